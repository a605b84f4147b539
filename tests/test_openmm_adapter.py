"""The OpenMM adapter (gluedmd_b200/openmm/B200GluedKernels.cpp) compiled against
minimal stand-ins of the OpenMM and GLUED declarations it uses
(tests/openmm_stub/include) and driven through a fake OpenMM runtime
(tests/openmm_stub/fake_openmm.cpp) the way OpenMM drives a kernel plugin:
registerKernelFactories() (CudaGluedKernelFactory.cpp:77-86), the factory's
createKernelImpl (:88-98), then initialize / updateState / execute /
getBiasStateBytes / getOPESMetrics of the CalcGluedForceKernel interface
(GluedKernels.h:23-105) as GluedForceImpl calls them (GluedForceImpl.cpp:36-165),
with OpenMM's device buffers read in place and an atom reorder announced
through a ReorderListener.

CPU: the adapter builds; its factory lands on the CUDA platform only; the
descriptor it builds from a GluedForce equals the force (same XML as the
library's own descriptor of the same calls); double precision is refused.
GPU: 40 steps of a context with distance/angle/dihedral/coordination CVs,
MetaD, OPES and a harmonic restraint against the FP64 oracle (fed the product's
CV values, as in test_gpu_paths.py): energies 1e-9 relative, forces 1e-4
relative (max-norm), MetaD grid 1e-12 and deposit count exact, OPES kernel
count exact and tables 1e-12, OPES metrics 1e-10; forces bit-identical after an
announced reorder."""
import ctypes
import math
import os
import sys

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "openmm_stub"))

_D, _I = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)


def _lib():
    import build as adapter_build
    from gluedmd_b200 import _native
    _native.lib()   # the product library first (the harness links against it)
    L = ctypes.CDLL(adapter_build.build())
    L.stub_error.restype = ctypes.c_char_p
    L.stub_new.restype = ctypes.c_void_p
    for name in ("stub_delete", "stub_add_particle", "stub_add_cv", "stub_add_bias", "stub_set_config",
                 "stub_describe_xml", "stub_create", "stub_set_box", "stub_execute", "stub_update_state",
                 "stub_notify_reordered", "stub_cv_values", "stub_bias_state", "stub_opes_metrics",
                 "stub_kernel_sigmas", "stub_last_bias"):
        getattr(L, name).argtypes = None
    L.stub_create.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_ulonglong,
                              ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int]
    L.stub_add_particle.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.stub_set_config.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _D, ctypes.c_int]
    return L


class Harness:
    def __init__(self, L, masses, cvs, biases, pbc=True, temperature=300.0, grad=None):
        self.L = L
        self.h = ctypes.c_void_p(L.stub_new())
        for m in masses:
            L.stub_add_particle(self.h, float(m))
        for t, a, p in cvs:
            a = np.ascontiguousarray(a, np.int32)
            p = np.ascontiguousarray(p, np.float64)
            L.stub_add_cv(self.h, int(t), a.ctypes.data_as(_I), len(a), p.ctypes.data_as(_D), len(p))
        for t, c, p, ip in biases:
            c = np.ascontiguousarray(c, np.int32)
            p = np.ascontiguousarray(p, np.float64)
            ip = np.ascontiguousarray(ip, np.int32)
            L.stub_add_bias(self.h, int(t), c.ctypes.data_as(_I), len(c), p.ctypes.data_as(_D), len(p),
                            ip.ctypes.data_as(_I), len(ip))
        g = np.ascontiguousarray([] if grad is None else grad, np.float64)
        L.stub_set_config(self.h, temperature, 1 if pbc else 0, g.ctypes.data_as(_D), len(g))

    def ok(self, rc):
        assert rc == 0, self.L.stub_error().decode()

    def xml(self):
        n = ctypes.c_size_t(0)
        self.L.stub_describe_xml(self.h, None, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        self.ok(self.L.stub_describe_xml(self.h, buf, ctypes.byref(n)))
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "h", None):
            self.L.stub_delete(self.h)
            self.h = None


def _system(seed=3):
    """Distance, angle, dihedral, coordination CVs on 300 atoms in a 2.5 nm box;
    MetaD on the two dihedrals' grid, OPES on (distance, angle), a harmonic
    restraint on the coordination number."""
    rng = np.random.default_rng(seed)
    n, L = 300, 2.5
    pos = rng.uniform(0, L, (n, 3))
    A = rng.choice(n, 40, replace=False)
    B = rng.choice(n, 90, replace=False)
    cvs = [(O.CV_DISTANCE, [3, 17], []), (O.CV_ANGLE, [5, 8, 40], []), (O.CV_DIHEDRAL, [1, 2, 3, 4], []),
           (O.CV_DIHEDRAL, [2, 3, 4, 5], []),
           (O.CV_COORDINATION, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.35, 6, 12])]
    biases = [(O.BIAS_METAD, [2, 3], [1.2, 0.35, 0.35, 10.0, 2.494338785, -math.pi, -math.pi, math.pi, math.pi],
               [3, 48, 48, 1, 1]),
              (O.BIAS_OPES, [0, 1], [2.494338785, 20.05, 0.1, 0.1, 0.01], [0, 2, 100000]),
              (O.BIAS_HARMONIC, [4], [5.0, 2.0], [0])]
    masses = rng.uniform(1, 16, n)
    return pos, masses, cvs, biases, L


def test_adapter_builds_and_registers_on_the_cuda_platform_only():
    L = _lib()
    assert L.stub_init_platforms() == 2


def test_adapter_descriptor_equals_the_force():
    from gluedmd_b200 import GluedForce
    L = _lib()
    pos, masses, cvs, biases, box = _system()
    h = Harness(L, masses, cvs, biases, pbc=True, temperature=310.0)
    f = GluedForce()
    f.setTemperature(310.0)
    f.setUsesPeriodicBoundaryConditions(True)
    for t, a, p in cvs:
        f.addCollectiveVariable(t, [int(x) for x in a], [float(x) for x in p])
    for t, c, p, ip in biases:
        f.addBias(t, c, p, ip)
    assert h.xml() == f.toXml()


def test_adapter_refuses_double_precision_contexts():
    L = _lib()
    L.stub_init_platforms()
    pos, masses, cvs, biases, box = _system()
    h = Harness(L, masses, cvs, biases)
    assert L.stub_create(h.h, 0, 0, 0, 320, 0, 1) == -1
    assert "double-precision" in L.stub_error().decode()


@pytest.mark.gpu
def test_adapter_drives_the_library_like_openmm():
    import torch
    L = _lib()
    assert L.stub_init_platforms() & 2
    pos0, masses, cvs, biases, box = _system()
    n = len(pos0)
    padded = 320
    rng = np.random.default_rng(9)
    perm = rng.permutation(n)                  # GPU slot s holds user atom perm[s]
    posq = torch.zeros((padded, 4), dtype=torch.float32, device="cuda")
    index = torch.zeros(padded, dtype=torch.int32, device="cuda")
    force = torch.zeros(3 * padded, dtype=torch.int64, device="cuda")
    index[:n] = torch.as_tensor(perm, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    h = Harness(L, masses, cvs, biases)
    h.ok(L.stub_create(h.h, posq.data_ptr(), index.data_ptr(), force.data_ptr(), padded, stream, 0))
    b9 = (ctypes.c_double * 9)(*np.diag([box] * 3).ravel())
    h.ok(L.stub_set_box(h.h, b9))
    orc = O.OracleSystem(cvs, biases, masses=masses, periodic=True, mode="f64", num_particles=n)

    def load(p, order):
        posq.zero_()
        posq[:n, :3] = torch.as_tensor(p[order], dtype=torch.float32, device="cuda")

    def forces(order):
        f = force.view(3, padded)[:, :n].cpu().numpy().astype(np.float64) / 4294967296.0
        out = np.zeros((n, 3))
        out[order] = f.T
        return out

    ncv = 5
    cvv = (ctypes.c_double * ncv)()
    walkers = [3, 17, 5, 8, 40]               # atoms of the OPES CVs (distance, angle) move further
    for step in range(40):
        p = pos0 + rng.normal(0, 0.03, pos0.shape)
        p[walkers] += rng.uniform(-0.3, 0.3, (len(walkers), 3))
        load(p, perm)
        force.zero_()
        h.ok(L.stub_update_state(h.h, step))
        orc.update_state(step)
        e = ctypes.c_double()
        h.ok(L.stub_execute(h.h, 1, 1, ctypes.byref(e)))
        h.ok(L.stub_cv_values(h.h, cvv, ncv))
        cv = np.array(cvv[:])
        ref = orc.execute(p, np.diag([box] * 3).ravel())
        np.testing.assert_allclose(cv, ref["cv_values"], rtol=1e-5, atol=1e-5)
        assert O.max_rel_force_err(forces(perm), ref["forces"]) < 1e-4
        # the next deposits start from the product's CV values and energies
        orc.cv_values = cv
        en = orc.evaluate_biases(cv)[0]
        assert abs(e.value - en.sum()) <= 1e-9 * max(1.0, abs(en.sum())), (step, e.value, en.sum())
        orc.bias_energies = en
    # OPES decisions and table, MetaD grid through the adapter's blob
    from gluedmd_b200.merger import BiasStateMerger
    from gluedmd_b200 import GluedForce
    f = GluedForce()
    for t, a, pp in cvs:
        f.addCollectiveVariable(t, [int(x) for x in a], [float(x) for x in pp])
    for t, c, pp, ip in biases:
        f.addBias(t, c, pp, ip)
    nb = ctypes.c_size_t(0)
    L.stub_bias_state(h.h, None, ctypes.byref(nb))
    buf = ctypes.create_string_buffer(nb.value)
    h.ok(L.stub_bias_state(h.h, buf, ctypes.byref(nb)))
    parsed = BiasStateMerger._parse(buf.raw[:nb.value], f)
    # the oracle's OPES deposits use its own per-bias energy at the product's CV
    # values (the adapter returns only the total), equal to the product's to
    # FP64 rounding: tables to 1e-12 (bit-exact decisions: test_gpu_paths.py)
    st = [s for s in orc.bias_state if s["type"] == O.BIAS_OPES][0]
    nk, su, ns, mean, m2, c, s_, lw = parsed["opes"][0]
    assert nk == int(st["ist"][0]) > 3
    np.testing.assert_allclose(np.frombuffer(c, "<f8"), st["centers"][:2 * nk], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(np.frombuffer(s_, "<f8"), st["sigmas"][:2 * nk], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(np.frombuffer(lw, "<f8"), st["logw"][:nk], rtol=1e-12, atol=1e-12)
    g = [s for s in orc.bias_state if s["type"] == O.BIAS_METAD][0]
    nd, grid = parsed["metad"][0]
    assert nd == g["deposited"] == 13
    np.testing.assert_allclose(np.frombuffer(grid, "<f8"), g["grid"], rtol=1e-12, atol=1e-12 * np.abs(g["grid"]).max())
    m = (ctypes.c_double * 4)()
    h.ok(L.stub_opes_metrics(h.h, 0, m))
    np.testing.assert_allclose(m[:], orc.opes_metrics(0), rtol=1e-10, atol=1e-12)
    # OpenMM reorders the atoms and tells its listeners: same forces, bitwise
    force.zero_()
    e1 = ctypes.c_double()
    h.ok(L.stub_execute(h.h, 1, 1, ctypes.byref(e1)))
    f1 = forces(perm)
    perm2 = rng.permutation(n)
    index[:n] = torch.as_tensor(perm2, dtype=torch.int32, device="cuda")
    load(p, perm2)
    h.ok(L.stub_notify_reordered(h.h))
    force.zero_()
    e2 = ctypes.c_double()
    h.ok(L.stub_execute(h.h, 1, 1, ctypes.byref(e2)))
    assert e1.value == e2.value
    assert np.array_equal(forces(perm2), f1)
