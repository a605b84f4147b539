"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline leg). The product package never imports this module.

Host-side restatement of GLUED's per-step orchestration over the C restatement in
``glued_oracle.cpp``:

* plan flattening and Jacobian-row layout in the reference's type order
  (platforms/common/src/CommonGluedKernels.cpp:3935-4230),
* ``execute()``: CV kernels in type order, bias evaluation in bias-type order with
  ``+=`` into the per-CV bias gradients, then the chain-rule scatter into the
  2^32 fixed-point force buffer (CommonGluedKernels.cpp:4736-5048),
* ``updateState(step)``: pace-gated OPES and MetaD deposition from the previous
  ``execute()``'s CV values and bias energies, skipped before the first execute
  and at step 0 (CommonGluedKernels.cpp:5050-5157).

``mode='f64'`` is the FP64 oracle; ``mode='f32'`` restates the reference's FP32
("real" = float) semantics.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libglued_oracle.so")

# CV / bias type codes (openmmapi/include/GluedForce.h:27-95).
CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION = 1, 2, 3, 4, 5
CV_COORDINATION, CV_RMSD, CV_PATH, CV_CONTACTMAP, CV_PCA = 6, 7, 10, 13, 21
BIAS_HARMONIC, BIAS_METAD, BIAS_PBMETAD, BIAS_OPES, BIAS_EXTERNAL = 1, 3, 4, 5, 6
# Extensions of this build (no reference counterpart).
CV_RMSD_KABSCH = 107
CV_COORDINATION_CUTOFF = 106
BIAS_METAD_HILLS = 103

KT_PER_K = 8.314462618e-3


def build(force: bool = False) -> str:
    """Compile the oracle shared library with gcc (no GPU needed)."""
    src = os.path.join(HERE, "glued_oracle.cpp")
    hdr = os.path.join(HERE, "..", "gluedmd_b200", "csrc", "glued_dmath.h")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    tmp = LIB_PATH + f".tmp{os.getpid()}"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                           src, "-o", tmp])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


_D, _I, _F, _L = ctypes.c_double, ctypes.c_int, ctypes.c_float, ctypes.c_longlong


def masses_or_ones(masses, n):
    return np.ones(n) if masses is None else np.asarray(masses, dtype=np.float64)


@dataclass
class _Kind:
    cv0: int = -1
    n: int = 0
    atoms: list = field(default_factory=list)
    extra: dict = field(default_factory=dict)


class OracleSystem:
    """A GluedForce-equivalent evaluated on the CPU.

    cvs    : list of (type, atoms, params) as passed to addCollectiveVariable.
    biases : list of (type, cvIndices, params, intParams) as passed to addBias.
    """

    def __init__(self, cvs, biases=(), masses=None, periodic=False, mode="f64",
                 test_bias_gradients=None, num_particles=None):
        self.mode = mode
        self.cvs = [(int(t), list(map(int, a)), list(map(float, p))) for t, a, p in cvs]
        self.biases = [(int(t), list(map(int, c)), list(map(float, p)), list(map(int, ip)))
                       for t, c, p, ip in biases]
        self.periodic = bool(periodic)
        self.test_grad = None if test_bias_gradients is None else np.asarray(test_bias_gradients, float)
        n_atoms = num_particles if num_particles is not None else 1 + max(
            [max(a) for t, a, p in self.cvs if a and t != CV_COORDINATION] +
            [max(a[1:]) for t, a, p in self.cvs if t == CV_COORDINATION] + [0])
        self.num_particles = n_atoms
        self.masses = masses_or_ones(masses, n_atoms)
        self._build_plan()
        self._setup_biases()
        self.cv_ready = False
        self.decisions_only = False  # skip the sum_uprob update in deposit replays
        self.last_update_step = -1
        self.cv_values = np.zeros(self.num_cvs)
        self.bias_energies = np.zeros(max(1, len(self.biases)))

    # ------------------------------------------------------------------ plan
    def _build_plan(self):
        order = [CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION, CV_COORDINATION,
                 CV_COORDINATION_CUTOFF, CV_RMSD, CV_RMSD_KABSCH, CV_PATH, CV_CONTACTMAP, CV_PCA]
        kinds = {t: _Kind() for t in order}
        v = 0
        for t, a, p in self.cvs:
            if t not in kinds:
                raise ValueError(f"oracle: CV type {t} not restated")
            k = kinds[t]
            if k.n == 0:
                k.cv0 = v
            k.n += 1
            k.atoms.append((a, p))
            v += 2 if t == CV_PATH else 1
        self.num_cvs = v
        self.kinds = kinds
        # Jacobian row offsets in the reference's order (CommonGluedKernels.cpp:4186-4230):
        # distance 2/CV, angle 3/CV, dihedral 4/CV, COM and gyration one per atom,
        # coordination one per group atom, RMSD one per atom, path two per atom,
        # contact map two per pair, PCA one per atom. Extension kinds follow their
        # reference sibling.
        def natoms(t):
            tot = 0
            for a, p in kinds[t].atoms:
                if t in (CV_COORDINATION, CV_COORDINATION_CUTOFF):
                    tot += len(a) - 1
                elif t == CV_PATH:
                    tot += 2 * len(a)
                elif t == CV_CONTACTMAP:
                    tot += 2 * (len(a) // 2)
                else:
                    tot += len(a)
            return tot
        sizes = [
            (CV_DISTANCE, 2 * kinds[CV_DISTANCE].n), (CV_ANGLE, 3 * kinds[CV_ANGLE].n),
            (CV_DIHEDRAL, 4 * kinds[CV_DIHEDRAL].n), (CV_COM_DISTANCE, natoms(CV_COM_DISTANCE)),
            (CV_GYRATION, natoms(CV_GYRATION)), (CV_COORDINATION, natoms(CV_COORDINATION)),
            (CV_COORDINATION_CUTOFF, natoms(CV_COORDINATION_CUTOFF)),
            (CV_RMSD, natoms(CV_RMSD)), (CV_RMSD_KABSCH, natoms(CV_RMSD_KABSCH)),
            (CV_PATH, natoms(CV_PATH)), (CV_CONTACTMAP, natoms(CV_CONTACTMAP)),
            (CV_PCA, natoms(CV_PCA)),
        ]
        off = 0
        self.jac0 = {}
        for t, s in sizes:
            self.jac0[t] = off
            off += s
        self.num_jac = off

    def _setup_biases(self):
        self.bias_state = []
        for slot, (t, cvi, p, ip) in enumerate(self.biases):
            D = len(cvi)
            st = {"type": t, "slot": slot, "idx": np.array(cvi, dtype=np.int32), "D": D}
            if t == BIAS_HARMONIC:
                prm = np.array(p[:2 * D], dtype=np.float32)
                st.update(prm=prm, periodic=(ip[0] if ip else 0))
            elif t == BIAS_METAD:
                # CommonBiasKernels.cpp:206-257
                h0 = p[0]; sigma = p[1:1 + D]; gamma = p[1 + D]; kT = p[2 + D]
                origin = p[3 + D:3 + 2 * D]; mx = p[3 + 2 * D:3 + 3 * D]
                pace = ip[0]; bins = ip[1:1 + D]; per = ip[1 + D:1 + 2 * D]
                inv = [bins[d] / (mx[d] - origin[d]) for d in range(D)]
                npts = [bins[d] + (0 if per[d] else 1) for d in range(D)]
                strides = [1] * D
                for d in range(1, D):
                    strides[d] = strides[d - 1] * npts[d - 1]
                total = strides[-1] * npts[-1]
                st.update(h0=h0, sigma=np.array(sigma), gamma=gamma, kT=kT,
                          origin=np.array(origin), inv=np.array(inv),
                          npts=np.array(npts, np.int32), strides=np.array(strides, np.int32),
                          per=np.array(per, np.int32), pace=pace, total=total,
                          grid=np.zeros(total), hif=(0.0 if gamma <= 1.0 else 1.0 / ((gamma - 1.0) * kT)),
                          deposited=0)
            elif t == BIAS_PBMETAD:
                # CommonBiasKernels.cpp:298-424: N 1-D sub-grids, one energy slot
                h0, gamma, kT = p[0], p[1], p[2]
                sigma = [p[3 + 3 * d] for d in range(D)]
                origin = [p[4 + 3 * d] for d in range(D)]
                mx = [p[5 + 3 * d] for d in range(D)]
                bins = [ip[1 + 2 * d] for d in range(D)]
                per = [ip[2 + 2 * d] for d in range(D)]
                npts = [bins[d] + (0 if per[d] else 1) for d in range(D)]
                goff = np.concatenate([[0], np.cumsum(npts)[:-1]]).astype(np.int32)
                st.update(h0=h0, gamma=gamma, kT=kT, sigma=np.array(sigma), origin=np.array(origin),
                          inv=np.array([bins[d] / (mx[d] - origin[d]) for d in range(D)]),
                          npts=np.array(npts, np.int32), per=np.array(per, np.int32), goff=goff,
                          grid=np.zeros(int(sum(npts))), pace=ip[0],
                          hif=(0.0 if gamma <= 1.0 else 1.0 / ((gamma - 1.0) * kT)),
                          V=np.zeros(D), W=np.full(D, 1.0 / D), deposited=[0] * D)
            elif t == BIAS_EXTERNAL:
                # CommonBiasKernels.cpp:425-488: fixed user grid, evaluated as the MetaD grid
                origin = p[:D]; mx = p[D:2 * D]
                bins = ip[:D]; per = ip[D:2 * D]
                inv = [bins[d] / (mx[d] - origin[d]) for d in range(D)]
                npts = [bins[d] + (0 if per[d] else 1) for d in range(D)]
                strides = [1] * D
                for d in range(1, D):
                    strides[d] = strides[d - 1] * npts[d - 1]
                total = strides[-1] * npts[-1]
                st.update(origin=np.array(origin), inv=np.array(inv), npts=np.array(npts, np.int32),
                          strides=np.array(strides, np.int32), per=np.array(per, np.int32), total=total,
                          grid=np.array(p[2 * D:2 * D + total], dtype=np.float64))
            elif t == BIAS_METAD_HILLS:
                h0 = p[0]; sigma = p[1:1 + D]; gamma = p[1 + D]; kT = p[2 + D]
                lo = p[3 + D:3 + 2 * D]; hi = p[3 + 2 * D:3 + 3 * D]
                pace = ip[0]; maxh = ip[1]; per = ip[2:2 + D]
                period = np.array([(hi[d] - lo[d]) if per[d] else 0.0 for d in range(D)])
                st.update(h0=h0, sigma=np.array(sigma), gamma=gamma, kT=kT, pace=pace, maxh=maxh,
                          period=period, centers=np.zeros((0, D)), heights=np.zeros(0),
                          hif=(0.0 if gamma <= 1.0 else 1.0 / ((gamma - 1.0) * kT)))
            elif t == BIAS_OPES:
                # CommonBiasKernels.cpp:489-588
                kT, gamma = p[0], p[1]
                sigma0 = list(p[2:2 + D]); smin = p[2 + D]
                variant = ip[0] if len(ip) > 0 else 0
                pace = ip[1] if len(ip) > 1 else 500
                maxk = ip[2] if len(ip) > 2 else 100000
                adaptive = sigma0[0] <= 0.0
                astride = (ip[3] if len(ip) > 3 else 10 * pace) if adaptive else 0
                if variant == 1:
                    invGF, cut2, eps, barrier = 1.0, 2.0 * gamma, 0.0, gamma * kT
                elif variant == 2:
                    invGF, cut2 = gamma - 1.0, 2.0 * gamma
                    eps, barrier = math.exp(-gamma / (gamma - 1.0)), gamma * kT
                    if not adaptive:
                        sigma0 = [s * math.sqrt(gamma) for s in sigma0]
                else:
                    invGF = (gamma - 1.0) / gamma
                    cut2 = 2.0 * gamma / invGF
                    eps = math.exp(-1.0 / (invGF * (1.0 - invGF)))
                    barrier = kT / (1.0 - invGF)
                st.update(kT=kT, gamma=gamma, sigma0=np.array(sigma0), smin=smin, variant=variant,
                          pace=pace, maxk=maxk, astride=astride, invGF=invGF, cut2=cut2, eps=eps,
                          barrier=barrier,
                          centers=np.zeros(maxk * D), sigmas=np.ones(maxk * D), logw=np.zeros(maxk),
                          dst=np.array([0.0, math.exp(-gamma), math.exp(-gamma), math.exp(-2.0 * gamma)]),
                          ist=np.zeros(4, np.int32), mean=np.zeros(D), m2=np.zeros(D), nsamp_cpu=0,
                          nker_cpu=0, decisions=[])
            else:
                raise ValueError(f"oracle: bias type {t} not restated")
            self.bias_state.append(st)

    # --------------------------------------------------------------- execute
    def _jac_arrays(self):
        n = max(1, self.num_jac)
        return (np.zeros(n, np.int32), np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n, np.int32))

    def evaluate_cvs(self, pos, box=None):
        """Returns (cv_values, (atom, gx, gy, gz, cv)) for positions pos[N,3] (nm)."""
        L = lib()
        sfx = "_" + self.mode
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        box9 = np.ascontiguousarray(np.eye(3).ravel() * 1e6 if box is None else np.asarray(box, float).ravel())
        per = 1 if self.periodic else 0
        cvv = np.zeros(max(1, self.num_cvs))
        ja, jx, jy, jz, jc = self._jac_arrays()
        J = (_p(ja, _I), _p(jx, _D), _p(jy, _D), _p(jz, _D), _p(jc, _I))
        P = _p(pos, _D)
        B = _p(box9, _D)
        C = _p(cvv, _D)
        k = self.kinds
        for t, fn, per_atoms in ((CV_DISTANCE, "orc_cv_distance", 2), (CV_ANGLE, "orc_cv_angle", 3),
                                 (CV_DIHEDRAL, "orc_cv_dihedral", 4)):
            if k[t].n:
                a = np.array([x for at, p in k[t].atoms for x in at[:per_atoms]], np.int32)
                getattr(L, fn + sfx)(P, _p(a, _I), k[t].n, k[t].cv0, self.jac0[t], B, per, C, *J)
        for t, fn in ((CV_COM_DISTANCE, "orc_cv_com_distance"), (CV_GYRATION, "orc_cv_gyration")):
            if not k[t].n:
                continue
            off, atoms, m, tm = [0], [], [], []
            for at, p in k[t].atoms:
                if t == CV_COM_DISTANCE:
                    ng1 = int(round(p[0])) if p else 1
                    g1, g2 = at[:ng1], at[ng1:]
                    off += [off[-1] + len(g1), off[-1] + len(g1) + len(g2)]
                    tm += [float(np.float32(sum(np.float32(self.masses[a]) for a in g1))),
                           float(np.float32(sum(np.float32(self.masses[a]) for a in g2)))]
                else:
                    off.append(off[-1] + len(at))
                    tm.append(float(np.float32(sum(np.float32(self.masses[a]) for a in at))))
                atoms += at
                m += [self.masses[a] for a in at]
            getattr(L, fn + sfx)(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                                 _p(np.array(m, np.float32), _F), _p(np.array(tm, np.float32), _F),
                                 k[t].n, k[t].cv0, self.jac0[t], B, per, C, *J)
        for t in (CV_COORDINATION, CV_COORDINATION_CUTOFF):
            if not k[t].n:
                continue
            # Each CV is its own call so that the cutoff can differ per CV.
            cum = 0
            for i, (at, p) in enumerate(k[t].atoms):
                na = at[0]
                grp = at[1:]
                off = np.array([cum, cum + na, cum + len(grp)], np.int32)
                atoms = np.zeros(cum + len(grp), np.int32)
                atoms[cum:] = grp
                prm = np.array(p[:3], np.float32)
                rc = p[3] if (t == CV_COORDINATION_CUTOFF and len(p) > 3) else 0.0
                getattr(L, "orc_cv_coordination" + sfx)(P, _p(off, _I), _p(atoms, _I), _p(prm, _F), 1,
                                                        k[t].cv0 + i, self.jac0[t], B, per, _D(rc), C, *J)
                cum += len(grp)
        if k[CV_RMSD].n:
            off, atoms, ref = [0], [], []
            for at, p in k[CV_RMSD].atoms:
                off.append(off[-1] + len(at)); atoms += at; ref += p[:3 * len(at)]
            L.__getattr__("orc_cv_rmsd" + sfx)(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                                               _p(np.array(ref, np.float32), _F), k[CV_RMSD].n, k[CV_RMSD].cv0,
                                               self.jac0[CV_RMSD], C, *J)
        if k[CV_RMSD_KABSCH].n:
            row = self.jac0[CV_RMSD_KABSCH]
            for i, (at, p) in enumerate(k[CV_RMSD_KABSCH].atoms):
                a = np.array(at, np.int32)
                ref = np.array(p[:3 * len(at)], np.float32)
                val = np.zeros(1); g = np.zeros(3 * len(at))
                L.orc_cv_rmsd_kabsch(P, _p(a, _I), _p(ref, _F), len(at), _p(val, _D), _p(g, _D))
                cvv[k[CV_RMSD_KABSCH].cv0 + i] = val[0]
                for j, at_j in enumerate(at):
                    ja[row] = at_j; jx[row], jy[row], jz[row] = g[3 * j:3 * j + 3]
                    jc[row] = k[CV_RMSD_KABSCH].cv0 + i
                    row += 1
        if k[CV_PATH].n:
            off, atoms, roff, ref, prm = [0], [], [], [], []
            rb = 0
            for at, p in k[CV_PATH].atoms:
                N = int(p[1]); M = len(at)
                off.append(off[-1] + M); atoms += at; roff.append(rb); rb += N * M
                prm += [p[0], p[1]]; ref += p[2:2 + 3 * N * M]
            L.__getattr__("orc_cv_path" + sfx)(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                                               _p(np.array(roff, np.int32), _I), _p(np.array(ref, np.float32), _F),
                                               _p(np.array(prm, np.float32), _F), k[CV_PATH].n, k[CV_PATH].cv0,
                                               self.jac0[CV_PATH], C, *J)
        if k[CV_CONTACTMAP].n:
            off, pairs, prm = [0], [], []
            for at, p in k[CV_CONTACTMAP].atoms:
                npair = len(at) // 2
                off.append(off[-1] + npair); pairs += at[:2 * npair]; prm += p[:4 * npair]
            L.__getattr__("orc_cv_contact_map" + sfx)(P, _p(np.array(off, np.int32), _I),
                                                      _p(np.array(pairs, np.int32), _I),
                                                      _p(np.array(prm, np.float32), _F), k[CV_CONTACTMAP].n,
                                                      k[CV_CONTACTMAP].cv0, self.jac0[CV_CONTACTMAP], B, per, C, *J)
        if k[CV_PCA].n:
            off, atoms, ref, ev = [0], [], [], []
            for at, p in k[CV_PCA].atoms:
                N = len(at)
                off.append(off[-1] + N); atoms += at; ref += p[:3 * N]; ev += p[3 * N:6 * N]
            L.__getattr__("orc_cv_pca" + sfx)(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                                              _p(np.array(ref, np.float32), _F), _p(np.array(ev, np.float32), _F),
                                              k[CV_PCA].n, k[CV_PCA].cv0, self.jac0[CV_PCA], C, *J)
        return cvv[:self.num_cvs].copy(), (ja, jx, jy, jz, jc)

    def evaluate_biases(self, cvv):
        """Bias evaluation in the reference's type order (CommonGluedKernels.cpp:4955-5026).
        Returns (energies per slot, dU/dCV)."""
        L = lib()
        grad = np.zeros(max(1, self.num_cvs))
        energies = np.zeros(max(1, len(self.biases)))
        C = _p(np.ascontiguousarray(cvv, dtype=np.float64), _D)
        cvv = np.ascontiguousarray(cvv, dtype=np.float64)
        G = _p(grad, _D)
        for typ in (BIAS_HARMONIC, BIAS_OPES, BIAS_METAD, BIAS_PBMETAD, BIAS_EXTERNAL, BIAS_METAD_HILLS):
            for st in self.bias_state:
                if st["type"] != typ:
                    continue
                idx = st["idx"]
                if typ == BIAS_HARMONIC:
                    L.orc_harmonic.restype = _D
                    e = L.orc_harmonic(C, _p(idx, _I), _p(st["prm"], _F), st["D"], st["periodic"], G)
                elif typ == BIAS_OPES:
                    L.orc_opes_eval.restype = _D
                    e = L.orc_opes_eval(C, _p(idx, _I), st["D"], _p(st["centers"], _D), _p(st["sigmas"], _D),
                                        _p(st["logw"], _D), int(st["ist"][0]), _D(st["invGF"]), _D(st["kT"]),
                                        _D(st["dst"][0]), _D(st["cut2"]), _D(st["eps"]), _D(st["barrier"]), G)
                elif typ == BIAS_PBMETAD:
                    L.orc_pbmetad_eval.restype = _D
                    e = L.orc_pbmetad_eval(C, _p(idx, _I), st["D"], _p(st["grid"], _D), _p(st["goff"], _I),
                                           _p(st["origin"], _D), _p(st["inv"], _D), _p(st["npts"], _I),
                                           _p(st["per"], _I), _D(st["kT"]), G, _p(st["V"], _D), _p(st["W"], _D))
                elif typ in (BIAS_METAD, BIAS_EXTERNAL):
                    L.orc_metad_eval.restype = _D
                    e = L.orc_metad_eval(C, _p(idx, _I), st["D"], _p(st["grid"], _D), _p(st["origin"], _D),
                                         _p(st["inv"], _D), _p(st["npts"], _I), _p(st["strides"], _I),
                                         _p(st["per"], _I), G)
                else:
                    L.orc_hills_eval.restype = _D
                    s = np.array([cvv[i] for i in idx])
                    dv = np.zeros(st["D"])
                    K = len(st["heights"])
                    cen = np.ascontiguousarray(st["centers"].ravel())
                    hts = np.ascontiguousarray(st["heights"])
                    e = L.orc_hills_eval(_p(s, _D), st["D"], _p(cen, _D), _p(hts, _D), K,
                                         _p(st["sigma"], _D), _p(st["period"], _D), _p(dv, _D))
                    for d, i in enumerate(idx):
                        grad[i] += dv[d]
                energies[st["slot"]] = e
        return energies, grad[:self.num_cvs]

    def execute(self, pos, box=None):
        """One force evaluation. Returns dict(energy, forces (N,3) double from the
        fixed-point buffer, force_fixed int64[3,N], cv_values, dUdCV, jacobian)."""
        cvv, jac = self.evaluate_cvs(pos, box)
        if self.test_grad is not None:
            grad = np.array(self.test_grad, float)
            energies = np.zeros(max(1, len(self.biases)))
        else:
            energies, grad = self.evaluate_biases(cvv)
        n = self.num_particles
        fbuf = np.zeros(3 * n, np.int64)
        ja, jx, jy, jz, jc = jac
        g = np.ascontiguousarray(np.resize(grad, max(1, self.num_cvs)), dtype=np.float64)
        lib().orc_scatter(_p(g, _D), _p(ja, _I), _p(jx, _D), _p(jy, _D), _p(jz, _D), _p(jc, _I),
                          self.num_jac, _p(fbuf, _L), n)
        self.cv_values = cvv
        self.bias_energies = energies
        self.cv_ready = True
        forces = fbuf.reshape(3, n).T.astype(np.float64) / 4294967296.0
        return dict(energy=float(energies.sum()), forces=forces, force_fixed=fbuf.reshape(3, n),
                    cv_values=cvv, dUdCV=grad, jacobian=jac, bias_energies=energies)

    # ----------------------------------------------------------- updateState
    def update_state(self, step):
        """Deposition at pace (CommonGluedKernels.cpp:5050-5157)."""
        L = lib()
        if not self.cv_ready or step == self.last_update_step:
            return
        if not any(st["type"] in (BIAS_OPES, BIAS_METAD, BIAS_PBMETAD, BIAS_METAD_HILLS) for st in self.bias_state):
            return
        self.last_update_step = step
        cvv = np.ascontiguousarray(self.cv_values, dtype=np.float64)
        C = _p(cvv, _D)
        for st in self.bias_state:
            if st["type"] != BIAS_OPES:
                continue
            if step == 0 or step % st["pace"] != 0:
                continue
            if st["nker_cpu"] >= st["maxk"]:
                continue
            will = st["astride"] == 0 or st["nsamp_cpu"] >= st["astride"]
            r = L.orc_opes_deposit_ex(C, _p(st["idx"], _I), st["D"], _p(st["mean"], _D), _p(st["m2"], _D),
                                      _p(st["sigma0"], _D), _D(st["smin"]), _p(st["centers"], _D),
                                      _p(st["sigmas"], _D), _p(st["logw"], _D), _p(st["dst"], _D),
                                      _p(st["ist"], _I), st["variant"], st["astride"],
                                      _D(self.bias_energies[st["slot"]]), _D(1.0 / st["kT"]), _D(st["cut2"]),
                                      st["maxk"], _D(st["gamma"]), 1 if self.decisions_only else 0)
            st["decisions"].append(int(r))
            if will:
                st["nker_cpu"] += 1
        for st in self.bias_state:
            if st["type"] == BIAS_METAD:
                if step == 0 or step % st["pace"] != 0:
                    continue
                center = np.array([cvv[i] for i in st["idx"]])
                L.orc_metad_deposit(_p(st["grid"], _D), st["D"], st["total"], _p(st["origin"], _D),
                                    _p(st["inv"], _D), _p(st["npts"], _I), _p(st["strides"], _I),
                                    _p(st["per"], _I), _p(center, _D), _p(st["sigma"], _D),
                                    _D(self.bias_energies[st["slot"]]), _D(st["h0"]), _D(st["hif"]))
                st["deposited"] += 1
            elif st["type"] == BIAS_METAD_HILLS:
                if step == 0 or step % st["pace"] != 0:
                    continue
                if len(st["heights"]) >= st["maxh"]:
                    continue
                V = self.bias_energies[st["slot"]]
                h = st["h0"] * math.exp(-V * st["hif"]) if st["hif"] > 0 else st["h0"]
                center = np.array([cvv[i] for i in st["idx"]])
                st["centers"] = np.vstack([st["centers"], center[None, :]])
                st["heights"] = np.append(st["heights"], h)
        for st in self.bias_state:
            if st["type"] != BIAS_PBMETAD or step == 0 or step % st["pace"] != 0:
                continue
            L.orc_pbmetad_deposit(_p(st["grid"], _D), _p(st["goff"], _I), st["D"], _p(st["origin"], _D),
                                  _p(st["inv"], _D), _p(st["npts"], _I), _p(st["per"], _I), C,
                                  _p(st["idx"], _I), _p(st["sigma"], _D), _p(st["V"], _D), _p(st["W"], _D),
                                  _D(st["h0"]), _D(st["hif"]))
            st["deposited"] = [n + 1 for n in st["deposited"]]

    def load_blob(self, blob: bytes):
        """Restore OPES / MetaD / hill-sum state from a 'GPUS' v1 bias-state blob
        (CommonSerialization.cpp:180-290 reader; hill section of this library)."""
        import struct
        p = 0
        if blob[:4] == b"GPUS":
            p = 8
        nb, = struct.unpack_from("<i", blob, p); p += 4
        opes = [st for st in self.bias_state if st["type"] == BIAS_OPES]
        assert nb == len(opes)
        for st in opes:
            D = st["D"]
            nk, su, ns = struct.unpack_from("<idi", blob, p); p += 16
            arr = np.frombuffer(blob, "<f8", count=2 * D + 2 * nk * D + nk, offset=p).copy()
            p += 8 * len(arr)
            st["mean"][:] = arr[:D]; st["m2"][:] = arr[D:2 * D]
            st["centers"][:nk * D] = arr[2 * D:2 * D + nk * D]
            st["sigmas"][:nk * D] = arr[2 * D + nk * D:2 * D + 2 * nk * D]
            st["logw"][:nk] = arr[2 * D + 2 * nk * D:]
            st["ist"][0] = nk; st["ist"][1] = ns; st["ist"][3] = nk
            st["dst"][0] = su
            st["dst"][1] = math.exp(-st["gamma"]) + float(np.exp(st["logw"][:nk]).sum())
            st["nker_cpu"] = nk; st["nsamp_cpu"] = ns
        if p < len(blob):
            p += 4  # ABMD count (0)
        if p < len(blob):
            nm, = struct.unpack_from("<i", blob, p); p += 4
            for st in [s_ for s_ in self.bias_state if s_["type"] == BIAS_METAD]:
                nd, = struct.unpack_from("<i", blob, p); p += 4
                st["grid"][:] = np.frombuffer(blob, "<f8", count=st["total"], offset=p)
                p += 8 * st["total"]
                st["deposited"] = nd
        if p < len(blob) and blob[p:p + 4] != b"HILL":
            npb, = struct.unpack_from("<i", blob, p); p += 4
            pbs = [s_ for s_ in self.bias_state if s_["type"] == BIAS_PBMETAD]
            assert npb == len(pbs)
            for st in pbs:
                nsub, = struct.unpack_from("<i", blob, p); p += 4
                assert nsub == st["D"]
                for d in range(nsub):
                    nd, = struct.unpack_from("<i", blob, p); p += 4
                    n, o = int(st["npts"][d]), int(st["goff"][d])
                    st["grid"][o:o + n] = np.frombuffer(blob, "<f8", count=n, offset=p)
                    p += 8 * n
                    st["deposited"][d] = nd
        p += 32  # EXTERNAL, LINEAR, WALL, OPES_EXPANDED, EXTLAG, EDS, MAXENT, MULTITHERMAL counts
        if blob[p:p + 4] == b"HILL":
            p += 8
            for st in [s_ for s_ in self.bias_state if s_["type"] == BIAS_METAD_HILLS]:
                n, = struct.unpack_from("<i", blob, p); p += 4
                D = st["D"]
                st["centers"] = np.frombuffer(blob, "<f8", count=n * D, offset=p).reshape(n, D).copy()
                p += 8 * n * D
                st["heights"] = np.frombuffer(blob, "<f8", count=n, offset=p).copy()
                p += 8 * n

    def _opes_states(self):
        return [st for st in self.bias_state if st["type"] == BIAS_OPES]

    def opes_metrics(self, opes_index):
        """[zed, rct, nker, neff] of the opes_index-th OPES bias
        (CommonGluedKernels.cpp:5164-5210): zed = sum_uprob / (KDEnorm nker) with
        KDEnorm the deposit counter for variant 2 (EXPLORE) and sum_weights
        otherwise; rct = kT ln(sum_weights / counter); neff = (1 + sum_w)^2 /
        (1 + sum_w2). State layout: dst = [sum_uprob, sum_weights, sum_w, sum_w2],
        ist = [numKernels, nSamples, counter, numAllocated]."""
        st = self._opes_states()[opes_index]
        nker = int(st["ist"][0])
        sum_up = float(st["dst"][0]) if nker > 0 else 0.0
        counter = float(st["ist"][2])
        kde = counter if st["variant"] == 2 else float(st["dst"][1])
        zed = sum_up / (kde * nker) if (nker > 0 and kde > 0.0) else 1.0
        rct = st["kT"] * math.log(st["dst"][1] / counter) if (counter > 0.0 and st["dst"][1] > 0.0) else 0.0
        sw, sw2 = float(st["dst"][2]), float(st["dst"][3])
        return [zed, rct, float(nker), (1.0 + sw) * (1.0 + sw) / (1.0 + sw2)]

    def kernel_sigmas(self, opes_index):
        """Kernel bandwidths of the live kernels, narrowed to float
        (CommonGluedKernels.cpp:5212-5232)."""
        st = self._opes_states()[opes_index]
        nk = int(st["ist"][0])
        return np.asarray(st["sigmas"][:nk * st["D"]], dtype=np.float32)

    def welford(self):
        """Per-execute Welford update for fully adaptive OPES (CommonGluedKernels.cpp:4976-4981)."""
        L = lib()
        cvv = np.ascontiguousarray(self.cv_values, dtype=np.float64)
        for st in self.bias_state:
            if st["type"] == BIAS_OPES and st["astride"] > 0:
                ns = np.array([st["ist"][1]], np.int32)
                L.orc_opes_welford(_p(cvv, _D), _p(st["idx"], _I), st["D"], _p(st["mean"], _D),
                                   _p(st["m2"], _D), _p(ns, _I))
                st["ist"][1] = ns[0]
                st["nsamp_cpu"] += 1


def fixed_point_forces(fbuf, n):
    """int64 field-major 2^32 fixed-point buffer -> (n,3) kJ/mol/nm."""
    f = np.asarray(fbuf, dtype=np.int64).reshape(3, -1)[:, :n]
    return f.T.astype(np.float64) / 4294967296.0


def max_rel_force_err(f, fref):
    """||f - fref||_inf / ||fref||_inf over all atoms and components."""
    den = np.max(np.abs(fref))
    return float(np.max(np.abs(np.asarray(f) - fref)) / den) if den > 0 else float(np.max(np.abs(f)))


def coordination_pair_list(pos, A, B, box9, rc, periodic=True, block=128):
    """Pairs (a, b) (indices into the groups A and B) that a cutoff coordination
    counts: 1e-20 <= r^2 < rc^2 with r^2 formed in FP64 as cv_coordination forms
    it (glued_oracle.cpp, cv_coordination and Box::image: d = p_a - p_b, then
    s = floor(d_z / c_z + 1/2), d -= s c; the same along b and a; r^2 = x^2 + y^2
    + z^2 left to right, each operation rounded on its own; rc^2 = rc * rc).
    numpy evaluates every elementwise operation with one rounding and no
    contraction, which is the oracle's arithmetic. Sorted by (a, b)."""
    pos = np.asarray(pos, np.float64)
    bx = np.asarray(box9, np.float64).reshape(3, 3)
    inv = np.array([1.0 / bx[0, 0], 1.0 / bx[1, 1], 1.0 / bx[2, 2]])
    rc2 = float(rc) * float(rc)
    pb = pos[np.asarray(B)]
    out = []
    A = np.asarray(A)
    for s in range(0, len(A), block):
        pa = pos[A[s:s + block]]
        d = pa[:, None, :] - pb[None, :, :]
        if periodic:
            for axis, vec in ((2, bx[2]), (1, bx[1]), (0, bx[0])):
                sh = np.floor(d[..., axis] * inv[axis] + 0.5)
                for k in range(axis + 1):
                    d[..., k] = d[..., k] - sh * vec[k]
        r2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
        ia, ib = np.nonzero((r2 >= 1e-20) & (r2 < rc2))
        out.append(np.stack([ia + s, ib], 1))
    p = np.concatenate(out) if out else np.zeros((0, 2), np.int64)
    return p[np.lexsort((p[:, 1], p[:, 0]))].astype(np.int32)
