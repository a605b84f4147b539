"""The allocation-free coordination entry point against the regular context path.

glued_coordination_noalloc serves callers that cannot allocate device memory
while they evaluate forces: its tile partials live in a fixed array inside the
library. Its CN and dCN/dx must agree with what glued_context_execute produces
for the same coordination CV (the CV value read back, and the forces with an
injected dU/dCN = 1, i.e. F = -dCN/dx), on two calls in a row that reuse the
array. Tolerances: CN 1e-6 relative, gradients 1e-5 of the largest force (the
1e-4 force gate of the other tests, tightened because both sides run the same
tile code)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(seed=21, n=3000, L=4.0, nA=700, nB=2000):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, L, (n, 3))
    perm = rng.permutation(n)
    A, B = perm[:nA], perm[nA:nA + nB]
    return pos, A, B, L


def test_noalloc_coordination_matches_context_path():
    import torch
    import gpu_util
    from gluedmd_b200 import _native

    pos, A, B, L = _system()
    cvs = [(6, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.35, 6, 12])]
    ctx, f = gpu_util.make_context(pos, cvs, pbc=True, box=np.eye(3) * L, grad=[1.0])
    _, F = ctx.computeForces()
    cn_ref = f.getLastCVValues(ctx)[0]

    lib = _native.lib()
    ga = torch.as_tensor(A, dtype=torch.int32, device="cuda")
    gb = torch.as_tensor(B, dtype=torch.int32, device="cuda")
    R = len(A) + len(B)
    cn = torch.empty(1, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * R, dtype=torch.float32, device="cuda")
    box = (ctypes.c_double * 9)(*(np.eye(3) * L).ravel())
    stream = torch.cuda.current_stream().cuda_stream
    atoms = np.concatenate([A, B])
    expect = -F[atoms]                       # rows A then B, (R, 3)
    scale = np.abs(expect).max()
    for call in range(2):
        cn.fill_(float("nan"))
        grad.fill_(float("nan"))
        rc = lib.glued_coordination_noalloc(ctypes.c_void_p(stream), ctypes.c_void_p(ctx.posq.data_ptr()),
                                            ctypes.c_void_p(ga.data_ptr()), len(A),
                                            ctypes.c_void_p(gb.data_ptr()), len(B), 0.35, 6.0, 12.0, 1, box,
                                            ctypes.c_void_p(cn.data_ptr()), ctypes.c_void_p(grad.data_ptr()))
        assert rc == 0, lib.glued_last_error().decode()
        torch.cuda.synchronize()
        assert abs(cn.item() - cn_ref) <= 1e-6 * abs(cn_ref), (call, cn.item(), cn_ref)
        g = grad.cpu().numpy().astype(np.float64).reshape(3, R).T
        assert np.max(np.abs(g - expect)) <= 1e-5 * scale, (call, np.max(np.abs(g - expect)), scale)


def test_noalloc_rejects_groups_beyond_the_fixed_array():
    import torch
    from gluedmd_b200 import _native
    lib = _native.lib()
    idx = torch.zeros(40000, dtype=torch.int32, device="cuda")
    posq = torch.zeros((40000, 4), dtype=torch.float32, device="cuda")
    cn = torch.empty(1, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * 80000, dtype=torch.float32, device="cuda")
    box = (ctypes.c_double * 9)(*(np.eye(3) * 5.0).ravel())
    rc = lib.glued_coordination_noalloc(None, ctypes.c_void_p(posq.data_ptr()), ctypes.c_void_p(idx.data_ptr()),
                                        40000, ctypes.c_void_p(idx.data_ptr()), 40000, 0.35, 6.0, 12.0, 1, box,
                                        ctypes.c_void_p(cn.data_ptr()), ctypes.c_void_p(grad.data_ptr()))
    assert rc == -1
    assert "GLUED_NOALLOC_SCRATCH_BYTES" in lib.glued_last_error().decode()
