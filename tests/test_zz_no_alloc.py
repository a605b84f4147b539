"""The allocation-free coordination entry point against the regular context path.

glued_coordination_noalloc serves callers that cannot allocate device memory
while they evaluate forces (an engine that reserves all device memory at
start-up, or manages the heap with its own allocator): its tile partials live in
a fixed array inside the library. Its CN and dCN/dx must agree with what
glued_context_execute produces for the same coordination CV (the CV value read
back, and the forces with an injected dU/dCN = 1, i.e. F = -dCN/dx), on two
calls in a row that reuse the array, for the three switch instantiations: the
6/12 closed form, another integer pair (8/14, S_n/S_m) and a non-integer pair
(6.5/11, the reference formula in FP64).

The two sides are different kernels: this entry point sums FP32 tile partials
in a fixed order, the context path adds per-step FP32 sums into 64-bit fixed
point. The difference is FP32 partial-sum rounding, measured on B200 at
9e-8 / 6e-10 / 2e-9 of the CN and 1.5e-6 / 1.4e-6 / 8.9e-6 of the largest
gradient (6/12, 8/14, 6.5/11; the non-integer switch has the longest tail, so
the most terms per sum); the gates are CN 1e-6 relative and gradients 3e-5 of
the largest gradient."""
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


def _call(lib, stream, posq, ga, nA, gb, nB, r0, n, m, box, cn, grad):
    return lib.glued_coordination_noalloc(ctypes.c_void_p(stream), ctypes.c_void_p(posq), ctypes.c_void_p(ga), nA,
                                          ctypes.c_void_p(gb), nB, ctypes.c_double(r0), ctypes.c_double(n),
                                          ctypes.c_double(m), 1, box, ctypes.c_void_p(cn), ctypes.c_void_p(grad))


@pytest.mark.parametrize("nm", [(6.0, 12.0), (8.0, 14.0), (6.5, 11.0)])
def test_noalloc_coordination_matches_context_path(nm):
    import torch
    import gpu_util
    from gluedmd_b200 import _native

    n_, m_ = nm
    pos, A, B, L = _system()
    cvs = [(6, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.35, n_, m_])]
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
        rc = _call(lib, stream, ctx.posq.data_ptr(), ga.data_ptr(), len(A), gb.data_ptr(), len(B), 0.35, n_, m_,
                   box, cn.data_ptr(), grad.data_ptr())
        assert rc == 0, lib.glued_last_error().decode()
        torch.cuda.synchronize()
        assert abs(cn.item() - cn_ref) <= 1e-6 * abs(cn_ref), (call, cn.item(), cn_ref)
        g = grad.cpu().numpy().astype(np.float64).reshape(3, R).T
        assert np.max(np.abs(g - expect)) <= 3e-5 * scale, (call, np.max(np.abs(g - expect)), scale)


def test_noalloc_rejects_invalid_arguments_and_oversize_groups():
    import torch
    from gluedmd_b200 import _native
    lib = _native.lib()
    idx = torch.zeros(40000, dtype=torch.int32, device="cuda")
    posq = torch.zeros((40000, 4), dtype=torch.float32, device="cuda")
    cn = torch.empty(1, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * 80000, dtype=torch.float32, device="cuda")
    box = (ctypes.c_double * 9)(*(np.eye(3) * 5.0).ravel())
    args = (lib, 0, posq.data_ptr(), idx.data_ptr())
    rc = _call(*args, 40000, idx.data_ptr(), 40000, 0.35, 6.0, 12.0, box, cn.data_ptr(), grad.data_ptr())
    assert rc == -1
    assert "GLUED_NOALLOC_SCRATCH_BYTES" in lib.glued_last_error().decode()
    for r0, n, m in ((float("inf"), 6.0, 12.0), (0.35, float("nan"), 12.0), (0.35, 6.0, 0.0), (0.35, -6.0, 12.0)):
        rc = _call(*args, 10, idx.data_ptr(), 10, r0, n, m, box, cn.data_ptr(), grad.data_ptr())
        assert rc == -1, (r0, n, m)
        assert "must be finite" in lib.glued_last_error().decode()
