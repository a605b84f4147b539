"""Differentiable contact-map + path + hill bias (gluedmd_b200.autograd).

* torch.autograd.gradcheck in float64 with eps = 1e-4 on positions, contact
  r0, path frames and hill heights (atol 1e-5, rtol 1e-3);
* forces -dE/dx against the FP64 oracle: the oracle's contact-map and path-CV
  values and Jacobians (CommonGluedKernels.cpp:1236-1323, :641-794 restated)
  combined with dE/dCV of the hill sum; FP32 kernels within 1e-4 relative
  (max-norm), FP64 kernels within 1e-8; on a small system and on the full C5
  size (30,000 atoms, 10,000 pairs, 50 frames x 500 atoms, 2,000 hills)."""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _system(n_atoms=60, n_pairs=40, F=6, M=8, K=20, seed=3, box=None):
    rng = np.random.default_rng(seed)
    L = 2.0
    pos = rng.uniform(0, L, (n_atoms, 3))
    pairs = np.stack([rng.integers(0, n_atoms, n_pairs), rng.integers(0, n_atoms, n_pairs)], 1)
    pairs[pairs[:, 0] == pairs[:, 1], 1] = (pairs[pairs[:, 0] == pairs[:, 1], 1] + 1) % n_atoms
    r0 = rng.uniform(0.4, 0.8, n_pairs)
    patoms = rng.choice(n_atoms, M, replace=False)
    frames = [pos[patoms] + rng.normal(0, 0.05, (M, 3))]
    for _ in range(F - 1):
        frames.append(frames[-1] + rng.normal(0, 0.05, (M, 3)))
    frames = np.array(frames)
    msd = np.mean([((frames[i + 1] - frames[i]) ** 2).sum(-1).mean() for i in range(F - 1)])
    lam = 2.3 / msd
    return pos, pairs, r0, patoms, frames, lam


def _oracle_forces(pos, pairs, r0, patoms, frames, lam, centers, heights, sigma):
    P = len(pairs)
    cm_params = [v for i in range(P) for v in (r0[i], 6.0, 12.0, 1.0)]
    cvs = [(O.CV_CONTACTMAP, list(pairs.ravel()), cm_params),
           (O.CV_PATH, list(patoms), [lam, len(frames)] + list(frames.ravel()))]
    # dE/dCV of the smooth hill sum on (CMAP, s)
    sysm = O.OracleSystem(cvs, mode="f64", num_particles=len(pos), test_bias_gradients=[0.0, 0.0, 0.0])
    cvv, _ = sysm.evaluate_cvs(pos)
    d0 = cvv[0] - centers[:, 0]
    d1 = cvv[1] - centers[:, 1]
    g = heights * np.exp(-d0 ** 2 / (2 * sigma[0] ** 2) - d1 ** 2 / (2 * sigma[1] ** 2))
    E = g.sum()
    dE = [(-g * d0 / sigma[0] ** 2).sum(), (-g * d1 / sigma[1] ** 2).sum(), 0.0]
    sysm.test_grad = np.array(dE)
    r = sysm.execute(pos)
    return E, r["forces"], cvv


def _torch_inputs(pos, r0, frames, heights, dtype):
    import torch
    return [torch.tensor(np.asarray(x), dtype=dtype, device="cuda", requires_grad=True)
            for x in (pos, r0, frames, heights)]


def test_gradcheck_fp64():
    import torch
    from gluedmd_b200.autograd import BiasTopology, glued_bias
    pos, pairs, r0, patoms, frames, lam = _system()
    rng = np.random.default_rng(9)
    # hills around the current CV values so that every gradient is exercised
    from gluedmd_b200.autograd import cv_values
    K = 20
    topo0 = BiasTopology.build(pairs, np.c_[r0, np.full(len(r0), 6.0), np.full(len(r0), 12.0), np.ones(len(r0))],
                               patoms, lam, np.zeros((K, 2)), (0.5, 0.6))
    p, r, f, h = _torch_inputs(pos, r0, frames, np.ones(K), torch.float64)
    _, cm, s, _ = cv_values(p, r, f, h, topo0)
    centers = np.c_[cm + rng.normal(0, 0.6, K), s + rng.normal(0, 0.8, K)]
    topo = BiasTopology.build(pairs, np.c_[r0, np.full(len(r0), 6.0), np.full(len(r0), 12.0), np.ones(len(r0))],
                              patoms, lam, centers, (0.5, 0.6))
    heights = rng.uniform(0.5, 1.5, K)
    inputs = _torch_inputs(pos, r0, frames, heights, torch.float64)
    assert torch.autograd.gradcheck(lambda a, b, c, d: glued_bias(a, b, c, d, topo), inputs, eps=1e-4, atol=1e-5,
                                    rtol=1e-3)


@pytest.mark.parametrize("full", [False, True])
def test_forces_vs_fp64_oracle(full):
    import torch
    from gluedmd_b200.autograd import BiasTopology, glued_bias, cv_values
    if full:
        from gluedmd_b200 import workloads as W
        w = W.config5()
        pos, pairs, r0 = w.positions, w.extra["pairs"], w.extra["r0"]
        patoms, frames, lam = w.extra["patoms"], w.extra["frames"], w.extra["lam"]
        K = 2000
    else:
        pos, pairs, r0, patoms, frames, lam = _system()
        K = 30
    # the oracle stores r0, frames and lambda as float (the reference's
    # parameter arrays); give the FP64 kernels the same float-representable values
    r0 = np.asarray(r0, np.float32).astype(np.float64)
    frames = np.asarray(frames, np.float32).astype(np.float64)
    lam = float(np.float32(lam))
    nmw = np.c_[r0, np.full(len(r0), 6.0), np.full(len(r0), 12.0), np.ones(len(r0))]
    sigma = (0.02 * max(1.0, len(r0) / 40.0), 0.35)
    topo0 = BiasTopology.build(pairs, nmw, patoms, lam, np.zeros((K, 2)), sigma)
    p, r, f, h = _torch_inputs(pos, r0, frames, np.ones(K), torch.float64)
    _, cm, s, _ = cv_values(p, r, f, h, topo0)
    rng = np.random.default_rng(2)
    centers = np.c_[cm + rng.uniform(-3, 3, K) * sigma[0], s + rng.uniform(-3, 3, K) * sigma[1]]
    heights = rng.uniform(0.2, 1.2, K)
    topo = BiasTopology.build(pairs, nmw, patoms, lam, centers, sigma)
    E_ref, F_ref, cvv = _oracle_forces(pos, pairs, r0, patoms, frames, lam, centers, heights, sigma)
    # FP64: 1e-8 (summation order over 10,000 pairs / 50 frames differs from the oracle's serial loops)
    for dtype, tol in ((torch.float32, 1e-4), (torch.float64, 1e-8)):
        p, r, f, h = _torch_inputs(pos, r0, frames, heights, dtype)
        E = glued_bias(p, r, f, h, topo)
        E.backward()
        F = -p.grad.double().cpu().numpy()
        assert O.max_rel_force_err(F, F_ref) < tol, (dtype, O.max_rel_force_err(F, F_ref))
        assert abs(E.item() - E_ref) <= max(tol, 1e-6) * max(1.0, abs(E_ref))
        # heights: dE/dh_k is the k-th Gaussian
        d0 = cvv[0] - centers[:, 0]
        d1 = cvv[1] - centers[:, 1]
        G = np.exp(-d0 ** 2 / (2 * sigma[0] ** 2) - d1 ** 2 / (2 * sigma[1] ** 2))
        np.testing.assert_allclose(h.grad.double().cpu().numpy(), G, rtol=max(tol, 1e-5) * 10,
                                   atol=max(tol, 1e-7))


def test_backward_is_bitwise_repeatable():
    import torch
    from gluedmd_b200.autograd import BiasTopology, glued_bias
    pos, pairs, r0, patoms, frames, lam = _system(n_atoms=400, n_pairs=600, F=10, M=40, K=50)
    nmw = np.c_[r0, np.full(len(r0), 6.0), np.full(len(r0), 12.0), np.ones(len(r0))]
    centers = np.random.default_rng(0).uniform(0, 5, (50, 2))
    topo = BiasTopology.build(pairs, nmw, patoms, lam, centers, (2.0, 2.0))
    grads = []
    for _ in range(2):
        p, r, f, h = _torch_inputs(pos, r0, frames, np.ones(50), torch.float32)
        glued_bias(p, r, f, h, topo).backward()
        grads.append(p.grad.cpu().numpy())
    assert np.array_equal(grads[0], grads[1])
