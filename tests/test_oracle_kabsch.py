"""Pins the oracle's Kabsch RMSD (CV_RMSD_KABSCH; the reference has only no-fit
RMSD, so the FP64 oracle is the definition the GPU path is checked against):

* value equal to an independent SVD solution of the same superposition problem
  (proper rotations only: the sign of the smallest singular direction is
  flipped when det(U V^T) < 0);
* analytic gradient equal to central finite differences (FP64, eps = 1e-4;
  1e-6 next to a degenerate rotation);
* zero for an identical structure and for a 180 degree rotation of it;
* near-degenerate eigenvalues (nearly collinear atoms): value and gradient
  still match SVD and finite differences.
"""
import math

import numpy as np
import pytest

import oracle as O


def _kabsch_svd(x, y):
    xc, yc = x - x.mean(0), y - y.mean(0)
    H = yc.T @ xc
    U, S, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(Vt.T @ U.T))
    D = np.diag([1.0, 1.0, d])
    R = Vt.T @ D @ U.T
    diff = xc - yc @ R.T
    return math.sqrt((diff * diff).sum() / len(x))


def _oracle(pos, ref):
    n = len(ref)
    cvs = [(O.CV_RMSD_KABSCH, list(range(n)), list(np.asarray(ref, float).ravel()))]
    s = O.OracleSystem(cvs, mode="f64", num_particles=len(pos))
    cvv, jac = s.evaluate_cvs(pos)
    ja, jx, jy, jz, jc = jac
    g = np.zeros((len(pos), 3))
    for r in range(len(ja)):
        g[ja[r]] += (jx[r], jy[r], jz[r])
    return cvv[0], g


def _rot(axis, angle):
    a = np.asarray(axis, float)
    a /= np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * K @ K


def _case(kind, n=40, seed=3):
    rng = np.random.default_rng(seed)
    if kind == "collinear":
        t = np.linspace(-1, 1, n)
        x = np.c_[t, 0.5 * t, -0.3 * t] + rng.normal(0, 1e-3, (n, 3))
    else:
        x = rng.uniform(0, 2, (n, 3))
    c = x.mean(0)
    if kind == "rot180":
        y = (x - c) @ _rot([0.2, 1.0, -0.4], math.pi).T + c
    else:
        y = (x - c) @ _rot(rng.normal(size=3), rng.uniform(0, math.pi)).T + c + rng.normal(0, 0.1, x.shape)
    # the oracle stores reference coordinates as float (the reference's parameter arrays)
    return x, y.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("kind", ["random", "collinear"])
def test_kabsch_value_matches_svd(kind):
    x, y = _case(kind)
    v, _ = _oracle(x, y)
    assert abs(v - _kabsch_svd(x, y)) < 1e-10 * max(1.0, v)


# Near the degenerate rotation (nearly collinear atoms) the RMSD has a large third
# derivative: the central-difference truncation error, O(eps^2), is 2.4e-4 relative
# at eps = 1e-4 for the oracle and for the SVD solution alike, and 2.4e-6 at 1e-5;
# that case uses eps = 1e-6.
@pytest.mark.parametrize("kind,eps", [("random", 1e-4), ("collinear", 1e-6)])
def test_kabsch_gradient_central_differences(kind, eps):
    x, y = _case(kind, n=25)
    v, g = _oracle(x, y)
    fd = np.zeros_like(x)
    for i in range(len(x)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, k] += eps
            xm[i, k] -= eps
            fd[i, k] = (_oracle(xp, y)[0] - _oracle(xm, y)[0]) / (2 * eps)
    assert np.abs(fd - g).max() < 1e-6 * np.abs(g).max()


def test_kabsch_zero_for_identity_and_half_turn():
    x, y = _case("rot180")
    v, _ = _oracle(x, y)
    assert v < 1e-6
    v0, g0 = _oracle(x, x)
    assert v0 < 1e-7
