"""Pins the PBMETAD and EXTERNAL oracle: the reference's own known answers
(tests/test_bias_pbmetad.py, tests/test_bias_external.py) restated on the FP64
oracle, and the restatement against the reference's kernels compiled for the
host (oracle/_ref: pbmetaDSubgridEval, pbmetaDCombine, pbmetaDDeposit,
metaDEvalBias)."""
import math

import numpy as np
import pytest

import oracle as O
from ref_runner import RefSystem

needs_ref = pytest.mark.skipif(not RefSystem.available(), reason="oracle/_ref not built (reference tree absent)")

KT = 2.479
DIST01 = [(O.CV_DISTANCE, [0, 1], [])]


def _pos(d):
    return np.array([[0.0, 0.0, 0.0], [d, 0.0, 0.0], [5.0, 5.0, 5.0]])


def _pb(h0, gamma, sub, pace=1000):
    """PBMETAD spec: sub = [(sigma, origin, max, bins, periodic), ...]."""
    params = [h0, gamma, KT]
    iparams = [pace]
    for sg, lo, hi, bins, per in sub:
        params += [sg, lo, hi]
        iparams += [bins, per]
    return (O.BIAS_PBMETAD, list(range(len(sub))), params, iparams)


def _ext(cvs, origin, mx, bins, per, grid):
    return (O.BIAS_EXTERNAL, list(cvs), list(origin) + list(mx) + list(grid), list(bins) + list(per))


def gaussian_grid_1d(height, center, sigma, origin, mx, bins):
    sp = (mx - origin) / bins
    return [height * math.exp(-((origin + i * sp - center) ** 2) / (2 * sigma ** 2)) for i in range(bins + 1)]


def _deposit_once(s, d):
    """Execute at distance d, then the step-0 (skipped) and step-1 (deposit) updates."""
    s.execute(_pos(d))
    s.update_state(0)
    s.update_state(1)


# ------------------------------------------------- known answers (PBMETAD)
def test_pbmetad_zero_before_deposit():
    s = O.OracleSystem(DIST01, [_pb(1.2, 10.0, [(0.1, 0.0, 2.0, 100, 0)])], mode="f64", num_particles=3)
    assert s.execute(_pos(1.0))["energy"] == 0.0


def test_pbmetad_two_cv_empty_grids():
    cvs = DIST01 + [(O.CV_DISTANCE, [0, 2], [])]
    s = O.OracleSystem(cvs, [_pb(2.0, 10.0, [(0.1, 0.0, 2.0, 50, 0), (0.1, 3.0, 8.0, 50, 0)])], mode="f64",
                       num_particles=3)
    r = s.execute(_pos(1.0))
    assert abs(r["energy"]) < 1e-12 and np.all(r["dUdCV"] == 0.0)


def test_pbmetad_deposit_raises_energy():
    """One fixed-height deposit at cv = 1.0 (a grid point): E there is h0."""
    s = O.OracleSystem(DIST01, [_pb(2.0, 1.0, [(0.2, 0.0, 2.0, 200, 0)], pace=1)], mode="f64", num_particles=3)
    _deposit_once(s, 1.0)
    assert s.bias_state[0]["deposited"] == [1]
    E = s.execute(_pos(1.0))["energy"]
    assert abs(E - 2.0) < 1e-12


def test_pbmetad_force_matches_finite_difference():
    """FD at the midpoint of bins 100-101 with dx = half a bin: exact on the
    piecewise-linear grid."""
    s = O.OracleSystem(DIST01, [_pb(2.0, 1.0, [(0.3, 0.0, 3.0, 300, 0)], pace=1)], mode="f64", num_particles=3)
    _deposit_once(s, 1.5)
    sp = 0.01
    x, dx = 100.5 * sp, 0.5 * sp
    Ep = s.execute(_pos(x + dx))["energy"]
    Em = s.execute(_pos(x - dx))["energy"]
    F = s.execute(_pos(x))["forces"][1, 0]
    Fnum = -(Ep - Em) / (2 * dx)
    assert abs(Fnum) > 1e-3 and abs(F - Fnum) < 1e-6 * abs(Fnum)


def test_pbmetad_log_sum_exp_of_two_subgrids():
    """Two sub-grids with one deposit each: E = -kT ln(mean exp(-V_d/kT)), the
    weights of the deposit are the softmax of the previous evaluation."""
    cvs = DIST01 + [(O.CV_DISTANCE, [0, 2], [])]
    s = O.OracleSystem(cvs, [_pb(1.5, 1.0, [(0.2, 0.0, 2.0, 100, 0), (0.2, 0.0, 2.0, 100, 0)], pace=1)],
                       mode="f64", num_particles=3)
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [0.6, 0, 0]])
    s.execute(pos)
    s.update_state(0)
    s.update_state(1)     # empty grids: weights 1/2 each, height 0.75 on both sub-grids
    st = s.bias_state[0]
    r = s.execute(pos)
    V = st["V"]
    assert abs(V[0] - 0.75) < 1e-12 and abs(V[1] - 0.75) < 1e-12
    Eexp = -KT * math.log(0.5 * (math.exp(-V[0] / KT) + math.exp(-V[1] / KT)))
    assert abs(r["energy"] - Eexp) < 1e-12
    np.testing.assert_allclose(st["W"], [0.5, 0.5], rtol=0, atol=1e-15)


# ------------------------------------------------ known answers (EXTERNAL)
def test_external_zero_grid():
    s = O.OracleSystem(DIST01, [_ext([0], [0.0], [2.0], [100], [0], [0.0] * 101)], mode="f64", num_particles=3)
    assert s.execute(_pos(1.0))["energy"] == 0.0


def test_external_gaussian_peak():
    g = gaussian_grid_1d(2.0, 1.0, 0.2, 0.0, 2.0, 200)
    s = O.OracleSystem(DIST01, [_ext([0], [0.0], [2.0], [200], [0], g)], mode="f64", num_particles=3)
    assert abs(s.execute(_pos(1.0))["energy"] - 2.0) < 0.02


def test_external_force_matches_finite_difference():
    g = gaussian_grid_1d(2.0, 1.5, 0.3, 0.0, 3.0, 300)
    s = O.OracleSystem(DIST01, [_ext([0], [0.0], [3.0], [300], [0], g)], mode="f64", num_particles=3)
    sp = 0.01
    x, dx = 100.5 * sp, 0.5 * sp
    Fnum = -(s.execute(_pos(x + dx))["energy"] - s.execute(_pos(x - dx))["energy"]) / (2 * dx)
    F = s.execute(_pos(x))["forces"][1, 0]
    assert abs(Fnum) > 1e-3 and abs(F - Fnum) < 1e-6 * abs(Fnum)


def test_external_two_biases_sum():
    cvs = DIST01 + [(O.CV_DISTANCE, [0, 2], [])]
    g0 = gaussian_grid_1d(2.0, 1.0, 0.2, 0.0, 2.0, 100)
    g1 = gaussian_grid_1d(3.0, 0.8, 0.15, 0.0, 2.0, 100)
    s = O.OracleSystem(cvs, [_ext([0], [0.0], [2.0], [100], [0], g0), _ext([1], [0.0], [2.0], [100], [0], g1)],
                       mode="f64", num_particles=3)
    E = s.execute(np.array([[0.0, 0, 0], [1.0, 0, 0], [0.8, 0, 0]]))["energy"]
    assert abs(E - 5.0) < 0.05


def test_external_matches_metad_after_deposit():
    """A fixed-height MetaD deposit at 1.0 and an EXTERNAL grid holding the same
    Gaussian give the same bias at 0.8."""
    m = O.OracleSystem(DIST01, [(O.BIAS_METAD, [0], [2.0, 0.2, 1.0, KT, 0.0, 2.0], [1, 200, 0])], mode="f64",
                       num_particles=3)
    _deposit_once(m, 1.0)
    Em = m.execute(_pos(0.8))["energy"]
    g = gaussian_grid_1d(2.0, 1.0, 0.2, 0.0, 2.0, 200)
    e = O.OracleSystem(DIST01, [_ext([0], [0.0], [2.0], [200], [0], g)], mode="f64", num_particles=3)
    assert abs(e.execute(_pos(0.8))["energy"] - Em) < 1e-12 * max(1.0, abs(Em))


# ------------------------------------------------ vs the reference kernels
def pbmetad_system(pace=2, gamma=10.0):
    """Two periodic dihedral sub-grids and one non-periodic distance sub-grid."""
    cvs = [(O.CV_DIHEDRAL, [0, 1, 2, 3], []), (O.CV_DIHEDRAL, [1, 2, 3, 4], []), (O.CV_DISTANCE, [0, 5], [])]
    sub = [(0.35, -math.pi, math.pi, 64, 1), (0.3, -math.pi, math.pi, 48, 1), (0.1, 0.0, 2.5, 100, 0)]
    return cvs, [_pb(1.2, gamma, sub, pace=pace)]


def external_system(seed=3):
    """2-D EXTERNAL grid of random values over a periodic dihedral and a distance."""
    cvs = [(O.CV_DIHEDRAL, [0, 1, 2, 3], []), (O.CV_DISTANCE, [0, 5], [])]
    rng = np.random.default_rng(seed)
    bins, per = [36, 50], [1, 0]
    grid = rng.uniform(-2.0, 5.0, 36 * 51)
    return cvs, [_ext([0, 1], [-math.pi, 0.0], [math.pi, 2.5], bins, per, grid)]


@needs_ref
@pytest.mark.parametrize("gamma", [10.0, 1.0])
def test_pbmetad_deposit_and_eval_vs_reference(gamma):
    """Pace-gated deposits on three sub-grids and the log-sum-exp evaluation over
    40 steps vs the reference kernels."""
    cvs, biases = pbmetad_system(pace=2, gamma=gamma)
    rng = np.random.default_rng(11)
    a = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    b = RefSystem(cvs, biases, mode="f64", num_particles=6)
    for step in range(40):
        pos = rng.uniform(0, 1.5, (6, 3))
        a.update_state(step); b.update_state(step)
        ra, rb = a.execute(pos), b.execute(pos)
        assert abs(ra["energy"] - rb["energy"]) < 1e-9 * max(1, abs(rb["energy"]))
        np.testing.assert_allclose(ra["dUdCV"], rb["dUdCV"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(a.bias_state[0]["grid"], b.bias_state[0]["grid"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(a.bias_state[0]["W"], b.bias_state[0]["W"], rtol=1e-12, atol=1e-15)
    assert a.bias_state[0]["deposited"] == b.bias_state[0]["deposited"] == [19, 19, 19]


@needs_ref
def test_external_eval_vs_reference():
    cvs, biases = external_system()
    rng = np.random.default_rng(5)
    a = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    b = RefSystem(cvs, biases, mode="f64", num_particles=6)
    for _ in range(20):
        pos = rng.uniform(0, 1.5, (6, 3))
        ra, rb = a.execute(pos), b.execute(pos)
        assert abs(ra["energy"] - rb["energy"]) < 1e-12 * max(1, abs(rb["energy"]))
        np.testing.assert_allclose(ra["dUdCV"], rb["dUdCV"], rtol=1e-12, atol=1e-12)
