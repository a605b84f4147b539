"""Pins the CPU oracle: known answers from the reference's tests, and the
restatement vs the reference's own kernels compiled for the host (oracle/_ref)."""
import math

import numpy as np
import pytest

import oracle as O
from cases import CASES, TOL_CV, TOL_F
from ref_runner import RefSystem


def _box(case):
    L = case.get("box")
    return None if L is None else np.diag([L, L, L]).ravel()


def _run(case, mode, cls=O.OracleSystem):
    pos = np.array(case["pos"], float)
    sysm = cls(case["cvs"], masses=case.get("masses"), periodic=case.get("pbc", False), mode=mode,
               test_bias_gradients=case.get("grad"), num_particles=len(pos))
    return sysm.execute(pos, _box(case))


def check_case(case, res):
    tol = case.get("tol", TOL_CV)
    cvv = res["cv_values"]
    for i, v in enumerate(case.get("cv", [])):
        assert abs(cvv[i] - v) < tol, (case["name"], i, cvv[i], v)
    for i, v in enumerate(case.get("cv_abs", [])):
        assert abs(abs(cvv[i]) - v) < tol, (case["name"], i, cvv[i], v)
    for i, v in enumerate(case.get("cv_below", [])):
        assert cvv[i] < v, (case["name"], i, cvv[i], v)
    F = res["forces"]
    for a, f in case.get("forces", {}).items():
        for c in range(3):
            assert abs(F[a][c] - f[c]) < TOL_F, (case["name"], a, c, F[a][c], f[c])
    if "force_sum_zero" in case:
        s = F[case["force_sum_zero"]].sum(axis=0)
        assert np.all(np.abs(s) < TOL_F), (case["name"], s)


@pytest.mark.parametrize("mode", ["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_known_answers(case, mode):
    check_case(case, _run(case, mode))


needs_ref = pytest.mark.skipif(not RefSystem.available(), reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_reference_kernels_known_answers(case):
    """The compiled reference kernels pass the same known answers (harness check)."""
    check_case(case, _run(case, "f32", RefSystem))


def random_system(seed, n_atoms=60, box=3.0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, box, (n_atoms, 3))
    perm = rng.permutation(n_atoms)
    cvs = [
        (O.CV_DISTANCE, list(perm[0:2]), []), (O.CV_DISTANCE, list(perm[2:4]), []),
        (O.CV_ANGLE, list(perm[4:7]), []),
        (O.CV_DIHEDRAL, list(perm[7:11]), []), (O.CV_DIHEDRAL, list(perm[11:15]), []),
        (O.CV_COM_DISTANCE, list(perm[15:25]), [4]),
        (O.CV_GYRATION, list(perm[20:40]), []),
        (O.CV_COORDINATION, [12] + list(perm[0:12]) + list(perm[30:55]), [0.45, 6, 12]),
        (O.CV_COORDINATION, [3] + list(perm[40:43]) + list(perm[5:15]), [0.6, 1, 2]),
        (O.CV_RMSD, list(perm[10:30]), list((pos[perm[10:30]] + rng.normal(0, 0.1, (20, 3))).ravel())),
        (O.CV_PATH, list(perm[30:36]),
         [1.7, 4] + list(np.concatenate([(pos[perm[30:36]] + rng.normal(0, 0.2, (6, 3))).ravel() for _ in range(4)]))),
        (O.CV_CONTACTMAP, list(perm[0:20]), [v for i in range(10) for v in (rng.uniform(0.4, 0.8), 6, 12, 1.0)]),
        (O.CV_PCA, list(perm[0:8]), list(rng.uniform(0, box, 24)) + list(rng.normal(0, 1, 24))),
    ]
    masses = rng.uniform(1, 16, n_atoms)
    return pos, cvs, masses, np.diag([box, box, box]).ravel()


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("periodic", [False, True])
def test_restatement_matches_reference_kernels(seed, periodic):
    """Restated FP32 semantics vs the compiled reference kernels, same inputs."""
    pos, cvs, masses, box = random_system(seed)
    ncv = sum(2 if t == O.CV_PATH else 1 for t, a, p in cvs)
    g = list(np.random.default_rng(seed + 100).normal(0, 1, ncv))
    mine = O.OracleSystem(cvs, masses=masses, periodic=periodic, mode="f32", test_bias_gradients=g,
                          num_particles=len(pos)).execute(pos, box)
    ref = RefSystem(cvs, masses=masses, periodic=periodic, mode="f32", test_bias_gradients=g,
                    num_particles=len(pos)).execute(pos, box)
    np.testing.assert_allclose(mine["cv_values"], ref["cv_values"], rtol=2e-6, atol=2e-6)
    # Same Jacobian layout: identical atom and CV index columns.
    assert np.array_equal(mine["jacobian"][0], ref["jacobian"][0])
    assert np.array_equal(mine["jacobian"][4], ref["jacobian"][4])
    for c in (1, 2, 3):
        np.testing.assert_allclose(mine["jacobian"][c], ref["jacobian"][c], rtol=1e-4, atol=2e-5)
    assert O.max_rel_force_err(mine["forces"], ref["forces"]) < 1e-4


@needs_ref
@pytest.mark.parametrize("seed", [4, 5])
def test_fp64_oracle_vs_reference_fp64_build(seed):
    pos, cvs, masses, box = random_system(seed)
    ncv = sum(2 if t == O.CV_PATH else 1 for t, a, p in cvs)
    g = list(np.random.default_rng(seed).normal(0, 1, ncv))
    mine = O.OracleSystem(cvs, masses=masses, periodic=True, mode="f64", test_bias_gradients=g,
                          num_particles=len(pos)).execute(pos, box)
    ref = RefSystem(cvs, masses=masses, periodic=True, mode="f64", test_bias_gradients=g,
                    num_particles=len(pos)).execute(pos, box)
    # The reference's double build still rounds some intermediates to float: group-B
    # positions in the coordination cache (CommonGluedKernels.cpp:959-965), path atom
    # positions (:700-706) and every stored Jacobian component. Agreement is therefore
    # at float resolution, not at double resolution.
    np.testing.assert_allclose(mine["cv_values"], ref["cv_values"], rtol=1e-6, atol=1e-7)
    assert O.max_rel_force_err(mine["forces"], ref["forces"]) < 1e-5


def metad_system(pace=1, D=2, periodic=1, gamma=10.0):
    cvs = [(O.CV_DIHEDRAL, [0, 1, 2, 3], []), (O.CV_DIHEDRAL, [1, 2, 3, 4], [])][:D]
    params = [1.2] + [0.35] * D + [gamma, 2.494338785] + [-math.pi] * D + [math.pi] * D
    iparams = [pace] + [64] * D + [periodic] * D
    return cvs, [(O.BIAS_METAD, list(range(D)), params, iparams)]


@needs_ref
def test_metad_grid_deposit_and_eval_vs_reference():
    """Pace-gated WT deposit + multilinear eval over 40 steps vs reference kernels."""
    cvs, biases = metad_system(pace=2)
    rng = np.random.default_rng(7)
    a = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    b = RefSystem(cvs, biases, mode="f64", num_particles=6)
    for step in range(40):
        pos = rng.uniform(0, 1.5, (6, 3))
        a.update_state(step); b.update_state(step)
        ra, rb = a.execute(pos), b.execute(pos)
        assert abs(ra["energy"] - rb["energy"]) < 1e-9 * max(1, abs(rb["energy"]))
        np.testing.assert_allclose(ra["dUdCV"], rb["dUdCV"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(a.bias_state[0]["grid"], b.bias_state[0]["grid"], rtol=1e-12, atol=1e-12)
    assert a.bias_state[0]["deposited"] == b.bias_state[0]["deposited"] == 19


def opes_system(variant=0, pace=1, sigma=0.3, maxk=100000):
    cvs = [(O.CV_DISTANCE, [0, 1], []), (O.CV_DISTANCE, [2, 3], [])]
    params = [2.494338785, 20.05, sigma, sigma, 0.02]
    return cvs, [(O.BIAS_OPES, [0, 1], params, [variant, pace, maxk])]


@needs_ref
@pytest.mark.parametrize("variant", [0, 2])
def test_opes_deposit_sequence_vs_reference(variant):
    """OPES deposits (Silverman sigma, merge/append decisions, sum_uprob) over 60
    steps agree with the reference kernels: same kernel counts, tables and bias."""
    cvs, biases = opes_system(variant)
    rng = np.random.default_rng(11)
    a = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    b = RefSystem(cvs, biases, mode="f64", num_particles=4)
    for step in range(60):
        pos = rng.uniform(0, 1.0, (4, 3))
        a.update_state(step); b.update_state(step)
        ra, rb = a.execute(pos), b.execute(pos)
        assert abs(ra["energy"] - rb["energy"]) < 1e-8 * max(1.0, abs(rb["energy"]))
    sa, sb = a.bias_state[0], b.bias_state[0]
    assert int(sa["ist"][0]) == int(sb["ist"][0])
    nk = int(sa["ist"][0])
    assert any(d >= 0 for d in sa["decisions"]), "replay should include merges"
    np.testing.assert_allclose(sa["centers"][:2 * nk], sb["centers"][:2 * nk], rtol=1e-12)
    np.testing.assert_allclose(sa["sigmas"][:2 * nk], sb["sigmas"][:2 * nk], rtol=1e-12)
    np.testing.assert_allclose(sa["logw"][:nk], sb["logw"][:nk], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(sa["dst"], sb["dst"], rtol=1e-11)


@pytest.mark.parametrize("variant", [0, 2])
def test_opes_decisions_only_replay_matches_full(variant):
    """The decisions-only deposit mode (no sum_uprob update) produces the same
    decisions and kernel tables as the full deposit when both are fed the same
    CV values and bias energies."""
    cvs, biases = opes_system(variant)
    rng = np.random.default_rng(4)
    a = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    b = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    b.decisions_only = True
    for step in range(80):
        pos = rng.uniform(0, 1.0, (4, 3))
        a.update_state(step); b.update_state(step)
        ra = a.execute(pos)
        b.cv_values = ra["cv_values"].copy(); b.bias_energies = ra["bias_energies"].copy(); b.cv_ready = True
    sa, sb = a.bias_state[0], b.bias_state[0]
    assert sa["decisions"] == sb["decisions"]
    assert any(d >= 0 for d in sa["decisions"]) and any(d == -1 for d in sa["decisions"])
    nk = int(sa["ist"][0])
    assert nk == int(sb["ist"][0])
    assert np.array_equal(sa["centers"][:2 * nk], sb["centers"][:2 * nk])
    assert np.array_equal(sa["sigmas"][:2 * nk], sb["sigmas"][:2 * nk])
    assert np.array_equal(sa["logw"][:nk], sb["logw"][:nk])
    assert sb["dst"][0] == 0.0 and sa["dst"][0] != 0.0


def test_deterministic_math_against_libm():
    """gd_exp / gd_log / gd_pow stay within a few ulp of the C library."""
    import ctypes
    # exercised through the OPES deposit on a 1-kernel case with known Silverman sigma
    cvs, biases = opes_system(variant=0, sigma=0.2)
    s = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    pos = np.array([[0, 0, 0], [0.5, 0, 0], [0, 0, 0], [0.7, 0, 0]], float)
    s.execute(pos)
    s.update_state(1)
    st = s.bias_state[0]
    g = st["gamma"]
    sw = 2 * math.exp(-g); sw2 = math.exp(-2 * g) + math.exp(-2 * g)
    neff = (1 + sw) ** 2 / (1 + sw2)
    sig = 0.2 * (neff * 4 / 4.0) ** (-1 / 6.0)
    assert abs(st["sigmas"][0] - sig) < 4e-16 * sig * 8
    lw = -g + math.log(0.2 / sig) * 2
    assert abs(st["logw"][0] - lw) < 1e-13
