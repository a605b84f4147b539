"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Tolerances: CV values 1e-5 relative (FP32 CV arithmetic vs FP64 oracle);
forces 1e-4 relative in max-norm against the FP64 oracle (the acceptance gate);
integer state (deposit counts, OPES decisions, kernel tables) bit-exact."""
import math

import numpy as np
import pytest

import oracle as O
from cases import CASES
from test_oracle import check_case, random_system, metad_system, opes_system

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4


def _gpu():
    import gpu_util
    return gpu_util


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_known_answers_gpu(case):
    L = case.get("box")
    box = None if L is None else np.diag([L, L, L])
    res = _gpu().run(case["pos"], case["cvs"], masses=case.get("masses"), pbc=case.get("pbc", False), box=box,
                     grad=case.get("grad"))
    check_case(case, res)


@pytest.mark.parametrize("seed", [1, 2, 3, 7])
@pytest.mark.parametrize("periodic", [False, True])
def test_random_systems_vs_fp64_oracle(seed, periodic):
    pos, cvs, masses, box = random_system(seed)
    ncv = sum(2 if t == O.CV_PATH else 1 for t, a, p in cvs)
    g = list(np.random.default_rng(seed + 100).normal(0, 1, ncv))
    ref = O.OracleSystem(cvs, masses=masses, periodic=periodic, mode="f64", test_bias_gradients=g,
                         num_particles=len(pos)).execute(pos, box)
    res = _gpu().run(pos, cvs, masses=masses, pbc=periodic, box=box.reshape(3, 3), grad=g)
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


@pytest.mark.parametrize("nm", [(6, 12), (8, 14), (4.5, 9.5)])
@pytest.mark.parametrize("periodic", [False, True])
def test_coordination_overlapping_groups_multi_tile(nm, periodic):
    """Groups sharing atoms (self pairs are excluded by the reference's r^2 >= 1e-20
    bound), ragged sizes that leave partial A tiles and B chunks, and two
    coordination CVs in one launch."""
    rng = np.random.default_rng(21)
    n, L = 1500, 2.5
    pos = rng.uniform(0, L, (n, 3))
    A = rng.choice(n, 203, replace=False)
    B = np.concatenate([A[:50], rng.choice(n, 331, replace=False)])
    A2 = rng.choice(n, 64, replace=False)
    B2 = rng.choice(n, 128, replace=False)
    cvs = [(O.CV_COORDINATION, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.3, nm[0], nm[1]]),
           (O.CV_COORDINATION, [len(A2)] + [int(x) for x in A2] + [int(x) for x in B2], [0.25, nm[0], nm[1]])]
    g = [0.7, -1.3]
    box = np.diag([L, L, L]).ravel()
    ref = O.OracleSystem(cvs, periodic=periodic, mode="f64", test_bias_gradients=g, num_particles=n).execute(pos, box)
    res = _gpu().run(pos, cvs, pbc=periodic, box=box.reshape(3, 3), grad=g)
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


def test_atom_reorder_gives_identical_forces():
    """OpenMM's GPU-slot reordering must not change anything (fixed-point sums are
    order independent): forces bit-identical with and without a permutation."""
    pos, cvs, masses, box = random_system(11)
    ncv = sum(2 if t == O.CV_PATH else 1 for t, a, p in cvs)
    g = list(np.random.default_rng(5).normal(0, 1, ncv))
    a = _gpu().run(pos, cvs, masses=masses, pbc=True, box=box.reshape(3, 3), grad=g)
    perm = np.random.default_rng(3).permutation(len(pos))
    b = _gpu().run(pos, cvs, masses=masses, pbc=True, box=box.reshape(3, 3), grad=g, reorder=perm)
    assert np.array_equal(a["forces"], b["forces"])
    assert np.array_equal(a["cv_values"], b["cv_values"])
    # reordering an existing context in place
    ctx = a["ctx"]
    ctx.reorderAtoms(perm)
    e, F = ctx.computeForces()
    assert np.array_equal(F, a["forces"])


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_fixed_point_io(mode):
    """setTestForce modes (tests/test_gpu_io.py:56-119): constant, per-user-atom and
    PBC distance written through the fixed-point buffer, with a reordered layout."""
    from gluedmd_b200.context import Context, System
    from gluedmd_b200 import GluedForce
    n = 8
    s = System()
    for _ in range(n):
        s.addParticle(1.0)
    f = GluedForce()
    f.setTestForce(mode, 0.25)
    f.setUsesPeriodicBoundaryConditions(True)
    s.addForce(f)
    s.setDefaultPeriodicBoxVectors([1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0])
    pos = np.zeros((n, 3)); pos[1] = [0.99, 0, 0]
    perm = np.arange(n)[::-1].copy()
    ctx = Context(s, pos, reorder=perm)
    e, F = ctx.computeForces()
    if mode == 1:
        assert np.allclose(F[:, 0], 0.25, atol=1e-9)
    elif mode == 2:
        assert np.allclose(F[:, 0], 0.25 * np.arange(n), atol=1e-9)
    else:
        # written to slot 0 -> user atom perm[0]
        assert abs(F[perm[0], 0] - 0.01) < 1e-5


def test_metad_grid_replay_vs_oracle():
    """Pace-gated WT grid deposits and evaluation over 40 steps (C1-like, 64x64
    periodic grid), the oracle depositing at its own FP64 CV values: energies agree
    to 1e-5 relative and the blob carries the 'GPUS' v1 header. The grid array and
    numDeposited are compared exactly in
    test_gpu_paths.py::test_metad_grid_and_deposit_count_replay."""
    cvs, biases = metad_system(pace=2)
    rng = np.random.default_rng(7)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    ctx, f = _gpu().make_context(np.zeros((6, 3)), cvs, biases)
    for step in range(40):
        pos = rng.uniform(0, 1.5, (6, 3))
        ctx.setPositions(pos)
        ctx.setStepCount(step)
        ctx.updateContextState()
        orc.update_state(step)
        e, F = ctx.computeForces()
        r = orc.execute(pos)
        # the oracle's own FP64 CV values: agreement to the FP32 CV resolution
        assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"]))
    blob = f.getBiasState()
    import struct
    assert blob[:4] == b"GPUS" and struct.unpack("<i", blob[4:8])[0] == 1


def test_opes_decisions_bit_exact():
    """OPES deposit replay: the oracle is fed the product's CV values and bias
    energy each step, then merge/append decisions, kernel centres, sigmas and
    log-weights must be bit-identical (FP64 decision path without FMA)."""
    cvs, biases = opes_system(variant=0, pace=1, sigma=0.3)
    rng = np.random.default_rng(11)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    ctx, f = _gpu().make_context(np.zeros((4, 3)), cvs, biases)
    nc = ctx.glued_context_for(f)
    dec_gpu = []
    for step in range(120):
        pos = rng.uniform(0, 1.0, (4, 3))
        ctx.setStepCount(step)
        ctx.updateContextState()
        if step > 0:
            dec_gpu.append(nc.opes_last_decision(0))
        # oracle deposit from the product's previous CVs / energy
        orc.update_state(step)
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        orc.cv_values = np.array(nc.cv_values())
        orc.bias_energies = np.array([e])
        orc.cv_ready = True
    st = orc.bias_state[0]
    dec_orc = [d for d in st["decisions"]]
    assert dec_gpu[:len(dec_orc)] == dec_orc
    assert any(d >= 0 for d in dec_orc) and any(d == -1 for d in dec_orc)
    blob = f.getBiasState()
    import struct
    nk = struct.unpack("<i", blob[12:16])[0]
    assert nk == int(st["ist"][0])
    off = 16 + 8 + 4 + 2 * 8 * 2
    c = np.frombuffer(blob[off:off + 16 * nk], "<f8")
    s_ = np.frombuffer(blob[off + 16 * nk:off + 32 * nk], "<f8")
    lw = np.frombuffer(blob[off + 32 * nk:off + 40 * nk], "<f8")
    assert np.array_equal(c, st["centers"][:2 * nk])
    assert np.array_equal(s_, st["sigmas"][:2 * nk])
    assert np.array_equal(lw, st["logw"][:nk])


def test_opes_decisions_bit_exact_c3_scale():
    """2,000 OPES deposits on the C3 system (50,000 atoms, COM distance + gyration
    of 5,000 atoms) starting from its 10,000-kernel compressed table: every
    merge/append decision and the final centres, sigmas and log-weights are
    bit-identical to the oracle fed the product's CV values and bias energy.
    The oracle skips the O(N^2) sum_uprob recomputation after merges (the sum
    enters the bias value, never a decision)."""
    import gpu_util
    from gluedmd_b200 import workloads as W
    import struct
    w = W.config3()
    n = len(w.positions)
    orc = O.OracleSystem(w.cvs, w.biases, mode="f64", num_particles=n, periodic=True)
    orc.load_blob(w.blob)
    orc.decisions_only = True
    ctx, f = gpu_util.make_context(w.positions, w.cvs, w.biases, masses=w.masses, pbc=True, box=w.box,
                                   blob=w.blob)
    nc = ctx.glued_context_for(f)
    pace = w.biases[0][3][1]
    sel = np.asarray(w.extra["sel"])
    half = sel[:len(sel) // 2]
    rng = np.random.default_rng(21)
    pos0 = np.asarray(w.positions, float)
    shift = np.zeros(3)
    scale = 1.0
    dec_gpu = []
    n_dep = 2000
    for k in range(n_dep + 1):
        step = k * pace
        ctx.setStepCount(step)
        ctx.updateContextState()
        if k > 0:
            dec_gpu.append(nc.opes_last_decision(0))
        orc.update_state(step)
        shift += rng.normal(0.0, 0.02, 3)
        scale = float(np.clip(scale + rng.normal(0.0, 0.004), 0.9, 1.1))
        pos = pos0.copy()
        cen = pos0[sel].mean(0)
        pos[sel] = cen + (pos0[sel] - cen) * scale
        pos[half] += shift
        ctx.setPositions(pos)
        e, _ = ctx.computeForces()
        orc.cv_values = np.array(nc.cv_values())
        orc.bias_energies = np.array([e])
        orc.cv_ready = True
    st = orc.bias_state[0]
    dec_orc = list(st["decisions"])
    assert len(dec_orc) == n_dep
    assert dec_gpu == dec_orc
    assert sum(d >= 0 for d in dec_orc) > 50 and sum(d == -1 for d in dec_orc) > 50
    blob = f.getBiasState()
    nk = struct.unpack("<i", blob[12:16])[0]
    assert nk == int(st["ist"][0])
    off = 16 + 8 + 4 + 2 * 8 * 2
    c = np.frombuffer(blob[off:off + 16 * nk], "<f8")
    s_ = np.frombuffer(blob[off + 16 * nk:off + 32 * nk], "<f8")
    lw = np.frombuffer(blob[off + 32 * nk:off + 40 * nk], "<f8")
    assert np.array_equal(c, st["centers"][:2 * nk])
    assert np.array_equal(s_, st["sigmas"][:2 * nk])
    assert np.array_equal(lw, st["logw"][:nk])


def test_opes_energy_vs_oracle():
    cvs, biases = opes_system(variant=0, pace=1, sigma=0.2)
    rng = np.random.default_rng(5)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    ctx, f = _gpu().make_context(np.zeros((4, 3)), cvs, biases)
    nc = ctx.glued_context_for(f)
    for step in range(30):
        pos = rng.uniform(0, 1.0, (4, 3))
        ctx.setStepCount(step)
        ctx.updateContextState()
        orc.update_state(step)
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        orc.cv_values = np.array(nc.cv_values())
        res = orc.evaluate_biases(orc.cv_values)
        orc.bias_energies = res[0]
        orc.cv_ready = True
        assert abs(e - res[0].sum()) < 1e-6 * max(1.0, abs(e))
    m = f.getOPESMetrics(ctx, 0)
    assert m[2] == orc.bias_state[0]["ist"][0]
    # zed, rct, nker, neff (CommonGluedKernels.cpp:5164-5210)
    np.testing.assert_allclose(m, orc.opes_metrics(0), rtol=1e-10, atol=1e-12)


def test_bias_state_round_trip():
    cvs, biases = opes_system(variant=0, pace=1, sigma=0.3)
    rng = np.random.default_rng(2)
    ctx, f = _gpu().make_context(np.zeros((4, 3)), cvs, biases)
    for step in range(20):
        ctx.setPositions(rng.uniform(0, 1, (4, 3)))
        ctx.setStepCount(step)
        ctx.updateContextState()
        ctx.computeForces()
    pos = rng.uniform(0, 1, (4, 3))
    ctx.setPositions(pos)
    e1, F1 = ctx.computeForces()
    blob = f.getBiasState()
    ctx2, f2 = _gpu().make_context(pos, cvs, biases)
    f2.setBiasState(blob)
    e2, F2 = ctx2.computeForces()
    assert e1 == e2 and np.array_equal(F1, F2)
    assert f2.getBiasState() == blob
    with pytest.raises(Exception):
        f2.setBiasState(blob[:-3])
