"""PBMETAD and EXTERNAL biases on the sm_100a path vs the FP64 oracle.

Tolerances: energies 1e-5 relative (FP32 CV values feed FP64 bias arithmetic);
forces 1e-4 relative in max-norm; grids after deposits 1e-5 relative (deposit
centres are the FP32-derived CV values); deposit counts and blob layout exact."""
import math
import struct

import numpy as np
import pytest

import oracle as O
from test_oracle_pbmetad import (DIST01, KT, _pb, _ext, _pos, gaussian_grid_1d, pbmetad_system,
                                 external_system)

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4


def _gpu():
    import gpu_util
    return gpu_util


def _pb_grid_from_blob(blob, cvs, biases, n):
    """Sub-grids and deposit counts of the first PBMETAD bias, read by the oracle's
    blob reader."""
    s = O.OracleSystem(cvs, biases, mode="f64", num_particles=n)
    s.load_blob(blob)
    st = [b for b in s.bias_state if b["type"] == O.BIAS_PBMETAD][0]
    return st["grid"], st["deposited"]


def test_pbmetad_replay_vs_oracle():
    """40 steps of pace-2 WT deposits on three sub-grids (two periodic): energies
    and forces every step, then the grids and deposit counts from the blob."""
    cvs, biases = pbmetad_system(pace=2, gamma=10.0)
    rng = np.random.default_rng(11)
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
        assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"])), (step, e, r["energy"])
        assert O.max_rel_force_err(F, r["forces"]) < FORCE_TOL, step
    g, nd = _pb_grid_from_blob(f.getBiasState(), cvs, biases, 6)
    st = orc.bias_state[0]
    assert nd == st["deposited"] == [19, 19, 19]
    np.testing.assert_allclose(g, st["grid"], rtol=1e-5, atol=1e-7 * np.abs(st["grid"]).max())


def test_pbmetad_known_answers_gpu():
    """The reference's PBMETAD acceptance cases on the product: zero before a
    deposit, h0 at the deposit point, FD force at a bin midpoint."""
    ctx, f = _gpu().make_context(_pos(1.0), DIST01, [_pb(1.2, 10.0, [(0.1, 0.0, 2.0, 100, 0)])])
    e, F = ctx.computeForces()
    assert e == 0.0 and np.all(F == 0.0)
    bias = [_pb(2.0, 1.0, [(0.2, 0.0, 2.0, 200, 0)], pace=1)]
    ctx, f = _gpu().make_context(_pos(1.0), DIST01, bias)
    ctx.computeForces()
    for step in (0, 1):
        ctx.setStepCount(step)
        ctx.updateContextState()
    e, _ = ctx.computeForces()
    assert abs(e - 2.0) < 1e-5
    bias = [_pb(2.0, 1.0, [(0.3, 0.0, 3.0, 300, 0)], pace=1)]
    ctx, f = _gpu().make_context(_pos(1.5), DIST01, bias)
    ctx.computeForces()
    for step in (0, 1):
        ctx.setStepCount(step)
        ctx.updateContextState()
    x, dx = 1.005, 0.005
    ctx.setPositions(_pos(x + dx)); ep, _ = ctx.computeForces()
    ctx.setPositions(_pos(x - dx)); em, _ = ctx.computeForces()
    ctx.setPositions(_pos(x)); _, F = ctx.computeForces()
    fnum = -(ep - em) / (2 * dx)
    assert abs(fnum) > 1e-3 and abs(F[1, 0] - fnum) < 5e-3


def test_pbmetad_restart_round_trip():
    """Blob of the product restores into a fresh context (same energy and forces,
    identical blob) and into the oracle (same energy)."""
    cvs, biases = pbmetad_system(pace=1, gamma=10.0)
    rng = np.random.default_rng(4)
    ctx, f = _gpu().make_context(np.zeros((6, 3)), cvs, biases)
    for step in range(12):
        ctx.setPositions(rng.uniform(0, 1.5, (6, 3)))
        ctx.setStepCount(step)
        ctx.updateContextState()
        ctx.computeForces()
    pos = rng.uniform(0, 1.5, (6, 3))
    ctx.setPositions(pos)
    e1, F1 = ctx.computeForces()
    blob = f.getBiasState()
    # PBMETAD section right after the empty OPES, ABMD and MetaD sections
    assert struct.unpack_from("<iiiiii", blob, 4) == (1, 0, 0, 0, 1, 3)
    ctx2, f2 = _gpu().make_context(pos, cvs, biases)
    f2.setBiasState(blob)
    e2, F2 = ctx2.computeForces()
    assert e1 == e2 and np.array_equal(F1, F2)
    assert f2.getBiasState() == blob
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    orc.load_blob(blob)
    r = orc.execute(pos)
    assert abs(e1 - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"]))
    with pytest.raises(Exception):
        f2.setBiasState(blob[:-3])


def test_external_vs_oracle():
    cvs, biases = external_system()
    rng = np.random.default_rng(5)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    ctx, f = _gpu().make_context(np.zeros((6, 3)), cvs, biases)
    for _ in range(10):
        pos = rng.uniform(0, 1.5, (6, 3))
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        r = orc.execute(pos)
        assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"]))
        assert O.max_rel_force_err(F, r["forces"]) < FORCE_TOL
    ctx.setStepCount(5)
    ctx.updateContextState()   # no deposition for a fixed grid
    blob = f.getBiasState()
    ctx.setPositions(pos)
    e2, _ = ctx.computeForces()
    assert e2 == e and f.getBiasState() == blob


def test_external_matches_metad_after_deposit_gpu():
    ctx, f = _gpu().make_context(_pos(1.0), DIST01, [(O.BIAS_METAD, [0], [2.0, 0.2, 1.0, KT, 0.0, 2.0], [1, 200, 0])])
    ctx.computeForces()
    for step in (0, 1):
        ctx.setStepCount(step)
        ctx.updateContextState()
    ctx.setPositions(_pos(0.8))
    em, Fm = ctx.computeForces()
    g = gaussian_grid_1d(2.0, 1.0, 0.2, 0.0, 2.0, 200)
    ctx2, _ = _gpu().make_context(_pos(0.8), DIST01, [_ext([0], [0.0], [2.0], [200], [0], g)])
    ee, Fe = ctx2.computeForces()
    assert abs(ee - em) < 2e-3 and em > 0.1
    assert O.max_rel_force_err(Fe, Fm) < 1e-3


def test_mixed_bias_types_vs_oracle():
    """HARMONIC, OPES, METAD, PBMETAD and EXTERNAL in one force, with deposits:
    the product's evaluation order and per-type deposition against the oracle."""
    cvs = [(O.CV_DIHEDRAL, [0, 1, 2, 3], []), (O.CV_DIHEDRAL, [1, 2, 3, 4], []), (O.CV_DISTANCE, [0, 5], [])]
    rng = np.random.default_rng(9)
    ext_grid = rng.uniform(0.0, 3.0, 101)
    biases = [
        (O.BIAS_EXTERNAL, [2], [0.0, 2.5] + list(ext_grid), [100, 0]),
        (O.BIAS_PBMETAD, [0, 1], [1.0, 8.0, KT, 0.35, -math.pi, math.pi, 0.35, -math.pi, math.pi], [3, 64, 1, 64, 1]),
        (O.BIAS_HARMONIC, [2], [50.0, 1.1], [0]),
        (O.BIAS_METAD, [0, 1], [1.2, 0.35, 0.35, 10.0, 2.494338785, -math.pi, -math.pi, math.pi, math.pi],
         [2, 64, 64, 1, 1]),
        (O.BIAS_OPES, [2], [2.494338785, 20.05, 0.05, 0.02], [0, 4, 1000]),
    ]
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    ctx, f = _gpu().make_context(np.zeros((6, 3)), cvs, biases)
    for step in range(30):
        pos = rng.uniform(0, 1.5, (6, 3))
        ctx.setPositions(pos)
        ctx.setStepCount(step)
        ctx.updateContextState()
        orc.update_state(step)
        e, F = ctx.computeForces()
        r = orc.execute(pos)
        assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"])), (step, e, r["energy"])
        assert O.max_rel_force_err(F, r["forces"]) < FORCE_TOL, step
    g, nd = _pb_grid_from_blob(f.getBiasState(), cvs, biases, 6)
    assert nd == orc.bias_state[1]["deposited"] == [9, 9]


def test_c1_pbmetad_workload_vs_oracle():
    """The bench's C1-pbmetad workload (PBMETAD sub-grids loaded from a blob, a
    256x256 EXTERNAL grid) at its positions and four perturbations of them."""
    from gluedmd_b200 import workloads as W
    w = W.config1("pbmetad")
    n = len(w.positions)
    orc = O.OracleSystem(w.cvs, w.biases, masses=w.masses, periodic=True, mode="f64", num_particles=n)
    orc.load_blob(w.blob)
    ctx, f = _gpu().make_context(w.positions, w.cvs, w.biases, masses=w.masses, pbc=True, box=w.box, blob=w.blob)
    rng = np.random.default_rng(6)
    for k in range(5):
        pos = w.positions + (0 if k == 0 else rng.normal(scale=0.05, size=w.positions.shape))
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        r = orc.execute(pos, np.asarray(w.box).ravel())
        assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"])), (k, e, r["energy"])
        assert O.max_rel_force_err(F, r["forces"]) < FORCE_TOL, k
