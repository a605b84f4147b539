"""Cutoff coordination on the device cell list (coord_cells.cu) against the FP64
oracle (no reference counterpart: the reference has no cutoff; the pair terms
are its CommonGluedKernels.cpp:969-1027).

* the pair list equals the oracle's bit for bit (sorted integer pairs; the
  oracle's decisions 1e-20 <= r^2 < rc^2 in FP64 from the FP32 positions) at the
  C2 cutoff workload (2,048 x 8,192 atoms, rc 1.2 nm, 5.9 nm box: 4 x 4 x 4
  cells) and in the edge cases: a box with fewer than three cells per side (one
  cell), a triclinic box and no periodicity (every B atom a candidate), atoms in
  both groups, positions outside the box, empty cells;
* CN, forces and energy of the C2 cutoff workload (5.9 nm box, and a 12 nm box
  at the same density: 8 x 8 x 8 cells) within the bench gates (forces 1e-4
  relative in max-norm, CV 1e-5, energy 1e-4), on the all-pairs tiles (the
  default) and on the cell list (params[4] = 1); the two agree to 5e-5 in
  forces (the tiles decide the cutoff in FP32 scaled units);
* an atom reorder leaves the cell-list forces bit-identical (candidate order is
  the B group order, not the GPU slot order).

The pair list (glued_context_coordination_pairs) comes from the cell-list
kernels whichever path evaluates the CV.
"""
import numpy as np
import pytest

import oracle as O
import parity as P

pytestmark = pytest.mark.gpu


def _ctx(pos, cvs, biases=(), box=None, pbc=True, reorder=None, blob=None):
    import gpu_util
    return gpu_util.make_context(pos, cvs, biases, pbc=pbc, box=box, reorder=reorder, blob=blob)


def _pairs_check(pos, A, B, box, rc, pbc=True, r0=0.35):
    pos32 = np.asarray(pos, np.float32).astype(np.float64)
    cvs = [(O.CV_COORDINATION_CUTOFF, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [r0, 6, 12, rc])]
    ctx, f = _ctx(pos32, cvs, box=box, pbc=pbc)
    ctx.computeForces()
    got = ctx.glued_context_for(f).coordination_pairs(0)
    box9 = np.asarray(box if box is not None else np.eye(3), float).ravel()
    ref = O.coordination_pair_list(pos32, A, B, box9, rc, periodic=pbc)
    assert got.shape == ref.shape, (got.shape, ref.shape)
    assert np.array_equal(got, ref)
    return ctx, f, len(ref)


def test_pair_list_c2_cutoff_bit_exact():
    from gluedmd_b200 import workloads as W
    w = W.config2_cutoff()
    n = _pairs_check(w.positions, w.extra["A"], w.extra["B"], w.box, 1.2)[2]
    assert n > 100000


@pytest.mark.parametrize("case", ["small_box", "triclinic", "nonperiodic", "overlap_outside_empty"])
def test_pair_list_edge_cases(case):
    rng = np.random.default_rng(5)
    if case == "small_box":
        L = 2.5   # floor(2.5 / 1.0) = 2 cells per side: one cell
        pos = rng.uniform(0, L, (600, 3))
        _pairs_check(pos, np.arange(100), np.arange(100, 600), np.eye(3) * L, 1.0)
    elif case == "triclinic":
        box = np.array([[4.0, 0, 0], [1.0, 4.0, 0], [-0.8, 0.7, 4.0]])
        pos = rng.uniform(0, 4.0, (900, 3))
        _pairs_check(pos, np.arange(200), np.arange(200, 900), box, 1.1)
    elif case == "nonperiodic":
        pos = rng.uniform(0, 3.0, (700, 3))
        _pairs_check(pos, np.arange(150), np.arange(150, 700), None, 0.9, pbc=False)
    else:
        # 8 x 8 x 8 cells of 0.75 nm (capped at 8 per side), the atoms in one corner
        # octant (most cells empty), some atoms in both groups, some far outside the box
        L = 6.0
        pos = rng.uniform(0, 2.0, (800, 3))
        pos[::7] += rng.integers(-3, 4, (len(pos[::7]), 3)) * L
        A = np.arange(0, 300)
        B = np.arange(250, 800)           # atoms 250..299 in both groups
        n = _pairs_check(pos, A, B, np.eye(3) * L, 0.6)[2]
        assert n > 0


def _gates(err, label):
    assert err["force"] < 1e-4, (label, err["force"])
    assert err["cv"] < 1e-5, (label, err["cv"])
    assert err["energy"] < 1e-4, (label, err["energy"])


@pytest.mark.parametrize("box", [5.9, 12.0])
def test_c2_cutoff_cells_and_tiles_vs_oracle(box):
    from gluedmd_b200 import workloads as W
    out = {}
    for method in (0, 1):
        w = W.config2_cutoff(method, box=box)
        ctx, f = _ctx(w.positions, w.cvs, w.biases, box=w.box, blob=w.blob)
        e, F = ctx.computeForces()
        cv = np.array(f.getLastCVValues(ctx))
        err = P.check_single(w, e, F, cv)
        _gates(err, w.name)
        out[method] = (F, cv)
    F0, F1 = out[0][0], out[1][0]
    assert np.abs(F0 - F1).max() <= 5e-5 * np.abs(F1).max()
    assert abs(out[0][1][0] - out[1][1][0]) <= 1e-6 * abs(out[1][1][0])


def test_cells_forces_bit_identical_after_reorder():
    rng = np.random.default_rng(8)
    L = 5.0
    pos = rng.uniform(0, L, (3000, 3))
    A, B = np.arange(500), np.arange(500, 3000)
    cvs = [(O.CV_COORDINATION_CUTOFF, [len(A)] + list(A) + list(B), [0.35, 6, 12, 1.1, 1.0])]
    import gpu_util
    res = []
    for reorder in (None, rng.permutation(3000)):
        ctx, f = gpu_util.make_context(pos, cvs, pbc=True, box=np.eye(3) * L, reorder=reorder, grad=[1.0])
        e, F = ctx.computeForces()
        res.append((F, f.getLastCVValues(ctx)[0]))
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]
