"""Merging the bias states of two walker groups evaluated on the sm_100a path.

Two contexts with the same force (2-D MetaD grid, PBMETAD, OPES, hill-sum MetaD)
deposit along different trajectories; their blobs are merged on the host and the
merged state is loaded into a third context. Checks: the third context writes
the merged blob back byte for byte; grids are the exact sums and OPES kernels
and hills the unions; energy and forces equal the FP64 oracle loaded with the
same merged blob (energy 1e-5 relative, forces 1e-4 relative max-norm)."""
import math

import numpy as np
import pytest

import oracle as O
from gluedmd_b200.merger import BiasStateMerger as M

pytestmark = pytest.mark.gpu

KT = 2.494338785
CVS = [(O.CV_DIHEDRAL, [0, 1, 2, 3], []), (O.CV_DIHEDRAL, [1, 2, 3, 4], []), (O.CV_DISTANCE, [0, 5], [])]
BIASES = [
    (O.BIAS_METAD, [0, 1], [1.2, 0.35, 0.35, 10.0, KT, -math.pi, -math.pi, math.pi, math.pi], [2, 48, 48, 1, 1]),
    (O.BIAS_PBMETAD, [0, 2], [1.0, 8.0, KT, 0.35, -math.pi, math.pi, 0.1, 0.0, 2.5], [3, 64, 1, 100, 0]),
    (O.BIAS_OPES, [2], [KT, 20.05, 0.05, 0.02], [0, 4, 1000]),
    (O.BIAS_METAD_HILLS, [1], [0.8, 0.3, 10.0, KT, -math.pi, math.pi], [2, 500, 1]),
]


def _group(seed, steps=24):
    import gpu_util
    rng = np.random.default_rng(seed)
    ctx, f = gpu_util.make_context(np.zeros((6, 3)), CVS, BIASES)
    for step in range(steps):
        ctx.setPositions(rng.uniform(0, 1.5, (6, 3)))
        ctx.setStepCount(step)
        ctx.updateContextState()
        ctx.computeForces()
    return ctx, f


def test_two_groups_merge_and_restore():
    import gpu_util
    (_, fa), (_, fb) = _group(1), _group(2)
    ba, bb = bytes(fa.getBiasState()), bytes(fb.getBiasState())
    pa, pb = M._parse(ba, fa), M._parse(bb, fa)
    assert M._pack(pa) == ba and M._pack(pb) == bb          # product blobs round-trip byte for byte
    merged = M.merge_additive([ba, bb], fa)
    pm = M._parse(merged, fa)
    ga, gb = (np.frombuffer(p["metad"][0][1], "<f8") for p in (pa, pb))
    assert np.array_equal(np.frombuffer(pm["metad"][0][1], "<f8"), ga + gb)
    assert pm["metad"][0][0] == pa["metad"][0][0] + pb["metad"][0][0] == 22
    for si in range(2):
        s = [np.frombuffer(p["pbmetad"][0][si][1], "<f8") for p in (pa, pb)]
        assert np.array_equal(np.frombuffer(pm["pbmetad"][0][si][1], "<f8"), s[0] + s[1])
    assert pm["opes"][0][0] == pa["opes"][0][0] + pb["opes"][0][0]
    assert pm["hills"][0][1] == pa["hills"][0][1] + pb["hills"][0][1] == 22

    pos = np.random.default_rng(9).uniform(0, 1.5, (6, 3))
    ctx, fc = gpu_util.make_context(pos, CVS, BIASES)
    fc.setBiasState(merged)
    assert bytes(fc.getBiasState()) == merged
    e, F = ctx.computeForces()
    orc = O.OracleSystem(CVS, BIASES, mode="f64", num_particles=6)
    orc.load_blob(merged)
    r = orc.execute(pos)
    assert abs(e - r["energy"]) < 1e-5 * max(1.0, abs(r["energy"])), (e, r["energy"])
    assert O.max_rel_force_err(F, r["forces"]) < 1e-4
