"""Bias-state blob parse / repack / merge (gluedmd_b200.merger) and the cross-rank
sync built on it, on CPU. The first four tests restate the reference's own merger
tests (tests/test_multi_gpu.py:458-570)."""
import math
import os
import socket
import struct

import numpy as np
import pytest
import torch.multiprocessing as mp

from gluedmd_b200.merger import BiasStateMerger as M


class FakeForce:
    """Stand-in for GluedForce: getNumBiases / getBiasParameters only."""

    def __init__(self, biases):
        self.biases = biases

    def getNumBiases(self):
        return len(self.biases)

    def getBiasParameters(self, i):
        return self.biases[i]


META1 = FakeForce([(3, [0], [], [10, 5, 0])])   # 1-D MetaD, 5 bins, not periodic: 6 points


def _metad_blob(grid, nd=5):
    b = bytearray(b"GPUS") + struct.pack("<iiii", 1, 0, 0, 1) + struct.pack("<i", nd)
    b += np.asarray(grid, "<f8").tobytes()
    b += struct.pack("<8i", 0, 0, 0, 0, 0, 0, 0, 0)  # PBMetaD .. MaxEnt
    return bytes(b)


def test_merge_additive_two_blobs():
    a, b = [1.0, 2, 3, 4, 5, 6], [0.5] * 6
    merged = M.merge_additive([_metad_blob(a, 10), _metad_blob(b, 5)], META1)
    nd, g = M._parse(merged, META1)["metad"][0]
    assert nd == 15
    np.testing.assert_array_equal(np.frombuffer(g, "<f8"), np.add(a, b))


def test_merge_single_blob_unchanged():
    blob = _metad_blob([1.0, 2, 3, 4, 5, 6])
    assert M.merge_additive([blob], META1) == blob


def test_merge_three_blobs():
    merged = M.merge_additive([_metad_blob([float(k)] * 6, 10) for k in (1, 2, 3)], META1)
    nd, g = M._parse(merged, META1)["metad"][0]
    assert nd == 30 and np.array_equal(np.frombuffer(g, "<f8"), np.full(6, 6.0))


def test_repack_round_trip_reference_blob():
    blob = _metad_blob([0.1 * i for i in range(6)], 7)
    p = M._parse(blob, META1)
    p2 = M._parse(M._pack(p), META1)
    assert p["metad"] == p2["metad"]


# ------------------------------------------------------------ every section
ALL = FakeForce([
    (5, [0, 1], [], [0, 10, 1000]),                 # OPES, D=2
    (7, [0], [], []),                               # ABMD, D=1
    (3, [0, 1], [], [10, 8, 12, 1, 0]),             # MetaD 8 (periodic) x 13
    (4, [0, 1], [], [10, 20, 0, 30, 1]),            # PBMetaD sub-grids 21, 30
    (6, [1], [], [40, 0]),                          # EXTERNAL
    (11, [0], [], []),                              # OPES_EXPANDED
    (12, [0, 1], [], []),                           # extended Lagrangian, D=2
    (14, [0, 1], [], []),                           # EDS, D=2
    (13, [1], [], []),                              # MaxEnt, D=1
    (15, [0], [], []),                              # OPES multithermal
    (103, [0, 1], [], [5, 100, 0, 0]),              # hill-sum MetaD, D=2
])


def _full_state(rng, nk=3, nh=4, ns=25):
    f = lambda n: rng.normal(size=n).astype("<f8").tobytes()  # noqa: E731
    return dict(
        opes=[(nk, 1.5, ns, f(2), np.abs(rng.normal(size=2)).tobytes(), f(2 * nk), f(2 * nk), f(nk))],
        abmd=[f(1)],
        metad=[(4, f(8 * 13))],
        pbmetad=[[(3, f(21)), (3, f(30))]],
        n_external=1, n_linear=0, n_wall=0,
        opes_expanded=[(0.25, 7)],
        ext_lag=[(f(2), f(2))],
        eds=[(f(2), f(2), f(2), f(2), np.arange(2, dtype="<i4").tobytes())],
        maxent=[f(1)],
        multithermal=[(3, f(3), f(1), f(1))],
        hills=[(2, nh, f(2 * nh), f(nh))],
    )


def test_every_section_round_trips_byte_exact():
    d = _full_state(np.random.default_rng(0))
    blob = M._pack(d)
    p = M._parse(blob, ALL)
    assert p == d
    assert M._pack(p) == blob


def test_metad_grid_size_follows_setup_layout():
    """[pace, bins_0, bins_1, periodic_0, periodic_1]: 8 periodic x 12 + 1 points."""
    d = _full_state(np.random.default_rng(1))
    p = M._parse(M._pack(d), ALL)
    assert len(p["metad"][0][1]) == 8 * 8 * 13


def test_count_mismatch_and_truncation_raise():
    blob = M._pack(_full_state(np.random.default_rng(2)))
    with pytest.raises(ValueError, match="truncated"):
        M._parse(blob[:-5], ALL)
    with pytest.raises(ValueError, match="MetaD count mismatch"):
        M._parse(_metad_blob([0.0] * 6), FakeForce([(3, [0], [], [10, 5, 0])] * 2))


def test_opes_union_merge_matches_pooled_statistics():
    """Chan's combination of the Welford accumulators equals the mean and M2 of the
    pooled samples; kernels are concatenated; logZ = log sum exp(logW)."""
    rng = np.random.default_rng(3)
    force = FakeForce([(5, [0, 1], [], [0, 10, 1000])])
    samples, blobs, lws = [], [], []
    for n, nk in ((40, 3), (65, 5), (1, 1)):
        x = rng.normal(size=(n, 2)) * [1.0, 3.0] + rng.normal(size=2)
        samples.append(x)
        mean = x.mean(0)
        m2 = ((x - mean) ** 2).sum(0)
        lw = rng.normal(size=nk)
        lws.append(lw)
        d = dict(opes=[(nk, 0.0, n, mean.tobytes(), m2.tobytes(), rng.normal(size=2 * nk).tobytes(),
                        rng.normal(size=2 * nk).tobytes(), lw.tobytes())],
                 abmd=[], metad=[], pbmetad=[], opes_expanded=[], ext_lag=[], eds=[], maxent=[])
        blobs.append(M._pack(d))
    nk, logz, ns, mb, m2b, cb, sb, lb = M._parse(M.merge_additive(blobs, force), force)["opes"][0]
    pooled = np.concatenate(samples)
    assert nk == 9 and ns == len(pooled)
    np.testing.assert_allclose(np.frombuffer(mb, "<f8"), pooled.mean(0), rtol=1e-12)
    np.testing.assert_allclose(np.frombuffer(m2b, "<f8"), ((pooled - pooled.mean(0)) ** 2).sum(0), rtol=1e-11)
    allw = np.concatenate(lws)
    assert abs(logz - math.log(np.exp(allw).sum())) < 1e-12
    assert np.array_equal(np.frombuffer(lb, "<f8"), allw)
    assert cb == b"".join(M._parse(b, force)["opes"][0][5] for b in blobs)


def test_incremental_merge_folds_only_deltas():
    """Second sync: shared + sum over groups of (now - baseline); grids, deposit
    counts and hill tables."""
    force = FakeForce([(3, [0], [], [10, 5, 0]), (4, [0], [], [10, 4, 1]), (103, [0], [], [5, 100, 0])])
    rng = np.random.default_rng(4)

    def state(g, pb, nd, hills):
        return M._pack(dict(opes=[], abmd=[], metad=[(nd, np.asarray(g, "<f8").tobytes())],
                            pbmetad=[[(nd, np.asarray(pb, "<f8").tobytes())]], opes_expanded=[], ext_lag=[], eds=[],
                            maxent=[], hills=[(1, len(hills), np.asarray(hills, "<f8").tobytes(),
                                               np.ones(len(hills), "<f8").tobytes())]))

    g0, g1 = rng.uniform(size=6), rng.uniform(size=6)
    p0, p1 = rng.uniform(size=4), rng.uniform(size=4)
    m1, base = M.merge_additive_incremental([state(g0, p0, 2, [0.1]), state(g1, p1, 3, [0.2, 0.3])], force)
    s1 = M._parse(m1, force)
    shared = np.frombuffer(s1["metad"][0][1], "<f8")
    np.testing.assert_array_equal(shared, g0 + g1)
    assert s1["metad"][0][0] == 5 and s1["hills"][0][1] == 3
    # both groups continue from the shared state and deposit more
    d0, d1 = rng.uniform(size=6), rng.uniform(size=6)
    hs = list(np.frombuffer(s1["hills"][0][2], "<f8"))
    b0 = state(shared + d0, np.frombuffer(s1["pbmetad"][0][0][1], "<f8") + 1.0, 6, hs + [0.4])
    b1 = state(shared + d1, np.frombuffer(s1["pbmetad"][0][0][1], "<f8") + 2.0, 7, hs + [0.5, 0.6])
    m2, _ = M.merge_additive_incremental([b0, b1], force, baselines=base)
    s2 = M._parse(m2, force)
    np.testing.assert_allclose(np.frombuffer(s2["metad"][0][1], "<f8"), shared + d0 + d1, rtol=1e-13)
    np.testing.assert_allclose(np.frombuffer(s2["pbmetad"][0][0][1], "<f8"), p0 + p1 + 3.0, rtol=1e-13)
    assert s2["metad"][0][0] == 5 + 1 + 2
    c = np.frombuffer(s2["hills"][0][2], "<f8")
    assert s2["hills"][0][1] == 6 and list(c) == [0.1, 0.2, 0.3, 0.4, 0.5, 0.6]


# ------------------------------------------------------------ 2-rank sync
def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _sync_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from gluedmd_b200 import dist as D
    dist = D.init("gloo", timeout_s=60)
    g = np.arange(6, dtype=float) * (rank + 1)
    merged, base = D.sync_bias_state(_metad_blob(g, 10 + rank), META1)
    shared = np.frombuffer(M._parse(merged, META1)["metad"][0][1], "<f8")
    merged2, _ = D.sync_bias_state(_metad_blob(shared + rank + 1.0, 20), META1, base)
    dist.barrier()
    q.put((rank, merged, merged2))
    dist.destroy_process_group()


def test_two_rank_gloo_bias_sync():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sync_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]   # identical on every rank
    nd, g = M._parse(out[0][1], META1)["metad"][0]
    assert nd == 21 and np.array_equal(np.frombuffer(g, "<f8"), np.arange(6) * 3.0)
    nd2, g2 = M._parse(out[0][2], META1)["metad"][0]
    # deltas since the shared state: +1 on rank 0, +2 on rank 1; counts 20 - 21 each
    assert nd2 == 21 + (20 - 21) * 2
    np.testing.assert_array_equal(np.frombuffer(g2, "<f8"), np.arange(6) * 3.0 + 3.0)


def test_workload_blob_round_trips_through_merger():
    """The C1-pbmetad bench workload's bias state (written by the workload
    builder): the merger parses it against the workload's biases, repacks it byte
    for byte, and the oracle reads the same sub-grids from it."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import oracle as O
    from gluedmd_b200 import workloads as W
    w = W.config1("pbmetad")
    force = FakeForce([(t, c, p, ip) for t, c, p, ip in w.biases])
    parsed = M._parse(w.blob, force)
    assert M._pack(parsed) == w.blob
    assert parsed["n_external"] == 1 and len(parsed["pbmetad"]) == 1 and len(parsed["pbmetad"][0]) == 2
    s = O.OracleSystem(w.cvs, w.biases, masses=w.masses, periodic=True, mode="f64", num_particles=len(w.positions))
    s.load_blob(w.blob)
    st = [b for b in s.bias_state if b["type"] == O.BIAS_PBMETAD][0]
    grids = np.concatenate([np.frombuffer(g, "<f8") for _, g in parsed["pbmetad"][0]])
    assert np.array_equal(st["grid"], grids)
    assert st["deposited"] == [nd for nd, _ in parsed["pbmetad"][0]]
