"""gluedmd_b200.merger pinned to the reference's own BiasStateMerger
(python/MultiGPUManager.py:132-716) on blobs this library wrote.

Fixtures (tests/golden/make_merger_fixtures.py): three walker groups per
scenario, each a context of this library on a B200, 30 steps of deposits
(round 1), merged, loaded back, 30 more steps (round 2); the reference merger's
outputs on those blobs (first sync, then incremental with its own baselines)
were recorded by importing the reference module unchanged.

The reference packer ends after the MaxEnt section; this library's serializer
also writes the OPES multithermal count (CommonSerialization.cpp:164-176; 0
here), so every merged blob of this library is the reference's followed by
four zero bytes. Everything else is equal byte for byte.

2-D MetaD: the reference helper reads grid sizes from an interleaved
[pace, bins_0, periodic_0, ...] layout, while the bias setup writes
[pace, bins_0, bins_1, periodic_0, periodic_1] (CommonBiasKernels.cpp:206-257);
on a 64 x 64 grid it reads 64 points and fails further on. The recorded
ValueError documents that; this library sums the full grids.
"""
import os
import struct
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_merger_fixtures as FX  # noqa: E402
from gluedmd_b200.merger import BiasStateMerger as M  # noqa: E402

BLOBS = FX.load_blobs()
EXPECTED = FX.load_expected()
AGREE = [n for n in BLOBS if n != "metad2d"]
TAIL = struct.pack("<i", 0)   # OPES multithermal count


def _ours(name):
    biases, r1, r2 = BLOBS[name]
    f = FX.SpecForce(biases)
    m1, base = M.merge_additive_incremental(r1, f, None)
    m2, _ = M.merge_additive_incremental(r2, f, base)
    return f, m1, m2


def test_fixture_blobs_repack_unchanged():
    for name, (biases, r1, r2) in BLOBS.items():
        f = FX.SpecForce(biases)
        for b in r1 + r2:
            assert M._pack(M._parse(b, f)) == b, name


@pytest.mark.parametrize("name", AGREE)
def test_merge_equals_reference_byte_for_byte(name):
    _, m1, m2 = _ours(name)
    e = EXPECTED[name]
    assert not e["r1_error"] and not e["r2_error"]
    assert m1 == e["r1"] + TAIL
    assert m2 == e["r2"] + TAIL


@pytest.mark.parametrize("name", AGREE)
def test_merged_state_is_nontrivial(name):
    """The fixtures exercise real merges: deposits in every group, and for OPES
    the Chan combination of adaptive-sigma statistics."""
    f, m1, m2 = _ours(name)
    p1, p2 = M._parse(m1, f), M._parse(m2, f)
    for nd, g in p1["metad"]:
        assert nd > 0 and np.abs(np.frombuffer(g, "<f8")).max() > 0
    for subs in p1["pbmetad"]:
        assert all(nd > 0 for nd, _ in subs)
    for o1, o2 in zip(p1["opes"], p2["opes"]):
        assert o1[0] > 0 and o2[0] > o1[0] and o2[2] > o1[2] > 0
        assert np.all(np.frombuffer(o2[4], "<f8") > 0)


def test_two_dimensional_metad_disagreement_is_documented():
    """The reference helper cannot parse a 2-D MetaD blob of the bias setup's
    parameter layout (it raised on the fixtures); this library merges it: the
    merged grid is the sum of the three groups' grids, deposit counts summed."""
    e = EXPECTED["metad2d"]
    assert e["r1_error"] and e["r1"].startswith("ValueError")
    biases, r1, _ = BLOBS["metad2d"]
    f = FX.SpecForce(biases)
    merged = M.merge_additive(r1, f)
    nd, g = M._parse(merged, f)["metad"][0]
    parts = [M._parse(b, f)["metad"][0] for b in r1]
    assert len(g) == 8 * 64 * 64
    assert nd == sum(p[0] for p in parts)
    np.testing.assert_array_equal(np.frombuffer(g, "<f8"), sum(np.frombuffer(p[1], "<f8") for p in parts))


# ------------------------------------------------- live, with the reference tree
REF = os.environ.get("GLUED_REFERENCE", "")
needs_ref = pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "python", "MultiGPUManager.py"))),
                               reason="GLUED_REFERENCE not set to a reference tree")


@needs_ref
@pytest.mark.parametrize("name", list(BLOBS))
def test_reference_merger_live(name):
    """The reference module itself, run here on the fixture blobs: it reproduces
    the recorded outputs, its parser reads this library's blobs into the same
    sections as this library's parser, and its merges equal this library's."""
    mod = FX.import_reference_merger(REF)
    biases, r1, r2 = BLOBS[name]
    got = FX.run_reference(mod, biases, r1, r2)
    e = EXPECTED[name]
    for k in ("r1", "r2"):
        assert got[k][1] == e[k + "_error"] and got[k][0] == e[k], (name, k)
    if name in AGREE:
        f = FX.SpecForce(biases)
        for b in r1 + r2:
            pr, po = mod.BiasStateMerger._parse(b, f), M._parse(b, f)
            for key, v in pr.items():
                assert po[key] == v, (name, key)
        _, m1, m2 = _ours(name)
        assert (m1, m2) == (got["r1"][0] + TAIL, got["r2"][0] + TAIL)
