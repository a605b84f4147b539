"""Batched multi-walker path vs the FP64 oracle evaluated walker by walker.

Gate: forces within 1e-4 relative (max-norm) of the FP64 oracle per walker, CV
values within 1e-5 relative, energies within 1e-4 relative; deposition centres
bit-exact (they are the walkers' CV values), heights to 1e-13 relative."""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _walkers(n_walkers=6, n_hills=3000, coord=(64, 256), seed=8):
    from gluedmd_b200 import workloads as W
    ws, hill = W.config4_walkers(n_walkers=n_walkers, n_hills=n_hills, coord=coord)
    return ws, hill


def _setup(ws, hill, with_hills=True, coord_restraint=True):
    import torch
    from gluedmd_b200.batch import Batch, Walker, force_for, c4_biases
    from gluedmd_b200 import workloads as W
    forces, walkers, specs = [], [], []
    for w in ws:
        cn0 = W.coordination_cn_fp64(w["pos"], w["A"], w["B"], w["L"]) if coord_restraint else None
        # restraint centres away from the current values, so that dU/dCV is not a
        # difference of nearly equal numbers (forces would be pure rounding noise);
        # the coordination centre 1% + 2 away, so that the CN error of FP32 pair
        # sums (~1e-8 relative for a CN of ~1e4) is not amplified by k / (CN - CN0)
        wr = dict(w, d0=w["d0"] + 0.05)
        biases = c4_biases(wr, hill["params"], hill["iparams"], cn0=None if cn0 is None else cn0 * 1.01 + 2.0)
        if not with_hills:
            biases = [b for b in biases if b[0] != 103]
        forces.append(force_for(w["cvs"], biases))
        walkers.append(Walker(w["pos"], w["box"]))
        specs.append(biases)
    b = Batch(forces, walkers)
    if with_hills:
        b.set_hills(hill["centers"], hill["heights"])
    return b, walkers, specs


def _oracle(w, biases, hill):
    s = O.OracleSystem(w["cvs"], biases, masses=w["masses"], periodic=True, mode="f64", num_particles=w["n"])
    for st in s.bias_state:
        if st["type"] == O.BIAS_METAD_HILLS:
            st["centers"] = np.array(hill["centers"], float)
            st["heights"] = np.array(hill["heights"], float)
    return s


@pytest.mark.parametrize("coord,parts,plain", [((64, 256), 0, 0), ((64, 256), 2, 0), ((64, 256), 5, 1),
                                                ((900, 1500), 0, 0)])
@pytest.mark.parametrize("with_hills", [False, True])
def test_batch_matches_fp64_oracle(with_hills, coord, parts, plain):
    """The batched step against the FP64 oracle: full coordination tiles with
    the fewest finalize parts per walker (one CTA for the walker and its 320
    rows, programmatic dependent launch), with a walker part and one row part,
    and with more parts than the rows need (plain launch); ragged tiles
    (partial A tiles and B chunks, 2,400 rows per walker: five row parts and
    the walker part)."""
    ws, hill = _walkers(coord=coord)
    b, walkers, specs = _setup(ws, hill, with_hills)
    b.set_tuning(8, parts, plain)
    rows = sum(coord)
    fewest = 1 if rows <= 512 else -(-rows // 512) + 1
    assert b.tuning["parts"] == max(parts, fewest)
    for wk in walkers:
        wk.force.zero_()
    b.execute()
    E = b.energies()
    cv = b.cv_values()
    assert b.status() == 0
    for i, w in enumerate(ws):
        r = _oracle(w, specs[i], hill).execute(w["pos"], w["box"].ravel())
        np.testing.assert_allclose(cv[i], r["cv_values"], rtol=1e-5, atol=1e-5)
        # energies carry restraint-amplified FP32 CV error: k * (s - s0) * dCV
        assert abs(E[i] - r["energy"]) <= 1e-4 * max(1.0, abs(r["energy"])), (i, E[i], r["energy"])
        err = O.max_rel_force_err(walkers[i].forces(), r["forces"])
        assert err < 1e-4, (i, err)


@pytest.mark.parametrize("group2,parts", [((32, 128), 0), ((32, 128), 3), ((96, 400), 0), ((96, 400), 5)])
def test_batch_two_coordination_items(group2, parts):
    """Two coordination CVs per walker, both restrained: the finalize's rows run
    over both items (item 0's A and B rows, then item 1's) and split across the
    row CTAs at arbitrary row boundaries. 480 rows fit one CTA (the fewest parts:
    one CTA completes the walker and takes every row; 3 parts: the walker CTA
    and two row CTAs); 816 rows need two row CTAs and the walker CTA (the
    fewest), or four."""
    import torch
    from gluedmd_b200.batch import Batch, Walker, force_for, c4_biases
    from gluedmd_b200 import workloads as W
    ws, hill = _walkers(n_walkers=4, coord=(64, 256))
    nA2, nB2 = group2
    forces, walkers, specs = [], [], []
    for i, w in enumerate(ws):
        rng = np.random.default_rng(77 + i)
        A2 = rng.choice(w["n"], nA2, replace=False)
        B2 = rng.choice(w["n"], nB2, replace=False)
        w["cvs"] = list(w["cvs"]) + [(W.CV_COORDINATION, [nA2] + [int(x) for x in A2] + [int(x) for x in B2],
                                      [0.35, 6, 12])]
        cn1 = W.coordination_cn_fp64(w["pos"], w["A"], w["B"], w["L"])
        cn2 = W.coordination_cn_fp64(w["pos"], A2, B2, w["L"])
        biases = c4_biases(dict(w, d0=w["d0"] + 0.05), hill["params"], hill["iparams"], cn0=cn1 * 1.01 + 2.0)
        biases.append((1, [4], [100.0, cn2 * 1.01 + 2.0], [0]))
        forces.append(force_for(w["cvs"], biases))
        walkers.append(Walker(w["pos"], w["box"]))
        specs.append(biases)
    b = Batch(forces, walkers)
    b.set_hills(hill["centers"], hill["heights"])
    b.set_tuning(8, parts, 0)
    rows = 64 + 256 + nA2 + nB2
    fewest = 1 if rows <= 512 else -(-rows // 512) + 1
    assert b.tuning["parts"] == max(parts, fewest)
    for wk in walkers:
        wk.force.zero_()
    b.execute()
    E = b.energies()
    cv = b.cv_values()
    assert b.status() == 0
    for i, w in enumerate(ws):
        r = _oracle(w, specs[i], hill).execute(w["pos"], w["box"].ravel())
        np.testing.assert_allclose(cv[i], r["cv_values"], rtol=1e-5, atol=1e-5)
        assert abs(E[i] - r["energy"]) <= 1e-4 * max(1.0, abs(r["energy"])), (i, E[i], r["energy"])
        err = O.max_rel_force_err(walkers[i].forces(), r["forces"])
        assert err < 1e-4, (i, err)


def test_batch_repeatable_and_autotuned():
    ws, hill = _walkers(n_walkers=5)
    b, walkers, specs = _setup(ws, hill, True)
    for wk in walkers:
        wk.force.zero_()
    b.execute()
    f1 = [w.forces() for w in walkers]
    for wk in walkers:
        wk.force.zero_()
    b.execute()
    f2 = [w.forces() for w in walkers]
    for a, c in zip(f1, f2):
        assert np.array_equal(a, c)  # deterministic reductions: bitwise repeatable
    t = b.autotune(use_cache=False)
    assert t["ra"] in (4, 8) and t["ch"] in (128, 256) and t["parts"] >= 1 and not b.tune_cached
    for wk in walkers:
        wk.force.zero_()
    b.execute()
    for i, w in enumerate(walkers):
        assert O.max_rel_force_err(w.forces(), f1[i]) < 2e-6
    assert b.status() == 0
    # a second batch of the same signature takes the cached choice without timing
    b2, walkers2, _ = _setup(ws, hill, True)
    assert b2.autotune() == t and b2.tune_cached


@pytest.mark.parametrize("ra,ch", [(8, 128), (4, 128), (8, 256), (4, 256)])
def test_batch_tile_shapes_agree(ra, ch):
    """Every tile shape the autotuner may pick: forces and CVs of all walkers
    within the FP64 oracle's gates (the walkers' groups are not multiples of the
    tiles, so ragged steps are included), and within 1e-6 of the default shape.
    The shapes group the FP32 pair terms differently before the 64-bit
    fixed-point sums, so they agree to FP32 rounding, not bit for bit."""
    ws, hill = _walkers(n_walkers=6, coord=(200, 700))   # full and ragged tiles in every shape
    b, walkers, specs = _setup(ws, hill, True)
    ref = []
    for shape in ((8, 128), (ra, ch)):
        b.set_tuning(ra=shape[0], ch=shape[1])
        assert b.tuning["ra"] == shape[0] and b.tuning["ch"] == shape[1]
        for wk in walkers:
            wk.force.zero_()
        b.execute()
        ref.append(([w.forces() for w in walkers], b.cv_values(), b.energies()))
    (f0, cv0, e0), (f1, cv1, e1) = ref
    for i in range(len(walkers)):
        assert O.max_rel_force_err(f1[i], f0[i]) < 1e-6, i
    np.testing.assert_allclose(cv1, cv0, rtol=1e-7)
    np.testing.assert_allclose(e1, e0, rtol=1e-6, atol=1e-9)
    for i, w in enumerate(ws):
        r = _oracle(w, specs[i], hill).execute(w["pos"], w["box"].ravel())
        assert O.max_rel_force_err(f1[i], r["forces"]) < 1e-4, i
    assert b.status() == 0


def test_batch_deposit_walker_order():
    ws, hill = _walkers(n_walkers=4, n_hills=500)
    hill["iparams"] = [2, 100000, 1, 0]  # pace 2
    b, walkers, specs = _setup(ws, hill, True, coord_restraint=False)
    n0 = b.num_hills()
    b.update_state(0)        # nothing before the first execute
    b.execute()
    cv = b.cv_values()
    E = b.energies()
    b.update_state(1)        # not a pace step
    assert b.num_hills() == n0
    b.update_state(2)
    assert b.num_hills() == n0 + 4
    b.update_state(2)        # once per step
    assert b.num_hills() == n0 + 4
    c, h = b.get_hills()
    hif = 1.0 / ((10.0 - 1.0) * 2.494338785)
    for i in range(4):
        assert c[n0 + i, 0] == cv[i, 2] and c[n0 + i, 1] == cv[i, 1]
        # hill-bias energy of walker i = its energy minus the distance restraint
        d = cv[i, 0] - np.float32(ws[i]["d0"] + 0.05)
        Vh = E[i] - 0.5 * 100.0 * d * d
        assert abs(h[n0 + i] - 1.2 * math.exp(-Vh * hif)) < 1e-9
    assert b.status() == 0


def test_batch_full_hill_table_sets_status():
    """A deposit that finds the table at its capacity keeps the hills that fit,
    drops the rest and raises bit 0 of the status word."""
    ws, hill = _walkers(n_walkers=4, n_hills=500)
    hill["iparams"] = [1, 502, 1, 0]  # pace 1, room for two more hills
    b, walkers, specs = _setup(ws, hill, True, coord_restraint=False)
    assert b.num_hills() == 500 and b.status() == 0
    b.execute()
    cv = b.cv_values()
    b.update_state(1)
    assert b.num_hills() == 502
    assert b.status() == 1
    c, h = b.get_hills()
    for i in range(2):
        assert c[500 + i, 0] == cv[i, 2] and c[500 + i, 1] == cv[i, 1]


def test_batch_rejects_unsupported_structure():
    from gluedmd_b200.batch import Batch, Walker, force_for
    from gluedmd_b200 import GluedError
    import numpy as np
    pos = np.random.default_rng(0).uniform(0, 2, (20, 3))
    f = force_for([(5, list(range(10)), [])], [])
    with pytest.raises(GluedError, match="not supported"):
        Batch([f], [Walker(pos, np.eye(3) * 2)])
    f1 = force_for([(1, [0, 1], [])], [])
    f2 = force_for([(2, [0, 1, 2], [])], [])
    with pytest.raises(GluedError, match="type differs|different"):
        Batch([f1, f2], [Walker(pos, np.eye(3) * 2), Walker(pos, np.eye(3) * 2)])
