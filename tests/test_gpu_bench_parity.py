"""Parity at the exact benchmark workloads: every configuration bench.py times,
built by the same workload functions at full size, against the FP64 oracle.

Gates (per system, per walker): forces within 1e-4 relative in max-norm of the
FP64 oracle; CV values within 1e-5 relative; energies within 1e-4 relative
(|dE| / max(1, |E|)).

* 64 walkers: 64 walkers of 1k-50k atoms, 256 x 1,024 coordination each,
  restraints just off the initial values, and the shared 50,000-hill table,
  in the tile shape the autotuner picks (as timed);
* C2: 2,048 x 8,192 coordination (16.8 M pairs) + RMSD over 1,000 atoms + the
  256 x 256 MetaD grid holding 20,000 hills;
* C1: 22 atoms, two dihedrals, 256 x 256 periodic grid of 2,000 WT hills; the
  same hills as PBMETAD sub-grids + EXTERNAL grid; and as a direct hill sum;
* C3: OPES on (COM distance, gyration) of 5,000 of 50,000 atoms with 10,000
  compressed kernels: energy and forces (the deposit decisions at this size are
  checked in test_gpu_parity.py).
"""
import numpy as np
import pytest

import oracle as O
import parity as P

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4
CV_TOL = 1e-5
ENERGY_TOL = 1e-4


@pytest.fixture(scope="module")
def c4():
    from gluedmd_b200 import workloads as W
    ws, hill = W.config4_walkers()
    W.config4_restraints(ws)
    return ws, hill


def _single(w):
    import gpu_util
    ctx, f = gpu_util.make_context(w.positions, w.cvs, w.biases, masses=w.masses, pbc=w.pbc, box=w.box,
                                   blob=w.blob)
    e, F = ctx.computeForces()
    return e, F, np.array(f.getLastCVValues(ctx))


def _assert(err, label):
    assert err["force"] < FORCE_TOL, (label, "force", err["force"])
    assert err["cv"] < CV_TOL, (label, "cv", err["cv"])
    assert err["energy"] < ENERGY_TOL, (label, "energy", err["energy"])


@pytest.mark.parametrize("tuned", [True, False])
def test_c4_64_walkers_full_size(c4, tuned):
    """All 64 walkers of the timed workload, with the autotuned tiling and with
    the default one: every walker's forces, CVs and energy vs the FP64 oracle."""
    from gluedmd_b200.batch import Batch, WalkerPool, force_for, c4_walker_biases
    ws, hill = c4
    specs = [c4_walker_biases(w, hill) for w in ws]
    pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
    b = Batch([force_for(w["cvs"], s) for w, s in zip(ws, specs)], pool.walkers)
    b.set_hills(hill["centers"], hill["heights"])
    if tuned:
        b.autotune()
    pool.force.zero_()
    b.execute()
    E, cv = b.energies(), b.cv_values()
    assert b.status() == 0
    errs = []
    for i, w in enumerate(ws):
        err = P.check_walker(w, specs[i], hill["centers"], hill["heights"], E[i], pool.walkers[i].forces(), cv[i])
        _assert(err, f"walker {i}")
        errs.append(err)
    # the restraint and hill forces are real forces, not rounding noise
    assert min(np.abs(e["ref"]["forces"]).max() for e in errs) > 1.0


def test_c2_full_size():
    from gluedmd_b200 import workloads as W
    w = W.config2()
    e, F, cv = _single(w)
    err = P.check_single(w, e, F, cv)
    _assert(err, "C2")


@pytest.mark.parametrize("form", ["grid", "pbmetad", "hills"])
def test_c1_full_size(form):
    from gluedmd_b200 import workloads as W
    w = W.config1(form)
    e, F, cv = _single(w)
    err = P.check_single(w, e, F, cv)
    _assert(err, f"C1-{form}")


def test_c3_full_size():
    from gluedmd_b200 import workloads as W
    w = W.config3()
    e, F, cv = _single(w)
    err = P.check_single(w, e, F, cv)
    _assert(err, "C3")
    # the 10,000-kernel sum is populated at these CVs (a non-trivial bias)
    assert abs(err["ref"]["energy"]) > 1.0
