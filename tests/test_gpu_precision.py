"""Sum-precision variants against the FP64 oracle, at the benchmark workloads.

* kernel sums (OPES, hill-sum MetaD) in FP32 and in two-sum compensated FP32
  (glued_context_set_sum_precision): C3 (10,000 OPES kernels) and the C1 hills
  form (2,000 hills) within the bench gates (forces 1e-4 relative in max-norm,
  CVs 1e-5, energies 1e-4);
* blocked coordination sums and the Kabsch RMSD (FP64 eigensolve) on C2;
* the 64-walker batch with two-sum hill sums and blocked coordination sums
  (glued_batch_set_sum_precision);
* OPES deposits with FP32 kernel sums still replay bit for bit against the
  oracle fed the product's CVs and energies (the kernel sum feeds the deposit
  only through the energy);
* argument checks of both setters.
"""
import numpy as np
import pytest

import oracle as O
import parity as P
from test_oracle import opes_system

pytestmark = pytest.mark.gpu

FORCE_TOL, CV_TOL, ENERGY_TOL = 1e-4, 1e-5, 1e-4


def _assert(err, label):
    assert err["force"] < FORCE_TOL, (label, "force", err["force"])
    assert err["cv"] < CV_TOL, (label, "cv", err["cv"])
    assert err["energy"] < ENERGY_TOL, (label, "energy", err["energy"])


def _single(w, kernel_sums, coord):
    import gpu_util
    ctx, f = gpu_util.make_context(w.positions, w.cvs, w.biases, masses=w.masses, pbc=w.pbc, box=w.box,
                                   blob=w.blob)
    nc = ctx.glued_context_for(f)
    nc.set_sum_precision(kernel_sums, coord)
    assert nc.sum_precision() == (kernel_sums, coord)
    e, F = ctx.computeForces()
    return P.check_single(w, e, F, np.array(f.getLastCVValues(ctx)))


@pytest.mark.parametrize("mode", [1, 2])
def test_c3_kernel_sums_fp32(mode):
    from gluedmd_b200 import workloads as W
    err = _single(W.config3(), mode, 0)
    _assert(err, f"C3 mode {mode}")
    assert abs(err["ref"]["energy"]) > 1.0


@pytest.mark.parametrize("mode", [1, 2])
def test_c1_hill_sums_fp32(mode):
    from gluedmd_b200 import workloads as W
    _assert(_single(W.config1("hills"), mode, 0), f"C1-hills mode {mode}")


@pytest.mark.parametrize("fit,blocked", [(False, 1), (True, 0), (True, 1)])
def test_c2_blocked_and_kabsch(fit, blocked):
    from gluedmd_b200 import workloads as W
    _assert(_single(W.config2(fit=fit), 0, blocked), f"C2 fit={fit} blocked={blocked}")


def test_c4_compensated_batch():
    from gluedmd_b200 import workloads as W
    from gluedmd_b200.batch import Batch, WalkerPool, force_for, c4_walker_biases
    ws, hill = W.config4_walkers()
    W.config4_restraints(ws)
    specs = [c4_walker_biases(w, hill) for w in ws]
    pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
    b = Batch([force_for(w["cvs"], s) for w, s in zip(ws, specs)], pool.walkers)
    b.set_hills(hill["centers"], hill["heights"])
    from gluedmd_b200 import GluedError
    for bad in (0, 3):
        with pytest.raises(GluedError):
            b.set_sum_precision(bad)
    b.set_sum_precision(2)
    assert b.sum_precision() == 2
    pool.force.zero_()
    b.execute()
    E, cv = b.energies(), b.cv_values()
    assert b.status() == 0
    for i, w in enumerate(ws):
        err = P.check_walker(w, specs[i], hill["centers"], hill["heights"], E[i], pool.walkers[i].forces(), cv[i])
        _assert(err, f"walker {i}")


@pytest.mark.parametrize("mode", [1, 2])
def test_opes_deposits_with_fp32_kernel_sums(mode):
    """150 steps of pace-1 OPES deposits (merges and appends): the kernel
    tables stay bit-identical to the oracle fed the product's CV values and
    bias energy; the energies agree with the oracle's FP64 sum to 1e-5."""
    import gpu_util
    cvs, biases = opes_system(variant=0, pace=1, sigma=0.3)
    rng = np.random.default_rng(11)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    ctx, f = gpu_util.make_context(np.zeros((4, 3)), cvs, biases)
    nc = ctx.glued_context_for(f)
    nc.set_sum_precision(mode, 0)
    for step in range(150):
        ctx.setStepCount(step)
        ctx.updateContextState()
        orc.update_state(step)
        ctx.setPositions(rng.uniform(0, 1.0, (4, 3)))
        e, F = ctx.computeForces()
        orc.cv_values = np.array(nc.cv_values())
        E_ref = orc.evaluate_biases(orc.cv_values)[0].sum()
        assert abs(e - E_ref) <= 1e-5 * max(1.0, abs(E_ref)), (step, e, E_ref)
        orc.bias_energies = np.array([e])
        orc.cv_ready = True
    from gluedmd_b200.merger import BiasStateMerger
    nk, logz, ns, mb, m2b, cb, sb, lb = BiasStateMerger._parse(f.getBiasState(), f)["opes"][0]
    st = orc.bias_state[0]
    assert nk == int(st["ist"][0]) and nk > 5
    assert np.array_equal(np.frombuffer(cb, "<f8"), st["centers"][:2 * nk])
    assert np.array_equal(np.frombuffer(sb, "<f8"), st["sigmas"][:2 * nk])
    assert np.array_equal(np.frombuffer(lb, "<f8"), st["logw"][:nk])


def test_sum_precision_argument_checks():
    import gpu_util
    from gluedmd_b200 import GluedError
    ctx, f = gpu_util.make_context(np.zeros((4, 3)), *opes_system())
    nc = ctx.glued_context_for(f)
    for bad in ((3, 0), (-1, 0), (0, 2)):
        with pytest.raises(GluedError):
            nc.set_sum_precision(*bad)
    assert nc.sum_precision() == (0, 0)
