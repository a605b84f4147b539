"""GPU parity of paths that the benchmark workloads do not reach.

* MetaD grid replay: the deposited grid (1e-12 relative) and numDeposited
  (bit-exact) against the oracle fed the product's CV values and bias energy
  each step (CommonGluedKernels.cpp:3645-3691, :5137-5145).
* OPES variants 0 (METAD), 1 (uniform), 2 (EXPLORE), with fixed and adaptive
  sigma (sigma0 <= 0: Welford statistics, CommonGluedKernels.cpp:3005-3027):
  merge/append decisions, kernel tables bit-exact; getOPESMetrics (zed, rct,
  nker, neff) and getKernelSigmas vs the oracle (:5164-5232).
* Multi-walker sharing (CudaGluedKernelFactory.cpp:30-46,
  CommonGluedKernels.cpp:5234-5262): a secondary context redirected to the
  primary's MetaD grid / OPES table; both walkers' deposits land in one table,
  replayed by two oracles that share their arrays.
* Kabsch RMSD (no reference counterpart): FP64 oracle, identity, 180 degree
  rotation and near-degenerate (nearly collinear) structures.
* Coordination with a hard cutoff (no reference counterpart) and coordination
  in a triclinic box.
"""
import math

import numpy as np
import pytest

import oracle as O
from test_oracle import metad_system, opes_system

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4


def _gpu():
    import gpu_util
    return gpu_util


def _parse(f):
    from gluedmd_b200.merger import BiasStateMerger
    return BiasStateMerger._parse(f.getBiasState(), f)


def _feed(orc, nc, e):
    """Give the oracle the product's CV values and bias energy of this step: the
    next deposit then starts from identical inputs (the FP32 CV values differ
    from the oracle's FP64 ones in the last bits)."""
    orc.cv_values = np.array(nc.cv_values())
    orc.bias_energies = np.array([e])
    orc.cv_ready = True


# ------------------------------------------------------------------ MetaD
def test_metad_grid_and_deposit_count_replay():
    """40 steps, pace 2, 64 x 64 periodic grid: after every step the product's
    energy equals the oracle's bias at the same CV values on the oracle's grid;
    at the end the grid agrees to 1e-12 and numDeposited is 19 on both sides."""
    cvs, biases = metad_system(pace=2)
    rng = np.random.default_rng(7)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=6)
    ctx, f = _gpu().make_context(np.zeros((6, 3)), cvs, biases)
    nc = ctx.glued_context_for(f)
    for step in range(40):
        pos = rng.uniform(0, 1.5, (6, 3))
        ctx.setStepCount(step)
        ctx.updateContextState()
        orc.update_state(step)
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        _feed(orc, nc, e)
        E_ref = orc.evaluate_biases(orc.cv_values)[0].sum()
        assert abs(e - E_ref) <= 1e-9 * max(1.0, abs(E_ref)), (step, e, E_ref)
    nd, g = _parse(f)["metad"][0]
    grid = np.frombuffer(g, "<f8")
    ref = orc.bias_state[0]["grid"]
    assert nd == orc.bias_state[0]["deposited"] == 19
    assert np.abs(ref).max() > 1.0
    np.testing.assert_allclose(grid, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


# ------------------------------------------------------------------- OPES
def _opes_replay(variant, adaptive, steps=150, seed=11):
    # variant 2 (EXPLORE) widens a fixed sigma0 by sqrt(gamma) = 4.5: a smaller
    # sigma0 keeps both merges and appends in the replay
    sigma = 0.0 if adaptive else (0.05 if variant == 2 else 0.3)
    cvs, biases = opes_system(variant=variant, pace=1, sigma=sigma)
    if adaptive:
        t, c, p, ip = biases[0]
        biases = [(t, c, p, list(ip) + [12])]  # adaptive stride: 12 samples before the first deposit
    rng = np.random.default_rng(seed)
    orc = O.OracleSystem(cvs, biases, mode="f64", num_particles=4)
    ctx, f = _gpu().make_context(np.zeros((4, 3)), cvs, biases)
    nc = ctx.glued_context_for(f)
    dec_gpu = []
    for step in range(steps):
        pos = rng.uniform(0, 1.0, (4, 3))
        ctx.setStepCount(step)
        ctx.updateContextState()
        if step > 0:
            dec_gpu.append(nc.opes_last_decision(0))
        orc.update_state(step)
        ctx.setPositions(pos)
        e, F = ctx.computeForces()
        _feed(orc, nc, e)
        if adaptive:
            orc.welford()
        E_ref = orc.evaluate_biases(orc.cv_values)[0].sum()
        assert abs(e - E_ref) <= 1e-9 * max(1.0, abs(E_ref)), (step, e, E_ref)
    return orc, ctx, f, dec_gpu


@pytest.mark.parametrize("variant,adaptive", [(0, False), (1, False), (2, False), (0, True), (2, True)])
def test_opes_variants_decisions_tables_metrics(variant, adaptive):
    orc, ctx, f, dec_gpu = _opes_replay(variant, adaptive)
    st = orc.bias_state[0]
    dec_orc = list(st["decisions"])
    assert dec_gpu == dec_orc
    assert sum(d >= 0 for d in dec_orc) > 5 and sum(d == -1 for d in dec_orc) > 5
    if adaptive:
        assert dec_orc[:11] == [-2] * 11 and dec_orc[11] != -2
    nk, su, ns, mean, m2, c, s, lw = _parse(f)["opes"][0]
    assert nk == int(st["ist"][0]) and ns == int(st["ist"][1])
    assert np.array_equal(np.frombuffer(c, "<f8"), st["centers"][:2 * nk])
    assert np.array_equal(np.frombuffer(s, "<f8"), st["sigmas"][:2 * nk])
    assert np.array_equal(np.frombuffer(lw, "<f8"), st["logw"][:nk])
    # Welford statistics (adaptive) in the same order, sum_uprob to FP64 summation order
    np.testing.assert_allclose(np.frombuffer(mean, "<f8"), st["mean"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(np.frombuffer(m2, "<f8"), st["m2"], rtol=1e-12, atol=1e-15)
    assert abs(su - st["dst"][0]) <= 1e-10 * abs(st["dst"][0])
    m = f.getOPESMetrics(ctx, 0)
    mr = orc.opes_metrics(0)
    assert m[2] == mr[2] == nk
    np.testing.assert_allclose(m, mr, rtol=1e-10, atol=1e-12)
    sig = np.asarray(f.getKernelSigmas(ctx, 0), dtype=np.float32)
    assert np.array_equal(sig, orc.kernel_sigmas(0))


# ---------------------------------------------------------- multi-walker
def test_multiwalker_metad_shared_grid():
    """Walker 1's MetaD grid pointer is redirected to walker 0's grid; both deposit
    every 2 steps into it (walker 0 first). Two oracles share one grid array."""
    cvs, biases = metad_system(pace=2)
    g = _gpu()
    ctxs = [g.make_context(np.zeros((6, 3)), cvs, biases) for _ in range(2)]
    (c0, f0), (c1, f1) = ctxs
    f1.setMultiWalkerPtrs(c1, 0, f0.getMultiWalkerPtrs(c0, 0))
    orcs = [O.OracleSystem(cvs, biases, mode="f64", num_particles=6) for _ in range(2)]
    orcs[1].bias_state[0]["grid"] = orcs[0].bias_state[0]["grid"]
    rng = np.random.default_rng(17)
    for step in range(30):
        for (ctx, f), orc in zip(ctxs, orcs):
            ctx.setStepCount(step)
            ctx.updateContextState()
            orc.update_state(step)
        for (ctx, f), orc in zip(ctxs, orcs):
            ctx.setPositions(rng.uniform(0, 1.5, (6, 3)))
            e, F = ctx.computeForces()
            _feed(orc, ctx.glued_context_for(f), e)
            E_ref = orc.evaluate_biases(orc.cv_values)[0].sum()
            assert abs(e - E_ref) <= 1e-9 * max(1.0, abs(E_ref)), (step, e, E_ref)
    nd, grid = _parse(f0)["metad"][0]
    ref = orcs[0].bias_state[0]["grid"]
    assert nd == orcs[0].bias_state[0]["deposited"] == 14
    assert orcs[1].bias_state[0]["deposited"] == 14
    np.testing.assert_allclose(np.frombuffer(grid, "<f8"), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_multiwalker_opes_shared_table():
    """Walker 1's OPES kernel table (centres, sigmas, log-weights, kernel count,
    slot counter) is walker 0's; each keeps its own sum_uprob and statistics.
    Decisions of both walkers and the shared table are bit-identical to two
    oracles that share those arrays."""
    cvs, biases = opes_system(variant=0, pace=1, sigma=0.3)
    g = _gpu()
    ctxs = [g.make_context(np.zeros((4, 3)), cvs, biases) for _ in range(2)]
    (c0, f0), (c1, f1) = ctxs
    f1.setMultiWalkerPtrs(c1, 0, f0.getMultiWalkerPtrs(c0, 0))
    orcs = [O.OracleSystem(cvs, biases, mode="f64", num_particles=4) for _ in range(2)]
    s0, s1 = orcs[0].bias_state[0], orcs[1].bias_state[0]
    for key in ("centers", "sigmas", "logw"):
        s1[key] = s0[key]

    def share(src, dst):
        dst["ist"][0] = src["ist"][0]   # numKernels
        dst["ist"][3] = src["ist"][3]   # numAllocated

    rng = np.random.default_rng(19)
    dec = [[], []]
    for step in range(80):
        for w, ((ctx, f), orc) in enumerate(zip(ctxs, orcs)):
            ctx.setStepCount(step)
            ctx.updateContextState()
            if step > 0:
                dec[w].append(ctx.glued_context_for(f).opes_last_decision(0))
            orc.update_state(step)
            share(orc.bias_state[0], orcs[1 - w].bias_state[0])
        for (ctx, f), orc in zip(ctxs, orcs):
            ctx.setPositions(rng.uniform(0, 1.0, (4, 3)))
            e, F = ctx.computeForces()
            _feed(orc, ctx.glued_context_for(f), e)
            E_ref = orc.evaluate_biases(orc.cv_values)[0].sum()
            assert abs(e - E_ref) <= 1e-9 * max(1.0, abs(E_ref)), (step, e, E_ref)
    assert dec[0] == list(s0["decisions"]) and dec[1] == list(s1["decisions"])
    assert sum(d >= 0 for d in dec[1]) > 5 and sum(d == -1 for d in dec[1]) > 5
    nk, su, ns, mean, m2, c, s, lw = _parse(f0)["opes"][0]
    assert nk == int(s0["ist"][0]) == int(s1["ist"][0])
    assert np.array_equal(np.frombuffer(c, "<f8"), s0["centers"][:2 * nk])
    assert np.array_equal(np.frombuffer(s, "<f8"), s0["sigmas"][:2 * nk])
    assert np.array_equal(np.frombuffer(lw, "<f8"), s0["logw"][:nk])


# ------------------------------------------------------------------ Kabsch
def _rot(axis, angle):
    a = np.asarray(axis, float)
    a /= np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * K @ K


def _kabsch_case(kind, n_atoms, seed=5):
    rng = np.random.default_rng(seed)
    n = n_atoms + 40
    pos = rng.uniform(0.5, 3.5, (n, 3))
    atoms = rng.choice(n, n_atoms, replace=False)
    x = pos[atoms]
    if kind == "collinear":
        # nearly collinear atoms: the two largest quaternion eigenvalues nearly coincide
        t = np.linspace(-1.0, 1.0, n_atoms)
        x = np.c_[2.0 + t, 2.0 + 0.5 * t, 2.0 - 0.3 * t] + rng.normal(0, 1e-3, (n_atoms, 3))
        pos[atoms] = x
    c = x.mean(0)
    if kind == "identity":
        ref = x.copy()
    elif kind == "rot180":
        ref = (x - c) @ _rot([0.3, -1.0, 0.5], math.pi).T + c + [0.2, -0.1, 0.4]
    elif kind == "rot180_noise":
        ref = (x - c) @ _rot([1.0, 0.2, 0.1], math.pi).T + c + rng.normal(0, 0.05, x.shape)
    else:  # random rotation + noise (also "collinear")
        ref = (x - c) @ _rot(rng.normal(size=3), rng.uniform(0, math.pi)).T + c + rng.normal(0, 0.1, x.shape)
    ref = ref.astype(np.float32).astype(np.float64)
    return pos, [(O.CV_RMSD_KABSCH, [int(a) for a in atoms], list(ref.ravel()))]


@pytest.mark.parametrize("kind,n_atoms", [("random", 50), ("random", 1000), ("random", 3000), ("identity", 200),
                                          ("rot180", 200), ("rot180_noise", 300), ("collinear", 100)])
def test_kabsch_rmsd_vs_fp64_oracle(kind, n_atoms):
    pos, cvs = _kabsch_case(kind, n_atoms)
    g = [1.7]
    ref = O.OracleSystem(cvs, mode="f64", test_bias_gradients=g, num_particles=len(pos)).execute(pos)
    res = _gpu().run(pos, cvs, grad=g)
    if kind in ("identity", "rot180"):
        # exact superposition: RMSD zero up to the FP32 positions
        assert ref["cv_values"][0] < 1e-6 and res["cv_values"][0] < 1e-5
        return
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-6)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


# ------------------------------------------------------------ coordination
@pytest.mark.parametrize("rc", [0.6, 1.2])
def test_coordination_cutoff_vs_fp64_oracle(rc):
    rng = np.random.default_rng(31)
    n, L = 3000, 3.2
    pos = rng.uniform(0, L, (n, 3))
    A = rng.choice(n, 300, replace=False)
    B = rng.choice(n, 1100, replace=False)
    cvs = [(O.CV_COORDINATION_CUTOFF, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.35, 6, 12, rc]),
           (O.CV_COORDINATION, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.35, 6, 12])]
    g = [0.9, -0.4]
    box = np.diag([L, L, L])
    ref = O.OracleSystem(cvs, periodic=True, mode="f64", test_bias_gradients=g,
                         num_particles=n).execute(pos, box.ravel())
    res = _gpu().run(pos, cvs, pbc=True, box=box, grad=g)
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert ref["cv_values"][0] < ref["cv_values"][1]  # the cutoff removes the tail
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


@pytest.mark.parametrize("nm", [(6, 12), (4.5, 9.5)])
def test_coordination_triclinic_box(nm):
    """Reduced triclinic box (a along x, b in the xy plane): coordination, distance
    and angle CVs through the box's minimum image (CommonGluedKernels.cpp:74-112)."""
    rng = np.random.default_rng(41)
    n, L = 1200, 2.6
    box = np.array([[L, 0, 0], [0.3 * L, L, 0], [-0.2 * L, 0.25 * L, L]])
    frac = rng.uniform(0, 1, (n, 3))
    pos = frac @ box
    A = rng.choice(n, 150, replace=False)
    B = rng.choice(n, 700, replace=False)
    cvs = [(O.CV_DISTANCE, [int(A[0]), int(B[0])], []), (O.CV_ANGLE, [int(A[1]), int(B[1]), int(A[2])], []),
           (O.CV_COORDINATION, [len(A)] + [int(x) for x in A] + [int(x) for x in B], [0.3, nm[0], nm[1]])]
    g = [0.5, -1.1, 0.8]
    ref = O.OracleSystem(cvs, periodic=True, mode="f64", test_bias_gradients=g,
                         num_particles=n).execute(pos, box.ravel())
    res = _gpu().run(pos, cvs, pbc=True, box=box, grad=g)
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL
