"""Group CVs on CTA clusters (COM distance, gyration, RMSD, PCA with groups of
>= 1,024 atoms) vs the FP64 oracle.

Tolerances as the other parity tests: CV values 1e-5 relative, forces 1e-4
relative in max-norm. Sizes cover slices of unequal length (group sizes not a
multiple of the cluster size, a COM-distance group boundary inside a slice),
empty trailing slices, and slices too large for the shared-memory cache."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4


def _system(seed, n_atoms, box, sizes):
    """Atoms uniform in a cube; CVs over disjoint seeded selections: COM distance
    (split n1 | n2), gyration, RMSD and PCA, each of the given sizes."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, box, (n_atoms, 3))
    perm = rng.permutation(n_atoms)
    k = 0

    def take(n):
        nonlocal k
        a = [int(x) for x in perm[k:k + n]]
        k += n
        return a

    cvs = []
    n1, n2 = sizes["com"]
    cvs.append((O.CV_COM_DISTANCE, take(n1) + take(n2), [n1]))
    cvs.append((O.CV_GYRATION, take(sizes["gyr"]), []))
    a = take(sizes["rmsd"])
    cvs.append((O.CV_RMSD, a, list((pos[a] + rng.normal(0, 0.1, (len(a), 3))).ravel())))
    a = take(sizes["pca"])
    cvs.append((O.CV_PCA, a, list((pos[a] + rng.normal(0, 0.1, (len(a), 3))).ravel()) +
                list(rng.normal(0, 1, 3 * len(a)))))
    masses = rng.uniform(1, 16, n_atoms)
    return pos, cvs, masses, np.diag([box, box, box])


@pytest.mark.parametrize("seed,sizes", [
    (1, dict(com=(700, 1331), gyr=1031, rmsd=1024, pca=1100)),
    (2, dict(com=(2500, 2500), gyr=5000, rmsd=1000, pca=1500)),
    (3, dict(com=(3, 1021), gyr=1025, rmsd=1030, pca=9)),   # 9 atoms: slices of 2, ranks 5-7 empty
])
@pytest.mark.parametrize("periodic", [False, True])
def test_cluster_group_cvs_vs_fp64_oracle(seed, sizes, periodic):
    n = sum(sizes["com"]) + sizes["gyr"] + sizes["rmsd"] + sizes["pca"] + 100
    pos, cvs, masses, box = _system(seed, n, 6.0, sizes)
    g = list(np.random.default_rng(seed + 50).normal(0, 1, len(cvs)))
    ref = O.OracleSystem(cvs, masses=masses, periodic=periodic, mode="f64", test_bias_gradients=g,
                         num_particles=n).execute(pos, box.ravel())
    import gpu_util
    res = gpu_util.run(pos, cvs, masses=masses, pbc=periodic, box=box, grad=g)
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


def test_cluster_gyration_beyond_shared_cache():
    """70,000-atom gyration: 8,750-atom slices exceed the 8,192-atom shared cache,
    so every CTA reads its slice from global memory."""
    rng = np.random.default_rng(4)
    n = 70000
    pos = rng.uniform(0, 9.0, (n, 3))
    cvs = [(O.CV_GYRATION, list(range(n)), [])]
    masses = rng.uniform(1, 16, n)
    ref = O.OracleSystem(cvs, masses=masses, periodic=True, mode="f64", test_bias_gradients=[0.7],
                         num_particles=n).execute(pos, np.diag([9.0] * 3).ravel())
    import gpu_util
    res = gpu_util.run(pos, cvs, masses=masses, pbc=True, box=np.diag([9.0] * 3), grad=[0.7])
    np.testing.assert_allclose(res["cv_values"], ref["cv_values"], rtol=1e-5)
    assert O.max_rel_force_err(res["forces"], ref["forces"]) < FORCE_TOL


def test_cluster_forces_repeatable():
    """Rank-ordered cluster sums: bitwise identical forces on repeated evaluation."""
    sizes = dict(com=(1200, 1300), gyr=2000, rmsd=1500, pca=1100)
    pos, cvs, masses, box = _system(5, 8000, 6.0, sizes)
    import gpu_util
    ctx, f = gpu_util.make_context(pos, cvs, masses=masses, pbc=True, box=box, grad=[0.3, -0.2, 0.5, 0.1])
    e1, F1 = ctx.computeForces()
    e2, F2 = ctx.computeForces()
    assert np.array_equal(F1, F2)


@pytest.mark.parametrize("periodic", [False, True])
def test_group_cvs_beside_coordination(periodic):
    """Coordination with a few single-CTA group CVs: the group kernel runs beside
    the coordination grid on the SMs it leaves free (launched after it, waiting
    for it only at its end); values and forces vs the FP64 oracle, and bitwise
    repeatable."""
    rng = np.random.default_rng(12)
    n, box = 6000, 4.0
    pos = rng.uniform(0, box, (n, 3))
    perm = [int(x) for x in rng.permutation(n)]
    A, B = perm[:300], perm[300:1500]
    r = perm[1500:2300]
    cvs = [(O.CV_COORDINATION, [len(A)] + A + B, [0.35, 6, 12]),
           (O.CV_RMSD, r, list((pos[r] + rng.normal(0, 0.1, (len(r), 3))).ravel())),
           (O.CV_GYRATION, perm[2300:2900], []),
           (O.CV_COM_DISTANCE, perm[2900:3100] + perm[3100:3500], [200])]
    masses = rng.uniform(1, 16, n)
    g = [0.01, 0.8, -0.6, 0.4]
    ref = O.OracleSystem(cvs, masses=masses, periodic=periodic, mode="f64", test_bias_gradients=g,
                         num_particles=n).execute(pos, np.diag([box] * 3).ravel())
    import gpu_util
    ctx, f = gpu_util.make_context(pos, cvs, masses=masses, pbc=periodic, box=np.diag([box] * 3), grad=g)
    e, F = ctx.computeForces()
    np.testing.assert_allclose(np.array(f.getLastCVValues(ctx)), ref["cv_values"], rtol=1e-5, atol=1e-5)
    assert O.max_rel_force_err(F, ref["forces"]) < FORCE_TOL
    _, F2 = ctx.computeForces()
    assert np.array_equal(F, F2)
