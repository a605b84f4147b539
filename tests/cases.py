"""Known-answer cases restated from the reference's acceptance tests.

Each case gives positions, CV specs (type, atoms, params) in the reference's
parameter encoding, optional injected dU/dCV (the reference's
setTestBiasGradients mock) and the analytic answers those tests assert. The
expected numbers are re-derived from the formulas the reference tests state;
the file:line of the test each case follows is in its 'ref' field.
"""
import math

CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION = 1, 2, 3, 4, 5
CV_COORDINATION, CV_RMSD, CV_PATH, CV_CONTACTMAP, CV_PCA = 6, 7, 10, 13, 21

TOL_CV = 1e-4
TOL_F = 1e-3


def _path_params(lam, frames):
    p = [lam, len(frames)]
    for fr in frames:
        for xyz in fr:
            p.extend(xyz)
    return p


def _sw(x, n, m):
    return (1 - x ** n) / (1 - x ** m)


CASES = [
    # ---- distance (tests/test_cv_distance.py:70-134)
    dict(name="distance_value", ref="tests/test_cv_distance.py:70-78",
         pos=[(0, 0, 0), (0.5, 0, 0), (5, 5, 5)], cvs=[(CV_DISTANCE, [0, 1], [])], cv=[0.5]),
    dict(name="distance_force", ref="tests/test_cv_distance.py:80-97",
         pos=[(0, 0, 0), (1.0, 0, 0), (5, 5, 5)], cvs=[(CV_DISTANCE, [0, 1], [])], grad=[1.0],
         forces={0: (1.0, 0, 0), 1: (-1.0, 0, 0)}),
    dict(name="distance_pbc", ref="tests/test_cv_distance.py:124-131",
         pos=[(0, 0, 0), (0.99, 0, 0)], cvs=[(CV_DISTANCE, [0, 1], [])], pbc=True, box=1.0, cv=[0.01]),
    dict(name="distance_multiple", ref="tests/test_cv_distance.py:134-142",
         pos=[(0, 0, 0), (1.0, 0, 0), (0, 2.0, 0), (5, 5, 5)],
         cvs=[(CV_DISTANCE, [0, 1], []), (CV_DISTANCE, [0, 2], [])], cv=[1.0, 2.0]),
    # ---- angle / dihedral (tests/test_cv_angle_dihedral.py:64-229)
    dict(name="angle_right", ref="tests/test_cv_angle_dihedral.py:64-71",
         pos=[(1, 0, 0), (0, 0, 0), (0, 1, 0)], cvs=[(CV_ANGLE, [0, 1, 2], [])], cv=[math.pi / 2]),
    dict(name="angle_60", ref="tests/test_cv_angle_dihedral.py:74-82",
         pos=[(1, 0, 0), (0, 0, 0), (0.5, math.sqrt(3) / 2, 0), (0.5, 0.5, 0.5)],
         cvs=[(CV_ANGLE, [0, 1, 2], [])], cv=[math.pi / 3]),
    dict(name="dihedral_zero", ref="tests/test_cv_angle_dihedral.py:135-143",
         pos=[(1, 0, 0), (0, 0, 0), (0, 0, 1), (1, 0, 1), (5, 5, 5)],
         cvs=[(CV_DIHEDRAL, [0, 1, 2, 3], [])], cv=[0.0]),
    dict(name="dihedral_pi", ref="tests/test_cv_angle_dihedral.py:146-155",
         pos=[(1, 0, 0), (0, 0, 0), (0, 0, 1), (-1, 0, 1), (5, 5, 5)],
         cvs=[(CV_DIHEDRAL, [0, 1, 2, 3], [])], cv_abs=[math.pi]),
    dict(name="dihedral_90", ref="tests/test_cv_angle_dihedral.py:158-167",
         pos=[(1, 0, 0), (0, 0, 0), (0, 0, 1), (0, 1, 1), (5, 5, 5)],
         cvs=[(CV_DIHEDRAL, [0, 1, 2, 3], [])], cv=[math.pi / 2]),
    # ---- COM distance / gyration (tests/test_cv_com_rg.py:70-244)
    dict(name="com_single", ref="tests/test_cv_com_rg.py:70-82",
         pos=[(0, 0, 0), (1, 0, 0), (0.5, 0.5, 0.5)], cvs=[(CV_COM_DISTANCE, [0, 1], [1])], cv=[1.0]),
    dict(name="com_two_atom_group", ref="tests/test_cv_com_rg.py:85-96",
         pos=[(0, 0, 0), (1, 0, 0), (2, 0, 0), (5, 5, 5)], cvs=[(CV_COM_DISTANCE, [0, 1, 2], [2])], cv=[1.5]),
    dict(name="com_weighted", ref="tests/test_cv_com_rg.py:99-111",
         pos=[(0, 0, 0), (1, 0, 0), (2, 0, 0), (5, 5, 5)], masses=[1.0, 3.0, 1.0, 1.0],
         cvs=[(CV_COM_DISTANCE, [0, 1, 2], [2])], cv=[1.25]),
    dict(name="com_force_sum", ref="tests/test_cv_com_rg.py:114-125",
         pos=[(0, 0, 0), (1, 0, 0), (2, 0, 0), (5, 5, 5)], cvs=[(CV_COM_DISTANCE, [0, 1, 2], [2])],
         grad=[1.0], force_sum_zero=[0, 1, 2]),
    dict(name="rg_symmetric", ref="tests/test_cv_com_rg.py:160-168",
         pos=[(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0)], cvs=[(CV_GYRATION, [0, 1, 2, 3], [])], cv=[1.0]),
    dict(name="rg_two_atoms", ref="tests/test_cv_com_rg.py:171-178",
         pos=[(0, 0, 0), (2, 0, 0), (5, 5, 5)], cvs=[(CV_GYRATION, [0, 1], [])], cv=[1.0]),
    dict(name="rg_weighted", ref="tests/test_cv_com_rg.py:181-189",
         pos=[(0, 0, 0), (10, 0, 0), (5, 5, 5)], masses=[9.0, 1.0, 1.0],
         cvs=[(CV_GYRATION, [0, 1], [])], cv=[3.0]),
    dict(name="rg_force_sum", ref="tests/test_cv_com_rg.py:192-202",
         pos=[(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1.5, 0)], cvs=[(CV_GYRATION, [0, 1, 2, 3], [])],
         grad=[1.0], force_sum_zero=[0, 1, 2, 3]),
    dict(name="com_rg_mixed", ref="tests/test_cv_com_rg.py:229-244",
         pos=[(0, 0, 0), (2, 0, 0), (4, 0, 0), (5, 5, 5)],
         cvs=[(CV_COM_DISTANCE, [0, 1, 2], [1]), (CV_GYRATION, [0, 1, 2], [])],
         cv=[3.0, math.sqrt(8.0 / 3.0)]),
    # ---- coordination (tests/test_cv_coordination.py:66-184)
    dict(name="coord_exact", ref="tests/test_cv_coordination.py:66-77",
         pos=[(0, 0, 0), (0.5, 0, 0), (5, 5, 5)], cvs=[(CV_COORDINATION, [1, 0, 1], [1.5, 1.0, 2.0])],
         cv=[0.75]),
    dict(name="coord_beyond_r0", ref="tests/test_cv_coordination.py:80-91",
         pos=[(0, 0, 0), (2.0, 0, 0), (5, 5, 5)], cvs=[(CV_COORDINATION, [1, 0, 1], [1.0, 6.0, 12.0])],
         cv=[(1 - 2.0 ** 6) / (1 - 2.0 ** 12)]),
    dict(name="coord_two_pairs", ref="tests/test_cv_coordination.py:94-108",
         pos=[(0, 0, 0), (0.5, 0, 0), (2.0, 0, 0), (5, 5, 5)],
         cvs=[(CV_COORDINATION, [1, 0, 1, 2], [1.0, 1.0, 2.0])], cv=[1.0]),
    dict(name="coord_force", ref="tests/test_cv_coordination.py:111-140",
         pos=[(0, 0, 0), (0.5, 0, 0), (5, 5, 5)], cvs=[(CV_COORDINATION, [1, 0, 1], [1.5, 1.0, 2.0])],
         grad=[1.0], forces={0: (-0.375, 0, 0)}, force_sum_zero=[0, 1]),
    dict(name="coord_2a2b", ref="tests/test_cv_coordination.py:168-184",
         pos=[(0, 0, 0), (0, 1.0, 0), (0.5, 0, 0), (0.5, 1.0, 0), (9, 9, 9)],
         cvs=[(CV_COORDINATION, [2, 0, 1, 2, 3], [1.0, 6.0, 12.0])],
         cv=[2 * _sw(0.5, 6, 12) + 2 * _sw(math.sqrt(1.25), 6, 12)]),
    # ---- RMSD no-fit (tests/test_cv_rmsd.py:65-140)
    dict(name="rmsd_single", ref="tests/test_cv_rmsd.py:65-75",
         pos=[(0.3, 0, 0), (5, 5, 5)], cvs=[(CV_RMSD, [0], [0, 0, 0])], cv=[0.3]),
    dict(name="rmsd_two_equal", ref="tests/test_cv_rmsd.py:78-90",
         pos=[(0.3, 0, 0), (-0.3, 0, 0), (5, 5, 5)], cvs=[(CV_RMSD, [0, 1], [0, 0, 0, 0, 0, 0])], cv=[0.3]),
    dict(name="rmsd_unequal", ref="tests/test_cv_rmsd.py:93-106",
         pos=[(0, 0, 0), (0.6, 0, 0), (5, 5, 5)], cvs=[(CV_RMSD, [0, 1], [0, 0, 0, 0, 0, 0])],
         cv=[math.sqrt(0.18)]),
    dict(name="rmsd_3d", ref="tests/test_cv_rmsd.py:109-118",
         pos=[(0.1, 0.2, 0.2), (5, 5, 5)], cvs=[(CV_RMSD, [0], [0, 0, 0])], cv=[0.3]),
    dict(name="rmsd_force", ref="tests/test_cv_rmsd.py:121-132",
         pos=[(0.3, 0, 0), (5, 5, 5)], cvs=[(CV_RMSD, [0], [0, 0, 0])], grad=[1.0], forces={0: (-1.0, 0, 0)}),
    # ---- path (tests/test_cv_path.py:76-128)
    dict(name="path_midpoint", ref="tests/test_cv_path.py:76-95",
         pos=[(1, 0, 0), (5, 5, 5)], cvs=[(CV_PATH, [0], _path_params(1.0, [[(0, 0, 0)], [(2, 0, 0)]]))],
         cv=[1.5, 1.0 - math.log(2.0)]),
    dict(name="path_at_frame0", ref="tests/test_cv_path.py:98-117",
         pos=[(0, 0, 0), (5, 5, 5)], cvs=[(CV_PATH, [0], _path_params(2.0, [[(0, 0, 0)], [(2, 0, 0)]]))],
         cv=[(1 + 2 * math.exp(-8)) / (1 + math.exp(-8)), -math.log(1 + math.exp(-8)) / 2.0]),
    dict(name="path_three_frames", ref="tests/test_cv_path.py:120-139",
         pos=[(1, 0, 0), (5, 5, 5)],
         cvs=[(CV_PATH, [0], _path_params(1.0, [[(0, 0, 0)], [(1, 0, 0)], [(2, 0, 0)]]))],
         cv=[(1 * math.exp(-1) + 2 + 3 * math.exp(-1)) / (1 + 2 * math.exp(-1)),
             -math.log(1 + 2 * math.exp(-1))]),
    # ---- contact map (tests/test_cv_contactmap.py:72-113): s = (1-x^n)/(1-x^m)
    dict(name="cmap_far", ref="tests/test_cv_contactmap.py:72-78",
         pos=[(0, 0, 0), (5.0, 0, 0)], cvs=[(CV_CONTACTMAP, [0, 1], [0.5, 6, 12, 1.0])], cv_below=[1e-4]),
    dict(name="cmap_near", ref="tests/test_cv_contactmap.py:81-87",
         pos=[(0, 0, 0), (0.01, 0, 0)], cvs=[(CV_CONTACTMAP, [0, 1], [0.5, 6, 12, 1.0])], cv=[1.0], tol=0.01),
    dict(name="cmap_three_pairs", ref="tests/test_cv_contactmap.py:90-101",
         pos=[(0.1, 0.2, 0.3), (0.5, 0.1, 0.7), (0.2, 0.9, 0.4), (0.6, 0.6, 0.1), (0.3, 0.3, 0.3), (0.8, 0.2, 0.9)],
         cvs=[(CV_CONTACTMAP, [0, 1, 2, 3, 4, 5], [0.5, 6, 12, 1.0, 0.4, 8, 16, 0.5, 0.6, 6, 12, 2.0])],
         cv=[1.0 * _sw(math.dist((0.1, 0.2, 0.3), (0.5, 0.1, 0.7)) / 0.5, 6, 12)
             + 0.5 * _sw(math.dist((0.2, 0.9, 0.4), (0.6, 0.6, 0.1)) / 0.4, 8, 16)
             + 2.0 * _sw(math.dist((0.3, 0.3, 0.3), (0.8, 0.2, 0.9)) / 0.6, 6, 12)]),
    dict(name="cmap_weight", ref="tests/test_cv_contactmap.py:104-113",
         pos=[(0, 0, 0), (0.2, 0, 0)], cvs=[(CV_CONTACTMAP, [0, 1], [0.5, 6, 12, 3.0])],
         cv=[3.0 * _sw(0.4, 6, 12)]),
    # ---- PCA (tests/test_cv_pca.py:58-123): CV = sum (r - mean) . ev, Jacobian = ev
    dict(name="pca_at_reference", ref="tests/test_cv_pca.py:58-68",
         pos=[(0.1 * i, 0.2 * i, 0.3 * i) for i in range(4)],
         cvs=[(CV_PCA, [0, 1, 2, 3], [v for i in range(4) for v in (0.1 * i, 0.2 * i, 0.3 * i)]
               + [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 1.0, 0, 0])], cv=[0.0]),
    dict(name="pca_single_atom_x", ref="tests/test_cv_pca.py:71-81",
         pos=[(0.7, 0.3, 0.1), (0, 0, 0), (0, 0, 0), (0, 0, 0)],
         cvs=[(CV_PCA, [0], [0.5, 0.3, 0.1, 1.0, 0, 0])], cv=[0.2]),
    dict(name="pca_force", ref="tests/test_cv_pca.py:104-123",
         pos=[(0.3, 0.1, 0.2), (0.5, 0.4, 0.6), (0, 0, 0), (0, 0, 0)],
         cvs=[(CV_PCA, [0, 1], [0.0] * 6 + [0.6, 0.8, 0.0, -0.8, 0.6, 0.0])], grad=[1.0],
         forces={0: (-0.6, -0.8, 0.0), 1: (0.8, -0.6, 0.0)}),
]
