"""ORACLE — test infrastructure only. Checker helpers that compare the product's
outputs on the benchmark workloads with the FP64 oracle (``oracle.OracleSystem``
in ``mode='f64'``). Used by ``tests/`` and by ``bench.py``'s correctness check,
which runs outside the timed region; nothing here is measured or shipped.

Error measures (the acceptance gate of the workloads):

* force: ||F - F_ref||_inf / ||F_ref||_inf over all atoms and components;
* energy: |E - E_ref| / max(1, |E_ref|);
* CV: max_k |s_k - s_ref,k| / max(1, |s_ref,k|).
"""
from __future__ import annotations

import numpy as np

import oracle as O


def rel_energy_err(e, e_ref):
    return abs(float(e) - float(e_ref)) / max(1.0, abs(float(e_ref)))


def rel_cv_err(cv, cv_ref):
    cv = np.asarray(cv, float).ravel()
    cv_ref = np.asarray(cv_ref, float).ravel()
    if cv.size == 0:
        return 0.0
    return float(np.max(np.abs(cv - cv_ref) / np.maximum(1.0, np.abs(cv_ref))))


def summary(errs, what):
    """Worst case over a list of per-walker / per-system error dicts."""
    return {"max_rel_force_err": max(e["force"] for e in errs),
            "energy_rel_err": max(e["energy"] for e in errs),
            "cv_rel_err": max(e["cv"] for e in errs),
            "oracle": "FP64 (oracle/glued_oracle.cpp, double)", "checked": what}


# ----------------------------------------------------------- single systems
IN_SCOPE_BIASES = (O.BIAS_HARMONIC, O.BIAS_METAD, O.BIAS_PBMETAD, O.BIAS_OPES, O.BIAS_EXTERNAL,
                   O.BIAS_METAD_HILLS)


def single_oracle(w):
    """FP64 oracle of a single-system workload (C1 / C2 / C3 of gluedmd_b200.workloads)
    with its bias state loaded from the workload's blob."""
    biases = [b for b in w.biases if b[0] in IN_SCOPE_BIASES]
    s = O.OracleSystem(w.cvs, biases, masses=w.masses, periodic=w.pbc, mode="f64",
                       num_particles=len(w.positions))
    if w.blob:
        s.load_blob(w.blob)
    return s


def check_single(w, energy, forces, cv_values):
    r = single_oracle(w).execute(np.asarray(w.positions, float), np.asarray(w.box, float).ravel())
    return {"force": O.max_rel_force_err(forces, r["forces"]), "energy": rel_energy_err(energy, r["energy"]),
            "cv": rel_cv_err(cv_values, r["cv_values"]), "ref": r}


# ------------------------------------------------------- batched walkers (C4)
def walker_oracle(w, biases, centers, heights):
    """FP64 oracle of one walker of the 64-walker workload with the shared hill
    table (centres (K, 2), heights (K,)) loaded into its hill-sum MetaD."""
    s = O.OracleSystem(w["cvs"], biases, masses=w["masses"], periodic=True, mode="f64", num_particles=w["n"])
    for st in s.bias_state:
        if st["type"] == O.BIAS_METAD_HILLS:
            st["centers"] = np.array(centers, float).reshape(-1, 2)
            st["heights"] = np.array(heights, float)
    return s


def check_walker(w, biases, centers, heights, energy, forces, cv_values):
    r = walker_oracle(w, biases, centers, heights).execute(w["pos"], np.asarray(w["box"], float).ravel())
    return {"force": O.max_rel_force_err(forces, r["forces"]), "energy": rel_energy_err(energy, r["energy"]),
            "cv": rel_cv_err(cv_values, r["cv_values"]), "ref": r}


# ------------------------------------------------- differentiable bias (C5)
def c5_reference(pos, pairs, r0, patoms, frames, lam, centers, heights, sigma):
    """FP64 energy and forces of the C5 bias: the oracle's contact-map and path-CV
    values and Jacobians combined with dE/dCV of the 2-D hill sum on (CMAP, s).
    r0, frames and lambda are rounded to float first, as the reference stores them."""
    r0 = np.asarray(r0, np.float32).astype(np.float64)
    frames = np.asarray(frames, np.float32).astype(np.float64)
    lam = float(np.float32(lam))
    P = len(pairs)
    cm_params = [v for i in range(P) for v in (r0[i], 6.0, 12.0, 1.0)]
    cvs = [(O.CV_CONTACTMAP, [int(x) for x in np.asarray(pairs).ravel()], cm_params),
           (O.CV_PATH, [int(x) for x in patoms], [lam, len(frames)] + list(np.asarray(frames).ravel()))]
    sysm = O.OracleSystem(cvs, mode="f64", num_particles=len(pos), test_bias_gradients=[0.0, 0.0, 0.0])
    cvv, _ = sysm.evaluate_cvs(pos)
    d0 = cvv[0] - centers[:, 0]
    d1 = cvv[1] - centers[:, 1]
    g = heights * np.exp(-d0 ** 2 / (2 * sigma[0] ** 2) - d1 ** 2 / (2 * sigma[1] ** 2))
    sysm.test_grad = np.array([(-g * d0 / sigma[0] ** 2).sum(), (-g * d1 / sigma[1] ** 2).sum(), 0.0])
    r = sysm.execute(pos)
    return float(g.sum()), r["forces"], cvv
