"""ORACLE — test infrastructure only.

Drives the reference's own kernels, compiled for the host by ``build_ref.py``
into ``oracle/_ref/``, with the same plan layout as ``oracle.OracleSystem``
(platforms/common/src/CommonGluedKernels.cpp:3935-4577 for the layout,
:4736-5048 for the execute order, :5050-5157 for deposition). Used to pin the
restatement in ``glued_oracle.cpp`` and, when present, as the CPU baseline
("kind": "reference"). ``RefSystem.available()`` is False where the reference
tree was not present at build time.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from oracle import (OracleSystem, CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION,
                    CV_COORDINATION, CV_RMSD, CV_PATH, CV_CONTACTMAP, CV_PCA, BIAS_HARMONIC,
                    BIAS_METAD, BIAS_OPES, BIAS_PBMETAD, BIAS_EXTERNAL)

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def ref_lib(mode):
    path = os.path.join(HERE, "_ref", f"libglued_ref_{mode}.so")
    if mode not in _libs:
        _libs[mode] = ctypes.CDLL(path)
    return _libs[mode]


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


_I, _F, _D, _UL = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_ulonglong


class RefSystem(OracleSystem):
    """OracleSystem whose CV, bias, scatter and deposit steps call the compiled
    reference kernels instead of the restatement."""

    @staticmethod
    def available():
        return all(os.path.exists(os.path.join(HERE, "_ref", f"libglued_ref_{m}.so")) for m in ("f32", "f64"))

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self.real = ctypes.c_float if self.mode == "f32" else ctypes.c_double
        self.np_real = np.float32 if self.mode == "f32" else np.float64

        class R4(ctypes.Structure):
            _fields_ = [("x", self.real), ("y", self.real), ("z", self.real), ("w", self.real)]
        self.R4 = R4
        self.L = ref_lib(self.mode)

    def _box_args(self, box):
        b = np.eye(3) * 1e6 if box is None else np.asarray(box, float).reshape(3, 3)
        R4 = self.R4
        size = R4(b[0, 0], b[1, 1], b[2, 2], 0)
        inv = R4(1.0 / b[0, 0], 1.0 / b[1, 1], 1.0 / b[2, 2], 0)
        return [size, inv, R4(*b[0], 0), R4(*b[1], 0), R4(*b[2], 0)]

    def evaluate_cvs(self, pos, box=None):
        L = self.L
        pos = np.asarray(pos, float).reshape(-1, 3)
        posq = np.zeros((len(pos), 4), self.np_real)
        posq[:, :3] = pos
        P = posq.ctypes.data_as(ctypes.POINTER(self.R4))
        n = max(1, self.num_jac)
        ja = np.zeros(n, np.int32); jc = np.zeros(n, np.int32)
        jx = np.zeros(n, np.float32); jy = np.zeros(n, np.float32); jz = np.zeros(n, np.float32)
        J = [_p(ja, _I), _p(jx, _F), _p(jy, _F), _p(jz, _F), _p(jc, _I)]
        cvv = np.zeros(max(1, self.num_cvs))
        C = _p(cvv, _D)
        boxa = self._box_args(box)
        per = 1 if self.periodic else 0
        k = self.kinds
        for t, fn, na in ((CV_DISTANCE, "cvDistance", 2), (CV_ANGLE, "cvAngle", 3), (CV_DIHEDRAL, "cvDihedral", 4)):
            if k[t].n:
                a = np.array([x for at, p in k[t].atoms for x in at[:na]], np.int32)
                getattr(L, fn)(P, _p(a, _I), k[t].n, k[t].cv0, self.jac0[t], C, *J, *boxa, per)
        for t, fn in ((CV_COM_DISTANCE, "cvCOMDistance"), (CV_GYRATION, "cvGyration")):
            if not k[t].n:
                continue
            off, atoms, m, tm = [0], [], [], []
            for at, p in k[t].atoms:
                if t == CV_COM_DISTANCE:
                    ng1 = int(round(p[0])) if p else 1
                    g1, g2 = at[:ng1], at[ng1:]
                    off += [off[-1] + len(g1), off[-1] + len(g1) + len(g2)]
                    tm += [np.float32(sum(np.float32(self.masses[a]) for a in g1)),
                           np.float32(sum(np.float32(self.masses[a]) for a in g2))]
                else:
                    off.append(off[-1] + len(at))
                    tm.append(np.float32(sum(np.float32(self.masses[a]) for a in at)))
                atoms += at
                m += [self.masses[a] for a in at]
            getattr(L, fn)(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                           _p(np.array(m, np.float32), _F), _p(np.array(tm, np.float32), _F),
                           k[t].n, k[t].cv0, self.jac0[t], C, *J, *boxa, per)
        if k[CV_COORDINATION].n:
            off, atoms, prm = [0], [], []
            cur = 0
            off = []
            for at, p in k[CV_COORDINATION].atoms:
                grp = at[1:]
                off += [cur, cur + at[0]]
                cur += len(grp)
                atoms += grp
                prm += p[:3]
            off.append(cur)
            L.cvCoordination(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                             _p(np.array(prm, np.float32), _F), k[CV_COORDINATION].n, k[CV_COORDINATION].cv0,
                             self.jac0[CV_COORDINATION], C, *J, *boxa, per)
        if k[CV_RMSD].n:
            off, atoms, ref = [0], [], []
            for at, p in k[CV_RMSD].atoms:
                off.append(off[-1] + len(at)); atoms += at; ref += p[:3 * len(at)]
            L.cvRMSD(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                     _p(np.array(ref, np.float32), _F), k[CV_RMSD].n, k[CV_RMSD].cv0, self.jac0[CV_RMSD],
                     C, *J, *boxa, per)
        if k[CV_PATH].n:
            off, atoms, roff, ref, prm = [0], [], [], [], []
            rb = 0
            for at, p in k[CV_PATH].atoms:
                N = int(p[1]); M = len(at)
                off.append(off[-1] + M); atoms += at; roff.append(rb); rb += N * M
                prm += [p[0], p[1]]; ref += p[2:2 + 3 * N * M]
            roff.append(rb)
            L.cvPath(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                     _p(np.array(roff, np.int32), _I), _p(np.array(ref, np.float32), _F),
                     _p(np.array(prm, np.float32), _F), k[CV_PATH].n, k[CV_PATH].cv0, self.jac0[CV_PATH],
                     C, *J, *boxa, per)
        if k[CV_CONTACTMAP].n:
            off, pairs, prm = [0], [], []
            for at, p in k[CV_CONTACTMAP].atoms:
                npair = len(at) // 2
                off.append(off[-1] + npair); pairs += at[:2 * npair]; prm += p[:4 * npair]
            L.cvContactMap(P, _p(np.array(off, np.int32), _I), _p(np.array(pairs, np.int32), _I),
                           _p(np.array(prm, np.float32), _F), k[CV_CONTACTMAP].n, k[CV_CONTACTMAP].cv0,
                           self.jac0[CV_CONTACTMAP], C, *J, *boxa, per)
        if k[CV_PCA].n:
            off, atoms, ref, ev = [0], [], [], []
            for at, p in k[CV_PCA].atoms:
                N = len(at)
                off.append(off[-1] + N); atoms += at; ref += p[:3 * N]; ev += p[3 * N:6 * N]
            L.cvPCA(P, _p(np.array(off, np.int32), _I), _p(np.array(atoms, np.int32), _I),
                    _p(np.array(ref, np.float32), _F), _p(np.array(ev, np.float32), _F), k[CV_PCA].n,
                    k[CV_PCA].cv0, self.jac0[CV_PCA], C, *J, 0)
        jac = (ja, jx.astype(np.float64), jy.astype(np.float64), jz.astype(np.float64), jc)
        return cvv[:self.num_cvs].copy(), jac

    def evaluate_biases(self, cvv):
        L = self.L
        grad = np.zeros(max(1, self.num_cvs))
        nslot = max(1, len(self.biases))
        energies = np.zeros(nslot)
        cvv = np.ascontiguousarray(np.resize(cvv, max(1, self.num_cvs)), dtype=np.float64)
        C, G, E = _p(cvv, _D), _p(grad, _D), _p(energies, _D)
        for typ in (BIAS_HARMONIC, BIAS_OPES, BIAS_METAD, BIAS_PBMETAD, BIAS_EXTERNAL):
            for st in self.bias_state:
                if st["type"] != typ:
                    continue
                idx = st["idx"]
                if typ == BIAS_HARMONIC:
                    L.harmonicEvalBias(C, _p(idx, _I), _p(st["prm"], _F), st["D"], G, E, st["slot"], st["periodic"])
                elif typ == BIAS_OPES:
                    nk = np.array([st["ist"][0]], np.int32)
                    su = np.array([st["dst"][0]]); sw = np.array([st["dst"][1]])
                    L.opesEvalBias(C, _p(idx, _I), _p(st["centers"], _D), _p(st["sigmas"], _D), _p(st["logw"], _D),
                                   _p(nk, _I), st["D"], _D(st["invGF"]), _D(st["kT"]), _p(su, _D), _p(sw, _D),
                                   _D(st["cut2"]), _D(st["eps"]), _D(st["barrier"]), G, E, st["slot"])
                elif typ == BIAS_PBMETAD:
                    # pbmetaDSubgridEval per sub-grid, then pbmetaDCombine
                    N = st["D"]
                    le, lg = np.zeros(N), np.zeros(N)
                    for d in range(N):
                        o = int(st["goff"][d])
                        sub = st["grid"][o:o + int(st["npts"][d])]
                        L.pbmetaDSubgridEval(C, _p(idx[d:d + 1], _I), _p(sub, _D), _p(st["origin"][d:d + 1], _D),
                                             _p(st["inv"][d:d + 1], _D), _p(st["npts"][d:d + 1], _I),
                                             _p(st["per"][d:d + 1], _I), _p(le, _D), _p(lg, _D), d)
                    L.pbmetaDCombine(_p(le, _D), _p(lg, _D), _p(idx, _I), N, _D(st["kT"]), E, st["slot"], G,
                                     _p(st["W"], _D))
                    st["V"][:] = le
                else:
                    L.metaDEvalBias(C, _p(idx, _I), _p(st["grid"], _D), _p(st["origin"], _D), _p(st["inv"], _D),
                                    _p(st["npts"], _I), _p(st["strides"], _I), _p(st["per"], _I), st["D"], G, E,
                                    st["slot"])
        return energies, grad[:self.num_cvs]

    def execute(self, pos, box=None):
        cvv, jac = self.evaluate_cvs(pos, box)
        if self.test_grad is not None:
            grad = np.array(self.test_grad, float)
            energies = np.zeros(max(1, len(self.biases)))
        else:
            energies, grad = self.evaluate_biases(cvv)
        n = self.num_particles
        fbuf = np.zeros(3 * n, np.uint64)
        ja, jx, jy, jz, jc = jac
        g = np.ascontiguousarray(np.resize(grad, max(1, self.num_cvs)), dtype=np.float64)
        fx, fy, fz = (np.ascontiguousarray(a, dtype=np.float32) for a in (jx, jy, jz))
        self.L.chainRuleScatter(_p(g, _D), _p(ja, _I), _p(fx, _F), _p(fy, _F), _p(fz, _F), _p(jc, _I),
                                _p(fbuf, _UL), n, self.num_jac)
        self.cv_values = cvv
        self.bias_energies = energies
        self.cv_ready = True
        fb = fbuf.view(np.int64)
        forces = fb.reshape(3, n).T.astype(np.float64) / 4294967296.0
        return dict(energy=float(energies.sum()), forces=forces, force_fixed=fb.reshape(3, n),
                    cv_values=cvv, dUdCV=grad, jacobian=jac, bias_energies=energies)

    def update_state(self, step):
        L = self.L
        if not self.cv_ready or step == self.last_update_step:
            return
        self.last_update_step = step
        cvv = np.ascontiguousarray(self.cv_values, dtype=np.float64)
        C = _p(cvv, _D)
        E = np.ascontiguousarray(self.bias_energies, dtype=np.float64)
        for st in self.bias_state:
            if st["type"] != BIAS_OPES or step == 0 or step % st["pace"] != 0:
                continue
            if st["nker_cpu"] >= st["maxk"]:
                continue
            nk = np.array([st["ist"][0]], np.int32); ns = np.array([st["ist"][1]], np.int32)
            sc = np.array([st["ist"][2]], np.int32); na = np.array([st["ist"][3]], np.int32)
            su = np.array([st["dst"][0]]); swt = np.array([st["dst"][1]]); sw = np.array(st["dst"][2:4])
            before = int(nk[0])
            L.opesGatherDeposit(C, _p(st["idx"], _I), _p(st["mean"], _D), _p(st["m2"], _D), _p(ns, _I),
                                _p(st["sigma0"], _D), _D(st["smin"]), _p(st["centers"], _D), _p(st["sigmas"], _D),
                                _p(st["logw"], _D), _p(su, _D), _p(nk, _I), st["D"], st["variant"], st["astride"],
                                _p(E, _D), st["slot"], _D(1.0 / st["kT"]), _p(swt, _D), _D(st["cut2"]),
                                _p(sw, _D), _p(sc, _I), _p(na, _I), st["maxk"], _D(st["gamma"]),
                                _D(st["barrier"]))
            st["ist"][:] = [nk[0], ns[0], sc[0], na[0]]
            st["dst"][:] = [su[0], swt[0], sw[0], sw[1]]
            st["decisions"].append(-1 if nk[0] > before else -4)
            if st["astride"] == 0 or st["nsamp_cpu"] >= st["astride"]:
                st["nker_cpu"] += 1
        for st in self.bias_state:
            if st["type"] != BIAS_METAD or step == 0 or step % st["pace"] != 0:
                continue
            center = np.array([cvv[i] for i in st["idx"]])
            sig = np.ascontiguousarray(st["sigma"], dtype=np.float64)
            L.metaDDeposit(_p(st["grid"], _D), _p(st["origin"], _D), _p(st["inv"], _D), _p(st["npts"], _I),
                           _p(st["strides"], _I), _p(st["per"], _I), st["D"], st["total"], _p(center, _D),
                           _p(sig, _D), _p(E, _D), st["slot"], _D(st["h0"]), _D(st["hif"]))
            st["deposited"] += 1
        for st in self.bias_state:
            if st["type"] != BIAS_PBMETAD or step == 0 or step % st["pace"] != 0:
                continue
            for d in range(st["D"]):
                o, n = int(st["goff"][d]), int(st["npts"][d])
                sub = np.ascontiguousarray(st["grid"][o:o + n])
                center = np.array([cvv[st["idx"][d]]])
                sig = np.array([st["sigma"][d]])
                L.pbmetaDDeposit(_p(sub, _D), _p(st["origin"][d:d + 1], _D), _p(st["inv"][d:d + 1], _D),
                                 _p(st["npts"][d:d + 1], _I), _p(st["per"][d:d + 1], _I), n, _p(center, _D),
                                 _p(sig, _D), _p(st["V"], _D), d, _D(st["h0"]), _D(st["hif"]), _p(st["W"], _D))
                st["grid"][o:o + n] = sub
            st["deposited"] = [k + 1 for k in st["deposited"]]
