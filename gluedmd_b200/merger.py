"""Parse, repack and merge 'GPUS' v1 bias-state blobs across walker groups.

Host-side counterpart of GLUED's ``BiasStateMerger``
(python/MultiGPUManager.py:132-716), with the same static methods
(``merge_additive``, ``merge_additive_incremental``, ``_parse``, ``_pack``,
``_merge_opes``, ``_merge_opes_expanded``) and the same parsed-dict keys, so
multi-group tooling written against the reference runs unchanged.

Layout (platforms/common/src/CommonSerialization.cpp:20-177): optional header
'GPUS' + int32 version, then OPES, ABMD, MetaD, PBMetaD, the stateless
EXTERNAL / LINEAR / WALL counts, OPES_EXPANDED, extended Lagrangian, EDS,
MaxEnt and OPES multithermal sections, each an int32 count followed by its
entries. Every section after OPES may be absent (older blobs).

Differences from the reference helper:
* the OPES multithermal section (written by the C++ serializer, skipped by the
  reference's Python parser) is parsed and repacked, and so is the 'HILL'
  section that this library appends for its hill-sum MetaD extension, so
  ``_pack(_parse(blob)) == blob`` for every blob this library writes;
* MetaD grid sizes follow the parameter layout the bias setup reads
  (``[pace, bins_0 .. bins_{D-1}, periodic_0 .. periodic_{D-1}]``,
  CommonBiasKernels.cpp:206-257); the reference helper reads an interleaved
  ``[pace, bins_0, periodic_0, ...]`` layout, which agrees only for 1-D grids;
* the hill tables of the hill-sum extension merge as a union: every group's
  hills deposited since its baseline are appended to the shared table.
"""
from __future__ import annotations

import math
import struct
from typing import List, Optional

import numpy as np

BIAS_METAD, BIAS_PBMETAD, BIAS_OPES, BIAS_ABMD = 3, 4, 5, 7
BIAS_OPES_EXPANDED, BIAS_EXT_LAGRANGIAN, BIAS_MAXENT, BIAS_EDS = 11, 12, 13, 14
BIAS_OPES_MULTITHERMAL = 15
BIAS_METAD_HILLS = 103

_HILL_TAG = b"HILL"


def _config(force):
    """Per-bias sizes the blob does not store, from the force's bias list."""
    cfg = dict(opes=[], abmd=[], metad=[], pbmetad=[], eds=[], maxent=[], ext_lag=[], opes_expanded=0,
               multithermal=[], hills=[])
    if force is None:
        return cfg
    for i in range(force.getNumBiases()):
        btype, cvs, params, ip = force.getBiasParameters(i)
        D = len(cvs)
        if btype == BIAS_OPES:
            cfg["opes"].append(D)
        elif btype == BIAS_ABMD:
            cfg["abmd"].append(D)
        elif btype == BIAS_METAD:
            G = 1
            for d in range(D):
                G *= ip[1 + d] + (0 if ip[1 + D + d] else 1)
            cfg["metad"].append(G)
        elif btype == BIAS_PBMETAD:
            cfg["pbmetad"].append([ip[1 + 2 * d] + (0 if ip[2 + 2 * d] else 1) for d in range(D)])
        elif btype == BIAS_EDS:
            cfg["eds"].append(D)
        elif btype == BIAS_MAXENT:
            cfg["maxent"].append(D)
        elif btype == BIAS_EXT_LAGRANGIAN:
            cfg["ext_lag"].append(D)
        elif btype == BIAS_OPES_EXPANDED:
            cfg["opes_expanded"] += 1
        elif btype == BIAS_OPES_MULTITHERMAL:
            cfg["multithermal"].append(None)
        elif btype == BIAS_METAD_HILLS:
            cfg["hills"].append(D)
    return cfg


def _grid(b):
    return np.frombuffer(bytes(b), dtype="<f8")


def _fold(cur, nd_cur, base, nd_base, shared, nd_shared):
    """shared + sum_g (cur_g - base_g), or sum_g cur_g without baselines."""
    if base is None:
        return sum(_grid(c) for c in cur), int(sum(nd_cur))
    out = _grid(shared).copy()
    nd = nd_shared
    for g in range(len(cur)):
        out = out + (_grid(cur[g]) - _grid(base[g]))
        nd += nd_cur[g] - nd_base[g]
    return out, int(nd)


class BiasStateMerger:
    """Parse, inspect and merge ``getBiasState()`` blobs (see the module docstring)."""

    @staticmethod
    def merge_additive(blobs: List[bytes], force) -> bytes:
        """Full additive merge: MetaD / PBMetaD grids and deposit counts summed, OPES
        kernel lists united with combined Welford statistics, OPES_EXPANDED logZ
        averaged by update counts, hill tables united; every other section from
        ``blobs[0]`` (python/MultiGPUManager.py:154-181)."""
        merged, _ = BiasStateMerger.merge_additive_incremental(blobs, force, baselines=None)
        return merged

    @staticmethod
    def merge_additive_incremental(blobs: List[bytes], force, baselines: Optional[list] = None):
        """Incremental additive merge (python/MultiGPUManager.py:184-302).

        Per grid cell: ``new_shared = shared + sum_g (G_g_now - G_g_baseline)``,
        with ``shared = baselines[0]`` (every group received the same state at the
        last sync); deposit counts fold the same way. Without usable baselines
        (None, or a different number of groups) the grids are summed in full.
        Returns ``(merged_blob, new_baselines)``: one parsed copy of the merged
        state per group, to pass back at the next sync.
        """
        if len(blobs) == 0:
            raise ValueError("no blobs to merge")
        if len(blobs) == 1:
            return blobs[0], [BiasStateMerger._parse(blobs[0], force)]
        parsed = [BiasStateMerger._parse(b, force) for b in blobs]
        inc = baselines is not None and len(baselines) == len(parsed)
        result = dict(parsed[0])

        merged_metad = []
        for i in range(len(parsed[0]["metad"])):
            cur = [p["metad"][i][1] for p in parsed]
            ndc = [p["metad"][i][0] for p in parsed]
            if inc:
                g, nd = _fold(cur, ndc, [b["metad"][i][1] for b in baselines], [b["metad"][i][0] for b in baselines],
                              baselines[0]["metad"][i][1], baselines[0]["metad"][i][0])
            else:
                g, nd = _fold(cur, ndc, None, None, None, None)
            merged_metad.append((nd, g.tobytes()))
        result["metad"] = merged_metad

        merged_pb = []
        for bi in range(len(parsed[0]["pbmetad"])):
            subs = []
            for si in range(len(parsed[0]["pbmetad"][bi])):
                cur = [p["pbmetad"][bi][si][1] for p in parsed]
                ndc = [p["pbmetad"][bi][si][0] for p in parsed]
                if inc:
                    g, nd = _fold(cur, ndc, [b["pbmetad"][bi][si][1] for b in baselines],
                                  [b["pbmetad"][bi][si][0] for b in baselines],
                                  baselines[0]["pbmetad"][bi][si][1], baselines[0]["pbmetad"][bi][si][0])
                else:
                    g, nd = _fold(cur, ndc, None, None, None, None)
                subs.append((nd, g.tobytes()))
            merged_pb.append(subs)
        result["pbmetad"] = merged_pb

        if parsed[0]["opes"]:
            result["opes"] = BiasStateMerger._merge_opes(parsed, np)
        if parsed[0]["opes_expanded"]:
            result["opes_expanded"] = BiasStateMerger._merge_opes_expanded(parsed)
        if parsed[0]["hills"]:
            result["hills"] = BiasStateMerger._merge_hills(parsed, baselines if inc else None)

        merged = BiasStateMerger._pack(result)
        mp = BiasStateMerger._parse(merged, force)
        return merged, [mp for _ in parsed]

    @staticmethod
    def _merge_opes(parsed: List[dict], np_=np) -> List[tuple]:
        """Union of the walkers' OPES kernel lists (python/MultiGPUManager.py:308-387):
        kernels concatenated in walker order, sample counts summed, Welford mean
        and M2 combined pairwise (Chan et al.: d = mB - mA, m = mA + d nB/n,
        M2 = M2A + M2B + d^2 nA nB / n), logZ = log sum_k exp(logW_k) over the union."""
        out = []
        for bi in range(len(parsed[0]["opes"])):
            D = len(parsed[0]["opes"][bi][3]) // 8
            n_acc, mean_acc, m2_acc = 0, np_.zeros(D), np_.zeros(D)
            cen, sig, lw = [], [], []
            for p in parsed:
                nk, logz, ns, mb, m2b, cb, sb, lb = p["opes"][bi]
                cen.append(bytes(cb)); sig.append(bytes(sb)); lw.append(bytes(lb))
                if ns <= 0:
                    continue
                mg, m2g = _grid(mb), _grid(m2b)
                if n_acc == 0:
                    n_acc, mean_acc, m2_acc = int(ns), mg.copy(), m2g.copy()
                else:
                    tot = n_acc + ns
                    d = mg - mean_acc
                    mean_acc = mean_acc + d * (ns / tot)
                    m2_acc = m2_acc + m2g + (d * d) * (n_acc * ns / tot)
                    n_acc = tot
            nk_tot = sum(p["opes"][bi][0] for p in parsed)
            lw_cat = b"".join(lw)
            if nk_tot > 0:
                w = _grid(lw_cat)
                m = float(w.max())
                logz = m + float(np_.log(np_.exp(w - m).sum()))
            else:
                logz = float(parsed[0]["opes"][bi][1])
            out.append((int(nk_tot), logz, int(n_acc), mean_acc.tobytes(), m2_acc.tobytes(), b"".join(cen),
                        b"".join(sig), lw_cat))
        return out

    @staticmethod
    def _merge_opes_expanded(parsed: List[dict]) -> List[tuple]:
        """OPES_EXPANDED (python/MultiGPUManager.py:390-417): update counts summed,
        exp(logZ) averaged with the counts as weights (plain mean of logZ when no
        walker has updates)."""
        out = []
        for ei in range(len(parsed[0]["opes_expanded"])):
            ent = [p["opes_expanded"][ei] for p in parsed]
            tot = sum(int(nu) for _, nu in ent)
            if tot > 0:
                m = max(lz for lz, _ in ent)
                acc = sum(nu * math.exp(lz - m) for lz, nu in ent if nu > 0)
                out.append((m + math.log(acc / tot), tot))
            else:
                out.append((sum(lz for lz, _ in ent) / len(ent), 0))
        return out

    @staticmethod
    def _merge_hills(parsed: List[dict], baselines: Optional[list]) -> List[tuple]:
        """Hill tables of the hill-sum extension: the shared table (baselines[0], or
        nothing on a first sync) followed by each group's hills past its baseline."""
        out = []
        for hi in range(len(parsed[0]["hills"])):
            D = parsed[0]["hills"][hi][0]
            if baselines is None:
                parts = [p["hills"][hi] for p in parsed]
                n = sum(x[1] for x in parts)
                c = b"".join(x[2] for x in parts)
                h = b"".join(x[3] for x in parts)
            else:
                sh = baselines[0]["hills"][hi]
                n, c, h = sh[1], [sh[2]], [sh[3]]
                for g, p in enumerate(parsed):
                    k0 = baselines[g]["hills"][hi][1]
                    _, k, cg, hg = p["hills"][hi]
                    if k < k0:
                        raise ValueError(f"hill table {hi} of group {g} shrank since the last sync")
                    c.append(cg[8 * D * k0:]); h.append(hg[8 * k0:])
                    n += k - k0
                c, h = b"".join(c), b"".join(h)
            out.append((D, int(n), c, h))
        return out

    # -------------------------------------------------------------- format
    @staticmethod
    def _parse(blob: bytes, force) -> dict:
        """Blob -> dict keyed like the reference parser (python/MultiGPUManager.py:420-640),
        plus ``multithermal`` and ``hills``. Counts are checked against the force's
        bias list when one is given; sizes the blob does not store (D, grid points)
        come from it."""
        blob = bytes(blob)
        cfg = _config(force)
        pos = [0]

        def left():
            return len(blob) - pos[0]

        def take(n):
            if n < 0 or n > left():
                raise ValueError(f"bias-state blob truncated: needed {n} bytes at offset {pos[0]} "
                                 f"but only {left()} remain")
            out = blob[pos[0]:pos[0] + n]
            pos[0] += n
            return out

        def i32():
            return struct.unpack("<i", take(4))[0]

        def f64():
            return struct.unpack("<d", take(8))[0]

        def more():
            return left() > 0 and blob[pos[0]:pos[0] + 4] != _HILL_TAG

        def count(section, key_len):
            n = i32()
            if key_len and n != key_len:
                raise ValueError(f"bias-state {section} count mismatch: blob declares {n} but force config has "
                                 f"{key_len}")
            return n

        def dim(lst, i, section):
            if i >= len(lst):
                raise ValueError(f"cannot parse {section} bias without force config (need its size)")
            return lst[i]

        if len(blob) >= 8 and blob[:4] == b"GPUS":
            pos[0] = 4
            if i32() != 1:
                raise ValueError("unknown bias-state blob version")
        out = dict(opes=[], abmd=[], metad=[], pbmetad=[], n_external=0, n_linear=0, n_wall=0, opes_expanded=[],
                   ext_lag=[], eds=[], maxent=[], multithermal=[], hills=[])
        n = count("OPES", len(cfg["opes"]))
        for i in range(n):
            D = dim(cfg["opes"], i, "OPES")
            nk, logz, ns = i32(), f64(), i32()
            out["opes"].append((nk, logz, ns, take(8 * D), take(8 * D), take(8 * nk * D), take(8 * nk * D),
                                take(8 * nk)))
        if more():
            for i in range(count("ABMD", len(cfg["abmd"]))):
                out["abmd"].append(take(8 * dim(cfg["abmd"], i, "ABMD")))
        if more():
            for i in range(count("MetaD", len(cfg["metad"]))):
                G = dim(cfg["metad"], i, "MetaD")
                nd = i32()
                out["metad"].append((nd, take(8 * G)))
        if more():
            for i in range(count("PBMetaD", len(cfg["pbmetad"]))):
                sizes = dim(cfg["pbmetad"], i, "PBMetaD")
                ns = i32()
                if ns != len(sizes):
                    raise ValueError(f"PBMetaD bias {i} sub-grid count mismatch: blob declares {ns} but force "
                                     f"config has {len(sizes)}")
                subs = []
                for G in sizes:
                    nd = i32()
                    subs.append((nd, take(8 * G)))
                out["pbmetad"].append(subs)
        for key in ("n_external", "n_linear", "n_wall"):
            if more():
                out[key] = i32()
        if more():
            n = i32()
            if cfg["opes_expanded"] and n != cfg["opes_expanded"]:
                raise ValueError(f"bias-state OPES_EXPANDED count mismatch: blob declares {n} but force config "
                                 f"has {cfg['opes_expanded']}")
            for _ in range(n):
                lz = f64()
                out["opes_expanded"].append((lz, i32()))
        if more():
            for i in range(count("EXT_LAGRANGIAN", len(cfg["ext_lag"]))):
                D = dim(cfg["ext_lag"], i, "EXT_LAGRANGIAN")
                out["ext_lag"].append((take(8 * D), take(8 * D)))
        if more():
            for i in range(count("EDS", len(cfg["eds"]))):
                D = dim(cfg["eds"], i, "EDS")
                out["eds"].append((take(8 * D), take(8 * D), take(8 * D), take(8 * D), take(4 * D)))
        if more():
            for i in range(count("MAXENT", len(cfg["maxent"]))):
                out["maxent"].append(take(8 * dim(cfg["maxent"], i, "MAXENT")))
        if more():
            # CommonSerialization.cpp:164-176: N, delta-F[N], rct, counter
            for _ in range(count("OPES multithermal", len(cfg["multithermal"]))):
                N = i32()
                out["multithermal"].append((N, take(8 * N), take(8), take(8)))
        if left() >= 8 and blob[pos[0]:pos[0] + 4] == _HILL_TAG:
            pos[0] += 4
            for i in range(count("hill-sum", len(cfg["hills"]))):
                D = dim(cfg["hills"], i, "hill-sum")
                k = i32()
                out["hills"].append((D, k, take(8 * k * D), take(8 * k)))
        return out

    @staticmethod
    def _pack(d: dict) -> bytes:
        """Parsed dict -> 'GPUS' v1 blob, sections in serializer order; the hill
        section only when the dict holds hill tables."""
        buf = bytearray(b"GPUS")
        i32 = lambda v: buf.extend(struct.pack("<i", int(v)))  # noqa: E731
        f64 = lambda v: buf.extend(struct.pack("<d", float(v)))  # noqa: E731
        i32(1)
        i32(len(d["opes"]))
        for nk, logz, ns, mb, m2b, cb, sb, lb in d["opes"]:
            i32(nk); f64(logz); i32(ns)
            for b in (mb, m2b, cb, sb, lb):
                buf.extend(b)
        i32(len(d["abmd"]))
        for b in d["abmd"]:
            buf.extend(b)
        i32(len(d["metad"]))
        for nd, g in d["metad"]:
            i32(nd); buf.extend(g)
        i32(len(d["pbmetad"]))
        for subs in d["pbmetad"]:
            i32(len(subs))
            for nd, g in subs:
                i32(nd); buf.extend(g)
        i32(d.get("n_external", 0)); i32(d.get("n_linear", 0)); i32(d.get("n_wall", 0))
        i32(len(d["opes_expanded"]))
        for lz, nu in d["opes_expanded"]:
            f64(lz); i32(nu)
        i32(len(d["ext_lag"]))
        for s, p in d["ext_lag"]:
            buf.extend(s); buf.extend(p)
        i32(len(d["eds"]))
        for parts in d["eds"]:
            for b in parts:
                buf.extend(b)
        i32(len(d["maxent"]))
        for b in d["maxent"]:
            buf.extend(b)
        mt = d.get("multithermal", [])
        i32(len(mt))
        for N, dF, rct, cnt in mt:
            i32(N); buf.extend(dF); buf.extend(rct); buf.extend(cnt)
        hills = d.get("hills", [])
        if hills:
            buf.extend(_HILL_TAG)
            i32(len(hills))
            for _D, k, c, h in hills:
                i32(k); buf.extend(c); buf.extend(h)
        return bytes(buf)
