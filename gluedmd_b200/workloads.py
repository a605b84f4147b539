"""Seeded synthetic inputs for the five benchmark configurations.

Positions are drawn with numpy ``default_rng(seed)``; "water density" is 100
atoms/nm^3. Pre-deposited bias state (MetaD hills / grids, OPES kernel tables)
is produced here as *input data* and loaded through the bias-state blob
('GPUS' v1), the reference's own checkpoint format.

C1  plain WT-MetaD, 22 atoms, 2 dihedrals, 2,000 hills (grid and hill-sum forms)
C2  single walker, 20,000 atoms: coordination 2,048 x 8,192 + RMSD over 1,000
    atoms, 2-D MetaD grid (256 x 256) with 20,000 hills
C3  OPES-METAD on (COM distance, gyration) of 5,000 of 50,000 atoms,
    10,000 merge-free kernels
C4  64 walkers of 1k-50k atoms (log-uniform), distance/angle/dihedral and
    256 x 1,024 coordination per walker, shared 50,000-hill WT MetaD
C5  30,000 atoms: contact map of 10,000 pairs + path CV (50 frames x 500 atoms)
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

KT300 = 2.494338785
CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION = 1, 2, 3, 4, 5
CV_COORDINATION, CV_RMSD, CV_PATH, CV_CONTACTMAP = 6, 7, 10, 13
CV_COORDINATION_CUTOFF, CV_RMSD_KABSCH = 106, 107
BIAS_HARMONIC, BIAS_METAD, BIAS_PBMETAD, BIAS_OPES, BIAS_EXTERNAL, BIAS_METAD_HILLS = 1, 3, 4, 5, 6, 103


@dataclass
class Workload:
    name: str
    positions: np.ndarray          # (N, 3) nm
    box: np.ndarray                # (3, 3) nm
    cvs: list                      # (type, atoms, params)
    biases: list = field(default_factory=list)  # (type, cvIdx, params, intParams)
    masses: np.ndarray = None
    pbc: bool = True
    blob: bytes = b""              # bias state to load ('GPUS' v1)
    extra: dict = field(default_factory=dict)


def _cube(L):
    return np.diag([L, L, L]).astype(np.float64)


# ------------------------------------------------------------------ MetaD data
def wt_hill_heights(centers, sigma, period, h0, gamma, kT, chunk=512):
    """Sequential well-tempered heights: h_k = h0 exp(-V_{k-1}(c_k) / ((gamma-1) kT)),
    V_{k-1} the truncated (exponent <= 8) hill sum of the previous hills. O(K^2),
    blocked so that only the within-block part is sequential. Large tables use
    torch float64 (on the GPU when one is present)."""
    if len(centers) > 4000:
        try:
            return _wt_hill_heights_torch(centers, sigma, period, h0, gamma, kT)
        except ImportError:
            pass
    c = np.asarray(centers, float)
    K, D = c.shape
    sig = np.asarray(sigma, float)
    per = np.asarray(period, float)
    hif = 0.0 if gamma <= 1.0 else 1.0 / ((gamma - 1.0) * kT)
    h = np.zeros(K)

    def kern(a, b):
        d = a[:, None, :] - b[None, :, :]
        for k in range(D):
            if per[k] > 0:
                d[..., k] -= np.round(d[..., k] / per[k]) * per[k]
        ex = np.sum(d * d / (2.0 * sig * sig), axis=-1)
        return np.where(ex <= 8.0, np.exp(-ex), 0.0)

    for s in range(0, K, chunk):
        e = min(K, s + chunk)
        Vpre = kern(c[s:e], c[:s]) @ h[:s] if s > 0 else np.zeros(e - s)
        W = kern(c[s:e], c[s:e])
        for i in range(e - s):
            V = Vpre[i] + (W[i, :i] @ h[s:s + i] if i else 0.0)
            h[s + i] = h0 * math.exp(-V * hif) if hif > 0 else h0
    return h


def _wt_hill_heights_torch(centers, sigma, period, h0, gamma, kT, chunk=1024):
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    c = torch.as_tensor(np.asarray(centers, float), dtype=torch.float64, device=dev)
    K, D = c.shape
    sig = torch.as_tensor(np.asarray(sigma, float), dtype=torch.float64, device=dev)
    per = [float(x) for x in period]
    hif = 0.0 if gamma <= 1.0 else 1.0 / ((gamma - 1.0) * kT)
    h = torch.zeros(K, dtype=torch.float64, device=dev)

    def kern(a, b):
        d = a[:, None, :] - b[None, :, :]
        for k in range(D):
            if per[k] > 0:
                d[..., k] -= torch.round(d[..., k] / per[k]) * per[k]
        ex = (d * d / (2.0 * sig * sig)).sum(-1)
        return torch.where(ex <= 8.0, torch.exp(-ex), torch.zeros_like(ex))

    for s in range(0, K, chunk):
        e = min(K, s + chunk)
        Vpre = kern(c[s:e], c[:s]) @ h[:s] if s > 0 else torch.zeros(e - s, dtype=torch.float64, device=dev)
        Wm = kern(c[s:e], c[s:e]).cpu().numpy()
        Vp = Vpre.cpu().numpy()
        hb = np.zeros(e - s)
        for i in range(e - s):
            V = Vp[i] + (Wm[i, :i] @ hb[:i] if i else 0.0)
            hb[i] = h0 * math.exp(-V * hif) if hif > 0 else h0
        h[s:e] = torch.as_tensor(hb, dtype=torch.float64, device=dev)
    return h.cpu().numpy()


def grid_from_hills_windowed(centers, heights, sigma, origin, maxv, bins, periodic):
    """Same grid as grid_from_hills, touching only each hill's +-4 sigma window."""
    D = len(bins)
    assert D == 2
    npts = [bins[d] + (0 if periodic[d] else 1) for d in range(D)]
    inv = [bins[d] / (maxv[d] - origin[d]) for d in range(D)]
    grid = np.zeros((npts[1], npts[0]))
    wins = []
    for d in range(D):
        half = int(math.ceil(4.0 * sigma[d] * inv[d])) + 1
        wins.append(np.arange(-half, half + 1))
    for c, h in zip(np.asarray(centers, float), heights):
        idx, dcs = [], []
        for d in range(D):
            b0 = int(math.floor((c[d] - origin[d]) * inv[d]))
            bi = b0 + wins[d]
            if periodic[d]:
                bi = np.unique(bi % npts[d])
            else:
                bi = bi[(bi >= 0) & (bi < npts[d])]
            pos = origin[d] + bi / inv[d]
            dc = pos - c[d]
            if periodic[d]:
                L = npts[d] / inv[d]
                dc = dc - np.round(dc / L) * L
            idx.append(bi)
            dcs.append(dc * dc / (2.0 * sigma[d] * sigma[d]))
        ex = dcs[1][:, None] + dcs[0][None, :]
        grid[np.ix_(idx[1], idx[0])] += np.where(ex <= 8.0, h * np.exp(-ex), 0.0)
    return grid.ravel()


def grid_from_hills(centers, heights, sigma, origin, maxv, bins, periodic):
    """Dense column-major MetaD grid holding the given hills with the reference's
    deposit rule (exponent <= 8 truncation, nearest periodic image;
    CommonGluedKernels.cpp:3645-3680)."""
    D = len(bins)
    npts = [bins[d] + (0 if periodic[d] else 1) for d in range(D)]
    inv = [bins[d] / (maxv[d] - origin[d]) for d in range(D)]
    axes = [origin[d] + np.arange(npts[d]) / inv[d] for d in range(D)]
    grid = np.zeros(npts[::-1])  # index [iD-1, ..., i0] -> column-major flat
    for c, h in zip(np.asarray(centers, float), heights):
        ex = None
        for d in range(D):
            dc = axes[d] - c[d]
            if periodic[d]:
                L = npts[d] / inv[d]
                dc = dc - np.round(dc / L) * L
            t = dc * dc / (2.0 * sigma[d] * sigma[d])
            shape = [1] * D
            shape[D - 1 - d] = npts[d]
            t = t.reshape(shape)
            ex = t if ex is None else ex + t
        grid += np.where(ex <= 8.0, h * np.exp(-ex), 0.0)
    return grid.ravel()  # C order over reversed axes == column-major over (i0, i1, ...)


def blob(opes=(), metad=(), hills=(), pbmetad=(), n_external=0):
    """'GPUS' v1 bias-state blob (CommonSerialization.cpp:20-177 layout).
    opes   : list of dict(nk, sum_uprob, nsamples, mean, m2, centers, sigmas, logw)
    metad  : list of (numDeposited, grid)
    pbmetad: list of [(numDeposited, sub-grid), ...] per bias
    hills  : list of (centers (n,D), heights (n,)) -- extension section 'HILL'."""
    out = bytearray(b"GPUS") + struct.pack("<i", 1)
    out += struct.pack("<i", len(opes))
    for o in opes:
        out += struct.pack("<idi", int(o["nk"]), float(o["sum_uprob"]), int(o.get("nsamples", 0)))
        for key in ("mean", "m2", "centers", "sigmas", "logw"):
            out += np.ascontiguousarray(o[key], dtype="<f8").tobytes()
    out += struct.pack("<i", 0)  # ABMD
    out += struct.pack("<i", len(metad))
    for nd, g in metad:
        out += struct.pack("<i", int(nd)) + np.ascontiguousarray(g, dtype="<f8").tobytes()
    out += struct.pack("<i", len(pbmetad))
    for subs in pbmetad:
        out += struct.pack("<i", len(subs))
        for nd, g in subs:
            out += struct.pack("<i", int(nd)) + np.ascontiguousarray(g, dtype="<f8").tobytes()
    out += struct.pack("<8i", int(n_external), *([0] * 7))
    if hills:
        out += b"HILL" + struct.pack("<i", len(hills))
        for c, h in hills:
            out += struct.pack("<i", len(h)) + np.ascontiguousarray(c, dtype="<f8").tobytes() + \
                np.ascontiguousarray(h, dtype="<f8").tobytes()
    return bytes(out)


# ------------------------------------------------------------------- configs
def config1(form="grid", n_hills=2000, bins=256):
    """C1: 22 atoms in a 3 nm cube (seed 1), dihedrals (4,6,8,14),(6,8,14,16),
    2,000 WT hills (seed 2), sigma 0.35 rad, h0 1.2, gamma 10, kT(300 K)."""
    rng = np.random.default_rng(1)
    pos = rng.uniform(0.0, 3.0, (22, 3))
    cvs = [(CV_DIHEDRAL, [4, 6, 8, 14], []), (CV_DIHEDRAL, [6, 8, 14, 16], [])]
    hr = np.random.default_rng(2)
    centers = hr.uniform(-math.pi, math.pi, (n_hills, 2))
    sigma, h0, gamma = [0.35, 0.35], 1.2, 10.0
    heights = wt_hill_heights(centers, sigma, [2 * math.pi] * 2, h0, gamma, KT300)
    lo, hi = [-math.pi] * 2, [math.pi] * 2
    if form == "grid":
        params = [h0] + sigma + [gamma, KT300] + lo + hi
        ip = [500, bins, bins, 1, 1]
        biases = [(BIAS_METAD, [0, 1], params, ip)]
        g = grid_from_hills_windowed(centers, heights, sigma, lo, hi, [bins, bins], [1, 1])
        b = blob(metad=[(n_hills, g)])
    elif form == "pbmetad":
        # PBMETAD on the two dihedrals (two periodic 1-D sub-grids holding the
        # hills' projections, half height each) + an EXTERNAL grid equal to the
        # 2-D MetaD grid of the same hills
        params = [h0, gamma, KT300]
        for d in range(2):
            params += [sigma[d], lo[d], hi[d]]
        biases = [(BIAS_PBMETAD, [0, 1], params, [500, bins, 1, bins, 1])]
        subs = [(n_hills, grid_from_hills(centers[:, d:d + 1], 0.5 * heights, sigma[d:d + 1], lo[d:d + 1],
                                          hi[d:d + 1], [bins], [1])) for d in range(2)]
        g = grid_from_hills_windowed(centers, heights, sigma, lo, hi, [bins, bins], [1, 1])
        biases.append((BIAS_EXTERNAL, [0, 1], lo + hi + list(g), [bins, bins, 1, 1]))
        b = blob(pbmetad=[subs], n_external=1)
    else:
        params = [h0] + sigma + [gamma, KT300] + lo + hi
        ip = [500, n_hills + 100000, 1, 1]
        biases = [(BIAS_METAD_HILLS, [0, 1], params, ip)]
        b = blob(hills=[(centers, heights)])
    return Workload(f"C1-{form}", pos, _cube(3.0), cvs, biases, np.ones(22), True, b,
                    dict(centers=centers, heights=heights))


def coordination_cn_fp64(pos, A, B, box_len, r0=0.35, n=6, m=12, chunk=256, rc=0.0):
    """Reference-semantics CN in FP64 (no cutoff unless rc > 0), used to place the C2 grid."""
    cn = 0.0
    pa, pb = pos[A], pos[B]
    for s in range(0, len(A), chunk):
        d = pa[s:s + chunk, None, :] - pb[None, :, :]
        d -= np.floor(d / box_len + 0.5) * box_len
        r = np.sqrt((d * d).sum(-1))
        x = r / r0
        with np.errstate(divide="ignore", invalid="ignore"):
            f = (1 - x ** n) / (1 - x ** m)
        f = np.where(np.abs(x - 1) < 1e-4, n / m, f)
        keep = (r * r >= 1e-20) & (x <= 1000)
        if rc > 0:
            keep &= r * r < rc * rc
        cn += f[keep].sum()
    return cn


def _cn_axis(cn0, bins):
    """Grid bounds on (CN, RMSD): CN over [0.9, 1.1] cn0 shifted so that cn0 sits
    0.37 of a cell past a grid node (on a node, the interpolated bias has a kink
    there and the FP32 CN's last bits would pick one side's gradient or the
    other), RMSD over [0, 0.5]."""
    sp = 0.2 * cn0 / bins
    lo = cn0 * 0.9 - 0.37 * sp
    return [lo, 0.0], [lo + 0.2 * cn0, 0.5]


def config2(n_hills=20000, bins=256, with_bias=True, fit=False):
    """C2: 20,000 atoms at water density (5.9 nm cube, seed 3); coordination
    between the first 2,048 and next 8,192 atoms of a seeded permutation (r0 0.35,
    6/12, no cutoff); RMSD over 1,000 atoms vs pos + N(0, 0.1) (seed 4); 2-D MetaD
    on (CN, RMSD), 256 x 256 non-periodic grid, 20,000 hills (seed 5). fit: the
    RMSD after optimal superposition (Kabsch, FP64 quaternion eigensolve) instead
    of the reference's no-fit RMSD; workload "C2-kabsch"."""
    L = 5.9
    rng = np.random.default_rng(3)
    pos = rng.uniform(0.0, L, (20000, 3))
    perm = rng.permutation(20000)
    A, B = perm[:2048], perm[2048:2048 + 8192]
    R = perm[2048 + 8192:2048 + 8192 + 1000]
    ref = pos[R] + np.random.default_rng(4).normal(0.0, 0.1, (1000, 3))
    cvs = [(CV_COORDINATION, [2048] + list(A) + list(B), [0.35, 6, 12]),
           (CV_RMSD_KABSCH if fit else CV_RMSD, list(R), list(ref.ravel()))]
    extra = dict(A=A, B=B, R=R)
    if not with_bias:
        return Workload("C2-cv", pos, _cube(L), cvs, [], np.ones(20000), True, b"", extra)
    cn0 = coordination_cn_fp64(pos, A, B, L)
    rmsd0 = float(np.sqrt(((pos[R] - ref) ** 2).sum(-1).mean()))
    lo, hi = _cn_axis(cn0, bins)
    sigma = [0.02 * (hi[0] - lo[0]), 0.02 * (hi[1] - lo[1])]
    hr = np.random.default_rng(5)
    centers = np.stack([hr.uniform(lo[0], hi[0], n_hills), hr.uniform(lo[1], hi[1], n_hills)], 1)
    heights = wt_hill_heights(centers, sigma, [0.0, 0.0], 1.2, 10.0, KT300)
    g = grid_from_hills_windowed(centers, heights, sigma, lo, hi, [bins, bins], [0, 0])
    params = [1.2] + sigma + [10.0, KT300] + lo + hi
    biases = [(BIAS_METAD, [0, 1], params, [500, bins, bins, 0, 0])]
    extra.update(cn0=cn0, rmsd0=rmsd0)
    return Workload("C2-kabsch" if fit else "C2", pos, _cube(L), cvs, biases, np.ones(20000), True,
                    blob(metad=[(n_hills, g)]), extra)


def config2_cutoff(method=0, rc=1.2, box=5.9):
    """C2 with the coordination restricted to pairs closer than rc = 1.2 nm
    (CV_COORDINATION_CUTOFF, no reference counterpart): 2,048 x 8,192 coordination
    and the 1,000-atom RMSD of a seeded permutation of atoms at C2's density
    (97.4 nm^-3) in a cube of side `box` (5.9 nm: C2's own atoms), 256 x 256
    MetaD grid on (CN, RMSD) centred on this CN. method 0: all-pairs tiles with
    a cutoff mask; 1: cell-list pair search. Positions are FP32-exact (as OpenMM's
    posq holds them), so the FP64 oracle's cutoff decisions see the same
    coordinates as the GPU."""
    if box == 5.9:
        w = config2()
        pos, A, B, R = w.positions, w.extra["A"], w.extra["B"], w.extra["R"]
        rmsd_cv = w.cvs[1]
    else:
        n = int(round(20000 * (box / 5.9) ** 3))
        rng = np.random.default_rng(13)
        pos = rng.uniform(0.0, box, (n, 3))
        perm = rng.permutation(n)
        A, B, R = perm[:2048], perm[2048:2048 + 8192], perm[2048 + 8192:2048 + 8192 + 1000]
        ref = pos[R] + np.random.default_rng(4).normal(0.0, 0.1, (1000, 3))
        rmsd_cv = (CV_RMSD, list(R), list(ref.ravel()))
    pos = np.asarray(pos, np.float32).astype(np.float64)
    cvs = [(CV_COORDINATION_CUTOFF, [len(A)] + list(A) + list(B), [0.35, 6, 12, rc, float(method)]), rmsd_cv]
    cn0 = coordination_cn_fp64(pos, A, B, box, rc=rc)
    lo, hi = _cn_axis(cn0, 256)
    sigma = [0.02 * (hi[0] - lo[0]), 0.02 * (hi[1] - lo[1])]
    hr = np.random.default_rng(5)
    n_hills, bins = 20000, 256
    centers = np.stack([hr.uniform(lo[0], hi[0], n_hills), hr.uniform(lo[1], hi[1], n_hills)], 1)
    heights = wt_hill_heights(centers, sigma, [0.0, 0.0], 1.2, 10.0, KT300)
    g = grid_from_hills_windowed(centers, heights, sigma, lo, hi, [bins, bins], [0, 0])
    biases = [(BIAS_METAD, [0, 1], [1.2] + sigma + [10.0, KT300] + lo + hi, [500, bins, bins, 0, 0])]
    extra = dict(A=A, B=B, R=R, cn0=cn0, rc=rc)
    name = "C2-cutoff" + ("" if box == 5.9 else f"-{box:g}nm") + ("-tiles" if method == 0 else "-cells")
    return Workload(name, pos, _cube(box), cvs, biases, np.ones(len(pos)), True, blob(metad=[(n_hills, g)]), extra)


def _opes_pair_sum(centers, sigmas, logw, cutoff2, chunk=1024):
    """sum_uprob = sum_{j,k} h_k (G(c_j; c_k, s_k) - eps), eps = exp(-cutoff2/2)
    (CommonGluedKernels.cpp:2982-3002), blocked over j."""
    eps = math.exp(-0.5 * cutoff2)
    h = np.exp(logw)
    tot = 0.0
    for s in range(0, len(centers), chunk):
        d = (centers[s:s + chunk, None, :] - centers[None, :, :]) / sigmas[None, :, :]
        n2 = (d * d).sum(-1)
        tot += np.where(n2 < cutoff2, h[None, :] * (np.exp(-0.5 * n2) - eps), 0.0).sum()
    return tot


def _c3_cv_estimate(pos, sel, L):
    """(COM distance of the two halves of sel, gyration of sel) with unit masses,
    minimum-image displacements: the C3 CV values, used only to order the kernels."""
    half = len(sel) // 2
    d = pos[sel[half:]].mean(0) - pos[sel[:half]].mean(0)
    d -= np.round(d / L) * L
    c = pos[sel].mean(0)
    r = pos[sel] - c
    r -= np.round(r / L) * L
    return np.array([np.linalg.norm(d), math.sqrt((r * r).sum(1).mean())])


def config3(n_kernels=10000):
    """C3: 50,000 atoms at water density (8 nm cube, seed 6); a seeded 5,000-atom
    selection; CV1 = COM distance of its two 2,500-atom halves, CV2 = gyration of
    all 5,000. OPES-METAD (gamma = 50 kJ/mol / kT) with 10,000 kernels whose sigma
    is U[0.02, 0.2] nm (seed 7), centres placed so that no kernel lies within
    1 sigma (Mahalanobis, with the existing kernel's sigma) of another, i.e. the
    table is already compressed; log-weights from a seeded bias trace."""
    L = 8.0
    n = 50000
    rng = np.random.default_rng(6)
    pos = rng.uniform(0.0, L, (n, 3))
    sel = rng.permutation(n)[:5000]
    cvs = [(CV_COM_DISTANCE, list(sel), [2500]), (CV_GYRATION, list(sel), [])]
    kT = KT300
    gamma = 50.0 / kT
    kr = np.random.default_rng(7)
    sig = kr.uniform(0.02, 0.2, (n_kernels, 2))
    # centres on a jittered lattice wide enough for a merge-free table
    side = int(math.ceil(math.sqrt(n_kernels)))
    spacing = 0.45
    grid = np.stack(np.meshgrid(np.arange(side), np.arange(side), indexing="ij"), -1).reshape(-1, 2)[:n_kernels]
    centers = (grid - side / 2.0) * spacing + kr.uniform(-0.02, 0.02, (n_kernels, 2))
    centers += np.array([0.05, 4.0])
    # enforce merge-freeness exactly as the deposit tests it (n2 < 1 with kernel k's sigma)
    keep = np.ones(n_kernels, bool)
    for s in range(0, n_kernels, 1024):
        d = (centers[s:s + 1024, None, :] - centers[None, :, :]) / sig[None, :, :]
        n2 = (d * d).sum(-1)
        np.fill_diagonal(n2[:, s:s + 1024], np.inf)
        keep[s:s + 1024] &= ~(n2 < 1.0).any(1)
    centers, sig = centers[keep], sig[keep]
    # deposition order of a run converging on the current state: the kernels
    # nearest the initial CV values (in sigma units) come last and so carry the
    # largest log-weights, which makes the bias and its forces non-trivial there
    s0 = _c3_cv_estimate(pos, sel, L)
    order = np.argsort(-np.sqrt((((centers - s0) / sig) ** 2).sum(1)), kind="stable")
    centers, sig = centers[order], sig[order]
    nk = len(centers)
    trace = np.cumsum(kr.normal(0.0, 0.3, nk)) - 2.0 * gamma * kT * np.linspace(1, 0, nk)
    logw = trace / kT
    invGF = (gamma - 1.0) / gamma
    cut2 = 2.0 * gamma / invGF
    su = _opes_pair_sum(centers, sig, logw, cut2)
    params = [kT, gamma, 0.1, 0.1, 0.005]
    biases = [(BIAS_OPES, [0, 1], params, [0, 500, 100000])]
    b = blob(opes=[dict(nk=nk, sum_uprob=su, nsamples=nk, mean=np.zeros(2), m2=np.zeros(2),
                        centers=centers.ravel(), sigmas=sig.ravel(), logw=logw)])
    return Workload("C3", pos, _cube(L), cvs, biases, np.ones(n), True, b,
                    dict(sel=sel, centers=centers, sigmas=sig, logw=logw, sum_uprob=su, gamma=gamma))


def config4_walkers(n_walkers=64, n_hills=50000, coord=(256, 1024)):
    """C4: walker sizes log-uniform in [1,000, 50,000] (seed 8), boxes at water
    density, positions seeded per walker (seed 1000 + w). Per walker: distance,
    angle and dihedral on seeded atoms and a 256 x 1,024 coordination (groups may
    overlap in walkers smaller than 1,280 atoms; identical-atom pairs are skipped
    by the r^2 < 1e-20 rule). Distance and coordination carry harmonic restraints
    (k = 100) whose centres config4_restraints places just off the initial values.
    All walkers share one WT hill-sum MetaD on
    (dihedral, angle): 50,000 hills, centres U over [-pi, pi) x [0, pi] (seed 9),
    sigma 0.35 rad, h0 1.2, gamma 10, kT(300 K), heights by the WT recursion."""
    sizes = np.exp(np.random.default_rng(8).uniform(math.log(1000), math.log(50000), n_walkers)).astype(int)
    walkers = []
    nA, nB = coord
    for w, n in enumerate(sizes):
        rng = np.random.default_rng(1000 + w)
        L = (n / 100.0) ** (1.0 / 3.0)
        pos = rng.uniform(0.0, L, (n, 3))
        quad = rng.choice(n, 4, replace=False)
        A = rng.choice(n, nA, replace=False)
        B = rng.choice(n, nB, replace=False)
        d0 = float(np.linalg.norm(pos[quad[1]] - pos[quad[0]]))
        cvs = [(CV_DISTANCE, [int(quad[0]), int(quad[1])], []),
               (CV_ANGLE, [int(quad[0]), int(quad[1]), int(quad[2])], []),
               (CV_DIHEDRAL, [int(x) for x in quad], []),
               (CV_COORDINATION, [nA] + [int(x) for x in A] + [int(x) for x in B], [0.35, 6, 12])]
        walkers.append(dict(n=int(n), L=L, pos=pos, cvs=cvs, box=_cube(L), masses=np.ones(n), d0=d0,
                            A=A, B=B, quad=quad))
    hr = np.random.default_rng(9)
    centers = np.stack([hr.uniform(-math.pi, math.pi, n_hills), hr.uniform(0.0, math.pi, n_hills)], 1)
    sigma = [0.35, 0.35]
    heights = wt_hill_heights(centers, sigma, [2 * math.pi, 0.0], 1.2, 10.0, KT300, chunk=1024)
    hill_params = [1.2] + sigma + [10.0, KT300, -math.pi, 0.0, math.pi, math.pi]
    hill_iparams = [500, n_hills + 100000, 1, 0]
    return walkers, dict(centers=centers, heights=heights, params=hill_params, iparams=hill_iparams)


def config4_restraints(walkers, restraint_k=100.0):
    """Harmonic restraint centres of the 64-walker workload, stored in each walker
    dict as ``restraint = (k, distance centre, coordination centre)``.

    The centres sit away from the walkers' initial CV values: distance d0 + 0.05 nm,
    coordination 1.01 CN0 + 2 with CN0 the FP64 coordination number of the initial
    positions. With a centre equal to the current value, dU/dCV = k (s - s0) is a
    difference of nearly equal numbers and the restraint forces are rounding noise
    of the CV; offset, they are forces of order k * 0.05 and k * (0.01 CN0 + 2) that a
    comparison with the FP64 oracle can resolve."""
    for w in walkers:
        if "cn_fp64" not in w:
            w["cn_fp64"] = coordination_cn_fp64(w["pos"], w["A"], w["B"], w["L"])
        w["restraint"] = (float(restraint_k), w["d0"] + 0.05, 1.01 * w["cn_fp64"] + 2.0)
    return walkers


def config5(n_pairs=10000, n_frames=50, n_path_atoms=500, n_hills=2000):
    """C5: 30,000 atoms at water density (seed 10); contact map of 10,000 seeded
    pairs with r0 ~ U[0.4, 0.8] nm (seed 11), n 6, m 12, w 1; path CV over 50
    frames of 500 atoms, frames = seeded base + cumulative N(0, 0.05 nm) drift
    (seed 12), lambda = 2.3 / mean adjacent-frame MSD; 2-D hill bias on (CMAP, s)."""
    n = 30000
    L = (n / 100.0) ** (1.0 / 3.0)
    rng = np.random.default_rng(10)
    pos = rng.uniform(0.0, L, (n, 3))
    pr = np.random.default_rng(11)
    pairs = np.stack([pr.integers(0, n, n_pairs), pr.integers(0, n, n_pairs)], 1)
    same = pairs[:, 0] == pairs[:, 1]
    pairs[same, 1] = (pairs[same, 1] + 1) % n
    r0 = pr.uniform(0.4, 0.8, n_pairs)
    cm_params = [v for i in range(n_pairs) for v in (r0[i], 6.0, 12.0, 1.0)]
    fr = np.random.default_rng(12)
    patoms = fr.choice(n, n_path_atoms, replace=False)
    base = pos[patoms]
    frames = [base.copy()]
    for _ in range(n_frames - 1):
        frames.append(frames[-1] + fr.normal(0.0, 0.05, base.shape))
    msd = np.mean([((frames[i + 1] - frames[i]) ** 2).sum(-1).mean() for i in range(n_frames - 1)])
    lam = 2.3 / msd
    path_params = [lam, n_frames] + list(np.concatenate([f.ravel() for f in frames]))
    cvs = [(CV_CONTACTMAP, [int(x) for x in pairs.ravel()], cm_params),
           (CV_PATH, [int(x) for x in patoms], path_params)]
    return Workload("C5", pos, _cube(L), cvs, [], np.ones(n), False, b"",
                    dict(pairs=pairs, r0=r0, patoms=patoms, frames=np.array(frames), lam=lam))
