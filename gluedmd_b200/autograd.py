"""Differentiable contact-map + path-CV + hill bias as a torch.autograd.Function.

    E = sum_k h_k exp(-(CMAP - c_k0)^2 / (2 sig0^2) - (s - c_k1)^2 / (2 sig1^2))

with CMAP the contact map over atom pairs (per-pair r0, integer n/m, weight w)
and s the path progress over reference frames. Forward and backward are CUDA
kernels (glued_ad_forward / glued_ad_backward): the backward gives dE/d(positions)
(minus the bias force), dE/d(r0), dE/d(frames) and dE/d(heights), recomputing the
per-pair switching values instead of storing them. float64 tensors run the FP64
kernels (for finite-difference checks), float32 the FP32 ones.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from ._native import call, c_int, c_double, c_void_p, P


class AdSpec(ctypes.Structure):
    _fields_ = [("pos", c_void_p), ("nAtoms", c_int), ("pairs", c_void_p), ("nPairs", c_int),
                ("r0", c_void_p), ("nmw", c_void_p), ("pathAtoms", c_void_p), ("M", c_int),
                ("frames", c_void_p), ("F", c_int), ("lam", c_double), ("hillC", c_void_p),
                ("heights", c_void_p), ("K", c_int), ("sig", c_double * 2), ("periodic", c_int),
                ("box", c_double * 3)]


@dataclass
class BiasTopology:
    """Non-differentiable description of the bias (device tensors)."""
    pairs: torch.Tensor       # int32 [P, 2]
    nmw: torch.Tensor         # float32 [P, 3]: n, m, w
    path_atoms: torch.Tensor  # int32 [M]
    lam: float
    hill_centers: torch.Tensor  # float64 [K, 2]
    sigma: tuple
    box: tuple = None         # rectangular box lengths, None = no PBC

    @classmethod
    def build(cls, pairs, r0_n_m_w, path_atoms, lam, hill_centers, sigma, box=None, device="cuda"):
        nmw = np.asarray(r0_n_m_w, np.float32)[:, 1:4]
        return cls(torch.as_tensor(np.asarray(pairs, np.int32).reshape(-1, 2), device=device),
                   torch.as_tensor(np.ascontiguousarray(nmw), device=device),
                   torch.as_tensor(np.asarray(path_atoms, np.int32), device=device), float(lam),
                   torch.as_tensor(np.asarray(hill_centers, np.float64).reshape(-1, 2), device=device),
                   tuple(float(s) for s in sigma), None if box is None else tuple(float(b) for b in box))


def _spec(topo, pos, r0, frames, heights):
    s = AdSpec()
    s.pos = pos.data_ptr(); s.nAtoms = pos.shape[0]
    s.pairs = topo.pairs.data_ptr(); s.nPairs = topo.pairs.shape[0]
    s.r0 = r0.data_ptr(); s.nmw = topo.nmw.data_ptr()
    s.pathAtoms = topo.path_atoms.data_ptr(); s.M = topo.path_atoms.shape[0]
    s.frames = frames.data_ptr(); s.F = frames.shape[0]
    s.lam = topo.lam
    s.hillC = topo.hill_centers.data_ptr(); s.heights = heights.data_ptr(); s.K = heights.shape[0]
    s.sig[0], s.sig[1] = topo.sigma
    s.periodic = 0 if topo.box is None else 1
    if topo.box is not None:
        for i in range(3):
            s.box[i] = topo.box[i]
    return s


def _dtype_code(t):
    if t.dtype == torch.float64:
        return 1
    if t.dtype == torch.float32:
        return 0
    raise TypeError("positions must be float32 or float64")


class GluedBias(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, r0, frames, heights, topo):
        pos, r0, frames, heights = (t.contiguous() for t in (pos, r0, frames, heights))
        dt = pos.dtype
        if not all(t.dtype == dt for t in (r0, frames, heights)):
            raise TypeError("positions, r0, frames and heights must share a dtype")
        F = frames.shape[0]
        out = torch.empty(7 + F, dtype=torch.float64, device=pos.device)
        n_part = max(1, min(1184, (topo.pairs.shape[0] + 255) // 256))
        part = torch.empty(n_part, dtype=torch.float64, device=pos.device)
        spec = _spec(topo, pos, r0, frames, heights)
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        call("glued_ad_forward", _dtype_code(pos), c_void_p(stream), ctypes.byref(spec),
             c_void_p(out.data_ptr()), c_void_p(part.data_ptr()), n_part)
        ctx.save_for_backward(pos, r0, frames, heights, out)
        ctx.topo = topo
        return out[0].to(dt)

    @staticmethod
    def backward(ctx, gE):
        pos, r0, frames, heights, out = ctx.saved_tensors
        topo = ctx.topo
        g = gE.detach().to(torch.float64).reshape(1).contiguous()
        gp, gr, gf, gh = (torch.empty_like(t) for t in (pos, r0, frames, heights))
        acc = torch.empty(3 * pos.shape[0], dtype=torch.int64, device=pos.device)
        spec = _spec(topo, pos, r0, frames, heights)
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        call("glued_ad_backward", _dtype_code(pos), c_void_p(stream), ctypes.byref(spec),
             c_void_p(out.data_ptr()), c_void_p(g.data_ptr()), c_void_p(acc.data_ptr()), c_void_p(gp.data_ptr()),
             c_void_p(gr.data_ptr()), c_void_p(gf.data_ptr()), c_void_p(gh.data_ptr()))
        return gp, gr, gf, gh, None


def glued_bias(pos, r0, frames, heights, topo):
    """Energy of the contact-map / path / hill bias; differentiable in all four tensors."""
    return GluedBias.apply(pos, r0, frames, heights, topo)


def cv_values(pos, r0, frames, heights, topo):
    """(E, CMAP, s, z) of the forward pass (no autograd)."""
    with torch.no_grad():
        pos, r0, frames, heights = (t.contiguous() for t in (pos, r0, frames, heights))
        F = frames.shape[0]
        out = torch.empty(7 + F, dtype=torch.float64, device=pos.device)
        n_part = max(1, min(1184, (topo.pairs.shape[0] + 255) // 256))
        part = torch.empty(n_part, dtype=torch.float64, device=pos.device)
        spec = _spec(topo, pos, r0, frames, heights)
        call("glued_ad_forward", _dtype_code(pos), c_void_p(torch.cuda.current_stream().cuda_stream),
             ctypes.byref(spec), c_void_p(out.data_ptr()), c_void_p(part.data_ptr()), n_part)
        return out[:4].cpu().numpy()
