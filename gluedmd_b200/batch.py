"""Batched multi-walker evaluation (glued_batch_* of include/glued_b200.h).

All walkers of one GPU are evaluated by one graph per step: a persistent
kernel for the coordination pairs, then a finalize kernel that also sums the
shared hill table per walker. Each walker owns a float4 posq buffer and an int64 fixed-point force
buffer in device memory (torch tensors here); walkers may have different atom
counts and boxes but the same CV / bias structure.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._native import WalkerDesc, call, lib, c_int, c_double, c_void_p, c_ll
from .gluedplugin import GluedForce

FIXED = 4294967296.0


class Walker:
    """Device buffers of one walker: posq (padded, 4) float32 and force (3*padded) int64."""

    def __init__(self, positions, box, device="cuda", padding=32):
        pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        self.n = len(pos)
        self.padded = ((self.n + padding - 1) // padding) * padding
        self.posq = torch.zeros((self.padded, 4), dtype=torch.float32, device=device)
        self.posq[: self.n, :3] = torch.as_tensor(pos, dtype=torch.float32, device=device)
        self.force = torch.zeros(3 * self.padded, dtype=torch.int64, device=device)
        self.box = np.asarray(box, dtype=np.float64).reshape(3, 3)

    def forces(self):
        f = self.force.view(3, self.padded)[:, : self.n].cpu().numpy().astype(np.float64) / FIXED
        return f.T.copy()


class WalkerPool:
    """Walkers whose posq and force buffers are views into one allocation each,
    so all positions move host->device in one copy and all forces back in one."""

    def __init__(self, positions_list, boxes, device="cuda", padding=32):
        ns = [len(np.asarray(p).reshape(-1, 3)) for p in positions_list]
        pads = [((n + padding - 1) // padding) * padding for n in ns]
        self.offsets = np.concatenate([[0], np.cumsum(pads)]).astype(np.int64)
        total = int(self.offsets[-1])
        self.posq = torch.zeros((total, 4), dtype=torch.float32, device=device)
        self.force = torch.zeros(3 * total, dtype=torch.int64, device=device)
        self.walkers = []
        for i, (p, box) in enumerate(zip(positions_list, boxes)):
            w = Walker.__new__(Walker)
            w.n, w.padded = ns[i], pads[i]
            o = int(self.offsets[i])
            w.posq = self.posq[o:o + pads[i]]
            w.force = self.force[3 * o:3 * (o + pads[i])]
            w.posq[: w.n, :3] = torch.as_tensor(np.asarray(p, dtype=np.float64).reshape(-1, 3),
                                                dtype=torch.float32, device=device)
            w.box = np.asarray(box, dtype=np.float64).reshape(3, 3)
            self.walkers.append(w)


class Batch:
    def __init__(self, forces, walkers, stream=None):
        if len(forces) != len(walkers):
            raise ValueError("one force per walker")
        self.forces = list(forces)
        self.walkers = list(walkers)
        W = len(walkers)
        descs = (WalkerDesc * W)()
        for i, w in enumerate(walkers):
            descs[i].posq = w.posq.data_ptr()
            descs[i].force_buffer = w.force.data_ptr()
            descs[i].num_atoms = w.n
            descs[i].padded_num_atoms = w.padded
            for k, v in enumerate(w.box.ravel()):
                descs[i].box[k] = float(v)
        fptrs = (c_void_p * W)(*[f._h.value for f in forces])
        h = c_void_p()
        call("glued_batch_create", fptrs, W, descs, ctypes.byref(h))
        self._h = h
        self.num_walkers = W
        s = torch.cuda.current_stream() if stream is None else stream
        call("glued_batch_set_stream", self._h, c_void_p(s.cuda_stream))
        n = c_int()
        call("glued_batch_num_cvs", self._h, ctypes.byref(n))
        self.num_cvs = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().glued_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def execute(self):
        call("glued_batch_execute", self._h)

    def update_state(self, step):
        call("glued_batch_update_state", self._h, int(step))

    def step(self, step):
        self.update_state(step)
        self.execute()

    def energies(self):
        out = (c_double * self.num_walkers)()
        call("glued_batch_get_energies", self._h, out)
        return np.array(out[:])

    def cv_values(self):
        out = (c_double * (self.num_walkers * max(1, self.num_cvs)))()
        call("glued_batch_get_cv_values", self._h, out)
        return np.array(out[: self.num_walkers * self.num_cvs]).reshape(self.num_walkers, self.num_cvs)

    def num_hills(self):
        n = c_int()
        call("glued_batch_num_hills", self._h, ctypes.byref(n))
        return n.value

    def set_hills(self, centers, heights):
        c = np.ascontiguousarray(centers, dtype=np.float64)
        h = np.ascontiguousarray(heights, dtype=np.float64)
        call("glued_batch_set_hills", self._h, c.ctypes.data_as(ctypes.POINTER(c_double)),
             h.ctypes.data_as(ctypes.POINTER(c_double)), len(h))

    def get_hills(self, D=2):
        n = self.num_hills()
        c = np.zeros(n * D)
        h = np.zeros(n)
        call("glued_batch_get_hills", self._h, c.ctypes.data_as(ctypes.POINTER(c_double)),
             h.ctypes.data_as(ctypes.POINTER(c_double)), n)
        return c.reshape(n, D), h

    def status(self):
        s = c_int()
        call("glued_batch_status", self._h, ctypes.byref(s))
        return s.value

    def launch_count(self):
        v = c_ll()
        call("glued_batch_launch_count", self._h, ctypes.byref(v))
        return v.value

    def phase_times(self):
        """One step between CUDA events, every CTA time-stamped (microseconds);
        see glued_batch_phase_times."""
        out = (c_double * 28)()
        call("glued_batch_phase_times", self._h, out)
        keys = ["step_us", "device_span_us", "stage_med_us", "stage_max_us", "coord_end_min_us",
                "coord_end_med_us", "coord_end_max_us", "runs_end_med_us", "runs_end_max_us",
                "fin_cta_med_us", "fin_cta_max_us", "fin_start_us", "coord_steps", "grid", "parts",
                "finalize_grid", "fin_record_us", "fin_cn_us", "fin_energy_us", "fin_coord_scatter_us",
                "fin_simple_rows_us", "hill_wait_us", "hill_eval_us", "hill_reduce_us", "runs_us", "finalize_us",
                "first_step_ready_us", "first_step_us"]
        self.phase_times_last = dict(zip(keys, out[:]))
        return dict(self.phase_times_last)

    def phase_stamps(self):
        """Raw records of the last phase_times call: (runs [grid, 11] = SM id,
        coordination steps, nine %globaltimer stamps in ns; finalize [CTAs, 6])."""
        n = c_ll()
        call("glued_batch_phase_stamps", self._h, None, 0, ctypes.byref(n))
        buf = (ctypes.c_ulonglong * max(1, n.value))()
        call("glued_batch_phase_stamps", self._h, buf, n.value, ctypes.byref(n))
        v = np.array(buf[:n.value], dtype=np.uint64)
        grid = int(self.phase_times_last["grid"]) if hasattr(self, "phase_times_last") else 0
        runs = v[:11 * grid].reshape(grid, 11)
        return runs, v[11 * grid:].reshape(-1, 6)

    @property
    def tuning(self):
        t = (c_int * 4)()
        call("glued_batch_get_tuning", self._h, t)
        return dict(ra=t[0], parts=t[1], plain=t[2], ch=t[3])

    def set_tuning(self, ra=8, parts=0, plain=0, ch=128):
        t = (c_int * 4)(ra, parts, plain, ch)
        call("glued_batch_set_tuning", self._h, t)

    def set_sum_precision(self, mode):
        """1: plain FP32 sums; 2: two-sum compensated hill sums, blocked coordination."""
        call("glued_batch_set_sum_precision", self._h, int(mode))

    def sum_precision(self):
        m = c_int()
        call("glued_batch_get_sum_precision", self._h, ctypes.byref(m))
        return m.value

    def autotune(self, use_cache=True):
        """glued_batch_autotune_ex: the fastest tiling (cached per batch signature
        for the process unless use_cache is False); self.tune_cached tells which."""
        t = (c_int * 4)()
        cached = c_int()
        call("glued_batch_autotune_ex", self._h, 1 if use_cache else 0, t, ctypes.byref(cached))
        self.tune_cached = bool(cached.value)
        return dict(ra=t[0], parts=t[1], plain=t[2], ch=t[3])


def force_for(cvs, biases, pbc=True):
    f = GluedForce()
    f.setUsesPeriodicBoundaryConditions(pbc)
    for t, a, p in cvs:
        f.addCollectiveVariable(t, [int(x) for x in a], [float(x) for x in p])
    for t, c, p, ip in biases:
        f.addBias(t, c, p, ip)
    return f


def c4_biases(walker, hill_params, hill_iparams, restraint_k=100.0, cn0=None, d0=None):
    """Per-walker biases of the 64-walker workload: harmonic restraints on the
    distance (CV 0, centre d0, default the walker's initial distance) and the
    coordination (CV 3, centre cn0; none when cn0 is None), and the shared hill-sum
    MetaD on (dihedral, angle) = CVs (2, 1)."""
    b = [(1, [0], [restraint_k, walker["d0"] if d0 is None else d0], [0])]
    if cn0 is not None:
        b.append((1, [3], [restraint_k, cn0], [0]))
    b.append((103, [2, 1], hill_params, hill_iparams))
    return b


def c4_walker_biases(walker, hill):
    """c4_biases with the restraint centres workloads.config4_restraints stored
    in the walker (the benchmark's definition of the 64-walker workload)."""
    k, d, cn = walker["restraint"]
    return c4_biases(walker, hill["params"], hill["iparams"], restraint_k=k, cn0=cn, d0=d)
