"""Benchmark of the per-step CV -> bias -> force-scatter path on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--config c4|c2|c1|c1pb|c3|c5] [--impl ours|reference]

A step is one pass of the hot path over one batch of synthetic input:
updateState(step) (pace-gated deposition) followed by execute(forces) for every
walker of the configuration. Inputs stay resident in HBM for `value`; `e2e`
repeats the measurement through the C ABI with host buffers (pinned host ->
device positions before, device -> host forces and energies after, every step).

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events on
the launching stream with a 256 MB L2 flush between steps (outside the events);
device time summed over steps, max over ranks. nvidia-smi clocks are sampled
during the timed region. Under torchrun each rank runs its own copy of the
workload (walkers shard across GPUs, no data-path collective: weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PAIR = 45.0      # coordination pair, FMA = 2 flops (per-pair count of the workload spec)
FLOP_HILL = 14.0      # one hill Gaussian + gradient (plus one exp)
# DRAM bytes (read + write) of one launch, from the ncu captures summarised under
# profiles/ (cold caches, one launch of the full workload)
TRAFFIC_C4_RUNS = 8.581e6
TRAFFIC_C2_COORD = 0.680e6


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


_CLOCK_SAMPLER = r"""
import sys, time, pynvml
pynvml.nvmlInit()
bus, idx, out = sys.argv[1], int(sys.argv[2]), sys.argv[3]
try:
    h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
except Exception:
    h = pynvml.nvmlDeviceGetHandleByIndex(idx)
with open(out, "w", buffering=1) as f:
    while True:
        t = time.time()
        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
        mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        f.write(f"{t:.6f} {sm} {mx} {rs}\n")
        time.sleep(0.001)
"""


class Clocks:
    """SM clocks and throttle reasons sampled during timing by a separate sampler
    process (NVML every millisecond, independent of this process's GIL; the GPU is
    matched to the CUDA device by PCI bus id). Only samples taken between the
    start and the end of the timed region are summarised; the raw samples (time,
    SM MHz, max SM MHz, reason bits) go to a file in the system temporary
    directory, or to $GLUED_BENCH_CLOCKS_DIR when that is set."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, index=0):
        import tempfile
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None
        d = os.environ.get("GLUED_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, f"glued_bench_clocks_{os.getpid()}.txt")

    def __enter__(self):
        import torch
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            if os.path.exists(self.path):
                os.remove(self.path)
            self.proc = subprocess.Popen([sys.executable, "-c", _CLOCK_SAMPLER, bus, str(self.index), self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            t = time.time()
            while time.time() - t < 10.0:
                if os.path.exists(self.path) and os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def __exit__(self, *a):
        self.t1 = time.time()
        if self.proc:
            time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path).read().splitlines():
                f = line.split()
                if len(f) == 4 and self.t0 <= float(f[0]) <= self.t1:
                    rows.append((int(f[1]), int(f[2]), int(f[3])))
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({name for r in rows for bit, name in self.REASONS.items() if r[2] & bit})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": float(max(r[1] for r in rows)),
                "reasons": reasons, "samples": len(rows), "source": "NVML every 1 ms in a sampler process"}


# ----------------------------------------------------------------- workloads
def build_single(w, torch, device):
    """One plain context for a single-walker workload (C1/C2/C3)."""
    from gluedmd_b200 import GluedForce
    from gluedmd_b200.context import Context, System
    s = System()
    for m in w.masses:
        s.addParticle(float(m))
    f = GluedForce()
    f.setUsesPeriodicBoundaryConditions(w.pbc)
    for t, a, p in w.cvs:
        f.addCollectiveVariable(t, [int(x) for x in a], [float(x) for x in p])
    for t, c, p, ip in w.biases:
        f.addBias(t, c, p, ip)
    s.addForce(f)
    s.setDefaultPeriodicBoxVectors(*w.box)
    ctx = Context(s, w.positions, device=device)
    if w.blob:
        f.setBiasState(w.blob)
    return ctx, f


def time_steps(torch, step_fn, steps, warmup, flush):
    stream = torch.cuda.current_stream()
    for i in range(warmup):
        step_fn(i)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    # NVTX range "timed": lets a profiler restrict its launch list to these steps
    torch.cuda.nvtx.range_push("timed")
    for i in range(steps):
        flush.add_(1.0)
        starts[i].record(stream)
        step_fn(warmup + i)
        ends[i].record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends))


def run_single(args, torch, cfg):
    from gluedmd_b200 import workloads as W, _native
    import ctypes
    w = {"c1": lambda: W.config1("grid"), "c1pb": lambda: W.config1("pbmetad"), "c1h": lambda: W.config1("hills"),
         "c2": W.config2, "c3": W.config3}[cfg]()
    ctx, f = build_single(w, torch, "cuda")
    nc = ctx.glued_context_for(f)
    # correctness of this exact workload against the FP64 oracle (untimed)
    e_chk, F_chk = ctx.computeForces()
    P = _checker()
    perr = P.check_single(w, e_chk, F_chk, np.array(f.getLastCVValues(ctx)))
    perr.pop("ref")
    parity = P.summary([perr], "one force evaluation of the timed workload, before the timed steps")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step(i):
        nc.update_state(i)
        nc.execute(True, False)

    launches0 = nc.launch_count()
    with Clocks(torch.cuda.current_device()) as clk:
        ms = time_steps(torch, step, args.steps, args.warmup, flush)
    launches = (nc.launch_count() - launches0)
    kernels_per_step = launches / float(args.steps + args.warmup)
    us = ms * 1e3 / args.steps
    # dominant kernel, timed with CUDA events on the launching stream
    phases = nc.profile_phases(20)
    names = ["simple_cvs", "group_cvs", "coord_pairs", "coord_finalize", "biases", "scatter"]
    dom = int(np.argmax(phases))
    # e2e through the C ABI with host buffers
    n = len(w.positions)
    host_pos = torch.zeros((ctx.padded, 4), dtype=torch.float32).pin_memory()
    host_pos[:n, :3] = torch.as_tensor(w.positions, dtype=torch.float32)
    host_f = torch.zeros(3 * ctx.padded, dtype=torch.int64).pin_memory()
    stream = torch.cuda.current_stream()

    def e2e_step(i):
        ctx.posq.copy_(host_pos, non_blocking=True)
        ctx.force_buf.zero_()
        nc.update_state(args.warmup + args.steps + i)
        e = nc.execute(True, True)  # synchronizing energy read
        host_f.copy_(ctx.force_buf, non_blocking=True)
        return e

    for i in range(args.warmup):
        e2e_step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        e2e_step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_us = e0.elapsed_time(e1) * 1e3 / args.steps
    info = dict(workload=w.name, us_per_step=us, phases_ms=dict(zip(names, phases)), dominant=names[dom],
                dom_ms=phases[dom], kernels_per_step=kernels_per_step, e2e_us=e2e_us,
                h2d=int(host_pos.numel() * 4), d2h=int(host_f.numel() * 8 + 8), clocks=clk.summary(), w=w,
                parity=parity)
    return info


def c5_inputs(torch, dtype):
    """C5: the 30,000-atom contact map (10,000 pairs) + 50-frame path CV with a
    2-D hill sum of 2,000 hills on (CMAP, s): centres spread over the current CV
    values +- 3 sigma (seed 2), heights U[0.2, 1.2]; all four tensors on the
    device, differentiable."""
    from gluedmd_b200 import workloads as W
    from gluedmd_b200.autograd import BiasTopology, cv_values
    w = W.config5()
    pos, pairs, r0 = w.positions, w.extra["pairs"], w.extra["r0"]
    patoms, frames, lam = w.extra["patoms"], w.extra["frames"], w.extra["lam"]
    K = 2000
    nmw = np.c_[r0, np.full(len(r0), 6.0), np.full(len(r0), 12.0), np.ones(len(r0))]
    sigma = (0.02 * max(1.0, len(r0) / 40.0), 0.35)

    def dev(x):
        return torch.tensor(np.asarray(x), dtype=dtype, device="cuda", requires_grad=True)

    topo0 = BiasTopology.build(pairs, nmw, patoms, lam, np.zeros((K, 2)), sigma)
    _, cm, s_, _ = cv_values(dev(pos), dev(r0), dev(frames), dev(np.ones(K)), topo0)
    rng = np.random.default_rng(2)
    centers = np.c_[cm + rng.uniform(-3, 3, K) * sigma[0], s_ + rng.uniform(-3, 3, K) * sigma[1]]
    heights = rng.uniform(0.2, 1.2, K)
    topo = BiasTopology.build(pairs, nmw, patoms, lam, centers, sigma)
    return w, topo, [dev(pos), dev(r0), dev(frames), dev(heights)], dict(
        pairs=pairs, r0=r0, patoms=patoms, frames=frames, lam=lam, centers=centers, heights=heights, sigma=sigma)


C5_KERNELS_PER_STEP = 5   # forward: pair partials, path + hills; backward: pairs, path, hills + convert (+ one memset node)


def run_c5(args, torch):
    """C5 through the library's C ABI: glued_ad_forward + glued_ad_backward (dL/dE
    = 1) on preallocated device buffers, captured once in a CUDA graph; one step
    = one replay (energy, forces and the gradients w.r.t. r0, frames and hill
    heights). The autograd wrapper (gluedmd_b200.autograd.glued_bias) issues the
    same two calls; its result is compared with the graph's once."""
    import ctypes
    from ctypes import c_void_p
    from gluedmd_b200._native import call
    from gluedmd_b200.autograd import _spec, glued_bias
    w, topo, (p, r, f, h), raw = c5_inputs(torch, torch.float32)
    pd, rd, fd, hd = (t.detach() for t in (p, r, f, h))
    out = torch.empty(7 + fd.shape[0], dtype=torch.float64, device="cuda")
    n_part = max(1, min(1184, (topo.pairs.shape[0] + 255) // 256))
    part = torch.empty(n_part, dtype=torch.float64, device="cuda")
    gE = torch.ones(1, dtype=torch.float64, device="cuda")
    acc = torch.empty(3 * pd.shape[0], dtype=torch.int64, device="cuda")
    gp, gr, gf, gh = (torch.empty_like(t) for t in (pd, rd, fd, hd))
    spec = _spec(topo, pd, rd, fd, hd)

    def enqueue(stream):
        call("glued_ad_forward", 0, c_void_p(stream), ctypes.byref(spec), c_void_p(out.data_ptr()),
             c_void_p(part.data_ptr()), n_part)
        call("glued_ad_backward", 0, c_void_p(stream), ctypes.byref(spec), c_void_p(out.data_ptr()),
             c_void_p(gE.data_ptr()), c_void_p(acc.data_ptr()), c_void_p(gp.data_ptr()), c_void_p(gr.data_ptr()),
             c_void_p(gf.data_ptr()), c_void_p(gh.data_ptr()))

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        enqueue(side.cuda_stream)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        enqueue(torch.cuda.current_stream().cuda_stream)
    # the graph's result against the autograd wrapper's
    graph.replay()
    glued_bias(p, r, f, h, topo).backward()
    torch.cuda.synchronize()
    diff = float((gp - p.grad).abs().max() / p.grad.abs().max().clamp_min(1e-30))
    if not diff < 1e-6:
        raise RuntimeError(f"C5 graph and autograd forces differ: {diff:.3e}")
    # energy and forces of this exact workload against the FP64 oracle (untimed)
    P = _checker()
    E_ref, F_ref, cv_ref = P.c5_reference(w.positions, raw["pairs"], raw["r0"], raw["patoms"], raw["frames"],
                                          raw["lam"], raw["centers"], raw["heights"], raw["sigma"])
    F_gpu = -gp.double().cpu().numpy()
    import oracle as _O
    parity = {"max_rel_force_err": _O.max_rel_force_err(F_gpu, F_ref),
              "energy_rel_err": P.rel_energy_err(float(out[0].item()), E_ref),
              "oracle": "FP64 (oracle/glued_oracle.cpp, double)",
              "checked": "one graph replay (forward + backward) of the timed workload, before the timed steps"}
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step(i):
        graph.replay()

    with Clocks(torch.cuda.current_device()) as clk:
        ms = time_steps(torch, step, args.steps, args.warmup, flush)
    us = ms * 1e3 / args.steps
    # e2e: positions from pinned host memory, energy and forces back to the host
    host_pos = torch.tensor(w.positions, dtype=torch.float32).pin_memory()
    host_f = torch.empty_like(host_pos).pin_memory()
    host_e = torch.empty(1, dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream()

    def e2e_step(i):
        pd.copy_(host_pos, non_blocking=True)
        graph.replay()
        host_f.copy_(gp, non_blocking=True)
        host_e.copy_(out[:1], non_blocking=True)

    for i in range(args.warmup):
        e2e_step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        e2e_step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_us = e0.elapsed_time(e1) * 1e3 / args.steps
    return dict(us_per_step=us, e2e_us=e2e_us, clocks=clk.summary(), raw=raw, w=w,
                h2d=int(host_pos.numel() * 4), d2h=int(host_f.numel() * 4 + 8), parity=parity)


def c5_raw_from_oracle():
    """The C5 inputs for the reference arm: hill centres placed around the FP64
    oracle's CV values (the GPU arm places them around its own)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from gluedmd_b200 import workloads as W
    w = W.config5()
    pairs, r0, patoms, frames, lam = (w.extra[k] for k in ("pairs", "r0", "patoms", "frames", "lam"))
    P = len(pairs)
    cm_params = [v for i in range(P) for v in (r0[i], 6.0, 12.0, 1.0)]
    cvs = [(O.CV_CONTACTMAP, [int(x) for x in pairs.ravel()], cm_params),
           (O.CV_PATH, [int(x) for x in patoms], [lam, len(frames)] + list(np.asarray(frames).ravel()))]
    cvv, _ = O.OracleSystem(cvs, mode="f64", num_particles=len(w.positions),
                            test_bias_gradients=[0.0, 0.0, 0.0]).evaluate_cvs(w.positions)
    K = 2000
    sigma = (0.02 * max(1.0, P / 40.0), 0.35)
    rng = np.random.default_rng(2)
    centers = np.c_[cvv[0] + rng.uniform(-3, 3, K) * sigma[0], cvv[1] + rng.uniform(-3, 3, K) * sigma[1]]
    heights = rng.uniform(0.2, 1.2, K)
    return w, dict(pairs=pairs, r0=r0, patoms=patoms, frames=np.asarray(frames), lam=lam, centers=centers,
                   heights=heights, sigma=sigma)


def cpu_baseline_c5(w, raw, budget_s=12.0):
    """The oracle's FP64 restatement of the C5 step on one host thread: CVs, the
    hill sum's dE/dCV, the chain rule to forces; bounded sample of steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    P = len(raw["pairs"])
    cm_params = [v for i in range(P) for v in (raw["r0"][i], 6.0, 12.0, 1.0)]
    cvs = [(O.CV_CONTACTMAP, [int(x) for x in raw["pairs"].ravel()], cm_params),
           (O.CV_PATH, [int(x) for x in raw["patoms"]], [raw["lam"], len(raw["frames"])] + list(raw["frames"].ravel()))]
    sysm = O.OracleSystem(cvs, mode="f64", num_particles=len(w.positions), test_bias_gradients=[0.0, 0.0, 0.0])
    c, hgt, sg = raw["centers"], raw["heights"], raw["sigma"]
    n = 0
    t0 = time.perf_counter()
    while n < 1 or time.perf_counter() - t0 < budget_s and n < 50:
        cvv, _ = sysm.evaluate_cvs(w.positions)
        d0, d1 = cvv[0] - c[:, 0], cvv[1] - c[:, 1]
        g = hgt * np.exp(-d0 ** 2 / (2 * sg[0] ** 2) - d1 ** 2 / (2 * sg[1] ** 2))
        sysm.test_grad = np.array([(-g * d0 / sg[0] ** 2).sum(), (-g * d1 / sg[1] ** 2).sum(), 0.0])
        sysm.execute(w.positions)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": dt / n * 1e6, "unit": "us/step", "cores": 1, "kind": "port",
            "sample": f"{n} steps of the C5 workload on one host thread (FP64 oracle: CVs twice per step, "
                      f"hill-sum dE/dCV in numpy)"}


def cpu_baseline_single(cfg, w, budget_s=12.0):
    """Reference kernels compiled for the host (oracle/_ref) when present, else the
    oracle's FP32 restatement; bounded sample of steps on one host thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ref_runner import RefSystem
    kind = "reference" if RefSystem.available() else "port"
    cls = RefSystem if kind == "reference" else O.OracleSystem
    biases = [b for b in w.biases if b[0] in (1, 3, 4, 5, 6)]
    sysm = cls(w.cvs, biases, masses=w.masses, periodic=w.pbc, mode="f32", num_particles=len(w.positions))
    if w.blob:
        sysm.load_blob(w.blob)
    box = np.asarray(w.box).ravel()
    t0 = time.perf_counter()
    n = 0
    while True:
        sysm.execute(w.positions, box)
        n += 1
        if time.perf_counter() - t0 > budget_s or n >= 50:
            break
    dt = (time.perf_counter() - t0) / n
    return dict(value=dt * 1e6, unit="us/step", cores=1, kind=kind,
                sample=f"{n} force evaluations of {w.name} ({'reference kernel text compiled for the host' if kind == 'reference' else 'oracle FP32 restatement'}), 1 thread")


def c4_inputs(n_walkers=64, n_hills=50000):
    from gluedmd_b200 import workloads as W
    ws, hill = W.config4_walkers(n_walkers=n_walkers, n_hills=n_hills)
    W.config4_restraints(ws)
    return ws, hill


def c4_biases(w, hill):
    from gluedmd_b200.batch import c4_walker_biases
    return c4_walker_biases(w, hill)


# Workload descriptions shared by both arms (the reference arm prints the same
# string; its bias form differs where the reference has no hill-sum kernel).
C4_WORKLOAD = ("C4: 64 walkers 1k-50k atoms (log-uniform), dist/angle/dihedral + 256x1024 coordination, "
               "harmonic restraints, shared 50,000-hill WT MetaD")
C4_FORM_OURS = "hill sum over the 50,000 shared hills"
C4_FORM_REF = "256x256 grid holding the 50,000 hills (the reference has no hill-sum kernel)"
C5_WORKLOAD = ("C5: 30,000 atoms, contact map 10,000 pairs + path CV 50 frames x 500 atoms, 2-D hill sum "
               "(2,000 hills); forward + backward (forces and the gradients w.r.t. r0, frames and hill heights)")


def _checker():
    """The FP64 oracle as the correctness checker (outside every timed region)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import parity
    return parity


def parity_c4(b, pool, ws, hill):
    """One batched step in the tuning the timed run uses, every walker's forces,
    CV values and energy against the FP64 oracle (max over walkers)."""
    P = _checker()
    pool.force.zero_()
    b.execute()
    E, cv = b.energies(), b.cv_values()
    errs = [P.check_walker(w, c4_biases(w, hill), hill["centers"], hill["heights"], E[i],
                           pool.walkers[i].forces(), cv[i]) for i, w in enumerate(ws)]
    return P.summary(errs, f"all {len(ws)} walkers, one step in the timed tiling, before the timed steps")


def run_c4(args, torch, ws, hill):
    from gluedmd_b200.batch import Batch, WalkerPool, force_for
    forces = [force_for(w["cvs"], c4_biases(w, hill)) for w in ws]
    pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
    walkers = pool.walkers
    b = Batch(forces, walkers)
    b.set_hills(hill["centers"], hill["heights"])
    tune = b.autotune()
    parity = parity_c4(b, pool, ws, hill)
    for wk in walkers:
        wk.force.zero_()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    W_ = len(ws)

    def step(i):
        b.update_state(i)
        b.execute()

    l0 = b.launch_count()
    with Clocks(torch.cuda.current_device()) as clk:
        ms = time_steps(torch, step, args.steps, args.warmup, flush)
    launches = b.launch_count() - l0
    status = b.status()
    # the persistent step kernel is the whole step: its per-launch time
    step_ms = ms / args.steps
    # plain per-walker path: one context per walker, stepped one after another
    plain_ctx = []
    from gluedmd_b200.context import Context, System
    from gluedmd_b200 import GluedForce, workloads as Wl
    hb = Wl.blob(hills=[(hill["centers"], hill["heights"])])
    for w in ws:
        s_ = System()
        for m in w["masses"]:
            s_.addParticle(float(m))
        f = force_for(w["cvs"], c4_biases(w, hill))
        s_.addForce(f)
        s_.setDefaultPeriodicBoxVectors(*w["box"])
        ctx = Context(s_, w["pos"])
        f.setBiasState(hb)
        plain_ctx.append((ctx, ctx.glued_context_for(f)))

    def plain_step(i):
        for ctx, nc in plain_ctx:
            nc.update_state(i)
            nc.execute(True, False)

    psteps = max(3, min(args.steps, 20))
    plain_ms = time_steps(torch, plain_step, psteps, 3, flush) / psteps
    plain_launches = sum(nc.launch_count() for _, nc in plain_ctx) / float(psteps + 3)
    del plain_ctx
    # e2e through the C ABI with host buffers: every walker's positions H2D from
    # pinned memory, one step, every force buffer and the energies D2H
    # one pooled buffer per direction: all walkers' positions in, all forces out
    host_pos = torch.zeros_like(pool.posq, device="cpu").pin_memory()
    host_f = torch.zeros_like(pool.force, device="cpu").pin_memory()
    host_pos.copy_(pool.posq)
    stream = torch.cuda.current_stream()

    def e2e_step(i):
        pool.posq.copy_(host_pos, non_blocking=True)
        pool.force.zero_()
        b.update_state(10 ** 6 + i)
        b.execute()
        host_f.copy_(pool.force, non_blocking=True)
        return b.energies()  # synchronizing read of the per-walker energies

    for i in range(args.warmup):
        e2e_step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        e2e_step(args.warmup + i)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    h2d = host_pos.numel() * 4
    d2h = host_f.numel() * 8 + 8 * W_
    pairs = sum(256 * 1024 for _ in ws)
    flops = pairs * FLOP_PAIR + W_ * b.num_hills() * FLOP_HILL
    # per-kernel durations (CUDA events around each launch of one step, L2 flushed
    # before every step): the dominant kernel is the coordination-runs kernel
    runs, fins, waits = [], [], []
    for i in range(20):
        flush.add_(1.0)
        pt = b.phase_times()
        runs.append(pt["runs_us"])
        fins.append(pt["finalize_us"])
        waits.append(pt["hill_wait_us"])
    runs_us = sum(runs) / len(runs)
    fin_us = sum(fins) / len(fins)
    hill_wait_us = float(np.median(waits))
    return dict(walkers=W_, step_ms=step_ms, value=W_ * 1e3 / step_ms, plain_ms=plain_ms,
                plain_value=W_ * 1e3 / plain_ms, plain_launches=plain_launches, e2e_value=W_ * 1e3 / e2e_ms,
                h2d=int(h2d), d2h=int(d2h), launches_per_step=launches / float(args.steps + args.warmup),
                flops=flops, clocks=clk.summary(), tune=tune, status=status, hills=b.num_hills(),
                graphed=True, runs_us=runs_us, finalize_us=fin_us, hill_wait_us=hill_wait_us, parity=parity)


def c4_phase_timeline(b, flush, calls=15):
    """Medians over `calls` steps (L2 flushed before each) of Batch.phase_times
    and, from the raw per-CTA stamps (%globaltimer), the finalize CTAs' six
    stamps per part relative to the exit of the last runs CTA (microseconds)."""
    pts, rel = [], []
    for _ in range(calls):
        flush.add_(1.0)
        pts.append(b.phase_times())
        runs, fin = b.phase_stamps()
        r, f = runs[:, 2:].astype(np.int64), fin.astype(np.int64)
        end = r[:, 5].max()
        parts = int(pts[-1]["parts"])
        part = np.arange(f.shape[0]) % parts
        rel.append([[float(np.median(f[part == q, k] - end)) * 1e-3 for k in range(6)] for q in range(parts)])
    return {"phase_times": {k: round(float(np.median([p[k] for p in pts])), 3) for k in pts[0]},
            "finalize_stamps_after_runs_end_us": np.round(np.median(np.array(rel), axis=0), 3).tolist()}


def cpu_reference_c4(ws, hill, steps_budget_s=20.0, threads=None):
    """The reference's kernels compiled for the host (oracle/_ref), one RefSystem
    per walker, walkers spread over host threads (ctypes releases the GIL).
    The reference's MetaD is grid-based: the 50,000 shared hills are deposited on
    its 256 x 256 grid over (dihedral, angle) and evaluated by its metaDEvalBias."""
    import concurrent.futures as cf
    import math as _m
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ref_runner import RefSystem
    from gluedmd_b200 import workloads as Wl
    kind = "reference" if RefSystem.available() else "port"
    cls = RefSystem if kind == "reference" else O.OracleSystem
    sig = [0.35, 0.35]
    lo, hi = [-_m.pi, 0.0], [_m.pi, _m.pi]
    grid = Wl.grid_from_hills_windowed(hill["centers"], hill["heights"], sig, lo, hi, [256, 256], [1, 0])
    systems = []
    for w in ws:
        biases = [b for b in c4_biases(w, hill) if b[0] == 1]
        biases.append((3, [2, 1], [1.2] + sig + [10.0, 2.494338785] + lo + hi, [500, 256, 256, 1, 0]))
        s_ = cls(w["cvs"], biases, masses=w["masses"], periodic=True, mode="f32", num_particles=w["n"])
        for st in s_.bias_state:
            if st["type"] == 3:
                st["grid"][:] = grid
        systems.append((s_, w))
    threads = threads or os.cpu_count() or 1
    pool = cf.ThreadPoolExecutor(max_workers=threads)

    def one(sw):
        s_, w = sw
        return s_.execute(w["pos"], w["box"].ravel())["energy"]

    list(pool.map(one, systems))  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        list(pool.map(one, systems))
        n += 1
        if time.perf_counter() - t0 > steps_budget_s or n >= 20:
            break
    dt = (time.perf_counter() - t0) / n
    pool.shutdown()
    return dict(value=len(ws) / dt, unit="walker-steps/s", cores=threads, kind=kind,
                sample=f"{n} steps x {len(ws)} walkers of the 64-walker workload on {threads} host threads "
                       f"({'reference kernel text compiled for the host' if kind == 'reference' else 'oracle FP32 restatement'}; "
                       "MetaD as the reference's 256x256 grid holding the same 50,000 hills)")


SUM_VARIANTS = {"fp64": (0, 0), "fp32": (1, 0), "fp32c": (2, 1)}


def precision_sweep(args, torch):
    """Step time (CUDA events, L2 flushed before every step) and error against the
    FP64 oracle of each sum-precision variant of one workload; one JSON line each.
    c1h / c3: kernel sums in FP64, FP32, FP32 two-sum (+ blocked coordination);
    c2cut: the C2 cutoff coordination on all-pairs tiles and on the cell list, in
    C2's 5.9 nm box and in a 12 nm box at the same density; c4tiles: every tile shape
    of the batch at the autotuned finalize setting;
    c2: no-fit RMSD or Kabsch RMSD (FP64 eigensolve), per-tile-run or blocked
    coordination sums; c4: the batch in plain FP32 and in two-sum FP32."""
    from gluedmd_b200 import workloads as W
    P = _checker()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = []

    def single(w, kernel_sums, coord, label):
        ctx, f = build_single(w, torch, "cuda")
        nc = ctx.glued_context_for(f)
        nc.set_sum_precision(kernel_sums, coord)
        e, F = ctx.computeForces()
        err = P.check_single(w, e, F, np.array(f.getLastCVValues(ctx)))
        err.pop("ref")

        def step(i):
            nc.update_state(i)
            nc.execute(True, False)

        ms = time_steps(torch, step, args.steps, args.warmup, flush)
        out.append({"sweep": args.config, "variant": label, "workload": w.name, "us_per_step": ms * 1e3 / args.steps,
                    "max_rel_force_err": err["force"], "energy_rel_err": err["energy"], "cv_rel_err": err["cv"],
                    "kernel_sums": kernel_sums, "coordination_blocked": coord})

    if args.config in ("c3", "c1h"):
        w = W.config3() if args.config == "c3" else W.config1("hills")
        for name, (k, c) in SUM_VARIANTS.items():
            single(w, k, c, name)
    elif args.config == "c2":
        for fit in (False, True):
            w = W.config2(fit=fit)
            for blocked in (0, 1):
                single(w, 0, blocked, ("kabsch" if fit else "nofit") + ("+blocked" if blocked else "+per-run"))
    elif args.config == "c2cut":
        for box in (5.9, 12.0):
            for method in (0, 1):
                single(W.config2_cutoff(method, box=box), 0, 0, ("tiles+mask" if method == 0 else "cells") +
                       f" box {box:g} nm")
    elif args.config == "c4tiles":
        # the batch's tile shapes (A atoms per warp x B chunk) at the fewest finalize parts
        from gluedmd_b200.batch import Batch, WalkerPool, force_for
        ws, hill = c4_inputs()
        pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
        b = Batch([force_for(w["cvs"], c4_biases(w, hill)) for w in ws], pool.walkers)
        b.set_hills(hill["centers"], hill["heights"])
        picked = b.autotune(use_cache=False)
        for ra, ch in ((8, 128), (4, 128), (8, 256), (4, 256)):
            b.set_tuning(ra=ra, parts=picked["parts"], plain=picked["plain"], ch=ch)
            par = parity_c4(b, pool, ws, hill)
            ms = time_steps(torch, lambda i: (b.update_state(i), b.execute()), args.steps, args.warmup, flush)
            runs = []
            for _ in range(10):
                flush.add_(1.0)
                runs.append(b.phase_times()["runs_us"])
            out.append({"sweep": "c4tiles", "variant": f"ra {ra} x chunk {ch}", "workload": C4_WORKLOAD,
                        "us_per_step": ms * 1e3 / args.steps, "runs_us": float(np.median(runs)),
                        "max_rel_force_err": par["max_rel_force_err"], "autotuned": picked})
    elif args.config == "c4":
        from gluedmd_b200.batch import Batch, WalkerPool, force_for
        ws, hill = c4_inputs()
        pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
        b = Batch([force_for(w["cvs"], c4_biases(w, hill)) for w in ws], pool.walkers)
        b.set_hills(hill["centers"], hill["heights"])
        tune = b.autotune()
        for mode, name in ((1, "fp32"), (2, "fp32c")):
            b.set_sum_precision(mode)
            par = parity_c4(b, pool, ws, hill)
            ms = time_steps(torch, lambda i: (b.update_state(i), b.execute()), args.steps, args.warmup, flush)
            out.append({"sweep": "c4", "variant": name, "workload": C4_WORKLOAD, "us_per_step": ms * 1e3 / args.steps,
                        "max_rel_force_err": par["max_rel_force_err"], "energy_rel_err": par["energy_rel_err"],
                        "cv_rel_err": par["cv_rel_err"], "tuning": tune, "status": b.status()})
    else:
        raise SystemExit("--precision-sweep: config must be c1h, c2, c2cut, c3, c4 or c4tiles")
    for line in out:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--config", default="c4", choices=["c1", "c1pb", "c1h", "c2", "c2cut", "c3", "c4", "c4tiles", "c5"])
    ap.add_argument("--precision-sweep", action="store_true",
                    help="time and check every sum-precision variant of --config (one JSON line each)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: warm-up + timed steps only, fixed tiling, no baselines (for ncu)")
    ap.add_argument("--walkers", type=int, default=64, help="C4 walker count (profiling of small cases)")
    ap.add_argument("--hills", type=int, default=50000, help="C4 hill count (profiling of small cases)")
    ap.add_argument("--tuning", default="8,0,0", help="fixed C4 tuning ra,finalize_parts,plain_finalize_launch (--profile)")
    ap.add_argument("--phases", action="store_true",
                    help="with --profile --config c4: per-CTA phase stamps of 15 more steps (Batch.phase_times)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # The reference's own CPU implementation of the path on the host cores;
        # rank 0 alone runs and prints.
        if rank != 0:
            return
        if args.config == "c4":
            ws, hill = c4_inputs()
            cb = cpu_reference_c4(ws, hill, steps_budget_s=min(60.0, max(10.0, 0.2 * args.steps)))
            line = {"impl": "reference", "metric": "walker-steps/s (CV+bias+force, 64 walkers)", "value": cb["value"],
                    "unit": "walker-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                    "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                    "config": {"workload": C4_WORKLOAD, "bias_form": C4_FORM_REF},
                    "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "walker-steps/s",
                                                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        elif args.config == "c5":
            w, raw = c5_raw_from_oracle()
            cb = cpu_baseline_c5(w, raw, budget_s=max(5.0, 0.5 * args.steps))
            line = {"impl": "reference", "metric": "CV+bias+force us/step", "value": cb["value"], "unit": "us/step",
                    "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                    "dtype": "f64", "data": "synthetic", "config": {"workload": C5_WORKLOAD},
                    "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "us/step", "h2d_bytes_per_step": 0,
                                                "d2h_bytes_per_step": 0}}
        else:
            from gluedmd_b200 import workloads as W
            w = {"c1": lambda: W.config1("grid"), "c1pb": lambda: W.config1("pbmetad"),
                 "c1h": lambda: W.config1("hills"), "c2": W.config2, "c3": W.config3}[args.config]()
            cb = cpu_baseline_single(args.config, w, budget_s=max(5.0, 0.5 * args.steps))
            line = {"impl": "reference", "metric": "CV+bias+force us/step", "value": cb["value"], "unit": "us/step",
                    "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                    "dtype": "f32", "data": "synthetic", "config": {"workload": w.name},
                    "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "us/step", "h2d_bytes_per_step": 0,
                                                "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    from gluedmd_b200 import dist as D
    torch.cuda.set_device(local)
    dist = D.init("nccl", timeout_s=120) if world > 1 else None

    def max_over_ranks(x):
        return D.max_over_ranks(x, device="cuda")

    from gluedmd_b200 import _native
    import ctypes
    pk, src = peaks()

    if args.precision_sweep:
        precision_sweep(args, torch)
        return

    if args.config == "c4" and args.profile:
        ws, hill = c4_inputs(args.walkers, args.hills)
        from gluedmd_b200.batch import Batch, WalkerPool, force_for
        pool = WalkerPool([w["pos"] for w in ws], [w["box"] for w in ws])
        b = Batch([force_for(w["cvs"], c4_biases(w, hill)) for w in ws], pool.walkers)
        b.set_hills(hill["centers"], hill["heights"])
        tv = [int(x) for x in args.tuning.split(",")] + [0, 0]
        b.set_tuning(tv[0], tv[1], tv[2])
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        ms = time_steps(torch, lambda i: (b.update_state(i), b.execute()), args.steps, args.warmup, flush)
        out = {"profile": "c4", "walkers": args.walkers, "hills": b.num_hills(), "ms_per_step": ms / args.steps,
               "status": b.status(), "tuning": b.tuning}
        if args.phases:
            out["phases"] = c4_phase_timeline(b, flush)
        print(json.dumps(out))
        return

    if args.config == "c4":
        ws, hill = c4_inputs()
        info = run_c4(args, torch, ws, hill)
        step_ms = max_over_ranks(info["step_ms"])
        if dist is not None:
            dist.barrier()
        if rank == 0:
            fp32 = ctypes.c_double()
            _native.call("glued_measure_fp32_peak", ctypes.byref(fp32))
            ach = info["flops"] / (info["runs_us"] * 1e-6) / 1e12
            roof = {"bound": "fp32", "kernel": "k_batch_runs (coordination pairs + hill table)", "achieved": ach,
                    "peak": fp32.value, "unit": "TFLOP/s", "frac": ach / fp32.value,
                    "traffic": TRAFFIC_C4_RUNS, "traffic_unit": "bytes per launch",
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture "
                                      "(profiles/k_batch_runs_c4.md)",
                    "launch_us": info["runs_us"],
                    "peak_source": "FP32 FMA microkernel measured in this run (MEASURED_PEAKS.json has no FP32 figure)",
                    "algorithmic": f"64 x 262144 pairs x {FLOP_PAIR:.0f} flop + 64 x {info['hills']} hills x {FLOP_HILL:.0f} flop",
                    "whole_step_frac": info["flops"] / (info["step_ms"] * 1e-3) / 1e12 / fp32.value,
                    "finalize_us": info["finalize_us"],
                    "hill_data_wait_us": info["hill_wait_us"]}
            cb = cb1 = None
            if not args.no_cpu_baseline and world == 1:
                cb = cpu_reference_c4(ws, hill, steps_budget_s=15.0)
                cb1 = cpu_reference_c4(ws, hill, steps_budget_s=8.0, threads=1)
            value = world * info["walkers"] * 1e3 / step_ms
            line = {
                "metric": "walker-steps/s (CV+bias+force, 64 walkers)", "value": value, "unit": "walker-steps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": C4_WORKLOAD, "bias_form": C4_FORM_OURS,
                           "walkers_per_gpu": info["walkers"], "l2": "flushed between steps (256 MB write)",
                           "parallelism": f"walkers x{world} GPUs (no data-path collective)", "tuning": info["tune"]},
                "e2e": {"value": world * info["e2e_value"], "unit": "walker-steps/s", "h2d_bytes_per_step": info["h2d"],
                        "d2h_bytes_per_step": info["d2h"]},
                "gpu_launches": int(round(info["launches_per_step"] * args.steps)),
                "roofline": roof, "cpu_baseline": cb, "cpu_baseline_1thread": cb1, "clocks": info["clocks"],
                "parity": info["parity"],
                "plain_per_walker_gpu": {"value": world * info["plain_value"], "unit": "walker-steps/s",
                                         "launches_per_step": info["plain_launches"],
                                         "speedup_batched_vs_plain": info["plain_ms"] / info["step_ms"]},
                "status": info["status"], "peaks_source": src,
            }
            print(json.dumps(line))
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.config == "c5":
        info = run_c5(args, torch)
        us = max_over_ranks(info["us_per_step"])
        if dist is not None:
            dist.barrier()
        if rank == 0:
            cb = None
            if not args.no_cpu_baseline and world == 1:
                cb = cpu_baseline_c5(info["w"], info["raw"])
            line = {
                "metric": "CV+bias+force us/step", "value": us, "unit": "us/step", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": us / 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": C5_WORKLOAD, "form": "through the C ABI, one CUDA graph",
                           "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}"},
                "e2e": {"value": info["e2e_us"], "unit": "us/step", "h2d_bytes_per_step": info["h2d"],
                        "d2h_bytes_per_step": info["d2h"]},
                "gpu_launches": C5_KERNELS_PER_STEP * args.steps,
                "roofline": None, "cpu_baseline": cb, "clocks": info["clocks"], "peaks_source": src,
                "parity": info["parity"],
            }
            print(json.dumps(line))
        if dist is not None:
            dist.destroy_process_group()
        return

    info = run_single(args, torch, args.config)
    us = max_over_ranks(info["us_per_step"])
    if dist is not None:
        dist.barrier()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    fp32 = ctypes.c_double()
    _native.call("glued_measure_fp32_peak", ctypes.byref(fp32))
    w = info["w"]
    roof = None
    if info["dominant"] == "coord_pairs":
        pairs = sum((len(a) - 1 - a[0]) * a[0] for t, a, p in w.cvs if t == 6)
        flops = pairs * FLOP_PAIR
        ach = flops / (info["dom_ms"] * 1e-3) / 1e12
        roof = {"bound": "fp32", "kernel": "k_coord_run", "achieved": ach, "peak": fp32.value,
                "unit": "TFLOP/s", "frac": ach / fp32.value, "traffic": TRAFFIC_C2_COORD,
                "traffic_unit": "bytes per launch",
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture "
                                  "(profiles/k_coord_run_c2.md)",
                "peak_source": "FP32 FMA microkernel measured in this run (MEASURED_PEAKS.json has no FP32 figure)",
                "algorithmic": f"{pairs} pairs x {FLOP_PAIR:.0f} flop"}
    cb = None
    if not args.no_cpu_baseline and world == 1:
        cb = cpu_baseline_single(args.config, w)
    line = {
        "metric": "CV+bias+force us/step", "value": us, "unit": "us/step", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": us / 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": info["workload"], "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": info["e2e_us"], "unit": "us/step", "h2d_bytes_per_step": info["h2d"],
                "d2h_bytes_per_step": info["d2h"]},
        "gpu_launches": int(round(info["kernels_per_step"] * args.steps)),
        "roofline": roof, "cpu_baseline": cb, "clocks": info["clocks"],
        "phases_ms": info["phases_ms"], "peaks_source": src, "parity": info["parity"],
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
