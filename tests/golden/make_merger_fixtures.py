"""Generates the bias-state merger fixtures in this folder.

Two stages, run on different machines:

``python tests/golden/make_merger_fixtures.py blobs``
    (GPU, this library) For each scenario, three walker groups (separate
    contexts, different seeded trajectories) run 30 steps and write their
    ``getBiasState()`` blobs (round 1); the groups' blobs are merged with
    ``gluedmd_b200.merger`` (first sync), every group loads the merged state,
    runs 30 more steps and writes its blob again (round 2).  Output:
    ``merger_blobs.npz`` (blobs + the bias lists as JSON).

``python tests/golden/make_merger_fixtures.py expected --reference <tree>``
    (CPU, the reference tree present) Imports the reference's
    ``python/MultiGPUManager.py`` unchanged (``openmm`` stubbed, ``gluedplugin``
    = this library's module, as the reference's own tests do with a stub) and
    runs its ``BiasStateMerger.merge_additive_incremental`` on round 1
    (baselines None) and on round 2 (with the baselines it returned).  Output:
    ``merger_expected.npz``: its merged blobs, or the error it raised.

Scenarios: 1-D MetaD (64 periodic bins), PBMETAD on two dihedrals, OPES on two
distances with adaptive sigma (Welford statistics, so the Chan combination is
exercised), all three in one force, and 2-D MetaD (64 x 64), whose grid size
the reference helper reads from an interleaved parameter layout.
"""
import argparse
import json
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
KT = 2.494338785

DIH = [(3, [0, 1, 2, 3], []), (3, [1, 2, 3, 4], [])]
DIST = [(1, [5, 6], []), (1, [7, 8], [])]
CVS = DIH + DIST          # CV 0, 1: dihedrals; CV 2, 3: distances
N_ATOMS = 9

METAD1 = (3, [0], [1.2, 0.35, 10.0, KT, -math.pi, math.pi], [2, 64, 1])
METAD2 = (3, [0, 1], [1.2, 0.35, 0.35, 10.0, KT, -math.pi, -math.pi, math.pi, math.pi], [2, 64, 64, 1, 1])
PBMETAD = (4, [0, 1], [1.0, 8.0, KT, 0.35, -math.pi, math.pi, 0.35, -math.pi, math.pi], [3, 64, 1, 64, 1])
OPES = (5, [2, 3], [KT, 20.05, 0.0, 0.0, 0.02], [0, 1, 100000, 6])

SCENARIOS = {
    "metad1d": [METAD1],
    "pbmetad": [PBMETAD],
    "opes_adaptive": [OPES],
    "combined": [OPES, METAD1, PBMETAD],
    "metad2d": [METAD2],
}
GROUPS, STEPS = 3, 30


class SpecForce:
    """getNumBiases / getBiasParameters over a fixed bias list: the only force
    methods either merger calls."""

    def __init__(self, biases):
        self.biases = [tuple(b) for b in biases]

    def getNumBiases(self):
        return len(self.biases)

    def getBiasParameters(self, i):
        t, c, p, ip = self.biases[i]
        return t, list(c), list(p), list(ip)


def load_blobs(path=os.path.join(HERE, "merger_blobs.npz")):
    """{scenario: (biases, [round-1 blobs], [round-2 blobs])}"""
    z = np.load(path)
    out = {}
    for name in json.loads(bytes(z["scenarios"]).decode()):
        biases = json.loads(bytes(z[f"{name}/biases"]).decode())
        r = [[bytes(z[f"{name}/r{k}/{g}"]) for g in range(GROUPS)] for k in (1, 2)]
        out[name] = (biases, r[0], r[1])
    return out


def load_expected(path=os.path.join(HERE, "merger_expected.npz")):
    """{scenario: {"r1": blob or error text, "r1_error": bool, "r2": ..., "r2_error": ...}}"""
    z = np.load(path)
    out = {}
    for name in json.loads(bytes(z["scenarios"]).decode()):
        e = {}
        for k in ("r1", "r2"):
            e[k + "_error"] = bool(z[f"{name}/{k}_error"])
            raw = bytes(z[f"{name}/{k}"])
            e[k] = raw.decode() if e[k + "_error"] else raw
        out[name] = e
    return out


def import_reference_merger(reference):
    """The reference's MultiGPUManager module, imported from its tree unchanged:
    ``openmm`` / ``openmm.unit`` are stand-ins whose every attribute is an empty
    class (the merger uses neither; annotations elsewhere in the module name them) and
    ``gluedplugin`` is this library's module (the merger reads its BIAS_*
    constants)."""
    import importlib.util
    sys.path.insert(0, ROOT)
    from gluedmd_b200 import gluedplugin
    mm = types.ModuleType("openmm")
    mm.__getattr__ = lambda name: type(name, (), {})   # annotations name mm.Context, mm.Platform, ...
    mm.unit = types.ModuleType("openmm.unit")
    saved = {k: sys.modules.get(k) for k in ("openmm", "openmm.unit", "gluedplugin")}
    sys.modules.update({"openmm": mm, "openmm.unit": mm.unit, "gluedplugin": gluedplugin})
    try:
        path = os.path.join(reference, "python", "MultiGPUManager.py")
        spec = importlib.util.spec_from_file_location("glued_ref_multigpu", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


def run_reference(mod, biases, r1, r2):
    """The reference merger on round 1 (first sync) and round 2 (incremental):
    (blob | error text, is_error) per round."""
    M = mod.BiasStateMerger
    f = SpecForce(biases)
    out = {}
    try:
        m1, base = M.merge_additive_incremental(r1, f, None)
        out["r1"] = (m1, False)
    except Exception as e:  # the recorded behaviour, e.g. a mis-sized 2-D grid
        out["r1"] = (f"{type(e).__name__}: {e}", True)
        out["r2"] = ("round 1 failed", True)
        return out
    try:
        m2, _ = M.merge_additive_incremental(r2, f, base)
        out["r2"] = (m2, False)
    except Exception as e:
        out["r2"] = (f"{type(e).__name__}: {e}", True)
    return out


def make_blobs(out_path):
    """Round-1 and round-2 blobs of every scenario from this library's contexts."""
    sys.path.insert(0, TESTS)
    sys.path.insert(0, ROOT)
    import gpu_util
    from gluedmd_b200.merger import BiasStateMerger
    arrays = {"scenarios": np.frombuffer(json.dumps(list(SCENARIOS)).encode(), np.uint8)}
    for si, (name, biases) in enumerate(SCENARIOS.items()):
        f_spec = SpecForce(biases)
        groups = []
        for g in range(GROUPS):
            ctx, f = gpu_util.make_context(np.zeros((N_ATOMS, 3)), CVS, biases)
            groups.append((ctx, f, np.random.default_rng(1000 * si + g)))

        def run(step0):
            for ctx, f, rng in groups:
                for step in range(step0, step0 + STEPS):
                    ctx.setStepCount(step)
                    ctx.updateContextState()
                    ctx.setPositions(rng.uniform(0.0, 1.5, (N_ATOMS, 3)))
                    ctx.computeForces()
                ctx.setStepCount(step0 + STEPS)
                ctx.updateContextState()   # the deposit of the last step
            return [bytes(f.getBiasState()) for _, f, _ in groups]

        r1 = run(0)
        merged, _ = BiasStateMerger.merge_additive_incremental(r1, f_spec, None)
        for _, f, _ in groups:
            f.setBiasState(merged)
        r2 = run(STEPS + 1)
        arrays[f"{name}/biases"] = np.frombuffer(json.dumps(biases).encode(), np.uint8)
        for k, r in ((1, r1), (2, r2)):
            for g, b in enumerate(r):
                arrays[f"{name}/r{k}/{g}"] = np.frombuffer(b, np.uint8)
    np.savez_compressed(out_path, **arrays)


def make_expected(reference, out_path):
    mod = import_reference_merger(reference)
    arrays = {}
    blobs = load_blobs()
    arrays["scenarios"] = np.frombuffer(json.dumps(list(blobs)).encode(), np.uint8)
    for name, (biases, r1, r2) in blobs.items():
        for k, (v, err) in run_reference(mod, biases, r1, r2).items():
            arrays[f"{name}/{k}"] = np.frombuffer(v.encode() if err else v, np.uint8)
            arrays[f"{name}/{k}_error"] = np.array(err)
    np.savez_compressed(out_path, **arrays)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["blobs", "expected"])
    ap.add_argument("--reference", default=os.environ.get("GLUED_REFERENCE", ""))
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.stage == "blobs":
        make_blobs(a.out or os.path.join(HERE, "merger_blobs.npz"))
    else:
        if not a.reference:
            sys.exit("expected: give --reference <tree> (or set GLUED_REFERENCE)")
        make_expected(a.reference, a.out or os.path.join(HERE, "merger_expected.npz"))
