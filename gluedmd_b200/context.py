"""Standalone host harness that drives GluedForce contexts the way OpenMM does.

OpenMM is not part of this library. ``System`` and ``Context`` here provide the
pieces of OpenMM's runtime the hot path touches: particle masses, a float4
``posq`` array in device memory with an optional GPU-slot reordering
(``atomIndexArray``), the 2^32 fixed-point ``int64`` force buffer, periodic box
vectors, the step counter, and the call order of one MD step (updateState before
the force evaluation, GluedForceImpl.cpp:100-119). Device memory and streams come
from PyTorch; all arithmetic runs in the native library.

No dynamics are integrated: ``step()`` advances the step counter and runs the
force evaluation with the current positions, so callers set positions between
steps (as the reference's tests do).
"""
from __future__ import annotations

import numpy as np
import torch

from .gluedplugin import GluedForce, NativeContext

FIXED = 4294967296.0  # 2^32


class System:
    """Masses, forces and default box: the parts of openmm.System used here."""

    def __init__(self):
        self.masses = []
        self.forces = []
        self.box = None

    def addParticle(self, mass=1.0):
        self.masses.append(float(mass))
        return len(self.masses) - 1

    def getNumParticles(self):
        return len(self.masses)

    def getParticleMass(self, i):
        return self.masses[i]

    def setParticleMass(self, i, m):
        self.masses[i] = float(m)

    def addForce(self, force):
        self.forces.append(force)
        return len(self.forces) - 1

    def setDefaultPeriodicBoxVectors(self, a, b, c):
        self.box = np.array([a, b, c], dtype=np.float64)


class State:
    def __init__(self, energy, forces, positions, step):
        self._e, self._f, self._p, self._s = energy, forces, positions, step

    def getPotentialEnergy(self):
        return self._e

    def getForces(self, asNumpy=True):
        return self._f

    def getPositions(self, asNumpy=True):
        return self._p

    def getStepCount(self):
        return self._s


class Context:
    """A device-resident context holding posq / force buffers for one system.

    reorder: optional permutation; ``posq[slot]`` holds user atom ``reorder[slot]``
    (OpenMM's atomIndexArray), to exercise the user -> slot mapping.
    """

    def __init__(self, system: System, positions=None, device="cuda:0", reorder=None, padding=32):
        self.system = system
        self.device = torch.device(device)
        self.n = system.getNumParticles()
        self.padded = ((self.n + padding - 1) // padding) * padding if self.n else padding
        self.posq = torch.zeros((self.padded, 4), dtype=torch.float32, device=self.device)
        self.force_buf = torch.zeros(3 * self.padded, dtype=torch.int64, device=self.device)
        perm = np.arange(self.n) if reorder is None else np.asarray(reorder, dtype=np.int64)
        self.atom_index = torch.as_tensor(perm, dtype=torch.int32, device=self.device)
        self._perm = perm
        self.step_count = 0
        self._last_update = {}
        self.stream = torch.cuda.current_stream(self.device)
        self._glued = {}
        box = system.box
        for f in system.forces:
            if isinstance(f, GluedForce):
                nc = NativeContext(f, self.n, system.masses)
                nc.bind(self.stream.cuda_stream, self.posq.data_ptr(), self.atom_index.data_ptr(),
                        self.force_buf.data_ptr(), self.padded)
                self._glued[id(f)] = (f, nc)
                self._last_update[id(f)] = -1
        if box is not None:
            self.setPeriodicBoxVectors(*box)
        if positions is not None:
            self.setPositions(positions)

    # ---------------------------------------------------------------- state
    def glued_context_for(self, force):
        try:
            return self._glued[id(force)][1]
        except KeyError:
            raise RuntimeError("this GluedForce is not part of the Context's System") from None

    def setPositions(self, positions):
        p = torch.as_tensor(np.asarray(positions, dtype=np.float64), dtype=torch.float32).reshape(-1, 3)
        if p.shape[0] != self.n:
            raise ValueError(f"expected {self.n} positions, got {p.shape[0]}")
        slots = torch.as_tensor(self._perm, dtype=torch.int64)
        host = torch.zeros((self.padded, 4), dtype=torch.float32)
        host[: self.n, :3] = p[slots]
        self.posq.copy_(host.to(self.device, non_blocking=False))

    def setPositionsDevice(self, posq_tensor):
        """Copy a device float4 posq array (slot order) in without a host round trip."""
        self.posq[: posq_tensor.shape[0]].copy_(posq_tensor)

    def setPeriodicBoxVectors(self, a, b, c):
        box = np.array([a, b, c], dtype=np.float64).reshape(9)
        for _, nc in self._glued.values():
            nc.set_box(box)

    def reorderAtoms(self, reorder):
        """Apply a new GPU-slot order (OpenMM's periodic atom reordering)."""
        pos = self.getPositions()
        self._perm = np.asarray(reorder, dtype=np.int64)
        self.atom_index.copy_(torch.as_tensor(self._perm, dtype=torch.int32, device=self.device))
        self.setPositions(pos)
        for _, nc in self._glued.values():
            nc.atoms_reordered()

    def getPositions(self):
        q = self.posq[: self.n, :3].double().cpu().numpy()
        out = np.empty_like(q)
        out[self._perm] = q
        return out

    # ------------------------------------------------------------- evaluate
    def computeForces(self, groups=0xFFFFFFFF, include_energy=True, include_forces=True):
        """calcForcesAndEnergy: zero the force buffer, run every GluedForce whose
        force group is selected. Returns (energy, forces (n,3) in user order)."""
        self.force_buf.zero_()
        e = 0.0
        for f, nc in self._glued.values():
            if groups & (1 << f.getForceGroup()):
                e += nc.execute(include_forces, include_energy)
        return e, self.forces_from_buffer() if include_forces else None

    def forces_from_buffer(self):
        fb = self.force_buf.view(3, self.padded)[:, : self.n].cpu().numpy().astype(np.float64) / FIXED
        out = np.empty((self.n, 3))
        out[self._perm] = fb.T
        return out

    def getState(self, getEnergy=False, getForces=False, getPositions=False, groups=0xFFFFFFFF):
        e, f = self.computeForces(groups, include_energy=True, include_forces=True)
        return State(e, f, self.getPositions() if getPositions else None, self.step_count)

    def updateContextState(self):
        """GluedForceImpl::updateContextState: updateState once per step."""
        for key, (f, nc) in self._glued.items():
            if self.step_count != self._last_update[key]:
                nc.update_state(self.step_count)
                self._last_update[key] = self.step_count

    def step(self, n=1):
        """Per step: updateState(step), force evaluation, step += 1."""
        for _ in range(n):
            self.updateContextState()
            self.computeForces(include_energy=False)
            self.step_count += 1

    def getStepCount(self):
        return self.step_count

    def setStepCount(self, s):
        self.step_count = int(s)
