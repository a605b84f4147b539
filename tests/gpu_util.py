"""Helpers shared by the GPU tests: build a product context from CV/bias specs
and run it, mirroring what the oracle runs."""
import numpy as np

from gluedmd_b200 import GluedForce
from gluedmd_b200.context import Context, System


def make_force(cvs, biases=(), pbc=False, grad=None, temperature=300.0):
    f = GluedForce()
    f.setTemperature(temperature)
    f.setUsesPeriodicBoundaryConditions(bool(pbc))
    for t, a, p in cvs:
        f.addCollectiveVariable(t, [int(x) for x in a], [float(x) for x in p])
    for t, c, p, ip in biases:
        f.addBias(t, c, p, ip)
    if grad is not None:
        f.setTestBiasGradients(list(grad))
    return f


def make_context(pos, cvs, biases=(), masses=None, pbc=False, box=None, grad=None, reorder=None, blob=None):
    pos = np.asarray(pos, float)
    n = len(pos)
    s = System()
    for i in range(n):
        s.addParticle(1.0 if masses is None else masses[i])
    f = make_force(cvs, biases, pbc, grad)
    s.addForce(f)
    if box is not None:
        b = np.asarray(box, float).reshape(3, 3)
        s.setDefaultPeriodicBoxVectors(b[0], b[1], b[2])
    ctx = Context(s, pos, reorder=reorder)
    if blob:
        f.setBiasState(blob)
    return ctx, f


def run(pos, cvs, biases=(), **kw):
    ctx, f = make_context(pos, cvs, biases, **kw)
    e, F = ctx.computeForces()
    return dict(energy=e, forces=F, cv_values=np.array(f.getLastCVValues(ctx)), ctx=ctx, force=f)
