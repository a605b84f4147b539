"""Python mirror of GLUED's SWIG module ``gluedplugin`` (python/gluedplugin.i).

``GluedForce`` has the reference's method names, argument meanings and error
behaviour, backed by the C ABI of include/glued_b200.h. Methods that take an
OpenMM ``Context`` in the reference take a :class:`gluedmd_b200.context.Context`
here (or any object exposing ``glued_context_for(force)``).

Importable as ``gluedplugin`` so that GLUED's own ``python/glued.py`` runs on top
of it unchanged (it needs only this module and ``openmm.vectori/vectord``).
"""
from __future__ import annotations

import ctypes

from ._native import (GluedError, call, int_array, dbl_array, c_int, c_double, c_size_t, c_void_p, c_float, c_ll,
                      lib)

__version__ = "0.1"


class OpenMMException(GluedError):
    """Alias so callers can catch the reference's exception name."""


def _ints(seq):
    return [int(x) for x in seq]


def _dbls(seq):
    return [float(x) for x in seq]


class GluedForce:
    """GluedForce (openmmapi/include/GluedForce.h:24-276)."""

    CV_DISTANCE, CV_ANGLE, CV_DIHEDRAL, CV_COM_DISTANCE, CV_GYRATION = 1, 2, 3, 4, 5
    CV_COORDINATION, CV_RMSD, CV_EXPRESSION, CV_PYTORCH, CV_PATH = 6, 7, 8, 9, 10
    CV_POSITION, CV_DRMSD, CV_CONTACTMAP, CV_PLANE, CV_PROJECTION = 11, 12, 13, 14, 15
    CV_PUCKERING, CV_DIPOLE, CV_VOLUME, CV_CELL, CV_SECONDARY_STRUCTURE = 16, 17, 18, 19, 20
    CV_PCA, CV_ERMSD, CV_ENERGY = 21, 22, 23
    # extensions of this library
    CV_COORDINATION_CUTOFF, CV_RMSD_KABSCH = 106, 107

    BIAS_HARMONIC, BIAS_MOVING_RESTRAINT, BIAS_METAD, BIAS_PBMETAD, BIAS_OPES = 1, 2, 3, 4, 5
    BIAS_EXTERNAL, BIAS_ABMD, BIAS_UPPER_WALL, BIAS_LOWER_WALL, BIAS_LINEAR = 6, 7, 8, 9, 10
    BIAS_OPES_EXPANDED, BIAS_EXT_LAGRANGIAN, BIAS_MAXENT, BIAS_EDS, BIAS_OPES_MULTITHERMAL = 11, 12, 13, 14, 15
    # extension: direct hill-sum metadynamics
    BIAS_METAD_HILLS = 103

    def __init__(self, *args):
        h = c_void_p()
        if len(args) == 1 and isinstance(args[0], GluedForce):
            call("glued_force_copy", args[0]._h, ctypes.byref(h))
        else:
            call("glued_force_create", ctypes.byref(h))
        self._h = h
        self._context = None  # most recently created context (GluedForce::impl_)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().glued_force_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------- CVs
    def addCollectiveVariable(self, type, atoms, parameters=()):
        a, na = int_array(_ints(atoms))
        p, np_ = dbl_array(_dbls(parameters))
        out = c_int()
        call("glued_force_add_cv", self._h, int(type), a, na, p, np_, ctypes.byref(out))
        return out.value

    def getNumCollectiveVariables(self):
        out = c_int(); call("glued_force_num_cv_values", self._h, ctypes.byref(out)); return out.value

    def getNumCollectiveVariableSpecs(self):
        out = c_int(); call("glued_force_num_cv_specs", self._h, ctypes.byref(out)); return out.value

    def getCollectiveVariableParameters(self, idx):
        t, na, np_ = c_int(), c_int(), c_int()
        call("glued_force_get_cv", self._h, int(idx), ctypes.byref(t), None, ctypes.byref(na), None, ctypes.byref(np_))
        a = (c_int * max(1, na.value))(); p = (c_double * max(1, np_.value))()
        call("glued_force_get_cv", self._h, int(idx), ctypes.byref(t), a, ctypes.byref(na), p, ctypes.byref(np_))
        return t.value, list(a[:na.value]), list(p[:np_.value])

    getCollectiveVariableInfo = getCollectiveVariableParameters

    def addExpressionCV(self, expression, inputCVIndices):
        a, n = int_array(_ints(inputCVIndices))
        out = c_int()
        call("glued_force_add_expression_cv", self._h, expression.encode(), a, n, ctypes.byref(out))
        return out.value

    def _cv_string(self, idx):
        n = c_size_t()
        call("glued_force_get_cv_string", self._h, int(idx), None, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        call("glued_force_get_cv_string", self._h, int(idx), buf, ctypes.byref(n))
        return buf.value.decode()

    def getExpressionCVInfo(self, specIdx):
        t, a, _ = self.getCollectiveVariableParameters(specIdx)
        if t != self.CV_EXPRESSION:
            raise OpenMMException(-1, "GluedForce: CV spec is not an expression CV")
        return self._cv_string(specIdx), a

    def addPyTorchCV(self, torchScriptPath, atomIndices, parameters=()):
        a, na = int_array(_ints(atomIndices))
        p, np_ = dbl_array(_dbls(parameters))
        out = c_int()
        call("glued_force_add_pytorch_cv", self._h, torchScriptPath.encode(), a, na, p, np_, ctypes.byref(out))
        return out.value

    def getPyTorchCVModelPath(self, specIdx):
        t, _, _ = self.getCollectiveVariableParameters(specIdx)
        if t != self.CV_PYTORCH:
            raise OpenMMException(-1, "GluedForce: CV spec is not a PyTorch CV")
        return self._cv_string(specIdx)

    # ----------------------------------------------------------- biases
    def addBias(self, type, cvIndices, parameters=(), integerParameters=()):
        c, nc = int_array(_ints(cvIndices))
        p, np_ = dbl_array(_dbls(parameters))
        ip, ni = int_array(_ints(integerParameters))
        out = c_int()
        call("glued_force_add_bias", self._h, int(type), c, nc, p, np_, ip, ni, ctypes.byref(out))
        return out.value

    def getNumBiases(self):
        out = c_int(); call("glued_force_num_biases", self._h, ctypes.byref(out)); return out.value

    def getBiasParameters(self, idx):
        t, nc, np_, ni = c_int(), c_int(), c_int(), c_int()
        call("glued_force_get_bias", self._h, int(idx), ctypes.byref(t), None, ctypes.byref(nc), None,
             ctypes.byref(np_), None, ctypes.byref(ni))
        c = (c_int * max(1, nc.value))(); p = (c_double * max(1, np_.value))(); ip = (c_int * max(1, ni.value))()
        call("glued_force_get_bias", self._h, int(idx), ctypes.byref(t), c, ctypes.byref(nc), p, ctypes.byref(np_),
             ip, ctypes.byref(ni))
        return t.value, list(c[:nc.value]), list(p[:np_.value]), list(ip[:ni.value])

    getBiasInfo = getBiasParameters

    # ----------------------------------------------------------- config
    def setTemperature(self, kelvin):
        call("glued_force_set_temperature", self._h, float(kelvin))

    def getTemperature(self):
        out = c_double(); call("glued_force_get_temperature", self._h, ctypes.byref(out)); return out.value

    @staticmethod
    def barrierToGamma(barrier_kJ, kT_kJ):
        return barrier_kJ / kT_kJ

    @staticmethod
    def kTFromTemperature(temperatureKelvin):
        return 8.314462618e-3 * temperatureKelvin

    def usesPeriodicBoundaryConditions(self):
        out = c_int(); call("glued_force_get_pbc", self._h, ctypes.byref(out)); return bool(out.value)

    def setUsesPeriodicBoundaryConditions(self, yes):
        call("glued_force_set_pbc", self._h, 1 if yes else 0)

    def setForceGroup(self, group):
        call("glued_force_set_force_group", self._h, int(group))

    def getForceGroup(self):
        out = c_int(); call("glued_force_get_force_group", self._h, ctypes.byref(out)); return out.value

    # -------------------------------------------------------- test hooks
    def setTestForce(self, mode, scale):
        call("glued_force_set_test_force", self._h, int(mode), float(scale))

    def getTestForceMode(self):
        m = c_int(); call("glued_force_get_test_force", self._h, ctypes.byref(m), None); return m.value

    def getTestForceScale(self):
        s = c_double(); call("glued_force_get_test_force", self._h, None, ctypes.byref(s)); return s.value

    def setTestBiasGradients(self, gradients):
        g, n = dbl_array(_dbls(gradients))
        call("glued_force_set_test_bias_gradients", self._h, g, n)

    def getTestBiasGradients(self):
        n = c_int()
        call("glued_force_get_test_bias_gradients", self._h, None, ctypes.byref(n))
        g = (c_double * max(1, n.value))()
        call("glued_force_get_test_bias_gradients", self._h, g, ctypes.byref(n))
        return list(g[:n.value])

    # --------------------------------------------------------------- XML
    def toXml(self):
        n = c_size_t()
        call("glued_force_serialize_xml", self._h, None, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value)
        call("glued_force_serialize_xml", self._h, buf, ctypes.byref(n))
        return buf.value.decode()

    @classmethod
    def fromXml(cls, xml):
        h = c_void_p()
        call("glued_force_deserialize_xml", xml.encode() if isinstance(xml, str) else xml, ctypes.byref(h))
        f = cls.__new__(cls)
        f._h = h
        f._context = None
        return f

    @staticmethod
    def cast(obj):
        return obj if isinstance(obj, GluedForce) else None

    # --------------------------------------------------- context-bound API
    def _ctx(self, context=None):
        if context is None:
            if self._context is None:
                raise OpenMMException(-3, "GluedForce::getBiasStateBytes: no Context created yet")
            return self._context
        return context.glued_context_for(self)

    def getBiasStateBytes(self):
        return self._ctx().get_bias_state()

    def setBiasStateBytes(self, data):
        self._ctx().set_bias_state(bytes(data))

    def getBiasState(self):
        return self._ctx().get_bias_state()

    def setBiasState(self, data):
        if not isinstance(data, (bytes, bytearray)):
            raise OpenMMException(-1, "setBiasState: expected bytes or bytearray")
        self._ctx().set_bias_state(bytes(data))

    def getCurrentCVValues(self, context):
        context.computeForces(groups=1 << self.getForceGroup(), include_energy=False)
        return self._ctx(context).cv_values()

    def getCurrentCollectiveVariables(self, context, values=None):
        v = self.getCurrentCVValues(context)
        if values is not None:
            values[:] = v
        return v

    def getLastCVValues(self, context):
        return self._ctx(context).cv_values()

    def getLastBias(self, context):
        return self._ctx(context).last_bias()

    def getOPESMetrics(self, context, biasIndex):
        return self._ctx(context).opes_metrics(biasIndex)

    def getKernelSigmas(self, context, biasIndex):
        return self._ctx(context).kernel_sigmas(biasIndex)

    def getMultiWalkerPtrs(self, context, biasIdx):
        return self._ctx(context).multiwalker_ptrs(biasIdx)

    def setMultiWalkerPtrs(self, context, biasIdx, ptrs):
        self._ctx(context).set_multiwalker_ptrs(biasIdx, ptrs)


class NativeContext:
    """One glued_context handle (the per-Context CalcGluedForceKernel)."""

    def __init__(self, force: GluedForce, num_particles: int, masses=None):
        m = None
        if masses is not None:
            m, _ = dbl_array(masses)
        h = c_void_p()
        call("glued_context_create", force._h, int(num_particles), m, ctypes.byref(h))
        self._h = h
        self.force = force
        self.num_particles = int(num_particles)
        force._context = self

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().glued_context_destroy(h)
            except Exception:
                pass
            self._h = None

    def bind(self, stream, posq_ptr, atom_index_ptr, force_ptr, padded):
        call("glued_context_bind", self._h, c_void_p(stream), c_void_p(posq_ptr), c_void_p(atom_index_ptr),
             c_void_p(force_ptr), int(padded))

    def atoms_reordered(self):
        call("glued_context_atoms_reordered", self._h)

    def set_box(self, box9):
        b, _ = dbl_array(box9)
        call("glued_context_set_box", self._h, b)

    def execute(self, include_forces=True, include_energy=True):
        e = c_double()
        call("glued_context_execute", self._h, 1 if include_forces else 0, 1 if include_energy else 0,
             ctypes.byref(e))
        return e.value

    def update_state(self, step):
        call("glued_context_update_state", self._h, int(step))

    def num_cvs(self):
        n = c_int()
        call("glued_context_device_arrays", self._h, None, None, None, None, None, None, None, ctypes.byref(n), None)
        return n.value

    def cv_values(self):
        n = self.num_cvs()
        out = (c_double * max(1, n))()
        call("glued_context_get_cv_values", self._h, out, n)
        return list(out[:n])

    def last_bias(self):
        e = c_double()
        call("glued_context_get_last_bias", self._h, ctypes.byref(e))
        return e.value

    def get_bias_state(self):
        n = c_size_t()
        call("glued_context_get_bias_state", self._h, None, ctypes.byref(n))
        buf = ctypes.create_string_buffer(max(1, n.value))
        call("glued_context_get_bias_state", self._h, buf, ctypes.byref(n))
        return buf.raw[:n.value]

    def set_bias_state(self, data: bytes):
        call("glued_context_set_bias_state", self._h, data, len(data))

    def opes_metrics(self, idx):
        out = (c_double * 4)()
        call("glued_context_opes_metrics", self._h, int(idx), out)
        return list(out)

    def kernel_sigmas(self, idx):
        n = c_int()
        call("glued_context_kernel_sigmas", self._h, int(idx), None, ctypes.byref(n))
        out = (c_float * max(1, n.value))()
        call("glued_context_kernel_sigmas", self._h, int(idx), out, ctypes.byref(n))
        return list(out[:n.value])

    def multiwalker_ptrs(self, idx):
        n = c_int()
        call("glued_context_multiwalker_ptrs", self._h, int(idx), None, ctypes.byref(n))
        out = (c_ll * max(1, n.value))()
        call("glued_context_multiwalker_ptrs", self._h, int(idx), out, ctypes.byref(n))
        return list(out[:n.value])

    def set_multiwalker_ptrs(self, idx, ptrs):
        arr = (c_ll * max(1, len(ptrs)))(*[int(p) for p in ptrs])
        call("glued_context_set_multiwalker_ptrs", self._h, int(idx), arr, len(ptrs))

    def opes_last_decision(self, idx):
        d = c_int()
        call("glued_context_opes_last_decision", self._h, int(idx), ctypes.byref(d))
        return d.value

    SUM_FP64, SUM_FP32, SUM_FP32_TWOSUM = 0, 1, 2

    def set_sum_precision(self, kernel_sums=0, coordination=0):
        """glued_context_set_sum_precision: kernel_sums 0 FP64 / 1 FP32 / 2 FP32
        two-sum; coordination 0 per tile run / 1 blocked."""
        call("glued_context_set_sum_precision", self._h, int(kernel_sums), int(coordination))

    def sum_precision(self):
        k, c = c_int(), c_int()
        call("glued_context_get_sum_precision", self._h, ctypes.byref(k), ctypes.byref(c))
        return k.value, c.value

    def coordination_pairs(self, cv_index):
        """glued_context_coordination_pairs: sorted (a, b) group indices, shape (n, 2)."""
        import numpy as np
        n = c_ll()
        call("glued_context_coordination_pairs", self._h, int(cv_index), None, 0, ctypes.byref(n))
        out = np.zeros(2 * max(1, n.value), dtype=np.int32)
        call("glued_context_coordination_pairs", self._h, int(cv_index),
             out.ctypes.data_as(ctypes.POINTER(c_int)), n.value, ctypes.byref(n))
        return out[:2 * n.value].reshape(-1, 2)

    def profile_phases(self, reps=20):
        n = c_int(6)
        out = (c_double * 6)()
        call("glued_context_profile_phases", self._h, int(reps), out, ctypes.byref(n))
        return list(out[:n.value])

    def launch_count(self):
        v = c_ll()
        call("glued_context_launch_count", self._h, ctypes.byref(v))
        return v.value

    def device_arrays(self):
        ptrs = [c_void_p() for _ in range(7)]
        nc, nr = c_int(), c_int()
        call("glued_context_device_arrays", self._h, *[ctypes.byref(p) for p in ptrs], ctypes.byref(nc),
             ctypes.byref(nr))
        return [p.value for p in ptrs], nc.value, nr.value
