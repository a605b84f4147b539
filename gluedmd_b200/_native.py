"""ctypes binding of the in-tree native library (include/glued_b200.h).

The library is the only implementation of the hot path: if it is missing the
import fails loudly (there is no CPU fallback)."""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libglued_b200.so")

c_int, c_double, c_float, c_char_p, c_void_p, c_size_t, c_ll = (
    ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t,
    ctypes.c_longlong)
P = ctypes.POINTER

GLUED_E = {-1: "invalid argument", -2: "CUDA error", -3: "invalid state", -4: "corrupt bias state",
           -5: "unsupported"}


class GluedError(RuntimeError):
    """Raised for every non-zero status of the C ABI (the reference raises
    OpenMMException for the same conditions)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class WalkerDesc(ctypes.Structure):
    _fields_ = [("posq", c_void_p), ("force_buffer", c_void_p), ("num_atoms", c_int),
                ("padded_num_atoms", c_int), ("box", c_double * 9)]


_SIGS = {
    "glued_force_create": [P(c_void_p)],
    "glued_force_copy": [c_void_p, P(c_void_p)],
    "glued_force_destroy": [c_void_p],
    "glued_force_add_cv": [c_void_p, c_int, P(c_int), c_int, P(c_double), c_int, P(c_int)],
    "glued_force_add_bias": [c_void_p, c_int, P(c_int), c_int, P(c_double), c_int, P(c_int), c_int, P(c_int)],
    "glued_force_add_expression_cv": [c_void_p, c_char_p, P(c_int), c_int, P(c_int)],
    "glued_force_add_pytorch_cv": [c_void_p, c_char_p, P(c_int), c_int, P(c_double), c_int, P(c_int)],
    "glued_force_num_cv_values": [c_void_p, P(c_int)],
    "glued_force_num_cv_specs": [c_void_p, P(c_int)],
    "glued_force_num_biases": [c_void_p, P(c_int)],
    "glued_force_get_cv": [c_void_p, c_int, P(c_int), P(c_int), P(c_int), P(c_double), P(c_int)],
    "glued_force_get_cv_string": [c_void_p, c_int, c_char_p, P(c_size_t)],
    "glued_force_get_bias": [c_void_p, c_int, P(c_int), P(c_int), P(c_int), P(c_double), P(c_int), P(c_int),
                             P(c_int)],
    "glued_force_set_temperature": [c_void_p, c_double],
    "glued_force_get_temperature": [c_void_p, P(c_double)],
    "glued_force_set_pbc": [c_void_p, c_int],
    "glued_force_get_pbc": [c_void_p, P(c_int)],
    "glued_force_set_force_group": [c_void_p, c_int],
    "glued_force_get_force_group": [c_void_p, P(c_int)],
    "glued_force_set_test_force": [c_void_p, c_int, c_double],
    "glued_force_get_test_force": [c_void_p, P(c_int), P(c_double)],
    "glued_force_set_test_bias_gradients": [c_void_p, P(c_double), c_int],
    "glued_force_get_test_bias_gradients": [c_void_p, P(c_double), P(c_int)],
    "glued_force_serialize_xml": [c_void_p, c_char_p, P(c_size_t)],
    "glued_force_deserialize_xml": [c_char_p, P(c_void_p)],
    "glued_context_create": [c_void_p, c_int, P(c_double), P(c_void_p)],
    "glued_context_destroy": [c_void_p],
    "glued_context_bind": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int],
    "glued_context_atoms_reordered": [c_void_p],
    "glued_context_set_box": [c_void_p, P(c_double)],
    "glued_context_set_step": [c_void_p, c_ll],
    "glued_context_execute": [c_void_p, c_int, c_int, P(c_double)],
    "glued_context_update_state": [c_void_p, c_int],
    "glued_context_get_cv_values": [c_void_p, P(c_double), c_int],
    "glued_context_get_last_bias": [c_void_p, P(c_double)],
    "glued_context_get_bias_state": [c_void_p, c_char_p, P(c_size_t)],
    "glued_context_set_bias_state": [c_void_p, c_char_p, c_size_t],
    "glued_context_opes_metrics": [c_void_p, c_int, P(c_double)],
    "glued_context_kernel_sigmas": [c_void_p, c_int, P(c_float), P(c_int)],
    "glued_context_multiwalker_ptrs": [c_void_p, c_int, P(c_ll), P(c_int)],
    "glued_context_set_multiwalker_ptrs": [c_void_p, c_int, P(c_ll), c_int],
    "glued_context_device_arrays": [c_void_p] + [P(c_void_p)] * 7 + [P(c_int), P(c_int)],
    "glued_context_opes_last_decision": [c_void_p, c_int, P(c_int)],
    "glued_context_set_sum_precision": [c_void_p, c_int, c_int],
    "glued_context_coordination_pairs": [c_void_p, c_int, P(c_int), c_ll, P(c_ll)],
    "glued_context_get_sum_precision": [c_void_p, P(c_int), P(c_int)],
    "glued_context_profile_phases": [c_void_p, c_int, P(c_double), P(c_int)],
    "glued_context_launch_count": [c_void_p, P(c_ll)],
    "glued_measure_fp32_peak": [P(c_double)],
    "glued_measure_hill_staging": [c_int, c_int, c_int, P(c_double), P(c_int)],
    "glued_ad_forward": [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int],
    "glued_ad_backward": [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                          c_void_p],
    "glued_coordination_noalloc": [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_double, c_double,
                                   c_double, c_int, P(c_double), c_void_p, c_void_p],
    "glued_batch_create": [P(c_void_p), c_int, P(WalkerDesc), P(c_void_p)],
    "glued_batch_destroy": [c_void_p],
    "glued_batch_set_stream": [c_void_p, c_void_p],
    "glued_batch_set_tuning": [c_void_p, P(c_int)],
    "glued_batch_get_tuning": [c_void_p, P(c_int)],
    "glued_batch_autotune": [c_void_p, P(c_int)],
    "glued_batch_autotune_ex": [c_void_p, c_int, P(c_int), P(c_int)],
    "glued_batch_set_sum_precision": [c_void_p, c_int],
    "glued_batch_get_sum_precision": [c_void_p, P(c_int)],
    "glued_batch_execute": [c_void_p],
    "glued_batch_update_state": [c_void_p, c_int],
    "glued_batch_get_energies": [c_void_p, P(c_double)],
    "glued_batch_get_cv_values": [c_void_p, P(c_double)],
    "glued_batch_num_cvs": [c_void_p, P(c_int)],
    "glued_batch_num_hills": [c_void_p, P(c_int)],
    "glued_batch_set_hills": [c_void_p, P(c_double), P(c_double), c_int],
    "glued_batch_get_hills": [c_void_p, P(c_double), P(c_double), c_int],
    "glued_batch_status": [c_void_p, P(c_int)],
    "glued_batch_launch_count": [c_void_p, P(c_ll)],
    "glued_batch_phase_times": [c_void_p, P(c_double)],
    "glued_batch_phase_stamps": [c_void_p, P(ctypes.c_ulonglong), c_ll, P(c_ll)],
}


def exported_symbols():
    return list(_SIGS) + ["glued_last_error", "glued_version"]


_lib = None


def lib():
    """Load the native library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"gluedmd_b200 native library not built: {LIB_PATH} missing "
                          "(run `python -m gluedmd_b200.build`)")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = c_int
    L.glued_last_error.restype = c_char_p
    L.glued_last_error.argtypes = []
    L.glued_version.restype = c_char_p
    L.glued_version.argtypes = []
    _lib = L
    return L


def check(rc):
    if rc != 0:
        msg = lib().glued_last_error().decode("utf-8", "replace")
        raise GluedError(rc, msg or GLUED_E.get(rc, f"error {rc}"))
    return rc


def call(name, *args):
    return check(getattr(lib(), name)(*args))


def int_array(seq):
    seq = [int(x) for x in seq]
    return (c_int * max(1, len(seq)))(*seq), len(seq)


def dbl_array(seq):
    seq = [float(x) for x in seq]
    return (c_double * max(1, len(seq)))(*seq), len(seq)
