"""ctypes binding of the C ABI in include/lfts_b200.h (liblfts_b200.so).

This is the binding a non-C++ host would add; the tests use it to call the
engine entry points directly.  Loading fails loudly when the shared library
has not been built: there is no CPU fallback.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblfts_b200.so")


class StepJob(C.Structure):
    _fields_ = [("in_", C.c_void_p), ("in_stride", C.c_longlong), ("out", C.c_void_p), ("out_stride", C.c_longlong),
                ("fac", C.c_void_p), ("bond", C.c_void_p), ("bond_half", C.c_void_p), ("spec", C.c_void_p),
                ("active", C.c_void_p), ("replica", C.c_int), ("pad", C.c_int)]


class JunctionJob(C.Structure):
    _fields_ = [("out", C.c_void_p), ("fac", C.c_void_p), ("ndeps", C.c_int), ("mode", C.c_int),
                ("dep_offset", C.c_int), ("pad", C.c_int)]


class DotJob(C.Structure):
    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p), ("w", C.c_void_p), ("scale", C.c_double)]


class PhiJob(C.Structure):
    _fields_ = [("q_left", C.c_void_p), ("q_right", C.c_void_p), ("fac", C.c_void_p), ("phi", C.c_void_p),
                ("norm", C.c_double), ("q_div", C.c_void_p), ("n_left", C.c_int), ("n_right", C.c_int),
                ("coef_offset", C.c_int), ("pad", C.c_int)]


class StressJob(C.Structure):
    _fields_ = [("q1", C.c_void_p), ("q2", C.c_void_p), ("bond", C.c_void_p), ("weight", C.c_double)]


_SIGS = {
    "lfts_ctx_create": [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int],
    "lfts_ctx_destroy": [C.c_void_p],
    "lfts_ctx_set_stream": [C.c_void_p, C.c_void_p],
    "lfts_ctx_info": [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_int)],
    "lfts_malloc": [C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t],
    "lfts_free": [C.c_void_p, C.c_void_p],
    "lfts_malloc_host": [C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t],
    "lfts_free_host": [C.c_void_p, C.c_void_p],
    "lfts_memset_async": [C.c_void_p, C.c_void_p, C.c_int, C.c_size_t],
    "lfts_memcpy_h2d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "lfts_memcpy_d2h": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "lfts_memcpy_d2d_async": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t],
    "lfts_synchronize": [C.c_void_p],
    "lfts_graph_begin": [C.c_void_p],
    "lfts_graph_end": [C.c_void_p, C.POINTER(C.c_void_p)],
    "lfts_graph_launch": [C.c_void_p, C.c_void_p],
    "lfts_graph_destroy": [C.c_void_p],
    "lfts_bond_tables": [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_void_p, C.c_void_p],
    "lfts_fourier_basis": [C.c_void_p, C.POINTER(C.c_double), C.c_void_p],
    "lfts_field_factors": [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p],
    "lfts_field_factors_batch": [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int],
    "lfts_step_continuous": [C.c_void_p, C.c_void_p, C.c_int, C.c_int],
    "lfts_step_discrete": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int],
    "lfts_junctions": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "lfts_dots": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "lfts_dots_static": [C.c_int, C.c_longlong, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "lfts_fft_forward": [C.c_void_p, C.c_void_p, C.c_int],
    "lfts_adam_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_double,
                         C.c_double, C.c_double, C.c_double, C.c_int],
    "lfts_sf_accumulate": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                           C.c_void_p],
    "lfts_phi_blocks": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p],
    "lfts_stress": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "lfts_am_dots": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_longlong, C.c_void_p, C.c_int, C.c_int],
    "lfts_am_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_longlong,
                       C.c_int, C.c_int],
    "lfts_am_simple": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_longlong],
    "lfts_lincomb": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong],
    "lfts_solvent": [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    "lfts_lfts_monomer_fields": [C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_lfts_field_deriv": [C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_lfts_langevin": [C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_lfts_row_moments": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_longlong,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_lfts_subtract_mean": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p],
    "lfts_am_batch_insert": [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p],
    "lfts_am_batch_dots": [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.c_void_p],
    "lfts_am_batch_update": [C.c_void_p, C.c_int, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_longlong],
    "lfts_saddle_control": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,
                            C.c_double, C.c_void_p],
    "lfts_am_batch_solve": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p],
    "lfts_status_post": [C.c_void_p, C.c_void_p, C.c_int],
    "lfts_status_wait": [C.c_void_p, C.c_int, C.c_void_p],
    "lfts_autotune": [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_size_t],
    "lfts_step_impl": [C.c_void_p, C.c_char_p, C.c_size_t],
    "lfts_realspace_tables": [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_step_realspace": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int],
    "lfts_set_step_impl": [C.c_void_p, C.c_char_p],
    "lfts_graph_while_begin": [C.c_void_p, C.POINTER(C.c_ulonglong)],
    "lfts_graph_while_end": [C.c_void_p],
    "lfts_saddle_begin": [C.c_void_p, C.c_int, C.c_double, C.c_void_p],
    "lfts_saddle_next": [C.c_void_p, C.c_ulonglong, C.c_void_p, C.c_int],
    "lfts_lfts_step_finish": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_double, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "lfts_pcg64_raw": [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p],
    "lfts_pcg64_normal": [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_double, C.c_void_p],
    "lfts_conv3d_bf16": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                         C.c_int, C.c_int, C.c_int, C.c_int],
    "lfts_relu_grad_bf16": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_int],
    "lfts_adamw_f32": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_double,
                       C.c_double, C.c_double, C.c_double, C.c_int],
    "lfts_conv3d_wgrad_bf16": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_int],
}

_lib = None


def lib():
    """Load liblfts_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run __graft_entry__.build() first")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.lfts_last_error.restype = C.c_char_p
        L.lfts_last_error.argtypes = []
        L.lfts_ctx_stream.restype = C.c_void_p
        L.lfts_ctx_stream.argtypes = [C.c_void_p]
        L.lfts_ctx_launches.restype = C.c_longlong
        L.lfts_ctx_launches.argtypes = [C.c_void_p]
        L.lfts_realspace_table_size.restype = C.c_longlong
        L.lfts_realspace_table_size.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def declared_symbols():
    """Names of every entry point declared in include/lfts_b200.h."""
    return list(_SIGS) + ["lfts_last_error", "lfts_ctx_stream", "lfts_ctx_launches", "lfts_realspace_table_size"]


def check(rc):
    if rc != 0:
        raise RuntimeError(lib().lfts_last_error().decode())


class Context:
    """Owns an lfts_ctx; convenience for tests and the benchmark."""

    def __init__(self, nx, precision=8, device=0):
        self.lib = lib()
        self.nx = list(nx)
        arr = (C.c_int * len(nx))(*nx)
        h = C.c_void_p()
        check(self.lib.lfts_ctx_create(C.byref(h), device, len(nx), arr, precision))
        self.h = h
        M, Mc, p = C.c_longlong(), C.c_longlong(), C.c_int()
        check(self.lib.lfts_ctx_info(h, C.byref(M), C.byref(Mc), C.byref(p)))
        self.M, self.Mc, self.prec = M.value, Mc.value, p.value
        self._allocs = []

    def close(self):
        for p in self._allocs:
            self.lib.lfts_free(self.h, p)
        self._allocs = []
        if self.h:
            self.lib.lfts_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def malloc(self, nbytes):
        p = C.c_void_p()
        check(self.lib.lfts_malloc(self.h, C.byref(p), nbytes))
        self._allocs.append(p.value)
        return p.value

    def h2d(self, dst, arr):
        import numpy as np
        a = np.ascontiguousarray(arr)
        check(self.lib.lfts_memcpy_h2d(self.h, dst, a.ctypes.data, a.nbytes))

    def d2h(self, src, shape, dtype):
        import numpy as np
        out = np.empty(shape, dtype=dtype)
        check(self.lib.lfts_memcpy_d2h(self.h, out.ctypes.data, src, out.nbytes))
        return out

    def upload(self, arr):
        import numpy as np
        a = np.ascontiguousarray(arr)
        p = self.malloc(max(a.nbytes, 16))
        self.h2d(p, a)
        return p

    def sync(self):
        check(self.lib.lfts_synchronize(self.h))
