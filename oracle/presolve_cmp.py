"""TEST INFRASTRUCTURE ONLY: the reference presolver against the fast one.

Wraps oracle/_ref/libpresolve_cmp.so (oracle/presolve_shim.cpp, built by
``make -C oracle presolve`` from the reference's sources): the reference's
presolve::Presolver::run and pdlpgpu::presolve_model run on the same
model::Model and their PresolveResults are compared field by field, doubles
by their bits. Also times either one on a model (the reference's timing leg
of the presolve measurement).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from optimisation_solver_b200 import native

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libpresolve_cmp.so")


def available() -> bool:
    return os.path.exists(LIB)


class PresolveCompare:
    def __init__(self):
        if not available():
            raise FileNotFoundError(f"{LIB} is not built (make -C oracle presolve)")
        native.lib()  # the shim links libpdlpgpu.so
        L = self.lib = C.CDLL(LIB)
        i64p = C.POINTER(C.c_int64)
        L.ps_compare.argtypes = [C.POINTER(native.PresolveModel), C.c_char_p, C.c_int, i64p]
        L.ps_compare_mps.argtypes = [C.c_char_p, C.c_char_p, C.c_int, i64p]
        L.ps_time.argtypes = [C.POINTER(native.PresolveModel), C.c_int,
                              C.POINTER(C.c_double), i64p]

    @staticmethod
    def _summary(s):
        return dict(infeasible=bool(s[0]), converged=bool(s[1]), presolved_variables=int(s[2]),
                    presolved_constraints=int(s[3]), transformations=int(s[4]),
                    removed_constraints=int(s[5]))

    def compare(self, model):
        """(rc, first difference or '', summary of the reference's result);
        rc 0 identical, 1 different, -1 an exception."""
        buf = model.buffers()
        msg, s = C.create_string_buffer(1024), np.zeros(6, np.int64)
        rc = self.lib.ps_compare(C.byref(buf.struct), msg, 1024, native.ptr(s, C.c_int64))
        return rc, msg.value.decode(), self._summary(s)

    def compare_mps(self, path: str):
        msg, s = C.create_string_buffer(1024), np.zeros(6, np.int64)
        rc = self.lib.ps_compare_mps(path.encode(), msg, 1024, native.ptr(s, C.c_int64))
        return rc, msg.value.decode(), self._summary(s)

    def time(self, model, which: str):
        """Seconds of one presolve: which = 'reference' or 'fast' (the facade,
        with its conversions from and to model::Model)."""
        buf = model.buffers()
        sec, s = C.c_double(), np.zeros(6, np.int64)
        rc = self.lib.ps_time(C.byref(buf.struct), 0 if which == "reference" else 1,
                              C.byref(sec), native.ptr(s, C.c_int64))
        if rc != 0:
            raise RuntimeError("presolve timing failed")
        return sec.value, self._summary(s)
