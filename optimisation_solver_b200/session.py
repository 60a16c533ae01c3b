"""Repeated batched solves of one LP family (include/pdlpgpu_session.h).

A ``Session`` fixes the constraint matrix and the batch size; each ``solve``
loads per-instance vectors -- numpy arrays (host) or device pointers such as
``torch.Tensor.data_ptr()`` of CUDA tensors already in HBM -- and solves every
instance to completion on the device.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import native
from .lp import CompiledLp, PdlpOptions, PdlpStatus

_PRECISIONS = {"fp64": 0, "mixed": 1}
_LAYOUTS = {"auto": 0, "sell": 1, "interleaved": 2}


def _caller_stream_done():
    """Device-pointer arguments are ordered after the caller's work on the
    legacy default stream by the library itself; a caller that enqueued
    them on another PyTorch stream is waited for here."""
    torch = sys.modules.get("torch")
    if torch is None or not torch.cuda.is_initialized():
        return
    current = torch.cuda.current_stream()
    if current != torch.cuda.default_stream(current.device):
        current.synchronize()


def _check_buffer(a, name, needed, on_device, in_place):
    """A buffer the library reads or writes as `needed` contiguous doubles.
    Host inputs are converted to contiguous float64 copies before the call,
    so only their element count matters; device inputs and every output are
    used in place (`in_place`), so they must already be contiguous float64
    storage of at least `needed` elements, on the side the call names. Raw
    integer device pointers are the caller's responsibility."""
    if a is None or isinstance(a, int):
        return
    if hasattr(a, "data_ptr"):   # a torch tensor
        if on_device != a.is_cuda:
            where = "a CUDA" if on_device else "a host"
            raise ValueError(f"{name}: {where} tensor expected")
        if in_place:
            import torch
            if a.dtype != torch.float64:
                raise ValueError(f"{name}: dtype {a.dtype}, float64 expected")
            if not a.is_contiguous():
                raise ValueError(f"{name}: tensor is not contiguous")
        size = a.numel()
    else:
        if on_device:
            raise ValueError(f"{name}: a device buffer (CUDA tensor or integer address) expected")
        if in_place and (not isinstance(a, np.ndarray) or a.dtype != np.float64
                         or not a.flags.c_contiguous or not a.flags.writeable):
            raise ValueError(f"{name}: a writeable C-contiguous float64 numpy array expected")
        size = np.size(a)
    if size < needed:
        raise ValueError(f"{name}: {size} elements, at least {needed} expected")


def _check_sizes(arrs, rows, n, m, on_device=False):
    """The library reads rows x length elements of each per-instance input
    (objective, row bounds, variable bounds, warm primal, warm dual, warm
    weight), the first rows of a larger one: a buffer with fewer elements, or
    device storage of another dtype or with gaps, is refused here rather than
    read past its end."""
    names = ("objective", "row_lower", "row_upper", "var_lower", "var_upper", "warm_primal",
             "warm_dual", "warm_weight")
    lengths = (n, m, m, n, n, n, m, 1)
    for a, name, k in zip(arrs, names, lengths):
        _check_buffer(a, name, rows * k, on_device, in_place=on_device)


def _check_output(a, name, needed, on_device):
    """An output the library writes in place: on the host a writeable
    C-contiguous float64 numpy array, on the device a contiguous float64 CUDA
    tensor (or an integer address), of at least `needed` elements."""
    _check_buffer(a, name, needed, on_device, in_place=True)


def _addr(a):
    """Address of a host numpy array, an integer device pointer, a CUDA tensor, or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class Session:
    def __init__(self, family: CompiledLp, batch: int, options: PdlpOptions | None = None,
                 precision: str = "fp64", device: int = 0, layout: str = "auto", **tuning):
        """`layout`: "interleaved" keeps the trial kernels' vectors as
        [line][instance] so a warp serves 32 instances; "sell" walks the
        matrix once per instance; "auto" picks interleaved from 16 instances."""
        self.family = family
        self.batch = int(batch)
        self.n, self.m = family.num_cols, family.num_rows
        self._h = native.LpHandle(family)
        self._o = native.options_struct(options or PdlpOptions())
        self._e = native.ext_struct(precision=_PRECISIONS[precision], device=device,
                                    layout=_LAYOUTS[layout], **tuning)
        self._s = C.c_void_p()
        rc = native.lib().pdlpgpu_session_create(C.byref(self._h.struct), self.batch,
                                                 C.byref(self._o), C.byref(self._e),
                                                 C.byref(self._s))
        if rc != 0:
            raise RuntimeError(f"session_create failed: {native.last_error()}")
        self._keep = []

    def close(self):
        if self._s:
            native.lib().pdlpgpu_session_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, objective=None, row_lower=None, row_upper=None, var_lower=None,
             var_upper=None, warm_primal=None, warm_dual=None, warm_weight=None,
             on_device: bool = False):
        arrs = [objective, row_lower, row_upper, var_lower, var_upper, warm_primal, warm_dual,
                warm_weight]
        _check_sizes(arrs, self.batch, self.n, self.m, on_device)
        if not on_device:
            arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        else:
            _caller_stream_done()
        self._keep = arrs
        rc = native.lib().pdlpgpu_session_load(self._s, int(on_device), *[_addr(a) for a in arrs])
        if rc != 0:
            raise RuntimeError(f"session_load failed: {native.last_error()}")

    def solve(self) -> int:
        k = native.lib().pdlpgpu_session_solve(self._s)
        if k < 0:
            raise RuntimeError(f"session_solve failed: {native.last_error()}")
        return k

    def read(self, primal=None, dual=None, on_device: bool = False):
        """Statuses, iterations and stats on the host; primal/dual into the
        given buffers (allocated on the host when None and on_device is False)."""
        _check_output(primal, "primal", self.batch * self.n, on_device)
        _check_output(dual, "dual", self.batch * self.m, on_device)
        if not on_device:
            if primal is None:
                primal = np.zeros((self.batch, self.n))
            if dual is None:
                dual = np.zeros((self.batch, self.m))
        else:
            _caller_stream_done()
        status = np.zeros(self.batch, dtype=np.int32)
        iters = np.zeros(self.batch, dtype=np.int64)
        stats = np.zeros((self.batch, 8))
        rc = native.lib().pdlpgpu_session_read(self._s, int(on_device), _addr(primal), _addr(dual),
                                               native.ptr(status, C.c_int32),
                                               native.ptr(iters, C.c_int64), native.ptr(stats))
        if rc != 0:
            raise RuntimeError(f"session_read failed: {native.last_error()}")
        return dict(primal=primal, dual=dual, status=[PdlpStatus(int(s)) for s in status],
                    iterations=iters, primal_objective=stats[:, 0], dual_objective=stats[:, 1],
                    primal_residual=stats[:, 2], dual_residual=stats[:, 3],
                    relative_gap=stats[:, 4], step_trials=stats[:, 5].astype(np.int64),
                    final_primal_weight=stats[:, 6], restart_count=stats[:, 7].astype(np.int64))

    def stream(self, count: int, objective=None, row_lower=None, row_upper=None, var_lower=None,
               var_upper=None, warm_primal=None, warm_dual=None, warm_weight=None, primal=None,
               dual=None, on_device: bool = False):
        """Solves `count` instances through the session's slots with refill.
        Host mode allocates primal/dual outputs when not given; device mode
        writes into the given device buffers (or none)."""
        arrs = [objective, row_lower, row_upper, var_lower, var_upper, warm_primal, warm_dual,
                warm_weight]
        _check_sizes(arrs, int(count), self.n, self.m, on_device)
        if not on_device:
            arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
            if primal is None:
                primal = np.zeros((count, self.n))
            if dual is None:
                dual = np.zeros((count, self.m))
        else:
            _caller_stream_done()
        _check_output(primal, "primal", int(count) * self.n, on_device)
        _check_output(dual, "dual", int(count) * self.m, on_device)
        status = np.zeros(count, dtype=np.int32)
        iters = np.zeros(count, dtype=np.int64)
        stats = np.zeros((count, 8))
        k = native.lib().pdlpgpu_session_stream(self._s, int(on_device), int(count),
                                                *[_addr(a) for a in arrs], _addr(primal),
                                                _addr(dual), native.ptr(status, C.c_int32),
                                                native.ptr(iters, C.c_int64), native.ptr(stats))
        if k < 0:
            raise RuntimeError(f"session_stream failed: {native.last_error()}")
        return dict(optimal=k, primal=primal, dual=dual,
                    status=[PdlpStatus(int(s)) for s in status], iterations=iters,
                    primal_objective=stats[:, 0], dual_objective=stats[:, 1],
                    primal_residual=stats[:, 2], dual_residual=stats[:, 3],
                    relative_gap=stats[:, 4], step_trials=stats[:, 5].astype(np.int64),
                    final_primal_weight=stats[:, 6], restart_count=stats[:, 7].astype(np.int64))

    def last_timing(self):
        s, n = C.c_double(), C.c_int64()
        native.lib().pdlpgpu_session_last_timing(self._s, C.byref(s), C.byref(n))
        return s.value, n.value

    def loop_timing(self) -> dict:
        """Live durations of the last solve or stream, from CUDA events
        recorded inside the captured iteration loop (one trial per chunk)."""
        out = np.zeros(15)
        if native.lib().pdlpgpu_session_loop_timing(self._s, native.ptr(out)) != 0:
            raise RuntimeError("loop_timing failed")
        return dict(primal_ms=out[0], dual_ms=out[1], samples=int(out[2]), chunk_ms=out[3],
                    chunks=int(out[4]), loop_seconds=out[5], check_ms=out[6],
                    by_slot=[(out[7 + 2 * k], out[8 + 2 * k]) for k in range(4)])

    def time_kernels(self, reps: int = 20) -> dict:
        out = np.zeros(6)
        rc = native.lib().pdlpgpu_session_time_kernels(self._s, reps, native.ptr(out))
        if rc != 0:
            raise RuntimeError(f"time_kernels failed: {native.last_error()}")
        return dict(primal_ms=out[0], dual_ms=out[1], primal_bytes=out[2], dual_bytes=out[3],
                    at_padding=out[4], a_padding=out[5])
