"""The learned warm start's network (include/pdlpgpu_mlp.h) over torch
device tensors (torch provides the device memory; every computation is the
library's own kernels)."""
from __future__ import annotations

import ctypes as C

from . import native


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Mlp:
    def __init__(self, inputs: int, hidden: int, outputs: int, batch: int, seed: int = 0,
                 device: int = 0):
        self.inputs, self.hidden, self.outputs, self.batch = inputs, hidden, outputs, batch
        self._h = C.c_void_p()
        rc = native.lib().pdlpgpu_mlp_create(inputs, hidden, outputs, batch, seed, device,
                                             C.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"mlp_create failed: {native.last_error()}")

    def close(self):
        if self._h:
            native.lib().pdlpgpu_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {native.last_error()}")

    def forward(self, x_bf16, out_f32):
        """x_bf16: CUDA bfloat16 [batch, inputs]; out_f32: CUDA float32 [batch, outputs]."""
        self._check(native.lib().pdlpgpu_mlp_forward(self._h, _p(x_bf16), _p(out_f32)), "forward")

    def train_step(self, x_bf16, target, weights, lr: float) -> float:
        loss = C.c_float()
        self._check(native.lib().pdlpgpu_mlp_train_step(self._h, _p(x_bf16), _p(target), _p(weights),
                                                        float(lr), C.byref(loss)), "train_step")
        return loss.value

    def gradients(self, x_bf16, target, weights, grads: dict) -> float:
        loss = C.c_float()
        keys = ["W1", "b1", "W2", "b2", "W3", "b3"]
        self._check(native.lib().pdlpgpu_mlp_gradients(self._h, _p(x_bf16), _p(target), _p(weights),
                                                       *[_p(grads.get(k)) for k in keys],
                                                       C.byref(loss)), "gradients")
        return loss.value

    def get_params(self, params: dict):
        keys = ["W1", "b1", "W2", "b2", "W3", "b3"]
        self._check(native.lib().pdlpgpu_mlp_get_params(self._h, *[_p(params.get(k)) for k in keys]),
                    "get_params")

    def set_params(self, params: dict):
        keys = ["W1", "b1", "W2", "b2", "W3", "b3"]
        self._check(native.lib().pdlpgpu_mlp_set_params(self._h, *[_p(params.get(k)) for k in keys]),
                    "set_params")

    def launches(self) -> int:
        return native.lib().pdlpgpu_mlp_launches(self._h)


def gemm_bf16(a_bf16, b_bf16, c_f32, splits: int = 1):
    """c = a @ b.T on the tensor cores (a [M,K], b [N,K] bfloat16 CUDA tensors)."""
    M, K = a_bf16.shape
    N = b_bf16.shape[0]
    rc = native.lib().pdlpgpu_gemm_bf16(M, N, K, _p(a_bf16), _p(b_bf16), _p(c_f32), splits)
    if rc != 0:
        raise RuntimeError(f"gemm failed: {native.last_error()}")
