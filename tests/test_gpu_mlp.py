"""The tensor-core GEMM and the warm-start network against the CPU oracle
(oracle/mlp_oracle.py, numpy FP64 with the device's BF16 rounding points).

Tolerances: GEMM outputs equal the FP64 product of the BF16 operands to
relative 1e-5 of the largest |product|-sum (FP32 accumulation); gradients
agree to 2e-2 relative in the Frobenius norm (BF16 re-rounding of
intermediate activations on either side can flip near-zero ReLU masks).
"""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _bf(t):
    import torch
    return torch.as_tensor(t, dtype=torch.float32).to("cuda").to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (256, 384, 512, 1), (256, 384, 512, 3),
                                           (200, 130, 136, 2), (256, 512, 22000, 18), (64, 256, 256, 1)])
def test_gemm_matches_numpy(M, N, K, splits):
    import torch
    from optimisation_solver_b200.mlp import gemm_bf16
    rng = np.random.default_rng(M * 7 + N + K)
    a = mo.bf16(rng.standard_normal((M, K)))
    b = mo.bf16(rng.standard_normal((N, K)))
    c = torch.empty((M, N), dtype=torch.float32, device="cuda")
    gemm_bf16(_bf(a), _bf(b), c, splits)
    torch.cuda.synchronize()
    got = c.cpu().numpy().astype(np.float64)
    want = a @ b.T
    scale = (np.abs(a) @ np.abs(b).T).max()
    assert np.abs(got - want).max() <= 1e-5 * scale


def _small_net(seed=0, I=256, H=128, O=192, B=128):
    import torch
    from optimisation_solver_b200.mlp import Mlp
    net = Mlp(I, H, O, B, seed=seed)
    rng = np.random.default_rng(seed)
    X = mo.bf16(rng.standard_normal((B, I)))
    T = rng.standard_normal((B, O))
    w = np.full(O, 1.0 / O)
    w[-7:] = 0.0
    P = {k: torch.empty(s, dtype=torch.float32, device="cuda") for k, s in
         dict(W1=(H, I), b1=(H,), W2=(H, H), b2=(H,), W3=(O, H), b3=(O,)).items()}
    # non-zero biases so every term is exercised
    net.get_params(P)
    for k in ("b1", "b2", "b3"):
        P[k].copy_(torch.as_tensor(rng.standard_normal(P[k].shape[0]) * 0.1, dtype=torch.float32))
    net.set_params(P)
    return net, X, T, w, P


def test_forward_matches_oracle():
    import torch
    net, X, T, w, P = _small_net(1)
    out = torch.empty((net.batch, net.outputs), dtype=torch.float32, device="cuda")
    net.forward(_bf(X), out)
    torch.cuda.synchronize()
    p = {k: v.cpu().numpy().astype(np.float64) for k, v in P.items()}
    want, _, _ = mo.forward(X, p["W1"], p["b1"], p["W2"], p["b2"], p["W3"], p["b3"])
    got = out.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-2 * np.linalg.norm(want)


def test_forward_waits_for_inputs_written_just_before():
    """Features still being copied in on the default stream, behind tens of
    milliseconds of other work, when the forward pass is called: the model
    waits for them, and its outputs are those of resident inputs."""
    import torch
    net, X, T, w, P = _small_net(2)
    ref = torch.empty((net.batch, net.outputs), dtype=torch.float32, device="cuda")
    x_ready = _bf(X)
    torch.cuda.synchronize()
    net.forward(x_ready, ref)
    x_late = torch.full_like(x_ready, float("nan"))
    x_host = x_ready.cpu().pin_memory()
    torch.cuda.synchronize()
    busy = torch.randn((4096, 4096), device="cuda")
    for _ in range(40):
        busy = torch.tanh(busy @ busy)
    x_late.copy_(x_host, non_blocking=True)
    out = torch.empty_like(ref)
    net.forward(x_late, out)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


def test_gradients_match_oracle():
    import torch
    net, X, T, w, P = _small_net(2)
    G = {k: torch.empty_like(v) for k, v in P.items()}
    Tt = torch.as_tensor(T, dtype=torch.float32, device="cuda")
    wt = torch.as_tensor(w, dtype=torch.float32, device="cuda")
    loss = net.gradients(_bf(X), Tt, wt, G)
    torch.cuda.synchronize()
    p = {k: v.cpu().numpy().astype(np.float64) for k, v in P.items()}
    want_loss, want = mo.gradients(X, T, w, p["W1"], p["b1"], p["W2"], p["b2"], p["W3"], p["b3"])
    assert abs(loss - want_loss) <= 2e-3 * abs(want_loss)
    for k in want:
        g = G[k].cpu().numpy()
        assert np.linalg.norm(g - want[k]) <= 2e-2 * max(np.linalg.norm(want[k]), 1e-12), k


def test_finite_differences_on_bias():
    """Directional check of db3 against a central difference of the loss
    (b3 enters the loss without BF16 rounding, so the difference is clean)."""
    import torch
    net, X, T, w, P = _small_net(3)
    G = {k: torch.empty_like(v) for k, v in P.items()}
    Tt = torch.as_tensor(T, dtype=torch.float32, device="cuda")
    wt = torch.as_tensor(w, dtype=torch.float32, device="cuda")
    Xb = _bf(X)
    net.gradients(Xb, Tt, wt, G)
    d = torch.zeros_like(P["b3"])
    d[:8] = 1.0
    h = 1e-2
    losses = []
    for sgn in (1.0, -1.0):
        Q = dict(P)
        Q["b3"] = P["b3"] + sgn * h * d
        net.set_params(Q)
        losses.append(net.gradients(Xb, Tt, wt, {}))
    net.set_params(P)
    fd = (losses[0] - losses[1]) / (2 * h)
    an = float((G["b3"] * d).sum())
    assert abs(fd - an) <= 1e-2 * max(abs(an), 1e-6)


def test_training_reduces_loss():
    import torch
    net, X, T, w, P = _small_net(4)
    Tt = torch.as_tensor(T * 0.1, dtype=torch.float32, device="cuda")
    wt = torch.as_tensor(w, dtype=torch.float32, device="cuda")
    Xb = _bf(X)
    first = net.train_step(Xb, Tt, wt, 1e-3)
    for _ in range(60):
        last = net.train_step(Xb, Tt, wt, 1e-3)
    assert last < 0.5 * first


@pytest.mark.parametrize("M,N,K,splits", [(1024, 1024, 2048, 1), (256, 512, 22000, 18)])
def test_gemm_timing_entry_point_computes_the_product(M, N, K, splits):
    """pdlpgpu_gemm_time runs the product `reps` times between CUDA events;
    the result left in C is the product, and the time is positive. Prints the
    throughput against the measured dense BF16 peak."""
    import ctypes as C
    import json
    import os

    import torch
    from optimisation_solver_b200 import native
    rng = np.random.default_rng(M + N + K)
    a = mo.bf16(rng.standard_normal((M, K)))
    b = mo.bf16(rng.standard_normal((N, K)))
    c = torch.empty((M, N), dtype=torch.float32, device="cuda")
    A, B = _bf(a), _bf(b)
    ms = C.c_double()
    rc = native.lib().pdlpgpu_gemm_time(M, N, K, C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()),
                                        C.c_void_p(c.data_ptr()), splits, 5, C.byref(ms))
    assert rc == 0, native.last_error()
    got = c.cpu().numpy().astype(np.float64)
    want = a @ b.T
    scale = (np.abs(a) @ np.abs(b).T).max()
    assert np.abs(got - want).max() <= 1e-5 * scale
    assert ms.value > 0.0
    peaks = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    peak = json.load(open(peaks)).get("bf16_tflops", 1590.0) if os.path.exists(peaks) else 1590.0
    tflops = 2.0 * M * N * K / (ms.value * 1e-3) / 1e12
    print(f"gemm {M}x{N}x{K} splits {splits}: {ms.value * 1e3:.1f} us, {tflops:.1f} TFLOP/s "
          f"({tflops / peak:.3f} of {peak})")
