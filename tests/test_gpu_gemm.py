"""The tcgen05 BF16 GEMM (vphys_gemm_tn_bf16) against a torch FP32 matmul of
the same BF16 operands.  FP32 accumulation in a different order: relative
tolerance 2e-3 of the output's scale (bf16 outputs: one bf16 ulp more)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import _ffi

    return torch, _ffi.get_lib(), _ffi


def P(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def gelu(x):
    import torch

    return 0.5 * x * (1.0 + torch.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    import torch

    t = torch.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * 0.7978845608028654 * (1 + 3 * 0.044715 * x * x)


def run(env, A, B, alpha=1.0, bias=None, zin=None, act=0, f32=True, bf16=False, bf16_t=False):
    torch, lib, _ffi = env
    M, K = A.shape
    N = B.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    o32 = torch.full((M, N), float("nan"), device="cuda") if f32 else None
    o16 = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda") if bf16 else None
    o16t = torch.zeros((N, M), dtype=torch.bfloat16, device="cuda") if bf16_t else None
    st = lib.vphys_gemm_tn_bf16(P(A), A.stride(0), P(B), B.stride(0), M, N, K, float(alpha), P(bias), P(zin), N,
                                act, P(o32), N, P(o16), N, P(o16t), M, P(err), None)
    assert st == 0, _ffi.last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return o32, o16, o16t


@pytest.mark.parametrize("M,N,K", [(128, 256, 160), (300, 80, 256), (1000, 160, 64), (77, 16, 8), (4096, 256, 256),
                                   (80, 256, 16384), (256, 160, 4104)])
def test_gemm_plain(env, M, N, K):
    torch = env[0]
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    o32, _, _ = run(env, A, B, alpha=0.5)
    ref = 0.5 * (A.float() @ B.float().T)
    scale = float(ref.abs().max())
    diff = float((o32 - ref).abs().max())
    assert diff <= 2e-3 * scale, (diff, scale)


def test_gemm_epilogue_gelu_bias_transposed(env):
    torch = env[0]
    M, N, K = 520, 256, 160
    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (0.1 * torch.randn(N, K, device="cuda", generator=g)).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    o32, o16, o16t = run(env, A, B, bias=bias, act=1, f32=True, bf16=True, bf16_t=True)
    z = A.float() @ B.float().T + bias
    assert float((o32 - z).abs().max()) <= 2e-3 * float(z.abs().max())
    a = gelu(z)
    tol = 2e-3 * float(a.abs().max()) + 1e-2 * float(a.abs().max()) / 128
    assert float((o16.float() - a).abs().max()) <= tol
    assert torch.equal(o16t, o16.T.contiguous())


@pytest.mark.parametrize("M,N,K", [(1000, 256, 160), (777, 256, 256)])
def test_gemm_inference_hidden_layer(env, M, N, K):
    """The hidden-layer inference form (alpha 1, bias, GELU, BF16 output only)
    against the general form of the same product and torch."""
    torch = env[0]
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (0.1 * torch.randn(N, K, device="cuda", generator=g)).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    _, o16, _ = run(env, A, B, bias=bias, act=1, f32=False, bf16=True)
    _, o16g, _ = run(env, A, B, bias=bias, act=1, f32=True, bf16=True)   # the general epilogue
    assert torch.equal(o16, o16g)
    a = gelu(A.float() @ B.float().T + bias)
    # the accumulation order (2e-3 of the scale) plus half a BF16 ulp of each value
    tol = 2e-3 * float(a.abs().max()) + a.abs() / 256
    assert bool(((o16.float() - a).abs() <= tol).all())


@pytest.mark.parametrize("M,N,K", [(1000, 80, 256), (4099, 80, 256)])
def test_gemm_inference_output_layer(env, M, N, K):
    """The output-layer inference form (alpha 1, bias, FP32 output only)."""
    torch = env[0]
    g = torch.Generator(device="cuda").manual_seed(M + 3 * N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    o32, _, _ = run(env, A, B, bias=bias)
    ref = A.float() @ B.float().T + bias
    assert float((o32 - ref).abs().max()) <= 2e-3 * float(ref.abs().max())
    assert not torch.isnan(o32).any()


def test_gemm_epilogue_gelu_backward(env):
    torch = env[0]
    M, N, K = 333, 256, 80
    g = torch.Generator(device="cuda").manual_seed(12)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    zin = torch.randn(M, N, device="cuda", generator=g)
    o32, _, _ = run(env, A, B, zin=zin)
    ref = (A.float() @ B.float().T) * gelu_grad(zin)
    assert float((o32 - ref).abs().max()) <= 2e-3 * float(ref.abs().max())


def test_gemm_strided_operands(env):
    """Operands that are column slices of wider matrices (row stride > K)."""
    torch = env[0]
    g = torch.Generator(device="cuda").manual_seed(13)
    Afull = torch.randn(256, 4096, device="cuda", generator=g).to(torch.bfloat16)
    Bfull = torch.randn(160, 4096, device="cuda", generator=g).to(torch.bfloat16)
    A, B = Afull[:, 1024:1024 + 2048], Bfull[:, 1024:1024 + 2048]
    o32, _, _ = run(env, A, B)
    ref = A.float() @ B.float().T
    assert float((o32 - ref).abs().max()) <= 2e-3 * float(ref.abs().max())


def test_gemm_rejects_bad_shapes(env):
    torch, lib, _ffi = env
    A = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    B = torch.zeros(24, 64, dtype=torch.bfloat16, device="cuda")   # N % 16 != 0
    st = lib.vphys_gemm_tn_bf16(P(A), 64, P(B), 64, 128, 24, 64, 1.0, None, None, 0, 0, None, 0, None, 0, None, 0,
                                None, None)
    assert st == _ffi.ERR_BAD_SHAPE


@pytest.mark.parametrize("M", [1000, 5003, 128])
def test_mlp3_equals_three_gemms(env, M):
    """vphys_mlp3_bf16 (the surrogate's three layers in one launch, hidden
    activations on chip) against the three inference GEMMs it replaces: the
    same products in the same order, so bit for bit."""
    torch, lib, _ffi = env
    g = torch.Generator(device="cuda").manual_seed(M)
    X = torch.zeros(M, 160, device="cuda", dtype=torch.bfloat16)
    X[:, :154] = torch.randn(M, 154, device="cuda", generator=g).to(torch.bfloat16)
    W1 = (0.1 * torch.randn(256, 160, device="cuda", generator=g)).to(torch.bfloat16)
    W2 = (0.06 * torch.randn(256, 256, device="cuda", generator=g)).to(torch.bfloat16)
    W3 = (0.06 * torch.randn(80, 256, device="cuda", generator=g)).to(torch.bfloat16)
    b1 = 0.1 * torch.randn(256, device="cuda", generator=g)
    b2 = 0.1 * torch.randn(256, device="cuda", generator=g)
    b3 = 0.1 * torch.randn(80, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    Y = torch.full((M, 80), float("nan"), device="cuda")
    st = lib.vphys_mlp3_bf16(P(X), M, P(W1), P(b1), P(W2), P(b2), P(W3), P(b3), P(Y), P(err), None)
    assert st == 0, _ffi.last_error()
    _, H1, _ = run(env, X, W1, bias=b1, act=1, f32=False, bf16=True)
    _, H2, _ = run(env, H1, W2, bias=b2, act=1, f32=False, bf16=True)
    Y3, _, _ = run(env, H2, W3, bias=b3)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(Y, Y3)
    ref = gelu(gelu(X.float() @ W1.float().T + b1).to(torch.bfloat16).float() @ W2.float().T + b2)
    ref = ref.to(torch.bfloat16).float() @ W3.float().T + b3
    assert float((Y - ref).abs().max()) <= 2e-2 * float(ref.abs().max())
