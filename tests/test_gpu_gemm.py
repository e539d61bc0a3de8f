"""The surrogate's tcgen05 BF16 GEMM (mx_gemm_bf16) against a plain PyTorch FP32 computation on the same BF16
operands: every epilogue, full and partial row tiles, the four column tile widths (64, 128, 192, 256), several K,
and a shape with many tiles per persistent CTA."""

import numpy as np
import pytest
import torch

from maxichem_b200 import abi

pytestmark = pytest.mark.gpu
STORE, BIAS, BIAS_SILU, DSILU = 0, 1, 2, 3


def run(mode, A, B, bias=None, z=None):
    M, K = A.shape
    N = B.shape[0]
    dev = A.device
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    if mode in (STORE, BIAS):
        out = torch.full((M, N), float("nan"), dtype=torch.float32, device=dev)
    else:
        out = torch.full((M, N), float("nan"), dtype=torch.bfloat16, device=dev)
    zt = z if z is not None else (torch.full((M, N), float("nan"), dtype=torch.float32, device=dev)
                                  if mode == BIAS_SILU else None)  # fmt: skip
    p = lambda t: None if t is None else t.data_ptr()
    rc = abi.library().mx_gemm_bf16(p(A), K, p(B), K, M, N, K, mode, p(bias), p(zt), N, p(out), N, p(flag),
                                    torch.cuda.current_stream(dev).cuda_stream)  # fmt: skip
    assert rc == 0
    torch.cuda.synchronize(dev)
    assert int(flag.item()) == 0
    return out, zt


# (65536, 512, 512): 1,024 tiles over the persistent CTAs (one per SM), so each CTA reuses both accumulators many times
# (20000, 192, 256), (300, 384, 128): 192-column tiles (TMEM accumulators rounded up to 512 columns)
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 128, 512), (1000, 320, 512), (4096, 512, 128), (77, 64, 192),
                                   (65536, 512, 512), (20000, 192, 256), (300, 384, 128), (65536, 384, 512)])
def test_every_epilogue_matches_an_fp32_product(gpu, M, N, K):
    g = torch.Generator(device=gpu)
    g.manual_seed(M + N + K)
    A = torch.randn(M, K, device=gpu, generator=g).to(torch.bfloat16)
    B = (torch.randn(N, K, device=gpu, generator=g) / K**0.5).to(torch.bfloat16)
    bias = torch.randn(N, device=gpu, generator=g)
    ref = A.float() @ B.float().T
    tol = 2e-5 * float(ref.abs().max())
    out, _ = run(STORE, A, B)
    assert float((out - ref).abs().max()) <= tol
    out, _ = run(BIAS, A, B, bias=bias)
    assert float((out - (ref + bias)).abs().max()) <= tol
    out, z = run(BIAS_SILU, A, B, bias=bias)
    zr = ref + bias
    assert float((z - zr).abs().max()) <= tol
    silu = zr * torch.sigmoid(zr)
    # one BF16 rounding of the output: half an ulp of 8 bits of mantissa, plus the product's FP32 difference
    assert bool(((out.float() - silu).abs() <= silu.abs() * 2**-8 + 2 * tol).all())
    zin = torch.randn(M, N, device=gpu, generator=g)
    out, _ = run(DSILU, A, B, z=zin)
    s = torch.sigmoid(zin)
    want = ref * s * (1 + zin * (1 - s))
    assert bool(((out.float() - want).abs() <= want.abs() * 2**-8 + 4 * tol).all())


def test_shapes_the_kernel_does_not_take_are_refused(gpu):
    A = torch.zeros(128, 100, dtype=torch.bfloat16, device=gpu)
    B = torch.zeros(64, 100, dtype=torch.bfloat16, device=gpu)
    out = torch.zeros(128, 64, dtype=torch.float32, device=gpu)
    flag = torch.zeros(1, dtype=torch.int32, device=gpu)
    rc = abi.library().mx_gemm_bf16(A.data_ptr(), 100, B.data_ptr(), 100, 128, 64, 100, STORE, None, None, 0,
                                    out.data_ptr(), 64, flag.data_ptr(), None)  # fmt: skip
    assert rc == 1  # K must be a multiple of 64
    assert np.isfinite(out.cpu().numpy()).all()


def test_unaligned_outputs_bias_or_z_are_refused(gpu):
    """Outputs, biases and z go through 16-byte stores and loads (TMA or plain): a pointer or a row pitch that is not a
    multiple of 16 bytes is refused before anything is launched, and the buffers stay as they were."""
    M, N, K = 128, 64, 64
    A = torch.zeros(M, K, dtype=torch.bfloat16, device=gpu)
    B = torch.zeros(N, K, dtype=torch.bfloat16, device=gpu)
    bias = torch.zeros(N + 4, device=gpu)
    out = torch.full((M * (N + 4),), 7.0, device=gpu)
    z = torch.full((M * (N + 4),), 7.0, device=gpu)
    flag = torch.zeros(1, dtype=torch.int32, device=gpu)
    lib = abi.library()
    p = lambda *a: lib.mx_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, *a, flag.data_ptr(), None)
    assert p(STORE, None, None, 0, out.data_ptr() + 4, N) == 1             # output 4 bytes off
    assert p(STORE, None, None, 0, out.data_ptr(), N + 1) == 1             # FP32 pitch of 260 bytes
    assert p(BIAS, bias.data_ptr() + 4, None, 0, out.data_ptr(), N) == 1   # bias 4 bytes off
    assert p(BIAS_SILU, bias.data_ptr(), None, 0, out.data_ptr(), N + 4) == 1   # BF16 pitch of 136 bytes
    assert p(BIAS_SILU, bias.data_ptr(), z.data_ptr(), N + 1, out.data_ptr(), N + 8) == 1  # z pitch
    assert p(DSILU, None, z.data_ptr() + 8, N, out.data_ptr(), N) == 1     # z 8 bytes off
    torch.cuda.synchronize(gpu)
    assert bool((out == 7.0).all()) and bool((z == 7.0).all())


@pytest.mark.parametrize("M,N,K", [(512, 512, 16384), (320, 512, 8192), (512, 128, 4096), (128, 64, 128)])
def test_the_split_k_product_matches_the_unsplit_one(gpu, M, N, K):
    """The weight gradients' shape (a few output tiles, a long K): K split across the SMs, the partial products
    added in split order by a second kernel; against the FP32 product, and the same bits twice."""
    g = torch.Generator(device=gpu)
    g.manual_seed(M + N + K + 1)
    A = torch.randn(M, K, device=gpu, generator=g).to(torch.bfloat16)
    B = (torch.randn(N, K, device=gpu, generator=g) / K**0.5).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    lib = abi.library()
    n_ws = lib.mx_gemm_split_workspace(M, N, K)
    if (M, N, K) != (128, 64, 128):
        assert n_ws > 0  # these shapes do split
    ws = torch.full((max(n_ws, 1),), float("nan"), device=gpu)
    flag = torch.zeros(1, dtype=torch.int32, device=gpu)
    outs = []
    for _ in range(2):
        out = torch.full((M, N + 4), float("nan"), device=gpu)
        rc = lib.mx_gemm_bf16_split(A.data_ptr(), K, B.data_ptr(), K, M, N, K, ws.data_ptr() if n_ws else None,
                                    out.data_ptr(), N + 4, flag.data_ptr(), None)  # fmt: skip
        assert rc == 0
        torch.cuda.synchronize(gpu)
        assert int(flag.item()) == 0
        outs.append(out)
    got = outs[0][:, :N]
    assert float((got - ref).abs().max()) <= 2e-5 * float(ref.abs().max()) + 1e-6 * K**0.5
    assert torch.equal(outs[0][:, :N], outs[1][:, :N])
    assert bool(torch.isnan(outs[0][:, N:]).all())
