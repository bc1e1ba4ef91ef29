"""The tcgen05 batched FP32 product (mpsqmc_tc_gemm) against an FP64 torch reference of the same
op: D_z = alpha A_{z/adiv} B_{z/bdiv}^T (+ D_z), operands K-major in zero-padded tiles.

Tolerances (relative to max |D|): 3 passes (TF32 head/tail split, FP32 accumulation) within 8x
the error of a plain FP32 product of the same inputs (torch, TF32 off), and at most 2e-5;
1 pass (TF32 operands) 4e-3.  Shapes cover the sweep's uses: a shared trial operand with walkers
stacked along N (M = 256, K = 512), per-walker operands with M = 64 (half-datapath accumulator
layout), padding of M, N and K to whole tiles, an operand shared by pairs of batch entries,
row- and column-major outputs (written through shared-memory boxes and TMA bulk stores when
nothing accumulates), and accumulation."""
import numpy as np
import pytest

from mpsqmc_b200 import capi

pytestmark = pytest.mark.gpu


def _pad(n, q):
    return (n + q - 1) // q * q


def run_case(M, N, K, Z, adiv, bdiv, bstack, passes, alpha=1.0, beta=0, colmajor=False, seed=0):
    import torch

    g = torch.Generator().manual_seed(seed)
    dev = "cuda"
    tm = 64 if M <= 64 else 128
    kp = _pad(K, 32)
    tn = _pad(N * bstack, 16) if bstack > 1 else min(256, _pad(N, 16))
    ar = _pad(M, tm)
    br = N if bstack > 1 else _pad(N, tn)
    za = 1 if adiv == 0 else (Z - 1) // adiv + 1
    zb = 1 if bdiv == 0 else (Z - 1) // bdiv + 1
    if bstack > 1:
        zb = _pad(zb, bstack)
    A = torch.zeros((za, ar, kp), dtype=torch.float32)
    B = torch.zeros((zb, br, kp), dtype=torch.float32)
    A[:, :M, :K] = torch.randn((za, M, K), generator=g)
    B[:, :N, :K] = torch.randn((zb, N, K), generator=g)
    D0 = torch.randn((Z, M, N), generator=g) if beta else torch.zeros((Z, M, N))
    ai = torch.tensor([z // adiv if adiv else 0 for z in range(Z)])
    bi = torch.tensor([z // bdiv if bdiv else 0 for z in range(Z)])
    ref = alpha * torch.einsum("zmk,znk->zmn", A[ai, :M, :K].double(), B[bi, :N, :K].double())
    if beta:
        ref = ref + D0.double()
    Ad, Bd = A.to(dev), B.to(dev)
    if colmajor:  # D_z stored (n, m): element (m, n) at z*M*N + n*M + m
        Dd = D0.transpose(1, 2).contiguous().to(dev)
        dz, dm, dn = M * N, 1, M
    else:
        Dd = D0.contiguous().to(dev)
        dz, dm, dn = M * N, N, 1
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = capi.tc_gemm(D=Dd.data_ptr(), A=Ad.data_ptr(), B=Bd.data_ptr(), M=M, N=N, K=K, lda=kp, a_zstride=ar * kp,
                      adiv=adiv, a_zcount=za, ldb=kp, b_zstride=br * kp, bdiv=bdiv, b_zcount=zb, Z=Z, bstack=bstack,
                      alpha=alpha, beta=beta, passes=passes, dz=dz, dm=dm, dn=dn, err=err.data_ptr(),
                      stream=torch.cuda.current_stream().cuda_stream)
    assert rc == 0, capi.load().mpsqmc_last_error().decode()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    out = Dd.cpu().double()
    if colmajor:
        out = out.transpose(1, 2)
    scale = float(ref.abs().max())
    # the same product in plain FP32 (TF32 off): the accuracy the 3-pass product should match
    keep = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    f32 = alpha * torch.einsum("zmk,znk->zmn", A[ai, :M, :K].to(dev), B[bi, :N, :K].to(dev)).double().cpu()
    torch.backends.cuda.matmul.allow_tf32 = keep
    if beta:
        f32 = f32 + D0.double()
    return float((out - ref).abs().max()) / scale, float((f32 - ref).abs().max()) / scale


CASES = [
    # M, N, K, Z, adiv, bdiv, bstack
    (256, 64, 512, 9, 0, 1, 4),     # trial x stacked walkers (8x8: M = 256, sigma-stacked K = 512)
    (64, 32, 64, 13, 0, 1, 8),      # chain64 trial products, 8 walkers per tile
    (64, 64, 32, 7, 1, 1, 1),       # walker products, M = 64
    (96, 40, 40, 3, 1, 1, 1),       # padding of M, N and K
    (128, 48, 64, 6, 1, 2, 1),      # B shared by pairs (a walker's site for its branches)
    (200, 256, 96, 2, 1, 1, 1),     # two M tiles, a full-width N tile
    (128, 300, 64, 2, 1, 1, 1),     # two N tiles per batch entry
]


def fp32_accurate(err, err_f32):
    # the head/tail scheme drops tail x tail and rounds the tail to TF32: about 2^-22 relative per
    # product term against FP32's 2^-24 (measured 3.6x - 5.4x the plain FP32 error)
    return err <= max(8.0 * err_f32, 2e-6) and err < 2e-5


@pytest.mark.parametrize("passes", [3, 1])
@pytest.mark.parametrize("case", CASES, ids=[f"M{c[0]}N{c[1]}K{c[2]}Z{c[3]}a{c[4]}b{c[5]}s{c[6]}" for c in CASES])
def test_tc_gemm_matches_fp64(case, passes):
    err, err_f32 = run_case(*case, passes=passes)
    print(f"{case} passes={passes}: {err:.3e} (plain FP32 {err_f32:.3e})")
    if passes == 3:
        assert fp32_accurate(err, err_f32), (err, err_f32)
    else:
        assert err < 4e-3


@pytest.mark.parametrize("colmajor", [False, True])
def test_tc_gemm_alpha_beta_and_layouts(colmajor):
    assert fp32_accurate(*run_case(128, 64, 64, 5, 1, 1, 1, 3, alpha=0.5, beta=1, colmajor=colmajor))
    assert fp32_accurate(*run_case(256, 32, 256, 8, 0, 1, 8, 3, alpha=-2.0, beta=1, colmajor=colmajor))
    # without accumulation the epilogue writes through TMA bulk stores (32-column boxes where the
    # tile allows, 16-column ones otherwise)
    assert fp32_accurate(*run_case(128, 64, 64, 5, 1, 1, 1, 3, alpha=0.5, beta=0, colmajor=colmajor))
    assert fp32_accurate(*run_case(256, 32, 256, 8, 0, 1, 8, 3, alpha=-2.0, beta=0, colmajor=colmajor))
    assert fp32_accurate(*run_case(64, 48, 32, 7, 1, 1, 1, 3, alpha=1.5, beta=0, colmajor=colmajor))


@pytest.mark.parametrize("case", CASES, ids=[f"M{c[0]}N{c[1]}K{c[2]}Z{c[3]}a{c[4]}b{c[5]}s{c[6]}" for c in CASES])
def test_tc_gemm_bf16_pass(case):
    """One bfloat16 pass (kind::f16): the product equals that of the operands rounded to bfloat16
    (nearest, ties to even), accumulated in FP32; against an FP64 product of the rounded inputs
    within FP32 accumulation error (5e-5 of max |D|), and within 1e-2 of the unrounded product."""
    import torch

    M, N, K, Z, adiv, bdiv, bstack = case
    g = torch.Generator().manual_seed(1)
    dev = "cuda"
    tm = 64 if M <= 64 else 128
    kp = _pad(K, 32)
    tn = _pad(N * bstack, 16) if bstack > 1 else min(256, _pad(N, 16))
    ar, br = _pad(M, tm), (N if bstack > 1 else _pad(N, tn))
    za = 1 if adiv == 0 else (Z - 1) // adiv + 1
    zb = 1 if bdiv == 0 else (Z - 1) // bdiv + 1
    if bstack > 1:
        zb = _pad(zb, bstack)
    A = torch.zeros((za, ar, kp))
    B = torch.zeros((zb, br, kp))
    A[:, :M, :K] = torch.randn((za, M, K), generator=g)
    B[:, :N, :K] = torch.randn((zb, N, K), generator=g)
    ai = torch.tensor([z // adiv if adiv else 0 for z in range(Z)])
    bi = torch.tensor([z // bdiv if bdiv else 0 for z in range(Z)])
    Ar, Br = A.bfloat16().double(), B.bfloat16().double()
    ref_r = torch.einsum("zmk,znk->zmn", Ar[ai, :M, :K], Br[bi, :N, :K])
    ref = torch.einsum("zmk,znk->zmn", A[ai, :M, :K].double(), B[bi, :N, :K].double())
    D = torch.zeros((Z, M, N), device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    Ad, Bd = A.to(dev), B.to(dev)
    rc = capi.tc_gemm(D=D.data_ptr(), A=Ad.data_ptr(), B=Bd.data_ptr(), M=M, N=N, K=K, lda=kp, a_zstride=ar * kp,
                      adiv=adiv, a_zcount=za, ldb=kp, b_zstride=br * kp, bdiv=bdiv, b_zcount=zb, Z=Z, bstack=bstack,
                      alpha=1.0, beta=0, passes=capi.TC_PASSES_BF16, dz=M * N, dm=N, dn=1, err=err.data_ptr(),
                      stream=torch.cuda.current_stream().cuda_stream)
    assert rc == 0, capi.load().mpsqmc_last_error().decode()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    out = D.cpu().double()
    scale = float(ref_r.abs().max())
    e_r = float((out - ref_r).abs().max()) / scale
    e = float((out - ref).abs().max()) / scale
    print(f"{case} bf16: {e_r:.2e} vs rounded inputs, {e:.2e} vs FP64")
    assert e_r < 5e-5
    assert e < 1e-2
