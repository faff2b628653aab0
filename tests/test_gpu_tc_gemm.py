"""The tensor-core batched GEMM (tcgen05 kind::tf32, TMA-staged operands)
that the wide-band factorization runs on in the TF32 forms, through the C
ABI, against an FP64 product of the same inputs rounded to TF32 (round to
nearest even at 10 mantissa bits, what the kernel's TMA descriptors do).

Against the FP64 product of the unrounded inputs each entry is held to
|C - C_ref| <= 2^-9 (|A| |B|)_ij (two TF32 input roundings and the FP32
accumulation), far below a layout, swizzle or descriptor error, which shows
as O(1) errors; against the product of the inputs rounded to nearest TF32
the bound is 2^-18 (|A| |B|)_ij, the FP32 accumulation alone.  Shapes cover ragged tiles in every
dimension, the three tile widths, sub-matrix views with leading dimensions
larger than the rows, batches, alpha / beta, K not a multiple of 32, and
grids with more tiles than resident CTAs (the persistent loop)."""
import numpy as np
import pytest

import saplibrary_b200 as sap

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def tf32_round(a: np.ndarray) -> np.ndarray:
    """FP32 -> TF32 by round to nearest even at 10 explicit mantissa bits."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 13) & 1
    u = (u + 0xFFF + lsb) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


def run_case(m, n, k, batch, alpha, beta, pad=(0, 0, 0), seed=0):
    rng = np.random.default_rng(seed)
    lda, ldb, ldc = m + pad[0], k + pad[1], m + pad[2]
    lda, ldb = (lda + 3) // 4 * 4, (ldb + 3) // 4 * 4
    sA, sB, sC = lda * k + 4 * pad[0], ldb * n + 8, ldc * n + 12
    A = rng.standard_normal((batch, sA)).astype(np.float32)
    B = rng.standard_normal((batch, sB)).astype(np.float32)
    C0 = rng.standard_normal((batch, sC)).astype(np.float32)
    dA, dB, dC = (torch.tensor(x.ravel(), device="cuda") for x in (A, B, C0))
    sap.tc_gemm_batched(m, n, k, alpha, dA, lda, sA, dB, ldb, sB, beta, dC, ldc, sC, batch)
    out = dC.cpu().numpy().reshape(batch, sC)
    worst_rne = 0.0
    for b in range(batch):
        Ax = A[b, :lda * k].reshape(k, lda).T[:m]
        Bx = B[b, :ldb * n].reshape(n, ldb).T[:k]
        Cb = C0[b, :ldc * n].reshape(n, ldc).T[:m].astype(np.float64)
        ref = alpha * (Ax.astype(np.float64) @ Bx.astype(np.float64)) + beta * Cb
        bound = abs(alpha) * (np.abs(Ax).astype(np.float64) @ np.abs(Bx).astype(np.float64)) + abs(beta) * np.abs(Cb)
        got = out[b, :ldc * n].reshape(n, ldc).T[:m]
        err = np.abs(got - ref)
        assert np.all(err <= 2.0 ** -9 * bound + 1e-30), (m, n, k, batch, b, float((err / (bound + 1e-30)).max()))
        rne = alpha * (tf32_round(Ax).astype(np.float64) @ tf32_round(Bx).astype(np.float64)) + beta * Cb
        worst_rne = max(worst_rne, float((np.abs(got - rne) / (bound + 1e-30)).max()))
        # entries outside the view (padding rows, the batch gap) are untouched
        full = out[b].copy()
        mask = np.ones(sC, bool)
        idx = (np.arange(n)[:, None] * ldc + np.arange(m)[None, :]).ravel()
        mask[idx] = False
        assert np.array_equal(full[mask], C0[b][mask])
    print(f"m={m} n={n} k={k} batch={batch}: max |C - C(rne tf32 inputs)| / (|A||B|) = {worst_rne:.2e}")
    # the inputs are rounded to nearest TF32: what is left is FP32 accumulation
    assert worst_rne <= 2.0 ** -18, worst_rne


@pytest.mark.parametrize("m,n,k,batch", [
    (128, 256, 32, 1), (1, 1, 1, 1), (31, 47, 5, 2), (129, 257, 33, 3), (128, 64, 64, 4), (200, 100, 300, 2),
    (384, 512, 1024, 2), (3168, 96, 64, 1), (96, 3168, 160, 1), (1000, 1000, 1000, 1),
    # more tiles than resident CTAs: every CTA walks several tiles, both accumulators in turn
    (800, 800, 96, 16), (1000, 50, 64, 40), (300, 120, 40, 70)])
def test_tc_gemm_matches_fp64_of_tf32_inputs(m, n, k, batch):
    run_case(m, n, k, batch, 1.0, 0.0, seed=m + n + k)


@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (1.0, 1.0), (0.5, -2.0)])
def test_tc_gemm_alpha_beta_and_views(alpha, beta):
    run_case(224, 224, 224, 3, alpha, beta, pad=(32, 8, 5), seed=7)
    run_case(160, 96, 96, 2, alpha, beta, pad=(4, 4, 1), seed=8)


def test_tc_gemm_rejects_unaligned_views():
    a = torch.zeros(4096, device="cuda")
    with pytest.raises(sap.LibraryError):
        sap.tc_gemm_batched(8, 8, 8, 1.0, a.data_ptr() + 4, 8, 64, a, 8, 64, 0.0, a, 8, 64, 1)
    with pytest.raises(sap.LibraryError):
        sap.tc_gemm_batched(8, 8, 8, 1.0, a, 9, 72, a, 8, 64, 0.0, a, 8, 64, 1)
