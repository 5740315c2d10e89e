"""GPU tests of the dense LU's own matrix products (cad_gemm_sub_dev:
C -= A B, column-major), FP64 on DMMA tensor cores and FP32 on TF32 tensor
cores through tcgen05 + TMA (or the FP32 CUDA-core kernel when the operands
do not meet TMA's alignment), against a plain PyTorch FP64 product.

Integer-valued operands are exact in TF32 and in FP64, and their products
sum exactly in FP32 below 2^24: those cases must match bit for bit, which
pins the tensor-memory and shared-memory descriptor layouts entry by entry.
Random operands check the rounding: FP64 to 1e-13 of the product's scale,
TF32 norm-wise to 2e-3 (10-bit mantissa inputs, FP32 accumulation).
Precision codes 2, 3, 4 are FP64 with the DMMA shapes m8n8k4, m16n8k8 and
m16n8k16, whose fragment layouts the integer cases pin element by element."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# the last two take the FP64 kernel's large tiles (at least two CTAs per SM), the others its small ones
SHAPES = [(128, 128, 32), (300, 200, 100), (1000, 700, 256), (4100, 130, 64), (37, 900, 300), (256, 256, 8),
          (2500, 1100, 96), (2600, 1200, 33)]


def _run(cad, prec, m, n, k, lda, ldb, ldc, a_off=0, b_off=0, integer=False, seed=0):
    import torch

    from cutanddisplacejulia_b200 import _lib
    dt = torch.float32 if prec == 1 else torch.float64
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(seed)

    def mat(rows, cols, ld, off):
        if integer:
            v = torch.randint(-4, 5, (off + ld * cols,), generator=g).to(torch.float64)
        else:
            v = torch.rand(off + ld * cols, generator=g, dtype=torch.float64) * 2 - 1
        return v.to(dt).to(dev)

    A = mat(m, k, lda, a_off)
    B = mat(k, n, ldb, b_off)
    C = mat(m, n, ldc, 0)
    C0 = C.clone()
    L = _lib.load()
    ctx = _lib.context(0)
    _lib.check(L.cad_gemm_sub_dev(ctx, prec, m, n, k, A.data_ptr() + a_off * A.element_size(), lda,
                                  B.data_ptr() + b_off * B.element_size(), ldb, C.data_ptr(), ldc), ctx)
    torch.cuda.synchronize()

    def view(v, off, rows, cols, ld):   # column-major rows x cols at offset off
        return v[off:off + ld * cols].view(cols, ld)[:, :rows].t().double()

    Ad, Bd, C0d, Cd = view(A, a_off, m, k, lda), view(B, b_off, k, n, ldb), view(C0, 0, m, n, ldc), view(C, 0, m, n, ldc)
    ref = C0d - Ad @ Bd
    # entries of C outside the m x n block are untouched
    mask = torch.ones(ldc * n, dtype=torch.bool, device=dev).view(n, ldc)
    mask[:, :m] = False
    assert torch.equal(C[:ldc * n].view(n, ldc)[mask], C0[:ldc * n].view(n, ldc)[mask])
    return Cd, ref, (Ad @ Bd)


@pytest.mark.parametrize("prec", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_integer_exact(cad, prec, m, n, k):
    ld = lambda r: (r + 3) // 4 * 4 + 4   # multiples of 4: the tcgen05 + TMA path for FP32
    got, ref, _ = _run(cad, prec, m, n, k, ld(m), ld(k), ld(m) + 1, integer=True)
    assert float((got - ref).abs().max()) == 0.0


@pytest.mark.parametrize("prec", [0, 1, 3, 4])
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_random(cad, prec, m, n, k):
    got, ref, prod = _run(cad, prec, m, n, k, m + 8, k + 12, m + 3, seed=1)
    if prec != 1:
        assert float((got - ref).abs().max()) <= 1e-13 * k
    else:
        assert float((got - ref).norm() / prod.norm()) <= 2e-3


@pytest.mark.parametrize("prec", [0, 1, 3, 4])
def test_gemm_offsets_and_odd_leading_dimensions(cad, prec):
    # sub-matrices at row offsets of the LU's trailing updates (multiples of
    # 4) and odd leading dimensions (FP64: any; FP32: the CUDA-core kernel)
    for (lda, ldb, a_off, b_off) in [(1003, 517, 4, 8), (1004, 516, 4, 8), (1001, 515, 1, 3)]:
        got, ref, prod = _run(cad, prec, 997, 300, 250, lda, ldb, 1000, a_off=a_off, b_off=b_off, integer=True)
        assert float((got - ref).abs().max()) == 0.0


def test_gemm_empty_and_bad_arguments(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    assert L.cad_gemm_sub_dev(ctx, 0, 0, 5, 5, None, 1, None, 5, None, 1) == 0
    assert L.cad_gemm_sub_dev(ctx, 1, 10, 5, 0, None, 10, None, 1, None, 10) == 0
    assert L.cad_gemm_sub_dev(ctx, 0, 10, 5, 5, None, 9, None, 5, None, 10) == _lib.CAD_ERR_ARG
    assert L.cad_gemm_sub_dev(ctx, 5, 10, 5, 5, None, 10, None, 5, None, 10) == _lib.CAD_ERR_ARG
    assert L.cad_gemm_sub_dev(ctx, -1, 10, 5, 5, None, 10, None, 5, None, 10) == _lib.CAD_ERR_ARG
