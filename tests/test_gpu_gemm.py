"""tcgen05 BF16 GEMM (FP32 accumulation in tensor memory) against a plain
PyTorch FP32 reference of the same products, through both operand paths
(TMA bulk tensor loads with swizzled shared-memory tiles, and per-thread
cp.async into the no-swizzle layout).  Tolerance: relative Frobenius error
<= 1e-5 (inputs are exact in BF16, so only FP32 summation order differs)."""
import ctypes as C

import pytest

from airtoolsii_b200 import _lib

pytestmark = pytest.mark.gpu


def set_path(path):
    f = _lib.lib().airt_test_gemm_path
    f.restype, f.argtypes = C.c_int, [C.c_int]
    assert f(path) == 0


@pytest.fixture(params=[0, 1], ids=["tma", "cpasync"])
def path(request):
    set_path(request.param)
    yield request.param
    set_path(0)


def _gemm(A, B, M, N, K, a_mn, b_mn, bn, ksplit=0, atomic_t=False):
    import torch
    L = _lib.lib()
    f = L.airt_test_gemm_bf16
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                  C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    if atomic_t:
        D = torch.zeros(N, M, dtype=torch.float32, device="cuda")
        ldd = M
    else:
        D = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
        ldd = N
    st = f(M, N, K, A.data_ptr(), A.shape[1], int(a_mn), B.data_ptr(), B.shape[1], int(b_mn),
           D.data_ptr(), ldd, bn, ksplit, int(atomic_t), torch.cuda.current_stream().cuda_stream)
    assert st == 0, L.airt_last_error()
    torch.cuda.synchronize()
    return D.t() if atomic_t else D


@pytest.mark.parametrize("a_mn,b_mn", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("bn", [32, 64, 128, 256])
def test_gemm_layouts(a_mn, b_mn, bn, path):
    import torch
    torch.manual_seed(bn + 2 * a_mn + b_mn)
    M, N, K = 200, 48 if bn == 32 else bn + 40, 192
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    ref = A.float() @ B.float().t()
    Ain = A.t().contiguous() if a_mn else A
    Bin = B.t().contiguous() if b_mn else B
    D = _gemm(Ain, Bin, M, N, K, a_mn, b_mn, bn)
    err = (D - ref).norm() / ref.norm()
    assert err.item() <= 1e-5


def test_gemm_splitk_atomic_transposed(path):
    import torch
    torch.manual_seed(3)
    M, N, K = 384, 64, 4096
    A = torch.randn(K, M, device="cuda").to(torch.bfloat16)   # MN-major A
    B = torch.randn(K, N, device="cuda").to(torch.bfloat16)   # MN-major B
    ref = A.float().t() @ B.float()
    D = _gemm(A, B, M, N, K, True, True, 64, ksplit=512, atomic_t=True)
    err = (D - ref).norm() / ref.norm()
    assert err.item() <= 1e-5


@pytest.mark.parametrize("K", [8, 40, 200, 1000])
def test_gemm_k_tails(K, path):
    """K not a multiple of the 64-wide slice: the TMA box reads zeros past K."""
    import torch
    torch.manual_seed(K)
    M, N = 300, 96
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    ref = A.float() @ B.float().t()
    D = _gemm(A, B, M, N, K, False, False, 128)
    assert ((D - ref).norm() / ref.norm()).item() <= 1e-5


def test_gemm_kmajor_splitk_atomic(path):
    import torch
    torch.manual_seed(5)
    M, N, K = 256, 128, 2048
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    ref = A.float() @ B.float().t()
    D = _gemm(A, B, M, N, K, False, False, 128, ksplit=256, atomic_t=True)
    assert ((D - ref).norm() / ref.norm()).item() <= 1e-5
