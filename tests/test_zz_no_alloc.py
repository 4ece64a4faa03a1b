"""fv_cg_noalloc against fv_cg, both called through the C ABI.

fv_cg_noalloc is for callers that are not allowed to allocate device memory
while they solve (their device memory is reserved up front or owned by
another runtime); it keeps its Krylov workspace in a static device array
instead of calling cudaMallocAsync.  It launches the same kernels in the same
order as fv_cg, so its solution and residual history are the same bits.  The
file name makes pytest collect it last, so a run that stops at the first
failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cases import diffusion_2d, equation

pytestmark = pytest.mark.gpu

# cuMemPoolGetAttribute / cuMemPoolSetAttribute attributes (cuda.h, CUmemPool_attribute)
RESERVED_MEM_CURRENT, USED_MEM_CURRENT, USED_MEM_HIGH = 5, 7, 8


def _call(fn, A, P, b, opts):
    import torch
    from fvb200._lib import SolverInfo
    x = torch.zeros(b.numel(), dtype=torch.float64, device="cuda")
    hist = np.zeros(int(opts.max_iterations) + 2)
    info = SolverInfo()
    info.history = hist.ctypes.data_as(C.POINTER(C.c_double))
    info.history_cap = len(hist)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = fn(A.handle, P.handle, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), opts, C.byref(info),
                stream)
    torch.cuda.synchronize()
    return status, x.cpu().numpy(), info, hist[: info.history_len].copy()


class _DefaultPool:
    """The device's default stream-ordered memory pool (the one cudaMallocAsync
    draws from), read through the driver API."""

    def __init__(self, device=0):
        self.cu = C.CDLL("libcuda.so.1")
        self.pool = C.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(C.byref(self.pool), C.c_int(device)) == 0

    def get(self, attr):
        v = C.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, C.c_int(attr), C.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = C.c_uint64(0)
        assert self.cu.cuMemPoolSetAttribute(self.pool, C.c_int(USED_MEM_HIGH), C.byref(zero)) == 0


def test_cg_noalloc_matches_cg_on_two_calls_in_a_row(fv):
    import torch
    from fvb200._lib import SolverOptions, lib
    case = diffusion_2d(fv, 48, seed=5)
    A, b = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    opts = SolverOptions(1e-10, 1e-10, 2000)
    g = torch.Generator(device="cpu").manual_seed(7)
    b2 = (b.data * (1.0 + torch.rand(b.data.numel(), generator=g, dtype=torch.float64).cuda())).contiguous()
    rhs = [b.data, b2]
    got = [_call(lib().fv_cg_noalloc, A, P, r, opts) for r in rhs]       # two calls in a row
    want = [_call(lib().fv_cg, A, P, r, opts) for r in rhs]
    for (s1, x1, i1, h1), (s0, x0, i0, h0) in zip(got, want):
        assert s1 == 0 and s0 == 0
        assert i1.iterations == i0.iterations and i1.iterations > 0
        assert np.array_equal(x1, x0)                      # same kernels, same order: same bits
        assert i1.final_residual == i0.final_residual
        assert i1.initial_residual == i0.initial_residual
        assert np.array_equal(h1, h0)
    # the second call did not inherit the first call's answer
    assert np.linalg.norm(got[1][1] - got[0][1]) > 0.0


def test_cg_noalloc_takes_no_device_memory_after_the_first_call(fv):
    """After one call on the device (which may load the solvers' CUDA module and
    with it the static array), later calls change neither the device's free
    memory nor the stream-ordered pool that fv_cg allocates from."""
    import torch
    from fvb200._lib import SolverOptions, lib
    case = diffusion_2d(fv, 40, seed=9)
    A, b = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    opts = SolverOptions(1e-10, 1e-10, 2000)
    x = torch.zeros(b.data.numel(), dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    from fvb200._lib import SolverInfo
    info = SolverInfo()

    def call():
        x.zero_()
        st = lib().fv_cg_noalloc(A.handle, P.handle, C.c_void_p(b.data.data_ptr()), C.c_void_p(x.data_ptr()), opts,
                                 C.byref(info), stream)
        torch.cuda.synchronize()
        assert st == 0 and info.iterations > 0

    call()  # warm-up: module, kernels and the static array are in place after it
    pool = _DefaultPool(torch.cuda.current_device())
    pool.reset_high()
    used0, reserved0 = pool.get(USED_MEM_CURRENT), pool.get(RESERVED_MEM_CURRENT)
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        call()
    free1, _ = torch.cuda.mem_get_info()
    # nothing taken: free memory did not shrink, the pool never held more than
    # before and reserved nothing more (it may only have trimmed what earlier
    # tests freed into it)
    assert free1 >= free0
    assert pool.get(USED_MEM_HIGH) == used0
    assert pool.get(RESERVED_MEM_CURRENT) <= reserved0


def test_cg_noalloc_rejects_sizes_beyond_its_limit(fv):
    from fvb200._lib import FV_ERR_INVALID, SolverInfo, SolverOptions, lib
    n = 262144 + 1  # FV_NOALLOC_MAX_ROWS + 1
    ptr = np.arange(n + 1, dtype=np.int32)
    A = fv.DistributedMatrix.from_csr(ptr, np.arange(n, dtype=np.int32), np.ones(n))
    b = fv.DistributedVector(np.ones(n))
    x = fv.DistributedVector.from_size(n)
    info = SolverInfo()
    st = lib().fv_cg_noalloc(A.handle, None, b.ptr(), x.ptr(), SolverOptions(1e-8, 1e-8, 10), C.byref(info), None)
    assert st == FV_ERR_INVALID
    assert b"FV_NOALLOC_MAX_ROWS" in lib().fv_last_error()
    small = fv.DistributedMatrix.from_csr(np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32), np.ones(4))
    st = lib().fv_cg_noalloc(small.handle, None, fv.DistributedVector(np.ones(4)).ptr(),
                             fv.DistributedVector.from_size(4).ptr(), SolverOptions(1e-8, 1e-8, 4094),
                             C.byref(info), None)
    assert st == FV_ERR_INVALID
