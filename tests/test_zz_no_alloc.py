"""fv_cg_noalloc against fv_cg, both called through the C ABI.

fv_cg_noalloc is for callers that are not allowed to allocate device memory
while they solve (their device memory is reserved up front or owned by
another runtime); it keeps its Krylov workspace in a static device array
instead of calling cudaMallocAsync.  The file name makes pytest collect it
last, so a run that stops at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from cases import diffusion_2d, equation

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # the solution tolerance of the other parity tests


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
        assert np.linalg.norm(x1 - x0) <= REL_TOL * np.linalg.norm(x0)
        assert abs(i1.final_residual - i0.final_residual) <= REL_TOL * abs(i0.final_residual)
        assert np.allclose(h1, h0, rtol=REL_TOL, atol=0.0)
    # the second call did not inherit the first call's answer
    assert np.linalg.norm(got[1][1] - got[0][1]) > 0.0


def test_cg_noalloc_rejects_sizes_beyond_its_limit(fv):
    from fvb200._lib import FV_ERR_INVALID, SolverOptions, lib
    n = 262144 + 1  # FV_NOALLOC_MAX_ROWS + 1
    ptr = np.arange(n + 1, dtype=np.int32)
    A = fv.DistributedMatrix.from_csr(ptr, np.arange(n, dtype=np.int32), np.ones(n))
    b = fv.DistributedVector(np.ones(n))
    x = fv.DistributedVector.from_size(n)
    info = __import__("fvb200._lib", fromlist=["SolverInfo"]).SolverInfo()
    st = lib().fv_cg_noalloc(A.handle, None, b.ptr(), x.ptr(), SolverOptions(1e-8, 1e-8, 10), C.byref(info), None)
    assert st == FV_ERR_INVALID
    assert b"FV_NOALLOC_MAX_ROWS" in lib().fv_last_error()
    small = fv.DistributedMatrix.from_csr(np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32), np.ones(4))
    st = lib().fv_cg_noalloc(small.handle, None, fv.DistributedVector(np.ones(4)).ptr(),
                             fv.DistributedVector.from_size(4).ptr(), SolverOptions(1e-8, 1e-8, 4094),
                             C.byref(info), None)
    assert st == FV_ERR_INVALID
