"""mxp_otf_gemv_noalloc: the residual GEMV for callers that cannot allocate
device memory (no workspace; its scratch is a fixed array inside the library).
Checked through the C ABI against the workspace entry point mxp_otf_gemv, at
the GEMV tolerance of the other tests, on two calls in a row (the second call
finds the first call's partial sums still in the shared array).  This file is
collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    f = L.mxp_otf_gemv_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_uint64, C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                  C.c_void_p]
    return f


def test_noalloc_gemv_matches_workspace_gemv_twice(mxp, orc, torch_cuda):
    torch = torch_cuda
    L = mxp.lib()
    noalloc = _bind(L)
    stream = torch.cuda.current_stream().cuda_stream
    # the largest n (two column splits fill the array exactly) and one just below it
    cases = [(4096, 42, -1.0, 1.0), (122880, 7, 0.5, 0.0), (262144, 3, -1.0, 1.0), (262080, 11, 1.0, -0.5)]
    for n, seed, alpha, beta in cases:
        _, d, _, _ = orc.matgen(n, seed, with_matrix=False) if n <= 8192 else (None, None, None, None)
        if d is None:
            dd = torch.empty(n, dtype=torch.float64, device="cuda")
            assert L.mxp_matgen(n, seed, 0, None, n, dd.data_ptr(), None, None, stream) == 0
        else:
            dd = torch.from_numpy(d).cuda()
        rng = np.random.default_rng(n)
        ws = mxp.Workspace(n, 256, 0)
        for call in range(2):
            x = torch.from_numpy(rng.standard_normal(n)).cuda()
            y0 = torch.from_numpy(rng.standard_normal(n)).cuda()
            y_ref = y0.clone()
            y_new = y0.clone()
            mxp.otf_gemv(n, seed, dd, alpha, x, beta, y_ref, ws)
            st = noalloc(n, seed, dd.data_ptr(), alpha, x.data_ptr(), beta, y_new.data_ptr(), stream)
            assert st == 0, L.mxp_last_error_string()
            torch.cuda.synchronize()
            a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
            # |A| x bound: |a_ij| <= 0.5 off the diagonal, d on it
            scale = abs(alpha) * (0.5 * np.abs(x.cpu().numpy()).sum() + dd.cpu().numpy() * np.abs(x.cpu().numpy())) \
                + abs(beta) * np.abs(y0.cpu().numpy())
            assert np.all(np.abs(a - b) <= 1e-14 * scale + 1e-300), (n, call)


def test_noalloc_gemv_rejects_too_large(mxp, torch_cuda):
    L = mxp.lib()
    noalloc = _bind(L)
    x = torch_cuda.zeros(8, dtype=torch_cuda.float64, device="cuda")
    st = noalloc(262145, 1, x.data_ptr(), 1.0, x.data_ptr(), 0.0, x.data_ptr(), None)
    assert st == mxp.INVALID_ARG
    assert b"262144" in L.mxp_last_error_string()
