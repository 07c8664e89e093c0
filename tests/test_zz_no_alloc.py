"""The allocation-free matvec entry point (dda_matvec_noalloc).

It serves callers that cannot allocate device memory where they need A.x:
serving loops whose latency budget rules out allocator calls, and host
applications whose device memory belongs to another framework's pool.  The
test calls it through the C ABI twice in a row, in every product mode, and
checks each result against the allocating entry point (dda_matvec, through
DDAOperator) with the tolerances the other matvec tests use.  It lives in its
own file named to be collected last, and passes alone in a fresh process or
after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu


def _problem(shape, seed):
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / 0.5
    d = 0.4 / k
    a = O.calculate_alpha(1.6 + 0.05j, d, k, method="RR")
    alpha = np.where(rng.random(shape) < 0.7, a, 0)
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    xs = [rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,)) for _ in range(2)]
    bs = [rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,)) for _ in range(2)]
    return k, d, ia, xs, bs


MODES = ["MV_AX", "MV_RESIDUAL", "MV_CONV", "MV_CONV_MASKED"]


def _allocating(op, mode, xt, bm):
    if mode == "MV_AX":
        return op.matvec(xt)
    if mode == "MV_RESIDUAL":
        return op.residual(bm, xt)
    if mode == "MV_CONV":
        return op.conv(xt)
    return op.conv_masked(xt)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 2e-5)])
@pytest.mark.parametrize("shape", [(8, 10, 12), (24, 16, 20)])
def test_noalloc_matches_allocating_matvec_twice(dtype, tol, shape, mode):
    import precondda_b200 as P
    from precondda_b200 import _lib as L
    k, d, ia, xs, bs = _problem(shape, seed=11)
    op = P.DDAOperator(ia, k, d, dtype=dtype)
    code = L.DDA_C128 if dtype == torch.complex128 else L.DDA_C64
    stream = torch.cuda.current_stream().cuda_stream
    for x, b in zip(xs, bs):                       # two calls in a row
        xt = torch.as_tensor(x, device="cuda").to(dtype).contiguous()
        # the residual mode takes b already masked, as dda_matvec does
        bm = (torch.as_tensor(b, device="cuda").to(dtype) * op.mask[..., None]).contiguous()
        y = torch.empty_like(xt)
        rc = L.lib().dda_matvec_noalloc(code, *op.shape, *op.L, op.ghat.data_ptr(), op.gscale,
                                        op.inv_alpha.data_ptr(), getattr(L, mode), xt.data_ptr(), y.data_ptr(),
                                        bm.data_ptr() if mode == "MV_RESIDUAL" else None, stream)
        assert rc == L.DDA_OK, L.lib().dda_last_error()
        ref = _allocating(op, mode, xt, bm)
        err = (y - ref).abs().max().item() / ref.abs().max().item()
        assert err < tol, (mode, err)


def test_noalloc_rejects_oversized_problem():
    from precondda_b200 import _lib as L
    # 256^3 box, FFT 512^3: far beyond the static scratch; rejected before any launch
    rc = L.lib().dda_matvec_noalloc(L.DDA_C64, 256, 256, 256, 512, 512, 512, ctypes.c_void_p(16), 1.0,
                                    ctypes.c_void_p(16), L.MV_AX, ctypes.c_void_p(16), ctypes.c_void_p(32), None,
                                    None)
    assert rc == L.DDA_ERR_BAD_SHAPE
    assert b"static buffer" in L.lib().dda_last_error()
