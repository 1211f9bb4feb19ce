"""GPU: the allocation-free matvec (sieb200_matvec_noalloc) against the
ordinary one (sieb200_matvec), both called through the C ABI.

The two differ only in how many column chunks the partial sums are split
into, so they agree to rounding: relative difference <= 1e-13 for
complex128 matrices and complex64 matrices (FP64 accumulation in both).
The file is collected last, so it runs both after the other tests and, on
its own, in a fresh process."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(fn, ctx, n, A, lda, prec, x, beta, y):
    from sieb200 import _lib
    _lib.check(fn(ctx.handle, n, A.data_ptr(), lda, prec, x.data_ptr(), ctypes.c_double(beta), y.data_ptr()))


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n,lda", [(1, 1), (300, 300), (1000, 1003), (6000, 6000)])
def test_noalloc_matvec_matches_matvec(prec, n, lda, gpu_ctx):
    import torch
    from sieb200 import _lib
    lib = _lib.lib()
    rng = np.random.default_rng(n + prec)
    dt = torch.complex128 if prec == 0 else torch.complex64
    A = torch.from_numpy(rng.standard_normal((n, lda)) + 1j * rng.standard_normal((n, lda))).to(dt).cuda()
    x = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    y0 = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    for beta in (0.0, 1.0):
        ref = y0.clone()
        _call(lib.sieb200_matvec, gpu_ctx, n, A, lda, prec, x, beta, ref)
        # two calls in a row: the fixed scratch is reused, nothing is reset
        for _ in range(2):
            got = y0.clone()
            torch.cuda.synchronize()
            _call(lib.sieb200_matvec_noalloc, gpu_ctx, n, A, lda, prec, x, beta, got)
            err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
            assert err <= 1e-13, (beta, err)


def test_noalloc_matvec_rejects_oversize(gpu_ctx):
    import torch
    from sieb200 import _lib
    lib = _lib.lib()
    n = 131073  # one more row than the fixed scratch holds; nothing is read
    A = torch.zeros(4, dtype=torch.complex128, device="cuda")
    x = torch.zeros(4, dtype=torch.complex128, device="cuda")
    y = torch.zeros(4, dtype=torch.complex128, device="cuda")
    st = lib.sieb200_matvec_noalloc(gpu_ctx.handle, n, A.data_ptr(), n, 0, x.data_ptr(), ctypes.c_double(0.0),
                                    y.data_ptr())
    assert st == _lib.INVALID_ARG
    assert b"131072" in lib.sieb200_last_error()


def test_noalloc_matvec_allocates_nothing(gpu_ctx):
    """After the set-up call, further calls leave the device's free memory
    unchanged (no cudaMalloc, no lazily loaded kernel code) and launch exactly
    the two kernels of the matvec each."""
    import torch
    from sieb200 import _lib
    lib = _lib.lib()
    n = 4096
    rng = np.random.default_rng(7)
    A = torch.from_numpy(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).cuda()
    x = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    ys = [torch.empty(n, dtype=torch.complex128, device="cuda") for _ in range(4)]
    _call(lib.sieb200_matvec_noalloc, gpu_ctx, n, A, n, 0, x, 0.0, ys[0])  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    launches0 = lib.sieb200_launch_count()
    for y in ys[1:]:
        _call(lib.sieb200_matvec_noalloc, gpu_ctx, n, A, n, 0, x, 0.0, y)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert lib.sieb200_launch_count() - launches0 == 2 * (len(ys) - 1)
    for y in ys[1:]:
        assert torch.equal(y, ys[0])
