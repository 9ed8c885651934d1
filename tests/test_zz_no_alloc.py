"""fwt_pdf_noalloc: the PDF entry point for callers that cannot allocate device memory.

Callers that run inside an allocator hook, between the capture and the replay of a fixed
memory plan, or under a byte-exact memory budget owned by someone else cannot let the library
call cudaMalloc.  fwt_pdf_noalloc keeps its scratch in a static device array instead.  This
test calls it through the C-ABI on a field built by the library and checks, on two calls in a
row (different data and bin counts, so stale scratch from the first call would show), that it
returns the same bins as the allocating entry point fwt_pdf: counts bit-exact, the REAL(4)
values and densities identical.

The file name sorts last, so a run that stops at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from helpers import gpu_params, oracle_inputs

pytestmark = pytest.mark.gpu


def _noalloc(F, d_ptr, nx, ny, nz, scale, nbins):
    L = F.library()
    f = L.fwt_pdf_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                  ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                  ctypes.POINTER(ctypes.c_uint64)]
    f.restype = ctypes.c_int
    val = np.zeros(nbins, dtype=np.float32)
    pdf = np.zeros(nbins, dtype=np.float32)
    cnt = np.zeros(nbins, dtype=np.uint64)
    rc = f(d_ptr, 32, nx, ny, nz, scale, nbins, None, val.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
           pdf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    assert rc == 0, F.api._err()
    return val, pdf, cnt


def test_pdf_noalloc_matches_pdf(orc):
    import torch

    import fastweavturb_b200 as F
    from fastweavturb_b200.configs import small

    w = small(N=32, seed=9, nlev=2, tubes0=1, nodes0=64)
    p, cl = oracle_inputs(orc, w)
    ctx = F.Context(gpu_params(F, w))
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    ctx.deposit()
    ctx.biot_savart()
    # raw (unnormalised) FP32 fields, exactly as stored on the device
    u_raw = np.stack([ctx.copy_field(1, c) for c in range(3)]).astype(np.float32)
    w_raw = np.stack([ctx.copy_field(0, c) for c in range(3)]).astype(np.float32)
    up = ctx.cal_helicity()["up"]
    N = w.N
    cases = [(u_raw, 0, -1, 1000, (N, N, 3 * N)),        # pooled u, the reference's pdf_um.dat
             (w_raw[0], 1, 0, 201, (N, N, N))]           # omega_x on 201 bins
    for data, which, comp, nbins, (nx, ny, nz) in cases:
        v_ref, p_ref, c_ref = ctx.export_pdf(which=which, component=comp, nbins=nbins)
        d = torch.from_numpy(np.ascontiguousarray(data).reshape(-1)).cuda()
        torch.cuda.synchronize()
        v, pdf, cnt = _noalloc(F, d.data_ptr(), nx, ny, nz, 1.0 / up, nbins)
        assert np.array_equal(cnt, c_ref), "bin counts differ"
        assert np.array_equal(v, v_ref)
        assert np.array_equal(pdf, p_ref)
        assert int(cnt.sum()) > 0.99 * data.size
    ctx.close()


def test_pdf_noalloc_rejects_too_many_bins():
    import torch

    import fastweavturb_b200 as F

    d = torch.zeros(8, device="cuda")
    L = F.library()
    f = L.fwt_pdf_noalloc
    f.restype = ctypes.c_int
    val = np.zeros(8193, dtype=np.float32)
    rc = f(ctypes.c_void_p(d.data_ptr()), 32, 2, 2, 2, ctypes.c_double(1.0), 8193, None,
           val.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), None, None)
    assert rc == -7   # FWT_E_RANGE
