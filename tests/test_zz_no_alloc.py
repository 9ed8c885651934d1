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


def _noalloc(F, d_ptr, precision, nx, ny, nz, scale, nbins, stream=None, want_counts=True):
    L = F.library()
    f = L.fwt_pdf_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                  ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                  ctypes.POINTER(ctypes.c_uint64)]
    f.restype = ctypes.c_int
    val = np.zeros(nbins, dtype=np.float32)
    pdf = np.zeros(nbins, dtype=np.float32)
    cnt = np.zeros(nbins, dtype=np.uint64)
    cptr = cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)) if want_counts else None
    rc = f(d_ptr, precision, nx, ny, nz, scale, nbins, stream, val.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
           pdf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), cptr)
    assert rc == 0, F.api._err()
    return val, pdf, (cnt if want_counts else None)


@pytest.mark.parametrize("precision", [32, 64])
def test_pdf_noalloc_matches_pdf(orc, precision):
    """Two calls in a row per case: the pooled u on the reference's 1000 bins, omega_x on 201
    bins, and u_y on 8192 bins (the largest count, above the default shared-memory limit);
    on the FP32 and the FP64 path, from a torch stream, and once without a count array."""
    import torch

    import fastweavturb_b200 as F
    from fastweavturb_b200.configs import small

    w = small(N=32, seed=9, nlev=2, tubes0=1, nodes0=64)
    p, cl = oracle_inputs(orc, w)
    ctx = F.Context(gpu_params(F, w, precision=precision, deposit_mode=0 if precision == 32 else 1))
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    ctx.deposit()
    ctx.biot_savart()
    # raw (unnormalised) fields, exactly as stored on the device
    dt = np.float32 if precision == 32 else np.float64
    u_raw = np.stack([ctx.copy_field(1, c) for c in range(3)]).astype(dt)
    w_raw = np.stack([ctx.copy_field(0, c) for c in range(3)]).astype(dt)
    up = ctx.cal_helicity()["up"]
    N = w.N
    stream = torch.cuda.Stream()
    cases = [(u_raw, 0, -1, 1000, (N, N, 3 * N), None, True),      # pooled u, the reference's pdf_um.dat
             (w_raw[0], 1, 0, 201, (N, N, N), None, True),           # omega_x on 201 bins
             (u_raw[1], 0, 1, 8192, (N, N, N), stream, True),        # u_y on 8192 bins, caller's stream
             (w_raw[2], 1, 2, 333, (N, N, N), stream, False)]        # omega_z, no count array
    for data, which, comp, nbins, (nx, ny, nz), st, want in cases:
        v_ref, p_ref, c_ref = ctx.export_pdf(which=which, component=comp, nbins=nbins)
        d = torch.from_numpy(np.ascontiguousarray(data).reshape(-1)).cuda()
        torch.cuda.synchronize()
        h = ctypes.c_void_p(st.cuda_stream) if st is not None else None
        v, pdf, cnt = _noalloc(F, d.data_ptr(), precision, nx, ny, nz, 1.0 / up, nbins, h, want)
        if want:
            assert np.array_equal(cnt, c_ref), "bin counts differ"
            assert int(cnt.sum()) > 0.99 * data.size
        assert np.array_equal(v, v_ref)
        assert np.array_equal(pdf, p_ref)
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
