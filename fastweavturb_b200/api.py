"""ctypes binding of libfwt (include/fwt.h).

The method names mirror the reference's Fortran routines so that a caller of the reference
finds the same steps:

=====================  ==========================================  =========================
method                 reference                                    C entry point
=====================  ==========================================  =========================
``load_inputs``        tube.f90:168-223, 341-379                    fwt_load_inputs
``set_centerlines``    tube.f90:353-379 (after the broadcasts)      fwt_set_centerlines
``deposit``            tube.f90:392-946                             fwt_deposit
``filter_spec``        subroutine.f90:1225-1277                     fwt_filter
``biot_savart``        tube.f90:972-1023                            fwt_biot_savart
``cal_helicity``       tube.f90:1026-1044                           fwt_normalize
``spectrum``           subroutine.f90:1604-1638                     fwt_spectrum
``export_pdf``         subroutine.f90:1-62                          fwt_pdf
``Sp_calculate``       subroutine.f90:64-129                        fwt_sp
``output_v``           tube.f90:1055-1071, subroutine.f90:1342      fwt_field_wh
``run``                tube.f90:392-1188                            fwt_run
``write_outputs``      the output tree of tube.f90                  fwt_write_outputs
=====================  ==========================================  =========================

Errors raise :class:`FwtError` with the library's message, as the reference would abort.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libfwt.so")
_lib = None


class FwtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libfwt error {code}: {msg}")
        self.code = code


class _Params(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("N_downsample", ctypes.c_int), ("line_s", ctypes.c_int), ("line_e", ctypes.c_int),
        ("sigma_ratio", ctypes.c_double), ("eta_t", ctypes.c_double), ("ntf_times", ctypes.c_int),
        ("ntf_pre", ctypes.c_int), ("Rtube_ratio", ctypes.c_double), ("dzeta_sup", ctypes.c_double),
        ("precision", ctypes.c_int), ("deposit_mode", ctypes.c_int), ("device", ctypes.c_int),
        ("stream", ctypes.c_void_p), ("if_pdf", ctypes.c_int), ("if_Sp", ctypes.c_int), ("Sp_order", ctypes.c_int),
        ("pdf_bins", ctypes.c_int), ("vorticity_output", ctypes.c_int), ("mem_cap", ctypes.c_size_t),
    ]


EXPORTS = [
    "fwt_default_params", "fwt_create", "fwt_destroy", "fwt_load_inputs", "fwt_check_inputs", "fwt_set_centerlines",
    "fwt_set_centerlines_async", "fwt_set_centerlines_device", "fwt_deposit", "fwt_filter", "fwt_biot_savart",
    "fwt_normalize", "fwt_spectrum",
    "fwt_pdf", "fwt_pdf_noalloc", "fwt_sp", "fwt_sp_exponents", "fwt_field_wh", "fwt_field_uw", "fwt_field_wd",
    "fwt_set_outputs", "fwt_copy_field", "fwt_field_device", "fwt_vsf_deviation", "fwt_helicity",
    "fwt_isosurface", "fwt_set_slab", "fwt_biot_savart_block", "fwt_sp_block",
    "fwt_write_outputs", "fwt_run_dir", "fwt_run",
    "fwt_timings", "fwt_kernel_times", "fwt_counters", "fwt_last_error", "fwt_fbb_generate", "fwt_fbb_signs",
    "fwt_set_tuning", "fwt_mlp_create", "fwt_mlp_destroy", "fwt_mlp_nparams", "fwt_mlp_get_params", "fwt_mlp_set_params",
    "fwt_mlp_forward", "fwt_mlp_loss_grad", "fwt_mlp_train_step", "fwt_gemm_bf16",
]


def library(path: str | None = None):
    """Load libfwt.so (built in-tree by fastweavturb_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or _LIB_PATH
    if not os.path.exists(p):
        raise FwtError(-2, f"{p} is missing: build it with `python -m fastweavturb_b200.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(p)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    sig = {
        "fwt_default_params": [ctypes.POINTER(_Params)],
        "fwt_create": [ctypes.POINTER(_Params), ctypes.POINTER(vp)],
        "fwt_destroy": [vp],
        "fwt_load_inputs": [vp, ctypes.c_char_p, ctypes.c_char_p],
        "fwt_check_inputs": [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_Params), ctypes.POINTER(ip), i64p],
        "fwt_set_centerlines": [vp, ip, i64p, dp, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
        "fwt_set_centerlines_async": [vp, ip, i64p, dp, dp, dp, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)],
        "fwt_set_centerlines_device": [vp, ip, i64p, vp, vp, vp, dp, dp, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)],
        "fwt_deposit": [vp, ip, ip],
        "fwt_filter": [vp, ctypes.c_double],
        "fwt_biot_savart": [vp],
        "fwt_normalize": [vp, dp, dp, dp],
        "fwt_spectrum": [vp, ip, dp, ip],
        "fwt_pdf": [vp, ip, ip, ip, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                    ctypes.POINTER(ctypes.c_uint64)],
        "fwt_sp": [vp, ip, ctypes.POINTER(ctypes.c_int), ip, dp],
        "fwt_sp_exponents": [dp, dp, ip, ip, dp, dp],
        "fwt_field_wh": [vp, ctypes.POINTER(ctypes.c_float)],
        "fwt_field_uw": [vp, ctypes.POINTER(ctypes.c_float)],
        "fwt_field_wd": [vp, ctypes.POINTER(ctypes.c_float)],
        "fwt_set_outputs": [vp, ip, ip],
        "fwt_copy_field": [vp, ip, ip, dp],
        "fwt_field_device": [vp, ip, ctypes.POINTER(vp)],
        "fwt_vsf_deviation": [vp, vp, dp],
        "fwt_helicity": [vp, dp],
        "fwt_isosurface": [vp, ctypes.c_float, ctypes.POINTER(ctypes.c_float), ctypes.c_int64, i64p,
                           ctypes.POINTER(ctypes.c_float)],
        "fwt_set_slab": [vp, ip, ip],
        "fwt_biot_savart_block": [vp, vp, ip, ip, dp],
        "fwt_sp_block": [vp, vp, ip, ip, ip, ip, ctypes.c_double, ctypes.POINTER(ctypes.c_int), ip, dp],
        "fwt_write_outputs": [vp, ctypes.c_char_p],
        "fwt_run_dir": [ctypes.c_char_p, ctypes.POINTER(_Params)],
        "fwt_run": [vp],
        "fwt_timings": [vp, dp, ip],
        "fwt_kernel_times": [vp, dp, i64p, ip],
        "fwt_counters": [vp, i64p, ip],
        "fwt_set_tuning": [vp, ip, ctypes.c_double],
        "fwt_last_error": [ctypes.c_char_p, ip],
        "fwt_fbb_generate": [vp, ctypes.c_uint64, ip, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), dp,
                             dp, vp, vp, vp],
        "fwt_fbb_signs": [ctypes.c_uint64, ip, ctypes.POINTER(ctypes.c_int)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    _lib = L
    return L


def _err():
    buf = ctypes.create_string_buffer(1024)
    library().fwt_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def _check(rc):
    if rc != 0:
        raise FwtError(rc, _err())
    return rc


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


@dataclass
class Params:
    """parameters_input.dat scalars plus the reference's compile-time switches."""
    N: int = 64
    N_downsample: int = 64
    line_s: int = 1
    line_e: int = 1
    sigma_ratio: float = 4.0
    eta_t: float = 0.0
    ntf_times: int = 50
    ntf_pre: int = 1000
    Rtube_ratio: float = 3.0
    dzeta_sup: float = 1e-4
    precision: int = 32
    deposit_mode: int = 0
    device: int = 0
    stream: int = 0
    if_pdf: int = 1
    if_Sp: int = 1
    Sp_order: int = 10
    pdf_bins: int = 1000
    vorticity_output: int = 1
    mem_cap: int = 0

    def to_c(self):
        p = _Params()
        for f, _ in _Params._fields_:
            v = getattr(self, f)
            setattr(p, f, v if f != "stream" else (v or None))
        return p


def sp_separations(N):
    """r_m = floor(sqrt(2.0)**m + 0.5), m = 0..2*floor(log2 N + 0.01), REAL(4) (subroutine.f90:78,98)."""
    f32 = np.float32
    lg2L = int(np.floor(f32(np.log(f32(N)) / np.log(f32(2.0))) + f32(0.01)))
    s2 = f32(np.sqrt(f32(2.0)))
    out = []
    for m in range(2 * lg2L + 1):
        p, base, e = f32(1.0), s2, m
        while e:
            if e & 1:
                p = f32(p * base)
            base = f32(base * base)
            e >>= 1
        out.append(int(np.floor(f32(p + f32(0.5)))))
    return np.array(out, dtype=np.int32)


class Context:
    """One libfwt context (device buffers, FFT plans, stream) for one field."""

    def __init__(self, params: Params | None = None, **kw):
        self.params = params or Params(**kw)
        L = library()
        self._h = ctypes.c_void_p()
        self._p = self.params.to_c()
        _check(L.fwt_create(ctypes.byref(self._p), ctypes.byref(self._h)))
        self.N = self.params.N

    # ------------------------------------------------------------------ life cycle
    def close(self):
        if self._h:
            library().fwt_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ inputs
    def load_inputs(self, centerline_path, params_path):
        _check(library().fwt_load_inputs(self._h, str(centerline_path).encode(), str(params_path).encode()))

    def set_centerlines(self, npoint, xyz, sigma, Gamma, n_T, if_filter=None, async_upload=False):
        """Host centerlines: npoint per line, xyz (npointall, 3) FP64.  async_upload: the copy
        runs behind the deposition (fwt_set_centerlines_async); the context keeps xyz alive
        until the next deposition returns, and xyz must not change before then."""
        npoint = np.ascontiguousarray(npoint, dtype=np.int64)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        nl = len(npoint)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        Gamma = np.ascontiguousarray(Gamma, dtype=np.float64)
        n_T = np.ascontiguousarray(n_T, dtype=np.int32)
        filt = np.ascontiguousarray(np.zeros(nl) if if_filter is None else if_filter, dtype=np.int32)
        f = library().fwt_set_centerlines_async if async_upload else library().fwt_set_centerlines
        self._upload = xyz if async_upload else None
        _check(f(self._h, nl, _ptr(npoint, ctypes.c_int64), _ptr(xyz, ctypes.c_double), _ptr(sigma, ctypes.c_double),
                 _ptr(Gamma, ctypes.c_double), _ptr(n_T, ctypes.c_int), _ptr(filt, ctypes.c_int)))

    def set_centerlines_device(self, npoint, dx, dy, dz, sigma, Gamma, n_T, if_filter=None):
        """dx, dy, dz: device pointers (int) to FP64 node coordinates on this context's GPU."""
        npoint = np.ascontiguousarray(npoint, dtype=np.int64)
        nl = len(npoint)
        sigma = np.ascontiguousarray(sigma, dtype=np.float64)
        Gamma = np.ascontiguousarray(Gamma, dtype=np.float64)
        n_T = np.ascontiguousarray(n_T, dtype=np.int32)
        filt = np.ascontiguousarray(np.zeros(nl) if if_filter is None else if_filter, dtype=np.int32)
        self._keep = (npoint, sigma, Gamma, n_T, filt)
        _check(library().fwt_set_centerlines_device(self._h, nl, _ptr(npoint, ctypes.c_int64), dx, dy, dz,
                                                    _ptr(sigma, ctypes.c_double), _ptr(Gamma, ctypes.c_double),
                                                    _ptr(n_T, ctypes.c_int), _ptr(filt, ctypes.c_int)))

    # ------------------------------------------------------------------ phases
    def deposit(self, line_s=None, line_e=None):
        _check(library().fwt_deposit(self._h, line_s or self.params.line_s, line_e or self.params.line_e))

    def filter_spec(self, k_c):
        _check(library().fwt_filter(self._h, float(k_c)))

    def biot_savart(self):
        _check(library().fwt_biot_savart(self._h))

    def cal_helicity(self):
        """Normalisation by u' (tube.f90:1026-1044); returns dict(up, Etot, Enstrophy)."""
        up, E, en = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(library().fwt_normalize(self._h, ctypes.byref(up), ctypes.byref(E), ctypes.byref(en)))
        return {"up": up.value, "Etot": E.value, "Enstrophy": en.value}

    def spectrum(self, which=1):
        out = np.zeros(self.N // 2)
        _check(library().fwt_spectrum(self._h, which, _ptr(out, ctypes.c_double), len(out)))
        return out

    def export_pdf(self, which=0, component=-1, nbins=1000):
        val = np.zeros(nbins, dtype=np.float32)
        pdf = np.zeros(nbins, dtype=np.float32)
        cnt = np.zeros(nbins, dtype=np.uint64)
        _check(library().fwt_pdf(self._h, which, component, nbins, _ptr(val, ctypes.c_float),
                                 _ptr(pdf, ctypes.c_float), _ptr(cnt, ctypes.c_uint64)))
        return val, pdf, cnt

    def Sp_calculate(self, pmax=10, r=None):
        r = sp_separations(self.N) if r is None else np.ascontiguousarray(r, dtype=np.int32)
        out = np.zeros(pmax * len(r))
        _check(library().fwt_sp(self._h, pmax, _ptr(r, ctypes.c_int), len(r), _ptr(out, ctypes.c_double)))
        return r, out.reshape(pmax, len(r))

    def output_v(self, out=None):
        """Downsampled |omega| and helicity of the normalised fields: (2, nd, nd, nd) [k, j, i]
        (field_wh.dat).  `out`: a C-contiguous float32 array of 2 nd^3 elements to write into
        (pinned host memory, e.g. a pinned torch tensor's numpy view, copies at the link's full
        rate; a fresh numpy array goes through the driver's pageable staging)."""
        nd = self.params.N_downsample
        if out is None:
            out = np.zeros(2 * nd ** 3, dtype=np.float32)
        elif out.dtype != np.float32 or out.size != 2 * nd ** 3 or not out.flags.c_contiguous:
            raise ValueError("out: a C-contiguous float32 array of 2 * N_downsample^3 elements")
        _check(library().fwt_field_wh(self._h, _ptr(out, ctypes.c_float)))
        return out.reshape(2, nd, nd, nd)

    def set_outputs(self, u_out=False, d_out=False):
        """The reference's u_out / d_out switches: write_outputs also writes field_uw.dat /
        field_wd.dat."""
        _check(library().fwt_set_outputs(self._h, int(bool(u_out)), int(bool(d_out))))

    def field_uw(self):
        """Downsampled ux, uy, uz, wx, wy, wz of the normalised fields: (6, nd, nd, nd) [k, j, i]."""
        nd = self.params.N_downsample
        out = np.zeros(6 * nd ** 3, dtype=np.float32)
        _check(library().fwt_field_uw(self._h, _ptr(out, ctypes.c_float)))
        return out.reshape(6, nd, nd, nd)

    def field_wd(self):
        """Downsampled |omega| and the dissipation S_ij S_ij: (2, nd, nd, nd) [k, j, i]."""
        nd = self.params.N_downsample
        out = np.zeros(2 * nd ** 3, dtype=np.float32)
        _check(library().fwt_field_wd(self._h, _ptr(out, ctypes.c_float)))
        return out.reshape(2, nd, nd, nd)

    def copy_field(self, which, component):
        """which 0: omega, 1: u; normalised once cal_helicity ran.  Array [k, j, i]."""
        nz = self._slab[1] if getattr(self, "_slab", None) else self.N
        out = np.zeros(self.N * self.N * nz)
        _check(library().fwt_copy_field(self._h, which, component, _ptr(out, ctypes.c_double)))
        return out.reshape(nz, self.N, self.N)

    def field(self, which):
        return np.stack([self.copy_field(which, c) for c in range(3)])

    def run(self):
        _check(library().fwt_run(self._h))

    def write_outputs(self, outdir):
        _check(library().fwt_write_outputs(self._h, str(outdir).encode()))

    def timings(self):
        t = np.zeros(5)
        library().fwt_timings(self._h, _ptr(t, ctypes.c_double), 5)
        return {"setup_ms": t[0], "deposit_ms": t[1], "spectral_ms": t[2], "stats_ms": t[3], "total_ms": t[4]}

    KERNEL_CATEGORIES = ("section_presample", "centerline_setup", "binning", "deposit", "biot_savart", "cufft",
                         "statistics", "generator")

    def kernel_times(self):
        """Per-category device ms and launch counts of the last run()."""
        ms = np.zeros(8)
        n = np.zeros(8, dtype=np.int64)
        library().fwt_kernel_times(self._h, _ptr(ms, ctypes.c_double), _ptr(n, ctypes.c_int64), 8)
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_CATEGORIES)}

    def set_piece_radius_limit(self, cells):
        """Tubes up to this truncation radius (grid spacings) take the chord-piece kernel."""
        _check(library().fwt_set_tuning(self._h, 1, float(cells)))

    def set_raster_radius_limit(self, cells):
        """Piece tubes up to this truncation radius (grid spacings) are rasterised once per piece
        (0: never, the default; negative: the default)."""
        _check(library().fwt_set_tuning(self._h, 2, float(cells)))

    def set_scatter_radius_limit(self, cells):
        """FP32 piece tubes up to this truncation radius (grid spacings) are deposited without
        tiles, with int64 global reductions (0: never; negative: the default, 5)."""
        _check(library().fwt_set_tuning(self._h, 3, float(cells)))

    def set_defer_limit(self, pairs):
        """Most entries the list of pairs handed from FP32 to FP64 grows to; more are listed
        and evaluated in windows of tiles or pieces (below 1: the default, 2^26)."""
        _check(library().fwt_set_tuning(self._h, 4, float(pairs)))

    def counters(self):
        v = np.zeros(7, dtype=np.int64)
        library().fwt_counters(self._h, _ptr(v, ctypes.c_int64), 7)
        return {"lines": int(v[0]), "sections": int(v[1]), "subsegments": int(v[2]), "pairs": int(v[3]),
                "launches": int(v[4]), "accepted": int(v[5]), "redone_fp64": int(v[6])}

    def vsf_deviation(self, phi_ptr=None):
        """cal_deviation (subroutine.f90:1519-1546) of omega against the scalar field at device
        address phi_ptr (N^3, the context's precision), or against |omega| when None."""
        out = ctypes.c_double()
        _check(library().fwt_vsf_deviation(self._h, phi_ptr, ctypes.byref(out)))
        return out.value

    def helicity(self):
        """Total helicity sum(omega . u) dv (cal_helicity of omega and u, subroutine.f90:1550-1569)."""
        out = ctypes.c_double()
        _check(library().fwt_helicity(self._h, ctypes.byref(out)))
        return out.value

    def isosurface(self, iso=0.0):
        """Triangles (T, 3, 4): vertices (x, y, z, helicity) of the |omega| isosurface of the
        field_wh box (output/field_wh_norm.py:56-89), and the iso value used (iso <= 0: the
        script's 3 rms(|omega|) / sqrt 2)."""
        n = ctypes.c_int64()
        used = ctypes.c_float()
        _check(library().fwt_isosurface(self._h, float(iso), None, 0, ctypes.byref(n), ctypes.byref(used)))
        tris = np.zeros((max(n.value, 1), 3, 4), dtype=np.float32)
        if n.value:
            _check(library().fwt_isosurface(self._h, float(used.value), _ptr(tris, ctypes.c_float), n.value,
                                            ctypes.byref(n), ctypes.byref(used)))
        return tris[:n.value], float(used.value)

    def set_slab(self, z0, nz):
        """Hold and deposit only planes z0 .. z0 + nz - 1 (fwt_set_slab); (0, 0): the whole grid."""
        _check(library().fwt_set_slab(self._h, int(z0), int(nz)))
        self._slab = (int(z0), int(nz)) if nz else None

    def biot_savart_block(self, spec_ptr, y0, ny):
        """fwt_biot_savart_block on a device y-pencil; returns (shells_w, shells_u, energy, enstrophy)
        of the pencil."""
        nek = self.N // 2
        out = np.zeros(2 * (nek + 1) + 2)
        _check(library().fwt_biot_savart_block(self._h, ctypes.c_void_p(spec_ptr), int(y0), int(ny),
                                               _ptr(out, ctypes.c_double)))
        return out[1:nek + 1], out[nek + 2:2 * nek + 2], out[2 * nek + 2], out[2 * nek + 3]

    def sp_block(self, u_ptr, n0, n1, n2, axis, scale, r):
        """fwt_sp_block: S_p sums (10, len(r)) of one component on a device box along `axis`."""
        r = np.ascontiguousarray(r, dtype=np.int32)
        out = np.zeros(10 * len(r))
        _check(library().fwt_sp_block(self._h, ctypes.c_void_p(u_ptr), n0, n1, n2, axis, float(scale),
                                      _ptr(r, ctypes.c_int), len(r), _ptr(out, ctypes.c_double)))
        return out.reshape(10, len(r))

    def field_tensor(self, which):
        """Zero-copy torch view (3, N, N, N), index [c, z, y, x], of the raw (unnormalised)
        field on the device (which = 0: omega, 1: u), in the context's precision.  Valid until
        the field is rebuilt or the context is closed."""
        import torch

        p = ctypes.c_void_p()
        _check(library().fwt_field_device(self._h, which, ctypes.byref(p)))
        N = self.N
        nz = getattr(self, "_slab", None)[1] if getattr(self, "_slab", None) else N
        dt = "<f4" if self.params.precision == 32 else "<f8"

        class _View:
            __cuda_array_interface__ = {"shape": (3, nz, N, N), "typestr": dt, "data": (p.value, False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_View(), device=torch.device("cuda", self.params.device))

    def fbb_generate(self, seed, tubes, nodes, H, dB, dx, dy, dz):
        tubes = np.ascontiguousarray(tubes, dtype=np.int32)
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        H = np.ascontiguousarray(H, dtype=np.float64)
        dB = np.ascontiguousarray(dB, dtype=np.float64)
        _check(library().fwt_fbb_generate(self._h, ctypes.c_uint64(seed), len(tubes), _ptr(tubes, ctypes.c_int),
                                          _ptr(nodes, ctypes.c_int), _ptr(H, ctypes.c_double),
                                          _ptr(dB, ctypes.c_double), dx, dy, dz))


def sp_exponents(rdr, Sp):
    """Scaling exponents zeta_p (p = 1..pmax) and flatness S_4/S_2^2 per separation of an
    S_p table (output/stat/Sp_zeta.m:3-23, output/stat/Flatness.m:14-19).

    rdr: nr separations r*dr; Sp: (pmax, nr).  Returns (zeta, flatness)."""
    rdr = np.ascontiguousarray(rdr, dtype=np.float64)
    Sp = np.ascontiguousarray(Sp, dtype=np.float64)
    pmax, nr = Sp.shape
    zeta = np.zeros(pmax)
    flat = np.zeros(nr)
    _check(library().fwt_sp_exponents(_ptr(rdr, ctypes.c_double), _ptr(Sp, ctypes.c_double), nr, pmax,
                                      _ptr(zeta, ctypes.c_double), _ptr(flat, ctypes.c_double)))
    return zeta, flat


def run_dir(rundir, params: Params | None = None):
    """The whole program in `rundir` (reads both input files, writes rundir/output)."""
    p = (params or Params()).to_c()
    _check(library().fwt_run_dir(str(rundir).encode(), ctypes.byref(p)))


def fbb_signs(seed, ntubes):
    out = np.zeros(ntubes, dtype=np.int32)
    _check(library().fwt_fbb_signs(ctypes.c_uint64(seed), ntubes, _ptr(out, ctypes.c_int)))
    return out


def check_inputs(rundir):
    """Read and validate rundir/centerline_input.dat and rundir/parameters_input.dat without a
    GPU (fwt_check_inputs); returns (params dict, nline, nodes) or raises FwtError."""
    p = _Params()
    _check(library().fwt_default_params(ctypes.byref(p)))
    nl = ctypes.c_int()
    nodes = ctypes.c_int64()
    _check(library().fwt_check_inputs(os.path.join(str(rundir), "centerline_input.dat").encode(),
                                      os.path.join(str(rundir), "parameters_input.dat").encode(), ctypes.byref(p),
                                      ctypes.byref(nl), ctypes.byref(nodes)))
    return {f: getattr(p, f) for f, _ in _Params._fields_}, nl.value, nodes.value


def write_ply(path, tris):
    """Write isosurface triangles (T, 3, 4): x, y, z, helicity per vertex (Context.isosurface)
    as a binary little-endian PLY mesh: 3T vertices with a float `helicity` property and T
    triangular faces.  The headless stand-in for the rendering script's screenshot
    (output/field_wh_norm.py:114-118): any mesh viewer colours it by the helicity."""
    tris = np.ascontiguousarray(tris, dtype="<f4").reshape(-1, 3, 4)
    T = tris.shape[0]
    head = ("ply\nformat binary_little_endian 1.0\ncomment |omega| isosurface coloured by the helicity omega.u\n"
            f"element vertex {3 * T}\nproperty float x\nproperty float y\nproperty float z\n"
            f"property float helicity\nelement face {T}\nproperty list uchar int vertex_indices\nend_header\n")
    faces = np.zeros(T, dtype=[("n", "u1"), ("v", "<i4", (3,))])
    faces["n"] = 3
    faces["v"] = np.arange(3 * T, dtype="<i4").reshape(T, 3)
    with open(path, "wb") as f:
        f.write(head.encode("ascii"))
        f.write(tris.tobytes())
        f.write(faces.tobytes())
