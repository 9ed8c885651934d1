"""FP64 CPU ORACLE for the woven-field construction path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
leg may import this module, and only as the checker.  The product path (the CUDA
library ``fastweavturb_b200``) never calls it.

It restates the reference program ``Weav_ver5_8_2`` (tube.f90 + subroutine.f90):

* deposition (tube.f90:392-904) -> C restatement in ``fwt_oracle.c`` (OpenMP over z-slabs)
* per-line spectral filter        -> :func:`filter_spec`   (subroutine.f90:1225-1277)
* 3-D FFT with 1/N per axis        -> :func:`fourier_forward` / :func:`fourier_backward`
                                      (subroutine.f90:983-1084, mathematically identical
                                      c2c transform via numpy's pocketfft)
* Biot-Savart                      -> :func:`biot_savart` (tube.f90:994-1007)
* energy normalisation             -> :func:`normalise` (tube.f90:1026-1044)
* spectrum                         -> :func:`spectrum` (subroutine.f90:1604-1638)
* PDF                              -> :func:`pdf` (subroutine.f90:1-62)
* structure functions              -> :func:`structure_functions` (subroutine.f90:64-129)
* field output                     -> :func:`field_wh` (tube.f90:1055-1073)

Parity status: UNPINNED against the reference binary (Fortran + MPI + FFTW; no Fortran
compiler exists in this image and the reference ships no golden outputs).  The oracle is
pinned by analytic known-answer tests instead (tests/test_oracle_kat.py).

Array convention: a field is a numpy array of shape (N, N, N) indexed [k, j, i] in C
order, i.e. the same memory order as the reference's column-major ``vor(i, j, k)``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")
_lib = None

PI = 3.141592653589793  # 4*datan(1d0)
PI2 = 2.0 * PI


def build() -> str:
    """Compile the C part of the oracle into oracle/_build/liborc.so (and the FMA-contracted
    variant liborc_fma.so)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load(path):
    """Load one build of the C restatement and declare its entry points."""
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.orc_line_prep.argtypes = [ctypes.c_int, dp, dp, dp, dp, dp, dp, dp]
    L.orc_line_ntf.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ctypes.c_int, ip, dp, dp, dp]
    L.orc_line_ntf.restype = ctypes.c_int
    L.orc_line_subsegs.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp]
    L.orc_line_subsegs.restype = ctypes.c_long
    L.orc_deposit_line.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp, dp, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, dp, dp, dp, ctypes.c_int, dp]
    L.orc_deposit_line.restype = ctypes.c_long
    L.orc_deposit_line_cond.argtypes = L.orc_deposit_line.argtypes + [dp]
    L.orc_deposit_line_cond.restype = ctypes.c_long
    L.orc_sp.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ip, ctypes.c_int, dp, ctypes.c_int]
    L.orc_philox.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                             ctypes.POINTER(ctypes.c_uint32)]
    u32p = ctypes.POINTER(ctypes.c_uint32)
    L.orc_philox_raw.argtypes = [u32p, u32p, u32p]
    L.orc_fbb_gauss.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, dp, dp]
    L.orc_fbb_shift.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
    L.orc_fbb_shift.restype = ctypes.c_double
    L.orc_fbb_sign.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
    L.orc_fbb_sign.restype = ctypes.c_int
    return L


def lib():
    global _lib
    if _lib is None:
        _lib = _load(_LIB_PATH)
    return _lib


_LIB_FMA_PATH = os.path.join(_HERE, "_build", "liborc_fma.so")
_lib_fma = None


def has_fma() -> bool:
    """Whether this host's CPU has fused multiply-add (the contracted build needs it)."""
    try:
        with open("/proc/cpuinfo") as f:
            return any(ln.startswith("flags") and " fma" in ln for ln in f)
    except OSError:
        return False


def lib_fma():
    """The same C restatement compiled with FMA contraction (-mfma -ffp-contract=fast): every
    a*b+c of the plain build fused, the operation order otherwise unchanged.  Two equally valid
    FP64 evaluations of the reference's algorithm; their distance is the reference's own
    rounding floor on a workload (its zeta interpolation amplifies ulp-level changes)."""
    global _lib_fma
    if _lib_fma is None:
        _lib_fma = _load(_LIB_FMA_PATH)
    return _lib_fma


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class _Grid(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("sigma_ratio", ctypes.c_double), ("eta0", ctypes.c_double),
                ("ntf_times", ctypes.c_int), ("ntf_pre", ctypes.c_int),
                ("Rtube_ratio", ctypes.c_double), ("dzeta_sup", ctypes.c_double)]


# ----------------------------------------------------------------------------- inputs

@dataclass
class Params:
    """Contents of parameters_input.dat (tube.f90:190-223)."""
    N: int = 64
    N_downsample: int = 64
    line_s: int = 1
    line_e: int = 1
    sigma_ratio: float = 1.0
    eta_t: float = 0.0
    ntf_times: int = 50
    ntf_pre: int = 1000
    Rtube_ratio: float = 3.0
    dzeta_sup: float = 1e-4
    sigma: np.ndarray = field(default_factory=lambda: np.zeros(0))
    Gamma: np.ndarray = field(default_factory=lambda: np.zeros(0))
    n_T: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int32))
    if_filter: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int32))


@dataclass
class Centerlines:
    """Contents of centerline_input.dat: nline, npoint per line, then x y z per node."""
    npoint: np.ndarray
    xyz: np.ndarray  # (npointall, 3)

    def line(self, i):
        off = int(np.sum(self.npoint[:i]))
        n = int(self.npoint[i])
        return self.xyz[off:off + n]


def read_centerlines(path) -> Centerlines:
    tok = open(path).read().split()
    nline = int(float(tok[0]))
    npoint = np.array([int(float(t)) for t in tok[1:1 + nline]], dtype=np.int64)
    vals = np.array([float(t) for t in tok[1 + nline:1 + nline + 3 * int(npoint.sum())]], dtype=np.float64)
    return Centerlines(npoint=npoint, xyz=vals.reshape(-1, 3))


def read_parameters(path, nline) -> Params:
    lines = [ln for ln in open(path).read().splitlines()]
    # label / value pairs in the order of tube.f90:192-217, then a header row and nline rows
    vals = [ln.split() for ln in lines]
    p = Params()
    p.N = int(vals[1][0])
    p.N_downsample = int(vals[3][0])
    p.line_s = int(vals[5][0])
    p.line_e = int(vals[7][0])
    p.sigma_ratio = float(vals[9][0])
    p.eta_t = float(vals[11][0])
    p.ntf_times = int(vals[14][0])
    p.ntf_pre = int(vals[16][0])
    p.Rtube_ratio = float(vals[18][0])
    p.dzeta_sup = float(vals[20][0])
    rows = [v for v in vals[23:23 + nline]]
    sig = np.zeros(nline)
    gam = np.zeros(nline)
    nT = np.zeros(nline, dtype=np.int32)
    filt = np.zeros(nline, dtype=np.int32)
    for r in rows:
        i = int(r[0]) - 1
        sig[i] = float(r[1]); gam[i] = float(r[2]); nT[i] = int(r[3]); filt[i] = int(r[4])
    p.sigma, p.Gamma, p.n_T, p.if_filter = sig, gam, nT, filt
    return p


# ----------------------------------------------------------------------------- construction

def line_ntf(xyz, ntf_times=50, ntf_pre=1000):
    """Per-section ntf (n_sec+1 entries), dtf and spline coefficients (tube.f90:598-657)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n = xyz.shape[0]
    cx, cy, cz = (np.ascontiguousarray(xyz[:, d]) for d in range(3))
    ntf = np.zeros(n + 1, dtype=np.int32)
    dtf = np.zeros(n + 1)
    coe = np.zeros((n + 1) * 18)
    L = ctypes.c_double()
    rc = lib().orc_line_ntf(n, _dp(cx), _dp(cy), _dp(cz), ntf_times, ntf_pre, _ip(ntf), _dp(dtf), _dp(coe),
                            ctypes.byref(L))
    if rc != 0:
        raise ValueError("line needs at least 2 nodes")
    return ntf, dtf, coe.reshape(n + 1, 3, 6), L.value


def line_prep(xyz):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n = xyz.shape[0]
    cx, cy, cz = (np.ascontiguousarray(xyz[:, d]) for d in range(3))
    cze = np.zeros(n); ck = np.zeros(3 * n); ckk = np.zeros(3 * n)
    L = ctypes.c_double()
    lib().orc_line_prep(n, _dp(cx), _dp(cy), _dp(cz), _dp(cze), _dp(ck), _dp(ckk), ctypes.byref(L))
    return cze, ck.reshape(3, n), ckk.reshape(3, n), L.value


def line_subsegs(xyz, ntf_times=50, ntf_pre=1000):
    """(nsub, 15) table: s0, s1, ci0[3], ci1[3], tci0[3], tci1[3], ndci0 (tube.f90:762-777)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n = xyz.shape[0]
    cx, cy, cz = (np.ascontiguousarray(xyz[:, d]) for d in range(3))
    cnt = lib().orc_line_subsegs(n, _dp(cx), _dp(cy), _dp(cz), ntf_times, ntf_pre, None)
    out = np.zeros(max(cnt, 1) * 15)
    lib().orc_line_subsegs(n, _dp(cx), _dp(cy), _dp(cz), ntf_times, ntf_pre, _dp(out))
    return out[:cnt * 15].reshape(cnt, 15)


def deposit(params: Params, cl: Centerlines, nthreads=None, line_s=None, line_e=None, vor=None, cond=None,
            contracted=False):
    """Deposit lines line_s..line_e (1-based, inclusive) into vor (3,N,N,N); applies the
    per-line spectral filter of lines flagged if_filter (tube.f90:528-946).

    contracted: run the FMA-contracted build (lib_fma) instead of the plain one.

    cond: optional (N,N,N) array; each point receives the maximum over its contributions of
    |1/(1 - kappa rho cos theta)|, the curved branch's amplification (1 when straight)."""
    N = params.N
    if vor is None:
        vor = np.zeros((3, N, N, N))
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    g = _Grid(N, params.sigma_ratio, params.eta_t, params.ntf_times, params.ntf_pre,
              params.Rtube_ratio, params.dzeta_sup)
    ls = params.line_s if line_s is None else line_s
    le = params.line_e if line_e is None else line_e
    stats = np.zeros(3)
    info = []
    vx, vy, vz = vor[0], vor[1], vor[2]
    for il in range(ls, le + 1):
        xyz = np.ascontiguousarray(cl.line(il - 1), dtype=np.float64)
        cx, cy, cz = (np.ascontiguousarray(xyz[:, d]) for d in range(3))
        args = (ctypes.byref(g), xyz.shape[0], _dp(cx), _dp(cy), _dp(cz), float(params.sigma[il - 1]),
                float(params.Gamma[il - 1]), int(params.n_T[il - 1]), _dp(vx), _dp(vy), _dp(vz), nthreads,
                _dp(stats))
        L = lib_fma() if contracted else lib()
        if cond is None:
            nsub = L.orc_deposit_line(*args)
        else:
            assert cond.shape == (N, N, N) and cond.dtype == np.float64 and cond.flags.c_contiguous
            nsub = L.orc_deposit_line_cond(*args, _dp(cond))
        if nsub < 0:
            raise ValueError(f"line {il}: needs at least 2 nodes")
        info.append((il, xyz.shape[0], int(stats[0]) // (xyz.shape[0] + 1), int(stats[1]), int(stats[2])))
        if params.if_filter[il - 1]:
            k_c = int(np.ceil(4.0 / params.sigma[il - 1]))
            filter_spec(k_c, vor)
    return vor, info


# ----------------------------------------------------------------------------- spectral

def wavenumbers(N):
    """kx(i) = (mod(i-1+N/2, N) - N/2) * (2pi/lx) with lx = 2pi (subroutine.f90:888-919)."""
    i = np.arange(N)
    return ((i + N // 2) % N - N // 2).astype(np.float64)


def k2_grid(N):
    k = wavenumbers(N)
    return k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2  # [kz, ky, kx]


_FFT_WORKERS = 1


def set_fft_workers(n):
    """Threads for the oracle's FFTs (scipy.fft's pocketfft; numpy's when scipy is absent)."""
    global _FFT_WORKERS
    _FFT_WORKERS = max(1, int(n))


def _fftn(a):
    try:
        import scipy.fft as sf
        return sf.fftn(a, workers=_FFT_WORKERS)
    except ImportError:
        return np.fft.fftn(a)


def _ifftn(a):
    try:
        import scipy.fft as sf
        return sf.ifftn(a, workers=_FFT_WORKERS)
    except ImportError:
        return np.fft.ifftn(a)


def fourier_forward(phy):
    """3-D forward transform scaled by 1/N per axis (subroutine.f90:983-1024)."""
    N = phy.shape[0]
    return _fftn(phy) / float(N) ** 3


def fourier_backward(spec):
    """Unscaled backward transform, real part (subroutine.f90:1037-1084)."""
    N = spec.shape[0]
    return np.real(_ifftn(spec)) * float(N) ** 3


def filter_spec(k_c, vor):
    """Sharp spectral cutoff |k|^2 > k_c^2 on each component (subroutine.f90:1225-1277)."""
    N = vor.shape[1]
    mask = k2_grid(N) > k_c ** 2
    for c in range(3):
        s = fourier_forward(vor[c])
        s[mask] = 0.0
        vor[c] = fourier_backward(s)
    return vor


def biot_savart(vor):
    """u = curl^-1 omega spectrally: u^ = i k x w^ / |k|^2, u^(0)=0 (tube.f90:991-1017)."""
    N = vor.shape[1]
    k = wavenumbers(N)
    kz, ky, kx = k[:, None, None], k[None, :, None], k[None, None, :]
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    k2s = k2.copy()
    k2s[0, 0, 0] = 1.0
    wx, wy, wz = (fourier_forward(vor[c]) for c in range(3))
    ux = 1j * (ky * wz - kz * wy) / k2s
    uy = 1j * (kz * wx - kx * wz) / k2s
    uz = 1j * (kx * wy - ky * wx) / k2s
    for s in (ux, uy, uz):
        s[0, 0, 0] = 0.0
    return np.stack([fourier_backward(ux), fourier_backward(uy), fourier_backward(uz)])


def cal_helicity(a, b, dv):
    """sum a.b * dv in the reference's serial order (subroutine.f90:1550-1569)."""
    return float(np.sum(a[0] * b[0] + a[1] * b[1] + a[2] * b[2], dtype=np.float64)) * dv


def normalise(vor, vel):
    """Scale omega and u by u' = sqrt(2E/3) (tube.f90:1026-1044).  Returns dict of scalars."""
    N = vor.shape[1]
    dx = PI2 / N
    dv = dx * dx * dx
    Etot = cal_helicity(vel, vel, dv)
    Etot = Etot / 2.0 / PI2 / PI2 / PI2
    up = np.sqrt(2 * Etot / 3)
    vor /= up
    vel /= up
    diss = cal_helicity(vor, vor, dv)
    enstrophy = diss / 2.0 / PI2 / PI2 / PI2
    return {"Etot": Etot, "up": up, "Enstrophy": enstrophy}


def spectrum(f, faithful=False):
    """Shell spectrum E(k) = sum_{nint|k|=i} 1/2 |f^|^2, i=1..nek (subroutine.f90:1604-1638).

    faithful=True reproduces the reference's REAL(4) per-mode values and REAL(4) shell sums
    (summation order within a shell is the memory order); otherwise FP64 throughout."""
    N = f.shape[1]
    nek = int(np.sqrt(np.float32((N * N * 3) / 12.0)))
    ik2 = (np.sqrt(k2_grid(N) + 0.00000001) + 0.5).astype(np.int64)
    if faithful:
        spec = np.zeros((N, N, N), dtype=np.float32)
        for c in range(3):
            s = fourier_forward(f[c])
            spec = (spec.astype(np.float64) + np.real(s * np.conj(s)) / 2.0).astype(np.float32)
        out = np.zeros(nek, dtype=np.float32)
        flat_i = ik2.ravel()
        flat_s = spec.ravel()
        for i in range(1, nek + 1):
            acc = np.float32(0.0)
            sel = flat_s[flat_i == i]
            for v in sel:  # serial float32 accumulation
                acc = np.float32(acc + v)
            out[i - 1] = acc
        return out
    e = np.zeros((N, N, N))
    for c in range(3):
        s = fourier_forward(f[c])
        e += 0.5 * (s.real ** 2 + s.imag ** 2)
    return np.bincount(ik2.ravel(), weights=e.ravel(), minlength=nek + 1)[1:nek + 1]


# ----------------------------------------------------------------------------- statistics

def pdf_edges(vmin, vmax, nbins):
    """Bin centres and edges in the reference's REAL(4) arithmetic (subroutine.f90:12-20,27)."""
    f32 = np.float32
    vmin, vmax = f32(vmin), f32(vmax)
    bsz = f32(f32(vmax - vmin) / f32(nbins))
    l = np.arange(nbins)
    # val(l) = min + 0.5d0*bin_size + real(l-1)*bin_size : the first sum is REAL(8), the
    # product real(l-1)*bin_size is REAL(4); the result is stored in REAL(4)
    val = (np.float64(vmin) + 0.5 * np.float64(bsz) + (l.astype(f32) * bsz).astype(np.float64)).astype(f32)
    half = f32(f32(0.5) * bsz)
    lo = (val - half).astype(f32)
    hi = (val + half).astype(f32)
    return val, lo, hi, bsz


def pdf_counts(data_f32, vmin, vmax, nbins):
    """Integer counts with the reference's first-match bin search (subroutine.f90:22-34):
    a value goes to the first l with lo(l) <= v < hi(l), or nowhere."""
    val, lo, hi, bsz = pdf_edges(vmin, vmax, nbins)
    v = np.asarray(data_f32, dtype=np.float32).ravel()
    # hi is non-decreasing: the first l with v < hi(l)
    l = np.searchsorted(hi, v, side="right")
    ok = l < nbins
    lc = np.minimum(l, nbins - 1)
    ok &= lo[lc] <= v
    counts = np.bincount(lc[ok], minlength=nbins).astype(np.int64)
    return val, counts, bsz


def pdf(data_f32, nbins=1000):
    """PDF of REAL(4) data shaped (nz, ny, nx) -- the pooled components stacked along z as in
    tube.f90:1169-1177 -- as (val, pdf) in REAL(4) plus integer counts (subroutine.f90:1-40)."""
    d = np.asarray(data_f32, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("pdf expects a 3-D (nz, ny, nx) array")
    vmin, vmax = d.min(), d.max()
    val, counts, bsz = pdf_counts(d, vmin, vmax, nbins)
    # pdf_v(l)/(bin_size*nx*ny*nzp*nproc), left to right in REAL(4)
    den = np.float32(bsz)
    for s in (d.shape[2], d.shape[1], d.shape[0]):
        den = np.float32(den * np.float32(s))
    p = (counts.astype(np.float32) / den).astype(np.float32)
    return val, p, counts


def sp_separations(N):
    """r_m = floor(sqrt(2.0)**m + 0.5), m = 0..2*lg2L, in REAL(4) (subroutine.f90:78,97-98)."""
    lg2L = int(np.floor(np.float32(np.log(np.float32(N)) / np.log(np.float32(2.0))) + np.float32(0.01)))
    s2 = np.float32(np.sqrt(np.float32(2.0)))
    rs = []
    for m in range(0, 2 * lg2L + 1):
        p = np.float32(1.0)
        # integer power by repeated squaring, as compilers lower x**n
        base, e = s2, m
        while e:
            if e & 1:
                p = np.float32(p * base)
            base = np.float32(base * base)
            e >>= 1
        rs.append(int(np.floor(np.float32(p + np.float32(0.5)))))
    return np.array(rs, dtype=np.int32)


def structure_functions(vel, pmax=10, r=None, nthreads=None):
    """S_p(r) = <du_x^p + du_y^p + du_z^p>/3 with longitudinal increments (subroutine.f90:64-129).
    Returns (r, Sp[pmax, nr])."""
    N = vel.shape[1]
    if r is None:
        r = sp_separations(N)
    r = np.ascontiguousarray(r, dtype=np.int32)
    out = np.zeros(pmax * len(r))
    ux, uy, uz = (np.ascontiguousarray(vel[c], dtype=np.float64) for c in range(3))
    lib().orc_sp(N, _dp(ux), _dp(uy), _dp(uz), pmax, _ip(r), len(r), _dp(out), nthreads or (os.cpu_count() or 1))
    return r, out.reshape(pmax, len(r))


def structure_functions_np(vel, pmax=10, r=None):
    """Vectorised FP64 restatement of the same sums (for speed on larger grids)."""
    N = vel.shape[1]
    if r is None:
        r = sp_separations(N)
    Sp = np.zeros((pmax, len(r)))
    for m, rr in enumerate(r):
        dux = np.roll(vel[0], -rr, axis=2) - vel[0]
        duy = np.roll(vel[1], -rr, axis=1) - vel[1]
        duz = np.roll(vel[2], -rr, axis=0) - vel[2]
        px = np.ones_like(dux); py = np.ones_like(duy); pz = np.ones_like(duz)
        for p in range(1, pmax + 1):
            px *= dux; py *= duy; pz *= duz
            Sp[p - 1, m] = np.sum(px + py + pz) / N / N / N / 3.0
    return np.asarray(r), Sp


def sp_exponents(rdr, Sp):
    """zeta_p = slope of the degree-1 least-squares fit of log|S_p| against log(r dr) over the
    1-based rows nr-9 .. nr-4 (output/stat/Sp_zeta.m:6-7,18-21); flatness S_4/S_2^2 per row
    (output/stat/Flatness.m:18)."""
    rdr = np.asarray(rdr, dtype=np.float64)
    Sp = np.asarray(Sp, dtype=np.float64)
    nr = len(rdr)
    ie = nr - 4
    rows = slice(ie - 6, ie)
    zeta = np.array([np.polyfit(np.log(rdr[rows]), np.log(np.abs(Sp[p, rows])), 1)[0] for p in range(Sp.shape[0])])
    flat = Sp[3] / Sp[1] ** 2
    return zeta, flat


def field_wh(vor, vel, n_d):
    """Downsampled |omega| and omega.u as REAL(4), Fortran order (tube.f90:1055-1071)."""
    N = vor.shape[1]
    r_d = N // n_d
    s = slice(r_d - 1, N, r_d)
    w = vor[:, s, s, s]
    u = vel[:, s, s, s]
    wm = np.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]).astype(np.float32)
    h = (w[0] * u[0] + w[1] * u[1] + w[2] * u[2]).astype(np.float32)
    return np.stack([wm, h])  # (2, nz, ny, nx) == Fortran (nx, ny, nz, 2)


def vsf_deviation(vor, phi):
    """cal_deviation (subroutine.f90:1519-1546): mean of |omega . grad phi| /
    (|omega| |grad phi| + 1e-11), grad phi by the reference's sixth-order central differences
    on the periodic grid (the ghost layers of wall_phiv, subroutine.f90:1575-1601, are the
    periodic images).  Arrays are [c, z, y, x]."""
    N = phi.shape[0]
    dx = 2.0 * np.pi / N

    def d6(axis):
        f = lambda o: np.roll(phi, -o, axis=axis)
        return (9.0 * f(-2) - f(-3) - 45.0 * f(-1) + 45.0 * f(1) - 9.0 * f(2) + f(3)) / 60.0 / dx

    gx, gy, gz = d6(2), d6(1), d6(0)
    graph = np.sqrt(gx ** 2 + gy ** 2 + gz ** 2)
    vorti = np.sqrt(vor[0] ** 2 + vor[1] ** 2 + vor[2] ** 2)
    dot = vor[0] * gx + vor[1] * gy + vor[2] * gz
    return float(np.sum(np.abs(dot) / (vorti * graph + 1.0e-11)) / N ** 3)


def helicity(vor, vel):
    """cal_helicity of omega and u (subroutine.f90:1550-1569): sum omega . u dv."""
    N = vor.shape[1]
    return cal_helicity(vor, vel, (2.0 * np.pi / N) ** 3)


def dx_dy_dz(phy, d):
    """dx_dy_dz_dp_dm with switch_d = d (1, 2, 3: d/dx, d/dy, d/dz; subroutine.f90:1128-1163):
    forward transform, times i k_d, backward transform, real part."""
    N = phy.shape[0]
    k = 1j * wavenumbers(N)
    spec = fourier_forward(phy)
    if d == 1:
        spec = spec * k[None, None, :]
    elif d == 2:
        spec = spec * k[None, :, None]
    else:
        spec = spec * k[:, None, None]
    return fourier_backward(spec)


def dissipation_field(vel):
    """sum_ij S_ij S_ij with S_ij = (du_i/dx_j + du_j/dx_i) / 2 (subroutine.f90:1086-1126)."""
    dudx = [[dx_dy_dz(vel[i], j + 1) for j in range(3)] for i in range(3)]
    disp = np.zeros_like(vel[0])
    for i in range(3):
        for j in range(3):
            s = 0.5 * (dudx[i][j] + dudx[j][i])
            disp += s * s
    return disp


def field_uw(vor, vel, n_d):
    """Downsampled ux, uy, uz, wx, wy, wz as REAL(4) (tube.f90:1075-1100)."""
    N = vor.shape[1]
    s = slice(N // n_d - 1, N, N // n_d)
    return np.concatenate([vel[:, s, s, s], vor[:, s, s, s]]).astype(np.float32)


def field_wd(vor, vel, n_d):
    """Downsampled |omega| and the dissipation field as REAL(4) (tube.f90:1102-1120)."""
    N = vor.shape[1]
    s = slice(N // n_d - 1, N, N // n_d)
    w = vor[:, s, s, s]
    wm = np.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]).astype(np.float32)
    return np.stack([wm, dissipation_field(vel)[s, s, s].astype(np.float32)])


# ----------------------------------------------------------------------------- pipeline

def run(params: Params, cl: Centerlines, nthreads=None, faithful_spectrum=False, sp_pmax=10):
    """The whole field-construction path of tube.f90:392-1188 in FP64.  Returns a dict."""
    vor, info = deposit(params, cl, nthreads=nthreads)
    out = {"line_info": info}
    out["spectrum_vor"] = spectrum(vor, faithful=faithful_spectrum)
    vel = biot_savart(vor)
    out.update(normalise(vor, vel))
    out["vor"] = vor
    out["vel"] = vel
    out["spectrum"] = spectrum(vel, faithful=faithful_spectrum)
    N = params.N
    out["pdf_u"] = pdf(vel.astype(np.float32).reshape(3 * N, N, N))
    out["pdf_w"] = pdf(vor.astype(np.float32).reshape(3 * N, N, N))
    out["Sp_r"], out["Sp"] = structure_functions(vel, pmax=sp_pmax, nthreads=nthreads)
    out["field_wh"] = field_wh(vor, vel, params.N_downsample)
    return out


# ----------------------------------------------------------------------------- fBb generator

def fbb_circulant_eigs(n, H):
    """Eigenvalues of the 2n circulant embedding of the fGn covariance (Davies-Harte)."""
    k = np.arange(n + 1, dtype=np.float64)
    g = 0.5 * (np.abs(k + 1) ** (2 * H) - 2 * np.abs(k) ** (2 * H) + np.abs(k - 1) ** (2 * H))
    c = np.concatenate([g, g[n - 1:0:-1]])
    lam = np.real(np.fft.fft(c))
    return np.maximum(lam, 0.0)


def fbb_tube(seed, tube, Np, H, dB):
    """One closed fBb centerline (FBB_with_parameters.m:76-120) -> (Np, 3) in [-pi, pi).

    fBm: Davies-Harte circulant embedding (published method, in place of MATLAB's closed
    wfbm) with Philox Gaussians; FP64 prefix sum; bridge f(j); rms-step normalisation to
    dB; uniform random shift; wrap mod 2pi - pi."""
    L = lib()
    M = 128 if Np < 128 else Np
    lam = fbb_circulant_eigs(M, H)
    n2 = 2 * M
    fbm = np.zeros((3, M))
    za = np.zeros(n2); zb = np.zeros(n2)
    for co in range(3):
        L.orc_fbb_gauss(ctypes.c_uint64(seed), tube, co, n2, _dp(za), _dp(zb))
        w = np.fft.fft(np.sqrt(lam / n2) * (za + 1j * zb))
        x = np.real(w[:M])
        fbm[co] = np.cumsum(x)
    if Np < 128:
        r_t = 128 // Np
        idx = np.ceil(np.arange(1, Np + 1) * r_t).astype(np.int64) - 1
        fbm = fbm[:, idx]
    j = np.arange(1, Np + 1, dtype=np.float64)
    f = 0.5 * ((j / Np) ** (2.0 * H) + 1 - (1.0 - j / Np) ** (2.0 * H))
    bb = fbm - f[None, :] * fbm[:, Np - 1:Np]
    d = np.diff(bb, axis=1)
    rms = float(np.sum(d * d / (Np - 1)))
    bb = bb * dB / np.sqrt(rms)
    for co in range(3):
        bb[co] = bb[co] + (L.orc_fbb_shift(ctypes.c_uint64(seed), tube, co) - 0.5) * 2 * PI
    bbp = np.mod(bb, 2 * PI) - PI
    return bbp.T.copy()


def fbb_sign(seed, tube):
    return lib().orc_fbb_sign(ctypes.c_uint64(seed), tube)


def philox_raw(ctr, key):
    """Philox4x32-10 block function on a 4-word counter and 2-word key (for KAT vectors)."""
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    lib().orc_philox_raw(c.ctypes.data_as(u32p), k.ctypes.data_as(u32p), out.ctypes.data_as(u32p))
    return out


# ----------------------------------------------------------------------------- isosurface

_TET_AXES = [(1, 2), (1, 4), (2, 1), (2, 4), (4, 1), (4, 2)]


def isosurface_iso(box_v):
    """output/field_wh_norm.py:71-73: iso_w = sqrt(mean(|omega|^2)) * 3 / sqrt(2)."""
    v = box_v.astype(np.float64)
    return np.float32(np.sqrt(np.sum(v * v) / v.size) * 3.0 / np.sqrt(2.0))


def isosurface(box_v, box_h, iso):
    """Marching tetrahedra on the field_wh box (arrays [k, j, i], float32), the restatement of
    the library's extraction: six tetrahedra per cube around the 0-7 diagonal, a vertex inside
    when its value exceeds iso, crossings interpolated from the edge's lower corner, triangles
    wound from inside to outside, in cube order (x fastest), then tetrahedron, then triangle.
    Every float32 operation is rounded on its own, as on the device.  Returns (T, 3, 4)
    vertices (x, y, z, helicity) at x_i = 2 pi i / (n - 1)."""
    f32 = np.float32
    n = box_v.shape[0]
    m1 = n - 1
    iso = f32(iso)
    step = f32(2.0 * np.pi / (n - 1))
    k, j, i = np.meshgrid(np.arange(m1), np.arange(m1), np.arange(m1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    q = i + m1 * (j + m1 * k)
    corner = lambda c: (k + ((c >> 2) & 1), j + ((c >> 1) & 1), i + (c & 1))
    val = [box_v[corner(c)].astype(f32) for c in range(8)]
    hel = [box_h[corner(c)].astype(f32) for c in range(8)]
    pos = [np.stack([(i + (c & 1)).astype(f32), (j + ((c >> 1) & 1)).astype(f32),
                     (k + ((c >> 2) & 1)).astype(f32)], axis=1) for c in range(8)]
    inside = [val[c] > iso for c in range(8)]

    def crossing(sel, a, b):
        if a > b:
            a, b = b, a
        va, vb = val[a][sel], val[b][sel]
        t = ((iso - va) / (vb - va)).astype(f32)
        xa, xb = pos[a][sel], pos[b][sel]
        p = ((xa + t[:, None] * (xb - xa)) * step).astype(f32)
        ha, hb = hel[a][sel], hel[b][sel]
        h = (ha + t * (hb - ha)).astype(f32)
        return np.concatenate([p, h[:, None]], axis=1)

    def wind(p, r, s, d):
        e1, e2 = r[:, :3] - p[:, :3], s[:, :3] - p[:, :3]
        nx = e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1]
        ny = e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2]
        nz = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]
        dot = (nx * d[0] + ny * d[1]) + nz * d[2]
        flip = (dot < f32(0.0))[:, None]
        return np.stack([p, np.where(flip, s, r), np.where(flip, r, s)], axis=1)

    tris, keys = [], []
    for tt, (a, b) in enumerate(_TET_AXES):
        cs = [0, a, a | b, 7]
        for mask in range(1, 15):
            ins = [c for s, c in enumerate(cs) if (mask >> s) & 1]
            outs = [c for s, c in enumerate(cs) if not (mask >> s) & 1]
            sel = np.ones(q.size, dtype=bool)
            for s, c in enumerate(cs):
                sel &= inside[c] == bool((mask >> s) & 1)
            if not sel.any():
                continue
            d = [f32(f32(sum((c >> ax) & 1 for c in outs)) / f32(len(outs)))
                 - f32(f32(sum((c >> ax) & 1 for c in ins)) / f32(len(ins))) for ax in range(3)]
            d = [f32(x) for x in d]
            if len(ins) == 1 or len(outs) == 1:
                lone = ins[0] if len(ins) == 1 else outs[0]
                oth = outs if len(ins) == 1 else ins
                p = [crossing(sel, lone, o) for o in oth]
                tris.append(wind(p[0], p[1], p[2], d))
                keys.append(np.stack([q[sel], np.full(sel.sum(), tt), np.zeros(sel.sum(), dtype=np.int64)], 1))
            else:
                p0 = crossing(sel, ins[0], outs[0])
                p1 = crossing(sel, ins[0], outs[1])
                p2 = crossing(sel, ins[1], outs[1])
                p3 = crossing(sel, ins[1], outs[0])
                tris.append(wind(p0, p1, p2, d))
                keys.append(np.stack([q[sel], np.full(sel.sum(), tt), np.zeros(sel.sum(), dtype=np.int64)], 1))
                tris.append(wind(p0, p2, p3, d))
                keys.append(np.stack([q[sel], np.full(sel.sum(), tt), np.ones(sel.sum(), dtype=np.int64)], 1))
    if not tris:
        return np.zeros((0, 3, 4), dtype=f32)
    tris = np.concatenate(tris)
    keys = np.concatenate(keys)
    order = np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))
    return tris[order]
