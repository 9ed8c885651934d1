"""Known-answer tests that pin the FP64 oracle (CPU only).

The reference ships no tests and no golden outputs, so the oracle is pinned by answers that
follow from the mathematics of each step: a straight periodic tube gives the analytic
truncated Gaussian core of the deposition formula; the quintic Hermite spline reproduces the
nodes and their derivatives; Biot-Savart gives a divergence-free u whose curl is omega's
solenoidal part; the shell spectrum obeys Parseval; normalisation gives E/u'^2 = 3/2; the PDF
bins agree with a literal first-match search and integrate to one; S_p of a single Fourier
mode is analytic; the random stream reproduces the published Philox4x32-10 vectors; the
fractional-Brownian-bridge increments scale as r^{2H}.
"""
import numpy as np
import pytest

PI = np.pi


# ----------------------------------------------------------------------------- random stream

def test_philox_kat_vectors(orc):
    """Philox4x32-10 known-answer vectors published with Random123 (Salmon et al., SC'11)."""
    kats = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for ctr, key, want in kats:
        assert list(orc.philox_raw(ctr, key)) == want


def test_fbb_gaussians_are_standard_normal(orc):
    import ctypes
    n = 1 << 16
    za = np.zeros(n)
    zb = np.zeros(n)
    orc.lib().orc_fbb_gauss(ctypes.c_uint64(7), 3, 1, n, orc._dp(za), orc._dp(zb))
    z = np.concatenate([za, zb])
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1.0) < 0.01
    assert abs(np.mean(z ** 4) - 3.0) < 0.06


def test_fbb_increments_scale_as_r_to_2H(orc):
    """S2(r) = <|x(j+r) - x(j)|^2> grows as r^{2H} (the reference's own generator check,
    FBB_with_parameters.m:150-166), with S2(1) = dB^2 by the rms normalisation."""
    H, dB, Np = 0.7, 0.05, 1024
    r = np.arange(1, 17)
    S2 = np.zeros(len(r))
    ntubes = 24
    for t in range(ntubes):
        x = orc.fbb_tube(11, t, Np, H, dB)
        for m, rr in enumerate(r):
            d = x[rr:] - x[:-rr]
            d = (d + PI) % (2 * PI) - PI            # minimum image of the wrapped coordinates
            S2[m] += np.mean(np.sum(d * d, axis=1)) / ntubes
    slope = np.polyfit(np.log(r), np.log(S2), 1)[0]
    assert abs(slope - 2 * H) < 0.08, slope
    assert abs(S2[0] / dB ** 2 - 1.0) < 0.05


def test_fbb_tube_is_wrapped_and_closed(orc):
    x = orc.fbb_tube(5, 0, 256, 0.6, 0.1)
    assert x.shape == (256, 3)
    assert np.all(x >= -PI) and np.all(x < PI)
    # the bridge closes the line: the last-to-first step is of the size of the others
    steps = np.diff(np.vstack([x, x[:1]]), axis=0)
    steps = (steps + PI) % (2 * PI) - PI
    n = np.linalg.norm(steps, axis=1)
    assert n[-1] < 5 * np.sqrt(np.mean(n[:-1] ** 2))


# ----------------------------------------------------------------------------- splines

def _poly(c, z):
    return sum(c[i] * z ** i for i in range(6))


def _dpoly(c, z):
    return sum(i * c[i] * z ** (i - 1) for i in range(1, 6))


def _d2poly(c, z):
    return sum(i * (i - 1) * c[i] * z ** (i - 2) for i in range(2, 6))


def test_spline_reproduces_nodes_and_derivatives(orc):
    """Section i of get_spline_5th_coe (subroutine.f90:440-461) interpolates node i at zeta=0
    and node i+1 (unwrapped) at the section length, with the central-difference c' and c''
    of tube.f90:470-515 at both ends."""
    xyz = orc.fbb_tube(3, 1, 64, 0.7, 0.2)
    n = xyz.shape[0]
    cze, ck, ckk, L = orc.line_prep(xyz)
    ntf, dtf, coe, L2 = orc.line_ntf(xyz)
    assert L == pytest.approx(L2, rel=1e-15)
    cze_pl = np.concatenate([cze, [2 * PI]])
    for i in range(n):
        j = (i + 1) % n
        zr = cze_pl[i + 1] * L - cze_pl[i] * L
        for d in range(3):
            c = coe[i, d]
            assert _poly(c, 0.0) == pytest.approx(xyz[i, d], abs=1e-13)
            right = _poly(c, zr)
            step = (xyz[j, d] - xyz[i, d] + PI) % (2 * PI) - PI   # the unwrapped right end
            assert right == pytest.approx(xyz[i, d] + step, abs=1e-11)
            assert _dpoly(c, 0.0) == pytest.approx(ck[d, i], abs=1e-12)
            assert _dpoly(c, zr) == pytest.approx(ck[d, j], rel=1e-9, abs=1e-10)
            assert _d2poly(c, 0.0) == pytest.approx(ckk[d, i], abs=1e-12)
            assert _d2poly(c, zr) == pytest.approx(ckk[d, j], rel=1e-8, abs=1e-8)
    # the periodic arc length runs over [0, 2 pi) and Len_Disc = length / 2 pi
    assert cze[0] == 0.0 and np.all(np.diff(cze) > 0) and cze[-1] < 2 * PI


def test_ntf_of_a_straight_line_is_one(orc):
    n = 32
    xyz = np.zeros((n, 3))
    xyz[:, 0] = -PI + 2 * PI * np.arange(n) / n
    xyz[:, 1] = 0.3
    xyz[:, 2] = -0.2
    ntf = orc.line_ntf(xyz)[0]
    assert np.all(ntf == 1)


def test_ntf_of_a_circle(orc):
    """A planar circle turns by 2 pi in total: sum over sections of ntf_times*theta/2pi = 50,
    so each of n sections gets ceil(50/n)+1 sub-segments."""
    n, R = 40, 1.0
    a = 2 * PI * np.arange(n) / n
    xyz = np.stack([R * np.cos(a), R * np.sin(a), np.full(n, 0.1)], axis=1)
    ntf = orc.line_ntf(xyz, ntf_times=50, ntf_pre=1000)[0]
    # per-section theta is 2 pi/n to within the central-difference error of c', c''
    assert np.all(np.abs(ntf[:n] - (np.ceil(50 / n) + 1)) <= 1)


# ----------------------------------------------------------------------------- deposition

def _straight_tube(N, sigma, Gamma, y0, z0, n=48, axis=0):
    from oracle.oracle import Centerlines, Params
    xyz = np.zeros((n, 3))
    xyz[:, axis] = -PI + 2 * PI * np.arange(n) / n
    others = [d for d in range(3) if d != axis]
    xyz[:, others[0]] = y0
    xyz[:, others[1]] = z0
    p = Params(N=N, N_downsample=N, line_s=1, line_e=1, sigma_ratio=1.0, sigma=np.array([sigma]),
               Gamma=np.array([Gamma]), n_T=np.array([1], dtype=np.int32), if_filter=np.zeros(1, dtype=np.int32))
    return p, Centerlines(npoint=np.array([n]), xyz=xyz)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_straight_tube_is_the_truncated_gaussian_core(orc, axis):
    """A straight periodic tube deposits, by the straight branch of tube.f90:854-866,
    omega = Gamma [exp(-rho^2/2s^2) - exp(-R^2/2s^2)]/(2 pi s^2) T for rho < R = 3 s,
    every grid point once."""
    N, sigma, Gamma = 32, 0.21, 1.7
    y0, z0 = 0.1234, -0.377
    p, cl = _straight_tube(N, sigma, Gamma, y0, z0, axis=axis)
    cond = np.zeros((N, N, N))
    vor, _ = orc.deposit(p, cl, nthreads=2, cond=cond)
    assert set(np.unique(cond)) <= {0.0, 1.0}          # the straight branch amplifies nothing
    x = -PI + 2 * PI * np.arange(N) / N
    R = 3.0 * sigma
    d1 = (x - y0 + PI) % (2 * PI) - PI
    d2 = (x - z0 + PI) % (2 * PI) - PI
    rho2 = d1[:, None] ** 2 + d2[None, :] ** 2          # [other0, other1]
    tp = (np.exp(-rho2 / (2 * sigma ** 2)) - np.exp(-R ** 2 / (2 * sigma ** 2))) / (2 * PI * sigma ** 2)
    tp[rho2 >= R * R] = 0.0
    # field arrays are [k(z), j(y), i(x)]
    if axis == 0:
        want = np.broadcast_to(tp.T[:, :, None], (N, N, N))      # [z, y] = tp[y, z].T
    elif axis == 1:
        want = np.broadcast_to(tp.T[:, None, :], (N, N, N))      # others: x, z -> [z, x]
    else:
        want = np.broadcast_to(tp.T[None, :, :], (N, N, N))      # others: x, y -> [y, x]
    got = vor[axis] / Gamma
    np.testing.assert_allclose(got, want, atol=1e-12)
    for d in range(3):
        if d != axis:
            assert np.max(np.abs(vor[d])) < 1e-12


def test_deposit_is_linear_in_gamma_and_additive(orc):
    from helpers import two_tubes
    p, cl = two_tubes(orc)
    v_all, _ = orc.deposit(p, cl, nthreads=2)
    v1, _ = orc.deposit(p, cl, nthreads=2, line_s=1, line_e=1)
    v2, _ = orc.deposit(p, cl, nthreads=2, line_s=2, line_e=2)
    np.testing.assert_allclose(v_all, v1 + v2, atol=1e-12)
    p.Gamma = p.Gamma * -2.5
    v_neg, _ = orc.deposit(p, cl, nthreads=2)
    np.testing.assert_allclose(v_neg, -2.5 * v_all, rtol=1e-12, atol=1e-12)


def test_deposit_threads_agree_bitwise(orc):
    """The OpenMP z-slab ownership gives the same sums for any thread count."""
    from helpers import two_tubes
    p, cl = two_tubes(orc)
    a, _ = orc.deposit(p, cl, nthreads=1)
    b, _ = orc.deposit(p, cl, nthreads=4)
    assert np.array_equal(a, b)


# ----------------------------------------------------------------------------- spectral

def _random_field(N, seed, kmax=None):
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((3, N, N, N))
    if kmax is not None:
        from oracle.oracle import fourier_backward, fourier_forward, k2_grid
        m = k2_grid(N) > kmax ** 2
        for c in range(3):
            s = fourier_forward(f[c])
            s[m] = 0
            f[c] = fourier_backward(s)
    return f


def test_biot_savart_divergence_free_and_curl(orc):
    N = 16
    w = _random_field(N, 1)
    u = orc.biot_savart(w)
    k = orc.wavenumbers(N)
    kz, ky, kx = k[:, None, None], k[None, :, None], k[None, None, :]
    U = [orc.fourier_forward(u[c]) for c in range(3)]
    W = [orc.fourier_forward(w[c]) for c in range(3)]
    # the Nyquist planes are not resolved by a centred difference; test the interior modes
    inner = (np.abs(kx) < N // 2) & (np.abs(ky) < N // 2) & (np.abs(kz) < N // 2)
    div = kx * U[0] + ky * U[1] + kz * U[2]
    assert np.max(np.abs(div[inner])) < 1e-13
    cx = 1j * (ky * U[2] - kz * U[1])
    cy = 1j * (kz * U[0] - kx * U[2])
    cz = 1j * (kx * U[1] - ky * U[0])
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    k2s = np.where(k2 == 0, 1.0, k2)
    kw = (kx * W[0] + ky * W[1] + kz * W[2]) / k2s
    Pw = [W[0] - kx * kw, W[1] - ky * kw, W[2] - kz * kw]   # solenoidal part of omega
    for c_got, c_want in zip((cx, cy, cz), Pw):
        m = inner & (k2 > 0)
        assert np.max(np.abs(c_got[m] - c_want[m])) < 1e-12


def test_spectrum_parseval(orc):
    """Sum over shells of E(k) equals <|f|^2>/2 for a zero-mean field band-limited inside
    shell N/2 (shell 0, the mean, is not part of the spectrum)."""
    N = 16
    f = _random_field(N, 2, kmax=N // 2 - 1)
    f -= f.mean(axis=(1, 2, 3), keepdims=True)
    E = orc.spectrum(f)
    assert len(E) == N // 2
    energy = 0.5 * np.mean(np.sum(f * f, axis=0))
    assert np.sum(E) == pytest.approx(energy, rel=1e-12)
    Ef = orc.spectrum(f, faithful=True)
    assert np.sum(Ef.astype(np.float64)) == pytest.approx(energy, rel=1e-5)


def test_spectrum_single_mode(orc):
    """u = (cos(3y), 0, 0) puts E = 1/4 in shell 3 and nothing elsewhere."""
    N = 16
    x = -PI + 2 * PI * np.arange(N) / N
    u = np.zeros((3, N, N, N))
    u[0] = np.cos(3 * x)[None, :, None]
    E = orc.spectrum(u)
    want = np.zeros(N // 2)
    want[2] = 0.25
    np.testing.assert_allclose(E, want, atol=1e-15)


def test_normalised_energy_is_three_halves(orc):
    N = 16
    w = _random_field(N, 3)
    u = orc.biot_savart(w)
    s = orc.normalise(w, u)
    dv = (2 * PI / N) ** 3
    E_after = orc.cal_helicity(u, u, dv) / 2 / (2 * PI) ** 3
    assert E_after == pytest.approx(1.5, rel=1e-13)
    assert s["Etot"] / s["up"] ** 2 == pytest.approx(1.5, rel=1e-13)


def test_filter_spec_is_a_sharp_cutoff(orc):
    N = 16
    w = _random_field(N, 4)
    orc.filter_spec(3, w)
    k2 = orc.k2_grid(N)
    for c in range(3):
        s = orc.fourier_forward(w[c])
        assert np.max(np.abs(s[k2 > 9])) < 1e-14
        assert np.max(np.abs(s[k2 <= 9])) > 1e-3


# ----------------------------------------------------------------------------- statistics

def _literal_cal_pdf(v, nbins):
    """subroutine.f90:12-34 as written: REAL(4) edges, then for each value the first bin
    l = 1..bin_num with lo(l) <= v < hi(l)."""
    vmin, vmax = np.float32(v.min()), np.float32(v.max())
    bsz = np.float32(np.float32(vmax - vmin) / np.float32(nbins))
    counts = np.zeros(nbins, dtype=np.int64)
    val = np.zeros(nbins, dtype=np.float32)
    for l in range(nbins):
        val[l] = np.float32(np.float64(vmin) + 0.5 * np.float64(bsz) + np.float64(np.float32(np.float32(l) * bsz)))
    half = np.float32(np.float32(0.5) * bsz)
    lo = (val - half).astype(np.float32)
    hi = (val + half).astype(np.float32)
    for x in v:
        for l in range(nbins):
            if lo[l] <= x < hi[l]:
                counts[l] += 1
                break
    return val, counts


@pytest.mark.parametrize("nbins", [1, 7, 50])
def test_pdf_bins_match_a_literal_first_match_search(orc, nbins):
    rng = np.random.default_rng(nbins)
    v = rng.standard_normal(3000).astype(np.float32)
    # values exactly on edges, the extremes, and repeats
    _, lo, hi, _ = orc.pdf_edges(v.min(), v.max(), nbins)
    v = np.concatenate([v, lo[: min(5, nbins)], hi[: min(5, nbins)], [v.max()] * 3, [v.min()] * 2]).astype(np.float32)
    val_ref, c_ref = _literal_cal_pdf(v, nbins)
    val, p, c = orc.pdf(v.reshape(1, 1, -1), nbins=nbins)
    assert np.array_equal(c, c_ref)
    assert np.array_equal(val, val_ref)


def test_pdf_integrates_to_one(orc):
    rng = np.random.default_rng(5)
    d = rng.standard_normal((12, 16, 16)).astype(np.float32)
    val, p, c = orc.pdf(d, nbins=1000)
    bsz = float(val[1] - val[0])
    # the maximum can fall outside the last half-open bin; everything else is counted
    assert d.size - 2 <= int(c.sum()) <= d.size
    assert float(np.sum(p.astype(np.float64)) * bsz) == pytest.approx(1.0, abs=2e-3)


def test_pdf_of_gaussian_data_matches_the_reference_gaussian_table(orc):
    """output/stat/pdf_um_gau.dat (fixture: every 50th row) is the standard normal density;
    the oracle's PDF of seeded N(0,1) samples follows it within sampling error."""
    import os
    tab = np.load(os.path.join(os.path.dirname(__file__), "golden", "gaussian_pdf_table.npz"))["table"]
    x, g = tab[:, 0], tab[:, 1]
    np.testing.assert_allclose(g, np.exp(-x * x / 2) / np.sqrt(2 * PI), rtol=1e-4, atol=1e-9)
    rng = np.random.default_rng(6)
    d = rng.standard_normal((64, 64, 64)).astype(np.float32)
    val, p, c = orc.pdf(d, nbins=100)
    gi = np.interp(val, x, g)
    core = np.abs(val) < 2.5
    err = np.abs(p[core] - gi[core]) / np.sqrt(gi[core] / (d.size * float(val[1] - val[0])))
    assert np.max(err) < 6.0        # within six standard errors of a bin count


def test_sp_separations_follow_sqrt2_powers(orc):
    assert list(orc.sp_separations(64)) == [1, 1, 2, 3, 4, 6, 8, 11, 16, 23, 32, 45, 64]
    assert len(orc.sp_separations(256)) == 17
    assert len(orc.sp_separations(1024)) == 21
    assert orc.sp_separations(256)[-1] == 256


def test_structure_functions_of_a_single_mode(orc):
    """u = (sin x, 0, 0): du_x(r) = sin(x+h) - sin(x) with h = r dx gives
    S_1 = 0, S_2 = (1 - cos h)/3, S_4 = (3/2)(1 - cos h)^2/3, odd orders 0."""
    N = 32
    x = -PI + 2 * PI * np.arange(N) / N
    u = np.zeros((3, N, N, N))
    u[0] = np.sin(x)[None, None, :]
    r = np.array([1, 2, 3, 5, 8], dtype=np.int32)
    rr, Sp = orc.structure_functions(u, pmax=4, r=r, nthreads=2)
    h = r * 2 * PI / N
    a = 1 - np.cos(h)
    np.testing.assert_allclose(Sp[0], 0.0, atol=1e-15)
    np.testing.assert_allclose(Sp[1], a / 3.0, rtol=1e-12)
    np.testing.assert_allclose(Sp[2], 0.0, atol=1e-14)
    np.testing.assert_allclose(Sp[3], 1.5 * a ** 2 / 3.0, rtol=1e-12)
    rr2, Sp2 = orc.structure_functions_np(u, pmax=4, r=r)
    np.testing.assert_allclose(Sp2, Sp, rtol=1e-12, atol=1e-15)


def test_field_wh_picks_every_rd_th_point(orc):
    N, nd = 16, 4
    rng = np.random.default_rng(7)
    w = rng.standard_normal((3, N, N, N))
    u = rng.standard_normal((3, N, N, N))
    out = orc.field_wh(w, u, nd)
    assert out.shape == (2, nd, nd, nd) and out.dtype == np.float32
    # Fortran sample index i*r_d (1-based) is 0-based i*r_d - 1
    i = 2 * (N // nd) - 1
    assert out[0, 0, 1, 1] == np.float32(np.sqrt(np.sum(w[:, N // nd - 1, i, i] ** 2)))


# ----------------------------------------------------------------------------- surrogate oracle

def test_mlp_oracle_gradients_by_finite_differences():
    """The FP64 network's backward pass against central differences of its loss."""
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(4)
    widths = [5, 16, 16, 7]
    n = sum(k * m + m for k, m in zip(widths[:-1], widths[1:]))
    p = rng.normal(0, 0.5, n)
    X = rng.uniform(-1, 1, (9, 5))
    T = rng.normal(0, 1, (9, 7))
    w = rng.uniform(0.5, 2, 7)
    loss, gp, gx = MO.loss_grad(p, widths, X, T, w, bf16_ops=False)
    h = 1e-6
    for i in rng.choice(n, 25, replace=False):
        e = np.zeros(n)
        e[i] = h
        fd = (MO.loss_grad(p + e, widths, X, T, w, False)[0] - MO.loss_grad(p - e, widths, X, T, w, False)[0]) / (2 * h)
        assert gp[i] == pytest.approx(fd, rel=1e-5, abs=1e-9)
    for (r, c) in [(0, 0), (3, 2), (8, 4)]:
        E = np.zeros_like(X)
        E[r, c] = h
        fd = (MO.loss_grad(p, widths, X + E, T, w, False)[0] - MO.loss_grad(p, widths, X - E, T, w, False)[0]) / (2 * h)
        assert gx[r, c] == pytest.approx(fd, rel=1e-5, abs=1e-9)


def test_bf16_rounding_is_round_to_nearest_even():
    from oracle import mlp_oracle as MO
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 3.0e38], dtype=np.float32)
    r = MO.bf16(x)
    assert list(r[:5]) == [1.0, 1.0, 1.0 + 2 ** -7, 1.0, -2.5]


def test_dissipation_of_a_shear_and_a_strain(orc):
    """dissipation_field (subroutine.f90:1086-1126) on fields with known strain: the shear
    u = (sin y, 0, 0) has S_12 = S_21 = cos(y)/2, so S_ij S_ij = cos(y)^2 / 2; the strain
    u = (sin x cos y, -cos x sin y, 0) has S_11 = -S_22 = cos x cos y and S_12 = 0, so
    S_ij S_ij = 2 cos^2 x cos^2 y."""
    N = 16
    x = np.arange(N) * 2 * np.pi / N - np.pi
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")          # [k, j, i]
    vel = np.stack([np.sin(Y), np.zeros_like(Y), np.zeros_like(Y)])
    assert np.allclose(orc.dissipation_field(vel), 0.5 * np.cos(Y) ** 2, atol=1e-12)
    vel = np.stack([np.sin(X) * np.cos(Y), -np.cos(X) * np.sin(Y), np.zeros_like(X)])
    assert np.allclose(orc.dissipation_field(vel), 2.0 * np.cos(X) ** 2 * np.cos(Y) ** 2, atol=1e-12)
    assert np.allclose(orc.dx_dy_dz(np.sin(2 * X), 1), 2 * np.cos(2 * X), atol=1e-12)


def test_vsf_deviation_and_helicity_known_answers(orc):
    """cal_deviation (subroutine.f90:1519-1546): omega along x with phi independent of x gives
    omega . grad phi = 0, deviation ~0; omega along x with phi = sin(x + 0.3) gives |omega . grad
    phi| = |omega| |grad phi|, deviation 1 (up to the 1e-11 guard).  The sixth-order stencil
    differentiates sin to O(dx^6).  cal_helicity: omega = u = (1, 0, 0) gives (2 pi)^3."""
    N = 32
    x = np.arange(N) * 2 * np.pi / N - np.pi
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    vor = np.stack([1.0 + 0.5 * np.cos(Y) * np.sin(Z), np.zeros_like(X), np.zeros_like(X)])
    # rounding leaves |d phi/dx| ~ 1e-16; where grad phi vanishes too (the extrema of phi) the
    # 1e-11 guard bounds such points' ratios by ~1e-5
    assert orc.vsf_deviation(vor, np.exp(np.cos(Y) + np.sin(2 * Z))) < 1e-6
    vor = np.stack([np.ones_like(X), np.zeros_like(X), np.zeros_like(X)])
    assert orc.vsf_deviation(vor, np.sin(X + 0.3)) == pytest.approx(1.0, abs=1e-8)
    # an oblique case: omega = (1, 1, 0) / sqrt2, phi = sin(x + 0.3): |cos| / sqrt2 / |cos| = 1/sqrt2
    vor = np.stack([np.ones_like(X), np.ones_like(X), np.zeros_like(X)]) / np.sqrt(2.0)
    assert orc.vsf_deviation(vor, np.sin(X + 0.3)) == pytest.approx(1.0 / np.sqrt(2.0), abs=1e-8)
    vel = np.stack([np.ones_like(X), np.zeros_like(X), np.zeros_like(X)])
    assert orc.helicity(vel, vel) == pytest.approx((2 * np.pi) ** 3, rel=1e-14)


def test_isosurface_of_a_sphere_is_closed_and_outward(orc):
    """Marching tetrahedra (the contour step of output/field_wh_norm.py:81) on a radial field:
    every vertex near the iso-radius, every edge shared by exactly two triangles (a closed
    surface), every normal pointing outward (to decreasing values), area close to 4 pi R^2, and
    the helicity scalar interpolated linearly (h = x gives the vertex x)."""
    n = 33
    x = np.linspace(0.0, 2 * np.pi, n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    c = np.pi
    r2 = (X - c) ** 2 + (Y - c) ** 2 + (Z - c) ** 2
    v = np.exp(-r2).astype(np.float32)
    R = 1.7
    iso = np.float32(np.exp(-R * R))
    tris = orc.isosurface(v, X.astype(np.float32), iso)
    assert tris.shape[1:] == (3, 4) and len(tris) > 500
    p = tris[:, :, :3].astype(np.float64)
    rad = np.linalg.norm(p - c, axis=2)
    assert np.abs(rad - R).max() < 0.05
    np.testing.assert_allclose(tris[:, :, 3], tris[:, :, 0], rtol=1e-5, atol=1e-5)
    e1, e2 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
    nrm = np.cross(e1, e2)
    area = 0.5 * np.linalg.norm(nrm, axis=1)
    cen = p.mean(axis=1) - c
    keep = area > 1e-9
    assert np.all(np.einsum("ij,ij->i", nrm[keep], cen[keep]) > 0)
    assert area.sum() == pytest.approx(4 * np.pi * R * R, rel=0.02)
    # closed: each undirected edge (by exact vertex coordinates) appears in two triangles
    from collections import Counter
    key = lambda a: tuple(np.round(a, 6))
    edges = Counter()
    for t in p:
        for s in range(3):
            a, b = key(t[s]), key(t[(s + 1) % 3])
            if a != b:
                edges[tuple(sorted((a, b)))] += 1
    assert set(edges.values()) == {2}
    assert orc.isosurface_iso(v) == pytest.approx(np.sqrt(np.mean(v.astype(np.float64) ** 2)) * 3 / np.sqrt(2),
                                                  rel=1e-6)


def test_fp64_floor_is_a_rounding_effect(orc):
    """The oracle's plain and FMA-contracted builds (helpers.fp64_floor) compute the same algorithm
    in the same order; their fields differ (the reference's zeta interpolation amplifies ulp-level
    changes) but only at the level of FP64 rounding, far below the FP32 tolerance.  This distance
    sets the FP64 tolerance of the GPU parity tests."""
    from fastweavturb_b200.configs import small
    from helpers import fp64_floor, oracle_inputs

    if not orc.has_fma():
        pytest.skip("no FMA on this host")
    w = small(N=32, seed=3, nlev=2, tubes0=2, nodes0=64, sigma0=0.4)
    p, cl = oracle_inputs(orc, w)
    floor, vor = fp64_floor(orc, p, cl)
    assert np.abs(vor).max() > 0
    assert 0.0 < floor < 1e-10
