"""Parity of the CUDA path (through the C-ABI) against the FP64 oracle on seeded inputs.

Tolerances: FP32 path <= 1e-5 relative L2 for omega, u and E(k); FP64 path within four times
the reference algorithm's own FP64 rounding floor on the same workload (helpers.fp64_floor,
the distance between the oracle's plain and FMA-contracted builds) and never below 1e-12.
Integer outputs (sub-segment counts, histogram counts given the same data) are bit-exact.
"""
import numpy as np
import pytest

from helpers import fp64_floor, gpu_params, oracle_inputs, rel_l2, tol64

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


@pytest.fixture(scope="module")
def small_case(orc):
    from fastweavturb_b200.configs import small

    w = small(N=32, seed=3, nlev=2, tubes0=2, nodes0=64, sigma0=0.4)
    p, cl = oracle_inputs(orc, w)
    ref = orc.run(p, cl)
    ref["tol64"] = tol64(fp64_floor(orc, p, cl)[0])
    return w, p, cl, ref


def _gpu_run(F, w, cl, p, precision, mode):
    ctx = F.Context(gpu_params(F, w, precision=precision, deposit_mode=mode))
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    ctx.run()
    return ctx


@pytest.mark.parametrize("precision,mode", [(32, 0), (32, 1), (64, 1), (64, 0)])
def test_fields_match_oracle(fwt, small_case, precision, mode):
    w, p, cl, ref = small_case
    tol = TOL32 if precision == 32 else ref["tol64"]
    ctx = _gpu_run(fwt, w, cl, p, precision, mode)
    vor = ctx.field(0)
    vel = ctx.field(1)
    e_w = rel_l2(vor, ref["vor"])
    e_u = rel_l2(vel, ref["vel"])
    assert e_w <= tol, f"omega rel L2 {e_w:.3e}"
    assert e_u <= tol, f"u rel L2 {e_u:.3e}"
    norm = ctx.cal_helicity()
    assert abs(norm["up"] - ref["up"]) <= tol * ref["up"]
    assert abs(norm["Enstrophy"] - ref["Enstrophy"]) <= tol * ref["Enstrophy"]
    ew = ctx.spectrum(0)
    eu = ctx.spectrum(1)
    assert rel_l2(ew, ref["spectrum_vor"]) <= tol
    assert rel_l2(eu, ref["spectrum"]) <= tol
    ctx.close()


def test_ntf_bit_exact(fwt, orc, small_case):
    """Sub-segment counts per section come out of FP64 presampling and must match exactly."""
    w, p, cl, ref = small_case
    ctx = _gpu_run(fwt, w, cl, p, 32, 0)
    c = ctx.counters()
    total = 0
    for i in range(len(cl.npoint)):
        ntf, _, _, _ = orc.line_ntf(cl.line(i), p.ntf_times, p.ntf_pre)
        total += int(ntf[:-1].sum())
    assert c["subsegments"] == total
    ctx.close()


def test_generator_matches_oracle(fwt, orc):
    import torch

    from fastweavturb_b200.configs import build_workload, small

    w = small(N=32, seed=11, nlev=2, tubes0=2, nodes0=64)
    ctx = fwt.Context(gpu_params(fwt, w))
    xyz, arrs = build_workload(ctx, w)
    g = xyz.cpu().numpy().T
    p, cl = oracle_inputs(orc, w)
    d = np.abs(g - cl.xyz)
    d = np.minimum(d, 2 * np.pi - d)   # coordinates live on the periodic box
    assert d.max() < 1e-9, d.max()
    assert np.array_equal(arrs[2], p.Gamma)
    ctx.close()
    del xyz
    torch.cuda.synchronize()


@pytest.mark.parametrize("H,dB_over_sigma", [(0.3, 10.0), (0.7, 10.0), (0.8, 40.0), (0.5, 3.0)])
def test_ntf_bit_exact_across_curvatures(fwt, orc, H, dB_over_sigma):
    """The sub-segment count of every section, ceil(ntf_times theta / 2 pi) + 1, decided by the
    quadrature estimate of the turning angle or its fallbacks, equals the oracle's FP64 sum
    over the reference's ntf_pre + 1 samples, for rough and smooth lines alike."""
    from fastweavturb_b200.configs import Level, Workload

    lv = [Level(tubes=6, nodes=256, sigma=0.1, Gamma=1.0, H=H, dB=dB_over_sigma * 0.1),
          Level(tubes=6, nodes=512, sigma=0.05, Gamma=0.5, H=H, dB=dB_over_sigma * 0.05)]
    w = Workload("ntf", 64, lv, seed=21)
    p, cl = oracle_inputs(orc, w)
    ctx = fwt.Context(gpu_params(fwt, w))
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    ctx.deposit()
    total = sum(int(orc.line_ntf(cl.line(i), p.ntf_times, p.ntf_pre)[0][:-1].sum()) for i in range(len(cl.npoint)))
    assert ctx.counters()["subsegments"] == total
    ctx.close()


@pytest.mark.parametrize("precision", [32, 64])
def test_rasterised_pieces_equal_searched_pieces(fwt, orc, precision):
    """Thin tubes (truncation radius 0.6-1.2 grid spacings on 64^3): the pieces rasterised once
    (radius limit 4 grid spacings) and the pieces searched in every tile (limit 0) accept the same
    points with the same test, so the FP32 fields are identical (int64 fixed-point sums) and the
    FP64 fields agree to the order of their FP64 additions; both match the oracle."""
    from fastweavturb_b200.configs import small
    w = small(N=64, seed=7, nlev=2, tubes0=3, nodes0=128, sigma0=0.04)
    p, cl = oracle_inputs(orc, w)
    fields = {}
    for cells in (4.0, 0.0):
        ctx = fwt.Context(gpu_params(fwt, w, precision=precision, deposit_mode=0))
        ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
        ctx.set_raster_radius_limit(cells)
        ctx.deposit(1, w.ntubes)
        fields[cells] = ctx.field(0).copy()
        ctx.close()
    assert np.abs(fields[4.0]).max() > 0
    if precision == 32:
        assert np.array_equal(fields[4.0], fields[0.0])
    else:
        assert rel_l2(fields[4.0], fields[0.0]) <= 1e-15
    floor, vor = fp64_floor(orc, p, cl)
    assert rel_l2(fields[4.0], vor) <= (TOL32 if precision == 32 else tol64(floor))


def test_piece_and_subsegment_kernels_agree(fwt, orc):
    """Thin tubes (Rtube 1.2-1.9 grid spacings on 64^3) deposited by the chord-piece kernel and
    by the sub-segment kernel: the same accepted points, evaluated by two forms of the same
    vorticity, agree to FP32 rounding; both match the FP64 oracle on every point, and so do
    both kernels of the FP64 tile path at FP64 rounding."""
    from fastweavturb_b200.configs import small
    w = small(N=64, seed=5, nlev=2, tubes0=3, nodes0=128, sigma0=0.04)
    p, cl = oracle_inputs(orc, w)
    fields = {}
    for precision in (32, 64):
        for cells in (0.0, 8.0):
            ctx = fwt.Context(gpu_params(fwt, w, precision=precision, deposit_mode=0))
            ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
            ctx.set_piece_radius_limit(cells)
            ctx.deposit(1, w.ntubes)
            fields[precision, cells] = ctx.field(0).copy()
            ctx.close()
    assert np.abs(fields[32, 8.0]).max() > 0
    assert rel_l2(fields[32, 8.0], fields[32, 0.0]) <= 1e-6
    floor, vor = fp64_floor(orc, p, cl)
    assert rel_l2(fields[32, 8.0], vor) <= TOL32
    assert rel_l2(fields[32, 0.0], vor) <= TOL32
    assert rel_l2(fields[64, 8.0], vor) <= tol64(floor)
    assert rel_l2(fields[64, 0.0], vor) <= tol64(floor)


@pytest.mark.parametrize("N", [36, 40])
@pytest.mark.parametrize("piece_cells", [None, 0.0])
@pytest.mark.parametrize("precision", [32, 64])
def test_partial_tiles(fwt, orc, N, piece_cells, precision):
    """Grids that are not a multiple of the 16 x 8 x 8 deposition tile (N = 36: partial tiles
    along every axis; N = 40: along x only), through the chord-piece kernel (default) and the
    sub-segment kernel (piece_cells = 0), in FP32 and in the FP64 tile path: omega matches the
    FP64 oracle on every point."""
    from fastweavturb_b200.configs import small
    w = small(N=N, seed=9, nlev=2, tubes0=2, nodes0=64, sigma0=0.2)
    p, cl = oracle_inputs(orc, w)
    ctx = fwt.Context(gpu_params(fwt, w, precision=precision, deposit_mode=0))
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    if piece_cells is not None:
        ctx.set_piece_radius_limit(piece_cells)
    ctx.deposit(1, w.ntubes)
    vor = ctx.field(0).copy()
    floor, vor_o = fp64_floor(orc, p, cl)
    assert np.abs(vor).max() > 0
    assert rel_l2(vor, vor_o) <= (TOL32 if precision == 32 else tol64(floor))
    ctx.close()


@pytest.mark.parametrize("precision,mode,tol_uw,tol_d", [(32, 0, 1e-5, 1e-4), (64, 1, 1e-6, 1e-6)])
def test_optional_field_outputs_match_oracle(fwt, orc, small_case, precision, mode, tol_uw, tol_d, tmp_path):
    """field_uw.dat and field_wd.dat (the reference's u_out / d_out outputs, tube.f90:1075-1120):
    the downsampled u and omega, and the dissipation S_ij S_ij from spectral derivatives
    (subroutine.f90:1086-1163), against the oracle's FP64 fields.  The boxes are REAL(4), so
    the FP64 path is held to float32 rounding.  A second call gives the same box, and
    write_outputs writes the same numbers when the switches are on."""
    w, p, cl, ref = small_case
    ctx = _gpu_run(fwt, w, cl, p, precision, mode)
    uw, wd = ctx.field_uw(), ctx.field_wd()
    uw_o = orc.field_uw(ref["vor"], ref["vel"], p.N_downsample)
    wd_o = orc.field_wd(ref["vor"], ref["vel"], p.N_downsample)
    assert uw.shape == uw_o.shape and wd.shape == wd_o.shape
    assert rel_l2(uw[:3], uw_o[:3]) <= tol_uw and rel_l2(uw[3:], uw_o[3:]) <= tol_uw
    assert rel_l2(wd[0], wd_o[0]) <= tol_uw
    assert wd_o[1].max() > 0 and rel_l2(wd[1], wd_o[1]) <= tol_d
    assert np.array_equal(ctx.field_wd(), wd)
    ctx.set_outputs(u_out=True, d_out=True)
    ctx.write_outputs(tmp_path / "output")
    assert np.array_equal(np.fromfile(tmp_path / "output" / "field_uw.dat", dtype=np.float32), uw.ravel())
    assert np.array_equal(np.fromfile(tmp_path / "output" / "field_wd.dat", dtype=np.float32), wd.ravel())
    ctx.close()


@pytest.mark.parametrize("sigma_ratio", [1.0, 4.0])
def test_scatter_equals_tile_pieces(fwt, orc, sigma_ratio):
    """Thin tubes (truncation radius 1.8-3.7 grid spacings on 64^3) through the scatter kernel
    (each piece searched once, int64 global sums; the FP32 default for piece lines) and through
    the piece tile kernel: the same accepted pairs and FP64 hand-overs, fields equal to FP32
    rounding (the tile path rounds omega to FP32 after every batch, the scatter path once), both
    matching the FP64 oracle.  sigma_ratio 4 takes the curved-branch terms (General)."""
    from fastweavturb_b200.configs import small
    w = small(N=64, seed=11, nlev=2, tubes0=3, nodes0=128, sigma0=0.12 / sigma_ratio)
    w.sigma_ratio = sigma_ratio
    p, cl = oracle_inputs(orc, w)
    fields, counts = {}, {}
    for cells in (8.0, 0.0):
        ctx = fwt.Context(gpu_params(fwt, w, precision=32, deposit_mode=0))
        ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
        ctx.set_scatter_radius_limit(cells)
        ctx.deposit(1, w.ntubes)
        fields[cells] = ctx.field(0).copy()
        counts[cells] = ctx.counters()
        ctx.close()
    assert np.abs(fields[8.0]).max() > 0
    assert counts[8.0]["accepted"] == counts[0.0]["accepted"]
    assert counts[8.0]["redone_fp64"] == counts[0.0]["redone_fp64"]
    assert counts[8.0]["pairs"] == 0 < counts[0.0]["pairs"]
    assert rel_l2(fields[8.0], fields[0.0]) <= 1e-6
    vor, _ = orc.deposit(p, cl)
    assert rel_l2(fields[8.0], vor) <= TOL32
    assert rel_l2(fields[0.0], vor) <= TOL32


@pytest.mark.parametrize("path", ["subsegment", "piece", "scatter"])
def test_deferred_list_windows_are_exact(fwt, orc, path):
    """The list of pairs handed from FP32 to FP64 limited to 16 entries: every launch overflows
    it and lists its deferred pairs again in windows of tiles (or chunks of pieces), evaluating
    one window at a time.  The FP64 contributions are int64 sums, so the field equals the one
    built with the default list bit for bit, through each of the three deposition kernels."""
    from fastweavturb_b200.configs import small
    w = small(N=64, seed=11, nlev=2, tubes0=3, nodes0=128, sigma0=0.03)
    w.sigma_ratio = 4.0
    p, cl = oracle_inputs(orc, w)
    piece, scatter = {"subsegment": (0.0, 0.0), "piece": (64.0, 0.0), "scatter": (64.0, 64.0)}[path]
    fields, counts = {}, {}
    for limit in (0, 16):
        ctx = fwt.Context(gpu_params(fwt, w, precision=32, deposit_mode=0))
        ctx.set_piece_radius_limit(piece)
        ctx.set_scatter_radius_limit(scatter)
        ctx.set_defer_limit(limit)
        ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
        ctx.deposit(1, w.ntubes)
        fields[limit] = ctx.field(0).copy()
        counts[limit] = ctx.counters()
        ctx.close()
    assert counts[16]["redone_fp64"] > 64
    assert counts[0] == counts[16]
    assert np.array_equal(fields[0], fields[16])
    vor, _ = orc.deposit(p, cl)
    assert rel_l2(fields[16], vor) <= TOL32


def test_async_node_upload_equals_synchronous(fwt, orc):
    """fwt_set_centerlines_async: the nodes' upload runs on its own stream and each batch of
    lines waits for its own nodes.  With a memory cap that splits the 74 K nodes into three
    batches, the field and the counters equal those of the synchronous upload bit for bit, and
    a second deposition after an asynchronous upload into the same context does too."""
    from fastweavturb_b200.configs import small
    w = small(N=64, seed=7, nlev=3, tubes0=4, nodes0=256, sigma0=0.2)
    p, cl = oracle_inputs(orc, w)
    assert cl.xyz.size // 3 > 2 * 32768
    out = {}
    for mode in ("sync", "async", "async-again"):
        if mode != "async-again":
            ctx = fwt.Context(gpu_params(fwt, w, precision=32, deposit_mode=0, mem_cap=512 << 20))
        ctx.set_centerlines(cl.npoint, cl.xyz.copy(), p.sigma, p.Gamma, p.n_T, async_upload=(mode != "sync"))
        ctx.deposit(1, w.ntubes)
        cnt = ctx.counters()
        cnt.pop("launches")   # the context's running launch count
        out[mode] = (ctx.field(0).copy(), cnt)
        if mode == "sync":
            ctx.close()
    ctx.close()
    for mode in ("async", "async-again"):
        assert np.array_equal(out[mode][0], out["sync"][0])
        assert out[mode][1] == out["sync"][1]
    assert np.abs(out["sync"][0]).max() > 0
