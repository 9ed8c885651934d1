"""Host-side logic of the workloads, the ensemble and the surrogate pipeline (no GPU)."""
import numpy as np

from fastweavturb_b200 import configs
from fastweavturb_b200.ensemble import Ensemble
from fastweavturb_b200.surrogate import (N_FLAT, N_OUT, N_SHELLS, PARAM_HI, PARAM_LO, Surrogate, draw_params,
                                         features, fit_error, within)


def test_level_seeds_are_deterministic_and_distinct():
    seeds = {(s, l): configs.level_seed(s, l) for s in range(4) for l in range(8)}
    assert all(0 <= v < 2 ** 64 for v in seeds.values())
    assert len(set(seeds.values())) == len(seeds)
    assert configs.level_seed(3, 2) == configs.level_seed(3, 2)


def test_surrogate_member_levels_counts_and_streams():
    w = configs.surrogate_member((0.55, 8.0, 1.5, 4.0, 1.35), seed=11, N=64)
    assert w.level_streams and w.N == 64 and len(w.levels) == 4
    assert [L.tubes for L in w.levels] == [max(1, int(round(1.5 * 4 * 4 ** l))) for l in range(4)]
    assert [L.nodes for L in w.levels] == [64 * 2 ** l for l in range(4)]
    sig = [L.sigma for L in w.levels]
    assert np.allclose(sig, [0.4 * 2.0 ** -l for l in range(4)])
    assert np.allclose([L.Gamma for L in w.levels], [(s / sig[0]) ** 1.35 for s in sig])
    # the benchmark workloads keep one stream numbered across levels
    assert not configs.cfg1().level_streams


def test_a_density_change_only_touches_the_end_of_a_level():
    a = configs.surrogate_member((0.5, 4.0, 1.0, 3.0, 1.3), seed=5)
    b = configs.surrogate_member((0.5, 4.0, 1.1, 3.0, 1.3), seed=5)
    ta, tb = [L.tubes for L in a.levels], [L.tubes for L in b.levels]
    assert ta != tb and all(y >= x for x, y in zip(ta, tb))
    # per-level streams: level l's first min(ta[l], tb[l]) tubes come from the same stream
    assert [configs.level_seed(a.seed, l) for l in range(3)] == [configs.level_seed(b.seed, l) for l in range(3)]


def test_ensemble_context_caps_per_grid_size():
    ens = Ensemble(workers=8, tune=False)
    assert ens.slots_for(64) == 8 and ens.slots_for(96) == 8
    assert ens.slots_for(128) == 2 and ens.slots_for(256) == 1
    assert Ensemble(workers=1).slots_for(256) == 1
    assert ens.ctx == {}            # nothing is created before a run


def test_ensemble_memory_plan_shares_the_device_by_volume():
    from fastweavturb_b200.ensemble import cfg3_members
    members = cfg3_members(64)
    ens = Ensemble(workers=4, tune=False)
    caps = ens.plan(members, total=180e9)
    sizes = sorted({w.N for w in members})
    assert sorted(caps) == sizes
    # the contexts' caps fill 80 % of the device and grow with the grid size
    used = sum(ens.slots_for(N) * caps[N] for N in sizes)
    assert 0.79 * 180e9 <= used <= 0.8 * 180e9
    assert all(caps[a] < caps[b] for a, b in zip(sizes, sizes[1:]))
    assert caps[sizes[0]] >= 2e9 and ens._cap(sizes[-1]) == caps[sizes[-1]]
    assert ens.plan(members, total=1.0) is caps     # planned once


def test_draw_params_stay_in_the_box():
    P = draw_params(np.random.default_rng(0), 2000)
    assert P.shape == (2000, 5)
    assert np.all(P >= PARAM_LO - 1e-12) and np.all(P <= PARAM_HI + 1e-12)
    assert set(np.unique(P[:, 3])) == {2.0, 3.0, 4.0}
    assert np.allclose(P[:, 1], 2.0 ** (P[:, 3] - 1))
    X = Surrogate.xin(P)
    assert np.all(np.abs(X) <= 1.0 + 1e-12)


def test_features_and_fit_error():
    N = 64
    k = np.arange(1, N // 2 + 1, dtype=np.float64)
    r = np.array([1, 1, 2, 3, 4, 6, 8, 11, 16, 23, 32, 45, 64])
    st = {"Ek": k ** (-5.0 / 3.0), "r": r, "flat": 3.0 + 0.01 * np.arange(len(r)),
          "zeta": np.array([0.35, 0.7, 1.0, 1.28, 1.55, 1.8])}
    y = features(st, N)
    assert y.shape == (N_OUT,)
    assert np.allclose(y[:N_SHELLS], -5.0 / 3.0 * np.log(np.exp(np.linspace(0, np.log(N / 2), N_SHELLS))))
    # the first 8 distinct separations (r = 1 appears twice in the reference's grid)
    assert np.allclose(y[N_SHELLS:N_SHELLS + N_FLAT], 3.0 + 0.01 * np.array([0, 2, 3, 4, 5, 6, 7, 8]))
    assert np.allclose(y[N_SHELLS + N_FLAT:], [0.7, 1.0, 1.28, 1.55, 1.8])
    assert fit_error(y, y) == (0.0, 0.0) and within(fit_error(y, y))
    z = y.copy()
    z[:N_SHELLS] += 0.03
    eE, eF = fit_error(z, y)
    assert abs(eE - 0.03) < 1e-12 and eF == 0.0 and not within((eE, eF))


def test_benchmark_workloads_follow_their_configurations():
    """cfg0: 64^3, 3 levels, sigma_l = 0.3 2^-l, n_l = 4 4^l; cfg1: 256^3, 6 levels, 0.4 2^-l,
    4 4^l; cfg2: 1024^3, 8 levels, 0.5 2^-l, 2 4^l; nodes 256 2^l, H = 0.7,
    Gamma_l = (sigma_l / sigma_0)^(4/3) in all three."""
    for w, N, nlev, s0, t0 in ((configs.cfg0(), 64, 3, 0.3, 4), (configs.cfg1(), 256, 6, 0.4, 4),
                               (configs.cfg2(), 1024, 8, 0.5, 2)):
        assert w.N == N and len(w.levels) == nlev and not w.level_streams
        for l, L in enumerate(w.levels):
            assert np.isclose(L.sigma, s0 * 2.0 ** -l) and L.tubes == t0 * 4 ** l and L.nodes == 256 * 2 ** l
            assert L.H == 0.7 and np.isclose(L.Gamma, (L.sigma / s0) ** (4.0 / 3.0))
    assert configs.cfg1().ntubes == 5460 and configs.cfg1().nnodes == 38347776
    assert configs.cfg2().ntubes == 43690


def test_write_ply_layout(tmp_path):
    """The PLY writer of isosurface triangles: header counts, vertex records of 4 floats and
    faces of (3, i, i+1, i+2)."""
    from fastweavturb_b200.api import write_ply
    tris = np.arange(2 * 3 * 4, dtype=np.float32).reshape(2, 3, 4)
    p = tmp_path / "m.ply"
    write_ply(p, tris)
    raw = p.read_bytes()
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    head = raw[:end].decode()
    assert "element vertex 6" in head and "element face 2" in head and "property float helicity" in head
    body = raw[end:]
    v = np.frombuffer(body[:6 * 16], dtype="<f4").reshape(6, 4)
    assert np.array_equal(v, tris.reshape(6, 4))
    f = np.frombuffer(body[6 * 16:], dtype=[("n", "u1"), ("v", "<i4", (3,))])
    assert list(f["n"]) == [3, 3] and f["v"].tolist() == [[0, 1, 2], [3, 4, 5]]


def test_autotuner_keeps_the_default_unless_clearly_faster():
    t = {("raster", 0.0): 1.00, ("raster", 1.5): 0.97, ("raster", 2.5): 1.20, ("raster", 4.0): 0.99}
    assert Ensemble.pick(t, "raster", (0.0, 1.5, 2.5, 4.0), 0.0) == 0.0      # 3 % is within the noise
    t[("raster", 2.5)] = 0.90
    assert Ensemble.pick(t, "raster", (0.0, 1.5, 2.5, 4.0), 0.0) == 2.5      # 10 % faster
    t = {("piece", 8.0): 2.0, ("piece", 5.0): 1.0}
    assert Ensemble.pick(t, "piece", (5.0, 8.0), 8.0) == 5.0
    assert Ensemble.pick(t, "piece", (5.0, 8.0), 5.0) == 5.0                 # the default is the fastest
