"""The committed golden fixtures (tests/golden/, written by make_golden.py) against the oracle,
and the reference's input file format (CPU only).

wt2_inputs.npz holds the reference's own shipped input pair (73 tubes x 148 nodes,
sigma_ratio 4, n_T 1/2/4); wt2_n64_oracle.npz the oracle's outputs on it at N = 64.  Re-running
the oracle must reproduce them, so a change to the oracle shows here before it can move the
GPU parity tests.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def wt2_inputs(O, N=64):
    z = np.load(os.path.join(GOLD, "wt2_inputs.npz"))
    s = z["scalars"]
    p = O.Params(N=N, N_downsample=N, line_s=int(s[2]), line_e=int(s[3]), sigma_ratio=float(s[4]),
                 eta_t=float(s[5]), ntf_times=int(s[6]), ntf_pre=int(s[7]), Rtube_ratio=float(s[8]),
                 dzeta_sup=float(s[9]), sigma=z["sigma"], Gamma=z["Gamma"], n_T=z["n_T"].astype(np.int32),
                 if_filter=z["if_filter"].astype(np.int32))
    return p, O.Centerlines(npoint=z["npoint"].astype(np.int64), xyz=z["xyz"])


def write_reference_inputs(d, p, cl, N=None):
    """Write centerline_input.dat / parameters_input.dat in the reference's layout
    (FBB_with_parameters.m:55-59,122-125,205-240; read by tube.f90:168-223,341-379)."""
    N = N or p.N
    with open(os.path.join(d, "centerline_input.dat"), "w") as f:
        f.write(f"{len(cl.npoint):18d}\n")
        for n in cl.npoint:
            f.write(f"{int(n):18d}\n")
        for x, y, z in cl.xyz:
            f.write(f"{x:24.16E} {y:24.16E} {z:24.16E}\n")
    rows = [("N", f"{N:8d}"), ("N_downsample", f"{N:8d}"), ("line_s", f"{p.line_s:8d}"),
            ("line_e", f"{p.line_e:8d}"), ("sigma_ratio", f"{p.sigma_ratio:18.5f}"),
            ("eta_t", f"{p.eta_t:18.5f}")]
    with open(os.path.join(d, "parameters_input.dat"), "w") as f:
        for k, v in rows:
            f.write(f"{k}\n{v}\n")
        f.write("---------------\n")
        for k, v in [("ntf_times", f"{p.ntf_times:8d}"), ("ntf_pre", f"{p.ntf_pre:8d}"),
                     ("Rtube_ratio", f"{p.Rtube_ratio:18.5f}"), ("dzeta_sup", f"{p.dzeta_sup:18.4f}")]:
            f.write(f"{k}\n{v}\n")
        f.write("---------------\n")
        f.write('variables="i_line","sigma","Gamma","n_T","if_filter"\n')
        for i in range(len(cl.npoint)):
            f.write(f"{i + 1:8d} {p.sigma[i]:17.7g} {p.Gamma[i]:17.7g} {int(p.n_T[i]):7d} {int(p.if_filter[i]):7d}\n")


def test_wt2_fixture_shape(orc):
    p, cl = wt2_inputs(orc)
    assert len(cl.npoint) == 73 and int(cl.npoint.sum()) == 73 * 148
    assert p.sigma_ratio == 4.0 and p.Rtube_ratio == 3.0 and p.ntf_times == 50 and p.ntf_pre == 1000
    assert set(np.unique(p.n_T)) == {1, 2, 4}
    assert np.all(cl.xyz >= -np.pi) and np.all(cl.xyz < np.pi)


def test_input_files_round_trip(orc, tmp_path):
    p, cl = wt2_inputs(orc)
    write_reference_inputs(str(tmp_path), p, cl)
    cl2 = orc.read_centerlines(str(tmp_path / "centerline_input.dat"))
    p2 = orc.read_parameters(str(tmp_path / "parameters_input.dat"), len(cl2.npoint))
    assert np.array_equal(cl2.npoint, cl.npoint)
    assert np.array_equal(cl2.xyz, cl.xyz)
    assert p2.N == 64 and p2.sigma_ratio == p.sigma_ratio and p2.dzeta_sup == p.dzeta_sup
    np.testing.assert_allclose(p2.sigma, p.sigma, rtol=1e-6)
    assert np.array_equal(p2.n_T, p.n_T)


@pytest.fixture(scope="module")
def wt2_run(orc):
    p, cl = wt2_inputs(orc)
    return p, cl, orc.run(p, cl, sp_pmax=10)


def test_oracle_reproduces_wt2_golden(orc, wt2_run):
    p, cl, out = wt2_run
    g = np.load(os.path.join(GOLD, "wt2_n64_oracle.npz"))
    for i in (0, 1, 72):
        assert np.array_equal(orc.line_ntf(cl.line(i), p.ntf_times, p.ntf_pre)[0], g[f"ntf_line{i + 1}"])
    assert np.array_equal(np.array([r[3] for r in out["line_info"]]), g["ntf_max"])
    assert np.array_equal(np.array([r[4] for r in out["line_info"]]), g["accepted"])
    np.testing.assert_allclose(out["vor"][:, ::4, ::4, ::4], g["vor_sample"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(out["spectrum_vor"], g["spectrum_vor"], rtol=1e-11)
    np.testing.assert_allclose(out["spectrum"], g["spectrum"], rtol=1e-11)
    np.testing.assert_allclose([out["up"], out["Etot"], out["Enstrophy"]], g["scalars"], rtol=1e-12)
    assert np.array_equal(out["pdf_u"][2], g["pdf_u_counts"])
    assert np.array_equal(out["pdf_u"][0], g["pdf_u_val"])
    assert np.array_equal(out["pdf_w"][2], g["pdf_w_counts"])
    assert np.array_equal(out["Sp_r"], g["Sp_r"])
    np.testing.assert_allclose(out["Sp"], g["Sp"], rtol=1e-10, atol=1e-300)


def test_wt2_physics(wt2_run):
    """Properties the reference's statistics must have on its own input: E/u'^2 = 3/2, S_1 ~ 0
    (homogeneity), S_2 > 0 growing at small r and zero at r = N (a full period), the PDF
    drops only the few values that fall in the gaps its REAL(4) edges leave between bins."""
    p, cl, out = wt2_run
    assert out["Etot"] / out["up"] ** 2 == pytest.approx(1.5, rel=1e-13)
    Sp = out["Sp"]
    assert np.all(np.abs(Sp[0]) < 1e-12)
    assert np.all(Sp[1][:-1] > 0) and Sp[1][2] > Sp[1][0]
    assert out["Sp_r"][-1] == p.N and Sp[1][-1] == 0.0
    N = p.N
    assert 0 <= 3 * N ** 3 - int(out["pdf_u"][2].sum()) <= 3 * N ** 3 // 10000
