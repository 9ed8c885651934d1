"""The grid split over ranks with the library's kernels (fwt_set_slab, fwt_biot_savart_block,
fwt_sp_block), the ranks run as threads on one GPU (distributed.ThreadComm: the exchanges are
host hand-overs between barriers; no kernel of one rank waits for another's), against the same
field built whole by one context.  The slab depositions add the same fixed-point
contributions, so omega is identical; u, the spectra and S_p differ only by the order of the
split transforms' FP32 rounding.
"""
import threading

import numpy as np
import pytest

from helpers import gpu_params, oracle_inputs, rel_l2, sp_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ranks", [2, 4])
def test_slab_ranks_equal_the_whole_grid(fwt, orc, ranks):
    import torch

    from fastweavturb_b200.configs import small
    from fastweavturb_b200.distributed import ThreadComm, build_field

    w = small(N=64, seed=4, nlev=2, tubes0=2, nodes0=64, sigma0=0.3)
    p, cl = oracle_inputs(orc, w)
    prm = gpu_params(fwt, w, precision=32, deposit_mode=0)
    ctx = fwt.Context(prm)
    ctx.set_centerlines(cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
    ctx.run()
    w_full = ctx.field_tensor(0).cpu().numpy()
    u_full = ctx.field_tensor(1).cpu().numpy()
    s = ctx.cal_helicity()
    ew, eu = ctx.spectrum(0), ctx.spectrum(1)
    r, Sp = ctx.Sp_calculate(pmax=10)
    ctx.close()

    comm = ThreadComm(ranks)
    out = [None] * ranks
    errs = []

    def run(rank):
        try:
            torch.cuda.set_device(0)
            out[rank] = build_field(comm.bind(rank), prm, cl.npoint, cl.xyz, p.sigma, p.Gamma, p.n_T)
        except Exception as e:   # surfaced below
            errs.append(e)
            comm._barrier.abort()

    th = [threading.Thread(target=run, args=(k,)) for k in range(ranks)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    w_d = np.concatenate([o["w"].cpu().numpy() for o in out], axis=1)
    u_d = np.concatenate([o["u"].cpu().numpy() for o in out], axis=1)
    assert np.array_equal(w_d, w_full)
    assert rel_l2(u_d, u_full) <= 1e-6
    o = out[0]
    assert o["up"] == pytest.approx(s["up"], rel=1e-6)
    assert o["Enstrophy"] == pytest.approx(s["Enstrophy"], rel=1e-6)
    assert rel_l2(o["spectrum_vor"], ew) <= 1e-6
    assert rel_l2(o["spectrum"], eu) <= 1e-6
    assert np.array_equal(o["Sp_r"], r)
    for q in range(1, 6):
        sp_close(o["Sp"], Sp, q, 1e-5)
    for k in range(1, ranks):
        np.testing.assert_allclose(out[k]["Sp"], o["Sp"], rtol=0, atol=0)
