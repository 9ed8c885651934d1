"""The grid split over ranks (fastweavturb_b200/distributed.py) on CPU: world_size-2 gloo ranks
run the distributed transforms, the slab <-> pencil all-to-alls and the S_p exchange on a
random FP64 vorticity field, with the per-pencil Biot-Savart and the per-box S_p sums restated
here in torch / numpy (the library's kernels need a GPU; the GPU test of the same driver with
them is in test_gpu_distributed.py).  The assembled velocity, spectra and S_p must equal the
oracle's single-grid results (oracle.biot_savart, spectrum, structure_functions_np) to FP64
rounding.
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = 16


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def pencil_block(P, y0, ny, N):
    """The Biot-Savart of fwt_biot_savart_block on a pencil (3, N kz, ny ky, N/2+1 kx), in torch:
    1/N^3 scaling, shells int(sqrt(k^2 + 1e-8) + 0.5), half-spectrum weights, u^ = i k' x w^/|k|^2
    with the Nyquist components of k' set to 0 (the real part of the reference's backward
    transform)."""
    import torch

    nh = N // 2 + 1
    jz = torch.arange(N).view(N, 1, 1)
    jy = (y0 + torch.arange(ny)).view(1, ny, 1)
    jx = torch.arange(nh).view(1, 1, nh)
    kz = (jz + N // 2) % N - N // 2
    ky = (jy + N // 2) % N - N // 2
    kx = jx
    k2 = (kx * kx + ky * ky + kz * kz).double()
    kxe = torch.where(jx == N // 2, 0, kx).double()
    kye = torch.where(jy == N // 2, 0, ky).double()
    kze = torch.where(jz == N // 2, 0, kz).double()
    w = P / float(N) ** 3
    wgt = torch.where((jx == 0) | (jx == N // 2), 1.0, 2.0).double()
    ew = 0.5 * wgt * (w.abs() ** 2).sum(0)
    ik2 = torch.where(k2 > 0, 1.0 / torch.where(k2 > 0, k2, 1.0), 0.0)
    a, b, c = w[0], w[1], w[2]
    u = torch.stack([1j * (kye * c - kze * b), 1j * (kze * a - kxe * c), 1j * (kxe * b - kye * a)]) * ik2
    P.copy_(u)
    eu = 0.5 * wgt * (u.abs() ** 2).sum(0)
    shell = torch.floor(torch.sqrt(k2 + 1e-8) + 0.5).long()
    nek = N // 2
    shw = torch.zeros(nek + 1, dtype=torch.float64).index_add_(0, shell.clamp(max=nek).view(-1),
                                                               torch.where(shell <= nek, ew, 0.0).view(-1))
    shu = torch.zeros(nek + 1, dtype=torch.float64).index_add_(0, shell.clamp(max=nek).view(-1),
                                                               torch.where(shell <= nek, eu, 0.0).view(-1))
    return shw[1:].numpy(), shu[1:].numpy(), float(eu.sum()), float(ew.sum())


def box_sums(box, n0, n1, n2, axis, r):
    """fwt_sp_block's sums on a box (x fastest) along `axis`, in numpy."""
    a = box.numpy().reshape(n2, n1, n0)
    ax = {0: 2, 1: 1, 2: 0}[axis]
    out = np.zeros((10, len(r)))
    for m, rr in enumerate(r):
        du = np.roll(a, -int(rr), axis=ax) - a
        pw = np.ones_like(du)
        for p in range(10):
            pw = pw * du
            out[p, m] = pw.sum()
    return out


def _rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from fastweavturb_b200.distributed import TorchComm, spectral_velocity, structure_function_sums
    from oracle.oracle import sp_separations

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        comm = TorchComm()
        vor = np.random.default_rng(5).standard_normal((3, N, N, N))
        nz = N // world
        w = torch.from_numpy(vor[:, rank * nz:(rank + 1) * nz].copy())
        u, shw, shu, E, Z = spectral_velocity(comm, w, N, lambda P, y0, ny: pencil_block(P, y0, ny, N))
        r = sp_separations(N)
        Sp = structure_function_sums(comm, u, N, 1.0, r, lambda b, n0, n1, n2, ax: box_sums(b, n0, n1, n2, ax, r))
        q.put((rank, u.numpy(), shw, shu, E, Z, Sp))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_distributed_transforms_equal_the_single_grid(orc):
    world = 2
    ctxmp = mp.get_context("spawn")
    q = ctxmp.Queue()
    port = _free_port()
    procs = [ctxmp.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    vor = np.random.default_rng(5).standard_normal((3, N, N, N))
    vel = orc.biot_savart(vor)
    u = np.concatenate([r[1] for r in res], axis=1)
    assert np.abs(u - vel).max() <= 1e-12 * np.abs(vel).max()
    # spectra and totals: every rank holds the all-reduced sums
    np.testing.assert_allclose(res[0][2], orc.spectrum(vor), rtol=1e-12)
    np.testing.assert_allclose(res[1][3], orc.spectrum(vel), rtol=1e-12)
    dv = (2 * np.pi / N) ** 3
    E = orc.cal_helicity(vel, vel, dv) / 2.0 / (2 * np.pi) ** 3
    assert res[0][4] == pytest.approx(E, rel=1e-12)
    _, Sp = orc.structure_functions_np(vel, pmax=10)
    np.testing.assert_allclose(res[0][6], Sp, rtol=1e-10, atol=1e-14 * np.abs(Sp).max())
