"""One woven field on a grid split over GPUs: the reference's MPI decomposition for N >= 2048,
where three N^3 fields no longer fit one GPU.

The reference splits the grid into z-slabs (tube.f90:261-265): every rank walks every
sub-segment box and keeps the points of its own planes (tube.f90:800-804), transforms by
pencil transposes (fourier_forward / fourier_backward, subroutine.f90:938-968) and gathers to
rank 0 for S_p (subroutine.f90:91-93).  Here, one process per GPU:

1. deposition: a z-slab context (fwt_set_slab) deposits every line into its planes only;
2. forward transform: R2C over (y, x) of the slab, transpose to y-pencils (all z, N/R values
   of ky) with an all-to-all, complex transform over z;
3. fwt_biot_savart_block on the pencil: u^ = i k x w^ / |k|^2, the pencil's spectra, energy
   and enstrophy, summed over the ranks with an all-reduce;
4. backward transform: over z, all-to-all back to slabs, C2R over (y, x);
5. S_p: the x and y increments on the slab, the z increments on a y-pencil of u_z (one more
   all-to-all), each with fwt_sp_block; the sums are all-reduced.

The transforms are cuFFT's (through torch.fft); the exchanges are the communicator's
all-to-all (NCCL over NVLink between GPUs: plain peer transfers, no multicast); the
Biot-Savart and S_p arithmetic are the library's kernels.  N must be divisible by 8 R (whole
deposition tiles per slab) and by R (pencils).

    python -m torch.distributed.run --nproc-per-node R fastweavturb_b200/distributed.py --config cfg2

prints rank 0's spectra and S_p summary as JSON.
"""
from __future__ import annotations

import math
import threading

import numpy as np


class TorchComm:
    """The communicator over torch.distributed (NCCL for CUDA tensors, gloo for CPU tensors)."""

    def __init__(self, group=None, device="cpu"):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.device = device      # where the all-reduce buffers live: "cpu" for gloo, a GPU for NCCL
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def all_to_all(self, chunks):
        """chunks[k] goes to rank k; returns the chunks received, rank order.  All chunks have
        one shape."""
        import torch

        real = chunks[0].is_complex()
        inp = torch.stack([torch.view_as_real(c) if real else c for c in chunks]).contiguous()
        out = torch.empty_like(inp)
        self.dist.all_to_all_single(out, inp, group=self.group)
        parts = list(out.unbind(0))
        return [torch.view_as_complex(p.contiguous()) for p in parts] if real else parts

    def all_reduce_sum(self, a):
        import torch

        t = torch.as_tensor(np.asarray(a, dtype=np.float64)).to(self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()


class ThreadComm:
    """The same exchanges between R ranks run as threads of one process (each rank a thread
    with its own context; one GPU).  The ranks hand tensors over through shared slots between
    barriers; no kernel of one rank waits for another's."""

    def __init__(self, world):
        self.world = world
        self._barrier = threading.Barrier(world)
        self._slots = [None] * world
        self._local = threading.local()

    def bind(self, rank):
        self._local.rank = rank
        return self

    @property
    def rank(self):
        return self._local.rank

    def _exchange(self, item):
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()
        self._slots[self.rank] = item
        self._barrier.wait()
        got = list(self._slots)
        self._barrier.wait()
        return got

    def all_to_all(self, chunks):
        got = self._exchange([c.contiguous() for c in chunks])
        return [got[j][self.rank] for j in range(self.world)]

    def all_reduce_sum(self, a):
        got = self._exchange(np.asarray(a, dtype=np.float64))
        return np.sum(got, axis=0)


# ---------------------------------------------------------------------------- transposes
def slab_to_pencil(comm, A, R):
    """(c, nz, N, m) slab of this rank (planes rank*nz..) -> (c, N, N/R, m) pencil of the ky
    (second) index rank*N/R.. with every z."""
    ny = A.shape[2] // R
    got = comm.all_to_all([A[:, :, k * ny:(k + 1) * ny] for k in range(R)])
    import torch

    return torch.cat(got, dim=1)


def pencil_to_slab(comm, P, R):
    """Inverse of slab_to_pencil."""
    nz = P.shape[1] // R
    got = comm.all_to_all([P[:, j * nz:(j + 1) * nz] for j in range(R)])
    import torch

    return torch.cat(got, dim=2)


# ---------------------------------------------------------------------------- the field
def spectral_velocity(comm, w, N, block):
    """u on this rank's slab from omega on it (both (3, nz, N, N), x fastest): the distributed
    transforms around block(P, y0, ny) -> (shells_w, shells_u, energy, enstrophy), which turns
    the pencil P (3, N, ny, N/2 + 1), unscaled transforms of omega, into u^ in place.  Returns u
    and the summed spectra and totals."""
    import torch

    R = comm.world
    ny = N // R
    W = torch.fft.rfft2(w, dim=(-2, -1))
    P = torch.fft.fft(slab_to_pencil(comm, W, R), dim=1).contiguous()
    if P.is_cuda:
        torch.cuda.synchronize()
    shw, shu, E, Z = block(P, comm.rank * ny, ny)
    tot = comm.all_reduce_sum(np.concatenate([shw, shu, [E, Z]]))
    nek = N // 2
    U = pencil_to_slab(comm, torch.fft.ifft(P, dim=1, norm="forward"), R)
    u = torch.fft.irfft2(U, s=(N, N), dim=(-2, -1), norm="forward").contiguous()
    if u.is_cuda:
        torch.cuda.synchronize()
    return u, tot[:nek], tot[nek:2 * nek], float(tot[2 * nek]), float(tot[2 * nek + 1])


def structure_function_sums(comm, u, N, scale, r, sp):
    """S_p (10, len(r)) of the slab velocity u (3, nz, N, N): x and y increments on the slab, z
    increments on a y-pencil of u_z; sp(box, n0, n1, n2, axis) -> sums of one box."""
    import torch

    R = comm.world
    nz, ny = u.shape[1], N // R
    S = sp(u[0], N, N, nz, 0) + sp(u[1], N, N, nz, 1)
    uz = u[2]
    got = comm.all_to_all([uz[:, k * ny:(k + 1) * ny, :] for k in range(R)])
    pencil = torch.cat(got, dim=0).contiguous()          # (N z, ny, N x)
    if pencil.is_cuda:
        torch.cuda.synchronize()
    S = S + sp(pencil, N, ny, N, 2)
    return comm.all_reduce_sum(S) / (3.0 * N ** 3)


def build_field(comm, params, npoint, xyz, sigma, Gamma, n_T, device=0):
    """This rank's share of one woven field: deposition on its slab, the distributed
    Biot-Savart and the statistics.  params: api.Params of the whole grid (deposit_mode 0).
    Returns a dict with the slab fields (raw), E(k) of omega and of u (normalised), u',
    Etot/u'^2, the enstrophy and S_p at the reference separations."""
    import torch

    from .api import Context, sp_separations

    N, R = params.N, comm.world
    if N % (8 * R) or N % R:
        raise ValueError("the grid must split into whole 8-plane slabs: N divisible by 8 R")
    nz = N // R
    ctx = Context(params)
    ctx.set_slab(comm.rank * nz, nz)
    ctx.set_centerlines(npoint, xyz, sigma, Gamma, n_T)
    ctx.deposit()
    w = ctx.field_tensor(0)

    def block(P, y0, ny):
        return ctx.biot_savart_block(P.data_ptr(), y0, ny)

    u, shw, shu, E, Z = spectral_velocity(comm, w, N, block)
    up = math.sqrt(2.0 * E / 3.0)
    r = sp_separations(N)

    def sp(box, n0, n1, n2, axis):
        return ctx.sp_block(box.data_ptr(), n0, n1, n2, axis, 1.0 / up, r)

    Sp = structure_function_sums(comm, u, N, 1.0 / up, r, sp)
    out = {"w": w.clone(), "u": u, "spectrum_vor": shw, "spectrum": shu / (up * up), "up": up,
           "Etot": E / (up * up), "Enstrophy": Z / (up * up), "Sp_r": r, "Sp": Sp}
    ctx.close()
    torch.cuda.synchronize()
    return out


def main(argv=None):
    import argparse
    import datetime
    import json
    import os

    import torch
    import torch.distributed as dist

    from .api import Params
    from .configs import CONFIGS, build_workload

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="cfg1")
    ap.add_argument("--precision", type=int, default=32)
    args = ap.parse_args(argv)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    comm = TorchComm(device=torch.device("cuda", local))
    w = CONFIGS[args.config](seed=0)
    prm = Params(N=w.N, N_downsample=w.N, line_s=1, line_e=w.ntubes, sigma_ratio=w.sigma_ratio, eta_t=w.eta_t,
                 ntf_times=w.ntf_times, ntf_pre=w.ntf_pre, Rtube_ratio=w.Rtube_ratio, dzeta_sup=w.dzeta_sup,
                 precision=args.precision, deposit_mode=0, device=local)
    from .api import Context
    gen = Context(prm)
    xyz, (npoint, sig, gam, nT) = build_workload(gen, w)
    host = xyz.T.contiguous().cpu().numpy()
    gen.close()
    out = build_field(comm, prm, npoint, host, sig, gam, nT, device=local)
    if comm.rank == 0:
        print(json.dumps({"config": w.name, "ranks": comm.world, "up": out["up"], "Enstrophy": out["Enstrophy"],
                          "spectrum_u_first": out["spectrum"][:4].tolist(), "S2": out["Sp"][1].tolist()}))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
