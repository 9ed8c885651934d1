"""Generate the committed golden fixtures under tests/golden/ (run once, in a checkout that has
the reference next to it; the tests only read the .npz files this writes).

Fixtures:

* ``wt2_inputs.npz`` -- the reference's own shipped input pair, ``centerline_input.dat``
  (73 closed tubes x 148 nodes) and ``parameters_input.dat`` (sigma_ratio 4, n_T 1/2/4,
  N 256), parsed into arrays.  It is the end-to-end fixture with the general deposition
  branch (varying core, twisted tubes).
* ``wt2_n64_oracle.npz`` -- the FP64 oracle's outputs on that input with N edited to 64:
  per-section ntf of three lines, per-line maximum ntf and accepted (point, sub-segment)
  pairs, E(k) of omega and of u, the normalisation scalars, integer PDF counts, S_p(r), and omega sampled every 4th point.
* ``gaussian_pdf_table.npz`` -- every 50th row of the reference's tabulated standard normal
  density (``output/stat/pdf_um_gau.dat``, 10000 rows on [-5, 5]), the known answer its
  plotting scripts compare the u-PDF with.

Usage:  python tests/golden/make_golden.py [reference_dir]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def main(ref):
    O.build()
    cl = O.read_centerlines(os.path.join(ref, "centerline_input.dat"))
    p = O.read_parameters(os.path.join(ref, "parameters_input.dat"), len(cl.npoint))
    np.savez_compressed(
        os.path.join(HERE, "wt2_inputs.npz"), npoint=cl.npoint, xyz=cl.xyz, sigma=p.sigma, Gamma=p.Gamma,
        n_T=p.n_T, if_filter=p.if_filter,
        scalars=np.array([p.N, p.N_downsample, p.line_s, p.line_e, p.sigma_ratio, p.eta_t, p.ntf_times, p.ntf_pre,
                          p.Rtube_ratio, p.dzeta_sup]))

    p.N = p.N_downsample = 64
    out = O.run(p, cl, sp_pmax=10)
    ntf = {f"ntf_line{i + 1}": O.line_ntf(cl.line(i), p.ntf_times, p.ntf_pre)[0] for i in (0, 1, 72)}
    ntf_max = np.array([row[3] for row in out["line_info"]], dtype=np.int64)
    accepted = np.array([row[4] for row in out["line_info"]], dtype=np.int64)
    np.savez_compressed(
        os.path.join(HERE, "wt2_n64_oracle.npz"), **ntf, ntf_max=ntf_max, accepted=accepted,
        spectrum_vor=out["spectrum_vor"], spectrum=out["spectrum"], scalars=np.array([out["up"], out["Etot"], out["Enstrophy"]]),
        pdf_u_counts=out["pdf_u"][2], pdf_u_val=out["pdf_u"][0], pdf_w_counts=out["pdf_w"][2],
        Sp_r=out["Sp_r"], Sp=out["Sp"], vor_sample=out["vor"][:, ::4, ::4, ::4].copy())

    tab = np.loadtxt(os.path.join(ref, "output", "stat", "pdf_um_gau.dat"))
    np.savez_compressed(os.path.join(HERE, "gaussian_pdf_table.npz"), table=tab[::50].copy())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
