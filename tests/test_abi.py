"""The C-ABI boundary (CPU only: nothing here launches a kernel).

libfwt.so must export every entry point include/fwt.h declares, the ctypes mirror of
fwt_params must have the C struct's layout (checked against a program compiled from the
header), host-only entry points must agree with the oracle, and on a machine without a GPU
fwt_create must fail loudly instead of falling back to a CPU path.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fwt.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(fwt_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("fwt_create", "fwt_destroy", "fwt_load_inputs", "fwt_set_centerlines", "fwt_deposit",
                 "fwt_filter", "fwt_biot_savart", "fwt_normalize", "fwt_spectrum", "fwt_pdf", "fwt_pdf_noalloc",
                 "fwt_sp", "fwt_write_outputs", "fwt_copy_field", "fwt_run_dir", "fwt_last_error"):
        assert must in names


def test_every_entry_point_is_documented_for_integrators():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    undocumented = [n for n in declared_functions() if n not in doc]
    assert not undocumented, undocumented


def test_library_exports_every_declared_symbol(fwt):
    L = fwt.library()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(fwt.api.EXPORTS) == declared_functions()


def test_params_layout_matches_the_header(fwt, tmp_path):
    fields = [f for f, _ in fwt.api._Params._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "fwt.h"', "int main(void) {",
            '  printf("%zu\\n", sizeof(fwt_params));']
    prog += [f'  printf("%zu\\n", offsetof(fwt_params, {f}));' for f in fields]
    prog += ["  return 0; }"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(fwt.api._Params)
    for f, off in zip(fields, out[1:]):
        assert getattr(fwt.api._Params, f).offset == off, f


def test_default_params_are_the_reference_defaults(fwt):
    p = fwt.api._Params()
    assert fwt.library().fwt_default_params(ctypes.byref(p)) == 0
    assert (p.ntf_times, p.ntf_pre, p.Rtube_ratio, p.dzeta_sup) == (50, 1000, 3.0, 1e-4)
    assert (p.if_pdf, p.if_Sp, p.Sp_order, p.pdf_bins, p.vorticity_output) == (1, 1, 10, 1000, 1)
    assert p.precision == 32 and p.deposit_mode == 0


def test_fbb_signs_match_the_oracle(fwt, orc):
    s = fwt.fbb_signs(12345, 257)
    want = [orc.fbb_sign(12345, t) for t in range(257)]
    assert list(s) == want
    assert 0.35 < np.mean(np.asarray(s) > 0) < 0.65


def test_errors_are_codes_with_messages(fwt):
    L = fwt.library()
    assert L.fwt_fbb_signs(ctypes.c_uint64(0), -1, None) == -1   # FWT_E_ARG
    buf = ctypes.create_string_buffer(256)
    L.fwt_last_error(buf, 256)
    assert buf.value
    assert L.fwt_default_params(None) == -1


def test_sp_separations_match_the_oracle(fwt, orc):
    for N in (32, 64, 96, 256, 1024):
        assert list(fwt.sp_separations(N)) == list(orc.sp_separations(N))


def test_create_fails_loudly_without_a_gpu(fwt):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fwt.FwtError) as e:
        fwt.Context(fwt.Params(N=16, N_downsample=16))
    assert e.value.code == -2       # FWT_E_CUDA: no CPU fallback


def test_sp_exponents_match_the_oracle(fwt, orc):
    """zeta_p and flatness of the reference's post-processing, through the C-ABI, on a
    synthetic table with known exponents S_p = c_p r^{p/3 + d_p}."""
    r = fwt.sp_separations(256).astype(np.float64) * (2 * np.pi / 256)
    p = np.arange(1, 11)[:, None]
    want = p[:, 0] / 3.0 + 0.01 * (p[:, 0] - 3) ** 2
    Sp = (0.5 + 0.1 * p) * r[None, :] ** want[:, None]
    Sp[2] *= -1.0                          # odd orders may be negative; the fit uses |S_p|
    zeta, flat = fwt.sp_exponents(r, Sp)
    z_o, f_o = orc.sp_exponents(r, Sp)
    np.testing.assert_allclose(zeta, want, rtol=1e-12)
    np.testing.assert_allclose(zeta, z_o, rtol=1e-12)
    np.testing.assert_allclose(flat, f_o, rtol=1e-14)
    with pytest.raises(fwt.FwtError):
        fwt.sp_exponents(r[:8], Sp[:, :8])
