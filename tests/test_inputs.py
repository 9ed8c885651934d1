"""Input-file validation on the host (fwt_check_inputs, no GPU): the reference's own input pair
reads back with its counts and scalars, and every kind of malformed file is refused with an
error that names the fault instead of reaching the device.
"""
import os

import pytest

from test_golden import write_reference_inputs, wt2_inputs


@pytest.fixture()
def rundir(orc, tmp_path):
    p, cl = wt2_inputs(orc)
    write_reference_inputs(str(tmp_path), p, cl, N=64)
    return tmp_path


def _lines(path):
    return open(path).read().splitlines(keepends=True)


def _write(path, lines):
    with open(path, "w") as f:
        f.writelines(lines)


def test_reference_inputs_read_back(fwt, rundir):
    p, nline, nodes = fwt.api.check_inputs(rundir)
    assert nline == 73 and nodes == 73 * 148
    assert p["N"] == 64 and p["N_downsample"] == 64 and p["ntf_times"] == 50 and p["ntf_pre"] == 1000
    assert p["sigma_ratio"] == 4.0 and p["Rtube_ratio"] == 3.0 and p["line_s"] == 1 and p["line_e"] == 73


def _expect(fwt, rundir, fragment):
    with pytest.raises(fwt.FwtError) as e:
        fwt.api.check_inputs(rundir)
    assert fragment in str(e.value), str(e.value)


def test_truncated_centerline_file(fwt, rundir):
    f = os.path.join(rundir, "centerline_input.dat")
    _write(f, _lines(f)[:-5])
    _expect(fwt, rundir, "truncated node list")


def test_non_finite_coordinate(fwt, rundir):
    f = os.path.join(rundir, "centerline_input.dat")
    L = _lines(f)
    L[80] = "  NaN  0.0  0.0\n"
    _write(f, L)
    _expect(fwt, rundir, "non-finite coordinate")


def test_line_with_one_node(fwt, rundir):
    f = os.path.join(rundir, "centerline_input.dat")
    L = _lines(f)
    L[1] = "1\n"
    _write(f, L)
    _expect(fwt, rundir, "need >= 2")


def test_bad_line_count(fwt, rundir):
    f = os.path.join(rundir, "centerline_input.dat")
    L = _lines(f)
    L[0] = "-3\n"
    _write(f, L)
    _expect(fwt, rundir, "bad nline")


def test_non_numeric_parameter(fwt, rundir):
    f = os.path.join(rundir, "parameters_input.dat")
    L = _lines(f)
    L[1] = "sixty-four\n"
    _write(f, L)
    _expect(fwt, rundir, "bad value on line 2")


def test_missing_line_rows(fwt, rundir):
    f = os.path.join(rundir, "parameters_input.dat")
    _write(f, _lines(f)[:-3])
    _expect(fwt, rundir, "fewer line rows than nline")


def test_duplicate_line_row_leaves_one_missing(fwt, rundir):
    f = os.path.join(rundir, "parameters_input.dat")
    L = _lines(f)
    L[-1] = L[-2]
    _write(f, L)
    _expect(fwt, rundir, "missing row for line 73")


def test_downsample_must_divide_N(fwt, rundir):
    f = os.path.join(rundir, "parameters_input.dat")
    L = _lines(f)
    L[3] = "      48\n"
    _write(f, L)
    _expect(fwt, rundir, "N_downsample must divide N")


def test_line_range_outside_the_lines(fwt, rundir):
    f = os.path.join(rundir, "parameters_input.dat")
    L = _lines(f)
    L[7] = "      99\n"
    _write(f, L)
    _expect(fwt, rundir, "line_s..line_e")


def test_missing_file(fwt, tmp_path):
    _expect(fwt, tmp_path, "cannot open")
