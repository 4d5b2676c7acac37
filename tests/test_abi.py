"""The C-ABI library without a GPU: it loads, exports every symbol that
include/lbm_b200.h declares, rejects bad input, and its host-side file
parsers read the reference's text formats."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import _abi, build, cases, io_formats


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _abi.load_library()


def test_library_exports_every_declared_symbol(lib):
    declared = _abi.header_declarations()
    assert len(declared) >= 20
    assert set(declared) == set(_abi.ABI), "ctypes table and header disagree"
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = set(declared) - exported
    assert not missing, missing
    assert all(name.startswith("lbm_") for name in exported), "library leaks non-ABI symbols"


def test_library_is_built_for_sm100a():
    """Every source is compiled and linked for sm_100a only (the GPU tests
    also ask the loaded kernels: lbm_device_check)."""
    flags = build.NVCC_FLAGS
    i = flags.index("-gencode")
    assert flags[i + 1] == "arch=compute_100a,code=sm_100a"
    assert flags.count("-gencode") == 1


def test_status_words_decode_to_codes_and_kernel_names(lib):
    """The device status word the kernels set becomes the call's status code
    and message (host logic, no device): an index error names every kernel
    that skipped an access and comes before the other errors."""
    buf = C.create_string_buffer(256)
    assert lib.lbm_describe_status(0, buf, 256) == _abi.LBM_OK and buf.value == b""
    for bit, kernel in _abi.LBM_ST_INDEX_KERNELS.items():
        assert lib.lbm_describe_status(bit | _abi.LBM_ST_SOLVER, buf, 256) == _abi.LBM_ERR_INDEX
        assert buf.value.decode().split(":")[-1].split() == [kernel]
    both = 0x4000 | 0x8000
    assert lib.lbm_describe_status(both, buf, 256) == _abi.LBM_ERR_INDEX
    assert buf.value.decode().split(":")[-1].split() == ["ib_tile_update", "ib_forces"]
    assert lib.lbm_describe_status(_abi.LBM_ST_RANGE, buf, 256) == _abi.LBM_ERR_RANGE
    assert lib.lbm_describe_status(_abi.LBM_ST_OVERFLOW, buf, 256) == _abi.LBM_ERR_RANGE
    assert lib.lbm_describe_status(_abi.LBM_ST_SOLVER, buf, 256) == _abi.LBM_ERR_SOLVER
    assert lib.lbm_describe_status(_abi.LBM_ST_NONFINITE, buf, 256) == _abi.LBM_ERR_NONFINITE
    assert lib.lbm_describe_status(_abi.LBM_ST_TIMEOUT, buf, 256) == _abi.LBM_ERR_CUDA
    # a short buffer gets a terminated prefix; a null buffer only the code
    small = C.create_string_buffer(8)
    assert lib.lbm_describe_status(0x100, small, 8) == _abi.LBM_ERR_INDEX
    assert len(small.value) == 7
    assert lib.lbm_describe_status(0x100, None, 0) == _abi.LBM_ERR_INDEX


def test_default_params_are_the_reference_parameters(lib):
    p = _abi.LbmParams()
    assert lib.lbm_default_params(C.byref(p)) == 0
    assert (p.nx, p.ny, p.wing_count, p.points_per_wing) == (4001, 2001, 2, 205)
    assert (p.uu, p.re, p.scale) == (0.01, 500.0, 0.01)
    assert list(p.s)[:7] == [0.0, 1.1, 1.05, 0.0, 1.2, 0.0, 1.2]
    assert p.delta_kernel == _abi.LBM_DELTA_SMOOTH


def test_create_rejects_bad_parameters(lib):
    p = cases.make_params(64, 64, 16, (20, 32), 0.05, 100.0)
    p.nx = 4
    h = C.c_void_p()
    assert lib.lbm_create(C.byref(p), C.byref(h)) == _abi.LBM_ERR_ARG
    p = cases.make_params(64, 64, 16, (20, 32), 0.05, 100.0)
    p.precision = 9
    assert lib.lbm_create(C.byref(p), C.byref(h)) == _abi.LBM_ERR_ARG
    assert lib.lbm_create(None, C.byref(h)) == _abi.LBM_ERR_ARG
    assert lib.lbm_destroy(None) == _abi.LBM_ERR_ARG
    assert lib.lbm_last_error(None)


def test_create_without_device_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = cases.make_params(64, 64, 16, (20, 32), 0.05, 100.0)
    h = C.c_void_p()
    assert lib.lbm_create(C.byref(p), C.byref(h)) == _abi.LBM_ERR_CUDA
    assert not h.value


def test_boundary_file_round_trip(lib, tmp_path):
    x, y = cases.naca0012(160)
    path = tmp_path / "boundary.dat"
    io_formats.write_boundary(path, x, y)
    line = open(path).readline()
    assert len(line.rstrip("\n")) == 28          # (2f14.8)
    rx, ry = io_formats.parse_boundary(str(path), len(x), lib)
    np.testing.assert_array_equal(rx, x)
    np.testing.assert_array_equal(ry, y)


def test_boundary_parser_errors(lib, tmp_path):
    p = tmp_path / "b.dat"
    p.write_text("   0.10000000   0.20000000\n")
    with pytest.raises(IOError):
        io_formats.parse_boundary(str(p), 5, lib)            # too few records
    p.write_text("abc def\n")
    with pytest.raises(IOError):
        io_formats.parse_boundary(str(p), 1, lib)            # not numbers
    with pytest.raises(IOError):
        io_formats.parse_boundary(str(tmp_path / "missing.dat"), 1, lib)


def test_motion_file_round_trip_and_blank_lines(lib, tmp_path):
    table = cases.plunge_pitch_table(50, 6.25e-4, heave=0.25, pitch_deg=10, freq=0.6)
    p = tmp_path / "motion_params.dat"
    io_formats.write_motion(p, table)
    with open(p, "a") as fh:
        fh.write("\n   \n")
    back = io_formats.parse_motion(str(p), table.shape[1], lib)
    np.testing.assert_array_equal(back, table)
    # Fortran D exponents and commas are list-directed input too
    p.write_text("0.0d0, 1.5D-1 2 3 4 5 6 7 8 9\n")
    np.testing.assert_allclose(io_formats.parse_motion(str(p), 10, lib)[0], [0, 0.15, 2, 3, 4, 5, 6, 7, 8, 9])


def test_motion_parser_errors(lib, tmp_path):
    p = tmp_path / "m.dat"
    p.write_text("")
    with pytest.raises(IOError):
        io_formats.parse_motion(str(p), 10, lib)             # empty (mode.f90:101-104)
    p.write_text("0.0 1.0 2.0\n")
    with pytest.raises(IOError):
        io_formats.parse_motion(str(p), 10, lib)             # short row (mode.f90:94-97)


def test_force_row_format():
    s = io_formats.format_force_row([0.0125, -1.23456789, 12.5])
    assert s == "     0.01250000    -1.23456789    12.50000000"


def test_fortran_interfaces_name_declared_entry_points():
    """Every bind(C, name=...) of the Fortran interfaces in INTEGRATION.md
    names an entry point the header declares (a maintainer who pastes them
    binds symbols that exist)."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "lbm_b200.h")).read()
    declared = set(re.findall(r"LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", header))
    doc = open(os.path.join(root, "INTEGRATION.md")).read()
    bound = set(re.findall(r"bind\(C,\s*name='(lbm_\w+)'\)", doc))
    assert bound, "no Fortran interfaces found"
    assert bound <= declared, sorted(bound - declared)
