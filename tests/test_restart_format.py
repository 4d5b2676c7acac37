"""The reference's restart file on the CPU: the library's writer and reader
(lbm_write_flow_field_file / lbm_read_flow_field_file) against a Python
restatement of saveflowfield's WRITE statements (solution.f90:1646-1672)
under nvfortran form='binary' (no record markers, native byte order), on a
small grid with two wings. The handle-based save and restart are GPU tests
(test_gpu_io.py)."""
import struct

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import io_formats

NX, NY, NW = 7, 5, 2


def reference_bytes(cycle, body, movenum, u, v, f, f0_edges, f2_edges):
    """saveflowfield (solution.f90:1649-1672) for one mesh, 0-based arrays:
    u, v (ny, nx), f (9, ny, nx); edges as dicts 'left', 'right' (ny, 9) and
    'up', 'down' (nx, 9) for f0 and for the f2 copies."""
    ny, nx = u.shape
    out = [struct.pack("<i", cycle), struct.pack("<i", body.shape[1])]
    out.append(struct.pack(f"<{body.size}d", *body.reshape(-1)))   # 11 arrays, each 1:wing_count
    out.append(struct.pack("<i", movenum))
    for j in range(ny):                       # do j=1,Ny; do i=1,Nx
        for i in range(nx):
            out.append(struct.pack("<11d", u[j, i], v[j, i], *f[:, j, i]))
    for j in range(1, ny - 1):                # do j=2,Ny-1
        out.append(struct.pack("<9d", *f2_edges["left"][j]))
        out.append(struct.pack("<9d", *f0_edges["left"][j]))
        out.append(struct.pack("<9d", *f2_edges["right"][j]))
        out.append(struct.pack("<9d", *f0_edges["right"][j]))
    for i in range(nx):                       # do j=1,Nx
        out.append(struct.pack("<9d", *f2_edges["up"][i]))
        out.append(struct.pack("<9d", *f0_edges["up"][i]))
        out.append(struct.pack("<9d", *f2_edges["down"][i]))
        out.append(struct.pack("<9d", *f0_edges["down"][i]))
    return b"".join(out)


def random_state(seed=5):
    rng = np.random.default_rng(seed)
    u, v = rng.normal(size=(NY, NX)), rng.normal(size=(NY, NX))
    f = rng.normal(size=(9, NY, NX))
    f0 = {"left": rng.normal(size=(NY, 9)), "right": rng.normal(size=(NY, 9)),
          "down": rng.normal(size=(NX, 9)), "up": rng.normal(size=(NX, 9))}
    # the corner nodes are one node each
    f0["left"][0], f0["left"][-1] = f0["down"][0], f0["up"][0]
    f0["right"][0], f0["right"][-1] = f0["down"][-1], f0["up"][-1]
    return u, v, f, f0


def edge_array(f0):
    """The library's edge_f0 layout: left column, right column, bottom row, top row."""
    return np.concatenate([f0["left"], f0["right"], f0["down"], f0["up"]])


def test_writer_matches_the_reference_layout(tmp_path):
    u, v, f, f0 = random_state()
    body = np.arange(11 * NW, dtype=np.float64).reshape(11, NW) * 0.25 - 1.0
    p = tmp_path / "saved_flow_feild.dat"
    io_formats.write_flow_field_file(p, 100000, u, v, f, edge_array(f0), body_state=body, movenum=-3)
    # on the one-mesh path leftf2 .. downf2 equal the edge f0 (solution.f90:60-63)
    want = reference_bytes(100000, body, -3, u, v, f, f0, f0)
    got = p.read_bytes()
    assert len(got) == len(want) == 12 + 88 * NW + 88 * NX * NY + 288 * (NY - 2 + NX)
    assert got == want


def test_writer_zero_body_state(tmp_path):
    u, v, f, f0 = random_state(6)
    p = tmp_path / "r.dat"
    io_formats.write_flow_field_file(p, 7, u, v, f, edge_array(f0))
    assert p.read_bytes() == reference_bytes(7, np.zeros((11, 0)), 0, u, v, f, f0, f0)


def test_reader_takes_the_reference_file_apart(tmp_path):
    u, v, f, f0 = random_state(7)
    f2 = {k: x + 100.0 for k, x in f0.items()}   # distinct f2 copies: the reader must take f0
    body = np.linspace(-1, 1, 11 * NW).reshape(11, NW)
    p = tmp_path / "saved_flow_feild.dat"
    p.write_bytes(reference_bytes(200000, body, 4, u, v, f, f0, f2))
    r = io_formats.read_flow_field_file(p, NX, NY, NW)
    assert r["cycle"] == 200000 and r["movenum"] == 4
    np.testing.assert_array_equal(r["body_state"], body)
    np.testing.assert_array_equal(r["u"], u)
    np.testing.assert_array_equal(r["v"], v)
    np.testing.assert_array_equal(r["f"], f)
    np.testing.assert_array_equal(r["edge_f0"], edge_array(f0))


def test_reader_refusals(tmp_path):
    u, v, f, f0 = random_state(8)
    body = np.zeros((11, NW))
    data = reference_bytes(3, body, 0, u, v, f, f0, f0)
    p = tmp_path / "a.dat"
    p.write_bytes(data[:-8])                                    # short: end= in the reference
    with pytest.raises(IOError, match="LBM_ERR_IO"):
        io_formats.read_flow_field_file(p, NX, NY, NW)
    p.write_bytes(data)
    with pytest.raises(IOError, match="LBM_ERR_STATE"):      # wing count of another build: the reference stops
        io_formats.read_flow_field_file(p, NX, NY, 1)
    with pytest.raises(IOError, match="LBM_ERR_IO"):          # another grid
        io_formats.read_flow_field_file(p, NX + 1, NY, NW)
    with pytest.raises(IOError, match="LBM_ERR_IO"):
        io_formats.read_flow_field_file(tmp_path / "missing.dat", NX, NY, NW)
    assert io_formats.read_flow_field_file(p, NX, NY, NW)["cycle"] == 3
