"""State files and VTU output (af_io_*; host code, no GPU)."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from atmospheric_flows_b200 import mesh as M


def _fields(m, P, seed=4):
    rng = np.random.default_rng(seed)
    n = m.n_cells * (P + 1) ** 2
    return rng.standard_normal(n), rng.standard_normal(2 * n), rng.standard_normal(n)


@pytest.mark.parametrize("periodic", [False, True])
def test_state_round_trip_is_bit_exact(tmp_path, periodic):
    from atmospheric_flows_b200 import io
    m = M.jitter_mesh(M.hill_mesh(7, 3, periodic_x=periodic), 0.1, seed=2)
    P = 3
    rho, u, p = _fields(m, P)
    f = tmp_path / "state.af"
    io.write_state(f, m, P, rho, u, p, time=12.5, step=25)
    m2, P2, t, step, r2, u2, p2 = io.read_state(f)
    assert (P2, t, step, m2.nx, m2.nz, m2.periodic_x) == (P, 12.5, 25, 7, 3, periodic)
    assert np.array_equal(m2.vertices, m.vertices)
    assert np.array_equal(r2, rho) and np.array_equal(u2, u) and np.array_equal(p2, p)


def test_state_read_rejects_other_files(tmp_path):
    from atmospheric_flows_b200 import io
    from atmospheric_flows_b200.operator import AFError
    f = tmp_path / "junk.bin"
    f.write_bytes(b"not a state file at all")
    with pytest.raises(AFError):
        io.read_state(f)


def _parse(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arr = {}
    for da in root.iter("DataArray"):
        name = da.get("Name") or "points"
        arr[name] = np.array(da.text.split(), dtype=float)
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), arr


@pytest.mark.parametrize("P", [1, 2, 4])
def test_vtu_patches_interpolate_polynomials_exactly(tmp_path, P):
    """On an affine mesh a field of degree <= P is reproduced at the equispaced patch points."""
    from atmospheric_flows_b200 import io
    m = M.box_mesh(3, 2, 0.0, 3.0, 0.0, 2.0)
    xz = M.dof_coordinates(m, P)  # (ncell, nd, 2)
    f = lambda x, z: 1.0 + 0.5 * x ** P - 0.25 * z ** P + 0.1 * x * z
    rho = f(xz[..., 0], xz[..., 1]).ravel()
    u = np.stack([xz[..., 0], -xz[..., 1]], axis=1).ravel()  # component-blocked per cell
    p = 2.0 * rho
    out = tmp_path / "sol.vtu"
    io.write_vtu(out, m, P, rho, u, p)
    npts, ncells, arr = _parse(out)
    assert npts == m.n_cells * (P + 1) ** 2 and ncells == m.n_cells * P * P
    pts = arr["points"].reshape(-1, 3)
    assert np.allclose(arr["rho"], f(pts[:, 0], pts[:, 1]), atol=1e-12)
    assert np.allclose(arr["p"], 2.0 * arr["rho"], atol=1e-12)
    uu = arr["u"].reshape(-1, 3)
    assert np.allclose(uu[:, 0], pts[:, 0], atol=1e-12) and np.allclose(uu[:, 1], -pts[:, 1], atol=1e-12)
    assert np.all(arr["types"] == 9) and arr["connectivity"].max() == npts - 1
    # each cell's corner points are its mesh vertices
    assert np.allclose(pts[0, :2], m.vertices[0, 0]) and np.allclose(pts[P, :2], m.vertices[0, 1])
