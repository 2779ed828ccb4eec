"""Reference file formats on the host: Mesh3d.dat (unformatted and text), wall_dist.dat,
flow3d.dat / SA3d.dat / SST3d.dat / Step_mess.dat round trips and conversions."""
import os
import struct

import numpy as np


def test_mesh3d_roundtrip_and_record_layout(tmp_path):
    from ocfd_b200 import cases
    from ocfd_b200.formats import case_from_files, read_mesh3d, write_mesh3d
    from ocfd_b200.connectivity import write_bc3d_inp
    p, case = cases.config2_small()
    path = str(tmp_path / "Mesh3d.dat")
    write_mesh3d(path, case.xyz)
    with open(path, "rb") as f:
        n, nb, n2 = struct.unpack("<iii", f.read(12))
    assert n == n2 == 4 and nb == len(case.xyz)          # first record: the block count
    back = read_mesh3d(path)
    assert all(np.array_equal(a, b) for a, b in zip(back, case.xyz))
    tpath = str(tmp_path / "Mesh3d_text.dat")
    write_mesh3d(tpath, case.xyz, formatted=True)
    assert all(np.array_equal(a, b) for a, b in zip(read_mesh3d(tpath, formatted=True), case.xyz))
    write_bc3d_inp(str(tmp_path / "bc3d.inp"), case.inp)
    c2 = case_from_files(path, str(tmp_path / "bc3d.inp"))
    assert c2.inc == case.inc and c2.dims == case.dims


def test_wall_dist_roundtrip(tmp_path):
    from ocfd_b200.formats import read_wall_dist, write_wall_dist
    rng = np.random.default_rng(3)
    dims = [(9, 7, 5), (4, 6, 3)]
    dw = [rng.random((nz - 1, ny - 1, nx - 1)) for nx, ny, nz in dims]
    write_wall_dist(str(tmp_path / "wall_dist.dat"), dw)
    assert all(np.array_equal(a, b) for a, b in zip(read_wall_dist(str(tmp_path / "wall_dist.dat"), dims), dw))


def test_flow_files_roundtrip(tmp_path):
    """write_flow -> read_flow reproduces the state on cells 0..n up to the primitive round trip
    (rounding of d*(m/d)), and fills the outer ghosts with the reference's allocation values."""
    from ocfd_b200 import cases
    from ocfd_b200.formats import read_flow, write_flow
    for turb, nv in ((0, 5), (2, 6), (3, 7)):
        p, case = cases.airfoil(ni=33, nj=9, turb=turb)
        rng = np.random.default_rng(turb)
        states = []
        for nx, ny, nz in case.dims:
            U = np.empty((nz + 7, ny + 7, nx + 7, nv))
            d = rng.uniform(0.5, 1.5, U.shape[:3])
            U[..., 0] = d
            U[..., 1:4] = d[..., None] * rng.uniform(-1, 1, U.shape[:3] + (3,))
            U[..., 4] = rng.uniform(2.0, 3.0, U.shape[:3])
            for m in range(5, nv):
                U[..., m] = rng.uniform(0, 1, U.shape[:3])
            states.append(U)
        write_flow(str(tmp_path), states, p, kstep=1234, tt=5.5)
        back, kstep, tt = read_flow(str(tmp_path), case.dims, p)
        assert kstep == 1234 and tt == 5.5
        for U, V in zip(states, back):
            inner = (slice(3, -3),) * 3
            np.testing.assert_allclose(V[inner], U[inner], rtol=1e-13, atol=1e-15)
            assert np.all(V[0, :, :, 0] == 1.0) and np.all(V[0, :, :, 1:4] == 0.0) and np.all(V[0, :, :, 4] == 1.0)
        for f in ("SA3d.dat", "SST3d.dat"):
            if os.path.exists(str(tmp_path / f)):
                os.remove(str(tmp_path / f))
