"""The reference's mesh, wall-distance and flow files, read and written on the host.

* ``Mesh3d.dat``     read_main_mesh (sub_IO.f90:4-93): block count, the (nx, ny, nz) of every
  block, then per block x(1:nx,1:ny,1:nz), y, z; Fortran unformatted sequential (default) or
  list-directed text (Mesh_File_Format = 1).
* ``wall_dist.dat``  read_dw (sub_IO.f90:97-161): per block dw(1:nx-1, 1:ny-1, 1:nz-1).
* ``flow3d.dat``     output_flow / read_flow_data (sub_IO.f90:350-484, 171-338): per block the
  primitive variables d, u, v, w, T on cells 0..nx x 0..ny x 0..nz; ``SA3d.dat`` holds U6 and
  ``SST3d.dat`` U6, U7 on the same cells; ``Step_mess.dat`` the step counter and time.

Unformatted files use the gfortran record layout: each record framed by 4-byte little-endian
lengths (records of more than 2**31-9 bytes, which gfortran splits into subrecords, are refused
with an error).  Together with
``connectivity.read_bc3d_inp`` / ``convert_inp_inc`` this lets a host program ingest a case and
restart from, or write, the reference's flow files without the Fortran code.
"""
import os
import struct

import numpy as np

from .meshgen import Case

_MAXREC = 2 ** 31 - 9


# ---- Fortran sequential records ----------------------------------------------------------
def _write_record(f, payload: bytes):
    n = len(payload)
    if n > _MAXREC:
        raise ValueError("record of %d bytes: longer than one Fortran record (split the block)" % n)
    f.write(struct.pack("<i", n))
    f.write(payload)
    f.write(struct.pack("<i", n))


def _read_record(f) -> bytes:
    hdr = f.read(4)
    if len(hdr) < 4:
        raise EOFError("unexpected end of Fortran unformatted file")
    n = struct.unpack("<i", hdr)[0]
    if n < 0:
        raise ValueError("Fortran subrecords (records over 2 GiB) are not supported")
    data = f.read(n)
    if struct.unpack("<i", f.read(4))[0] != n:
        raise ValueError("corrupt Fortran record markers")
    return data


def _fortran(a):
    """Array (k, j, i) C order -> bytes of the Fortran array (i fastest)."""
    return np.ascontiguousarray(a, dtype="<f8").tobytes()


# ---- Mesh3d.dat --------------------------------------------------------------------------
def write_mesh3d(path, xyz, formatted=False):
    """xyz: per block (3, nz, ny, nx) node coordinates."""
    dims = [(a.shape[3], a.shape[2], a.shape[1]) for a in xyz]
    if formatted:
        with open(path, "w") as f:
            f.write("%d\n" % len(dims))
            f.write(" ".join("%d %d %d" % d for d in dims) + "\n")
            for a in xyz:
                for c in range(3):
                    np.savetxt(f, a[c].reshape(-1), fmt="%.17e")
        return
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<i", len(dims)))
        _write_record(f, np.array(dims, dtype="<i4").tobytes())
        for a in xyz:
            _write_record(f, b"".join(_fortran(a[c]) for c in range(3)))


def read_mesh3d(path, formatted=False):
    """Returns the per-block node coordinates, each (3, nz, ny, nx) float64."""
    if formatted:
        with open(path) as f:
            toks = f.read().split()
        nb = int(toks[0])
        dims = [tuple(int(v) for v in toks[1 + 3 * q:4 + 3 * q]) for q in range(nb)]
        vals = np.array(toks[1 + 3 * nb:], dtype=np.float64)
        out, o = [], 0
        for nx, ny, nz in dims:
            n = nx * ny * nz
            out.append(vals[o:o + 3 * n].reshape(3, nz, ny, nx).copy())
            o += 3 * n
        return out
    with open(path, "rb") as f:
        nb = struct.unpack("<i", _read_record(f))[0]
        dims = np.frombuffer(_read_record(f), dtype="<i4").reshape(nb, 3)
        out = []
        for nx, ny, nz in dims:
            a = np.frombuffer(_read_record(f), dtype="<f8")
            out.append(a.reshape(3, nz, ny, nx).copy())
    return out


def case_from_files(mesh_path, inp_path, name=None, formatted=False):
    """A Case (mesh + connectivity) from the reference's Mesh3d.dat and bc3d.inp."""
    from .connectivity import read_bc3d_inp
    xyz = read_mesh3d(mesh_path, formatted)
    inp = read_bc3d_inp(inp_path)
    if [(b.nx, b.ny, b.nz) for b in inp] != [(a.shape[3], a.shape[2], a.shape[1]) for a in xyz]:
        raise ValueError("block sizes in %s and %s differ" % (mesh_path, inp_path))
    return Case(name or os.path.basename(os.path.dirname(os.path.abspath(mesh_path))), xyz, inp)


# ---- bc3d.inc ------------------------------------------------------------------------------
def write_bc3d_inc(path, case):
    """bc3d.inc as convert_inp_inc writes it (sub_convert_inp.f90:103-114) and read_inc reads it
    (sub_IO.f90:656-743): a title line, the block count, then per block its node counts, a label
    line, its subface count and per subface the 9 + 12 integers of the .inc record."""
    nijk, _, nsub, inc = case.flat()
    rec = np.asarray(inc).reshape(-1, 21)
    with open(path, "w") as f:
        f.write(" Inp-liked file of OpenCFD-EC\n")
        f.write(" %d\n" % len(case.dims))
        t = 0
        for b, (nx, ny, nz) in enumerate(case.dims):
            f.write(" %d %d %d\n" % (nx, ny, nz))
            f.write(" Block %d\n" % (b + 1))
            f.write(" %d\n" % nsub[b])
            for _ in range(nsub[b]):
                f.write("".join("%6d" % v for v in rec[t, :9]) + "\n")
                f.write("".join("%6d" % v for v in rec[t, 9:]) + "\n")
                t += 1


def write_case_files(directory, case, formatted=False):
    """Mesh3d.dat and bc3d.inc of a case, the two files the reference's driver reads."""
    write_mesh3d(os.path.join(directory, "Mesh3d.dat"), case.xyz, formatted)
    write_bc3d_inc(os.path.join(directory, "bc3d.inc"), case)


# ---- wall_dist.dat -----------------------------------------------------------------------
def write_wall_dist(path, dw):
    """dw: per block cell-centre distances, (nz-1, ny-1, nx-1)."""
    with open(path, "wb") as f:
        for d in dw:
            _write_record(f, _fortran(d))


def read_wall_dist(path, dims):
    out = []
    with open(path, "rb") as f:
        for nx, ny, nz in dims:
            out.append(np.frombuffer(_read_record(f), dtype="<f8").reshape(nz - 1, ny - 1, nx - 1).copy())
    return out


# ---- flow files --------------------------------------------------------------------------
def _cv(params):
    return 1.0 / (params.gamma * (params.gamma - 1.0) * params.ma * params.ma)


def conservative_to_flow(U, nvar, cv):
    """output_flow (sub_IO.f90:404-423): state box (nz+7, ny+7, nx+7, nvar), cells -3..n+3 ->
    (nvar, nz+1, ny+1, nx+1) of d, u, v, w, T [, U6 [, U7]] on cells 0..n."""
    B = U[3:-3, 3:-3, 3:-3, :]
    d = B[..., 0]
    u, v, w = B[..., 1] / d, B[..., 2] / d, B[..., 3] / d
    T = (B[..., 4] - 0.5 * d * (u ** 2 + v ** 2 + w ** 2)) / (cv * d)
    out = [d, u, v, w, T] + [B[..., m] for m in range(5, nvar)]
    return np.stack(out)


def flow_to_conservative(P, nvar, cv):
    """read_flow_data (sub_IO.f90:300-320): (d, u, v, w, T, ...) -> conservative."""
    d, u, v, w, T = P[0], P[1], P[2], P[3], P[4]
    out = [d, d * u, d * v, d * w, cv * d * T + 0.5 * d * (u ** 2 + v ** 2 + w ** 2)] + [P[m] for m in range(5, nvar)]
    return np.stack(out, axis=-1)


def write_flow(directory, states, params, kstep=0, tt=0.0, numbered=False):
    """output_flow: states = per block conservative boxes as ocfd_get_state returns them."""
    nvar, cv = int(params.nvar), _cv(params)
    name = "flow3d-%08d.dat" % kstep if numbered else "flow3d.dat"
    prims = [conservative_to_flow(U, nvar, cv) for U in states]
    with open(os.path.join(directory, name), "wb") as f:
        for P in prims:
            _write_record(f, b"".join(_fortran(P[m]) for m in range(5)))
    if nvar == 6:
        with open(os.path.join(directory, "SA3d.dat"), "wb") as f:
            for P in prims:
                _write_record(f, _fortran(P[5]))
    if nvar == 7:
        with open(os.path.join(directory, "SST3d.dat"), "wb") as f:
            for P in prims:
                _write_record(f, _fortran(P[5]) + _fortran(P[6]))
    with open(os.path.join(directory, "Step_mess.dat"), "w") as f:
        f.write(" %d %.17g\n ---time Step, time ----\n" % (kstep, tt))


def read_flow(directory, dims, params):
    """read_flow_data: per block the conservative state box (nz+7, ny+7, nx+7, nvar) for
    ocfd_set_state, plus (kstep, tt).  Cells 0..n come from the files; the other ghost layers
    keep the values the reference allocates U with (sub_init.f90:518-525): d=1, momentum 0,
    energy 1, U6=1 (SA) or U6=0, U7=1 (SST).  Without SA3d.dat / SST3d.dat the turbulence
    variables on 0..n are 1/Re (SA) or Kt_Inf, Wt_Inf (SST), as the reference sets them."""
    nvar, cv = int(params.nvar), _cv(params)
    tdir = os.path.join(directory, "SA3d.dat" if nvar == 6 else "SST3d.dat")
    ft = open(tdir, "rb") if nvar > 5 and os.path.exists(tdir) else None
    out = []
    with open(os.path.join(directory, "flow3d.dat"), "rb") as f:
        for nx, ny, nz in dims:
            shp = (nz + 1, ny + 1, nx + 1)
            n = int(np.prod(shp))
            P = list(np.frombuffer(_read_record(f), dtype="<f8").reshape(5, *shp))
            if nvar > 5:
                if ft is not None:
                    P += list(np.frombuffer(_read_record(ft), dtype="<f8").reshape(nvar - 5, *shp))
                elif nvar == 6:
                    P.append(np.full(shp, 1.0 / params.re))
                else:
                    P += [np.full(shp, params.kt_inf), np.full(shp, params.wt_inf)]
            box = np.zeros((nz + 7, ny + 7, nx + 7, nvar))
            box[..., 0] = 1.0
            box[..., 4] = 1.0
            if nvar == 6:
                box[..., 5] = 1.0
            if nvar == 7:
                box[..., 6] = 1.0
            box[3:-3, 3:-3, 3:-3, :] = flow_to_conservative(np.stack(P), nvar, cv)
            out.append(box)
            del n
    if ft is not None:
        ft.close()
    kstep, tt = 0, 0.0
    sm = os.path.join(directory, "Step_mess.dat")
    if os.path.exists(sm):
        with open(sm) as f:
            toks = f.readline().split()
            kstep, tt = int(toks[0]), float(toks[1])
    return out, kstep, tt
