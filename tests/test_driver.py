"""The compiled C++ caller (opencfd-ec_b200/driver/ocfd_drive.cpp) reads the reference's input
files as the Fortran driver does: Mesh3d.dat (read_main_mesh, Fortran unformatted records) and
bc3d.inc (read_inc, text).  Here, without a GPU: the files written by ocfd_b200.formats are read
back by the driver's --check mode (no device call) and must give the case's block sizes,
subface records and coordinates."""
import math
import subprocess

import numpy as np


def _driver():
    from ocfd_b200 import build
    build.build()
    return build.build_driver()


def test_driver_reads_reference_input_files(tmp_path):
    from ocfd_b200 import cases
    from ocfd_b200.formats import write_case_files
    drv = _driver()
    for _, case in (cases.config2_small(), cases.config1(scale=0.25, cuts_i=(12,))):
        write_case_files(str(tmp_path), case)
        out = subprocess.run([drv, str(tmp_path), "--check"], capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stderr
        lines = out.stdout.splitlines()
        nijk, xyz, nsub, inc = case.flat()
        assert lines[0] == "blocks %d" % len(case.dims)
        for b, (nx, ny, nz) in enumerate(case.dims):
            assert lines[1 + b] == "block %d %d %d %d nsub %d" % (b + 1, nx, ny, nz, nsub[b])
        got = [int(v) for v in lines[1 + len(case.dims)].split()[1:]]
        assert got == [int(v) for v in inc]
        want = math.fsum(float(v) for a in xyz for v in np.ravel(a))
        assert math.isclose(float(lines[-1].split()[1]), want, rel_tol=1e-12)
