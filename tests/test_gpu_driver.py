"""The drop-in boundary from a compiled caller: the C++ driver (opencfd-ec_b200/driver/
ocfd_drive.cpp) runs the reference's time loop through include/ocfd_ec_gpu.h only
(ocfd_default_params / ocfd_finalize_params from namelist-style values, ocfd_create from
Mesh3d.dat + bc3d.inc, ocfd_advance every step, ocfd_forces + ocfd_residual every Kstep_show
steps, output_flow at the end).  Its printed monitor history and its flow3d.dat must equal, bit
for bit, the same run through the Python binding with the same raw parameters."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    from ocfd_b200 import cases, meshgen
    bump = meshgen.channel_bump(33, 17, 5, cuts_i=(12,), name="bump")
    foil = meshgen.airfoil_omesh(ni=65, nj=17, nk=3, m=0.02, p=0.4, t=0.12, ds=2e-6, name="foil")
    return {
        "bump2_euler": (bump, dict(ma=0.5, aoa=0.0, if_viscous=0, iflag_scheme=5, iflag_flux=4, time_method=0, cfl=5.0)),
        "foil_sa": (foil, dict(ma=0.7, aoa=2.0, re=6.0e6, if_viscous=1, iflag_turbulence_model=2, iflag_scheme=5,
                               iflag_flux=6, time_method=0, cfl=5.0,
                               ref_s=float(foil.xyz[0][2].max() - foil.xyz[0][2].min()))),
    }


@pytest.mark.parametrize("name", list(_cases()))
def test_driver_equals_python_binding(gpu, tmp_path, name):
    from ocfd_b200 import build
    from ocfd_b200.formats import write_case_files, write_flow
    from ocfd_b200.params import make_params
    case, raw = _cases()[name]
    steps, show = 12, 4
    drv = build.build_driver()
    cdir, pdir = tmp_path / "case", tmp_path / "py"
    cdir.mkdir()
    pdir.mkdir()
    write_case_files(str(cdir), case)
    args = [drv, str(cdir), "steps=%d" % steps, "show=%d" % show] + ["%s=%r" % (k, v) for k, v in raw.items()]
    out = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    hist = [l.split() for l in out.stdout.splitlines() if l.startswith("step ")]
    assert len(hist) == steps // show
    p = make_params(**raw)
    g = gpu.Solver(p, case)
    rows = []
    for k in range(1, steps + 1):
        kk, tt = g.advance(1)
        if k % show == 0:
            ft, cl, cd, cs = g.forces()
            mx, rms = g.residual()
            rows.append((kk, tt, mx, rms, ft, cl, cd, cs))
    for h, (kk, tt, mx, rms, ft, cl, cd, cs) in zip(hist, rows):
        assert int(h[1]) == kk
        vals = np.array([float(v) for v in h[2:]])
        want = np.concatenate([[tt], mx, rms, ft, [cl, cd, cs]])
        assert np.array_equal(vals, want), (vals - want)
    write_flow(str(pdir), [g.get_state(b) for b in range(g.nblk)], p, kstep=kk, tt=tt)
    g.close()
    for f in ("flow3d.dat", "Step_mess.dat"):
        assert open(os.path.join(cdir, f), "rb").read() == open(os.path.join(pdir, f), "rb").read(), f
