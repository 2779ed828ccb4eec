"""Every LU-SGS wavefront variant gives the hyperplane-order bits.

The creation-time autotuner picks a tile width (32 or 64 columns) and a wavefront kernel version
(3: inputs staged by element; 4: staged by 32-byte sector, helper warps off the step phases, or
with both sweeps in one launch when OCFD_LU_ONE_LAUNCH is set; 5:
inputs packed in sweep order and fetched by one bulk copy per step, 64-column tiles) per case; the
choice must never change a result.  Each variant is forced here through its switches and
compared bit for bit with the one-launch-per-hyperplane sweep (OCFD_LUSGS_PLANES=1), on cases that
cover NV = 5, 6 and 7, dual time, block edges that cut tiles, blocks thinner than a tile, and both
precisions (in the mixed form the wavefront's flux difference is FP32 while the hyperplane form's
is FP64, so there the two versions are compared with each other).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SWITCHES = ("OCFD_LU_V3", "OCFD_LU_V4", "OCFD_LU_V5", "OCFD_LU_TC", "OCFD_LUSGS_PLANES", "OCFD_NO_AUTOTUNE",
            "OCFD_LU_ONE_LAUNCH")
# (version, tile width, extra switches): version 4 also with both sweeps in one launch
ONE = {"OCFD_LU_ONE_LAUNCH": "1"}
VARIANTS = (("3", "32", {}), ("3", "64", {}), ("4", "32", {}), ("4", "64", {}), ("4", "32", ONE), ("4", "64", ONE),
            ("5", "64", {}))


def run(gpu, p, case, env, nsteps):
    old = {k: os.environ.get(k) for k in SWITCHES}
    for k in SWITCHES:
        os.environ.pop(k, None)
    os.environ.update(env)
    try:
        s = gpu.Solver(p, case)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    ver, tc = s.lu_kernel_version(), s.lu_tile_width()
    run.one_launch = s.lu_one_launch()
    s.advance(nsteps)
    U = [s.get_state(b) for b in range(s.nblk)]
    DU = [s.get_array(b, "DU")[0] for b in range(s.nblk)]
    s.close()
    return U, DU, ver, tc


def bits_equal(a, b):
    return all(np.array_equal(x.view(np.uint64), y.view(np.uint64)) for x, y in zip(a, b))


def case_list():
    from meshes import wavy_box
    from ocfd_b200 import cases
    from ocfd_b200.params import make_params
    out = {
        "config2_small_sa": cases.config2_small(),
        "config3_small_sst": cases.config3_small(),
        "config1_euler_2blk": cases.config1(scale=0.5, cuts_i=(20,)),
        "config2_small_dual": cases.config2_small(time_method=-1, dt_global=0.05, step_inner_limit=3, res_inner_limit=1e-14),
    }
    ragged = wavy_box(nx=21, ny=11, nz=7, cuts=(2, 4, 15))
    out["ragged_sa"] = (make_params(ma=0.5, aoa=3.0, if_viscous=1, iflag_turbulence_model=2, iflag_scheme=5, iflag_flux=4,
                                    re=1e5, cfl=2.0), ragged)
    return out


NAMES = ["config2_small_sa", "config3_small_sst", "config1_euler_2blk", "config2_small_dual", "ragged_sa"]


@pytest.mark.parametrize("name", NAMES)
def test_every_wavefront_variant_equals_hyperplanes(gpu, name):
    p, case = case_list()[name]
    refU, refDU, _, _ = run(gpu, p, case, {"OCFD_LUSGS_PLANES": "1"}, 3)
    for ver, tc, extra in VARIANTS:
        U, DU, v, t = run(gpu, p, case, dict({"OCFD_LU_V" + ver: "1", "OCFD_LU_TC": tc}, **extra), 3)
        assert (v, t) == (int(ver), int(tc))
        assert run.one_launch == (extra is ONE)
        assert bits_equal(U, refU), (name, ver, tc, extra)
        assert bits_equal(DU, refDU), (name, ver, tc, extra)


@pytest.mark.parametrize("name", ["config2_small_sa", "config3_small_sst"])
def test_mixed_wavefront_versions_agree(gpu, name):
    """Versions 3 and 4 agree bit for bit in the mixed form.  Version 5's mixed form takes the
    off-diagonal products in FP32 and multiplies by the diagonal's FP64 reciprocal (the north star
    keeps only the diagonal inverse and the accumulation in FP64), and the compiler may contract
    its FP32 operations differently: the FP32 flux difference F(U+DU) - F(U) is a cancellation
    that keeps ~1e-4 of DU's digits, so the state after three steps agrees to 1e-5 of each
    variable's scale (the converged state, where Res = 0, does not depend on the sweep's
    rounding)."""
    p, case = case_list()[name]
    p = p.copy()
    p.precision = 1
    base = None
    for ver, tc, extra in VARIANTS:
        U, DU, v, t = run(gpu, p, case, dict({"OCFD_LU_V" + ver: "1", "OCFD_LU_TC": tc}, **extra), 3)
        assert (v, t) == (int(ver), int(tc))
        if base is None:
            base = (U, DU)
        elif ver != "5":
            assert bits_equal(U, base[0]), (name, ver, tc)
            assert bits_equal(DU, base[1]), (name, ver, tc)
        else:
            for a, b in zip(U, base[0]):
                scale = np.maximum(np.abs(b).max(axis=(0, 1, 2)), 1e-30)
                assert (np.abs(a - b).max(axis=(0, 1, 2)) / scale).max() <= 1e-5, (name, ver, tc)


def test_autotuner_picks_a_known_variant(gpu):
    from ocfd_b200 import cases
    p, case = cases.config2_small()
    _, _, v, t = run(gpu, p, case, {}, 1)
    assert v in (3, 4, 5) and t in (32, 64)
    assert not run.one_launch or v == 4
    _, _, v, t = run(gpu, p, case, {"OCFD_NO_AUTOTUNE": "1"}, 1)
    assert (v, t) == (4, 32)
