"""Host-side logic without a GPU: the C-ABI library's exports and argument checks, parameter
finalisation (C and Python agree), connectivity conversion, mesh generators, the bench model."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ocfd_ec_gpu.h")
# the reference's case folder (M6-wing, M6-wing-SEC, DLR-F4 with their bc3d.inp decks), when a
# checkout of the reference is at hand: OCFD_REF_CASES=<reference>/cases
REF_CASES = os.environ.get("OCFD_REF_CASES", "")


@pytest.fixture(scope="module")
def clib():
    from ocfd_b200 import build, capi
    build.build()
    return capi.lib()


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(ocfd_[a-z0-9_]+)\s*\(", src, flags=re.M)))


def test_library_exports_every_header_symbol(clib):
    names = header_functions()
    assert len(names) >= 20, names
    for n in names:
        assert hasattr(clib, n), "libocfd_b200.so does not export %s" % n
    from ocfd_b200 import capi
    assert set(capi.EXPORTED) == set(names), set(capi.EXPORTED) ^ set(names)


def test_version_string(clib):
    from ocfd_b200 import capi
    v = capi.version()
    assert "sm_100a" in v or "opencfd" in v.lower(), v


def test_params_default_and_finalize_match_python(clib):
    """ocfd_default_params + ocfd_finalize_params (C) == default_params + finalize (Python),
    both restating sub_read_parameter.f90:30-106 and 371-429."""
    from ocfd_b200.params import OcfdParams, default_params, finalize
    for raw in (dict(), dict(ma=0.8, aoa=3.0, re=1e7, iflag_turbulence_model=2),
                dict(if_viscous=0, iflag_turbulence_model=3, cood_y_up=0, aos=1.5, bound_scheme=-1, iflag_scheme=7),
                dict(iflag_turbulence_model=3, twall=300.0, t_inf=250.0)):
        c = OcfdParams()
        assert clib.ocfd_default_params(ctypes.byref(c)) == 0
        for k, v in raw.items():
            setattr(c, k, v)
        assert clib.ocfd_finalize_params(ctypes.byref(c)) == 0
        py = finalize(default_params(**raw))
        assert bytes(c) == bytes(py), (raw, c.as_dict(), py.as_dict())


def test_create_rejects_bad_arguments_before_touching_the_device(clib):
    from ocfd_b200 import cases
    from ocfd_b200.capi import OCFD_ERR_ARG, OCFD_ERR_UNSUPPORTED
    p, case = cases.config1(scale=0.25)
    nijk, xyz, nsub, inc = case.flat()
    IP = ctypes.POINTER(ctypes.c_int)
    DP = ctypes.POINTER(ctypes.c_double)
    xp = (DP * 1)(xyz[0].ctypes.data_as(DP))
    h = ctypes.c_void_p()
    call = lambda pp, nb, nj: clib.ocfd_create(ctypes.byref(pp) if pp is not None else None, nb,  # noqa: E731
                                               nj.ctypes.data_as(IP), xp, nsub.ctypes.data_as(IP),
                                               inc.ctypes.data_as(IP), None, ctypes.byref(h))
    assert call(None, 1, nijk) == OCFD_ERR_ARG
    assert call(p, 0, nijk) == OCFD_ERR_ARG
    bad = nijk.copy()
    bad[0] = 1
    assert call(p, 1, bad) == OCFD_ERR_ARG
    q = p.copy()
    q.if_viscous = 1
    q.iflag_turbulence_model = 1   # Baldwin-Lomax: not on the hot path
    assert call(q, 1, nijk) == OCFD_ERR_UNSUPPORTED
    q = p.copy()
    q.time_method = 2              # no such time method (sub_time_advance.f90:10-19)
    assert call(q, 1, nijk) == OCFD_ERR_UNSUPPORTED
    q = p.copy()
    q.if_residual_smoothing = 2
    assert call(q, 1, nijk) == OCFD_ERR_ARG
    q = p.copy()
    q.iflag_flux = 9
    assert call(q, 1, nijk) == OCFD_ERR_ARG
    assert not h.value


def test_null_handle_calls_return_arg_error(clib):
    from ocfd_b200.capi import OCFD_ERR_ARG
    a = np.zeros(7)
    dp = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert clib.ocfd_residual(None, dp, dp) == OCFD_ERR_ARG
    assert clib.ocfd_advance(None, 1, None, None) == OCFD_ERR_ARG
    assert clib.ocfd_get_state(None, 0, dp) == OCFD_ERR_ARG
    assert clib.ocfd_destroy(None) in (0, OCFD_ERR_ARG)


def _check_inc_consistency(inp, inc):
    """Every inner subface's partner record points back at it with the same extents."""
    nsub = 0
    for b, recs in enumerate(inc):
        assert len(recs) == len(inp[b].subs)
        for q, r in enumerate(recs):
            assert len(r) == 21
            ib, ie, jb, je, kb, ke, bc, face, f_no = r[:9]
            assert f_no == q + 1
            assert 1 <= ib <= ie <= inp[b].nx and 1 <= jb <= je <= inp[b].ny and 1 <= kb <= ke <= inp[b].nz
            lo = (ib, jb, kb)[(face - 1) % 3]
            hi = (ie, je, ke)[(face - 1) % 3]
            assert lo == hi
            nsub += 1
            if bc >= 0:
                continue
            nb1, face1, f_no1 = r[15], r[16], r[17]
            partner = inc[nb1 - 1][f_no1 - 1]
            assert partner[15] == b + 1 and partner[17] == q + 1 and partner[16] == face
            assert partner[7] == face1
            # the orientation maps are inverse permutations of each other
            L = [abs(x) for x in r[18:21]]
            L1 = [abs(x) for x in partner[18:21]]
            assert sorted(L) == [1, 2, 3]
            assert [L1[L[d] - 1] for d in range(3)] == [1, 2, 3]
            # same number of points on both sides
            n0 = (ie - ib + 1) * (je - jb + 1) * (ke - kb + 1)
            n1 = (r[10] - r[9] + 1) * (r[12] - r[11] + 1) * (r[14] - r[13] + 1)
            assert n0 == n1
    return nsub


@pytest.mark.parametrize("name", ["M6-wing", "M6-wing-SEC", "DLR-F4"])
def test_convert_reference_bc3d_inp(name):
    """.inp -> .inc conversion (sub_convert_inp.f90:25-248) of the reference's own case decks:
    every inner subface finds its partner and the orientation maps are mutually inverse."""
    path = os.path.join(REF_CASES, name, "bc3d.inp")
    if not REF_CASES or not os.path.exists(path):
        pytest.skip("set OCFD_REF_CASES to the reference's cases folder to run this test")
    from ocfd_b200.connectivity import convert_inp_inc, read_bc3d_inp
    inp = read_bc3d_inp(path)
    inc = convert_inp_inc(inp)
    assert _check_inc_consistency(inp, inc) > 0


def test_generated_cases_roundtrip_bc3d_inp(tmp_path):
    from ocfd_b200 import cases
    from ocfd_b200.connectivity import convert_inp_inc, read_bc3d_inp, write_bc3d_inp
    for p, case in (cases.config1(scale=0.25, cuts_i=(12,)), cases.config2_small(), cases.airfoil(ni=65, nj=17)):
        f = tmp_path / (case.name + ".inp")
        write_bc3d_inp(str(f), case.inp)
        back = read_bc3d_inp(str(f))
        assert [(b.nx, b.ny, b.nz) for b in back] == [(b.nx, b.ny, b.nz) for b in case.inp]
        assert convert_inp_inc(back) == case.inc
        _check_inc_consistency(case.inp, case.inc)


def test_interface_nodes_coincide():
    """Generated multi-block meshes: the node planes two blocks share are the same points."""
    from ocfd_b200 import cases
    for p, case in (cases.config1(scale=0.25, cuts_i=(12,)), cases.config2_small()):
        for b, recs in enumerate(case.inc):
            for r in recs:
                if r[6] >= 0:
                    continue
                ib, ie, jb, je, kb, ke = r[:6]
                ib1, ie1, jb1, je1, kb1, ke1, nb1 = r[9:16]
                L = r[18:21]
                A = case.xyz[b][:, kb - 1:ke, jb - 1:je, ib - 1:ie]
                Bx = case.xyz[nb1 - 1]
                lo1, hi1 = (ib1, jb1, kb1), (ie1, je1, ke1)
                for kk in range(kb, ke + 1):
                    for jj in range(jb, je + 1):
                        for ii in range(ib, ie + 1):
                            t = [ii - ib, jj - jb, kk - kb]
                            idx = [0, 0, 0]
                            for d in range(3):
                                s = t[abs(L[d]) - 1] if L[d] != 0 else 0
                                idx[d] = lo1[d] + s if L[d] > 0 else hi1[d] - s
                            pa = case.xyz[b][:, kk - 1, jj - 1, ii - 1]
                            pb = Bx[:, idx[2] - 1, idx[1] - 1, idx[0] - 1]
                            assert np.allclose(pa, pb, atol=1e-12), (case.name, b, r, (ii, jj, kk), idx)
                del A


def test_config_sizes():
    """The benchmark workloads have the sizes they are named for."""
    from ocfd_b200 import cases
    p, c1 = cases.config1()
    assert c1.ncells == 128 * 64 * 16 == 131072 and p.nvar == 5
    p, c2 = cases.config2()
    assert len(c2.dims) == 8 and 2.0e6 <= c2.ncells <= 2.2e6 and p.nvar == 6
    batch = cases.config4_batch(n=8)
    assert len(batch) == 8 and all(q.precision == 1 for q, _ in batch)


def test_bench_bytes_model():
    """Algorithmic bytes per cell-update of the roofline: K1 + K2 + K3 per LU-SGS iteration."""
    import bench
    tot = {k: sum(v.values()) for k, v in bench.BYTES.items()}
    assert tot[("fp64", 5)] == 760 and tot[("fp64", 6)] == 1192 and tot[("fp64", 7)] == 1256
    assert tot[("mixed", 5)] == 500 and tot[("mixed", 6)] == 740 and tot[("mixed", 7)] == 796


def test_bench_reference_arm_runs_on_cpu():
    """bench.py's reference arm (the CPU restatement on the host cores) prints its JSON line on a
    small workload, and every leg the GPU arm calls is defined."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "config1",
                          "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "cell-updates/s"
    assert {"workload", "cells", "parallelism", "l2"} <= set(line["config"])
    sys.path.insert(0, ROOT)
    import bench
    for name in ("mixed_leg", "batch_leg", "config3_leg", "serving_leg", "sweep_serving_leg", "converged_leg",
                 "bench_config", "cpu_sample", "run_reference", "diverges_at", "open_solver", "make_case", "shard_main"):
        assert callable(getattr(bench, name)), name
