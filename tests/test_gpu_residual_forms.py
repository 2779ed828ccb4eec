"""The forms of the residual give the bits of the face-flux form.

The Navier-Stokes part of the residual computes each direction's face fluxes in its own kernel,
stores them to face planes and assembles Res from them (k_inv_flux, k_inv_kbc, k_visc_flux,
k_assemble); the opt-in tile forms (OCFD_RES_FUSED=1: all fluxes of a tile of cells in shared
memory; 2: the inviscid ones, the viscous ones still from k_visc_flux; 3: the viscous ones, the
inviscid ones from k_inv_flux) must give the same FP64 results, bit for bit.  The SA part runs as
one tile kernel by default (k_sa_tile); OCFD_SA_SPLIT restores k_sa_flux + k_sa_res.  By default
the viscosity / turbulence chain runs on a second stream beside the inviscid fluxes; the
residual issued on one stream (OCFD_RES_STREAMS=0), or with the inviscid fluxes forked instead
(1), must give the same bits too.  Cases cover the OverLimit path, physical k faces (the central
flux of k_inv_kbc), several blocks, tiles cut by block edges (OCFD_RES_TILE) and both
reconstructions.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SWITCHES = ("OCFD_RES_FUSED", "OCFD_RES_TILE", "OCFD_SA_SPLIT", "OCFD_RES_STREAMS")


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
    s.advance(nsteps)
    U = [s.get_state(b) for b in range(s.nblk)]
    R = [s.get_array(b, "Res")[0] for b in range(s.nblk)]
    f = s.forces()
    s.close()
    return U, R, f


def bits_equal(a, b):
    return all(np.array_equal(np.asarray(x).view(np.uint64), np.asarray(y).view(np.uint64)) for x, y in zip(a, b))


def case_list():
    from ocfd_b200 import cases
    return {
        "wing8_sa": cases.config2_small(),
        "wing24_sst": cases.config3_small(),
        "bump_euler_2blk": cases.config1(scale=0.5, cuts_i=(20,)),
        "foil_sa_char": cases.airfoil(ni=65, nj=17, scheme=5, flux=2, turb=2, iflag_reconstruction=2),
    }


CASES = case_list()
FORMS = {
    "fused1": {"OCFD_RES_FUSED": "1"},
    "fused2": {"OCFD_RES_FUSED": "2"},
    "fused2_8x6x4": {"OCFD_RES_FUSED": "2", "OCFD_RES_TILE": "8,4,200"},
    "fused1_32x16x2": {"OCFD_RES_FUSED": "1", "OCFD_RES_TILE": "32,2,1024"},
    "fused3": {"OCFD_RES_FUSED": "3"},
    "fused3_8x6x4": {"OCFD_RES_FUSED": "3", "OCFD_RES_TILE": "8,4,200"},
    "sa_split": {"OCFD_SA_SPLIT": "1"},
    "one_stream": {"OCFD_RES_STREAMS": "0"},
    "inviscid_forked": {"OCFD_RES_STREAMS": "1"},
    "sa_tile_8x6x4_fused1": {"OCFD_RES_FUSED": "1", "OCFD_RES_TILE": "8,4,200"},
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("form", list(FORMS))
def test_tile_form_bits(gpu, name, form):
    p, case = CASES[name]
    ref = run(gpu, p, case, {}, 4)
    got = run(gpu, p, case, FORMS[form], 4)
    assert bits_equal(ref[0], got[0]), "state"
    assert bits_equal(ref[1], got[1]), "Res"
    assert np.array_equal(ref[2][0], got[2][0]) and ref[2][1:] == got[2][1:], "forces"


def test_tile_form_overlimit(gpu):
    """A block in OverLimit (UD1, no viscous flux, zero viscous wall flux) takes the same path in
    the tile forms: the limiter is made to fire by tight bounds from a prepared state."""
    import branch_cases
    p, case, warm, preps, steps = branch_cases.limiter_cases()["foil_sa_lusgs"]()
    outs = []
    for env in ({}, {"OCFD_RES_FUSED": "1"}, {"OCFD_RES_FUSED": "2"}, {"OCFD_RES_FUSED": "3"}, {"OCFD_SA_SPLIT": "1"}):
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
        branch_cases.prepare(s, p, warm, preps)
        s.advance(steps)
        st = [s.limiter_status(b) for b in range(s.nblk)]
        outs.append(([s.get_state(b) for b in range(s.nblk)], st, s.forces()))
        s.close()
    assert any(ov for _, ov in outs[0][1]), "the limiter did not leave a block in OverLimit"
    for o in outs[1:]:
        assert o[1] == outs[0][1]
        assert bits_equal(outs[0][0], o[0])
        assert np.array_equal(outs[0][2][0], o[2][0]) and outs[0][2][1:] == o[2][1:]
