"""ocfd_residual_static: the allocation-free residual norms agree bit for bit with
ocfd_residual, on two calls in a row, across handles sharing the static scratch; a fresh handle
whose first read-back is this call leaves the device's free memory unchanged; handles larger than
the static area (in solves or in norm chunks) are refused with a clear error, and a NaN gives
OCFD_ERR_NAN.  Collected last on purpose: it must pass alone and after every other test in the
process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_residual_equals_residual(gpu):
    from ocfd_b200 import cases
    p, case = cases.config2_small()
    s = gpu.Solver(p, case)
    for _ in range(2):
        s.advance(2)
        a_max, a_rms = s.residual()
        b_max, b_rms = s.residual_static()
        assert np.array_equal(a_max, b_max) and np.array_equal(a_rms, b_rms)
        c_max, c_rms = s.residual_static()      # a second call in a row, no step between
        assert np.array_equal(b_max, c_max) and np.array_equal(b_rms, c_rms)
    # a second handle on the same device uses the same static area
    q, case2 = cases.config1(scale=0.25)
    t = gpu.Solver(q, case2)
    t.advance(3)
    assert all(np.array_equal(x, y) for x, y in zip(t.residual(), t.residual_static()))
    assert all(np.array_equal(x, y) for x, y in zip(s.residual(), s.residual_static()))
    t.close()
    s.close()


def test_static_residual_rejects_oversize_handle(gpu):
    from ocfd_b200 import cases
    items = [cases.airfoil(ni=17, nj=5, aoa=0.01 * q) for q in range(257)]   # 257 solves > 256
    b = gpu.Batch(items)
    with pytest.raises(gpu.OcfdError) as e:
        b.residual_static()
    assert e.value.code == gpu.OCFD_ERR_ARG and "256 solves" in str(e.value)
    b.close()


def test_static_residual_first_call_allocates_nothing(gpu):
    """A fresh handle calls ocfd_residual_static before any other read-back (so the pinned
    read-back area of ocfd_residual is never set up): the device's free memory stays the same
    over repeated calls, and the norms equal ocfd_residual's afterwards."""
    import torch
    from ocfd_b200 import cases
    p, case = cases.airfoil(ni=65, nj=17)
    s = gpu.Solver(p, case)
    s.advance(2)
    s.synchronize()
    first = s.residual_static()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        again = s.residual_static()
        assert all(np.array_equal(x, y) for x, y in zip(first, again))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert all(np.array_equal(x, y) for x, y in zip(s.residual(), first))
    s.close()


def test_static_residual_rejects_too_many_chunks(gpu):
    """241 solves of 17 small blocks each: 4097 norm chunks (one per block) with only 262,208
    cells and fewer than 256 solves; refused with OCFD_ERR_ARG and the chunk count."""
    from meshes import wavy_box
    from ocfd_b200.params import make_params
    case = wavy_box(nx=69, ny=5, nz=5, cuts=tuple(range(5, 69, 4)))
    assert len(case.dims) == 17
    p = make_params(ma=0.5, if_viscous=0, iflag_scheme=5, iflag_flux=4, cfl=2.0)
    b = gpu.Batch([(p, case)] * 241)
    with pytest.raises(gpu.OcfdError) as e:
        b.residual_static()
    assert e.value.code == gpu.OCFD_ERR_ARG and "4097 norm chunks" in str(e.value), str(e.value)
    b.close()


def test_static_residual_reports_nan(gpu):
    from ocfd_b200 import cases
    p, case = cases.airfoil(ni=65, nj=17)
    s = gpu.Solver(p, case)
    s.advance(2)
    U = s.get_state(0)
    U[3 + 1, 3 + 6, 3 + 20, 0] = float("nan")
    s.set_state(0, U)
    s.advance(1)
    with pytest.raises(FloatingPointError) as e:
        s.residual_static()
    assert "NaN" in str(e.value)
    s.close()
