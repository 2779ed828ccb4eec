"""ocfd_residual_static: the allocation-free residual norms agree bit for bit with
ocfd_residual, on two calls in a row, across handles sharing the static scratch, and refuse
handles larger than the static area with a clear error.  Collected last on purpose: it must pass
alone and after every other test in the process."""
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
