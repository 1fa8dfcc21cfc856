"""Failure detection without a GPU fault.

* A bounded device wait runs out: the Kaczmarz sweep kernel's first step is
  made to wait for a completion stamp that nothing writes (test hook), with
  a short cycle budget.  The kernel raises its error flag, every warp
  leaves, airt_art returns AIRT_ERR_TIMEOUT, and the next normal call in the
  same process succeeds and matches the oracle.
* A device allocation fails (host-side injection): the call returns
  AIRT_ERR_OOM with its message, and the next call succeeds.
"""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from airtoolsii_b200 import _lib
from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture()
def hooks_off():
    L = _lib.lib()
    yield L
    L.airt_test_inject_stall(0)
    L.airt_test_set_wait_budget(4_000_000_000)
    L.airt_test_fail_alloc(-1)


def test_kaczmarz_wait_runs_out_then_recovers(hooks_off):
    L = hooks_off
    A_ref = O.paralleltomo_matrix(32, np.arange(0.0, 180.0, 6.0))
    A = airt.afun_matrix(A_ref)
    b = A_ref @ O.shepplogan(32)
    assert L.airt_test_set_wait_budget(2_000_000) == _lib.AIRT_OK      # ~1 ms
    L.airt_test_inject_stall(1)
    with pytest.raises(airt.AirtError) as e:
        airt.kaczmarz(A, b, [2])
    assert e.value.code == _lib.AIRT_ERR_TIMEOUT
    assert "bounded device wait" in str(e.value)
    L.airt_test_inject_stall(0)
    L.airt_test_set_wait_budget(4_000_000_000)
    X, info = airt.kaczmarz(A, b, [2])
    Xo, _ = O.art("kaczmarz", A_ref, b, [2])
    assert info["finaliter"] == 2 and relerr(X[:, -1], Xo[:, -1]) <= 1e-5


def test_injected_allocation_failure(hooks_off):
    L = hooks_off
    theta = np.arange(0.0, 180.0, 4.0)
    L.airt_test_fail_alloc(0)
    with pytest.raises(airt.AirtError) as e:
        airt.paralleltomo(24, theta)
    assert e.value.code == _lib.AIRT_ERR_OOM
    assert "injected allocation failure" in str(e.value)
    A, b, x, *_ = airt.paralleltomo(24, theta)            # the countdown is spent: normal again
    # a failure in the middle of a solve leaves the handle usable
    L.airt_test_fail_alloc(3)
    with pytest.raises(airt.AirtError) as e:
        airt.cimmino(A, b, [5], None, {"rho": 1.0})
    assert e.value.code == _lib.AIRT_ERR_OOM
    L.airt_test_fail_alloc(-1)
    X, info = airt.cimmino(A, b, [5], None, {"rho": 1.0})
    Xo, _, _ = O.sirt("cimmino", O.paralleltomo_matrix(24, theta), b, [5], None, {"rho": 1.0})
    assert relerr(X[:, -1], Xo[:, -1]) <= 1e-5
