"""Failure paths on the GPU, made without a GPU fault.

* The tensor-core kernels' bounded mbarrier wait is run on a barrier that
  nothing arrives at: it must give up after its poll limit, record the
  timeout and return, and the context must stay usable.
* A NaN planted on the host in one block of a matrix (through the
  reference's wire format: Pack, change one double, Unpack) must surface as
  HM_ERR_NUMERICAL from EstimateTwoNorm, from SchulzInvert and, after an H*H
  product whose roundings meet it, from the next synchronization; the context
  stays usable afterwards."""
import ctypes as C
import struct

import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu
HM_ERR_NUMERICAL = 5


def test_bounded_wait_gives_up_and_context_survives():
    t = C.c_int(-1)
    _lib.check(_lib.lib().hm_check_bounded_wait(0, 1 << 14, C.byref(t)))
    assert t.value == 1
    fx = load("weak")
    ctx = D.Context(0)
    H = build(D, fx, ctx)
    assert relerr(H.Multiply(1.0, fx["probes"]), fx["matvec"]) < 1e-13


def _with_nan(H):
    """Copy of H whose last stored double (the last entry of the last block
    in the wire format's depth-first order) is NaN."""
    b = bytearray(H.Pack())
    pos = len(b) - 4 - 8              # the format ends with 4 bytes after the data
    (v,) = struct.unpack_from("d", b, pos)
    assert np.isfinite(v)
    struct.pack_into("d", b, pos, float("nan"))
    return type(H).Unpack(bytes(b), ctx=H.ctx)


def test_nan_block_reported_as_numerical():
    fx = load("ragged")
    ctx = D.Context(0)
    H = build(D, fx, ctx)
    H.SetToRandom()
    Hn = _with_nan(H)
    y = Hn.Multiply(1.0, fx["probes"])
    assert not np.all(np.isfinite(y))            # the NaN is in the operator
    with pytest.raises(D.HMError) as e:
        D.EstimateTwoNorm(Hn, 1.5, 6.0)
    assert e.value.status == HM_ERR_NUMERICAL
    C2 = Hn.Multiply(1.0, Hn)                    # roundings meet the NaN
    with pytest.raises(D.HMError) as e:
        ctx.synchronize()
    assert e.value.status == HM_ERR_NUMERICAL
    ctx.synchronize()                            # the flag was cleared
    del C2
    with pytest.raises(D.HMError) as e:
        _with_nan(H).SchulzInvert(2)
    assert e.value.status == HM_ERR_NUMERICAL
    # the context still computes correctly
    assert relerr(H.Multiply(1.0, fx["probes"]), fx["random"]) < 1e-13
