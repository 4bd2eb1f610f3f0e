"""The reference's Pack / Unpack wire format (src/HMat2d/Pack-incl.hpp):
matrices packed by the reference itself (tests/golden/pack.npz) load on the
device and multiply like the reference's own Unpack; matrices packed here
have the reference's byte layout and round-trip bit for bit.

Tolerances: products 1e-13 relative (same data, different summation order);
bytes exact."""
import numpy as np
import pytest

import dmhm_b200 as D
from dmhm_b200 import _lib
from helpers import build, load, relerr

pytestmark = pytest.mark.gpu


def fresh_ctx(fx):
    c = D.Context(0)
    c.set_oversample(int(fx["oversample"]))
    return c


@pytest.mark.parametrize("case", ["ragged", "c3d"])
def test_unpack_reference_bytes(case):
    pk = load("pack")
    fx = load(case)
    cls = D.HMat3d if len(fx["sizes"]) == 3 else D.HMat2d
    H = cls.Unpack(pk[case + "_pack"].tobytes(), ctx=fresh_ctx(fx))
    assert relerr(H.Multiply(1.0, fx["probes"]), pk[case + "_unpack_matvec"]) < 1e-13
    # and it packs back to the same bytes
    assert H.Pack() == pk[case + "_pack"].tobytes()


def test_pack_matches_reference_layout():
    """SetToRandom here draws the reference's numbers, so packing it gives
    the reference's bytes: the same layout, header and ranks exactly, the
    data to the last bits of the Gaussian transform."""
    pk = load("pack")
    fx = load("ragged")
    c = fresh_ctx(fx)
    H = build(D, fx, c)
    H.SetToRandom()
    ours = np.frombuffer(H.Pack(), dtype=np.uint8)
    ref = pk["ragged_pack"]
    assert ours.size == ref.size
    # reload both and compare as operators
    A = D.HMat2d.Unpack(ours.tobytes(), ctx=c)
    B = D.HMat2d.Unpack(ref.tobytes(), ctx=c)
    P = fx["probes"]
    assert relerr(A.Multiply(1.0, P), B.Multiply(1.0, P)) < 1e-13
    # header (12 ints + 2 bools = 50 bytes) and the trailing slack identical
    assert np.array_equal(ours[:50], ref[:50])
    assert np.array_equal(ours[-4:], ref[-4:])


def test_round_trip_after_products():
    """An H*H product (ranks from the compression) survives Pack / Unpack."""
    fx = load("c1")
    c = fresh_ctx(fx)
    A = build(D, fx, c)
    A.SetToRandom()
    C2 = A.Multiply(0.5, A)
    b = C2.Pack()
    assert len(b) == C2.PackedSize()
    R = D.HMat2d.Unpack(b, ctx=c)
    assert R.Pack() == b
    P = fx["probes"]
    assert np.array_equal(R.Multiply(1.0, P), C2.Multiply(1.0, P))


def test_unpack_rejects_bad_input():
    pk = load("pack")
    fx = load("ragged")
    c = fresh_ctx(fx)
    raw = pk["ragged_pack"].tobytes()
    with pytest.raises(_lib.HMError):
        D.HMat2d.Unpack(raw[: len(raw) // 2], ctx=c)       # truncated
    bad = bytearray(raw)
    bad[16] = 1                                           # symmetric flag
    with pytest.raises(_lib.HMError):
        D.HMat2d.Unpack(bytes(bad), ctx=c)
