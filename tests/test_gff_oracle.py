"""The CPU restatement of the flow-field cache formats (``oracle/gff.py``) on known answers.

No .gff/.tke file of the reference exists to pin against, so the restatement is checked three
ways: conversions against hand-computed values (truncation, half-to-even rounding, clamping, NaN),
whole payloads against byte-by-byte loop restatements that follow the reference's writer loops
literally (GFFWrite.cs), and the reader against the writer (round trips, every rejection the
reference's reader makes, GFFRead.cs).
"""
import struct

import numpy as np
import pytest

from oracle import gff


def test_conversions_known_answers():
    # modes -1/-2: float32 product, clamp, truncation toward zero, NaN -> 0
    x = np.array([1.234, -1.239, -0.005, 0.0099, 400.0, -400.0, np.inf, -np.inf, np.nan, 327.5, -327.68],
                 np.float32)
    assert gff.to_i16_trunc(x).tolist() == [123, -123, 0, 0, 32767, -32768, 32767, -32768, 0, 32750, -32768]
    # mode -3: MathF.Round (half to even) before the clamp
    y = np.array([0.125, 0.375, -0.125, -0.375, 0.0049, 1.0, 500.0, np.nan], np.float32)
    assert gff.to_i16_round(y).tolist() == [12, 38, -12, -38, 0, 100, 32767, 0]
    # reader: one float32 multiply
    assert gff.from_i16(np.array([123, -32768, 1], np.int16)).tolist() == [
        float(np.float32(123) * np.float32(0.01)), float(np.float32(-32768) * np.float32(0.01)),
        float(np.float32(0.01))]


def _fields(nii, njj, nkk, seed, scale=3.0):
    rng = np.random.default_rng(seed)
    shape = (nii + 2, njj + 2, nkk + 2)
    return [(rng.standard_normal(shape) * scale).astype(np.float32) for _ in range(3)]


def _i16(v):
    """(Int16) of an already clamped float, as the reference casts it."""
    return int(np.trunc(np.float32(v))) if v == v else 0


def _loop_writer(mode, U, V, W, KK, hdr):
    """GFFWrite.cs:189-220 (mode 0), :279-328 (mode 1), :411-499 (mode 2) as literal loops."""
    nii, njj, nkk = U.shape[0] - 2, U.shape[1] - 2, U.shape[2] - 2
    out = bytearray(hdr)

    def trunc(x):
        v = np.float32(x) * np.float32(100)
        if v != v:
            return 0
        return _i16(min(max(v, np.float32(-32768)), np.float32(32767)))

    def rnd(x):
        v = np.rint(np.float32(x) * np.float32(100))
        if v > 32767:
            return 32767
        if v < -32768:
            return -32768
        return _i16(v)

    if mode == 0:
        for i in range(1, nii + 2):
            for j in range(1, njj + 2):
                for k in range(1, nkk + 2):
                    out += struct.pack("<hhh", trunc(U[i, j, k - 1]), trunc(V[i, j, k - 1]), trunc(W[i, j, k]))
    elif mode == 1:
        for k in range(1, nkk + 2):
            for i in range(1, nii + 2):
                for arr, kk in ((U, k - 1), (V, k - 1), (W, k)):
                    for j in range(1, njj + 2):
                        out += struct.pack("<h", trunc(arr[i, j, kk]))
    else:
        for i in range(1, nii + 1):
            for j in range(1, njj + 1):
                out += struct.pack("<h", int(KK[i, j]))
        for i in range(1, nii + 2):
            for j in range(1, njj + 2):
                k0 = max(int(KK[i, j]), 1)
                for k in range(k0, nkk + 2):
                    out += struct.pack("<h", rnd(U[i, j, k - 1]))
                for k in range(k0, nkk + 2):
                    out += struct.pack("<h", rnd(V[i, j, k - 1]))
                for k in range(k0, nkk + 2):
                    out += struct.pack("<h", rnd(W[i, j, k]))
    return bytes(out)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_pack_matches_reference_loops(mode):
    nii, njj, nkk = 5, 4, 6
    U, V, W = _fields(nii, njj, nkk, seed=mode)
    U[2, 3, 4] = np.nan
    V[1, 1, 0] = 500.0
    W[3, 2, 6] = -np.inf
    U[5, 4, 1] = np.float32(0.125)      # half-way cases of the terrain format's rounding
    V[4, 4, 3] = np.float32(-0.375)
    rng = np.random.default_rng(7)
    KK = rng.integers(0, 4, size=(nii + 2, njj + 2)).astype(np.int16)
    KK[1, 1] = nkk + 1                  # a column holding only its top level
    got = gff.pack(mode, U, V, W, kkart=KK, wind_dir=225.5, wind_speed=3.25, stab=4, dxk=2.0)
    nkk_word = nkk if mode == 0 else -nkk
    hdr = struct.pack("<iiiffifi", nkk_word, njj, nii, 225.5, 3.25, 4, 2.0, -1 - mode)
    assert got == _loop_writer(mode, U, V, W, KK, hdr)


def test_tke_payload():
    nii, njj, nkk = 3, 4, 5
    T = np.abs(_fields(nii, njj, nkk, seed=9)[0])
    T[1, 2, 3] = np.float32(0.125)
    T[2, 2, 2] = 1000.0
    got = gff.pack(gff.TKE, T, T, T, turb=T, wind_dir=10.0, wind_speed=1.0, stab=2, dxk=4.0)
    want = bytearray(struct.pack("<iiiffifi", nkk, njj, nii, 10.0, 1.0, 2, 4.0, -1))
    for i in range(1, nii + 1):                  # GFFWrite.cs:121-130
        for j in range(1, njj + 1):
            for k in range(1, nkk + 1):
                v = min(max(np.float32(T[i, j, k]) * np.float32(100), np.float32(-32768)), np.float32(32767))
                want += struct.pack("<h", int(np.rint(v)))
    assert got == bytes(want)
    assert struct.unpack_from("<h", got, 32 + 2 * (((1 - 1) * njj + (2 - 1)) * nkk + (3 - 1)))[0] == 12
    T[2, 3, 4] = np.nan
    with pytest.raises(ValueError):
        gff.pack(gff.TKE, T, T, T, turb=T)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_round_trip(mode):
    nii, njj, nkk = 6, 5, 7
    U, V, W = _fields(nii, njj, nkk, seed=10 + mode)
    KK = np.random.default_rng(3).integers(0, 5, size=(nii + 2, njj + 2)).astype(np.int16)
    p = gff.pack(mode, U, V, W, kkart=KK, dxk=1.5, stab=3, wind_dir=90.0, wind_speed=2.0)
    u, v, w, info = gff.unpack(p, nii, njj, nkk, 1.5, kkart=KK)
    assert info == (90.0, 2.0, 3, -1 - mode)
    conv = gff.to_i16_round if mode == 2 else gff.to_i16_trunc
    for got, src, ks in ((u, U, slice(0, nkk + 1)), (v, V, slice(0, nkk + 1)), (w, W, slice(1, nkk + 2))):
        want = np.zeros_like(src)
        want[1:, 1:, ks] = gff.from_i16(conv(src[1:, 1:, ks]))
        if mode == 2:     # levels below KKART are zero after reading the terrain format
            for i in range(1, nii + 2):
                for j in range(1, njj + 2):
                    k0 = max(int(KK[i, j]), 1)
                    lo = k0 - 1 if ks.start == 0 else k0
                    want[i, j, ks.start:lo] = 0.0
        np.testing.assert_array_equal(got, want)


def test_reader_rejections():
    nii, njj, nkk = 4, 3, 5
    U, V, W = _fields(nii, njj, nkk, seed=1)
    KK = np.ones((nii + 2, njj + 2), np.int16)
    p = gff.pack(2, U, V, W, kkart=KK, dxk=2.0)
    with pytest.raises(ValueError, match="z-direction"):
        gff.unpack(p, nii, njj, nkk + 1, 2.0, kkart=KK)
    with pytest.raises(ValueError, match="y-direction"):
        gff.unpack(p, nii, njj + 1, nkk, 2.0, kkart=KK)
    with pytest.raises(ValueError, match="x-direction"):
        gff.unpack(p, nii + 1, njj, nkk, 2.0, kkart=KK)
    with pytest.raises(ValueError, match="grid size"):
        gff.unpack(p, nii, njj, nkk, 2.5, kkart=KK)
    other = KK.copy()
    other[2, 2] = 3
    with pytest.raises(ValueError, match="terrain"):
        gff.unpack(p, nii, njj, nkk, 2.0, kkart=other)
    with pytest.raises(ValueError, match="shorter"):
        gff.unpack(p[:-2], nii, njj, nkk, 2.0, kkart=KK)
    q = gff.pack(0, U, V, W, dxk=2.0)
    with pytest.raises(ValueError, match="shorter"):
        gff.unpack(q[:-1], nii, njj, nkk, 2.0)
    # an unknown format flag: the reference's reader reads no further and reports success
    r = q[:28] + struct.pack("<i", -7) + q[32:]
    assert gff.unpack(r, nii, njj, nkk, 2.0)[:3] == (None, None, None)
