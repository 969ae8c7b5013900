"""CPU restatement of GRAL's flow-field (.gff) and turbulence (.tke) cache formats.

Test infrastructure only: the tests, the smoke check and the bench's CPU baseline compare the
device pack/unpack of ``libgralprog.so`` with these functions; nothing in the product imports
this module.  Parity unpinned: the reference holds no .gff/.tke files and its .NET runtime is not
available here, so these functions follow the reference source line by line (cited per function)
and are pinned only by hand-computed known answers in the tests.

Fields are flat ``[NII+2][NJJ+2][NKK+2]`` float32 arrays, k fastest, as the solver's ABI holds
them: ``UK[i][j][k]`` of the reference is ``uk[i, j, k]``.  Payloads are the bytes of the zip
entry (header + data); the zip container is not part of the format functions.
"""

import struct

import numpy as np

HEADER = struct.Struct("<iiiffifi")   # NKK, NJJ, NII, WindDirGral, WindVelGral, StabClass, DXK, flag
HEADER_BYTES = HEADER.size

COLUMNS, LEVELS, TERRAIN, TKE = 0, 1, 2, 3
_F100 = np.float32(100.0)
_F001 = np.float32(0.01)


def _clamp_cast(v):
    """Clamp float32 ``v`` to [-32768, 32767] and convert toward zero; NaN gives 0.

    ``(Int16)(Math.Max(Int16.MinValue, Math.Min(Int16.MaxValue, v)))`` (GFFWrite.cs:196-216) and
    the if/else clamp before ``(Int16)_val`` (GFFWrite.cs:296-309) agree on every input.  NaN:
    Math.Min/Max propagate it (IEEE 754-2019) and the x64 truncating conversion gives
    0x80000000, whose low 16 bits are 0; newer .NET runtimes saturate NaN to 0 too.
    """
    v = np.asarray(v, np.float32)
    nan = np.isnan(v)
    c = np.clip(np.where(nan, np.float32(0), v), np.float32(-32768), np.float32(32767))
    return np.trunc(c).astype(np.int16)


def to_i16_trunc(x):
    """int16 of ``x * 100`` as modes -1 and -2 write it (float32 product, GFFWrite.cs:198, 296)."""
    return _clamp_cast(np.asarray(x, np.float32) * _F100)


def to_i16_round(x):
    """``MathF.Round(x * 100)`` (half to even), then clamp and cast (GFFWrite.cs:446-458)."""
    return _clamp_cast(np.rint(np.asarray(x, np.float32) * _F100))


def from_i16(s):
    """``(float)(int16 * 0.01F)`` (GFFRead.cs:223, 249, 298): one float32 multiply."""
    return np.asarray(s, np.int16).astype(np.float32) * _F001


def header(nkk_word, njj, nii, wind_dir, wind_speed, stab, dxk, flag):
    """The 32-byte header of every payload (GFFWrite.cs:180-188, 269-277, 401-409, 113-121)."""
    return HEADER.pack(int(nkk_word), int(njj), int(nii), float(np.float32(wind_dir)),
                       float(np.float32(wind_speed)), int(stab), float(np.float32(dxk)), int(flag))


def _dims(uk):
    ni2, nj2, nk2 = uk.shape
    return ni2 - 2, nj2 - 2, nk2 - 2


def pack(mode, uk, vk, wk, *, kkart=None, turb=None, wind_dir=0.0, wind_speed=0.0, stab=0, dxk=1.0):
    """Payload bytes of ``mode`` for one situation (GFFWrite.cs).

    mode 0 (:167-254) i, j outer, k inner: U[k-1], V[k-1], W[k];
    mode 1 (:256-386) k outer, rows i, each row U, V, W over j;
    mode 2 (:388-520) KKART of the inner columns, then per column k = max(KKART,1)..NKK+1 of U,
    then V, then W, rounded half to even;
    mode 3 (:83-133) .tke: TURB of i = 1..NII, j = 1..NJJ, k = 1..NKK via Convert.ToInt16, which
    rounds half to even and throws on NaN (raised here as ValueError).
    """
    uk = np.asarray(uk, np.float32)
    nii, njj, nkk = _dims(uk)
    I = slice(1, nii + 2)
    J = slice(1, njj + 2)
    if mode == COLUMNS:
        body = np.stack([to_i16_trunc(uk[I, J, 0:nkk + 1]), to_i16_trunc(vk[I, J, 0:nkk + 1]),
                         to_i16_trunc(wk[I, J, 1:nkk + 2])], axis=-1)          # [i][j][k][c]
        hdr = header(nkk, njj, nii, wind_dir, wind_speed, stab, dxk, -1)
    elif mode == LEVELS:
        comp = [to_i16_trunc(uk[I, J, 0:nkk + 1]), to_i16_trunc(vk[I, J, 0:nkk + 1]),
                to_i16_trunc(wk[I, J, 1:nkk + 2])]                              # [i][j][k]
        body = np.stack([c.transpose(2, 0, 1) for c in comp], axis=2)           # [k][i][c][j]
        hdr = header(-nkk, njj, nii, wind_dir, wind_speed, stab, dxk, -2)
    elif mode == TERRAIN:
        kk = np.asarray(kkart, np.int16)
        parts = [kk[1:nii + 1, 1:njj + 1].astype(np.int16).ravel()]
        for i in range(1, nii + 2):
            for j in range(1, njj + 2):
                k0 = max(int(kk[i, j]), 1)
                if nkk + 2 - k0 < 0:
                    raise ValueError("KKART above NKK+1 leaves no room for a terrain-format record")
                parts += [to_i16_round(uk[i, j, k0 - 1:nkk + 1]), to_i16_round(vk[i, j, k0 - 1:nkk + 1]),
                          to_i16_round(wk[i, j, k0:nkk + 2])]
        body = np.concatenate(parts)
        hdr = header(-nkk, njj, nii, wind_dir, wind_speed, stab, dxk, -3)
    elif mode == TKE:
        v = np.asarray(turb, np.float32)[1:nii + 1, 1:njj + 1, 1:nkk + 1] * _F100
        if np.isnan(v).any():
            raise ValueError("non-finite TKE value: Convert.ToInt16 throws")
        body = np.rint(np.clip(v, np.float32(-32768), np.float32(32767))).astype(np.int16)
        hdr = header(nkk, njj, nii, wind_dir, wind_speed, stab, dxk, -1)
    else:
        raise ValueError(f"unknown payload mode {mode}")
    return hdr + np.ascontiguousarray(body, dtype="<i2").tobytes()


def unpack(payload, nii, njj, nkk, dxk, kkart=None):
    """Fields read from a flow-field payload (GFFRead.cs:181-320).

    Returns ``(uk, vk, wk, info)``: flat ``[NII+2][NJJ+2][NKK+2]`` float32 arrays holding the
    entries the file sets (levels below KKART set to 0 in the terrain format) and 0 elsewhere,
    and ``info = (wind_dir, wind_speed, stability_class, flag)``.  A header that does not match
    the grid or DXK, a terrain KKART that differs from ``kkart`` or a payload too short for its
    grid raises ValueError, as the reference's reader fails on such a file.  A flag other than
    -1, -2, -3 reads nothing further (the reference then returns success): the arrays are None.
    """
    if len(payload) < HEADER_BYTES:
        raise ValueError("payload shorter than its header")
    h0, h1, h2, wdir, wspd, stab, cell, flag = HEADER.unpack_from(payload, 0)
    if h0 == -2 ** 31 or abs(h0) != nkk:
        raise ValueError("field dimension in z-direction does not match")
    if h1 != njj:
        raise ValueError("field dimension in y-direction does not match")
    if h2 != nii:
        raise ValueError("field dimension in x-direction does not match")
    if np.float32(cell) != np.float32(dxk):
        raise ValueError("horizontal grid size does not match")
    info = (wdir, wspd, stab, flag)
    if flag not in (-1, -2, -3):
        return None, None, None, info
    data = np.frombuffer(payload, dtype="<i2", offset=HEADER_BYTES,
                         count=(len(payload) - HEADER_BYTES) // 2)
    shape = (nii + 2, njj + 2, nkk + 2)
    uk, vk, wk = (np.zeros(shape, np.float32) for _ in range(3))
    ni, nj, nk = nii + 1, njj + 1, nkk + 1
    I = slice(1, nii + 2)
    J = slice(1, njj + 2)
    if flag in (-1, -2):
        n = 3 * ni * nj * nk
        if data.size < n:
            raise ValueError("payload shorter than its grid")
        if flag == -1:
            d = data[:n].reshape(ni, nj, nk, 3)                                  # [i][j][k][c]
            u, v, w = d[..., 0], d[..., 1], d[..., 2]
        else:
            d = data[:n].reshape(nk, ni, 3, nj)                                  # [k][i][c][j]
            u, v, w = (d[:, :, c, :].transpose(1, 2, 0) for c in range(3))
        uk[I, J, 0:nkk + 1] = from_i16(u)
        vk[I, J, 0:nkk + 1] = from_i16(v)
        wk[I, J, 1:nkk + 2] = from_i16(w)
        return uk, vk, wk, info
    kk = np.asarray(kkart, np.int16)
    if data.size < nii * njj or not np.array_equal(data[:nii * njj].reshape(nii, njj), kk[1:nii + 1, 1:njj + 1]):
        raise ValueError("building or terrain of flow field does not match")
    pos = nii * njj
    for i in range(1, nii + 2):
        for j in range(1, njj + 2):
            k0 = max(int(kk[i, j]), 1)
            n = nkk + 2 - k0
            if n < 0:
                raise ValueError("KKART above NKK+1 leaves no room for a terrain-format record")
            if pos + 3 * n > data.size:
                raise ValueError("payload shorter than its grid")
            rec = data[pos:pos + 3 * n]
            pos += 3 * n
            uk[i, j, k0 - 1:nkk + 1] = from_i16(rec[:n])
            vk[i, j, k0 - 1:nkk + 1] = from_i16(rec[n:2 * n])
            wk[i, j, k0:nkk + 2] = from_i16(rec[2 * n:])
    return uk, vk, wk, info
