"""ERS IM level-0 packet walk (oracle restatement; TEST INFRASTRUCTURE ONLY).

Plain-Python restatement of the reference's two host passes over an ERS_SAR_0P measurement
data set, used to check the library's host forecast and its GPU unpack kernel:

* ``forecast``: FetchErsL0ImForecastMeta (envisat_format/src/ers_im_parse.cc:228-354);
* ``parse``: ParseErsLevel0ImPackets (envisat_format/src/ers_im_parse.cc:356-580), the parts
  that reach the focusing path (measurement bytes, SWST and PRI codes, the ISP-length and
  auxiliary-marker checks).

The reference parser needs Boost date_time and GDAL headers and so is not compiled here; no
reference test pins this path (parity of these two functions is unpinned).  No PATC
sensing-time correction is applied (ers_sbt.cc:56-84 applies one only when registered).
"""
from __future__ import annotations

import numpy as np

MDSR_BYTES = 11498      # ers_env_format.h:26
MEAS_BYTES = 11232      # ers_env_format.h:34
MEAS_OFFSET = 266       # 12 + 20 + 4 + 10 + 220 (ers_env_format.h:27-33)
DR_NO_MAX = 0xFFFFFFFF  # MaxValueForBits<uint32_t, 32>


def _be32(b, o):
    return (int(b[o]) << 24) | (int(b[o + 1]) << 16) | (int(b[o + 2]) << 8) | int(b[o + 3])


def _be16(b, o):
    return (int(b[o]) << 8) | int(b[o + 1])


def counter_gap(last: int, cur: int, limit: int) -> int:
    """parseutil::CounterGap (envisat_format/include/parse_util.h:33-46), unsigned 32-bit."""
    if (last + 1) & 0xFFFFFFFF == cur:
        return 1
    if cur < last:
        return (limit - last + cur + 1) & 0xFFFFFFFF
    return cur - last


def _dr_before(b, o) -> int:
    """InitializeDataRecordNo (ers_im_parse.cc:93-103)."""
    v = _be32(b, o + 32)
    return v - 1 if v != 0 else DR_NO_MAX


def forecast(blob: np.ndarray, start: tuple, stop: tuple, before_limit: int, after_limit: int):
    """FetchErsL0ImForecastMeta: (list of (offset, (days, s, us))), packets before start, after stop."""
    b = np.asarray(blob, dtype=np.uint8)
    n = b.size // MDSR_BYTES
    fc = []
    before = after = 0
    last_dr = _dr_before(b, 0)
    for i in range(n):
        o = i * MDSR_BYTES
        t = (_be32(b, o) - (1 << 32) if _be32(b, o) & 0x80000000 else _be32(b, o), _be32(b, o + 4), _be32(b, o + 8))
        if _be16(b, o + 24) != 11465:
            raise ValueError("FEP annotation's ISP length shall be 11465")
        dr = _dr_before(b, o)
        gap = counter_gap(last_dr, dr, DR_NO_MAX)
        if gap > 1:
            if not fc:
                raise ValueError("data record no. discontinuity before any packet")
            fill = gap - 1
            if fill > 900:
                raise ValueError(f"There are {fill} packets missing")
            prev = fc[-1]
            fc.extend([prev] * fill)
            if prev[1] < tuple(start):
                before += fill
            if prev[1] > tuple(stop):
                after += fill
        else:
            if t < tuple(start):
                before += 1
            if t > tuple(stop):
                after += 1
        if after > after_limit:
            after -= 1
            break
        last_dr = dr
        fc.append((o, t))
    if before > before_limit:
        drop = before - before_limit
        fc = fc[drop:]
        before -= drop
        if before_limit == 0:
            while fc and fc[0][1] < tuple(start):
                fc.pop(0)
    return fc, before, after


def parse(blob: np.ndarray, offsets) -> dict:
    """ParseErsLevel0ImPackets for the listed packets: raw lines, SWST / PRI codes, check bits."""
    b = np.asarray(blob, dtype=np.uint8)
    n = len(offsets)
    raw = np.empty((n, MEAS_BYTES), dtype=np.uint8)
    swst = np.empty(n, dtype=np.uint16)
    pri = np.empty(n, dtype=np.uint16)
    err = 0
    for y, o in enumerate(offsets):
        o = int(o)
        if _be16(b, o + 24) != 11465:
            err |= 1
        if b[o + 46] != 0xAA:
            err |= 2
        swst[y] = _be16(b, o + 58)
        pri[y] = _be16(b, o + 60)
        raw[y] = b[o + MEAS_OFFSET:o + MEAS_OFFSET + MEAS_BYTES]
    return dict(raw=raw, swst=swst, pri=pri, errors=err)
