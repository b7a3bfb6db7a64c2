"""ERS IM and ENVISAT ASAR IM level-0 packet walks (oracle restatement; TEST INFRASTRUCTURE ONLY).

Plain-Python restatement of the reference's two host passes over an ERS_SAR_0P measurement
data set, used to check the library's host forecast and its GPU unpack kernel:

* ``forecast``: FetchErsL0ImForecastMeta (envisat_format/src/ers_im_parse.cc:228-354);
* ``parse``: ParseErsLevel0ImPackets (envisat_format/src/ers_im_parse.cc:356-580), the parts
  that reach the focusing path (measurement bytes, SWST and PRI codes, the ISP-length and
  auxiliary-marker checks).

And of the ENVISAT ASAR IM (ASA_IM__0P) walk:

* ``asar_forecast``: FetchEnvisatL0ImForecastMeta (envisat_format/src/envisat_im_parse.cc:297-385);
* ``asar_parse``: ParseEnvisatLevel0ImPackets (:387-676) with ForecastMaxBlockDataLength
  (:159-197): FBAQ4 records (2-byte little-endian length, sample blocks), SWST / PRI codes and
  sensing times per line.  The reference leaves the bytes after a record's blocks
  uninitialised; here they are zero.

The reference parsers need Boost date_time and GDAL headers and so are not compiled here; no
reference test pins this path (parity of these functions is unpinned).  No PATC
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


# ---------------------------------------------------------------- ENVISAT ASAR IM
def _asar_header(b, o):
    """FetchPacketFrom (envisat_im_parse.cc:246-272) plus the fields the parse reads."""
    t = (_be32(b, o) - (1 << 32) if _be32(b, o) & 0x80000000 else _be32(b, o), _be32(b, o + 4), _be32(b, o + 8))
    return dict(time=t, isp_length=_be16(b, o + 24), packet_length=_be16(b, o + 36),
                datafield_length=_be16(b, o + 38), mode=int(b[o + 41]), echo=bool(b[o + 52] & 0x80),
                cal=bool(b[o + 52] & 0x20), pri=_be16(b, o + 54), swst=_be16(b, o + 56),
                next=o + 39 + _be16(b, o + 24))


def asar_forecast(blob, num_dsr: int, start: tuple, stop: tuple, before_limit: int, after_limit: int):
    """FetchEnvisatL0ImForecastMeta: (list of (offset, time)), packets before start, after stop."""
    b = np.asarray(blob, dtype=np.uint8)
    fc = []
    before = after = 0
    cal = False
    o = 0
    for _ in range(num_dsr):
        h = _asar_header(b, o)
        if h["datafield_length"] != 29:
            raise ValueError("Date Field Header Length should be 29")
        cur = (o, h["time"])
        o = h["next"]
        cal = h["cal"]
        if not fc and not h["echo"]:
            continue
        if not h["echo"] and not h["cal"]:
            continue
        if h["time"] < tuple(start):
            before += 1
        if h["time"] > tuple(stop):
            after += 1
        if after > after_limit:
            after -= 1
            break
        fc.append(cur)
    if before > before_limit:
        drop = before - before_limit
        fc = fc[drop:]
        before -= drop
        while fc:
            if _asar_header(b, fc[0][0])["echo"]:
                break
            if not cal:
                raise ValueError("Programming error detected")
            fc.pop(0)
            before -= 1
    return fc, before, after


def _block_samples(n: int) -> int:
    return (n // 64) * 63 + n % 64 - (1 if n % 64 else 0)


def _add_micros(t, add):
    d, s, u = t
    u += add
    s += u // 1_000_000
    u %= 1_000_000
    d += s // 86400
    s %= 86400
    return (d, s, u)


def asar_parse(blob, offsets, range_sampling_rate: float) -> dict:
    """ParseEnvisatLevel0ImPackets for the listed packets: FBAQ4 records, codes, times."""
    b = np.asarray(blob, dtype=np.uint8)
    n = len(offsets)
    o = int(offsets[0])
    most_len, echoes = 0, 0
    for _ in range(n):            # ForecastMaxBlockDataLength: n consecutive packets
        h = _asar_header(b, o)
        if h["echo"]:
            most_len = max(most_len, (h["packet_length"] - 29) & 0xFFFF)
            echoes += 1
        o = h["next"]
    if echoes < 10:
        raise ValueError("Could not gather atleast 10 echo packets")
    stride = most_len + 2
    rec = np.zeros((n, stride), dtype=np.uint8)
    swst = np.zeros(n, dtype=np.uint16)
    pri = np.zeros(n, dtype=np.uint16)
    times = [None] * n
    most = 0
    for k, off in enumerate(offsets):
        off = int(off)
        h = _asar_header(b, off)
        if h["mode"] != 0x54:
            raise ValueError("Expected only IM mode packets")
        if h["echo"]:
            ln = (h["packet_length"] - 29) & 0xFFFF
            rec[k, 0], rec[k, 1] = ln & 0xFF, ln >> 8
            rec[k, 2:2 + ln] = b[off + 68:off + 68 + ln]
            swst[k], pri[k], times[k] = h["swst"], h["pri"], h["time"]
            most = max(most, _block_samples(ln))
        elif h["cal"] and k > 0:
            rec[k] = rec[k - 1]
            swst[k], pri[k] = swst[k - 1], pri[k - 1]
            prf = np.float32(range_sampling_rate) / np.float32(pri[k - 1])
            add = int(np.float64(np.float32(1.0) / prf) * 10e5)
            times[k] = _add_micros(times[k - 1], add)
        else:
            raise ValueError("Programming error detected")
    if most != _block_samples(most_len):
        raise ValueError("Post-parse max samples do not equal with forecast")
    return dict(records=rec, swst=swst, pri=pri, times=times, record_bytes=stride, max_samples=most)
