"""ERS IM (ERS_SAR_0P) and ENVISAT ASAR IM (ASA_IM__0P) level-0 packets in and out of the library.

* ``forecast``: the packet list of the product's lines (asarf_ers_l0_forecast: record-number
  gaps filled with copies of the previous packet, sensing-time window), on the host.
* ``unpack``: the listed packets' measurement bytes, SWST and PRI codes gathered into device
  raw lines on the GPU (asarf_ers_l0_unpack), ready for ``FocusPlan.focus``.
* ``write_packets``: a synthetic measurement data set from raw lines and header fields, in the
  MDSR layout the reference parses (for tests and benchmarks; no L0 product is available).

MDSR layout (11498 bytes, big-endian fields): ISP sensing time (days, seconds, microseconds:
3 x 4 bytes), FEP annotation (20 bytes, ISP length 11465 at bytes 24-25), data record number
(32-35), IDHT header (36-45: packet counter, subcommutation counter, 8 bytes), auxiliary data
(46-265: 0xAA, orbit byte, 4-byte on-board time, activity, flags, 4-byte image format
counter, SWST code at 58-59, PRI code at 60-61, calibration data), measurement data
(266-11497: 5616 I/Q byte pairs).

ASAR IM source packets (variable length, big-endian fields): ISP sensing time (0-11), FEP
annotation (12-31: its time, ISP length at 24-25), packet ID (32-33), sequence control
(34-35), packet length (36-37), data field header length 29 (38-39), data field header (40-67:
mode ID 0x54 at 41, 40-bit on-board time at 42-46, mode packet count at 48-50, beam set and
compression ratio at 51, echo / noise / calibration flags and the cycle packet count at 52-53,
PRI code at 54-55, SWST code at 56-57, echo window code at 58-59, converter / polarisation at
60-61, tx pulse code at 62-63, chirp bandwidth code at 64, aux monitor level at 65, resampling
factor at 66-67), then packet length - 29 bytes of FBAQ4 sample blocks.  The next packet
starts 39 + ISP length bytes on.  ``asar_forecast`` / ``asar_lines`` / ``asar_unpack`` are the
ASAR counterparts of the ERS functions (asarf_asar_l0_*): the unpack writes FBAQ4 records.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

MDSR_BYTES = 11498
MEASUREMENT_BYTES = 11232
MEASUREMENT_OFFSET = 266
ERR_ISP_LENGTH = 1
ERR_AUX_MARKER = 2


class Mjd(C.Structure):
    _fields_ = [("days", C.c_int32), ("seconds", C.c_uint32), ("micros", C.c_uint32)]


def mjd(us_since_2000: int) -> tuple[int, int, int]:
    """(days, seconds of day, microseconds) of a time in microseconds since 2000-01-01."""
    d, r = divmod(int(us_since_2000), 86_400_000_000)
    s, u = divmod(r, 1_000_000)
    return int(d), int(s), int(u)


def write_packets(raw_lines: np.ndarray, swst: np.ndarray, pri: np.ndarray, record_numbers: np.ndarray,
                  times_us: np.ndarray, isp_length: int = 11465, aux_marker: int = 0xAA) -> np.ndarray:
    """Measurement data set (uint8 [n * 11498]) holding one packet per raw line."""
    raw_lines = np.ascontiguousarray(raw_lines, dtype=np.uint8)
    n = raw_lines.shape[0]
    if raw_lines.shape[1] != MEASUREMENT_BYTES:
        raise ValueError("ERS measurement data are 11232 bytes (5616 I/Q pairs) per line")
    pk = np.zeros((n, MDSR_BYTES), dtype=np.uint8)
    t = np.array([mjd(v) for v in times_us], dtype=np.int64).reshape(n, 3)

    def put32(col, vals):
        v = np.asarray(vals, dtype=np.uint64) & 0xFFFFFFFF
        for k in range(4):
            pk[:, col + k] = (v >> np.uint64(8 * (3 - k))) & np.uint64(0xFF)

    def put16(col, vals):
        v = np.asarray(vals, dtype=np.uint32)
        pk[:, col] = (v >> 8) & 0xFF
        pk[:, col + 1] = v & 0xFF

    put32(0, t[:, 0] & 0xFFFFFFFF)
    put32(4, t[:, 1])
    put32(8, t[:, 2])
    put16(24, np.full(n, isp_length))
    put32(32, record_numbers)
    pk[:, 36] = (np.arange(n) // 1679 + 1) & 0xFF           # packet counter
    pk[:, 37] = np.arange(n) % 48 + 1                          # subcommutation counter
    pk[:, 46] = aux_marker
    put32(48, np.arange(n) // 4)                               # on-board time, every 4th PRI
    pk[:, 52] = 0b10101000                                     # echo
    put32(54, np.arange(n) + 1)                                # image format counter
    put16(58, swst)
    put16(60, pri)
    pk[:, MEASUREMENT_OFFSET:] = raw_lines
    return pk.reshape(-1)


def forecast(blob: np.ndarray, start: tuple, stop: tuple, before: int, after: int, lib=None):
    """(offsets int64 [lines], sensing times [(days, s, us)], packets before start, after stop)."""
    lib = lib or _lib.load_library()
    blob = np.ascontiguousarray(blob, dtype=np.uint8)
    n = blob.size // MDSR_BYTES
    fn = lib.asarf_ers_l0_forecast
    fn.restype = C.c_int

    def call(offs, times, cap):
        b, a, cnt = C.c_int64(int(before)), C.c_int64(int(after)), C.c_int64()
        _lib.check(lib, fn(C.c_void_p(blob.ctypes.data), C.c_int64(blob.size), C.c_int64(n), C.c_int64(MDSR_BYTES),
                           C.byref(Mjd(*start)), C.byref(Mjd(*stop)), C.byref(b), C.byref(a),
                           None if offs is None else C.c_void_p(offs.ctypes.data), times, C.c_int64(cap),
                           C.byref(cnt)), "ers_l0_forecast")
        return b.value, a.value, cnt.value

    _, _, k = call(None, None, 0)          # the line count first
    offs = np.empty(max(k, 1), dtype=np.int64)
    times = (Mjd * max(k, 1))()
    b, a, k = call(offs, times, k)
    return offs[:k].copy(), [(times[i].days, times[i].seconds, times[i].micros) for i in range(k)], b, a


def unpack(d_blob, d_offsets, lines: int, d_raw, d_swst=None, d_pri=None, d_errors=None, lib=None, stream: int = 0):
    """Gather the listed packets into raw lines on the device (torch tensors or device pointers)."""
    lib = lib or _lib.load_library()

    def ptr(x):
        return None if x is None else (x if isinstance(x, int) else (x.ctypes.data if isinstance(x, np.ndarray)
                                                                    else x.data_ptr()))
    fn = lib.asarf_ers_l0_unpack
    fn.restype = C.c_int
    _lib.check(lib, fn(C.c_void_p(ptr(d_blob)), C.c_void_p(ptr(d_offsets)), C.c_int32(lines), C.c_void_p(ptr(d_raw)),
                       C.c_void_p(ptr(d_swst)), C.c_void_p(ptr(d_pri)), C.c_void_p(ptr(d_errors)),
                       C.c_void_p(stream)), "ers_l0_unpack")


# ---------------------------------------------------------------- ENVISAT ASAR IM
ASAR_HEADER_BYTES = 68
FLAG_ECHO, FLAG_NOISE, FLAG_CAL = 0x80, 0x40, 0x20
ERR_DATA_FIELD, ERR_MODE, ERR_LENGTH = 1, 2, 4


def write_asar_packets(records: np.ndarray, swst: np.ndarray, pri: np.ndarray, times_us: np.ndarray,
                       flags: np.ndarray | None = None, mode_id: int = 0x54, datafield_length: int = 29):
    """(measurement data set uint8 [bytes], packet count): one source packet per FBAQ4 record
    (2-byte little-endian block-data length, then the blocks), its sample blocks the record's.
    ``flags`` per packet (FLAG_ECHO default, FLAG_CAL, FLAG_NOISE)."""
    records = np.ascontiguousarray(records, dtype=np.uint8)
    n = records.shape[0]
    flags = np.full(n, FLAG_ECHO, dtype=np.uint8) if flags is None else np.asarray(flags, dtype=np.uint8)
    lengths = records[:, 0].astype(np.int64) | (records[:, 1].astype(np.int64) << 8)
    sizes = ASAR_HEADER_BYTES + lengths
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    blob = np.zeros(int(sizes.sum()), dtype=np.uint8)

    def be(v, nbytes):
        return [(int(v) >> (8 * (nbytes - 1 - k))) & 0xFF for k in range(nbytes)]

    for i in range(n):
        o = int(starts[i])
        d, s, u = mjd(int(times_us[i]))
        hdr = np.zeros(ASAR_HEADER_BYTES, dtype=np.uint8)
        t = be(d & 0xFFFFFFFF, 4) + be(s, 4) + be(u, 4)
        hdr[0:12] = t
        hdr[12:24] = t                                  # FEP time
        hdr[24:26] = be(lengths[i] + 29, 2)             # ISP length: the packet is 39 + it bytes
        hdr[32:34] = be(0x0CB0, 2)                      # packet ID
        hdr[34:36] = be(0xC000 | (i & 0x3FFF), 2)       # sequence control
        hdr[36:38] = be(lengths[i] + 29, 2)             # packet length
        hdr[38:40] = be(datafield_length, 2)
        hdr[41] = mode_id
        hdr[42:47] = be(i * 7, 5)                       # on-board time
        hdr[48:51] = be(i, 3)                           # mode packet count
        hdr[51] = (1 << 2) | 1                          # beam set 1, compression ratio 1
        hdr[52] = int(flags[i]) | ((i >> 8) & 0x0F)
        hdr[53] = i & 0xFF
        hdr[54:56] = be(pri[i], 2)
        hdr[56:58] = be(swst[i], 2)
        hdr[58:60] = be(max(0, lengths[i] - (lengths[i] + 63) // 64), 2)   # echo window code
        blob[o:o + ASAR_HEADER_BYTES] = hdr
        blob[o + ASAR_HEADER_BYTES:o + int(sizes[i])] = records[i, 2:2 + lengths[i]]
    return blob, n


def asar_forecast(blob: np.ndarray, num_dsr: int, start: tuple, stop: tuple, before: int, after: int, lib=None):
    """(offsets int64 [lines], sensing times, packets before start, after stop): asarf_asar_l0_forecast."""
    lib = lib or _lib.load_library()
    blob = np.ascontiguousarray(blob, dtype=np.uint8)
    fn = lib.asarf_asar_l0_forecast
    fn.restype = C.c_int

    def call(offs, times, cap):
        b, a, cnt = C.c_int64(int(before)), C.c_int64(int(after)), C.c_int64()
        _lib.check(lib, fn(C.c_void_p(blob.ctypes.data), C.c_int64(blob.size), C.c_int64(int(num_dsr)),
                           C.byref(Mjd(*start)), C.byref(Mjd(*stop)), C.byref(b), C.byref(a),
                           None if offs is None else C.c_void_p(offs.ctypes.data), times, C.c_int64(cap),
                           C.byref(cnt)), "asar_l0_forecast")
        return b.value, a.value, cnt.value

    _, _, k = call(None, None, 0)
    offs = np.empty(max(k, 1), dtype=np.int64)
    times = (Mjd * max(k, 1))()
    b, a, k = call(offs, times, k)
    return offs[:k].copy(), [(times[i].days, times[i].seconds, times[i].micros) for i in range(k)], b, a


def asar_lines(blob: np.ndarray, offsets: np.ndarray, range_sampling_rate: float, lib=None):
    """(source packet offsets int64 [lines], sensing times, record_bytes, max samples):
    asarf_asar_l0_lines."""
    lib = lib or _lib.load_library()
    blob = np.ascontiguousarray(blob, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    k = offsets.size
    src = np.empty(max(k, 1), dtype=np.int64)
    times = (Mjd * max(k, 1))()
    rb, ms = C.c_int32(), C.c_int32()
    fn = lib.asarf_asar_l0_lines
    fn.restype = C.c_int
    _lib.check(lib, fn(C.c_void_p(blob.ctypes.data), C.c_int64(blob.size), C.c_void_p(offsets.ctypes.data),
                       C.c_int64(k), C.c_float(range_sampling_rate), C.c_void_p(src.ctypes.data), times,
                       C.byref(rb), C.byref(ms)), "asar_l0_lines")
    return src[:k].copy(), [(times[i].days, times[i].seconds, times[i].micros) for i in range(k)], rb.value, ms.value


def asar_unpack(d_blob, d_src_offsets, lines: int, record_bytes: int, d_records, d_swst=None, d_pri=None,
                d_errors=None, lib=None, stream: int = 0):
    """FBAQ4 records of the listed lines on the device (asarf_asar_l0_unpack)."""
    lib = lib or _lib.load_library()

    def ptr(x):
        return None if x is None else (x if isinstance(x, int) else (x.ctypes.data if isinstance(x, np.ndarray)
                                                                    else x.data_ptr()))
    fn = lib.asarf_asar_l0_unpack
    fn.restype = C.c_int
    _lib.check(lib, fn(C.c_void_p(ptr(d_blob)), C.c_void_p(ptr(d_src_offsets)), C.c_int32(lines),
                       C.c_int32(record_bytes), C.c_void_p(ptr(d_records)), C.c_void_p(ptr(d_swst)),
                       C.c_void_p(ptr(d_pri)), C.c_void_p(ptr(d_errors)), C.c_void_p(stream)), "asar_l0_unpack")
