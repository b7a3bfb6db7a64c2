"""ENVISAT ASAR FBAQ4 raw records: layout helpers, a synthetic instrument table and an encoder.

Record layout (what ConvertAsarImBlocksToComplex reads, envisat_format/src/envisat_format_kernels.cu:160-209):
a 2-byte little-endian length L of the block data, then 64-byte blocks of one block-id byte and
63 codeword bytes, the I code in the high nibble and the Q code in the low one.  A code is
sign-magnitude (bit 3 = sign); the instrument file's reconstruction table holds 4096 floats at
index 256 * level + block id, level 0..15 from the most negative to the most positive value
(Fbaq4IndexCalc, envisat_format/include/envisat_parse_util.cuh:75-84).

The real tables come from the ASAR instrument auxiliary file, which is not available here; the
synthetic table below is a 16-level Gaussian quantiser (Max, IRE Trans. IT-6, 1960) scaled by a
block-id gain of 0.25 dB per step, which is the structure of the on-board adaptive quantiser.
"""
from __future__ import annotations

import numpy as np

# output levels of the 16-level minimum-mean-square-error quantiser of a unit Gaussian (Max 1960)
_MAX16 = np.array([0.1284, 0.3881, 0.6568, 0.9424, 1.2562, 1.6181, 2.0690, 2.7326])
LEVELS = np.concatenate([-_MAX16[::-1], _MAX16])  # level 0 .. 15, ascending
SIGMA0 = 0.5       # block id 0 scale
STEP_DB = 0.25     # scale step per block id


def block_bytes(samples: int) -> int:
    """Block-data bytes holding `samples` samples: 63 per 64-byte block, one id byte per block."""
    full, rem = divmod(int(samples), 63)
    return 64 * full + (rem + 1 if rem else 0)


def record_samples(length: int) -> int:
    """Samples in a record whose block data is `length` bytes (envisat_im_parse.cc:589-592)."""
    return (length // 64) * 63 + length % 64 - (1 if length % 64 else 0)


def level_of_code(code):
    """Level (0..15) of a 4-bit sign-magnitude code."""
    code = np.asarray(code)
    return np.where(code > 7, 15 - code, 8 + code)


def code_of_level(level):
    level = np.asarray(level)
    return np.where(level >= 8, level - 8, 15 - level)


def table_index(block, code):
    """Fbaq4Index: 256 * level + block id."""
    return 256 * level_of_code(code) + np.asarray(block)


def block_scale(block_ids) -> np.ndarray:
    return SIGMA0 * 10.0 ** (np.asarray(block_ids, dtype=np.float64) * STEP_DB / 20.0)


def synthetic_tables(q_gain: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """(i_lut, q_lut): 4096 float32 each, index 256 * level + block id."""
    sig = block_scale(np.arange(256))
    t = (LEVELS[:, None] * sig[None, :]).astype(np.float32).reshape(-1)
    return t, (LEVELS[:, None] * sig[None, :] * q_gain).astype(np.float32).reshape(-1)


def encode(iv: np.ndarray, qv: np.ndarray, samples: np.ndarray, record_bytes: int, q_gain: float = 1.0,
           chunk: int = 1024) -> np.ndarray:
    """Encode float I/Q rows [na, n] into FBAQ4 records [na, record_bytes] with the synthetic
    tables: per 63-sample block the block id whose scale is nearest (in dB) to the block RMS,
    per sample the nearest table level.  Record y holds samples[y] samples."""
    na, n = iv.shape
    samples = np.asarray(samples, dtype=np.int64)
    out = np.zeros((na, record_bytes), dtype=np.uint8)
    nb = (n + 62) // 63
    thr = (LEVELS[1:] + LEVELS[:-1]) / 2
    col = np.arange(nb * 63)
    for y0 in range(0, na, chunk):
        y1 = min(na, y0 + chunk)
        m = y1 - y0
        keep = col[None, :] < samples[y0:y1, None]
        ivp = np.zeros((m, nb * 63))
        qvp = np.zeros((m, nb * 63))
        ivp[:, :n] = iv[y0:y1]
        qvp[:, :n] = qv[y0:y1]
        ivp = np.where(keep, ivp, 0.0).reshape(m, nb, 63)
        qvp = np.where(keep, qvp, 0.0).reshape(m, nb, 63)
        cnt = np.maximum(keep.reshape(m, nb, 63).sum(axis=2), 1)
        rms = np.sqrt((ivp ** 2 + qvp ** 2).sum(axis=2) / (2 * cnt))
        bid = np.clip(np.rint(20 * np.log10(np.maximum(rms, 1e-12) / SIGMA0) / STEP_DB), 0, 255).astype(np.int64)
        sig = block_scale(bid)[:, :, None]
        li = np.searchsorted(thr, ivp / sig)
        lq = np.searchsorted(thr, qvp / (sig * q_gain))
        cw = (code_of_level(li) << 4 | code_of_level(lq)).astype(np.uint8)
        blocks = np.concatenate([bid.astype(np.uint8)[:, :, None], cw], axis=2).reshape(m, nb * 64)
        for k in range(m):
            length = block_bytes(int(samples[y0 + k]))
            out[y0 + k, 0] = length & 0xFF
            out[y0 + k, 1] = length >> 8
            out[y0 + k, 2:2 + length] = blocks[k, :length]
    return out
