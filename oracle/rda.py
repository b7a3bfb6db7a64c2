"""CPU restatement of the reference's range-Doppler focusing chain.

Layout follows the reference: a padded complex image ``img[az_pad][rg_pad]``
(row = azimuth line, column = range sample), data block top-left
(cuda_util/device_padded_image.cuh:13-27).  FFTs are FP64 (scipy.fft); the
reference runs them in float32 through cuFFT, so agreement is to float32
rounding, not bit-exact.  Values on which the reference branches are computed
with its float32 operation order (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

from . import geometry as geo

F32 = np.float32
PI32 = F32(math.pi)


def _workers() -> int:
    import os
    return max(1, os.cpu_count() or 1)


# --------------------------------------------------------------------------- float32 helpers

def _fix_midpoints(s, err):
    """Round binary64 s (+ residual err) to float32 correctly."""
    r = s.astype(np.float32)
    rd = r.astype(np.float64)
    # only a value exactly halfway between two float32 neighbours can round wrongly
    nb = np.where(rd > s, np.nextafter(r, np.float32(-np.inf)), np.nextafter(r, np.float32(np.inf)))
    mid = (rd + nb.astype(np.float64)) / 2
    is_mid = (s == mid)
    toward_nb = np.where(nb.astype(np.float64) > rd, err > 0, err < 0)
    away_nb = np.where(nb.astype(np.float64) > rd, err < 0, err > 0)
    out = np.where(is_mid & toward_nb, nb, r)
    out = np.where(is_mid & away_nb, r, out)
    return out.astype(np.float32)


def fmaf(a, b, c) -> np.ndarray:
    """Exact float32 fused multiply-add (vectorised)."""
    a = np.asarray(a, dtype=np.float32).astype(np.float64)
    b = np.asarray(b, dtype=np.float32).astype(np.float64)
    c = np.asarray(c, dtype=np.float32).astype(np.float64)
    p = a * b
    s = p + c
    bb = s - p
    err = (p - (s - bb)) + (c - bb)
    return _fix_midpoints(s, err)


def polyval_f32(poly, x) -> np.ndarray:
    """Device ``Polyval<N>`` in float32 with contracted multiply-add
    (sar/range_doppler_algorithm.cu:97-105, sar/srgr.cu:40-47)."""
    x = np.asarray(x, dtype=np.float32)
    r = np.zeros_like(x, dtype=np.float32)
    for e in np.asarray(poly, dtype=np.float64):
        r = fmaf(r, x, np.float32(e))
    return r


def roundf_away(v: np.ndarray) -> np.ndarray:
    """std::roundf / std::round (half away from zero) on float32 input."""
    v64 = np.asarray(v, dtype=np.float32).astype(np.float64)
    return np.sign(v64) * np.floor(np.abs(v64) + 0.5)


def blackman16() -> np.ndarray:
    """numpy.blackman(16) in float32, the RCMC tap window (sar/range_doppler_algorithm.cu:46-52)."""
    n = np.arange(16, dtype=np.float64)
    w = 0.42 - 0.5 * np.cos(2 * np.pi * n / 15) + 0.08 * np.cos(4 * np.pi * n / 15)
    return w.astype(np.float32)


# --------------------------------------------------------------------------- stage 1: decode

def decode_ers(raw: np.ndarray, samples_per_line: int, swst: np.ndarray | None, range_size: int) -> np.ndarray:
    """ConvertErsImSamplesToComplexKernel (envisat_format/src/envisat_format_kernels.cu:116-134)
    after the NaN pre-fill (main_flow.cc:537-540).  Even byte = I, odd byte = Q; line y starts
    at 4*(swst[y]-min(swst)).  Bit-exact: float(uint8)."""
    na = raw.shape[0]
    out = np.full((na, range_size), np.complex64(complex(np.nan, np.nan)), dtype=np.complex64)
    if swst is None:
        swst = np.zeros(na, dtype=np.int64)
    swst = np.asarray(swst, dtype=np.int64)
    mn = swst.min()
    iv = raw[:, 0:2 * samples_per_line:2].astype(np.float32)
    qv = raw[:, 1:2 * samples_per_line:2].astype(np.float32)
    for y in range(na):
        off = 4 * int(swst[y] - mn)
        seg = out[y, off:off + samples_per_line]
        n = seg.shape[0]
        out.real[y, off:off + n] = iv[y, :n]
        out.imag[y, off:off + n] = qv[y, :n]
    return out


def fbaq4_index(block, code):
    """Fbaq4IndexCalc (envisat_format/include/envisat_parse_util.cuh:75-84): table index
    256 * level + block id, level = 15 - code for codes above 7, else 8 + code."""
    code = np.asarray(code, dtype=np.int64)
    return 256 * np.where(code > 7, 15 - code, 8 + code) + np.asarray(block, dtype=np.int64)


def decode_asar_fbaq(raw: np.ndarray, swst: np.ndarray | None, range_size: int, i_lut: np.ndarray,
                     q_lut: np.ndarray, chunk: int = 1024) -> np.ndarray:
    """ConvertAsarImBlocksToComplexKernel (envisat_format/src/envisat_format_kernels.cu:160-209)
    after the NaN pre-fill (main_flow.cc:537-540).  Record y (raw[y], its byte stride the record
    size): 2-byte little-endian block-data length L, then per byte j < L of the block data that is
    not a block id (j % 64 != 0) the sample j - (j // 64 + 1), shifted right by swst[y] - min(swst),
    I from the high nibble and Q from the low nibble of the byte through the tables.  The
    reference indexes the output flat (y * range_size + sample) without a range check, so a
    record longer than range_size would continue into the next row; that is kept here (writes
    past the last row are dropped).  Bit-exact: table lookups only."""
    na, rec = raw.shape
    out_re = np.full(na * range_size, np.nan, dtype=np.float32)
    out_im = np.full(na * range_size, np.nan, dtype=np.float32)
    sw = np.zeros(na, dtype=np.int64) if swst is None else np.asarray(swst, dtype=np.int64)
    off = sw - sw.min()
    j = np.arange(rec - 2, dtype=np.int64)
    b = j // 64
    not_id = (j % 64) != 0
    for y0 in range(0, na, chunk):
        y1 = min(na, y0 + chunk)
        r8 = raw[y0:y1].astype(np.int64)
        length = r8[:, 0] | (r8[:, 1] << 8)
        valid = (j[None, :] < length[:, None]) & not_id[None, :]
        bid = r8[:, 2 + 64 * b]
        cw = r8[:, 2 + j]
        ii = fbaq4_index(bid, cw >> 4)
        qi = fbaq4_index(bid, cw & 15)
        valid &= (ii < i_lut.shape[0]) & (qi < q_lut.shape[0])
        flat = (np.arange(y0, y1)[:, None] * range_size + j[None, :] - (b[None, :] + 1) + off[y0:y1, None])
        keep = valid & (flat < na * range_size)
        out_re[flat[keep]] = i_lut[ii[keep]]
        out_im[flat[keep]] = q_lut[qi[keep]]
    out = np.empty(na * range_size, dtype=np.complex64)
    out.real = out_re
    out.imag = out_im
    return out.reshape(na, range_size)


def decode(raw: np.ndarray, scene: dict) -> np.ndarray:
    """The decoder of the scene's record format (main_flow.cc:530-583)."""
    if scene.get("raw_format", "ers") == "fbaq4":
        ti, tq = scene["fbaq_tables"]
        return decode_asar_fbaq(raw, scene.get("swst"), scene["range_size"], ti, tq)
    return decode_ers(raw, scene["samples_per_line"], scene.get("swst"), scene["range_size"])


def pad_image(data: np.ndarray, rg_pad: int, az_pad: int) -> np.ndarray:
    """InitPadded + ZeroMemory + cudaMemcpy2D of the decoded block (main.cc:233-238)."""
    na, nr = data.shape
    img = np.zeros((az_pad, rg_pad), dtype=np.complex64)
    img[:na, :nr] = data
    return img


# --------------------------------------------------------------------------- level-1 records

def condition_slc(img: np.ndarray, cal: float, hdr: int) -> np.ndarray:
    """CalibrateClampToBigEndian (envisat_format/src/envisat_format_kernels.cu:28-61): per row
    `hdr` zero bytes, then per complex pixel int16 I and Q of clamp(value * cal) truncated toward
    zero (NaN converts to 0 on the device), each most significant byte first."""
    y, x = img.shape
    out = np.zeros((y, hdr + 4 * x), dtype=np.uint8)

    def i16(v):
        s = (v.astype(np.float32) * np.float32(cal)).astype(np.float32)
        c = np.where(s > 32767, np.float32(32767), np.where(s < -32768, np.float32(-32768), s))
        return np.where(np.isnan(c), 0, np.trunc(np.nan_to_num(c))).astype(np.int64)

    i, q = i16(img.real), i16(img.imag)
    pay = out[:, hdr:].reshape(y, x, 4)
    pay[:, :, 0] = (i >> 8) & 0xFF
    pay[:, :, 1] = i & 0xFF
    pay[:, :, 2] = (q >> 8) & 0xFF
    pay[:, :, 3] = q & 0xFF
    return out


def condition_detected(img: np.ndarray, cal: float, hdr: int) -> np.ndarray:
    """CalibrateClampToBigEndianDetected (envisat_format/src/envisat_format_kernels.cu:63-93): per
    row `hdr` zero bytes, then per pixel uint16(min(10 * log10f(value * cal), 65535)) truncated
    toward zero (negative, -inf and NaN convert to 0 on the device), least significant byte
    first.  log10 here is numpy's float32 one; CUDA's log10f may differ by an ulp, which moves a
    value only where 10 log10 lands within an ulp of an integer."""
    y, x = img.shape
    out = np.zeros((y, hdr + 2 * x), dtype=np.uint8)
    v = (img.astype(np.float32) * np.float32(cal)).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        db = (np.float32(10) * np.log10(v)).astype(np.float32)
    db = np.where(np.float32(65535) < db, np.float32(65535), db)
    u = np.where(np.isnan(db) | (db <= 0), 0, np.trunc(np.nan_to_num(db, neginf=0.0))).astype(np.int64)
    pay = out[:, hdr:].reshape(y, x, 2)
    pay[:, :, 0] = u & 0xFF
    pay[:, :, 1] = (u >> 8) & 0xFF
    return out


def _mean_dev(x: np.ndarray, y: np.ndarray):
    """DevicePaddedImage::CalcMean / CalcStdDev (cuda_util/device_padded_image.cu:331-414) over
    pairs (x, y), NaN pairs skipped, divided by the number of all pairs, float results."""
    n = F32(x.size)
    ok = ~(np.isnan(x) | np.isnan(y))
    xd, yd = x[ok].astype(np.float64), y[ok].astype(np.float64)
    mx, my = F32(F32(xd.sum()) / n), F32(F32(yd.sum()) / n)
    dx = F32(((xd - np.float64(mx)) ** 2).sum())
    dy = F32(((yd - np.float64(my)) ** 2).sum())
    return mx, my, F32(np.sqrt(F32(dx / n))), F32(np.sqrt(F32(dy / n)))


def product_statistics_ims(slc: np.ndarray, cal: float = 1.0) -> np.ndarray:
    """CalculateStatistics (main_flow.cc:666-670) of the subset SLC, scaled as main.cc:384-390."""
    mx, my, ex, ey = _mean_dev(slc.real.ravel(), slc.imag.ravel())
    return np.array([mx, my, ex, ey], dtype=np.float64) * float(cal)


def product_statistics_imp(detected: np.ndarray, slc: np.ndarray, cal: float = 1.0) -> np.ndarray:
    """CalculateStatisticsImaged (main_flow.cc:672-676) as main.cc:327-342 calls it: the
    ground-range floats are written over the start of the subset SLC's buffer and that buffer is
    viewed as a complex image of the ground-range size, so its 2 N floats (N pixels) are the
    N ground-range values followed by the SLC floats at positions N .. 2N - 1 of the buffer."""
    n = detected.size
    buf = np.concatenate([detected.astype(np.float32).ravel(), slc.astype(np.complex64).view(np.float32).ravel()[n:2 * n]])
    mx, my, ex, ey = _mean_dev(buf[0::2], buf[1::2])
    return np.array([F32((mx + my) / F32(2)), 0.0, F32((ex + ey) / F32(2)), 0.0], dtype=np.float64) * \
        np.array([cal, 1.0, cal, 1.0])


# --------------------------------------------------------------------------- stage 2: IQ correction

@dataclass
class IqResults:
    dc_i: float
    dc_q: float
    iq_gain: float
    phase_error: float
    stddev_i: float
    stddev_q: float
    sin_corr: float
    cos_corr: float


def raw_data_correction(img: np.ndarray, x_size: int, y_size: int, n_total: int,
                        ref_compat: bool = True) -> IqResults:
    """RawDataCorrection (sar/iq_correction.cu:188-274), in place on the padded image.

    The mean (CalcMean, cuda_util/device_padded_image.cu:331-371) runs over x < XSize; the
    DC subtraction and the gain / phase reductions run over x < XStride, so with
    ``ref_compat`` the range padding (zeros -> -dc) enters the gain and phase statistics
    exactly as in the reference.  ``ref_compat=False`` restricts them to the data block."""
    x_stat = img.shape[1] if ref_compat else x_size
    blk = img[:y_size, :x_size]
    re = blk.real.astype(np.float64)
    im = blk.imag.astype(np.float64)
    ok = ~(np.isnan(re) | np.isnan(im))
    total = F32(n_total)
    mean_i = F32(F32(re[ok].sum()) / total)
    mean_q = F32(F32(im[ok].sum()) / total)
    di = (blk.real[ok] - mean_i).astype(np.float32).astype(np.float64)
    dq = (blk.imag[ok] - mean_q).astype(np.float32).astype(np.float64)
    std_i = F32(np.sqrt(F32(F32((di * di).sum()) / total)))
    std_q = F32(np.sqrt(F32(F32((dq * dq).sum()) / total)))

    reg = img[:y_size, :x_stat]
    reg.real[...] = reg.real - mean_i
    reg.imag[...] = reg.imag - mean_q

    re = reg.real.astype(np.float64)
    im = reg.imag.astype(np.float64)
    ok = ~(np.isnan(re) | np.isnan(im))
    i_sq = float((re[ok] ** 2).sum())
    q_sq = float((im[ok] ** 2).sum())
    gain = math.sqrt(i_sq / q_sq)
    reg.real[...] = (reg.real / F32(gain)).astype(np.float32)

    re = reg.real.astype(np.float64)
    ok = ~(np.isnan(re) | np.isnan(im))
    iq = float((re[ok] * im[ok]).sum())
    i_sq2 = float((re[ok] ** 2).sum())
    delta = iq / i_sq2
    sin_c = F32(delta)
    cos_c = F32(1 - delta * delta)
    q_new = fmaf(reg.real, -sin_c, reg.imag) / cos_c
    reg.imag[...] = q_new.astype(np.float32)
    phase_err = 360 * math.asin(delta) / (2 * math.pi)
    return IqResults(float(mean_i), float(mean_q), gain, phase_err, float(std_i), float(std_q),
                     float(sin_c), float(cos_c))


def apply_iq_correction(block: np.ndarray, dc_i: float, dc_q: float, gain_f32: float, sin_c: float,
                        cos_c: float) -> np.ndarray:
    """The three correction kernels of RawDataCorrection on a complex64 block with given
    float constants (sar/iq_correction.cu:140-178): I = (I - dc_i) / g; Q = fma(-I, s, Q - dc_q) / c.
    NaN samples stay NaN."""
    i1 = (block.real - F32(dc_i)).astype(np.float32)
    q1 = (block.imag - F32(dc_q)).astype(np.float32)
    i2 = (i1 / F32(gain_f32)).astype(np.float32)
    q2 = fmaf(-i2, F32(sin_c), q1) / F32(cos_c)
    out = np.empty_like(block)
    out.real = i2
    out.imag = q2.astype(np.float32)
    return out


def zero_nans(img: np.ndarray) -> None:
    """DevicePaddedImage::ZeroNaNs (cuda_util/device_padded_image.cu:69-85, 322-329)."""
    r = img.real
    i = img.imag
    r[np.isnan(r)] = 0
    i[np.isnan(i)] = 0


# --------------------------------------------------------------------------- stage 3: Doppler centroid

def doppler_centroid(img: np.ndarray, x_size: int, y_size: int, prf: float):
    """CalculateDopplerCentroid (sar/fractional_doppler_centroid.cu:98-139): ACCC over
    range blocks of XSize//32 columns; the last block may run into the range padding
    (the kernel bounds only by x_end).  Returns (poly float64[3], block centres, block Hz)."""
    step = x_size // 32
    dcs, idx = [], []
    a = img[:y_size]
    for xb in range(0, x_size, step):
        xe = xb + step
        blk = a[:, xb:xe].astype(np.complex128)
        acc = (np.conj(blk[:-1]) * blk[1:]).sum()
        ang = math.atan2(acc.imag, acc.real)
        dcs.append(prf * ang / (2 * math.pi))
        idx.append((xb + xe) // 2)
    return geo.polyfit(idx, dcs, 2), np.array(idx), np.array(dcs)


# --------------------------------------------------------------------------- stage 4: chirp + RC

def generate_chirp(kr: float, fs: float, n_samples: int, apply_window: bool, padding: int) -> np.ndarray:
    """GenerateChirpData (sar/sar_chirp.cc:70-104).  The windowed power scale uses Parseval
    (sum |C_k|^2 / N == sum |c_n|^2) in FP64 instead of a float FFT round trip."""
    i = np.arange(n_samples, dtype=np.int64)
    t = (i - n_samples // 2) * (1.0 / fs)
    ph = np.pi * kr * t * t
    c = (np.cos(ph).astype(np.float32) + 1j * np.sin(ph).astype(np.float32)).astype(np.complex64)
    if apply_window:
        m = (0.54 - 0.46 * np.cos(2 * np.pi * i / n_samples)).astype(np.float32)
        cr = c.real * m
        ci = c.imag * m
        c = np.empty_like(c)
        c.real = cr
        c.imag = ci
    out = np.zeros(padding, dtype=np.complex64)
    out[:n_samples] = c
    if apply_window:
        scale = float((np.abs(out.astype(np.complex128)) ** 2).sum())
    else:
        scale = float(n_samples)
    d = F32(math.sqrt(scale))
    # complex<float> /= float divides each component (a complex division would round differently)
    res = np.empty_like(out)
    res.real = out.real / d
    res.imag = out.imag / d
    return res


def range_compression(img: np.ndarray, y_size: int, x_size: int, chirp: np.ndarray, chirp_samples: int) -> int:
    """RangeCompression (sar/range_compression.cu:57-111) in place; returns the new XSize."""
    n = img.shape[1]
    if chirp.shape[0] != n:
        raise ValueError("Range padding and chirp size mismatch")
    cf = np.conj(sfft.fft(chirp.astype(np.complex128)))
    rows = sfft.fft(img[:y_size].astype(np.complex128), axis=1, workers=_workers())
    rows *= cf[None, :]
    rows = sfft.ifft(rows, axis=1, workers=_workers()) * n      # cuFFT inverse is unnormalised
    new_x = x_size - chirp_samples
    mult = F32(1.0 / n)
    rows[:, :new_x] *= np.float64(mult)
    rows[:, new_x:] = 0
    img[:y_size] = rows.astype(np.complex64)
    return new_x


# --------------------------------------------------------------------------- stage 5: RDA

@dataclass
class RdaArgs:
    prf: float
    wavelength: float
    az_bw_frac: float
    range_spacing: float
    slant_range: float
    dc_poly: np.ndarray
    vr_poly: np.ndarray
    absolute_phase: bool = False


def _bin_freq(az_pad: int, step32):
    y = np.arange(az_pad)
    yy = np.where(y < az_pad // 2, y, y - az_pad).astype(np.float32)
    return (yy * step32).astype(np.float32)


def rcmc_shift(args: RdaArgs, az_pad: int, x: np.ndarray):
    """Per (frequency row, column) RCMC walk of RangeCellMigrationCorrection
    (sar/range_doppler_algorithm.cu:117-154).  Returns (shift float32[az_pad, nx], walk int)."""
    prf = F32(args.prf)
    step = F32(prf / F32(az_pad))
    xf = x.astype(np.float32)
    dc = polyval_f32(args.dc_poly, xf)[None, :]
    fn = _bin_freq(az_pad, step)[:, None] * np.ones((1, x.size), np.float32)
    half = F32(prf * F32(0.5))
    hi = (half + dc).astype(np.float32)
    lo = (-half + dc).astype(np.float32)
    fn = np.where((dc < 0) & (fn > hi), (fn - prf).astype(np.float32), fn)
    fn = np.where((dc > 0) & (fn < lo), (fn + prf).astype(np.float32), fn).astype(np.float32)
    r0 = args.slant_range + x.astype(np.float64) * args.range_spacing
    vr = polyval_f32(args.vr_poly, xf)[None, :]
    lam = F32(args.wavelength)
    num = (((lam * lam) * fn).astype(np.float32) * fn).astype(np.float32)
    den = ((F32(8.0) * vr).astype(np.float32) * vr).astype(np.float32)
    dr = (num / den).astype(np.float32).astype(np.float64) * r0[None, :]
    shift = (dr / args.range_spacing).astype(np.float32)
    walk = roundf_away(shift).astype(np.int64)
    return shift, walk


def rcmc(src: np.ndarray, nk: int, args: RdaArgs) -> np.ndarray:
    """RangeCellMigrationCorrection (sar/range_doppler_algorithm.cu:107-195): 16-tap
    Blackman-windowed sinc, taps [calc_x-8, calc_x+8), sum-of-weights normalised, zero when
    the window leaves [0, XSize)."""
    az_pad, rg_pad = src.shape
    out = np.zeros_like(src)
    win = blackman16()
    x = np.arange(nk)
    shift, walk = rcmc_shift(args, az_pad, x)

    def rows_block(r0: int, r1: int) -> None:
        # every output row reads its own frequency row only: blocks of rows are independent
        sh, wk = shift[r0:r1], walk[r0:r1]
        calc = x[None, :] + wk
        valid = (calc - 8 >= 0) & (calc + 8 < nk)
        off = ((sh - wk.astype(np.float32)).astype(np.float32) + F32(8)).astype(np.float32)
        acc = np.zeros((r1 - r0, nk), dtype=np.complex128)
        norm = np.zeros((r1 - r0, nk), dtype=np.float64)
        rows = np.arange(r0, r1)[:, None]
        for i in range(16):
            arg = (off - F32(i)).astype(np.float32)
            pa = (PI32 * arg).astype(np.float32)
            with np.errstate(invalid="ignore", divide="ignore"):
                s = (np.sin(pa.astype(np.float64)).astype(np.float32) / pa).astype(np.float32)
            s = np.where(arg == 0, F32(1), s)
            w = (win[i] * s).astype(np.float32)
            w = np.where(valid, w, F32(0))
            col = np.clip(calc - 8 + i, 0, rg_pad - 1)
            acc += src[rows, col].astype(np.complex128) * w
            norm += w
        with np.errstate(invalid="ignore", divide="ignore"):
            res = np.where(norm != 0, acc / np.where(norm != 0, norm, 1), 0)
        out[r0:r1, :nk] = res.astype(np.complex64)

    # numpy releases the GIL in these element-wise passes: row blocks run on a thread pool
    from concurrent.futures import ThreadPoolExecutor
    step = 512
    with ThreadPoolExecutor(max_workers=_workers()) as ex:
        list(ex.map(lambda r0: rows_block(r0, min(az_pad, r0 + step)), range(0, az_pad, step)))
    return out


def azimuth_filter(az_pad: int, nk: int, args: RdaArgs) -> np.ndarray:
    """The azimuth reference of AzimuthReferenceMultiply (sar/range_doppler_algorithm.cu:197-309)
    as a complex128 array [az_pad, nk] (zero in the discarded band)."""
    prf = F32(args.prf)
    step = F32(prf / F32(az_pad))
    x = np.arange(nk)
    xf = x.astype(np.float32)
    dc = polyval_f32(args.dc_poly, xf)[None, :]
    dc_steps = roundf_away((dc / step).astype(np.float32)).astype(np.float32)
    dc_off = (dc_steps * step).astype(np.float32)
    bf = _bin_freq(az_pad, step)[:, None] * np.ones((1, nk), np.float32)
    half = F32(prf * F32(0.5))
    absf = bf.copy()
    absf = np.where((dc < 0) & (bf > (half + dc).astype(np.float32)), (absf - prf).astype(np.float32), absf)
    absf = np.where((dc > 0) & (absf < (-half + dc).astype(np.float32)), (absf + prf).astype(np.float32), absf)
    frac = F32(args.az_bw_frac)
    cut_hi = fmaf(half, frac, dc_off)
    cut_lo = fmaf(-half, frac, dc_off)
    keep = ~((absf < cut_lo) | (absf > cut_hi))
    fc = (bf - dc_off).astype(np.float32)
    fc = np.where(fc > half, (fc - prf).astype(np.float32), np.where(fc < -half, (fc + prf).astype(np.float32), fc))
    r0 = args.slant_range + args.range_spacing * x.astype(np.float64)
    vr = polyval_f32(args.vr_poly, xf)
    ka = (((F32(2) * vr).astype(np.float32) * vr).astype(np.float32).astype(np.float64)
          / (np.float64(F32(args.wavelength)) * r0)).astype(np.float32)[None, :]
    mf_phase = (((PI32 * fc).astype(np.float32) * fc).astype(np.float32) / ka).astype(np.float32)
    sh_phase = (((F32(2) * PI32) * (dc_off / ka).astype(np.float32)).astype(np.float32) * bf).astype(np.float32)
    mf = np.exp(-1j * mf_phase.astype(np.float64)) * np.exp(-1j * sh_phase.astype(np.float64))
    if args.absolute_phase:
        # the range-dependent azimuth reference phase 4 pi R0 / lambda (about 1.9e8 rad at
        # 850 km), reduced modulo 2 pi in FP64: no term of this kind exists in the reference
        # (sar/range_doppler_algorithm.cu:265-290), whose SLC phase keeps -4 pi R0 / lambda
        ph = np.fmod(4.0 * np.pi * r0 / float(args.wavelength), 2.0 * np.pi)
        # and the constant the Doppler-centroid shift leaves, pi dc_off^2 / Ka: with it the
        # filter is exp(-j pi f^2 / Ka) in the unaliased frequency, the zero-Doppler phase kept
        ph = ph + np.fmod(np.pi * dc_off[0].astype(np.float64) ** 2 / ka[0].astype(np.float64), 2.0 * np.pi)
        mf = mf * np.exp(1j * ph)[None, :]
    return np.where(keep, mf, 0)


def range_doppler(img: np.ndarray, nk: int, na: int, args: RdaArgs) -> np.ndarray:
    """RangeDopplerAlgorithm (sar/range_doppler_algorithm.cu:312-407).  Returns the new image
    (same padded shape); valid block [:na, :nk]."""
    az_pad = img.shape[0]
    cols = sfft.fft(img[:, :nk].astype(np.complex128), axis=0, workers=_workers())
    src = img.copy()
    src[:, :nk] = cols.astype(np.complex64)
    out = rcmc(src, nk, args)
    h = azimuth_filter(az_pad, nk, args)
    blk = out[:, :nk].astype(np.complex128) * h
    blk = sfft.ifft(blk, axis=0, workers=_workers()) * az_pad
    blk[:na] *= np.float64(F32(F32(1.0) / F32(az_pad)))
    out[:, :nk] = blk.astype(np.complex64)
    return out


# --------------------------------------------------------------------------- stage 6: detected tail

def azimuth_multilook(slc: np.ndarray, azimuth_spacing: float):
    """AzimuthMultiLook / TimeDomainAzimuthLook (sar/az_multilook.cu:25-98).  Returns
    (float32 [out_az, nx], ratio float32)."""
    in_y, nx = slc.shape
    ratio = F32(12.5 / azimuth_spacing)
    out_y = int(roundf_away(np.float32(F32(in_y) / ratio)))
    inten = (slc.real.astype(np.float64) ** 2 + slc.imag.astype(np.float64) ** 2)
    cs = np.concatenate([np.zeros((1, nx)), np.cumsum(inten, axis=0)], axis=0)
    y = np.arange(out_y)
    in_idx = (y.astype(np.float32) * ratio).astype(np.float32)
    mu = (in_idx - np.trunc(in_idx.astype(np.float64)).astype(np.float32)).astype(np.float32)

    def box(lo_off, hi_off):
        s = np.trunc((in_idx + F32(lo_off)).astype(np.float32).astype(np.float64)).astype(np.int64)
        e = np.trunc((in_idx + F32(hi_off)).astype(np.float32).astype(np.float64)).astype(np.int64)
        s = np.maximum(s, 0)
        e = np.minimum(e, in_y)
        cnt = np.maximum(e - s, 0)
        tot = cs[np.maximum(e, s)] - cs[s]
        with np.errstate(invalid="ignore", divide="ignore"):
            m = np.where(cnt[:, None] > 0, tot / np.maximum(cnt, 1)[:, None], 0)
        return m, cnt

    s0, c0 = box(-2, 2)
    s1, c1 = box(-1, 3)
    val = s0 + (s1 - s0) * mu.astype(np.float64)[:, None]
    val = np.where(((c0 > 0) & (c1 > 0))[:, None], val, 0)
    return val.astype(np.float32), ratio


def srgr(ml: np.ndarray, start: np.ndarray, frac: np.ndarray) -> np.ndarray:
    """SrGrInterpolation (sar/srgr.cu:49-71): linear interpolation at the per-column index."""
    v0 = ml[:, start].astype(np.float64)
    v1 = ml[:, np.minimum(start + 1, ml.shape[1] - 1)].astype(np.float64)
    return (v0 + frac.astype(np.float64)[None, :] * (v1 - v0)).astype(np.float32)


# --------------------------------------------------------------------------- whole chain

@dataclass
class FocusResult:
    iq: IqResults
    dc_poly: np.ndarray
    dc_blocks: np.ndarray
    vr_poly: np.ndarray
    rg_pad: int
    az_pad: int
    nk: int
    window: dict
    slc: np.ndarray              # subset complex image (IMS tail input)
    ml: np.ndarray               # multilooked + RSL float image
    detected: np.ndarray         # ground-range float image (IMP tail output)
    srgr_start: np.ndarray
    srgr_frac: np.ndarray
    grsr_poly: np.ndarray
    extra: dict = field(default_factory=dict)


def _range_doppler_image(raw: np.ndarray, scene: dict, ref_compat: bool = True):
    """main.cc:233-287 for one block: decode .. RangeDopplerAlgorithm.  Returns the padded
    range-Doppler-processed image, nk, the Doppler polynomial and the Vr polynomial."""
    nr = scene["range_size"]
    na = scene["azimuth_size"]
    nc = scene["chirp_samples"]
    rg_pad, az_pad = geo.reference_padding(nr, nc, na)
    img = pad_image(decode(raw, scene), rg_pad, az_pad)
    raw_data_correction(img, nr, na, scene["total_raw_samples"], ref_compat)
    zero_nans(img)
    osv = [geo.Osv(*o) for o in scene["osv"]]
    if scene.get("vr_poly") is not None:
        vr_poly = np.asarray(scene["vr_poly"], dtype=np.float64)
    else:
        vr_poly = geo.estimate_processing_velocity(
            osv, scene["first_line_time_us"], scene["line_time_interval"], scene["center_point"],
            scene["slant_range_first"], scene["range_spacing"], scene["carrier_frequency"],
            scene["vr_poly_init"], scene["prf"], scene["az_bw_frac"], nr, nc, na)
    chirp = generate_chirp(scene["chirp_kr"], scene["range_sampling_rate"], nc, scene["apply_window"], rg_pad)
    dc_poly, _, _ = doppler_centroid(img, nr, na, scene["prf"])
    nk = range_compression(img, na, nr, chirp, nc)
    args = RdaArgs(scene["prf"], scene["wavelength"], scene["az_bw_frac"], scene["range_spacing"],
                   scene["slant_range_first"], dc_poly, vr_poly)
    return range_doppler(img, nk, na, args), nk, dc_poly, vr_poly


def _round_away(v: float) -> int:
    """llround: nearest integer, halves away from zero."""
    return int(math.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)


def strip_layout(na: int, block: int, overlap: int, max_ap: int, lines_before: int = 0, lines_after: int = 0):
    """Block starts and kept block-relative line ranges of a strip of na lines in blocks of
    `block` lines overlapping by `overlap` (seams at the overlap midpoints, one synthetic
    aperture dropped at each strip end).  Returns (starts, keep_lo, keep_hi, first_line)."""
    B = min(block, na)
    nb = 1 if na <= B else 1 + (na - B + (B - overlap) - 1) // (B - overlap)
    starts = [min(k * (B - overlap), na - B) for k in range(nb)]
    sm, em = max(lines_before, max_ap), max(lines_after, max_ap)
    lo, hi = [], []
    for k, s in enumerate(starts):
        lo.append(sm if k == 0 else (starts[k - 1] + B + s) // 2 - s)
        hi.append(B - em if k == nb - 1 else (s + B + starts[k + 1]) // 2 - s)
    return starts, lo, hi, sm


def focus_strip(raw: np.ndarray, scene: dict, block: int, overlap: int, ref_compat: bool = True):
    """Overlapped-block strip focusing: each block focused as its own scene (own statistics,
    Doppler estimate and orbit time), its kept lines assembled into one strip SLC, then one
    multilook + range-spreading-loss + SRGR pass over the strip.  Returns (detected, slc)."""
    na = scene["azimuth_size"]
    nr, nc = scene["range_size"], scene["chirp_samples"]
    ap = geo.calc_aperture_pixels(scene["carrier_frequency"], scene["vr_poly_init"], [], scene["prf"],
                                  scene["az_bw_frac"], scene["slant_range_first"], scene["range_spacing"], nr, nc)
    starts, lo, hi, first = strip_layout(na, block, overlap, max(ap), scene["lines_before"], scene["lines_after"])
    B = min(block, na)
    parts = []
    for s, a, b in zip(starts, lo, hi):
        bs = dict(scene)
        bs["azimuth_size"] = B
        bs["total_raw_samples"] = scene["samples_per_line"] * B
        bs["first_line_time_us"] = scene["first_line_time_us"] + _round_away(s * scene["line_time_interval"] * 1e6)
        if scene.get("swst") is not None:
            bs["swst"] = np.asarray(scene["swst"])[s:s + B]
        out, nk, _, _ = _range_doppler_image(raw[s:s + B], bs, ref_compat)
        parts.append(out[a:b, : nk])
    nk = parts[0].shape[1]
    half = geo.RCMC_WINDOW // 2
    slc = np.concatenate(parts, axis=0)[:, half: nk - half]
    ml, ratio = azimuth_multilook(slc, scene["azimuth_spacing"])
    sub_first = scene["slant_range_first"] + half * scene["range_spacing"]
    ml = (ml * geo.rsl_table(slc.shape[1], sub_first, scene["range_spacing"])[None, :]).astype(np.float32)
    osv = [geo.Osv(*o) for o in scene["osv"]]
    t0 = scene["first_line_time_us"] + _round_away(first * scene["line_time_interval"] * 1e6)
    lti_ml = float(np.float64(1.0 / scene["prf"]) * np.float64(ratio))
    grsr, ng = geo.srgr_polynomial(osv, t0, lti_ml, ml.shape[0], scene["center_point"], sub_first,
                                   scene["range_spacing"], slc.shape[1])
    start, frac = geo.srgr_index_map(grsr, scene["range_spacing"], ng)
    return srgr(ml, start, frac), slc


def focus(raw: np.ndarray, scene: dict, ref_compat: bool = True, keep_intermediate: bool = False,
          absolute_phase: bool = False) -> FocusResult:
    """main.cc:233-327 for a scene described by ``scene`` (see ``asarf.scene.Scene.to_dict``):
    ERS byte-I/Q or ASAR FBAQ4 records.  ``absolute_phase`` adds the azimuth reference phase
    4 pi R0 / lambda per range column (not in the reference)."""
    nr = scene["range_size"]
    na = scene["azimuth_size"]
    nc = scene["chirp_samples"]
    rg_pad, az_pad = geo.reference_padding(nr, nc, na)
    data = decode(raw, scene)
    img = pad_image(data, rg_pad, az_pad)
    del data
    iq = raw_data_correction(img, nr, na, scene["total_raw_samples"], ref_compat)
    zero_nans(img)
    extra = {}
    if keep_intermediate:
        extra["corrected"] = img[:na, :nr].copy()
    osv = [geo.Osv(*o) for o in scene["osv"]]
    aperture = geo.calc_aperture_pixels(scene["carrier_frequency"], scene["vr_poly_init"], [], scene["prf"],
                                        scene["az_bw_frac"], scene["slant_range_first"], scene["range_spacing"],
                                        nr, nc)
    if scene.get("vr_poly") is not None:
        vr_poly = np.asarray(scene["vr_poly"], dtype=np.float64)
    else:
        vr_poly = geo.estimate_processing_velocity(
            osv, scene["first_line_time_us"], scene["line_time_interval"], scene["center_point"],
            scene["slant_range_first"], scene["range_spacing"], scene["carrier_frequency"],
            scene["vr_poly_init"], scene["prf"], scene["az_bw_frac"], nr, nc, na)
    chirp = generate_chirp(scene["chirp_kr"], scene["range_sampling_rate"], nc, scene["apply_window"], rg_pad)
    dc_poly, dc_idx, dc_hz = doppler_centroid(img, nr, na, scene["prf"])
    nk = range_compression(img, na, nr, chirp, nc)
    if keep_intermediate:
        extra["rc"] = img[:na, :nk].copy()
    args = RdaArgs(scene["prf"], scene["wavelength"], scene["az_bw_frac"], scene["range_spacing"],
                   scene["slant_range_first"], dc_poly, vr_poly, absolute_phase)
    out = range_doppler(img, nk, na, args)
    del img
    win = geo.results_window(dc_poly[-1], scene["lines_before"], scene["lines_after"], max(aperture))
    first = win["first_line"]
    last = na - win["drop_end"]
    slc = out[first:last, win["near"]:nk - win["far"]].copy()
    del out
    ml, ratio = azimuth_multilook(slc, scene["azimuth_spacing"])
    sub_first = scene["slant_range_first"] + win["near"] * scene["range_spacing"]
    rsl = geo.rsl_table(slc.shape[1], sub_first, scene["range_spacing"])
    ml = (ml * rsl[None, :]).astype(np.float32)
    lti_ml = float(np.float64(1.0 / scene["prf"]) * np.float64(ratio))
    grsr, ng = geo.srgr_polynomial(osv, scene["first_line_time_us"], lti_ml, ml.shape[0], scene["center_point"],
                                   sub_first, scene["range_spacing"], slc.shape[1])
    start, frac = geo.srgr_index_map(grsr, scene["range_spacing"], ng)
    det = srgr(ml, start, frac)
    return FocusResult(iq, dc_poly, dc_hz, vr_poly, rg_pad, az_pad, nk, win, slc, ml, det, start, frac, grsr,
                       dict(extra, aperture=aperture, dc_idx=dc_idx, ratio=ratio))
