"""Point-target impulse-response analysis (test utility; the reference has none).

For each expected target position in a complex image: locate the peak, cut a window,
upsample it by 2-D FFT zero padding, then measure along the range and azimuth cuts through
the interpolated peak:

* resolution: -3 dB width in input samples;
* PSLR: highest sidelobe outside the main lobe (first nulls) relative to the peak, dB;
* ISLR: sidelobe energy / main-lobe energy over the 2-D window, dB (main lobe = the
  rectangle spanned by the first nulls of the two cuts);
* phase: argument of the interpolated peak, rad.
"""
from __future__ import annotations

import numpy as np


def _upsample(win: np.ndarray, f: int) -> np.ndarray:
    n0, n1 = win.shape
    spec = np.fft.fftshift(np.fft.fft2(win))
    big = np.zeros((n0 * f, n1 * f), dtype=np.complex128)
    o0 = (n0 * f - n0) // 2
    o1 = (n1 * f - n1) // 2
    big[o0:o0 + n0, o1:o1 + n1] = spec
    return np.fft.ifft2(np.fft.ifftshift(big)) * (f * f)


def _cut_metrics(p: np.ndarray, k: int, f: int):
    """p: power along a cut, peak at k, f: upsampling factor."""
    peak = p[k]
    half = peak / 2
    lo = k
    while lo > 0 and p[lo] > half:
        lo -= 1
    hi = k
    while hi < len(p) - 1 and p[hi] > half:
        hi += 1

    def interp(i0, i1):
        a, b = p[i0], p[i1]
        return i0 + (half - a) / (b - a) if b != a else float(i0)

    width = (interp(hi - 1, hi) - interp(lo, lo + 1)) / f if hi > lo + 1 else 0.0
    # first nulls: local minima walking out from the peak
    nl = k
    while nl > 0 and p[nl - 1] < p[nl]:
        nl -= 1
    nr = k
    while nr < len(p) - 1 and p[nr + 1] < p[nr]:
        nr += 1
    side = np.concatenate([p[:nl], p[nr + 1:]])
    pslr = 10 * np.log10(side.max() / peak) if side.size and side.max() > 0 else -np.inf
    return width, pslr, nl, nr


def analyse(img: np.ndarray, y: float, x: float, search: int = 8, win: int = 32, up: int = 16) -> dict:
    """IRF of the target expected near (line y, column x) of complex image img."""
    ny, nx = img.shape
    yi, xi = int(round(y)), int(round(x))
    y0, y1 = max(0, yi - search), min(ny, yi + search + 1)
    x0, x1 = max(0, xi - search), min(nx, xi + search + 1)
    sub = np.abs(img[y0:y1, x0:x1])
    py, px = np.unravel_index(np.argmax(sub), sub.shape)
    py += y0
    px += x0
    h = win // 2
    if py - h < 0 or px - h < 0 or py + h > ny or px + h > nx:
        return {}
    w = img[py - h:py + h, px - h:px + h].astype(np.complex128)
    u = _upsample(w, up)
    pw = np.abs(u) ** 2
    ky, kx = np.unravel_index(np.argmax(pw), pw.shape)
    az_w, az_pslr, an0, an1 = _cut_metrics(pw[:, kx], ky, up)
    rg_w, rg_pslr, rn0, rn1 = _cut_metrics(pw[ky, :], kx, up)
    main = pw[an0:an1 + 1, rn0:rn1 + 1].sum()
    tot = pw.sum()
    islr = 10 * np.log10((tot - main) / main) if main > 0 and tot > main else -np.inf
    return dict(y=py - h + ky / up, x=px - h + kx / up, peak=float(pw[ky, kx]), phase=float(np.angle(u[ky, kx])),
                res_az=az_w, res_rg=rg_w, pslr_az=az_pslr, pslr_rg=rg_pslr, islr=islr)


def compare(a: dict, b: dict) -> dict:
    """Differences between two IRF measurements of the same target."""
    dphi = np.angle(np.exp(1j * (a["phase"] - b["phase"])))
    return dict(res_az_rel=abs(a["res_az"] / b["res_az"] - 1), res_rg_rel=abs(a["res_rg"] / b["res_rg"] - 1),
                pslr_az_db=abs(a["pslr_az"] - b["pslr_az"]), pslr_rg_db=abs(a["pslr_rg"] - b["pslr_rg"]),
                islr_db=abs(a["islr"] - b["islr"]), phase_rad=abs(float(dphi)))
