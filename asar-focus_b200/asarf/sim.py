"""Seeded synthetic raw-data generator (test inputs; no public dataset exists for this path).

A scene is circular complex Gaussian clutter plus a grid of point targets plus thermal
noise, then the I/Q front-end impairments (DC bias, gain imbalance, quadrature skew) and
quantisation to 5- or 8-bit offset-binary bytes, interleaved I,Q per sample as the ERS
byte decoder expects, or adaptive 4-bit block quantisation into ENVISAT ASAR FBAQ4 records
(``asarf.fbaq``).

* point targets: exact hyperbolic range history R(eta) = sqrt(R0^2 + Vr^2 (eta-eta0)^2)
  (so range migration is present), transmitted chirp exp(j pi Kr t^2), carrier phase
  exp(-j 4 pi R / lambda), azimuth beam cos^2 centred on the Doppler centroid;
* clutter: white reflectivity shaped in range by the chirp spectrum and in azimuth by the
  same beam and the stationary-phase azimuth chirp, so its azimuth spectrum sits on the
  Doppler centroid (which the ACCC estimator then measures).

Runs on any torch device (the CUDA path only for speed on big scenes).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import fbaq
from .scene import SOL, Scene


def _poly(p, x):
    v = 0.0
    for c in p:
        v = v * x + c
    return v


def target_grid(sc: Scene) -> list[tuple[float, float]]:
    """(range pixel, zero-Doppler azimuth line) of every point target."""
    nk = sc.range_size - sc.chirp_samples
    gx, gy = sc.grid
    xs = np.linspace(0.15 * nk, 0.85 * nk, gx)
    ys = np.linspace(0.3 * sc.azimuth_size, 0.7 * sc.azimuth_size, gy)
    return [(float(round(x)) + 0.0, float(round(y)) + 0.0) for y in ys for x in xs]


def _orbit_state(sc: Scene, time_us: int):
    """Position and velocity of the scene's circular orbit at an absolute time (analytic,
    the curve the state vectors of Scene.build_orbit sample)."""
    from .scene import GM, R_EARTH
    rs = R_EARTH + sc.altitude
    w = math.sqrt(GM / rs ** 3)
    inc = math.radians(98.5)
    e1 = np.array([1.0, 0.0, 0.0])
    e2 = np.array([0.0, math.cos(inc), math.sin(inc)])
    t_scene = sc.azimuth_size / sc.prf
    t = (time_us - sc.first_line_time_us) * 1e-6
    th = math.radians(30.0) + w * (t - t_scene / 2)
    return rs * (math.cos(th) * e1 + math.sin(th) * e2), rs * w * (-math.sin(th) * e1 + math.cos(th) * e2)


def truth_vr_poly(sc: Scene) -> tuple:
    """Effective velocity of the simulated world, quadratic in range pixel (highest power first).

    It is the hyperbolic range-history coefficient of a point on the WGS84 ellipsoid seen from
    the analytic orbit, fitted over 9 positions across the synthetic aperture at 10 range
    positions, so that a processor that estimates Vr from the state vectors recovers it.  It
    depends only on the scene description, not on any processor's estimate, so every
    process simulating a scene produces the same raw bytes.
    """
    if sc.vr_given is not None:
        return (0.0, 0.0, float(sc.vr_given))
    if not sc.osv:
        sc.build_orbit()
    a_e, b_e = 6378137.0, 6356752.314245
    lti = 1.0 / sc.prf
    mid = sc.azimuth_size // 2
    tc = sc.first_line_time_us + (int(lti * mid * 1e6) & 0xFFFFFFFF)
    pc, vc = _orbit_state(sc, tc)
    up = pc / np.linalg.norm(pc)
    right = np.cross(vc / np.linalg.norm(vc), up)
    nk = sc.range_size - sc.chirp_samples
    step = nk // 10
    vr_init = math.sqrt(0.88) * float(np.linalg.norm(vc))
    xs, vs = [], []
    for x in range(0, nk, step):
        r0 = sc.slant_range_first + x * sc.range_spacing
        ground = math.sqrt(max(r0 ** 2 - sc.altitude ** 2, 1.0))
        t = up + (ground / a_e) * right
        t = t / np.linalg.norm(t) * a_e
        for _ in range(60):  # zero Doppler, slant range r0, on the ellipsoid
            d = t - pc
            f = np.array([vc @ d, d @ d - r0 * r0, (t[0] / a_e) ** 2 + (t[1] / a_e) ** 2 + (t[2] / b_e) ** 2 - 1])
            jac = np.array([vc, 2 * d, [2 * t[0] / a_e ** 2, 2 * t[1] / a_e ** 2, 2 * t[2] / b_e ** 2]])
            dt = np.linalg.solve(jac, -f)
            t = t + dt
            if np.linalg.norm(dt) < 1e-6:
                break
        ka = 2 * vr_init * vr_init / (sc.wavelength * r0)
        ap = int(math.floor((sc.prf * sc.az_bw_frac / 2) / ka * sc.prf + 0.5))
        hs = int(ap / 8)
        ts, ys = [], []
        for i in range(9):
            idx = mid + (i - 4) * hs
            ti = sc.first_line_time_us + (int(lti * idx * 1e6) & 0xFFFFFFFF)
            p, _ = _orbit_state(sc, ti)
            dd = p - t
            ys.append(dd @ dd - r0 * r0)
            ts.append((tc - ti) * 1e-6)
        ts = np.asarray(ts)
        coef = np.linalg.lstsq(np.stack([np.ones(9), ts * ts], axis=1), np.asarray(ys), rcond=None)[0]
        xs.append(x)
        vs.append(math.sqrt(coef[1]))
    return tuple(float(c) for c in np.polyfit(np.asarray(xs, float), np.asarray(vs), 2))


def simulate(sc: Scene, device: str | torch.device = "cpu", noise_rel: float = 0.25,
             return_field: bool = False):
    """Return (raw uint8 numpy [Na, 2*spl], truth dict)."""
    dev = torch.device(device)
    na, nr = sc.azimuth_size, sc.range_size
    nc = sc.chirp_samples
    fs = sc.range_sampling_rate
    kr = sc.chirp_kr
    prf = sc.prf
    lam = sc.wavelength
    dr = sc.range_spacing
    vr_poly = truth_vr_poly(sc)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(sc.seed))
    cdt = torch.complex64
    rdt = torch.float32

    # ---------------------------------------------------------------- clutter
    clut = torch.complex(torch.randn(na, nr, generator=gen, device=dev, dtype=rdt),
                         torch.randn(na, nr, generator=gen, device=dev, dtype=rdt)) * (1 / math.sqrt(2))
    n = torch.arange(nc, device=dev, dtype=torch.float64)
    t = (n - nc // 2) / fs
    chirp = torch.polar(torch.ones_like(t), math.pi * kr * t * t).to(cdt)
    hr = torch.fft.fft(torch.nn.functional.pad(chirp, (0, nr - nc)))
    clut = torch.fft.ifft(torch.fft.fft(clut, dim=1) * hr[None, :], dim=1)
    # azimuth: per range column spectrum A(f - fdc) exp(j pi f^2 / Ka) * PRF / sqrt(Ka)
    x = torch.arange(nr, device=dev, dtype=torch.float64)
    r0 = sc.slant_range_first + x * dr
    vr = _poly(vr_poly, x)
    ka = 2 * vr * vr / (lam * r0)
    fdc = torch.as_tensor(sc.dc_truth(np.arange(nr), na / 2), device=dev, dtype=torch.float64)
    beam_bw = 0.95 * prf
    spec = torch.fft.fft(clut, dim=0)
    fb = torch.fft.fftfreq(na, d=1.0 / prf, device=dev).to(torch.float64)
    chunk = max(1, (1 << 24) // na)
    for c0 in range(0, nr, chunk):
        c1 = min(nr, c0 + chunk)
        f = fb[:, None] + torch.zeros(1, c1 - c0, device=dev, dtype=torch.float64)
        d = fdc[None, c0:c1]
        fa = f + prf * torch.round((d - f) / prf)          # unaliased Doppler within fdc +- prf/2
        off = fa - d
        beam = torch.where(off.abs() < beam_bw / 2, torch.cos(math.pi * off / beam_bw) ** 2,
                           torch.zeros_like(off))
        ph = torch.remainder(math.pi * fa * fa / ka[None, c0:c1], 2 * math.pi)
        h = torch.polar(beam * (prf / torch.sqrt(ka[None, c0:c1])), ph)
        spec[:, c0:c1] *= h.to(cdt)
    clut = torch.fft.ifft(spec, dim=0)
    del spec
    if sc.dc_kind == "sin" and sc.dc_drift:
        # azimuth drift of the clutter's Doppler centroid: line y is shifted in frequency by
        # dc_truth(y) - dc_truth(mid-scene) through the integrated phase of that shift
        yy = np.arange(na, dtype=np.float64)
        shift = sc.dc_drift * np.sin(2 * np.pi * yy / na) - sc.dc_drift * np.sin(np.pi)
        phase = 2 * np.pi * np.cumsum(shift) / prf
        clut = clut * torch.polar(torch.ones(na, device=dev, dtype=torch.float64),
                                  torch.as_tensor(np.remainder(phase, 2 * np.pi), device=dev))[:, None].to(cdt)
    clut_std = float(torch.sqrt(torch.mean(clut.real ** 2 + clut.imag ** 2) / 2))

    # ---------------------------------------------------------------- point targets
    field = clut
    amp = 10 ** (sc.target_db / 20)
    targets = target_grid(sc)
    for (xt, yt) in targets:
        r0t = sc.slant_range_first + xt * dr
        vrt = _poly(vr_poly, xt)
        kat = 2 * vrt * vrt / (lam * r0t)
        fd = float(sc.dc_truth(np.array([xt]), yt)[0])
        eta0 = yt / prf
        etac = eta0 - fd / kat
        half = beam_bw / (2 * kat)
        y_lo = max(0, int(math.ceil((etac - half) * prf)))
        y_hi = min(na - 1, int(math.floor((etac + half) * prf)))
        if y_hi < y_lo:
            continue
        ys = torch.arange(y_lo, y_hi + 1, device=dev, dtype=torch.float64)
        eta = ys / prf
        rr = torch.sqrt(r0t * r0t + vrt * vrt * (eta - eta0) ** 2)
        finst = -2 * vrt * vrt * (eta - eta0) / (lam * rr)
        off = finst - fd
        beam = torch.where(off.abs() < beam_bw / 2, torch.cos(math.pi * off / beam_bw) ** 2,
                           torch.zeros_like(off))
        p = (rr - sc.slant_range_first) / dr
        i0 = torch.ceil(p)
        k = torch.arange(nc, device=dev, dtype=torch.float64)
        ii = i0[:, None] + k[None, :]
        u = ii - p[:, None]
        tt = (u - nc // 2) / fs
        carrier = torch.remainder(-4 * math.pi * rr / lam, 2 * math.pi)
        phase = torch.remainder(carrier[:, None] + math.pi * kr * tt * tt, 2 * math.pi)
        val = torch.polar((amp * beam)[:, None].expand_as(phase), phase)
        ok = (ii >= 0) & (ii < nr)
        yy = ys[:, None].expand_as(ii).long()
        field.index_put_((yy[ok], ii[ok].long()), val[ok].to(cdt), accumulate=True)

    # ---------------------------------------------------------------- front end
    bits = sc.bits
    full = float(2 ** bits)
    fbaq4 = sc.raw_format == "fbaq4"
    sigma_raw = 8.0 if fbaq4 else (4.0 if bits == 5 else 30.0)
    scale = sigma_raw / max(clut_std, 1e-30)
    z = field * scale
    z = z + torch.complex(torch.randn(na, nr, generator=gen, device=dev, dtype=rdt),
                          torch.randn(na, nr, generator=gen, device=dev, dtype=rdt)) * (noise_rel * sigma_raw)
    skew = math.radians(sc.iq_skew_deg)
    iv = z.real * sc.iq_gain
    qv = z.imag * math.cos(skew) + z.real * math.sin(skew)
    truth = dict(targets=target_grid(sc), clutter_scale=scale, amp=amp)
    if return_field:
        truth["field"] = field
    if fbaq4:
        # adaptive 4-bit block quantisation of the (biased, imbalanced) I/Q; record y holds the
        # samples from its SWST offset on
        ivn = (iv + sc.iq_bias[0]).cpu().numpy()
        qvn = (qv + sc.iq_bias[1]).cpu().numpy()
        spl = sc.samples_per_line
        if sc.swst_codes is not None:
            sw = np.asarray(sc.swst_codes, dtype=np.int64)
            offs = sc.swst_step * (sw - sw.min())
            ivn = np.stack([ivn[y, offs[y]:offs[y] + spl] for y in range(na)])
            qvn = np.stack([qvn[y, offs[y]:offs[y] + spl] for y in range(na)])
        else:
            ivn, qvn = ivn[:, :spl], qvn[:, :spl]
        raw = fbaq.encode(ivn, qvn, sc.record_counts, sc.raw_line_bytes, sc.fbaq_q_gain)
        return raw, truth
    bias = full / 2 - 0.5
    iq = torch.stack([iv + bias + sc.iq_bias[0], qv + bias + sc.iq_bias[1]], dim=-1)
    iq = torch.clamp(torch.round(iq), 0, full - 1).to(torch.uint8)
    if sc.swst_codes is not None:
        sw = np.asarray(sc.swst_codes, dtype=np.int64)
        offs = 4 * (sw - sw.min())
        spl = sc.samples_per_line
        out = torch.empty(na, spl, 2, dtype=torch.uint8, device=dev)
        for y in range(na):
            out[y] = iq[y, offs[y]:offs[y] + spl]
        iq = out
    raw = iq.reshape(na, -1).contiguous().cpu().numpy()
    return raw, truth
