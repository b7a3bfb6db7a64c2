"""Scene descriptions: the metadata the focusing path reads (SARMetadata subset) plus the
truth parameters of the synthetic raw-data generator.

The five workloads are ERS / ENVISAT-like stripmap scenes:

* ``ers_small``  — 2048 x 4096 5-bit, 3x3 point grid, constant Doppler 300 Hz, Vr 7100 m/s given.
* ``ers_full``   — 5616 x 28000 5-bit, 20x20 grid, Doppler linear 250..350 Hz, Vr from 5 orbit vectors.
* ``asar_im``    — 5616 x 30000 8-bit, ASAR-like chirp / PRF / wavelength, Doppler quadratic -200..150 Hz.
* ``batch16``    — 16 segments of ERS / ASAR parameters, range 2048 | 5616, azimuth U[4000, 30000].
* ``asar_strip`` — 5616 x 120000 8-bit strip, sinusoidal Doppler drift +-100 Hz.

The orbit is a circular 800 km orbit in an Earth-fixed frame (no Earth rotation); the
scene centre is geolocated with the library's own zero-Doppler solver, and the processing
velocity is either given or estimated from the orbit, exactly as the focusing path uses it.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace

import numpy as np

from . import _lib, fbaq

SOL = 299792458.0
GM = 3.986004418e14
R_EARTH = 6378137.0


@dataclass
class Scene:
    name: str
    range_size: int
    azimuth_size: int
    bits: int
    # chirp
    range_sampling_rate: float
    pulse_duration: float
    chirp_bandwidth: float
    apply_window: bool = True
    # radar / geometry
    prf: float = 1680.0
    wavelength: float = 0.05656
    slant_range_first: float = 830000.0
    azimuth_spacing: float = 2.5
    az_bw_frac: float = 0.8
    altitude: float = 800000.0
    vr_given: float | None = None          # constant processing velocity; None = estimate from orbit
    lines_before: int = 0
    lines_after: int = 0
    # simulation truth
    dc_coeffs: tuple = (300.0,)            # Doppler centroid vs normalised range u in [0,1]: sum c_k u^k
    dc_kind: str = "poly"                  # "poly" or "sin" (azimuth drift, strip)
    dc_drift: float = 0.0
    grid: tuple = (3, 3)
    target_db: float = 30.0
    seed: int = 1000
    iq_bias: tuple = (0.3, 0.3)
    iq_gain: float = 1.02
    iq_skew_deg: float = 2.0
    swst_codes: np.ndarray | None = None
    # raw record format: "ers" (byte I/Q) or "fbaq4" (ENVISAT ASAR FBAQ4 blocks, synthetic tables)
    raw_format: str = "ers"
    fbaq_q_gain: float = 1.0               # Q table scale relative to I
    record_samples: np.ndarray | None = None  # fbaq4: samples held by each record (default: all)
    # filled by prepare()
    osv: list = field(default_factory=list)
    center_point: tuple = (0.0, 0.0, 0.0)
    vr_poly: tuple | None = None
    vr_poly_init: tuple = (0.0, 0.0, 7000.0)
    first_line_time_us: int = 0

    # ------------------------------------------------------------------ derived
    @property
    def chirp_samples(self) -> int:
        return int(round(self.pulse_duration / (1.0 / self.range_sampling_rate)))

    @property
    def chirp_kr(self) -> float:
        return self.chirp_bandwidth / self.pulse_duration

    @property
    def range_spacing(self) -> float:
        return SOL / (2 * self.range_sampling_rate)

    @property
    def carrier_frequency(self) -> float:
        return SOL / self.wavelength

    @property
    def swst_step(self) -> int:
        """Range samples per SWST code step: 4 for ERS records, 1 for ASAR."""
        return 1 if self.raw_format == "fbaq4" else 4

    @property
    def samples_per_line(self) -> int:
        if self.swst_codes is None:
            return self.range_size
        return self.range_size - self.swst_step * int(self.swst_codes.max() - self.swst_codes.min())

    @property
    def raw_line_bytes(self) -> int:
        if self.raw_format == "fbaq4":
            return 2 + fbaq.block_bytes(self.samples_per_line)
        return 2 * self.samples_per_line

    @property
    def record_counts(self) -> np.ndarray:
        """Samples held by each raw record."""
        if self.record_samples is not None:
            return np.asarray(self.record_samples, dtype=np.int64)
        return np.full(self.azimuth_size, self.samples_per_line, dtype=np.int64)

    @property
    def total_raw_samples(self) -> int:
        return int(self.record_counts.sum())

    @property
    def fbaq_tables(self) -> tuple[np.ndarray, np.ndarray] | None:
        if self.raw_format != "fbaq4":
            return None
        if getattr(self, "_tables", None) is None:
            self._tables = fbaq.synthetic_tables(self.fbaq_q_gain)
        return self._tables

    @property
    def line_time_interval(self) -> float:
        return 1.0 / self.prf

    def dc_truth(self, x: np.ndarray, y: np.ndarray | float = 0.0) -> np.ndarray:
        """True Doppler centroid (Hz) at range pixel x (and azimuth line y for the strip)."""
        u = np.asarray(x, dtype=np.float64) / max(1, self.range_size - 1)
        v = np.zeros_like(u)
        for k, c in enumerate(self.dc_coeffs):
            v = v + c * u ** k
        if self.dc_kind == "sin":
            v = v + self.dc_drift * np.sin(2 * np.pi * np.asarray(y, dtype=np.float64) / self.azimuth_size)
        return v

    # ------------------------------------------------------------------ geometry setup
    def build_orbit(self) -> "Scene":
        """State vectors of the circular 800 km orbit, centred on the scene (pure Python)."""
        rs = R_EARTH + self.altitude
        w = math.sqrt(GM / rs ** 3)
        inc = math.radians(98.5)
        e1 = np.array([1.0, 0.0, 0.0])
        e2 = np.array([0.0, math.cos(inc), math.sin(inc)])
        t_scene = self.azimuth_size / self.prf
        theta_c = math.radians(30.0)
        # 5 state vectors 10 s apart centred on the scene (more for long strips)
        n_osv = max(5, int(math.ceil(t_scene / 10.0)) + 3)
        t0_us = 1_000_000_000
        self.first_line_time_us = t0_us
        osv = []
        for k in range(n_osv):
            t = -10.0 * ((n_osv - 1) // 2) + 10.0 * k + t_scene / 2
            th = theta_c + w * (t - t_scene / 2)
            pos = rs * (math.cos(th) * e1 + math.sin(th) * e2)
            vel = rs * w * (-math.sin(th) * e1 + math.cos(th) * e2)
            osv.append((t0_us + int(round(t * 1e6)), tuple(pos), tuple(vel)))
        self.osv = osv
        return self

    def prepare(self, lib=None, geometry=None) -> "Scene":
        """Build the orbit, geolocate the scene centre, fix the processing velocity.

        ``geometry`` supplies the three FP64 steps (``interpolate_orbit(osv, time_us) ->
        (pos, vel)``, ``geolocate(vel, pos, guess, slant_range) -> xyz``,
        ``estimate_vr(scene) -> vr_poly``); by default they are the library's
        asarf_interpolate_orbit, asarf_geolocate and asarf_estimate_processing_velocity.
        """
        if geometry is None:
            geometry = LibraryGeometry(lib or _lib.load_library())
        self.build_orbit()
        osv = self.osv
        # scene centre: right of the ground track at the mid slant range
        tc = self.first_line_time_us + int(self.line_time_interval * (self.azimuth_size // 2) * 1e6)
        pos, vel = geometry.interpolate_orbit(osv, tc)
        pos = np.asarray(pos, dtype=np.float64)
        vel = np.asarray(vel, dtype=np.float64)
        up = pos / np.linalg.norm(pos)
        right = np.cross(vel / np.linalg.norm(vel), up)
        nk = self.range_size - self.chirp_samples
        r_mid = self.slant_range_first + (nk // 2) * self.range_spacing
        ground = math.sqrt(max(r_mid ** 2 - self.altitude ** 2, 1.0))
        guess = (up + (ground / R_EARTH) * right)
        guess = guess / np.linalg.norm(guess) * R_EARTH
        self.center_point = tuple(float(v) for v in geometry.geolocate(vel, pos, guess, r_mid))
        vp = float(np.linalg.norm(osv[len(osv) // 2][2]))
        self.vr_poly_init = (0.0, 0.0, math.sqrt(0.88 * vp * vp))
        if self.vr_given is not None:
            self.vr_poly = (0.0, 0.0, float(self.vr_given))
        else:
            self.vr_poly = tuple(float(v) for v in geometry.estimate_vr(self))
        return self

    # ------------------------------------------------------------------ exports
    def to_c(self, estimate: bool = False):
        """(SceneC, keep-alive osv array)."""
        arr = (_lib.Osv * len(self.osv))(*[_lib.Osv(t, (C.c_double * 3)(*p), (C.c_double * 3)(*v))
                                           for t, p, v in self.osv])
        s = _lib.SceneC()
        s.range_size = self.range_size
        s.azimuth_size = self.azimuth_size
        s.samples_per_line = self.samples_per_line
        s.raw_line_bytes = self.raw_line_bytes
        s.total_raw_samples = self.total_raw_samples
        s.range_sampling_rate = self.range_sampling_rate
        s.chirp_kr = self.chirp_kr
        s.pulse_duration = self.pulse_duration
        s.chirp_samples = self.chirp_samples
        s.apply_window = int(self.apply_window)
        s.prf = self.prf
        s.wavelength = self.wavelength
        s.carrier_frequency = self.carrier_frequency
        s.range_spacing = self.range_spacing
        s.slant_range_first = self.slant_range_first
        s.azimuth_spacing = self.azimuth_spacing
        s.az_bw_frac = self.az_bw_frac
        if self.vr_poly is not None and not estimate:
            s.vr_poly = (C.c_double * 3)(*self.vr_poly)
            s.vr_poly_given = 1
        else:
            s.vr_poly_given = 0
        s.vr_poly_init = (C.c_double * 3)(*self.vr_poly_init)
        s.n_osv = len(self.osv)
        s.osv = C.cast(arr, C.POINTER(_lib.Osv))
        s.first_line_time_us = self.first_line_time_us
        s.line_time_interval = self.line_time_interval
        s.center_point = (C.c_double * 3)(*self.center_point)
        s.lines_before = self.lines_before
        s.lines_after = self.lines_after
        if self.raw_format == "fbaq4":
            ti, tq = self.fbaq_tables
            s.raw_format = _lib.RAW_ASAR_FBAQ4
            s.fbaq_i_lut = ti.ctypes.data_as(C.POINTER(C.c_float))
            s.fbaq_q_lut = tq.ctypes.data_as(C.POINTER(C.c_float))
        return s, arr

    def to_dict(self) -> dict:
        """Scene as the oracle reads it."""
        return dict(
            range_size=self.range_size, azimuth_size=self.azimuth_size, samples_per_line=self.samples_per_line,
            total_raw_samples=self.total_raw_samples, chirp_samples=self.chirp_samples,
            chirp_kr=self.chirp_kr, range_sampling_rate=self.range_sampling_rate, apply_window=self.apply_window,
            prf=self.prf, wavelength=self.wavelength, carrier_frequency=self.carrier_frequency,
            range_spacing=self.range_spacing, slant_range_first=self.slant_range_first,
            azimuth_spacing=self.azimuth_spacing, az_bw_frac=self.az_bw_frac,
            vr_poly=None if self.vr_poly is None else list(self.vr_poly), vr_poly_init=list(self.vr_poly_init),
            osv=[(t, p, v) for t, p, v in self.osv], first_line_time_us=self.first_line_time_us,
            line_time_interval=self.line_time_interval, center_point=tuple(self.center_point),
            lines_before=self.lines_before, lines_after=self.lines_after,
            swst=None if self.swst_codes is None else np.asarray(self.swst_codes),
            raw_format=self.raw_format, raw_line_bytes=self.raw_line_bytes,
            fbaq_tables=self.fbaq_tables,
        )


class LibraryGeometry:
    """The FP64 geometry steps of Scene.prepare through the library's C ABI."""

    def __init__(self, lib):
        self.lib = lib

    def interpolate_orbit(self, osv, time_us):
        arr = (_lib.Osv * len(osv))(*[_lib.Osv(t, (C.c_double * 3)(*p), (C.c_double * 3)(*v)) for t, p, v in osv])
        o = _lib.Osv()
        _lib.check(self.lib, self.lib.asarf_interpolate_orbit(arr, len(osv), int(time_us), C.byref(o)),
                   "interpolate_orbit")
        return tuple(o.pos[:]), tuple(o.vel[:])

    def geolocate(self, vel, pos, guess, slant_range):
        out = (C.c_double * 3)()
        _lib.check(self.lib, self.lib.asarf_geolocate((C.c_double * 3)(*vel), (C.c_double * 3)(*pos),
                                                      (C.c_double * 3)(*guess), float(slant_range), out), "geolocate")
        return tuple(out[:])

    def estimate_vr(self, scene):
        sc = scene.to_c(estimate=True)
        vr = (C.c_double * 3)()
        _lib.check(self.lib, self.lib.asarf_estimate_processing_velocity(C.byref(sc[0]), vr), "estimate_vr")
        return tuple(vr[:])


# ---------------------------------------------------------------------- the workloads

def ers_small(**kw) -> Scene:
    """2048 x 4096 ERS-like 5-bit scene (constant DC 300 Hz, Vr = 7100 m/s given)."""
    base = dict(name="ers_small", range_size=2048, azimuth_size=4096, bits=5, range_sampling_rate=18.96e6,
                pulse_duration=37.12e-6, chirp_bandwidth=15.55e6, prf=1680.0, wavelength=0.05656,
                slant_range_first=830000.0, vr_given=7100.0, dc_coeffs=(300.0,), grid=(3, 3), seed=1000)
    base.update(kw)
    return Scene(**base)


def ers_full(**kw) -> Scene:
    """5616 x 28000 ERS-like 5-bit scene (DC linear 250..350 Hz, Vr from 5 orbit vectors)."""
    base = dict(name="ers_full", range_size=5616, azimuth_size=28000, bits=5, range_sampling_rate=18.96e6,
                pulse_duration=37.12e-6, chirp_bandwidth=15.55e6, prf=1680.0, wavelength=0.05656,
                slant_range_first=830000.0, vr_given=None, dc_coeffs=(250.0, 100.0), grid=(20, 20), seed=1001)
    base.update(kw)
    return Scene(**base)


def asar_im(**kw) -> Scene:
    """5616 x 30000 ENVISAT ASAR IM-like 8-bit scene (DC quadratic -200..150 Hz)."""
    base = dict(name="asar_im", range_size=5616, azimuth_size=30000, bits=8, range_sampling_rate=19.208e6,
                pulse_duration=27.1e-6, chirp_bandwidth=16.0e6, prf=1652.0, wavelength=0.05624,
                slant_range_first=830000.0, vr_given=None, dc_coeffs=(-200.0, 250.0, 100.0), grid=(20, 20),
                seed=1002)
    base.update(kw)
    return Scene(**base)


def asar_strip(**kw) -> Scene:
    """5616 x 120000 ASAR-like strip with a sinusoidal Doppler drift of +-100 Hz."""
    base = dict(name="asar_strip", range_size=5616, azimuth_size=120000, bits=8, range_sampling_rate=19.208e6,
                pulse_duration=27.1e-6, chirp_bandwidth=16.0e6, prf=1652.0, wavelength=0.05624,
                slant_range_first=830000.0, vr_given=None, dc_coeffs=(0.0,), dc_kind="sin", dc_drift=100.0,
                grid=(20, 60), seed=1004)
    base.update(kw)
    return Scene(**base)


def batch16(seed: int = 1003) -> list[Scene]:
    """16 uneven segments mixing the ERS (5-bit) and ASAR (8-bit) parameter sets."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(16):
        ers = bool(rng.integers(0, 2))
        rg = int(rng.choice([2048, 5616]))
        az = int(rng.integers(4000, 30001))
        mk = ers_full if ers else asar_im
        sc = mk(name=f"seg{k:02d}", range_size=rg, azimuth_size=az, seed=seed * 100 + k,
                grid=(4, 6), dc_coeffs=(float(rng.uniform(-300, 300)), float(rng.uniform(-50, 50))))
        out.append(sc)
    return out


def tiny(**kw) -> Scene:
    """Small ERS-like scene for fast tests: 768 range x 1024 lines, 6 us chirp, 100 km slant
    range from an 80 km orbit so the synthetic aperture is ~130 lines."""
    base = dict(name="tiny", range_size=768, azimuth_size=1024, bits=5, range_sampling_rate=18.96e6,
                pulse_duration=6.0e-6, chirp_bandwidth=15.55e6, prf=1680.0, wavelength=0.05656,
                slant_range_first=100000.0, altitude=80000.0, vr_given=7100.0, dc_coeffs=(300.0,),
                grid=(2, 2), seed=7, az_bw_frac=0.8)
    base.update(kw)
    return Scene(**base)


def asar_fbaq(**kw) -> Scene:
    """5616 x 30000 ENVISAT ASAR IM-like scene in FBAQ4 records (synthetic instrument tables)."""
    base = dict(name="asar_fbaq", raw_format="fbaq4", seed=1005)
    base.update(kw)
    return asar_im(**base)


def tiny_fbaq(**kw) -> Scene:
    """The small test scene in FBAQ4 records."""
    base = dict(name="tiny_fbaq", raw_format="fbaq4", seed=8)
    base.update(kw)
    return tiny(**base)


def ers_mid(**kw) -> Scene:
    """5616 x 8192 cut of the ERS scene: profiling case (complex images 324 MB, above L2)."""
    base = dict(name="ers_mid", azimuth_size=8192, grid=(10, 6))
    base.update(kw)
    return ers_full(**base)


def asar_fbaq_mid(**kw) -> Scene:
    """5616 x 8192 cut of the FBAQ4 scene: profiling case (complex images above L2)."""
    base = dict(name="asar_fbaq_mid", azimuth_size=8192)
    base.update(kw)
    return asar_fbaq(**base)


WORKLOADS = {"ers_small": ers_small, "ers_full": ers_full, "asar_im": asar_im, "asar_strip": asar_strip,
             "tiny": tiny, "ers_mid": ers_mid, "asar_fbaq": asar_fbaq, "tiny_fbaq": tiny_fbaq,
             "asar_fbaq_mid": asar_fbaq_mid}


def with_sizes(sc: Scene, **kw) -> Scene:
    return replace(sc, **kw)
