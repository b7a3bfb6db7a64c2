"""C ABI: the product library loads, exports every symbol include/*.h declares, and its
host-only entry points follow the reference rules.  No device work here."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import asarf
from asarf import _lib
from asarf import scene as S

ROOT = Path(__file__).resolve().parent.parent


def _declared() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(asarf_[a-z0-9_]+)\s*\(", txt))
    return names


def test_product_library_exports_every_declared_symbol():
    lib = asarf.load_library()  # raises when the CUDA library is not built
    names = _declared()
    assert "asarf_focus" in names and "asarf_plan_create" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_emulation_library_exports_the_same_abi(emu_lib):
    missing = [n for n in sorted(_declared()) if not hasattr(emu_lib, n)]
    assert not missing


def test_fft_size_rule_matches_reference_padding():
    # upper_bound over 2^a3^b5^c7^d: strictly greater (main.cc:217, 223)
    lib = asarf.load_library()
    cases = {2048 + 704: 2800, 4096: 4116, 5616 + 704: 6400, 28000: 28125, 5616 + 521: 6144, 30000: 30240,
             120000: 120050, 16384: 16464, 4095: 4096, 4116: 4200}
    for v, want in cases.items():
        assert lib.asarf_fft_size_above(v) == want, v
    from oracle import geometry as geo
    for v in list(cases) + [1, 7, 1000, 99999]:
        assert lib.asarf_fft_size_above(v) == geo.fft_upper_bound(v)


def test_invalid_scene_is_rejected_with_message():
    lib = asarf.load_library()
    sc = S.tiny()
    sc.prepare(lib)
    c, keep = sc.to_c()
    c.range_size = -5
    h = C.c_void_p()
    rc = lib.asarf_plan_create(C.byref(c), None, C.byref(h))
    assert rc == -1 and not h.value
    assert b"positive" in lib.asarf_last_error()
    c.range_size = sc.range_size
    c.raw_line_bytes = 3
    assert lib.asarf_plan_create(C.byref(c), None, C.byref(h)) == -1
    assert b"raw_line_bytes" in lib.asarf_last_error()


def test_null_arguments_are_errors_not_crashes():
    lib = asarf.load_library()
    assert lib.asarf_focus(None, None, None, 0, None, None) == -1
    assert lib.asarf_plan_results(None, None, None) == -1
    assert lib.asarf_polyfit(None, None, 3, 2, None) == -1
    lib.asarf_plan_destroy(None)


def test_polyfit_matches_least_squares():
    lib = asarf.load_library()
    rng = np.random.default_rng(3)
    x = np.linspace(0, 5600, 33)
    y = 250 + 0.02 * x - 3e-6 * x * x + rng.normal(0, 1, x.size)
    out = (C.c_double * 3)()
    xa = (C.c_double * x.size)(*x)
    ya = (C.c_double * y.size)(*y)
    assert lib.asarf_polyfit(xa, ya, x.size, 2, out) == 0
    ref = np.polyfit(x, y, 2)
    assert np.allclose(out[:], ref, rtol=1e-9, atol=1e-12)
