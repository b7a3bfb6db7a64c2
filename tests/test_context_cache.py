"""Host logic of the allocation-free statistics entry point, on the CPU.

* Its scratch address is cached per CUDA context id, not per device: a new context (after
  cudaDeviceReset, or a host application's own driver context) must trigger a new lookup
  and must never be handed the address resolved under an earlier context.  Driven through
  a test hook of the host-emulation library with made-up context ids; no GPU involved.
* The Doppler-block count stays inside the static scratch's 80 entries for every range
  size; at range_size 63 (the largest count, 63 one-sample blocks) the entry point's
  per-block estimates match the oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from asarf import _lib
from oracle import rda


def _probe(lib, ids):
    f = lib.asarf_emu_context_cache_probe
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_ulonglong), C.c_int, C.POINTER(C.c_ulonglong)]
    arr = (C.c_ulonglong * len(ids))(*ids)
    out = (C.c_ulonglong * len(ids))()
    n = f(arr, len(ids), out)
    return n, list(out)


def test_scratch_address_is_resolved_again_for_a_new_context(emu_lib):
    # context 11 twice, then a "reset" gives context 12 on the same device, then 11 again
    n, addrs = _probe(emu_lib, [11, 11, 12, 12, 11])
    assert n == 2
    assert addrs[0] == addrs[1] == addrs[4]
    assert addrs[2] == addrs[3]
    assert addrs[2] != addrs[0]  # the new context never sees the old context's address


def test_oldest_context_entry_is_overwritten_when_the_table_is_full(emu_lib):
    # the probe's table has 4 slots: five new contexts push the first one out
    n, addrs = _probe(emu_lib, [101, 102, 103, 104, 105, 101])
    assert n == 6
    assert addrs[5] != addrs[0]


def test_doppler_block_count_never_exceeds_scratch():
    counts = []
    for nr in range(32, 70000):
        step = nr // 32
        counts.append((nr + step - 1) // step)
    assert max(counts) == 63 < 80


def test_range_size_63_blocks_match_oracle(emu_lib):
    rng = np.random.default_rng(63)
    nr, na = 63, 512
    iq = rng.integers(0, 32, size=(na, nr, 2), dtype=np.uint8)
    raw = np.ascontiguousarray(iq.reshape(na, 2 * nr))
    out = _lib.RawStats()
    rc = emu_lib.asarf_raw_statistics_noalloc(raw.ctypes.data, 2 * nr, nr, nr, na, None, 0, nr * na, 0, 1680.0,
                                              C.addressof(out), None)
    _lib.check(emu_lib, rc, "raw_statistics_noalloc")
    assert out.errors == 0
    assert out.n_dc_blocks == 63
    img = rda.decode_ers(raw, nr, None, nr)
    rda.raw_data_correction(img, nr, na, nr * na)
    _, _, hz = rda.doppler_centroid(img, nr, na, 1680.0)
    assert len(hz) == 63
    np.testing.assert_allclose(np.array(out.dc_block_hz[:63]), hz, rtol=0, atol=2e-3)
