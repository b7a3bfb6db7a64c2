"""CPU oracle for the asar-focus range-Doppler focusing path.

TEST INFRASTRUCTURE ONLY.  This package is a plain numpy restatement of the
reference's algorithm (cgi-estonia-space/asar-focus, ``sar/``, ``cuda_util/``,
``main.cc``, ``main_flow.cc``), used as the checker for the CUDA product path.
Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product path
(``asar-focus_b200/asarf``) never imports, links or executes anything here.

Precision policy: FFTs and accumulations run in FP64; every quantity on which
the reference takes a discrete decision (RCMC walk, Doppler-bin quantisation,
band cut, multilook indices, SRGR index) or whose float32 rounding dominates
the result (azimuth matched-filter phase) is recomputed with the reference's
float32 operation sequence.

Parity pinning: the reference ships no golden vectors or known-answer tests for
this path (its unit tests cover only parsing helpers).  The oracle is pinned
against the reference's own CUDA build (``oracle/ref_build``: the reference's
``sar/`` + ``cuda_util/`` sources compiled for sm_100a, run on a B200): the stored
reference outputs in ``tests/golden`` are checked on the CPU by ``tests/test_golden.py``,
and the reference build runs beside the oracle on the GPU in ``tests/test_gpu_parity.py``.
"""
