"""Generate the golden fixtures of the reference's own focusing code.

Runs on a machine with a CUDA GPU and the reference build (oracle/_ref/libasar_ref.so,
made by `make -C oracle/ref_build`): simulates seeded scenes on the CPU (so any machine can
regenerate the identical raw bytes, checked by SHA-256), runs the reference chain, and
stores its IQ statistics, Doppler polynomial, results window, the first rows of the
IQ-corrected and range-compressed images and of the detected output, plus image-wide
summary numbers.  tests/test_golden.py checks the CPU oracle against these on any machine.

Usage: python tests/golden/make_golden.py [outdir]
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "asar-focus_b200"))


def generate(name: str, factory, out_dir: Path, rows: int) -> Path:
    import asarf
    from asarf import sim
    from oracle import ref_lib

    lib = asarf.load_library()
    sc = factory()
    sc.prepare(lib)
    raw, _ = sim.simulate(sc, device="cpu")
    scc, keep = sc.to_c()
    det, r, d = ref_lib.ref_focus(scc, sc.vr_poly, raw, dumps=True)
    path = out_dir / f"ref_{name}.npz"
    np.savez_compressed(
        path,
        raw_sha256=np.frombuffer(hashlib.sha256(raw.tobytes()).digest(), dtype=np.uint8),
        stats=np.array([r["dc_i"], r["dc_q"], r["iq_gain"], r["phase_error"], r["stddev_i"], r["stddev_q"]]),
        dc_poly=np.array(r["dc_poly"]), grsr_poly=np.array(r["grsr_poly"]),
        window=np.array([r["first_line"], r["n_lines"], r["slc_cols"], r["out_rows"], r["out_cols"],
                         r["max_aperture"]]),
        corrected_head=d["corrected"][:rows], rc_head=d["rc"][:rows], detected_head=det[:rows],
        detected_sum=np.array([det.astype(np.float64).sum(), (det.astype(np.float64) ** 2).sum()]),
        vr_poly=np.array(sc.vr_poly),
    )
    return path


if __name__ == "__main__":
    from asarf import scene as S
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    out.mkdir(parents=True, exist_ok=True)
    print(generate("tiny", S.tiny, out, 16))
    print(generate("ers_small", S.ers_small, out, 4))
