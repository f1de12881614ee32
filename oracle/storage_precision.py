"""Storage-precision study with the oracle's C restatement (test
infrastructure; run on the CPU, needs oracle/_ref and oracle/build).

    python oracle/storage_precision.py [work_dir]

A CGFDM half-space (48 x 48 x 40, DH = 100 m, 8-layer PML, Mxy point source
at 1.5 km depth, 4 Hz, 8 surface stations, 800 steps) is set up by the
reference's CPU build, then stepped by the restatement four ways: FP64
(the oracle), FP32, and FP32 arithmetic with the stored state -- wavefield,
RK sum, step start, PML auxiliaries -- rounded after every write to 11
significand bits (FP16 storage with ideal per-field scaling: the FP32
exponent range is kept) or 8 bits (BF16).  A second pass rounds only the
metric/medium array (CJM) and keeps the state in FP32.  Prints the
relative L2 error of the velocity seismograms against FP64 over the first
100, 200, 400 and 800 steps.
"""

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, os.path.join(ROOT, "cgfdm3d-eqr-sc_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import refrun  # noqa: E402
import restated  # noqa: E402
from cgfdm import cases  # noqa: E402


def _round_bits(a: np.ndarray, bits: int) -> np.ndarray:
    u = a.astype(np.float32).view(np.uint32).copy()
    drop = 24 - bits
    lsb = (u >> drop) & 1
    u = (u + np.uint32((1 << (drop - 1)) - 1) + lsb) & ~np.uint32((1 << drop) - 1)
    return u.view(np.float32)


def main(work: str) -> None:
    d = os.path.join(work, "run")
    c = cases.halfspace_case(NX=48, NY=48, NZ=40, nPML=8, steps=800, n_stations=8, depth_m=1500.0, fc=4.0)
    cases.write_case(c, d)
    refrun.run(d)
    b = restated.make_bundle(d, os.path.join(d, "bundle"), "CGFDM")
    ref = restated.run(b, "f64")["stations"][:, :, :3].astype(np.float64)

    def err(st):
        st = st[:, :, :3].astype(np.float64)
        return [np.linalg.norm(st[:, :n] - ref[:, :n]) / np.linalg.norm(ref[:, :n]) for n in (100, 200, 400, 800)]

    print("seismogram rel L2 vs FP64 after 100 / 200 / 400 / 800 steps")
    for p, label in (("f32", "FP32 state"), ("s11", "state at 11 bits (FP16)"), ("s8", "state at 8 bits (BF16)")):
        print(f"  {label:32s}", " ".join(f"{e:.2e}" for e in err(restated.run(b, p)["stations"])))
    b2 = os.path.join(d, "bundle_cjm")
    cjm = np.fromfile(os.path.join(b, "cjm.bin"), np.float32)
    for bits, label in ((11, "CJM at 11 bits, FP32 state"), (8, "CJM at 8 bits, FP32 state")):
        if os.path.exists(b2):
            shutil.rmtree(b2)
        shutil.copytree(b, b2)
        _round_bits(cjm, bits).tofile(os.path.join(b2, "cjm.bin"))
        print(f"  {label:32s}", " ".join(f"{e:.2e}" for e in err(restated.run(b2, "f32")["stations"])))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/tmp/cgfdm_storage_precision")
