"""Generates tests/golden/c1_halfspace.npz: the reference's CPU-runnable
benchmark case run through the reference's own CPU build and through the
FP64 oracle.

The case is the homogeneous half-space of cgfdm.cases.halfspace_case with
its defaults: 128 x 128 x 96 points, DH = 100 m, Vp 6000 / Vs 3464 m/s,
rho 2670 kg/m^3, flat free surface, 12-layer PML on five faces, one Mxy
point source of 1e16 N m (a finite-fault file with one real and one dummy
point) with a 2 Hz Ricker rate at 3 km depth, DT at 0.8 of the reference's
CFL bound, 1000 RK4 steps, 16 surface stations on a line.

Outputs kept: the reference build's station traces (all nine components),
PGV, the final wavefield's surface plane and per-component sums and norms;
the FP64 oracle's velocity traces, surface-plane velocities and
per-component norms.  About 13 core-minutes for each of the two runs (they
run side by side).

    make -C oracle/refbuild && make -C oracle/restated && python tests/golden/make_golden_c1.py
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "cgfdm3d-eqr-sc_b200"), os.path.join(ROOT, "oracle")]

import refrun  # noqa: E402
import restated  # noqa: E402
from cgfdm import cases  # noqa: E402


def c1_case():
    return cases.halfspace_case()


def main(out_path=os.path.join(HERE, "c1_halfspace.npz")):
    tmp = tempfile.mkdtemp()
    try:
        d = os.path.join(tmp, "c1")
        cases.write_case(c1_case(), d, scheme="CGFDM")
        # the reference run writes the model dumps the FP64 oracle starts from,
        # so it goes first; a copy of the directory runs nothing else
        secs = refrun.run(d, "CGFDM", timeout=7200)
        ref = refrun.read_outputs(d, "CGFDM")
        b = restated.make_bundle(d, os.path.join(d, "bundle"), "CGFDM")
        with ThreadPoolExecutor(1) as ex:
            f64 = ex.submit(restated.run, b, "f64", 7200).result()
        W = ref["W"].astype(np.float64)
        W64 = f64["W"].astype(np.float64)
        ks = W.shape[0] - 4   # surface layer, k = _nz - 1
        np.savez_compressed(
            out_path,
            stations=ref["stations"],
            station_xyz=ref["station_xyz"],
            PGV=ref["PGV"],
            W_sum=W.sum(axis=(0, 1, 2)),
            W_l2=np.sqrt((W * W).sum(axis=(0, 1, 2))),
            W_plane_z=ref["W"][ks],
            stations64=f64["stations"][:, :, :3],
            W_l2_64=np.sqrt((W64 * W64).sum(axis=(0, 1, 2))),
            W_plane_z64=f64["W"][ks][:, :, :3],
            ref_seconds=np.float64(secs),
        )
        print("c1: reference", secs, "s; stations", ref["stations"].shape)
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    main(*sys.argv[1:])
