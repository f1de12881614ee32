"""Generates the committed golden fixtures from the reference's own CPU build.

Each fixture is a small run directory written by cgfdm.cases, run through
oracle/_ref/{cgfdm,scfdm}_ref (compiled from the reference sources by
oracle/refbuild), and reduced to what a test needs: station traces, PGV,
three wavefield planes through the source, and per-component sums and
norms of the final wavefield and of CJM.  The run directories are
re-created from the same seeded generators when a test needs them, so only
the outputs are stored.

    make -C oracle/refbuild && python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "cgfdm3d-eqr-sc_b200"), os.path.join(ROOT, "oracle")]

import golden_cases  # noqa: E402
import refrun  # noqa: E402
from cgfdm import cases  # noqa: E402


def reduce(res: dict, case) -> dict:
    W = res["W"].astype(np.float64)
    out = {
        "stations": res["stations"],
        "station_xyz": res["station_xyz"],
        "PGV": res["PGV"],
        "W_sum": W.sum(axis=(0, 1, 2)),
        "W_l2": np.sqrt((W * W).sum(axis=(0, 1, 2))),
        "CJM_sum": res["CJM"].astype(np.float64).sum(axis=(0, 1, 2)),
        "W_plane_z": res["W"][res["W"].shape[0] - 4],        # surface layer k = _nz - 1
        "W_plane_y": res["W"][:, res["W"].shape[1] // 2],
    }
    return out


def main():
    for name, (mk, scheme) in golden_cases.CASES.items():
        tmp = tempfile.mkdtemp()
        try:
            d = os.path.join(tmp, name)
            cases.write_case(mk(), d, scheme=scheme)
            refrun.run(d, scheme)
            res = refrun.read_outputs(d, scheme)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **reduce(res, None))
            print(name, "stations", res["stations"].shape)
        finally:
            shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
