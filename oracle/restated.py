"""Runs the C restatement of the time-stepping path (oracle/restated/stepper.c)
on a run directory the reference's own CPU build has already processed.

Test infrastructure: only tests, the smoke check and the benchmark's
CPU-baseline leg use this module.

The restatement covers the hot path -- the time loop -- and takes the
model the reference built as its input: the metric and medium (CJM), the
CGFDM free-surface matrices, the finite-fault table before its scaling,
the station indices and the scalars of the run, all of which the
reference build's dump hooks write into OUT (oracle/refbuild/
ref_drivers.cpp).  ``precision="f32"`` follows the reference's FP32
arithmetic; ``precision="f64"`` is the FP64 oracle.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from typing import Dict

import numpy as np

import refrun

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")


def binary(precision: str = "f32") -> str:
    """f32, f64, or m16 (FP32 arithmetic with the mixed-precision storage of the CGFDM path)."""
    return os.path.join(BUILD, f"stepper_{precision}")


def available() -> bool:
    return os.access(binary("f32"), os.X_OK) and os.access(binary("f64"), os.X_OK)


def make_bundle(run_dir: str, bundle: str, scheme: str = "CGFDM") -> str:
    """Collects the restatement's inputs from a processed run directory."""
    p = refrun._params(run_dir)
    out = os.path.join(run_dir, p.get("out", "./output"))
    os.makedirs(bundle, exist_ok=True)
    meta = {}
    with open(os.path.join(out, "oracle_meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = v
    sc = scheme.upper() != "CGFDM"
    meta["scheme"] = "1" if sc else "0"
    meta["pml"] = "0" if sc else "1"          # the two reference builds' switches
    meta["exp_decay"] = "1" if sc else "0"
    with open(os.path.join(bundle, "meta.txt"), "w") as f:
        for k, v in meta.items():
            f.write(f"{k} {v}\n")
    shutil.copyfile(os.path.join(out, "oracle_CJM.bin"), os.path.join(bundle, "cjm.bin"))
    if not sc:
        shutil.copyfile(os.path.join(out, "oracle_rDZ.bin"), os.path.join(bundle, "rdz.bin"))
    src = os.path.join(out, "oracle_src.bin")
    if os.path.exists(src):
        shutil.copyfile(src, os.path.join(bundle, "src.bin"))
    ref = refrun.read_outputs(run_dir, scheme)
    # the station file holds global (unpadded) indices (src/station.cpp:412-443)
    xyz = ref.get("station_xyz", np.zeros((0, 3), np.int32)).astype(np.int32) + 3
    xyz.tofile(os.path.join(bundle, "stations.bin"))
    return bundle


def run(bundle: str, precision: str = "f32", timeout: float = 3600.0) -> Dict[str, np.ndarray]:
    subprocess.run([binary(precision), bundle], check=True, timeout=timeout)
    meta = {}
    with open(os.path.join(bundle, "meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = float(v)
    nx, ny, nz, NT = int(meta["nx"]), int(meta["ny"]), int(meta["nz"]), int(meta["NT"])
    nst = os.path.getsize(os.path.join(bundle, "stations.bin")) // 12
    return {
        "stations": np.fromfile(os.path.join(bundle, "out_stations.bin"), np.float32).reshape(nst, NT, 9),
        "W": np.fromfile(os.path.join(bundle, "out_W.bin"), np.float32).reshape(nz + 6, ny + 6, nx + 6, 9),
        "PGV": np.fromfile(os.path.join(bundle, "out_pgv.bin"), np.float32).reshape(ny, nx, 2),
    }
