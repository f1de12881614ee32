"""Runs the reference's own CPU build (oracle/_ref/{cgfdm,scfdm}_ref) on a run
directory and reads back what it wrote.  Test infrastructure: only tests,
the smoke check and the benchmark's CPU-baseline leg use this module.

The binaries are built from the reference sources by oracle/refbuild
(``make -C oracle/refbuild``).  They read params.json and station.json from
their working directory (src/getParams.cpp:20, src/station.cpp:95) and write
into OUT: station_mpi_0_0_0.bin, PGV_Z_mpi_0_0_0.bin, and, through the
oracle's dump hooks, oracle_CJM.bin, oracle_rDZ.bin and oracle_final_W.bin.
"""

from __future__ import annotations

import json
import os
import shutil
import subprocess
import time
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ref_binary(scheme: str = "CGFDM", displacement: bool = False, pga: bool = False) -> str:
    """The build of one scheme; ``displacement`` picks the one compiled with
    SOLVE_DISPLACEMENT (src/propagate.cpp:101-104, 264-266, 305-307), which
    also writes FreeSurfUx/Uy/Uz with the free-surface snapshots; ``pga``
    the one compiled with SOLVE_PGA (a four-field PGV file, src/PGV.cpp:61-175)."""
    name = "cgfdm_ref" if scheme.upper() == "CGFDM" else "scfdm_ref"
    return os.path.join(REF_DIR, name + ("_dis" if displacement else "") + ("_pga" if pga else ""))


def available(scheme: str = "CGFDM", displacement: bool = False, pga: bool = False) -> bool:
    return os.access(ref_binary(scheme, displacement, pga), os.X_OK)


def _params(run_dir: str) -> dict:
    with open(os.path.join(run_dir, "params.json")) as f:
        p = json.load(f)
    return {k.lower(): v for k, v in p.items()}


def run(run_dir: str, scheme: str = "CGFDM", timeout: float = 3600.0, log: Optional[str] = None,
        displacement: bool = False, pga: bool = False) -> float:
    """Runs the reference binary in run_dir; returns wall seconds."""
    out = os.path.join(run_dir, _params(run_dir).get("out", "./output"))
    os.makedirs(out, exist_ok=True)
    t0 = time.perf_counter()
    with open(log or os.path.join(run_dir, "ref.log"), "w") as lf:
        subprocess.run([ref_binary(scheme, displacement, pga)], cwd=run_dir, stdout=lf, stderr=subprocess.STDOUT, check=True,
                       timeout=timeout)
    return time.perf_counter() - t0


def run_many(run_dirs, scheme: str = "CGFDM", timeout: float = 3600.0) -> None:
    """Runs the reference binary in several run directories at once, one
    process each (at most one per host core)."""
    from concurrent.futures import ThreadPoolExecutor

    workers = max(1, min(len(run_dirs), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as ex:
        for f in [ex.submit(run, d, scheme, timeout) for d in run_dirs]:
            f.result()


def read_outputs(run_dir: str, scheme: str = "CGFDM") -> Dict[str, np.ndarray]:
    p = _params(run_dir)
    NX, NY, NZ = p["nx"], p["ny"], p["nz"]
    nxp, nyp, nzp = NX + 6, NY + 6, NZ + 6
    NT = int(p["tmax"] / float(np.float32(p["dt"])))
    out = os.path.join(run_dir, p.get("out", "./output"))
    res: Dict[str, np.ndarray] = {}
    sp = os.path.join(out, "station_mpi_0_0_0.bin")
    if os.path.exists(sp):
        raw = np.fromfile(sp, dtype=np.uint8)
        nst = raw.size // (12 + NT * 36)
        res["station_xyz"] = np.frombuffer(raw[: nst * 12].tobytes(), np.int32).reshape(nst, 3)
        res["stations"] = np.frombuffer(raw[nst * 12:].tobytes(), np.float32).reshape(nst, NT, 9)
    wp = os.path.join(out, "oracle_final_W.bin")
    if os.path.exists(wp):
        res["W"] = np.fromfile(wp, np.float32).reshape(nzp, nyp, nxp, 9)
    cp = os.path.join(out, "oracle_CJM.bin")
    if os.path.exists(cp):
        nf = 13 if scheme.upper() == "CGFDM" else 19
        res["CJM"] = np.fromfile(cp, np.float32).reshape(nzp, nyp, nxp, nf)
    pg = os.path.join(out, "PGV_Z_mpi_0_0_0.bin")
    if os.path.exists(pg):
        raw = np.fromfile(pg, np.float32)
        res["PGV"] = raw.reshape(NY, NX, raw.size // (NY * NX))   # 2 fields, 4 with SOLVE_PGA
    return res


def run_copy(run_dir: str, work_dir: str, scheme: str = "CGFDM", **kw) -> Dict[str, np.ndarray]:
    """Copies a run directory, runs the reference there and reads its outputs."""
    if os.path.exists(work_dir):
        shutil.rmtree(work_dir)
    shutil.copytree(run_dir, work_dir)
    run(work_dir, scheme, **kw)
    return read_outputs(work_dir, scheme)
