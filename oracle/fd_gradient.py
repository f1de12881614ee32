"""FP64 central finite differences of the seismogram misfit, for checking
the adjoint gradient.  Test infrastructure: only tests use this module.

The misfit is J = 1/2 sum over stations, samples and the three velocity
components of (v - d)^2, v from the FP64 restatement of the CGFDM time loop
(oracle/restated/stepper.c) run on a bundle of the reference's own model
(oracle/restated.py make_bundle).  A parameter of one grid point is
perturbed through the bundle's perturb.txt: Vp, Vs or rho of the point,
mapped to (mu, lambda, buoyancy) by mu = rho Vs^2, lambda = rho (Vp^2 -
2 Vs^2), buoyancy = 1 / rho (src/CJM.cpp:52-77), in double.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Sequence, Tuple

import numpy as np

import restated

PARAMS = ("vp", "vs", "rho")


def perturbation(param: str, vs: float, vp: float, rho: float, delta: float) -> Tuple[float, float, float]:
    """(dmu, dlambda, dbuoyancy) of adding delta to Vp, Vs or rho."""
    if param == "vp":
        return 0.0, rho * ((vp + delta) ** 2 - vp ** 2), 0.0
    if param == "vs":
        dmu = rho * ((vs + delta) ** 2 - vs ** 2)
        return dmu, -2.0 * dmu, 0.0
    if param == "rho":
        return delta * vs * vs, delta * (vp * vp - 2.0 * vs * vs), 1.0 / (rho + delta) - 1.0 / rho
    raise ValueError(param)


def misfit(stations64: np.ndarray, observed: np.ndarray) -> float:
    r = stations64[:, :, :3].astype(np.float64) - observed.astype(np.float64)
    return 0.5 * float(np.sum(r * r))


def _run_one(bundle: str, work: str, lines: Sequence[str]) -> np.ndarray:
    os.makedirs(work, exist_ok=True)
    for name in os.listdir(bundle):
        if name.startswith("out_") or name == "perturb.txt":
            continue
        dst = os.path.join(work, name)
        if not os.path.exists(dst):
            os.symlink(os.path.abspath(os.path.join(bundle, name)), dst)
    with open(os.path.join(work, "perturb.txt"), "w") as f:
        f.write("\n".join(lines) + ("\n" if lines else ""))
    subprocess.run([restated.binary("f64"), work], check=True, timeout=3600)
    meta = {}
    with open(os.path.join(bundle, "meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = float(v)
    NT = int(meta["NT"])
    nst = os.path.getsize(os.path.join(bundle, "stations.bin")) // 12
    return np.fromfile(os.path.join(work, "out_stations64.bin"), np.float64).reshape(nst, NT, 9)


def fd_gradient(bundle: str, work_dir: str, medium: np.ndarray, cells: Sequence[Tuple[int, int, int]],
                observed: np.ndarray, rel_step: float = 1e-4, workers: int = 0) -> Dict[str, np.ndarray]:
    """dJ/dVp, dJ/dVs, dJ/drho at `cells` (padded-grid (i, j, k)) by central
    differences with step rel_step times the parameter.  medium is the run's
    [nzp][nyp][nxp][3] (Vs, Vp, rho) volume.  Returns {param: [len(cells)]}
    and "J" (the unperturbed misfit)."""
    jobs: List[Tuple[str, int, int, str, List[str]]] = []
    for c, (i, j, k) in enumerate(cells):
        vs, vp, rho = (float(x) for x in medium[k, j, i])
        base = {"vp": vp, "vs": vs, "rho": rho}
        for p in PARAMS:
            d = rel_step * base[p]
            for sgn in (1, -1):
                dm, dl, db = perturbation(p, vs, vp, rho, sgn * d)
                jobs.append((p, c, sgn, os.path.join(work_dir, f"{p}_{c}_{'p' if sgn > 0 else 'm'}"),
                             [f"{i} {j} {k} {dm!r} {dl!r} {db!r}"]))
    jobs.append(("J", 0, 0, os.path.join(work_dir, "base"), []))
    workers = workers or max(1, os.cpu_count() or 1)
    with ThreadPoolExecutor(workers) as ex:
        res = list(ex.map(lambda jb: misfit(_run_one(bundle, jb[3], jb[4]), observed), jobs))
    out = {p: np.zeros(len(cells)) for p in PARAMS}
    Jp: Dict[Tuple[str, int, int], float] = {}
    for jb, J in zip(jobs, res):
        Jp[(jb[0], jb[1], jb[2])] = J
    for c, (i, j, k) in enumerate(cells):
        vs, vp, rho = (float(x) for x in medium[k, j, i])
        base = {"vp": vp, "vs": vs, "rho": rho}
        for p in PARAMS:
            d = rel_step * base[p]
            out[p][c] = (Jp[(p, c, 1)] - Jp[(p, c, -1)]) / (2.0 * d)
    out["J"] = np.array([Jp[("J", 0, 0)]])
    shutil.rmtree(work_dir, ignore_errors=True)
    return out
