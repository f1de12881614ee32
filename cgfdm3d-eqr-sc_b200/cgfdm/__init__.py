"""Python view of libcgfdm, the B200 velocity-stress time-stepping library.

The library itself is C++/CUDA behind the C ABI in ``include/cgfdm.h``;
this module loads it with ctypes and wraps a session.  There is no CPU
fallback: if the compiled library is missing, importing a session raises.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import cases  # noqa: F401  (input writers)

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIBDIR = os.path.join(os.path.dirname(_PKG), "lib")
_libs = {}


class CgfdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cgfdm error {code}: {msg}")
        self.code = code


class Info(ctypes.Structure):
    _fields_ = [
        ("scheme", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nxp", ctypes.c_int), ("nyp", ctypes.c_int), ("nzp", ctypes.c_int),
        ("NT", ctypes.c_int), ("steps_done", ctypes.c_int), ("n_stations", ctypes.c_int),
        ("n_fault_cells", ctypes.c_longlong),
        ("DT", ctypes.c_float), ("DH", ctypes.c_float), ("dtmax", ctypes.c_float),
        ("H_min", ctypes.c_float), ("Vp_max", ctypes.c_float),
        ("device_bytes", ctypes.c_double), ("h2d_bytes", ctypes.c_double),
        ("kernel_launches", ctypes.c_longlong),
        ("algo_bytes_per_step", ctypes.c_double),
        ("stage_kernels_per_step", ctypes.c_int),
        ("pgv_fields", ctypes.c_int),
    ]


def lib_path(flavor: str = "fast") -> str:
    """lib/libcgfdm.so ("fast"), lib/libcgfdm_<flavor>.so, or an explicit .so path."""
    if flavor.endswith(".so"):
        return os.path.abspath(flavor)
    name = "libcgfdm.so" if flavor == "fast" else f"libcgfdm_{flavor}.so"
    return os.path.join(_LIBDIR, name)


def load(flavor: str = "fast") -> ctypes.CDLL:
    """Loads lib/libcgfdm[_flavor].so; raises if it has not been built."""
    if flavor in _libs:
        return _libs[flavor]
    path = lib_path(flavor)
    if not os.path.exists(path):
        raise ImportError(f"{path} not built; run `make -C {os.path.dirname(_LIBDIR)}`")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.cgfdm_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]
    L.cgfdm_run.argtypes = [vp, ctypes.c_int]
    L.cgfdm_run_timed.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.cgfdm_info_get.argtypes = [vp, ctypes.POINTER(Info)]
    L.cgfdm_profile_stages.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    fp = ctypes.POINTER(ctypes.c_float)
    L.cgfdm_model_medium.argtypes = [ctypes.c_char_p, ctypes.c_char_p, fp, ctypes.c_longlong,
                                     ctypes.POINTER(ctypes.c_int)]
    L.cgfdm_model_coord.argtypes = [ctypes.c_char_p, ctypes.c_char_p, fp, ctypes.c_longlong, fp,
                                    ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]
    L.cgfdm_get_stations.argtypes = [vp, fp, ctypes.c_longlong]
    L.cgfdm_get_wavefield.argtypes = [vp, fp, ctypes.c_longlong]
    L.cgfdm_get_cjm.argtypes = [vp, fp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]
    L.cgfdm_get_pgv.argtypes = [vp, fp, ctypes.c_longlong]
    L.cgfdm_get_array.argtypes = [vp, ctypes.c_char_p, vp, ctypes.POINTER(ctypes.c_longlong)]
    L.cgfdm_write_outputs.argtypes = [vp]
    L.cgfdm_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.cgfdm_checkpoint.argtypes = [vp, vp, ctypes.c_longlong]
    L.cgfdm_restore.argtypes = [vp, vp, ctypes.c_longlong]
    L.cgfdm_destroy.argtypes = [vp]
    L.cgfdm_set_wavefield.argtypes = [vp, fp, ctypes.c_longlong]
    L.cgfdm_set_medium.argtypes = [vp, fp, ctypes.c_longlong]
    L.cgfdm_adjoint_apply.argtypes = [vp, ctypes.c_int, fp, ctypes.c_longlong]
    L.cgfdm_gradient_profile.argtypes = [vp, fp]
    ip = ctypes.POINTER(ctypes.c_int)
    L.cgfdm_autotune.argtypes = [vp, ctypes.c_int, ip, ip, ctypes.POINTER(ctypes.c_float)]
    L.cgfdm_set_tiling.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.cgfdm_get_tiling.argtypes = [vp, ip, ip]
    L.cgfdm_set_stage_tile.argtypes = [vp, ctypes.c_int]
    L.cgfdm_get_stage_tile.argtypes = [vp, ip]
    L.cgfdm_batch_set_stage_tile.argtypes = [vp, ctypes.c_int]
    L.cgfdm_batch_get_stage_tile.argtypes = [vp, ip]
    L.cgfdm_batch_autotune.argtypes = [vp, ctypes.c_int, ip, ip, ctypes.POINTER(ctypes.c_float)]
    L.cgfdm_gradient.argtypes = [vp, fp, ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(ctypes.c_double), fp,
                                 ctypes.c_longlong]
    L.cgfdm_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    L.cgfdm_batch_run.argtypes = [vp, ctypes.c_int]
    L.cgfdm_batch_run_timed.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.cgfdm_batch_destroy.argtypes = [vp]
    L.cgfdm_batch_last_error.argtypes = [vp]
    L.cgfdm_batch_last_error.restype = ctypes.c_char_p
    L.cgfdm_last_error.argtypes = [vp]
    L.cgfdm_last_error.restype = ctypes.c_char_p
    L.cgfdm_build_flavor.restype = ctypes.c_char_p
    _libs[flavor] = L
    return L


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def model_medium(run_dir: str, options: Optional[str] = None, flavor: str = "fast") -> np.ndarray:
    """The medium a run directory describes, [nzp][nyp][nxp][3] (Vs, Vp, rho),
    built on the host without a GPU (cgfdm_model_medium)."""
    L = load(flavor)
    dims = (ctypes.c_int * 3)()
    o = options.encode() if options else None
    rc = L.cgfdm_model_medium(run_dir.encode(), o, None, 0, dims)
    if rc:
        raise CgfdmError(rc, L.cgfdm_last_error(None).decode())
    out = np.zeros((dims[0], dims[1], dims[2], 3), np.float32)
    rc = L.cgfdm_model_medium(run_dir.encode(), o, _fptr(out), out.size, dims)
    if rc:
        raise CgfdmError(rc, L.cgfdm_last_error(None).decode())
    return out


def model_coord(run_dir: str, options: Optional[str] = None, flavor: str = "fast"):
    """The surface height [nyp][nxp] and the coordinates [nzp][nyp][nxp][3]
    (x, y, z) a run directory describes, built on the host without a GPU
    (cgfdm_model_coord)."""
    L = load(flavor)
    dims = (ctypes.c_int * 3)()
    o = options.encode() if options else None
    rc = L.cgfdm_model_coord(run_dir.encode(), o, None, 0, None, 0, dims)
    if rc:
        raise CgfdmError(rc, L.cgfdm_last_error(None).decode())
    terrain = np.zeros((dims[1], dims[2]), np.float32)
    coord = np.zeros((dims[0], dims[1], dims[2], 3), np.float32)
    rc = L.cgfdm_model_coord(run_dir.encode(), o, _fptr(terrain), terrain.size, _fptr(coord), coord.size, dims)
    if rc:
        raise CgfdmError(rc, L.cgfdm_last_error(None).decode())
    return terrain, coord


class Session:
    """One run directory simulated on one GPU (``cgfdm_create`` ... ``cgfdm_destroy``)."""

    def __init__(self, run_dir: str, options: Optional[str] = None, device: int = 0, flavor: str = "fast"):
        self.L = load(flavor)
        self._h = ctypes.c_void_p()
        rc = self.L.cgfdm_create(run_dir.encode(), options.encode() if options else None, device,
                                 ctypes.byref(self._h))
        if rc:
            raise CgfdmError(rc, self.L.cgfdm_last_error(None).decode())
        self.run_dir = run_dir

    def _check(self, rc: int):
        if rc:
            raise CgfdmError(rc, self.L.cgfdm_last_error(self._h).decode())

    @property
    def info(self) -> Info:
        i = Info()
        self._check(self.L.cgfdm_info_get(self._h, ctypes.byref(i)))
        return i

    def run(self, nsteps: int) -> None:
        self._check(self.L.cgfdm_run(self._h, int(nsteps)))

    def run_timed(self, nsteps: int) -> float:
        ms = ctypes.c_float()
        self._check(self.L.cgfdm_run_timed(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def profile_stages(self, nsteps: int) -> float:
        ms = ctypes.c_float()
        self._check(self.L.cgfdm_profile_stages(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def checkpoint(self) -> np.ndarray:
        """The time-stepping state at the current step boundary (cgfdm_checkpoint)."""
        n = ctypes.c_longlong()
        self._check(self.L.cgfdm_checkpoint_size(self._h, ctypes.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(self.L.cgfdm_checkpoint(self._h, buf.ctypes.data_as(ctypes.c_void_p), buf.size))
        return buf

    def restore(self, buf: np.ndarray) -> None:
        """Loads a checkpoint of a session of the same run directory (cgfdm_restore)."""
        buf = np.ascontiguousarray(buf, np.uint8)
        self._check(self.L.cgfdm_restore(self._h, buf.ctypes.data_as(ctypes.c_void_p), buf.size))

    def stations(self) -> np.ndarray:
        i = self.info
        out = np.zeros((i.n_stations, i.NT, 9), np.float32)
        self._check(self.L.cgfdm_get_stations(self._h, _fptr(out), out.size))
        return out

    def wavefield(self) -> np.ndarray:
        i = self.info
        out = np.zeros((i.nzp, i.nyp, i.nxp, 9), np.float32)
        self._check(self.L.cgfdm_get_wavefield(self._h, _fptr(out), out.size))
        return out

    def cjm(self) -> np.ndarray:
        i = self.info
        nf = ctypes.c_int()
        self._check(self.L.cgfdm_get_cjm(self._h, None, 0, ctypes.byref(nf)))
        out = np.zeros((i.nzp, i.nyp, i.nxp, nf.value), np.float32)
        self._check(self.L.cgfdm_get_cjm(self._h, _fptr(out), out.size, ctypes.byref(nf)))
        return out

    def pgv(self) -> np.ndarray:
        i = self.info
        out = np.zeros((i.ny, i.nx, i.pgv_fields), np.float32)
        self._check(self.L.cgfdm_get_pgv(self._h, _fptr(out), out.size))
        return out

    _ARRAY_DTYPES = {"srcIndex": np.int64, "stationXYZ": np.int32}

    def array(self, name: str) -> np.ndarray:
        """A model array in the reference's layout (cgfdm_get_array): rDZ_DX,
        rDZ_DY, pml_{alpha,beta,d}_{x,y,z}, srcIndex, momentRate, stationXYZ."""
        n = ctypes.c_longlong(0)
        self._check(self.L.cgfdm_get_array(self._h, name.encode(), None, ctypes.byref(n)))
        dt = np.dtype(self._ARRAY_DTYPES.get(name, np.float32))
        out = np.zeros(n.value // dt.itemsize, dt)
        self._check(self.L.cgfdm_get_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p),
                                           ctypes.byref(n)))
        return out

    def write_outputs(self) -> None:
        self._check(self.L.cgfdm_write_outputs(self._h))

    def check_finite(self):
        """(count, first) of NaN/Inf values in the state (cgfdm_check_finite):
        first = ((k * ny + j) * nx + i) * 9 + field over interior indices, -1
        when count is 0."""
        self.L.cgfdm_check_finite.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                              ctypes.POINTER(ctypes.c_longlong)]
        c, f = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.L.cgfdm_check_finite(self._h, ctypes.byref(c), ctypes.byref(f)))
        return c.value, f.value

    def set_wavefield(self, w: np.ndarray) -> None:
        """Overwrites the wavefield, [nzp][nyp][nxp][9] (cgfdm_set_wavefield)."""
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.L.cgfdm_set_wavefield(self._h, _fptr(w), w.size))

    def set_medium(self, medium: np.ndarray) -> None:
        """New (Vs, Vp, rho) medium, [nzp][nyp][nxp][3]; back to step 0 (cgfdm_set_medium)."""
        medium = np.ascontiguousarray(medium, np.float32)
        self._check(self.L.cgfdm_set_medium(self._h, _fptr(medium), medium.size))

    def adjoint_apply(self, state: np.ndarray, nsteps: int) -> np.ndarray:
        """Transpose of the last ``nsteps`` steps applied to ``state`` (cgfdm_adjoint_apply)."""
        out = np.array(state, np.float32, copy=True, order="C")
        self._check(self.L.cgfdm_adjoint_apply(self._h, int(nsteps), _fptr(out), out.size))
        return out

    def gradient(self, observed: np.ndarray, checkpoint_every: int = 100):
        """Misfit J = 1/2 sum (v - d)^2 over the station velocities and its
        gradient [3][nz][ny][nx] with respect to (Vp, Vs, rho) (cgfdm_gradient).
        ``observed`` is [n_stations][NT][3]."""
        i = self.info
        obs = np.ascontiguousarray(observed, np.float32)
        if obs.shape != (i.n_stations, i.NT, 3):
            raise ValueError(f"observed must be ({i.n_stations}, {i.NT}, 3), got {obs.shape}")
        grad = np.zeros((3, i.nz, i.ny, i.nx), np.float32)
        J = ctypes.c_double()
        self._check(self.L.cgfdm_gradient(self._h, _fptr(obs), obs.size, int(checkpoint_every), ctypes.byref(J),
                                          _fptr(grad), grad.size))
        return J.value, grad

    def autotune(self, trial_steps: int = 4):
        """Times candidate work decompositions of the stage kernel and keeps
        the fastest (cgfdm_autotune); returns (kchunk, ctas, ms_per_step)."""
        kc, ct, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.L.cgfdm_autotune(self._h, int(trial_steps), ctypes.byref(kc), ctypes.byref(ct),
                                          ctypes.byref(ms)))
        return kc.value, ct.value, ms.value

    def run_precise(self, nsteps: int, bits: int = 64, wavefield: bool = False):
        """The time loop from step 0 in reference form with state and
        arithmetic in FP64 (``bits`` 64) or FP32 (32) on this session's model
        (cgfdm_run_precise).  Returns (stations [n][nsteps][9], pgv
        [ny][nx][2], wavefield [nzp][nyp][nxp][9] or None), all float64."""
        i = self.info
        dp = ctypes.POINTER(ctypes.c_double)
        self.L.cgfdm_run_precise.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, ctypes.c_longlong, dp,
                                             ctypes.c_longlong, dp, ctypes.c_longlong]
        st = np.zeros((i.n_stations, int(nsteps), 9), np.float64)
        pgv = np.zeros((i.ny, i.nx, 2), np.float64)
        W = np.zeros((i.nzp, i.nyp, i.nxp, 9), np.float64) if wavefield else None

        def p(a):
            return a.ctypes.data_as(dp) if a is not None and a.size else None

        self._check(self.L.cgfdm_run_precise(self._h, int(nsteps), int(bits), p(st), st.size, p(pgv), pgv.size,
                                             p(W), W.size if W is not None else 0))
        return st, pgv, W

    def create_profile(self) -> dict:
        """Host wall ms of the set-up (cgfdm_create_profile)."""
        ms = (ctypes.c_double * 14)()
        self.L.cgfdm_create_profile.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        self._check(self.L.cgfdm_create_profile(self._h, ms))
        return {"model_from_files_ms": ms[0], "device_setup_ms": ms[1], "create_ms": ms[2],
                "graph_capture_ms": ms[3],
                "model_parts_ms": {"coordinates_terrain": ms[4], "medium": ms[5], "ranges_pml": ms[6],
                                   "sources": ms[7], "stations": ms[8]},
                "device_setup_parts_ms": {"alloc_upload_cfl": ms[9], "enqueue_rest": ms[10], "complete": ms[11],
                                          "of_which_alloc": ms[12], "of_which_upload": ms[13]}}

    def test_stall(self, item: int, fill: int, wait_cycles: int) -> None:
        """Test hook (cgfdm_test_stall): the next stage launch's work item
        ``item`` leaves plane copy ``fill`` unissued, once, and the stage
        kernel's bounded waits give up after ``wait_cycles`` clocks."""
        self.L.cgfdm_test_stall.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_longlong]
        self._check(self.L.cgfdm_test_stall(self._h, int(item), int(fill), int(wait_cycles)))

    def set_tiling(self, kchunk: int, ctas: int) -> None:
        self._check(self.L.cgfdm_set_tiling(self._h, int(kchunk), int(ctas)))

    def tiling(self):
        kc, ct = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.cgfdm_get_tiling(self._h, ctypes.byref(kc), ctypes.byref(ct)))
        return kc.value, ct.value

    def set_stage_tile(self, rows: int) -> None:
        """Column-tile height of the CGFDM stage kernel (cgfdm_set_stage_tile):
        4 or 8 rows of 32; 8 needs FP32 storage and a whole grid (not a part)."""
        self._check(self.L.cgfdm_set_stage_tile(self._h, int(rows)))

    def stage_tile(self) -> int:
        r = ctypes.c_int()
        self._check(self.L.cgfdm_get_stage_tile(self._h, ctypes.byref(r)))
        return r.value

    def gradient_profile(self):
        """Device ms of the last gradient's phases: forward with checkpoints,
        segment re-runs storing the stage RHS, adjoint steps."""
        ms = np.zeros(3, np.float32)
        self._check(self.L.cgfdm_gradient_profile(self._h, _fptr(ms)))
        return tuple(float(x) for x in ms)

    def close(self) -> None:
        if self._h:
            self.L.cgfdm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """CGFDM sessions advanced together, one persistent stage launch for all
    (``cgfdm_batch_create`` ... ``cgfdm_batch_destroy``).  The sessions stay
    owned by the caller and must outlive the batch."""

    def __init__(self, sessions):
        self.sessions = list(sessions)
        self.L = self.sessions[0].L
        arr = (ctypes.c_void_p * len(self.sessions))(*[s._h.value for s in self.sessions])
        self._h = ctypes.c_void_p()
        rc = self.L.cgfdm_batch_create(arr, len(self.sessions), ctypes.byref(self._h))
        if rc:
            raise CgfdmError(rc, self.L.cgfdm_batch_last_error(None).decode())

    def _check(self, rc: int):
        if rc:
            raise CgfdmError(rc, self.L.cgfdm_batch_last_error(self._h).decode())

    def run(self, nsteps: int) -> None:
        self._check(self.L.cgfdm_batch_run(self._h, int(nsteps)))

    def run_timed(self, nsteps: int) -> float:
        ms = ctypes.c_float()
        self._check(self.L.cgfdm_batch_run_timed(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def autotune(self, trial_steps: int = 4):
        """Tunes the batched launch's work decomposition (cgfdm_batch_autotune);
        returns (kchunk, ctas, ms_per_step)."""
        kc, ct, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.L.cgfdm_batch_autotune(self._h, int(trial_steps), ctypes.byref(kc), ctypes.byref(ct),
                                                ctypes.byref(ms)))
        return kc.value, ct.value, ms.value

    def set_stage_tile(self, rows: int) -> None:
        """Rows (4 or 8) of the 32-column tiles of the batched stage launch
        (cgfdm_batch_set_stage_tile)."""
        self._check(self.L.cgfdm_batch_set_stage_tile(self._h, int(rows)))

    def stage_tile(self) -> int:
        r = ctypes.c_int()
        self._check(self.L.cgfdm_batch_get_stage_tile(self._h, ctypes.byref(r)))
        return r.value

    def close(self) -> None:
        if self._h:
            self.L.cgfdm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
