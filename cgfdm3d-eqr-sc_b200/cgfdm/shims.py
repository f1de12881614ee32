"""ctypes binding of the per-function entry points (include/cgfdm_shims.h):
the reference's step drivers -- waveDeriv, freeSurfaceDeriv, pmlDeriv,
pmlFreeSurfaceDeriv, waveRk, pmlRk, calculateMomentRate, addMomenteRate,
storageStation, comparePGV, SolveDisplacement, storage_W_pre and, for
ME-AWENO, waveDeriv_alternative_flux_FD, waveRk_tvd, charfreeSurfaceDeriv,
expDecayLayers -- on device
arrays in the reference's layouts, here torch CUDA tensors.  Argument names
and meanings are the reference's (src/propagate.cpp:186-309); the grid is
passed as the padded sizes (_nx_, _ny_, _nz_).  Errors raise CgfdmError
with the library's message."""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

from . import CgfdmError, load

_i, _f, _ll, _p = ctypes.c_int, ctypes.c_float, ctypes.c_longlong, ctypes.c_void_p
_pp = ctypes.POINTER(ctypes.c_void_p)
_ip = ctypes.POINTER(ctypes.c_int)

_SIGS = {
    "cgfdm_waveDeriv": [_i, _i, _i, _f, _p, _p, _p, _p, _p, _p, _i, _i, _i, _f, _p],
    "cgfdm_freeSurfaceDeriv": [_i, _i, _i, _f, _p, _p, _p, _p, _p, _p, _p, _i, _i, _i, _f, _p],
    "cgfdm_pmlDeriv": [_i, _i, _i, _i, _f, _p, _p, _p, _pp, _pp, _ip, _i, _i, _i, _i, _f, _p],
    "cgfdm_pmlFreeSurfaceDeriv": [_i, _i, _i, _i, _f, _p, _p, _pp, _p, _p, _p, _p, _ip, _i, _i, _f, _p],
    "cgfdm_waveRk": [_i, _i, _i, _i, _p, _p, _p, _p, _p],
    "cgfdm_pmlRk": [_i, _i, _i, _i, _i, _pp, _ip, _i, _p],
    "cgfdm_calculateMomentRate": [_ll, _ll, _p, _p, _p, _f, _i, _p],
    "cgfdm_addMomenteRate": [_ll, _i, _f, _p, _p, _p, _p, _i, _i, _f, _i, _p, _p],
    "cgfdm_storageStation": [_i, _i, _i, _i, _i, _p, _p, _p, _i, _i, _p, _p],
    "cgfdm_comparePGV": [_i, _i, _i, _p, _p, _f, _i, _i, _p, _p, _p],
    "cgfdm_SolveDisplacement": [_i, _i, _i, _p, _p, _i, _p, _f, _p],
    "cgfdm_storage_W_pre": [_i, _i, _i, _p, _p, _p],
    "cgfdm_loadPointSource_ricker": [_i, _i, _i, _i, _i, _i, _p, _p, _i, _i, _f, _f, _f, _i, _p],
    "cgfdm_loadPointSource_double_couple": [_i, _i, _i, _i, _i, _i, _p, _p, _i, _i, _f, _f, _f, _f, _f, _f, _f,
                                            _i, _p],
    "cgfdm_waveDeriv_alternative_flux_FD": [_i, _i, _i, _f, _p, _p, _p, _p, _f, _f, _p],
    "cgfdm_waveRk_tvd": [_i, _i, _i, _i, _p, _p, _p, _p],
    "cgfdm_charfreeSurfaceDeriv": [_i, _i, _i, _p, _p, _p],
    "cgfdm_expDecayLayers": [_i, _i, _i, _p, _i, _p],
}


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _ptrs(ts: Sequence) -> ctypes.Array:
    return (ctypes.c_void_p * len(ts))(*[_ptr(t) for t in ts])


class Shims:
    """The entry points of one library flavour ("fast" or "exact")."""

    def __init__(self, flavor: str = "fast"):
        self.L = load(flavor)
        for name, args in _SIGS.items():
            fn = getattr(self.L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        self.L.cgfdm_shim_last_error.restype = ctypes.c_char_p

    def _call(self, name: str, *args):
        rc = getattr(self.L, name)(*args)
        if rc:
            raise CgfdmError(rc, self.L.cgfdm_shim_last_error().decode())

    def waveDeriv(self, g, h_W, W, CJM, pml_beta, FB, DT, stream=None):
        bx, by, bz = pml_beta if pml_beta is not None else (None, None, None)
        self._call("cgfdm_waveDeriv", *g, g.rDH, _ptr(h_W), _ptr(W), _ptr(CJM), _ptr(bx), _ptr(by), _ptr(bz),
                   *FB, DT, stream)

    def freeSurfaceDeriv(self, g, h_W, W, CJM, rDZ_DX, rDZ_DY, pml_beta, FB, DT, stream=None):
        bx, by = (pml_beta[0], pml_beta[1]) if pml_beta is not None else (None, None)
        self._call("cgfdm_freeSurfaceDeriv", *g, g.rDH, _ptr(h_W), _ptr(W), _ptr(CJM), _ptr(rDZ_DX), _ptr(rDZ_DY),
                   _ptr(bx), _ptr(by), *FB, DT, stream)

    def pmlDeriv(self, g, nPML, h_W, W, CJM, aux, pml, border, free_surface, FB, DT, stream=None):
        self._call("cgfdm_pmlDeriv", *g, nPML, g.rDH, _ptr(h_W), _ptr(W), _ptr(CJM), _ptrs(aux), _ptrs(pml),
                   (ctypes.c_int * 6)(*border), int(free_surface), *FB, DT, stream)

    def pmlFreeSurfaceDeriv(self, g, nPML, W, CJM, aux, rDZ_DX, rDZ_DY, pml_d_x, pml_d_y, border, FB, DT,
                            stream=None):
        self._call("cgfdm_pmlFreeSurfaceDeriv", *g, nPML, g.rDH, _ptr(W), _ptr(CJM), _ptrs(aux), _ptr(rDZ_DX),
                   _ptr(rDZ_DY), _ptr(pml_d_x), _ptr(pml_d_y), (ctypes.c_int * 6)(*border), FB[0], FB[1], DT, stream)

    def waveRk(self, g, irk, h_W, W, t_W, m_W, stream=None):
        self._call("cgfdm_waveRk", *g, irk, _ptr(h_W), _ptr(W), _ptr(t_W), _ptr(m_W), stream)

    def pmlRk(self, nx, ny, nz, nPML, irk, aux, border, free_surface, stream=None):
        self._call("cgfdm_pmlRk", nx, ny, nz, nPML, irk, _ptrs(aux), (ctypes.c_int * 6)(*border),
                   int(free_surface), stream)

    def calculateMomentRate(self, npts, nt, CJM, momentRate, srcIndex, DH, scheme=0, stream=None):
        self._call("cgfdm_calculateMomentRate", npts, nt, _ptr(CJM), _ptr(momentRate), _ptr(srcIndex), DH, scheme,
                   stream)

    def addMomenteRate(self, npts, nt, dt, W, srcIndex, momentRate, momentRateSlice, it, irk, DT, scheme=0,
                       CJM=None, stream=None):
        self._call("cgfdm_addMomenteRate", npts, nt, dt, _ptr(W), _ptr(srcIndex), _ptr(momentRate),
                   _ptr(momentRateSlice), it, irk, DT, scheme, _ptr(CJM), stream)

    def loadPointSource_ricker(self, g, S, W, CJM, it, irk, DT, DH, rickerfc, scheme=0, stream=None):
        self._call("cgfdm_loadPointSource_ricker", *g, *S, _ptr(W), _ptr(CJM), it, irk, DT, DH, rickerfc, scheme,
                   stream)

    def loadPointSource_double_couple(self, g, S, W, CJM, it, irk, DT, DH, strike, dip, rake, Mw, duration,
                                      scheme=0, stream=None):
        self._call("cgfdm_loadPointSource_double_couple", *g, *S, _ptr(W), _ptr(CJM), it, irk, DT, DH, strike, dip,
                   rake, Mw, duration, scheme, stream)

    def storageStation(self, g, NT, stationNum, XYZ, wave, W, it, scheme=0, CJM=None, stream=None):
        self._call("cgfdm_storageStation", *g, NT, stationNum, _ptr(XYZ), _ptr(wave), _ptr(W), it, scheme,
                   _ptr(CJM), stream)

    def comparePGV(self, nx, ny, nz, W, pgv, DT, it, scheme=0, CJM=None, W_pre=None, stream=None):
        self._call("cgfdm_comparePGV", nx, ny, nz, _ptr(W), _ptr(pgv), DT, it, scheme, _ptr(CJM), _ptr(W_pre),
                   stream)

    def SolveDisplacement(self, g, W, Dis, DT, scheme=0, CJM=None, stream=None):
        self._call("cgfdm_SolveDisplacement", *g, _ptr(W), _ptr(Dis), scheme, _ptr(CJM), DT, stream)

    def storage_W_pre(self, g, W_pre, W, stream=None):
        self._call("cgfdm_storage_W_pre", *g, _ptr(W_pre), _ptr(W), stream)

    def waveDeriv_alternative_flux_FD(self, g, h_W, W, Riemann_flux, CJM, alpha, DT, stream=None):
        self._call("cgfdm_waveDeriv_alternative_flux_FD", *g, g.rDH, _ptr(h_W), _ptr(W), _ptr(Riemann_flux),
                   _ptr(CJM), alpha, DT, stream)

    def waveRk_tvd(self, g, irk, h_W, W, m_W, stream=None):
        self._call("cgfdm_waveRk_tvd", *g, irk, _ptr(h_W), _ptr(W), _ptr(m_W), stream)

    def charfreeSurfaceDeriv(self, g, W, CJM, stream=None):
        self._call("cgfdm_charfreeSurfaceDeriv", *g, _ptr(W), _ptr(CJM), stream)

    def expDecayLayers(self, g, W, free_surface=True, stream=None):
        self._call("cgfdm_expDecayLayers", *g, _ptr(W), int(free_surface), stream)


class Grid(tuple):
    """(_nx_, _ny_, _nz_) with rDH, the GRID fields the drivers read."""

    def __new__(cls, nxp: int, nyp: int, nzp: int, rDH: float):
        t = super().__new__(cls, (nxp, nyp, nzp))
        t.rDH = rDH
        return t
