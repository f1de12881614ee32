"""Domain decomposition of a CGFDM run over parts (cgfdm_create_part ...).

A grid is split into parts[0] x parts[1] x parts[2] sub-domains, as the
reference's MPI ranks hold it (src/init_grid.cpp, src/MPI_send_recv_FLOAT.cpp);
each part is one session.  A step is five phases (the source, then the four
RK stages); after each of the first four every part refreshes the halos at
its internal faces, axis by axis, from its neighbours.

* ``plan`` -- the decomposition's arithmetic (extents, neighbours), host only;
* ``run_local`` -- every part in one process on one GPU, halos moved by
  device copies: a decomposed run on one device, which must reproduce the
  single-domain run bit for bit;
* ``run_distributed`` -- one part per rank of a torch.distributed group
  (NCCL between GPUs), halos sent with send/recv.

The exchange itself (``exchange``) only needs a part object with
``halo_count``, ``pack`` and ``unpack`` and a transport, so its logic is
tested on the CPU with gloo ranks and array-backed parts.
"""

from __future__ import annotations

import ctypes
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import CgfdmError, Session, load

FACES = 6   # 0 x-low, 1 x-high, 2 y-low, 3 y-high, 4 z-low, 5 z-high


# ------------------------------------------------------------------ plan
def extent(N: int, n: int, c: int) -> Tuple[int, int]:
    """Interior offset and size of part c of n along an axis of N points
    (sizes as even as possible, the first N % n parts one larger)."""
    base, rem = divmod(N, n)
    return c * base + min(c, rem), base + (1 if c < rem else 0)


def neighbour(parts: Sequence[int], coord: Sequence[int], face: int) -> Optional[Tuple[int, int, int]]:
    """The part on side `face` of part `coord`, or None at the boundary."""
    axis, side = divmod(face, 2)
    c = list(coord)
    c[axis] += 1 if side else -1
    if c[axis] < 0 or c[axis] >= parts[axis]:
        return None
    return tuple(c)


def rank_of(parts: Sequence[int], coord: Sequence[int]) -> int:
    """x fastest, as the reference numbers its ranks (src/init_MPI.cpp)."""
    return coord[0] + parts[0] * (coord[1] + parts[1] * coord[2])


def coord_of(parts: Sequence[int], rank: int) -> Tuple[int, int, int]:
    x = rank % parts[0]
    y = (rank // parts[0]) % parts[1]
    return (x, y, rank // (parts[0] * parts[1]))


def plan(shape: Sequence[int], parts: Sequence[int]) -> List[dict]:
    """Every part of the decomposition: coord, rank, interior lo and n,
    whether it holds the free surface, and its neighbours by face."""
    out = []
    for r in range(parts[0] * parts[1] * parts[2]):
        c = coord_of(parts, r)
        lo, n = zip(*(extent(shape[a], parts[a], c[a]) for a in range(3)))
        out.append(dict(coord=c, rank=r, lo=lo, n=n, top=c[2] == parts[2] - 1,
                        neighbours={f: neighbour(parts, c, f) for f in range(FACES)}))
    return out


# -------------------------------------------------------------- exchange
def exchange(part, coord, parts, which: int, transport: Callable) -> None:
    """Refresh the halos of one part's internal faces, x then y then z.

    transport(send: {face: buffer}, recv: {face: buffer}) moves, for every
    face with a neighbour, the packed buffer to that neighbour and fills
    recv[face] with what the neighbour packed on the opposite face."""
    for axis in range(3):
        faces = [f for f in (2 * axis, 2 * axis + 1) if neighbour(parts, coord, f) is not None]
        if not faces:
            transport({}, {})
            continue
        send = {f: part.new_buffer(part.halo_count(f, which)) for f in faces}
        recv = {f: part.new_buffer(part.halo_count(f, which)) for f in faces}
        for f in faces:
            part.pack(f, which, send[f])
        transport(send, recv)
        for f in faces:
            part.unpack(f, which, recv[f])


class Part(Session):
    """One part of a decomposed run directory (cgfdm_create_part)."""

    def __init__(self, run_dir: str, parts: Sequence[int], coord: Sequence[int], options: Optional[str] = None,
                 device: int = 0, flavor: str = "fast"):
        self.L = load(flavor)
        L = self.L
        L.cgfdm_create_part.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.cgfdm_part_info.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 3
        L.cgfdm_part_station_ids.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.cgfdm_part_advance.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.cgfdm_part_launch.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.cgfdm_part_finish.argtypes = [ctypes.c_void_p]
        L.cgfdm_part_link.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.cgfdm_part_handle.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong]
        L.cgfdm_part_link_handle.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.cgfdm_halo_count.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.cgfdm_halo_count.restype = ctypes.c_longlong
        L.cgfdm_halo_pack.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.cgfdm_halo_unpack.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        self._h = ctypes.c_void_p()
        P, C = (ctypes.c_int * 3)(*parts), (ctypes.c_int * 3)(*coord)
        rc = L.cgfdm_create_part(run_dir.encode(), options.encode() if options else None, P, C, device,
                                 ctypes.byref(self._h))
        if rc:
            raise CgfdmError(rc, L.cgfdm_last_error(None).decode())
        self.run_dir, self.parts, self.coord, self.device = run_dir, tuple(parts), tuple(coord), device
        lo, n, top = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), ctypes.c_int()
        self._check(L.cgfdm_part_info(self._h, lo, n, ctypes.byref(top)))
        self.lo, self.n, self.top = tuple(lo), tuple(n), bool(top.value)
        nst = self.info.n_stations
        ids = (ctypes.c_int * max(nst, 1))()
        self._check(L.cgfdm_part_station_ids(self._h, ids, nst))
        self.station_ids = list(ids)[:nst]

    def advance(self) -> int:
        ph = ctypes.c_int()
        self._check(self.L.cgfdm_part_advance(self._h, ctypes.byref(ph)))
        return ph.value

    def launch(self) -> int:
        """Enqueue the next phase (finish() waits for it)."""
        ph = ctypes.c_int()
        self._check(self.L.cgfdm_part_launch(self._h, ctypes.byref(ph)))
        return ph.value

    def finish(self) -> None:
        self._check(self.L.cgfdm_part_finish(self._h))

    def link(self, face: int, nbr: "Part") -> None:
        """Stages store the layers next to `face` into nbr's halo directly."""
        self._check(self.L.cgfdm_part_link(self._h, face, nbr._h))

    HANDLE_BYTES = 512

    def handle(self) -> bytes:
        """This part's stage buffers for a neighbour in another process."""
        buf = ctypes.create_string_buffer(self.HANDLE_BYTES)
        self._check(self.L.cgfdm_part_handle(self._h, buf, self.HANDLE_BYTES))
        return buf.raw

    def link_handle(self, face: int, handle: bytes) -> None:
        buf = ctypes.create_string_buffer(handle, len(handle))
        self._check(self.L.cgfdm_part_link_handle(self._h, face, buf, len(handle)))

    def halo_count(self, face: int, which: int) -> int:
        return int(self.L.cgfdm_halo_count(self._h, face, which))

    def new_buffer(self, n: int):
        import torch
        return torch.empty(n, dtype=torch.float32, device=f"cuda:{self.device}")

    def pack(self, face: int, which: int, buf) -> None:
        self._check(self.L.cgfdm_halo_pack(self._h, face, which, buf.data_ptr()))

    def unpack(self, face: int, which: int, buf) -> None:
        self._check(self.L.cgfdm_halo_unpack(self._h, face, which, buf.data_ptr()))


def _exchange_all_local(ps: Dict, parts, which: int) -> None:
    """Halo exchange among parts of one process: per axis, every part packs,
    then every part unpacks its neighbours' buffers (device copies)."""
    for axis in range(3):
        packed = {}
        for c, p in ps.items():
            for f in (2 * axis, 2 * axis + 1):
                if neighbour(parts, c, f) is not None:
                    b = p.new_buffer(p.halo_count(f, which))
                    p.pack(f, which, b)
                    packed[(c, f)] = b
        for c, p in ps.items():
            for f in (2 * axis, 2 * axis + 1):
                q = neighbour(parts, c, f)
                if q is not None:
                    p.unpack(f, which, packed[(q, f ^ 1)])


def _assemble(ps: Dict, shape, nst_total: int, NT: int):
    nx, ny, nz = shape
    W = np.zeros((nz, ny, nx, 9), np.float32)
    st = np.zeros((nst_total, NT, 9), np.float32)
    pgv = np.zeros((ny, nx, 2), np.float32)
    for p in ps.values():
        (x0, y0, z0), (lx, ly, lz) = p.lo, p.n
        W[z0:z0 + lz, y0:y0 + ly, x0:x0 + lx] = p.wavefield()[3:-3, 3:-3, 3:-3]
        if p.station_ids:
            st[p.station_ids] = p.stations()
        if p.top:
            pgv[y0:y0 + ly, x0:x0 + lx] = p.pgv()[..., :2]
    return W, st, pgv


class LocalDomain:
    """Every part of a decomposition in this process on one GPU, halos moved
    by device copies (or, fused, stored by the stage kernels)."""

    def __init__(self, run_dir: str, parts: Sequence[int], options: Optional[str] = None, device: int = 0,
                 flavor: str = "fast", fused: bool = False):
        self.parts, self.fused = tuple(parts), fused
        self.ps: Dict = {}
        try:
            for r in range(parts[0] * parts[1] * parts[2]):
                c = coord_of(self.parts, r)
                self.ps[c] = Part(run_dir, self.parts, c, options, device, flavor)
            _exchange_all_local(self.ps, self.parts, 1)      # metric and medium halos
            if fused:
                for c, p in self.ps.items():
                    for f in range(FACES):
                        q = neighbour(self.parts, c, f)
                        if q is not None:
                            p.link(f, self.ps[q])
        except Exception:
            self.close()
            raise
        any_part = next(iter(self.ps.values()))
        self.NT = any_part.info.NT
        self.it = 0
        self.shape = tuple(max(p.lo[a] + p.n[a] for p in self.ps.values()) for a in range(3))

    def step(self, n: int) -> None:
        n = min(n, self.NT - self.it)
        for _ in range(n):
            for phase in range(5):
                for p in self.ps.values():        # the parts' kernels run concurrently
                    assert p.launch() == phase
                for p in self.ps.values():
                    p.finish()
                if phase == 0 or (phase < 4 and not self.fused):
                    _exchange_all_local(self.ps, self.parts, 0)
        self.it += n

    def outputs(self):
        """Interior wavefield, station traces in the run's order, PGV."""
        nst_total = 1 + max([max(p.station_ids) for p in self.ps.values() if p.station_ids], default=-1)
        return _assemble(self.ps, self.shape, nst_total, self.NT)

    def write_outputs(self) -> None:
        for p in self.ps.values():
            p.write_outputs()

    def close(self) -> None:
        for p in self.ps.values():
            p.close()
        self.ps = {}


def run_local(run_dir: str, parts: Sequence[int], nsteps: Optional[int] = None, options: Optional[str] = None,
              device: int = 0, flavor: str = "fast", fused: bool = False, write_outputs: bool = False):
    """Every part on one GPU; returns the interior wavefield [nz][ny][nx][9],
    the station traces [n][NT][9] in the run's station order and the PGV
    [ny][nx][2], assembled from the parts.  fused: the stages store their
    boundary layers into the neighbours' halos (cgfdm_part_link), leaving
    one explicit exchange per step, after the source.  write_outputs: every
    part writes its station and PGV files under its rank coordinates, as
    the reference's ranks do."""
    dom = LocalDomain(run_dir, parts, options, device, flavor, fused)
    try:
        dom.step(dom.NT if nsteps is None else nsteps)
        if write_outputs:
            dom.write_outputs()
        return dom.outputs()
    finally:
        dom.close()


def torch_transport(group, parts, coord):
    """transport() over torch.distributed point-to-point: every face's buffer
    to the neighbour's rank, the neighbour's opposite face into recv."""
    import torch.distributed as dist

    def move(send, recv):
        ops = []
        for f, b in send.items():
            ops.append(dist.P2POp(dist.isend, b, rank_of(parts, neighbour(parts, coord, f)), group))
        for f, b in recv.items():
            ops.append(dist.P2POp(dist.irecv, b, rank_of(parts, neighbour(parts, coord, f)), group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
    return move


def link_neighbours(part, coord, parts, group=None) -> None:
    """Every rank publishes its part's handle; each part links the handles
    of its face neighbours (the stages then write their halos directly)."""
    import torch.distributed as dist

    handles = [None] * dist.get_world_size(group)
    dist.all_gather_object(handles, part.handle(), group=group)
    for f in range(FACES):
        q = neighbour(parts, coord, f)
        if q is not None:
            part.link_handle(f, handles[rank_of(parts, q)])


def step_distributed(part, coord, parts, nsteps: int, move, barrier, fused: bool, sync=lambda: None) -> None:
    """nsteps steps of one part: the five phases, after each either the
    exchange (phase 0 always; 1..3 unless fused) or, when fused, a barrier
    so that no part starts a phase before its neighbours' stores landed."""
    for _ in range(nsteps):
        for phase in range(5):
            part.advance()
            sync()
            if phase == 0 or (phase < 4 and not fused):
                exchange(part, coord, parts, 0, move)
            elif fused:
                barrier()


def run_distributed(run_dir: str, parts: Sequence[int], nsteps: Optional[int] = None,
                    options: Optional[str] = None, group=None, fused: bool = False):
    """One part per rank (rank r holds coord_of(parts, r), on cuda:LOCAL_RANK);
    returns this part's session after the steps, for its outputs.  fused:
    neighbours' buffers are linked through CUDA IPC and the stage kernels
    store into them over NVLink."""
    import os

    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    coord = coord_of(parts, rank)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    p = Part(run_dir, parts, coord, options, dev)
    move = torch_transport(group, parts, coord)
    exchange(p, coord, parts, 1, move)
    if fused:
        link_neighbours(p, coord, parts, group)
    NT = p.info.NT
    step_distributed(p, coord, parts, NT if nsteps is None else min(nsteps, NT), move,
                     lambda: dist.barrier(group), fused, lambda: torch.cuda.synchronize(dev))
    return p
