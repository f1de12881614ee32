"""Domain decomposition (cgfdm_create_part, cgfdm.domain): a grid split into
parts, one session each, the halos at internal faces refreshed after every
phase of a step, as the reference's MPI ranks exchange them
(src/MPI_send_recv_FLOAT.cpp).

GPU: every part on one device (halos moved by device copies) must reproduce
the single-domain run bit for bit -- interior wavefield, station traces in
the run's order, surface PGV -- for several decompositions of a curvilinear
grid with PML on five faces, the free surface and a finite fault whose cells
fall in several parts.

CPU: the decomposition's arithmetic, and the exchange orchestration between
two gloo ranks with array-backed parts: each rank's halos must equal its
neighbour's interior layers afterwards."""

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import parity_util as pu
from cgfdm import Session, cases, domain


def test_plan_covers_grid_once():
    shape, parts = (34, 30, 26), (3, 2, 2)
    cover = np.zeros(shape[::-1], int)
    P = domain.plan(shape, parts)
    assert len(P) == 12 and sum(p["top"] for p in P) == 6
    for p in P:
        (x, y, z), (nx, ny, nz) = p["lo"], p["n"]
        cover[z:z + nz, y:y + ny, x:x + nx] += 1
        assert domain.rank_of(parts, p["coord"]) == p["rank"]
        for f, q in p["neighbours"].items():
            if q is not None:
                assert domain.neighbour(parts, q, f ^ 1) == p["coord"]
    assert (cover == 1).all()
    assert [domain.extent(10, 3, c) for c in range(3)] == [(0, 4), (4, 3), (7, 3)]


class ArrayPart:
    """A part backed by a padded numpy array [nz+6][ny+6][nx+6][nf] whose
    interior holds the global index of each point; pack/unpack as the
    library's kernels do (three layers next to / beyond the face, the other
    axes over their padded extent)."""

    def __init__(self, shape, parts, coord, nf=2):
        lo, n = zip(*(domain.extent(shape[a], parts[a], coord[a]) for a in range(3)))
        self.lo, self.n, self.nf = lo, n, nf
        self.a = np.full((n[2] + 6, n[1] + 6, n[0] + 6, nf), -1.0, np.float32)
        z, y, x = np.meshgrid(*(np.arange(lo[a], lo[a] + n[a]) for a in (2, 1, 0)), indexing="ij")
        g = (z * shape[1] + y) * shape[0] + x
        for f in range(nf):
            self.a[3:-3, 3:-3, 3:-3, f] = g + 1000000 * f

    def _box(self, face, send):
        axis, hi = divmod(face, 2)
        n = self.n[axis]
        start = (n if hi else 3) if send else (n + 3 if hi else 0)
        sl = [slice(None)] * 3
        sl[2 - axis] = slice(start, start + 3)   # array axes are z, y, x
        return tuple(sl)

    def halo_count(self, face, which):
        return int(self.a[self._box(face, True)].size)

    def new_buffer(self, n):
        return torch.zeros(n, dtype=torch.float32)

    def pack(self, face, which, buf):
        buf.copy_(torch.from_numpy(np.ascontiguousarray(self.a[self._box(face, True)]).reshape(-1)))

    def unpack(self, face, which, buf):
        box = self._box(face, False)
        self.a[box] = buf.numpy().reshape(self.a[box].shape)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, shape, parts, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        coord = domain.coord_of(parts, rank)
        p = ArrayPart(shape, parts, coord)
        domain.exchange(p, coord, parts, 0, domain.torch_transport(None, parts, coord))
        np.save(os.path.join(out, f"part{rank}.npy"), p.a)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("parts", [(2, 1, 1), (1, 1, 2)])
def test_exchange_between_gloo_ranks(tmp_path, parts):
    shape = (14, 9, 12)
    world = parts[0] * parts[1] * parts[2]
    mp.spawn(_worker, args=(world, _free_port(), shape, parts, str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        c = domain.coord_of(parts, r)
        a = np.load(tmp_path / f"part{r}.npy")
        ref = ArrayPart(shape, parts, c)
        # every halo layer on an internal face now holds the neighbour's points
        for f in range(6):
            if domain.neighbour(parts, c, f) is None:
                continue
            axis, hi = divmod(f, 2)
            lo, n = ref.lo[axis], ref.n[axis]
            idx = np.arange(lo + n, lo + n + 3) if hi else np.arange(lo - 3, lo)
            box = ref._box(f, False)
            sub = [slice(3, -3)] * 3
            sub[2 - axis] = slice(None)
            got = a[box][tuple(sub)][..., 0]
            zz, yy, xx = [np.arange(ref.lo[b], ref.lo[b] + ref.n[b]) for b in (2, 1, 0)]
            axes = [zz, yy, xx]
            axes[2 - axis] = idx
            Z, Y, X = np.meshgrid(*axes, indexing="ij")
            np.testing.assert_array_equal(got, (Z * shape[1] + Y) * shape[0] + X)


class LinkPart(ArrayPart):
    """An array-backed part that records its links, phases and exchanges."""

    def __init__(self, shape, parts, coord, rank):
        super().__init__(shape, parts, coord)
        self.rank, self.links, self.phases, self.packs = rank, {}, 0, 0

    def handle(self):
        return f"part-of-rank-{self.rank}".encode().ljust(32, b"\0")

    def link_handle(self, face, handle):
        self.links[face] = handle.rstrip(b"\0").decode()

    def advance(self):
        self.phases += 1

    def pack(self, face, which, buf):
        self.packs += 1
        super().pack(face, which, buf)


def _link_worker(rank, world, port, shape, parts, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        coord = domain.coord_of(parts, rank)
        p = LinkPart(shape, parts, coord, rank)
        domain.link_neighbours(p, coord, parts)
        barriers = []
        domain.step_distributed(p, coord, parts, 3, domain.torch_transport(None, parts, coord),
                                lambda: (barriers.append(1), dist.barrier()), True)
        np.save(os.path.join(out, f"r{rank}.npy"),
                np.array([p.phases, p.packs, len(barriers)] + sorted(p.links)))
        with open(os.path.join(out, f"r{rank}.txt"), "w") as f:
            f.write(",".join(p.links[k] for k in sorted(p.links)))
    finally:
        dist.destroy_process_group()


def test_fused_orchestration_between_gloo_ranks(tmp_path):
    """Handles reach the face neighbours; with the stores fused, a step is
    five phases, one exchange (after the source) and four barriers."""
    shape, parts = (14, 9, 12), (3, 1, 1)
    mp.spawn(_link_worker, args=(3, _free_port(), shape, parts, str(tmp_path)), nprocs=3, join=True)
    expect_links = {0: [1], 1: [0, 1], 2: [0]}
    for r in range(3):
        v = np.load(tmp_path / f"r{r}.npy")
        nfaces = len(expect_links[r])
        assert v[0] == 15 and v[1] == 3 * nfaces and v[2] == 12
        assert list(v[3:]) == expect_links[r]
        names = open(tmp_path / f"r{r}.txt").read().split(",")
        nb = [domain.rank_of(parts, domain.neighbour(parts, domain.coord_of(parts, r), f)) for f in expect_links[r]]
        assert names == [f"part-of-rank-{q}" for q in nb]


def _case():
    c = pu.multi_fault(steps=24, courant=0.45)
    c.gauss_hill = 1
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("parts,fused", [((2, 1, 2), False), ((1, 2, 1), False), ((2, 2, 2), False),
                                         ((2, 1, 2), True), ((2, 2, 2), True), ((3, 1, 1), True)])
def test_decomposed_run_matches_single_domain(tmp_path, parts, fused):
    """fused: the stage kernels store their boundary layers into the
    neighbours' halos (cgfdm_part_link); only the exchange after the source
    stays explicit."""
    c = _case()
    d = cases.write_case(c, str(tmp_path / "run"))
    with Session(d) as s:
        s.run(s.info.NT)
        ref = (s.wavefield()[3:-3, 3:-3, 3:-3], s.stations(), s.pgv()[..., :2])
        assert s.info.n_fault_cells > 1
    got = domain.run_local(d, parts, fused=fused)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    assert np.abs(got[0]).max() > 0


def _staged_transport(parts, coord):
    """send/recv of device buffers through host memory (gloo moves CPU
    tensors only)."""
    def move(send, recv):
        cs = {f: b.cpu() for f, b in send.items()}
        cr = {f: torch.empty(b.numel()) for f, b in recv.items()}
        peer = lambda f: domain.rank_of(parts, domain.neighbour(parts, coord, f))
        ops = [dist.P2POp(dist.isend, cs[f], peer(f)) for f in cs] + [dist.P2POp(dist.irecv, cr[f], peer(f)) for f in cr]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for f, b in recv.items():
            b.copy_(cr[f])
    return move


def _ipc_worker(rank, world, port, run_dir, parts, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        coord = domain.coord_of(parts, rank)
        p = domain.Part(run_dir, parts, coord, device=0)
        move = _staged_transport(parts, coord)
        domain.exchange(p, coord, parts, 1, move)
        domain.link_neighbours(p, coord, parts)
        domain.step_distributed(p, coord, parts, p.info.NT, move, dist.barrier, True, torch.cuda.synchronize)
        np.savez(os.path.join(out, f"part{rank}.npz"), W=p.wavefield()[3:-3, 3:-3, 3:-3], st=p.stations(),
                 pgv=p.pgv()[..., :2], lo=p.lo, n=p.n, ids=np.array(p.station_ids, int), top=p.top)
        dist.barrier()   # no part unmaps its buffers while a neighbour may still use them
        p.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_fused_parts_in_two_processes_match_single_domain(tmp_path):
    """Two processes, one part each, on one GPU: the neighbours' stage
    buffers linked through CUDA IPC handles, the stage kernels storing their
    boundary layers into the other process's memory, host barriers between
    phases (no kernel waits on another).  Bit-identical to one session."""
    c = _case()
    d = cases.write_case(c, str(tmp_path / "run"))
    parts = (2, 1, 1)
    mp.spawn(_ipc_worker, args=(2, _free_port(), d, parts, str(tmp_path)), nprocs=2, join=True)
    with Session(d) as s:
        s.run(s.info.NT)
        ref = (s.wavefield()[3:-3, 3:-3, 3:-3], s.stations(), s.pgv()[..., :2])
    W = np.zeros_like(ref[0])
    st = np.zeros_like(ref[1])
    pgv = np.zeros_like(ref[2])
    for r in range(2):
        z = np.load(tmp_path / f"part{r}.npz")
        (x0, y0, z0), (lx, ly, lz) = z["lo"], z["n"]
        W[z0:z0 + lz, y0:y0 + ly, x0:x0 + lx] = z["W"]
        if len(z["ids"]):
            st[z["ids"]] = z["st"]
        if z["top"]:
            pgv[y0:y0 + ly, x0:x0 + lx] = z["pgv"]
    for a, b in zip((W, st, pgv), ref):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_parts_write_per_rank_files(tmp_path):
    """Each part writes station_mpi_X_Y_Z.bin (its stations' global indices
    and traces) and, in the top parts, PGV_Z_mpi_X_Y_Z.bin; together they
    hold exactly the single-domain run's files."""
    c = _case()
    d = cases.write_case(c, str(tmp_path / "run"))
    with Session(d) as s:
        s.run(s.info.NT)
        s.write_outputs()
        NT, NX, NY = s.info.NT, s.info.nx, s.info.ny
    out = os.path.join(d, "output")
    ref_st = np.fromfile(os.path.join(out, "station_mpi_0_0_0.bin"), np.uint8)
    ref_pgv = np.fromfile(os.path.join(out, "PGV_Z_mpi_0_0_0.bin"), np.float32).reshape(NY, NX, 2)
    os.remove(os.path.join(out, "station_mpi_0_0_0.bin"))
    os.remove(os.path.join(out, "PGV_Z_mpi_0_0_0.bin"))
    parts = (2, 1, 2)
    domain.run_local(d, parts, write_outputs=True)
    rows = {}
    pgv = np.zeros_like(ref_pgv)
    for p in domain.plan((NX, NY, c.NZ), parts):
        tag = "_mpi_%d_%d_%d.bin" % p["coord"]
        f = os.path.join(out, "station" + tag)
        if os.path.exists(f):
            raw = np.fromfile(f, np.uint8)
            n = raw.size // (12 + NT * 36)
            xyz = np.frombuffer(raw[: n * 12].tobytes(), np.int32).reshape(n, 3)
            tr = np.frombuffer(raw[n * 12:].tobytes(), np.float32).reshape(n, NT, 9)
            for a, b in zip(xyz, tr):
                rows[tuple(a)] = b
        g = os.path.join(out, "PGV_Z" + tag)
        assert os.path.exists(g) == p["top"]
        if p["top"]:
            (x0, y0, _), (lx, ly, _) = p["lo"], p["n"]
            pgv[y0:y0 + ly, x0:x0 + lx] = np.fromfile(g, np.float32).reshape(ly, lx, 2)
    n = ref_st.size // (12 + NT * 36)
    xyz = np.frombuffer(ref_st[: n * 12].tobytes(), np.int32).reshape(n, 3)
    tr = np.frombuffer(ref_st[n * 12:].tobytes(), np.float32).reshape(n, NT, 9)
    assert len(rows) == n
    for a, b in zip(xyz, tr):
        np.testing.assert_array_equal(rows[tuple(a)], b)
    np.testing.assert_array_equal(pgv, ref_pgv)


@pytest.mark.gpu
def test_part_refuses_plain_run(tmp_path):
    from cgfdm import CgfdmError

    d = cases.write_case(_case(), str(tmp_path / "run"))
    p = domain.Part(d, (2, 1, 1), (0, 0, 0))
    try:
        with pytest.raises(CgfdmError):
            p.run(1)
    finally:
        p.close()
