"""The z-slab domain decomposition (md-bench_b200/domain.py) on CPU.

Two ranks over gloo run the decomposition's host logic (slab ownership,
migration at rebuild, halo selection and shifts, the two-phase neighbour
exchange, thermo sums) with a small NumPy engine: Verlet lists built at every
rebuild, each atom's pair forces summed in a canonical order (by neighbour
global id, then image position). Halo positions are made exactly as ghost
images are (one FP64 addition of the box length per coordinate), so a 2-slab
run and an undivided run of the same engine give bit-identical forces,
positions and velocities, across a rebuild with atoms changing slabs.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

CELLS = 6
STEPS = 26        # one rebuild (step 19) with migration, then 6 more steps
EVERY = 20


def _np(a):
    return a.numpy() if hasattr(a, "numpy") else np.asarray(a)


class NumpyLJ:
    """LJ full lists (epsilon = sigma = 1) and the velocity Verlet of
    verletlist/integrate.c:21-42 on NumPy; periodic in x, y and, without
    halo atoms, z."""

    def __init__(self, box, cutforce, cutneigh, dt, dtforce, periodic_z):
        self.box = np.asarray(box, dtype=np.float64)
        self.rc2, self.rl2 = cutforce ** 2, cutneigh ** 2
        self.dt, self.dtf = dt, dtforce
        zs = (-1, 0, 1) if periodic_z else (0,)
        self.shifts = np.array([(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in zs],
                               dtype=np.float64) * self.box

    def load(self, x, v, t, hx, ht, ids):
        # the driver hands over torch tensors on the host (NumPy arrays here)
        x, v, t, hx = (_np(a) for a in (x, v, t, hx))
        self.x, self.v = np.array(x, dtype=np.float64), np.array(v, dtype=np.float64)
        self.t = np.asarray(t)
        self.hx = np.array(hx, dtype=np.float64).reshape(-1, 3)
        self.gall = np.concatenate([_np(ids[0]), _np(ids[1])]).astype(np.int64)
        self.n = len(self.x)
        self._build()
        self.force()

    def _images(self):
        allx = np.concatenate([self.x, self.hx])
        # one addition per coordinate, as a ghost image is made
        return allx[None, :, :] + self.shifts[:, None, :]

    def _build(self):
        img = self._images()                             # (S, A, 3)
        S, A = img.shape[:2]
        pi, pj, ps = [], [], []
        for i in range(self.n):
            d = self.x[i][None, None, :] - img
            r2 = np.sum(d * d, axis=2)
            s, j = np.nonzero(r2 < self.rl2)
            keep = ~((j == i) & np.all(self.shifts[s] == 0.0, axis=1))
            s, j = s[keep], j[keep]
            p = img[s, j]
            # canonical order: neighbour global id, then its image position
            order = np.lexsort((p[:, 2], p[:, 1], p[:, 0], self.gall[j]))
            pi.append(np.full(len(j), i))
            pj.append(j[order])
            ps.append(s[order])
        self.pi, self.pj, self.ps = np.concatenate(pi), np.concatenate(pj), np.concatenate(ps)
        self.starts = np.searchsorted(self.pi, np.arange(self.n))

    def force(self):
        img = self._images()
        d = self.x[self.pi] - img[self.ps, self.pj]
        r2 = np.sum(d * d, axis=1)
        sr2 = np.where(r2 < self.rc2, 1.0 / r2, 0.0)
        sr6 = sr2 * sr2 * sr2
        fpair = 48.0 * sr6 * (sr6 - 0.5) * sr2
        self.f = np.zeros((self.n, 3))
        for i in range(self.n):
            a, b = self.starts[i], self.starts[i + 1] if i + 1 < self.n else len(self.pi)
            self.f[i] = np.sum(d[a:b] * fpair[a:b, None], axis=0)

    def positions(self, idx, sz):
        p = self.x[np.asarray(idx)].copy()
        p[:, 2] += sz
        return torch.from_numpy(p)

    def set_halo_positions(self, recv):
        self.hx = np.concatenate([_np(r).astype(np.float64).reshape(-1, 3) for r in recv])

    def initial_integrate(self):
        self.v += self.dtf * self.f
        self.x += self.dt * self.v

    def final_integrate(self):
        self.v += self.dtf * self.f

    def owned_state(self):
        return self.x.copy(), self.v.copy(), self.t.copy()

    def owned_forces(self):
        return self.f.copy()

    def kinetic(self):
        return float(np.sum(self.v * self.v))


def initial_state():
    sys.path[:0] = [os.path.join(ROOT, "md-bench_b200")]
    import mdb
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS)
    x, v, t = mdb.create_fcc(hp)
    return hp, x, v, t


def undivided(hp, x, v, t):
    """The same engine on the whole periodic box, the reference's loop."""
    sys.path[:0] = [os.path.join(ROOT, "md-bench_b200")]
    import domain as D
    box = (hp.xprd, hp.yprd, hp.zprd)
    e = NumpyLJ(box, hp.cutforce, hp.cutneigh, hp.dt, hp.dtforce, periodic_z=True)
    sl = D.Slabs(box, hp.cutneigh, 1, 0)
    gid = np.arange(len(t))
    e.load(sl.wrap(x), v, t, np.zeros((0, 3)), np.zeros(0, np.int32), (gid, gid[:0]))
    f0 = e.f.copy()
    for n in range(STEPS):
        e.initial_integrate()
        if (n + 1) % EVERY == 0:
            e.load(sl.wrap(e.x), e.v, e.t, np.zeros((0, 3)), np.zeros(0, np.int32),
                   (gid, gid[:0]))
        else:
            e.force()
        e.final_integrate()
    return f0, e.x, e.v, e.f


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "md-bench_b200"), os.path.join(ROOT, "tests")]
    import datetime

    import domain as D
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        hp, x, v, t = initial_state()
        box = (hp.xprd, hp.yprd, hp.zprd)
        sl = D.Slabs(box, hp.cutneigh, world, rank)
        eng = NumpyLJ(box, hp.cutforce, hp.cutneigh, hp.dt, hp.dtforce, periodic_z=False)
        run = D.SlabRun(sl, D.DistTransport(torch, dist, "cpu"), eng, EVERY)
        run.start(x, v, t, np.arange(len(t)))
        g0, _, _, f0 = run.gather()
        n0 = len(g0)
        run.run(STEPS)
        g, xs, vs, fs = run.gather()
        T = run.temperature(len(t))
        q.put((rank, g0, f0, g, xs, vs, fs, T, n0, len(g)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_slabs_bit_identical_to_one_domain():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    hp, x, v, t = initial_state()
    n = len(t)
    F0, X, V, F = undivided(hp, x, v, t)
    got0, gotf, gotx, gotv, owned = (np.full((n, 3), np.nan) for _ in range(5))
    T = None
    counts = []
    for rank, g0, f0, g, xs, vs, fs, Tr, n0, n1 in res:
        got0[g0] = f0
        gotx[g], gotv[g], gotf[g] = xs, vs, fs
        T = Tr
        counts.append((n0, n1))
    # every atom owned by exactly one rank, before and after the migration,
    # and the rebuild moved some atoms to the other slab
    assert sum(c[0] for c in counts) == n and sum(c[1] for c in counts) == n
    moved = sum(len(set(r[1].tolist()) ^ set(r[3].tolist())) for r in res)
    assert moved > 0
    assert np.array_equal(got0, F0)
    # positions are wrapped at the rebuild on both sides
    assert np.array_equal(gotx, X) and np.array_equal(gotv, V) and np.array_equal(gotf, F)
    assert T == pytest.approx(float(np.sum(V * V)) / (3 * n - 3), rel=1e-14)


def _empty_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [os.path.join(ROOT, "md-bench_b200")]
    import datetime

    import domain as D
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        tr = D.DistTransport(torch, dist, "cpu")
        other = 1 - rank
        # rank 0 sends nothing down and three rows up; rank 1 the reverse
        down = np.zeros((0, 3)) if rank == 0 else np.arange(9.0).reshape(3, 3) + 100 * rank
        up = np.arange(9.0).reshape(3, 3) + 100 * rank if rank == 0 else np.zeros((0, 3))
        fb, fa = tr.exchange(tr.wrap(down), tr.wrap(up), other, other)
        q.put((rank, tr.to_host(fb).tolist(), tr.to_host(fa).tolist()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_exchange_with_empty_messages():
    """Empty halves of an exchange (no atom leaving in one direction) travel
    as padding and arrive as zero rows."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_empty_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r, (fb, fa)) for r, fb, fa in [q.get(timeout=90) for _ in range(2)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rows = np.arange(9.0).reshape(3, 3)
    # rank 0: from below (rank 1's up) nothing; from above (rank 1's down) 3 rows
    assert res[0][0] == [] and res[0][1] == (rows + 100).tolist()
    # rank 1: from below (rank 0's up) 3 rows; from above (rank 0's down) nothing
    assert res[1][0] == rows.tolist() and res[1][1] == []


def test_one_slab_is_its_own_neighbour():
    """One rank: the halo is the slab's own z images (shifted by the box
    length both ways), exchanged with itself through host queues; atoms never
    leave. Bit-identical to the undivided periodic run, across two rebuilds."""
    sys.path[:0] = [os.path.join(ROOT, "md-bench_b200")]
    import domain as D
    hp, x, v, t = initial_state()
    box = (hp.xprd, hp.yprd, hp.zprd)
    eng = NumpyLJ(box, hp.cutforce, hp.cutneigh, hp.dt, hp.dtforce, periodic_z=False)
    run = D.SlabRun(D.Slabs(box, hp.cutneigh, 1, 0),
                    D.ThreadTransport(D.ThreadTransport.Hub(1), 0), eng, EVERY)
    run.start(x, v, t, np.arange(len(t)))
    run.run(STEPS + EVERY)
    g, xs, vs, fs = run.gather()
    assert len(g) == len(t) and np.array_equal(np.sort(g), np.arange(len(t)))
    ref = NumpyLJ(box, hp.cutforce, hp.cutneigh, hp.dt, hp.dtforce, periodic_z=True)
    sl = D.Slabs(box, hp.cutneigh, 1, 0)
    gid = np.arange(len(t))
    ref.load(sl.wrap(x), v, t, np.zeros((0, 3)), np.zeros(0, np.int32), (gid, gid[:0]))
    for n in range(STEPS + EVERY):
        ref.initial_integrate()
        if (n + 1) % EVERY == 0:
            ref.load(sl.wrap(ref.x), ref.v, ref.t, np.zeros((0, 3)), np.zeros(0, np.int32),
                     (gid, gid[:0]))
        else:
            ref.force()
        ref.final_integrate()
    order = np.argsort(g)
    assert np.array_equal(xs[order], ref.x) and np.array_equal(vs[order], ref.v)
    assert np.array_equal(fs[order], ref.f)


def test_slab_geometry_and_halo_plan():
    sys.path[:0] = [os.path.join(ROOT, "md-bench_b200")]
    import domain as D
    box = (10.0, 10.0, 12.0)
    s0, s1, s2 = (D.Slabs(box, 2.8, 3, r) for r in range(3))
    assert (s0.zlo, s0.zhi, s2.zlo, s2.zhi) == (0.0, 4.0, 8.0, 12.0)
    assert list(s0.owner(np.array([0.0, 3.999, 4.0, 11.999]))) == [0, 0, 1, 2]
    x = np.array([[1.0, 1.0, 0.5], [1.0, 1.0, 2.0], [1.0, 1.0, 3.5]])
    (pb, down, sd), (pa, up, su) = s0.halo_plan(x)
    assert (pb, pa) == (2, 1) and sd == 12.0 and su == 0.0
    assert list(down) == [0, 1] and list(up) == [1, 2]
    (pb, down, sd), (pa, up, su) = s2.halo_plan(x + [0, 0, 8.0])
    assert (pb, pa) == (1, 0) and sd == 0.0 and su == -12.0
    w = s0.wrap(np.array([[-0.5, 10.0, 12.5]]))
    assert np.array_equal(w, [[9.5, 0.0, 0.5]])
    with pytest.raises(ValueError):
        D.Slabs(box, 5.0, 3, 0)
