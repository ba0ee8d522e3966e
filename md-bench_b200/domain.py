"""z-slab domain decomposition of the Verlet-list timestep over ranks.

The reference runs one MPI rank per subdomain and moves atoms between them
with a 6-swap halo (common/comm.c:233-631, driven by forward() and
updateAtoms()/reneighbour() in verletlist/main.c:150-161, 115-135 and
common/shell_methods.h:28-54). Here the box is cut into slabs along z, one per
rank (one GPU each), periodic in x and y inside every rank. Per rebuild
period:

* at a rebuild step each rank wraps its atoms into the box, sends the atoms
  that left its slab to the rank that now owns them (atoms move less than
  the skin in a period, but any rank is reachable), and sends every owned
  atom within cutneigh of a slab face to the neighbouring rank across it,
  shifted by the box length where that face is the box boundary; the rank
  then holds its owned atoms followed by that halo (``mdb_set_owned``) and
  builds its ghosts (x, y images) and lists;
* at every other step the same halo atoms' positions are sent again, after
  the initial integration and before the force (``mdb_gather_positions`` /
  ``mdb_set_halo_positions``).

The halo covers both z faces, as the reference's fullShell method, whose
reverse() moves nothing (common/shell_methods.h:59-88): each rank computes the
forces of its own atoms from owned and halo neighbours. With half lists a
halo atom is listed like a ghost and gets no reaction, so a pair across a slab
face is computed on both ranks, each for its own atom; there is no reverse
exchange of forces. Thermo sums are reduced over ranks.

The exchange goes through a ``Transport``: ``DistTransport`` uses
torch.distributed point-to-point calls (NCCL with device tensors between
GPUs, gloo with host tensors on CPU); the driver itself (``SlabRun``) is the
same for any engine with the small interface of ``MdbEngine``.
"""
import numpy as np


def _is_tensor(a):
    return type(a).__module__.startswith("torch")


class Slabs:
    """Slab geometry: rank r owns z in [r * Lz / P, (r + 1) * Lz / P)."""

    def __init__(self, box, cutneigh, world, rank):
        self.box = np.asarray(box, dtype=np.float64)
        self.cut = float(cutneigh)
        self.world, self.rank = int(world), int(rank)
        self.lz = self.box[2] / self.world
        if self.world > 1 and self.lz < self.cut:
            raise ValueError("slabs thinner than the neighbour cutoff")
        self.zlo = self.rank * self.lz
        self.zhi = self.box[2] if self.rank == self.world - 1 else (self.rank + 1) * self.lz

    # NumPy arrays or torch tensors (on the host or a GPU): the same FP64
    # operations either way

    def owner(self, z):
        """The rank owning each z (wrapped positions)."""
        if _is_tensor(z):
            import torch
            return torch.clamp(torch.floor(z / self.lz).long(), 0, self.world - 1)
        r = np.floor(np.asarray(z) / self.lz).astype(np.int64)
        return np.clip(r, 0, self.world - 1)

    def wrap(self, x):
        """updateAtomsPbcCPU (verletlist/pbc.c:62-87): one box length back
        into [0, L) per coordinate (both tests on the unwrapped value)."""
        if _is_tensor(x):
            import torch
            x = x.clone()
            for d in range(3):
                c = x[:, d]
                lo, hi = c < 0.0, c >= float(self.box[d])
                x[:, d] = torch.where(lo, c + float(self.box[d]),
                                      torch.where(hi, c - float(self.box[d]), c))
            return x
        x = np.array(x, dtype=np.float64, copy=True)
        for d in range(3):
            lo, hi = x[:, d] < 0.0, x[:, d] >= self.box[d]
            x[lo, d] += self.box[d]
            x[hi, d] -= self.box[d]
        return x

    def halo_plan(self, x):
        """For each direction (below, above): (peer rank, indices of owned atoms
        within cutneigh of that face, z shift into the peer's frame)."""
        z = x[:, 2]
        below = (self.rank - 1) % self.world
        above = (self.rank + 1) % self.world
        sdown = float(self.box[2]) if self.rank == 0 else 0.0
        sup = -float(self.box[2]) if self.rank == self.world - 1 else 0.0
        if _is_tensor(x):
            import torch
            down = torch.nonzero(z < self.zlo + self.cut).flatten()
            up = torch.nonzero(z >= self.zhi - self.cut).flatten()
        else:
            down = np.nonzero(z < self.zlo + self.cut)[0]
            up = np.nonzero(z >= self.zhi - self.cut)[0]
        return [(below, down, sdown), (above, up, sup)]


class DistTransport:
    """Neighbour exchange over torch.distributed point-to-point calls (NCCL
    with device tensors, gloo with host tensors). Every exchange runs in two
    phases, all ranks sending down and receiving from above, then sending up
    and receiving from below, so each phase has one message per direction
    between any two ranks and NCCL's in-order matching pairs them correctly
    even when the ranks below and above are the same (two ranks)."""

    def __init__(self, torch, dist, device):
        self.torch, self.dist, self.device = torch, dist, device

    def wrap(self, rows):
        if _is_tensor(rows):
            return rows.contiguous().to(self.device)
        return self.torch.from_numpy(np.ascontiguousarray(rows)).to(self.device)

    def to_host(self, t):
        return t.cpu().numpy()

    def _phase(self, dest, t, src, shape_rows):
        """Send t to dest, receive shape_rows rows from src. Empty messages
        travel as one padding row (dropped on arrival), so no point-to-point
        call ever moves zero elements."""
        torch, dist = self.torch, self.dist
        if t.shape[0] == 0:
            t = torch.zeros((1, t.shape[1]), dtype=t.dtype, device=self.device)
        r = torch.empty((max(shape_rows, 1), t.shape[1]), dtype=t.dtype, device=self.device)
        ops = [dist.P2POp(dist.isend, t.contiguous(), dest), dist.P2POp(dist.irecv, r, src)]
        for q in dist.batch_isend_irecv(ops):
            q.wait()
        return r[:shape_rows]

    def exchange(self, down, up, below, above, sizes=None):
        """down / up: rows for the rank below / above. Returns (rows from below,
        rows from above); sizes: their row counts when known (between rebuilds)."""
        torch = self.torch
        if sizes is None:
            n = []
            for dest, t, src in ((below, down, above), (above, up, below)):
                c = torch.tensor([[t.shape[0]]], dtype=torch.int64, device=self.device)
                n.append(int(self._phase(dest, c, src, 1).item()))
            sizes = (n[1], n[0])
        from_above = self._phase(below, down, above, sizes[1])
        from_below = self._phase(above, up, below, sizes[0])
        return from_below, from_above

    def sum(self, values):
        t = self.torch.tensor(values, dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t)
        return t.tolist()


class ThreadTransport:
    """Ranks as host threads of one process (tests, or a decomposition run on
    fewer GPUs than ranks): messages pass through queues on the host, so no
    kernel ever waits on another rank's kernel. One shared hub per run."""

    class Hub:
        def __init__(self, world):
            import queue
            import threading
            self.world = world
            self.q = {(r, k): queue.Queue() for r in range(world) for k in ("below", "above")}
            self.barrier = threading.Barrier(world)
            self.acc = [0.0]
            self.lock = threading.Lock()

    def __init__(self, hub, rank):
        self.hub, self.rank = hub, rank

    def wrap(self, rows):
        return rows

    def to_host(self, t):
        return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)

    def exchange(self, down, up, below, above, sizes=None):
        h = self.hub
        h.q[(below, "above")].put(down)
        h.q[(above, "below")].put(up)
        return h.q[(self.rank, "below")].get(timeout=120), h.q[(self.rank, "above")].get(timeout=120)

    def sum(self, values):
        h = self.hub
        h.barrier.wait(timeout=120)
        if self.rank == 0:
            h.acc = [0.0] * len(values)
        h.barrier.wait(timeout=120)
        with h.lock:
            h.acc = [a + float(v) for a, v in zip(h.acc, values)]
        h.barrier.wait(timeout=120)
        out = list(h.acc)
        h.barrier.wait(timeout=120)
        return out


class SlabRun:
    """One rank of a slab-decomposed run. ``engine`` holds this rank's atoms
    (see MdbEngine for the interface); atoms carry global ids so that results
    can be compared with an undivided run. The atom state between the engine
    and the transport stays in torch tensors on the engine's device
    (``engine.tensor_device``, the host when the engine has none): a GPU
    engine's migration, halo selection and exchange never pass through host
    memory."""

    def __init__(self, slabs, transport, engine, reneigh_every=20):
        self.sl, self.tr, self.eng = slabs, transport, engine
        self.every = int(reneigh_every)
        w, r = slabs.world, slabs.rank
        self.below, self.above = (r - 1) % w, (r + 1) % w
        self.dev = getattr(engine, "tensor_device", "cpu")

    def _t(self, a, dtype):
        import torch
        if _is_tensor(a):
            return a.to(device=self.dev, dtype=dtype)
        return torch.as_tensor(np.asarray(a), dtype=dtype, device=self.dev)

    def start(self, x, v, t, gid):
        """Every rank passes the full initial state; each keeps its slab."""
        import torch
        x = self.sl.wrap(self._t(x, torch.float64).reshape(-1, 3))
        v = self._t(v, torch.float64).reshape(-1, 3)
        t, gid = self._t(t, torch.int32), self._t(gid, torch.int64)
        mine = self.sl.owner(x[:, 2]) == self.sl.rank
        self._load(x[mine], v[mine], t[mine], gid[mine])

    def _load(self, x, v, t, gid):
        import torch
        order = torch.argsort(gid, stable=True)
        x, v, t, gid = x[order], v[order], t[order], gid[order]
        self.gid = gid
        (_, down, sdown), (_, up, sup) = self.sl.halo_plan(x)

        # halo rows: position shifted into the receiver's frame, type, global id
        def rows(idx, sz):
            return torch.stack([x[idx, 0], x[idx, 1], x[idx, 2] + sz, t[idx].double(),
                                gid[idx].double()], dim=1)
        fb, fa = self.tr.exchange(self.tr.wrap(rows(down, sdown)), self.tr.wrap(rows(up, sup)),
                                  self.below, self.above)
        halo = torch.cat([self._t(fb, torch.float64).reshape(-1, 5),
                          self._t(fa, torch.float64).reshape(-1, 5)])
        self.send = ((down, sdown), (up, sup))
        self.nhalo = (int(fb.shape[0]), int(fa.shape[0]))
        self.halo_gid = halo[:, 4].long()
        self.eng.load(x, v, t, halo[:, :3].contiguous(), halo[:, 3].int(),
                      ids=(gid, self.halo_gid))

    def _migrate(self):
        """updateAtoms + reneighbour (verletlist/main.c:115-161): wrap, hand the
        atoms that left the slab to the neighbour that owns them, then a new
        halo and new lists."""
        import torch
        x, v, t = self.eng.owned_state()
        x = self.sl.wrap(self._t(x, torch.float64))
        v, t = self._t(v, torch.float64), self._t(t, torch.int32)
        dest = self.sl.owner(x[:, 2])
        stay = dest == self.sl.rank
        # one rank is its own neighbour: nothing leaves
        go_down = (dest == self.below) & ~stay
        go_up = (dest == self.above) & (dest != self.below) & ~stay
        if not bool(torch.all(stay | go_down | go_up)):
            raise RuntimeError("an atom moved past a whole slab in one rebuild period")
        rows = torch.cat([x, v, t.double()[:, None], self.gid.double()[:, None]], dim=1)
        if self.sl.world == 1:
            got = rows
        else:
            fb, fa = self.tr.exchange(self.tr.wrap(rows[go_down]), self.tr.wrap(rows[go_up]),
                                      self.below, self.above)
            got = torch.cat([rows[stay], self._t(fb, torch.float64).reshape(-1, 8),
                             self._t(fa, torch.float64).reshape(-1, 8)])
        self._load(got[:, 0:3].contiguous(), got[:, 3:6].contiguous(), got[:, 6].int(),
                   got[:, 7].long())

    def _forward(self):
        """The halo's positions of this step (forward(),
        common/shell_methods.h:28-54)."""
        (down, sdown), (up, sup) = self.send
        fb, fa = self.tr.exchange(self.eng.positions(down, sdown), self.eng.positions(up, sup),
                                  self.below, self.above, sizes=self.nhalo)
        self.eng.set_halo_positions([fb, fa])

    def step(self, n):
        """Timestep n as verletlist/main.c:383-407 runs it."""
        self.eng.initial_integrate()
        if (n + 1) % self.every == 0:
            self._migrate()
        else:
            self._forward()
        self.eng.force()
        self.eng.final_integrate()

    def run(self, nsteps, first_step=0):
        for n in range(first_step, first_step + nsteps):
            self.step(n)

    def temperature(self, natoms):
        """T over all ranks (computeThermo, common/thermo.c:60-100, LJ units)."""
        ke = self.tr.sum([self.eng.kinetic()])[0]
        return ke / (3 * natoms - 3)

    def gather(self):
        """(gid, x, v, f) of this rank's owned atoms, as NumPy arrays."""
        def host(a):
            return a.cpu().numpy() if _is_tensor(a) else np.asarray(a)
        x, v, _ = self.eng.owned_state()
        return host(self.gid), host(x), host(v), host(self.eng.owned_forces())


class MdbEngine:
    """A rank's atoms in a libmdb Verlet-list context (FP64 or mixed, full or
    half lists): owned atoms, then the halo. The atom state moves between the
    context and torch tensors on the GPU (mdb_set_atoms / mdb_get_atoms take
    device arrays), halo positions with mdb_gather_positions /
    mdb_set_halo_positions; nothing passes through host memory."""

    tensor_device = "cuda"

    def __init__(self, torch, mdb, hp, device, precision="fp64", half_neigh=0):
        self.torch, self.mdb, self.hp = torch, mdb, hp
        self.device, self.precision, self.half_neigh = device, precision, half_neigh
        self.sys = None
        self._idx = {}  # int32 copies of the halo index tensors, per load

    def load(self, x, v, t, hx, ht, ids=None):
        torch, mdb = self.torch, self.mdb
        n, nh = int(t.shape[0]), int(ht.shape[0])
        if self.sys is None:
            # periodic in x and y only: z neighbours come as halo atoms
            self.sys = mdb.system_from_host(self.hp, n + nh, precision=self.precision,
                                            device=self.device, pbc=(1, 1, 0),
                                            half_neigh=self.half_neigh)
        xa = torch.cat([x, hx.to(x.device)]).contiguous()
        va = torch.cat([v, torch.zeros((nh, 3), dtype=v.dtype, device=v.device)]).contiguous()
        ta = torch.cat([t.int(), ht.to(t.device).int()]).contiguous()
        # xa, va, ta come from torch's stream; the context copies them on its own
        torch.cuda.current_stream().synchronize()
        self.sys.set_atoms_ptr(n + nh, xa.data_ptr(), va.data_ptr(), ta.data_ptr())
        self.sys.set_owned(n)
        self._idx = {}
        self.n, self.nh = n, nh
        self.sys.setup_pbc()
        self.sys.update_pbc()
        self.sys.build_neighbor()
        self.sys.compute_force()

    def _streams(self):
        # the context's own stream as a torch stream, and torch's current one:
        # the halo moves between them by stream order, with no host wait
        if getattr(self, "_es", None) is None or self._es_sys is not self.sys:
            self._es = self.torch.cuda.ExternalStream(self.sys.stream)
            self._es_sys = self.sys
        return self._es, self.torch.cuda.current_stream()

    def positions(self, idx, sz):
        torch = self.torch
        # the same index tensors serve every step of a rebuild period
        key = id(idx)
        if key not in self._idx:
            self._idx[key] = (idx, torch.as_tensor(idx, device="cuda").to(torch.int32)
                              .contiguous())
        d_idx = self._idx[key][1]
        out = torch.empty((int(d_idx.shape[0]), 3), dtype=torch.float64, device="cuda")
        es, cur = self._streams()
        es.wait_stream(cur)   # d_idx and out exist on torch's stream first
        self.sys.gather_positions(d_idx.data_ptr(), int(d_idx.shape[0]), (0.0, 0.0, sz),
                                  out.data_ptr())
        out.record_stream(es)
        cur.wait_stream(es)   # torch's later uses of out follow the gather
        return out

    def set_halo_positions(self, recv):
        torch = self.torch
        buf = torch.cat([r.to("cuda") for r in recv]).contiguous()
        # the received rows and buf come from torch's stream (NCCL receives
        # complete there); the context reads buf on its own stream, after it
        es, cur = self._streams()
        es.wait_stream(cur)
        self.sys.set_halo_positions(buf.data_ptr(), buf.shape[0])
        self.sys.update_pbc()
        buf.record_stream(es)  # not reused before the context has read it

    def initial_integrate(self):
        self.sys.initial_integrate()

    def force(self):
        self.sys.compute_force()

    def final_integrate(self):
        self.sys.final_integrate()

    def _state(self, what):
        torch = self.torch
        nl = self.n + self.nh
        bufs = {k: torch.empty((nl, 3), dtype=torch.float64, device="cuda") for k in what
                if k != "t"}
        if "t" in what:
            bufs["t"] = torch.empty(nl, dtype=torch.int32, device="cuda")
        torch.cuda.current_stream().synchronize()
        self.sys.atoms_ptr(*(bufs[k].data_ptr() if k in bufs else None
                             for k in ("x", "v", "f", "t")))
        return bufs

    def owned_state(self):
        b = self._state(("x", "v", "t"))
        return b["x"][:self.n], b["v"][:self.n], b["t"][:self.n]

    def owned_forces(self):
        return self._state(("f",))["f"][:self.n]

    def kinetic(self):
        _, v, _ = self.owned_state()
        return float((v * v).sum()) * self.hp.mass
