"""MD-Bench short-range timestep on B200: atom-steps/s, mixed FP32 vs FP64.

One bench step = one rebuild period of the reference loop (reneigh_every = 20
MD timesteps: 19 plain steps and one step with the full rebuild), thermo
sampled every nstat = 100 steps as the reference does.

Headline (``value``): the cluster-pair scheme (GROMACS-style 4x4 clusters,
bounding-box pruned lists) on LJ fcc 64^3 cells = 1,048,576 atoms, reduced
density 0.8442, T 1.44, cutoff 2.5 + skin 0.3, half lists, mixed precision.
The same run reports every other cluster-pair variant (4x4/4x8, full/half,
mixed/FP64), the Verlet-list scheme on the same workload and both EAM paths on
Cu fcc 32^3 cells (131,072 atoms, a = 3.615 A, 1600 K, funcfl Cu_u3), each
mixed variant with its force error against FP64 and the energy drifts.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun) every rank runs one independent replica for the
headline (value is the sum over ranks, timing the max over ranks), and the
line's ``sharded`` key runs the Verlet-list LJ system decomposed into z-slabs
over all ranks (halo exchange every step, atoms migrating at rebuilds).
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "md-bench_b200"))

LJ_CELLS = 64
C5_CELLS = 128
C4_REPLICAS = 256
STUB_ATOMS = 1 << 20
EAM_CELLS = 32
EAM_A = 3.615
EAM_T = 1600.0
EAM_FILE = os.path.join(ROOT, "md-bench_b200", "data", "Cu_u3.eam")
REF_CP = {shape: os.path.join(ROOT, "oracle", "_ref", f"MDBench-CP-{shape}")
          for shape in ("4x4", "4x8")}
METRIC = "atom-steps/s, LJ+EAM mixed-FP32 vs FP64 on 1 B200 at stated force error"
# headline workload: GROMACS-style 4x4 cluster pairs, half lists, mixed precision
HEAD = {"kind": "cp44", "precision": "mixed", "half": 1, "path": 0}
HEAD_WORKLOAD = f"lj-fcc-{LJ_CELLS}^3-clusterpair-4x4-half-mixed"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50, help="timed bench steps (20 MD steps each)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-variants", action="store_true", help="headline only")
    ap.add_argument("--profile", choices=[f"{k}_{p}{h}" for k in ("lj", "eam", "cp44", "cp48")
                                          for p in ("mixed", "fp64") for h in ("", "_half")]
                    + [f"{k}_mixed{h}_pairs" for k in ("cp44", "cp48") for h in ("", "_half")]
                    + ["c5_mixed", "c5_mixed_pairs", "c5_fp64", "c4_mixed", "stub",
                       "cp44_mixed_half_checked"]
                    + [k for k in VARIANT_SPEC if "mixedcomp" in k],
                    help="run one variant only (W+K bench steps + force timing), for ncu")
    ap.add_argument("--cells", type=int, default=None, help="fcc cells per side (profiling)")
    ap.add_argument("--tune", default=None, help="key=value[,key=value] context tuning")
    ap.add_argument("--replicas", type=int, default=C4_REPLICAS, help="ensemble size")
    ap.add_argument("--no-autotune", action="store_true", help="ensemble with default choices")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi clock and throttle-reason sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.p = None
        if shutil.which("nvidia-smi"):
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "-i", str(device),
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                                      errors="replace")

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") == 5]
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[2 + k].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].strip().isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def lj_workload(mdb, precision, device, cells=None, half=0):
    c = cells or LJ_CELLS
    hp = mdb.host_params(nx=c, ny=c, nz=c, half_neigh=half)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t), precision=precision, device=device)
    return s, (x, v, t)


def cp_workload(mdb, precision, device, cells=None, half=0, cluster_n=4, types=None):
    """The cluster-pair scheme (GROMACS-style 4xN clusters) on the LJ workload;
    ``types`` = (epsilon_per_type, sigma_per_type) gives the multi-type liquid
    (types drawn by createAtom, cutoff 2.5 sigma_max)."""
    c = cells or LJ_CELLS
    kw = {}
    if types is not None:
        import workloads as W
        kw = dict(types=types, cutforce=W.c5_cutoff(types[1]))
    hp = mdb.host_params(nx=c, ny=c, nz=c, half_neigh=half, **kw)
    x, v, t = mdb.create_fcc(hp)
    eps = sig = None
    if types is not None:
        eps, sig = list(types[0]), list(types[1])
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=cluster_n, half_neigh=half,
                          precision=precision, device=device, xprd=hp.xprd, yprd=hp.yprd,
                          zprd=hp.zprd, cutforce=hp.cutforce, cutneigh=hp.cutneigh, dt=hp.dt,
                          dtforce=hp.dtforce, mass=hp.mass, epsilon=hp.epsilon,
                          sigma=hp.sigma, ntypes=hp.ntypes, reneigh_every=hp.reneigh_every,
                          nstat=hp.nstat, epsilon_per_type=eps, sigma_per_type=sig)
    return s, (x, v, t)


def eam_workload(mdb, precision, device, cells=None, half=0):
    c = cells or EAM_CELLS
    tab = mdb.read_funcfl(EAM_FILE)
    hp = mdb.host_params(eam=tab, nx=c, ny=c, nz=c, rho=4.0 / EAM_A ** 3, temp=EAM_T)
    x, v, t = mdb.create_fcc(hp)
    # the reference reads this configuration from a dump (-i): cutneigh/2 bins
    hp.from_file = 1
    s = mdb.system_from_host(hp, len(t), eam=tab, precision=precision, device=device)
    return s, (x, v, t)


def time_run(torch, s, steps, warmup, rebuild_every, first=0):
    """Device time of `steps` bench steps, events on the library's stream."""
    stream = torch.cuda.ExternalStream(s.stream)
    n = first
    samples = []
    for _ in range(warmup):
        samples += s.run(rebuild_every, first_step=n)
        n += rebuild_every
    s.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = s.launches
    e0.record(stream)
    for _ in range(steps):
        samples += s.run(rebuild_every, first_step=n)
        n += rebuild_every
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, s.launches - l0, samples, n


def force_kernel_time(torch, s, reps=20):
    """Average duration of one force launch (no energy), on the launching stream."""
    stream = torch.cuda.ExternalStream(s.stream)
    for _ in range(3):
        s.compute_force()
    s.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        s.compute_force()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def algorithmic_bytes(kind, precision, natoms, mean_list):
    """Bytes one force launch must move (per atom: list + count + own position +
    one read of each neighbour position + force write; EAM: two list passes,
    rho/fp arrays)."""
    pos = 32 if precision == "fp64" else 16
    if kind == "lj":
        per = 4 * mean_list + 4 + pos + pos + 24
    else:
        per = 2 * (4 * mean_list + 4 + pos) + pos + 8 + 8 + 24
    return per * natoms, per


def rel_force_err(a, b):
    rms = np.sqrt(np.mean(np.sum(b * b, axis=1)))
    d = np.sqrt(np.sum((a - b) ** 2, axis=1))
    return float(np.sqrt(np.mean(d * d)) / rms), float(d.max() / rms)


def make_system(mdb, kind, precision, args, device, half=0, path=0):
    """A workload's context and initial state; path 1: the pair-list force path
    of the mixed cluster-pair scheme."""
    if kind == "c5":
        import workloads as W
        s, init = cp_workload(mdb, precision, device, args.cells or C5_CELLS, 1, cluster_n=4,
                              types=W.c5_types())
    elif kind.startswith("cp"):
        s, init = cp_workload(mdb, precision, device, args.cells, half, cluster_n=int(kind[3]))
    else:
        make = lj_workload if kind == "lj" else eam_workload
        s, init = make(mdb, precision, device, args.cells, half)
    if kind.startswith("c") and path:
        s.tune("force_path", 1)
    for kv in (args.tune.split(",") if getattr(args, "tune", None) else []):
        k, val = kv.split("=")
        if kind.startswith("c") != k.startswith("eam"):
            s.tune(k, int(val))
    return s, init


def measure(torch, mdb, kind, precision, args, device, half=0, steps=None, path=0):
    steps = steps or args.steps
    s, (x, v, t) = make_system(mdb, kind, precision, args, device, half, path)
    s.set_atoms(x, v, t)
    s.setup()
    th0 = s.thermo()
    nat = len(t)
    every = s.params.reneigh_every
    d0 = s.pair_stats()[0] if path else 0
    secs, launches, samples, nsteps = time_run(torch, s, steps, args.warmup, every)
    mean_list = float(s.numneigh().mean())
    out = dict(system=s, natoms=nat, secs=secs, launches=launches, samples=samples,
               nsteps=nsteps, th0=th0, mean_list=mean_list,
               value=nat * every * steps / secs, ms_per_step=1e3 * secs / steps,
               init=(x, v, t))
    if path:
        d1, codes = s.pair_stats()
        # derivations of the pair codes during the warm-up and timed periods,
        # and the pair slots the force kernel evaluates per atom
        out["pair_stats"] = {"pair_derivations": d1 - d0,
                             "pair_md_steps": (args.warmup + steps) * every,
                             "pair_slots_per_atom": round(2.0 * codes / nat, 2)}
    return out


def checked_rebuilds(torch, mdb, args, device, limit=0.15):
    """The headline workload with displacement-checked rebuilds (any atom
    moving farther than skin / 2 since the last build also rebuilds, besides
    the fixed schedule), the decision taken on the device (a conditional CUDA
    graph per step) and on the host (one synchronisation per step); W + K
    bench steps of 20 MD steps each, device-timed like the headline."""
    out = {"max_displacement": limit}
    for mode, host in (("device", 0), ("host", 1)):
        s, (x, v, t) = make_system(mdb, HEAD["kind"], HEAD["precision"], args, device,
                                   HEAD["half"], HEAD["path"])
        s.tune("check_on_host", host)
        s.set_rebuild_check(limit)
        s.set_atoms(x, v, t)
        s.setup()
        secs, launches, _, _ = time_run(torch, s, args.steps, args.warmup, 20)
        sched, trig = s.rebuilds()
        out[mode] = {"value": len(t) * 20 * args.steps / secs,
                     "ms_per_step": 1e3 * secs / args.steps, "rebuilds_scheduled": sched,
                     "rebuilds_checked": trig, "device_decided_steps": s.check_stats()[0],
                     "gpu_launches": launches}
        s.close()
    return out


def stub_bench(torch, mdb, device, natoms=STUB_ATOMS, nneighs=76, reps=20):
    """The stub gather benchmark (verletlist/main-stub.c) on the GPU: the FP64
    full-list LJ force alone on synthetic lists (seq: the next 76 atoms, fix:
    the same 76 atoms for all, rand: 76 random atoms), atoms on a diagonal,
    every listed pair inside the cutoff. Reports the reference stub's figure,
    atom updates per second, with ns per neighbour and the gather rate."""
    out = {}
    for pattern in ("seq", "fix", "rand"):
        x, v, t, num, nb = mdb.stub_system(natoms, pattern, nneighs)
        s, _, _ = mdb.stub_context(x, v, t, num, nb, device=device)
        secs = force_kernel_time(torch, s, reps=reps)
        s.close()
        # list entry + the gathered double4 position per neighbour, plus per
        # atom its own position, row length and force
        bytes_per_atom = nneighs * (4 + 32) + 32 + 4 + 24
        out[pattern] = {"atom_updates_per_s": natoms / secs,
                        "ns_per_neighbor": secs / (natoms * nneighs) * 1e9,
                        "force_us": secs * 1e6,
                        # list entries plus gathered positions per second: the
                        # positions (32 MB) are served from L2/L1, not HBM, so
                        # this is no HBM roofline figure
                        "cache_served_gather_gb_per_s": natoms * bytes_per_atom / secs / 1e9}
    return {"natoms": natoms, "nneighs": nneighs, "precision": "fp64", "list": "full",
            "patterns": out}


def c4_specs(count):
    import workloads as W
    return [{"cells": n, "rho": rho, "temp": T, "natoms": 4 * n ** 3}
            for n, rho, T in W.c4_replicas(count)]


class Replicas:
    """Initial states of ensemble replicas (createAtom at each replica's cells,
    density and temperature) and set-up mixed-precision systems built from them."""

    def __init__(self, mdb, device):
        self.mdb, self.device, self.cache = mdb, device, {}

    def state(self, sp):
        key = (sp["cells"], sp["rho"], sp["temp"])
        if key not in self.cache:
            c = sp["cells"]
            hp = self.mdb.host_params(nx=c, ny=c, nz=c, rho=sp["rho"], temp=sp["temp"])
            x, v, t = self.mdb.create_fcc(hp)
            self.cache[key] = (hp, x, v, t)
        return self.cache[key]

    def build(self, sp, cluster_n, half, column_edge=100, choice=None, precision="mixed",
              check=0.0):
        import autotune as AT
        hp, x, v, t = self.state(sp)
        s = self.mdb.ClusterSystem(natoms=len(t), cluster_n=cluster_n, half_neigh=half,
                                   column_edge=column_edge,
                                   precision=precision, device=self.device, xprd=hp.xprd,
                                   yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
                                   cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce,
                                   mass=hp.mass, reneigh_every=hp.reneigh_every,
                                   nstat=hp.nstat, ntypes=hp.ntypes)
        if choice is not None and precision == "mixed":
            AT.apply_launch(s, choice)
        if check > 0.0:
            s.set_rebuild_check(check)
        s.set_atoms(x, v, t)
        s.setup()
        return s


def run_ensemble(torch, mdb, members, args, every=20, check_on_host=None):
    """Device time of args.steps rebuild periods of an ensemble (after
    args.warmup untimed ones) and the energy drift of every member."""
    ens = mdb.Ensemble(members)
    if check_on_host is not None:
        ens.tune("check_on_host", check_on_host)
    th0 = [m.thermo() for m in members]
    stream = torch.cuda.ExternalStream(ens.stream)
    n = 0
    for _ in range(args.warmup):
        ens.run(every, first_step=n, max_samples=0)
        n += every
    torch.cuda.synchronize()
    samples = [[] for _ in members]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = ens.launches
    e0.record(stream)
    for _ in range(args.steps):
        out = ens.run(every, first_step=n, max_samples=1)
        for k, q in enumerate(out):
            samples[k] += q
        n += every
    e1.record(stream)
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    launches = ens.launches - l0
    ens.close()
    drifts = [(q[-1]["E"] - t["E"]) / abs(t["E"]) if q else 0.0
              for q, t in zip(samples, th0)]
    return secs, launches, np.array(drifts), n


def sharded(torch, dist, mdb, rank, world, device, md_steps=40):
    """The z-slab domain decomposition of the Verlet-list scheme (full lists,
    mixed) on LJ fcc 64^3: every rank owns a slab of the same system and
    exchanges its halo's positions every step and atoms at each rebuild
    (md-bench_b200/domain.py). Several ranks exchange over torch.distributed
    point-to-point calls (NCCL); one rank gets its slab's own z images
    through host queues, as its own neighbour. One untimed rebuild period,
    then md_steps steps timed with CUDA events after a device synchronisation
    on both sides (the loop is host-driven: host work is inside), max over
    ranks. value = all atoms x md_steps / that time."""
    import domain as D
    hp = mdb.host_params(nx=LJ_CELLS, ny=LJ_CELLS, nz=LJ_CELLS)
    x, v, t = mdb.create_fcc(hp)
    box = (hp.xprd, hp.yprd, hp.zprd)
    tr = (D.DistTransport(torch, dist, "cuda") if world > 1
          else D.ThreadTransport(D.ThreadTransport.Hub(1), 0))
    eng = D.MdbEngine(torch, mdb, hp, device, "mixed")
    run = D.SlabRun(D.Slabs(box, hp.cutneigh, world, rank), tr, eng, hp.reneigh_every)
    run.start(x, v, t, np.arange(len(t)))
    run.run(hp.reneigh_every)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run.run(md_steps, first_step=hp.reneigh_every)
    torch.cuda.synchronize()
    e1.record()
    e1.synchronize()
    secs = reduce_scalar(torch, dist, e0.elapsed_time(e1) / 1e3, "max", "cuda")
    temp = run.temperature(len(t))
    owned = reduce_scalar(torch, dist, eng.n, "max", "cuda")
    halo = reduce_scalar(torch, dist, eng.nh, "max", "cuda")
    eng.sys.close()
    return {"value": len(t) * md_steps / secs, "unit": "atom-steps/s", "ranks": world,
            "scaling": "strong", "workload": HEAD_WORKLOAD.replace("clusterpair-4x4-half",
                                                                  "verletlist-full-zslabs"),
            "md_steps": md_steps, "max_owned_atoms": int(owned), "max_halo_atoms": int(halo),
            "T_end": temp,
            "exchange": "NCCL point-to-point" if world > 1 else "one slab: its own z images"}


def reduce_scalar(torch, dist, x, op, device):
    """x reduced over all ranks (op "max" or "sum"); x itself without a group."""
    if dist is None:
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def c4_ensemble(torch, mdb, args, device, rank=0, world=1, dist=None):
    """256 LJ replicas of uneven size, density and temperature advanced as one
    ensemble (one graph launch per timestep, batched kernels over all
    replicas), autotuned per size class; the same replicas in FP64 give the
    energy drift the mixed path is compared with. With several ranks the
    replicas are bin-packed by atom count over the GPUs (no exchange); the
    time is the slowest rank's."""
    import autotune as AT
    import workloads as W
    specs = c4_specs(args.replicas)
    total_atoms = sum(sp["natoms"] for sp in specs)
    if world > 1:
        mine = W.assign_replicas([sp["natoms"] for sp in specs], world)[rank]
        specs = [specs[i] for i in mine]
    pool = Replicas(mdb, device)
    t0 = time.perf_counter()
    if args.no_autotune:
        choice, trials = {}, []
    else:
        choice, trials = AT.tune_ensemble(specs, lambda sp, n, h, e: pool.build(sp, n, h, e),
                                          rounds=2)
    tune_secs = time.perf_counter() - t0
    pick = [choice.get(AT.size_class(sp["natoms"]), AT.DEFAULT) for sp in specs]
    every = 20
    members = [pool.build(sp, c["cluster_n"], c["half"], c["column_edge"], c)
               for sp, c in zip(specs, pick)]
    secs, launches, d32, n = run_ensemble(torch, mdb, members, args, every)
    secs = reduce_scalar(torch, dist, secs, "max", "cuda")
    # the same replicas advanced one after another (each its own graph loop)
    t1 = time.perf_counter()
    for m in members:
        m.run(every, first_step=n, max_samples=0)
    serial = time.perf_counter() - t1
    for m in members:
        m.close()
    members = [pool.build(sp, c["cluster_n"], c["half"], c["column_edge"], None, "fp64")
               for sp, c in zip(specs, pick)]
    secs64, _, d64, _ = run_ensemble(torch, mdb, members, args, every)
    secs64 = reduce_scalar(torch, dist, secs64, "max", "cuda")
    serial = reduce_scalar(torch, dist, serial, "max", "cuda")
    for m in members:
        m.close()
    # displacement-checked rebuilds (limit skin / 2, a member rebuilds when its
    # own flag trips), decided on the device (a conditional graph per step) and
    # on the host (one synchronisation per step)
    checked = {"max_displacement": 0.15}
    for mode, host in (("device", 0), ("host", 1)):
        members = [pool.build(sp, c["cluster_n"], c["half"], c["column_edge"], c, check=0.15)
                   for sp, c in zip(specs, pick)]
        sc, _, _, _ = run_ensemble(torch, mdb, members, args, every, check_on_host=host)
        sc = reduce_scalar(torch, dist, sc, "max", "cuda")
        checked[mode] = {"value": total_atoms * every * args.steps / sc,
                         "rebuilds_scheduled": members[0].rebuilds()[0],
                         "rebuilds_checked": members[0].rebuilds()[1]}
        for m in members:
            m.close()
    nat = total_atoms
    shapes = {}
    for c in pick:
        key = f"4x{c['cluster_n']}-{'half' if c['half'] else 'full'}-edge{c['column_edge']}"
        shapes[key] = shapes.get(key, 0) + 1
    return {"value": nat * every * args.steps / secs, "ms_per_step": 1e3 * secs / args.steps,
            "natoms": nat, "replicas": len(specs), "md_steps": every * args.steps,
            "gpu_launches": launches, "graph_launches_per_md_step": 1,
            "energy_drift_max_abs": reduce_scalar(torch, dist, np.abs(d32).max(), "max", "cuda"),
            "energy_drift_fp64_max_abs": reduce_scalar(torch, dist, np.abs(d64).max(), "max",
                                                       "cuda"),
            "excess_drift_vs_fp64_max_abs": reduce_scalar(torch, dist, np.abs(d32 - d64).max(),
                                                          "max", "cuda"),
            "excess_drift_vs_fp64_median_abs": float(np.median(np.abs(d32 - d64))),
            "fp64_value": nat * every * args.steps / secs64,
            "checked_rebuilds": checked,
            "serial_value": nat * every / serial,
            "autotune": {"seconds": round(tune_secs, 2), "trials": len(trials),
                         "choice_per_size_class": {str(k): v for k, v in choice.items()},
                         "replicas_per_shape": shapes}}


# systems in flight in the end-to-end measurement (each its own context,
# device buffers, stream and host thread): measured 3.0-3.4e9 atom-steps/s
# with two, 3.7-3.9e9 with three, 3.6-3.9e9 with four
E2E_INFLIGHT = 3


def e2e(torch, systems, init, steps, every, device):
    """Same metric through the public C ABI with host buffers: each step
    uploads one system's atoms from pinned host memory, runs setup + one
    rebuild period and reads positions and velocities back into pinned host
    memory. ``systems`` are independent contexts, each driven by its own host
    thread (the ABI calls release the GIL), so that one step's copies and
    host-side waits overlap another step's kernels, as a caller feeding a
    stream of systems would run them; every step's copies stay inside the
    timed region."""
    import threading
    x, v, t = init
    n = len(t)

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    hx, hv, ht = pinned(x), pinned(v), pinned(t)
    bi = hx.nbytes + hv.nbytes + ht.nbytes
    bo = 2 * 3 * 8 * n + 4 * n
    # results land in pinned host buffers as well, one set per system
    outs = [tuple(pinned(np.empty_like(a)) for a in (hx, hv, ht)) for _ in systems]
    share = [steps // len(systems) + (1 if k < steps % len(systems) else 0)
             for k in range(len(systems))]
    errors = []

    def work(k):
        try:
            torch.cuda.set_device(device)
            s, out = systems[k], outs[k]
            for _ in range(share[k]):
                s.set_atoms(hx, hv, ht)
                s.setup()
                s.run(every, first_step=0)
                s.atoms(out=out)
            s.synchronize()
        except Exception as e:  # re-raised on the calling thread
            errors.append(e)

    # one untimed step per system: first-use allocations and graph captures
    for s, out in zip(systems, outs):
        s.set_atoms(hx, hv, ht)
        s.setup()
        s.run(every, first_step=0)
        s.atoms(out=out)
        s.synchronize()
    workers = [threading.Thread(target=work, args=(k,)) for k in range(len(systems))]
    t0 = time.perf_counter()
    for w in workers:
        w.start()
    for w in workers:
        w.join()
    secs = time.perf_counter() - t0
    if errors:
        raise errors[0]
    for k, out in enumerate(outs):
        if share[k] and not np.all(np.isfinite(out[0])):
            raise RuntimeError("end-to-end run returned non-finite positions")
    return dict(value=n * every * steps / secs, unit="atom-steps/s", h2d_bytes_per_step=bi,
                d2h_bytes_per_step=bo, systems_in_flight=len(systems))


def host_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            return "avx512f" in f.read()
    except OSError:
        return False


def ref_cp_binary():
    """The fastest reference cluster-pair build this host can run."""
    if host_has_avx512() and os.path.exists(REF_CP["4x8"]):
        return REF_CP["4x8"], "4x8 AVX-512"
    if os.path.exists(REF_CP["4x4"]):
        return REF_CP["4x4"], "4x4 AVX2"
    return None, None


def cpu_baseline(md_steps=20, half=1):
    """The reference CPU cluster-pair build on this host (all cores), a bounded
    sample of the headline workload: LJ fcc 64^3, half lists when the headline
    uses them, md_steps steps with one rebuild."""
    cores = os.cpu_count() or 1
    binary, shape = ref_cp_binary()
    if binary is not None:
        env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_SCHEDULE="static",
                   OMP_PROC_BIND="close")
        out = subprocess.run([binary, "-nx", str(LJ_CELLS), "-ny", str(LJ_CELLS), "-nz",
                              str(LJ_CELLS), "-n", str(md_steps), "-half", str(half)], env=env,
                             capture_output=True, text=True, errors="replace",
                             timeout=1200).stdout  # it may print stray bytes
        for line in out.splitlines():
            if "atom updates/us" in line:
                val = float(line.split("|")[1].split()[0]) * 1e6
                return dict(value=val, unit="atom-steps/s", cores=cores, kind="reference",
                            sample=f"reference cluster-pair {shape} build (-Ofast, OpenMP), "
                                   f"LJ {LJ_CELLS}^3 (1,048,576 atoms), "
                                   f"{'half' if half else 'full'} lists, {md_steps} steps "
                                   "incl. one rebuild; its own Performance line")
        raise RuntimeError("reference run printed no performance line")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # checker only: timed as the CPU baseline
    o = oracle.Oracle(nx=32, ny=32, nz=32)
    o.lattice()
    o.setup()
    o.force()
    t0 = time.perf_counter()
    o.run(md_steps)
    secs = time.perf_counter() - t0
    return dict(value=32 ** 3 * 4 * md_steps / secs, unit="atom-steps/s", cores=1,
                kind="port", sample=f"C restatement, LJ 32^3, {md_steps} steps")


def reference_arm(args, rank):
    if rank != 0:
        return
    steps = 20 * max(args.steps // 5, 1)
    cb = cpu_baseline(steps, half=HEAD["half"])
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"],
            "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": HEAD_WORKLOAD, "natoms": 1048576, "md_steps": steps},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def fp32_peak(mdb=None, device=0):
    """FP32 peak: measured in this run by mdb_fp32_fma_rate (packed FMA chains
    on all SMs; the pool's MEASURED_PEAKS.json has no FP32 figure), with the
    figure derived from its max SM clock (148 SMs x 128 FP32 lanes x 2 flops
    per FMA) beside it."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f)["sm_max_mhz"])
        dsrc = "sm_max_mhz of MEASURED_PEAKS.json"
    except Exception:
        mhz, dsrc = 1965.0, "the nominal 1965 MHz"
    derived = 148 * 128 * 2 * mhz * 1e6 / 1e12
    if mdb is not None:
        measured = mdb.fp32_fma_rate(device) / 1e12
        if measured > 0:
            return measured, ("measured in this run: mdb_fp32_fma_rate, packed FP32 FMA "
                              f"chains on all SMs (derived from {dsrc}: {derived:.1f})")
    return derived, f"derived from {dsrc}"


def pairs_in_cutoff(x, box, rc):
    """P_c: ordered atom pairs inside the force cutoff per atom (periodic)."""
    from scipy.spatial import cKDTree
    xw = np.mod(x, box)
    tree = cKDTree(xw, boxsize=box)
    return (tree.count_neighbors(tree, rc) - len(x)) / len(x)


def cp_flops_per_atom(pc, half):
    """Algorithmic flops per atom-step of the cluster-pair LJ force: 24 per
    in-cutoff pair (3 sub, 3 mul + 2 add, 1 cmp, 1 div, 3 mul, 5 force, 6 for the
    accumulation), half lists P_c/2 pairs x (24 + 3 for the reaction)."""
    return pc / 2 * 27 if half else pc * 24


# the fixed window of the energy-drift comparison (MD steps; the multi-type
# liquid runs its configuration's 500)
DRIFT_STEPS = 1000


def _variant_spec():
    """key -> (kind, precision, half lists, force path) of every variant in the
    line; force path 1 is the pair-list kernel of the mixed cluster-pair scheme."""
    spec = {}
    for kind in ("cp44", "cp48"):
        for half in (0, 1):
            h = "_half" if half else ""
            spec[f"{kind}_mixed{h}"] = (kind, "mixed", half, 0)
            spec[f"{kind}_mixed{h}_pairs"] = (kind, "mixed", half, 1)
            spec[f"{kind}_fp64{h}"] = (kind, "fp64", half, 0)
    for prec in ("mixed", "fp64"):
        spec[f"vl_{prec}"] = ("lj", prec, 0, 0)
        spec[f"eam_{prec}"] = ("eam", prec, 0, 0)
        spec[f"c5_{prec}"] = ("c5", prec, 1, 0)
    spec["c5_mixed_pairs"] = ("c5", "mixed", 1, 1)
    # compensated sums (and, on the cluster-pair scheme, FP64 cutoff decisions
    # near r_c on the pair-list kernel)
    spec["cp44_mixedcomp_half"] = ("cp44", "mixed_comp", 1, 1)
    spec["c5_mixedcomp"] = ("c5", "mixed_comp", 1, 1)
    spec["vl_mixedcomp"] = ("lj", "mixed_comp", 0, 0)
    spec["eam_mixedcomp"] = ("eam", "mixed_comp", 0, 0)
    return spec


VARIANT_SPEC = _variant_spec()


def _twin(key):
    kind, prec, half, _ = VARIANT_SPEC[key]
    return f"{key.split('_')[0]}_fp64{'_half' if half and kind != 'c5' else ''}"


# the FP64 variant each mixed one is compared with
FP64_TWIN = {k: _twin(k) for k in VARIANT_SPEC if "_mixed" in k}


def drift_window(mdb, kind, precision, args, device, half=0, path=0, md_steps=DRIFT_STEPS):
    """Total-energy drift (E_end - E_0) / |E_0| over md_steps MD steps from the
    workload's initial state, whatever --steps is; returns the system at the
    window's end with it."""
    s, (x, v, t) = make_system(mdb, kind, precision, args, device, half, path)
    s.set_atoms(x, v, t)
    s.setup()
    e0 = s.thermo()["E"]
    e1 = s.run(md_steps)[-1]["E"]
    return s, float((e1 - e0) / abs(e0))


def force_compare(sm, sf, kind):
    """Mixed force against FP64 on the FP64 system's current state (both systems
    get the same atoms and rebuild)."""
    if kind.startswith("c"):
        x, v, t = sf.atoms()
        for s in (sf, sm):
            s.set_atoms(x, v, t)
            s.setup()
        nat = sm.iclusters()[0]
        valid = np.concatenate([np.arange(4) < k for k in nat])
        fm = sm.slots()[2][:len(valid)][valid]
        ff = sf.slots()[2][:len(valid)][valid]
    else:
        x, v, _, t = sf.atoms()
        for s in (sf, sm):
            s.set_atoms(x, v, t)
            s.setup()
        fm, ff = sm.atoms()[2], sf.atoms()[2]
    return rel_force_err(fm, ff)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    import torch
    import mdb

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    if args.profile == "stub":
        print(json.dumps(dict(profile=args.profile, **stub_bench(torch, mdb, local))),
              flush=True)
        return
    if args.profile == "cp44_mixed_half_checked":
        print(json.dumps(dict(profile=args.profile, **checked_rebuilds(torch, mdb, args, local))),
              flush=True)
        return
    if args.profile == "c4_mixed":
        res = c4_ensemble(torch, mdb, args, local, rank, world, dist)
        if rank == 0:
            print(json.dumps(dict(profile=args.profile, n_gpus=world, **res)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.profile:
        if args.profile in VARIANT_SPEC:
            kind, prec, half, path = VARIANT_SPEC[args.profile]
        else:
            kind, prec = args.profile.split("_")[:2]
            half = 1 if "_half" in args.profile or kind == "c5" else 0
            path = 1 if args.profile.endswith("_pairs") else 0
        m = measure(torch, mdb, kind, prec, args, local, half, path=path)
        kt = force_kernel_time(torch, m["system"], reps=3)
        print(json.dumps({"profile": args.profile, "natoms": m["natoms"],
                          "value": m["value"], "ms_per_step": m["ms_per_step"],
                          "force_ms": kt * 1e3, "mean_list": m["mean_list"],
                          "launches": m["launches"]}), flush=True)
        return

    # headline: the cluster-pair scheme on LJ 1M atoms, mixed precision
    barrier()
    clk = Clocks(local)
    head = measure(torch, mdb, HEAD["kind"], HEAD["precision"], args, local, HEAD["half"],
                   path=HEAD["path"])
    clocks = clk.stop()
    secs = reduce_scalar(torch, dist, head["secs"], "max", "cuda")
    value = head["natoms"] * 20 * args.steps * world / secs

    s = head["system"]
    kt = force_kernel_time(torch, s)
    xh, _, _ = s.atoms()
    box = np.array([s.params.xprd, s.params.yprd, s.params.zprd])
    pc = pairs_in_cutoff(xh, box, s.params.cutforce)
    fpa = cp_flops_per_atom(pc, HEAD["half"])
    peak, src = fp32_peak(mdb, local)
    achieved = fpa * head["natoms"] / kt / 1e12
    # DRAM bytes of one launch from the ncu capture recorded in profiles/ (not
    # a counter of this run)
    traffic, tsrc = None, None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    tkey = "cp_pairs_bytes_per_atom" if HEAD["path"] else "cp_head_bytes_per_atom"
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        if tkey in tj:
            traffic = tj[tkey] * head["natoms"]
            tsrc = "profiles/traffic.json (ncu dram__bytes of one launch; not measured in this run)"
    if HEAD["path"]:
        # pair slots the pair-list kernel evaluates: two per listed j atom code
        computed = head["pair_stats"]["pair_slots_per_atom"]
        kname = "k_force_pairs<4, %s> (cluster-pair pair list, uniform types)"
    else:
        computed = float(s.numneigh().mean()) * 4
        kname = "k_force_mixed<4, %s> (cluster-pair, uniform types)"
    credited = pc / 2 if HEAD["half"] else pc
    roof = {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 1),
            "unit": "TFLOP/s", "frac": round(achieved / peak, 4), "traffic": traffic,
            "traffic_source": tsrc,
            "kernel": kname % ("half" if HEAD["half"] else "full"),
            "kernel_ms": round(kt * 1e3, 4), "pairs_in_cutoff_per_atom": round(pc, 2),
            "flops_per_atom": round(fpa, 1),
            "computed_pairs_per_atom": round(computed, 1),
            # pairs credited above over the pair slots the kernel evaluates,
            # and the rate with every such slot credited (the FP32 pipe's view;
            # the roofline fraction counts only in-cutoff pairs)
            "cluster_efficiency": round(credited / computed, 3),
            "achieved_all_computed_pairs": round(achieved * computed / credited, 3),
            "peak_source": src}

    extra = {}
    # the variants are one-GPU measurements: only in the one-rank run, so that
    # no rank waits on them inside a collective
    if not args.no_variants and world == 1:
        runs = {}
        for key, (kind, prec, half, path) in VARIANT_SPEC.items():
            if (kind, prec, half, path) == (HEAD["kind"], HEAD["precision"], HEAD["half"],
                                            HEAD["path"]):
                runs[key] = head
            else:
                # the multi-type liquid (128^3 cells) times half as many periods
                steps = max(args.steps // 2, 1) if kind == "c5" else None
                runs[key] = measure(torch, mdb, kind, prec, args, local, half, steps, path)
        var = {}
        for key, m in runs.items():
            var[key] = {"value": m["value"], "ms_per_step": m["ms_per_step"],
                        "natoms": m["natoms"], "md_steps_timed": m["nsteps"],
                        "mean_list": m["mean_list"]}
            if "pair_stats" in m:
                var[key].update(m["pair_stats"])
        for m in runs.values():
            if m is not head:
                m["system"].close()
        # energy drift over a fixed window from the initial state, mixed and
        # FP64 twins, and the mixed force error on the FP64 window's final state
        spec = {k: v for k, v in VARIANT_SPEC.items() if k in runs}
        f64_end = {}
        for key, (kind, prec, half, path) in spec.items():
            if prec != "fp64":
                continue
            n = 500 if kind == "c5" else DRIFT_STEPS
            sf, d = drift_window(mdb, kind, prec, args, local, half, 0, n)
            f64_end[key] = sf
            var[key]["drift_window_md_steps"] = n
            var[key]["energy_drift"] = d
        for key, (kind, prec, half, path) in spec.items():
            if prec == "fp64":
                continue
            ref = FP64_TWIN[key]
            n = var[ref]["drift_window_md_steps"]
            sm, d = drift_window(mdb, kind, prec, args, local, half, path, n)
            var[key]["drift_window_md_steps"] = n
            var[key]["energy_drift"] = d
            var[key]["energy_drift_fp64"] = var[ref]["energy_drift"]
            var[key]["excess_drift_vs_fp64"] = d - var[ref]["energy_drift"]
            rms, mx = force_compare(sm, f64_end[ref], kind)
            var[key]["force_rms_rel_err"] = rms
            var[key]["force_max_rel_err"] = mx
            var[key]["force_err_state"] = f"FP64 state after {n} MD steps"
            sm.close()
        for sf in f64_end.values():
            sf.close()
        extra = {"variants": var,
                 "mixed_over_fp64": {k.replace("_mixed", ""): var[k]["value"] /
                                     var[FP64_TWIN[k]]["value"] for k in var if k in FP64_TWIN},
                 "drift_note": "energy_drift: (E - E0)/|E0| over the fixed window "
                               "drift_window_md_steps from each workload's initial state; the "
                               "reference's LJ and EAM potentials are not shifted at the "
                               "cutoff, so the FP64 path itself drifts past 1e-4 per 1000 "
                               "steps on these workloads; excess_drift_vs_fp64 is the mixed "
                               "path's part"}
        var["cp44_mixed_half_checked"] = checked_rebuilds(torch, mdb, args, local)
        var["c4_ensemble_mixed"] = c4_ensemble(torch, mdb, args, local)
        var["stub_gather_fp64"] = stub_bench(torch, mdb, local)

    # end to end from the state the timed run reached (a liquid, as in use)
    extra_sys = [make_system(mdb, HEAD["kind"], HEAD["precision"], args, local, HEAD["half"],
                             HEAD["path"])[0] for _ in range(E2E_INFLIGHT - 1)]
    e2 = e2e(torch, [s] + extra_sys, s.atoms(), max(args.steps // 4, 4 * E2E_INFLIGHT), 20,
             local)
    for es in extra_sys:
        es.close()
    e2["value"] = reduce_scalar(torch, dist, e2["value"], "sum", "cuda")
    # the same LJ system split into z-slabs over all ranks
    barrier()
    try:
        dd = sharded(torch, dist, mdb, rank, world, local)
    except (mdb.MdbError, RuntimeError, ValueError) as e:
        dd = {"error": str(e)[:300]}
    cb = cpu_baseline(half=HEAD["half"]) if (rank == 0 and world == 1) else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32-mixed",
                "data": "synthetic",
                "config": {"workload": HEAD_WORKLOAD,
                           "natoms_per_gpu": head["natoms"], "md_steps_per_bench_step": 20,
                           "rebuild_every": 20, "thermo_every": 100, "density": 0.8442,
                           "cutoff": 2.5, "skin": 0.3, "cluster": "4x4",
                           "force_path": "pair list (listed cluster pairs' pairs within "
                                         "r_c + skin, re-derived when an atom moves past "
                                         "skin / 2)" if HEAD["path"] else "cluster pair",
                           "i_clusters_per_warp": 4, "j_atoms_per_lane": 2,
                           "lists": "half" if HEAD["half"] else "full",
                           "l2": "inputs larger than L2 (cluster list %.0f MB, "
                                 "positions and velocities %.0f MB)"
                                 % (head["mean_list"] * 4 * head["natoms"] / 4 / 1e6,
                                    head["natoms"] * 96 / 1e6),
                           "parallelism": f"replicas{world}"},
                "roofline": roof, "cpu_baseline": cb, "e2e": e2, "clocks": clocks,
                "gpu_launches": head["launches"], "sharded": dd}
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
