"""Autotuner for the cluster-pair scheme's free choices.

The reference fixes its cluster shape at compile time (CLUSTER_N = the SIMD
width: 4x4 for AVX2, 4x8 for AVX-512; clusterpair/atom.h) and its list form on
the command line (-half); the column grid then follows from the cluster shape
(setupNeighbor, clusterpair/neighbor.c:108-215: columns of max(M, N) / rho
atoms). Every choice below is therefore one of the reference's own valid
configurations, and lists stay bit-exact against the reference build of the
chosen shape, except for a bin size other than the reference's. The tuner
picks, per system size:

* cluster shape N = 4 or 8 (which also fixes the column size),
* list form: full or half (half-list reactions use atomics),
* the bin size: the column grid's xy edge (``column_edge``, percent of the
  reference's edge for the chosen shape; 100 keeps the reference's lists,
  other values give other clusters and lists with the same pairs inside the
  list cutoff, so the same forces up to summation order),
* the mixed force kernel's launch: threads per block (``force_block``),
  ``force_variant`` (prefetch depth, register budget), i-clusters per warp
  (``force_cpw``: 1, 2, 4, or 8 with 4x4 clusters) and j atoms per lane
  (``force_jpl``: 1, or 2 with four i-clusters per warp),

by measurement on the device. A single large system is tuned on the force
kernel's own time (``ClusterSystem.time_force``, CUDA events). Members of an
ensemble run concurrently and share the GPU, so an ensemble is tuned on the
throughput of the whole ensemble (atom-steps per second over whole rebuild
periods, graph and rebuild costs included), one size class and one setting at
a time: a size class tuned alone does not fill the GPU and favours choices
(full lists, small blocks) that lose once every replica shares it.
"""
import math
import time

import mdb

SHAPES = (4, 8)
FORMS = (0, 1)
BLOCKS = (64, 128, 256)
VARIANTS = (0, 1, 2, 3)
CPWS = (1, 2, 4, 8)
JPLS = (1, 2)
EDGES = (80, 100, 125)
DEFAULT = {"cluster_n": 4, "half": 1, "column_edge": 100, "force_block": 128,
           "force_variant": 2, "force_cpw": 4, "force_jpl": 1}


def valid(choice):
    """force_cpw 8 needs 4x4 clusters; several clusters per warp prefetch one
    block ahead (variant 1 runs as 0 there; 3 is a budget for 6 blocks)."""
    if choice.get("force_cpw", 1) == 8 and choice["cluster_n"] != 4:
        return False
    if choice.get("force_jpl", 1) == 2 and choice.get("force_cpw", 1) != 4:
        return False
    return not (choice.get("force_cpw", 1) > 1 and choice.get("force_variant", 0) == 1)


def size_class(natoms):
    """Octave of the atom count: replicas within a factor of two share a choice."""
    return int(math.log2(max(int(natoms), 1)))


def apply_launch(system, choice):
    """Launch settings of a choice on a (mixed-precision) system."""
    system.tune("force_block", choice["force_block"])
    system.tune("force_variant", choice["force_variant"])
    system.tune("force_cpw", choice["force_cpw"])
    system.tune("force_jpl", choice.get("force_jpl", 1))


def tune_system(build, precision="mixed", reps=20, shapes=SHAPES, forms=FORMS, edges=EDGES):
    """Best choice for one system. ``build(cluster_n, half, column_edge)``
    returns a set-up ClusterSystem; the choice minimises the force launch time
    (per step)."""
    best, trials = None, []
    for n in shapes:
        for half in forms:
            for edge in edges:
                s = build(n, half, edge)
                t = s.time_force(reps)
                base = {"cluster_n": n, "half": half, "column_edge": edge}
                trials.append((base, t))
                if precision == "mixed":
                    for blk, var, cpw, jpl in ((b, v, w, p) for b in BLOCKS for v in VARIANTS
                                               for w in CPWS for p in JPLS):
                        c = dict(base, force_block=blk, force_variant=var, force_cpw=cpw,
                                 force_jpl=jpl)
                        if not valid(c):
                            continue
                        apply_launch(s, c)
                        t = s.time_force(reps)
                        trials.append((c, t))
                        if best is None or t < best[1]:
                            best = (c, t)
                elif best is None or t < best[1]:
                    best = (base, t)
                s.close()
    choice = dict(DEFAULT)
    choice.update(best[0])
    return choice, trials


def _ensemble_rate(members, steps, rounds):
    ens = mdb.Ensemble(members)
    ens.run(steps, max_samples=0)  # graph capture, warm-up
    nat = sum(m.nlocal for m in members)
    t0 = time.perf_counter()
    for r in range(rounds):
        ens.run(steps, first_step=steps * (r + 1), max_samples=0)
    secs = time.perf_counter() - t0
    ens.close()
    return nat * steps * rounds / secs


def tune_ensemble(specs, build, steps=20, rounds=2, shapes=SHAPES, forms=FORMS, margin=0.02,
                  rate=None, edges=EDGES):
    """Choice per size class for an ensemble, by coordinate descent on the whole
    ensemble's throughput. ``specs`` is a list of replica descriptions with an
    ``natoms`` entry; ``build(spec, cluster_n, half, column_edge)`` returns a
    set-up mixed-precision ClusterSystem (with ``close()``). Every class starts
    at DEFAULT; classes are visited largest (total atoms) first, each trying
    the other shapes and list forms, then the other bin sizes of its shape,
    then the other threads per block and kernel variants, with every other
    class at its current choice. A change is kept
    only if the ensemble gets faster by more than ``margin`` (timing noise).
    ``rate(members)`` measures the throughput (default: an mdb.Ensemble run of
    ``rounds`` rebuild periods of ``steps`` steps after one untimed period).
    Returns ({size_class: choice}, trials), trials = (class, choice, rate)."""
    if rate is None:
        def rate(members):
            return _ensemble_rate(members, steps, rounds)
    classes = {}
    for sp in specs:
        classes.setdefault(size_class(sp["natoms"]), []).append(sp)
    order = sorted(classes, key=lambda c: (-sum(sp["natoms"] for sp in classes[c]), c))
    choice = {c: dict(DEFAULT) for c in classes}
    members = {c: [build(sp, DEFAULT["cluster_n"], DEFAULT["half"], DEFAULT["column_edge"])
                   for sp in classes[c]] for c in classes}

    def everyone():
        return [m for c in sorted(members) for m in members[c]]

    best = rate(everyone())
    trials = [(None, dict(DEFAULT), best)]

    def close(ms):
        for m in ms:
            m.close()

    def rebuild(c, trial):
        # a choice fixed at build time: new members, kept only if faster
        nonlocal best
        old = members[c]
        members[c] = [build(sp, trial["cluster_n"], trial["half"], trial["column_edge"])
                      for sp in classes[c]]
        for m in members[c]:
            apply_launch(m, trial)
        r = rate(everyone())
        trials.append((c, dict(trial), r))
        if r > best * (1.0 + margin):
            best, choice[c] = r, trial
            close(old)
        else:
            close(members[c])
            members[c] = old

    for c in order:
        for n in shapes:
            for half in forms:
                if (n, half) == (choice[c]["cluster_n"], choice[c]["half"]):
                    continue
                trial = dict(choice[c], cluster_n=n, half=half)
                if valid(trial):
                    rebuild(c, trial)
        start = choice[c]["column_edge"]
        for edge in edges:
            if edge not in (start, choice[c]["column_edge"]):
                rebuild(c, dict(choice[c], column_edge=edge))
    for c in order:
        for key, values in (("force_block", BLOCKS), ("force_variant", VARIANTS),
                            ("force_cpw", CPWS), ("force_jpl", JPLS)):
            for val in values:
                if val == choice[c][key]:
                    continue
                trial = dict(choice[c], **{key: val})
                if not valid(trial):
                    continue
                for m in members[c]:
                    apply_launch(m, trial)
                r = rate(everyone())
                trials.append((c, dict(trial), r))
                if r > best * (1.0 + margin):
                    best, choice[c] = r, trial
                else:
                    for m in members[c]:
                        apply_launch(m, choice[c])
    close(everyone())
    return choice, trials
