"""The ensemble autotuner's search (coordinate descent on the whole ensemble's
throughput), run on fake members with a throughput model in place of the
device: it must find the choices the model rewards beyond the noise margin,
keep the defaults where a change gains less, and close every system it
builds (the tuned members too: the caller builds its own from the choice)."""
import itertools

import pytest

import autotune as AT


class FakeMember:
    def __init__(self, sp, n, half, edge, log):
        self.natoms, self.nlocal = sp["natoms"], sp["natoms"]
        self.cluster_n, self.half, self.edge = n, half, edge
        self.launch = {k: AT.DEFAULT[k]
                       for k in ("force_block", "force_variant", "force_cpw", "force_jpl")}
        self.closed = False
        log.append(self)

    def tune(self, key, value):
        assert not self.closed
        self.launch[key] = value

    def close(self):
        assert not self.closed
        self.closed = True


def model_rate(members):
    """Time of the ensemble = sum over members of natoms x cost, where the model
    rewards: 4x8 half lists for the 500-atom class (-20 %), full lists for the 4000-atom
    class (-1 %, inside the margin), 256 threads for the 4000-atom class
    (-10 %), eight i-clusters per warp for the 32,000-atom class (-8 %), a
    column edge of 125 % for the 32,000-atom class (-6 %; 80 % costs +5 %); plus
    one launch per distinct (shape, form, launch) group."""
    t, groups = 0.0, set()
    for m in members:
        assert not m.closed
        cls = AT.size_class(m.natoms)
        c = 1.0
        if cls == AT.size_class(500) and m.cluster_n == 8 and m.half:
            c *= 0.8
        if cls == AT.size_class(4000) and not m.half:
            c *= 0.99
        if cls == AT.size_class(4000) and m.launch["force_block"] == 256:
            c *= 0.9
        if cls == AT.size_class(32000) and m.launch["force_cpw"] == 8:
            c *= 0.92
        if cls == AT.size_class(32000):
            c *= {80: 1.05, 100: 1.0, 125: 0.94}[m.edge]
        if m.launch["force_variant"] != AT.DEFAULT["force_variant"]:
            c *= 1.05
        t += m.natoms * c
        groups.add((m.cluster_n, m.half, m.launch["force_block"], m.launch["force_variant"],
                    m.launch["force_cpw"], m.launch["force_jpl"]))
    t += 50.0 * len(groups)
    return sum(m.natoms for m in members) / t


def test_coordinate_descent_finds_rewarded_choices():
    # classes of 20,000 / 20,000 / 32,000 atoms: the rewards below are worth
    # 5.5 % and 2.7 % of the ensemble, the full-list gain 0.3 %
    specs = [{"natoms": 500}] * 40 + [{"natoms": 4000}] * 5 + [{"natoms": 32000}]
    log = []
    choice, trials = AT.tune_ensemble(specs, lambda sp, n, h, e: FakeMember(sp, n, h, e, log),
                                      rate=model_rate)
    c512, c4k, c32k = (choice[AT.size_class(n)] for n in (500, 4000, 32000))
    assert (c512["cluster_n"], c512["half"]) == (8, 1)
    assert c512["force_block"] == AT.DEFAULT["force_block"]
    assert (c4k["cluster_n"], c4k["half"]) == (4, 1)      # full lists gain < margin
    assert c4k["force_block"] == 256
    assert c32k == dict(AT.DEFAULT, force_cpw=8, column_edge=125)
    # the bin size stays the reference's where nothing rewards another
    assert c512["column_edge"] == c4k["column_edge"] == 100
    # the tuned members were built with their bin size
    assert any(m.edge == 125 for m in log) and any(m.edge == 80 for m in log)
    # force_cpw 8 was never tried on a 4x8 shape
    assert all(t[1]["force_cpw"] != 8 or t[1]["cluster_n"] == 4 for t in trials)
    assert all(c["force_variant"] == AT.DEFAULT["force_variant"] for c in choice.values())
    # every system built was closed, and trials start from the default ensemble
    assert log and all(m.closed for m in log)
    assert trials[0][0] is None and trials[0][1] == AT.DEFAULT
    # the largest class (by total atoms) is visited first
    assert trials[1][0] == AT.size_class(32000)


def test_no_change_within_noise():
    specs = [{"natoms": 1000}] * 3
    log = []
    flat = itertools.cycle([1.0, 1.01, 0.99, 1.015, 1.0, 1.019, 0.98, 1.0, 1.0, 1.0, 1.012,
                            1.0, 0.99, 1.0, 1.005])
    choice, trials = AT.tune_ensemble(specs, lambda sp, n, h, e: FakeMember(sp, n, h, e, log),
                                      rate=lambda ms: next(flat))
    assert choice == {AT.size_class(1000): AT.DEFAULT}
    assert all(m.closed for m in log)


class FakeSystem:
    """A single system whose force time the model below gives."""

    def __init__(self, n, half, edge, log):
        self.cluster_n, self.half, self.edge = n, half, edge
        self.launch = {}
        self.closed = False
        log.append(self)

    def tune(self, key, value):
        self.launch[key] = value

    def time_force(self, reps):
        # 4x4 half lists with a 125 % column edge and four i-clusters per warp
        # are fastest; everything else costs more
        t = 1.0
        t *= 1.0 if (self.cluster_n, self.half) == (4, 1) else 1.3
        t *= {80: 1.1, 100: 1.0, 125: 0.95}[self.edge]
        t *= 1.0 if self.launch.get("force_cpw", 4) == 4 else 1.2
        return t

    def close(self):
        self.closed = True


def test_single_system_search_covers_bin_sizes():
    log = []
    choice, trials = AT.tune_system(lambda n, h, e: FakeSystem(n, h, e, log))
    assert (choice["cluster_n"], choice["half"], choice["column_edge"]) == (4, 1, 125)
    assert choice["force_cpw"] == 4
    # every shape, list form and bin size was built once, and closed
    assert sorted((m.cluster_n, m.half, m.edge) for m in log) == sorted(
        (n, h, e) for n in AT.SHAPES for h in AT.FORMS for e in AT.EDGES)
    assert all(m.closed for m in log)
    assert all(AT.valid(c) for c, _ in trials if "force_cpw" in c)
