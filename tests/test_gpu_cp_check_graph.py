"""Displacement-checked rebuilds decided on the device (conditional CUDA graph
nodes, no host synchronisation per step) against the same check decided on
the host (tuning key "check_on_host" = 1, the host reads the flag after every
integration). Both take the same decisions, so FP64 and mixed full-list runs
(no atomics) end bit for bit equal, with the same rebuild counts; a device
rebuild that overflows the list capacity stops the call's later steps on the
device, and the host grows the list, replays that build and resumes, ending
where the host-decided run (which grows at once) ends.
"""
import numpy as np
import pytest

import mdb

from test_gpu_cp import _force_error_vs_fresh_build, _local_state

pytestmark = pytest.mark.gpu


def hot(check, host, precision="fp64", maxneighs=0, n=6, rho=0.95, temp=2.0):
    hp = mdb.host_params(nx=n, ny=n, nz=n, rho=rho, temp=temp, nstat=10)
    x, v, t = mdb.create_fcc(hp)
    kw = dict(xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
              cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
              reneigh_every=hp.reneigh_every, nstat=hp.nstat, natoms=len(t), cluster_n=4,
              precision=precision, ntypes=hp.ntypes)
    s = mdb.ClusterSystem(maxneighs=maxneighs, **kw)
    s.tune("check_on_host", host)
    s.set_rebuild_check(check)
    s.set_atoms(x, v, t)
    s.setup()
    return s, kw


def assert_same_state(a, b):
    for u, w in zip(_local_state(a), _local_state(b)):
        assert np.array_equal(u, w)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_decisions_match_host_decisions(precision):
    a, kw = hot(0.05, 0, precision)
    b, _ = hot(0.05, 1, precision)
    sa = a.run(57, max_samples=8)
    sb = b.run(57, max_samples=8)
    assert sa == sb and [q["step"] for q in sa] == [10, 20, 30, 40, 50]
    assert a.rebuilds() == b.rebuilds()
    sched, trig = a.rebuilds()
    assert sched == 2 and trig >= 3
    steps, replays = a.check_stats()
    assert steps > 20 and replays == 0
    assert b.check_stats() == (0, 0)
    assert_same_state(a, b)
    if precision == "fp64":
        assert _force_error_vs_fresh_build(a, kw) <= 1e-12
    # a second call continues from the first's state
    a.run(23, first_step=57, max_samples=0)
    b.run(23, first_step=57, max_samples=0)
    assert a.rebuilds() == b.rebuilds()
    assert_same_state(a, b)
    a.close()
    b.close()


def test_overflowing_device_rebuild_is_replayed():
    """The list capacity is one more than the lattice's longest row, so the
    first rebuild of the melting lattice with a longer row overflows it: on
    the device that rebuild stops the call's later steps, the host grows the
    list (1.2 x the longest row, as buildNeighbor does), replays the build and
    resumes. The end state equals the host-decided run's, which grows the list
    in the same rebuild."""
    probe, _ = hot(0.05, 1)
    longest = int(probe.numneigh().max())
    probe.close()
    a, kw = hot(0.05, 0, maxneighs=longest + 1)
    b, _ = hot(0.05, 1, maxneighs=longest + 1)
    assert a.counts()["maxneighs"] == longest + 1
    sa = a.run(57, max_samples=8)
    sb = b.run(57, max_samples=8)
    steps, replays = a.check_stats()
    assert replays >= 1 and steps > 20
    assert a.counts()["maxneighs"] == b.counts()["maxneighs"] > longest + 1
    assert sa == sb
    assert a.rebuilds() == b.rebuilds()
    assert_same_state(a, b)
    assert _force_error_vs_fresh_build(a, kw) <= 1e-12
    a.close()
    b.close()


def test_cold_system_never_rebuilds_on_the_device():
    a, _ = hot(0.15, 0, n=5, rho=0.8442, temp=0.01)
    b, _ = hot(0.0, 0, n=5, rho=0.8442, temp=0.01)
    sa = a.run(45, max_samples=8)
    sb = b.run(45, max_samples=8)
    assert sa == sb
    assert a.rebuilds()[1] == 0 and a.check_stats()[0] > 30
    assert_same_state(a, b)
    a.close()
    b.close()


def ensemble_members(host_check, maxneighs=None):
    """A hot dense replica, a mild one and a cold one (mixed, full lists), all
    with the displacement check; maxneighs: list capacity of the hot one."""
    specs = [(6, 0.95, 2.0), (4, 0.8, 0.5), (5, 0.8442, 0.02)]
    out = []
    for k, (n, rho, temp) in enumerate(specs):
        s, _ = hot(0.05, host_check, "mixed", maxneighs if (k == 0 and maxneighs) else 0,
                   n, rho, temp)
        out.append(s)
    return out


@pytest.mark.parametrize("squeeze", [False, True])
def test_ensemble_device_decisions_match_host_decisions(squeeze):
    """Batched ensemble with the check decided on the device (one conditional
    graph per step over all replicas; the members whose flag is up rebuild)
    against the host reading the flags every step: the same samples, rebuild
    counts and end states, bit for bit. With
    the hot replica's list capacity one more than its lattice's longest row,
    a device rebuild overflows it and is replayed by the host."""
    maxneighs = None
    if squeeze:
        probe, _ = hot(0.05, 1, "mixed")
        maxneighs = int(probe.numneigh().max()) + 1
        probe.close()
    a = ensemble_members(0, maxneighs)
    b = ensemble_members(1, maxneighs)
    ea, eb = mdb.Ensemble(a), mdb.Ensemble(b)
    ea.tune("check_on_host", 0)
    eb.tune("check_on_host", 1)
    ga = ea.run(57, max_samples=8)
    gb = eb.run(57, max_samples=8)
    assert ga == gb
    steps, replays = ea.check_stats()
    assert steps > 20 and eb.check_stats() == (0, 0)
    assert replays >= 1 if squeeze else replays == 0
    for u, w in zip(a, b):
        assert u.rebuilds() == w.rebuilds()
        assert_same_state(u, w)
    # each member rebuilds on its own flag: the hot one trips, the cold one not
    assert a[0].rebuilds()[1] > 0 and a[2].rebuilds()[1] == 0
    if squeeze:
        assert a[0].counts()["maxneighs"] == b[0].counts()["maxneighs"] > maxneighs
    ga = ea.run(23, first_step=57, max_samples=0)
    gb = eb.run(23, first_step=57, max_samples=0)
    for u, w in zip(a, b):
        assert_same_state(u, w)
    ea.close()
    eb.close()
    for s in a + b:
        s.close()
