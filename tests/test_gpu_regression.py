"""The reference's regression case on the GPU paths: the default LJ run (32^3
fcc, 131,072 atoms, 200 steps, lists rebuilt every 20 steps) must end at the
temperature and pressure of tests/sim_copper_fcc_regression.sh in the
reference (T 7.961676e-01, P 6.721195e-01, within 1e-4 and 1e-3 relative: the
script's own tolerances), through both schemes, both list forms and both
precisions. The FP64 Verlet-list path with full lists, bit-identical to the
oracle, must print exactly what the strict FP64 reference build prints. The
cluster-pair runs end, as the reference's, with updateAtoms before the thermo.
"""
import pytest

import mdb

pytestmark = pytest.mark.gpu

REF_TEMP, REF_PRESS = 7.961676e-01, 6.721195e-01
TEMP_TOL, PRESS_TOL = 1e-4, 1e-3
STEPS = 200


def check(th):
    assert abs(th["T"] - REF_TEMP) / REF_TEMP <= TEMP_TOL, th["T"]
    assert abs(th["P"] - REF_PRESS) / REF_PRESS <= PRESS_TOL, th["P"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("half", [0, 1])
def test_verlet_list_default_case(precision, half):
    hp = mdb.host_params(half_neigh=half)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t), precision=precision)
    s.set_atoms(x, v, t)
    s.setup()
    s.run(STEPS)
    th = s.thermo()
    check(th)
    if precision == "fp64" and not half:
        assert f"{th['T']:.6e}" == "7.961535e-01"
        assert f"{th['P']:.6e}" == "6.721076e-01"
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("half", [0, 1])
@pytest.mark.parametrize("N", [4, 8])
def test_cluster_pair_default_case(N, half, precision):
    hp = mdb.host_params(half_neigh=half)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.ClusterSystem(natoms=len(t), cluster_n=N, half_neigh=half, precision=precision,
                          xprd=hp.xprd, yprd=hp.yprd, zprd=hp.zprd, cutforce=hp.cutforce,
                          cutneigh=hp.cutneigh, dt=hp.dt, dtforce=hp.dtforce, mass=hp.mass,
                          epsilon=hp.epsilon, sigma=hp.sigma, ntypes=hp.ntypes,
                          reneigh_every=hp.reneigh_every, nstat=hp.nstat)
    s.set_atoms(x, v, t)
    s.setup()
    s.run(STEPS)
    # the reference's last updateAtoms before its final thermo line: the atom
    # arrays then hold the full-step velocities (during the run they are
    # refreshed only at rebuilds, clusterpair/neighbor.c:2096-2149)
    s.update_single_atoms()
    check(s.thermo())
    s.close()
