"""The z-slab domain decomposition on libmdb contexts, on one GPU.

Two slab contexts (owned atoms + halo atoms from the other slab, periodic in x
and y only) are driven by two host threads of one process through
domain.ThreadTransport: the halo moves between them through the host, so no
kernel waits on the other context's kernels. Their forces, positions and
velocities are compared with one undivided context on the same initial
state, after setup and after a run across a rebuild with atoms changing
slabs. The per-atom neighbour order differs between the two (different bins
and ghost sets), so the FP64 sums agree to rounding, not bit for bit; the CPU
test (tests/test_domain.py) checks the host logic bit for bit.
"""
import threading

import numpy as np
import pytest

import mdb

pytestmark = pytest.mark.gpu

CELLS = 10
STEPS = 26
FP64_REL = 1e-12


def scale(f):
    return max(np.sqrt(np.mean(np.sum(f * f, axis=1))), 1.0)


@pytest.mark.parametrize("precision,half", [("fp64", 0), ("mixed", 0), ("fp64", 1),
                                            ("mixed", 1)])
def test_two_slab_contexts_match_one(precision, half):
    """Half lists: a pair across the slab face is computed by both slabs, each
    for its own atom (no reverse exchange); the undivided context computes it
    once with the reaction. Same pairs, so the same forces to rounding."""
    torch = pytest.importorskip("torch")
    import domain as D
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS, half_neigh=half)
    x, v, t = mdb.create_fcc(hp)
    n = len(t)
    one = mdb.system_from_host(hp, n, precision=precision)
    one.set_atoms(x, v, t)
    one.setup()
    F0 = one.atoms()[2]
    for k in range(STEPS):
        one.step(k)
    X, V, F, _ = one.atoms()
    T = one.thermo()["T"]

    box = (hp.xprd, hp.yprd, hp.zprd)
    hub = D.ThreadTransport.Hub(2)
    out, errors = [None, None], []

    def rank(r):
        try:
            torch.cuda.set_device(0)
            run = D.SlabRun(D.Slabs(box, hp.cutneigh, 2, r), D.ThreadTransport(hub, r),
                            D.MdbEngine(torch, mdb, hp, 0, precision, half),
                            hp.reneigh_every)
            run.start(x, v, t, np.arange(n))
            g0, _, _, f0 = run.gather()
            run.run(STEPS)
            out[r] = (g0, f0) + run.gather() + (run.temperature(n),)
        except Exception as e:  # re-raised by the test
            errors.append(e)

    th = [threading.Thread(target=rank, args=(r,)) for r in range(2)]
    for w in th:
        w.start()
    for w in th:
        w.join(timeout=300)
    if errors:
        raise errors[0]
    f0s, xs, vs, fs = (np.full((n, 3), np.nan) for _ in range(4))
    for g0, f0, g, xr, vr, fr, _ in out:
        f0s[g0] = f0
        xs[g], vs[g], fs[g] = xr, vr, fr
    moved = sum(len(set(o[0].tolist()) ^ set(o[2].tolist())) for o in out)
    assert moved > 0  # the rebuild handed atoms to the other slab
    if precision == "fp64":
        assert np.abs(f0s - F0).max() <= FP64_REL * scale(F0)
        # periodic positions: compare modulo the box
        d = np.abs((xs - X + 0.5 * np.array(box)) % np.array(box) - 0.5 * np.array(box))
        assert d.max() < 1e-10
        assert np.abs(vs - V).max() < 1e-10
        assert np.abs(fs - F).max() <= 1e-9 * scale(F)
        assert out[0][-1] == pytest.approx(T, rel=1e-10)
    else:
        # the lattice's forces cancel to ~1e-6 of a pair force: the scale is
        # at least 1 (FP32 sums of O(1) pair forces in another order)
        assert np.sqrt(np.mean(np.sum((f0s - F0) ** 2, axis=1))) / scale(F0) <= 1e-6
        assert out[0][-1] == pytest.approx(T, rel=1e-4)


def test_one_slab_context_matches_undivided():
    """One rank: the slab context's halo is its own z images, refreshed every
    step through host queues; across two rebuilds it follows the periodic
    context (FP64: same pairs, summation order differs at the box faces)."""
    torch = pytest.importorskip("torch")
    import domain as D
    hp = mdb.host_params(nx=CELLS, ny=CELLS, nz=CELLS)
    x, v, t = mdb.create_fcc(hp)
    n = len(t)
    one = mdb.system_from_host(hp, n, precision="fp64")
    one.set_atoms(x, v, t)
    one.setup()
    for k in range(45):
        one.step(k)
    X, V, F, _ = one.atoms()
    box = np.array([hp.xprd, hp.yprd, hp.zprd])
    eng = D.MdbEngine(torch, mdb, hp, 0, "fp64")
    run = D.SlabRun(D.Slabs(box, hp.cutneigh, 1, 0),
                    D.ThreadTransport(D.ThreadTransport.Hub(1), 0), eng, hp.reneigh_every)
    run.start(x, v, t, np.arange(n))
    run.run(45)
    g, xs, vs, fs = run.gather()
    assert eng.n == n and np.array_equal(np.sort(g), np.arange(n))
    d = np.abs((xs - X[g] + 0.5 * box) % box - 0.5 * box)
    assert d.max() < 1e-10
    assert np.abs(vs - V[g]).max() < 1e-10
    assert np.abs(fs - F[g]).max() <= 1e-9 * scale(F)


def test_halo_entry_points_reject_bad_use():
    torch = pytest.importorskip("torch")
    from test_gpu_vl import EAM_FILE
    tab = mdb.read_funcfl(EAM_FILE)
    hp = mdb.host_params(eam=tab, nx=4, ny=4, nz=4)
    x, v, t = mdb.create_fcc(hp)
    s = mdb.system_from_host(hp, len(t), eam=tab)
    s.set_atoms(x, v, t)
    with pytest.raises(mdb.MdbError):  # EAM would need the F'(rho) exchange
        s.set_owned(len(t) - 10)
    f = mdb.host_params(nx=4, ny=4, nz=4)
    x, v, t = mdb.create_fcc(f)
    s = mdb.system_from_host(f, len(t), pbc=(1, 1, 0))
    s.set_atoms(x, v, t)
    s.set_owned(len(t) - 10)
    buf = torch.zeros((5, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(mdb.MdbError):  # 10 halo atoms, 5 positions
        s.set_halo_positions(buf.data_ptr(), 5)
    s.setup_pbc()
    s.update_pbc()
    s.build_neighbor()
    with pytest.raises(mdb.MdbError):  # halo atoms: the caller drives the steps
        s.run(2)
