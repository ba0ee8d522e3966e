"""Generate the golden fixtures in tests/golden/ from the MD-Bench reference itself.

Runs the reference's own Verlet-list sources (compiled from the reference tree
by ``make -C oracle`` into oracle/_ref/libmdbref_vl.so) on small seeded inputs
and stores what they produce, so that tests on machines without the reference
tree (the GPU box) still compare against reference output.

    python tests/golden/make_golden.py       # needs oracle/_ref built

Fixtures (npz):
  lj_full_5x5x5   default LJ case at 5^3 cells, full list: initial state, list
                  (reference order), setup forces, state and thermo after 45 steps
  lj_half_5x5x5   the same with half lists (reference run single-threaded)
  eam_cu_6x6x6    Cu fcc a = 3.615 A at 1600 K written as a dump and read back
                  by the reference (-i file.dmp -f eam), forces, fp and state
                  after 25 steps
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "md-bench_b200"))

import oracle as O  # noqa: E402

EAM = os.path.join(HERE, "data", "Cu_u3.eam")


def cu_dump(path, n=6, a=3.615, temp=1600.0, seed=20241203):
    """Seeded fcc Cu dump (ids 1-based, type 1 as in data/copper_melting)."""
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.array([[i, j, k] for k in range(n) for j in range(n) for i in range(n)])
    x = ((cells[:, None, :] + base[None, :, :]) * a).reshape(-1, 3)
    mass, kb, mvv2e = 63.55, 8.617343e-05, 1.036427e-04
    v = rng.normal(size=x.shape) * np.sqrt(kb * temp / (mass * mvv2e))
    v -= v.mean(axis=0)
    t = np.ones(len(x), dtype=np.int32)
    box = n * a
    with open(path, "w") as f:
        f.write(f"ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n{len(x)}\n")
        f.write("ITEM: BOX BOUNDS pp pp pp\n")
        for _ in range(3):
            f.write(f"0.0 {box:.17g}\n")
        f.write("ITEM: ATOMS id type x y z vx vy vz\n")
        for i in range(len(x)):
            f.write(f"{i + 1} {t[i]} " + " ".join(f"{c:.17g}" for c in (*x[i], *v[i])) + "\n")
    return x, v, t, box


def ordered_list(r):
    nn, nb = r.neighbor_list()
    return nn, nb


def lj(half):
    r = O.RefVL(nx=5, ny=5, nz=5, half=half)
    x0, v0, _, t0 = r.atoms()
    nn, nb = ordered_list(r)
    bm, pb = r.ghosts()
    r.force()
    _, _, f0, _ = r.atoms()
    for n in range(45):
        r.step(n)
    x1, v1, f1, _ = r.atoms()
    th = r.thermo()
    return dict(x0=x0, v0=v0, type=t0, numneigh=nn, neighbors=nb, border_map=bm, pbc=pb,
                f0=f0, x45=x1, v45=v1, f45=f1, T45=th["T"], P45=th["P"])


def eam():
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "cu.dmp")
        x, v, t, box = cu_dump(path)
        r = O.RefVL(force_field=1, input_file=path, eam_file=EAM)
        x0, v0, _, t0 = r.atoms()
        nn, nb = ordered_list(r)
        r.force()
        _, _, f0, _ = r.atoms()
        for n in range(25):
            r.step(n)
        x1, v1, f1, _ = r.atoms()
        th = r.thermo()
    return dict(x0=x0, v0=v0, type=t0, box=np.array([box] * 3), numneigh=nn, neighbors=nb,
                f0=f0, x25=x1, v25=v1, f25=f1, T25=th["T"], P25=th["P"])


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/libmdbref_vl.so missing: run `make -C oracle` with the "
                 "reference tree present")
    np.savez_compressed(os.path.join(HERE, "lj_full_5x5x5.npz"), **lj(0))
    np.savez_compressed(os.path.join(HERE, "lj_half_5x5x5.npz"), **lj(1))
    np.savez_compressed(os.path.join(HERE, "eam_cu_6x6x6.npz"), **eam())
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
