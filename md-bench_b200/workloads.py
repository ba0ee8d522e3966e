"""Seeded synthetic workloads of the benchmark configurations.

MD-Bench has no public dataset: its own generators (fcc lattice, Park-Miller
velocities, glibc rand() types; createAtom in verletlist/atom.c:104-246) define
the inputs. The configurations below add what those generators leave open, with
a documented counter-based generator (splitmix64, Steele et al., OOPSLA 2014) so
every value is reproducible without any library's random stream:

* multi-type liquid (``c5_types``): 4 atom types, epsilon_t ~ U[0.5, 1.5] and
  sigma_t ~ U[0.8, 1.2], geometric mixing, cutoff 2.5 sigma_max, written the way
  the reference's types_file holds them (common/parameter.c:126-184, one
  "epsilon sigma" line per type);
* ensemble (``c4_replicas``): replica r of 256 has n = 5 + (h mod 16) fcc cells
  per side (500 to 32,000 atoms), reduced density ~ U[0.75, 0.95] and
  temperature ~ U[0.7, 2.0], with h = splitmix64(r).
"""
MASK64 = (1 << 64) - 1


def splitmix64(x):
    """One splitmix64 output for state x (the state advances by the golden gamma)."""
    z = (x + 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def uniform(h):
    """Uniform double in [0, 1) from the top 53 bits of a 64-bit hash."""
    return (h >> 11) * (1.0 / (1 << 53))


def c5_types(seed=5, ntypes=4):
    """(epsilon_per_type, sigma_per_type) of the multi-type liquid."""
    eps, sig = [], []
    h = splitmix64(seed)
    for _ in range(ntypes):
        h = splitmix64(h)
        eps.append(0.5 + uniform(h))
        h = splitmix64(h)
        sig.append(0.8 + 0.4 * uniform(h))
    return eps, sig


def c5_cutoff(sigma_per_type):
    return 2.5 * max(sigma_per_type)


def write_types_file(path, eps, sig):
    """The reference's types_file format: one 'epsilon sigma' line per type."""
    with open(path, "w") as f:
        f.write("# epsilon sigma (one line per atom type)\n")
        for e, s in zip(eps, sig):
            f.write(f"{e:.17g} {s:.17g}\n")


def c4_replicas(count=256):
    """Per replica: (cells per side, reduced density, temperature)."""
    out = []
    for r in range(count):
        h = splitmix64(r)
        n = 5 + (h % 16)
        h2 = splitmix64(h)
        h3 = splitmix64(h2)
        out.append((int(n), 0.75 + 0.2 * uniform(h2), 0.7 + 1.3 * uniform(h3)))
    return out


def assign_replicas(natoms, nranks):
    """Replicas bin-packed by atom count over nranks GPUs (longest first, each
    to the least-loaded rank, ties to the lower rank): the ensemble's
    multi-GPU split, with no exchange between ranks. Returns one sorted index
    list per rank."""
    load = [0] * nranks
    out = [[] for _ in range(nranks)]
    for i in sorted(range(len(natoms)), key=lambda k: (-natoms[k], k)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += natoms[i]
    return [sorted(o) for o in out]
