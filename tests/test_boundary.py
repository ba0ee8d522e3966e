"""The drop-in boundary seen from the reference's side.

md-bench_b200/host/ref_hooks.c binds MD-Bench's Verlet-list hooks to libmdb and
replaces three reference files (common/device.c, verletlist/force.c,
verletlist/pbc.c) in a link of the reference's own main.c and sources
(oracle/Makefile builds it as oracle/_ref/MDBench-VL-libmdb). CPU tests: the
adapter compiles against the reference's headers with the reference's flags,
defines exactly the symbols of the files it replaces, calls libmdb, and the
linked program depends on libmdb.so. GPU tests: that program, the reference's
own CPU build and this repository's driver MDBench-B200 (graph-captured loop
and per-hook loop) print the same thermo lines on the reference's default case
(fcc 32^3 LJ, 200 steps), which carry the golden values of
tests/sim_copper_fcc_regression.sh:23-26 in the reference.
"""
import os
import re
import subprocess

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOOKS = os.path.join(ROOT, "md-bench_b200", "host", "ref_hooks.c")
LINKED = os.path.join(ROOT, "oracle", "_ref", "MDBench-VL-libmdb")
REF_VL = os.path.join(ROOT, "oracle", "_ref", "MDBench-VL")
DRIVER = os.path.join(ROOT, "md-bench_b200", "MDBench-B200")
# the reference's own strict FP64 build prints these at step 200 (its
# regression test expects 7.961676e-01 / 6.721195e-01 within 1e-4 / 1e-3)
T200, P200 = "7.961535e-01", "6.721076e-01"
REPLACED = ["initDevice", "GPUfree", "allocateGPU", "reallocateGPU", "memcpyToGPU",
            "memcpyFromGPU", "memsetGPU", "computeForce", "initForce", "updatePbc",
            "updateAtomsPbc", "initPbc", "setupPbc", "NmaxGhost", "PBCx", "PBCy", "PBCz"]


def _defined(obj):
    out = subprocess.run(["nm", "-g", "--defined-only", obj], capture_output=True, text=True,
                         check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


def test_adapter_compiles_against_reference_headers(tmp_path):
    tree = O.reference_tree()
    if tree is None:
        pytest.skip("reference tree not present")
    src = os.path.join(tree, "src")
    obj = str(tmp_path / "ref_hooks.o")
    subprocess.run(["gcc", "-c", "-std=c11", "-Wall", "-Werror", "-D_GNU_SOURCE",
                    "-DATOM_POSITION_AOS", "-DNBLIST_AOS", "-DPRECISION=2", "-DLJ_COMB_RULE=1",
                    "-I" + os.path.join(src, "verletlist"), "-I" + os.path.join(src, "common"),
                    "-I" + os.path.join(ROOT, "include"), HOOKS, "-o", obj], check=True)
    assert set(REPLACED) <= _defined(obj)
    undef = subprocess.run(["nm", "-u", obj], capture_output=True, text=True,
                           check=True).stdout
    for entry in ("mdb_create", "mdb_set_atoms", "mdb_setup_pbc", "mdb_update_pbc",
                  "mdb_update_atoms_pbc", "mdb_build_neighbor", "mdb_compute_force",
                  "mdb_initial_integrate", "mdb_final_integrate", "mdb_get_atoms",
                  "mdb_set_eam"):
        assert entry in undef, entry


def test_replaced_files_define_the_same_symbols():
    """The adapter stands in for exactly what the three reference files export
    (checked on objects of the reference files compiled here)."""
    tree = O.reference_tree()
    if tree is None:
        pytest.skip("reference tree not present")
    src = os.path.join(tree, "src")
    flags = ["-std=c11", "-D_GNU_SOURCE", "-DALIGNMENT=64", "-DATOM_POSITION_AOS", "-DNBLIST_AOS",
             "-DPRECISION=2", "-DLJ_COMB_RULE=1", "-I" + os.path.join(src, "verletlist"),
             "-I" + os.path.join(src, "common")]
    import tempfile
    want = set()
    with tempfile.TemporaryDirectory() as d:
        for rel in ("common/device.c", "verletlist/force.c", "verletlist/pbc.c"):
            obj = os.path.join(d, os.path.basename(rel) + ".o")
            subprocess.run(["gcc", "-c"] + flags + [os.path.join(src, rel), "-o", obj],
                           check=True)
            want |= _defined(obj)
    # the reference's CPU kernels of pbc.c (updatePbcCPU, updateAtomsPbcCPU) are
    # not hooks; everything else it exports is provided
    assert want - {"updatePbcCPU", "updateAtomsPbcCPU"} <= set(REPLACED), want


def test_linked_program_depends_on_libmdb():
    if not os.path.exists(LINKED):
        pytest.skip("reference tree not present at build time")
    out = subprocess.run(["readelf", "-d", LINKED], capture_output=True, text=True,
                         check=True).stdout
    assert "libmdb.so" in out


def thermo_lines(text):
    """(step, 'T', 'P') rows of a SIMULATION PROGRESS table."""
    rows = re.findall(r"^\s+(\d+)\s+(\S+e[+-]\d+)\s+(\S+e[+-]\d+)\s*$", text, re.M)
    return [(int(s), t, p) for s, t, p in rows]


def run(cmd, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=e)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


@pytest.mark.gpu
def test_reference_main_with_libmdb_hooks_prints_the_reference_thermo():
    if not os.path.exists(LINKED):
        pytest.skip("reference tree not present at build time")
    ours = thermo_lines(run([LINKED]))
    assert (200, T200, P200) in ours, ours
    if os.path.exists(REF_VL):
        ref = thermo_lines(run([REF_VL], {"OMP_NUM_THREADS": str(os.cpu_count() or 1)}))
        assert ours == ref, (ours, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [[], ["--hooks"]])
def test_driver_prints_the_reference_thermo(mode):
    if not os.path.exists(DRIVER):
        pytest.skip("driver not built")
    ours = thermo_lines(run([DRIVER] + mode))
    assert (200, T200, P200) in ours, ours
