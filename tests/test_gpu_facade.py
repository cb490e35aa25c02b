"""The C++ facade include/exafmm_b200.hpp run on the GPU: a driver in the shape
of examples/fmm.cxx (tests/facade/fmm_driver.cpp) against the engine's own
path on the same bodies.  Same engine, same bounds and trees, so the bodies'
order, the cells and the potentials and gradients agree exactly; the driver's
own check against the direct sum (examples/fmm.cxx:107-124) is reported too."""
import os
import subprocess

import numpy as np
import pytest

from test_facade import compile_facade

pytestmark = pytest.mark.gpu


def read_driver(path):
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(8), np.int64)[0])
        bodies = np.frombuffer(f.read(8 * 9 * n), np.float64).reshape(n, 9)
        nc = int(np.frombuffer(f.read(8), np.int64)[0])
        cells = np.frombuffer(f.read(4 * 5 * nc), np.int32).reshape(nc, 5)
        err = np.frombuffer(f.read(16), np.float64)
    return bodies, cells, err


@pytest.fixture(scope="module")
def driver(ex, tmp_path_factory):
    return compile_facade("fmm_driver.cpp", str(tmp_path_factory.mktemp("facade") / "fmm_driver"), ex,
                          defines=("EXAFMM_COUNT_LIST=1",))


@pytest.mark.parametrize("n,dist,P,theta,ncrit,nspawn,images,inej", [
    (20000, "plummer", 8, 0.35, 32, 5000, 0, 0),
    (6000, "cube", 6, 0.4, 16, 1000, 1, 0),
    (5000, "cube", 6, 0.4, 16, 5000, 0, 1),
])
def test_facade_driver_matches_engine(ex, datasets, driver, tmp_path, n, dist, P, theta, ncrit, nspawn, images, inej):
    out = str(tmp_path / "out.bin")
    r = subprocess.run([driver, out, str(n), dist, str(P), str(theta), str(ncrit), str(nspawn), str(images), str(inej)],
                       capture_output=True, text=True, cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    bodies, cells, err = read_driver(out)
    x = datasets.reference_bodies(n, dist, 0)
    jx = None
    if inej:
        x[:, 0] = (x[:, 0] + np.pi) * 0.5
        jx = datasets.reference_bodies(n, dist, 1)
        jx[:, 0] = (jx[:, 0] - np.pi) * 0.5
    f = ex.Fmm(P=P, theta=theta, ncrit=ncrit, nspawn=nspawn, images=images, cycle=2 * np.pi)
    f.set_bodies(x)
    if inej:
        f.set_sources(jx)
    f.solve()
    trg = f.results()
    perm = f.perm()
    ints, _ = f.cells()
    f.close()
    # the bodies come back in the tree's order, with their IBODY and results
    np.testing.assert_array_equal(bodies[:, 4].astype(np.int64), perm)
    np.testing.assert_array_equal(bodies[:, :4], x[perm])
    np.testing.assert_array_equal(cells, ints)
    np.testing.assert_array_equal(bodies[:, 5:], trg[perm])
    assert os.path.exists(tmp_path / "list000000.dat")
    # the time file: the driver's timer with the engine's phases, as the reference writes it
    names = [ln[:20].rstrip() for ln in (tmp_path / "time000000.dat").read_text().splitlines()]
    assert {"Total FMM", "Get bounds", "Grow tree", "Upward pass", "Traverse", "Downward pass"} <= set(names)
    assert names == sorted(names)
    # examples/fmm.cxx's accuracy check on 100 sampled targets (the method's
    # truncation at these P and theta; images 1 is the 27 nearest cells' sum
    # for both)
    assert err[0] < 1e-3 and err[1] < 1e-2, err


def test_facade_kernel_chain_matches_reference(ex, tmp_path):
    """examples/kernel.cxx's chain through the facade's Kernel, against the
    reference's own values (tests/golden/kernel_kat.npz)."""
    from conftest import GOLDEN, load_golden, rel_l2
    exe = compile_facade("kernel_driver.cpp", str(tmp_path / "kernel_driver"), ex)
    g = load_golden(os.path.join(GOLDEN, "kernel_kat.npz"))
    for P in (4, 8, 10, 14):
        out = str(tmp_path / f"k{P}.bin")
        r = subprocess.run([exe, out, str(P)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        nt = P * (P + 1) // 2
        raw = np.fromfile(out, dtype=np.float64)
        E = raw[:8 * nt].view(np.complex128).reshape(4, nt)
        trg, direct = raw[8 * nt:8 * nt + 4], raw[8 * nt + 4:]
        for k, name in enumerate(("Mj", "MJ", "LI", "Li")):
            ref = g[f"P{P}_{name}"]
            assert np.abs(E[k] - ref).max() <= 1e-13 * np.abs(ref).max(), (P, name)
        assert rel_l2(trg, g[f"P{P}_trg"].reshape(-1)) < 1e-13
        assert rel_l2(direct, g[f"P{P}_direct"].reshape(-1)) < 1e-15


def _rel_errors(stdout):
    vals = {}
    for line in stdout.splitlines():
        if line.startswith("Rel. L2 Error (pot)") or line.startswith("Rel. L2 Error (acc)"):
            vals[line[15:18]] = float(line.split(":")[1])
    return vals


def test_reference_fmm_example_runs_on_the_engine(ex, tmp_path):
    """The reference's examples/fmm.cxx, compiled unchanged against the facade
    (oracle/_ref/examples/fmm), with -n 20000 -P 10 -t 0.4 -c 64 -d c: its own
    accuracy check against the direct sum, its regression files and its timing
    loop run to the end (the driver aborts when a regression fails)."""
    from test_facade import reference_examples
    paths = reference_examples(ex)
    if paths is None:
        pytest.skip("the reference examples were not built (no reference tree at the build step)")
    out = str(tmp_path) + "/"
    r = subprocess.run([paths["fmm"], "-n", "20000", "-P", "10", "-t", "0.4", "-c", "64", "-d", "c", "-v", "-w",
                        "-p", out], capture_output=True, text=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    err = _rel_errors(r.stdout)
    # the method's truncation at P = 10, theta = 0.4 on 100 sampled targets
    assert 0 < err["pot"] < 2e-5 and 0 < err["acc"] < 2e-4, err
    assert "passed accuracy regression" in r.stdout and "passed time regression" in r.stdout
    assert (tmp_path / "accuracy.reg").exists()
    # the driver resets its "Total FMM" timer before writeTime; the engine's phases remain
    names = [ln[:20].rstrip() for ln in (tmp_path / "time000000.dat").read_text().splitlines()]
    assert {"Get bounds", "Grow tree", "Link tree", "Upward pass", "Traverse", "Downward pass"} <= set(names)
    # a second run reads the records the first one wrote and still passes
    r2 = subprocess.run([paths["fmm"], "-n", "20000", "-P", "10", "-t", "0.4", "-c", "64", "-d", "c", "-a", "-v",
                         "-p", out], capture_output=True, text=True, cwd=str(tmp_path), timeout=600)
    assert r2.returncode == 0 and _rel_errors(r2.stdout) == err, r2.stdout[-2000:]


def test_reference_kernel_example_matches_its_known_answers(ex, tmp_path):
    """examples/kernel.cxx (the P2M-M2M-M2L-L2L-L2P chain against P2P) through the
    facade: the printed errors equal the ones the reference's own values give
    (tests/golden/kernel_kat.npz)."""
    from test_facade import reference_examples
    from conftest import GOLDEN, load_golden
    paths = reference_examples(ex)
    if paths is None:
        pytest.skip("the reference examples were not built (no reference tree at the build step)")
    g = load_golden(os.path.join(GOLDEN, "kernel_kat.npz"))
    for P in (4, 8, 10, 14):
        r = subprocess.run([paths["kernel"], "-P", str(P)], capture_output=True, text=True, cwd=str(tmp_path),
                           timeout=120)
        assert r.returncode == 0, r.stderr
        trg, direct = g[f"P{P}_trg"].reshape(-1, 4), g[f"P{P}_direct"].reshape(-1, 4)
        want_pot = np.sqrt(np.sum((trg[:, 0] - direct[:, 0]) ** 2) / np.sum(trg[:, 0] ** 2))
        want_acc = np.sqrt(np.sum((trg[:, 1:] - direct[:, 1:]) ** 2) / np.sum(trg[:, 1:] ** 2))
        # its unconditional line "P pot-error acc-error" (Verify::print is silent unless verbose)
        fields = r.stdout.split()
        assert int(fields[0]) == P, r.stdout
        pot, acc = float(fields[1]), float(fields[2])
        assert abs(pot / want_pot - 1) < 1e-5 and abs(acc / want_acc - 1) < 1e-5, (P, pot, acc, want_pot, want_acc)
    assert len((tmp_path / "kernel.dat").read_text().splitlines()) == 4


def test_reference_tree_example_times_the_engine_build(ex, tmp_path):
    """examples/tree.cxx through the facade: buildTree twice per repeat, with
    the engine's Grow tree / Link tree phases read from logger::timer."""
    from test_facade import reference_examples
    paths = reference_examples(ex)
    if paths is None:
        pytest.skip("the reference examples were not built (no reference tree at the build step)")
    r = subprocess.run([paths["tree"], "-n", "200000", "-r", "3", "-d", "p"], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stderr
    grow = [ln for ln in r.stdout.splitlines() if ln.startswith("Grow1:") or ln.startswith("Grow2:")]
    assert len(grow) == 2
    for ln in grow:
        t = float(ln.split()[1].split("+-")[0])
        assert 0 < t < 1.0, ln
    assert (tmp_path / "time.dat").read_text().split()[0] == "200000"
