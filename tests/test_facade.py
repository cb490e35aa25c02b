"""The C++ facade include/exafmm_b200.hpp (the reference's classes over the C
ABI): a driver in the shape of examples/fmm.cxx compiles and links against it,
and its Dataset reproduces the reference's generators bit for bit (pinned by
tests/golden/datasets_reference.npz).  CPU only: nothing here opens the GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def compile_facade(src, out, ex, defines=()):
    pkg = os.path.dirname(ex.LIB_PATH)
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           *[f"-D{d}" for d in defines],
           os.path.join(HERE, "facade", src), "-L", pkg, "-lexafmm_b200", f"-Wl,-rpath,{pkg}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("src", ["fmm_driver.cpp", "kernel_driver.cpp"])
def test_drivers_compile_and_link(ex, tmp_path, src):
    exe = compile_facade(src, str(tmp_path / src[:-4]), ex)
    assert os.path.exists(exe)


def test_facade_dataset_matches_reference(ex, tmp_path):
    exe = compile_facade("dataset_dump.cpp", str(tmp_path / "dump"), ex)
    with np.load(os.path.join(GOLDEN, "datasets_reference.npz")) as z:
        gold = {k: z[k] for k in z.files if not k.startswith("drand48")}
    for key, ref in gold.items():
        dist, n, rank, size, ns = key.split("_")
        out = str(tmp_path / f"{key}.bin")
        subprocess.run([exe, out, n, dist, rank, size, ns], check=True)
        mine = np.fromfile(out, dtype=np.float64).reshape(-1, 4)
        assert mine.shape == ref.shape, key
        np.testing.assert_array_equal(mine, ref, err_msg=key)


def test_facade_verify_regression_matches_reference(ex, tmp_path, monkeypatch):
    """Verify::regression of the facade against the reference's own
    (include/verify.h:118-175, compiled in oracle/_ref/libexafmm_ref_dataset.so):
    the same pass / fail answers and byte-identical regression files over a
    sequence of accuracy (two values) and time calls on one object."""
    import ctypes
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libexafmm_ref_dataset.so")
    if not os.path.exists(ref_path):
        pytest.skip("oracle/_ref was not built here (needs the reference tree)")
    lib = ctypes.CDLL(ref_path)
    lib.ref_verify_sequence.argtypes = [ctypes.c_char_p, ctypes.c_int] + [ctypes.c_void_p] * 6
    monkeypatch.setenv("WORKERNAME", "box")
    calls = [  # key, time, iteration, value, value2
        (3, 0, 0, 1e-5, 2e-4), (3, 0, 1, 1.05e-5, 2.1e-4), (3, 0, 2, 9e-5, 2e-4), (77, 0, 0, 6e-4, 1e-4),
        (77, 0, 0, 3e-4, 6e-3), (3, 0, 0, 1e-5, 1e-4), (12345678901, 0, 3, 2e-6, 3e-5),
        (5, 1, 0, 0.25, 0.0), (5, 1, 1, 0.24, 0.0), (5, 1, 0, 0.5, 0.0), (9, 1, 2, 1.5, 0.0), (5, 1, 0, 0.2, 0.0),
    ]
    ref_dir, my_dir = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    my_dir.mkdir()
    keys = np.array([c[0] for c in calls], np.uint64)
    tm = np.array([c[1] for c in calls], np.int32)
    it = np.array([c[2] for c in calls], np.int32)
    v = np.array([c[3] for c in calls])
    v2 = np.array([c[4] for c in calls])
    ref_pass = np.zeros(len(calls), np.int32)
    lib.ref_verify_sequence((str(ref_dir) + "/").encode(), len(calls), keys.ctypes.data, tm.ctypes.data,
                            it.ctypes.data, v.ctypes.data, v2.ctypes.data, ref_pass.ctypes.data)
    exe = compile_facade("verify_driver.cpp", str(tmp_path / "verify_driver"), ex)
    args = [exe, str(my_dir) + "/"]
    for c in calls:
        args += [str(c[0]), str(c[1]), str(c[2]), repr(c[3]), repr(c[4])]
    out = subprocess.run(args, capture_output=True, text=True, check=True).stdout.split()
    assert [int(t) for t in out] == ref_pass.tolist()
    assert 0 < ref_pass.sum() < len(calls)  # both outcomes exercised
    for name in ("accuracy.reg", "time_box.reg"):
        assert (my_dir / name).read_bytes() == (ref_dir / name).read_bytes(), name


def test_facade_logger_time_file(ex, tmp_path):
    """logger's timers accumulate per event and writeTime writes them in the
    reference's time file format (the same writer as exafmm_write_time,
    byte-compared with the reference in test_gpu_records.py), then clears."""
    exe = compile_facade("logger_driver.cpp", str(tmp_path / "logger_driver"), ex)
    subprocess.run([exe, str(tmp_path) + "/"], check=True)
    lines = (tmp_path / "time000002.dat").read_text().splitlines()
    names = [ln[:20].rstrip() for ln in lines]
    vals = [float(ln[21:]) for ln in lines]
    assert names == ["Direct sum", "Total FMM"]
    assert 0.015 < vals[0] < 0.5 and 0.05 < vals[1] < 1.0
    assert (tmp_path / "time000003.dat").read_text() == ""
    # another name width: the file follows logger::stringLength, as the reference's does
    wide = tmp_path / "wide"
    wide.mkdir()
    subprocess.run([exe, str(wide) + "/", "26"], check=True)
    lines = (wide / "time000002.dat").read_text().splitlines()
    assert [ln[:26].rstrip() for ln in lines] == ["Direct sum", "Total FMM"]
    assert all(ln[26] == " " and float(ln[27:]) > 0 for ln in lines)


EXAMPLES = ("fmm", "kernel", "tree")


def reference_examples(ex):
    """The reference's examples/{fmm,kernel,tree}.cxx compiled unchanged against the
    facade (oracle/Makefile `examples`): built here when EXAFMM_REFERENCE_ROOT names
    the exafmm-beta tree, else taken as built by the build step; None if absent."""
    sys_path = os.path.join(ROOT, "oracle")
    root = os.environ.get("EXAFMM_REFERENCE_ROOT")
    if root and os.path.isdir(os.path.join(root, "examples")):
        subprocess.run(["make", "-s", "-C", sys_path, "examples", f"REFERENCE_ROOT={root}"], check=True)
    paths = {e: os.path.join(sys_path, "_ref", "examples", e) for e in EXAMPLES}
    return paths if all(os.path.exists(p) for p in paths.values()) else None


def test_reference_examples_build_against_the_facade(ex):
    """examples/fmm.cxx, kernel.cxx and tree.cxx, unmodified, compile against
    include/exafmm_compat/ + the facade and link only the engine library."""
    paths = reference_examples(ex)
    if paths is None:
        pytest.skip("the reference tree was not available to the build step")
    for name, p in paths.items():
        assert os.access(p, os.X_OK), name
        libs = subprocess.run(["ldd", p], capture_output=True, text=True).stdout
        assert "libexafmm_b200.so" in libs and "not found" not in libs, (name, libs)


def test_facade_args_match_the_reference_command_line(ex, tmp_path):
    """Args: the reference's options, defaults and getKey, exercised by a driver."""
    exe = compile_facade("args_driver.cpp", str(tmp_path / "args_driver"), ex)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    d = dict(zip(out[0::2], out[1::2]))
    assert d == {"ncrit": "64", "P": "10", "theta": "0.4", "numBodies": "1000000", "distribution": "cube",
                 "images": "0", "nspawn": "5000", "threads": "16", "repeat": "1", "dual": "0", "IneJ": "0",
                 "path": "./", "verbose": "0", "key": str(_reference_key(64, "c", 0, 0, 0, 1000000, 10, 5000, 0.4, 16))}
    argv = ["-n", "20000", "-P", "8", "-t", "0.35", "-c", "32", "-d", "p", "-i", "2", "-s", "1000", "-j", "-D", "-r",
            "3", "-T", "4", "-v", "--path", "out/"]
    out = subprocess.run([exe, *argv], capture_output=True, text=True, check=True).stdout.split()
    d = dict(zip(out[0::2], out[1::2]))
    assert (d["numBodies"], d["P"], d["theta"], d["ncrit"], d["distribution"], d["images"], d["nspawn"], d["IneJ"],
            d["dual"], d["repeat"], d["threads"], d["verbose"], d["path"]) == \
        ("20000", "8", "0.35", "32", "plummer", "2", "1000", "1", "1", "3", "4", "1", "out/")
    assert d["key"] == str(_reference_key(32, "p", 1, 2, 1, 20000, 8, 1000, 0.35, 4))
    bad = subprocess.run([exe, "-x"], capture_output=True, text=True)
    assert bad.returncode != 0 and "Usage" in bad.stderr


def _reference_key(ncrit, dist, dual, images, inej, n, P, nspawn, theta, threads):
    """include/args.h getKey bit layout (Laplace, no build switches, one rank)."""
    lg = lambda v, b: int(round(np.log(v) / np.log(b)))
    code = {"c": 0, "l": 1, "o": 2, "p": 3, "s": 4}[dist]
    return (lg(ncrit, 2) | code << 4 | dual << 7 | images << 12 | inej << 14 | lg(n, 10) << 15 | P << 19
            | lg(nspawn, 10) << 25 | int(theta * 14) << 28 | lg(threads, 2) << 31)
