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


def compile_facade(src, out, ex):
    pkg = os.path.dirname(ex.LIB_PATH)
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
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
