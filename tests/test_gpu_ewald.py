"""Ewald summation on the GPU (exafmm_ewald, include/ewald.h) against the
reference and the C restatement, and the periodic FMM (images = 3, dipole
correction) against it on a small water box."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _box(n, L, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n, 4))
    x[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
    q = rng.uniform(-1, 1, n)
    x[:, 3] = q - q.mean()
    return x


def test_ewald_bins_match_reference(ex, reference):
    L = 2 * np.pi
    x = _box(2000, L, 3)
    kw = dict(ksize=11, alpha=11 / L, sigma=0.25 / np.pi, cutoff=L / 4, cycle=L)  # 4 bins a side
    g = ex.ewald(x, **kw)
    r = reference.ewald(x, ncrit=16, **kw)
    assert rel_l2(g[:, 0], r[:, 0]) < 1e-12
    assert rel_l2(g[:, 1:], r[:, 1:]) < 1e-12


def test_ewald_all_pairs_match_oracle(ex, oracle):
    L = 10.0
    x = _box(1500, L, 4)
    x[:5, :3] += L  # bodies outside the box are taken modulo L
    kw = dict(ksize=9, alpha=0.9, sigma=0.25 / np.pi, cutoff=0.45 * L, cycle=L)  # 2 bins: all-pairs pass
    g = ex.ewald(x, **kw)
    o = oracle.ewald(x, **kw)
    assert rel_l2(g[:, 0], o[:, 0]) < 1e-12
    assert rel_l2(g[:, 1:], o[:, 1:]) < 1e-12


def test_periodic_fmm_matches_ewald_on_water(ex, datasets):
    x, L = datasets.water_box(1000, seed=8)
    f = ex.Fmm(P=10, theta=0.4, ncrit=32, images=3, cycle=L)
    f.set_bodies(x)
    f.solve()
    f.dipole_correction(f.get_dipole())
    fmm = f.results()
    f.close()
    # real part to erfc(3.6) = 4e-7, wave part to exp(-K^2 / 4 alpha^2) = 3e-8 at |k| = 19
    ew = ex.ewald(x, ksize=19, alpha=3.6 / (L / 4), sigma=0.25 / np.pi, cutoff=L / 4, cycle=L)
    q = x[:, 3]
    # potentials differ by a constant: compare the energy sum q.phi (zero net charge) and the forces
    e_fmm, e_ew = float(q @ fmm[:, 0]), float(q @ ew[:, 0])
    assert abs(e_fmm - e_ew) / abs(e_ew) < 1e-4
    assert rel_l2(fmm[:, 1:], ew[:, 1:]) < 1e-3
