"""Generate the golden fixtures in this folder from the reference itself.

The exafmm-beta Laplace headers are compiled in place into
oracle/_ref/libexafmm_ref.so (``make -C oracle ref``) and run here on seeded
inputs; their outputs are stored as compressed .npz files.  The reference
commits no golden values of its own (its .reg regression files are written at
run time), so these fixtures are what pins both the CPU restatement (oracle/)
and the GPU engine to the reference's behaviour.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from bindings import Reference, build  # noqa: E402

spec = importlib.util.spec_from_file_location("exafmm_datasets", os.path.join(ROOT, "exafmm-beta_b200", "datasets.py"))
datasets = importlib.util.module_from_spec(spec)
spec.loader.exec_module(datasets)

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, generator, n, seed, P, theta, ncrit, nspawn, keep expansions)
CASES = [
    ("cube_n2000_p6", "cube", 2000, 11, 6, 0.4, 16, 5000, False),
    ("cube_n500_p6_expansions", "cube", 500, 17, 6, 0.4, 8, 5000, True),
    ("plummer_n3000_p8", "plummer", 3000, 12, 8, 0.35, 32, 5000, False),
    ("sphere_n1500_p10", "sphere", 1500, 13, 10, 0.4, 64, 1000, False),
    ("cube_n1000_p4_nspawn1", "cube", 1000, 14, 4, 0.5, 8, 1, False),
    ("single_body", "cube", 1, 15, 6, 0.4, 64, 5000, True),
    ("root_leaf_n40", "cube", 40, 16, 6, 0.4, 64, 5000, True),
]


def sorted_pairs(p: np.ndarray) -> np.ndarray:
    if len(p) == 0:
        return p.reshape(0, 2)
    order = np.lexsort((p[:, 1], p[:, 0]))
    return p[order]


def make_case(ref: Reference, name, gen, n, seed, P, theta, ncrit, nspawn, keep_exp):
    x = getattr(datasets, gen)(n, seed)
    run = ref.solve(x, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn, threads=1, record_lists=True,
                    expansions=keep_exp)
    data = dict(xyzq=x, params=np.array([P, theta, ncrit, nspawn], dtype=np.float64), bounds=run.bounds,
                perm=run.perm, cells_int=run.cells_int, cells_real=run.cells_real, m2l=sorted_pairs(run.m2l),
                p2p=sorted_pairs(run.p2p), trg=run.trg)
    if keep_exp:
        data["M"] = run.M
        data["L"] = run.L
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(f"{name}: cells={len(run.cells_int)} m2l={len(run.m2l)} p2p={len(run.p2p)}")


def make_kat(ref: Reference):
    """The examples/kernel.cxx chain: P2M -> M2M -> M2L -> L2L -> L2P against P2P."""
    src = np.array([[2.0, 2.0, 2.0, 1.0]])
    tgt = np.array([[-2.0, 2.0, 2.0, 1.0]])
    Xj, XJ, XI, Xi = [3.0, 1.0, 1.0], [4.0, 0.0, 0.0], [-4.0, 0.0, 0.0], [-3.0, 1.0, 1.0]
    data = {}
    for P in (4, 8, 10, 14):
        Mj = ref.p2m(P, Xj, src)
        MJ = ref.m2m(P, XJ, np.array([Xj]), Mj[None, :])
        LI = ref.m2l(P, XI, XJ, MJ)
        Li = ref.l2l(P, Xi, XI, LI)
        trg = ref.l2p(P, Xi, Li, tgt)
        direct = ref.p2p(tgt, src)
        data.update({f"P{P}_Mj": Mj, f"P{P}_MJ": MJ, f"P{P}_LI": LI, f"P{P}_Li": Li, f"P{P}_trg": trg,
                     f"P{P}_direct": direct})
    np.savez_compressed(os.path.join(OUT, "kernel_kat.npz"), **data)
    print("kernel_kat: P in (4, 8, 10, 14)")


# Periodic systems (Traversal::traverse with images, traversePeriodic and
# UpDownPass::dipoleCorrection): bodies in the reference's box [-pi, pi]^3,
# cycle 2 pi.  (name, generator, n, seed, P, theta, ncrit, nspawn, images)
PERIODIC_CASES = [
    ("periodic_cube_n600_p6_images2", "cube", 600, 21, 6, 0.4, 16, 5000, 2),
    ("periodic_cube_n800_p8_images3", "cube", 800, 22, 8, 0.4, 32, 5000, 3),
]


def make_periodic_case(ref: Reference, name, gen, n, seed, P, theta, ncrit, nspawn, images):
    x = getattr(datasets, gen)(n, seed)
    x[:, :3] *= np.pi
    cycle = 2 * np.pi
    run = ref.solve(x, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn, images=images, cycle=cycle, threads=1,
                    record_lists=True, dipole_correction=True)
    nc = len(run.cells_int)
    # the log also holds traversePeriodic's M2Ls from temporary cells outside the tree
    lattice = (run.m2l[:, 1] >= nc) | (run.m2l[:, 1] < 0)
    data = dict(xyzq=x, params=np.array([P, theta, ncrit, nspawn, images, cycle], dtype=np.float64),
                bounds=run.bounds, perm=run.perm, cells_int=run.cells_int, cells_real=run.cells_real,
                m2l=sorted_pairs(run.m2l[~lattice]), p2p=sorted_pairs(run.p2p), trg=run.trg,
                n_lattice=np.array([lattice.sum()]))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(f"{name}: cells={nc} m2l={len(data['m2l'])} (+{lattice.sum()} lattice) p2p={len(run.p2p)}")


def main():
    build(reference=True)
    ref = Reference()
    for c in CASES:
        make_case(ref, *c)
    for c in PERIODIC_CASES:
        make_periodic_case(ref, *c)
    make_kat(ref)


if __name__ == "__main__":
    main()
