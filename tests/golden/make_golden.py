"""Generate the golden fixtures in this folder from the reference itself.

The exafmm-beta Laplace headers are compiled in place into
oracle/_ref/libexafmm_ref.so (``make -C oracle ref``) and run here on seeded
inputs; their outputs are stored as compressed .npz files.  The reference
commits no golden values of its own (its .reg regression files are written at
run time), so these fixtures are what pins both the CPU restatement (oracle/)
and the GPU engine to the reference's behaviour.

Run from the repository root, with EXAFMM_REFERENCE_ROOT naming the
exafmm-beta source tree (read only):

    EXAFMM_REFERENCE_ROOT=/root/reference python tests/golden/make_golden.py [solve periodic kat records md inej datasets large]
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


# Records in the reference's file formats: Traversal::writeList (EXAFMM_COUNT_LIST)
# of a tree 19 levels deep (a Plummer sphere plus a tight cluster, so cell keys
# of levels >= 11 wrap as the compiled reference computes them) and of a
# periodic case, and logger::writeTime of fixed events.
RECORD_EVENTS = {"Get bounds": 0.00123, "Grow tree": 1.5e-05, "Link tree": 0.25, "Upward pass": 12.5,
                 "Traverse": 3.0, "Traverse periodic": 0.0, "Downward pass": 1e-07, "Total FMM": 123456.789}


def records_input():
    x = datasets.plummer(5000, 21)
    rng = np.random.default_rng(22)
    c = np.zeros((200, 4))
    c[:, :3] = np.array([0.3, -0.2, 0.1]) + 1e-4 * rng.standard_normal((200, 3))
    c[:, 3] = 1.0 / 5200
    return np.vstack([x, c])


def make_records(ref: Reference):
    import tempfile
    out = {}
    for tag, x, kw in (("deep", records_input(), dict(P=6, theta=0.4, ncrit=8, nspawn=5000, images=0)),
                       ("periodic", datasets.cube(600, 31) * np.array([np.pi, np.pi, np.pi, 1.0]),
                        dict(P=6, theta=0.4, ncrit=16, nspawn=5000, images=2, cycle=2 * np.pi))):
        d = tempfile.mkdtemp() + "/"
        run = ref.solve(x, threads=1, record_lists=False, list_path=d, **kw)
        with open(d + "list000000.dat", "rb") as f:
            text = f.read()
        out[f"{tag}_xyzq"] = x
        out[f"{tag}_params"] = np.array([kw["P"], kw["theta"], kw["ncrit"], kw["nspawn"], kw["images"],
                                         kw.get("cycle", 2 * np.pi)])
        out[f"{tag}_icell"] = run.icell
        out[f"{tag}_cells_real"] = run.cells_real
        out[f"{tag}_list"] = np.frombuffer(text, dtype=np.uint8)
        print(f"records {tag}: cells={len(run.cells_int)} list bytes={len(text)}")
    d = tempfile.mkdtemp() + "/"
    ref.write_time(RECORD_EVENTS, d)
    with open(d + "time000000.dat", "rb") as f:
        out["time_text"] = np.frombuffer(f.read(), dtype=np.uint8)
    out["time_names"] = np.array(list(RECORD_EVENTS.keys()))
    out["time_values"] = np.array(list(RECORD_EVENTS.values()))
    np.savez_compressed(os.path.join(OUT, "records.npz"), **out)


# The MD ABI (wrappers/gromacs.cxx, driven as wrappers/test_gromacs.cxx drives it):
# 1000 random charges with zero net charge in [-cycle/2, cycle/2)^3, cycle = 2 pi,
# images 3, Ewald ksize 11, alpha 10/cycle, sigma 0.25/pi, cutoff cycle/2.  The
# wrapper needs MPI, which is not here, so its single-rank recipe runs through
# the harness: bodies shifted by -cycle/2 and wrapped (vec.h wrap), bounds of
# BoundBox::getBounds narrowed by Partition::octsection with one rank, FMM with
# P 10, theta 0.5, ncrit 32, nspawn 1000 and the dipole correction, and Ewald on
# the wrapped, unshifted bodies.
def md_wrap(X, w):
    X = X.copy()
    for d in range(3):
        lo = X[:, d] < -w / 2
        X[lo, d] += w
        hi = X[:, d] > w / 2
        X[hi, d] -= w
    return X


def make_md(ref: Reference):
    rng = np.random.default_rng(41)
    n = 1000
    cycle32 = np.float32(2 * np.pi)
    x32 = (rng.uniform(size=(n, 3)) * cycle32 - cycle32 / np.float32(2)).astype(np.float32)
    q32 = (rng.uniform(size=n) - 0.5).astype(np.float32)
    q32 = (q32 - np.float32(q32.astype(np.float64).mean())).astype(np.float32)
    c = float(cycle32)
    # FMM_Coulomb's bodies and bounds
    X = md_wrap(x32.astype(np.float64) - c / 2, c)
    xyzq = np.column_stack([X, q32.astype(np.float64)])
    g = ref.solve(xyzq, P=10, theta=0.5, ncrit=32, nspawn=1000, images=0, record_lists=False).bounds
    part = (g[3:] - g[:3]) / 1
    local = np.concatenate([g[:3] + 0 * part, g[:3] + 1 * part])
    fmm = ref.solve(xyzq, P=10, theta=0.5, ncrit=32, nspawn=1000, images=3, cycle=c, bounds=local,
                    record_lists=False, dipole_correction=True)
    # Ewald_Coulomb's bodies
    Xe = md_wrap(x32.astype(np.float64), c)
    ew = ref.ewald(np.column_stack([Xe, q32.astype(np.float64)]), 11, 10 / c, 0.25 / np.pi, c / 2, c)
    # at cutoff L/2 the reference's real part takes each pair's image from its leaf
    # cells' centers and drops some pairs; the nearest-image sum is the oracle's
    from bindings import Oracle
    ew_nearest = Oracle().ewald(np.column_stack([Xe, q32.astype(np.float64)]), 11, 10 / c, 0.25 / np.pi, c / 2, c)
    np.savez_compressed(os.path.join(OUT, "md_gromacs.npz"), x=x32, q=q32, cycle=np.array([c]), bounds=local,
                        perm=fmm.perm, fmm_trg=fmm.trg, ewald_trg=ew, ewald_nearest_trg=ew_nearest)
    e_fmm, e_ew = np.sum(fmm.trg[:, 0] * q32), np.sum(ew[:, 0] * q32)
    acc = np.sqrt(np.sum((fmm.trg[:, 1:] - ew[:, 1:]) ** 2) / np.sum(ew[:, 1:] ** 2))
    print(f"md_gromacs: energy fmm {e_fmm:.8e} ewald {e_ew:.8e} rel {abs(e_fmm - e_ew) / abs(e_ew):.2e}, "
          f"force rel-L2 {acc:.2e}")


# wrappers/md_distributed.cxx's recipe as wrappers/test_md_distributed.cxx drives
# it (images 3, theta 0.4, cutoff L/2, cycle 2 pi, Ewald ksize 11, alpha 10/L,
# sigma 1/(4 pi)) on seeded bodies: the bodies wrapped without a shift,
# Set_Index's tree in the bounds of getBounds, FMM_Partition's in those bounds
# narrowed by the one-rank octsection, FMM_FMM's solve in the latter with the
# dipole correction, and Ewald on the wrapped bodies.
def make_md_distributed(ref: Reference):
    from bindings import Oracle
    rng = np.random.default_rng(43)
    n = 1000
    c = 2 * np.pi
    x = rng.uniform(size=(n, 3)) * c - c / 2
    x[:7] += c * np.array([1.0, -1.0, 0.0])  # a few bodies given at another image
    q = rng.uniform(size=n) - 0.5
    q -= q.mean()
    X = md_wrap(x, c)
    xyzq = np.column_stack([X, q])
    idx = ref.solve(xyzq, P=10, theta=0.4, ncrit=32, nspawn=1000, images=0, record_lists=False)
    g = idx.bounds
    part = (g[3:] - g[:3]) / 1
    local = np.concatenate([g[:3] + 0 * part, g[:3] + 1 * part])
    fmm = ref.solve(xyzq, P=10, theta=0.4, ncrit=32, nspawn=1000, images=3, cycle=c, bounds=local,
                    record_lists=False, dipole_correction=True)
    ew = ref.ewald(xyzq, 11, 10 / c, 0.25 / np.pi, c / 2, c)
    ew_nearest = Oracle().ewald(xyzq, 11, 10 / c, 0.25 / np.pi, c / 2, c)
    np.savez_compressed(os.path.join(OUT, "md_distributed.npz"), x=x, q=q, cycle=np.array([c]),
                        index_bounds=g, index_perm=idx.perm, index_cells=idx.cells_int, bounds=local,
                        perm=fmm.perm, fmm_trg=fmm.trg, ewald_trg=ew, ewald_nearest_trg=ew_nearest)
    e_fmm, e_ew = np.sum(fmm.trg[:, 0] * q), np.sum(ew[:, 0] * q)
    print(f"md_distributed: cells={len(idx.cells_int)} energy fmm {e_fmm:.8e} ewald {e_ew:.8e} "
          f"rel {abs(e_fmm - e_ew) / abs(e_ew):.2e}")


# Separate source bodies (examples/fmm.cxx -j IneJ): (name, target generator, n,
# seed, source generator, n, seed, split, P, theta, ncrit, nspawn).  split applies
# fmm.cxx's transform (targets x -> (x + pi) / 2, sources x -> (x - pi) / 2).
INEJ_CASES = [
    ("inej_split_cube", "cube", 2000, 31, "cube", 1500, 32, True, 6, 0.4, 16, 5000),
    ("inej_overlap_plummer", "plummer", 3000, 33, "plummer", 2500, 34, False, 8, 0.35, 32, 5000),
    ("inej_overlap_cube_nspawn", "cube", 1500, 35, "sphere", 2000, 36, False, 4, 0.5, 8, 100),
]


def make_inej(ref: Reference, name, gen, n, seed, jgen, nj, jseed, split, P, theta, ncrit, nspawn):
    x = getattr(datasets, gen)(n, seed)
    jx = getattr(datasets, jgen)(nj, jseed)
    if split:
        x[:, 0] = (x[:, 0] + np.pi) * 0.5
        jx[:, 0] = (jx[:, 0] - np.pi) * 0.5
    run, (ji, jr, jp) = ref.solve_inej(x, jx, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn)
    data = dict(xyzq=x, jxyzq=jx, params=np.array([P, theta, ncrit, nspawn], dtype=np.float64), bounds=run.bounds,
                perm=run.perm, cells_int=run.cells_int, cells_real=run.cells_real, jcells_int=ji, jcells_real=jr,
                jperm=jp, m2l=sorted_pairs(run.m2l), p2p=sorted_pairs(run.p2p), trg=run.trg)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(f"{name}: cells={len(run.cells_int)} jcells={len(ji)} m2l={len(run.m2l)} p2p={len(run.p2p)}")


# Dataset::initBodies (include/dataset.h:229-257) from the reference compiled
# without fast-math (oracle/_ref/libexafmm_ref_dataset.so):
# (distribution, n, mpirank, mpisize, numSplit).
DATASET_CASES = [("lattice", 1000, 0, 1, 1), ("lattice", 300, 1, 2, 1), ("cube", 1000, 0, 1, 1),
                 ("cube", 997, 2, 1, 3), ("sphere", 1000, 1, 1, 1), ("octant", 1000, 0, 1, 2),
                 ("plummer", 2000, 0, 1, 1), ("plummer", 777, 5, 1, 4)]


def make_datasets():
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libexafmm_ref_dataset.so"))
    lib.ref_dataset_init_bodies.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    lib.ref_drand48.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    data = {}
    for dist, n, rank, size, ns in DATASET_CASES:
        buf = np.zeros((n * size + 8, 4))
        m = lib.ref_dataset_init_bodies(n, dist.encode(), rank, size, ns, buf.ctypes.data, len(buf))
        data[f"{dist}_{n}_{rank}_{size}_{ns}"] = buf[:m].copy()
    d = np.zeros(5000)
    lib.ref_drand48(12345, 5000, d.ctypes.data)
    data["drand48_12345"] = d
    np.savez_compressed(os.path.join(OUT, "datasets_reference.npz"), **data)
    print("datasets_reference:", ", ".join(f"{k} {v.shape}" for k, v in data.items()))


# Large all-positive case (the single large adaptive solve's distribution at a
# size the reference finishes in about a minute on a few cores): the bodies are
# regenerated from the seed at test time (their SHA-256 is stored to check
# that), and the reference's results are kept on 4,096 strided targets plus
# whole-run sums.
# (name, generator, n, seed, P, theta, ncrit, nspawn, sample)
LARGE_CASES = [
    ("large_plummer_n1048576_p8", "plummer", 1 << 20, 77, 8, 0.35, 64, 5000, 4096),
]


def make_large(ref: Reference, name, gen, n, seed, P, theta, ncrit, nspawn, sample):
    import hashlib
    import time
    x = getattr(datasets, gen)(n, seed)
    t0 = time.perf_counter()
    run = ref.solve(x, P=P, theta=theta, ncrit=ncrit, nspawn=nspawn, threads=os.cpu_count() or 1,
                    record_lists=True)
    dt = time.perf_counter() - t0
    idx = datasets.strided_sample(n, sample)
    data = dict(params=np.array([P, theta, ncrit, nspawn], dtype=np.float64), n=np.int64(n), seed=np.int64(seed),
                generator=np.array(gen), xyzq_sha256=np.array(hashlib.sha256(x.tobytes()).hexdigest()),
                bounds=run.bounds, ncells=np.int64(len(run.cells_int)), n_m2l=np.int64(len(run.m2l)),
                n_p2p=np.int64(len(run.p2p)), idx=idx, trg=run.trg[idx],
                pot_sum=np.float64(run.trg[:, 0].sum()), pot_sq_sum=np.float64((run.trg[:, 0] ** 2).sum()),
                acc_sq_sum=np.float64((run.trg[:, 1:] ** 2).sum()))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
    print(f"{name}: cells={len(run.cells_int)} m2l={len(run.m2l)} p2p={len(run.p2p)} ({dt:.1f} s)")


def main(which=("solve", "periodic", "kat", "records", "md", "inej", "datasets", "large")):
    root = os.environ.get("EXAFMM_REFERENCE_ROOT")
    if not root or not os.path.isdir(os.path.join(root, "include")):
        raise SystemExit("set EXAFMM_REFERENCE_ROOT to the exafmm-beta source tree")
    build(reference_root=root, examples=False)
    ref = Reference()
    if "solve" in which:
        for c in CASES:
            make_case(ref, *c)
    if "periodic" in which:
        for c in PERIODIC_CASES:
            make_periodic_case(ref, *c)
    if "kat" in which:
        make_kat(ref)
    if "records" in which:
        make_records(ref)
    if "md" in which:
        make_md(ref)
        make_md_distributed(ref)
    if "inej" in which:
        for c in INEJ_CASES:
            make_inej(ref, *c)
    if "datasets" in which:
        make_datasets()
    if "large" in which:
        for c in LARGE_CASES:
            make_large(ref, *c)


if __name__ == "__main__":
    # optional arguments: a subset of solve, periodic, kat, records, md, inej, datasets, large
    main(tuple(sys.argv[1:]) or ("solve", "periodic", "kat", "records", "md", "inej", "datasets", "large"))
