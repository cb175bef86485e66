"""Generates the statistical golden ensembles from the reference's CPU solvers.

Run where the reference tree is present (oracle/Makefile builds
oracle/_ref/libref_cpu_solvers.so from the reference sources):

    python tests/golden/make_ensembles.py

ensembles/nsm_bimolecular_<edge>.npz
    lm::rdme::NextSubvolumeSolver (the reference's exact RDME solver) on the
    bimolecular A + B <-> C model (lattice_microbes_b200.configs.config0) at
    lattice edges 32 and 16: independent replicates (XORShift seeds), species
    counts every 0.05 s to t = 0.5 s (10,000 MPD timesteps of 50 us).
    Replicate k starts from the lattice config0(seed=k + 1, edge), the same
    initial lattices the MPD ensemble tests use.
ensembles/nsm_rodcell.npz
    NextSubvolumeSolver on the rod-cell model (configs.config1: membrane-only
    binding, three site types; no homodimer reaction, whose propensity MPD
    counts differently from NSM), 256 replicates from the lattices
    config1(seed=k + 1), species counts every 5 ms to t = 50 ms (2,000 MPD
    timesteps of 25 us).
ensembles/gillespie_two_state.npz
    lm::cme::GillespieDSolver on the two-state gene model
    (configs.two_state_gene) to t = 3600 s, counts every 600 s.

    python tests/golden/make_ensembles.py [bimolecular] [rodcell] [gillespie]

makes the named sets (all three when none is named).

The MPD and CME ensemble tests compare the GPU ensembles with these counts
(two-sample KS, means within 2 sigma); the reference files do not travel to
the GPU machine, these fixtures do.
"""
import multiprocessing as mp
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ensembles")

NSM_CASES = [  # edge, replicates
    (32, 512),
    (16, 512),
]
NSM_T_END, NSM_DT = 0.5, 0.05
NSM_SEED = 2024
ROD_REPLICATES = 256
ROD_T_END, ROD_DT = 0.05, 0.005
ROD_SEED = 515
GD_REPLICATES = 8192
GD_SEED = 77


def _nsm_worker(args):
    edge, k = args
    sys.path.insert(0, ROOT)
    from lattice_microbes_b200 import configs
    from tests import ref_cpu_lib
    spec = configs.config0(seed=k + 1, edge=edge)
    t, c = ref_cpu_lib.nsm_run(spec, NSM_SEED, k + 1, NSM_T_END, NSM_DT)
    return t, c


def _rod_worker(k):
    sys.path.insert(0, ROOT)
    from lattice_microbes_b200 import configs
    from tests import ref_cpu_lib
    spec = configs.config1(seed=k + 1)
    return ref_cpu_lib.nsm_run(spec, ROD_SEED, k + 1, ROD_T_END, ROD_DT)


def _gd_worker(chunk):
    sys.path.insert(0, ROOT)
    from lattice_microbes_b200 import configs
    from tests import ref_cpu_lib
    m = configs.two_state_gene()
    out = []
    for k in chunk:
        t, c = ref_cpu_lib.gillespie_run(m.ns, m.rtype, m.K, m.S, m.D, m.init, GD_SEED, k + 1, m.max_time,
                                         m.write_interval)
        out.append((t, c))
    return out


def main(which):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    os.makedirs(OUT, exist_ok=True)
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        if "bimolecular" in which:
            for edge, reps in NSM_CASES:
                t0 = time.time()
                res = pool.map(_nsm_worker, [(edge, k) for k in range(reps)])
                times = res[0][0]
                counts = np.stack([r[1] for r in res]).astype(np.uint16)  # [rep, entry, species]
                np.savez_compressed(os.path.join(OUT, "nsm_bimolecular_%d.npz" % edge), times=times,
                                    counts=counts, edge=edge, seed=NSM_SEED, t_end=NSM_T_END)
                print("nsm edge %d: %d replicates in %.1f s" % (edge, reps, time.time() - t0))
        if "rodcell" in which:
            t0 = time.time()
            res = pool.map(_rod_worker, range(ROD_REPLICATES))
            times = res[0][0]
            counts = np.stack([r[1] for r in res]).astype(np.uint16)
            np.savez_compressed(os.path.join(OUT, "nsm_rodcell.npz"), times=times, counts=counts, seed=ROD_SEED,
                                t_end=ROD_T_END)
            print("nsm rod cell: %d replicates in %.1f s" % (ROD_REPLICATES, time.time() - t0))
        if "gillespie" in which:
            t0 = time.time()
            chunks = np.array_split(np.arange(GD_REPLICATES), 64)
            res = [x for part in pool.map(_gd_worker, chunks) for x in part]
            times = res[0][0]
            counts = np.stack([r[1] for r in res]).astype(np.uint32)
            np.savez_compressed(os.path.join(OUT, "gillespie_two_state.npz"), times=times, counts=counts,
                                seed=GD_SEED)
            print("gillespie: %d replicates in %.1f s" % (GD_REPLICATES, time.time() - t0))


if __name__ == "__main__":
    main(set(sys.argv[1:]) or {"bimolecular", "rodcell", "gillespie"})
