"""Generates the golden MPD-RDME fixtures from the reference's own code.

Run where the reference tree is present (it builds oracle/_ref/ from the
reference sources through oracle/Makefile):

    python tests/golden/make_golden.py

Each fixture holds one seeded problem (device tables, native lattice, site
types, seed, first timestep, step count) and the lattice the reference's
device functions produce for it, run on the CPU by oracle/ref_host_harness.cpp.
hash_kat.npz holds known answers of the reference's device hash
(xor_random_dev.cu:46-81) and of its reaction probability (double exp,
byte_reaction_dev.cu:130-137).
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lattice_microbes_b200 import configs  # noqa: E402
from tests.cases import oracle_tables  # noqa: E402
from tests.oracle_lib import reference, reference_run  # noqa: E402

CASES = [
    # name, generator kwargs, seed, step0, nsteps
    ("byte8_dense", dict(seed=11, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=2.5, nst=2), 501, 0, 12),
    ("byte8_sparse", dict(seed=12, X=64, Y=8, Z=16, slots=8, bytes_per_slot=1, density=0.3, nst=3), 502, 40, 20),
    ("byte16_dense", dict(seed=13, X=32, Y=8, Z=8, slots=16, bytes_per_slot=1, density=4.0, nst=2), 503, 7, 10),
    ("int16_dense", dict(seed=14, X=32, Y=8, Z=8, slots=16, bytes_per_slot=4, density=5.0, nst=3, ns=9), 504, 3, 10),
    ("int8_mixed", dict(seed=15, X=32, Y=16, Z=8, slots=8, bytes_per_slot=4, density=1.5, nst=3), 505, 0, 10),
    ("byte8_diffusion_only", dict(seed=16, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=1.0, nr=0), 506, 100, 25),
]


def build_refs():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref"], check=True)


def make_case(name, kw, seed, step0, nsteps):
    nr = kw.pop("nr", 8)
    spec = configs.random_problem(nr=nr, **kw)
    t = oracle_tables(spec)
    out, rc, ovf, rx = reference_run(t, spec.lattice, spec.sites, seed, step0, nsteps)
    assert rc == 0, (name, rc)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        X=t.X, Y=t.Y, Z=t.Z, slots=t.slots, bytes_per_slot=t.bytes_per_slot, ns=t.ns, nst=t.nst,
        T=t.T, qp0=t.qp0, qp1=t.qp1, qp2=t.qp2, order=t.order[: t.nr], D1=t.D1[: t.nr],
        D2=t.D2[: t.nr], rate=t.rate[: t.nr], S=t.S[: t.nr * t.ns], RL=t.RL[: t.nr * t.nst],
        lattice_in=spec.lattice, sites=spec.sites, seed=seed, step0=step0, nsteps=nsteps,
        lattice_out=out, overflows=ovf, reactions=rx)
    print(name, "overflows", ovf, "reactions", rx)


def make_hash_kat():
    lib = reference("byte", 8)
    rng = np.random.default_rng(2024)
    keys = rng.integers(0, 2 ** 63, size=256, dtype=np.uint64)
    ths = rng.integers(0, 2 ** 63, size=256, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    h = np.array([lib.ref_device_hash(int(k), int(t)) for k, t in zip(keys, ths)], dtype=np.uint32)
    v1 = rng.integers(0, 2 ** 22, size=256, dtype=np.uint32)
    v2 = rng.integers(0, 8, size=256, dtype=np.uint32)
    hf = np.array([lib.ref_device_hash_float(int(a), 3, int(b), int(t)) for a, b, t in zip(v1, v2, ths)],
                  dtype=np.float32)
    rates = np.concatenate([np.exp(rng.uniform(np.log(1e-9), np.log(5.0), size=512)),
                            [1e-30, 1e-12, 2e-4, 0.5, 1.0, 3.0]]).astype(np.float32)
    prob = np.array([lib.ref_reaction_probability(float(r)) for r in rates], dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "hash_kat.npz"), keys=keys, ths=ths, hash=h, v1=v1, v2=v2,
                        hash_float=hf, rates=rates, prob=prob)


if __name__ == "__main__":
    build_refs()
    make_hash_kat()
    for name, kw, seed, step0, nsteps in CASES:
        make_case(name, dict(kw), seed, step0, nsteps)
