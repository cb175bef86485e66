"""Loads the golden fixtures made by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from tests.oracle_lib import DeviceTables

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def case_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not p.endswith("hash_kat.npz"))


def load_case(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: z[k] for k in z.files}
    t = DeviceTables(int(g["X"]), int(g["Y"]), int(g["Z"]), int(g["slots"]), int(g["bytes_per_slot"]),
                     int(g["ns"]), int(g["nst"]), g["T"], g["qp0"], g["qp1"], g["qp2"], g["order"],
                     g["D1"], g["D2"], g["rate"], g["S"], g["RL"])
    return t, g


def load_kat():
    z = np.load(os.path.join(GOLDEN, "hash_kat.npz"))
    return {k: z[k] for k in z.files}
