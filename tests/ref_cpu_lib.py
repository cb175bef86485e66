"""ctypes access to the reference's CPU solvers (test infrastructure).

oracle/_ref/libref_cpu_solvers.so holds lm::rdme::NextSubvolumeSolver and
lm::cme::GillespieDSolver compiled from the reference sources
(oracle/ref_cpu_solvers.cpp).  They are the statistical comparator for
MPD-RDME ensembles and CME ensembles and the timed CPU baseline.  Only
tests/ and bench.py's CPU legs import this module.
"""
import ctypes as C
import os

import numpy as np

from lattice_microbes_b200 import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_ref", "libref_cpu_solvers.so")

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)
f64p = C.POINTER(C.c_double)

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference CPU solvers not built (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        L.ref_nsm_run.restype = C.c_int
        L.ref_nsm_run.argtypes = [
            C.c_uint32, C.c_uint32, u32p, u32p, f64p, i32p, u32p, C.c_uint32, f64p, u32p,
            C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, u8p, u8p,
            C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32, f64p, u32p, u32p, u8p,
            C.c_char_p, C.c_size_t]
        L.ref_record_walls.restype = C.c_uint32
        L.ref_record_walls.argtypes = [f64p, C.c_uint32]
        L.ref_gillespie_run.restype = C.c_int
        L.ref_gillespie_run.argtypes = [
            C.c_uint32, C.c_uint32, u32p, u32p, f64p, C.c_uint32, i32p, u32p, C.c_uint32, C.c_uint32,
            C.c_double, C.c_double, C.c_uint32, f64p, u32p, u32p, C.c_char_p, C.c_size_t]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def row_major(spec):
    """Native word-planar lattice -> row-major [x][y][z][p] uint8 particles and
    [x][y][z] site types (RDMESolver::setLatticeData's input order)."""
    X, Y, Z = spec.X, spec.Y, spec.Z
    slots = configs.native_to_slots(spec.lattice, X, Y, Z, spec.slots, spec.bytes_per_slot)  # [N, S]
    lat = slots.reshape(Z, Y, X, spec.slots).transpose(2, 1, 0, 3)
    sites = spec.sites.reshape(Z, Y, X).transpose(2, 1, 0)
    return (np.ascontiguousarray(lat, dtype=np.uint8).reshape(-1),
            np.ascontiguousarray(sites, dtype=np.uint8).reshape(-1))


def nsm_run(spec, seed, replicate, max_time, write_interval, final_lattice=False):
    """One NextSubvolumeSolver trajectory of `spec` (Byte lattice).  Returns
    (times[E], counts[E, NS]) and, if asked, the final row-major lattice."""
    L = lib()
    if spec.bytes_per_slot != 1:
        raise ValueError("NextSubvolumeSolver runs ByteLattices only")
    lat_rm, sites_rm = row_major(spec)
    ns, nr, nst = spec.ns, spec.nr, spec.nst
    init = configs.species_counts(spec.lattice, spec.nsites, spec.slots, spec.bytes_per_slot, ns)[1:]
    init = np.ascontiguousarray(init, dtype=np.uint32)
    rtype = np.ascontiguousarray(spec.rtype, dtype=np.uint32)
    K = np.ascontiguousarray(spec.K, dtype=np.float64)
    S = np.ascontiguousarray(spec.S, dtype=np.int32).reshape(-1)
    D = np.ascontiguousarray(spec.D, dtype=np.uint32).reshape(-1)
    DF = np.ascontiguousarray(spec.DF, dtype=np.float64).reshape(-1)
    RL = np.ascontiguousarray(spec.RL, dtype=np.uint32).reshape(-1)
    cap = int(max_time / write_interval) + 8
    times = np.zeros(cap, dtype=np.float64)
    counts = np.zeros((cap, ns), dtype=np.uint32)
    entries = np.zeros(1, dtype=np.uint32)
    fin = np.zeros(lat_rm.size, dtype=np.uint8) if final_lattice else None
    err = C.create_string_buffer(512)
    rc = L.ref_nsm_run(ns, nr, _p(init, u32p), _p(rtype, u32p), _p(K, f64p), _p(S, i32p), _p(D, u32p), nst,
                       _p(DF, f64p), _p(RL, u32p), spec.X, spec.Y, spec.Z, spec.slots, spec.spacing,
                       _p(lat_rm, u8p), _p(sites_rm, u8p), seed, replicate, max_time, write_interval, cap,
                       _p(times, f64p), _p(counts, u32p), _p(entries, u32p),
                       _p(fin, u8p) if fin is not None else None, err, 512)
    if rc != 0:
        raise RuntimeError("NextSubvolumeSolver: %s" % err.value.decode())
    n = int(entries[0])
    out = (times[:n], counts[:n])
    return out + (fin,) if final_lattice else out


def record_walls():
    """Wall-clock seconds (steady clock) at which the last trajectory run on
    this thread took each species-count record: entry 0 follows the solver's
    set-up, entry k is the record at k write intervals."""
    L = lib()
    n = L.ref_record_walls(None, 0)
    w = np.zeros(max(n, 1), dtype=np.float64)
    L.ref_record_walls(_p(w, f64p), n)
    return w[:n]


def gillespie_run(ns, rtype, K, S, D, init, seed, replicate, max_time, write_interval):
    """One GillespieDSolver trajectory.  K is [R, k_cols]; S and D are
    species-major [NS, R].  Returns (times[E], counts[E, NS])."""
    L = lib()
    rtype = np.ascontiguousarray(rtype, dtype=np.uint32)
    K = np.ascontiguousarray(np.atleast_2d(np.asarray(K, dtype=np.float64).T).T)
    nr, kcols = K.shape
    Kf = np.ascontiguousarray(K.reshape(-1))
    S = np.ascontiguousarray(S, dtype=np.int32).reshape(-1)
    D = np.ascontiguousarray(D, dtype=np.uint32).reshape(-1)
    init = np.ascontiguousarray(init, dtype=np.uint32)
    cap = int(max_time / write_interval) + 8
    times = np.zeros(cap, dtype=np.float64)
    counts = np.zeros((cap, ns), dtype=np.uint32)
    entries = np.zeros(1, dtype=np.uint32)
    err = C.create_string_buffer(512)
    rc = L.ref_gillespie_run(ns, nr, _p(init, u32p), _p(rtype, u32p), _p(Kf, f64p), kcols, _p(S, i32p),
                             _p(D, u32p), seed, replicate, max_time, write_interval, cap, _p(times, f64p),
                             _p(counts, u32p), _p(entries, u32p), err, 512)
    if rc != 0:
        raise RuntimeError("GillespieDSolver: %s" % err.value.decode())
    n = int(entries[0])
    return times[:n], counts[:n]
