"""ctypes access to the checkers under oracle/ (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  It loads:
  oracle/libmpd_oracle.so      the C restatement (mpd_oracle.c)
  oracle/_ref/libref_*.so      the reference's device functions built for the
                               host from the reference sources
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
i8p = C.POINTER(C.c_int8)
u8p = C.POINTER(C.c_uint8)


class OrcModel(C.Structure):
    _fields_ = [
        ("X", C.c_uint32), ("Y", C.c_uint32), ("Z", C.c_uint32),
        ("slots", C.c_uint32), ("bytes_per_slot", C.c_uint32),
        ("ns", C.c_uint32), ("nst", C.c_uint32), ("nr", C.c_uint32),
        ("T", f32p), ("qp0", f32p), ("qp1", f32p), ("qp2", f32p),
        ("order", u32p), ("D1", u32p), ("D2", u32p), ("rate", f32p),
        ("S", i8p), ("RL", u8p), ("overflow_capacity", C.c_uint32),
    ]


class OrcStats(C.Structure):
    _fields_ = [("overflows", C.c_uint64), ("reactions", C.c_uint64),
                ("unresolved", C.c_uint64), ("steps_done", C.c_uint32)]


def _ptr(a, t):
    return a.ctypes.data_as(t)


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        path = os.path.join(ORACLE_DIR, "libmpd_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run make -C oracle")
        lib = C.CDLL(path)
        lib.orc_timestep_hash.restype = C.c_uint64
        lib.orc_timestep_hash.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        lib.orc_hash.restype = C.c_uint32
        lib.orc_hash.argtypes = [C.c_uint64, C.c_uint64]
        lib.orc_hash_float.restype = C.c_float
        lib.orc_hash_float.argtypes = [C.c_uint64, C.c_uint64]
        lib.orc_compose_seed.restype = C.c_uint32
        lib.orc_compose_seed.argtypes = [C.c_uint32, C.c_uint32]
        lib.orc_run.restype = C.c_int
        lib.orc_run.argtypes = [C.POINTER(OrcModel), u32p, u8p, C.c_uint32, C.c_uint32,
                                C.c_uint32, C.c_int, C.POINTER(OrcStats)]
        lib.orc_counts.argtypes = [C.POINTER(OrcModel), u32p, u64p]
        lib.orc_build_T.restype = C.c_int
        lib.orc_build_T.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_double), C.c_double,
                                    C.c_double, f32p]
        lib.orc_compute_propensities.restype = C.c_int
        lib.orc_compute_propensities.argtypes = [
            C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.POINTER(C.c_double), C.c_uint32, u32p,
            C.c_double, C.c_uint32, C.c_uint32, C.c_uint32, f32p, f32p, f32p, f32p, u32p, u32p, u32p]
        lib.orc_transpose_S.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_int32), i8p]
        _oracle = lib
    return _oracle


_refs = {}


def reference(kind, slots):
    """The reference's device code built for the host ('byte'|'int', 8|16)."""
    key = (kind, slots)
    if key not in _refs:
        path = os.path.join(REF_DIR, "libref_%s%d.so" % (kind, slots))
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        lib.ref_device_hash.restype = C.c_uint32
        lib.ref_device_hash.argtypes = [C.c_uint64, C.c_uint64]
        lib.ref_device_hash_float.restype = C.c_float
        lib.ref_device_hash_float.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        lib.ref_reaction_probability.restype = C.c_float
        lib.ref_reaction_probability.argtypes = [C.c_float]
        lib.ref_set_model.restype = C.c_int
        lib.ref_set_model.argtypes = [C.c_uint32] * 6 + [f32p, f32p, f32p, f32p, u32p, u32p, u32p,
                                                         f32p, i8p, u8p]
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = [u32p, u8p, u64p, C.c_uint32, u64p, u64p]
        lib.ref_rowmajor_to_native.restype = C.c_int
        lib.ref_rowmajor_to_native.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, u32p]
        lib.ref_particle_counts.restype = C.c_int
        lib.ref_particle_counts.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u64p]
        _refs[key] = lib
    return _refs[key]


class DeviceTables:
    """FP32 device tables of one model + lattice geometry (numpy-owned)."""

    def __init__(self, X, Y, Z, slots, bytes_per_slot, ns, nst, T, qp0, qp1, qp2,
                 order, D1, D2, rate, S, RL, overflow_capacity=2048):
        self.X, self.Y, self.Z = X, Y, Z
        self.slots, self.bytes_per_slot = slots, bytes_per_slot
        self.ns, self.nst = ns, nst
        self.nr = len(order)
        self.T = np.ascontiguousarray(T, dtype=np.float32)
        self.qp0 = np.ascontiguousarray(qp0, dtype=np.float32)
        self.qp1 = np.ascontiguousarray(qp1, dtype=np.float32)
        self.qp2 = np.ascontiguousarray(qp2, dtype=np.float32)
        pad = lambda a, dt: np.ascontiguousarray(a if len(a) else np.zeros(1), dtype=dt)
        self.order = pad(order, np.uint32)
        self.D1 = pad(D1, np.uint32)
        self.D2 = pad(D2, np.uint32)
        self.rate = pad(rate, np.float32)
        self.S = pad(np.asarray(S).reshape(-1), np.int8)
        self.RL = pad(np.asarray(RL).reshape(-1), np.uint8)
        self.overflow_capacity = overflow_capacity

    @property
    def words(self):
        return self.slots // 4 if self.bytes_per_slot == 1 else self.slots

    @property
    def nsites(self):
        return self.X * self.Y * self.Z

    def orc(self):
        m = OrcModel()
        m.X, m.Y, m.Z = self.X, self.Y, self.Z
        m.slots, m.bytes_per_slot = self.slots, self.bytes_per_slot
        m.ns, m.nst, m.nr = self.ns, self.nst, self.nr
        m.T, m.qp0, m.qp1, m.qp2 = (_ptr(self.T, f32p), _ptr(self.qp0, f32p),
                                    _ptr(self.qp1, f32p), _ptr(self.qp2, f32p))
        m.order, m.D1, m.D2 = _ptr(self.order, u32p), _ptr(self.D1, u32p), _ptr(self.D2, u32p)
        m.rate, m.S, m.RL = _ptr(self.rate, f32p), _ptr(self.S, i8p), _ptr(self.RL, u8p)
        m.overflow_capacity = self.overflow_capacity
        return m


def oracle_run(tables, lattice, sites, seed, step0, nsteps, mode=0):
    """Runs the C restatement in place on a copy; returns (lattice, rc, stats)."""
    lat = np.ascontiguousarray(lattice, dtype=np.uint32).copy()
    st = np.ascontiguousarray(sites, dtype=np.uint8)
    m = tables.orc()
    stats = OrcStats()
    rc = oracle().orc_run(C.byref(m), _ptr(lat, u32p), _ptr(st, u8p), seed, step0, nsteps, mode,
                          C.byref(stats))
    return lat, rc, stats


def oracle_counts(tables, lattice):
    m = tables.orc()
    counts = np.zeros(tables.ns + 1, dtype=np.uint64)
    lat = np.ascontiguousarray(lattice, dtype=np.uint32)
    oracle().orc_counts(C.byref(m), _ptr(lat, u32p), _ptr(counts, u64p))
    return counts


def timestep_hashes(seed, step0, nsteps):
    lib = oracle()
    return np.array([lib.orc_timestep_hash(seed, step0 + s, k)
                     for s in range(nsteps) for k in range(4)], dtype=np.uint64)


def reference_run(tables, lattice, sites, seed, step0, nsteps):
    """Runs the host-built reference device functions; None if not built."""
    kind = "byte" if tables.bytes_per_slot == 1 else "int"
    lib = reference(kind, tables.slots)
    if lib is None:
        return None
    t = tables
    rc = lib.ref_set_model(t.X, t.Y, t.Z, t.ns, t.nst, t.nr, _ptr(t.T, f32p), _ptr(t.qp0, f32p),
                           _ptr(t.qp1, f32p), _ptr(t.qp2, f32p), _ptr(t.order, u32p),
                           _ptr(t.D1, u32p), _ptr(t.D2, u32p), _ptr(t.rate, f32p),
                           _ptr(t.S, i8p), _ptr(t.RL, u8p))
    assert rc == 0
    lat = np.ascontiguousarray(lattice, dtype=np.uint32).copy()
    st = np.ascontiguousarray(sites, dtype=np.uint8)
    th = timestep_hashes(seed, step0, nsteps)
    ovf = C.c_uint64(0)
    rx = C.c_uint64(0)
    rc = lib.ref_run(_ptr(lat, u32p), _ptr(st, u8p), _ptr(th, u64p), nsteps, C.byref(ovf), C.byref(rx))
    return lat, rc, ovf.value, rx.value


_refg = {}


def reference_gpu(kind, slots, nofma=False):
    """The reference's device functions compiled for sm_100a (oracle/_ref)."""
    key = (kind, slots, nofma)
    if key not in _refg:
        path = os.path.join(REF_DIR, "libref_gpu_%s%d%s.so" % (kind, slots, "_nofma" if nofma else ""))
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        lib.refg_set_model.restype = C.c_int
        lib.refg_set_model.argtypes = [C.c_uint32] * 6 + [f32p, f32p, f32p, f32p, u32p, u32p, u32p,
                                                          f32p, i8p, u8p]
        lib.refg_supported.restype = C.c_int
        lib.refg_supported.argtypes = [C.c_uint32] * 3
        lib.refg_run.restype = C.c_int
        lib.refg_run.argtypes = [u32p, u8p, u64p, C.c_uint32, u64p]
        lib.refg_time.restype = C.c_int
        lib.refg_time.argtypes = [u32p, u8p, u64p, C.c_uint32, C.POINTER(C.c_double)]
        _refg[key] = lib
    return _refg[key]


def _refg_prepare(tables, nofma=False):
    kind = "byte" if tables.bytes_per_slot == 1 else "int"
    lib = reference_gpu(kind, tables.slots, nofma)
    if lib is None or not lib.refg_supported(tables.X, tables.Y, tables.Z):
        return None
    t = tables
    rc = lib.refg_set_model(t.X, t.Y, t.Z, t.ns, t.nst, t.nr, _ptr(t.T, f32p), _ptr(t.qp0, f32p),
                            _ptr(t.qp1, f32p), _ptr(t.qp2, f32p), _ptr(t.order, u32p), _ptr(t.D1, u32p),
                            _ptr(t.D2, u32p), _ptr(t.rate, f32p), _ptr(t.S, i8p), _ptr(t.RL, u8p))
    assert rc == 0, rc
    return lib


def reference_gpu_run(tables, lattice, sites, seed, step0, nsteps, nofma=False):
    """Replays through the reference kernels on the GPU; None if unavailable."""
    lib = _refg_prepare(tables, nofma)
    if lib is None:
        return None
    lat = np.ascontiguousarray(lattice, dtype=np.uint32).copy()
    st = np.ascontiguousarray(sites, dtype=np.uint8)
    th = timestep_hashes(seed, step0, nsteps)
    ovf = C.c_uint64(0)
    rc = lib.refg_run(_ptr(lat, u32p), _ptr(st, u8p), _ptr(th, u64p), nsteps, C.byref(ovf))
    return lat, rc, ovf.value


def reference_gpu_time(tables, lattice, sites, seed, step0, nsteps):
    """Wall time (ms) of the reference's timestep loop on the GPU."""
    lib = _refg_prepare(tables)
    if lib is None:
        return None
    lat = np.ascontiguousarray(lattice, dtype=np.uint32).copy()
    st = np.ascontiguousarray(sites, dtype=np.uint8)
    th = timestep_hashes(seed, step0, nsteps)
    ms = C.c_double(0)
    rc = lib.refg_time(_ptr(lat, u32p), _ptr(st, u8p), _ptr(th, u64p), nsteps, C.byref(ms))
    return rc, ms.value, lat
