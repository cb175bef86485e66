"""Builds the oracle's device tables from a ModelSpec (test infrastructure).

The tables come from the oracle's restatement of the reference's host model
building (MpdRdmeSolver.cu:265-321, :407-421, :697-774); the product builds
its own through the C ABI and tests compare the two.
"""
import ctypes as C

import numpy as np

from tests.oracle_lib import DeviceTables, oracle, f32p, u32p, i8p


def oracle_tables(spec, overflow_capacity=2048):
    lib = oracle()
    ns, nst, nr = spec.ns, spec.nst, spec.nr
    DF = np.ascontiguousarray(spec.DF, dtype=np.float64).reshape(-1)
    T = np.zeros(nst * nst * ns, dtype=np.float32)
    rc = lib.orc_build_T(nst, ns, DF.ctypes.data_as(C.POINTER(C.c_double)), spec.tau, spec.spacing,
                         T.ctypes.data_as(f32p))
    if rc != 0:
        raise ValueError("diffusion coefficient too high for the timestep")
    rate = np.zeros(max(nr, 1), dtype=np.float32)
    qp0 = np.zeros(nst, dtype=np.float32)
    qp1 = np.zeros(nst * ns, dtype=np.float32)
    qp2 = np.zeros(nst * ns * ns, dtype=np.float32)
    order = np.zeros(max(nr, 1), dtype=np.uint32)
    s1, s2 = spec.reactants()
    D1 = np.zeros(max(nr, 1), dtype=np.uint32)
    D2 = np.zeros(max(nr, 1), dtype=np.uint32)
    D1[:nr] = s1
    D2[:nr] = s2
    rtype = np.ascontiguousarray(spec.rtype, dtype=np.uint32)
    K = np.ascontiguousarray(spec.K, dtype=np.float64)
    RL = np.ascontiguousarray(spec.RL, dtype=np.uint32).reshape(-1)
    if nr:
        rc = lib.orc_compute_propensities(ns, nr, nst, rtype.ctypes.data_as(u32p),
                                          K.ctypes.data_as(C.POINTER(C.c_double)), 1,
                                          RL.ctypes.data_as(u32p), spec.tau, spec.X, spec.Y, spec.Z,
                                          rate.ctypes.data_as(f32p), qp0.ctypes.data_as(f32p),
                                          qp1.ctypes.data_as(f32p), qp2.ctypes.data_as(f32p),
                                          order.ctypes.data_as(u32p), D1.ctypes.data_as(u32p),
                                          D2.ctypes.data_as(u32p))
        assert rc == 0
    Sm = np.ascontiguousarray(spec.S, dtype=np.int32).reshape(-1)
    St = np.zeros(max(ns * nr, 1), dtype=np.int8)
    if nr:
        lib.orc_transpose_S(ns, nr, Sm.ctypes.data_as(C.POINTER(C.c_int32)), St.ctypes.data_as(i8p))
    return DeviceTables(spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot, ns, nst, T, qp0, qp1,
                        qp2, order[:nr], D1[:nr], D2[:nr], rate[:nr], St[: ns * nr],
                        RL.astype(np.uint8), overflow_capacity)
