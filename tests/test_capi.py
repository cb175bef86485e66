"""The C ABI library on the CPU: it loads, it exports every entry point that
include/lmb.h declares, and its host-only pieces agree with the oracle.
No device work is done here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.oracle_lib import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(lmb_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from lattice_microbes_b200 import _lib as L
    lib = C.CDLL(L.LIB_PATH)
    declared = declared_entry_points()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    # The Python binding covers each of them too.
    assert not [n for n in declared if n not in L.PROTOTYPES], "binding out of date"


def test_binding_constants_equal_the_header():
    """Every integer LMB_* constant the Python binding defines has the value
    include/lmb.h gives it, and the header's schedules, status codes and
    overflow modes are all bound."""
    from lattice_microbes_b200 import _lib as L
    text = open(os.path.join(ROOT, "include", "lmb.h")).read()
    header = {n: int(v) for n, v in re.findall(r"#define\s+(LMB_\w+)\s+\(?(-?\d+)\)?", text)}
    assert len(header) >= 20
    for name, value in header.items():
        if hasattr(L, name):
            assert getattr(L, name) == value, name
    for prefix in ("LMB_SCHEDULE_", "LMB_E_", "LMB_OVERFLOW_"):
        unbound = [n for n in header if n.startswith(prefix) and not hasattr(L, n)]
        assert not unbound, unbound


def test_abi_version_and_status_strings():
    from lattice_microbes_b200 import _lib as L
    assert L.lib().lmb_abi_version() == 1
    assert b"overflow" in L.lib().lmb_status_string(L.LMB_E_OVERFLOW_EXHAUSTED)
    assert b"available site" in L.lib().lmb_status_string(L.LMB_E_OVERFLOW_UNRESOLVED)


def test_seed_and_timestep_hash_match_oracle():
    from lattice_microbes_b200 import _lib as L
    orc = oracle()
    for seed in (0, 1, 0xFFFFFFFF, 123456789):
        for step in (0, 1, 77, 2 ** 31 + 5):
            for sub in range(4):
                assert L.lib().lmb_timestep_hash(seed, step, sub) == orc.orc_timestep_hash(seed, step, sub)
    assert L.lib().lmb_compose_seed(0x10001, 0x12345) == orc.orc_compose_seed(0x10001, 0x12345)


def _build_tables(spec):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import _p
    ns, nst, nr = spec.ns, spec.nst, spec.nr
    keep = dict(rtype=np.ascontiguousarray(spec.rtype, np.uint32), K=np.ascontiguousarray(spec.K, np.float64),
                S=np.ascontiguousarray(spec.S, np.int32).reshape(-1),
                D=np.ascontiguousarray(spec.D, np.uint32).reshape(-1),
                DF=np.ascontiguousarray(spec.DF, np.float64).reshape(-1),
                RL=np.ascontiguousarray(spec.RL, np.uint32).reshape(-1))
    d = L.ModelDesc()
    d.number_species, d.number_reactions, d.number_site_types = ns, nr, nst
    d.reaction_types, d.K, d.k_cols = _p(keep["rtype"], L.u32p), _p(keep["K"], L.f64p), 1
    d.S, d.D = _p(keep["S"], L.i32p), _p(keep["D"], L.u32p)
    d.DF, d.RL = _p(keep["DF"], L.f64p), _p(keep["RL"], L.u32p)
    d.timestep, d.lattice_spacing = spec.tau, spec.spacing
    out = dict(T=np.zeros(nst * nst * ns, np.float32), qp0=np.zeros(nst, np.float32),
               qp1=np.zeros(nst * ns, np.float32), qp2=np.zeros(nst * ns * ns, np.float32),
               order=np.zeros(nr, np.uint32), D1=np.zeros(nr, np.uint32), D2=np.zeros(nr, np.uint32),
               rate=np.zeros(nr, np.float32), S=np.zeros(nr * ns, np.int8), RL=np.zeros(nr * nst, np.uint8))
    rc = L.lib().lmb_tables_build(C.byref(d), spec.X, spec.Y, spec.Z, _p(out["T"], L.f32p), _p(out["qp0"], L.f32p),
                                  _p(out["qp1"], L.f32p), _p(out["qp2"], L.f32p), _p(out["order"], L.u32p),
                                  _p(out["D1"], L.u32p), _p(out["D2"], L.u32p), _p(out["rate"], L.f32p),
                                  _p(out["S"], L.i8p), _p(out["RL"], L.u8p))
    return rc, out


@pytest.mark.parametrize("maker", [
    lambda: configs.config0(seed=1),
    lambda: configs.config1(seed=1, X=32, Y=32, Z=64),
    lambda: configs.random_problem(3, X=16, Y=8, Z=8, nr=12),
    lambda: configs.random_problem(4, X=16, Y=8, Z=8, slots=16, bytes_per_slot=4, ns=9, nr=20),
])
def test_model_tables_match_oracle(maker):
    spec = maker()
    rc, ours = _build_tables(spec)
    assert rc == 0
    ref = oracle_tables(spec)
    for k in ("T", "qp0", "qp1", "qp2"):
        assert np.array_equal(ours[k], getattr(ref, k)), k
    for k in ("order", "D1", "D2", "rate", "S", "RL"):
        assert np.array_equal(ours[k], getattr(ref, k)[: len(ours[k])]), k


def test_model_rejects_fast_diffusion_and_bad_dependencies():
    from lattice_microbes_b200 import _lib as L
    spec = configs.config0(seed=1)
    spec.DF = spec.DF * 1e6  # q far above 0.5 (MpdRdmeSolver.cu:415-421)
    rc, _ = _build_tables(spec)
    assert rc == L.LMB_E_MODEL
    spec = configs.config0(seed=1)
    spec.D = spec.D.copy()
    spec.D[2, 0] = 1  # a second-order reaction with three reactants
    rc, _ = _build_tables(spec)
    assert rc == L.LMB_E_MODEL


def test_context_without_device_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from lattice_microbes_b200 import _lib as L
    h = L.vp()
    assert L.lib().lmb_ctx_create(0, C.byref(h)) in (L.LMB_E_CUDA, L.LMB_E_ARG)
