"""ctypes binding of liblmb200.so (declarations in include/lmb.h).

The CUDA library is the only implementation of the solver: if it is missing
or cannot be loaded, importing this module raises.  There is no CPU path.
"""
import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblmb200.so")

LMB_OK = 0
LMB_E_ARG = -1
LMB_E_CUDA = -2
LMB_E_NOMEM = -3
LMB_E_MODEL = -4
LMB_E_STATE = -5
LMB_E_OVERFLOW_EXHAUSTED = -6
LMB_E_OVERFLOW_UNRESOLVED = -7
LMB_E_TIMEOUT = -8
LMB_E_UNSUPPORTED = -9
LMB_E_IO = -10

LMB_OVERFLOW_CLASSIC = 0
LMB_OVERFLOW_RELAXED = 1

LMB_NOALLOC_MAX_SPECIES = 4095

LMB_SCHEDULE_FUSED = 0
LMB_SCHEDULE_PHASES = 1
LMB_SCHEDULE_CLUSTER = 2
LMB_SCHEDULE_GRID = 3
LMB_CME_KERNEL_AUTO = 0
LMB_CME_KERNEL_GENERIC = 1

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i8p = C.POINTER(C.c_int8)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p


class ModelDesc(C.Structure):
    _fields_ = [
        ("number_species", C.c_uint32), ("number_reactions", C.c_uint32),
        ("number_site_types", C.c_uint32), ("reaction_types", u32p), ("K", f64p),
        ("k_cols", C.c_uint32), ("S", i32p), ("D", u32p), ("DF", f64p), ("RL", u32p),
        ("timestep", C.c_double), ("lattice_spacing", C.c_double),
    ]


class Tables(C.Structure):
    _fields_ = [
        ("number_species", C.c_uint32), ("number_reactions", C.c_uint32),
        ("number_site_types", C.c_uint32), ("T", f32p), ("qp0", f32p), ("qp1", f32p),
        ("qp2", f32p), ("order", u32p), ("D1", u32p), ("D2", u32p), ("rate", f32p),
        ("S", i8p), ("RL", u8p),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("steps_done", C.c_uint32), ("failed_step", C.c_uint32),
        ("unresolved", C.c_uint32), ("overflows", C.c_uint64), ("reactions", C.c_uint64),
    ]


class Request(C.Structure):
    _fields_ = [
        ("id", C.c_uint64), ("model", C.POINTER(ModelDesc)), ("X", C.c_uint32), ("Y", C.c_uint32),
        ("Z", C.c_uint32), ("particles", u32p), ("sites", u8p), ("seed", C.c_uint32), ("timesteps", C.c_uint32),
    ]


class ResultInfo(C.Structure):
    _fields_ = [
        ("id", C.c_uint64), ("stats", RunStats), ("X", C.c_uint32), ("Y", C.c_uint32), ("Z", C.c_uint32),
        ("number_species", C.c_uint32), ("t_submit", C.c_double), ("t_admit", C.c_double),
        ("t_done", C.c_double),
    ]


class ServerStatus(C.Structure):
    _fields_ = [
        ("active", C.c_uint32), ("queued", C.c_uint32), ("ready", C.c_uint32), ("peak_active", C.c_uint32),
        ("bytes_in_use", C.c_uint64), ("peak_bytes", C.c_uint64), ("completed", C.c_uint64),
        ("next_ready_words", C.c_uint64),
    ]


# name -> (restype, argtypes); kept in the order of include/lmb.h.
PROTOTYPES = {
    "lmb_abi_version": (C.c_int, []),
    "lmb_status_string": (C.c_char_p, [C.c_int]),
    "lmb_compose_seed": (C.c_uint32, [C.c_uint32, C.c_uint32]),
    "lmb_timestep_hash": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "lmb_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "lmb_ctx_create_on_stream": (C.c_int, [C.c_int, vp, C.POINTER(vp)]),
    "lmb_ctx_destroy": (C.c_int, [vp]),
    "lmb_ctx_stream": (vp, [vp]),
    "lmb_ctx_synchronize": (C.c_int, [vp]),
    "lmb_model_create": (C.c_int, [vp, C.POINTER(ModelDesc), C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.POINTER(vp)]),
    "lmb_tables_build": (C.c_int, [C.POINTER(ModelDesc), C.c_uint32, C.c_uint32, C.c_uint32, f32p, f32p, f32p,
                                   f32p, u32p, u32p, u32p, f32p, i8p, u8p]),
    "lmb_model_create_from_tables": (C.c_int, [vp, C.POINTER(Tables), C.POINTER(vp)]),
    "lmb_model_get_tables": (C.c_int, [vp, f32p, f32p, f32p, f32p, u32p, u32p, u32p, f32p, i8p, u8p]),
    "lmb_model_set_reaction_rate": (C.c_int, [vp, C.c_uint32, C.c_double]),
    "lmb_model_destroy": (C.c_int, [vp]),
    "lmb_lattice_create": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.POINTER(vp)]),
    "lmb_lattice_destroy": (C.c_int, [vp]),
    "lmb_lattice_set_native": (C.c_int, [vp, u32p, u8p]),
    "lmb_lattice_get_native": (C.c_int, [vp, u32p, u8p]),
    "lmb_lattice_set_row_major": (C.c_int, [vp, vp, u8p, C.c_uint32, C.c_uint32]),
    "lmb_lattice_get_row_major": (C.c_int, [vp, vp, u8p]),
    "lmb_lattice_set_schedule": (C.c_int, [vp, C.c_int, C.c_uint32, C.c_uint32]),
    "lmb_lattice_get_schedule": (C.c_int, [vp, C.POINTER(C.c_int), u32p, u32p]),
    "lmb_lattice_autotune": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_int), u32p, u32p,
                                       f32p]),
    "lmb_lattice_device_buffers": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp)]),
    "lmb_lattice_species_counts": (C.c_int, [vp, C.c_uint32, u64p]),
    "lmb_species_counts_noalloc": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.c_uint32, u64p, vp]),
    "lmb_run": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(RunStats)]),
    "lmb_run_async": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int]),
    "lmb_run_wait": (C.c_int, [vp, C.POINTER(RunStats)]),
    "lmb_run_native_async": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, vp, vp, vp]),
    "lmb_run_counts_async": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32]),
    "lmb_run_counts_wait": (C.c_int, [vp, C.POINTER(RunStats), u64p]),
    "lmb_run_profiled": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, f32p, u32p,
                                   C.POINTER(RunStats)]),
    "lmb_batch_create": (C.c_int, [vp, C.c_uint32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "lmb_batch_run": (C.c_int, [vp, u32p, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(RunStats)]),
    "lmb_batch_run_async": (C.c_int, [vp, u32p, C.c_uint32, C.c_uint32, C.c_int]),
    "lmb_batch_wait": (C.c_int, [vp, C.POINTER(RunStats)]),
    "lmb_batch_run_ranges_async": (C.c_int, [vp, u32p, u32p, u32p, C.c_int]),
    "lmb_batch_set_lattices": (C.c_int, [vp, C.c_uint32, C.POINTER(vp), C.POINTER(vp)]),
    "lmb_batch_destroy": (C.c_int, [vp]),
    "lmb_batch_autotune": (C.c_int, [vp, u32p, C.c_uint32, C.c_uint32, f32p]),
    "lmb_batch_plan": (C.c_int, [vp, u32p, u32p]),
    "lmb_server_create": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32,
                                    C.POINTER(vp)]),
    "lmb_server_destroy": (C.c_int, [vp]),
    "lmb_server_submit": (C.c_int, [vp, C.POINTER(Request)]),
    "lmb_server_step": (C.c_int, [vp, u32p, u32p]),
    "lmb_server_pop_result": (C.c_int, [vp, C.POINTER(ResultInfo), u32p, C.c_uint64, u64p, C.c_uint32]),
    "lmb_server_status": (C.c_int, [vp, C.POINTER(ServerStatus)]),
    "lmb_cme_create": (C.c_int, [vp, C.c_uint32, C.c_uint32, u32p, f64p, C.c_uint32, i32p, u32p, C.c_uint32,
                                 C.POINTER(vp)]),
    "lmb_cme_destroy": (C.c_int, [vp]),
    "lmb_cme_set_initial_counts": (C.c_int, [vp, u32p, C.c_int]),
    "lmb_cme_begin": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_double]),
    "lmb_cme_advance_async": (C.c_int, [vp, C.c_double]),
    "lmb_cme_run": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_double]),
    "lmb_cme_entries": (C.c_int, [vp, u32p]),
    "lmb_cme_get_counts": (C.c_int, [vp, u32p]),
    "lmb_cme_device_counts": (C.c_int, [vp, C.POINTER(vp)]),
    "lmb_cme_stats": (C.c_int, [vp, u64p, u32p]),
    "lmb_cme_set_kernel": (C.c_int, [vp, C.c_int]),
    "lmb_kernel_launches": (C.c_uint64, []),
    # include/lmb_lmfile.h
    "lmb_lmfile_create": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "lmb_lmfile_set_parameter": (C.c_int, [vp, C.c_char_p, C.c_char_p]),
    "lmb_lmfile_set_reaction_model": (C.c_int, [vp, C.c_uint32, C.c_uint32, u32p, u32p, f64p, f64p, i32p, u32p]),
    "lmb_lmfile_set_diffusion_model": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32,
                                                 C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, f64p, u32p]),
    "lmb_lmfile_set_diffusion_model_lattice": (C.c_int, [vp, vp, u8p]),
    "lmb_lmfile_append_species_counts": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, f64p, i32p]),
    "lmb_lmfile_append_lattice": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32,
                                            C.c_uint32, C.c_uint32, vp]),
    "lmb_lmfile_append_lattice_device": (C.c_int, [vp, C.c_uint32, C.c_double, vp]),
    "lmb_lmfile_append_sites": (C.c_int, [vp, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32, u8p]),
    "lmb_lmfile_append_sites_device": (C.c_int, [vp, C.c_uint32, C.c_double, vp]),
    "lmb_lmfile_write_max_counts": (C.c_int, [vp, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32]),
    "lmb_lmfile_create_group": (C.c_int, [vp, C.c_char_p]),
    "lmb_lmfile_set_attribute": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_int, C.c_uint32, u64p, vp, C.c_uint32]),
    "lmb_lmfile_write_dataset": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_int, C.c_uint32, u64p, u64p, C.c_int,
                                           C.c_int, vp]),
    "lmb_lmfile_flush": (C.c_int, [vp]),
    "lmb_lmfile_checkpoint": (C.c_int, [vp, C.c_char_p, C.c_uint64]),
    "lmb_lmfile_stats": (C.c_int, [vp, u64p, u64p]),
    "lmb_lmfile_close": (C.c_int, [vp]),
}


class LmbError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib.lmb_status_string(status).decode() if _lib is not None else str(status)
        super().__init__("%s (status %d)%s" % (msg, status, (": " + what) if what else ""))


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("liblmb200.so not built; run `python -m lattice_microbes_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None
_lib = _load()


def lib():
    return _lib


def check(status, what=""):
    if status != LMB_OK:
        raise LmbError(status, what)
    return status
