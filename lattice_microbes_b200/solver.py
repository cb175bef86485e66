"""Python face of the C ABI: contexts, models, lattices and timestep runs.

This mirrors the pieces of the reference's ``lm`` module the MPD-RDME path
uses (a solver's model upload, its CUDA lattice and ``runTimestep`` loop); the
work happens in liblmb200.so.
"""
import ctypes as C

import numpy as np

from lattice_microbes_b200 import _lib as L


def _p(a, t):
    return a.ctypes.data_as(t)


class Context:
    """One device and one CUDA stream (lmb_ctx)."""

    def __init__(self, device=0, stream=None):
        h = L.vp()
        if stream is None:
            L.check(L.lib().lmb_ctx_create(device, C.byref(h)), "lmb_ctx_create")
        else:
            L.check(L.lib().lmb_ctx_create_on_stream(device, C.c_void_p(stream), C.byref(h)),
                    "lmb_ctx_create_on_stream")
        self.handle = h
        self.device = device

    @property
    def stream(self):
        return L.lib().lmb_ctx_stream(self.handle)

    def synchronize(self):
        L.check(L.lib().lmb_ctx_synchronize(self.handle))

    def close(self):
        if self.handle:
            L.lib().lmb_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Model:
    """Device model tables (lmb_model)."""

    def __init__(self, ctx, handle, ns, nst, nr):
        self.ctx, self.handle = ctx, handle
        self.ns, self.nst, self.nr = ns, nst, nr

    @classmethod
    def from_spec(cls, ctx, spec):
        """Builds from reference-style inputs (a configs.ModelSpec or any
        object with the same fields)."""
        ns, nst, nr = spec.ns, spec.nst, spec.nr
        keep = dict(
            rtype=np.ascontiguousarray(spec.rtype, dtype=np.uint32) if nr else np.zeros(1, np.uint32),
            K=np.ascontiguousarray(spec.K, dtype=np.float64) if nr else np.zeros(1),
            S=np.ascontiguousarray(spec.S, dtype=np.int32).reshape(-1) if nr else np.zeros(1, np.int32),
            D=np.ascontiguousarray(spec.D, dtype=np.uint32).reshape(-1) if nr else np.zeros(1, np.uint32),
            DF=np.ascontiguousarray(spec.DF, dtype=np.float64).reshape(-1),
            RL=np.ascontiguousarray(spec.RL, dtype=np.uint32).reshape(-1) if nr else np.zeros(1, np.uint32),
        )
        d = L.ModelDesc()
        d.number_species, d.number_reactions, d.number_site_types = ns, nr, nst
        d.reaction_types = _p(keep["rtype"], L.u32p)
        d.K = _p(keep["K"], L.f64p)
        d.k_cols = 1
        d.S = _p(keep["S"], L.i32p)
        d.D = _p(keep["D"], L.u32p)
        d.DF = _p(keep["DF"], L.f64p)
        d.RL = _p(keep["RL"], L.u32p)
        d.timestep = spec.tau
        d.lattice_spacing = spec.spacing
        h = L.vp()
        L.check(L.lib().lmb_model_create(ctx.handle, C.byref(d), spec.X, spec.Y, spec.Z, C.byref(h)),
                "lmb_model_create")
        return cls(ctx, h, ns, nst, nr)

    @classmethod
    def from_tables(cls, ctx, t):
        """From ready FP32 tables (an object with T, qp0.. RL arrays)."""
        arrs = dict(T=np.ascontiguousarray(t.T, np.float32), qp0=np.ascontiguousarray(t.qp0, np.float32),
                    qp1=np.ascontiguousarray(t.qp1, np.float32), qp2=np.ascontiguousarray(t.qp2, np.float32),
                    order=np.ascontiguousarray(t.order, np.uint32), D1=np.ascontiguousarray(t.D1, np.uint32),
                    D2=np.ascontiguousarray(t.D2, np.uint32), rate=np.ascontiguousarray(t.rate, np.float32),
                    S=np.ascontiguousarray(t.S, np.int8), RL=np.ascontiguousarray(t.RL, np.uint8))
        tb = L.Tables()
        tb.number_species, tb.number_reactions, tb.number_site_types = t.ns, t.nr, t.nst
        tb.T, tb.qp0, tb.qp1, tb.qp2 = (_p(arrs["T"], L.f32p), _p(arrs["qp0"], L.f32p),
                                        _p(arrs["qp1"], L.f32p), _p(arrs["qp2"], L.f32p))
        tb.order, tb.D1, tb.D2 = _p(arrs["order"], L.u32p), _p(arrs["D1"], L.u32p), _p(arrs["D2"], L.u32p)
        tb.rate, tb.S, tb.RL = _p(arrs["rate"], L.f32p), _p(arrs["S"], L.i8p), _p(arrs["RL"], L.u8p)
        h = L.vp()
        L.check(L.lib().lmb_model_create_from_tables(ctx.handle, C.byref(tb), C.byref(h)),
                "lmb_model_create_from_tables")
        return cls(ctx, h, t.ns, t.nst, t.nr)

    def tables(self):
        ns, nst, nr = self.ns, self.nst, self.nr
        out = dict(T=np.zeros(nst * nst * ns, np.float32), qp0=np.zeros(nst, np.float32),
                   qp1=np.zeros(nst * ns, np.float32), qp2=np.zeros(nst * ns * ns, np.float32),
                   order=np.zeros(max(nr, 1), np.uint32), D1=np.zeros(max(nr, 1), np.uint32),
                   D2=np.zeros(max(nr, 1), np.uint32), rate=np.zeros(max(nr, 1), np.float32),
                   S=np.zeros(max(nr * ns, 1), np.int8), RL=np.zeros(max(nr * nst, 1), np.uint8))
        L.check(L.lib().lmb_model_get_tables(
            self.handle, _p(out["T"], L.f32p), _p(out["qp0"], L.f32p), _p(out["qp1"], L.f32p),
            _p(out["qp2"], L.f32p), _p(out["order"], L.u32p), _p(out["D1"], L.u32p), _p(out["D2"], L.u32p),
            _p(out["rate"], L.f32p), _p(out["S"], L.i8p), _p(out["RL"], L.u8p)))
        for k in ("order", "D1", "D2", "rate"):
            out[k] = out[k][:nr]
        out["S"] = out["S"][: nr * ns]
        out["RL"] = out["RL"][: nr * nst]
        return out

    def set_reaction_rate(self, reaction, rate):
        L.check(L.lib().lmb_model_set_reaction_rate(self.handle, reaction, rate))

    def close(self):
        if self.handle:
            L.lib().lmb_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """Device lattice (lmb_lattice): two particle buffers + site types."""

    def __init__(self, ctx, X, Y, Z, slots, bytes_per_slot):
        h = L.vp()
        L.check(L.lib().lmb_lattice_create(ctx.handle, X, Y, Z, slots, bytes_per_slot, C.byref(h)),
                "lmb_lattice_create")
        self.ctx, self.handle = ctx, h
        self.X, self.Y, self.Z = X, Y, Z
        self.slots, self.bytes_per_slot = slots, bytes_per_slot
        self.words = slots // 4 if bytes_per_slot == 1 else slots

    @property
    def nsites(self):
        return self.X * self.Y * self.Z

    def set_native(self, particles=None, sites=None):
        p = None if particles is None else np.ascontiguousarray(particles, dtype=np.uint32)
        s = None if sites is None else np.ascontiguousarray(sites, dtype=np.uint8)
        if p is not None and p.size != self.words * self.nsites:
            raise ValueError("particle array size")
        if s is not None and s.size != self.nsites:
            raise ValueError("site array size")
        L.check(L.lib().lmb_lattice_set_native(self.handle, None if p is None else _p(p, L.u32p),
                                               None if s is None else _p(s, L.u8p)))

    def get_native(self):
        p = np.zeros(self.words * self.nsites, dtype=np.uint32)
        s = np.zeros(self.nsites, dtype=np.uint8)
        L.check(L.lib().lmb_lattice_get_native(self.handle, _p(p, L.u32p), _p(s, L.u8p)))
        return p, s

    def set_row_major(self, particles, sites, number_species, number_site_types):
        dt = np.uint8 if self.bytes_per_slot == 1 else np.uint32
        p = np.ascontiguousarray(particles, dtype=dt)
        s = np.ascontiguousarray(sites, dtype=np.uint8)
        L.check(L.lib().lmb_lattice_set_row_major(self.handle, p.ctypes.data_as(C.c_void_p), _p(s, L.u8p),
                                                  number_species, number_site_types))

    def get_row_major(self):
        dt = np.uint8 if self.bytes_per_slot == 1 else np.uint32
        p = np.zeros((self.X, self.Y, self.Z, self.slots), dtype=dt)
        s = np.zeros((self.X, self.Y, self.Z), dtype=np.uint8)
        L.check(L.lib().lmb_lattice_get_row_major(self.handle, p.ctypes.data_as(C.c_void_p), _p(s, L.u8p)))
        return p, s

    def set_schedule(self, schedule, Ty=0, Tz=0):
        L.check(L.lib().lmb_lattice_set_schedule(self.handle, schedule, Ty, Tz), "lmb_lattice_set_schedule")

    def schedule(self):
        s, ty, tz = C.c_int(), C.c_uint32(), C.c_uint32()
        L.check(L.lib().lmb_lattice_get_schedule(self.handle, C.byref(s), C.byref(ty), C.byref(tz)))
        return s.value, ty.value, tz.value

    def autotune(self, model, seed, first_timestep, timesteps):
        s, ty, tz, ms = C.c_int(), C.c_uint32(), C.c_uint32(), C.c_float()
        L.check(L.lib().lmb_lattice_autotune(self.handle, model.handle, seed, first_timestep, timesteps,
                                             C.byref(s), C.byref(ty), C.byref(tz), C.byref(ms)), "autotune")
        return s.value, ty.value, tz.value, ms.value

    def device_buffers(self):
        a, b = L.vp(), L.vp()
        L.check(L.lib().lmb_lattice_device_buffers(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def species_counts(self, ns):
        c = np.zeros(ns + 1, dtype=np.uint64)
        L.check(L.lib().lmb_lattice_species_counts(self.handle, ns, _p(c, L.u64p)))
        return c

    def run(self, model, seed, first_timestep, timesteps, overflow_mode=L.LMB_OVERFLOW_CLASSIC, check=True):
        st = L.RunStats()
        rc = L.lib().lmb_run(self.handle, model.handle, seed, first_timestep, timesteps, overflow_mode,
                             C.byref(st))
        if check:
            L.check(rc, "lmb_run")
        return rc, st

    def run_counts(self, model, seed, first_timestep, timesteps, number_species,
                   overflow_mode=L.LMB_OVERFLOW_CLASSIC, check=True):
        """lmb_run with the species totals at the end of the run taken in the
        run's own work (lmb_run_counts_async / lmb_run_counts_wait); returns
        (status, stats, counts[0..number_species])."""
        L.check(L.lib().lmb_run_counts_async(self.handle, model.handle, seed, first_timestep, timesteps,
                                             overflow_mode, number_species), "lmb_run_counts_async")
        st = L.RunStats()
        c = np.zeros(number_species + 1, dtype=np.uint64)
        rc = L.lib().lmb_run_counts_wait(self.handle, C.byref(st), _p(c, L.u64p))
        if check:
            L.check(rc, "lmb_run_counts_wait")
        return rc, st, c

    def run_profiled(self, model, seed, first_timestep, timesteps, overflow_mode=L.LMB_OVERFLOW_CLASSIC):
        """Runs with CUDA events around every kernel; returns (stats, phase
        milliseconds [x, y, z, reaction, overflow, fused], launches per phase)."""
        st = L.RunStats()
        ms = np.zeros(6, dtype=np.float32)
        n = np.zeros(6, dtype=np.uint32)
        L.check(L.lib().lmb_run_profiled(self.handle, model.handle, seed, first_timestep, timesteps, overflow_mode,
                                         _p(ms, L.f32p), _p(n, L.u32p), C.byref(st)), "lmb_run_profiled")
        return st, ms, n

    def run_async(self, model, seed, first_timestep, timesteps, overflow_mode=L.LMB_OVERFLOW_CLASSIC):
        L.check(L.lib().lmb_run_async(self.handle, model.handle, seed, first_timestep, timesteps, overflow_mode))

    def run_native_async(self, model, seed, first_timestep, timesteps, particles_in=0, sites_in=0,
                         particles_out=0, overflow_mode=L.LMB_OVERFLOW_CLASSIC):
        """lmb_run_native_async: upload, run and download queued as one solve
        on the lattice's stream; wait() ends it.  The buffers are host
        addresses (ints, e.g. a pinned tensor's data_ptr(); 0 for none) of
        words * N uint32 particles and N uint8 site types, valid until wait()."""
        L.check(L.lib().lmb_run_native_async(self.handle, model.handle, seed, first_timestep, timesteps,
                                             overflow_mode, particles_in or None, sites_in or None,
                                             particles_out or None), "lmb_run_native_async")

    def wait(self, check=True):
        st = L.RunStats()
        rc = L.lib().lmb_run_wait(self.handle, C.byref(st))
        if check:
            L.check(rc, "lmb_run_wait")
        return rc, st

    def close(self):
        if self.handle:
            L.lib().lmb_lattice_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many lattices advanced together (lmb_batch): one launch per timestep
    for all of them.  Each lattice ends where lmb_run alone would take it."""

    def __init__(self, ctx, lattices, models):
        n = len(lattices)
        la = (L.vp * n)(*[l.handle for l in lattices])
        mo = (L.vp * n)(*[m.handle for m in models])
        h = L.vp()
        L.check(L.lib().lmb_batch_create(ctx.handle, n, la, mo, C.byref(h)), "lmb_batch_create")
        self.ctx, self.handle = ctx, h
        self.lattices, self.models = list(lattices), list(models)

    def run(self, seeds, first_timestep, timesteps, overflow_mode=L.LMB_OVERFLOW_CLASSIC, check=True):
        n = len(self.lattices)
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        stats = (L.RunStats * n)()
        rc = L.lib().lmb_batch_run(self.handle, _p(sd, L.u32p), first_timestep, timesteps, overflow_mode, stats)
        if check:
            L.check(rc, "lmb_batch_run")
        return rc, list(stats)

    def run_async(self, seeds, first_timestep, timesteps, overflow_mode=L.LMB_OVERFLOW_CLASSIC):
        self._seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        L.check(L.lib().lmb_batch_run_async(self.handle, _p(self._seeds, L.u32p), first_timestep, timesteps,
                                            overflow_mode), "lmb_batch_run_async")

    def wait(self, check=True):
        n = len(self.lattices)
        stats = (L.RunStats * n)()
        rc = L.lib().lmb_batch_wait(self.handle, stats)
        if check:
            L.check(rc, "lmb_batch_wait")
        return rc, list(stats)

    def run_ranges_async(self, seeds, firsts, counts, overflow_mode=L.LMB_OVERFLOW_CLASSIC):
        """Lattice j runs timesteps firsts[j] .. firsts[j] + counts[j] - 1."""
        self._seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        self._firsts = np.ascontiguousarray(firsts, dtype=np.uint32)
        self._counts = np.ascontiguousarray(counts, dtype=np.uint32)
        L.check(L.lib().lmb_batch_run_ranges_async(self.handle, _p(self._seeds, L.u32p), _p(self._firsts, L.u32p),
                                                   _p(self._counts, L.u32p), overflow_mode),
                "lmb_batch_run_ranges_async")

    def autotune(self, seeds, first_timestep, timesteps):
        """Chooses each lattice size's tile shape by timing the whole batch
        (lmb_batch_autotune); the lattices end where they started.  Returns
        the best trial's milliseconds."""
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        ms = C.c_float()
        L.check(L.lib().lmb_batch_autotune(self.handle, _p(sd, L.u32p), first_timestep, timesteps, C.byref(ms)),
                "lmb_batch_autotune")
        return ms.value

    def plan(self):
        """(Ty, Tz) tile of each lattice."""
        n = len(self.lattices)
        ty = np.zeros(n, dtype=np.uint32)
        tz = np.zeros(n, dtype=np.uint32)
        L.check(L.lib().lmb_batch_plan(self.handle, _p(ty, L.u32p), _p(tz, L.u32p)), "lmb_batch_plan")
        return list(zip(ty.tolist(), tz.tolist()))

    def set_lattices(self, lattices, models):
        n = len(lattices)
        la = (L.vp * n)(*[l.handle for l in lattices])
        mo = (L.vp * n)(*[m.handle for m in models])
        L.check(L.lib().lmb_batch_set_lattices(self.handle, n, la, mo), "lmb_batch_set_lattices")
        self.lattices, self.models = list(lattices), list(models)

    def close(self):
        if self.handle:
            L.lib().lmb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _model_desc(spec):
    """lmb_model_desc for a ModelSpec-like object; returns (desc, arrays to keep alive)."""
    ns, nst, nr = spec.ns, spec.nst, spec.nr
    keep = dict(
        rtype=np.ascontiguousarray(spec.rtype, dtype=np.uint32) if nr else np.zeros(1, np.uint32),
        K=np.ascontiguousarray(spec.K, dtype=np.float64) if nr else np.zeros(1),
        S=np.ascontiguousarray(spec.S, dtype=np.int32).reshape(-1) if nr else np.zeros(1, np.int32),
        D=np.ascontiguousarray(spec.D, dtype=np.uint32).reshape(-1) if nr else np.zeros(1, np.uint32),
        DF=np.ascontiguousarray(spec.DF, dtype=np.float64).reshape(-1),
        RL=np.ascontiguousarray(spec.RL, dtype=np.uint32).reshape(-1) if nr else np.zeros(1, np.uint32),
    )
    d = L.ModelDesc()
    d.number_species, d.number_reactions, d.number_site_types = ns, nr, nst
    d.reaction_types = _p(keep["rtype"], L.u32p)
    d.K = _p(keep["K"], L.f64p)
    d.k_cols = 1
    d.S = _p(keep["S"], L.i32p)
    d.D = _p(keep["D"], L.u32p)
    d.DF = _p(keep["DF"], L.f64p)
    d.RL = _p(keep["RL"], L.u32p)
    d.timestep = spec.tau
    d.lattice_spacing = spec.spacing
    return d, keep


class Server:
    """Continuous batching of MPD-RDME solves (lmb_server): admitted solves
    stay resident on the device and advance together, one launch per
    timestep for all of them; admission is in arrival order under a slot
    count and a device-memory budget."""

    def __init__(self, ctx, slots=8, bytes_per_slot=1, hbm_budget_bytes=150 << 30, max_active=256,
                 chunk_timesteps=256):
        h = L.vp()
        L.check(L.lib().lmb_server_create(ctx.handle, slots, bytes_per_slot, hbm_budget_bytes, max_active,
                                          chunk_timesteps, C.byref(h)), "lmb_server_create")
        self.ctx, self.handle = ctx, h
        self.words_per_site = slots // 4 if bytes_per_slot == 1 else slots

    def submit(self, request_id, spec, seed, timesteps, lattice=None, sites=None):
        """Queues a solve of `spec` (ModelSpec-like; its lattice and site types
        unless given) for `timesteps` timesteps with the composed `seed`."""
        d, keep = _model_desc(spec)
        lat = np.ascontiguousarray(spec.lattice if lattice is None else lattice, dtype=np.uint32)
        st = np.ascontiguousarray(spec.sites if sites is None else sites, dtype=np.uint8)
        r = L.Request()
        r.id = request_id
        r.model = C.pointer(d)
        r.X, r.Y, r.Z = spec.X, spec.Y, spec.Z
        r.particles = _p(lat, L.u32p)
        r.sites = _p(st, L.u8p)
        r.seed = seed
        r.timesteps = timesteps
        L.check(L.lib().lmb_server_submit(self.handle, C.byref(r)), "lmb_server_submit")

    def step(self):
        a, q = C.c_uint32(), C.c_uint32()
        L.check(L.lib().lmb_server_step(self.handle, C.byref(a), C.byref(q)), "lmb_server_step")
        return a.value, q.value

    def status(self):
        st = L.ServerStatus()
        L.check(L.lib().lmb_server_status(self.handle, C.byref(st)))
        return st

    def pop_result(self, with_lattice=True):
        """(info, native lattice or None, species counts) of the oldest
        finished solve, or None."""
        st = self.status()
        if st.ready == 0:
            return None
        info = L.ResultInfo()
        lat = np.zeros(max(1, st.next_ready_words), dtype=np.uint32) if with_lattice else None
        counts = np.zeros(4096, dtype=np.uint64)
        L.check(L.lib().lmb_server_pop_result(self.handle, C.byref(info), _p(lat, L.u32p) if with_lattice else None,
                                              lat.size if with_lattice else 0, _p(counts, L.u64p), counts.size))
        n = info.number_species + 1
        return info, (lat[:st.next_ready_words] if with_lattice else None), counts[:n].copy()

    def close(self):
        if getattr(self, "handle", None):
            L.lib().lmb_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CMEEnsemble:
    """Independent replicates of a well-mixed model advanced by the direct
    method (lmb_cme), the GPU form of running one GillespieDSolver per
    replicate.  ``spec`` is a configs.CMESpec or any object with ns, rtype,
    K, S, D, init."""

    def __init__(self, ctx, spec, replicates):
        self.ctx, self.ns, self.replicates = ctx, spec.ns, replicates
        nr = len(spec.rtype)
        self._keep = dict(
            rtype=np.ascontiguousarray(spec.rtype, dtype=np.uint32),
            K=np.ascontiguousarray(spec.K, dtype=np.float64).reshape(-1),
            S=np.ascontiguousarray(spec.S, dtype=np.int32).reshape(-1),
            D=np.ascontiguousarray(spec.D, dtype=np.uint32).reshape(-1),
        )
        kcols = self._keep["K"].size // nr
        h = L.vp()
        L.check(L.lib().lmb_cme_create(ctx.handle, spec.ns, nr, _p(self._keep["rtype"], L.u32p),
                                       _p(self._keep["K"], L.f64p), kcols, _p(self._keep["S"], L.i32p),
                                       _p(self._keep["D"], L.u32p), replicates, C.byref(h)), "lmb_cme_create")
        self.handle = h
        self.set_initial_counts(spec.init)

    def set_initial_counts(self, counts):
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        per = 1 if c.ndim == 2 else 0
        L.check(L.lib().lmb_cme_set_initial_counts(self.handle, _p(c, L.u32p), per))

    def set_kernel(self, kernel):
        """L.LMB_CME_KERNEL_AUTO (register-resident form for small models) or
        L.LMB_CME_KERNEL_GENERIC; both give the same trajectories."""
        L.check(L.lib().lmb_cme_set_kernel(self.handle, kernel), "lmb_cme_set_kernel")

    def run(self, seed, t_end, write_interval):
        L.check(L.lib().lmb_cme_run(self.handle, seed, t_end, write_interval), "lmb_cme_run")

    def begin(self, seed, t_end, write_interval):
        L.check(L.lib().lmb_cme_begin(self.handle, seed, t_end, write_interval))

    def advance_async(self, until):
        L.check(L.lib().lmb_cme_advance_async(self.handle, until))

    def entries(self):
        n = C.c_uint32()
        L.check(L.lib().lmb_cme_entries(self.handle, C.byref(n)))
        return n.value

    def counts(self):
        """[replicates, entries, species] uint32."""
        out = np.zeros((self.replicates, self.entries(), self.ns), dtype=np.uint32)
        L.check(L.lib().lmb_cme_get_counts(self.handle, _p(out, L.u32p)))
        return out

    def stats(self):
        ev = C.c_uint64()
        fin = C.c_uint32()
        L.check(L.lib().lmb_cme_stats(self.handle, C.byref(ev), C.byref(fin)))
        return ev.value, fin.value

    def close(self):
        if getattr(self, "handle", None):
            L.lib().lmb_cme_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compose_seed(seed_top, replicate):
    return L.lib().lmb_compose_seed(seed_top, replicate)


def kernel_launches():
    return L.lib().lmb_kernel_launches()
