// lmb_serve.cu -- continuous batching of MPD-RDME solves on one device.
//
// The reference runs one solve per replicate thread, each with its own
// solver, lattice and stream (core/ReplicateRunner.cpp:84-166,
// core/ResourceAllocator.cpp), so solves of different sizes run one after
// another or compete for the device.  Here a server keeps every admitted
// solve's lattice resident on the device and advances all of them together:
// each step of the server admits queued requests while the device-memory
// budget and the slot count allow, then runs one chunk of timesteps for
// every resident lattice in one batch (one launch per timestep covering all
// of them, each lattice within its own timestep range), then retires the
// solves that reached their last timestep.  A solve gives the same lattice
// as lmb_run on it alone: every decision depends only on (seed, timestep,
// site, slot) and the lattice's own state.
//
// Small solves share the batched launches, where they would otherwise each
// pay a launch per timestep for little work; a solve of at least
// SOLO_SITES sites fills the device by itself and runs its chunks on its own
// stream, beside the batch.  There are SOLO_STREAMS such streams; a large
// solve is given one at admission (in turn), and each stream advances its
// oldest solve in every step, so that large solves finish in arrival order
// per stream instead of all finishing late.  A large solve takes the
// schedule that suits its particle density: the per-phase kernels for dense
// lattices, the fused kernel for sparse ones.
//
// Host code only; it drives the device through the C ABI of lmb_capi.cu.
#include <chrono>
#include <cstring>
#include <deque>
#include <new>
#include <vector>

#include "lmb.h"
#include "lmb_internal.h"

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t id;
    uint32_t X, Y, Z, seed, timesteps;
    uint32_t ns, nr, nst, kcols;
    std::vector<uint32_t> rtype, D, RL, particles;
    std::vector<int32_t> S;
    std::vector<double> K, DF;
    std::vector<uint8_t> sites;
    double timestep, spacing;
    double t_submit;
    uint64_t bytes;
};

struct Active {
    Request req;
    lmb_lattice *lat;
    lmb_model *model;
    uint32_t done;
    double t_admit;
    lmb_run_stats stats;
    bool solo;
    uint32_t stream;  // large solves: which solo stream
};

constexpr uint64_t SOLO_SITES = 1u << 17;      // 128 Ki sites (about 51^3)
constexpr uint32_t SOLO_STREAMS = 2;
constexpr double DENSE_PARTICLES_PER_SITE = 0.05;

// Particles in a native lattice (nonzero slots).
uint64_t count_particles(const std::vector<uint32_t> &w, uint32_t bytes_per_particle)
{
    uint64_t n = 0;
    for (uint32_t v : w) {
        if (!v) continue;
        if (bytes_per_particle == 4) n++;
        else n += (v & 0xFFu ? 1 : 0) + (v & 0xFF00u ? 1 : 0) + (v & 0xFF0000u ? 1 : 0) + (v & 0xFF000000u ? 1 : 0);
    }
    return n;
}

struct Result {
    lmb_result_info info;
    std::vector<uint32_t> particles;
    std::vector<uint64_t> counts;
};

}  // namespace

struct lmb_server {
    lmb_ctx *ctx;
    // Large solves run on their own streams, beside the small solves' batch.
    lmb_ctx *solo_ctx[SOLO_STREAMS];
    uint32_t next_stream;
    uint32_t slots, bps, words;
    uint64_t budget;
    uint32_t max_active, chunk;
    std::deque<Request> queue;
    std::vector<Active> active;
    std::deque<Result> ready;
    lmb_batch *batch;
    bool members_changed;
    uint64_t bytes_in_use;
    uint64_t peak_bytes;
    uint32_t peak_active;
    uint64_t completed;
};

// Device bytes a resident solve holds: two particle buffers, site types, the
// overflow queue and run state (lmb_lattice_create), the reaction site list
// of the per-phase schedule (N / 8 + 4096 entries of 8 bytes), and the model tables
// (lmb_model_create).
static uint64_t request_bytes(const lmb_server *s, const Request &r)
{
    const uint64_t N = (uint64_t)r.X * r.Y * r.Z;
    const uint64_t lattice = 2ull * s->words * N * 4 + N + 2048ull * 16 + 256 + 8ull * (N / 8 + 4096);
    const uint64_t tables = 4ull * ((uint64_t)r.nst * r.nst * r.ns + r.nst + (uint64_t)r.nst * r.ns +
                                    (uint64_t)r.nst * r.ns * r.ns + 8ull * r.nr) +
                            (uint64_t)r.nr * (r.ns + r.nst) + 4096;
    return lattice + tables;
}

extern "C" int lmb_server_create(lmb_ctx *ctx, uint32_t particles_per_site, uint32_t bytes_per_particle,
                                 uint64_t hbm_budget_bytes, uint32_t max_active, uint32_t chunk_timesteps,
                                 lmb_server **out)
{
    if (!ctx || !out || max_active == 0 || chunk_timesteps == 0) return LMB_E_ARG;
    if (bytes_per_particle != 1 && bytes_per_particle != 4) return LMB_E_ARG;
    *out = nullptr;
    lmb_server *s = new (std::nothrow) lmb_server;
    if (!s) return LMB_E_NOMEM;
    s->ctx = ctx;
    ctx_retain(ctx);
    s->next_stream = 0;
    for (uint32_t k = 0; k < SOLO_STREAMS; k++) s->solo_ctx[k] = nullptr;
    for (uint32_t k = 0; k < SOLO_STREAMS; k++) {
        const int rc = lmb_ctx_create(ctx->device, &s->solo_ctx[k]);
        if (rc != LMB_OK) {
            for (uint32_t q = 0; q < k; q++) lmb_ctx_destroy(s->solo_ctx[q]);
            ctx_release(ctx);
            delete s;
            return rc;
        }
    }
    s->slots = particles_per_site;
    s->bps = bytes_per_particle;
    s->words = bytes_per_particle == 1 ? particles_per_site / 4 : particles_per_site;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->chunk = chunk_timesteps;
    s->batch = nullptr;
    s->members_changed = false;
    s->bytes_in_use = 0;
    s->peak_bytes = 0;
    s->peak_active = 0;
    s->completed = 0;
    *out = s;
    return LMB_OK;
}

static void release_active(lmb_server *s, Active &a)
{
    if (a.lat) lmb_lattice_destroy(a.lat);
    if (a.model) lmb_model_destroy(a.model);
    a.lat = nullptr;
    a.model = nullptr;
    s->bytes_in_use -= a.req.bytes;
}

extern "C" int lmb_server_destroy(lmb_server *s)
{
    if (!s) return LMB_E_ARG;
    if (s->batch) lmb_batch_destroy(s->batch);
    for (Active &a : s->active) release_active(s, a);
    lmb_ctx *c = s->ctx;
    for (uint32_t k = 0; k < SOLO_STREAMS; k++)
        if (s->solo_ctx[k]) lmb_ctx_destroy(s->solo_ctx[k]);
    delete s;
    ctx_release(c);
    return LMB_OK;
}

extern "C" int lmb_server_submit(lmb_server *s, const lmb_request *q)
{
    if (!s || !q || !q->model || !q->particles || !q->sites) return LMB_E_ARG;
    const lmb_model_desc *d = q->model;
    if (q->X == 0 || q->Y == 0 || q->Z == 0 || q->timesteps == 0 || d->k_cols == 0) return LMB_E_ARG;
    Request r;
    r.id = q->id;
    r.X = q->X;
    r.Y = q->Y;
    r.Z = q->Z;
    r.seed = q->seed;
    r.timesteps = q->timesteps;
    r.ns = d->number_species;
    r.nr = d->number_reactions;
    r.nst = d->number_site_types;
    r.kcols = d->k_cols;
    const size_t N = (size_t)q->X * q->Y * q->Z;
    if (r.nr) {
        if (!d->reaction_types || !d->K || !d->S || !d->D || !d->RL) return LMB_E_ARG;
        r.rtype.assign(d->reaction_types, d->reaction_types + r.nr);
        r.K.assign(d->K, d->K + (size_t)r.nr * r.kcols);
        r.S.assign(d->S, d->S + (size_t)r.ns * r.nr);
        r.D.assign(d->D, d->D + (size_t)r.ns * r.nr);
        r.RL.assign(d->RL, d->RL + (size_t)r.nr * r.nst);
    }
    if (!d->DF) return LMB_E_ARG;
    r.DF.assign(d->DF, d->DF + (size_t)r.nst * r.nst * r.ns);
    r.particles.assign(q->particles, q->particles + (size_t)s->words * N);
    r.sites.assign(q->sites, q->sites + N);
    r.timestep = d->timestep;
    r.spacing = d->lattice_spacing;
    r.t_submit = now_s();
    r.bytes = request_bytes(s, r);
    s->queue.push_back(std::move(r));
    return LMB_OK;
}

// Finishes a solve: copies its lattice and species counts out and frees its
// device memory.
static void retire(lmb_server *s, Active &a)
{
    Result res;
    memset(&res.info, 0, sizeof res.info);
    res.info.id = a.req.id;
    res.info.stats = a.stats;
    res.info.stats.steps_done = a.done;
    res.info.X = a.req.X;
    res.info.Y = a.req.Y;
    res.info.Z = a.req.Z;
    res.info.number_species = a.req.ns;
    res.info.t_submit = a.req.t_submit;
    res.info.t_admit = a.t_admit;
    if (a.lat) {
        const size_t N = (size_t)a.req.X * a.req.Y * a.req.Z;
        res.particles.resize((size_t)s->words * N);
        res.counts.resize(a.req.ns + 1);
        int rc = lmb_lattice_get_native(a.lat, res.particles.data(), nullptr);
        if (rc == LMB_OK) rc = lmb_lattice_species_counts(a.lat, a.req.ns, res.counts.data());
        if (rc != LMB_OK && res.info.stats.status == LMB_OK) res.info.stats.status = rc;
    }
    res.info.t_done = now_s();
    release_active(s, a);
    s->ready.push_back(std::move(res));
    s->completed++;
}

// Admits queued requests in arrival order while the slot count and the
// memory budget allow (a request larger than the whole budget is rejected).
static int admit(lmb_server *s)
{
    while (!s->queue.empty() && s->active.size() < s->max_active) {
        Request &r = s->queue.front();
        if (r.bytes > s->budget) {
            Active a;
            a.req = std::move(r);
            s->queue.pop_front();
            a.lat = nullptr;
            a.model = nullptr;
            a.done = 0;
            a.solo = false;
            a.t_admit = now_s();
            memset(&a.stats, 0, sizeof a.stats);
            a.stats.status = LMB_E_NOMEM;
            s->bytes_in_use += a.req.bytes;  // released again by retire
            retire(s, a);
            continue;
        }
        if (s->bytes_in_use + r.bytes > s->budget) break;
        Active a;
        a.req = std::move(r);
        s->queue.pop_front();
        a.lat = nullptr;
        a.model = nullptr;
        a.done = 0;
        a.solo = false;
        memset(&a.stats, 0, sizeof a.stats);
        lmb_model_desc d;
        d.number_species = a.req.ns;
        d.number_reactions = a.req.nr;
        d.number_site_types = a.req.nst;
        d.reaction_types = a.req.rtype.data();
        d.K = a.req.K.data();
        d.k_cols = a.req.kcols;
        d.S = a.req.S.data();
        d.D = a.req.D.data();
        d.DF = a.req.DF.data();
        d.RL = a.req.RL.data();
        d.timestep = a.req.timestep;
        d.lattice_spacing = a.req.spacing;
        s->bytes_in_use += a.req.bytes;
        const uint64_t nsites = (uint64_t)a.req.X * a.req.Y * a.req.Z;
        a.solo = nsites >= SOLO_SITES;
        a.stream = 0;
        if (a.solo) {
            a.stream = s->next_stream;
            s->next_stream = (s->next_stream + 1) % SOLO_STREAMS;
        }
        lmb_ctx *c = a.solo ? s->solo_ctx[a.stream] : s->ctx;
        int rc = lmb_model_create(c, &d, a.req.X, a.req.Y, a.req.Z, &a.model);
        if (rc == LMB_OK) rc = lmb_lattice_create(c, a.req.X, a.req.Y, a.req.Z, s->slots, s->bps, &a.lat);
        if (rc == LMB_OK) rc = lmb_lattice_set_native(a.lat, a.req.particles.data(), a.req.sites.data());
        if (rc == LMB_OK && a.solo) {
            const double density = (double)count_particles(a.req.particles, s->bps) / (double)nsites;
            if (density >= DENSE_PARTICLES_PER_SITE) rc = lmb_lattice_set_schedule(a.lat, LMB_SCHEDULE_PHASES, 0, 0);
        }
        a.t_admit = now_s();
        if (rc != LMB_OK) {
            a.stats.status = rc;
            retire(s, a);
            continue;
        }
        // Host copies are no longer needed once the lattice is on the device.
        std::vector<uint32_t>().swap(a.req.particles);
        std::vector<uint8_t>().swap(a.req.sites);
        if (!a.solo) s->members_changed = true;
        s->active.push_back(std::move(a));
    }
    if (s->bytes_in_use > s->peak_bytes) s->peak_bytes = s->bytes_in_use;
    if (s->active.size() > s->peak_active) s->peak_active = (uint32_t)s->active.size();
    return LMB_OK;
}

extern "C" int lmb_server_step(lmb_server *s, uint32_t *active_out, uint32_t *queued_out)
{
    if (!s) return LMB_E_ARG;
    int rc = admit(s);
    if (rc) return rc;
    const uint32_t n = (uint32_t)s->active.size();
    if (n > 0) {
        std::vector<lmb_run_stats> st(n);
        // Small solves: one batch, one launch per timestep for all of them.
        std::vector<uint32_t> small;
        for (uint32_t j = 0; j < n; j++)
            if (!s->active[j].solo) small.push_back(j);
        if (!small.empty()) {
            const uint32_t nb = (uint32_t)small.size();
            std::vector<lmb_lattice *> lats(nb);
            std::vector<const lmb_model *> models(nb);
            std::vector<uint32_t> seeds(nb), firsts(nb), counts(nb);
            for (uint32_t q = 0; q < nb; q++) {
                Active &a = s->active[small[q]];
                lats[q] = a.lat;
                models[q] = a.model;
                seeds[q] = a.req.seed;
                firsts[q] = a.done;
                const uint32_t left = a.req.timesteps - a.done;
                counts[q] = left < s->chunk ? left : s->chunk;
            }
            if (!s->batch) rc = lmb_batch_create(s->ctx, nb, lats.data(), models.data(), &s->batch);
            else if (s->members_changed) rc = lmb_batch_set_lattices(s->batch, nb, lats.data(), models.data());
            if (rc) return rc;
            s->members_changed = false;
            rc = lmb_batch_run_ranges_async(s->batch, seeds.data(), firsts.data(), counts.data(),
                                            LMB_OVERFLOW_CLASSIC);
            if (rc) return rc;
        }
        // Large solves: the oldest one of each solo stream runs its chunk in
        // this step, beside the batch and the other stream's.
        int solo[SOLO_STREAMS];
        for (uint32_t k = 0; k < SOLO_STREAMS; k++) solo[k] = -1;
        for (uint32_t j = 0; j < n && rc == LMB_OK; j++) {
            Active &a = s->active[j];
            if (!a.solo || solo[a.stream] >= 0) continue;
            const uint32_t left = a.req.timesteps - a.done;
            rc = lmb_run_async(a.lat, a.model, a.req.seed, a.done, left < s->chunk ? left : s->chunk,
                               LMB_OVERFLOW_CLASSIC);
            if (rc == LMB_OK) solo[a.stream] = (int)j;
        }
        int rc_batch = LMB_OK;
        if (!small.empty()) {
            std::vector<lmb_run_stats> bst(small.size());
            rc_batch = lmb_batch_wait(s->batch, bst.data());
            for (size_t q = 0; q < small.size(); q++) st[small[q]] = bst[q];
        }
        for (uint32_t k = 0; k < SOLO_STREAMS; k++) {
            if (solo[k] < 0) continue;
            const int r = lmb_run_wait(s->active[solo[k]].lat, &st[solo[k]]);
            if (rc == LMB_OK) rc = r;
        }
        if (rc != LMB_OK && rc != LMB_E_OVERFLOW_EXHAUSTED && rc != LMB_E_OVERFLOW_UNRESOLVED) return rc;
        if (rc_batch != LMB_OK && rc_batch != LMB_E_OVERFLOW_EXHAUSTED && rc_batch != LMB_E_OVERFLOW_UNRESOLVED)
            return rc_batch;
        rc = LMB_OK;
        // Retire finished and failed solves; keep the order of the rest.
        std::vector<Active> keep;
        keep.reserve(n);
        for (uint32_t j = 0; j < n; j++) {
            Active &a = s->active[j];
            a.done += st[j].steps_done;
            a.stats.overflows += st[j].overflows;
            a.stats.reactions += st[j].reactions;
            if (st[j].status != LMB_OK) {
                a.stats.status = st[j].status;
                a.stats.failed_step = st[j].failed_step;
            }
            if (a.stats.status != LMB_OK || a.done >= a.req.timesteps) {
                if (!a.solo) s->members_changed = true;
                retire(s, a);
            } else {
                keep.push_back(std::move(a));
            }
        }
        s->active.swap(keep);
    }
    if (active_out) *active_out = (uint32_t)s->active.size();
    if (queued_out) *queued_out = (uint32_t)s->queue.size();
    return LMB_OK;
}

extern "C" int lmb_server_pop_result(lmb_server *s, lmb_result_info *info, uint32_t *particles,
                                     uint64_t particles_words, uint64_t *species_counts, uint32_t counts_len)
{
    if (!s || !info) return LMB_E_ARG;
    if (s->ready.empty()) return LMB_E_STATE;
    Result &r = s->ready.front();
    if (particles && r.particles.size() > particles_words) return LMB_E_ARG;
    *info = r.info;
    if (particles && !r.particles.empty()) memcpy(particles, r.particles.data(), r.particles.size() * 4);
    if (species_counts) {
        const size_t n = r.counts.size() < counts_len ? r.counts.size() : counts_len;
        if (n) memcpy(species_counts, r.counts.data(), n * 8);
    }
    s->ready.pop_front();
    return LMB_OK;
}

extern "C" int lmb_server_status(const lmb_server *s, lmb_server_status_info *st)
{
    if (!s || !st) return LMB_E_ARG;
    st->active = (uint32_t)s->active.size();
    st->queued = (uint32_t)s->queue.size();
    st->ready = (uint32_t)s->ready.size();
    st->peak_active = s->peak_active;
    st->bytes_in_use = s->bytes_in_use;
    st->peak_bytes = s->peak_bytes;
    st->completed = s->completed;
    st->next_ready_words = s->ready.empty() ? 0 : s->ready.front().particles.size();
    return LMB_OK;
}
