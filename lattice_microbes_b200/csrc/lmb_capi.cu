// lmb_capi.cu -- the C ABI declared in include/lmb.h.
//
// Host side of the solver: model building (the reference's
// MpdRdmeSolver::buildModel / buildDiffusionModel / computePropensities,
// restated), device buffers, and the timestep loop that queues the per-phase
// kernels of lmb_kernels.cu on the context stream.  Nothing here throws; every
// entry returns a status code.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_fused.h"
#include "lmb_internal.h"

using namespace lmb;

namespace lmb {
static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches += n; }
}  // namespace lmb

struct lmb_model {
    lmb_ctx *ctx;
    uint32_t ns, nst, nr;
    uint32_t X, Y, Z;
    bool has_desc;
    // Reference-side inputs kept for setReactionRate.
    std::vector<uint32_t> rtype, s1, s2;
    std::vector<double> K;
    std::vector<uint32_t> RLin;
    double tau;
    // Host copy of the FP32 tables.
    std::vector<float> T, qp0, qp1, qp2, rate;
    std::vector<uint32_t> order, D1, D2;
    std::vector<int8_t> S;
    std::vector<uint8_t> RL;
    std::vector<uint32_t> st_off, st_sp;
    std::vector<int32_t> st_d;
    std::vector<float> qpmax;  // per site type: largest qp1, then largest qp2 entry
    std::vector<uint32_t> rx_off, rx_list;  // reactions by first reactant (DevTables::rx_off)
    // Device copy.
    void *dev_block;
    size_t dev_bytes;
    DevTables dev;
    bool dirty;
};

struct lmb_lattice {
    lmb_ctx *ctx;
    Geometry g;
    uint32_t bps, slots, words;
    uint32_t *buf[2];
    int cur;
    uint8_t *sites;
    RunState *rs;
    RunState *rs_host;  // pinned
    OverflowEntry *list;
    uint32_t cap;
    // Per-phase schedule: sites the z sweep lists for the reaction step,
    // rx_cap entries of two words (allocated when the schedule is first
    // chosen).
    uint32_t *rx_sites;
    uint32_t rx_cap;
    // Per-phase schedule, X a multiple of 32: plane bounds of buf[0] (first
    // nseg words) and buf[1] (next nseg), one per segment of 32 sites.
    uint32_t *pb;
    uint32_t nseg;
    unsigned long long *counts_dev;
    uint32_t counts_len;
    // Species counts of the last lmb_run_counts_async (pinned), and the
    // species count they were taken for (~0u: none pending).
    unsigned long long *counts_host;
    uint32_t counts_host_len;
    uint32_t pending_count_ns;
    bool validated;
    uint32_t max_species, max_site_type;
    // Schedule: fused tile kernel (one launch per timestep) or per-phase kernels.
    int schedule;
    TileShape tile;
    // Captured timestep graphs, one per starting buffer parity.
    struct Graph {
        cudaGraphExec_t exec;
        const void *model;
        const void *tables;
        int schedule;
        uint32_t Ty, Tz;
        bool reaction;
        uint64_t kernels;
    } graph[2];
    // Pending async run.
    bool pending;
    int pending_cur0;
    uint32_t pending_first, pending_n;
    bool pending_check;  // its new contents are checked on the device (lmb_run_native_async)
};

#define CK(call)                                      \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

static int cuda_status(cudaError_t e)
{
    if (e == cudaErrorMemoryAllocation) return LMB_E_NOMEM;
    return LMB_E_CUDA;
}

// Schedules that hold the lattice in shared memory and run every timestep of
// a run in one launch.
static bool resident_schedule(int schedule)
{
    return schedule == LMB_SCHEDULE_CLUSTER || schedule == LMB_SCHEDULE_GRID;
}

// The one launch of a run on a resident schedule, from the current buffer.
static cudaError_t launch_resident(lmb_lattice *l, const lmb_model *m, cudaStream_t stream)
{
    uint32_t *a = l->buf[l->cur], *b = l->buf[l->cur ^ 1];
    if (l->schedule == LMB_SCHEDULE_GRID)
        return launch_fused_grid((int)l->bps, (int)l->slots, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap,
                                 l->tile, m->nr > 0, stream);
    return launch_cluster_run((int)l->bps, (int)l->slots, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap,
                              stream);
}

extern "C" int lmb_abi_version(void) { return LMB_ABI_VERSION; }

extern "C" const char *lmb_status_string(int s)
{
    switch (s) {
    case LMB_OK: return "ok";
    case LMB_E_ARG: return "invalid argument";
    case LMB_E_CUDA: return "CUDA error";
    case LMB_E_NOMEM: return "device out of memory";
    case LMB_E_MODEL: return "model rejected";
    case LMB_E_STATE: return "invalid call order or state";
    case LMB_E_OVERFLOW_EXHAUSTED: return "Too many particle overflows for the available buffer";
    case LMB_E_OVERFLOW_UNRESOLVED: return "Unable to find an available site to handle a particle overflow";
    case LMB_E_TIMEOUT: return "device wait timed out";
    case LMB_E_UNSUPPORTED: return "unsupported lattice layout or size";
    case LMB_E_IO: return "file could not be created or written";
    default: return "unknown status";
    }
}

extern "C" uint32_t lmb_compose_seed(uint32_t seed_top, uint32_t replicate)
{
    return (uint32_t)((seed_top << 16) | (replicate & 0xFFFFu));
}

extern "C" uint64_t lmb_timestep_hash(uint32_t seed, uint32_t timestep, uint32_t substep)
{
    return timestep_hash(seed, timestep, substep);
}

extern "C" uint64_t lmb_kernel_launches(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------

extern "C" int lmb_ctx_create_on_stream(int device, void *stream, lmb_ctx **out)
{
    if (!out) return LMB_E_ARG;
    *out = nullptr;
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return LMB_E_ARG;
    CK(cudaSetDevice(device));
    lmb_ctx *c = new (std::nothrow) lmb_ctx;
    if (!c) return LMB_E_NOMEM;
    c->device = device;
    c->refs.store(1);
    c->own_stream = stream == nullptr;
    if (stream) c->stream = (cudaStream_t)stream;
    else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            return cuda_status(e);
        }
    }
    *out = c;
    return LMB_OK;
}

extern "C" int lmb_ctx_create(int device, lmb_ctx **out) { return lmb_ctx_create_on_stream(device, nullptr, out); }

extern "C" int lmb_ctx_destroy(lmb_ctx *c)
{
    if (!c) return LMB_E_ARG;
    ctx_release(c);
    return LMB_OK;
}

extern "C" void *lmb_ctx_stream(lmb_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" int lmb_ctx_synchronize(lmb_ctx *c)
{
    if (!c) return LMB_E_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    return LMB_OK;
}

// ---------------------------------------------------------------------------
// Model
// ---------------------------------------------------------------------------

// computePropensities (MpdRdmeSolver.cu:697-774): per-reaction scaled rates
// and the per-site-type qp0/qp1/qp2 tables.  "float += double" expressions of
// the reference round once after a double add, and are evaluated that way.
static void compute_propensities(lmb_model *m)
{
    const uint32_t X = m->X, Y = m->Y, Z = m->Z, ns = m->ns, nst = m->nst, nr = m->nr;
    const double tau = m->tau;
    const uint32_t nsites_u = X * Y * Z;
    for (uint32_t r = 0; r < nr; r++) {
        const double k = m->K[r];
        switch (m->rtype[r]) {
        case LMB_REACTION_ZEROTH: m->rate[r] = (float)(k * tau / (double)nsites_u); break;
        case LMB_REACTION_FIRST: m->rate[r] = (float)(k * tau); break;
        default: m->rate[r] = (float)(k * tau * X * Y * Z); break;
        }
    }
    const float scale = (float)nsites_u;
    for (uint32_t st = 0; st < nst; st++) {
        const size_t o1 = (size_t)st * ns, o2 = (size_t)st * ns * ns;
        m->qp0[st] = 0.0f;
        std::fill(m->qp1.begin() + o1, m->qp1.begin() + o1 + ns, 0.0f);
        std::fill(m->qp2.begin() + o2, m->qp2.begin() + o2 + (size_t)ns * ns, 0.0f);
        for (uint32_t r = 0; r < nr; r++) {
            if (!m->RLin[(size_t)r * nst + st]) continue;
            const double k = m->K[r];
            const uint32_t a = m->s1[r], b = m->s2[r];
            switch (m->rtype[r]) {
            case LMB_REACTION_ZEROTH: m->qp0[st] = (float)((double)m->qp0[st] + k * tau / (double)scale); break;
            case LMB_REACTION_FIRST: m->qp1[o1 + a] = (float)((double)m->qp1[o1 + a] + k * tau); break;
            case LMB_REACTION_SECOND:
                // Assignment, not accumulation (MpdRdmeSolver.cu:760-764).
                m->qp2[o2 + (size_t)a * ns + b] = (float)(k * tau * (double)scale);
                m->qp2[o2 + (size_t)b * ns + a] = (float)(k * tau * (double)scale);
                break;
            case LMB_REACTION_SECOND_SELF: {
                const size_t e = o2 + (size_t)a * ns + a;
                m->qp2[e] = (float)((double)m->qp2[e] + k * tau * (double)scale * 2);
                break;
            }
            }
        }
    }
}

static int upload_model(lmb_model *m)
{
    lmb_ctx *c = m->ctx;
    CK(cudaSetDevice(c->device));
    // Largest single-particle and pair table entries per site type: they
    // bound a site's total propensity from its particle count alone.
    m->qpmax.assign(2 * (size_t)m->nst, 0.0f);
    for (uint32_t st = 0; st < m->nst; st++) {
        float a = 0.0f, b = 0.0f;
        for (uint32_t i = 0; i < m->ns; i++) a = std::max(a, m->qp1[(size_t)st * m->ns + i]);
        for (size_t i = 0; i < (size_t)m->ns * m->ns; i++) b = std::max(b, m->qp2[(size_t)st * m->ns * m->ns + i]);
        m->qpmax[st] = a;
        m->qpmax[m->nst + st] = b;
    }
    // Reactions by first reactant (zeroth-order ones first), ascending.
    m->rx_off.assign((size_t)m->ns + 2, 0);
    m->rx_list.clear();
    for (uint32_t sp = 0; sp <= m->ns; sp++) {
        m->rx_off[sp] = (uint32_t)m->rx_list.size();
        for (uint32_t r = 0; r < m->nr; r++) {
            const bool zeroth = m->order[r] == 1;
            if ((sp == 0 && zeroth) || (sp > 0 && !zeroth && m->D1[r] == sp)) m->rx_list.push_back(r);
        }
    }
    m->rx_off[m->ns + 1] = (uint32_t)m->rx_list.size();
    // One device block holding every table, 256-byte aligned pieces.
    std::vector<std::pair<const void *, size_t>> parts = {
        {m->T.data(), m->T.size() * 4},          {m->qp0.data(), m->qp0.size() * 4},
        {m->qp1.data(), m->qp1.size() * 4},      {m->qp2.data(), m->qp2.size() * 4},
        {m->order.data(), m->order.size() * 4},  {m->D1.data(), m->D1.size() * 4},
        {m->D2.data(), m->D2.size() * 4},        {m->rate.data(), m->rate.size() * 4},
        {m->RL.data(), m->RL.size()},            {m->st_off.data(), m->st_off.size() * 4},
        {m->st_sp.data(), m->st_sp.size() * 4},  {m->st_d.data(), m->st_d.size() * 4},
        {m->qpmax.data(), m->qpmax.size() * 4},  {m->rx_off.data(), m->rx_off.size() * 4},
        {m->rx_list.data(), m->rx_list.size() * 4}};
    std::vector<size_t> off(parts.size());
    size_t total = 0;
    for (size_t i = 0; i < parts.size(); i++) {
        off[i] = total;
        total += (parts[i].second + 255) & ~(size_t)255;
        if (parts[i].second == 0) total += 256;
    }
    if (!m->dev_block || m->dev_bytes < total) {
        if (m->dev_block) cudaFree(m->dev_block);
        m->dev_block = nullptr;
        CK(cudaMalloc(&m->dev_block, total));
        m->dev_bytes = total;
    }
    std::vector<uint8_t> staging(total, 0);
    for (size_t i = 0; i < parts.size(); i++)
        if (parts[i].second) memcpy(staging.data() + off[i], parts[i].first, parts[i].second);
    CK(cudaMemcpyAsync(m->dev_block, staging.data(), total, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    uint8_t *b = (uint8_t *)m->dev_block;
    m->dev.ns = m->ns;
    m->dev.nst = m->nst;
    m->dev.nr = m->nr;
    m->dev.T = (const float *)(b + off[0]);
    m->dev.qp0 = (const float *)(b + off[1]);
    m->dev.qp1 = (const float *)(b + off[2]);
    m->dev.qp2 = (const float *)(b + off[3]);
    m->dev.order = (const uint32_t *)(b + off[4]);
    m->dev.D1 = (const uint32_t *)(b + off[5]);
    m->dev.D2 = (const uint32_t *)(b + off[6]);
    m->dev.rate = (const float *)(b + off[7]);
    m->dev.RL = (const uint8_t *)(b + off[8]);
    m->dev.stoich_off = (const uint32_t *)(b + off[9]);
    m->dev.stoich_sp = (const uint32_t *)(b + off[10]);
    m->dev.stoich_d = (const int32_t *)(b + off[11]);
    m->dev.qpmax = (const float *)(b + off[12]);
    m->dev.rx_off = (const uint32_t *)(b + off[13]);
    m->dev.rx_list = (const uint32_t *)(b + off[14]);
    m->dev.nnz = (uint32_t)m->st_sp.size();
    m->dev.stage_bytes = 0;
    {
        // Tables small enough to copy into shared memory per block (16-byte
        // aligned pieces, in the order the fused kernel lays them out).
        size_t bytes = 0;
        const size_t pieces[] = {m->T.size() * 4, m->qp0.size() * 4, m->qp1.size() * 4, m->qp2.size() * 4,
                                 (size_t)m->nr * 4, (size_t)m->nr * 4, (size_t)m->nr * 4, (size_t)m->nr * 4,
                                 m->RL.size(), ((size_t)m->nr + 1) * 4, m->st_sp.size() * 4, m->st_d.size() * 4,
                                 m->qpmax.size() * 4, m->rx_off.size() * 4, m->rx_list.size() * 4};
        for (size_t p : pieces) bytes += (p + 15) & ~(size_t)15;
        if (bytes <= 8 * 1024) m->dev.stage_bytes = (uint32_t)bytes;
    }
    m->dirty = false;
    return LMB_OK;
}

// Sparse per-reaction stoichiometry from the transposed S (ascending species).
static int build_stoich(lmb_model *m)
{
    m->st_off.assign(m->nr + 1, 0);
    m->st_sp.clear();
    m->st_d.clear();
    for (uint32_t r = 0; r < m->nr; r++) {
        m->st_off[r] = (uint32_t)m->st_sp.size();
        uint32_t cnt = 0;
        for (uint32_t s = 0; s < m->ns; s++) {
            const int8_t v = m->S[(size_t)r * m->ns + s];
            if (v != 0) {
                m->st_sp.push_back(s);
                m->st_d.push_back(v);
                cnt++;
            }
        }
        if (cnt > 32) return LMB_E_UNSUPPORTED;
    }
    m->st_off[m->nr] = (uint32_t)m->st_sp.size();
    return LMB_OK;
}

extern "C" int lmb_model_get_tables(const lmb_model *m, float *T, float *qp0, float *qp1, float *qp2,
                                    uint32_t *order, uint32_t *D1, uint32_t *D2, float *rate, int8_t *S,
                                    uint8_t *RL);
static void free_model(lmb_model *m);

static lmb_model *new_model(lmb_ctx *c, uint32_t ns, uint32_t nst, uint32_t nr)
{
    lmb_model *m = new (std::nothrow) lmb_model;
    if (!m) return nullptr;
    m->ctx = c;
    if (c) ctx_retain(c);
    m->ns = ns;
    m->nst = nst;
    m->nr = nr;
    m->X = m->Y = m->Z = 0;
    m->has_desc = false;
    m->tau = 0;
    m->dev_block = nullptr;
    m->dev_bytes = 0;
    m->dirty = true;
    m->T.assign((size_t)nst * nst * ns, 0.0f);
    m->qp0.assign(nst, 0.0f);
    m->qp1.assign((size_t)nst * ns, 0.0f);
    m->qp2.assign((size_t)nst * ns * ns, 0.0f);
    m->rate.assign(nr, 0.0f);
    m->order.assign(nr, 0);
    m->D1.assign(nr, 0);
    m->D2.assign(nr, 0);
    m->S.assign((size_t)nr * ns, 0);
    m->RL.assign((size_t)nr * nst, 0);
    return m;
}

// Fills a model's host tables from reference-style inputs; no device work.
static int build_model_host(const lmb_model_desc *d, uint32_t X, uint32_t Y, uint32_t Z, lmb_model *m)
{
    const uint32_t ns = d->number_species, nr = d->number_reactions, nst = d->number_site_types;
    m->X = X;
    m->Y = Y;
    m->Z = Z;
    m->has_desc = true;
    m->tau = d->timestep;
    m->rtype.assign(d->reaction_types, d->reaction_types + nr);
    m->K.resize(nr);
    for (uint32_t r = 0; r < nr; r++) m->K[r] = d->K[(size_t)r * d->k_cols];
    m->RLin.assign(d->RL, d->RL + (size_t)nr * nst);
    m->s1.assign(nr, 0);
    m->s2.assign(nr, 0);
    // Reactants from the dependency columns (CMESolver.cpp:340-430) and the
    // device order / 1-based ids (MpdRdmeSolver.cu:265-302).
    for (uint32_t r = 0; r < nr; r++) {
        uint32_t deps[3], nd = 0;
        for (uint32_t s = 0; s < ns; s++)
            if (d->D[(size_t)s * nr + r] == 1) {
                if (nd < 3) deps[nd] = s;
                nd++;
            }
        const uint32_t t = m->rtype[r];
        bool ok = (t == LMB_REACTION_ZEROTH && nd == 0) || (t == LMB_REACTION_FIRST && nd == 1) ||
                  (t == LMB_REACTION_SECOND && nd == 2) || (t == LMB_REACTION_SECOND_SELF && nd == 1);
        if (!ok) return LMB_E_MODEL;
        m->order[r] = t + 1;
        if (nd >= 1) m->s1[r] = deps[0];
        if (nd >= 2) m->s2[r] = deps[1];
        m->D1[r] = t == LMB_REACTION_ZEROTH ? 0 : m->s1[r] + 1;
        m->D2[r] = t == LMB_REACTION_SECOND ? m->s2[r] + 1 : 0;
    }
    // T[src][dst][sp] = (float)(DF * tau / spacing^2), q > 0.5 rejected
    // (MpdRdmeSolver.cu:407-421).
    for (size_t i = 0; i < m->T.size(); i++) {
        const float q = (float)(d->DF[i] * d->timestep / pow(d->lattice_spacing, 2));
        if (q > 0.50f) return LMB_E_MODEL;
        m->T[i] = q;
    }
    // SG[rx][sp] = S[sp][rx] (MpdRdmeSolver.cu:312-321); RL as bytes.
    for (uint32_t r = 0; r < nr; r++)
        for (uint32_t s = 0; s < ns; s++) m->S[(size_t)r * ns + s] = (int8_t)d->S[(size_t)s * nr + r];
    for (size_t i = 0; i < m->RL.size(); i++) m->RL[i] = (uint8_t)m->RLin[i];
    int rc = build_stoich(m);
    if (rc != LMB_OK) return rc;
    compute_propensities(m);
    return LMB_OK;
}

static int check_desc(const lmb_model_desc *d, uint32_t X, uint32_t Y, uint32_t Z)
{
    if (!d || X == 0 || Y == 0 || Z == 0) return LMB_E_ARG;
    const uint32_t ns = d->number_species, nr = d->number_reactions, nst = d->number_site_types;
    if (ns == 0 || nst == 0 || nst > 256) return LMB_E_ARG;
    if (nr > 0 && (!d->reaction_types || !d->K || d->k_cols == 0 || !d->S || !d->D || !d->RL)) return LMB_E_ARG;
    if (!d->DF || !(d->timestep > 0.0) || !(d->lattice_spacing > 0.0)) return LMB_E_ARG;
    return LMB_OK;
}

extern "C" int lmb_model_create(lmb_ctx *c, const lmb_model_desc *d, uint32_t X, uint32_t Y, uint32_t Z,
                                lmb_model **out)
{
    if (!c || !out) return LMB_E_ARG;
    *out = nullptr;
    int rc = check_desc(d, X, Y, Z);
    if (rc) return rc;
    lmb_model *m = new_model(c, d->number_species, d->number_site_types, d->number_reactions);
    if (!m) return LMB_E_NOMEM;
    rc = build_model_host(d, X, Y, Z, m);
    if (rc == LMB_OK) rc = upload_model(m);
    if (rc != LMB_OK) {
        free_model(m);
        return rc;
    }
    *out = m;
    return LMB_OK;
}

extern "C" int lmb_tables_build(const lmb_model_desc *d, uint32_t X, uint32_t Y, uint32_t Z, float *T, float *qp0,
                                float *qp1, float *qp2, uint32_t *order, uint32_t *D1, uint32_t *D2, float *rate,
                                int8_t *S, uint8_t *RL)
{
    int rc = check_desc(d, X, Y, Z);
    if (rc) return rc;
    lmb_model *m = new_model(nullptr, d->number_species, d->number_site_types, d->number_reactions);
    if (!m) return LMB_E_NOMEM;
    rc = build_model_host(d, X, Y, Z, m);
    if (rc == LMB_OK) rc = lmb_model_get_tables(m, T, qp0, qp1, qp2, order, D1, D2, rate, S, RL);
    free_model(m);
    return rc;
}

extern "C" int lmb_model_create_from_tables(lmb_ctx *c, const lmb_tables *t, lmb_model **out)
{
    if (!c || !t || !out || t->number_species == 0 || t->number_site_types == 0 || t->number_site_types > 256)
        return LMB_E_ARG;
    *out = nullptr;
    const uint32_t ns = t->number_species, nst = t->number_site_types, nr = t->number_reactions;
    if (!t->T || !t->qp0 || !t->qp1 || !t->qp2) return LMB_E_ARG;
    if (nr && (!t->order || !t->D1 || !t->D2 || !t->rate || !t->S || !t->RL)) return LMB_E_ARG;
    lmb_model *m = new_model(c, ns, nst, nr);
    if (!m) return LMB_E_NOMEM;
    std::copy(t->T, t->T + m->T.size(), m->T.begin());
    std::copy(t->qp0, t->qp0 + m->qp0.size(), m->qp0.begin());
    std::copy(t->qp1, t->qp1 + m->qp1.size(), m->qp1.begin());
    std::copy(t->qp2, t->qp2 + m->qp2.size(), m->qp2.begin());
    if (nr) {
        std::copy(t->order, t->order + nr, m->order.begin());
        std::copy(t->D1, t->D1 + nr, m->D1.begin());
        std::copy(t->D2, t->D2 + nr, m->D2.begin());
        std::copy(t->rate, t->rate + nr, m->rate.begin());
        std::copy(t->S, t->S + m->S.size(), m->S.begin());
        std::copy(t->RL, t->RL + m->RL.size(), m->RL.begin());
    }
    for (float q : m->T)
        if (q > 0.50f) {
            free_model(m);
            return LMB_E_MODEL;
        }
    int rc = build_stoich(m);
    if (rc == LMB_OK) rc = upload_model(m);
    if (rc != LMB_OK) {
        free_model(m);
        return rc;
    }
    *out = m;
    return LMB_OK;
}

extern "C" int lmb_model_get_tables(const lmb_model *m, float *T, float *qp0, float *qp1, float *qp2,
                                    uint32_t *order, uint32_t *D1, uint32_t *D2, float *rate, int8_t *S,
                                    uint8_t *RL)
{
    if (!m) return LMB_E_ARG;
    if (T) std::copy(m->T.begin(), m->T.end(), T);
    if (qp0) std::copy(m->qp0.begin(), m->qp0.end(), qp0);
    if (qp1) std::copy(m->qp1.begin(), m->qp1.end(), qp1);
    if (qp2) std::copy(m->qp2.begin(), m->qp2.end(), qp2);
    if (order) std::copy(m->order.begin(), m->order.end(), order);
    if (D1) std::copy(m->D1.begin(), m->D1.end(), D1);
    if (D2) std::copy(m->D2.begin(), m->D2.end(), D2);
    if (rate) std::copy(m->rate.begin(), m->rate.end(), rate);
    if (S) std::copy(m->S.begin(), m->S.end(), S);
    if (RL) std::copy(m->RL.begin(), m->RL.end(), RL);
    return LMB_OK;
}

extern "C" int lmb_model_set_reaction_rate(lmb_model *m, uint32_t reaction, double rate)
{
    if (!m || reaction >= m->nr) return LMB_E_ARG;
    if (!m->has_desc) return LMB_E_STATE;
    m->K[reaction] = rate;
    compute_propensities(m);
    m->dirty = true;
    return LMB_OK;
}

static void free_model(lmb_model *m)
{
    if (m->dev_block && m->ctx) {
        cudaSetDevice(m->ctx->device);
        cudaStreamSynchronize(m->ctx->stream);
        cudaFree(m->dev_block);
    }
    if (m->ctx) ctx_release(m->ctx);
    delete m;
}

extern "C" int lmb_model_destroy(lmb_model *m)
{
    if (!m) return LMB_E_ARG;
    free_model(m);
    return LMB_OK;
}

// ---------------------------------------------------------------------------
// Lattice
// ---------------------------------------------------------------------------

static const uint32_t DEFAULT_OVERFLOW_CAPACITY = 2048;  // TUNE_MPD_MAX_PARTICLE_OVERFLOWS

extern "C" int lmb_lattice_create(lmb_ctx *c, uint32_t X, uint32_t Y, uint32_t Z, uint32_t slots, uint32_t bps,
                                  lmb_lattice **out)
{
    if (!c || !out || X == 0 || Y == 0 || Z == 0) return LMB_E_ARG;
    *out = nullptr;
    if (!slots_supported((int)bps, (int)slots)) return LMB_E_UNSUPPORTED;
    const uint64_t N = (uint64_t)X * Y * Z;
    if (N > 0xFFFFFFFFull) return LMB_E_UNSUPPORTED;  // site indices are 32-bit
    CK(cudaSetDevice(c->device));
    lmb_lattice *l = new (std::nothrow) lmb_lattice;
    if (!l) return LMB_E_NOMEM;
    memset((void *)l, 0, sizeof(*l));
    l->ctx = c;
    ctx_retain(c);
    l->g.X = X;
    l->g.Y = Y;
    l->g.Z = Z;
    l->g.XY = X * Y;
    l->g.N = (uint32_t)N;
    l->bps = bps;
    l->slots = slots;
    l->words = bps == 1 ? slots / 4 : slots;
    l->cap = DEFAULT_OVERFLOW_CAPACITY;
    const size_t wbytes = (size_t)l->words * N * sizeof(uint32_t);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&l->buf[0], wbytes);
    if (e == cudaSuccess) e = cudaMalloc(&l->buf[1], wbytes);
    if (e == cudaSuccess) e = cudaMalloc(&l->sites, N);
    if (e == cudaSuccess) e = cudaMalloc(&l->rs, sizeof(RunState));
    if (e == cudaSuccess) e = cudaMalloc(&l->list, sizeof(OverflowEntry) * l->cap);
    if (e == cudaSuccess) e = cudaMallocHost(&l->rs_host, sizeof(RunState));
    if (e == cudaSuccess) e = cudaMemsetAsync(l->buf[0], 0, wbytes, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l->buf[1], 0, wbytes, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l->sites, 0, N, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l->rs, 0, sizeof(RunState), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        lmb_lattice_destroy(l);
        return cuda_status(e);
    }
    l->validated = false;
    l->schedule = LMB_SCHEDULE_FUSED;
    if (!fused_default_shape(l->g, (int)bps, (int)slots, l->tile)) {
        const int rc = lmb_lattice_set_schedule(l, LMB_SCHEDULE_PHASES, 0, 0);
        if (rc != LMB_OK) {
            lmb_lattice_destroy(l);
            return rc;
        }
    }
    *out = l;
    return LMB_OK;
}

// Room for one eighth of the sites plus 4096: sparse lattices list a small
// fraction of their sites; denser ones overflow it and react over every site.
static uint32_t reaction_list_capacity(const Geometry &g) { return g.N / 8 + 4096; }

extern "C" int lmb_lattice_set_schedule(lmb_lattice *l, int schedule, uint32_t Ty, uint32_t Tz)
{
    if (!l) return LMB_E_ARG;
    if (schedule == LMB_SCHEDULE_PHASES) {
        if (!l->rx_sites) {
            CK(cudaSetDevice(l->ctx->device));
            const uint32_t cap = reaction_list_capacity(l->g);
            CK(cudaMalloc(&l->rx_sites, (size_t)cap * 2 * sizeof(uint32_t)));
            l->rx_cap = cap;
        }
        // Plane bounds need every warp of a sweep tile to hold one whole
        // segment: x rows a multiple of 32 sites.
        if (!l->pb && l->g.X % 32u == 0) {
            CK(cudaSetDevice(l->ctx->device));
            const uint32_t nseg = l->g.N >> PB_SHIFT;
            CK(cudaMalloc(&l->pb, (size_t)nseg * 2 * sizeof(uint32_t)));
            l->nseg = nseg;
        }
        l->schedule = schedule;
        return LMB_OK;
    }
    if (schedule == LMB_SCHEDULE_CLUSTER) {
        // The plan is checked with the largest staged tables (8 KiB).
        uint32_t C = 0, P = 0;
        CK(cudaSetDevice(l->ctx->device));
        if (!cluster_plan(l->g, (int)l->bps, (int)l->slots, l->cap, 8 * 1024, C, P)) return LMB_E_UNSUPPORTED;
        l->schedule = schedule;
        return LMB_OK;
    }
    if (schedule == LMB_SCHEDULE_GRID) {
        // Every tile resident at once, checked with the largest staged tables (8 KiB).
        CK(cudaSetDevice(l->ctx->device));
        TileShape t;
        const bool ok = (Ty == 0 && Tz == 0)
                            ? fused_grid_default_shape(l->g, (int)l->bps, (int)l->slots, l->cap, 8 * 1024, t)
                            : fused_make_shape(l->g, (int)l->bps, (int)l->slots, Ty, Tz, t) &&
                                  fused_grid_fits(l->g, (int)l->bps, (int)l->slots, l->cap, 8 * 1024, t);
        if (!ok) return LMB_E_UNSUPPORTED;
        l->tile = t;
        l->schedule = schedule;
        return LMB_OK;
    }
    if (schedule != LMB_SCHEDULE_FUSED) return LMB_E_ARG;
    TileShape t;
    bool ok = (Ty == 0 && Tz == 0) ? fused_default_shape(l->g, (int)l->bps, (int)l->slots, t)
                                   : fused_make_shape(l->g, (int)l->bps, (int)l->slots, Ty, Tz, t);
    if (!ok) return LMB_E_UNSUPPORTED;
    l->tile = t;
    l->schedule = schedule;
    return LMB_OK;
}

extern "C" int lmb_lattice_get_schedule(lmb_lattice *l, int *schedule, uint32_t *Ty, uint32_t *Tz)
{
    if (!l) return LMB_E_ARG;
    if (schedule) *schedule = l->schedule;
    const bool tiled = l->schedule == LMB_SCHEDULE_FUSED || l->schedule == LMB_SCHEDULE_GRID;
    if (Ty) *Ty = tiled ? l->tile.Ty : 0;
    if (Tz) *Tz = tiled ? l->tile.Tz : 0;
    return LMB_OK;
}

extern "C" int lmb_lattice_destroy(lmb_lattice *l)
{
    if (!l) return LMB_E_ARG;
    cudaSetDevice(l->ctx->device);
    cudaStreamSynchronize(l->ctx->stream);
    if (l->buf[0]) cudaFree(l->buf[0]);
    if (l->buf[1]) cudaFree(l->buf[1]);
    if (l->sites) cudaFree(l->sites);
    if (l->rs) cudaFree(l->rs);
    if (l->list) cudaFree(l->list);
    if (l->rx_sites) cudaFree(l->rx_sites);
    if (l->pb) cudaFree(l->pb);
    if (l->counts_dev) cudaFree(l->counts_dev);
    if (l->counts_host) cudaFreeHost(l->counts_host);
    if (l->rs_host) cudaFreeHost(l->rs_host);
    for (auto &gr : l->graph)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    lmb_ctx *c = l->ctx;
    delete l;
    ctx_release(c);
    return LMB_OK;
}

static void reset_overflow_queue(lmb_lattice *l)
{
    // A new lattice state drops whatever the relaxed handler had queued.
    RunState z;
    memset(&z, 0, sizeof(z));
    *l->rs_host = z;
}

extern "C" int lmb_lattice_set_native(lmb_lattice *l, const uint32_t *particles, const uint8_t *sites)
{
    if (!l || l->pending) return l ? LMB_E_STATE : LMB_E_ARG;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    if (particles)
        CK(cudaMemcpyAsync(l->buf[l->cur], particles, (size_t)l->words * l->g.N * 4, cudaMemcpyHostToDevice, c->stream));
    if (sites) CK(cudaMemcpyAsync(l->sites, sites, l->g.N, cudaMemcpyHostToDevice, c->stream));
    reset_overflow_queue(l);
    CK(cudaMemcpyAsync(l->rs, l->rs_host, sizeof(RunState), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    l->validated = false;
    return LMB_OK;
}

extern "C" int lmb_lattice_get_native(lmb_lattice *l, uint32_t *particles, uint8_t *sites)
{
    if (!l || l->pending) return l ? LMB_E_STATE : LMB_E_ARG;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    if (particles)
        CK(cudaMemcpyAsync(particles, l->buf[l->cur], (size_t)l->words * l->g.N * 4, cudaMemcpyDeviceToHost, c->stream));
    if (sites) CK(cudaMemcpyAsync(sites, l->sites, l->g.N, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return LMB_OK;
}

extern "C" int lmb_lattice_set_row_major(lmb_lattice *l, const void *particles, const uint8_t *sites,
                                         uint32_t number_species, uint32_t number_site_types)
{
    if (!l || !particles || !sites) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    const size_t pbytes = (size_t)l->g.N * l->slots * l->bps;
    void *tmp = nullptr;
    uint8_t *tmp_sites = nullptr;
    CK(cudaMalloc(&tmp, pbytes));
    cudaError_t e = cudaMalloc(&tmp_sites, l->g.N);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, particles, pbytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp_sites, sites, l->g.N, cudaMemcpyHostToDevice, c->stream);
    reset_overflow_queue(l);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l->rs, l->rs_host, sizeof(RunState), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = launch_row_major_to_native((int)l->bps, (int)l->slots, tmp, tmp_sites, l->buf[l->cur], l->sites, l->g,
                                       l->rs, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l->rs_host, l->rs, sizeof(RunState), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (tmp_sites) cudaFree(tmp_sites);
    if (e != cudaSuccess) return cuda_status(e);
    // RDMESolver.cpp:160-185 rejects invalid species ids and site types.
    if (l->rs_host->max_species > number_species || l->rs_host->max_site_type >= number_site_types) {
        return LMB_E_ARG;
    }
    l->validated = false;
    return LMB_OK;
}

extern "C" int lmb_lattice_get_row_major(lmb_lattice *l, void *particles, uint8_t *sites)
{
    if (!l || !particles) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    const size_t pbytes = (size_t)l->g.N * l->slots * l->bps;
    void *tmp = nullptr;
    uint8_t *tmp_sites = nullptr;
    CK(cudaMalloc(&tmp, pbytes));
    cudaError_t e = sites ? cudaMalloc(&tmp_sites, l->g.N) : cudaSuccess;
    if (e == cudaSuccess)
        e = launch_native_to_row_major((int)l->bps, (int)l->slots, l->buf[l->cur], l->sites, tmp, tmp_sites, l->g,
                                       c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(particles, tmp, pbytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && sites) e = cudaMemcpyAsync(sites, tmp_sites, l->g.N, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (tmp_sites) cudaFree(tmp_sites);
    if (e != cudaSuccess) return cuda_status(e);
    return LMB_OK;
}

int lmb::lattice_view(const lmb_lattice *l, LatticeView *v)
{
    if (!l || !v) return LMB_E_ARG;
    v->ctx = l->ctx;
    v->g = l->g;
    v->bytes_per_slot = l->bps;
    v->slots = l->slots;
    v->particles = l->buf[l->cur];
    v->sites = l->sites;
    v->pending = l->pending;
    return LMB_OK;
}

extern "C" int lmb_lattice_device_buffers(lmb_lattice *l, void **particles, void **sites)
{
    if (!l) return LMB_E_ARG;
    if (particles) *particles = l->buf[l->cur];
    if (sites) *sites = l->sites;
    return LMB_OK;
}

// Device counters for ns + 1 species totals (kept between calls).
static int ensure_counts_dev(lmb_lattice *l, uint32_t ns)
{
    if (!l->counts_dev || l->counts_len < ns + 1) {
        if (l->counts_dev) cudaFree(l->counts_dev);
        l->counts_dev = nullptr;
        CK(cudaMalloc(&l->counts_dev, sizeof(unsigned long long) * (ns + 1)));
        l->counts_len = ns + 1;
    }
    return LMB_OK;
}

extern "C" int lmb_lattice_species_counts(lmb_lattice *l, uint32_t ns, uint64_t *counts)
{
    if (!l || !counts) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    int rc = ensure_counts_dev(l, ns);
    if (rc) return rc;
    CK(cudaMemsetAsync(l->counts_dev, 0, sizeof(unsigned long long) * (ns + 1), c->stream));
    CK(launch_counts((int)l->bps, (int)l->slots, l->buf[l->cur], l->g, ns, l->counts_dev, c->stream));
    CK(cudaMemcpyAsync(counts, l->counts_dev, sizeof(uint64_t) * (ns + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    counts[0] = 0;
    return LMB_OK;
}

// ---------------------------------------------------------------------------
// Timesteps
// ---------------------------------------------------------------------------


// ---------------------------------------------------------------------------
// Timestep enqueue and graph capture
// ---------------------------------------------------------------------------

static const uint32_t GRAPH_STEPS = 32;  // even: a replay returns to the same buffer parity

// Plane bounds of buffer b, or null when the lattice keeps none.
static uint32_t *plane_bounds(lmb_lattice *l, int b) { return l->pb ? l->pb + (size_t)b * l->nseg : nullptr; }

// Queues one timestep (schedule of the lattice) and flips the buffer index.
static cudaError_t enqueue_step(lmb_lattice *l, lmb_model *m, cudaStream_t st)
{
    const int bps = (int)l->bps, S = (int)l->slots;
    uint32_t *a = l->buf[l->cur], *b = l->buf[l->cur ^ 1];
    cudaError_t e;
    if (l->schedule == LMB_SCHEDULE_FUSED) {
        e = launch_fused(bps, S, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, l->tile, m->nr > 0, st);
        l->cur ^= 1;
        return e;
    }
    uint32_t *rx = m->nr > 0 ? l->rx_sites : nullptr;
    uint32_t *pa = plane_bounds(l, l->cur), *pbb = plane_bounds(l, l->cur ^ 1);
    if ((e = launch_sweep(bps, S, 0, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, nullptr, 0, pa, pbb,
                          st)) != cudaSuccess)
        return e;
    if ((e = launch_sweep(bps, S, 1, b, a, l->sites, l->g, m->dev, l->rs, l->list, l->cap, nullptr, 0, pbb, pa,
                          st)) != cudaSuccess)
        return e;
    if ((e = launch_sweep(bps, S, 2, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, rx, l->rx_cap, pa, pbb,
                          st)) != cudaSuccess)
        return e;
    l->cur ^= 1;
    if (m->nr > 0 && (e = launch_reaction(bps, S, l->buf[l->cur], l->sites, l->g, m->dev, l->rs, l->list, l->cap,
                                          rx, l->rx_cap, pbb, st)) != cudaSuccess)
        return e;
    return launch_resolve(bps, S, l->buf[l->cur], l->sites, l->g, l->rs, l->list, l->cap, rx ? l->rx_cap : 0, pbb,
                          st);
}

// Both buffers' plane bounds set to every plane: the start of a per-phase
// run, whatever was written to the buffers since the last one.
static cudaError_t reset_plane_bounds(lmb_lattice *l, cudaStream_t st)
{
    if (!l->pb || l->schedule != LMB_SCHEDULE_PHASES) return cudaSuccess;
    return launch_fill_bounds(l->pb, 2 * l->nseg, l->words, st);
}

// Captures GRAPH_STEPS timesteps starting at the current buffer parity, or
// keeps the graph captured before for the same model storage and schedule.
// Every kernel reads the step index from the run state, so one graph serves
// any run.
static int ensure_graph(lmb_lattice *l, lmb_model *m)
{
    lmb_lattice::Graph &gr = l->graph[l->cur];
    const bool same = gr.exec && gr.model == m && gr.tables == m->dev_block && gr.schedule == l->schedule &&
                      gr.Ty == l->tile.Ty && gr.Tz == l->tile.Tz && gr.reaction == (m->nr > 0);
    if (same) return LMB_OK;
    if (gr.exec) {
        cudaGraphExecDestroy(gr.exec);
        gr.exec = nullptr;
    }
    cudaStream_t st = l->ctx->stream;
    const int cur0 = l->cur;
    const uint64_t launches0 = lmb_kernel_launches();
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return LMB_E_UNSUPPORTED;
    }
    cudaError_t e = cudaSuccess;
    for (uint32_t s = 0; s < GRAPH_STEPS && e == cudaSuccess; s++) e = enqueue_step(l, m, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    l->cur = cur0;
    const uint64_t captured = lmb_kernel_launches() - launches0;
    count_launch((uint64_t)0 - captured);  // captured launches run only when replayed
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_status(e != cudaSuccess ? e : e2);
    }
    e = cudaGraphInstantiate(&gr.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        gr.exec = nullptr;
        return cuda_status(e);
    }
    gr.model = m;
    gr.tables = m->dev_block;
    gr.schedule = l->schedule;
    gr.Ty = l->tile.Ty;
    gr.Tz = l->tile.Tz;
    gr.reaction = m->nr > 0;
    gr.kernels = captured;
    return LMB_OK;
}

static int validate_for_model(lmb_lattice *l, const lmb_model *m)
{
    if (!l->validated) {
        lmb_ctx *c = l->ctx;
        CK(cudaMemcpyAsync(l->rs_host, l->rs, sizeof(RunState), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        l->rs_host->max_species = 0;
        l->rs_host->max_site_type = 0;
        CK(cudaMemcpyAsync(l->rs, l->rs_host, sizeof(RunState), cudaMemcpyHostToDevice, c->stream));
        CK(launch_validate((int)l->bps, (int)l->slots, l->buf[l->cur], l->sites, l->g, l->rs, c->stream));
        CK(cudaMemcpyAsync(l->rs_host, l->rs, sizeof(RunState), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        l->max_species = l->rs_host->max_species;
        l->max_site_type = l->rs_host->max_site_type;
        l->validated = true;
    }
    // Species ids index the qp tables unchecked on the device
    // (MpdRdmeSolver.cu:1617-1636), as the reference assumes after
    // RDMESolver::setLatticeData validated them.
    if (l->max_species > m->ns || l->max_site_type >= m->nst) return LMB_E_ARG;
    return LMB_OK;
}

// count_ns ~0u: no species count; otherwise the lattice's species totals at
// the end of the run are taken in the run's own work (lmb_run_counts_async).
// device_check: the lattice's contents were just uploaded in the same
// stream; they are checked by kernels queued ahead of the timesteps (a bad
// species id or site type fails the run with LMB_E_ARG) instead of by a host
// round trip.
static int run_async(lmb_lattice *l, const lmb_model *mc, uint32_t seed, uint32_t first, uint32_t n, int mode,
                     uint32_t count_ns, bool device_check = false)
{
    if (!l || !mc) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    if (mode != LMB_OVERFLOW_CLASSIC && mode != LMB_OVERFLOW_RELAXED) return LMB_E_ARG;
    lmb_model *m = const_cast<lmb_model *>(mc);
    if (m->ctx->device != l->ctx->device) return LMB_E_ARG;
    if (m->has_desc && (m->X != l->g.X || m->Y != l->g.Y || m->Z != l->g.Z)) return LMB_E_ARG;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    if (m->dirty) {
        int rc = upload_model(m);
        if (rc) return rc;
    }
    int rc = device_check ? LMB_OK : validate_for_model(l, m);
    if (rc) return rc;
    const bool counting = count_ns != ~0u;
    // The fused kernel counts in its last launch when its work list can hold
    // the histogram; otherwise one pass over the final lattice follows the run.
    const bool in_kernel = counting && n > 0 && l->schedule == LMB_SCHEDULE_FUSED && count_ns + 1 <= l->tile.R;
    if (counting) {
        rc = ensure_counts_dev(l, count_ns);
        if (rc) return rc;
        if (!l->counts_host || l->counts_host_len < count_ns + 1) {
            if (l->counts_host) cudaFreeHost(l->counts_host);
            l->counts_host = nullptr;
            CK(cudaMallocHost(&l->counts_host, sizeof(unsigned long long) * (count_ns + 1)));
            l->counts_host_len = count_ns + 1;
        }
        CK(cudaMemsetAsync(l->counts_dev, 0, sizeof(unsigned long long) * (count_ns + 1), c->stream));
    }
    // The shared-memory-resident schedules resolve overflows the classic way only.
    if (resident_schedule(l->schedule) && mode != LMB_OVERFLOW_CLASSIC) return LMB_E_UNSUPPORTED;
    CK(launch_begin_run(l->rs, seed, first, n, (uint32_t)mode, c->stream, in_kernel ? first + n - 1 : ~0u, count_ns,
                        l->counts_dev));
    if (device_check) {
        CK(launch_validate((int)l->bps, (int)l->slots, l->buf[l->cur], l->sites, l->g, l->rs, c->stream));
        CK(launch_check_contents(l->rs, m->ns, m->nst, c->stream));
    }
    CK(reset_plane_bounds(l, c->stream));
    l->pending_cur0 = l->cur;
    l->pending_check = device_check;
    uint32_t done = 0;
    if (resident_schedule(l->schedule) && n > 0) {
        // Every timestep in one launch, ending in the buffer n's parity gives.
        CK(launch_resident(l, m, c->stream));
        l->cur ^= (int)(n & 1u);
        done = n;
    }
    // Whole graphs of GRAPH_STEPS timesteps, then single launches.
    // A stream that cannot be captured (the legacy default stream) runs
    // every timestep as single launches.
    if (n >= 2 * GRAPH_STEPS && ensure_graph(l, m) == LMB_OK) {
        lmb_lattice::Graph &gr = l->graph[l->cur];
        for (; done + GRAPH_STEPS <= n; done += GRAPH_STEPS) {
            CK(cudaGraphLaunch(gr.exec, c->stream));
            count_launch(gr.kernels);
        }
    }
    for (; done < n; done++) CK(enqueue_step(l, m, c->stream));
    if (counting) {
        if (!in_kernel) {
            // After a per-phase run the current buffer's plane bounds hold:
            // only the planes below them are read.
            const uint32_t *pb = l->schedule == LMB_SCHEDULE_PHASES && n > 0 ? plane_bounds(l, l->cur) : nullptr;
            CK(launch_counts((int)l->bps, (int)l->slots, l->buf[l->cur], l->g, count_ns, l->counts_dev, c->stream,
                             pb));
        }
        CK(cudaMemcpyAsync(l->counts_host, l->counts_dev, sizeof(unsigned long long) * (count_ns + 1),
                           cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaMemcpyAsync(l->rs_host, l->rs, sizeof(RunState), cudaMemcpyDeviceToHost, c->stream));
    l->pending = true;
    l->pending_first = first;
    l->pending_n = n;
    l->pending_count_ns = count_ns;
    return LMB_OK;
}

extern "C" int lmb_run_async(lmb_lattice *l, const lmb_model *mc, uint32_t seed, uint32_t first, uint32_t n, int mode)
{
    return run_async(l, mc, seed, first, n, mode, ~0u);
}

extern "C" int lmb_run_counts_async(lmb_lattice *l, const lmb_model *mc, uint32_t seed, uint32_t first, uint32_t n,
                                    int mode, uint32_t number_species)
{
    if (number_species == ~0u) return LMB_E_ARG;
    return run_async(l, mc, seed, first, n, mode, number_species);
}

extern "C" int lmb_run_counts_wait(lmb_lattice *l, lmb_run_stats *st, uint64_t *counts)
{
    if (!l || !counts) return LMB_E_ARG;
    if (!l->pending || l->pending_count_ns == ~0u) return LMB_E_STATE;
    const uint32_t ns = l->pending_count_ns;
    const int rc = lmb_run_wait(l, st);
    for (uint32_t s = 0; s <= ns; s++) counts[s] = l->counts_host[s];
    counts[0] = 0;
    return rc;
}

extern "C" int lmb_run_native_async(lmb_lattice *l, const lmb_model *m, uint32_t seed, uint32_t first, uint32_t n,
                                    int mode, const uint32_t *in_particles, const uint8_t *in_sites,
                                    uint32_t *out_particles)
{
    if (!l || !m) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    const size_t bytes = (size_t)l->words * l->g.N * 4;
    if (in_particles || in_sites) {
        // As lmb_lattice_set_native, without its wait; the new contents are
        // checked on the device ahead of the timesteps.
        if (in_particles) CK(cudaMemcpyAsync(l->buf[l->cur], in_particles, bytes, cudaMemcpyHostToDevice, c->stream));
        if (in_sites) CK(cudaMemcpyAsync(l->sites, in_sites, l->g.N, cudaMemcpyHostToDevice, c->stream));
        reset_overflow_queue(l);
        CK(cudaMemcpyAsync(l->rs, l->rs_host, sizeof(RunState), cudaMemcpyHostToDevice, c->stream));
        l->validated = false;
    }
    int rc = run_async(l, m, seed, first, n, mode, ~0u, in_particles || in_sites);
    if (rc) return rc;
    // The buffer the run ends in when it succeeds (run_async tracks the
    // parity as it queues the timesteps).
    if (out_particles)
        CK(cudaMemcpyAsync(out_particles, l->buf[l->cur], bytes, cudaMemcpyDeviceToHost, c->stream));
    return LMB_OK;
}

extern "C" int lmb_run_wait(lmb_lattice *l, lmb_run_stats *st)
{
    if (!l) return LMB_E_ARG;
    if (!l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    l->pending = false;
    CK(cudaStreamSynchronize(c->stream));
    const RunState &h = *l->rs_host;
    uint32_t done = h.status == LMB_OK ? l->pending_n : h.failed_step - l->pending_first;
    const bool refused = l->pending_check && h.status == LMB_E_ARG;
    if (l->pending_check) {
        // The device's check of the contents, kept as the host's would be.
        l->max_species = h.max_species;
        l->max_site_type = h.max_site_type;
        l->validated = true;
        l->pending_check = false;
    }
    if (refused) {
        // Refused before the first timestep: the lattice is where it was.
        done = 0;
        l->cur = l->pending_cur0;
    } else if (h.status != LMB_OK) {
        // Kernels after the failing step did nothing: the lattice sits in the
        // buffer reached after done + 1 steps (each step flips once).
        l->cur = l->pending_cur0 ^ (int)((done + 1) & 1u);
    }
    if (st) {
        st->status = h.status;
        st->steps_done = done;
        st->failed_step = h.status == LMB_OK ? 0 : h.failed_step;
        st->unresolved = h.mode == LMB_OVERFLOW_RELAXED ? h.ovf_count : 0;
        st->overflows = h.overflows;
        st->reactions = h.reactions;
    }
    return h.status;
}

extern "C" int lmb_run_profiled(lmb_lattice *l, const lmb_model *mc, uint32_t seed, uint32_t first, uint32_t n,
                                int mode, float *phase_ms, uint32_t *phase_launches, lmb_run_stats *st)
{
    // Same work as lmb_run with a CUDA event pair around every kernel, on the
    // lattice's stream.  phase order: x, y, z sweeps, reaction, overflow,
    // fused timestep.
    if (!l || !mc || !phase_ms || !phase_launches) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_model *m = const_cast<lmb_model *>(mc);
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    if (m->dirty) {
        int rc = upload_model(m);
        if (rc) return rc;
    }
    int rc = validate_for_model(l, m);
    if (rc) return rc;
    CK(launch_begin_run(l->rs, seed, first, n, (uint32_t)mode, c->stream));
    CK(reset_plane_bounds(l, c->stream));
    std::vector<cudaEvent_t> ev((size_t)n * 12);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    const int bps = (int)l->bps, S = (int)l->slots;
    const int cur0 = l->cur;
    const bool cluster = resident_schedule(l->schedule);
    const bool fused = l->schedule == LMB_SCHEDULE_FUSED || cluster;
    if (cluster && mode != LMB_OVERFLOW_CLASSIC) return LMB_E_UNSUPPORTED;
    for (uint32_t s = 0; s < n; s++) {
        uint32_t *a = l->buf[l->cur], *b = l->buf[l->cur ^ 1];
        cudaEvent_t *E = &ev[(size_t)s * 12];
        if (cluster) {
            // One launch runs every timestep; its time counts under the
            // fused-timestep entry, one launch per timestep.
            CK(cudaEventRecord(E[10], c->stream));
            if (s == 0) {
                CK(launch_resident(l, m, c->stream));
                l->cur ^= (int)(n & 1u);
            }
            CK(cudaEventRecord(E[11], c->stream));
            continue;
        }
        if (fused) {
            CK(cudaEventRecord(E[10], c->stream));
            CK(launch_fused(bps, S, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, l->tile, m->nr > 0,
                            c->stream));
            CK(cudaEventRecord(E[11], c->stream));
            l->cur ^= 1;
            continue;
        }
        CK(cudaEventRecord(E[0], c->stream));
        uint32_t *rx = m->nr > 0 ? l->rx_sites : nullptr;
        uint32_t *pa = plane_bounds(l, l->cur), *pbb = plane_bounds(l, l->cur ^ 1);
        CK(launch_sweep(bps, S, 0, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, nullptr, 0, pa, pbb,
                        c->stream));
        CK(cudaEventRecord(E[1], c->stream));
        CK(cudaEventRecord(E[2], c->stream));
        CK(launch_sweep(bps, S, 1, b, a, l->sites, l->g, m->dev, l->rs, l->list, l->cap, nullptr, 0, pbb, pa,
                        c->stream));
        CK(cudaEventRecord(E[3], c->stream));
        CK(cudaEventRecord(E[4], c->stream));
        CK(launch_sweep(bps, S, 2, a, b, l->sites, l->g, m->dev, l->rs, l->list, l->cap, rx, l->rx_cap, pa, pbb,
                        c->stream));
        CK(cudaEventRecord(E[5], c->stream));
        l->cur ^= 1;
        CK(cudaEventRecord(E[6], c->stream));
        if (m->nr > 0)
            CK(launch_reaction(bps, S, l->buf[l->cur], l->sites, l->g, m->dev, l->rs, l->list, l->cap, rx, l->rx_cap,
                               pbb, c->stream));
        CK(cudaEventRecord(E[7], c->stream));
        CK(cudaEventRecord(E[8], c->stream));
        CK(launch_resolve(bps, S, l->buf[l->cur], l->sites, l->g, l->rs, l->list, l->cap, rx ? l->rx_cap : 0, pbb,
                          c->stream));
        CK(cudaEventRecord(E[9], c->stream));
    }
    CK(cudaMemcpyAsync(l->rs_host, l->rs, sizeof(RunState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int p = 0; p < 6; p++) {
        phase_ms[p] = 0.0f;
        phase_launches[p] = 0;
    }
    for (uint32_t s = 0; s < n; s++)
        for (int p = 0; p < 6; p++) {
            if (fused != (p == 5)) continue;
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ev[(size_t)s * 12 + 2 * p], ev[(size_t)s * 12 + 2 * p + 1]));
            phase_ms[p] += ms;
            if (p != 3 || m->nr > 0) phase_launches[p] += 1;
        }
    for (auto &e : ev) cudaEventDestroy(e);
    const RunState &h = *l->rs_host;
    const uint32_t done = h.status == LMB_OK ? n : h.failed_step - first;
    if (h.status != LMB_OK) l->cur = cur0 ^ (int)((done + 1) & 1u);
    if (st) {
        st->status = h.status;
        st->steps_done = done;
        st->failed_step = h.status == LMB_OK ? 0 : h.failed_step;
        st->unresolved = h.mode == LMB_OVERFLOW_RELAXED ? h.ovf_count : 0;
        st->overflows = h.overflows;
        st->reactions = h.reactions;
    }
    return h.status;
}

extern "C" int lmb_run(lmb_lattice *l, const lmb_model *m, uint32_t seed, uint32_t first, uint32_t n, int mode,
                       lmb_run_stats *st)
{
    int rc = lmb_run_async(l, m, seed, first, n, mode);
    if (rc != LMB_OK) return rc;
    return lmb_run_wait(l, st);
}

// Times each candidate schedule for `timesteps` on a copy of the lattice
// state (restored afterwards) and keeps the fastest.
extern "C" int lmb_lattice_autotune(lmb_lattice *l, const lmb_model *m, uint32_t seed, uint32_t first,
                                    uint32_t timesteps, int *schedule, uint32_t *Ty, uint32_t *Tz, float *best_ms)
{
    if (!l || !m || timesteps == 0) return LMB_E_ARG;
    if (l->pending) return LMB_E_STATE;
    lmb_ctx *c = l->ctx;
    CK(cudaSetDevice(c->device));
    const size_t wbytes = (size_t)l->words * l->g.N * 4;
    uint32_t *save = nullptr;
    CK(cudaMalloc(&save, wbytes));
    cudaError_t e = cudaMemcpyAsync(save, l->buf[l->cur], wbytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) {
        cudaFree(save);
        return cuda_status(e);
    }
    const int cur0 = l->cur;
    const int sched0 = l->schedule;
    const TileShape tile0 = l->tile;
    struct Cand { int sched; uint32_t ty, tz; };
    std::vector<Cand> cands = {{LMB_SCHEDULE_PHASES, 0, 0}, {LMB_SCHEDULE_CLUSTER, 0, 0}};
    const uint32_t dims[] = {1, 2, 4, 8, 16};
    for (uint32_t ty : dims)
        for (uint32_t tz : dims) {
            TileShape t;
            if (fused_make_shape(l->g, (int)l->bps, (int)l->slots, ty, tz, t)) cands.push_back({LMB_SCHEDULE_FUSED, ty, tz});
        }
    // LMB_SCHEDULE_GRID is not a candidate: on one lattice it times as its
    // fused plan does, and its cooperative launch cannot overlap another
    // lattice's run on a second stream, as fused launches do.
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    Cand bestc = {sched0, tile0.Ty, tile0.Tz};
    int rc = LMB_OK;
    for (const Cand &cd : cands) {
        if (lmb_lattice_set_schedule(l, cd.sched, cd.ty, cd.tz) != LMB_OK) continue;
        // warm-up launch, then the timed one, each from the saved state
        for (int rep = 0; rep < 2 && rc == LMB_OK; rep++) {
            l->cur = cur0;
            cudaMemcpyAsync(l->buf[l->cur], save, wbytes, cudaMemcpyDeviceToDevice, c->stream);
            cudaEventRecord(e0, c->stream);
            rc = lmb_run_async(l, m, seed, first, timesteps, LMB_OVERFLOW_CLASSIC);
            if (rc != LMB_OK && resident_schedule(cd.sched) && rc == LMB_E_CUDA) {
                // A cluster the device would not launch: not a candidate.
                cudaGetLastError();
                rc = LMB_OK;
                break;
            }
            if (rc != LMB_OK) break;
            cudaEventRecord(e1, c->stream);
            lmb_run_stats st;
            rc = lmb_run_wait(l, &st);
            if (rc != LMB_OK) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 1 && ms < best) {
                best = ms;
                bestc = cd;
            }
        }
        if (rc != LMB_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    l->cur = cur0;
    cudaMemcpyAsync(l->buf[l->cur], save, wbytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(save);
    if (rc != LMB_OK) {
        l->schedule = sched0;
        l->tile = tile0;
        return rc;
    }
    lmb_lattice_set_schedule(l, bestc.sched, bestc.ty, bestc.tz);
    if (schedule) *schedule = bestc.sched;
    if (Ty) *Ty = bestc.ty;
    if (Tz) *Tz = bestc.tz;
    if (best_ms) *best_ms = best;
    return LMB_OK;
}

// ---------------------------------------------------------------------------
// Batches: many lattices advanced by one launch per timestep
// ---------------------------------------------------------------------------

struct lmb_batch {
    lmb_ctx *ctx;
    std::vector<lmb_lattice *> lats;
    std::vector<const lmb_model *> models;
    int bps, slots;
    uint32_t capacity;  // lattices the device arrays hold
    // Device side: job table, run-state pointers, seeds, per-lattice
    // timestep ranges, gathered states.
    FusedJob *jobs;
    RunState **rs_ptrs;
    uint32_t *seeds;
    uint32_t *firsts;
    uint32_t *counts;
    RunState *states;
    RunState *states_host;  // pinned
    std::vector<FusedJob> jobs_host;
    std::vector<TileShape> tiles;  // batch plan per lattice
    uint32_t total_tiles;
    size_t smem;
    cudaGraphExec_t graph;
    uint64_t graph_kernels;
    uint32_t graph_tiles;  // launch shape the graph was captured with
    uint32_t graph_jobs;
    size_t graph_smem;
    bool pending;
    std::vector<uint32_t> pending_first, pending_n;
    std::vector<int> cur0;
    // Tiles lmb_batch_autotune chose, by lattice size (X, Y, Z): used for
    // every member of that size, now and after lmb_batch_set_lattices.
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, std::pair<uint32_t, uint32_t>> tuned;
};

static const uint32_t BATCH_GRAPH_STEPS = 32;

static std::tuple<uint32_t, uint32_t, uint32_t> size_key(const Geometry &g) { return {g.X, g.Y, g.Z}; }

static void batch_free_arrays(lmb_batch *b)
{
    if (b->jobs) cudaFree(b->jobs);
    if (b->rs_ptrs) cudaFree(b->rs_ptrs);
    if (b->seeds) cudaFree(b->seeds);
    if (b->firsts) cudaFree(b->firsts);
    if (b->counts) cudaFree(b->counts);
    if (b->states) cudaFree(b->states);
    if (b->states_host) cudaFreeHost(b->states_host);
    b->jobs = nullptr;
    b->rs_ptrs = nullptr;
    b->seeds = b->firsts = b->counts = nullptr;
    b->states = b->states_host = nullptr;
    b->capacity = 0;
}

static int batch_reserve(lmb_batch *b, uint32_t count)
{
    if (count <= b->capacity) return LMB_OK;
    CK(cudaStreamSynchronize(b->ctx->stream));
    batch_free_arrays(b);
    cudaError_t e = cudaMalloc(&b->jobs, sizeof(FusedJob) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->rs_ptrs, sizeof(RunState *) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->seeds, sizeof(uint32_t) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->firsts, sizeof(uint32_t) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->counts, sizeof(uint32_t) * count);
    if (e == cudaSuccess) e = cudaMalloc(&b->states, sizeof(RunState) * count);
    if (e == cudaSuccess) e = cudaMallocHost(&b->states_host, sizeof(RunState) * count);
    if (e != cudaSuccess) {
        batch_free_arrays(b);
        return cuda_status(e);
    }
    b->capacity = count;
    return LMB_OK;
}

// Checks and plans a member set; fills `plan`.
static int batch_check_members(lmb_ctx *c, uint32_t count, lmb_lattice *const *lattices,
                               const lmb_model *const *models, int bps, int slots, std::vector<TileShape> &plan)
{
    plan.resize(count);
    for (uint32_t j = 0; j < count; j++) {
        lmb_lattice *l = lattices[j];
        const lmb_model *m = models[j];
        if (!l || !m || l->ctx != c || m->ctx != c) return LMB_E_ARG;
        if ((int)l->bps != bps || (int)l->slots != slots) return LMB_E_ARG;
        if (m->has_desc && (m->X != l->g.X || m->Y != l->g.Y || m->Z != l->g.Z)) return LMB_E_ARG;
        if (!fused_batch_shape(l->g, bps, slots, plan[j])) return LMB_E_UNSUPPORTED;
    }
    return LMB_OK;
}

static int batch_set(lmb_batch *b, uint32_t count, lmb_lattice *const *lattices, const lmb_model *const *models,
                     std::vector<TileShape> &plan)
{
    int rc = batch_reserve(b, count);
    if (rc) return rc;
    for (uint32_t j = 0; j < count; j++) {
        const auto it = b->tuned.find(size_key(lattices[j]->g));
        TileShape t;
        if (it != b->tuned.end() &&
            fused_batch_shape_ok(lattices[j]->g, b->bps, b->slots, it->second.first, it->second.second, t))
            plan[j] = t;
    }
    b->lats.assign(lattices, lattices + count);
    b->models.assign(models, models + count);
    b->tiles.swap(plan);
    std::vector<RunState *> ptrs(count);
    for (uint32_t j = 0; j < count; j++) ptrs[j] = lattices[j]->rs;
    CK(cudaMemcpyAsync(b->rs_ptrs, ptrs.data(), sizeof(RunState *) * count, cudaMemcpyHostToDevice,
                       b->ctx->stream));
    CK(cudaStreamSynchronize(b->ctx->stream));
    return LMB_OK;
}

extern "C" int lmb_batch_create(lmb_ctx *c, uint32_t count, lmb_lattice *const *lattices,
                                const lmb_model *const *models, lmb_batch **out)
{
    if (!c || !lattices || !models || !out || count == 0 || !lattices[0]) return LMB_E_ARG;
    *out = nullptr;
    const int bps = (int)lattices[0]->bps, slots = (int)lattices[0]->slots;
    std::vector<TileShape> plan;
    int rc = batch_check_members(c, count, lattices, models, bps, slots, plan);
    if (rc) return rc;
    CK(cudaSetDevice(c->device));
    lmb_batch *b = new (std::nothrow) lmb_batch;
    if (!b) return LMB_E_NOMEM;
    b->ctx = c;
    ctx_retain(c);
    b->bps = bps;
    b->slots = slots;
    b->capacity = 0;
    b->jobs = nullptr;
    b->rs_ptrs = nullptr;
    b->seeds = b->firsts = b->counts = nullptr;
    b->states = nullptr;
    b->states_host = nullptr;
    b->graph = nullptr;
    b->graph_kernels = 0;
    b->graph_tiles = 0;
    b->graph_jobs = 0;
    b->graph_smem = 0;
    b->pending = false;
    b->total_tiles = 0;
    b->smem = 0;
    rc = batch_set(b, count, lattices, models, plan);
    if (rc) {
        lmb_batch_destroy(b);
        return rc;
    }
    *out = b;
    return LMB_OK;
}

extern "C" int lmb_batch_set_lattices(lmb_batch *b, uint32_t count, lmb_lattice *const *lattices,
                                      const lmb_model *const *models)
{
    if (!b || !lattices || !models || count == 0) return LMB_E_ARG;
    if (b->pending) return LMB_E_STATE;
    std::vector<TileShape> plan;
    int rc = batch_check_members(b->ctx, count, lattices, models, b->bps, b->slots, plan);
    if (rc) return rc;
    CK(cudaSetDevice(b->ctx->device));
    return batch_set(b, count, lattices, models, plan);
}

extern "C" int lmb_batch_destroy(lmb_batch *b)
{
    if (!b) return LMB_E_ARG;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    batch_free_arrays(b);
    lmb_ctx *c = b->ctx;
    delete b;
    ctx_release(c);
    return LMB_OK;
}

// Fills the job table for a run starting from every lattice's current buffer.
static int batch_prepare(lmb_batch *b)
{
    const uint32_t count = (uint32_t)b->lats.size();
    b->jobs_host.resize(count);
    b->cur0.resize(count);
    uint32_t tiles = 0;
    size_t smem = 0;
    for (uint32_t j = 0; j < count; j++) {
        lmb_lattice *l = b->lats[j];
        lmb_model *m = const_cast<lmb_model *>(b->models[j]);
        if (l->pending) return LMB_E_STATE;
        if (m->dirty) {
            int rc = upload_model(m);
            if (rc) return rc;
        }
        int rc = validate_for_model(l, m);
        if (rc) return rc;
        FusedJob &jb = b->jobs_host[j];
        jb.buf[0] = l->buf[0];
        jb.buf[1] = l->buf[1];
        jb.sites = l->sites;
        jb.g = l->g;
        jb.m = m->dev;
        jb.rs = l->rs;
        jb.list = l->list;
        jb.cap = l->cap;
        jb.ts = b->tiles[j];
        jb.with_reaction = m->nr > 0;
        jb.cur0 = (uint32_t)l->cur;
        jb.tile_begin = tiles;
        b->cur0[j] = l->cur;
        tiles += b->tiles[j].tiles_y * b->tiles[j].tiles_z;
        const size_t sm = fused_smem_bytes(b->tiles[j], l->g.X, l->words, l->cap, m->dev.stage_bytes);
        if (sm > smem) smem = sm;
    }
    b->total_tiles = tiles;
    b->smem = smem;
    CK(cudaMemcpyAsync(b->jobs, b->jobs_host.data(), sizeof(FusedJob) * count, cudaMemcpyHostToDevice,
                       b->ctx->stream));
    return LMB_OK;
}

// Queues a batch run: lattice j advances through timesteps firsts[j] ..
// firsts[j] + counts[j] - 1 (or first .. first + n - 1 for all when the
// arrays are null); the launch count is the longest range, and a lattice
// whose range is done sits out the remaining launches.
static int batch_run(lmb_batch *b, const uint32_t *seeds, uint32_t first, uint32_t n, const uint32_t *firsts,
                     const uint32_t *counts, int mode)
{
    if (!b || !seeds) return LMB_E_ARG;
    if (b->pending) return LMB_E_STATE;
    if (mode != LMB_OVERFLOW_CLASSIC && mode != LMB_OVERFLOW_RELAXED) return LMB_E_ARG;
    lmb_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    int rc = batch_prepare(b);
    if (rc) return rc;
    const uint32_t count = (uint32_t)b->lats.size();
    b->pending_first.assign(count, first);
    b->pending_n.assign(count, n);
    uint32_t launches = n;
    if (firsts && counts) {
        launches = 0;
        for (uint32_t j = 0; j < count; j++) {
            b->pending_first[j] = firsts[j];
            b->pending_n[j] = counts[j];
            if (counts[j] > launches) launches = counts[j];
        }
        CK(cudaMemcpyAsync(b->firsts, firsts, sizeof(uint32_t) * count, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(b->counts, counts, sizeof(uint32_t) * count, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaMemcpyAsync(b->seeds, seeds, sizeof(uint32_t) * count, cudaMemcpyHostToDevice, c->stream));
    CK(launch_begin_batch(b->rs_ptrs, b->seeds, count, first, n, firsts && counts ? b->firsts : nullptr,
                          firsts && counts ? b->counts : nullptr, (uint32_t)mode, c->stream));
    uint32_t done = 0;
    if (launches >= 2 * BATCH_GRAPH_STEPS) {
        // One graph of BATCH_GRAPH_STEPS launches (parities 0, 1, ...) serves
        // every run: the job table it reads is rewritten before each run.
        static_assert(BATCH_GRAPH_STEPS % 2 == 0, "graph must return to parity 0");
        if (b->graph && (b->graph_tiles != b->total_tiles || b->graph_smem != b->smem || b->graph_jobs != count)) {
            cudaGraphExecDestroy(b->graph);  // the member set or a tile plan changed
            b->graph = nullptr;
        }
        if (!b->graph) {
            const uint64_t l0 = lmb_kernel_launches();
            if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                cudaError_t e = cudaSuccess;
                for (uint32_t s = 0; s < BATCH_GRAPH_STEPS && e == cudaSuccess; s++)
                    e = launch_fused_batch(b->bps, b->slots, b->jobs, count, b->total_tiles, b->smem, s & 1u, c->stream);
                cudaGraph_t graph = nullptr;
                const cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
                const uint64_t captured = lmb_kernel_launches() - l0;
                count_launch((uint64_t)0 - captured);
                if (e == cudaSuccess && e2 == cudaSuccess && cudaGraphInstantiate(&b->graph, graph, 0) == cudaSuccess) {
                    b->graph_kernels = captured;
                    b->graph_tiles = b->total_tiles;
                    b->graph_jobs = count;
                    b->graph_smem = b->smem;
                } else {
                    b->graph = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
            } else {
                cudaGetLastError();
            }
        }
        if (b->graph) {
            for (; done + BATCH_GRAPH_STEPS <= launches; done += BATCH_GRAPH_STEPS) {
                CK(cudaGraphLaunch(b->graph, c->stream));
                count_launch(b->graph_kernels);
            }
        }
    }
    for (; done < launches; done++)
        CK(launch_fused_batch(b->bps, b->slots, b->jobs, count, b->total_tiles, b->smem, done & 1u, c->stream));
    CK(launch_gather_states(b->rs_ptrs, count, b->states, c->stream));
    CK(cudaMemcpyAsync(b->states_host, b->states, sizeof(RunState) * count, cudaMemcpyDeviceToHost, c->stream));
    b->pending = true;
    for (lmb_lattice *l : b->lats) l->pending = true;
    return LMB_OK;
}

extern "C" int lmb_batch_run_async(lmb_batch *b, const uint32_t *seeds, uint32_t first, uint32_t n, int mode)
{
    return batch_run(b, seeds, first, n, nullptr, nullptr, mode);
}

extern "C" int lmb_batch_run_ranges_async(lmb_batch *b, const uint32_t *seeds, const uint32_t *firsts,
                                          const uint32_t *counts, int mode)
{
    if (!firsts || !counts) return LMB_E_ARG;
    return batch_run(b, seeds, 0, 0, firsts, counts, mode);
}

extern "C" int lmb_batch_wait(lmb_batch *b, lmb_run_stats *stats)
{
    if (!b) return LMB_E_ARG;
    if (!b->pending) return LMB_E_STATE;
    lmb_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    b->pending = false;
    for (lmb_lattice *l : b->lats) l->pending = false;
    CK(cudaStreamSynchronize(c->stream));
    int first_error = LMB_OK;
    for (size_t j = 0; j < b->lats.size(); j++) {
        const RunState &h = b->states_host[j];
        lmb_lattice *l = b->lats[j];
        const uint32_t done = h.status == LMB_OK ? b->pending_n[j] : h.failed_step - b->pending_first[j];
        l->cur = b->cur0[j] ^ (int)((h.status == LMB_OK ? done : done + 1) & 1u);
        if (stats) {
            stats[j].status = h.status;
            stats[j].steps_done = done;
            stats[j].failed_step = h.status == LMB_OK ? 0 : h.failed_step;
            stats[j].unresolved = h.mode == LMB_OVERFLOW_RELAXED ? h.ovf_count : 0;
            stats[j].overflows = h.overflows;
            stats[j].reactions = h.reactions;
        }
        if (h.status != LMB_OK && first_error == LMB_OK) first_error = h.status;
    }
    return first_error;
}

extern "C" int lmb_batch_run(lmb_batch *b, const uint32_t *seeds, uint32_t first, uint32_t n, int mode,
                             lmb_run_stats *stats)
{
    int rc = lmb_batch_run_async(b, seeds, first, n, mode);
    if (rc != LMB_OK) return rc;
    return lmb_batch_wait(b, stats);
}

extern "C" int lmb_batch_autotune(lmb_batch *b, const uint32_t *seeds, uint32_t first, uint32_t timesteps,
                                  float *best_ms)
{
    // Per lattice size, largest total size first: every tile shape a batch
    // may use is timed on the whole batch (the launch's shared memory is the
    // largest any member needs, so the choices interact), each trial from
    // the same saved states; the fastest stays.  The lattices end where they
    // started.
    if (!b || !seeds || timesteps == 0) return LMB_E_ARG;
    if (b->pending) return LMB_E_STATE;
    lmb_ctx *c = b->ctx;
    CK(cudaSetDevice(c->device));
    const uint32_t count = (uint32_t)b->lats.size();
    std::vector<size_t> off(count);
    size_t total = 0;
    for (uint32_t j = 0; j < count; j++) {
        off[j] = total;
        total += (size_t)b->lats[j]->words * b->lats[j]->g.N * sizeof(uint32_t);
    }
    uint8_t *save = nullptr;
    CK(cudaMalloc(&save, total));
    std::vector<int> cur0(count);
    for (uint32_t j = 0; j < count; j++) {
        lmb_lattice *l = b->lats[j];
        cur0[j] = l->cur;
        cudaMemcpyAsync(save + off[j], l->buf[l->cur], (size_t)l->words * l->g.N * 4, cudaMemcpyDeviceToDevice,
                        c->stream);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto restore = [&]() {
        for (uint32_t j = 0; j < count; j++) {
            lmb_lattice *l = b->lats[j];
            l->cur = cur0[j];
            cudaMemcpyAsync(l->buf[l->cur], save + off[j], (size_t)l->words * l->g.N * 4,
                            cudaMemcpyDeviceToDevice, c->stream);
        }
    };
    // Time of one trial (the better of two), or a large value when it fails.
    auto trial = [&]() -> float {
        float best = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            restore();
            cudaEventRecord(e0, c->stream);
            if (batch_run(b, seeds, first, timesteps, nullptr, nullptr, LMB_OVERFLOW_CLASSIC) != LMB_OK) return 1e30f;
            cudaEventRecord(e1, c->stream);
            if (lmb_batch_wait(b, nullptr) != LMB_OK) return 1e30f;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms;
        }
        return best;
    };
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, std::vector<uint32_t>> classes;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, uint64_t> sites;
    for (uint32_t j = 0; j < count; j++) {
        classes[size_key(b->lats[j]->g)].push_back(j);
        sites[size_key(b->lats[j]->g)] += b->lats[j]->g.N;
    }
    std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> order;
    for (auto &kv : classes) order.push_back(kv.first);
    std::sort(order.begin(), order.end(), [&](const auto &a, const auto &z) { return sites[a] > sites[z]; });
    trial();  // warm-up
    float best = trial();
    const uint32_t cands[] = {1, 2, 4, 8, 16};
    for (const auto &key : order) {
        const std::vector<uint32_t> &members = classes[key];
        const Geometry g = b->lats[members[0]]->g;
        TileShape keep = b->tiles[members[0]];
        for (uint32_t Ty : cands)
            for (uint32_t Tz : cands) {
                TileShape t;
                if (!fused_batch_shape_ok(g, b->bps, b->slots, Ty, Tz, t)) continue;
                if (t.Ty == keep.Ty && t.Tz == keep.Tz) continue;
                for (uint32_t j : members) b->tiles[j] = t;
                const float ms = trial();
                if (ms < best) {
                    best = ms;
                    keep = t;
                }
            }
        for (uint32_t j : members) b->tiles[j] = keep;
        b->tuned[key] = {keep.Ty, keep.Tz};
    }
    restore();
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_status(e);
    if (best_ms) *best_ms = best;
    return LMB_OK;
}

extern "C" int lmb_batch_plan(lmb_batch *b, uint32_t *Ty, uint32_t *Tz)
{
    if (!b || !Ty || !Tz) return LMB_E_ARG;
    for (size_t j = 0; j < b->tiles.size(); j++) {
        Ty[j] = b->tiles[j].Ty;
        Tz[j] = b->tiles[j].Tz;
    }
    return LMB_OK;
}
