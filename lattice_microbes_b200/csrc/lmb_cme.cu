// lmb_cme.cu -- well-mixed CME ensembles on the GPU: the direct method of
// lm::cme::GillespieDSolver (cme/GillespieDSolver.cpp:107-382) for many
// independent replicates, one thread per replicate.
//
// Per event, as the reference does: draw an exponential and a uniform number,
// advance time by expR / a0, record the counts at every write time passed
// (counts before the event), pick the reaction by a linear scan of the
// propensities with the last reaction as the fallback, apply its
// stoichiometry, recompute the dependent propensities and the total.
// Differences by design: species counts are int32 and propensities FP32 (time
// stays FP64); the random numbers come from the counter hash of the MPD
// solver keyed by (seed, replicate, event), so that a replicate's trajectory
// does not depend on how the ensemble is cut into launches or on which other
// replicates run beside it.
//
// The run can be cut into time segments: a replicate pauses before an event
// whose time lies past the segment end and resumes with it, so any cut gives
// the trajectory of one uninterrupted run.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_internal.h"

using namespace lmb;

namespace {

constexpr int CME_MAX_SPECIES = 32;
constexpr int CME_MAX_REACTIONS = 64;
constexpr int CME_THREADS = 128;

// Model in device memory (and staged into shared memory by each block).
struct CmeModel {
    uint32_t ns, nr;
    uint32_t type[CME_MAX_REACTIONS];
    float k[CME_MAX_REACTIONS];
    uint32_t s1[CME_MAX_REACTIONS], s2[CME_MAX_REACTIONS];
    // Reactions whose propensity changes when reaction r fires.
    unsigned long long dep[CME_MAX_REACTIONS];
    // Sparse stoichiometry: nonzero changes of reaction r at
    // [off[r], off[r+1]).
    uint32_t off[CME_MAX_REACTIONS + 1];
    uint8_t sp[CME_MAX_REACTIONS * CME_MAX_SPECIES];
    int32_t d[CME_MAX_REACTIONS * CME_MAX_SPECIES];
    // Compact form (models of up to 8 species and 16 reactions whose
    // changes lie in -8..7): reaction r's type | s1 << 2 | s2 << 7, and its
    // change of species s in bits 4s..4s+3 (two's complement).
    uint32_t code[CME_MAX_REACTIONS];
    uint32_t delta4[CME_MAX_REACTIONS];
    uint32_t compact;
};

// Per-replicate state, structure of arrays.
struct CmeState {
    int32_t *counts;            // [ns][reps]
    double *t;                  // time of the last event applied
    double *t_next;             // time of the pending event (INFINITY: none)
    double *next_write;         // next recording time
    uint32_t *next_entry;       // next recording index
    unsigned long long *events; // events applied
    uint32_t *done;             // 1 once the trajectory reached t_end
};

// Count of species s from the register array without dynamic indexing.
template <int NS>
__device__ __forceinline__ int32_t getx(const int32_t (&x)[NS], uint32_t s)
{
    int32_t v = 0;
#pragma unroll
    for (int q = 0; q < NS; q++)
        if ((uint32_t)q == s) v = x[q];
    return v;
}

// Propensity of reaction r (CMESolver.cpp:797-822) in FP32: k, k*x,
// k*x1*x2, and k*x*(x-1)/2 for a homodimer.
template <int NS>
__device__ __forceinline__ float propensity(const CmeModel &m, int r, const int32_t (&x)[NS])
{
    const float k = m.k[r];
    switch (m.type[r]) {
    case LMB_REACTION_ZEROTH: return k;
    case LMB_REACTION_FIRST: return __fmul_rn(k, (float)getx(x, m.s1[r]));
    case LMB_REACTION_SECOND:
        return __fmul_rn(__fmul_rn(k, (float)getx(x, m.s1[r])), (float)getx(x, m.s2[r]));
    default: {
        const int32_t n = getx(x, m.s1[r]);
        if (n < 2) return 0.0f;
        return __fmul_rn(__fmul_rn(__fmul_rn(0.5f, k), (float)n), (float)(n - 1));
    }
    }
}

// Exponential variate for event ev: u in (0, 1] from the event's first draw,
// -log(u).
__device__ __forceinline__ float exp_draw(unsigned long long ev, unsigned long long th)
{
    const uint32_t r = mix_hash(ev << 1, th);
    const float u = __fmul_rn((float)r + 1.0f, 2.32830643654e-10f);
    return -logf(u);
}

template <int NR>
__device__ __forceinline__ float total(const float (&a)[NR], uint32_t nr)
{
    float a0 = 0.0f;
#pragma unroll
    for (int q = 0; q < NR; q++)
        if ((uint32_t)q < nr) a0 = __fadd_rn(a0, a[q]);
    return a0;
}

template <int NS, int NR>
__global__ void __launch_bounds__(CME_THREADS) cme_segment_kernel(const CmeModel *__restrict__ gm, CmeState st,
                                                                  int32_t *__restrict__ out, uint32_t reps,
                                                                  uint32_t entries, uint32_t seed, double seg_end,
                                                                  double t_end, double write_interval)
{
    __shared__ CmeModel m;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(gm);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&m);
        for (uint32_t i = threadIdx.x; i < sizeof(CmeModel) / 4; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const uint32_t rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= reps || st.done[rep]) return;

    const uint32_t ns = m.ns, nr = m.nr;
    int32_t x[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) x[s] = (uint32_t)s < ns ? st.counts[(size_t)s * reps + rep] : 0;
    float a[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) a[q] = (uint32_t)q < nr ? propensity(m, q, x) : 0.0f;

    const unsigned long long th = timestep_hash(seed, rep, 0);
    double t = st.t[rep];
    double t_next = st.t_next[rep];
    double next_write = st.next_write[rep];
    uint32_t next_entry = st.next_entry[rep];
    unsigned long long ev = st.events[rep];
    bool finished = false;

    // Records the current counts at every write time up to `limit`.
    auto record_until = [&](double limit) {
        while (next_entry < entries && next_write <= limit) {
#pragma unroll
            for (int s = 0; s < NS; s++)
                if ((uint32_t)s < ns) out[((size_t)next_entry * ns + s) * reps + rep] = x[s];
            next_entry++;
            next_write += write_interval;
        }
    };

    for (;;) {
        if (t_next >= t_end) {  // the reference stops at maxTime (or when a0 = 0)
            t = t_end;
            record_until(t_end + 1e-9);
            finished = true;
            break;
        }
        if (t_next >= seg_end) break;  // resume with this event in the next segment
        record_until(t_next + 1e-9);   // counts before the event
        // Which reaction: linear scan, the last reaction as the fallback
        // (GillespieDSolver.cpp:222-230).
        const float a0 = total(a, nr);
        const float u = __fmul_rn(__uint2float_rn(mix_hash((ev << 1) | 1ull, th)), 2.32830643654e-10f);
        float rv = __fmul_rn(u, a0);
        uint32_t pick = nr - 1;
        bool found = false;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            if ((uint32_t)q + 1 < nr && !found) {
                if (rv < a[q]) {
                    pick = q;
                    found = true;
                } else {
                    rv = __fsub_rn(rv, a[q]);
                }
            }
        }
        for (uint32_t j = m.off[pick]; j < m.off[pick + 1]; j++) {
            const uint32_t s = m.sp[j];
            const int32_t d = m.d[j];
#pragma unroll
            for (int q = 0; q < NS; q++)
                if ((uint32_t)q == s) x[q] += d;
        }
        const unsigned long long dep = m.dep[pick];
#pragma unroll
        for (int q = 0; q < NR; q++)
            if ((uint32_t)q < nr && ((dep >> q) & 1ull)) a[q] = propensity(m, q, x);
        t = t_next;
        ev++;
        const float a1 = total(a, nr);
        t_next = a1 > 0.0f ? t + (double)exp_draw(ev, th) / (double)a1 : INFINITY;
    }

#pragma unroll
    for (int s = 0; s < NS; s++)
        if ((uint32_t)s < ns) st.counts[(size_t)s * reps + rep] = x[s];
    st.t[rep] = t;
    st.t_next[rep] = t_next;
    st.next_write[rep] = next_write;
    st.next_entry[rep] = next_entry;
    st.events[rep] = ev;
    if (finished) st.done[rep] = 1;
}

// The segment kernel for compact models: each reaction's rate and reactant
// code live in registers, its change vector is one shared word, and the
// total propensity is carried from one event to the next.  The arithmetic
// is the generic kernel's, operation for operation, so the trajectories are
// the same bit for bit.
template <int NS, int NR>
__global__ void __launch_bounds__(CME_THREADS) cme_compact_kernel(const CmeModel *__restrict__ gm, CmeState st,
                                                                  int32_t *__restrict__ out, uint32_t reps,
                                                                  uint32_t entries, uint32_t seed, double seg_end,
                                                                  double t_end, double write_interval)
{
    static_assert(NS <= 8 && NR <= 32, "compact models have at most 8 species");
    __shared__ uint32_t s_delta[NR];
    __shared__ unsigned long long s_dep[NR];
    const uint32_t nr = gm->nr, ns = gm->ns;
    float kq[NR];
    uint32_t code[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        kq[q] = (uint32_t)q < nr ? gm->k[q] : 0.0f;
        code[q] = (uint32_t)q < nr ? gm->code[q] : 0u;
    }
    for (uint32_t q = threadIdx.x; q < NR; q += blockDim.x) {
        s_delta[q] = q < nr ? gm->delta4[q] : 0u;
        s_dep[q] = q < nr ? gm->dep[q] : 0ull;
    }
    __syncthreads();
    const uint32_t rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= reps || st.done[rep]) return;

    int32_t x[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) x[s] = (uint32_t)s < ns ? st.counts[(size_t)s * reps + rep] : 0;
    // Propensity of reaction q (CMESolver.cpp:797-822), as propensity().
    auto prop = [&](int q) {
        const uint32_t c = code[q], type = c & 3u;
        const float k = kq[q];
        const int32_t n1 = getx(x, (c >> 2) & 31u);
        if (type == LMB_REACTION_ZEROTH) return k;
        if (type == LMB_REACTION_FIRST) return __fmul_rn(k, (float)n1);
        if (type == LMB_REACTION_SECOND) return __fmul_rn(__fmul_rn(k, (float)n1), (float)getx(x, (c >> 7) & 31u));
        if (n1 < 2) return 0.0f;
        return __fmul_rn(__fmul_rn(__fmul_rn(0.5f, k), (float)n1), (float)(n1 - 1));
    };
    float a[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) a[q] = (uint32_t)q < nr ? prop(q) : 0.0f;
    float atot = total(a, nr);

    const unsigned long long th = timestep_hash(seed, rep, 0);
    double t = st.t[rep];
    double t_next = st.t_next[rep];
    double next_write = st.next_write[rep];
    uint32_t next_entry = st.next_entry[rep];
    unsigned long long ev = st.events[rep];
    bool finished = false;

    auto record_until = [&](double limit) {
        while (next_entry < entries && next_write <= limit) {
#pragma unroll
            for (int s = 0; s < NS; s++)
                if ((uint32_t)s < ns) out[((size_t)next_entry * ns + s) * reps + rep] = x[s];
            next_entry++;
            next_write += write_interval;
        }
    };

    for (;;) {
        if (t_next >= t_end) {
            t = t_end;
            record_until(t_end + 1e-9);
            finished = true;
            break;
        }
        if (t_next >= seg_end) break;
        record_until(t_next + 1e-9);
        const float u = __fmul_rn(__uint2float_rn(mix_hash((ev << 1) | 1ull, th)), 2.32830643654e-10f);
        float rv = __fmul_rn(u, atot);
        uint32_t pick = nr - 1;
        bool found = false;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            if ((uint32_t)q + 1 < nr && !found) {
                if (rv < a[q]) {
                    pick = q;
                    found = true;
                } else {
                    rv = __fsub_rn(rv, a[q]);
                }
            }
        }
        const uint32_t dv = s_delta[pick];
#pragma unroll
        for (int s = 0; s < NS; s++) x[s] += (int32_t)(dv << (28 - 4 * s)) >> 28;
        const unsigned long long dep = s_dep[pick];
#pragma unroll
        for (int q = 0; q < NR; q++)
            if ((uint32_t)q < nr && ((dep >> q) & 1ull)) a[q] = prop(q);
        t = t_next;
        ev++;
        atot = total(a, nr);
        t_next = atot > 0.0f ? t + (double)exp_draw(ev, th) / (double)atot : INFINITY;
    }

#pragma unroll
    for (int s = 0; s < NS; s++)
        if ((uint32_t)s < ns) st.counts[(size_t)s * reps + rep] = x[s];
    st.t[rep] = t;
    st.t_next[rep] = t_next;
    st.next_write[rep] = next_write;
    st.next_entry[rep] = next_entry;
    st.events[rep] = ev;
    if (finished) st.done[rep] = 1;
}

// Sets up every replicate at t = 0: counts and the first event's time; the
// first segment records entry 0.
template <int NS, int NR>
__global__ void cme_begin_kernel(const CmeModel *__restrict__ gm, CmeState st, const int32_t *__restrict__ init,
                                 uint32_t per_replicate, uint32_t reps, uint32_t seed)
{
    const uint32_t rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= reps) return;
    const CmeModel &m = *gm;
    int32_t x[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        x[s] = 0;
        if ((uint32_t)s < m.ns) {
            x[s] = init[per_replicate ? (size_t)rep * m.ns + s : (size_t)s];
            st.counts[(size_t)s * reps + rep] = x[s];
        }
    }
    float a[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) a[q] = (uint32_t)q < m.nr ? propensity(m, q, x) : 0.0f;
    const float a0 = total(a, m.nr);
    const unsigned long long th = timestep_hash(seed, rep, 0);
    st.t[rep] = 0.0;
    st.t_next[rep] = a0 > 0.0f ? (double)exp_draw(0, th) / (double)a0 : INFINITY;
    st.next_write[rep] = 0.0;
    st.next_entry[rep] = 0;
    st.events[rep] = 0;
    st.done[rep] = 0;
}

}  // namespace

struct lmb_cme {
    lmb_ctx *ctx;
    uint32_t ns, nr, reps;
    CmeModel host;
    CmeModel *dev_model;
    void *state_block;
    CmeState st;
    int32_t *init_dev;
    uint32_t init_per_replicate;
    int32_t *out;
    size_t out_entries;
    uint32_t entries;
    double t_end, write_interval;
    uint32_t seed;
    double t_done;
    bool begun;
    int kernel;  // LMB_CME_KERNEL_*
};

#define CKC(call)                                                                    \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) return e_ == cudaErrorMemoryAllocation ? LMB_E_NOMEM : LMB_E_CUDA; \
    } while (0)

// The number of entries GillespieDSolver records for a run to t_end: one at
// t = 0, then every write interval up to t_end + 1e-9, the write time advanced
// by repeated addition (GillespieDSolver.cpp:145-147, 202-213, 329-338).
static uint32_t entries_for(double t_end, double dt)
{
    uint32_t n = 1;
    double w = dt;
    while (w <= t_end + 1e-9 && n < (1u << 30)) {
        n++;
        w += dt;
    }
    return n;
}

extern "C" int lmb_cme_create(lmb_ctx *ctx, uint32_t ns, uint32_t nr, const uint32_t *rtype, const double *K,
                              uint32_t k_cols, const int32_t *S, const uint32_t *D, uint32_t replicates,
                              lmb_cme **out)
{
    if (!ctx || !out || !rtype || !K || !S || !D || replicates == 0 || k_cols == 0) return LMB_E_ARG;
    *out = nullptr;
    if (ns == 0 || ns > CME_MAX_SPECIES || nr == 0 || nr > CME_MAX_REACTIONS) return LMB_E_UNSUPPORTED;
    CmeModel h;
    memset(&h, 0, sizeof h);
    h.ns = ns;
    h.nr = nr;
    // Reactants from the dependency matrix, as CMESolver::buildModel reads
    // them (CMESolver.cpp:340-430): the first one or two species with D = 1.
    for (uint32_t r = 0; r < nr; r++) {
        uint32_t deps[3], nd = 0;
        for (uint32_t s = 0; s < ns; s++)
            if (D[(size_t)s * nr + r] == 1) {
                if (nd < 3) deps[nd] = s;
                nd++;
            }
        const uint32_t t = rtype[r];
        if (t == LMB_REACTION_ZEROTH) {
            if (nd != 0) return LMB_E_MODEL;
        } else if (t == LMB_REACTION_FIRST || t == LMB_REACTION_SECOND_SELF) {
            if (nd != 1) return LMB_E_MODEL;
            h.s1[r] = deps[0];
        } else if (t == LMB_REACTION_SECOND) {
            if (nd != 2) return LMB_E_MODEL;
            h.s1[r] = deps[0];
            h.s2[r] = deps[1];
        } else {
            return LMB_E_UNSUPPORTED;  // Hill / Michaelis-Menten types run on the CPU solvers only
        }
        h.type[r] = t;
        h.k[r] = (float)K[(size_t)r * k_cols];
    }
    // Stoichiometry and dependencies (CMESolver.cpp:440-560 builds the same
    // dependent-species / dependent-reaction tables).
    uint32_t nnz = 0;
    for (uint32_t r = 0; r < nr; r++) {
        h.off[r] = nnz;
        for (uint32_t s = 0; s < ns; s++) {
            const int32_t d = S[(size_t)s * nr + r];
            if (d != 0) {
                h.sp[nnz] = (uint8_t)s;
                h.d[nnz] = d;
                nnz++;
            }
        }
    }
    h.off[nr] = nnz;
    h.compact = ns <= 8 && nr <= 16;
    for (uint32_t r = 0; r < nr; r++) {
        h.code[r] = h.type[r] | (h.s1[r] << 2) | (h.s2[r] << 7);
        uint32_t packed = 0;
        for (uint32_t j = h.off[r]; j < h.off[r + 1]; j++) {
            if (h.d[j] < -8 || h.d[j] > 7) h.compact = 0;
            packed |= ((uint32_t)h.d[j] & 0xFu) << (4 * h.sp[j]);
        }
        h.delta4[r] = packed;
    }
    for (uint32_t r = 0; r < nr; r++) {
        unsigned long long dep = 0;
        for (uint32_t j = h.off[r]; j < h.off[r + 1]; j++) {
            const uint32_t s = h.sp[j];
            for (uint32_t q = 0; q < nr; q++) {
                const bool uses = (h.type[q] != LMB_REACTION_ZEROTH && h.s1[q] == s) ||
                                  (h.type[q] == LMB_REACTION_SECOND && h.s2[q] == s);
                if (uses) dep |= 1ull << q;
            }
        }
        h.dep[r] = dep;
    }

    lmb_cme *c = new (std::nothrow) lmb_cme;
    if (!c) return LMB_E_NOMEM;
    memset(c, 0, sizeof *c);
    c->ctx = ctx;
    c->ns = ns;
    c->nr = nr;
    c->reps = replicates;
    c->host = h;
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        delete c;
        return LMB_E_CUDA;
    }
    const size_t R = replicates;
    // One device block, sub-allocated at 256-byte boundaries.
    const size_t parts[] = {sizeof(CmeModel), R * ns * 4, R * 8, R * 8, R * 8, R * 4, R * 8, R * 4, R * ns * 4};
    size_t bytes = 0;
    for (size_t p : parts) bytes += (p + 255) & ~(size_t)255;
    char *blk = nullptr;
    if (cudaMalloc(&blk, bytes) != cudaSuccess) {
        delete c;
        return LMB_E_NOMEM;
    }
    c->state_block = blk;
    size_t o = 0;
    auto take = [&](size_t n) {
        char *p = blk + o;
        o += (n + 255) & ~(size_t)255;
        return p;
    };
    c->dev_model = (CmeModel *)take(sizeof(CmeModel));
    c->st.counts = (int32_t *)take(R * ns * 4);
    c->st.t = (double *)take(R * 8);
    c->st.t_next = (double *)take(R * 8);
    c->st.next_write = (double *)take(R * 8);
    c->st.next_entry = (uint32_t *)take(R * 4);
    c->st.events = (unsigned long long *)take(R * 8);
    c->st.done = (uint32_t *)take(R * 4);
    c->init_dev = (int32_t *)take(R * ns * 4);
    if (cudaMemcpyAsync(c->dev_model, &c->host, sizeof(CmeModel), cudaMemcpyHostToDevice, ctx->stream) !=
        cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaFree(blk);
        delete c;
        return LMB_E_CUDA;
    }
    ctx_retain(ctx);
    *out = c;
    return LMB_OK;
}

extern "C" int lmb_cme_destroy(lmb_cme *c)
{
    if (!c) return LMB_E_ARG;
    cudaSetDevice(c->ctx->device);
    cudaStreamSynchronize(c->ctx->stream);
    if (c->out) cudaFree(c->out);
    if (c->state_block) cudaFree(c->state_block);
    lmb_ctx *ctx = c->ctx;
    delete c;
    ctx_release(ctx);
    return LMB_OK;
}

extern "C" int lmb_cme_set_initial_counts(lmb_cme *c, const uint32_t *counts, int per_replicate)
{
    if (!c || !counts) return LMB_E_ARG;
    CKC(cudaSetDevice(c->ctx->device));
    const size_t n = per_replicate ? (size_t)c->reps * c->ns : c->ns;
    for (size_t i = 0; i < n; i++)
        if (counts[i] > 0x7FFFFFFFu) return LMB_E_ARG;
    CKC(cudaMemcpyAsync(c->init_dev, counts, n * 4, cudaMemcpyHostToDevice, c->ctx->stream));
    CKC(cudaStreamSynchronize(c->ctx->stream));
    c->init_per_replicate = per_replicate ? 1 : 0;
    c->begun = false;
    return LMB_OK;
}

template <int NS, int NR>
static cudaError_t launch_begin(lmb_cme *c)
{
    const uint32_t blocks = (c->reps + CME_THREADS - 1) / CME_THREADS;
    cme_begin_kernel<NS, NR><<<blocks, CME_THREADS, 0, c->ctx->stream>>>(c->dev_model, c->st, c->init_dev,
                                                                     c->init_per_replicate, c->reps, c->seed);
    count_launch();
    return cudaGetLastError();
}

template <int NS, int NR>
static cudaError_t launch_segment(lmb_cme *c, double seg_end)
{
    const uint32_t blocks = (c->reps + CME_THREADS - 1) / CME_THREADS;
    cme_segment_kernel<NS, NR><<<blocks, CME_THREADS, 0, c->ctx->stream>>>(
        c->dev_model, c->st, c->out, c->reps, c->entries, c->seed, seg_end, c->t_end, c->write_interval);
    count_launch();
    return cudaGetLastError();
}

template <int NS, int NR>
static cudaError_t launch_compact(lmb_cme *c, double seg_end)
{
    const uint32_t blocks = (c->reps + CME_THREADS - 1) / CME_THREADS;
    cme_compact_kernel<NS, NR><<<blocks, CME_THREADS, 0, c->ctx->stream>>>(
        c->dev_model, c->st, c->out, c->reps, c->entries, c->seed, seg_end, c->t_end, c->write_interval);
    count_launch();
    return cudaGetLastError();
}

// Register-resident variants: (species, reactions) up to (4, 8), (8, 16) and
// (32, 64).
static cudaError_t dispatch_begin(lmb_cme *c)
{
    if (c->ns <= 4 && c->nr <= 8) return launch_begin<4, 8>(c);
    if (c->ns <= 8 && c->nr <= 16) return launch_begin<8, 16>(c);
    return launch_begin<CME_MAX_SPECIES, CME_MAX_REACTIONS>(c);
}

static cudaError_t dispatch_segment(lmb_cme *c, double seg_end)
{
    if (c->host.compact && c->kernel == LMB_CME_KERNEL_AUTO) {
        if (c->ns <= 4 && c->nr <= 8) return launch_compact<4, 8>(c, seg_end);
        return launch_compact<8, 16>(c, seg_end);
    }
    if (c->ns <= 4 && c->nr <= 8) return launch_segment<4, 8>(c, seg_end);
    if (c->ns <= 8 && c->nr <= 16) return launch_segment<8, 16>(c, seg_end);
    return launch_segment<CME_MAX_SPECIES, CME_MAX_REACTIONS>(c, seg_end);
}

extern "C" int lmb_cme_set_kernel(lmb_cme *c, int kernel)
{
    if (!c || (kernel != LMB_CME_KERNEL_AUTO && kernel != LMB_CME_KERNEL_GENERIC)) return LMB_E_ARG;
    c->kernel = kernel;
    return LMB_OK;
}

extern "C" int lmb_cme_begin(lmb_cme *c, uint32_t seed, double t_end, double write_interval)
{
    if (!c || !(t_end > 0.0) || !(write_interval > 0.0)) return LMB_E_ARG;
    CKC(cudaSetDevice(c->ctx->device));
    const uint32_t entries = entries_for(t_end, write_interval);
    const size_t need = (size_t)entries * c->ns * c->reps;
    if (need > c->out_entries) {
        if (c->out) cudaFree(c->out);
        c->out = nullptr;
        c->out_entries = 0;
        CKC(cudaMalloc(&c->out, need * 4));
        c->out_entries = need;
    }
    c->entries = entries;
    c->t_end = t_end;
    c->write_interval = write_interval;
    c->seed = seed;
    c->t_done = 0.0;
    CKC(dispatch_begin(c));
    c->begun = true;
    return LMB_OK;
}

extern "C" int lmb_cme_advance_async(lmb_cme *c, double until)
{
    if (!c) return LMB_E_ARG;
    if (!c->begun) return LMB_E_STATE;
    CKC(cudaSetDevice(c->ctx->device));
    const double seg_end = until >= c->t_end ? c->t_end : until;
    CKC(dispatch_segment(c, seg_end));
    if (seg_end > c->t_done) c->t_done = seg_end;
    return LMB_OK;
}

extern "C" int lmb_cme_run(lmb_cme *c, uint32_t seed, double t_end, double write_interval)
{
    int rc = lmb_cme_begin(c, seed, t_end, write_interval);
    if (rc) return rc;
    rc = lmb_cme_advance_async(c, t_end);
    if (rc) return rc;
    CKC(cudaStreamSynchronize(c->ctx->stream));
    return LMB_OK;
}

extern "C" int lmb_cme_entries(const lmb_cme *c, uint32_t *entries)
{
    if (!c || !entries) return LMB_E_ARG;
    *entries = c->entries;
    return LMB_OK;
}

extern "C" int lmb_cme_get_counts(lmb_cme *c, uint32_t *counts)
{
    if (!c || !counts) return LMB_E_ARG;
    if (!c->begun) return LMB_E_STATE;
    CKC(cudaSetDevice(c->ctx->device));
    const size_t n = (size_t)c->entries * c->ns * c->reps;
    std::vector<int32_t> planar(n);
    CKC(cudaMemcpyAsync(planar.data(), c->out, n * 4, cudaMemcpyDeviceToHost, c->ctx->stream));
    CKC(cudaStreamSynchronize(c->ctx->stream));
    // [entry][species][replicate] -> [replicate][entry][species]
    for (uint32_t e = 0; e < c->entries; e++)
        for (uint32_t s = 0; s < c->ns; s++) {
            const int32_t *row = planar.data() + ((size_t)e * c->ns + s) * c->reps;
            for (uint32_t r = 0; r < c->reps; r++)
                counts[((size_t)r * c->entries + e) * c->ns + s] = (uint32_t)row[r];
        }
    return LMB_OK;
}

extern "C" int lmb_cme_device_counts(lmb_cme *c, void **counts)
{
    if (!c || !counts) return LMB_E_ARG;
    *counts = c->out;
    return LMB_OK;
}

extern "C" int lmb_cme_stats(lmb_cme *c, uint64_t *events, uint32_t *finished)
{
    if (!c) return LMB_E_ARG;
    CKC(cudaSetDevice(c->ctx->device));
    std::vector<unsigned long long> ev(c->reps);
    std::vector<uint32_t> done(c->reps);
    CKC(cudaMemcpyAsync(ev.data(), c->st.events, c->reps * 8, cudaMemcpyDeviceToHost, c->ctx->stream));
    CKC(cudaMemcpyAsync(done.data(), c->st.done, c->reps * 4, cudaMemcpyDeviceToHost, c->ctx->stream));
    CKC(cudaStreamSynchronize(c->ctx->stream));
    uint64_t tot = 0;
    uint32_t fin = 0;
    for (uint32_t r = 0; r < c->reps; r++) {
        tot += ev[r];
        fin += done[r];
    }
    if (events) *events = tot;
    if (finished) *finished = fin;
    return LMB_OK;
}
