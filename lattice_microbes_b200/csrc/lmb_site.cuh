// lmb_site.cuh -- the per-site MPD rules, shared by the per-phase kernels and
// the fused timestep kernel.
//
// sweep_site: new content of one site after a 1-D hop sweep, from its own
// slots and its two neighbours' slots along the sweep axis
// (byte_diffusion_1d_dev.cu:86-122 choices, :199-269 propagation).
// react_site: the precomputed-table reaction step of one site
// (MpdRdmeSolver.cu:1590-1675 with byte_reaction_dev.cu:121-258).
#pragma once

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_internal.h"

namespace lmb {

// Appends particles to a new site in order; the (S+1)-th and later ones
// overflow with seq = position - S, if `record` (only the owner of a site
// records; halo recomputations do not).
template <int BPS, int S>
struct SiteBuilder {
    SiteWords<BPS, S> out;
    int n;
    __device__ __forceinline__ void init()
    {
        out.clear();
        n = 0;
    }
    __device__ __forceinline__ void push(uint32_t p, bool record, RunState *rs, OverflowEntry *list, uint32_t cap,
                                         uint32_t phase, uint32_t site)
    {
        if (n < S) out.put(n, p);
        else if (record) push_overflow(rs, list, cap, phase, site, (uint32_t)(n - S), p);
        n++;
    }
};

// gi/gim/gip: lattice indices of the site and its minus / plus neighbours
// (they key the hash); t/tm/tp: their site types.
template <int BPS, int S>
__device__ __forceinline__ SiteWords<BPS, S> sweep_site(const SiteWords<BPS, S> &own, const SiteWords<BPS, S> &mn,
                                                        const SiteWords<BPS, S> &pl, uint32_t t, uint32_t tm,
                                                        uint32_t tp, uint32_t gi, uint32_t gim, uint32_t gip,
                                                        unsigned long long th, const DevTables &m, bool record,
                                                        uint32_t phase, RunState *rs, OverflowEntry *list,
                                                        uint32_t cap)
{
    SiteBuilder<BPS, S> b;
    b.init();
    constexpr int CB = CountBits<S>::value;
    // Stayers of this site, slot order.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = own.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)gi << CB) | (unsigned)k, th);
            const float qm = lookup_T(m, p, t, tm);
            const float qp = lookup_T(m, p, t, tp);
            const bool plus = (r >= 0.5f) && (r < __fadd_rn(qp, 0.5f));
            if (!plus && !(r < qm)) b.push(p, record, rs, list, cap, phase, gi);
        }
    }
    // PLUS movers of the minus neighbour.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = mn.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)gim << CB) | (unsigned)k, th);
            const float qp = lookup_T(m, p, tm, t);
            if ((r >= 0.5f) && (r < __fadd_rn(qp, 0.5f))) b.push(p, record, rs, list, cap, phase, gi);
        }
    }
    // MINUS movers of the plus neighbour.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = pl.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)gip << CB) | (unsigned)k, th);
            const float qm = lookup_T(m, p, tp, t);
            if (r < qm) b.push(p, record, rs, list, cap, phase, gi);
        }
    }
    return b.out;
}

// Per-reaction propensity from FP32 counts (byte_reaction_dev.cu:62-102,
// MPD_GLOBAL_R_MATRIX branch: the self reaction is rate*n*(n-1)).
template <int BPS, int S>
__device__ __forceinline__ float reaction_propensity(const DevTables &m, uint32_t t, const SiteWords<BPS, S> &s,
                                                     uint32_t rx)
{
    if (!tload(m.RL + (size_t)rx * m.nst + t)) return 0.0f;
    const uint32_t d1 = tload(m.D1 + rx), d2 = tload(m.D2 + rx);
    float n1 = 0.0f, n2 = 0.0f;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = s.slot(k);
        if (p > 0) {
            n1 = __fadd_rn(n1, p == d1 ? 1.0f : 0.0f);
            n2 = __fadd_rn(n2, p == d2 ? 1.0f : 0.0f);
        }
    }
    const float rate = tload(m.rate + rx);
    switch (tload(m.order + rx)) {
    case 1: return rate;
    case 2: return __fmul_rn(rate, n1);
    case 3: return __fmul_rn(__fmul_rn(rate, n1), n2);
    case 4: return __fmul_rn(__fmul_rn(rate, n1), __fsub_rn(n1, 1.0f));
    default: return 0.0f;
    }
}

constexpr int MAX_STOICH = 32;

// Table propensity sum in slot order, double precision probability, at most
// one reaction; returns true when the site changed (s updated in place).
template <int BPS, int S>
__device__ __forceinline__ bool react_site(SiteWords<BPS, S> &s, uint32_t t, uint32_t gi, unsigned long long th,
                                           const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap)
{
    float a = tload(m.qp0 + t);
    if (s.empty() && a == 0.0f) return false;
    const size_t o1 = (size_t)t * m.ns, o2 = (size_t)t * m.ns * m.ns;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p1 = s.slot(k);
        if (p1 > 0) {
            a = __fadd_rn(a, tload(m.qp1 + o1 + (p1 - 1)));
#pragma unroll
            for (int j = k + 1; j < S; j++) {
                const uint32_t p2 = s.slot(j);
                if (p2 > 0) a = __fadd_rn(a, tload(m.qp2 + o2 + (size_t)(p1 - 1) * m.ns + (p2 - 1)));
            }
        }
    }
    if (a == 0.0f) return false;
    const float prob = (float)(1.0 - exp(-(double)a));
    const float r0 = hash_float(((unsigned long long)gi << 1) | 0ull, th);
    if (!(prob > 0.0f && r0 <= prob)) return false;

    float rp = __fmul_rn(hash_float(((unsigned long long)gi << 1) | 1ull, th), a);
    uint32_t idx = 0;
    for (uint32_t rx = 0; rx < m.nr; rx++) {
        const float prop = reaction_propensity<BPS, S>(m, t, s, rx);
        if (prop > 0.0f) {
            if (rp > 0.0f) idx = rx;
            rp = __fsub_rn(rp, prop);
        }
    }
    atomicAdd(&rs->reactions, 1ull);

    // Stoichiometry of the chosen reaction, ascending species.
    const uint32_t e0 = tload(m.stoich_off + idx), e1 = tload(m.stoich_off + idx + 1);
    const int ne = (int)(e1 - e0) < MAX_STOICH ? (int)(e1 - e0) : MAX_STOICH;
    uint32_t sp[MAX_STOICH];
    int dlt[MAX_STOICH];
    for (int e = 0; e < ne; e++) {
        sp[e] = tload(m.stoich_sp + e0 + e);
        dlt[e] = tload(m.stoich_d + e0 + e);
    }
    // Survivors in slot order; a consumed reactant bumps its count.
    SiteWords<BPS, S> out;
    out.clear();
    int n = 0;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t q = s.slot(k);
        if (q > 0) {
            bool consumed = false;
            for (int e = 0; e < ne; e++) {
                if (sp[e] == q - 1) {
                    if (dlt[e] < 0) {
                        dlt[e]++;
                        consumed = true;
                    }
                    break;
                }
            }
            if (!consumed) out.put(n++, q);
        }
    }
    // Products by ascending species id; extra ones overflow.  A stoichiometry
    // left negative (reactant missing) adds nothing.
    uint32_t seq = 0;
    for (int e = 0; e < ne; e++) {
        for (int j = 0; j < dlt[e]; j++) {
            const uint32_t p = sp[e] + 1;
            if (n < S) out.put(n++, p);
            else push_overflow(rs, list, cap, 4u, gi, seq++, p);
        }
    }
    s = out;
    return true;
}

}  // namespace lmb
