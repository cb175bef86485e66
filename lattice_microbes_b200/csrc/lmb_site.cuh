// lmb_site.cuh -- the per-site MPD rules, shared by the per-phase kernels and
// the fused timestep kernel.
//
// site_choices / assemble_site: one 1-D hop sweep, as the reference splits it
// into choices (byte_diffusion_1d_dev.cu:86-122) and propagation (:199-269):
// each particle's choice is drawn once, then every output site assembles its
// new content from its own and its two neighbours' choices.
// sweep_site: one sweep of one site, drawing its neighbours' choices too.
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

// A site's hop choices for one sweep, one bit per slot and direction: bit k
// of the low half set when the particle in slot k moves to the minus
// neighbour, bit S + k when it moves to the plus neighbour; neither bit for a
// stayer or an empty slot.  32 bits cover up to 16 slots, 64 bits 32 slots.
template <int S>
struct ChoiceCode {
    using type = uint32_t;
};
template <>
struct ChoiceCode<32> {
    using type = unsigned long long;
};

// Bit k set when slot k holds a particle (slots may have holes in a lattice
// given by the caller, so every slot is looked at, as the reference does).
template <int BPS, int S>
__device__ __forceinline__ uint32_t occupied_slots(const SiteWords<BPS, S> &s)
{
    uint32_t m = 0;
    if (BPS == 1) {
#pragma unroll
        for (int k = 0; k < SiteWords<BPS, S>::W; k++) {
            const uint32_t w = s.w[k];
            // High bit of each byte set when the byte is nonzero, then the
            // four bits gathered into bits 28..31 by one multiply.
            const uint32_t hi = (w | ((w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu)) & 0x80808080u;
            m |= (((hi >> 7) * 0x10204080u) >> 28) << (4 * k);
        }
    } else {
#pragma unroll
        for (int k = 0; k < S; k++) m |= (s.w[k] != 0u ? 1u : 0u) << k;
    }
    return m;
}

// The particle in slot k for a slot index known only at run time (no
// dynamic register indexing: the word is selected, then the byte).
template <int BPS, int S>
__device__ __forceinline__ uint32_t slot_at(const SiteWords<BPS, S> &s, uint32_t k)
{
    constexpr int W = SiteWords<BPS, S>::W;
    if (BPS == 1) {
        uint32_t w = s.w[0];
#pragma unroll
        for (int j = 1; j < W; j++)
            if ((k >> 2) == (uint32_t)j) w = s.w[j];
        return (w >> (8 * (k & 3u))) & 0xFFu;
    }
    uint32_t v = s.w[0];
#pragma unroll
    for (int j = 1; j < W; j++)
        if (k == (uint32_t)j) v = s.w[j];
    return v;
}

// Choices of every particle of a site of type t whose minus / plus
// neighbours have types tm / tp, keyed by the site's lattice index gi
// (byte_diffusion_1d_dev.cu:86-122, word_diffusion_1d_dev.cu:83-112): draw
// r; PLUS when 0.5 <= r < q(t->tp) + 0.5, else MINUS when r < q(t->tm),
// else STAY.  One hash per particle per sweep.
template <int BPS, int S>
__device__ __forceinline__ typename ChoiceCode<S>::type site_choices(const SiteWords<BPS, S> &s, uint32_t t,
                                                                     uint32_t tm, uint32_t tp, uint32_t gi,
                                                                     unsigned long long th, const DevTables &m)
{
    using Code = typename ChoiceCode<S>::type;
    constexpr int CB = CountBits<S>::value;
    Code c = 0;
    uint32_t occ = occupied_slots<BPS, S>(s);
    while (occ) {
        const uint32_t k = __ffs(occ) - 1;
        occ &= occ - 1;
        const uint32_t p = slot_at<BPS, S>(s, k);
        const float r = hash_float(((unsigned long long)gi << CB) | k, th);
        const float qp = lookup_T(m, p, t, tp);
        if ((r >= 0.5f) && (r < __fadd_rn(qp, 0.5f))) {
            c |= (Code)1 << (S + k);
        } else {
            const float qm = lookup_T(m, p, t, tm);
            if (r < qm) c |= (Code)1 << k;
        }
    }
    return c;
}

// Byte compaction: the bytes of word w whose bits are set in the 4-bit mask
// m, moved to the low end in order (one byte permute; the selector of mask m
// is entry m of a 16-entry table of 16-bit selectors, kept in four 64-bit
// constants).
__device__ __forceinline__ uint32_t compact_bytes(uint32_t w, uint32_t m)
{
    const unsigned long long q = m < 8u ? (m < 4u ? 0x4410444144404444ull : 0x4210442144204442ull)
                                        : (m < 12u ? 0x4310443144304443ull : 0x3210432143204432ull);
    return __byte_perm(w, 0u, (uint32_t)(q >> (16u * (m & 3u))) & 0xFFFFu);
}

// A site's bytes selected by an S-bit slot mask, packed from the low end of
// a 128-bit value (lo, hi); n = number of bytes.  S <= 16.
template <int S>
__device__ __forceinline__ void compact_site(const uint32_t *w, uint32_t mask, unsigned long long &lo,
                                             unsigned long long &hi, uint32_t &n)
{
    lo = 0;
    hi = 0;
    n = 0;
    // Words past the mask's highest bit contribute nothing (a packed site's
    // particles sit in its first words).
    const uint32_t top = 32u - __clz(mask);
#pragma unroll
    for (int k = 0; k < S / 4; k++) {
        if (4u * k >= top) break;
        const uint32_t m = (mask >> (4 * k)) & 0xFu;
        const unsigned long long c = compact_bytes(w[k], m);
        // Append the (up to 4) bytes at byte offset n (< 16).
        const uint32_t sh = 8u * n;
        if (sh < 64u) {
            lo |= c << sh;
            if (sh > 32u) hi |= c >> (64u - sh);
        } else {
            hi |= c << (sh - 64u);
        }
        n += __popc(m);
    }
}

// (lo, hi) |= (a_lo, a_hi) << (8 * nb), for nb < 16 and bits beyond 128 dropped.
__device__ __forceinline__ void or_shifted(unsigned long long &lo, unsigned long long &hi, unsigned long long a_lo,
                                           unsigned long long a_hi, uint32_t nb)
{
    const uint32_t sh = 8u * nb;
    if (sh == 0u) {
        lo |= a_lo;
        hi |= a_hi;
    } else if (sh < 64u) {
        lo |= a_lo << sh;
        hi |= (a_hi << sh) | (a_lo >> (64u - sh));
    } else {
        hi |= a_lo << (sh - 64u);
    }
}

// New content of a site after a sweep (byte_diffusion_1d_dev.cu:199-269):
// its stayers in slot order, then the PLUS movers of the minus neighbour,
// then the MINUS movers of the plus neighbour, each in slot order; the
// (S+1)-th and later particles overflow (queued with seq = position - S when
// `record`: only the owner of a site records, halo recomputations do not).
template <int BPS, int S>
__device__ __forceinline__ SiteWords<BPS, S> assemble_site(const SiteWords<BPS, S> &own,
                                                           typename ChoiceCode<S>::type c_own,
                                                           const SiteWords<BPS, S> &mn,
                                                           typename ChoiceCode<S>::type c_mn,
                                                           const SiteWords<BPS, S> &pl,
                                                           typename ChoiceCode<S>::type c_pl, uint32_t gi,
                                                           bool record, uint32_t phase, RunState *rs,
                                                           OverflowEntry *list, uint32_t cap)
{
    constexpr uint32_t LOW = S >= 32 ? 0xFFFFFFFFu : ((1u << S) - 1u);
    if (BPS == 1 && S <= 16) {
        // Byte lattices: three byte compactions and two shifts, no loop,
        // unless the site overflows (then the ordered loop below queues the
        // extra particles).
        const uint32_t stay = occupied_slots<BPS, S>(own) & ~((uint32_t)c_own | (uint32_t)(c_own >> S)) & LOW;
        const uint32_t in_m = (uint32_t)(c_mn >> S) & LOW, in_p = (uint32_t)c_pl & LOW;
        const uint32_t total = __popc(stay) + __popc(in_m) + __popc(in_p);
        if (total <= (uint32_t)S) {
            unsigned long long lo, hi, blo, bhi, clo, chi;
            uint32_t na, nb, nc;
            compact_site<S>(own.w, stay, lo, hi, na);
            compact_site<S>(mn.w, in_m, blo, bhi, nb);
            compact_site<S>(pl.w, in_p, clo, chi, nc);
            or_shifted(lo, hi, blo, bhi, na);
            or_shifted(lo, hi, clo, chi, na + nb);
            SiteWords<BPS, S> out;
#pragma unroll
            for (int k = 0; k < SiteWords<BPS, S>::W; k++)
                out.w[k] = (uint32_t)((k < 2 ? lo : hi) >> (32 * (k & 1)));
            return out;
        }
    }
    SiteBuilder<BPS, S> b;
    b.init();
    uint32_t stay = occupied_slots<BPS, S>(own) & ~((uint32_t)c_own | (uint32_t)(c_own >> S)) & LOW;
    while (stay) {
        const uint32_t k = __ffs(stay) - 1;
        stay &= stay - 1;
        b.push(slot_at<BPS, S>(own, k), record, rs, list, cap, phase, gi);
    }
    uint32_t in_m = (uint32_t)(c_mn >> S) & LOW;
    while (in_m) {
        const uint32_t k = __ffs(in_m) - 1;
        in_m &= in_m - 1;
        b.push(slot_at<BPS, S>(mn, k), record, rs, list, cap, phase, gi);
    }
    uint32_t in_p = (uint32_t)c_pl & LOW;
    while (in_p) {
        const uint32_t k = __ffs(in_p) - 1;
        in_p &= in_p - 1;
        b.push(slot_at<BPS, S>(pl, k), record, rs, list, cap, phase, gi);
    }
    return b.out;
}

// sweep_site: the same sweep for one output site in one call, drawing the
// choices of its own and its two neighbours' particles itself (three hashes
// per particle over the sweep, no exchange between threads).  The fused
// kernel uses it: at the low occupancy it serves, exchanging choices through
// shared memory costs more (a pass, a barrier and shared memory) than the
// extra hashes.
// gi/gim/gip: lattice indices of the site and its minus / plus neighbours
// (they key the hash); t/tm/tp: their site types.
// Transition-table access for sweep_site, two forms giving the same values:
// TTable keeps the table's base and sizes in registers and reads through a
// site's rows; TableSet reads through the table set for every lookup (fewer
// live registers).
struct TTable {
    const float *T;
    uint32_t ns, nst;
    __device__ __forceinline__ TRow row(uint32_t src, uint32_t dst) const { return TRow(T, ns, nst, src, dst); }
};

struct TableSetRow {
    const DevTables *m;
    uint32_t src, dst;
    __device__ __forceinline__ float operator()(uint32_t p) const { return lookup_T(*m, p, src, dst); }
};

struct TableSet {
    const DevTables *m;
    __device__ __forceinline__ TableSetRow row(uint32_t src, uint32_t dst) const { return TableSetRow{m, src, dst}; }
};

template <int BPS, int S, class Tables>
__device__ __forceinline__ SiteWords<BPS, S> sweep_site(const SiteWords<BPS, S> &own, const SiteWords<BPS, S> &mn,
                                                        const SiteWords<BPS, S> &pl, uint32_t t, uint32_t tm,
                                                        uint32_t tp, uint32_t gi, uint32_t gim, uint32_t gip,
                                                        unsigned long long th, const Tables &tabs, bool record,
                                                        uint32_t phase, RunState *rs, OverflowEntry *list,
                                                        uint32_t cap)
{
    SiteBuilder<BPS, S> b;
    b.init();
    constexpr int CB = CountBits<S>::value;
    // The four rows of T the site's particles use.
    const auto own_m = tabs.row(t, tm), own_p = tabs.row(t, tp), mn_p = tabs.row(tm, t), pl_m = tabs.row(tp, t);
    // Stayers of this site, slot order.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = own.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)gi << CB) | (unsigned)k, th);
            const float qm = own_m(p);
            const float qp = own_p(p);
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
            const float qp = mn_p(p);
            if ((r >= 0.5f) && (r < __fadd_rn(qp, 0.5f))) b.push(p, record, rs, list, cap, phase, gi);
        }
    }
    // MINUS movers of the plus neighbour.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = pl.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)gip << CB) | (unsigned)k, th);
            const float qm = pl_m(p);
            if (r < qm) b.push(p, record, rs, list, cap, phase, gi);
        }
    }
    return b.out;
}

// Per-reaction propensity from FP32 counts (byte_reaction_dev.cu:62-102,
// MPD_GLOBAL_R_MATRIX branch: the self reaction is rate*n*(n-1)).
// hi: slots at and above it are empty (an unrolled loop stops there).
// The same from a reaction's table entries (D1, D2, order, rate), for a
// reaction allowed on the site's type.
template <int BPS, int S>
__device__ __forceinline__ float propensity_of(const SiteWords<BPS, S> &s, int hi, uint32_t d1, uint32_t d2,
                                               uint32_t order, float rate)
{
    float n1 = 0.0f, n2 = 0.0f;
#pragma unroll
    for (int k = 0; k < S; k++) {
        if (k >= hi) break;
        const uint32_t p = s.slot(k);
        if (p > 0) {
            n1 = __fadd_rn(n1, p == d1 ? 1.0f : 0.0f);
            n2 = __fadd_rn(n2, p == d2 ? 1.0f : 0.0f);
        }
    }
    switch (order) {
    case 1: return rate;
    case 2: return __fmul_rn(rate, n1);
    case 3: return __fmul_rn(__fmul_rn(rate, n1), n2);
    case 4: return __fmul_rn(__fmul_rn(rate, n1), __fsub_rn(n1, 1.0f));
    default: return 0.0f;
    }
}

template <int BPS, int S>
__device__ __forceinline__ float reaction_propensity(const DevTables &m, uint32_t t, const SiteWords<BPS, S> &s,
                                                     uint32_t rx, int hi)
{
    if (!tload(m.RL + (size_t)rx * m.nst + t)) return 0.0f;
    return propensity_of<BPS, S>(s, hi, tload(m.D1 + rx), tload(m.D2 + rx), tload(m.order + rx), tload(m.rate + rx));
}

// The first two exits of react_site, for a site of type t holding n
// particles whose zeroth-order propensity is a0 and whose reaction draw is
// r0: false when the reaction step cannot change the site.  The reaction
// probability never exceeds the total propensity a (see the bound before
// the double exp in react_site), and a itself -- a float sum of qp0, one qp1
// entry per particle and one qp2 entry per pair, at most 137 terms -- never
// exceeds U = qp0 + n max(qp1) + n(n-1)/2 max(qp2) by more than its rounding,
// (1 + 2^-24)^136 < 1.0001.  So a draw above U * 1.0001 * (1 + 2^-20) + 2^-60
// cannot react.  The z sweep evaluates the same function on the site it has
// just assembled, so the sites it leaves out are exactly those react_site
// would leave unchanged.
// The per-type inputs of the bound: qp0, max qp1 and max qp2 of type t (a
// kernel may load them ahead of the site's count).
struct ReactBound {
    float a0, q1, q2;
};

__device__ __forceinline__ ReactBound react_bound(uint32_t t, const DevTables &m)
{
    return ReactBound{tload(m.qp0 + t), tload(m.qpmax + t), tload(m.qpmax + m.nst + t)};
}

__device__ __forceinline__ bool reaction_may_fire(uint32_t n, const ReactBound &b, float r0)
{
    if (n == 0 && b.a0 == 0.0f) return false;
    const float nf = (float)n;
    const float pairs = __fmul_rn(nf, __fmul_rn(__fsub_rn(nf, 1.0f), 0.5f));
    float u = __fadd_ru(b.a0, __fmul_ru(nf, b.q1));
    u = __fadd_ru(u, __fmul_ru(pairs, b.q2));
    u = __fmul_ru(u, 1.0001f);
    return !(r0 > __fadd_ru(__fmul_ru(u, 1.00000095367431640625f), 8.67361738e-19f));
}

__device__ __forceinline__ bool reaction_may_fire(uint32_t n, float a0, uint32_t t, float r0, const DevTables &m)
{
    if (n == 0 && a0 == 0.0f) return false;
    return reaction_may_fire(n, ReactBound{a0, tload(m.qpmax + t), tload(m.qpmax + m.nst + t)}, r0);
}

// Table propensity sum in slot order, double precision probability, at most
// one reaction; returns true when the site changed (s updated in place).
// CAP > 0: the reaction's candidates are sorted in a list of CAP registers
// (nothing in local memory; for kernels whose registers are scarce and whose
// models have few candidates per site); CAP == 0: in a 64-entry array.
template <int BPS, int S, int CAP>
__device__ __forceinline__ bool react_site(SiteWords<BPS, S> &s, uint32_t t, uint32_t gi, unsigned long long th,
                                           const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap)
{
    float a = tload(m.qp0 + t);
    if (s.empty() && a == 0.0f) return false;
    // The table sums and the double exp are evaluated only for draws below
    // the bound of reaction_may_fire.
    const float r0 = hash_float(((unsigned long long)gi << 1) | 0ull, th);
    const uint32_t occ = occupied_slots<BPS, S>(s);
    if (!reaction_may_fire((uint32_t)__popc(occ), a, t, r0, m)) return false;
    // Every slot loop below stops at the highest occupied slot: the slots
    // above it add nothing (sites are packed after a sweep, so this is the
    // particle count, which keeps the unrolled loops short).
    const int hi = 32 - __clz((int)occ);
    const size_t o1 = (size_t)t * m.ns, o2 = (size_t)t * m.ns * m.ns;
#pragma unroll
    for (int k = 0; k < S; k++) {
        if (k >= hi) break;
        const uint32_t p1 = s.slot(k);
        if (p1 > 0) {
            a = __fadd_rn(a, tload(m.qp1 + o1 + (p1 - 1)));
#pragma unroll
            for (int j = k + 1; j < S; j++) {
                if (j >= hi) break;
                const uint32_t p2 = s.slot(j);
                if (p2 > 0) a = __fadd_rn(a, tload(m.qp2 + o2 + (size_t)(p1 - 1) * m.ns + (p2 - 1)));
            }
        }
    }
    if (a == 0.0f) return false;
    // prob = (float)(1 - exp(-a)) below never exceeds a: mathematically
    // 1 - e^-a < a for a > 0, the double evaluation adds at most a few units
    // of 2^-53, and rounding to float at most one float ulp of a.  A draw
    // above a * (1 + 2^-20) + 2^-60 therefore cannot react, and the double
    // exp is evaluated only for draws below that bound.
    if (r0 > __fadd_ru(__fmul_ru(a, 1.00000095367431640625f), 8.67361738e-19f)) return false;
    const float prob = (float)(1.0 - exp(-(double)a));
    if (!(prob > 0.0f && r0 <= prob)) return false;

    float rp = __fmul_rn(hash_float(((unsigned long long)gi << 1) | 1ull, th), a);
    uint32_t idx = 0;
    // determineReactionIndex (byte_reaction_dev.cu:146-176) visits every
    // reaction in index order; a reaction whose propensity is 0 changes
    // nothing, and only the zeroth-order reactions and those whose first
    // reactant is in the site can have a nonzero one.  Those candidates are
    // gathered from the reaction lists of the zeroth-order reactions and of
    // each species held, sorted, repeats dropped (a species held twice gives
    // its reactions once), and visited in index order; when there are more
    // than the list holds, every reaction is visited instead.
    auto visit = [&](uint32_t rx) {
        const float prop = reaction_propensity<BPS, S>(m, t, s, rx, hi);
        if (prop > 0.0f) {
            if (rp > 0.0f) idx = rx;
            rp = __fsub_rn(rp, prop);
        }
    };
    constexpr int LEN = CAP > 0 ? CAP : 64;
    // CAP == 0, models of up to BMW * 32 reactions: the candidates are the
    // set bits of a bitmap indexed by reaction, which keeps them sorted and
    // drops repeats whatever their number (a full site of one species, say).
    constexpr uint32_t BMW = CAP > 0 ? 1 : 128;
    const bool bitmap = CAP == 0 && m.nr <= BMW * 32;
    // Only its first nbw words are used, each cleared below before any bit
    // is set (the compiler cannot see that the two conditions agree).
#pragma nv_diag_suppress 549
    uint32_t bm[BMW];
    uint32_t cand[LEN];
    int nc = 0;
    bool all = false;
    // CAP > 0: insertion by compare-and-swap over fixed positions (unused
    // ones hold ~0u, above every index, so carrying the larger value forward
    // keeps the list sorted); CAP == 0 without the bitmap: appended, sorted
    // below.
    auto insert = [&](uint32_t v) {
        if (CAP > 0) {
            bool dup = false;
#pragma unroll
            for (int j = 0; j < LEN; j++) dup |= cand[j] == v;
            if (dup) return;
            if (nc == LEN) {
                all = true;
                return;
            }
            uint32_t carry = v;
#pragma unroll
            for (int j = 0; j < LEN; j++) {
                const uint32_t c = cand[j];
                const bool sw = c > carry;
                cand[j] = sw ? carry : c;
                carry = sw ? c : carry;
            }
            nc++;
        } else if (bitmap) {
            bm[v >> 5] |= 1u << (v & 31u);
        } else {
            if (nc < LEN) cand[nc++] = v;
            else all = true;
        }
    };
    if (CAP > 0) {
#pragma unroll
        for (int j = 0; j < LEN; j++) cand[j] = 0xFFFFFFFFu;
    }
    const uint32_t nbw = (m.nr + 31u) / 32u;
    if (bitmap)
        for (uint32_t w = 0; w < nbw; w++) bm[w] = 0u;
    {
        const uint32_t z0 = tload(m.rx_off), z1 = tload(m.rx_off + 1);
        for (uint32_t e = z0; e < z1 && !all; e++) insert(tload(m.rx_list + e));
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (k >= hi) break;
            const uint32_t p = s.slot(k);
            if (p > 0 && p <= m.ns && !all) {
                const uint32_t e0 = tload(m.rx_off + p), e1 = tload(m.rx_off + p + 1);
                for (uint32_t e = e0; e < e1 && !all; e++) insert(tload(m.rx_list + e));
            }
        }
    }
    if (all) {
        for (uint32_t rx = 0; rx < m.nr; rx++) visit(rx);
    } else if (CAP > 0) {
        // Smallest off the front, the rest shifted down.
        for (int q = 0; q < nc; q++) {
            const uint32_t rx = cand[0];
#pragma unroll
            for (int j = 0; j + 1 < LEN; j++) cand[j] = cand[j + 1];
            visit(rx);
        }
    } else if (bitmap) {
        // Candidates in ascending order, RXB at a time: every table entry of
        // the batch is loaded before any propensity is formed (one round trip
        // per batch instead of two per candidate), then the batch is visited
        // in order with the same arithmetic as visit().
        constexpr int RXB = 4;
        uint32_t rxs[RXB];
        int nb = 0;
        auto flush = [&]() {
            uint32_t rl[RXB], d1[RXB], d2[RXB], ord[RXB];
            float rate[RXB];
#pragma unroll
            for (int j = 0; j < RXB; j++) {
                const uint32_t rx = j < nb ? rxs[j] : rxs[0];
                rl[j] = tload(m.RL + (size_t)rx * m.nst + t);
                d1[j] = tload(m.D1 + rx);
                d2[j] = tload(m.D2 + rx);
                ord[j] = tload(m.order + rx);
                rate[j] = tload(m.rate + rx);
            }
#pragma unroll
            for (int j = 0; j < RXB; j++) {
                if (j >= nb) break;
                const float prop = rl[j] ? propensity_of<BPS, S>(s, hi, d1[j], d2[j], ord[j], rate[j]) : 0.0f;
                if (prop > 0.0f) {
                    if (rp > 0.0f) idx = rxs[j];
                    rp = __fsub_rn(rp, prop);
                }
            }
            nb = 0;
        };
        for (uint32_t w = 0; w < nbw; w++) {
            uint32_t bits = bm[w];
            while (bits) {
                const uint32_t k = __ffs(bits) - 1;
                bits &= bits - 1;
                rxs[nb++] = w * 32u + k;
                if (nb == RXB) flush();
            }
        }
        if (nb > 0) flush();
    } else {
        // Insertion sort of the few entries; repeats skipped.
        for (int a = 1; a < nc; a++) {
            const uint32_t v = cand[a];
            int b = a - 1;
            while (b >= 0 && cand[b] > v) {
                cand[b + 1] = cand[b];
                b--;
            }
            cand[b + 1] = v;
        }
        for (int q = 0; q < nc; q++) {
            if (q > 0 && cand[q] == cand[q - 1]) continue;
            visit(cand[q]);
        }
    }
#pragma nv_diag_default 549
    atomicAdd(&rs->reactions, 1ull);

    // evaluateReaction (byte_reaction_dev.cu:179-258) with the chosen
    // reaction's sparse stoichiometry (ascending species): reactants are
    // taken out in slot order, products appended by ascending species id.
    // The consumed species are held in two registers (a reaction of order
    // two or less consumes at most two); a stoichiometry with more negative
    // entries goes through a per-entry count.
    const uint32_t e0 = tload(m.stoich_off + idx), e1 = tload(m.stoich_off + idx + 1);
    uint32_t c_sp0 = 0xFFFFFFFFu, c_sp1 = 0xFFFFFFFFu;
    int c_n0 = 0, c_n1 = 0, negatives = 0;
    for (uint32_t e = e0; e < e1; e++) {
        const int d = tload(m.stoich_d + e);
        if (d < 0) {
            if (negatives == 0) {
                c_sp0 = tload(m.stoich_sp + e);
                c_n0 = -d;
            } else if (negatives == 1) {
                c_sp1 = tload(m.stoich_sp + e);
                c_n1 = -d;
            }
            negatives++;
        }
    }
    SiteWords<BPS, S> out;
    out.clear();
    int n = 0;
    if (negatives <= 2) {
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (k >= hi) break;
            const uint32_t q = s.slot(k);
            if (q > 0) {
                if (q - 1 == c_sp0 && c_n0 > 0) c_n0--;
                else if (q - 1 == c_sp1 && c_n1 > 0) c_n1--;
                else out.put(n++, q);
            }
        }
    } else {
        // Any number of consumed species: the entry of each particle's
        // species is looked up and its remaining count kept in a bit of
        // `used` per consumed particle (S <= 32 slots, so at most S taken).
        uint32_t taken_bits = 0;  // bit k: slot k consumed
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (k >= hi) break;
            const uint32_t q = s.slot(k);
            if (q > 0) {
                int need = 0;
                for (uint32_t e = e0; e < e1; e++)
                    if (tload(m.stoich_sp + e) == q - 1) {
                        need = -tload(m.stoich_d + e);
                        break;
                    }
                // Consumed when fewer of this species than it needs were
                // taken in the slots before.
                int before = 0;
#pragma unroll
                for (int j = 0; j < k; j++)
                    if (((taken_bits >> j) & 1u) && s.slot(j) == q) before++;
                if (need > before) taken_bits |= 1u << k;
                else out.put(n++, q);
            }
        }
    }
    // Products by ascending species id; extra ones overflow.  A stoichiometry
    // left negative (reactant missing) adds nothing.
    uint32_t seq = 0;
    for (uint32_t e = e0; e < e1; e++) {
        const int d = tload(m.stoich_d + e);
        const uint32_t p = tload(m.stoich_sp + e) + 1;
        for (int j = 0; j < d; j++) {
            if (n < S) out.put(n++, p);
            else push_overflow(rs, list, cap, 4u, gi, seq++, p);
        }
    }
    s = out;
    return true;
}

}  // namespace lmb
