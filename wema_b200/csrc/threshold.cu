// threshold.cu - the reference's adaptive threshold, bit for bit.
//
// The reference computes thr = (sum|x| / N) * 0.2 over the 6-slot flat
// coefficient array (wema.c:719-723, phase_amp.c:25-29; the batch route uses
// (0.2 / N) * sum, wema_batch.c:272-276).  Its -Ofast build vectorises the
// sum as eight sequential FP32 lane sums (lane j = elements 8t + j), reduced
// ((l0+l4)+(l2+l6)) + ((l1+l5)+(l3+l7)), plus a 4-wide/scalar epilogue for the
// last N mod 8 elements.  A mask bit |x| > thr flips if thr is off by one ulp,
// so the lane sums must be reproduced exactly - each is a chain of N/8
// dependent FP32 adds (518k at 1080p).
//
// Parallel exact method.  While the running sum s stays in one binade
// [2^e, 2^(e+1)), s = m * u with u = 2^(e-23) and m a 24-bit integer, and
// fl(s + a) = u * rne(m + a/u): the increment is round(a/u) unless a/u is an
// exact half, where it rounds to the even result, i.e. depends on m's parity.
// So a run of elements acts on m as  m -> m + d[m & 1]  - a two-entry
// "parity monoid" {d0, d1}, composable in any grouping:
//   (A then B)[p] = A[p] + B[(p + A[p]) & 1].
// A lane is cut into sub-chunks of G = 256 lane-elements.  Kernels:
//   thr_partials, thr_prefix - FP64 lane sums per sub-chunk and their prefix
//                   (first call only: no binade history yet);
//   thr_monoids   - per (sub-chunk, lane) monoids of one or two candidate
//                   binades: the binade the previous frame's walk recorded at
//                   the sub-chunk start (a video's coefficient statistics move
//                   slowly) and a neighbour near a recorded binade change
//                   (first call: from the FP64 prefix); also FP32 sub-chunk
//                   sums for the walk's own prediction;
//   thr_walk      - one CTA per (lane, channel).  An FP64 prefix of the
//                   sub-chunk sums predicts the binade at each sub-chunk start
//                   and picks that candidate's monoid.  All warps compose the
//                   monoids of each run of equal predicted binade (a
//                   "segment") into prefix and suffix compositions in shared
//                   memory and copy in the elements of the sub-chunks where a
//                   binade change is predicted; then one warp walks: a segment
//                   whose end stays below 2^24 is accepted in one step, a
//                   crossing is located from the prefix compositions and its
//                   sub-chunk is summed with plain sequential FP32 adds from
//                   the exact value before it.  Anything unpredicted (another
//                   binade, a crossing elsewhere) takes a window scan over the
//                   stored monoids or the sequential adds.  The lane that
//                   finishes last reduces the eight lane sums and divides.
// Predictions only decide speed, never the result.
#include <string.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

namespace wema {

constexpr int LANES = 8;
constexpr int THR_THREADS = 256;
constexpr int G = 256;             // lane-elements per sub-chunk
constexpr int EPT = G / 32;        // lane-elements per thread in the per-sub-chunk kernels
constexpr int SAT = 1 << 25;       // saturated increment: certainly leaves the binade
constexpr int PAGE = 2048;         // sub-chunks of one lane staged in shared memory at a time
constexpr int NPRE = 32;           // predicted-crossing sub-chunks staged per page
constexpr int SPT = 4;             // sub-chunks per thread in a slow-path window
constexpr int WIN = 32 * SPT;
constexpr unsigned FULL = 0xffffffffu;

struct Mono { int d0, d1; };

__device__ __forceinline__ Mono mono_id() { return {0, 0}; }

__device__ __forceinline__ Mono compose(Mono a, Mono b) {   // a first, then b
    Mono r;
    r.d0 = min(a.d0 + ((a.d0 & 1) ? b.d1 : b.d0), SAT);
    r.d1 = min(a.d1 + (((a.d1 + 1) & 1) ? b.d1 : b.d0), SAT);
    return r;
}

__device__ __forceinline__ int apply(int m, Mono d) { return m + ((m & 1) ? d.d1 : d.d0); }
__device__ __forceinline__ int apply(int m, int2 d) { return m + ((m & 1) ? d.y : d.x); }

// effect of adding |x| (bits ua, sign cleared) to any s of biased exponent eb
__device__ __forceinline__ Mono elem_mono(uint32_t ua, int eb) {
    const int ea_raw = (int)(ua >> 23);
    const int ea = max(ea_raw, 1);
    const uint32_t ma = (ua & 0x7FFFFFu) | (ea_raw ? 0x800000u : 0u);
    const int sh = eb - ea;
    const int shc = min(max(sh, 1), 31);
    const int q = (int)(ma >> shc);
    const uint32_t r2 = ma << (32 - shc);          // remainder bits, aligned to the top
    const int up = r2 > 0x80000000u;
    const int tie = r2 == 0x80000000u;
    const int qo = q & 1;
    Mono m;
    m.d0 = q + (up | (tie & qo));
    m.d1 = q + (up | (tie & (qo ^ 1)));
    if (sh <= 0) m = {SAT, SAT};
    return m;
}

__device__ __forceinline__ float from_m(int m, int eb) {
    return __uint_as_float(((uint32_t)eb << 23) | ((uint32_t)m & 0x7FFFFFu));
}

// Sequential reader of the 6-slot flat array (slots 3-5 mirror 2-0).
// cur_seek() places it on the (level, slot) segment holding index i;
// cur_addr() advances segment by segment, so a run of nearby indices costs one
// division.  levels == 0 views coef as a plain flat array of off6[0] elements.
struct Cursor {
    const float* base;           // element at seg0
    long long seg0, seg1;        // current segment [seg0, seg1)
    int l, slot;
};

__device__ __forceinline__ void cur_set(const PyrView& v, Cursor& c) {
    const int band = c.slot < 3 ? c.slot : 5 - c.slot;
    c.seg0 = v.off6[c.l] + c.slot * v.n[c.l];
    c.seg1 = c.seg0 + v.n[c.l];
    c.base = v.coef + v.uoff[c.l] + band * v.n[c.l];
}

__device__ __forceinline__ void cur_seek(const PyrView& v, Cursor& c, long long i) {
    if (v.levels == 0) {
        c.base = v.coef;
        c.seg0 = 0;
        c.seg1 = 0x7fffffffffffffffLL;
        return;
    }
    int l = 0;
#pragma unroll
    for (int k = 1; k < 4; k++)
        if (k < v.levels && i >= v.off6[k]) l = k;
    c.l = l;
    const long long r = i - v.off6[l];
    c.slot = (r < 0x7fffffffLL && v.n[l] < 0x7fffffffLL) ? (int)((int)r / (int)v.n[l])
                                                           : (int)(r / v.n[l]);
    if (c.slot > 5) c.slot = 5;
    cur_set(v, c);
}

__device__ __forceinline__ const float* cur_addr(const PyrView& v, Cursor& c, long long i) {
    while (i >= c.seg1) {
        if (++c.slot == 6) { c.slot = 0; c.l++; }
        cur_set(v, c);
    }
    return c.base + (i - c.seg0);
}

// Addresses of the EPT lane-elements t0 .. t0+EPT-1 of lane j (null past the
// lane's end).  A run almost always lies inside one (level, slot) segment:
// then it is one seek and fixed offsets.
__device__ __forceinline__ void run_addrs(const PyrView& v, long long nlane, long long t0, int j,
                                          const float* (&addr)[EPT]) {
    if (t0 >= nlane) {
#pragma unroll
        for (int k = 0; k < EPT; k++) addr[k] = nullptr;
        return;
    }
    Cursor cu;
    const long long i0 = 8 * t0 + j;
    cur_seek(v, cu, i0);
    if (t0 + EPT <= nlane && i0 + 8 * (EPT - 1) < cu.seg1) {
        const float* p = cu.base + (i0 - cu.seg0);
#pragma unroll
        for (int k = 0; k < EPT; k++) addr[k] = p + 8 * k;
        return;
    }
#pragma unroll
    for (int k = 0; k < EPT; k++) addr[k] = (t0 + k < nlane) ? cur_addr(v, cu, i0 + 8 * k) : nullptr;
}

// |x| bits of the EPT lane-elements t0 .. t0+EPT-1 of lane j (0 past the
// lane's end): all addresses first, then all loads, so they are in flight together
__device__ __forceinline__ void load_run(const PyrView& v, long long nlane, long long t0, int j,
                                         uint32_t (&out)[EPT]) {
    const float* addr[EPT];
    run_addrs(v, nlane, t0, j, addr);
#pragma unroll
    for (int k = 0; k < EPT; k++) out[k] = addr[k] ? (__float_as_uint(__ldg(addr[k])) & 0x7FFFFFFFu) : 0u;
}

__device__ __forceinline__ uint32_t v6_bits(const PyrView& v, long long i) {
    Cursor c;
    cur_seek(v, c, i);
    return __float_as_uint(*cur_addr(v, c, i)) & 0x7FFFFFFFu;
}

struct ThrGeom {
    long long n6, main, nlane;   // main = elements summed by the 8 lanes
    int nsub;                    // sub-chunks per lane
};

__host__ __device__ inline ThrGeom thr_geom(long long n6) {
    ThrGeom g;
    g.n6 = n6;
    g.main = (n6 - 1 <= 6) ? 0 : (n6 & ~7LL);
    g.nlane = g.main / LANES;
    g.nsub = (int)((g.nlane + G - 1) / G);
    return g;
}

// entries of each lane-major array: at least T16_MAXBLK (the FP16-plane
// threshold's per-block partial sums use `part`)
constexpr int T16_MAXBLK = 1024;
static size_t thr_per(const ThrGeom& g) { return std::max<size_t>((size_t)g.nsub * LANES, T16_MAXBLK); }

size_t thr_scratch_bytes(long long n6) {
    const ThrGeom g = thr_geom(n6);
    const size_t per = thr_per(g);
    return per * (2 * sizeof(double) + sizeof(int4) + sizeof(int2) + sizeof(int)) + 256;
}

void thr_scratch_bind(ThrScratch& s, void* base, long long n6) {
    const ThrGeom g = thr_geom(n6);
    const size_t per = thr_per(g);
    char* p = (char*)base;
    s.part = (double*)p;    p += per * sizeof(double);
    s.prefix = (double*)p;  p += per * sizeof(double);
    s.candp = (int4*)p;     p += per * sizeof(int4);
    s.candq = (int2*)p;     p += per * sizeof(int2);
    s.hist = (int*)p;       p += per * sizeof(int);   // per is a multiple of 8: stays 32-aligned
    s.lanes = (float*)p;    p += LANES * sizeof(float);
    s.counter = (unsigned*)p;
}

struct ThrArgs {
    PyrView v[3];
    ThrScratch s[3];
    float* thr;
    float* sums;
    int batch_form;
    int use_hist;
    int sub0;                   // monoids: first sub-chunk of this launch (a split launch)
};

// ---- FP64 partial sums: thread (lane j, block tb) covers EPT lane-elements
__device__ __forceinline__ void thr_partials_body(const ThrArgs& a, int bx, int by) {
    const int ch = by;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const int sub = bx;
    if (sub >= g.nsub) return;
    const int j = threadIdx.x & 7, tb = threadIdx.x >> 3;
    const long long t0 = (long long)sub * G + (long long)tb * EPT;
    uint32_t val[EPT];
    load_run(v, g.nlane, t0, j, val);
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < EPT; k++) acc += (double)__uint_as_float(val[k]);
    acc += __shfl_xor_sync(FULL, acc, 8);
    acc += __shfl_xor_sync(FULL, acc, 16);
    __shared__ double ws[8][8];
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln < 8) ws[warp][ln] = acc;
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s += ws[w][threadIdx.x];
        a.s[ch].part[(long long)threadIdx.x * g.nsub + sub] = s;
    }
}

// ---- exclusive FP64 prefix per lane: one CTA per (lane, channel)
__device__ __forceinline__ void thr_prefix_body(const ThrArgs& a, int bx, int by) {
    const int j = bx, ch = by;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const double* part = a.s[ch].part + (long long)j * g.nsub;
    double* pre = a.s[ch].prefix + (long long)j * g.nsub;
    __shared__ double wsum[THR_THREADS / 32];
    __shared__ double carry_s;
    double carry = 0.0;
    const int ln = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < g.nsub; base += THR_THREADS * 8) {
        double x[8];
        double local = 0.0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int c = base + threadIdx.x * 8 + k;
            x[k] = c < g.nsub ? part[c] : 0.0;
            local += x[k];
        }
        double incl = local;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_up_sync(FULL, incl, d);
            if (ln >= d) incl += o;
        }
        if (ln == 31) wsum[warp] = incl;
        __syncthreads();
        double wpre = 0.0;
        for (int w = 0; w < warp; w++) wpre += wsum[w];
        double run = carry + wpre + incl - local;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int c = base + threadIdx.x * 8 + k;
            if (c < g.nsub) pre[c] = run;
            run += x[k];
        }
        if (threadIdx.x == THR_THREADS - 1) carry_s = run;
        __syncthreads();
        carry = carry_s;
        __syncthreads();
    }
}

// ---- monoids of the candidate binades of each (sub-chunk, lane)
//   primary   = binade of s at the sub-chunk start in the previous frame (or
//               of the FP64 prefix without history);
//   secondary = the binade one above when a binade change was recorded within
//               max(2, sub/16) sub-chunks after (the change may come earlier),
//               else one below when one was recorded as far before (it may
//               come later); without history the neighbour nearer the prefix.
// One warp per sub-chunk (2048 flat elements).  Without an exact half the
// increments do not depend on parity, a monoid is a plain integer sum and the
// order of summation is free: thread ln reads float4s 32k + ln (coalesced),
// which always hold lanes 4(ln & 1) .. 4(ln & 1) + 3, and the sums meet by
// shuffles.  A warp that meets an exact half takes lane_monoids.
// Sub-chunks per CTA.  A warp that meets an exact half takes the much slower
// lane_monoids; small CTAs free their slot as soon as their own warps finish
// instead of holding it for the slowest of eight.
constexpr int MON_WARPS = 2;
// CTAs per SM asked of the register allocator: 10 x 2 warps at 96 registers
// (8 would allow 128 registers but only 16 warps per SM for a latency-bound kernel)
constexpr int MON_MINB = 10;

__device__ __forceinline__ void sub_candidates(const ThrArgs& a, const ThrScratch& sc,
                                               const ThrGeom& g, long long row, int sub,
                                               int& ep, int& eq) {
    if (a.use_hist) {
        const int* h = sc.hist + row;
        ep = h[sub];
        const int D = max(2, sub >> 4);
        const int hi = h[min(sub + D, g.nsub - 1)], lo = h[max(sub - D, 0)];
        eq = hi > ep ? ep + 1 : (lo < ep && lo > 0 ? ep - 1 : 0);
    } else {
        const float f = (float)sc.prefix[row + sub];
        const uint32_t fb = __float_as_uint(f);
        ep = (int)(fb >> 23);
        const bool low_half = (fb & 0x7FFFFFu) < 0x400000u;
        eq = low_half ? ep - 1 : ep + 1;
    }
    if (ep <= 0 || ep >= 255) ep = 0;
    if (ep == 0 || eq <= 0 || eq >= 255) eq = 0;
}

// The increment of |x| in binade eb as a float: q = |x| * 2^(150-eb) is exact,
// and (q + 2^23) - 2^23 rounds it to the nearest integer, ties to even, for
// q < 2^23; an element with q >= 2^23 leaves the binade from any m, and its
// float is then large enough to say so.  Sums of these integers are exact
// below 2^24; anything larger means the binade is left anyway.  |q - r| ==
// 0.5 marks an exact half, where the increment depends on m's parity.
// scale_of is 0 when eb is too small to scale within the float range; such a
// candidate is dropped.
__device__ __forceinline__ float scale_of(int eb) {
    return (eb >= 24 && eb <= 254) ? __uint_as_float((uint32_t)(277 - eb) << 23) : 0.0f;
}
constexpr float RND = 8388608.0f;   // 2^23

// Monoids of this thread's four lanes (4 * (ln & 1) + i) over a sub-chunk
// that contains exact halves (or elements of 2^23 increments and more).  The
// elements are reloaded through the first-level cache in the warp's float4
// layout: thread ln holds lane-elements 16k + (ln >> 1), k < 16.  An exact half
// rounds m + n + 1/2 to the even neighbour, so m is even after it: only a
// lane's first half depends on the start parity p, and each half adds n plus
// (parity of m before it) xor (n & 1), where that parity counts the odd
// increments since the start (p included) or since the previous half.
// Ballots in lane-element order give those counts.
__device__ __forceinline__ void lane_monoids(const PyrView& v, long long main, long long i0,
                                             const float* p, bool vec, bool one, int ln,
                                             const float (&scale)[4], Mono (&out)[4]) {
    const int half = ln & 1;
    const unsigned hmask = half ? 0xAAAAAAAAu : 0x55555555u;
#pragma unroll 1
    for (int i = 0; i < 4; i++) {
        const float sci = i == 0 ? scale[0] : i == 1 ? scale[1] : i == 2 ? scale[2] : scale[3];
        float S = 0.0f;
        int cp = 0, first = 1, c1 = 0, cfix = 0;
        Cursor cl;
        if (!vec && !one && i0 < main) cur_seek(v, cl, i0);
#pragma unroll 2
        for (int k = 0; k < 2 * G / 32; k++) {
            float x;
            if (vec) {
                const float4 x4 = __ldg(reinterpret_cast<const float4*>(p) + 32 * k + ln);
                x = i == 0 ? x4.x : i == 1 ? x4.y : i == 2 ? x4.z : x4.w;
            } else {
                const long long e = 4 * (32 * k + ln) + i;
                x = one ? __ldg(p + e) : (i0 + e < main ? *cur_addr(v, cl, i0 + e) : 0.0f);
            }
            const float q = fabsf(x) * sci;
            const float r = __fsub_rn(__fadd_rn(q, RND), RND);
            const bool tie = fabsf(q - r) == 0.5f;
            const float n = tie ? __fsub_rn(q, 0.5f) : r;
            S += n;
            const int nbit = tie ? ((int)n & 1) : 0;
            const int pbit = tie ? 0 : ((int)fminf(r, 16777216.0f) & 1);
            const unsigned tm0 = __ballot_sync(FULL, tie) & hmask;
            const unsigned pm = __ballot_sync(FULL, pbit) & hmask;
            const unsigned nm = __ballot_sync(FULL, nbit) & hmask;
            unsigned tm = tm0, done = 0u;
            while (tm) {
                const unsigned b = tm & (0u - tm);
                cp ^= __popc(pm & (b - 1u) & ~done) & 1;
                const int nb = (nm & b) != 0;
                if (first) { c1 = cp ^ nb; first = 0; }
                else cfix += cp ^ nb;
                cp = 0;
                done = (b << 1) - 1u;
                tm &= tm - 1u;
            }
            cp ^= __popc(pm & ~done) & 1;
        }
#pragma unroll
        for (int d = 2; d < 32; d <<= 1) S += __shfl_xor_sync(FULL, S, d);
        const int base = (int)fminf(S, (float)SAT) + cfix;
        const Mono m = {min(base + (first ? 0 : c1), SAT), min(base + (first ? 0 : (1 ^ c1)), SAT)};
        if (i == 0) out[0] = m;
        else if (i == 1) out[1] = m;
        else if (i == 2) out[2] = m;
        else out[3] = m;
    }
}

// The 64 elements of thread ln in the warp's float4 layout when the
// sub-chunk straddles a (level, slot) segment or is not 16-byte aligned.  Out
// of line (and reading the view from shared memory) so that the common path
// stays small in the instruction cache.
__device__ __noinline__ void load_generic(const PyrView* sv, long long main, long long i0,
                                          const float* p, bool one, int ln, float* out) {
    Cursor cu;
    if (!one && i0 < main) cur_seek(*sv, cu, i0);
    for (int k = 0; k < 2 * G / 32; k++)
        for (int i = 0; i < 4; i++) {
            const long long e = 4 * (32 * k + ln) + i;
            out[4 * k + i] = one ? __ldg(p + e) : (i0 + e < main ? *cur_addr(*sv, cu, i0 + e) : 0.0f);
        }
}

__device__ __forceinline__ void thr_monoids_body(const ThrArgs& a, int bx, int by) {
    const int ch = by;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const ThrScratch& sc = a.s[ch];
    __shared__ PyrView sv;
    if (threadIdx.x == 0) {
        sv = v;
        if (bx == 0 && a.sub0 == 0) *sc.counter = 0u;   // the walk's lane counter
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const int sub = a.sub0 + bx * MON_WARPS + warp;
    if (sub >= g.nsub) return;   // whole warps only; no block barrier follows
    const int half = ln & 1;     // this thread's lanes: 4 * half + i
    const long long i0 = (long long)sub * (8 * G);
    Cursor cu;
    const bool any = i0 < g.main;
    if (any) cur_seek(v, cu, i0);
    const float* p = any ? cu.base + (i0 - cu.seg0) : nullptr;
    const bool one = any && i0 + 8 * G <= g.main && i0 + 8 * G - 1 < cu.seg1;
    const bool vec = one && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    // all sixteen float4s in flight before anything else
    float xv[2 * G / 32][4];
    if (vec) {
#pragma unroll
        for (int k = 0; k < 2 * G / 32; k++) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(p) + 32 * k + ln);
            xv[k][0] = x.x; xv[k][1] = x.y; xv[k][2] = x.z; xv[k][3] = x.w;
        }
    } else {
        float tmp[8 * G / 32];
        load_generic(&sv, g.main, i0, p, one, ln, tmp);
#pragma unroll
        for (int k = 0; k < 2 * G / 32; k++)
#pragma unroll
            for (int i = 0; i < 4; i++) xv[k][i] = tmp[4 * k + i];
    }
    int ep, eq;                  // candidates of lane ln & 7
    sub_candidates(a, sc, g, (long long)(ln & 7) * g.nsub, sub, ep, eq);
    int EP[4], EQ[4];
    float sc4[4], sq4[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        EP[i] = __shfl_sync(FULL, ep, 4 * half + i);
        EQ[i] = __shfl_sync(FULL, eq, 4 * half + i);
        sc4[i] = scale_of(EP[i]);
        sq4[i] = scale_of(EQ[i]);
    }
    float sp[4], sq[4], ps[4];
    float dmax = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; i++) { sp[i] = 0.0f; sq[i] = 0.0f; ps[i] = 0.0f; }
#pragma unroll
    for (int k = 0; k < 2 * G / 32; k++) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float a = fabsf(xv[k][i]);
            const float q = a * sc4[i];
            const float r = __fsub_rn(__fadd_rn(q, RND), RND);
            sp[i] += r;
            dmax = fmaxf(dmax, fabsf(q - r));
            ps[i] += a;
        }
    }
    const bool has_q = __any_sync(FULL, (EQ[0] | EQ[1] | EQ[2] | EQ[3]) != 0);
    if (has_q) {   // secondary candidates
#pragma unroll
        for (int k = 0; k < 2 * G / 32; k++) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float q = fabsf(xv[k][i]) * sq4[i];
                const float r = __fsub_rn(__fadd_rn(q, RND), RND);
                sq[i] += r;
                dmax = fmaxf(dmax, fabsf(q - r));
            }
        }
    }
    // |q - r| reaches 0.5 only at an exact half or at q >= 2^23
    Mono mp4[4], mq4[4];
    if (__any_sync(FULL, dmax >= 0.5f)) {
        lane_monoids(v, g.main, i0, p, vec, one, ln, sc4, mp4);
        if (has_q) {
            lane_monoids(v, g.main, i0, p, vec, one, ln, sq4, mq4);
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) mq4[i] = mono_id();
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int d = 2; d < 32; d <<= 1) {
                sp[i] += __shfl_xor_sync(FULL, sp[i], d);
                sq[i] += __shfl_xor_sync(FULL, sq[i], d);
            }
            const int a0 = (int)fminf(sp[i], (float)SAT), a1 = (int)fminf(sq[i], (float)SAT);
            mp4[i] = {a0, a0};
            mq4[i] = {a1, a1};
        }
    }
    int EPw[4];   // candidate actually written (0 when it cannot be scaled)
#pragma unroll
    for (int i = 0; i < 4; i++) {
#pragma unroll
        for (int d = 2; d < 32; d <<= 1) ps[i] += __shfl_xor_sync(FULL, ps[i], d);
        EPw[i] = (EP[i] > 0 && sc4[i] == 0.0f) ? 0 : EP[i];
    }
    // thread L < 8 takes lane L from thread L >> 2, entry L & 3
    const int src = (ln >> 2) & 1, ent = ln & 3;
    Mono MP = mono_id(), MQ = mono_id();
    float rs = 0.0f;
    int epw = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int a0 = __shfl_sync(FULL, mp4[i].d0, src), a1 = __shfl_sync(FULL, mp4[i].d1, src);
        const int b0 = __shfl_sync(FULL, mq4[i].d0, src), b1 = __shfl_sync(FULL, mq4[i].d1, src);
        const float a2 = __shfl_sync(FULL, ps[i], src);
        const int e2 = __shfl_sync(FULL, EPw[i], src);
        if (ent == i) {
            MP = {a0, a1};
            MQ = {b0, b1};
            rs = a2;
            epw = e2;
        }
    }
    if (ln < 8) {   // lane ln: its own ep / eq
        ep = epw;
        if (ep == 0 || scale_of(eq) == 0.0f) eq = 0;
        const long long row = (long long)ln * g.nsub;
        sc.part[row + sub] = (double)rs;
        sc.candp[row + sub] = make_int4(ep, MP.d0, MP.d1, eq);
        sc.candq[row + sub] = make_int2(MQ.d0, MQ.d1);
    }
}

// ---- the walk
// Page arrays are padded so that a thread's eight consecutive entries fall in
// distinct banks across the warp: one int per 32 entries (sw), one int2 per
// 16 (sw2), one int4 per 8 (sw4).
__device__ __forceinline__ int sw(int c) { return c + (c >> 5); }
__device__ __forceinline__ int sw2(int c) { return c + (c >> 4); }
__device__ __forceinline__ int sw4(int c) { return c + (c >> 3); }
constexpr int LOGN = 256;          // accepted runs remembered for the history write-back

struct WalkSmem {
    int eb[PAGE + PAGE / 32];      // primary binade of each sub-chunk of the page (-1: none)
    int4 rec[PAGE + PAGE / 8];     // {binade, segment end | head << 30, suffix composition}
    int2 S[PAGE + PAGE / 16];      // composition from the segment start to c
    float pre[NPRE][G];            // elements of the predicted-crossing sub-chunks
    float wbuf[G];                 // elements of an unpredicted resolve
    int4 log[LOGN];                // {first, last, binade} of each accepted run
    int pre_sub[NPRE];
    int npre, nlog;
    int wf[8], we[8], wc[8];
    int2 wa[8];
    double wd[8];
};

struct Agg { int f; Mono m; int e; };   // segmented-scan element: head flag, composition, end

__device__ __forceinline__ Agg shfl_up_agg(Agg x, int d) {
    Agg o;
    o.f = __shfl_up_sync(FULL, x.f, d);
    o.m.d0 = __shfl_up_sync(FULL, x.m.d0, d);
    o.m.d1 = __shfl_up_sync(FULL, x.m.d1, d);
    o.e = __shfl_up_sync(FULL, x.e, d);
    return o;
}
__device__ __forceinline__ Agg shfl_down_agg(Agg x, int d) {
    Agg o;
    o.f = __shfl_down_sync(FULL, x.f, d);
    o.m.d0 = __shfl_down_sync(FULL, x.m.d0, d);
    o.m.d1 = __shfl_down_sync(FULL, x.m.d1, d);
    o.e = __shfl_down_sync(FULL, x.e, d);
    return o;
}
// a (earlier in c) then b, segments restart at heads
__device__ __forceinline__ Agg comb_fwd(const Agg& a, const Agg& b) {
    if (b.f) return b;
    return {a.f, compose(a.m, b.m), b.e};
}
// suffix direction: b (earlier in c) then a (later); b's own segment end wins
__device__ __forceinline__ Agg comb_rev(const Agg& a, const Agg& b) {
    if (b.f) return b;
    return {a.f, compose(b.m, a.m), a.e};
}

// sum of |x| over one sub-chunk's G lane-elements from s with sequential FP32 adds
__device__ __forceinline__ float serial_sum(const float* src, float s) {
    const float4* q = reinterpret_cast<const float4*>(src);
#pragma unroll 16
    for (int k = 0; k < G / 4; k++) {
        const float4 x = q[k];
        s = __fadd_rn(s, fabsf(x.x));
        s = __fadd_rn(s, fabsf(x.y));
        s = __fadd_rn(s, fabsf(x.z));
        s = __fadd_rn(s, fabsf(x.w));
    }
    return s;
}

// Addresses of lane-elements e = 32k + ln (k < EPT) of sub-chunk `sub` of lane
// j (null past the lane's end).  Interleaved so that a warp's load touches
// 1 KB (8 lines) rather than 8 KB.
__device__ __forceinline__ void sub_addrs(const PyrView& v, const ThrGeom& g, int j, long long sub,
                                          int ln, const float* (&addr)[EPT]) {
    const long long t0 = sub * G;
    const long long i0 = 8 * t0 + j;
    Cursor cu;
    cur_seek(v, cu, i0);
    if (t0 + G <= g.nlane && i0 + 8LL * (G - 1) < cu.seg1) {
        const float* p = cu.base + (i0 - cu.seg0) + 8 * ln;
#pragma unroll
        for (int k = 0; k < EPT; k++) addr[k] = p + 256 * k;
        return;
    }
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        const long long t = t0 + 32 * k + ln;
        addr[k] = nullptr;
        if (t < g.nlane) {
            Cursor c2;
            cur_seek(v, c2, 8 * t + j);
            addr[k] = cur_addr(v, c2, 8 * t + j);
        }
    }
}

// the G elements of a sub-chunk into shared memory (signs kept)
__device__ __forceinline__ void stage_sub(const PyrView& v, const ThrGeom& g, int j, long long sub,
                                          int ln, float* dst) {
    const float* addr[EPT];
    sub_addrs(v, g, j, sub, ln, addr);
    float x[EPT];
#pragma unroll
    for (int k = 0; k < EPT; k++) x[k] = addr[k] ? __ldg(addr[k]) : 0.0f;
#pragma unroll
    for (int k = 0; k < EPT; k++) dst[32 * k + ln] = x[k];
}

// the same with cp.async (completes at the next cp.async.wait_all)
__device__ __forceinline__ void stage_sub_async(const PyrView& v, const ThrGeom& g, int j,
                                                long long sub, int ln, float* dst) {
    const float* addr[EPT];
    sub_addrs(v, g, j, sub, ln, addr);
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        float* d = dst + 32 * k + ln;
        if (addr[k]) {
            const unsigned sa = (unsigned)__cvta_generic_to_shared(d);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(addr[k]) : "memory");
        } else {
            *d = 0.0f;
        }
    }
}

__device__ __forceinline__ bool cand_mono(const int4& P, const int2& Q, int eb, Mono& m) {
    if (eb <= 0) return false;
    if (P.x == eb) { m = {P.y, P.z}; return true; }
    if (P.w == eb) { m = {Q.x, Q.y}; return true; }
    return false;
}

__device__ __forceinline__ Mono warp_scan(Mono t, int ln) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        Mono o;
        o.d0 = __shfl_up_sync(FULL, t.d0, d);
        o.d1 = __shfl_up_sync(FULL, t.d1, d);
        if (ln >= d) t = compose(o, t);
    }
    return t;
}

__device__ __forceinline__ void thr_walk_body(const ThrArgs& a, int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WalkSmem& sm = *reinterpret_cast<WalkSmem*>(smem_raw);
    const int j = bx, ch = by;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const ThrScratch& sc = a.s[ch];
    const long long row = (long long)j * g.nsub;
    int* hist = sc.hist + row;
    const int tid = threadIdx.x, ln = tid & 31, warp = tid >> 5;
    float s = 0.0f;        // the running lane sum (warp 0)
    double pcarry = 0.0;   // FP64 sum of the earlier pages' sub-chunks

    for (int p0 = 0; p0 < g.nsub; p0 += PAGE) {
        const int np = min(PAGE, g.nsub - p0);
        // ---- FP64 prefix of the lane's sub-chunk sums -> predicted binade of
        // s at each sub-chunk start; the primary monoid is the stored candidate
        // of that binade (none: eb -1, never accepted, so the walk resolves it)
        double pv[8];
        int4 q4[8];
        int2 r2[8];
        double loc = 0.0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int c = tid * 8 + i;
            pv[i] = c < np ? sc.part[row + p0 + c] : 0.0;
            q4[i] = c < np ? sc.candp[row + p0 + c] : make_int4(-2, 0, 0, 0);
            r2[i] = c < np ? sc.candq[row + p0 + c] : make_int2(0, 0);
            loc += pv[i];
        }
        double incl_d = loc;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_up_sync(FULL, incl_d, d);
            if (ln >= d) incl_d += o;
        }
        if (ln == 31) sm.wd[warp] = incl_d;
        __syncthreads();
        double run_d = pcarry + incl_d - loc;
        double page_tot = 0.0;
        for (int w = 0; w < 8; w++) {
            if (w < warp) run_d += sm.wd[w];
            page_tot += sm.wd[w];
        }
        pcarry += page_tot;
        Mono P[8];
        int e8[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int c = tid * 8 + i;
            const int pred = (int)(__float_as_uint((float)run_d) >> 23);
            run_d += pv[i];
            P[i] = mono_id();
            e8[i] = -1;
            if (c >= np) continue;
            if (q4[i].x == pred) {
                e8[i] = pred;
                P[i] = {q4[i].y, q4[i].z};
            } else if (q4[i].w == pred && pred > 0) {
                e8[i] = pred;
                P[i] = {r2[i].x, r2[i].y};
            }
            sm.eb[sw(c)] = e8[i];
        }
        __syncthreads();
        unsigned head = 0, tail = 0;   // bit i: sub-chunk tid*8+i starts / ends a segment
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int c = tid * 8 + i;
            if (c < np) {
                if (c == 0 || sm.eb[sw(c - 1)] != e8[i]) head |= 1u << i;
                if (c == np - 1 || sm.eb[sw(c + 1)] != e8[i]) tail |= 1u << i;
            }
        }
        // ---- list the predicted crossings (segment ends but the lane's last
        // sub-chunk; sub-chunk 0 always) and start copying the first NPRE of
        // them into shared memory while the compositions are built
        {
            unsigned flag = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int c = tid * 8 + i;
                const bool f = ((tail >> i & 1) && p0 + c != g.nsub - 1) || (p0 + c == 0 && np > 0);
                if (f && c < np) flag |= 1u << i;
            }
            const int cnt = __popc(flag);
            int incl = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(FULL, incl, d);
                if (ln >= d) incl += o;
            }
            if (ln == 31) sm.wc[warp] = incl;
            __syncthreads();
            int pos = incl - cnt, total = 0;
            for (int w = 0; w < 8; w++) {
                if (w < warp) pos += sm.wc[w];
                total += sm.wc[w];
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                if (flag >> i & 1) {
                    if (pos < NPRE) sm.pre_sub[pos] = tid * 8 + i;
                    pos++;
                }
            }
            if (tid == 0) sm.npre = min(total, NPRE);
            __syncthreads();
            for (int k = warp; k < sm.npre; k += 8)
                stage_sub_async(v, g, j, (long long)p0 + sm.pre_sub[k], ln, sm.pre[k]);
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        // ---- forward segmented scan -> S
        {
            Agg t{0, mono_id(), 0};
#pragma unroll
            for (int i = 0; i < 8; i++) {
                if (head >> i & 1) { t.f = 1; t.m = P[i]; }
                else t.m = compose(t.m, P[i]);
            }
            Agg x = t;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const Agg o = shfl_up_agg(x, d);
                if (ln >= d) x = comb_fwd(o, x);
            }
            Agg ex = shfl_up_agg(x, 1);
            if (ln == 0) ex = {0, mono_id(), 0};
            if (ln == 31) { sm.wf[warp] = x.f; sm.wa[warp] = make_int2(x.m.d0, x.m.d1); }
            __syncthreads();
            Agg carry{0, mono_id(), 0};
            for (int w = 0; w < warp; w++)
                carry = comb_fwd(carry, Agg{sm.wf[w], {sm.wa[w].x, sm.wa[w].y}, 0});
            Mono run = comb_fwd(carry, ex).m;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int c = tid * 8 + i;
                run = (head >> i & 1) ? P[i] : compose(run, P[i]);
                if (c < np) sm.S[sw2(c)] = make_int2(run.d0, run.d1);
            }
            __syncthreads();
        }
        // ---- reverse segmented scan -> suffix compositions and segment ends
        {
            Agg t{0, mono_id(), -1};
#pragma unroll
            for (int i = 7; i >= 0; i--) {
                if (tail >> i & 1) { t.f = 1; t.m = P[i]; t.e = tid * 8 + i; }
                else t.m = compose(P[i], t.m);
            }
            Agg x = t;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const Agg o = shfl_down_agg(x, d);
                if (ln + d < 32) x = comb_rev(o, x);
            }
            Agg ex = shfl_down_agg(x, 1);
            if (ln == 31) ex = {0, mono_id(), -1};
            if (ln == 0) {
                sm.wf[warp] = x.f;
                sm.wa[warp] = make_int2(x.m.d0, x.m.d1);
                sm.we[warp] = x.e;
            }
            __syncthreads();
            Agg carry{0, mono_id(), -1};
            for (int w = 7; w > warp; w--)
                carry = comb_rev(carry, Agg{sm.wf[w], {sm.wa[w].x, sm.wa[w].y}, sm.we[w]});
            const Agg in = comb_rev(carry, ex);
            Mono run = in.m;
            int re = in.e;
#pragma unroll
            for (int i = 7; i >= 0; i--) {
                const int c = tid * 8 + i;
                if (tail >> i & 1) { run = P[i]; re = c; }
                else run = compose(P[i], run);
                if (c < np)
                    sm.rec[sw4(c)] = make_int4(e8[i], re | (int)((head >> i & 1) << 30), run.d0, run.d1);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();

        // ---- walk (warp 0)
        if (warp == 0) {
            const int npre = sm.npre;
            int kp = 0, nlog = 0;
            auto note = [&](int c0, int c1, int eb) {   // page sub-chunks c0..c1 start in eb
                if (nlog < LOGN) {
                    if (ln == 0) sm.log[nlog] = make_int4(c0, c1, eb, 0);
                    nlog++;
                } else {
                    for (int i = c0 + ln; i <= c1; i += 32) hist[p0 + i] = eb;
                }
            };
            auto resolve = [&](int r, float x) -> float {
                while (kp < npre && sm.pre_sub[kp] < r) kp++;
                const float* src;
                if (kp < npre && sm.pre_sub[kp] == r) {
                    src = sm.pre[kp];
                } else {
                    stage_sub(v, g, j, (long long)p0 + r, ln, sm.wbuf);
                    __syncwarp();
                    src = sm.wbuf;
                }
                x = serial_sum(src, x);
                __syncwarp();
                return x;
            };
            auto getS = [&](int c) { return sm.S[sw2(c)]; };
            int c = 0;
            while (c < np) {
                const uint32_t sb = __float_as_uint(s);
                const int eb = (int)(sb >> 23);
                if (eb == 0) {   // zero or subnormal running sum: sequential adds
                    note(c, c, 0);
                    s = resolve(c, s);
                    c++;
                    continue;
                }
                const int m = (int)(sb & 0x7FFFFFu) | 0x800000;
                const int4 R = sm.rec[sw4(c)];
                const int e = max(R.y & 0x3FFFFFFF, c);
                if (eb == R.x) {
                    const int mend = apply(m, make_int2(R.z, R.w));
                    if (mend < (1 << 24)) {   // the rest of the segment stays in this binade
                        note(c, e, eb);
                        s = from_m(mend, eb);
                        c = e + 1;
                        continue;
                    }
                    if (R.y >> 30) {   // segment start: S is the prefix from c
                        int r = e;
                        int2 Sr = e > c ? getS(e - 1) : make_int2(0, 0);
                        if (e > c && apply(m, Sr) >= (1 << 24)) {
                            r = e - 1;
                            for (int b = c; b < e; b += 32) {
                                const int i = b + ln;
                                const bool hit = i < e && apply(m, getS(i)) >= (1 << 24);
                                const unsigned bal = __ballot_sync(FULL, hit);
                                if (bal) { r = b + __ffs(bal) - 1; break; }
                            }
                            Sr = r > c ? getS(r - 1) : make_int2(0, 0);
                        }
                        const int ms = r > c ? apply(m, Sr) : m;
                        note(c, r, eb);
                        s = resolve(r, from_m(ms, eb));
                        c = r + 1;
                        continue;
                    }
                }
                // ---- slow path: window scan over the stored candidates of
                // c .. min(c + WIN, segment end + 1), first failure resolved
                const int wend = min(np, min(c + WIN, e + 1));
                const int4* cp = sc.candp + row + p0;
                const int2* cq = sc.candq + row + p0;
                Mono mine[SPT];
                bool ok[SPT];
                Mono t = mono_id();
                bool broken = false;
#pragma unroll
                for (int q = 0; q < SPT; q++) {
                    const int r = c + ln * SPT + q;
                    ok[q] = false;
                    mine[q] = mono_id();
                    if (r < wend && !broken) {
                        Mono mq;
                        if (cand_mono(cp[r], cq[r], eb, mq)) {
                            ok[q] = true;
                            mine[q] = mq;
                            t = compose(t, mq);
                        } else {
                            broken = true;
                        }
                    }
                }
                const Mono incl = warp_scan(t, ln);
                Mono ex;
                ex.d0 = __shfl_up_sync(FULL, incl.d0, 1);
                ex.d1 = __shfl_up_sync(FULL, incl.d1, 1);
                if (ln == 0) ex = mono_id();
                int mm = apply(m, ex);
                int stop = 0x7fffffff;
#pragma unroll
                for (int q = 0; q < SPT; q++) {
                    const int r = c + ln * SPT + q;
                    if (r >= wend || stop != 0x7fffffff) continue;
                    if (!ok[q]) { stop = r; continue; }
                    const int mn = apply(mm, mine[q]);
                    if (mn >= (1 << 24)) { stop = r; continue; }
                    mm = mn;
                }
                int first = stop;
#pragma unroll
                for (int d = 16; d >= 1; d >>= 1) first = min(first, __shfl_xor_sync(FULL, first, d));
                if (first == 0x7fffffff) {
                    const int mend = __shfl_sync(FULL, mm, (wend - 1 - c) / SPT);
                    note(c, wend - 1, eb);
                    s = from_m(mend, eb);
                    c = wend;
                    continue;
                }
                const int ms = __shfl_sync(FULL, mm, (first - c) / SPT);
                note(c, first, eb);
                s = resolve(first, from_m(ms, eb));
                c = first + 1;
            }
            if (ln == 0) sm.nlog = min(nlog, LOGN);
        }
        __syncthreads();
        // ---- binade history of the page from the run log (all warps)
        for (int k = warp; k < sm.nlog; k += 8) {
            const int4 L = sm.log[k];
            for (int i = L.x + ln; i <= L.y; i += 32) hist[p0 + i] = L.z;
        }
        __syncthreads();
    }

    // ---- lane sum out; the last lane of the channel reduces and divides
    if (tid == 0) {
        sc.lanes[j] = s;
        __threadfence();
        const unsigned done = atomicAdd(sc.counter, 1u);
        if (done == LANES - 1) {
            __threadfence();
            const volatile float* L = sc.lanes;
            float h[4] = {0.f, 0.f, 0.f, 0.f};
            float tot = 0.0f;
            long long i = g.main;
            if (g.main > 0) {
                for (int k = 0; k < 4; k++) h[k] = __fadd_rn(L[k], L[k + 4]);
                tot = __fadd_rn(__fadd_rn(h[0], h[2]), __fadd_rn(h[1], h[3]));
            }
            if (g.n6 - i >= 4) {   // the 4-wide epilogue block
                float q[4];
                for (int k = 0; k < 4; k++) q[k] = __fadd_rn(h[k], __uint_as_float(v6_bits(v, i + k)));
                tot = __fadd_rn(__fadd_rn(q[0], q[2]), __fadd_rn(q[1], q[3]));
                i += 4;
            }
            for (; i < g.n6; i++) tot = __fadd_rn(tot, __uint_as_float(v6_bits(v, i)));
            const float nf = __ll2float_rn(g.n6);
            const float thr = a.batch_form ? __fmul_rn(__fdiv_rn(0.2f, nf), tot)
                                           : __fmul_rn(__fdiv_rn(tot, nf), 0.2f);
            a.thr[ch] = thr;
            if (a.sums) a.sums[ch] = tot;
            *sc.counter = 0u;
        }
    }
}

// ---- the planes_fp16 precision variant: the threshold of FP16 planes.
// Not the reference's vectorised FP32 sum: the sum of |x| over the 6-slot
// array (each unique band twice - slots 3-5 mirror 2-0) in FP64 from
// per-block partial sums, which the last block to finish adds in block
// order (the result does not depend on timing), then (S / N6) * 0.2 or
// (0.2 / N6) * S in FP64, rounded to FP32 once.  Grid: nblk x channels.
constexpr int T16_THREADS = 256;

__device__ __forceinline__ void thr16_body(const ThrArgs& a, int bx, int by, int nblk) {
    const int ch = by;
    const PyrView& v = a.v[ch];
    const ThrScratch& sc = a.s[ch];
    const long long pu = v.off6[v.levels] / 2;             // unique positions: half the 6-slot count
    const __half* x = reinterpret_cast<const __half*>(v.coef);
    double acc = 0.0;
    for (long long u = (long long)bx * T16_THREADS + threadIdx.x; u < pu; u += (long long)nblk * T16_THREADS)
        acc += (double)fabsf(__half2float(x[u]));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(FULL, acc, d);
    __shared__ double ws[T16_THREADS / 32];
    __shared__ bool last;
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln == 0) ws[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < T16_THREADS / 32; w++) b += ws[w];
        sc.part[bx] = b;
        __threadfence();
        last = atomicAdd(sc.counter, 1u) == (unsigned)(nblk - 1);
    }
    __syncthreads();
    if (!last || warp != 0) return;
    __threadfence();
    const volatile double* part = sc.part;
    double t = 0.0;
    for (int i = ln; i < nblk; i += 32) t += part[i];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) t += __shfl_xor_sync(FULL, t, d);
    if (ln == 0) {
        const double s6 = 2.0 * t, n6 = (double)v.off6[v.levels];
        a.thr[ch] = (float)(a.batch_form ? (0.2 / n6) * s6 : (s6 / n6) * 0.2);
        if (a.sums) a.sums[ch] = (float)s6;
        *sc.counter = 0u;
    }
}

static int thr16_blocks(const PyrView& v) {
    const long long pu = v.off6[v.levels] / 2;
    const long long b = (pu + 8LL * T16_THREADS - 1) / (8LL * T16_THREADS);
    return (int)std::min<long long>(std::max<long long>(b, 1), T16_MAXBLK);
}

// ------------------------------------------------------------- wrappers
__global__ void __launch_bounds__(T16_THREADS) k_thr16(ThrArgs a, int nblk) {
    thr16_body(a, blockIdx.x, blockIdx.y, nblk);
}
__global__ void __launch_bounds__(T16_THREADS)
    k_thr16_multi(const ThrArgs* __restrict__ as, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    thr16_body(as[t.task], t.x, t.y, map[map[0] + 2 + t.task]);
}
__global__ void __launch_bounds__(THR_THREADS) k_thr_partials(ThrArgs a) {
    thr_partials_body(a, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(THR_THREADS) k_thr_prefix(ThrArgs a) {
    thr_prefix_body(a, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(32 * MON_WARPS, MON_MINB) k_thr_monoids(ThrArgs a) {
    thr_monoids_body(a, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(THR_THREADS, 2) k_thr_walk(ThrArgs a) {
    thr_walk_body(a, blockIdx.x, blockIdx.y);
}
// batched: task = one stream's ThrArgs
__global__ void __launch_bounds__(THR_THREADS)
    k_thr_partials_multi(const ThrArgs* __restrict__ as, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    thr_partials_body(as[t.task], t.x, t.y);
}
__global__ void __launch_bounds__(THR_THREADS)
    k_thr_prefix_multi(const ThrArgs* __restrict__ as, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    thr_prefix_body(as[t.task], t.x, t.y);
}
__global__ void __launch_bounds__(32 * MON_WARPS, MON_MINB)
    k_thr_monoids_multi(const ThrArgs* __restrict__ as, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    thr_monoids_body(as[t.task], t.x, t.y);
}
__global__ void __launch_bounds__(THR_THREADS, 2)
    k_thr_walk_multi(const ThrArgs* __restrict__ as, const int* __restrict__ map) {
    const TaskBlock t = task_block(map, blockIdx.x);
    thr_walk_body(as[t.task], t.x, t.y);
}

cudaError_t thr_prepare_device() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned char> done[64];
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
    // the walk: two CTAs per SM (about 101 KB of shared memory and at most 128
    // registers each), so a batch's lanes x streams take fewer waves
    e = cudaFuncSetAttribute(k_thr_walk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(WalkSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_thr_walk_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(WalkSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_thr_walk, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_thr_walk_multi, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev].store(1, std::memory_order_release);
    return e;
}

cudaError_t launch_threshold(const PyrView* views, int nch, ThrScratch* scratch, float* thr,
                             float* sums, int batch_form, int use_hist, int h16, cudaStream_t st) {
    if (nch < 1 || nch > 3) return cudaErrorInvalidValue;
    cudaError_t e = thr_prepare_device();
    if (e != cudaSuccess) return e;
    ThrArgs a{};
    int nsub = 0;
    for (int c = 0; c < nch; c++) {
        a.v[c] = views[c];
        a.s[c] = scratch[c];
        nsub = max(nsub, thr_geom(views[c].off6[views[c].levels]).nsub);
    }
    a.thr = thr;
    a.sums = sums;
    a.batch_form = batch_form;
    a.use_hist = use_hist;
    if (h16) {
        const int nb = thr16_blocks(views[0]);
        k_thr16<<<dim3(nb, nch), T16_THREADS, 0, st>>>(a, nb);
        return cudaGetLastError();
    }
    if (!use_hist && nsub > 0) {
        k_thr_partials<<<dim3(nsub, nch), THR_THREADS, 0, st>>>(a);
        k_thr_prefix<<<dim3(LANES, nch), THR_THREADS, 0, st>>>(a);
    }
    k_thr_monoids<<<dim3(max((nsub + MON_WARPS - 1) / MON_WARPS, 1), nch), 32 * MON_WARPS, 0, st>>>(a);
    k_thr_walk<<<dim3(LANES, nch), THR_THREADS, sizeof(WalkSmem), st>>>(a);
    return cudaGetLastError();
}

// ---- batched threshold (the host fills one ThrArgs per stream)
size_t thr_args_bytes() { return sizeof(ThrArgs); }

cudaError_t thr_args_fill(void* dst, const PyrView* views, int nch, const ThrScratch* scratch,
                          float* thr, float* sums, int batch_form, int use_hist, unsigned grids[5][2]) {
    if (nch < 1 || nch > 3) return cudaErrorInvalidValue;
    ThrArgs a{};
    int nsub = 0;
    for (int c = 0; c < nch; c++) {
        a.v[c] = views[c];
        a.s[c] = scratch[c];
        nsub = max(nsub, thr_geom(views[c].off6[views[c].levels]).nsub);
    }
    a.thr = thr;
    a.sums = sums;
    a.batch_form = batch_form;
    a.use_hist = use_hist;
    memcpy(dst, &a, sizeof a);
    grids[0][0] = (unsigned)nsub;                                         // partials
    grids[1][0] = LANES;                                                  // prefix
    grids[2][0] = (unsigned)max((nsub + MON_WARPS - 1) / MON_WARPS, 1);   // monoids
    grids[3][0] = LANES;                                                  // walk
    grids[4][0] = (unsigned)thr16_blocks(views[0]);                        // FP16 planes
    for (int k = 0; k < 5; k++) grids[k][1] = (unsigned)nch;
    if (nsub == 0) grids[0][0] = 0;
    return cudaSuccess;
}

int thr_level0_subchunks(const PyrView& v) {
    if (v.levels < 2) return 0;
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    return (int)std::min<long long>(v.off6[1] / (LANES * G), g.nsub);
}

unsigned thr_args_monoid_part(void* args, int sub0, int sub1) {
    ThrArgs a;
    memcpy(&a, args, sizeof a);
    if (sub1 < 0)
        for (int c = 0; c < 3; c++) sub1 = max(sub1, thr_geom(a.v[c].off6[a.v[c].levels]).nsub);
    a.sub0 = sub0;
    memcpy(args, &a, sizeof a);
    return (unsigned)((sub1 - sub0 + MON_WARPS - 1) / MON_WARPS);
}

cudaError_t launch_threshold_multi(int stage, const void* d_args, const int* d_map, unsigned blocks,
                                   cudaStream_t st) {
    if (blocks == 0) return cudaSuccess;
    cudaError_t e = thr_prepare_device();
    if (e != cudaSuccess) return e;
    const ThrArgs* as = static_cast<const ThrArgs*>(d_args);
    switch (stage) {
        case 0: k_thr_partials_multi<<<blocks, THR_THREADS, 0, st>>>(as, d_map); break;
        case 1: k_thr_prefix_multi<<<blocks, THR_THREADS, 0, st>>>(as, d_map); break;
        case 2: k_thr_monoids_multi<<<blocks, 32 * MON_WARPS, 0, st>>>(as, d_map); break;
        case 3: k_thr_walk_multi<<<blocks, THR_THREADS, sizeof(WalkSmem), st>>>(as, d_map); break;
        case 4: k_thr16_multi<<<blocks, T16_THREADS, 0, st>>>(as, d_map); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace wema
