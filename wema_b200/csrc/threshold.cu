// threshold.cu - the reference's adaptive threshold, bit for bit.
//
// The reference computes thr = (sum|x| / N) * 0.2 over the 6-slot flat
// coefficient array (wema.c:719-723, phase_amp.c:25-29; the batch route uses
// (0.2 / N) * sum, wema_batch.c:272-276).  Its -Ofast build vectorises the
// sum as eight sequential FP32 lane sums (lane j = elements 8t + j), reduced
// ((l0+l4)+(l2+l6)) + ((l1+l5)+(l3+l7)), plus a 4-wide/scalar epilogue for the
// last N mod 8 elements.  A mask bit |x| > thr flips if thr is off by one ulp,
// so the lane sums must be reproduced exactly - each is a chain of N/8
// dependent FP32 adds (516k at 1080p).
//
// Parallel exact method.  While the running sum s stays in one binade
// [2^e, 2^(e+1)), s = m * u with u = 2^(e-23) and m a 24-bit integer, and
// fl(s + a) = u * rne(m + a/u): the increment is round(a/u) unless a/u is an
// exact half, where it rounds to the even result, i.e. depends on m's parity.
// So a run of elements acts on m as  m -> m + d[m & 1]  - a two-entry
// "parity monoid" {d0, d1}, composable in any grouping:
//   (A then B)[p] = A[p] + B[(p + A[p]) & 1].
// Kernels:
//   thr_partials  - per (sub-chunk, lane) FP64 sum of |x| (exact enough to
//                   predict the binade of s at each sub-chunk start);
//   thr_prefix    - exclusive FP64 prefix per lane;
//                   (both skipped when the previous frame's walk recorded the
//                   binade at every sub-chunk start: a video's coefficient
//                   statistics move slowly, and a wrong guess only costs time)
//   thr_monoids   - per (sub-chunk, lane) monoids for the three binades
//                   around the predicted one;
//   thr_walk      - one warp per lane composes 32 sub-chunks at a time by a
//                   warp scan, accepts the prefix that stays inside the
//                   binade, and resolves a crossing (or an unpredicted
//                   binade) element by element: the element where s leaves
//                   the binade is added with a real FP32 add from the exact
//                   value before it.  Then the epilogue and the division.
// The prediction only decides speed, never the result.
#include "common.cuh"
#include "kernels.h"

namespace wema {

constexpr int LANES = 8;
constexpr int THR_THREADS = 256;
constexpr int SAT = 1 << 25;      // saturated increment: certainly leaves the binade
constexpr int NCAND = 3;          // binades tried per sub-chunk: top, top-1, top-2

struct Mono { int d0, d1; };

__device__ __forceinline__ Mono mono_id() { return {0, 0}; }

__device__ __forceinline__ Mono compose(Mono a, Mono b) {   // a first, then b
    Mono r;
    r.d0 = min(a.d0 + ((a.d0 & 1) ? b.d1 : b.d0), SAT);
    r.d1 = min(a.d1 + (((a.d1 + 1) & 1) ? b.d1 : b.d0), SAT);
    return r;
}

// effect of adding |x| (bits ua, sign cleared) to any s of biased exponent eb
__device__ __forceinline__ Mono elem_mono(uint32_t ua, int eb) {
    int ea = ua >> 23;
    int ma = ua & 0x7FFFFF;
    if (ea) ma |= 0x800000; else ea = 1;
    const int shift = eb - ea;
    if (shift <= 0) return {SAT, SAT};
    if (shift >= 25) return {0, 0};
    const int q = ma >> shift;
    const int r = ma & ((1 << shift) - 1);
    const int half = 1 << (shift - 1);
    if (r > half) return {q + 1, q + 1};
    if (r < half) return {q, q};
    return {q + (q & 1), q + 1 - (q & 1)};
}

__device__ __forceinline__ float from_m(int m, int eb) {
    return __uint_as_float(((uint32_t)eb << 23) | ((uint32_t)m & 0x7FFFFFu));
}

// Sequential reader of |element| of the 6-slot flat array (slots 3-5 mirror
// 2-0).  seek() places it on the (level, slot) segment holding index i; get()
// advances segment by segment, so a run of nearby indices costs one division.
// levels == 0 views coef as a plain flat array of off6[0] elements.
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

__device__ __forceinline__ uint32_t cur_get(const PyrView& v, Cursor& c, long long i) {
    return __float_as_uint(*cur_addr(v, c, i)) & 0x7FFFFFFFu;
}

// |x| bits of the EPT lane-elements t0 .. t0+EPT-1 of lane j: all addresses
// first, then all loads, so they are in flight together
template <int EPT>
__device__ __forceinline__ void load_run(const PyrView& v, long long nlane, long long t0, int j,
                                         uint32_t (&out)[EPT]) {
    const float* addr[EPT];
    Cursor cu;
    if (t0 < nlane) cur_seek(v, cu, 8 * t0 + j);
#pragma unroll
    for (int k = 0; k < EPT; k++) addr[k] = (t0 + k < nlane) ? cur_addr(v, cu, 8 * (t0 + k) + j) : nullptr;
#pragma unroll
    for (int k = 0; k < EPT; k++) out[k] = addr[k] ? (__float_as_uint(__ldg(addr[k])) & 0x7FFFFFFFu) : 0u;
}

__device__ __forceinline__ uint32_t v6_bits(const PyrView& v, long long i) {
    Cursor c;
    cur_seek(v, c, i);
    return cur_get(v, c, i);
}

struct ThrGeom {
    long long n6, main, nlane;   // main = elements summed by the 8 lanes
    int G, nsub;                 // lane-elements per sub-chunk, sub-chunks per lane
};

__host__ __device__ inline ThrGeom thr_geom(long long n6) {
    ThrGeom g;
    g.n6 = n6;
    g.main = (n6 - 1 <= 6) ? 0 : (n6 & ~7LL);
    g.nlane = g.main / LANES;
    g.G = 256;
    while (g.G < 1024 && (g.nlane + g.G - 1) / g.G > 2048) g.G *= 2;
    g.nsub = (int)((g.nlane + g.G - 1) / g.G);
    return g;
}

size_t thr_scratch_bytes(long long n6) {
    ThrGeom g = thr_geom(n6);
    size_t per = (size_t)g.nsub * LANES;
    return per * (sizeof(double) * 2 + sizeof(int4) * 2 + sizeof(int)) + 256;
}

void thr_scratch_bind(ThrScratch& s, void* base, long long n6) {
    ThrGeom g = thr_geom(n6);
    size_t per = (size_t)g.nsub * LANES;
    char* p = (char*)base;
    s.part = (double*)p;   p += per * sizeof(double);
    s.prefix = (double*)p; p += per * sizeof(double);
    s.cand = (int4*)p;     p += per * 2 * sizeof(int4);   // two int4 per (sub-chunk, lane)
    s.hist = (int*)p;
}

struct ThrArgs {
    PyrView v[3];
    ThrScratch s[3];
    float* thr;
    float* sums;
    int batch_form;
    int use_hist;
};

// ---- partial sums: thread (lane j, block tb) covers G/32 lane-elements
template <int EPT>
__global__ void __launch_bounds__(THR_THREADS) k_thr_partials(ThrArgs a) {
    const int ch = blockIdx.y;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const int sub = blockIdx.x;
    const int j = threadIdx.x & 7, tb = threadIdx.x >> 3;
    const long long t0 = (long long)sub * g.G + (long long)tb * EPT;
    uint32_t val[EPT];
    load_run<EPT>(v, g.nlane, t0, j, val);
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < EPT; k++) acc += (double)__uint_as_float(val[k]);
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    __shared__ double ws[8][8];
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln < 8) ws[warp][ln] = acc;
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s += ws[w][threadIdx.x];
        a.s[ch].part[(long long)sub * LANES + threadIdx.x] = s;
    }
}

// ---- exclusive prefix per lane: one CTA per (lane, channel), 8 entries per
// thread per pass, block-wide scan in shared memory
__global__ void __launch_bounds__(THR_THREADS) k_thr_prefix(ThrArgs a) {
    const int j = blockIdx.x, ch = blockIdx.y;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const double* part = a.s[ch].part;
    double* pre = a.s[ch].prefix;
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
            x[k] = c < g.nsub ? part[(long long)c * LANES + j] : 0.0;
            local += x[k];
        }
        double incl = local;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_up_sync(0xffffffffu, incl, d);
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
            if (c < g.nsub) pre[(long long)c * LANES + j] = run;
            run += x[k];
        }
        if (threadIdx.x == THR_THREADS - 1) carry_s = run;
        __syncthreads();
        carry = carry_s;
        __syncthreads();
    }
}

__device__ __forceinline__ int predicted_top_binade(double s) {
    float f = (float)(s * (1.0 + 1.0 / 512.0));
    return (int)(__float_as_uint(f) >> 23);   // 0 for zero / subnormal
}

// ---- monoids for the candidate binades of each (sub-chunk, lane)
template <int EPT>
__global__ void __launch_bounds__(THR_THREADS) k_thr_monoids(ThrArgs a) {
    const int ch = blockIdx.y;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const int sub = blockIdx.x;
    const int j = threadIdx.x & 7, tb = threadIdx.x >> 3;
    const int etop = a.use_hist ? a.s[ch].hist[(long long)sub * LANES + j] + 1
                                : predicted_top_binade(a.s[ch].prefix[(long long)sub * LANES + j]);
    Mono m[NCAND];
#pragma unroll
    for (int c = 0; c < NCAND; c++) m[c] = mono_id();
    const long long t0 = (long long)sub * g.G + (long long)tb * EPT;
    uint32_t val[EPT];
    load_run<EPT>(v, g.nlane, t0, j, val);
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        const long long t = t0 + k;
        if (t < g.nlane) {
            const uint32_t ua = val[k];
#pragma unroll
            for (int c = 0; c < NCAND; c++) m[c] = compose(m[c], elem_mono(ua, etop - c));
        }
    }
    // ordered combine over tb: lanes j, j+8, j+16, j+24 of a warp hold tb = 4w..4w+3
#pragma unroll
    for (int d = 8; d <= 16; d <<= 1) {
#pragma unroll
        for (int c = 0; c < NCAND; c++) {
            Mono o;
            o.d0 = __shfl_down_sync(0xffffffffu, m[c].d0, d);
            o.d1 = __shfl_down_sync(0xffffffffu, m[c].d1, d);
            if (((threadIdx.x & 31) & d) == 0) m[c] = compose(m[c], o);
        }
    }
    __shared__ Mono wm[8][8][NCAND];
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln < 8) {
#pragma unroll
        for (int c = 0; c < NCAND; c++) wm[warp][ln][c] = m[c];
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        Mono r[NCAND];
#pragma unroll
        for (int c = 0; c < NCAND; c++) {
            r[c] = mono_id();
            for (int w = 0; w < 8; w++) r[c] = compose(r[c], wm[w][threadIdx.x][c]);
        }
        int4* out = a.s[ch].cand + 2 * ((long long)sub * LANES + threadIdx.x);
        out[0] = make_int4(etop, r[0].d0, r[0].d1, r[1].d0);
        out[1] = make_int4(r[1].d1, r[2].d0, r[2].d1, 0);
    }
}

// ---- the walk
__device__ __forceinline__ Mono warp_scan(Mono t, int ln) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        Mono o;
        o.d0 = __shfl_up_sync(0xffffffffu, t.d0, d);
        o.d1 = __shfl_up_sync(0xffffffffu, t.d1, d);
        if (ln >= d) t = compose(o, t);
    }
    return t;
}

// exact sum over sub-chunk `sub` of lane j starting from s (warp-collective)
template <int EPT>
__device__ float resolve_sub(const PyrView& v, const ThrGeom& g, int j, int sub, float s, int ln) {
    uint32_t val[EPT];
    load_run<EPT>(v, g.nlane, (long long)sub * g.G + (long long)ln * EPT, j, val);
    int pos = 0;
    while (pos < 32) {
        const uint32_t sb = __float_as_uint(s);
        const int eb = sb >> 23;
        if (eb == 0) {   // zero or subnormal running sum: plain adds for one thread's run
            float x = s;
            if (ln == pos) {
#pragma unroll
                for (int k = 0; k < EPT; k++) x = __fadd_rn(x, __uint_as_float(val[k]));
            }
            s = __shfl_sync(0xffffffffu, x, pos);
            pos++;
            continue;
        }
        const int m = (sb & 0x7FFFFF) | 0x800000;
        Mono t = mono_id();
        if (ln >= pos) {
#pragma unroll
            for (int k = 0; k < EPT; k++) t = compose(t, elem_mono(val[k], eb));
        }
        t = warp_scan(t, ln);
        const int mend = m + ((m & 1) ? t.d1 : t.d0);
        const unsigned cross = __ballot_sync(0xffffffffu, ln >= pos && mend >= (1 << 24));
        if (!cross) {
            s = from_m(__shfl_sync(0xffffffffu, mend, 31), eb);
            break;
        }
        const int tc = __ffs(cross) - 1;
        const int mprev = __shfl_sync(0xffffffffu, mend, tc > 0 ? tc - 1 : 0);
        float x = from_m(tc > pos ? mprev : m, eb);
        if (ln == tc) {
#pragma unroll
            for (int k = 0; k < EPT; k++) x = __fadd_rn(x, __uint_as_float(val[k]));
        }
        s = __shfl_sync(0xffffffffu, x, tc);
        pos = tc + 1;
    }
    return s;
}

// monoid of a sub-chunk for binade eb from its stored candidates, if present
__device__ __forceinline__ bool cand_mono(const int4& k0, const int4& k1, int eb, Mono& m) {
    const int dlt = k0.x - eb;
    if (k0.x <= 0 || dlt < 0 || dlt >= NCAND) return false;
    if (dlt == 0) m = {k0.y, k0.z};
    else if (dlt == 1) m = {k0.w, k1.x};
    else m = {k1.y, k1.z};
    return true;
}

constexpr int SPT = 4;                // sub-chunks per lane-thread in a walk window
constexpr int WIN = 32 * SPT;

template <int EPT>
__global__ void __launch_bounds__(THR_THREADS, 1) k_thr_walk(ThrArgs a) {
    const int ch = blockIdx.x;
    const PyrView& v = a.v[ch];
    const ThrGeom g = thr_geom(v.off6[v.levels]);
    const int j = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const int4* cand = a.s[ch].cand;
    float s = 0.0f;
    int4 k0[SPT], k1[SPT], n0[SPT], n1[SPT];
    auto load = [&](int c0, int4* K0, int4* K1) {
#pragma unroll
        for (int q = 0; q < SPT; q++) {
            const int c = c0 + ln * SPT + q;
            if (c < g.nsub) {
                K0[q] = cand[2 * ((long long)c * LANES + j)];
                K1[q] = cand[2 * ((long long)c * LANES + j) + 1];
            } else {
                K0[q] = make_int4(0, 0, 0, 0);
                K1[q] = make_int4(0, 0, 0, 0);
            }
        }
    };
    if (g.nsub > 0) load(0, k0, k1);
    for (int c0 = 0; c0 < g.nsub; c0 += WIN) {
        if (c0 + WIN < g.nsub) load(c0 + WIN, n0, n1);   // prefetch the next window
        const int wend = min(WIN, g.nsub - c0);
        const int my0 = ln * SPT;
        int off = 0;
        while (off < wend) {
            const uint32_t sb = __float_as_uint(s);
            const int eb = sb >> 23;
            if (eb == 0) {   // zero / subnormal running sum: exact element walk
                if (ln == 0) a.s[ch].hist[(long long)(c0 + off) * LANES + j] = 0;
                s = resolve_sub<EPT>(v, g, j, c0 + off, s, ln);
                off++;
                continue;
            }
            const int m = (sb & 0x7FFFFF) | 0x800000;
            int* hist = a.s[ch].hist + j;
            // my sub-chunks' composition, up to my first missing candidate
            Mono t = mono_id();
#pragma unroll
            for (int q = 0; q < SPT; q++) {
                const int r = my0 + q;
                if (r >= off && r < wend) {
                    Mono mq;
                    if (!cand_mono(k0[q], k1[q], eb, mq)) break;
                    t = compose(t, mq);
                }
            }
            const Mono incl = warp_scan(t, ln);
            Mono ex;
            ex.d0 = __shfl_up_sync(0xffffffffu, incl.d0, 1);
            ex.d1 = __shfl_up_sync(0xffffffffu, incl.d1, 1);
            if (ln == 0) ex = mono_id();
            // exact m at my first sub-chunk, valid if nothing went wrong before it
            int mm = m + ((m & 1) ? ex.d1 : ex.d0);
            int stop = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < SPT; q++) {
                const int r = my0 + q;
                if (r < off || r >= wend || stop != 0x7fffffff) continue;
                Mono mq;
                if (!cand_mono(k0[q], k1[q], eb, mq)) { stop = r; continue; }
                const int mn = mm + ((mm & 1) ? mq.d1 : mq.d0);
                if (mn >= (1 << 24)) { stop = r; continue; }
                mm = mn;
                hist[(long long)(c0 + r) * LANES] = eb;   // accepted: starts in binade eb
            }
            int first = stop;
#pragma unroll
            for (int d = 16; d >= 1; d >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, d));
            if (first == 0x7fffffff) {   // the rest of the window stays in this binade
                s = from_m(__shfl_sync(0xffffffffu, mm, (wend - 1) / SPT), eb);
                break;
            }
            const int mp = __shfl_sync(0xffffffffu, mm, first / SPT);
            if (first > off) s = from_m(mp, eb);
            if (ln == 0) hist[(long long)(c0 + first) * LANES] = eb;
            s = resolve_sub<EPT>(v, g, j, c0 + first, s, ln);
            off = first + 1;
        }
#pragma unroll
        for (int q = 0; q < SPT; q++) { k0[q] = n0[q]; k1[q] = n1[q]; }
    }
    __shared__ float lane_sum[LANES];
    if (ln == 0) lane_sum[j] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        // reduction of the vector accumulator and the epilogue (N mod 8)
        float h[4] = {0.f, 0.f, 0.f, 0.f};
        float tot = 0.0f;
        long long i = g.main;
        if (g.main > 0) {
            for (int k = 0; k < 4; k++) h[k] = __fadd_rn(lane_sum[k], lane_sum[k + 4]);
            tot = __fadd_rn(__fadd_rn(h[0], h[2]), __fadd_rn(h[1], h[3]));
        }
        if (g.n6 - i >= 4) {
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
    }
}

template <int EPT>
static cudaError_t thr_launch(const ThrArgs& a, int nch, int nsub_max, cudaStream_t st) {
    if (nsub_max > 0) {
        if (!a.use_hist) {
            k_thr_partials<EPT><<<dim3(nsub_max, nch), THR_THREADS, 0, st>>>(a);
            k_thr_prefix<<<dim3(LANES, nch), THR_THREADS, 0, st>>>(a);
        }
        k_thr_monoids<EPT><<<dim3(nsub_max, nch), THR_THREADS, 0, st>>>(a);
    }
    k_thr_walk<EPT><<<nch, THR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_threshold(const PyrView* views, int nch, ThrScratch* scratch, float* thr,
                             float* sums, int batch_form, int use_hist, cudaStream_t st) {
    if (nch < 1 || nch > 3) return cudaErrorInvalidValue;
    ThrArgs a{};
    int G = 0;
    for (int c = 0; c < nch; c++) {
        a.v[c] = views[c];
        a.s[c] = scratch[c];
        ThrGeom g = thr_geom(views[c].off6[views[c].levels]);
        if (c > 0 && g.G != G) return cudaErrorInvalidValue;   // channels share a geometry
        G = g.G;
    }
    a.thr = thr;
    a.sums = sums;
    a.batch_form = batch_form;
    a.use_hist = use_hist;
    const int nsub = thr_geom(views[0].off6[views[0].levels]).nsub;
    switch (G) {
        case 256: return thr_launch<8>(a, nch, nsub, st);
        case 512: return thr_launch<16>(a, nch, nsub, st);
        case 1024: return thr_launch<32>(a, nch, nsub, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace wema
