// FP32 compensated periodic direct sum (sm_100a).
//
// Same field as E_MQ_DirectSum (src/FieldStructure.cpp:106-156), rewritten as
//   E_i = sum_j q_j g(d_ij) - c * sum_j q_j d_ij,   g(d) = d / (2 sqrt(d^2 + eps^2)),
//   d_ij = x_i - x_j wrapped into [-L/2, L/2],       c = 1 / sqrt(L^2 + 4 eps^2).
// The second (neutralising-background) term is linear in d and is evaluated
// exactly in FP64 from prefix sums over the x-sorted sources.  Only g is
// evaluated per pair, in FP32:
//
//  * Sources are wrapped into [0, L), sorted by x and cut into tiles of kS.
//    Each tile stores FP32 offsets s_j = x_j - b_t from an FP64 tile base b_t,
//    and q_j/2.  Per (target, tile) the target offset tau = x_i + shift - b_t
//    is formed in FP64 and rounded once, so d = tau - s_j is accurate to the
//    tile's scale, not to L.
//  * The periodic image of every pair is fixed by one index J_i per target
//    (sources before / after J_i take one of two images); the FP64 background
//    term uses the same split, so both halves of the kernel agree exactly on
//    which image a pair uses.
//  * Per target the sources split into far pairs (|d| > 16 eps) and a band
//    (|d| <= 16 eps), by index (binary searches in FP64).  A far pair
//    contributes sign(d) q/2 (1 - c(v)) with v = eps^2/(d^2+eps^2) <= 1/257:
//    the sign(d) q/2 part is summed exactly in FP64 from prefix sums of the
//    FP64 charges; the pair kernel only accumulates q/2 * c(v) in FP32, with
//    the shifted one-term series c = a1 / (d^2 + 3 eps^2 / 4), a1 = eps^2/2,
//    whose error is below v^2/16 of c and which carries FP32's relative error
//    on a quantity of order eps^2/d^2.  Band pairs (about 2% on the two-stream
//    deck) are evaluated in FP64, q/2 d / sqrt(d^2 + eps^2), from FP64 source
//    records staged beside the FP32 ones.  Every tile's partial sum is added
//    into an FP64 accumulator.
//  * Far pairs need no square root: per two targets FFMA2 (d), FFMA2
//    (d^2 + 3 eps^2/4), FMUL + one MUFU.RCP for both reciprocals, FMUL, FFMA2:
//    4 FP32 lane-operations and 0.5 MUFU op per pair, loading the FP32
//    datapath (128 lanes/clk/SM) and MUFU (16/clk/SM) equally.  Source tiles
//    move global->shared by TMA bulk copies (cp.async.bulk, no multicast),
//    double-buffered on mbarriers.
//
// Work is split into (target block, source chunk) items, taken from an atomic
// counter by a one-wave persistent grid in an order estimated on the device
// (band-heavy items spread over the queue, light ones last); chunk partials are
// summed in a fixed order by the finalize kernel, which also applies the fused
// RK4 stage epilogue.
#include <cub/cub.cuh>

#include <cstdlib>
#include <mutex>

#include "fs_device.cuh"

namespace fsb {

namespace {

#ifndef FS_TILE_SOURCES
#define FS_TILE_SOURCES 256
#endif
constexpr int kS = FS_TILE_SOURCES;  // sources per shared-memory tile
// Threads per CTA: two warps (64) measured 1.3-1.5% faster than four (128)
// on the two-stream and batch workloads (eight CTAs per SM instead of four, so
// a CTA's barrier per tile holds fewer warps), one warp (32) no faster.
#ifndef FS_NT
#define FS_NT 64
#endif
constexpr int kNT = FS_NT;       // threads per CTA
constexpr int kRMax = 8;         // largest number of targets per thread
constexpr int kTBPad = kNT * kRMax;  // target counts are padded to a multiple of this

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared (TMA), completion signalled on `bar`.
// Source and destination are 16-byte aligned and bytes is a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, "
        "p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Polls of one bounded mbarrier wait before it gives up (each poll may itself
// suspend the thread for a short, hardware-chosen time).
constexpr long long kMbarPolls = 1LL << 22;
// The bound the pair kernels use for the waits on their source tiles.
// fs_debug_set_wait_limits lowers it (0 = give up at once) so that tests can
// drive the timeout path; the drain waits of that path always use kMbarPolls.
__device__ long long g_mbar_polls = kMbarPolls;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long polls) {
    for (long long it = 0; it < polls; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}


__device__ __forceinline__ double key_to_x(uint64_t k) { return __longlong_as_double((long long)k); }

// Band pair in FP64, accumulated: acc + (q/2) d / sqrt(r), r = d^2 + eps^2,
// from the source's q/4.  1/sqrt(r) is the hardware approximation y refined
// by one Newton-Raphson step y (3 - r y^2) / 2 (which squares its relative
// error); the step's 1/2 is folded into the stored q/4:
//   (q/2) d y (3 - r y^2) / 2 = ((q/4) d y) (3 - r y^2),
// 7 FP64 operations per pair with the difference and r.
__device__ __forceinline__ double band_acc64(double q4, double d, double r, double acc) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r));
    const double a = (q4 * d) * y;
    const double v = fma(-r, y * y, 3.0);
    return fma(a, v, acc);
}

// x -> [0, L) and its order-preserving key (non-negative doubles sort as
// unsigned integers).
__global__ void k_wrap_keys(const double* __restrict__ x, int n, double L, uint64_t* __restrict__ keys,
                            int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double w = x[i] - L * floor(x[i] / L);
    if (w >= L) w -= L;
    if (w < 0.0) w = 0.0;
    w = w + 0.0;  // -0 -> +0
    keys[i] = (uint64_t)__double_as_longlong(w);
    idx[i] = i;
}

// Sorted sources -> tile-relative FP32 records {s, q/2, q/2 a1, q/2 a2}
// (pads all zero), the FP64 tile bases, and the FP64 q and q*x the exact sums
// are formed from.  a1 = eps^2/2, a2 = eps^4/8 are the far-pair series
// coefficients, folded into the source's charge once here.
__global__ void k_gather_sources(const uint64_t* __restrict__ skeys, const int* __restrict__ sidx,
                                 const double* __restrict__ q, int ns, int ns_pad, double a1, double a2,
                                 float4* __restrict__ src, double2* __restrict__ src64, double* __restrict__ tbase,
                                 double* __restrict__ qs, double* __restrict__ qx) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns_pad) return;
    if (j >= ns) {
        src[j] = make_float4(0.f, 0.f, 0.f, 0.f);
        src64[j] = make_double2(0.0, 0.0);
        return;
    }
    const double xj = key_to_x(skeys[j]);
    const double base = key_to_x(skeys[(j / kS) * kS]);
    if (j % kS == 0) tbase[j / kS] = base;
    const double qj = q[sidx[j]];
    const float qh = (float)(0.5 * qj);
    src[j] = make_float4((float)(xj - base), qh, (float)((double)qh * a1), (float)((double)qh * a2));
    src64[j] = make_double2(xj, 0.25 * qj);
    qs[j] = qj;
    qx[j] = qj * xj;
}

// Position along the target's periodic window.  Sources are visited in the
// cyclic order J, J+1, ..., n-1, 0, ..., J-1 ("unrolled" index u in [J, J+n));
// X(u) = x_(u mod n) + L*(u >= n) increases with u and d(u) = tlo + L - X(u).
__device__ __forceinline__ double unrolled_x(const uint64_t* __restrict__ skeys, int n, double L, int u) {
    return (u >= n) ? key_to_x(skeys[u - n]) + L : key_to_x(skeys[u]);
}
__device__ __forceinline__ int unrolled_lower_bound(const uint64_t* __restrict__ skeys, int n, double L, int lo,
                                                    int hi, double v, bool strict) {
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        const double xm = unrolled_x(skeys, n, L, mid);
        if (strict ? (xm <= v) : (xm < v)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// exclusive prefix of the periodic extension: sum of w over unrolled [0, u)
__device__ __forceinline__ double unrolled_prefix(const double* __restrict__ incl, int n, int u) {
    const int k = u / n, r = u - k * n;
    return k * incl[n - 1] + (r ? incl[r - 1] : 0.0);
}

// Per sorted target: the image split J, the near band [U1, U2) in unrolled
// index space (|d| <= band), and the far-band sign sum.
__global__ void k_target_info(const uint64_t* __restrict__ tkeys, int nt, int nt_pad,
                              const uint64_t* __restrict__ skeys, int ns, double L, double band,
                              const double* __restrict__ pq, TargetInfo* __restrict__ info) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt_pad) return;
    TargetInfo T;
    T.pad = 0;
    if (i >= nt) {
        T.tlo = 0.0;
        T.ffar = 0.0;
        T.J = T.U1 = T.U2 = 0;
        info[i] = T;
        return;
    }
    const double xw = key_to_x(tkeys[i]);
    const double half = 0.5 * L;
    double th;
    if (xw < half) {
        th = xw + half;   // sources at or beyond x_i + L/2 use the image +L
        T.tlo = xw;
    } else {
        th = xw - half;   // sources below x_i - L/2 use the image -L
        T.tlo = xw - L;
    }
    int lo = 0, hi = ns;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key_to_x(skeys[mid]) < th) lo = mid + 1;
        else hi = mid;
    }
    T.J = lo;
    const double c = T.tlo + L;  // d(u) = c - X(u)
    T.U1 = unrolled_lower_bound(skeys, ns, L, T.J, T.J + ns, c - band, false);  // first d <= band
    T.U2 = unrolled_lower_bound(skeys, ns, L, T.U1, T.J + ns, c + band, true);  // first d < -band
    const double p_J = unrolled_prefix(pq, ns, T.J), p_1 = unrolled_prefix(pq, ns, T.U1);
    const double p_2 = unrolled_prefix(pq, ns, T.U2), p_e = unrolled_prefix(pq, ns, T.J + ns);
    T.ffar = 0.5 * ((p_1 - p_J) - (p_e - p_2));
    info[i] = T;
}

// Far tiles restart their FP32 sums every kFarChunk sources (0: one sum per
// tile), moving the partial sums into the FP64 accumulators: the rounding of a
// sequential FP32 sum of n similar terms grows like n^1.5.
#ifndef FS_FAR_CHUNK
#define FS_FAR_CHUNK 0
#endif
constexpr int kFarChunk = FS_FAR_CHUNK;
static_assert(kFarChunk == 0 || (kFarChunk % 8 == 0 && 256 % kFarChunk == 0), "far chunk: a multiple of 8 dividing 256");
// FP64 source records for the band pairs: staged into shared memory with the
// FP32 ones (1), or read from global memory by the band and mixed tiles that
// need them (0).
#ifndef FS_STAGE64
#define FS_STAGE64 1
#endif
// band tiles: sources per unrolled body
#ifndef FS_BAND_UNROLL
#define FS_BAND_UNROLL 4
#endif
constexpr int kBandUnroll = FS_BAND_UNROLL;
// far tiles: sources per unrolled body
#ifndef FS_FAR_UNROLL
#define FS_FAR_UNROLL 8
#endif
constexpr int kFarUnroll = FS_FAR_UNROLL;
static_assert(kS % kFarUnroll == 0, "far unroll must divide the tile");
// one simulation's persistent launch: about this many items per CTA
#ifndef FS_ITEMS_PER_CTA
#define FS_ITEMS_PER_CTA 32
#endif
constexpr int kItemsPerCta = FS_ITEMS_PER_CTA;
// targets assigned contiguously per warp (1) or interleaved across the CTA (0)
#ifndef FS_WARP_CONTIG
#define FS_WARP_CONTIG 1
#endif
constexpr bool kWarpContig = FS_WARP_CONTIG;
constexpr int kTStride = kWarpContig ? 32 : kNT;
constexpr bool kStage64 = FS_STAGE64;

// Far pairs: q/2 * d*y = sign(d) * q/2 * (1 - c), c = 1 - sqrt(1 - v),
// v = eps^2 w, w = 1/(d^2 + eps^2), v <= 1/(1 + kBand^2).  The sign part is
// summed in FP64 (ffar); the pair kernel accumulates q/2 * c with the shifted
// form c = (v/2) / (1 - v/4) = a1 / (d^2 + 3 eps^2 / 4), a1 = eps^2/2, whose
// series v/2 + v^2/8 + v^3/32 + ... matches c = v/2 + v^2/8 + v^3/16 + ... to
// second order: the error is below v^2/16 <= 1e-6 of c at the band edge
// (2e-9 of the pair's q/2) and falls off as 1/d^6.  Far pairs need no square
// root, and two targets share one MUFU.RCP and one scalar product:
// q a1 / r_a = (q a1 / (r_a r_b)) r_b.
#ifndef FS_PAIR_BAND
#define FS_PAIR_BAND 16.0
#endif
constexpr double kBand = FS_PAIR_BAND;  // near band half-width in units of eps
constexpr int kMaxChunks = 64;

// One (target block, source chunk) of a job: kR targets per thread, the
// chunk's tiles moved into shared memory by TMA bulk copies on two mbarriers.
// `gk` counts the tiles this CTA has consumed (buffer = gk & 1, barrier phase
// = (gk >> 1) & 1), so the barriers keep alternating across work items.
// Returns false when a bounded wait gave up (flag set, CTA must stop).
template <int kR>
__device__ __forceinline__ bool pair_block(const PairJob& Jb, int tb, int chunk, float4 (*buf)[kS],
                                           double2 (*buf64)[kS], uint64_t* bar,
                                           uint32_t& gk, int* __restrict__ err) {
    constexpr int kTB = kNT * kR;
    const int tid = threadIdx.x;
    const int t0 = chunk * Jb.tpc;
    const int t1 = min(Jb.ntiles, t0 + Jb.tpc);
    if (t0 >= t1) return true;
    const float eps2 = Jb.eps2, a1 = Jb.a1, a2 = Jb.a2;
    const double L = Jb.L;
    const int ns = Jb.ns;
    // targets of this thread: ibase + r * kTStride.  Per warp (kTStride = 32)
    // a warp's 32 kR targets are contiguous in x, so fewer of its tiles mix
    // band and far pairs; per CTA (kTStride = kNT) they interleave with the
    // other warps'.
    const int ibase = kWarpContig ? tb * kTB + (tid >> 5) * (32 * kR) + (tid & 31) : tb * kTB + tid;
    double tl[kR], acc64[kR];
    int J[kR], U1[kR], U2[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
        const TargetInfo T = Jb.info[ibase + r * kTStride];  // nt_pad is a multiple of kTB
        tl[r] = T.tlo;
        J[r] = T.J;
        U1[r] = T.U1;
        U2[r] = T.U2;
        acc64[r] = 0.0;
    }
    // each tile: the FP32 records and the FP64 records of the same sources,
    // two bulk copies completing on one barrier
    constexpr uint32_t kBytes = kS * sizeof(float4);
    constexpr uint32_t kBytes64 = kStage64 ? kS * sizeof(double2) : 0;
    const long long polls = g_mbar_polls;
    if (tid == 0) {
        fence_proxy_async();
        mbar_expect_tx(&bar[gk & 1], kBytes + kBytes64);
        bulk_load(buf[gk & 1], Jb.src + (size_t)t0 * kS, kBytes, &bar[gk & 1]);
        if (kStage64) bulk_load(buf64[gk & 1], Jb.src64 + (size_t)t0 * kS, kBytes64, &bar[gk & 1]);
    }
    for (int t = t0; t < t1; ++t, ++gk) {
        const int b = gk & 1;
        if (tid == 0 && t + 1 < t1) {
            fence_proxy_async();
            mbar_expect_tx(&bar[b ^ 1], kBytes + kBytes64);
            bulk_load(buf[b ^ 1], Jb.src + (size_t)(t + 1) * kS, kBytes, &bar[b ^ 1]);
            if (kStage64) bulk_load(buf64[b ^ 1], Jb.src64 + (size_t)(t + 1) * kS, kBytes64, &bar[b ^ 1]);
        }
        const bool ok = mbar_wait_bounded(&bar[b], (gk >> 1) & 1, polls);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {
                atomicExch(err, (int)FS_ERR_TIMEOUT);
                // Both copies this CTA issued may still be in flight: the one
                // into buf[b] whose wait gave up, and the prefetch into
                // buf[b ^ 1].  Shared memory is released when the CTA exits,
                // so let both land first (bounded waits).
                (void)mbar_wait_bounded(&bar[b], (gk >> 1) & 1, kMbarPolls);
                if (t + 1 < t1) (void)mbar_wait_bounded(&bar[b ^ 1], ((gk + 1) >> 1) & 1, kMbarPolls);
            }
            return false;
        }
        const double base = Jb.tbase[t];
        const int jlo = t * kS;
        const int jend = min(jlo + kS, ns);  // real sources in this tile
        float tau[kR], tauh[kR], sg[kR], acc[kR];
        bool careful = false, inband = true;
#pragma unroll
        for (int r = 0; r < kR; ++r) {
            const double lo = tl[r] - base;
            tau[r] = (float)lo;
            tauh[r] = (float)(lo + L);
            float sgn = 0.f;
            bool band = false;
            if (jend <= J[r]) {          // whole tile on the lo image: u = j + n
                if (jend + ns <= U1[r]) sgn = 1.f;
                else if (jlo + ns >= U2[r]) sgn = -1.f;
                band = (jlo + ns >= U1[r]) && (jend + ns <= U2[r]);
            } else if (jlo >= J[r]) {    // whole tile on the hi image: u = j
                tau[r] = tauh[r];
                if (jend <= U1[r]) sgn = 1.f;
                else if (jlo >= U2[r]) sgn = -1.f;
                band = (jlo >= U1[r]) && (jend <= U2[r]);
            }
            sg[r] = sgn;
            acc[r] = 0.f;
            careful |= (sgn == 0.f);
            inband &= band;
        }
        const float4* tile = buf[b];
        if (__any_sync(0xffffffffu, careful) && __all_sync(0xffffffffu, inband)) {
            // band tiles (every pair of the warp within |d| <= band, one image
            // per target): q/2 * d / sqrt(d^2 + eps^2) in FP64 from the FP64
            // records.  Band terms are O(q/2) and cancel to the (possibly much
            // smaller) field; FP64 keeps their rounding below the field's size.
            const double2* tile64 = kStage64 ? buf64[b] : Jb.src64 + (size_t)jlo;
            const double e2d = Jb.eps2d;
            double T[kR];
#pragma unroll
            for (int r = 0; r < kR; ++r) T[r] = (jend <= J[r]) ? tl[r] : tl[r] + L;  // the tile's image
#pragma unroll(kBandUnroll)
            for (int j = 0; j < kS; ++j) {
                const double2 e = tile64[j];
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    const double d = T[r] - e.x;
                    acc64[r] = band_acc64(e.y, d, fma(d, d, e2d), acc64[r]);
                }
            }
        } else if (!__any_sync(0xffffffffu, careful)) {
            // far tiles: accumulate q/2 * c(v) = (q/2 a1) w', w' = 1/(d^2 + 3 eps^2/4),
            // two targets per packed FP32x2 op, one MUFU.RCP per two targets
            const float2 e2v = make_float2(Jb.e2f, Jb.e2f), m1 = make_float2(-1.f, -1.f);
            float2 tau2[kR / 2], acc2[kR / 2];
#pragma unroll
            for (int h = 0; h < kR / 2; ++h) {
                tau2[h] = make_float2(tau[2 * h], tau[2 * h + 1]);
                acc2[h] = make_float2(0.f, 0.f);
            }
            // Eight sources per unrolled body (unroll 4 measured 3.5% slower,
            // 16 no faster); per two targets one reciprocal and one scalar
            // product: q/2 a1 / r_a = (q/2 a1 W) r_b with W = 1/(r_a r_b), i.e.
            // 4 FP32 lane-ops and 0.5 MUFU.RCP per pair, which load the FMA pipe
            // and MUFU equally.  (One reciprocal per four targets -- 4.5
            // lane-ops and 0.25 MUFU per pair -- for 1/8 to 1/2 of the sources
            // measured 0.5-3.7% slower, and for 1, 2 or all 4 of a CTA's warps
            // 3-4% slower.  One or two of the four target pairs on the idle
            // FP64 pipe instead, with a reciprocal from an integer seed and
            // Newton steps, for every first, second or fourth source, measured
            // 8-33% slower: 6.5 issue slots per pair there against 3.  An
            // explicit software pipeline issuing each source's reciprocal one
            // source ahead of its accumulation measured 15% slower.)  The
            // FP32 sums are moved into the FP64 accumulators every kFarChunk
            // sources.
            constexpr int kChunk = kFarChunk ? kFarChunk : kS;
#pragma unroll 1
            for (int c = 0; c < kS; c += kChunk) {
#pragma unroll 1
                for (int j0 = c; j0 < c + kChunk; j0 += kFarUnroll) {
#pragma unroll
                    for (int k = 0; k < kFarUnroll; ++k) {
                        const float4 e = tile[j0 + k];
                        const float2 sx2 = make_float2(e.x, e.x);
#pragma unroll
                        for (int h = 0; h < kR / 2; ++h) {
                            const float2 d = __ffma2_rn(sx2, m1, tau2[h]);  // tau - s, exact product by -1
                            const float2 r2 = __ffma2_rn(d, d, e2v);
                            const float qW = e.z * rcp_approx(r2.x * r2.y);
                            acc2[h] = __ffma2_rn(r2, make_float2(qW, qW), acc2[h]);
                        }
                    }
                }
                // (qW r_a, qW r_b) are the terms of targets 2h+1 and 2h:
                // acc2[h].x holds target 2h+1 and .y target 2h
#pragma unroll
                for (int h = 0; h < kR / 2; ++h) {
                    acc64[2 * h] -= (double)sg[2 * h] * (double)acc2[h].y;
                    acc64[2 * h + 1] -= (double)sg[2 * h + 1] * (double)acc2[h].x;
                    acc2[h] = make_float2(0.f, 0.f);
                }
            }

        } else {
            // near band / image split: per-pair image and band; band pairs
            // q/2 * d / sqrt(d^2 + eps^2) in FP64 (as in band tiles), far pairs
            // -+ q/2 * c in FP32 with a Kahan sum
            const double2* tile64 = kStage64 ? buf64[b] : Jb.src64 + (size_t)jlo;
            const double e2d = Jb.eps2d;
            float cmp[kR];
#pragma unroll
            for (int r = 0; r < kR; ++r) cmp[r] = 0.f;
            for (int j = 0; j < kS; ++j) {
                const float4 e = tile[j];
                const int idx = jlo + j;
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    const bool lo_img = idx < J[r];
                    const int u = lo_img ? idx + ns : idx;
                    if (u >= U1[r] && u < U2[r]) {
                        const double2 e64 = tile64[j];
                        const double d = (lo_img ? tl[r] : tl[r] + L) - e64.x;
                        acc64[r] = band_acc64(e64.y, d, fma(d, d, e2d), acc64[r]);
                    } else {
                        const float d = (lo_img ? tau[r] : tauh[r]) - e.x;
                        const float y = rsqrt_approx(fmaf(d, d, eps2));
                        const float z = y * y;
                        const float c = z * fmaf(z, a2, a1);
                        const float val = (u < U1[r]) ? -c : c;
                        const float v = fmaf(e.y, val, -cmp[r]);
                        const float sum = acc[r] + v;
                        cmp[r] = (sum - acc[r]) - v;
                        acc[r] = sum;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < kR; ++r) acc64[r] += (double)acc[r] - (double)cmp[r];
        }
        __syncthreads();
    }
    double* out = Jb.partial + (size_t)chunk * Jb.nt_pad;
#pragma unroll
    for (int r = 0; r < kR; ++r) out[ibase + r * kTStride] = acc64[r];
    return true;
}

__device__ __forceinline__ void init_bars(uint64_t* bar) {
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// One job, grid (target blocks, source chunks).
template <int kR>
__global__ void __launch_bounds__(kNT) k_pairs32(PairJob job, int* __restrict__ err) {
    __shared__ __align__(128) float4 buf[2][kS];
    __shared__ __align__(128) double2 buf64[2][kS];
    __shared__ __align__(8) uint64_t bar[2];
    if ((int)blockIdx.y * job.tpc >= job.ntiles) return;
    init_bars(bar);
    uint32_t gk = 0;
    (void)pair_block<kR>(job, blockIdx.x, blockIdx.y, buf, buf64, bar, gk, err);
}

// Many jobs (one per simulation of a batch), persistent: a fixed grid of CTAs
// takes (job, target block, chunk) items from an atomic counter, in the order
// `order` gives (band-heavy items spread over the queue) or the host's order
// (longest first) when it is null.
// CTAs per SM (in 64-thread units) the batched kernel is compiled for: 16 at
// 4 targets per thread (64 registers; measured 4% faster than 12 CTAs at 80
// registers on the 64-instance batch), 8 at 8 targets (128 registers, no spills)
#ifndef FS_BATCH_MIN_BLOCKS4
#define FS_BATCH_MIN_BLOCKS4 16
#endif
template <int kR>
__global__ void __launch_bounds__(kNT, (kR >= 8 ? 8 : FS_BATCH_MIN_BLOCKS4) * 64 / kNT) k_pairs32_batched(const PairJob* __restrict__ jobs, const int4* __restrict__ items,
                                                         int nitems, const int* __restrict__ order,
                                                         int* __restrict__ counter, int* __restrict__ err) {
    __shared__ __align__(128) float4 buf[2][kS];
    __shared__ __align__(128) double2 buf64[2][kS];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_item;
    init_bars(bar);
    uint32_t gk = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(counter, 1);
            s_item = (order && k < nitems) ? order[k] : k;
        }
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= nitems) break;
        const int4 it = items[item];
        const PairJob job = jobs[it.x];
        if (!pair_block<kR>(job, it.y, it.z, buf, buf64, bar, gk, err)) return;
    }
}

// CTAs per SM (counted in 128-thread units) the 8-targets-per-thread
// persistent kernel is compiled for: 3 (up to 168 registers per thread, 12
// warps per SM) measured 0.9% faster than 4 (128 registers, 16 warps)
#ifndef FS_MIN_BLOCKS8
#define FS_MIN_BLOCKS8 3
#endif
constexpr int kMinBlocks8 = FS_MIN_BLOCKS8;

// One job, persistent: a grid of one wave of CTAs takes (chunk, target block)
// items from an atomic counter, in the order `order` gives (band-heavy items
// spread over the queue, light ones last) or in chunk-major order when it is
// null.
template <int kR>
__global__ void __launch_bounds__(kNT, (kR >= 8 ? kMinBlocks8 : 8) * 128 / kNT) k_pairs32_persistent(PairJob job, int tblocks, int nitems,
                                                            const int* __restrict__ order,
                                                            int* __restrict__ counter, int* __restrict__ err) {
    __shared__ __align__(128) float4 buf[2][kS];
    __shared__ __align__(128) double2 buf64[2][kS];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_item;
    init_bars(bar);
    uint32_t gk = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(counter, 1);
            s_item = (order && k < nitems) ? order[k] : k;
        }
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= nitems) break;
        if (!pair_block<kR>(job, item % tblocks, item / tblocks, buf, buf64, bar, gk, err)) return;
    }
}

// Estimated cost of a (target block, source chunk) item: its tiles, plus
// kNearTileCost - 1 more for every tile within the band of the block's
// x-range (band and mixed tiles run the FP64 / per-pair paths, several times a
// far tile's time).  Items with such tiles ("heavy") are spread evenly over
// the launch's queue, heaviest first, with light items in the gaps and alone
// in the last two waves: the launch does not end on a heavy item, and heavy
// items' FP64 work runs beside other items' FP32 work on the same SMs rather
// than all at once.  Only the order of the items depends on this; every item
// writes its own partial sums.
constexpr int kNearTileCost = 4;
#ifndef FS_ITEM_ORDER
#define FS_ITEM_ORDER 1
#endif
constexpr bool kItemOrder = FS_ITEM_ORDER;
#ifndef FS_ITEM_SPREAD
#define FS_ITEM_SPREAD 1
#endif
constexpr bool kItemSpread = FS_ITEM_SPREAD;
constexpr int kCostBits = 24;           // sort keys: cost < 2^23, plus the heavy bit
constexpr int kHeavy = 1 << 23;

__device__ __forceinline__ double target_x(const TargetInfo& T, double L) { return T.tlo < 0.0 ? T.tlo + L : T.tlo; }

// Sort key of an item: its estimated cost, with kHeavy set when it has tiles
// within the band; counts heavy items into *nheavy.
__device__ int item_key(const PairJob& J, int tb, int c, int ttb, int* __restrict__ nheavy) {
    const int t0 = c * J.tpc, t1 = min(J.ntiles, t0 + J.tpc);
    if (t0 >= t1 || J.nt <= 0) return 0;
    // the block's real targets, sorted by x: the first and the last bound it
    const int first = min(tb * ttb, J.nt - 1), last = min(tb * ttb + ttb, J.nt) - 1;
    const double xa = target_x(J.info[first], J.L), xb = target_x(J.info[last], J.L);
    const double band = kBand * sqrt(J.eps2d);
    int near = 0;
    for (int t = t0; t < t1; ++t) {
        const double ya = J.tbase[t];
        const double yb = (t + 1 < J.ntiles) ? J.tbase[t + 1] : J.L;
        double gap = 1e300;
        for (int k = -1; k <= 1; ++k) {
            const double sh = k * J.L;
            gap = fmin(gap, fmax(0.0, fmax(ya + sh - xb, xa - (yb + sh))));
        }
        near += (gap <= band);
    }
    const int cost = min((t1 - t0) + (kNearTileCost - 1) * near, kHeavy - 1);
    if (near == 0) return cost;
    atomicAdd(nheavy, 1);
    return cost | kHeavy;
}

// item i = chunk * tblocks + target block, as k_pairs32_persistent reads it
__global__ void k_item_cost(PairJob J, int nitems, int tblocks, int ttb, int* __restrict__ key,
                            int* __restrict__ ids, int* __restrict__ nheavy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    key[i] = item_key(J, i % tblocks, i / tblocks, ttb, nheavy);
    ids[i] = i;
}

__global__ void k_item_cost_batched(const PairJob* __restrict__ jobs, const int4* __restrict__ items, int nitems,
                                    int ttb, int* __restrict__ key, int* __restrict__ ids,
                                    int* __restrict__ nheavy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const int4 it = items[i];
    key[i] = item_key(jobs[it.x], it.y, it.z, ttb, nheavy);
    ids[i] = i;
}

// From the n items sorted by key (the H heavy ones first): heavy item j at
// position floor(j span / H), span = n - guard, light items in the remaining
// positions in their sorted order.  The heavy positions below p number
// min(H, ceil(p H / span)).  With span < H there is nothing to spread: the
// sorted order stands.
__global__ void k_item_spread(const int* __restrict__ sorted, int n, const int* __restrict__ nheavy, int guard,
                              int* __restrict__ out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const long long H = *nheavy, span = n - guard;
    if (H == 0 || span < H || !kItemSpread) {
        out[p] = sorted[p];
        return;
    }
    const long long below = min(H, (p * H + span - 1) / span);
    const long long upto = min(H, ((p + 1) * H + span - 1) / span);
    out[p] = (upto > below) ? sorted[below] : sorted[H + (p - below)];
}

// Bytes of CUB scratch for ordering n items.
size_t item_order_tmp_bytes(int n) {
    size_t b = 0;
    FS_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, b, (const int*)nullptr, (int*)nullptr,
                                                      (const int*)nullptr, (int*)nullptr, n, 0, kCostBits));
    return std::max<size_t>(b, 1);
}

// key holds 2 n + 1 ints (the heavy count last, already set), ids 3 n: the
// sorted ids go to ids + n and the final order to ids + 2 n, which is returned.
const int* order_items(int n, int* key, int* ids, int guard, void* tmp, size_t tmp_bytes, cudaStream_t st) {
    FS_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, key, key + n, ids, ids + n, n, 0, kCostBits,
                                                      st));
    const int T = 256;
    k_item_spread<<<(n + T - 1) / T, T, 0, st>>>(ids + n, n, key + 2 * n, guard, ids + 2 * n);
    FS_LAUNCHED(1);
    return ids + 2 * n;
}

// Targets per thread of the pair kernel: 2, 4 or 8 (register use vs. reuse of
// each shared-memory source record).
void launch_pairs(int R, dim3 grid, cudaStream_t st, const PairJob& job, int* err) {
    switch (R) {
        case 2: k_pairs32<2><<<grid, kNT, 0, st>>>(job, err); break;
        case 8: k_pairs32<8><<<grid, kNT, 0, st>>>(job, err); break;
        default: k_pairs32<4><<<grid, kNT, 0, st>>>(job, err); break;
    }
}

int persistent_grid(int R) {
    int per_sm = 0;
    switch (R) {
        case 2: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_persistent<2>, kNT, 0)); break;
        case 8: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_persistent<8>, kNT, 0)); break;
        default: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_persistent<4>, kNT, 0)); break;
    }
    return std::max(1, per_sm) * sm_count();
}

void launch_pairs_persistent(int R, int grid, cudaStream_t st, const PairJob& job, int tblocks, int nitems,
                             const int* order, int* counter, int* err) {
    FS_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    switch (R) {
        case 2: k_pairs32_persistent<2><<<grid, kNT, 0, st>>>(job, tblocks, nitems, order, counter, err); break;
        case 8: k_pairs32_persistent<8><<<grid, kNT, 0, st>>>(job, tblocks, nitems, order, counter, err); break;
        default: k_pairs32_persistent<4><<<grid, kNT, 0, st>>>(job, tblocks, nitems, order, counter, err); break;
    }
}

}  // namespace

void launch_pairs_batched(int R, int grid, cudaStream_t st, const PairJob* jobs, const int4* items, int nitems,
                          ItemOrder* ord, int* counter, int* err) {
    const int* order = nullptr;
    if (kItemOrder && ord && nitems > grid) {
        const int T = 256;
        FS_CUDA(cudaMemsetAsync(ord->cost.p + 2 * (size_t)nitems, 0, sizeof(int), st));
        k_item_cost_batched<<<(nitems + T - 1) / T, T, 0, st>>>(jobs, items, nitems, kNT * R, ord->cost.p,
                                                                ord->ids.p, ord->cost.p + 2 * (size_t)nitems);
        FS_LAUNCHED(1);
        order = order_items(nitems, ord->cost.p, ord->ids.p, 2 * grid, ord->tmp.p, ord->tmp.n, st);
    }
    FS_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    switch (R) {
        case 2: k_pairs32_batched<2><<<grid, kNT, 0, st>>>(jobs, items, nitems, order, counter, err); break;
        case 8: k_pairs32_batched<8><<<grid, kNT, 0, st>>>(jobs, items, nitems, order, counter, err); break;
        default: k_pairs32_batched<4><<<grid, kNT, 0, st>>>(jobs, items, nitems, order, counter, err); break;
    }
    FS_LAUNCHED(1);
}

void ItemOrder::reserve(int nitems) {
    cost.ensure(2 * (size_t)std::max(nitems, 1) + 1);
    ids.ensure(3 * (size_t)std::max(nitems, 1));
    tmp.ensure(item_order_tmp_bytes(std::max(nitems, 1)));
}

void pair_job_items(const PairJob& job, int job_index, int R, std::vector<int4>& items, std::vector<double>& cost) {
    const int tblocks = job.nt_pad / (kNT * R);
    const int nchunks = (job.ntiles + job.tpc - 1) / job.tpc;
    for (int c = 0; c < nchunks; ++c) {
        const int tiles = std::min(job.tpc, job.ntiles - c * job.tpc);
        for (int b = 0; b < tblocks; ++b) {
            items.push_back(make_int4(job_index, b, c, 0));
            cost.push_back((double)tiles * kNT * R);
        }
    }
}

int pairs_batched_grid(int R) {
    int per_sm = 0;
    switch (R) {
        case 2: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_batched<2>, kNT, 0)); break;
        case 8: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_batched<8>, kNT, 0)); break;
        default: FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs32_batched<4>, kNT, 0)); break;
    }
    return std::max(1, per_sm) * sm_count();
}

namespace {

// Sum the chunk partials in a fixed order, add the exact far-band sign sum,
// subtract the FP64 background and apply the stage epilogue at the target's
// original index.
__global__ void k_finalize32(const double* __restrict__ partial, int nchunks, int nt_pad, int nt,
                             const TargetInfo* __restrict__ info, const double* __restrict__ pq,
                             const double* __restrict__ qxsum, int ns, double L, double cbg,
                             const int* __restrict__ tperm, Stage S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    double E = 0.0;
    for (int c = 0; c < nchunks; ++c) E += partial[(size_t)c * nt_pad + i];
    if (ns > 0) {
        const TargetInfo T = info[i];
        const double Q = pq[ns - 1];
        const double PJ = (T.J > 0) ? pq[T.J - 1] : 0.0;
        const double B = T.tlo * Q - qxsum[0] + L * (Q - PJ);
        E += T.ffar;
        E -= cbg * B;
    }
    apply_stage(S, tperm[i], E);
}

// Band pairs of an evaluation (sum over targets of U2 - U1), for the
// profile's roofline: they run on the FP64 pipe, the far pairs on FP32/MUFU.
__global__ void k_band_count(int nt, const TargetInfo* __restrict__ info, double* __restrict__ out) {
    __shared__ double sh[256];
    double c = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x)
        c += (double)(info[i].U2 - info[i].U1);
    sh[threadIdx.x] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, sh[0]);
}

class Direct32c final : public FieldEngine {
   public:
    Direct32c(double L, double eps) : L_(L), eps_(eps) {
        cbg_ = 1 / std::sqrt(L * L + 4 * eps * eps);
        // tuning knob: targets per thread of the pair kernel (2, 4 or 8)
        if (const char* v = std::getenv("FS_B200_PAIR_TARGETS")) {
            const int r = std::atoi(v);
            if (r == 2 || r == 4 || r == 8) R_ = r;
        }
    }


    void eval(const double* d_t, int nt, const double* d_s, const double* d_q, int ns, const Stage& stage,
              cudaStream_t st) override {
        // a standalone launch: one persistent wave over about 32 items per CTA
        const int ntiles = (ns + kS - 1) / kS;
        const int nt_pad = (nt + kTBPad - 1) / kTBPad * kTBPad;
        const int tblocks = nt_pad / (kNT * R_);
        if (!grid_) grid_ = persistent_grid(R_);
        const int want = grid_ * kItemsPerCta;
        int nchunks = ntiles ? std::min(ntiles, std::max(1, (want + tblocks - 1) / tblocks)) : 1;
        const int tpc = ntiles ? (ntiles + nchunks - 1) / nchunks : 1;
        PairJob job;
        if (prepare(d_t, nt, d_s, d_q, ns, stage, st, tpc, &job)) {
            nchunks = (job.ntiles + job.tpc - 1) / job.tpc;
            const int nitems = tblocks * nchunks;
            const int* order = kItemOrder && nitems > grid_ ? item_order(nitems, tblocks, job, st) : nullptr;
            ProfScope prof("k_pairs32", st, last_pairs);
            launch_pairs_persistent(R_, std::min(grid_, nitems), st, job, tblocks, nitems, order, counter_.p,
                                    err_.p);
            FS_LAUNCHED(1);
        }
        finalize(st);
    }

    bool prepare(const double* d_t, int nt, const double* d_s, const double* d_q, int ns, const Stage& stage,
                 cudaStream_t st, int tpc, PairJob* job) override {
        last_pairs = (double)nt * (double)ns;
        last_nt_ = 0;
        fin_ = Fin{};
        if (nt <= 0) return false;
        const bool same = (d_t == d_s) && (nt == ns);
        const int ntiles = (ns + kS - 1) / kS;
        const int ns_pad = ntiles * kS;
        const int nt_pad = (nt + kTBPad - 1) / kTBPad * kTBPad;
        // at most kMaxChunks source chunks: bounds the partial sums to
        // 8 * kMaxChunks bytes per target whatever the item shape
        tpc = std::max(std::max(1, tpc), (ntiles + kMaxChunks - 1) / kMaxChunks);
        const int nchunks = ntiles ? (ntiles + tpc - 1) / tpc : 1;
        reserve(std::max(ns, 1), ns_pad, same ? 0 : nt, nt_pad, (size_t)nchunks * nt_pad, ntiles);
        const int T = 256;
        const double e2 = eps_ * eps_;
        if (ns > 0) {
            k_wrap_keys<<<(ns + T - 1) / T, T, 0, st>>>(d_s, ns, L_, kin_.p, iin_.p);
            size_t tb = cub_.bytes();
            FS_CUDA(cub::DeviceRadixSort::SortPairs(cub_.p, tb, kin_.p, kout_.p, iin_.p, iout_.p, ns, 0, 63, st));
            k_gather_sources<<<(ns_pad + T - 1) / T, T, 0, st>>>(kout_.p, iout_.p, d_q, ns, ns_pad, e2 / 2,
                                                                 e2 * e2 / 8, src_.p, src64_.p, tbase_.p, qs_.p,
                                                                 qx_.p);
            scan_f64_inclusive(qs_.p, pq_.p, ns, scan_.p, st);
            sum_f64(qx_.p, ns, scan_.p, qxsum_.p, st);
            FS_LAUNCHED(2);  // k_wrap_keys, k_gather_sources (the sort is CUB's; the scan and sum count themselves)
        }
        const uint64_t* tkeys;
        const int* tperm;
        if (same) {
            tkeys = kout_.p;
            tperm = iout_.p;
        } else {
            k_wrap_keys<<<(nt + T - 1) / T, T, 0, st>>>(d_t, nt, L_, tkin_.p, tiin_.p);
            size_t tb = cub_.bytes();
            FS_CUDA(cub::DeviceRadixSort::SortPairs(cub_.p, tb, tkin_.p, tkout_.p, tiin_.p, tiout_.p, nt, 0, 63, st));
            tkeys = tkout_.p;
            tperm = tiout_.p;
            FS_LAUNCHED(1);
        }
        fin_ = Fin{true, nt, ns, nt_pad, ns > 0 ? nchunks : 1, tperm, stage};
        if (ns <= 0) {
            FS_CUDA(cudaMemsetAsync(partial_.p, 0, sizeof(double) * nt_pad, st));
            return false;
        }
        k_target_info<<<(nt_pad + T - 1) / T, T, 0, st>>>(tkeys, nt, nt_pad, kout_.p, ns, L_, kBand * eps_, pq_.p,
                                                         info_.p);
        FS_LAUNCHED(1);
        last_nt_ = nt;
        *job = PairJob{src_.p, src64_.p, tbase_.p, info_.p, partial_.p, ns, ntiles, tpc, nt_pad, L_, (float)e2,
                       (float)(e2 / 2), (float)(e2 * e2 / 8), (float)(0.75 * e2), e2, nt};
        return true;
    }

    void finalize(cudaStream_t st) override {
        if (!fin_.pending) return;
        const int T = 256;
        k_finalize32<<<(fin_.nt + T - 1) / T, T, 0, st>>>(partial_.p, fin_.nchunks, fin_.nt_pad, fin_.nt, info_.p,
                                                           pq_.p, qxsum_.p, fin_.ns, L_, cbg_, fin_.tperm, fin_.stage);
        FS_LAUNCHED(1);
        fin_.pending = false;
    }

    int* error_flag() override { return err_.p; }

    // Pairs of the last evaluation (each evaluated); while profiling, also the
    // band pairs among them, recorded as "pairs32_band_pairs".
    double actual_work(cudaStream_t st) override {
        if (last_pairs > 0 && last_nt_ > 0) prof_add_work("pairs32_band_pairs", band_pairs(st));
        return last_pairs;
    }

    double band_pairs(cudaStream_t st) override {
        if (last_pairs <= 0 || last_nt_ <= 0) return 0.0;
        FS_CUDA(cudaMemsetAsync(bandcount_.p, 0, sizeof(double), st));
        k_band_count<<<148, 256, 0, st>>>(last_nt_, info_.p, bandcount_.p);
        FS_LAUNCHED(1);
        double h = 0.0;
        FS_CUDA(cudaMemcpyAsync(&h, bandcount_.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        FS_CUDA(cudaStreamSynchronize(st));
        return h;
    }

   private:
    // The persistent launch's items in the order of order_items (heavy items
    // spread over the queue, light ones last).
    const int* item_order(int nitems, int tblocks, const PairJob& job, cudaStream_t st) {
        cost_.ensure(2 * (size_t)nitems + 1);
        ids_.ensure(3 * (size_t)nitems);
        const size_t tb = item_order_tmp_bytes(nitems);
        ordtmp_.ensure(tb);
        const int T = 256;
        FS_CUDA(cudaMemsetAsync(cost_.p + 2 * (size_t)nitems, 0, sizeof(int), st));
        k_item_cost<<<(nitems + T - 1) / T, T, 0, st>>>(job, nitems, tblocks, job.nt_pad / tblocks, cost_.p, ids_.p,
                                                        cost_.p + 2 * (size_t)nitems);
        FS_LAUNCHED(1);
        return order_items(nitems, cost_.p, ids_.p, 2 * std::min(grid_, nitems), ordtmp_.p, tb, st);
    }

    void reserve(int ns, int ns_pad, int nt_sep, int nt_pad, size_t npartial, int ntiles) {
        kin_.ensure(ns);
        kout_.ensure(ns);
        iin_.ensure(ns);
        iout_.ensure(ns);
        src_.ensure(ns_pad);
        src64_.ensure(ns_pad);
        qs_.ensure(ns);
        qx_.ensure(ns);
        pq_.ensure(ns);
        qxsum_.ensure(1);
        scan_.ensure(scan_f64_scratch(ns));
        tbase_.ensure(std::max(ntiles, 1));
        info_.ensure(nt_pad);
        partial_.ensure(npartial);
        if (!err_.p) {
            err_.ensure(1);
            FS_CUDA(cudaMemset(err_.p, 0, sizeof(int)));
            counter_.ensure(1);
            bandcount_.ensure(1);
        }
        const int nsort = std::max(ns, nt_sep);
        if (nt_sep) {
            tkin_.ensure(nt_sep);
            tkout_.ensure(nt_sep);
            tiin_.ensure(nt_sep);
            tiout_.ensure(nt_sep);
        }
        size_t need = 0, b = 0;
        FS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, (int*)nullptr,
                                                (int*)nullptr, nsort, 0, 63));
        need = std::max(need, b);
        cub_.ensure(need);
    }

    struct Fin {
        bool pending = false;
        int nt = 0, ns = 0, nt_pad = 0, nchunks = 1;
        const int* tperm = nullptr;
        Stage stage;
    };
    double L_, eps_, cbg_;
    int R_ = 8;
    int grid_ = 0;
    Fin fin_;
    DevBuf<uint64_t> kin_, kout_, tkin_, tkout_;
    DevBuf<int> iin_, iout_, tiin_, tiout_;
    DevBuf<float4> src_;
    DevBuf<double2> src64_;
    DevBuf<double> bandcount_;
    int last_nt_ = 0;
    DevBuf<int> cost_, ids_;
    DevBuf<unsigned char> ordtmp_;
    DevBuf<double> qs_, qx_, pq_, qxsum_, tbase_, partial_, scan_;
    DevBuf<TargetInfo> info_;
    DevBuf<int> err_, counter_;
    DevBuf<unsigned char> cub_;
};

}  // namespace

FieldEngine* make_direct32c(double L, double eps) { return new Direct32c(L, eps); }

// ---------------------------------------------------------------------------
// Allocation-free variant of the FP32-compensated self-field.
//
// Some callers cannot allocate device memory when they need the field: code
// running inside a memory pool or arena that owns the whole device, embedded
// or real-time hosts whose allocation happens once at start-up, and hosts that
// forbid cudaMalloc/cudaFree on their calling thread because those calls
// synchronise the device.  This variant keeps all of its scratch (sort keys,
// tile records, prefix sums, per-target bands, chunk partials, the sort's
// temporary storage, the timeout flag) in one file-scope device array, so a
// call allocates nothing.  The array's size is fixed (kNoAllocBytes, about
// 9 MiB) and every GPU that loads this library holds it until the process
// exits; it bounds the problem size to kNoAllocMaxPoints points.
//
// The array is shared by every call on a device and keeps the previous call's
// contents: everything a call reads is written by that call first, and the
// timeout flag is cleared at the start of each call.  Calls whose work overlaps
// on the same GPU (different streams or threads) race on the array; serialise
// them.
void set_mbar_polls(long long polls) {
    const long long v = polls < 0 ? kMbarPolls : polls;
    FS_CUDA(cudaMemcpyToSymbol(g_mbar_polls, &v, sizeof(v)));
}

constexpr int kNoAllocMaxPoints = 32768;
constexpr int kNoAllocMaxChunks = 16;
constexpr size_t kNoAllocCubBytes = size_t(2) << 20;

namespace {

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct NoAllocLayout {
    size_t kin, kout, iin, iout, src, src64, tbase, qs, qx, pq, qxsum, info, partial, err, cub, total;
};

constexpr NoAllocLayout noalloc_layout() {
    NoAllocLayout L{};
    size_t o = 0;
    const size_t n = kNoAllocMaxPoints;
    L.kin = o;     o += align256(n * sizeof(uint64_t));
    L.kout = o;    o += align256(n * sizeof(uint64_t));
    L.iin = o;     o += align256(n * sizeof(int));
    L.iout = o;    o += align256(n * sizeof(int));
    L.src = o;     o += align256(n * sizeof(float4));
    L.src64 = o;   o += align256(n * sizeof(double2));
    L.tbase = o;   o += align256((n / kS) * sizeof(double));
    L.qs = o;      o += align256(n * sizeof(double));
    L.qx = o;      o += align256(n * sizeof(double));
    L.pq = o;      o += align256(n * sizeof(double));
    L.qxsum = o;   o += align256(sizeof(double));
    L.info = o;    o += align256(n * sizeof(TargetInfo));
    L.partial = o; o += align256((size_t)kNoAllocMaxChunks * n * sizeof(double));
    L.err = o;     o += align256(sizeof(int));
    L.cub = o;     o += kNoAllocCubBytes;
    L.total = o;
    return L;
}

constexpr NoAllocLayout kNoAlloc = noalloc_layout();
constexpr size_t kNoAllocBytes = kNoAlloc.total;
static_assert(kNoAllocMaxPoints % kTBPad == 0 && kNoAllocMaxPoints % kS == 0, "max size must fill whole blocks");

// The scratch itself.  Host code must not use this symbol as an address: it
// gets the device address from cudaGetSymbolAddress (noalloc_scratch()).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this; cudaGetSymbolAddress does
// not allocate).
unsigned char* noalloc_scratch() {
    int dev = 0;
    FS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(FS_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            (void)cudaGetLastError();
            fail(FS_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                                  cudaGetErrorString(e));
        }
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

void direct32c_noalloc(double L, double eps, double* d_es, const double* d_x, const double* d_q, int n,
                       cudaStream_t st) {
    if (!(L > 0) || !(eps > 0)) fail(FS_ERR_ARG, "L and epsilon must be positive");
    if (n < 0) fail(FS_ERR_ARG, "n must be >= 0");
    if (n > kNoAllocMaxPoints)
        fail(FS_ERR_ARG, "fs_field_eval_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                             std::to_string(kNoAllocMaxPoints) + " points");
    if (n == 0) return;
    if (!d_es || !d_x || !d_q) fail(FS_ERR_ARG, "null device pointer");
    unsigned char* base = noalloc_scratch();
    auto at = [&](size_t off) { return base + off; };
    uint64_t* kin = reinterpret_cast<uint64_t*>(at(kNoAlloc.kin));
    uint64_t* kout = reinterpret_cast<uint64_t*>(at(kNoAlloc.kout));
    int* iin = reinterpret_cast<int*>(at(kNoAlloc.iin));
    int* iout = reinterpret_cast<int*>(at(kNoAlloc.iout));
    float4* src = reinterpret_cast<float4*>(at(kNoAlloc.src));
    double2* src64 = reinterpret_cast<double2*>(at(kNoAlloc.src64));
    double* tbase = reinterpret_cast<double*>(at(kNoAlloc.tbase));
    double* qs = reinterpret_cast<double*>(at(kNoAlloc.qs));
    double* qx = reinterpret_cast<double*>(at(kNoAlloc.qx));
    double* pq = reinterpret_cast<double*>(at(kNoAlloc.pq));
    double* qxsum = reinterpret_cast<double*>(at(kNoAlloc.qxsum));
    TargetInfo* info = reinterpret_cast<TargetInfo*>(at(kNoAlloc.info));
    double* partial = reinterpret_cast<double*>(at(kNoAlloc.partial));
    int* err = reinterpret_cast<int*>(at(kNoAlloc.err));
    void* cub_tmp = at(kNoAlloc.cub);

    const int ntiles = (n + kS - 1) / kS;
    const int ns_pad = ntiles * kS;
    constexpr int R = 4;
    const int nt_pad = (n + kTBPad - 1) / kTBPad * kTBPad;
    const int tblocks = nt_pad / (kNT * R);
    const int want = sm_count() * 8 * 4;
    int nchunks = std::min(std::min(ntiles, kNoAllocMaxChunks), std::max(1, (want + tblocks - 1) / tblocks));
    const int tpc = (ntiles + nchunks - 1) / nchunks;
    nchunks = (ntiles + tpc - 1) / tpc;
    size_t need = 0, b = 0;
    FS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, kin, kout, iin, iout, n, 0, 63));
    need = std::max(need, b);
    need = std::max(need, scan_f64_scratch(n) * sizeof(double));
    if (need > kNoAllocCubBytes) fail(FS_ERR_UNSUPPORTED, "sort scratch larger than the static reserve");

    FS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    const int T = 256;
    k_wrap_keys<<<(n + T - 1) / T, T, 0, st>>>(d_x, n, L, kin, iin);
    size_t tb = kNoAllocCubBytes;
    FS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, tb, kin, kout, iin, iout, n, 0, 63, st));
    const double e2 = eps * eps;
    k_gather_sources<<<(ns_pad + T - 1) / T, T, 0, st>>>(kout, iout, d_q, n, ns_pad, e2 / 2, e2 * e2 / 8, src, src64,
                                                         tbase, qs, qx);
    scan_f64_inclusive(qs, pq, n, reinterpret_cast<double*>(cub_tmp), st);  // the sort is done with cub_tmp
    sum_f64(qx, n, reinterpret_cast<double*>(cub_tmp), qxsum, st);
    k_target_info<<<(nt_pad + T - 1) / T, T, 0, st>>>(kout, n, nt_pad, kout, n, L, kBand * eps, pq, info);
    const PairJob job{src, src64, tbase, info, partial, n, ntiles, tpc, nt_pad, L, (float)e2, (float)(e2 / 2),
                      (float)(e2 * e2 / 8), (float)(0.75 * e2), e2, n};
    launch_pairs(R, dim3(tblocks, nchunks), st, job, err);
    Stage S;
    S.kind = STAGE_STORE;
    S.out = d_es;
    const double cbg = 1 / std::sqrt(L * L + 4 * eps * eps);
    k_finalize32<<<(n + T - 1) / T, T, 0, st>>>(partial, nchunks, nt_pad, n, info, pq, qxsum, n, L, cbg, iout, S);
    FS_LAUNCHED(6);
    int h = 0;
    FS_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    FS_CUDA(cudaStreamSynchronize(st));
    if (h) fail((fs_status)h, "device wait timed out in the field kernel");
}

}  // namespace fsb

extern "C" fs_status fs_field_eval_noalloc(double L, double epsilon, double* d_es, const double* d_x,
                                           const double* d_q_ws, int n, void* stream) {
    return fsb::guard([&] { fsb::direct32c_noalloc(L, epsilon, d_es, d_x, d_q_ws, n, (cudaStream_t)stream); });
}
