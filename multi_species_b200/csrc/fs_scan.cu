// Deterministic inclusive prefix sum and sum of doubles (sm_100a).
//
// The field kernels form exact-in-FP64 sign sums and background terms from
// prefix sums of the sorted charges.  A single-pass scan with decoupled
// look-back groups its additions by which predecessor tiles happen to have
// finished, so its floating-point results can differ from run to run.  This
// scan fixes every association: each block of kScanT threads owns a segment
// of kScanT * kScanPer elements, each thread a run of kScanPer; runs are summed
// left to right, threads combined by a Kogge-Stone scan inside each warp and
// across the warps, blocks by one block scanning the block totals the same way.
// Three launches: block totals, their scan, and the final pass that rescans
// each block from its offset.  sum_f64 is the same first pass and one CTA
// summing the block totals.
#include "fs_device.cuh"

namespace fsb {

namespace {

constexpr int kScanT = 256;
constexpr int kScanPer = 8;
constexpr int kScanSeg = kScanT * kScanPer;
constexpr int kScanWarps = kScanT / 32;

// Exclusive scan of one value per thread over a CTA of kScanT threads, in a
// fixed association; returns the exclusive prefix and sets *total.
__device__ __forceinline__ double block_scan_excl(double v, double* sh, double* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        double w = lane < kScanWarps ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        if (lane < kScanWarps) sh[kScanWarps + lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const double before = warp ? sh[kScanWarps + warp - 1] : 0.0;
    *total = sh[2 * kScanWarps - 1];
    __syncthreads();  // sh is reused by the caller's next scan
    double ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) ex = 0.0;
    return before + ex;
}

__device__ __forceinline__ double run_sum(const double* __restrict__ in, int n, int a) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) s += (a + k < n) ? in[a + k] : 0.0;
    return s;
}

__global__ void __launch_bounds__(kScanT) k_scan_totals(const double* __restrict__ in, int n,
                                                         double* __restrict__ bsum) {
    __shared__ double sh[2 * kScanWarps];
    const int a = blockIdx.x * kScanSeg + threadIdx.x * kScanPer;
    double total;
    (void)block_scan_excl(run_sum(in, n, a), sh, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// One CTA: bsum[0..nb) -> exclusive prefixes, in place.
__global__ void __launch_bounds__(kScanT) k_scan_offsets(double* __restrict__ bsum, int nb) {
    __shared__ double sh[2 * kScanWarps];
    const int per = (nb + kScanT - 1) / kScanT;
    const int a = threadIdx.x * per, e = min(nb, a + per);
    double s = 0.0;
    for (int i = a; i < e; ++i) s += bsum[i];
    double total;
    double run = block_scan_excl(s, sh, &total);
    for (int i = a; i < e; ++i) {
        const double v = bsum[i];
        bsum[i] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kScanT) k_scan_final(const double* __restrict__ in, int n,
                                                        const double* __restrict__ boff, double* __restrict__ out) {
    __shared__ double sh[2 * kScanWarps];
    const int a = blockIdx.x * kScanSeg + threadIdx.x * kScanPer;
    double total;
    double run = boff[blockIdx.x] + block_scan_excl(run_sum(in, n, a), sh, &total);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (a + k < n) {
            run += in[a + k];
            out[a + k] = run;
        }
    }
}

// One CTA: out[0] = the sum of bsum[0..nb), in a fixed association.
__global__ void __launch_bounds__(kScanT) k_sum_totals(const double* __restrict__ bsum, int nb,
                                                        double* __restrict__ out) {
    __shared__ double sh[2 * kScanWarps];
    const int per = (nb + kScanT - 1) / kScanT;
    const int a = threadIdx.x * per, e = min(nb, a + per);
    double s = 0.0;
    for (int i = a; i < e; ++i) s += bsum[i];
    double total;
    (void)block_scan_excl(s, sh, &total);
    if (threadIdx.x == 0) out[0] = total;
}

}  // namespace

void sum_f64(const double* in, int n, double* scratch, double* out, cudaStream_t st) {
    if (n <= 0) {
        FS_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
        return;
    }
    const int nb = (n + kScanSeg - 1) / kScanSeg;
    k_scan_totals<<<nb, kScanT, 0, st>>>(in, n, scratch);
    k_sum_totals<<<1, kScanT, 0, st>>>(scratch, nb, out);
    FS_LAUNCHED(2);
}

size_t scan_f64_scratch(int n) { return (size_t)std::max(1, (n + kScanSeg - 1) / kScanSeg); }

void scan_f64_inclusive(const double* in, double* out, int n, double* scratch, cudaStream_t st) {
    if (n <= 0) return;
    const int nb = (n + kScanSeg - 1) / kScanSeg;
    k_scan_totals<<<nb, kScanT, 0, st>>>(in, n, scratch);
    k_scan_offsets<<<1, kScanT, 0, st>>>(scratch, nb);
    k_scan_final<<<nb, kScanT, 0, st>>>(in, n, scratch, out);
    FS_LAUNCHED(3);
}

}  // namespace fsb
