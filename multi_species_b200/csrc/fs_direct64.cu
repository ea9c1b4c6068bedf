// Plain FP64 periodic direct sum: the reference's arithmetic on the GPU.
//
// E_MQ_DirectSum::operator() (src/FieldStructure.cpp:106-156) evaluated one
// target per thread with the sources streamed through shared-memory tiles in
// their original order, so every target's sum is formed in the same order and
// with the same roundings (explicit _rn intrinsics, no contraction, IEEE
// division and square root) as the reference's sequential loop: the result is
// bit-identical to E_MQ_DirectSum.  This is the parity path and the "plain
// FP64 GPU" comparator; it is bound by the FP64 pipe (two divisions and one
// square root per pair).
#include <cfloat>

#include "fs_device.cuh"

namespace fsb {

namespace {

constexpr int kThreads64 = 128;
constexpr int kTile64 = 1024;

__global__ void __launch_bounds__(kThreads64)
k_direct64(const double* __restrict__ tx, int nt, const double* __restrict__ sx,
           const double* __restrict__ sq, int ns, double L, double eps, double norm_const,
           Stage S) {
    __shared__ double sh_x[kTile64];
    __shared__ double sh_q[kTile64];
    const int i = blockIdx.x * kThreads64 + threadIdx.x;
    const double xi = (i < nt) ? tx[i] : 0.0;
    const double four_eps2 = dmul(dmul(4.0, eps), eps);
    double ei = 0.0;
    for (int base = 0; base < ns; base += kTile64) {
        const int cnt = min(kTile64, ns - base);
        for (int k = threadIdx.x; k < cnt; k += kThreads64) {
            sh_x[k] = sx[base + k];
            sh_q[k] = sq[base + k];
        }
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            double z = ddiv(dsub(xi, sh_x[j]), L);
            z = dsub(z, round(z));
            if (fabs(dsub(z, 0.5)) < DBL_MIN || fabs(dadd(z, 0.5)) < DBL_MIN || fabs(z) < DBL_MIN) continue;
            const double r2 = dadd(dmul(dmul(dmul(dmul(4.0, z), z), L), L), four_eps2);
            const double inv = ddiv(1.0, __dsqrt_rn(r2));
            const double term = dmul(dmul(dmul(dmul(sh_q[j], -1.0), z), L), dsub(norm_const, inv));
            ei = dadd(ei, term);
        }
        __syncthreads();
    }
    if (i < nt) apply_stage(S, i, ei);
}

// Open boundaries, E_MQ_DirectSum_openbcs::operator() (src/FieldStructure.cpp:170-192):
// es_i = sum_j ((q_j * 0.5) * z) / sqrt(z*z + eps^2) - x_i, z = x_i - x_j, in the
// reference's order and roundings (bit-identical).
__global__ void __launch_bounds__(kThreads64)
k_direct64_open(const double* __restrict__ tx, int nt, const double* __restrict__ sx, const double* __restrict__ sq,
                int ns, double eps, Stage S) {
    __shared__ double sh_x[kTile64];
    __shared__ double sh_q[kTile64];
    const int i = blockIdx.x * kThreads64 + threadIdx.x;
    const double xi = (i < nt) ? tx[i] : 0.0;
    const double eps_sq = dmul(eps, eps);
    double ei = 0.0;
    for (int base = 0; base < ns; base += kTile64) {
        const int cnt = min(kTile64, ns - base);
        for (int k = threadIdx.x; k < cnt; k += kThreads64) {
            sh_x[k] = sx[base + k];
            sh_q[k] = sq[base + k];
        }
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            const double z = dsub(xi, sh_x[j]);
            ei = dadd(ei, ddiv(dmul(dmul(sh_q[j], 0.5), z), __dsqrt_rn(dadd(dmul(z, z), eps_sq))));
        }
        __syncthreads();
    }
    if (i < nt) apply_stage(S, i, dsub(ei, xi));
}

class Direct64Open final : public FieldEngine {
   public:
    explicit Direct64Open(double eps) : eps_(eps) {}
    void eval(const double* d_t, int nt, const double* d_s, const double* d_q, int ns, const Stage& stage,
              cudaStream_t st) override {
        last_pairs = (double)nt * (double)ns;
        if (nt <= 0) return;
        const int blocks = (nt + kThreads64 - 1) / kThreads64;
        ProfScope prof("k_direct64_open", st, last_pairs);
        k_direct64_open<<<blocks, kThreads64, 0, st>>>(d_t, nt, d_s, d_q, ns, eps_, stage);
        FS_LAUNCHED(1);
    }

   private:
    double eps_;
};

class Direct64 final : public FieldEngine {
   public:
    Direct64(double L, double eps) : L_(L), eps_(eps) {
        // same expression as the reference: 1/sqrt(L*L + 4*epsilon*epsilon)
        norm_const_ = 1 / std::sqrt(L * L + 4 * eps * eps);
    }
    void eval(const double* d_t, int nt, const double* d_s, const double* d_q, int ns,
              const Stage& stage, cudaStream_t st) override {
        last_pairs = (double)nt * (double)ns;
        if (nt <= 0) return;
        const int blocks = (nt + kThreads64 - 1) / kThreads64;
        ProfScope prof("k_direct64", st, last_pairs);
        k_direct64<<<blocks, kThreads64, 0, st>>>(d_t, nt, d_s, d_q, ns, L_, eps_, norm_const_, stage);
        FS_LAUNCHED(1);
    }

   private:
    double L_, eps_, norm_const_;
};

}  // namespace

FieldEngine* make_direct64(double L, double eps) { return new Direct64(L, eps); }
FieldEngine* make_direct64_open(double eps) { return new Direct64Open(eps); }

}  // namespace fsb
