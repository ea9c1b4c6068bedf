// Device helpers shared by the kernels of libfs_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fs_internal.h"

namespace fsb {

// FP64 arithmetic with one rounding per operation.  The reference is plain C++
// compiled without fused multiply-adds; using these (never contracted)
// intrinsics everywhere a bit-identical FP64 result is claimed keeps the device
// arithmetic the same as the reference's, whatever -fmad says.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double stage_qm(const Stage& S, int o) {
    double qm = S.qm[0];
#pragma unroll
    for (int s = 1; s < 8; ++s)
        if (s < S.nsp && o >= S.start[s]) qm = S.qm[s];
    return qm;
}

// Position velocity of stage momentum p.  rk4_step moves x with p itself
// (AMRSimulation_step.cpp:163, :184, :208, :245); with the opt-in relativistic
// push it is relativistic_momentum_push's v = (p/m) / sqrt(1 + (p/m)^2)
// (AMRSimulation_step.cpp:101-111), correctly rounded so it matches the host.
__device__ __forceinline__ double stage_v(const Stage& S, int o, double p) {
    if (!S.rel) return p;
    double m = S.m[0];
#pragma unroll
    for (int s = 1; s < 8; ++s)
        if (s < S.nsp && o >= S.start[s]) m = S.m[s];
    const double u = __ddiv_rn(p, m);
    return __ddiv_rn(u, __dsqrt_rn(dadd(1.0, dmul(u, u))));
}

// RK4 epilogue for point o given the raw field E at that point
// (src/simulation_files/AMRSimulation_step.cpp:178-248).
__device__ __forceinline__ void apply_stage(const Stage& S, int o, double E) {
    // evaluate_field (AMRSimulation_field.cpp:164-173): the drive field is
    // added to the field before the stage uses it, es += a sin(k x - omega t)
    if (S.ext_x) E = dadd(E, dmul(S.ext_a, sin(dsub(dmul(S.ext_k, S.ext_x[o]), S.ext_omt))));
    switch (S.kind) {
        case STAGE_STORE:
            S.out[o] = E;
            break;
        case STAGE_RK2: {
            const double ef = dmul(E, stage_qm(S, o));
            const double p2 = S.pst[o];
            const double v2 = stage_v(S, o, p2);
            S.xk[o] = dadd(S.x[o], dmul(S.hdt, v2));
            S.accX[o] = dadd(S.accX[o], dmul(2.0, v2));
            S.accP[o] = dadd(S.accP[o], dmul(2.0, ef));
            S.pst[o] = dadd(S.p[o], dmul(S.hdt, ef));  // p3
            break;
        }
        case STAGE_RK3: {
            const double ef = dmul(E, stage_qm(S, o));
            const double p3 = S.pst[o];
            const double v3 = stage_v(S, o, p3);
            S.xk[o] = dadd(S.x[o], dmul(S.dt, v3));
            S.accX[o] = dadd(S.accX[o], dmul(2.0, v3));
            S.accP[o] = dadd(S.accP[o], dmul(2.0, ef));
            S.pst[o] = dadd(S.p[o], dmul(S.dt, ef));  // p4
            break;
        }
        case STAGE_RK4: {
            const double ef = dmul(E, stage_qm(S, o));
            const double p4 = S.pst[o];
            const double ax = dadd(S.accX[o], stage_v(S, o, p4));
            const double ap = dadd(S.accP[o], ef);
            S.x[o] = dadd(S.x[o], dmul(S.dt6, ax));
            S.p[o] = dadd(S.p[o], dmul(S.dt6, ap));
            break;
        }
        default:
            break;
    }
}

// Bounded spin limit for every device-side wait (mbarrier, flags).
constexpr long long kSpinLimit = 1LL << 26;

// One MUFU.RSQ (callers pass arguments >= eps^2 > 0, never denormal).
__device__ __forceinline__ float rsqrt_approx(float v) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v));
    return y;
}
// One MUFU.RCP (callers pass products of two values in [eps^2, L^2/4+eps^2]).
__device__ __forceinline__ float rcp_approx(float v) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v));
    return y;
}

}  // namespace fsb
