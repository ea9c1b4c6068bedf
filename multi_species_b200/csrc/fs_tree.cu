// Barycentric Lagrange treecode on the device (E_MQ_Treecode,
// src/FieldStructure.cpp:230-1020).
//
// Same tree, lists and moments as the reference, rebuilt every call like the
// reference does, but on the GPU:
//   k_tree_keys/sort   particles_x = fmod(x, L) (:235-247), sorted (CUB radix)
//   k_build_tree       one CTA, level-synchronous midpoint bisection over the
//                      root interval [min - 0.1234, max + 0.001] (:506-632,
//                      :1032-1050): a node with n >= max_source points splits at
//                      0.5 (x0 + x1), points with x <= mid go left, children only
//                      when non-empty.  Member ranges are contiguous in sorted
//                      order, so a split is one binary search.
//   k_lists            one thread per leaf: the reference's traversal from the
//                      root (build_interaction_list :663-702) -- any leaf reached
//                      is near, a node is far when (r_b + r_p) / R < theta with the
//                      periodic R = min(|dxc|, L - |dxc|), else recurse -- in the
//                      same IEEE arithmetic, so far/near decisions are identical.
//   k_moment_items /   Chebyshev-Lobatto t_k = x0 + (cos(k pi/P) + 1)/2 (x1 - x0) and
//   k_moment_reduce    M_{c,k} = sum_j lambda_j a_k(x_j) / sum_k a_k(x_j) for every
//                      node but the root (alloc_set_cluster_list :775-866),
//                      as fixed-size member chunks reduced in a fixed order
//                      (deterministic).  cos(k pi/P) comes from the host C library.
//   k_far_near64       per target: far list then near list (Call_BL :904-961,
//                      Call_Ds :963-1020), the reference's arithmetic in FP64.
//   k_far32 + k_near32 FP32-compensated form: far field in FP64 with a
//                      reciprocal-square-root kernel evaluation, near field as
//                      FP32 tiles of the near leaves' sources with Kahan sums.
// The kernel of the reference treecode is sqrt(L^2+4 eps^2)/L times the direct
// sum's (:949, :1008 vs :150); both forms keep that normalisation.
#include <cub/cub.cuh>

#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

#include "fs_device.cuh"

namespace fsb {

namespace {

constexpr int kMaxDegree = 16;
constexpr int kMaxDepth = 60;
constexpr int kFarCap = 256;   // far-list entries per leaf
constexpr int kNearCap = 64;   // near-list entries per leaf
constexpr int kChunk = 8192;   // member points per moment work item

struct TNode {
    double x0, x1, xc;
    int m0, m1;       // inclusive member range in sorted order
    int child0, child1;
    int parent, level;
};

// Per-instance constants (device array of 2 x (kMaxDegree+1) doubles):
//   cheb[k] = cos(k pi / P) from the host C library, w[k] = (-1)^k (1/2 at the ends).

// signed double -> order-preserving unsigned key
__device__ __forceinline__ uint64_t order_key(double v) {
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_value(uint64_t k) {
    const uint64_t b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__global__ void k_tree_keys(const double* __restrict__ x, int n, double L, uint64_t* __restrict__ keys,
                            int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = order_key(fmod(x[i], L));
    idx[i] = i;
}

__global__ void k_tree_gather(const uint64_t* __restrict__ skeys, const int* __restrict__ sidx,
                              const double* __restrict__ q, int n, double* __restrict__ sx,
                              double* __restrict__ lam) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    sx[j] = key_value(skeys[j]);
    lam[j] = q[sidx[j]];
}

__device__ __forceinline__ int upper_bound(const double* __restrict__ a, int lo, int hi, double v) {
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (a[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// meta: [0] nodes, [1] leaves, [2] error code, [3] depth
__global__ void __launch_bounds__(1024) k_build_tree(const double* __restrict__ sx, int n, int N0, int cap_nodes,
                                                     int cap_leaves, TNode* __restrict__ nodes,
                                                     int* __restrict__ leaves, int* __restrict__ meta) {
    __shared__ int s_begin, s_end, s_next, s_nleaf, s_err;
    __shared__ int s_scan[1024];
    __shared__ int s_lscan[1024];
    const int tid = threadIdx.x;
    if (tid == 0) {
        TNode r;
        r.x0 = sx[0] - 0.1234;
        r.x1 = sx[n - 1] + 0.001;
        r.xc = 0.5 * (r.x0 + r.x1);
        r.m0 = 0;
        r.m1 = n - 1;
        r.child0 = r.child1 = -1;
        r.parent = -1;
        r.level = 0;
        nodes[0] = r;
        s_begin = 0;
        s_end = 1;
        s_next = 1;
        s_nleaf = 0;
        s_err = 0;
    }
    __syncthreads();
    int level = 0;
    while (s_begin < s_end) {
        if (level > kMaxDepth) {
            if (tid == 0) s_err = FS_ERR_TREE;
            break;
        }
        const int begin = s_begin, end = s_end;
        for (int base = begin; base < end; base += blockDim.x) {
            const int i = base + tid;
            int nchild = 0, isleaf = 0, k = 0;
            TNode nd;
            if (i < end) {
                nd = nodes[i];
                const int cnt = nd.m1 - nd.m0 + 1;
                if (cnt >= N0) {
                    const double mid = 0.5 * (nd.x0 + nd.x1);
                    k = upper_bound(sx, nd.m0, nd.m1 + 1, mid);
                    nchild = (k > nd.m0) + (k <= nd.m1);
                } else {
                    isleaf = 1;
                }
            }
            s_scan[tid] = nchild;
            s_lscan[tid] = isleaf;
            __syncthreads();
            for (int off = 1; off < (int)blockDim.x; off <<= 1) {  // inclusive scans
                const int a = (tid >= off) ? s_scan[tid - off] : 0;
                const int b = (tid >= off) ? s_lscan[tid - off] : 0;
                __syncthreads();
                s_scan[tid] += a;
                s_lscan[tid] += b;
                __syncthreads();
            }
            const int cfirst = s_next + s_scan[tid] - nchild;
            const int lslot = s_nleaf + s_lscan[tid] - isleaf;
            if (i < end) {
                if (isleaf) {
                    if (lslot < cap_leaves) leaves[lslot] = i;
                } else if (nchild) {
                    const double mid = 0.5 * (nd.x0 + nd.x1);
                    int c = cfirst;
                    int c0 = -1, c1 = -1;
                    if (k > nd.m0 && c < cap_nodes) {
                        TNode ch;
                        ch.x0 = nd.x0;
                        ch.x1 = mid;
                        ch.xc = 0.5 * (ch.x0 + ch.x1);
                        ch.m0 = nd.m0;
                        ch.m1 = k - 1;
                        ch.child0 = ch.child1 = -1;
                        ch.parent = i;
                        ch.level = level + 1;
                        nodes[c] = ch;
                        c0 = c++;
                    }
                    if (k <= nd.m1 && c < cap_nodes) {
                        TNode ch;
                        ch.x0 = mid;
                        ch.x1 = nd.x1;
                        ch.xc = 0.5 * (ch.x0 + ch.x1);
                        ch.m0 = k;
                        ch.m1 = nd.m1;
                        ch.child0 = ch.child1 = -1;
                        ch.parent = i;
                        ch.level = level + 1;
                        nodes[c] = ch;
                        if (c0 < 0) c0 = c;
                        else c1 = c;
                        ++c;
                    }
                    nodes[i].child0 = c0;
                    nodes[i].child1 = c1;
                }
            }
            __syncthreads();
            if (tid == blockDim.x - 1) {
                s_next += s_scan[tid];
                s_nleaf += s_lscan[tid];
                if (s_next > cap_nodes || s_nleaf > cap_leaves) s_err = FS_ERR_TREE;
            }
            __syncthreads();
            if (s_err) break;
        }
        if (s_err) break;
        if (tid == 0) {
            s_begin = end;
            s_end = s_next;
        }
        ++level;
        __syncthreads();
    }
    if (tid == 0) {
        meta[0] = min(s_next, cap_nodes);
        meta[1] = min(s_nleaf, cap_leaves);
        meta[2] = s_err;
        meta[3] = level;
    }
}

__global__ void k_mark_leaves(const TNode* __restrict__ nodes, const int* __restrict__ leaves,
                              const int* __restrict__ meta, int* __restrict__ leaf_of) {
    const int l = blockIdx.x;
    if (l >= meta[1] || meta[2]) return;
    const TNode nd = nodes[leaves[l]];
    for (int j = nd.m0 + threadIdx.x; j <= nd.m1; j += blockDim.x) leaf_of[j] = l;
}

// build_interaction_list (src/FieldStructure.cpp:663-702) for one leaf.
__global__ void k_lists(const TNode* __restrict__ nodes, const int* __restrict__ leaves, const int* __restrict__ meta,
                        double L, double sqrt_sq_theta, int* __restrict__ far_list, int* __restrict__ far_n,
                        int* __restrict__ near_list, int* __restrict__ near_n, int* __restrict__ err) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= meta[1] || meta[2]) return;
    const TNode b = nodes[leaves[l]];
    int stack[2 * kMaxDepth + 4];
    int sp = 0;
    stack[sp++] = 0;
    int nf = 0, nn = 0;
    while (sp > 0) {
        const int pi = stack[--sp];
        const TNode p = nodes[pi];
        const double r_dist = fabs(b.xc - p.xc);
        const double dfbpx = fmin(r_dist, L - r_dist);
        const double dfbx = b.x1 - b.xc;
        const double dfpx = p.x1 - p.xc;
        const double sq_R = dfbpx * dfbpx, sq_rb = dfbx * dfbx, sq_rp = dfpx * dfpx;
        if (p.child0 < 0 && p.child1 < 0) {
            if (nn < kNearCap) near_list[(size_t)l * kNearCap + nn] = pi;
            ++nn;
        } else if ((__dsqrt_rn(sq_rb) + __dsqrt_rn(sq_rp)) / __dsqrt_rn(sq_R) < sqrt_sq_theta) {
            if (nf < kFarCap) far_list[(size_t)l * kFarCap + nf] = pi;
            ++nf;
        } else {
            if (sp + 2 > 2 * kMaxDepth + 4) {
                atomicCAS(err, 0, (int)FS_ERR_TREE);
                return;
            }
            if (p.child1 >= 0) stack[sp++] = p.child1;  // pop order: child0 first
            if (p.child0 >= 0) stack[sp++] = p.child0;
        }
    }
    if (nf > kFarCap || nn > kNearCap) atomicCAS(err, 0, (int)FS_ERR_TREE);
    far_n[l] = min(nf, kFarCap);
    near_n[l] = min(nn, kNearCap);
}

// Work items for the moments: (node, chunk) pairs, chunk = kChunk members.
__global__ void k_item_counts(const TNode* __restrict__ nodes, const int* __restrict__ meta, int cap_nodes,
                              int* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap_nodes) return;
    int c = 0;
    if (i > 0 && i < meta[0] && !meta[2]) c = (nodes[i].m1 - nodes[i].m0 + kChunk) / kChunk;
    counts[i] = c;
}

// Partial moments of a member chunk of one node, one CTA per work item
// (grid-stride over the items).  Per point the reference's arithmetic
// (alloc_set_cluster_list :826-860) with one rounding per operation.
// kPP > 0 fixes the number of Chebyshev nodes (degree + 1) at compile time, so
// that the per-point arrays live in registers (with kPP = 0, read from P at
// run time, they sit in local memory); the arithmetic is the same either way.
// 1/x in FP64 for the FP32c treecode's moments: the hardware approximation
// and two Newton-Raphson steps (relative error ~1e-16 for normal x).
__device__ __forceinline__ double rcp_nr64(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// FP32c treecode moments with rcp_nr64 products instead of IEEE divisions:
// measured 0.9% faster per full-size treecode step.
#ifndef FS_FAST_MOMENTS
#define FS_FAST_MOMENTS 1
#endif
constexpr bool kFastMoments = FS_FAST_MOMENTS;
// kFast (the FP32c treecode): divisions as products with rcp_nr64 instead of
// IEEE divisions; the FP64 treecode keeps the reference's arithmetic.
template <int kPP, bool kFast>
__global__ void __launch_bounds__(256) k_moment_items(const TNode* __restrict__ nodes, const int* __restrict__ meta,
                                                      int cap_nodes, const int* __restrict__ item_start,
                                                      int cap_items, int P, const double* __restrict__ consts,
                                                      const double* __restrict__ sx, const double* __restrict__ lam,
                                                      double* __restrict__ partial) {
    const int nnodes = min(meta[0], cap_nodes);
    if (meta[2] || nnodes < 2) return;
    const int total = min(cap_items, item_start[nnodes - 1] +
                                         (nodes[nnodes - 1].m1 - nodes[nnodes - 1].m0 + kChunk) / kChunk);
    const double* cheb = consts;
    const double* wk = consts + (kMaxDegree + 1);
    const int PP = kPP > 0 ? kPP : P + 1;
    __shared__ double red[8 * (kMaxDegree + 1)];  // per warp (256 threads), per moment
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        // node owning this item: last node with item_start <= item (nodes 1..nnodes-1)
        int lo = 1, hi = nnodes - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (item_start[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        const TNode nd = nodes[lo];
        const int chunk = item - item_start[lo];
        const int a = nd.m0 + chunk * kChunk;
        const int e = min(nd.m1, a + kChunk - 1);
        double t[kMaxDegree + 1], acc[kMaxDegree + 1];
#pragma unroll
        for (int k = 0; k < PP; ++k) {
            t[k] = dadd(nd.x0, dmul(dmul(dadd(cheb[k], 1.0), 0.5), dsub(nd.x1, nd.x0)));
            acc[k] = 0.0;
        }
        for (int j = a + threadIdx.x; j <= e; j += blockDim.x) {
            const double x = sx[j];
            double ak[kMaxDegree + 1];
            int exact = -1;
            double sum = 0.0;
            // w_k / dx_k, two nodes per division where both differences are
            // clear of zero: 1/dx_a = dx_b / (dx_a dx_b) (a few ulps; |dx| lies
            // between the spacing of doubles near x and the node width, so the
            // product neither underflows nor overflows)
            int k = 0;
#pragma unroll
            for (; k + 1 < PP; k += 2) {
                const double da = dsub(x, t[k]), db = dsub(x, t[k + 1]);
                if (fabs(da) <= DBL_MIN || fabs(db) <= DBL_MIN) {
                    if (fabs(da) <= DBL_MIN) {
                        exact = k;
                        ak[k] = 0.0;
                    } else {
                        ak[k] = (kFast ? wk[k] * rcp_nr64(da) : ddiv(wk[k], da));
                        sum = dadd(sum, ak[k]);
                    }
                    if (fabs(db) <= DBL_MIN) {
                        exact = k + 1;
                        ak[k + 1] = 0.0;
                    } else {
                        ak[k + 1] = (kFast ? wk[k + 1] * rcp_nr64(db) : ddiv(wk[k + 1], db));
                        sum = dadd(sum, ak[k + 1]);
                    }
                } else {
                    const double r = (kFast ? rcp_nr64(dmul(da, db)) : ddiv(1.0, dmul(da, db)));
                    ak[k] = dmul(wk[k], dmul(db, r));
                    ak[k + 1] = dmul(wk[k + 1], dmul(da, r));
                    sum = dadd(dadd(sum, ak[k]), ak[k + 1]);
                }
            }
            if (k < PP) {
                const double dx = dsub(x, t[k]);
                if (fabs(dx) <= DBL_MIN) {
                    exact = k;
                    ak[k] = 0.0;
                } else {
                    ak[k] = (kFast ? wk[k] * rcp_nr64(dx) : ddiv(wk[k], dx));
                    sum = dadd(sum, ak[k]);
                }
            }
            if (exact > -1) {
                sum = 1.0;
#pragma unroll
                for (int k = 0; k < PP; ++k) ak[k] = (k == exact) ? 1.0 : 0.0;
            }
            const double D = (kFast ? rcp_nr64(sum) : ddiv(1.0, sum));
            const double l = lam[j];
#pragma unroll
            for (int k = 0; k < PP; ++k) acc[k] = dadd(acc[k], dmul(dmul(ak[k], D), l));
        }
        // block reduction of PP values in a fixed order: a shuffle tree within
        // each warp, then the eight warp sums in warp order
        double* out = partial + (size_t)item * (kMaxDegree + 1);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < PP; ++k) {
            double v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = dadd(v, __shfl_down_sync(0xffffffffu, v, o));
            if (lane == 0) red[warp * (kMaxDegree + 1) + k] = v;
        }
        __syncthreads();
        if (threadIdx.x < PP) {
            double sum = red[threadIdx.x];
            for (int w = 1; w < 8; ++w) sum = dadd(sum, red[w * (kMaxDegree + 1) + threadIdx.x]);
            out[threadIdx.x] = sum;
        }
        __syncthreads();
    }
}

__global__ void k_moment_reduce(const TNode* __restrict__ nodes, const int* __restrict__ meta, int cap_nodes,
                                const int* __restrict__ item_start, int P, const double* __restrict__ partial,
                                double* __restrict__ mom) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nnodes = min(meta[0], cap_nodes);
    if (i >= nnodes || meta[2]) return;
    const int PP = P + 1;
    double* m = mom + (size_t)i * (kMaxDegree + 1);
    if (i == 0) {  // the root's moments are never formed (and never used)
        for (int k = 0; k < PP; ++k) m[k] = 0.0;
        return;
    }
    const int nitems = (nodes[i].m1 - nodes[i].m0 + kChunk) / kChunk;
    for (int k = 0; k < PP; ++k) {
        double s = 0.0;
        for (int c = 0; c < nitems; ++c) s = dadd(s, partial[(size_t)(item_start[i] + c) * (kMaxDegree + 1) + k]);
        m[k] = s;
    }
}

// One term of the reference sum, FP64, same association and roundings as
// `w * -1.0 * s * (1 - sqrt(deno / (4*s*s*L*L + 4*eps*eps)))`
// (src/FieldStructure.cpp:940-950, :1000-1010); skipped pairs add nothing.
__device__ __forceinline__ double tc_term(double w, double xi, double xj, double L, double deno, double four_eps2,
                                          bool& skip) {
    double s = ddiv(dsub(xi, xj), L);
    s = dsub(s, round(s));
    skip = fabs(dsub(s, 0.5)) < DBL_MIN || fabs(dadd(s, 0.5)) < DBL_MIN || fabs(s) < DBL_MIN;
    const double den = dadd(dmul(dmul(dmul(dmul(4.0, s), s), L), L), four_eps2);
    return dmul(dmul(dmul(w, -1.0), s), dsub(1.0, __dsqrt_rn(ddiv(deno, den))));
}

// FP64 per target: far field (Call_BL) then near field (Call_Ds), reference
// arithmetic and order; result through the stage epilogue at the original index.
__global__ void k_far_near64(const TNode* __restrict__ nodes, const int* __restrict__ meta,
                             const int* __restrict__ leaf_of, const int* __restrict__ leaves,
                             const int* __restrict__ far_list, const int* __restrict__ far_n,
                             const int* __restrict__ near_list, const int* __restrict__ near_n,
                             const double* __restrict__ mom, const double* __restrict__ consts,
                             const double* __restrict__ sx, const double* __restrict__ lam,
                             const int* __restrict__ sidx, int n, int P, double L, double eps, Stage S) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || meta[2]) return;
    const double* cheb = consts;
    const int PP = P + 1;
    const double deno = dadd(dmul(L, L), dmul(dmul(4.0, eps), eps));
    const double four_eps2 = dmul(dmul(4.0, eps), eps);
    const int l = leaf_of[j];
    const double x = sx[j];
    double far = 0.0;
    for (int f = 0; f < far_n[l]; ++f) {
        const int fi = far_list[(size_t)l * kFarCap + f];
        const TNode nd = nodes[fi];
        const double* m = mom + (size_t)fi * (kMaxDegree + 1);
        for (int k = 0; k < PP; ++k) {
            const double t = dadd(nd.x0, dmul(dmul(dadd(cheb[k], 1.0), 0.5), dsub(nd.x1, nd.x0)));
            bool skip;
            const double v = tc_term(m[k], x, t, L, deno, four_eps2, skip);
            if (!skip) far = dadd(far, v);
        }
    }
    double near = 0.0;
    for (int q = 0; q < near_n[l]; ++q) {
        const TNode nd = nodes[near_list[(size_t)l * kNearCap + q]];
        for (int i = nd.m0; i <= nd.m1; ++i) {
            bool skip;
            const double v = tc_term(lam[i], x, sx[i], L, deno, four_eps2, skip);
            if (!skip) near = dadd(near, v);
        }
    }
    apply_stage(S, sidx[j], dadd(dadd(0.0, far), near));
}

// FP32-compensated form, far part: FP64 with the kernel written through one
// reciprocal square root, K_tc(d) = norm * (d / (2 sqrt(d^2+eps^2)) - c d).
// k_far32's per-node arithmetic: the nearest image by a product with 1/L and
// 1/sqrt by the hardware approximation and one Newton step (1), or by an IEEE
// division and the library's FP64 rsqrt (0).  (1) measured 4% faster per step
// of the three-species treecode workload, with E changed by about 2e-14.
#ifndef FS_FAR32_FAST
#define FS_FAR32_FAST 1
#endif
constexpr bool kFar32Fast = FS_FAR32_FAST;

__global__ void k_far32(const TNode* __restrict__ nodes, const int* __restrict__ meta, const int* __restrict__ leaf_of,
                        const int* __restrict__ far_list, const int* __restrict__ far_n,
                        const double* __restrict__ mom, const double* __restrict__ consts,
                        const double* __restrict__ sx, int n, int P, double L, double eps, double norm, double cbg,
                        double* __restrict__ efar) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || meta[2]) return;
    const double* cheb = consts;
    const int PP = P + 1;
    const int l = leaf_of[j];
    const double x = sx[j];
    const double e2 = eps * eps;
    const double invL = 1.0 / L;
    double far = 0.0;
    for (int f = 0; f < far_n[l]; ++f) {
        const int fi = far_list[(size_t)l * kFarCap + f];
        const TNode nd = nodes[fi];
        const double* m = mom + (size_t)fi * (kMaxDegree + 1);
        for (int k = 0; k < PP; ++k) {
            const double t = nd.x0 + (cheb[k] + 1.0) * 0.5 * (nd.x1 - nd.x0);
            double d = x - t;
            if (kFar32Fast) {
                // nearest image by a product with 1/L, 1/sqrt from the hardware
                // approximation and one Newton step (relative error ~1e-14)
                d -= L * rint(d * invL);
                const double r = d * d + e2;
                double y;
                asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r));
                y = y * fma(-0.5 * r, y * y, 1.5);
                far += m[k] * (d * (0.5 * y - cbg));
            } else {
                d -= L * rint(d / L);
                far += m[k] * (d * (0.5 * rsqrt(d * d + e2) - cbg));
            }
        }
    }
    efar[j] = norm * far;
}

// FP32-compensated form, near part: one CTA per (leaf, block of
// kNearThreads x kNearR targets), kNearR targets per thread.
//   K_tc(d) / norm = d/(2 sqrt(d^2+eps^2)) - c d,  d = xt - x_j  (xt = image of x_i)
// The linear term c d is summed exactly in FP64 from prefix sums of lambda and
// lambda x.  For each near leaf, when every target of the CTA sees the whole
// leaf in one periodic image and within the band |d| <= band (the usual case:
// near leaves are neighbours a few leaf widths away), the pairs are
// lambda/2 d y, y = rsqrt(d^2+eps^2), accumulated in packed FP32x2 over two
// targets with Kahan compensation per tile and reduced in FP64 across tiles.
// Otherwise every target of the CTA takes the general path for that leaf: the
// leaf's sources are cut where their image changes (at most three images), and
// beyond the band the sign part sign(d) lambda/2 is summed exactly in FP64 while
// the kernel accumulates -+ lambda/2 c(v) (c = v/2 + v^2/8, v = eps^2 y^2).
// Sources are staged through shared memory as FP32 offsets from an FP64 tile
// base; each image's target offset is formed in FP64 before rounding.
#ifndef FS_NEAR_THREADS
#define FS_NEAR_THREADS 128
#endif
#ifndef FS_NEAR_R
#define FS_NEAR_R 4
#endif
constexpr int kNearThreads = FS_NEAR_THREADS;
constexpr int kNearR = FS_NEAR_R;
constexpr int kNearBlock = kNearThreads * kNearR;
constexpr int kNearTile = 256;
constexpr double kNearBand = 24.0;
// near items taken by a persistent grid in decreasing order of work (1) or one
// CTA per item in leaf order (0).  At 6.3M points (1) measured 0.5% slower per
// treecode step than (0): the plain grid of ~12k CTAs leaves little tail.
#ifndef FS_NEAR_ORDER
#define FS_NEAR_ORDER 0
#endif
constexpr bool kNearOrder = FS_NEAR_ORDER;

struct NearImage {
    double xt;    // target coordinate in this image
    int start;    // first source index of the image's subrange
    int U1, U2;   // band [U1, U2): |d| <= band
};

__device__ __forceinline__ int lower_bound_d(const double* __restrict__ a, int lo, int hi, double v) {
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int upper_bound_d(const double* __restrict__ a, int lo, int hi, double v) {
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (a[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ double range_sum(const double* __restrict__ incl, int a, int e) {
    // sum over [a, e) of the series whose inclusive prefix is incl
    if (e <= a) return 0.0;
    return incl[e - 1] - (a > 0 ? incl[a - 1] : 0.0);
}

// General path for one target and one near leaf (all threads of the CTA call
// it together: it stages tiles through `sh` with barriers).
__device__ void near_general(const TNode& nd, double x, const double* __restrict__ sx,
                             const double* __restrict__ lam, const double* __restrict__ pl,
                             const double* __restrict__ plx, double L, double band, double cbg, float eps2, float a1,
                             float a2, float4* sh, double& exact, double& fp, int* __restrict__ err) {
    NearImage im[3];
    int nim = 0;
    int a = nd.m0;
    while (a <= nd.m1 && nim < 3) {
        // image of source j: m_j = round((x - x_j) / L), the reference's
        // choice (z - round(z)); m_j is non-increasing in j
        const double m = round((x - sx[a]) / L);
        const double xt = x - m * L;
        int e;  // first source of the next image
        {
            int lo = a + 1, hi = nd.m1 + 1;
            while (lo < hi) {
                const int mid = lo + ((hi - lo) >> 1);
                if (round((x - sx[mid]) / L) < m) hi = mid;
                else lo = mid + 1;
            }
            e = lo;
        }
        const int U1 = lower_bound_d(sx, a, e, xt - band);
        const int U2 = upper_bound_d(sx, U1, e, xt + band);  // first x_j > xt + band
        exact += 0.5 * (range_sum(pl, a, U1) - range_sum(pl, U2, e)) -
                 cbg * (xt * range_sum(pl, a, e) - range_sum(plx, a, e));
        im[nim].xt = xt;
        im[nim].start = a;
        im[nim].U1 = U1;
        im[nim].U2 = U2;
        ++nim;
        a = e;
    }
    if (a <= nd.m1) atomicCAS(err, 0, (int)FS_ERR_TREE);
    for (int k = nim; k < 3; ++k) {
        im[k].xt = im[nim - 1].xt;
        im[k].start = INT_MAX;
        im[k].U1 = im[k].U2 = 0;
    }
    for (int t0 = nd.m0; t0 <= nd.m1; t0 += kNearTile) {
        const int cnt = min(kNearTile, nd.m1 - t0 + 1);
        const double base = sx[t0];
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += kNearThreads) {
            const float lh = (float)(0.5 * lam[t0 + k]);
            sh[k] = make_float4((float)(sx[t0 + k] - base), lh, lh * a1, lh * a2);
        }
        __syncthreads();
        const float tau0 = (float)(im[0].xt - base), tau1 = (float)(im[1].xt - base),
                    tau2 = (float)(im[2].xt - base);
        const int s1 = im[1].start, s2 = im[2].start;
        const int u10 = im[0].U1, u11 = im[1].U1, u12 = im[2].U1;
        const int u20 = im[0].U2, u21 = im[1].U2, u22 = im[2].U2;
        float acc = 0.f, cmp = 0.f;
        for (int k = 0; k < cnt; ++k) {
            const int jj = t0 + k;
            const bool g1 = jj >= s1, g2 = jj >= s2;
            const float tr = g2 ? tau2 : (g1 ? tau1 : tau0);
            const int U1 = g2 ? u12 : (g1 ? u11 : u10);
            const int U2 = g2 ? u22 : (g1 ? u21 : u20);
            const float4 e = sh[k];
            const float d = tr - e.x;
            const float y = rsqrt_approx(fmaf(d, d, eps2));
            const float z = y * y;
            const float c = z * fmaf(z, e.w, e.z);
            const float v = (jj < U1) ? -c : ((jj >= U2) ? c : e.y * (d * y));
            const float w = v - cmp;
            const float t = acc + w;
            cmp = (t - acc) - w;
            acc = t;
        }
        fp += (double)acc - (double)cmp;
    }
}

struct NearArgs {
    const TNode* nodes;
    const int* meta;
    const int* leaves;
    const int* near_list;
    const int* near_n;
    const double* sx;
    const double* lam;
    const double* pl;
    const double* plx;
    const double* efar;
    const int* sidx;
    double L, eps, cbg, norm;
    Stage S;
    int* err;
};

// Near field of target block yb of leaf l (all threads of the CTA together).
__device__ void near_item(const NearArgs& A, int l, int yb, float4* shg, float2 (*shb)[kNearTile]) {
    const TNode* __restrict__ nodes = A.nodes;
    const int* __restrict__ near_list = A.near_list;
    const double* __restrict__ sx = A.sx;
    const double* __restrict__ lam = A.lam;
    const double* __restrict__ pl = A.pl;
    const double* __restrict__ plx = A.plx;
    const double L = A.L, eps = A.eps, cbg = A.cbg;
    int* __restrict__ err = A.err;
    if (l >= A.meta[1] || A.meta[2]) return;
    const TNode leaf = nodes[A.leaves[l]];
    const int tb0 = leaf.m0 + yb * kNearBlock;
    if (tb0 > leaf.m1) return;  // whole CTA beyond the leaf
    const double band = kNearBand * eps;
    const double e2d = eps * eps;
    const float eps2 = (float)e2d, a1 = (float)(e2d / 2), a2 = (float)(e2d * e2d / 8);
    int jt[kNearR];
    double x[kNearR], exact[kNearR], fp[kNearR];
#pragma unroll
    for (int r = 0; r < kNearR; ++r) {
        jt[r] = tb0 + threadIdx.x + r * kNearThreads;
        x[r] = (jt[r] <= leaf.m1) ? sx[jt[r]] : sx[leaf.m0];  // padded targets repeat a real one
        exact[r] = 0.0;
        fp[r] = 0.0;
    }
    for (int q = 0; q < A.near_n[l]; ++q) {
        const TNode nd = nodes[near_list[(size_t)l * kNearCap + q]];
        const double xlo = sx[nd.m0], xhi = sx[nd.m1];
        double xt[kNearR];
        bool simple = true;
#pragma unroll
        for (int r = 0; r < kNearR; ++r) {
            const double m = round((x[r] - xlo) / L);
            xt[r] = x[r] - m * L;
            simple = simple && (round((x[r] - xhi) / L) == m) && (xlo >= xt[r] - band) && (xhi <= xt[r] + band);
        }
        if (__syncthreads_and(simple)) {
            const double sl = range_sum(pl, nd.m0, nd.m1 + 1), slx = range_sum(plx, nd.m0, nd.m1 + 1);
#pragma unroll
            for (int r = 0; r < kNearR; ++r) exact[r] -= cbg * (xt[r] * sl - slx);
            const float2 e2v = make_float2(eps2, eps2), m1 = make_float2(-1.f, -1.f);
            // software pipeline: each thread holds two sources of the next tile
            // in registers while the current tile is computed; one barrier per tile
            constexpr int kPer = kNearTile / kNearThreads;
            double nx[kPer], nl[kPer];
            double nbase = sx[nd.m0];
            auto fetch = [&](int t0) {
#pragma unroll
                for (int i = 0; i < kPer; ++i) {
                    const int j = t0 + threadIdx.x + i * kNearThreads;
                    nx[i] = (j <= nd.m1) ? sx[j] : 0.0;
                    nl[i] = (j <= nd.m1) ? lam[j] : 0.0;
                }
                nbase = sx[t0];
            };
            fetch(nd.m0);
            int buf = 0;
            for (int t0 = nd.m0; t0 <= nd.m1; t0 += kNearTile, buf ^= 1) {
                const int cnt = min(kNearTile, nd.m1 - t0 + 1);
                const double base = nbase;
#pragma unroll
                for (int i = 0; i < kPer; ++i) {
                    const int k = threadIdx.x + i * kNearThreads;
                    // padding sources (q = 0, s = 0) complete the last pair
                    shb[buf][k] = (k < cnt) ? make_float2((float)(nx[i] - base), (float)(0.5 * nl[i]))
                                            : make_float2(0.f, 0.f);
                }
                __syncthreads();
                if (t0 + kNearTile <= nd.m1) fetch(t0 + kNearTile);
                float2 tau2[kNearR / 2], acc2[kNearR / 2], ncmp2[kNearR / 2];
#pragma unroll
                for (int h = 0; h < kNearR / 2; ++h) {
                    tau2[h] = make_float2((float)(xt[2 * h] - base), (float)(xt[2 * h + 1] - base));
                    acc2[h] = make_float2(0.f, 0.f);
                    ncmp2[h] = make_float2(0.f, 0.f);
                }
                const float4* pairs = reinterpret_cast<const float4*>(shb[buf]);
                const int npair = (cnt + 1) >> 1;
#pragma unroll 2
                for (int k = 0; k < npair; ++k) {
                    const float4 e4 = pairs[k];  // two sources per shared-memory load
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const float2 sx2 = u ? make_float2(e4.z, e4.z) : make_float2(e4.x, e4.x);
                        const float2 qh = u ? make_float2(e4.w, e4.w) : make_float2(e4.y, e4.y);
#pragma unroll
                        for (int h = 0; h < kNearR / 2; ++h) {
                            // differences as FMAs with -1 (exact products): no sign
                            // flips; Kahan with the negated compensation nc = -c
                            const float2 d = __ffma2_rn(sx2, m1, tau2[h]);
                            const float2 r2 = __ffma2_rn(d, d, e2v);
                            const float2 y = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                            const float2 g = __fmul2_rn(d, y);
                            const float2 v = __ffma2_rn(qh, g, ncmp2[h]);
                            const float2 sum = __fadd2_rn(acc2[h], v);
                            const float2 t = __ffma2_rn(acc2[h], m1, sum);
                            ncmp2[h] = __ffma2_rn(t, m1, v);
                            acc2[h] = sum;
                        }
                    }
                }
#pragma unroll
                for (int h = 0; h < kNearR / 2; ++h) {
                    fp[2 * h] += (double)acc2[h].x + (double)ncmp2[h].x;
                    fp[2 * h + 1] += (double)acc2[h].y + (double)ncmp2[h].y;
                }
            }
            __syncthreads();  // the general path and the next leaf reuse shared memory
        } else {
#pragma unroll 1
            for (int r = 0; r < kNearR; ++r)
                near_general(nd, x[r], sx, lam, pl, plx, L, band, cbg, eps2, a1, a2, shg, exact[r], fp[r], err);
        }
    }
#pragma unroll
    for (int r = 0; r < kNearR; ++r)
        if (jt[r] <= leaf.m1) apply_stage(A.S, A.sidx[jt[r]], A.efar[jt[r]] + A.norm * (exact[r] + fp[r]));
}

// One CTA per (leaf, target block): grid (leaf capacity, blocks per leaf).
__global__ void __launch_bounds__(kNearThreads) k_near32(NearArgs A) {
    __shared__ float4 shg[kNearTile];          // general path: {s, lambda/2, lambda/2 a1, lambda/2 a2}
    __shared__ __align__(16) float2 shb[2][kNearTile];  // band path: {s, lambda/2}, double-buffered
    near_item(A, blockIdx.x, blockIdx.y, shg, shb);
}

// Work of item i = l * nyb + yb: its targets times the sources of its leaf's
// near list (0 for items beyond the tree's leaves or their points).
__global__ void k_near_cost(NearArgs A, int nitems, int nyb, unsigned* __restrict__ cost, int* __restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const int l = i / nyb, yb = i - l * nyb;
    unsigned c = 0;
    if (l < A.meta[1] && !A.meta[2]) {
        const TNode leaf = A.nodes[A.leaves[l]];
        const int tb0 = leaf.m0 + yb * kNearBlock;
        if (tb0 <= leaf.m1) {
            const int nt = min(kNearBlock, leaf.m1 - tb0 + 1);
            long long ns = 0;
            for (int q = 0; q < A.near_n[l]; ++q) {
                const TNode nd = A.nodes[A.near_list[(size_t)l * kNearCap + q]];
                ns += nd.m1 - nd.m0 + 1;
            }
            c = (unsigned)min((long long)nt * ns / 64 + 1, (long long)UINT_MAX);
        }
    }
    cost[i] = c;
    ids[i] = i;
}

// Persistent: a one-wave grid takes items from an atomic counter in the order
// `order` gives (most work first), so that the launch does not end on a
// leaf with a long near list; items of no work come last and are skipped.
__global__ void __launch_bounds__(kNearThreads) k_near32_persistent(NearArgs A, int nitems, int nyb,
                                                                     const int* __restrict__ order,
                                                                     int* __restrict__ counter) {
    __shared__ float4 shg[kNearTile];
    __shared__ __align__(16) float2 shb[2][kNearTile];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(counter, 1);
            s_item = k < nitems ? order[k] : -1;
        }
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item < 0) break;
        near_item(A, item / nyb, item % nyb, shg, shb);
    }
}

__global__ void k_mul(const double* __restrict__ a, const double* __restrict__ b, int n, double* __restrict__ c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] * b[i];
}

// near pairs + far cluster terms of this call
__global__ void k_count_work(const TNode* __restrict__ nodes, const int* __restrict__ meta,
                             const int* __restrict__ leaves, const int* __restrict__ far_n,
                             const int* __restrict__ near_list, const int* __restrict__ near_n, int P,
                             double* __restrict__ work) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= meta[1] || meta[2]) return;
    const TNode lf = nodes[leaves[l]];
    const double nt = lf.m1 - lf.m0 + 1;
    double ns = 0.0;
    for (int q = 0; q < near_n[l]; ++q) {
        const TNode nd = nodes[near_list[(size_t)l * kNearCap + q]];
        ns += nd.m1 - nd.m0 + 1;
    }
    atomicAdd(&work[0], nt * ns);
    atomicAdd(&work[1], nt * far_n[l] * (double)(P + 1));
}

__global__ void k_copy_meta_error(const int* __restrict__ meta, int* __restrict__ err) {
    if (meta[2]) atomicCAS(err, 0, meta[2]);
}

// k_moment_items for PP = degree + 1 Chebyshev nodes: compiled for each
// supported node count, so that its per-point arrays stay in registers.
template <bool kFast>
void launch_moment_items_t(int PP, int grid, cudaStream_t st, const TNode* nodes, const int* meta, int cap_nodes,
                           const int* item_start, int cap_items, int P, const double* consts, const double* sx,
                           const double* lam, double* partial) {
#define FS_MOMENT_CASE(n)                                                                                      \
    case n:                                                                                                   \
        k_moment_items<n, kFast><<<grid, 256, 0, st>>>(nodes, meta, cap_nodes, item_start, cap_items, P, consts, \
                                                       sx, lam, partial);                                     \
        break;
    switch (PP) {
        FS_MOMENT_CASE(2) FS_MOMENT_CASE(3) FS_MOMENT_CASE(4) FS_MOMENT_CASE(5) FS_MOMENT_CASE(6)
        FS_MOMENT_CASE(7) FS_MOMENT_CASE(8) FS_MOMENT_CASE(9) FS_MOMENT_CASE(10) FS_MOMENT_CASE(11)
        FS_MOMENT_CASE(12) FS_MOMENT_CASE(13) FS_MOMENT_CASE(14) FS_MOMENT_CASE(15) FS_MOMENT_CASE(16)
        FS_MOMENT_CASE(17)
        default:
            k_moment_items<0, kFast><<<grid, 256, 0, st>>>(nodes, meta, cap_nodes, item_start, cap_items, P, consts,
                                                           sx, lam, partial);
    }
#undef FS_MOMENT_CASE
}

void launch_moment_items(bool fast, int PP, int grid, cudaStream_t st, const TNode* nodes, const int* meta,
                         int cap_nodes, const int* item_start, int cap_items, int P, const double* consts,
                         const double* sx, const double* lam, double* partial) {
    if (fast && kFastMoments)
        launch_moment_items_t<true>(PP, grid, st, nodes, meta, cap_nodes, item_start, cap_items, P, consts, sx, lam,
                                    partial);
    else
        launch_moment_items_t<false>(PP, grid, st, nodes, meta, cap_nodes, item_start, cap_items, P, consts, sx, lam,
                                     partial);
}

class Treecode final : public FieldEngine {
   public:
    Treecode(double L, double eps, double mac, int degree, int max_source, bool fp32_near)
        : L_(L), eps_(eps), mac_(mac), P_(degree), N0_(max_source), fp32_(fp32_near) {
        if (degree < 1 || degree > kMaxDegree) fail(FS_ERR_ARG, "treecode degree must be 1..16");
        if (max_source < 2) fail(FS_ERR_ARG, "treecode max_source must be >= 2");
        // Chebyshev points and barycentric weights exactly as the reference
        // forms them (pi constant and expressions of :790-806), on the host.
        const double pi = 3.14159265358979323846;
        const double h = pi / P_;
        std::vector<double> c(2 * (kMaxDegree + 1), 0.0);
        for (int i = 0; i <= P_; ++i) c[i] = std::cos(i * h);
        for (int j = 0; j <= P_; ++j) {
            const double dj = (j == 0 || j == P_) ? 0.5 : 1.0;
            c[kMaxDegree + 1 + j] = ((j % 2 == 0) ? 1 : -1) * dj;
        }
        consts_.ensure(c.size());
        FS_CUDA(cudaMemcpy(consts_.p, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
        FS_CUDA(cudaStreamSynchronize(nullptr));  // the copy lands before the engine's non-blocking streams read it
        norm_ = std::sqrt(L * L + 4 * eps * eps) / L;
        cbg_ = 1 / std::sqrt(L * L + 4 * eps * eps);
    }

    int* error_flag() override { return err_.p; }

    double actual_work(cudaStream_t st) override {
        if (last_pairs <= 0) return 0.0;
        FS_CUDA(cudaMemsetAsync(work_.p, 0, 2 * sizeof(double), st));
        k_count_work<<<(cap_leaves_ + 127) / 128, 128, 0, st>>>(nodes_.p, meta_.p, leaves_.p, far_n_.p, near_.p,
                                                                near_n_.p, P_, work_.p);
        FS_LAUNCHED(1);
        double h[2] = {0, 0};
        FS_CUDA(cudaMemcpyAsync(h, work_.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        FS_CUDA(cudaStreamSynchronize(st));
        prof_add_work("treecode_near_pairs", h[0]);
        prof_add_work("treecode_far_terms", h[1]);
        return h[0] + h[1];
    }

    void eval(const double* d_t, int nt, const double* d_s, const double* d_q, int ns, const Stage& stage,
              cudaStream_t st) override {
        (void)d_t;
        if (nt != ns) fail(FS_ERR_ARG, "treecode evaluates at the sources: nt must equal ns");
        last_pairs = (double)ns * (double)ns;
        if (ns <= 0) return;
        const int n = ns;
        const int cap_leaves = 2 * (n / N0_ + 1) + 16;
        const int cap_nodes = 2 * kMaxDepth * (n / N0_ + 1) + 64;
        const int cap_items = cap_nodes + (int)(((long long)n * (kMaxDepth + 1)) / kChunk) + 1;
        reserve(n, cap_nodes, cap_leaves, cap_items);
        cap_leaves_ = cap_leaves;
        const int T = 256;
        k_tree_keys<<<(n + T - 1) / T, T, 0, st>>>(d_s, n, L_, kin_.p, iin_.p);
        size_t tb = cub_.bytes();
        FS_CUDA(cub::DeviceRadixSort::SortPairs(cub_.p, tb, kin_.p, kout_.p, iin_.p, iout_.p, n, 0, 64, st));
        k_tree_gather<<<(n + T - 1) / T, T, 0, st>>>(kout_.p, iout_.p, d_q, n, sx_.p, lam_.p);
        k_build_tree<<<1, 1024, 0, st>>>(sx_.p, n, N0_, cap_nodes, cap_leaves, nodes_.p, leaves_.p, meta_.p);
        k_mark_leaves<<<cap_leaves, 256, 0, st>>>(nodes_.p, leaves_.p, meta_.p, leaf_of_.p);
        k_lists<<<(cap_leaves + 127) / 128, 128, 0, st>>>(nodes_.p, leaves_.p, meta_.p, L_, std::sqrt(mac_ * mac_),
                                                          far_.p, far_n_.p, near_.p, near_n_.p, err_.p);
        k_item_counts<<<(cap_nodes + T - 1) / T, T, 0, st>>>(nodes_.p, meta_.p, cap_nodes, counts_.p);
        tb = cub_.bytes();
        FS_CUDA(cub::DeviceScan::ExclusiveSum(cub_.p, tb, counts_.p, item_start_.p, cap_nodes, st));
        launch_moment_items(fp32_, P_ + 1, sm_count() * 8, st, nodes_.p, meta_.p, cap_nodes, item_start_.p, cap_items,
                            P_, consts_.p, sx_.p, lam_.p, mpart_.p);
        k_moment_reduce<<<(cap_nodes + T - 1) / T, T, 0, st>>>(nodes_.p, meta_.p, cap_nodes, item_start_.p, P_,
                                                              mpart_.p, mom_.p);
        k_copy_meta_error<<<1, 1, 0, st>>>(meta_.p, err_.p);
        if (!fp32_) {
            ProfScope prof("k_far_near64", st, last_pairs);
            k_far_near64<<<(n + 127) / 128, 128, 0, st>>>(nodes_.p, meta_.p, leaf_of_.p, leaves_.p, far_.p, far_n_.p,
                                                         near_.p, near_n_.p, mom_.p, consts_.p, sx_.p, lam_.p,
                                                         iout_.p, n, P_, L_, eps_, stage);
            FS_LAUNCHED(10);
        } else {
            {
                ProfScope prof("k_far32", st);
                k_far32<<<(n + 127) / 128, 128, 0, st>>>(nodes_.p, meta_.p, leaf_of_.p, far_.p, far_n_.p, mom_.p,
                                                        consts_.p, sx_.p, n, P_, L_, eps_, norm_, cbg_, efar_.p);
            }
            // leaves hold < max_source points: at most ceil(max_source/kNearBlock) target blocks each
            const int nyb = (N0_ + kNearBlock - 1) / kNearBlock;
            scan_f64_inclusive(lam_.p, pl_.p, n, scan_.p, st);
            k_mul<<<(n + T - 1) / T, T, 0, st>>>(lam_.p, sx_.p, n, lx_.p);
            scan_f64_inclusive(lx_.p, plx_.p, n, scan_.p, st);
            const NearArgs A{nodes_.p, meta_.p, leaves_.p, near_.p, near_n_.p, sx_.p, lam_.p, pl_.p, plx_.p, efar_.p,
                             iout_.p, L_, eps_, cbg_, norm_, stage, err_.p};
            if (kNearOrder) {
                // items in decreasing order of work, taken by a one-wave persistent grid
                const int nitems = cap_leaves * nyb;
                k_near_cost<<<(nitems + T - 1) / T, T, 0, st>>>(A, nitems, nyb, ncost_.p, nids_.p);
                size_t tbn = ntmp_.bytes();
                FS_CUDA(cub::DeviceRadixSort::SortPairsDescending(ntmp_.p, tbn, ncost_.p, ncost_.p + nitems,
                                                                  nids_.p, nids_.p + nitems, nitems, 0, 32, st));
                FS_CUDA(cudaMemsetAsync(ncounter_.p, 0, sizeof(int), st));
                if (!near_grid_) {
                    int per_sm = 0;
                    FS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_near32_persistent, kNearThreads,
                                                                          0));
                    near_grid_ = std::max(1, per_sm) * sm_count();
                }
                ProfScope prof("k_near32", st, last_pairs);
                k_near32_persistent<<<std::min(near_grid_, nitems), kNearThreads, 0, st>>>(A, nitems, nyb,
                                                                                          nids_.p + nitems,
                                                                                          ncounter_.p);
                FS_LAUNCHED(13);
            } else {
                ProfScope prof("k_near32", st, last_pairs);
                k_near32<<<dim3(cap_leaves, nyb), kNearThreads, 0, st>>>(A);
                FS_LAUNCHED(12);
            }
        }
    }

   private:

    void reserve(int n, int cap_nodes, int cap_leaves, int cap_items) {
        kin_.ensure(n);
        kout_.ensure(n);
        iin_.ensure(n);
        iout_.ensure(n);
        sx_.ensure(n);
        lam_.ensure(n);
        leaf_of_.ensure(n);
        efar_.ensure(n);
        if (fp32_) {
            pl_.ensure(n);
            plx_.ensure(n);
            lx_.ensure(n);
            scan_.ensure(scan_f64_scratch(n));
            const int nitems = cap_leaves * ((N0_ + kNearBlock - 1) / kNearBlock);
            ncost_.ensure(2 * (size_t)nitems);
            nids_.ensure(2 * (size_t)nitems);
            ncounter_.ensure(1);
            size_t b = 0;
            FS_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr,
                                                              (const int*)nullptr, (int*)nullptr, nitems, 0, 32));
            ntmp_.ensure(std::max<size_t>(b, 1));
        }
        nodes_.ensure(cap_nodes);
        leaves_.ensure(cap_leaves);
        meta_.ensure(4);
        work_.ensure(2);
        far_.ensure((size_t)cap_leaves * kFarCap);
        far_n_.ensure(cap_leaves);
        near_.ensure((size_t)cap_leaves * kNearCap);
        near_n_.ensure(cap_leaves);
        counts_.ensure(cap_nodes);
        item_start_.ensure(cap_nodes);
        mpart_.ensure((size_t)cap_items * (kMaxDegree + 1));
        mom_.ensure((size_t)cap_nodes * (kMaxDegree + 1));
        if (!err_.p) {
            err_.ensure(1);
            FS_CUDA(cudaMemset(err_.p, 0, sizeof(int)));
        }
        size_t need = 0, b = 0;
        FS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, (int*)nullptr,
                                                (int*)nullptr, n, 0, 64));
        need = std::max(need, b);
        FS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, cap_nodes));
        need = std::max(need, b);
        cub_.ensure(need);
    }

    double L_, eps_, mac_;
    int P_, N0_;
    bool fp32_;
    double norm_ = 1, cbg_ = 0;
    DevBuf<uint64_t> kin_, kout_;
    DevBuf<int> iin_, iout_, leaf_of_, leaves_, meta_, far_, far_n_, near_, near_n_, counts_, item_start_, err_;
    DevBuf<double> sx_, lam_, efar_, mpart_, mom_, consts_, pl_, plx_, lx_, work_, scan_;
    DevBuf<unsigned> ncost_;
    DevBuf<int> nids_, ncounter_;
    DevBuf<unsigned char> ntmp_;
    int near_grid_ = 0;
    int cap_leaves_ = 0;
    DevBuf<TNode> nodes_;
    DevBuf<unsigned char> cub_;
};

}  // namespace

FieldEngine* make_treecode(double L, double eps, double mac, int degree, int max_source, bool fp32_near) {
    return new Treecode(L, eps, mac, degree, max_source, fp32_near);
}

}  // namespace fsb
