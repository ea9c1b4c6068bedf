// Device-resident FARRSIGHT simulation: RK4 step, remesh, reduced-grid field.
//
// Host control flow follows AMRSimulation::step (src/simulation_files/AMRSimulation_step.cpp:5-99):
//   RK4 (3 field evaluations at stage positions, epilogues fused into the field
//   kernels) -> iter++, t += dt -> remesh + reduced-grid field every
//   remesh_period steps, otherwise a 4th field evaluation at the new positions.
// All species live in one concatenated SoA (x, p, f, q_w, E) in HBM, species
// ranges contiguous, so AMRSimulation::gather/scatter
// (AMRSimulation_gather_scatter.cpp:3-51) are index ranges, not copies.
//
// Remesh per species (AMRStructure::remesh, AMRStructure_amr.cpp:1156-1202):
//   k_panel_fit    one thread per old leaf: 9x9 LU fit of f about point 4
//                  (interpolate_from_panel_to_points, AMRStructure_interp.cpp:795-975)
//   k_shift        per point: periodic shift into the sheared root (shift_xs :429-491)
//   k_row_sort     per lattice row (one CTA): sort by shifted x, the order the
//                  reference's global sort gives (:525-558)
//   k_walk_first_column / k_walk_rows
//                  the reference's neighbour walk (find_leaf_containing_point_from_neighbor
//                  :12-230) in the reference's order: first point from the root,
//                  the first column sequentially, then one thread per row, each
//                  walk starting at the previous point's leaf.  In a strongly
//                  deformed (tangled) mesh a point can lie in more than one old
//                  panel, and only this order reproduces the reference's choice.
//   k_eval_points  per point: the located panel's fit or f_beyond_boundary
//   k_reset_points x,p <- lattice, f <- new f, q_w <- w0 * f
//                  (set_leaves_weights :1084-1151 with cached w0).
// Reduced grid (evaluate_field_uniform_grid, AMRSimulation_field.cpp:5-162,
// get_reduced_xs_ws AMRStructure.cpp:147-196): the lattice's unique x and the
// point->unique map are fixed, so they are cached; per remesh only the
// per-column charge sums (in the reference's summation order) are formed.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <filesystem>
#include <fstream>
#include <mutex>
#include <thread>
#include <array>
#include <map>
#include <memory>
#include <set>
#include <string>

#include "fs_device.cuh"

namespace fsb {

namespace {

constexpr int kT = 256;
// A walk keeps every panel it visited in its own kHist-int slice of global
// scratch (it stops at the first revisit, as the reference's visited set
// does); a walk longer than kHist panels stops with FS_ERR_WALK instead of
// forgetting where it has been.
constexpr int kHist = 1024;
// Walk length at which a walk gives up (<= kHist); fs_debug_set_wait_limits
// lowers it so that tests can drive FS_ERR_WALK.
__device__ int g_walk_limit = kHist;

__device__ __forceinline__ void raise_status(int* status, int code) { atomicCAS(status, 0, code); }

// ---------------------------------------------------------------- RK4 stage 1
// ef1 = E*qm, p2 = p + hdt*ef1, xk = x + hdt*v(p), accX = v(p), accP = ef1
// (AMRSimulation_step.cpp:148-165; v(p) = p unless the relativistic push is on).
__global__ void k_rk_stage1(int n, Stage S, double* __restrict__ e, double* __restrict__ xk) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const double ef = dmul(e[o], stage_qm(S, o));
    const double p1 = S.p[o];
    const double v1 = stage_v(S, o, p1);
    S.pst[o] = dadd(p1, dmul(S.hdt, ef));
    xk[o] = dadd(S.x[o], dmul(S.hdt, v1));
    S.accX[o] = v1;
    S.accP[o] = ef;
}

// ---------------------------------------------------------------- 9-point fit
// Row pivoting by the largest |a| (first on ties); the algorithm class of the
// reference's Eigen PartialPivLU (AMRStructure_interp.cpp:935).
// The 9x9 solve of one leaf, in the thread's own slice of shared memory (the
// partial pivoting swaps rows at run time; in registers that indexing would
// put the matrix in local memory, which for a leaf per thread spills to DRAM).
// A[i][j] = a[9 i + j]; b holds the right-hand side, then the solution.
// Partial pivoting by the largest |a| (first index on ties), the algorithm of
// Eigen's PartialPivLU (AMRStructure_interp.cpp:935), one rounding per
// operation.
__device__ void lu_solve9(double* a, double* b, int* perm) {
#pragma unroll
    for (int i = 0; i < 9; ++i) perm[i] = i;
    for (int k = 0; k < 9; ++k) {
        int piv = k;
        double best = fabs(a[9 * k + k]);
        for (int i = k + 1; i < 9; ++i) {
            const double v = fabs(a[9 * i + k]);
            if (v > best) {
                best = v;
                piv = i;
            }
        }
        if (piv != k) {
            for (int j = 0; j < 9; ++j) {
                const double t = a[9 * k + j];
                a[9 * k + j] = a[9 * piv + j];
                a[9 * piv + j] = t;
            }
            const int t = perm[k];
            perm[k] = perm[piv];
            perm[piv] = t;
        }
        if (best != 0.0)
            for (int i = k + 1; i < 9; ++i) a[9 * i + k] = ddiv(a[9 * i + k], a[9 * k + k]);
        for (int i = k + 1; i < 9; ++i)
            for (int j = k + 1; j < 9; ++j) a[9 * i + j] = dsub(a[9 * i + j], dmul(a[9 * i + k], a[9 * k + j]));
    }
    double y[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) y[i] = b[perm[i]];
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int i = k + 1; i < 9; ++i) y[i] = dsub(y[i], dmul(y[k], a[9 * i + k]));
#pragma unroll
    for (int k = 8; k >= 0; --k) {
        y[k] = ddiv(y[k], a[9 * k + k]);
#pragma unroll
        for (int i = 0; i < k; ++i) y[i] = dsub(y[i], dmul(y[k], a[9 * i + k]));
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) b[i] = y[i];
}

// Shared memory of one thread of k_panel_fit: the matrix, the right-hand side
// and the row permutation.
constexpr int kFitThreads = 64;
constexpr size_t kFitSmemPerThread = (81 + 9) * sizeof(double) + 9 * sizeof(int);

// Per leaf: the 9 old points' (x, p, f), the monomial basis
// {1, dx, dx dp, dp, dx^2, dx^2 dp, dx^2 dp^2, dx dp^2, dp^2} about point 4,
// and the 11-double fit record (9 coefficients, centre x, p)
// (interpolate_from_panel_to_points, AMRStructure_interp.cpp:795-975).
__global__ void __launch_bounds__(kFitThreads) k_panel_fit(int nleaves, const int* __restrict__ leaves,
                                                           const int* __restrict__ rec, const double* __restrict__ ox,
                                                           const double* __restrict__ op,
                                                           const double* __restrict__ of, double* __restrict__ coef) {
    extern __shared__ __align__(16) unsigned char fit_smem[];
    double* a = reinterpret_cast<double*>(fit_smem) + (size_t)threadIdx.x * 81;
    double* c = reinterpret_cast<double*>(fit_smem) + (size_t)kFitThreads * 81 + (size_t)threadIdx.x * 9;
    int* perm = reinterpret_cast<int*>(fit_smem + (size_t)kFitThreads * 90 * sizeof(double)) + threadIdx.x * 9;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nleaves) return;
    const int* r = rec + (size_t)leaves[l] * 18;
    double px[9], pp[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        px[i] = ox[r[i]];
        pp[i] = op[r[i]];
        c[i] = of[r[i]];
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const double dx = dsub(px[i], px[4]), dp = dsub(pp[i], pp[4]);
        a[9 * i + 0] = 1;
        a[9 * i + 1] = dx;
        a[9 * i + 2] = dmul(dx, dp);
        a[9 * i + 3] = dp;
        a[9 * i + 4] = dmul(dx, dx);
        a[9 * i + 5] = dmul(dmul(dx, dx), dp);
        a[9 * i + 6] = dmul(dmul(dmul(dx, dx), dp), dp);
        a[9 * i + 7] = dmul(dmul(dx, dp), dp);
        a[9 * i + 8] = dmul(dp, dp);
    }
    lu_solve9(a, c, perm);
    double* o = coef + (size_t)l * 11;
#pragma unroll
    for (int i = 0; i < 9; ++i) o[i] = c[i];
    o[9] = px[4];
    o[10] = pp[4];
}

struct MeshView {
    const int* rec;        // 18 ints per panel
    const int* leaf_slot;  // panel -> leaf slot (or -1)
    const double* lat_x;
    const double* lat_p;
    const double* coef;
    int npx, npp, n;
    double xmin, pmin, Lx, dxp, dpp;
    double f_beyond;
};

__device__ __forceinline__ bool edge_right(double x_tr, double p_tr, double x_br, double p_br, double tx, double tp) {
    return dmul(dsub(x_tr, x_br), dsub(tp, p_br)) > dmul(dsub(p_tr, p_br), dsub(tx, x_br));
}
__device__ __forceinline__ bool edge_left(double x_tl, double p_tl, double x_bl, double p_bl, double tx, double tp) {
    return dmul(dsub(x_tl, x_bl), dsub(tp, p_bl)) <= dmul(dsub(p_tl, p_bl), dsub(tx, x_bl));
}
__device__ __forceinline__ bool edge_top(double x_tr, double p_tr, double x_tl, double p_tl, double tx, double tp) {
    return dmul(dsub(x_tr, x_tl), dsub(tp, p_tl)) < dmul(dsub(p_tr, p_tl), dsub(tx, x_tl));
}
__device__ __forceinline__ bool edge_bottom(double x_br, double p_br, double x_bl, double p_bl, double tx, double tp) {
    return dmul(dsub(x_br, x_bl), dsub(tp, p_bl)) >= dmul(dsub(p_br, p_bl), dsub(tx, x_bl));
}

// find_leaf_containing_point_from_neighbor (AMRStructure_interp.cpp:12-230):
// starting at `leaf`, apply the half-open edge tests of the current panel and
// step to the neighbour across the first failed edge (right, top, bottom, left
// priority), shifting tx by Lx across the periodic seam; stop at the first
// panel already visited.  beyond_boundary is or-ed over every visited panel.
// Bounded: returns -1 when the walk would visit more than `cap` panels (cap
// <= the entries of hist).
__device__ int walk_from(const MeshView& M, const double* __restrict__ ox, const double* __restrict__ op,
                         double& tx, double tp, int leaf, bool& beyond, int* __restrict__ hist, int cap) {
    const double Lx = M.Lx;
    const int* R = M.rec;
    const int limit = cap;
    int nh = 0;
    hist[nh++] = leaf;
    for (;;) {
        if (leaf == 0) return 0;
        const int* P = R + (size_t)leaf * 18;
        const double x_bl = ox[P[0]], p_bl = op[P[0]];
        const double x_tl = ox[P[2]], p_tl = op[P[2]];
        const double x_mid = ox[P[4]];
        const double x_br = ox[P[6]], p_br = op[P[6]];
        const double x_tr = ox[P[8]], p_tr = op[P[8]];
        if (dsub(tx, x_mid) >= Lx / 2) tx = dsub(tx, Lx);
        if (dsub(tx, x_mid) < -Lx / 2) tx = dadd(tx, Lx);
        const bool ir = edge_right(x_tr, p_tr, x_br, p_br, tx, tp);
        const bool il = edge_left(x_tl, p_tl, x_bl, p_bl, tx, tp);
        const bool it = edge_top(x_tr, p_tr, x_tl, p_tl, tx, tp);
        const bool ib = edge_bottom(x_br, p_br, x_bl, p_bl, tx, tp);
        const int left = P[13], top = P[14], right = P[15], bottom = P[16], flags = P[17], parent = P[10];
        int nl = leaf;
        if (!ir && right != -2) {
            if (flags & 2) tx = dsub(tx, Lx);
            if (right == -1) nl = R[(size_t)parent * 18 + 15];
            else nl = (R[(size_t)right * 18 + 17] & 4) ? R[(size_t)right * 18 + 12] : right;
        } else if (!it && top != -2) {
            if (top == -1) nl = R[(size_t)parent * 18 + 14];
            else nl = (R[(size_t)top * 18 + 17] & 4) ? R[(size_t)top * 18 + 12] : top;
        } else if (!ib && bottom != -2) {
            if (bottom == -1) nl = R[(size_t)parent * 18 + 16];
            else nl = (R[(size_t)bottom * 18 + 17] & 4) ? R[(size_t)bottom * 18 + 12] + 1 : bottom;
        } else if (!il && left != -2) {
            if (flags & 1) tx = dadd(tx, Lx);
            if (left == -1) nl = R[(size_t)parent * 18 + 13];
            else nl = (R[(size_t)left * 18 + 17] & 4) ? R[(size_t)left * 18 + 12] + 2 : left;
        }
        if ((!ir && right == -2) || (!il && left == -2) || (!it && top == -2) || (!ib && bottom == -2))
            beyond = true;
        bool seen = false;
        for (int h = 0; h < nh; ++h) seen |= (hist[h] == nl);
        if (seen) return nl;
        if (nh >= limit) return -1;
        hist[nh++] = nl;
        leaf = nl;
    }
}

// find_leaf_containing_xp_recursively (AMRStructure_interp.cpp:232-426), used
// for the first point only; x is updated in place as in the reference.
__device__ int find_from_root(const MeshView& M, const double* __restrict__ ox, const double* __restrict__ op,
                              double& x, double p, bool& beyond) {
    const int* R = M.rec;
    const double Lx = M.Lx;
    int pi = 0;
    for (int depth = 0; depth < 64; ++depth) {
        const int* P = R + (size_t)pi * 18;
        const int flags = P[17], cs = P[12];
        const bool xp = flags & 4, pr = flags & 8;
        if (!(xp || pr)) {
            const double x_bl = ox[P[0]], p_bl = op[P[0]], x_tl = ox[P[2]], p_tl = op[P[2]];
            const double x_br = ox[P[6]], p_br = op[P[6]], x_tr = ox[P[8]], p_tr = op[P[8]];
            const bool ir = edge_right(x_tr, p_tr, x_br, p_br, x, p);
            const bool il = edge_left(x_tl, p_tl, x_bl, p_bl, x, p);
            const bool it = edge_top(x_tr, p_tr, x_tl, p_tl, x, p);
            const bool ib = edge_bottom(x_br, p_br, x_bl, p_bl, x, p);
            if ((!il && P[13] == -2) || (!ir && P[15] == -2) || (!it && P[14] == -2) || (!ib && P[16] == -2))
                beyond = true;
            return pi;
        }
        double xc[9], pc[9];
        for (int i = 0; i < 9; ++i) {
            xc[i] = ox[P[i]];
            pc[i] = op[P[i]];
        }
        // a >= b  <=>  (xa - xb)*(p - pb) >= (pa - pb)*(x - xb) style tests on the panel's mid lines
        auto ge = [&](int a, int b) { return dmul(dsub(xc[a], xc[b]), dsub(p, pc[b])) >= dmul(dsub(pc[a], pc[b]), dsub(x, xc[b])); };
        auto le = [&](int a, int b) { return dmul(dsub(xc[a], xc[b]), dsub(p, pc[b])) <= dmul(dsub(pc[a], pc[b]), dsub(x, xc[b])); };
        const bool i1b = ge(4, 1), i1r = ge(5, 4), i3b = ge(7, 4);
        const int* C = R;
        int sub;
        if (i1b && i1r) {
            const int c1 = cs + 1;
            const bool i1t = le(5, 2);
            if (i1t || C[(size_t)c1 * 18 + 14] < 0) {
                const bool i1l = le(2, 1);
                if (i1l || C[(size_t)c1 * 18 + 13] < 0) sub = c1;
                else {
                    sub = C[(size_t)c1 * 18 + 13];
                    if (flags & 1) x = dadd(x, Lx);
                }
            } else sub = C[(size_t)c1 * 18 + 14];
        } else if (i3b && !i1r) {
            const int c3 = pr ? cs + 1 : cs + 3;
            const bool i3t = le(8, 5);
            if (i3t || C[(size_t)c3 * 18 + 14] < 0) {
                const bool i3r = le(8, 7);
                if (!i3r || C[(size_t)c3 * 18 + 15] < 0) sub = c3;
                else {
                    sub = C[(size_t)c3 * 18 + 15];
                    if (flags & 2) x = dsub(x, Lx);
                }
            } else sub = C[(size_t)c3 * 18 + 14];
        } else {
            const bool i0r = ge(4, 3);
            if (i0r) {
                const int c0 = cs;
                const bool i0b = ge(3, 0);
                if (i0b || C[(size_t)c0 * 18 + 16] < 0) {
                    const bool i0l = le(1, 0);
                    if (i0l || C[(size_t)c0 * 18 + 13] < 0) sub = c0;
                    else {
                        sub = C[(size_t)c0 * 18 + 13];
                        if (flags & 1) x = dadd(x, Lx);
                    }
                } else sub = C[(size_t)c0 * 18 + 16];
            } else {
                const int c2 = pr ? cs : cs + 2;
                const bool i2b = ge(6, 3);
                if (i2b || C[(size_t)c2 * 18 + 16] < 0) {
                    const bool i2r = le(7, 6);
                    if (!i2r || C[(size_t)c2 * 18 + 15] < 0) sub = c2;
                    else {
                        sub = C[(size_t)c2 * 18 + 15];
                        if (flags & 2) x = dsub(x, Lx);
                    }
                } else sub = C[(size_t)c2 * 18 + 16];
            }
        }
        pi = sub;
    }
    return -1;
}

// shift_xs (AMRStructure_interp.cpp:429-491): lattice x -> the periodic image
// inside the sheared root panel (old points 0, 2, 6, 8).
__global__ void k_shift(int n, const double* __restrict__ lat_x, const double* __restrict__ lat_p, double Lx,
                        const double* __restrict__ ox, const double* __restrict__ op, double* __restrict__ sx,
                        int* __restrict__ status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double tp = lat_p[k];
    double tx = lat_x[k];
    const double x_bl = ox[0], p_bl = op[0], x_tl = ox[2], p_tl = op[2];
    const double x_br = ox[6], p_br = op[6], x_tr = ox[8], p_tr = op[8];
    int cnt = 0;
    while (!edge_left(x_tl, p_tl, x_bl, p_bl, tx, tp)) {
        tx = dadd(tx, Lx);
        if (++cnt > 10) {
            raise_status(status, FS_ERR_SHIFT);
            break;
        }
    }
    cnt = 0;
    while (!edge_right(x_tr, p_tr, x_br, p_br, tx, tp)) {
        tx = dsub(tx, Lx);
        if (++cnt > 10) {
            raise_status(status, FS_ERR_SHIFT);
            break;
        }
    }
    sx[k] = tx;
}

// The reference sorts all points by p row, then shifted x (AMRStructure_interp.cpp:525-558).
// Lattice rows are separated by far more than the sort threshold, so this is a
// per-row sort by (shifted x, point index): one CTA per row, bitonic sort in
// shared memory.  Writes sorted x, p and the point index of each sorted slot.
__global__ void k_row_sort(int nx, int pow2, const int* __restrict__ row_pts, const double* __restrict__ sx,
                           const double* __restrict__ lat_p, double* __restrict__ sortx, double* __restrict__ sortp,
                           int* __restrict__ order) {
    extern __shared__ unsigned char smem_raw[];
    double* kx = reinterpret_cast<double*>(smem_raw);
    int* ki = reinterpret_cast<int*>(kx + pow2);
    const int row = blockIdx.x;
    for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
        if (t < nx) {
            const int pt = row_pts[(size_t)row * nx + t];
            kx[t] = sx[pt];
            ki[t] = pt;
        } else {
            kx[t] = INFINITY;
            ki[t] = INT_MAX;
        }
    }
    __syncthreads();
    for (int size = 2; size <= pow2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
                const int u = t ^ stride;
                if (u > t) {
                    const bool up = ((t & size) == 0);
                    const bool gt = (kx[t] > kx[u]) || (kx[t] == kx[u] && ki[t] > ki[u]);
                    if (gt == up) {
                        const double a = kx[t];
                        kx[t] = kx[u];
                        kx[u] = a;
                        const int b = ki[t];
                        ki[t] = ki[u];
                        ki[u] = b;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < nx; t += blockDim.x) {
        const size_t o = (size_t)row * nx + t;
        sortx[o] = kx[t];
        sortp[o] = lat_p[ki[t]];
        order[o] = ki[t];
    }
}

// First point from the root, then the first column row by row, each walk
// starting where the previous one ended (AMRStructure_interp.cpp:608-650).
// One thread: the reference's dependency chain.
__global__ void k_walk_first_column(MeshView M, int nx, int np, const double* __restrict__ ox,
                                    const double* __restrict__ op, double* __restrict__ sortx,
                                    const double* __restrict__ sortp, int* __restrict__ first_col,
                                    int* __restrict__ leaf_of, int* __restrict__ hist, int* __restrict__ status) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    bool beyond = false;
    int leaf = find_from_root(M, ox, op, sortx[0], sortp[0], beyond);
    if (leaf < 0) {
        raise_status(status, FS_ERR_WALK);
        return;
    }
    for (int ii = 0; ii < np; ++ii) {
        const int pt = ii * nx;
        beyond = false;
        double tx = sortx[pt];
        leaf = walk_from(M, ox, op, tx, sortp[pt], leaf, beyond, hist, min(g_walk_limit, kHist));
        if (leaf < 0) {
            raise_status(status, FS_ERR_WALK);
            return;
        }
        sortx[pt] = tx;
        first_col[ii] = leaf;
        leaf_of[pt] = beyond ? 0 : leaf;
    }
}

// Every row: walk its sorted points left to right, each from the previous
// point's leaf (AMRStructure_interp.cpp:689-722).  One thread per row.
__global__ void k_walk_rows(MeshView M, int nx, int np, const double* __restrict__ ox, const double* __restrict__ op,
                            double* __restrict__ sortx, const double* __restrict__ sortp,
                            const int* __restrict__ first_col, int* __restrict__ leaf_of, int* __restrict__ hist,
                            int* __restrict__ status) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= np) return;
    int lc = first_col[ii];
    for (int jj = 1; jj < nx; ++jj) {
        const int pt = ii * nx + jj;
        bool beyond = false;
        double tx = sortx[pt];
        lc = walk_from(M, ox, op, tx, sortp[pt], lc, beyond, hist + (size_t)ii * kHist, min(g_walk_limit, kHist));
        if (lc < 0) {
            raise_status(status, FS_ERR_WALK);
            return;
        }
        sortx[pt] = tx;
        leaf_of[pt] = beyond ? 0 : lc;
    }
}

// ---------------------------------------------------------------- parallel point location
// The walks above form one chain per lattice row, hung from one chain down the
// first column: each point's walk starts at the leaf where the previous
// point's walk ended.  The same result is computed in parallel:
//   1. a guess of every point's leaf (k_leaf_xmid, k_guess): the leaf of the
//      old uniform mesh in the point's p-row whose centre is nearest in x;
//   2. every point's walk at once, each starting at the guess for its
//      predecessor (k_walk_spec), with a short local history;
//   3. a warp per chain (k_repair_column, then k_repair_rows) checks in order,
//      32 points at a time, that each walk started where its predecessor's
//      final walk ended, and walks again, with the full history, wherever it
//      did not.  Every final result is then a walk from the final result of
//      its predecessor: the chain's own result, whatever the guesses were.
// Used for species whose previous mesh is the uniform lattice mesh (every
// non-adaptive remesh); adaptive meshes keep the chain kernels above.
constexpr int kSpecHist = 32;  // local history of a speculative walk

// Centre x of every leaf of the old uniform mesh, by lattice cell (ip, ix).
__global__ void k_leaf_xmid(int ncell, const int* __restrict__ leaf_grid, const int* __restrict__ rec,
                            const double* __restrict__ ox, double* __restrict__ xmid) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    xmid[c] = ox[rec[(size_t)leaf_grid[c] * 18 + 4]];
}

// Guess of the old leaf holding each sorted slot: its p-row by p, then the
// leaf of that row whose centre is nearest in x, periodically; then a short
// walk from there (at most kGuessWalk panels) onto the panel the edge tests
// select -- lattice points on a row boundary belong to the row above or
// below depending on how the old boundary moved.
constexpr int kGuessWalk = 8;
__global__ void k_guess(MeshView M, const double* __restrict__ ox, const double* __restrict__ op, int n,
                        const double* __restrict__ sortx, const double* __restrict__ sortp, double pmin,
                        double dpp, int npx, int npp, double Lx, const double* __restrict__ xmid,
                        const int* __restrict__ leaf_grid, int* __restrict__ guess) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int ip = (int)floor((sortp[k] - pmin) / dpp);
    ip = min(max(ip, 0), npp - 1);
    const double* xm = xmid + (size_t)ip * npx;
    const double x0 = xm[0];
    double u = sortx[k] - x0;
    u -= Lx * floor(u / Lx);
    int lo = 0, hi = npx;  // first ix with xm[ix] - x0 > u
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (xm[mid] - x0 <= u) lo = mid + 1;
        else hi = mid;
    }
    int ix = lo - 1;  // xm[ix] - x0 <= u < xm[ix + 1] - x0
    if (ix < 0) ix = 0;
    const double right = (ix + 1 < npx) ? (xm[ix + 1] - x0) : Lx;
    if (right - u < u - (xm[ix] - x0)) ix = (ix + 1) % npx;
    const int g = leaf_grid[(size_t)ip * npx + ix];
    int hist[kGuessWalk];
    bool beyond = false;
    double tx = sortx[k];
    const int w = walk_from(M, ox, op, tx, sortp[k], g, beyond, hist, min(kGuessWalk, g_walk_limit));
    guess[k] = w >= 0 ? w : g;
}

// Every sorted slot's walk from the guess for its predecessor (slot 0: from
// the root search, as the chain does).  Writes the walk's end leaf R, the
// start it used S (-2: the walk did not finish within the local history or
// the walk bound, so the repair walks it again), its beyond-boundary flag B
// and its x after the periodic shifts TX.
__global__ void k_walk_spec(MeshView M, int nx, int n, const double* __restrict__ ox, const double* __restrict__ op,
                            const double* __restrict__ sortx, const double* __restrict__ sortp,
                            const int* __restrict__ guess, int* __restrict__ wR, int* __restrict__ wS,
                            int* __restrict__ wB, double* __restrict__ wTX, int* __restrict__ root_leaf,
                            double* __restrict__ root_x, int* __restrict__ status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double tx = sortx[k];
    int start;
    if (k == 0) {
        bool bb = false;
        start = find_from_root(M, ox, op, tx, sortp[0], bb);
        root_leaf[0] = start;
        root_x[0] = tx;
        if (start < 0) {
            raise_status(status, FS_ERR_WALK);
            wR[0] = 0;
            wS[0] = -2;
            wB[0] = 0;
            wTX[0] = tx;
            return;
        }
    } else {
        start = (k % nx == 0) ? guess[k - nx] : guess[k - 1];
    }
    int hist[kSpecHist];
    bool beyond = false;
    const int r = walk_from(M, ox, op, tx, sortp[k], start, beyond, hist, min(kSpecHist, g_walk_limit));
    wR[k] = r < 0 ? start : r;
    wS[k] = r < 0 ? -2 : start;
    wB[k] = beyond ? 1 : 0;
    wTX[k] = tx;
}

// One warp walks a chain again where needed.  pos(i) is the slot of the i-th
// point of the chain (i = 0 .. len-1), start0 the leaf the chain starts from.
// Returns false after a walk error (status set).
__device__ bool repair_chain(const MeshView& M, const double* __restrict__ ox, const double* __restrict__ op,
                             const double* __restrict__ sortx, const double* __restrict__ sortp, int* wR, int* wS,
                             int* wB, double* wTX, int* __restrict__ hist, int* __restrict__ status, int first_slot,
                             int stride, int len, int start0, double x0_override, bool use_x0) {
    const int lane = threadIdx.x & 31;
    const int cap = min(g_walk_limit, kHist);
    int i = 0;
    while (i < len) {
        const int ii = i + lane;
        bool bad = false;
        if (ii < len) {
            const int k = first_slot + ii * stride;
            const int want = (ii == 0) ? start0 : wR[k - stride];
            bad = (wS[k] != want);
        }
        const unsigned m = __ballot_sync(0xffffffffu, bad);
        if (!m) {
            i += 32;
            continue;
        }
        const int f = i + __ffs(m) - 1;
        int ok = 1;
        if (lane == 0) {
            const int k = first_slot + f * stride;
            const int want = (f == 0) ? start0 : wR[k - stride];
            double tx = (f == 0 && use_x0) ? x0_override : sortx[k];
            bool beyond = false;
            const int r = walk_from(M, ox, op, tx, sortp[k], want, beyond, hist, cap);
            if (r < 0) {
                raise_status(status, FS_ERR_WALK);
                ok = 0;
            } else {
                wR[k] = r;
                wS[k] = want;
                wB[k] = beyond ? 1 : 0;
                wTX[k] = tx;
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        if (!ok) return false;
        i = f + 1;
    }
    return true;
}

// The first column: one warp.
__global__ void k_repair_column(MeshView M, int nx, int np, const double* __restrict__ ox,
                                const double* __restrict__ op, const double* __restrict__ sortx,
                                const double* __restrict__ sortp, int* wR, int* wS, int* wB, double* wTX,
                                const int* __restrict__ root_leaf, const double* __restrict__ root_x,
                                int* __restrict__ hist, int* __restrict__ status) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    if (root_leaf[0] < 0) return;  // the root search failed (status set)
    (void)repair_chain(M, ox, op, sortx, sortp, wR, wS, wB, wTX, hist, status, 0, nx, np, root_leaf[0], root_x[0],
                       true);
}

// Every row: one warp per row, then the row's final leaves (0 beyond the
// p-range) and shifted x.
__global__ void k_repair_rows(MeshView M, int nx, int np, const double* __restrict__ ox, const double* __restrict__ op,
                              double* __restrict__ sortx, const double* __restrict__ sortp, int* wR, int* wS, int* wB,
                              double* wTX, int* __restrict__ leaf_of, int* __restrict__ hist,
                              int* __restrict__ status) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= np) return;
    const int lane = threadIdx.x & 31;
    const int first = row * nx;
    // the first column failed: one read for the whole warp, so that no lane
    // leaves while the others enter the warp-wide scan
    int failed = (lane == 0) ? *(volatile int*)status : 0;
    failed = __shfl_sync(0xffffffffu, failed, 0);
    if (failed) return;
    const bool ok = repair_chain(M, ox, op, sortx, sortp, wR, wS, wB, wTX, hist + (size_t)row * kHist, status,
                                 first + 1, 1, nx - 1, wR[first], 0.0, false);
    if (!ok) return;
    for (int j = lane; j < nx; j += 32) {
        const int k = first + j;
        leaf_of[k] = wB[k] ? 0 : wR[k];
        sortx[k] = wTX[k];
    }
}

// Evaluate the located panel's fit (or f_beyond_boundary) at every sorted
// slot and scatter back to point order.
__global__ void k_eval_points(MeshView M, const double* __restrict__ sortx, const double* __restrict__ sortp,
                              const int* __restrict__ order, const int* __restrict__ leaf_of,
                              double* __restrict__ fnew) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M.n) return;
    const int leaf = leaf_of[k];
    const int slot = (leaf > 0) ? M.leaf_slot[leaf] : -1;
    double v;
    if (slot < 0) {
        v = M.f_beyond;
    } else {
        const double* c = M.coef + (size_t)slot * 11;
        const double dx = dsub(sortx[k], c[9]), dp = dsub(sortp[k], c[10]);
        const double dxsq = dmul(dx, dx), dpsq = dmul(dp, dp);
        const double D[9] = {1.0, dx, dmul(dx, dp), dp, dxsq, dmul(dxsq, dp), dmul(dxsq, dpsq), dmul(dx, dpsq), dpsq};
        v = 0.0;
        for (int j = 0; j < 9; ++j) v = dadd(v, dmul(D[j], c[j]));
    }
    fnew[order[k]] = v;
}

// interpolate_from_mesh (AMRStructure_interp.cpp:1094-1143) for the points an
// adaptive refinement adds: shift_xs, the recursive search from the root of
// the previous mesh, then its leaf's fit in the single-point expression
// (:1086-1088) with one rounding per operation.
__global__ void k_interp_points(MeshView M, const double* __restrict__ ox, const double* __restrict__ op, int n,
                                const double* __restrict__ px, const double* __restrict__ pp,
                                double* __restrict__ fout, int* __restrict__ status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double tp = pp[k];
    double tx = px[k];
    const double x_bl = ox[0], p_bl = op[0], x_tl = ox[2], p_tl = op[2];
    const double x_br = ox[6], p_br = op[6], x_tr = ox[8], p_tr = op[8];
    int cnt = 0;
    while (!edge_left(x_tl, p_tl, x_bl, p_bl, tx, tp)) {
        tx = dadd(tx, M.Lx);
        if (++cnt > 10) {
            raise_status(status, FS_ERR_SHIFT);
            fout[k] = 0.0;
            return;
        }
    }
    cnt = 0;
    while (!edge_right(x_tr, p_tr, x_br, p_br, tx, tp)) {
        tx = dsub(tx, M.Lx);
        if (++cnt > 10) {
            raise_status(status, FS_ERR_SHIFT);
            fout[k] = 0.0;
            return;
        }
    }
    bool beyond = false;
    const int leaf = find_from_root(M, ox, op, tx, tp, beyond);
    const int slot = (!beyond && leaf > 0) ? M.leaf_slot[leaf] : -1;
    if (slot < 0) {
        if (leaf < 0) raise_status(status, FS_ERR_WALK);
        fout[k] = M.f_beyond;
        return;
    }
    const double* c = M.coef + (size_t)slot * 11;
    const double dx = dsub(tx, c[9]), dp = dsub(tp, c[10]);
    double v = c[0];
    v = dadd(v, dmul(c[1], dx));
    v = dadd(v, dmul(dmul(c[2], dx), dp));
    v = dadd(v, dmul(c[3], dp));
    v = dadd(v, dmul(dmul(c[4], dx), dx));
    v = dadd(v, dmul(dmul(dmul(c[5], dx), dx), dp));
    v = dadd(v, dmul(dmul(dmul(dmul(c[6], dx), dx), dp), dp));
    v = dadd(v, dmul(dmul(dmul(c[7], dx), dp), dp));
    v = dadd(v, dmul(dmul(c[8], dp), dp));
    fout[k] = v;
}

// The new state of a remeshed species.  Skipped when an earlier kernel of the
// remesh reported a failure (status set), so that a failed remesh leaves the
// state it started from.
__global__ void k_reset_points(int n, const double* __restrict__ lat_x, const double* __restrict__ lat_p,
                               const double* __restrict__ w0, const double* __restrict__ fnew, double* __restrict__ x,
                               double* __restrict__ p, double* __restrict__ f, double* __restrict__ qw,
                               const int* __restrict__ status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    x[k] = lat_x[k];
    p[k] = lat_p[k];
    f[k] = fnew[k];
    qw[k] = dmul(w0[k], fnew[k]);
}

// reduced_ws[u] = sum of q_w over the points of unique x u, in point order
__global__ void k_column_sums(int nu, const int* __restrict__ off, const int* __restrict__ idx,
                              const double* __restrict__ qw, double* __restrict__ rw) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    double s = 0.0;
    for (int k = off[u]; k < off[u + 1]; ++k) s = dadd(s, qw[idx[k]]);
    rw[u] = s;
}

// E of every point from the reduced grid; skipped, like k_reset_points, after
// a failure earlier in the same remesh.
__global__ void k_scatter_reduced(int n, const int* __restrict__ inv, const double* __restrict__ re,
                                  double* __restrict__ e, const int* __restrict__ status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || *status) return;
    e[k] = re[inv[k]];
}

// Host-to-device copy that has landed when it returns.  cudaMemcpy from pageable
// memory may return once the data is staged, with the DMA still queued on the
// legacy default stream, which the library's non-blocking streams do not wait
// for; the legacy stream is synchronised before any kernel can read the data.
inline void h2d(void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    FS_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    FS_CUDA(cudaStreamSynchronize(nullptr));
}

template <class T>
void upload(DevBuf<T>& b, const std::vector<T>& h) {
    b.ensure(h.size());
    h2d(b.p, h.data(), sizeof(T) * h.size());
}

inline int blocks(int n, int per = kT) { return (n + per - 1) / per; }

}  // namespace

struct SpeciesState {
    HostMesh mesh;       // current mesh (uniform, or refined adaptively)
    HostMesh base_mesh;  // the uniform mesh (adaptive species)
    bool adaptive = false;
    int max_height = 0, neps = 0;
    double eps[5] = {0, 0, 0, 0, 0};
    int nbase = 0;       // lattice points: the first nbase points of the species
    int start = 0, n = 0;
    double q = 0, m = 0, qm = 0, f_beyond = 0;
    int nleaves = 0, npx = 0, npp = 0;
    DevBuf<double> lat_x, lat_p, w0, coef, fnew;
    DevBuf<int> rec, leaf_slot, leaves, row_pts;
    DevBuf<double> sx, sortx, sortp;
    DevBuf<int> order, leaf_of, first_col, walk_hist;
    int nxl = 0, npl = 0, pow2 = 1;
    // parallel point location (uniform previous mesh): leaf of each lattice
    // cell, leaf centres, guesses and the speculative walks' results
    bool grid_ok = false;
    DevBuf<int> leaf_grid, wG, wR, wS, wB, wroot;
    DevBuf<double> xmid, wTX, wroot_x;
    // reduced grid
    int nu = 0, roff = 0;
    DevBuf<int> inv, col_off, col_idx;
};

// ------------------------------------------------------------------ diagnostic output
// The reference's dump files (AMRStructure_io.cpp:8-101, AMRStructure_restart.cpp:33-98,
// AMRSimulation_field.cpp:81-111), under <sim_dir>simulation_output/:
//   <species>/xs/xs_<iter>, ps/ps_<iter>, fs/fs_<iter>    raw FP64, one per point
//   <species>/panels/leaf_point_inds_<iter>                int32 x 9 per leaf, leaf order
//   <species>/panels/full_tree_<iter>                      int64 count, then one
//       80-byte record per panel: index, level, parent, which child, 9 point
//       indices, left/top/right/bottom neighbours, first child (int32), then
//       left/right boundary, refined in xp / in p, needs refinement (int8), 3 pad
//   reduce_xs/xs_<iter>, reduced_es/es_<iter>              raw FP64, reduced grid
// Particle files are written every diag_phase_space_period steps (and at
// iteration 0), reduced-grid files at reduced evaluations (start, remesh) on
// multiples of diag_period.  The state is copied to pinned host memory on the
// simulation stream and a writer thread writes the files while the next steps
// run; two buffer sets alternate.
struct DiagOutput {
    // one full_tree record: 18 int32 (72 bytes), 5 int8 flags, 3 pad bytes
    static constexpr size_t kTreeRecord = 18 * sizeof(int32_t) + 8;
    static_assert(kTreeRecord == 80, "panel record layout");
    // What one dump writes for a species: its place in the state arrays and
    // the files of its mesh as it stood when the dump was queued.
    struct Species {
        std::string name;
        int start = 0, n = 0;
        std::vector<int32_t> leaf_inds;
        std::vector<unsigned char> tree;
    };
    struct Slot {
        double* host = nullptr;
        size_t cap = 0;  // doubles
        cudaEvent_t ev = nullptr;
        bool busy = false, particles = false, reduced = false;
        int iter = 0, N = 0, U = 0;
        std::vector<Species> sp;
    };
    std::string out;  // <sim_dir>simulation_output/
    std::vector<std::string> names;
    int diag_period = 1, phase_period = 1, device = 0;
    Slot slot[2];
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int> queue;
    bool stop = false;
    std::string error;

    ~DiagOutput() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (th.joinable()) th.join();
        for (auto& s : slot) {
            if (s.host) cudaFreeHost(s.host);
            if (s.ev) cudaEventDestroy(s.ev);
        }
    }

    void start() {
        for (auto& s : slot) FS_CUDA(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
        th = std::thread([this] { writer(); });
    }

    // The files of a mesh: leaf point indices and the full panel tree.
    static Species snapshot(const std::string& name, int start, int n, const HostMesh& M) {
        Species q;
        q.name = name;
        q.start = start;
        q.n = n;
        q.leaf_inds.reserve(M.leaves.size() * 9);
        for (int l : M.leaves)
            for (int k = 0; k < 9; ++k) q.leaf_inds.push_back(M.panels[l].pts[k]);
        q.tree.assign(8 + kTreeRecord * M.panels.size(), 0);
        const int64_t np = (int64_t)M.panels.size();
        std::memcpy(q.tree.data(), &np, 8);
        for (size_t i = 0; i < M.panels.size(); ++i) {
            const HostPanel& P = M.panels[i];
            const int32_t v[18] = {(int32_t)i, P.level, P.parent, P.which, P.pts[0], P.pts[1], P.pts[2],
                                   P.pts[3], P.pts[4], P.pts[5], P.pts[6], P.pts[7], P.pts[8], P.left,
                                   P.top, P.right, P.bottom, P.child};
            unsigned char* r = q.tree.data() + 8 + kTreeRecord * i;
            std::memcpy(r, v, sizeof(v));
            const int8_t b[5] = {(int8_t)(P.lb ? 1 : 0), (int8_t)(P.rb ? 1 : 0), (int8_t)(P.xp ? 1 : 0),
                                 (int8_t)(P.pr ? 1 : 0), (int8_t)(P.needs ? 1 : 0)};
            std::memcpy(r + sizeof(v), b, 5);
        }
        return q;
    }

    // Copy the state (N points) and the reduced grid (U values) for iteration
    // `iter` on `st`; `sp` describes the species.
    void enqueue(cudaStream_t st, int iter, bool particles, bool reduced, int N, int U, std::vector<Species> sp,
                 const double* x, const double* p, const double* f, const double* rx, const double* re) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !slot[0].busy || !slot[1].busy; });
        if (!error.empty()) fail(FS_ERR_STATE, "diagnostic output failed: " + error);
        const int k = slot[0].busy ? 1 : 0;
        Slot& S = slot[k];
        S.busy = true;
        lk.unlock();
        const size_t need = 3 * (size_t)N + 2 * (size_t)U;
        if (S.cap < need) {
            if (S.host) FS_CUDA(cudaFreeHost(S.host));
            S.host = nullptr;
            S.cap = 0;
            FS_CUDA(cudaHostAlloc((void**)&S.host, sizeof(double) * std::max<size_t>(need, 1), 0));
            S.cap = need;
        }
        S.iter = iter;
        S.particles = particles;
        S.reduced = reduced;
        S.N = N;
        S.U = U;
        S.sp = std::move(sp);
        const size_t n = sizeof(double) * (size_t)N, u = sizeof(double) * (size_t)U;
        if (particles) {
            FS_CUDA(cudaMemcpyAsync(S.host, x, n, cudaMemcpyDeviceToHost, st));
            FS_CUDA(cudaMemcpyAsync(S.host + N, p, n, cudaMemcpyDeviceToHost, st));
            FS_CUDA(cudaMemcpyAsync(S.host + 2 * (size_t)N, f, n, cudaMemcpyDeviceToHost, st));
        }
        if (reduced) {
            FS_CUDA(cudaMemcpyAsync(S.host + 3 * (size_t)N, rx, u, cudaMemcpyDeviceToHost, st));
            FS_CUDA(cudaMemcpyAsync(S.host + 3 * (size_t)N + U, re, u, cudaMemcpyDeviceToHost, st));
        }
        FS_CUDA(cudaEventRecord(S.ev, st));
        lk.lock();
        queue.push_back(k);
        cv.notify_all();
    }

    void flush() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return queue.empty() && !slot[0].busy && !slot[1].busy; });
        if (!error.empty()) {
            const std::string e = error;
            error.clear();
            fail(FS_ERR_STATE, "diagnostic output failed: " + e);
        }
    }

    static void write_file(const std::string& path, const void* data, size_t bytes) {
        std::filesystem::create_directories(std::filesystem::path(path).parent_path());
        std::ofstream o(path, std::ios::out | std::ios::binary);
        if (!o) throw std::runtime_error("unable to open " + path);
        o.write(static_cast<const char*>(data), (std::streamsize)bytes);
        if (!o.good()) throw std::runtime_error("error writing " + path);
    }

    void write_slot(const Slot& S) {
        const std::string it = std::to_string(S.iter);
        const size_t N = S.N;
        if (S.particles) {
            for (const auto& q : S.sp) {
                const std::string d = out + q.name + "/";
                write_file(d + "xs/xs_" + it, S.host + q.start, sizeof(double) * q.n);
                write_file(d + "ps/ps_" + it, S.host + N + q.start, sizeof(double) * q.n);
                write_file(d + "fs/fs_" + it, S.host + 2 * N + q.start, sizeof(double) * q.n);
                write_file(d + "panels/leaf_point_inds_" + it, q.leaf_inds.data(), sizeof(int32_t) * q.leaf_inds.size());
                write_file(d + "panels/full_tree_" + it, q.tree.data(), q.tree.size());
            }
        }
        if (S.reduced) {
            write_file(out + "reduce_xs/xs_" + it, S.host + 3 * N, sizeof(double) * S.U);
            write_file(out + "reduced_es/es_" + it, S.host + 3 * N + S.U, sizeof(double) * S.U);
        }
    }

    void writer() {
        cudaSetDevice(device);
        for (;;) {
            int k;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                k = queue.front();
                queue.pop_front();
            }
            std::string err;
            if (cudaEventSynchronize(slot[k].ev) != cudaSuccess) {
                (void)cudaGetLastError();
                err = "copy to host failed";
            } else {
                try {
                    write_slot(slot[k]);
                } catch (const std::exception& e) {
                    err = e.what();
                }
            }
            std::lock_guard<std::mutex> lk(mu);
            if (!err.empty() && error.empty()) error = err;
            slot[k].busy = false;
            cv.notify_all();
        }
    }
};

// Drive-field amplitude at time t (src/FieldStructure.cpp:15-96): ExternalTanh
// (type 0, its factor k included) switches on around t = 69 and off around
// t = 307 with widths 20, normalised to start from zero at t = 0; ExternalSine
// (1) ramps up to t = 50, holds to 150 and ramps down to 200; ExternalLogistic
// (2) switches on at t = 10 and off at t = 110.  Host double arithmetic in the
// reference's expression order.
double tanh_switch(double t) { return 0.5 * (std::tanh((t - 69.0) / 20.0) - std::tanh((t - 307.0) / 20.0)); }
double drive_amplitude(int type, double Am, double k, double t) {
    if (type == 1) {
        if (t < 50.0) return Am * std::sin(t * M_PI / 100);
        if (t < 150.0) return Am;
        if (t < 200.0) return Am * std::cos((t - 150) * M_PI / 100);
        return 0.0;
    }
    if (type == 2) {
        if (t < 60.0) return Am / (1.0 + std::exp(-40.0 * (t - 10.0)));
        return Am * (1.0 - 1.0 / (1.0 + std::exp(-40.0 * (t - 110.0))));
    }
    const double e0 = tanh_switch(0.0);
    return (tanh_switch(t) - e0) / (1 - e0) * Am * k;
}

struct Sim {
    fs_sim_params prm{};
    int N = 0, U = 0, iter = 0;
    double L = 0, t = 0, pairs = 0, evals = 0;
    std::vector<std::unique_ptr<SpeciesState>> sp;
    DevBuf<double> x, p, f, qw, e, xkA, xkB, pst, accX, accP, rx, rw, re;
    DevBuf<int> status;
    std::unique_ptr<FieldEngine> field;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<double> step_ms;
    Stage base;

    bool own_stream = true;
    std::unique_ptr<DiagOutput> out;
    int last_reduced_iter = 0;  // iteration of the last reduced-grid evaluation

    ~Sim() {
        out.reset();  // writes what is queued
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st && own_stream) cudaStreamDestroy(st);
    }

    void check_status() {
        FS_CUDA(cudaStreamSynchronize(st));
        int h = 0;
        FS_CUDA(cudaMemcpy(&h, status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (h == 0 && field) {
            if (int* fe = field_error_flag(field.get())) {
                FS_CUDA(cudaMemcpy(&h, fe, sizeof(int), cudaMemcpyDeviceToHost));
                if (h) FS_CUDA(cudaMemset(fe, 0, sizeof(int)));
            }
        }
        if (h) {
            FS_CUDA(cudaMemset(status.p, 0, sizeof(int)));
            fail((fs_status)h, h == FS_ERR_WALK    ? "remesh point location did not converge"
                               : h == FS_ERR_SHIFT ? "remesh: too many periodic shifts"
                                                   : "device wait timed out");
        }
    }

    // Panel records, leaf list and leaf slots of the species' current mesh.
    void upload_mesh(SpeciesState& ss) {
        const HostMesh& M = ss.mesh;
        std::vector<int> rec(M.panels.size() * 18);
        M.panel_records(rec.data());
        upload(ss.rec, rec);
        upload(ss.leaves, M.leaves);
        std::vector<int> slot(M.panels.size(), -1);
        for (size_t l = 0; l < M.leaves.size(); ++l) slot[M.leaves[l]] = (int)l;
        upload(ss.leaf_slot, slot);
        ss.nleaves = (int)M.leaves.size();
        ss.coef.ensure((size_t)ss.nleaves * 11);
        // lattice cell of every leaf when the mesh is the uniform npx x npp one
        // (each leaf covers the 3 x 3 lattice points from (2 ix, 2 ip))
        ss.grid_ok = false;
        if (!ss.adaptive && ss.npx > 0 && ss.npp > 0 && (int)M.leaves.size() == ss.npx * ss.npp) {
            const double hx = (M.xmax - M.xmin) / ss.npx / 2, hp = (M.pmax - M.pmin) / ss.npp / 2;
            std::vector<int> grid((size_t)ss.npx * ss.npp, -1);
            bool ok = true;
            for (int l : M.leaves) {
                const int* r = &rec[(size_t)l * 18];
                const double c0 = (M.xs[r[0]] - M.xmin) / hx, r0 = (M.ps[r[0]] - M.pmin) / hp;
                const double c8 = (M.xs[r[8]] - M.xmin) / hx, r8 = (M.ps[r[8]] - M.pmin) / hp;
                const long ic = std::lround(c0), ir = std::lround(r0);
                if (std::fabs(c0 - ic) > 1e-6 || std::fabs(r0 - ir) > 1e-6 || std::fabs(c8 - (ic + 2)) > 1e-6 ||
                    std::fabs(r8 - (ir + 2)) > 1e-6 || (ic & 1) || (ir & 1)) {
                    ok = false;
                    break;
                }
                const long ix = ic / 2, ip = ir / 2;
                if (ix < 0 || ix >= ss.npx || ip < 0 || ip >= ss.npp || grid[(size_t)ip * ss.npx + ix] != -1) {
                    ok = false;
                    break;
                }
                grid[(size_t)ip * ss.npx + ix] = l;
            }
            if (ok) {
                upload(ss.leaf_grid, grid);
                ss.xmid.ensure(grid.size());
                ss.grid_ok = true;
            }
        }
    }

    // Reduced grid of a species (get_reduced_xs_ws, AMRStructure.cpp:147-185):
    // unique x strictly increasing, point -> unique map (global, offset by
    // ss.roff), per-unique point lists in ascending point index.  Returns the
    // unique x.
    std::vector<double> reduced_maps(SpeciesState& ss, const std::vector<double>& xs) {
        const int n = ss.n;
        std::vector<int> order(n);
        for (int i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return xs[a] < xs[b]; });
        std::vector<int> inv(n);
        std::vector<double> ux;
        double val = xs[order[0]];
        ux.push_back(val);
        inv[order[0]] = 0;
        for (int k = 1; k < n; ++k) {
            const double v = xs[order[k]];
            if (v > val) {
                val = v;
                ux.push_back(v);
            }
            inv[order[k]] = (int)ux.size() - 1;
        }
        ss.nu = (int)ux.size();
        std::vector<int> off(ss.nu + 1, 0), idx(n);
        for (int i = 0; i < n; ++i) off[inv[i] + 1]++;
        for (int u = 0; u < ss.nu; ++u) off[u + 1] += off[u];
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (int i = 0; i < n; ++i) idx[fill[inv[i]]++] = i;
        std::vector<int> inv_global(n);
        for (int i = 0; i < n; ++i) inv_global[i] = inv[i] + ss.roff;
        upload(ss.inv, inv_global);
        upload(ss.col_off, off);
        upload(ss.col_idx, idx);
        return ux;
    }

    // Load the remesh kernels on this device at creation: with the CUDA
    // runtime's lazy module loading the first remesh would otherwise pay for
    // loading them (about 0.3-0.8 ms measured on a 0.4 ms remesh).
    static void preload_remesh_kernels(int device) {
        static std::mutex mu;
        static std::vector<int> done;
        std::lock_guard<std::mutex> lk(mu);
        if (std::find(done.begin(), done.end(), device) != done.end()) return;
        const void* fns[] = {(const void*)k_panel_fit,         (const void*)k_shift,
                             (const void*)k_row_sort,          (const void*)k_leaf_xmid,
                             (const void*)k_guess,             (const void*)k_walk_spec,
                             (const void*)k_repair_column,     (const void*)k_repair_rows,
                             (const void*)k_walk_first_column, (const void*)k_walk_rows,
                             (const void*)k_eval_points,       (const void*)k_reset_points};
        for (const void* f : fns) {
            cudaFuncAttributes a;
            FS_CUDA(cudaFuncGetAttributes(&a, f));
        }
        done.push_back(device);
    }

    void create(const fs_sim_params& P, cudaStream_t external = nullptr) {
        prm = P;
        if (P.num_species < 1 || P.num_species > 8) fail(FS_ERR_ARG, "num_species must be 1..8");
        if (!(P.xmax > P.xmin)) fail(FS_ERR_ARG, "xmax must exceed xmin");
        if (P.remesh_period < 1) fail(FS_ERR_ARG, "remesh_period must be >= 1");
        if (P.field_kind == FS_FIELD_DIRECT64_OPEN)
            fail(FS_ERR_UNSUPPORTED, "open boundaries are supported by the field plugin only, not by the session");
        if (P.use_external_field && (P.external_type < 0 || P.external_type > 2))
            fail(FS_ERR_ARG, "external_type must be 0 (tanh), 1 (sine) or 2 (logistic)");
        FS_CUDA(cudaSetDevice(P.device));
        preload_remesh_kernels(P.device);
        if (external) {
            st = external;
            own_stream = false;
        } else {
            FS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        }
        FS_CUDA(cudaEventCreate(&ev0));
        FS_CUDA(cudaEventCreate(&ev1));
        L = P.xmax - P.xmin;
        std::vector<double> hx, hp, hf, hqw;
        std::vector<double> hrx;
        base.nsp = P.num_species;
        for (int s = 0; s < P.num_species; ++s) {
            const fs_species_params& S = P.species[s];
            auto ss = std::make_unique<SpeciesState>();
            ss->mesh.build(S.initial_height, S.p_height, P.xmin, P.xmax, S.pmin, S.pmax);
            HostMesh& M = ss->mesh;
            ss->nbase = (int)M.xs.size();
            // initial condition (AMRStructure ctor / generate_mesh at the initial step)
            const InitialDistribution dist(S, P.xmin, P.xmax);
            std::vector<double> f0(M.xs.size());
            for (size_t i = 0; i < f0.size(); ++i) f0[i] = dist(M.xs[i], M.ps[i]);
            ss->adaptive = S.do_adaptively_refine && S.n_amr_eps > 0;
            if (ss->adaptive) {
                if (S.n_amr_eps > 5) fail(FS_ERR_ARG, "at most 5 amr_epsilons");
                ss->max_height = S.max_height;
                ss->neps = S.n_amr_eps;
                for (int k = 0; k < S.n_amr_eps; ++k) ss->eps[k] = S.amr_eps[k];
                ss->base_mesh = M;
                M.adapt(f0, ss->eps, ss->neps, ss->max_height,
                        [&](const double* x, const double* p, int n, double* out) {
                            for (int i = 0; i < n; ++i) out[i] = dist(x[i], p[i]);
                        });
            }
            ss->start = N;
            ss->n = (int)M.xs.size();
            ss->q = S.q;
            ss->m = S.m;
            ss->qm = S.q / S.m;
            ss->npx = 1 << S.initial_height;
            ss->npp = 1 << (S.initial_height + S.p_height);
            ss->nleaves = (int)M.leaves.size();
            base.start[s] = N;
            base.qm[s] = ss->qm;
            base.m[s] = ss->m;
            N += ss->n;
            // weights (set_leaves_weights)
            std::vector<double> w0 = M.base_weights(S.q, P.quadrature);
            double fmin = 0;
            for (int i = 0; i < ss->n; ++i) {
                const double fv = f0[i];
                hx.push_back(M.xs[i]);
                hp.push_back(M.ps[i]);
                hf.push_back(fv);
                hqw.push_back(w0[i] * fv);
                if (i == 0 || fv < fmin) fmin = fv;
            }
            ss->f_beyond = fmin;
            upload(ss->lat_x, std::vector<double>(M.xs.begin(), M.xs.begin() + ss->nbase));
            upload(ss->lat_p, std::vector<double>(M.ps.begin(), M.ps.begin() + ss->nbase));
            upload(ss->w0, w0);
            upload_mesh(*ss);
            // lattice rows (ascending p), each listing its points by column
            ss->nxl = M.nx();
            ss->npl = M.np();
            {
                const double hx = L / ss->npx / 2, hp = (S.pmax - S.pmin) / ss->npp / 2;
                std::vector<int> rows((size_t)ss->nxl * ss->npl, -1);
                for (int i = 0; i < ss->nbase; ++i) {
                    const int c = (int)std::lround((M.xs[i] - P.xmin) / hx);
                    const int r = (int)std::lround((M.ps[i] - S.pmin) / hp);
                    if (c < 0 || c >= ss->nxl || r < 0 || r >= ss->npl || rows[(size_t)r * ss->nxl + c] != -1)
                        fail(FS_ERR_STATE, "mesh points do not form the expected lattice");
                    rows[(size_t)r * ss->nxl + c] = i;
                }
                upload(ss->row_pts, rows);
            }
            while (ss->pow2 < ss->nxl) ss->pow2 <<= 1;
            if ((size_t)ss->pow2 * (sizeof(double) + sizeof(int)) > 200 * 1024)
                fail(FS_ERR_UNSUPPORTED, "mesh rows longer than the row sort supports");
            ss->sx.ensure(ss->nbase);
            ss->sortx.ensure(ss->nbase);
            ss->sortp.ensure(ss->nbase);
            ss->order.ensure(ss->nbase);
            ss->leaf_of.ensure(ss->nbase);
            ss->first_col.ensure(ss->npl);
            ss->walk_hist.ensure((size_t)ss->npl * kHist);
            for (DevBuf<int>* b : {&ss->wG, &ss->wR, &ss->wS, &ss->wB}) b->ensure(ss->nbase);
            ss->wTX.ensure(ss->nbase);
            ss->wroot.ensure(1);
            ss->wroot_x.ensure(1);
            ss->fnew.ensure(ss->nbase);
            ss->roff = U;
            const std::vector<double> ux = reduced_maps(*ss, M.xs);
            U += ss->nu;
            hrx.insert(hrx.end(), ux.begin(), ux.end());
            sp.push_back(std::move(ss));
        }
        base.start[P.num_species] = N;
        for (int s = P.num_species + 1; s < 9; ++s) base.start[s] = N;
        base.rel = P.relativistic_push ? 1 : 0;
        base.dt = P.dt;
        base.hdt = 0.5 * P.dt;
        base.dt6 = P.dt / 6.0;
        upload(x, hx);
        upload(p, hp);
        upload(f, hf);
        upload(qw, hqw);
        e.ensure(N);
        xkA.ensure(N);
        xkB.ensure(N);
        pst.ensure(N);
        accX.ensure(N);
        accP.ensure(N);
        upload(rx, hrx);
        rw.ensure(U);
        re.ensure(U);
        status.ensure(1);
        FS_CUDA(cudaMemset(status.p, 0, sizeof(int)));
        switch (P.field_kind) {
            case FS_FIELD_DIRECT64: field.reset(make_direct64(L, P.greens_epsilon)); break;
            case FS_FIELD_DIRECT32C: field.reset(make_direct32c(L, P.greens_epsilon)); break;
            case FS_FIELD_TREECODE64:
            case FS_FIELD_TREECODE32C:
                field.reset(make_treecode(L, P.greens_epsilon, P.mac, P.degree, P.max_source,
                                          P.field_kind == FS_FIELD_TREECODE32C));
                break;
            default: fail(FS_ERR_ARG, "unknown field kind");
        }
        base.x = x.p;
        base.p = p.p;
        base.pst = pst.p;
        base.accX = accX.p;
        base.accP = accP.p;
        reduced_field();  // AMRSimulation ctor: evaluate_field_uniform_grid(0)
        check_status();
    }

    // direct-equivalent pairs always; kernel-level evaluations when profiling
    void account() {
        pairs += field->last_pairs;
        evals += profiling_enabled() ? field->actual_work(st) : field->last_pairs;
    }

    Stage stage(int kind, double* xk_out) const {
        Stage S = base;
        S.kind = kind;
        S.xk = xk_out;
        return S;
    }

    // One field evaluation: targets == sources == x (n points), weights q.
    struct FieldCall {
        const double* x;
        int n;
        const double* q;
        Stage stage;
    };

    void run_call(const FieldCall& fc) {
        field->eval(fc.x, fc.n, fc.x, fc.q, fc.n, fc.stage, st);
        account();
    }

    // Reduced grid (evaluate_field_uniform_grid): column sums, one field call
    // on the unique x, scatter back to the points.
    void reduced_pre() {
        for (auto& s : sp) {
            k_column_sums<<<blocks(s->nu), kT, 0, st>>>(s->nu, s->col_off.p, s->col_idx.p, qw.p + s->start,
                                                       rw.p + s->roff);
        }
        FS_LAUNCHED((long long)sp.size());
    }
    // The drive field at time tc on the call's targets (evaluate_field and
    // evaluate_field_uniform_grid add it after the field).
    FieldCall with_drive(FieldCall fc, double tc) const {
        if (prm.use_external_field) {
            fc.stage.ext_x = fc.x;
            fc.stage.ext_a = drive_amplitude(prm.external_type, prm.external_Am, prm.external_k, tc);
            fc.stage.ext_k = prm.external_k;
            fc.stage.ext_omt = prm.external_omega * tc;
        }
        return fc;
    }
    FieldCall reduced_call() const {
        Stage S = base;
        S.kind = STAGE_STORE;
        S.out = re.p;
        return with_drive(FieldCall{rx.p, U, rw.p, S}, t);
    }
    void reduced_post() {
        for (auto& s : sp) {
            k_scatter_reduced<<<blocks(s->n), kT, 0, st>>>(s->n, s->inv.p, re.p, e.p + s->start, status.p);
        }
        FS_LAUNCHED((long long)sp.size());
    }
    void reduced_field() {
        last_reduced_iter = iter;
        reduced_pre();
        run_call(reduced_call());
        reduced_post();
    }

    // AMRStructure::remesh for every species (interpolation + weights).
    MeshView mesh_view(const SpeciesState& ss) const {
        MeshView M;
        M.rec = ss.rec.p;
        M.leaf_slot = ss.leaf_slot.p;
        M.lat_x = ss.lat_x.p;
        M.lat_p = ss.lat_p.p;
        M.coef = ss.coef.p;
        M.npx = ss.npx;
        M.npp = ss.npp;
        M.n = ss.nbase;
        M.xmin = prm.xmin;
        M.pmin = ss.mesh.pmin;
        M.Lx = L;
        M.dxp = L / ss.npx;
        M.dpp = (ss.mesh.pmax - ss.mesh.pmin) / ss.npp;
        M.f_beyond = ss.f_beyond;
        return M;
    }

    void remesh_kernels() {
        bool any_adaptive = false;
        long long launches = 0;
        for (auto& s : sp) {
            const int a = s->start;
            const int nb = s->nbase;
            ProfScope prof("remesh", st);
            k_panel_fit<<<blocks(s->nleaves, kFitThreads), kFitThreads, kFitThreads * kFitSmemPerThread, st>>>(
                s->nleaves, s->leaves.p, s->rec.p, x.p + a, p.p + a, f.p + a, s->coef.p);
            const MeshView M = mesh_view(*s);
            k_shift<<<blocks(nb), kT, 0, st>>>(nb, s->lat_x.p, s->lat_p.p, L, x.p + a, p.p + a, s->sx.p, status.p);
            const size_t smem = (size_t)s->pow2 * (sizeof(double) + sizeof(int));
            if (smem > 48 * 1024)
                FS_CUDA(cudaFuncSetAttribute(k_row_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_row_sort<<<s->npl, 512, smem, st>>>(s->nxl, s->pow2, s->row_pts.p, s->sx.p, s->lat_p.p, s->sortx.p,
                                                  s->sortp.p, s->order.p);
            if (s->grid_ok) {
                const int ncell = s->npx * s->npp;
                k_leaf_xmid<<<blocks(ncell), kT, 0, st>>>(ncell, s->leaf_grid.p, s->rec.p, x.p + a, s->xmid.p);
                k_guess<<<blocks(nb, 128), 128, 0, st>>>(M, x.p + a, p.p + a, nb, s->sortx.p, s->sortp.p, M.pmin,
                                                         M.dpp, s->npx, s->npp, L, s->xmid.p, s->leaf_grid.p, s->wG.p);
                k_walk_spec<<<blocks(nb, 128), 128, 0, st>>>(M, s->nxl, nb, x.p + a, p.p + a, s->sortx.p, s->sortp.p,
                                                             s->wG.p, s->wR.p, s->wS.p, s->wB.p, s->wTX.p, s->wroot.p,
                                                             s->wroot_x.p, status.p);
                k_repair_column<<<1, 32, 0, st>>>(M, s->nxl, s->npl, x.p + a, p.p + a, s->sortx.p, s->sortp.p,
                                                  s->wR.p, s->wS.p, s->wB.p, s->wTX.p, s->wroot.p, s->wroot_x.p,
                                                  s->walk_hist.p, status.p);
                k_repair_rows<<<blocks(s->npl, 4), 128, 0, st>>>(M, s->nxl, s->npl, x.p + a, p.p + a, s->sortx.p,
                                                                 s->sortp.p, s->wR.p, s->wS.p, s->wB.p, s->wTX.p,
                                                                 s->leaf_of.p, s->walk_hist.p, status.p);
                launches += 5;
            } else {
                k_walk_first_column<<<1, 32, 0, st>>>(M, s->nxl, s->npl, x.p + a, p.p + a, s->sortx.p, s->sortp.p,
                                                      s->first_col.p, s->leaf_of.p, s->walk_hist.p, status.p);
                k_walk_rows<<<blocks(s->npl, 64), 64, 0, st>>>(M, s->nxl, s->npl, x.p + a, p.p + a, s->sortx.p,
                                                               s->sortp.p, s->first_col.p, s->leaf_of.p,
                                                               s->walk_hist.p, status.p);
                launches += 2;
            }
            k_eval_points<<<blocks(nb), kT, 0, st>>>(M, s->sortx.p, s->sortp.p, s->order.p, s->leaf_of.p,
                                                     s->fnew.p);
            launches += 4;  // fit, shift, row sort, evaluation
            if (s->adaptive) {
                any_adaptive = true;  // f at the lattice stays in fnew; the old state is still needed
            } else {
                k_reset_points<<<blocks(nb), kT, 0, st>>>(nb, s->lat_x.p, s->lat_p.p, s->w0.p, s->fnew.p, x.p + a,
                                                         p.p + a, f.p + a, qw.p + a, status.p);
                launches += 1;
            }
        }
        FS_LAUNCHED(launches);
        if (any_adaptive) adaptive_remesh();
    }

    // generate_mesh after a step for adaptive species (AMRStructure_amr.cpp:841-941):
    // the lattice values from the walk, then refinement passes on the host whose
    // new points are interpolated on the device from the previous mesh.  The
    // point counts change, so the state is laid out again.
    void adaptive_remesh() {
        check_status();
        const int ns = (int)sp.size();
        std::vector<std::vector<double>> hx(ns), hp(ns), hf(ns), hq(ns);
        DevBuf<double> dx, dp, df;
        for (int k = 0; k < ns; ++k) {
            SpeciesState& S = *sp[k];
            const int a = S.start;
            if (!S.adaptive) {
                for (auto* v : {&hx[k], &hp[k], &hf[k], &hq[k]}) v->resize(S.n);
                FS_CUDA(cudaMemcpy(hx[k].data(), x.p + a, 8 * (size_t)S.n, cudaMemcpyDeviceToHost));
                FS_CUDA(cudaMemcpy(hp[k].data(), p.p + a, 8 * (size_t)S.n, cudaMemcpyDeviceToHost));
                FS_CUDA(cudaMemcpy(hf[k].data(), f.p + a, 8 * (size_t)S.n, cudaMemcpyDeviceToHost));
                FS_CUDA(cudaMemcpy(hq[k].data(), qw.p + a, 8 * (size_t)S.n, cudaMemcpyDeviceToHost));
                continue;
            }
            std::vector<double> fv(S.nbase);
            FS_CUDA(cudaMemcpy(fv.data(), S.fnew.p, 8 * (size_t)S.nbase, cudaMemcpyDeviceToHost));
            HostMesh nm = S.base_mesh;
            const MeshView M = mesh_view(S);
            nm.adapt(fv, S.eps, S.neps, S.max_height, [&](const double* xs, const double* ps, int n, double* out) {
                dx.ensure(n);
                dp.ensure(n);
                df.ensure(n);
                h2d(dx.p, xs, 8 * (size_t)n);
                h2d(dp.p, ps, 8 * (size_t)n);
                k_interp_points<<<blocks(n), kT, 0, st>>>(M, x.p + a, p.p + a, n, dx.p, dp.p, df.p, status.p);
                FS_LAUNCHED(1);
                check_status();
                FS_CUDA(cudaMemcpy(out, df.p, 8 * (size_t)n, cudaMemcpyDeviceToHost));
            });
            const std::vector<double> w = nm.base_weights(S.q, prm.quadrature);
            hq[k].resize(nm.xs.size());
            for (size_t i = 0; i < nm.xs.size(); ++i) hq[k][i] = w[i] * fv[i];
            hx[k] = nm.xs;
            hp[k] = nm.ps;
            hf[k] = std::move(fv);
            S.mesh = std::move(nm);
            upload(S.w0, w);
        }
        relayout(hx, hp, hf, hq);
    }

    // Lay the species' states out again after their point counts changed.
    void relayout(const std::vector<std::vector<double>>& hx, const std::vector<std::vector<double>>& hp,
                  const std::vector<std::vector<double>>& hf, const std::vector<std::vector<double>>& hq) {
        const int ns = (int)sp.size();
        std::vector<double> ax, ap, af, aq, arx;
        N = 0;
        U = 0;
        for (int k = 0; k < ns; ++k) {
            SpeciesState& S = *sp[k];
            S.start = N;
            S.n = (int)hx[k].size();
            base.start[k] = N;
            N += S.n;
            ax.insert(ax.end(), hx[k].begin(), hx[k].end());
            ap.insert(ap.end(), hp[k].begin(), hp[k].end());
            af.insert(af.end(), hf[k].begin(), hf[k].end());
            aq.insert(aq.end(), hq[k].begin(), hq[k].end());
            if (S.adaptive) upload_mesh(S);
            S.roff = U;
            const std::vector<double> ux = reduced_maps(S, hx[k]);
            U += S.nu;
            arx.insert(arx.end(), ux.begin(), ux.end());
        }
        for (int k = ns; k < 9; ++k) base.start[k] = N;
        upload(x, ax);
        upload(p, ap);
        upload(f, af);
        upload(qw, aq);
        for (auto* b : {&e, &xkA, &xkB, &pst, &accX, &accP}) b->ensure(N);
        base.x = x.p;
        base.p = p.p;
        base.pst = pst.p;
        base.accX = accX.p;
        base.accP = accP.p;
        upload(rx, arx);
        rw.ensure(U);
        re.ensure(U);
    }

    void remesh() {
        remesh_kernels();
        reduced_field();
    }

    // Restart from the dump files of iteration `it` (AMRSimulation.cpp:65-84,
    // AMRStructure::load_restart, AMRStructure_restart.cpp:101-229): per species
    // xs/ps/fs and the full panel tree; weights from the loaded leaves at the
    // loaded positions (set_leaves_weights, as the reference does: equal to the
    // carried weights only for a dump taken right after a remesh), t = it * dt,
    // then the reduced-grid field on the loaded state.
    void restart(const std::string& sim_dir, const std::vector<std::string>& names, int it) {
        if (it < 0) fail(FS_ERR_ARG, "restart iteration must be >= 0");
        const std::string out = sim_dir + ((sim_dir.empty() || sim_dir.back() == '/') ? "" : "/") + "simulation_output/";
        const int ns = (int)sp.size();
        std::vector<std::vector<double>> hx(ns), hp(ns), hf(ns), hq(ns);
        std::vector<HostMesh> meshes(ns);
        auto read_all = [](const std::string& path) {
            std::ifstream in(path, std::ios::in | std::ios::binary | std::ios::ate);
            if (!in) fail(FS_ERR_ARG, "unable to open " + path);
            const std::streamsize n = in.tellg();
            std::vector<unsigned char> b(n > 0 ? (size_t)n : 0);
            in.seekg(0);
            if (n > 0) in.read(reinterpret_cast<char*>(b.data()), n);
            if (!in) fail(FS_ERR_ARG, "error reading " + path);
            return b;
        };
        auto doubles = [&](const std::string& path) {
            const std::vector<unsigned char> b = read_all(path);
            if (b.size() % sizeof(double)) fail(FS_ERR_ARG, "bad file size for " + path);
            std::vector<double> v(b.size() / sizeof(double));
            if (!v.empty()) std::memcpy(v.data(), b.data(), b.size());
            return v;
        };
        for (int k = 0; k < ns; ++k) {
            SpeciesState& S = *sp[k];
            const std::string name = k < (int)names.size() && !names[k].empty() ? names[k] : "species" + std::to_string(k);
            const std::string d = out + name + "/";
            const std::string its = std::to_string(it);
            hx[k] = doubles(d + "xs/xs_" + its);
            hp[k] = doubles(d + "ps/ps_" + its);
            hf[k] = doubles(d + "fs/fs_" + its);
            if (hx[k].size() != hp[k].size() || hp[k].size() != hf[k].size() || hx[k].empty())
                fail(FS_ERR_ARG, "mismatched xs/ps/fs sizes in the restart files of " + name);
            const std::vector<unsigned char> tree = read_all(d + "panels/full_tree_" + its);
            int64_t np = 0;
            if (tree.size() < 8) fail(FS_ERR_ARG, "bad panel tree header for " + name);
            std::memcpy(&np, tree.data(), 8);
            const size_t rec = DiagOutput::kTreeRecord;
            if (np <= 0 || tree.size() != 8 + rec * (size_t)np) fail(FS_ERR_ARG, "bad panel tree size for " + name);
            HostMesh& M = meshes[k];
            M = S.base_mesh.panels.empty() ? S.mesh : S.base_mesh;  // heights and bounds
            M.panels.assign((size_t)np, HostPanel{});
            const int npts = (int)hx[k].size();
            for (int64_t i = 0; i < np; ++i) {
                const unsigned char* r = tree.data() + 8 + rec * (size_t)i;
                int32_t v[18];
                std::memcpy(v, r, sizeof(v));
                HostPanel& P = M.panels[(size_t)i];
                std::memset(&P, 0, sizeof(P));
                P.level = v[1];
                P.parent = v[2];
                P.which = v[3];
                for (int q = 0; q < 9; ++q) {
                    P.pts[q] = v[4 + q];
                    if (P.pts[q] < 0 || P.pts[q] >= npts) fail(FS_ERR_ARG, "panel tree of " + name + " points outside its xs");
                }
                P.left = v[13];
                P.top = v[14];
                P.right = v[15];
                P.bottom = v[16];
                P.child = v[17];
                const int8_t* b = reinterpret_cast<const int8_t*>(r + sizeof(v));
                P.lb = b[0] != 0;
                P.rb = b[1] != 0;
                P.xp = b[2] != 0;
                P.pr = b[3] != 0;
                P.needs = b[4] != 0;
                const int nc = P.xp ? 4 : (P.pr ? 2 : 0);
                if (nc && (P.child <= (int)i || P.child + nc > np))
                    fail(FS_ERR_ARG, "panel tree of " + name + " has children out of order");
                // every index the device walks follow must name a panel: the
                // point location reads the records of neighbours and parents
                bool ok = P.parent >= -1 && P.parent < np && (i == 0) == (P.parent == -1);
                for (int nb : {P.left, P.top, P.right, P.bottom}) ok = ok && nb >= -2 && nb < np && (nb != -1 || P.parent >= 0);
                if (!ok) fail(FS_ERR_ARG, "panel tree of " + name + " has links outside the tree");
            }
            M.xs = hx[k];
            M.ps = hp[k];
            M.restart_leaves();
            if (!S.adaptive && npts != S.nbase)
                fail(FS_ERR_ARG, "restart files of " + name + " hold " + std::to_string(npts) +
                                     " points; the deck's uniform mesh has " + std::to_string(S.nbase));
            const std::vector<double> w = M.base_weights(S.q, prm.quadrature);
            hq[k].resize(npts);
            for (int i = 0; i < npts; ++i) hq[k][i] = w[i] * hf[k][i];
        }
        FS_CUDA(cudaStreamSynchronize(st));
        for (int k = 0; k < ns; ++k) {
            sp[k]->mesh = std::move(meshes[k]);
            upload_mesh(*sp[k]);
        }
        relayout(hx, hp, hf, hq);
        iter = it;
        t = it * prm.dt;
        remeshing = false;
        reduced_field();
        check_status();
    }

    // A step (AMRSimulation::step, AMRSimulation_step.cpp:5-99) is four field
    // evaluations with work before and after each:
    //   0: RK stage 1 kernel, field at xk (epilogue: stage 2)
    //   1: field at xk (epilogue: stage 3)
    //   2: field at xk (epilogue: final combination)
    //   3: iter++, t += dt; either remesh + reduced-grid field, or the field
    //      at the new positions.
    // Stage positions alternate between two buffers so no kernel writes the
    // positions it reads.
    bool remeshing = false;

    void pre_call(int c) {
        if (c == 0) {
            Stage S1 = base;
            k_rk_stage1<<<blocks(N), kT, 0, st>>>(N, S1, e.p, xkA.p);
            FS_LAUNCHED(1);
        } else if (c == 3) {
            iter += 1;
            t += prm.dt;
            remeshing = (iter % prm.remesh_period == 0);
            if (remeshing) {
                last_reduced_iter = iter;
                remesh_kernels();
                reduced_pre();
            }
        }
    }
    // Stage times of rk4_step (AMRSimulation_step.cpp:170, :201, :224):
    // t2 = t + dt/2 for the second and third stages, t + dt for the fourth;
    // the end-of-step evaluation and the remesh use the advanced t (:84-89).
    FieldCall call(int c) const {
        const double t2 = t + prm.dt * 0.5, t4 = t + prm.dt;
        switch (c) {
            case 0: return with_drive(FieldCall{xkA.p, N, qw.p, stage(STAGE_RK2, xkB.p)}, t2);
            case 1: return with_drive(FieldCall{xkB.p, N, qw.p, stage(STAGE_RK3, xkA.p)}, t2);
            case 2: return with_drive(FieldCall{xkA.p, N, qw.p, stage(STAGE_RK4, nullptr)}, t4);
            default: {
                if (remeshing) return reduced_call();
                Stage S = base;
                S.kind = STAGE_STORE;
                S.out = e.p;
                return with_drive(FieldCall{x.p, N, qw.p, S}, t);
            }
        }
    }
    void post_call(int c) {
        if (c == 3 && remeshing) reduced_post();
    }

    void step() {
        for (int c = 0; c < 4; ++c) {
            pre_call(c);
            run_call(call(c));
            post_call(c);
        }
        dump(remeshing);
    }

    // AMRSimulation::step writes the particles every diag_phase_space_period
    // steps (AMRSimulation_step.cpp:94-96); evaluate_field_uniform_grid writes the
    // reduced grid on multiples of diag_period (AMRSimulation_field.cpp:81).
    void dump(bool reduced_now) {
        if (!out) return;
        const bool particles = iter % out->phase_period == 0;
        const bool reduced = reduced_now && iter % out->diag_period == 0;
        if (!particles && !reduced) return;
        std::vector<DiagOutput::Species> q;
        if (particles)
            for (size_t k = 0; k < sp.size(); ++k)
                q.push_back(DiagOutput::snapshot(out->names[k], sp[k]->start, sp[k]->n, sp[k]->mesh));
        out->enqueue(st, iter, particles, reduced, N, U, std::move(q), x.p, p.p, f.p, rx.p, re.p);
    }

    void set_output(const std::string& sim_dir, const std::vector<std::string>& names, int diag_period,
                    int phase_period) {
        if (diag_period < 1 || phase_period < 1) fail(FS_ERR_ARG, "diagnostic periods must be >= 1");
        out.reset();
        auto o = std::make_unique<DiagOutput>();
        o->out = sim_dir + ((sim_dir.empty() || sim_dir.back() == '/') ? "" : "/") + "simulation_output/";
        o->diag_period = diag_period;
        o->phase_period = phase_period;
        o->device = prm.device;
        for (size_t k = 0; k < sp.size(); ++k)
            o->names.push_back(k < names.size() && !names[k].empty() ? names[k] : "species" + std::to_string(k));
        o->start();
        out = std::move(o);
        // the state as it stands (the ctor's dump at iteration 0)
        dump(last_reduced_iter == iter);
    }

    static int* field_error_flag(FieldEngine* fe) { return fe->error_flag(); }
};

}  // namespace fsb

// ------------------------------------------------------------------ C ABI (session)
struct fs_sim {
    fsb::Sim impl;
};

extern "C" {

fs_status fs_debug_set_wait_limits(int device, long long mbar_polls, int walk_panels) {
    return fsb::guard([&] {
        int prev = 0;
        FS_CUDA(cudaGetDevice(&prev));
        FS_CUDA(cudaSetDevice(device));
        fsb::set_mbar_polls(mbar_polls);
        const int w = (walk_panels <= 0 || walk_panels > fsb::kHist) ? fsb::kHist : walk_panels;
        FS_CUDA(cudaMemcpyToSymbol(fsb::g_walk_limit, &w, sizeof(w)));
        FS_CUDA(cudaSetDevice(prev));
    });
}

fs_status fs_sim_create(const fs_sim_params* params, fs_sim** out) {
    if (!params || !out) return fsb::guard([] { fsb::fail(FS_ERR_ARG, "null argument"); });
    *out = nullptr;
    auto* s = new fs_sim();
    fs_status rc = fsb::guard([&] { s->impl.create(*params); });
    if (rc != FS_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return FS_OK;
}

fs_status fs_sim_destroy(fs_sim* sim) {
    return fsb::guard([&] {
        if (sim) {
            cudaSetDevice(sim->impl.prm.device);
            delete sim;
        }
    });
}

fs_status fs_sim_step(fs_sim* sim, int nsteps) {
    return fsb::guard([&] {
        if (!sim || nsteps < 0) fsb::fail(FS_ERR_ARG, "bad argument");
        auto& S = sim->impl;
        FS_CUDA(cudaSetDevice(S.prm.device));
        S.step_ms.clear();
        for (int k = 0; k < nsteps; ++k) {
            FS_CUDA(cudaEventRecord(S.ev0, S.st));
            S.step();
            FS_CUDA(cudaEventRecord(S.ev1, S.st));
            S.check_status();
            float ms = 0.f;
            FS_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
            S.step_ms.push_back(ms);
        }
    });
}

fs_status fs_sim_remesh(fs_sim* sim) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null sim");
        FS_CUDA(cudaSetDevice(sim->impl.prm.device));
        sim->impl.remesh();
        if (sim->impl.out && sim->impl.iter % sim->impl.out->diag_period == 0)
            sim->impl.out->enqueue(sim->impl.st, sim->impl.iter, false, true, sim->impl.N, sim->impl.U, {}, nullptr,
                                   nullptr, nullptr, sim->impl.rx.p, sim->impl.re.p);
        sim->impl.check_status();
    });
}

fs_status fs_sim_set_output(fs_sim* sim, const char* sim_dir, const char* const* species_names, int diag_period,
                            int diag_phase_space_period) {
    return fsb::guard([&] {
        if (!sim || !sim_dir) fsb::fail(FS_ERR_ARG, "null argument");
        auto& S = sim->impl;
        FS_CUDA(cudaSetDevice(S.prm.device));
        std::vector<std::string> names;
        for (int k = 0; k < S.prm.num_species; ++k)
            names.push_back(species_names && species_names[k] ? species_names[k] : "");
        S.set_output(sim_dir, names, diag_period, diag_phase_space_period);
    });
}

fs_status fs_sim_restart(fs_sim* sim, const char* sim_dir, const char* const* species_names, int iter) {
    return fsb::guard([&] {
        if (!sim || !sim_dir) fsb::fail(FS_ERR_ARG, "null argument");
        auto& S = sim->impl;
        FS_CUDA(cudaSetDevice(S.prm.device));
        std::vector<std::string> names;
        for (int k = 0; k < S.prm.num_species; ++k)
            names.push_back(species_names && species_names[k] ? species_names[k] : "");
        S.restart(sim_dir, names, iter);
    });
}

fs_status fs_sim_flush_output(fs_sim* sim) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null sim");
        if (sim->impl.out) sim->impl.out->flush();
    });
}

fs_status fs_sim_num_points(const fs_sim* sim, int species, int* n) {
    return fsb::guard([&] {
        if (!sim || !n) fsb::fail(FS_ERR_ARG, "null argument");
        if (species < 0) *n = sim->impl.N;
        else if (species < (int)sim->impl.sp.size()) *n = sim->impl.sp[species]->n;
        else fsb::fail(FS_ERR_ARG, "species out of range");
    });
}

fs_status fs_sim_export(fs_sim* sim, double* xs, double* ps, double* fs, double* q_ws, double* es) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null sim");
        auto& S = sim->impl;
        FS_CUDA(cudaSetDevice(S.prm.device));
        FS_CUDA(cudaStreamSynchronize(S.st));
        const size_t b = sizeof(double) * S.N;
        if (xs) FS_CUDA(cudaMemcpy(xs, S.x.p, b, cudaMemcpyDeviceToHost));
        if (ps) FS_CUDA(cudaMemcpy(ps, S.p.p, b, cudaMemcpyDeviceToHost));
        if (fs) FS_CUDA(cudaMemcpy(fs, S.f.p, b, cudaMemcpyDeviceToHost));
        if (q_ws) FS_CUDA(cudaMemcpy(q_ws, S.qw.p, b, cudaMemcpyDeviceToHost));
        if (es) FS_CUDA(cudaMemcpy(es, S.e.p, b, cudaMemcpyDeviceToHost));
    });
}

fs_status fs_sim_import_xp(fs_sim* sim, const double* xs, const double* ps, const double* es) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null sim");
        auto& S = sim->impl;
        FS_CUDA(cudaSetDevice(S.prm.device));
        FS_CUDA(cudaStreamSynchronize(S.st));
        const size_t b = sizeof(double) * S.N;
        if (xs) fsb::h2d(S.x.p, xs, b);
        if (ps) fsb::h2d(S.p.p, ps, b);
        if (es) fsb::h2d(S.e.p, es, b);
    });
}

fs_status fs_sim_iter(const fs_sim* sim, int* iter, double* t) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null sim");
        if (iter) *iter = sim->impl.iter;
        if (t) *t = sim->impl.t;
    });
}

fs_status fs_sim_step_times(const fs_sim* sim, double* ms, int cap, int* n) {
    return fsb::guard([&] {
        if (!sim || !n) fsb::fail(FS_ERR_ARG, "null argument");
        const auto& v = sim->impl.step_ms;
        const int k = std::min<int>((int)v.size(), std::max(cap, 0));
        for (int i = 0; i < k && ms; ++i) ms[i] = v[i];
        *n = k;
    });
}

fs_status fs_sim_pair_count(const fs_sim* sim, double* pairs) {
    return fsb::guard([&] {
        if (!sim || !pairs) fsb::fail(FS_ERR_ARG, "null argument");
        *pairs = sim->impl.pairs;
    });
}

fs_status fs_sim_work(const fs_sim* sim, double* direct_pairs, double* kernel_evals) {
    return fsb::guard([&] {
        if (!sim) fsb::fail(FS_ERR_ARG, "null argument");
        if (direct_pairs) *direct_pairs = sim->impl.pairs;
        if (kernel_evals) *kernel_evals = sim->impl.evals;
    });
}

fs_status fs_initial_f0(const fs_sim_params* params, int species, int n, const double* x,
                        const double* p, double* f) {
    return fsb::guard([&] {
        if (!params || n < 0 || (n > 0 && (!x || !p || !f))) fsb::fail(FS_ERR_ARG, "null argument");
        if (species < 0 || species >= params->num_species || species >= 8) fsb::fail(FS_ERR_ARG, "species out of range");
        if (!(params->xmax > params->xmin)) fsb::fail(FS_ERR_ARG, "xmax must exceed xmin");
        const fsb::InitialDistribution dist(params->species[species], params->xmin, params->xmax);
        for (int i = 0; i < n; ++i) f[i] = dist(x[i], p[i]);
    });
}

}  // extern "C"

// ======================================================================
// Batch: many independent simulations stepped together.
//
// Members share one stream.  For each of a step's four field evaluations,
// every member runs its own preparation (RK stage kernels, sort, tile records,
// band searches) and then the FP32 pair work of ALL members runs as one
// persistent launch (k_pairs32_batched) over (member, target block, source
// chunk) items taken longest first from an atomic counter, so simulations of
// very different sizes share the GPU without tails.  Members whose field kind
// cannot join (FP64 reference kernel, treecode) evaluate on their own in the
// same stream.  The first step autotunes the items (targets per thread x
// source tiles per item) by timing the batched launch; later steps are
// captured once into a CUDA graph per step kind (with / without remesh) and
// replayed while all members are in phase.
// ======================================================================
namespace fsb {

struct Batch {
    // Device copy of one batched launch's job and item arrays, with the host
    // bytes they were made from.
    struct Slot {
        DevBuf<PairJob> jobs;
        DevBuf<int4> items;
        std::vector<unsigned char> host;  // jobs then items, as uploaded
        int njobs = 0, nitems = 0;
    };
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        unsigned long long epoch = 0;
        long long launches = 0;
        std::vector<double> dpairs, devals;  // per member, per step
        std::vector<ProfNode> prof;          // profiled regions recorded in the graph
    };
    struct Capturing {};  // thrown when a captured step would need a host upload

    // Members run their own work on kSide side streams (round robin), forked
    // from and joined back into the batch stream around each phase, so small
    // members' kernels overlap; the shared pair launch runs on `st`.
    static constexpr int kSide = 8;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaStream_t side[kSide] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kSide] = {};
    int next_side = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<std::unique_ptr<Sim>> sims;
    std::vector<int> ids;
    int next_id = 1;
    int R = 4, tpc = 32;
    bool tuned = false;
    DevBuf<int> counter, err;
    ItemOrder order;  // device cost order of the batched launch's items
    // slots and graphs are keyed by the step's remesh mask (one char per member)
    std::map<std::string, std::array<Slot, 4>> slots;
    std::map<std::string, Graph> graphs;
    std::set<std::string> warmed, uncapturable;
    bool use_graphs = true;
    bool capturing = false;
    std::vector<double> step_ms;
    double pairs = 0;
    long long graph_steps = 0, plain_steps = 0;

    ~Batch() {
        reset_graphs();
        if (st) cudaStreamSynchronize(st);
        for (auto& q : side)
            if (q) cudaStreamSynchronize(q);
        sims.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (auto& e : ev_join)
            if (e) cudaEventDestroy(e);
        for (auto& q : side)
            if (q) cudaStreamDestroy(q);
        if (st) cudaStreamDestroy(st);
    }

    void init(int dev) {
        device = dev;
        FS_CUDA(cudaSetDevice(dev));
        FS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        FS_CUDA(cudaEventCreate(&ev0));
        FS_CUDA(cudaEventCreate(&ev1));
        FS_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        for (int k = 0; k < kSide; ++k) {
            FS_CUDA(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
            FS_CUDA(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
        }
        counter.ensure(1);
        err.ensure(1);
        FS_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    }

    void reset_graphs() {
        for (auto& kv : graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            prof_release(kv.second.prof);
        }
        graphs.clear();
        warmed.clear();
        uncapturable.clear();
        slots.clear();
    }

    int add(const fs_sim_params& P) {
        if (P.device != device) fail(FS_ERR_ARG, "simulation device differs from the batch device");
        FS_CUDA(cudaStreamSynchronize(st));
        auto s = std::make_unique<Sim>();
        s->create(P, side[next_side++ % kSide]);
        sims.push_back(std::move(s));
        ids.push_back(next_id);
        reset_graphs();
        return next_id++;
    }

    // Take a simulation created on its own stream (synchronised) into the
    // batch: from now on it runs on one of the batch's side streams.
    int adopt(std::unique_ptr<Sim> s) {
        FS_CUDA(cudaStreamSynchronize(s->st));
        if (s->own_stream) FS_CUDA(cudaStreamDestroy(s->st));
        s->st = side[next_side++ % kSide];
        s->own_stream = false;
        sims.push_back(std::move(s));
        ids.push_back(next_id);
        reset_graphs();
        return next_id++;
    }

    int index_of(int id) const {
        for (size_t i = 0; i < ids.size(); ++i)
            if (ids[i] == id) return (int)i;
        fail(FS_ERR_ARG, "no simulation with id " + std::to_string(id));
    }

    void remove(int id) {
        const int i = index_of(id);
        FS_CUDA(cudaStreamSynchronize(st));
        reset_graphs();
        sims.erase(sims.begin() + i);
        ids.erase(ids.begin() + i);
    }

    // Items of all jobs, longest first, in host bytes (jobs then items).
    std::vector<unsigned char> pack(const std::vector<PairJob>& jobs, int R_, int& nitems) const {
        std::vector<int4> items;
        std::vector<double> cost;
        for (size_t j = 0; j < jobs.size(); ++j) pair_job_items(jobs[j], (int)j, R_, items, cost);
        std::vector<int> order(items.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        nitems = (int)items.size();
        std::vector<unsigned char> bytes(sizeof(PairJob) * jobs.size() + sizeof(int4) * items.size());
        std::memcpy(bytes.data(), jobs.data(), sizeof(PairJob) * jobs.size());
        // the item block starts after the jobs, which need not leave it
        // 16-byte aligned, so copy bytewise rather than through an int4 pointer
        unsigned char* dst = bytes.data() + sizeof(PairJob) * jobs.size();
        for (size_t i = 0; i < order.size(); ++i) std::memcpy(dst + i * sizeof(int4), &items[order[i]], sizeof(int4));
        return bytes;
    }

    // Bring the slot's device arrays up to date (never while capturing).
    void stage(Slot& sl, const std::vector<PairJob>& jobs, int R_) {
        int nitems = 0;
        std::vector<unsigned char> bytes = pack(jobs, R_, nitems);
        if (bytes == sl.host && sl.jobs.p) return;
        if (capturing) throw Capturing{};
        sl.jobs.ensure(jobs.size());
        sl.items.ensure(std::max(nitems, 1));
        order.reserve(nitems);
        FS_CUDA(cudaMemcpyAsync(sl.jobs.p, bytes.data(), sizeof(PairJob) * jobs.size(), cudaMemcpyHostToDevice, st));
        FS_CUDA(cudaMemcpyAsync(sl.items.p, bytes.data() + sizeof(PairJob) * jobs.size(), sizeof(int4) * nitems,
                                cudaMemcpyHostToDevice, st));
        FS_CUDA(cudaStreamSynchronize(st));
        sl.host = std::move(bytes);
        sl.njobs = (int)jobs.size();
        sl.nitems = nitems;
    }

    void launch(const Slot& sl, int R_) {
        launch_pairs_batched(R_, pairs_batched_grid(R_), st, sl.jobs.p, sl.items.p, sl.nitems, &order, counter.p,
                             err.p);
    }

    static bool joins(const Sim& s) { return s.prm.field_kind == FS_FIELD_DIRECT32C; }

    void fork() {
        FS_CUDA(cudaEventRecord(ev_fork, st));
        for (int k = 0; k < kSide; ++k) FS_CUDA(cudaStreamWaitEvent(side[k], ev_fork, 0));
    }
    void join() {
        for (int k = 0; k < kSide; ++k) {
            FS_CUDA(cudaEventRecord(ev_join[k], side[k]));
            FS_CUDA(cudaStreamWaitEvent(st, ev_join[k], 0));
        }
    }

    void run_call(int c, std::array<Slot, 4>& sl) {
        std::vector<PairJob> jobs;
        std::vector<Sim*> joined;
        double w = 0;
        {
            // members' work before the shared launch, each on its side stream:
            // RK stage, remesh, sort, source records, band searches (and whole
            // evaluations of members that do not join)
            ProfScope prof("batch_prepare", st);
            fork();
            for (auto& s : sims) {
                s->pre_call(c);
                const Sim::FieldCall fc = s->call(c);
                PairJob j{};
                if (s->field->prepare(fc.x, fc.n, fc.x, fc.q, fc.n, fc.stage, s->st, tpc, &j)) {
                    jobs.push_back(j);
                    joined.push_back(s.get());
                    w += s->field->last_pairs;
                }
                s->pairs += s->field->last_pairs;
                s->evals += s->field->last_pairs;
                pairs += s->field->last_pairs;
            }
            join();
        }
        if (!jobs.empty()) {
            stage(sl[c], jobs, R);
            ProfScope prof("k_pairs32_batched", st, w);
            launch(sl[c], R);
        }
        ProfScope prof("batch_finalize", st);
        fork();
        for (auto* s : joined) s->field->finalize(s->st);
        for (auto& s : sims) s->post_call(c);
        join();
    }

    std::string mask() const {
        std::string m(sims.size(), '0');
        for (size_t i = 0; i < sims.size(); ++i)
            if ((sims[i]->iter + 1) % sims[i]->prm.remesh_period == 0) m[i] = '1';
        return m;
    }

    void step_direct(const std::string& key) {
        auto& sl = slots[key];
        for (int c = 0; c < 4; ++c) run_call(c, sl);
    }

    // Time the batched pair launch of the first field call for each
    // candidate (targets per thread x source tiles per item); keep the fastest.
    void autotune() {
        tuned = true;
        bool any = false;
        for (auto& s : sims) any = any || joins(*s);
        if (!any) return;
        static const int kRs[] = {4, 8};
        static const int kTpcs[] = {8, 16, 32, 64};
        fork();
        for (auto& s : sims)
            if (joins(*s)) s->pre_call(0);  // stage-1 kernel; the step recomputes it
        join();
        float best = 1e30f;
        int bR = R, bT = tpc;
        for (int r : kRs)
            for (int t : kTpcs) {
                fork();
                std::vector<PairJob> jobs;
                for (auto& s : sims) {
                    if (!joins(*s)) continue;
                    const Sim::FieldCall fc = s->call(0);
                    PairJob j{};
                    if (s->field->prepare(fc.x, fc.n, fc.x, fc.q, fc.n, fc.stage, s->st, t, &j)) jobs.push_back(j);
                }
                join();
                Slot sl;
                stage(sl, jobs, r);
                launch(sl, r);  // warm
                FS_CUDA(cudaEventRecord(ev0, st));
                launch(sl, r);
                FS_CUDA(cudaEventRecord(ev1, st));
                FS_CUDA(cudaEventSynchronize(ev1));
                float ms = 0.f;
                FS_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
                if (ms < best) {
                    best = ms;
                    bR = r;
                    bT = t;
                }
            }
        R = bR;
        tpc = bT;
        slots.clear();
        check();
    }

    void check() {
        FS_CUDA(cudaStreamSynchronize(st));
        int h = 0;
        FS_CUDA(cudaMemcpy(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            FS_CUDA(cudaMemset(err.p, 0, sizeof(int)));
            fail((fs_status)h, "device wait timed out in the batched pair kernel");
        }
        for (auto& s : sims) s->check_status();
    }

    // Captured kernels keep their arguments: members whose drive field changes
    // with time, or whose field kind synchronises with the host, step launch by launch.
    bool graphable() const {
        for (auto& s : sims) {
            if (s->prm.field_kind != FS_FIELD_DIRECT32C && s->prm.field_kind != FS_FIELD_DIRECT64) return false;
            if (s->prm.use_external_field) return false;
            for (const auto& q : s->sp)
                if (q->adaptive) return false;  // point counts change at remesh
        }
        return true;
    }

    // Capture one step of this mask.  Host bookkeeping done during the capture
    // is kept (the graph is launched right after); on failure it is rolled back
    // and false is returned.
    bool capture(const std::string& key) {
        struct Saved {
            int iter;
            double t, pairs, evals;
            bool remeshing;
        };
        std::vector<Saved> saved;
        for (auto& s : sims) saved.push_back({s->iter, s->t, s->pairs, s->evals, s->remeshing});
        const double saved_pairs = pairs;
        const long long l0 = fs_kernel_launches();
        const unsigned long long e0 = alloc_epoch().load();
        cudaGraph_t g = nullptr;
        Graph G;
        FS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        prof_capture_sink(&G.prof);
        bool ok = true;
        try {
            step_direct(key);
        } catch (...) {
            ok = false;
        }
        prof_capture_sink(nullptr);
        capturing = false;
        const cudaError_t ee = cudaStreamEndCapture(st, &g);
        if (ee != cudaSuccess) ok = false;
        (void)cudaGetLastError();
        if (ok && g && alloc_epoch().load() == e0) {
            ok = cudaGraphInstantiate(&G.exec, g, 0) == cudaSuccess;
            (void)cudaGetLastError();
        } else {
            ok = false;
        }
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            if (G.exec) cudaGraphExecDestroy(G.exec);
            prof_release(G.prof);
            for (size_t i = 0; i < sims.size(); ++i) {
                sims[i]->iter = saved[i].iter;
                sims[i]->t = saved[i].t;
                sims[i]->pairs = saved[i].pairs;
                sims[i]->evals = saved[i].evals;
                sims[i]->remeshing = saved[i].remeshing;
            }
            pairs = saved_pairs;
            return false;
        }
        G.epoch = e0;
        G.launches = fs_kernel_launches() - l0;
        for (size_t i = 0; i < sims.size(); ++i) {
            G.dpairs.push_back(sims[i]->pairs - saved[i].pairs);
            G.devals.push_back(sims[i]->evals - saved[i].evals);
        }
        graphs[key] = std::move(G);
        return true;
    }

    void replay_bookkeeping(const Graph& G) {
        for (size_t i = 0; i < sims.size(); ++i) {
            Sim& s = *sims[i];
            s.iter += 1;
            s.t += s.prm.dt;
            s.remeshing = (s.iter % s.prm.remesh_period == 0);
            s.pairs += G.dpairs[i];
            s.evals += G.devals[i];
            pairs += G.dpairs[i];
        }
    }

    void step_one() {
        if (sims.empty()) return;
        if (!tuned) autotune();
        const std::string key = mask();
        FS_CUDA(cudaEventRecord(ev0, st));
        bool done = false;
        const Graph* launched = nullptr;
        if (use_graphs && graphable() && warmed.count(key)) {
            auto it = graphs.find(key);
            if (it != graphs.end() && it->second.epoch != alloc_epoch().load()) {
                cudaGraphExecDestroy(it->second.exec);
                graphs.erase(it);
                it = graphs.end();
                warmed.erase(key);
            }
            if (it != graphs.end()) {
                replay_bookkeeping(it->second);
                FS_CUDA(cudaGraphLaunch(it->second.exec, st));
                count_launches(it->second.launches);
                launched = &it->second;
                done = true;
                ++graph_steps;
            } else if (warmed.count(key) && !uncapturable.count(key)) {
                if (capture(key)) {
                    FS_CUDA(cudaGraphLaunch(graphs[key].exec, st));
                    launched = &graphs[key];
                    done = true;
                    ++graph_steps;
                } else {
                    uncapturable.insert(key);
                }
            }
        }
        if (!done) {
            step_direct(key);
            warmed.insert(key);
            ++plain_steps;
        }
        FS_CUDA(cudaEventRecord(ev1, st));
        check();
        if (launched) prof_harvest(launched->prof);
        float ms = 0.f;
        FS_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        step_ms.push_back(ms);
    }
};

}  // namespace fsb

struct fs_batch {
    fsb::Batch impl;
};

extern "C" {

fs_status fs_batch_create(int device, fs_batch** out) {
    if (!out) return fsb::guard([] { fsb::fail(FS_ERR_ARG, "null argument"); });
    *out = nullptr;
    auto* b = new fs_batch();
    fs_status rc = fsb::guard([&] { b->impl.init(device); });
    if (rc != FS_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return FS_OK;
}

fs_status fs_batch_destroy(fs_batch* b) {
    return fsb::guard([&] {
        if (b) {
            cudaSetDevice(b->impl.device);
            delete b;
        }
    });
}

fs_status fs_batch_add(fs_batch* b, const fs_sim_params* params, int* id) {
    return fsb::guard([&] {
        if (!b || !params || !id) fsb::fail(FS_ERR_ARG, "null argument");
        FS_CUDA(cudaSetDevice(b->impl.device));
        *id = b->impl.add(*params);
    });
}

fs_status fs_batch_remove(fs_batch* b, int id) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        FS_CUDA(cudaSetDevice(b->impl.device));
        b->impl.remove(id);
    });
}

fs_status fs_batch_step(fs_batch* b, int nsteps) {
    return fsb::guard([&] {
        if (!b || nsteps < 0) fsb::fail(FS_ERR_ARG, "bad argument");
        FS_CUDA(cudaSetDevice(b->impl.device));
        b->impl.step_ms.clear();
        for (int k = 0; k < nsteps; ++k) b->impl.step_one();
    });
}

fs_status fs_batch_export(fs_batch* b, int id, double* xs, double* ps, double* fs, double* q_ws, double* es) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        auto& S = *b->impl.sims[b->impl.index_of(id)];
        FS_CUDA(cudaSetDevice(b->impl.device));
        FS_CUDA(cudaStreamSynchronize(S.st));
        const size_t n = sizeof(double) * S.N;
        if (xs) FS_CUDA(cudaMemcpy(xs, S.x.p, n, cudaMemcpyDeviceToHost));
        if (ps) FS_CUDA(cudaMemcpy(ps, S.p.p, n, cudaMemcpyDeviceToHost));
        if (fs) FS_CUDA(cudaMemcpy(fs, S.f.p, n, cudaMemcpyDeviceToHost));
        if (q_ws) FS_CUDA(cudaMemcpy(q_ws, S.qw.p, n, cudaMemcpyDeviceToHost));
        if (es) FS_CUDA(cudaMemcpy(es, S.e.p, n, cudaMemcpyDeviceToHost));
    });
}

fs_status fs_batch_info(fs_batch* b, int id, int* npoints, int* iter, double* t, double* pairs) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        auto& S = *b->impl.sims[b->impl.index_of(id)];
        if (npoints) *npoints = S.N;
        if (iter) *iter = S.iter;
        if (t) *t = S.t;
        if (pairs) *pairs = S.pairs;
    });
}

fs_status fs_batch_step_times(fs_batch* b, double* ms, int cap, int* n) {
    return fsb::guard([&] {
        if (!b || !n) fsb::fail(FS_ERR_ARG, "null argument");
        const auto& v = b->impl.step_ms;
        const int k = std::min<int>((int)v.size(), std::max(cap, 0));
        for (int i = 0; i < k && ms; ++i) ms[i] = v[i];
        *n = k;
    });
}

fs_status fs_batch_work(fs_batch* b, double* pairs) {
    return fsb::guard([&] {
        if (!b || !pairs) fsb::fail(FS_ERR_ARG, "null argument");
        *pairs = b->impl.pairs;
    });
}

fs_status fs_batch_band_pairs(fs_batch* b, double* band_pairs, double* pairs) {
    return fsb::guard([&] {
        if (!b || !band_pairs || !pairs) fsb::fail(FS_ERR_ARG, "null argument");
        FS_CUDA(cudaStreamSynchronize(b->impl.st));
        double band = 0.0, all = 0.0;
        for (auto& s : b->impl.sims) {
            if (s->prm.field_kind != FS_FIELD_DIRECT32C) continue;
            band += s->field->band_pairs(s->st);
            all += s->field->last_pairs;
        }
        *band_pairs = band;
        *pairs = all;
    });
}

fs_status fs_batch_stats(fs_batch* b, int* targets_per_thread, int* tiles_per_item, long long* graph_steps,
                         long long* plain_steps) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        if (targets_per_thread) *targets_per_thread = b->impl.R;
        if (tiles_per_item) *tiles_per_item = b->impl.tpc;
        if (graph_steps) *graph_steps = b->impl.graph_steps;
        if (plain_steps) *plain_steps = b->impl.plain_steps;
    });
}

fs_status fs_batch_set_tuning(fs_batch* b, int targets_per_thread, int tiles_per_item) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        if (targets_per_thread != 4 && targets_per_thread != 8)
            fsb::fail(FS_ERR_ARG, "targets_per_thread must be 4 or 8");
        if (tiles_per_item < 1 || tiles_per_item > 4096) fsb::fail(FS_ERR_ARG, "tiles_per_item must be 1..4096");
        FS_CUDA(cudaStreamSynchronize(b->impl.st));
        b->impl.R = targets_per_thread;
        b->impl.tpc = tiles_per_item;
        b->impl.tuned = true;
        b->impl.reset_graphs();
    });
}

fs_status fs_batch_set_graphs(fs_batch* b, int on) {
    return fsb::guard([&] {
        if (!b) fsb::fail(FS_ERR_ARG, "null batch");
        FS_CUDA(cudaStreamSynchronize(b->impl.st));
        b->impl.use_graphs = (on != 0);
        b->impl.reset_graphs();
    });
}

}  // extern "C"

// ======================================================================
// Pool: a request loop over one Batch (continuous batching).
//
// Client threads submit simulations (deck parameters + number of steps) and
// return at once.  One device-owner thread admits queued requests in arrival
// order while the HBM budget (estimated bytes of live members) and the slot
// count allow, steps every live member one step per iteration (their pair
// work shares one persistent launch per field evaluation), and retires
// members that reached their step count: the final state is copied to host
// memory and the device state freed.  Requests that arrive while others are
// running join at the next iteration.  Per-request step latencies are the
// wall times of the iterations in which the request advanced.
// ======================================================================
namespace fsb {

// Device bytes of a simulation of N points (state, stage buffers, mesh and
// remesh arrays, FP32 field engine with at most 64 source chunks), with
// margin; checked against cudaMemGetInfo in the tests.
double estimate_sim_bytes(const fs_sim_params& P) {
    double n = 0;
    for (int s = 0; s < P.num_species && s < 8; ++s) {
        const fs_species_params& S = P.species[s];
        const double h = S.initial_height, ph = S.p_height;
        double pts = (2.0 * std::pow(2.0, h) + 1.0) * (2.0 * std::pow(2.0, h + ph) + 1.0);
        // adaptive refinement can split leaves up to max_height: each level at
        // most quadruples the points (bounded at 64x)
        if (S.do_adaptively_refine && S.n_amr_eps > 0)
            pts *= std::min(64.0, std::pow(4.0, std::max(0, S.max_height - S.initial_height - S.p_height)));
        n += pts;
    }
    double per_point = 1100.0;
    if (P.field_kind == FS_FIELD_TREECODE64 || P.field_kind == FS_FIELD_TREECODE32C) per_point = 1400.0;
    return n * per_point + 8.0 * 1024 * 1024;
}

struct Pool {
    enum State { QUEUED = 0, RUNNING = 1, DONE = 2, FAILED = 3, CANCELLED = 4 };
    struct Request {
        long long id = 0;
        fs_sim_params prm{};
        int nsteps = 0;
        State state = QUEUED;
        int steps_done = 0;
        int member = 0;  // batch id while running
        double est_bytes = 0;
        int npoints = 0;
        double pairs = 0;
        std::vector<double> step_ms;
        std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
        std::vector<double> xs, ps, fs, qws, es;  // final state
        std::string error;
        bool cancel = false;
    };

    int device = 0;
    double budget = 0, in_use = 0;
    int max_live = 64;
    std::mutex mu;
    std::condition_variable cv_work, cv_prep, cv_done;
    std::deque<long long> queue;                                       // submitted, not admitted
    std::deque<std::pair<long long, std::unique_ptr<Sim>>> ready;      // created, not yet in the batch
    std::map<long long, std::unique_ptr<Request>> reqs;
    std::vector<long long> live;                                       // in the batch
    int preparing = 0;
    long long next_id = 1;
    bool stopping = false;
    std::string broken;
    std::thread worker, preparer;
    Batch batch;  // used by the worker thread only
    std::vector<double> all_step_ms;
    double pairs_done = 0, busy_ms = 0;
    long long n_completed = 0, n_failed = 0, n_cancelled = 0, n_admitted = 0, iterations = 0;

    void start(int dev, double hbm_budget, int slots, int tpt, int tpi) {
        device = dev;
        budget = hbm_budget;
        max_live = slots;
        batch.init(dev);
        if (tpt) {
            batch.R = tpt;
            batch.tpc = tpi;
            batch.tuned = true;
        }
        worker = std::thread([this] { run(); });
        preparer = std::thread([this] { prepare_loop(); });
    }

    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
        }
        cv_work.notify_all();
        cv_prep.notify_all();
        if (preparer.joinable()) preparer.join();
        if (worker.joinable()) worker.join();
    }

    long long submit(const fs_sim_params& P, int nsteps) {
        auto r = std::make_unique<Request>();
        r->prm = P;
        r->prm.device = device;
        r->nsteps = nsteps;
        r->est_bytes = estimate_sim_bytes(P);
        r->t_submit = std::chrono::steady_clock::now();
        std::lock_guard<std::mutex> lk(mu);
        if (!broken.empty()) fail(FS_ERR_STATE, "pool stopped after a device error: " + broken);
        if (stopping) fail(FS_ERR_STATE, "pool is shutting down");
        if (r->est_bytes > budget)
            fail(FS_ERR_NOMEM, "request needs about " + std::to_string((long long)(r->est_bytes / 1e6)) +
                                   " MB of device memory, above the pool's HBM budget");
        r->id = next_id++;
        const long long id = r->id;
        queue.push_back(id);
        reqs[id] = std::move(r);
        cv_prep.notify_all();
        return id;
    }

    void cancel(long long id) {
        std::lock_guard<std::mutex> lk(mu);
        Request& r = get(id);
        r.cancel = true;
        if (r.state == QUEUED) {
            auto it = std::find(queue.begin(), queue.end(), id);
            if (it != queue.end()) {
                queue.erase(it);
                finish(r, CANCELLED);
                cv_done.notify_all();
            }
        }
        cv_work.notify_all();
    }

    // --- under mu -----------------------------------------------------------
    void finish(Request& r, State st, const std::string& err = std::string()) {
        r.state = st;
        r.error = err;
        r.t_done = std::chrono::steady_clock::now();
        if (st == DONE) ++n_completed;
        if (st == FAILED) ++n_failed;
        if (st == CANCELLED) ++n_cancelled;
    }
    int occupied() const { return (int)live.size() + (int)ready.size() + preparing; }
    bool front_fits() {
        if (queue.empty() || occupied() >= max_live) return false;
        return in_use + reqs[queue.front()]->est_bytes <= budget;
    }

    // --- preparer thread: admission and simulation set-up ---------------------
    // Creating a simulation (host mesh, f0, upload, initial reduced field) runs
    // on its own stream here, overlapping the worker's steps.
    void prepare_loop() {
        cudaSetDevice(device);
        for (;;) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_prep.wait(lk, [&] { return stopping || !broken.empty() || front_fits(); });
                if (stopping || !broken.empty()) return;
                r = reqs[queue.front()].get();
                size_t fr = 0, tot = 0;
                if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && (double)fr < r->est_bytes + 512.0 * 1024 * 1024 &&
                    occupied() > 0) {
                    // the device is fuller than the estimates say: wait for a member to leave
                    cv_prep.wait_for(lk, std::chrono::milliseconds(50));
                    continue;
                }
                (void)cudaGetLastError();
                queue.pop_front();
                in_use += r->est_bytes;
                ++preparing;
                r->state = RUNNING;
                r->t_admit = std::chrono::steady_clock::now();
                ++n_admitted;
            }
            std::unique_ptr<Sim> sim;
            std::string err;
            try {
                sim = std::make_unique<Sim>();
                sim->create(r->prm);
            } catch (const FsError& e) {
                err = e.msg.empty() ? "simulation set-up failed" : e.msg;
            } catch (const std::exception& e) {
                err = e.what();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                --preparing;
                if (!err.empty() || stopping) {
                    in_use -= r->est_bytes;
                    finish(*r, err.empty() ? CANCELLED : FAILED, err);
                    sim.reset();
                    cv_done.notify_all();
                    cv_prep.notify_all();
                } else {
                    r->npoints = sim->N;
                    ready.emplace_back(r->id, std::move(sim));
                    cv_work.notify_all();
                }
            }
        }
    }

    // --- worker thread ---------------------------------------------------------
    // Move the member's final state to host memory and free its device state.
    void retire(Request& r, State st, const std::string& err = std::string()) {
        if (st == DONE) {
            auto& S = *batch.sims[batch.index_of(r.member)];
            const size_t n = S.N;
            r.xs.resize(n);
            r.ps.resize(n);
            r.fs.resize(n);
            r.qws.resize(n);
            r.es.resize(n);
            FS_CUDA(cudaStreamSynchronize(batch.st));
            FS_CUDA(cudaMemcpy(r.xs.data(), S.x.p, 8 * n, cudaMemcpyDeviceToHost));
            FS_CUDA(cudaMemcpy(r.ps.data(), S.p.p, 8 * n, cudaMemcpyDeviceToHost));
            FS_CUDA(cudaMemcpy(r.fs.data(), S.f.p, 8 * n, cudaMemcpyDeviceToHost));
            FS_CUDA(cudaMemcpy(r.qws.data(), S.qw.p, 8 * n, cudaMemcpyDeviceToHost));
            FS_CUDA(cudaMemcpy(r.es.data(), S.e.p, 8 * n, cudaMemcpyDeviceToHost));
        }
        batch.remove(r.member);
        std::lock_guard<std::mutex> lk(mu);
        in_use -= r.est_bytes;
        live.erase(std::find(live.begin(), live.end(), r.id));
        finish(r, st, err);
        cv_prep.notify_all();
    }

    // Members created by the preparer join the batch.
    void adopt_ready() {
        for (;;) {
            std::pair<long long, std::unique_ptr<Sim>> item;
            Request* r = nullptr;
            {
                // counted in `live` from here on, so the slot stays taken
                std::lock_guard<std::mutex> lk(mu);
                if (ready.empty()) return;
                item = std::move(ready.front());
                ready.pop_front();
                r = reqs.at(item.first).get();
                live.push_back(r->id);
            }
            r->member = batch.adopt(std::move(item.second));
            if (r->nsteps == 0) retire(*r, DONE);
        }
    }

    void iterate() {
        adopt_ready();
        std::vector<Request*> running;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (long long id : live) running.push_back(reqs[id].get());
        }
        for (Request* r : running)
            if (r->cancel) retire(*r, CANCELLED);
        running.erase(std::remove_if(running.begin(), running.end(), [](Request* r) { return r->state != RUNNING; }),
                      running.end());
        if (running.empty()) return;
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<double> before;
        for (Request* r : running) before.push_back(batch.sims[batch.index_of(r->member)]->pairs);
        batch.step_one();
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        {
            std::lock_guard<std::mutex> lk(mu);
            ++iterations;
            busy_ms += ms;
            for (size_t i = 0; i < running.size(); ++i) {
                Request* r = running[i];
                const double w = batch.sims[batch.index_of(r->member)]->pairs - before[i];
                r->pairs += w;
                pairs_done += w;
                r->steps_done += 1;
                r->step_ms.push_back(ms);
                all_step_ms.push_back(ms);
            }
        }
        for (Request* r : running)
            if (r->steps_done >= r->nsteps) retire(*r, DONE);
        cv_done.notify_all();
    }

    void fail_all_live(const std::string& why) {
        std::vector<Request*> running;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (long long id : live) running.push_back(reqs[id].get());
        }
        for (Request* r : running) {
            try {
                retire(*r, FAILED, why);
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu);
                in_use -= r->est_bytes;
                live.erase(std::find(live.begin(), live.end(), r->id));
                finish(*r, FAILED, why);
            }
        }
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stopping || !ready.empty() || !live.empty(); });
                if (stopping) break;
            }
            try {
                iterate();
            } catch (const FsError& e) {
                // a member's remesh failure or a timed-out wait: the members of
                // this iteration cannot be told apart, so all of them fail
                fail_all_live(e.msg);
                if (e.code == FS_ERR_CUDA) {
                    std::lock_guard<std::mutex> lk(mu);
                    broken = e.msg;
                    for (long long id : queue) finish(*reqs[id], FAILED, "pool stopped: " + e.msg);
                    queue.clear();
                    cv_prep.notify_all();
                }
            } catch (const std::exception& e) {
                fail_all_live(e.what());
            }
            cv_done.notify_all();
            {
                std::lock_guard<std::mutex> lk(mu);
                if (!broken.empty()) break;
            }
        }
        // shut down: what is left is cancelled
        std::vector<Request*> running;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (long long id : live) running.push_back(reqs[id].get());
            for (long long id : queue) finish(*reqs[id], CANCELLED);
            queue.clear();
        }
        for (Request* r : running) {
            try {
                retire(*r, CANCELLED);
            } catch (...) {
            }
        }
        cv_done.notify_all();
    }

    void drain_ready_after_stop() {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& it : ready) {
            Request& r = *reqs.at(it.first);
            in_use -= r.est_bytes;
            finish(r, CANCELLED);
        }
        ready.clear();
        cv_done.notify_all();
    }

    Request& get(long long id) {
        auto it = reqs.find(id);
        if (it == reqs.end()) fail(FS_ERR_ARG, "no request with id " + std::to_string(id));
        return *it->second;
    }

    static double percentile(std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        const double pos = q * (v.size() - 1);
        const size_t i = (size_t)pos;
        const double f = pos - i;
        return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
    }
};

}  // namespace fsb

struct fs_pool {
    fsb::Pool impl;
};

extern "C" {

fs_status fs_pool_create(const fs_pool_params* params, fs_pool** out) {
    if (!params || !out) return fsb::guard([] { fsb::fail(FS_ERR_ARG, "null argument"); });
    *out = nullptr;
    const fs_pool_params P = *params;
    fs_status rc = fsb::guard([&] {
        if (!(P.hbm_budget_bytes > 0)) fsb::fail(FS_ERR_ARG, "hbm_budget_bytes must be positive");
        if (P.max_live < 1) fsb::fail(FS_ERR_ARG, "max_live must be >= 1");
        if (P.targets_per_thread != 0 && P.targets_per_thread != 4 && P.targets_per_thread != 8)
            fsb::fail(FS_ERR_ARG, "targets_per_thread must be 0 (autotune), 4 or 8");
        if (P.targets_per_thread != 0 && P.tiles_per_item < 1) fsb::fail(FS_ERR_ARG, "tiles_per_item must be >= 1");
    });
    if (rc != FS_OK) return rc;
    auto* p = new fs_pool();
    rc = fsb::guard([&] {
        FS_CUDA(cudaSetDevice(P.device));
        p->impl.start(P.device, P.hbm_budget_bytes, P.max_live, P.targets_per_thread, P.tiles_per_item);
    });
    if (rc != FS_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return FS_OK;
}

fs_status fs_pool_destroy(fs_pool* p) {
    return fsb::guard([&] {
        if (!p) return;
        p->impl.stop();
        p->impl.drain_ready_after_stop();
        cudaSetDevice(p->impl.device);
        delete p;
    });
}

fs_status fs_pool_submit(fs_pool* p, const fs_sim_params* params, int nsteps, long long* id) {
    return fsb::guard([&] {
        if (!p || !params || !id) fsb::fail(FS_ERR_ARG, "null argument");
        if (nsteps < 0) fsb::fail(FS_ERR_ARG, "nsteps must be >= 0");
        if (params->num_species < 1 || params->num_species > 8) fsb::fail(FS_ERR_ARG, "num_species must be 1..8");
        *id = p->impl.submit(*params, nsteps);
    });
}

fs_status fs_pool_cancel(fs_pool* p, long long id) {
    return fsb::guard([&] {
        if (!p) fsb::fail(FS_ERR_ARG, "null pool");
        p->impl.cancel(id);
    });
}

fs_status fs_pool_poll(fs_pool* p, long long id, fs_request_info* info) {
    return fsb::guard([&] {
        if (!p || !info) fsb::fail(FS_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(p->impl.mu);
        const auto& r = p->impl.get(id);
        info->state = (int)r.state;
        info->steps_done = r.steps_done;
        info->nsteps = r.nsteps;
        info->npoints = r.npoints;
        info->pairs = r.pairs;
        info->step_ms_p50 = fsb::Pool::percentile(r.step_ms, 0.5);
        info->step_ms_p99 = fsb::Pool::percentile(r.step_ms, 0.99);
        using ms = std::chrono::duration<double, std::milli>;
        const bool admitted = r.state != fsb::Pool::QUEUED && r.t_admit.time_since_epoch().count() != 0;
        info->queue_ms = admitted ? ms(r.t_admit - r.t_submit).count() : -1.0;
        info->total_ms = (r.state >= fsb::Pool::DONE) ? ms(r.t_done - r.t_submit).count() : -1.0;
        std::snprintf(info->error, sizeof(info->error), "%s", r.error.c_str());
    });
}

fs_status fs_pool_wait(fs_pool* p, long long id, double timeout_ms, int* state) {
    return fsb::guard([&] {
        if (!p) fsb::fail(FS_ERR_ARG, "null pool");
        std::unique_lock<std::mutex> lk(p->impl.mu);
        auto done = [&] { return p->impl.get(id).state >= fsb::Pool::DONE; };
        if (timeout_ms < 0) {
            p->impl.cv_done.wait(lk, done);
        } else {
            p->impl.cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done);
        }
        if (state) *state = (int)p->impl.get(id).state;
    });
}

fs_status fs_pool_result(fs_pool* p, long long id, double* xs, double* ps, double* fs, double* q_ws, double* es) {
    return fsb::guard([&] {
        if (!p) fsb::fail(FS_ERR_ARG, "null pool");
        std::lock_guard<std::mutex> lk(p->impl.mu);
        auto& r = p->impl.get(id);
        if (r.state != fsb::Pool::DONE) fsb::fail(FS_ERR_STATE, "request has not completed");
        const size_t n = r.xs.size();
        if (xs) std::memcpy(xs, r.xs.data(), 8 * n);
        if (ps) std::memcpy(ps, r.ps.data(), 8 * n);
        if (fs) std::memcpy(fs, r.fs.data(), 8 * n);
        if (q_ws) std::memcpy(q_ws, r.qws.data(), 8 * n);
        if (es) std::memcpy(es, r.es.data(), 8 * n);
    });
}

fs_status fs_pool_release(fs_pool* p, long long id) {
    return fsb::guard([&] {
        if (!p) fsb::fail(FS_ERR_ARG, "null pool");
        std::lock_guard<std::mutex> lk(p->impl.mu);
        auto& r = p->impl.get(id);
        if (r.state < fsb::Pool::DONE) fsb::fail(FS_ERR_STATE, "request is still queued or running");
        p->impl.reqs.erase(id);
    });
}

fs_status fs_pool_step_times(fs_pool* p, long long id, double* ms, int cap, int* n) {
    return fsb::guard([&] {
        if (!p || !n) fsb::fail(FS_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(p->impl.mu);
        const auto& v = p->impl.get(id).step_ms;
        const int k = std::min<int>((int)v.size(), std::max(cap, 0));
        for (int i = 0; i < k && ms; ++i) ms[i] = v[i];
        *n = k;
    });
}

fs_status fs_pool_stats(fs_pool* p, fs_pool_stats_t* s) {
    return fsb::guard([&] {
        if (!p || !s) fsb::fail(FS_ERR_ARG, "null argument");
        std::lock_guard<std::mutex> lk(p->impl.mu);
        auto& P = p->impl;
        s->submitted = P.next_id - 1;
        s->admitted = P.n_admitted;
        s->completed = P.n_completed;
        s->failed = P.n_failed;
        s->cancelled = P.n_cancelled;
        s->queued = (long long)P.queue.size();
        s->live = (long long)P.live.size();
        s->iterations = P.iterations;
        s->hbm_in_use_bytes = P.in_use;
        s->pairs = P.pairs_done;
        s->busy_ms = P.busy_ms;
        s->step_ms_p50 = fsb::Pool::percentile(P.all_step_ms, 0.5);
        s->step_ms_p99 = fsb::Pool::percentile(P.all_step_ms, 0.99);
    });
}

fs_status fs_pool_estimate_bytes(const fs_sim_params* params, double* bytes) {
    return fsb::guard([&] {
        if (!params || !bytes) fsb::fail(FS_ERR_ARG, "null argument");
        *bytes = fsb::estimate_sim_bytes(*params);
    });
}

}  // extern "C"
