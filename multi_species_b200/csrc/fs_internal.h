// Internal declarations of libfs_b200 (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <functional>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fs_b200.h"

namespace fsb {

// ------------------------------------------------------------------ errors
// Internal code throws FsError; the C ABI layer converts it to an fs_status
// and records the message for fs_last_error().
struct FsError {
    fs_status code;
    std::string msg;
};

void set_last_error(const std::string& msg);
[[noreturn]] void fail(fs_status code, const std::string& msg);
void cuda_check(cudaError_t e, const char* what, const char* file, int line);

#define FS_CUDA(call) ::fsb::cuda_check((call), #call, __FILE__, __LINE__)
#define FS_LAUNCHED(n) do { ::fsb::count_launches(n); FS_CUDA(cudaGetLastError()); } while (0)

void count_launches(long long n);
long long launches();

// Number of SMs of the current device (cached per device).
int sm_count();

// Device-time profiling of named kernels (enabled by fs_profile_enable).
// Records a CUDA event pair on `st` around the enclosed launches.
class ProfScope {
   public:
    // `work`: algorithmic units done by the enclosed launches (pairs, bytes)
    ProfScope(const char* name, cudaStream_t st, double work = 0.0);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

   private:
    const char* name_;
    cudaStream_t st_;
    double work_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
    bool captured_ = false;
};
bool profiling_enabled();

// Profiled regions inside a captured CUDA graph: while a sink is set on this
// thread, a ProfScope on a capturing stream records its two events as graph
// nodes (external event records) and appends them to the sink; the graph's
// owner adds their times to the profile after each replay.
struct ProfNode {
    const char* name;
    cudaEvent_t a, b;
    double work;
};
void prof_capture_sink(std::vector<ProfNode>* sink);
void prof_harvest(const std::vector<ProfNode>& nodes);  // events must have completed
void prof_release(std::vector<ProfNode>& nodes);
// Adds algorithmic work counted apart from any launch (e.g. the treecode's
// near pairs and far terms) under `name` while profiling is enabled.
void prof_add_work(const char* name, double work);

// ------------------------------------------------------------------ device buffers
// Bumped by every device (re)allocation of a DevBuf; a captured CUDA graph
// records it and is discarded when it changed, since the graph's kernels hold
// raw device pointers.
inline std::atomic<unsigned long long>& alloc_epoch() {
    static std::atomic<unsigned long long> e{0};
    return e;
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void ensure(size_t count) {
        if (count <= n && p) return;
        release();
        alloc_epoch().fetch_add(1);
        size_t bytes = (count ? count : 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            (void)cudaGetLastError();
            fail(FS_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        n = count;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------------ RK4 stage epilogue
// Fused into the last kernel of each field evaluation.  kind:
//   STAGE_STORE  out[o] = E
//   STAGE_RK2    E is the field at the stage-2 positions: ef2 = E*qm,
//                p3 = p + hdt*ef2, xk = x + hdt*p2, accX += 2 p2, accP += 2 ef2
//   STAGE_RK3    ef3 = E*qm, p4 = p + dt*ef3, xk = x + dt*p3, accX += 2 p3, accP += 2 ef3
//   STAGE_RK4    ef4 = E*qm, x += dt6*(accX + p4), p += dt6*(accP + ef4)
// (src/simulation_files/AMRSimulation_step.cpp:158-248, same operation order).
enum StageKind { STAGE_STORE = 0, STAGE_RK2 = 1, STAGE_RK3 = 2, STAGE_RK4 = 3 };

struct Stage {
    int kind = STAGE_STORE;
    double* out = nullptr;
    double *x = nullptr, *p = nullptr, *xk = nullptr, *pst = nullptr, *accX = nullptr, *accP = nullptr;
    double dt = 0, hdt = 0, dt6 = 0;
    int nsp = 1;
    int start[9] = {0};
    double qm[8] = {0};
    // relativistic position push (rel != 0): stage positions move with
    // v = (p/m) / sqrt(1 + (p/m)^2), m the species mass
    int rel = 0;
    double m[8] = {0};
    // drive field: E += ext_a * sin(ext_k * ext_x[o] - ext_omt) when ext_x is set
    // (ext_x = the evaluation's targets, in the caller's order)
    const double* ext_x = nullptr;
    double ext_a = 0, ext_k = 0, ext_omt = 0;
};

// ------------------------------------------------------------------ host mesh
struct HostPanel {
    int pts[9];
    int level, parent, which, child;
    int left, top, right, bottom;
    uint8_t lb, rb, xp, pr, needs;
};

struct HostMesh {
    int h = 0, ph = 0;
    double xmin = 0, xmax = 0, pmin = 0, pmax = 0;
    std::vector<HostPanel> panels;
    std::vector<double> xs, ps;
    std::vector<int> leaves;
    int min_unrefined = 1;  // first panel of the last uniform generation
    void build(int h, int ph, double xmin, double xmax, double pmin, double pmax);
    // Adaptive refinement (generate_mesh, AMRStructure_amr.cpp:901-941): f holds
    // the values at the current points and grows with the mesh; eval(x, p, n, out)
    // gives f at new points.
    void adapt(std::vector<double>& f, const double* eps, int neps, int max_height,
               const std::function<void(const double*, const double*, int, double*)>& eval);
    // Leaves (DFS order) of panels loaded from a restart file.
    void restart_leaves();
    std::vector<double> base_weights(double q, int quadrature) const;
    void panel_records(int* out) const;  // 18 ints per panel
    int nx() const { return 2 * (1 << h) + 1; }
    int np() const { return 2 * (1 << (h + ph)) + 1; }
};

// Initial distribution of one species (make_f0_return_ptr,
// AMRSimulation_load.cpp:139-225): tables of the Friedman beam and the
// relativistic wave are built once, K_1(mu) is evaluated once.
struct InitialDistribution {
    int ics;
    double pth, pstr, amp, mu, wave_beta, k = 0;
    double fb_xcf = 0, fb_nhat = 0, fb_pth = 0, fb_dx = 0;
    std::vector<double> fb_N;          // Friedman envelope density, step 0.01
    double k1mu = 0, gstr = 0;         // K_1(mu), sqrt(1 + pstr^2)
    std::vector<double> wv_x, wv_p;    // cold travelling-wave orbit, 100 nodes
    InitialDistribution(const fs_species_params& S, double xmin, double xmax);
    double operator()(double x, double p) const;
};

// ------------------------------------------------------------------ field engines
// Per sorted target of the FP32 direct sum (csrc/fs_direct32.cu).
struct TargetInfo {
    double tlo;   // target coordinate for sources before J (after J: tlo + L)
    double ffar;  // exact FP64 sum of sign(d) * q/2 over the far band (FP64 q)
    int J, U1, U2;
    int pad;
};

// One field evaluation's FP32 pair work, as the pair kernels see it.
struct PairJob {
    const float4* src;        // tile-relative source records {s, q/2, q/2 a1, q/2 a2}
    const double2* src64;     // the same sources in FP64: {x (wrapped), q/4}, for band pairs
    const double* tbase;      // FP64 tile bases
    const TargetInfo* info;   // per sorted target (nt_pad entries)
    double* partial;          // chunks * nt_pad
    int ns, ntiles, tpc, nt_pad;
    double L;
    float eps2, a1, a2;  // near band: eps^2, eps^2/2, eps^4/8
    float e2f;           // far pairs: 3 eps^2 / 4
    double eps2d;        // band pairs (FP64): eps^2
    int nt;              // targets: the first nt of the nt_pad entries of info are real
};

class FieldEngine {
   public:
    virtual ~FieldEngine() = default;
    // Field at targets from sources (device pointers), result through the
    // stage epilogue, enqueued on `st`.  For targets == sources pass the same
    // pointer and nt == ns.
    virtual void eval(const double* d_targets, int nt, const double* d_sources, const double* d_q,
                      int ns, const Stage& stage, cudaStream_t st) = 0;
    // Device int set non-zero by a kernel whose bounded wait gave up (or null).
    virtual int* error_flag() { return nullptr; }
    // Kernel-level evaluations of the last call (pairs for the direct sums;
    // near pairs + far cluster terms for the treecode).  May synchronise `st`;
    // called only when profiling is enabled.
    virtual double actual_work(cudaStream_t st) {
        (void)st;
        return last_pairs;
    }
    // Pairs of the last evaluation that the FP32c direct sum evaluates in FP64
    // (|d| <= 16 eps); 0 for the other kinds.  Synchronises `st`.
    virtual double band_pairs(cudaStream_t st) {
        (void)st;
        return 0.0;
    }
    // Batched use.  prepare() runs everything before the pair kernel with
    // `tpc` source tiles per work chunk and fills *job, returning true; the
    // caller then runs the pair work (alone or batched with other jobs) and
    // calls finalize().  Engines whose work cannot join a batched launch
    // evaluate completely here and return false (no finalize).
    virtual bool prepare(const double* d_t, int nt, const double* d_s, const double* d_q, int ns,
                         const Stage& stage, cudaStream_t st, int tpc, PairJob* job) {
        (void)tpc;
        (void)job;
        eval(d_t, nt, d_s, d_q, ns, stage, st);
        return false;
    }
    virtual void finalize(cudaStream_t st) { (void)st; }
    // Pair interactions (direct-equivalent) of the last call.
    double last_pairs = 0;
};

// Runs fn, converting FsError / exceptions into an fs_status and recording the
// message for fs_last_error().
fs_status guard(const std::function<void()>& fn);

// Device scratch for ordering the items of a batched launch by their
// estimated cost (reserve() before any graph capture; it may allocate).
struct ItemOrder {
    DevBuf<int> cost, ids;
    DevBuf<unsigned char> tmp;
    void reserve(int nitems);
};

// Batched FP32 pair work (csrc/fs_direct32.cu): one persistent launch over the
// (job, target block, source chunk) items of many field evaluations, in the
// order of the device's cost estimate when `ord` is given (reserved for at
// least nitems): band-heavy items spread over the queue, light ones last.
void launch_pairs_batched(int R, int grid, cudaStream_t st, const PairJob* jobs, const int4* items, int nitems,
                          ItemOrder* ord, int* counter, int* err);
int pairs_batched_grid(int R);
// Items of one job for R targets per thread (target blocks x chunks) and the
// work of each (tiles x targets), appended to `items` / `cost`.
void pair_job_items(const PairJob& job, int job_index, int R, std::vector<int4>& items, std::vector<double>& cost);

// Inclusive prefix sum of n doubles with a fixed association, so that its
// results are the same on every run (csrc/fs_scan.cu); `scratch` holds
// scan_f64_scratch(n) doubles.
size_t scan_f64_scratch(int n);
void scan_f64_inclusive(const double* in, double* out, int n, double* scratch, cudaStream_t st);
// out[0] = sum of in[0..n), with the same fixed association (same scratch).
void sum_f64(const double* in, int n, double* scratch, double* out, cudaStream_t st);

// Polls of the pair kernels' tile waits on the current device (< 0: the
// default bound); a test hook behind fs_debug_set_wait_limits.
void set_mbar_polls(long long polls);

FieldEngine* make_direct64(double L, double eps);
FieldEngine* make_direct64_open(double eps);
FieldEngine* make_direct32c(double L, double eps);
FieldEngine* make_treecode(double L, double eps, double mac, int degree, int max_source, bool fp32_near);

}  // namespace fsb
