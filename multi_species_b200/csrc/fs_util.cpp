// Error reporting, launch accounting and device queries for libfs_b200.
#include <map>
#include <mutex>
#include <utility>

#include "fs_internal.h"

namespace fsb {

namespace {
thread_local std::string t_last_error;
std::atomic<long long> g_launches{0};
std::mutex g_sm_mu;
std::vector<int> g_sm_cache;
}  // namespace

void set_last_error(const std::string& msg) { t_last_error = msg; }

void fail(fs_status code, const std::string& msg) { throw FsError{code, msg}; }

void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return;
    std::string m = std::string(what) + " failed at " + file + ":" + std::to_string(line) + ": " +
                    cudaGetErrorString(e);
    fail(FS_ERR_CUDA, m);
}

void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches() { return g_launches.load(std::memory_order_relaxed); }

int sm_count() {
    int dev = 0;
    FS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_sm_mu);
    if ((int)g_sm_cache.size() <= dev) g_sm_cache.resize(dev + 1, 0);
    if (!g_sm_cache[dev]) {
        int n = 0;
        FS_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        g_sm_cache[dev] = n;
    }
    return g_sm_cache[dev];
}

const char* last_error_cstr() { return t_last_error.c_str(); }

// ------------------------------------------------------------------ profiling
namespace {
struct Pending {
    std::string name;
    cudaEvent_t a, b;
    double work;
};
struct Total {
    long long launches = 0;
    double ms = 0.0, work = 0.0;
};
std::atomic<bool> g_prof{false};
std::mutex g_prof_mu;
std::vector<Pending> g_pending;
std::map<std::string, Total> g_totals;

void collect_locked() {
    for (auto& p : g_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            auto& t = g_totals[p.name];
            t.launches += 1;
            t.ms += ms;
            t.work += p.work;
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    g_pending.clear();
    (void)cudaGetLastError();
}
}  // namespace

bool profiling_enabled() { return g_prof.load(std::memory_order_relaxed); }

namespace {
thread_local std::vector<ProfNode>* t_sink = nullptr;
}

void prof_capture_sink(std::vector<ProfNode>* sink) { t_sink = sink; }

ProfScope::ProfScope(const char* name, cudaStream_t st, double work) : name_(name), st_(st), work_(work) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st_, &cs) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    if (cs != cudaStreamCaptureStatusNone) {
        if (!t_sink) return;
        if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
            if (a_) cudaEventDestroy(a_);
            a_ = b_ = nullptr;
            (void)cudaGetLastError();
            return;
        }
        captured_ = true;
        cudaEventRecordWithFlags(a_, st_, cudaEventRecordExternal);
        return;
    }
    if (!profiling_enabled()) return;
    if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
        a_ = b_ = nullptr;
        (void)cudaGetLastError();
        return;
    }
    cudaEventRecord(a_, st_);
}
ProfScope::~ProfScope() {
    if (!a_) return;
    if (captured_) {
        cudaEventRecordWithFlags(b_, st_, cudaEventRecordExternal);
        if (t_sink) t_sink->push_back({name_, a_, b_, work_});
        return;
    }
    cudaEventRecord(b_, st_);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_pending.push_back({name_, a_, b_, work_});
}

void prof_harvest(const std::vector<ProfNode>& nodes) {
    if (!profiling_enabled()) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (const auto& n : nodes) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, n.a, n.b) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        Total& t = g_totals[n.name];
        t.launches += 1;
        t.ms += ms;
        t.work += n.work;
    }
}

void prof_add_work(const char* name, double work) {
    if (!profiling_enabled()) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_totals[name].work += work;
}

void prof_release(std::vector<ProfNode>& nodes) {
    for (auto& n : nodes) {
        cudaEventDestroy(n.a);
        cudaEventDestroy(n.b);
    }
    nodes.clear();
}

}  // namespace fsb

extern "C" {

fs_status fs_profile_enable(int on) {
    fsb::g_prof.store(on != 0);
    return FS_OK;
}

fs_status fs_profile_read(const char* kernel, long long* launches, double* total_ms, double* total_work) {
    std::lock_guard<std::mutex> lk(fsb::g_prof_mu);
    fsb::collect_locked();
    auto it = fsb::g_totals.find(kernel ? kernel : "");
    const bool hit = it != fsb::g_totals.end();
    if (launches) *launches = hit ? it->second.launches : 0;
    if (total_ms) *total_ms = hit ? it->second.ms : 0.0;
    if (total_work) *total_work = hit ? it->second.work : 0.0;
    return FS_OK;
}

fs_status fs_profile_reset(void) {
    std::lock_guard<std::mutex> lk(fsb::g_prof_mu);
    fsb::collect_locked();
    fsb::g_totals.clear();
    return FS_OK;
}

}  // extern "C"

namespace fsb {

}  // namespace fsb
