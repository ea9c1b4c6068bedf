// Oracle harness around the reference's own simulation code (TEST INFRASTRUCTURE).
//
// oracle/Makefile compiles this file together with the UNMODIFIED reference
// sources -- src/structure_files/*.cpp, src/simulation_files/*.cpp and
// src/FieldStructure.cpp, taken from where they lie -- into
// oracle/_ref/libamr_ref.so.  The reference's headers are read from a copy made
// by the recipe with three mechanical edits (the absolute Boost include lines
// inc/AMRSimulation.hpp:47-48 and inc/initial_distributions.hpp:17-19 point at
// the shims in oracle/refshim/, and AMRSimulation gets the three restart
// members that AMRSimulation.cpp:65-121 and AMRSimulation_load.cpp:43-44 use
// but the header never declares).  Eigen and Boost are absent from this image;
// oracle/refshim/ holds stand-ins for the few calls the reference makes.
//
// The C ABI below drives AMRSimulation exactly as run_FARRSIGHT2.cpp does
// (constructor from a deck.json, then step()), and reads the reference's
// public members: the species' points, weights, f, E, panel trees and reduced
// grids.  Only tests/ and the generator of tests/golden/ load this library;
// the product never does.
//
// Three things are needed to run the reference code unchanged:
//  * Its prints go to std::cout; they are muted by swapping the stream buffer
//    around each call.  AMRSimulation's constructor opens "debug.txt" in the
//    working directory (AMRSimulation.cpp:6), so the constructor runs with the
//    simulation directory as the working directory.
//  * refine_panels and refine_panels_refine_v keep a Panel* into `panels`
//    across panels.push_back, which may reallocate, and then read the split
//    panel's point indices and boundary flags through it
//    (AMRStructure_amr.cpp:793-818, :461-480).  With the system allocator those
//    reads may see allocator bookkeeping or unmapped memory.  This harness
//    replaces the global scalar operator new/delete for this shared object
//    (linked -Bsymbolic): blocks freed while a harness call runs stay intact in
//    a quarantine until the call returns, so those reads see the panel exactly
//    as it was before the append -- the values the code means to read.
//  * E_MQ_Treecode frees its arrays twice (src/FieldStructure.cpp:313-378 vs
//    :466-470); the array operators new[]/delete[] ignore the second delete and
//    pad every block with zeroed bytes, as oracle/ref_harness.cpp does.
#include "AMRSimulation.hpp"

#include <unistd.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

constexpr size_t kArrayTailPad = 8192;

// The bookkeeping containers allocate with malloc: the replaced operator new
// below takes the heap lock, so they must not call it.
template <typename T>
struct MallocAllocator {
    typedef T value_type;
    MallocAllocator() = default;
    template <typename U>
    MallocAllocator(const MallocAllocator<U>&) {}
    T* allocate(size_t n) {
        void* p = std::malloc(n * sizeof(T));
        if (!p) throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t) { std::free(p); }
    template <typename U>
    bool operator==(const MallocAllocator<U>&) const { return true; }
    template <typename U>
    bool operator!=(const MallocAllocator<U>&) const { return false; }
};

typedef std::unordered_set<void*, std::hash<void*>, std::equal_to<void*>, MallocAllocator<void*>> PtrSet;
typedef std::vector<void*, MallocAllocator<void*>> PtrList;

struct Heap {
    std::mutex mu;
    PtrSet scalar_live, array_live;
    PtrList quarantine;
    int depth = 0;
};

Heap& heap() {
    // constructed in static storage, never destroyed (used until exit), and
    // not allocated through the replaced operator new
    alignas(Heap) static unsigned char storage[sizeof(Heap)];
    static Heap* h = new (storage) Heap();
    return *h;
}

void* scalar_alloc(size_t n) {
    void* p = std::calloc(1, n ? n : 1);
    if (!p) throw std::bad_alloc();
    Heap& h = heap();
    std::lock_guard<std::mutex> lk(h.mu);
    h.scalar_live.insert(p);
    return p;
}

void scalar_free(void* p) {
    if (!p) return;
    Heap& h = heap();
    std::lock_guard<std::mutex> lk(h.mu);
    auto it = h.scalar_live.find(p);
    if (it == h.scalar_live.end()) {  // allocated by the C++ runtime's own operator new
        std::free(p);
        return;
    }
    h.scalar_live.erase(it);
    if (h.depth > 0) h.quarantine.push_back(p);
    else std::free(p);
}

void* array_alloc(size_t n) {
    void* p = std::calloc(1, n + kArrayTailPad);
    if (!p) throw std::bad_alloc();
    Heap& h = heap();
    std::lock_guard<std::mutex> lk(h.mu);
    h.array_live.insert(p);
    return p;
}

void array_free(void* p) {
    if (!p) return;
    Heap& h = heap();
    std::lock_guard<std::mutex> lk(h.mu);
    auto it = h.array_live.find(p);
    if (it == h.array_live.end()) return;  // second delete[] of the same block: ignored
    h.array_live.erase(it);
    if (h.depth > 0) h.quarantine.push_back(p);
    else std::free(p);
}

// One harness call: stdout muted, frees quarantined until the call returns.
struct CallScope {
    std::streambuf* saved;
    std::ostringstream sink;
    CallScope() {
        saved = std::cout.rdbuf(sink.rdbuf());
        std::lock_guard<std::mutex> lk(heap().mu);
        heap().depth++;
    }
    ~CallScope() {
        std::cout.rdbuf(saved);
        PtrList release;
        {
            std::lock_guard<std::mutex> lk(heap().mu);
            if (--heap().depth == 0) release.swap(heap().quarantine);
        }
        for (void* p : release) std::free(p);
    }
};

struct RefSim {
    AMRSimulation* sim = nullptr;
    std::string dir;
};

// Species arrays are current after scatter (AMRSimulation_gather_scatter.cpp:36-51);
// rk4_step leaves the simulation-level arrays newer (need_scatter).
void sync_species(AMRSimulation* s) {
    if (s->need_scatter) s->scatter(true);
}

}  // namespace

void* operator new(size_t n) { return scalar_alloc(n); }
void* operator new(size_t n, const std::nothrow_t&) noexcept {
    try { return scalar_alloc(n); } catch (...) { return nullptr; }
}
void operator delete(void* p) noexcept { scalar_free(p); }
void operator delete(void* p, size_t) noexcept { scalar_free(p); }
void operator delete(void* p, const std::nothrow_t&) noexcept { scalar_free(p); }
void* operator new[](size_t n) { return array_alloc(n); }
void* operator new[](size_t n, const std::nothrow_t&) noexcept {
    try { return array_alloc(n); } catch (...) { return nullptr; }
}
void operator delete[](void* p) noexcept { array_free(p); }
void operator delete[](void* p, size_t) noexcept { array_free(p); }
void operator delete[](void* p, const std::nothrow_t&) noexcept { array_free(p); }

extern "C" {

// AMRSimulation(sim_dir, deck_address) (AMRSimulation.cpp:5-91).  sim_dir ends
// with '/' and already holds simulation_output/<species>/{xs,ps,fs,panels}
// and simulation_output/{reduce_xs,reduced_es}.  Returns NULL on failure.
void* amrref_sim_create(const char* sim_dir, const char* deck_path) {
    CallScope scope;
    RefSim* r = new RefSim();
    r->dir = sim_dir;
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) { delete r; return nullptr; }
    if (chdir(sim_dir) != 0) { delete r; return nullptr; }
    try {
        r->sim = new AMRSimulation(std::string(sim_dir), std::string(deck_path));
    } catch (...) {
        r->sim = nullptr;
    }
    if (chdir(cwd) != 0) { /* the caller's directory vanished: nothing to restore */ }
    if (!r->sim || r->sim->species_list.empty()) {
        delete r->sim;
        delete r;
        return nullptr;
    }
    return r;
}

void amrref_sim_destroy(void* h) {
    if (!h) return;
    CallScope scope;
    RefSim* r = static_cast<RefSim*>(h);
    delete r->sim;
    delete r;
}

// n x AMRSimulation::step() (AMRSimulation_step.cpp:5-99).
int amrref_sim_step(void* h, int n) {
    CallScope scope;
    AMRSimulation* s = static_cast<RefSim*>(h)->sim;
    try {
        for (int i = 0; i < n; ++i) s->step();
    } catch (...) {
        return 1;
    }
    return 0;
}

// AMRSimulation::remesh() on the current state (AMRSimulation_remesh.cpp:3-48).
int amrref_sim_remesh(void* h) {
    CallScope scope;
    AMRSimulation* s = static_cast<RefSim*>(h)->sim;
    try {
        s->remesh();
    } catch (...) {
        return 1;
    }
    return 0;
}

int amrref_sim_nspecies(void* h) { return static_cast<RefSim*>(h)->sim->N_sp; }

int amrref_sim_species_points(void* h, int sp) {
    return int(static_cast<RefSim*>(h)->sim->species_list[sp]->xs.size());
}

int amrref_sim_iter(void* h, double* t) {
    AMRSimulation* s = static_cast<RefSim*>(h)->sim;
    if (t) *t = s->t;
    return s->iter_num;
}

// Concatenated species state (species in deck order); any pointer may be NULL.
int amrref_sim_state(void* h, double* xs, double* ps, double* fs, double* qws, double* es) {
    CallScope scope;
    AMRSimulation* s = static_cast<RefSim*>(h)->sim;
    sync_species(s);
    size_t o = 0;
    for (AMRStructure* sp : s->species_list) {
        size_t n = sp->xs.size();
        if (xs) std::memcpy(xs + o, sp->xs.data(), n * sizeof(double));
        if (ps) std::memcpy(ps + o, sp->ps.data(), n * sizeof(double));
        if (fs) std::memcpy(fs + o, sp->fs.data(), n * sizeof(double));
        if (qws) std::memcpy(qws + o, sp->q_ws.data(), n * sizeof(double));
        if (es) {
            if (sp->es.size() == n) std::memcpy(es + o, sp->es.data(), n * sizeof(double));
            else std::memset(es + o, 0, n * sizeof(double));
        }
        o += n;
    }
    return 0;
}

// Overwrite the species' positions and velocities (concatenated, deck order);
// the next step gathers them (need_gather), as after a restart load.
int amrref_sim_set_xp(void* h, const double* xs, const double* ps) {
    CallScope scope;
    AMRSimulation* s = static_cast<RefSim*>(h)->sim;
    sync_species(s);
    size_t o = 0;
    for (AMRStructure* sp : s->species_list) {
        size_t n = sp->xs.size();
        std::memcpy(sp->xs.data(), xs + o, n * sizeof(double));
        std::memcpy(sp->ps.data(), ps + o, n * sizeof(double));
        o += n;
    }
    s->need_gather = true;
    return 0;
}

int amrref_sim_npanels(void* h, int sp) {
    return int(static_cast<RefSim*>(h)->sim->species_list[sp]->panels.size());
}

// Panel records as 18 ints: point_inds[9], level, parent_ind, which_child,
// child_inds_start, left, top, right, bottom neighbours, flags (1 is_left_bdry,
// 2 is_right_bdry, 4 is_refined_xp, 8 is_refined_p)  (inc/Panel.hpp:41-61).
int amrref_sim_panels(void* h, int sp, int* out) {
    const std::vector<Panel>& P = static_cast<RefSim*>(h)->sim->species_list[sp]->panels;
    for (size_t i = 0; i < P.size(); ++i) {
        int* r = out + i * 18;
        for (int k = 0; k < 9; ++k) r[k] = P[i].point_inds[k];
        r[9] = P[i].level;
        r[10] = P[i].parent_ind;
        r[11] = P[i].which_child;
        r[12] = P[i].child_inds_start;
        r[13] = P[i].left_nbr_ind;
        r[14] = P[i].top_nbr_ind;
        r[15] = P[i].right_nbr_ind;
        r[16] = P[i].bottom_nbr_ind;
        r[17] = (P[i].is_left_bdry ? 1 : 0) | (P[i].is_right_bdry ? 2 : 0) | (P[i].is_refined_xp ? 4 : 0) |
                (P[i].is_refined_p ? 8 : 0);
    }
    return int(P.size());
}

int amrref_sim_nleaves(void* h, int sp) {
    return int(static_cast<RefSim*>(h)->sim->species_list[sp]->leaf_inds.size());
}

int amrref_sim_leaves(void* h, int sp, int* out) {
    const std::vector<int>& L = static_cast<RefSim*>(h)->sim->species_list[sp]->leaf_inds;
    std::memcpy(out, L.data(), L.size() * sizeof(int));
    return int(L.size());
}

// The species' reduced grid of its last get_reduced_xs_ws / get_reduced_es
// (AMRStructure.cpp:147-196): unique x, summed weights and the reduced field.
int amrref_sim_nreduced(void* h, int sp) {
    return int(static_cast<RefSim*>(h)->sim->species_list[sp]->reduced_xs.size());
}

int amrref_sim_reduced(void* h, int sp, double* rx, double* rw, double* re) {
    AMRStructure* s = static_cast<RefSim*>(h)->sim->species_list[sp];
    size_t u = s->reduced_xs.size();
    if (rx) std::memcpy(rx, s->reduced_xs.data(), u * sizeof(double));
    if (rw) std::memcpy(rw, s->reduced_ws.data(), u * sizeof(double));
    if (re) {
        if (s->sort_es.size() == u) std::memcpy(re, s->sort_es.data(), u * sizeof(double));
        else std::memset(re, 0, u * sizeof(double));
    }
    return int(u);
}

double amrref_sim_f_beyond(void* h, int sp) {
    return static_cast<RefSim*>(h)->sim->species_list[sp]->f_beyond_boundary;
}

// The species' initial distribution (the object make_f0_return_ptr built,
// AMRSimulation_load.cpp:139-225) at n points.
int amrref_sim_f0(void* h, int sp, int n, const double* x, const double* p, double* out) {
    CallScope scope;
    distribution* f0 = static_cast<RefSim*>(h)->sim->ic_list[sp];
    try {
        for (int i = 0; i < n; ++i) out[i] = (*f0)(x[i], p[i]);
    } catch (...) {
        return 1;
    }
    return 0;
}

}  // extern "C"
