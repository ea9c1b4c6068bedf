// C ABI of libfs_b200: field plugin, host mesh and misc entry points.
// (The session entry points fs_sim_* live next to the simulation in fs_sim.cu.)
#include <functional>
#include <memory>

#include "fs_internal.h"

namespace fsb {

const char* last_error_cstr();

fs_status guard(const std::function<void()>& fn) {
    try {
        fn();
        set_last_error("");
        return FS_OK;
    } catch (const FsError& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return FS_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return FS_ERR_STATE;
    }
}

}  // namespace fsb

struct fs_field {
    fs_field_params prm{};
    std::unique_ptr<fsb::FieldEngine> engine;
    cudaStream_t st = nullptr;
    fsb::DevBuf<double> t, s, q, e;
    ~fs_field() {
        if (st) cudaStreamDestroy(st);
    }
    void check_errors(cudaStream_t stream) {
        FS_CUDA(cudaStreamSynchronize(stream));
        if (int* fe = engine->error_flag()) {
            int h = 0;
            FS_CUDA(cudaMemcpy(&h, fe, sizeof(int), cudaMemcpyDeviceToHost));
            if (h) {
                FS_CUDA(cudaMemset(fe, 0, sizeof(int)));
                fsb::fail((fs_status)h, "device wait timed out in the field kernel");
            }
        }
    }
};

extern "C" {

fs_status fs_field_create(const fs_field_params* params, fs_field** out) {
    if (!params || !out) return fsb::guard([] { fsb::fail(FS_ERR_ARG, "null argument"); });
    *out = nullptr;
    auto* f = new fs_field();
    fs_status rc = fsb::guard([&] {
        const fs_field_params& P = *params;
        if (!(P.epsilon > 0)) fsb::fail(FS_ERR_ARG, "epsilon must be positive");
        if (P.kind != FS_FIELD_DIRECT64_OPEN && !(P.L > 0)) fsb::fail(FS_ERR_ARG, "L must be positive");
        f->prm = P;
        FS_CUDA(cudaSetDevice(P.device));
        FS_CUDA(cudaStreamCreateWithFlags(&f->st, cudaStreamNonBlocking));
        switch (P.kind) {
            case FS_FIELD_DIRECT64: f->engine.reset(fsb::make_direct64(P.L, P.epsilon)); break;
            case FS_FIELD_DIRECT32C: f->engine.reset(fsb::make_direct32c(P.L, P.epsilon)); break;
            case FS_FIELD_DIRECT64_OPEN: f->engine.reset(fsb::make_direct64_open(P.epsilon)); break;
            case FS_FIELD_TREECODE64:
            case FS_FIELD_TREECODE32C:
                if (P.degree < 1 || P.degree > 16) fsb::fail(FS_ERR_ARG, "treecode degree must be 1..16");
                if (P.max_source < 2) fsb::fail(FS_ERR_ARG, "treecode max_source must be >= 2");
                f->engine.reset(fsb::make_treecode(P.L, P.epsilon, P.mac, P.degree, P.max_source,
                                                   P.kind == FS_FIELD_TREECODE32C));
                break;
            default: fsb::fail(FS_ERR_ARG, "unknown field kind");
        }
    });
    if (rc != FS_OK) {
        delete f;
        return rc;
    }
    *out = f;
    return FS_OK;
}

fs_status fs_field_destroy(fs_field* field) {
    return fsb::guard([&] {
        if (field) {
            cudaSetDevice(field->prm.device);
            delete field;
        }
    });
}

fs_status fs_field_eval(fs_field* field, double* es, const double* targets, int nt, const double* sources,
                        const double* q_ws, int ns) {
    return fsb::guard([&] {
        if (!field || nt < 0 || ns < 0) fsb::fail(FS_ERR_ARG, "bad argument");
        if ((nt > 0 && (!es || !targets)) || (ns > 0 && (!sources || !q_ws))) fsb::fail(FS_ERR_ARG, "null array");
        const bool tree = field->prm.kind == FS_FIELD_TREECODE64 || field->prm.kind == FS_FIELD_TREECODE32C;
        if (tree && nt != ns) fsb::fail(FS_ERR_ARG, "treecode evaluates at the sources: nt must equal ns");
        FS_CUDA(cudaSetDevice(field->prm.device));
        cudaStream_t st = field->st;
        field->t.ensure(std::max(nt, 1));
        field->s.ensure(std::max(ns, 1));
        field->q.ensure(std::max(ns, 1));
        field->e.ensure(std::max(nt, 1));
        const bool same = (targets == sources) && nt == ns;
        if (ns) {
            FS_CUDA(cudaMemcpyAsync(field->s.p, sources, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
            FS_CUDA(cudaMemcpyAsync(field->q.p, q_ws, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
        }
        if (nt && !same)
            FS_CUDA(cudaMemcpyAsync(field->t.p, targets, sizeof(double) * nt, cudaMemcpyHostToDevice, st));
        fsb::Stage S;
        S.kind = fsb::STAGE_STORE;
        S.out = field->e.p;
        if (nt) {
            field->engine->eval(same ? field->s.p : field->t.p, nt, field->s.p, field->q.p, ns, S, st);
            FS_CUDA(cudaMemcpyAsync(es, field->e.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, st));
        }
        field->check_errors(st);
    });
}

fs_status fs_field_eval_device(fs_field* field, double* d_es, const double* d_targets, int nt,
                               const double* d_sources, const double* d_q_ws, int ns, void* stream) {
    return fsb::guard([&] {
        if (!field || nt < 0 || ns < 0) fsb::fail(FS_ERR_ARG, "bad argument");
        const bool tree = field->prm.kind == FS_FIELD_TREECODE64 || field->prm.kind == FS_FIELD_TREECODE32C;
        if (tree && nt != ns) fsb::fail(FS_ERR_ARG, "treecode evaluates at the sources: nt must equal ns");
        FS_CUDA(cudaSetDevice(field->prm.device));
        cudaStream_t st = stream ? (cudaStream_t)stream : field->st;
        fsb::Stage S;
        S.kind = fsb::STAGE_STORE;
        S.out = d_es;
        if (nt) field->engine->eval(d_targets, nt, d_sources, d_q_ws, ns, S, st);
    });
}

fs_status fs_mesh_sizes(int initial_height, int p_height, int* npoints, int* npanels, int* nleaves) {
    return fsb::guard([&] {
        fsb::HostMesh m;
        m.build(initial_height, p_height, 0.0, 1.0, 0.0, 1.0);
        if (npoints) *npoints = (int)m.xs.size();
        if (npanels) *npanels = (int)m.panels.size();
        if (nleaves) *nleaves = (int)m.leaves.size();
    });
}

fs_status fs_mesh_fill(int initial_height, int p_height, double xmin, double xmax, double pmin, double pmax,
                       double q, int quadrature, double* xs, double* ps, int* panels, int* leaves,
                       double* base_weights) {
    return fsb::guard([&] {
        fsb::HostMesh m;
        m.build(initial_height, p_height, xmin, xmax, pmin, pmax);
        if (xs) std::memcpy(xs, m.xs.data(), sizeof(double) * m.xs.size());
        if (ps) std::memcpy(ps, m.ps.data(), sizeof(double) * m.ps.size());
        if (panels) m.panel_records(panels);
        if (leaves) std::memcpy(leaves, m.leaves.data(), sizeof(int) * m.leaves.size());
        if (base_weights) {
            std::vector<double> w = m.base_weights(q, quadrature);
            std::memcpy(base_weights, w.data(), sizeof(double) * w.size());
        }
    });
}

const char* fs_last_error(void) { return fsb::last_error_cstr(); }

int fs_version(void) { return 100; }

long long fs_kernel_launches(void) { return fsb::launches(); }

}  // extern "C"
