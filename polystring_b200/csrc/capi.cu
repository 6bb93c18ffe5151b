// capi.cu -- extern "C" entry points declared in include/polystring_b200.h.
// Every function catches C++ exceptions and maps them to status codes.
#include "polystring_b200.h"
#include "engine.h"
#include "field_kernels.h"
#include "string_ab.h"
#include "batch_ab.h"

#include <string>
#include <vector>

namespace ps {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return PS_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return PS_ERR_INVALID;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return PS_ERR_INVALID;
    }
}

static Cell to_cell(const ps_unit_cell* c) {
    if (!c) throw Error(PS_ERR_INVALID, "null unit cell");
    Cell r;
    r.dim = c->dim; r.system = c->system;
    r.a = c->a; r.b = c->b; r.c = c->c;
    r.alpha = c->alpha; r.beta = c->beta; r.gamma = c->gamma;
    return r;
}

static void check_dims(int dim, int Lx, int Ly, int Lz) {
    if (Lx < 1 || Ly < 1 || Lz < 1) throw Error(PS_ERR_INVALID, "grid sizes must be positive");
    if (dim < 1 || dim > 3) throw Error(PS_ERR_INVALID, "dimension must be 1, 2 or 3");
    if (dim == 1 && (Ly != 1 || Lz != 1)) throw Error(PS_ERR_INVALID, "1D grids need Ly = Lz = 1");
    if (dim == 2 && Lz != 1) throw Error(PS_ERR_INVALID, "2D grids need Lz = 1");
}

}  // namespace ps

using namespace ps;

struct ps_updater { UpdaterCtx* ctx; };
struct ps_model_ab { ModelAB* ctx; };
struct ps_string_ab { StringAB* ctx; };
struct ps_batch_ab { BatchAB* ctx; };
struct ps_model_abc { ModelABC* ctx; };

extern "C" {

const char* ps_version(void) { return "polystring_b200 0.1 (sm_100a, FP64)"; }

const char* ps_tuning_log(void) { return tuning_log(); }

const char* ps_last_error(void) { return g_last_error.c_str(); }

int ps_updater_create(int scheme, const ps_unit_cell* cell, int Lx, int Ly, int Lz, double ds, ps_updater** out) {
    return guarded([&] {
        if (!out) throw Error(PS_ERR_INVALID, "null output handle");
        if (scheme != PS_MDE_RQM4 && scheme != PS_MDE_OS2 && scheme != PS_MDE_ETDRK4)
            throw Error(PS_ERR_INVALID, "unknown MDE scheme");
        Cell c = to_cell(cell);
        check_dims(c.dim, Lx, Ly, Lz);
        const int sc = scheme == PS_MDE_RQM4 ? SCHEME_RQM4 : scheme == PS_MDE_OS2 ? SCHEME_OS2 : SCHEME_ETDRK4;
        *out = new ps_updater{new UpdaterCtx(sc, c, Lx, Ly, Lz, ds)};
    });
}

int ps_updater_create_etdrk4(const ps_unit_cell* cell, int Lx, int Ly, int Lz, double ds, int M, ps_updater** out) {
    return guarded([&] {
        if (!out) throw Error(PS_ERR_INVALID, "null output handle");
        if (M < 1) throw Error(PS_ERR_INVALID, "ETDRK4 needs at least one contour point");
        Cell c = to_cell(cell);
        check_dims(c.dim, Lx, Ly, Lz);
        *out = new ps_updater{new UpdaterCtx(SCHEME_ETDRK4, c, Lx, Ly, Lz, ds, M)};
    });
}

int ps_updater_clone(const ps_updater* u, ps_updater** out) {
    return guarded([&] {
        if (!u || !out) throw Error(PS_ERR_INVALID, "null handle");
        *out = new ps_updater{u->ctx->clone()};
    });
}

void ps_updater_destroy(ps_updater* u) {
    if (!u) return;
    delete u->ctx;
    delete u;
}

int ps_updater_solve(ps_updater* u, const double* w, double* qs, int len) {
    return guarded([&] {
        if (!u || !w || !qs) throw Error(PS_ERR_INVALID, "null argument");
        u->ctx->solve_host(w, qs, len);
    });
}

int ps_updater_solve_device(ps_updater* u, const double* w, double* qs, int len, void* stream) {
    return guarded([&] {
        if (!u || !w || !qs) throw Error(PS_ERR_INVALID, "null argument");
        u->ctx->solve_device(w, qs, len, (cudaStream_t)stream);
    });
}

int ps_density_solve_device(int rule, const double* q, const double* qc, int len, long long M, double ds, double cc,
                            double* phi, void* stream) {
    return guarded([&] {
        if (!q || !qc || !phi || M < 1 || len < 2) throw Error(PS_ERR_INVALID, "bad density arguments");
        std::vector<double> c;
        if (!contour_weights(rule, len - 1, c)) throw Error(PS_ERR_QUADRATURE, "contour rule precondition fails");
        cudaStream_t st = (cudaStream_t)stream;
        DevBuf dc(c.size());
        PS_CUDA(cudaMemcpyAsync(dc.p, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice, st));
        launch_density(q, qc, len - 1, (long)M, dc.p, ds, nullptr, cc, phi, 1, 0, 0, nullptr, st);
        // dc is freed on return: wait for the kernel that reads it
        PS_CUDA(cudaStreamSynchronize(st));
    });
}

int ps_density_solve(int rule, const double* q, const double* qc, int len, long long M, double ds, double cc,
                     double* phi) {
    return guarded([&] {
        if (!q || !qc || !phi || M < 1 || len < 2) throw Error(PS_ERR_INVALID, "bad density arguments");
        std::vector<double> c;
        if (!contour_weights(rule, len - 1, c)) throw Error(PS_ERR_QUADRATURE, "contour rule precondition fails");
        size_t n = (size_t)len * (size_t)M;
        DevBuf dq(n), dqc(n), dphi((size_t)M), dc(c.size());
        PS_CUDA(cudaMemcpy(dq.p, q, sizeof(double) * n, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMemcpy(dqc.p, qc, sizeof(double) * n, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMemcpy(dc.p, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
        launch_density(dq.p, dqc.p, len - 1, (long)M, dc.p, ds, nullptr, cc, dphi.p, 1, 0, 0, nullptr, 0);
        PS_CUDA(cudaMemcpy(phi, dphi.p, sizeof(double) * (size_t)M, cudaMemcpyDeviceToHost));
    });
}

int ps_grid_mean_device(const double* x, long long M, double* out_host, void* stream) {
    return guarded([&] {
        if (!x || !out_host || M < 1) throw Error(PS_ERR_INVALID, "bad arguments");
        cudaStream_t st = (cudaStream_t)stream;
        DevBuf partial((size_t)kRedBlocks * 8), res(1);
        launch_mean(x, (long)M, partial.p, res.p, st);
        PS_CUDA(cudaMemcpyAsync(out_host, res.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        PS_CUDA(cudaStreamSynchronize(st));
    });
}

static ModelABParams to_params(const ps_model_ab_params* p) {
    if (!p) throw Error(PS_ERR_INVALID, "null parameters");
    check_dims(p->dim, p->Lx, p->Ly, p->Lz);
    if (p->cell.dim != p->dim) throw Error(PS_ERR_INVALID, "cell dimension differs from grid dimension");
    if (p->mde != PS_MDE_RQM4 && p->mde != PS_MDE_OS2 && p->mde != PS_MDE_ETDRK4)
        throw Error(PS_ERR_INVALID, "unknown MDE scheme");
    if (p->scft != PS_SCFT_EM && p->scft != PS_SCFT_ANDERSON) throw Error(PS_ERR_INVALID, "unknown SCFT algorithm");
    ModelABParams q;
    q.dim = p->dim; q.Lx = p->Lx; q.Ly = p->Ly; q.Lz = p->Lz;
    q.cell = to_cell(&p->cell);
    q.sA = p->sA; q.sB = p->sB; q.chiN = p->chiN;
    q.lamA = p->lamA; q.lamB = p->lamB; q.lamYita = p->lamYita;
    q.mde = p->mde; q.scft = p->scft; q.n_anderson = p->n_anderson;
    q.compressible = p->compressible; q.contour = p->contour;
    q.etd_M = p->etdrk4_M;
    return q;
}

static ModelABCParams to_abc_params(const ps_model_abc_params* p) {
    if (!p) throw Error(PS_ERR_INVALID, "null parameters");
    check_dims(p->dim, p->Lx, p->Ly, p->Lz);
    if (p->cell.dim != p->dim) throw Error(PS_ERR_INVALID, "cell dimension differs from grid dimension");
    if (p->scft != PS_SCFT_EM && p->scft != PS_SCFT_ANDERSON) throw Error(PS_ERR_INVALID, "unknown SCFT algorithm");
    ModelABCParams q;
    q.dim = p->dim; q.Lx = p->Lx; q.Ly = p->Ly; q.Lz = p->Lz;
    q.cell = to_cell(&p->cell);
    q.s[0] = p->sA; q.s[1] = p->sB; q.s[2] = p->sC;
    q.chi[0] = p->chiAB; q.chi[1] = p->chiBC; q.chi[2] = p->chiAC;
    q.lam[0] = p->lamA; q.lam[1] = p->lamB; q.lam[2] = p->lamC; q.lam[3] = p->lamYita;
    q.scft = p->scft; q.n_anderson = p->n_anderson; q.contour = p->contour;
    return q;
}

int ps_model_abc_create(const ps_model_abc_params* p, ps_model_abc** out) {
    return guarded([&] {
        if (!p || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = new ps_model_abc{new ModelABC(to_abc_params(p))};
    });
}

void ps_model_abc_destroy(ps_model_abc* m) {
    if (!m) return;
    delete m->ctx;
    delete m;
}

int ps_model_abc_set_fields(ps_model_abc* m, const double* wA, const double* wB, const double* wC) {
    return guarded([&] {
        if (!m || !wA || !wB || !wC) throw Error(PS_ERR_INVALID, "null argument");
        const double* w[3] = {wA, wB, wC};
        m->ctx->set_fields(w, false);
    });
}

int ps_model_abc_update(ps_model_abc* m, int n_iter) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        m->ctx->update(n_iter);
    });
}

int ps_model_abc_Q(ps_model_abc* m, double* Q) {
    return guarded([&] {
        if (!m || !Q) throw Error(PS_ERR_INVALID, "null argument");
        *Q = m->ctx->Q();
    });
}

int ps_model_abc_H(ps_model_abc* m, double* H, double* Hw, double* Hs) {
    return guarded([&] {
        if (!m || !H || !Hw || !Hs) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->H(H, Hw, Hs);
    });
}

int ps_model_abc_residual(ps_model_abc* m, double* res) {
    return guarded([&] {
        if (!m || !res) throw Error(PS_ERR_INVALID, "null argument");
        *res = m->ctx->residual();
    });
}

int ps_model_abc_get(ps_model_abc* m, int which, double* out) {
    return guarded([&] {
        if (!m || !out) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->get(which, out, false);
    });
}

int ps_model_abc_synchronize(ps_model_abc* m) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        PS_CUDA(cudaStreamSynchronize(m->ctx->stream()));
    });
}

int ps_model_ab_create(const ps_model_ab_params* p, ps_model_ab** out) {
    return guarded([&] {
        if (!p || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = new ps_model_ab{new ModelAB(to_params(p))};
    });
}

void ps_model_ab_destroy(ps_model_ab* m) {
    if (!m) return;
    delete m->ctx;
    delete m;
}

int ps_model_ab_set_fields(ps_model_ab* m, const double* wA, const double* wB) {
    return guarded([&] {
        if (!m || !wA || !wB) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->set_fields(wA, wB, false);
    });
}

int ps_model_ab_set_fields_device(ps_model_ab* m, const double* wA, const double* wB) {
    return guarded([&] {
        if (!m || !wA || !wB) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->set_fields(wA, wB, true);
    });
}

int ps_model_ab_update(ps_model_ab* m, int n_iter) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        m->ctx->update(n_iter);
    });
}

int ps_model_ab_update_timed(ps_model_ab* m, int n_iter, double* total_ms, double* propagator_ms) {
    return guarded([&] {
        if (!m || !total_ms || !propagator_ms) throw Error(PS_ERR_INVALID, "null argument");
        *total_ms = m->ctx->update_timed(n_iter, propagator_ms);
    });
}

int ps_model_ab_propagate(ps_model_ab* m, int n_iter) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        m->ctx->propagate(n_iter);
    });
}

int ps_model_ab_H(ps_model_ab* m, double* H, double* Hw, double* Hs) {
    return guarded([&] {
        if (!m || !H || !Hw || !Hs) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->H(H, Hw, Hs);
    });
}

int ps_model_ab_residual(ps_model_ab* m, double* res) {
    return guarded([&] {
        if (!m || !res) throw Error(PS_ERR_INVALID, "null argument");
        *res = m->ctx->residual();
    });
}

int ps_model_ab_Q(ps_model_ab* m, double* Q) {
    return guarded([&] {
        if (!m || !Q) throw Error(PS_ERR_INVALID, "null argument");
        *Q = m->ctx->Q();
    });
}

int ps_model_ab_forward(ps_model_ab* m) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        m->ctx->forward_only();
    });
}

int ps_model_ab_grad_w(ps_model_ab* m, const double* dL_dphiA, const double* dL_dphiB, double dL_dQ,
                       double* dL_dwA, double* dL_dwB) {
    return guarded([&] {
        if (!m || !dL_dphiA || !dL_dphiB || !dL_dwA || !dL_dwB) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->grad_w(dL_dphiA, dL_dphiB, dL_dQ, dL_dwA, dL_dwB);
    });
}

int ps_model_ab_stress_checkpointed(ps_model_ab* m, int k, double* dF_dl) {
    return guarded([&] {
        if (!m || !dF_dl) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->stress_checkpointed(k, dF_dl);
    });
}

int ps_model_ab_stress(ps_model_ab* m, double* dF_dl) {
    return guarded([&] {
        if (!m || !dF_dl) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->stress(dF_dl);
    });
}

int ps_model_ab_get(ps_model_ab* m, int which, double* out) {
    return guarded([&] {
        if (!m || !out) throw Error(PS_ERR_INVALID, "null argument");
        m->ctx->get(which, out, false);
    });
}

int ps_model_ab_device_ptr(ps_model_ab* m, int which, double** out) {
    return guarded([&] {
        if (!m || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = m->ctx->device_ptr(which);
    });
}

int ps_model_ab_synchronize(ps_model_ab* m) {
    return guarded([&] {
        if (!m) throw Error(PS_ERR_INVALID, "null handle");
        m->ctx->sync();
    });
}

int ps_model_ab_launches_per_iteration(ps_model_ab* m) { return m ? m->ctx->launches_per_iteration() : -1; }

int ps_model_ab_launches_per_propagate(ps_model_ab* m) { return m ? m->ctx->launches_per_propagate() : -1; }

void* ps_model_ab_stream(ps_model_ab* m) { return m ? (void*)m->ctx->stream() : nullptr; }

int ps_string_ab_create(const ps_model_ab_params* p, int m, int max_iter, ps_string_ab** out) {
    return guarded([&] {
        if (!p || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = new ps_string_ab{new StringAB(to_params(p), m, max_iter)};
    });
}

int ps_string_ab_create_shard(const ps_model_ab_params* p, int m, int max_iter, int lo, int hi, ps_string_ab** out) {
    return guarded([&] {
        if (!p || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = new ps_string_ab{new StringAB(to_params(p), m, max_iter, lo, hi)};
    });
}

int ps_string_ab_relax(ps_string_ab* s) {
    return guarded([&] {
        if (!s) throw Error(PS_ERR_INVALID, "null handle");
        s->ctx->relax();
    });
}

int ps_string_ab_reparameterize(ps_string_ab* s) {
    return guarded([&] {
        if (!s) throw Error(PS_ERR_INVALID, "null handle");
        s->ctx->reparameterize();
    });
}

int ps_string_ab_device_ptr(ps_string_ab* s, int which, double** out) {
    return guarded([&] {
        if (!s || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = s->ctx->device_ptr(which);
    });
}

void* ps_string_ab_stream(ps_string_ab* s) { return s ? (void*)s->ctx->stream() : nullptr; }

void ps_string_ab_destroy(ps_string_ab* s) {
    if (!s) return;
    delete s->ctx;
    delete s;
}

int ps_string_ab_set_images(ps_string_ab* s, const double* wa, const double* wb) {
    return guarded([&] {
        if (!s || !wa || !wb) throw Error(PS_ERR_INVALID, "null argument");
        s->ctx->set_images(wa, wb, false);
    });
}

int ps_string_ab_iterate(ps_string_ab* s, int n) {
    return guarded([&] {
        if (!s) throw Error(PS_ERR_INVALID, "null handle");
        s->ctx->iterate(n);
    });
}

int ps_string_ab_H(ps_string_ab* s, double* H) {
    return guarded([&] {
        if (!s || !H) throw Error(PS_ERR_INVALID, "null argument");
        s->ctx->H(H);
    });
}

int ps_string_ab_S(ps_string_ab* s, double* S) {
    return guarded([&] {
        if (!s || !S) throw Error(PS_ERR_INVALID, "null argument");
        s->ctx->S(S);
    });
}

int ps_string_ab_get(ps_string_ab* s, int which, double* out) {
    return guarded([&] {
        if (!s || !out) throw Error(PS_ERR_INVALID, "null argument");
        s->ctx->get(which, out, false);
    });
}

int ps_string_ab_synchronize(ps_string_ab* s) {
    return guarded([&] {
        if (!s) throw Error(PS_ERR_INVALID, "null handle");
        s->ctx->sync();
    });
}

int ps_string_ab_launches_per_iteration(ps_string_ab* s) { return s ? s->ctx->launches_per_iteration() : -1; }

int ps_batch_ab_create(const ps_model_ab_params* p, int n, ps_batch_ab** out) {
    return guarded([&] {
        if (!p || !out || n < 1) throw Error(PS_ERR_INVALID, "bad batch arguments");
        std::vector<ModelABParams> ps;
        for (int k = 0; k < n; k++) ps.push_back(to_params(p + k));
        *out = new ps_batch_ab{new BatchAB(ps)};
    });
}

int ps_batch_ab_create_mixed(const ps_model_ab_params* p, int n, const ps_model_abc_params* q, int nq,
                             ps_batch_ab** out) {
    return guarded([&] {
        if (!out || n < 0 || nq < 0 || n + nq < 1 || (n > 0 && !p) || (nq > 0 && !q))
            throw Error(PS_ERR_INVALID, "bad batch arguments");
        std::vector<ModelABParams> ps;
        std::vector<ModelABCParams> qs;
        for (int k = 0; k < n; k++) ps.push_back(to_params(p + k));
        for (int k = 0; k < nq; k++) {
            qs.push_back(to_abc_params(q + k));
            if (qs.back().dim < 2) throw Error(PS_ERR_UNSUPPORTED, "batched solves need 2D or 3D grids");
        }
        *out = new ps_batch_ab{new BatchAB(ps, qs)};
    });
}

int ps_batch_ab_set_fields_abc(ps_batch_ab* b, int k, const double* wA, const double* wB, const double* wC) {
    return guarded([&] {
        if (!b || !wA || !wB || !wC) throw Error(PS_ERR_INVALID, "null argument");
        const double* w[3] = {wA, wB, wC};
        b->ctx->set_fields_abc(k, w, false);
    });
}

void ps_batch_ab_destroy(ps_batch_ab* b) {
    if (!b) return;
    delete b->ctx;
    delete b;
}

int ps_batch_ab_set_fields(ps_batch_ab* b, int k, const double* wA, const double* wB) {
    return guarded([&] {
        if (!b || !wA || !wB) throw Error(PS_ERR_INVALID, "null argument");
        b->ctx->set_fields(k, wA, wB, false);
    });
}

int ps_batch_ab_update(ps_batch_ab* b, int n_iter) {
    return guarded([&] {
        if (!b) throw Error(PS_ERR_INVALID, "null handle");
        b->ctx->update(n_iter);
    });
}

int ps_batch_ab_update_timed(ps_batch_ab* b, int n_iter, double* total_ms) {
    return guarded([&] {
        if (!b || !total_ms) throw Error(PS_ERR_INVALID, "null argument");
        *total_ms = b->ctx->update_timed(n_iter);
    });
}

int ps_batch_ab_H(ps_batch_ab* b, int k, double* H, double* Hw, double* Hs) {
    return guarded([&] {
        if (!b || !H || !Hw || !Hs) throw Error(PS_ERR_INVALID, "null argument");
        b->ctx->sync();
        if (k >= b->ctx->size_ab()) b->ctx->model_abc(k).H(H, Hw, Hs);
        else b->ctx->model(k).H(H, Hw, Hs);
    });
}

int ps_batch_ab_residual(ps_batch_ab* b, int k, double* res) {
    return guarded([&] {
        if (!b || !res) throw Error(PS_ERR_INVALID, "null argument");
        b->ctx->sync();
        *res = k >= b->ctx->size_ab() ? b->ctx->model_abc(k).residual() : b->ctx->model(k).residual();
    });
}

int ps_batch_ab_get(ps_batch_ab* b, int k, int which, double* out) {
    return guarded([&] {
        if (!b || !out) throw Error(PS_ERR_INVALID, "null argument");
        b->ctx->sync();
        if (k >= b->ctx->size_ab()) b->ctx->model_abc(k).get(which, out, false);
        else b->ctx->model(k).get(which, out, false);
    });
}

int ps_batch_ab_synchronize(ps_batch_ab* b) {
    return guarded([&] {
        if (!b) throw Error(PS_ERR_INVALID, "null handle");
        b->ctx->sync();
    });
}

int ps_batch_ab_launches_per_iteration(ps_batch_ab* b) { return b ? b->ctx->launches_per_iteration() : -1; }

int ps_batch_ab_launches_per_propagate(ps_batch_ab* b) { return b ? b->ctx->launches_per_propagate() : -1; }

int ps_batch_ab_gridpoint_steps(ps_batch_ab* b, double* out) {
    return guarded([&] {
        if (!b || !out) throw Error(PS_ERR_INVALID, "null argument");
        *out = b->ctx->gridpoint_steps_per_iteration();
    });
}

}  // extern "C"
