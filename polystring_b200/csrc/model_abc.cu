// model_abc.cu -- a linear A-B-C triblock melt on the device.
//
// The reference has no periodic ABC melt model (its polystring_ABC drives an
// AB diblock with a grafted C brush in a Chebyshev slab), so this model is
// defined here, by extending Model_AB (Model_AB.cc:85-371) term by term:
//   * blocks of sA, sB, sC contour points, L = LA + LB + LC, fX = LX / L,
//     dsX = fX / LX;
//   * forward chain qA -> qB -> qC from 1, complementary chain qCc -> qBc ->
//     qAc from 1, each block's head the previous block's tail
//     (Model_AB.cc:187-193 with a third block); Q = mean(qC tail);
//   * phiX = dsX / Q sum_s c_s qX[s] qXc[LX - s] with Simpson or Quad4_Closed
//     by the parity of Ms (Model_AB.cc:713-735);
//   * targets wA* = chiAB phiB + chiAC phiC + eta, wB* = chiAB phiA +
//     chiBC phiC + eta, wC* = chiAC phiA + chiBC phiB + eta;
//   * simple mixing: eta += lam_eta (phiA + phiB + phiC - 1), then
//     wX = wX (1 - lamX) + lamX wX* (Field.cc:51-59, Yita.cc:49-55);
//   * Anderson mixing: eta = (wA + wB + wC - chiAB (phiA + phiB) - chiBC
//     (phiB + phiC) - chiAC (phiA + phiC)) / 3, so that the targets sum to
//     the current fields (Model_AB's 0.5 (wA + wB - chiN) is the two-block
//     case with phiA + phiB = 1); one FieldAX ring per field and one
//     coefficient set from U = UA + UB + UC, V = VA + VB + VC;
//   * Hw = mean(chiAB phiA phiB + chiBC phiB phiC + chiAC phiA phiC -
//     sum_X wX phiX), Hs = -ln Q; the residuals of Model_AB with a third field.
// Incompressible, RQM4, orthogonal k^2 table.  Propagation: the 64^3 sweep
// (sweep64.cu) on 64^3 grids and the generic persistent sweep (sweep.cu) on
// 32^3 and 48^3 grids, each given three factor sets; the packed line passes
// (PairChain) on other grids.
#include <cmath>
#include <cstdlib>
#include <string>

#include "engine.h"
#include "field_kernels.h"

namespace ps {

ModelABC::ModelABC(const ModelABCParams& p) : p_(p) {
    cell_init(p_.cell);
    M_ = (long)p.Lx * p.Ly * p.Lz;
    if (p.scft == 1 && (p.n_anderson < 1 || ax_nmax(p.n_anderson) == 0))
        throw Error(-1, "n_Anderson_mixing must be 1..31");
    Ns_ = 0;
    for (int x = 0; x < 3; x++) {
        if (p.s[x] < 2) throw Error(-1, "every block needs at least two contour points");
        L_[x] = p.s[x] - 1;
        Ns_ += L_[x];
    }
    std::vector<double> cw[3];
    for (int x = 0; x < 3; x++) {
        const double f = 1.0 * L_[x] / Ns_;
        ds_[x] = f / L_[x];
        const int rule = p.contour == 0 ? 0 : ((p.s[x] % 2 != 0) ? 1 : 2);
        if (!contour_weights(rule, L_[x], cw[x]))
            throw Error(-4, "contour quadrature precondition fails for block " + std::to_string(x) + " (Ms " +
                                std::to_string(p.s[x]) + ")");
    }
    PS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    chain_ = new PairChain(p.Lx, p.Ly, p.Lz, SCHEME_RQM4, 1);
    // the packed lanes share the block-A tables; the three ds agree to a
    // few ulps (each rounds 1 / L)
    std::vector<double> k2 = k2_orthogonal(p_.cell, p.Lx, p.Ly, p.Lz);
    std::vector<double> L1(M_), L2(M_);
    for (long m = 0; m < M_; m++) {
        L1[m] = exp(ds_[0] * k2[m]);
        L2[m] = exp(0.5 * ds_[0] * k2[m]);
    }
    chain_->set_tables(L1, L2);
    const char* force = getenv("PS_B200_LINE_PASSES");
    const char* generic = getenv("PS_B200_GENERIC_SWEEP");
    const bool allow = !(force && force[0] == '1');
    // 64^3 grids take the 64^3 sweep where its clusters fit (as Model_AB)
    use_sweep64_ = allow && sweep64_supported(p.Lx, p.Ly, p.Lz) && !(generic && generic[0] == '1');
    if (use_sweep64_) {
        sweep_grid_ = sweep64_prepare();
        use_sweep64_ = sweep_grid_ > 0;
    }
    use_sweep_ = allow && !use_sweep64_ && sweep_supported(p.Lx, p.Ly, p.Lz);
    if (use_sweep64_) {
        swZ_.alloc(6 * (size_t)M_);
        const std::vector<double> tab = sweep64_axis_tables(p_.cell.l, ds_[0]);
        swTab_.alloc(tab.size());
        PS_CUDA(cudaMemcpy(swTab_.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
        PS_CUDA(cudaMalloc(&swbar_, 64 * sizeof(unsigned)));
        PS_CUDA(cudaMalloc(&swerr_, sizeof(int)));
        PS_CUDA(cudaMemset(swerr_, 0, sizeof(int)));
    }
    if (use_sweep_) {
        sweep_grid_ = sweep_prepare(p.Lx, p.Ly, p.Lz);
        swZ_.alloc(6 * (size_t)M_);
        swU_.alloc(2 * (size_t)M_);
        swL1_.alloc(M_);
        swL2_.alloc(M_);
        PS_CUDA(cudaMemcpy(swL1_.p, L1.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMemcpy(swL2_.p, L2.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMalloc(&swbar_, 32 * sizeof(unsigned)));
        PS_CUDA(cudaMalloc(&swerr_, sizeof(int)));
        PS_CUDA(cudaMemset(swerr_, 0, sizeof(int)));
    }
    hf_.alloc((size_t)(Ns_ + 1) * M_);
    hc_.alloc((size_t)(Ns_ + 1) * M_);
    yita_.alloc(M_);
    for (int x = 0; x < 3; x++) {
        w_[x].alloc(M_); phi_[x].alloc(M_); eF_[x].alloc(M_); eH_[x].alloc(M_);
        c_[x].alloc(cw[x].size());
        PS_CUDA(cudaMemcpy(c_[x].p, cw[x].data(), sizeof(double) * cw[x].size(), cudaMemcpyHostToDevice));
    }
    scal_.alloc(32);
    partial_.alloc((size_t)kRedBlocks * 128);
    if (p.scft == 1) {
        const size_t n1 = (size_t)p.n_anderson + 1;
        for (int x = 0; x < 3; x++) {
            hw_[x].alloc(n1 * M_); hd_[x].alloc(n1 * M_); B_[x].alloc(n1 * n1);
        }
        PS_CUDA(cudaMalloc(&axs_, sizeof(AXState)));
    }
    launch_fill(hf_.p, M_, 1.0, st_);
    launch_fill(hc_.p, M_, 1.0, st_);
    launch_fill(yita_.p, M_, 0.0, st_);
    if (!use_sweep_ && !use_sweep64_) chain_->autotune(st_);
    PS_CUDA(cudaStreamSynchronize(st_));
}

ModelABC::~ModelABC() {
    if (graph_) cudaGraphExecDestroy(graph_);
    delete chain_;
    if (axs_) cudaFree(axs_);
    if (swbar_) cudaFree(swbar_);
    if (swerr_) cudaFree(swerr_);
    if (st_) cudaStreamDestroy(st_);
}

void ModelABC::set_fields(const double* const w[3], bool dev) {
    const auto kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int x = 0; x < 3; x++)
        PS_CUDA(cudaMemcpyAsync(w_[x].p, w[x], sizeof(double) * M_, kind, st_));
    launch_fill(yita_.p, M_, 0.0, st_);
    if (p_.scft == 1) {
        const int n = p_.n_anderson;
        const size_t n1 = (size_t)n + 1;
        for (int x = 0; x < 3; x++) {
            PS_CUDA(cudaMemsetAsync(hw_[x].p, 0, sizeof(double) * n1 * M_, st_));
            PS_CUDA(cudaMemsetAsync(hd_[x].p, 0, sizeof(double) * n1 * M_, st_));
            PS_CUDA(cudaMemsetAsync(B_[x].p, 0, sizeof(double) * n1 * n1, st_));
            // FieldAX::update_w0 (FieldAX.cc:274-280): w(n) = w0
            PS_CUDA(cudaMemcpyAsync(hw_[x].p + (size_t)n * M_, w[x], sizeof(double) * M_, kind, st_));
        }
        AXState s{};
        s.n = n; s.k = 0; s.cur = n; s.cur_old = n; s.cur_new = n;
        s.lamA = p_.lam[0]; s.lamB = p_.lam[1]; s.lamC = p_.lam[2];
        PS_CUDA(cudaMemcpyAsync(axs_, &s, sizeof(AXState), cudaMemcpyHostToDevice, st_));
    }
    // exp(-w ds/2), exp(-w ds/4) of the first iteration
    launch_factors(w_[0].p, w_[1].p, M_, ds_[0], ds_[1], eF_[0].p, eH_[0].p, eF_[1].p, eH_[1].p, 1, 0, st_);
    launch_factors(w_[2].p, w_[2].p, M_, ds_[2], ds_[2], eF_[2].p, eH_[2].p, eF_[2].p, eH_[2].p, 1, 0, st_);
    PS_CUDA(cudaStreamSynchronize(st_));
    iter_ = 0;
    fields_set_ = true;
}

SweepArgs ModelABC::sweep_descriptor() const {
    if (!use_sweep_) throw Error(-2, "this solve has no generic persistent sweep");
    SweepArgs a{};
    a.hf = hf_.p; a.hc = hc_.p;
    a.Z1 = swZ_.c(); a.Z2 = swZ_.c() + M_; a.Z3 = swZ_.c() + 2 * M_;
    a.uf = swU_.p; a.uc = swU_.p + M_;
    a.eFA = eF_[0].p; a.eHA = eH_[0].p; a.eFB = eF_[1].p; a.eHB = eH_[1].p; a.eFC = eF_[2].p; a.eHC = eH_[2].p;
    a.L1 = swL1_.p; a.L2 = swL2_.p;
    a.LA = L_[0]; a.LB = L_[1]; a.LC = L_[2]; a.Ns = Ns_;
    a.bar = swbar_; a.err = swerr_;
    return a;
}

void ModelABC::enqueue_propagate(cudaStream_t s) {
    if (use_sweep64_) {
        SweepArgs a{};
        a.hf = hf_.p; a.hc = hc_.p;
        a.Z1 = swZ_.c(); a.Z2 = swZ_.c() + M_; a.Z3 = swZ_.c() + 2 * M_;
        a.eFA = eF_[0].p; a.eHA = eH_[0].p; a.eFB = eF_[1].p; a.eHB = eH_[1].p; a.eFC = eF_[2].p; a.eHC = eH_[2].p;
        a.LA = L_[0]; a.LB = L_[1]; a.LC = L_[2]; a.Ns = Ns_;
        a.bar = swbar_; a.err = swerr_;
        PS_CUDA(cudaMemsetAsync(swbar_, 0, 64 * sizeof(unsigned), s));
        sweep64_launch(a, swTab_.p, sweep_grid_, s);
        return;
    }
    if (use_sweep_) {
        const SweepArgs a = sweep_descriptor();
        PS_CUDA(cudaMemsetAsync(swbar_, 0, 32 * sizeof(unsigned), s));
        sweep_launch(a, p_.Lx, p_.Ly, p_.Lz, sweep_grid_, 1, s, sweep_default_variant(p_.Lx, p_.Ly, p_.Lz));
        return;
    }
    // lane f: A for t < LA, B up to LA + LB, then C; lane c: C, B, A
    LaneFactors lf{{eF_[0].p, eF_[1].p, eF_[2].p}, {eH_[0].p, eH_[1].p, eH_[2].p}, L_[0], L_[0] + L_[1]};
    LaneFactors lc{{eF_[2].p, eF_[1].p, eF_[0].p}, {eH_[2].p, eH_[1].p, eH_[0].p}, L_[2], L_[2] + L_[1]};
    chain_->enqueue(hf_.p, hc_.p, 0, Ns_, lf, lc, 0, s);
}

void ModelABC::enqueue_post(cudaStream_t st) {
    double* dQ = scal_.p + 0;
    launch_mean(hf_.p + (long)Ns_ * M_, M_, partial_.p, dQ, st);
    // block X spans forward slices [oX, oX + LX]; its complementary slices
    // run backwards from Ns - oX
    const long o[3] = {0, L_[0], (long)L_[0] + L_[1]};
    for (int x = 0; x < 3; x++) {
        const long oc = Ns_ - o[x] - L_[x];
        launch_density(hf_.p + o[x] * M_, hc_.p + oc * M_, L_[x], M_, c_[x].p, ds_[x], dQ, 0.0, phi_[x].p, 1, 0, 0,
                       nullptr, st);
    }
    if (p_.scft == 1) {
        AXArgs a{};
        a.state = axs_; a.n = p_.n_anderson; a.M = M_; a.nf = 3;
        a.phiA = phi_[0].p; a.phiB = phi_[1].p; a.phiC = phi_[2].p;
        a.dataA = w_[0].p; a.dataB = w_[1].p; a.dataC = w_[2].p;
        a.wA = hw_[0].p; a.dA = hd_[0].p; a.wB = hw_[1].p; a.dB = hd_[1].p; a.wC = hw_[2].p; a.dC = hd_[2].p;
        a.BA = B_[0].p; a.BB = B_[1].p; a.BC = B_[2].p;
        a.yita = yita_.p;
        a.dsA = ds_[0]; a.dsB = ds_[1]; a.dsC = ds_[2];
        a.eFA = eF_[0].p; a.eHA = eH_[0].p; a.eFB = eF_[1].p; a.eHB = eH_[1].p; a.eFC = eF_[2].p; a.eHC = eH_[2].p;
        for (int k = 0; k < 3; k++) a.chi[k] = p_.chi[k];
        launch_anderson(a, partial_.p, st);
    } else {
        EMABCArgs a{};
        for (int x = 0; x < 3; x++) {
            a.phi[x] = phi_[x].p; a.w[x] = w_[x].p; a.eF[x] = eF_[x].p; a.eH[x] = eH_[x].p;
            a.ds[x] = ds_[x]; a.chi[x] = p_.chi[x];
        }
        for (int k = 0; k < 4; k++) a.lam[k] = p_.lam[k];
        a.yita = yita_.p;
        a.M = M_;
        launch_em_update_abc(a, st);
    }
}

void ModelABC::enqueue_iteration(cudaStream_t st) {
    if (!fields_set_) throw Error(-6, "fields are not set");
    enqueue_propagate(st);
    enqueue_post(st);
}

void ModelABC::update(int n) {
    if (!fields_set_) throw Error(-6, "fields are not set");
    if (!graph_) {
        PS_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t g = nullptr;
        try {
            enqueue_iteration(st_);
        } catch (...) {
            cudaStreamEndCapture(st_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        PS_CUDA(cudaStreamEndCapture(st_, &g));
        cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Error(-3, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    for (int i = 0; i < n; i++) PS_CUDA(cudaGraphLaunch(graph_, st_));
    iter_ += n > 0 ? n : 0;
}

double ModelABC::Q() {
    if (iter_ == 0) throw Error(-6, "no iteration has run");
    double q = 0;
    PS_CUDA(cudaMemcpyAsync(&q, scal_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    return q;
}

void ModelABC::H(double* H, double* Hw, double* Hs) {
    if (iter_ == 0) throw Error(-6, "no iteration has run");
    const double* phi[3] = {phi_[0].p, phi_[1].p, phi_[2].p};
    const double* w[3] = {w_[0].p, w_[1].p, w_[2].p};
    launch_Hw_abc(phi, w, p_.chi, M_, partial_.p, scal_.p + 1, st_);
    double h[2];
    PS_CUDA(cudaMemcpyAsync(h, scal_.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    *Hw = h[1];
    *Hs = -log(h[0]);
    *H = *Hw + *Hs;
}

double ModelABC::residual() {
    if (iter_ == 0) throw Error(-6, "no iteration has run");
    if (p_.scft == 1) {
        const int n = p_.n_anderson;
        const int cur = n - (int)(iter_ % (n + 1));
        int pos = cur + 1;
        if (pos > n) pos = 0;
        const double* d[3];
        const double* w[3];
        for (int x = 0; x < 3; x++) {
            d[x] = hd_[x].p + (long)pos * M_;
            w[x] = hw_[x].p + (long)pos * M_;
        }
        launch_residual_ax_abc(d, w, M_, partial_.p, scal_.p + 2, st_);
        double e[6];
        PS_CUDA(cudaMemcpyAsync(e, scal_.p + 2, sizeof(double) * 6, cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        return sqrt((e[0] + e[2] + e[4]) / (e[1] + e[3] + e[5]));
    }
    const double* phi[3] = {phi_[0].p, phi_[1].p, phi_[2].p};
    const double* w[3] = {w_[0].p, w_[1].p, w_[2].p};
    launch_residual_em_abc(phi, w, yita_.p, p_.chi, M_, partial_.p, scal_.p + 2, st_);
    double v[11];
    PS_CUDA(cudaMemcpyAsync(v, scal_.p + 2, sizeof(double) * 11, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    double res = 0.0;
    for (int x = 0; x < 3; x++) res += v[3 * x] / (v[3 * x + 1] + v[3 * x + 2]);
    res += v[9] / (1.0 + v[10]);
    return res / 4.0;
}

void ModelABC::get(int which, double* out, bool device_dst) {
    const double* src = nullptr;
    if (which >= 0 && which < 3) src = w_[which].p;
    else if (which >= 3 && which < 6) src = phi_[which - 3].p;
    else if (which == 6) src = yita_.p;
    else throw Error(-1, "unknown field");
    PS_CUDA(cudaMemcpyAsync(out, src, sizeof(double) * M_, device_dst ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

int ModelABC::status() {
    int st = 0;
    if (axs_) {
        AXState s;
        PS_CUDA(cudaMemcpyAsync(&s, axs_, sizeof(AXState), cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        st |= s.status;
    }
    if (swerr_) {
        int e = 0;
        PS_CUDA(cudaMemcpyAsync(&e, swerr_, sizeof(int), cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        if (e) st |= 2;
    }
    return st;
}

}  // namespace ps
