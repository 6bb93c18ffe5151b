// adjoint.cu -- reverse-mode differentiation of the discrete RQM4 chain.
//
// Forward map at fixed fields (Model_AB.cc:136-199): chains f (qA -> qB) and
// c (qBc -> qAc), Q = mean f[Ns], phiA = dsA sum_t cA_t f[t] c[Ns-t] / Q,
// phiB likewise.  Every split step S = e (.) K (e (.) x) with
// K = F^-1 diag(L) F / M is symmetric, hence so is the RQM4 step
// A = (4 S' S' - S) / 3, and the adjoint recursion
//
//     lambda[t] = A lambda[t+1] + D[t]          (D: direct density terms)
//
// is the same step applied backwards.  One adjoint step packs q[t] (from
// the stored forward history) in the real lane and lambda[t+1] in the
// imaginary lane of one complex field; its intermediates give the exact
// discrete w-gradient of the step (line_pass.cu MODE_END_ADJ) and, from the
// spectra of the three packed fields, the derivative with respect to the cell
// lengths through the k-space factors exp(-h k^2):
//
//   lambda' dS/dl q = (1/M) sum_k dL_k/dl conj(F[e lambda])_k F[e q]_k
//                   = (1/2M) sum_k dL_k/dl Im(Z_k Z_-k)   (Z = F[e q + i e lambda])
//
// The forward histories q are the ones the densities already need, resident
// in HBM after forward_only(); the reverse sweep reads them instead of
// recomputing them.  d(-ln Q)/dl at fixed fields is the stress used for cell
// optimisation (at an SCFT saddle point it equals dF/dl up to the contour
// quadrature error of the densities).
#include "engine.h"
#include "field_kernels.h"

#include <cmath>

namespace ps {

namespace {

constexpr int kAT = 256;
constexpr int kAG = 148;   // blocks of the per-step stress reductions

__global__ void lam_init_kernel(double* lam, long M, const double* pA, const double* pB, double wA, double wB,
                                const double* other, double cst) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        double v = cst;
        if (pA) v += (wA * pA[i] + wB * pB[i]) * other[i];
        lam[i] = v;
    }
}

__global__ void scale2_kernel(const double* a, const double* b, double s, double* oa, double* ob, long M) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        oa[i] = a[i] * s;
        ob[i] = b[i] * s;
    }
}

// per-step partial sums of the cell-length derivative of lambda' A q:
// (4/3)[lambda' dS' u + v' dS' q] - (1/3) lambda' dS q, times M, for the
// three cell lengths; spec0 = F[eF(q + i lambda)], spec1 = F[eH(q + i lambda)],
// spec2 = F[eH(u + i v)] with u = S'q, v = S'lambda.
struct StressArgs {
    const double2 *s0, *s1, *s2;
    const double *L1, *L2;
    int Lx, Ly, Lz;
    double cx, cy, cz;      // ds 8 pi^2 / l^3 per axis (full step); half step uses ds/2
    double* partial;        // [gridDim.x][3]
};

__global__ void __launch_bounds__(kAT) stress_step_kernel(StressArgs a) {
    const long M = (long)a.Lx * a.Ly * a.Lz;
    double acc[3] = {0.0, 0.0, 0.0};
    const long stride = (long)gridDim.x * blockDim.x;
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < M; g += stride) {
        const int kz = (int)(g % a.Lz);
        const int ky = (int)((g / a.Lz) % a.Ly);
        const int kx = (int)(g / ((long)a.Ly * a.Lz));
        const int nx = (a.Lx - kx) % a.Lx, ny = (a.Ly - ky) % a.Ly, nz = (a.Lz - kz) % a.Lz;
        const long gn = ((long)nx * a.Ly + ny) * a.Lz + nz;
        const double2 z1 = a.s0[g], z1n = a.s0[gn];
        const double2 z2 = a.s1[g], z2n = a.s1[gn];
        const double2 z3 = a.s2[g], z3n = a.s2[gn];
        // 0.5 Im(Z1_k Z1_-k) = Re(conj(F[eF lambda]) F[eF q])
        const double t1 = 0.5 * (z1.x * z1n.y + z1.y * z1n.x);
        // F[eH q] = (Z2 + conj Z2n)/2, F[eH lambda] = (Z2 - conj Z2n)/(2i), same for u, v from Z3
        const double fq_r = 0.5 * (z2.x + z2n.x), fq_i = 0.5 * (z2.y - z2n.y);
        const double fl_r = 0.5 * (z2.y + z2n.y), fl_i = -0.5 * (z2.x - z2n.x);
        const double fu_r = 0.5 * (z3.x + z3n.x), fu_i = 0.5 * (z3.y - z3n.y);
        const double fv_r = 0.5 * (z3.y + z3n.y), fv_i = -0.5 * (z3.x - z3n.x);
        // Re(conj(Fl) Fu + conj(Fv) Fq)
        const double t2 = (fl_r * fu_r + fl_i * fu_i) + (fv_r * fq_r + fv_i * fq_i);
        const int rx = (kx < a.Lx / 2 + 1) ? kx : a.Lx - kx;
        const int ry = (ky < a.Ly / 2 + 1) ? ky : a.Ly - ky;
        const int rz = (kz < a.Lz / 2 + 1) ? kz : a.Lz - kz;
        const double l1 = a.L1[g], l2 = a.L2[g];
        const double r2[3] = {(double)rx * rx, (double)ry * ry, (double)rz * rz};
        const double cc[3] = {a.cx, a.cy, a.cz};
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const double d1 = l1 * cc[i] * r2[i];          // dL1/dl_i
            const double d2 = l2 * (0.5 * cc[i]) * r2[i];  // dL2/dl_i
            acc[i] += (4.0 / 3.0) * t2 * d2 - (1.0 / 3.0) * t1 * d1;
        }
    }
    __shared__ double sh[3][kAT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double v = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[i][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int w = 0; w < kAT / 32; w++) s += sh[threadIdx.x][w];
        a.partial[(long)blockIdx.x * 3 + threadIdx.x] = s;
    }
}

// sum of all per-step partials in a fixed order
__global__ void stress_final_kernel(const double* partial, long n, double scale, double* out) {
    if (threadIdx.x >= 3 || blockIdx.x != 0) return;
    double s = 0.0;
    for (long j = 0; j < n; j++) s += partial[j * 3 + threadIdx.x];
    out[threadIdx.x] = s * scale;
}

int egrid(long M) {
    long g = (M + kAT - 1) / kAT;
    if (g > 148L * 8) g = 148L * 8;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

// One adjoint sweep of a chain (see the file comment and AdjointSweep).
void PairChain::enqueue_adjoint(AdjointSweep& s, cudaStream_t st) {
    if (scheme_ != SCHEME_RQM4) throw Error(-2, "the adjoint is provided for RQM4");
    if (plan_.naxes < 2) throw Error(-2, "the adjoint needs a 2D or 3D grid");
    const long M = M_;
    const int Ns = s.Ns;
    const LineGeom& in = plan_.ax[0];
    const LineGeom& out = plan_.ax[plan_.naxes - 1];
    const LineGeom* mid = (plan_.naxes == 3) ? &plan_.ax[1] : nullptr;
    if (half_.n < 2 * (size_t)M) half_.alloc(2 * (size_t)M);
    const int t_hi = s.t_hi > 0 ? s.t_hi : Ns, t_lo = s.t_lo;
    int cur = s.lam_cur;
    if (t_hi == Ns) {
        // lambda[Ns]
        lam_init_kernel<<<egrid(M), kAT, 0, st>>>(s.lam[0], M, s.pbarA, s.pbarB, s.wd[0][Ns], s.wd[1][Ns],
                                                    s.ho, s.cst_Ns);
        PS_CUDA(cudaGetLastError());
        cur = 0;
    }
    for (int t = t_hi - 1; t >= t_lo; t--) {
        const int X = s.blk[t];
        StepPtrs p{};
        p.M = (double)M;
        p.bstride_z = M; p.bstride_u = M;
        p.u[0] = u_[0].p; p.u[1] = u_[1].p;
        p.half[0] = half_.p; p.half[1] = half_.p + M;
        p.z[0] = z_[0].c(); p.z[1] = z_[1].c(); p.z[2] = z_[2].c();
        p.L[0] = L1_.p; p.L[1] = L2_.p; p.L[2] = L2_.p;
        p.qin[0] = s.hq + (long)(t - s.hq_base) * M;
        p.qin[1] = s.lam[cur];
        p.qout[1] = s.lam[cur ^ 1];
        p.qout[0] = nullptr;
        p.eF[0] = p.eF[1] = s.eF[X];
        p.eH[0] = p.eH[1] = s.eH[X];
        p.grad = s.grad[X];
        p.gds = s.ds[X];
        if (s.pbarA) {
            p.pbarA = s.pbarA; p.pbarB = s.pbarB;
            p.other = s.ho + (long)(Ns - t) * M;
            p.wdA = s.wd[0][t]; p.wdB = s.wd[1][t];
        }
        if (t > t_lo) {
            const int Xn = s.blk[t - 1];
            p.chain_next = 1;
            p.nF[0] = p.nF[1] = s.eF[Xn];
            p.nH[0] = p.nH[1] = s.eH[Xn];
            p.next_qf = s.hq + (long)(t - 1 - s.hq_base) * M;
        }
        if (s.spec) { p.spec[0] = s.spec; p.spec[1] = s.spec + M; }
        if (t == t_hi - 1) launch_line_pass(MODE_FIRST_RQM4, in, p, 1, st);
        p.nfield = 2;
        if (mid) launch_line_pass(MODE_FWD, *mid, p, 1, st);
        launch_line_pass(MODE_OUTER, out, p, 1, st);
        if (mid) launch_line_pass(MODE_INV, *mid, p, 1, st);
        launch_line_pass(MODE_MID_RQM4, in, p, 1, st);
        StepPtrs p3 = p;
        p3.nfield = 1;
        p3.z[0] = z_[2].c();
        p3.L[0] = L2_.p;
        p3.spec[0] = s.spec ? s.spec + 2 * M : nullptr;
        p3.spec[1] = nullptr;
        if (mid) launch_line_pass(MODE_FWD, *mid, p3, 1, st);
        launch_line_pass(MODE_OUTER, out, p3, 1, st);
        if (mid) launch_line_pass(MODE_INV, *mid, p3, 1, st);
        launch_line_pass(MODE_END_ADJ, in, p, 1, st);
        if (s.spec) {
            StressArgs a{};
            a.s0 = s.spec; a.s1 = s.spec + M; a.s2 = s.spec + 2 * M;
            a.L1 = L1_.p; a.L2 = L2_.p;
            a.Lx = Lx_; a.Ly = Ly_; a.Lz = Lz_;
            a.cx = s.ds[X] * s.cl[0]; a.cy = s.ds[X] * s.cl[1]; a.cz = s.ds[X] * s.cl[2];
            a.partial = s.stress_partial + (long)t * kAG * 3;
            stress_step_kernel<<<kAG, kAT, 0, st>>>(a);
            PS_CUDA(cudaGetLastError());
        }
        cur ^= 1;
    }
    s.lam_cur = cur;   // lambda[t_lo] is in s.lam[cur]
}

void PairChain::prepare_adjoint() {
    if (plan_.naxes < 2) return;
    prepare_line_pass(MODE_END_ADJ, plan_.ax[0]);
}

// ---------------------------------------------------------------------------
// ModelAB: forward map, w-gradient, stress
// ---------------------------------------------------------------------------
void ModelAB::forward_only() {
    if (!fields_set_) throw Error(-6, "fields are not set");
    ensure_graphs();
    PS_CUDA(cudaGraphLaunch(gprop_, st_));
    double* dQ = scal_.p + 0;
    launch_mean(hf_.p + (long)Ns_ * M_, M_, partial_.p, dQ, st_);
    launch_density(hf_.p, hc_.p + (long)LB_ * M_, LA_, M_, cA_.p, dsA_, dQ, 0.0, phiA_.p, 1, 0, 0, nullptr, st_);
    launch_density(hf_.p + (long)LA_ * M_, hc_.p, LB_, M_, cB_.p, dsB_, dQ, 0.0, phiB_.p, 1, 0, 0, nullptr, st_);
    forward_done_ = true;
}

void ModelAB::adjoint_weights(std::vector<double>& wAf, std::vector<double>& wBf) const {
    // weight of pbar A / B at forward-chain index t (slice t of hf pairs with slice Ns - t of hc)
    std::vector<double> cA, cB;
    contour_weights(ruleA_, LA_, cA);
    contour_weights(ruleB_, LB_, cB);
    wAf.assign(Ns_ + 1, 0.0);
    wBf.assign(Ns_ + 1, 0.0);
    for (int t = 0; t <= LA_; t++) wAf[t] = dsA_ * cA[t];
    for (int t = LA_; t <= Ns_; t++) wBf[t] = dsB_ * cB[t - LA_];
}

void ModelAB::ensure_adjoint_buffers(bool spec) {
    if (lam_.n == 0) {
        lam_.alloc(2 * (size_t)M_);
        gA_.alloc(M_); gB_.alloc(M_);
        pbA_.alloc(M_); pbB_.alloc(M_);
        chain_->prepare_adjoint();
    }
    if (spec && spec_.n == 0) {
        spec_.alloc(6 * (size_t)M_);
        stress_part_.alloc((size_t)Ns_ * 148 * 3);
    }
}

void ModelAB::grad_w(const double* phiA_bar, const double* phiB_bar, double Q_bar, double* gA, double* gB) {
    if (!fields_set_) throw Error(-6, "fields are not set");
    if (p_.mde != 0) throw Error(-2, "the adjoint is provided for RQM4");
    ensure_adjoint_buffers(false);
    forward_only();
    // pbar = phi_bar / Q; Qbar_total = Q_bar - (1/Q) sum(phi_bar phi)
    PS_CUDA(cudaMemcpyAsync(pbA_.p, phiA_bar, sizeof(double) * M_, cudaMemcpyHostToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(pbB_.p, phiB_bar, sizeof(double) * M_, cudaMemcpyHostToDevice, st_));
    std::vector<double> pa(M_), pb(M_);
    PS_CUDA(cudaMemcpyAsync(pa.data(), phiA_.p, sizeof(double) * M_, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaMemcpyAsync(pb.data(), phiB_.p, sizeof(double) * M_, cudaMemcpyDeviceToHost, st_));
    double Q = 0;
    PS_CUDA(cudaMemcpyAsync(&Q, scal_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    double dot = 0.0;
    for (long i = 0; i < M_; i++) dot += phiA_bar[i] * pa[i] + phiB_bar[i] * pb[i];
    const double Qbar = Q_bar - dot / Q;
    scale2_kernel<<<egrid(M_), kAT, 0, st_>>>(pbA_.p, pbB_.p, 1.0 / Q, pbA_.p, pbB_.p, M_);
    PS_CUDA(cudaGetLastError());
    PS_CUDA(cudaMemsetAsync(gA_.p, 0, sizeof(double) * M_, st_));
    PS_CUDA(cudaMemsetAsync(gB_.p, 0, sizeof(double) * M_, st_));

    std::vector<double> wAf, wBf;
    adjoint_weights(wAf, wBf);
    // forward chain f: step t in block A for t < LA; direct weights at index t
    AdjointSweep s{};
    s.Ns = Ns_;
    s.hq = hf_.p; s.ho = hc_.p;
    s.lam[0] = lam_.p; s.lam[1] = lam_.p + M_;
    s.eF[0] = eFA_.p; s.eF[1] = eFB_.p; s.eH[0] = eHA_.p; s.eH[1] = eHB_.p;
    s.grad[0] = gA_.p; s.grad[1] = gB_.p;
    s.ds[0] = dsA_; s.ds[1] = dsB_;
    s.pbarA = pbA_.p; s.pbarB = pbB_.p;
    std::vector<int> blk(Ns_);
    for (int t = 0; t < Ns_; t++) blk[t] = t < LA_ ? 0 : 1;
    s.blk = blk.data();
    s.wd[0] = wAf.data(); s.wd[1] = wBf.data();
    s.cst_Ns = Qbar / (double)M_;
    chain_->enqueue_adjoint(s, st_);
    // complementary chain c: step t in block B for t < LB; slice t pairs with
    // forward index Ns - t
    std::vector<double> wAc(Ns_ + 1), wBc(Ns_ + 1);
    for (int i = 0; i <= Ns_; i++) { wAc[i] = wAf[Ns_ - i]; wBc[i] = wBf[Ns_ - i]; }
    std::vector<int> blkc(Ns_);
    for (int t = 0; t < Ns_; t++) blkc[t] = t < LB_ ? 1 : 0;
    AdjointSweep c = s;
    c.hq = hc_.p; c.ho = hf_.p;
    c.blk = blkc.data();
    c.wd[0] = wAc.data(); c.wd[1] = wBc.data();
    c.cst_Ns = 0.0;
    chain_->enqueue_adjoint(c, st_);
    PS_CUDA(cudaMemcpyAsync(gA, gA_.p, sizeof(double) * M_, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaMemcpyAsync(gB, gB_.p, sizeof(double) * M_, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

void ModelAB::stress(double* dFdl) {
    if (!fields_set_) throw Error(-6, "fields are not set");
    if (p_.mde != 0) throw Error(-2, "the adjoint is provided for RQM4");
    ensure_adjoint_buffers(true);
    forward_only();
    PS_CUDA(cudaMemsetAsync(gA_.p, 0, sizeof(double) * M_, st_));
    PS_CUDA(cudaMemsetAsync(gB_.p, 0, sizeof(double) * M_, st_));
    std::vector<double> zero(Ns_ + 1, 0.0);
    AdjointSweep s{};
    s.Ns = Ns_;
    s.hq = hf_.p; s.ho = hc_.p;
    s.lam[0] = lam_.p; s.lam[1] = lam_.p + M_;
    s.eF[0] = eFA_.p; s.eF[1] = eFB_.p; s.eH[0] = eHA_.p; s.eH[1] = eHB_.p;
    s.grad[0] = gA_.p; s.grad[1] = gB_.p;
    s.ds[0] = dsA_; s.ds[1] = dsB_;
    std::vector<int> blk(Ns_);
    for (int t = 0; t < Ns_; t++) blk[t] = t < LA_ ? 0 : 1;
    s.blk = blk.data();
    s.wd[0] = zero.data(); s.wd[1] = zero.data();
    s.cst_Ns = 1.0 / (double)M_;          // d Q / d f[Ns]
    s.spec = reinterpret_cast<double2*>(spec_.p);
    s.stress_partial = stress_part_.p;
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < 3; i++) {
        double l = p_.cell.l[i];
        s.cl[i] = (i < p_.dim && l > 0) ? 8.0 * PI * PI / (l * l * l) : 0.0;
    }
    chain_->enqueue_adjoint(s, st_);
    // dQ/dl = (1/M) sum over steps and k; dF/dl = -(1/Q) dQ/dl
    stress_final_kernel<<<1, 32, 0, st_>>>(stress_part_.p, (long)Ns_ * kAG, 1.0 / (double)M_, scal_.p + 16);
    PS_CUDA(cudaGetLastError());
    double Q = 0.0, dQ[3];
    PS_CUDA(cudaMemcpyAsync(&Q, scal_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaMemcpyAsync(dQ, scal_.p + 16, sizeof(double) * 3, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    for (int i = 0; i < 3; i++) dFdl[i] = -dQ[i] / Q;
}

void ModelAB::stress_checkpointed(int k, double* dFdl) {
    if (!fields_set_) throw Error(-6, "fields are not set");
    if (p_.mde != 0) throw Error(-2, "the adjoint is provided for RQM4");
    if (k <= 0) k = (int)std::ceil(std::sqrt((double)Ns_));
    if (k > Ns_) k = Ns_;
    const int nseg = (Ns_ + k - 1) / k;
    ensure_adjoint_buffers(true);
    ck_.alloc((size_t)nseg * M_);
    seg_.alloc((size_t)(k + 1) * M_);
    if (zero_.n == 0) {
        zero_.alloc(M_);
        scratch_.alloc(M_);
        launch_fill(zero_.p, M_, 0.0, st_);
    }
    // forward chain f only (lane c of the packed field carries zeros),
    // keeping slice j k of every segment j
    launch_fill(ck_.p, M_, 1.0, st_);
    auto segment = [&](int j) {
        const int t0 = j * k, n = std::min(k, Ns_ - t0);
        PS_CUDA(cudaMemcpyAsync(seg_.p, ck_.p + (long)j * M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
        LaneFactors lf{{eFA_.p, eFB_.p}, {eHA_.p, eHB_.p}, LA_ - t0};
        LaneFactors lc{{zero_.p, zero_.p}, {zero_.p, zero_.p}, 0};
        chain_->enqueue(seg_.p, nullptr, 0, n, lf, lc, 0, st_, zero_.p, scratch_.p);
        return n;
    };
    for (int j = 0; j < nseg; j++) {
        const int n = segment(j);
        if (j + 1 < nseg)
            PS_CUDA(cudaMemcpyAsync(ck_.p + (long)(j + 1) * M_, seg_.p + (long)n * M_, sizeof(double) * M_,
                                    cudaMemcpyDeviceToDevice, st_));
    }
    // Q = mean f[Ns]: the last slice of the last segment
    const int nlast = Ns_ - (nseg - 1) * k;
    double* dQ = scal_.p + 20;
    launch_mean(seg_.p + (long)nlast * M_, M_, partial_.p, dQ, st_);
    // reverse sweep, one recomputed segment at a time (the last one is still in seg_)
    std::vector<double> zero(Ns_ + 1, 0.0);
    std::vector<int> blk(Ns_);
    for (int t = 0; t < Ns_; t++) blk[t] = t < LA_ ? 0 : 1;
    AdjointSweep s{};
    s.Ns = Ns_;
    s.lam[0] = lam_.p; s.lam[1] = lam_.p + M_;
    s.eF[0] = eFA_.p; s.eF[1] = eFB_.p; s.eH[0] = eHA_.p; s.eH[1] = eHB_.p;
    s.grad[0] = gA_.p; s.grad[1] = gB_.p;
    s.ds[0] = dsA_; s.ds[1] = dsB_;
    s.blk = blk.data();
    s.wd[0] = zero.data(); s.wd[1] = zero.data();
    s.cst_Ns = 1.0 / (double)M_;
    s.spec = reinterpret_cast<double2*>(spec_.p);
    s.stress_partial = stress_part_.p;
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < 3; i++) {
        double l = p_.cell.l[i];
        s.cl[i] = (i < p_.dim && l > 0) ? 8.0 * PI * PI / (l * l * l) : 0.0;
    }
    s.hq = seg_.p;
    for (int j = nseg - 1; j >= 0; j--) {
        const int n = (j == nseg - 1) ? nlast : segment(j);
        s.t_lo = j * k;
        s.t_hi = j * k + n;
        s.hq_base = j * k;
        chain_->enqueue_adjoint(s, st_);
    }
    stress_final_kernel<<<1, 32, 0, st_>>>(stress_part_.p, (long)Ns_ * kAG, 1.0 / (double)M_, scal_.p + 16);
    PS_CUDA(cudaGetLastError());
    double Q = 0.0, dQl[3];
    PS_CUDA(cudaMemcpyAsync(&Q, dQ, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaMemcpyAsync(dQl, scal_.p + 16, sizeof(double) * 3, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    for (int i = 0; i < 3; i++) dFdl[i] = -dQl[i] / Q;
}

}  // namespace ps
