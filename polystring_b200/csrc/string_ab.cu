// string_ab.cu -- the string method of polystring_AB (scft/polystring_AB.cc)
// with all images advanced together on the device.
//
// One string iteration (polystring_AB.cc:125-150) is captured once as a CUDA
// graph and replayed:
//   * every image restarts from its string fields with a fresh Yita = 0
//     (resetInString, Model_AB.cc:52-83, DATA_INIT -> init_data_field) and
//     runs max_iter simple-mixing SCFT iterations (scft::relax); every
//     propagator pass of that loop is ONE launch for all images (batch in
//     gridDim.z), as are Q, densities and the field update;
//   * H of every image (Model_AB::H);
//   * arc length S from wa (parameterize_string, :283-296);
//   * per-grid-point natural cubic spline re-sampling of wa and wb at
//     uniform s (redistribute_stringBeads, :298-319), ends restored (:321-328).
#include "engine.h"
#include "field_kernels.h"
#include "string_ab.h"
#include "sweep.h"

#include <cmath>
#include <cstdlib>

namespace ps {

namespace {

constexpr int kBT = 256;

// per-image two-stage deterministic reductions: out[b * 8 + slot] (+= stride)
template <class F, int K>
__global__ void __launch_bounds__(kBT) breduce_partial(F f, long M, double* partial) {
    const int b = blockIdx.y;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        double v[K];
        f(b, i, v);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += v[k];
    }
    __shared__ double sh[K][kBT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < kBT / 32; w++) s += sh[threadIdx.x][w];
        partial[((long)b * gridDim.x + blockIdx.x) * K + threadIdx.x] = s;
    }
}

template <int K>
__global__ void __launch_bounds__(kBT) breduce_final(const double* partial, int G, double scale, double* out,
                                                      int slot) {
    const int b = blockIdx.x;
    __shared__ double sh[K][kBT / 32];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += partial[((long)b * G + g) * K + k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < kBT / 32; w++) s += sh[threadIdx.x][w];
        out[b * 8 + slot + threadIdx.x] = s * scale;
    }
}

constexpr int kBG = 64;   // blocks per image in batched reductions

struct TailMeanF {   // Q: mean of the last forward-chain slice of image b
    const double* hf;
    long hstride, tail_off;
    __device__ void operator()(int b, long i, double* v) const { v[0] = hf[b * hstride + tail_off + i]; }
};

struct HwBF {
    const double *phiA, *phiB, *wA, *wB;
    long M;
    double chiN, lamYita;
    int compressible;
    __device__ void operator()(int b, long i, double* v) const {
        long j = b * M + i;
        double a = phiA[j], c = phiB[j];
        double g = chiN * a * c;
        if (compressible) g += lamYita / 2.0 * (a + c - 1.0) * (a + c - 1.0);
        g -= wA[j] * a;
        g -= wB[j] * c;
        v[0] = g;
    }
};

struct ArcBF {   // image b >= 1: (wa[b] - wa[b-1])^2; image 0 contributes 0
    const double* wa;
    long M;
    __device__ void operator()(int b, long i, double* v) const {
        if (b == 0) { v[0] = 0.0; return; }
        double d = wa[b * M + i] - wa[(b - 1) * M + i];
        v[0] = d * d;
    }
};

// S[0] = 0, S[s] = S[s-1] + sqrt(arc2[s]); normalised by S[m-1]
__global__ void arclength_kernel(const double* scal, int m, double* S) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    S[0] = 0.0;
    for (int s = 1; s < m; s++) S[s] = S[s - 1] + sqrt(scal[s * 8 + 2]);
    double last = S[m - 1];
    for (int s = 0; s < m; s++) S[s] = 1.0 * S[s] / last;
}

// Natural cubic spline through (S[z], f[z][i]) evaluated at z/(m-1), per
// grid point i; b (half second derivatives) by forward elimination and back
// substitution of the tridiagonal system; abscissae equal to a knot x_j
// (j > 0) use the piece to their left.  Same steps as the oracle.
__global__ void spline_kernel(double* f, const double* S, int m, long M) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    double y[kMaxImages], bb[kMaxImages], cp[kMaxImages], rhs[kMaxImages];
    for (int z = 0; z < m; z++) y[z] = f[(long)z * M + i];
    bb[0] = 0.0; bb[m - 1] = 0.0; cp[0] = 0.0; rhs[0] = 0.0;
    for (int j = 1; j < m - 1; j++) {
        double hl = S[j] - S[j - 1], hr = S[j + 1] - S[j];
        double lo = hl / 3.0, di = 2.0 * (S[j + 1] - S[j - 1]) / 3.0, up = hr / 3.0;
        double r = (y[j + 1] - y[j]) / hr - (y[j] - y[j - 1]) / hl;
        double den = di - lo * cp[j - 1];
        cp[j] = up / den;
        rhs[j] = (r - lo * rhs[j - 1]) / den;
    }
    for (int j = m - 2; j >= 1; j--) bb[j] = rhs[j] - cp[j] * bb[j + 1];
    int idx = 0;
    for (int z = 0; z < m; z++) {
        double t = 1.0 * z / (m - 1);
        while (idx < m - 1 && S[idx + 1] < t) idx++;
        int k = idx > m - 2 ? m - 2 : idx;
        double h = t - S[k];
        double hi = S[k + 1] - S[k];
        double a = (bb[k + 1] - bb[k]) / (3.0 * hi);
        double c = (y[k + 1] - y[k]) / hi - (2.0 * bb[k] + bb[k + 1]) * hi / 3.0;
        f[(long)z * M + i] = ((a * h + bb[k]) * h + c) * h + y[k];
    }
}

int rgrid(long M) {
    long g = (M + kBT - 1) / kBT;
    return (int)(g < kBG ? g : kBG);
}

}  // namespace

StringAB::StringAB(const ModelABParams& p, int m, int max_iter, int lo, int hi)
    : p_(p), m_(m), max_iter_(max_iter) {
    if (m < 3 || m > kMaxImages) throw Error(-1, "number of images must be in 3.." + std::to_string(kMaxImages));
    if (hi < 0) hi = m;
    if (lo < 0 || hi > m || lo >= hi) throw Error(-1, "the shard must be a non-empty range of the images");
    lo_ = lo;
    nloc_ = hi - lo;
    if (max_iter < 1) throw Error(-1, "max_iter must be positive");
    if (p.scft != 0) throw Error(-2, "the string method runs simple mixing (DATA_INIT fields)");
    if (p.sA < 2 || p.sB < 2) throw Error(-1, "Ms must be at least [2, 2]");
    cell_init(p_.cell);
    M_ = (long)p.Lx * p.Ly * p.Lz;
    LA_ = p.sA - 1;
    LB_ = p.sB - 1;
    Ns_ = LA_ + LB_;
    double fA = 1.0 * LA_ / (LA_ + LB_), fB = 1.0 * LB_ / (LA_ + LB_);
    dsA_ = fA / LA_;
    dsB_ = fB / LB_;
    int ruleA = p.contour == 0 ? 0 : ((p.sA % 2 != 0) ? 1 : 2);
    int ruleB = p.contour == 0 ? 0 : ((p.sB % 2 != 0) ? 1 : 2);
    std::vector<double> cA, cB;
    if (!contour_weights(ruleA, LA_, cA) || !contour_weights(ruleB, LB_, cB))
        throw Error(-4, "contour quadrature precondition fails");
    if (p.mde != 0 && p.mde != 1) throw Error(-2, "string images use RQM4 or OS2");
    PS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    chain_ = new PairChain(p.Lx, p.Ly, p.Lz, p.mde == 1 ? SCHEME_OS2 : SCHEME_RQM4, nloc_);
    if (p.mde == 1) {
        chain_->set_tables(k_laplacian(p_.cell, p.Lx, p.Ly, p.Lz, dsA_), {});
    } else {
        std::vector<double> k2 = k2_orthogonal(p_.cell, p.Lx, p.Ly, p.Lz);
        std::vector<double> L1(M_), L2(M_);
        for (long i = 0; i < M_; i++) {
            L1[i] = exp(dsA_ * k2[i]);
            L2[i] = exp(0.5 * dsA_ * k2[i]);
        }
        chain_->set_tables(L1, L2);
        // every image's propagators in one cluster-resident sweep per SCFT
        // iteration where the 2D grid has one (PS_B200_LINE_PASSES=1 keeps
        // the batched line passes)
        const char* force = getenv("PS_B200_LINE_PASSES");
        if (cluster_sweep_supported(p.Lx, p.Ly, p.Lz) && !(force && force[0] == '1')) {
            use_cluster_ = true;
            cluster_sweep_prepare(p.Lx, p.Ly, p.Lz, nloc_);
            // per-axis factors exp(h k_x^2), exp(h k_y^2) for h = ds, ds/2: the
            // orthogonal k2 along each axis (the other indices 0)
            std::vector<double> kt;
            for (double h : {dsA_, 0.5 * dsA_}) {
                for (int x = 0; x < p.Lx; x++) kt.push_back(exp(h * k2[(long)x * p.Ly * p.Lz]));
                for (int y = 0; y < p.Ly; y++) kt.push_back(exp(h * k2[(long)y * p.Lz]));
            }
            clK_.alloc(kt.size());
            PS_CUDA(cudaMemcpy(clK_.p, kt.data(), sizeof(double) * kt.size(), cudaMemcpyHostToDevice));
        }
    }
    if (!use_cluster_) chain_->autotune(st_);
    const size_t mM = (size_t)m * M_, nM = (size_t)nloc_ * M_;
    hf_.alloc((size_t)(Ns_ + 1) * nM);
    hc_.alloc((size_t)(Ns_ + 1) * nM);
    wa_.alloc(mM); wb_.alloc(mM); phiA_.alloc(mM); phiB_.alloc(mM);
    yita_.alloc(nM); eFA_.alloc(nM); eHA_.alloc(nM); eFB_.alloc(nM); eHB_.alloc(nM);
    ends_.alloc(4 * (size_t)M_);
    cA_.alloc(cA.size()); cB_.alloc(cB.size());
    PS_CUDA(cudaMemcpy(cA_.p, cA.data(), sizeof(double) * cA.size(), cudaMemcpyHostToDevice));
    PS_CUDA(cudaMemcpy(cB_.p, cB.data(), sizeof(double) * cB.size(), cudaMemcpyHostToDevice));
    scal_.alloc((size_t)8 * m);
    S_.alloc(m);
    partial_.alloc((size_t)kBG * m * 8);
    // heads of both chains of every image of the shard
    for (int b = 0; b < nloc_; b++) {
        launch_fill(hf_.p + (size_t)b * (Ns_ + 1) * M_, M_, 1.0, st_);
        launch_fill(hc_.p + (size_t)b * (Ns_ + 1) * M_, M_, 1.0, st_);
    }
    PS_CUDA(cudaMemsetAsync(scal_.p, 0, sizeof(double) * 8 * m, st_));
    PS_CUDA(cudaMemsetAsync(phiA_.p, 0, sizeof(double) * mM, st_));
    PS_CUDA(cudaMemsetAsync(phiB_.p, 0, sizeof(double) * mM, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

StringAB::~StringAB() {
    if (giter_) cudaGraphExecDestroy(giter_);
    if (grelax_) cudaGraphExecDestroy(grelax_);
    if (grepar_) cudaGraphExecDestroy(grepar_);
    delete chain_;
    if (st_) cudaStreamDestroy(st_);
}

void StringAB::set_images(const double* wa, const double* wb, bool dev) {
    auto kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const size_t mM = (size_t)m_ * M_;
    PS_CUDA(cudaMemcpyAsync(wa_.p, wa, sizeof(double) * mM, kind, st_));
    PS_CUDA(cudaMemcpyAsync(wb_.p, wb, sizeof(double) * mM, kind, st_));
    // ends kept aside (polystring_AB.cc:214-221)
    PS_CUDA(cudaMemcpyAsync(ends_.p, wa_.p, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(ends_.p + M_, wa_.p + (size_t)(m_ - 1) * M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(ends_.p + 2 * M_, wb_.p, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(ends_.p + 3 * M_, wb_.p + (size_t)(m_ - 1) * M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    iters_ = 0;
    relaxed_ = false;
    ready_ = true;
}

// one SCFT iteration (Model_AB::update, EM branch) of the shard's images
void StringAB::enqueue_scft_iteration() {
    const long hstride = (long)(Ns_ + 1) * M_;
    const long off = (long)lo_ * M_;
    double *wa = wa_.p + off, *wb = wb_.p + off, *phiA = phiA_.p + off, *phiB = phiB_.p + off;
    double* scal = scal_.p + 8 * lo_;
    if (use_cluster_) {
        SweepArgs a{};
        a.hf = hf_.p; a.hc = hc_.p;
        a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p;
        a.ktab = clK_.p;
        a.LA = LA_; a.LB = LB_; a.Ns = Ns_;
        a.bstride_batch = M_; a.bstride_hist = hstride; a.bstride_L = 0;
        cluster_sweep_launch(a, p_.Lx, p_.Ly, p_.Lz, nloc_, st_);
    } else {
        LaneFactors lf{{eFA_.p, eFB_.p}, {eHA_.p, eHB_.p}, LA_};
        LaneFactors lc{{eFB_.p, eFA_.p}, {eHB_.p, eHA_.p}, LB_};
        chain_->enqueue(hf_.p, hc_.p, hstride, Ns_, lf, lc, M_, st_);
    }
    // Q of every image
    dim3 g(rgrid(M_), nloc_);
    breduce_partial<TailMeanF, 1><<<g, kBT, 0, st_>>>(TailMeanF{hf_.p, hstride, (long)Ns_ * M_}, M_, partial_.p);
    PS_CUDA(cudaGetLastError());
    breduce_final<1><<<nloc_, kBT, 0, st_>>>(partial_.p, rgrid(M_), 1.0 / (double)M_, scal, 0);
    PS_CUDA(cudaGetLastError());
    launch_density(hf_.p, hc_.p + (long)LB_ * M_, LA_, M_, cA_.p, dsA_, nullptr, 0.0, phiA, nloc_, hstride, M_,
                   scal, st_);
    launch_density(hf_.p + (long)LA_ * M_, hc_.p, LB_, M_, cB_.p, dsB_, nullptr, 0.0, phiB, nloc_, hstride, M_,
                   scal, st_);
    EMArgs a{};
    a.phiA = phiA; a.phiB = phiB; a.wA = wa; a.wB = wb; a.yita = yita_.p;
    a.M = M_; a.chiN = p_.chiN; a.lamA = p_.lamA; a.lamB = p_.lamB; a.lamYita = p_.lamYita;
    a.dsA = dsA_; a.dsB = dsB_; a.compressible = p_.compressible;
    a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p; a.bstride = M_;
    launch_em_update(a, nloc_, st_);
}

// run_scftInString (polystring_AB.cc:256-281) for the shard's images: fresh
// Yita and Boltzmann factors of the string fields (resetInString), max_iter
// SCFT iterations, H = Hw - ln Q per image (Hw into slot 1)
void StringAB::enqueue_relax() {
    const long off = (long)lo_ * M_;
    launch_fill(yita_.p, (long)nloc_ * M_, 0.0, st_);
    launch_factors(wa_.p + off, wb_.p + off, M_, dsA_, dsB_, eFA_.p, eHA_.p, eFB_.p, eHB_.p, nloc_, M_, st_);
    for (int it = 0; it < max_iter_; it++) enqueue_scft_iteration();
    dim3 g(rgrid(M_), nloc_);
    breduce_partial<HwBF, 1><<<g, kBT, 0, st_>>>(
        HwBF{phiA_.p + off, phiB_.p + off, wa_.p + off, wb_.p + off, M_, p_.chiN, p_.lamYita, p_.compressible}, M_,
        partial_.p);
    PS_CUDA(cudaGetLastError());
    breduce_final<1><<<nloc_, kBT, 0, st_>>>(partial_.p, rgrid(M_), 1.0 / (double)M_, scal_.p + 8 * lo_, 1);
    PS_CUDA(cudaGetLastError());
}

// parameterize_string and redistribute_stringBeads (polystring_AB.cc:283-329)
// over all m images
void StringAB::enqueue_reparameterize() {
    // arc length from wa (slot 2 of image s: mean (wa[s] - wa[s-1])^2)
    dim3 g(rgrid(M_), m_);
    breduce_partial<ArcBF, 1><<<g, kBT, 0, st_>>>(ArcBF{wa_.p, M_}, M_, partial_.p);
    PS_CUDA(cudaGetLastError());
    breduce_final<1><<<m_, kBT, 0, st_>>>(partial_.p, rgrid(M_), 1.0 / (double)M_, scal_.p, 2);
    PS_CUDA(cudaGetLastError());
    arclength_kernel<<<1, 32, 0, st_>>>(scal_.p, m_, S_.p);
    PS_CUDA(cudaGetLastError());
    // re-sample wa and wb, restore the ends
    const int sb = (int)((M_ + 127) / 128);
    spline_kernel<<<sb, 128, 0, st_>>>(wa_.p, S_.p, m_, M_);
    PS_CUDA(cudaGetLastError());
    spline_kernel<<<sb, 128, 0, st_>>>(wb_.p, S_.p, m_, M_);
    PS_CUDA(cudaGetLastError());
    PS_CUDA(cudaMemcpyAsync(wa_.p, ends_.p, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(wa_.p + (size_t)(m_ - 1) * M_, ends_.p + M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(wb_.p, ends_.p + 2 * M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(wb_.p + (size_t)(m_ - 1) * M_, ends_.p + 3 * M_, sizeof(double) * M_, cudaMemcpyDeviceToDevice, st_));
}

void StringAB::enqueue_string_iteration() {
    enqueue_relax();
    enqueue_reparameterize();
}

cudaGraphExec_t StringAB::capture(void (StringAB::*enq)()) {
    PS_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
        (this->*enq)();
    } catch (...) {
        cudaStreamEndCapture(st_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    PS_CUDA(cudaStreamEndCapture(st_, &g));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw Error(-3, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return ex;
}

void StringAB::iterate(int n) {
    if (!ready_) throw Error(-6, "string images are not set");
    if (nloc_ != m_) throw Error(-6, "a context that relaxes a shard of the images runs relax and reparameterize");
    if (!giter_) giter_ = capture(&StringAB::enqueue_string_iteration);
    for (int i = 0; i < n; i++) PS_CUDA(cudaGraphLaunch(giter_, st_));
    iters_ += n;
}

void StringAB::relax() {
    if (!ready_) throw Error(-6, "string images are not set");
    if (!grelax_) grelax_ = capture(&StringAB::enqueue_relax);
    PS_CUDA(cudaGraphLaunch(grelax_, st_));
    relaxed_ = true;
}

void StringAB::reparameterize() {
    if (!ready_) throw Error(-6, "string images are not set");
    if (!grepar_) grepar_ = capture(&StringAB::enqueue_reparameterize);
    PS_CUDA(cudaGraphLaunch(grepar_, st_));
    iters_ += 1;
}

double* StringAB::device_ptr(int which) {
    switch (which) {
    case 0: return wa_.p;
    case 1: return wb_.p;
    case 2: return phiA_.p;
    case 3: return phiB_.p;
    }
    throw Error(-1, "unknown string array");
}

void StringAB::sync() { PS_CUDA(cudaStreamSynchronize(st_)); }

void StringAB::H(double* out) {
    if (iters_ == 0 && !relaxed_) throw Error(-6, "no string iteration has run");
    std::vector<double> sc((size_t)8 * m_);
    PS_CUDA(cudaMemcpyAsync(sc.data(), scal_.p, sizeof(double) * 8 * m_, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    for (int b = 0; b < m_; b++)   // images outside the shard have no H here
        out[b] = (b >= lo_ && b < lo_ + nloc_) ? sc[b * 8 + 1] + (-log(sc[b * 8 + 0])) : nan("");
}

void StringAB::S(double* out) {
    PS_CUDA(cudaMemcpyAsync(out, S_.p, sizeof(double) * m_, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

void StringAB::get(int which, double* out, bool dev) {
    double* src = nullptr;
    switch (which) {
    case 0: src = wa_.p; break;
    case 1: src = wb_.p; break;
    case 2: src = phiA_.p; break;
    case 3: src = phiB_.p; break;
    default: throw Error(-1, "unknown string array");
    }
    PS_CUDA(cudaMemcpyAsync(out, src, sizeof(double) * m_ * M_, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

int StringAB::launches_per_iteration() const {
    const int prop = use_cluster_ ? 1 : chain_->launches_per_step() * Ns_ + (chain_->plan().naxes > 1 ? 1 : 0);
    const int scft = prop + 2 + 2 + 1;
    return 2 + max_iter_ * scft + 2 + 2 + 1 + 2;
}

}  // namespace ps
