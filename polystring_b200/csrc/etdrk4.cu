// etdrk4.cu -- the ETDRK4 propagator step (Etdrk4_PBC.cc:110-184) for two
// real chains packed into one complex field (lane f in the real part, lane c
// in the imaginary part).
//
// Cox-Matthews ETDRK4 with the Kassam-Trefethen coefficients: the spectrum v
// of the chain is carried from step to step, and each step is
//     Nv = F[-w q_s]
//     a  = E2 v + Q Nv              Na = F[-w Re(F^-1 a) / M]
//     b  = E2 v + Q Na              Nb = F[-w Re(F^-1 b) / M]
//     c  = E2 a + Q (2 Nb - Nv)     Nc = F[-w Re(F^-1 c) / M]
//     v  = E v + f1 Nv + 2 f2 (Na + Nb) + f3 Nc
//     q_{s+1} = Re(F^-1 v) / M
// with E = exp(ds L), E2 = exp(ds L / 2) and L = -k^2 (calc_k2_orthogonal).
// Every spectral operation multiplies by real tables that are even in k, so
// the packed field carries both lanes' spectra at once; the nonlinear term
// takes each lane's own w.  The transforms are the line passes of
// line_pass.cu (MODE_FWD / MODE_INV over every axis); the elementwise work
// of the step is in the kernels below.
#include "engine.h"
#include "ps_internal.h"

#include <cmath>
#include <complex>

namespace ps {

namespace {

constexpr int kEtdThreads = 256;

inline unsigned etd_blocks(long n) {
    long b = (n + kEtdThreads - 1) / kEtdThreads;
    return (unsigned)(b < 148 * 16 ? b : 148 * 16);
}

// T = qf + i qc (a chain's spectrum from its real slices: init) or
// T = -(wf qf) - i (wc qc) (the nonlinear term of the slices: Nv)
__global__ void etd_slices_kernel(double2* __restrict__ T, const double* __restrict__ qf,
                                  const double* __restrict__ qc, const double* __restrict__ wf,
                                  const double* __restrict__ wc, long M, int nonlin) {
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < M; m += (long)gridDim.x * blockDim.x) {
        const double xf = qf[m], xc = qc[m];
        T[m] = nonlin ? make_double2(-wf[m] * xf, -wc[m] * xc) : make_double2(xf, xc);
    }
}

// T = -(wf Re(T) / M) - i (wc Im(T) / M): the nonlinear term of an inverse
// transform (Etdrk4_PBC.cc, x = Re(b) / M)
__global__ void etd_nonlin_kernel(double2* __restrict__ T, const double* __restrict__ wf,
                                  const double* __restrict__ wc, long M, double rM) {
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < M; m += (long)gridDim.x * blockDim.x) {
        const double2 t = T[m];
        const double xf = t.x / rM, xc = t.y / rM;
        T[m] = make_double2(-wf[m] * xf, -wc[m] * xc);
    }
}

struct EtdFields {
    double2 *T, *V, *Nv, *A, *Na, *Nb;
    const double *E, *E2, *Q, *f1, *f2, *f3;
};

__device__ __forceinline__ double2 lin2(double a, double2 x, double b, double2 y) {
    return make_double2(a * x.x + b * y.x, a * x.y + b * y.y);
}

// the spectral stages of one step; T holds the forward transform of the
// stage's nonlinear term on entry and the next spectrum to invert on exit
//   0: Nv = T; a = E2 v + Q Nv; T = a
//   1: Na = T; T = E2 v + Q Na
//   2: Nb = T; T = E2 a + Q (2 Nb - Nv)
//   3: v = E v + f1 Nv + 2 f2 (Na + Nb) + f3 T; T = v
__global__ void etd_combine_kernel(EtdFields f, long M, int stage) {
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < M; m += (long)gridDim.x * blockDim.x) {
        const double2 t = f.T[m];
        if (stage == 0) {
            f.Nv[m] = t;
            const double2 a = lin2(f.E2[m], f.V[m], f.Q[m], t);
            f.A[m] = a;
            f.T[m] = a;
        } else if (stage == 1) {
            f.Na[m] = t;
            f.T[m] = lin2(f.E2[m], f.V[m], f.Q[m], t);
        } else if (stage == 2) {
            f.Nb[m] = t;
            const double2 nv = f.Nv[m];
            const double2 d = make_double2(2.0 * t.x - nv.x, 2.0 * t.y - nv.y);
            f.T[m] = lin2(f.E2[m], f.A[m], f.Q[m], d);
        } else {
            const double2 v = f.V[m], nv = f.Nv[m], na = f.Na[m], nb = f.Nb[m];
            const double e = f.E[m], g1 = f.f1[m], c2 = 2.0 * f.f2[m], g3 = f.f3[m];
            const double2 r = make_double2(e * v.x + g1 * nv.x + c2 * (na.x + nb.x) + g3 * t.x,
                                           e * v.y + g1 * nv.y + c2 * (na.y + nb.y) + g3 * t.y);
            f.V[m] = r;
            f.T[m] = r;
        }
    }
}

// q_f = Re(T) / M, q_c = Im(T) / M (q_c may be null)
__global__ void etd_store_kernel(const double2* __restrict__ T, double* __restrict__ qf, double* __restrict__ qc,
                                 long M, double rM) {
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < M; m += (long)gridDim.x * blockDim.x) {
        const double2 t = T[m];
        qf[m] = t.x / rM;
        if (qc) qc[m] = t.y / rM;
    }
}

}  // namespace

// Etdrk4_PBC's tables (Etdrk4_PBC.cc:14-24, :43-99): E = exp(ds L),
// E2 = exp(ds L / 2) and Q, f1, f2, f3 as ds times the mean over Mc points
// r = exp(i pi (j + 1/2) / Mc) of the upper half circle of the real parts of
//   Q  = (e^{x/2} - 1) / x,            f1 = (e^x (x^2 - 3x + 4) - x - 4) / x^3,
//   f2 = (e^x (x - 2) + x + 2) / x^3,  f3 = (e^x (4 - x) - x^2 - 3x - 4) / x^3
// at x = ds L + r (the contour integral that avoids the cancellation of the
// closed forms near L = 0).  L is the k2_orthogonal table (-|k|^2).
void PairChain::set_tables_etd(const std::vector<double>& k2, double ds, int Mc) {
    if (scheme_ != SCHEME_ETDRK4) throw Error(-2, "set_tables_etd on a chain that is not ETDRK4");
    if (Mc < 1) throw Error(-1, "ETDRK4 needs at least one contour point");
    const long M = M_;
    std::vector<double> tab(6 * (size_t)M);
    const double PI = 3.14159265358979323846;
    std::vector<std::complex<double>> r(Mc);
    for (int j = 0; j < Mc; j++) r[j] = std::exp(std::complex<double>(0.0, PI * (j + 0.5) / Mc));
    for (long m = 0; m < M; m++) {
        const double L = k2[m];
        tab[0 * M + m] = exp(ds * L);
        tab[1 * M + m] = exp(ds * L / 2.0);
        double sq = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int j = 0; j < Mc; j++) {
            const std::complex<double> x = ds * L + r[j];
            const std::complex<double> ex = std::exp(x), x2 = x * x, x3 = x2 * x;
            sq += ((std::exp(x / 2.0) - 1.0) / x).real();
            s1 += ((ex * (x2 - 3.0 * x + 4.0) - x - 4.0) / x3).real();
            s2 += ((ex * (x - 2.0) + x + 2.0) / x3).real();
            s3 += ((ex * (4.0 - x) - x2 - 3.0 * x - 4.0) / x3).real();
        }
        tab[2 * M + m] = ds * (sq / Mc);
        tab[3 * M + m] = ds * (s1 / Mc);
        tab[4 * M + m] = ds * (s2 / Mc);
        tab[5 * M + m] = ds * (s3 / Mc);
    }
    etdtab_.alloc(tab.size());
    PS_CUDA(cudaMemcpy(etdtab_.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
}

// forward (MODE_FWD) or inverse (MODE_INV, unnormalised) transform of one
// packed field over every axis of the grid
void PairChain::transform(double2* z, int mode, cudaStream_t st) const {
    StepPtrs p{};
    p.z[0] = z;
    p.nfield = 1;
    p.M = (double)M_;
    for (int a = 0; a < plan_.naxes; a++) launch_line_pass(mode, plan_.ax[a], p, 1, st);
}

// ETDRK4 steps t = 0 .. nsteps-1 of the pair: lane f's w is lf.F(t), lane c's
// lc.F(t) (the factor slots carry the fields w themselves for this scheme).
// A lane that starts a new block at step t starts a new solve there: the
// carried spectrum is rebuilt from the real slices of both lanes at t = 0
// and at each lane's switch step (Etdrk4_PBC::solve starts from F[q_0]).
void PairChain::enqueue_etd(double* hf, double* hc, int nsteps, const LaneFactors& lf, const LaneFactors& lc,
                            cudaStream_t st, const double* c_in_fixed, double* c_out_fixed) {
    const long M = M_;
    const double rM = (double)M;
    const unsigned nb = etd_blocks(M);
    double2* T = z_[0].c();
    EtdFields f;
    f.T = T;
    f.V = etd_.c(); f.Nv = f.V + M; f.A = f.V + 2 * M; f.Na = f.V + 3 * M; f.Nb = f.V + 4 * M;
    f.E = etdtab_.p; f.E2 = f.E + M; f.Q = f.E + 2 * M; f.f1 = f.E + 3 * M; f.f2 = f.E + 4 * M; f.f3 = f.E + 5 * M;
    for (int t = 0; t < nsteps; t++) {
        const double* qf = hf + (long)t * M;
        const double* qc = c_in_fixed ? c_in_fixed : hc + (long)t * M;
        const double* wf = lf.F(t);
        const double* wc = lc.F(t);
        if (t == 0 || t == lf.switch_t || t == lc.switch_t) {
            etd_slices_kernel<<<nb, kEtdThreads, 0, st>>>(f.V, qf, qc, nullptr, nullptr, M, 0);
            PS_CUDA(cudaGetLastError());
            transform(f.V, MODE_FWD, st);
        }
        etd_slices_kernel<<<nb, kEtdThreads, 0, st>>>(T, qf, qc, wf, wc, M, 1);
        PS_CUDA(cudaGetLastError());
        for (int stage = 0; stage < 4; stage++) {
            if (stage > 0) {
                etd_nonlin_kernel<<<nb, kEtdThreads, 0, st>>>(T, wf, wc, M, rM);
                PS_CUDA(cudaGetLastError());
            }
            transform(T, MODE_FWD, st);
            etd_combine_kernel<<<nb, kEtdThreads, 0, st>>>(f, M, stage);
            PS_CUDA(cudaGetLastError());
            transform(T, MODE_INV, st);
        }
        double* of = hf + (long)(t + 1) * M;
        double* oc = c_in_fixed ? c_out_fixed : hc + (long)(t + 1) * M;
        etd_store_kernel<<<nb, kEtdThreads, 0, st>>>(T, of, oc, M, rM);
        PS_CUDA(cudaGetLastError());
    }
}

}  // namespace ps
