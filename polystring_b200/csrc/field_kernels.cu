// field_kernels.cu -- bandwidth-bound kernels around the propagator:
// contour integral of q q^dagger into densities, deterministic grid
// reductions (Q, H, residuals, Anderson inner products), the simple-mixing
// field update fused with the Boltzmann factors of the next iteration, and
// the Anderson combination.
//
// Reductions are two-stage with a fixed grid (kRedBlocks x kRedThreads) and a
// fixed tree order, so a result is bit-identical from run to run.
#include "ps_internal.h"
#include "field_kernels.h"

namespace ps {

namespace {

// ---------------------------------------------------------------------------
// deterministic block reduction of K values per thread
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void block_reduce_store(double (&acc)[K], double* out) {
    __shared__ double sh[K][kRedThreads / 32];
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
        for (int w = 0; w < kRedThreads / 32; w++) s += sh[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

template <class F, int K>
__global__ void __launch_bounds__(kRedThreads) reduce_partial_kernel(F f, long M, double* partial) {
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        double v[K];
        f(i, v);
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += v[k];
    }
    block_reduce_store<K>(acc, partial + (long)blockIdx.x * K);
}

// out[k] = scale * sum_b partial[b][k]; one block, fixed order
template <int K>
__global__ void __launch_bounds__(kRedThreads) reduce_final_kernel(const double* partial, int G, double scale, double* out) {
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += partial[(long)b * K + k];
    }
    __shared__ double res[K];
    block_reduce_store<K>(acc, res);
    __syncthreads();
    if (threadIdx.x < K) out[threadIdx.x] = res[threadIdx.x] * scale;
}

template <class F, int K>
void reduce_launch(F f, long M, double* partial, double* out, double scale, cudaStream_t st) {
    reduce_partial_kernel<F, K><<<kRedBlocks, kRedThreads, 0, st>>>(f, M, partial);
    PS_CUDA(cudaGetLastError());
    reduce_final_kernel<K><<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, scale, out);
    PS_CUDA(cudaGetLastError());
}

struct MeanF {
    const double* x;
    __device__ void operator()(long i, double* v) const { v[0] = x[i]; }
};

// Model_AB::Hw integrand (Model_AB.cc:263-289)
struct HwF {
    const double *phiA, *phiB, *wA, *wB;
    double chiN, lamYita;
    int compressible;
    __device__ void operator()(long i, double* v) const {
        double a = phiA[i], b = phiB[i];
        double g = chiN * a * b;
        if (compressible) g += lamYita / 2.0 * (a + b - 1.0) * (a + b - 1.0);
        g -= wA[i] * a;
        g -= wB[i] * b;
        v[0] = g;
    }
};

// Model_AB::residual_error, EM branch (Model_AB.cc:317-369):
// sums of |g2A|, |wA|, |g1A|, |g2B|, |wB|, |g1B|, |phiA+phiB-1|, |phiA+phiB|
struct ResidualEMF {
    const double *phiA, *phiB, *wA, *wB, *yita;
    double chiN, lamYita;
    int compressible;
    __device__ void operator()(long i, double* v) const {
        double a = phiA[i], b = phiB[i];
        double ya = compressible ? lamYita * (a + b - 1.0) : yita[i];
        double g1A = chiN * b + ya;
        double g1B = chiN * a + ya;
        v[0] = fabs(g1A - wA[i]); v[1] = fabs(wA[i]); v[2] = fabs(g1A);
        v[3] = fabs(g1B - wB[i]); v[4] = fabs(wB[i]); v[5] = fabs(g1B);
        double s = a + b;
        v[6] = fabs(s - 1.0); v[7] = fabs(s);
    }
};

// Anderson residual sums (Model_AB.cc:309-316 with FieldAX.cc:106-150)
struct ResidualAXF {
    const double *dA, *dB, *wA, *wB;
    __device__ void operator()(long i, double* v) const {
        v[0] = dA[i] * dA[i]; v[1] = wA[i] * wA[i];
        v[2] = dB[i] * dB[i]; v[3] = wB[i] * wB[i];
    }
};

// Model_ABC (linear ABC triblock): Hw integrand and residual sums, the
// two-block ones with a third field; chi = (chiAB, chiBC, chiAC) N
struct HwABCF {
    const double *phiA, *phiB, *phiC, *wA, *wB, *wC;
    double xab, xbc, xac;
    __device__ void operator()(long i, double* v) const {
        double a = phiA[i], b = phiB[i], c = phiC[i];
        double g = xab * a * b + xbc * b * c + xac * a * c;
        g -= wA[i] * a;
        g -= wB[i] * b;
        g -= wC[i] * c;
        v[0] = g;
    }
};

// EM branch: per field |w* - w|, |w|, |w*|; then |phiA+phiB+phiC-1|, |phiA+phiB+phiC|
struct ResidualEMABCF {
    const double *phiA, *phiB, *phiC, *wA, *wB, *wC, *yita;
    double xab, xbc, xac;
    __device__ void operator()(long i, double* v) const {
        double a = phiA[i], b = phiB[i], c = phiC[i], y = yita[i];
        double tA = xab * b + xac * c + y;
        double tB = xab * a + xbc * c + y;
        double tC = xac * a + xbc * b + y;
        v[0] = fabs(tA - wA[i]); v[1] = fabs(wA[i]); v[2] = fabs(tA);
        v[3] = fabs(tB - wB[i]); v[4] = fabs(wB[i]); v[5] = fabs(tB);
        v[6] = fabs(tC - wC[i]); v[7] = fabs(wC[i]); v[8] = fabs(tC);
        double t = a + b + c;
        v[9] = fabs(t - 1.0); v[10] = fabs(t);
    }
};

struct ResidualAXABCF {
    const double *dA, *dB, *dC, *wA, *wB, *wC;
    __device__ void operator()(long i, double* v) const {
        v[0] = dA[i] * dA[i]; v[1] = wA[i] * wA[i];
        v[2] = dB[i] * dB[i]; v[3] = wB[i] * wB[i];
        v[4] = dC[i] * dC[i]; v[5] = wC[i] * wC[i];
    }
};

struct ArcF {
    const double *a, *b;
    __device__ void operator()(long i, double* v) const { double d = a[i] - b[i]; v[0] = d * d; }
};

// ---------------------------------------------------------------------------
// density
// ---------------------------------------------------------------------------
// phi[m] = (cc * ds) * sum_{s=0}^{n} c_s q[s][m] qc[n-s][m]; cc = 1/Q from
// device memory when Qdev != nullptr, else cc_host.
__global__ void density_kernel(const double* __restrict__ q, const double* __restrict__ qc, int n, long M,
                               const double* __restrict__ c, double ds, const double* Qdev, double cc_host,
                               double* __restrict__ phi, long bstride_q, long bstride_phi, const double* Qbatch) {
    const long b = blockIdx.y;
    q += b * bstride_q;
    qc += b * bstride_q;
    phi += b * bstride_phi;
    double cc = cc_host;
    if (Qdev) cc = 1.0 / Qdev[0];
    if (Qbatch) cc = 1.0 / Qbatch[b * 8];
    const double scale = cc * ds;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M; m += stride) {
        double acc = 0.0;
        for (int s = 0; s <= n; s++) acc += c[s] * (q[(long)s * M + m] * qc[(long)(n - s) * M + m]);
        phi[m] = acc * scale;
    }
}

// ---------------------------------------------------------------------------
// simple mixing (Field.cc:51-59, Yita.cc:49-55, Model_AB.cc:205-259) fused
// with exp(-w ds/2), exp(-w ds/4) of the updated fields
// ---------------------------------------------------------------------------
__global__ void em_update_kernel(EMArgs a) {
    const long b = blockIdx.y;
    const long off = b * a.bstride;
    const double* phiA = a.phiA + off;
    const double* phiB = a.phiB + off;
    double* wA = a.wA + off;
    double* wB = a.wB + off;
    double* yita = a.yita ? a.yita + off : nullptr;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.M; i += stride) {
        double pa = phiA[i], pb = phiB[i];
        double ua, ub;
        if (a.compressible) {
            double eta = a.lamYita * (pa + pb - 1.0);
            ua = a.chiN * pb + eta;
            ub = a.chiN * pa + eta;
        } else {
            double y = yita[i] + a.lamYita * (pa + pb - 1.0);
            yita[i] = y;
            ua = a.chiN * pb + y;
            ub = a.chiN * pa + y;
        }
        double na = wA[i] * (1.0 - a.lamA) + a.lamA * ua;
        double nb = wB[i] * (1.0 - a.lamB) + a.lamB * ub;
        wA[i] = na;
        wB[i] = nb;
        if (a.eFA) {
            a.eFA[off + i] = exp(-0.5 * a.dsA * na);
            a.eHA[off + i] = exp(-0.25 * a.dsA * na);
            a.eFB[off + i] = exp(-0.5 * a.dsB * nb);
            a.eHB[off + i] = exp(-0.25 * a.dsB * nb);
        }
    }
}

// Model_ABC simple mixing (incompressible): eta += lam_eta (phiA + phiB +
// phiC - 1), wX = wX (1 - lamX) + lamX wX*, fused with the next factors
__global__ void em_update_abc_kernel(EMABCArgs a) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < a.M; i += stride) {
        const double pa = a.phi[0][i], pb = a.phi[1][i], pc = a.phi[2][i];
        const double y = a.yita[i] + a.lam[3] * (pa + pb + pc - 1.0);
        a.yita[i] = y;
        const double t[3] = {a.chi[0] * pb + a.chi[2] * pc + y, a.chi[0] * pa + a.chi[1] * pc + y,
                             a.chi[2] * pa + a.chi[1] * pb + y};
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const double nw = a.w[x][i] * (1.0 - a.lam[x]) + a.lam[x] * t[x];
            a.w[x][i] = nw;
            a.eF[x][i] = exp(-0.5 * a.ds[x] * nw);
            a.eH[x][i] = exp(-0.25 * a.ds[x] * nw);
        }
    }
}

__global__ void factors_kernel(const double* __restrict__ wA, const double* __restrict__ wB, long M, double dsA,
                               double dsB, double* eFA, double* eHA, double* eFB, double* eHB, long bstride) {
    const long b = blockIdx.y;
    const long off = b * bstride;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        double a = wA[off + i], c = wB[off + i];
        eFA[off + i] = exp(-0.5 * dsA * a);
        eHA[off + i] = exp(-0.25 * dsA * a);
        eFB[off + i] = exp(-0.5 * dsB * c);
        eHB[off + i] = exp(-0.25 * dsB * c);
    }
}

__global__ void fill_kernel(double* x, long n, double v) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = v;
}

int grid_for(long M) {
    long g = (M + 255) / 256;
    if (g > 148L * 8) g = 148L * 8;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

void launch_mean(const double* x, long M, double* partial, double* out, cudaStream_t st) {
    reduce_launch<MeanF, 1>(MeanF{x}, M, partial, out, 1.0 / (double)M, st);
}

void launch_Hw(const double* phiA, const double* phiB, const double* wA, const double* wB, long M, double chiN,
               double lamYita, int compressible, double* partial, double* out, cudaStream_t st) {
    reduce_launch<HwF, 1>(HwF{phiA, phiB, wA, wB, chiN, lamYita, compressible}, M, partial, out, 1.0 / (double)M, st);
}

void launch_residual_em(const double* phiA, const double* phiB, const double* wA, const double* wB,
                        const double* yita, long M, double chiN, double lamYita, int compressible, double* partial,
                        double* out8, cudaStream_t st) {
    reduce_launch<ResidualEMF, 8>(ResidualEMF{phiA, phiB, wA, wB, yita, chiN, lamYita, compressible}, M, partial,
                                  out8, 1.0 / (double)M, st);
}

void launch_residual_ax(const double* dA, const double* dB, const double* wA, const double* wB, long M,
                        double* partial, double* out4, cudaStream_t st) {
    reduce_launch<ResidualAXF, 4>(ResidualAXF{dA, dB, wA, wB}, M, partial, out4, 1.0 / (double)M, st);
}

void launch_Hw_abc(const double* const phi[3], const double* const w[3], const double chi[3], long M,
                   double* partial, double* out, cudaStream_t st) {
    reduce_launch<HwABCF, 1>(HwABCF{phi[0], phi[1], phi[2], w[0], w[1], w[2], chi[0], chi[1], chi[2]}, M, partial,
                             out, 1.0 / (double)M, st);
}

void launch_residual_em_abc(const double* const phi[3], const double* const w[3], const double* yita,
                            const double chi[3], long M, double* partial, double* out11, cudaStream_t st) {
    reduce_launch<ResidualEMABCF, 11>(
        ResidualEMABCF{phi[0], phi[1], phi[2], w[0], w[1], w[2], yita, chi[0], chi[1], chi[2]}, M, partial, out11,
        1.0 / (double)M, st);
}

void launch_residual_ax_abc(const double* const d[3], const double* const w[3], long M, double* partial,
                            double* out6, cudaStream_t st) {
    reduce_launch<ResidualAXABCF, 6>(ResidualAXABCF{d[0], d[1], d[2], w[0], w[1], w[2]}, M, partial, out6,
                                     1.0 / (double)M, st);
}

void launch_em_update_abc(const EMABCArgs& a, cudaStream_t st) {
    em_update_abc_kernel<<<grid_for(a.M), 256, 0, st>>>(a);
    PS_CUDA(cudaGetLastError());
}

void launch_arc_sq(const double* a, const double* b, long M, double* partial, double* out, cudaStream_t st) {
    reduce_launch<ArcF, 1>(ArcF{a, b}, M, partial, out, 1.0 / (double)M, st);
}

void launch_density(const double* q, const double* qc, int n, long M, const double* c, double ds,
                    const double* Qdev, double cc_host, double* phi, int nbatch, long bstride_q, long bstride_phi,
                    const double* Qbatch, cudaStream_t st) {
    dim3 grid(grid_for(M), nbatch);
    density_kernel<<<grid, 256, 0, st>>>(q, qc, n, M, c, ds, Qdev, cc_host, phi, bstride_q, bstride_phi, Qbatch);
    PS_CUDA(cudaGetLastError());
}

void launch_em_update(const EMArgs& a, int nbatch, cudaStream_t st) {
    dim3 grid(grid_for(a.M), nbatch);
    em_update_kernel<<<grid, 256, 0, st>>>(a);
    PS_CUDA(cudaGetLastError());
}

void launch_factors(const double* wA, const double* wB, long M, double dsA, double dsB, double* eFA, double* eHA,
                    double* eFB, double* eHB, int nbatch, long bstride, cudaStream_t st) {
    dim3 grid(grid_for(M), nbatch);
    factors_kernel<<<grid, 256, 0, st>>>(wA, wB, M, dsA, dsB, eFA, eHA, eFB, eHB, bstride);
    PS_CUDA(cudaGetLastError());
}

void launch_fill(double* x, long n, double v, cudaStream_t st) {
    fill_kernel<<<grid_for(n), 256, 0, st>>>(x, n, v);
    PS_CUDA(cudaGetLastError());
}

}  // namespace ps
