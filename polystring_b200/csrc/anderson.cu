// anderson.cu -- Anderson mixing of the A and B fields kept on the device
// (restates FieldAX, src/FieldAX.cc:152-427, as driven by Model_AB::update,
// src/Model_AB.cc:206-253).
//
// History layout per field: w(i), d(i), i = 0..n, each M doubles; the ring
// position cur and the iteration count k live in device memory (AXState) so
// that one SCFT iteration can be captured once in a CUDA graph and replayed.
//
// Per iteration:
//   ax_prepare  d(cur) = w_target - w(cur) for A and B       (update_d)
//   ax_dots     partial sums of d(cur) . d(find_index(j)), j = 0..nn (4 j per CTA row)
//   ax_solve    B shift + new row (update_B), U = UA + UB, V = VA + VB,
//               C = U^-1 V by Gaussian elimination with partial pivoting,
//               ramp 1 - lambda^(k+1), ring position update     (one block, shared memory)
//   ax_combine  W = w(cur) + sum C (w(kk) - w(cur)), D likewise,
//               w(cur') = W + ramp D, plus the next Boltzmann factors
#include "ps_internal.h"
#include "field_kernels.h"
#include "anderson.h"

namespace ps {

namespace {

__device__ __forceinline__ int find_index(int cur, int n, int j) {
    int i = j + cur;
    if (i > n) i -= (n + 1);
    return i;
}

// yita / eta and d(cur) for every field
template <int NF>
__global__ void ax_prepare_kernel(AXArgs a) {
    const AXState* s = a.state;
    const int cur = s->cur;
    const long M = a.M;
    double* dA = a.dA + (long)cur * M;
    double* dB = a.dB + (long)cur * M;
    const double* wA = a.wA + (long)cur * M;
    const double* wB = a.wB + (long)cur * M;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        double pa = a.phiA[i], pb = a.phiB[i];
        if constexpr (NF == 2) {
            double y;
            if (a.compressible) {
                y = a.lamYita * (pa + pb - 1.0);
            } else {
                y = 0.5 * (a.dataA[i] + a.dataB[i] - a.chiN);
                a.yita[i] = y;
            }
            dA[i] = (a.chiN * pb + y) - wA[i];
            dB[i] = (a.chiN * pa + y) - wB[i];
        } else {
            const double pc = a.phiC[i];
            const double xab = a.chi[0], xbc = a.chi[1], xac = a.chi[2];
            const double sw = a.dataA[i] + a.dataB[i] + a.dataC[i];
            const double y = (sw - xab * (pa + pb) - xbc * (pb + pc) - xac * (pa + pc)) / 3.0;
            a.yita[i] = y;
            dA[i] = (xab * pb + xac * pc + y) - wA[i];
            dB[i] = (xab * pa + xbc * pc + y) - wB[i];
            a.dC[(long)cur * M + i] = (xac * pa + xbc * pb + y) - a.wC[(long)cur * M + i];
        }
    }
}

// partial sums of d(cur) . d(find_index(j)) for j = 4 blockIdx.y .. + 3
// (every field); every thread visits the same points i in the same order
// for every j, so the sums do not depend on the split over blockIdx.y
constexpr int kJC = 4;

template <int NF, int NMAX>
__global__ void __launch_bounds__(kRedThreads) ax_dots_kernel(AXArgs a, double* partial) {
    const AXState* s = a.state;
    const int n = s->n, cur = s->cur;
    const int nn = s->k < n ? s->k : n;
    const long M = a.M;
    const int j0 = blockIdx.y * kJC;
    const double* dF[3] = {a.dA, a.dB, NF == 3 ? a.dC : a.dA};
    double acc[NF * kJC];
#pragma unroll
    for (int j = 0; j < NF * kJC; j++) acc[j] = 0.0;
    long kk[kJC];
#pragma unroll
    for (int j = 0; j < kJC; j++) kk[j] = (long)find_index(cur, n, j0 + j <= nn ? j0 + j : 0) * M;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
#pragma unroll
        for (int f = 0; f < NF; f++) {
            const double x = dF[f][(long)cur * M + i];
#pragma unroll
            for (int j = 0; j < kJC; j++)
                if (j0 + j <= nn) acc[f * kJC + j] += x * dF[f][kk[j] + i];
        }
    }
    // block reduction
    __shared__ double sh[NF * kJC][kRedThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NF * kJC; j++) {
        double v = acc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[j][warp] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NF * kJC; q += blockDim.x) {
        const int f = q / kJC, j = j0 + (q % kJC);
        if (j >= NMAX) continue;
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; w++) t += sh[q][w];
        partial[(long)blockIdx.x * NF * NMAX + f * NMAX + j] = t;
    }
}

// update_B, U = UA + UB, V = VA + VB and C = U^-1 V by Gaussian elimination
// with partial pivoting, in shared memory across the block.  Every matrix
// element gets the same operations as in the oracle's orc_solve_small (row i
// of step k: f = A[i][k] / piv, A[i][j] -= f A[k][j]); the pivot is the first
// row of largest |A[i][k]|; back substitution runs in order on one thread.
template <int NF, int NMAX>
__global__ void __launch_bounds__(kRedThreads) ax_solve_kernel(AXArgs a, const double* partial, int G) {
    AXState* s = a.state;
    const int n = s->n;
    const int N1 = n + 1;
    const int nn = s->k < n ? s->k : n;
    const int tid = threadIdx.x, nt = blockDim.x;
    __shared__ double row[NF * NMAX];
    __shared__ double sB[NF][(NMAX + 1) * (NMAX + 1)];
    __shared__ double U[NMAX * NMAX], V[NMAX], C[NMAX], F[NMAX];
    __shared__ int piv_row, singular;
    // fixed-order reduction of the partial sums
    for (int j = tid; j < NF * NMAX; j += nt) {
        double t = 0.0;
        for (int b = 0; b < G; b++) t += partial[(long)b * NF * NMAX + j];
        row[j] = t / (double)a.M;
    }
    double* BG[3] = {a.BA, a.BB, a.BC};
    for (int f = 0; f < NF; f++)
        for (int e = tid; e < N1 * N1; e += nt) sB[f][e] = BG[f][e];
    if (tid == 0) singular = 0;
    __syncthreads();
    // update_B (FieldAX.cc:321-345): shift the upper triangle down the diagonal
    double shifted[NF][((NMAX + 1) * (NMAX + 1) + kRedThreads - 1) / kRedThreads];
    for (int f = 0; f < NF; f++) {
        int c = 0;
        for (int e = tid; e < N1 * N1; e += nt, c++) {
            const int i = e / N1, j = e - i * N1;
            shifted[f][c] = (i >= 1 && j >= i) ? sB[f][(i - 1) * N1 + (j - 1)] : sB[f][e];
        }
    }
    __syncthreads();
    for (int f = 0; f < NF; f++) {
        int c = 0;
        for (int e = tid; e < N1 * N1; e += nt, c++) sB[f][e] = shifted[f][c];
    }
    __syncthreads();
    for (int j = tid; j <= nn; j += nt)     // new row 0
        for (int f = 0; f < NF; f++) sB[f][j] = row[f * NMAX + j];
    __syncthreads();
    for (int f = 0; f < NF; f++)            // symmetrise
        for (int e = tid; e < N1 * N1; e += nt) {
            const int i = e / N1, j = e - i * N1;
            if (j < i) sB[f][e] = sB[f][j * N1 + i];
        }
    __syncthreads();
    for (int f = 0; f < NF; f++)
        for (int e = tid; e < N1 * N1; e += nt) BG[f][e] = sB[f][e];
    // U = UA + UB (+ UC), V = VA + VB (+ VC) (FieldAX.cc:352-381)
    for (int e = tid; e < nn * nn; e += nt) {
        const int i = e / nn, j = e - i * nn;
        double u = 0.0;
        for (int f = 0; f < NF; f++) {
            const double* Bf = sB[f];
            u = u + (Bf[0] - Bf[(i + 1) * N1] - Bf[j + 1] + Bf[(i + 1) * N1 + (j + 1)]);
        }
        U[e] = u;
    }
    for (int i = tid; i < nn; i += nt) {
        double v = 0.0;
        for (int f = 0; f < NF; f++) v = v + (sB[f][0] - sB[f][(i + 1) * N1]);
        V[i] = v;
    }
    __syncthreads();
    for (int k = 0; k < nn; k++) {
        if (tid == 0) {
            int p = k;
            double best = fabs(U[k * nn + k]);
            for (int i = k + 1; i < nn; i++) {
                const double v = fabs(U[i * nn + k]);
                if (v > best) { best = v; p = i; }
            }
            piv_row = p;
            if (best == 0.0) singular = 1;
        }
        __syncthreads();
        if (singular) break;
        const int p = piv_row;
        if (p != k) {
            for (int j = tid; j < nn; j += nt) {
                const double t = U[k * nn + j];
                U[k * nn + j] = U[p * nn + j];
                U[p * nn + j] = t;
            }
            if (tid == 0) {
                const double t = V[k];
                V[k] = V[p];
                V[p] = t;
            }
        }
        __syncthreads();
        const double pv = U[k * nn + k];
        for (int i = k + 1 + tid; i < nn; i += nt) F[i] = U[i * nn + k] / pv;
        __syncthreads();
        const int w = nn - k - 1;           // columns k+1 .. nn-1 of rows k+1 .. nn-1
        for (int e = tid; e < w * w; e += nt) {
            const int i = k + 1 + e / w, j = k + 1 + e % w;
            U[i * nn + j] -= F[i] * U[k * nn + j];
        }
        for (int i = k + 1 + tid; i < nn; i += nt) {
            U[i * nn + k] = 0.0;
            V[i] -= F[i] * V[k];
        }
        __syncthreads();
    }
    if (tid != 0) return;
    int nc = 0;
    if (nn > 0) {
        if (singular) {
            s->status |= 1;
            for (int i = 0; i < nn; i++) C[i] = 0.0;
        } else {
            for (int i = nn - 1; i >= 0; i--) {
                double t = V[i];
                for (int j = i + 1; j < nn; j++) t -= U[i * nn + j] * C[j];
                C[i] = t / U[i * nn + i];
            }
        }
        nc = nn;
    }
    for (int i = 0; i < nc; i++) s->C[i] = C[i];
    s->nc = nc;
    s->rampA = 1.0 - pow(s->lamA, (double)(s->k + 1));
    s->rampB = 1.0 - pow(s->lamB, (double)(s->k + 1));
    if (NF == 3) s->rampC = 1.0 - pow(s->lamC, (double)(s->k + 1));
    s->cur_old = s->cur;
    s->cur_new = s->cur > 0 ? s->cur - 1 : n;
    s->cur = s->cur_new;
    s->k += 1;
}

// W and D of one field at point i, w(cur') = W + ramp D
__device__ __forceinline__ double ax_mix(const double* w, const double* d, long oc, long i, const double* C,
                                         const long* kk, int nc, double ramp) {
    const double wc = w[oc + i], dc = d[oc + i];
    double W = wc, D = dc;
    for (int j = 0; j < nc; j++) {
        W += C[j] * (w[kk[j] + i] - wc);
        D += C[j] * (d[kk[j] + i] - dc);
    }
    return W + ramp * D;
}

template <int NF>
__global__ void ax_combine_kernel(AXArgs a) {
    const AXState* s = a.state;
    const int n = s->n, co = s->cur_old, cn = s->cur_new, nc = s->nc;
    const long M = a.M;
    __shared__ double C[kAXMaxHist];
    __shared__ long kk[kAXMaxHist];
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        C[i] = s->C[i];
        kk[i] = (long)find_index(co, n, i + 1) * M;
    }
    __syncthreads();
    const double rA = s->rampA, rB = s->rampB, rC = s->rampC;
    const long oc = (long)co * M, on = (long)cn * M;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
        const double na = ax_mix(a.wA, a.dA, oc, i, C, kk, nc, rA);
        const double nb = ax_mix(a.wB, a.dB, oc, i, C, kk, nc, rB);
        a.wA[on + i] = na;
        a.wB[on + i] = nb;
        a.dataA[i] = na;
        a.dataB[i] = nb;
        if (a.eFA) {
            a.eFA[i] = exp(-0.5 * a.dsA * na);
            a.eHA[i] = exp(-0.25 * a.dsA * na);
            a.eFB[i] = exp(-0.5 * a.dsB * nb);
            a.eHB[i] = exp(-0.25 * a.dsB * nb);
        }
        if constexpr (NF == 3) {
            const double nc3 = ax_mix(a.wC, a.dC, oc, i, C, kk, nc, rC);
            a.wC[on + i] = nc3;
            a.dataC[i] = nc3;
            if (a.eFC) {
                a.eFC[i] = exp(-0.5 * a.dsC * nc3);
                a.eHC[i] = exp(-0.25 * a.dsC * nc3);
            }
        }
    }
}

int grid_for(long M) {
    long g = (M + 255) / 256;
    if (g > 148L * 8) g = 148L * 8;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

int ax_nmax(int n) {
    if (n + 1 <= 8) return 8;
    if (n + 1 <= 16) return 16;
    if (n + 1 <= 32) return 32;
    return 0;
}

template <int NF, int NMAX>
void launch_ax_nf(const AXArgs& a, double* partial, cudaStream_t st) {
    ax_dots_kernel<NF, NMAX><<<dim3(kRedBlocks, (NMAX + kJC) / kJC), kRedThreads, 0, st>>>(a, partial);
    ax_solve_kernel<NF, NMAX><<<1, kRedThreads, 0, st>>>(a, partial, kRedBlocks);
}

template <int NF>
void launch_anderson_nf(const AXArgs& a, double* partial, cudaStream_t st) {
    const int nmax = ax_nmax(a.n);
    if (nmax == 0) throw Error(-2, "Anderson history longer than 31 is not supported");
    ax_prepare_kernel<NF><<<grid_for(a.M), 256, 0, st>>>(a);
    PS_CUDA(cudaGetLastError());
    switch (nmax) {
    case 8: launch_ax_nf<NF, 8>(a, partial, st); break;
    case 16: launch_ax_nf<NF, 16>(a, partial, st); break;
    default: launch_ax_nf<NF, 32>(a, partial, st); break;
    }
    PS_CUDA(cudaGetLastError());
    ax_combine_kernel<NF><<<grid_for(a.M), 256, 0, st>>>(a);
    PS_CUDA(cudaGetLastError());
}

void launch_anderson(const AXArgs& a, double* partial, cudaStream_t st) {
    if (a.nf == 3) {
        if (a.compressible) throw Error(-2, "three-field Anderson mixing is incompressible");
        launch_anderson_nf<3>(a, partial, st);
    } else {
        launch_anderson_nf<2>(a, partial, st);
    }
}

}  // namespace ps
