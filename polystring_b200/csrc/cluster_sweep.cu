// cluster_sweep.cu -- RQM4 propagator sweeps of a batch of 2D problems, one
// thread-block cluster per problem, both packed fields resident in the
// cluster's distributed shared memory for the whole sweep.
//
// The string method advances m images of the same small 2D grid at once
// (polystring_AB.cc:111-208 runs one SCFT solve per image).  An image's two
// packed complex work fields (lane f = forward chain in the real part, lane c
// = complementary chain in the imaginary part, as in the line passes) fit in
// the shared memory of C CTAs: CTA r of the cluster owns rows x in
// [r LX/C, (r+1) LX/C) in "row layout" (y lines contiguous, pitch LY + 1).
// A 2D transform is
//
//   y FFTs in row layout | cluster transpose | x FFTs in column layout
//
// where the column layout gives CTA r the columns y in [r LY/C, (r+1) LY/C)
// for every x.  The transposes read the peers' shared memory (DSMEM) into
// registers between hardware cluster barriers, then overwrite the local
// buffer in place, so each field needs one buffer per CTA.
//
// One contour step (RQM4.cc:66-92, same operation order as sweep.cu):
//   A = e^{-w ds/2} q, B = e^{-w ds/4} q      (row layout)
//   A <- F^-1 L1 F A, B <- F^-1 L2 F B
//   u = e^{-w ds/2} A / M  (kept in A's buffer), B <- e^{-w ds/4} (e^{-w ds/4} B / M)
//   B <- F^-1 L2 F B
//   q[t+1] = (4 e^{-w ds/4} B / M - u) / 3    -> history, next step's A and B
//
// No grid barrier and no spin wait: the cluster barrier is a hardware
// barrier every thread of every CTA of the cluster reaches the same number of
// times, and clusters are independent, so they need not be co-resident.
#include <cooperative_groups.h>

#include <cstdio>

#include "ps_internal.h"
#include "fft_core.cuh"
#include "smem_line_fft.cuh"
#include "engine.h"
#include "sweep.h"

namespace cg = cooperative_groups;

namespace ps {

namespace {

constexpr int kCT = 256;   // threads per CTA

template <int LX, int LY, int C>
struct CGeo {
    static constexpr int XR = LX / C;          // rows per CTA (row layout)
    static constexpr int YC = LY / C;          // columns per CTA (column layout)
    static constexpr int RP = LY + 1;          // row pitch in double2
    static constexpr int FS = XR * RP;         // one field's buffer (double2)
    static constexpr int E = XR * LY;          // points per CTA (= LX * YC)
    static constexpr int EPT = E / kCT;        // points per thread
    static constexpr long M = (long)LX * LY;
    static_assert(LX % C == 0 && LY % C == 0, "C must divide both axes");
    static_assert(E % kCT == 0 && E / kCT >= 1, "whole points per thread");
    static_assert(LX * YC == E && E <= FS, "column layout fits the row buffer");
};

// row-layout index of CTA-local point e (x_local = e / LY, y = e % LY)
template <class G, int LY>
__device__ __forceinline__ int ridx(int e) { return (e / LY) * G::RP + (e % LY); }

// peers' row-layout points -> this CTA's column-layout points (e = x * YC + yl)
template <class G>
__device__ __forceinline__ void gather_rc(double2 (&v)[G::EPT], double2* fld, int r, cg::cluster_group& cl) {
#pragma unroll
    for (int k = 0; k < G::EPT; k++) {
        const int e = threadIdx.x + k * kCT;
        const int x = e / G::YC, yl = e % G::YC;
        const double2* src = cl.map_shared_rank(fld, (unsigned)(x / G::XR));
        v[k] = src[(x % G::XR) * G::RP + r * G::YC + yl];
    }
}
template <class G>
__device__ __forceinline__ void put_c(const double2 (&v)[G::EPT], double2* fld) {
#pragma unroll
    for (int k = 0; k < G::EPT; k++) fld[threadIdx.x + k * kCT] = v[k];
}
// peers' column-layout points -> this CTA's row-layout points
template <class G, int LY>
__device__ __forceinline__ void gather_cr(double2 (&v)[G::EPT], double2* fld, int r, cg::cluster_group& cl) {
#pragma unroll
    for (int k = 0; k < G::EPT; k++) {
        const int e = threadIdx.x + k * kCT;
        const int xl = e / LY, y = e % LY;
        const double2* src = cl.map_shared_rank(fld, (unsigned)(y / G::YC));
        v[k] = src[(r * G::XR + xl) * G::YC + (y % G::YC)];
    }
}
template <class G, int LY>
__device__ __forceinline__ void put_r(const double2 (&v)[G::EPT], double2* fld) {
#pragma unroll
    for (int k = 0; k < G::EPT; k++) fld[ridx<G, LY>(threadIdx.x + k * kCT)] = v[k];
}

template <int LX, int LY, int C, class PX, class PY>
__global__ void __launch_bounds__(kCT, 3) cluster_sweep2d_kernel(SweepArgs a) {
    using G = CGeo<LX, LY, C>;
    // One field at a time: an in-place pass holds all of a thread's points in
    // registers across its barrier, 8 double2 per field at 128^2 / 8 CTAs.
    // y lines (row layout: element y of row xl at xl * RP + y)
    using YF = SmemLineFFT<LY, G::XR, 1, OffMul<G::RP>, -1, kCT, PY>;
    using YI = SmemLineFFT<LY, G::XR, 1, OffMul<G::RP>, +1, kCT, PY>;
    // x lines (column layout: element x of column yl at x * YC + yl)
    using XF = SmemLineFFT<LX, G::YC, G::YC, OffMul<1>, -1, kCT, PX>;
    using XI = SmemLineFFT<LX, G::YC, G::YC, OffMul<1>, +1, kCT, PX>;

    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const long img = blockIdx.x / C;

    extern __shared__ double2 sm[];
    double2* twx = sm;
    double2* twy = twx + LX;
    double2* A = twy + LY;
    double2* B = A + G::FS;
    for (int i = threadIdx.x; i < LX; i += kCT) twx[i] = a.twx[i];
    for (int i = threadIdx.x; i < LY; i += kCT) twy[i] = a.twy[i];

    const long M = G::M;
    const double Md = (double)M;
    const double rMd = 1.0 / Md;
    const bool mpow2 = (M & (M - 1)) == 0;   // x / M == x * (1 / M) exactly
    const long boff = img * a.bstride_batch;
    double* hf = a.hf + img * a.bstride_hist;
    double* hc = a.hc + img * a.bstride_hist;
    const double* L1 = a.L1 + img * a.bstride_L;
    const double* L2 = a.L2 + img * a.bstride_L;
    const long g0 = (long)r * G::E;          // this CTA's rows in natural order
    auto eF = [&](int lane, int t) -> const double* {   // e^{-w ds/2} of the lane's block at step t
        int blk = lane == 0 ? (t < a.LA ? 0 : 1) : (t < a.LB ? 1 : 0);
        return (blk == 0 ? a.eFA : a.eFB) + boff;
    };
    auto eH = [&](int lane, int t) -> const double* {
        int blk = lane == 0 ? (t < a.LA ? 0 : 1) : (t < a.LB ? 1 : 0);
        return (blk == 0 ? a.eHA : a.eHB) + boff;
    };
    double2 v[G::EPT];

    // k-space multiply in column layout: B by L2 (half step), A by L1 (full step)
    auto kmul = [&](bool both) {
#pragma unroll 4
        for (int k = 0; k < G::EPT; k++) {
            const int e = threadIdx.x + k * kCT;
            const long kx = (long)(e / G::YC) * LY + r * G::YC + (e % G::YC);
            double l2 = L2[kx];
            double2 b = B[e];
            B[e] = make_double2(b.x * l2, b.y * l2);
            if (both) {
                double l1 = L1[kx];
                double2 c = A[e];
                A[e] = make_double2(c.x * l1, c.y * l1);
            }
        }
        __syncthreads();
    };

    // step 0 inputs: A = e^{-w ds/2} q[0], B = e^{-w ds/4} q[0]
    {
        const double *ef = eF(0, 0), *ec = eF(1, 0), *hfp = eH(0, 0), *hcp = eH(1, 0);
#pragma unroll 4
        for (int k = 0; k < G::EPT; k++) {
            const int e = threadIdx.x + k * kCT;
            const long g = g0 + e;
            const int si = ridx<G, LY>(e);
            const double qf = hf[g], qc = hc[g];
            A[si] = make_double2(ef[g] * qf, ec[g] * qc);
            B[si] = make_double2(hfp[g] * qf, hcp[g] * qc);
        }
    }
    __syncthreads();

    for (int t = 0; t < a.Ns; t++) {
        // ---- full step (A, L1) and first half step (B, L2) -------------------
        YF::run(A, twy, OffMul<G::RP>());
        YF::run(B, twy, OffMul<G::RP>());
        cl.sync();                                   // rows of every CTA final
        gather_rc<G>(v, A, r, cl);
        cl.sync();                                   // no CTA reads A any more
        put_c<G>(v, A);
        gather_rc<G>(v, B, r, cl);
        cl.sync();                                   // no CTA reads B any more
        put_c<G>(v, B);
        __syncthreads();
        XF::run(A, twx, OffMul<1>());
        XF::run(B, twx, OffMul<1>());
        kmul(true);
        XI::run(A, twx, OffMul<1>());
        XI::run(B, twx, OffMul<1>());
        cl.sync();                                   // columns of every CTA final
        gather_cr<G, LY>(v, A, r, cl);
        cl.sync();
        put_r<G, LY>(v, A);
        gather_cr<G, LY>(v, B, r, cl);
        cl.sync();
        put_r<G, LY>(v, B);
        __syncthreads();
        YI::run(A, twy, OffMul<G::RP>());
        YI::run(B, twy, OffMul<G::RP>());
        {
            const double *ef = eF(0, t), *ec = eF(1, t), *hfp = eH(0, t), *hcp = eH(1, t);
#pragma unroll 4
            for (int k = 0; k < G::EPT; k++) {
                const int e = threadIdx.x + k * kCT;
                const long g = g0 + e;
                const int si = ridx<G, LY>(e);
                const double2 z1 = A[si];
                A[si] = make_double2(div_pow2_or_rn(z1.x * ef[g], Md, rMd, mpow2),
                                     div_pow2_or_rn(z1.y * ec[g], Md, rMd, mpow2));
                const double2 z2 = B[si];
                const double ha = hfp[g], hb = hcp[g];
                const double qtf = div_pow2_or_rn(z2.x * ha, Md, rMd, mpow2);
                const double qtc = div_pow2_or_rn(z2.y * hb, Md, rMd, mpow2);
                B[si] = make_double2(ha * qtf, hb * qtc);
            }
        }
        __syncthreads();
        // ---- second half step (B, L2) -----------------------------------------
        YF::run(B, twy, OffMul<G::RP>());
        cl.sync();
        gather_rc<G>(v, B, r, cl);
        cl.sync();
        put_c<G>(v, B);
        __syncthreads();
        XF::run(B, twx, OffMul<1>());
        kmul(false);
        XI::run(B, twx, OffMul<1>());
        cl.sync();
        gather_cr<G, LY>(v, B, r, cl);
        cl.sync();
        put_r<G, LY>(v, B);
        __syncthreads();
        YI::run(B, twy, OffMul<G::RP>());
        // ---- q[t+1] = (4 qt2 - u) / 3; next step's A and B --------------------
        {
            const bool next = t + 1 < a.Ns;
            const double *hfp = eH(0, t), *hcp = eH(1, t);
            const double *nf1 = eF(0, t + 1), *nc1 = eF(1, t + 1), *nf2 = eH(0, t + 1), *nc2 = eH(1, t + 1);
            double* of = hf + (long)(t + 1) * M;
            double* oc = hc + (long)(t + 1) * M;
#pragma unroll 4
            for (int k = 0; k < G::EPT; k++) {
                const int e = threadIdx.x + k * kCT;
                const long g = g0 + e;
                const int si = ridx<G, LY>(e);
                const double2 z3 = B[si];
                const double2 u = A[si];
                double qf = div_pow2_or_rn(z3.x * hfp[g], Md, rMd, mpow2);
                double qc = div_pow2_or_rn(z3.y * hcp[g], Md, rMd, mpow2);
                qf = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
                qc = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
                of[g] = qf;
                oc[g] = qc;
                if (next) {
                    A[si] = make_double2(nf1[g] * qf, nc1[g] * qc);
                    B[si] = make_double2(nf2[g] * qf, nc2[g] * qc);
                }
            }
        }
        __syncthreads();
    }
    cl.sync();   // no peer reads this CTA's shared memory after it exits
}

template <int LX, int LY, int C>
auto kernel_of() {
    return cluster_sweep2d_kernel<LX, LY, C, Plan<LX>, Plan<LY>>;
}

template <int LX, int LY, int C>
size_t cl_smem() {
    using G = CGeo<LX, LY, C>;
    return sizeof(double2) * ((size_t)LX + LY + 2 * (size_t)G::FS);
}

template <int LX, int LY, int C>
cudaLaunchConfig_t cl_config(int nbatch, cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * nbatch), 1, 1);
    cfg.blockDim = dim3(kCT, 1, 1);
    cfg.dynamicSmemBytes = cl_smem<LX, LY, C>();
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <int LX, int LY, int C>
int cluster_prepare_t(int nbatch) {
    auto k = kernel_of<LX, LY, C>();
    PS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cl_smem<LX, LY, C>()));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cl_config<LX, LY, C>(nbatch, nullptr, attr);
    int n = 0, per_sm = 0;
    PS_CUDA(cudaOccupancyMaxActiveClusters(&n, k, &cfg));
    PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kCT, cl_smem<LX, LY, C>()));
    char line[200];
    std::snprintf(line, sizeof(line), "grid %dx%dx1 cluster sweep: %d CTAs per problem, %d CTAs per SM, "
                  "%d clusters resident at once, batch %d\n", LX, LY, C, per_sm, n, nbatch);
    tuning_note(line);
    twiddle_table(LX);
    twiddle_table(LY);
    return n;
}

template <int LX, int LY, int C>
void cluster_launch_t(SweepArgs a, int nbatch, cudaStream_t st) {
    a.twx = twiddle_table(LX);
    a.twy = twiddle_table(LY);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cl_config<LX, LY, C>(nbatch, st, attr);
    PS_CUDA(cudaLaunchKernelEx(&cfg, kernel_of<LX, LY, C>(), a));
}

}  // namespace

// (LX, LY, CTAs per cluster)
#define PS_CLUSTER_SHAPES(X) X(32, 32, 4) X(64, 64, 4) X(128, 128, 8)

bool cluster_sweep_supported(int Lx, int Ly, int Lz) {
#define PS_X(x, y, c) if (Lx == x && Ly == y && Lz == 1) return true;
    PS_CLUSTER_SHAPES(PS_X)
#undef PS_X
    return false;
}

int cluster_sweep_prepare(int Lx, int Ly, int Lz, int nbatch) {
#define PS_X(x, y, c) if (Lx == x && Ly == y && Lz == 1) return cluster_prepare_t<x, y, c>(nbatch);
    PS_CLUSTER_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no cluster sweep for this grid");
}

void cluster_sweep_launch(const SweepArgs& a, int Lx, int Ly, int Lz, int nbatch, cudaStream_t st) {
#define PS_X(x, y, c) if (Lx == x && Ly == y && Lz == 1) { cluster_launch_t<x, y, c>(a, nbatch, st); return; }
    PS_CLUSTER_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no cluster sweep for this grid");
}

}  // namespace ps
