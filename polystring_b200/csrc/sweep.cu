// sweep.cu -- one persistent cooperative kernel per propagator sweep.
//
// The paired chains (lane f in the real part, lane c in the imaginary part
// of a packed complex field; see line_pass.cu) are advanced through all Ns
// RQM4 contour steps inside a single launch.  Each contour step is four
// phases separated by grid barriers:
//
//   plane   2D FFT (y, z) of whole x-slabs in shared memory, fused with the
//           real-space work of the step (e^{-w h/2} multiplies, 1/M, the
//           Richardson combination (4 q_half - q_full)/3, history writes)
//   x-pass  FFT along x of column tiles, k-space multiply, inverse FFT
//
//   step t:  x-pass(Z1, Z2)  |  plane: Z1 -> u ; Z2 -> qt -> Z3  |
//            x-pass(Z3)      |  plane: Z3 -> q[t+1] -> Z1', Z2' (step t+1)
//
// Z1 carries the full ds step, Z2 and Z3 the two ds/2 steps (RQM4.cc:66-92).
// Line FFTs are Stockham radix passes with every thread's butterfly inputs
// staged in registers, so each transform runs in place in one buffer.  All
// shapes are compile-time, so the index arithmetic is constant division.
//
// Grid barriers are counter based with a bounded spin: on timeout a CTA
// raises the error flag, every CTA sees the flag and returns, and the host
// reports the failure.  The launch is cooperative, so all CTAs are resident.
//
// Two launch forms share the body: one problem (or a strided batch) at 512
// threads a CTA, one CTA an SM; and a batch of independent problems of one
// shape described by per-problem descriptors (uneven batches), at 256
// threads a CTA, two CTAs an SM.  The thread count and the x-tile width
// change which thread computes what, never the arithmetic, so a batched
// problem's results equal its single solve's bit for bit.
#include "ps_internal.h"
#include "fft_core.cuh"
#include "smem_line_fft.cuh"
#include "sweep.h"

namespace ps {

namespace {

constexpr int kNT = 512;                 // threads per CTA (one problem a launch)
constexpr int kNTB = 256;                // threads per CTA of the descriptor batches (2 CTAs an SM)
constexpr long long kSpinLimit = 20000000; // polls before a barrier gives up

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Returns false when the sweep must stop (error flag raised).
__device__ __forceinline__ bool grid_barrier(unsigned* count, int* err, unsigned target) {
    __syncthreads();
    __shared__ int stop;
    if (threadIdx.x == 0) {
        int s = 0;
        __threadfence();
        red_release_add(count, 1u);
        long long spins = 0;
        while (ld_acquire(count) < target) {
            if (*((volatile int*)err)) { s = 1; break; }
            if (++spins > kSpinLimit) {
                atomicExch(err, 2);
                s = 1;
                break;
            }
        }
        __threadfence();
        stop = s;
    }
    __syncthreads();
    return stop == 0;
}

// in-place line FFTs with register staging (smem_line_fft.cuh), NT threads;
// 48-point lines in two passes (16 then 3) rather than the three of Plan<48>
// (measured: 48^3 contour step 79 -> 65 us)
struct Plan16x3 { static constexpr int P = 2, r0 = 16, r1 = 3, r2 = 1; };
template <int N> struct SweepPlan { using type = Plan<N>; };
template <> struct SweepPlan<48> { using type = Plan16x3; };
template <int N, int NL, int ES, class Off, int SIGN, int NT>
using LineFFT = SmemLineFFT<N, NL, ES, Off, SIGN, NT, typename SweepPlan<N>::type>;

constexpr int largest_div_le(int n, int cap) {
    int t = cap < n ? cap : n;
    while (t > 1 && n % t != 0) t--;
    return t < 1 ? 1 : t;
}

// XTC: elements per x line of an x tile at most (tile columns = XTC / LX)
template <int LX, int LY, int LZ, int XTC = 2048>
struct Geo {
    static constexpr int P = LY * LZ;                       // points per x-slab
    static constexpr long M = (long)LX * P;
    static constexpr int PR = (P >= 4096) ? 1 : largest_div_le(LX, 4096 / P);  // slabs per plane task
    static constexpr int PT = PR * P;                       // points per plane task
    static constexpr int NPT = LX / PR;                     // plane tasks per role
    static constexpr int ZP = (LZ > 1 && LZ % 2 == 0) ? LZ + 1 : LZ;  // smem row pitch
    static constexpr int XT = largest_div_le(P, (XTC + LX - 1) / LX);  // columns per x tile
    static constexpr int NXT = P / XT;                      // x tiles
    static constexpr int PLANE_SMEM = PR * LY * ZP;         // double2
    static constexpr int XTILE_SMEM = 2 * LX * XT;          // double2 (two fields)
    static constexpr int SMEM = (PLANE_SMEM > XTILE_SMEM ? PLANE_SMEM : XTILE_SMEM);
};

// smem index of plane-task point p (natural order inside the task's slabs)
template <class G, int LZ>
__device__ __forceinline__ int pidx(int p) {
    return (p / LZ) * G::ZP + (p % LZ);
}

template <int LX, int LY, int LZ, int SIGN, int NT>
__device__ __forceinline__ void plane_fft(double2* buf, const double2* twy, const double2* twz) {
    using G = Geo<LX, LY, LZ>;
    if constexpr (LZ > 1) {
        // z lines: line l = (pr, y), element z at l*ZP + z
        LineFFT<LZ, G::PR * LY, 1, OffMul<G::ZP>, SIGN, NT>::run(buf, twz, OffMul<G::ZP>());
    }
    if constexpr (LY > 1) {
        // y lines: line l = (pr, z), element y at pr*LY*ZP + y*ZP + z
        LineFFT<LY, G::PR * LZ, G::ZP, OffSplit<LZ, LY * G::ZP>, SIGN, NT>::run(buf, twy, OffSplit<LZ, LY * G::ZP>());
    }
}

// The sweep of one problem; bidx scales the batch strides of a (the problem's
// index in a strided batch, 0 when a describes the problem by its own pointers);
// NT threads a CTA (the thread count changes which thread computes what, not
// the arithmetic).
// XTC caps the elements of an x tile: the single-solve kernel comes in the
// x-tile variants kXtc (the autotuner times them per grid; a 48^3 solve ran
// 65 -> 57 us per step with 18-column rather than 36-column tiles, as more
// CTAs share its x passes); the shared batch launches keep 2048 (they fill the
// GPU with several solves).  The tile never changes the arithmetic, and shared
// memory is sized for the largest tile.
constexpr int kXtc[3] = {512, 1024, 2048};

template <int LX, int LY, int LZ, int NT, int XTC>
__device__ __forceinline__ void sweep_body(const SweepArgs& a, long bidx) {
    using G = Geo<LX, LY, LZ, XTC>;
    constexpr int EPT = (G::PT + NT - 1) / NT;   // plane elements per thread
    extern __shared__ double2 sm[];
    double2* twx = sm;
    double2* twy = twx + LX;
    double2* twz = twy + LY;
    double2* buf = twz + LZ;

    for (int m = threadIdx.x; m < LX; m += NT) twx[m] = a.twx[m];
    for (int m = threadIdx.x; m < LY; m += NT) twy[m] = a.twy[m];
    for (int m = threadIdx.x; m < LZ; m += NT) twz[m] = a.twz[m];
    __syncthreads();

    const long M = G::M;
    const double Md = (double)M;
    const double rMd = 1.0 / Md;
    const bool mpow2 = (M & (M - 1)) == 0;   // x / M == x * (1 / M) exactly
    const int nb = gridDim.x;
    const long boff = bidx * a.bstride_batch;   // batch offset of per-problem arrays
    unsigned bar_target = 0;
    unsigned* bar = a.bar + 32 * bidx;
    const int Ns = a.Ns;

    double* hf = a.hf + bidx * a.bstride_hist;
    double* hc = a.hc + bidx * a.bstride_hist;
    double2* Z1 = a.Z1 + boff;
    double2* Z2 = a.Z2 + boff;
    double2* Z3 = a.Z3 + boff;
    double* uf = a.uf + boff;
    double* uc = a.uc + boff;
    const double* L1 = a.L1 + bidx * a.bstride_L;
    const double* L2 = a.L2 + bidx * a.bstride_L;
    // block (0 A, 1 B, 2 C) of a lane at step t
    auto block = [&](int lane, int t) -> int {
        if (!a.eFC) return lane == 0 ? (t < a.LA ? 0 : 1) : (t < a.LB ? 1 : 0);
        if (lane == 0) return t < a.LA ? 0 : (t < a.LA + a.LB ? 1 : 2);
        return t < a.LC ? 2 : (t < a.LC + a.LB ? 1 : 0);
    };
    auto eF = [&](int lane, int t) -> const double* {   // e^{-w ds/2} of the lane's block at step t
        const int blk = block(lane, t);
        return (blk == 0 ? a.eFA : blk == 1 ? a.eFB : a.eFC) + boff;
    };
    auto eH = [&](int lane, int t) -> const double* {
        const int blk = block(lane, t);
        return (blk == 0 ? a.eHA : blk == 1 ? a.eHB : a.eHC) + boff;
    };

    // ---- plane task helpers -------------------------------------------------
    auto load_plane = [&](const double2* Z, long slab0) {
#pragma unroll 4
        for (int k = 0; k < EPT; k++) {
            int p = threadIdx.x + k * NT;
            if (G::PT % NT == 0 || p < G::PT) buf[pidx<G, LZ>(p)] = Z[slab0 + p];
        }
        __syncthreads();
    };
    auto store_plane = [&](double2* Z, long slab0) {
#pragma unroll 4
        for (int k = 0; k < EPT; k++) {
            int p = threadIdx.x + k * NT;
            if (G::PT % NT == 0 || p < G::PT) Z[slab0 + p] = buf[pidx<G, LZ>(p)];
        }
    };

    // initial forward transforms of step 0: Z1 = e^{-w ds/2} q[0], Z2 = e^{-w ds/4} q[0]
    for (int task = blockIdx.x; task < 2 * G::NPT; task += nb) {
        const int role = task / G::NPT;
        const long s0 = (long)(task % G::NPT) * G::PT;
        const double* ef = role == 0 ? eF(0, 0) : eH(0, 0);
        const double* ec = role == 0 ? eF(1, 0) : eH(1, 0);
#pragma unroll 2
        for (int k = 0; k < EPT; k++) {
            int p = threadIdx.x + k * NT;
            if (G::PT % NT == 0 || p < G::PT) {
                long g = s0 + p;
                buf[pidx<G, LZ>(p)] = make_double2(ef[g] * hf[g], ec[g] * hc[g]);
            }
        }
        __syncthreads();
        plane_fft<LX, LY, LZ, -1, NT>(buf, twy, twz);
        store_plane(role == 0 ? Z1 : Z2, s0);
        __syncthreads();
    }
    bar_target += nb;
    if (!grid_barrier(bar, a.err, bar_target)) return;

    for (int t = 0; t < Ns; t++) {
        // ---- x-pass on Z1 (table L1) and Z2 (table L2) ------------------------
        for (int phase = 0; phase < 2; phase++) {
            const int nf = phase == 0 ? 2 : 1;
            for (int task = blockIdx.x; task < G::NXT; task += nb) {
                const long c0 = (long)task * G::XT;
                // load: element (x, c) of field f at buf[f*LX*XT + x*XT + c]
                constexpr int XE = LX * G::XT;
                constexpr int XEPT = (XE + NT - 1) / NT;
                for (int f = 0; f < nf; f++) {
                    const double2* Z = phase == 0 ? (f == 0 ? Z1 : Z2) : Z3;
                    double2* xb = buf + f * XE;
#pragma unroll 2
                    for (int k = 0; k < XEPT; k++) {
                        int e = threadIdx.x + k * NT;
                        if (XE % NT == 0 || e < XE) {
                            int x = e / G::XT, c = e % G::XT;
                            xb[e] = Z[(long)x * G::P + c0 + c];
                        }
                    }
                }
                __syncthreads();
                for (int f = 0; f < nf; f++) {
                    double2* xb = buf + f * XE;
                    LineFFT<LX, G::XT, G::XT, OffMul<1>, -1, NT>::run(xb, twx, OffMul<1>());
                    const double* L = (phase == 0 && f == 0) ? L1 : L2;
#pragma unroll 2
                    for (int k = 0; k < XEPT; k++) {
                        int e = threadIdx.x + k * NT;
                        if (XE % NT == 0 || e < XE) {
                            int x = e / G::XT, c = e % G::XT;
                            double lv = L[(long)x * G::P + c0 + c];
                            double2 v = xb[e];
                            xb[e] = make_double2(v.x * lv, v.y * lv);
                        }
                    }
                    __syncthreads();
                    LineFFT<LX, G::XT, G::XT, OffMul<1>, +1, NT>::run(xb, twx, OffMul<1>());
                }
                for (int f = 0; f < nf; f++) {
                    double2* Z = phase == 0 ? (f == 0 ? Z1 : Z2) : Z3;
                    double2* xb = buf + f * XE;
#pragma unroll 2
                    for (int k = 0; k < XEPT; k++) {
                        int e = threadIdx.x + k * NT;
                        if (XE % NT == 0 || e < XE) {
                            int x = e / G::XT, c = e % G::XT;
                            Z[(long)x * G::P + c0 + c] = xb[e];
                        }
                    }
                }
                __syncthreads();
            }
            bar_target += nb;
            if (!grid_barrier(bar, a.err, bar_target)) return;

            if (phase == 0) {
                // ---- plane: Z1 -> u (full step); Z2 -> qt -> Z3 (second half step)
                for (int task = blockIdx.x; task < 2 * G::NPT; task += nb) {
                    const int role = task / G::NPT;
                    const long s0 = (long)(task % G::NPT) * G::PT;
                    load_plane(role == 0 ? Z1 : Z2, s0);
                    plane_fft<LX, LY, LZ, +1, NT>(buf, twy, twz);
                    if (role == 0) {
                        const double* ef = eF(0, t);
                        const double* ec = eF(1, t);
#pragma unroll 2
                        for (int k = 0; k < EPT; k++) {
                            int p = threadIdx.x + k * NT;
                            if (G::PT % NT == 0 || p < G::PT) {
                                long g = s0 + p;
                                double2 v = buf[pidx<G, LZ>(p)];
                                uf[g] = div_pow2_or_rn(v.x * ef[g], Md, rMd, mpow2);
                                uc[g] = div_pow2_or_rn(v.y * ec[g], Md, rMd, mpow2);
                            }
                        }
                        __syncthreads();
                    } else {
                        const double* hfp = eH(0, t);
                        const double* hcp = eH(1, t);
#pragma unroll 2
                        for (int k = 0; k < EPT; k++) {
                            int p = threadIdx.x + k * NT;
                            if (G::PT % NT == 0 || p < G::PT) {
                                long g = s0 + p;
                                int si = pidx<G, LZ>(p);
                                double2 v = buf[si];
                                double ha = hfp[g], hb = hcp[g];
                                double qtf = div_pow2_or_rn(v.x * ha, Md, rMd, mpow2);
                                double qtc = div_pow2_or_rn(v.y * hb, Md, rMd, mpow2);
                                buf[si] = make_double2(ha * qtf, hb * qtc);
                            }
                        }
                        __syncthreads();
                        plane_fft<LX, LY, LZ, -1, NT>(buf, twy, twz);
                        store_plane(Z3, s0);
                        __syncthreads();
                    }
                }
                bar_target += nb;
                if (!grid_barrier(bar, a.err, bar_target)) return;
            }
        }

        // ---- plane: Z3 -> q[t+1] = (4 qt2 - u)/3; next step's Z1 / Z2 ----------
        const bool next = (t + 1 < Ns);
        for (int task = blockIdx.x; task < 2 * G::NPT; task += nb) {
            const int role = task / G::NPT;
            const long s0 = (long)(task % G::NPT) * G::PT;
            if (!next && role == 1) continue;
            load_plane(Z3, s0);
            plane_fft<LX, LY, LZ, +1, NT>(buf, twy, twz);
            const double* hfp = eH(0, t);
            const double* hcp = eH(1, t);
            const double* nf = next ? (role == 0 ? eF(0, t + 1) : eH(0, t + 1)) : nullptr;
            const double* nc = next ? (role == 0 ? eF(1, t + 1) : eH(1, t + 1)) : nullptr;
            double* of = hf + (long)(t + 1) * M;
            double* oc = hc + (long)(t + 1) * M;
#pragma unroll 2
            for (int k = 0; k < EPT; k++) {
                int p = threadIdx.x + k * NT;
                if (G::PT % NT == 0 || p < G::PT) {
                    long g = s0 + p;
                    int si = pidx<G, LZ>(p);
                    double2 v = buf[si];
                    double qf = div_pow2_or_rn(v.x * hfp[g], Md, rMd, mpow2);
                    double qc = div_pow2_or_rn(v.y * hcp[g], Md, rMd, mpow2);
                    qf = div_rn(4.0 * qf - uf[g], 3.0, 1.0 / 3.0);
                    qc = div_rn(4.0 * qc - uc[g], 3.0, 1.0 / 3.0);
                    if (role == 0) { of[g] = qf; oc[g] = qc; }
                    if (next) buf[si] = make_double2(nf[g] * qf, nc[g] * qc);
                }
            }
            __syncthreads();
            if (next) {
                plane_fft<LX, LY, LZ, -1, NT>(buf, twy, twz);
                store_plane(role == 0 ? Z1 : Z2, s0);
                __syncthreads();
            }
        }
        if (next) {
            bar_target += nb;
            if (!grid_barrier(bar, a.err, bar_target)) return;
        }
    }
}

// a strided batch: problem blockIdx.y at blockIdx.y times the strides of a
template <int LX, int LY, int LZ, int XTC>
__global__ void __launch_bounds__(kNT, 1) sweep_rqm4_kernel(SweepArgs a) {
    sweep_body<LX, LY, LZ, kNT, XTC>(a, blockIdx.y);
}

template <int LX, int LY, int LZ>
auto sweep_kernel_of(int variant) {
    return variant == 0 ? sweep_rqm4_kernel<LX, LY, LZ, kXtc[0]>
         : variant == 1 ? sweep_rqm4_kernel<LX, LY, LZ, kXtc[1]> : sweep_rqm4_kernel<LX, LY, LZ, kXtc[2]>;
}

// a batch of independent problems, problem blockIdx.y described by d[blockIdx.y]
template <int LX, int LY, int LZ>
// (kNTB threads, two CTAs an SM: more solves share the GPU at full width;
// measured on the C5 sample 8.65e9 -> 9.71e9 gridpt*steps/s)
__global__ void __launch_bounds__(kNTB, 2) sweep_rqm4_desc_kernel(const SweepArgs* __restrict__ d) {
    const SweepArgs a = d[blockIdx.y];
    sweep_body<LX, LY, LZ, kNTB, 2048>(a, 0);
}

template <int LX, int LY, int LZ>
size_t smem_bytes() {
    using G = Geo<LX, LY, LZ>;
    return sizeof(double2) * ((size_t)LX + LY + LZ + G::SMEM);
}

template <int LX, int LY, int LZ>
int sweep_prepare_t(int* grid_out) {
    const size_t smem = smem_bytes<LX, LY, LZ>();
    PS_CUDA(cudaFuncSetAttribute(sweep_rqm4_desc_kernel<LX, LY, LZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int dev = 0, sms = 0, occ = 1 << 30, occ_d = 0;
    PS_CUDA(cudaGetDevice(&dev));
    PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int v = 0; v < kSweepVariants; v++) {
        int o = 0;
        PS_CUDA(cudaFuncSetAttribute(sweep_kernel_of<LX, LY, LZ>(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, sweep_kernel_of<LX, LY, LZ>(v), kNT, smem));
        occ = o < occ ? o : occ;   // one grid size for every variant
    }
    PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, sweep_rqm4_desc_kernel<LX, LY, LZ>, kNTB, smem));
    if (occ < 1 || occ_d < 1) throw Error(-2, "sweep kernel does not fit on an SM");
    grid_out[0] = sms * occ;
    grid_out[1] = sms * occ_d;
    twiddle_table(LX); twiddle_table(LY); twiddle_table(LZ);
    return 0;
}

template <int LX, int LY, int LZ>
void sweep_launch_t(SweepArgs a, int grid, int nbatch, cudaStream_t st, int variant) {
    a.twx = twiddle_table(LX);
    a.twy = twiddle_table(LY);
    a.twz = twiddle_table(LZ);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, (unsigned)nbatch, 1);
    cfg.blockDim = dim3(kNT, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes<LX, LY, LZ>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PS_CUDA(cudaLaunchKernelEx(&cfg, sweep_kernel_of<LX, LY, LZ>(variant), a));
}

template <int LX, int LY, int LZ>
void sweep_launch_desc_t(const SweepArgs* d, int per, int n, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)per, (unsigned)n, 1);
    cfg.blockDim = dim3(kNTB, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes<LX, LY, LZ>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PS_CUDA(cudaLaunchKernelEx(&cfg, sweep_rqm4_desc_kernel<LX, LY, LZ>, d));
}

}  // namespace

#define PS_SWEEP_SHAPES(X) \
    X(64, 64, 64) X(48, 48, 48) X(32, 32, 32)

bool sweep_supported(int Lx, int Ly, int Lz) {
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) return true;
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    return false;
}

int sweep_prepare(int Lx, int Ly, int Lz) {
    int grid[2] = {0, 0};
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) { sweep_prepare_t<a, b, c>(grid); return grid[0]; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

void sweep_launch(const SweepArgs& a, int Lx, int Ly, int Lz, int grid, int nbatch, cudaStream_t st, int variant) {
    if (variant < 0 || variant >= kSweepVariants) throw Error(-1, "unknown sweep variant");
#define PS_X(x, y, z) if (Lx == x && Ly == y && Lz == z) { sweep_launch_t<x, y, z>(a, grid, nbatch, st, variant); return; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

int sweep_default_variant(int Lx, int Ly, int Lz) { return Lx == 48 ? 1 : 2; }

int sweep_xtile_columns(int Lx, int Ly, int Lz, int variant) {
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) { \
        return variant == 0 ? Geo<a, b, c, kXtc[0]>::XT : variant == 1 ? Geo<a, b, c, kXtc[1]>::XT : Geo<a, b, c, kXtc[2]>::XT; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

int sweep_desc_prepare(int Lx, int Ly, int Lz) {
    int grid[2] = {0, 0};
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) { sweep_prepare_t<a, b, c>(grid); return grid[1]; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

int sweep_tasks_per_phase(int Lx, int Ly, int Lz) {
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) { using G = Geo<a, b, c>; \
        return 2 * G::NPT > G::NXT ? 2 * G::NPT : G::NXT; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

int sweep_rounds_per_step(int Lx, int Ly, int Lz, int per) {
    if (per < 1) per = 1;
#define PS_X(a, b, c) if (Lx == a && Ly == b && Lz == c) { using G = Geo<a, b, c>; \
        return 2 * ((G::NXT + per - 1) / per) + 2 * ((2 * G::NPT + per - 1) / per); }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

void sweep_launch_desc(const SweepArgs* d, int Lx, int Ly, int Lz, int per, int n, cudaStream_t st) {
#define PS_X(x, y, z) if (Lx == x && Ly == y && Lz == z) { sweep_launch_desc_t<x, y, z>(d, per, n, st); return; }
    PS_SWEEP_SHAPES(PS_X)
#undef PS_X
    throw Error(-2, "no persistent sweep for this grid");
}

}  // namespace ps
