// sweep64.cu -- persistent RQM4 sweep specialised for 64^3 grids.
//
// Same phase structure as sweep.cu (x-pass | plane | x-pass | plane per
// contour step, grid barriers in between), built around a register-resident
// 64 = 8 x 8 four-step FFT:
//
//   a 64-point line is owned by 8 lanes of one warp; lane t holds the
//   stride-8 set x[8 n1 + t].  Pass 1 is an 8-point DFT over n1 and the
//   twiddle W64^(t k1); the 8 x 8 transpose goes through shared memory with
//   a rotation swizzle (element (k1, n2) at slot 8 k1 + ((n2 + k1) & 7), no
//   bank conflicts) and __syncwarp only; pass 2 is an 8-point DFT over n2,
//   after which lane t holds X[t + 8 k2] -- again a stride-8 set with offset
//   t.  So an inverse transform, elementwise work and the next forward
//   transform chain in registers with no shared-memory round trip.
//
// A 2D (y, z) plane FFT is one sweep over the 64 rows (z lines) and one over
// the 64 columns (y lines) with a single CTA barrier between them.  x-pass
// tasks are warp-sized (4 columns) and need no CTA barrier at all.
//
// Plane work is statically mapped: CTA b < 128 owns slab s = b % 64 in role
// b / 64 for the whole sweep, keeps the slab's e^{-w ds/4} factors of both
// blocks in shared memory, and prefetches the full-step slab u with a 1D
// bulk copy (cp.async.bulk, no multicast) completed on an mbarrier.
// e^{-w ds/2} is formed as (e^{-w ds/4})^2, and the k-space factors as
// products of per-axis tables; both agree with the reference's direct exp()
// evaluations to a few ulps.
#include "ps_internal.h"
#include "fft_core.cuh"
#include "sweep.h"

namespace ps {

namespace {

constexpr int N64 = 64;
constexpr int P64 = 64 * 64;          // points per slab
constexpr long M64 = 64L * 64 * 64;
constexpr int NT = 512;
constexpr int PITCH = 65;             // smem row pitch of the plane (complex)
constexpr long long kSpin = 20000000;

// shared memory map (bytes)
constexpr int OFF_PLANE = 0;                                   // 64 x 65 double2 (also x-pass scratch)
constexpr int SZ_PLANE = 64 * PITCH * 16;
// the slab's e^{-w ds/4} tables, row pitch EHP doubles: a warp reads 4 rows x 8
// consecutive z, and a pitch of 72 (not 64) puts alternate rows on the other
// 16 banks (2 wavefronts a read instead of 4)
constexpr int EHP = 72;
constexpr int OFF_EHA = OFF_PLANE + SZ_PLANE;                  // 64 x EHP double
constexpr int OFF_EHB = OFF_EHA + 64 * EHP * 8;
constexpr int OFF_U = OFF_EHB + 64 * EHP * 8;                  // 4096 double2 (16-byte aligned)
constexpr int OFF_TW = OFF_U + P64 * 16;                       // 64 double2
constexpr int OFF_TAB = OFF_TW + 64 * 16;                      // 6 x 64 double: x,y,z tables for L1 then L2
constexpr int OFF_MBAR = OFF_TAB + 6 * 64 * 8;                 // mbarrier (8 B)
constexpr int SMEM64 = OFF_MBAR + 16;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_add_release(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Counter grid barrier: every CTA adds one with release semantics and polls
// the counter (acquire) until all CTAs of barrier `idx` have arrived, with a
// bounded spin.  The counter is zeroed before each launch.  The CTA barrier
// before the arrival orders the CTA's writes before thread 0's release (PTX
// memory model: bar.sync then a release at gpu scope is cumulative); the
// acquire load and the CTA barrier after it order the CTA's later reads.
// Compared with a last-arriver flag, the arrival needs no round trip.
__device__ __forceinline__ bool grid_sync(unsigned* ctr, int* err, unsigned idx) {
    __syncthreads();
    __shared__ int stop;
    if (threadIdx.x == 0) {
        int s = 0;
        red_add_release(ctr, 1u);
        const unsigned target = idx * gridDim.x;
        long long spins = 0;
        while (ld_acquire(ctr) < target) {
            if ((spins & 63) == 63 && *((volatile int*)err)) { s = 1; break; }
            if (++spins > kSpin) { atomicExch(err, 2); s = 1; break; }
        }
        stop = s;
    }
    __syncthreads();
    return stop == 0;
}

// ---- mbarrier + bulk copy (global -> shared) -----------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(void* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, void* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bounded wait on the mbarrier phase; returns false on timeout
__device__ __forceinline__ bool mbar_wait(void* bar, unsigned parity) {
    unsigned ok = 0;
    long long spins = 0;
    while (!ok) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (++spins > kSpin) return false;
    }
    return true;
}

// ---- 64-point four-step FFT, 8 lanes per line ----------------------------
// tw8[k1 * 8 + t] = W64^(t k1): lanes t = 0..7 read consecutive entries
template <int SIGN>
__device__ __forceinline__ void pass1(double2 (&v)[8], int t, const double2* tw8) {
    Dft<8, SIGN>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < 8; k1++) {
        double2 w = tw8[k1 * 8 + t];
        if (SIGN > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
}
// v[k1] of lane t -> slot 8 k1 + ((t + k1) & 7) of the line
__device__ __forceinline__ void xstore(double2* line, int es, int t, const double2 (&v)[8]) {
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) line[(8 * k1 + ((t + k1) & 7)) * es] = v[k1];
}
// lane t gathers element (k1 = t, n2) from slot 8 t + ((n2 + t) & 7)
__device__ __forceinline__ void xload(const double2* line, int es, int t, double2 (&v)[8]) {
#pragma unroll
    for (int n2 = 0; n2 < 8; n2++) v[n2] = line[(8 * t + ((n2 + t) & 7)) * es];
}
// full transform: on entry lane t holds x[8 n1 + t] in v[n1]; on exit
// X[t + 8 k2] in v[k2].  `line` is the 64-slot exchange area (stride es).
template <int SIGN>
__device__ __forceinline__ void fft64(double2 (&v)[8], int t, double2* line, int es, const double2* tw) {
    pass1<SIGN>(v, t, tw);
    __syncwarp();
    xstore(line, es, t, v);
    __syncwarp();
    xload(line, es, t, v);
    Dft<8, SIGN>::run(v);
}

struct S64 {
    double2* plane;
    const double* ehA;
    const double* ehB;
    double2* u;
    const double2* tw;
    const double* tab;   // [0..63] x full, [64..] y full, [128..] z full, [192..] x half, ...
};

// forward plane FFT: v holds row y = r, z = 8 n1 + t (the z-line input set).
// Writes the spectrum of the slab to global Zg (natural order).
__device__ __forceinline__ void plane_forward(double2 (&v)[8], const S64& s, double2* Zg) {
    const int tid = threadIdx.x, t = tid & 7, r = tid >> 3;
    double2* row = s.plane + r * PITCH;
    fft64<-1>(v, t, row, 1, s.tw);
    __syncwarp();
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) row[t + 8 * k2] = v[k2];
    __syncthreads();
    // y lines: column c = r
    double2* col = s.plane + r;
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) v[n1] = col[(8 * n1 + t) * PITCH];
    fft64<-1>(v, t, col, PITCH, s.tw);
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) Zg[(t + 8 * k2) * 64 + r] = v[k2];
    __syncthreads();   // plane buffer is reused by the caller
}

// inverse plane FFT of the slab spectrum Zg (global, natural order); on exit
// v holds row y = r, z = t + 8 k2 of the (unnormalised) inverse.
__device__ __forceinline__ void plane_inverse(double2 (&v)[8], const S64& s, const double2* Zg) {
    const int tid = threadIdx.x, t = tid & 7, r = tid >> 3;
    double2* col = s.plane + r;
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) v[n1] = Zg[(8 * n1 + t) * 64 + r];
    fft64<+1>(v, t, col, PITCH, s.tw);
    __syncwarp();
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) col[(t + 8 * k2) * PITCH] = v[k2];
    __syncthreads();
    double2* row = s.plane + r * PITCH;
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) v[n1] = row[8 * n1 + t];
    fft64<+1>(v, t, row, 1, s.tw);
    __syncthreads();   // plane buffer is reused by the caller
}

// x-pass of one field over all columns; warp task = 4 columns.
// half = 0: k table of the full step, 1: of the half step
__device__ __forceinline__ void xpass(double2* Z, int half, const S64& s, int gwarp, int nwarps) {
    const int lane = threadIdx.x & 31, t = lane & 7, cq = lane >> 3;
    double2* scratch = s.plane + (threadIdx.x >> 5) * 256 + cq * 64;
    const double* tx = s.tab + half * 192;
    const double* ty = tx + 64;
    const double* tz = tx + 128;
    for (int task = gwarp; task < P64 / 4; task += nwarps) {
        const int c = task * 4 + cq;          // column = (ky, kz) = (c / 64, c % 64)
        double2 v[8];
#pragma unroll
        for (int n1 = 0; n1 < 8; n1++) v[n1] = Z[(long)(8 * n1 + t) * P64 + c];
        fft64<-1>(v, t, scratch, 1, s.tw);
        const double tyz = ty[c >> 6] * tz[c & 63];
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) {
            double lv = tx[t + 8 * k2] * tyz;
            v[k2] = make_double2(v[k2].x * lv, v[k2].y * lv);
        }
        __syncwarp();
        fft64<+1>(v, t, scratch, 1, s.tw);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) Z[(long)(t + 8 * k2) * P64 + c] = v[k2];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(NT, 1) sweep64_kernel(SweepArgs a, const double* __restrict__ tables) {
    extern __shared__ __align__(128) unsigned char smraw[];
    S64 s;
    s.plane = reinterpret_cast<double2*>(smraw + OFF_PLANE);
    double* ehA = reinterpret_cast<double*>(smraw + OFF_EHA);
    double* ehB = reinterpret_cast<double*>(smraw + OFF_EHB);
    s.ehA = ehA;
    s.ehB = ehB;
    s.u = reinterpret_cast<double2*>(smraw + OFF_U);
    double2* tw = reinterpret_cast<double2*>(smraw + OFF_TW);
    double* tab = reinterpret_cast<double*>(smraw + OFF_TAB);
    void* mbar = smraw + OFF_MBAR;
    s.tw = tw;
    s.tab = tab;

    const int tid = threadIdx.x, t = tid & 7, r = tid >> 3;
    const int b = blockIdx.x;
    const bool planar = b < 128;
    const int slab = b & 63, role = b >> 6;
    const long soff = (long)slab * P64;
    const double Md = (double)M64;
    const double rMd = 1.0 / Md;   // M = 2^18: multiplying by 1/M rounds exactly like dividing
    unsigned* ctr = a.bar;
    unsigned bidx = 0;
    unsigned mphase = 0;

    for (int i = tid; i < 64; i += NT) tw[i] = a.twx[((i & 7) * (i >> 3)) & 63];   // [k1][t]
    for (int i = tid; i < 6 * 64; i += NT) tab[i] = tables[i];
    if (planar) {
        for (int i = tid; i < P64; i += NT) {
            ehA[(i >> 6) * EHP + (i & 63)] = a.eHA[soff + i];
            ehB[(i >> 6) * EHP + (i & 63)] = a.eHB[soff + i];
        }
    }
    if (tid == 0) mbar_init(mbar);
    __syncthreads();

    // x-pass warp index, CTA-fastest so that a phase's tasks spread over all SMs
    const int gwarp = (tid >> 5) * gridDim.x + b;
    const int nwarps = gridDim.x * (NT / 32);
    double2* Z1 = a.Z1;
    double2* Z2 = a.Z2;
    double2* Z3 = a.Z3;
    double2* ug = reinterpret_cast<double2*>(a.uf);   // interleaved (u_f, u_c)

    // lane block at step t: lane f is in A for t < LA, lane c in B for t < LB
    auto eh_f = [&](int st) { return st < a.LA ? s.ehA : s.ehB; };
    auto eh_c = [&](int st) { return st < a.LB ? s.ehB : s.ehA; };
    const int zb = r * 64 + t;   // slab index of (y = r, z = t) ; + 8 k of z
    const int zbe = r * EHP + t; // the same point in the factor tables

    // ---- step 0 forward transforms ----------------------------------------
    if (planar) {
        const double* ef = eh_f(0);
        const double* ec = eh_c(0);
        double2 v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int zi = zb + 8 * k, ze = zbe + 8 * k;
            double hf = ef[ze], hc = ec[ze];
            if (role == 0) { hf *= hf; hc *= hc; }
            v[k] = make_double2(hf * a.hf[soff + zi], hc * a.hc[soff + zi]);
        }
        plane_forward(v, s, (role == 0 ? Z1 : Z2) + soff);
    }
    if (!grid_sync(ctr, a.err, ++bidx)) return;

    for (int st = 0; st < a.Ns; st++) {
        // ---- x-pass on Z1 (full step) and Z2 (half step) ---------------------
        {
            const int half = gwarp & 1;
            xpass(half ? Z2 : Z1, half, s, gwarp >> 1, nwarps >> 1);
        }
        if (!grid_sync(ctr, a.err, ++bidx)) return;

        // ---- plane: Z1 -> u ; Z2 -> qt -> Z3 ---------------------------------
        if (planar) {
            const double* ef = eh_f(st);
            const double* ec = eh_c(st);
            double2 v[8];
            plane_inverse(v, s, (role == 0 ? Z1 : Z2) + soff);
            if (role == 0) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int zi = zb + 8 * k, ze = zbe + 8 * k;
                    double hf = ef[ze], hc = ec[ze];
                    ug[soff + zi] = make_double2((v[k].x * (hf * hf)) * rMd, (v[k].y * (hc * hc)) * rMd);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int ze = zbe + 8 * k;
                    double hf = ef[ze], hc = ec[ze];
                    double qf = (v[k].x * hf) * rMd, qc = (v[k].y * hc) * rMd;
                    v[k] = make_double2(hf * qf, hc * qc);
                }
                plane_forward(v, s, Z3 + soff);
            }
        }
        if (!grid_sync(ctr, a.err, ++bidx)) return;

        // ---- x-pass on Z3 (half step) -----------------------------------------
        xpass(Z3, 1, s, gwarp, nwarps);
        if (!grid_sync(ctr, a.err, ++bidx)) return;

        // ---- plane: Z3 -> q[st+1] = (4 qt2 - u) / 3 -> next Z1 / Z2 ------------
        const bool next = st + 1 < a.Ns;
        if (planar && (role == 0 || next)) {
            if (tid == 0) {
                // order earlier generic-proxy accesses (other CTAs' u stores,
                // this CTA's reads of s.u) before the async-proxy bulk copy
                asm volatile("fence.proxy.async;" ::: "memory");
                bulk_load(s.u, ug + soff, P64 * 16, mbar);
            }
            const double* ef = eh_f(st);
            const double* ec = eh_c(st);
            double2 v[8];
            plane_inverse(v, s, Z3 + soff);
            if (!mbar_wait(mbar, mphase)) { atomicExch(a.err, 3); }
            mphase ^= 1u;
            const double* nf = next ? eh_f(st + 1) : ef;
            const double* nc = next ? eh_c(st + 1) : ec;
            double* of = a.hf + (long)(st + 1) * M64 + soff;
            double* oc = a.hc + (long)(st + 1) * M64 + soff;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int zi = zb + 8 * k, ze = zbe + 8 * k;
                double hf = ef[ze], hc = ec[ze];
                double2 u = s.u[zi];
                double qf = (v[k].x * hf) * rMd, qc = (v[k].y * hc) * rMd;
                qf = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
                qc = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
                if (role == 0) of[zi] = qf;
                if (role == 1 || !next) oc[zi] = qc;
                double gf = nf[ze], gc = nc[ze];
                if (role == 0) { gf *= gf; gc *= gc; }
                v[k] = make_double2(gf * qf, gc * qc);
            }
            if (next) plane_forward(v, s, (role == 0 ? Z1 : Z2) + soff);
            __syncthreads();
        }
        if (next) {
            if (!grid_sync(ctr, a.err, ++bidx)) return;
        }
    }
}

}  // namespace

bool sweep64_supported(int Lx, int Ly, int Lz) { return Lx == 64 && Ly == 64 && Lz == 64; }

int sweep64_prepare() {
    PS_CUDA(cudaFuncSetAttribute(sweep64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM64));
    int dev = 0, sms = 0, occ = 0;
    PS_CUDA(cudaGetDevice(&dev));
    PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sweep64_kernel, NT, SMEM64));
    if (occ < 1 || sms < 128) throw Error(-2, "64^3 sweep needs 128 resident CTAs");
    twiddle_table(64);
    return sms;   // one CTA per SM
}

void sweep64_launch(const SweepArgs& a0, const double* tables, int grid, cudaStream_t st) {
    SweepArgs a = a0;
    a.twx = a.twy = a.twz = twiddle_table(64);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = SMEM64;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PS_CUDA(cudaLaunchKernelEx(&cfg, sweep64_kernel, a, tables));
}

}  // namespace ps
