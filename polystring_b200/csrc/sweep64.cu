// sweep64.cu -- persistent RQM4 sweep specialised for 64^3 grids.
//
// Built around a register-resident 64 = 8 x 8 four-step FFT:
//
//   a 64-point line is owned by 8 lanes of one warp; lane t holds the
//   stride-8 set x[8 n1 + t].  Pass 1 is an 8-point DFT over n1 and the
//   twiddle W64^(t k1); the 8 x 8 transpose goes through shared memory with
//   a rotation swizzle (element (k1, n2) at slot 8 k1 + ((n2 + k1) & 7), no
//   bank conflicts) and __syncwarp only; pass 2 is an 8-point DFT over n2,
//   after which lane t holds X[t + 8 k2] -- again a stride-8 set with offset
//   t.  So a forward transform, the k-space factor and the inverse transform
//   of one line operator chain in registers, and so do consecutive operators.
//
// For an orthogonal cell exp(-h k^2) is the product of per-axis factors, so
// each split step's F^-1 exp(-h k^2) F is a product Dx Dy Dz of commuting
// line operators.  A contour step is two grid-wide phases with a grid barrier
// after each: an x-pass over the 4096 (y, z) columns (warp-sized tasks, no CTA
// barrier) and a plane phase over the 64 x-slabs (Dy and Dz with one transpose
// through shared memory each way).
//
// Plane work is statically mapped: CTA b < 128 owns slab s = b % 64 in role
// b / 64 for the whole sweep, keeps the slab's e^{-w ds/4} factors of both
// blocks in shared memory, and prefetches the full-step slab u with a 1D
// bulk copy (cp.async.bulk, no multicast) completed on an mbarrier.
// e^{-w ds/2} is formed as (e^{-w ds/4})^2, and the k-space factors as
// per-axis tables; both agree with the reference's direct exp() evaluations
// to a few ulps.
#include "ps_internal.h"
#include "fft_core.cuh"
#include "sweep.h"

namespace ps {

namespace {

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

// Per-axis k factors in shared memory: tab[h * 192 + axis * 64 + k] =
// exp(h' ds k_axis^2) for h = 0 (full step) and 1 (half step), axis 0 x, 1 y, 2 z.
__device__ __forceinline__ const double* ktab(const double* tab, int half, int axis) {
    return tab + half * 192 + axis * 64;
}

// Line operator D = F^-1 diag(L) F of one 64-point line held as the stride-8
// set of lane t (v[j] = element t + 8 j on entry and on exit); `line` is the
// line's 64-slot exchange area (stride es), L the axis factor table.
__device__ __forceinline__ void line_op(double2 (&v)[8], int t, double2* line, int es, const double2* tw,
                                        const double* L) {
    fft64<-1>(v, t, line, es, tw);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const double f = L[t + 8 * k];
        v[k] = make_double2(v[k].x * f, v[k].y * f);
    }
    __syncwarp();
    fft64<+1>(v, t, line, es, tw);
}

// x-pass task of 4 columns c = (y, z) (8 lanes a column, lane t holds the
// stride-8 set x = t + 8 j).
//   Z1 columns: Dx of the full step, then u = e^{-w ds/2} v / M  -> ug
//   Z2 columns: Dx of the half step, qt = e^{-w ds/4} v / M, the second half
//               step's input e^{-w ds/4} qt and its Dx                -> Z3
// eAB: (e^{-w ds/4} of block A, of block B) per point; fB, cB: whether lane f
// and lane c are in block B at this step.  One 16-byte load gives both lanes'
// factors of a point.
__device__ __forceinline__ void xtask(bool full, const double2* Zin, double2* Zout, const double2* eAB,
                                      bool fB, bool cB, double2* scratch, double2* estage, int c, int t,
                                      const double2* tw, const double* tab, double rMd) {
    double2 v[8];
    double hf[8], hc[8];
    // the factors travel to this lane's staging slots (estage[32 j]) by
    // asynchronous copies while the first operator runs: no registers held
#pragma unroll
    for (int j = 0; j < 8; j++) {
        v[j] = Zin[(long)(t + 8 * j) * P64 + c];
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(estage + 32 * j)),
                     "l"(eAB + (long)(t + 8 * j) * P64 + c)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    line_op(v, t, scratch, 1, tw, ktab(tab, full ? 0 : 1, 0));
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const double2 e = estage[32 * j];
        hf[j] = fB ? e.y : e.x;
        hc[j] = cB ? e.y : e.x;
    }
    if (full) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            Zout[(long)(t + 8 * j) * P64 + c] =
                make_double2((v[j].x * (hf[j] * hf[j])) * rMd, (v[j].y * (hc[j] * hc[j])) * rMd);
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const double qf = (v[j].x * hf[j]) * rMd, qc = (v[j].y * hc[j]) * rMd;
            v[j] = make_double2(hf[j] * qf, hc[j] * qc);
        }
        __syncwarp();
        line_op(v, t, scratch, 1, tw, ktab(tab, 1, 0));
#pragma unroll
        for (int j = 0; j < 8; j++) Zout[(long)(t + 8 * j) * P64 + c] = v[j];
    }
    __syncwarp();
}

// Dy then Dz of the slab held in y-line order (thread (r, t): column z = r,
// y = t + 8 j) -> z-line order (row y = r, z = t + 8 j).  One CTA barrier
// for the transpose through the plane buffer; a second one before the
// caller reuses the buffer.
template <class MID>
__device__ __forceinline__ void slab_yz(double2 (&v)[8], double2* plane, int r, int t, const double2* tw,
                                        const double* tab, int half, MID&& mid) {
    double2* col = plane + r;
    line_op(v, t, col, PITCH, tw, ktab(tab, half, 1));
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; j++) col[(t + 8 * j) * PITCH] = v[j];
    __syncthreads();
    mid();   // every thread's loads before the operator are done here
    double2* row = plane + r * PITCH;
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = row[8 * j + t];
    line_op(v, t, row, 1, tw, ktab(tab, half, 2));
    __syncthreads();
}

// Dz then Dy of the slab held in z-line order -> y-line order.
__device__ __forceinline__ void slab_zy(double2 (&v)[8], double2* plane, int r, int t, const double2* tw,
                                        const double* tab, int half) {
    double2* row = plane + r * PITCH;
    line_op(v, t, row, 1, tw, ktab(tab, half, 2));
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; j++) row[t + 8 * j] = v[j];
    __syncthreads();
    double2* col = plane + r;
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = col[(8 * j + t) * PITCH];
    line_op(v, t, col, PITCH, tw, ktab(tab, half, 1));
    __syncthreads();
}

// The diffusion operator F^-1 exp(-h k^2) F of an orthogonal cell is the
// product Dx Dy Dz of commuting line operators (exp(-h k^2) is the product of
// the per-axis factors), so a contour step needs only two grid-wide phases:
//
//   x-pass  (4096 columns): Dx of the full step on Z1 -> u; Dx of the first
//            half step on Z2, the pointwise e^{-w ds/4} work, Dx of the second
//            half step -> Z3
//   plane   (slab x = s): Dy Dz of the second half step on Z3 -> qt2,
//            q[t+1] = (4 qt2 - u) / 3 -> history; the next step's inputs
//            e^{-w ds/2} q (role 0) and e^{-w ds/4} q (role 1) with their
//            Dz Dy -> Z1, Z2
//
// The divisions by M come after the last inverse transform of each operator,
// where the reference divides.
__global__ void __launch_bounds__(NT, 1) sweep64_kernel(SweepArgs a, const double* __restrict__ tables) {
    extern __shared__ __align__(128) unsigned char smraw[];
    double2* plane = reinterpret_cast<double2*>(smraw + OFF_PLANE);
    double* ehA = reinterpret_cast<double*>(smraw + OFF_EHA);
    double* ehB = reinterpret_cast<double*>(smraw + OFF_EHB);
    double2* su = reinterpret_cast<double2*>(smraw + OFF_U);
    double2* tw = reinterpret_cast<double2*>(smraw + OFF_TW);
    double* tab = reinterpret_cast<double*>(smraw + OFF_TAB);
    void* mbar = smraw + OFF_MBAR;

    const int tid = threadIdx.x, t = tid & 7, r = tid >> 3;
    const int b = blockIdx.x;
    const bool planar = b < 128;
    const int slab = b & 63, role = b >> 6;
    const long soff = (long)slab * P64;
    const double rMd = 1.0 / (double)M64;   // M = 2^18: multiplying by 1/M rounds exactly like dividing
    unsigned* ctr = a.bar;
    unsigned bidx = 0;
    unsigned mphase = 0;

    for (int i = tid; i < 64; i += NT) tw[i] = a.twx[((i & 7) * (i >> 3)) & 63];   // [k1][t]
    for (int i = tid; i < 6 * 64; i += NT) tab[i] = tables[i];
    if (planar) {
        for (int i = tid; i < P64; i += NT) {
            const double fa = a.eHA[soff + i], fb = a.eHB[soff + i];
            ehA[(i >> 6) * EHP + (i & 63)] = fa;
            ehB[(i >> 6) * EHP + (i & 63)] = fb;
            if (role == 0) a.eHAB[soff + i] = make_double2(fa, fb);   // for the x-pass (after the first grid barrier)
        }
    }
    if (tid == 0) mbar_init(mbar);
    __syncthreads();

    // x-pass warp index, CTA-fastest so that a phase's tasks spread over all SMs
    const int gwarp = (tid >> 5) * gridDim.x + b;
    const int nwarps = gridDim.x * (NT / 32);
    const int lane = tid & 31, cq = lane >> 3;
    double2* scratch = plane + (tid >> 5) * 256 + cq * 64;
    double2* estage = su + (tid >> 5) * 256 + lane;   // x-pass factor staging (su is idle then)
    double2* ug = reinterpret_cast<double2*>(a.uf);   // interleaved (u_f, u_c)

    // lane block at step t: lane f is in A for t < LA, lane c in B for t < LB
    auto sh_f = [&](int st) { return st < a.LA ? ehA : ehB; };          // slab tables (shared)
    auto sh_c = [&](int st) { return st < a.LB ? ehB : ehA; };

    const int zb = r * 64 + t;   // slab index of (y = r, z = t); + 8 j of z
    const int zbe = r * EHP + t; // the same point in the factor tables

    // next step's input of this CTA's role from q (z-line order), its Dz Dy,
    // stored as Z1 (role 0) or Z2 (role 1)
    auto next_inputs = [&](double2 (&v)[8], int st) {
        const double* nf = sh_f(st);
        const double* nc = sh_c(st);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int ze = zbe + 8 * j;
            double gf = nf[ze], gc = nc[ze];
            if (role == 0) { gf *= gf; gc *= gc; }
            v[j] = make_double2(gf * v[j].x, gc * v[j].y);
        }
        slab_zy(v, plane, r, t, tw, tab, role);
        double2* Zg = (role == 0 ? a.Z1 : a.Z2) + soff;
#pragma unroll
        for (int j = 0; j < 8; j++) Zg[(t + 8 * j) * 64 + r] = v[j];
    };

    // ---- step 0 inputs --------------------------------------------------------
    if (planar) {
        double2 v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = make_double2(a.hf[soff + zb + 8 * j], a.hc[soff + zb + 8 * j]);
        next_inputs(v, 0);
    }
    if (!grid_sync(ctr, a.err, ++bidx)) return;

    for (int st = 0; st < a.Ns; st++) {
        // ---- x-pass: Z1 -> u, Z2 -> Z3 (the longer Z2 tasks first) ------------
        for (int task = gwarp; task < 2 * (P64 / 4); task += nwarps) {
            const bool full = task >= P64 / 4;
            const int c = (full ? task - P64 / 4 : task) * 4 + cq;
            xtask(full, full ? a.Z1 : a.Z2, full ? ug : a.Z3, a.eHAB, st >= a.LA, st < a.LB, scratch, estage, c, t,
                  tw, tab, rMd);
        }
        if (!grid_sync(ctr, a.err, ++bidx)) return;

        // ---- plane: Z3 -> q[st+1] -> next Z1 / Z2 ------------------------------
        const bool next = st + 1 < a.Ns;
        if (planar && (role == 0 || next)) {
            const double* ef = sh_f(st);
            const double* ec = sh_c(st);
            double2 v[8];
            // Z3 in y-line order (column z = r, y = t + 8 j)
            const double2* Z3 = a.Z3 + soff;
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = Z3[(8 * j + t) * 64 + r];
            // u's bulk copy starts once the Z3 loads are done (they share L2
            // bandwidth; u is needed only after Dy Dz)
            slab_yz(v, plane, r, t, tw, tab, 1, [&] {
                if (tid == 0) {
                    // order earlier generic-proxy accesses (other CTAs' u stores,
                    // this CTA's reads and staging writes of su) before the
                    // async-proxy bulk copy
                    asm volatile("fence.proxy.async;" ::: "memory");
                    bulk_load(su, ug + soff, P64 * 16, mbar);
                }
            });
            if (!mbar_wait(mbar, mphase)) { atomicExch(a.err, 3); }
            mphase ^= 1u;
            double* of = a.hf + (long)(st + 1) * M64 + soff;
            double* oc = a.hc + (long)(st + 1) * M64 + soff;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int zi = zb + 8 * j, ze = zbe + 8 * j;
                const double hf = ef[ze], hc = ec[ze];
                const double2 u = su[zi];
                double qf = (v[j].x * hf) * rMd, qc = (v[j].y * hc) * rMd;
                qf = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
                qc = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
                if (role == 0) of[zi] = qf;
                if (role == 1 || !next) oc[zi] = qc;
                v[j] = make_double2(qf, qc);
            }
            if (next) next_inputs(v, st + 1);
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
