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
// barrier) and a plane phase over the 64 x-slabs (Dy and Dz).
//
// The grid is made of two-CTA thread-block clusters, one CTA per SM.  In the
// plane phase cluster s < 64 owns slab x = s for the whole sweep, and CTA c of
// the pair owns the columns z and the rows y in [32 c, 32 c + 32): it runs
// Dy on its columns, reads its rows from both CTAs' shared memory (DSMEM)
// after a cluster barrier, runs Dz, combines, writes the history and forms
// both next inputs of its rows, runs Dz on them, and after a second cluster
// barrier reads its columns of both from both CTAs and runs Dy.  So every
// line operator of the plane phase runs once, on half the lines a CTA.  The
// CTA keeps its rows' e^{-w ds/4} factors of both blocks in shared memory for
// the whole sweep and prefetches its rows of the full-step result u with a 1D
// bulk copy (cp.async.bulk, no multicast) completed on an mbarrier.
// e^{-w ds/2} is formed as (e^{-w ds/4})^2, and the k-space factors as
// per-axis tables; both agree with the reference's direct exp() evaluations
// to a few ulps.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>

#include "ps_internal.h"
#include "fft_core.cuh"
#include "engine.h"
#include "sweep.h"

namespace cg = cooperative_groups;

namespace ps {

namespace {

constexpr int P64 = 64 * 64;          // points per slab
constexpr int H64 = 32 * 64;          // points of a CTA's half slab (32 rows)
constexpr long M64 = 64L * 64 * 64;
constexpr int NT = 512;
constexpr long long kSpin = 20000000;

// shared memory map (bytes)
//   RA: the two next inputs of the CTA's 32 rows after Dz (row pitch QP),
//       read by both CTAs for Dy; Dz exchange areas
//   RB: Z3 after Dy, the CTA's 32 columns (64 rows of pitch PB), read by both
//       CTAs for Dz, and behind it the CTA's rows of u (bulk copy); the Dy
//       exchange areas of the next inputs (64 lines, slot pitch SP); x-pass
//       exchange areas
//   FC: the x-pass factors of each warp's four columns, loaded in the first
//       x-pass and kept for the sweep (a warp's task is the same every step)
constexpr int QP = 65;                                         // complex
constexpr int PB = 33;
constexpr int SP = 65;
constexpr int OFF_RA = 0;
constexpr int SZ_RA = 2 * 32 * QP * 16;
constexpr int OFF_RB = OFF_RA + SZ_RA;
constexpr int SZ_RB = 64 * SP * 16;
// the rows' e^{-w ds/4} tables, row pitch EHP doubles: a warp reads 4 rows x 8
// consecutive z, and a pitch of 72 (not 64) puts alternate rows on the other
// 16 banks (2 wavefronts a read instead of 4)
constexpr int EHP = 72;
constexpr int OFF_EHA = OFF_RB + SZ_RB;                        // 32 x EHP double
constexpr int OFF_EHB = OFF_EHA + 32 * EHP * 8;
constexpr int OFF_U = OFF_RB + 64 * PB * 16;                   // 2048 double2 behind the Z3 columns
constexpr int XW = 14;                                         // x-pass warps a CTA with a task (2048 tasks)
constexpr int OFF_FC = OFF_EHB + 32 * EHP * 8;                 // XW x 256 double2
constexpr int OFF_TW = OFF_FC + XW * 256 * 16;                 // 64 double2
constexpr int OFF_TAB = OFF_TW + 64 * 16;                      // 6 x 64 double: x,y,z tables for L1 then L2
constexpr int OFF_MBAR = OFF_TAB + 6 * 64 * 8;                 // mbarrier (8 B)
constexpr int OFF_STOP = OFF_MBAR + 8;                         // grid barriers no longer waited (int)
constexpr int SMEM64 = OFF_MBAR + 16;
static_assert(64 * PB * 16 + H64 * 16 <= SZ_RB, "Z3 columns and u fit in RB");
static_assert(16 * 256 * 16 <= SZ_RB, "x-pass scratch fits");
static_assert(OFF_U % 16 == 0 && OFF_FC % 16 == 0 && OFF_MBAR % 8 == 0, "alignment");
static_assert(SMEM64 <= 232448, "shared memory of one CTA");

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
// After a timeout, or once another CTA has raised the error flag, the CTA
// marks itself stopped (*stopped, shared memory, zeroed by the kernel's
// prologue) and no longer waits at later barriers: the sweep runs on to its
// end without waiting, so that the two CTAs of a cluster keep meeting at the
// same cluster barriers, and the host reads the error flag.
__device__ __forceinline__ void grid_sync(unsigned* ctr, int* err, unsigned idx, int* stopped) {
    __syncthreads();
    if (threadIdx.x == 0 && !*stopped) {
        red_add_release(ctr, 1u);
        const unsigned target = idx * gridDim.x;
        long long spins = 0;
        while (ld_acquire(ctr) < target) {
            if ((spins & 63) == 63 && *((volatile int*)err)) { *stopped = 1; break; }
            if (++spins > kSpin) { atomicExch(err, 2); *stopped = 1; break; }
        }
    }
    __syncthreads();
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

// Index of (x, y, z) in the x-pass layout of the work fields Z1, Z2, Z3 and
// of the x-pass factor table: [y][z / 4][x][z % 4].  An x-pass warp (4
// columns z = 4 q .. 4 q + 3 of one y, 8 lanes each, lane t holding
// x = t + 8 j) then reads and writes 512 contiguous bytes per instruction, and
// the plane phase (4 consecutive z of 8 rows y per instruction) 8 runs of 64
// bytes as in natural order.  Column c = 64 y + z starts at (c / 4) 256 + c % 4.
__device__ __forceinline__ long xq(int x, int y, int z) { return ((long)((y << 4) + (z >> 2)) * 64 + x) * 4 + (z & 3); }

// x-pass task of 4 columns c = (y, z) (8 lanes a column, lane t holds the
// stride-8 set x = t + 8 j).
//   Z1 columns: Dx of the full step, then u = e^{-w ds/2} v / M  -> ug
//   Z2 columns: Dx of the half step, qt = e^{-w ds/4} v / M, the second half
//               step's input e^{-w ds/4} qt and its Dx                -> Z3
// Zin and Z3 are in the x-pass layout (xcol: element x = t of column c; + 32 j
// for x = t + 8 j), u in natural order.  fc[32 j]: this lane's slots of the
// warp's factor cache, (e^{-w ds/4} of block A, of block B) of point x = t + 8 j
// (filled by the kernel's prologue); fB, cB: whether lane f and lane c are in
// block B at this step.
__device__ __forceinline__ long xcol(int c, int t) { return (long)(c >> 2) * 256 + (c & 3) + 4 * t; }
__device__ __forceinline__ void xtask(bool full, const double2* Zin, double2* Zout, bool fB, bool cB,
                                      double2* scratch, const double2* fc, int c, int t, const double2* tw,
                                      const double* tab, double rMd) {
    double2 v[8];
    double hf[8], hc[8];
    const long cx = xcol(c, t);   // x = t in the x-pass layout; + 32 j
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = Zin[cx + 32 * j];
    line_op(v, t, scratch, 1, tw, ktab(tab, full ? 0 : 1, 0));
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const double2 e = fc[32 * j];
        hf[j] = fB ? e.y : e.x;
        hc[j] = cB ? e.y : e.x;
    }
    if (full) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            Zout[(long)(t + 8 * j) * P64 + c] =   // u: natural order
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
        for (int j = 0; j < 8; j++) Zout[cx + 32 * j] = v[j];   // Z3: x-pass layout
    }
    __syncwarp();
}

// Address of the same shared-memory offset in CTA `rank` of the cluster, and a
// 16-byte load through it (the CTA's own shared memory or a peer's).
__device__ __forceinline__ unsigned cluster_addr(const void* p, unsigned rank) {
    unsigned d;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(smem_u32(p)), "r"(rank));
    return d;
}
__device__ __forceinline__ double2 ld_cluster(unsigned addr) {
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
    return v;
}

// Indices of the plane phase: cluster rank c (CTA c owns rows and columns
// [32 c, 32 c + 32) of slab blockIdx.x / 2), field f (0: the full-step input,
// 1: the half-step input), row or column r, lane t of the line; the slab's and
// the CTA's rows' offsets; the factor-table entry of (row r, z = t).  Read
// from the special registers where they are used (volatile reads, so the
// compiler keeps none of them live through the x-pass, whose line operators
// use every register).
struct PlaneIx {
    int c, f, r, t, ze0;
    long soff, hoff;
};
__device__ __forceinline__ PlaneIx plane_ix() {
    unsigned tid, cta;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(tid));
    asm volatile("mov.u32 %0, %%ctaid.x;" : "=r"(cta));
    PlaneIx p;
    p.c = (int)(cta & 1);
    p.f = (int)(tid >> 8);
    p.r = (int)((tid >> 3) & 31);
    p.t = (int)(tid & 7);
    p.ze0 = p.r * EHP + p.t;
    p.soff = (long)(cta >> 1) * P64;
    p.hoff = p.soff + (long)p.c * H64;
    return p;
}

// Hardware barrier of every thread of both CTAs of the cluster.  The
// release/acquire pair orders each CTA's shared-memory writes before the
// peer's reads after the barrier, and each CTA's reads of the peer's shared
// memory before the peer's writes after it.
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// The diffusion operator F^-1 exp(-h k^2) F of an orthogonal cell is the
// product Dx Dy Dz of commuting line operators (exp(-h k^2) is the product of
// the per-axis factors), so a contour step needs only two grid-wide phases:
//
//   x-pass  (4096 columns): Dx of the full step on Z1 -> u; Dx of the first
//            half step on Z2, the pointwise e^{-w ds/4} work, Dx of the second
//            half step -> Z3
//   plane   (slab x = s, CTA c of the cluster: columns and rows [32 c, 32 c + 32)):
//            Dy of the second half step on Z3 (columns) | cluster barrier |
//            Dz (rows), q[t+1] = (4 qt2 - u) / 3 -> history; the next step's
//            inputs e^{-w ds/2} q and e^{-w ds/4} q with their Dz (rows) |
//            cluster barrier | Dy (columns) -> Z1, Z2
//
// The divisions by M come after the last inverse transform of each operator,
// where the reference divides.
__global__ void __launch_bounds__(NT, 1) sweep64_kernel(SweepArgs a, const double* __restrict__ tables) {
    extern __shared__ __align__(128) unsigned char smraw[];
    double2* RA = reinterpret_cast<double2*>(smraw + OFF_RA);
    double2* RB = reinterpret_cast<double2*>(smraw + OFF_RB);
    double* ehA = reinterpret_cast<double*>(smraw + OFF_EHA);
    double* ehB = reinterpret_cast<double*>(smraw + OFF_EHB);
    double2* su = reinterpret_cast<double2*>(smraw + OFF_U);
    double2* fcache = reinterpret_cast<double2*>(smraw + OFF_FC);
    double2* tw = reinterpret_cast<double2*>(smraw + OFF_TW);
    double* tab = reinterpret_cast<double*>(smraw + OFF_TAB);
    void* mbar = smraw + OFF_MBAR;
    int* stopped = reinterpret_cast<int*>(smraw + OFF_STOP);

    const int b = blockIdx.x;
    const bool planar = (b >> 1) < 64;          // the same for both CTAs of a cluster
    const int tid = threadIdx.x, t = tid & 7;
    const double rMd = 1.0 / (double)M64;       // M = 2^18: multiplying by 1/M rounds exactly like dividing
    unsigned* ctr = a.bar;
    unsigned bidx = 0;
    unsigned mphase = 0;

    for (int i = tid; i < 64; i += NT) tw[i] = a.twx[((i & 7) * (i >> 3)) & 63];   // [k1][t]
    for (int i = tid; i < 6 * 64; i += NT) tab[i] = tables[i];
    if (planar) {
        const long hoff = plane_ix().hoff;
        for (int i = tid; i < H64; i += NT) {
            const double fa = a.eHA[hoff + i], fb = a.eHB[hoff + i];
            ehA[(i >> 6) * EHP + (i & 63)] = fa;
            ehB[(i >> 6) * EHP + (i & 63)] = fb;
        }
    }
    if (tid == 0) {
        mbar_init(mbar);
        *stopped = 0;
    }

    // x-pass warp index, CTA-fastest so that a phase's tasks spread over all SMs
    const int gwarp = (tid >> 5) * gridDim.x + b;
    const int nwarps = gridDim.x * (NT / 32);
    const int lane = tid & 31, cq = lane >> 3;
    double2* scratch = RB + (tid >> 5) * 256 + cq * 64;
    double2* fc = fcache + (tid >> 5) * 256 + lane;   // this lane's x-pass factors (warps < XW)
    double2* ug = reinterpret_cast<double2*>(a.uf);   // interleaved (u_f, u_c)
    // the factors (e^{-w ds/4} of A, of B) of the warp's x-pass task, x = t + 8 j
    // of its column, for the whole sweep (the task is the same every step)
    if (gwarp < 2 * (P64 / 4) && (tid >> 5) < XW) {
        const int column = (gwarp >= P64 / 4 ? gwarp - P64 / 4 : gwarp) * 4 + cq;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const long i = (long)(t + 8 * j) * P64 + column;
            fc[32 * j] = make_double2(a.eHA[i], a.eHB[i]);
        }
    }
    __syncthreads();

    // lane block at step t: lane f is in A for t < LA, lane c in B for t < LB
    auto sh_f = [&](int st) { return st < a.LA ? ehA : ehB; };          // the rows' tables (shared)
    auto sh_c = [&](int st) { return st < a.LB ? ehB : ehA; };

    auto gsync = [&]() { grid_sync(ctr, a.err, ++bidx, stopped); };

    // The next step's inputs from q[st] (rows, held by the threads of field 0:
    // row r, z = t + 8 j): e^{-w ds/2} q (field 0) and e^{-w ds/4} q (field 1),
    // Dz on the rows, cluster barrier, Dy on the columns -> Z1, Z2
    auto next_inputs = [&](double2 (&v)[8], int st) {
        const PlaneIx ix = plane_ix();
        const int c = ix.c, r = ix.r, f = ix.f, ze0 = ix.ze0;
        const double* nf = sh_f(st);
        const double* nc = sh_c(st);
        double2* Q1 = RA + 32 * QP;
        if (f == 0) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                Q1[r * QP + t + 8 * j] = v[j];
                const double gf = nf[ze0 + 8 * j], gc = nc[ze0 + 8 * j];
                v[j] = make_double2((gf * gf) * v[j].x, (gc * gc) * v[j].y);
            }
        }
        __syncthreads();
        if (f == 1) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const double2 q = Q1[r * QP + t + 8 * j];
                v[j] = make_double2(nf[ze0 + 8 * j] * q.x, nc[ze0 + 8 * j] * q.y);
            }
        }
        double2* row = RA + (f * 32 + r) * QP;
        line_op(v, t, row, 1, tw, ktab(tab, f, 2));
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 8; j++) row[t + 8 * j] = v[j];
        cluster_sync_all();
        // column z = 32 c + r of field f; element y = t + 8 j is row t + 8 (j & 3) of CTA j / 4
        {
            // RA of CTA 0 (rows [0, 32)) and of CTA 1 ([32, 64))
            const double2* p = RA + f * 32 * QP + 32 * c + r + t * QP;
            const unsigned lo = cluster_addr(p, 0), hi = cluster_addr(p, 1);
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = ld_cluster((j < 4 ? lo : hi) + 16 * 8 * QP * (j & 3));
        }
        line_op(v, t, RB + f * 32 + r, SP, tw, ktab(tab, f, 1));
        double2* Zg = (f == 0 ? a.Z1 : a.Z2) + xq((int)(ix.soff >> 12), t, 32 * c + r);
#pragma unroll
        for (int j = 0; j < 8; j++) Zg[8 * j * 16 * 256] = v[j];   // y = t + 8 j
    };

    // Step st = -1 forms the first inputs from the chain heads; every later
    // step is an x-pass and a plane phase.
    for (int st = -1; st < a.Ns; st++) {
        if (st >= 0) {
            // ---- x-pass: Z1 -> u, Z2 -> Z3 (the longer Z2 tasks first) --------
            for (int task = gwarp; task < 2 * (P64 / 4); task += nwarps) {
                // one task a warp, by warps < XW (the launcher's grid ensures it)
                if ((tid >> 5) >= XW || task + nwarps < 2 * (P64 / 4)) { atomicExch(a.err, 4); break; }
                const bool full = task >= P64 / 4;
                const int column = (full ? task - P64 / 4 : task) * 4 + cq;
                xtask(full, full ? a.Z1 : a.Z2, full ? ug : a.Z3, st >= a.LA, st < a.LB, scratch, fc, column, t, tw,
                      tab, rMd);
            }
            gsync();
        }

        // ---- plane: Z3 -> q[st+1] -> next Z1 / Z2 ------------------------------
        const bool next = st + 1 < a.Ns;
        if (planar) {
            double2 v[8];
            const PlaneIx ix = plane_ix();
            const int c = ix.c, r = ix.r, f = ix.f, ze0 = ix.ze0;
            const long soff = ix.soff, hoff = ix.hoff;
            if (st < 0) {
                if (f == 0) {
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const long i = hoff + r * 64 + t + 8 * j;
                        v[j] = make_double2(a.hf[i], a.hc[i]);
                    }
                }
            } else {
                if (f == 0) {
                    // Dy of column z = 32 c + r (y = t + 8 j)
                    const double2* Z3 = a.Z3 + xq((int)(soff >> 12), t, 32 * c + r);
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] = Z3[8 * j * 16 * 256];   // y = t + 8 j
                    double2* col = RB + r;
                    line_op(v, t, col, PB, tw, ktab(tab, 1, 1));
                    if (tid == 0) {
                        // this CTA's rows of u, by a bulk copy once the Z3 loads are
                        // done (they share L2 bandwidth; u is needed after Dz).  The
                        // proxy fence orders earlier generic-proxy accesses (other
                        // CTAs' u stores, this CTA's reads of su) before the copy.
                        asm volatile("fence.proxy.async;" ::: "memory");
                        bulk_load(su, ug + hoff, H64 * 16, mbar);
                    }
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 8; j++) col[(t + 8 * j) * PB] = v[j];
                }
                cluster_sync_all();
                if (f == 0) {
                    // Dz of row y = 32 c + r; element z = t + 8 j is column t + 8 (j & 3) of CTA j / 4
                    {
                        // RB of CTA 0 (columns [0, 32)) and of CTA 1 ([32, 64))
                        const double2* p = RB + (32 * c + r) * PB + t;
                        const unsigned lo = cluster_addr(p, 0), hi = cluster_addr(p, 1);
#pragma unroll
                        for (int j = 0; j < 8; j++) v[j] = ld_cluster((j < 4 ? lo : hi) + 16 * 8 * (j & 3));
                    }
                    line_op(v, t, RA + r * QP, 1, tw, ktab(tab, 1, 2));
                    if (!mbar_wait(mbar, mphase)) atomicExch(a.err, 3);
                    const double* ef = sh_f(st);
                    const double* ec = sh_c(st);
                    double* of = a.hf + (long)(st + 1) * M64 + hoff + r * 64 + t;
                    double* oc = a.hc + (long)(st + 1) * M64 + hoff + r * 64 + t;
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const double hf = ef[ze0 + 8 * j], hc = ec[ze0 + 8 * j];
                        const double2 u = su[r * 64 + t + 8 * j];
                        double qf = (v[j].x * hf) * rMd, qc = (v[j].y * hc) * rMd;
                        qf = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
                        qc = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
                        of[8 * j] = qf;
                        oc[8 * j] = qc;
                        v[j] = make_double2(qf, qc);
                    }
                }
                mphase ^= 1u;
            }
            if (next) next_inputs(v, st + 1);
        }
        if (next) gsync();
    }
    if (planar) cluster_sync_all();   // no peer reads this CTA's shared memory after it exits
}

// Launch configuration: two-CTA clusters, one CTA per SM.  The grid barriers
// need every CTA resident at once; sweep64_prepare sizes the grid by
// cudaOccupancyMaxActiveClusters, and a barrier that waits too long ends the
// sweep with an error instead of spinning on.  (The cooperative launch
// attribute is not combined with the cluster dimension: profilers refuse such
// launches.)
cudaLaunchConfig_t sweep64_config(int grid, cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = SMEM64;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

}  // namespace

bool sweep64_supported(int Lx, int Ly, int Lz) { return Lx == 64 && Ly == 64 && Lz == 64; }

int sweep64_prepare() {
    PS_CUDA(cudaFuncSetAttribute(sweep64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM64));
    int dev = 0, sms = 0;
    PS_CUDA(cudaGetDevice(&dev));
    PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = sweep64_config(sms & ~1, nullptr, attr);
    int nclusters = 0;
    PS_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, sweep64_kernel, &cfg));
    nclusters = std::min(nclusters, sms / 2);
    // 64 clusters own the slabs; every x-pass warp with a task keeps its
    // factors resident, so the 2048 tasks need one warp each among the first
    // XW warps of every CTA
    if (nclusters < 64 || 2 * nclusters * XW < 2 * (P64 / 4)) return 0;
    char line[160];
    std::snprintf(line, sizeof(line), "64^3 sweep: %d clusters of 2 CTAs resident, grid %d\n", nclusters,
                  2 * nclusters);
    tuning_note(line);
    twiddle_table(64);
    return 2 * nclusters;
}

void sweep64_launch(const SweepArgs& a0, const double* tables, int grid, cudaStream_t st) {
    SweepArgs a = a0;
    a.twx = a.twy = a.twz = twiddle_table(64);
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = sweep64_config(grid, st, attr);
    PS_CUDA(cudaLaunchKernelEx(&cfg, sweep64_kernel, a, tables));
}

}  // namespace ps
