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
// Dy on its columns of the half-step field Z3 and of the full-step field W,
// reads its rows of both from both CTAs' shared memory (DSMEM) after a
// cluster barrier, runs Dz on Z3, combines, writes the history and forms both
// next inputs of its rows, runs Dz on them (W is stored then; its Dx and Dy
// follow in the next x-pass and plane phase), and after a second cluster
// barrier reads its columns of the half-step input from both CTAs and runs
// Dy.  So every line operator of the plane phase runs once, on half a slab a
// CTA.  The CTA keeps its rows' e^{-w ds/4} factors of both blocks in shared
// memory for the whole sweep, and so does each x-pass warp for its columns.
// e^{-w ds/2} is formed as (e^{-w ds/4})^2, and the k-space factors as
// per-axis tables; both agree with the reference's direct exp() evaluations
// to a few ulps.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "ps_internal.h"
#include "fft_core.cuh"
#include "engine.h"
#include "sweep.h"

namespace ps {

namespace {

constexpr int P64 = 64 * 64;          // points per slab
constexpr int H64 = 32 * 64;          // points of a CTA's half slab (32 rows)
constexpr long M64 = 64L * 64 * 64;
constexpr int NT = 512;
constexpr long long kSpin = 20000000;

// shared memory map (bytes)
//   RA: 64 rows of pitch QP: rows 0-31 the Dz exchange areas of Z3 and of the
//       full-step input; rows 32-63 the Dy exchange areas of W's columns, then
//       q and the half-step input, whose rows after Dz both CTAs read for Dy
//   RB: Z3 after Dy, the CTA's 32 columns (64 rows of pitch PB), and behind
//       it the full-step result after Dy, the CTA's 32 columns (64 rows of 32,
//       swizzled), both read by both CTAs for the rows; the Dy exchange areas
//       of the half-step input (32 lines, slot pitch SP); x-pass exchange areas
//   EH: the CTA's 32 rows of e^{-w ds/4} of each block (A, B and, for a
//       linear ABC triblock, C), for the whole sweep
//   FC: the factor pair (lane f's block, lane c's block) of the four columns
//       of each warp with a half-step x-pass task; a warp's task is the same
//       every step, so the pairs are loaded again only when a lane changes
//       block
constexpr int QP = 65;                                         // complex
constexpr int PB = 33;
constexpr int SP = 65;
constexpr int UC = 64 * PB;                                    // RB offset of the full-step columns
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
constexpr int XW = 14;                                         // x-pass warps a CTA with a task (2048 tasks)
constexpr int XH = 7;                                          // of them with a half-step task (1024 tasks)
constexpr int OFF_FC = OFF_EHB + 32 * EHP * 8;                 // XH x 256 double2
constexpr int OFF_TW = OFF_FC + XH * 256 * 16;                 // 64 double2
constexpr int OFF_TAB = OFF_TW + 64 * 16;                      // 6 x 64 double: x,y,z tables for L1 then L2
constexpr int OFF_STOP = OFF_TAB + 6 * 64 * 8;                 // grid barriers no longer waited (int)
constexpr int SMEM64 = OFF_STOP + 16;
// block C's rows, at the end: only the launches of linear ABC triblocks ask
// for the extra shared memory (the diblocks' launches keep it as L1 cache)
constexpr int OFF_EHC = SMEM64;
constexpr int SMEM64_ABC = OFF_EHC + 32 * EHP * 8;
static_assert((UC + H64) * 16 <= SZ_RB, "Z3 and full-step columns fit in RB");
static_assert(16 * 256 * 16 <= SZ_RB && (31 + 63 * SP + 1) * 16 <= SZ_RB, "exchange areas fit in RB");
static_assert(OFF_FC % 16 == 0 && OFF_STOP % 8 == 0, "alignment");
static_assert(SMEM64_ABC <= 232448, "shared memory of one CTA");

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

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
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
// stride-8 set x = t + 8 j), fields in the x-pass layout (xcol: element x = t
// of column c; + 32 j for x = t + 8 j).
//   full step (Z1, in place): Dx of the full step (Dz came before, Dy and the
//               factor e^{-w ds/2} / M follow in the plane phase)
//   half step (Z2 -> Z3): Dx of the half step, qt = e^{-w ds/4} v / M, the
//               second half step's input e^{-w ds/4} qt and its Dx
// fc[32 j]: this lane's slots of the warp's factor cache, a pair of e^{-w ds/4}
// at point x = t + 8 j: for a diblock (block A, block B) for the whole sweep,
// fB and cB telling whether lane f and lane c are in block B at this step; for
// a triblock (lane f's block, lane c's block), loaded again by xfill when a
// lane changes block, fB = false and cB = true.
__device__ __forceinline__ long xcol(int c, int t) { return (long)(c >> 2) * 256 + (c & 3) + 4 * t; }
__device__ __forceinline__ void xtask_full(double2* Z, double2* scratch, int c, int t, const double2* tw,
                                           const double* tab) {
    double2 v[8];
    const long cx = xcol(c, t);
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = Z[cx + 32 * j];
    line_op(v, t, scratch, 1, tw, ktab(tab, 0, 0));
#pragma unroll
    for (int j = 0; j < 8; j++) Z[cx + 32 * j] = v[j];
    __syncwarp();
}
__device__ __forceinline__ void xfill(const double* ef, const double* ec, double2* fc, int c, int t) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const long i = (long)(t + 8 * j) * P64 + c;   // natural order
        fc[32 * j] = make_double2(ef[i], ec[i]);
    }
}
__device__ __forceinline__ void xtask_half(const double2* Zin, double2* Zout, bool fB, bool cB, double2* scratch,
                                           const double2* fc, int c, int t, const double2* tw, const double* tab,
                                           double rMd) {
    double2 v[8];
    const long cx = xcol(c, t);
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = Zin[cx + 32 * j];
    line_op(v, t, scratch, 1, tw, ktab(tab, 1, 0));
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const double2 e = fc[32 * j];
        const double hf = fB ? e.y : e.x, hc = cB ? e.y : e.x;
        const double qf = (v[j].x * hf) * rMd, qc = (v[j].y * hc) * rMd;
        v[j] = make_double2(hf * qf, hc * qc);
    }
    __syncwarp();
    line_op(v, t, scratch, 1, tw, ktab(tab, 1, 0));
#pragma unroll
    for (int j = 0; j < 8; j++) Zout[cx + 32 * j] = v[j];
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
//   x-pass  (4096 columns): Dx of the full step on W (in place); Dx of the
//            first half step on Z2, the pointwise e^{-w ds/4} work, Dx of the
//            second half step -> Z3
//   plane   (slab x = s, CTA c of the cluster: columns and rows [32 c, 32 c + 32)):
//            Dy of the second half step on Z3 and Dy of the full step on W
//            (columns) | cluster barrier | Dz of Z3 (rows), u = e^{-w ds/2} W / M,
//            q[t+1] = (4 qt2 - u) / 3 -> history; the next step's inputs
//            e^{-w ds/2} q with its Dz -> W, and e^{-w ds/4} q with its Dz
//            (rows) | cluster barrier | Dy (columns) -> Z2
//
// so the full-step field gets Dz at the end of one plane phase, Dx in the
// x-pass and Dy at the start of the next plane phase (whose first operators
// have half the lines of its last ones).  The divisions by M come after the
// last inverse transform of each operator, where the reference divides.
template <bool TRI>   // TRI: a linear ABC triblock (three factor sets)
__global__ void __launch_bounds__(NT, 1) sweep64_kernel(SweepArgs a, const double* __restrict__ tables) {
    extern __shared__ __align__(128) unsigned char smraw[];
    double2* RA = reinterpret_cast<double2*>(smraw + OFF_RA);
    double2* RB = reinterpret_cast<double2*>(smraw + OFF_RB);
    double* ehA = reinterpret_cast<double*>(smraw + OFF_EHA);
    double* ehB = reinterpret_cast<double*>(smraw + OFF_EHB);
    double* ehC = reinterpret_cast<double*>(smraw + OFF_EHC);
    double2* fcache = reinterpret_cast<double2*>(smraw + OFF_FC);
    double2* tw = reinterpret_cast<double2*>(smraw + OFF_TW);
    double* tab = reinterpret_cast<double*>(smraw + OFF_TAB);
    int* stopped = reinterpret_cast<int*>(smraw + OFF_STOP);

    const int b = blockIdx.x;
    const bool planar = (b >> 1) < 64;          // the same for both CTAs of a cluster
    const int tid = threadIdx.x, t = tid & 7;
    const double rMd = 1.0 / (double)M64;       // M = 2^18: multiplying by 1/M rounds exactly like dividing
    unsigned* ctr = a.bar;
    unsigned bidx = 0;

    for (int i = tid; i < 64; i += NT) tw[i] = a.twx[((i & 7) * (i >> 3)) & 63];   // [k1][t]
    for (int i = tid; i < 6 * 64; i += NT) tab[i] = tables[i];
    if (planar) {
        const long hoff = plane_ix().hoff;
        for (int i = tid; i < H64; i += NT) {
            ehA[(i >> 6) * EHP + (i & 63)] = a.eHA[hoff + i];
            ehB[(i >> 6) * EHP + (i & 63)] = a.eHB[hoff + i];
            if constexpr (TRI) ehC[(i >> 6) * EHP + (i & 63)] = a.eHC[hoff + i];
        }
    }
    if (tid == 0) *stopped = 0;

    // x-pass warp index, CTA-fastest so that a phase's tasks spread over all SMs
    const int gwarp = (tid >> 5) * gridDim.x + b;
    const int nwarps = gridDim.x * (NT / 32);
    const int lane = tid & 31, cq = lane >> 3;
    double2* scratch = RB + (tid >> 5) * 256 + cq * 64;
    double2* fc = fcache + (tid >> 5) * 256 + lane;   // this lane's x-pass factors (warps < XH)
    if constexpr (!TRI) {
        // a diblock's (A, B) factor pairs of the warp's half-step x-pass task, x =
        // t + 8 j of its column, for the whole sweep (the task is the same every step)
        if (gwarp < P64 / 4 && (tid >> 5) < XH) xfill(a.eHA, a.eHB, fc, gwarp * 4 + cq, t);
    }
    __syncthreads();

    // block (0 A, 1 B, 2 C) of a lane at step st: lane f runs A then B, switching
    // at LA, and lane c B then A, switching at LB; for a linear ABC triblock
    // lane f runs A, B, C switching at LA and LA + LB, and lane c C, B, A
    // switching at LC and LC + LB
    auto blk_f = [&](int st) { return st < a.LA ? 0 : (!TRI || st < a.LA + a.LB) ? 1 : 2; };
    auto blk_c = [&](int st) { return TRI ? (st < a.LC ? 2 : st < a.LC + a.LB ? 1 : 0) : (st < a.LB ? 1 : 0); };
    auto gl_of = [&](int k) { return k == 0 ? a.eHA : k == 1 ? a.eHB : a.eHC; };
    // the rows' tables (shared) of lane f's and lane c's block
    auto sh_f = [&](int st) {
        if constexpr (TRI) {
            const int k = blk_f(st);
            return k == 0 ? ehA : k == 1 ? ehB : ehC;
        } else {
            return st < a.LA ? ehA : ehB;
        }
    };
    auto sh_c = [&](int st) {
        if constexpr (TRI) {
            const int k = blk_c(st);
            return k == 0 ? ehA : k == 1 ? ehB : ehC;
        } else {
            return st < a.LB ? ehB : ehA;
        }
    };

    auto gsync = [&]() { grid_sync(ctr, a.err, ++bidx, stopped); };

    // The next step's inputs from q[st] (rows, held by the threads of field 0:
    // row r, z = t + 8 j): e^{-w ds/2} q (field 0) gets Dz and goes to W (its Dx
    // and Dy follow); e^{-w ds/4} q (field 1) gets Dz, and after a cluster
    // barrier Dy on the columns -> Z2
    auto next_inputs = [&](double2 (&v)[8], int st) {
        const PlaneIx ix = plane_ix();
        const int c = ix.c, r = ix.r, f = ix.f, ze0 = ix.ze0;
        const int slab = (int)(ix.soff >> 12);
        const double* nf = sh_f(st);
        const double* nc = sh_c(st);
        double2* row = RA + (f * 32 + r) * QP;   // field f's row r: Dz exchange area (field 1: and result)
        if (f == 0) {
#pragma unroll
            for (int j = 0; j < 8; j++) row[32 * QP + t + 8 * j] = v[j];   // q for field 1
        }
        __syncthreads();
        if (f == 0) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const double gf = nf[ze0 + 8 * j], gc = nc[ze0 + 8 * j];
                v[j] = make_double2((gf * gf) * v[j].x, (gc * gc) * v[j].y);
            }
            line_op(v, t, row, 1, tw, ktab(tab, 0, 2));
            // row y = 32 c + r, z = t + 8 j in the x-pass layout
            double2* W = a.Z1 + xq(slab, 32 * c + r, t);
#pragma unroll
            for (int j = 0; j < 8; j++) W[512 * j] = v[j];
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const double2 q = row[t + 8 * j];
                v[j] = make_double2(nf[ze0 + 8 * j] * q.x, nc[ze0 + 8 * j] * q.y);
            }
            line_op(v, t, row, 1, tw, ktab(tab, 1, 2));
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 8; j++) row[t + 8 * j] = v[j];
        }
        cluster_sync_all();
        if (f == 1) {
            // column z = 32 c + r; element y = t + 8 j is row t + 8 (j & 3) of CTA j / 4
            {
                const double2* p = RA + 32 * QP + 32 * c + r + t * QP;
                const unsigned lo = cluster_addr(p, 0), hi = cluster_addr(p, 1);
#pragma unroll
                for (int j = 0; j < 8; j++) v[j] = ld_cluster((j < 4 ? lo : hi) + 16 * 8 * QP * (j & 3));
            }
            line_op(v, t, RB + r, SP, tw, ktab(tab, 1, 1));
            double2* Zg = a.Z2 + xq(slab, t, 32 * c + r);
#pragma unroll
            for (int j = 0; j < 8; j++) Zg[8 * j * 16 * 256] = v[j];   // y = t + 8 j
        }
    };

    // Step st = -1 forms the first inputs from the chain heads; every later
    // step is an x-pass and a plane phase.
    for (int st = -1; st < a.Ns; st++) {
        if (st >= 0) {
            // ---- x-pass: W in place, Z2 -> Z3 (the longer Z2 tasks first) -----
            for (int task = gwarp; task < 2 * (P64 / 4); task += nwarps) {
                // one task a warp; the half-step tasks on warps < XH (the
                // launcher's grid ensures both)
                if ((tid >> 5) >= XW || task + nwarps < 2 * (P64 / 4) || (task < P64 / 4 && (tid >> 5) >= XH)) {
                    atomicExch(a.err, 4);
                    break;
                }
                if (task < P64 / 4) {
                    if constexpr (TRI) {
                        // the warp's factor pairs, again whenever a lane changes block
                        if (st == 0 || blk_f(st) != blk_f(st - 1) || blk_c(st) != blk_c(st - 1))
                            xfill(gl_of(blk_f(st)), gl_of(blk_c(st)), fc, task * 4 + cq, t);
                        xtask_half(a.Z2, a.Z3, false, true, scratch, fc, task * 4 + cq, t, tw, tab, rMd);
                    } else {
                        xtask_half(a.Z2, a.Z3, st >= a.LA, st < a.LB, scratch, fc, task * 4 + cq, t, tw, tab, rMd);
                    }
                } else
                    xtask_full(a.Z1, scratch, (task - P64 / 4) * 4 + cq, t, tw, tab);
            }
            gsync();
        }

        // ---- plane: Z3, W -> q[st+1] -> next W, Z2 -----------------------------
        const bool next = st + 1 < a.Ns;
        if (planar) {
            double2 v[8];
            const PlaneIx ix = plane_ix();
            const int c = ix.c, r = ix.r, f = ix.f, ze0 = ix.ze0;
            const int slab = (int)(ix.soff >> 12);
            const long hoff = ix.hoff;
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
                    // Dy (second half step) of Z3's column z = 32 c + r (y = t + 8 j)
                    const double2* Z3 = a.Z3 + xq(slab, t, 32 * c + r);
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] = Z3[8 * j * 16 * 256];
                    double2* col = RB + r;
                    line_op(v, t, col, PB, tw, ktab(tab, 1, 1));
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 8; j++) col[(t + 8 * j) * PB] = v[j];
                } else {
                    // Dy (full step) of W's column z = 32 c + r, stored with row y
                    // at RB[UC + 32 y + (r ^ (y & 7))] (conflict-free both ways)
                    const double2* W = a.Z1 + xq(slab, t, 32 * c + r);
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] = W[8 * j * 16 * 256];
                    line_op(v, t, RA + (32 + r) * QP, 1, tw, ktab(tab, 0, 1));
#pragma unroll
                    for (int j = 0; j < 8; j++) RB[UC + (t + 8 * j) * 32 + (r ^ t)] = v[j];
                }
                cluster_sync_all();
                if (f == 0) {
                    // Dz of row y = 32 c + r; element z = t + 8 j is column t + 8 (j & 3) of CTA j / 4
                    {
                        const double2* p = RB + (32 * c + r) * PB + t;
                        const unsigned lo = cluster_addr(p, 0), hi = cluster_addr(p, 1);
#pragma unroll
                        for (int j = 0; j < 8; j++) v[j] = ld_cluster((j < 4 ? lo : hi) + 16 * 8 * (j & 3));
                    }
                    line_op(v, t, RA + r * QP, 1, tw, ktab(tab, 1, 2));
                    const double* ef = sh_f(st);
                    const double* ec = sh_c(st);
                    double* of = a.hf + (long)(st + 1) * M64 + hoff + r * 64 + t;
                    double* oc = a.hc + (long)(st + 1) * M64 + hoff + r * 64 + t;
                    // W of row y: column z = t + 8 j sits at column (t ^ (y & 7)) + 8 (j & 3) of CTA j / 4
                    const double2* pu = RB + UC + (32 * c + r) * 32 + (t ^ (r & 7));
                    const unsigned ulo = cluster_addr(pu, 0), uhi = cluster_addr(pu, 1);
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const double hf = ef[ze0 + 8 * j], hc = ec[ze0 + 8 * j];
                        const double2 w = ld_cluster((j < 4 ? ulo : uhi) + 16 * 8 * (j & 3));
                        const double uf = (w.x * (hf * hf)) * rMd, uc = (w.y * (hc * hc)) * rMd;
                        double qf = (v[j].x * hf) * rMd, qc = (v[j].y * hc) * rMd;
                        qf = div_rn(4.0 * qf - uf, 3.0, 1.0 / 3.0);
                        qc = div_rn(4.0 * qc - uc, 3.0, 1.0 / 3.0);
                        of[8 * j] = qf;
                        oc[8 * j] = qc;
                        v[j] = make_double2(qf, qc);
                    }
                }
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
cudaLaunchConfig_t sweep64_config(int grid, int smem, cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
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

std::vector<double> sweep64_axis_tables(const double l[3], double ds) {
    const double PI = 3.14159265358979323846;
    std::vector<double> tab(6 * 64);
    for (int half = 0; half < 2; half++)
        for (int ax = 0; ax < 3; ax++) {
            const double cc = -4.0 * PI * PI / (l[ax] * l[ax]);
            const double h = half ? 0.5 * ds : ds;
            for (int i = 0; i < 64; i++) {
                const int ri = (i < 64 / 2 + 1) ? i : 64 - i;
                tab[half * 192 + ax * 64 + i] = exp(h * (cc * ri * ri));
            }
        }
    return tab;
}

int sweep64_prepare() {
    PS_CUDA(cudaFuncSetAttribute(sweep64_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM64));
    PS_CUDA(cudaFuncSetAttribute(sweep64_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM64_ABC));
    int dev = 0, sms = 0;
    PS_CUDA(cudaGetDevice(&dev));
    PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = sweep64_config(sms & ~1, SMEM64_ABC, nullptr, attr);
    int nclusters = 0;
    PS_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, sweep64_kernel<true>, &cfg));
    nclusters = std::min(nclusters, sms / 2);
    // 64 clusters own the slabs; every x-pass warp with a half-step task keeps
    // its factors resident, so the 2048 tasks need one warp each among the
    // first XW warps of every CTA, the 1024 half-step tasks among the first XH
    if (nclusters < 64 || 2 * nclusters * XW < 2 * (P64 / 4) || 2 * nclusters * XH < P64 / 4) return 0;
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
    cudaLaunchConfig_t cfg = sweep64_config(grid, a.eHC ? SMEM64_ABC : SMEM64, st, attr);
    if (a.eHC)
        PS_CUDA(cudaLaunchKernelEx(&cfg, sweep64_kernel<true>, a, tables));
    else
        PS_CUDA(cudaLaunchKernelEx(&cfg, sweep64_kernel<false>, a, tables));
}

}  // namespace ps
