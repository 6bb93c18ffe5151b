// cluster_sweep.cu -- RQM4 propagator sweeps of a batch of 2D problems, one
// thread-block cluster per problem, both packed fields resident in the
// cluster's distributed shared memory for the whole sweep.
//
// The string method advances m images of the same small 2D grid at once
// (polystring_AB.cc:111-208 runs one SCFT solve per image).  An image's two
// packed complex work fields (lane f = forward chain in the real part, lane c
// = complementary chain in the imaginary part, as in the line passes) fit in
// the shared memory of C CTAs: CTA r of the cluster owns rows x in
// [r LX/C, (r+1) LX/C) in "row layout" (y lines contiguous, pitch LY + 1,
// y swizzled within aligned groups of 8).
// A 2D transform is
//
//   y FFTs in row layout | cluster transpose | x FFTs in column layout
//
// where the column layout gives CTA r the columns y in [r LY/C, (r+1) LY/C)
// for every x.  The transposes read the peers' shared memory (DSMEM) into
// registers between hardware cluster barriers, then overwrite the local
// buffer in place, so each field needs one buffer per CTA.
//
// For an orthogonal cell F^-1 exp(-h k^2) F = Dx Dy, two commuting line
// operators (exp(-h k^2) is the product of the axis factors), so Dy runs on
// the y lines of the row layout and Dx on the x lines of the column layout.
// One contour step (RQM4.cc:66-92, the reference's operation order for the
// pointwise work and the divisions by M):
//   rows:    A = e^{-w ds/2} q, B = e^{-w ds/4} q;  Dy (full) A, Dy (half) B
//   -> columns (A, B)
//   columns: Dx (full) A -> u = e^{-w ds/2} A / M;  Dx (half) B ->
//            qt = e^{-w ds/4} B / M -> B = e^{-w ds/4} qt;  Dx (half) B
//   -> rows (B, and u copied)
//   rows:    Dy (half) B -> q[t+1] = (4 e^{-w ds/4} B / M - u) / 3
//            -> history, next step's A and B
// Two cluster transposes a step (four field transposes).
//
// No grid barrier and no spin wait: the cluster barrier is a hardware
// barrier every thread of every CTA of the cluster reaches the same number of
// times, and clusters are independent, so they need not be co-resident.
#include <cooperative_groups.h>

#include <cstdio>

#include "ps_internal.h"
#include "fft_core.cuh"
#include "engine.h"
#include "sweep.h"

namespace cg = cooperative_groups;

namespace ps {

namespace {

constexpr int kCT = 128;   // threads per CTA (168 registers a thread at 3 CTAs per SM)

// The CTA's shared memory: twiddles, then field A, then field B.  Passes
// address it by offset, so the compiler knows every such access is a shared
// one (and cannot alias the global factor tables and histories).
extern __shared__ double2 csm[];

// two radix passes per line length: r0 first (no twiddles), then r1
template <int N> struct Plan2;
template <> struct Plan2<32> { static constexpr int r0 = 8, r1 = 4; };
template <> struct Plan2<64> { static constexpr int r0 = 8, r1 = 8; };
template <> struct Plan2<128> { static constexpr int r0 = 16, r1 = 8; };

template <int LX, int LY, int C, int NT>
struct CGeo {
    static constexpr int XR = LX / C;          // rows per CTA (row layout)
    static constexpr int YC = LY / C;          // columns per CTA (column layout)
    static constexpr int RP = LY + 1;          // row pitch in double2
    static constexpr int FS = XR * RP;         // one field's buffer (double2)
    static constexpr int E = XR * LY;          // points per CTA (= LX * YC)
    static constexpr int EPT = E / NT;         // points per thread
    static constexpr long M = (long)LX * LY;
    static constexpr int TWX = (Plan2<LX>::r1 - 1) * Plan2<LX>::r0;   // stage twiddles (x passes)
    static constexpr int TWY = (Plan2<LY>::r1 - 1) * Plan2<LY>::r0;
    // per-axis k factors (doubles): x full, y full, x half, y half, after the fields
    static constexpr int KT = TWX + TWY + 2 * FS;          // offset in double2
    static constexpr int NKT = 2 * (LX + LY);              // doubles
    static_assert(LX % C == 0 && LY % C == 0, "C must divide both axes");
    static_assert(E % NT == 0 && E / NT >= 1, "whole points per thread");
    static_assert(LX * YC == E && E <= FS, "column layout fits the row buffer");
};

// butterfly b of a pass over NL lines with NB butterflies a line: LFAST puts
// consecutive threads on consecutive lines, otherwise on consecutive
// butterflies of one line (consecutive elements of the line)
template <int NL, int NB, bool LFAST>
__device__ __forceinline__ void bmap(int b, int& l, int& j) {
    if (LFAST) { l = b % NL; j = b / NL; } else { j = b % NB; l = b / NB; }
}

// One Stockham butterfly of N-point lines: inputs v[r] = x[j + r N/R] after
// the twiddles of stage NS, outputs y[(j / NS) NS R + j % NS + r NS].  Only
// the last pass of a two-pass plan (NS R = N) has twiddles, W_N^{jm r}, read
// from the stage table tw[(r - 1) NS + jm] (consecutive jm, consecutive banks).
template <int N, int R, int NS, int SIGN>
__device__ __forceinline__ void butterfly(double2 (&v)[R], int j, const double2* tw) {
    static_assert(NS == 1 || NS * R == N, "twiddles only in the last of two passes");
    if (NS > 1) {
        const int jm = j % NS;
#pragma unroll
        for (int r = 1; r < R; r++) {
            double2 w = tw[(r - 1) * NS + jm];
            if (SIGN > 0) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
    }
    Dft<R, SIGN>::run(v);
}
template <int R, int NS>
__device__ __forceinline__ int out_base(int j) { return (j / NS) * NS * R + j % NS; }

struct NoEpi {
    __device__ __forceinline__ double2 operator()(int, int, double2 v) const { return v; }
};

// One in-place pass over NL lines of this CTA's buffer: ad(l, n) is the index
// of element n of line l; epi(l, n, value) gives what is stored at output n
// (the pass's fused epilogue).  The CTA synchronises after the loads and,
// with TAIL, after the stores; without TAIL the caller orders the stores
// before the next reads of this buffer (another pass's load barrier or a
// cluster barrier).
template <int N, int R, int NS, int SIGN, int NL, bool LFAST, bool TAIL, class Ad, class Epi>
__device__ __noinline__ void local_pass(int buf, int tw, Ad ad, Epi epi) {
    constexpr int NB = N / R, TOTAL = NL * NB, BPT = (TOTAL + kCT - 1) / kCT;
    double2 v[BPT][R];
    int ll[BPT], jj[BPT];
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        const int b = threadIdx.x + k * kCT;
        jj[k] = -1;
        if (TOTAL % kCT == 0 || b < TOTAL) {
            bmap<NL, NB, LFAST>(b, ll[k], jj[k]);
#pragma unroll
            for (int r = 0; r < R; r++) v[k][r] = csm[buf + ad(ll[k], jj[k] + r * NB)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        if (jj[k] < 0) continue;
        butterfly<N, R, NS, SIGN>(v[k], jj[k], csm + tw);
        const int o = out_base<R, NS>(jj[k]);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int n = o + r * NS;
            csm[buf + ad(ll[k], n)] = epi(ll[k], n, v[k][r]);
        }
    }
    if (TAIL) __syncthreads();
}

// The last pass of an inverse transform along the lines (radix R1 after
// stages of R0, so butterfly jj holds the outputs jj + R0 r), a pointwise
// epilogue, and the first pass of the next forward transform (radix R0, no
// twiddles: butterfly j takes x[j + R1 r']), fused in registers: thread
// (l, j), j < R1, runs the inverse butterflies j + R1 m (m < R0 / R1), whose
// outputs are exactly forward butterfly j's inputs (r' = m + (R0 / R1) r).
// epi(l, n, value) maps the inverse output at n to the forward input.  One
// load barrier and one store barrier instead of two passes' four.
template <int N, int R0, int R1, int NL, bool LFAST, class Ad, class Epi>
__device__ __noinline__ void inv_epi_fwd_pass(int buf, int tw, Ad ad, Epi epi) {
    static_assert(R0 * R1 == N && R0 % R1 == 0, "two-pass plan with R1 dividing R0");
    constexpr int Q = R0 / R1;
    constexpr int TOTAL = NL * R1, BPT = (TOTAL + kCT - 1) / kCT;
    double2 v[BPT][R0];
    int ll[BPT], jj[BPT];
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        const int b = threadIdx.x + k * kCT;
        jj[k] = -1;
        if (TOTAL % kCT == 0 || b < TOTAL) {
            bmap<NL, R1, LFAST>(b, ll[k], jj[k]);
#pragma unroll
            for (int m = 0; m < Q; m++)
#pragma unroll
                for (int r = 0; r < R1; r++) v[k][m + Q * r] = csm[buf + ad(ll[k], jj[k] + R1 * m + R0 * r)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        if (jj[k] < 0) continue;
        const int j = jj[k], l = ll[k];
#pragma unroll
        for (int m = 0; m < Q; m++) {
            double2 w[R1];
#pragma unroll
            for (int r = 0; r < R1; r++) w[r] = v[k][m + Q * r];
            butterfly<N, R1, R0, +1>(w, j + R1 * m, csm + tw);   // outputs at j + R1 m + R0 r
#pragma unroll
            for (int r = 0; r < R1; r++) v[k][m + Q * r] = w[r];
        }
#pragma unroll
        for (int q = 0; q < R0; q++) v[k][q] = epi(l, j + R1 * q, v[k][q]);
        butterfly<N, R0, 1, -1>(v[k], j, nullptr);                  // outputs at j R0 + r''
#pragma unroll
        for (int q = 0; q < R0; q++) csm[buf + ad(l, j * R0 + q)] = v[k][q];
    }
    __syncthreads();
}

// The same fusion at the end of a contour step, with two outputs: epi(l, n,
// value) returns the next step's inputs of both fields (.a for field A, .b
// for field B) from B's inverse output at n, reading this CTA's field A at n
// (the full-step result u).  B's forward outputs are stored after the load
// barrier; A's only after a second barrier, once no thread reads u any more.
struct FieldPair { double2 a, b; };
template <int N, int R0, int R1, int NL, class Ad, class Epi>
__device__ __noinline__ void inv_epi_fwd2_pass(int bufB, int bufA, int tw, Ad ad, Epi epi) {
    static_assert(R0 * R1 == N && R0 % R1 == 0, "two-pass plan with R1 dividing R0");
    constexpr int Q = R0 / R1;
    constexpr int TOTAL = NL * R1, BPT = (TOTAL + kCT - 1) / kCT;
    double2 v[BPT][R0];
    int ll[BPT], jj[BPT];
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        const int b = threadIdx.x + k * kCT;
        jj[k] = -1;
        if (TOTAL % kCT == 0 || b < TOTAL) {
            ll[k] = b / R1;
            jj[k] = b % R1;
#pragma unroll
            for (int m = 0; m < Q; m++)
#pragma unroll
                for (int r = 0; r < R1; r++) v[k][m + Q * r] = csm[bufB + ad(ll[k], jj[k] + R1 * m + R0 * r)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        if (jj[k] < 0) continue;
        const int j = jj[k], l = ll[k];
#pragma unroll
        for (int m = 0; m < Q; m++) {
            double2 w[R1];
#pragma unroll
            for (int r = 0; r < R1; r++) w[r] = v[k][m + Q * r];
            butterfly<N, R1, R0, +1>(w, j + R1 * m, csm + tw);
#pragma unroll
            for (int r = 0; r < R1; r++) v[k][m + Q * r] = w[r];
        }
        double2 av[R0];
#pragma unroll
        for (int q = 0; q < R0; q++) {
            const FieldPair pr = epi(l, j + R1 * q, v[k][q]);
            av[q] = pr.a;
            v[k][q] = pr.b;
        }
        butterfly<N, R0, 1, -1>(v[k], j, nullptr);
#pragma unroll
        for (int q = 0; q < R0; q++) csm[bufB + ad(l, j * R0 + q)] = v[k][q];
        butterfly<N, R0, 1, -1>(av, j, nullptr);
#pragma unroll
        for (int q = 0; q < R0; q++) v[k][q] = av[q];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        if (jj[k] < 0) continue;
#pragma unroll
        for (int q = 0; q < R0; q++) csm[bufA + ad(ll[k], jj[k] * R0 + q)] = v[k][q];
    }
    __syncthreads();
}

// The first radix pass of the other axis fused with the cluster transpose:
// the butterfly inputs come from the peers' buffers (src(l, n) points at
// element n of line l there), the butterflies run in registers, a cluster
// barrier makes sure no CTA still reads this CTA's buffer, then the outputs
// overwrite it (ad(l, n) as in local_pass).  The caller has synchronised the
// cluster after the peers' buffers became final.
template <int N, int R, int SIGN, int NL, bool LFAST, class Src, class Ad>
__device__ __noinline__ void gather_pass(int buf, Src src, Ad ad) {
    constexpr int NB = N / R, TOTAL = NL * NB, BPT = (TOTAL + kCT - 1) / kCT;
    double2 v[BPT][R];
    int ll[BPT], jj[BPT];
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        const int b = threadIdx.x + k * kCT;
        jj[k] = -1;
        if (TOTAL % kCT == 0 || b < TOTAL) {
            bmap<NL, NB, LFAST>(b, ll[k], jj[k]);
#pragma unroll
            for (int r = 0; r < R; r++) v[k][r] = *src(ll[k], jj[k] + r * NB);
        }
    }
#pragma unroll
    for (int k = 0; k < BPT; k++)
        if (jj[k] >= 0) butterfly<N, R, 1, SIGN>(v[k], jj[k], nullptr);
    // every value read from the peers is consumed above, so the reads are
    // complete: a relaxed cluster barrier (no fence) orders them before the
    // peers overwrite their buffers, and this CTA's before it overwrites its own
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        if (jj[k] < 0) continue;
        const int o = out_base<R, 1>(jj[k]);
#pragma unroll
        for (int r = 0; r < R; r++) csm[buf + ad(ll[k], o + r)] = v[k][r];
    }
}

// The cluster transpose of a field that needs no transform next (the
// full-step result u): the values of NL lines of N points come from the
// peers' buffers (src(l, n)), a cluster barrier orders the reads before any
// CTA overwrites its buffer, then they are stored in this CTA's layout
// (ad(l, n)).  With LFAST false consecutive threads take consecutive n.
// Unlike gather_pass, nothing consumes the loaded values before the barrier,
// so the loads may still be in flight when a thread arrives: the arrival
// has release semantics (not relaxed), which orders them before it.
template <int N, int NL, bool LFAST, class Src, class Ad>
__device__ __noinline__ void gather_copy(int buf, Src src, Ad ad) {
    constexpr int TOTAL = NL * N, BPT = (TOTAL + kCT - 1) / kCT;
    double2 v[BPT];
    int ll[BPT], nn[BPT];
#pragma unroll
    for (int k = 0; k < BPT; k++) {
        const int b = threadIdx.x + k * kCT;
        nn[k] = -1;
        if (TOTAL % kCT == 0 || b < TOTAL) {
            bmap<NL, N, LFAST>(b, ll[k], nn[k]);
            v[k] = *src(ll[k], nn[k]);
        }
    }
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
#pragma unroll
    for (int k = 0; k < BPT; k++)
        if (nn[k] >= 0) csm[buf + ad(ll[k], nn[k])] = v[k];
}

template <int LX, int LY, int C>
__global__ void __launch_bounds__(kCT, 3) cluster_sweep2d_kernel(SweepArgs a) {
    using G = CGeo<LX, LY, C, kCT>;
    constexpr int X0 = Plan2<LX>::r0, X1 = Plan2<LX>::r1;
    constexpr int Y0 = Plan2<LY>::r0, Y1 = Plan2<LY>::r1;
    // gathers: x lines (one per local column) from the peers' rows, y lines
    // (one per local row) from the peers' columns, consecutive threads on
    // consecutive peer addresses

    cg::cluster_group cl = cg::this_cluster();
    const int rk = (int)cl.block_rank();
    const long img = blockIdx.x / C;

    // offsets in csm: stage twiddle tables of the x and y passes, fields A, B
    constexpr int twx = 0, twy = G::TWX, A = G::TWX + G::TWY, B = A + G::FS;
    for (int i = threadIdx.x; i < G::TWX; i += kCT)   // W_LX^{jm r}, r = i / X0 + 1, jm = i % X0
        csm[twx + i] = a.twx[((i % X0) * (i / X0 + 1)) % LX];
    for (int i = threadIdx.x; i < G::TWY; i += kCT)
        csm[twy + i] = a.twy[((i % Y0) * (i / Y0 + 1)) % LY];
    for (int i = threadIdx.x; i < G::NKT; i += kCT) reinterpret_cast<double*>(csm + G::KT)[i] = a.ktab[i];

    const long M = G::M;
    const double Md = (double)M;
    const double rMd = 1.0 / Md;
    const bool mpow2 = (M & (M - 1)) == 0;   // x / M == x * (1 / M) exactly
    const long boff = img * a.bstride_batch;
    double* hf = a.hf + img * a.bstride_hist;
    double* hc = a.hc + img * a.bstride_hist;
    const long g0 = (long)rk * G::E;         // this CTA's rows in natural order
    auto eF = [&](int lane, int t) -> const double* {   // e^{-w ds/2} of the lane's block at step t
        int blk = lane == 0 ? (t < a.LA ? 0 : 1) : (t < a.LB ? 1 : 0);
        return (blk == 0 ? a.eFA : a.eFB) + boff;
    };
    auto eH = [&](int lane, int t) -> const double* {
        int blk = lane == 0 ? (t < a.LA ? 0 : 1) : (t < a.LB ? 1 : 0);
        return (blk == 0 ? a.eHA : a.eHB) + boff;
    };

    // layouts: row (l = local row, n = y) and column (l = local column, n = x)
    // (row layout: y swizzled within aligned groups of 8, n ^ ((n / 16) % 8), so
    // that the 16 outputs of one radix-16 butterfly, 16 apart in a row, fall
    // in different banks; the pitch LY + 1 separates the rows)
    auto rowAd = [](int l, int n) { return l * G::RP + (n ^ ((n >> 4) & 7)); };
    auto colAd = [](int l, int n) { return n * G::YC + l; };
    // element n = x of local column l, from the row layout of the CTA owning x
    auto fromRows = [&](int fld) {
        return [fld, rk](int l, int n) -> const double2* {
            const int y = rk * G::YC + l;
            return cg::this_cluster().map_shared_rank(csm + fld, (unsigned)(n / G::XR)) + (n % G::XR) * G::RP +
                   (y ^ ((y >> 4) & 7));
        };
    };
    // element n = y of local row l, from the column layout of the CTA owning y
    auto fromCols = [&](int fld) {
        return [fld, rk](int l, int n) -> const double2* {
            return cg::this_cluster().map_shared_rank(csm + fld, (unsigned)(n / G::YC)) + (rk * G::XR + l) * G::YC +
                   (n % G::YC);
        };
    };
    // The diffusion operator F^-1 exp(-h k^2) F of an orthogonal cell is the
    // product of two commuting line operators, Dy = F_y^-1 exp(-h k_y^2) F_y
    // on the y lines and Dx on the x lines.  Dy runs in row layout and Dx in
    // column layout, each as a forward line transform whose last pass
    // multiplies by the axis factor (kept in shared memory), then an inverse
    // line transform.  The inverse transforms are unnormalised; the division
    // by M comes after both, where the reference divides.  A contour step
    // then needs two cluster transposes (four field transposes) instead of
    // the four (six) of whole 2D transforms.
    auto ky = [](int half) {      // row layout: element n of a row is k_y index n
        return [half](int, int n, double2 v) {
            const double f = reinterpret_cast<const double*>(csm + G::KT)[half * (LX + LY) + LX + n];
            return make_double2(v.x * f, v.y * f);
        };
    };
    auto kx = [](int half) {      // column layout: element n of a column is k_x index n
        return [half](int, int n, double2 v) {
            const double f = reinterpret_cast<const double*>(csm + G::KT)[half * (LX + LY) + n];
            return make_double2(v.x * f, v.y * f);
        };
    };
    // Dy after its first forward pass: A with the full-step factor, B with the
    // half-step one, passes interleaved (each pass's load barrier orders the
    // other field's stores); the last inverse pass leaves the stores to the
    // cluster barrier of the transpose that follows
    auto dy2 = [&]() {
        local_pass<LY, Y1, Y0, -1, G::XR, false, false>(A, twy, rowAd, ky(0));
        local_pass<LY, Y1, Y0, -1, G::XR, false, false>(B, twy, rowAd, ky(1));
        local_pass<LY, Y0, 1, +1, G::XR, false, false>(A, twy, rowAd, NoEpi());
        local_pass<LY, Y0, 1, +1, G::XR, false, false>(B, twy, rowAd, NoEpi());
        local_pass<LY, Y1, Y0, +1, G::XR, false, false>(A, twy, rowAd, NoEpi());
        local_pass<LY, Y1, Y0, +1, G::XR, false, false>(B, twy, rowAd, NoEpi());
    };
    // peers' rows -> first forward x pass -> this CTA's columns, both fields
    auto rows_to_cols2 = [&]() {
        cl.sync();                                   // every CTA's rows final
        gather_pass<LX, X0, -1, G::YC, true>(B, fromRows(B), colAd);
        gather_pass<LX, X0, -1, G::YC, true>(A, fromRows(A), colAd);
        __syncthreads();
    };
    // peers' columns -> this CTA's rows: B with the first forward y pass, and
    // A (the full-step result u) copied as it is
    auto cols_to_rows2 = [&]() {
        cl.sync();                                   // every CTA's columns final
        gather_pass<LY, Y0, -1, G::XR, false>(B, fromCols(B), rowAd);
        gather_copy<LY, G::XR, false>(A, fromCols(A), rowAd);
        __syncthreads();
    };
    // global index of element n of local column l (column layout)
    auto gcol = [rk](int l, int n) -> long { return (long)n * LY + rk * G::YC + l; };

    // step 0 inputs: A = e^{-w ds/2} q[0], B = e^{-w ds/4} q[0]
    {
        const double *ef = eF(0, 0), *ec = eF(1, 0), *hfp = eH(0, 0), *hcp = eH(1, 0);
#pragma unroll 4
        for (int k = 0; k < G::EPT; k++) {
            const int e = threadIdx.x + k * kCT;
            const long g = g0 + e;
            const int si = rowAd(e / LY, e % LY);
            const double qf = hf[g], qc = hc[g];
            csm[A + si] = make_double2(__ldg(ef + g) * qf, __ldg(ec + g) * qc);
            csm[B + si] = make_double2(__ldg(hfp + g) * qf, __ldg(hcp + g) * qc);
        }
    }
    __syncthreads();

    for (int t = 0; t < a.Ns; t++) {
        const double *ef = eF(0, t), *ec = eF(1, t), *hfp = eH(0, t), *hcp = eH(1, t);
        // ---- Dy of the full step (A) and of the first half step (B) ----------
        // (after step 0 the first forward pass was fused into the previous
        // step's end)
        if (t == 0) {
            local_pass<LY, Y0, 1, -1, G::XR, false, false>(A, twy, rowAd, NoEpi());
            local_pass<LY, Y0, 1, -1, G::XR, false, false>(B, twy, rowAd, NoEpi());
        }
        dy2();
        rows_to_cols2();
        // ---- Dx of both in column layout -------------------------------------
        local_pass<LX, X1, X0, -1, G::YC, true, false>(A, twx, colAd, kx(0));
        local_pass<LX, X1, X0, -1, G::YC, true, false>(B, twx, colAd, kx(1));
        local_pass<LX, X0, 1, +1, G::YC, true, false>(A, twx, colAd, NoEpi());
        local_pass<LX, X0, 1, +1, G::YC, true, false>(B, twx, colAd, NoEpi());
        // u = e^{-w ds/2} A / M stays in A
        local_pass<LX, X1, X0, +1, G::YC, true, false>(A, twx, colAd, [=](int l, int n, double2 v) {
            const long g = gcol(l, n);
            return make_double2(div_pow2_or_rn(v.x * __ldg(ef + g), Md, rMd, mpow2),
                                div_pow2_or_rn(v.y * __ldg(ec + g), Md, rMd, mpow2));
        });
        // B's last inverse x pass, qt = e^{-w ds/4} B / M, the second half
        // step's input e^{-w ds/4} qt and its first forward x pass, in registers
        inv_epi_fwd_pass<LX, X0, X1, G::YC, true>(B, twx, colAd, [=](int l, int n, double2 v) {
            const long g = gcol(l, n);
            const double ha = __ldg(hfp + g), hb = __ldg(hcp + g);
            const double qtf = div_pow2_or_rn(v.x * ha, Md, rMd, mpow2);
            const double qtc = div_pow2_or_rn(v.y * hb, Md, rMd, mpow2);
            return make_double2(ha * qtf, hb * qtc);
        });
        // ---- second half step: Dx in column layout, then Dy in row layout ------
        local_pass<LX, X1, X0, -1, G::YC, true, true>(B, twx, colAd, kx(1));
        local_pass<LX, X0, 1, +1, G::YC, true, true>(B, twx, colAd, NoEpi());
        local_pass<LX, X1, X0, +1, G::YC, true, false>(B, twx, colAd, NoEpi());
        cols_to_rows2();
        local_pass<LY, Y1, Y0, -1, G::XR, false, true>(B, twy, rowAd, ky(1));
        local_pass<LY, Y0, 1, +1, G::XR, false, true>(B, twy, rowAd, NoEpi());
        // last inverse y pass fused with q[t+1] = (4 qt2 - u) / 3, the history
        // write and the next step's inputs A = e^{-w ds/2} q, B = e^{-w ds/4} q
        const bool next = t + 1 < a.Ns;
        const double *nf1 = eF(0, t + 1), *nc1 = eF(1, t + 1), *nf2 = eH(0, t + 1), *nc2 = eH(1, t + 1);
        double* of = hf + (long)(t + 1) * M;
        double* oc = hc + (long)(t + 1) * M;
        // (three straight-line variants, chosen once per step: the last step
        // prepares no next inputs, and the next step's e^{-w ds/4} tables are
        // this step's unless a chain crosses its block boundary at t + 1)
        auto fin = [=](int l, int n, double2 v, const double* gf2, const double* gc2, bool reuse) {
            const long g = g0 + l * LY + n;
            const double2 u = csm[A + rowAd(l, n)];
            const double ha = __ldg(hfp + g), hb = __ldg(hcp + g);
            double qf = div_pow2_or_rn(v.x * ha, Md, rMd, mpow2);
            double qc = div_pow2_or_rn(v.y * hb, Md, rMd, mpow2);
            qf = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
            qc = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
            of[g] = qf;
            oc[g] = qc;
            FieldPair p;
            p.a = make_double2(__ldg(nf1 + g) * qf, __ldg(nc1 + g) * qc);
            p.b = reuse ? make_double2(ha * qf, hb * qc) : make_double2(__ldg(gf2 + g) * qf, __ldg(gc2 + g) * qc);
            return p;
        };
        if (!next) {
            local_pass<LY, Y1, Y0, +1, G::XR, false, true>(B, twy, rowAd, [=](int l, int n, double2 v) {
                const long g = g0 + l * LY + n;
                const int si = rowAd(l, n);
                const double2 u = csm[A + si];
                double qf = div_pow2_or_rn(v.x * __ldg(hfp + g), Md, rMd, mpow2);
                double qc = div_pow2_or_rn(v.y * __ldg(hcp + g), Md, rMd, mpow2);
                of[g] = div_rn(4.0 * qf - u.x, 3.0, 1.0 / 3.0);
                oc[g] = div_rn(4.0 * qc - u.y, 3.0, 1.0 / 3.0);
                return v;
            });
        } else if (nf2 == hfp && nc2 == hcp) {
            // (with the next step's first forward pass of both fields)
            inv_epi_fwd2_pass<LY, Y0, Y1, G::XR>(B, A, twy, rowAd,
                [=](int l, int n, double2 v) { return fin(l, n, v, nullptr, nullptr, true); });
        } else {
            inv_epi_fwd2_pass<LY, Y0, Y1, G::XR>(B, A, twy, rowAd,
                [=](int l, int n, double2 v) { return fin(l, n, v, nf2, nc2, false); });
        }
    }
    cl.sync();   // no peer reads this CTA's shared memory after it exits
}

template <int LX, int LY, int C>
auto kernel_of() {
    return cluster_sweep2d_kernel<LX, LY, C>;
}

template <int LX, int LY, int C>
size_t cl_smem() {
    using G = CGeo<LX, LY, C, kCT>;
    return sizeof(double2) * (size_t)G::KT + sizeof(double) * (size_t)G::NKT;
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
    // the whole unified L1 as shared memory, so three CTAs fit on an SM
    PS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
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
