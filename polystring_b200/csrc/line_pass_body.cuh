// line_pass_body.cuh -- the device side of one line pass (see line_pass.cu):
// tile staging, the shared-memory Stockham FFT and the fused elementwise work
// of every pass mode, as a device function of (tile, field, batch element) so
// that the per-chain kernels (line_pass.cu) and the grouped kernels over many
// independent solves (grouped_pass.cu) run the same code.
#pragma once

#include "ps_internal.h"
#include "fft_core.cuh"

namespace ps {
namespace lp {

// M a power of two: x / M == x * (1 / M) exactly
__device__ __forceinline__ bool is_pow2(double M) {
    const long long m = (long long)M;
    return m > 0 && (m & (m - 1)) == 0;
}

constexpr int kThreads = 256;
constexpr int kMaxEPT = 8;   // tiles hold at most 2048 elements (make_axis_plan)

// loop over this thread's tile elements: a fixed, unrolled count with a
// guard, so that independent global loads are issued back to back
#define PS_ELEMS(e) _Pragma("unroll") for (int k_ = 0, e = threadIdx.x; k_ < kMaxEPT; k_++, e += kThreads) if (e < nel)

struct TileAddr {
    long base, nstride, lstride;
};

__device__ __forceinline__ TileAddr tile_addr(const LineGeom& g, long tile) {
    long l0 = tile * g.T;
    TileAddr a;
    if (g.S == 1) {
        a.base = l0 * g.N; a.nstride = 1; a.lstride = g.N;
    } else {
        long o = l0 / g.S, i0 = l0 % g.S;
        a.base = o * (long)g.N * g.S + i0; a.nstride = g.S; a.lstride = 1;
    }
    return a;
}

// element e of a tile -> (n, line); global offset; smem index
struct Elem {
    int n, l;
    long goff;
    int sidx;
};

template <int N>
__device__ __forceinline__ Elem elem(const LineGeom& g, const TileAddr& a, int e) {
    Elem r;
    if (g.S == 1) { r.l = e / N; r.n = e - r.l * N; }
    else if (g.tshift >= 0) { r.n = e >> g.tshift; r.l = e & (g.T - 1); }
    else          { r.n = e / g.T; r.l = e - r.n * g.T; }
    r.goff = a.base + (long)r.n * a.nstride + (long)r.l * a.lstride;
    r.sidx = r.n * g.LP + r.l;
    return r;
}

template <int N, int R, int NS, int SIGN>
__device__ __forceinline__ void run_pass(const double2* in, double2* out, int T, int LP, const double2* tw) {
    const int total = T * (N / R);
    const int tsh = (T & (T - 1)) == 0 ? __ffs(T) - 1 : -1;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int j = tsh >= 0 ? b >> tsh : b / T;
        int l = b - j * T;
        butterfly<N, R, NS, SIGN>(in, out, LP, l, j, tw);
    }
}

// Full line FFT of the tile held in A (B is the ping-pong partner).  Returns
// the buffer that holds the result.  Caller synchronises before the call.
template <int N, int SIGN>
__device__ __forceinline__ double2* tile_fft(double2* A, double2* B, int T, int LP, const double2* tw) {
    using P = Plan<N>;
    if constexpr (P::P >= 1) { run_pass<N, P::r0, 1, SIGN>(A, B, T, LP, tw); __syncthreads(); }
    if constexpr (P::P >= 2) { run_pass<N, P::r1, P::r0, SIGN>(B, A, T, LP, tw); __syncthreads(); }
    if constexpr (P::P >= 3) { run_pass<N, P::r2, P::r0 * P::r1, SIGN>(A, B, T, LP, tw); __syncthreads(); }
    return (P::P % 2 == 1) ? B : A;
}

__device__ __forceinline__ double2* other(double2* r, double2* A, double2* B) { return r == A ? B : A; }

// One line pass over tile `tile` of field fy of batch element bz (the CTA's
// share of the pass); the kernels below map their blocks onto these indices.
template <int N, int MODE>
__device__ __forceinline__ void line_pass_body(const LineGeom& g, const StepPtrs& p, const double2* __restrict__ gtw,
                                               const long tile, const int fy, const long bz) {
    extern __shared__ double2 smem[];
    double2* twf = smem;
    double2* twi = smem + N;
    const int tile_elems = N * g.LP;
    double2* A = smem + 2 * N;
    double2* B = A + tile_elems;
    double2* C = B + tile_elems;   // END / FULL modes: chain values (lane f, lane c)
    double2* D = C + tile_elems;   // FULL RQM4: full-step result u

    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double2 t = gtw[m];
        twf[m] = t;
        twi[m] = make_double2(t.x, -t.y);
    }

    const TileAddr ta = tile_addr(g, tile);
    const int nel = N * g.T;
    const double M = p.M;
    const double rM = 1.0 / M;
    const bool mpow2 = is_pow2(M);

    const long oz = bz * p.bstride_z, oq = bz * p.bstride_q, oe = bz * p.bstride_e, oL = bz * p.bstride_L;
    const long ou = bz * p.bstride_u;

    if constexpr (MODE == MODE_FWD || MODE == MODE_INV || MODE == MODE_OUTER) {
        double2* z = p.z[fy] + oz;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            A[el.sidx] = z[el.goff];
        }
        __syncthreads();
        double2* r;
        if constexpr (MODE == MODE_INV) {
            r = tile_fft<N, +1>(A, B, g.T, g.LP, twi);
        } else {
            r = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
        }
        if constexpr (MODE == MODE_OUTER) {
            if (p.spec[fy]) {
                double2* sp = p.spec[fy] + oz;
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    sp[el.goff] = r[el.sidx];
                }
            }
            const double* L = p.L[fy] + oL;
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double lv = L[el.goff];
                double2 v = r[el.sidx];
                r[el.sidx] = make_double2(v.x * lv, v.y * lv);
            }
            __syncthreads();
            r = tile_fft<N, +1>(r, other(r, A, B), g.T, g.LP, twi);
        }
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            z[el.goff] = r[el.sidx];
        }
    } else if constexpr (MODE == MODE_FIRST_RQM4 || MODE == MODE_FIRST_OS2) {
        // Z = (e_f q_f) + i (e_c q_c); RQM4: y = 0 uses e^{-w ds/2} (full
        // step), y = 1 uses e^{-w ds/4} (first half step).
        const double* ef = (fy == 0 ? p.eF[0] : p.eH[0]) + oe;
        const double* ec = (fy == 0 ? p.eF[1] : p.eH[1]) + oe;
        const double* qf = p.qin[0] + oq;
        const double* qc = p.qin[1] + oq;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            A[el.sidx] = make_double2(ef[el.goff] * qf[el.goff], ec[el.goff] * qc[el.goff]);
        }
        __syncthreads();
        double2* r = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
        double2* z = p.z[fy] + oz;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            z[el.goff] = r[el.sidx];
        }
    } else if constexpr (MODE == MODE_MID_RQM4) {
        if (fy == 0) {
            // full step: u = Re/Im(F^-1 Z1) e^{-w ds/2} / M
            double2* z = p.z[0] + oz;
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                A[el.sidx] = z[el.goff];
            }
            __syncthreads();
            double2* r = tile_fft<N, +1>(A, B, g.T, g.LP, twi);
            const double* ef = p.eF[0] + oe;
            const double* ec = p.eF[1] + oe;
            double* uf = p.u[0] + ou;
            double* uc = p.u[1] + ou;
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double2 v = r[el.sidx];
                uf[el.goff] = div_pow2_or_rn(v.x * ef[el.goff], M, rM, mpow2);
                uc[el.goff] = div_pow2_or_rn(v.y * ec[el.goff], M, rM, mpow2);
            }
        } else {
            // first half step finishes, second half step starts
            double2* z = p.z[1] + oz;
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                A[el.sidx] = z[el.goff];
            }
            __syncthreads();
            double2* r = tile_fft<N, +1>(A, B, g.T, g.LP, twi);
            const double* hf = p.eH[0] + oe;
            const double* hc = p.eH[1] + oe;
            double* sf = p.half[0];
            double* sc = p.half[1];
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double2 v = r[el.sidx];
                double a = hf[el.goff], b = hc[el.goff];
                double qtf = div_pow2_or_rn(v.x * a, M, rM, mpow2);
                double qtc = div_pow2_or_rn(v.y * b, M, rM, mpow2);
                if (sf) {
                    sf[ou + el.goff] = qtf;
                    sc[ou + el.goff] = qtc;
                }
                r[el.sidx] = make_double2(a * qtf, b * qtc);
            }
            __syncthreads();
            double2* r2 = tile_fft<N, -1>(r, other(r, A, B), g.T, g.LP, twf);
            double2* z3 = p.z[2] + oz;
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                z3[el.goff] = r2[el.sidx];
            }
        }
    } else if constexpr (MODE == MODE_END_ADJ) {
        // lane f: q_t (forward slice), lane c: lambda_{t+1}.  qt2 = S'S'q,
        // vv = S'S'lambda; lambda_t = (4 vv - S lambda)/3 + direct term; the
        // step's w-gradient -(ds/3)[lam qt2 + 2 u v + q vv] + (ds/6)[lam Sq + q Slam]
        double2* zin = p.z[2] + oz;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            A[el.sidx] = zin[el.goff];
        }
        __syncthreads();
        double2* r = tile_fft<N, +1>(A, B, g.T, g.LP, twi);
        const double* hf = p.eH[0] + oe;
        const double* hc = p.eH[1] + oe;
        const double* qv = p.qin[0] + oq;
        const double* lv = p.qin[1];
        double* lout = p.qout[1];
        const double ds = p.gds;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            const long i = el.goff;
            double2 v = r[el.sidx];
            double qt2 = div_pow2_or_rn(v.x * hf[i], M, rM, mpow2);
            double vv = div_pow2_or_rn(v.y * hc[i], M, rM, mpow2);
            double sq = p.u[0][ou + i], sl = p.u[1][ou + i];
            double uh = p.half[0][ou + i], vh = p.half[1][ou + i];
            double q = qv[i], lam = lv[i];
            double lt = div_rn(4.0 * vv - sl, 3.0, 1.0 / 3.0);
            if (p.pbarA) lt += (p.wdA * p.pbarA[i] + p.wdB * p.pbarB[i]) * p.other[i];
            lout[i] = lt;
            if (p.grad)
                p.grad[i] += -(ds / 3.0) * (lam * qt2 + 2.0 * uh * vh + q * vv) + (ds / 6.0) * (lam * sq + q * sl);
            C[el.sidx] = make_double2(0.0, lt);
        }
        if (p.chain_next) {
            for (int k = 0; k < 2; k++) {
                const double* nf = (k == 0 ? p.nF[0] : p.nH[0]) + oe;
                const double* nc = (k == 0 ? p.nF[1] : p.nH[1]) + oe;
                __syncthreads();
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    double2 qq = C[el.sidx];
                    A[el.sidx] = make_double2(nf[el.goff] * p.next_qf[el.goff], nc[el.goff] * qq.y);
                }
                __syncthreads();
                double2* r2 = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
                double2* z = p.z[k] + oz;
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    z[el.goff] = r2[el.sidx];
                }
            }
        }
    } else if constexpr (MODE == MODE_END_RQM4 || MODE == MODE_END_OS2) {
        double2* zin = (MODE == MODE_END_RQM4 ? p.z[2] : p.z[0]) + oz;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            A[el.sidx] = zin[el.goff];
        }
        __syncthreads();
        double2* r = tile_fft<N, +1>(A, B, g.T, g.LP, twi);
        const double* hf = (MODE == MODE_END_RQM4 ? p.eH[0] : p.eF[0]) + oe;
        const double* hc = (MODE == MODE_END_RQM4 ? p.eH[1] : p.eF[1]) + oe;
        double* of = p.qout[0] + oq;
        double* oc = p.qout[1] + oq;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            double2 v = r[el.sidx];
            double qf = div_pow2_or_rn(v.x * hf[el.goff], M, rM, mpow2);
            double qc = div_pow2_or_rn(v.y * hc[el.goff], M, rM, mpow2);
            if constexpr (MODE == MODE_END_RQM4) {
                qf = div_rn(4.0 * qf - p.u[0][ou + el.goff], 3.0, 1.0 / 3.0);
                qc = div_rn(4.0 * qc - p.u[1][ou + el.goff], 3.0, 1.0 / 3.0);
            }
            of[el.goff] = qf;
            oc[el.goff] = qc;
            C[el.sidx] = make_double2(qf, qc);
        }
        if (p.chain_next) {
            const int nz = (MODE == MODE_END_RQM4) ? 2 : 1;
            for (int k = 0; k < nz; k++) {
                const double* nf = (k == 0 ? p.nF[0] : p.nH[0]) + oe;
                const double* nc = (k == 0 ? p.nF[1] : p.nH[1]) + oe;
                __syncthreads();
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    double2 q = C[el.sidx];
                    A[el.sidx] = make_double2(nf[el.goff] * q.x, nc[el.goff] * q.y);
                }
                __syncthreads();
                double2* r2 = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
                double2* z = p.z[k] + oz;
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    z[el.goff] = r2[el.sidx];
                }
            }
        }
    } else if constexpr (MODE == MODE_FULL_RQM4 || MODE == MODE_FULL_OS2) {
        // single-axis grids: the whole step inside one tile
        const double* qf = p.qin[0] + oq;
        const double* qc = p.qin[1] + oq;
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            C[el.sidx] = make_double2(qf[el.goff], qc[el.goff]);
        }
        const double* ef = p.eF[0] + oe;
        const double* ec = p.eF[1] + oe;
        const double* L1 = p.L[0] + oL;
        // sub-step 1: full ds step
        __syncthreads();
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            double2 q = C[el.sidx];
            A[el.sidx] = make_double2(ef[el.goff] * q.x, ec[el.goff] * q.y);
        }
        __syncthreads();
        double2* r = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
        PS_ELEMS(e) {
            Elem el = elem<N>(g, ta, e);
            double lv = L1[el.goff];
            double2 v = r[el.sidx];
            r[el.sidx] = make_double2(v.x * lv, v.y * lv);
        }
        __syncthreads();
        r = tile_fft<N, +1>(r, other(r, A, B), g.T, g.LP, twi);
        double* of = p.qout[0] + oq;
        double* oc = p.qout[1] + oq;
        if constexpr (MODE == MODE_FULL_OS2) {
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double2 v = r[el.sidx];
                of[el.goff] = div_pow2_or_rn(v.x * ef[el.goff], M, rM, mpow2);
                oc[el.goff] = div_pow2_or_rn(v.y * ec[el.goff], M, rM, mpow2);
            }
        } else {
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double2 v = r[el.sidx];
                D[el.sidx] = make_double2(div_pow2_or_rn(v.x * ef[el.goff], M, rM, mpow2), div_pow2_or_rn(v.y * ec[el.goff], M, rM, mpow2));
            }
            const double* hf = p.eH[0] + oe;
            const double* hc = p.eH[1] + oe;
            const double* L2 = p.L[1] + oL;
            // two ds/2 steps: start from C, keep the intermediate in C
            for (int h = 0; h < 2; h++) {
                __syncthreads();
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    double2 q = C[el.sidx];
                    A[el.sidx] = make_double2(hf[el.goff] * q.x, hc[el.goff] * q.y);
                }
                __syncthreads();
                r = tile_fft<N, -1>(A, B, g.T, g.LP, twf);
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    double lv = L2[el.goff];
                    double2 v = r[el.sidx];
                    r[el.sidx] = make_double2(v.x * lv, v.y * lv);
                }
                __syncthreads();
                r = tile_fft<N, +1>(r, other(r, A, B), g.T, g.LP, twi);
                PS_ELEMS(e) {
                    Elem el = elem<N>(g, ta, e);
                    double2 v = r[el.sidx];
                    C[el.sidx] = make_double2(div_pow2_or_rn(v.x * hf[el.goff], M, rM, mpow2), div_pow2_or_rn(v.y * hc[el.goff], M, rM, mpow2));
                }
            }
            __syncthreads();
            PS_ELEMS(e) {
                Elem el = elem<N>(g, ta, e);
                double2 q = C[el.sidx];
                double2 u = D[el.sidx];
                of[el.goff] = div_rn(4.0 * q.x - u.x, 3.0, 1.0 / 3.0);
                oc[el.goff] = div_rn(4.0 * q.y - u.y, 3.0, 1.0 / 3.0);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Register-resident passes (power-of-two lengths 32..256): a line belongs to
// G lanes of one warp (RegPlan<N>), each warp handles 32/G lines, and a CTA's
// warps are independent -- the only shared-memory traffic is one swizzled
// exchange per transform, synchronised with __syncwarp.  Lanes of lines past
// the end of the field still take part in every exchange (their loads and
// stores are skipped), so the warp-wide synchronisation stays complete.
// ---------------------------------------------------------------------------
template <int N>
constexpr bool reg_capable() { return N == 32 || N == 64 || N == 128 || N == 256; }

template <int N, int MODE>
constexpr bool reg_body() {
    return reg_capable<N>() && (MODE == MODE_FWD || MODE == MODE_INV || MODE == MODE_OUTER ||
                                MODE == MODE_FIRST_RQM4 || MODE == MODE_MID_RQM4 || MODE == MODE_END_RQM4);
}

template <int N, int SIGN>
__device__ __forceinline__ void reg_fft(double2 (&v)[RegPlan<N>::E], int t, double2* xbuf, const double2* tw) {
    constexpr int E = RegPlan<N>::E, G = RegPlan<N>::G;
    reg_stage_a<N, SIGN>(v, t, tw);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < E; k1++) xbuf[xslot<G>(k1, t)] = v[k1];
    __syncwarp();
    reg_stage_b<N, SIGN>(v, t, xbuf);
}

template <int N, int MODE>
__device__ __forceinline__ void line_pass_body_reg(const LineGeom& g, const StepPtrs& p,
                                                   const double2* __restrict__ gtw, const long cta, const int fy,
                                                   const long bz) {
    constexpr int G = RegPlan<N>::G, E = RegPlan<N>::E, LS = N + RegPlan<N>::PAD, LW = 32 / G;
    extern __shared__ double2 smem[];
    double2* tw = smem;
    for (int m = threadIdx.x; m < N; m += blockDim.x) tw[m] = gtw[m];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lw = lane / G, t = lane % G;
    double2* xbuf = smem + N + (warp * LW + lw) * LS;
    const long line = (cta * (kThreads / 32) + warp) * LW + lw;
    const bool valid = line < g.nlines;
    long base = 0, ns = 1;
    if (g.S == 1) {
        base = line * N;
    } else {
        const long o = line / g.S, i0 = line - o * g.S;
        base = o * (long)N * g.S + i0;
        ns = g.S;
    }
    const double M = p.M;
    const double rM = 1.0 / M;
    const bool mpow2 = is_pow2(M);
    const long oz = bz * p.bstride_z, oq = bz * p.bstride_q, oe = bz * p.bstride_e, oL = bz * p.bstride_L;
    const long ou = bz * p.bstride_u;
    // register m of every lane holds element t + G m of its line
    auto off = [&](int m) { return base + (long)(t + G * m) * ns; };
    double2 v[E];

    if constexpr (MODE == MODE_FWD || MODE == MODE_INV || MODE == MODE_OUTER) {
        double2* z = p.z[fy] + oz;
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = valid ? z[off(m)] : make_double2(0.0, 0.0);
        if constexpr (MODE == MODE_INV) {
            reg_fft<N, +1>(v, t, xbuf, tw);
        } else {
            reg_fft<N, -1>(v, t, xbuf, tw);
        }
        if constexpr (MODE == MODE_OUTER) {
            if (p.spec[fy] && valid) {
                double2* sp = p.spec[fy] + oz;
#pragma unroll
                for (int m = 0; m < E; m++) sp[off(m)] = v[m];
            }
            const double* L = p.L[fy] + oL;
#pragma unroll
            for (int m = 0; m < E; m++) {
                const double lv = valid ? L[off(m)] : 0.0;
                v[m] = make_double2(v[m].x * lv, v[m].y * lv);
            }
            reg_fft<N, +1>(v, t, xbuf, tw);
        }
        if (valid) {
#pragma unroll
            for (int m = 0; m < E; m++) z[off(m)] = v[m];
        }
    } else if constexpr (MODE == MODE_FIRST_RQM4) {
        const double* ef = (fy == 0 ? p.eF[0] : p.eH[0]) + oe;
        const double* ec = (fy == 0 ? p.eF[1] : p.eH[1]) + oe;
        const double* qf = p.qin[0] + oq;
        const double* qc = p.qin[1] + oq;
#pragma unroll
        for (int m = 0; m < E; m++) {
            if (valid) {
                const long i = off(m);
                v[m] = make_double2(ef[i] * qf[i], ec[i] * qc[i]);
            } else {
                v[m] = make_double2(0.0, 0.0);
            }
        }
        reg_fft<N, -1>(v, t, xbuf, tw);
        if (valid) {
            double2* z = p.z[fy] + oz;
#pragma unroll
            for (int m = 0; m < E; m++) z[off(m)] = v[m];
        }
    } else if constexpr (MODE == MODE_MID_RQM4) {
        const double2* zin = p.z[fy == 0 ? 0 : 1] + oz;
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = valid ? zin[off(m)] : make_double2(0.0, 0.0);
        reg_fft<N, +1>(v, t, xbuf, tw);
        if (fy == 0) {
            // full step: u = Re/Im(F^-1 Z1) e^{-w ds/2} / M
            const double* ef = p.eF[0] + oe;
            const double* ec = p.eF[1] + oe;
            if (valid) {
#pragma unroll
                for (int m = 0; m < E; m++) {
                    const long i = off(m);
                    p.u[0][ou + i] = div_pow2_or_rn(v[m].x * ef[i], M, rM, mpow2);
                    p.u[1][ou + i] = div_pow2_or_rn(v[m].y * ec[i], M, rM, mpow2);
                }
            }
        } else {
            // first half step finishes, second half step starts
            const double* hf = p.eH[0] + oe;
            const double* hc = p.eH[1] + oe;
#pragma unroll
            for (int m = 0; m < E; m++) {
                if (valid) {
                    const long i = off(m);
                    const double a = hf[i], b = hc[i];
                    const double qtf = div_pow2_or_rn(v[m].x * a, M, rM, mpow2);
                    const double qtc = div_pow2_or_rn(v[m].y * b, M, rM, mpow2);
                    if (p.half[0]) {
                        p.half[0][ou + i] = qtf;
                        p.half[1][ou + i] = qtc;
                    }
                    v[m] = make_double2(a * qtf, b * qtc);
                } else {
                    v[m] = make_double2(0.0, 0.0);
                }
            }
            reg_fft<N, -1>(v, t, xbuf, tw);
            if (valid) {
                double2* z3 = p.z[2] + oz;
#pragma unroll
                for (int m = 0; m < E; m++) z3[off(m)] = v[m];
            }
        }
    } else if constexpr (MODE == MODE_END_RQM4) {
        const double2* zin = p.z[2] + oz;
#pragma unroll
        for (int m = 0; m < E; m++) v[m] = valid ? zin[off(m)] : make_double2(0.0, 0.0);
        reg_fft<N, +1>(v, t, xbuf, tw);
        const double* hf = p.eH[0] + oe;
        const double* hc = p.eH[1] + oe;
        double2 q[E];
#pragma unroll
        for (int m = 0; m < E; m++) {
            if (valid) {
                const long i = off(m);
                double qf = div_pow2_or_rn(v[m].x * hf[i], M, rM, mpow2);
                double qc = div_pow2_or_rn(v[m].y * hc[i], M, rM, mpow2);
                qf = div_rn(4.0 * qf - p.u[0][ou + i], 3.0, 1.0 / 3.0);
                qc = div_rn(4.0 * qc - p.u[1][ou + i], 3.0, 1.0 / 3.0);
                p.qout[0][oq + i] = qf;
                p.qout[1][oq + i] = qc;
                q[m] = make_double2(qf, qc);
            } else {
                q[m] = make_double2(0.0, 0.0);
            }
        }
        if (p.chain_next) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const double* nf = (k == 0 ? p.nF[0] : p.nH[0]) + oe;
                const double* nc = (k == 0 ? p.nF[1] : p.nH[1]) + oe;
#pragma unroll
                for (int m = 0; m < E; m++) {
                    if (valid) {
                        const long i = off(m);
                        v[m] = make_double2(nf[i] * q[m].x, nc[i] * q[m].y);
                    } else {
                        v[m] = make_double2(0.0, 0.0);
                    }
                }
                reg_fft<N, -1>(v, t, xbuf, tw);
                if (valid) {
                    double2* z = p.z[k] + oz;
#pragma unroll
                    for (int m = 0; m < E; m++) z[off(m)] = v[m];
                }
            }
        }
    }
}

}  // namespace lp
}  // namespace ps
