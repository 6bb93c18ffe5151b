// smem_line_fft.cuh -- in-place line FFTs of a shared-memory buffer with
// register staging, for kernels that keep whole fields on chip (sweep.cu,
// cluster_sweep.cu).
//
// Lines l = 0..NL-1 of length N; element n of line l sits at
// buf[off(l) + n * ES].  Each Stockham radix pass loads every butterfly's
// inputs into registers, synchronises the CTA, then writes the outputs back
// to the same buffer, so one buffer holds the transform in place (and each
// thread holds all its points of the pass in registers across the barrier).
// Every CTA thread (NT of them) must call run(); it ends with the buffer
// consistent.
#pragma once

#include "fft_core.cuh"

namespace ps {

template <int N, int NL, int ES, class Off, int SIGN, int NT, class PL = Plan<N>>
struct SmemLineFFT {
    template <int R, int NS>
    __device__ __forceinline__ static void pass(double2* buf, const double2* tw, const Off& off) {
        constexpr int NB = N / R;
        constexpr int TOTAL = NL * NB;
        constexpr int BPT = (TOTAL + NT - 1) / NT;
        double2 v[BPT][R];
        int base[BPT], jj[BPT];
#pragma unroll
        for (int k = 0; k < BPT; k++) {
            const int b = threadIdx.x + k * NT;
            jj[k] = -1;
            if (TOTAL % NT == 0 || b < TOTAL) {
                const int l = b % NL, j = b / NL;
                jj[k] = j;
                base[k] = off(l);
#pragma unroll
                for (int r = 0; r < R; r++) v[k][r] = buf[base[k] + (j + r * NB) * ES];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BPT; k++) {
            if (jj[k] < 0) continue;
            const int j = jj[k];
            const int jm = j % NS;
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    const int m = (jm * r * (N / (NS * R))) % N;
                    double2 w = tw[m];
                    if (SIGN > 0) w.y = -w.y;
                    v[k][r] = cmul(v[k][r], w);
                }
            }
            Dft<R, SIGN>::run(v[k]);
            const int idxD = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; r++) buf[base[k] + (idxD + r * NS) * ES] = v[k][r];
        }
        __syncthreads();
    }
    __device__ __noinline__ static void run(double2* buf, const double2* tw, const Off& off) {
        if constexpr (PL::P >= 1) pass<PL::r0, 1>(buf, tw, off);
        if constexpr (PL::P >= 2) pass<PL::r1, PL::r0>(buf, tw, off);
        if constexpr (PL::P >= 3) pass<PL::r2, PL::r0 * PL::r1>(buf, tw, off);
    }
};

template <int A>
struct OffMul {   // off(l) = l * A
    __device__ __forceinline__ int operator()(int l) const { return l * A; }
};
template <int INNER, int OUTER_STRIDE>
struct OffSplit {  // off(l) = (l / INNER) * OUTER_STRIDE + (l % INNER)
    __device__ __forceinline__ int operator()(int l) const { return (l / INNER) * OUTER_STRIDE + (l % INNER); }
};

}  // namespace ps
