// fft_core.cuh -- FP64 complex DFT building blocks shared by the CUDA line
// passes and by the host-side unit test of the index arithmetic.
//
// The transforms are mixed-radix Stockham autosort FFTs (the formulation of
// Govindaraju, Lloyd, Dotsenko, Smith and Manferdelli, "High performance
// discrete Fourier transforms on graphics processors", SC 2008):
//
//   pass p, radix R, Ns = product of the radices of the earlier passes,
//   butterfly j in [0, N/R):
//     v[r]  = in[j + r N/R] * W_N^{ (j mod Ns) r N/(Ns R) },   r = 0..R-1
//     v     = DFT_R(v)
//     out[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
//
// with W_N = exp(sign 2 pi i / N).  After the last pass the output is in
// natural order.  Forward transforms use sign = -1 and inverse ones +1; both
// are unnormalised, like the FFTW c2c plans of the reference (RQM4.cc:22-32).
#pragma once

#ifdef __CUDACC__
#define PS_HD __host__ __device__ __forceinline__
#else
#define PS_HD inline
#include <cmath>
struct double2 { double x, y; };
#endif

namespace ps {

PS_HD double2 mk(double a, double b) { double2 r; r.x = a; r.y = b; return r; }
PS_HD double2 add(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
PS_HD double2 sub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
PS_HD double2 cmul(double2 a, double2 b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by sign*i: forward (sign -1) -> -i, inverse -> +i
template <int SIGN> PS_HD double2 mul_si(double2 a) {
    return SIGN < 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

// x / d rounded to nearest, from r = RN(1/d): q = RN(x r) is within an ulp
// of x/d, the remainder x - d q is exact in one fma, and one correction step
// RN(q + (x - d q) r) is the correctly rounded quotient (P. Markstein, IBM
// J. Res. Dev. 34(1), 1990).  Three FP64 operations instead of a division.
PS_HD double div_rn(double x, double d, double r) {
    const double q = x * r;
    return fma(fma(-d, q, x), r, q);
}

// x / d for d = 2^k given r = 1/d (exact): one multiply, the same rounding
// as the division; otherwise div_rn
PS_HD double div_pow2_or_rn(double x, double d, double r, bool pow2) { return pow2 ? x * r : div_rn(x, d, r); }

// sqrt(1/2) and sin(2 pi/3) rounded to double
#define PS_SQRT1_2 0.70710678118654752440
#define PS_SIN60 0.86602540378443864676

template <int R, int SIGN> struct Dft;

template <int SIGN> struct Dft<1, SIGN> {
    PS_HD static void run(double2* v) { (void)v; }
};

template <int SIGN> struct Dft<2, SIGN> {
    PS_HD static void run(double2* v) {
        double2 a = v[0], b = v[1];
        v[0] = add(a, b);
        v[1] = sub(a, b);
    }
};

template <int SIGN> struct Dft<3, SIGN> {
    // X0 = a+b+c; X1,2 = a - (b+c)/2 -/+ i*sign*... with W3 = exp(sign 2 pi i/3)
    PS_HD static void run(double2* v) {
        double2 a = v[0], b = v[1], c = v[2];
        double2 s = add(b, c);
        double2 d = sub(b, c);
        double2 m = mk(a.x - 0.5 * s.x, a.y - 0.5 * s.y);
        // sign*i*sin60*d
        double2 t = mul_si<SIGN>(mk(PS_SIN60 * d.x, PS_SIN60 * d.y));
        v[0] = add(a, s);
        v[1] = add(m, t);
        v[2] = sub(m, t);
    }
};

template <int SIGN> struct Dft<4, SIGN> {
    PS_HD static void run(double2* v) {
        double2 t0 = add(v[0], v[2]);
        double2 t1 = sub(v[0], v[2]);
        double2 t2 = add(v[1], v[3]);
        double2 t3 = mul_si<SIGN>(sub(v[1], v[3]));
        v[0] = add(t0, t2);
        v[2] = sub(t0, t2);
        v[1] = add(t1, t3);
        v[3] = sub(t1, t3);
    }
};

template <int SIGN> struct Dft<8, SIGN> {
    // decimation in frequency: radix-2 over (n, n+4), twiddle W8^n on the
    // difference half, then two radix-4 transforms (even and odd outputs).
    PS_HD static void run(double2* v) {
        double2 b0 = add(v[0], v[4]), b4 = sub(v[0], v[4]);
        double2 b1 = add(v[1], v[5]), b5 = sub(v[1], v[5]);
        double2 b2 = add(v[2], v[6]), b6 = sub(v[2], v[6]);
        double2 b3 = add(v[3], v[7]), b7 = sub(v[3], v[7]);
        // W8^1 = (1 + sign i)/sqrt2, W8^2 = sign i, W8^3 = (-1 + sign i)/sqrt2
        double2 t5 = add(b5, mul_si<SIGN>(b5));
        b5 = mk(PS_SQRT1_2 * t5.x, PS_SQRT1_2 * t5.y);
        b6 = mul_si<SIGN>(b6);
        double2 t7 = sub(mul_si<SIGN>(b7), b7);
        b7 = mk(PS_SQRT1_2 * t7.x, PS_SQRT1_2 * t7.y);
        double2 e[4] = {b0, b1, b2, b3};
        double2 o[4] = {b4, b5, b6, b7};
        Dft<4, SIGN>::run(e);
        Dft<4, SIGN>::run(o);
        v[0] = e[0]; v[2] = e[1]; v[4] = e[2]; v[6] = e[3];
        v[1] = o[0]; v[3] = o[1]; v[5] = o[2]; v[7] = o[3];
    }
};

template <int SIGN> struct Dft<11, SIGN> {
    // Direct 11-point DFT over the symmetric pairs (x[n], x[11 - n]):
    // X[k], X[11 - k] = x0 + sum_n (x[n] + x[11-n]) cos(2 pi n k / 11)
    //                  +/- sign i sum_n (x[n] - x[11-n]) sin(2 pi n k / 11), n = 1..5.
    // cos, sin(2 pi m / 11), m = 1..5, rounded to double from 50-digit values.
    PS_HD static void run(double2* v) {
        const double C[5] = {0.84125353283118120551, 0.41541501300188643508, -0.14231483827328514358,
                             -0.65486073394528510061, -0.95949297361449736865};
        const double S[5] = {0.54064081745559755543, 0.90963199535451833011, 0.98982144188093268422,
                             0.75574957435425826890, 0.28173255684142967104};
        double2 a[5], b[5];
#pragma unroll
        for (int n = 1; n <= 5; n++) {
            a[n - 1] = add(v[n], v[11 - n]);
            b[n - 1] = sub(v[n], v[11 - n]);
        }
        const double2 x0 = v[0];
        double2 sum = x0;
#pragma unroll
        for (int n = 0; n < 5; n++) sum = add(sum, a[n]);
#pragma unroll
        for (int k = 1; k <= 5; k++) {
            double2 t = x0, u = mk(0.0, 0.0);
#pragma unroll
            for (int n = 1; n <= 5; n++) {
                const int m = (n * k) % 11;
                const double c = m <= 5 ? C[m - 1] : C[10 - m];
                const double sn = m <= 5 ? S[m - 1] : -S[10 - m];
                t = mk(t.x + a[n - 1].x * c, t.y + a[n - 1].y * c);
                u = mk(u.x + b[n - 1].x * sn, u.y + b[n - 1].y * sn);
            }
            const double2 iu = mul_si<SIGN>(u);
            v[k] = add(t, iu);
            v[11 - k] = sub(t, iu);
        }
        v[0] = sum;
    }
};

template <int SIGN> struct Dft<16, SIGN> {
    // 16 = 4 x 4: DFT4 over n1 of x[4 n1 + n2], twiddle W16^(n2 k1), DFT4
    // over n2; X[k1 + 4 k2].  W16^m = cos(pi m/8) + sign i sin(pi m/8).
    PS_HD static void run(double2* v) {
        const double C1 = 0.92387953251128675613, S1 = 0.38268343236508977173;
        double2 a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            double2 q[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<4, SIGN>::run(q);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) a[k1][n2] = q[k1];
        }
        const double sg = (double)SIGN;
        // W^1, W^2, W^3, W^6, W^9 (W^4 = sign i)
        const double2 w1 = mk(C1, sg * S1), w2 = mk(PS_SQRT1_2, sg * PS_SQRT1_2), w3 = mk(S1, sg * C1);
        const double2 w6 = mk(-PS_SQRT1_2, sg * PS_SQRT1_2), w9 = mk(-C1, -sg * S1);
        a[1][1] = cmul(a[1][1], w1); a[1][2] = cmul(a[1][2], w2); a[1][3] = cmul(a[1][3], w3);
        a[2][1] = cmul(a[2][1], w2); a[2][2] = mul_si<SIGN>(a[2][2]); a[2][3] = cmul(a[2][3], w6);
        a[3][1] = cmul(a[3][1], w3); a[3][2] = cmul(a[3][2], w6); a[3][3] = cmul(a[3][3], w9);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            Dft<4, SIGN>::run(a[k1]);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = a[k1][k2];
        }
    }
};

// Register-resident line FFT (four-step, N = E x G): a line is owned by G
// lanes of one warp, lane t holding the stride-G set x[G n + t], n < E.
//   stage A (in registers): DFT_E over n, then twiddle W_N^(t k1);
//   exchange (shared memory, one line's G lanes): lane t stores its E values
//     at slots xslot(k1, t); lane t' then gathers (k1, t) for k1 = t' + G j;
//   stage B (in registers): DFT_G over t for each j, giving X[k1 + E k2].
// Lane t' ends with X[t' + G m], m = j + (E / G) k2: again the stride-G set
// of offset t', so inverse transform, elementwise work and forward transform
// chain without leaving registers.  The slot rotation (t + k1) mod G makes
// both the stores and the gathers of a quarter-warp hit distinct bank groups.
template <int N> struct RegPlan;
template <> struct RegPlan<32>  { static constexpr int G = 4, E = 8, PAD = 4; };
template <> struct RegPlan<64>  { static constexpr int G = 8, E = 8, PAD = 0; };
template <> struct RegPlan<128> { static constexpr int G = 8, E = 16, PAD = 0; };
template <> struct RegPlan<256> { static constexpr int G = 16, E = 16, PAD = 0; };

template <int G> PS_HD int xslot(int k1, int t) { return k1 * G + ((t + k1) % G); }

// stage A of lane t: tw[m] = W_N^m of the forward direction (conjugated for SIGN > 0)
template <int N, int SIGN>
PS_HD void reg_stage_a(double2* v, int t, const double2* tw) {
    constexpr int E = RegPlan<N>::E;
    Dft<E, SIGN>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < E; k1++) {
        double2 w = tw[(t * k1) & (N - 1)];
        if (SIGN > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
}

// stage B of lane t from the exchange area of its line (after the stores)
template <int N, int SIGN>
PS_HD void reg_stage_b(double2* v, int t, const double2* line) {
    constexpr int E = RegPlan<N>::E, G = RegPlan<N>::G;
#pragma unroll
    for (int j = 0; j < E / G; j++) {
        double2 w[G];
        const int k1 = t + G * j;
#pragma unroll
        for (int s = 0; s < G; s++) w[s] = line[xslot<G>(k1, s)];
        Dft<G, SIGN>::run(w);
#pragma unroll
        for (int k2 = 0; k2 < G; k2++) v[j + (E / G) * k2] = w[k2];
    }
}

// Radix plans per line length (compile time).  Every supported length is
// 2^a 3^b with at most three passes.
template <int N> struct Plan;
template <> struct Plan<1>   { static constexpr int P = 0; static constexpr int r0 = 1, r1 = 1, r2 = 1; };
template <> struct Plan<2>   { static constexpr int P = 1; static constexpr int r0 = 2, r1 = 1, r2 = 1; };
template <> struct Plan<4>   { static constexpr int P = 1; static constexpr int r0 = 4, r1 = 1, r2 = 1; };
template <> struct Plan<8>   { static constexpr int P = 1; static constexpr int r0 = 8, r1 = 1, r2 = 1; };
template <> struct Plan<12>  { static constexpr int P = 2; static constexpr int r0 = 4, r1 = 3, r2 = 1; };
template <> struct Plan<16>  { static constexpr int P = 2; static constexpr int r0 = 4, r1 = 4, r2 = 1; };
template <> struct Plan<24>  { static constexpr int P = 2; static constexpr int r0 = 8, r1 = 3, r2 = 1; };
template <> struct Plan<32>  { static constexpr int P = 2; static constexpr int r0 = 8, r1 = 4, r2 = 1; };
template <> struct Plan<48>  { static constexpr int P = 3; static constexpr int r0 = 4, r1 = 4, r2 = 3; };
template <> struct Plan<64>  { static constexpr int P = 2; static constexpr int r0 = 8, r1 = 8, r2 = 1; };
template <> struct Plan<96>  { static constexpr int P = 3; static constexpr int r0 = 8, r1 = 4, r2 = 3; };
template <> struct Plan<128> { static constexpr int P = 3; static constexpr int r0 = 8, r1 = 4, r2 = 4; };
template <> struct Plan<192> { static constexpr int P = 3; static constexpr int r0 = 8, r1 = 8, r2 = 3; };
template <> struct Plan<256> { static constexpr int P = 3; static constexpr int r0 = 8, r1 = 8, r2 = 4; };
template <> struct Plan<352> { static constexpr int P = 3; static constexpr int r0 = 8, r1 = 4, r2 = 11; };

// One Stockham butterfly on a tile stored "line fastest": element n of line
// l sits at buf[n * LP + l] (LP = line pitch).  tw[m] = W_N^m for the
// transform direction.
template <int N, int R, int NS, int SIGN>
PS_HD void butterfly(const double2* in, double2* out, int LP, int l, int j, const double2* tw) {
    double2 v[R];
    const int jm = j % NS;
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[(j + r * (N / R)) * LP + l];
    if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) {
            const int m = (jm * r * (N / (NS * R))) % N;
            v[r] = cmul(v[r], tw[m]);
        }
    }
    Dft<R, SIGN>::run(v);
    const int idxD = (j / NS) * NS * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) out[(idxD + r * NS) * LP + l] = v[r];
}

}  // namespace ps
