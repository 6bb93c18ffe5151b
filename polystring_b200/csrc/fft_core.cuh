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
