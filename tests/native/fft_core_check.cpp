// Host-side check of polystring_b200/csrc/fft_core.cuh: runs every supported
// line length through the Stockham passes on the CPU and compares with a
// direct DFT evaluated in long double.  Prints "N sign maxerr" per case and
// exits non-zero when an error exceeds 1e-14 relative.
#include <cmath>
#include <cstdio>
#include <vector>
#include "../../polystring_b200/csrc/fft_core.cuh"

using namespace ps;

template <int N, int R, int NS, int SIGN>
static void pass(std::vector<double2>& in, std::vector<double2>& out, int L, const double2* tw) {
    for (int l = 0; l < L; l++)
        for (int j = 0; j < N / R; j++) butterfly<N, R, NS, SIGN>(in.data(), out.data(), L, l, j, tw);
    in.swap(out);
}

// two-pass plans of particular kernels besides Plan<N> (48 in the generic
// sweep, 128 in the string cluster sweep)
struct Plan16x3 { static constexpr int P = 2, r0 = 16, r1 = 3, r2 = 1; };
struct Plan16x8 { static constexpr int P = 2, r0 = 16, r1 = 8, r2 = 1; };

template <int N, int SIGN, class PL = Plan<N>>
static double run() {
    const int L = 3;
    std::vector<double2> a(N * L), b(N * L), ref(N * L);
    std::vector<double2> tw(N);
    for (int m = 0; m < N; m++) {
        long double ang = 2.0L * 3.141592653589793238462643383279502884L * m / N;
        tw[m] = mk((double)cosl(ang), SIGN * (double)sinl(ang));
    }
    unsigned s = 12345u;
    for (auto& v : a) {
        s = s * 1103515245u + 12345u; v.x = ((s >> 8) & 0xffff) / 65536.0 - 0.5;
        s = s * 1103515245u + 12345u; v.y = ((s >> 8) & 0xffff) / 65536.0 - 0.5;
    }
    for (int l = 0; l < L; l++)
        for (int k = 0; k < N; k++) {
            long double sr = 0, si = 0;
            for (int n = 0; n < N; n++) {
                long double ang = SIGN * 2.0L * 3.141592653589793238462643383279502884L * ((long)n * k % N) / N;
                long double c = cosl(ang), sn = sinl(ang);
                sr += a[n * L + l].x * c - a[n * L + l].y * sn;
                si += a[n * L + l].x * sn + a[n * L + l].y * c;
            }
            ref[k * L + l] = mk((double)sr, (double)si);
        }
    constexpr int r0 = PL::r0, r1 = PL::r1, r2 = PL::r2;
    if (PL::P >= 1) pass<N, r0, 1, SIGN>(a, b, L, tw.data());
    if (PL::P >= 2) pass<N, r1, r0, SIGN>(a, b, L, tw.data());
    if (PL::P >= 3) pass<N, r2, r0 * r1, SIGN>(a, b, L, tw.data());
    double err = 0, mx = 0;
    for (int i = 0; i < N * L; i++) {
        err = fmax(err, fmax(fabs(a[i].x - ref[i].x), fabs(a[i].y - ref[i].y)));
        mx = fmax(mx, fmax(fabs(ref[i].x), fabs(ref[i].y)));
    }
    printf("%d %d %.3e\n", N, SIGN, err / mx);
    return err / mx;
}

// div_rn against IEEE division for the divisors the kernels use (3 and the
// point counts of supported grids), over magnitudes 1e-30 .. 1e30
static double check_div() {
    const double ds[] = {3.0, 4096.0, 16384.0, 32768.0, 110592.0, 262144.0, 884736.0, 9216.0, 1536.0, 36864.0};
    unsigned long long s = 88172645463325252ull;
    long bad = 0;
    for (double d : ds) {
        const double r = 1.0 / d;
        for (int i = 0; i < 200000; i++) {
            s ^= s << 13; s ^= s >> 7; s ^= s << 17;
            double u = (double)(s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
            double x = u * pow(10.0, (int)(s % 61) - 30);
            if (ps::div_rn(x, d, r) != x / d) bad++;
        }
        printf("div %g %ld\n", d, bad);
    }
    return (double)bad;
}

// the register-resident four-step FFT, every lane emulated in turn: stage A,
// the swizzled stores, stage B; against the long-double DFT
template <int N, int SIGN>
static double run_reg() {
    constexpr int E = ps::RegPlan<N>::E, G = ps::RegPlan<N>::G;
    std::vector<double2> x(N), tw(N), line(E * G);
    for (int i = 0; i < N; i++) {
        x[i] = ps::mk(std::sin(0.37 * i + 0.1) + 0.25 * i / N, std::cos(1.3 * i) - 0.5);
        long double a = -2.0L * 3.14159265358979323846264338327950288L * i / N;
        tw[i] = ps::mk((double)cosl(a), (double)sinl(a));
    }
    std::vector<std::vector<double2>> v(G, std::vector<double2>(E));
    for (int t = 0; t < G; t++) {
        for (int n = 0; n < E; n++) v[t][n] = x[G * n + t];
        ps::reg_stage_a<N, SIGN>(v[t].data(), t, tw.data());
        for (int k1 = 0; k1 < E; k1++) line[ps::xslot<G>(k1, t)] = v[t][k1];
    }
    double err = 0, mx = 0;
    for (int t = 0; t < G; t++) {
        ps::reg_stage_b<N, SIGN>(v[t].data(), t, line.data());
        for (int m = 0; m < E; m++) {
            const int k = t + G * m;
            long double re = 0, im = 0;
            for (int n = 0; n < N; n++) {
                long double a = SIGN * 2.0L * 3.14159265358979323846264338327950288L * ((long)k * n % N) / N;
                re += x[n].x * cosl(a) - x[n].y * sinl(a);
                im += x[n].x * sinl(a) + x[n].y * cosl(a);
            }
            err = fmax(err, fmax(fabs((double)(v[t][m].x - re)), fabs((double)(v[t][m].y - im))));
            mx = fmax(mx, fmax(fabs((double)re), fabs((double)im)));
        }
    }
    printf("reg%d %d %.3e\n", N, SIGN, err / mx);
    return err / mx;
}

int main() {
    double e = check_div();
    e = fmax(e, run_reg<32, -1>()); e = fmax(e, run_reg<64, -1>()); e = fmax(e, run_reg<128, -1>());
    e = fmax(e, run_reg<256, -1>()); e = fmax(e, run_reg<32, 1>()); e = fmax(e, run_reg<128, 1>());
    e = fmax(e, run_reg<256, 1>());
    e = fmax(e, run<2, -1>());   e = fmax(e, run<4, -1>());   e = fmax(e, run<8, -1>());
    e = fmax(e, run<12, -1>());  e = fmax(e, run<16, -1>());  e = fmax(e, run<24, -1>());
    e = fmax(e, run<32, -1>());  e = fmax(e, run<48, -1>());  e = fmax(e, run<64, -1>());
    e = fmax(e, run<96, -1>());  e = fmax(e, run<128, -1>()); e = fmax(e, run<192, -1>());
    e = fmax(e, run<256, -1>()); e = fmax(e, run<352, -1>()); e = fmax(e, run<352, 1>());
    e = fmax(e, run<8, 1>());    e = fmax(e, run<48, 1>());   e = fmax(e, run<64, 1>());
    e = fmax(e, run<128, 1>());  e = fmax(e, run<12, 1>());   e = fmax(e, run<256, 1>());
    e = fmax(e, run<48, -1, Plan16x3>());  e = fmax(e, run<48, 1, Plan16x3>());
    e = fmax(e, run<128, -1, Plan16x8>()); e = fmax(e, run<128, 1, Plan16x8>());
    return e < 1e-14 ? 0 : 1;
}
