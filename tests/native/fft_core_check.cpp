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

template <int N, int SIGN>
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
    constexpr int r0 = Plan<N>::r0, r1 = Plan<N>::r1, r2 = Plan<N>::r2;
    if (Plan<N>::P >= 1) pass<N, r0, 1, SIGN>(a, b, L, tw.data());
    if (Plan<N>::P >= 2) pass<N, r1, r0, SIGN>(a, b, L, tw.data());
    if (Plan<N>::P >= 3) pass<N, r2, r0 * r1, SIGN>(a, b, L, tw.data());
    double err = 0, mx = 0;
    for (int i = 0; i < N * L; i++) {
        err = fmax(err, fmax(fabs(a[i].x - ref[i].x), fabs(a[i].y - ref[i].y)));
        mx = fmax(mx, fmax(fabs(ref[i].x), fabs(ref[i].y)));
    }
    printf("%d %d %.3e\n", N, SIGN, err / mx);
    return err / mx;
}

int main() {
    double e = 0;
    e = fmax(e, run<2, -1>());   e = fmax(e, run<4, -1>());   e = fmax(e, run<8, -1>());
    e = fmax(e, run<12, -1>());  e = fmax(e, run<16, -1>());  e = fmax(e, run<24, -1>());
    e = fmax(e, run<32, -1>());  e = fmax(e, run<48, -1>());  e = fmax(e, run<64, -1>());
    e = fmax(e, run<96, -1>());  e = fmax(e, run<128, -1>()); e = fmax(e, run<192, -1>());
    e = fmax(e, run<256, -1>());
    e = fmax(e, run<8, 1>());    e = fmax(e, run<48, 1>());   e = fmax(e, run<64, 1>());
    e = fmax(e, run<128, 1>());  e = fmax(e, run<12, 1>());   e = fmax(e, run<256, 1>());
    return e < 1e-14 ? 0 : 1;
}
