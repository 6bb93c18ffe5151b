// twiddles.cu -- device tables of W_N^m = exp(-2 pi i m / N).
//
// Computed on the host in long double (x87 80-bit) and rounded once to
// double, so every entry is the correctly rounded root up to the long
// double evaluation error (well below half an ulp of a double).
#include "ps_internal.h"

#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace ps {

namespace {
std::mutex g_tw_mutex;
std::map<std::pair<int, int>, double2*> g_tw;   // (device, N) -> table
}

const double2* twiddle_table(int N) {
    int dev = 0;
    PS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_tw_mutex);
    auto key = std::make_pair(dev, N);
    auto it = g_tw.find(key);
    if (it != g_tw.end()) return it->second;
    std::vector<double2> h(N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < N; m++) {
        long double a = 2.0L * pi * (long double)m / (long double)N;
        h[m].x = (double)cosl(a);
        h[m].y = -(double)sinl(a);
    }
    double2* d = nullptr;
    PS_CUDA(cudaMalloc(&d, sizeof(double2) * N));
    PS_CUDA(cudaMemcpy(d, h.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    g_tw[key] = d;
    return d;
}

}  // namespace ps
