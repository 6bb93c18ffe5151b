// density_noalloc.cu -- the contour density of ps_density_solve_device for
// callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc or cudaFree: code
// running inside a host program that hands out all device memory from its
// own pool (a foreign allocation there either fails under the pool's memory
// cap or escapes its accounting), and loops that cannot accept the
// device-wide synchronisation that cudaFree implies.  ps_density_solve_device
// allocates a small device table of contour weights on every call; the entry
// point here keeps that table in a fixed array compiled into the library, so
// it allocates nothing.  The caller still owns q, qc and phi.
//
// The table holds at most PS_DENSITY_NOALLOC_MAX_LEN doubles (64 KiB).  Every
// GPU that loads the library holds one copy until the process exits.  All
// calls on a device share it and each call overwrites entries 0..len-1 before
// its density kernel reads them; nothing has to start at zero.  Two calls whose
// kernels overlap on the GPU (different streams, no ordering between them)
// race on the table.
#include "polystring_b200.h"
#include "engine.h"
#include "field_kernels.h"

#include <mutex>
#include <string>

// contour weights of the most recent call on this device
static __device__ __align__(256) double ps_noalloc_contour_weights[PS_DENSITY_NOALLOC_MAX_LEN];

namespace ps {

void set_last_error(const std::string& msg);

namespace {

// weight c_s of contour point s of rule `rule` on n intervals: the same
// values as contour_weights() (Simpson.cc, Quadrature4.cc, Density.cc)
__device__ double rule_weight(int rule, int n, int s) {
    switch (rule) {
    case 0:
        return (s == 0 || s == n) ? 0.5 : 1.0;
    case 1:
        if (s == 0 || s == n) return 1.0 / 3.0;
        return (s & 1) ? 4.0 / 3.0 : 2.0 / 3.0;
    case 2:
        if (s == 0 || s == n) return 0.375;
        if (s == 1 || s == n - 1) return 7 / 6.0;
        if (s == 2 || s == n - 2) return 23 / 24.0;
        return 1.0;
    case 3:
        if (s == 0 || s == n) return 0.0;
        if (s == 1 || s == n - 1) return 55 / 24.0;
        if (s == 2 || s == n - 2) return -1 / 6.0;
        if (s == 3 || s == n - 3) return 33 / 24.0;
        return 1.0;
    case 4:
        if (s == 0) return 0.0;
        if (s == 1) return 55 / 24.0;
        if (s == 2) return -1 / 6.0;
        if (s == 3) return 33 / 24.0;
        if (s == n - 2) return 23 / 24.0;
        if (s == n - 1) return 7 / 6.0;
        if (s == n) return 0.375;
        return 1.0;
    case 5:
        if (s == 0) return 0.375;
        if (s == 1) return 7 / 6.0;
        if (s == 2) return 23 / 24.0;
        if (s == n - 3) return 33 / 24.0;
        if (s == n - 2) return -1 / 6.0;
        if (s == n - 1) return 55 / 24.0;
        if (s == n) return 0.0;
        return 1.0;
    }
    return 0.0;
}

__global__ void fill_weights_kernel(int rule, int n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= n; s += gridDim.x * blockDim.x)
        ps_noalloc_contour_weights[s] = rule_weight(rule, n, s);
}

// the preconditions contour_weights() checks, without building the table
bool rule_valid(int rule, int n) {
    switch (rule) {
    case 0: return n >= 1;
    case 1: return n % 2 == 0 && n >= 4;
    case 2: return n >= 7;
    case 3: return n >= 9;
    case 4: case 5: return n >= 8;
    }
    return false;
}

constexpr int kMaxDevices = 64;
std::mutex g_table_mu;
// per device ordinal: the context the address was looked up in, and the address
void* g_table_ctx[kMaxDevices] = {};
double* g_table[kMaxDevices] = {};

// the calling thread's current driver context (cuCtxGetCurrent, reached
// through the runtime's driver entry-point table so that the library needs
// no link against libcuda); nullptr if it cannot be queried
void* current_context() {
    typedef int (*CtxGetCurrent)(void**);
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (CtxGetCurrent) nullptr;
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// device address of the table on the current device.  The host-side name of
// the array is not a device address, so it is looked up once per device and
// context: a cudaDeviceReset (or any other end of the primary context) loads
// the module again at a new address in the next context, and the changed
// context handle triggers a new look-up.
double* table_address() {
    int dev = -1;
    PS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(PS_ERR_UNSUPPORTED, "device ordinal beyond 63");
    void* ctx = current_context();   // null before the runtime has made a context current
    std::lock_guard<std::mutex> lock(g_table_mu);
    if (!g_table[dev] || !ctx || ctx != g_table_ctx[dev]) {
        double* p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), ps_noalloc_contour_weights);
        if (rc != cudaSuccess)
            throw Error(PS_ERR_CUDA, std::string("cudaGetSymbolAddress of the contour table: ") + cudaGetErrorString(rc));
        g_table[dev] = p;
        g_table_ctx[dev] = current_context();   // current now: the look-up initialised the runtime
    }
    return g_table[dev];
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" int ps_density_solve_device_noalloc(int rule, const double* q, const double* qc, int len, long long M,
                                               double ds, double cc, double* phi, void* stream) {
    try {
        if (!q || !qc || !phi || M < 1 || len < 2) throw Error(PS_ERR_INVALID, "bad density arguments");
        if (len > PS_DENSITY_NOALLOC_MAX_LEN)
            throw Error(PS_ERR_INVALID, "len " + std::to_string(len) + " exceeds the fixed contour table of " +
                                            std::to_string(PS_DENSITY_NOALLOC_MAX_LEN) +
                                            " points; use ps_density_solve_device");
        if (!rule_valid(rule, len - 1)) throw Error(PS_ERR_QUADRATURE, "contour rule precondition fails");
        cudaStream_t st = (cudaStream_t)stream;
        double* table = table_address();
        const int n = len - 1;
        const int threads = 256;
        const int blocks = (len + threads - 1) / threads;
        fill_weights_kernel<<<blocks, threads, 0, st>>>(rule, n);
        PS_CUDA(cudaGetLastError());
        launch_density(q, qc, n, (long)M, table, ds, nullptr, cc, phi, 1, 0, 0, nullptr, st);
        return PS_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return PS_ERR_INVALID;
    }
}
