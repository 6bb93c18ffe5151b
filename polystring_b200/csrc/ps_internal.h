// ps_internal.h -- shared declarations of the polystring_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <stdexcept>

namespace ps {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define PS_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess)                                                     \
            throw ::ps::Error(-3, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// line passes (kernels in line_pass.cu)
// ---------------------------------------------------------------------------
enum PassMode {
    MODE_FWD = 0,        // forward line FFT of every field
    MODE_INV = 1,        // inverse line FFT of every field
    MODE_OUTER = 2,      // forward, multiply by the k-space table, inverse
    MODE_FIRST_RQM4 = 3, // real chain slices -> Z1 (ds step), Z2 (ds/2 step), forward
    MODE_MID_RQM4 = 4,   // inverse Z1 -> full-step result u; inverse Z2 -> qt -> Z3, forward
    MODE_END_RQM4 = 5,   // inverse Z3 -> qt2, q = (4 qt2 - u)/3 (+ next step's FIRST)
    MODE_FIRST_OS2 = 6,  // real chain slices -> Z, forward
    MODE_END_OS2 = 7,    // inverse Z -> q (+ next step's FIRST)
    MODE_FULL_RQM4 = 8,  // whole RQM4 step when the grid has a single axis
    MODE_FULL_OS2 = 9,   // whole OS2 step when the grid has a single axis
    MODE_END_ADJ = 10,   // adjoint RQM4 step end: lambda_t, w-gradient, next step's FIRST
};

// Geometry of one line pass over a (batch of) field(s) of M points.
struct LineGeom {
    int N;        // line length (FFT size)
    long S;       // element stride of a line
    int T;        // lines per tile
    int LP;       // smem line pitch (T or T + 1)
    long nlines;  // lines per field (M / N)
    long ntiles;  // tiles per field (nlines / T)
    int tshift;   // log2(T) when T is a power of two, else -1
    int reg;      // schedule of the RQM4 / FFT passes of this axis: 0 Stockham in shared memory,
                  // 1 register-resident four-step (one CTA per SM), 2 the same at two CTAs per SM
    long rtiles;  // CTAs per field of a register-resident pass
};

// Register-resident line FFT (fft_core.cuh RegPlan): lines per 256-thread
// CTA for the supported lengths (0 = not supported), and the pass modes that
// have a register-resident body.
__host__ __device__ inline int reg_lines_per_cta(int N) {
    switch (N) {
    case 32: return 64;
    case 64: return 32;
    case 128: return 32;
    case 256: return 16;
    default: return 0;
    }
}

// Pointers used by the fused first / last passes.  A "lane" is one of the
// two real chains packed into one complex field: lane f in the real part,
// lane c in the imaginary part.
struct StepPtrs {
    double2* z[3];           // packed complex work fields W1, W2, W3
    const double* L[3];      // k-space tables for the OUTER pass of z[i]
    const double* qin[2];    // real inputs (chain slices s), lanes f, c
    double* qout[2];         // real outputs (chain slices s + 1)
    double* u[2];            // RQM4 full-step scratch (lanes f, c)
    const double* eF[2];     // exp(-w ds / 2) for the current step, per lane
    const double* eH[2];     // exp(-w ds / 4) (RQM4 half steps), per lane
    const double* nF[2];     // next step's factors (END modes with chaining)
    const double* nH[2];
    int chain_next;          // END modes: also run the next step's FIRST
    int nfield;              // FWD / INV / OUTER: number of fields in z[]
    double M;                // grid points (normalisation of the inverse)
    long bstride_z;          // batch strides (elements) for batched launches
    long bstride_q;          // history slices (qin / qout)
    long bstride_u;          // u scratch buffers
    long bstride_e;          // factor arrays
    long bstride_L;          // k tables
    // adjoint sweeps (lane f = forward slice q_t, lane c = adjoint lambda_{t+1})
    double* half[2];         // MID: save S'q and S'lambda (first half-step results)
    double2* spec[3];        // OUTER: save the spectrum after the forward FFT (field index)
    double* grad;            // END_ADJ: w-gradient of the step's block, accumulated
    double gds;              // END_ADJ: ds of the step's block
    const double* pbarA;     // END_ADJ: direct term (wdA pbarA + wdB pbarB) * other
    const double* pbarB;
    const double* other;
    double wdA, wdB;
    const double* next_qf;   // END_ADJ chaining: lane f input of the next step
};

__host__ __device__ inline bool reg_mode(int mode) {
    return mode == MODE_FWD || mode == MODE_INV || mode == MODE_OUTER || mode == MODE_FIRST_RQM4 ||
           mode == MODE_MID_RQM4 || mode == MODE_END_RQM4;
}
// CTAs per field of a pass of `mode` on axis g
__host__ __device__ inline long pass_tiles(const LineGeom& g, int mode) { return (g.reg && reg_mode(mode)) ? g.rtiles : g.ntiles; }

void launch_line_pass(int mode, const LineGeom& g, const StepPtrs& p, int nbatch, cudaStream_t st);
// sets kernel attributes and builds twiddles; call outside stream capture
void prepare_line_pass(int mode, const LineGeom& g);
size_t line_pass_smem_bytes(int mode, const LineGeom& g);
constexpr size_t kLinePassSmemLimit = 200 * 1024;   // dynamic shared memory of one line-pass CTA
bool line_size_supported(int N);

// ---------------------------------------------------------------------------
// twiddles
// ---------------------------------------------------------------------------
// Device table of W_N^m = exp(-2 pi i m / N) (forward) for a supported N,
// computed on the host in long double and rounded once.
const double2* twiddle_table(int N);

}  // namespace ps
