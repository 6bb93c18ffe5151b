// line_pass.cu -- shared-memory Stockham line FFTs over one axis of a
// periodic grid, with the elementwise work of the propagator step fused into
// the first and last passes.
//
// A pass works on tiles of T lines of length N.  A tile is staged in shared
// memory "line fastest" (element n of line l at buf[n * LP + l]) so that
// consecutive threads touch consecutive lines: the global loads are
// coalesced for both contiguous lines (innermost axis, S == 1, the tile is one
// contiguous block) and strided lines (outer axes, the T lines of a tile are
// contiguous for every n).  Radix passes ping-pong between two tile buffers.
//
// The step being computed is the reference's RQM4 / OS2 split step
// (RQM4.cc:66-92, PseudoSpectral.cc:248-260)
//     q' = e^{-w h/2} F^-1[ exp(-h k^2) F[ e^{-w h/2} q ] ] / M
// for two independent real chains packed into one complex field (lane f in
// the real part, lane c in the imaginary part).  Both lanes share the k-space
// table, which is real and even in k, so the packed transform carries both
// real transforms exactly.
#include "line_pass_body.cuh"

namespace ps {

namespace {

using namespace lp;

template <int N, int MODE>
__global__ void __launch_bounds__(kThreads) line_pass_kernel(LineGeom g, StepPtrs p, const double2* __restrict__ gtw) {
    line_pass_body<N, MODE>(g, p, gtw, blockIdx.x, blockIdx.y, blockIdx.z);
}

// register-resident passes, compiled apart from the Stockham ones so that
// each keeps its own register budget; OCC = resident CTAs per SM the
// compiler must allow (1: no spills, 2: twice the warps, may spill at 128+)
template <int N, int MODE, int OCC>
__global__ void __launch_bounds__(kThreads, OCC)
    line_pass_reg_kernel(LineGeom g, StepPtrs p, const double2* __restrict__ gtw) {
    if constexpr (reg_body<N, MODE>()) line_pass_body_reg<N, MODE>(g, p, gtw, blockIdx.x, blockIdx.y, blockIdx.z);
}

constexpr int kMaxSmem = (int)kLinePassSmemLimit;

int buffers_for_mode(int mode) {
    switch (mode) {
    case MODE_END_RQM4: case MODE_END_OS2: case MODE_FULL_OS2: case MODE_END_ADJ: return 3;
    case MODE_FULL_RQM4: return 4;
    default: return 2;
    }
}

int grid_y_for_mode(int mode, int nfield) {
    switch (mode) {
    case MODE_FWD: case MODE_INV: case MODE_OUTER: return nfield;
    case MODE_FIRST_RQM4: case MODE_MID_RQM4: return 2;
    default: return 1;
    }
}

template <int N, int MODE>
void prepare_nm() {
    PS_CUDA(cudaFuncSetAttribute(line_pass_kernel<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kMaxSmem));
    if constexpr (reg_body<N, MODE>()) {
        PS_CUDA(cudaFuncSetAttribute(line_pass_reg_kernel<N, MODE, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kMaxSmem));
        PS_CUDA(cudaFuncSetAttribute(line_pass_reg_kernel<N, MODE, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kMaxSmem));
    }
}

template <int N, int MODE>
void launch_nm(const LineGeom& g, const StepPtrs& p, int nbatch, cudaStream_t st, bool prepare_only) {
    if (prepare_only) { prepare_nm<N, MODE>(); return; }
    size_t smem = line_pass_smem_bytes(MODE, g);
    if (smem > (size_t)kMaxSmem) throw Error(-2, "line pass tile does not fit in shared memory");
    dim3 grid((unsigned)pass_tiles(g, MODE), (unsigned)grid_y_for_mode(MODE, p.nfield), (unsigned)nbatch);
    if constexpr (reg_body<N, MODE>()) {
        if (g.reg == 1) {
            line_pass_reg_kernel<N, MODE, 1><<<grid, kThreads, smem, st>>>(g, p, twiddle_table(N));
            PS_CUDA(cudaGetLastError());
            return;
        }
        if (g.reg == 2) {
            line_pass_reg_kernel<N, MODE, 2><<<grid, kThreads, smem, st>>>(g, p, twiddle_table(N));
            PS_CUDA(cudaGetLastError());
            return;
        }
    }
    line_pass_kernel<N, MODE><<<grid, kThreads, smem, st>>>(g, p, twiddle_table(N));
    PS_CUDA(cudaGetLastError());
}

template <int N>
void launch_n(int mode, const LineGeom& g, const StepPtrs& p, int nbatch, cudaStream_t st, bool po) {
    switch (mode) {
    case MODE_FWD: launch_nm<N, MODE_FWD>(g, p, nbatch, st, po); break;
    case MODE_INV: launch_nm<N, MODE_INV>(g, p, nbatch, st, po); break;
    case MODE_OUTER: launch_nm<N, MODE_OUTER>(g, p, nbatch, st, po); break;
    case MODE_FIRST_RQM4: launch_nm<N, MODE_FIRST_RQM4>(g, p, nbatch, st, po); break;
    case MODE_MID_RQM4: launch_nm<N, MODE_MID_RQM4>(g, p, nbatch, st, po); break;
    case MODE_END_RQM4: launch_nm<N, MODE_END_RQM4>(g, p, nbatch, st, po); break;
    case MODE_FIRST_OS2: launch_nm<N, MODE_FIRST_OS2>(g, p, nbatch, st, po); break;
    case MODE_END_OS2: launch_nm<N, MODE_END_OS2>(g, p, nbatch, st, po); break;
    case MODE_FULL_RQM4: launch_nm<N, MODE_FULL_RQM4>(g, p, nbatch, st, po); break;
    case MODE_FULL_OS2: launch_nm<N, MODE_FULL_OS2>(g, p, nbatch, st, po); break;
    case MODE_END_ADJ: launch_nm<N, MODE_END_ADJ>(g, p, nbatch, st, po); break;
    default: throw Error(-1, "unknown line pass mode");
    }
}

}  // namespace

bool line_size_supported(int N) {
    switch (N) {
    case 2: case 4: case 8: case 12: case 16: case 24: case 32: case 48: case 64:
    case 96: case 128: case 192: case 256: case 352: return true;
    default: return false;
    }
}

namespace {
void dispatch(int mode, const LineGeom& g, const StepPtrs& p, int nbatch, cudaStream_t st, bool po) {
    switch (g.N) {
    case 2: launch_n<2>(mode, g, p, nbatch, st, po); break;
    case 4: launch_n<4>(mode, g, p, nbatch, st, po); break;
    case 8: launch_n<8>(mode, g, p, nbatch, st, po); break;
    case 12: launch_n<12>(mode, g, p, nbatch, st, po); break;
    case 16: launch_n<16>(mode, g, p, nbatch, st, po); break;
    case 24: launch_n<24>(mode, g, p, nbatch, st, po); break;
    case 32: launch_n<32>(mode, g, p, nbatch, st, po); break;
    case 48: launch_n<48>(mode, g, p, nbatch, st, po); break;
    case 64: launch_n<64>(mode, g, p, nbatch, st, po); break;
    case 96: launch_n<96>(mode, g, p, nbatch, st, po); break;
    case 128: launch_n<128>(mode, g, p, nbatch, st, po); break;
    case 192: launch_n<192>(mode, g, p, nbatch, st, po); break;
    case 256: launch_n<256>(mode, g, p, nbatch, st, po); break;
    case 352: launch_n<352>(mode, g, p, nbatch, st, po); break;
    default: throw Error(-2, "unsupported FFT line length " + std::to_string(g.N));
    }
}
}  // namespace

size_t line_pass_smem_bytes(int mode, const LineGeom& g) {
    if (g.reg && reg_mode(mode)) {
        // twiddles + one exchange area per line of the CTA (RegPlan pads N = 32)
        const size_t ls = g.N + (g.N == 32 ? 4 : 0);
        return sizeof(double2) * ((size_t)g.N + (size_t)reg_lines_per_cta(g.N) * ls);
    }
    return sizeof(double2) * (2 * (size_t)g.N + (size_t)buffers_for_mode(mode) * g.N * g.LP);
}

void prepare_line_pass(int mode, const LineGeom& g) {
    StepPtrs p{};
    dispatch(mode, g, p, 1, 0, true);
    twiddle_table(g.N);
    if (line_pass_smem_bytes(mode, g) > (size_t)kMaxSmem)
        throw Error(-2, "line pass tile does not fit in shared memory");
}

void launch_line_pass(int mode, const LineGeom& g, const StepPtrs& p, int nbatch, cudaStream_t st) {
    dispatch(mode, g, p, nbatch, st, false);
}

}  // namespace ps
