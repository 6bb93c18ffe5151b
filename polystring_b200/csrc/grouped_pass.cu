// grouped_pass.cu -- one launch runs the same line pass of step t for every
// active solve of a batch of independent Model_AB solves.  Each CTA finds its
// solve by a binary search over the per-solve CTA offsets, builds the solve's
// step pointers from its descriptor and t (the same pointers PairChain::enqueue
// gives the per-chain launches), and runs the line-pass body for that solve's
// line length; so every solve gets bit-for-bit the arithmetic of its own
// per-chain passes while a pass of the whole batch costs one launch.
#include "grouped_pass.h"
#include "line_pass_body.cuh"

namespace ps {

namespace {

using namespace lp;

__device__ __forceinline__ int find_solve(const int* __restrict__ prefix, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// PATH 0: Stockham body for every supported length; PATH 1 / 2: the
// register-resident body (lengths 32, 64, 128), compiled into separate
// kernels so that each keeps its own register budget
template <int MODE, int PATH>
__device__ __forceinline__ void dispatch_n(const LineGeom& g, const StepPtrs& p, const double2* tw, long tile, int fy) {
    if constexpr (PATH == 0) {
        switch (g.N) {
        case 16: line_pass_body<16, MODE>(g, p, tw, tile, fy, 0); break;
        case 24: line_pass_body<24, MODE>(g, p, tw, tile, fy, 0); break;
        case 32: line_pass_body<32, MODE>(g, p, tw, tile, fy, 0); break;
        case 48: line_pass_body<48, MODE>(g, p, tw, tile, fy, 0); break;
        case 64: line_pass_body<64, MODE>(g, p, tw, tile, fy, 0); break;
        case 96: line_pass_body<96, MODE>(g, p, tw, tile, fy, 0); break;
        case 128: line_pass_body<128, MODE>(g, p, tw, tile, fy, 0); break;
        default: break;   // rejected on the host (grouped_size_supported)
        }
    } else {
        switch (g.N) {
        case 32: line_pass_body_reg<32, MODE>(g, p, tw, tile, fy, 0); break;
        case 64: line_pass_body_reg<64, MODE>(g, p, tw, tile, fy, 0); break;
        case 128: line_pass_body_reg<128, MODE>(g, p, tw, tile, fy, 0); break;
        default: break;   // the host groups only register-capable lengths here
        }
    }
}

// factor set of a lane at step t
__device__ __forceinline__ int gset(const int* sw, int t) { return t < sw[0] ? 0 : (t < sw[1] ? 1 : 2); }

template <int MODE, int AX, int P3, int PATH>
__global__ void __launch_bounds__(kThreads, PATH == 2 ? 2 : 1)
    grouped_pass_kernel(const GroupSolve* __restrict__ solves, const int* __restrict__ prefix, int nactive, int t) {
    const int s = find_solve(prefix, nactive, blockIdx.x);
    const GroupSolve& D = solves[s];
    const int a = AX == GROUP_AX_IN ? 0 : (AX == GROUP_AX_MID ? 1 : D.naxes - 1);
    const LineGeom g = D.ax[a];
    const int local = blockIdx.x - prefix[s];
    const long nt = pass_tiles(g, MODE);
    const long tile = local % nt;
    const int fy = (int)(local / nt);
    const long M = (long)D.M;
    StepPtrs p{};
    p.M = D.M;
    p.bstride_z = M; p.bstride_u = M;
    p.u[0] = D.u[0]; p.u[1] = D.u[1];
    p.z[0] = D.z[0]; p.z[1] = D.z[1]; p.z[2] = D.z[2];
    p.L[0] = D.L1; p.L[1] = D.L2; p.L[2] = D.L2;
    p.qin[0] = D.hf + (long)t * M;
    p.qout[0] = D.hf + (long)(t + 1) * M;
    p.qin[1] = D.hc + (long)t * M;
    p.qout[1] = D.hc + (long)(t + 1) * M;
    const int sf = gset(D.swf, t), sc = gset(D.swc, t);
    p.eF[0] = D.fF[sf]; p.eF[1] = D.cF[sc];
    p.eH[0] = D.fH[sf]; p.eH[1] = D.cH[sc];
    if (t + 1 < D.Ns) {
        p.chain_next = 1;
        const int nf = gset(D.swf, t + 1), nc = gset(D.swc, t + 1);
        p.nF[0] = D.fF[nf]; p.nF[1] = D.cF[nc];
        p.nH[0] = D.fH[nf]; p.nH[1] = D.cH[nc];
    }
    p.nfield = P3 ? 1 : 2;
    if (P3) {
        p.z[0] = D.z[2];
        p.L[0] = D.L2;
    }
    dispatch_n<MODE, PATH>(g, p, D.tw[a], tile, fy);
}

template <int MODE, int AX, int P3, int PATH>
void launch_one(const GroupSolve* s, const int* prefix, int nactive, int nblocks, size_t smem, int t, cudaStream_t st,
                bool prepare) {
    if (prepare) {
        PS_CUDA(cudaFuncSetAttribute(grouped_pass_kernel<MODE, AX, P3, PATH>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLinePassSmemLimit));
        return;
    }
    grouped_pass_kernel<MODE, AX, P3, PATH><<<nblocks, kThreads, smem, st>>>(s, prefix, nactive, t);
    PS_CUDA(cudaGetLastError());
}

template <int MODE, int AX, int P3>
void launch_path(int path, const GroupSolve* s, const int* prefix, int nactive, int nblocks, size_t smem, int t,
                 cudaStream_t st, bool prepare) {
    if (path == 1) return launch_one<MODE, AX, P3, 1>(s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (path == 2) return launch_one<MODE, AX, P3, 2>(s, prefix, nactive, nblocks, smem, t, st, prepare);
    return launch_one<MODE, AX, P3, 0>(s, prefix, nactive, nblocks, smem, t, st, prepare);
}

void dispatch(int mode, int ax, int p3, int path, const GroupSolve* s, const int* prefix, int nactive, int nblocks,
              size_t smem, int t, cudaStream_t st, bool prepare) {
    if (mode == MODE_FIRST_RQM4 && ax == GROUP_AX_IN) return launch_path<MODE_FIRST_RQM4, 0, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (mode == MODE_MID_RQM4 && ax == GROUP_AX_IN) return launch_path<MODE_MID_RQM4, 0, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (mode == MODE_END_RQM4 && ax == GROUP_AX_IN) return launch_path<MODE_END_RQM4, 0, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (mode == MODE_FWD && ax == GROUP_AX_MID)
        return p3 ? launch_path<MODE_FWD, 1, 1>(path, s, prefix, nactive, nblocks, smem, t, st, prepare)
                  : launch_path<MODE_FWD, 1, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (mode == MODE_INV && ax == GROUP_AX_MID)
        return p3 ? launch_path<MODE_INV, 1, 1>(path, s, prefix, nactive, nblocks, smem, t, st, prepare)
                  : launch_path<MODE_INV, 1, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    if (mode == MODE_OUTER && ax == GROUP_AX_OUT)
        return p3 ? launch_path<MODE_OUTER, 2, 1>(path, s, prefix, nactive, nblocks, smem, t, st, prepare)
                  : launch_path<MODE_OUTER, 2, 0>(path, s, prefix, nactive, nblocks, smem, t, st, prepare);
    throw Error(-1, "no grouped pass for this mode and axis");
}

}  // namespace

bool grouped_size_supported(int N) {
    switch (N) {
    case 16: case 24: case 32: case 48: case 64: case 96: case 128: return true;
    default: return false;
    }
}

void grouped_prepare() {
    const int modes[][3] = {{MODE_FIRST_RQM4, 0, 0}, {MODE_MID_RQM4, 0, 0}, {MODE_END_RQM4, 0, 0},
                            {MODE_FWD, 1, 0},        {MODE_FWD, 1, 1},      {MODE_INV, 1, 0},
                            {MODE_INV, 1, 1},        {MODE_OUTER, 2, 0},    {MODE_OUTER, 2, 1}};
    for (auto& m : modes)
        for (int path = 0; path < 3; path++) dispatch(m[0], m[1], m[2], path, nullptr, nullptr, 0, 0, 0, 0, 0, true);
    for (int N : {16, 24, 32, 48, 64, 96, 128}) twiddle_table(N);
}

int grouped_ctas(const GroupSolve& s, int mode, int ax, int p3) {
    const int a = ax == GROUP_AX_IN ? 0 : (ax == GROUP_AX_MID ? 1 : s.naxes - 1);
    int gy = 1;
    if (mode == MODE_FIRST_RQM4 || mode == MODE_MID_RQM4) gy = 2;
    if (mode == MODE_FWD || mode == MODE_INV || mode == MODE_OUTER) gy = p3 ? 1 : 2;
    return (int)pass_tiles(s.ax[a], mode) * gy;
}

void grouped_launch(int mode, int ax, int p3, int path, const GroupSolve* solves_dev, const int* prefix_dev,
                    int nactive, int nblocks, size_t smem, int t, cudaStream_t st) {
    if (nactive <= 0 || nblocks <= 0) return;
    dispatch(mode, ax, p3, path, solves_dev, prefix_dev, nactive, nblocks, smem, t, st, false);
}

}  // namespace ps
