// grouped_pass.h -- line passes of many independent propagator solves (of
// different grids, contour lengths and block fractions) in one launch each.
#pragma once

#include "ps_internal.h"

namespace ps {

// One solve of a grouped launch: the paired chains of one Model_AB (lane f:
// qA -> qB, lane c: qBc -> qAc) or Model_ABC (lane f: qA -> qB -> qC, lane c:
// qCc -> qBc -> qAc), its work fields and tables, and its line geometry.
// Step t of the solve reads slice t of the histories and writes slice t + 1;
// a lane uses its factor set 0 for t < sw[0], set 1 for t < sw[1], then set 2.
struct GroupSolve {
    LineGeom ax[3];
    int naxes, Ns;
    int swf[2], swc[2];         // switch steps of lane f and lane c
    double M;
    double* hf;
    double* hc;
    double2* z[3];
    double* u[2];
    const double* L1;
    const double* L2;
    const double* fF[3];        // lane f: e^{-w ds/2} of its blocks in chain order
    const double* fH[3];        // lane f: e^{-w ds/4}
    const double* cF[3];        // lane c
    const double* cH[3];
    const double2* tw[3];       // twiddles of each axis
};

// axis role of a pass: 0 = innermost (FIRST / MID / END), 1 = middle axis of
// a 3D grid, 2 = outermost (OUTER)
enum { GROUP_AX_IN = 0, GROUP_AX_MID = 1, GROUP_AX_OUT = 2 };

bool grouped_size_supported(int N);
void grouped_prepare();
// CTAs of one solve in a pass of `mode` on axis role `ax` (p3: the single
// field of the second half step)
int grouped_ctas(const GroupSolve& s, int mode, int ax, int p3);
// one grouped pass over solves[0 .. nactive): block b belongs to solve k when
// prefix[k] <= b < prefix[k + 1]; smem = the largest tile any of them needs
// path: the schedule of the pass's axis in every solve of the launch (LineGeom::reg; 1 and 2 only
// for lengths 32, 64, 128)
void grouped_launch(int mode, int ax, int p3, int path, const GroupSolve* solves_dev, const int* prefix_dev,
                    int nactive, int nblocks, size_t smem, int t, cudaStream_t st);

}  // namespace ps
