// anderson.h -- device-resident Anderson mixing state and launcher.
#pragma once

#include <cuda_runtime.h>

namespace ps {

constexpr int kAXMaxHist = 32;

// Ring bookkeeping of FieldAX (FieldAX.h:95-143), shared by the A and B
// fields, which are always updated together.
struct AXState {
    int n;          // history length
    int k;          // iterations performed
    int cur;        // cur_pos
    int cur_old;    // cur_pos before the last update (slot of the newest d)
    int cur_new;    // cur_pos after the last update
    int nc;         // number of mixing coefficients used by the last update
    int status;     // bit 0: singular U met (C set to 0)
    int pad;
    double lamA, lamB;    // FieldAX::_lambda of A and B
    double rampA, rampB;  // 1 - lambda^(k+1) of the last update
    double C[kAXMaxHist];
    double lamC, rampC;   // the third field of a triblock (Model_ABC)
};

struct AXArgs {
    AXState* state;
    int n;
    long M;
    const double *phiA, *phiB;
    double *dataA, *dataB;       // current fields (Grid::_data)
    double *wA, *dA, *wB, *dB;   // histories, (n+1) x M each
    double *BA, *BB;             // (n+1) x (n+1)
    double* yita;                // incompressible: 0.5 (wA + wB - chiN)
    double chiN, lamYita, dsA, dsB;
    int compressible;
    double *eFA, *eHA, *eFB, *eHB;   // next Boltzmann factors (nullable)
    // three fields (Model_ABC): nf = 3, field C and the pair interactions
    // chi = (chiAB, chiBC, chiAC) N; eta = (wA + wB + wC - chiAB (phiA + phiB)
    // - chiBC (phiB + phiC) - chiAC (phiA + phiC)) / 3 (incompressible only)
    int nf;                          // 0 or 2: A and B; 3: A, B, C
    const double* phiC;
    double *dataC, *wC, *dC, *BC;
    double dsC;
    double *eFC, *eHC;
    double chi[3];
};

int ax_nmax(int n);
// partial: kRedBlocks x 64 doubles of scratch (x 96 with three fields)
void launch_anderson(const AXArgs& a, double* partial, cudaStream_t st);

}  // namespace ps
