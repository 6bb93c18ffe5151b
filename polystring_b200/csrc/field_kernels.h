// field_kernels.h -- launchers of the bandwidth-bound field kernels.
#pragma once

#include <cuda_runtime.h>

namespace ps {

constexpr int kRedBlocks = 296;   // 2 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kRedMaxK = 11;      // widest fixed reduction (triblock EM residual)

struct EMArgs {
    const double *phiA, *phiB;
    double *wA, *wB, *yita;
    long M;
    double chiN, lamA, lamB, lamYita, dsA, dsB;
    int compressible;
    double *eFA, *eHA, *eFB, *eHB;   // nullable: skip the factors
    long bstride;
};

// Model_ABC simple mixing (incompressible), fused with the next factors
struct EMABCArgs {
    const double* phi[3];
    double* w[3];
    double* yita;
    double* eF[3];
    double* eH[3];
    long M;
    double chi[3];   // chiAB, chiBC, chiAC (times N)
    double lam[4];   // lamA, lamB, lamC, lamYita
    double ds[3];
};

// out[0] = mean(x)
void launch_mean(const double* x, long M, double* partial, double* out, cudaStream_t st);
void launch_Hw(const double* phiA, const double* phiB, const double* wA, const double* wB, long M, double chiN,
               double lamYita, int compressible, double* partial, double* out, cudaStream_t st);
void launch_residual_em(const double* phiA, const double* phiB, const double* wA, const double* wB,
                        const double* yita, long M, double chiN, double lamYita, int compressible, double* partial,
                        double* out8, cudaStream_t st);
void launch_residual_ax(const double* dA, const double* dB, const double* wA, const double* wB, long M,
                        double* partial, double* out4, cudaStream_t st);
// Model_ABC reductions: Hw; EM residual sums (11); Anderson residual sums (6)
void launch_Hw_abc(const double* const phi[3], const double* const w[3], const double chi[3], long M,
                   double* partial, double* out, cudaStream_t st);
void launch_residual_em_abc(const double* const phi[3], const double* const w[3], const double* yita,
                            const double chi[3], long M, double* partial, double* out11, cudaStream_t st);
void launch_residual_ax_abc(const double* const d[3], const double* const w[3], long M, double* partial,
                            double* out6, cudaStream_t st);
void launch_em_update_abc(const EMABCArgs& a, cudaStream_t st);
void launch_arc_sq(const double* a, const double* b, long M, double* partial, double* out, cudaStream_t st);
void launch_density(const double* q, const double* qc, int n, long M, const double* c, double ds,
                    const double* Qdev, double cc_host, double* phi, int nbatch, long bstride_q, long bstride_phi,
                    const double* Qbatch, cudaStream_t st);
void launch_em_update(const EMArgs& a, int nbatch, cudaStream_t st);
void launch_factors(const double* wA, const double* wB, long M, double dsA, double dsB, double* eFA, double* eHA,
                    double* eFB, double* eHB, int nbatch, long bstride, cudaStream_t st);
void launch_fill(double* x, long n, double v, cudaStream_t st);

}  // namespace ps
