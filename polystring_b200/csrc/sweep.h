// sweep.h -- persistent cooperative RQM4 sweep of a paired chain.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace ps {

struct SweepArgs {
    double *hf, *hc;                 // histories, (Ns + 1) x M each (slice 0 = head)
    double2 *Z1, *Z2, *Z3;           // packed complex work fields, M each
    double *uf, *uc;                 // full-step results, M each
    const double *eFA, *eHA, *eFB, *eHB;   // Boltzmann factors of the A and B blocks
    const double *L1, *L2;           // exp(ds k2), exp(ds k2 / 2)
    const double2 *twx, *twy, *twz;  // twiddles (set by the launcher)
    int LA, LB, Ns;
    unsigned* bar;                   // one barrier counter per problem (stride 32), zeroed per launch
    int* err;                        // nonzero after a barrier timeout
    long bstride_batch;              // per-problem stride of M-sized arrays
    long bstride_hist;               // per-problem stride of the histories
    long bstride_L;                  // per-problem stride of the k tables (0: shared)
    const double* ktab;              // cluster sweep: per-axis exp(h k_x^2), exp(h k_y^2), h = ds then ds/2
    // linear A-B-C triblock (generic sweep only; eFC == nullptr: diblock):
    // lane f runs A, B, C switching at LA and LA + LB; lane c runs C, B, A
    // switching at LC and LC + LB
    const double *eFC, *eHC;
    int LC;
};

bool sweep_supported(int Lx, int Ly, int Lz);
// 64^3 specialisation (sweep64.cu); uses hf, hc, Z1-Z3, eHA, eHB, LA, LB,
// Ns, bar (64 zeroed words) and err; tables = 6 x 64 per-axis k factors
bool sweep64_supported(int Lx, int Ly, int Lz);
// sets kernel attributes, builds twiddles; returns the grid (two-CTA clusters,
// one CTA per SM), or 0 when too few clusters can be resident on this device
int sweep64_prepare();
// the sweep's per-axis k-space factors exp(h cc_axis r^2) of a 64^3 grid on an
// orthogonal cell of lengths l, h = ds (full step) then ds / 2: 6 x 64 doubles
std::vector<double> sweep64_axis_tables(const double l[3], double ds);
void sweep64_launch(const SweepArgs& a, const double* tables, int grid, cudaStream_t st);
// sets kernel attributes, builds twiddles; returns the cooperative grid size
int sweep_prepare(int Lx, int Ly, int Lz);
// x-tile variants of the single-solve sweep (same arithmetic, different
// tile widths): the autotuner's choices; sweep_default_variant is the one used
// untuned; sweep_xtile_columns the columns of an x tile of a variant
constexpr int kSweepVariants = 3;
int sweep_default_variant(int Lx, int Ly, int Lz);
int sweep_xtile_columns(int Lx, int Ly, int Lz, int variant);
void sweep_launch(const SweepArgs& a, int Lx, int Ly, int Lz, int grid, int nbatch, cudaStream_t st, int variant);
// Independent problems of one shape in one cooperative launch: d (device
// memory) holds n descriptors with their own pointers (batch strides 0, bar =
// 32 zeroed words each), per CTAs work on each problem (per * n must not
// exceed sweep_desc_prepare's count of resident CTAs).  Problem k runs
// d[k].Ns steps; the twiddle pointers come from twiddle_table.
int sweep_desc_prepare(int Lx, int Ly, int Lz);
// plane tasks / x tiles of the busiest phase: CTAs one problem can keep busy
int sweep_tasks_per_phase(int Lx, int Ly, int Lz);
// rounds of tasks per contour step (two x-passes, two plane phases) when one
// problem has per CTAs: the step time in units of a task
int sweep_rounds_per_step(int Lx, int Ly, int Lz, int per);
void sweep_launch_desc(const SweepArgs* d, int Lx, int Ly, int Lz, int per, int n, cudaStream_t st);
// batches of 2D problems, one thread-block cluster per problem (cluster_sweep.cu):
// uses hf, hc, the factors, ktab (2 (Lx + Ly) doubles), LA, LB, Ns and the
// batch strides of SweepArgs
bool cluster_sweep_supported(int Lx, int Ly, int Lz);
// sets kernel attributes, builds twiddles; returns how many clusters fit at once
int cluster_sweep_prepare(int Lx, int Ly, int Lz, int nbatch);
void cluster_sweep_launch(const SweepArgs& a, int Lx, int Ly, int Lz, int nbatch, cudaStream_t st);

}  // namespace ps
