// engine.h -- host-side engine of the polystring_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "ps_internal.h"
#include "anderson.h"
#include "sweep.h"

namespace ps {

// RAII device array of doubles
struct DevBuf {
    double* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(size_t count);
    void release();
    double2* c() const { return reinterpret_cast<double2*>(p); }
};

// Unit cell (UnitCell.cc:149-296): reciprocal shape matrix g and lengths l
struct Cell {
    int dim = 3, system = 0;
    double a = 0, b = 0, c = 0, alpha = 0, beta = 0, gamma = 0;
    double g[9] = {0};
    double l[3] = {0};
};
void cell_init(Cell& c);   // throws on bad parameters

// -k^2 on an orthogonal cell (UnitCell.cc:368-418)
std::vector<double> k2_orthogonal(const Cell& c, int Lx, int Ly, int Lz);
// exp(-ds |q|^2), 27-image minimum (UnitCell.cc:321-359)
std::vector<double> k_laplacian(const Cell& c, int Lx, int Ly, int Lz, double ds);

// Line-pass plan of a grid: the axes longer than one, innermost first.
struct AxisPlan {
    int naxes = 0;
    LineGeom ax[3];
};
AxisPlan make_axis_plan(int Lx, int Ly, int Lz);
// tile of about `elems` elements: T lines, T a divisor of the line count
// (contiguous axis) or of the stride (outer axes)
void set_tile_elems(LineGeom& g, int elems);
// the tile choices of the autotuner so far, one line per tuned chain
const char* tuning_log();
void tuning_note(const char* line);   // appends one line to the tuning log

enum { SCHEME_RQM4 = 0, SCHEME_OS2 = 1, SCHEME_ETDRK4 = 2 };

// Which Boltzmann factors a lane uses at step t: set 0 before switch_t,
// set 1 from switch_t on (a chain crossing the A/B junction); a triblock
// chain (eF[2] set) uses set 2 from switch2 on.  switch_t may be negative
// (a step range that starts past the junction).
struct LaneFactors {
    const double* eF[3];
    const double* eH[3];
    int switch_t;
    int switch2;
    int set(int t) const { return t < switch_t ? 0 : (eF[2] && t >= switch2 ? 2 : 1); }
    const double* F(int t) const { return eF[set(t)]; }
    const double* H(int t) const { return eH[set(t)]; }
};

// One reverse sweep through a chain of Ns RQM4 steps (adjoint.cu).  Step t
// maps slice t to slice t + 1 of the history hq and runs in block blk[t]
// (0 = A, 1 = B).  lambda[Ns] = cst_Ns + (wd[0][Ns] pbarA + wd[1][Ns] pbarB)
// ho[0]; lambda[t] = A_t' lambda[t+1] + (wd[0][t] pbarA + wd[1][t] pbarB)
// ho[Ns - t].  The w-gradient of every step accumulates into grad[blk[t]].
struct AdjointSweep {
    int Ns;
    const double* hq;          // (Ns + 1) x M history of the chain
    const double* ho;          // (Ns + 1) x M history of the partner chain
    double* lam[2];            // two M buffers (ping-pong); lambda[0] ends in one
    const double* eF[2];       // e^{-w ds/2} of block A / B
    const double* eH[2];       // e^{-w ds/4}
    double* grad[2];           // accumulated w-gradient of block A / B
    double ds[2];
    const double* pbarA;       // direct terms (nullable: none)
    const double* pbarB;
    const int* blk;            // Ns entries
    const double* wd[2];       // Ns + 1 weights each
    double cst_Ns;
    double2* spec;             // 3 M spectra for the stress (nullable)
    double* stress_partial;    // Ns x 148 x 3
    double cl[3];              // 8 pi^2 / l^3 per axis (times the step's ds)
    // steps t_hi-1 .. t_lo of the sweep (t_hi = 0: all Ns); slice t of the
    // chain is at hq + (t - hq_base) M.  lambda[Ns] is set when t_hi = Ns;
    // lam_cur carries the ping-pong index from one range to the next.
    int t_lo, t_hi, hq_base, lam_cur;
};

// Work space and pass sequence for two real chains advanced together in one
// packed complex field.  Histories hold (nsteps + 1) slices of M doubles.
class PairChain {
public:
    PairChain(int Lx, int Ly, int Lz, int scheme, int nbatch);
    // RQM4: L1 = exp(ds k2), L2 = exp(ds k2 / 2); OS2: L1 = exp(-ds q^2)
    void set_tables(const std::vector<double>& L1, const std::vector<double>& L2);
    // batched tables: nbatch consecutive tables of M values each
    void set_tables_batched(const std::vector<double>& L1, const std::vector<double>& L2);
    // ETDRK4 (etdrk4.cu): E, E2, Q, f1, f2, f3 from the k2_orthogonal table,
    // Mc contour points (Etdrk4_PBC.cc:43-99)
    void set_tables_etd(const std::vector<double>& k2, double ds, int Mc);
    // c_in_fixed / c_out_fixed: lane c reads and writes fixed slices instead
    // of a history (single-chain solves).  ETDRK4: the factor slots of lf and
    // lc carry the fields w of each lane's blocks.
    void enqueue(double* hf, double* hc, long hist_bstride, int nsteps, const LaneFactors& lf,
                 const LaneFactors& lc, long fac_bstride, cudaStream_t st, const double* c_in_fixed = nullptr,
                 double* c_out_fixed = nullptr);
    // reverse sweep of one chain for the w-gradient and the cell stress (RQM4, 2D/3D)
    void enqueue_adjoint(AdjointSweep& s, cudaStream_t st);
    void prepare_adjoint();
    // choose each axis's tile height by timing whole contour steps (after set_tables*)
    void autotune(cudaStream_t st);
    // kernel launches per pair step
    int launches_per_step() const;
    long M() const { return M_; }
    const AxisPlan& plan() const { return plan_; }
    // work fields and tables (for grouped launches over many chains)
    double2* z(int i) const { return z_[i].c(); }
    double* u(int i) const { return u_[i].p; }
    const double* L1() const { return L1_.p; }
    const double* L2() const { return L2_.p; }

private:
    void enqueue_etd(double* hf, double* hc, int nsteps, const LaneFactors& lf, const LaneFactors& lc,
                     cudaStream_t st, const double* c_in_fixed, double* c_out_fixed);
    void transform(double2* z, int mode, cudaStream_t st) const;

    int Lx_, Ly_, Lz_, scheme_, nbatch_;
    long M_;
    AxisPlan plan_;
    DevBuf z_[3], u_[2], L1_, L2_, half_;
    DevBuf etd_, etdtab_;   // ETDRK4: V, Nv, A, Na, Nb (packed spectra); E, E2, Q, f1, f2, f3
    bool batched_tables_ = false;
};

// Model_AB on the device (Model_AB.cc:85-371 for a periodic cell)
struct ModelABParams {
    int dim, Lx, Ly, Lz;
    Cell cell;
    int sA, sB;
    double chiN, lamA, lamB, lamYita;
    int mde, scft, n_anderson, compressible, contour;
    int etd_M;   // ETDRK4 contour points (Etdrk4_PBC's M)
};

class ModelAB {
public:
    // batch_member: the propagators run in launches of a BatchAB (persistent
    // sweeps where the shape has one, else grouped line passes; no tile
    // tuning of its own)
    explicit ModelAB(const ModelABParams& p, bool batch_member = false);
    ~ModelAB();
    void set_fields(const double* wA, const double* wB, bool device_ptrs);
    void update(int n);
    // update() with CUDA events around the whole run and around every
    // propagator-graph replay; after synchronising returns the total device
    // time (ms) and sets *prop_ms to the summed propagator time
    double update_timed(int n, double* prop_ms);
    // replay only the propagator sweeps (the four Propagator::update calls)
    void propagate(int n);
    void H(double* H, double* Hw, double* Hs);
    double residual();
    double Q();
    void get(int which, double* out, bool device_dst);
    double* device_ptr(int which);
    void sync();
    cudaStream_t stream() const { return st_; }
    int launches_per_iteration() const { return launches_per_iter_; }
    int launches_per_propagate() const { return launches_per_prop_; }
    long M() const { return M_; }
    int Ns() const { return Ns_; }
    long iterations() const { return iter_; }
    int status();
    const ModelABParams& params() const { return p_; }
    bool persistent_sweep() const { return use_sweep_; }       // generic sweep (sweep.cu)
    bool persistent_sweep64() const { return use_sweep64_; }   // 64^3 sweep (sweep64.cu)
    // the generic sweep's arguments for this solve (its own pointers, batch
    // strides 0, its barrier words and error flag)
    SweepArgs sweep_descriptor() const;
    // the propagator sweeps of one iteration on stream s
    void enqueue_propagate(cudaStream_t s);
    // Adjoint of the forward map (wA, wB) -> (phiA, phiB, Q) at fixed fields:
    // forward_only() evaluates the map; grad_w() returns the gradient (per
    // point of M) of sum(phiA_bar phiA + phiB_bar phiB) + Q_bar Q with respect
    // to wA, wB; stress() returns d(-ln Q)/dl for the three cell lengths
    void forward_only();
    void grad_w(const double* phiA_bar, const double* phiB_bar, double Q_bar, double* gA, double* gB);
    void stress(double* dFdl);
    // the same stress with the forward chain kept only at checkpoints every
    // k slices (k <= 0: ceil(sqrt(Ns))), recomputed segment by segment during
    // the reverse sweep; (Ns/k + k + 4) M doubles instead of (Ns + 1) M
    void stress_checkpointed(int k, double* dFdl);
    // for BatchAB: the chain histories and factors, the post-propagator work
    // (Q, densities, field update) on a given stream, and the iteration count
    PairChain* chain() const { return chain_; }
    double* hist_f() const { return hf_.p; }
    double* hist_c() const { return hc_.p; }
    const double* factor(int full, int block) const {
        return full ? (block ? eFB_.p : eFA_.p) : (block ? eHB_.p : eHA_.p);
    }
    int LA() const { return LA_; }
    int LB() const { return LB_; }
    void enqueue_post(cudaStream_t s);
    void advance(int n) { iter_ += n; }
    bool has_fields() const { return fields_set_; }

private:
    void enqueue_propagate();
    void enqueue_post() { enqueue_post(st_); }
    void ensure_graphs();
    void init_anderson(const double* wA, const double* wB, bool device_ptrs);
    void tune_sweep();
    void adjoint_weights(std::vector<double>& wAf, std::vector<double>& wBf) const;
    void ensure_adjoint_buffers(bool spec);
    ModelABParams p_;
    long M_;
    int LA_, LB_, Ns_;
    double dsA_, dsB_;
    int ruleA_, ruleB_;
    PairChain* chain_ = nullptr;
    // persistent sweep (RQM4 on the shapes sweep_supported() lists)
    bool use_sweep_ = false;
    bool use_sweep64_ = false;
    int sweep_grid_ = 0;
    int sweep_variant_ = 0;              // x-tile variant of the generic sweep (tune_sweep)
    DevBuf swZ_, swU_, swL1_, swL2_, swTab_;
    unsigned* swbar_ = nullptr;
    int* swerr_ = nullptr;
    cudaStream_t st_ = nullptr;
    cudaGraphExec_t gprop_ = nullptr, gpost_ = nullptr;
    DevBuf hf_, hc_, wA_, wB_, yita_, phiA_, phiB_, eFA_, eHA_, eFB_, eHB_;
    DevBuf cA_, cB_, scal_, partial_;
    // Anderson
    DevBuf hwA_, hdA_, hwB_, hdB_, BA_, BB_;
    AXState* axs_ = nullptr;
    DevBuf lam_, gA_, gB_, pbA_, pbB_, spec_, stress_part_;
    DevBuf ck_, seg_, zero_, scratch_;   // checkpointed stress
    long iter_ = 0;
    bool fields_set_ = false;
    bool forward_done_ = false;   // Q, phi of the current fields are valid (forward_only)
    int launches_per_iter_ = 0;
    int launches_per_prop_ = 0;
};

// Linear A-B-C triblock melt on the device (model_abc.cu; no counterpart in
// the reference, which has no periodic ABC melt): Model_AB's steps with a
// third block and field, incompressible, RQM4.  The forward chain A -> B -> C
// and the complementary chain C -> B -> A share one packed field (three
// factor sets a lane, two switch steps); propagation runs the line passes.
struct ModelABCParams {
    int dim, Lx, Ly, Lz;
    Cell cell;
    int s[3];         // Ms of blocks A, B, C
    double chi[3];    // chiAB, chiBC, chiAC (times N)
    double lam[4];    // lamA, lamB, lamC, lamYita
    int scft, n_anderson, contour;
};

class ModelABC {
public:
    explicit ModelABC(const ModelABCParams& p);
    ~ModelABC();
    // w: three fields of M values (host or device)
    void set_fields(const double* const w[3], bool device_ptrs);
    void update(int n);
    void enqueue_iteration(cudaStream_t st);   // one iteration on stream st (fields set)
    double Q();
    void H(double* H, double* Hw, double* Hs);
    double residual();
    // 0..2 wA, wB, wC; 3..5 phiA, phiB, phiC; 6 yita
    void get(int which, double* out, bool device_dst);
    int status();
    long M() const { return M_; }
    int Ns() const { return Ns_; }
    int L(int x) const { return L_[x]; }
    cudaStream_t stream() const { return st_; }
    void count_iterations(int n) { iter_ += n; }
    bool has_fields() const { return fields_set_; }
    // for batches (batch_ab.cu): the packed chain, histories and factors
    PairChain* chain() const { return chain_; }
    double* hist_f() const { return hf_.p; }
    double* hist_c() const { return hc_.p; }
    const double* factor(int full, int block) const { return full ? eF_[block].p : eH_[block].p; }
    void enqueue_propagate(cudaStream_t s);
    void enqueue_post(cudaStream_t s);
    int launches_post() const { return 2 + 3 + (p_.scft == 1 ? 4 : 1); }
    // the generic persistent sweep (32^3, 48^3 grids; 64^3 where the 64^3
    // sweep cannot run) with three factor sets
    bool persistent_sweep() const { return use_sweep_; }
    // the 64^3 sweep (sweep64.cu) with three factor sets
    bool persistent_sweep64() const { return use_sweep64_; }
    SweepArgs sweep_descriptor() const;
    const ModelABCParams& params() const { return p_; }

private:

    ModelABCParams p_;
    long M_;
    int L_[3], Ns_;
    double ds_[3];
    PairChain* chain_ = nullptr;
    cudaStream_t st_ = nullptr;
    DevBuf hf_, hc_, w_[3], yita_, phi_[3], eF_[3], eH_[3], c_[3], scal_, partial_;
    DevBuf hw_[3], hd_[3], B_[3];
    AXState* axs_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    long iter_ = 0;
    bool fields_set_ = false;
    bool use_sweep_ = false;
    bool use_sweep64_ = false;
    int sweep_grid_ = 0;
    DevBuf swZ_, swU_, swL1_, swL2_, swTab_;
    unsigned* swbar_ = nullptr;
    int* swerr_ = nullptr;
};

// Single propagator updater behind the Updater C-ABI (RQM4 / OS2 / ETDRK4)
class UpdaterCtx {
public:
    UpdaterCtx(int scheme, const Cell& cell, int Lx, int Ly, int Lz, double ds, int etd_M = 32);
    ~UpdaterCtx();
    UpdaterCtx* clone() const;
    void solve_device(const double* w, double* qs, int len, cudaStream_t st);
    void solve_host(const double* w, double* qs, int len);
    int scheme() const { return scheme_; }

private:
    int scheme_, Lx_, Ly_, Lz_;
    Cell cell_;
    double ds_;
    int etd_M_;
    long M_;
    PairChain* chain_ = nullptr;
    DevBuf eF_, eH_, zero_, scratch_, dw_, dqs_;
    cudaStream_t st_ = nullptr;
};

// contour weights c_s of a rule (Simpson.cc, Quadrature4.cc, Density.cc);
// returns false when the rule's precondition fails
bool contour_weights(int rule, int n, std::vector<double>& c);

}  // namespace ps
