/*
 * polystring_b200.h -- C ABI of the B200 (sm_100a) implementation of
 * PolyOrder's periodic pseudospectral SCFT path.
 *
 * Plain C: opaque handles, pointers and sizes; no C++ or torch types.  Every
 * entry point returns PS_OK (0) or a negative status and never lets a C++
 * exception cross the boundary; ps_last_error() gives the message of the
 * last failure on the calling thread.
 *
 * Arrays are FP64, row-major (x, y, z) with z fastest, M = Lx*Ly*Lz points;
 * a propagator history is len consecutive slices of M (slice s at qs + s*M),
 * as Propagator stores _qs(len, Lx, Ly, Lz) (src/Propagator.cc:12-18).
 * 2D grids use Lz = 1, 1D grids Ly = Lz = 1.  Supported axis lengths: 1, 2,
 * 4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 352 (= 8 x 4 x 11, the
 * 128 x 352 grid of the reference's string example).
 *
 * Each context owns its device memory and one CUDA stream; a context is safe
 * to use from one host thread at a time.  "_device" entry points take device
 * pointers and a cudaStream_t passed as void* (NULL: the context's stream)
 * and return without synchronising; the others take host pointers and
 * return after the result is in host memory.
 *
 * Paths in the citations are relative to the reference project root.
 */
#ifndef POLYSTRING_B200_H
#define POLYSTRING_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define PS_OK 0
#define PS_ERR_INVALID (-1)      /* bad argument or cell                     */
#define PS_ERR_UNSUPPORTED (-2)  /* grid size / history length not supported */
#define PS_ERR_CUDA (-3)         /* CUDA runtime failure                     */
#define PS_ERR_QUADRATURE (-4)   /* contour rule precondition fails          */
#define PS_ERR_STATE (-6)        /* call out of order (e.g. H before update) */

/* ---- enumerations ---------------------------------------------------- */
/* MDE schemes, Config::algo_mde_type (src/Config.cc:1099-1111) */
#define PS_MDE_RQM4 0            /* "RQM4" / "OS4": src/RQM4.cc              */
#define PS_MDE_OS2 1             /* "OS2" / "PseudoSpectral": src/PseudoSpectral.cc */
#define PS_MDE_ETDRK4 2          /* "ETDRK4": src/Etdrk4_PBC.cc (Cox-Matthews) */
/* SCFT field update, Config::algo_scft_type (src/Config.cc:1219-1235) */
#define PS_SCFT_EM 0
#define PS_SCFT_ANDERSON 1
/* contour integration rules */
#define PS_CONTOUR_TRAPEZOID 0         /* Density::_update, src/Density.cc:107-121 */
#define PS_CONTOUR_SIMPSON 1           /* Simpson::solve, src/Simpson.cc:14-45     */
#define PS_CONTOUR_QUAD4_CLOSED 2      /* src/Quadrature4.cc:17-53                 */
#define PS_CONTOUR_QUAD4_OPEN 3        /* src/Quadrature4.cc:62-102                */
#define PS_CONTOUR_QUAD4_SEMIOPEN_LEFT 4  /* src/Quadrature4.cc:111-155            */
#define PS_CONTOUR_QUAD4_SEMIOPEN_RIGHT 5 /* src/Quadrature4.cc:164-197            */
/* crystal systems, UnitCell::calc_shape_matrix{1,2,3} (src/UnitCell.cc:149-296) */
#define PS_CELL_LAMELLAR 0
#define PS_CELL_SQUARE 1
#define PS_CELL_RECTANGULAR 2
#define PS_CELL_HEXAGONAL2 3
#define PS_CELL_OBLIQUE 4
#define PS_CELL_CUBIC 5
#define PS_CELL_TETRAGONAL 6
#define PS_CELL_ORTHORHOMBIC 7
#define PS_CELL_HEXAGONAL3 8
#define PS_CELL_TRIGONAL 9
#define PS_CELL_MONOCLINIC 10
#define PS_CELL_TRICLINIC 11
/* ps_model_ab_get / ps_model_ab_device_ptr: which array */
#define PS_FIELD_WA 0
#define PS_FIELD_WB 1
#define PS_FIELD_PHIA 2
#define PS_FIELD_PHIB 3
#define PS_FIELD_YITA 4
#define PS_FIELD_QA 5    /* sA slices */
#define PS_FIELD_QB 6    /* sB slices */
#define PS_FIELD_QAC 7   /* sA slices */
#define PS_FIELD_QBC 8   /* sB slices */

/* UnitCell parameters ([UnitCell] a, b, c, alpha, beta, gamma; angles in
 * radians), replacing UnitCell(const Config&) (include/UnitCell.h:39-98). */
typedef struct ps_unit_cell {
    int dim;
    int system;
    double a, b, c;
    double alpha, beta, gamma;
} ps_unit_cell;

typedef struct ps_updater ps_updater;
typedef struct ps_model_ab ps_model_ab;

const char* ps_version(void);
/* Tile schedules the line-pass autotuner chose in this process, one line per
 * tuned grid / scheme / batch (no counterpart in the reference).  Tuning runs
 * when a model or string context is created; PS_B200_AUTOTUNE=0 disables it. */
const char* ps_tuning_log(void);
const char* ps_last_error(void);
/* FP64 fused multiply-add throughput of the current GPU in TFLOP/s, timed
 * with CUDA events over a few launches of a kernel of independent FMA chains
 * on every SM (no counterpart in the reference; the denominator of the FP64
 * roofline fraction of the propagator sweeps).  Allocates and frees a small
 * buffer; synchronous. */
int ps_measure_fp64_peak(double* tflops);

/* ---- propagator updaters (the Updater interface, include/Updater.h:44-69) */

/* RQM4(const UnitCell&, Lx, Ly, Lz, ds)            src/RQM4.cc:9-16
 * PseudoSpectral(const UnitCell&, Lx, Ly, Lz, ds)  src/PseudoSpectral.cc:190-195
 * Etdrk4_PBC(const UnitCell&, Lx, Ly, Lz, ds)      src/Etdrk4_PBC.cc:12-24 (M = 32)
 * scheme = PS_MDE_RQM4, PS_MDE_OS2 or PS_MDE_ETDRK4.  ETDRK4 uses the
 * orthogonal k^2 table, as Etdrk4_PBC does. */
int ps_updater_create(int scheme, const ps_unit_cell* cell, int Lx, int Ly, int Lz, double ds,
                      ps_updater** out);
/* Etdrk4_PBC(const UnitCell&, Lx, Ly, Lz, ds, M)   include/Etdrk4_PBC.h:47-51:
 * M contour points for the coefficients (M >= 1). */
int ps_updater_create_etdrk4(const ps_unit_cell* cell, int Lx, int Ly, int Lz, double ds, int M,
                             ps_updater** out);
/* Updater::clone() (include/Updater.h:67) */
int ps_updater_clone(const ps_updater* u, ps_updater** out);
void ps_updater_destroy(ps_updater* u);
/* Updater::solve(Propagator& q, const Grid& w) (include/Updater.h:55;
 * src/RQM4.cc:41-93, src/PseudoSpectral.cc:226-261): qs[0] is the head on
 * entry; slices 1..len-1 are overwritten. */
int ps_updater_solve(ps_updater* u, const double* w, double* qs, int len);
int ps_updater_solve_device(ps_updater* u, const double* w, double* qs, int len, void* stream);

/* ---- density (Updater::solve(data, q, qc, cc), include/Updater.h:57-58) */
/* phi = cc * ds * sum_s c_s q[s] qc[len-1-s] with the weights of `rule`.
 * Returns PS_ERR_QUADRATURE when the rule's precondition fails (the
 * reference prints to cerr and leaves phi unchanged, src/Simpson.cc:18-26). */
int ps_density_solve(int rule, const double* q, const double* qc, int len, long long M, double ds, double cc,
                     double* phi);
int ps_density_solve_device(int rule, const double* q, const double* qc, int len, long long M, double ds,
                            double cc, double* phi, void* stream);
/* No counterpart in the reference.  ps_density_solve_device for callers that
 * cannot allocate device memory (a host program that owns all device memory
 * through its own pool, or a loop that cannot afford the synchronisation of
 * cudaMalloc / cudaFree): same arguments and result, but the contour-weight
 * table lives in a fixed device array compiled into the library, so nothing
 * is allocated.  len (contour points) may not exceed
 * PS_DENSITY_NOALLOC_MAX_LEN; larger values return PS_ERR_INVALID.  The first
 * call on a device looks up the table's device address on the current device
 * (and the first call after the device's context was reset, which reloads the
 * library's device code at a new address); make that first call before any
 * stream capture.  Asynchronous on `stream`.
 * All calls share one table per device: calls whose kernels may overlap on
 * the GPU (different streams with no ordering) race on it. */
#define PS_DENSITY_NOALLOC_MAX_LEN 8192
int ps_density_solve_device_noalloc(int rule, const double* q, const double* qc, int len, long long M, double ds,
                                    double cc, double* phi, void* stream);

/* Grid::quadrature on a regular grid: the mean (src/Grid.cc:329-374); with
 * a propagator slice this is Propagator::Q(s) (src/Propagator.cc:85-89). */
int ps_grid_mean_device(const double* x, long long M, double* out_host, void* stream);

/* ---- Model_AB: the whole SCFT iteration on the device ---------------- */
/* Fields of the reference's config file that Model_AB reads. */
typedef struct ps_model_ab_params {
    int dim, Lx, Ly, Lz;       /* [Grid] dimension, Lx, Ly, Lz                  */
    ps_unit_cell cell;         /* [UnitCell]                                    */
    int sA, sB;                /* [Algorithm_MDE] Ms                            */
    double chiN;               /* [Model] chiN                                  */
    double lamA, lamB, lamYita;/* [Algorithm_SCFT] lam                          */
    int mde;                   /* PS_MDE_*                                      */
    int scft;                  /* PS_SCFT_*                                     */
    int n_anderson;            /* [Algorithm_SCFT] n_Anderson_mixing (1..31)    */
    int compressible;          /* [Model] is_compressible                       */
    int contour;               /* 0 trapezoid, 1 Simpson (Simpson / Quad4_Closed
                                  by parity of Ms, src/Model_AB.cc:713-735)     */
    int etdrk4_M;              /* [Algorithm_MDE] etdrk4_M: ETDRK4 contour points;
                                  <= 0 gives Etdrk4_PBC's default 32
                                  (src/Model_AB.cc:746-763)                     */
} ps_model_ab_params;

/* Model_AB::init (src/Model_AB.cc:85-134) for a periodic cell */
int ps_model_ab_create(const ps_model_ab_params* p, ps_model_ab** out);
void ps_model_ab_destroy(ps_model_ab* m);
/* DATA_INIT fields (Model_AB::init_data_field, src/Model_AB.cc:672-675;
 * resetInString, :52-83): sets wA, wB, zeroes yita, restarts Anderson. */
int ps_model_ab_set_fields(ps_model_ab* m, const double* wA, const double* wB);
int ps_model_ab_set_fields_device(ps_model_ab* m, const double* wA, const double* wB);
/* n_iter x Model_AB::update (src/Model_AB.cc:136-261), the loop body of
 * scft::relax (src/scft.cc:395-397).  Asynchronous on the context stream. */
int ps_model_ab_update(ps_model_ab* m, int n_iter);
/* ps_model_ab_update with CUDA events on the context stream around the
 * whole run and around every propagator sweep; synchronises, then returns
 * the device time of the run and the summed sweep time, in milliseconds. */
int ps_model_ab_update_timed(ps_model_ab* m, int n_iter, double* total_ms, double* propagator_ms);
/* n_iter x the four Propagator::update calls of Model_AB::update only
 * (qA, qB, qBc, qAc; src/Model_AB.cc:187-193), no density or mixing. */
int ps_model_ab_propagate(ps_model_ab* m, int n_iter);
/* Model_AB::H / Hw / Hs (src/Model_AB.cc:263-300) */
int ps_model_ab_H(ps_model_ab* m, double* H, double* Hw, double* Hs);
/* Model_AB::residual_error (src/Model_AB.cc:307-371) */
int ps_model_ab_residual(ps_model_ab* m, double* res);
/* qB->Qt() of the last update (src/Model_AB.cc:195) */
int ps_model_ab_Q(ps_model_ab* m, double* Q);
/* Forward map at fixed fields: the four propagators, Q and both densities of
 * Model_AB::update (src/Model_AB.cc:186-199) without the field update.
 * Afterwards ps_model_ab_Q, ps_model_ab_H and ps_model_ab_get (PHIA, PHIB)
 * report the map's outputs. */
int ps_model_ab_forward(ps_model_ab* m);
/* Reverse mode of that map (RQM4, 2D/3D grids; no counterpart in the
 * reference, which has no derivatives): with the current fields, writes
 * dL/dwA and dL/dwB (M doubles each, host memory) for
 * L = sum_r (dL_dphiA phiA + dL_dphiB phiB) + dL_dQ Q, exact for the
 * discrete RQM4 chain and contour rule; the forward map is re-evaluated. */
int ps_model_ab_grad_w(ps_model_ab* m, const double* dL_dphiA, const double* dL_dphiB, double dL_dQ,
                       double* dL_dwA, double* dL_dwB);
/* Cell stress d(-ln Q)/dl_i at the current fields for the three cell
 * lengths l_i of the orthogonal k^2 table (UnitCell.cc:368-418; zero for
 * unused axes).  At an SCFT saddle point this is dF/dl, the derivative the
 * reference's Brent cell search (src/scft.cc:589-609) estimates from
 * converged free energies. */
int ps_model_ab_stress(ps_model_ab* m, double* dF_dl);
/* The same stress computed with the forward chain kept only at checkpoints
 * every k contour slices (k <= 0: ceil(sqrt(Ns))): the reverse sweep
 * recomputes one segment at a time, so the chain needs (Ns/k + k) slices of M
 * doubles instead of Ns + 1, for one extra forward pass. */
int ps_model_ab_stress_checkpointed(ps_model_ab* m, int k, double* dF_dl);
/* copy one array (PS_FIELD_*) to host memory */
int ps_model_ab_get(ps_model_ab* m, int which, double* out);
/* device address of one array (PS_FIELD_*), owned by the context */
int ps_model_ab_device_ptr(ps_model_ab* m, int which, double** out);
int ps_model_ab_synchronize(ps_model_ab* m);
/* kernel launches of one iteration / of one propagator sweep pair */
int ps_model_ab_launches_per_iteration(ps_model_ab* m);
int ps_model_ab_launches_per_propagate(ps_model_ab* m);
/* CUDA stream of the context (cudaStream_t as void*) */
void* ps_model_ab_stream(ps_model_ab* m);

/* ---- Model_ABC: a linear A-B-C triblock melt (no counterpart in the
 * reference, which has no periodic ABC melt model) -------------------------
 * Model_AB's steps with a third block and field: blocks of sA, sB, sC
 * contour points (ds = 1 / (sA + sB + sC - 3) up to rounding), Simpson or
 * Quad4_Closed by parity of each block's Ms, targets
 *   wA* = chiAB phiB + chiAC phiC + eta, wB* = chiAB phiA + chiBC phiC + eta,
 *   wC* = chiAC phiA + chiBC phiB + eta,
 * simple mixing with eta += lamYita (phiA + phiB + phiC - 1), or Anderson
 * mixing (one ring per field, one coefficient set) with
 *   eta = (wA + wB + wC - chiAB (phiA + phiB) - chiBC (phiB + phiC)
 *          - chiAC (phiA + phiC)) / 3;
 * H = mean(chiAB phiA phiB + chiBC phiB phiC + chiAC phiA phiC
 *          - wA phiA - wB phiB - wC phiC) - ln Q.
 * Incompressible, RQM4, orthogonal cells. */
typedef struct ps_model_abc_params {
    int dim, Lx, Ly, Lz;
    ps_unit_cell cell;
    int sA, sB, sC;
    double chiAB, chiBC, chiAC;            /* times N                         */
    double lamA, lamB, lamC, lamYita;
    int scft;                              /* PS_SCFT_*                       */
    int n_anderson;                        /* 1..31                           */
    int contour;                           /* 0 trapezoid, 1 Simpson / Quad4  */
} ps_model_abc_params;
typedef struct ps_model_abc ps_model_abc;
int ps_model_abc_create(const ps_model_abc_params* p, ps_model_abc** out);
void ps_model_abc_destroy(ps_model_abc* m);
int ps_model_abc_set_fields(ps_model_abc* m, const double* wA, const double* wB, const double* wC);
int ps_model_abc_update(ps_model_abc* m, int n_iter);
int ps_model_abc_Q(ps_model_abc* m, double* Q);
int ps_model_abc_H(ps_model_abc* m, double* H, double* Hw, double* Hs);
int ps_model_abc_residual(ps_model_abc* m, double* res);
/* which: 0..2 wA, wB, wC; 3..5 phiA, phiB, phiC; 6 eta (M values, host) */
int ps_model_abc_get(ps_model_abc* m, int which, double* out);
int ps_model_abc_synchronize(ps_model_abc* m);

/* ---- string method: all images of the string on the device ----------- */
typedef struct ps_string_ab ps_string_ab;
/* polystring_AB (scft/polystring_AB.cc:111-152) with m images of the model
 * in p (p->scft must be PS_SCFT_EM: images restart from DATA_INIT fields,
 * Model_AB.cc:52-83) and max_iter SCFT iterations per image per string
 * iteration ([Algorithm_SCFT] max_iter).  3 <= m <= 64.  H of images outside
 * a context's shard (ps_string_ab_create_shard) reads as NaN. */
int ps_string_ab_create(const ps_model_ab_params* p, int m, int max_iter, ps_string_ab** out);
void ps_string_ab_destroy(ps_string_ab* s);
/* initial string, m x M per field, image-major (initialize_string,
 * polystring_AB.cc:184-222); images 0 and m-1 are the fixed ends */
int ps_string_ab_set_images(ps_string_ab* s, const double* wa, const double* wb);
/* n string iterations: SCFT of every image (run_scftInString :256-281),
 * arc length (parameterize_string :283-296), per-point natural cubic spline
 * re-sampling and end restoration (redistribute_stringBeads :298-329) */
int ps_string_ab_iterate(ps_string_ab* s, int n);
/* H of every image after the last iteration (m values) */
int ps_string_ab_H(ps_string_ab* s, double* H);
/* normalised arc length of every image (m values) */
int ps_string_ab_S(ps_string_ab* s, double* S);
/* which: 0 wa, 1 wb, 2 phiA, 3 phiB; m x M values */
int ps_string_ab_get(ps_string_ab* s, int which, double* out);
int ps_string_ab_synchronize(ps_string_ab* s);
int ps_string_ab_launches_per_iteration(ps_string_ab* s);
/* The string with its images partitioned over processes (one per GPU): this
 * context holds the string fields of all m images but relaxes only images
 * lo <= s < hi (no counterpart in the reference, whose archived threaded
 * driver runs one std::thread per image, scft/polystring_AB_back/
 * polystring_AB_backThread.cc:256-258,412-423).  A sharded string iteration
 * is ps_string_ab_relax on every rank, an all-gather of the shards' wa and
 * wb (ps_string_ab_device_ptr), then ps_string_ab_reparameterize on every
 * rank (the same arithmetic everywhere, so the ranks keep identical strings).
 * ps_string_ab_iterate is the two in one graph and needs lo = 0, hi = m. */
int ps_string_ab_create_shard(const ps_model_ab_params* p, int m, int max_iter, int lo, int hi,
                              ps_string_ab** out);
/* run_scftInString (polystring_AB.cc:256-281) for the images of the shard:
 * fresh Yita, max_iter SCFT iterations, H.  Asynchronous on the context's
 * stream. */
int ps_string_ab_relax(ps_string_ab* s);
/* parameterize_string and redistribute_stringBeads (polystring_AB.cc:283-329)
 * over all m images: arc length, spline re-sampling, ends restored.
 * Asynchronous on the context's stream. */
int ps_string_ab_reparameterize(ps_string_ab* s);
/* device address of the m x M array `which` (0 wa, 1 wb, 2 phiA, 3 phiB) */
int ps_string_ab_device_ptr(ps_string_ab* s, int which, double** out);
/* CUDA stream of the context (cudaStream_t as void*) */
void* ps_string_ab_stream(ps_string_ab* s);

/* ---- independent solves of uneven grids and Ns, advanced together ------- */
/* The reference runs independent solves one per host thread
 * (scft/polystring_AB_backThread.cc).  A batch holds n Model_AB solves,
 * each with its own parameters p[k] (RQM4; 2D or 3D grids with axis lengths
 * 16, 24, 32, 48, 64, 96 or 128; Ms, chiN, cell, EM or Anderson may all
 * differ).  Each line pass of contour step t is one launch over every solve
 * that has a step t; one batch iteration (= one Model_AB::update of every
 * solve) is one CUDA graph.  Results equal those of each solve run alone on
 * the per-pass path. */
typedef struct ps_batch_ab ps_batch_ab;
int ps_batch_ab_create(const ps_model_ab_params* p, int n, ps_batch_ab** out);
/* A batch of n Model_AB solves (members 0 .. n-1) and nq linear ABC
 * triblock solves (members n .. n+nq-1, see ps_model_abc_params; 2D or 3D
 * grids; always on grouped line passes).  ps_batch_ab_H / _residual / _get
 * take either kind of member (_get with the ps_model_abc_get numbering for
 * ABC members). */
int ps_batch_ab_create_mixed(const ps_model_ab_params* p, int n, const ps_model_abc_params* q, int nq,
                             ps_batch_ab** out);
int ps_batch_ab_set_fields_abc(ps_batch_ab* b, int k, const double* wA, const double* wB, const double* wC);
void ps_batch_ab_destroy(ps_batch_ab* b);
int ps_batch_ab_set_fields(ps_batch_ab* b, int k, const double* wA, const double* wB);
int ps_batch_ab_update(ps_batch_ab* b, int n_iter);
/* update between CUDA events on the batch stream; device milliseconds */
int ps_batch_ab_update_timed(ps_batch_ab* b, int n_iter, double* total_ms);
int ps_batch_ab_H(ps_batch_ab* b, int k, double* H, double* Hw, double* Hs);
int ps_batch_ab_residual(ps_batch_ab* b, int k, double* res);
int ps_batch_ab_get(ps_batch_ab* b, int k, int which, double* out);
int ps_batch_ab_synchronize(ps_batch_ab* b);
int ps_batch_ab_launches_per_iteration(ps_batch_ab* b);
/* of them, the propagator launches (persistent sweeps and grouped line passes);
   the rest are the members' Q, density and field-update kernels */
int ps_batch_ab_launches_per_propagate(ps_batch_ab* b);
/* sum over solves of 2 Ns M: gridpoint contour steps of one batch iteration */
int ps_batch_ab_gridpoint_steps(ps_batch_ab* b, double* out);

#ifdef __cplusplus
}
#endif

#endif /* POLYSTRING_B200_H */
