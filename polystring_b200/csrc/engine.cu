// engine.cu -- pass sequencing, k-space tables, the Model_AB device context
// (one SCFT iteration captured once as a CUDA graph and replayed), and the
// single-propagator Updater context.
#include "engine.h"
#include "field_kernels.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

namespace ps {

// ---------------------------------------------------------------------------
// DevBuf
// ---------------------------------------------------------------------------
void DevBuf::alloc(size_t count) {
    release();
    if (count == 0) return;
    PS_CUDA(cudaMalloc(&p, sizeof(double) * count));
    n = count;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
}

// ---------------------------------------------------------------------------
// unit cell and k tables
// ---------------------------------------------------------------------------
static void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// UnitCell::calc_shape_matrix{1,2,3} (UnitCell.cc:149-296)
void cell_init(Cell& c) {
    const double PI = 3.14159265358979323846;
    const double pi2 = PI / 2.0, pi3 = 2.0 * PI / 3.0, twopi = 2.0 * PI;
    std::memset(c.g, 0, sizeof(c.g));
    double a = c.a, b = c.b, cc = c.c, alpha = c.alpha, beta = c.beta, gamma = c.gamma;
    if (c.dim == 1) {
        if (a <= 0) throw Error(-1, "bad cell parameters (1D)");
        c.l[0] = a; c.l[1] = 0; c.l[2] = 0;
        c.g[0] = twopi / a; c.g[4] = twopi; c.g[8] = twopi;
        return;
    }
    if (c.dim == 2) {
        if (a <= 0) throw Error(-1, "bad cell parameters (2D)");
        switch (c.system) {
        case 1: b = a; gamma = pi2; break;                                  // SQUARE
        case 2: if (b <= 0) throw Error(-1, "bad RECTANGULAR cell"); gamma = pi2; break;
        case 3: b = a; gamma = pi3; break;                                  // HEXAGONAL
        default: if (b <= 0 || gamma <= 0) throw Error(-1, "bad 2D cell"); break;
        }
        double va[3] = {a, 0, 0}, vb[3] = {b * cos(gamma), b * sin(gamma), 0};
        c.l[0] = a; c.l[1] = b; c.l[2] = 0;
        double acb[3], t[3], as[3], bs[3];
        cross3(va, vb, acb);
        double denom = dot3(acb, acb);
        cross3(vb, acb, t); for (int i = 0; i < 3; i++) as[i] = t[i] / denom;
        cross3(acb, va, t); for (int i = 0; i < 3; i++) bs[i] = t[i] / denom;
        c.g[0] = twopi * as[0]; c.g[1] = twopi * bs[0];
        c.g[3] = twopi * as[1]; c.g[4] = twopi * bs[1];
        c.g[8] = twopi;
        return;
    }
    switch (c.system) {
    case 5: b = a; cc = a; alpha = beta = gamma = pi2; break;   // CUBIC
    case 6: b = a; alpha = beta = gamma = pi2; break;           // TETRAGONAL
    case 7: alpha = beta = gamma = pi2; break;                  // ORTHORHOMBIC
    case 8: b = a; alpha = pi2; beta = pi2; gamma = pi3; break; // HEXAGONAL
    case 9: b = a; cc = a; alpha = gamma; beta = gamma; break;  // TRIGONAL
    case 10: alpha = pi2; gamma = pi2; break;                   // MONOCLINIC
    case 11: break;                                             // TRICLINIC
    default: throw Error(-1, "unknown crystal system");
    }
    if (a <= 0 || b <= 0 || cc <= 0) throw Error(-1, "bad 3D cell");
    double va[3] = {a, 0, 0}, vb[3] = {b * cos(gamma), b * sin(gamma), 0};
    double cx = cc * cos(beta), cy = cc * (cos(alpha) - cos(beta) * cos(gamma));
    double cz = sqrt(cc * cc - cx * cx - cy * cy);
    double vc[3] = {cx, cy, cz};
    c.l[0] = a; c.l[1] = b; c.l[2] = cc;
    double bcc[3], cca[3], acb[3];
    cross3(vb, vc, bcc); cross3(vc, va, cca); cross3(va, vb, acb);
    double denom = dot3(va, bcc);
    for (int i = 0; i < 3; i++) {
        c.g[3 * i + 0] = twopi * (bcc[i] / denom);
        c.g[3 * i + 1] = twopi * (cca[i] / denom);
        c.g[3 * i + 2] = twopi * (acb[i] / denom);
    }
}

std::vector<double> k2_orthogonal(const Cell& c, int Lx, int Ly, int Lz) {
    const double PI = 3.14159265358979323846;
    double ccx = 0, ccy = 0, ccz = 0;
    if (c.dim >= 1) ccx = -4.0 * PI * PI / (c.l[0] * c.l[0]);
    if (c.dim >= 2) ccy = -4.0 * PI * PI / (c.l[1] * c.l[1]);
    if (c.dim >= 3) ccz = -4.0 * PI * PI / (c.l[2] * c.l[2]);
    std::vector<double> k2((size_t)Lx * Ly * Lz);
    for (int i = 0; i < Lx; i++)
        for (int j = 0; j < Ly; j++)
            for (int k = 0; k < Lz; k++) {
                int ri = (i < Lx / 2 + 1) ? i : Lx - i;
                int rj = (j < Ly / 2 + 1) ? j : Ly - j;
                int rk = (k < Lz / 2 + 1) ? k : Lz - k;
                k2[((size_t)i * Ly + j) * Lz + k] = ccx * ri * ri + ccy * rj * rj + ccz * rk * rk;
            }
    return k2;
}

std::vector<double> k_laplacian(const Cell& c, int Na, int Nb, int Nc, double ds) {
    std::vector<double> out((size_t)Na * Nb * Nc);
    for (int i = 0; i < Na; i++)
        for (int j = 0; j < Nb; j++)
            for (int k = 0; k < Nc; k++) {
                double q2min = 1.0e300;
                for (int ii = 1; ii > -2; ii--)
                    for (int jj = 1; jj > -2; jj--)
                        for (int kk = 1; kk > -2; kk--) {
                            double bq[3] = {(double)(ii * Na) + i, (double)(jj * Nb) + j, (double)(kk * Nc) + k};
                            double qt[3];
                            for (int r = 0; r < 3; r++)
                                qt[r] = c.g[3 * r + 0] * bq[0] + c.g[3 * r + 1] * bq[1] + c.g[3 * r + 2] * bq[2];
                            double q2 = dot3(qt, qt);
                            if (q2 < q2min) q2min = q2;
                        }
                out[((size_t)i * Nb + j) * Nc + k] = exp(-ds * q2min);
            }
    return out;
}

// ---------------------------------------------------------------------------
// axis plan
// ---------------------------------------------------------------------------
static int largest_divisor_le(long n, long cap) {
    if (cap < 1) cap = 1;
    for (long t = std::min(n, cap); t >= 1; t--)
        if (n % t == 0) return (int)t;
    return 1;
}

void set_tile_elems(LineGeom& g, int elems) {
    const int lpc = reg_lines_per_cta(g.N);
    g.rtiles = lpc > 0 ? (g.nlines + lpc - 1) / lpc : 0;
    const long target = std::max(1, elems / g.N);
    g.T = (g.S == 1) ? largest_divisor_le(g.nlines, target) : largest_divisor_le(g.S, target);
    g.LP = (g.S == 1 && g.T % 2 == 0) ? g.T + 1 : g.T;
    g.ntiles = g.nlines / g.T;
    g.tshift = -1;
    for (int b = 0; b < 12; b++)
        if ((1 << b) == g.T) g.tshift = b;
}

AxisPlan make_axis_plan(int Lx, int Ly, int Lz) {
    AxisPlan ap;
    const long M = (long)Lx * Ly * Lz;
    const int sizes[3] = {Lz, Ly, Lx};
    const long strides[3] = {1, (long)Lz, (long)Ly * Lz};
    for (int a = 0; a < 3; a++) {
        int N = sizes[a];
        if (N <= 1) continue;
        if (!line_size_supported(N))
            throw Error(-2, "unsupported grid size " + std::to_string(N) +
                                " (supported: 2, 4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 352)");
        LineGeom g;
        g.N = N;
        g.S = strides[a];
        g.nlines = M / N;
        set_tile_elems(g, 2048);
        // default schedule: Stockham passes (fastest in the measurements made
        // so far); the autotuner tries the register-resident four-step where
        // the length supports it; PS_B200_REG_FFT=0/1/2 forces a schedule
        const char* rf = getenv("PS_B200_REG_FFT");
        g.reg = 0;
        if (rf && rf[0] >= '0' && rf[0] <= '2' && reg_lines_per_cta(N) > 0) g.reg = rf[0] - '0';
        ap.ax[ap.naxes++] = g;
    }
    if (ap.naxes == 0) throw Error(-2, "grid has no axis longer than one point");
    return ap;
}

// ---------------------------------------------------------------------------
// PairChain
// ---------------------------------------------------------------------------
PairChain::PairChain(int Lx, int Ly, int Lz, int scheme, int nbatch)
    : Lx_(Lx), Ly_(Ly), Lz_(Lz), scheme_(scheme), nbatch_(nbatch) {
    M_ = (long)Lx * Ly * Lz;
    plan_ = make_axis_plan(Lx, Ly, Lz);
    const int nz = (scheme == SCHEME_RQM4) ? 3 : 1;
    for (int i = 0; i < nz; i++) z_[i].alloc(2 * (size_t)M_ * nbatch);
    if (scheme == SCHEME_RQM4) {
        u_[0].alloc((size_t)M_ * nbatch);
        u_[1].alloc((size_t)M_ * nbatch);
    }
    // attributes and twiddles before any capture
    const LineGeom& in = plan_.ax[0];
    if (scheme == SCHEME_ETDRK4) {
        if (nbatch != 1) throw Error(-2, "ETDRK4 chains are not batched");
        etd_.alloc(10 * (size_t)M_);
        for (int a = 0; a < plan_.naxes; a++) {
            prepare_line_pass(MODE_FWD, plan_.ax[a]);
            prepare_line_pass(MODE_INV, plan_.ax[a]);
        }
    } else if (plan_.naxes == 1) {
        prepare_line_pass(scheme == SCHEME_RQM4 ? MODE_FULL_RQM4 : MODE_FULL_OS2, in);
    } else {
        const LineGeom& out = plan_.ax[plan_.naxes - 1];
        if (scheme == SCHEME_RQM4) {
            prepare_line_pass(MODE_FIRST_RQM4, in);
            prepare_line_pass(MODE_MID_RQM4, in);
            prepare_line_pass(MODE_END_RQM4, in);
        } else {
            prepare_line_pass(MODE_FIRST_OS2, in);
            prepare_line_pass(MODE_END_OS2, in);
        }
        prepare_line_pass(MODE_OUTER, out);
        if (plan_.naxes == 3) {
            prepare_line_pass(MODE_FWD, plan_.ax[1]);
            prepare_line_pass(MODE_INV, plan_.ax[1]);
        }
    }
}

void PairChain::set_tables(const std::vector<double>& L1, const std::vector<double>& L2) {
    L1_.alloc(M_);
    PS_CUDA(cudaMemcpy(L1_.p, L1.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
    if (scheme_ == SCHEME_RQM4) {
        L2_.alloc(M_);
        PS_CUDA(cudaMemcpy(L2_.p, L2.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
    }
    batched_tables_ = false;
}

void PairChain::set_tables_batched(const std::vector<double>& L1, const std::vector<double>& L2) {
    L1_.alloc((size_t)M_ * nbatch_);
    PS_CUDA(cudaMemcpy(L1_.p, L1.data(), sizeof(double) * M_ * nbatch_, cudaMemcpyHostToDevice));
    if (scheme_ == SCHEME_RQM4) {
        L2_.alloc((size_t)M_ * nbatch_);
        PS_CUDA(cudaMemcpy(L2_.p, L2.data(), sizeof(double) * M_ * nbatch_, cudaMemcpyHostToDevice));
    }
    batched_tables_ = true;
}

int PairChain::launches_per_step() const {
    // slices, 4 x (forward transform, combine, inverse transform), 3 nonlinear terms, store
    if (scheme_ == SCHEME_ETDRK4) return 1 + 4 * (2 * plan_.naxes + 1) + 3 + 1;
    if (plan_.naxes == 1) return 1;
    if (scheme_ == SCHEME_RQM4) return plan_.naxes == 3 ? 8 : 4;
    return plan_.naxes == 3 ? 4 : 2;
}

void PairChain::enqueue(double* hf, double* hc, long hist_bstride, int nsteps, const LaneFactors& lf,
                        const LaneFactors& lc, long fac_bstride, cudaStream_t st, const double* c_in_fixed,
                        double* c_out_fixed) {
    const long M = M_;
    StepPtrs base{};
    base.M = (double)M;
    base.bstride_z = M;         // in double2 elements
    base.bstride_q = hist_bstride;
    base.bstride_u = M;
    base.bstride_e = fac_bstride;
    base.bstride_L = batched_tables_ ? M : 0;
    base.u[0] = u_[0].p;
    base.u[1] = u_[1].p;
    const int na = plan_.naxes;
    const LineGeom& in = plan_.ax[0];
    const LineGeom& out = plan_.ax[na - 1];
    const LineGeom* mid = (na == 3) ? &plan_.ax[1] : nullptr;
    const bool rq = (scheme_ == SCHEME_RQM4);
    if (scheme_ == SCHEME_ETDRK4) {
        if (hist_bstride != 0 || fac_bstride != 0) throw Error(-2, "ETDRK4 chains are not batched");
        enqueue_etd(hf, hc, nsteps, lf, lc, st, c_in_fixed, c_out_fixed);
        return;
    }

    for (int t = 0; t < nsteps; t++) {
        StepPtrs p = base;
        p.z[0] = z_[0].c(); p.z[1] = rq ? z_[1].c() : nullptr; p.z[2] = rq ? z_[2].c() : nullptr;
        p.L[0] = L1_.p; p.L[1] = rq ? L2_.p : nullptr; p.L[2] = p.L[1];
        p.qin[0] = hf + (long)t * M;
        p.qout[0] = hf + (long)(t + 1) * M;
        if (c_in_fixed) {
            p.qin[1] = c_in_fixed;
            p.qout[1] = c_out_fixed;
        } else {
            p.qin[1] = hc + (long)t * M;
            p.qout[1] = hc + (long)(t + 1) * M;
        }
        p.eF[0] = lf.F(t); p.eF[1] = lc.F(t);
        p.eH[0] = lf.H(t); p.eH[1] = lc.H(t);
        if (t + 1 < nsteps) {
            p.chain_next = 1;
            p.nF[0] = lf.F(t + 1); p.nF[1] = lc.F(t + 1);
            p.nH[0] = lf.H(t + 1); p.nH[1] = lc.H(t + 1);
        }
        if (na == 1) {
            p.nfield = 1;
            launch_line_pass(rq ? MODE_FULL_RQM4 : MODE_FULL_OS2, in, p, nbatch_, st);
            continue;
        }
        if (rq) {
            if (t == 0) launch_line_pass(MODE_FIRST_RQM4, in, p, nbatch_, st);
            p.nfield = 2;
            if (mid) launch_line_pass(MODE_FWD, *mid, p, nbatch_, st);
            launch_line_pass(MODE_OUTER, out, p, nbatch_, st);
            if (mid) launch_line_pass(MODE_INV, *mid, p, nbatch_, st);
            launch_line_pass(MODE_MID_RQM4, in, p, nbatch_, st);
            StepPtrs p3 = p;
            p3.nfield = 1;
            p3.z[0] = z_[2].c();
            p3.L[0] = L2_.p;
            if (mid) launch_line_pass(MODE_FWD, *mid, p3, nbatch_, st);
            launch_line_pass(MODE_OUTER, out, p3, nbatch_, st);
            if (mid) launch_line_pass(MODE_INV, *mid, p3, nbatch_, st);
            launch_line_pass(MODE_END_RQM4, in, p, nbatch_, st);
        } else {
            if (t == 0) launch_line_pass(MODE_FIRST_OS2, in, p, nbatch_, st);
            p.nfield = 1;
            if (mid) launch_line_pass(MODE_FWD, *mid, p, nbatch_, st);
            launch_line_pass(MODE_OUTER, out, p, nbatch_, st);
            if (mid) launch_line_pass(MODE_INV, *mid, p, nbatch_, st);
            launch_line_pass(MODE_END_OS2, in, p, nbatch_, st);
        }
    }
}

// ---------------------------------------------------------------------------
// contour weights (Density.cc:107-121, Simpson.cc:14-45, Quadrature4.cc)
// ---------------------------------------------------------------------------
bool contour_weights(int rule, int n, std::vector<double>& c) {
    c.assign(n + 1, 0.0);
    switch (rule) {
    case 0:
        for (int s = 0; s <= n; s++) c[s] = 1.0;
        c[0] -= 0.5; c[n] -= 0.5;
        return n >= 1;
    case 1:
        if (n % 2 != 0 || n < 4) return false;
        c[0] = c[n] = 1.0 / 3.0;
        for (int s = 1; s <= n - 1; s += 2) c[s] = 4.0 / 3.0;
        for (int s = 2; s <= n - 2; s += 2) c[s] = 2.0 / 3.0;
        return true;
    case 2:
        if (n < 7) return false;
        for (int s = 3; s <= n - 3; s++) c[s] = 1.0;
        c[0] = c[n] = 0.375; c[1] = c[n - 1] = 7 / 6.0; c[2] = c[n - 2] = 23 / 24.0;
        return true;
    case 3:
        if (n < 9) return false;
        for (int s = 4; s <= n - 4; s++) c[s] = 1.0;
        c[1] = c[n - 1] = 55 / 24.0; c[2] = c[n - 2] = -1 / 6.0; c[3] = c[n - 3] = 33 / 24.0;
        return true;
    case 4:
        if (n < 8) return false;
        for (int s = 4; s <= n - 3; s++) c[s] = 1.0;
        c[1] = 55 / 24.0; c[2] = -1 / 6.0; c[3] = 33 / 24.0;
        c[n - 2] = 23 / 24.0; c[n - 1] = 7 / 6.0; c[n] = 0.375;
        return true;
    case 5:
        if (n < 8) return false;
        for (int s = 3; s <= n - 4; s++) c[s] = 1.0;
        c[0] = 0.375; c[1] = 7 / 6.0; c[2] = 23 / 24.0;
        c[n - 3] = 33 / 24.0; c[n - 2] = -1 / 6.0; c[n - 1] = 55 / 24.0;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// ModelAB
// ---------------------------------------------------------------------------
ModelAB::ModelAB(const ModelABParams& p, bool batch_member) : p_(p) {
    if (p.sA < 2 || p.sB < 2) throw Error(-1, "Ms must be at least [2, 2]");
    if (p.scft == 1 && (p.n_anderson < 1 || ax_nmax(p.n_anderson) == 0))
        throw Error(-2, "n_Anderson_mixing must be in 1..31");
    cell_init(p_.cell);
    M_ = (long)p.Lx * p.Ly * p.Lz;
    LA_ = p.sA - 1;
    LB_ = p.sB - 1;
    Ns_ = LA_ + LB_;
    // Model_AB::init (Model_AB.cc:100-111)
    double fA = 1.0 * LA_ / (LA_ + LB_);
    double fB = 1.0 * LB_ / (LA_ + LB_);
    dsA_ = fA / LA_;
    dsB_ = fB / LB_;
    // Model_AB::init_density (Model_AB.cc:713-735)
    if (p.contour == 0) {
        ruleA_ = ruleB_ = 0;
    } else {
        ruleA_ = (p.sA % 2 != 0) ? 1 : 2;
        ruleB_ = (p.sB % 2 != 0) ? 1 : 2;
    }
    std::vector<double> cA, cB;
    if (!contour_weights(ruleA_, LA_, cA) || !contour_weights(ruleB_, LB_, cB))
        throw Error(-4, "contour quadrature precondition fails for Ms = [" + std::to_string(p.sA) + ", " +
                            std::to_string(p.sB) + "]");
    PS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    chain_ = new PairChain(p.Lx, p.Ly, p.Lz, p.mde == 1 ? SCHEME_OS2 : p.mde == 2 ? SCHEME_ETDRK4 : SCHEME_RQM4, 1);
    // k tables.  ds of the two blocks agree to within two ulps (both round
    // 1/(LA+LB)); the packed lanes share the block-A table.
    if (p.mde == 1) {
        chain_->set_tables(k_laplacian(p_.cell, p.Lx, p.Ly, p.Lz, dsA_), {});
    } else if (p.mde == 2) {
        // Etdrk4_PBC(uc, Lx, Ly, Lz, dsA, etdrk4_M) (Model_AB.cc:746-763; M = 32 when unset)
        chain_->set_tables_etd(k2_orthogonal(p_.cell, p.Lx, p.Ly, p.Lz), dsA_, p.etd_M > 0 ? p.etd_M : 32);
    } else {
        std::vector<double> k2 = k2_orthogonal(p_.cell, p.Lx, p.Ly, p.Lz);
        std::vector<double> L1(M_), L2(M_);
        for (long m = 0; m < M_; m++) {
            L1[m] = exp(dsA_ * k2[m]);
            L2[m] = exp(0.5 * dsA_ * k2[m]);
        }
        chain_->set_tables(L1, L2);
    }
    const char* force = getenv("PS_B200_LINE_PASSES");
    const char* generic = getenv("PS_B200_GENERIC_SWEEP");
    const bool allow = !(force && force[0] == '1');
    use_sweep64_ = allow && p.mde == 0 && sweep64_supported(p.Lx, p.Ly, p.Lz) && !(generic && generic[0] == '1');
    // the 64^3 sweep needs its clusters resident (74 two-CTA clusters on a
    // 148-SM B200); where fewer fit, the generic sweep runs the grid
    if (use_sweep64_) {
        sweep_grid_ = sweep64_prepare();
        use_sweep64_ = sweep_grid_ > 0;
    }
    use_sweep_ = allow && p.mde == 0 && !use_sweep64_ && sweep_supported(p.Lx, p.Ly, p.Lz);
    if (use_sweep64_) {
        swZ_.alloc(6 * (size_t)M_);
        const std::vector<double> tab = sweep64_axis_tables(p_.cell.l, dsA_);
        swTab_.alloc(tab.size());
        PS_CUDA(cudaMemcpy(swTab_.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
        PS_CUDA(cudaMalloc(&swbar_, 64 * sizeof(unsigned)));
        PS_CUDA(cudaMalloc(&swerr_, sizeof(int)));
        PS_CUDA(cudaMemset(swerr_, 0, sizeof(int)));
    }
    if (use_sweep_) {
        sweep_grid_ = sweep_prepare(p.Lx, p.Ly, p.Lz);
        swZ_.alloc(6 * (size_t)M_);
        swU_.alloc(2 * (size_t)M_);
        std::vector<double> k2 = k2_orthogonal(p_.cell, p.Lx, p.Ly, p.Lz);
        std::vector<double> L1(M_), L2(M_);
        for (long m = 0; m < M_; m++) {
            L1[m] = exp(dsA_ * k2[m]);
            L2[m] = exp(0.5 * dsA_ * k2[m]);
        }
        swL1_.alloc(M_);
        swL2_.alloc(M_);
        PS_CUDA(cudaMemcpy(swL1_.p, L1.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMemcpy(swL2_.p, L2.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
        PS_CUDA(cudaMalloc(&swbar_, 32 * sizeof(unsigned)));
        PS_CUDA(cudaMalloc(&swerr_, sizeof(int)));
        PS_CUDA(cudaMemset(swerr_, 0, sizeof(int)));
    }
    hf_.alloc((size_t)(Ns_ + 1) * M_);
    hc_.alloc((size_t)(Ns_ + 1) * M_);
    wA_.alloc(M_); wB_.alloc(M_); yita_.alloc(M_);
    phiA_.alloc(M_); phiB_.alloc(M_);
    eFA_.alloc(M_); eHA_.alloc(M_); eFB_.alloc(M_); eHB_.alloc(M_);
    cA_.alloc(cA.size()); cB_.alloc(cB.size());
    PS_CUDA(cudaMemcpy(cA_.p, cA.data(), sizeof(double) * cA.size(), cudaMemcpyHostToDevice));
    PS_CUDA(cudaMemcpy(cB_.p, cB.data(), sizeof(double) * cB.size(), cudaMemcpyHostToDevice));
    scal_.alloc(32);
    partial_.alloc((size_t)kRedBlocks * 64);
    if (p.scft == 1) {
        const size_t n1 = (size_t)p.n_anderson + 1;
        hwA_.alloc(n1 * M_); hdA_.alloc(n1 * M_); hwB_.alloc(n1 * M_); hdB_.alloc(n1 * M_);
        BA_.alloc(n1 * n1); BB_.alloc(n1 * n1);
        PS_CUDA(cudaMalloc(&axs_, sizeof(AXState)));
    }
    // heads of the forward chain (qA[0] = 1) and of the complementary chain
    // (qBc[0] = 1), Model_AB.cc:779-782
    launch_fill(hf_.p, M_, 1.0, st_);
    launch_fill(hc_.p, M_, 1.0, st_);
    launch_fill(yita_.p, M_, 0.0, st_);
    if (!use_sweep_ && !use_sweep64_ && !batch_member) chain_->autotune(st_);
    if (use_sweep_) {
        sweep_variant_ = sweep_default_variant(p.Lx, p.Ly, p.Lz);
        if (!batch_member) tune_sweep();
    }
    PS_CUDA(cudaStreamSynchronize(st_));
    launches_per_prop_ = (use_sweep_ || use_sweep64_) ? 1 : chain_->launches_per_step() * Ns_ + (chain_->plan().naxes > 1 ? 1 : 0);
    launches_per_iter_ = launches_per_prop_ + 2 + 2 + (p.scft == 1 ? 4 : 1);
}

ModelAB::~ModelAB() {
    if (gprop_) cudaGraphExecDestroy(gprop_);
    if (gpost_) cudaGraphExecDestroy(gpost_);
    delete chain_;
    if (axs_) cudaFree(axs_);
    if (swbar_) cudaFree(swbar_);
    if (swerr_) cudaFree(swerr_);
    if (st_) cudaStreamDestroy(st_);
}

void ModelAB::init_anderson(const double* wA, const double* wB, bool dev) {
    const int n = p_.n_anderson;
    const size_t n1 = (size_t)n + 1;
    auto kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PS_CUDA(cudaMemsetAsync(hwA_.p, 0, sizeof(double) * n1 * M_, st_));
    PS_CUDA(cudaMemsetAsync(hwB_.p, 0, sizeof(double) * n1 * M_, st_));
    PS_CUDA(cudaMemsetAsync(hdA_.p, 0, sizeof(double) * n1 * M_, st_));
    PS_CUDA(cudaMemsetAsync(hdB_.p, 0, sizeof(double) * n1 * M_, st_));
    PS_CUDA(cudaMemsetAsync(BA_.p, 0, sizeof(double) * n1 * n1, st_));
    PS_CUDA(cudaMemsetAsync(BB_.p, 0, sizeof(double) * n1 * n1, st_));
    // FieldAX::update_w0 (FieldAX.cc:274-280): w(n) = w0
    PS_CUDA(cudaMemcpyAsync(hwA_.p + (size_t)n * M_, wA, sizeof(double) * M_, kind, st_));
    PS_CUDA(cudaMemcpyAsync(hwB_.p + (size_t)n * M_, wB, sizeof(double) * M_, kind, st_));
    AXState s{};
    s.n = n; s.k = 0; s.cur = n; s.cur_old = n; s.cur_new = n; s.nc = 0; s.status = 0;
    s.lamA = p_.lamA; s.lamB = p_.lamB;
    PS_CUDA(cudaMemcpyAsync(axs_, &s, sizeof(AXState), cudaMemcpyHostToDevice, st_));
}

void ModelAB::set_fields(const double* wA, const double* wB, bool dev) {
    auto kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PS_CUDA(cudaMemcpyAsync(wA_.p, wA, sizeof(double) * M_, kind, st_));
    PS_CUDA(cudaMemcpyAsync(wB_.p, wB, sizeof(double) * M_, kind, st_));
    // a freshly initialised Yita starts at zero (Model_AB.cc:709-710)
    launch_fill(yita_.p, M_, 0.0, st_);
    if (p_.scft == 1) init_anderson(wA, wB, dev);
    launch_factors(wA_.p, wB_.p, M_, dsA_, dsB_, eFA_.p, eHA_.p, eFB_.p, eHB_.p, 1, 0, st_);
    PS_CUDA(cudaStreamSynchronize(st_));
    iter_ = 0;
    fields_set_ = true;
    forward_done_ = false;
}

// The x-tile variant of the generic persistent sweep for this grid, timed
// once per device and grid shape in a process (whole sweeps on this solve's
// buffers, before its fields are set; the variants compute the same values,
// so the choice only changes the time) and cached.  PS_B200_AUTOTUNE=0
// keeps the default variant, PS_B200_SWEEP_VARIANT=v forces variant v.
void ModelAB::tune_sweep() {
    const char* force = getenv("PS_B200_SWEEP_VARIANT");
    if (force && force[0] >= '0' && force[0] < '0' + kSweepVariants) {
        sweep_variant_ = force[0] - '0';
        return;
    }
    const char* at = getenv("PS_B200_AUTOTUNE");
    if (at && at[0] == '0') return;
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, int> cache;   // (device, Lx, Ly, Lz) -> variant
    int dev = 0;
    PS_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, p_.Lx, p_.Ly, p_.Lz);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
        sweep_variant_ = it->second;
        return;
    }
    // finite data for the timed sweeps (set_fields overwrites the factors)
    for (double* f : {eFA_.p, eHA_.p, eFB_.p, eHB_.p}) launch_fill(f, M_, 1.0, st_);
    const SweepArgs a = sweep_descriptor();
    cudaEvent_t e0, e1;
    PS_CUDA(cudaEventCreate(&e0));
    PS_CUDA(cudaEventCreate(&e1));
    double best = 1e30;
    char line[512];
    int n = std::snprintf(line, sizeof(line), "grid %dx%dx%d persistent sweep, x-tile columns (us per step):",
                          p_.Lx, p_.Ly, p_.Lz);
    for (int v = 0; v < kSweepVariants; v++) {
        auto run = [&]() {
            PS_CUDA(cudaMemsetAsync(swbar_, 0, 32 * sizeof(unsigned), st_));
            sweep_launch(a, p_.Lx, p_.Ly, p_.Lz, sweep_grid_, 1, st_, v);
        };
        run();
        PS_CUDA(cudaEventRecord(e0, st_));
        for (int r = 0; r < 3; r++) run();
        PS_CUDA(cudaEventRecord(e1, st_));
        PS_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double us = 1e3 * ms / 3.0 / Ns_;
        if (n > 0 && n < (int)sizeof(line))
            n += std::snprintf(line + n, sizeof(line) - n, " %d=%.1f", sweep_xtile_columns(p_.Lx, p_.Ly, p_.Lz, v), us);
        if (us < best) {
            best = us;
            sweep_variant_ = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int err = 0;
    PS_CUDA(cudaMemcpy(&err, swerr_, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) throw Error(-3, "persistent sweep reported an error while it was timed");
    if (n > 0 && n < (int)sizeof(line))
        std::snprintf(line + n, sizeof(line) - n, " -> %d\n", sweep_xtile_columns(p_.Lx, p_.Ly, p_.Lz, sweep_variant_));
    tuning_note(line);
    cache[key] = sweep_variant_;
}

SweepArgs ModelAB::sweep_descriptor() const {
    if (!use_sweep_) throw Error(-2, "this solve has no generic persistent sweep");
    SweepArgs a{};
    a.hf = hf_.p; a.hc = hc_.p;
    a.Z1 = swZ_.c(); a.Z2 = swZ_.c() + M_; a.Z3 = swZ_.c() + 2 * M_;
    a.uf = swU_.p; a.uc = swU_.p + M_;
    a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p;
    a.L1 = swL1_.p; a.L2 = swL2_.p;
    a.LA = LA_; a.LB = LB_; a.Ns = Ns_;
    a.bar = swbar_; a.err = swerr_;
    a.bstride_batch = 0; a.bstride_hist = 0; a.bstride_L = 0;
    return a;
}

void ModelAB::enqueue_propagate() { enqueue_propagate(st_); }

void ModelAB::enqueue_propagate(cudaStream_t s) {
    // propagators: forward chain qA -> qB, complementary chain qBc -> qAc
    // (Model_AB.cc:139-145, 187-193)
    if (use_sweep64_) {
        SweepArgs a{};
        a.hf = hf_.p; a.hc = hc_.p;
        a.Z1 = swZ_.c(); a.Z2 = swZ_.c() + M_; a.Z3 = swZ_.c() + 2 * M_;
        a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p;
        a.LA = LA_; a.LB = LB_; a.Ns = Ns_;
        a.bar = swbar_; a.err = swerr_;
        PS_CUDA(cudaMemsetAsync(swbar_, 0, 64 * sizeof(unsigned), s));
        sweep64_launch(a, swTab_.p, sweep_grid_, s);
        return;
    }
    if (use_sweep_) {
        const SweepArgs a = sweep_descriptor();
        PS_CUDA(cudaMemsetAsync(swbar_, 0, 32 * sizeof(unsigned), s));
        sweep_launch(a, p_.Lx, p_.Ly, p_.Lz, sweep_grid_, 1, s, sweep_variant_);
        return;
    }
    if (p_.mde == 2) {
        // ETDRK4 takes the fields themselves: N(q) = -w q
        LaneFactors lf{{wA_.p, wB_.p}, {wA_.p, wB_.p}, LA_};
        LaneFactors lc{{wB_.p, wA_.p}, {wB_.p, wA_.p}, LB_};
        chain_->enqueue(hf_.p, hc_.p, 0, Ns_, lf, lc, 0, s);
        return;
    }
    LaneFactors lf{{eFA_.p, eFB_.p}, {eHA_.p, eHB_.p}, LA_};
    LaneFactors lc{{eFB_.p, eFA_.p}, {eHB_.p, eHA_.p}, LB_};
    chain_->enqueue(hf_.p, hc_.p, 0, Ns_, lf, lc, 0, s);
}

void ModelAB::enqueue_post(cudaStream_t st) {
    // Q = qB->Qt() (Model_AB.cc:195, Propagator.cc:85-93)
    double* dQ = scal_.p + 0;
    launch_mean(hf_.p + (long)Ns_ * M_, M_, partial_.p, dQ, st);
    // phiA = (1/Q) dsA sum c_s qA[s] qAc[LA - s]; phiB likewise (Model_AB.cc:196-199)
    launch_density(hf_.p, hc_.p + (long)LB_ * M_, LA_, M_, cA_.p, dsA_, dQ, 0.0, phiA_.p, 1, 0, 0, nullptr, st);
    launch_density(hf_.p + (long)LA_ * M_, hc_.p, LB_, M_, cB_.p, dsB_, dQ, 0.0, phiB_.p, 1, 0, 0, nullptr, st);
    if (p_.scft == 1) {
        AXArgs a{};
        a.state = axs_; a.n = p_.n_anderson; a.M = M_;
        a.phiA = phiA_.p; a.phiB = phiB_.p; a.dataA = wA_.p; a.dataB = wB_.p;
        a.wA = hwA_.p; a.dA = hdA_.p; a.wB = hwB_.p; a.dB = hdB_.p; a.BA = BA_.p; a.BB = BB_.p;
        a.yita = yita_.p; a.chiN = p_.chiN; a.lamYita = p_.lamYita; a.dsA = dsA_; a.dsB = dsB_;
        a.compressible = p_.compressible;
        a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p;
        launch_anderson(a, partial_.p, st);
    } else {
        EMArgs a{};
        a.phiA = phiA_.p; a.phiB = phiB_.p; a.wA = wA_.p; a.wB = wB_.p; a.yita = yita_.p;
        a.M = M_; a.chiN = p_.chiN; a.lamA = p_.lamA; a.lamB = p_.lamB; a.lamYita = p_.lamYita;
        a.dsA = dsA_; a.dsB = dsB_; a.compressible = p_.compressible;
        a.eFA = eFA_.p; a.eHA = eHA_.p; a.eFB = eFB_.p; a.eHB = eHB_.p; a.bstride = 0;
        launch_em_update(a, 1, st);
    }
}

template <class F>
static cudaGraphExec_t capture(cudaStream_t st, F&& body) {
    PS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    PS_CUDA(cudaStreamEndCapture(st, &g));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw Error(-3, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return ex;
}

void ModelAB::ensure_graphs() {
    if (!fields_set_) throw Error(-6, "fields are not set");
    if (!gprop_) gprop_ = capture(st_, [&] { enqueue_propagate(); });
    if (!gpost_) gpost_ = capture(st_, [&] { enqueue_post(); });
}

void ModelAB::update(int n) {
    ensure_graphs();
    for (int i = 0; i < n; i++) {
        PS_CUDA(cudaGraphLaunch(gprop_, st_));
        PS_CUDA(cudaGraphLaunch(gpost_, st_));
    }
    iter_ += n > 0 ? n : 0;
}

double ModelAB::update_timed(int n, double* prop_ms) {
    ensure_graphs();
    *prop_ms = 0.0;
    if (n <= 0) return 0.0;
    std::vector<cudaEvent_t> ev(2 * (size_t)n + 2);
    for (auto& e : ev) PS_CUDA(cudaEventCreate(&e));
    PS_CUDA(cudaEventRecord(ev[2 * n], st_));
    for (int i = 0; i < n; i++) {
        PS_CUDA(cudaEventRecord(ev[2 * i], st_));
        PS_CUDA(cudaGraphLaunch(gprop_, st_));
        PS_CUDA(cudaEventRecord(ev[2 * i + 1], st_));
        PS_CUDA(cudaGraphLaunch(gpost_, st_));
    }
    PS_CUDA(cudaEventRecord(ev[2 * n + 1], st_));
    iter_ += n;
    PS_CUDA(cudaStreamSynchronize(st_));
    double total = 0.0;
    for (int i = 0; i < n; i++) {
        float ms = 0.f;
        PS_CUDA(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
        total += ms;
    }
    float all = 0.f;
    PS_CUDA(cudaEventElapsedTime(&all, ev[2 * n], ev[2 * n + 1]));
    for (auto& e : ev) cudaEventDestroy(e);
    *prop_ms = total;
    return all;
}

void ModelAB::propagate(int n) {
    ensure_graphs();
    for (int i = 0; i < n; i++) PS_CUDA(cudaGraphLaunch(gprop_, st_));
}

void ModelAB::sync() { PS_CUDA(cudaStreamSynchronize(st_)); }

double ModelAB::Q() {
    if (iter_ == 0 && !forward_done_) throw Error(-6, "no iteration has run");
    double q = 0;
    PS_CUDA(cudaMemcpyAsync(&q, scal_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    return q;
}

void ModelAB::H(double* H, double* Hw, double* Hs) {
    if (iter_ == 0 && !forward_done_) throw Error(-6, "no iteration has run");
    launch_Hw(phiA_.p, phiB_.p, wA_.p, wB_.p, M_, p_.chiN, p_.lamYita, p_.compressible, partial_.p, scal_.p + 1, st_);
    double h[2];
    PS_CUDA(cudaMemcpyAsync(h, scal_.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    *Hw = h[1];
    *Hs = -log(h[0]);
    *H = *Hw + *Hs;
}

double ModelAB::residual() {
    if (iter_ == 0) throw Error(-6, "no iteration has run");
    if (p_.scft == 1) {
        const int n = p_.n_anderson;
        int cur = n - (int)(iter_ % (n + 1));
        int pos = cur + 1;
        if (pos > n) pos = 0;
        launch_residual_ax(hdA_.p + (long)pos * M_, hdB_.p + (long)pos * M_, hwA_.p + (long)pos * M_,
                           hwB_.p + (long)pos * M_, M_, partial_.p, scal_.p + 2, st_);
        double e[4];
        PS_CUDA(cudaMemcpyAsync(e, scal_.p + 2, sizeof(double) * 4, cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        return sqrt((e[0] + e[2]) / (e[1] + e[3]));
    }
    launch_residual_em(phiA_.p, phiB_.p, wA_.p, wB_.p, yita_.p, M_, p_.chiN, p_.lamYita, p_.compressible,
                       partial_.p, scal_.p + 2, st_);
    double v[8];
    PS_CUDA(cudaMemcpyAsync(v, scal_.p + 2, sizeof(double) * 8, cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
    double res = 0.0;
    res += v[0] / (v[1] + v[2]);
    res += v[3] / (v[4] + v[5]);
    if (!p_.compressible) {
        res += v[6] / (1.0 + v[7]);
        res /= 3.0;
    } else {
        res /= 2.0;
    }
    return res;
}

int ModelAB::status() {
    int st = 0;
    if (axs_) {
        AXState s;
        PS_CUDA(cudaMemcpyAsync(&s, axs_, sizeof(AXState), cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        st |= s.status;
    }
    if (swerr_) {
        int e = 0;
        PS_CUDA(cudaMemcpyAsync(&e, swerr_, sizeof(int), cudaMemcpyDeviceToHost, st_));
        PS_CUDA(cudaStreamSynchronize(st_));
        if (e) st |= 2;
    }
    return st;
}

double* ModelAB::device_ptr(int which) {
    switch (which) {
    case 0: return wA_.p;
    case 1: return wB_.p;
    case 2: return phiA_.p;
    case 3: return phiB_.p;
    case 4: return yita_.p;
    case 5: return hf_.p;                         // qA: slices 0..LA of the forward chain
    case 6: return hf_.p + (long)LA_ * M_;        // qB: slices LA..Ns
    case 7: return hc_.p + (long)LB_ * M_;        // qAc: slices LB..Ns of the complementary chain
    case 8: return hc_.p;                         // qBc: slices 0..LB
    }
    throw Error(-1, "unknown field index");
}

void ModelAB::get(int which, double* out, bool device_dst) {
    size_t count = (size_t)M_;
    if (which == 5 || which == 7) count = (size_t)p_.sA * M_;
    if (which == 6 || which == 8) count = (size_t)p_.sB * M_;
    double* src = device_ptr(which);
    PS_CUDA(cudaMemcpyAsync(out, src, sizeof(double) * count,
                            device_dst ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

// ---------------------------------------------------------------------------
// UpdaterCtx
// ---------------------------------------------------------------------------
UpdaterCtx::UpdaterCtx(int scheme, const Cell& cell, int Lx, int Ly, int Lz, double ds, int etd_M)
    : scheme_(scheme), Lx_(Lx), Ly_(Ly), Lz_(Lz), cell_(cell), ds_(ds), etd_M_(etd_M) {
    if (!(ds > 0)) throw Error(-1, "ds must be positive");
    cell_init(cell_);
    M_ = (long)Lx * Ly * Lz;
    PS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    chain_ = new PairChain(Lx, Ly, Lz, scheme, 1);
    if (scheme == SCHEME_OS2) {
        chain_->set_tables(k_laplacian(cell_, Lx, Ly, Lz, ds), {});
    } else if (scheme == SCHEME_ETDRK4) {
        chain_->set_tables_etd(k2_orthogonal(cell_, Lx, Ly, Lz), ds, etd_M);
    } else {
        std::vector<double> k2 = k2_orthogonal(cell_, Lx, Ly, Lz);
        std::vector<double> L1(M_), L2(M_);
        for (long m = 0; m < M_; m++) {
            L1[m] = exp(ds * k2[m]);
            L2[m] = exp(0.5 * ds * k2[m]);
        }
        chain_->set_tables(L1, L2);
    }
    eF_.alloc(2 * M_);
    eH_.alloc(2 * M_);
    zero_.alloc(M_);
    scratch_.alloc(M_);
    launch_fill(zero_.p, M_, 0.0, st_);
    PS_CUDA(cudaStreamSynchronize(st_));
}

UpdaterCtx::~UpdaterCtx() {
    delete chain_;
    if (st_) cudaStreamDestroy(st_);
}

UpdaterCtx* UpdaterCtx::clone() const { return new UpdaterCtx(scheme_, cell_, Lx_, Ly_, Lz_, ds_, etd_M_); }

void UpdaterCtx::solve_device(const double* w, double* qs, int len, cudaStream_t st) {
    if (len < 1) throw Error(-1, "propagator length must be at least 1");
    if (len == 1) return;
    if (!st) st = st_;
    if (scheme_ == SCHEME_ETDRK4) {
        // Etdrk4_PBC::solve (Etdrk4_PBC.cc:110-184) reads w itself
        LaneFactors lf{{w, w}, {w, w}, len};
        LaneFactors lc{{zero_.p, zero_.p}, {zero_.p, zero_.p}, len};
        chain_->enqueue(qs, nullptr, 0, len - 1, lf, lc, 0, st, zero_.p, scratch_.p);
        return;
    }
    // exp(-w ds/2), exp(-w ds/4) (RQM4.cc:49-52, PseudoSpectral.cc:234-235)
    launch_factors(w, w, M_, ds_, ds_, eF_.p, eH_.p, eF_.p + M_, eH_.p + M_, 1, 0, st);
    // lane c carries nothing: zero factors, zero input, scratch output
    LaneFactors lf{{eF_.p, eF_.p}, {eH_.p, eH_.p}, len};
    LaneFactors lc{{zero_.p, zero_.p}, {zero_.p, zero_.p}, len};
    chain_->enqueue(qs, nullptr, 0, len - 1, lf, lc, 0, st, zero_.p, scratch_.p);
}

void UpdaterCtx::solve_host(const double* w, double* qs, int len) {
    if (len < 1) throw Error(-1, "propagator length must be at least 1");
    if (dw_.n < (size_t)M_) dw_.alloc(M_);
    if (dqs_.n < (size_t)len * M_) dqs_.alloc((size_t)len * M_);
    PS_CUDA(cudaMemcpyAsync(dw_.p, w, sizeof(double) * M_, cudaMemcpyHostToDevice, st_));
    PS_CUDA(cudaMemcpyAsync(dqs_.p, qs, sizeof(double) * M_, cudaMemcpyHostToDevice, st_));
    solve_device(dw_.p, dqs_.p, len, st_);
    if (len > 1)
        PS_CUDA(cudaMemcpyAsync(qs + M_, dqs_.p + M_, sizeof(double) * (size_t)(len - 1) * M_,
                                cudaMemcpyDeviceToHost, st_));
    PS_CUDA(cudaStreamSynchronize(st_));
}

}  // namespace ps
