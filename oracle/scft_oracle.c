/*
 * scft_oracle.c -- CPU FP64 restatement of PolyOrder's periodic
 * pseudospectral SCFT path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA product
 * is checked against and the CPU baseline that bench.py times.  The product
 * library (polystring_b200) never links, loads or calls it.
 *
 * Every routine follows the reference step for step and cites the file:line
 * it restates (paths are relative to the reference project root):
 *
 *   k tables        src/UnitCell.cc:149-296 (shape matrices),
 *                   :321-359 (calc_kLaplacian, 27-image minimum),
 *                   :368-418 (calc_k2_orthogonal, returns -k^2)
 *   RQM4            src/RQM4.cc:9-16 (tables), :41-93 (solve)
 *   OS2             src/PseudoSpectral.cc:190-195, :226-261
 *   ETDRK4          src/Etdrk4_PBC.cc:14-24 (tables), :43-99 (contour
 *                   coefficients), :110-184 (solve, carried spectrum)
 *   Propagator      src/Propagator.cc:85-93 (Q = mean of a slice)
 *   densities       src/Density.cc:107-121 (trapezoid), src/Simpson.cc:14-45,
 *                   src/Quadrature4.cc:17-197
 *   Model_AB        src/Model_AB.cc:85-134 (init, Ms -> f, ds),
 *                   :136-261 (update), :263-300 (H), :307-371 (residual),
 *                   :713-735 (quadrature choice)
 *   Field / Yita    src/Field.cc:51-59, src/Yita.cc:49-55
 *   FieldAX         src/FieldAX.cc:152-427 (ring history, B, U, V, W, D)
 *   Model_ABC       (no reference counterpart) linear ABC triblock melt built
 *                   from the Model_AB steps above, defined in its own block
 *   string method   scft/polystring_AB.cc:283-329 (arc length, per-point
 *                   natural cubic spline, ends restored)
 *
 * The FFT is written here (mixed-radix Stockham, radices 2/3/4/5, generic
 * DFT for any other prime factor), complex-to-complex and unnormalised like
 * the FFTW_ESTIMATE c2c plans of the reference (RQM4.cc:22-32).  FFTW itself
 * is not available; the restatement is pinned instead against the
 * reference's own converged free energies and analytic identities (see the
 * tests that import this library).
 *
 * The only deliberate choice where the reference delegates to a third-party
 * library: Armadillo's solve(U, V) (FieldAX.cc:386-390) is restated as
 * Gaussian elimination with partial pivoting; the same algorithm, in the
 * same operation order, runs in the CUDA product.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.141592653589793238462643383279502884L

/* ------------------------------------------------------------------------ */
/* threads                                                                   */
/* ------------------------------------------------------------------------ */
static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n > 0 ? n : 1; }
int orc_get_threads(void) { return g_threads; }
int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* 1D complex FFT: Stockham autosort, mixed radix                            */
/* ------------------------------------------------------------------------ */
typedef struct { double re, im; } cpx;

typedef struct {
    int n;
    int nf;
    int fac[32];
    cpx *tw_fwd;   /* exp(-2 pi i m / n), m = 0..n-1, rounded from long double */
    cpx *tw_bwd;   /* exp(+2 pi i m / n) */
} fft_plan1d;

static void factorize(int n, int *nf, int *fac) {
    int k = 0;
    /* radix 4 first, then 2, 3, 5, then any remaining prime */
    while (n % 4 == 0) { fac[k++] = 4; n /= 4; }
    while (n % 2 == 0) { fac[k++] = 2; n /= 2; }
    while (n % 3 == 0) { fac[k++] = 3; n /= 3; }
    while (n % 5 == 0) { fac[k++] = 5; n /= 5; }
    for (int p = 7; n > 1; p += 2) {
        while (n % p == 0) { fac[k++] = p; n /= p; }
    }
    *nf = k;
}

static fft_plan1d *plan1d_create(int n) {
    fft_plan1d *p = (fft_plan1d *)calloc(1, sizeof(fft_plan1d));
    p->n = n;
    factorize(n, &p->nf, p->fac);
    p->tw_fwd = (cpx *)malloc(sizeof(cpx) * (size_t)n);
    p->tw_bwd = (cpx *)malloc(sizeof(cpx) * (size_t)n);
    for (int m = 0; m < n; m++) {
        long double a = 2.0L * ORC_PI * (long double)m / (long double)n;
        double c = (double)cosl(a), s = (double)sinl(a);
        p->tw_fwd[m].re = c; p->tw_fwd[m].im = -s;
        p->tw_bwd[m].re = c; p->tw_bwd[m].im = s;
    }
    return p;
}

static void plan1d_destroy(fft_plan1d *p) {
    if (!p) return;
    free(p->tw_fwd); free(p->tw_bwd); free(p);
}

static inline cpx cmul(cpx a, cpx b) {
    cpx r; r.re = a.re * b.re - a.im * b.im; r.im = a.re * b.im + a.im * b.re; return r;
}

/* small DFT of length R on v (in place); w = table of exp(sign 2 pi i m/n),
 * stride = n / R so that w[stride*m] = exp(sign 2 pi i m / R). */
static void small_dft(cpx *v, int R, const cpx *w, int stride, int sign) {
    if (R == 2) {
        cpx a = v[0], b = v[1];
        v[0].re = a.re + b.re; v[0].im = a.im + b.im;
        v[1].re = a.re - b.re; v[1].im = a.im - b.im;
        return;
    }
    if (R == 4) {
        cpx a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
        cpx t0 = {a0.re + a2.re, a0.im + a2.im};
        cpx t1 = {a0.re - a2.re, a0.im - a2.im};
        cpx t2 = {a1.re + a3.re, a1.im + a3.im};
        cpx t3 = {a1.re - a3.re, a1.im - a3.im};
        /* multiply t3 by sign*i : forward (sign=-1) -> -i */
        cpx t3r;
        if (sign < 0) { t3r.re = t3.im; t3r.im = -t3.re; }
        else          { t3r.re = -t3.im; t3r.im = t3.re; }
        v[0].re = t0.re + t2.re;  v[0].im = t0.im + t2.im;
        v[2].re = t0.re - t2.re;  v[2].im = t0.im - t2.im;
        v[1].re = t1.re + t3r.re; v[1].im = t1.im + t3r.im;
        v[3].re = t1.re - t3r.re; v[3].im = t1.im - t3r.im;
        return;
    }
    cpx out[64];
    for (int k = 0; k < R; k++) {
        double sr = 0.0, si = 0.0;
        for (int m = 0; m < R; m++) {
            cpx wk = w[(size_t)stride * (size_t)((k * m) % R)];
            sr += v[m].re * wk.re - v[m].im * wk.im;
            si += v[m].re * wk.im + v[m].im * wk.re;
        }
        out[k].re = sr; out[k].im = si;
    }
    for (int k = 0; k < R; k++) v[k] = out[k];
}

/* Stockham autosort passes (Govindaraju et al., SC'08 formulation):
 *   for pass with radix R and Ns = product of earlier radices,
 *   butterfly j in [0, n/R): inputs in[j + r n/R], twiddle
 *   exp(sign 2 pi i (j mod Ns) r / (Ns R)), R-point DFT, outputs to
 *   out[(j/Ns) Ns R + (j mod Ns) + r Ns].                                  */
static void fft1d_exec(const fft_plan1d *p, cpx *x, cpx *work, int sign) {
    int n = p->n;
    if (n == 1) return;
    const cpx *w = sign < 0 ? p->tw_fwd : p->tw_bwd;
    cpx *in = x, *out = work;
    int Ns = 1;
    cpx v[64];
    for (int f = 0; f < p->nf; f++) {
        int R = p->fac[f];
        int nR = n / R;
        for (int j = 0; j < nR; j++) {
            int jm = j % Ns;
            int twstep = n / (Ns * R);
            for (int r = 0; r < R; r++) {
                cpx a = in[j + r * nR];
                int m = (jm * r * twstep) % n;
                v[r] = (m == 0) ? a : cmul(a, w[m]);
            }
            small_dft(v, R, w, n / R, sign);
            int idxD = (j / Ns) * Ns * R + jm;
            for (int r = 0; r < R; r++) out[idxD + r * Ns] = v[r];
        }
        cpx *t = in; in = out; out = t;
        Ns *= R;
    }
    if (in != x) memcpy(x, in, sizeof(cpx) * (size_t)n);
}

/* ------------------------------------------------------------------------ */
/* 3D c2c FFT over (Lx, Ly, Lz), row-major with z fastest                     */
/* ------------------------------------------------------------------------ */
typedef struct {
    int Lx, Ly, Lz;
    fft_plan1d *px, *py, *pz;
} fft_plan3d;

static fft_plan3d *plan3d_create(int Lx, int Ly, int Lz) {
    fft_plan3d *p = (fft_plan3d *)calloc(1, sizeof(fft_plan3d));
    p->Lx = Lx; p->Ly = Ly; p->Lz = Lz;
    p->px = plan1d_create(Lx); p->py = plan1d_create(Ly); p->pz = plan1d_create(Lz);
    return p;
}

static void plan3d_destroy(fft_plan3d *p) {
    if (!p) return;
    plan1d_destroy(p->px); plan1d_destroy(p->py); plan1d_destroy(p->pz); free(p);
}

static void fft3d_exec(const fft_plan3d *p, cpx *a, int sign) {
    int Lx = p->Lx, Ly = p->Ly, Lz = p->Lz;
    int maxn = Lx > Ly ? Lx : Ly; if (Lz > maxn) maxn = Lz;
    /* z lines (contiguous) */
    if (Lz > 1) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int l = 0; l < Lx * Ly; l++) {
            cpx work[1024];
            fft1d_exec(p->pz, a + (size_t)l * Lz, work, sign);
        }
    }
    if (Ly > 1) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int l = 0; l < Lx * Lz; l++) {
            int i = l / Lz, k = l % Lz;
            cpx line[1024], work[1024];
            for (int j = 0; j < Ly; j++) line[j] = a[((size_t)i * Ly + j) * Lz + k];
            fft1d_exec(p->py, line, work, sign);
            for (int j = 0; j < Ly; j++) a[((size_t)i * Ly + j) * Lz + k] = line[j];
        }
    }
    if (Lx > 1) {
        size_t P = (size_t)Ly * Lz;
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (long l = 0; l < (long)P; l++) {
            cpx line[1024], work[1024];
            for (int i = 0; i < Lx; i++) line[i] = a[(size_t)i * P + l];
            fft1d_exec(p->px, line, work, sign);
            for (int i = 0; i < Lx; i++) a[(size_t)i * P + l] = line[i];
        }
    }
    (void)maxn;
}

/* exported for the FFT round-trip tests: data interleaved (re, im) */
int orc_fft3(int Lx, int Ly, int Lz, double *data, int sign) {
    if (Lx > 1024 || Ly > 1024 || Lz > 1024 || Lx < 1 || Ly < 1 || Lz < 1) return -1;
    fft_plan3d *p = plan3d_create(Lx, Ly, Lz);
    fft3d_exec(p, (cpx *)data, sign < 0 ? -1 : 1);
    plan3d_destroy(p);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* UnitCell                                                                  */
/* ------------------------------------------------------------------------ */
/* crystal systems, numbered as in the C-ABI header (polystring_b200.h) */
enum {
    ORC_LAMELLAR = 0,
    ORC_SQUARE = 1, ORC_RECTANGULAR = 2, ORC_HEXAGONAL2 = 3, ORC_OBLIQUE = 4,
    ORC_CUBIC = 5, ORC_TETRAGONAL = 6, ORC_ORTHORHOMBIC = 7, ORC_HEXAGONAL3 = 8,
    ORC_TRIGONAL = 9, ORC_MONOCLINIC = 10, ORC_TRICLINIC = 11
};

static void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* UnitCell::calc_shape_matrix{1,2,3} (UnitCell.cc:149-296).  Outputs the
 * reciprocal shape matrix g (row-major 3x3, g = 2 pi [a* b* c*] as columns)
 * and the cell lengths l = (lx, ly, lz).  Returns 0, or -1 on a bad cell. */
int orc_unit_cell(int dim, int system, double a, double b, double c,
                  double alpha, double beta, double gamma, double *g, double *l) {
    const double PI = (double)ORC_PI;
    const double pi2 = PI / 2.0, pi3 = 2.0 * PI / 3.0, twopi = 2.0 * PI;
    memset(g, 0, 9 * sizeof(double));
    if (dim == 1) {
        if (a <= 0) return -1;
        l[0] = a; l[1] = 0.0; l[2] = 0.0;
        g[0] = twopi / a; g[4] = twopi; g[8] = twopi;
        return 0;
    }
    if (dim == 2) {
        if (a <= 0) return -1;
        switch (system) {
        case ORC_SQUARE: b = a; gamma = pi2; break;
        case ORC_RECTANGULAR: if (b <= 0) return -1; gamma = pi2; break;
        case ORC_HEXAGONAL2: b = a; gamma = pi3; break;
        default: if (b <= 0 || gamma <= 0) return -1; break;
        }
        double va[3] = {a, 0.0, 0.0};
        double vb[3] = {b * cos(gamma), b * sin(gamma), 0.0};
        l[0] = a; l[1] = b; l[2] = 0.0;
        double acb[3]; cross3(va, vb, acb);
        double denom = dot3(acb, acb);
        double as[3], bs[3], t[3];
        cross3(vb, acb, t); for (int i = 0; i < 3; i++) as[i] = t[i] / denom;
        cross3(acb, va, t); for (int i = 0; i < 3; i++) bs[i] = t[i] / denom;
        g[0] = twopi * as[0]; g[1] = twopi * bs[0]; g[2] = 0.0;
        g[3] = twopi * as[1]; g[4] = twopi * bs[1]; g[5] = 0.0;
        g[6] = 0.0;           g[7] = 0.0;           g[8] = twopi;
        return 0;
    }
    switch (system) {
    case ORC_CUBIC: b = a; c = a; alpha = beta = gamma = pi2; break;
    case ORC_TETRAGONAL: b = a; alpha = beta = gamma = pi2; break;
    case ORC_ORTHORHOMBIC: alpha = beta = gamma = pi2; break;
    case ORC_HEXAGONAL3: b = a; alpha = pi2; beta = pi2; gamma = pi3; break;
    case ORC_TRIGONAL: b = a; c = a; alpha = gamma; beta = gamma; break;
    case ORC_MONOCLINIC: alpha = pi2; gamma = pi2; break;
    case ORC_TRICLINIC: break;
    default: return -1;
    }
    double va[3] = {a, 0.0, 0.0};
    double vb[3] = {b * cos(gamma), b * sin(gamma), 0.0};
    double cx = c * cos(beta);
    double cy = c * (cos(alpha) - cos(beta) * cos(gamma));
    double cz = sqrt(c * c - cx * cx - cy * cy);
    double vc[3] = {cx, cy, cz};
    l[0] = a; l[1] = b; l[2] = c;
    double bcc[3], cca[3], acb[3];
    cross3(vb, vc, bcc); cross3(vc, va, cca); cross3(va, vb, acb);
    double denom = dot3(va, bcc);
    for (int i = 0; i < 3; i++) {
        g[3 * i + 0] = twopi * (bcc[i] / denom);
        g[3 * i + 1] = twopi * (cca[i] / denom);
        g[3 * i + 2] = twopi * (acb[i] / denom);
    }
    return 0;
}

/* UnitCell::calc_k2_orthogonal (UnitCell.cc:368-418): returns -|k|^2 */
void orc_k2_orthogonal(int dim, double lx, double ly, double lz,
                       int Lx, int Ly, int Lz, double *k2) {
    const double PI = (double)ORC_PI;
    double ccx = 0.0, ccy = 0.0, ccz = 0.0;
    if (dim >= 1) ccx = -4.0 * PI * PI / (lx * lx);
    if (dim >= 2) ccy = -4.0 * PI * PI / (ly * ly);
    if (dim >= 3) ccz = -4.0 * PI * PI / (lz * lz);
    for (int i = 0; i < Lx; i++)
        for (int j = 0; j < Ly; j++)
            for (int k = 0; k < Lz; k++) {
                int ri = (i < Lx / 2 + 1) ? i : Lx - i;
                int rj = (j < Ly / 2 + 1) ? j : Ly - j;
                int rk = (k < Lz / 2 + 1) ? k : Lz - k;
                k2[((size_t)i * Ly + j) * Lz + k] = ccx * ri * ri + ccy * rj * rj + ccz * rk * rk;
            }
}

/* UnitCell::calc_k2 + calc_kLaplacian (UnitCell.cc:321-359): exp(-ds |q|^2)
 * with |q|^2 minimised over the 27 neighbouring images. */
void orc_k_laplacian(const double *g, int Na, int Nb, int Nc, double ds, double *out) {
    for (int i = 0; i < Na; i++)
        for (int j = 0; j < Nb; j++)
            for (int k = 0; k < Nc; k++) {
                double q2min = 1.0e300;
                for (int ii = 1; ii > -2; ii--)
                    for (int jj = 1; jj > -2; jj--)
                        for (int kk = 1; kk > -2; kk--) {
                            double bq[3] = {(double)(ii * Na) + i, (double)(jj * Nb) + j,
                                            (double)(kk * Nc) + k};
                            double qt[3];
                            for (int r = 0; r < 3; r++)
                                qt[r] = g[3 * r + 0] * bq[0] + g[3 * r + 1] * bq[1] + g[3 * r + 2] * bq[2];
                            double q2 = dot3(qt, qt);
                            if (q2 < q2min) q2min = q2;
                        }
                out[((size_t)i * Nb + j) * Nc + k] = exp(-ds * q2min);
            }
}

/* ------------------------------------------------------------------------ */
/* Propagator updaters                                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
    int scheme;           /* 0 = RQM4, 1 = OS2, 2 = ETDRK4 */
    int Lx, Ly, Lz;
    size_t M;
    double ds;
    double *lap;          /* RQM4: exp(ds * k2); OS2: exp(-ds q^2); ETDRK4: E = exp(ds k2) */
    double *lap2;         /* RQM4: exp(0.5 ds k2); ETDRK4: E2 = exp(ds k2 / 2) */
    double *eq, *f1, *f2, *f3;   /* ETDRK4 contour coefficients Q, f1, f2, f3 */
    fft_plan3d *plan;
    cpx *buf;
} orc_updater;

/* RQM4::RQM4 (RQM4.cc:9-16): k2 = calc_k2_orthogonal (already -k^2) */
orc_updater *orc_rqm4_create(const double *k2, int Lx, int Ly, int Lz, double ds) {
    orc_updater *u = (orc_updater *)calloc(1, sizeof(orc_updater));
    u->scheme = 0; u->Lx = Lx; u->Ly = Ly; u->Lz = Lz;
    u->M = (size_t)Lx * Ly * Lz; u->ds = ds;
    u->lap = (double *)malloc(sizeof(double) * u->M);
    u->lap2 = (double *)malloc(sizeof(double) * u->M);
    for (size_t m = 0; m < u->M; m++) {
        u->lap[m] = exp(ds * k2[m]);
        u->lap2[m] = exp(0.5 * ds * k2[m]);
    }
    u->plan = plan3d_create(Lx, Ly, Lz);
    u->buf = (cpx *)malloc(sizeof(cpx) * u->M);
    return u;
}

/* PseudoSpectral(laplace) (PseudoSpectral.cc:190-201): lap = calc_kLaplacian */
orc_updater *orc_os2_create(const double *lap, int Lx, int Ly, int Lz, double ds) {
    orc_updater *u = (orc_updater *)calloc(1, sizeof(orc_updater));
    u->scheme = 1; u->Lx = Lx; u->Ly = Ly; u->Lz = Lz;
    u->M = (size_t)Lx * Ly * Lz; u->ds = ds;
    u->lap = (double *)malloc(sizeof(double) * u->M);
    memcpy(u->lap, lap, sizeof(double) * u->M);
    u->plan = plan3d_create(Lx, Ly, Lz);
    u->buf = (cpx *)malloc(sizeof(cpx) * u->M);
    return u;
}

/* Etdrk4_PBC(uc, Lx, Ly, Lz, ds, Mc) (Etdrk4_PBC.cc:14-24, :43-99): L = -k^2
 * (calc_k2_orthogonal), E = exp(ds L), E2 = exp(ds L / 2), and Q, f1, f2, f3
 * as ds times the mean over Mc points r = exp(i pi (j + 1/2) / Mc) of the
 * Kassam-Trefethen expressions at x = ds L + r:
 *   Q  = (e^{x/2} - 1) / x,            f1 = (e^x (x^2 - 3x + 4) - x - 4) / x^3,
 *   f2 = (e^x (x - 2) + x + 2) / x^3,  f3 = (e^x (4 - x) - x^2 - 3x - 4) / x^3 */
orc_updater *orc_etdrk4_create(const double *k2, int Lx, int Ly, int Lz, double ds, int Mc) {
    orc_updater *u = (orc_updater *)calloc(1, sizeof(orc_updater));
    u->scheme = 2; u->Lx = Lx; u->Ly = Ly; u->Lz = Lz;
    u->M = (size_t)Lx * Ly * Lz; u->ds = ds;
    size_t M = u->M;
    u->lap = (double *)malloc(sizeof(double) * M);
    u->lap2 = (double *)malloc(sizeof(double) * M);
    u->eq = (double *)malloc(sizeof(double) * M);
    u->f1 = (double *)malloc(sizeof(double) * M);
    u->f2 = (double *)malloc(sizeof(double) * M);
    u->f3 = (double *)malloc(sizeof(double) * M);
    const double PI = 3.14159265358979323846;
    for (size_t m = 0; m < M; m++) {
        const double L = k2[m];
        u->lap[m] = exp(ds * L);
        u->lap2[m] = exp(ds * L / 2.0);
        double sq = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int j = 0; j < Mc; j++) {
            double complex r = cexp(I * (PI * (j + 0.5) / Mc));
            double complex x = ds * L + r;
            double complex ex = cexp(x), x2 = x * x, x3 = x2 * x;
            sq += creal((cexp(x / 2.0) - 1.0) / x);
            s1 += creal((ex * (x2 - 3.0 * x + 4.0) - x - 4.0) / x3);
            s2 += creal((ex * (x - 2.0) + x + 2.0) / x3);
            s3 += creal((ex * (4.0 - x) - x2 - 3.0 * x - 4.0) / x3);
        }
        u->eq[m] = ds * (sq / Mc);
        u->f1[m] = ds * (s1 / Mc);
        u->f2[m] = ds * (s2 / Mc);
        u->f3[m] = ds * (s3 / Mc);
    }
    u->plan = plan3d_create(Lx, Ly, Lz);
    u->buf = (cpx *)malloc(sizeof(cpx) * M);
    return u;
}

void orc_updater_destroy(orc_updater *u) {
    if (!u) return;
    free(u->lap); free(u->lap2); free(u->eq); free(u->f1); free(u->f2); free(u->f3);
    plan3d_destroy(u->plan); free(u->buf); free(u);
}

/* N(x) = F[-w x] with x = Re(b) / M taken from an inverse transform in b
 * (inv != 0) or x = the real slice q (inv == 0) */
static void etd_nonlin(orc_updater *u, const double *w, const cpx *b, const double *q, int inv, cpx *out) {
    size_t M = u->M;
    double rM = (double)M;
    for (size_t m = 0; m < M; m++) {
        double x = inv ? b[m].re / rM : q[m];
        out[m].re = -w[m] * x;
        out[m].im = 0.0;
    }
    fft3d_exec(u->plan, out, -1);
}

/* Etdrk4_PBC::solve (Etdrk4_PBC.cc:110-184), Cox-Matthews: the spectrum v of
 * q is carried from step to step; each step takes four forward and four
 * inverse transforms. */
static int etdrk4_solve(orc_updater *u, const double *w, double *qs, int len) {
    size_t M = u->M;
    double rM = (double)M;
    cpx *v = (cpx *)malloc(sizeof(cpx) * M), *Nv = (cpx *)malloc(sizeof(cpx) * M);
    cpx *a = (cpx *)malloc(sizeof(cpx) * M), *Na = (cpx *)malloc(sizeof(cpx) * M);
    cpx *Nb = (cpx *)malloc(sizeof(cpx) * M), *Nc = (cpx *)malloc(sizeof(cpx) * M);
    cpx *t = u->buf;
    for (size_t m = 0; m < M; m++) { v[m].re = qs[m]; v[m].im = 0.0; }
    fft3d_exec(u->plan, v, -1);
    for (int s = 0; s < len - 1; s++) {
        const double *q1 = qs + (size_t)s * M;
        double *q2 = qs + (size_t)(s + 1) * M;
        etd_nonlin(u, w, NULL, q1, 0, Nv);
        for (size_t m = 0; m < M; m++) {      /* a = E2 v + Q Nv */
            a[m].re = u->lap2[m] * v[m].re + u->eq[m] * Nv[m].re;
            a[m].im = u->lap2[m] * v[m].im + u->eq[m] * Nv[m].im;
            t[m] = a[m];
        }
        fft3d_exec(u->plan, t, +1);
        etd_nonlin(u, w, t, NULL, 1, Na);
        for (size_t m = 0; m < M; m++) {      /* b = E2 v + Q Na */
            t[m].re = u->lap2[m] * v[m].re + u->eq[m] * Na[m].re;
            t[m].im = u->lap2[m] * v[m].im + u->eq[m] * Na[m].im;
        }
        fft3d_exec(u->plan, t, +1);
        etd_nonlin(u, w, t, NULL, 1, Nb);
        for (size_t m = 0; m < M; m++) {      /* c = E2 a + Q (2 Nb - Nv) */
            t[m].re = u->lap2[m] * a[m].re + u->eq[m] * (2.0 * Nb[m].re - Nv[m].re);
            t[m].im = u->lap2[m] * a[m].im + u->eq[m] * (2.0 * Nb[m].im - Nv[m].im);
        }
        fft3d_exec(u->plan, t, +1);
        etd_nonlin(u, w, t, NULL, 1, Nc);
        for (size_t m = 0; m < M; m++) {      /* v = E v + f1 Nv + 2 f2 (Na + Nb) + f3 Nc */
            double c2 = 2.0 * u->f2[m];
            v[m].re = u->lap[m] * v[m].re + u->f1[m] * Nv[m].re + c2 * (Na[m].re + Nb[m].re) + u->f3[m] * Nc[m].re;
            v[m].im = u->lap[m] * v[m].im + u->f1[m] * Nv[m].im + c2 * (Na[m].im + Nb[m].im) + u->f3[m] * Nc[m].im;
            t[m] = v[m];
        }
        fft3d_exec(u->plan, t, +1);
        for (size_t m = 0; m < M; m++) q2[m] = t[m].re / rM;
    }
    free(v); free(Nv); free(a); free(Na); free(Nb); free(Nc);
    return 0;
}

/* one split-step e^{-w h/2} F^-1[ L F[e^{-w h/2} q] ] / M  (RQM4.cc:71-75) */
static void split_step(orc_updater *u, const double *e, const double *L,
                       const double *qin, double *qout) {
    size_t M = u->M;
    cpx *b = u->buf;
    for (size_t m = 0; m < M; m++) { b[m].re = e[m] * qin[m]; b[m].im = 0.0; }
    fft3d_exec(u->plan, b, -1);
    for (size_t m = 0; m < M; m++) { b[m].re *= L[m]; b[m].im *= L[m]; }
    fft3d_exec(u->plan, b, +1);
    double inv = (double)M;
    for (size_t m = 0; m < M; m++) qout[m] = (b[m].re * e[m]) / inv;
}

/* RQM4::solve (RQM4.cc:41-93) / PseudoSpectral::solve (PseudoSpectral.cc:226-261).
 * qs holds len slices of M; qs[0] is the head on entry. */
int orc_updater_solve(orc_updater *u, const double *w, double *qs, int len) {
    if (u->scheme == 2) return etdrk4_solve(u, w, qs, len);
    size_t M = u->M;
    double ds = u->ds;
    double *expq = (double *)malloc(sizeof(double) * M);
    double *expq2 = (double *)malloc(sizeof(double) * M);
    double *qt = (double *)malloc(sizeof(double) * M);
    for (size_t m = 0; m < M; m++) {
        expq[m] = exp(-0.5 * ds * w[m]);
        expq2[m] = exp(-0.25 * ds * w[m]);
    }
    for (int s = 0; s < len - 1; s++) {
        const double *q1 = qs + (size_t)s * M;
        double *q2 = qs + (size_t)(s + 1) * M;
        split_step(u, expq, u->lap, q1, q2);
        if (u->scheme == 0) {
            split_step(u, expq2, u->lap2, q1, qt);
            split_step(u, expq2, u->lap2, qt, qt);
            for (size_t m = 0; m < M; m++) q2[m] = (4.0 * qt[m] - q2[m]) / 3.0;
        }
    }
    free(expq); free(expq2); free(qt);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Grid reductions                                                           */
/* ------------------------------------------------------------------------ */
/* Grid::quadrature on a regular grid is the mean (Grid.cc:329-374) */
double orc_mean(const double *a, size_t M) {
    double s = 0.0;
    for (size_t m = 0; m < M; m++) s += a[m];
    return s / (double)M;
}

static double mean_abs(const double *a, size_t M) {
    double s = 0.0;
    for (size_t m = 0; m < M; m++) s += fabs(a[m]);
    return s / (double)M;
}

/* ------------------------------------------------------------------------ */
/* Density: contour quadratures                                              */
/* ------------------------------------------------------------------------ */
enum { ORC_TRAPEZOID = 0, ORC_SIMPSON = 1, ORC_QUAD4_CLOSED = 2, ORC_QUAD4_OPEN = 3,
       ORC_QUAD4_SEMIOPEN_LEFT = 4, ORC_QUAD4_SEMIOPEN_RIGHT = 5 };

/* weights c_s (s = 0..n) such that phi = cc * ds * sum_s c_s q[s] qc[n-s].
 * Returns -1 when the rule's precondition fails (the reference prints to
 * cerr and leaves phi untouched: Simpson.cc:18-26, Quadrature4.cc:22-25). */
int orc_contour_weights(int rule, int n, double *c) {
    for (int s = 0; s <= n; s++) c[s] = 0.0;
    switch (rule) {
    case ORC_TRAPEZOID:               /* Density.cc:107-121 */
        for (int s = 0; s <= n; s++) c[s] = 1.0;
        c[0] -= 0.5; c[n] -= 0.5;
        return 0;
    case ORC_SIMPSON:                 /* Simpson.cc:14-45 */
        if (n % 2 != 0 || n < 4) return -1;
        c[0] = 1.0 / 3.0; c[n] = 1.0 / 3.0;
        for (int s = 1; s <= n - 1; s += 2) c[s] = 4.0 / 3.0;
        for (int s = 2; s <= n - 2; s += 2) c[s] = 2.0 / 3.0;
        return 0;
    case ORC_QUAD4_CLOSED:            /* Quadrature4.cc:17-53 */
        if (n < 7) return -1;
        for (int s = 3; s <= n - 3; s++) c[s] = 1.0;
        c[0] = c[n] = 0.375; c[1] = c[n - 1] = 7 / 6.0; c[2] = c[n - 2] = 23 / 24.0;
        return 0;
    case ORC_QUAD4_OPEN:              /* Quadrature4.cc:62-102 */
        if (n < 9) return -1;
        for (int s = 4; s <= n - 4; s++) c[s] = 1.0;
        c[1] = c[n - 1] = 55 / 24.0; c[2] = c[n - 2] = -1 / 6.0; c[3] = c[n - 3] = 33 / 24.0;
        return 0;
    case ORC_QUAD4_SEMIOPEN_LEFT:     /* Quadrature4.cc:111-155 */
        if (n < 8) return -1;
        for (int s = 4; s <= n - 3; s++) c[s] = 1.0;
        c[1] = 55 / 24.0; c[2] = -1 / 6.0; c[3] = 33 / 24.0;
        c[n - 2] = 23 / 24.0; c[n - 1] = 7 / 6.0; c[n] = 0.375;
        return 0;
    case ORC_QUAD4_SEMIOPEN_RIGHT:    /* Quadrature4.cc:164-197 */
        if (n < 8) return -1;
        for (int s = 3; s <= n - 4; s++) c[s] = 1.0;
        c[0] = 0.375; c[1] = 7 / 6.0; c[2] = 23 / 24.0;
        c[n - 3] = 33 / 24.0; c[n - 2] = -1 / 6.0; c[n - 1] = 55 / 24.0;
        return 0;
    }
    return -2;
}

/* Density update: phi = cc * ds * sum_s c_s q[s] * qc[n-s].  The reference
 * builds qq = q * reverse(qc) and sums along s (Simpson.cc:31-44); the sum
 * here accumulates in s order per grid point. */
int orc_density(int rule, const double *q, const double *qc, int len, size_t M,
                double ds, double cc, double *phi) {
    int n = len - 1;
    double *c = (double *)malloc(sizeof(double) * (size_t)len);
    int rc = orc_contour_weights(rule, n, c);
    if (rc != 0) { free(c); return rc; }
    for (size_t m = 0; m < M; m++) {
        double acc = 0.0;
        for (int s = 0; s <= n; s++) acc += c[s] * (q[(size_t)s * M + m] * qc[(size_t)(n - s) * M + m]);
        phi[m] = acc * (cc * ds);
    }
    free(c);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Small dense solve for Anderson mixing                                     */
/* ------------------------------------------------------------------------ */
/* Solves U C = V (n x n, row-major U), Gaussian elimination with partial
 * pivoting (first maximal |pivot| wins), then back substitution.  Returns 0,
 * or -1 when a pivot is exactly zero. */
int orc_solve_small(int n, const double *Uin, const double *Vin, double *C) {
    double A[64 * 64], b[64];
    if (n > 64) return -2;
    for (int i = 0; i < n * n; i++) A[i] = Uin[i];
    for (int i = 0; i < n; i++) b[i] = Vin[i];
    for (int k = 0; k < n; k++) {
        int p = k; double best = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; i++) {
            double v = fabs(A[i * n + k]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0.0) return -1;
        if (p != k) {
            for (int j = 0; j < n; j++) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        double piv = A[k * n + k];
        for (int i = k + 1; i < n; i++) {
            double f = A[i * n + k] / piv;
            A[i * n + k] = 0.0;
            for (int j = k + 1; j < n; j++) A[i * n + j] -= f * A[k * n + j];
            b[i] -= f * b[k];
        }
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= A[i * n + j] * C[j];
        C[i] = s / A[i * n + i];
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FieldAX: Anderson mixing history (FieldAX.cc)                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n;            /* history length; w(i), d(i), i = 0..n */
    int cur;          /* cur_pos */
    long k;           /* iterations performed */
    double lambda;
    size_t M;
    double *w;        /* (n+1) x M */
    double *d;        /* (n+1) x M */
    double *B;        /* (n+1) x (n+1) */
    double *data;     /* current field (Grid::_data) */
} orc_fieldax;

static void fax_init(orc_fieldax *f, int n, double lambda, size_t M, const double *w0) {
    f->n = n; f->cur = n; f->k = 0; f->lambda = lambda; f->M = M;
    f->w = (double *)calloc((size_t)(n + 1) * M, sizeof(double));
    f->d = (double *)calloc((size_t)(n + 1) * M, sizeof(double));
    f->B = (double *)calloc((size_t)(n + 1) * (n + 1), sizeof(double));
    f->data = (double *)malloc(sizeof(double) * M);
    memcpy(f->data, w0, sizeof(double) * M);
    memcpy(f->w + (size_t)n * M, w0, sizeof(double) * M);   /* update_w0, FieldAX.cc:274-280 */
}

static void fax_free(orc_fieldax *f) { free(f->w); free(f->d); free(f->B); free(f->data); }

static int fax_find_index(const orc_fieldax *f, int j) {    /* FieldAX.cc:262-267 */
    int i = j + f->cur;
    if (i > f->n) i -= (f->n + 1);
    return i;
}

static int fax_nn(const orc_fieldax *f) { return f->k < f->n ? (int)f->k : f->n; }

/* pre_update (FieldAX.cc:188-199): update_d then update_B */
static void fax_pre_update(orc_fieldax *f, const double *wt) {
    size_t M = f->M;
    int n = f->n, N1 = n + 1;
    double *dc = f->d + (size_t)f->cur * M;
    const double *wc = f->w + (size_t)f->cur * M;
    for (size_t m = 0; m < M; m++) dc[m] = wt[m] - wc[m];               /* update_d :311-313 */
    for (int i = n; i >= 1; i--)                                         /* update_B :321-345 */
        for (int j = n; j >= i; j--) f->B[i * N1 + j] = f->B[(i - 1) * N1 + (j - 1)];
    int nn = fax_nn(f);
    for (int j = 0; j <= nn; j++) {
        const double *dk = f->d + (size_t)fax_find_index(f, j) * M;
        double s = 0.0;
        for (size_t m = 0; m < M; m++) s += dc[m] * dk[m];
        f->B[0 * N1 + j] = s / (double)M;
    }
    for (int i = 0; i < N1; i++)                                         /* symmatu */
        for (int j = i + 1; j < N1; j++) f->B[j * N1 + i] = f->B[i * N1 + j];
}

/* calc_U / calc_V (FieldAX.cc:352-381), accumulated into U, V */
static void fax_add_UV(const orc_fieldax *f, double *U, double *V) {
    int nn = fax_nn(f), N1 = f->n + 1;
    const double *B = f->B;
    for (int i = 0; i < nn; i++) {
        for (int j = 0; j < nn; j++)
            U[i * nn + j] += B[0] - B[(i + 1) * N1 + 0] - B[0 * N1 + (j + 1)] + B[(i + 1) * N1 + (j + 1)];
        V[i] += B[0] - B[(i + 1) * N1 + 0];
    }
}

/* update(C) (FieldAX.cc:201-223, calc_W :395-410, calc_D :415-427,
 * update_w :286-305) */
static void fax_update(orc_fieldax *f, const double *C, int nc, double *Wtmp, double *Dtmp) {
    size_t M = f->M;
    const double *wc = f->w + (size_t)f->cur * M;
    const double *dc = f->d + (size_t)f->cur * M;
    memcpy(Wtmp, wc, sizeof(double) * M);
    memcpy(Dtmp, dc, sizeof(double) * M);
    for (int i = 1; i <= nc; i++) {
        int kk = fax_find_index(f, i);
        const double *wk = f->w + (size_t)kk * M;
        const double *dk = f->d + (size_t)kk * M;
        double ci = C[i - 1];
        for (size_t m = 0; m < M; m++) {
            Wtmp[m] += ci * (wk[m] - wc[m]);
            Dtmp[m] += ci * (dk[m] - dc[m]);
        }
    }
    if (f->cur > 0) f->cur--; else f->cur = f->n;
    double lam = 1.0 - pow(f->lambda, (double)(f->k + 1));
    double *wn = f->w + (size_t)f->cur * M;
    for (size_t m = 0; m < M; m++) {
        double v = Wtmp[m] + lam * Dtmp[m];
        wn[m] = v;
        f->data[m] = v;
    }
    f->k++;
}

/* ------------------------------------------------------------------------ */
/* Model_AB                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    int dim, Lx, Ly, Lz;
    int sA, sB;
    double chiN;
    double lamA, lamB, lamYita;
    int mde;              /* 0 = RQM4, 1 = OS2, 2 = ETDRK4 */
    int scft;             /* 0 = EM, 1 = Anderson */
    int n_anderson;
    int compressible;
    int contour;          /* 0 = trapezoid, 1 = Simpson (Simpson/Quad4 by parity) */
    const double *k2;     /* RQM4: -k^2 table (calc_k2_orthogonal), M values */
    const double *lapA;   /* OS2: exp(-dsA q^2) table */
    const double *lapB;   /* OS2: exp(-dsB q^2) table */
} orc_ab_params;

typedef struct {
    orc_ab_params p;
    size_t M;
    double fA, fB, dsA, dsB;
    int ruleA, ruleB;
    orc_updater *upA, *upB;
    double *qA, *qB, *qAc, *qBc;       /* histories */
    double *wA, *wB, *yita;            /* EM fields */
    orc_fieldax axA, axB;              /* Anderson fields */
    double *phiA, *phiB;
    double Q;
    double *tmp1, *tmp2, *tmp3;
    int last_rc;
} orc_model_ab;

static const double *cur_wA(const orc_model_ab *m) { return m->p.scft == 1 ? m->axA.data : m->wA; }
static const double *cur_wB(const orc_model_ab *m) { return m->p.scft == 1 ? m->axB.data : m->wB; }

/* Model_AB::init (Model_AB.cc:85-134) with init_density (:713-735) and
 * init_propagator (:737-824); fields come from the caller (DATA_INIT). */
orc_model_ab *orc_model_ab_create(const orc_ab_params *p, const double *wA0, const double *wB0) {
    orc_model_ab *m = (orc_model_ab *)calloc(1, sizeof(orc_model_ab));
    m->p = *p;
    size_t M = (size_t)p->Lx * p->Ly * p->Lz;
    m->M = M;
    int LA = p->sA - 1, LB = p->sB - 1;
    m->fA = 1.0 * LA / (LA + LB);
    m->fB = 1.0 * LB / (LA + LB);
    m->dsA = m->fA / LA;
    m->dsB = m->fB / LB;
    if (p->contour == 0) { m->ruleA = m->ruleB = ORC_TRAPEZOID; }
    else {
        m->ruleA = (p->sA % 2 != 0) ? ORC_SIMPSON : ORC_QUAD4_CLOSED;
        m->ruleB = (p->sB % 2 != 0) ? ORC_SIMPSON : ORC_QUAD4_CLOSED;
    }
    if (p->mde == 0) {
        m->upA = orc_rqm4_create(p->k2, p->Lx, p->Ly, p->Lz, m->dsA);
        m->upB = orc_rqm4_create(p->k2, p->Lx, p->Ly, p->Lz, m->dsB);
    } else if (p->mde == 2) {
        /* the Propagator's default Etdrk4_PBC (Propagator.cc:115), M = 32 */
        m->upA = orc_etdrk4_create(p->k2, p->Lx, p->Ly, p->Lz, m->dsA, 32);
        m->upB = orc_etdrk4_create(p->k2, p->Lx, p->Ly, p->Lz, m->dsB, 32);
    } else {
        m->upA = orc_os2_create(p->lapA, p->Lx, p->Ly, p->Lz, m->dsA);
        m->upB = orc_os2_create(p->lapB, p->Lx, p->Ly, p->Lz, m->dsB);
    }
    m->qA = (double *)calloc((size_t)p->sA * M, sizeof(double));
    m->qAc = (double *)calloc((size_t)p->sA * M, sizeof(double));
    m->qB = (double *)calloc((size_t)p->sB * M, sizeof(double));
    m->qBc = (double *)calloc((size_t)p->sB * M, sizeof(double));
    for (size_t i = 0; i < M; i++) { m->qA[i] = 1.0; m->qBc[i] = 1.0; }
    m->phiA = (double *)calloc(M, sizeof(double));
    m->phiB = (double *)calloc(M, sizeof(double));
    m->tmp1 = (double *)malloc(sizeof(double) * M);
    m->tmp2 = (double *)malloc(sizeof(double) * M);
    m->tmp3 = (double *)malloc(sizeof(double) * M);
    if (p->scft == 1) {
        fax_init(&m->axA, p->n_anderson, p->lamA, M, wA0);
        fax_init(&m->axB, p->n_anderson, p->lamB, M, wB0);
    } else {
        m->wA = (double *)malloc(sizeof(double) * M);
        m->wB = (double *)malloc(sizeof(double) * M);
        memcpy(m->wA, wA0, sizeof(double) * M);
        memcpy(m->wB, wB0, sizeof(double) * M);
    }
    if (!p->compressible) m->yita = (double *)calloc(M, sizeof(double));
    return m;
}

void orc_model_ab_destroy(orc_model_ab *m) {
    if (!m) return;
    orc_updater_destroy(m->upA); orc_updater_destroy(m->upB);
    free(m->qA); free(m->qAc); free(m->qB); free(m->qBc);
    free(m->phiA); free(m->phiB); free(m->tmp1); free(m->tmp2); free(m->tmp3);
    if (m->p.scft == 1) { fax_free(&m->axA); fax_free(&m->axB); }
    else { free(m->wA); free(m->wB); }
    free(m->yita);
    free(m);
}

/* Model_AB::update (Model_AB.cc:136-261), periodic cell, no NBC_by_PBC mirror */
int orc_model_ab_update(orc_model_ab *m) {
    size_t M = m->M;
    const orc_ab_params *p = &m->p;
    const double *wA = cur_wA(m), *wB = cur_wB(m);
    orc_updater_solve(m->upA, wA, m->qA, p->sA);
    memcpy(m->qB, m->qA + (size_t)(p->sA - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->upB, wB, m->qB, p->sB);
    orc_updater_solve(m->upB, wB, m->qBc, p->sB);
    memcpy(m->qAc, m->qBc + (size_t)(p->sB - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->upA, wA, m->qAc, p->sA);

    double Q = orc_mean(m->qB + (size_t)(p->sB - 1) * M, M);
    m->Q = Q;
    int rc = 0;
    rc |= orc_density(m->ruleA, m->qA, m->qAc, p->sA, M, m->dsA, 1.0 / Q, m->phiA);
    rc |= orc_density(m->ruleB, m->qB, m->qBc, p->sB, M, m->dsB, 1.0 / Q, m->phiB);
    m->last_rc = rc;

    const double chiN = p->chiN;
    if (p->compressible) {
        double *eta = m->tmp3;
        for (size_t i = 0; i < M; i++) eta[i] = p->lamYita * (m->phiA[i] + m->phiB[i] - 1.0);
        if (p->scft == 1) {
            for (size_t i = 0; i < M; i++) {
                m->tmp1[i] = chiN * m->phiB[i] + eta[i];
                m->tmp2[i] = chiN * m->phiA[i] + eta[i];
            }
        } else {
            for (size_t i = 0; i < M; i++) {
                m->wA[i] = m->wA[i] * (1.0 - p->lamA) + p->lamA * (chiN * m->phiB[i] + eta[i]);
                m->wB[i] = m->wB[i] * (1.0 - p->lamB) + p->lamB * (chiN * m->phiA[i] + eta[i]);
            }
            return rc;
        }
    } else {
        if (p->scft == 1) {
            for (size_t i = 0; i < M; i++)
                m->yita[i] = 0.5 * (m->axA.data[i] + m->axB.data[i] - chiN);
            for (size_t i = 0; i < M; i++) {
                m->tmp1[i] = chiN * m->phiB[i] + m->yita[i];
                m->tmp2[i] = chiN * m->phiA[i] + m->yita[i];
            }
        } else {
            for (size_t i = 0; i < M; i++) m->yita[i] += p->lamYita * (m->phiA[i] + m->phiB[i] - 1.0);
            for (size_t i = 0; i < M; i++) {
                m->wA[i] = m->wA[i] * (1.0 - p->lamA) + p->lamA * (chiN * m->phiB[i] + m->yita[i]);
                m->wB[i] = m->wB[i] * (1.0 - p->lamB) + p->lamB * (chiN * m->phiA[i] + m->yita[i]);
            }
            return rc;
        }
    }
    /* Anderson: pre_update x2, U = UA + UB, V = VA + VB, C = solve(U, V), update(C) */
    fax_pre_update(&m->axA, m->tmp1);
    fax_pre_update(&m->axB, m->tmp2);
    int nn = fax_nn(&m->axA);
    double U[64 * 64], V[64], C[64];
    memset(U, 0, sizeof(U)); memset(V, 0, sizeof(V));
    fax_add_UV(&m->axA, U, V);
    fax_add_UV(&m->axB, U, V);
    int nc = 0;
    if (nn > 0) {
        if (orc_solve_small(nn, U, V, C) != 0) rc |= 4;
        nc = nn;
    }
    fax_update(&m->axA, C, nc, m->tmp1, m->tmp2);
    fax_update(&m->axB, C, nc, m->tmp1, m->tmp2);
    return rc;
}

/* Model_AB::Hw / Hs / H (Model_AB.cc:263-300) */
void orc_model_ab_H(const orc_model_ab *m, double *H, double *Hw, double *Hs) {
    size_t M = m->M;
    const double *wA = cur_wA(m), *wB = cur_wB(m);
    double s = 0.0;
    for (size_t i = 0; i < M; i++) {
        double a = m->phiA[i], b = m->phiB[i];
        double g = m->p.chiN * a * b;
        if (m->p.compressible) g += m->p.lamYita / 2.0 * (a + b - 1.0) * (a + b - 1.0);
        g -= wA[i] * a;
        g -= wB[i] * b;
        s += g;
    }
    double hw = s / (double)M;
    double hs = -log(m->Q);
    *Hw = hw; *Hs = hs; *H = hw + hs;
}

/* Model_AB::residual_error (Model_AB.cc:307-371) */
double orc_model_ab_residual(const orc_model_ab *m) {
    size_t M = m->M;
    const orc_ab_params *p = &m->p;
    double res = 0.0;
    if (p->scft == 1) {
        /* current_d2_quadrature / current_w2_quadrature: slot cur_pos + 1 */
        int posA = m->axA.cur + 1; if (posA > m->axA.n) posA = 0;
        int posB = m->axB.cur + 1; if (posB > m->axB.n) posB = 0;
        const double *dA = m->axA.d + (size_t)posA * M, *dB = m->axB.d + (size_t)posB * M;
        const double *wA = m->axA.w + (size_t)posA * M, *wB = m->axB.w + (size_t)posB * M;
        double eA1 = 0, eA2 = 0, eB1 = 0, eB2 = 0;
        for (size_t i = 0; i < M; i++) { eA1 += dA[i] * dA[i]; eA2 += wA[i] * wA[i]; }
        for (size_t i = 0; i < M; i++) { eB1 += dB[i] * dB[i]; eB2 += wB[i] * wB[i]; }
        eA1 /= (double)M; eA2 /= (double)M; eB1 /= (double)M; eB2 /= (double)M;
        return sqrt((eA1 + eB1) / (eA2 + eB2));
    }
    double *g1 = m->tmp1, *g2 = m->tmp2;
    const double chiN = p->chiN;
    if (!p->compressible) {
        for (size_t i = 0; i < M; i++) { g1[i] = chiN * m->phiB[i] + m->yita[i]; g2[i] = g1[i] - m->wA[i]; }
        res += mean_abs(g2, M) / (mean_abs(m->wA, M) + mean_abs(g1, M));
        for (size_t i = 0; i < M; i++) { g1[i] = chiN * m->phiA[i] + m->yita[i]; g2[i] = g1[i] - m->wB[i]; }
        res += mean_abs(g2, M) / (mean_abs(m->wB, M) + mean_abs(g1, M));
        for (size_t i = 0; i < M; i++) { g1[i] = m->phiA[i] + m->phiB[i]; g2[i] = g1[i] - 1.0; }
        res += mean_abs(g2, M) / (1.0 + mean_abs(g1, M));
        res /= 3.0;
    } else {
        for (size_t i = 0; i < M; i++) {
            g1[i] = chiN * m->phiB[i] + p->lamYita * (m->phiA[i] + m->phiB[i] - 1.0);
            g2[i] = g1[i] - m->wA[i];
        }
        res += mean_abs(g2, M) / (mean_abs(m->wA, M) + mean_abs(g1, M));
        for (size_t i = 0; i < M; i++) {
            g1[i] = chiN * m->phiA[i] + p->lamYita * (m->phiA[i] + m->phiB[i] - 1.0);
            g2[i] = g1[i] - m->wB[i];
        }
        res += mean_abs(g2, M) / (mean_abs(m->wB, M) + mean_abs(g1, M));
        res /= 2.0;
    }
    return res;
}

double orc_model_ab_Q(const orc_model_ab *m) { return m->Q; }
int orc_model_ab_last_rc(const orc_model_ab *m) { return m->last_rc; }

/* copy state out: which = 0 wA, 1 wB, 2 phiA, 3 phiB, 4 yita,
 * 5 qA history (sA*M), 6 qB, 7 qAc, 8 qBc */
int orc_model_ab_get(const orc_model_ab *m, int which, double *out) {
    size_t M = m->M;
    switch (which) {
    case 0: memcpy(out, cur_wA(m), sizeof(double) * M); return 0;
    case 1: memcpy(out, cur_wB(m), sizeof(double) * M); return 0;
    case 2: memcpy(out, m->phiA, sizeof(double) * M); return 0;
    case 3: memcpy(out, m->phiB, sizeof(double) * M); return 0;
    case 4: if (!m->yita) return -1; memcpy(out, m->yita, sizeof(double) * M); return 0;
    case 5: memcpy(out, m->qA, sizeof(double) * M * m->p.sA); return 0;
    case 6: memcpy(out, m->qB, sizeof(double) * M * m->p.sB); return 0;
    case 7: memcpy(out, m->qAc, sizeof(double) * M * m->p.sA); return 0;
    case 8: memcpy(out, m->qBc, sizeof(double) * M * m->p.sB); return 0;
    }
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Model_ABC: linear A-B-C triblock melt (defined here; the reference has no  */
/* periodic ABC melt model).  It extends Model_AB term by term:               */
/*   chain A (sA slices) - B (sB) - C (sC), L = LA + LB + LC, fX = LX / L,    */
/*   dsX = fX / LX; forward qA -> qB -> qC from 1, complementary qCc -> qBc ->*/
/*   qAc from 1; Q = mean(qC[sC-1]); phiX = density(ruleX, qX, qXc) / Q;      */
/*   targets  wA* = xAB phiB + xAC phiC + eta, wB* = xAB phiA + xBC phiC + eta,*/
/*            wC* = xAC phiA + xBC phiB + eta;                                */
/*   EM:       eta += lam_eta (phiA + phiB + phiC - 1), wX += lamX (wX* - wX)  */
/*             (Model_AB.cc:184-193, 254-259 with a third field);             */
/*   Anderson: eta = (wA + wB + wC - xAB (phiA + phiB) - xBC (phiB + phiC)    */
/*             - xAC (phiA + phiC)) / 3, the value that makes the targets sum */
/*             to the current fields (Model_AB's 0.5 (wA + wB - chiN) is the  */
/*             two-block case with phiA + phiB = 1); one ring per field, one  */
/*             coefficient set from U = UA + UB + UC, V = VA + VB + VC;       */
/*   Hw = mean(xAB phiA phiB + xBC phiB phiC + xAC phiA phiC - sum wX phiX),  */
/*   Hs = -ln Q;  residual as Model_AB's (Anderson: sqrt(sum d^2 / sum w^2);  */
/*   EM: mean of the three field terms and the incompressibility term).       */
/* Incompressible, RQM4 only.                                                 */
/* ------------------------------------------------------------------------ */
typedef struct {
    int dim, Lx, Ly, Lz;
    int s[3];             /* sA, sB, sC */
    double chi[3];        /* xAB, xBC, xAC (times N) */
    double lam[4];        /* lamA, lamB, lamC, lamYita */
    int scft;             /* 0 = EM, 1 = Anderson */
    int n_anderson;
    int contour;          /* 0 = trapezoid, 1 = Simpson (Simpson/Quad4 by parity) */
    const double *k2;     /* -k^2 table (calc_k2_orthogonal), M values */
} orc_abc_params;

typedef struct {
    orc_abc_params p;
    size_t M;
    double ds[3];
    int rule[3];
    orc_updater *up[3];
    double *q[3], *qc[3];              /* histories: forward and complementary, block X */
    double *w[3], *yita;               /* EM fields */
    orc_fieldax ax[3];                 /* Anderson fields */
    double *phi[3];
    double Q;
    double *tgt[3];
    int last_rc;
} orc_model_abc;

static const double *abc_w(const orc_model_abc *m, int x) { return m->p.scft == 1 ? m->ax[x].data : m->w[x]; }

orc_model_abc *orc_model_abc_create(const orc_abc_params *p, const double *wA0, const double *wB0,
                                    const double *wC0) {
    orc_model_abc *m = (orc_model_abc *)calloc(1, sizeof(orc_model_abc));
    m->p = *p;
    size_t M = (size_t)p->Lx * p->Ly * p->Lz;
    m->M = M;
    int L[3] = {p->s[0] - 1, p->s[1] - 1, p->s[2] - 1};
    int Lt = L[0] + L[1] + L[2];
    const double *w0[3] = {wA0, wB0, wC0};
    for (int x = 0; x < 3; x++) {
        double f = 1.0 * L[x] / Lt;
        m->ds[x] = f / L[x];
        m->rule[x] = p->contour == 0 ? ORC_TRAPEZOID : ((p->s[x] % 2 != 0) ? ORC_SIMPSON : ORC_QUAD4_CLOSED);
        m->up[x] = orc_rqm4_create(p->k2, p->Lx, p->Ly, p->Lz, m->ds[x]);
        m->q[x] = (double *)calloc((size_t)p->s[x] * M, sizeof(double));
        m->qc[x] = (double *)calloc((size_t)p->s[x] * M, sizeof(double));
        m->phi[x] = (double *)calloc(M, sizeof(double));
        m->tgt[x] = (double *)malloc(sizeof(double) * M);
        if (p->scft == 1) {
            fax_init(&m->ax[x], p->n_anderson, p->lam[x], M, w0[x]);
        } else {
            m->w[x] = (double *)malloc(sizeof(double) * M);
            memcpy(m->w[x], w0[x], sizeof(double) * M);
        }
    }
    for (size_t i = 0; i < M; i++) { m->q[0][i] = 1.0; m->qc[2][i] = 1.0; }
    m->yita = (double *)calloc(M, sizeof(double));
    return m;
}

void orc_model_abc_destroy(orc_model_abc *m) {
    if (!m) return;
    for (int x = 0; x < 3; x++) {
        orc_updater_destroy(m->up[x]);
        free(m->q[x]); free(m->qc[x]); free(m->phi[x]); free(m->tgt[x]);
        if (m->p.scft == 1) fax_free(&m->ax[x]); else free(m->w[x]);
    }
    free(m->yita);
    free(m);
}

/* the three targets wX* for the current phi and eta */
static void abc_targets(orc_model_abc *m, const double *eta) {
    const double xab = m->p.chi[0], xbc = m->p.chi[1], xac = m->p.chi[2];
    for (size_t i = 0; i < m->M; i++) {
        double a = m->phi[0][i], b = m->phi[1][i], c = m->phi[2][i];
        m->tgt[0][i] = xab * b + xac * c + eta[i];
        m->tgt[1][i] = xab * a + xbc * c + eta[i];
        m->tgt[2][i] = xac * a + xbc * b + eta[i];
    }
}

int orc_model_abc_update(orc_model_abc *m) {
    size_t M = m->M;
    const orc_abc_params *p = &m->p;
    const int *s = p->s;
    /* forward A -> B -> C */
    orc_updater_solve(m->up[0], abc_w(m, 0), m->q[0], s[0]);
    memcpy(m->q[1], m->q[0] + (size_t)(s[0] - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->up[1], abc_w(m, 1), m->q[1], s[1]);
    memcpy(m->q[2], m->q[1] + (size_t)(s[1] - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->up[2], abc_w(m, 2), m->q[2], s[2]);
    /* complementary C -> B -> A */
    orc_updater_solve(m->up[2], abc_w(m, 2), m->qc[2], s[2]);
    memcpy(m->qc[1], m->qc[2] + (size_t)(s[2] - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->up[1], abc_w(m, 1), m->qc[1], s[1]);
    memcpy(m->qc[0], m->qc[1] + (size_t)(s[1] - 1) * M, sizeof(double) * M);
    orc_updater_solve(m->up[0], abc_w(m, 0), m->qc[0], s[0]);

    double Q = orc_mean(m->q[2] + (size_t)(s[2] - 1) * M, M);
    m->Q = Q;
    int rc = 0;
    for (int x = 0; x < 3; x++) rc |= orc_density(m->rule[x], m->q[x], m->qc[x], s[x], M, m->ds[x], 1.0 / Q, m->phi[x]);
    m->last_rc = rc;

    const double xab = p->chi[0], xbc = p->chi[1], xac = p->chi[2];
    if (p->scft == 0) {
        for (size_t i = 0; i < M; i++) m->yita[i] += p->lam[3] * (m->phi[0][i] + m->phi[1][i] + m->phi[2][i] - 1.0);
        abc_targets(m, m->yita);
        for (int x = 0; x < 3; x++)
            for (size_t i = 0; i < M; i++) m->w[x][i] = m->w[x][i] * (1.0 - p->lam[x]) + p->lam[x] * m->tgt[x][i];
        return rc;
    }
    for (size_t i = 0; i < M; i++) {
        double a = m->phi[0][i], b = m->phi[1][i], c = m->phi[2][i];
        double sw = m->ax[0].data[i] + m->ax[1].data[i] + m->ax[2].data[i];
        m->yita[i] = (sw - xab * (a + b) - xbc * (b + c) - xac * (a + c)) / 3.0;
    }
    abc_targets(m, m->yita);
    for (int x = 0; x < 3; x++) fax_pre_update(&m->ax[x], m->tgt[x]);
    int nn = fax_nn(&m->ax[0]);
    double U[64 * 64], V[64], C[64];
    memset(U, 0, sizeof(U)); memset(V, 0, sizeof(V));
    for (int x = 0; x < 3; x++) fax_add_UV(&m->ax[x], U, V);
    int nc = 0;
    if (nn > 0) {
        if (orc_solve_small(nn, U, V, C) != 0) rc |= 4;
        nc = nn;
    }
    double *W = (double *)malloc(sizeof(double) * M), *D = (double *)malloc(sizeof(double) * M);
    for (int x = 0; x < 3; x++) fax_update(&m->ax[x], C, nc, W, D);
    free(W); free(D);
    return rc;
}

void orc_model_abc_H(const orc_model_abc *m, double *H, double *Hw, double *Hs) {
    size_t M = m->M;
    const double xab = m->p.chi[0], xbc = m->p.chi[1], xac = m->p.chi[2];
    const double *wa = abc_w(m, 0), *wb = abc_w(m, 1), *wc = abc_w(m, 2);
    double sum = 0.0;
    for (size_t i = 0; i < M; i++) {
        double a = m->phi[0][i], b = m->phi[1][i], c = m->phi[2][i];
        double g = xab * a * b + xbc * b * c + xac * a * c;
        g -= wa[i] * a;
        g -= wb[i] * b;
        g -= wc[i] * c;
        sum += g;
    }
    double hw = sum / (double)M, hs = -log(m->Q);
    *Hw = hw; *Hs = hs; *H = hw + hs;
}

double orc_model_abc_residual(const orc_model_abc *m) {
    size_t M = m->M;
    if (m->p.scft == 1) {
        double e1 = 0.0, e2 = 0.0;
        for (int x = 0; x < 3; x++) {
            int pos = m->ax[x].cur + 1; if (pos > m->ax[x].n) pos = 0;
            const double *d = m->ax[x].d + (size_t)pos * M, *w = m->ax[x].w + (size_t)pos * M;
            double a1 = 0.0, a2 = 0.0;
            for (size_t i = 0; i < M; i++) { a1 += d[i] * d[i]; a2 += w[i] * w[i]; }
            e1 += a1 / (double)M;
            e2 += a2 / (double)M;
        }
        return sqrt(e1 / e2);
    }
    /* EM: the targets of the fields after the update (this iteration's phi, eta) */
    orc_model_abc *mm = (orc_model_abc *)m;
    abc_targets(mm, m->yita);
    double res = 0.0;
    double *g = (double *)malloc(sizeof(double) * M);
    for (int x = 0; x < 3; x++) {
        for (size_t i = 0; i < M; i++) g[i] = m->tgt[x][i] - m->w[x][i];
        res += mean_abs(g, M) / (mean_abs(m->w[x], M) + mean_abs(m->tgt[x], M));
    }
    double *t = (double *)malloc(sizeof(double) * M);
    for (size_t i = 0; i < M; i++) { t[i] = m->phi[0][i] + m->phi[1][i] + m->phi[2][i]; g[i] = t[i] - 1.0; }
    res += mean_abs(g, M) / (1.0 + mean_abs(t, M));
    free(g); free(t);
    return res / 4.0;
}

double orc_model_abc_Q(const orc_model_abc *m) { return m->Q; }

/* which = 0..2 wA, wB, wC; 3..5 phiA, phiB, phiC; 6 yita */
int orc_model_abc_get(const orc_model_abc *m, int which, double *out) {
    size_t M = m->M;
    if (which >= 0 && which < 3) { memcpy(out, abc_w(m, which), sizeof(double) * M); return 0; }
    if (which >= 3 && which < 6) { memcpy(out, m->phi[which - 3], sizeof(double) * M); return 0; }
    if (which == 6) { memcpy(out, m->yita, sizeof(double) * M); return 0; }
    return -1;
}

/* ------------------------------------------------------------------------ */
/* String method: arc length and per-point natural cubic spline              */
/* ------------------------------------------------------------------------ */
/* parameterize_string (polystring_AB.cc:283-296): S[0] = 0,
 * S[s] = S[s-1] + sqrt(mean((wa[s]-wa[s-1])^2)), normalised by S[m-1]. */
void orc_string_arclength(const double *wa, int m, size_t M, double *S) {
    S[0] = 0.0;
    for (int s = 1; s < m; s++) {
        const double *a = wa + (size_t)s * M, *b = wa + (size_t)(s - 1) * M;
        double acc = 0.0;
        for (size_t i = 0; i < M; i++) { double d = a[i] - b[i]; acc += d * d; }
        S[s] = S[s - 1] + sqrt(acc / (double)M);
    }
    double last = S[m - 1];
    for (int s = 0; s < m; s++) S[s] = 1.0 * S[s] / last;
}

/* Natural cubic spline through (x[i], y[i]), evaluated at t[z] = z/(m-1).
 * Piece i on [x_i, x_{i+1}] is y_i + c_i h + b_i h^2 + a_i h^3 with
 * b = half the second derivative, b_0 = b_{m-1} = 0 (zero end curvature,
 * the default of the spline used by polystring_AB.cc:298-319).  The
 * tridiagonal system for b is solved by forward elimination and back
 * substitution.  An abscissa equal to a knot x_i (i > 0) is evaluated on
 * the piece to its left, and the last knot with the last piece. */
static void natural_spline_resample(const double *x, const double *y, int m,
                                    double *b, double *cp, double *out) {
    /* rows i = 1..m-2: h_{i-1}/3 b_{i-1} + 2(h_{i-1}+h_i)/3 b_i + h_i/3 b_{i+1}
     *                  = (y_{i+1}-y_i)/h_i - (y_i-y_{i-1})/h_{i-1}            */
    double *rhs = out;  /* scratch; overwritten by the results at the end */
    b[0] = 0.0; b[m - 1] = 0.0;
    cp[0] = 0.0; rhs[0] = 0.0;
    for (int i = 1; i < m - 1; i++) {
        double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
        double lo = hl / 3.0, di = 2.0 * (x[i + 1] - x[i - 1]) / 3.0, up = hr / 3.0;
        double r = (y[i + 1] - y[i]) / hr - (y[i] - y[i - 1]) / hl;
        double den = di - lo * cp[i - 1];
        cp[i] = up / den;
        rhs[i] = (r - lo * rhs[i - 1]) / den;
    }
    for (int i = m - 2; i >= 1; i--) b[i] = rhs[i] - cp[i] * b[i + 1];
    for (int z = 0; z < m; z++) {
        double t = 1.0 * z / (m - 1);
        int idx = 0;
        while (idx < m - 1 && x[idx + 1] < t) idx++;   /* first knot >= t, minus one */
        if (idx > m - 2) idx = m - 2;
        double h = t - x[idx];
        double hi = x[idx + 1] - x[idx];
        double a = (b[idx + 1] - b[idx]) / (3.0 * hi);
        double c = (y[idx + 1] - y[idx]) / hi - (2.0 * b[idx] + b[idx + 1]) * hi / 3.0;
        out[z] = ((a * h + b[idx]) * h + c) * h + y[idx];
    }
}

/* redistribute_stringBeads (polystring_AB.cc:298-329) for one field:
 * f is m x M (image-major); ends are restored from the stored end images. */
int orc_string_redistribute(double *f, const double *S, int m, size_t M,
                            const double *end0, const double *end1) {
    if (m < 3 || m > 4096) return -1;
    double *y = (double *)malloc(sizeof(double) * (size_t)m * 4);
    double *b = y + m, *cp = b + m, *out = cp + m;
    for (size_t i = 0; i < M; i++) {
        for (int z = 0; z < m; z++) y[z] = f[(size_t)z * M + i];
        natural_spline_resample(S, y, m, b, cp, out);
        for (int z = 0; z < m; z++) f[(size_t)z * M + i] = out[z];
    }
    free(y);
    memcpy(f, end0, sizeof(double) * M);
    memcpy(f + (size_t)(m - 1) * M, end1, sizeof(double) * M);
    return 0;
}
