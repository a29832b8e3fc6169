/*
 * nlo_oracle.c -- CPU FP64 restatement of the reference NLO BK hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * nlo_bk_optimized_b200/csrc: tests, __graft_entry__.smoke() and the bench's
 * CPU-baseline leg call it; nothing on the product path links or executes it.
 *
 * It restates, in plain C, the algorithm of the reference package
 * (HaowuDuan/nlo_bk_optimized, torch_nlo_clean/src/nlo_torch):
 *
 *   coupling              coupling.py:10-46, 81-97     (bk_alpha_s: fixed, smooth
 *                         freeze for NF <= 3, flavour thresholds for NF = 5)
 *   natural cubic spline  numerics/interpolation.py:10-92, 124-149
 *   log-log spline        numerics/interpolation.py:95-121
 *   edge rules            bk/derivatives.py:761-772     (_evaluate_loglog)
 *   K1 pointwise kernel   bk_kernels/k1.py:20-155       (Kernel_lo: every Order,
 *                         RC_LO and RESUM_RC; production NLO_RESUM_DLOG_SLOG,
 *                         BALITSKY_LO, RESUM_RC_SMALLEST)
 *   K1 integrand          bk/derivatives.py:434-468     (_lo_integrand)
 *   kinematical constr.   bk/derivatives.py:469-487, 712-758 (shifted rapidity,
 *                         6-point natural splines of the history rows in r,
 *                         linear in y)
 *   K1 fixed rule         custom_kernels/bk/k1/kernel.cu:2040-2092
 *                         (8 GL nodes in log z per r-grid interval x 24 GL nodes
 *                          in v with theta = pi v^2)
 *   K2 / Kf kernels       bk_kernels/k2.py:8-39, bk_kernels/kf.py:10-41
 *   K2+Kf integrand       bk/derivatives.py:490-612     (_nlo_integrand) and the
 *                         log-variable Jacobian at bk/derivatives.py:322-335
 *   K2+Kf box             bk/derivatives.py:424-431     (nlo_vegas_bounds)
 *   K2+Kf coupling        bk/derivatives.py:615-632     (_nlo_alpha_s: smallest
 *                         size, or the parent for PARENT_NLO)
 *   dN/dY assembly        bk/evolution.py:329-351, 354-488
 *   steppers              bk/evolution.py:110-122 (Euler), 190-236 (Kutta RK3);
 *                         RK4 is the classical four-stage rule (no reference
 *                         counterpart) wrapped around the same derivative.
 *   Sobol points          torch.quasirandom.SobolEngine (torch 2.11), used by
 *                         dis/fixed_sobol.py:87-92: Gray-code XOR of the engine's
 *                         scrambled direction numbers, scaled by 2^-30.
 *
 * Numerical form.  The reference evaluates K2/Kf and the Balitsky LO kernel as
 * differences of O(1/|z-z'|^4) (resp. O(1/z^2)) terms whose true value is
 * O(r^2); in FP64 those differences lose all precision for r below ~1e-4.
 * This restatement uses algebraically identical, cancellation-free forms:
 *   X^2 = (r-z)^2 + 4 r z sin^2(theta/2)                  (k1/kernel.cu:467-470)
 *   a - b = XY2^2 - X2Y^2 = r [ r (z'^2 - z^2) - 2 z z' (z' cos th - z cos th') ]
 *   log(a/b)/(a-b) = 2 h(t)/(a+b),  h(t) = atanh(t)/t,  t = (a-b)/(a+b)
 *   (a+b) log(a/b)/(a-b) - 2 = 2 (h(t) - 1)
 *   alpha_Y - alpha_X from log1p/expm1 of the exact X^2 - Y^2
 *   S = 1 - N stored as log S = log1p(-N); N = -expm1(log S)
 * The quad-precision functions at the end evaluate the reference's literal
 * formulas; tests use them to show that the two forms agree wherever the
 * literal one is well conditioned and that the stable one is the exact value
 * elsewhere.
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.14159265358979323846
#define OR_MIN_LOG (-40.0) /* interpolation.py:8 MIN_LOG_VALUE */

double or_bessel_i1(double x);

typedef struct or_physics {
    double nc;            /* BKConfig.NC */
    double nf;            /* BKConfig.NF */
    double lambda_qcd;    /* BKConfig.LambdaQCD */
    double c2;            /* BKConfig.C2 */
    double minr;          /* BKConfig.MINR (double-log switch, k1.py:117) */
    double ksub;          /* BKConfig.KSUB */
    int symmetrize;       /* BKConfig.SYMMETRIZE_Z_Z2_INTEGRATION */
    int fixed_coupling;   /* RC_LO/RC_NLO FIXED */
    double fixed_alpha_s; /* BKConfig.FIXED_AS */
    double alpha_cap;     /* >0: cap alpha_s at this value (frozen variant) */
    int order;            /* Order: 0 NLO_RESUM_DLOG_SLOG, 1 NLO_RESUM_DLOG, 2 NLO,
                             3 LO_RESUM_DLOG_SLOG, 4 LO_RESUM_DLOG, 5 LO */
    int rc_lo;            /* RC_LO: 0 BALITSKY (and FIXED), 1 PARENT, 2 SMALLEST, 3 FAC, 4 BEUF */
    int resum_rc;         /* RESUM_RC: 0 SMALLEST, 1 PARENT, 2 FIXED */
    int rc_nlo;           /* RC_NLO: 0 SMALLEST (and FIXED), 1 PARENT */
} or_physics;

/* One log-log spline over the r grid: knots x = log r, coefficients per interval. */
typedef struct or_spline {
    int n;              /* knots */
    const double* x;    /* [n] log r_i */
    const double* a;    /* [n-1] */
    const double* b;
    const double* c;
    const double* d;
    double rmin, rmax;  /* r_grid[0], r_grid[n-1] */
} or_spline;

/* ------------------------------------------------------------------------ */
/* coupling.py:81-97 (_smooth_alpha_s): 1/(b0 * c * logaddexp(2/c log mu0, log scale / c)) */
static double alpha_thresholds(double r, const or_physics* p)
{
    /* coupling.py:25-45: Nf = 3/4/5 by 4 C2/r^2 against 1.3^2 and 4.5^2 */
    const double dipolescale = 4.0 * p->c2 / (r * r);
    const double nf = dipolescale < 1.3 * 1.3 ? 3.0 : (dipolescale < 4.5 * 4.5 ? 4.0 : 5.0);
    const double lambda = nf == 3.0 ? 0.146159 : (nf == 4.0 ? 0.122944 : 0.0904389);
    const double b0 = 11.0 - 2.0 * nf / 3.0;
    const double log_arg = 4.0 * p->c2 / (r * r * lambda * lambda);
    const double a = 4.0 * OR_PI / (b0 * log(log_arg));
    return (log_arg < 1.0 || a > 1.0) ? 1.0 : a;
}

static double alpha_from_log_distance(double log_d, const or_physics* p)
{
    if (p->fixed_coupling) return p->fixed_alpha_s;
    if (p->nf > 3.0) return alpha_thresholds(exp(log_d), p);
    const double b0 = (11.0 * p->nc - 2.0 * p->nf) / (12.0 * OR_PI);
    const double c = 0.2;
    const double left = 2.0 / c * log(2.5);
    /* log scale = log(4 C2 / (d^2 Lambda^2)) */
    const double log_scale = log(4.0 * p->c2 / (p->lambda_qcd * p->lambda_qcd)) - 2.0 * log_d;
    const double right = log_scale / c;
    const double m = fmax(left, right);
    const double lae = m + log1p(exp(-fabs(left - right)));
    double a = 1.0 / (b0 * c * lae);
    if (p->alpha_cap > 0.0 && a > p->alpha_cap) a = p->alpha_cap;
    return a;
}

double or_alpha_s(double r, const or_physics* p) { return alpha_from_log_distance(log(r), p); }

/* logaddexp(c, t + delta) - logaddexp(c, t) without cancellation.
 * With sigma = e^t/(e^c + e^t) the difference is log(1 + sigma expm1(delta))
 * = log((1 - sigma) + sigma e^delta); the second form is used when the
 * argument of log1p would be close to -1. */
static double lae_difference(double c, double t, double delta)
{
    const double sigma = 1.0 / (1.0 + exp(c - t));
    const double v = sigma * expm1(delta);
    if (v > -0.5) return log1p(v);
    const double sigma_c = 1.0 / (1.0 + exp(t - c));
    return log(sigma_c + sigma * exp(delta));
}

/* ------------------------------------------------------------------------ */
/* interpolation.py:10-92 + 124-149: natural cubic spline via the Thomas algorithm. */
void or_natural_spline(const double* x, const double* y, int n,
                       double* a, double* b, double* c, double* d)
{
    const int m = n - 2; /* interior second derivatives */
    double* h = (double*)malloc(sizeof(double) * (size_t)(n - 1));
    double* upper = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* sol = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* second = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n - 1; ++i) h[i] = x[i + 1] - x[i];
    /* diagonal_i = 2 (h_i + h_{i+1}); off_i = h_{i+1}; rhs_i = 6 (slope_{i+1} - slope_i) */
    if (m == 1) {
        const double rhs = 6.0 * ((y[2] - y[1]) / h[1] - (y[1] - y[0]) / h[0]);
        sol[0] = rhs / (2.0 * (h[0] + h[1]));
    } else if (m > 1) {
        double diag = 2.0 * (h[0] + h[1]);
        upper[0] = h[1] / diag;
        sol[0] = 6.0 * ((y[2] - y[1]) / h[1] - (y[1] - y[0]) / h[0]) / diag;
        for (int i = 1; i < m; ++i) {
            const double off = h[i];
            const double denom = 2.0 * (h[i] + h[i + 1]) - off * upper[i - 1];
            if (i < m - 1) upper[i] = h[i + 1] / denom;
            const double rhs = 6.0 * ((y[i + 2] - y[i + 1]) / h[i + 1] - (y[i + 1] - y[i]) / h[i]);
            sol[i] = (rhs - off * sol[i - 1]) / denom;
        }
        for (int i = m - 2; i >= 0; --i) sol[i] -= upper[i] * sol[i + 1];
    }
    second[0] = 0.0;
    second[n - 1] = 0.0;
    for (int i = 0; i < m; ++i) second[i + 1] = sol[i];
    for (int i = 0; i < n - 1; ++i) {
        a[i] = y[i];
        b[i] = (y[i + 1] - y[i]) / h[i] - h[i] * (2.0 * second[i] + second[i + 1]) / 6.0;
        c[i] = second[i] / 2.0;
        d[i] = (second[i + 1] - second[i]) / (6.0 * h[i]);
    }
    free(h); free(upper); free(sol); free(second);
}

/*
 * Knot values of the two evolution splines (evolution.py:548-560):
 *   kind 0: log N with N clamped to [0,1] (the lower clamp only with force_positive)
 *   kind 1: log S with S = 1 - N clamped to [0,1] (the upper clamp only with
 *           force_positive); computed as log1p(-N) so that S near 1 keeps the
 *           relative precision of N.
 * Non-positive values map to -40 (interpolation.py:8,113).
 */
void or_loglog_knots(const double* N, int n, int kind, int force_positive, double* out)
{
    for (int i = 0; i < n; ++i) {
        double v = N[i];
        if (kind == 0) {
            if (v > 1.0) v = 1.0;
            if (force_positive && v < 0.0) v = 0.0;
            out[i] = v > 0.0 ? log(v) : OR_MIN_LOG;
        } else {
            /* S = 1 - N; S < 0 -> 0; force_positive: S > 1 -> 1 (i.e. N < 0 -> N = 0) */
            double nn = v;
            if (force_positive && nn < 0.0) nn = 0.0;
            out[i] = nn < 1.0 ? log1p(-nn) : OR_MIN_LOG;
        }
    }
}

static inline int spline_interval(const or_spline* s, double lx)
{
    /* searchsorted(x, lx, right=True) - 1, clamped to [0, n-2] */
    int lo = 0, hi = s->n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (lx >= s->x[mid]) lo = mid + 1; else hi = mid;
    }
    int i = lo - 1;
    if (i < 0) i = 0;
    if (i > s->n - 2) i = s->n - 2;
    return i;
}

static inline double spline_poly(const or_spline* s, double lx)
{
    const int i = spline_interval(s, lx);
    const double dx = lx - s->x[i];
    return s->a[i] + dx * (s->b[i] + dx * (s->c[i] + dx * s->d[i]));
}

/* N from the log N spline, with the edge rules of derivatives.py:761-772
 * (0 below r_min, 1 above r_max, non-finite -> 0) and min(., 1) (derivatives.py:452-463). */
double or_n_from_nspline(const or_spline* s, double r)
{
    if (r < s->rmin) return 0.0;
    if (r > s->rmax) return 1.0;
    double v = exp(spline_poly(s, log(r)));
    if (!isfinite(v)) v = 0.0;
    return v < 1.0 ? v : 1.0;
}

/* N = 1 - S from the log S spline (edge rules: S = 1 below r_min, 0 above r_max). */
double or_n_from_sspline(const or_spline* s, double r)
{
    if (r < s->rmin) return 0.0;
    if (r > s->rmax) return 1.0;
    const double p = spline_poly(s, log(r));
    const double sv = exp(p);
    if (!isfinite(sv)) return 1.0; /* S non-finite -> S = 0 */
    return -expm1(p);
}

/* Amplitude at one distance with its log-spline value, so that differences of
 * nearby amplitudes can be formed without cancellation. */
typedef struct nsv {
    double p;  /* spline value (log N or log S); meaningful when edge == 0 */
    double N;
    double S;
    int edge;  /* -1 below r_min, 0 inside, +1 above r_max */
} nsv;

/* log S spline (K2+Kf): S = 1 below r_min, 0 above r_max, non-finite S -> 0. */
static nsv eval_s(const or_spline* s, double r)
{
    nsv v;
    if (r < s->rmin) { v.p = 0.0; v.N = 0.0; v.S = 1.0; v.edge = -1; return v; }
    if (r > s->rmax) { v.p = 0.0; v.N = 1.0; v.S = 0.0; v.edge = 1; return v; }
    v.edge = 0;
    v.p = spline_poly(s, log(r));
    v.S = exp(v.p);
    if (!isfinite(v.S)) { v.S = 0.0; v.N = 1.0; v.edge = 1; return v; }
    v.N = -expm1(v.p);
    return v;
}

/* N_A - N_B = S_B - S_A = S_A expm1(p_B - p_A) for log S values. */
static double ndiff_s(const nsv* A, const nsv* B)
{
    if (A->edge == 0 && B->edge == 0) return A->S * expm1(B->p - A->p);
    /* one side clamped: subtract whichever representation is small */
    if (A->N < 0.5 && B->N < 0.5) return A->N - B->N;
    return B->S - A->S;
}

/* Spline value at lx minus the knot value a_i, without cancellation when lx
 * lies in interval i or i-1 (Taylor form of the cubic about knot i). */
static double spline_delta_from_knot(const or_spline* s, int i, double lx)
{
    if (lx < s->x[0]) lx = s->x[0];
    if (lx > s->x[s->n - 1]) lx = s->x[s->n - 1];
    const int j = spline_interval(s, lx);
    const double dx = lx - s->x[i];
    if (j == i) return dx * (s->b[i] + dx * (s->c[i] + dx * s->d[i]));
    if (j == i - 1) {
        const double h = s->x[i] - s->x[i - 1];
        const double b1 = s->b[i - 1] + h * (2.0 * s->c[i - 1] + 3.0 * h * s->d[i - 1]);
        const double c1 = s->c[i - 1] + 3.0 * h * s->d[i - 1];
        return dx * (b1 + dx * (c1 + dx * s->d[i - 1]));
    }
    return spline_poly(s, lx) - s->a[i];
}

/* K1 dipole N_X + N_Y - N_r - N_X N_Y for a parent at knot i of the log N
 * spline (derivatives.py:452-467 with the min(N, 1) clamps), written as
 * S_r (N_Y + D_X) - D_X D_Y with D = N - N_r from spline differences. */
static double k1_dipole(const or_spline* s, int i, double X, double Y)
{
    const double pr = s->a[i] ; /* value at knot i */
    const double Nr = fmin(exp(pr), 1.0);
    const double Sr = pr < 0.0 ? -expm1(pr) : 0.0;
    double N[2], D[2];
    const double dist[2] = {X, Y};
    for (int k = 0; k < 2; ++k) {
        const double x = dist[k];
        if (x < s->rmin) { N[k] = 0.0; D[k] = -Nr; continue; }
        if (x > s->rmax) { N[k] = 1.0; D[k] = Sr; continue; }
        const double dp = spline_delta_from_knot(s, i, log(x));
        const double pv = pr + dp;
        double nv = exp(pv);
        if (!isfinite(nv)) nv = 0.0;
        if (nv >= 1.0) { N[k] = 1.0; D[k] = Sr; continue; }
        N[k] = nv;
        D[k] = Nr * expm1(dp);
    }
    const double base = N[1] <= N[0] ? N[1] + D[0] : N[0] + D[1];
    return Sr * base - D[0] * D[1];
}

static int knot_index(const or_spline* s, double r)
{
    /* the parent sizes of the evolution are grid points; return the nearest knot */
    const double lr = log(r);
    int i = spline_interval(s, lr);
    if (i + 1 < s->n && fabs(s->x[i + 1] - lr) < fabs(s->x[i] - lr)) i = i + 1;
    return i;
}

/* ------------------------------------------------------------------------ */
/* K1: Kernel_lo (k1.py:20-155) x dipole (derivatives.py:452-468), stable form.
 * RC_LO picks the kernel (k1.py:37-94); Order LO and NLO stop at the bare kernel
 * (k1.py:97-98); RESUM_RC picks the resummation coupling (k1.py:100-107). */
static double kernel_lo_value(double r, double z, double theta, const or_physics* p)
{
    const double sh = sin(0.5 * theta);
    const double s2 = sh * sh;
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * s2;
    if (Xsq < 1e-40 || z < 1e-20 || r < 1e-20) return 0.0;
    const double X = sqrt(Xsq);
    const double Y = z;
    const double Ysq = z * z;
    const double nc = p->nc;

    const double log_r = log(r), log_X = 0.5 * log(Xsq), log_Y = log(z);
    const double alpha_r = alpha_from_log_distance(log_r, p);
    const double alpha_X = alpha_from_log_distance(log_X, p);
    const double alpha_Y = alpha_from_log_distance(log_Y, p);
    const double log_min = fmin(fmin(log_X, log_Y), log_r);
    const double alpha_min = alpha_from_log_distance(log_min, p);

    /* X^2 - Y^2 = r (r - 2 z cos theta), exact. */
    const double cos_t = 1.0 - 2.0 * s2;
    const double XmY = r * (r - 2.0 * z * cos_t);
    /* alpha_Y - alpha_X without cancellation for the smooth coupling (fixed: 0). */
    double dalpha = 0.0;
    if (!p->fixed_coupling && p->alpha_cap <= 0.0 && p->nf <= 3.0) {
        const double b0 = (11.0 * nc - 2.0 * p->nf) / (12.0 * OR_PI);
        const double c = 0.2;
        const double left = 2.0 / c * log(2.5);
        const double right_Y = (log(4.0 * p->c2 / (p->lambda_qcd * p->lambda_qcd)) - 2.0 * log_Y) / c;
        /* right_X - right_Y = -(1/c) log(X^2/Y^2) */
        const double delta = -log1p(XmY / Ysq) / c;
        /* Lambda = c * lae; alpha = 1/(b0 Lambda):
           alpha_Y - alpha_X = alpha_X alpha_Y b0 c (lae_X - lae_Y) */
        dalpha = alpha_X * alpha_Y * b0 * c * lae_difference(left, right_Y, delta);
    } else if (!p->fixed_coupling) {
        dalpha = alpha_Y - alpha_X;
    }
    const double pref = nc / (2.0 * OR_PI * OR_PI);
    const double rxy2 = r * r / (Xsq * Ysq);
    double lo_kernel, alpha_scale;
    switch (p->rc_lo) {
    case 1: /* PARENT_LO */
        alpha_scale = alpha_r;
        lo_kernel = pref * alpha_r * rxy2;
        break;
    case 2: /* SMALLEST_LO */
        alpha_scale = alpha_min;
        lo_kernel = pref * alpha_min * rxy2;
        break;
    case 3: { /* FAC_LO: 1/(2pi) / (1/abar_r + (X^2-Y^2)/r^2 (abar_X - abar_Y)/(abar_X abar_Y)) r^2/(X^2Y^2)
                 with (abar_X - abar_Y)/(abar_X abar_Y) = -(pi/Nc) (alpha_Y - alpha_X)/(alpha_X alpha_Y) */
        alpha_scale = alpha_r;
        const double den = 1.0 / alpha_r - XmY / (r * r) * dalpha / (alpha_X * alpha_Y);
        lo_kernel = pref * rxy2 / den;
        break;
    }
    case 4: { /* BEUF_LO: r_eff^2 = r^2 (Y^2/X^2)^((X^2-Y^2)/r^2) */
        const double log_reff = log_r - 0.5 * XmY / (r * r) * log1p(XmY / Ysq);
        alpha_scale = alpha_from_log_distance(log_reff, p);
        lo_kernel = pref * alpha_scale * rxy2;
        break;
    }
    default: { /* BALITSKY_LO (and FIXED_LO):
                  r^2/(X^2Y^2) + (aY/aX - 1)/Y^2 + (aX/aY - 1)/X^2
                  = [r^2 + dA (aY (X^2-Y^2) + Y^2 dA)/(aX aY)] / (X^2 Y^2) */
        alpha_scale = alpha_r;
        const double bracket =
            (r * r + dalpha * (alpha_Y * XmY + Ysq * dalpha) / (alpha_X * alpha_Y)) / (Xsq * Ysq);
        lo_kernel = pref * alpha_r * bracket;
    }
    }
    if (!isfinite(lo_kernel)) lo_kernel = 0.0;
    const int resum = p->order != 2 && p->order != 5;
    const int slog_on = p->order == 0 || p->order == 3;
    if (!resum) return lo_kernel;

    const double alpha_res = p->resum_rc == 1 ? alpha_r : (p->resum_rc == 2 ? p->fixed_alpha_s : alpha_min);
    const double min_xy = fmin(X, Y);
    const double xarg = 4.0 * (log_X - log_r) * (log_Y - log_r);
    const double as_x = sqrt(alpha_res * nc / OR_PI * fabs(xarg));
    double dlog;
    if (as_x == 0.0) {
        dlog = 1.0;
    } else {
        dlog = (xarg >= 0.0 ? j1(2.0 * as_x) : or_bessel_i1(2.0 * as_x)) / as_x;
    }
    if (!(r > 1.01 * p->minr)) dlog = 1.0;
    if (!isfinite(dlog)) return 0.0;

    const double alphabar = alpha_res * nc / OR_PI;
    const double A1 = 11.0 / 12.0;
    const double ratio = r / min_xy;
    double slog = 1.0, slog_exp = 0.0;
    if (slog_on) {
        slog = exp(-alphabar * A1 * fabs(log(p->ksub * ratio * ratio)));
        slog_exp = -alphabar * A1 * fabs(2.0 * log(sqrt(p->ksub) * r / min_xy));
    }
    const double lo_single = alpha_scale * pref * rxy2;
    const double subtract = lo_single * slog_exp;
    const double k1fin = lo_kernel * alpha_scale * nc / (4.0 * OR_PI) *
                         (67.0 / 9.0 - OR_PI * OR_PI / 3.0 - 10.0 / 9.0 * p->nf / nc);
    const double result = dlog * slog * lo_kernel - subtract + k1fin;
    return isfinite(result) ? result : 0.0;
}

static double k1_integrand_at(double r, int knot, double z, double theta, const or_spline* nspl,
                              const or_physics* p)
{
    const double sh = sin(0.5 * theta);
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * sh * sh;
    if (Xsq < 1e-40 || z < 1e-20 || r < 1e-20) return 0.0;
    const double value = kernel_lo_value(r, z, theta, p) * k1_dipole(nspl, knot, sqrt(Xsq), z);
    return isfinite(value) ? value : 0.0;
}

/* Amplitude history for the kinematical constraint: rows hN[rows][n] at rapidities hy[rows]
 * on the grid rg[n] (the last row the current amplitude). */
typedef struct or_history {
    const double* rg;
    const double* hy;
    const double* hN;
    int n, rows;
} or_history;

/* _interpolate_history_N (bk/derivatives.py:712-758) at one distance d and rapidity yv,
 * for yind < rows - 1: natural spline through the 6 grid points from max(rind-3, 0)
 * of rows yind and yind+1 (1 when that window runs past the grid), linear in y. */
static double history_amplitude(const or_history* H, double d, double yv, int yind)
{
    int lo = 0, hi = H->n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (d >= H->rg[mid]) lo = mid + 1; else hi = mid;
    }
    const int rind = lo - 1;
    const int start = rind - 3 < 0 ? 0 : rind - 3;
    if (start + 6 > H->n) return 1.0;
    const double* x = H->rg + start;
    double ev = d;
    if (ev < x[0]) ev = x[0] * 1.00001;
    if (ev > x[5]) ev = x[5] * 0.999999;
    int j = 0;
    while (j < 4 && ev >= x[j + 1]) ++j;
    double v[2];
    for (int k = 0; k < 2; ++k) {
        double a[5], b[5], c[5], dd[5];
        or_natural_spline(x, H->hN + (size_t)(yind + k) * H->n + start, 6, a, b, c, dd);
        const double dx = ev - x[j];
        v[k] = a[j] + dx * (b[j] + dx * (c[j] + dx * dd[j]));
    }
    const double frac = (yv - H->hy[yind]) / (H->hy[yind + 1] - H->hy[yind]);
    const double out = v[0] + frac * (v[1] - v[0]);
    return out < 0.0 ? 0.0 : (out > 1.0 ? 1.0 : out);
}

/* _lo_integrand with KINEMATICAL_CONSTRAINT (bk/derivatives.py:469-487): where
 * min(X, Y) > r the daughters are taken at y - log(min(X^2, Y^2)/r^2) from the history
 * (no contribution when that is negative); the dipole (1 - N_r) - (1 - N_X')(1 - N_Y')
 * is formed as N_X' + N_Y' - N_r - N_X' N_Y'. */
static double k1_integrand_history(double r, int knot, double z, double theta, const or_spline* nspl,
                                   const or_physics* p, const or_history* H)
{
    const double sh = sin(0.5 * theta);
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * sh * sh;
    if (Xsq < 1e-40 || z < 1e-20 || r < 1e-20) return 0.0;
    const double X = sqrt(Xsq);
    const double rapidity = H->hy[H->rows - 1];
    const double dmin = fmin(0.5 * log(Xsq), log(z)) - log(r);
    double dipole;
    if (dmin > 0.0) {
        const double shifted = rapidity - 2.0 * dmin;
        if (shifted < 0.0) return 0.0;
        int lo = 0, hi = H->rows;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (H->hy[mid] <= shifted) lo = mid + 1; else hi = mid;
        }
        const int yind = lo - 1 < 0 ? 0 : lo - 1;
        if (yind >= H->rows - 1) {
            dipole = k1_dipole(nspl, knot, X, z);
        } else {
            const double NX = history_amplitude(H, X, shifted, yind);
            const double NY = history_amplitude(H, z, shifted, yind);
            const double Nr = or_n_from_nspline(nspl, r);
            dipole = NX + NY - Nr - NX * NY;
        }
    } else {
        dipole = k1_dipole(nspl, knot, X, z);
    }
    const double value = kernel_lo_value(r, z, theta, p) * dipole;
    return isfinite(value) ? value : 0.0;
}

double or_k1_integrand_history(double r, double z, double theta, const or_spline* nspl, const or_physics* p,
                               const double* rg, int n, const double* hy, const double* hN, int rows)
{
    const or_history H = {rg, hy, hN, n, rows};
    return k1_integrand_history(r, knot_index(nspl, r), z, theta, nspl, p, &H);
}

/* The fixed K1 rule (k1/kernel.cu:2040-2092 nodes) with the kinematical constraint,
 * for many parents. */
void or_k1_fixed_history_many(const double* rpar, int nr, const or_spline* nspl, const or_physics* p,
                              const double* x8, const double* w8, const double* x24, const double* w24,
                              const double* rg, int n, const double* hy, const double* hN, int rows, double* out)
{
    const or_history H = {rg, hy, hN, n, rows};
#pragma omp parallel for schedule(dynamic, 1)
    for (int q = 0; q < nr; ++q) {
        const double r = rpar[q];
        const int knot = knot_index(nspl, r);
        double total = 0.0;
        for (int i = 0; i < nspl->n - 1; ++i) {
            const double lower = nspl->x[i], upper = nspl->x[i + 1];
            const double center = 0.5 * (lower + upper), hw = 0.5 * (upper - lower);
            for (int k = 0; k < 8; ++k) {
                const double lz = center + hw * x8[k];
                const double z = exp(lz);
                const double rw = hw * w8[k];
                for (int j = 0; j < 24; ++j) {
                    const double v = 0.5 * (x24[j] + 1.0);
                    const double theta = OR_PI * v * v;
                    const double aw = w24[j] * OR_PI * v;
                    total += k1_integrand_history(r, knot, z, theta, nspl, p, &H) * (2.0 * z * z) * rw * aw;
                }
            }
        }
        out[q] = total;
    }
}

double or_k1_integrand(double r, double z, double theta, const or_spline* nspl, const or_physics* p)
{
    return k1_integrand_at(r, knot_index(nspl, r), z, theta, nspl, p);
}

/* Modified Bessel I1 (the reference calls torch.special.modified_bessel_i1).
 * Power series sum_k (x/2)^{2k+1}/(k!(k+1)!) below 30 (all terms positive),
 * Hankel asymptotic expansion e^x/sqrt(2 pi x) (1 - 3/(8x) - 15/(128x^2) - ...) above. */
double or_bessel_i1(double x)
{
    const double ax = fabs(x);
    double v;
    if (ax < 30.0) {
        const double h = 0.5 * ax;
        double term = h, sum = h;
        for (int k = 1; k < 200; ++k) {
            term *= h * h / ((double)k * (double)(k + 1));
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        v = sum;
    } else {
        /* mu = 4; terms (-1)^k prod_{j=1..k} (mu - (2j-1)^2) / (k! (8x)^k) */
        const double mu = 4.0;
        double term = 1.0, sum = 1.0;
        for (int k = 1; k < 40; ++k) {
            const double f = (mu - (2.0 * k - 1.0) * (2.0 * k - 1.0));
            term *= -f / ((double)k * 8.0 * ax);
            sum += term;
            if (fabs(term) < 1e-18 * fabs(sum)) break;
        }
        v = exp(ax) / sqrt(2.0 * OR_PI * ax) * sum;
    }
    return x < 0.0 ? -v : v;
}

/* Fixed K1 rule for one parent: k1/kernel.cu:2040-2092 restated.
 * gl8/gl24: Gauss-Legendre nodes/weights on [-1,1] (ascending). */
double or_k1_fixed(double r, const or_spline* nspl, const or_physics* p,
                   const double* x8, const double* w8, const double* x24, const double* w24)
{
    const int knot = knot_index(nspl, r);
    double total = 0.0;
    for (int i = 0; i < nspl->n - 1; ++i) {
        const double lower = nspl->x[i], upper = nspl->x[i + 1];
        const double center = 0.5 * (lower + upper), hw = 0.5 * (upper - lower);
        for (int k = 0; k < 8; ++k) {
            const double lz = center + hw * x8[k];
            const double z = exp(lz);
            const double rw = hw * w8[k];
            for (int j = 0; j < 24; ++j) {
                const double v = 0.5 * (x24[j] + 1.0);
                const double theta = OR_PI * v * v;
                const double aw = w24[j] * OR_PI * v;
                total += k1_integrand_at(r, knot, z, theta, nspl, p) * (2.0 * z * z) * rw * aw;
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* K2/Kf kernels (k2.py, kf.py) in the stable form.  out: k2, k2_swap, kf. */
static void nlo_kernels_stable(double r, double z, double z2, double c1, double c2, double c12,
                               double Xsq, double X2sq, double zzsq, double nf_over_nc,
                               double* k2, double* k2s, double* kf)
{
    const double a = Xsq * z2 * z2;
    const double b = X2sq * z * z;
    const double s = a + b;
    const double dd = r * (r * (z2 * z2 - z * z) - 2.0 * z * z2 * (z2 * c1 - z * c2));
    const double t = dd / s;
    double hm1; /* h(t) - 1 with h = atanh(t)/t */
    double Ld;  /* log(a/b) = 2 atanh(t) */
    if (fabs(t) < 0.1) {
        const double t2 = t * t;
        double series = 0.0;
        for (int k = 12; k >= 1; --k) series = series * t2 + 1.0 / (2.0 * k + 1.0);
        hm1 = t2 * series;
        Ld = 2.0 * t * (1.0 + hm1);
    } else {
        /* |t| >= 0.1: log(a/b) directly (1 - |t| = 2 min(a,b)/s may be tiny) */
        Ld = log(a / b);
        hm1 = Ld / (2.0 * t) - 1.0;
    }
    const double L = 2.0 * (1.0 + hm1) / s;
    const double f = 2.0 * hm1;
    const double q = 1.0 / zzsq;
    const double r2 = r * r;
    const double C0 = f * q * q - 4.0 * r2 * L * q;
    /* L r^4/a + log(a/b) r^2 q/a = L r^2 q (r^2 zz^2 + a - b)/a, and
       r^2 zz^2 + a - b = 2 r z' [r z' - r z cos(th-th') - z z' cos th + z^2 cos th'],
       which removes the cancellation as z' -> 0 (and symmetrically for the swap). */
    const double B1 = r * z2 - r * z * c12 - z * z2 * c1 + z * z * c2;
    const double B2 = r * z - r * z2 * c12 - z * z2 * c2 + z2 * z2 * c1;
    *k2 = C0 + L * r2 * q * 2.0 * r * B1 / (Xsq * z2);
    *k2s = C0 + L * r2 * q * 2.0 * r * B2 / (X2sq * z);
    *kf = (r2 * L * q - f * q * q) * nf_over_nc;
}

void or_nlo_kernels(double r, double lz, double lz2, double th, double th2, double nf, double nc, double* out)
{
    const double z = exp(lz), z2 = exp(lz2);
    const double s1 = sin(0.5 * th), s2 = sin(0.5 * th2), s12 = sin(0.5 * (th - th2));
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * s1 * s1;
    const double X2sq = (r - z2) * (r - z2) + 4.0 * r * z2 * s2 * s2;
    const double zzsq = (z - z2) * (z - z2) + 4.0 * z * z2 * s12 * s12;
    nlo_kernels_stable(r, z, z2, cos(th), cos(th2), cos(th - th2), Xsq, X2sq, zzsq, nf / nc, &out[0], &out[1],
                       &out[2]);
}

/* Per-sample r-independent data of the K2+Kf integrand. */
typedef struct k2_point {
    double z, z2, c1, c2, c12, s1, s2, zzsq, log_min_pt;
    nsv Y, Y2, zz;
    double dN;  /* N_Y2 - N_Y */
    double jac; /* exp(2 log z + 2 log z') (derivatives.py:335) */
    int invalid;
} k2_point;

static void k2_prepare(double lz, double lz2, double th, double th2, const or_spline* sspl, k2_point* pt)
{
    pt->z = exp(lz);
    pt->z2 = exp(lz2);
    const double s1 = sin(0.5 * th), s2 = sin(0.5 * th2), s12 = sin(0.5 * (th - th2));
    pt->s1 = s1 * s1;
    pt->s2 = s2 * s2;
    pt->c1 = cos(th);
    pt->c2 = cos(th2);
    pt->c12 = cos(th - th2);
    pt->zzsq = (pt->z - pt->z2) * (pt->z - pt->z2) + 4.0 * pt->z * pt->z2 * s12 * s12;
    pt->invalid = pt->zzsq < 1e-40 || pt->z < 1e-20 || pt->z2 < 1e-20;
    const double zz = sqrt(pt->zzsq);
    pt->log_min_pt = fmin(fmin(lz, lz2), 0.5 * log(pt->zzsq));
    pt->Y = eval_s(sspl, pt->z);
    pt->Y2 = eval_s(sspl, pt->z2);
    pt->zz = eval_s(sspl, zz);
    pt->dN = ndiff_s(&pt->Y2, &pt->Y);
    pt->jac = exp(2.0 * lz + 2.0 * lz2);
}

/* _nlo_integrand x Jacobian for one (sample, parent); returns K2 and Kf parts. */
static void k2_eval(double r, double log_r, const k2_point* pt, const or_spline* sspl, const or_physics* p,
                    double* k2out, double* kfout)
{
    *k2out = 0.0;
    *kfout = 0.0;
    if (pt->invalid) return;
    const double z = pt->z, z2 = pt->z2;
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * pt->s1;
    const double X2sq = (r - z2) * (r - z2) + 4.0 * r * z2 * pt->s2;
    if (Xsq < 1e-40 || X2sq < 1e-40 || r < 1e-20) return;
    const nsv vX = eval_s(sspl, sqrt(Xsq)), vX2 = eval_s(sspl, sqrt(X2sq));
    double k2, k2s, kf;
    nlo_kernels_stable(r, z, z2, pt->c1, pt->c2, pt->c12, Xsq, X2sq, pt->zzsq, p->nf / p->nc, &k2, &k2s, &kf);
    if (!isfinite(k2)) k2 = 0.0;
    if (!isfinite(k2s)) k2s = 0.0;
    if (!isfinite(kf)) kf = 0.0;
    /* dipole = -(S_X S_zz S_Y2 - S_X S_Y) = S_X (S_Y N_zz + S_zz (N_Y2 - N_Y)) */
    double dip = vX.S * (pt->Y.S * pt->zz.N + pt->zz.S * pt->dN);
    double dips = vX2.S * (pt->Y2.S * pt->zz.N - pt->zz.S * pt->dN);
    if (fabs(k2) > 1e10 && fabs(dip) < 1e-10) { k2 = 0.0; dip = 0.0; }
    if (fabs(k2s) > 1e10 && fabs(dips) < 1e-10) { k2s = 0.0; dips = 0.0; }
    double k2res = p->symmetrize ? 0.5 * (k2 * dip + k2s * dips) : k2 * dip;
    double kfres = 0.0;
    if (p->nf > 0.0) {
        /* dipole_f = S_Y (S_X2 - S_X); symmetric sum = (N_X - N_X2)(N_Y2 - N_Y) */
        const double dNX = ndiff_s(&vX, &vX2);
        const double fermion = p->symmetrize ? 0.5 * kf * dNX * pt->dN : kf * pt->Y.S * dNX;
        kfres = -fermion;
    }
    const double log_min = fmin(fmin(log_r, pt->log_min_pt), 0.5 * fmin(log(Xsq), log(X2sq)));
    /* _nlo_alpha_s (bk/derivatives.py:615-632): smallest size, or the parent (PARENT_NLO) */
    const double alpha = alpha_from_log_distance(p->rc_nlo == 1 ? log_r : log_min, p);
    const double scale = (alpha * p->nc) * (alpha * p->nc) / (8.0 * OR_PI * OR_PI * OR_PI * OR_PI) * pt->jac;
    k2res *= scale;
    kfres *= scale;
    *k2out = isfinite(k2res) ? k2res : 0.0;
    *kfout = isfinite(kfres) ? kfres : 0.0;
}

/* Single-sample integrand (tests). x = (log z, log z', theta_z, theta_z'). */
void or_k2kf_integrand(double r, const double* x, const or_spline* sspl, const or_physics* p, double* out)
{
    k2_point pt;
    k2_prepare(x[0], x[1], x[2], x[3], sspl, &pt);
    k2_eval(r, log(r), &pt, sspl, p, &out[0], &out[1]);
}

/* _nlo_integrand x Jacobian at n box points xs[n][4] = (log z, log z', theta_z, theta_z')
 * for one parent (the Vegas samples): out_k2[i], out_kf[i]. */
void or_k2kf_values(double r, const double* xs, long n, const or_spline* sspl, const or_physics* p, double* out_k2,
                    double* out_kf)
{
    const double lr = log(r);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        k2_point pt;
        k2_prepare(xs[4 * i], xs[4 * i + 1], xs[4 * i + 2], xs[4 * i + 3], sspl, &pt);
        k2_eval(r, lr, &pt, sspl, p, &out_k2[i], &out_kf[i]);
    }
}

/*
 * Sums over n box samples for each of nr parents.  pts: [n][4] unit-cube
 * coordinates u (values already rounded to the generator's precision).
 * The map x = lower + width * u is applied in float32 (map_f32=1, the mixed
 * device build) or float64 (map_f32=0), each operation rounded separately.
 * out: [nr][3] = sum K2 w, sum Kf w, sum (K2+Kf)^2 w^2, with w = volume.
 */
void or_k2kf_sums(const double* rpar, int nr, const double* pts, long n, const double* lower,
                  const double* width, int map_f32, const or_spline* sspl, const or_physics* p,
                  double* out)
{
    double volume = width[0] * width[1] * width[2] * width[3];
    if (map_f32) {
        const float v01 = (float)width[0] * (float)width[1];
        const float v23 = (float)width[2] * (float)width[3];
        volume = (double)(v01 * v23);
    }
    k2_point* prep = (k2_point*)malloc(sizeof(k2_point) * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        double x[4];
        for (int dmn = 0; dmn < 4; ++dmn) {
            if (map_f32) {
                volatile float prod = (float)width[dmn] * (float)pts[i * 4 + dmn];
                volatile float sum = (float)lower[dmn] + prod;
                x[dmn] = (double)sum;
            } else {
                volatile double prod = width[dmn] * pts[i * 4 + dmn];
                x[dmn] = lower[dmn] + prod;
            }
        }
        k2_prepare(x[0], x[1], x[2], x[3], sspl, &prep[i]);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < nr; ++j) {
        const double r = rpar[j];
        const double lr = log(r);
        double s_k2 = 0.0, s_kf = 0.0, s_sq = 0.0;
        for (long i = 0; i < n; ++i) {
            double k2, kf;
            k2_eval(r, lr, &prep[i], sspl, p, &k2, &kf);
            k2 *= volume;
            kf *= volume;
            s_k2 += k2;
            s_kf += kf;
            s_sq += (k2 + kf) * (k2 + kf);
        }
        out[j * 3 + 0] = s_k2;
        out[j * 3 + 1] = s_kf;
        out[j * 3 + 2] = s_sq;
    }
    free(prep);
}

/* K1 fixed rule for many parents (parallel over parents). */
void or_k1_fixed_many(const double* rpar, int nr, const or_spline* nspl, const or_physics* p,
                      const double* x8, const double* w8, const double* x24, const double* w24, double* out)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < nr; ++j) out[j] = or_k1_fixed(rpar[j], nspl, p, x8, w8, x24, w24);
}

/* ------------------------------------------------------------------------ */
/* Sobol points: torch.quasirandom.SobolEngine draws (dims <= 8).
 * state: [dims][30] scrambled direction numbers, shift: [dims].
 * Point i = shift ^ (xor of state[:, j] over the set bits j of gray(i)), times 2^-30.
 * float32 output rounds the integer to float32 first (torch's copy into a
 * float32 result, then multiply by 2^-30).  In float64 the reference's first
 * point is computed in float32 and cast (torch/quasirandom.py _first_point). */
void or_sobol(const int64_t* state, const int64_t* shift, int dims, long offset, long n, int as_f32,
              double* out)
{
    const double scale = 1.0 / 1073741824.0;
    for (long k = 0; k < n; ++k) {
        const uint64_t i = (uint64_t)(offset + k);
        const uint64_t g = i ^ (i >> 1);
        for (int d = 0; d < dims; ++d) {
            int64_t v = shift[d];
            for (int j = 0; j < 30; ++j)
                if ((g >> j) & 1u) v ^= state[d * 30 + j];
            double u;
            if (as_f32 || i == 0) {
                const float fv = (float)v;
                u = (double)(fv * (float)scale);
            } else {
                u = (double)v * scale;
            }
            out[k * dims + d] = u;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Quad-precision evaluation of the reference's literal formulas (pinning only). */
typedef __float128 qd;

static qd q_alpha(qd r, const or_physics* p)
{
    if (p->fixed_coupling) return (qd)p->fixed_alpha_s;
    const qd b0 = ((qd)11 * p->nc - (qd)2 * p->nf) / ((qd)12 * M_PIq);
    const qd c = (qd)0.2Q;
    const qd left = (qd)2 / c * logq((qd)2.5Q);
    const qd scale = (qd)4 * p->c2 / (r * r * (qd)p->lambda_qcd * (qd)p->lambda_qcd);
    const qd right = logq(scale) / c;
    const qd m = left > right ? left : right;
    const qd lae = m + log1pq(expq(-fabsq(left - right)));
    qd a = (qd)1 / (b0 * c * lae);
    if (p->alpha_cap > 0.0 && a > (qd)p->alpha_cap) a = (qd)p->alpha_cap;
    return a;
}

/* Kernel_nlo / Kernel_nlo_fermion (k2.py:8-39, kf.py:10-41) with the distances of
 * derivatives.py:521-529 (law of cosines), all in quad precision. out: k2, k2s, kf. */
void or_nlo_kernels_literal_q(double r_, double lz, double lz2, double th, double th2, double nf, double nc,
                              double* out)
{
    const qd r = r_;
    const qd z = expq((qd)lz), z2 = expq((qd)lz2);
    const qd X = sqrtq(r * r + z * z - 2 * r * z * cosq((qd)th));
    const qd X2 = sqrtq(r * r + z2 * z2 - 2 * r * z2 * cosq((qd)th2));
    const qd zz = sqrtq(z * z + z2 * z2 - 2 * z * z2 * cosq((qd)th - (qd)th2));
    const qd Y = z, Y2 = z2;
    qd res[2];
    for (int sw = 0; sw < 2; ++sw) {
        const qd x1 = sw ? X2 : X, y1 = sw ? Y2 : Y, x2 = sw ? X : X2, y2 = sw ? Y : Y2;
        const qd XY2sq = (x1 * y2) * (x1 * y2), X2Ysq = (x2 * y1) * (x2 * y1);
        const qd diff = XY2sq - X2Ysq;
        const qd zz4 = zz * zz * zz * zz;
        qd k = -(qd)2 / zz4;
        k += ((XY2sq + X2Ysq - 4 * (r * zz) * (r * zz)) / (zz4 * diff) + r * r * r * r / (XY2sq * diff) +
              r * r / ((x1 * y2 * zz) * (x1 * y2 * zz))) *
             2 * logq(x1 * y2 / (x2 * y1));
        res[sw] = k;
    }
    const qd XY2sq = (X * Y2) * (X * Y2), X2Ysq = (X2 * Y) * (X2 * Y);
    const qd zz4 = zz * zz * zz * zz;
    qd kf = (qd)2 / zz4 - (XY2sq + X2Ysq - (r * zz) * (r * zz)) / (zz4 * (XY2sq - X2Ysq)) * 2 * logq(X * Y2 / (X2 * Y));
    kf = kf * (qd)nf / (qd)nc;
    out[0] = (double)res[0];
    out[1] = (double)res[1];
    out[2] = (double)kf;
}

/* Kernel_lo literal (k1.py:20-155, production order) in quad precision;
 * the Bessel factor uses the FP64 functions (it is well conditioned). */
double or_lo_kernel_literal_q(double r_, double z_, double theta, const or_physics* p)
{
    const qd r = r_, z = z_;
    const qd Xsq = r * r + z * z - 2 * r * z * cosq((qd)theta);
    if (Xsq <= 0) return 0.0;
    const qd X = sqrtq(Xsq), Y = z;
    const qd nc = p->nc;
    const qd ar = q_alpha(r, p), aX = q_alpha(X, p), aY = q_alpha(Y, p);
    const qd lo = nc / (2 * M_PIq * M_PIq) * ar *
                  (r * r / (X * X * Y * Y) + (aY / aX - 1) / (Y * Y) + (aX / aY - 1) / (X * X));
    const qd mn = fminq(fminq(X, Y), r);
    const qd amin = q_alpha(mn, p);
    const double xarg = (double)(4 * logq(X / r) * logq(Y / r));
    const double as_x = sqrt((double)amin * p->nc / OR_PI * fabs(xarg));
    double dlog = as_x == 0.0 ? 1.0 : (xarg >= 0 ? j1(2 * as_x) : or_bessel_i1(2 * as_x)) / as_x;
    if (!(r_ > 1.01 * p->minr)) dlog = 1.0;
    const qd alphabar = amin * nc / M_PIq;
    const qd minxy = fminq(X, Y);
    const qd slog = expq(-alphabar * (qd)11 / 12 * fabsq(logq((qd)p->ksub * (r / minxy) * (r / minxy))));
    const qd slog_exp = -alphabar * (qd)11 / 12 * fabsq(2 * logq(sqrtq((qd)p->ksub) * r / minxy));
    const qd lo_single = ar * nc / (2 * M_PIq * M_PIq) * (r / (X * Y)) * (r / (X * Y));
    const qd k1fin = lo * ar * nc / (4 * M_PIq) * ((qd)67 / 9 - M_PIq * M_PIq / 3 - (qd)10 / 9 * (qd)p->nf / nc);
    const qd res = (qd)dlog * slog * lo - lo_single * slog_exp + k1fin;
    return (double)res;
}

/* Stable lo-kernel alone (same as or_k1_integrand without the dipole), for tests. */
double or_lo_kernel(double r, double z, double theta, const or_physics* p)
{
    return kernel_lo_value(r, z, theta, p);
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Quad-precision literal dipoles from the same spline coefficients (pinning only). */
static qd q_poly(const or_spline* s, qd lx)
{
    if (lx < (qd)s->x[0]) lx = (qd)s->x[0];
    if (lx > (qd)s->x[s->n - 1]) lx = (qd)s->x[s->n - 1];
    int lo = 0, hi = s->n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (lx >= (qd)s->x[mid]) lo = mid + 1; else hi = mid;
    }
    int i = lo - 1;
    if (i < 0) i = 0;
    if (i > s->n - 2) i = s->n - 2;
    const qd dx = lx - (qd)s->x[i];
    return (qd)s->a[i] + dx * ((qd)s->b[i] + dx * ((qd)s->c[i] + dx * (qd)s->d[i]));
}

static qd q_n_nspline(const or_spline* s, qd r)
{
    if (r < (qd)s->rmin) return 0;
    if (r > (qd)s->rmax) return 1;
    qd v = expq(q_poly(s, logq(r)));
    return v < 1 ? v : (qd)1;
}

static qd q_s_sspline(const or_spline* s, qd r)
{
    if (r < (qd)s->rmin) return 1;
    if (r > (qd)s->rmax) return 0;
    return expq(q_poly(s, logq(r)));
}

/* N_X + N_Y - N_r - N_X N_Y for the K1 integrand; X from the law of cosines. */
double or_k1_dipole_literal_q(const or_spline* s, double r_, double z_, double theta)
{
    const qd r = r_, z = z_;
    const qd X = sqrtq(r * r + z * z - 2 * r * z * cosq((qd)theta));
    const qd NX = q_n_nspline(s, X), NY = q_n_nspline(s, z), Nr = q_n_nspline(s, r);
    return (double)(NX + NY - Nr - NX * NY);
}

double or_k1_dipole(const or_spline* s, double r, double z, double theta)
{
    const double sh = sin(0.5 * theta);
    const double Xsq = (r - z) * (r - z) + 4.0 * r * z * sh * sh;
    return k1_dipole(s, knot_index(s, r), sqrt(Xsq), z);
}

/* K2 dipoles S_X (S_Y - S_zz S_Y2), S_X2 (S_Y2 - S_zz S_Y) and the fermion
 * factor (S_X2 - S_X)(S_Y - S_Y2): quad literal (out_q) and stable FP64 (out). */
void or_k2_dipoles(const or_spline* s, double r, const double* x, double* out, double* out_q)
{
    k2_point pt;
    k2_prepare(x[0], x[1], x[2], x[3], s, &pt);
    const double Xsq = (r - pt.z) * (r - pt.z) + 4.0 * r * pt.z * pt.s1;
    const double X2sq = (r - pt.z2) * (r - pt.z2) + 4.0 * r * pt.z2 * pt.s2;
    const nsv vX = eval_s(s, sqrt(Xsq)), vX2 = eval_s(s, sqrt(X2sq));
    out[0] = vX.S * (pt.Y.S * pt.zz.N + pt.zz.S * pt.dN);
    out[1] = vX2.S * (pt.Y2.S * pt.zz.N - pt.zz.S * pt.dN);
    out[2] = ndiff_s(&vX, &vX2) * pt.dN;
    const qd rq = r, z = expq((qd)x[0]), z2 = expq((qd)x[1]);
    const qd X = sqrtq(rq * rq + z * z - 2 * rq * z * cosq((qd)x[2]));
    const qd X2 = sqrtq(rq * rq + z2 * z2 - 2 * rq * z2 * cosq((qd)x[3]));
    const qd zz = sqrtq(z * z + z2 * z2 - 2 * z * z2 * cosq((qd)x[2] - (qd)x[3]));
    const qd SX = q_s_sspline(s, X), SX2 = q_s_sspline(s, X2), SY = q_s_sspline(s, z),
             SY2 = q_s_sspline(s, z2), Szz = q_s_sspline(s, zz);
    out_q[0] = (double)(-(SX * Szz * SY2 - SX * SY));
    out_q[1] = (double)(-(SX2 * Szz * SY - SX2 * SY2));
    out_q[2] = (double)((SX2 - SX) * (SY - SY2));
}
