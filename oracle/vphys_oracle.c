/* vphys_oracle.c -- CPU FP64 restatement of Roundabout's vertical-physics hot
 * path.  TEST INFRASTRUCTURE ONLY (see vphys_oracle.h).  Each routine cites
 * the reference lines it restates; loop variables are 1-based like the
 * Fortran so the index arithmetic can be read against it line by line.
 *
 * Build: gcc -O3 -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared
 * (oracle/Makefile).
 */
#include "vphys_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- constants (src/core/rdb_constants.F90:37, 44, 67, 85, 94) ---- */
static const double GRAVITY = 9.80665;
static const double H_VANISHED = 1.5e-4;
static const double H_DIV_EPS = 1.0e-20;
static const double PI_ = 3.141592653589793115997963468544185161590576171875; /* 4*atan(1) */

/* Fortran MAX/MIN on finite operands. */
static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return a < b ? a : b; }

/* 1-based Fortran-order accessors. */
#define C3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)nx * (((size_t)(j) - 1) + (size_t)ny * ((size_t)(k) - 1))]
#define C2(a, i, j) (a)[((size_t)(i) - 1) + (size_t)nx * ((size_t)(j) - 1)]
#define U3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)(nx + 1) * (((size_t)(j) - 1) + (size_t)ny * ((size_t)(k) - 1))]
#define V3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)nx * (((size_t)(j) - 1) + (size_t)(ny + 1) * ((size_t)(k) - 1))]

void vpo_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int vpo_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* =====================================================================
 * Position-independent math: restatement of rdb_sm_cbrt
 * (src/shared_module_utilities/rdb_safe_math_pow.inc:107-142) and
 * rdb_sm_atan (rdb_safe_math_atan.inc:7-44) with the coefficient tables of
 * rdb_safe_math_consts.inc:65-100.  Only IEEE + - * / and exact exponent
 * manipulation, so the value is the same on every IEEE machine built without
 * FMA contraction.
 * ===================================================================== */
static const double SM_CBRT_C[5] = {
    0.5189978361037301813, 0.6542973117201534849, -0.2158001895775201462,
    0.04437845996234061896, -0.003660165019409192949};
static const double SM_ATAN_C[12] = {
    1.0, -0.3333333333333333148, 0.1999999999999998446,
    -0.1428571428571007162, 0.1111111111054328693, -0.09090909045700855395,
    0.07692305406260263601, -0.06666590357759735741, 0.05880646170199485545,
    -0.05237747786578652448, 0.04518284953605152671, -0.0295457862073798469};
static const double SM_PIO2_HI = 1.570796326794896558;
static const double SM_PIO2_LO = 6.1232339957367660359e-17;
static const double SM_SQRT3 = 1.7320508075688771932;
static const double SM_PIO6_HI = 0.52359877559829892668;
static const double SM_PIO6_LO = -5.3604088322554549242e-17;
static const double SM_TAN_PIO12 = 0.2679491924311226958;

/* rdb_sm_exp (rdb_safe_math_core.inc:81-137) with its constants
 * (rdb_safe_math_consts.inc:39-52): k = nearest integer to x/ln2 (halves away
 * from zero), r = x - k ln2 with ln2 split so k*LN2_HI is exact, degree-13
 * Taylor polynomial (coefficients 1/i!), scaled by 2**k; results below the
 * smallest normal are exactly 0. */
static const double SM_LN2_HI = 0.69314718060195446014;
static const double SM_LN2_LO = -4.2009150726810845979e-11;
static const double SM_INV_LN2 = 1.442695040888963387;
static const double SM_EXP_MAX = 709.78271289338399679;
static const double SM_EXP_MIN = -745.1332191019412;
static const double SM_EXP_C[14] = {1.0,           1.0,              1.0 / 2.0,         1.0 / 6.0,
                                    1.0 / 24.0,    1.0 / 120.0,      1.0 / 720.0,       1.0 / 5040.0,
                                    1.0 / 40320.0, 1.0 / 362880.0,   1.0 / 3628800.0,   1.0 / 39916800.0,
                                    1.0 / 479001600.0, 1.0 / 6227020800.0};

/* rdb_sm_exp_core (rdb_safe_math_core.inc:81-114): exp(x + c) for finite x
 * in range and a small correction c added to the reduced argument (0 for
 * plain exp; the tail of a double-double exponent for pow). */
static double sm_exp_core(double x, double c)
{
    double kr = round(x * SM_INV_LN2);
    int k = (int)kr;
    double r = x - kr * SM_LN2_HI;
    r = r - kr * SM_LN2_LO;
    r = r + c;
    double p = SM_EXP_C[13];
    for (int i = 12; i >= 0; --i) p = p * r + SM_EXP_C[i];
    double y = (k > 1000) ? 2.0 * ldexp(p, k - 1) : ldexp(p, k);
    if (y < DBL_MIN) y = 0.0;
    return y;
}

double vpo_sm_exp(double x)
{
    if (isnan(x)) return x;
    if (x > SM_EXP_MAX) return INFINITY;
    if (x < SM_EXP_MIN) return 0.0;
    return sm_exp_core(x, 0.0);
}

/* rdb_sm_log (rdb_safe_math_core.inc:139-206): x = m 2^k with m in
 * [sqrt(1/2), sqrt(2)), log m = 2 atanh f, f = (m-1)/(m+1), the odd series
 * in f to 1/19 (Cody & Waite 1980, ch. 5), k ln 2 added as head + tail. */
static const double SM_SPLIT = 134217729.0;   /* 2^27 + 1, the Veltkamp split */
static const double SM_LOG_C[10] = {1.0,        1.0 / 3.0,  1.0 / 5.0,  1.0 / 7.0,  1.0 / 9.0,
                                    1.0 / 11.0, 1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0, 1.0 / 19.0};
static const double SM_SQRT_HALF = 0.70710678118654757274;
static const double SM_TWO54 = 18014398509481984.0;

double vpo_sm_log(double x)
{
    if (isnan(x)) return x;
    if (x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x < DBL_MIN && x * SM_TWO54 == 0.0) return -INFINITY;
    if (!isfinite(x)) return x;
    double xs = x;
    int kadj = 0;
    if (x < DBL_MIN) {
        xs = x * SM_TWO54;
        kadj = -54;
    }
    int e;
    double m = frexp(xs, &e);   /* Fortran fraction / exponent: m in [1/2, 1) */
    int k = e + kadj;
    if (m < SM_SQRT_HALF) {
        m = 2.0 * m;
        k = k - 1;
    }
    const double f = (m - 1.0) / (m + 1.0);
    const double u = f * f;
    double p = SM_LOG_C[9];
    for (int i = 8; i >= 1; --i) p = p * u + SM_LOG_C[i];
    const double kr = (double)k;
    const double s = kr * SM_LN2_HI + 2.0 * f;
    const double w = (2.0 * f) * u * p + kr * SM_LN2_LO;
    return s + w;
}

/* Knuth's exact sum and Dekker's exact product without FMA (Veltkamp split
 * by 2^27 + 1): s + e == a + b, p + e == a * b (rdb_safe_math_core.inc:53-79). */
static void sm_two_sum(double a, double b, double *s, double *e)
{
    *s = a + b;
    const double bb = *s - a;
    *e = (a - (*s - bb)) + (b - bb);
}
static void sm_two_prod(double a, double b, double *p, double *e)
{
    double c = SM_SPLIT * a;
    const double ah = c - (c - a);
    const double al = a - ah;
    c = SM_SPLIT * b;
    const double bh = c - (c - b);
    const double bl = b - bh;
    *p = a * b;
    *e = (((ah * bh - *p) + ah * bl) + al * bh) + al * bl;
}

/* rdb_sm_log_dd (rdb_safe_math_core.inc:208-249): log x as head + tail, the
 * quotient f = (m-1)/(m+1) carried to ~106 bits so y log x keeps its bits. */
static void sm_log_dd(double x, double *lh, double *ll)
{
    if (x < DBL_MIN && x * SM_TWO54 == 0.0) {
        *lh = -INFINITY;
        *ll = 0.0;
        return;
    }
    double xs = x;
    int kadj = 0;
    if (x < DBL_MIN) {
        xs = x * SM_TWO54;
        kadj = -54;
    }
    int e;
    double m = frexp(xs, &e);
    int k = e + kadj;
    if (m < SM_SQRT_HALF) {
        m = 2.0 * m;
        k = k - 1;
    }
    const double a = m - 1.0;
    double bh, bl;
    sm_two_sum(m, 1.0, &bh, &bl);
    const double q1 = a / bh;
    double p1, p2;
    sm_two_prod(q1, bh, &p1, &p2);
    const double rr = ((a - p1) - p2) - q1 * bl;
    const double q2 = rr / bh;
    const double fh = q1 + q2;
    const double fl = q2 - (fh - q1);
    const double u = fh * fh;
    double p = SM_LOG_C[9];
    for (int i = 8; i >= 1; --i) p = p * u + SM_LOG_C[i];
    const double tail = (2.0 * fh) * u * p;
    const double kr = (double)k;
    double ss, ee;
    sm_two_sum(kr * SM_LN2_HI, 2.0 * fh, &ss, &ee);
    *lh = ss;
    *ll = ee + ((2.0 * fl + tail) + kr * SM_LN2_LO);
}

/* rdb_sm_pow (rdb_safe_math_pow.inc:6-105): the C99 pow special values
 * except that a NaN anywhere gives NaN; for finite x > 0 exp(y log x) with
 * the log as head + tail and y*log x formed exactly (Dekker 1971). */
double vpo_sm_pow(double x, double y)
{
    if (isnan(x) || isnan(y)) return NAN;
    if (y == 0.0 || x == 1.0) return 1.0;
    const double ax = fabs(x), ay = fabs(y);
    int yint, yodd;
    if (isfinite(y)) {
        if (ay >= 9007199254740992.0) {
            yint = 1;
            yodd = 0;
        } else {
            yint = (ay == round(ay));
            const double h = 0.5 * ay;
            yodd = yint && (h != round(h));
        }
    } else {
        yint = 0;
        yodd = 0;
    }
    const int xneg = (x < 0.0) || (x == 0.0 && signbit(x));
    double r;
    if (!isfinite(y)) {
        if (ax == 1.0)
            r = 1.0;
        else if ((ax < 1.0) == (y > 0.0))
            r = 0.0;
        else
            r = INFINITY;
        return r;
    }
    if (ax == 0.0) {
        r = (y > 0.0) ? 0.0 : INFINITY;
        if (xneg && yodd) r = -r;
        return r;
    }
    if (!isfinite(x)) {
        r = (y > 0.0) ? INFINITY : 0.0;
        if (xneg && yodd) r = -r;
        return r;
    }
    if (xneg && !yint) return NAN;
    double lh, ll;
    sm_log_dd(ax, &lh, &ll);
    const double t = y * lh;
    if (t > 800.0) {
        r = INFINITY;
    } else if (t < -800.0) {
        r = 0.0;
    } else {
        double ph, pl, ee, c2;
        sm_two_prod(y, lh, &ph, &pl);
        const double c = pl + y * ll;
        sm_two_sum(ph, c, &ee, &c2);
        if (ee > SM_EXP_MAX)
            r = INFINITY;
        else if (ee < SM_EXP_MIN)
            r = 0.0;
        else
            r = sm_exp_core(ee, c2);
    }
    if (xneg && yodd) r = -r;
    return r;
}

/* rdb_sm_erfc (rdb_safe_math_erfc.inc): a series in x^2 below |x| = 1/2;
 * beyond, exp(-x^2) formed as exp(-xh^2 - xl (x + xh)) on a Veltkamp split,
 * times a rational fit on [1/2, 2) and [2, 4) or the asymptotic form
 * (1 + w P(w)/Q(w))/(x sqrt(pi)), w = 1/x^2, beyond 4.  The fitted tables
 * are the reference's (rdb_safe_math_consts.inc:99-128). */
static const double SM_ERF_C[12] = {
    1.128379167095512559,      -0.376126389031837538,    0.1128379167095512614,
    -0.02686617064513124181,   0.005223977625441806293,  -0.0008548327023363942604,
    0.0001205533296923066544,  -0.00001492564916290355896, 1.64620383639705829e-6,
    -1.636264690374603956e-7,  1.472152117638980096e-8,  -1.095865453884735107e-9};
static const double SM_ERFC_A_P[7] = {0.9999999993850857694, 1.248626834329117141, 0.7867094724888269441,
                                      0.2819428661917610102, 0.05719027224971907214, 0.005247572786535052193,
                                      4.820036176802313081e-8};
static const double SM_ERFC_A_Q[7] = {1.0, 2.377005991883625935, 2.468873583018134976, 1.443014856236056964,
                                      0.5046949490889137691, 0.1013327241858480304, 0.009303534974169982985};
static const double SM_ERFC_B_P[7] = {0.9999921569124016196, 1.494269944137282868, 1.086387126830294259,
                                      0.4598879010194165118, 0.1135948493973390344, 0.01390038004034872994,
                                      1.000103316758091609e-9};
static const double SM_ERFC_B_Q[7] = {1.0, 2.622591678871410537, 3.045871297831376889, 2.025960043609839722,
                                      0.8274770365185684096, 0.2013396690397278865, 0.02463786793791475013};
static const double SM_ERFC_C_P[6] = {-0.4999999999999982792, -12.20993252402114315, -95.49719132910308872,
                                      -273.5933562329464053, -231.8021338423288, -12.38208675658035851};
static const double SM_ERFC_C_Q[6] = {1.0, 25.91986504803799107, 226.1241802321382579, 802.2984884770494318,
                                      1100.222105092567517, 428.3053107970796418};
static const double SM_INV_SQRTPI = 0.56418958354775627928;

double vpo_sm_erfc(double x)
{
    if (isnan(x)) return x;
    const double ax = fabs(x);
    if (ax < 0.5) {
        const double v = x * x;
        double p = SM_ERF_C[11];
        for (int i = 10; i >= 0; --i) p = p * v + SM_ERF_C[i];
        return 1.0 - x * p;
    }
    double ex;
    if (ax > 27.3) {
        ex = 0.0;
    } else {
        const double c = SM_SPLIT * ax;
        const double xh = c - (c - ax);
        const double xl = ax - xh;
        ex = sm_exp_core(-(xh * xh), -(xl * (ax + xh)));
    }
    double p, q;
    if (ax < 2.0) {
        p = SM_ERFC_A_P[6];
        q = SM_ERFC_A_Q[6];
        for (int i = 5; i >= 0; --i) {
            p = p * ax + SM_ERFC_A_P[i];
            q = q * ax + SM_ERFC_A_Q[i];
        }
        ex = ex * (p / q);
    } else if (ax < 4.0) {
        p = SM_ERFC_B_P[6];
        q = SM_ERFC_B_Q[6];
        for (int i = 5; i >= 0; --i) {
            p = p * ax + SM_ERFC_B_P[i];
            q = q * ax + SM_ERFC_B_Q[i];
        }
        ex = ex * (p / q);
    } else {
        const double rax = 1.0 / ax;
        const double w = rax * rax;
        p = SM_ERFC_C_P[5];
        q = SM_ERFC_C_Q[5];
        for (int i = 4; i >= 0; --i) {
            p = p * w + SM_ERFC_C_P[i];
            q = q * w + SM_ERFC_C_Q[i];
        }
        ex = ((ex * SM_INV_SQRTPI) * rax) * (1.0 + w * (p / q));
    }
    if (ex < DBL_MIN) ex = 0.0;
    return (x < 0.0) ? 2.0 - ex : ex;
}

static inline double sm_flush(double r)
{
    /* rdb_sm_flush (rdb_safe_math_core.inc:40-51) */
    if (fabs(r) < DBL_MIN) return copysign(0.0, r);
    return r;
}

double vpo_sm_cbrt(double x)
{
    if (isnan(x) || !isfinite(x)) return x;
    double ax = fabs(x);
    if (ax < DBL_MIN) return copysign(0.0, x);
    int e;
    double f = frexp(ax, &e);          /* Fortran fraction()/exponent() */
    int rem = ((e % 3) + 3) % 3;       /* modulo(e, 3) */
    int q = (e - rem) / 3;
    double m = ldexp(f, rem);          /* in [1/2, 4) */
    double y0 = SM_CBRT_C[4];
    for (int i = 3; i >= 0; --i) y0 = y0 * m + SM_CBRT_C[i];
    for (int it = 0; it < 2; ++it) {
        double y3 = (y0 * y0) * y0;
        y0 = y0 + y0 * ((m - y3) / ((y3 + y3) + m));
    }
    double y = ldexp(y0, q);
    if (x < 0.0) y = -y;
    return y;
}

double vpo_sm_atan(double x)
{
    if (isnan(x)) return x;
    double ax = fabs(x);
    int inv = ax > 1.0;
    double t = inv ? 1.0 / ax : ax;
    int mid = t > SM_TAN_PIO12;
    double a = mid ? (SM_SQRT3 * t - 1.0) / (SM_SQRT3 + t) : t;
    double u = a * a;
    double p = SM_ATAN_C[11];
    for (int i = 10; i >= 0; --i) p = p * u + SM_ATAN_C[i];
    double y = a * p;
    if (mid) y = SM_PIO6_HI + (y + SM_PIO6_LO);
    if (inv) y = (SM_PIO2_HI - y) + SM_PIO2_LO;
    return sm_flush(copysign(y, x));
}

/* =====================================================================
 * Wright (1997) EOS at p_ref (src/equation_of_state/rdb_eos.F90:200-217,
 * 909-959).
 * ===================================================================== */
#define WRIGHT_A0 7.057924e-4
#define WRIGHT_A1 3.480336e-7
#define WRIGHT_A2 -1.112733e-7
#define WRIGHT_B0 5.790749e8
#define WRIGHT_B1 3.516535e6
#define WRIGHT_B2 -4.002714e4
#define WRIGHT_B3 2.084372e2
#define WRIGHT_B4 5.944068e5
#define WRIGHT_B5 -9.643486e3
#define WRIGHT_C0 1.704853e5
#define WRIGHT_C1 7.904722e2
#define WRIGHT_C2 -7.984422e0
#define WRIGHT_C3 5.140652e-2
#define WRIGHT_C4 -2.302158e2
#define WRIGHT_C5 -3.079464e0

void vpo_eos_wright(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double *S = s->tr[c->idx_salinity], *T = s->tr[c->idx_temperature];
    const double p_ref = c->eos_p_ref, rho0 = c->rho0;
#pragma omp parallel for
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                if (C3(s->h, i, j, k) > H_VANISHED) {
                    double S_k = C3(S, i, j, k), T_k = C3(T, i, j, k);
                    double T_sq = T_k * T_k;
                    double T_cu = T_sq * T_k;
                    double alpha_0 = WRIGHT_A0 + WRIGHT_A1 * T_k + WRIGHT_A2 * S_k;
                    double p_0 = WRIGHT_B0 + WRIGHT_B1 * T_k + WRIGHT_B2 * T_sq + WRIGHT_B3 * T_cu +
                                 WRIGHT_B4 * S_k + WRIGHT_B5 * S_k * T_k;
                    double lambda = WRIGHT_C0 + WRIGHT_C1 * T_k + WRIGHT_C2 * T_sq + WRIGHT_C3 * T_cu +
                                    WRIGHT_C4 * S_k + WRIGHT_C5 * S_k * T_k;
                    double p_plus_p0 = p_ref + p_0;
                    double denom = lambda + alpha_0 * p_plus_p0;
                    C3(s->rho, i, j, k) = p_plus_p0 / denom;
                } else {
                    C3(s->rho, i, j, k) = rho0;
                }
            }
}

/* eos_buoyancy_coeffs, Wright branch (rdb_eos.F90:1624-1736, the Wright arm
 * 1716-1733): alpha_T = -d(rho)/dT, beta_S = +d(rho)/dS of rho = P/D with
 * P = p + p0(T,S), D = lambda(T,S) + alpha0(T,S) P, by the quotient rule. */
void vpo_eos_buoyancy_coeffs(double T, double S, double p, double *alpha_T, double *beta_S)
{
    double T_sq = T * T;
    double alpha_0 = WRIGHT_A0 + WRIGHT_A1 * T + WRIGHT_A2 * S;
    double p_0 = WRIGHT_B0 + WRIGHT_B1 * T + WRIGHT_B2 * T_sq + WRIGHT_B3 * T_sq * T + WRIGHT_B4 * S + WRIGHT_B5 * S * T;
    double lambda = WRIGHT_C0 + WRIGHT_C1 * T + WRIGHT_C2 * T_sq + WRIGHT_C3 * T_sq * T + WRIGHT_C4 * S +
                    WRIGHT_C5 * S * T;
    double dp0_dt = WRIGHT_B1 + 2.0 * WRIGHT_B2 * T + 3.0 * WRIGHT_B3 * T_sq + WRIGHT_B5 * S;
    double dlam_dt = WRIGHT_C1 + 2.0 * WRIGHT_C2 * T + 3.0 * WRIGHT_C3 * T_sq + WRIGHT_C5 * S;
    double dp0_ds = WRIGHT_B4 + WRIGHT_B5 * T;
    double dlam_ds = WRIGHT_C4 + WRIGHT_C5 * T;
    double big_p = p + p_0;
    double denom = lambda + alpha_0 * big_p;
    double inv_d2 = 1.0 / (denom * denom);
    *alpha_T = -(dp0_dt * denom - big_p * (dlam_dt + WRIGHT_A1 * big_p + alpha_0 * dp0_dt)) * inv_d2;
    *beta_S = (dp0_ds * denom - big_p * (dlam_ds + WRIGHT_A2 * big_p + alpha_0 * dp0_ds)) * inv_d2;
}

/* |tau| at cell centres (rdb_ocean_surface_stress.F90:858-875). */
void vpo_stress_mag(vpo_state *s)
{
    const int nx = s->nx, ny = s->ny;
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double tx = 0.5 * (s->tau_x[(i - 1) + (nx + 1) * (j - 1)] + s->tau_x[i + (nx + 1) * (j - 1)]);
            double ty = 0.5 * (s->tau_y[(i - 1) + nx * (j - 1)] + s->tau_y[(i - 1) + nx * j]);
            C2(s->stress_mag, i, j) = sqrt(tx * tx + ty * ty);
        }
}

/* =====================================================================
 * PP81 (rdb_ocean_vmix.F90:1007-1074)
 * ===================================================================== */
void vpo_pp81(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    double *kv = s->kv, *kt = s->kt;
    const double *u = s->u, *v = s->v, *h = s->h, *rho = s->rho;
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            C3(kv, i, j, 1) = 0.0;
            C3(kt, i, j, 1) = 0.0;
            C3(kv, i, j, nz + 1) = 0.0;
            C3(kt, i, j, nz + 1) = 0.0;
        }
#pragma omp parallel for
    for (int k = 2; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double u_km1 = 0.5 * (U3(u, i, j, k - 1) + U3(u, i + 1, j, k - 1));
                double v_km1 = 0.5 * (V3(v, i, j, k - 1) + V3(v, i, j + 1, k - 1));
                double u_k = 0.5 * (U3(u, i, j, k) + U3(u, i + 1, j, k));
                double v_k = 0.5 * (V3(v, i, j, k) + V3(v, i, j + 1, k));
                double dz_face = 0.5 * (C3(h, i, j, k - 1) + C3(h, i, j, k));
                if (dz_face <= 0.0) {
                    C3(kv, i, j, k) = c->pp81_nu_bg;
                    C3(kt, i, j, k) = c->pp81_kappa_bg;
                    continue;
                }
                double du_dz = (u_k - u_km1) / dz_face;
                double dv_dz = (v_k - v_km1) / dz_face;
                double shear2 = fmx(du_dz * du_dz + dv_dz * dv_dz, c->shear2_floor);
                double n2 = -(GRAVITY * (C3(rho, i, j, k) - C3(rho, i, j, k - 1)) / (c->rho0 * dz_face));
                double ri = n2 / shear2;
                double denom = 1.0 + c->pp81_alpha * fmx(ri, 0.0);
                double ri_factor = 1.0 / (denom * denom);
                C3(kv, i, j, k) = c->pp81_nu_bg + c->pp81_nu0 * ri_factor;
                C3(kt, i, j, k) = c->pp81_kappa_bg + c->pp81_nu0 * ri_factor / denom;
            }
}

/* =====================================================================
 * Bryan-Lewis background fill (rdb_ocean_vmix.F90:2387-2434)
 * ===================================================================== */
static void bkgnd_fill(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double inv_pi = 1.0 / PI_;
    const double kd_sfc = c->bkgnd_kd_sfc, kd_deep = c->bkgnd_kd_deep;
    const double z0 = c->bkgnd_z0, delta = c->bkgnd_delta;
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double depth = 0.0;
            for (int k = nz; k >= 2; --k) {
                depth = depth + C3(s->h, i, j, k);
                C3(s->kd_bg, i, j, k) =
                    kd_sfc + (kd_deep - kd_sfc) * (0.5 + vpo_sm_atan((depth - z0) / delta) * inv_pi);
            }
        }
}

/* interior_closure = "none" seed (rdb_ocean_vmix.F90:676-797; Henyey not
 * supported here). */
void vpo_seed_interior_none(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    if (c->bkgnd_profile) {
        double pr_bl = 1.0;
        if (c->bkgnd_prandtl > 0.0) pr_bl = c->bkgnd_prandtl;
        bkgnd_fill(c, s);
        for (int k = 1; k <= nz + 1; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    if (k == 1 || k == nz + 1) {
                        C3(s->kv, i, j, k) = 0.0;
                        C3(s->kt, i, j, k) = 0.0;
                    } else {
                        C3(s->kv, i, j, k) = pr_bl * C3(s->kd_bg, i, j, k);
                        C3(s->kt, i, j, k) = C3(s->kd_bg, i, j, k);
                    }
                }
    } else {
        double kv_seed = c->kv_bg, kt_seed = c->kt_bg;
        if (c->bkgnd_prandtl > 0.0) kv_seed = c->bkgnd_prandtl * c->kt_bg + c->kv_bg;
        for (int k = 1; k <= nz + 1; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    if (k == 1 || k == nz + 1) {
                        C3(s->kv, i, j, k) = 0.0;
                        C3(s->kt, i, j, k) = 0.0;
                    } else {
                        C3(s->kv, i, j, k) = kv_seed;
                        C3(s->kt, i, j, k) = kt_seed;
                    }
                }
    }
}

/* rdb_vl_first_live (rdb_vanished_layer.inc:82-110) */
static inline int first_live(const double *h, int nx, int ny, int i, int j, int kstart)
{
    int r = kstart;
    for (int k = kstart; k >= 1; --k) {
        if (C3(h, i, j, k) > H_VANISHED) {
            r = k;
            break;
        }
    }
    return r;
}

/* kpp_surface_buoyancy_flux (rdb_ocean_vmix.F90:1518-1559) */
static inline double kpp_b0(double alpha_T, double beta_S, double rho0, double qT, double qS)
{
    return (GRAVITY / rho0) * (alpha_T * qT - beta_S * qS);
}

/* sw_transmission (rdb_ocean_surface_flux.F90:1401-1415): the two-band
 * normalised downward irradiance at depth d, R e^(-d/zeta1) + (1-R) e^(-d/zeta2). */
static inline double sw_transmission(const vphys_config *c, double d)
{
    return c->sw_band_ratio * vpo_sm_exp(-d / c->sw_zeta1) + (1.0 - c->sw_band_ratio) * vpo_sm_exp(-d / c->sw_zeta2);
}

/* sw_band_fractions (rdb_ocean_surface_flux.F90:767-782): band n (1-based)
 * of nb carries blue 0.42 / (1 - blue) 0.42 of the visible, or an even share
 * of the near-infrared 0.58 for n >= 3. */
double vpo_sw_band_frac(int n, int nb, double blue)
{
    const double vis = 0.42;
    if (n == 1) return blue * vis;
    if (n == 2) return (1.0 - blue) * vis;
    return (1.0 - vis) / (double)(nb - 2);
}

/* sw_transmission_nb (:795-812): sum_n frac_n exp(-kappa_n(i,j) d). */
double vpo_sw_transmission_nb(const vphys_config *c, const vpo_state *s, int i, int j, double d)
{
    const int nx = s->nx, ny = s->ny;
    double trans = 0.0;
    for (int n = 1; n <= c->sw_nbands; ++n)
        trans = trans + vpo_sw_band_frac(n, c->sw_nbands, c->sw_blue_frac) *
                            vpo_sm_exp(-(s->sw_kappa[(size_t)(i - 1) + (size_t)nx * (j - 1) + (size_t)nx * ny * (n - 1)] * d));
    return trans;
}

/* sw_chl_fill_kappa -> sw_kappa_band_impl (rdb_ocean_sw_chl.F90:160-190) with
 * sw_opacity_manizza (rdb_ocean_surface_flux.F90:784-793): kappa_n =
 * a_n + b_n rdb_sm_pow(max(chl, 1e-4), p_n) on wet columns, the land value
 * elsewhere. */
void vpo_sw_chl_kappa(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny;
    for (int n = 1; n <= c->sw_nbands; ++n)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const size_t at = (size_t)(i - 1) + (size_t)nx * (j - 1) + (size_t)nx * ny * (n - 1);
                s->sw_kappa[at] = C2(s->wet, i, j) > 0.5
                                      ? c->sw_opacity_coef[2 * n - 2] +
                                            c->sw_opacity_coef[2 * n - 1] *
                                                vpo_sm_pow(fmx(C2(s->sw_chl, i, j), 1.0e-4), c->sw_chl_power[n - 1])
                                      : c->sw_opacity_land;
            }
}

/* The kinematic heat flux B0 charges (rdb_ocean_vmix.F90:1321-1348 in pass 1
 * with the lagged h_b, 1440-1466 in pass 2 with the new one): with
 * shortwave penetration on, Q_heat minus the penetrating part that passes
 * the boundary layer (MXL) or the surface layer (LV1), sw_pen_frac times the
 * selected shortwave source (sw_src, :1102-1117); all of it otherwise. */
static inline double kpp_q_t_kin(const vphys_config *c, const vpo_state *s, int i, int j, int k_sfc, double h_b)
{
    const int nx = s->nx, ny = s->ny;
    if (c->sw_pen_frac != 0.0) {
        const double *sw = vpo_sw_source(c, s);
        double q_bl = C2(s->q_heat, i, j);
        if (c->sw_chl) {   /* the N-band twin, :1326-1336 */
            if (c->kpp_sw_method == VPHYS_KPP_SW_MXL)
                q_bl = q_bl - c->sw_pen_frac * C2(sw, i, j) * vpo_sw_transmission_nb(c, s, i, j, h_b);
            else if (c->kpp_sw_method == VPHYS_KPP_SW_LV1)
                q_bl = q_bl - c->sw_pen_frac * C2(sw, i, j) * vpo_sw_transmission_nb(c, s, i, j, C3(s->h, i, j, k_sfc));
        } else if (c->kpp_sw_method == VPHYS_KPP_SW_MXL)
            q_bl = q_bl - c->sw_pen_frac * C2(sw, i, j) * sw_transmission(c, h_b);
        else if (c->kpp_sw_method == VPHYS_KPP_SW_LV1)
            q_bl = q_bl - c->sw_pen_frac * C2(sw, i, j) * sw_transmission(c, C3(s->h, i, j, k_sfc));
        return q_bl / (c->rho0 * c->cp);
    }
    return C2(s->q_heat, i, j) / (c->rho0 * c->cp);
}

/* The coefficient pair of B0 (rdb_ocean_vmix.F90:1357-1376, 1469-1488): the
 * constants, or with buoyancy_coeffs = "eos" the Wright derivatives at the
 * first live layer's (T, S) and p_ref when that layer is live. */
static inline double kpp_b0_col(const vphys_config *c, const vpo_state *s, int i, int j, int k_sfc, double qT,
                                double qS)
{
    const int nx = s->nx, ny = s->ny;
    double a = c->alpha_T, b = c->beta_S;
    if (c->buoyancy_coeffs && C3(s->h, i, j, k_sfc) > H_VANISHED)
        vpo_eos_buoyancy_coeffs(C3(s->tr[c->idx_temperature], i, j, k_sfc), C3(s->tr[c->idx_salinity], i, j, k_sfc),
                                c->eos_p_ref, &a, &b);
    return kpp_b0(a, b, c->rho0, qT, qS);
}

/* =====================================================================
 * KPP overlay (rdb_ocean_vmix.F90:1121-1516), constant buoyancy
 * coefficients, no penetrating shortwave (sw_active = .false.).
 * ===================================================================== */
void vpo_kpp_overlay(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double rho0 = c->rho0;
    const double *h = s->h, *u = s->u, *v = s->v, *rho = s->rho;
    for (size_t n = 0; n < (size_t)nx * ny * (nz + 1); ++n) {
        s->gamma_t[n] = 0.0;
        s->gamma_s[n] = 0.0;
    }
    /* ---- pass 1: BL depth ---- */
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            int k_sfc = first_live(h, nx, ny, i, j, nz);
            double u_ref = 0.5 * (U3(u, i, j, k_sfc) + U3(u, i + 1, j, k_sfc));
            double v_ref = 0.5 * (V3(v, i, j, k_sfc) + V3(v, i, j + 1, k_sfc));
            double b_ref = -(GRAVITY * C3(rho, i, j, k_sfc) / rho0);
            double d_centre_ref = 0.5 * C3(h, i, j, k_sfc);
            double tau_mag = C2(s->stress_mag, i, j);
            double u_star = sqrt(tau_mag / rho0);
            double h_b_lagged = C2(s->bl_depth, i, j);
            double q_T_kin = kpp_q_t_kin(c, s, i, j, k_sfc, h_b_lagged);
            double q_S_kin = C2(s->q_salt, i, j) / rho0;
            double B_0 = kpp_b0_col(c, s, i, j, k_sfc, q_T_kin, q_S_kin);
            double wstar3_lagged = fmx(0.0, -B_0) * h_b_lagged;
            double cb = vpo_sm_cbrt(wstar3_lagged);
            double w_s_col = sqrt(u_star * u_star + cb * cb);
            double ri_prev = 0.0, d_prev = d_centre_ref, h_b = 0.0;
            int crossing_found = 0;
            double d_centre_k = d_centre_ref;
            for (int k = k_sfc - 1; k >= 1; --k) {
                if (!crossing_found) {
                    d_centre_k = d_centre_k + 0.5 * (C3(h, i, j, k + 1) + C3(h, i, j, k));
                    double u_k = 0.5 * (U3(u, i, j, k) + U3(u, i + 1, j, k));
                    double v_k = 0.5 * (V3(v, i, j, k) + V3(v, i, j + 1, k));
                    double b_k = -(GRAVITY * C3(rho, i, j, k) / rho0);
                    double delta_d = d_centre_k - d_centre_ref;
                    double delta_b = b_ref - b_k;
                    double n_brunt = sqrt(fmx(0.0, delta_b / delta_d));
                    double vt2 = (c->c_vt2 / c->ri_crit) * d_centre_k * n_brunt * w_s_col;
                    double shear2 = fmx((u_k - u_ref) * (u_k - u_ref) + (v_k - v_ref) * (v_k - v_ref) + vt2,
                                        c->shear2_floor);
                    double ri_bulk = delta_b * delta_d / shear2;
                    if (ri_bulk >= c->ri_crit) {
                        double denom = ri_bulk - ri_prev;
                        double frac;
                        if (fabs(denom) > 1.0e-12)
                            frac = (c->ri_crit - ri_prev) / denom;
                        else
                            frac = 0.5;
                        h_b = d_prev + frac * (d_centre_k - d_prev);
                        crossing_found = 1;
                    }
                    ri_prev = ri_bulk;
                    d_prev = d_centre_k;
                }
            }
            if (!crossing_found) {
                h_b = 0.0;
                for (int k = 1; k <= k_sfc; ++k) h_b = h_b + C3(h, i, j, k);
            }
            C2(s->bl_depth, i, j) = h_b;
        }
    /* ---- pass 2: overlay ---- */
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            int k_sfc = first_live(h, nx, ny, i, j, nz);
            double tau_mag = C2(s->stress_mag, i, j);
            double u_star = sqrt(tau_mag / rho0);
            double h_b = C2(s->bl_depth, i, j);
            double q_T_kin = kpp_q_t_kin(c, s, i, j, k_sfc, h_b);
            double q_S_kin = C2(s->q_salt, i, j) / rho0;
            double B_0 = kpp_b0_col(c, s, i, j, k_sfc, q_T_kin, q_S_kin);
            C2(s->b0, i, j) = B_0;
            int destabilizing = B_0 < 0.0;
            double wstar3 = fmx(0.0, -B_0) * h_b;
            double w_star = vpo_sm_cbrt(wstar3);
            double w_s = sqrt(u_star * u_star + w_star * w_star);
            if (h_b > 0.0 && w_s > 0.0) {
                double d_running = 0.0;
                for (int k = k_sfc; k >= 1; --k) {
                    d_running = d_running + C3(h, i, j, k);
                    double d_face_k = d_running;
                    if (k > 1 && d_face_k < h_b) {
                        double sigma = d_face_k / h_b;
                        double g_shape = sigma * (1.0 - sigma) * (1.0 - sigma);
                        double kv_kpp = h_b * w_s * g_shape;
                        C3(s->kv, i, j, k) = fmx(C3(s->kv, i, j, k), kv_kpp);
                        C3(s->kt, i, j, k) = fmx(C3(s->kt, i, j, k), kv_kpp);
                        if (destabilizing) {
                            double gamma_factor = c->cs_nonlocal * g_shape;
                            C3(s->gamma_t, i, j, k) = gamma_factor * q_T_kin;
                            C3(s->gamma_s, i, j, k) = gamma_factor * q_S_kin;
                        }
                    }
                }
            }
        }
}

/* KV_ML_INVZ2 surface band (rdb_ocean_vmix.F90:1716-1766) */
void vpo_kv_ml_invz2(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    if (c->kv_ml_invz2 <= 0.0) return;
    if (c->hmix_fixed <= 0.0) return;
    double hmix = c->hmix_fixed;
    double hmix_sq = hmix * hmix;
    double dz_min_safe = 0.5 * hmix / (double)(nz > 1 ? nz : 1);
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double z = 0.0;
            for (int k = nz; k >= 2; --k) {
                z = z + C3(s->h, i, j, k);
                if (z >= hmix) break;
                double zz = fmx(z, dz_min_safe);
                double kv_extra = c->kv_ml_invz2 * hmix_sq / (zz * zz);
                C3(s->kv, i, j, k) = C3(s->kv, i, j, k) + kv_extra;
            }
        }
}

/* Convective adjustment (rdb_ocean_vmix.F90:1768-1849), masked below the
 * KPP bl_depth. */
void vpo_convection(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    if (!c->conv_enable) return;
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double z = 0.0;
            for (int k = nz; k >= 2; --k) {
                z = z + C3(s->h, i, j, k);
                double dz_face = 0.5 * (C3(s->h, i, j, k - 1) + C3(s->h, i, j, k));
                if (dz_face <= H_VANISHED) continue;
                if (z < (c->epbl ? C2(s->mld_epbl, i, j) : C2(s->bl_depth, i, j))) continue;
                double n2 = -(GRAVITY * (C3(s->rho, i, j, k) - C3(s->rho, i, j, k - 1)) / (c->rho0 * dz_face));
                if (n2 < c->conv_n2_thresh) {
                    C3(s->kt, i, j, k) = fmx(C3(s->kt, i, j, k), c->conv_kd);
                    C3(s->kv, i, j, k) = fmx(C3(s->kv, i, j, k), c->conv_prandtl * c->conv_kd);
                }
            }
        }
}

/* ks := kt (rdb_ocean_vmix.F90:1921-1934) */
void vpo_split(const vphys_config *c, vpo_state *s)
{
    (void)c;
    size_t n = (size_t)s->nx * s->ny * (s->nz + 1);
    memcpy(s->ks, s->kt, n * sizeof(double));
}

static void smooth_121(vpo_state *s, double *fld, double *scratch)
{
    /* vmix_smooth_121_impl (rdb_ocean_vmix.F90:2699-2748) */
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double *wet = s->wet;
    size_t n = (size_t)nx * ny * (nz + 1);
    memcpy(scratch, fld, n * sizeof(double));
    for (int k = 2; k <= nz; ++k)
        for (int j = 2; j <= ny - 1; ++j)
            for (int i = 2; i <= nx - 1; ++i) {
                double w_c = 4.0 * C2(wet, i, j);
                double w_e = 2.0 * C2(wet, i + 1, j);
                double w_w = 2.0 * C2(wet, i - 1, j);
                double w_n = 2.0 * C2(wet, i, j + 1);
                double w_s = 2.0 * C2(wet, i, j - 1);
                double w_ne = C2(wet, i + 1, j + 1);
                double w_nw = C2(wet, i - 1, j + 1);
                double w_se = C2(wet, i + 1, j - 1);
                double w_sw = C2(wet, i - 1, j - 1);
                double wsum = w_c + w_e + w_w + w_n + w_s + w_ne + w_nw + w_se + w_sw;
                if (wsum <= 0.0 || C2(wet, i, j) == 0.0) {
                    C3(fld, i, j, k) = C3(scratch, i, j, k);
                } else {
                    C3(fld, i, j, k) =
                        (w_c * C3(scratch, i, j, k) + w_e * C3(scratch, i + 1, j, k) +
                         w_w * C3(scratch, i - 1, j, k) + w_n * C3(scratch, i, j + 1, k) +
                         w_s * C3(scratch, i, j - 1, k) + w_ne * C3(scratch, i + 1, j + 1, k) +
                         w_nw * C3(scratch, i - 1, j + 1, k) + w_se * C3(scratch, i + 1, j - 1, k) +
                         w_sw * C3(scratch, i - 1, j - 1, k)) /
                        wsum;
                }
            }
}

/* vmix_assemble (rdb_ocean_vmix.F90:2183-2366): guard, floors, ceilings,
 * smoothing.  Returns 1 when the guard tripped, else 0. */
int vpo_assemble_gate(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    int status = 0;
    if (c->vmix_guard) {
        long bad = 0;
        for (int k = 2; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    double a = C3(s->kv, i, j, k), b = C3(s->kt, i, j, k), d = C3(s->ks, i, j, k);
                    if (a < 0.0 || a != a) bad++;
                    if (b < 0.0 || b != b) bad++;
                    if (d < 0.0 || d != d) bad++;
                }
        if (bad > 0) status = 1;
    }
    if (c->bkgnd_profile) {
        double pr_bl = 1.0;
        if (c->bkgnd_prandtl > 0.0) pr_bl = c->bkgnd_prandtl;
        bkgnd_fill(c, s);
#pragma omp parallel for
        for (int k = 2; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    double kdb = C3(s->kd_bg, i, j, k);
                    C3(s->kv, i, j, k) = fmn(fmx(C3(s->kv, i, j, k), pr_bl * kdb), c->kv_max);
                    C3(s->kt, i, j, k) = fmn(fmx(C3(s->kt, i, j, k), kdb), c->kd_max);
                    C3(s->ks, i, j, k) = fmn(fmx(C3(s->ks, i, j, k), kdb), c->kd_max);
                }
    } else {
        double kv_floor = c->kv_bg;
        if (c->bkgnd_prandtl > 0.0) kv_floor = c->bkgnd_prandtl * c->kt_bg + c->kv_bg;
#pragma omp parallel for
        for (int k = 2; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    C3(s->kv, i, j, k) = fmn(fmx(C3(s->kv, i, j, k), kv_floor), c->kv_max);
                    C3(s->kt, i, j, k) = fmn(fmx(C3(s->kt, i, j, k), c->kt_bg), c->kd_max);
                    C3(s->ks, i, j, k) = fmn(fmx(C3(s->ks, i, j, k), c->ks_bg), c->kd_max);
                }
    }
    if (c->kd_smooth_iterations > 0) {
        size_t n = (size_t)nx * ny * (nz + 1);
        double *scratch = (double *)malloc(n * sizeof(double));
        for (int it = 0; it < c->kd_smooth_iterations; ++it) {
            smooth_121(s, s->kv, scratch);
            smooth_121(s, s->kt, scratch);
            smooth_121(s, s->ks, scratch);
        }
        free(scratch);
    }
    return status;
}

/* vmix_build_coefficients (rdb_ocean_dyn.F90:1473-1634) with the EPBL and
 * kappa-shear merges of the kd_epbl / kd_shear last computed (1546-1583); no
 * tidal / BBL mixing. */
int vpo_build_coefficients(const vphys_config *c, vpo_state *s)
{
    if (c->interior_closure == VPHYS_INTERIOR_PP81)
        vpo_pp81(c, s);
    else
        vpo_seed_interior_none(c, s);
    if (c->use_kpp && !c->epbl) vpo_kpp_overlay(c, s);   /* EPBL replaces KPP (rdb_ocean_dyn.F90:1539) */
    if (c->epbl) vpo_epbl_merge(c, s);   /* with combine = max_shear it merges kappa-shear first */
    if (c->kappa_shear && !(c->epbl && c->epbl_combine == 3)) vpo_kappa_shear_merge(c, s);
    vpo_kv_ml_invz2(c, s);
    if (c->conv_enable) vpo_convection(c, s);
    vpo_split(c, s);
    return vpo_assemble_gate(c, s);
}

/* =====================================================================
 * Tracer vertical diffusion (rdb_ocean_vdiff.F90:1107-1414, 1928-1962)
 * ===================================================================== */
static inline double face_thick(double ha, double hb, int use_harmonic)
{
    if (use_harmonic) {
        double sum_h = ha + hb;
        if (sum_h > 1.0e-30) return 2.0 * ha * hb / sum_h;
        return 0.5 * sum_h;
    }
    return 0.5 * (ha + hb);
}

/* build_factorize_tracer_matrix for one column; col arrays are 1-based. */
static void factor_column(int nz, int use_harmonic, double dt, const double *kvc /* nz+1 */,
                          const double *hcol /* nz */, double *a, double *b, double *cc)
{
    double hc = fmx(hcol[0], H_VANISHED);
    double alpha = 0.0;
    if (nz > 1) {
        double hp = fmx(hcol[1], H_VANISHED);
        double dz_face = face_thick(hc, hp, use_harmonic);
        alpha = dt * kvc[1] / (hc * dz_face);
        if (hcol[0] <= H_VANISHED || hcol[1] <= H_VANISHED) alpha = 0.0;
    }
    a[0] = 0.0;
    cc[0] = -alpha;
    b[0] = 1.0 + alpha;
    for (int k = 2; k <= nz - 1; ++k) {
        double hm = fmx(hcol[k - 2], H_VANISHED);
        hc = fmx(hcol[k - 1], H_VANISHED);
        double hp = fmx(hcol[k], H_VANISHED);
        double beta = dt * kvc[k - 1] / (hc * face_thick(hm, hc, use_harmonic));
        alpha = dt * kvc[k] / (hc * face_thick(hc, hp, use_harmonic));
        if (hcol[k - 1] <= H_VANISHED || hcol[k - 2] <= H_VANISHED) beta = 0.0;
        if (hcol[k - 1] <= H_VANISHED || hcol[k] <= H_VANISHED) alpha = 0.0;
        a[k - 1] = -beta;
        cc[k - 1] = -alpha;
        b[k - 1] = 1.0 + alpha + beta;
    }
    if (nz > 1) {
        double hm = fmx(hcol[nz - 2], H_VANISHED);
        hc = fmx(hcol[nz - 1], H_VANISHED);
        double dz_face = face_thick(hm, hc, use_harmonic);
        double beta = dt * kvc[nz - 1] / (hc * dz_face);
        if (hcol[nz - 1] <= H_VANISHED || hcol[nz - 2] <= H_VANISHED) beta = 0.0;
        a[nz - 1] = -beta;
        cc[nz - 1] = 0.0;
        b[nz - 1] = 1.0 + beta;
    }
    cc[0] = cc[0] / b[0];
    for (int k = 2; k <= nz; ++k) {
        double denom = b[k - 1] - a[k - 1] * cc[k - 2];
        cc[k - 1] = cc[k - 1] / denom;
        b[k - 1] = denom;
    }
}

/* apply_factored_tracer for one column (in place on ccol). */
static void apply_column(int nz, const double *hcol, double *ccol, const double *a, const double *b,
                         const double *cc, double *rhs, double *budget_col /* may be NULL */)
{
    for (int k = 0; k < nz; ++k) rhs[k] = ccol[k];
    rhs[0] = rhs[0] / b[0];
    for (int k = 2; k <= nz; ++k) rhs[k - 1] = (rhs[k - 1] - a[k - 1] * rhs[k - 2]) / b[k - 1];
    for (int k = nz - 1; k >= 1; --k) rhs[k - 1] = rhs[k - 1] - cc[k - 1] * rhs[k];
    if (budget_col) {
        for (int k = 0; k < nz; ++k) {
            double p_new = hcol[k] * rhs[k];
            double p_old = hcol[k] * ccol[k];
            budget_col[k] = budget_col[k] + (p_new - p_old);
            ccol[k] = rhs[k];
        }
    } else {
        for (int k = 0; k < nz; ++k) ccol[k] = rhs[k];
    }
}

static void tracer_pass(const vphys_config *c, vpo_state *s, double dt, const double *ksrc, int temperature_pass)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel
    {
        double kvc[VPHYS_NZ_MAX + 1], hcol[VPHYS_NZ_MAX], a[VPHYS_NZ_MAX], b[VPHYS_NZ_MAX], cc[VPHYS_NZ_MAX];
        double rhs[VPHYS_NZ_MAX], ccol[VPHYS_NZ_MAX], bud[VPHYS_NZ_MAX];
#pragma omp for
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                for (int k = 1; k <= nz + 1; ++k) kvc[k - 1] = C3(ksrc, i, j, k);
                for (int k = 1; k <= nz; ++k) hcol[k - 1] = C3(s->h, i, j, k);
                factor_column(nz, c->use_harmonic, dt, kvc, hcol, a, b, cc);
                for (int t = 0; t < s->ntr; ++t) {
                    int is_T = (t == c->idx_temperature);
                    if (temperature_pass != is_T) continue;
                    double *trc = s->tr[t];
                    double *budget = NULL;
                    if (c->budgets) {
                        if (is_T) budget = s->heat_budget;
                        else if (t == c->idx_salinity) budget = s->salt_budget;
                    }
                    for (int k = 1; k <= nz; ++k) ccol[k - 1] = C3(trc, i, j, k);
                    if (budget)
                        for (int k = 1; k <= nz; ++k) bud[k - 1] = C3(budget, i, j, k);
                    apply_column(nz, hcol, ccol, a, b, cc, rhs, budget ? bud : NULL);
                    for (int k = 1; k <= nz; ++k) C3(trc, i, j, k) = ccol[k - 1];
                    if (budget)
                        for (int k = 1; k <= nz; ++k) C3(budget, i, j, k) = bud[k - 1];
                }
            }
    }
}

/* vdiff_apply_tracers with kt_source and ks_source (case 3). */
void vpo_vdiff_tracers(const vphys_config *c, vpo_state *s, double dt)
{
    tracer_pass(c, s, dt, s->kt, 1);
    tracer_pass(c, s, dt, s->ks, 0);
}

/* =====================================================================
 * KPP non-local tendencies (rdb_ocean_vmix.F90:1605-1714,
 * rdb_tracer_conc.inc:36-53)
 * ===================================================================== */
static inline double nonlocal_face_flux(double gamma, double h_below, double h_above)
{
    if (h_below > H_VANISHED && h_above > H_VANISHED) return gamma;
    return 0.0;
}

static inline double conc_add_source(double cval, double h, double src)
{
    if (h > H_VANISHED) return cval + src / (h + H_DIV_EPS);
    return cval;
}

static void nonlocal_one(vpo_state *s, double dt, const double *gam, double *trc)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double f_up = 0.0, f_dn = 0.0;
                if (k < nz) f_up = nonlocal_face_flux(C3(gam, i, j, k + 1), C3(s->h, i, j, k), C3(s->h, i, j, k + 1));
                if (k > 1) f_dn = nonlocal_face_flux(C3(gam, i, j, k), C3(s->h, i, j, k - 1), C3(s->h, i, j, k));
                C3(trc, i, j, k) = conc_add_source(C3(trc, i, j, k), C3(s->h, i, j, k), dt * (f_up - f_dn));
            }
}

void vpo_nonlocal(const vphys_config *c, vpo_state *s, double dt)
{
    if (c->idx_temperature >= 0) nonlocal_one(s, dt, s->gamma_t, s->tr[c->idx_temperature]);
    if (c->idx_salinity >= 0) nonlocal_one(s, dt, s->gamma_s, s->tr[c->idx_salinity]);
    if (c->idx_pseudo_salt >= 0) nonlocal_one(s, dt, s->gamma_s, s->tr[c->idx_pseudo_salt]);
}

/* =====================================================================
 * Momentum vertical viscosity (rdb_ocean_vdiff.F90:1416-1926, 1964-2115,
 * rdb_bed_live_face.inc), without the ice-shelf top drag and the corner
 * viscosity add-on.  `xf` selects u faces (nu = nx+1, nv = ny) or v faces.
 * ===================================================================== */
#define EPS_HVEL 1.0e-30
#define STRESS_H_MIN 1.0e-3

static inline void face_layer(double hl_c, double hr_c, double u_k, int k, int kb, int hvel_mom6,
                              int hvel_harmonic, int hvel_upwind, int zlevel_faces, double d_min,
                              double i_hbbl, double *zacc, double *zcol_l, double *zcol_r, double *hvel,
                              double *zint)
{
    double h_harm, h_arith, h_delta, z_clear, z2, botfn;
    *zint = 0.0;
    if (hvel_mom6 && !hvel_harmonic) {
        h_harm = 2.0 * hl_c * hr_c / (hl_c + hr_c + EPS_HVEL);
        h_arith = 0.5 * (hl_c + hr_c);
        h_delta = hr_c - hl_c;
        *zcol_l = *zcol_l + hl_c;
        *zcol_r = *zcol_r + hr_c;
        if (k >= kb) *zacc = *zacc + h_harm;
        z_clear = fmx(*zcol_l, *zcol_r) + d_min;
        *zint = fmx(*zacc, z_clear) * i_hbbl;
        *hvel = h_arith;
        if (u_k * h_delta > 0.0) {
            z2 = *zint;
            botfn = 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
            *hvel = (1.0 - botfn) * h_arith + botfn * h_harm;
        }
    } else if (hvel_mom6) {
        h_harm = 2.0 * hl_c * hr_c / (hl_c + hr_c + EPS_HVEL);
        h_arith = 0.5 * (hl_c + hr_c);
        h_delta = hr_c - hl_c;
        *hvel = h_harm;
        if (hvel_upwind && u_k * h_delta < 0.0) {
            z2 = *zacc;
            botfn = 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
            *hvel = (1.0 - botfn) * h_harm + botfn * h_arith;
        }
        if (k >= kb) *zacc = *zacc + h_harm * i_hbbl;
        *zint = *zacc;
    } else {
        *hvel = 0.5 * (hl_c + hr_c);
    }
    if (zlevel_faces) *hvel = fmn(hl_c, hr_c);
}

static inline void interface_coupling(double hv_lo, double hv_hi, double zint_lo, double dt, int hvel_mom6,
                                      int use_harmonic, int bbl_glue, double kv_bbl, double kv_bbl_bg,
                                      double bbl_thick, int zlevel_faces, double kv_l, double kv_r, double *num,
                                      double *dz, int *cut)
{
    double hf_lo = fmx(hv_lo, H_VANISHED);
    double hf_hi = fmx(hv_hi, H_VANISHED);
    if (hvel_mom6)
        *dz = 0.5 * (hf_lo + hf_hi);
    else
        *dz = face_thick(hf_lo, hf_hi, use_harmonic);
    double nu_f = 0.5 * (kv_l + kv_r);
    if (bbl_glue) {
        double z = zint_lo;
        double botfn_int = 1.0 / (1.0 + 0.09 * z * z * z * z * z * z);
        nu_f = fmx(0.0, nu_f + (kv_bbl - kv_bbl_bg) * botfn_int);
        if (*dz > bbl_thick) *dz = (1.0 - botfn_int) * (*dz) + botfn_int * bbl_thick;
    }
    *num = dt * nu_f;
    *cut = zlevel_faces && (hv_lo <= H_VANISHED || hv_hi <= H_VANISHED);
}

static void diffuse_faces(const vphys_config *c, vpo_state *s, double dt, int xf)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int nu = xf ? nx + 1 : nx;
    const int nv = xf ? ny : ny + 1;
    double *uf = xf ? s->u : s->v;
    const double *tau = xf ? s->tau_x : s->tau_y;
    const double *lam = xf ? s->lambda_bot_u : s->lambda_bot_v;
    double *vrem = xf ? s->visc_rem_u : s->visc_rem_v;
    const int *ktopf = xf ? s->k_top_u : s->k_top_v;
    const int *kbotf = xf ? s->k_bot_u : s->k_bot_v;
    const double *h = s->h, *kvc = s->kv, *wet = s->wet;
    const int do_stress = c->implicit_stress, do_drag = c->implicit_drag, do_remnant = c->remnant;
    const double inv_rho0 = 1.0 / c->rho0;
#define F3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)nu * (((size_t)(j) - 1) + (size_t)nv * ((size_t)(k) - 1))]
#define F2(a, i, j) (a)[((size_t)(i) - 1) + (size_t)nu * ((size_t)(j) - 1)]
#pragma omp parallel
    {
        double cdiag[VPHYS_NZ_MAX], rhs[VPHYS_NZ_MAX];
#pragma omp for
        for (int j = 1; j <= nv; ++j)
            for (int i = 1; i <= nu; ++i) {
                int i_left, i_right, j_below, j_above;
                if (xf) {
                    i_left = i - 1 > 1 ? i - 1 : 1;
                    i_right = i < nx ? i : nx;
                    j_below = j;
                    j_above = j;
                } else {
                    i_left = i;
                    i_right = i;
                    j_below = j - 1 > 1 ? j - 1 : 1;
                    j_above = j < ny ? j : ny;
                }
                int kb = F2(kbotf, i, j);
                int ktop = F2(ktopf, i, j);
                double kv_bbl = 0.0, bbl_thick = c->hbbl_visc;
                if (c->bbl_glue) {
                    kv_bbl = c->bbl_piston * c->hbbl_visc;
                    bbl_thick = c->hbbl_visc;
                }
                double i_hbbl = 1.0 / (bbl_thick + EPS_HVEL);
                double zacc = 0.0, zcol_l = 0.0, zcol_r = 0.0;
                if (c->hvel_mom6 && !c->hvel_harmonic) {
                    for (int k = 1; k <= nz; ++k) {
                        zcol_l = zcol_l - C3(h, i_left, j_below, k);
                        zcol_r = zcol_r - C3(h, i_right, j_above, k);
                    }
                }
                double d_min = fmn(-zcol_l, -zcol_r);
                int kb_live = kb;
                for (int k = kb; k <= nz; ++k) {
                    int live = c->zlevel_faces ? (fmn(C3(h, i_left, j_below, k), C3(h, i_right, j_above, k)) > H_VANISHED)
                                               : 1;
                    if (live) {
                        kb_live = k;
                        break;
                    }
                }
                double hv_0, hv_p, zi_0, zi_p;
                face_layer(C3(h, i_left, j_below, 1), C3(h, i_right, j_above, 1), F3(uf, i, j, 1), 1, kb,
                           c->hvel_mom6, c->hvel_harmonic, c->hvel_upwind, c->zlevel_faces, d_min, i_hbbl, &zacc,
                           &zcol_l, &zcol_r, &hv_p, &zi_p);
                hv_0 = 0.0;
                zi_0 = 0.0;
                double num_t = 0.0, dz_t = 1.0;
                int cut_t = 0;
                double cp_prev = 0.0, dp_prev = 0.0, gp_prev = 0.0;
                double cp = 0.0, dp = 0.0, gp = 0.0;
                for (int k = 1; k <= nz; ++k) {
                    hv_0 = hv_p;
                    zi_0 = zi_p;
                    double num_b = num_t, dz_b = dz_t;
                    int cut_b = cut_t;
                    if (k < nz) {
                        face_layer(C3(h, i_left, j_below, k + 1), C3(h, i_right, j_above, k + 1), F3(uf, i, j, k + 1),
                                   k + 1, kb, c->hvel_mom6, c->hvel_harmonic, c->hvel_upwind, c->zlevel_faces, d_min,
                                   i_hbbl, &zacc, &zcol_l, &zcol_r, &hv_p, &zi_p);
                        if (k >= kb_live && k <= ktop) {
                            interface_coupling(hv_0, hv_p, zi_0, dt, c->hvel_mom6, c->use_harmonic, c->bbl_glue,
                                               kv_bbl, c->kv_bbl_bg, bbl_thick, c->zlevel_faces,
                                               C3(kvc, i_left, j_below, k + 1), C3(kvc, i_right, j_above, k + 1),
                                               &num_t, &dz_t, &cut_t);
                        }
                    }
                    double a_k = 0.0, b_k = 1.0, c_k = 0.0;
                    double hf_k = fmx(hv_0, H_VANISHED);
                    if (k == kb_live && k <= ktop) {
                        double alpha = 0.0;
                        if (kb_live < nz) {
                            alpha = num_t / (hf_k * dz_t);
                            if (cut_t) alpha = 0.0;
                        }
                        c_k = -alpha;
                        b_k = 1.0 + alpha;
                        if (c->bbl_glue) b_k = b_k + dt * kv_bbl / (hf_k * (fmn(0.5 * hv_0, bbl_thick) + EPS_HVEL));
                        if (do_drag && !c->bbl_glue) b_k = b_k + dt * F2(lam, i, j);
                    }
                    if (k == ktop && k > kb_live) {
                        double beta = num_b / (hf_k * dz_b);
                        if (cut_b) beta = 0.0;
                        a_k = -beta;
                        b_k = 1.0 + beta;
                    }
                    if (k > kb_live && k < ktop) {
                        double beta = num_b / (hf_k * dz_b);
                        double alpha = num_t / (hf_k * dz_t);
                        if (cut_b) beta = 0.0;
                        if (cut_t) alpha = 0.0;
                        a_k = -beta;
                        c_k = -alpha;
                        b_k = 1.0 + alpha + beta;
                    }
                    double r_k = F3(uf, i, j, k);
                    if (k == ktop) {
                        if (do_stress) {
                            double wind_open = 1.0;
                            r_k = r_k + dt * F2(tau, i, j) * wind_open *
                                            fmn(C2(wet, i_left, j_below), C2(wet, i_right, j_above)) * inv_rho0 /
                                            fmx(hf_k, STRESS_H_MIN);
                        }
                    }
                    if (k == 1) {
                        cp = c_k / b_k;
                        dp = r_k / b_k;
                        gp = 1.0 / b_k;
                    } else {
                        double denom = b_k - a_k * cp_prev;
                        cp = c_k / denom;
                        dp = (r_k - a_k * dp_prev) / denom;
                        gp = (1.0 - a_k * gp_prev) / denom;
                    }
                    cdiag[k - 1] = cp;
                    rhs[k - 1] = dp;
                    if (do_remnant) F3(vrem, i, j, k) = gp;
                    cp_prev = cp;
                    dp_prev = dp;
                    gp_prev = gp;
                }
                double u_next = dp_prev;
                double g_next = fmn(gp_prev, 1.0);
                F3(uf, i, j, nz) = u_next;
                if (do_remnant) F3(vrem, i, j, nz) = g_next;
                for (int k = nz - 1; k >= 1; --k) {
                    double cpk = cdiag[k - 1];
                    u_next = rhs[k - 1] - cpk * u_next;
                    F3(uf, i, j, k) = u_next;
                    if (do_remnant) {
                        g_next = fmn(F3(vrem, i, j, k) - cpk * g_next, 1.0);
                        F3(vrem, i, j, k) = g_next;
                    }
                }
            }
    }
#undef F3
#undef F2
}

void vpo_vdiff_momentum(const vphys_config *c, vpo_state *s, double dt)
{
    diffuse_faces(c, s, dt, 1);
    diffuse_faces(c, s, dt, 0);
}

/* One vmix_apply_in_stage on a thermo step (rdb_ocean_dyn.F90:1636-1900). */
/* ocean_surface_flux_apply_tracers (rdb_ocean_surface_flux.F90:959-1070):
 * the surface heat and salt fluxes stamped onto the first live layer from the
 * top (rdb_vl_first_live from k_top = nz) of T, S and the pseudo-salt mirror,
 * apply_surface_src_2d_impl (1093-1142) with its budget contributor and the
 * nobudget twin (1175-1203) for pseudo-salt; content -> concentration through
 * rdb_conc_add_source, the budget books rdb_conc_accepted_source
 * (rdb_tracer_conc.inc:33-63). */
void vpo_surface_flux(const vphys_config *c, vpo_state *s, double dt)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double inv_heat = dt / (c->rho0 * c->cp);
    const double inv_salt = dt / c->rho0;
    const int iT = c->idx_temperature, iS = c->idx_salinity, iPS = c->idx_pseudo_salt;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= ny; ++j) {
        for (int i = 1; i <= nx; ++i) {
            const int kt = first_live(s->h, nx, ny, i, j, nz);
            const double hk = C3(s->h, i, j, kt);
            const double w = C2(s->wet, i, j);
            /* apply_surface_src_2d_dyn_impl (1144-1225): the dynamic mask
             * multiplies after the static one */
            const int dyn = c->use_wet_dyn;
            if (iT >= 0) {
                double cell = inv_heat * C2(s->q_heat, i, j) * w;
                if (dyn) cell = cell * C2(s->wet_dyn, i, j);
                double *T = s->tr[iT];
                C3(T, i, j, kt) = conc_add_source(C3(T, i, j, kt), hk, cell);
                if (c->budgets) C3(s->heat_budget_surface, i, j, kt) += (hk > H_VANISHED) ? cell : 0.0;
            }
            if (iS >= 0) {
                double cell = inv_salt * C2(s->q_salt, i, j) * w;
                if (dyn) cell = cell * C2(s->wet_dyn, i, j);
                double *S = s->tr[iS];
                C3(S, i, j, kt) = conc_add_source(C3(S, i, j, kt), hk, cell);
                if (c->budgets) C3(s->salt_budget_surface, i, j, kt) += (hk > H_VANISHED) ? cell : 0.0;
            }
            if (iPS >= 0) {
                double cell = inv_salt * C2(s->q_salt, i, j) * w;
                if (dyn) cell = cell * C2(s->wet_dyn, i, j);
                double *PS = s->tr[iPS];
                C3(PS, i, j, kt) = conc_add_source(C3(PS, i, j, kt), hk, cell);
            }
            /* bound_salinity_top_impl (1072-1091), after the salt deposit:
             * the static mask, a thickness above H_DIV_EPS, not booked */
            if (c->bound_salinity && iS >= 0 && w > 0.5 && hk > H_DIV_EPS) {
                double *S = s->tr[iS];
                C3(S, i, j, kt) = fmx(C3(S, i, j, kt), c->min_salinity);
            }
        }
    }
}

/* ocean_surface_flux_apply_sw_penetration -> apply_sw_penetration_impl
 * (rdb_ocean_surface_flux.F90:1255-1370, 1451-1530) with k_top = nz and
 * k_bot = 1: the penetrating part I0 of the surface lump leaves the first
 * live layer and is spread as I0 (T(d_top) - T(d_bottom)) over the live
 * layers, the deepest live layer taking the rest (opaque bed); vanished
 * layers pass the light on. */
void vpo_sw_penetration(const vphys_config *c, vpo_state *s, double dt)
{
    if (c->sw_pen_frac == 0.0 || c->idx_temperature < 0) return;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double inv_scale = dt / (c->rho0 * c->cp);
    double *T = s->tr[c->idx_temperature];
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = 1; j <= ny; ++j) {
        for (int i = 1; i <= nx; ++i) {
            const int kt = first_live(s->h, nx, ny, i, j, nz);
            /* the chlorophyll scheme absorbs all of the source (apply_sw_penetration_nb_impl, 1606-1668) */
            const int nbs = c->sw_chl;
            double i0col = nbs ? C2(vpo_sw_source(c, s), i, j) * C2(s->wet, i, j)
                               : c->sw_pen_frac * C2(vpo_sw_source(c, s), i, j) * C2(s->wet, i, j);
            /* apply_sw_penetration_cover_impl / _nb_cover_impl (1532-1604, 1670-1730) */
            if (c->use_cover_frac) i0col = i0col * (1.0 - C2(s->cover_frac, i, j));
            int k_dep = 1;
            for (int k = 1; k <= nz; ++k) {
                if (C3(s->h, i, j, k) > H_VANISHED) {
                    k_dep = k;
                    break;
                }
            }
            double d_top = 0.0;
            double trans_top = nbs ? vpo_sw_transmission_nb(c, s, i, j, d_top) : sw_transmission(c, d_top);
            for (int k = nz; k >= k_dep; --k) {
                const double hk = C3(s->h, i, j, k);
                const double d_bot = d_top + hk;
                const double trans_bot =
                    (k > k_dep) ? (nbs ? vpo_sw_transmission_nb(c, s, i, j, d_bot) : sw_transmission(c, d_bot)) : 0.0;
                if (hk > H_VANISHED) {
                    const double absorbed = i0col * (trans_top - trans_bot);
                    double add = inv_scale * absorbed;
                    if (k == kt) add = add - inv_scale * i0col;
                    C3(T, i, j, k) = conc_add_source(C3(T, i, j, k), hk, add);
                    if (c->budgets) C3(s->heat_budget_surface, i, j, k) += add;
                    trans_top = trans_bot;
                }
                d_top = d_bot;
            }
        }
    }
}

int vpo_step(const vphys_config *c, vpo_state *s, double dt, int n_steps)
{
    int st = 0;
    for (int n = 0; n < n_steps; ++n) {
        if (c->eos_in_step) vpo_eos_wright(c, s);
        if (c->surface_flux) {
            vpo_surface_flux(c, s, dt);
            vpo_sw_penetration(c, s, dt);
        }
        if (c->epbl) vpo_epbl(c, s, dt);
        if (c->kappa_shear) vpo_kappa_shear(c, s, dt);
        st |= vpo_build_coefficients(c, s);
        vpo_vdiff_momentum(c, s, dt);
        vpo_vdiff_tracers(c, s, dt);
        if (c->use_kpp && !c->epbl) vpo_nonlocal(c, s, dt);   /* under EPBL its gamma is 0: a no-op */
    }
    return st;
}

/* =====================================================================
 * Compensated column content (the diagnostic of cfg.column_integrals)
 * ===================================================================== */
/* Neumaier's improvement of Kahan summation (Z. Angew. Math. Mech. 54, 1974):
 * the rounding error of every addition is carried in *cmp, whichever of the
 * two operands is larger. */
static inline void neumaier_add(double *sum, double *cmp, double x)
{
    const double t = *sum + x;
    if (fabs(*sum) >= fabs(x))
        *cmp += (*sum - t) + x;
    else
        *cmp += (x - t) + *sum;
    *sum = t;
}

void vpo_column_content(const vpo_state *s, int descending, double *out)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const size_t plane = (size_t)nx * ny;
#pragma omp parallel for
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            int lo = 0, hi = 0;
            for (int k = 1; k <= nz; ++k)
                if (C3(s->h, i, j, k) > H_VANISHED) {
                    lo = k;
                    break;
                }
            if (lo > 0)
                for (int k = nz; k >= lo; --k)
                    if (C3(s->h, i, j, k) > H_VANISHED) {
                        hi = k;
                        break;
                    }
            const size_t col = (size_t)(i - 1) + (size_t)nx * (j - 1);
            for (int t = 0; t < s->ntr; ++t) {
                double sum = 0.0, cmp = 0.0;
                if (lo > 0) {
                    for (int n = 0; n <= hi - lo; ++n) {
                        const int k = descending ? hi - n : lo + n;
                        neumaier_add(&sum, &cmp, C3(s->h, i, j, k) * C3(s->tr[t], i, j, k));
                    }
                }
                out[(size_t)t * plane + col] = sum + cmp;
            }
        }
}
