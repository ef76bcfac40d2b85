// vphys_device.cuh -- device-side building blocks of the vertical-physics
// kernels: constants, the position-independent cbrt/atan, and the per-level
// pieces of the momentum face column.  Every routine follows the operation
// order of the Fortran it cites, and the kernels are compiled without FMA
// contraction (-fmad=false), so a column's result is bit-identical to the CPU
// restatement built with -ffp-contract=off.
#pragma once

#include <cstdint>

#include "../../include/vphys.h"

namespace vphys {

constexpr double GRAVITY = 9.80665;        // rdb_constants.F90:37
constexpr double H_VANISHED = 1.5e-4;      // rdb_constants.F90:67
constexpr double H_DIV_EPS = 1.0e-20;      // rdb_constants.F90:85
constexpr double PI_D = 3.141592653589793115997963468544185161590576171875;  // 4*atan(1)
constexpr double EPS_HVEL = 1.0e-30;       // rdb_ocean_vdiff.F90 diffuse_velocity_columns_impl
constexpr double STRESS_H_MIN = 1.0e-3;
constexpr double DBL_TINY = 2.2250738585072014e-308;

// Wright (1997) reduced-range coefficients (rdb_eos.F90:200-217, Table A1)
constexpr double WRIGHT_A0 = 7.057924e-4, WRIGHT_A1 = 3.480336e-7, WRIGHT_A2 = -1.112733e-7;
constexpr double WRIGHT_B0 = 5.790749e8, WRIGHT_B1 = 3.516535e6, WRIGHT_B2 = -4.002714e4, WRIGHT_B3 = 2.084372e2,
                 WRIGHT_B4 = 5.944068e5, WRIGHT_B5 = -9.643486e3;
constexpr double WRIGHT_C0 = 1.704853e5, WRIGHT_C1 = 7.904722e2, WRIGHT_C2 = -7.984422e0, WRIGHT_C3 = 5.140652e-2,
                 WRIGHT_C4 = -2.302158e2, WRIGHT_C5 = -3.079464e0;

// ---- exact division helpers ----------------------------------------------
// xdiv(a, b) == a / b for every input.  A zero numerator is answered directly
// (the quotient is a zero carrying the XOR of the signs): the general IEEE
// division takes a slow path of ~90 instructions for a zero operand, and the
// path divides zeros all the time (a non-local source that is zero below the
// boundary layer, an ideal-age tracer that starts at zero, the harmonic mean
// of two vanished layers).
__device__ __forceinline__ double xdiv(double a, double b)
{
    if (a == 0.0 && b != 0.0 && isfinite(b))
        return ((__double_as_longlong(a) ^ __double_as_longlong(b)) < 0) ? -0.0 : 0.0;
    return a / b;
}

// Division of several numerators by one denominator with a single correctly
// rounded reciprocal y = RN(1/b) and Markstein's correction (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(a*y), r = a - b*q0
// (exact with an FMA), q = RN(q0 + r*y) is RN(a/b) when y is within half an
// ulp of 1/b, q0 within one ulp of a/b and nothing over- or underflows.  The
// operands are kept inside [2^-500, 2^500] for that; anything else (zeros,
// extremes, NaN, Inf) takes xdiv.  tests/test_gpu_division.py checks the
// result against a/b bit for bit.
struct Rcp {
    double b, y;
    bool fast;
};
__device__ __forceinline__ Rcp rcp_of(double b)
{
    Rcp r;
    r.b = b;
    r.y = 1.0 / b;
    const double ab = fabs(b);
    r.fast = ab >= 0x1p-500 && ab <= 0x1p500;
    return r;
}
__device__ __forceinline__ double qdiv(double a, const Rcp &r)
{
    const double aa = fabs(a);
    if (r.fast && aa >= 0x1p-500 && aa <= 0x1p500) {
        const double q0 = __dmul_rn(a, r.y);
        const double rem = __fma_rn(-r.b, q0, a);
        return __fma_rn(rem, r.y, q0);
    }
    return xdiv(a, r.b);
}

// Fortran MAX/MIN (finite operands); the same ternary as the CPU restatement.
__device__ __forceinline__ double fmx(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double fmn(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ float fmx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }

// Precision-generic spellings used by the templated kernels: for double they
// are the exact helpers above (value-identical to a/b); for float (the
// mixed-precision path, no bitwise contract) the hardware fast forms.
__device__ __forceinline__ double rdiv(double a, double b) { return xdiv(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdividef(a, b); }
struct RcpF {
    float y;
};
__device__ __forceinline__ RcpF rcp_of(float b) { return RcpF{__frcp_rn(b)}; }
__device__ __forceinline__ float qdiv(float a, const RcpF &r) { return a * r.y; }

// ---- position-independent cube root: rdb_sm_cbrt
// (rdb_safe_math_pow.inc:107-142): exponent split modulo 3, degree-4 seed on
// the mantissa in [1/2, 4), two Halley steps; tables rdb_safe_math_consts.inc:90-92.
__device__ __forceinline__ double sm_cbrt(double x)
{
    if (isnan(x) || !isfinite(x)) return x;
    double ax = fabs(x);
    if (ax < DBL_TINY) return copysign(0.0, x);
    int e;
    double f = frexp(ax, &e);
    int rem = ((e % 3) + 3) % 3;
    int q = (e - rem) / 3;
    double m = ldexp(f, rem);
    double y0 = -0.003660165019409192949;
    y0 = y0 * m + 0.04437845996234061896;
    y0 = y0 * m + -0.2158001895775201462;
    y0 = y0 * m + 0.6542973117201534849;
    y0 = y0 * m + 0.5189978361037301813;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        double y3 = (y0 * y0) * y0;
        y0 = y0 + y0 * xdiv(m - y3, (y3 + y3) + m);
    }
    double y = ldexp(y0, q);
    return x < 0.0 ? -y : y;
}

// ---- position-independent exponential: rdb_sm_exp
// (rdb_safe_math_core.inc:81-137, constants rdb_safe_math_consts.inc:39-52):
// k = nearest integer to x/ln2 (halves away from zero), r = x - k ln2 with
// ln2 split so k*LN2_HI is exact, degree-13 Taylor polynomial (1/i!), 2**k;
// results below the smallest normal are exactly 0.
// exp(x + c): the correction c joins the reduced argument (0 for plain exp;
// the tail of a double-double exponent for sm_pow), rdb_sm_exp_core
// (rdb_safe_math_core.inc:81-114)
__device__ __forceinline__ double sm_exp_core(double x, double c)
{
    const double kr = round(x * 1.442695040888963387);
    const int k = (int)kr;
    double r = x - kr * 0.69314718060195446014;
    r = r - kr * -4.2009150726810845979e-11;
    r = r + c;
    double p = 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 1.0 / 2.0;
    p = p * r + 1.0;
    p = p * r + 1.0;
    double y = (k > 1000) ? 2.0 * ldexp(p, k - 1) : ldexp(p, k);
    if (y < DBL_TINY) y = 0.0;
    return y;
}
__device__ __forceinline__ double sm_exp(double x)
{
    if (isnan(x)) return x;
    if (x > 709.78271289338399679) return __longlong_as_double(0x7ff0000000000000LL);
    if (x < -745.1332191019412) return 0.0;
    return sm_exp_core(x, 0.0);
}

// ---- position-independent natural logarithm: rdb_sm_log
// (rdb_safe_math_core.inc:139-206): x = m 2^k with m in [sqrt(1/2), sqrt(2))
// (subnormals scaled by 2^54 first), log m = 2 atanh f with f = (m-1)/(m+1)
// and the odd series in f to 1/19 (Cody & Waite 1980, ch. 5), k ln 2 added as
// head + tail.  Bit-identical to the CPU restatement without FMA contraction.
__device__ __forceinline__ double sm_log(double x)
{
    if (isnan(x)) return x;
    if (x < 0.0) return __longlong_as_double(0x7ff8000000000000LL);
    if (x == 0.0) return __longlong_as_double((long long)0xfff0000000000000ULL);
    if (isinf(x)) return x;
    double xs = x;
    int kadj = 0;
    if (x < DBL_TINY) {
        xs = x * 18014398509481984.0;   // 2^54
        kadj = -54;
    }
    int e;
    double m = frexp(xs, &e);   // m in [1/2, 1), exact
    int k = e + kadj;
    if (m < 0.70710678118654757274) {
        m = 2.0 * m;
        k = k - 1;
    }
    const double f = xdiv(m - 1.0, m + 1.0);
    const double u = f * f;
    double p = 1.0 / 19.0;
    p = p * u + 1.0 / 17.0;
    p = p * u + 1.0 / 15.0;
    p = p * u + 1.0 / 13.0;
    p = p * u + 1.0 / 11.0;
    p = p * u + 1.0 / 9.0;
    p = p * u + 1.0 / 7.0;
    p = p * u + 1.0 / 5.0;
    p = p * u + 1.0 / 3.0;
    const double kr = (double)k;
    const double s = kr * 0.69314718060195446014 + 2.0 * f;
    const double w = (2.0 * f) * u * p + kr * -4.2009150726810845979e-11;
    return s + w;
}

// ---- exact sum (Knuth) and exact product without FMA (Dekker, Veltkamp
// split by 2^27 + 1), rdb_safe_math_core.inc:53-79: s + e == a + b,
// p + e == a * b.  The _rn intrinsics keep every operation separately
// rounded whatever the file's contraction setting.
__device__ __forceinline__ void sm_two_sum(double a, double b, double &s, double &e)
{
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void sm_two_prod(double a, double b, double &p, double &e)
{
    double c = __dmul_rn(134217729.0, a);
    const double ah = __dsub_rn(c, __dsub_rn(c, a));
    const double al = __dsub_rn(a, ah);
    c = __dmul_rn(134217729.0, b);
    const double bh = __dsub_rn(c, __dsub_rn(c, b));
    const double bl = __dsub_rn(b, bh);
    p = __dmul_rn(a, b);
    e = __dadd_rn(__dadd_rn(__dadd_rn(__dsub_rn(__dmul_rn(ah, bh), p), __dmul_rn(ah, bl)), __dmul_rn(al, bh)),
                  __dmul_rn(al, bl));
}

// ---- log x as head + tail, rdb_sm_log_dd (rdb_safe_math_core.inc:208-249):
// the quotient f = (m-1)/(m+1) carried to ~106 bits, the series tail in
// plain double; lh + ll is good to ~1e-18 relative.
__device__ __forceinline__ void sm_log_dd(double x, double &lh, double &ll)
{
    double xs = x;
    int kadj = 0;
    if (x < DBL_TINY) {
        xs = x * 18014398509481984.0;   // 2^54
        kadj = -54;
    }
    int e;
    double m = frexp(xs, &e);
    int k = e + kadj;
    if (m < 0.70710678118654757274) {
        m = 2.0 * m;
        k = k - 1;
    }
    const double a = m - 1.0;
    double bh, bl;
    sm_two_sum(m, 1.0, bh, bl);
    const double q1 = xdiv(a, bh);
    double p1, p2;
    sm_two_prod(q1, bh, p1, p2);
    const double rr = ((a - p1) - p2) - q1 * bl;
    const double q2 = xdiv(rr, bh);
    const double fh = q1 + q2;
    const double fl = q2 - (fh - q1);
    const double u = fh * fh;
    double p = 1.0 / 19.0;
    p = p * u + 1.0 / 17.0;
    p = p * u + 1.0 / 15.0;
    p = p * u + 1.0 / 13.0;
    p = p * u + 1.0 / 11.0;
    p = p * u + 1.0 / 9.0;
    p = p * u + 1.0 / 7.0;
    p = p * u + 1.0 / 5.0;
    p = p * u + 1.0 / 3.0;
    const double tail = (2.0 * fh) * u * p;
    const double kr = (double)k;
    double ss, ee;
    sm_two_sum(kr * 0.69314718060195446014, 2.0 * fh, ss, ee);
    lh = ss;
    ll = ee + ((2.0 * fl + tail) + kr * -4.2009150726810845979e-11);
}

// ---- position-independent power: rdb_sm_pow (rdb_safe_math_pow.inc:6-105):
// the C99 pow special values except that a NaN anywhere gives NaN; for finite
// x > 0, exp(y log x) with the log as head + tail and y*log x formed exactly.
__device__ __forceinline__ double sm_pow(double x, double y)
{
    const double NaN = __longlong_as_double(0x7ff8000000000000LL);
    const double Inf = __longlong_as_double(0x7ff0000000000000LL);
    if (isnan(x) || isnan(y)) return NaN;
    if (y == 0.0 || x == 1.0) return 1.0;
    const double ax = fabs(x), ay = fabs(y);
    bool yint = false, yodd = false;
    if (isfinite(y)) {
        if (ay >= 9007199254740992.0) {
            yint = true;
        } else {
            yint = (ay == round(ay));
            const double h = 0.5 * ay;
            yodd = yint && (h != round(h));
        }
    }
    const bool xneg = (x < 0.0) || (x == 0.0 && signbit(x));
    double r;
    if (!isfinite(y)) {
        if (ax == 1.0) return 1.0;
        return ((ax < 1.0) == (y > 0.0)) ? 0.0 : Inf;
    }
    if (ax == 0.0) {
        r = (y > 0.0) ? 0.0 : Inf;
        return (xneg && yodd) ? -r : r;
    }
    if (!isfinite(x)) {
        r = (y > 0.0) ? Inf : 0.0;
        return (xneg && yodd) ? -r : r;
    }
    if (xneg && !yint) return NaN;
    double lh, ll;
    sm_log_dd(ax, lh, ll);
    const double t = y * lh;
    if (t > 800.0) {
        r = Inf;
    } else if (t < -800.0) {
        r = 0.0;
    } else {
        double ph, pl, ee, c2;
        sm_two_prod(y, lh, ph, pl);
        const double c = pl + y * ll;
        sm_two_sum(ph, c, ee, c2);
        if (ee > 709.78271289338399679)
            r = Inf;
        else if (ee < -745.1332191019412)
            r = 0.0;
        else
            r = sm_exp_core(ee, c2);
    }
    return (xneg && yodd) ? -r : r;
}

// ---- position-independent complementary error function: rdb_sm_erfc
// (rdb_safe_math_erfc.inc): a series in x^2 below |x| = 1/2; beyond,
// exp(-x^2) as sm_exp_core(-xh^2, -xl (x + xh)) on a Veltkamp split, times a
// rational fit on [1/2, 2) and [2, 4) or the asymptotic form beyond 4 (the
// reference's fitted tables, rdb_safe_math_consts.inc:99-128).
__device__ __forceinline__ double sm_erfc(double x)
{
    if (isnan(x)) return x;
    const double ax = fabs(x);
    if (ax < 0.5) {
        const double v = x * x;
        double p = -1.095865453884735107e-9;
        p = p * v + 1.472152117638980096e-8;
        p = p * v + -1.636264690374603956e-7;
        p = p * v + 1.64620383639705829e-6;
        p = p * v + -0.00001492564916290355896;
        p = p * v + 0.0001205533296923066544;
        p = p * v + -0.0008548327023363942604;
        p = p * v + 0.005223977625441806293;
        p = p * v + -0.02686617064513124181;
        p = p * v + 0.1128379167095512614;
        p = p * v + -0.376126389031837538;
        p = p * v + 1.128379167095512559;
        return 1.0 - x * p;
    }
    double ex = 0.0;
    if (!(ax > 27.3)) {
        const double c = __dmul_rn(134217729.0, ax);
        const double xh = __dsub_rn(c, __dsub_rn(c, ax));
        const double xl = __dsub_rn(ax, xh);
        ex = sm_exp_core(-(xh * xh), -(xl * (ax + xh)));
    }
    double p, q;
    if (ax < 2.0) {
        p = 4.820036176802313081e-8;
        q = 0.009303534974169982985;
        p = p * ax + 0.005247572786535052193;
        q = q * ax + 0.1013327241858480304;
        p = p * ax + 0.05719027224971907214;
        q = q * ax + 0.5046949490889137691;
        p = p * ax + 0.2819428661917610102;
        q = q * ax + 1.443014856236056964;
        p = p * ax + 0.7867094724888269441;
        q = q * ax + 2.468873583018134976;
        p = p * ax + 1.248626834329117141;
        q = q * ax + 2.377005991883625935;
        p = p * ax + 0.9999999993850857694;
        q = q * ax + 1.0;
        ex = ex * xdiv(p, q);
    } else if (ax < 4.0) {
        p = 1.000103316758091609e-9;
        q = 0.02463786793791475013;
        p = p * ax + 0.01390038004034872994;
        q = q * ax + 0.2013396690397278865;
        p = p * ax + 0.1135948493973390344;
        q = q * ax + 0.8274770365185684096;
        p = p * ax + 0.4598879010194165118;
        q = q * ax + 2.025960043609839722;
        p = p * ax + 1.086387126830294259;
        q = q * ax + 3.045871297831376889;
        p = p * ax + 1.494269944137282868;
        q = q * ax + 2.622591678871410537;
        p = p * ax + 0.9999921569124016196;
        q = q * ax + 1.0;
        ex = ex * xdiv(p, q);
    } else {
        const double rax = 1.0 / ax;
        const double w = rax * rax;
        p = -12.38208675658035851;
        q = 428.3053107970796418;
        p = p * w + -231.8021338423288;
        q = q * w + 1100.222105092567517;
        p = p * w + -273.5933562329464053;
        q = q * w + 802.2984884770494318;
        p = p * w + -95.49719132910308872;
        q = q * w + 226.1241802321382579;
        p = p * w + -12.20993252402114315;
        q = q * w + 25.91986504803799107;
        p = p * w + -0.4999999999999982792;
        q = q * w + 1.0;
        ex = ((ex * 0.56418958354775627928) * rax) * (1.0 + w * xdiv(p, q));
    }
    if (ex < DBL_TINY) ex = 0.0;
    return (x < 0.0) ? 2.0 - ex : ex;
}

// ---- position-independent arctangent: rdb_sm_atan
// (rdb_safe_math_atan.inc:7-44, Cody & Waite reduction, fitted degree-11
// polynomial of rdb_safe_math_consts.inc:85-89).
__device__ __forceinline__ double sm_atan(double x)
{
    if (isnan(x)) return x;
    double ax = fabs(x);
    bool inv = ax > 1.0;
    double t = inv ? 1.0 / ax : ax;
    bool mid = t > 0.2679491924311226958;
    double a = mid ? xdiv(1.7320508075688771932 * t - 1.0, 1.7320508075688771932 + t) : t;
    double u = a * a;
    double p = -0.0295457862073798469;
    p = p * u + 0.04518284953605152671;
    p = p * u + -0.05237747786578652448;
    p = p * u + 0.05880646170199485545;
    p = p * u + -0.06666590357759735741;
    p = p * u + 0.07692305406260263601;
    p = p * u + -0.09090909045700855395;
    p = p * u + 0.1111111111054328693;
    p = p * u + -0.1428571428571007162;
    p = p * u + 0.1999999999999998446;
    p = p * u + -0.3333333333333333148;
    p = p * u + 1.0;
    double y = a * p;
    if (mid) y = 0.52359877559829892668 + (y + -5.3604088322554549242e-17);
    if (inv) y = (1.570796326794896558 - y) + 6.1232339957367660359e-17;
    y = copysign(y, x);
    if (fabs(y) < DBL_TINY) y = copysign(0.0, y);
    return y;
}

__device__ __forceinline__ double ratan(double x) { return sm_atan(x); }
__device__ __forceinline__ float ratan(float x) { return atanf(x); }

// face_thick (rdb_ocean_vdiff.F90:1928-1962)
__device__ __forceinline__ double face_thick(double ha, double hb, bool use_harmonic)
{
    if (use_harmonic) {
        double sum_h = ha + hb;
        if (sum_h > 1.0e-30) return xdiv(2.0 * ha * hb, sum_h);
        return 0.5 * sum_h;
    }
    return 0.5 * (ha + hb);
}
__device__ __forceinline__ float face_thick(float ha, float hb, bool use_harmonic)
{
    if (use_harmonic) {
        const float sum_h = ha + hb;
        if (sum_h > 1.0e-30f) return __fdividef(2.0f * ha * hb, sum_h);
        return 0.5f * sum_h;
    }
    return 0.5f * (ha + hb);
}

// rdb_conc_add_source (rdb_tracer_conc.inc:36-53)
__device__ __forceinline__ double conc_add_source(double c, double h, double src)
{
    return (h > H_VANISHED) ? c + xdiv(src, h + H_DIV_EPS) : c;
}
// the same with the quotient from r = rcp_of(h + H_DIV_EPS), made once for
// the tracers a layer deposits into (qdiv(src, r) is src / (h + H_DIV_EPS)
// bit for bit)
__device__ __forceinline__ double conc_add_source_r(double c, double h, double src, const Rcp &r)
{
    return (h > H_VANISHED) ? c + qdiv(src, r) : c;
}

// 1 / b for the mixed-precision solves, which carry no bitwise contract:
// the hardware's approximate FP64 reciprocal refined by two Newton-Raphson
// steps y <- y + y (1 - b y), each of which squares the relative error, so
// the result is within an ulp or two of 1/b (b positive and normal here: a
// layer thickness plus H_DIV_EPS, a boundary-layer depth)
__device__ __forceinline__ double rcp_nr(double b)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    return fma(y, e, y);
}
// conc_add_source of the mixed-precision solves: the quotient as a product
// with r = rcp_nr(h + H_DIV_EPS)
__device__ __forceinline__ double conc_add_source_mp(double c, double h, double src, double r)
{
    return (h > H_VANISHED) ? c + src * r : c;
}

// nonlocal_face_flux (rdb_ocean_vmix.F90:1694-1714)
__device__ __forceinline__ double nonlocal_face_flux(double gamma, double h_below, double h_above)
{
    return (h_below > H_VANISHED && h_above > H_VANISHED) ? gamma : 0.0;
}

// ---- L2 residency hints (PTX createpolicy + cache_hint) ----
// Intermediates that a thread writes and reads back later in the same kernel
// (in-place Thomas sweeps) are stored evict_last so the round trip stays in
// the 126 MB L2; data read once are loaded evict_first.
__device__ __forceinline__ unsigned long long l2_policy_evict_last()
{
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_normal()
{
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_first()
{
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_hint(const double *ptr, unsigned long long pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_hint(double *ptr, double v, unsigned long long pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(ptr), "d"(v), "l"(pol) : "memory");
}

// eos_buoyancy_coeffs, Wright branch (rdb_eos.F90:1716-1733): alpha_T =
// -d(rho)/dT and beta_S = +d(rho)/dS of rho = P/D, P = p + p0(T,S),
// D = lambda(T,S) + alpha0(T,S) P, by the quotient rule, in the reference's
// operation order.
__device__ __forceinline__ void wright_buoyancy_coeffs(double T, double S, double p, double &alpha_T, double &beta_S)
{
    const double T_sq = T * T;
    const double alpha_0 = WRIGHT_A0 + WRIGHT_A1 * T + WRIGHT_A2 * S;
    const double p_0 = WRIGHT_B0 + WRIGHT_B1 * T + WRIGHT_B2 * T_sq + WRIGHT_B3 * T_sq * T + WRIGHT_B4 * S +
                       WRIGHT_B5 * S * T;
    const double lambda = WRIGHT_C0 + WRIGHT_C1 * T + WRIGHT_C2 * T_sq + WRIGHT_C3 * T_sq * T + WRIGHT_C4 * S +
                          WRIGHT_C5 * S * T;
    const double dp0_dt = WRIGHT_B1 + 2.0 * WRIGHT_B2 * T + 3.0 * WRIGHT_B3 * T_sq + WRIGHT_B5 * S;
    const double dlam_dt = WRIGHT_C1 + 2.0 * WRIGHT_C2 * T + 3.0 * WRIGHT_C3 * T_sq + WRIGHT_C5 * S;
    const double dp0_ds = WRIGHT_B4 + WRIGHT_B5 * T;
    const double dlam_ds = WRIGHT_C4 + WRIGHT_C5 * T;
    const double big_p = p + p_0;
    const double denom = lambda + alpha_0 * big_p;
    const double inv_d2 = xdiv(1.0, denom * denom);
    alpha_T = -(dp0_dt * denom - big_p * (dlam_dt + WRIGHT_A1 * big_p + alpha_0 * dp0_dt)) * inv_d2;
    beta_S = (dp0_ds * denom - big_p * (dlam_ds + WRIGHT_A2 * big_p + alpha_0 * dp0_ds)) * inv_d2;
}

// The KPP surface buoyancy flux B0 (kpp_surface_buoyancy_flux,
// rdb_ocean_vmix.F90:1518-1559) with the coefficient pair of
// buoyancy_coeffs (1357-1376): the constants, or with "eos" the Wright
// derivatives at the first live layer's (T_sfc, S_sfc) and p_ref when that
// layer is live (h_sfc > H_VANISHED).
__device__ __forceinline__ double kpp_surface_b0(const vphys_config &c, double q_T_kin, double q_S_kin, double h_sfc,
                                                 double T_sfc, double S_sfc)
{
    double a = c.alpha_T, b = c.beta_S;
    if (c.buoyancy_coeffs && h_sfc > H_VANISHED) wright_buoyancy_coeffs(T_sfc, S_sfc, c.eos_p_ref, a, b);
    return (GRAVITY / c.rho0) * (a * q_T_kin - b * q_S_kin);
}

// sw_transmission (rdb_ocean_surface_flux.F90:1401-1415): the two-band
// normalised downward irradiance at depth d.
__device__ __forceinline__ double sw_transmission(const vphys_config &c, double d)
{
    return c.sw_band_ratio * sm_exp(xdiv(-d, c.sw_zeta1)) + (1.0 - c.sw_band_ratio) * sm_exp(xdiv(-d, c.sw_zeta2));
}

// The kinematic heat flux KPP's B0 charges (rdb_ocean_vmix.F90:1321-1348 in
// pass 1 with the lagged h_b, 1440-1466 in pass 2 with the new one): with
// shortwave penetration on, Q_heat minus the penetrating part that passes the
// boundary layer (MXL) or the surface layer h_sfc (LV1), the part of
// sw_pen_frac times the shortwave source *sw (Q_heat, or SW_NET under
// sw_source = 1; read only with penetration on).
// (the exponentials out of line, with scalar arguments, so the kernels that
// call this keep their registers when shortwave penetration is off)
static __device__ __noinline__ double sw_q_bl(double q_heat, const double *sw, double d, double pen, double R,
                                               double zeta1, double zeta2)
{
    return q_heat - pen * *sw * (R * sm_exp(xdiv(-d, zeta1)) + (1.0 - R) * sm_exp(xdiv(-d, zeta2)));
}
// The chlorophyll scheme's share of the shortwave in band n (1-based) of nb
// (sw_band_fractions, rdb_ocean_surface_flux.F90:767-782): the visible 0.42
// split blue / red, the near infrared shared evenly by bands 3..nb.
constexpr double SW_VIS_FRAC = 0.42;
__device__ __forceinline__ double sw_band_frac(int n, int nb, double blue)
{
    if (n == 1) return blue * SW_VIS_FRAC;
    if (n == 2) return (1.0 - blue) * SW_VIS_FRAC;
    return xdiv(1.0 - SW_VIS_FRAC, (double)(nb - 2));
}
// sw_transmission_nb (:795-812): sum_n frac_n exp(-kappa_n d), kappa_n at
// kap[col + (n-1) plane] (kap is the opacity field's base: the column offset is
// applied here, so a null field is never offset)
static __device__ __noinline__ double sw_transmission_nb(double d, const double *kap, size_t col, size_t plane, int nb,
                                                         double blue)
{
    double trans = 0.0;
    for (int n = 1; n <= nb; ++n) trans = trans + sw_band_frac(n, nb, blue) * sm_exp(-(kap[col + (size_t)(n - 1) * plane] * d));
    return trans;
}
__device__ __forceinline__ double kpp_q_t_kin(const vphys_config &c, double q_heat, const double *sw, const double *kap,
                                              size_t col, size_t plane, double h_b, double h_sfc)
{
    if (c.sw_pen_frac != 0.0 && c.kpp_sw_method != VPHYS_KPP_SW_ALL) {
        const double d = (c.kpp_sw_method == VPHYS_KPP_SW_MXL) ? h_b : h_sfc;
        if (c.sw_chl)
            return xdiv(q_heat - c.sw_pen_frac * *sw * sw_transmission_nb(d, kap, col, plane, c.sw_nbands, c.sw_blue_frac),
                        c.rho0 * c.cp);
        return xdiv(sw_q_bl(q_heat, sw, d, c.sw_pen_frac, c.sw_band_ratio, c.sw_zeta1, c.sw_zeta2), c.rho0 * c.cp);
    }
    return xdiv(q_heat, c.rho0 * c.cp);
}

// The tracer-solve knobs of the default (benchmark) configuration: no
// budgets, arithmetic face thickness, constant buoyancy coefficients, no
// shortwave; a solve instantiated for them folds the other branches out.
__host__ __device__ __forceinline__ bool is_default_tracer_knobs(const vphys_config &c)
{
    return !c.budgets && !c.use_harmonic && !c.buoyancy_coeffs && c.sw_pen_frac == 0.0 && !c.column_integrals;
}
__device__ __forceinline__ void default_tracer_knobs(vphys_config &c)
{
    c.budgets = 0;
    c.use_harmonic = 0;
    c.buoyancy_coeffs = 0;
    c.sw_pen_frac = 0.0;
    c.column_integrals = 0;
}

// Neumaier's improvement of Kahan summation (Z. Angew. Math. Mech. 54, 1974):
// the rounding error of every addition is carried in cmp, whichever of the
// two operands is larger (the column-content diagnostic; the oracle's
// neumaier_add, operation for operation).
__device__ __forceinline__ void neumaier_add(double &sum, double &cmp, double x)
{
    const double t = sum + x;
    if (fabs(sum) >= fabs(x))
        cmp += (sum - t) + x;
    else
        cmp += (x - t) + sum;
    sum = t;
}

}  // namespace vphys
