// vphys_device.cuh -- device-side building blocks of the vertical-physics
// kernels: constants, the position-independent cbrt/atan, and the per-level
// pieces of the momentum face column.  Every routine follows the operation
// order of the Fortran it cites, and the kernels are compiled without FMA
// contraction (-fmad=false), so a column's result is bit-identical to the CPU
// restatement built with -ffp-contract=off.
#pragma once

#include <cstdint>

namespace vphys {

constexpr double GRAVITY = 9.80665;        // rdb_constants.F90:37
constexpr double H_VANISHED = 1.5e-4;      // rdb_constants.F90:67
constexpr double H_DIV_EPS = 1.0e-20;      // rdb_constants.F90:85
constexpr double PI_D = 3.141592653589793115997963468544185161590576171875;  // 4*atan(1)
constexpr double EPS_HVEL = 1.0e-30;       // rdb_ocean_vdiff.F90 diffuse_velocity_columns_impl
constexpr double STRESS_H_MIN = 1.0e-3;
constexpr double DBL_TINY = 2.2250738585072014e-308;

// Fortran MAX/MIN (finite operands); the same ternary as the CPU restatement.
__device__ __forceinline__ double fmx(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double fmn(double a, double b) { return a < b ? a : b; }

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
        y0 = y0 + y0 * ((m - y3) / ((y3 + y3) + m));
    }
    double y = ldexp(y0, q);
    return x < 0.0 ? -y : y;
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
    double a = mid ? (1.7320508075688771932 * t - 1.0) / (1.7320508075688771932 + t) : t;
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

// face_thick (rdb_ocean_vdiff.F90:1928-1962)
__device__ __forceinline__ double face_thick(double ha, double hb, bool use_harmonic)
{
    if (use_harmonic) {
        double sum_h = ha + hb;
        if (sum_h > 1.0e-30) return 2.0 * ha * hb / sum_h;
        return 0.5 * sum_h;
    }
    return 0.5 * (ha + hb);
}

// rdb_conc_add_source (rdb_tracer_conc.inc:36-53)
__device__ __forceinline__ double conc_add_source(double c, double h, double src)
{
    return (h > H_VANISHED) ? c + src / (h + H_DIV_EPS) : c;
}

// nonlocal_face_flux (rdb_ocean_vmix.F90:1694-1714)
__device__ __forceinline__ double nonlocal_face_flux(double gamma, double h_below, double h_above)
{
    return (h_below > H_VANISHED && h_above > H_VANISHED) ? gamma : 0.0;
}

}  // namespace vphys
