// vphys_faces.cuh -- velocity-face thickness and interface coupling of the
// momentum solve, templated on the arithmetic type (double: the exact path,
// float: the mixed-precision path).
#pragma once

#include "vphys_device.cuh"
#include "../../include/vphys.h"

namespace vphys {

// The momentum knobs of the default (benchmark) configuration; a face solve
// instantiated for them folds the other options' branches out.
__host__ __device__ __forceinline__ bool is_default_face_knobs(const vphys_config &c)
{
    return c.hvel_mom6 && !c.hvel_harmonic && !c.remnant && !c.bbl_glue && !c.implicit_stress &&
           !c.implicit_drag && !c.zlevel_faces;
}
__host__ __device__ __forceinline__ void default_face_knobs(vphys_config &c)
{
    c.hvel_mom6 = 1;
    c.hvel_harmonic = 0;
    c.remnant = 0;
    c.bbl_glue = 0;
    c.implicit_stress = 0;
    c.implicit_drag = 0;
    c.zlevel_faces = 0;
}

template <typename R>
__device__ __forceinline__ void face_layer(const vphys_config &c, R hl_c, R hr_c, R u_k, int k, int kb, R d_min,
                                           R i_hbbl, R &zacc, R &zcol_l, R &zcol_r, R &hvel, R &zint)
{
    // vdiff_face_layer (rdb_ocean_vdiff.F90:1964-2056)
    zint = 0;
    if (c.hvel_mom6 && !c.hvel_harmonic) {
        const R h_harm = rdiv(R(2.0) * hl_c * hr_c, hl_c + hr_c + R(EPS_HVEL));
        const R h_arith = R(0.5) * (hl_c + hr_c);
        const R h_delta = hr_c - hl_c;
        zcol_l = zcol_l + hl_c;
        zcol_r = zcol_r + hr_c;
        if (k >= kb) zacc = zacc + h_harm;
        const R z_clear = fmx(zcol_l, zcol_r) + d_min;
        zint = fmx(zacc, z_clear) * i_hbbl;
        hvel = h_arith;
        if (u_k * h_delta > R(0)) {
            const R z2 = zint;
            const R botfn = rdiv(R(1.0), R(1.0) + R(0.09) * z2 * z2 * z2 * z2 * z2 * z2);
            hvel = (R(1.0) - botfn) * h_arith + botfn * h_harm;
        }
    } else if (c.hvel_mom6) {
        const R h_harm = rdiv(R(2.0) * hl_c * hr_c, hl_c + hr_c + R(EPS_HVEL));
        const R h_arith = R(0.5) * (hl_c + hr_c);
        const R h_delta = hr_c - hl_c;
        hvel = h_harm;
        if (c.hvel_upwind && u_k * h_delta < R(0)) {
            const R z2 = zacc;
            const R botfn = rdiv(R(1.0), R(1.0) + R(0.09) * z2 * z2 * z2 * z2 * z2 * z2);
            hvel = (R(1.0) - botfn) * h_harm + botfn * h_arith;
        }
        if (k >= kb) zacc = zacc + h_harm * i_hbbl;
        zint = zacc;
    } else {
        hvel = R(0.5) * (hl_c + hr_c);
    }
    if (c.zlevel_faces) hvel = fmn(hl_c, hr_c);
}

template <typename R>
__device__ __forceinline__ void interface_coupling(const vphys_config &c, R hv_lo, R hv_hi, R zint_lo, R dt, R kv_bbl,
                                                   R bbl_thick, R kv_l, R kv_r, R &num, R &dz, bool &cut)
{
    // vdiff_interface_coupling (rdb_ocean_vdiff.F90:2058-2115)
    const R HV = (R)H_VANISHED;
    const R hf_lo = fmx(hv_lo, HV);
    const R hf_hi = fmx(hv_hi, HV);
    if (c.hvel_mom6)
        dz = R(0.5) * (hf_lo + hf_hi);
    else
        dz = face_thick(hf_lo, hf_hi, c.use_harmonic);
    R nu_f = R(0.5) * (kv_l + kv_r);
    if (c.bbl_glue) {
        const R z = zint_lo;
        const R botfn_int = rdiv(R(1.0), R(1.0) + R(0.09) * z * z * z * z * z * z);
        nu_f = fmx(R(0), nu_f + (kv_bbl - (R)c.kv_bbl_bg) * botfn_int);
        if (dz > bbl_thick) dz = (R(1.0) - botfn_int) * dz + botfn_int * bbl_thick;
    }
    num = dt * nu_f;
    cut = c.zlevel_faces && (hv_lo <= HV || hv_hi <= HV);
}

}  // namespace vphys
