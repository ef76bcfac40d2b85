// vphys_api.cu -- host runtime and C ABI of libvphys (include/vphys.h).
//
// A handle owns the grid shape, the configuration, a CUDA stream and one
// device buffer per field.  Core fields are allocated in HBM at create;
// optional ones (remnant, budgets, gamma diagnostics, drag rates, k_top/k_bot
// overrides, smoothing scratch) the first time a stage or the caller needs
// them.  Any field can instead be bound to a caller-owned device array.
// Stage entry points enqueue kernels on the handle's stream and return.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vphys.h"
#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

using vphys::Params;

namespace {

// ---------------------------------------------------------------------------
// error ring (rdb_ocean_last_error contract, include/rdb_ocean.h:305-314)
// ---------------------------------------------------------------------------
std::mutex g_err_mu;
std::deque<std::string> g_err;
constexpr size_t ERR_RING = 32;

int push_error(int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err.emplace_front(buf);
    while (g_err.size() > ERR_RING) g_err.pop_back();
    return status;
}

int cuda_status(cudaError_t e, const char *where)
{
    if (e == cudaSuccess) return VPHYS_OK;
    return push_error(VPHYS_ERR_CUDA, "%s: CUDA error %d (%s)", where, (int)e, cudaGetErrorString(e));
}

constexpr int NFIXED = 48;
constexpr unsigned MAGIC = 0x56504859u;   // "VPHY"

struct Field {
    void *own = nullptr;     // handle-owned device buffer
    void *bound = nullptr;   // caller-owned device buffer
    size_t n = 0;            // elements
    bool is_int = false;
    void *ptr() const { return bound ? bound : own; }
    size_t bytes() const { return n * (is_int ? sizeof(int) : sizeof(double)); }
};

}  // namespace

struct vphys_handle_s {
    unsigned magic = MAGIC;
    int nx = 0, ny = 0, nz = 0, ntr = 0;
    vphys_config cfg{};
    cudaStream_t stream = nullptr;
    int gen = 0;
    std::vector<Field> f;             // NFIXED fixed fields, then ntr tracers
    unsigned long long *guard_dev = nullptr;
    double *smooth_scratch = nullptr;
    double *budget_scratch = nullptr;
    int *span = nullptr;              // live spans of the columns (mixed-precision tracer solve)
    unsigned *mp_redo = nullptr;      // the mixed tracer solve's FP64 re-solve list (count + entries)
    unsigned *work_ctr = nullptr;     // the work counter of the dynamically scheduled mixed tracer solve
    // kernel variants of the mixed solves (vphys_autotune); the defaults are
    // the faster ones on 1440x1080x75 with 4 tracers
    int var_mom = vphys::VAR_MOM_REGISTER;
    int var_tr = vphys::VAR_TR_SMEM1;
    double *zcol = nullptr;           // column depths for the momentum face thickness
    unsigned char *mom_tiles = nullptr;   // skip flags of the TMA-staged momentum solve's face tiles
    unsigned *dev_err = nullptr;      // bounded waits of the TMA-staged solves that ran out (0: none)
    // ks is bitwise kt: the assembly gate last wrote both under floors that
    // agree, and the caller has written neither since, so a tracer solve may
    // factorise once.  While a pointer to either has been handed out or a
    // buffer is bound to either, a standalone tracer solve never assumes it.
    bool ks_is_kt = false;
    bool k_ptr_given = false;
    // learned KPP surrogate (vphys_kpp_attach): the caller's weights and the scratch of one inference
    vphys_kpp_model kpp{};
    bool kpp_attached = false;
    void *kX = nullptr;
    float *kY = nullptr, *kcolH = nullptr, *kpred = nullptr, *kcheck = nullptr;
    unsigned char *kgate = nullptr;
    unsigned long long *kstats = nullptr;
    int *kerr = nullptr;
    unsigned kgen = 0;
    // vphys_step_graph: the captured launches of n steps and what they were captured with
    cudaStream_t cap_stream = nullptr;
    cudaStream_t aux_stream = nullptr;   // the momentum solve, forked from `stream` after the assembly
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int *ks_work = nullptr;            // kappa-shear: each column's cost in the last solve
    int *ks_order = nullptr;           // kappa-shear: the solve order built from ks_work
    unsigned *ks_hist = nullptr;       // kappa-shear: cost-bucket counts / offsets (1024)
    unsigned char gsig[sizeof(Params) + sizeof(vphys_kpp_model) + 32] = {};
};

namespace {

bool valid(vphys_handle h) { return h != nullptr && h->magic == MAGIC; }

bool is_k_field(int field) { return field == VPHYS_FIELD_KT || field == VPHYS_FIELD_KS; }

// A tracer solve run on its own factorises once only when ks is the gate's
// copy of kt; coefficients a caller wrote or can write get two
// factorisations (kt for temperature, ks for the rest).
void standalone_k(vphys_handle h, Params &p)
{
    if (!h->ks_is_kt || h->k_ptr_given || h->f[VPHYS_FIELD_KT].bound || h->f[VPHYS_FIELD_KS].bound)
        p.ks_equals_kt = 0;
}

// After the gate has written kt and ks: ks is bitwise kt where the floors agree.
void gate_wrote_k(vphys_handle h) { h->ks_is_kt = h->cfg.bkgnd_profile || h->cfg.kt_bg == h->cfg.ks_bg; }

int slot_of(const vphys_handle_s *h, int field)
{
    if (field >= 0 && field < NFIXED) return field;
    if (field >= VPHYS_FIELD_TRACER0 && field < VPHYS_FIELD_TRACER0 + h->ntr) return NFIXED + (field - VPHYS_FIELD_TRACER0);
    return -1;
}

size_t field_count(int nx, int ny, int nz, int field, bool *is_int)
{
    const size_t X = nx, Y = ny, Z = nz;
    *is_int = false;
    if (field >= VPHYS_FIELD_TRACER0) return X * Y * Z;
    switch (field) {
    case VPHYS_FIELD_H:
    case VPHYS_FIELD_RHO:
    case VPHYS_FIELD_HEAT_BUDGET:
    case VPHYS_FIELD_SALT_BUDGET:
    case VPHYS_FIELD_HEAT_BUDGET_SURFACE:
    case VPHYS_FIELD_SALT_BUDGET_SURFACE: return X * Y * Z;
    case VPHYS_FIELD_U:
    case VPHYS_FIELD_VISC_REM_U: return (X + 1) * Y * Z;
    case VPHYS_FIELD_V:
    case VPHYS_FIELD_VISC_REM_V: return X * (Y + 1) * Z;
    case VPHYS_FIELD_KV:
    case VPHYS_FIELD_KT:
    case VPHYS_FIELD_KS:
    case VPHYS_FIELD_GAMMA_T:
    case VPHYS_FIELD_GAMMA_S:
    case VPHYS_FIELD_KD_SHEAR:
    case VPHYS_FIELD_TKE_SHEAR:
    case VPHYS_FIELD_KD_EPBL: return X * Y * (Z + 1);
    case VPHYS_FIELD_SW_KAPPA: return X * Y * VPHYS_SW_NB_MAX;
    case VPHYS_FIELD_CONTENT_OLD:
    case VPHYS_FIELD_CONTENT_NEW: return X * Y;   // times the tracer count: set by vphys_create
    case VPHYS_FIELD_BL_DEPTH:
    case VPHYS_FIELD_B0:
    case VPHYS_FIELD_STRESS_MAG:
    case VPHYS_FIELD_Q_HEAT:
    case VPHYS_FIELD_Q_SALT:
    case VPHYS_FIELD_WET:
    case VPHYS_FIELD_CORIOLIS:
    case VPHYS_FIELD_SW_NET:
    case VPHYS_FIELD_WET_DYN:
    case VPHYS_FIELD_SW_CHL:
    case VPHYS_FIELD_COVER_FRAC:
    case VPHYS_FIELD_MLD_EPBL:
    case VPHYS_FIELD_LA_EPBL:
    case VPHYS_FIELD_EPBL_TKE_WIND:
    case VPHYS_FIELD_EPBL_TKE_CONV:
    case VPHYS_FIELD_EPBL_TKE_FORCING:
    case VPHYS_FIELD_EPBL_TKE_MIXING:
    case VPHYS_FIELD_EPBL_TKE_MECH_DECAY:
    case VPHYS_FIELD_EPBL_TKE_CONV_DECAY: return X * Y;
    case VPHYS_FIELD_TAU_X:
    case VPHYS_FIELD_LAMBDA_BOT_U: return (X + 1) * Y;
    case VPHYS_FIELD_TAU_Y:
    case VPHYS_FIELD_LAMBDA_BOT_V: return X * (Y + 1);
    case VPHYS_FIELD_K_TOP_U:
    case VPHYS_FIELD_K_BOT_U: *is_int = true; return (X + 1) * Y;
    case VPHYS_FIELD_K_TOP_V:
    case VPHYS_FIELD_K_BOT_V: *is_int = true; return X * (Y + 1);
    default: return 0;
    }
}

// ---- fills used at allocation ------------------------------------------
__global__ void k_fill_double(double *p, size_t n, double v)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_fill_int(int *p, size_t n, int v)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
// interface seed: interior value, 0 on the bed (k=1) and surface (k=nz+1)
__global__ void k_fill_interfaces(double *p, size_t plane, int nz, double interior)
{
    const size_t n = plane * (size_t)(nz + 1);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t k = i / plane;
        p[i] = (k == 0 || k == (size_t)nz) ? 0.0 : interior;
    }
}

int fill_blocks(size_t n)
{
    size_t b = (n + 255) / 256;
    return (int)(b < 4096 ? (b ? b : 1) : 4096);
}

// Initial contents of a freshly allocated field (vmix_seed_backgrounds,
// rdb_ocean_vmix.F90:843-913, and ocean_multilayer_state init defaults).
int init_field(vphys_handle h, int field, Field &fl)
{
    const size_t plane = (size_t)h->nx * h->ny;
    cudaStream_t s = h->stream;
    switch (field) {
    case VPHYS_FIELD_WET:
    case VPHYS_FIELD_WET_DYN:
    case VPHYS_FIELD_SW_KAPPA: k_fill_double<<<fill_blocks(fl.n), 256, 0, s>>>((double *)fl.own, fl.n, 1.0); break;
    case VPHYS_FIELD_SW_CHL: k_fill_double<<<fill_blocks(fl.n), 256, 0, s>>>((double *)fl.own, fl.n, 1.0e-4); break;
    case VPHYS_FIELD_KV: k_fill_interfaces<<<fill_blocks(fl.n), 256, 0, s>>>((double *)fl.own, plane, h->nz, h->cfg.pp81_nu_bg); break;
    case VPHYS_FIELD_KT:
    case VPHYS_FIELD_KS: k_fill_interfaces<<<fill_blocks(fl.n), 256, 0, s>>>((double *)fl.own, plane, h->nz, h->cfg.pp81_kappa_bg); break;
    case VPHYS_FIELD_K_TOP_U:
    case VPHYS_FIELD_K_TOP_V: k_fill_int<<<fill_blocks(fl.n), 256, 0, s>>>((int *)fl.own, fl.n, h->nz); break;
    case VPHYS_FIELD_K_BOT_U:
    case VPHYS_FIELD_K_BOT_V: k_fill_int<<<fill_blocks(fl.n), 256, 0, s>>>((int *)fl.own, fl.n, 1); break;
    default: {
        cudaError_t e = cudaMemsetAsync(fl.own, 0, fl.bytes(), s);
        if (e != cudaSuccess) return cuda_status(e, "init_field");
    }
    }
    return cuda_status(cudaGetLastError(), "init_field");
}

int ensure(vphys_handle h, int field)
{
    int sl = slot_of(h, field);
    if (sl < 0) return push_error(VPHYS_ERR_NOT_FOUND, "unknown field id %d", field);
    Field &fl = h->f[sl];
    if (fl.ptr()) return VPHYS_OK;
    cudaError_t e = cudaMalloc(&fl.own, fl.bytes());
    if (e != cudaSuccess) {
        fl.own = nullptr;
        cudaGetLastError();
        return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of %zu bytes for field %d failed (%s)", fl.bytes(), field,
                          cudaGetErrorString(e));
    }
    return init_field(h, field, fl);
}

bool present(vphys_handle h, int field) { return h->f[slot_of(h, field)].ptr() != nullptr; }

// The forcing fields a configuration reads: SW_NET under sw_source = 1,
// WET_DYN under use_wet_dyn.  Held from create / set_config on (and
// restored by an unbind), so every launch finds them.
int prepare_sources(vphys_handle h)
{
    int st = VPHYS_OK;
    if (h->cfg.sw_source && (st = ensure(h, VPHYS_FIELD_SW_NET))) return st;
    if (h->cfg.use_wet_dyn && (st = ensure(h, VPHYS_FIELD_WET_DYN))) return st;
    if (h->cfg.sw_chl && (st = ensure(h, VPHYS_FIELD_SW_CHL))) return st;
    if (h->cfg.sw_chl && (st = ensure(h, VPHYS_FIELD_SW_KAPPA))) return st;
    if (h->cfg.use_cover_frac && (st = ensure(h, VPHYS_FIELD_COVER_FRAC))) return st;
    return st;
}

// What the handle stores after validation: the chlorophyll scheme absorbs the
// whole shortwave, so an unset penetrating fraction (0) becomes 1
// (set_sw_chl, rdb_ocean_sw_chl.F90:87-103).
static void normalize_config(vphys_config &c)
{
    if (c.sw_chl && c.sw_pen_frac == 0.0) c.sw_pen_frac = 1.0;
}

int validate(const vphys_config *c, int ntr)
{
    if (!c->use_closure)
        return push_error(VPHYS_ERR_CONFIG, "use_closure = 0 selects the scalar K_v_* vdiff path, which is not "
                                            "part of this library (vmix closure path only)");
    if (c->interior_closure != VPHYS_INTERIOR_PP81 && c->interior_closure != VPHYS_INTERIOR_NONE)
        return push_error(VPHYS_ERR_CONFIG, "interior_closure %d has no kernel (only PP81=1 and NONE=4)",
                          c->interior_closure);
    if (c->idx_temperature >= ntr || c->idx_salinity >= ntr || c->idx_pseudo_salt >= ntr)
        return push_error(VPHYS_ERR_CONFIG, "tracer role index beyond ntracer=%d", ntr);
    if (c->idx_pseudo_salt >= 0 && (c->idx_pseudo_salt == c->idx_salinity || c->idx_pseudo_salt == c->idx_temperature))
        return push_error(VPHYS_ERR_CONFIG, "pseudo-salt must be a tracer of its own");
    if (c->idx_temperature >= 0 && c->idx_temperature == c->idx_salinity)
        return push_error(VPHYS_ERR_CONFIG, "temperature and salinity must be different tracers");
    if (c->kd_smooth_iterations < 0) return push_error(VPHYS_ERR_CONFIG, "kd_smooth_iterations < 0");
    if (c->mixed_precision < 0 || c->mixed_precision > 2)
        return push_error(VPHYS_ERR_CONFIG, "mixed_precision %d: 0 (FP64), 1 (mixed solves) or 2 (mixed solves and assembly)",
                          c->mixed_precision);
    if (c->surface_flux < 0 || c->surface_flux > 1) return push_error(VPHYS_ERR_CONFIG, "surface_flux must be 0 or 1");
    if (c->sw_pen_frac != 0.0) {
        if (c->kpp_sw_method < VPHYS_KPP_SW_ALL || c->kpp_sw_method > VPHYS_KPP_SW_LV1)
            return push_error(VPHYS_ERR_CONFIG, "kpp_sw_method must be 1 (all), 2 (mxl) or 3 (lv1)");
        if (!(c->sw_zeta1 > 0.0) || !(c->sw_zeta2 > 0.0))
            return push_error(VPHYS_ERR_CONFIG, "sw_zeta1 and sw_zeta2 must be positive");
    }
    if (c->buoyancy_coeffs < 0 || c->buoyancy_coeffs > 1)
        return push_error(VPHYS_ERR_CONFIG, "buoyancy_coeffs must be 0 (constant) or 1 (eos)");
    if (c->buoyancy_coeffs && c->use_kpp && (c->idx_temperature < 0 || c->idx_salinity < 0))
        return push_error(VPHYS_ERR_CONFIG, "buoyancy_coeffs = eos needs temperature and salinity tracers");
    if (c->rho0 <= 0.0 || c->cp <= 0.0) return push_error(VPHYS_ERR_CONFIG, "rho0 and cp must be positive");
    if (c->use_kpp && c->ri_crit <= 0.0) return push_error(VPHYS_ERR_CONFIG, "ri_crit must be positive");
    if (c->bkgnd_profile && c->bkgnd_delta == 0.0) return push_error(VPHYS_ERR_CONFIG, "bkgnd_delta must be nonzero");
    if (c->bkgnd_prandtl == 0.0)
        return push_error(VPHYS_ERR_CONFIG, "bkgnd_prandtl = 0 is refused (use -1 for off), as the reference does");
    if (c->kappa_shear < 0 || c->kappa_shear > 1) return push_error(VPHYS_ERR_CONFIG, "kappa_shear must be 0 or 1");
    if (c->ks_massless_merge < 0 || c->ks_massless_merge > 1)
        return push_error(VPHYS_ERR_CONFIG, "ks_massless_merge must be 0 or 1");
    if (c->sw_source < 0 || c->sw_source > 1)
        return push_error(VPHYS_ERR_CONFIG, "sw_source must be 0 (net_heat) or 1 (q_sw)");
    if (c->bound_salinity < 0 || c->bound_salinity > 1)
        return push_error(VPHYS_ERR_CONFIG, "bound_salinity must be 0 or 1");
    if (c->use_wet_dyn < 0 || c->use_wet_dyn > 1) return push_error(VPHYS_ERR_CONFIG, "use_wet_dyn must be 0 or 1");
    if (c->epbl_sw_ctke < 0 || c->epbl_sw_ctke > 1) return push_error(VPHYS_ERR_CONFIG, "epbl_sw_ctke must be 0 or 1");
    if (c->sw_chl < 0 || c->sw_chl > 1) return push_error(VPHYS_ERR_CONFIG, "sw_chl must be 0 or 1");
    if (c->use_cover_frac < 0 || c->use_cover_frac > 1)
        return push_error(VPHYS_ERR_CONFIG, "use_cover_frac must be 0 or 1");
    if (c->column_integrals < 0 || c->column_integrals > 1)
        return push_error(VPHYS_ERR_CONFIG, "column_integrals must be 0 or 1");
    if (c->sw_chl) {
        // rdb_config_validate.F90:291-310, rdb_ocean_sw_chl.F90:87-103
        // 0 means "unset" there and is raised to 1 when the handle stores the
        // configuration (normalize_config); any other value is refused
        if (c->sw_pen_frac != 1.0 && c->sw_pen_frac != 0.0)
            return push_error(VPHYS_ERR_CONFIG, "sw_chl band-absorbs the whole shortwave: sw_pen_frac must be 1 (or 0, "
                                                "which selects 1)");
        if (c->sw_nbands < 3 || c->sw_nbands > VPHYS_SW_NB_MAX)
            return push_error(VPHYS_ERR_CONFIG, "sw_nbands must be in [3, %d]", VPHYS_SW_NB_MAX);
        for (int n = 0; n < c->sw_nbands; ++n)
            if (!(c->sw_opacity_coef[2 * n] > 0.0))
                return push_error(VPHYS_ERR_CONFIG, "sw_opacity_coef: band %d needs a positive clear-water opacity",
                                  n + 1);
    }
    // the inner solve must run at least once (the substep's adaptive-dt bands
    // read its decay lengths); both caps bound the per-column work
    if (c->ks_max_inner_it < 1 || c->ks_max_inner_it > 10000)
        return push_error(VPHYS_ERR_CONFIG, "ks_max_inner_it must be in [1, 10000]");
    if (c->ks_max_substep_it < 0 || c->ks_max_substep_it > 10000)
        return push_error(VPHYS_ERR_CONFIG, "ks_max_substep_it must be in [0, 10000]");
    if (c->eos_variant < 0 || c->eos_variant > 1) return push_error(VPHYS_ERR_CONFIG, "eos_variant must be 0 (Wright) or 1 (linear)");
    if (c->ks_lambda == 0.0 || c->ks_lz_rescale == 0.0 || c->ks_src_max_chg == 0.0)
        return push_error(VPHYS_ERR_CONFIG, "ks_lambda, ks_lz_rescale and ks_src_max_chg must be nonzero");
    if (c->epbl < 0 || c->epbl > 1) return push_error(VPHYS_ERR_CONFIG, "epbl must be 0 or 1");
    if (c->epbl) {
        if (c->epbl_mstar_scheme < 1 || c->epbl_mstar_scheme > 3)
            return push_error(VPHYS_ERR_CONFIG, "epbl_mstar_scheme must be 1 (constant), 2 (OM4) or 3 (RH18)");
        if (c->epbl_vstar_scheme < 1 || c->epbl_vstar_scheme > 2)
            return push_error(VPHYS_ERR_CONFIG, "epbl_vstar_scheme must be 1 (cube root) or 2 (RH18)");
        if (c->epbl_combine < 1 || c->epbl_combine > 3)
            return push_error(VPHYS_ERR_CONFIG, "epbl_combine must be 1 (add), 2 (max) or 3 (max_shear)");
        if (c->learned_kpp) return push_error(VPHYS_ERR_CONFIG, "EPBL replaces KPP: learned_kpp must be 0");
        if (c->epbl_use_lt < 0 || c->epbl_use_lt > 1) return push_error(VPHYS_ERR_CONFIG, "epbl_use_lt must be 0 or 1");
        if (c->epbl_tke_diags < 0 || c->epbl_tke_diags > 1)
            return push_error(VPHYS_ERR_CONFIG, "epbl_tke_diags must be 0 or 1");
        if (c->epbl_use_lt && (c->epbl_lt_scheme < 1 || c->epbl_lt_scheme > 2))
            return push_error(VPHYS_ERR_CONFIG, "epbl_lt_scheme must be 1 (rescale) or 2 (additive)");
        if (c->epbl_mld_max_its < 1 || c->epbl_mld_max_its > 1000)
            return push_error(VPHYS_ERR_CONFIG, "epbl_mld_max_its must be in [1, 1000]");
        if (!(c->epbl_ustar_min > 0.0)) return push_error(VPHYS_ERR_CONFIG, "epbl_ustar_min must be positive");
    }
    return VPHYS_OK;
}

Params make_params(vphys_handle h)
{
    Params p{};
    p.nx = h->nx;
    p.ny = h->ny;
    p.nz = h->nz;
    p.ntr = h->ntr;
    p.plane = (size_t)h->nx * h->ny;
    p.plane_u = (size_t)(h->nx + 1) * h->ny;
    p.plane_v = (size_t)h->nx * (h->ny + 1);
    p.cfg = h->cfg;
    auto D = [&](int fid) { return (double *)h->f[fid].ptr(); };
    auto I = [&](int fid) { return (const int *)h->f[fid].ptr(); };
    p.h = D(VPHYS_FIELD_H);
    p.rho = D(VPHYS_FIELD_RHO);
    p.u = D(VPHYS_FIELD_U);
    p.v = D(VPHYS_FIELD_V);
    p.kv = D(VPHYS_FIELD_KV);
    p.kt = D(VPHYS_FIELD_KT);
    p.ks = D(VPHYS_FIELD_KS);
    p.bl_depth = D(VPHYS_FIELD_BL_DEPTH);
    p.b0 = D(VPHYS_FIELD_B0);
    p.stress_mag = D(VPHYS_FIELD_STRESS_MAG);
    p.q_heat = D(VPHYS_FIELD_Q_HEAT);
    p.q_salt = D(VPHYS_FIELD_Q_SALT);
    p.wet = D(VPHYS_FIELD_WET);
    p.sw_src = h->cfg.sw_source ? D(VPHYS_FIELD_SW_NET) : p.q_heat;
    p.wet_dyn = h->cfg.use_wet_dyn ? D(VPHYS_FIELD_WET_DYN) : nullptr;
    p.sw_kappa = h->cfg.sw_chl ? D(VPHYS_FIELD_SW_KAPPA) : nullptr;
    p.cover_frac = h->cfg.use_cover_frac ? D(VPHYS_FIELD_COVER_FRAC) : nullptr;
    p.content_old = h->cfg.column_integrals ? D(VPHYS_FIELD_CONTENT_OLD) : nullptr;
    p.content_new = h->cfg.column_integrals ? D(VPHYS_FIELD_CONTENT_NEW) : nullptr;
    p.tau_x = D(VPHYS_FIELD_TAU_X);
    p.tau_y = D(VPHYS_FIELD_TAU_Y);
    p.lambda_bot_u = D(VPHYS_FIELD_LAMBDA_BOT_U);
    p.lambda_bot_v = D(VPHYS_FIELD_LAMBDA_BOT_V);
    p.visc_rem_u = D(VPHYS_FIELD_VISC_REM_U);
    p.visc_rem_v = D(VPHYS_FIELD_VISC_REM_V);
    p.gamma_t = D(VPHYS_FIELD_GAMMA_T);
    p.gamma_s = D(VPHYS_FIELD_GAMMA_S);
    p.heat_budget = D(VPHYS_FIELD_HEAT_BUDGET);
    p.salt_budget = D(VPHYS_FIELD_SALT_BUDGET);
    p.heat_budget_surface = D(VPHYS_FIELD_HEAT_BUDGET_SURFACE);
    p.salt_budget_surface = D(VPHYS_FIELD_SALT_BUDGET_SURFACE);
    p.k_top_u = I(VPHYS_FIELD_K_TOP_U);
    p.k_top_v = I(VPHYS_FIELD_K_TOP_V);
    p.k_bot_u = I(VPHYS_FIELD_K_BOT_U);
    p.k_bot_v = I(VPHYS_FIELD_K_BOT_V);
    for (int t = 0; t < h->ntr && t < vphys::NTR_MAX; ++t) p.tr[t] = (double *)h->f[NFIXED + t].ptr();
    p.guard_count = h->guard_dev;
    p.budget_scratch = h->budget_scratch;
    p.span = h->span;
    p.mp_redo = h->mp_redo;
    p.work_ctr = h->work_ctr;
    p.var_mom = h->var_mom;
    p.var_tr = h->var_tr;
    p.zcol = h->zcol;
    p.mom_tile_skip = h->mom_tiles;
    p.dev_err = h->dev_err;
    p.coriolis = D(VPHYS_FIELD_CORIOLIS);
    p.kd_shear = D(VPHYS_FIELD_KD_SHEAR);
    p.tke_shear = D(VPHYS_FIELD_TKE_SHEAR);
    p.kd_epbl = D(VPHYS_FIELD_KD_EPBL);
    p.mld_epbl = D(VPHYS_FIELD_MLD_EPBL);
    p.la_epbl = D(VPHYS_FIELD_LA_EPBL);
    for (int d = 0; d < 6; ++d) p.epbl_tke[d] = h->cfg.epbl_tke_diags ? D(VPHYS_FIELD_EPBL_TKE_WIND + d) : nullptr;
    p.ks_equals_kt = (h->cfg.bkgnd_profile || h->cfg.kt_bg == h->cfg.ks_bg) ? 1 : 0;
    p.write_gamma = (p.gamma_t && p.gamma_s) ? 1 : 0;
    return p;
}

// Stage preconditions: allocate what the configuration needs.
int prepare_momentum(vphys_handle h)
{
    int st = VPHYS_OK;
    if (h->cfg.hvel_mom6 && !h->cfg.hvel_harmonic && !h->zcol) {
        cudaError_t e = cudaMalloc(&h->zcol, (size_t)h->nx * h->ny * sizeof(double));
        if (e != cudaSuccess) {
            h->zcol = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the column depths failed");
        }
    }
    if (h->cfg.hvel_mom6 && !h->cfg.hvel_harmonic && !h->mom_tiles) {
        Params q{};
        q.nx = h->nx;
        q.ny = h->ny;
        cudaError_t e = cudaMalloc(&h->mom_tiles, (size_t)vphys::momentum_tma_tiles(q));
        if (e != cudaSuccess) {
            h->mom_tiles = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the momentum tile flags failed");
        }
    }
    if (h->cfg.remnant) {
        if ((st = ensure(h, VPHYS_FIELD_VISC_REM_U))) return st;
        if ((st = ensure(h, VPHYS_FIELD_VISC_REM_V))) return st;
    }
    if (h->cfg.implicit_drag) {
        if ((st = ensure(h, VPHYS_FIELD_LAMBDA_BOT_U))) return st;
        if ((st = ensure(h, VPHYS_FIELD_LAMBDA_BOT_V))) return st;
    }
    return st;
}

int prepare_tracers(vphys_handle h)
{
    int st = VPHYS_OK;
    if (h->cfg.column_integrals) {
        if ((st = ensure(h, VPHYS_FIELD_CONTENT_OLD))) return st;
        if ((st = ensure(h, VPHYS_FIELD_CONTENT_NEW))) return st;
    }
    if (h->cfg.mixed_precision && !h->span) {
        cudaError_t e = cudaMalloc(&h->span, (size_t)h->nx * h->ny * sizeof(int));
        if (e != cudaSuccess) {
            h->span = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the column spans failed");
        }
    }
    if (h->cfg.mixed_precision && !h->work_ctr) {
        cudaError_t e = cudaMalloc(&h->work_ctr, 4 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(h->work_ctr, 0, 4 * sizeof(unsigned), h->stream);
        if (e != cudaSuccess) {
            if (h->work_ctr) cudaFree(h->work_ctr);
            h->work_ctr = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the work counter failed");
        }
    }
    if (h->cfg.mixed_precision && !h->mp_redo) {
        const size_t n = 1 + (size_t)((h->nx + 31) / 32) * h->ny * (size_t)(h->ntr > 0 ? h->ntr : 1);
        cudaError_t e = cudaMalloc(&h->mp_redo, n * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(h->mp_redo, 0, sizeof(unsigned), h->stream);
        if (e != cudaSuccess) {
            if (h->mp_redo) cudaFree(h->mp_redo);
            h->mp_redo = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the mixed-solve re-solve list failed");
        }
    }
    if (h->cfg.budgets) {
        if ((st = ensure(h, VPHYS_FIELD_HEAT_BUDGET))) return st;
        if ((st = ensure(h, VPHYS_FIELD_SALT_BUDGET))) return st;
        if (!h->budget_scratch) {
            size_t n = 2 * (size_t)h->nx * h->ny * h->nz;
            cudaError_t e = cudaMalloc(&h->budget_scratch, n * sizeof(double));
            if (e != cudaSuccess) {
                h->budget_scratch = nullptr;
                cudaGetLastError();
                return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the budget scratch failed");
            }
        }
    }
    return st;
}

int prepare_surface_flux(vphys_handle h)
{
    int st = VPHYS_OK;
    if (h->cfg.budgets) {
        if ((st = ensure(h, VPHYS_FIELD_HEAT_BUDGET_SURFACE))) return st;
        if ((st = ensure(h, VPHYS_FIELD_SALT_BUDGET_SURFACE))) return st;
    }
    return st;
}

// dt/(rho0 cp) and dt/rho0, the deposit's column-invariant multipliers
// (rdb_ocean_surface_flux.F90:1048-1064), divided on the host in IEEE double
void surface_flux_scales(const vphys_config &c, double dt, double *inv_heat, double *inv_salt)
{
    *inv_heat = dt / (c.rho0 * c.cp);
    *inv_salt = dt / c.rho0;
}

int prepare_kappa_shear(vphys_handle h)
{
    int st = VPHYS_OK;
    if ((st = ensure(h, VPHYS_FIELD_KD_SHEAR))) return st;
    if ((st = ensure(h, VPHYS_FIELD_TKE_SHEAR))) return st;
    if (!h->ks_work) {
        const size_t n = (size_t)h->nx * h->ny;
        cudaError_t e = cudaMalloc(&h->ks_work, n * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&h->ks_order, n * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&h->ks_hist, 1024 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(h->ks_work, 0, n * sizeof(int), h->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaFree(h->ks_work);
            cudaFree(h->ks_order);
            cudaFree(h->ks_hist);
            h->ks_work = h->ks_order = nullptr;
            h->ks_hist = nullptr;
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the kappa-shear scheduling arrays failed");
        }
    }
    return st;
}

void launch_kappa_shear(vphys_handle h, const Params &p, double dt)
{
    vphys::launch_kappa_shear(p, dt, h->ks_work, h->ks_order, h->ks_hist, true, h->stream);
}

int prepare_epbl(vphys_handle h)
{
    int st = VPHYS_OK;
    if ((st = ensure(h, VPHYS_FIELD_KD_EPBL))) return st;
    if ((st = ensure(h, VPHYS_FIELD_LA_EPBL))) return st;
    if (h->cfg.epbl_tke_diags)
        for (int d = 0; d < 6; ++d)
            if ((st = ensure(h, VPHYS_FIELD_EPBL_TKE_WIND + d))) return st;
    return ensure(h, VPHYS_FIELD_MLD_EPBL);
}

int prepare_assemble(vphys_handle h)
{
    if (h->cfg.kappa_shear) {
        int st = prepare_kappa_shear(h);
        if (st) return st;
    }
    if (h->cfg.epbl) {
        int st = prepare_epbl(h);
        if (st) return st;
    }
    if (h->cfg.kd_smooth_iterations > 0 && !h->smooth_scratch) {
        size_t n = (size_t)h->nx * h->ny * (h->nz + 1);
        cudaError_t e = cudaMalloc(&h->smooth_scratch, n * sizeof(double));
        if (e != cudaSuccess) {
            h->smooth_scratch = nullptr;
            cudaGetLastError();
            return push_error(VPHYS_ERR_ALLOC, "cudaMalloc of the smoothing scratch failed");
        }
    }
    return VPHYS_OK;
}

// The learned KPP pre-stage of an assembly: counters, features, the MLP on the
// tensor cores, the gate/check/fallback decision per column.  Afterwards the
// assembly reads p.kpp_pred / p.kpp_check.
int run_learned_kpp(vphys_handle h, Params &p)
{
    if (!h->cfg.learned_kpp || !h->cfg.use_kpp) return VPHYS_OK;
    if (!h->kpp_attached)
        return push_error(VPHYS_ERR_NOT_INITIALISED, "learned_kpp = 1 but no surrogate attached (vphys_kpp_attach)");
    const vphys_kpp_model &m = h->kpp;
    cudaStream_t s = h->stream;
    const int ncols = h->nx * h->ny;
    vphys::launch_kpp_roll(h->kstats, m.fail_fraction, s);
    vphys::launch_kpp_features(p, nullptr, h->kX, nullptr, 0, m.feat_mean, m.feat_istd, m.gate_limit, h->kgate,
                               h->kcolH, s);
    int st;
    // the three layers in one launch, the hidden activations on chip
    if ((st = vphys::mlp3_bf16(h->kX, ncols, m.w1, m.b1, m.w2, m.b2, m.w3, m.b3, h->kY, h->kerr, s))) return st;
    vphys::launch_kpp_apply((size_t)ncols, h->kY, m.target_mean0, m.target_std0, h->kgate, h->kcolH, h->kpred,
                            h->kcheck, h->kstats, h->kgen++, m.check_fraction, s);
    p.kpp_pred = h->kpred;
    p.kpp_check = h->kcheck;
    p.kpp_stats = h->kstats;
    p.kpp_tol = m.check_tolerance;
    return cuda_status(cudaGetLastError(), "learned KPP launch");
}

void free_kpp(vphys_handle h)
{
    void *bufs[] = {h->kX, h->kY, h->kcolH, h->kpred, h->kcheck, h->kgate, h->kstats, h->kerr};
    for (void *b : bufs)
        if (b) cudaFree(b);
    h->kX = nullptr;
    h->kY = h->kcolH = h->kpred = h->kcheck = nullptr;
    h->kgate = nullptr;
    h->kstats = nullptr;
    h->kerr = nullptr;
    h->kpp_attached = false;
}

int run_assemble(vphys_handle h, const Params &p);

// The launches of n whole steps (vmix_apply_in_stage on a thermo step,
// rdb_ocean_dyn.F90:1636-1900): EOS, [surface deposit + shortwave],
// [kappa-shear], [learned KPP], assembly (with the kappa-shear merge), momentum,
// tracers with the non-local tendency.  All asynchronous
// on h->stream.
// The momentum and tracer solves after the assembly touch disjoint data
// (u, v, kv / tracers, kt, ks, b0), so the momentum solve runs on an
// auxiliary stream forked from the handle's stream and joined before the next
// step; one kernel's tail overlaps the other (1440x1080x75: step 11.67 ->
// 11.56 ms FP64, 9.20 -> 9.15 ms mixed).  VPHYS_FORK_SOLVES=0 keeps both on
// the handle's stream.  The stream and events are made before any capture
// (prepare_fork).
bool fork_solves()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VPHYS_FORK_SOLVES");
        on = (e && atoi(e) == 0) ? 0 : 1;
    }
    return on == 1;
}

int prepare_fork(vphys_handle h)
{
    if (!fork_solves() || h->aux_stream) return VPHYS_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&h->aux_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
    return cuda_status(e, "solve fork stream");
}

int launch_steps(vphys_handle h, const Params &p, double dt, int n_steps)
{
    int st;
    const bool fork = h->aux_stream && h->ntr > 0;
    // KPP's non-local tendency; under EPBL KPP does not run and its gamma is 0
    const bool kpp_nonlocal = h->cfg.use_kpp && !h->cfg.epbl;
    double inv_heat, inv_salt;
    surface_flux_scales(h->cfg, dt, &inv_heat, &inv_salt);
    for (int n = 0; n < n_steps; ++n) {
        if (h->cfg.eos_in_step) vphys::launch_eos_wright(p, h->stream);
        if (h->cfg.surface_flux) {
            vphys::launch_surface_flux(p, inv_heat, inv_salt, h->stream);
            if (h->cfg.sw_pen_frac != 0.0 && h->cfg.idx_temperature >= 0)
                vphys::launch_sw_penetration(p, inv_heat, h->stream);
        }
        if (h->cfg.epbl && h->cfg.idx_temperature >= 0 && h->cfg.idx_salinity >= 0) vphys::launch_epbl(p, dt, h->stream);
        if (h->cfg.kappa_shear && h->cfg.idx_temperature >= 0 && h->cfg.idx_salinity >= 0)
            launch_kappa_shear(h, p, dt);
        Params pa = p;
        if ((st = run_learned_kpp(h, pa))) return st;
        if ((st = run_assemble(h, pa))) return st;
        if (fork) {
            cudaEventRecord(h->ev_fork, h->stream);
            cudaStreamWaitEvent(h->aux_stream, h->ev_fork, 0);
            vphys::launch_momentum(p, dt, h->aux_stream);
            vphys::launch_tracers(p, dt, true, kpp_nonlocal, h->stream);
            cudaEventRecord(h->ev_join, h->aux_stream);
            cudaStreamWaitEvent(h->stream, h->ev_join, 0);
        } else {
            vphys::launch_momentum(p, dt, h->stream);
            if (h->ntr > 0) vphys::launch_tracers(p, dt, true, kpp_nonlocal, h->stream);
        }
        h->gen += 1;
    }
    return VPHYS_OK;
}

int run_assemble(vphys_handle h, const Params &p)
{
    vphys::launch_assemble(p, h->stream);
    for (int it = 0; it < h->cfg.kd_smooth_iterations; ++it) {
        vphys::launch_smooth(p, p.kv, h->smooth_scratch, h->stream);
        vphys::launch_smooth(p, p.kt, h->smooth_scratch, h->stream);
        vphys::launch_smooth(p, p.ks, h->smooth_scratch, h->stream);
    }
    return cuda_status(cudaGetLastError(), "vphys_assemble launch");
}

// A bounded wait of a TMA-staged solve that ran out leaves a nonzero code in
// h->dev_err (its results are then not to be trusted); read after a
// synchronisation, reported once and cleared.
int check_dev_err(vphys_handle h)
{
    unsigned code = 0;
    cudaError_t e = cudaMemcpy(&code, h->dev_err, sizeof code, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "device error word");
    if (code == 0) return VPHYS_OK;
    cudaMemset(h->dev_err, 0, sizeof code);
    return push_error(VPHYS_ERR_CUDA, "a bounded wait of a TMA-staged solve ran out (code %u); the last step's "
                                      "results are incomplete", code);
}

int read_guard(vphys_handle h, int *status)
{
    unsigned long long bad = 0;
    cudaError_t e = cudaMemcpyAsync(&bad, h->guard_dev, sizeof bad, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_status(e, "guard readback");
    *status = VPHYS_OK;
    if (bad > 0)
        *status = push_error(VPHYS_ERR_GUARD, "vmix_assemble: %llu negative or NaN diffusivities detected", bad);
    return VPHYS_OK;
}

}  // namespace

int vphys::report_error(int status, const char *msg) { return push_error(status, "%s", msg); }

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *vphys_version(void) { return "vphys 0.1 (sm_100a, FP64)"; }

size_t vphys_config_sizeof(void) { return sizeof(vphys_config); }

int vphys_selftest_division(long long n_pairs, unsigned long long seed, int emin, int erange,
                            unsigned long long *mismatches)
{
    if (!mismatches || n_pairs < 0 || erange < 1 || emin < -1000 || emin + erange > 1000)
        return push_error(VPHYS_ERR_CONFIG, "vphys_selftest_division: bad arguments");
    unsigned long long *bad = nullptr;
    cudaError_t e = cudaMalloc(&bad, sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_status(e, "vphys_selftest_division");
    const long long threads = 148LL * 4 * 256;
    const long long per = (n_pairs + threads - 1) / threads;
    e = cudaMemset(bad, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        vphys::launch_selftest_division(seed, per, emin, erange, bad, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(mismatches, bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(bad);
    return cuda_status(e, "vphys_selftest_division");
}

int vphys_last_error(int idx, char *buf, int cap)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (idx < 0 || (size_t)idx >= g_err.size() || cap <= 0 || buf == nullptr) return 0;
    const std::string &m = g_err[(size_t)idx];
    size_t n = m.size() < (size_t)cap - 1 ? m.size() : (size_t)cap - 1;
    memcpy(buf, m.data(), n);
    buf[n] = '\0';
    return (int)m.size();
}

int vphys_config_default(vphys_config *c)
{
    if (!c) return push_error(VPHYS_ERR_CONFIG, "vphys_config_default: NULL");
    memset(c, 0, sizeof *c);
    c->use_closure = 1;
    c->epbl_sw_ctke = 1;
    // Manizza (2005) three-band defaults (rdb_config.F90:336-360)
    c->sw_nbands = 3;
    c->sw_blue_frac = 0.5;
    const double coef[6] = {0.0232, 0.074, 0.225, 0.037, 2.86, 0.0};
    for (int n = 0; n < 6; ++n) c->sw_opacity_coef[n] = coef[n];
    c->sw_chl_power[0] = 0.674;
    c->sw_chl_power[1] = 0.629;
    c->sw_opacity_land = 10.0;
    c->interior_closure = VPHYS_INTERIOR_PP81;
    c->pp81_nu0 = 1.0e-2;
    c->pp81_nu_bg = 1.0e-4;
    c->pp81_kappa_bg = 1.0e-5;
    c->pp81_alpha = 5.0;
    c->rho0 = 1035.0;
    c->shear2_floor = 1.0e-10;
    c->ri_crit = 0.3;
    c->cs_nonlocal = 6.3;
    c->c_vt2 = 1.8;
    c->kpp_sw_method = VPHYS_KPP_SW_MXL;
    c->sw_band_ratio = 0.58;
    c->sw_zeta1 = 0.35;
    c->sw_zeta2 = 23.0;
    c->alpha_T = 1.7e-4;
    c->beta_S = 7.6e-4;
    c->cp = 3992.0;
    c->hmix_fixed = 20.0;
    c->conv_kd = 1.0;
    c->conv_prandtl = 1.0;
    c->kv_bg = 1.0e-4;
    c->kt_bg = 1.0e-5;
    c->ks_bg = 1.0e-5;
    c->kv_max = 1.7976931348623157e308;
    c->kd_max = 1.7976931348623157e308;
    c->bkgnd_kd_sfc = 1.0e-5;
    c->bkgnd_kd_deep = 1.3e-4;
    c->bkgnd_z0 = 2500.0;
    c->bkgnd_delta = 222.0;
    c->bkgnd_prandtl = -1.0;
    c->hvel_mom6 = 1;
    c->hvel_upwind = 1;
    c->hbbl_visc = 10.0;
    c->bbl_piston = 3.0e-4;
    c->kv_bbl_bg = 1.0e-4;
    c->idx_temperature = 1;
    c->idx_salinity = 0;
    c->idx_pseudo_salt = -1;
    c->ks_max_inner_it = 50;
    c->ks_max_substep_it = 13;
    c->ks_ri_crit = 0.25;
    c->ks_shearmix_rate = 0.089;
    c->ks_fri_curvature = -0.97;
    c->ks_c_n = 0.24;
    c->ks_c_s = 0.14;
    c->ks_lambda = 0.82;
    c->ks_lz_rescale = 1.0;
    c->ks_kappa_0 = 1.0e-7;
    c->ks_kappa_seed = 1.0;
    c->ks_kappa_trunc = 1.0e-9;
    c->ks_tol_err = 0.1;
    c->ks_src_max_chg = 10.0;
    c->ks_prandtl_turb = 1.0;
    c->epbl_mstar_scheme = 2;
    c->epbl_vstar_scheme = 1;
    c->epbl_combine = 1;
    c->epbl_mld_iteration = 1;
    c->epbl_mld_max_its = 20;
    c->epbl_mstar_const = 1.2;
    c->epbl_mstar_cap = -1.0;
    c->epbl_mstar_coef1 = 0.3;
    c->epbl_c_ek = 0.085;
    c->epbl_nstar = 0.2;
    c->epbl_tke_decay = 2.5;
    c->epbl_wstar_ustar_coef = 1.0;
    c->epbl_vstar_scale_fac = 1.0;
    c->epbl_vstar_surf_fac = 1.2;
    c->epbl_von_karman = 0.41;
    c->epbl_ekman_scale_coef = 1.0;
    c->epbl_mixlen_exponent = 2.0;
    c->epbl_translay_scale = 0.1;
    c->epbl_mld_tol = 1.0;
    c->epbl_omega = 7.2921e-05;
    c->epbl_ustar_min = 1e-08;
    c->epbl_prandtl = 1.0;
    c->epbl_rh18_cn1 = 0.275;
    c->epbl_rh18_cn2 = 8.0;
    c->epbl_rh18_cn3 = -5.0;
    c->epbl_rh18_cs1 = 0.2;
    c->epbl_rh18_cs2 = 0.4;
    c->epbl_lt_scheme = 1;
    c->epbl_lt_enhance_coef = 0.447;
    c->epbl_lt_enhance_exp = -1.33;
    c->epbl_lt_max_enhance = 5.0;
    c->epbl_la_frac_hbl = 0.04;
    c->epbl_lt_lac1 = -0.87;
    c->epbl_lt_lac4 = 0.95;
    c->epbl_lt_lac5 = 0.95;
    return VPHYS_OK;
}

int vphys_create(int nx, int ny, int nz, int ntracer, const vphys_config *cfg, vphys_handle *out)
{
    if (!out) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_create: NULL out");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nz < 1) return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_create: bad shape %d x %d x %d", nx, ny, nz);
    if (ny > 65534) return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_create: ny=%d > 65534 (grid y limit)", ny);
    if (nz > VPHYS_NZ_MAX) return push_error(VPHYS_ERR_TOO_DEEP, "vphys_create: nz=%d > VPHYS_NZ_MAX=%d", nz, VPHYS_NZ_MAX);
    if (ntracer < 0 || ntracer > vphys::NTR_MAX)
        return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_create: ntracer=%d outside [0, %d]", ntracer, vphys::NTR_MAX);
    vphys_config c;
    if (cfg)
        c = *cfg;
    else
        vphys_config_default(&c);
    int st = validate(&c, ntracer);
    if (st) return st;
    normalize_config(c);
    vphys_handle h = new vphys_handle_s();
    h->nx = nx;
    h->ny = ny;
    h->nz = nz;
    h->ntr = ntracer;
    h->cfg = c;
    h->f.resize(NFIXED + ntracer);
    for (int id = 0; id < NFIXED; ++id) h->f[id].n = field_count(nx, ny, nz, id, &h->f[id].is_int);
    for (int t = 0; t < ntracer; ++t) h->f[NFIXED + t].n = (size_t)nx * ny * nz;
    h->f[VPHYS_FIELD_CONTENT_OLD].n = h->f[VPHYS_FIELD_CONTENT_NEW].n = (size_t)nx * ny * (ntracer > 0 ? ntracer : 1);
    cudaError_t e = cudaMalloc(&h->guard_dev, sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return push_error(VPHYS_ERR_ALLOC, "vphys_create: cudaMalloc failed (%s)", cudaGetErrorString(e));
    }
    cudaMemset(h->guard_dev, 0, sizeof(unsigned long long));
    e = cudaMalloc(&h->dev_err, sizeof(unsigned));
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(h->guard_dev);
        delete h;
        return push_error(VPHYS_ERR_ALLOC, "vphys_create: cudaMalloc failed (%s)", cudaGetErrorString(e));
    }
    cudaMemset(h->dev_err, 0, sizeof(unsigned));
    const int core[] = {VPHYS_FIELD_H,        VPHYS_FIELD_RHO,        VPHYS_FIELD_U,      VPHYS_FIELD_V,
                        VPHYS_FIELD_KV,       VPHYS_FIELD_KT,         VPHYS_FIELD_KS,     VPHYS_FIELD_BL_DEPTH,
                        VPHYS_FIELD_B0,       VPHYS_FIELD_STRESS_MAG, VPHYS_FIELD_Q_HEAT, VPHYS_FIELD_Q_SALT,
                        VPHYS_FIELD_WET,      VPHYS_FIELD_TAU_X,      VPHYS_FIELD_TAU_Y};
    for (int id : core) {
        if ((st = ensure(h, id))) {
            vphys_destroy(&h);
            return st;
        }
    }
    for (int t = 0; t < ntracer; ++t) {
        if ((st = ensure(h, VPHYS_FIELD_TRACER0 + t))) {
            vphys_destroy(&h);
            return st;
        }
    }
    if ((st = prepare_sources(h))) {
        vphys_destroy(&h);
        return st;
    }
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        st = cuda_status(e, "vphys_create");
        vphys_destroy(&h);
        return st;
    }
    *out = h;
    return VPHYS_OK;
}

int vphys_destroy(vphys_handle *hp)
{
    if (!hp || !*hp) return VPHYS_OK;
    vphys_handle h = *hp;
    *hp = nullptr;
    if (!valid(h)) return VPHYS_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    for (auto &fl : h->f)
        if (fl.own) cudaFree(fl.own);
    if (h->guard_dev) cudaFree(h->guard_dev);
    if (h->smooth_scratch) cudaFree(h->smooth_scratch);
    if (h->budget_scratch) cudaFree(h->budget_scratch);
    if (h->span) cudaFree(h->span);
    if (h->mp_redo) cudaFree(h->mp_redo);
    if (h->work_ctr) cudaFree(h->work_ctr);
    if (h->zcol) cudaFree(h->zcol);
    if (h->mom_tiles) cudaFree(h->mom_tiles);
    if (h->dev_err) cudaFree(h->dev_err);
    if (h->ks_work) cudaFree(h->ks_work);
    if (h->ks_order) cudaFree(h->ks_order);
    if (h->ks_hist) cudaFree(h->ks_hist);
    free_kpp(h);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->aux_stream) cudaStreamDestroy(h->aux_stream);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    h->magic = 0;
    delete h;
    return VPHYS_OK;
}

int vphys_set_config(vphys_handle h, const vphys_config *cfg)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_set_config: bad handle");
    if (!cfg) return push_error(VPHYS_ERR_CONFIG, "vphys_set_config: NULL");
    int st = validate(cfg, h->ntr);
    if (st) return st;
    h->cfg = *cfg;
    normalize_config(h->cfg);
    return prepare_sources(h);
}

int vphys_get_config(vphys_handle h, vphys_config *cfg)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_get_config: bad handle");
    if (!cfg) return push_error(VPHYS_ERR_CONFIG, "vphys_get_config: NULL");
    *cfg = h->cfg;
    return VPHYS_OK;
}

int vphys_set_stream(vphys_handle h, void *stream)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_set_stream: bad handle");
    h->stream = (cudaStream_t)stream;
    return VPHYS_OK;
}

int vphys_bind(vphys_handle h, int field, void *device_ptr)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_bind: bad handle");
    int sl = slot_of(h, field);
    if (sl < 0) return push_error(VPHYS_ERR_NOT_FOUND, "vphys_bind: unknown field id %d", field);
    h->f[sl].bound = device_ptr;
    if (device_ptr && h->f[sl].own) {
        // the caller's array replaces the handle's own buffer: free it (a
        // later unbind allocates a fresh one), so binding every large field
        // does not hold two copies of the state
        cudaFree(h->f[sl].own);
        h->f[sl].own = nullptr;
    }
    if (!device_ptr && !h->f[sl].own) {
        // restore a handle-owned buffer only for core fields / tracers
        if (sl < VPHYS_FIELD_LAMBDA_BOT_U || sl >= NFIXED) return ensure(h, field);
        if (sl == VPHYS_FIELD_SW_NET || sl == VPHYS_FIELD_WET_DYN || sl == VPHYS_FIELD_SW_CHL ||
            sl == VPHYS_FIELD_SW_KAPPA || sl == VPHYS_FIELD_COVER_FRAC)
            return prepare_sources(h);
    }
    return VPHYS_OK;
}

int vphys_set_field(vphys_handle h, int field, const void *host, size_t n)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_set_field: bad handle");
    int sl = slot_of(h, field);
    if (sl < 0) return push_error(VPHYS_ERR_NOT_FOUND, "vphys_set_field: unknown field id %d", field);
    if (n != h->f[sl].n)
        return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_set_field: field %d holds %zu elements, got %zu", field, h->f[sl].n, n);
    if (!host) return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_set_field: NULL host buffer");
    int st = ensure(h, field);
    if (st) return st;
    if (is_k_field(field)) h->ks_is_kt = false;
    cudaError_t e = cudaMemcpyAsync(h->f[sl].ptr(), host, h->f[sl].bytes(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return cuda_status(e, "vphys_set_field");
}

int vphys_get_field(vphys_handle h, int field, void *host, size_t n)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_get_field: bad handle");
    int sl = slot_of(h, field);
    if (sl < 0) return push_error(VPHYS_ERR_NOT_FOUND, "vphys_get_field: unknown field id %d", field);
    if (n != h->f[sl].n)
        return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_get_field: field %d holds %zu elements, got %zu", field, h->f[sl].n, n);
    if (!host) return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_get_field: NULL host buffer");
    int st = ensure(h, field);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(host, h->f[sl].ptr(), h->f[sl].bytes(), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if ((st = cuda_status(e, "vphys_get_field"))) return st;
    return check_dev_err(h);
}

namespace {
// Checks shared by the asynchronous copies; returns the slot or a status < 0.
int copy_slot(vphys_handle h, int field, const void *host, size_t n, const char *who, int *st)
{
    *st = VPHYS_OK;
    if (!valid(h)) {
        *st = push_error(VPHYS_ERR_BAD_HANDLE, "%s: bad handle", who);
        return -1;
    }
    int sl = slot_of(h, field);
    if (sl < 0) {
        *st = push_error(VPHYS_ERR_NOT_FOUND, "%s: unknown field id %d", who, field);
        return -1;
    }
    if (n != h->f[sl].n) {
        *st = push_error(VPHYS_ERR_BAD_SHAPE, "%s: field %d holds %zu elements, got %zu", who, field, h->f[sl].n, n);
        return -1;
    }
    if (!host) {
        *st = push_error(VPHYS_ERR_BAD_SHAPE, "%s: NULL host buffer", who);
        return -1;
    }
    if ((*st = ensure(h, field))) return -1;
    return sl;
}
}  // namespace

int vphys_set_field_async(vphys_handle h, int field, const void *host, size_t n)
{
    int st;
    const int sl = copy_slot(h, field, host, n, "vphys_set_field_async", &st);
    if (sl < 0) return st;
    if (is_k_field(field)) h->ks_is_kt = false;
    return cuda_status(cudaMemcpyAsync(h->f[sl].ptr(), host, h->f[sl].bytes(), cudaMemcpyHostToDevice, h->stream),
                       "vphys_set_field_async");
}

int vphys_get_field_async(vphys_handle h, int field, void *host, size_t n)
{
    int st;
    const int sl = copy_slot(h, field, host, n, "vphys_get_field_async", &st);
    if (sl < 0) return st;
    return cuda_status(cudaMemcpyAsync(host, h->f[sl].ptr(), h->f[sl].bytes(), cudaMemcpyDeviceToHost, h->stream),
                       "vphys_get_field_async");
}

int vphys_get_ptr(vphys_handle h, int field, void **ptr, int *nx, int *ny, int *nz, int *gen)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_get_ptr: bad handle");
    int sl = slot_of(h, field);
    if (sl < 0) return push_error(VPHYS_ERR_NOT_FOUND, "vphys_get_ptr: unknown field id %d", field);
    int st = ensure(h, field);
    if (st) return st;
    if (is_k_field(field)) h->k_ptr_given = true;
    if (ptr) *ptr = h->f[sl].ptr();
    bool is_int;
    size_t n = field_count(h->nx, h->ny, h->nz, field, &is_int);
    int X = h->nx, Y = h->ny, Z = 1;
    if (field == VPHYS_FIELD_CONTENT_OLD || field == VPHYS_FIELD_CONTENT_NEW) n = 0, Z = h->ntr > 0 ? h->ntr : 1;
    if (n == (size_t)(h->nx + 1) * h->ny * h->nz || n == (size_t)(h->nx + 1) * h->ny) X = h->nx + 1;
    if (n == (size_t)h->nx * (h->ny + 1) * h->nz || n == (size_t)h->nx * (h->ny + 1)) Y = h->ny + 1;
    if (n == (size_t)X * Y * h->nz) Z = h->nz;
    if (n == (size_t)X * Y * (h->nz + 1)) Z = h->nz + 1;
    if (nx) *nx = X;
    if (ny) *ny = Y;
    if (nz) *nz = Z;
    if (gen) *gen = h->gen;
    return VPHYS_OK;
}

int vphys_eos_wright(vphys_handle h)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_eos_wright: bad handle");
    if (h->cfg.idx_temperature < 0 || h->cfg.idx_salinity < 0)
        return push_error(VPHYS_ERR_CONFIG, "vphys_eos_wright: needs temperature and salinity tracers");
    Params p = make_params(h);
    vphys::launch_eos_wright(p, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_eos_wright launch");
}

int vphys_surface_flux(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_surface_flux: bad handle");
    int st = prepare_surface_flux(h);
    if (st) return st;
    double inv_heat, inv_salt;
    surface_flux_scales(h->cfg, dt, &inv_heat, &inv_salt);
    Params p = make_params(h);
    vphys::launch_surface_flux(p, inv_heat, inv_salt, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_surface_flux launch");
}

int vphys_sw_penetration(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_sw_penetration: bad handle");
    if (h->cfg.sw_pen_frac == 0.0 || h->cfg.idx_temperature < 0) return VPHYS_OK;
    int st = prepare_surface_flux(h);
    if (st) return st;
    double inv_heat, inv_salt;
    surface_flux_scales(h->cfg, dt, &inv_heat, &inv_salt);
    Params p = make_params(h);
    vphys::launch_sw_penetration(p, inv_heat, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_sw_penetration launch");
}

int vphys_sw_chl_apply(vphys_handle h)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_sw_chl_apply: bad handle");
    if (!h->cfg.sw_chl) return push_error(VPHYS_ERR_CONFIG, "vphys_sw_chl_apply: sw_chl is 0");
    int st = prepare_sources(h);
    if (st) return st;
    Params p = make_params(h);
    vphys::launch_sw_chl_kappa(p, (const double *)h->f[VPHYS_FIELD_SW_CHL].ptr(), h->stream);
    return cuda_status(cudaGetLastError(), "vphys_sw_chl_apply");
}

int vphys_kappa_shear(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_kappa_shear: bad handle");
    if (h->cfg.idx_temperature < 0 || h->cfg.idx_salinity < 0) return VPHYS_OK;
    int st = prepare_kappa_shear(h);
    if (st) return st;
    Params p = make_params(h);
    launch_kappa_shear(h, p, dt);
    return cuda_status(cudaGetLastError(), "vphys_kappa_shear launch");
}

int vphys_epbl(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_epbl: bad handle");
    if (h->cfg.idx_temperature < 0 || h->cfg.idx_salinity < 0) return VPHYS_OK;
    int st = prepare_epbl(h);
    if (st) return st;
    Params p = make_params(h);
    vphys::launch_epbl(p, dt, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_epbl launch");
}

int vphys_mixed_redo_count(vphys_handle h, unsigned *groups)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_mixed_redo_count: bad handle");
    if (!groups) return VPHYS_OK;
    *groups = 0;
    if (!h->mp_redo) return VPHYS_OK;
    cudaError_t e = cudaMemcpyAsync(groups, h->mp_redo, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return cuda_status(e, "vphys_mixed_redo_count");
}

int vphys_stress_mag(vphys_handle h)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_stress_mag: bad handle");
    Params p = make_params(h);
    vphys::launch_stress_mag(p, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_stress_mag launch");
}

int vphys_assemble(vphys_handle h)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_assemble: bad handle");
    int st = prepare_assemble(h);
    if (st) return st;
    if (h->cfg.vmix_guard) {
        cudaError_t e = cudaMemsetAsync(h->guard_dev, 0, sizeof(unsigned long long), h->stream);
        if (e != cudaSuccess) return cuda_status(e, "vphys_assemble guard reset");
    }
    Params p = make_params(h);
    if ((st = run_learned_kpp(h, p))) return st;
    if ((st = run_assemble(h, p))) return st;
    gate_wrote_k(h);
    if (h->cfg.vmix_guard) {
        int gs = VPHYS_OK;
        if ((st = read_guard(h, &gs))) return st;
        return gs;
    }
    return VPHYS_OK;
}

int vphys_vdiff_momentum(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_vdiff_momentum: bad handle");
    int st = prepare_momentum(h);
    if (st) return st;
    Params p = make_params(h);
    vphys::launch_momentum(p, dt, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_vdiff_momentum launch");
}

int vphys_vdiff_tracers(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_vdiff_tracers: bad handle");
    int st = prepare_tracers(h);
    if (st) return st;
    if (h->ntr == 0) return VPHYS_OK;
    Params p = make_params(h);
    standalone_k(h, p);
    vphys::launch_tracers(p, dt, true, false, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_vdiff_tracers launch");
}

int vphys_nonlocal(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_nonlocal: bad handle");
    if (h->ntr == 0 || !h->cfg.use_kpp || h->cfg.epbl) return VPHYS_OK;
    Params p = make_params(h);
    vphys::launch_tracers(p, dt, false, true, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_nonlocal launch");
}

int vphys_vdiff_tracers_nonlocal(vphys_handle h, double dt)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_vdiff_tracers_nonlocal: bad handle");
    int st = prepare_tracers(h);
    if (st) return st;
    if (h->ntr == 0) return VPHYS_OK;
    Params p = make_params(h);
    standalone_k(h, p);
    vphys::launch_tracers(p, dt, true, h->cfg.use_kpp && !h->cfg.epbl, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_vdiff_tracers_nonlocal launch");
}

int vphys_set_variants(vphys_handle h, int momentum, int tracers)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_set_variants: bad handle");
    if (momentum < 0 || momentum >= vphys::N_VAR_MOM || tracers < 0 || tracers >= vphys::N_VAR_TR)
        return push_error(VPHYS_ERR_CONFIG, "vphys_set_variants: momentum in [0, %d), tracers in [0, %d)",
                          vphys::N_VAR_MOM, vphys::N_VAR_TR);
    h->var_mom = momentum;
    h->var_tr = tracers;
    return VPHYS_OK;
}

int vphys_autotune(vphys_handle h, double dt, int reps, double *ms, int n_ms, int *chosen)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_autotune: bad handle");
    if (reps < 1 || reps > 100) return push_error(VPHYS_ERR_CONFIG, "vphys_autotune: reps must be in [1, 100]");
    if (ms && n_ms > 0)
        for (int i = 0; i < n_ms; ++i) ms[i] = -1.0;
    if (!h->cfg.mixed_precision) {   // the exact solves have one form
        if (chosen) chosen[0] = h->var_mom, chosen[1] = h->var_tr;
        return VPHYS_OK;
    }
    int st;
    if ((st = prepare_assemble(h)) || (st = prepare_momentum(h)) || (st = prepare_tracers(h))) return st;
    // the handle's state, restored after the trials: every allocated real field
    std::vector<std::pair<int, void *>> saved;
    auto release = [&]() {
        for (auto &s : saved) cudaFree(s.second);
        saved.clear();
    };
    for (int id = 0; id < (int)h->f.size(); ++id) {
        const Field &fl = h->f[id];
        if (!fl.ptr() || fl.is_int) continue;
        void *b = nullptr;
        cudaError_t e = cudaMalloc(&b, fl.bytes());
        if (e == cudaSuccess) e = cudaMemcpyAsync(b, fl.ptr(), fl.bytes(), cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) {
            if (b) cudaFree(b);
            cudaGetLastError();
            release();
            return push_error(VPHYS_ERR_ALLOC, "vphys_autotune: no room for a copy of the state (%s)",
                              cudaGetErrorString(e));
        }
        saved.emplace_back(id, b);
    }
    auto restore = [&]() {
        for (auto &s : saved)
            cudaMemcpyAsync(h->f[s.first].ptr(), s.second, h->f[s.first].bytes(), cudaMemcpyDeviceToDevice, h->stream);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // the coefficients the solves read, as in a step
    {
        Params p = make_params(h);
        if (h->cfg.eos_in_step) vphys::launch_eos_wright(p, h->stream);
        if ((st = run_assemble(h, p))) {
            release();
            return st;
        }
    }
    const bool kpp_nonlocal = h->cfg.use_kpp && !h->cfg.epbl;
    auto trial = [&](auto launch) -> double {
        float total = 0.0f;
        for (int r = 0; r <= reps; ++r) {   // the first run is a warm-up
            restore();
            cudaEventRecord(e0, h->stream);
            launch();
            cudaEventRecord(e1, h->stream);
            cudaEventSynchronize(e1);
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r > 0) total += t;
        }
        return (double)total / reps;
    };
    double best_m = 1e30, best_t = 1e30;
    int pick_m = h->var_mom, pick_t = h->var_tr;
    for (int v = 0; v < vphys::N_VAR_MOM; ++v) {
        Params p = make_params(h);
        p.var_mom = v;
        if (v == vphys::VAR_MOM_RING && !vphys::momentum_tma_eligible(p)) continue;
        const double t = trial([&]() { vphys::launch_momentum(p, dt, h->stream); });
        if (ms && v < n_ms) ms[v] = t;
        if (t < best_m) best_m = t, pick_m = v;
    }
    for (int v = 0; v < vphys::N_VAR_TR && h->ntr > 0; ++v) {
        Params p = make_params(h);
        p.var_tr = v;
        // variants other than one tracer per warp need one factorisation (ks = kt);
        // the tensor-memory rows also need the default tracer knobs
        if (v != vphys::VAR_TR_SMEM1 && !p.ks_equals_kt) continue;
        if (v == vphys::VAR_TR_TMEM && !vphys::is_default_tracer_knobs(p.cfg)) continue;
        const double t = trial([&]() { vphys::launch_tracers(p, dt, true, kpp_nonlocal, h->stream); });
        if (ms && vphys::N_VAR_MOM + v < n_ms) ms[vphys::N_VAR_MOM + v] = t;
        if (t < best_t) best_t = t, pick_t = v;
    }
    restore();
    st = cuda_status(cudaStreamSynchronize(h->stream), "vphys_autotune");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release();
    if (st) return st;
    h->var_mom = pick_m;
    h->var_tr = pick_t;
    if (chosen) chosen[0] = pick_m, chosen[1] = pick_t;
    return VPHYS_OK;
}

int vphys_step(vphys_handle h, double dt, int n_steps)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_step: bad handle");
    if (n_steps <= 0) return VPHYS_OK;
    int st;
    if ((st = prepare_assemble(h)) || (st = prepare_momentum(h)) || (st = prepare_tracers(h)) ||
        (h->cfg.surface_flux && (st = prepare_surface_flux(h))) || (st = prepare_fork(h)))
        return st;
    if (h->cfg.eos_in_step && (h->cfg.idx_temperature < 0 || h->cfg.idx_salinity < 0))
        return push_error(VPHYS_ERR_CONFIG, "vphys_step: eos_in_step needs temperature and salinity tracers");
    if (h->cfg.vmix_guard) {
        cudaError_t e = cudaMemsetAsync(h->guard_dev, 0, sizeof(unsigned long long), h->stream);
        if (e != cudaSuccess) return cuda_status(e, "vphys_step guard reset");
    }
    Params p = make_params(h);
    if ((st = launch_steps(h, p, dt, n_steps))) return st;
    if ((st = cuda_status(cudaGetLastError(), "vphys_step launch"))) return st;
    gate_wrote_k(h);
    if (h->cfg.vmix_guard) {
        int gs = VPHYS_OK;
        if ((st = read_guard(h, &gs))) return st;
        return gs;
    }
    return VPHYS_OK;
}

int vphys_step_graph(vphys_handle h, double dt, int n_steps)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_step_graph: bad handle");
    if (n_steps <= 0) return VPHYS_OK;
    int st;
    if ((st = prepare_assemble(h)) || (st = prepare_momentum(h)) || (st = prepare_tracers(h)) ||
        (h->cfg.surface_flux && (st = prepare_surface_flux(h))) || (st = prepare_fork(h)))
        return st;
    if (h->cfg.eos_in_step && (h->cfg.idx_temperature < 0 || h->cfg.idx_salinity < 0))
        return push_error(VPHYS_ERR_CONFIG, "vphys_step_graph: eos_in_step needs temperature and salinity tracers");
    if (h->cfg.vmix_guard) {
        cudaError_t e = cudaMemsetAsync(h->guard_dev, 0, sizeof(unsigned long long), h->stream);
        if (e != cudaSuccess) return cuda_status(e, "vphys_step_graph guard reset");
    }
    Params p = make_params(h);
    // what the launches depend on: every pointer and knob (Params), dt, n and
    // the surrogate; any change (a bind, a new config, an attach) recaptures
    unsigned char sig[sizeof h->gsig] = {};
    memcpy(sig, &p, sizeof p);
    memcpy(sig + sizeof p, &h->kpp, sizeof h->kpp);
    memcpy(sig + sizeof p + sizeof h->kpp, &dt, sizeof dt);
    memcpy(sig + sizeof p + sizeof h->kpp + 8, &n_steps, sizeof n_steps);
    sig[sizeof p + sizeof h->kpp + 12] = h->kpp_attached ? 1 : 0;
    if (!h->gexec || memcmp(sig, h->gsig, sizeof sig) != 0) {
        if (h->gexec) {
            cudaGraphExecDestroy(h->gexec);
            h->gexec = nullptr;
        }
        cudaError_t e = cudaSuccess;
        if (!h->cap_stream) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e, "vphys_step_graph stream");
        cudaStream_t user = h->stream;
        const int gen0 = h->gen;
        const unsigned kgen0 = h->kgen;
        h->stream = h->cap_stream;
        e = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeRelaxed);
        int lst = (e == cudaSuccess) ? launch_steps(h, p, dt, n_steps) : VPHYS_OK;
        cudaGraph_t graph = nullptr;
        cudaError_t e2 = (e == cudaSuccess) ? cudaStreamEndCapture(h->cap_stream, &graph) : e;
        h->stream = user;
        h->gen = gen0;
        h->kgen = kgen0 + (unsigned)n_steps;
        if (e != cudaSuccess || e2 != cudaSuccess || lst != VPHYS_OK) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (lst != VPHYS_OK) return lst;
            return cuda_status(e != cudaSuccess ? e : e2, "vphys_step_graph capture");
        }
        e = cudaGraphInstantiate(&h->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            h->gexec = nullptr;
            return cuda_status(e, "vphys_step_graph instantiate");
        }
        memcpy(h->gsig, sig, sizeof sig);
    }
    cudaError_t e = cudaGraphLaunch(h->gexec, h->stream);
    if (e != cudaSuccess) return cuda_status(e, "vphys_step_graph launch");
    h->gen += n_steps;
    gate_wrote_k(h);
    if (h->cfg.vmix_guard) {
        int gs = VPHYS_OK;
        if ((st = read_guard(h, &gs))) return st;
        return gs;
    }
    return VPHYS_OK;
}

int vphys_synchronize(vphys_handle h)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_synchronize: bad handle");
    int st = cuda_status(cudaStreamSynchronize(h->stream), "vphys_synchronize");
    if (st) return st;
    if (h->aux_stream && (st = cuda_status(cudaStreamSynchronize(h->aux_stream), "vphys_synchronize"))) return st;
    return check_dev_err(h);
}

int vphys_kpp_attach(vphys_handle h, const vphys_kpp_model *m)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_kpp_attach: bad handle");
    if (!m) {
        free_kpp(h);
        return VPHYS_OK;
    }
    if (!m->w1 || !m->w2 || !m->w3 || !m->b1 || !m->b2 || !m->b3 || !m->feat_mean || !m->feat_istd)
        return push_error(VPHYS_ERR_CONFIG, "vphys_kpp_attach: a weight, bias or standardisation pointer is NULL");
    if (!(m->target_std0 > 0.0f) || !(m->gate_limit > 0.0f) || m->check_fraction < 0.0f || m->check_fraction > 1.0f)
        return push_error(VPHYS_ERR_CONFIG, "vphys_kpp_attach: target_std0 and gate_limit must be > 0, "
                                            "check_fraction in [0, 1]");
    if ((((uintptr_t)m->w1) | ((uintptr_t)m->w2) | ((uintptr_t)m->w3)) & 15)
        return push_error(VPHYS_ERR_BAD_SHAPE, "vphys_kpp_attach: weights must be 16-byte aligned");
    free_kpp(h);
    const size_t nc = (size_t)h->nx * h->ny;
    struct {
        void **p;
        size_t bytes;
    } want[] = {{&h->kX, nc * vphys::LK_INP * 2},
                {(void **)&h->kY, nc * vphys::LK_OUTP * sizeof(float)},
                {(void **)&h->kcolH, nc * sizeof(float)},
                {(void **)&h->kpred, nc * sizeof(float)},
                {(void **)&h->kcheck, nc * sizeof(float)},
                {(void **)&h->kgate, nc},
                {(void **)&h->kstats, 16 * sizeof(unsigned long long)},
                {(void **)&h->kerr, sizeof(int)}};
    for (auto &w : want) {
        if (cudaMalloc(w.p, w.bytes) != cudaSuccess) {
            cudaGetLastError();
            free_kpp(h);
            return push_error(VPHYS_ERR_ALLOC, "vphys_kpp_attach: cudaMalloc of the surrogate's scratch failed");
        }
    }
    cudaMemsetAsync(h->kstats, 0, 16 * sizeof(unsigned long long), h->stream);
    cudaMemsetAsync(h->kerr, 0, sizeof(int), h->stream);
    h->kpp = *m;
    h->kpp_attached = true;
    h->kgen = 0;
    return cuda_status(cudaGetLastError(), "vphys_kpp_attach");
}

int vphys_kpp_stats(vphys_handle h, unsigned long long *out, int n)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_kpp_stats: bad handle");
    if (!h->kpp_attached) return push_error(VPHYS_ERR_NOT_INITIALISED, "vphys_kpp_stats: no surrogate attached");
    if (!out || n <= 0) return VPHYS_OK;
    unsigned long long tmp[16];
    int gemm_err = 0;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(tmp, h->kstats, sizeof tmp, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&gemm_err, h->kerr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "vphys_kpp_stats");
    tmp[10] = (unsigned long long)gemm_err;
    for (int i = 0; i < n && i < 16; ++i) out[i] = tmp[i];
    if (gemm_err) return push_error(VPHYS_ERR_CUDA, "learned KPP: a tensor-core GEMM gave up waiting (code %d)", gemm_err);
    return VPHYS_OK;
}

int vphys_kpp_features(vphys_handle h, const float *mean, const float *istd, float gate_limit, float *raw, void *X,
                       void *XT, long long ld_t, unsigned char *gate, float *colH)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_kpp_features: bad handle");
    if ((mean == nullptr) != (istd == nullptr))
        return push_error(VPHYS_ERR_CONFIG, "vphys_kpp_features: mean and istd go together");
    Params p = make_params(h);
    vphys::launch_kpp_features(p, raw, X, XT, ld_t, mean, istd, gate_limit, gate, colH, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_kpp_features launch");
}

int vphys_kpp_targets(vphys_handle h, float *T)
{
    if (!valid(h)) return push_error(VPHYS_ERR_BAD_HANDLE, "vphys_kpp_targets: bad handle");
    if (!T) return push_error(VPHYS_ERR_CONFIG, "vphys_kpp_targets: NULL");
    Params p = make_params(h);
    vphys::launch_kpp_targets(p, T, h->stream);
    return cuda_status(cudaGetLastError(), "vphys_kpp_targets launch");
}

}  // extern "C"
