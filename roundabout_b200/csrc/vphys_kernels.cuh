// vphys_kernels.cuh -- launch parameters shared by the host runtime and the
// kernels of libvphys.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/vphys.h"

namespace vphys {

constexpr int NZ_MAX = VPHYS_NZ_MAX + 1;   // per-column local arrays (>= nz + 1)

// Kernel variants of the mixed-precision solves that vphys_autotune chooses
// between (the same results up to FP32 rounding order; each applies where
// its eligibility test passes, the register forms everywhere).
constexpr int VAR_MOM_REGISTER = 0;   // k_momentum_mp: loads prefetched in registers
constexpr int VAR_MOM_RING = 1;       // k_momentum_mp_tma: TMA-staged ring (vphys_mom_ring.cuh)
constexpr int VAR_TR_SMEM1 = 0;       // k_tracers_mp, rows in shared memory, one tracer per warp
constexpr int VAR_TR_SMEM2 = 1;       // the same, two tracers per warp (one factorisation)
constexpr int VAR_TR_SMEM4 = 2;       // the same, four tracers per warp
constexpr int VAR_TR_TMEM = 3;        // k_tracers_mp_tm, rows in tensor memory
constexpr int N_VAR_MOM = 2, N_VAR_TR = 4;
constexpr int NTR_MAX = 16;                // tracers a handle may carry

// learned KPP surrogate: 75 feature levels below the surface layer,
// 154 inputs (K padded to 160), 256 hidden, 77 outputs (padded to 80)
constexpr int LK_LEV = 75;
constexpr int LK_IN = 154;
constexpr int LK_INP = 160;
constexpr int LK_HID = 256;
constexpr int LK_OUT = 77;
constexpr int LK_OUTP = 80;

// Everything a kernel needs: the grid, the knobs and the device pointers.
struct Params {
    int nx, ny, nz, ntr;
    size_t plane;        // nx*ny: stride between levels of cell/interface arrays
    size_t plane_u;      // (nx+1)*ny
    size_t plane_v;      // nx*(ny+1)
    vphys_config cfg;
    // state
    const double *h;
    double *rho, *u, *v, *kv, *kt, *ks;
    double *bl_depth, *b0;
    const double *stress_mag, *q_heat, *q_salt, *wet;
    // the shortwave source the host selected (q_heat, or SW_NET under
    // sw_source = 1) and the dynamic wet mask (NULL unless use_wet_dyn)
    const double *sw_src, *wet_dyn;
    // the chlorophyll scheme's band opacities, (nx, ny, VPHYS_SW_NB_MAX); NULL unless sw_chl
    const double *sw_kappa;
    const double *cover_frac;   // ice-shelf cover fraction; NULL unless use_cover_frac
    // compensated column content before / after the tracer diffusion, (nx, ny, ntr); NULL unless column_integrals
    double *content_old, *content_new;
    const double *tau_x, *tau_y, *lambda_bot_u, *lambda_bot_v;
    double *visc_rem_u, *visc_rem_v;
    double *gamma_t, *gamma_s;       // nullptr: not written
    double *heat_budget, *salt_budget;
    double *heat_budget_surface, *salt_budget_surface;   // surface-flux deposit books (budgets on)
    double *budget_scratch;          // 2 planes x nz: forward-swept T and S when budgets are on
    const int *k_top_u, *k_top_v, *k_bot_u, *k_bot_v;   // nullptr: nz / 1
    double *tr[NTR_MAX];
    unsigned long long *guard_count;  // vmix_guard counter (device)
    int *span;                        // per column: first | last live layer << 16 (0: none), scratch
    unsigned *mp_redo;                // mixed solves: count, then (group << 5 | tracer) re-solved in FP64
    unsigned *work_ctr;               // next work item of a dynamically scheduled solve (reset by k_spans)
    int var_mom;                      // mixed face solve: VAR_MOM_REGISTER or VAR_MOM_RING (where eligible)
    int var_tr;                       // mixed tracer solve: VAR_TR_* (where eligible)
    double *zcol;                     // per column: -sum_k h, k = 1..nz in order (momentum z_clear), scratch
    unsigned char *mom_tile_skip;     // per face tile of the TMA-staged momentum solve: 1 = nothing to solve
    unsigned *dev_err;                // bounded waits that ran out (bit 0: consumer, 1: producer, 2: drain)
    const double *coriolis;           // (nx, ny) f, or nullptr (learned KPP features, kappa-shear f^2)
    double *kd_shear, *tke_shear;     // (nx, ny, nz+1) kappa-shear diffusivity and TKE, or nullptr
    double *kd_epbl, *mld_epbl;       // (nx, ny, nz+1) EPBL diffusivity, (nx, ny) its MLD, or nullptr
    double *la_epbl;                  // (nx, ny) EPBL Langmuir number, or nullptr
    double *epbl_tke[6];              // (nx, ny) EPBL TKE budget terms (wind, conv, forcing, mixing,
                                      // mech_decay, conv_decay), or nullptr when not requested
    const float *kpp_pred;            // per column: the surrogate's h_b, < 0: run pass 1; nullptr: plain KPP
    const float *kpp_check;           // per column: h_b to compare with pass 1 (>= 0), or nullptr
    unsigned long long *kpp_stats;    // learned KPP counters (k_kpp_roll)
    float kpp_tol;                    // relative h_b difference counted as a failed check
    int ks_equals_kt;                 // ks is bitwise kt after the gate
    int write_gamma;
};

// Push a message onto the library's error ring and return `status` (vphys_api.cu).
int report_error(int status, const char *msg);

// Launchers (vphys_kernels.cu); all asynchronous on `stream`.
void launch_eos_wright(const Params &p, cudaStream_t stream);
// surface heat/salt deposit on the first live layer; inv_heat = dt/(rho0 cp), inv_salt = dt/rho0
void launch_surface_flux(const Params &p, double inv_heat, double inv_salt, cudaStream_t stream);
// the penetrating shortwave spread down the column; inv_scale = dt/(rho0 cp)
void launch_sw_penetration(const Params &p, double inv_scale, cudaStream_t stream);
void launch_stress_mag(const Params &p, cudaStream_t stream);
// kappa-shear column solve into p.kd_shear / p.tke_shear (vphys_kshear.cu).
// work (per column, zeroed before the first call) carries each column's cost
// from one call to the next; with `ordered`, the columns are solved heaviest
// first through order (per column) bucketed in hist (1024 counts).
void launch_sw_chl_kappa(const Params &p, const double *chl, cudaStream_t stream);
void launch_kappa_shear(const Params &p, double dt, int *work, int *order, unsigned *hist, bool ordered,
                        cudaStream_t stream);
// EPBL column solve into p.kd_epbl / p.mld_epbl (vphys_epbl.cu)
void launch_epbl(const Params &p, double dt, cudaStream_t stream);
void launch_assemble(const Params &p, cudaStream_t stream);
void launch_smooth(const Params &p, double *fld, double *scratch, cudaStream_t stream);
void launch_momentum(const Params &p, double dt, cudaStream_t stream);
// the TMA-staged ring of the mixed-precision face solve (vphys_mixed.cu,
// host side in vphys_momentum_tma.cu): false when the configuration or the
// buffers do not qualify (the caller runs k_momentum_mp)
bool launch_momentum_mp_tma(const Params &p, double dt, cudaStream_t stream);
bool momentum_tma_eligible(const Params &p);
int momentum_tma_tiles(const Params &p);

// -sum of h over each column, accumulated k = 1..nz as vdiff's z_clear does (into p.zcol)
void launch_column_depth(const Params &p, cudaStream_t stream);
void launch_tracers(const Params &p, double dt, bool diffuse, bool nonlocal, cudaStream_t stream);
// mixed-precision solves (vphys_mixed.cu), dispatched by the two above when cfg.mixed_precision
void launch_momentum_mp(const Params &p, double dt, cudaStream_t stream);
void launch_tracers_mp(const Params &p, double dt, bool nonlocal, cudaStream_t stream);
// the FP64 re-solve of the groups the mixed tracer kernel listed in p.mp_redo (vphys_tracers.cu)
void launch_tracers_redo(const Params &p, double dt, bool nonlocal, cudaStream_t stream);
// learned KPP (vphys_learned.cu)
void launch_kpp_features(const Params &p, float *raw, void *X, void *XT, long long ld_t, const float *mean,
                         const float *istd, float limit, unsigned char *gate, float *colH, cudaStream_t s);
void launch_kpp_targets(const Params &p, float *T, cudaStream_t s);
void launch_kpp_roll(unsigned long long *st, float fail_fraction, cudaStream_t s);
void launch_kpp_apply(size_t ncols, const float *Y, float tmean0, float tstd0, const unsigned char *gate,
                      const float *colH, float *pred, float *check, unsigned long long *st, unsigned gen,
                      float check_fraction, cudaStream_t s);
// tcgen05 GEMM (vphys_gemm.cu)
int gemm_tn_bf16(const void *A, long long lda, const void *B, long long ldb, int M, int N, int K, float alpha,
                 const float *bias, const float *zin, int ld_z, int act, float *out_f32, int ld_f32, void *out_bf16,
                 int ld_bf16, void *out_bf16_t, int ld_t, int *err, cudaStream_t stream);
int mlp3_bf16(const void *X, int M, const void *W1, const float *b1, const void *W2, const float *b2, const void *W3,
              const float *b3, float *Y, int *err, cudaStream_t stream);
void launch_selftest_division(unsigned long long seed, long long per_thread, int emin, int erange,
                              unsigned long long *bad, cudaStream_t stream);

}  // namespace vphys
