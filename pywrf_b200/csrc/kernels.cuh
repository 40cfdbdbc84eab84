// Launchers of the step kernels (one group per reference phase).  Each
// returns the number of kernels it enqueued.
#pragma once
#include "wrf_common.cuh"
#include "bc.cuh"

namespace wrf {

// column kernels keep one vertical column per thread in local arrays
constexpr int kMaxNz = 64;

// the kernel form wrf_set_kernel_form selected (WRF_FORM_FAST or WRF_FORM_POINT)
int kernel_form();
int set_kernel_form(int form);  // returns the previous form

// rk_step_prep: calculate_full, calc_mu_uv, couple_momentum, calc_ww_cp,
// calc_cq, calc_alt, calc_php (k_prep.cu)
int launch_prep(const Grid& g, const S& s, cudaStream_t st);
// compute_diff_metrics (k_prep.cu)
int launch_diff_metrics(const Grid& g, const S& s, cudaStream_t st);
// cal_deform_and_div (defor11/22/12 and defor12's boundary copies) alone,
// and with calculate_km_kh (k_prep.cu)
int launch_deform(const Grid& g, const S& s, cudaStream_t st);
int launch_km(const Grid& g, const S& s, cudaStream_t st);
// horizontal_diffusion u/v/w/theta + relax_bdytend u/v/ph/t/mu (k_prep.cu)
int launch_hdiff_relax(const Grid& g, const S& s, cudaStream_t st);
// relax_bdytend + spec_bdytend of qv into moist_tend (k_prep.cu)
int launch_relax_qv(const Grid& g, const S& s, cudaStream_t st);

// advection of u, v, w, theta and the pressure-gradient / buoyancy /
// Coriolis / curvature forces (k_tend.cu)
int launch_advect_forces(const Grid& g, const S& s, cudaStream_t st);
// k_forces in its tiled tensor-map form (k_forces_tma.cu); 0 (nothing
// launched) when nx is not a multiple of 4, a map is refused or the point form
// is selected
int launch_forces_tma(const Grid& g, const S& s, cudaStream_t st);
// the tendency terms selected by a mask (1 rhs_ph, 2 pressure gradient,
// 4 pg_buoy_w, 8 coriolis, 16 curvature) with the point kernel (k_tend.cu),
// and their adjoint (k_adjoint_forces.cu)
int launch_forces_terms(const Grid& g, const S& s, int terms, cudaStream_t st);
int launch_forces_adj(const Grid& g, const S& s, const S& b, int terms, cudaStream_t st);
// sumflux, spec_bdyupdate (var 't', 'u', 'v' 3-D or 'm' 2-D) and
// spec_bdyupdate_ph as stand-alone operators, and their adjoints
// (k_adjoint_subbdy.cu)
int launch_sumflux(const Grid& g, const S& s, int iteration, int nsub, cudaStream_t st);
int launch_sumflux_adj(const Grid& g, const S& s, const S& b, int iteration, int nsub, cudaStream_t st);
int launch_spec_update(const Grid& g, float* field, const float* tend, float dt, char var, bool two_d, cudaStream_t st);
int launch_spec_update_adj(const Grid& g, const float* field_bar, float* tend_bar, float dt, char var, bool two_d,
                           cudaStream_t st);
int launch_spec_ph(const Grid& g, const S& s, float dt, cudaStream_t st);
int launch_spec_ph_adj(const Grid& g, const S& s, const S& b, float dt, cudaStream_t st);
// rk_step_prep's functions selected by a mask (1 calculate_full, 2
// calc_mu_uv, 4 couple_momentum, 8 calc_ww_cp, 16 calc_cq, 32 calc_alt, 64
// calc_php) and their adjoints (k_adjoint_prep.cu)
int launch_prep_ops(const Grid& g, const S& s, int ops, cudaStream_t st);
int launch_prep_ops_adj(const Grid& g, const S& s, const S& b, int ops, cudaStream_t st);
// rk_addtend_dry and spec_bdytend as stand-alone operators, and their
// adjoints (k_adjoint_tend.cu); bt4: the x-start, x-end, y-start, y-end
// boundary tendencies of the variable
int launch_addtend_op(const Grid& g, const S& s, int rk_step, cudaStream_t st);
int launch_addtend_op_adj(const Grid& g, const S& s, const S& b, int rk_step, cudaStream_t st);
int launch_spec_tend(const Grid& g, float* tend, const float* const* bt4, char var, cudaStream_t st);
int launch_spec_tend_adj(const Grid& g, float* tend_bar, char var, cudaStream_t st);
// the first stage's horizontal diffusion of one field ('u', 'v', 'w', or
// 'm' for a mass-point scalar, about base when given), the eddy viscosities
// and mass_weight as stand-alone operators with their adjoints
// (k_adjoint_diff.cu)
int launch_hdiff_op(const Grid& g, const S& s, char var, const float* f, const float* base, const float* mut,
                    const float* K, float* tend, cudaStream_t st);
int launch_hdiff_op_adj(const Grid& g, const S& s, char var, const float* f, const float* base, const float* mut,
                        const float* K, const float* tbar, float* fbar, float* mutbar, float* Kbar, cudaStream_t st);
int launch_km_op(const Grid& g, const S& s, cudaStream_t st);
int launch_km_op_adj(const Grid& g, const S& s, const S& b, float* work, cudaStream_t st);
int launch_mass_weight(const Grid& g, const float* f, const float* mut, float* out, int nk, cudaStream_t st);
int launch_mass_weight_adj(const Grid& g, const float* f, const float* mut, const float* ob, float* fb, float* mb,
                           int nk, cudaStream_t st);
// rk_addtend_dry + spec_bdytend (k_tend.cu)
int launch_addtend(const Grid& g, const S& s, int rk_step, cudaStream_t st);
// moisture advection with the time-averaged fluxes (k_tend.cu)
int launch_advect_moist(const Grid& g, const S& s, cudaStream_t st);
// tiled scalar advection (k_advect_tiled.cu): the six moisture species with
// ru_m / rv_m / ww_m into advect_tend, theta with ru / rv / ww into t_tend
int launch_advect_moist_tiled(const Grid& g, const S& s, cudaStream_t st);
int launch_advect_theta_tiled(const Grid& g, const S& s, cudaStream_t st);
// advect_u / advect_v / advect_w of the components comp0 .. comp0+ncomp-1
// (0 u, 1 v, 2 w) in one tiled TMA launch (k_advect_tiled.cu); 0 (nothing
// launched) when nx is not a multiple of 4 or a map is refused
int launch_advect_mom_tma(const Grid& g, const S& s, int comp0, int ncomp, cudaStream_t st);
// the same with one thread per point (k_tend.cu), components as a bit mask
int launch_advect_mom_point(const Grid& g, const S& s, int comps, cudaStream_t st);
// stand-alone advect_scalar (k_tend.cu)
int launch_advect_scalar(const Grid& g, const S& s, const float* field, float* tend, const float* ru,
                          const float* rv, const float* rom, cudaStream_t st);

// adjoint of advect_scalar w.r.t. the field and ru / rv / rom (k_adjoint.cu);
// accumulates into qbar, rubar, rvbar, rombar
int launch_advance_uv_adj(const Grid& g, const S& s, const S& b, float dts, cudaStream_t st);
int launch_calc_p_rho(const Grid& g, const S& s, int step, cudaStream_t st);
int launch_advance_mu_t(const Grid& g, const S& s, float dts, cudaStream_t st);
int launch_advance_w(const Grid& g, const S& s, float dts, cudaStream_t st);
int launch_advance_w_adj(const Grid& g, const S& s, const S& b, float dts, float* work, cudaStream_t st);
int launch_advance_mu_t_adj(const Grid& g, const S& s, const S& b, float dts, int ref_no_grad, float* work,
                            cudaStream_t st);
int launch_calc_p_rho_adj(const Grid& g, const S& s, const S& b, int step, cudaStream_t st);
// work: advect_mom_adj_work_floats(g) floats (the faces' stencil slots)
size_t advect_mom_adj_work_floats(const Grid& g);
int launch_advect_mom_adj(const Grid& g, int component, const float* q, const float* ru, const float* rv,
                          const float* rom, const float* msf, const float* msf2, const float* fzm, const float* fzp,
                          const float* rdz, const float* tbar, float* qbar, float* rubar, float* rvbar,
                          float* rombar, float* work, cudaStream_t st);
// work: advect_scalar_adj_work_floats(g) floats (the faces' stencil slots)
size_t advect_scalar_adj_work_floats(const Grid& g);
int launch_advect_scalar_adj(const Grid& g, const float* q, const float* ru, const float* rv, const float* rom,
                             const float* msftx, const float* fnm, const float* fnp, const float* rdnw,
                             const float* tbar, float* qbar, float* rubar, float* rvbar, float* rombar, float* work,
                             cudaStream_t st);

// relax_bdytend on one field (bdy8: xs xe ys ye txs txe tys tye device
// arrays) and its adjoint w.r.t. the field (k_adjoint.cu)
int launch_relax_field(const Grid& g, const float* field, float* tend, const float* const* bdy8, char var, float dtbc,
                       cudaStream_t st);
int launch_relax_field_adj(const Grid& g, const float* tbar, float* fbar, char var, cudaStream_t st);

// the implicit w solve of advance_w on ncol columns of nz levels, and its
// adjoint (accumulates into xbar, abar, alphabar, gammabar) (k_adjoint.cu)
int launch_vsolve_w(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma, float* w,
                    cudaStream_t st);
int launch_vsolve_w_adj(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                        const float* wbar, float* xbar, float* abar, float* alphabar, float* gammabar,
                        cudaStream_t st);

// calc_coef_w's adjoint w.r.t. cqw, c2a and mut (accumulates) (k_adjoint.cu)
int launch_coef_w_adj(const Grid& g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                      const float* rdnw, float dts, const float* abar, const float* alphabar, const float* gammabar,
                      float* mutbar, float* cqwbar, float* c2abar, cudaStream_t st);
// calc_coef_w alone on caller arrays (k_acoustic.cu)
int launch_coef_w(const Grid& g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                  const float* rdnw, float dts, float* a, float* alpha, float* gamma, cudaStream_t st);

// acoustic steps (k_acoustic.cu)
int launch_small_step_prep(const Grid& g, const S& s, int rk_step, float dts, cudaStream_t st);
int launch_advance_uv(const Grid& g, const S& s, float dts, cudaStream_t st);
int launch_acoustic_col(const Grid& g, const S& s, float dts, int iteration, int nsub, cudaStream_t st);
int launch_small_step_finish(const Grid& g, const S& s, float dts, int nsub, int rk_step, cudaStream_t st);
// small_step_prep without the calc_p_rho / calc_coef_w that follow it in the
// step (k_acoustic.cu), and the adjoints of small_step_prep and of
// calc_mu_uv_1 + small_step_finish (k_adjoint_ssp.cu)
int launch_ssp_only(const Grid& g, const S& s, int rk_step, cudaStream_t st);
int launch_small_step_prep_adj(const Grid& g, const S& s, const S& b, int rk_step, float* work, cudaStream_t st);
int launch_small_step_finish_adj(const Grid& g, const S& s, const S& b, float dts, int nsub, int rk_step, float* work,
                                 cudaStream_t st);

// moisture (k_moist.cu)
int launch_hdiff_moist(const Grid& g, const S& s, cudaStream_t st);
// calc_p_rho_phi alone (k_moist.cu)
int launch_eos(const Grid& g, const S& s, cudaStream_t st);
int launch_moist(const Grid& g, const S& s, int rk_step, float dt_rk, cudaStream_t st);
// its adjoint (k_adjoint_moist.cu); work: nz*ny*nx floats
int launch_moist_adj(const Grid& g, const S& s, const S& b, int rk_step, float dt_rk, float* work, cudaStream_t st);
// calc_p_rho_phi's reverse with the state's own qv (k_adjoint_moist.cu)
int launch_eos_adj(const Grid& g, const S& s, const S& b, cudaStream_t st);
// the microphysics block's reverse (the equation of state after it, then
// prep + WSM6 + finish by a per-column tape, forward-mode tangents for the
// columns whose tape outgrows its capacity; k_adjoint_wsm6.cu): s holds the
// block's inputs, post the state after it; work holds
// microphysics_adj_work_floats(g) floats; values (optional) receives the
// taped code's own outputs
size_t microphysics_adj_work_floats(const Grid& g);
// the tape capacity in entries per column (0: the default, which grows with
// the levels); returns the previous setting
int set_microphysics_tape_capacity(int entries);
int launch_physics_adj(const Grid& g, const S& s, const S& post, const S& b, float* work, float dt, cudaStream_t st,
                       const S* values);
int launch_bdy_final(const Grid& g, const S& s, cudaStream_t st);
// spec_bdy_final + set_w_surface as a stand-alone operator and its adjoint
// (k_adjoint_end.cu)
int launch_bdy_final_op(const Grid& g, const S& s, cudaStream_t st);
int launch_bdy_final_op_adj(const Grid& g, const S& s, const S& b, cudaStream_t st);

// microphysics (k_wsm6.cu)
int launch_physics(const Grid& g, const S& s, cudaStream_t st);
int launch_wsm6(const Grid& g, float* const* f, float delt, cudaStream_t st);
// WSM6 with a fixed file-scope device scratch (returns kernels or WRF_E*, *err set)
int launch_wsm6_noalloc(const Grid& g, float* const* f, float delt, cudaStream_t st, const char** err);

}  // namespace wrf
