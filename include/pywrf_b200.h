/*
 * pywrf_b200 C ABI: the ARW integration step of PyWRF on sm_100a.
 *
 * Everything here is plain C: device pointers, sizes and a cudaStream_t
 * (passed as void*).  The caller owns all memory (no allocation inside any
 * entry point) and launches run asynchronously on the given stream.  Return
 * value: 0 on success, negative WRF_E* codes on bad arguments or CUDA launch
 * errors.  Device-side failures (NaN in the diagnosed pressure, exhausted
 * bounded waits) are recorded in the WF_STATUS int array and read with
 * wrf_status_read after the stream is synchronised.
 *
 * Layout: 3-D fields are [nz][ny][nx] float32 (x fastest) with the
 * reference's 5-cell frame: ids = jds = 5, ide = nx - 5, jde = ny - 5
 * (pywrf/config_params.py:67-99); 2-D fields [ny][nx]; vertical profiles
 * [nz]; the 7 moisture slots [7][nz][ny][nx] (slot 0 unused, 1..6 =
 * qv qc qr qi qs qg, config_params.py:102-108); lateral-boundary arrays in
 * the reference's permuted layout: x sides [nzb][ny][5], y sides [nzb][5][nx]
 * with nzb = nz (nzb = 1 for mu) (pywrf/solver.py:468-482).
 */
#ifndef PYWRF_B200_H
#define PYWRF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WRF_OK 0
#define WRF_EINVAL (-1)   /* bad grid / null pointer / unsupported option */
#define WRF_ECUDA (-2)    /* a kernel launch failed (see wrf_last_error) */

/* kinds of the fields in the state table */
#define WRF_K3 3      /* [nz][ny][nx] */
#define WRF_K2 2      /* [ny][nx] */
#define WRF_K1 1      /* [nz] */
#define WRF_K4 4      /* [7][nz][ny][nx] */
#define WRF_KBX 10    /* [nz][ny][5] */
#define WRF_KBY 11    /* [nz][5][nx] */
#define WRF_KBX2 12   /* [1][ny][5] */
#define WRF_KBY2 13   /* [1][5][nx] */
#define WRF_KSF 20    /* float[16] device scalars */
#define WRF_KSI 21    /* int32[16] device status words */

/* status words (WF_STATUS) */
#define WRF_ST_NAN_P 0        /* NaN points met in the diagnosed p (summed over RK stages) */
#define WRF_ST_STEP 1         /* completed steps (device step counter) */
#define WRF_ST_WAIT 2         /* thread blocks whose bounded wait on a tile load ran out (tiled advection) */

/* the persistent state of one integration, in table order */
#define WRF_FIELD_TABLE(X) \
  X(U, WRF_K3) X(V, WRF_K3) X(W, WRF_K3) X(T, WRF_K3) X(PH, WRF_K3) X(P, WRF_K3) X(AL, WRF_K3) \
  X(PB, WRF_K3) X(PHB, WRF_K3) X(T_INIT, WRF_K3) X(ALB, WRF_K3) X(RU, WRF_K3) X(RV, WRF_K3) \
  X(RW, WRF_K3) X(WW, WRF_K3) X(WW1, WRF_K3) X(CQU, WRF_K3) X(CQV, WRF_K3) X(CQW, WRF_K3) \
  X(ALT, WRF_K3) X(PHP, WRF_K3) X(RU_TENDF, WRF_K3) X(RV_TENDF, WRF_K3) X(RW_TENDF, WRF_K3) \
  X(PH_TENDF, WRF_K3) X(T_TENDF, WRF_K3) X(RU_TEND, WRF_K3) X(RV_TEND, WRF_K3) X(RW_TEND, WRF_K3) \
  X(PH_TEND, WRF_K3) X(T_TEND, WRF_K3) X(U_SAVE, WRF_K3) X(V_SAVE, WRF_K3) X(W_SAVE, WRF_K3) \
  X(PH_SAVE, WRF_K3) X(T_SAVE, WRF_K3) X(RDZW, WRF_K3) X(ZX, WRF_K3) X(ZY, WRF_K3) \
  X(DEFOR11, WRF_K3) X(DEFOR22, WRF_K3) X(DEFOR12, WRF_K3) X(XKMH, WRF_K3) X(XKHH, WRF_K3) \
  X(U_1, WRF_K3) X(V_1, WRF_K3) X(W_1, WRF_K3) X(T_1, WRF_K3) X(PH_1, WRF_K3) X(C2A, WRF_K3) \
  X(PM1, WRF_K3) X(A, WRF_K3) X(ALPHA, WRF_K3) X(GAMMA, WRF_K3) X(RU_M, WRF_K3) X(RV_M, WRF_K3) \
  X(WW_M, WRF_K3) X(T_2SAVE, WRF_K3) X(H_DIABATIC, WRF_K3) X(QV_DIABATIC, WRF_K3) \
  X(QC_DIABATIC, WRF_K3) X(WSM_T, WRF_K3) X(WSM_QR0S, WRF_K3) \
  X(MU, WRF_K2) X(MUB, WRF_K2) X(MSFU, WRF_K2) X(MSFV, WRF_K2) X(MSFVX_INV, WRF_K2) \
  X(MSFT, WRF_K2) X(MSFTX, WRF_K2) X(MSFTY, WRF_K2) X(MSFUX, WRF_K2) X(MSFUY, WRF_K2) \
  X(MSFVX, WRF_K2) X(MSFVY, WRF_K2) X(F, WRF_K2) X(E, WRF_K2) X(SINA, WRF_K2) X(COSA, WRF_K2) \
  X(HT, WRF_K2) X(RAINNC, WRF_K2) X(RAINNCV, WRF_K2) X(SNOWNC, WRF_K2) X(SNOWNCV, WRF_K2) \
  X(GRAUPELNC, WRF_K2) X(GRAUPELNCV, WRF_K2) X(SR, WRF_K2) X(MUT, WRF_K2) X(MUU, WRF_K2) \
  X(MUV, WRF_K2) X(MU_TENDF, WRF_K2) X(MU_TEND, WRF_K2) X(MU_SAVE, WRF_K2) X(MU_1, WRF_K2) \
  X(MUUS, WRF_K2) X(MUVS, WRF_K2) X(MUTS, WRF_K2) X(MUDF, WRF_K2) X(MUAVE, WRF_K2) \
  X(RDNW, WRF_K1) X(RDN, WRF_K1) X(C1H, WRF_K1) X(FNM, WRF_K1) X(FNP, WRF_K1) X(DN, WRF_K1) \
  X(DNW, WRF_K1) \
  X(MOIST, WRF_K4) X(MOIST_TEND, WRF_K4) X(ADVECT_TEND, WRF_K4) X(MOIST_OLD, WRF_K4) \
  X(U_BXS, WRF_KBX) X(U_BXE, WRF_KBX) X(U_BYS, WRF_KBY) X(U_BYE, WRF_KBY) \
  X(U_BTXS, WRF_KBX) X(U_BTXE, WRF_KBX) X(U_BTYS, WRF_KBY) X(U_BTYE, WRF_KBY) \
  X(V_BXS, WRF_KBX) X(V_BXE, WRF_KBX) X(V_BYS, WRF_KBY) X(V_BYE, WRF_KBY) \
  X(V_BTXS, WRF_KBX) X(V_BTXE, WRF_KBX) X(V_BTYS, WRF_KBY) X(V_BTYE, WRF_KBY) \
  X(PH_BXS, WRF_KBX) X(PH_BXE, WRF_KBX) X(PH_BYS, WRF_KBY) X(PH_BYE, WRF_KBY) \
  X(PH_BTXS, WRF_KBX) X(PH_BTXE, WRF_KBX) X(PH_BTYS, WRF_KBY) X(PH_BTYE, WRF_KBY) \
  X(T_BXS, WRF_KBX) X(T_BXE, WRF_KBX) X(T_BYS, WRF_KBY) X(T_BYE, WRF_KBY) \
  X(T_BTXS, WRF_KBX) X(T_BTXE, WRF_KBX) X(T_BTYS, WRF_KBY) X(T_BTYE, WRF_KBY) \
  X(MU_BXS, WRF_KBX2) X(MU_BXE, WRF_KBX2) X(MU_BYS, WRF_KBY2) X(MU_BYE, WRF_KBY2) \
  X(MU_BTXS, WRF_KBX2) X(MU_BTXE, WRF_KBX2) X(MU_BTYS, WRF_KBY2) X(MU_BTYE, WRF_KBY2) \
  X(QV_BXS, WRF_KBX) X(QV_BXE, WRF_KBX) X(QV_BYS, WRF_KBY) X(QV_BYE, WRF_KBY) \
  X(QV_BTXS, WRF_KBX) X(QV_BTXE, WRF_KBX) X(QV_BTYS, WRF_KBY) X(QV_BTYE, WRF_KBY) \
  X(DSCAL, WRF_KSF) X(STATUS, WRF_KSI)

#define WRF_ENUM_ENTRY(name, kind) WF_##name,
enum WrfFieldId { WRF_FIELD_TABLE(WRF_ENUM_ENTRY) WF_COUNT };
#undef WRF_ENUM_ENTRY

/* Grid, time step and the scalar coefficients read from the input file
 * (CF1..CFN1, pywrf/solver.py:267-271).  Index bounds follow the reference's
 * python-style WRF index sets. */
typedef struct WrfGrid {
  int nx, ny, nz;
  int ids, ide, jds, jde;
  int soundsteps;
  int spec_zone;
  int bdy_interval;
  int top_lid;
  float dx, dy, dt;
  float smdiv, emdiv, epssm, khdif, kvdif;
  float cf1, cf2, cf3, cfn, cfn1;
} WrfGrid;

/* device pointers of every state field, indexed by WrfFieldId */
typedef struct WrfState {
  void* f[WF_COUNT];
} WrfState;

/* optional host callback invoked after each phase of wrf_rk3_step (the
 * stream is not synchronised by the library; the callback may do so) */
typedef void (*wrf_probe_fn)(const char* phase, void* user);

/* table introspection (names are the lower-case reference variable names) */
int wrf_field_count(void);
const char* wrf_field_name(int id);
int wrf_field_kind(int id);
const char* wrf_last_error(void);

/* Replaces one time step of WrfSolver.solve (pywrf/solver.py:709-1910): the
 * three RK stages with their acoustic substeps, moisture transport, WSM6 and
 * the end-of-step lateral-boundary updates.  The step number used for the
 * boundary time (solver.py:713) is the device counter STATUS[WRF_ST_STEP]+1,
 * so the call can be captured once in a CUDA graph and replayed. */
int wrf_rk3_step(const WrfGrid* g, const WrfState* s, void* stream, wrf_probe_fn probe, void* user);

/* The same step one phase at a time, for a caller that drives the RK3 loop
 * itself as WrfSolver.solve does (pywrf/solver.py:709-1910).  Calling, in
 * this order,
 *   wrf_step_begin;
 *   for rk_step = 1, 2, 3:
 *     wrf_rk_prep(rk_step); if rk_step == 1: wrf_diff_stage1;
 *     wrf_tend_stage(rk_step); wrf_acoustic_prep(rk_step);
 *     for iteration = 1 .. nsub: wrf_acoustic_substep(rk_step, iteration)
 *       (nsub = 1, soundsteps / 2, soundsteps for rk_step 1, 2, 3);
 *     wrf_acoustic_finish(rk_step); wrf_moist_stage(rk_step);
 *   wrf_microphysics; wrf_step_end
 * enqueues exactly the kernels of one wrf_rk3_step.  The phases:
 *   step_begin        boundary time of the step (solver.py:713-718)
 *   rk_prep           rk_step_prep and its halo copies (solver.py:736-778)
 *   diff_stage1       first stage only: physics tendencies zeroed, diffusion
 *                     metrics, deformation, eddy viscosities (solver.py:880-985)
 *   tend_stage        advection, pressure gradient, buoyancy, Coriolis,
 *                     curvature; first-stage horizontal diffusion and
 *                     relaxation; rk_addtend_dry (solver.py:987-1256)
 *   acoustic_prep     small_step_prep, calc_p_rho, calc_coef_w (solver.py:1258-1345)
 *   acoustic_substep  advance_uv, advance_mu_t, advance_w, sumflux,
 *                     calc_p_rho, lateral updates (solver.py:1350-1492)
 *   acoustic_finish   small_step_finish (solver.py:1494-1546)
 *   moist_stage       moisture transport and update (solver.py:1548-1710)
 *   microphysics      WSM6 and calc_p_rho_phi (solver.py:1714-1766)
 *   step_end          end-of-step lateral boundaries (solver.py:1776-1910)
 * rk_step outside 1..3 or an iteration outside 1..nsub is WRF_EINVAL. */
int wrf_step_begin(const WrfGrid* g, const WrfState* s, void* stream);
int wrf_rk_prep(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
int wrf_diff_stage1(const WrfGrid* g, const WrfState* s, void* stream);
int wrf_tend_stage(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
int wrf_acoustic_prep(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
int wrf_acoustic_substep(const WrfGrid* g, const WrfState* s, int rk_step, int iteration, void* stream);
int wrf_acoustic_finish(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
int wrf_moist_stage(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
int wrf_microphysics(const WrfGrid* g, const WrfState* s, void* stream);
int wrf_step_end(const WrfGrid* g, const WrfState* s, void* stream);

/* Reference function-level entry points (same arguments as the step
 * driver; each runs exactly the reference function named). */
/* wrf_dynamics.py:1841-2028 advect_scalar: tend += flux-form advection of field */
int wrf_advect_scalar(const WrfGrid* g, const float* field, float* tend, const float* ru,
                      const float* rv, const float* rom, const float* msftx, const float* fzm,
                      const float* fzp, const float* rdzw, void* stream);
/* wrf_dynamics.py:1112-1331 advect_u, 1332-1534 advect_v, 1535-1823
 * advect_w: tend += the flux-form advection of one momentum component
 * (component 0: field = u, msf = msfux; 1: field = v, msf = msfvy,
 * msf2 = msfvx; 2: field = w, msf = msftx), with the coupled velocities ru,
 * rv, rom, the profiles fzm, fzp and rdz (rdnw for u and v, rdn for w).
 * form 0 runs the fastest kernel the arrays allow (the tiled tensor-map
 * kernel when nx is a multiple of 4 and the arrays are 16-byte aligned),
 * form 1 the one-thread-per-point kernel; both perform the reference's
 * operations in the reference's order. */
int wrf_advect_momentum(const WrfGrid* g, int component, const float* field, float* tend, const float* ru,
                        const float* rv, const float* rom, const float* msf, const float* msf2, const float* fzm,
                        const float* fzp, const float* rdz, int form, void* stream);
/* Adjoint of wrf_advect_scalar (reverse mode): given the cotangent tend_bar of
 * the updated tendency, accumulates (+=) the cotangents of field, ru, rv and
 * rom.  The cotangent of the incoming tendency is tend_bar itself.  The
 * reference obtains this product from torch autograd through
 * wrf_dynamics.py:1841-2028.  work: device scratch of at least
 * wrf_advect_scalar_adj_work floats (work_floats, checked). */
int wrf_advect_scalar_adj(const WrfGrid* g, const float* field, const float* ru, const float* rv,
                          const float* rom, const float* msftx, const float* fzm, const float* fzp,
                          const float* rdzw, const float* tend_bar, float* field_bar, float* ru_bar,
                          float* rv_bar, float* rom_bar, float* work, size_t work_floats, void* stream);
/* The number of floats of work wrf_advect_scalar_adj needs for the grid. */
int wrf_advect_scalar_adj_work(const WrfGrid* g, size_t* floats);
/* wrf_dynamics.py:2031-2620 the large-step tendency terms selected by the
 * mask `terms` (1 rhs_ph, 2 horizontal_pressure_gradient, 4 pg_buoy_w, 8
 * coriolis, 16 curvature) on the state table, with the solver's arguments:
 * adds to ph_tend, ru_tend, rv_tend, rw_tend; pg_buoy_w also replaces cqw by
 * 1 / (1 + cqw) on levels 1 .. nz-2 of the mass points (wrf_dynamics.py:2453).
 * The step itself runs these terms fused in one tiled kernel. */
int wrf_forces(const WrfGrid* g, const WrfState* s, int terms, void* stream);
/* Its adjoint: sbar's PH_TEND, RU_TEND, RV_TEND, RW_TEND and CQW hold the
 * cotangents of the updated fields and are rewritten to those of the inputs
 * (the tendencies' pass through, except ph_tend's top level, which rhs_ph
 * sets); the cotangents of u, v, w, ww, ph, phb, mut, muu, muv, alt, p, pb,
 * al, php, cqu, cqv, mu, mub, ru, rv and rw are accumulated (+=), all
 * required.  Accumulation order is not fixed (atomic adds). */
int wrf_forces_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int terms, void* stream);
/* wrf_dynamics.py:3799-3839 sumflux on the state table, with the solver's
 * arguments: u, v, ww, u_save, v_save, ww1, muu, muv, msfuy, msfvx_inv;
 * updates ru_m, rv_m, ww_m (zeroed first at iteration 1, averaged at
 * iteration nsub).  The step fuses it into its acoustic column kernel. */
int wrf_sumflux(const WrfGrid* g, const WrfState* s, int iteration, int nsub, void* stream);
/* Its adjoint: sbar's RU_M, RV_M, WW_M hold the cotangents of the updated
 * sums and are rewritten to those of the incoming sums; those of u, v, ww,
 * u_save, v_save, ww1, muu, muv are accumulated (+=). */
int wrf_sumflux_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int iteration, int nsub,
                    void* stream);
/* wrf_boundary.py:244-294 spec_bdyupdate: field += dt * tend on the
 * specified rows of stagger var ('t', 'u', 'v': [nz][ny][nx] fields, levels
 * below nz-1; 'm': [ny][nx]). */
int wrf_spec_bdyupdate(const WrfGrid* g, float* field, const float* tend, float dt, char var, void* stream);
/* Its adjoint: tend_bar += dt * field_bar on those rows (the field's own
 * cotangent passes through). */
int wrf_spec_bdyupdate_adj(const WrfGrid* g, const float* field_bar, float* tend_bar, float dt, char var,
                           void* stream);
/* wrf_boundary.py:297-355 spec_bdyupdate_ph on the state table (ph, ph_save,
 * ph_tend, mu_tend, muts): the specified rows of ph with the mass
 * re-weighting mu_old = muts - dt * mu_tend, all levels. */
int wrf_spec_bdyupdate_ph(const WrfGrid* g, const WrfState* s, float dt, void* stream);
/* Its adjoint: sbar's PH holds the cotangent of the updated ph and is
 * rewritten to that of the incoming ph; those of ph_save, ph_tend, mu_tend
 * and muts are accumulated (+=). */
int wrf_spec_bdyupdate_ph_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float dt, void* stream);
/* wrf_dynamics.py:30-159 rk_step_prep's functions selected by the mask ops
 * (1 calculate_full, 2 calc_mu_uv, 4 couple_momentum, 8 calc_ww_cp, 16
 * calc_cq, 32 calc_alt, 64 calc_php), in that order, on the state table with
 * the solver's arguments (couple_momentum divides by msfu and msft, calc_cq
 * sums all seven moisture slots; c1h, dnw, msftx, msfuy, msfvx_inv).  The
 * step computes them fused in its prep kernels. */
int wrf_prep(const WrfGrid* g, const WrfState* s, int ops, void* stream);
/* Its adjoint: the cotangents of the outputs (mut, muu, muv, ru, rv, rw,
 * ww levels 1 .. nz-2, cqu, cqv, cqw, alt, php) are read on each function's
 * region and set to zero there (the functions overwrite them); those of the
 * inputs (mu, mub, u, v, w, ww level 0, moist, al, alb, ph, phb, and muu,
 * muv, mut where a later function reads them) are accumulated (+=). */
int wrf_prep_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int ops, void* stream);
/* wrf_dynamics.py:164-278 set_physical_bc3d (two_d 0, [nz][ny][nx]) /
 * set_physical_bc2d (two_d 1, [ny][nx]) of one field for the stagger letter
 * var, in place: the reference's open-boundary halo copies, x sides first. */
int wrf_halo(const WrfGrid* g, float* field, char var, int two_d, void* stream);
/* Its adjoint: the cotangent of the copied field is added (+=) into in_bar,
 * the cotangent of the field before the copies (a separate array). */
int wrf_halo_adj(const WrfGrid* g, const float* field_bar, float* in_bar, char var, int two_d, void* stream);
/* wrf_boundary.py:358-400 zero_grad_bdy of w (all levels), in place. */
int wrf_zero_grad_w(const WrfGrid* g, float* w, void* stream);
/* Its adjoint: w_bar is added (+=) into in_bar (a separate array). */
int wrf_zero_grad_w_adj(const WrfGrid* g, const float* w_bar, float* in_bar, void* stream);
/* wrf_dynamics.py:3152-3266 small_step_prep on the state table (without the
 * calc_p_rho / calc_coef_w the step runs after it): mu_1, muts, muus, muvs,
 * mu_save, mu, the _1 and _save copies, the perturbation forms of u, v, t,
 * w, ph, c2a and ww1, at RK stage rk_step. */
int wrf_small_step_prep(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
/* Its adjoint: sbar holds the cotangents of the updated fields and is
 * rewritten to those of the incoming state (overwritten fields get zero);
 * work: caller-owned scratch of 3 * ny * nx floats (the column masses the
 * forward formed). */
int wrf_small_step_prep_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int rk_step, float* work,
                            void* stream);
/* wrf_dynamics.py:3844-3930 calc_mu_uv_1 then small_step_finish on the state
 * table (back from the perturbation form; h_diabatic enters at rk_step 3). */
int wrf_small_step_finish(const WrfGrid* g, const WrfState* s, float dts, int nsub, int rk_step, void* stream);
/* Its adjoint: as wrf_small_step_prep_adj; work: 2 * ny * nx floats. */
int wrf_small_step_finish_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float dts, int nsub,
                              int rk_step, float* work, void* stream);
/* wrf_dynamics.py:3100-3148 rk_addtend_dry on the state table: at rk_step 1
 * the physics tendencies take the saved fields first; every stage adds them
 * (divided by the map factor) to ru/rv/rw/ph/t_tend, theta also mut
 * h_diabatic / msfty, and mu_tend += mu_tendf. */
int wrf_addtend(const WrfGrid* g, const WrfState* s, int rk_step, void* stream);
/* Its adjoint: the tendencies' cotangents pass through; those of the
 * updated physics tendencies are rewritten to the incoming ones'; the saved
 * fields, mut and h_diabatic accumulate (+=). */
int wrf_addtend_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int rk_step, void* stream);
/* wrf_boundary.py:189-241 spec_bdytend: the specified rows of tend take the
 * boundary tendency (x sides [nk][ny][5], y sides [nk][5][nx]; var 'u', 'v',
 * 't' below level nz-1, 'h' all levels, 'm' 2-D). */
int wrf_spec_bdytend(const WrfGrid* g, float* tend, const float* txs, const float* txe, const float* tys,
                     const float* tye, char var, void* stream);
/* Its adjoint: sets those rows of tend_bar to zero (in place). */
int wrf_spec_bdytend_adj(const WrfGrid* g, float* tend_bar, char var, void* stream);
/* wrf_dynamics.py:491-536, 539-813, 816-995 the first stage's eddy
 * viscosities on the state table: compute_diff_metrics (rdzw, zx, zy from
 * ph, phb) with their halo copies, cal_deform_and_div's defor11, defor22,
 * defor12 (from u, v) and the 2-D Smagorinsky calculate_km_kh (xkmh, xkhh);
 * rdzw, zx, zy and the defor fields are scratch the call overwrites. */
int wrf_eddy_viscosity(const WrfGrid* g, const WrfState* s, void* stream);
/* Its adjoint: the cotangents of xkmh and xkhh are rewritten to those of
 * their incoming values (which reach the output only where the region's
 * formula does not apply); u, v and ph accumulate.  The scratch fields are
 * recomputed from s; work: 6 * nz * ny * nx floats. */
int wrf_eddy_viscosity_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float* work, void* stream);
/* wrf_dynamics.py:2623-2838 horizontal_diffusion of u ('u'), v ('v'), w
 * ('w') or a mass-point scalar ('m'; with base, horizontal_diffusion_3dmp at
 * :2841-2915, the diffusion of field - base): tend += the diffusion of
 * field with column mass mut and eddy viscosity xk; s supplies the map
 * factors (msfux, msfuy, msfvx, msfvy, msftx, msfty, msfvx_inv). */
int wrf_horizontal_diffusion(const WrfGrid* g, const WrfState* s, char var, const float* field, const float* base,
                             const float* mut, const float* xk, float* tend, void* stream);
/* Its adjoint: field_bar, mut_bar and xk_bar accumulate (each may be null
 * when not wanted; they must not overlap each other, tend_bar or the
 * operands); tend_bar passes through unchanged. */
int wrf_horizontal_diffusion_adj(const WrfGrid* g, const WrfState* s, char var, const float* field,
                                 const float* base, const float* mut, const float* xk, const float* tend_bar,
                                 float* field_bar, float* mut_bar, float* xk_bar, void* stream);
/* wrf_boundary.py:408-414 mass_weight: out = field * mut on levels below nk
 * of the mass points (other points of out are left as they are). */
int wrf_mass_weight(const WrfGrid* g, const float* field, const float* mut, float* out, int nk, void* stream);
/* Its adjoint: field_bar and mut_bar accumulate. */
int wrf_mass_weight_adj(const WrfGrid* g, const float* field, const float* mut, const float* out_bar,
                        float* field_bar, float* mut_bar, int nk, void* stream);
/* wrf_boundary.py:511-587, wrf_dynamics.py:4218-4324 the end-of-step
 * lateral boundaries on the state table: spec_bdy_final of u, v, t, ph and
 * qv (the specified rows take msf (bdy + dtbc bdy_tend) / mu with mu = muus,
 * muvs or muts; dtbc is DSCAL[0]) then set_w_surface (w at the lowest
 * level from the lowest three levels of u and v and the terrain ht). */
int wrf_bdy_final(const WrfGrid* g, const WrfState* s, void* stream);
/* Its adjoint: the cotangents of u, v, t, ph, qv and w are rewritten to
 * those of their incoming values; muus, muvs and muts accumulate (the
 * boundary arrays and ht are data). */
int wrf_bdy_final_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, void* stream);
/* solver.py:1714-1766 the step's microphysics on the state table:
 * moist_physics_prep_em, wsm6 on the solver's column block,
 * moist_physics_finish_em and calc_p_rho_phi (wrf_physics.py:27-91,
 * 137-1214, 2106-2137; wrf_dynamics.py:4124-4164).  The table needs t,
 * moist, al, alb, p, pb, ph, phb, mu, muts, rdnw, h_diabatic, qv_diabatic,
 * qc_diabatic, the precipitation accumulators and the wsm_t / wsm_qr0s
 * scratch; the grid's dt is the step's. */
int wrf_microphysics_op(const WrfGrid* g, const WrfState* s, void* stream);
/* The number of floats of work wrf_microphysics_adj needs for the grid. */
int wrf_microphysics_adj_work(const WrfGrid* g, size_t* floats);
/* Its adjoint.  s holds the block's inputs (t, moist, al, alb, p, pb, ph,
 * phb, mu, muts, rdnw), post the same fields after the block; sbar the
 * cotangents of the outputs t, moist, al, p and h_diabatic, rewritten to
 * those of the inputs, while ph, mu, muts, alb and pb accumulate.  The
 * equation of state is reversed exactly; prep + WSM6 + finish by reverse
 * mode over a per-column restatement of the scheme (the derivative of the
 * branch taken): each column runs once on taped scalars and one reverse
 * sweep of its tape gives its inputs' cotangents; a column whose tape
 * outgrows the capacity takes forward-mode tangents of the same
 * restatement instead.  values (optional: t, moist, h_diabatic) receives
 * that restatement's own outputs, for checking it against the forward. */
int wrf_microphysics_adj(const WrfGrid* g, const WrfState* s, const WrfState* post, const WrfState* sbar,
                         float* work, size_t work_floats, const WrfState* values, void* stream);
/* The tape capacity of wrf_microphysics_adj in entries per column, for the
 * whole library (0 restores the default, 480 entries per level plus the
 * inputs, at most 65535); *previous (optional) receives the setting it
 * replaces.  A capacity below the column's input count sends every column
 * to the tangents.  Call wrf_microphysics_adj_work again after changing
 * it. */
int wrf_set_microphysics_tape_capacity(int entries, int* previous);
/* wrf_dynamics.py:4124-4164 calc_p_rho_phi on the state table: al and p on
 * the mass points below the top level from ph, t, qv (moist slot 1), alb,
 * pb, mu, muts, rdnw; NaN in p is counted in the status words. */
int wrf_calc_p_rho_phi(const WrfGrid* g, const WrfState* s, void* stream);
/* wrf_dynamics.py:4055-4164, wrf_boundary.py:470-508 the moisture update of
 * an RK stage on the state table: rk_update_scalar of qv .. qg (moist_old,
 * moist_tend, advect_tend, mu_1, mu, mub, msfty), flow_dep_bdy of qc .. qg
 * (ru_m, rv_m) and calc_p_rho_phi (al, p from ph, t, qv, alb, pb, mu, muts);
 * NaN in the diagnosed p is counted in the status words. */
int wrf_moist_update(const WrfGrid* g, const WrfState* s, int rk_step, float dt_rk, void* stream);
/* Its adjoint: the cotangents of moist (and at rk_step 1 moist_old), al and
 * p are rewritten to those of the incoming values; those of moist_tend,
 * advect_tend, mu_1, mu, mub, alb, muts, ph, pb, t (and moist_old after the
 * first stage) are accumulated; work: nz * ny * nx floats. */
int wrf_moist_update_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int rk_step, float dt_rk,
                         float* work, void* stream);
/* wrf_dynamics.py:3391-3525 advance_uv followed by spec_bdyupdate of u and
 * v (wrf_boundary.py:244-290), as the acoustic substep calls them
 * (solver.py:1350-1377): u and v of the state table are updated in place
 * from the table's ru_tend, rv_tend, p, pb, ph, php, alt, al, mu, muu, muv,
 * cqu, cqv, mudf, msfux, msfuy, msfvx, msfvx_inv, msfvy, fnm, fnp, rdnw and
 * the grid's emdiv, cf1..cf3 (spec_zone 1); fields it does not read may be
 * null.  Runs the kernel of the form wrf_set_kernel_form selects. */
int wrf_advance_uv(const WrfGrid* g, const WrfState* s, float dts, void* stream);
/* Its adjoint (reverse mode): sbar holds, under the same field ids, the
 * cotangents of the updated u and v (which are also those of the incoming
 * u and v: du'/du = 1) and accumulates (+=) those of ru_tend, rv_tend, p, pb,
 * ph, php, alt, al, mu, muu, muv, cqu, cqv and mudf, all required.  The
 * reference's autograd cannot differentiate advance_uv (an in-place update
 * of a saved operand), so the product is checked against finite differences
 * of its forward. */
int wrf_advance_uv_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float dts, void* stream);
/* wrf_dynamics.py:3641-3796 advance_w on the state table, in place, with
 * the solver's arguments: w, rw_tend, ww, w_save, u, v, muave, muts, mut,
 * t_2ave (T_2SAVE), t_2 (T), t_1 (T_SAVE), ph, ph_1 (PH_SAVE), phb, ph_tend,
 * ht, c2a, cqw, alt, a, alpha, gamma, msftx, msfty, fnm, fnp, rdnw, rdn and
 * the grid's epssm, cf1..cf3 (top_lid 0); updates t_2save, w and ph. */
int wrf_advance_w(const WrfGrid* g, const WrfState* s, float dts, void* stream);
/* Its adjoint: sbar's W, PH, T_2SAVE hold the cotangents of the updated
 * fields and are rewritten to those of the inputs; those of the other 20
 * operands above (u, v, ht included, through the lower boundary) are
 * accumulated (+=).  work: caller-owned scratch of ny*nx floats.  The
 * reference's autograd cannot run backward through its in-place sweeps. */
int wrf_advance_w_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float dts, float* work,
                      void* stream);
/* wrf_dynamics.py:3528-3638 advance_mu_t on the state table, in place, with
 * the solver's arguments (solver.py:1380-1393): ww (WW), ww_1 (WW1), u,
 * u_1 (U_SAVE), v, v_1 (V_SAVE), mu, mut, muave, muts, muu, muv, mudf, t,
 * t_1 (T_SAVE), t_ave (T_2SAVE), ft (T_TEND), mu_tend and the profiles dnw,
 * fnm, fnp, rdnw and map factors msfuy, msfvx_inv, msftx, msfty, with the
 * grid's epssm; updates ww, t, t_2save, mu, muts, mudf and muave. */
int wrf_advance_mu_t(const WrfGrid* g, const WrfState* s, float dts, void* stream);
/* Its adjoint: sbar holds, under the same ids, the cotangents of the seven
 * updated fields (rewritten to those of the inputs of the same name) and
 * accumulates (+=) those of ww_1, u, u_1, v, v_1, mut, muu, muv, t_1, ft,
 * mu_tend.  work: caller-owned scratch of nz*ny*nx floats.  ref_no_grad != 0
 * reproduces the reference's autograd, which runs the mu / muts / mudf /
 * muave update under torch.no_grad() (wrf_dynamics.py:3597-3604): those
 * four outputs then pass their cotangents to the inputs of the same name and
 * nothing else; ref_no_grad = 0 gives the derivative of the operator. */
int wrf_advance_mu_t_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, float dts,
                         int ref_no_grad, float* work, void* stream);
/* wrf_dynamics.py:3269-3313 calc_p_rho on the state table, in place: al, p
 * and pm1 from ph, alt, t_2 (field T), t_1 (T_SAVE), c2a, mu, mut (MUTS)
 * and rdnw, with the grid's smdiv; step 0 sets pm1 to a copy of the whole
 * new p, a later step applies the divergence damping p += smdiv (p - pm1)
 * and keeps the undamped p in pm1 (the acoustic substep's use). */
int wrf_calc_p_rho(const WrfGrid* g, const WrfState* s, int step, void* stream);
/* Its adjoint: sbar's AL, P, PM1 hold the cotangents of the updated al, p,
 * pm1 and are rewritten to those of the incoming al, p, pm1; the cotangents
 * of ph, alt, T, T_SAVE, c2a (3-D) and mu, MUTS (2-D) are accumulated (+=).
 * The reference obtains this product from torch autograd through
 * wrf_dynamics.py:3269-3313. */
int wrf_calc_p_rho_adj(const WrfGrid* g, const WrfState* s, const WrfState* sbar, int step, void* stream);
/* Adjoint of wrf_advect_momentum (reverse mode): given the cotangent tend_bar
 * of the updated tendency, accumulates (+=) the cotangents of the advected
 * component (field) and of ru, rv and rom; the arguments are those of
 * wrf_advect_momentum.  The reference obtains this product from torch
 * autograd through wrf_dynamics.py:1112-1331 (advect_u) and 1332-1534
 * (advect_v); its advect_w (1535-1823) cannot be differentiated by its
 * autograd (an in-place update of a saved operand), the product is the
 * same transpose of the linearised operator.  work: device scratch of at
 * least wrf_advect_momentum_adj_work floats (work_floats, checked). */
int wrf_advect_momentum_adj(const WrfGrid* g, int component, const float* field, const float* ru,
                            const float* rv, const float* rom, const float* msf, const float* msf2,
                            const float* fzm, const float* fzp, const float* rdz, const float* tend_bar,
                            float* field_bar, float* ru_bar, float* rv_bar, float* rom_bar, float* work,
                            size_t work_floats, void* stream);
/* The number of floats of work wrf_advect_momentum_adj needs for the grid. */
int wrf_advect_momentum_adj_work(const WrfGrid* g, size_t* floats);
/* wrf_boundary.py:52-147 relax_bdytend on one field: tend += the relaxation
 * toward bdy + dtbc * bdy_tend over the zone rows 1..3.  bdy8: device arrays
 * xs xe ys ye (values) and txs txe tys tye (tendencies) in the solver's
 * permuted layout ([nz][ny][5] and [nz][5][nx]); variable: the reference's
 * stagger letter ('u', 'v', 'h' for all nz levels, 'm' for the 2-D mu
 * (one level), else nz - 1), with the weights fcx / gcx the solver passes
 * (solver.py:440-441). */
int wrf_relax_bdytend(const WrfGrid* g, const float* field, float* tend, const float* const* bdy8,
                      char variable, float dtbc, void* stream);
/* its adjoint w.r.t. the field: field_bar += d(tend)/d(field)^T tend_bar (the
 * operator is linear in the field; no counterpart in the reference, which
 * gets it from torch autograd) */
int wrf_relax_bdytend_adj(const WrfGrid* g, const float* tend_bar, float* field_bar, char variable,
                          void* stream);
/* The vertically implicit w solve of advance_w (wrf_dynamics.py:3761-3767)
 * on ncol columns of nz levels ([nz][ncol] arrays, any column stride folded
 * into ncol): forward sweep w(k) = (x(k) - a(k) w(k-1)) alpha(k), then
 * w(k) -= gamma(k) w(k+1); w(0) = x(0).  The reference runs it inline. */
int wrf_vsolve_w(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                 float* w, void* stream);
/* its adjoint (the transposed solve and the coefficient cotangents):
 * accumulates (+=) into x_bar, a_bar, alpha_bar, gamma_bar given w_bar */
int wrf_vsolve_w_adj(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                     const float* w_bar, float* x_bar, float* a_bar, float* alpha_bar, float* gamma_bar,
                     void* stream);
/* wrf_dynamics.py:3316-3388 calc_coef_w on the mass columns [ids, ide-1) x
 * [jds, jde-1): the tridiagonal coefficients a, alpha, gamma of the implicit
 * w solve from mut (2-D), cqw, c2a (3-D), rdn, rdnw (profiles); epssm and
 * top_lid from the grid */
int wrf_coef_w(const WrfGrid* g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
               const float* rdnw, float dts, float* a, float* alpha, float* gamma, void* stream);
/* its adjoint w.r.t. mut, cqw and c2a (accumulates into the *_bar outputs,
 * which must not overlap the inputs or each other); the reference obtains
 * it from torch autograd */
int wrf_coef_w_adj(const WrfGrid* g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                   const float* rdnw, float dts, const float* a_bar, const float* alpha_bar,
                   const float* gamma_bar, float* mut_bar, float* cqw_bar, float* c2a_bar, void* stream);
/* wrf_physics.py:94-136 microphysics_driver -> wsm6 on the solver's column block */
int wrf_wsm6(const WrfGrid* g, float* th, float* qv, float* qc, float* qr, float* qi, float* qs,
             float* qg, const float* rho, const float* pii, const float* p, const float* dz8w,
             float delt, float* rainnc, float* rainncv, float* snownc, float* snowncv,
             float* graupelnc, float* graupelncv, float* sr, void* stream);

/* wrf_wsm6's computation without caller scratch and without any device
 * allocation; no counterpart in the reference.  For callers that pass only
 * the scheme's own arrays and must not allocate device memory themselves:
 * its two intermediate fields live in a fixed file-scope device array of
 * 2 x 2,097,152 floats (16 MiB), enough for the block of a 240x240x41 grid.
 * Larger blocks, and delt >= 240 s (two time-split loops), return WRF_EINVAL.
 * The first call in each CUDA context looks up the array's address (make it
 * before any stream capture on that device; after a device reset the next
 * call looks it up again); calls that overlap on the GPU share the array and
 * race. */
int wrf_wsm6_noalloc(const WrfGrid* g, float* th, float* qv, float* qc, float* qr, float* qi, float* qs,
                     float* qg, const float* rho, const float* pii, const float* p, const float* dz8w,
                     float delt, float* rainnc, float* rainncv, float* snownc, float* snowncv,
                     float* graupelnc, float* graupelncv, float* sr, void* stream);

/* copies the 16 device status words to host memory (synchronises the stream) */
int wrf_status_read(const WrfState* s, void* stream, int* out16);

/* number of kernels the calling thread's last wrf_rk3_step enqueued (the
 * reference has no counterpart; used to report launch counts) */
int wrf_last_launch_count(void);

/* Kernel forms for cross-checks (process-wide; no counterpart in the
 * reference).  WRF_FORM_FAST (the default) runs the tiled tensor-map kernels
 * where the arrays allow them, and the boundary relaxation over the boundary
 * band only; WRF_FORM_POINT runs, for the same launches, the
 * one-thread-per-point (momentum advection, advance_uv, forces) and
 * cp.async-tiled (scalar advection) kernels and the relaxation over every
 * point.  Both forms perform the reference's operations
 * in the same order and give bit-identical results.  A CUDA graph keeps the
 * form that was set when it was captured.  Returns the previous form, or
 * WRF_EINVAL for an unknown one. */
#define WRF_FORM_FAST 0
#define WRF_FORM_POINT 1
int wrf_set_kernel_form(int form);

/* ------------------------------------------------------------------------
 * Per-column microphysics network: a learned stand-in for wsm6
 * (pywrf/wrf_physics.py:137-1214).  The reference has no counterpart of
 * anything below; the layout of the network's rows is given by
 * wrf_mlp_layout.  A column is a mass column of the WSM6 block
 * (i in [ids+1, ide-2), j in [jds+1, jde-2)), numbered
 * (j - jds - 1) * ncx + (i - ids - 1).
 * ------------------------------------------------------------------------ */
#define WRF_MLP_LAYERS 4

typedef struct WrfMlpNet {
  int dims[WRF_MLP_LAYERS + 1];    /* widths: d0 (input), hidden x 3, d4 (output) */
  const void* w[WRF_MLP_LAYERS];   /* bf16 [dims[l+1]][dims[l]] */
  const float* b[WRF_MLP_LAYERS];  /* fp32 [dims[l+1]] */
  const float* norm;               /* fp32 [2 d0 + 2 d4]: input mean, input 1/std, output mean, output std */
  float tol_neg;                   /* gate: a species below -tol_neg (kg/kg) before clipping rejects the column */
  float tol_sat;                   /* gate: qv above (1 + tol_sat) x saturation over water rejects the column */
} WrfMlpNet;

typedef struct WrfMlpWork {        /* caller-owned device scratch of one surrogate call */
  int capacity;                    /* columns the buffers hold (>= ncols) */
  void* x;                         /* bf16 [capacity][d0] */
  void* h[2];                      /* bf16 [capacity][max hidden width] */
  float* y;                        /* fp32 [capacity][d4] */
  int* list;                       /* int [16 + capacity]: [0] rejected columns, [1] quiet columns (no
                                      condensate, subsaturated: zero increments without the network),
                                      [2] [3] [4] rejections for positivity / supersaturation / a non-finite
                                      output, [16..] the rejected columns' j * nx + i */
  int* err;                        /* int: set to 1 if a tensor-core kernel's bounded wait ran out */
  void* colstat;                   /* optional uint8 [capacity]: 0 network, 1 quiet, 2 rejected */
} WrfMlpWork;

/* one-time set-up of the network's kernels on the current device; call it
 * before capturing any of the calls below into a CUDA graph */
int wrf_mlp_init(void);

/* out8 = km, ncx, ncy, ncols, nfeat (9 km), d0, nout (7 km + 3), d4 */
int wrf_mlp_layout(const WrfGrid* g, int* out8);

/* wrf_rk3_step with the microphysics call replaced by the network: features,
 * four tcgen05 GEMMs, apply with the positivity / supersaturation gate, and
 * WSM6 (the fused column kernel) on the rejected columns */
int wrf_rk3_step_mlp(const WrfGrid* g, const WrfState* s, const WrfMlpNet* net, const WrfMlpWork* work,
                     void* stream, wrf_probe_fn probe, void* user);

/* the network alone on m rows: x bf16 [m][d0] -> y fp32 [m][d4] (h0, h1: bf16 [m][max hidden]) */
int wrf_mlp_forward(const WrfMlpNet* net, const void* x, int m, void* h0, void* h1, float* y, int* err,
                    void* stream);

/* network rows of the state's columns: x (bf16, standardised with norm) if
 * raw is NULL, else raw (fp32 [ncols][10 km]: T p rho qv qc qr qi qs qg theta') */
int wrf_mlp_features(const WrfGrid* g, const WrfState* s, const float* norm, void* x, float* raw, void* stream);
/* raw increments [ncols][nout] of one microphysics call, given the raw rows before it */
int wrf_mlp_targets(const WrfGrid* g, const WrfState* s, const float* raw_in, float* raw_out, void* stream);
/* n raw rows -> bf16 inputs [n][d0] and fp32 standardised targets [n][d4] */
int wrf_mlp_normalize(const WrfGrid* g, const float* norm, const float* raw_in, const float* raw_out, long long n,
                      void* x, float* t, void* stream);

/* out = a b^T on the tensor cores (a: m x k, b: n x k, bf16 row-major; n a
 * multiple of 16, k of 64) with epilogue epi: 0 fp32 (+ bias; a split
 * reduction writes `splits` partial sums split_stride apart), 1 bf16
 * gelu(acc + bias) with the pre-activation in out_z, 2 bf16 acc * gelu'(aux),
 * 3 bf16 (+ bias); out_t (optional) receives the stored values transposed */
int wrf_gemm_bf16(const void* a, const void* b, int m, int n, int k, int splits, int epi, const float* bias,
                  const void* aux, void* out, int ldo, long long split_stride, void* out_z, void* out_t, int ldt,
                  int* err, void* stream);
/* number of partial sums wrf_gemm_bf16 writes for a requested split count */
int wrf_gemm_splits(int k, int splits);
/* dy = scale (y - t) (zero beyond column nvalid), row-major and transposed; *loss += sum (y - t)^2 */
int wrf_mse_grad(const float* y, const float* t, int m, int n, int nvalid, float scale, void* dy, void* dyt,
                 float* loss, void* stream);
/* out[r] = sum of row r of a bf16 [rows][cols] */
int wrf_rowsum_bf16(const void* a, int rows, int cols, float* out, void* stream);
/* Adam step (decoupled weight decay wd) on fp32 w [r][c] with the gradient summed from nsplit partials;
 * refreshes the bf16 copy wb [r][c] and the transposed copy wtb [c][r] (either may be NULL) */
int wrf_adam(float* w, const float* gpart, int nsplit, long long split_stride, float* m, float* v, int r, int c,
             void* wb, void* wtb, float lr, float beta1, float beta2, float eps, float wd, int step, void* stream);
/* out [c][r] = a [r][c]^T (bf16) */
int wrf_transpose_bf16(const void* a, int r, int c, void* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PYWRF_B200_H */
