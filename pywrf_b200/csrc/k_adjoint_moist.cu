// Adjoint of the moisture update of an RK stage (the step's k_moist_update +
// k_eos_flowdep, launch_moist): rk_update_scalar (wrf_dynamics.py:4055-4119),
// flow_dep_bdy of qc .. qg (wrf_boundary.py:470-508) and calc_p_rho_phi
// (wrf_dynamics.py:4124-4164), reversed in the opposite order.  The
// equation of state reads the updated qv, which the reverse pass recomputes
// into caller scratch first.  flow_dep_bdy copies an inner neighbour into
// the outer row (or zero, by the sign of the averaged mass flux, which is
// data): its reverse moves each outer point's cotangent onto its source.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

struct MoistRegions {
  bool full, inner;
};

__device__ __forceinline__ MoistRegions moist_regions(const Grid& g, int k, int j, int i) {
  MoistRegions r;
  r.full = k < g.nz - 1 && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1;
  r.inner = r.full && j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  return r;
}

// the updated qv (k_moist_update's arithmetic for slot 1) into qv_new
__global__ void k_qv_update(Grid g, S s, int rk_step, float dt, float* qv_new) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const MoistRegions r = moist_regions(g, k, j, i);
  const float cur = s[WF_MOIST][n3 + p];
  if (!r.full) {
    qv_new[p] = cur;
    return;
  }
  const float muold = s[WF_MU_1][c] + s[WF_MUB][c], munew = s[WF_MU][c] + s[WF_MUB][c];
  const float qo = rk_step != 1 ? s[WF_MOIST_OLD][n3 + p] : cur;
  float tend = r.inner ? s[WF_ADVECT_TEND][n3 + p] * s[WF_MSFTY][c] : 0.f;
  tend = tend + s[WF_MOIST_TEND][n3 + p];
  qv_new[p] = (muold * qo + dt * tend) / munew;
}

// calc_p_rho_phi's reverse on the mass points (al and p are overwritten)
__global__ void k_eos_adj(Grid g, S s, S b, const float* qv_new) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= g.nz - 1 || j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * lev + c;
  const float muts = s[WF_MUTS][c], mu = s[WF_MU][c], alb = s[WF_ALB][p], rdk = s[WF_RDNW][k];
  const float dph = s[WF_PH][p + lev] - s[WF_PH][p];
  const float al = -1.0f / muts * (alb * mu + rdk * dph);
  const float qv = qv_new[p], tk = s[WF_T][p];
  const float qvf = 1.0f + (float)RVOVRD * qv;
  const float den = (float)P0 * (al + alb);
  const float temp = ((float)R_D * ((float)T0 + tk) * qvf) / den;
  const float pp = wpow_eos(temp, (float)CPOVCV);
  const float P = b[WF_P][p];
  b[WF_PB][p] += -P;
  // d p / d temp = P0 cpovcv pp / temp
  const float Tb = (float)P0 * (float)CPOVCV * pp / temp * P;
  b[WF_T][p] += Tb * (float)R_D * qvf / den;
  b[WF_MOIST][n3 + p] += Tb * (float)R_D * ((float)T0 + tk) * (float)RVOVRD / den;
  const float denb = -Tb * temp / (al + alb);  // d temp / d (al + alb)
  const float A = b[WF_AL][p] + denb;
  b[WF_ALB][p] += denb - A * mu / muts;
  acc(b[WF_MU], c, -A * alb / muts);
  acc(b[WF_MUTS], c, A * (alb * mu + rdk * dph) / (muts * muts));
  acc(b[WF_PH], p + lev, -A * rdk / muts);
  acc(b[WF_PH], p, A * rdk / muts);
  b[WF_AL][p] = 0.f;
  b[WF_P][p] = 0.f;
}

// flow_dep_bdy's reverse for qc .. qg (levels below nz-1), in place: an
// outer-row point hands its cotangent to its source (an inner point, never
// an outer one) when the copy happened, and its own becomes zero
__global__ void k_flowdep_adj(Grid g, S s, S b) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= g.nz - 1) return;
  const int nx = g.nx, its = g.ids, jts = g.jds, itf = g.ide - 1, jtf = g.jde - 1;
  const size_t lev = (size_t)g.ny * nx, n3 = g.n3(), base = (size_t)k * lev;
  const float* um = s[WF_RU_M];
  const float* vm = s[WF_RV_M];
  int mode = 0, sj = 0, si = 0;
  bool cond = false;
  if (j == jts && i >= its && i < itf) {
    if (i == its) { mode = 1; sj = jts + 1; si = its + 1; }
    else if (i == itf - 1) { mode = 1; sj = jts + 1; si = itf - 2; }
    else { mode = 2; sj = jts + 1; si = i; cond = vm[base + (size_t)jts * nx + i] < 0.f; }
  } else if (j == jtf - 1 && i >= its && i < itf) {
    if (i == its) { mode = 1; sj = jtf - 2; si = its + 1; }
    else if (i == itf - 1) { mode = 1; sj = jtf - 2; si = itf - 2; }
    else { mode = 2; sj = jtf - 2; si = i; cond = vm[base + (size_t)jtf * nx + i] > 0.f; }
  } else if (j > jts && j < jtf - 1 && i == its) {
    mode = 2; sj = j; si = its + 1; cond = um[base + (size_t)j * nx + its] < 0.f;
  } else if (j > jts && j < jtf - 1 && i == itf - 1) {
    mode = 2; sj = j; si = itf - 2; cond = um[base + (size_t)j * nx + itf] > 0.f;
  }
  if (!mode) return;
  const size_t p = base + (size_t)j * nx + i, q = base + (size_t)sj * nx + si;
  float* fb = b[WF_MOIST];
  float v[5];  // the five species' loads before the first store
#pragma unroll
  for (int m = 2; m < 7; ++m) v[m - 2] = fb[m * n3 + p];
#pragma unroll
  for (int m = 2; m < 7; ++m) {
    fb[m * n3 + p] = 0.f;
    if (mode == 1 || cond) acc(fb, m * n3 + q, v[m - 2]);
  }
}

// rk_update_scalar's reverse, all six species.  The arrays may alias as far
// as the compiler knows, so the six species' loads are all written before
// the first store and issue together.
__global__ void k_moist_update_adj(Grid g, S s, S b, int rk_step, float dt) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const MoistRegions r = moist_regions(g, k, j, i);
  const bool first = rk_step == 1;
  float* qb = b[WF_MOIST];
  float* qob = b[WF_MOIST_OLD];
  if (!r.full) {
    // outside the updated region only the first stage's copy moist_old =
    // moist passes its cotangent back
    if (!first) return;
    float qv[6], qo[6];
#pragma unroll
    for (int m = 1; m < 7; ++m) {
      qv[m - 1] = qb[(size_t)m * n3 + p];
      qo[m - 1] = qob[(size_t)m * n3 + p];
    }
#pragma unroll
    for (int m = 1; m < 7; ++m) {
      qob[(size_t)m * n3 + p] = 0.f;
      qb[(size_t)m * n3 + p] = qv[m - 1] + qo[m - 1];
    }
    return;
  }
  const float muold = s[WF_MU_1][c] + s[WF_MUB][c];
  const float munew = s[WF_MU][c] + s[WF_MUB][c];
  const float msfty = s[WF_MSFTY][c];
  float Q[6], QO[6], qo[6], adv[6], mt[6], advb[6], mtb[6];
#pragma unroll
  for (int m = 1; m < 7; ++m) {
    const size_t o = (size_t)m * n3 + p;
    Q[m - 1] = qb[o];
    QO[m - 1] = qob[o];
    qo[m - 1] = first ? s[WF_MOIST][o] : s[WF_MOIST_OLD][o];
    adv[m - 1] = r.inner ? s[WF_ADVECT_TEND][o] : 0.f;
    advb[m - 1] = r.inner ? b[WF_ADVECT_TEND][o] : 0.f;
    mt[m - 1] = s[WF_MOIST_TEND][o];
    mtb[m - 1] = b[WF_MOIST_TEND][o];
  }
  float mu1b = 0.f, mub2 = 0.f;
#pragma unroll
  for (int m = 1; m < 7; ++m) {
    const size_t o = (size_t)m * n3 + p;
    const float q = Q[m - 1];
    // at the first stage moist_old became a copy of the incoming moist
    float qin_b = first ? QO[m - 1] : 0.f;
    const float tend = (r.inner ? adv[m - 1] * msfty : 0.f) + mt[m - 1];
    const float Tb = dt / munew * q;
    if (r.inner) b[WF_ADVECT_TEND][o] = advb[m - 1] + Tb * msfty;
    b[WF_MOIST_TEND][o] = mtb[m - 1] + Tb;
    const float qob_v = muold / munew * q;
    if (first) {
      qin_b += qob_v;
      qob[o] = 0.f;
    } else {
      qob[o] = QO[m - 1] + qob_v;
    }
    mu1b += qo[m - 1] * q / munew;
    mub2 += -(muold * qo[m - 1] + dt * tend) / (munew * munew) * q;
    qb[o] = qin_b;  // the updated value replaced the incoming one
  }
  acc(b[WF_MU_1], c, mu1b);
  acc(b[WF_MU], c, mub2);
  acc(b[WF_MUB], c, mu1b + mub2);
}

}  // namespace

// calc_p_rho_phi's reverse alone, with the state's own qv (the equation of
// state after the microphysics)
int launch_eos_adj(const Grid& g, const S& s, const S& b, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_eos_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, s[WF_MOIST] + g.n3());
  return 1;
}

// work: caller-owned scratch of nz * ny * nx floats
int launch_moist_adj(const Grid& g, const S& s, const S& b, int rk_step, float dt_rk, float* work, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_qv_update<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step, dt_rk, work);
  k_eos_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, work);
  k_flowdep_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b);
  k_moist_update_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, rk_step, dt_rk);
  return 4;
}

}  // namespace wrf
