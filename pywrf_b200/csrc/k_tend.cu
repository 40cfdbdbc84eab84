// Large-step (RK stage) tendencies.
//   k_advect  advect_u, advect_v, advect_w (wrf_dynamics.py:1112-1823) for rows
//             that are not a multiple of 16 bytes (else k_advect_mom_tma):
//             5th-order upwind-biased fluxes, 3rd/2nd order on the rows next
//             to each boundary (theta and the moisture species: k_advect_tiled)
//   k_forces  rhs_ph, horizontal_pressure_gradient, pg_buoy_w, coriolis,
//             curvature (wrf_dynamics.py:2031-2620)
//   k_addtend rk_addtend_dry + spec_bdytend (wrf_dynamics.py:3100-3148,
//             wrf_boundary.py:189-241)
// Each thread owns one (k, j, i) point and recomputes the two fluxes of its
// cell faces in each direction; tendencies accumulate in the reference's order
// (y, x, z advection, then forces).
#include "kernels.cuh"

namespace wrf {

// ------------------------------------------------------------ face fluxes

// u momentum, y faces (v points), column i (wrf_dynamics.py:1157-1182)
__device__ __forceinline__ float fqy_u(const Grid& g, const float* u, const float* rv, int k, int jf, int i) {
  const int jds = g.jds, jde = g.jde, nx = g.nx;
  const size_t base = (size_t)k * g.ny * nx;
  auto U = [&](int jj) { return u[base + (size_t)jj * nx + i]; };
  auto vel = [&](int jj) { return 0.5f * (rv[base + (size_t)jj * nx + i] + rv[base + (size_t)jj * nx + i - 1]); };
  if (jf >= jds + 3 && jf < jde - 3) {
    const float v = vel(jf);
    return v * flux5(U(jf - 3), U(jf - 2), U(jf - 1), U(jf), U(jf + 1), U(jf + 2), v);
  }
  if (jf == jds + 1) return 0.25f * (rv[base + (size_t)(jds + 1) * nx + i] + rv[base + (size_t)(jds + 1) * nx + i - 1]) * (U(jds + 1) + U(jds));
  if (jf == jds + 2) { const float v = vel(jds + 2); return v * flux3(U(jds), U(jds + 1), U(jds + 2), U(jds + 3), v); }
  if (jf == jde - 2) return 0.25f * (rv[base + (size_t)(jde - 2) * nx + i] + rv[base + (size_t)(jde - 2) * nx + i - 1]) * (U(jde - 2) + U(jde - 3));
  if (jf == jde - 3) {  // upwind sign from row jde-2, where the reference never set vel (0 -> +1)
    const float v = vel(jde - 3);
    return v * flux3(U(jde - 5), U(jde - 4), U(jde - 3), U(jde - 2), 0.0f);
  }
  return 0.f;
}

// u momentum, x faces (mass points) (wrf_dynamics.py:1212-1246)
__device__ __forceinline__ float fqx_u(const Grid& g, const float* u, const float* ru, int k, int j, int f) {
  const int ids = g.ids, ide = g.ide;
  const size_t r = ((size_t)k * g.ny + j) * g.nx;
  auto U = [&](int ii) { return u[r + ii]; };
  auto R = [&](int ii) { return ru[r + ii]; };
  if (f >= ids + 3 && f < ide - 2) {
    const float v = 0.5f * (R(f) + R(f - 1));
    return v * flux5(U(f - 3), U(f - 2), U(f - 1), U(f), U(f + 1), U(f + 2), v);
  }
  if (f == ids + 1) {
    const float ub = U(ids + 1) < 0.f ? U(ids + 1) : U(ids);
    return 0.25f * (R(ids + 1) + R(ids)) * (U(ids + 1) + ub);
  }
  if (f == ids + 2) { const float v = 0.5f * (R(ids + 2) + R(ids + 1)); return v * flux3(U(ids), U(ids + 1), U(ids + 2), U(ids + 3), v); }
  if (f == ide - 1) {
    const float ub = U(ide - 2) > 0.f ? U(ide - 2) : U(ide - 1);
    return 0.25f * (R(ide - 1) + R(ide - 2)) * (U(ide - 2) + ub);
  }
  if (f == ide - 2) { const float v = 0.5f * (R(ide - 2) + R(ide - 3)); return v * flux3(U(ide - 4), U(ide - 3), U(ide - 2), U(ide - 1), v); }
  return 0.f;
}

// u momentum, w levels (wrf_dynamics.py:1265-1300); rom averaged to u points
__device__ __forceinline__ float vf_u(const Grid& g, const S& s, const float* u, const float* rom, int kf, int j, int i) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t c = (size_t)j * g.nx + i;
  auto U = [&](int kk) { return u[kk * lev + c]; };
  auto vel = [&](int kk) { return 0.5f * (rom[kk * lev + c] + rom[kk * lev + c - 1]); };
  if (kf >= 3 && kf < ktf - 2) { const float v = vel(kf); return v * flux5(U(kf - 3), U(kf - 2), U(kf - 1), U(kf), U(kf + 1), U(kf + 2), -v); }
  if (kf == 1) return vel(1) * (s[WF_FNM][1] * U(1) + s[WF_FNP][1] * U(0));
  if (kf == 2) { const float v = vel(2); return v * flux3(U(0), U(1), U(2), U(3), -v); }
  if (kf == ktf - 2) { const float v = vel(kf); return v * flux3(U(kf - 2), U(kf - 1), U(kf), U(kf + 1), -v); }
  if (kf == ktf - 1) return vel(kf) * (s[WF_FNM][kf] * U(kf) + s[WF_FNP][kf] * U(kf - 1));
  return 0.f;
}

// v momentum, y faces (mass rows) (wrf_dynamics.py:1373-1407)
__device__ __forceinline__ float fqy_v(const Grid& g, const float* v, const float* rv, int k, int jf, int i) {
  const int jds = g.jds, jde = g.jde, nx = g.nx;
  const size_t base = (size_t)k * g.ny * nx + i;
  auto V = [&](int jj) { return v[base + (size_t)jj * nx]; };
  auto R = [&](int jj) { return rv[base + (size_t)jj * nx]; };
  if (jf >= jds + 3 && jf < jde - 2) {
    const float w = 0.5f * (R(jf) + R(jf - 1));
    return w * flux5(V(jf - 3), V(jf - 2), V(jf - 1), V(jf), V(jf + 1), V(jf + 2), w);
  }
  if (jf == jds + 1) {
    const float vb = V(jds + 1) < 0.f ? V(jds + 1) : V(jds);
    return 0.25f * (R(jds + 1) + R(jds)) * (V(jds + 1) + vb);
  }
  if (jf == jds + 2) { const float w = 0.5f * (R(jds + 2) + R(jds + 1)); return w * flux3(V(jds), V(jds + 1), V(jds + 2), V(jds + 3), w); }
  if (jf == jde - 1) {
    const float vb = V(jde - 2) > 0.f ? V(jde - 2) : V(jde - 1);
    return 0.25f * (R(jde - 1) + R(jde - 2)) * (V(jde - 2) + vb);
  }
  if (jf == jde - 2) { const float w = 0.5f * (R(jde - 2) + R(jde - 3)); return w * flux3(V(jde - 4), V(jde - 3), V(jde - 2), V(jde - 1), w); }
  return 0.f;
}

// v momentum, x faces (u points) (wrf_dynamics.py:1434-1463)
__device__ __forceinline__ float fqx_v(const Grid& g, const float* v, const float* ru, int k, int j, int f) {
  const int ids = g.ids, ide = g.ide, nx = g.nx;
  const size_t r = ((size_t)k * g.ny + j) * nx;
  auto V = [&](int ii) { return v[r + ii]; };
  auto R = [&](int ii) { return ru[r + ii] + ru[r - nx + ii]; };
  if (f >= ids + 3 && f < ide - 3) {
    const float w = 0.5f * R(f);
    return w * flux5(V(f - 3), V(f - 2), V(f - 1), V(f), V(f + 1), V(f + 2), w);
  }
  if (f == ids + 1) return 0.25f * R(ids + 1) * (V(ids + 1) + V(ids));
  if (f == ids + 2) { const float w = 0.5f * R(ids + 2); return w * flux3(V(ids), V(ids + 1), V(ids + 2), V(ids + 3), w); }
  if (f == ide - 2) return 0.25f * R(ide - 2) * (V(ide - 2) + V(ide - 3));
  if (f == ide - 3) { const float w = 0.5f * R(ide - 3); return w * flux3(V(ide - 5), V(ide - 4), V(ide - 3), V(ide - 2), w); }
  return 0.f;
}

// v momentum, w levels (wrf_dynamics.py:1482-1524); the ktf-2 row takes +vel
__device__ __forceinline__ float vf_v(const Grid& g, const S& s, const float* v, const float* rom, int kf, int j, int i) {
  const int ktf = g.nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const size_t c = (size_t)j * nx + i;
  auto V = [&](int kk) { return v[kk * lev + c]; };
  auto vel = [&](int kk) { return 0.5f * (rom[kk * lev + c] + rom[kk * lev + c - nx]); };
  if (kf >= 3 && kf < ktf - 2) { const float w = vel(kf); return w * flux5(V(kf - 3), V(kf - 2), V(kf - 1), V(kf), V(kf + 1), V(kf + 2), -w); }
  if (kf == 1) return vel(1) * (s[WF_FNM][1] * V(1) + s[WF_FNP][1] * V(0));
  if (kf == 2) { const float w = vel(2); return w * flux3(V(0), V(1), V(2), V(3), -w); }
  if (kf == ktf - 2) { const float w = vel(kf); return w * flux3(V(kf - 2), V(kf - 1), V(kf), V(kf + 1), w); }
  if (kf == ktf - 1) return vel(kf) * (s[WF_FNM][kf] * V(kf) + s[WF_FNP][kf] * V(kf - 1));
  return 0.f;
}

// w: coupled horizontal velocity interpolated to w level k (top: extrapolated)
__device__ __forceinline__ float wvel(const Grid& g, const S& s, const float* r, int k, size_t c) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  if (k < ktf) return s[WF_FNM][k] * r[k * lev + c] + s[WF_FNP][k] * r[(k - 1) * lev + c];
  return (2.0f - s[WF_FNM][ktf - 1]) * r[(ktf - 1) * lev + c] - s[WF_FNP][ktf - 1] * r[(ktf - 2) * lev + c];
}

// w, y faces (wrf_dynamics.py:1578-1656)
__device__ __forceinline__ float fqy_w(const Grid& g, const S& s, const float* w, const float* rv, int k, int jf, int i) {
  const int jds = g.jds, jde = g.jde, nx = g.nx;
  const size_t base = (size_t)k * g.ny * nx + i;
  auto W = [&](int jj) { return w[base + (size_t)jj * nx]; };
  const float vel = wvel(g, s, rv, k, (size_t)jf * nx + i);
  if (jf >= jds + 3 && jf < jde - 3) return vel * flux5(W(jf - 3), W(jf - 2), W(jf - 1), W(jf), W(jf + 1), W(jf + 2), vel);
  if (jf == jds + 1) return 0.5f * vel * (W(jds + 1) + W(jds));
  if (jf == jds + 2) return vel * flux3(W(jds), W(jds + 1), W(jds + 2), W(jds + 3), vel);
  if (jf == jde - 2) return 0.5f * vel * (W(jde - 2) + W(jde - 3));
  if (jf == jde - 3) return vel * flux3(W(jde - 5), W(jde - 4), W(jde - 3), W(jde - 2), vel);
  return 0.f;
}

// w, x faces (wrf_dynamics.py:1681-1758)
__device__ __forceinline__ float fqx_w(const Grid& g, const S& s, const float* w, const float* ru, int k, int j, int f) {
  const int ids = g.ids, ide = g.ide, nx = g.nx;
  const size_t r = ((size_t)k * g.ny + j) * nx;
  auto W = [&](int ii) { return w[r + ii]; };
  const float vel = wvel(g, s, ru, k, (size_t)j * nx + f);
  if (f >= ids + 3 && f < ide - 3) return vel * flux5(W(f - 3), W(f - 2), W(f - 1), W(f), W(f + 1), W(f + 2), vel);
  if (f == ids + 1) return 0.5f * vel * (W(ids + 1) + W(ids));
  if (f == ids + 2) return vel * flux3(W(ids), W(ids + 1), W(ids + 2), W(ids + 3), vel);
  if (f == ide - 2) return 0.5f * vel * (W(ide - 2) + W(ide - 3));
  if (f == ide - 3) return vel * flux3(W(ide - 5), W(ide - 4), W(ide - 3), W(ide - 2), vel);
  return 0.f;
}

// w, mass levels (wrf_dynamics.py:1773-1811); the ktf-1 row takes +vel
__device__ __forceinline__ float vf_w(const Grid& g, const float* w, const float* rom, int kf, size_t c) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  auto W = [&](int kk) { return w[kk * lev + c]; };
  auto R = [&](int kk) { return rom[kk * lev + c]; };
  if (kf >= 3 && kf < ktf - 1) { const float v = 0.5f * (R(kf) + R(kf - 1)); return v * flux5(W(kf - 3), W(kf - 2), W(kf - 1), W(kf), W(kf + 1), W(kf + 2), -v); }
  if (kf == 1) return 0.25f * (R(1) + R(0)) * (W(1) + W(0));
  if (kf == 2) { const float v = 0.5f * (R(2) + R(1)); return v * flux3(W(0), W(1), W(2), W(3), -v); }
  if (kf == ktf - 1) { const float v = 0.5f * (R(kf) + R(kf - 1)); return v * flux3(W(kf - 2), W(kf - 1), W(kf), W(kf + 1), v); }
  if (kf == ktf) return 0.25f * (R(ktf) + R(ktf - 1)) * (W(ktf) + W(ktf - 1));
  return 0.f;
}

// mass-point scalar, y faces (wrf_dynamics.py:1889-1910)
__device__ __forceinline__ float fqy_s(const Grid& g, const float* q, const float* rv, int k, int jf, int i) {
  const int jds = g.jds, jde = g.jde, nx = g.nx;
  const size_t base = (size_t)k * g.ny * nx + i;
  auto Q = [&](int jj) { return q[base + (size_t)jj * nx]; };
  const float r = rv[base + (size_t)jf * nx];
  if (jf >= jds + 3 && jf < jde - 3) return r * flux5(Q(jf - 3), Q(jf - 2), Q(jf - 1), Q(jf), Q(jf + 1), Q(jf + 2), r);
  if (jf == jds + 1) return 0.5f * r * (Q(jds + 1) + Q(jds));
  if (jf == jds + 2) return r * flux3(Q(jds), Q(jds + 1), Q(jds + 2), Q(jds + 3), r);
  if (jf == jde - 2) return 0.5f * r * (Q(jde - 2) + Q(jde - 3));
  if (jf == jde - 3) return r * flux3(Q(jde - 5), Q(jde - 4), Q(jde - 3), Q(jde - 2), r);
  return 0.f;
}

// mass-point scalar, x faces (wrf_dynamics.py:1941-1971); the ide-3 face
// takes its upwind sign from ru at ide-2
__device__ __forceinline__ float fqx_s(const Grid& g, const float* q, const float* ru, int k, int j, int f) {
  const int ids = g.ids, ide = g.ide;
  const size_t r0 = ((size_t)k * g.ny + j) * g.nx;
  auto Q = [&](int ii) { return q[r0 + ii]; };
  const float r = ru[r0 + f];
  if (f >= ids + 3 && f < ide - 3) return r * flux5(Q(f - 3), Q(f - 2), Q(f - 1), Q(f), Q(f + 1), Q(f + 2), r);
  if (f == ids + 1) return 0.5f * r * (Q(ids + 1) + Q(ids));
  if (f == ids + 2) return r * flux3(Q(ids), Q(ids + 1), Q(ids + 2), Q(ids + 3), r);
  if (f == ide - 2) return 0.5f * r * (Q(ide - 2) + Q(ide - 3));
  if (f == ide - 3) return r * flux3(Q(ide - 5), Q(ide - 4), Q(ide - 3), Q(ide - 2), ru[r0 + ide - 2]);
  return 0.f;
}

// mass-point scalar, w levels (wrf_dynamics.py:1991-2015)
__device__ __forceinline__ float vf_s(const Grid& g, const S& s, const float* q, const float* rom, int kf, size_t c) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  auto Q = [&](int kk) { return q[kk * lev + c]; };
  const float r = rom[kf * lev + c];
  if (kf >= 3 && kf < ktf - 2) return r * flux5(Q(kf - 3), Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), Q(kf + 2), -r);
  if (kf == 1) return r * (s[WF_FNM][1] * Q(1) + s[WF_FNP][1] * Q(0));
  if (kf == 2) return r * flux3(Q(0), Q(1), Q(2), Q(3), -r);
  if (kf == ktf - 2) return r * flux3(Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), -r);
  if (kf == ktf - 1) return r * (s[WF_FNM][kf] * Q(kf) + s[WF_FNP][kf] * Q(kf - 1));
  return 0.f;
}

// advect_scalar for one mass field into ``tend`` at (k, j, i)
__device__ __forceinline__ void advect_scalar_point(const Grid& g, const S& s, const float* q, float* tend, const float* ru,
                                                    const float* rv, const float* rom, int k, int j, int i) {
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  if (k >= ktf || i < ids || i >= ide - 1 || j < jds || j >= jde - 1) return;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  float t = tend[p];
  const float msftx = s[WF_MSFTX][c];
  if (j >= jds + 1 && j < jde - 2) t = t - (msftx * g.rdy) * (fqy_s(g, q, rv, k, j + 1, i) - fqy_s(g, q, rv, k, j, i));
  if (i >= ids + 1 && i < ide - 2) t = t - (msftx * g.rdx) * (fqx_s(g, q, ru, k, j, i + 1) - fqx_s(g, q, ru, k, j, i));
  t = t - s[WF_RDNW][k] * (vf_s(g, s, q, rom, k + 1, c) - vf_s(g, s, q, rom, k, c));
  tend[p] = t;
}

// comps: bit 0 u, bit 1 v, bit 2 w
__global__ void k_advect(Grid g, S s, int comps) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const float* ru = s[WF_RU];
  const float* rv = s[WF_RV];
  const float* ww = s[WF_WW];
  const float rdx = g.rdx, rdy = g.rdy;
  // u
  if ((comps & 1) && k < ktf && j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1) {
    const float* u = s[WF_U];
    const float msfux = s[WF_MSFUX][c];
    float t = s[WF_RU_TEND][p];
    if (j >= jds + 1 && j < jde - 2) t = t - (msfux * rdy) * (fqy_u(g, u, rv, k, j + 1, i) - fqy_u(g, u, rv, k, j, i));
    t = t - (msfux * rdx) * (fqx_u(g, u, ru, k, j, i + 1) - fqx_u(g, u, ru, k, j, i));
    t = t - s[WF_RDNW][k] * (vf_u(g, s, u, ww, k + 1, j, i) - vf_u(g, s, u, ww, k, j, i));
    s[WF_RU_TEND][p] = t;
  }
  // v
  if ((comps & 2) && k < ktf && j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1) {
    const float* v = s[WF_V];
    const float msfvy = s[WF_MSFVY][c];
    float t = s[WF_RV_TEND][p];
    t = t - (msfvy * rdy) * (fqy_v(g, v, rv, k, j + 1, i) - fqy_v(g, v, rv, k, j, i));
    if (i >= ids + 1 && i < ide - 2) t = t - (msfvy * rdx) * (fqx_v(g, v, ru, k, j, i + 1) - fqx_v(g, v, ru, k, j, i));
    t = t - ((msfvy / s[WF_MSFVX][c]) * s[WF_RDNW][k]) * (vf_v(g, s, v, ww, k + 1, j, i) - vf_v(g, s, v, ww, k, j, i));
    s[WF_RV_TEND][p] = t;
  }
  // w (levels 1..ktf)
  if ((comps & 4) && k >= 1 && j >= jds && j < jde - 1 && i >= ids && i < ide - 1) {
    const float* w = s[WF_W];
    const float msftx = s[WF_MSFTX][c];
    float t = s[WF_RW_TEND][p];
    if (j >= jds + 1 && j < jde - 2) t = t - (msftx * rdy) * (fqy_w(g, s, w, rv, k, j + 1, i) - fqy_w(g, s, w, rv, k, j, i));
    if (i >= ids + 1 && i < ide - 2) t = t - (msftx * rdx) * (fqx_w(g, s, w, ru, k, j, i + 1) - fqx_w(g, s, w, ru, k, j, i));
    if (k < ktf)
      t = t - s[WF_RDN][k] * (vf_w(g, w, ww, k + 1, c) - vf_w(g, w, ww, k, c));
    else
      t = t + 2.0f * s[WF_RDN][ktf - 1] * vf_w(g, w, ww, ktf, c);
    s[WF_RW_TEND][p] = t;
  }
  // theta: k_advect_tiled
}

// ------------------------------------------------------------------ forces

__device__ __forceinline__ float d6(const float* a, size_t p, int st) {
  return 45.0f * (a[p + st] - a[p - st]) - 9.0f * (a[p + 2 * st] - a[p - 2 * st]) + (a[p + 3 * st] - a[p - 3 * st]);
}

__global__ void k_forces(Grid g, S s, int terms) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const float gf = (float)G;
  const float rdx = g.rdx, rdy = g.rdy;
  const bool mass = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const float* ph = s[WF_PH];
  const float* phb = s[WF_PHB];
  const float* rdnw = s[WF_RDNW];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  // ---------------- rhs_ph (wrf_dynamics.py:2031-2297)
  if ((terms & 1) && mass && k >= 1) {
    const float* ww = s[WF_WW];
    const float* u = s[WF_U];
    const float* v = s[WF_V];
    const float* muu = s[WF_MUU];
    const float* muv = s[WF_MUV];
    const float* msfux = s[WF_MSFUX];
    const float* msfvy = s[WF_MSFVY];
    const float msfty = s[WF_MSFTY][c];
    float t = s[WF_PH_TEND][p];
    if (k < nz - 1) {
      auto wdwn = [&](int kk) {
        const size_t q = kk * lev + c, qm = q - lev;
        return 0.5f * (ww[q] + ww[qm]) * rdnw[kk - 1] * (ph[q] - ph[qm] + phb[q] - phb[qm]);
      };
      t = t - (fnm[k] * wdwn(k + 1) + fnp[k] * wdwn(k));
    } else {
      t = 0.f;
    }
    t = t + s[WF_MUT][c] * gf * s[WF_W][p] / msfty;
    const bool top = (k == nz - 1);
    const float cfn = g.cfn, cfn1 = g.cfn1;
    // y advection of phi
    auto fly = [&](int jj) {
      const size_t cc = (size_t)jj * nx + i;
      if (!top) return muv[cc] * (v[k * lev + cc] + v[(k - 1) * lev + cc]) * msfvy[cc];
      return muv[cc] * (cfn * v[(nz - 2) * lev + cc] + cfn1 * v[(nz - 3) * lev + cc]) * msfvy[cc];
    };
    const float ky = top ? (float)(0.5 * g.rdyd) : (float)(0.25 * g.rdyd);
    if (j >= jds + 3 && j < jde - 4) {
      const float dd = d6(ph, p, nx) + 45.0f * (phb[p + nx] - phb[p - nx]) - 9.0f * (phb[p + 2 * nx] - phb[p - 2 * nx]) + (phb[p + 3 * nx] - phb[p - 3 * nx]);
      t = t - (ky / msfty) * ((fly(j + 1) + fly(j)) * (float)(1.0 / 60.0) * dd);
    } else if (j == jds + 2 || j == jde - 4) {
      const float dd = 8.0f * (ph[p + nx] - ph[p - nx]) - (ph[p + 2 * nx] - ph[p - 2 * nx]) + 8.0f * (phb[p + nx] - phb[p - nx]) -
                       (phb[p + 2 * nx] - phb[p - 2 * nx]);
      t = t - (ky / msfty) * ((fly(j + 1) + fly(j)) * (float)(1.0 / 12.0) * dd);
    } else if (j == jds + 1 || j == jde - 3) {
      auto dp = [&](int d) { const size_t q = p + d * nx; return phb[q] - phb[q - nx] + ph[q] - ph[q - nx]; };
      t = t - (ky / msfty) * (fly(j + 1) * dp(1) + fly(j) * dp(0));
    }
    // x advection of phi (6th order interior, 2nd order at ids+1 and ide-3)
    auto flx = [&](int ii) {
      const size_t cc = (size_t)j * nx + ii;
      if (!top) return muu[cc] * (u[k * lev + cc] + u[(k - 1) * lev + cc]) * msfux[cc];
      return muu[cc] * (cfn * u[(nz - 2) * lev + cc] + cfn1 * u[(nz - 3) * lev + cc]) * msfux[cc];
    };
    const float kx = top ? (float)(0.5 * g.rdxd) : (float)(0.25 * g.rdxd);
    if (i >= ids + 3 && i < ide - 4) {
      const float dd = d6(ph, p, 1) + 45.0f * (phb[p + 1] - phb[p - 1]) - 9.0f * (phb[p + 2] - phb[p - 2]) + (phb[p + 3] - phb[p - 3]);
      t = t - (kx / msfty) * ((flx(i + 1) + flx(i)) * (float)(1.0 / 60.0) * dd);
    } else if (i == ids + 1 || i == ide - 3) {
      auto dp = [&](int d) { const size_t q = p + d; return phb[q] - phb[q - 1] + ph[q] - ph[q - 1]; };
      t = t - (kx / msfty) * (flx(i + 1) * dp(1) + flx(i) * dp(0));
    }
    s[WF_PH_TEND][p] = t;
  }
  // ---------------- horizontal pressure gradient (wrf_dynamics.py:2300-2421)
  const float* pp = s[WF_P];
  const float* pb = s[WF_PB];
  const float* al = s[WF_AL];
  const float* alt = s[WF_ALT];
  const float* php = s[WF_PHP];
  const float* mu = s[WF_MU];
  auto dpn = [&](int kk, size_t ca, size_t cb) {  // p at w level kk between two columns
    if (kk == 0)
      return 0.5f * (g.cf1 * (pp[cb] + pp[ca]) + g.cf2 * (pp[lev + cb] + pp[lev + ca]) + g.cf3 * (pp[2 * lev + cb] + pp[2 * lev + ca]));
    if (kk == nz - 1) return 0.f;
    return 0.5f * (fnm[kk] * (pp[kk * lev + cb] + pp[kk * lev + ca]) + fnp[kk] * (pp[(kk - 1) * lev + cb] + pp[(kk - 1) * lev + ca]));
  };
  if ((terms & 2) && k < ktf && j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1) {  // u
    const float r = s[WF_MSFUX][c] / s[WF_MSFUY][c];
    const size_t q = p, qm = p - 1;
    float dpx = r * 0.5f * rdx * s[WF_MUU][c] *
                ((ph[q + lev] - ph[qm + lev] + ph[q] - ph[qm]) + (alt[q] + alt[qm]) * (pp[q] - pp[qm]) + (al[q] + al[qm]) * (pb[q] - pb[qm]));
    dpx = dpx + r * rdx * (php[q] - php[qm]) * (rdnw[k] * (dpn(k + 1, c, c - 1) - dpn(k, c, c - 1)) - 0.5f * (mu[c - 1] + mu[c]));
    s[WF_RU_TEND][p] = s[WF_RU_TEND][p] - s[WF_CQU][p] * dpx;
  }
  if ((terms & 2) && k < ktf && j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1) {  // v
    const float r = s[WF_MSFVY][c] / s[WF_MSFVX][c];
    const size_t q = p, qm = p - nx;
    float dpy = r * 0.5f * rdy * s[WF_MUV][c] *
                ((ph[q + lev] - ph[qm + lev] + ph[q] - ph[qm]) + (alt[q] + alt[qm]) * (pp[q] - pp[qm]) + (al[q] + al[qm]) * (pb[q] - pb[qm]));
    dpy = dpy + r * rdy * (php[q] - php[qm]) * (rdnw[k] * (dpn(k + 1, c, c - nx) - dpn(k, c, c - nx)) - 0.5f * (mu[c - nx] + mu[c]));
    s[WF_RV_TEND][p] = s[WF_RV_TEND][p] - s[WF_CQV][p] * dpy;
  }
  // ---------------- pg_buoy_w (wrf_dynamics.py:2424-2460); cqw becomes 1/(1+cqw)
  if ((terms & 4) && mass && k >= 1 && k < nz - 1) {
    float* cqw = s[WF_CQW];
    const float rm = 1.0f / s[WF_MSFTY][c];
    const float mub = s[WF_MUB][c];
    if (k == nz - 2) {  // the top level reads the unmodified cqw of level nz-2
      const float cq1 = 1.0f / (1.0f + cqw[p]);
      const float cq2 = cqw[p] * cq1;
      const size_t pt = p + lev;
      s[WF_RW_TEND][pt] = s[WF_RW_TEND][pt] + rm * gf * (cq1 * 2.0f * rdnw[nz - 2] * (-pp[p]) - mu[c] - cq2 * mub);
    }
    const float cq1 = 1.0f / (1.0f + cqw[p]);
    const float cq2 = cqw[p] * cq1;
    cqw[p] = cq1;
    s[WF_RW_TEND][p] = s[WF_RW_TEND][p] + rm * gf * (cq1 * s[WF_RDN][k] * (pp[p] - pp[p - lev]) - mu[c] - cq2 * mub);
  }
  // ---------------- coriolis and curvature (wrf_dynamics.py:2463-2620)
  const float* ru = s[WF_RU];
  const float* rv = s[WF_RV];
  const float* rw = s[WF_RW];
  const float* f = s[WF_F];
  const float* e = s[WF_E];
  const float* sina = s[WF_SINA];
  const float* cosa = s[WF_COSA];
  const float rr = (float)RERADIUS;
  if ((terms & 24) && k < ktf && j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1) {  // u
    const float rvs = rv[p + nx - 1] + rv[p + nx] + rv[p - 1] + rv[p];
    const float rws = rw[p + lev - 1] + rw[p - 1] + rw[p + lev] + rw[p];
    float t = s[WF_RU_TEND][p];
    if (terms & 8)
      t = t + (s[WF_MSFUX][c] / s[WF_MSFUY][c]) * 0.5f * (f[c] + f[c - 1]) * 0.25f * rvs -
        0.5f * (e[c] + e[c - 1]) * 0.5f * (cosa[c] + cosa[c - 1]) * 0.25f * rws;
    const float* u = s[WF_U];
    const float* v = s[WF_V];
    auto vx = [&](int cc, size_t qq) {
      return 0.5f * (u[qq] + u[qq + 1]) * (s[WF_MSFVX][cc + nx] - s[WF_MSFVX][cc]) * rdy -
             0.5f * (v[qq] + v[qq + nx]) * (s[WF_MSFUY][cc + 1] - s[WF_MSFUY][cc]) * rdx;
    };
    if (terms & 16) t = t + 0.5f * (vx(c, p) + vx(c - 1, p - 1)) * 0.25f * rvs - u[p] * rr * 0.25f * rws;
    s[WF_RU_TEND][p] = t;
  }
  if ((terms & 24) && k < ktf && j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1) {  // v
    const float r = s[WF_MSFVY][c] / s[WF_MSFVX][c];
    const float rus = ru[p] + ru[p + 1] + ru[p - nx] + ru[p - nx + 1];
    const float rws = rw[p + lev - nx] + rw[p - nx] + rw[p + lev] + rw[p];
    float t = s[WF_RV_TEND][p];
    if (terms & 8) t = t - r * 0.5f * (f[c] + f[c - nx]) * 0.25f * rus + r * 0.5f * (e[c] + e[c - nx]) * 0.5f * (sina[c] + sina[c - nx]) * 0.25f * rws;
    const float* u = s[WF_U];
    const float* v = s[WF_V];
    auto vx = [&](int cc, size_t qq) {
      return 0.5f * (u[qq] + u[qq + 1]) * (s[WF_MSFVX][cc + nx] - s[WF_MSFVX][cc]) * rdy -
             0.5f * (v[qq] + v[qq + nx]) * (s[WF_MSFUY][cc + 1] - s[WF_MSFUY][cc]) * rdx;
    };
    if (terms & 16) t = t - 0.5f * (vx(c, p) + vx(c - nx, p - nx)) * 0.25f * rus - r * v[p] * rr * 0.25f * rws;
    s[WF_RV_TEND][p] = t;
  }
  if ((terms & 24) && mass && k >= 1 && k < ktf) {  // w
    const float fm = fnm[k], fp = fnp[k];
    const float A = fm * (ru[p] + ru[p + 1]) + fp * (ru[p - lev] + ru[p - lev + 1]);
    const float B = fm * (rv[p] + rv[p + nx]) + fp * (rv[p - lev] + rv[p - lev + nx]);
    const float rmt = s[WF_MSFTX][c] / s[WF_MSFTY][c];
    float t = s[WF_RW_TEND][p];
    if (terms & 8) t = t + e[c] * (cosa[c] * 0.5f * A - rmt * sina[c] * 0.5f * B);
    const float* u = s[WF_U];
    const float* v = s[WF_V];
    const float Cu = fm * (u[p] + u[p + 1]) + fp * (u[p - lev] + u[p - lev + 1]);
    const float Cv = fm * (v[p] + v[p + nx]) + fp * (v[p - lev] + v[p - lev + nx]);
    if (terms & 16) t = t + rr * (0.5f * A * 0.5f * Cu + rmt * 0.5f * B * 0.5f * Cv);
    s[WF_RW_TEND][p] = t;
  }
}

// the tendency terms selected by `terms` alone (1 rhs_ph, 2 the pressure
// gradient, 4 pg_buoy_w, 8 coriolis, 16 curvature), with the point kernel
int launch_forces_terms(const Grid& g, const S& s, int terms, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_forces<<<point_grid(g, b3), b3, 0, st>>>(g, s, terms);
  return 1;
}

// -------------------------------------------- tendency accumulation + spec rows

__global__ void k_addtend(Grid g, S s, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, nx = g.nx, ny = g.ny;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * ny * nx + c;
  const bool mass = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  auto ys0 = [&](int bid, int kk, int ii) { return s[bid][((size_t)kk * 5 + 0) * nx + ii]; };
  auto xs0 = [&](int bid, int kk, int jj) { return s[bid][((size_t)kk * ny + jj) * 5]; };
  // specified rows: field_tend = bdy_tend (y rows first, x columns overwrite)
  auto spec = [&](float& t, int btxs, int ibe, int jbe) {
    if (i >= ids && i < ibe && j == jds) t = ys0(btxs + 2, k, i);
    if (i >= ids && i < ibe && j == jbe - 1) t = ys0(btxs + 3, k, i);
    if (j >= jds && j < jbe && i == ids) t = xs0(btxs + 0, k, j);
    if (j >= jds && j < jbe && i == ibe - 1) t = xs0(btxs + 1, k, j);
  };
  // operands first, then the specified-row overrides, then the stores (a
  // store would hold back the later fields' loads)
  const bool r1 = rk_step == 1;
  const bool du = k < nz - 1 && j >= jds && j < jde - 1 && i >= ids && i < ide;
  const bool dv = k < nz - 1 && j >= jds && j < jde && i >= ids && i < ide - 1;
  const bool dt = mass && k < nz - 1;
  const bool dmu = mass && k == 0;
  float tfu = 0.f, usv = 0.f, mfuy = 1.f, rtu = 0.f;
  if (du) {
    tfu = s[WF_RU_TENDF][p];
    mfuy = s[WF_MSFUY][c];
    if (r1) usv = s[WF_U_SAVE][p];
    rtu = s[WF_RU_TEND][p];
  }
  float tfv = 0.f, vsv = 0.f, mfvx = 0.f, mvxi = 0.f, rtv = 0.f;
  if (dv) {
    tfv = s[WF_RV_TENDF][p];
    if (r1) {
      vsv = s[WF_V_SAVE][p];
      mfvx = s[WF_MSFVX][c];
    }
    mvxi = s[WF_MSFVX_INV][c];
    rtv = s[WF_RV_TEND][p];
  }
  float msfty = 1.f, tfw = 0.f, wsv = 0.f, rtw = 0.f, tfp = 0.f, phs = 0.f, rtp = 0.f;
  float tft = 0.f, tsv = 0.f, rtt = 0.f, mutc = 0.f, hd = 0.f, mut0 = 0.f, mutf0 = 0.f;
  if (mass) {
    msfty = s[WF_MSFTY][c];
    tfw = s[WF_RW_TENDF][p];
    rtw = s[WF_RW_TEND][p];
    tfp = s[WF_PH_TENDF][p];
    rtp = s[WF_PH_TEND][p];
    if (r1) {
      wsv = s[WF_W_SAVE][p];
      phs = s[WF_PH_SAVE][p];
    }
  }
  if (dt) {
    tft = s[WF_T_TENDF][p];
    if (r1) tsv = s[WF_T_SAVE][p];
    rtt = s[WF_T_TEND][p];
    mutc = s[WF_MUT][c];
    hd = s[WF_H_DIABATIC][p];
  }
  if (dmu) {
    mut0 = s[WF_MU_TEND][c];
    mutf0 = s[WF_MU_TENDF][c];
  }
  float ou = 0.f, ov = 0.f, ow = 0.f, oph = 0.f, ot = 0.f, omu = 0.f;
  if (du) {  // u
    if (r1) tfu = tfu + usv * mfuy;
    ou = rtu + tfu / mfuy;
    spec(ou, WF_U_BTXS, ide, jde - 1);
  }
  if (dv) {  // v
    if (r1) tfv = tfv + vsv * mfvx;
    ov = rtv + tfv * mvxi;
    spec(ov, WF_V_BTXS, ide - 1, jde);
  }
  if (mass) {
    if (r1) tfw = tfw + wsv * msfty;
    ow = rtw + tfw / msfty;
    if (r1) tfp = tfp + phs;
    oph = rtp + tfp / msfty;
    spec(oph, WF_PH_BTXS, ide - 1, jde - 1);
  }
  if (dt) {
    if (r1) tft = tft + tsv;
    ot = rtt + tft / msfty + mutc * hd / msfty;
    spec(ot, WF_T_BTXS, ide - 1, jde - 1);
  }
  if (dmu) {
    omu = mut0 + mutf0;
    spec(omu, WF_MU_BTXS, ide - 1, jde - 1);
  }
  if (du) {
    if (r1) s[WF_RU_TENDF][p] = tfu;
    s[WF_RU_TEND][p] = ou;
  }
  if (dv) {
    if (r1) s[WF_RV_TENDF][p] = tfv;
    s[WF_RV_TEND][p] = ov;
  }
  if (mass) {
    if (r1) {
      s[WF_RW_TENDF][p] = tfw;
      s[WF_PH_TENDF][p] = tfp;
    }
    s[WF_RW_TEND][p] = ow;
    s[WF_PH_TEND][p] = oph;
  }
  if (dt) {
    if (r1) s[WF_T_TENDF][p] = tft;
    s[WF_T_TEND][p] = ot;
  }
  if (dmu) s[WF_MU_TEND][c] = omu;
}

// stand-alone advect_scalar on caller arrays (s carries msftx, fnm, fnp, rdnw)
__global__ void k_advect_scalar(Grid g, S s, const float* q, float* tend, const float* ru, const float* rv,
                                const float* rom) {
  WRF_POINT_INDEX(g, k, j, i);
  advect_scalar_point(g, s, q, tend, ru, rv, rom, k, j, i);
}

int launch_advect_mom_point(const Grid& g, const S& s, int comps, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_advect<<<point_grid(g, b3), b3, 0, st>>>(g, s, comps);
  return 1;
}

int launch_advect_forces(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  int n = launch_advect_mom_tma(g, s, 0, 3, st);
  if (n == 0) n = launch_advect_mom_point(g, s, 7, st);
  n += launch_advect_theta_tiled(g, s, st);
  if (launch_forces_tma(g, s, st) == 0) k_forces<<<point_grid(g, b3), b3, 0, st>>>(g, s, 31);
  return n + 1;
}

int launch_addtend(const Grid& g, const S& s, int rk_step, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_addtend<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step);
  return 1;
}

int launch_advect_scalar(const Grid& g, const S& s, const float* field, float* tend, const float* ru,
                          const float* rv, const float* rom, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_advect_scalar<<<point_grid(g, b3), b3, 0, st>>>(g, s, field, tend, ru, rv, rom);
  return 1;
}

int launch_advect_moist(const Grid& g, const S& s, cudaStream_t st) { return launch_advect_moist_tiled(g, s, st); }

}  // namespace wrf
