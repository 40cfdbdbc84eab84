// rk_step_prep's functions (wrf_dynamics.py:30-159) one at a time, and their
// adjoints, selected by a bit of `ops`:
//   1 calculate_full   mut = mub + mu
//   2 calc_mu_uv       muu, muv: two-point averages of mu + mub
//   4 couple_momentum  ru = u muu / msfu, rv = v muv msfvx_inv, rw = w mut / msft
//   8 calc_ww_cp       column divergence, its k-sum and the upward ww scan
//  16 calc_cq          cqu, cqv, cqw from the sum of the moisture slots
//  32 calc_alt         alt = al + alb
//  64 calc_php         php: four-point average of ph + phb
// (the step computes them fused in k_rk_prep2d / k_rk_prep3d / k_ww_cp).
// Each function overwrites its outputs on its region: the adjoint reads an
// output's cotangent there, adds its contributions to the inputs'
// cotangents (atomically where inputs are shared by several outputs) and sets
// the output's cotangent to zero (its incoming value does not reach the
// result).  calc_ww_cp reads ww at level 0 and overwrites levels 1 .. nz-2.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

// ---- forward

__global__ void k_prep2d_ops(Grid g, S s, int ops) {
  WRF_COLUMN_INDEX(g, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int c = g.i2(j, i), nx = g.nx;
  const float* mu = s[WF_MU];
  const float* mub = s[WF_MUB];
  if ((ops & 1) && j >= jds && j < jde - 1 && i >= ids && i < ide - 1) s[WF_MUT][c] = mub[c] + mu[c];
  if (ops & 2) {
    if (j >= jds && j < jde - 1 && i >= ids && i < ide) {
      float v;
      if (i == ids) v = mu[c] + mub[c];
      else if (i == ide - 1) v = mu[c - 1] + mub[c - 1];
      else v = 0.5f * (mu[c] + mu[c - 1] + mub[c] + mub[c - 1]);
      s[WF_MUU][c] = v;
    }
    if (j >= jds && j < jde && i >= ids && i < ide - 1) {
      float v;
      if (j == jds) v = mu[c] + mub[c];
      else if (j == jde - 1) v = mu[c - nx] + mub[c - nx];
      else v = 0.5f * (mu[c] + mu[c - nx] + mub[c] + mub[c - nx]);
      s[WF_MUV][c] = v;
    }
  }
}

__device__ __forceinline__ float qsum(const S& s, size_t p, size_t n3) {
  const float* m = s[WF_MOIST];
  float q = m[p];
  for (int e = 1; e < 7; ++e) q = q + m[e * n3 + p];
  return q;
}

__global__ void k_prep3d_ops(Grid g, S s, int ops) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx, n3 = lev * nz;
  const size_t p = k * lev + c;
  const bool ur = k < ktf && j >= jds && j < jde - 1 && i >= ids && i < ide;
  const bool vr = k < ktf && j >= jds && j < jde && i >= ids && i < ide - 1;
  const bool wr = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool mr = k < ktf && wr;
  if (ops & 4) {
    if (ur) s[WF_RU][p] = s[WF_U][p] * s[WF_MUU][c] / s[WF_MSFU][c];
    if (vr) s[WF_RV][p] = s[WF_V][p] * s[WF_MUV][c] * s[WF_MSFVX_INV][c];
    if (wr) s[WF_RW][p] = s[WF_W][p] * s[WF_MUT][c] / s[WF_MSFT][c];
  }
  if (ops & 16) {
    if (ur) s[WF_CQU][p] = 1.0f / (1.0f + 0.5f * (qsum(s, p, n3) + qsum(s, p - 1, n3)));
    if (vr) s[WF_CQV][p] = 1.0f / (1.0f + 0.5f * (qsum(s, p, n3) + qsum(s, p - nx, n3)));
    if (mr && k >= 1) s[WF_CQW][p] = 0.5f * (qsum(s, p, n3) + qsum(s, p - lev, n3));
  }
  if ((ops & 32) && mr) s[WF_ALT][p] = s[WF_AL][p] + s[WF_ALB][p];
  if ((ops & 64) && mr) {
    const float* ph = s[WF_PH];
    const float* phb = s[WF_PHB];
    s[WF_PHP][p] = 0.5f * (phb[p] + phb[p + lev] + ph[p] + ph[p + lev]);
  }
}

// calc_ww_cp, one thread per mass column
__global__ void k_ww_cp_op(Grid g, S s) {
  WRF_COLUMN_INDEX(g, j, i);
  if (j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const int ktf = g.nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* dnw = s[WF_DNW];
  const float* c1h = s[WF_C1H];
  float* ww = s[WF_WW];
  auto divv = [&](int k) {
    const size_t p = k * lev + c;
    const float fu1 = s[WF_MUU][c + 1] * u[p + 1] / s[WF_MSFUY][c + 1], fu0 = s[WF_MUU][c] * u[p] / s[WF_MSFUY][c];
    const float fv1 = s[WF_MUV][c + nx] * v[p + nx] * s[WF_MSFVX_INV][c + nx], fv0 = s[WF_MUV][c] * v[p] * s[WF_MSFVX_INV][c];
    return (s[WF_MSFTX][c] * dnw[k]) * (g.rdx * (fu1 - fu0) + g.rdy * (fv1 - fv0));
  };
  float dmdt = 0.f;
  for (int k = 0; k < ktf; ++k) dmdt = dmdt + divv(k);
  float w = ww[c];
  for (int k = 0; k < ktf - 1; ++k) {
    w = w - (dnw[k] * c1h[k]) * dmdt - divv(k);
    ww[(k + 1) * lev + c] = w;
  }
}

// ---- adjoint

__global__ void k_prep2d_ops_adj(Grid g, S s, S b, int ops) {
  WRF_COLUMN_INDEX(g, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int c = g.i2(j, i), nx = g.nx;
  if ((ops & 1) && j >= jds && j < jde - 1 && i >= ids && i < ide - 1) {
    const float M = b[WF_MUT][c];
    acc(b[WF_MUB], c, M);
    acc(b[WF_MU], c, M);
    b[WF_MUT][c] = 0.f;
  }
  if (ops & 2) {
    if (j >= jds && j < jde - 1 && i >= ids && i < ide) {
      const float M = b[WF_MUU][c];
      if (i == ids) {
        acc(b[WF_MU], c, M);
        acc(b[WF_MUB], c, M);
      } else if (i == ide - 1) {
        acc(b[WF_MU], c - 1, M);
        acc(b[WF_MUB], c - 1, M);
      } else {
        acc(b[WF_MU], c, 0.5f * M);
        acc(b[WF_MUB], c, 0.5f * M);
        acc(b[WF_MU], c - 1, 0.5f * M);
        acc(b[WF_MUB], c - 1, 0.5f * M);
      }
      b[WF_MUU][c] = 0.f;
    }
    if (j >= jds && j < jde && i >= ids && i < ide - 1) {
      const float M = b[WF_MUV][c];
      if (j == jds) {
        acc(b[WF_MU], c, M);
        acc(b[WF_MUB], c, M);
      } else if (j == jde - 1) {
        acc(b[WF_MU], c - nx, M);
        acc(b[WF_MUB], c - nx, M);
      } else {
        acc(b[WF_MU], c, 0.5f * M);
        acc(b[WF_MUB], c, 0.5f * M);
        acc(b[WF_MU], c - nx, 0.5f * M);
        acc(b[WF_MUB], c - nx, 0.5f * M);
      }
      b[WF_MUV][c] = 0.f;
    }
  }
}

__global__ void k_prep3d_ops_adj(Grid g, S s, S b, int ops) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx, n3 = lev * nz;
  const size_t p = k * lev + c;
  const bool ur = k < ktf && j >= jds && j < jde - 1 && i >= ids && i < ide;
  const bool vr = k < ktf && j >= jds && j < jde && i >= ids && i < ide - 1;
  const bool wr = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool mr = k < ktf && wr;
  if (ops & 4) {
    if (ur) {
      const float R = b[WF_RU][p], m = s[WF_MSFU][c];
      acc(b[WF_U], p, s[WF_MUU][c] / m * R);
      acc(b[WF_MUU], c, s[WF_U][p] / m * R);
      b[WF_RU][p] = 0.f;
    }
    if (vr) {
      const float R = b[WF_RV][p], m = s[WF_MSFVX_INV][c];
      acc(b[WF_V], p, s[WF_MUV][c] * m * R);
      acc(b[WF_MUV], c, s[WF_V][p] * m * R);
      b[WF_RV][p] = 0.f;
    }
    if (wr) {
      const float R = b[WF_RW][p], m = s[WF_MSFT][c];
      acc(b[WF_W], p, s[WF_MUT][c] / m * R);
      acc(b[WF_MUT], c, s[WF_W][p] / m * R);
      b[WF_RW][p] = 0.f;
    }
  }
  if (ops & 16) {
    auto qs_bar = [&](size_t q, float v) {
      if (v == 0.f) return;
      for (int e = 0; e < 7; ++e) atomicAdd(&b[WF_MOIST][e * n3 + q], v);
    };
    if (ur) {
      const float cq = 1.0f / (1.0f + 0.5f * (qsum(s, p, n3) + qsum(s, p - 1, n3)));
      const float d = -0.5f * cq * cq * b[WF_CQU][p];
      qs_bar(p, d);
      qs_bar(p - 1, d);
      b[WF_CQU][p] = 0.f;
    }
    if (vr) {
      const float cq = 1.0f / (1.0f + 0.5f * (qsum(s, p, n3) + qsum(s, p - nx, n3)));
      const float d = -0.5f * cq * cq * b[WF_CQV][p];
      qs_bar(p, d);
      qs_bar(p - nx, d);
      b[WF_CQV][p] = 0.f;
    }
    if (mr && k >= 1) {
      const float d = 0.5f * b[WF_CQW][p];
      qs_bar(p, d);
      qs_bar(p - lev, d);
      b[WF_CQW][p] = 0.f;
    }
  }
  if ((ops & 32) && mr) {
    const float A = b[WF_ALT][p];
    acc(b[WF_AL], p, A);
    acc(b[WF_ALB], p, A);
    b[WF_ALT][p] = 0.f;
  }
  if ((ops & 64) && mr) {
    const float P = 0.5f * b[WF_PHP][p];
    acc(b[WF_PHB], p, P);
    acc(b[WF_PHB], p + lev, P);
    acc(b[WF_PH], p, P);
    acc(b[WF_PH], p + lev, P);
    b[WF_PHP][p] = 0.f;
  }
}

// calc_ww_cp's adjoint, one thread per mass column: with W(m) the cotangent
// of ww(m) (m = 1 .. ktf-1) and S(k) = sum of W(m) over m > k, the incoming
// ww(0) gets W(0) + sum W, dmdt gets -sum_k dnw(k) c1h(k) S(k), and divv(k)
// gets that minus S(k) (k < ktf-1); divv's cotangents go to u, v, muu, muv.
__global__ void k_ww_cp_op_adj(Grid g, S s, S b) {
  WRF_COLUMN_INDEX(g, j, i);
  if (j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const int ktf = g.nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  const float* dnw = s[WF_DNW];
  const float* c1h = s[WF_C1H];
  float* wwb = b[WF_WW];
  // the arrays may alias as far as the compiler knows: the column's loads
  // are written before its stores (in blocks of kChunk levels below), so
  // they issue together
  constexpr int kChunk = 8;
  float Wk[kMaxNz], Sk[kMaxNz];
#pragma unroll 8
  for (int k = 0; k < ktf; ++k) Wk[k] = wwb[k * lev + c];
  float run = 0.f, sumw = 0.f, dmb = 0.f;
#pragma unroll 8
  for (int k = ktf - 2; k >= 0; --k) {  // S(k) = W(k+1) + S(k+1)
    const float W = Wk[k + 1];
    run = run + W;
    Sk[k] = run;
    sumw = sumw + W;
    dmb = dmb - (dnw[k] * c1h[k]) * run;
  }
  const float msftx = s[WF_MSFTX][c];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float muu0 = s[WF_MUU][c], muu1 = s[WF_MUU][c + 1], mfu0 = s[WF_MSFUY][c], mfu1 = s[WF_MSFUY][c + 1];
  const float muv0 = s[WF_MUV][c], muv1 = s[WF_MUV][c + nx], mfv0 = s[WF_MSFVX_INV][c],
              mfv1 = s[WF_MSFVX_INV][c + nx];
  for (int k = 1; k < ktf; ++k) wwb[k * lev + c] = 0.f;
  wwb[c] = Wk[0] + sumw;
  float amuu0 = 0.f, amuu1 = 0.f, amuv0 = 0.f, amuv1 = 0.f;
  for (int k0 = 0; k0 < ktf; k0 += kChunk) {
    float u0[kChunk], u1[kChunk], v0[kChunk], v1[kChunk], dn[kChunk];
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
      const size_t p = (size_t)(k0 + q < ktf ? k0 + q : 0) * lev + c;
      u0[q] = u[p];
      u1[q] = u[p + 1];
      v0[q] = v[p];
      v1[q] = v[p + nx];
      dn[q] = dnw[k0 + q < ktf ? k0 + q : 0];
    }
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
      const int k = k0 + q;
      if (k >= ktf) break;
      const float D = dmb - (k < ktf - 1 ? Sk[k] : 0.f);
      const float E = msftx * dn[q] * D;
      const size_t p = k * lev + c;
      const float fu1b = g.rdx * E, fv1b = g.rdy * E;
      acc(b[WF_U], p + 1, muu1 / mfu1 * fu1b);
      amuu1 += u1[q] / mfu1 * fu1b;
      acc(b[WF_U], p, -muu0 / mfu0 * fu1b);
      amuu0 += -u0[q] / mfu0 * fu1b;
      acc(b[WF_V], p + nx, muv1 * mfv1 * fv1b);
      amuv1 += v1[q] * mfv1 * fv1b;
      acc(b[WF_V], p, -muv0 * mfv0 * fv1b);
      amuv0 += -v0[q] * mfv0 * fv1b;
    }
  }
  acc(b[WF_MUU], c + 1, amuu1);
  acc(b[WF_MUU], c, amuu0);
  acc(b[WF_MUV], c + nx, amuv1);
  acc(b[WF_MUV], c, amuv0);
}

}  // namespace

int launch_prep_ops(const Grid& g, const S& s, int ops, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  int n = 0;
  if (ops & 3) {
    k_prep2d_ops<<<col_grid(g, b2), b2, 0, st>>>(g, s, ops);
    ++n;
  }
  if (ops & 8) {
    k_ww_cp_op<<<col_grid(g, b2), b2, 0, st>>>(g, s);
    ++n;
  }
  if (ops & (4 | 16 | 32 | 64)) {
    k_prep3d_ops<<<point_grid(g, b3), b3, 0, st>>>(g, s, ops);
    ++n;
  }
  return n;
}

int launch_prep_ops_adj(const Grid& g, const S& s, const S& b, int ops, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  int n = 0;
  if (ops & (4 | 16 | 32 | 64)) {
    k_prep3d_ops_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, ops);
    ++n;
  }
  if (ops & 8) {
    k_ww_cp_op_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b);
    ++n;
  }
  if (ops & 3) {
    k_prep2d_ops_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b, ops);
    ++n;
  }
  return n;
}

}  // namespace wrf
