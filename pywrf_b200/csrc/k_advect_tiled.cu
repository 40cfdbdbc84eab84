// Tiled flux-form advection of mass-point scalars (advect_scalar,
// wrf_dynamics.py:1841-2028): the six moisture species with the time-averaged
// mass fluxes (rk_scalar_tend, wrf_dynamics.py:3982-4051) and theta with the
// stage's coupled velocities.
//
// A block of TX x TY threads owns (TX-1) x (TY-1) columns and marches up
// through KCH levels.  For each level the species' values of the tile and its
// halo are staged in shared memory (cp.async, double-buffered: the next level
// streams in while this one computes) and every thread forms exactly one x face
// flux and one y face flux (the tile's TX x TY faces); the vertical face flux
// is carried from one level to the next (each thread keeps a 7-level window
// of its column).  Face fluxes use the reference's orders:
// 5th order inside, 3rd order on the second face and 2nd order on the first
// face from each boundary; the tendency is accumulated y, then x, then z.
#include "kernels.cuh"

namespace wrf {

constexpr int kAdvTX = 32, kAdvTY = 8, kAdvKCH = 10;
constexpr int kAdvCX = kAdvTX - 1, kAdvCY = kAdvTY - 1;  // cells per tile; faces = threads
constexpr int kHX = kAdvTX + 5, kHY = kAdvTY + 5;        // staged tile: faces - 3 .. faces + 2

// up to six scalars; a block takes the group blockIdx.z % ngroup of NSP of them
struct AdvArgs {
  const float* q[6];
  float* tend[6];
  const float *ru, *rv, *rom;
  int ngroup;
};

// y face jf (between rows jf-1 and jf) from the tile column (wrf_dynamics.py:1889-1910)
__device__ __forceinline__ float yface(const Grid& g, const float* col /* col[y'] for y' = jj - (j0-3) */, int j0, int jf,
                                       float r) {
  const int jds = g.jds, jde = g.jde;
  auto Q = [&](int jj) { return col[(jj - (j0 - 3)) * kHX]; };
  if (jf >= jds + 3 && jf < jde - 3) return r * flux5(Q(jf - 3), Q(jf - 2), Q(jf - 1), Q(jf), Q(jf + 1), Q(jf + 2), r);
  if (jf == jds + 1) return 0.5f * r * (Q(jds + 1) + Q(jds));
  if (jf == jds + 2) return r * flux3(Q(jds), Q(jds + 1), Q(jds + 2), Q(jds + 3), r);
  if (jf == jde - 2) return 0.5f * r * (Q(jde - 2) + Q(jde - 3));
  if (jf == jde - 3) return r * flux3(Q(jde - 5), Q(jde - 4), Q(jde - 3), Q(jde - 2), r);
  return 0.f;
}

// x face f (between columns f-1 and f) from the tile row (wrf_dynamics.py:1941-1971);
// the ide-3 face takes its upwind sign from ru at ide-2 (rsgn)
__device__ __forceinline__ float xface(const Grid& g, const float* row /* row[x'] for x' = ii - (i0-3) */, int i0, int f,
                                       float r, float rsgn) {
  const int ids = g.ids, ide = g.ide;
  auto Q = [&](int ii) { return row[ii - (i0 - 3)]; };
  if (f >= ids + 3 && f < ide - 3) return r * flux5(Q(f - 3), Q(f - 2), Q(f - 1), Q(f), Q(f + 1), Q(f + 2), r);
  if (f == ids + 1) return 0.5f * r * (Q(ids + 1) + Q(ids));
  if (f == ids + 2) return r * flux3(Q(ids), Q(ids + 1), Q(ids + 2), Q(ids + 3), r);
  if (f == ide - 2) return 0.5f * r * (Q(ide - 2) + Q(ide - 3));
  if (f == ide - 3) return r * flux3(Q(ide - 5), Q(ide - 4), Q(ide - 3), Q(ide - 2), rsgn);
  return 0.f;
}

// vertical face kf from the column window w[0..6] = q(kc-3 .. kc+3), kf in {kc, kc+1}
// (wrf_dynamics.py:1991-2015)
__device__ __forceinline__ float zface(int ktf, const float* fnm, const float* fnp, const float* w, int kc, int kf, float r) {
  auto Q = [&](int kk) { return w[kk - kc + 3]; };
  if (kf >= 3 && kf < ktf - 2) return r * flux5(Q(kf - 3), Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), Q(kf + 2), -r);
  if (kf == 1) return r * (__ldg(&fnm[1]) * Q(1) + __ldg(&fnp[1]) * Q(0));
  if (kf == 2) return r * flux3(Q(0), Q(1), Q(2), Q(3), -r);
  if (kf == ktf - 2) return r * flux3(Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), -r);
  if (kf == ktf - 1) return r * (__ldg(&fnm[kf]) * Q(kf) + __ldg(&fnp[kf]) * Q(kf - 1));
  return 0.f;
}

// ACCUM: add to the tendency already in tend (else tend = the advection alone,
// and the points of [0, nz) x [jds, jde) x [ids, ide) outside the advected
// region are set to zero, as the reference zeroes advect_tend first)
template <int NSP, bool ACCUM>
__global__ void __launch_bounds__(kAdvTX * kAdvTY) k_advect_tiled(Grid g, S s, AdvArgs a) {
  __shared__ float tq[2][NSP][kHY][kHX];  // double buffer: level k computes while k+1 loads
  __shared__ float fx[NSP][kAdvTY][kAdvTX];
  __shared__ float fy[NSP][kAdvTY][kAdvTX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = g.ids + blockIdx.x * kAdvCX, j0 = g.jds + blockIdx.y * kAdvCY;
  const int i = i0 + tx, j = j0 + ty;
  const int nx = g.nx, ny = g.ny, ktf = g.nz - 1;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const size_t lev = (size_t)ny * nx;
  const int grp = blockIdx.z % a.ngroup;
  const int k0 = (blockIdx.z / a.ngroup) * kAdvKCH, k1 = min(k0 + kAdvKCH, g.nz);
  const float* qs[NSP];
  float* ts[NSP];
#pragma unroll
  for (int m = 0; m < NSP; ++m) {
    qs[m] = a.q[grp * NSP + m];
    ts[m] = a.tend[grp * NSP + m];
  }
  const bool inner = tx < kAdvCX && ty < kAdvCY;
  const bool cell = inner && i < ide - 1 && j < jde - 1;  // advected column
  const bool zreg = inner && i < ide && j < jde;          // zeroed column
  const bool xf = j < jde - 1 && i >= ids + 1 && i <= ide - 2;  // x face i of row j is used
  const bool yf = i < ide - 1 && j >= jds + 1 && j <= jde - 2;  // y face j of column i is used
  const bool doy = j >= jds + 1 && j < jde - 2;
  const bool dox = i >= ids + 1 && i < ide - 2;
  const int c = g.i2(min(j, ny - 1), min(i, nx - 1));
  const float msftx = cell ? __ldg(&s[WF_MSFTX][c]) : 0.f;
  const float cy = msftx * g.rdy, cx = msftx * g.rdx;
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  // column windows q(k-3 .. k+3) and the flux through the bottom face
  float win[NSP][7], fbot[NSP];
  auto colq = [&](int m, int kk) -> float {
    return (cell && kk >= 0 && kk < g.nz) ? __ldg(&qs[m][kk * lev + c]) : 0.f;
  };
#pragma unroll
  for (int m = 0; m < NSP; ++m) {
#pragma unroll
    for (int d = 0; d < 7; ++d) win[m][d] = colq(m, k0 - 3 + d);
    const float r = cell && k0 < g.nz ? __ldg(&a.rom[k0 * lev + c]) : 0.f;
    fbot[m] = zface(ktf, fnm, fnp, win[m], k0, k0, r);
  }
  // asynchronous copy of a level's tile (and halo) of every species into a
  // buffer; points outside the allocation are zero-filled
  auto stage = [&](int k, int buf) {
    for (int e = ty * kAdvTX + tx; e < kHY * kHX; e += kAdvTX * kAdvTY) {
      const int yy = e / kHX, xx = e % kHX;
      const int jj = j0 - 3 + yy, ii = i0 - 3 + xx;
      const bool in = jj >= 0 && jj < ny && ii >= 0 && ii < nx;
      const size_t p = in ? (size_t)k * lev + (size_t)jj * nx + ii : 0;
#pragma unroll
      for (int m = 0; m < NSP; ++m) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(&tq[buf][m][yy][xx]);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(qs[m] + p), "r"(in ? 4 : 0));
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  if (k0 < k1) stage(k0, 0);
  for (int k = k0; k < k1; ++k) {
    const int buf = (k - k0) & 1;
    if (k + 1 < k1) {
      stage(k + 1, buf ^ 1);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    const size_t pc = (size_t)k * lev + c;
    if (k < ktf) {
      // one x face (i, between i-1 and i) and one y face (j) per thread
      const float rl = xf ? __ldg(&a.ru[pc]) : 0.f;
      const float rs3 = xf ? __ldg(&a.ru[(size_t)k * lev + (size_t)j * nx + (ide - 2)]) : 0.f;
      const float rb = yf ? __ldg(&a.rv[pc]) : 0.f;
#pragma unroll
      for (int m = 0; m < NSP; ++m) {
        fx[m][ty][tx] = xf ? xface(g, &tq[buf][m][ty + 3][0], i0, i, rl, rs3) : 0.f;
        fy[m][ty][tx] = yf ? yface(g, &tq[buf][m][0][tx + 3], j0, j, rb) : 0.f;
      }
    }
    __syncthreads();
    const float rtop = (cell && k + 1 < g.nz) ? __ldg(&a.rom[pc + lev]) : 0.f;
#pragma unroll
    for (int m = 0; m < NSP; ++m) {
      const float ftop = zface(ktf, fnm, fnp, win[m], k, k + 1, rtop);
      if (cell && k < ktf) {
        float t = ACCUM ? ts[m][pc] : 0.f;
        if (doy) t = t - cy * (fy[m][ty + 1][tx] - fy[m][ty][tx]);
        if (dox) t = t - cx * (fx[m][ty][tx + 1] - fx[m][ty][tx]);
        t = t - __ldg(&rdnw[k]) * (ftop - fbot[m]);
        ts[m][pc] = t;
      } else if (!ACCUM && zreg) {
        ts[m][pc] = 0.f;
      }
      fbot[m] = ftop;
#pragma unroll
      for (int d = 0; d < 6; ++d) win[m][d] = win[m][d + 1];
      win[m][6] = colq(m, k + 4);
    }
  }
}

int launch_advect_moist_tiled(const Grid& g, const S& s, cudaStream_t st) {
  AdvArgs a;
  const size_t n3 = g.n3();
  for (int m = 0; m < 6; ++m) {
    a.q[m] = s[WF_MOIST] + (m + 1) * n3;
    a.tend[m] = s[WF_ADVECT_TEND] + (m + 1) * n3;
  }
  a.ru = s[WF_RU_M];
  a.rv = s[WF_RV_M];
  a.rom = s[WF_WW_M];
  a.ngroup = 3;
  const dim3 b(kAdvTX, kAdvTY);
  const dim3 gr((g.ide - g.ids + kAdvCX - 1) / kAdvCX, (g.jde - g.jds + kAdvCY - 1) / kAdvCY,
                3 * ((g.nz + kAdvKCH - 1) / kAdvKCH));
  k_advect_tiled<2, false><<<gr, b, 0, st>>>(g, s, a);
  return 1;
}

int launch_advect_theta_tiled(const Grid& g, const S& s, cudaStream_t st) {
  AdvArgs a{};
  a.q[0] = s[WF_T];
  a.tend[0] = s[WF_T_TEND];
  a.ru = s[WF_RU];
  a.rv = s[WF_RV];
  a.rom = s[WF_WW];
  a.ngroup = 1;
  const dim3 b(kAdvTX, kAdvTY);
  const dim3 gr((g.ide - g.ids + kAdvCX - 1) / kAdvCX, (g.jde - g.jds + kAdvCY - 1) / kAdvCY,
                (g.nz + kAdvKCH - 1) / kAdvKCH);
  k_advect_tiled<1, true><<<gr, b, 0, st>>>(g, s, a);
  return 1;
}

}  // namespace wrf
