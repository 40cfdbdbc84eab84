// Tiled flux-form advection of mass-point scalars (advect_scalar,
// wrf_dynamics.py:1841-2028): the six moisture species with the time-averaged
// mass fluxes (rk_scalar_tend, wrf_dynamics.py:3982-4051) and theta with the
// stage's coupled velocities.
//
// A block of TX x TY threads owns (TX-1) x (TY-1) columns and marches up
// through KCH levels.  For each level the species' values of the tile and its
// halo are staged in shared memory together with everything else the level
// reads (the thread's face velocities, the rom of its top face, the column
// value three levels up and, when accumulating, its tendency): cp.async,
// double-buffered, so the next level streams in while this one computes and
// no global load waits between the level's barriers.  Every thread forms
// exactly one x face flux and one y face flux (the tile's TX x TY faces); the
// vertical face flux is carried from one level to the next (each thread keeps
// a 7-level window of its column).  Face fluxes use the reference's orders:
// 5th order inside, 3rd order on the second face and 2nd order on the first
// face from each boundary; the tendency is accumulated y, then x, then z.
#include "kernels.cuh"
#include "tma.cuh"

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

// y face jf (between rows jf-1 and jf) from the tile column, rows STRIDE
// floats apart (wrf_dynamics.py:1889-1910)
template <int STRIDE = kHX>
__device__ __forceinline__ float yface(const Grid& g, const float* col /* col[y'] for y' = jj - (j0-3) */, int j0, int jf,
                                       float r) {
  const int jds = g.jds, jde = g.jde;
  auto Q = [&](int jj) { return col[(jj - (j0 - 3)) * STRIDE]; };
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

__device__ __forceinline__ void cp_async4(void* dst, const float* src, bool in) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(in ? 4 : 0));
}

// What one level reads besides the tile: per thread its x-face ru, the ru at
// ide-2 of its row (the ide-3 face's upwind sign), its y-face rv, the rom of
// its cell's top face, its column's value three levels up and, when
// accumulating, its tendency.
template <int NSP>
struct AdvLevel {
  float ru[kAdvTY][kAdvTX], rs3[kAdvTY][kAdvTX], rv[kAdvTY][kAdvTX], rtop[kAdvTY][kAdvTX];
  float qup[NSP][kAdvTY][kAdvTX], tv[NSP][kAdvTY][kAdvTX];
};

// ACCUM: add to the tendency already in tend (else tend = the advection alone,
// and the points of [0, nz) x [jds, jde) x [ids, ide) outside the advected
// region are set to zero, as the reference zeroes advect_tend first)
template <int NSP, bool ACCUM>
__global__ void __launch_bounds__(kAdvTX * kAdvTY) k_advect_tiled(Grid g, S s, AdvArgs a) {
  __shared__ float tq[2][NSP][kHY][kHX];  // double buffer: level k computes while k+1 loads
  __shared__ AdvLevel<NSP> lv[2];
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
  const size_t crs3 = (size_t)min(j, ny - 1) * nx + (ide - 2);
  const float msftx = cell ? __ldg(&s[WF_MSFTX][c]) : 0.f;
  const float cy = msftx * g.rdy, cx = msftx * g.rdx;
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  // column windows q(k-3 .. k+3) and the flux through the bottom face
  float win[NSP][7], fbot[NSP];
#pragma unroll
  for (int m = 0; m < NSP; ++m) {
#pragma unroll
    for (int d = 0; d < 7; ++d) {
      const int kk = k0 - 3 + d;
      win[m][d] = (cell && kk >= 0 && kk < g.nz) ? __ldg(&qs[m][kk * lev + c]) : 0.f;
    }
    const float r = cell && k0 < g.nz ? __ldg(&a.rom[k0 * lev + c]) : 0.f;
    fbot[m] = zface(ktf, fnm, fnp, win[m], k0, k0, r);
  }
  // asynchronous copy of everything level k reads into buffer buf; points
  // outside the allocation or unused by the thread are zero-filled
  auto stage = [&](int k, int buf) {
    for (int e = ty * kAdvTX + tx; e < kHY * kHX; e += kAdvTX * kAdvTY) {
      const int yy = e / kHX, xx = e % kHX;
      const int jj = j0 - 3 + yy, ii = i0 - 3 + xx;
      const bool in = jj >= 0 && jj < ny && ii >= 0 && ii < nx;
      const size_t p = in ? (size_t)k * lev + (size_t)jj * nx + ii : 0;
#pragma unroll
      for (int m = 0; m < NSP; ++m) cp_async4(&tq[buf][m][yy][xx], qs[m] + p, in);
    }
    const size_t kl = (size_t)k * lev;
    const bool hz = k < ktf;
    AdvLevel<NSP>& L = lv[buf];
    cp_async4(&L.ru[ty][tx], a.ru + (xf && hz ? kl + c : 0), xf && hz);
    cp_async4(&L.rs3[ty][tx], a.ru + (xf && hz ? kl + crs3 : 0), xf && hz);
    cp_async4(&L.rv[ty][tx], a.rv + (yf && hz ? kl + c : 0), yf && hz);
    const bool top = cell && k + 1 < g.nz;
    cp_async4(&L.rtop[ty][tx], a.rom + (top ? kl + lev + c : 0), top);
    const bool up = cell && k + 3 < g.nz;
#pragma unroll
    for (int m = 0; m < NSP; ++m) {
      cp_async4(&L.qup[m][ty][tx], qs[m] + (up ? kl + 3 * lev + c : 0), up);
      if (ACCUM) cp_async4(&L.tv[m][ty][tx], ts[m] + (cell && hz ? kl + c : 0), cell && hz);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  if (k0 < k1) stage(k0, 0);
  for (int k = k0; k < k1; ++k) {
    const int buf = (k - k0) & 1;
    const float rdk = __ldg(&rdnw[k]);
    if (k + 1 < k1) {
      stage(k + 1, buf ^ 1);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    const AdvLevel<NSP>& L = lv[buf];
    const size_t pc = (size_t)k * lev + c;
    if (k < ktf) {
      // one x face (i, between i-1 and i) and one y face (j) per thread
      const float rl = L.ru[ty][tx], rs3 = L.rs3[ty][tx], rb = L.rv[ty][tx];
#pragma unroll
      for (int m = 0; m < NSP; ++m) {
        fx[m][ty][tx] = xf ? xface(g, &tq[buf][m][ty + 3][0], i0, i, rl, rs3) : 0.f;
        fy[m][ty][tx] = yf ? yface(g, &tq[buf][m][0][tx + 3], j0, j, rb) : 0.f;
      }
    }
    __syncthreads();
    const float rtop = L.rtop[ty][tx];
#pragma unroll
    for (int m = 0; m < NSP; ++m) {
      win[m][6] = L.qup[m][ty][tx];  // q(k+3)
      const float ftop = zface(ktf, fnm, fnp, win[m], k, k + 1, rtop);
      if (cell && k < ktf) {
        float t = ACCUM ? L.tv[m][ty][tx] : 0.f;
        if (doy) t = t - cy * (fy[m][ty + 1][tx] - fy[m][ty][tx]);
        if (dox) t = t - cx * (fx[m][ty][tx + 1] - fx[m][ty][tx]);
        t = t - rdk * (ftop - fbot[m]);
        ts[m][pc] = t;
      } else if (!ACCUM && zreg) {
        ts[m][pc] = 0.f;
      }
      fbot[m] = ftop;
#pragma unroll
      for (int d = 0; d < 6; ++d) win[m][d] = win[m][d + 1];
    }
  }
}

// ------------------------------------------------------------------------
// TMA form, for arrays whose rows are a multiple of 16 bytes (nx % 4 == 0).
// A block of 32 x 8 threads owns 32 x 8 columns (one per thread) and a chunk
// of levels.  One thread issues, per level, tile loads of the scalars (box
// 44 x 14 from x = floor4(i0 - 3), y = j0 - 3: the tile plus its 3-cell
// halo) and of the level's face velocities, top-face rom and (accumulating)
// tendency (boxes 40 x 9 from x = floor4(i0), y = j0) into shared rings
// completed on mbarriers, kTRing - 1 levels ahead for the scalars and
// kARing - 1 for the rest; out-of-range elements arrive as zeros.  The other
// threads spend no instructions on staging.  Each thread forms the x face
// west of its cell and the y face south of it; warp 6 adds the tile's east
// faces and warp 7 its north faces.  Blocks wholly inside the 5th-order
// region take the fluxes without the boundary branches.  The arithmetic and
// its order are those of the cp.async form above.
//
// Every wait on a tile is bounded (~2 s); a block whose wait runs out stops,
// waits (bounded) for the copies it issued, adds 1 to STATUS[WRF_ST_WAIT]
// and returns.
constexpr int kTTX = 32, kTTY = 8;
constexpr int kQW = 44, kQH = kTTY + 6;        // scalar box
constexpr int kAW = 40, kAH = kTTY + 1;        // per-level box
constexpr uint32_t kQBytes = kQW * kQH * 4, kABytes = kAW * kAH * 4;
constexpr int kQSlot = 640, kASlot = 384;      // floats per ring slot (128-byte multiples)
constexpr int kTRing = 5, kARing = 3;
constexpr int kTKCH = 10;                      // levels per block, at most (chunks balanced over nz)
constexpr long long kAdvWaitCycles = 4000000000LL;
static_assert(kQBytes <= kQSlot * 4 && kABytes <= kASlot * 4, "a ring slot holds one box");
static_assert(kTRing >= 5, "the column window reads the tile three levels up, issued a level earlier");

struct AdvTmaArgs {
  CUtensorMap q;                  // the scalars: [nw][nz][ny][nx], box kQW x kQH
  CUtensorMap ru, rv, rom, tend;  // box kAW x kAH (tend: accumulating form only)
  const float* qg[6];             // the scalars, for the column window's direct loads
  float* tout[6];                 // tendencies written
  const float* romg;              // rom, for the chunk's bottom face
  int qw0, tw0;                   // array index of the first scalar in q / tend
  int ngroup, nchunk;
};

template <int NSP, bool ACCUM>
struct __align__(128) AdvTmaSmem {
  float q[kTRing][NSP][kQSlot];
  float aux[kARing][3 + (ACCUM ? NSP : 0)][kASlot];
  float fx[NSP][kTTY][kTTX + 1];
  float fy[NSP][kTTY + 1][kTTX];
  uint64_t qbar[kTRing], abar[kARing];
};

#ifndef WRF_ADV_MINB
#define WRF_ADV_MINB 4
#endif
template <int NSP, bool ACCUM>
__global__ void __launch_bounds__(kTTX * kTTY, WRF_ADV_MINB) k_advect_tma(Grid g, S s, const __grid_constant__ AdvTmaArgs a) {
  constexpr int NA = 3 + (ACCUM ? NSP : 0);
  __shared__ AdvTmaSmem<NSP, ACCUM> sm;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTTX + tx;
  const int nx = g.nx, ny = g.ny, nz = g.nz, ktf = nz - 1;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int i0 = ids + blockIdx.x * kTTX, j0 = jds + blockIdx.y * kTTY;
  const int i = i0 + tx, j = j0 + ty;
  const int qx = (i0 - 3) & ~3, ax = i0 & ~3;  // box origins, multiples of 4 (floor for negatives)
  const int oq = i0 - 3 - qx, oa = i0 - ax;    // tile columns of i0 - 3 and of i0
  const size_t lev = (size_t)ny * nx;
  const int grp = blockIdx.z % a.ngroup, chunk = blockIdx.z / a.ngroup;
  const int k0 = chunk * nz / a.nchunk, k1 = (chunk + 1) * nz / a.nchunk;
  const int qw = a.qw0 + grp * NSP, tw = a.tw0 + grp * NSP;
  const bool cell = i < ide - 1 && j < jde - 1;  // advected column
  const bool zreg = i < ide && j < jde;          // zeroed column
  const bool doy = j >= jds + 1 && j < jde - 2;
  const bool dox = i >= ids + 1 && i < ide - 2;
  // the whole block in the 5th-order region (x faces i0 .. i0+32, y faces j0 .. j0+8)
  const bool xin = i0 >= ids + 3 && i0 + kTTX < ide - 3;
  const bool yin = j0 >= jds + 3 && j0 + kTTY < jde - 3;
  const int c = min(j, ny - 1) * nx + min(i, nx - 1);
  const float msftx = cell ? __ldg(&s[WF_MSFTX][c]) : 0.f;
  const float cy = msftx * g.rdy, cx = msftx * g.rdx;
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  const int rs3x = ide - 2 - ax;  // column of ru(ide-2) in the per-level box
  const bool rs3in = rs3x >= 0 && rs3x < kAW;

  if (tid == 0) {
    for (int r = 0; r < kTRing; ++r) tma::mbar_init(&sm.qbar[r], 1);
    for (int r = 0; r < kARing; ++r) tma::mbar_init(&sm.abar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tma::prefetch_map(&a.q);
    tma::prefetch_map(&a.ru);
    tma::prefetch_map(&a.rv);
    tma::prefetch_map(&a.rom);
    if (ACCUM) tma::prefetch_map(&a.tend);
  }
  __syncthreads();
  auto issue_q = [&](int k) {
    const int r = (k - k0) % kTRing;
    tma::mbar_expect_tx(&sm.qbar[r], NSP * kQBytes);
#pragma unroll
    for (int m = 0; m < NSP; ++m) tma::load_4d(sm.q[r][m], &a.q, qx, j0 - 3, k, qw + m, &sm.qbar[r]);
  };
  auto issue_a = [&](int k) {
    const int r = (k - k0) % kARing;
    tma::mbar_expect_tx(&sm.abar[r], NA * kABytes);
    tma::load_4d(sm.aux[r][0], &a.ru, ax, j0, k, 0, &sm.abar[r]);
    tma::load_4d(sm.aux[r][1], &a.rv, ax, j0, k, 0, &sm.abar[r]);
    tma::load_4d(sm.aux[r][2], &a.rom, ax, j0, k + 1, 0, &sm.abar[r]);  // top face; k + 1 == nz reads zeros
    if (ACCUM) {
#pragma unroll
      for (int m = 0; m < NSP; ++m) tma::load_4d(sm.aux[r][3 + m], &a.tend, ax, j0, k, tw + m, &sm.abar[r]);
    }
  };
  // levels issued so far (thread 0's record, for the bounded drain on abort)
  int q_hi = k0 - 1, a_hi = k0 - 1;
  if (tid == 0) {
    for (int k = k0; k < min(k0 + kTRing - 1, k1); ++k) issue_q(k);
    for (int k = k0; k < min(k0 + kARing - 1, k1); ++k) issue_a(k);
    q_hi = min(k0 + kTRing - 1, k1) - 1;
    a_hi = min(k0 + kARing - 1, k1) - 1;
  }
  // column windows q(k-3 .. k+3), the values q(k1 .. k1+2) above the chunk
  // (read directly; the rings hold the chunk's own levels) and the flux
  // through the bottom face
  float win[NSP][7], wtop[NSP][3], fbot[NSP];
  const float rbot = cell && k0 < nz ? __ldg(&a.romg[k0 * lev + c]) : 0.f;
#pragma unroll
  for (int m = 0; m < NSP; ++m) {
    const float* q = a.qg[grp * NSP + m];
#pragma unroll
    for (int d = 0; d < 7; ++d) {
      const int kk = k0 - 3 + d;
      win[m][d] = (cell && kk >= 0 && kk < nz) ? __ldg(&q[kk * lev + c]) : 0.f;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int kk = k1 + d;
      wtop[m][d] = (cell && kk < nz) ? __ldg(&q[kk * lev + c]) : 0.f;
    }
    fbot[m] = zface(ktf, fnm, fnp, win[m], k0, k0, rbot);
  }
  int kstop = k1;  // the level at which a bounded wait ran out (k1: none did)
  for (int k = k0; k < k1; ++k) {
    const int it = k - k0;
    const float rdk = __ldg(&rdnw[k]);
    bool ok = tma::mbar_wait_bounded(&sm.qbar[it % kTRing], (it / kTRing) & 1, kAdvWaitCycles);
    ok = ok && tma::mbar_wait_bounded(&sm.abar[it % kARing], (it / kARing) & 1, kAdvWaitCycles);
    if (k + 3 < k1)
      ok = ok && tma::mbar_wait_bounded(&sm.qbar[(it + 3) % kTRing], ((it + 3) / kTRing) & 1,
                                        kAdvWaitCycles);
    if (__syncthreads_or(!ok)) {
      kstop = k;
      break;
    }
    // every thread is past level k-1: its ring slots take levels k+kTRing-1 / k+kARing-1
    if (tid == 0) {
      if (k + kTRing - 1 < k1) {
        issue_q(k + kTRing - 1);
        q_hi = k + kTRing - 1;
      }
      if (k + kARing - 1 < k1) {
        issue_a(k + kARing - 1);
        a_hi = k + kARing - 1;
      }
    }
    const float* A = sm.aux[it % kARing][0];
    if (k < ktf) {
#pragma unroll
      for (int m = 0; m < NSP; ++m) {
        const float* T = sm.q[it % kTRing][m];
        // x face i0 + tx of row ty; y face j0 + ty of column tx
        const float* row = T + (ty + 3) * kQW + oq;
        const float rl = A[ty * kAW + oa + tx];
        const float rs3 = rs3in ? A[ty * kAW + rs3x] : 0.f;
        if (xin) {
          const float* Q = row + tx;
          sm.fx[m][ty][tx] = rl * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], rl);
        } else {
          sm.fx[m][ty][tx] = xface(g, row, i0, i, rl, rs3);
        }
        const float* col = T + tx + 3 + oq;
        const float rb = A[kASlot + ty * kAW + oa + tx];
        if (yin) {
          const float* Q = col + ty * kQW;
          sm.fy[m][ty][tx] = rb * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], rb);
        } else {
          sm.fy[m][ty][tx] = yface<kQW>(g, col, j0, j, rb);
        }
        if (ty == 6 && tx < kTTY) {  // east faces i0 + 32, row tx
          const float* erow = T + (tx + 3) * kQW + oq;
          const float re = A[tx * kAW + oa + kTTX];
          const float rse = rs3in ? A[tx * kAW + rs3x] : 0.f;
          if (xin) {
            const float* Q = erow + kTTX;
            sm.fx[m][tx][kTTX] = re * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], re);
          } else {
            sm.fx[m][tx][kTTX] = xface(g, erow, i0, i0 + kTTX, re, rse);
          }
        }
        if (ty == 7) {  // north faces j0 + 8, column tx
          const float rn = A[kASlot + kTTY * kAW + oa + tx];
          if (yin) {
            const float* Q = col + kTTY * kQW;
            sm.fy[m][kTTY][tx] = rn * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], rn);
          } else {
            sm.fy[m][kTTY][tx] = yface<kQW>(g, col, j0, j0 + kTTY, rn);
          }
        }
      }
    }
    __syncthreads();
    const float rtop = A[2 * kASlot + ty * kAW + oa + tx];
#pragma unroll
    for (int m = 0; m < NSP; ++m) {
      // q(k+3): from the ring inside the chunk, else the direct loads
      if (k + 3 < k1) {
        win[m][6] = sm.q[(it + 3) % kTRing][m][(ty + 3) * kQW + oq + 3 + tx];
      } else {
        win[m][6] = wtop[m][0];
        wtop[m][0] = wtop[m][1];
        wtop[m][1] = wtop[m][2];
      }
      const float ftop = zface(ktf, fnm, fnp, win[m], k, k + 1, rtop);
      float* tout = a.tout[grp * NSP + m] + (size_t)k * lev + c;
      if (cell && k < ktf) {
        float t = ACCUM ? A[(3 + m) * kASlot + ty * kAW + oa + tx] : 0.f;
        if (doy) t = t - cy * (sm.fy[m][ty + 1][tx] - sm.fy[m][ty][tx]);
        if (dox) t = t - cx * (sm.fx[m][ty][tx + 1] - sm.fx[m][ty][tx]);
        t = t - rdk * (ftop - fbot[m]);
        *tout = t;
      } else if (!ACCUM && zreg) {
        *tout = 0.f;
      }
      fbot[m] = ftop;
#pragma unroll
      for (int d = 0; d < 6; ++d) win[m][d] = win[m][d + 1];
    }
  }
  if (kstop < k1 && tid == 0) {
    // let the copies still in flight land before the block's shared memory
    // goes (levels below kstop were all consumed)
    for (int k = kstop; k <= q_hi; ++k)
      tma::mbar_wait_bounded(&sm.qbar[(k - k0) % kTRing], ((k - k0) / kTRing) & 1, kAdvWaitCycles);
    for (int k = kstop; k <= a_hi; ++k)
      tma::mbar_wait_bounded(&sm.abar[(k - k0) % kARing], ((k - k0) / kARing) & 1, kAdvWaitCycles);
    atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_WAIT, 1);
  }
}

namespace {
// the TMA form applies when every row is a multiple of 16 bytes and the
// arrays are 16-byte aligned (the encoder checks the bases)
bool tma_form(const Grid& g) { return g.nx % 4 == 0 && g.ids >= 0 && g.jds >= 0; }

int nchunks(const Grid& g) { return (g.nz + kTKCH - 1) / kTKCH; }

dim3 tma_grid(const Grid& g, int ngroup) {
  return dim3((g.ide - g.ids + kTTX - 1) / kTTX, (g.jde - g.jds + kTTY - 1) / kTTY, ngroup * nchunks(g));
}

bool aux_maps(AdvTmaArgs& a, const Grid& g, const float* ru, const float* rv, const float* rom) {
  const char* err = nullptr;
  return tma::encode_f32_4d(&a.ru, ru, g.nx, g.ny, g.nz, 1, kAW, kAH, &err) &&
         tma::encode_f32_4d(&a.rv, rv, g.nx, g.ny, g.nz, 1, kAW, kAH, &err) &&
         tma::encode_f32_4d(&a.rom, rom, g.nx, g.ny, g.nz, 1, kAW, kAH, &err);
}
}  // namespace

int launch_advect_moist_tiled(const Grid& g, const S& s, cudaStream_t st) {
  const size_t n3 = g.n3();
  if (tma_form(g)) {
    AdvTmaArgs a{};
    const char* err = nullptr;
    if (tma::encode_f32_4d(&a.q, s[WF_MOIST], g.nx, g.ny, g.nz, 7, kQW, kQH, &err) &&
        aux_maps(a, g, s[WF_RU_M], s[WF_RV_M], s[WF_WW_M])) {
      a.tend = a.rom;  // unused by the non-accumulating form
      for (int m = 0; m < 6; ++m) {
        a.qg[m] = s[WF_MOIST] + (m + 1) * n3;
        a.tout[m] = s[WF_ADVECT_TEND] + (m + 1) * n3;
      }
      a.romg = s[WF_WW_M];
      a.qw0 = 1;
      a.tw0 = 1;
      a.ngroup = 3;
      a.nchunk = nchunks(g);
      k_advect_tma<2, false><<<tma_grid(g, 3), dim3(kTTX, kTTY), 0, st>>>(g, s, a);
      return 1;
    }
  }
  AdvArgs a;
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
  if (tma_form(g)) {
    AdvTmaArgs a{};
    const char* err = nullptr;
    if (tma::encode_f32_4d(&a.q, s[WF_T], g.nx, g.ny, g.nz, 1, kQW, kQH, &err) &&
        tma::encode_f32_4d(&a.tend, s[WF_T_TEND], g.nx, g.ny, g.nz, 1, kAW, kAH, &err) &&
        aux_maps(a, g, s[WF_RU], s[WF_RV], s[WF_WW])) {
      a.qg[0] = s[WF_T];
      a.tout[0] = s[WF_T_TEND];
      a.romg = s[WF_WW];
      a.qw0 = 0;
      a.tw0 = 0;
      a.ngroup = 1;
      a.nchunk = nchunks(g);
      k_advect_tma<1, true><<<tma_grid(g, 1), dim3(kTTX, kTTY), 0, st>>>(g, s, a);
      return 1;
    }
  }
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
