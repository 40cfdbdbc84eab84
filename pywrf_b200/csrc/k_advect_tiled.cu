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

// The face f (between cells f-1 and f) of [lo, hi) from the six values
// q[0..5] = q(f-3 .. f+2), the cases of xface / yface in their priority
// order but without a branch: every lane forms the 5th-, 3rd- and 2nd-order
// values and keeps its own, so a warp whose faces straddle a boundary does
// not run the cases one after another.  The hi-3 face takes its upwind sign
// from s3 (ru at ide-2 for x faces, r for y faces); the 2nd-order faces are
// r2 * (q(f) + q(f-1)) (r2 = 0.5 r for a scalar).
__device__ __forceinline__ float face_sel(const float* q, int stride, int f, int lo, int hi, float r, float s3,
                                         float r2) {
  const float q0 = q[0], q1 = q[stride], q2 = q[2 * stride], q3 = q[3 * stride], q4 = q[4 * stride],
              q5 = q[5 * stride];
  const float v5 = r * flux5(q0, q1, q2, q3, q4, q5, r);
  const float v3 = r * flux3(q1, q2, q3, q4, (f == hi - 3 && f != lo + 2) ? s3 : r);
  const float v2 = r2 * (q3 + q2);
  float v = 0.f;  // lowest priority first
  v = f == hi - 3 ? v3 : v;
  v = f == hi - 2 ? v2 : v;
  v = f == lo + 2 ? v3 : v;
  v = f == lo + 1 ? v2 : v;
  v = (f >= lo + 3 && f < hi - 3) ? v5 : v;
  return v;
}

// vertical face kf from the column window w[0..6] = q(kc-3 .. kc+3), kf in {kc, kc+1}
// (wrf_dynamics.py:1991-2015)
__device__ __forceinline__ float zface(int ktf, const float* fnm, const float* fnp, const float* w, int kc, int kf, float r) {
  auto Q = [&](int kk) { return w[kk - kc + 3]; };
  if (kf >= 3 && kf < ktf - 2) return r * flux5(Q(kf - 3), Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), Q(kf + 2), -r);
  if (kf == 1) return r * (__ldg(&fnm[1]) * Q(kf) + __ldg(&fnp[1]) * Q(kf - 1));
  if (kf == 2) return r * flux3(Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), -r);
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
  auto issue_q = [&](int k, int r) {
    tma::mbar_expect_tx(&sm.qbar[r], NSP * kQBytes);
#pragma unroll
    for (int m = 0; m < NSP; ++m) tma::load_4d(sm.q[r][m], &a.q, qx, j0 - 3, k, qw + m, &sm.qbar[r]);
  };
  auto issue_a = [&](int k, int r) {
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
    for (int k = k0; k < min(k0 + kTRing - 1, k1); ++k) issue_q(k, k - k0);
    for (int k = k0; k < min(k0 + kARing - 1, k1); ++k) issue_a(k, k - k0);
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
  // ring slots and phase parities of levels k and k+3 (scalars) and k (the rest)
  int qs = 0, q3s = 3 % kTRing, as = 0;
  uint32_t qp = 0, q3p = 3 / kTRing, ap = 0;
  auto next = [](int& slot, uint32_t& par, int ring) {
    if (++slot == ring) {
      slot = 0;
      par ^= 1u;
    }
  };
  // this thread's offsets in a scalar tile and in a per-level box
  const int offX = (ty + 3) * kQW + oq + tx;  // x face: q(i-3) of row j
  const int offY = ty * kQW + oq + 3 + tx;    // y face: q(j-3) of column i
  const int offC = offX + 3;                  // the cell itself
  const int offA = ty * kAW + oa + tx;
  float* tb[NSP];
#pragma unroll
  for (int m = 0; m < NSP; ++m) tb[m] = a.tout[grp * NSP + m] + (size_t)k0 * lev + c;
  for (int k = k0; k < k1; ++k) {
    const float rdk = __ldg(&rdnw[k]);
    bool ok = tma::mbar_wait_bounded(&sm.qbar[qs], qp, kAdvWaitCycles);
    ok = ok && tma::mbar_wait_bounded(&sm.abar[as], ap, kAdvWaitCycles);
    if (k + 3 < k1) ok = ok && tma::mbar_wait_bounded(&sm.qbar[q3s], q3p, kAdvWaitCycles);
    if (__syncthreads_or(!ok)) {
      kstop = k;
      break;
    }
    // every thread is past level k-1: its ring slots take levels k+kTRing-1 / k+kARing-1
    if (tid == 0) {
      if (k + kTRing - 1 < k1) {
        issue_q(k + kTRing - 1, qs == 0 ? kTRing - 1 : qs - 1);
        q_hi = k + kTRing - 1;
      }
      if (k + kARing - 1 < k1) {
        issue_a(k + kARing - 1, as == 0 ? kARing - 1 : as - 1);
        a_hi = k + kARing - 1;
      }
    }
    const float* A = sm.aux[as][0];
    const float* T0 = sm.q[qs][0];
    if (k < ktf) {
      const float rl = A[offA];
      const float rb = A[kASlot + offA];
      const float rs3 = rs3in ? A[ty * kAW + rs3x] : 0.f;
#pragma unroll
      for (int m = 0; m < NSP; ++m) {
        const float* T = T0 + m * kQSlot;
        // x face i0 + tx of row ty; y face j0 + ty of column tx
        if (xin) {
          const float* Q = T + offX;
          sm.fx[m][ty][tx] = rl * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], rl);
        } else {
          sm.fx[m][ty][tx] = face_sel(T + offX, 1, i, ids, ide, rl, rs3, 0.5f * rl);
        }
        if (yin) {
          const float* Q = T + offY;
          sm.fy[m][ty][tx] = rb * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], rb);
        } else {
          sm.fy[m][ty][tx] = yface<kQW>(g, T + tx + 3 + oq, j0, j, rb);
        }
        if (ty == 6 && tx < kTTY) {  // east faces i0 + 32, row tx
          const float* erow = T + (tx + 3) * kQW + oq;
          const float re = A[tx * kAW + oa + kTTX];
          const float rse = rs3in ? A[tx * kAW + rs3x] : 0.f;
          if (xin) {
            const float* Q = erow + kTTX;
            sm.fx[m][tx][kTTX] = re * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], re);
          } else {
            sm.fx[m][tx][kTTX] = face_sel(erow + kTTX, 1, i0 + kTTX, ids, ide, re, rse, 0.5f * re);
          }
        }
        if (ty == 7) {  // north faces j0 + 8, column tx
          const float rn = A[kASlot + kTTY * kAW + oa + tx];
          const float* col = T + tx + 3 + oq;
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
    const float rtop = A[2 * kASlot + offA];
    const float* T3 = sm.q[q3s][0];
#pragma unroll
    for (int m = 0; m < NSP; ++m) {
      // q(k+3): from the ring inside the chunk, else the direct loads
      if (k + 3 < k1) {
        win[m][6] = T3[m * kQSlot + offC];
      } else {
        win[m][6] = wtop[m][0];
        wtop[m][0] = wtop[m][1];
        wtop[m][1] = wtop[m][2];
      }
      const float ftop = zface(ktf, fnm, fnp, win[m], k, k + 1, rtop);
      if (cell && k < ktf) {
        float t = ACCUM ? A[(3 + m) * kASlot + offA] : 0.f;
        if (doy) t = t - cy * (sm.fy[m][ty + 1][tx] - sm.fy[m][ty][tx]);
        if (dox) t = t - cx * (sm.fx[m][ty][tx + 1] - sm.fx[m][ty][tx]);
        t = t - rdk * (ftop - fbot[m]);
        *tb[m] = t;
      } else if (!ACCUM && zreg) {
        *tb[m] = 0.f;
      }
      tb[m] += lev;
      fbot[m] = ftop;
#pragma unroll
      for (int d = 0; d < 6; ++d) win[m][d] = win[m][d + 1];
    }
    next(qs, qp, kTRing);
    next(q3s, q3p, kTRing);
    next(as, ap, kARing);
  }
  if (kstop < k1 && tid == 0) {
    // let the copies still in flight land before the block's shared memory
    // goes (levels below kstop were all consumed)
    for (int k = kstop; k <= q_hi; ++k)
      tma::mbar_wait_bounded(&sm.qbar[(k - k0) % kTRing], ((k - k0) / kTRing) & 1, kAdvWaitCycles);
    for (int k = kstop; k <= a_hi; ++k)
      tma::mbar_wait_bounded(&sm.abar[(k - k0) % kARing], ((k - k0) / kARing) & 1, kAdvWaitCycles);
    if (s[WF_STATUS]) atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_WAIT, 1);
  }
}

// ------------------------------------------------------------------------
// Momentum advection, TMA form: advect_u, advect_v, advect_w
// (wrf_dynamics.py:1112-1823) on the same plan as the scalar kernel above -
// one launch, blockIdx.z = component * chunks + chunk; a 32 x 8 tile of the
// component's cells per block, its field tile (box 44 x 14) and the level's
// coupled velocities and tendency (boxes 40 x 10 from x = floor4(i0 - 1),
// y = j0 - 1, so that the i-1 and j-1 neighbours of every face are in the box)
// streamed through mbarrier rings.  Face formulas and their order are those of
// the point kernel (k_tend.cu: fqx_u .. vf_w); boundary blocks take the
// branch-free select forms.

// the face f of a momentum component normal to it (u in x, v in y) of
// [lo, hi) from q[0..5] = q(f-3 .. f+2) and the coupled velocities ra, rb
// either side (wrf_dynamics.py:1212-1246, 1373-1407): upwind 2nd order at
// lo+1 and hi-1, 3rd order at lo+2 and hi-2, 5th order between
__device__ __forceinline__ float face_normal(const float* q, int stride, int f, int lo, int hi, float ra, float rb) {
  const float q0 = q[0], q1 = q[stride], q2 = q[2 * stride], q3 = q[3 * stride], q4 = q[4 * stride],
              q5 = q[5 * stride];
  const float vel = 0.5f * (ra + rb);
  const float r4 = 0.25f * (ra + rb);
  const float v5 = vel * flux5(q0, q1, q2, q3, q4, q5, vel);
  const float v3 = vel * flux3(q1, q2, q3, q4, vel);
  const float vl = r4 * (q3 + (q3 < 0.f ? q3 : q2));
  const float vh = r4 * (q2 + (q2 > 0.f ? q2 : q3));
  float v = 0.f;  // lowest priority first
  v = f == hi - 2 ? v3 : v;
  v = f == hi - 1 ? vh : v;
  v = f == lo + 2 ? v3 : v;
  v = f == lo + 1 ? vl : v;
  v = (f >= lo + 3 && f < hi - 2) ? v5 : v;
  return v;
}

// vertical face of v (vf_v, wrf_dynamics.py:1482-1524): zface with +vel on the ktf-2 face
__device__ __forceinline__ float zface_v(int ktf, const float* fnm, const float* fnp, const float* w, int kc, int kf,
                                         float r) {
  auto Q = [&](int kk) { return w[kk - kc + 3]; };
  if (kf >= 3 && kf < ktf - 2) return r * flux5(Q(kf - 3), Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), Q(kf + 2), -r);
  if (kf == 1) return r * (__ldg(&fnm[1]) * Q(kf) + __ldg(&fnp[1]) * Q(kf - 1));
  if (kf == 2) return r * flux3(Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), -r);
  if (kf == ktf - 2) return r * flux3(Q(kf - 2), Q(kf - 1), Q(kf), Q(kf + 1), r);
  if (kf == ktf - 1) return r * (__ldg(&fnm[kf]) * Q(kf) + __ldg(&fnp[kf]) * Q(kf - 1));
  return 0.f;
}

// vertical face of w at mass level kf (vf_w, wrf_dynamics.py:1773-1811),
// ra = rom(kf), rb = rom(kf-1)
__device__ __forceinline__ float zface_w(int ktf, const float* w, int kc, int kf, float ra, float rb) {
  auto W = [&](int kk) { return w[kk - kc + 3]; };
  if (kf >= 3 && kf < ktf - 1) {
    const float v = 0.5f * (ra + rb);
    return v * flux5(W(kf - 3), W(kf - 2), W(kf - 1), W(kf), W(kf + 1), W(kf + 2), -v);
  }
  if (kf == 1) return 0.25f * (ra + rb) * (W(kf) + W(kf - 1));
  if (kf == 2) {
    const float v = 0.5f * (ra + rb);
    return v * flux3(W(kf - 2), W(kf - 1), W(kf), W(kf + 1), -v);
  }
  if (kf == ktf - 1) {
    const float v = 0.5f * (ra + rb);
    return v * flux3(W(kf - 2), W(kf - 1), W(kf), W(kf + 1), v);
  }
  if (kf == ktf) return 0.25f * (ra + rb) * (W(kf) + W(kf - 1));
  return 0.f;
}

constexpr int kMW = 40, kMH = kTTY + 2;        // per-level box of the momentum kernel
constexpr uint32_t kMBytes = kMW * kMH * 4;
constexpr int kMSlot = 416;                    // floats per box slot (1664 B)
constexpr int kMomKCH = 10;
static_assert(kMBytes <= kMSlot * 4 && (kMSlot * 4) % 128 == 0, "a ring slot holds one box");

struct MomTmaArgs {
  CUtensorMap q[3];               // u, v, w: box kQW x kQH
  CUtensorMap ru, rv, rom;        // box kMW x kMH
  CUtensorMap tend[3];            // ru_tend, rv_tend, rw_tend
  const float* qg[3];
  float* tout[3];
  const float* romg;
  int nchunk, comp0;  // blockIdx.z = (component - comp0) * nchunk + chunk
};

// per-level boxes: u, v: ru(k) rv(k) rom(k+1) tend(k); w: ru(k) ru(k-1) rv(k)
// rv(k-1) rom(k+1) tend(k) (at the top level ru, rv of ktf-1 and ktf-2)
template <int C>
struct MomLayout {
  static constexpr int NA = C == 2 ? 6 : 4;
};
constexpr int kMomSmemFloats = kTRing * kQSlot + kARing * 6 * kMSlot + kTTY * (kTTX + 1) + (kTTY + 1) * kTTX;

template <int C>
__device__ __forceinline__ void advect_mom_block(const Grid& g, const S& s, const MomTmaArgs& a, float* smf,
                                                 uint64_t* qbar, uint64_t* abar, int chunk) {
  constexpr int NA = MomLayout<C>::NA;
  float* sq = smf;                                      // [kTRing][kQSlot]
  float* saux = smf + kTRing * kQSlot;                  // [kARing][NA][kMSlot]
  float (*fx)[kTTX + 1] = reinterpret_cast<float (*)[kTTX + 1]>(saux + kARing * 6 * kMSlot);
  float (*fy)[kTTX] = reinterpret_cast<float (*)[kTTX]>(saux + kARing * 6 * kMSlot + kTTY * (kTTX + 1));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTTX + tx;
  const int nx = g.nx, ny = g.ny, nz = g.nz, ktf = nz - 1;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int i0 = ids + blockIdx.x * kTTX, j0 = jds + blockIdx.y * kTTY;
  const int i = i0 + tx, j = j0 + ty;
  const int qx = (i0 - 3) & ~3, mx = (i0 - 1) & ~3;
  const int oq = i0 - 3 - qx, om = i0 - mx;  // om in 1..4
  const size_t lev = (size_t)ny * nx;
  // levels: u, v 0 .. ktf-1; w 1 .. ktf
  const int kb = C == 2 ? 1 : 0, nlev = ktf;
  const int k0 = kb + chunk * nlev / a.nchunk, k1 = kb + (chunk + 1) * nlev / a.nchunk;
  bool cell, doy, dox;
  float msf_y, msf_x, zfac = 0.f;
  const int c = min(j, ny - 1) * nx + min(i, nx - 1);
  if (C == 0) {
    cell = j < jde - 1 && i >= ids + 1 && i < ide - 1;
    doy = j >= jds + 1 && j < jde - 2;
    dox = true;
    const float m = cell ? __ldg(&s[WF_MSFUX][c]) : 0.f;
    msf_y = m * g.rdy;
    msf_x = m * g.rdx;
  } else if (C == 1) {
    cell = j >= jds + 1 && j < jde - 1 && i < ide - 1;
    doy = true;
    dox = i >= ids + 1 && i < ide - 2;
    const float my = cell ? __ldg(&s[WF_MSFVY][c]) : 0.f;
    const float mxv = cell ? __ldg(&s[WF_MSFVX][c]) : 1.f;
    msf_y = my * g.rdy;
    msf_x = my * g.rdx;
    zfac = my / mxv;
  } else {
    cell = j < jde - 1 && i < ide - 1;
    doy = j >= jds + 1 && j < jde - 2;
    dox = i >= ids + 1 && i < ide - 2;
    const float m = cell ? __ldg(&s[WF_MSFTX][c]) : 0.f;
    msf_y = m * g.rdy;
    msf_x = m * g.rdx;
  }
  // whole block in the 5th-order region of its faces (x faces i0 .. i0+32, y faces j0 .. j0+8)
  const bool xin = C == 0 ? (i0 >= ids + 3 && i0 + kTTX < ide - 2) : (i0 >= ids + 3 && i0 + kTTX < ide - 3);
  const bool yin = C == 1 ? (j0 >= jds + 3 && j0 + kTTY < jde - 2) : (j0 >= jds + 3 && j0 + kTTY < jde - 3);
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdz = C == 2 ? s[WF_RDN] : s[WF_RDNW];

  if (tid == 0) {
    for (int r = 0; r < kTRing; ++r) tma::mbar_init(&qbar[r], 1);
    for (int r = 0; r < kARing; ++r) tma::mbar_init(&abar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tma::prefetch_map(&a.q[C]);
    tma::prefetch_map(&a.ru);
    tma::prefetch_map(&a.rv);
    tma::prefetch_map(&a.rom);
    tma::prefetch_map(&a.tend[C]);
  }
  __syncthreads();
  auto issue_q = [&](int k, int r) {
    tma::mbar_expect_tx(&qbar[r], kQBytes);
    tma::load_4d(sq + r * kQSlot, &a.q[C], qx, j0 - 3, k, 0, &qbar[r]);
  };
  auto issue_a = [&](int k, int r) {
    float* d = saux + r * NA * kMSlot;
    tma::mbar_expect_tx(&abar[r], NA * kMBytes);
    if (C == 2) {
      const int kr = k < ktf ? k : ktf - 1;  // wvel's levels: k, k-1 (top: ktf-1, ktf-2)
      tma::load_4d(d + 0 * kMSlot, &a.ru, mx, j0 - 1, kr, 0, &abar[r]);
      tma::load_4d(d + 1 * kMSlot, &a.ru, mx, j0 - 1, kr - 1, 0, &abar[r]);
      tma::load_4d(d + 2 * kMSlot, &a.rv, mx, j0 - 1, kr, 0, &abar[r]);
      tma::load_4d(d + 3 * kMSlot, &a.rv, mx, j0 - 1, kr - 1, 0, &abar[r]);
      tma::load_4d(d + 4 * kMSlot, &a.rom, mx, j0 - 1, k + 1, 0, &abar[r]);  // k + 1 == nz reads zeros
      tma::load_4d(d + 5 * kMSlot, &a.tend[C], mx, j0 - 1, k, 0, &abar[r]);
    } else {
      tma::load_4d(d + 0 * kMSlot, &a.ru, mx, j0 - 1, k, 0, &abar[r]);
      tma::load_4d(d + 1 * kMSlot, &a.rv, mx, j0 - 1, k, 0, &abar[r]);
      tma::load_4d(d + 2 * kMSlot, &a.rom, mx, j0 - 1, k + 1, 0, &abar[r]);
      tma::load_4d(d + 3 * kMSlot, &a.tend[C], mx, j0 - 1, k, 0, &abar[r]);
    }
  };
  int q_hi = k0 - 1, a_hi = k0 - 1;
  if (tid == 0) {
    for (int k = k0; k < min(k0 + kTRing - 1, k1); ++k) issue_q(k, k - k0);
    for (int k = k0; k < min(k0 + kARing - 1, k1); ++k) issue_a(k, k - k0);
    q_hi = min(k0 + kTRing - 1, k1) - 1;
    a_hi = min(k0 + kARing - 1, k1) - 1;
  }
  // column window of the component, its values above the chunk, the bottom-face flux
  const float* qg = a.qg[C];
  float win[7], wtop[3];
#pragma unroll
  for (int d = 0; d < 7; ++d) {
    const int kk = k0 - 3 + d;
    win[d] = (cell && kk >= 0 && kk < nz) ? __ldg(&qg[kk * lev + c]) : 0.f;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int kk = k1 + d;
    wtop[d] = (cell && kk < nz) ? __ldg(&qg[kk * lev + c]) : 0.f;
  }
  float fbot, rprev = 0.f;
  {
    const float* rom = a.romg;
    if (C == 0) {
      const float vel = cell ? 0.5f * (__ldg(&rom[k0 * lev + c]) + __ldg(&rom[k0 * lev + c - 1])) : 0.f;
      fbot = zface(ktf, fnm, fnp, win, k0, k0, vel);
    } else if (C == 1) {
      const float vel = cell ? 0.5f * (__ldg(&rom[k0 * lev + c]) + __ldg(&rom[k0 * lev + c - nx])) : 0.f;
      fbot = zface_v(ktf, fnm, fnp, win, k0, k0, vel);
    } else {
      rprev = cell ? __ldg(&rom[k0 * lev + c]) : 0.f;
      const float rb = cell ? __ldg(&rom[(k0 - 1) * lev + c]) : 0.f;
      fbot = zface_w(ktf, win, k0, k0, rprev, rb);
    }
  }
  int kstop = k1;
  int qs = 0, q3s = 3 % kTRing, as = 0;
  uint32_t qp = 0, q3p = 3 / kTRing, ap = 0;
  auto next = [](int& slot, uint32_t& par, int ring) {
    if (++slot == ring) {
      slot = 0;
      par ^= 1u;
    }
  };
  const int offX = (ty + 3) * kQW + oq + tx;  // x face f = i: q(f-3) of row j
  const int offY = ty * kQW + oq + 3 + tx;    // y face jf = j: q(jf-3) of column i
  const int offC = offX + 3;                  // the cell
  const int oA = (ty + 1) * kMW + om + tx;    // (j, i) in a per-level box; -1: i-1, -kMW: j-1
  float* tb = a.tout[C] + (size_t)k0 * lev + c;
  for (int k = k0; k < k1; ++k) {
    const float rdk = __ldg(&rdz[C == 2 && k == ktf ? ktf - 1 : k]);
    bool ok = tma::mbar_wait_bounded(&qbar[qs], qp, kAdvWaitCycles);
    ok = ok && tma::mbar_wait_bounded(&abar[as], ap, kAdvWaitCycles);
    if (k + 3 < k1) ok = ok && tma::mbar_wait_bounded(&qbar[q3s], q3p, kAdvWaitCycles);
    if (__syncthreads_or(!ok)) {
      kstop = k;
      break;
    }
    if (tid == 0) {
      if (k + kTRing - 1 < k1) {
        issue_q(k + kTRing - 1, qs == 0 ? kTRing - 1 : qs - 1);
        q_hi = k + kTRing - 1;
      }
      if (k + kARing - 1 < k1) {
        issue_a(k + kARing - 1, as == 0 ? kARing - 1 : as - 1);
        a_hi = k + kARing - 1;
      }
    }
    const float* A = saux + as * NA * kMSlot;
    const float* T = sq + qs * kQSlot;
    // w's interpolation of ru / rv to level k (top: extrapolated from ktf-1, ktf-2)
    float c0 = 0.f, c1 = 0.f;
    if (C == 2) {
      if (k < ktf) {
        c0 = __ldg(&fnm[k]);
        c1 = __ldg(&fnp[k]);
      } else {
        c0 = 2.0f - __ldg(&fnm[ktf - 1]);
        c1 = -__ldg(&fnp[ktf - 1]);
      }
    }
    // the faces west / south of the cell, and the tile's east / north faces
    auto xflux = [&](const float* Q, int f, int o) -> float {  // o: box index of (row, f)
      if (C == 0) {
        const float ra = A[o], rb = A[o - 1];
        if (xin) {
          const float vel = 0.5f * (ra + rb);
          return vel * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], vel);
        }
        return face_normal(Q, 1, f, ids, ide, ra, rb);
      } else if (C == 1) {
        const float R = A[o] + A[o - kMW];
        const float w = 0.5f * R;
        if (xin) return w * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], w);
        return face_sel(Q, 1, f, ids, ide, w, w, 0.25f * R);
      } else {
        const float vel = c0 * A[o] + c1 * A[kMSlot + o];
        if (xin) return vel * flux5(Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], vel);
        return face_sel(Q, 1, f, ids, ide, vel, vel, 0.5f * vel);
      }
    };
    auto yflux = [&](const float* Q, int f, int o) -> float {  // o: box index of (f, column)
      if (C == 0) {
        const float ra = A[kMSlot + o], rb = A[kMSlot + o - 1];
        const float vel = 0.5f * (ra + rb);
        if (yin) return vel * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], vel);
        return face_sel(Q, kQW, f, jds, jde, vel, 0.0f, 0.25f * (ra + rb));
      } else if (C == 1) {
        const float ra = A[kMSlot + o], rb = A[kMSlot + o - kMW];
        if (yin) {
          const float vel = 0.5f * (ra + rb);
          return vel * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], vel);
        }
        return face_normal(Q, kQW, f, jds, jde, ra, rb);
      } else {
        const float vel = c0 * A[2 * kMSlot + o] + c1 * A[3 * kMSlot + o];
        if (yin) return vel * flux5(Q[0], Q[kQW], Q[2 * kQW], Q[3 * kQW], Q[4 * kQW], Q[5 * kQW], vel);
        return face_sel(Q, kQW, f, jds, jde, vel, vel, 0.5f * vel);
      }
    };
    const bool faces = C == 2 || k < ktf;
    if (faces) {
      fx[ty][tx] = xflux(T + offX, i, oA);
      fy[ty][tx] = yflux(T + offY, j, oA);
      if (ty == 6 && tx < kTTY)  // east faces i0 + 32, row tx
        fx[tx][kTTX] = xflux(T + (tx + 3) * kQW + oq + kTTX, i0 + kTTX, (tx + 1) * kMW + om + kTTX);
      if (ty == 7)  // north faces j0 + 8, column tx
        fy[kTTY][tx] = yflux(T + kTTY * kQW + oq + 3 + tx, j0 + kTTY, (kTTY + 1) * kMW + om + tx);
    }
    __syncthreads();
    // q(k+3): from the ring inside the chunk, else the direct loads
    if (k + 3 < k1) {
      win[6] = sq[q3s * kQSlot + offC];
    } else {
      win[6] = wtop[0];
      wtop[0] = wtop[1];
      wtop[1] = wtop[2];
    }
    float ftop = 0.f;
    if (C == 0) {
      ftop = zface(ktf, fnm, fnp, win, k, k + 1, 0.5f * (A[2 * kMSlot + oA] + A[2 * kMSlot + oA - 1]));
    } else if (C == 1) {
      ftop = zface_v(ktf, fnm, fnp, win, k, k + 1, 0.5f * (A[2 * kMSlot + oA] + A[2 * kMSlot + oA - kMW]));
    } else if (k < ktf) {
      const float ra = A[4 * kMSlot + oA];
      ftop = zface_w(ktf, win, k, k + 1, ra, rprev);
      rprev = ra;
    }
    if (cell) {
      float t = A[(NA - 1) * kMSlot + oA];
      if (doy) t = t - msf_y * (fy[ty + 1][tx] - fy[ty][tx]);
      if (dox) t = t - msf_x * (fx[ty][tx + 1] - fx[ty][tx]);
      if (C == 1) {
        t = t - (zfac * rdk) * (ftop - fbot);
      } else if (C == 2 && k == ktf) {
        t = t + 2.0f * rdk * fbot;
      } else {
        t = t - rdk * (ftop - fbot);
      }
      *tb = t;
    }
    tb += lev;
    fbot = ftop;
#pragma unroll
    for (int d = 0; d < 6; ++d) win[d] = win[d + 1];
    next(qs, qp, kTRing);
    next(q3s, q3p, kTRing);
    next(as, ap, kARing);
  }
  if (kstop < k1 && tid == 0) {
    for (int k = kstop; k <= q_hi; ++k)
      tma::mbar_wait_bounded(&qbar[(k - k0) % kTRing], ((k - k0) / kTRing) & 1, kAdvWaitCycles);
    for (int k = kstop; k <= a_hi; ++k)
      tma::mbar_wait_bounded(&abar[(k - k0) % kARing], ((k - k0) / kARing) & 1, kAdvWaitCycles);
    if (s[WF_STATUS]) atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_WAIT, 1);
  }
}

__global__ void __launch_bounds__(kTTX * kTTY, WRF_ADV_MINB) k_advect_mom_tma(Grid g, S s,
                                                                             const __grid_constant__ MomTmaArgs a) {
  __shared__ __align__(128) float smf[kMomSmemFloats];
  __shared__ uint64_t qbar[kTRing], abar[kARing];
  const int comp = a.comp0 + blockIdx.z / a.nchunk, chunk = blockIdx.z % a.nchunk;
  if (comp == 0)
    advect_mom_block<0>(g, s, a, smf, qbar, abar, chunk);
  else if (comp == 1)
    advect_mom_block<1>(g, s, a, smf, qbar, abar, chunk);
  else
    advect_mom_block<2>(g, s, a, smf, qbar, abar, chunk);
}

namespace {
// the TMA form applies when every row is a multiple of 16 bytes and the
// arrays are 16-byte aligned (the encoder checks the bases)
bool tma_form(const Grid& g) { return kernel_form() == WRF_FORM_FAST && g.nx % 4 == 0 && g.ids >= 0 && g.jds >= 0; }

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

// advection of the momentum components comp0 .. comp0+ncomp-1 (0 u, 1 v,
// 2 w) into ru_tend / rv_tend / rw_tend (TMA form); returns 0 (nothing
// launched) when the arrays do not allow tensor maps
int launch_advect_mom_tma(const Grid& g, const S& s, int comp0, int ncomp, cudaStream_t st) {
  if (!tma_form(g) || g.nz < 4 || comp0 < 0 || ncomp < 1 || comp0 + ncomp > 3) return 0;
  MomTmaArgs a{};
  const char* err = nullptr;
  const int f[3] = {WF_U, WF_V, WF_W}, t[3] = {WF_RU_TEND, WF_RV_TEND, WF_RW_TEND};
  for (int m = comp0; m < comp0 + ncomp; ++m) {
    if (!tma::encode_f32_4d(&a.q[m], s[f[m]], g.nx, g.ny, g.nz, 1, kQW, kQH, &err) ||
        !tma::encode_f32_4d(&a.tend[m], s[t[m]], g.nx, g.ny, g.nz, 1, kMW, kMH, &err))
      return 0;
    a.qg[m] = s[f[m]];
    a.tout[m] = s[t[m]];
  }
  if (!tma::encode_f32_4d(&a.ru, s[WF_RU], g.nx, g.ny, g.nz, 1, kMW, kMH, &err) ||
      !tma::encode_f32_4d(&a.rv, s[WF_RV], g.nx, g.ny, g.nz, 1, kMW, kMH, &err) ||
      !tma::encode_f32_4d(&a.rom, s[WF_WW], g.nx, g.ny, g.nz, 1, kMW, kMH, &err))
    return 0;
  a.romg = s[WF_WW];
  a.nchunk = min((g.nz - 1 + kMomKCH - 1) / kMomKCH, g.nz - 1);
  a.comp0 = comp0;
  const dim3 gr((g.ide - g.ids + kTTX - 1) / kTTX, (g.jde - g.jds + kTTY - 1) / kTTY, ncomp * a.nchunk);
  k_advect_mom_tma<<<gr, dim3(kTTX, kTTY), 0, st>>>(g, s, a);
  return 1;
}

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
