// Hand-written adjoints of step operators (reverse mode, one cotangent per call).
//
//   k_advect_scalar_faces + k_advect_scalar_gather
//                        adjoint of advect_scalar (wrf_dynamics.py:1841-2028,
//                        forward: k_advect_scalar / k_advect_tiled) with
//                        respect to the advected field and the three mass
//                        fluxes ru, rv, rom.
//
// Forward, per mass point c of [ids, ide-1) x [jds, jde-1) x [0, nz-1):
//   tend(c) -= a_y(c) (Fy(j+1) - Fy(j)) + a_x(c) (Fx(i+1) - Fx(i)) + rdnw(k) (Fz(k+1) - Fz(k))
// with a_y = msftx rdy on rows [jds+1, jde-2) (else 0), a_x likewise, and each
// face flux F = r Phi(q; sign r), Phi the 5th-, 3rd- or 2nd-order face value
// the reference selects for that face (fortran_sign(1, r) upwinding; minus
// sign of rom vertically).  The sign is piecewise constant, so
//   Fbar(f)  = a(cell above f) tbar(cell above) - a(cell below f) tbar(cell below)
//   qbar(m) += sum over faces f whose stencil holds m of Fbar(f) r(f) dPhi_f/dq(m)
//   rbar(f) += Fbar(f) Phi(f)
// The faces pass forms each face once (its rbar, and its field terms stored
// by stencil offset in 18 slot arrays of caller work); the gather pass sums,
// per point, the slots that address it in a fixed order.  Each output
// element is written by one thread, so results do not depend on scheduling;
// tend's own cotangent is tbar unchanged (the caller passes it through).
//
//   k_advect_mom_faces<C> + k_advect_mom_gather<C>
//                        adjoint of advect_u (C = 0, wrf_dynamics.py:1112-1331),
//                        advect_v (1, :1332-1534) and advect_w (2, :1535-1823),
//                        forward k_advect / k_advect_mom_tma, with respect to
//                        the advected component and ru, rv, rom.  Every face
//                        flux of those operators is a product F = V Phi of a
//                        velocity V linear in one of ru / rv / rom (a two-point
//                        average, or the fnm / fnp interpolation of advect_w's
//                        horizontal faces) and a face value Phi linear in the
//                        component for fixed upwind choices (the sign of V, or
//                        of the component itself at advect_u's / advect_v's
//                        outermost faces).  face_lin<C, D> lists both linear
//                        forms of a face.  k_advect_mom_faces<C> forms each
//                        face once and stores its contributions by stencil
//                        slot, k_advect_mom_gather<C> sums, per point, the
//                        slots that address it:
//   qbar(m) += sum_f Fbar(f) V(f) dPhi_f/dq(m),  rbar(n) += sum_f Fbar(f) Phi(f) dV_f/dr(n)
//                        with Fbar(f) from the tendency cotangent of the cells
//                        either side of f (one writer per output element).
//
//   k_advance_uv_adj / k_advance_uv_adj_col  adjoint of advance_uv
//                        (wrf_dynamics.py:3391-3525) with spec_bdyupdate of
//                        u and v (wrf_boundary.py:244-290), forward
//                        k_advance_uv / k_advance_uv_tma.  At an updated
//                        u point, u' = u + dts ru_tend - dts cqu dp + mudf_xy
//                        with dp = A B + C D:
//     A = r rdx muu / 2,  B = dph(k+1) + dph(k) + (alt + alt_w) dp_x + (al + al_w) dpb_x,
//     C = r rdx dphp_x,   D = rdnw(k) (dpn(k+1) - dpn(k)) - (mu + mu_w) / 2
//                        (r = msfux / msfuy, _w the west neighbour, _x the
//                        difference to it, dpn the vertical pressure average
//                        of the two columns); v likewise in y.  The point
//                        kernel gathers the 3-D cotangents from the u and v
//                        points whose stencils hold the point (forming of
//                        each only the factors that reach the point), the column
//                        kernel sums the 2-D ones (muu, muv, mu, mudf) over
//                        the levels.  The cotangents of u and v pass through
//                        (du'/du = 1).
//
//   k_calc_p_rho / k_calc_p_rho_adj*  calc_p_rho (wrf_dynamics.py:3269-3313)
//                        on the mass points: al = -(alt mu + rdnw dph) / mut,
//                        p1 = c2a (alt (t_2 - mu t_1) / (mut (t0 + t_1)) - al),
//                        then p = p1, pm1 = p (the whole array) at step 0, or
//                        p = p1 + smdiv (p1 - pm1), pm1 = p1 after it.  The
//                        adjoint runs in three passes - the 3-D cotangents
//                        (ph gathered from the two cells either side of a
//                        level), the 2-D ones (mu, mut summed over the column)
//                        and last the in-place rewrite of the cotangents of
//                        al, p, pm1 from those of the outputs to those of the
//                        inputs - so no pass reads what another writes.
//
//   k_advance_mu_t / k_advance_mu_t_adj_*  advance_mu_t (wrf_dynamics.py:
//                        3528-3638) on the columns [ids+1, ide-2) x [jds+1,
//                        jde-2): the horizontal divergence dvdxi(k), its
//                        column sum dmdt, the mu / mudf / muts / muave update,
//                        the ww scan W(k) = W(k-1) - dnw(k-1) (dmdt + dvdxi(k-1)
//                        + mu_tend) / msfty (ww' = W - ww_1) and the theta
//                        update with the fluxes wdtn = ww' (fnm t_1 + fnp t_1).
//                        The adjoint: (1) per column, the cotangent of
//                        dvdxi at every level into the caller's work array
//                        (reverse ww scan as a suffix sum); (2) per point, the
//                        gathers of u, v, u_1, v_1 and the horizontal part of
//                        t_1 from the columns whose stencils hold the point;
//                        (3) per column, muu, muv from the work array, the
//                        column-local cotangents and the in-place rewrite of
//                        those of the outputs (ww, t, t_ave, mu, muts, mudf,
//                        muave) to those of the inputs.  With ref_no_grad the
//                        mu / muts / mudf / muave update is treated as the
//                        reference's autograd sees it (computed under
//                        torch.no_grad(): each passes its cotangent to the
//                        input of the same name and nothing to dmdt, mut or
//                        mu_tend).
//
//   k_advance_w_lp / k_advance_w_adj_lp / k_advance_w_adj_bc  advance_w
//                        (wrf_dynamics.py:3641-3796) on the columns [ids+1,
//                        ide-2) x [jds+1, jde-2): t_2ave, the right-hand side
//                        rhs = ph + msfty R / mut (R from ph_tend, w and the
//                        vertical phi fluxes wdwn), the explicit w x(k), the
//                        lower boundary x(0) from the terrain slope and the
//                        near-surface winds, the implicit solve with a, alpha,
//                        gamma, the Rayleigh damping of the upper levels and
//                        the phi update.  The adjoint runs each column's
//                        chain backwards over a block's level groups (forward
//                        values recomputed into shared column arrays, the
//                        per-level parts on all threads in gather form, the
//                        solve transposed as in k_vsolve_w_adj on one thread
//                        per column; the damping weight's sin^2
//                        differentiated in ph_1 and phb through hk and htop)
//                        and leaves the cotangent of x(0) in a work array, from
//                        which a second kernel gathers those of u, v (levels
//                        0..2) and ht.
//
//   k_relax_field / k_relax_field_adj  relax_bdytend (wrf_boundary.py:52-147)
//                        on one field, and its adjoint with respect to the
//                        field: at a relaxation point P of distance b,
//   tend(P) += fcx_b f0 - gcx_b (f1 + f2 + f3 + f4 - 4 f0),  fN = bdy_N - field(N)
//                        so field(P) carries -(fcx_b + 4 gcx_b) and each of its
//                        four neighbours +gcx_b.  The adjoint gathers, for each
//                        point m, its own term and its neighbours' terms.
//
//   k_vsolve_w / k_vsolve_w_adj  the vertically implicit w solve of
//                        advance_w (wrf_dynamics.py:3761-3767) on every
//                        column, and its transposed (adjoint) solve with
//                        respect to the right-hand side and the coefficients
//                        a, alpha, gamma of calc_coef_w:
//   y(0) = x(0);  y(k) = (x(k) - a(k) y(k-1)) alpha(k),  k = 1..nz-1
//   w(nz-1) = y(nz-1);  w(k) = y(k) - gamma(k) w(k+1),  k = nz-2..1;  w(0) = y(0)
//                        The reverse sweep runs the two recurrences backwards
//                        (one thread per column; the column's y and w are
//                        recomputed into local arrays).
//
//   k_coef_w_adj         adjoint of calc_coef_w (wrf_dynamics.py:3316-3388)
//                        with respect to cqw, c2a and mut: the column's
//                        forward recurrence alpha(k) = 1 / (b(k) - a(k)
//                        gamma(k-1)), gamma(k) = c(k) alpha(k) is recomputed
//                        into local arrays and run backwards.
#include "kernels.cuh"
#include "relax.cuh"

namespace wrf {
namespace {

// dPhi/dq at stencil offset o = m - f of a 5th-order face (o in [-3, 2]),
// Phi = (37(q0+qm1) - 8(qp1+qm2) + (qp2+qm3))/60 - s ((qp2-qm3) - 5(qp1-qm2) + 10(q0-qm1))/60
__device__ __forceinline__ float w5(int o, float s) {
  switch (o) {
    case -3: return (1.f + s) * (1.f / 60.f);
    case -2: return (-8.f - 5.f * s) * (1.f / 60.f);
    case -1: return (37.f + 10.f * s) * (1.f / 60.f);
    case 0: return (37.f - 10.f * s) * (1.f / 60.f);
    case 1: return (-8.f + 5.f * s) * (1.f / 60.f);
    case 2: return (1.f - s) * (1.f / 60.f);
    default: return 0.f;
  }
}

// 3rd-order face, o in [-2, 1]:
// Phi = (7(q0+qm1) - (qp1+qm2))/12 + s ((qp1-qm2) - 3(q0-qm1))/12
__device__ __forceinline__ float w3(int o, float s) {
  switch (o) {
    case -2: return (-1.f - s) * (1.f / 12.f);
    case -1: return (7.f + 3.f * s) * (1.f / 12.f);
    case 0: return (7.f - 3.f * s) * (1.f / 12.f);
    case 1: return (-1.f + s) * (1.f / 12.f);
    default: return 0.f;
  }
}

// order class of a horizontal face index f in [lo, hi) (lo = ids or jds,
// hi = ide or jde): 5, 3, 2, or 0 (no flux), as in fqx_s / fqy_s
__device__ __forceinline__ int horder(int f, int lo, int hi) {
  if (f >= lo + 3 && f < hi - 3) return 5;
  if (f == lo + 2 || f == hi - 3) return 3;
  if (f == lo + 1 || f == hi - 2) return 2;
  return 0;
}

// vertical face kf (as in vf_s): 5, 3, 1 (the fnm / fnp average), or 0
__device__ __forceinline__ int vorder(int kf, int ktf) {
  if (kf >= 3 && kf < ktf - 2) return 5;
  if (kf == 2 || kf == ktf - 2) return 3;
  if (kf == 1 || kf == ktf - 1) return 1;
  return 0;
}

struct AdvArgs0 {
  const float *q, *ru, *rv, *rom, *msftx, *fnm, *fnp, *rdnw;
};

// The face cotangent Fbar of advect_scalar's faces and the cell coefficients
// it is formed from: every mass cell of the update set subtracts coef
// (F(upper face) - F(lower face)) in each direction
struct ScalarFaces {
  const Grid& g;
  const AdvArgs0& a;
  const float* tbar;
  size_t lev;
  __device__ bool inset(int kk, int jj, int ii) const {
    return kk >= 0 && kk < g.nz - 1 && ii >= g.ids && ii < g.ide - 1 && jj >= g.jds && jj < g.jde - 1;
  }
  __device__ float tb(int kk, int jj, int ii) const { return tbar[(size_t)kk * lev + (size_t)jj * g.nx + ii]; }
  __device__ float ay(int kk, int jj, int ii) const {
    return (inset(kk, jj, ii) && jj >= g.jds + 1 && jj < g.jde - 2) ? a.msftx[(size_t)jj * g.nx + ii] * g.rdy : 0.f;
  }
  __device__ float ax(int kk, int jj, int ii) const {
    return (inset(kk, jj, ii) && ii >= g.ids + 1 && ii < g.ide - 2) ? a.msftx[(size_t)jj * g.nx + ii] * g.rdx : 0.f;
  }
  __device__ float az(int kk, int jj, int ii) const { return inset(kk, jj, ii) ? a.rdnw[kk] : 0.f; }
  __device__ float fby(int kk, int jf, int ii) const {
    float v = 0.f;
    if (jf < g.ny) { const float cf = ay(kk, jf, ii); if (cf != 0.f) v += cf * tb(kk, jf, ii); }
    if (jf >= 1) { const float cf = ay(kk, jf - 1, ii); if (cf != 0.f) v -= cf * tb(kk, jf - 1, ii); }
    return v;
  }
  __device__ float fbx(int kk, int jj, int f) const {
    float v = 0.f;
    if (f < g.nx) { const float cf = ax(kk, jj, f); if (cf != 0.f) v += cf * tb(kk, jj, f); }
    if (f >= 1) { const float cf = ax(kk, jj, f - 1); if (cf != 0.f) v -= cf * tb(kk, jj, f - 1); }
    return v;
  }
  __device__ float fbz(int kf, int jj, int ii) const {
    float v = 0.f;
    if (kf < g.nz) { const float cf = az(kf, jj, ii); if (cf != 0.f) v += cf * tb(kf, jj, ii); }
    if (kf >= 1) { const float cf = az(kf - 1, jj, ii); if (cf != 0.f) v -= cf * tb(kf - 1, jj, ii); }
    return v;
  }
};

// one face's contributions Fbar r dPhi/dq(f + o) to the slots o + 3 of
// direction D (ord 5: o in [-3, 2], 3: [-2, 1], 2: the two-point average,
// 1: the fnm / fnp average of the vertical faces next to the ends)
__device__ __forceinline__ void scalar_slots(float* Q, size_t n3, int D, size_t p, int ord, float fbr, float s,
                                             float c0, float cm1) {
#pragma unroll
  for (int o = -3; o <= 2; ++o) {
    float w = 0.f;
    if (ord == 5) w = w5(o, s);
    else if (ord == 3) w = w3(o, s);
    else if (ord == 2) w = (o == 0 || o == -1) ? 0.5f : 0.f;
    else if (ord == 1) w = o == 0 ? c0 : (o == -1 ? cm1 : 0.f);
    Q[(size_t)(D * 6 + o + 3) * n3 + p] = fbr * w;
  }
}

}  // namespace

// Pass 1 of advect_scalar's reverse: one thread per point p, taken as the y
// face jf = j, the x face f = i and the vertical face kf = k.  Each face's
// cotangent Fbar (from the cells either side), velocity r and upwind sign
// give its contributions to the field at its stencil offsets (slots, as in
// the momentum reverse) and its own velocity cotangent rbar = Fbar Phi,
// which only this thread writes.
__global__ void k_advect_scalar_faces(Grid g, AdvArgs0 a, const float* tbar, float* Q, float* rubar, float* rvbar,
                                      float* rombar) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, n3 = g.n3();
  const size_t p = (size_t)k * lev + (size_t)j * nx + i;
  const ScalarFaces F{g, a, tbar, lev};
  const float* q = a.q;
  auto Qv = [&](size_t base, int off, int st) { return q[base + (size_t)((long long)off * st)]; };
  {  // y face jf = j at (k, i)
    const int ord = horder(j, jds, jde);
    const float fb = ord ? F.fby(k, j, i) : 0.f;
    const float r = a.rv[p];
    scalar_slots(Q, n3, 0, p, fb != 0.f ? ord : 0, fb * r, sgnf(r), 0.f, 0.f);
    if (fb != 0.f) {
      float phi;
      if (ord == 5) phi = flux5(Qv(p, -3, nx), Qv(p, -2, nx), Qv(p, -1, nx), Qv(p, 0, nx), Qv(p, 1, nx), Qv(p, 2, nx), r);
      else if (ord == 3) phi = flux3(Qv(p, -2, nx), Qv(p, -1, nx), Qv(p, 0, nx), Qv(p, 1, nx), r);
      else phi = 0.5f * (Qv(p, 0, nx) + Qv(p, -1, nx));
      rvbar[p] += fb * phi;
    }
  }
  {  // x face f = i at (k, j)
    const int ord = horder(i, ids, ide);
    const float fb = ord ? F.fbx(k, j, i) : 0.f;
    const size_t row = (size_t)k * lev + (size_t)j * nx;
    const float r = a.ru[p];
    const float rs = (i == ide - 3 && ord) ? a.ru[row + ide - 2] : r;  // the reference's sign source of that face
    scalar_slots(Q, n3, 1, p, fb != 0.f ? ord : 0, fb * r, sgnf(rs), 0.f, 0.f);
    if (fb != 0.f) {
      float phi;
      if (ord == 5) phi = flux5(Qv(p, -3, 1), Qv(p, -2, 1), Qv(p, -1, 1), Qv(p, 0, 1), Qv(p, 1, 1), Qv(p, 2, 1), rs);
      else if (ord == 3) phi = flux3(Qv(p, -2, 1), Qv(p, -1, 1), Qv(p, 0, 1), Qv(p, 1, 1), rs);
      else phi = 0.5f * (Qv(p, 0, 1) + Qv(p, -1, 1));
      rubar[p] += fb * phi;
    }
  }
  {  // vertical face kf = k at (j, i)
    const int ord = vorder(k, ktf);
    const float fb = ord ? F.fbz(k, j, i) : 0.f;
    const float r = a.rom[p];
    scalar_slots(Q, n3, 2, p, fb != 0.f ? ord : 0, fb * r, sgnf(-r), ord == 1 ? a.fnm[k] : 0.f,
                 ord == 1 ? a.fnp[k] : 0.f);
    if (fb != 0.f) {
      const int st = (int)lev;
      float phi;
      if (ord == 5) phi = flux5(Qv(p, -3, st), Qv(p, -2, st), Qv(p, -1, st), Qv(p, 0, st), Qv(p, 1, st), Qv(p, 2, st), -r);
      else if (ord == 3) phi = flux3(Qv(p, -2, st), Qv(p, -1, st), Qv(p, 0, st), Qv(p, 1, st), -r);
      else phi = a.fnm[k] * Qv(p, 0, st) + a.fnp[k] * Qv(p, -1, st);
      rombar[p] += fb * phi;
    }
  }
}

// Pass 2: the field cotangent of each point, summed in a fixed order over
// the slots of the faces whose stencils hold it (faces on the point's own
// line in each direction)
__global__ void k_advect_scalar_gather(Grid g, const float* Q, float* qbar) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const size_t m = (size_t)k * lev + (size_t)j * g.nx + i;
  float aq = 0.f;
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const int o = s - 3;
    if (j - o >= 0 && j - o < g.ny) aq += Q[(size_t)(0 * 6 + s) * n3 + (m - (long long)o * g.nx)];
    if (i - o >= 0 && i - o < g.nx) aq += Q[(size_t)(1 * 6 + s) * n3 + (m - o)];
    if (k - o >= 0 && k - o < g.nz) aq += Q[(size_t)(2 * 6 + s) * n3 + (m - (long long)o * lev)];
  }
  if (aq != 0.f) qbar[m] += aq;
}

// ------------------------------------------------------------ advance_uv

namespace {

// the points advance_uv updates (spec_zone 1) and the specified rows that
// spec_bdyupdate updates, as in k_advance_uv
__device__ __forceinline__ bool uv_in(const Grid& g, int V, int j, int i) {
  return V == 0 ? (j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 1)
                : (j >= g.jds + 1 && j < g.jde - 1 && i >= g.ids + 1 && i < g.ide - 2);
}
__device__ __forceinline__ bool uv_spec(const Grid& g, int V, int j, int i) {
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  return V == 0 ? (((j == jds || j == jde - 2) && i >= ids && i < ide) ||
                   (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 1)))
                : (((j == jds || j == jde - 1) && i >= ids && i < ide - 1) ||
                   (j >= jds + 1 && j < jde - 1 && (i == ids || i == ide - 2)));
}

__device__ __forceinline__ float uv_dpn(const Grid& g, const S& s, int kk, size_t ca, size_t cb) {
  const size_t lev = (size_t)g.ny * g.nx;
  const float* pp = s[WF_P];
  if (kk == 0)
    return 0.5f * (g.cf1 * (pp[ca] + pp[cb]) + g.cf2 * (pp[lev + ca] + pp[lev + cb]) + g.cf3 * (pp[2 * lev + ca] + pp[2 * lev + cb]));
  if (kk == g.nz - 1) return 0.f;
  return 0.5f * (s[WF_FNM][kk] * (pp[kk * lev + ca] + pp[kk * lev + cb]) +
                 s[WF_FNP][kk] * (pp[(kk - 1) * lev + ca] + pp[(kk - 1) * lev + cb]));
}

// d dpn(kk) / d p(k) at either column of the pair
__device__ __forceinline__ float uv_dpn_coef(const Grid& g, const S& s, int kk, int k) {
  if (kk == 0) return k == 0 ? 0.5f * g.cf1 : k == 1 ? 0.5f * g.cf2 : k == 2 ? 0.5f * g.cf3 : 0.f;
  if (kk < 0 || kk >= g.nz - 1) return 0.f;
  if (k == kk) return 0.5f * s[WF_FNM][kk];
  if (k == kk - 1) return 0.5f * s[WF_FNP][kk];
  return 0.f;
}

// the factors of dp at an updated point of u (V = 0) or v (V = 1), the
// cotangent ub of its new value and dpb = d L / d dp
struct UvTerm {
  float ub, dpb, A, B, Cf, C, D;
};

template <bool kB = true, bool kD = true>
__device__ UvTerm uv_term(const Grid& g, const S& s, const S& b, float dts, int V, int k, int j, int i) {
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t c = (size_t)j * g.nx + i, p = k * lev + c, no = V ? (size_t)g.nx : 1;
  const float* ph = s[WF_PH];
  const float* pp = s[WF_P];
  const float* alt = s[WF_ALT];
  const float* al = s[WF_AL];
  const float* pb = s[WF_PB];
  const float* php = s[WF_PHP];
  const float* mu = s[WF_MU];
  const float r = V ? s[WF_MSFVY][c] / s[WF_MSFVX][c] : s[WF_MSFUX][c] / s[WF_MSFUY][c];
  const float rd = V ? g.rdy : g.rdx;
  UvTerm t;
  t.ub = b[V ? WF_V : WF_U][p];
  t.dpb = -dts * s[V ? WF_CQV : WF_CQU][p] * t.ub;
  t.A = r * 0.5f * rd * s[V ? WF_MUV : WF_MUU][c];
  t.B = 0.f;
  if (kB)
    t.B = ((ph[p + lev] - ph[p + lev - no]) + (ph[p] - ph[p - no])) + (alt[p] + alt[p - no]) * (pp[p] - pp[p - no]) +
          (al[p] + al[p - no]) * (pb[p] - pb[p - no]);
  t.Cf = r * rd;
  t.C = t.Cf * (php[p] - php[p - no]);
  t.D = 0.f;
  if (kD)
    t.D = s[WF_RDNW][k] * (uv_dpn(g, s, k + 1, c, c - no) - uv_dpn(g, s, k, c, c - no)) - 0.5f * (mu[c - no] + mu[c]);
  return t;
}

}  // namespace

__global__ void k_advance_uv_adj(Grid g, S s, S b, float dts) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ktf = g.nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const size_t m = (size_t)k * lev + (size_t)j * nx + i;
  if (k < ktf) {
    if (uv_in(g, 0, j, i) || uv_spec(g, 0, j, i)) b[WF_RU_TEND][m] += dts * b[WF_U][m];
    if (uv_in(g, 1, j, i) || uv_spec(g, 1, j, i)) b[WF_RV_TEND][m] += dts * b[WF_V][m];
  }
  float aph = 0.f, aalt = 0.f, aal = 0.f, apb = 0.f, aphp = 0.f, ap = 0.f;
  for (int V = 0; V < 2; ++V) {
    const size_t no = V ? (size_t)nx : 1;
    // the points P = (kP, j + V e, i + (1 - V) e), e = 0 (m is P's own
    // column, sign +) or 1 (m is P's west / south neighbour, sign -)
    for (int e = 0; e < 2; ++e) {
      const int jP = j + V * e, iP = i + (1 - V) * e;
      if (jP >= g.ny || iP >= nx || !uv_in(g, V, jP, iP)) continue;
      const float sg = e == 0 ? 1.f : -1.f;
      for (int kP = k - 2; kP <= k + 1; ++kP) {
        if (kP < 0 || kP >= ktf) continue;
        // B enters the gathered cotangents only through A (and the own
        // point's cqu / cqv, below), D only at kP == k
        const UvTerm t = kP == k ? uv_term<false, true>(g, s, b, dts, V, kP, jP, iP)
                                 : uv_term<false, false>(g, s, b, dts, V, kP, jP, iP);
        if (t.dpb == 0.f) continue;
        const float Bb = t.dpb * t.A, Db = t.dpb * t.C;
        const size_t P = (size_t)kP * lev + (size_t)jP * nx + iP;
        if (kP == k || kP == k - 1) aph += sg * Bb;  // ph at kP and kP + 1
        if (kP == k) {
          aalt += Bb * (s[WF_P][P] - s[WF_P][P - no]);
          aal += Bb * (s[WF_PB][P] - s[WF_PB][P - no]);
          apb += sg * Bb * (s[WF_AL][P] + s[WF_AL][P - no]);
          ap += sg * Bb * (s[WF_ALT][P] + s[WF_ALT][P - no]);
          aphp += sg * t.dpb * t.Cf * t.D;
        }
        // p through dpn(kP + 1) - dpn(kP) (both columns of the pair, sign +)
        const float rw = s[WF_RDNW][kP] * Db;
        ap += rw * (uv_dpn_coef(g, s, kP + 1, k) - uv_dpn_coef(g, s, kP, k));
      }
    }
  }
  if (k < ktf) {
    if (uv_in(g, 0, j, i)) {
      const UvTerm t = uv_term(g, s, b, dts, 0, k, j, i);
      b[WF_CQU][m] += -dts * (t.A * t.B + t.C * t.D) * t.ub;
    }
    if (uv_in(g, 1, j, i)) {
      const UvTerm t = uv_term(g, s, b, dts, 1, k, j, i);
      b[WF_CQV][m] += -dts * (t.A * t.B + t.C * t.D) * t.ub;
    }
  }
  if (aph != 0.f) b[WF_PH][m] += aph;
  if (aalt != 0.f) b[WF_ALT][m] += aalt;
  if (aal != 0.f) b[WF_AL][m] += aal;
  if (apb != 0.f) b[WF_PB][m] += apb;
  if (aphp != 0.f) b[WF_PHP][m] += aphp;
  if (ap != 0.f) b[WF_P][m] += ap;
}

// the column sums by kColLevels level groups (threadIdx.y, levels ty,
// ty + kColLevels, ...) of 32 columns of a row, added up in a fixed order
constexpr int kColLevels = 8;

__global__ void __launch_bounds__(32 * kColLevels) k_advance_uv_adj_col(Grid g, S s, S b, float dts) {
  __shared__ float red[4][kColLevels][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const int ktf = g.nz - 1, nx = g.nx;
  const bool on = i < nx;
  const size_t c = (size_t)j * nx + (on ? i : 0);
  const float eu = (float)(-(double)g.emdiv * g.dxd), ev = (float)(-(double)g.emdiv * g.dyd);
  float amuu = 0.f, amuv = 0.f, amu = 0.f, amudf = 0.f;
  for (int V = 0; V < 2; ++V)
    for (int e = 0; e < 2; ++e) {
      const int jP = j + V * e, iP = i + (1 - V) * e;
      if (!on || jP >= g.ny || iP >= nx || !uv_in(g, V, jP, iP)) continue;
      const size_t cP = (size_t)jP * nx + iP;
      const float sg = e == 0 ? 1.f : -1.f;
      const float em = V ? ev * s[WF_MSFVX_INV][cP] : eu / s[WF_MSFUY][cP];
#pragma unroll 2
      for (int k = ty; k < ktf; k += kColLevels) {
        const UvTerm t = e == 0 ? uv_term<true, false>(g, s, b, dts, V, k, jP, iP)
                                : uv_term<false, false>(g, s, b, dts, V, k, jP, iP);
        if (e == 0) {
          const float r = V ? s[WF_MSFVY][cP] / s[WF_MSFVX][cP] : s[WF_MSFUX][cP] / s[WF_MSFUY][cP];
          const float d = t.dpb * (r * 0.5f * (V ? g.rdy : g.rdx)) * t.B;
          if (V) amuv += d;
          else amuu += d;
        }
        amu += -0.5f * t.dpb * t.C;
        amudf += sg * t.ub * em;
      }
    }
  red[0][ty][tx] = amuu;
  red[1][ty][tx] = amuv;
  red[2][ty][tx] = amu;
  red[3][ty][tx] = amudf;
  __syncthreads();
  if (ty != 0 || !on) return;
  amuu = amuv = amu = amudf = 0.f;
#pragma unroll
  for (int y = 0; y < kColLevels; ++y) {
    amuu += red[0][y][tx];
    amuv += red[1][y][tx];
    amu += red[2][y][tx];
    amudf += red[3][y][tx];
  }
  if (amuu != 0.f) b[WF_MUU][c] += amuu;
  if (amuv != 0.f) b[WF_MUV][c] += amuv;
  if (amu != 0.f) b[WF_MU][c] += amu;
  if (amudf != 0.f) b[WF_MUDF][c] += amudf;
}

int launch_advance_uv_adj(const Grid& g, const S& s, const S& b, float dts, cudaStream_t st) {
  const dim3 b3(32, 4), b2(32, 8);
  k_advance_uv_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, dts);
  k_advance_uv_adj_col<<<dim3((g.nx + 31) / 32, g.ny), dim3(32, kColLevels), 0, st>>>(g, s, b, dts);
  return 2;
}

// ------------------------------------------------------------ calc_p_rho
// state-table operands: al AL, p P, ph PH, alt ALT, t_2 T, t_1 T_SAVE,
// c2a C2A, pm1 PM1, mu MU, mut MUTS, rdnw RDNW (the acoustic substep's
// arguments, solver.py calc_p_rho calls)

namespace {

__device__ __forceinline__ bool prho_in(const Grid& g, int k, int j, int i) {
  return k < g.nz - 1 && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1;
}

// forward values at a mass point and the cotangents that reach p1 and al
struct PrhoTerm {
  float al, N, Dn, X, p1, p1b, Ab;
};

__device__ PrhoTerm prho_term(const Grid& g, const S& s, const S& b, int step, int k, int j, int i) {
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t c = (size_t)j * g.nx + i, p = k * lev + c;
  const float mut = s[WF_MUTS][c], mu = s[WF_MU][c];
  const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p], t2 = s[WF_T][p], c2 = s[WF_C2A][p];
  PrhoTerm t;
  t.al = -1.0f / mut * (alt * mu + s[WF_RDNW][k] * (s[WF_PH][p + lev] - s[WF_PH][p]));
  t.N = t2 - mu * t1;
  t.Dn = mut * ((float)T0 + t1);
  t.X = alt * t.N / t.Dn;
  t.p1 = c2 * (t.X - t.al);
  const float Pb = b[WF_P][p], Mb = b[WF_PM1][p];
  t.p1b = step == 0 ? Pb + Mb : (1.0f + g.smdiv) * Pb + Mb;
  t.Ab = b[WF_AL][p] - c2 * t.p1b;
  return t;
}

}  // namespace

__global__ void k_calc_p_rho(Grid g, S s, int step) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  float* pp = s[WF_P];
  if (prho_in(g, k, j, i)) {
    const float muts = s[WF_MUTS][c], mu = s[WF_MU][c];
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float al = -1.0f / muts * (alt * mu + s[WF_RDNW][k] * (s[WF_PH][p + lev] - s[WF_PH][p]));
    const float p1 = s[WF_C2A][p] * (alt * (s[WF_T][p] - mu * t1) / (muts * ((float)T0 + t1)) - al);
    s[WF_AL][p] = al;
    if (step == 0) {
      pp[p] = p1;
      s[WF_PM1][p] = p1;
    } else {
      pp[p] = p1 + g.smdiv * (p1 - s[WF_PM1][p]);
      s[WF_PM1][p] = p1;
    }
  } else if (step == 0) {
    s[WF_PM1][p] = pp[p];  // pm1 is a copy of the whole p
  }
}

__global__ void k_calc_p_rho_adj(Grid g, S s, S b, int step) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const float mut = s[WF_MUTS][c], mu = s[WF_MU][c];
  if (prho_in(g, k, j, i)) {
    const PrhoTerm t = prho_term(g, s, b, step, k, j, i);
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float Xb = s[WF_C2A][p] * t.p1b;
    b[WF_C2A][p] += t.p1b * (t.X - t.al);
    b[WF_ALT][p] += Xb * t.N / t.Dn + t.Ab * (-mu / mut);
    b[WF_T][p] += Xb * alt / t.Dn;
    b[WF_T_SAVE][p] += Xb * alt * (-mu) / t.Dn - Xb * t.X / ((float)T0 + t1);
  }
  // ph(k): +rdnw(k) / mut from cell k, -rdnw(k-1) / mut from cell k-1
  float aph = 0.f;
  if (prho_in(g, k, j, i)) aph += prho_term(g, s, b, step, k, j, i).Ab * (s[WF_RDNW][k] / mut);
  if (k >= 1 && prho_in(g, k - 1, j, i)) aph -= prho_term(g, s, b, step, k - 1, j, i).Ab * (s[WF_RDNW][k - 1] / mut);
  if (aph != 0.f) b[WF_PH][p] += aph;
}

__global__ void __launch_bounds__(32 * kColLevels) k_calc_p_rho_adj_col(Grid g, S s, S b, int step) {
  __shared__ float red[2][kColLevels][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const bool on = i < g.nx && prho_in(g, 0, j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const int c = g.i2(j, on ? i : 0);
  const float mut = on ? s[WF_MUTS][c] : 1.f;
  float amu = 0.f, amut = 0.f;
#pragma unroll 2
  for (int k = ty; on && k < g.nz - 1; k += kColLevels) {
    const size_t p = k * lev + c;
    const PrhoTerm t = prho_term(g, s, b, step, k, j, i);
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float Xb = s[WF_C2A][p] * t.p1b;
    amu += Xb * alt * (-t1) / t.Dn + t.Ab * (-alt / mut);
    amut += -Xb * t.X / mut + t.Ab * (-t.al / mut);
  }
  red[0][ty][tx] = amu;
  red[1][ty][tx] = amut;
  __syncthreads();
  if (ty != 0 || !on) return;
  amu = amut = 0.f;
#pragma unroll
  for (int y = 0; y < kColLevels; ++y) {
    amu += red[0][y][tx];
    amut += red[1][y][tx];
  }
  b[WF_MU][c] += amu;
  b[WF_MUTS][c] += amut;
}

__global__ void k_calc_p_rho_adj_out(Grid g, S b, int step) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t p = (size_t)k * g.ny * g.nx + g.i2(j, i);
  if (prho_in(g, k, j, i)) {
    const float Pb = b[WF_P][p];
    b[WF_AL][p] = 0.f;
    b[WF_P][p] = 0.f;
    b[WF_PM1][p] = step == 0 ? 0.f : -g.smdiv * Pb;
  } else if (step == 0) {
    b[WF_P][p] = b[WF_P][p] + b[WF_PM1][p];
    b[WF_PM1][p] = 0.f;
  }
}

int launch_calc_p_rho(const Grid& g, const S& s, int step, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_calc_p_rho<<<point_grid(g, b3), b3, 0, st>>>(g, s, step);
  return 1;
}

int launch_calc_p_rho_adj(const Grid& g, const S& s, const S& b, int step, cudaStream_t st) {
  const dim3 b3(32, 4), b2(32, 8);
  k_calc_p_rho_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, step);
  k_calc_p_rho_adj_col<<<dim3((g.nx + 31) / 32, g.ny), dim3(32, kColLevels), 0, st>>>(g, s, b, step);
  k_calc_p_rho_adj_out<<<point_grid(g, b3), b3, 0, st>>>(g, b, step);
  return 3;
}

// ------------------------------------------------------------ advance_mu_t
// state-table operands: ww WW, ww_1 WW1, u U, u_1 U_SAVE, v V, v_1 V_SAVE,
// mu MU, mut MUT, muave MUAVE, muts MUTS, muu MUU, muv MUV, mudf MUDF, t T,
// t_1 T_SAVE, t_ave T_2SAVE, ft T_TEND, mu_tend MU_TEND (solver.py:1380-1393)

namespace {

__device__ __forceinline__ bool mut_in(const Grid& g, int j, int i) {
  return j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
}

__device__ __forceinline__ float mut_dvdxi(const Grid& g, const S& s, int k, int j, int i) {
  const int nx = g.nx;
  const size_t c = (size_t)j * nx + i, p = (size_t)k * g.ny * nx + c;
  const float vn = s[WF_V][p + nx] + s[WF_MUV][c + nx] * s[WF_V_SAVE][p + nx] * s[WF_MSFVX_INV][c + nx];
  const float vs = s[WF_V][p] + s[WF_MUV][c] * s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c];
  const float ue = s[WF_U][p + 1] + s[WF_MUU][c + 1] * s[WF_U_SAVE][p + 1] / s[WF_MSFUY][c + 1];
  const float uw = s[WF_U][p] + s[WF_MUU][c] * s[WF_U_SAVE][p] / s[WF_MSFUY][c];
  return s[WF_MSFTX][c] * s[WF_MSFTY][c] * (g.rdy * (vn - vs) + g.rdx * (ue - uw));
}

// a column's forward values: dvdxi, dmdt and the new ww (ww' = W - ww_1)
struct MutCol {
  float dv[kMaxNz], wwp[kMaxNz];
  float dmdt;
};

constexpr int kMutChunk = 8;  // levels whose loads a column kernel issues together

__device__ void mut_column(const Grid& g, const S& s, int j, int i, MutCol& m) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, c = (size_t)j * g.nx + i;
  const float* dnw = s[WF_DNW];
  m.dmdt = 0.f;
#pragma unroll 8
  for (int k = 0; k < ktf; ++k) {
    m.dv[k] = mut_dvdxi(g, s, k, j, i);
    m.dmdt = m.dmdt + dnw[k] * m.dv[k];
  }
  const float mt = s[WF_MU_TEND][c], msfty = s[WF_MSFTY][c];
  float W = s[WF_WW][c];
  m.wwp[0] = W - s[WF_WW1][c];
#pragma unroll 8
  for (int k = 1; k < ktf; ++k) {
    W = W - dnw[k - 1] * (m.dmdt + m.dv[k - 1] + mt) / msfty;
    m.wwp[k] = W - s[WF_WW1][k * lev + c];
  }
}

// the cotangents of wdtn(kk), kk in [1, ktf), and of ww'(k), k in [0, ktf)
__device__ void mut_ww_bar(const Grid& g, const S& s, const S& b, float dts, int j, int i, const MutCol& m,
                           float* wdb, float* wwb) {
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, c = (size_t)j * g.nx + i;
  const float dm = dts * s[WF_MSFTY][c];
  const float* rdnw = s[WF_RDNW];
  const float* t1 = s[WF_T_SAVE];
#pragma unroll 8
  for (int k = 0; k < ktf; ++k) {
    wdb[k] = 0.f;
    if (k >= 1) wdb[k] = -dm * rdnw[k - 1] * b[WF_T][(k - 1) * lev + c] + dm * rdnw[k] * b[WF_T][k * lev + c];
    const float tavg = k >= 1 ? s[WF_FNM][k] * t1[k * lev + c] + s[WF_FNP][k] * t1[(k - 1) * lev + c] : 0.f;
    wwb[k] = b[WF_WW][k * lev + c] + (k >= 1 ? wdb[k] * tavg : 0.f);
  }
}

// mu' is the new mu; the cotangent reaching it from mu', muts', muave'
__device__ __forceinline__ float mut_mu_bar(const Grid& g, const S& b, size_t c) {
  const float ep1 = (float)(1.0 + (double)g.epssm);
  return b[WF_MU][c] + b[WF_MUTS][c] + 0.5f * ep1 * b[WF_MUAVE][c];
}

}  // namespace

__global__ void k_advance_mu_t(Grid g, S s, float dts) {
  WRF_COLUMN_INDEX(g, j, i);
  if (!mut_in(g, j, i)) return;
  const int ktf = g.nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, c = (size_t)j * nx + i;
  MutCol m;
  mut_column(g, s, j, i, m);
  const float ep1 = (float)(1.0 + (double)g.epssm), em1 = (float)(1.0 - (double)g.epssm);
  const float mu0 = s[WF_MU][c], mt = s[WF_MU_TEND][c];
  const float mu1 = mu0 + dts * (m.dmdt + mt);
  s[WF_MU][c] = mu1;
  s[WF_MUDF][c] = m.dmdt + mt;
  s[WF_MUTS][c] = s[WF_MUT][c] + mu1;
  s[WF_MUAVE][c] = 0.5f * (ep1 * mu1 + em1 * mu0);
  for (int k = 0; k < ktf; ++k) s[WF_WW][k * lev + c] = m.wwp[k];
  const float msfty = s[WF_MSFTY][c], msftx = s[WF_MSFTX][c], rdx = g.rdx, rdy = g.rdy;
  const float* t1 = s[WF_T_SAVE];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  auto wdtn = [&](int k) {
    if (k < 1 || k >= ktf) return 0.f;
    return m.wwp[k] * (s[WF_FNM][k] * t1[k * lev + c] + s[WF_FNP][k] * t1[(k - 1) * lev + c]);
  };
  // kMutChunk levels at a time, every load of the block before its stores
  for (int k0 = 0; k0 < ktf; k0 += kMutChunk) {
    float tk[kMutChunk], tt[kMutChunk], h[kMutChunk], rd[kMutChunk], wd[kMutChunk + 1];
#pragma unroll
    for (int q = 0; q <= kMutChunk; ++q) wd[q] = wdtn(k0 + q);
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      const size_t p = (size_t)(k < ktf ? k : 0) * lev + c;
      tk[q] = s[WF_T][p];
      tt[q] = s[WF_T_TEND][p];
      h[q] = 0.5f * rdy * (v[p + nx] * (t1[p + nx] + t1[p]) - v[p] * (t1[p] + t1[p - nx])) +
             0.5f * rdx * (u[p + 1] * (t1[p + 1] + t1[p]) - u[p] * (t1[p] + t1[p - 1]));
      rd[q] = s[WF_RDNW][k < ktf ? k : 0];
    }
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      if (k >= ktf) break;
      const size_t p = k * lev + c;
      s[WF_T_2SAVE][p] = tk[q];
      const float t1v = tk[q] + msfty * dts * tt[q];
      s[WF_T][p] = t1v - dts * msfty * (msftx * h[q] + rd[q] * (wd[q + 1] - wd[q]));
    }
  }
}

__global__ void k_advance_mu_t_adj_dv(Grid g, S s, S b, float dts, int ref_no_grad, float* work) {
  WRF_COLUMN_INDEX(g, j, i);
  if (!mut_in(g, j, i)) return;
  const int ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, c = (size_t)j * g.nx + i;
  MutCol m;
  mut_column(g, s, j, i, m);
  float wdb[kMaxNz], wwb[kMaxNz], qb[kMaxNz];
  mut_ww_bar(g, s, b, dts, j, i, m, wdb, wwb);
  const float msfty = s[WF_MSFTY][c];
  float S_ = 0.f, qsum = 0.f;
#pragma unroll 8
  for (int k = ktf - 1; k >= 1; --k) {
    S_ += wwb[k];
    qb[k - 1] = -s[WF_DNW][k - 1] / msfty * S_;
    qsum += qb[k - 1];
  }
  const float dmdtb = qsum + (ref_no_grad ? 0.f : dts * mut_mu_bar(g, b, c) + b[WF_MUDF][c]);
  for (int k0 = 0; k0 < ktf; k0 += kMutChunk) {  // dnw loaded before the block's stores
    float dn[kMutChunk];
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) dn[q] = s[WF_DNW][k0 + q < ktf ? k0 + q : 0];
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      if (k >= ktf) break;
      work[k * lev + c] = (k <= ktf - 2 ? qb[k] : 0.f) + dn[q] * dmdtb;
    }
  }
}

__global__ void k_advance_mu_t_adj_pt(Grid g, S s, S b, float dts, const float* work) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ktf = g.nz - 1, nx = g.nx;
  if (k >= ktf) return;
  const size_t lev = (size_t)g.ny * nx, c = (size_t)j * nx + i, p = k * lev + c;
  const float rdx = g.rdx, rdy = g.rdy;
  auto mm = [&](size_t cc) { return s[WF_MSFTX][cc] * s[WF_MSFTY][cc]; };
  // divergence: u, u_1 at columns i (east face of column i-1, sign +) and
  // (west face of column i, sign -); v, v_1 likewise in y
  float ub = 0.f, vb = 0.f;
  if (i >= 1 && mut_in(g, j, i - 1)) ub += mm(c - 1) * rdx * work[p - 1];
  if (mut_in(g, j, i)) ub -= mm(c) * rdx * work[p];
  if (j >= 1 && mut_in(g, j - 1, i)) vb += mm(c - nx) * rdy * work[p - nx];
  if (mut_in(g, j, i)) vb -= mm(c) * rdy * work[p];
  float u1b = ub * s[WF_MUU][c] / s[WF_MSFUY][c];
  float v1b = vb * s[WF_MUV][c] * s[WF_MSFVX_INV][c];
  // theta fluxes: Hb(P) = -dts msfty msftx tbar at the updated columns P
  auto hb = [&](int jj, int ii) {
    if (jj < 0 || ii < 0 || jj >= g.ny || ii >= nx || !mut_in(g, jj, ii)) return 0.f;
    const size_t cc = (size_t)jj * nx + ii;
    return -dts * s[WF_MSFTY][cc] * s[WF_MSFTX][cc] * b[WF_T][k * lev + cc];
  };
  const float hc = hb(j, i), hs = hb(j - 1, i), hn = hb(j + 1, i), hw = hb(j, i - 1), he = hb(j, i + 1);
  const float* t1 = s[WF_T_SAVE];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  if (hs != 0.f || hc != 0.f) vb += 0.5f * rdy * (t1[p] + t1[p - nx]) * (hs - hc);
  if (hw != 0.f || hc != 0.f) ub += 0.5f * rdx * (t1[p] + t1[p - 1]) * (hw - hc);
  float t1b = 0.f;
  if (hs != 0.f) t1b += 0.5f * rdy * hs * v[p];
  if (hc != 0.f) t1b += 0.5f * rdy * hc * (v[p + nx] - v[p]) + 0.5f * rdx * hc * (u[p + 1] - u[p]);
  if (hn != 0.f) t1b -= 0.5f * rdy * hn * v[p + nx];
  if (hw != 0.f) t1b += 0.5f * rdx * hw * u[p];
  if (he != 0.f) t1b -= 0.5f * rdx * he * u[p + 1];
  if (ub != 0.f) b[WF_U][p] += ub;
  if (vb != 0.f) b[WF_V][p] += vb;
  if (u1b != 0.f) b[WF_U_SAVE][p] += u1b;
  if (v1b != 0.f) b[WF_V_SAVE][p] += v1b;
  if (t1b != 0.f) b[WF_T_SAVE][p] += t1b;
}

__global__ void k_advance_mu_t_adj_col(Grid g, S s, S b, float dts, int ref_no_grad, const float* work) {
  WRF_COLUMN_INDEX(g, j, i);
  const int ktf = g.nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, c = (size_t)j * nx + i;
  const float rdx = g.rdx, rdy = g.rdy;
  // muu, muv: the u / v terms of the divergence at this column
  {
    float amuu = 0.f, amuv = 0.f;
    const bool w = i >= 1 && mut_in(g, j, i - 1), o = mut_in(g, j, i), sth = j >= 1 && mut_in(g, j - 1, i);
    if (w || o || sth) {
      const float mw = w ? s[WF_MSFTX][c - 1] * s[WF_MSFTY][c - 1] : 0.f;
      const float mo = o ? s[WF_MSFTX][c] * s[WF_MSFTY][c] : 0.f;
      const float ms = sth ? s[WF_MSFTX][c - nx] * s[WF_MSFTY][c - nx] : 0.f;
#pragma unroll 8
      for (int k = 0; k < ktf; ++k) {
        const size_t p = k * lev + c;
        float ub = 0.f, vb = 0.f;
        if (w) ub += mw * rdx * work[p - 1];
        if (o) ub -= mo * rdx * work[p];
        if (sth) vb += ms * rdy * work[p - nx];
        if (o) vb -= mo * rdy * work[p];
        amuu += ub * s[WF_U_SAVE][p] / s[WF_MSFUY][c];
        amuv += vb * s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c];
      }
      if (amuu != 0.f) b[WF_MUU][c] += amuu;
      if (amuv != 0.f) b[WF_MUV][c] += amuv;
    }
  }
  if (!mut_in(g, j, i)) return;
  MutCol m;
  mut_column(g, s, j, i, m);
  float wdb[kMaxNz], wwb[kMaxNz];
  mut_ww_bar(g, s, b, dts, j, i, m, wdb, wwb);
  const float msfty = s[WF_MSFTY][c];
  // ww, ww_1 (the scan passes every ww' cotangent down to ww(0))
  float wsum = 0.f, qsum = 0.f, S_ = 0.f;
#pragma unroll 8
  for (int k = ktf - 1; k >= 1; --k) {
    S_ += wwb[k];
    qsum += -s[WF_DNW][k - 1] / msfty * S_;
  }
  // (the arrays may alias as far as the compiler knows: each block of
  // kMutChunk levels loads everything it reads before its first store, so
  // the loads issue together)
  for (int k0 = 0; k0 < ktf; k0 += kMutChunk) {
    float w1[kMutChunk];
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) w1[q] = k0 + q < ktf ? b[WF_WW1][(k0 + q) * lev + c] : 0.f;
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      if (k >= ktf) break;
      wsum += wwb[k];
      b[WF_WW1][k * lev + c] = w1[q] - wwb[k];
      if (k >= 1) b[WF_WW][k * lev + c] = 0.f;
    }
  }
  b[WF_WW][c] = wsum;
  // theta: t_ave = t, ft, the vertical fluxes' t_1 (t_1(k) takes level k's
  // fnm term, then level k + 1's fnp term)
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  for (int k0 = 0; k0 < ktf; k0 += kMutChunk) {
    float tb[kMutChunk], tt[kMutChunk], t2s[kMutChunk], tsv[kMutChunk], fm[kMutChunk], fp[kMutChunk];
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      const size_t p = (size_t)(k < ktf ? k : 0) * lev + c;
      tb[q] = k < ktf ? b[WF_T][p] : 0.f;
      tt[q] = k < ktf ? b[WF_T_TEND][p] : 0.f;
      t2s[q] = k < ktf ? b[WF_T_2SAVE][p] : 0.f;
      tsv[q] = k < ktf ? b[WF_T_SAVE][p] : 0.f;
      fm[q] = k >= 1 && k < ktf ? fnm[k] : 0.f;
      fp[q] = k + 1 < ktf ? fnp[k + 1] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < kMutChunk; ++q) {
      const int k = k0 + q;
      if (k >= ktf) break;
      const size_t p = k * lev + c;
      b[WF_T_TEND][p] = tt[q] + msfty * dts * tb[q];
      b[WF_T][p] = tb[q] + t2s[q];
      b[WF_T_2SAVE][p] = 0.f;
      float x = tsv[q];
      if (k >= 1) x += wdb[k] * m.wwp[k] * fm[q];
      if (k + 1 < ktf) x += wdb[k + 1] * m.wwp[k + 1] * fp[q];
      b[WF_T_SAVE][p] = x;
    }
  }
  // the mu update
  if (ref_no_grad) {
    b[WF_MU_TEND][c] += qsum;
  } else {
    const float em1 = (float)(1.0 - (double)g.epssm);
    const float mub = mut_mu_bar(g, b, c);
    b[WF_MU_TEND][c] += qsum + dts * mub + b[WF_MUDF][c];
    b[WF_MUT][c] += b[WF_MUTS][c];
    b[WF_MU][c] = mub + 0.5f * em1 * b[WF_MUAVE][c];
    b[WF_MUTS][c] = 0.f;
    b[WF_MUDF][c] = 0.f;
    b[WF_MUAVE][c] = 0.f;
  }
}

int launch_advance_mu_t(const Grid& g, const S& s, float dts, cudaStream_t st) {
  const dim3 b2(32, 4);
  k_advance_mu_t<<<col_grid(g, b2), b2, 0, st>>>(g, s, dts);
  return 1;
}

int launch_advance_mu_t_adj(const Grid& g, const S& s, const S& b, float dts, int ref_no_grad, float* work,
                            cudaStream_t st) {
  const dim3 b2(32, 4), b3(32, 4);
  k_advance_mu_t_adj_dv<<<col_grid(g, b2), b2, 0, st>>>(g, s, b, dts, ref_no_grad, work);
  k_advance_mu_t_adj_pt<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, dts, work);
  k_advance_mu_t_adj_col<<<col_grid(g, b2), b2, 0, st>>>(g, s, b, dts, ref_no_grad, work);
  return 3;
}

// ------------------------------------------------------------ advance_w
// state-table operands (solver.py advance_w call): w W, rw_tend RW_TEND, ww WW,
// w_save W_SAVE, u U, v V, muave MUAVE, muts MUTS, mut MUT, t_2ave T_2SAVE,
// t_2 T, t_1 T_SAVE, ph PH, ph_1 PH_SAVE, phb PHB, ph_tend PH_TEND, ht HT,
// c2a C2A, cqw CQW, alt ALT, a A, alpha ALPHA, gamma GAMMA, with msftx, msfty,
// fnm, fnp, rdnw, rdn

namespace {

constexpr float kAwHdepth = 5000.0f;

// one column's forward values

__device__ float aw_bc(const Grid& g, const S& s, int j, int i) {
  const int nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, c = (size_t)j * nx + i;
  const float* ht = s[WF_HT];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  auto cv = [&](size_t cc) { return g.cf1 * v[cc] + g.cf2 * v[lev + cc] + g.cf3 * v[2 * lev + cc]; };
  auto cu = [&](size_t cc) { return g.cf1 * u[cc] + g.cf2 * u[lev + cc] + g.cf3 * u[2 * lev + cc]; };
  return s[WF_MSFTY][c] * 0.5f * g.rdy * ((ht[c + nx] - ht[c]) * cv(c + nx) + (ht[c] - ht[c - nx]) * cv(c)) +
         s[WF_MSFTX][c] * 0.5f * g.rdx * ((ht[c + 1] - ht[c]) * cu(c + 1) + (ht[c] - ht[c - 1]) * cu(c));
}


}  // namespace

// advance_w's reverse with a column's levels spread over the threads of a
// block: 32 adjacent columns of one row (threadIdx.x) x kAwGroups level
// groups (threadIdx.y; group y takes levels y, y + kAwGroups, ...).  The
// per-level parts of the forward recomputation and of the reverse run on
// all threads, each written in gather form (a level's thread forms every
// contribution that lands on its level, from its own level's terms and
// from the neighbouring levels' terms), so every cotangent element has one
// writer; the three vertical recurrences (the forward's two sweeps of the
// implicit solve, the transposed sweeps) run on the threads of group 0,
// one per column, through the column arrays in shared memory
// ([array][level][column]: a warp's lanes read neighbouring words).  The
// column sums (mut, muts, muave, and the damping top's height) are reduced
// across the groups at the end.
constexpr int kAwGroups = 8, kAwLevels = kMaxNz / kAwGroups;
constexpr int kAwArrays = 12;  // t2a, wd, R, rhs, P, x, y, z, zb (then xb), yb, Pb, rhsb

size_t advance_w_adj_smem(const Grid& g) { return ((size_t)kAwArrays * g.nz * 32 + 4 * kAwGroups * 32) * sizeof(float); }

// the forward recomputation of advance_w over a block's level groups, in
// the reference's order: t_2ave, wdwn, R, rhs, P and the explicit w x in
// the column arrays, then the solve's two sweeps (y, z) on group 0, the
// solve's coefficients staged first; ends with the block synchronised
struct AwLp {
  const Grid& g;
  const S& s;
  float* sm;
  int nz, ktf, tx, ty;
  bool on;
  size_t lev, c;
  int j, i;
  float dts, ep1, em1, gf, t0, muave, muts, mut, msfty, minv;
  enum { T2A, WD, RR, RHS, PP, XX, YY, ZZ, ZB, YB, PB, RHSB };
  enum { CA = RHS, CAL = RHSB, CG = PB };
  __device__ float& A(int arr, int k) const { return sm[((size_t)arr * nz + k) * 32 + tx]; }
  __device__ float F(int id, int k) const { return s[id][k * lev + c]; }
  __device__ void forward() const {
    const float* rdnw = s[WF_RDNW];
    const float* rdn = s[WF_RDN];
    if (on)
  #pragma unroll
      for (int l = 0; l < kAwLevels; ++l) {
        const int k = ty + kAwGroups * l;
        if (k < ktf) {
          const float tt = 0.5f * (ep1 * F(WF_T, k) + em1 * F(WF_T_2SAVE, k));
          A(T2A, k) = (tt + muave * t0) / (muts * (t0 + F(WF_T_SAVE, k)));
        }
        if (k == 0) A(WD, 0) = 0.f;
        if (k >= 1 && k <= ktf)
          A(WD, k) = 0.5f * (F(WF_WW, k) + F(WF_WW, k - 1)) * rdnw[k - 1] *
                     (F(WF_PH_SAVE, k) - F(WF_PH_SAVE, k - 1) + F(WF_PHB, k) - F(WF_PHB, k - 1));
      }
    __syncthreads();
    if (on)
  #pragma unroll
      for (int l = 0; l < kAwLevels; ++l) {
        const int k = ty + kAwGroups * l;
        if (k == 0) A(RHS, 0) = 0.f;
        if (k >= 1 && k <= ktf) {
          float r = dts * (F(WF_PH_TEND, k) + 0.5f * gf * em1 * F(WF_W, k));
          if (k < ktf) r = r - dts * (s[WF_FNM][k] * A(WD, k + 1) + s[WF_FNP][k] * A(WD, k));
          A(RR, k) = r;
          A(RHS, k) = F(WF_PH, k) + msfty * r / mut;
        }
      }
    __syncthreads();
    if (on)
  #pragma unroll
      for (int l = 0; l < kAwLevels; ++l) {
        const int k = ty + kAwGroups * l;
        if (k < ktf) A(PP, k) = ep1 * (A(RHS, k + 1) - A(RHS, k)) + em1 * (F(WF_PH, k + 1) - F(WF_PH, k));
      }
    __syncthreads();
    if (on)
  #pragma unroll
      for (int l = 0; l < kAwLevels; ++l) {
        const int k = ty + kAwGroups * l;
        if (k == 0) A(XX, 0) = aw_bc(g, s, j, i);
        if (k >= 1 && k < ktf) {
          const float X1 = F(WF_C2A, k) * rdnw[k] / mut * A(PP, k);
          const float X2 = F(WF_C2A, k - 1) * rdnw[k - 1] / mut * A(PP, k - 1);
          A(XX, k) = F(WF_W, k) + dts * F(WF_RW_TEND, k) + minv * F(WF_CQW, k) * (0.5f * dts * gf * rdn[k] * (X1 - X2)) +
                     dts * gf * minv *
                         (rdn[k] * (F(WF_C2A, k) * F(WF_ALT, k) * A(T2A, k) -
                                    F(WF_C2A, k - 1) * F(WF_ALT, k - 1) * A(T2A, k - 1)) -
                          muave);
        }
        if (k == ktf) {
          const float rm = rdnw[k - 1];
          A(XX, k) = F(WF_W, k) + dts * F(WF_RW_TEND, k) +
                     minv * (-0.5f * dts * gf / mut * (rm * rm) * 2.0f * F(WF_C2A, k - 1) * A(PP, k - 1) -
                             dts * gf * (2.0f * rm * F(WF_C2A, k - 1) * F(WF_ALT, k - 1) * A(T2A, k - 1) + muave));
        }
        // the solve's coefficients, staged for the sweeps (in arrays free until
        // the reverse writes them: rhs is done, Pb and rhsb come later)
        if (k >= 1 && k <= ktf) {
          A(CA, k) = F(WF_A, k);
          A(CAL, k) = F(WF_ALPHA, k);
          A(CG, k) = F(WF_GAMMA, k);
        }
      }
    __syncthreads();
    if (on && ty == 0) {  // the implicit solve's two sweeps
      A(YY, 0) = A(XX, 0);
      for (int k = 1; k <= ktf; ++k) A(YY, k) = (A(XX, k) - A(CA, k) * A(YY, k - 1)) * A(CAL, k);
      A(ZZ, ktf) = A(YY, ktf);
      for (int k = ktf - 1; k >= 1; --k) A(ZZ, k) = A(YY, k) - A(CG, k) * A(ZZ, k + 1);
      A(ZZ, 0) = A(YY, 0);
    }
    __syncthreads();
  }
};

__global__ void __launch_bounds__(32 * kAwGroups) k_advance_w_adj_lp(Grid g, S s, S b, float dts, float* work) {
  extern __shared__ float awsm[];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const bool on = i < g.nx && j < g.ny && mut_in(g, j, i);
  const int nz = g.nz, ktf = nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, c = (size_t)j * g.nx + (on ? i : 0);
  float* red = awsm + (size_t)kAwArrays * nz * 32;  // [4][kAwGroups][32]
  const float ep1 = (float)(1.0 + (double)g.epssm), em1 = (float)(1.0 - (double)g.epssm);
  const float gf = (float)G, t0 = (float)T0;
  float muave = 0.f, muts = 1.f, mut = 1.f, msfty = 1.f;
  if (on) muave = s[WF_MUAVE][c], muts = s[WF_MUTS][c], mut = s[WF_MUT][c], msfty = s[WF_MSFTY][c];
  const float minv = 1.0f / msfty;
  const float* rdnw = s[WF_RDNW];
  const float* rdn = s[WF_RDN];
  const AwLp L{g, s, awsm, nz, ktf, tx, ty, on, lev, c, j, i, dts, ep1, em1, gf, t0, muave, muts, mut, msfty, minv};
  auto A = [&](int arr, int k) -> float& { return L.A(arr, k); };
  auto F = [&](int id, int k) { return s[id][k * lev + c]; };
  auto B = [&](int id, int k) -> float& { return b[id][k * lev + c]; };
  enum { T2A = AwLp::T2A, WD = AwLp::WD, RR = AwLp::RR, PP = AwLp::PP, XX = AwLp::XX, YY = AwLp::YY,
         ZZ = AwLp::ZZ, ZB = AwLp::ZB, YB = AwLp::YB, PB = AwLp::PB, RHSB = AwLp::RHSB, CA = AwLp::CA,
         CAL = AwLp::CAL, CG = AwLp::CG };
  L.forward();
  // ---- reverse
  const float dampmag = (float)((double)dts * 0.2), hpi = (float)(0.5 * 3.14159265359);
  const float cph = msfty * 0.5f * dts * gf * ep1;
  float mutb = 0.f, mutsb = 0.f, muaveb = 0.f, hbotb = 0.f;
  float ph1b[kAwLevels], phbb[kAwLevels], wib[kAwLevels], pbin[kAwLevels];
#pragma unroll
  for (int l = 0; l < kAwLevels; ++l) ph1b[l] = phbb[l] = wib[l] = pbin[l] = 0.f;
  // phi update and damping, per level
  if (on) {
    const float hbot = (F(WF_PH_SAVE, ktf) + F(WF_PHB, ktf)) / gf - kAwHdepth;
#pragma unroll
    for (int l = 0; l < kAwLevels; ++l) {
      const int k = ty + kAwGroups * l;
      if (k == 0) A(ZB, 0) = B(WF_W, 0);
      if (k >= 1 && k <= ktf) {
        const float hk = (F(WF_PH_SAVE, k) + F(WF_PHB, k)) / gf;
        float dk = 0.f;
        if (hk >= hbot) {
          const float sn = sinf(hpi * (hk - hbot) / kAwHdepth);
          dk = dampmag * (sn * sn);
        }
        const float ws = F(WF_W_SAVE, k), den = 1.0f + dk;
        const float wf = (A(ZZ, k) - dk * mut * ws) / den;
        const float pbk = B(WF_PH, k);
        const float wfb = B(WF_W, k) + pbk * cph / muts;
        mutsb += -pbk * cph * wf / (muts * muts);
        A(ZB, k) = wfb / den;
        B(WF_W_SAVE, k) += -wfb * dk * mut / den;
        mutb += -wfb * dk * ws / den;
        if (hk >= hbot) {
          const float db = wfb * (-mut * ws - wf) / den;
          const float th = hpi * (hk - hbot) / kAwHdepth;
          const float thb = db * dampmag * sinf(2.0f * th);
          const float hkb = thb * hpi / kAwHdepth;
          hbotb += -hkb;
          ph1b[l] += hkb / gf;
          phbb[l] += hkb / gf;
        }
      }
    }
  }
  red[(3 * kAwGroups + ty) * 32 + tx] = hbotb;
  __syncthreads();
  if (on && ty == 0) {  // hbot = htop - hdepth, htop = (ph_1 + phb)(ktf) / g: the top level's thread adds it below
    float hb = 0.f;
    for (int y = 0; y < kAwGroups; ++y) hb += red[(3 * kAwGroups + y) * 32 + tx];
    red[(3 * kAwGroups) * 32 + tx] = hb;
    // the transposed solve: z = y - gamma z(k+1) backwards, y = (x - a y(k-1))
    // alpha forwards; the coefficients' cotangents are formed per level after
    // it from the sweeps' values kept in shared memory (zb in wd's array)
    float carry = 0.f;
    for (int k = 1; k <= ktf - 1; ++k) {
      const float zbk = A(ZB, k) + carry;
      A(YB, k) = zbk;
      A(WD, k) = zbk;
      carry = -A(CG, k) * zbk;
    }
    A(YB, ktf) = A(ZB, ktf) + carry;
    A(YB, 0) = A(ZB, 0);
    float yc = 0.f;
    for (int k = ktf; k >= 1; --k) {
      const float ybk = A(YB, k) + yc;
      const float al = A(CAL, k), ak = A(CA, k);
      A(ZB, k) = al * ybk;  // xb
      A(YB, k) = ybk;
      yc = -ak * al * ybk;
    }
    A(ZB, 0) = A(YB, 0) + yc;  // xb(0)
  }
  __syncthreads();
  // explicit w (and t_2ave's reverse), per level in gather form
  if (on) {
    const float hbt = red[(3 * kAwGroups) * 32 + tx];
#pragma unroll
    for (int l = 0; l < kAwLevels; ++l) {
      const int k = ty + kAwGroups * l;
      if (k > ktf) continue;
      if (k == ktf) {
        ph1b[l] += hbt / gf;
        phbb[l] += hbt / gf;
      }
      if (k >= 1) {  // the solve's coefficients
        const float ybk = A(YB, k), al = A(CAL, k);
        if (k <= ktf - 1) B(WF_GAMMA, k) += -A(ZZ, k + 1) * A(WD, k);
        B(WF_A, k) += -A(YY, k - 1) * al * ybk;
        B(WF_ALPHA, k) += (A(XX, k) - A(CA, k) * A(YY, k - 1)) * ybk;
      }
      float c2ab = 0.f, altb = 0.f, pbk = 0.f, t2ab = 0.f;
      if (k >= 1 && k < ktf) {  // the level's own terms
        const float x_b = A(ZB, k);
        if (x_b != 0.f) {
          wib[l] += x_b;
          B(WF_RW_TEND, k) += dts * x_b;
          const float X1 = F(WF_C2A, k) * rdnw[k] / mut * A(PP, k);
          const float X2 = F(WF_C2A, k - 1) * rdnw[k - 1] / mut * A(PP, k - 1);
          const float C1 = minv * F(WF_CQW, k) * 0.5f * dts * gf * rdn[k];
          B(WF_CQW, k) += x_b * minv * 0.5f * dts * gf * rdn[k] * (X1 - X2);
          const float X1b = x_b * C1, X2b = -x_b * C1;
          c2ab += X1b * rdnw[k] / mut * A(PP, k);
          mutb += -X1b * X1 / mut;
          pbk += X1b * F(WF_C2A, k) * rdnw[k] / mut;
          mutb += -X2b * X2 / mut;
          const float Bx = dts * gf * minv * x_b;
          c2ab += Bx * rdn[k] * F(WF_ALT, k) * A(T2A, k);
          altb += Bx * rdn[k] * F(WF_C2A, k) * A(T2A, k);
          t2ab += Bx * rdn[k] * F(WF_C2A, k) * F(WF_ALT, k);
          muaveb += -Bx;
        }
      }
      if (k + 1 >= 1 && k + 1 < ktf) {  // level k + 1's terms on level k
        const float x_b = A(ZB, k + 1);
        if (x_b != 0.f) {
          const float C1 = minv * F(WF_CQW, k + 1) * 0.5f * dts * gf * rdn[k + 1];
          const float X2b = -x_b * C1;
          c2ab += X2b * rdnw[k] / mut * A(PP, k);
          pbk += X2b * F(WF_C2A, k) * rdnw[k] / mut;
          const float Bx = dts * gf * minv * x_b;
          c2ab += -Bx * rdn[k + 1] * F(WF_ALT, k) * A(T2A, k);
          altb += -Bx * rdn[k + 1] * F(WF_C2A, k) * A(T2A, k);
          t2ab += -Bx * rdn[k + 1] * F(WF_C2A, k) * F(WF_ALT, k);
        }
      }
      if (k == ktf) {  // the top level's own terms
        const float x_b = A(ZB, k), rm = rdnw[k - 1];
        wib[l] += x_b;
        B(WF_RW_TEND, k) += dts * x_b;
        const float Ct = minv * (-0.5f * dts * gf / mut * (rm * rm) * 2.0f);
        const float term1 = Ct * F(WF_C2A, k - 1) * A(PP, k - 1);
        mutb += -x_b * term1 / mut;
        muaveb += -minv * dts * gf * x_b;
      }
      if (k == ktf - 1) {  // the top level's terms on the level below it
        const float x_b = A(ZB, ktf), rm = rdnw[ktf - 1];
        const float Ct = minv * (-0.5f * dts * gf / mut * (rm * rm) * 2.0f);
        c2ab += x_b * Ct * A(PP, k);
        pbk += x_b * Ct * F(WF_C2A, k);
        const float Bt = -minv * dts * gf * x_b;
        c2ab += Bt * 2.0f * rm * F(WF_ALT, k) * A(T2A, k);
        altb += Bt * 2.0f * rm * F(WF_C2A, k) * A(T2A, k);
        t2ab += Bt * 2.0f * rm * F(WF_C2A, k) * F(WF_ALT, k);
      }
      if (c2ab != 0.f) B(WF_C2A, k) += c2ab;
      if (altb != 0.f) B(WF_ALT, k) += altb;
      if (k < ktf) {
        A(PB, k) = pbk;
        // t_2ave(k) = (0.5 ((1+e) t_2 + (1-e) t_2ave) + muave t0) / (muts (t0 + t_1))
        const float T = B(WF_T_2SAVE, k) + t2ab;
        const float t1 = F(WF_T_SAVE, k), Dm = muts * (t0 + t1);
        const float ttb = T / Dm;
        muaveb += T * t0 / Dm;
        mutsb += -T * A(T2A, k) / muts;
        B(WF_T_SAVE, k) += -T * A(T2A, k) / (t0 + t1);
        B(WF_T, k) += ttb * 0.5f * ep1;
        B(WF_T_2SAVE, k) = ttb * 0.5f * em1;
      }
    }
  }
  __syncthreads();
  // P(k) = (1+e) (rhs(k+1) - rhs(k)) + (1-e) (ph(k+1) - ph(k)) and
  // rhs(k) = ph(k) + msfty R(k) / mut, per level
  if (on)
#pragma unroll
    for (int l = 0; l < kAwLevels; ++l) {
      const int k = ty + kAwGroups * l;
      if (k > ktf) continue;
      float rhsb = 0.f, pb = k == 0 ? B(WF_PH, 0) : 0.f;
      if (k >= 1) {
        rhsb += B(WF_PH, k) + ep1 * A(PB, k - 1);
        pb += em1 * A(PB, k - 1);
      }
      if (k < ktf) {
        if (k >= 1) rhsb += -ep1 * A(PB, k);
        pb += -em1 * A(PB, k);
      }
      if (k >= 1) {
        pb += rhsb;
        const float Rb = rhsb * msfty / mut;
        mutb += -rhsb * msfty * A(RR, k) / (mut * mut);
        B(WF_PH_TEND, k) += dts * Rb;
        wib[l] += dts * 0.5f * gf * em1 * Rb;
      }
      A(RHSB, k) = rhsb;
      pbin[l] = pb;
    }
  __syncthreads();
  // wdwn(k) = (ww(k) + ww(k-1)) / 2 rdnw(k-1) (ph_1 + phb)(k) - (ph_1 + phb)(k-1),
  // then the level's results
  if (on) {
    const float* fnm = s[WF_FNM];
    const float* fnp = s[WF_FNP];
    auto wdb = [&](int kk) {  // wdwn's cotangent at level kk (1 .. ktf)
      float v = 0.f;
      if (kk - 1 >= 1 && kk - 1 < ktf) v += -dts * fnm[kk - 1] * (A(RHSB, kk - 1) * msfty / mut);
      if (kk >= 1 && kk < ktf) v += -dts * fnp[kk] * (A(RHSB, kk) * msfty / mut);
      return v;
    };
#pragma unroll
    for (int l = 0; l < kAwLevels; ++l) {
      const int k = ty + kAwGroups * l;
      if (k > ktf) continue;
      float wwb = 0.f;
      if (k >= 1) {
        const float w = wdb(k);
        if (w != 0.f) {
          const float h = 0.5f * rdnw[k - 1];
          const float dph = F(WF_PH_SAVE, k) - F(WF_PH_SAVE, k - 1) + F(WF_PHB, k) - F(WF_PHB, k - 1);
          wwb += w * h * dph;
          const float dphb = w * h * (F(WF_WW, k) + F(WF_WW, k - 1));
          ph1b[l] += dphb;
          phbb[l] += dphb;
        }
      }
      if (k + 1 <= ktf) {
        const float w = wdb(k + 1);
        if (w != 0.f) {
          const float h = 0.5f * rdnw[k];
          const float dph = F(WF_PH_SAVE, k + 1) - F(WF_PH_SAVE, k) + F(WF_PHB, k + 1) - F(WF_PHB, k);
          wwb += w * h * dph;
          const float dphb = w * h * (F(WF_WW, k + 1) + F(WF_WW, k));
          ph1b[l] += -dphb;
          phbb[l] += -dphb;
        }
      }
      if (wwb != 0.f) B(WF_WW, k) += wwb;
      B(WF_PH_SAVE, k) += ph1b[l];
      B(WF_PHB, k) += phbb[l];
      B(WF_PH, k) = pbin[l];
      B(WF_W, k) = wib[l];  // w(0) is replaced by the lower boundary value: wib = 0 there
    }
  }
  red[(0 * kAwGroups + ty) * 32 + tx] = mutb;
  red[(1 * kAwGroups + ty) * 32 + tx] = mutsb;
  red[(2 * kAwGroups + ty) * 32 + tx] = muaveb;
  __syncthreads();
  if (on && ty == 0) {
    float m0 = 0.f, m1 = 0.f, m2 = 0.f;
    for (int y = 0; y < kAwGroups; ++y) {
      m0 += red[(0 * kAwGroups + y) * 32 + tx];
      m1 += red[(1 * kAwGroups + y) * 32 + tx];
      m2 += red[(2 * kAwGroups + y) * 32 + tx];
    }
    b[WF_MUT][c] += m0;
    b[WF_MUTS][c] += m1;
    b[WF_MUAVE][c] += m2;
    work[c] = A(ZB, 0);
  }
}

// advance_w forward over a block's level groups (the stand-alone operator;
// in the step k_acoustic_col does this work): the recomputation above, then
// per level the Rayleigh damping, w and the phi update
__global__ void __launch_bounds__(32 * kAwGroups) k_advance_w_lp(Grid g, S s, float dts) {
  extern __shared__ float awsm[];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  const bool on = i < g.nx && j < g.ny && mut_in(g, j, i);
  const int nz = g.nz, ktf = nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, c = (size_t)j * g.nx + (on ? i : 0);
  const float ep1 = (float)(1.0 + (double)g.epssm), em1 = (float)(1.0 - (double)g.epssm);
  const float gf = (float)G, t0 = (float)T0;
  float muave = 0.f, muts = 1.f, mut = 1.f, msfty = 1.f;
  if (on) muave = s[WF_MUAVE][c], muts = s[WF_MUTS][c], mut = s[WF_MUT][c], msfty = s[WF_MSFTY][c];
  const AwLp L{g, s, awsm, nz, ktf, tx, ty, on, lev, c, j, i, dts, ep1, em1, gf, t0, muave, muts, mut, msfty,
               1.0f / msfty};
  L.forward();
  if (!on) return;
  const float dampmag = (float)((double)dts * 0.2), hpi = (float)(0.5 * 3.14159265359);
  const float hbot = (L.F(WF_PH_SAVE, ktf) + L.F(WF_PHB, ktf)) / gf - kAwHdepth;
#pragma unroll
  for (int l = 0; l < kAwLevels; ++l) {
    const int k = ty + kAwGroups * l;
    if (k > ktf) continue;
    if (k < ktf) s[WF_T_2SAVE][k * lev + c] = L.A(AwLp::T2A, k);
    if (k == 0) {
      s[WF_W][c] = L.A(AwLp::ZZ, 0);
      continue;
    }
    const float hk = (L.F(WF_PH_SAVE, k) + L.F(WF_PHB, k)) / gf;
    float dw = 0.f;
    if (hk >= hbot) {
      const float sn = sinf(hpi * (hk - hbot) / kAwHdepth);
      dw = dampmag * (sn * sn);
    }
    const float wf = (L.A(AwLp::ZZ, k) - dw * mut * L.F(WF_W_SAVE, k)) / (1.0f + dw);
    const float rhs = L.F(WF_PH, k) + msfty * L.A(AwLp::RR, k) / mut;
    s[WF_W][k * lev + c] = wf;
    s[WF_PH][k * lev + c] = rhs + msfty * 0.5f * dts * gf * ep1 * wf / muts;
  }
}

__global__ void k_advance_w_adj_bc(Grid g, S s, S b, const float* work) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k > 2) return;
  const int nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, c = (size_t)j * nx + i, p = k * lev + c;
  const float* ht = s[WF_HT];
  auto Y = [&](int jj, int ii) {
    if (jj < 0 || ii < 0 || jj >= g.ny || ii >= nx || !mut_in(g, jj, ii)) return 0.f;
    return work[(size_t)jj * nx + ii] * s[WF_MSFTY][(size_t)jj * nx + ii];
  };
  auto Xx = [&](int jj, int ii) {
    if (jj < 0 || ii < 0 || jj >= g.ny || ii >= nx || !mut_in(g, jj, ii)) return 0.f;
    return work[(size_t)jj * nx + ii] * s[WF_MSFTX][(size_t)jj * nx + ii];
  };
  const float cfk = k == 0 ? g.cf1 : k == 1 ? g.cf2 : g.cf3;
  const float ys = Y(j - 1, i), yc = Y(j, i), xw = Xx(j, i - 1), xc = Xx(j, i);
  if (ys != 0.f || yc != 0.f) b[WF_V][p] += cfk * 0.5f * g.rdy * (ht[c] - ht[c - nx]) * (ys + yc);
  if (xw != 0.f || xc != 0.f) b[WF_U][p] += cfk * 0.5f * g.rdx * (ht[c] - ht[c - 1]) * (xw + xc);
  if (k == 0) {
    const float* u = s[WF_U];
    const float* v = s[WF_V];
    auto cv = [&](size_t cc) { return g.cf1 * v[cc] + g.cf2 * v[lev + cc] + g.cf3 * v[2 * lev + cc]; };
    auto cu = [&](size_t cc) { return g.cf1 * u[cc] + g.cf2 * u[lev + cc] + g.cf3 * u[2 * lev + cc]; };
    const float yn = Y(j + 1, i), xe = Xx(j, i + 1);
    float h = 0.f;
    if (ys != 0.f) h += 0.5f * g.rdy * ys * cv(c);
    if (yc != 0.f) h += 0.5f * g.rdy * yc * (cv(c) - cv(c + nx));
    if (yn != 0.f) h += -0.5f * g.rdy * yn * cv(c + nx);
    if (xw != 0.f) h += 0.5f * g.rdx * xw * cu(c);
    if (xc != 0.f) h += 0.5f * g.rdx * xc * (cu(c) - cu(c + 1));
    if (xe != 0.f) h += -0.5f * g.rdx * xe * cu(c + 1);
    if (h != 0.f) b[WF_HT][c] += h;
  }
}

int launch_advance_w(const Grid& g, const S& s, float dts, cudaStream_t st) {
  const size_t smem = advance_w_adj_smem(g);
  static size_t granted = 48 * 1024;
  if (smem > granted) {
    cudaFuncSetAttribute(k_advance_w_lp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    granted = smem;
  }
  k_advance_w_lp<<<dim3((g.nx + 31) / 32, g.ny), dim3(32, kAwGroups), smem, st>>>(g, s, dts);
  return 1;
}

int launch_advance_w_adj(const Grid& g, const S& s, const S& b, float dts, float* work, cudaStream_t st) {
  const dim3 bl(32, kAwGroups), b3(32, 4);
  const size_t smem = advance_w_adj_smem(g);
  static size_t granted = 48 * 1024;
  if (smem > granted) {
    cudaFuncSetAttribute(k_advance_w_adj_lp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    granted = smem;
  }
  k_advance_w_adj_lp<<<dim3((g.nx + 31) / 32, g.ny), bl, smem, st>>>(g, s, b, dts, work);
  k_advance_w_adj_bc<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, work);
  return 2;
}

// stagger of a relaxed field: the bounds of relax_bdytend's zones and levels
// ('u': ibe = ide, 'v': jbe = jde, 'h'/'m': all nz levels, else nz - 1)
struct RelaxShape {
  int ibe, jbe, nk;
};

__host__ __device__ inline RelaxShape relax_shape(const Grid& g, char var) {
  RelaxShape r{g.ide - 1, g.jde - 1, g.nz - 1};
  if (var == 'u') r.ibe = g.ide;
  if (var == 'v') r.jbe = g.jde;
  if (var == 'h' || var == 'm') r.nk = g.nz;
  return r;
}

__global__ void k_relax_field(Grid g, S s, RelaxShape r, const float* field, float* tend, float dtbc) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= r.nk) return;
  const int nx = g.nx, ny = g.ny;
  float* o = tend + ((size_t)k * ny + j) * nx + i;
  relax_point(g, s, 0, k, j, i, r.ibe, r.jbe, r.nk,
              [&](int kk, int jj, int ii) { return field[((size_t)kk * ny + jj) * nx + ii]; }, dtbc, o);
}

__global__ void k_relax_field_adj(Grid g, RelaxShape r, const float* tbar, float* fbar) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= r.nk) return;
  const int nx = g.nx, ny = g.ny;
  const size_t p = ((size_t)k * ny + j) * nx + i;
  float acc = 0.f;
  const int b0 = relax_zone_b(g, j, i, r.ibe, r.jbe);
  if (b0) acc -= (kFcx[b0] + 4.0f * kGcx[b0]) * tbar[p];
  const int dj[4] = {0, 0, -1, 1}, di[4] = {-1, 1, 0, 0};
  for (int n = 0; n < 4; ++n) {
    const int jj = j + dj[n], ii = i + di[n];
    if (jj < 0 || jj >= ny || ii < 0 || ii >= nx) continue;
    const int b = relax_zone_b(g, jj, ii, r.ibe, r.jbe);
    if (b) acc += kGcx[b] * tbar[((size_t)k * ny + jj) * nx + ii];
  }
  if (acc != 0.f) fbar[p] += acc;
}

int launch_relax_field(const Grid& g, const float* field, float* tend, const float* const* bdy8, char var, float dtbc,
                       cudaStream_t st) {
  S s{};
  for (int q = 0; q < 8; ++q) s.f[q] = const_cast<float*>(bdy8[q]);
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (var == 'm') g2.nz = 1;  // mu is 2-D
  k_relax_field<<<point_grid(g2, b3), b3, 0, st>>>(g2, s, relax_shape(g2, var), field, tend, dtbc);
  return 1;
}

int launch_relax_field_adj(const Grid& g, const float* tbar, float* fbar, char var, cudaStream_t st) {
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (var == 'm') g2.nz = 1;
  k_relax_field_adj<<<point_grid(g2, b3), b3, 0, st>>>(g2, relax_shape(g2, var), tbar, fbar);
  return 1;
}

__global__ void k_vsolve_w(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                           float* w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t lev = (size_t)ncol;
  const int kend = nz - 1;
  float prev = x[c];
  w[c] = prev;
  for (int k = 1; k <= kend; ++k) {
    const size_t p = k * lev + c;
    prev = (x[p] - a[p] * prev) * alpha[p];
    w[p] = prev;
  }
  for (int k = kend - 1; k >= 1; --k) {
    const size_t p = k * lev + c;
    prev = w[p] - gamma[p] * prev;
    w[p] = prev;
  }
}

__global__ void k_vsolve_w_adj(int ncol, int nz, const float* x, const float* a, const float* alpha,
                               const float* gamma, const float* wbar, float* xbar, float* abar, float* alphabar,
                               float* gammabar) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const size_t lev = (size_t)ncol;
  const int kend = nz - 1;
  float y[kMaxNz], z[kMaxNz], zb[kMaxNz], yb[kMaxNz];
  // forward recomputation
  y[0] = x[c];
  for (int k = 1; k <= kend; ++k) {
    const size_t p = k * lev + c;
    y[k] = (x[p] - a[p] * y[k - 1]) * alpha[p];
  }
  z[kend] = y[kend];
  for (int k = kend - 1; k >= 1; --k) z[k] = y[k] - gamma[k * lev + c] * z[k + 1];
  z[0] = y[0];
  for (int k = 0; k <= kend; ++k) {
    zb[k] = wbar[k * lev + c];
    yb[k] = 0.f;
  }
  // back-substitution in reverse (it computed k = kend-1 down to 1)
  for (int k = 1; k <= kend - 1; ++k) {
    const size_t p = k * lev + c;
    yb[k] += zb[k];
    gammabar[p] += -z[k + 1] * zb[k];
    zb[k + 1] += -gamma[p] * zb[k];
  }
  yb[kend] += zb[kend];
  yb[0] += zb[0];
  // forward sweep in reverse (it computed k = 1 up to kend)
  for (int k = kend; k >= 1; --k) {
    const size_t p = k * lev + c;
    const float al = alpha[p], ak = a[p];
    xbar[p] += al * yb[k];
    abar[p] += -y[k - 1] * al * yb[k];
    alphabar[p] += (x[p] - ak * y[k - 1]) * yb[k];
    yb[k - 1] += -ak * al * yb[k];
  }
  xbar[c] += yb[0];
}

int launch_vsolve_w(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma, float* w,
                    cudaStream_t st) {
  k_vsolve_w<<<(ncol + 127) / 128, 128, 0, st>>>(ncol, nz, x, a, alpha, gamma, w);
  return 1;
}

int launch_vsolve_w_adj(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                        const float* wbar, float* xbar, float* abar, float* alphabar, float* gammabar,
                        cudaStream_t st) {
  k_vsolve_w_adj<<<(ncol + 127) / 128, 128, 0, st>>>(ncol, nz, x, a, alpha, gamma, wbar, xbar, abar, alphabar,
                                                      gammabar);
  return 1;
}

// one column of calc_coef_w's adjoint; the forward is k_coef_w (k_acoustic.cu)
// (the cotangent arrays are the caller's own buffers, distinct from the
// operands: __restrict__ lets the level loops' loads run ahead of their
// stores)
__global__ void k_coef_w_adj(Grid g, const float* __restrict__ mut_, const float* __restrict__ cqw,
                             const float* __restrict__ c2a, const float* __restrict__ rdn,
                             const float* __restrict__ rdnw, float dts, const float* __restrict__ abar,
                             const float* __restrict__ alphabar, const float* __restrict__ gammabar,
                             float* __restrict__ mutbar, float* __restrict__ cqwbar, float* __restrict__ c2abar) {
  WRF_COLUMN_INDEX(g, j, i);
  if (j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const int nz = g.nz;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const double cofd = (0.5 * (double)dts * G * (1.0 + (double)g.epssm)) * (0.5 * (double)dts * G * (1.0 + (double)g.epssm));
  const float cof = (float)cofd, cofm2 = (float)(-2.0 * cofd), cof2 = (float)(2.0 * cofd);
  const float mut = mut_[c];
  const float mm = mut * mut;
  const float lid = g.top_lid ? 0.f : 1.f;
  float ak[kMaxNz], bk[kMaxNz], ck[kMaxNz], al[kMaxNz], gm[kMaxNz];
  // forward recomputation (k_coef_w's arithmetic)
  const float c2t = c2a[(nz - 2) * lev + c], rwt = rdnw[nz - 2];
  const float atop = cofm2 * (rwt * rwt) * c2t * lid / mm;
  gm[0] = 0.f;
#pragma unroll 4
  for (int k = 1; k < nz - 1; ++k) {
    const size_t p = k * lev + c;
    const float cw = cqw[p];
    ak[k] = k >= 2 ? -cw * cof * rdn[k] * rdnw[k - 1] * c2a[p - lev] / mm : 0.f;
    bk[k] = 1.0f + cw * cof * rdn[k] * (rdnw[k] * c2a[p] / mm + rdnw[k - 1] * c2a[p - lev] / mm);
    ck[k] = -cw * cof * rdn[k] * rdnw[k] * c2a[p] / mm;
    al[k] = 1.0f / (bk[k] - ak[k] * gm[k - 1]);
    gm[k] = ck[k] * al[k];
  }
  const float btop = 1.0f + cof2 * (rwt * rwt) * c2t / mm;
  const float altop = 1.0f / (btop - atop * gm[nz - 2]);
  // reverse
  float mmb = 0.f, c2tb = 0.f;
  float gmb = 0.f;  // cotangent of gm[k] flowing down from level k+1
  {
    const float alb = alphabar[(nz - 1) * lev + c];
    const float bb = -altop * altop * alb;
    const float atb = abar[(nz - 1) * lev + c] + altop * altop * gm[nz - 2] * alb;
    gmb = altop * altop * atop * alb;
    // btop = 1 + cof2 rwt^2 c2t / mm ; atop = cofm2 rwt^2 c2t lid / mm
    c2tb += bb * cof2 * (rwt * rwt) / mm + atb * cofm2 * (rwt * rwt) * lid / mm;
    mmb += -bb * (btop - 1.0f) / mm - atb * atop / mm;
  }
  float c2b_next = 0.f;  // cotangent of c2a at level k (from the k+1 step's c2a(k) terms)
#pragma unroll 4
  for (int k = nz - 2; k >= 1; --k) {
    const size_t p = k * lev + c;
    const float cw = cqw[p];
    const float g_k = gammabar[p] + gmb;               // total cotangent of gm[k]
    const float ccb = g_k * al[k];
    const float alb = alphabar[p] + g_k * ck[k];        // total cotangent of al[k]
    const float a2 = al[k] * al[k];
    const float bb = -a2 * alb;
    const float akb = (k >= 2 ? abar[p] : 0.f) + a2 * gm[k - 1] * alb;
    gmb = a2 * ak[k] * alb;                             // to gm[k-1]
    const float base = cof * rdn[k] / mm;
    const float c2k = c2a[p], c2m = c2a[p - lev];
    // cqw
    float cwb = bb * base * (rdnw[k] * c2k + rdnw[k - 1] * c2m) - ccb * base * rdnw[k] * c2k;
    if (k >= 2) cwb += -akb * base * rdnw[k - 1] * c2m;
    cqwbar[p] += cwb;
    // c2a(k) and c2a(k-1)
    float c2kb = bb * cw * base * rdnw[k] - ccb * cw * base * rdnw[k] + c2b_next;
    float c2mb = bb * cw * base * rdnw[k - 1];
    if (k >= 2) c2mb += -akb * cw * base * rdnw[k - 1];
    if (k == nz - 2) c2kb += c2tb;
    c2abar[p] += c2kb;
    c2b_next = c2mb;
    // mm
    mmb += -bb * (bk[k] - 1.0f) / mm - ccb * ck[k] / mm - (k >= 2 ? akb * ak[k] / mm : 0.f);
  }
  c2abar[c] += c2b_next;  // c2a(0), from level 1
  mutbar[c] += mmb * 2.0f * mut;
}

int launch_coef_w_adj(const Grid& g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                      const float* rdnw, float dts, const float* abar, const float* alphabar, const float* gammabar,
                      float* mutbar, float* cqwbar, float* c2abar, cudaStream_t st) {
  const dim3 b2(32, 8);
  k_coef_w_adj<<<col_grid(g, b2), b2, 0, st>>>(g, mut, cqw, c2a, rdn, rdnw, dts, abar, alphabar, gammabar, mutbar,
                                               cqwbar, c2abar);
  return 1;
}

// ------------------------------------------------------- momentum advection

namespace {

// the linear forms of one face flux F = V Phi: Phi = sum qc[n] q[qi[n]],
// V = sum rc[n] r[ri[n]] (r: ru for x faces, rv for y faces, rom for z faces)
struct FaceLin {
  int nq = 0, nr = 0;
  size_t qi[6];
  float qc[6];
  size_t ri[2];
  float rc[2];
};

struct MomAdjArgs {
  const float *q, *ru, *rv, *rom, *msf, *msf2, *fzm, *fzp, *rdz;
};

__device__ __forceinline__ size_t off(size_t b, int o, size_t st) {
  return (size_t)((long long)b + (long long)o * (long long)st);
}
__device__ __forceinline__ void put5(FaceLin& L, size_t b, size_t st, float s) {
  L.nq = 6;
  for (int o = -3; o <= 2; ++o) {
    L.qi[o + 3] = off(b, o, st);
    L.qc[o + 3] = w5(o, s);
  }
}
__device__ __forceinline__ void put3(FaceLin& L, size_t b, size_t st, float s) {
  L.nq = 4;
  for (int o = -2; o <= 1; ++o) {
    L.qi[o + 2] = off(b, o, st);
    L.qc[o + 2] = w3(o, s);
  }
}
__device__ __forceinline__ void put2(FaceLin& L, size_t i0, float c0, size_t i1, float c1) {
  L.nq = 2;
  L.qi[0] = i0;
  L.qc[0] = c0;
  L.qi[1] = i1;
  L.qc[1] = c1;
}
// V = c0 r[i0] + c1 r[i1], returned
__device__ __forceinline__ float putr(FaceLin& L, const float* r, size_t i0, float c0, size_t i1, float c1) {
  L.nr = 2;
  L.ri[0] = i0;
  L.rc[0] = c0;
  L.ri[1] = i1;
  L.rc[1] = c1;
  return c0 * r[i0] + c1 * r[i1];
}

// Face D (0 y, 1 x, 2 z) of component C at (k, j, i): the face index is j,
// i or k along D.  Returns false where the forward has no flux.  The cases
// and their order are those of fqy_u .. vf_w (k_tend.cu).
template <int C, int D>
__device__ bool face_lin(const Grid& g, const MomAdjArgs& a, int k, int j, int i, FaceLin& L) {
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const size_t p = (size_t)k * lev + (size_t)j * nx + i;
  const float* q = a.q;
  if (D == 0) {  // y faces, rv
    const int jf = j;
    float v;
    if (C == 0) {
      v = putr(L, a.rv, p, 0.5f, p - 1, 0.5f);
      if (jf >= jds + 3 && jf < jde - 3) put5(L, p, nx, sgnf(v));
      else if (jf == jds + 1) put2(L, p, 0.5f, p - nx, 0.5f);
      else if (jf == jds + 2) put3(L, p, nx, sgnf(v));
      else if (jf == jde - 2) put2(L, p, 0.5f, p - nx, 0.5f);
      else if (jf == jde - 3) put3(L, p, nx, 1.0f);  // the reference's sign source there is 0
      else return false;
    } else if (C == 1) {
      v = putr(L, a.rv, p, 0.5f, p - nx, 0.5f);
      if (jf >= jds + 3 && jf < jde - 2) put5(L, p, nx, sgnf(v));
      else if (jf == jds + 1) {
        if (q[p] < 0.f) put2(L, p, 1.0f, p - nx, 0.0f);
        else put2(L, p, 0.5f, p - nx, 0.5f);
      } else if (jf == jds + 2) put3(L, p, nx, sgnf(v));
      else if (jf == jde - 1) {
        if (q[p - nx] > 0.f) put2(L, p - nx, 1.0f, p, 0.0f);
        else put2(L, p - nx, 0.5f, p, 0.5f);
      } else if (jf == jde - 2) put3(L, p, nx, sgnf(v));
      else return false;
    } else {
      if (k < 1) return false;
      v = k < ktf ? putr(L, a.rv, p, a.fzm[k], p - lev, a.fzp[k])
                  : putr(L, a.rv, p - lev, 2.0f - a.fzm[ktf - 1], p - 2 * lev, -a.fzp[ktf - 1]);
      if (jf >= jds + 3 && jf < jde - 3) put5(L, p, nx, sgnf(v));
      else if (jf == jds + 1) put2(L, p, 0.5f, p - nx, 0.5f);
      else if (jf == jds + 2) put3(L, p, nx, sgnf(v));
      else if (jf == jde - 2) put2(L, p, 0.5f, p - nx, 0.5f);
      else if (jf == jde - 3) put3(L, p, nx, sgnf(v));
      else return false;
    }
    return true;
  } else if (D == 1) {  // x faces, ru
    const int f = i;
    float v;
    if (C == 0) {
      v = putr(L, a.ru, p, 0.5f, p - 1, 0.5f);
      if (f >= ids + 3 && f < ide - 2) put5(L, p, 1, sgnf(v));
      else if (f == ids + 1) {
        if (q[p] < 0.f) put2(L, p, 1.0f, p - 1, 0.0f);
        else put2(L, p, 0.5f, p - 1, 0.5f);
      } else if (f == ids + 2) put3(L, p, 1, sgnf(v));
      else if (f == ide - 1) {
        if (q[p - 1] > 0.f) put2(L, p - 1, 1.0f, p, 0.0f);
        else put2(L, p - 1, 0.5f, p, 0.5f);
      } else if (f == ide - 2) put3(L, p, 1, sgnf(v));
      else return false;
    } else if (C == 1) {
      v = putr(L, a.ru, p, 0.5f, p - nx, 0.5f);
      if (f >= ids + 3 && f < ide - 3) put5(L, p, 1, sgnf(v));
      else if (f == ids + 1) put2(L, p, 0.5f, p - 1, 0.5f);
      else if (f == ids + 2) put3(L, p, 1, sgnf(v));
      else if (f == ide - 2) put2(L, p, 0.5f, p - 1, 0.5f);
      else if (f == ide - 3) put3(L, p, 1, sgnf(v));
      else return false;
    } else {
      if (k < 1) return false;
      v = k < ktf ? putr(L, a.ru, p, a.fzm[k], p - lev, a.fzp[k])
                  : putr(L, a.ru, p - lev, 2.0f - a.fzm[ktf - 1], p - 2 * lev, -a.fzp[ktf - 1]);
      if (f >= ids + 3 && f < ide - 3) put5(L, p, 1, sgnf(v));
      else if (f == ids + 1) put2(L, p, 0.5f, p - 1, 0.5f);
      else if (f == ids + 2) put3(L, p, 1, sgnf(v));
      else if (f == ide - 2) put2(L, p, 0.5f, p - 1, 0.5f);
      else if (f == ide - 3) put3(L, p, 1, sgnf(v));
      else return false;
    }
    return true;
  } else {  // vertical faces, rom
    const int kf = k;
    if (kf < 1) return false;
    if (C == 0 || C == 1) {
      const size_t nb = C == 0 ? 1 : (size_t)nx;  // the second rom point: i-1 (u) or j-1 (v)
      const float v = putr(L, a.rom, p, 0.5f, p - nb, 0.5f);
      if (kf >= 3 && kf < ktf - 2) put5(L, p, lev, sgnf(-v));
      else if (kf == 1) put2(L, p, a.fzm[kf], p - lev, a.fzp[kf]);
      else if (kf == 2) put3(L, p, lev, sgnf(-v));
      else if (kf == ktf - 2) put3(L, p, lev, C == 0 ? sgnf(-v) : sgnf(v));
      else if (kf == ktf - 1) put2(L, p, a.fzm[kf], p - lev, a.fzp[kf]);
      else return false;
    } else {
      const float v = putr(L, a.rom, p, 0.5f, p - lev, 0.5f);
      if (kf >= 3 && kf < ktf - 1) put5(L, p, lev, sgnf(-v));
      else if (kf == 1) put2(L, p, 0.5f, p - lev, 0.5f);
      else if (kf == 2) put3(L, p, lev, sgnf(-v));
      else if (kf == ktf - 1) put3(L, p, lev, sgnf(v));
      else if (kf == ktf) put2(L, p, 0.5f, p - lev, 0.5f);
      else return false;
    }
    return true;
  }
}

// the tendency coefficient of direction D in cell (k, j, i) of component C
// (0 outside the cells that direction updates); advect_w's top cell, which
// adds 2 rdz(ktf-1) F(ktf), is handled by fbar
template <int C, int D>
__device__ __forceinline__ float cell_coef(const Grid& g, const MomAdjArgs& a, int k, int j, int i) {
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  if (k < 0 || j < 0 || i < 0 || j >= g.ny || i >= g.nx) return 0.f;
  const int c = j * g.nx + i;
  if (C == 0) {
    if (!(k < ktf && j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1)) return 0.f;
    if (D == 0) return (j >= jds + 1 && j < jde - 2) ? a.msf[c] * g.rdy : 0.f;
    if (D == 1) return a.msf[c] * g.rdx;
    return a.rdz[k];
  } else if (C == 1) {
    if (!(k < ktf && j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1)) return 0.f;
    if (D == 0) return a.msf[c] * g.rdy;
    if (D == 1) return (i >= ids + 1 && i < ide - 2) ? a.msf[c] * g.rdx : 0.f;
    return (a.msf[c] / a.msf2[c]) * a.rdz[k];
  } else {
    if (!(k >= 1 && k <= ktf && j >= jds && j < jde - 1 && i >= ids && i < ide - 1)) return 0.f;
    if (D == 0) return (j >= jds + 1 && j < jde - 2) ? a.msf[c] * g.rdy : 0.f;
    if (D == 1) return (i >= ids + 1 && i < ide - 2) ? a.msf[c] * g.rdx : 0.f;
    return k < ktf ? a.rdz[k] : 0.f;
  }
}

// Fbar of face D at (k, j, i): each cell subtracts coef (F(upper) - F(lower))
template <int C, int D>
__device__ float fbar(const Grid& g, const MomAdjArgs& a, const float* tbar, int k, int j, int i) {
  if (k < 0 || k >= g.nz || j < 0 || j >= g.ny || i < 0 || i >= g.nx) return 0.f;
  const size_t lev = (size_t)g.ny * g.nx;
  auto tb = [&](int kk, int jj, int ii) { return tbar[(size_t)kk * lev + (size_t)jj * g.nx + ii]; };
  float v = 0.f;
  const float c0 = cell_coef<C, D>(g, a, k, j, i);
  if (c0 != 0.f) v += c0 * tb(k, j, i);
  const int k1 = D == 2 ? k - 1 : k, j1 = D == 0 ? j - 1 : j, i1 = D == 1 ? i - 1 : i;
  const float c1 = cell_coef<C, D>(g, a, k1, j1, i1);
  if (c1 != 0.f) v -= c1 * tb(k1, j1, i1);
  if (C == 2 && D == 2 && k == g.nz - 1) {  // advect_w's top cell: tend += 2 rdz(ktf-1) F(ktf)
    const int ktf = g.nz - 1;
    if (j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1) v += 2.0f * a.rdz[ktf - 1] * tb(ktf, j, i);
  }
  return v;
}

// The two passes of the momentum adjoint.  Pass 1 (one thread per point,
// taken as the face index of each direction D) forms every face once: its
// cotangent Fbar, velocity V and face value Phi, then the face's
// contributions Fbar V dPhi/dq to the field at its stencil offsets o in
// [-3, 2] along D, stored in slot o + 3 of the face (Q, 6 slots per
// direction), and Fbar Phi dV/dr to the velocity points p - d (R, one slot
// per distance d of the component's velocity forms: d in {0, 1} for u,
// {0, nx} for v, {0, lev, 2 lev} for w).  Pass 2 gathers each point's
// cotangents from the slots that address it, in a fixed order (one writer
// per output element, no atomics).
template <int C>
__device__ __forceinline__ int r_slot(size_t d, size_t nx, size_t lev) {
  if (C == 0) return (int)d;
  if (C == 1) return d == 0 ? 0 : 1;
  return d == 0 ? 0 : (d == lev ? 1 : 2);
}
template <int C>
__device__ __forceinline__ size_t r_dist(int s, size_t nx, size_t lev) {
  if (C == 0) return (size_t)s;
  if (C == 1) return s == 0 ? 0 : nx;
  return (size_t)s * lev;
}
template <int C>
__host__ __device__ constexpr int r_slots() {
  return C == 2 ? 3 : 2;
}

template <int C, int D>
__device__ __forceinline__ void face_pass(const Grid& g, const MomAdjArgs& a, const float* tbar, int k, int j, int i,
                                          size_t p, size_t n3, float* Q, float* R) {
  const size_t lev = (size_t)g.ny * g.nx, nx = g.nx;
  float q6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, r3[3] = {0.f, 0.f, 0.f};
  const float fb = fbar<C, D>(g, a, tbar, k, j, i);
  FaceLin L;
  if (fb != 0.f && face_lin<C, D>(g, a, k, j, i, L)) {
    const float* r = D == 0 ? a.rv : D == 1 ? a.ru : a.rom;
    const long long st = D == 0 ? (long long)nx : D == 1 ? 1 : (long long)lev;
    float v = 0.f, phi = 0.f;
    for (int n = 0; n < L.nr; ++n) v += L.rc[n] * r[L.ri[n]];
    for (int n = 0; n < L.nq; ++n) phi += L.qc[n] * a.q[L.qi[n]];
    const float gv = fb * v, gp = fb * phi;
    for (int n = 0; n < L.nq; ++n) {
      const int slot = (int)(((long long)L.qi[n] - (long long)p) / st) + 3;
#pragma unroll
      for (int s = 0; s < 6; ++s) q6[s] += slot == s ? gv * L.qc[n] : 0.f;
    }
    for (int n = 0; n < L.nr; ++n) {
      const int slot = r_slot<C>(p - L.ri[n], nx, lev);
#pragma unroll
      for (int s = 0; s < 3; ++s) r3[s] += slot == s ? gp * L.rc[n] : 0.f;
    }
  }
#pragma unroll
  for (int s = 0; s < 6; ++s) Q[(size_t)(D * 6 + s) * n3 + p] = q6[s];
#pragma unroll
  for (int s = 0; s < r_slots<C>(); ++s) R[(size_t)(D * 3 + s) * n3 + p] = r3[s];
}

}  // namespace

template <int C>
__global__ void k_advect_mom_faces(Grid g, MomAdjArgs a, const float* tbar, float* Q, float* R) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t n3 = g.n3(), p = ((size_t)k * g.ny + j) * g.nx + i;
  face_pass<C, 0>(g, a, tbar, k, j, i, p, n3, Q, R);
  face_pass<C, 1>(g, a, tbar, k, j, i, p, n3, Q, R);
  face_pass<C, 2>(g, a, tbar, k, j, i, p, n3, Q, R);
}

template <int C>
__global__ void k_advect_mom_gather(Grid g, const float* Q, const float* R, float* qbar, float* rubar, float* rvbar,
                                    float* rombar) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t n3 = g.n3(), lev = (size_t)g.ny * g.nx, nx = g.nx;
  const size_t m = ((size_t)k * g.ny + j) * g.nx + i;
  float aq = 0.f;
#pragma unroll
  for (int D = 0; D < 3; ++D) {
    const long long st = D == 0 ? (long long)nx : D == 1 ? 1 : (long long)lev;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const long long f = (long long)m - (long long)(s - 3) * st;
      if (f >= 0 && f < (long long)n3) aq += Q[(size_t)(D * 6 + s) * n3 + (size_t)f];
    }
  }
  if (aq != 0.f) qbar[m] += aq;
  float ar[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int D = 0; D < 3; ++D)
#pragma unroll
    for (int s = 0; s < r_slots<C>(); ++s) {
      const size_t f = m + r_dist<C>(s, nx, lev);
      if (f < n3) ar[D] += R[(size_t)(D * 3 + s) * n3 + f];
    }
  if (ar[0] != 0.f) rvbar[m] += ar[0];
  if (ar[1] != 0.f) rubar[m] += ar[1];
  if (ar[2] != 0.f) rombar[m] += ar[2];
}

size_t advect_mom_adj_work_floats(const Grid& g) { return (size_t)(18 + 9) * g.n3(); }

int launch_advect_mom_adj(const Grid& g, int component, const float* q, const float* ru, const float* rv,
                          const float* rom, const float* msf, const float* msf2, const float* fzm, const float* fzp,
                          const float* rdz, const float* tbar, float* qbar, float* rubar, float* rvbar,
                          float* rombar, float* work, cudaStream_t st) {
  const dim3 b3(32, 4);
  const MomAdjArgs a{q, ru, rv, rom, msf, msf2, fzm, fzp, rdz};
  float* Q = work;
  float* R = work + 18 * g.n3();
  if (component == 0) {
    k_advect_mom_faces<0><<<point_grid(g, b3), b3, 0, st>>>(g, a, tbar, Q, R);
    k_advect_mom_gather<0><<<point_grid(g, b3), b3, 0, st>>>(g, Q, R, qbar, rubar, rvbar, rombar);
  } else if (component == 1) {
    k_advect_mom_faces<1><<<point_grid(g, b3), b3, 0, st>>>(g, a, tbar, Q, R);
    k_advect_mom_gather<1><<<point_grid(g, b3), b3, 0, st>>>(g, Q, R, qbar, rubar, rvbar, rombar);
  } else {
    k_advect_mom_faces<2><<<point_grid(g, b3), b3, 0, st>>>(g, a, tbar, Q, R);
    k_advect_mom_gather<2><<<point_grid(g, b3), b3, 0, st>>>(g, Q, R, qbar, rubar, rvbar, rombar);
  }
  return 2;
}

size_t advect_scalar_adj_work_floats(const Grid& g) { return (size_t)18 * g.n3(); }

int launch_advect_scalar_adj(const Grid& g, const float* q, const float* ru, const float* rv, const float* rom,
                             const float* msftx, const float* fnm, const float* fnp, const float* rdnw,
                             const float* tbar, float* qbar, float* rubar, float* rvbar, float* rombar, float* work,
                             cudaStream_t st) {
  const dim3 b3(32, 4);
  AdvArgs0 a{q, ru, rv, rom, msftx, fnm, fnp, rdnw};
  k_advect_scalar_faces<<<point_grid(g, b3), b3, 0, st>>>(g, a, tbar, work, rubar, rvbar, rombar);
  k_advect_scalar_gather<<<point_grid(g, b3), b3, 0, st>>>(g, work, qbar);
  return 2;
}

}  // namespace wrf
