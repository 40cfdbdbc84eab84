// C ABI and the host-side step driver: the launch sequence of one ARW time
// step in the order of WrfSolver.solve (pywrf/solver.py:709-1910).
//
// The driver only enqueues kernels and memsets on the caller's stream; it
// allocates nothing and never synchronises (a probe callback may).  The
// boundary time of the step is derived on the device from the step counter
// STATUS[WRF_ST_STEP], so one captured CUDA graph replays every step.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <cctype>
#include <string>
#include "kernels.cuh"
#include "mlp.cuh"
#include "tc_gemm.cuh"

namespace wrf {
namespace {

thread_local std::string g_err;
thread_local int g_last_launches = 0;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int check_launch(const char* where) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(WRF_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
  return WRF_OK;
}

#define WRF_NAME_ENTRY(name, kind) #name,
const char* const kUpperNames[WF_COUNT] = {WRF_FIELD_TABLE(WRF_NAME_ENTRY)};
#undef WRF_NAME_ENTRY
#define WRF_KIND_ENTRY(name, kind) kind,
const int kKinds[WF_COUNT] = {WRF_FIELD_TABLE(WRF_KIND_ENTRY)};
#undef WRF_KIND_ENTRY

struct LowerNames {
  char buf[WF_COUNT][24];
  LowerNames() {
    for (int i = 0; i < WF_COUNT; ++i) {
      size_t n = strlen(kUpperNames[i]);
      if (n > 23) n = 23;
      for (size_t c = 0; c < n; ++c) buf[i][c] = (char)tolower((unsigned char)kUpperNames[i][c]);
      buf[i][n] = 0;
    }
  }
};
const LowerNames kLower;

int make_grid(const WrfGrid* in, Grid& g) {
  if (!in) return fail(WRF_EINVAL, "null grid");
  g.nx = in->nx; g.ny = in->ny; g.nz = in->nz;
  g.ids = in->ids; g.ide = in->ide; g.jds = in->jds; g.jde = in->jde;
  g.soundsteps = in->soundsteps; g.spec_zone = in->spec_zone; g.top_lid = in->top_lid;
  if (g.nz < 12 || g.nz > kMaxNz) return fail(WRF_EINVAL, "nz must lie in [12, 64]");
  if (g.ids != 5 || g.jds != 5 || g.ide != g.nx - 5 || g.jde != g.ny - 5)
    return fail(WRF_EINVAL, "the 5-cell frame needs ids = jds = 5, ide = nx - 5, jde = ny - 5");
  if (g.nx < 24 || g.ny < 24) return fail(WRF_EINVAL, "nx and ny must be at least 24");
  if (g.spec_zone != 1) return fail(WRF_EINVAL, "spec_zone must be 1 (relax zone 4, bdy width 5)");
  if (g.soundsteps < 2 || (g.soundsteps % 2) != 0) return fail(WRF_EINVAL, "soundsteps must be even and >= 2");
  if (in->kvdif != 0.0f) return fail(WRF_EINVAL, "kvdif != 0 (vertical diffusion) is not supported");
  if (in->bdy_interval < 1) return fail(WRF_EINVAL, "bdy_interval must be >= 1");
  if (!(in->dx > 0.f) || !(in->dy > 0.f) || !(in->dt > 0.f)) return fail(WRF_EINVAL, "dx, dy, dt must be > 0");
  g.dx = in->dx; g.dy = in->dy; g.dt = in->dt;
  g.dxd = in->dx; g.dyd = in->dy; g.dtd = in->dt;
  g.rdxd = 1.0 / g.dxd; g.rdyd = 1.0 / g.dyd;
  g.rdx = (float)g.rdxd; g.rdy = (float)g.rdyd;
  g.smdiv = in->smdiv; g.emdiv = in->emdiv; g.epssm = in->epssm;
  g.cf1 = in->cf1; g.cf2 = in->cf2; g.cf3 = in->cf3; g.cfn = in->cfn; g.cfn1 = in->cfn1;
  return WRF_OK;
}

int make_state(const WrfState* in, S& s) {
  if (!in) return fail(WRF_EINVAL, "null state");
  for (int i = 0; i < WF_COUNT; ++i) {
    s.f[i] = static_cast<float*>(in->f[i]);
    if (!s.f[i]) return fail(WRF_EINVAL, std::string("null field ") + kLower.buf[i]);
  }
  return WRF_OK;
}

// boundary time of this step from the device step counter (solver.py:713-718)
__global__ void k_step_begin(float* dscal, const int* status, int bdy_interval, double dt) {
  const int step = status[WRF_ST_STEP] + 1;
  const int it_bdy = bdy_interval > 1 ? (step - 1) / bdy_interval : 0;
  dscal[DS_DTBC] = (float)(dt * (double)(step - it_bdy * bdy_interval));
  dscal[DS_STEP] = (float)step;
}

__global__ void k_step_end(int* status) { status[WRF_ST_STEP] += 1; }

// zeroes a batch of fields in one launch (in place of one memset node per
// field in the captured step): blockIdx.y picks the field, the blocks of x
// stride over it with 16-byte stores
constexpr int kZeroMax = 16;
struct ZeroBatch {
  float* p[kZeroMax];
  unsigned long long n[kZeroMax];  // floats
  int count;
};
__global__ void __launch_bounds__(256) k_zero_batch(ZeroBatch b) {
  const int f = blockIdx.y;
  float* p = b.p[f];
  const unsigned long long n = b.n[f];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
    const unsigned long long n4 = n / 4;
    float4* q = reinterpret_cast<float4*>(p);
    for (unsigned long long e = t0; e < n4; e += stride) q[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (unsigned long long e = n4 * 4 + t0; e < n; e += stride) p[e] = 0.f;
  } else {
    for (unsigned long long e = t0; e < n; e += stride) p[e] = 0.f;
  }
}

struct Driver {
  Grid g;
  S s;
  cudaStream_t st;
  wrf_probe_fn probe;
  void* user;
  const MlpNetDev* net = nullptr;   // surrogate microphysics when set
  const MlpWorkDev* work = nullptr;
  int rc = WRF_OK;
  int n = 0;  // kernels enqueued


  bool ok(const char* where) {
    if (rc != WRF_OK) return false;
    rc = check_launch(where);
    return rc == WRF_OK;
  }
  // zero the listed fields (id, kind: 3 = [nz][ny][nx], 2 = [ny][nx], 4 = the 7 moisture slots) in one launch
  void zero(std::initializer_list<std::pair<int, int>> fields) {
    if (rc != WRF_OK) return;
    ZeroBatch b{};
    for (auto& e : fields) {
      b.p[b.count] = s[e.first];
      b.n[b.count] = e.second == 2 ? g.n2() : (e.second == 4 ? 7 * g.n3() : g.n3());
      ++b.count;
    }
    k_zero_batch<<<dim3(std::min<unsigned>(592u, (unsigned)((g.n3() / 4 + 255) / 256)), b.count), 256, 0, st>>>(b);
    ++n;
  }
  void phase(const char* name) {
    if (!ok(name)) return;
    if (probe) probe(name, user);
  }
  // halo copies of the listed 3-D and 2-D fields (and, with moist, of the
  // six moisture species) in as few launches as the batch allows
  void bc(std::initializer_list<std::pair<int, char>> f3, std::initializer_list<std::pair<int, char>> f2 = {},
          bool moist = false, bool zero_grad_w = false) {
    BcBatch b;
    auto add = [&](const BcItem& it) {
      if (b.n == kBcMax) {
        n += launch_bc(g, b, st);
        b.n = 0;
      }
      b.add(it);
    };
    for (auto& e : f3) add(bc_item(g, s[e.first], e.second, false));
    for (auto& e : f2) add(bc_item(g, s[e.first], e.second, true));
    if (moist)
      for (int m = 1; m < 7; ++m) add(bc_item(g, s[WF_MOIST] + m * g.n3(), 'p', false));
    if (zero_grad_w) b.zgw = s[WF_W];
    n += launch_bc(g, b, st);
  }

  // dt_rk, dts_rk and the substep count of RK stage rk (solver.py:722-735)
  void stage(int rk, float& dt_rk, float& dts_rk, int& nsub) const {
    const float dts = (float)(g.dtd / g.soundsteps);
    if (rk == 1) { dt_rk = (float)(g.dtd / 3.0); dts_rk = dt_rk; nsub = 1; }
    else if (rk == 2) { dt_rk = (float)(0.5 * g.dtd); dts_rk = dts; nsub = g.soundsteps / 2; }
    else { dt_rk = g.dt; dts_rk = dts; nsub = g.soundsteps; }
  }

  // boundary time of the step from the device step counter (solver.py:713)
  void step_begin() {
    if (rc != WRF_OK) return;
    k_step_begin<<<1, 1, 0, st>>>(s[WF_DSCAL], reinterpret_cast<const int*>(s[WF_STATUS]), bdy_interval, g.dtd);
    ++n;
    ok("step_begin");
  }
  // rk_step_prep (solver.py:736-778)
  void rk_prep(int rk) {
    if (rc != WRF_OK) return;
    char tag[32];
    n += launch_prep(g, s, st);
    bc({{WF_RU, 'u'}, {WF_RV, 'v'}, {WF_RW, 'w'}, {WF_WW, 'w'}, {WF_PHP, 'w'}, {WF_ALT, 't'}, {WF_P, 'p'},
        {WF_AL, 'p'}, {WF_PH, 'w'}},
       {{WF_MUU, 'u'}, {WF_MUV, 'v'}, {WF_MUT, 't'}});
    snprintf(tag, sizeof tag, "s%d.prep", rk);
    phase(tag);
  }
  // first stage: physics tendencies start from zero; diffusion metrics and
  // eddy viscosities (solver.py:880-985)
  void diff_stage1() {
    if (rc != WRF_OK) return;
    zero({{WF_RU_TENDF, 3}, {WF_RV_TENDF, 3}, {WF_RW_TENDF, 3}, {WF_PH_TENDF, 3}, {WF_T_TENDF, 3}, {WF_MU_TENDF, 2},
          {WF_MOIST_TEND, 4}});
    n += launch_diff_metrics(g, s, st);
    bc({{WF_RDZW, 'w'}, {WF_ZX, 'e'}, {WF_ZY, 'f'}});
    n += launch_km(g, s, st);
    bc({{WF_XKMH, 't'}, {WF_XKHH, 't'}});
    phase("s1.km");
  }
  // large-step tendencies: advection and forces, first-stage diffusion and
  // relaxation, rk_addtend_dry (solver.py:987-1256)
  void tend_stage(int rk) {
    if (rc != WRF_OK) return;
    char tag[32];
    zero({{WF_RU_TEND, 3}, {WF_RV_TEND, 3}, {WF_RW_TEND, 3}, {WF_T_TEND, 3}, {WF_PH_TEND, 3}, {WF_U_SAVE, 3},
          {WF_V_SAVE, 3}, {WF_W_SAVE, 3}, {WF_PH_SAVE, 3}, {WF_T_SAVE, 3}, {WF_MU_TEND, 2}, {WF_MU_SAVE, 2}});
    n += launch_advect_forces(g, s, st);
    snprintf(tag, sizeof tag, "s%d.forces", rk);
    phase(tag);
    if (rk == 1) {
      n += launch_hdiff_relax(g, s, st);
      phase("s1.diff");
    }
    n += launch_addtend(g, s, rk, st);
    snprintf(tag, sizeof tag, "s%d.tend", rk);
    phase(tag);
  }
  // acoustic set-up (solver.py:1258-1345)
  void acoustic_prep(int rk) {
    if (rc != WRF_OK) return;
    char tag[32];
    float dt_rk, dts_rk;
    int nsub;
    stage(rk, dt_rk, dts_rk, nsub);
    n += launch_small_step_prep(g, s, rk, dts_rk, st);
    bc({{WF_RU_TEND, 'u'}, {WF_RV_TEND, 'v'}, {WF_PH, 'w'}, {WF_AL, 'p'}, {WF_P, 'p'}, {WF_T_1, 't'},
        {WF_T_SAVE, 't'}},
       {{WF_MU_1, 't'}, {WF_MU, 't'}, {WF_MUDF, 't'}});
    snprintf(tag, sizeof tag, "s%d.acprep", rk);
    phase(tag);
  }
  // one acoustic substep: advance_uv, then the column update (mu/theta,
  // w/phi, sumflux, p/al), then zero_grad_bdy(w) and the halo copies
  // (solver.py:1350-1492)
  void acoustic_substep(int rk, int it) {
    if (rc != WRF_OK) return;
    char tag[32];
    float dt_rk, dts_rk;
    int nsub;
    stage(rk, dt_rk, dts_rk, nsub);
    n += launch_advance_uv(g, s, dts_rk, st);
    snprintf(tag, sizeof tag, "s%d.sub%d.uv", rk, it);
    phase(tag);
    n += launch_acoustic_col(g, s, dts_rk, it, nsub, st);
    snprintf(tag, sizeof tag, "s%d.sub%d.col", rk, it);
    phase(tag);
    // zero_grad_bdy(w) rides in the halo launch (disjoint fields)
    bc({{WF_PH, 'w'}, {WF_AL, 'p'}, {WF_P, 'p'}}, {{WF_MUTS, 't'}, {WF_MU, 't'}, {WF_MUDF, 't'}}, false, true);
    snprintf(tag, sizeof tag, "s%d.sub%d", rk, it);
    phase(tag);
  }
  // small_step_finish (solver.py:1494-1546)
  void acoustic_finish(int rk) {
    if (rc != WRF_OK) return;
    char tag[32];
    float dt_rk, dts_rk;
    int nsub;
    stage(rk, dt_rk, dts_rk, nsub);
    n += launch_small_step_finish(g, s, dts_rk, nsub, rk, st);
    if (rk == 3) bc({{WF_RU_M, 'u'}, {WF_RV_M, 'v'}, {WF_WW_M, 'w'}}, {{WF_MUT, 't'}, {WF_MUTS, 't'}});
    snprintf(tag, sizeof tag, "s%d.acfinish", rk);
    phase(tag);
  }
  // moisture transport and the stage's halo copies (solver.py:1548-1710)
  void moist_stage(int rk) {
    if (rc != WRF_OK) return;
    char tag[32];
    float dt_rk, dts_rk;
    int nsub;
    stage(rk, dt_rk, dts_rk, nsub);
    n += launch_advect_moist(g, s, st);
    if (rk == 1) {
      n += launch_hdiff_moist(g, s, st);
      n += launch_relax_qv(g, s, st);
    }
    n += launch_moist(g, s, rk, dt_rk, st);
    if (rk < 3) {
      bc({{WF_U, 'U'}, {WF_V, 'V'}, {WF_W, 'w'}, {WF_T, 'p'}, {WF_PH, 'w'}}, {{WF_MU, 't'}}, true);
    }
    snprintf(tag, sizeof tag, "s%d.moist", rk);
    phase(tag);
  }
  // microphysics (solver.py:1714-1766), or its learned stand-in
  void microphysics() {
    if (rc != WRF_OK) return;
    if (net) {
      const char* err = nullptr;
      const int r = launch_physics_mlp(g, s, *net, *work, st, &err);
      if (r < 0) {
        rc = fail(r, err ? err : "surrogate microphysics failed");
        return;
      }
      n += r;
    } else {
      n += launch_physics(g, s, st);
    }
    phase("mp");
  }
  // end-of-step boundaries and the step counter (solver.py:1776-1910)
  void step_end() {
    if (rc != WRF_OK) return;
    bc({{WF_U_1, 'U'}, {WF_U, 'U'}, {WF_V_1, 'V'}, {WF_V, 'V'}, {WF_W_1, 'w'}, {WF_W, 'w'}, {WF_T_1, 'p'},
        {WF_T, 'p'}, {WF_PH_1, 'w'}, {WF_PH, 'w'}},
       {{WF_MU_1, 't'}, {WF_MU, 't'}}, true);
    n += launch_bdy_final(g, s, st);
    k_step_end<<<1, 1, 0, st>>>(reinterpret_cast<int*>(s[WF_STATUS]));
    ++n;
    phase("end");
  }

  void run() {
    step_begin();
    for (int rk = 1; rk <= 3; ++rk) {
      float dt_rk, dts_rk;
      int nsub;
      stage(rk, dt_rk, dts_rk, nsub);
      rk_prep(rk);
      if (rk == 1) diff_stage1();
      tend_stage(rk);
      acoustic_prep(rk);
      for (int it = 1; it <= nsub; ++it) acoustic_substep(rk, it);
      acoustic_finish(rk);
      moist_stage(rk);
    }
    microphysics();
    step_end();
  }
  int bdy_interval = 360;
};

}  // namespace
}  // namespace wrf

using namespace wrf;

namespace wrf {
namespace {
std::atomic<int> g_form{WRF_FORM_FAST};
}
int kernel_form() { return g_form.load(std::memory_order_relaxed); }
int set_kernel_form(int form) { return g_form.exchange(form); }
}  // namespace wrf

extern "C" {

int wrf_field_count(void) { return WF_COUNT; }

const char* wrf_field_name(int id) {
  if (id < 0 || id >= WF_COUNT) return nullptr;
  return kLower.buf[id];
}

int wrf_field_kind(int id) {
  if (id < 0 || id >= WF_COUNT) return WRF_EINVAL;
  return kKinds[id];
}

const char* wrf_last_error(void) { return g_err.c_str(); }

int wrf_last_launch_count(void) { return g_last_launches; }

int wrf_set_kernel_form(int form) {
  if (form != WRF_FORM_FAST && form != WRF_FORM_POINT) return fail(WRF_EINVAL, "unknown kernel form");
  return wrf::set_kernel_form(form);
}

int wrf_rk3_step(const WrfGrid* gin, const WrfState* sin, void* stream, wrf_probe_fn probe, void* user) {
  Driver d;
  int rc = make_grid(gin, d.g);
  if (rc) return rc;
  rc = make_state(sin, d.s);
  if (rc) return rc;
  d.st = static_cast<cudaStream_t>(stream);
  d.probe = probe;
  d.user = user;
  d.bdy_interval = gin->bdy_interval;
  cudaGetLastError();  // clear a stale error from an unrelated earlier call
  d.run();
  g_last_launches = d.n;
  return d.rc;
}

}  // extern "C"

namespace {
// one phase of the step on a fresh driver (no probe)
template <typename F>
int run_phase(const WrfGrid* gin, const WrfState* sin, void* stream, int rk, int it, F body) {
  Driver d;
  int rc = make_grid(gin, d.g);
  if (rc) return rc;
  rc = make_state(sin, d.s);
  if (rc) return rc;
  if (rk != 0) {
    if (rk < 1 || rk > 3) return fail(WRF_EINVAL, "rk_step must be 1, 2 or 3");
    float dt_rk, dts_rk;
    int nsub;
    d.stage(rk, dt_rk, dts_rk, nsub);
    if (it != 0 && (it < 1 || it > nsub)) return fail(WRF_EINVAL, "acoustic iteration outside 1 .. substeps of the stage");
  }
  d.st = static_cast<cudaStream_t>(stream);
  d.probe = nullptr;
  d.user = nullptr;
  d.bdy_interval = gin->bdy_interval;
  cudaGetLastError();
  body(d);
  g_last_launches = d.n;
  return d.rc;
}
}  // namespace

extern "C" {

int wrf_step_begin(const WrfGrid* g, const WrfState* s, void* stream) {
  return run_phase(g, s, stream, 0, 0, [](Driver& d) { d.step_begin(); });
}
int wrf_rk_prep(const WrfGrid* g, const WrfState* s, int rk_step, void* stream) {
  return run_phase(g, s, stream, rk_step, 0, [&](Driver& d) { d.rk_prep(rk_step); });
}
int wrf_diff_stage1(const WrfGrid* g, const WrfState* s, void* stream) {
  return run_phase(g, s, stream, 0, 0, [](Driver& d) { d.diff_stage1(); });
}
int wrf_tend_stage(const WrfGrid* g, const WrfState* s, int rk_step, void* stream) {
  return run_phase(g, s, stream, rk_step, 0, [&](Driver& d) { d.tend_stage(rk_step); });
}
int wrf_acoustic_prep(const WrfGrid* g, const WrfState* s, int rk_step, void* stream) {
  return run_phase(g, s, stream, rk_step, 0, [&](Driver& d) { d.acoustic_prep(rk_step); });
}
int wrf_acoustic_substep(const WrfGrid* g, const WrfState* s, int rk_step, int iteration, void* stream) {
  if (iteration < 1) return fail(WRF_EINVAL, "acoustic iteration outside 1 .. substeps of the stage");
  return run_phase(g, s, stream, rk_step, iteration, [&](Driver& d) { d.acoustic_substep(rk_step, iteration); });
}
int wrf_acoustic_finish(const WrfGrid* g, const WrfState* s, int rk_step, void* stream) {
  return run_phase(g, s, stream, rk_step, 0, [&](Driver& d) { d.acoustic_finish(rk_step); });
}
int wrf_moist_stage(const WrfGrid* g, const WrfState* s, int rk_step, void* stream) {
  return run_phase(g, s, stream, rk_step, 0, [&](Driver& d) { d.moist_stage(rk_step); });
}
int wrf_microphysics(const WrfGrid* g, const WrfState* s, void* stream) {
  return run_phase(g, s, stream, 0, 0, [](Driver& d) { d.microphysics(); });
}
int wrf_step_end(const WrfGrid* g, const WrfState* s, void* stream) {
  return run_phase(g, s, stream, 0, 0, [](Driver& d) { d.step_end(); });
}

int wrf_advect_scalar(const WrfGrid* gin, const float* field, float* tend, const float* ru, const float* rv,
                      const float* rom, const float* msftx, const float* fzm, const float* fzp, const float* rdzw,
                      void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !tend || !ru || !rv || !rom || !msftx || !fzm || !fzp || !rdzw)
    return fail(WRF_EINVAL, "null argument");
  S s{};
  s.f[WF_MSFTX] = const_cast<float*>(msftx);
  s.f[WF_FNM] = const_cast<float*>(fzm);
  s.f[WF_FNP] = const_cast<float*>(fzp);
  s.f[WF_RDNW] = const_cast<float*>(rdzw);
  cudaGetLastError();
  launch_advect_scalar(g, s, field, tend, ru, rv, rom, static_cast<cudaStream_t>(stream));
  return check_launch("advect_scalar");
}

int wrf_advect_momentum(const WrfGrid* gin, int component, const float* field, float* tend, const float* ru,
                        const float* rv, const float* rom, const float* msf, const float* msf2, const float* fzm,
                        const float* fzp, const float* rdz, int form, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (component < 0 || component > 2 || (form != 0 && form != 1))
    return fail(WRF_EINVAL, "advect_momentum: component 0..2, form 0 or 1");
  if (!field || !tend || !ru || !rv || !rom || !msf || (component == 1 && !msf2) || !fzm || !fzp || !rdz)
    return fail(WRF_EINVAL, "null argument");
  S s{};
  const int fld[3] = {WF_U, WF_V, WF_W}, tnd[3] = {WF_RU_TEND, WF_RV_TEND, WF_RW_TEND};
  s.f[fld[component]] = const_cast<float*>(field);
  s.f[tnd[component]] = tend;
  s.f[WF_RU] = const_cast<float*>(ru);
  s.f[WF_RV] = const_cast<float*>(rv);
  s.f[WF_WW] = const_cast<float*>(rom);
  if (component == 0) s.f[WF_MSFUX] = const_cast<float*>(msf);
  if (component == 1) {
    s.f[WF_MSFVY] = const_cast<float*>(msf);
    s.f[WF_MSFVX] = const_cast<float*>(msf2);
  }
  if (component == 2) s.f[WF_MSFTX] = const_cast<float*>(msf);
  s.f[WF_FNM] = const_cast<float*>(fzm);
  s.f[WF_FNP] = const_cast<float*>(fzp);
  s.f[component == 2 ? WF_RDN : WF_RDNW] = const_cast<float*>(rdz);
  cudaGetLastError();
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (form == 1 || launch_advect_mom_tma(g, s, component, 1, st) == 0) launch_advect_mom_point(g, s, 1 << component, st);
  return check_launch("advect_momentum");
}

int wrf_advect_scalar_adj(const WrfGrid* gin, const float* field, const float* ru, const float* rv, const float* rom,
                          const float* msftx, const float* fzm, const float* fzp, const float* rdzw,
                          const float* tend_bar, float* field_bar, float* ru_bar, float* rv_bar, float* rom_bar,
                          float* work, size_t work_floats, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !ru || !rv || !rom || !msftx || !fzm || !fzp || !rdzw || !tend_bar || !field_bar || !ru_bar ||
      !rv_bar || !rom_bar || !work)
    return fail(WRF_EINVAL, "null argument");
  if (work_floats < advect_scalar_adj_work_floats(g))
    return fail(WRF_EINVAL, "advect_scalar_adj: work smaller than wrf_advect_scalar_adj_work gives");
  cudaGetLastError();
  launch_advect_scalar_adj(g, field, ru, rv, rom, msftx, fzm, fzp, rdzw, tend_bar, field_bar, ru_bar, rv_bar, rom_bar,
                           work, static_cast<cudaStream_t>(stream));
  return check_launch("advect_scalar_adj");
}

int wrf_advect_scalar_adj_work(const WrfGrid* gin, size_t* floats) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!floats) return fail(WRF_EINVAL, "null argument");
  *floats = advect_scalar_adj_work_floats(g);
  return WRF_OK;
}

namespace {
// the forward operands of advance_uv in the state table
constexpr int kUvOperands[] = {WF_U, WF_V, WF_RU_TEND, WF_RV_TEND, WF_P, WF_PB, WF_PH, WF_PHP, WF_ALT, WF_AL, WF_MU,
                               WF_MUU, WF_MUV, WF_CQU, WF_CQV, WF_MUDF, WF_MSFUX, WF_MSFUY, WF_MSFVX, WF_MSFVX_INV,
                               WF_MSFVY, WF_FNM, WF_FNP, WF_RDNW};
// the cotangents it reads (U, V) and accumulates
constexpr int kUvCotangents[] = {WF_U, WF_V, WF_RU_TEND, WF_RV_TEND, WF_P, WF_PB, WF_PH, WF_PHP, WF_ALT, WF_AL,
                                 WF_MU, WF_MUU, WF_MUV, WF_CQU, WF_CQV, WF_MUDF};

// the tendency terms' operands (rhs_ph, horizontal_pressure_gradient,
// pg_buoy_w, coriolis, curvature) and the cotangents their adjoint reads or
// accumulates
constexpr int kForcesOperands[] = {WF_PH_TEND, WF_RU_TEND, WF_RV_TEND, WF_RW_TEND, WF_CQW, WF_U, WF_V, WF_W, WF_WW,
                                   WF_PH, WF_PHB, WF_MUT, WF_MUU, WF_MUV, WF_ALT, WF_P, WF_PB, WF_AL, WF_PHP, WF_CQU,
                                   WF_CQV, WF_MU, WF_MUB, WF_RU, WF_RV, WF_RW, WF_MSFUX, WF_MSFUY, WF_MSFVX, WF_MSFVY,
                                   WF_MSFTX, WF_MSFTY, WF_F, WF_E, WF_SINA, WF_COSA, WF_FNM, WF_FNP, WF_RDNW, WF_RDN};
constexpr int kForcesCotangents[] = {WF_PH_TEND, WF_RU_TEND, WF_RV_TEND, WF_RW_TEND, WF_CQW, WF_U, WF_V, WF_W,
                                     WF_WW, WF_PH, WF_PHB, WF_MUT, WF_MUU, WF_MUV, WF_ALT, WF_P, WF_PB, WF_AL,
                                     WF_PHP, WF_CQU, WF_CQV, WF_MU, WF_MUB, WF_RU, WF_RV, WF_RW};

// sumflux and spec_bdyupdate_ph operands and cotangents
constexpr int kSumfluxOperands[] = {WF_U, WF_V, WF_WW, WF_U_SAVE, WF_V_SAVE, WF_WW1, WF_MUU, WF_MUV, WF_RU_M,
                                    WF_RV_M, WF_WW_M, WF_MSFUY, WF_MSFVX_INV};
constexpr int kSumfluxCotangents[] = {WF_U, WF_V, WF_WW, WF_U_SAVE, WF_V_SAVE, WF_WW1, WF_MUU, WF_MUV, WF_RU_M,
                                      WF_RV_M, WF_WW_M};
constexpr int kSpecPhOperands[] = {WF_PH, WF_PH_SAVE, WF_PH_TEND, WF_MU_TEND, WF_MUTS};

// rk_step_prep's operands and the cotangents its adjoint reads or accumulates
constexpr int kPrepOperands[] = {WF_MU, WF_MUB, WF_MUT, WF_MUU, WF_MUV, WF_U, WF_V, WF_W, WF_RU, WF_RV, WF_RW,
                                 WF_WW, WF_MOIST, WF_CQU, WF_CQV, WF_CQW, WF_AL, WF_ALB, WF_ALT, WF_PH, WF_PHB,
                                 WF_PHP, WF_MSFU, WF_MSFVX_INV, WF_MSFT, WF_MSFTX, WF_MSFUY, WF_DNW, WF_C1H};
constexpr int kPrepCotangents[] = {WF_MU, WF_MUB, WF_MUT, WF_MUU, WF_MUV, WF_U, WF_V, WF_W, WF_RU, WF_RV, WF_RW,
                                   WF_WW, WF_MOIST, WF_CQU, WF_CQV, WF_CQW, WF_AL, WF_ALB, WF_ALT, WF_PH, WF_PHB,
                                   WF_PHP};

// small_step_prep and calc_mu_uv_1 + small_step_finish operands and cotangents
constexpr int kSspOperands[] = {WF_MU, WF_MU_1, WF_MUB, WF_MUDF, WF_MUTS, WF_MU_SAVE, WF_MUU, WF_MUV, WF_MUUS,
                                WF_MUVS, WF_MUT, WF_U, WF_U_1, WF_U_SAVE, WF_V, WF_V_1, WF_V_SAVE, WF_T, WF_T_1,
                                WF_T_SAVE, WF_W, WF_W_1, WF_W_SAVE, WF_PH, WF_PH_1, WF_PH_SAVE, WF_WW, WF_WW1,
                                WF_C2A, WF_PB, WF_P, WF_ALT, WF_MSFUY, WF_MSFVX_INV, WF_MSFTY};
constexpr int kSspCotangents[] = {WF_MU, WF_MU_1, WF_MUB, WF_MUDF, WF_MUTS, WF_MU_SAVE, WF_MUU, WF_MUV, WF_MUUS,
                                  WF_MUVS, WF_MUT, WF_U, WF_U_1, WF_U_SAVE, WF_V, WF_V_1, WF_V_SAVE, WF_T, WF_T_1,
                                  WF_T_SAVE, WF_W, WF_W_1, WF_W_SAVE, WF_PH, WF_PH_1, WF_PH_SAVE, WF_WW, WF_WW1,
                                  WF_C2A, WF_PB, WF_P, WF_ALT};
constexpr int kSsfOperands[] = {WF_U, WF_U_SAVE, WF_V, WF_V_SAVE, WF_W, WF_W_SAVE, WF_PH, WF_PH_SAVE, WF_WW, WF_WW1,
                                WF_T, WF_T_SAVE, WF_H_DIABATIC, WF_MU, WF_MU_SAVE, WF_MUT, WF_MUTS, WF_MUU, WF_MUV,
                                WF_MUUS, WF_MUVS, WF_MSFUY, WF_MSFVX, WF_MSFTY};
constexpr int kSsfCotangents[] = {WF_U, WF_U_SAVE, WF_V, WF_V_SAVE, WF_W, WF_W_SAVE, WF_PH, WF_PH_SAVE, WF_WW, WF_WW1,
                                  WF_T, WF_T_SAVE, WF_H_DIABATIC, WF_MU, WF_MU_SAVE, WF_MUT, WF_MUTS, WF_MUU, WF_MUV,
                                  WF_MUUS, WF_MUVS};

// the eddy viscosities' operands (metrics, deformations, calculate_km_kh;
// rdzw, zx, zy and the defor fields are scratch) and cotangents
constexpr int kKmOperands[] = {WF_U, WF_V, WF_PH, WF_PHB, WF_XKMH, WF_XKHH, WF_RDZW, WF_ZX, WF_ZY, WF_DEFOR11,
                               WF_DEFOR22, WF_DEFOR12, WF_MSFUX, WF_MSFUY, WF_MSFVX, WF_MSFVY, WF_MSFTX, WF_MSFTY,
                               WF_FNM, WF_FNP, WF_DN, WF_DNW};
constexpr int kKmCotangents[] = {WF_U, WF_V, WF_PH, WF_XKMH, WF_XKHH};
// horizontal_diffusion's map factors
constexpr int kHdiffOperands[] = {WF_MSFUX, WF_MSFUY, WF_MSFVX, WF_MSFVY, WF_MSFTX, WF_MSFTY, WF_MSFVX_INV};

// the end-of-step boundaries' operands (spec_bdy_final of u, v, t, ph, qv;
// set_w_surface) and cotangents
constexpr int kBdyFinalOperands[] = {
    WF_U, WF_V, WF_T, WF_PH, WF_MOIST, WF_W, WF_MUUS, WF_MUVS, WF_MUTS, WF_MSFUY, WF_MSFVX, WF_MSFTX, WF_MSFTY,
    WF_HT, WF_DSCAL, WF_U_BXS, WF_U_BXS + 1, WF_U_BXS + 2, WF_U_BXS + 3, WF_U_BXS + 4, WF_U_BXS + 5, WF_U_BXS + 6,
    WF_U_BXS + 7, WF_V_BXS, WF_V_BXS + 1, WF_V_BXS + 2, WF_V_BXS + 3, WF_V_BXS + 4, WF_V_BXS + 5, WF_V_BXS + 6,
    WF_V_BXS + 7, WF_T_BXS, WF_T_BXS + 1, WF_T_BXS + 2, WF_T_BXS + 3, WF_T_BXS + 4, WF_T_BXS + 5, WF_T_BXS + 6,
    WF_T_BXS + 7, WF_PH_BXS, WF_PH_BXS + 1, WF_PH_BXS + 2, WF_PH_BXS + 3, WF_PH_BXS + 4, WF_PH_BXS + 5,
    WF_PH_BXS + 6, WF_PH_BXS + 7, WF_QV_BXS, WF_QV_BXS + 1, WF_QV_BXS + 2, WF_QV_BXS + 3, WF_QV_BXS + 4,
    WF_QV_BXS + 5, WF_QV_BXS + 6, WF_QV_BXS + 7};
constexpr int kBdyFinalCotangents[] = {WF_U, WF_V, WF_T, WF_PH, WF_MOIST, WF_W, WF_MUUS, WF_MUVS, WF_MUTS};

// the microphysics block's operands (moist_physics_prep_em, WSM6,
// moist_physics_finish_em, calc_p_rho_phi), those its reverse reads, and
// the cotangents
constexpr int kMpOperands[] = {WF_T, WF_MOIST, WF_AL, WF_ALB, WF_P, WF_PB, WF_PH, WF_PHB, WF_MU, WF_MUTS, WF_RDNW,
                               WF_H_DIABATIC, WF_QV_DIABATIC, WF_QC_DIABATIC, WF_RAINNC, WF_RAINNCV, WF_SNOWNC,
                               WF_SNOWNCV, WF_GRAUPELNC, WF_GRAUPELNCV, WF_SR, WF_WSM_T, WF_WSM_QR0S};
constexpr int kMpAdjOperands[] = {WF_T, WF_MOIST, WF_AL, WF_ALB, WF_P, WF_PB, WF_PH, WF_PHB, WF_MU, WF_MUTS, WF_RDNW};
constexpr int kMpCotangents[] = {WF_T, WF_MOIST, WF_AL, WF_ALB, WF_P, WF_PB, WF_PH, WF_MU, WF_MUTS, WF_H_DIABATIC};

// calc_p_rho_phi's operands
constexpr int kEosOperands[] = {WF_AL, WF_ALB, WF_MU, WF_MUTS, WF_PH, WF_P, WF_PB, WF_T, WF_MOIST, WF_RDNW,
                                WF_STATUS};

// rk_addtend_dry's operands and cotangents
constexpr int kAddtendOperands[] = {WF_RU_TEND, WF_RV_TEND, WF_RW_TEND, WF_PH_TEND, WF_T_TEND, WF_MU_TEND,
                                    WF_RU_TENDF, WF_RV_TENDF, WF_RW_TENDF, WF_PH_TENDF, WF_T_TENDF, WF_MU_TENDF,
                                    WF_U_SAVE, WF_V_SAVE, WF_W_SAVE, WF_PH_SAVE, WF_T_SAVE, WF_H_DIABATIC, WF_MUT,
                                    WF_MSFTY, WF_MSFUY, WF_MSFVX, WF_MSFVX_INV};
constexpr int kAddtendCotangents[] = {WF_RU_TEND, WF_RV_TEND, WF_RW_TEND, WF_PH_TEND, WF_T_TEND, WF_MU_TEND,
                                      WF_RU_TENDF, WF_RV_TENDF, WF_RW_TENDF, WF_PH_TENDF, WF_T_TENDF, WF_MU_TENDF,
                                      WF_U_SAVE, WF_V_SAVE, WF_W_SAVE, WF_PH_SAVE, WF_T_SAVE, WF_H_DIABATIC, WF_MUT};

// the moisture update's operands (rk_update_scalar, flow_dep_bdy,
// calc_p_rho_phi) and cotangents
constexpr int kMoistOperands[] = {WF_MOIST, WF_MOIST_OLD, WF_MOIST_TEND, WF_ADVECT_TEND, WF_MU, WF_MU_1, WF_MUB,
                                  WF_MSFTY, WF_RU_M, WF_RV_M, WF_AL, WF_ALB, WF_MUTS, WF_PH, WF_P, WF_PB, WF_T,
                                  WF_RDNW, WF_STATUS};
constexpr int kMoistCotangents[] = {WF_MOIST, WF_MOIST_OLD, WF_MOIST_TEND, WF_ADVECT_TEND, WF_MU, WF_MU_1, WF_MUB,
                                    WF_AL, WF_ALB, WF_MUTS, WF_PH, WF_P, WF_PB, WF_T};

int state_of(const WrfState* in, const int* ids, int n, S& s) {
  if (!in) return fail(WRF_EINVAL, "null state");
  s = S{};
  for (int q = 0; q < WF_COUNT; ++q) s.f[q] = static_cast<float*>(in->f[q]);
  for (int e = 0; e < n; ++e)
    if (!s.f[ids[e]]) return fail(WRF_EINVAL, "a field the operator needs is null");
  return 0;
}
}  // namespace

namespace {
constexpr int kPrhoOperands[] = {WF_AL, WF_P, WF_PH, WF_ALT, WF_T, WF_T_SAVE, WF_C2A, WF_PM1, WF_MU, WF_MUTS, WF_RDNW};
constexpr int kPrhoCotangents[] = {WF_AL, WF_P, WF_PH, WF_ALT, WF_T, WF_T_SAVE, WF_C2A, WF_PM1, WF_MU, WF_MUTS};
}  // namespace

namespace {
constexpr int kMutOperands[] = {WF_WW, WF_WW1, WF_U, WF_U_SAVE, WF_V, WF_V_SAVE, WF_MU, WF_MUT, WF_MUAVE, WF_MUTS,
                                WF_MUU, WF_MUV, WF_MUDF, WF_T, WF_T_SAVE, WF_T_2SAVE, WF_T_TEND, WF_MU_TEND,
                                WF_DNW, WF_FNM, WF_FNP, WF_RDNW, WF_MSFUY, WF_MSFVX_INV, WF_MSFTX, WF_MSFTY};
constexpr int kMutCotangents[] = {WF_WW, WF_WW1, WF_U, WF_U_SAVE, WF_V, WF_V_SAVE, WF_MU, WF_MUT, WF_MUAVE,
                                  WF_MUTS, WF_MUU, WF_MUV, WF_MUDF, WF_T, WF_T_SAVE, WF_T_2SAVE, WF_T_TEND,
                                  WF_MU_TEND};
}  // namespace

namespace {
constexpr int kAwCotangents[] = {WF_W, WF_RW_TEND, WF_WW, WF_W_SAVE, WF_U, WF_V, WF_MUAVE, WF_MUTS, WF_MUT,
                                 WF_T_2SAVE, WF_T, WF_T_SAVE, WF_PH, WF_PH_SAVE, WF_PHB, WF_PH_TEND, WF_HT, WF_C2A,
                                 WF_CQW, WF_ALT, WF_A, WF_ALPHA, WF_GAMMA};
constexpr int kAwOperands[] = {WF_W, WF_RW_TEND, WF_WW, WF_W_SAVE, WF_U, WF_V, WF_MUAVE, WF_MUTS, WF_MUT,
                               WF_T_2SAVE, WF_T, WF_T_SAVE, WF_PH, WF_PH_SAVE, WF_PHB, WF_PH_TEND, WF_HT, WF_C2A,
                               WF_CQW, WF_ALT, WF_A, WF_ALPHA, WF_GAMMA, WF_MSFTX, WF_MSFTY, WF_FNM, WF_FNP,
                               WF_RDNW, WF_RDN};
}  // namespace

int wrf_advance_w(const WrfGrid* gin, const WrfState* sin, float dts, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kAwOperands, sizeof(kAwOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_advance_w(g, s, dts, static_cast<cudaStream_t>(stream));
  return check_launch("advance_w");
}

int wrf_advance_w_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float dts, float* work,
                      void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!work) return fail(WRF_EINVAL, "advance_w_adj: null work array");
  S s, b;
  if ((rc = state_of(sin, kAwOperands, sizeof(kAwOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kAwCotangents, sizeof(kAwCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_advance_w_adj(g, s, b, dts, work, static_cast<cudaStream_t>(stream));
  return check_launch("advance_w_adj");
}

int wrf_advance_mu_t(const WrfGrid* gin, const WrfState* sin, float dts, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kMutOperands, sizeof(kMutOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_advance_mu_t(g, s, dts, static_cast<cudaStream_t>(stream));
  return check_launch("advance_mu_t");
}

int wrf_advance_mu_t_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float dts, int ref_no_grad,
                         float* work, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!work) return fail(WRF_EINVAL, "advance_mu_t_adj: null work array");
  S s, b;
  if ((rc = state_of(sin, kMutOperands, sizeof(kMutOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kMutCotangents, sizeof(kMutCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_advance_mu_t_adj(g, s, b, dts, ref_no_grad ? 1 : 0, work, static_cast<cudaStream_t>(stream));
  return check_launch("advance_mu_t_adj");
}

int wrf_calc_p_rho(const WrfGrid* gin, const WrfState* sin, int step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (step < 0) return fail(WRF_EINVAL, "calc_p_rho: step >= 0");
  S s;
  if ((rc = state_of(sin, kPrhoOperands, sizeof(kPrhoOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_calc_p_rho(g, s, step, static_cast<cudaStream_t>(stream));
  return check_launch("calc_p_rho");
}

int wrf_calc_p_rho_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (step < 0) return fail(WRF_EINVAL, "calc_p_rho_adj: step >= 0");
  S s, b;
  if ((rc = state_of(sin, kPrhoOperands, sizeof(kPrhoOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kPrhoCotangents, sizeof(kPrhoCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_calc_p_rho_adj(g, s, b, step, static_cast<cudaStream_t>(stream));
  return check_launch("calc_p_rho_adj");
}

int wrf_advance_uv(const WrfGrid* gin, const WrfState* sin, float dts, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kUvOperands, sizeof(kUvOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_advance_uv(g, s, dts, static_cast<cudaStream_t>(stream));
  return check_launch("advance_uv");
}

int wrf_forces(const WrfGrid* gin, const WrfState* sin, int terms, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (terms < 1 || terms > 31) return fail(WRF_EINVAL, "forces: terms is a mask of 1 .. 31");
  S s;
  if ((rc = state_of(sin, kForcesOperands, sizeof(kForcesOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_forces_terms(g, s, terms, static_cast<cudaStream_t>(stream));
  return check_launch("forces");
}

int wrf_forces_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int terms, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (terms < 1 || terms > 31) return fail(WRF_EINVAL, "forces_adj: terms is a mask of 1 .. 31");
  S s, b;
  if ((rc = state_of(sin, kForcesOperands, sizeof(kForcesOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kForcesCotangents, sizeof(kForcesCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_forces_adj(g, s, b, terms, static_cast<cudaStream_t>(stream));
  return check_launch("forces_adj");
}

int wrf_sumflux(const WrfGrid* gin, const WrfState* sin, int iteration, int nsub, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (nsub < 1 || iteration < 1 || iteration > nsub) return fail(WRF_EINVAL, "sumflux: needs 1 <= iteration <= nsub");
  S s;
  if ((rc = state_of(sin, kSumfluxOperands, sizeof(kSumfluxOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_sumflux(g, s, iteration, nsub, static_cast<cudaStream_t>(stream));
  return check_launch("sumflux");
}

int wrf_sumflux_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int iteration, int nsub,
                    void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (nsub < 1 || iteration < 1 || iteration > nsub) return fail(WRF_EINVAL, "sumflux_adj: needs 1 <= iteration <= nsub");
  S s, b;
  if ((rc = state_of(sin, kSumfluxOperands, sizeof(kSumfluxOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kSumfluxCotangents, sizeof(kSumfluxCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_sumflux_adj(g, s, b, iteration, nsub, static_cast<cudaStream_t>(stream));
  return check_launch("sumflux_adj");
}

int wrf_spec_bdyupdate(const WrfGrid* gin, float* field, const float* tend, float dt, char var, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !tend) return fail(WRF_EINVAL, "null argument");
  if (var != 't' && var != 'u' && var != 'v' && var != 'm') return fail(WRF_EINVAL, "spec_bdyupdate: var is t, u, v or m");
  cudaGetLastError();
  launch_spec_update(g, field, tend, dt, var, var == 'm', static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdyupdate");
}

int wrf_spec_bdyupdate_adj(const WrfGrid* gin, const float* field_bar, float* tend_bar, float dt, char var,
                           void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field_bar || !tend_bar) return fail(WRF_EINVAL, "null argument");
  if (var != 't' && var != 'u' && var != 'v' && var != 'm') return fail(WRF_EINVAL, "spec_bdyupdate_adj: var is t, u, v or m");
  cudaGetLastError();
  launch_spec_update_adj(g, field_bar, tend_bar, dt, var, var == 'm', static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdyupdate_adj");
}

int wrf_spec_bdyupdate_ph(const WrfGrid* gin, const WrfState* sin, float dt, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kSpecPhOperands, sizeof(kSpecPhOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_spec_ph(g, s, dt, static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdyupdate_ph");
}

int wrf_spec_bdyupdate_ph_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float dt, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s, b;
  if ((rc = state_of(sin, kSpecPhOperands, sizeof(kSpecPhOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kSpecPhOperands, sizeof(kSpecPhOperands) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_spec_ph_adj(g, s, b, dt, static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdyupdate_ph_adj");
}

int wrf_prep(const WrfGrid* gin, const WrfState* sin, int ops, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (ops < 1 || ops > 127) return fail(WRF_EINVAL, "prep: ops is a mask of 1 .. 127");
  S s;
  if ((rc = state_of(sin, kPrepOperands, sizeof(kPrepOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_prep_ops(g, s, ops, static_cast<cudaStream_t>(stream));
  return check_launch("prep");
}

int wrf_prep_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int ops, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (ops < 1 || ops > 127) return fail(WRF_EINVAL, "prep_adj: ops is a mask of 1 .. 127");
  S s, b;
  if ((rc = state_of(sin, kPrepOperands, sizeof(kPrepOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kPrepCotangents, sizeof(kPrepCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_prep_ops_adj(g, s, b, ops, static_cast<cudaStream_t>(stream));
  return check_launch("prep_adj");
}

namespace {
bool halo_var(char v) {
  return v == 'u' || v == 'v' || v == 'w' || v == 't' || v == 'p' || v == 'd' || v == 'e' || v == 'f' || v == 'x' ||
         v == 'y' || v == 'r' || v == 'U' || v == 'V';
}
}  // namespace

int wrf_halo(const WrfGrid* gin, float* field, char var, int two_d, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field) return fail(WRF_EINVAL, "null argument");
  if (!halo_var(var)) return fail(WRF_EINVAL, "halo: unknown stagger letter");
  cudaGetLastError();
  launch_halo(g, field, var, two_d != 0, static_cast<cudaStream_t>(stream));
  return check_launch("halo");
}

int wrf_halo_adj(const WrfGrid* gin, const float* field_bar, float* in_bar, char var, int two_d, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field_bar || !in_bar || field_bar == in_bar) return fail(WRF_EINVAL, "halo_adj: two distinct arrays needed");
  if (!halo_var(var)) return fail(WRF_EINVAL, "halo_adj: unknown stagger letter");
  cudaGetLastError();
  launch_halo_adj(g, field_bar, in_bar, var, two_d != 0, static_cast<cudaStream_t>(stream));
  return check_launch("halo_adj");
}

int wrf_zero_grad_w(const WrfGrid* gin, float* w, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!w) return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  launch_zero_grad_w(g, w, static_cast<cudaStream_t>(stream));
  return check_launch("zero_grad_w");
}

int wrf_zero_grad_w_adj(const WrfGrid* gin, const float* w_bar, float* in_bar, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!w_bar || !in_bar || w_bar == in_bar) return fail(WRF_EINVAL, "zero_grad_w_adj: two distinct arrays needed");
  cudaGetLastError();
  launch_zero_grad_w_adj(g, w_bar, in_bar, static_cast<cudaStream_t>(stream));
  return check_launch("zero_grad_w_adj");
}

int wrf_small_step_prep(const WrfGrid* gin, const WrfState* sin, int rk_step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "small_step_prep: rk_step is 1, 2 or 3");
  S s;
  if ((rc = state_of(sin, kSspOperands, sizeof(kSspOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_ssp_only(g, s, rk_step, static_cast<cudaStream_t>(stream));
  return check_launch("small_step_prep");
}

int wrf_small_step_prep_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int rk_step, float* work,
                            void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "small_step_prep_adj: rk_step is 1, 2 or 3");
  if (!work) return fail(WRF_EINVAL, "small_step_prep_adj: work (3 ny*nx floats) is required");
  S s, b;
  if ((rc = state_of(sin, kSspOperands, sizeof(kSspOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kSspCotangents, sizeof(kSspCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_small_step_prep_adj(g, s, b, rk_step, work, static_cast<cudaStream_t>(stream));
  return check_launch("small_step_prep_adj");
}

int wrf_small_step_finish(const WrfGrid* gin, const WrfState* sin, float dts, int nsub, int rk_step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3 || nsub < 1) return fail(WRF_EINVAL, "small_step_finish: rk_step 1..3, nsub >= 1");
  S s;
  if ((rc = state_of(sin, kSsfOperands, sizeof(kSsfOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_small_step_finish(g, s, dts, nsub, rk_step, static_cast<cudaStream_t>(stream));
  return check_launch("small_step_finish");
}

int wrf_small_step_finish_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float dts, int nsub,
                              int rk_step, float* work, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3 || nsub < 1) return fail(WRF_EINVAL, "small_step_finish_adj: rk_step 1..3, nsub >= 1");
  if (!work) return fail(WRF_EINVAL, "small_step_finish_adj: work (2 ny*nx floats) is required");
  S s, b;
  if ((rc = state_of(sin, kSsfOperands, sizeof(kSsfOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kSsfCotangents, sizeof(kSsfCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_small_step_finish_adj(g, s, b, dts, nsub, rk_step, work, static_cast<cudaStream_t>(stream));
  return check_launch("small_step_finish_adj");
}

int wrf_addtend(const WrfGrid* gin, const WrfState* sin, int rk_step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "addtend: rk_step is 1, 2 or 3");
  S s;
  if ((rc = state_of(sin, kAddtendOperands, sizeof(kAddtendOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_addtend_op(g, s, rk_step, static_cast<cudaStream_t>(stream));
  return check_launch("addtend");
}

int wrf_addtend_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int rk_step, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "addtend_adj: rk_step is 1, 2 or 3");
  S s, b;
  if ((rc = state_of(sin, kAddtendOperands, sizeof(kAddtendOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kAddtendCotangents, sizeof(kAddtendCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_addtend_op_adj(g, s, b, rk_step, static_cast<cudaStream_t>(stream));
  return check_launch("addtend_adj");
}

int wrf_spec_bdytend(const WrfGrid* gin, float* tend, const float* txs, const float* txe, const float* tys,
                     const float* tye, char var, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!tend || !txs || !txe || !tys || !tye) return fail(WRF_EINVAL, "null argument");
  if (var != 'u' && var != 'v' && var != 't' && var != 'h' && var != 'm')
    return fail(WRF_EINVAL, "spec_bdytend: var is u, v, t, h or m");
  const float* bt4[4] = {txs, txe, tys, tye};
  cudaGetLastError();
  launch_spec_tend(g, tend, bt4, var, static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdytend");
}

int wrf_spec_bdytend_adj(const WrfGrid* gin, float* tend_bar, char var, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!tend_bar) return fail(WRF_EINVAL, "null argument");
  if (var != 'u' && var != 'v' && var != 't' && var != 'h' && var != 'm')
    return fail(WRF_EINVAL, "spec_bdytend_adj: var is u, v, t, h or m");
  cudaGetLastError();
  launch_spec_tend_adj(g, tend_bar, var, static_cast<cudaStream_t>(stream));
  return check_launch("spec_bdytend_adj");
}

int wrf_eddy_viscosity(const WrfGrid* gin, const WrfState* sin, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kKmOperands, sizeof(kKmOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_km_op(g, s, static_cast<cudaStream_t>(stream));
  return check_launch("eddy_viscosity");
}

int wrf_eddy_viscosity_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float* work,
                           void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!work) return fail(WRF_EINVAL, "eddy_viscosity_adj: work (6*nz*ny*nx floats) is required");
  S s, b;
  if ((rc = state_of(sin, kKmOperands, sizeof(kKmOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kKmCotangents, sizeof(kKmCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_km_op_adj(g, s, b, work, static_cast<cudaStream_t>(stream));
  return check_launch("eddy_viscosity_adj");
}

namespace {
int hdiff_args(const Grid& g, char var, const float* field, const float* mut, const float* xk, const void* out) {
  (void)g;
  if (var != 'u' && var != 'v' && var != 'w' && var != 'm')
    return fail(WRF_EINVAL, "horizontal_diffusion: var is u, v, w or m");
  if (!field || !mut || !xk || !out) return fail(WRF_EINVAL, "null argument");
  return 0;
}
}  // namespace

int wrf_horizontal_diffusion(const WrfGrid* gin, const WrfState* sin, char var, const float* field, const float* base,
                             const float* mut, const float* xk, float* tend, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if ((rc = hdiff_args(g, var, field, mut, xk, tend))) return rc;
  if (base && var != 'm') return fail(WRF_EINVAL, "horizontal_diffusion: base is for a mass-point scalar");
  S s;
  if ((rc = state_of(sin, kHdiffOperands, sizeof(kHdiffOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_hdiff_op(g, s, var, field, base, mut, xk, tend, static_cast<cudaStream_t>(stream));
  return check_launch("horizontal_diffusion");
}

int wrf_horizontal_diffusion_adj(const WrfGrid* gin, const WrfState* sin, char var, const float* field,
                                 const float* base, const float* mut, const float* xk, const float* tend_bar,
                                 float* field_bar, float* mut_bar, float* xk_bar, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if ((rc = hdiff_args(g, var, field, mut, xk, tend_bar))) return rc;
  if (base && var != 'm') return fail(WRF_EINVAL, "horizontal_diffusion_adj: base is for a mass-point scalar");
  S s;
  if ((rc = state_of(sin, kHdiffOperands, sizeof(kHdiffOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_hdiff_op_adj(g, s, var, field, base, mut, xk, tend_bar, field_bar, mut_bar, xk_bar,
                      static_cast<cudaStream_t>(stream));
  return check_launch("horizontal_diffusion_adj");
}

int wrf_mass_weight(const WrfGrid* gin, const float* field, const float* mut, float* out, int nk, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !mut || !out) return fail(WRF_EINVAL, "null argument");
  if (nk < 1 || nk > g.nz) return fail(WRF_EINVAL, "mass_weight: 1 <= nk <= nz");
  cudaGetLastError();
  launch_mass_weight(g, field, mut, out, nk, static_cast<cudaStream_t>(stream));
  return check_launch("mass_weight");
}

int wrf_mass_weight_adj(const WrfGrid* gin, const float* field, const float* mut, const float* out_bar,
                        float* field_bar, float* mut_bar, int nk, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !mut || !out_bar || !field_bar || !mut_bar) return fail(WRF_EINVAL, "null argument");
  if (nk < 1 || nk > g.nz) return fail(WRF_EINVAL, "mass_weight_adj: 1 <= nk <= nz");
  cudaGetLastError();
  launch_mass_weight_adj(g, field, mut, out_bar, field_bar, mut_bar, nk, static_cast<cudaStream_t>(stream));
  return check_launch("mass_weight_adj");
}

int wrf_bdy_final(const WrfGrid* gin, const WrfState* sin, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kBdyFinalOperands, sizeof(kBdyFinalOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_bdy_final_op(g, s, static_cast<cudaStream_t>(stream));
  return check_launch("bdy_final");
}

int wrf_bdy_final_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s, b;
  if ((rc = state_of(sin, kBdyFinalOperands, sizeof(kBdyFinalOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kBdyFinalCotangents, sizeof(kBdyFinalCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_bdy_final_op_adj(g, s, b, static_cast<cudaStream_t>(stream));
  return check_launch("bdy_final_adj");
}

int wrf_microphysics_op(const WrfGrid* gin, const WrfState* sin, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kMpOperands, sizeof(kMpOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_physics(g, s, static_cast<cudaStream_t>(stream));
  return check_launch("microphysics_op");
}

int wrf_microphysics_adj_work(const WrfGrid* gin, size_t* floats) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!floats) return fail(WRF_EINVAL, "null argument");
  *floats = microphysics_adj_work_floats(g);
  return WRF_OK;
}

int wrf_microphysics_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* spost, const WrfState* sbar,
                         float* work, size_t work_floats, const WrfState* values, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!work || work_floats < microphysics_adj_work_floats(g))
    return fail(WRF_EINVAL, "microphysics_adj: work smaller than wrf_microphysics_adj_work gives");
  S s, post, b, vo;
  if ((rc = state_of(sin, kMpAdjOperands, sizeof(kMpAdjOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(spost, kMpAdjOperands, sizeof(kMpAdjOperands) / sizeof(int), post))) return rc;
  if ((rc = state_of(sbar, kMpCotangents, sizeof(kMpCotangents) / sizeof(int), b))) return rc;
  const int kVals[] = {WF_T, WF_MOIST, WF_H_DIABATIC};
  if (values && (rc = state_of(values, kVals, 3, vo))) return rc;
  cudaGetLastError();
  launch_physics_adj(g, s, post, b, work, g.dt, static_cast<cudaStream_t>(stream), values ? &vo : nullptr);
  return check_launch("microphysics_adj");
}

int wrf_set_microphysics_tape_capacity(int entries, int* previous) {
  if (entries < 0) return fail(WRF_EINVAL, "microphysics tape capacity: negative");
  const int prev = set_microphysics_tape_capacity(entries);
  if (previous) *previous = prev;
  return WRF_OK;
}

int wrf_calc_p_rho_phi(const WrfGrid* gin, const WrfState* sin, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s;
  if ((rc = state_of(sin, kEosOperands, sizeof(kEosOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_eos(g, s, static_cast<cudaStream_t>(stream));
  return check_launch("calc_p_rho_phi");
}

int wrf_moist_update(const WrfGrid* gin, const WrfState* sin, int rk_step, float dt_rk, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "moist_update: rk_step is 1, 2 or 3");
  S s;
  if ((rc = state_of(sin, kMoistOperands, sizeof(kMoistOperands) / sizeof(int), s))) return rc;
  cudaGetLastError();
  launch_moist(g, s, rk_step, dt_rk, static_cast<cudaStream_t>(stream));
  return check_launch("moist_update");
}

int wrf_moist_update_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, int rk_step, float dt_rk,
                         float* work, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (rk_step < 1 || rk_step > 3) return fail(WRF_EINVAL, "moist_update_adj: rk_step is 1, 2 or 3");
  if (!work) return fail(WRF_EINVAL, "moist_update_adj: work (nz*ny*nx floats) is required");
  S s, b;
  if ((rc = state_of(sin, kMoistOperands, sizeof(kMoistOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kMoistCotangents, sizeof(kMoistCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_moist_adj(g, s, b, rk_step, dt_rk, work, static_cast<cudaStream_t>(stream));
  return check_launch("moist_update_adj");
}

int wrf_advance_uv_adj(const WrfGrid* gin, const WrfState* sin, const WrfState* sbar, float dts, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  S s, b;
  if ((rc = state_of(sin, kUvOperands, sizeof(kUvOperands) / sizeof(int), s))) return rc;
  if ((rc = state_of(sbar, kUvCotangents, sizeof(kUvCotangents) / sizeof(int), b))) return rc;
  cudaGetLastError();
  launch_advance_uv_adj(g, s, b, dts, static_cast<cudaStream_t>(stream));
  return check_launch("advance_uv_adj");
}

int wrf_advect_momentum_adj(const WrfGrid* gin, int component, const float* field, const float* ru, const float* rv,
                            const float* rom, const float* msf, const float* msf2, const float* fzm, const float* fzp,
                            const float* rdz, const float* tend_bar, float* field_bar, float* ru_bar, float* rv_bar,
                            float* rom_bar, float* work, size_t work_floats, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (component < 0 || component > 2) return fail(WRF_EINVAL, "advect_momentum_adj: component 0..2");
  if (!field || !ru || !rv || !rom || !msf || (component == 1 && !msf2) || !fzm || !fzp || !rdz || !tend_bar ||
      !field_bar || !ru_bar || !rv_bar || !rom_bar || !work)
    return fail(WRF_EINVAL, "null argument");
  if (work_floats < advect_mom_adj_work_floats(g))
    return fail(WRF_EINVAL, "advect_momentum_adj: work smaller than wrf_advect_momentum_adj_work gives");
  cudaGetLastError();
  launch_advect_mom_adj(g, component, field, ru, rv, rom, msf, msf2, fzm, fzp, rdz, tend_bar, field_bar, ru_bar,
                        rv_bar, rom_bar, work, static_cast<cudaStream_t>(stream));
  return check_launch("advect_momentum_adj");
}

int wrf_advect_momentum_adj_work(const WrfGrid* gin, size_t* floats) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!floats) return fail(WRF_EINVAL, "null argument");
  *floats = advect_mom_adj_work_floats(g);
  return WRF_OK;
}

int wrf_relax_bdytend(const WrfGrid* gin, const float* field, float* tend, const float* const* bdy8, char variable,
                      float dtbc, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!field || !tend || !bdy8) return fail(WRF_EINVAL, "null argument");
  for (int q = 0; q < 8; ++q)
    if (!bdy8[q]) return fail(WRF_EINVAL, "null boundary array");
  cudaGetLastError();
  launch_relax_field(g, field, tend, bdy8, variable, dtbc, static_cast<cudaStream_t>(stream));
  return check_launch("relax_bdytend");
}

int wrf_relax_bdytend_adj(const WrfGrid* gin, const float* tend_bar, float* field_bar, char variable, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!tend_bar || !field_bar) return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  launch_relax_field_adj(g, tend_bar, field_bar, variable, static_cast<cudaStream_t>(stream));
  return check_launch("relax_bdytend_adj");
}

int wrf_vsolve_w(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma, float* w,
                 void* stream) {
  if (!x || !a || !alpha || !gamma || !w) return fail(WRF_EINVAL, "null argument");
  if (ncol < 1 || nz < 3 || nz > kMaxNz) return fail(WRF_EINVAL, "vsolve_w: needs ncol >= 1 and 3 <= nz <= 64");
  cudaGetLastError();
  launch_vsolve_w(ncol, nz, x, a, alpha, gamma, w, static_cast<cudaStream_t>(stream));
  return check_launch("vsolve_w");
}

int wrf_vsolve_w_adj(int ncol, int nz, const float* x, const float* a, const float* alpha, const float* gamma,
                     const float* w_bar, float* x_bar, float* a_bar, float* alpha_bar, float* gamma_bar,
                     void* stream) {
  if (!x || !a || !alpha || !gamma || !w_bar || !x_bar || !a_bar || !alpha_bar || !gamma_bar)
    return fail(WRF_EINVAL, "null argument");
  if (ncol < 1 || nz < 3 || nz > kMaxNz) return fail(WRF_EINVAL, "vsolve_w_adj: needs ncol >= 1 and 3 <= nz <= 64");
  cudaGetLastError();
  launch_vsolve_w_adj(ncol, nz, x, a, alpha, gamma, w_bar, x_bar, a_bar, alpha_bar, gamma_bar,
                      static_cast<cudaStream_t>(stream));
  return check_launch("vsolve_w_adj");
}

int wrf_coef_w(const WrfGrid* gin, const float* mut, const float* cqw, const float* c2a, const float* rdn,
               const float* rdnw, float dts, float* a, float* alpha, float* gamma, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!mut || !cqw || !c2a || !rdn || !rdnw || !a || !alpha || !gamma) return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  launch_coef_w(g, mut, cqw, c2a, rdn, rdnw, dts, a, alpha, gamma, static_cast<cudaStream_t>(stream));
  return check_launch("coef_w");
}

int wrf_coef_w_adj(const WrfGrid* gin, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                   const float* rdnw, float dts, const float* a_bar, const float* alpha_bar, const float* gamma_bar,
                   float* mut_bar, float* cqw_bar, float* c2a_bar, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!mut || !cqw || !c2a || !rdn || !rdnw || !a_bar || !alpha_bar || !gamma_bar || !mut_bar || !cqw_bar || !c2a_bar)
    return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  launch_coef_w_adj(g, mut, cqw, c2a, rdn, rdnw, dts, a_bar, alpha_bar, gamma_bar, mut_bar, cqw_bar, c2a_bar,
                    static_cast<cudaStream_t>(stream));
  return check_launch("coef_w_adj");
}

int wrf_wsm6(const WrfGrid* gin, float* th, float* qv, float* qc, float* qr, float* qi, float* qs, float* qg,
             const float* rho, const float* pii, const float* p, const float* dz8w, float delt, float* rainnc,
             float* rainncv, float* snownc, float* snowncv, float* graupelnc, float* graupelncv, float* sr,
             void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  float* f[18] = {th, qv, qc, qr, qi, qs, qg, const_cast<float*>(rho), const_cast<float*>(pii),
                  const_cast<float*>(p), const_cast<float*>(dz8w), rainnc, rainncv, snownc, snowncv,
                  graupelnc, graupelncv, sr};
  for (float* x : f)
    if (!x) return fail(WRF_EINVAL, "null argument");
  if (!(delt > 0.f)) return fail(WRF_EINVAL, "delt must be > 0");
  cudaGetLastError();
  launch_wsm6(g, f, delt, static_cast<cudaStream_t>(stream));
  return check_launch("wsm6");
}

int wrf_wsm6_noalloc(const WrfGrid* gin, float* th, float* qv, float* qc, float* qr, float* qi, float* qs,
                     float* qg, const float* rho, const float* pii, const float* p, const float* dz8w, float delt,
                     float* rainnc, float* rainncv, float* snownc, float* snowncv, float* graupelnc,
                     float* graupelncv, float* sr, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  float* f[18] = {th, qv, qc, qr, qi, qs, qg, const_cast<float*>(rho), const_cast<float*>(pii),
                  const_cast<float*>(p), const_cast<float*>(dz8w), rainnc, rainncv, snownc, snowncv,
                  graupelnc, graupelncv, sr};
  for (float* x : f)
    if (!x) return fail(WRF_EINVAL, "null argument");
  if (!(delt > 0.f)) return fail(WRF_EINVAL, "delt must be > 0");
  cudaGetLastError();
  const char* err = nullptr;
  rc = launch_wsm6_noalloc(g, f, delt, static_cast<cudaStream_t>(stream), &err);
  if (rc < 0) return fail(rc, err ? err : "wrf_wsm6_noalloc failed");
  return check_launch("wsm6_noalloc");
}

int wrf_status_read(const WrfState* sin, void* stream, int* out16) {
  if (!sin || !sin->f[WF_STATUS] || !out16) return fail(WRF_EINVAL, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(out16, sin->f[WF_STATUS], 16 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return check_launch("status_read");
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("status_read");
  return WRF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- network
namespace {
MlpLayout layout_of(const Grid& g) { return MlpLayout::make(g.nx, g.ny, g.nz, g.ids, g.ide, g.jds, g.jde); }
int ret_launch(int r, const char* err, const char* where) {
  if (r < 0) return fail(r, err ? err : where);
  return check_launch(where);
}
}  // namespace

extern "C" {

int wrf_mlp_init(void) {
  if (mlp_prepare_device() != WRF_OK) return fail(WRF_ECUDA, "mlp_init: cannot set the kernels' shared-memory limits");
  return WRF_OK;
}

int wrf_mlp_layout(const WrfGrid* gin, int* out8) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!out8) return fail(WRF_EINVAL, "null argument");
  const MlpLayout L = layout_of(g);
  const int v[8] = {L.km, L.ncx, L.ncy, L.ncols, L.nfeat, L.d0, L.nout, L.d4};
  for (int i = 0; i < 8; ++i) out8[i] = v[i];
  return WRF_OK;
}

}  // extern "C"

namespace {
MlpNetDev net_of(const WrfMlpNet* net) {
  MlpNetDev nd;
  for (int l = 0; l <= kMlpLayers; ++l) nd.dims[l] = net->dims[l];
  for (int l = 0; l < kMlpLayers; ++l) {
    nd.w[l] = net->w[l];
    nd.b[l] = net->b[l];
  }
  nd.norm = net->norm;
  nd.tol_neg = net->tol_neg;
  nd.tol_sat = net->tol_sat;
  return nd;
}
}  // namespace

extern "C" {

int wrf_mlp_forward(const WrfMlpNet* net, const void* x, int m, void* h0, void* h1, float* y, int* err,
                    void* stream) {
  if (!net || !x || !h0 || !h1 || !y || m < 1) return fail(WRF_EINVAL, "null argument or m < 1");
  for (int l = 0; l < kMlpLayers; ++l)
    if (!net->w[l] || !net->b[l]) return fail(WRF_EINVAL, "null weight or bias");
  const MlpNetDev nd = net_of(net);
  cudaGetLastError();
  const char* msg = nullptr;
  const int r = launch_mlp_forward(nd, x, m, h0, h1, y, err, static_cast<cudaStream_t>(stream), &msg);
  return ret_launch(r, msg, "mlp_forward");
}

int wrf_rk3_step_mlp(const WrfGrid* gin, const WrfState* sin, const WrfMlpNet* net, const WrfMlpWork* work,
                     void* stream, wrf_probe_fn probe, void* user) {
  if (!net || !work) return fail(WRF_EINVAL, "null network or work buffers");
  const MlpNetDev nd = net_of(net);
  MlpWorkDev wd;
  wd.capacity = work->capacity;
  wd.x = work->x;
  wd.h[0] = work->h[0];
  wd.h[1] = work->h[1];
  wd.y = work->y;
  wd.list = work->list;
  wd.err = work->err;
  wd.colstat = work->colstat;
  Driver d;
  int rc = make_grid(gin, d.g);
  if (rc) return rc;
  rc = make_state(sin, d.s);
  if (rc) return rc;
  d.st = static_cast<cudaStream_t>(stream);
  d.probe = probe;
  d.user = user;
  d.bdy_interval = gin->bdy_interval;
  d.net = &nd;
  d.work = &wd;
  cudaGetLastError();
  d.run();
  g_last_launches = d.n;
  return d.rc;
}

int wrf_mlp_features(const WrfGrid* gin, const WrfState* sin, const float* norm, void* x, float* raw, void* stream) {
  Grid g;
  S s;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  rc = make_state(sin, s);
  if (rc) return rc;
  if (!raw && (!x || !norm)) return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  const int r = launch_mlp_features(g, s, layout_of(g), norm, x, raw, static_cast<cudaStream_t>(stream));
  return ret_launch(r, nullptr, "mlp_features");
}

int wrf_mlp_targets(const WrfGrid* gin, const WrfState* sin, const float* raw_in, float* raw_out, void* stream) {
  Grid g;
  S s;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  rc = make_state(sin, s);
  if (rc) return rc;
  if (!raw_in || !raw_out) return fail(WRF_EINVAL, "null argument");
  cudaGetLastError();
  return ret_launch(launch_mlp_targets(g, s, layout_of(g), raw_in, raw_out, static_cast<cudaStream_t>(stream)),
                    nullptr, "mlp_targets");
}

int wrf_mlp_normalize(const WrfGrid* gin, const float* norm, const float* raw_in, const float* raw_out, long long n,
                      void* x, float* t, void* stream) {
  Grid g;
  int rc = make_grid(gin, g);
  if (rc) return rc;
  if (!norm || !raw_in || !raw_out || !x || !t || n < 0) return fail(WRF_EINVAL, "null argument or n < 0");
  cudaGetLastError();
  return ret_launch(launch_mlp_normalize(layout_of(g), norm, raw_in, raw_out, n, x, t,
                                         static_cast<cudaStream_t>(stream)),
                    nullptr, "mlp_normalize");
}

int wrf_gemm_bf16(const void* a, const void* b, int m, int n, int k, int splits, int epi, const float* bias,
                  const void* aux, void* out, int ldo, long long split_stride, void* out_z, void* out_t, int ldt,
                  int* err, void* stream) {
  GemmEpi e{};
  e.kind = epi;
  e.bias = bias;
  e.aux = static_cast<const __nv_bfloat16*>(aux);
  e.out = out;
  e.ldo = ldo;
  e.split_stride = split_stride;
  e.out_z = static_cast<__nv_bfloat16*>(out_z);
  e.out_t = static_cast<__nv_bfloat16*>(out_t);
  e.ldt = ldt;
  e.err = err;
  if (epi == EPI_F32 && gemm_splits_used(k, splits) > 1 && split_stride < (long long)m * ldo)
    return fail(WRF_EINVAL, "gemm: split_stride smaller than one partial sum");
  if (epi == EPI_F32 && (split_stride % 4)) return fail(WRF_EINVAL, "gemm: split_stride must be a multiple of 4");
  cudaGetLastError();
  const char* msg = nullptr;
  const int r = launch_gemm_tc(a, b, m, n, k, splits, e, static_cast<cudaStream_t>(stream), &msg);
  return ret_launch(r, msg, "gemm_bf16");
}

int wrf_gemm_splits(int k, int splits) { return gemm_splits_used(k, splits); }

int wrf_mse_grad(const float* y, const float* t, int m, int n, int nvalid, float scale, void* dy, void* dyt,
                 float* loss, void* stream) {
  if (!y || !t || !dy || !dyt || !loss || m < 1 || n < 1) return fail(WRF_EINVAL, "null argument or empty matrix");
  cudaGetLastError();
  return ret_launch(launch_mse_grad(y, t, m, n, nvalid, scale, dy, dyt, loss, static_cast<cudaStream_t>(stream)),
                    nullptr, "mse_grad");
}

int wrf_rowsum_bf16(const void* a, int rows, int cols, float* out, void* stream) {
  if (!a || !out || rows < 1 || cols < 1) return fail(WRF_EINVAL, "null argument or empty matrix");
  cudaGetLastError();
  return ret_launch(launch_rowsum_bf16(a, rows, cols, out, static_cast<cudaStream_t>(stream)), nullptr,
                    "rowsum_bf16");
}

int wrf_adam(float* w, const float* gpart, int nsplit, long long split_stride, float* m, float* v, int r, int c,
             void* wb, void* wtb, float lr, float beta1, float beta2, float eps, float wd, int step, void* stream) {
  if (!w || !gpart || !m || !v || r < 1 || c < 1 || nsplit < 1 || step < 1)
    return fail(WRF_EINVAL, "null argument, empty matrix, or step < 1");
  const float bc1 = (float)(1.0 - pow((double)beta1, step)), bc2 = (float)(1.0 - pow((double)beta2, step));
  cudaGetLastError();
  return ret_launch(launch_adam(w, gpart, nsplit, split_stride, m, v, r, c, wb, wtb, lr, beta1, beta2, eps, wd, bc1,
                                bc2, static_cast<cudaStream_t>(stream)),
                    nullptr, "adam");
}

int wrf_transpose_bf16(const void* a, int r, int c, void* out, void* stream) {
  if (!a || !out || r < 1 || c < 1) return fail(WRF_EINVAL, "null argument or empty matrix");
  cudaGetLastError();
  return ret_launch(launch_transpose_bf16(a, r, c, out, static_cast<cudaStream_t>(stream)), nullptr,
                    "transpose_bf16");
}

}  // extern "C"
