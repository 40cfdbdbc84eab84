// Reverse-mode differentiation of scalar device code by a per-thread tape.
//
// Tv carries a float value and the index of the tape entry that produced it
// (-1 for a constant).  Every arithmetic operation or elementary function on
// a Tv appends one entry -- the indices of its (at most two) operands and
// the partial derivatives with respect to them -- to the calling thread's
// tape; selections (vmin, vmax, sel, the branches of the code) append
// nothing: the result is the chosen operand itself, so the derivative is
// that of the branch taken.  Adding a constant appends nothing either (the
// result keeps its operand's entry).  After the forward code has run, the
// reverse sweep walks the thread's entries backwards and accumulates the
// adjoints of the operands.
//
// A thread's tape lives in global memory, interleaved across the threads of
// a launch (entry n of lane t at n * stride + t), so that threads running
// the same operation store and load neighbouring words: the two operand
// indices packed in 16 bits each (0xffff for none), the two partials, and
// the entry's adjoint (zeroed when the entry is recorded).  The per-thread
// entry count sits in shared memory (blocks of at most kTapeBlock threads)
// beside the launch's tape context.  Entries past the capacity are counted
// but not stored; the caller compares the count with the capacity and
// treats such a thread's tape as unusable.
#pragma once
#include "dual.cuh"

namespace wrf {

constexpr int kTapeBlock = 64;
constexpr int kTapeMaxEntries = 0xffff;  // operand indices fit in 16 bits

struct TapeCtx {
  unsigned* ab;  // packed operand indices of entry n of lane t at [n * stride + t]
  float2* dd;    // partials
  float* adj;    // adjoints
  int stride, cap;
};

// the block's tape context and the per-thread entry counts
__shared__ TapeCtx g_tape;
__shared__ int g_tape_n[kTapeBlock];

struct Tv {
  float v;
  int id;
};

__device__ __forceinline__ int tape_lane() { return blockIdx.x * blockDim.x + threadIdx.x; }

__device__ __forceinline__ int tape_rec(int a, int b, float da, float db) {
  if (a < 0 && b < 0) return -1;  // constant operands: a constant
  const int t = threadIdx.x;
  const int n = g_tape_n[t];
  g_tape_n[t] = n + 1;
  if (n < g_tape.cap) {
    const size_t q = (size_t)n * g_tape.stride + tape_lane();
    g_tape.ab[q] = (unsigned)(a & 0xffff) | ((unsigned)(b & 0xffff) << 16);
    g_tape.dd[q] = make_float2(da, db);
    g_tape.adj[q] = 0.f;
  }
  return n;
}

// reserve entries [0, n) for the independent variables (the inputs of the
// taped code): Tv{value, index} with index < n then names input index
__device__ __forceinline__ void tape_reserve(int n) {
  const int t = threadIdx.x;
  const int m = n < g_tape.cap ? n : g_tape.cap;
  for (int k = 0; k < m; ++k) g_tape.adj[(size_t)k * g_tape.stride + tape_lane()] = 0.f;
  g_tape_n[t] = n;
}

__device__ __forceinline__ float val(const Tv& x) { return x.v; }

__device__ __forceinline__ Tv operator+(const Tv& a, const Tv& b) {
  return Tv{a.v + b.v, tape_rec(a.id, b.id, 1.f, 1.f)};
}
__device__ __forceinline__ Tv operator-(const Tv& a, const Tv& b) {
  return Tv{a.v - b.v, tape_rec(a.id, b.id, 1.f, -1.f)};
}
__device__ __forceinline__ Tv operator-(const Tv& a) { return Tv{-a.v, tape_rec(a.id, -1, -1.f, 0.f)}; }
__device__ __forceinline__ Tv operator*(const Tv& a, const Tv& b) {
  return Tv{a.v * b.v, tape_rec(a.id, b.id, b.v, a.v)};
}
__device__ __forceinline__ Tv operator/(const Tv& a, const Tv& b) {
  const float r = a.v / b.v;
  const float ib = 1.0f / b.v;
  return Tv{r, tape_rec(a.id, b.id, ib, -r * ib)};
}
__device__ __forceinline__ Tv operator+(const Tv& a, float b) { return Tv{a.v + b, a.id}; }
__device__ __forceinline__ Tv operator+(float a, const Tv& b) { return Tv{a + b.v, b.id}; }
__device__ __forceinline__ Tv operator-(const Tv& a, float b) { return Tv{a.v - b, a.id}; }
__device__ __forceinline__ Tv operator-(float a, const Tv& b) { return Tv{a - b.v, tape_rec(b.id, -1, -1.f, 0.f)}; }
__device__ __forceinline__ Tv operator*(const Tv& a, float b) { return Tv{a.v * b, tape_rec(a.id, -1, b, 0.f)}; }
__device__ __forceinline__ Tv operator*(float a, const Tv& b) { return Tv{a * b.v, tape_rec(b.id, -1, a, 0.f)}; }
__device__ __forceinline__ Tv operator/(const Tv& a, float b) { return Tv{a.v / b, tape_rec(a.id, -1, 1.0f / b, 0.f)}; }
__device__ __forceinline__ Tv operator/(float a, const Tv& b) {
  const float r = a / b.v;
  return Tv{r, tape_rec(b.id, -1, -r / b.v, 0.f)};
}

// elementary functions: the value by the library's float function, the
// partial from its closed form (as in the dual numbers)
__device__ __forceinline__ Tv vsqrt(const Tv& x) {
  const float v = sqrtf(x.v);
  return Tv{v, tape_rec(x.id, -1, v > 0.f ? 0.5f / v : 0.f, 0.f)};
}
__device__ __forceinline__ Tv vexp(const Tv& x) {
  const float v = wexp(x.v);
  return Tv{v, tape_rec(x.id, -1, v, 0.f)};
}
__device__ __forceinline__ Tv vlog(const Tv& x) { return Tv{wlog(x.v), tape_rec(x.id, -1, 1.0f / x.v, 0.f)}; }
__device__ __forceinline__ Tv vpow(const Tv& x, float e) {
  const float v = wpow(x.v, e);
  return Tv{v, tape_rec(x.id, -1, x.v != 0.f ? e * v / x.v : 0.f, 0.f)};
}
__device__ __forceinline__ Tv vabs(const Tv& x) { return x.v < 0.f ? -x : x; }
__device__ __forceinline__ Tv vmin(const Tv& a, const Tv& b) { return b.v < a.v ? b : a; }
__device__ __forceinline__ Tv vmax(const Tv& a, const Tv& b) { return b.v > a.v ? b : a; }
__device__ __forceinline__ Tv vmin(const Tv& a, float b) { return b < a.v ? Tv{b, -1} : a; }
__device__ __forceinline__ Tv vmax(const Tv& a, float b) { return b > a.v ? Tv{b, -1} : a; }
__device__ __forceinline__ Tv vmin(float a, const Tv& b) { return b.v < a ? b : Tv{a, -1}; }
__device__ __forceinline__ Tv vmax(float a, const Tv& b) { return b.v > a ? b : Tv{a, -1}; }

template <>
struct Lift<Tv> {
  __device__ static Tv c(float x) { return Tv{x, -1}; }
};

// one contribution c to the adjoint of entry a (0xffff: none) during the
// sweep's step t, after the load of step t + D: to the window's
// accumulator of a's step when it lies inside the window (steps t + 1 ..
// t + D), else a fire-and-forget reduction in memory
template <int D>
__device__ __forceinline__ void tape_give(const TapeCtx& tc, size_t lane, int n0, int n, int t, unsigned a, float c,
                                          float (&acc)[D]) {
  if (a == 0xffffu || c == 0.f) return;
  const int ta = n - 1 - (int)a;
  if ((int)a >= n0 && ta <= t + D) {
    const int slot = ta & (D - 1);
#pragma unroll
    for (int u = 0; u < D; ++u) acc[u] += slot == u ? c : 0.f;
  } else {
    atomicAdd(tc.adj + (size_t)a * tc.stride + lane, c);
  }
}

// the reverse sweep of lane's entries [n0, n) (n within the capacity):
// adj[a] += da adj[e], adj[b] += db adj[e] from the last entry down.  The
// sweep is software-pipelined over a window of D entries held in
// registers: entry e's record and adjoint are loaded D steps before they
// are used, a contribution to an entry inside the window goes to the
// window's accumulator registers (kept apart from the loaded values, so
// that no contribution waits for a load in flight), and one to an entry
// below the window is a fire-and-forget reduction in memory, which the
// entry's own load (issued later in program order) sees.  The window's
// slot of step t (entry n - 1 - t) is t mod D.
template <int D>
__device__ __forceinline__ void tape_sweep(const TapeCtx& tc, size_t lane, int n0, int n) {
  static_assert((D & (D - 1)) == 0, "window of a power of two");
  const size_t st = tc.stride;
  const int steps = n - n0;
  float w[D], acc[D];
  unsigned ab[D];
  float2 dd[D];
#pragma unroll
  for (int u = 0; u < D; ++u) {
    acc[u] = 0.f;
    w[u] = 0.f;
    ab[u] = 0xffffffffu;
    dd[u] = make_float2(0.f, 0.f);
    if (u < steps) {
      const size_t q = (size_t)(n - 1 - u) * st + lane;
      w[u] = __ldcg(tc.adj + q);
      ab[u] = __ldcs(tc.ab + q);
      dd[u] = __ldcs(tc.dd + q);
    }
  }
  for (int t0 = 0; t0 < steps; t0 += D) {
#pragma unroll
    for (int u = 0; u < D; ++u) {
      const int t = t0 + u;
      if (t < steps) {
        const float wv = w[u] + acc[u];
        const unsigned abv = ab[u];
        const float2 ddv = dd[u];
        acc[u] = 0.f;
        if (t + D < steps) {
          const size_t q = (size_t)(n - 1 - t - D) * st + lane;
          w[u] = __ldcg(tc.adj + q);
          ab[u] = __ldcs(tc.ab + q);
          dd[u] = __ldcs(tc.dd + q);
        }
        if (wv != 0.f) {
          tape_give<D>(tc, lane, n0, n, t, abv & 0xffffu, ddv.x * wv, acc);
          tape_give<D>(tc, lane, n0, n, t, abv >> 16, ddv.y * wv, acc);
        }
      }
    }
  }
}

}  // namespace wrf
