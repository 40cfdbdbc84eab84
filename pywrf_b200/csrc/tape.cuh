// Reverse-mode differentiation of scalar device code by a per-thread tape.
//
// Tv carries a float value, the index of a tape entry (-1 for a constant)
// and the multiple of that entry's value it is.  Every arithmetic operation
// or elementary function of taped operands appends one entry -- the indices
// of its (at most two) operands and the partial derivatives with respect to
// them -- to the calling thread's tape; selections (vmin, vmax, sel, the
// branches of the code) append nothing: the result is the chosen operand
// itself, so the derivative is that of the branch taken.  Adding a
// constant, scaling by one and negating append nothing either: the multiple
// changes and enters the partials of the next entry that uses the value.
// After the forward code has run, the reverse sweep walks the thread's
// entries backwards and accumulates the adjoints of the operands.
//
// A thread's tape lives in global memory, contiguous per thread (entry n of
// lane t at t * cap + n): the lanes of a warp are mostly at different
// entries, so a warp's accesses fall on different cache lines whatever the
// layout, and a contiguous tape lets the consecutive entries a thread
// writes, then reads back in reverse, share lines and DRAM bursts.  An
// entry is one 16-byte record -- the two operand indices packed in 16 bits
// each (0xffff for none), the two partials, and the entry's adjoint (zeroed
// when the entry is recorded) -- written by one vector store and read back
// by one vector load.  The per-thread entry count sits in shared memory
// (blocks of at most kTapeBlock threads) beside the launch's tape context.
// Entries past the capacity are counted but not stored; the caller
// compares the count with the capacity and treats such a thread's tape as
// unusable.
#pragma once
#include "dual.cuh"

namespace wrf {

constexpr int kTapeBlock = 64;
constexpr int kTapeMaxEntries = 0xffff;  // operand indices fit in 16 bits

// an entry: x the packed operand indices, y and z the partials (float
// bits), w the adjoint
using TapeRec = uint4;

struct TapeCtx {
  TapeRec* rec;  // entry n of lane t at rec[t * cap + n]
  int stride;    // the interleave stride of the caller's column arrays (lanes)
  int cap;
  __device__ __forceinline__ TapeRec* at(size_t n, size_t lane) const { return rec + lane * (size_t)cap + n; }
  // the adjoint of entry n of lane
  __device__ __forceinline__ float* adj(size_t n, size_t lane) const {
    return reinterpret_cast<float*>(at(n, lane)) + 3;
  }
};

// the block's tape context and the per-thread entry counts
__shared__ TapeCtx g_tape;
__shared__ int g_tape_n[kTapeBlock];

// a taped value: v the value, id the entry it is a multiple of (-1: a
// constant) and s that multiple, so that scaling by a constant, negation
// and adding a constant record nothing
struct Tv {
  float v;
  int id;
  float s;
};

__device__ __forceinline__ int tape_lane() { return blockIdx.x * blockDim.x + threadIdx.x; }

__device__ __forceinline__ int tape_rec(int a, int b, float da, float db) {
  if (a < 0 && b < 0) return -1;  // constant operands: a constant
  const int t = threadIdx.x;
  const int n = g_tape_n[t];
  g_tape_n[t] = n + 1;
  if (n < g_tape.cap)
    *g_tape.at(n, tape_lane()) =
        make_uint4((unsigned)(a & 0xffff) | ((unsigned)(b & 0xffff) << 16), __float_as_uint(da), __float_as_uint(db), 0u);
  return n;
}

// reserve entries [0, n) for the independent variables (the inputs of the
// taped code): Tv{value, index, 1} with index < n then names input index
__device__ __forceinline__ void tape_reserve(int n) {
  const int t = threadIdx.x;
  const int m = n < g_tape.cap ? n : g_tape.cap;
  for (int k = 0; k < m; ++k) *g_tape.at(k, tape_lane()) = make_uint4(0xffffffffu, 0u, 0u, 0u);
  g_tape_n[t] = n;
}

__device__ __forceinline__ float val(const Tv& x) { return x.v; }

// a new entry with operands a and b (partials with respect to the values)
__device__ __forceinline__ Tv tape_op(float v, const Tv& a, float da, const Tv& b, float db) {
  return Tv{v, tape_rec(a.id, b.id, da * a.s, db * b.s), 1.f};
}
__device__ __forceinline__ Tv tape_op1(float v, const Tv& x, float dx) {
  return Tv{v, tape_rec(x.id, -1, dx * x.s, 0.f), 1.f};
}

__device__ __forceinline__ Tv operator+(const Tv& a, const Tv& b) {
  if (b.id < 0) return Tv{a.v + b.v, a.id, a.s};
  if (a.id < 0) return Tv{a.v + b.v, b.id, b.s};
  return tape_op(a.v + b.v, a, 1.f, b, 1.f);
}
__device__ __forceinline__ Tv operator-(const Tv& a, const Tv& b) {
  if (b.id < 0) return Tv{a.v - b.v, a.id, a.s};
  if (a.id < 0) return Tv{a.v - b.v, b.id, -b.s};
  return tape_op(a.v - b.v, a, 1.f, b, -1.f);
}
__device__ __forceinline__ Tv operator-(const Tv& a) { return Tv{-a.v, a.id, -a.s}; }
__device__ __forceinline__ Tv operator*(const Tv& a, const Tv& b) {
  if (b.id < 0) return Tv{a.v * b.v, a.id, a.s * b.v};
  if (a.id < 0) return Tv{a.v * b.v, b.id, b.s * a.v};
  return tape_op(a.v * b.v, a, b.v, b, a.v);
}
__device__ __forceinline__ Tv operator/(const Tv& a, const Tv& b) {
  const float r = a.v / b.v;
  if (b.id < 0) return Tv{r, a.id, a.s / b.v};
  const float ib = 1.0f / b.v;
  return tape_op(r, a, ib, b, -r * ib);
}
__device__ __forceinline__ Tv operator+(const Tv& a, float b) { return Tv{a.v + b, a.id, a.s}; }
__device__ __forceinline__ Tv operator+(float a, const Tv& b) { return Tv{a + b.v, b.id, b.s}; }
__device__ __forceinline__ Tv operator-(const Tv& a, float b) { return Tv{a.v - b, a.id, a.s}; }
__device__ __forceinline__ Tv operator-(float a, const Tv& b) { return Tv{a - b.v, b.id, -b.s}; }
__device__ __forceinline__ Tv operator*(const Tv& a, float b) { return Tv{a.v * b, a.id, a.s * b}; }
__device__ __forceinline__ Tv operator*(float a, const Tv& b) { return Tv{a * b.v, b.id, b.s * a}; }
__device__ __forceinline__ Tv operator/(const Tv& a, float b) { return Tv{a.v / b, a.id, a.s / b}; }
__device__ __forceinline__ Tv operator/(float a, const Tv& b) {
  const float r = a / b.v;
  return tape_op1(r, b, -r / b.v);
}

// elementary functions: the value by the library's float function, the
// partial from its closed form (as in the dual numbers)
__device__ __forceinline__ Tv vsqrt(const Tv& x) {
  const float v = sqrtf(x.v);
  return tape_op1(v, x, v > 0.f ? 0.5f / v : 0.f);
}
__device__ __forceinline__ Tv vexp(const Tv& x) {
  const float v = wexp(x.v);
  return tape_op1(v, x, v);
}
__device__ __forceinline__ Tv vlog(const Tv& x) { return tape_op1(wlog(x.v), x, 1.0f / x.v); }
__device__ __forceinline__ Tv vpow(const Tv& x, float e) {
  const float v = wpow(x.v, e);
  return tape_op1(v, x, x.v != 0.f ? e * v / x.v : 0.f);
}
__device__ __forceinline__ Tv vabs(const Tv& x) { return x.v < 0.f ? -x : x; }
__device__ __forceinline__ Tv vmin(const Tv& a, const Tv& b) { return b.v < a.v ? b : a; }
__device__ __forceinline__ Tv vmax(const Tv& a, const Tv& b) { return b.v > a.v ? b : a; }
__device__ __forceinline__ Tv vmin(const Tv& a, float b) { return b < a.v ? Tv{b, -1, 0.f} : a; }
__device__ __forceinline__ Tv vmax(const Tv& a, float b) { return b > a.v ? Tv{b, -1, 0.f} : a; }
__device__ __forceinline__ Tv vmin(float a, const Tv& b) { return b.v < a ? b : Tv{a, -1, 0.f}; }
__device__ __forceinline__ Tv vmax(float a, const Tv& b) { return b.v > a ? b : Tv{a, -1, 0.f}; }

template <>
struct Lift<Tv> {
  __device__ static Tv c(float x) { return Tv{x, -1, 0.f}; }
};

// the reverse sweep of lane's entries [n0, n) (n within the capacity):
// adj[a] += da adj[e], adj[b] += db adj[e] from the last entry down, by
// the threads of a block of B threads.  Entry e's record (operands,
// partials and the adjoint it holds in memory) is loaded D steps before it
// is used, into a window of registers.  A contribution to one of the next
// A - 1 entries goes to the thread's ring of A accumulators in shared
// memory (acc[slot * B + thread], conflict-free across the warp; the slot
// of step t, entry n - 1 - t, is t mod A), read and cleared when its step
// comes; one to an entry further down is a fire-and-forget reduction into
// the entry's record, which the record's own load (issued at least A - D
// steps later in program order) sees.
template <int D, int A, int B>
__device__ __forceinline__ void tape_sweep(const TapeCtx& tc, size_t lane, int n0, int n, float* acc) {
  static_assert((D & (D - 1)) == 0 && (A & (A - 1)) == 0 && A > D, "windows of powers of two");
  const int steps = n - n0;
  const TapeRec* mine = tc.at(0, lane);
  float* my = acc + threadIdx.x;
#pragma unroll 4
  for (int u = 0; u < A; ++u) my[u * B] = 0.f;
  float w[D];
  unsigned ab[D];
  float2 dd[D];
#pragma unroll
  for (int u = 0; u < D; ++u) {
    w[u] = 0.f;
    ab[u] = 0xffffffffu;
    dd[u] = make_float2(0.f, 0.f);
    if (u < steps) {
      const uint4 r = __ldcg(mine + (n - 1 - u));
      ab[u] = r.x;
      dd[u] = make_float2(__uint_as_float(r.y), __uint_as_float(r.z));
      w[u] = __uint_as_float(r.w);
    }
  }
  auto give = [&](int t, unsigned a, float c) {
    if (a == 0xffffu || c == 0.f) return;
    const int ta = n - 1 - (int)a;
    if ((int)a >= n0 && ta < t + A) my[(ta & (A - 1)) * B] += c;
    else atomicAdd(tc.adj(a, lane), c);
  };
  for (int t0 = 0; t0 < steps; t0 += D) {
#pragma unroll
    for (int u = 0; u < D; ++u) {
      const int t = t0 + u;
      if (t < steps) {
        float* slot = my + (t & (A - 1)) * B;
        const float wv = w[u] + *slot;
        *slot = 0.f;
        const unsigned abv = ab[u];
        const float2 ddv = dd[u];
        if (t + D < steps) {
          const uint4 r = __ldcg(mine + (n - 1 - t - D));
          ab[u] = r.x;
          dd[u] = make_float2(__uint_as_float(r.y), __uint_as_float(r.z));
          w[u] = __uint_as_float(r.w);
        }
        if (wv != 0.f) {
          give(t, abv & 0xffffu, ddv.x * wv);
          give(t, abv >> 16, ddv.y * wv);
        }
      }
    }
  }
}

}  // namespace wrf
