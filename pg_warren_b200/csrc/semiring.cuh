// semiring.cuh — the reference's element semantics on the device.
//
// compute/semiring.rs:15-388 (BinaryOp, Monoid, SemiringElement for f64,
// f32, i64 and bool), compute/cast.rs:42-64 (weight casts) and
// compute/dtype.rs:69-160 (SQL order: NaN above every number, ties keep the
// first operand), as device functions specialised at compile time per
// semiring, as the reference's `specialised!` macro specialises its inner
// loops (compute/product/kernel.rs:50-70).  A failing operation returns a
// wc_status instead of aborting; kernels raise it in the call's error word.
#pragma once

#include <cstdint>

#include "../../include/warren_cuda.h"
#include "runtime.cuh"

namespace wc {

typedef unsigned char bool8;  // the bool dtype: one byte, 0 or 1

__host__ __device__ inline int sql_cmp_f(double a, double b) {
  bool an = a != a, bn = b != b;
  if (an && bn) return 0;
  if (an) return 1;
  if (bn) return -1;
  return a < b ? -1 : (a > b ? 1 : 0);
}

template <class E> struct Elem;

template <> struct Elem<double> {
  __device__ static int cmp(double a, double b) { return sql_cmp_f(a, b); }
  __device__ static bool nonzero(double a) { return a != 0.0; }
  __device__ static int32_t from_weight(double w, double* o) { *o = w; return 0; }
};
template <> struct Elem<float> {
  __device__ static int cmp(float a, float b) { return sql_cmp_f(a, b); }
  __device__ static bool nonzero(float a) { return a != 0.0f; }
  // float8 -> float4: an error rather than a silent infinity or zero.
  __device__ static int32_t from_weight(double w, float* o) {
    float n = (float)w;
    if (isinf(n) && !isinf(w)) return WC_FLOAT_OVERFLOW;
    if (n == 0.0f && w != 0.0) return WC_FLOAT_UNDERFLOW;
    *o = n;
    return 0;
  }
};
template <> struct Elem<int64_t> {
  __device__ static int cmp(int64_t a, int64_t b) { return a < b ? -1 : (a > b ? 1 : 0); }
  __device__ static bool nonzero(int64_t a) { return a != 0; }
  // float8 -> int8: round half to even, then range-check.
  __device__ static int32_t from_weight(double w, int64_t* o) {
    double r = rint(w);
    if (!(r >= -9223372036854775808.0 && r < 9223372036854775808.0)) return WC_BIGINT_OUT_OF_RANGE;
    *o = (int64_t)r;
    return 0;
  }
};
template <> struct Elem<bool8> {
  __device__ static int cmp(bool8 a, bool8 b) { return (int)(a != 0) - (int)(b != 0); }
  __device__ static bool nonzero(bool8 a) { return a != 0; }
  __device__ static int32_t from_weight(double w, bool8* o) { *o = w != 0.0; return 0; }
};

template <class E> __device__ inline E least(E a, E b) { return Elem<E>::cmp(b, a) < 0 ? b : a; }
template <class E> __device__ inline E greatest(E a, E b) { return Elem<E>::cmp(b, a) > 0 ? b : a; }

__device__ inline bool fnz(double a) { return a != 0.0 || a != a; }

// BinaryOp::apply (semiring.rs:283-295, 317-329, 371-378).
template <class E, int OP> struct Apply;

template <int OP> struct Apply<double, OP> {
  __device__ static int32_t go(double a, double b, double* o) {
    switch (OP) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = a; break;
      case WC_OP_SECOND: *o = b; break;
      case WC_OP_PAIR: *o = 1.0; break;
      case WC_OP_PLUS: *o = a + b; break;
      case WC_OP_TIMES: *o = a * b; break;
      case WC_OP_MIN: *o = least(a, b); break;
      case WC_OP_MAX: *o = greatest(a, b); break;
      case WC_OP_LOR: *o = (fnz(a) || fnz(b)) ? 1.0 : 0.0; break;
      case WC_OP_LAND: *o = (fnz(a) && fnz(b)) ? 1.0 : 0.0; break;
    }
    return 0;
  }
};
template <int OP> struct Apply<float, OP> {
  __device__ static int32_t go(float a, float b, float* o) {
    switch (OP) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = a; break;
      case WC_OP_SECOND: *o = b; break;
      case WC_OP_PAIR: *o = 1.0f; break;
      case WC_OP_PLUS: *o = a + b; break;
      case WC_OP_TIMES: *o = a * b; break;
      case WC_OP_MIN: *o = least(a, b); break;
      case WC_OP_MAX: *o = greatest(a, b); break;
      case WC_OP_LOR: *o = (fnz(a) || fnz(b)) ? 1.0f : 0.0f; break;
      case WC_OP_LAND: *o = (fnz(a) && fnz(b)) ? 1.0f : 0.0f; break;
    }
    return 0;
  }
};
template <int OP> struct Apply<int64_t, OP> {
  __device__ static int32_t go(int64_t a, int64_t b, int64_t* o) {
    switch (OP) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = a; break;
      case WC_OP_SECOND: *o = b; break;
      case WC_OP_PAIR: *o = 1; break;
      case WC_OP_PLUS: {  // checked_add
        long long r = (long long)((unsigned long long)a + (unsigned long long)b);
        if (((a ^ r) & (b ^ r)) < 0) return WC_BIGINT_OUT_OF_RANGE;
        *o = r;
        break;
      }
      case WC_OP_TIMES: {  // checked_mul: the 128-bit product must fit 64 bits
        long long lo = (long long)((unsigned long long)a * (unsigned long long)b);
        long long hi = __mul64hi((long long)a, (long long)b);
        if (hi != (lo >> 63)) return WC_BIGINT_OUT_OF_RANGE;
        *o = lo;
        break;
      }
      case WC_OP_MIN: *o = a < b ? a : b; break;
      case WC_OP_MAX: *o = a > b ? a : b; break;
      case WC_OP_LOR: *o = (a != 0 || b != 0); break;
      case WC_OP_LAND: *o = (a != 0 && b != 0); break;
    }
    return 0;
  }
};
template <int OP> struct Apply<bool8, OP> {
  __device__ static int32_t go(bool8 a, bool8 b, bool8* o) {
    bool x = a != 0, y = b != 0;
    switch (OP) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = x; break;
      case WC_OP_SECOND: *o = y; break;
      case WC_OP_PAIR: *o = 1; break;
      case WC_OP_PLUS: case WC_OP_MAX: case WC_OP_LOR: *o = x || y; break;
      default: *o = x && y; break;
    }
    return 0;
  }
};

// The same with the operator chosen at run time (accumulators).
template <class E> __device__ inline int32_t apply_rt(int op, E a, E b, E* o) {
  switch (op) {
    case WC_OP_FIRST: return Apply<E, WC_OP_FIRST>::go(a, b, o);
    case WC_OP_SECOND: return Apply<E, WC_OP_SECOND>::go(a, b, o);
    case WC_OP_PAIR: return Apply<E, WC_OP_PAIR>::go(a, b, o);
    case WC_OP_PLUS: return Apply<E, WC_OP_PLUS>::go(a, b, o);
    case WC_OP_TIMES: return Apply<E, WC_OP_TIMES>::go(a, b, o);
    case WC_OP_MIN: return Apply<E, WC_OP_MIN>::go(a, b, o);
    case WC_OP_MAX: return Apply<E, WC_OP_MAX>::go(a, b, o);
    case WC_OP_LOR: return Apply<E, WC_OP_LOR>::go(a, b, o);
    case WC_OP_LAND: return Apply<E, WC_OP_LAND>::go(a, b, o);
    default: return Apply<E, WC_OP_ANY>::go(a, b, o);
  }
}

// Monoid identities (semiring.rs:298-304, 332-338, 381-383).
template <class E> struct Identity;
template <> struct Identity<double> {
  __host__ __device__ static double of(int m) {
    return m == WC_OP_MIN ? (double)INFINITY : (m == WC_OP_MAX ? -(double)INFINITY : 0.0);
  }
};
template <> struct Identity<float> {
  __host__ __device__ static float of(int m) {
    return m == WC_OP_MIN ? INFINITY : (m == WC_OP_MAX ? -INFINITY : 0.0f);
  }
};
template <> struct Identity<int64_t> {
  __host__ __device__ static int64_t of(int m) {
    return m == WC_OP_MIN ? INT64_MAX : (m == WC_OP_MAX ? INT64_MIN : 0);
  }
};
template <> struct Identity<bool8> {
  __host__ __device__ static bool8 of(int m) { return m == WC_OP_MIN ? 1 : 0; }
};

// The ⊕ and ⊗ of each semiring (semiring.rs:170-191).
__host__ __device__ constexpr int semiring_add(int s) {
  return (s == WC_PLUS_TIMES || s == WC_PLUS_PAIR || s == WC_PLUS_FIRST || s == WC_PLUS_SECOND)
             ? WC_OP_PLUS
             : (s == WC_MIN_PLUS || s == WC_MIN_TIMES || s == WC_MIN_FIRST || s == WC_MIN_SECOND)
                   ? WC_OP_MIN
                   : (s == WC_MAX_PLUS || s == WC_MAX_TIMES || s == WC_MAX_SECOND)
                         ? WC_OP_MAX
                         : (s == WC_LOR_LAND ? WC_OP_LOR : WC_OP_ANY);
}
__host__ __device__ constexpr int semiring_mul(int s) {
  return (s == WC_PLUS_TIMES || s == WC_MAX_TIMES || s == WC_MIN_TIMES)
             ? WC_OP_TIMES
             : (s == WC_MIN_PLUS || s == WC_MAX_PLUS)
                   ? WC_OP_PLUS
                   : (s == WC_LOR_LAND)
                         ? WC_OP_LAND
                         : (s == WC_ANY_PAIR || s == WC_PLUS_PAIR)
                               ? WC_OP_PAIR
                               : (s == WC_PLUS_FIRST || s == WC_MIN_FIRST) ? WC_OP_FIRST
                                                                           : WC_OP_SECOND;
}

// ⊗(weight, value) in a semiring whose ⊕ is ADD (semiring.rs:254-261,
// 340-363): for i64 the min identity MAX and the max identity MIN stand for
// ±∞ and absorb plus, and times by a weight above zero.
template <class E, int ADD, int MUL> struct Multiply {
  __device__ static int32_t go(E w, E v, E* o) { return Apply<E, MUL>::go(w, v, o); }
};
template <int ADD, int MUL> struct Multiply<int64_t, ADD, MUL> {
  __device__ static int32_t go(int64_t w, int64_t v, int64_t* o) {
    bool infinite = (ADD == WC_OP_MIN && v == INT64_MAX) || (ADD == WC_OP_MAX && v == INT64_MIN);
    bool absorbs = MUL == WC_OP_PLUS || (MUL == WC_OP_TIMES && w > 0);
    if (infinite && absorbs) {
      *o = v;
      return 0;
    }
    return Apply<int64_t, MUL>::go(w, v, o);
  }
};

// The product of one entry (product/kernel.rs:39-47): the weight is cast
// only if ⊗ reads it.  `W` is the stored weight type: double (cast by
// from_weight), int32_t (the integral copy, exact for any element type) or
// void (unweighted: every weight 1).
template <class E, int SEMIRING, class W> struct Entry {
  static constexpr int ADD = semiring_add(SEMIRING);
  static constexpr int MUL = semiring_mul(SEMIRING);
  static constexpr bool reads_weight = MUL != WC_OP_SECOND && MUL != WC_OP_PAIR;
  __device__ static int32_t product(double w, E v, E* o) {
    E we{};
    if (reads_weight) {
      int32_t s = Elem<E>::from_weight(w, &we);
      if (s) return s;
    }
    return Multiply<E, ADD, MUL>::go(we, v, o);
  }
  __device__ static int32_t product_int(int32_t w, E v, E* o) {
    E we{};
    if (reads_weight) we = (E)w;
    return Multiply<E, ADD, MUL>::go(we, v, o);
  }
};

// Raises `status` in the call's error word: the first status wins.
__device__ inline void raise(DeviceError* e, int32_t status, uint64_t aux = 0) {
  if (status && atomicCAS(&e->status, 0, status) == 0) e->aux = aux;
}

// An accumulator for ⊕ that tree reductions combine in order (left operand
// first), so min / max with first-on-tie, lor, any, and i64 checked sums
// give what a sequential fold gives.  For i64 plus it tracks the range of
// every prefix sum in 128 bits, so an overflow anywhere in the sequential
// order is found whatever the tree's shape.
template <class E, int ADD> struct Acc {
  E v;
  __device__ static Acc of(E p) { return Acc{p}; }
  __device__ static Acc combine(Acc a, Acc b) {
    Acc r;
    Apply<E, ADD>::go(a.v, b.v, &r.v);
    return r;
  }
  __device__ int32_t value(E* o) const { *o = v; return 0; }
  __device__ Acc shfl_down(unsigned off) const {
    Acc r;
    r.v = shfl_down_e(v, off);
    return r;
  }
  __device__ static E shfl_down_e(E x, unsigned off);
};

template <class E, int ADD>
__device__ inline E Acc<E, ADD>::shfl_down_e(E x, unsigned off) {
  if constexpr (sizeof(E) == 8) {
    long long t;
    memcpy(&t, &x, 8);
    t = __shfl_down_sync(0xffffffffu, t, off);
    E r;
    memcpy(&r, &t, 8);
    return r;
  } else if constexpr (sizeof(E) == 4) {
    int t;
    memcpy(&t, &x, 4);
    t = __shfl_down_sync(0xffffffffu, t, off);
    E r;
    memcpy(&r, &t, 4);
    return r;
  } else {
    int t = (int)x;
    t = __shfl_down_sync(0xffffffffu, t, off);
    return (E)t;
  }
}

template <> struct Acc<int64_t, WC_OP_PLUS> {
  __int128 sum, lo, hi;
  __device__ static Acc of(int64_t p) { return Acc{p, p, p}; }
  __device__ static Acc combine(Acc a, Acc b) {
    Acc r;
    r.sum = a.sum + b.sum;
    __int128 l = a.sum + b.lo, h = a.sum + b.hi;
    r.lo = a.lo < l ? a.lo : l;
    r.hi = a.hi > h ? a.hi : h;
    return r;
  }
  __device__ int32_t value(int64_t* o) const {
    if (lo < (__int128)INT64_MIN || hi > (__int128)INT64_MAX) return WC_BIGINT_OUT_OF_RANGE;
    *o = (int64_t)sum;
    return 0;
  }
  __device__ static __int128 shfl128(__int128 x, unsigned off) {
    unsigned long long lo64 = (unsigned long long)x, hi64 = (unsigned long long)(x >> 64);
    lo64 = __shfl_down_sync(0xffffffffu, lo64, off);
    hi64 = __shfl_down_sync(0xffffffffu, hi64, off);
    return ((__int128)hi64 << 64) | (__int128)lo64;
  }
  __device__ Acc shfl_down(unsigned off) const {
    return Acc{shfl128(sum, off), shfl128(lo, off), shfl128(hi, off)};
  }
};

}  // namespace wc
