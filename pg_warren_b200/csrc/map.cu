// map.cu — wc_vector_map: compute/map (vector_map) on the device.
//
// The reference evaluates its expression IR a chunk at a time, column by
// column, under a mask of the elements SQL would evaluate each node for
// (map/eval.rs); where an element fails, it evaluates the chunk again one
// element at a time and reports the first failing element's error
// (map/mod.rs:96-150).  An element's value and its first error are those of
// evaluating the tree for that element alone, children in order and lazy
// branches only where taken, which is what a thread does here: the host
// compiles the tree into a short stack program (jumps for CASE, COALESCE,
// AND and OR), checking every operand reference in the order the
// reference's evaluation visits them, and each thread runs the program for
// one element.  The first failing element is an atomic minimum of
// (position, status).
//
// Arithmetic and casts follow map/arithmetic.rs and compute/cast.rs bit for
// bit (SQL float overflow / underflow / division checks, checked bigint
// arithmetic, round-half-even); exp, ln, log and power call the device's
// functions, which are within 2 units in the last place of the host's.
#include <cmath>
#include <vector>

#include "operand.h"
#include "runtime.cuh"
#include "semiring.cuh"

namespace wc {

enum MapCode : uint8_t {
  I_LIT, I_NULL, I_VEC, I_CAST, I_NEG, I_ABS, I_ARITH, I_MOD, I_CALL, I_POW, I_CMP, I_NOT,
  I_JUMP, I_JIF_NOT_TRUE, I_JIF_NOT_NULL, I_CONN, I_CONN_STEP, I_NULLIF, I_EXTREME
};

struct MapIns {
  uint8_t code;
  uint8_t type;  // the result's wc_dtype (CMP: the operands'; CAST: the target)
  uint8_t sub;   // arithmetic / comparison / function; CONN: the stop value; EXTREME: greatest
  uint8_t from;  // CAST: the source type
  uint32_t target;  // jumps; EXTREME: the argument count
  int64_t i;
  double f;
};

constexpr int kMapStack = 32;
constexpr int kMapOperands = 16;

struct MapOperand {
  const void* p;
  int32_t dtype;
  uint32_t width;
};
struct MapOperands {
  MapOperand op[kMapOperands];
};

struct Val {
  union {
    double d;
    float f;
    long long i;
    int b;
  };
  int null;
};

// ------------------------------------------------------------ arithmetic

// map/arithmetic.rs:49-79 (float): a op b with Postgres's checks.
template <class F>
__device__ inline int32_t sql_arith(int op, F a, F b, F* o) {
  if (op == 3 && b == F(0) && !(a != a)) return WC_DIVISION_BY_ZERO;
  F r;
  switch (op) {
    case 0: r = a + b; break;
    case 1: r = a - b; break;
    case 2: r = a * b; break;
    default: r = a / b;
  }
  const bool finite_operands = op == 3 ? !isinf(a) : (!isinf(a) && !isinf(b));
  if (isinf(r) && finite_operands) return WC_FLOAT_OVERFLOW;
  const bool underflowed = op == 2 ? (a != F(0) && b != F(0))
                                   : (op == 3 ? (a != F(0) && !isinf(b)) : false);
  if (r == F(0) && underflowed) return WC_FLOAT_UNDERFLOW;
  *o = r;
  return 0;
}

// map/arithmetic.rs:83-110 (int, int_modulo).
__device__ inline int32_t int_arith(int op, long long a, long long b, long long* o) {
  if (op == 3) {
    if (b == 0) return WC_DIVISION_BY_ZERO;
    if (a == LLONG_MIN && b == -1) return WC_BIGINT_OUT_OF_RANGE;
    *o = a / b;
    return 0;
  }
  __int128 r;
  switch (op) {
    case 0: r = (__int128)a + b; break;
    case 1: r = (__int128)a - b; break;
    default: r = (__int128)a * b;
  }
  if (r > (__int128)LLONG_MAX || r < (__int128)LLONG_MIN) return WC_BIGINT_OUT_OF_RANGE;
  *o = (long long)r;
  return 0;
}

// A finite pow or exp result (arithmetic.rs:160-169).
__device__ inline int32_t checked_result(double r, double base, double* o) {
  if (isinf(r)) return WC_FLOAT_OVERFLOW;
  if (r == 0.0 && base != 0.0) return WC_FLOAT_UNDERFLOW;
  *o = r;
  return 0;
}

// arithmetic.rs:116-157 (call).
__device__ inline int32_t f64_call(int fn, double a, double* o) {
  switch (fn) {
    case 0: *o = fabs(a); return 0;
    case 1:
      if (a < 0.0) return WC_SQRT_OF_NEGATIVE;
      *o = sqrt(a);
      return 0;
    case 2:
      if (a != a) { *o = a; return 0; }
      if (isinf(a)) { *o = a > 0.0 ? a : 0.0; return 0; }
      return checked_result(exp(a), a, o);
    case 3: case 4:
      if (a == 0.0) return WC_LOG_OF_ZERO;
      if (a < 0.0) return WC_LOG_OF_NEGATIVE;
      *o = fn == 3 ? log(a) : log10(a);
      return 0;
    case 5: *o = floor(a); return 0;
    case 6: *o = ceil(a); return 0;
    case 7: *o = rint(a); return 0;  // half to even
    default: *o = a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : 0.0); return 0;
  }
}

// arithmetic.rs:171-218 (power).
__device__ inline int32_t f64_power(double a, double b, double* o) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  if (a != a) { *o = (b != b || b != 0.0) ? nan : 1.0; return 0; }
  if (b != b) { *o = a != 1.0 ? nan : 1.0; return 0; }
  if (a == 0.0 && b < 0.0) return WC_ZERO_TO_NEGATIVE_POWER;
  if (a < 0.0 && floor(b) != b) return WC_COMPLEX_POWER;
  if (isinf(b)) {
    const double mag = fabs(a);
    if (mag == 1.0) *o = 1.0;
    else if ((b > 0.0) == (mag > 1.0)) *o = __longlong_as_double(0x7ff0000000000000ll);
    else *o = 0.0;
    return 0;
  }
  if (isinf(a)) {
    if (b == 0.0) { *o = 1.0; return 0; }
    if (a > 0.0) { *o = b > 0.0 ? a : 0.0; return 0; }
    const double half = b / 2.0;
    const bool odd = floor(half) != half;
    if (b > 0.0) *o = odd ? a : -a;
    else *o = odd ? -0.0 : 0.0;
    return 0;
  }
  return checked_result(pow(a, b), a, o);
}

// compute/cast.rs: `from` to `to`.
__device__ inline int32_t sql_cast(int from, int to, const Val& v, Val* o) {
  o->null = 0;
  double d = 0.0;  // the source as a double, for the float sources
  switch (from) {
    case WC_F64: d = v.d; break;
    case WC_F32: d = (double)v.f; break;
    default: break;
  }
  switch (to) {
    case WC_F64:
      if (from == WC_I64) o->d = (double)v.i;
      else if (from == WC_BOOL) o->d = v.b ? 1.0 : 0.0;
      else o->d = d;
      return 0;
    case WC_F32:
      if (from == WC_I64) { o->f = (float)v.i; return 0; }
      if (from == WC_BOOL) { o->f = v.b ? 1.0f : 0.0f; return 0; }
      if (from == WC_F32) { o->f = v.f; return 0; }
      {
        const float narrowed = (float)d;  // float4_from_float8 (cast.rs:38-47)
        if (isinf(narrowed) && !isinf(d)) return WC_FLOAT_OVERFLOW;
        if (narrowed == 0.0f && d != 0.0) return WC_FLOAT_UNDERFLOW;
        o->f = narrowed;
        return 0;
      }
    case WC_I64:
      if (from == WC_I64) { o->i = v.i; return 0; }
      if (from == WC_BOOL) { o->i = v.b ? 1 : 0; return 0; }
      {
        const double r = rint(d);  // int8_from_float8 (cast.rs:49-56)
        if (!(r >= -9223372036854775808.0 && r < 9223372036854775808.0))
          return WC_BIGINT_OUT_OF_RANGE;
        o->i = (long long)r;
        return 0;
      }
    default:
      if (from == WC_I64) o->b = v.i != 0;
      else if (from == WC_BOOL) o->b = v.b;
      else o->b = d != 0.0;  // NaN is true
      return 0;
  }
}

// SQL order of two values of `type` (NaN above every number and equal to
// itself; -0 equals 0).
__device__ inline int val_cmp(int type, const Val& a, const Val& b) {
  switch (type) {
    case WC_F64: return sql_cmp_f(a.d, b.d);
    case WC_F32: return sql_cmp_f(a.f, b.f);
    case WC_I64: return a.i < b.i ? -1 : (a.i > b.i ? 1 : 0);
    default: return (a.b != 0) - (b.b != 0);
  }
}

__device__ inline Val load_operand(const MapOperand& m, uint64_t p, uint64_t row) {
  const uint64_t i = m.width == 1 ? row : p;
  Val v;
  v.null = 0;
  switch (m.dtype) {
    case WC_F64: v.d = static_cast<const double*>(m.p)[i]; break;
    case WC_F32: v.f = static_cast<const float*>(m.p)[i]; break;
    case WC_I64: v.i = static_cast<const long long*>(m.p)[i]; break;
    default: v.b = static_cast<const uint8_t*>(m.p)[i] != 0;
  }
  return v;
}

// The program for element p (row `row`): 0 and the value, or the status of
// its first error.
__device__ int32_t map_element(const MapIns* prog, uint32_t len, const MapOperands& ops,
                               uint64_t p, uint64_t row, Val* out) {
  Val st[kMapStack];
  int sp = 0;
  for (uint32_t pc = 0; pc < len;) {
    const MapIns in = prog[pc++];
    int32_t e = 0;
    switch (in.code) {
      case I_LIT: {
        Val v;
        v.null = 0;
        if (in.type == WC_F64) v.d = in.f;
        else if (in.type == WC_F32) v.f = (float)in.f;
        else if (in.type == WC_I64) v.i = in.i;
        else v.b = in.i != 0;
        st[sp++] = v;
        break;
      }
      case I_NULL: {
        Val v;
        v.i = 0;
        v.null = 1;
        st[sp++] = v;
        break;
      }
      case I_VEC: st[sp++] = load_operand(ops.op[in.i], p, row); break;
      case I_CAST:
        if (!st[sp - 1].null) e = sql_cast(in.from, in.type, st[sp - 1], &st[sp - 1]);
        break;
      case I_NEG: {
        Val& a = st[sp - 1];
        if (a.null) break;
        if (in.type == WC_F64) a.d = -a.d;
        else if (in.type == WC_F32) a.f = -a.f;
        else if (a.i == LLONG_MIN) e = WC_BIGINT_OUT_OF_RANGE;
        else a.i = -a.i;
        break;
      }
      case I_ABS: {
        Val& a = st[sp - 1];
        if (a.null) break;
        if (in.type == WC_F64) a.d = fabs(a.d);
        else if (in.type == WC_F32) a.f = fabsf(a.f);
        else if (a.i == LLONG_MIN) e = WC_BIGINT_OUT_OF_RANGE;
        else a.i = a.i < 0 ? -a.i : a.i;
        break;
      }
      case I_CALL: {
        Val& a = st[sp - 1];
        if (!a.null) e = f64_call(in.sub, a.d, &a.d);
        break;
      }
      case I_ARITH: case I_MOD: case I_POW: case I_CMP: {
        const Val b = st[--sp];
        Val& a = st[sp - 1];
        if (a.null || b.null) {
          a.null = 1;
          break;
        }
        if (in.code == I_CMP) {
          const int c = val_cmp(in.type, a, b);
          bool r;
          switch (in.sub) {
            case 0: r = c == 0; break;
            case 1: r = c != 0; break;
            case 2: r = c < 0; break;
            case 3: r = c <= 0; break;
            case 4: r = c > 0; break;
            default: r = c >= 0;
          }
          a.b = r;
        } else if (in.code == I_POW) {
          e = f64_power(a.d, b.d, &a.d);
        } else if (in.code == I_MOD) {
          if (b.i == 0) e = WC_DIVISION_BY_ZERO;
          else a.i = b.i == -1 ? 0 : a.i % b.i;
        } else if (in.type == WC_F64) {
          e = sql_arith<double>(in.sub, a.d, b.d, &a.d);
        } else if (in.type == WC_F32) {
          e = sql_arith<float>(in.sub, a.f, b.f, &a.f);
        } else {
          e = int_arith(in.sub, a.i, b.i, &a.i);
        }
        break;
      }
      case I_NOT:
        if (!st[sp - 1].null) st[sp - 1].b = !st[sp - 1].b;
        break;
      case I_JUMP: pc = in.target; break;
      case I_JIF_NOT_TRUE: {
        const Val c = st[--sp];
        if (c.null || !c.b) pc = in.target;
        break;
      }
      case I_JIF_NOT_NULL:
        if (!st[sp - 1].null) pc = in.target;
        else sp--;
        break;
      case I_CONN: {
        Val v;
        v.i = 0;
        v.b = !in.sub;
        v.null = 0;
        st[sp++] = v;
        break;
      }
      case I_CONN_STEP: {
        const Val v = st[--sp];
        Val& acc = st[sp - 1];
        if (v.null) {
          acc.null = 1;
        } else if ((v.b != 0) == (in.sub != 0)) {
          acc.b = in.sub;
          acc.null = 0;
          pc = in.target;
        }
        break;
      }
      case I_NULLIF: {
        const Val b = st[--sp];
        Val& a = st[sp - 1];
        if (!a.null && !b.null && val_cmp(in.type, a, b) == 0) a.null = 1;
        break;
      }
      case I_EXTREME: {
        const int n = (int)in.target;
        Val best;
        best.i = 0;
        best.null = 1;
        for (int j = 0; j < n; j++) {
          const Val& v = st[sp - n + j];
          if (v.null) continue;
          const int c = best.null ? 0 : val_cmp(in.type, v, best);
          if (best.null || (in.sub ? c > 0 : c < 0)) best = v;
        }
        sp -= n;
        st[sp++] = best;
        break;
      }
    }
    if (e) return e;
  }
  *out = st[0];
  return 0;
}

__global__ void __launch_bounds__(256) map_kernel(const MapIns* prog, uint32_t len,
                                                  MapOperands ops, uint64_t total, uint32_t width,
                                                  int32_t out_type, void* out,
                                                  unsigned long long* first_error) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < total;
       p += (uint64_t)gridDim.x * blockDim.x) {
    Val v;
    int32_t e = map_element(prog, len, ops, p, p / width, &v);
    if (!e) {
      switch (out_type) {
        case WC_F64:
          static_cast<double*>(out)[p] = v.null ? __longlong_as_double(0x7ff8000000000000ll) : v.d;
          break;
        case WC_F32:
          static_cast<float*>(out)[p] = v.null ? __int_as_float(0x7fc00000) : v.f;
          break;
        case WC_I64:
          if (v.null) e = WC_NULL_RESULT;
          else static_cast<long long*>(out)[p] = v.i;
          break;
        default:
          if (v.null) e = WC_NULL_RESULT;
          else static_cast<uint8_t*>(out)[p] = v.b ? 1 : 0;
      }
    }
    if (e) atomicMin(first_error, (unsigned long long)(p << 8) | (unsigned long long)e);
  }
}

// ------------------------------------------------------------ the compiler

struct MapCompiler {
  const wc_map_node* nodes;
  uint32_t node_count;
  const uint32_t* children;
  uint32_t child_count;
  const wc_dtype* operand_dtypes;
  uint32_t operand_count;
  wc_error_detail* detail;
  std::vector<MapIns> prog;
  int depth = 0, max_depth = 0;

  void emit(MapIns in, int effect) {
    prog.push_back(in);
    depth += effect;
    max_depth = std::max(max_depth, depth);
  }
  static MapIns ins(uint8_t code, int type, int sub = 0) {
    MapIns in{};
    in.code = code;
    in.type = (uint8_t)type;
    in.sub = (uint8_t)sub;
    return in;
  }
  wc_status child(const wc_map_node& n, uint32_t k, uint32_t* out) {
    if (k >= n.count || (uint64_t)n.first + k >= child_count) return WC_INVALID_ARGUMENT;
    *out = children[n.first + k];
    return *out < node_count ? WC_OK : WC_INVALID_ARGUMENT;
  }
  // Compiles node `id` (of `type`, or any type if -1) with the operand
  // references checked in the reference's visiting order.
  wc_status node(uint32_t id, int type, int nesting) {
    if (nesting > 512 || id >= node_count) return WC_INVALID_ARGUMENT;
    const wc_map_node& n = nodes[id];
    if (n.type < WC_F32 || n.type > WC_BOOL || (type >= 0 && n.type != type))
      return WC_INVALID_ARGUMENT;
    const int t = n.type;
    uint32_t a = 0, b = 0;
    switch (n.kind) {
      case WC_MAP_LITERAL: {
        MapIns in = ins(n.is_null ? I_NULL : I_LIT, t);
        in.i = n.i;
        in.f = n.f;
        emit(in, 1);
        return WC_OK;
      }
      case WC_MAP_VECTOR: {
        if (n.i < 0 || (uint64_t)n.i >= operand_count) {
          if (detail) detail->node = (uint64_t)n.i, detail->expected = operand_count;
          set_message(detail, "expression refers to operand %lld, but %u were given",
                      (long long)n.i, operand_count);
          return WC_UNKNOWN_OPERAND;
        }
        if (operand_dtypes[n.i] != t) {
          if (detail)
            detail->node = (uint64_t)n.i, detail->expected = t, detail->found = operand_dtypes[n.i];
          set_message(detail, "expression reads operand %lld as dtype %d, but it is %d",
                      (long long)n.i, t, operand_dtypes[n.i]);
          return WC_OPERAND_TYPE;
        }
        MapIns in = ins(I_VEC, t);
        in.i = n.i;
        emit(in, 1);
        return WC_OK;
      }
      case WC_MAP_CAST: {
        WC_TRY(child(n, 0, &a));
        WC_TRY(node(a, -1, nesting + 1));
        MapIns in = ins(I_CAST, t);
        in.from = (uint8_t)nodes[a].type;
        emit(in, 0);
        return WC_OK;
      }
      case WC_MAP_CASE: {
        // condition, JIF_NOT_TRUE next; value; JUMP end; next: ...; else
        const uint32_t pairs = (n.count - (n.has_else ? 1 : 0)) / 2;
        if (n.count < (n.has_else ? 1u : 0u) || pairs * 2 + (n.has_else ? 1 : 0) != n.count)
          return WC_INVALID_ARGUMENT;
        std::vector<size_t> ends;
        const int base = depth;
        for (uint32_t q = 0; q < pairs; q++) {
          WC_TRY(child(n, 2 * q, &a));
          WC_TRY(child(n, 2 * q + 1, &b));
          WC_TRY(node(a, WC_BOOL, nesting + 1));
          const size_t jif = prog.size();
          emit(ins(I_JIF_NOT_TRUE, WC_BOOL), -1);
          WC_TRY(node(b, t, nesting + 1));
          ends.push_back(prog.size());
          emit(ins(I_JUMP, t), 0);
          depth = base;
          prog[jif].target = (uint32_t)prog.size();
        }
        if (n.has_else) {
          WC_TRY(child(n, n.count - 1, &a));
          WC_TRY(node(a, t, nesting + 1));
        } else {
          emit(ins(I_NULL, t), 1);
        }
        for (size_t j : ends) prog[j].target = (uint32_t)prog.size();
        return WC_OK;
      }
      case WC_MAP_NULLIF: {
        WC_TRY(child(n, 0, &a));
        WC_TRY(child(n, 1, &b));
        WC_TRY(node(a, t, nesting + 1));
        WC_TRY(node(b, t, nesting + 1));
        emit(ins(I_NULLIF, t), -1);
        return WC_OK;
      }
      case WC_MAP_COALESCE: {
        if (n.count == 0) {
          emit(ins(I_NULL, t), 1);
          return WC_OK;
        }
        std::vector<size_t> ends;
        for (uint32_t q = 0; q < n.count; q++) {
          WC_TRY(child(n, q, &a));
          WC_TRY(node(a, t, nesting + 1));
          if (q + 1 < n.count) {
            ends.push_back(prog.size());
            emit(ins(I_JIF_NOT_NULL, t), -1);  // the fall-through pops
          }
        }
        for (size_t j : ends) prog[j].target = (uint32_t)prog.size();
        return WC_OK;
      }
      case WC_MAP_LEAST: case WC_MAP_GREATEST: {
        if (n.count == 0) {
          emit(ins(I_NULL, t), 1);
          return WC_OK;
        }
        for (uint32_t q = 0; q < n.count; q++) {
          WC_TRY(child(n, q, &a));
          WC_TRY(node(a, t, nesting + 1));
        }
        MapIns in = ins(I_EXTREME, t, n.kind == WC_MAP_GREATEST);
        in.target = n.count;
        emit(in, 1 - (int)n.count);
        return WC_OK;
      }
      case WC_MAP_NEGATE: case WC_MAP_ABS: {
        if (t == WC_BOOL || (n.kind == WC_MAP_ABS && t == WC_F64)) return WC_INVALID_ARGUMENT;
        WC_TRY(child(n, 0, &a));
        WC_TRY(node(a, t, nesting + 1));
        emit(ins(n.kind == WC_MAP_NEGATE ? I_NEG : I_ABS, t), 0);
        return WC_OK;
      }
      case WC_MAP_CALL: {
        if (t != WC_F64 || n.op < 0 || n.op > 8) return WC_INVALID_ARGUMENT;
        WC_TRY(child(n, 0, &a));
        WC_TRY(node(a, t, nesting + 1));
        emit(ins(I_CALL, t, n.op), 0);
        return WC_OK;
      }
      case WC_MAP_ARITHMETIC: case WC_MAP_MODULO: case WC_MAP_POWER: case WC_MAP_COMPARE: {
        const bool cmp = n.kind == WC_MAP_COMPARE;
        if (cmp ? (t != WC_BOOL || n.op < 0 || n.op > 5) : false) return WC_INVALID_ARGUMENT;
        if (n.kind == WC_MAP_ARITHMETIC && (t == WC_BOOL || n.op < 0 || n.op > 3))
          return WC_INVALID_ARGUMENT;
        if (n.kind == WC_MAP_MODULO && t != WC_I64) return WC_INVALID_ARGUMENT;
        if (n.kind == WC_MAP_POWER && t != WC_F64) return WC_INVALID_ARGUMENT;
        WC_TRY(child(n, 0, &a));
        WC_TRY(child(n, 1, &b));
        const int operand_type = cmp ? nodes[a].type : t;
        WC_TRY(node(a, operand_type, nesting + 1));
        WC_TRY(node(b, operand_type, nesting + 1));
        const uint8_t code = cmp ? I_CMP : n.kind == WC_MAP_MODULO ? I_MOD
                             : n.kind == WC_MAP_POWER ? I_POW : I_ARITH;
        emit(ins(code, operand_type, n.op), -1);
        return WC_OK;
      }
      case WC_MAP_NOT: {
        if (t != WC_BOOL) return WC_INVALID_ARGUMENT;
        WC_TRY(child(n, 0, &a));
        WC_TRY(node(a, WC_BOOL, nesting + 1));
        emit(ins(I_NOT, t), 0);
        return WC_OK;
      }
      case WC_MAP_AND: case WC_MAP_OR: {
        if (t != WC_BOOL) return WC_INVALID_ARGUMENT;
        const int stop = n.kind == WC_MAP_OR;
        emit(ins(I_CONN, t, stop), 1);
        std::vector<size_t> steps;
        for (uint32_t q = 0; q < n.count; q++) {
          WC_TRY(child(n, q, &a));
          WC_TRY(node(a, WC_BOOL, nesting + 1));
          steps.push_back(prog.size());
          emit(ins(I_CONN_STEP, t, stop), -1);
        }
        for (size_t j : steps) prog[j].target = (uint32_t)prog.size();
        return WC_OK;
      }
      default: return WC_INVALID_ARGUMENT;
    }
  }
};

static uint32_t dtype_bytes(int32_t dtype) {
  switch (dtype) {
    case WC_F64: case WC_I64: return 8;
    case WC_F32: return 4;
    case WC_BOOL: return 1;
    default: return 0;
  }
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_vector_map(wc_version* v, const wc_call* call, const wc_map_node* nodes,
                        uint32_t node_count, const uint32_t* children, uint32_t child_count,
                        uint32_t root, const void* const* operands, const wc_dtype* operand_dtypes,
                        const uint64_t* operand_id_spaces, const uint32_t* operand_widths,
                        uint32_t operand_count, void* out, uint32_t* out_width) {
  wc_error_detail* d = call ? call->detail : nullptr;
  if (!v || !nodes || root >= node_count || (child_count && !children) ||
      (operand_count && (!operands || !operand_dtypes || !operand_id_spaces || !operand_widths)))
    return WC_INVALID_ARGUMENT;
  // map/mod.rs:57-71: the widest operand's width; every operand over the id
  // space, of width 1 or that width.
  uint32_t width = 1;
  for (uint32_t q = 0; q < operand_count; q++) width = std::max(width, operand_widths[q]);
  for (uint32_t q = 0; q < operand_count; q++) {
    if (!dtype_bytes(operand_dtypes[q])) return WC_INVALID_ARGUMENT;
    if (operand_id_spaces[q] != v->n) {
      if (d) d->expected = v->n, d->found = operand_id_spaces[q];
      return WC_ID_SPACE_MISMATCH;
    }
    if (operand_widths[q] != 1 && operand_widths[q] != width) {
      if (d) d->expected = width, d->found = operand_widths[q];
      return WC_WIDTH_MISMATCH;
    }
  }
  MapCompiler comp{nodes, node_count, children, child_count, operand_dtypes, operand_count, d};
  WC_TRY(comp.node(root, -1, 0));
  if (comp.max_depth > kMapStack || operand_count > (uint32_t)kMapOperands) {
    set_message(d, "expressions are served up to %d stack values and %d operands", kMapStack,
                kMapOperands);
    return WC_UNSUPPORTED;
  }
  const int32_t out_type = nodes[root].type;
  if (out_width) *out_width = width;
  if (!out && v->n) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), d);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  const uint64_t total = v->n * width;
  if (total == 0) return ctx.finish();
  DevBuf *pb, *eb;
  WC_TRY(ctx.scratch(POOL_MAP_PROGRAM, comp.prog.size() * sizeof(MapIns), &pb));
  WC_TRY(ctx.scratch(POOL_MAP_ERROR, 8, &eb));
  WC_CUDA(cudaMemcpyAsync(pb->ptr, comp.prog.data(), comp.prog.size() * sizeof(MapIns),
                          cudaMemcpyHostToDevice, ctx.stream), ctx.detail);
  WC_CUDA(cudaMemsetAsync(eb->ptr, 0xff, 8, ctx.stream), ctx.detail);
  MapOperands ops{};
  Operand staged[kMapOperands] = {Operand(POOL_MAP_OPERAND_0), Operand(POOL_MAP_OPERAND_0 + 1),
                                  Operand(POOL_MAP_OPERAND_0 + 2), Operand(POOL_MAP_OPERAND_0 + 3),
                                  Operand(POOL_MAP_OPERAND_0 + 4), Operand(POOL_MAP_OPERAND_0 + 5),
                                  Operand(POOL_MAP_OPERAND_0 + 6), Operand(POOL_MAP_OPERAND_0 + 7),
                                  Operand(POOL_MAP_OPERAND_0 + 8), Operand(POOL_MAP_OPERAND_0 + 9),
                                  Operand(POOL_MAP_OPERAND_0 + 10), Operand(POOL_MAP_OPERAND_0 + 11),
                                  Operand(POOL_MAP_OPERAND_0 + 12), Operand(POOL_MAP_OPERAND_0 + 13),
                                  Operand(POOL_MAP_OPERAND_0 + 14), Operand(POOL_MAP_OPERAND_0 + 15)};
  for (uint32_t q = 0; q < operand_count; q++) {
    WC_TRY(staged[q].in(ctx, operands[q],
                        v->n * operand_widths[q] * dtype_bytes(operand_dtypes[q])));
    ops.op[q] = MapOperand{staged[q].dev, operand_dtypes[q], operand_widths[q]};
  }
  Operand O(POOL_MAP_OUT);
  WC_TRY(O.output(ctx, out, total * dtype_bytes(out_type)));
  const uint32_t grid = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(max_blocks(8), (total + 255) / 256));
  note_launch(), map_kernel<<<grid, 256, 0, ctx.stream>>>(
      pb->as<MapIns>(), (uint32_t)comp.prog.size(), ops, total, width, out_type, O.dev,
      eb->as<unsigned long long>());
  unsigned long long first = 0;
  WC_CUDA(cudaMemcpyAsync(&first, eb->ptr, 8, cudaMemcpyDeviceToHost, ctx.stream), ctx.detail);
  WC_TRY(ctx.finish());
  if (first != ~0ull) {
    const wc_status e = (wc_status)(first & 0xff);
    if (d) {
      d->node = first >> 8;
      if (e == WC_NULL_RESULT) d->expected = out_type;
    }
    return e;
  }
  WC_TRY(O.out(ctx));
  return ctx.finish();
}

}  // extern "C"
