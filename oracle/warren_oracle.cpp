// warren_oracle.cpp — TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement, in C++, of the reference warren-core functions on the
// whole-graph compute path.  It is the checker the CUDA backend is compared
// against and the CPU baseline the benchmark times; nothing in the product
// links or calls it.  The reference (Rust, rayon) cannot be built here: no
// Rust toolchain, and its crates are not vendored.  So this file restates the
// algorithm of each cited file:line, keeping the reference's summation orders
// (sequential folds, 65536-element chunks combined in chunk order, ascending
// column order within a row) so that results are bit-identical to it.  It is
// pinned by the reference's own known-answer tests (tests/test_oracle_*.py).
//
// Exported entry points are `extern "C"` with the prefix `wo_` and reuse the
// status codes of include/warren_cuda.h.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <queue>
#include <array>
#include <thread>
#include <vector>

#include "../include/warren_cuda.h"

namespace {

using Status = int32_t;

// ------------------------------------------------------------- threading
// compute/workers.rs:37-143 runs tasks on a rayon pool; results never depend
// on the thread count (every reduction combines in task order), so a plain
// std::thread pool over the same task sizes stands in for it.

int g_threads = 0;

int threads() {
  if (g_threads > 0) return g_threads;
  unsigned hw = std::thread::hardware_concurrency();
  return hw ? (int)hw : 1;
}

// Runs body(task) for task in [0, tasks) on up to threads() threads.  The
// status of the lowest-numbered failing task is returned (deterministic).
Status parallel_tasks(size_t tasks, const std::function<Status(size_t)>& body) {
  int t = std::min<size_t>(threads(), std::max<size_t>(tasks, 1));
  std::vector<Status> first(tasks, WC_OK);
  if (t <= 1) {
    for (size_t i = 0; i < tasks; i++) {
      Status s = body(i);
      if (s != WC_OK) return s;
    }
    return WC_OK;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  for (int w = 0; w < t; w++)
    pool.emplace_back([&]() {
      for (;;) {
        size_t i = next.fetch_add(1);
        if (i >= tasks) break;
        first[i] = body(i);
      }
    });
  for (auto& th : pool) th.join();
  for (size_t i = 0; i < tasks; i++)
    if (first[i] != WC_OK) return first[i];
  return WC_OK;
}

// ------------------------------------------------------------- elements
// compute/dtype.rs:69-160: SQL order (NaN above every number, NaN == NaN),
// non-zero test (NaN is non-zero), as f64.

template <class E> struct El;

inline int float_cmp(double a, double b) {
  bool an = std::isnan(a), bn = std::isnan(b);
  if (an && bn) return 0;
  if (an) return 1;
  if (bn) return -1;
  return a < b ? -1 : (a > b ? 1 : 0);
}

// map/arithmetic.rs:49-79: float8 operators with SQL's errors.
enum Arith { ADD, SUB, MUL, DIV };
template <class F> Status sql_float(Arith op, F a, F b, F* out) {
  if (op == DIV && b == F(0) && !std::isnan(a)) return WC_DIVISION_BY_ZERO;
  F r;
  switch (op) {
    case ADD: r = a + b; break;
    case SUB: r = a - b; break;
    case MUL: r = a * b; break;
    default: r = a / b; break;
  }
  bool finite_operands = op == DIV ? !std::isinf(a) : (!std::isinf(a) && !std::isinf(b));
  if (std::isinf(r) && finite_operands) return WC_FLOAT_OVERFLOW;
  bool underflowed = false;
  if (op == MUL) underflowed = a != F(0) && b != F(0);
  if (op == DIV) underflowed = a != F(0) && !std::isinf(b);
  if (r == F(0) && underflowed) return WC_FLOAT_UNDERFLOW;
  *out = r;
  return WC_OK;
}

// compute/cast.rs:43-64.
Status float4_from_float8(double v, float* out) {
  float n = (float)v;
  if (std::isinf(n) && !std::isinf(v)) return WC_FLOAT_OVERFLOW;
  if (n == 0.0f && v != 0.0) return WC_FLOAT_UNDERFLOW;
  *out = n;
  return WC_OK;
}
Status int8_from_float8(double v, int64_t* out) {
  double r = std::nearbyint(v);  // round half to even in the default mode
  if (!(r >= -9223372036854775808.0 && r < 9223372036854775808.0)) return WC_BIGINT_OUT_OF_RANGE;
  *out = (int64_t)r;
  return WC_OK;
}

template <> struct El<double> {
  static constexpr int dtype = WC_F64;
  static int cmp(double a, double b) { return float_cmp(a, b); }
  static bool nonzero(double a) { return a != 0.0; }
  static double f64(double a) { return a; }
  static Status from_weight(double w, double* o) { *o = w; return WC_OK; }
};
template <> struct El<float> {
  static constexpr int dtype = WC_F32;
  static int cmp(float a, float b) { return float_cmp(a, b); }
  static bool nonzero(float a) { return a != 0.0f; }
  static double f64(float a) { return a; }
  static Status from_weight(double w, float* o) { return float4_from_float8(w, o); }
};
template <> struct El<int64_t> {
  static constexpr int dtype = WC_I64;
  static int cmp(int64_t a, int64_t b) { return a < b ? -1 : (a > b ? 1 : 0); }
  static bool nonzero(int64_t a) { return a != 0; }
  static double f64(int64_t a) { return (double)a; }
  static Status from_weight(double w, int64_t* o) { return int8_from_float8(w, o); }
};
template <> struct El<uint8_t> {  // bool, one byte, 0 or 1
  static constexpr int dtype = WC_BOOL;
  static int cmp(uint8_t a, uint8_t b) { return (int)(a != 0) - (int)(b != 0); }
  static bool nonzero(uint8_t a) { return a != 0; }
  static double f64(uint8_t a) { return a ? 1.0 : 0.0; }
  static Status from_weight(double w, uint8_t* o) { *o = w != 0.0; return WC_OK; }
};

// compute/semiring.rs:264-278: LEAST / GREATEST keep the first on a tie.
template <class E> E least(E a, E b) { return El<E>::cmp(b, a) < 0 ? b : a; }
template <class E> E greatest(E a, E b) { return El<E>::cmp(b, a) > 0 ? b : a; }

// compute/semiring.rs:280-388: BinaryOp applied to each element type.
template <class E> struct Ops;
template <class F> Status float_apply(int op, F a, F b, F* o) {
  switch (op) {
    case WC_OP_FIRST: case WC_OP_ANY: *o = a; break;
    case WC_OP_SECOND: *o = b; break;
    case WC_OP_PAIR: *o = 1; break;
    case WC_OP_PLUS: *o = a + b; break;
    case WC_OP_TIMES: *o = a * b; break;
    case WC_OP_MIN: *o = least(a, b); break;
    case WC_OP_MAX: *o = greatest(a, b); break;
    case WC_OP_LOR: *o = (a != 0 || b != 0 || std::isnan(a) || std::isnan(b)) ? 1 : 0; break;
    case WC_OP_LAND: *o = ((a != 0 || std::isnan(a)) && (b != 0 || std::isnan(b))) ? 1 : 0; break;
  }
  return WC_OK;
}
template <> struct Ops<double> {
  static Status apply(int op, double a, double b, double* o) { return float_apply(op, a, b, o); }
  static double identity(int monoid) {
    return monoid == WC_OP_MIN ? INFINITY : (monoid == WC_OP_MAX ? -INFINITY : 0.0);
  }
};
template <> struct Ops<float> {
  static Status apply(int op, float a, float b, float* o) { return float_apply(op, a, b, o); }
  static float identity(int monoid) {
    return monoid == WC_OP_MIN ? INFINITY : (monoid == WC_OP_MAX ? -INFINITY : 0.0f);
  }
};
template <> struct Ops<int64_t> {
  static Status apply(int op, int64_t a, int64_t b, int64_t* o) {
    switch (op) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = a; break;
      case WC_OP_SECOND: *o = b; break;
      case WC_OP_PAIR: *o = 1; break;
      case WC_OP_PLUS: if (__builtin_add_overflow(a, b, o)) return WC_BIGINT_OUT_OF_RANGE; break;
      case WC_OP_TIMES: if (__builtin_mul_overflow(a, b, o)) return WC_BIGINT_OUT_OF_RANGE; break;
      case WC_OP_MIN: *o = std::min(a, b); break;
      case WC_OP_MAX: *o = std::max(a, b); break;
      case WC_OP_LOR: *o = (a != 0 || b != 0); break;
      case WC_OP_LAND: *o = (a != 0 && b != 0); break;
    }
    return WC_OK;
  }
  static int64_t identity(int monoid) {
    return monoid == WC_OP_MIN ? INT64_MAX : (monoid == WC_OP_MAX ? INT64_MIN : 0);
  }
};
template <> struct Ops<uint8_t> {
  static Status apply(int op, uint8_t a, uint8_t b, uint8_t* o) {
    bool x = a != 0, y = b != 0;
    switch (op) {
      case WC_OP_FIRST: case WC_OP_ANY: *o = x; break;
      case WC_OP_SECOND: *o = y; break;
      case WC_OP_PAIR: *o = 1; break;
      case WC_OP_PLUS: case WC_OP_MAX: case WC_OP_LOR: *o = x || y; break;
      default: *o = x && y; break;  // times, min, land
    }
    return WC_OK;
  }
  static uint8_t identity(int monoid) { return monoid == WC_OP_MIN ? 1 : 0; }
};

// compute/semiring.rs:170-191: ⊕ and ⊗ of each semiring.
const int kAdd[13] = {WC_OP_PLUS, WC_OP_MIN, WC_OP_MAX, WC_OP_MAX, WC_OP_MIN, WC_OP_LOR,
                      WC_OP_ANY,  WC_OP_PLUS, WC_OP_PLUS, WC_OP_PLUS, WC_OP_MIN, WC_OP_MIN,
                      WC_OP_MAX};
const int kMul[13] = {WC_OP_TIMES, WC_OP_PLUS,  WC_OP_PLUS,   WC_OP_TIMES, WC_OP_TIMES,
                      WC_OP_LAND,  WC_OP_PAIR,  WC_OP_PAIR,   WC_OP_FIRST, WC_OP_SECOND,
                      WC_OP_FIRST, WC_OP_SECOND, WC_OP_SECOND};

// compute/semiring.rs:254-261 and 340-363: ⊗(weight, value), with the i64
// ±∞ identities absorbing plus and times by a positive weight.
template <class E> Status multiply(int add, int mul, E weight, E value, E* o) {
  if constexpr (std::is_same_v<E, int64_t>) {
    bool infinite = (add == WC_OP_MIN && value == INT64_MAX) || (add == WC_OP_MAX && value == INT64_MIN);
    bool absorbs = mul == WC_OP_PLUS || (mul == WC_OP_TIMES && weight > 0);
    if (infinite && absorbs) { *o = value; return WC_OK; }
  }
  return Ops<E>::apply(mul, weight, value, o);
}

// compute/product/kernel.rs:39-47: the weight is cast only if ⊗ reads it.
template <class E> Status times(int add, int mul, double w, E value, E* o) {
  E weight{};
  if (mul != WC_OP_SECOND && mul != WC_OP_PAIR) {
    Status s = El<E>::from_weight(w, &weight);
    if (s) return s;
  }
  return multiply<E>(add, mul, weight, value, o);
}

// ------------------------------------------------------------------ graph

struct Csr {
  uint64_t n = 0;
  std::vector<uint64_t> off;  // n + 1
  std::vector<uint32_t> tgt;
  std::vector<double> w;      // empty: unweighted
  bool weighted() const { return !w.empty(); }
};

// graph/csr/transpose.rs:14-44: counting transpose, scattering while sources
// are scanned in order, so every reverse row comes out ascending.
Csr transpose(const Csr& c) {
  Csr r;
  r.n = c.n;
  r.off.assign(c.n + 1, 0);
  for (uint32_t t : c.tgt) r.off[t + 1]++;
  for (uint64_t i = 0; i < c.n; i++) r.off[i + 1] += r.off[i];
  std::vector<uint64_t> cur(r.off.begin(), r.off.end() - 1);
  r.tgt.resize(c.tgt.size());
  if (c.weighted()) r.w.resize(c.w.size());
  for (uint64_t s = 0; s < c.n; s++)
    for (uint64_t e = c.off[s]; e < c.off[s + 1]; e++) {
      uint64_t p = cur[c.tgt[e]]++;
      r.tgt[p] = (uint32_t)s;
      if (c.weighted()) r.w[p] = c.w[e];
    }
  return r;
}

// graph/csr/build/deduplication.rs:1-7, 16-79: each relation's rows sorted by
// target (stably, for weights), parallel edges folded with weights summed in
// input order; the merged CSR sums the relations' folded weights in relation
// order.  Unweighted rows just drop repeats.
struct Edge { uint32_t rel; uint64_t s, t; double w; uint64_t order; };

Csr build_merged(uint64_t n, uint32_t relations, std::vector<Edge> edges, bool weighted) {
  // Per relation: group (s, t) pairs in input order.
  std::stable_sort(edges.begin(), edges.end(), [](const Edge& a, const Edge& b) {
    if (a.s != b.s) return a.s < b.s;
    if (a.t != b.t) return a.t < b.t;
    return a.rel < b.rel;  // stable: input order within (s, t, rel)
  });
  Csr c;
  c.n = n;
  c.off.assign(n + 1, 0);
  for (size_t i = 0; i < edges.size();) {
    size_t j = i;
    double total = 0.0;
    bool first_relation = true;
    // Relations in order (merge_weighted, deduplication.rs:117-150), each
    // relation's weights in input order (relation_sum / fold_weighted: the
    // first weight, then `+=` each later one).
    while (j < edges.size() && edges[j].s == edges[i].s && edges[j].t == edges[i].t) {
      uint32_t rel = edges[j].rel;
      double sum = edges[j].w;
      j++;
      while (j < edges.size() && edges[j].s == edges[i].s && edges[j].t == edges[i].t &&
             edges[j].rel == rel) {
        sum += edges[j].w;
        j++;
      }
      total = first_relation ? sum : total + sum;
      first_relation = false;
    }
    c.tgt.push_back((uint32_t)edges[i].t);
    if (weighted) c.w.push_back(total);
    c.off[edges[i].s + 1]++;
    i = j;
  }
  for (uint64_t r = 0; r < n; r++) c.off[r + 1] += c.off[r];
  (void)relations;
  return c;
}

struct Graph {
  Csr fwd, rev;
  bool has_rev = false;
};

// ------------------------------------------------------------------ product

struct Mask {
  const void* values = nullptr;
  int dtype = WC_F64;
  bool complement = false;
  bool selects(uint64_t row) const {
    bool set = false;
    switch (dtype) {
      case WC_F32: set = ((const float*)values)[row] != 0.0f || std::isnan(((const float*)values)[row]); break;
      case WC_F64: set = ((const double*)values)[row] != 0.0 || std::isnan(((const double*)values)[row]); break;
      case WC_I64: set = ((const int64_t*)values)[row] != 0; break;
      default: set = ((const uint8_t*)values)[row] != 0; break;
    }
    return set != complement;
  }
};

struct Product {
  int semiring = WC_PLUS_TIMES;
  bool transpose = false;
  int weighted = -1;
  const Mask* mask = nullptr;
  bool replace = false;
  int accumulate = WC_OP_NONE;
};

// compute/product/kernel.rs:200-240 (Write::row).
template <class E> Status write_row(const Product& p, uint64_t row, E* out, const E* t, size_t width) {
  E identity = Ops<E>::identity(kAdd[p.semiring]);
  if (p.mask && !p.mask->selects(row)) {
    if (p.replace) std::fill(out, out + width, identity);
    return WC_OK;
  }
  if (p.accumulate == WC_OP_NONE) {
    if (t) std::copy(t, t + width, out);
    else std::fill(out, out + width, identity);
  } else if (t) {
    for (size_t k = 0; k < width; k++) {
      Status s = Ops<E>::apply(p.accumulate, out[k], t[k], &out[k]);
      if (s) return s;
    }
  }
  return WC_OK;
}

const size_t ROWS_PER_TASK = 4096;  // compute/product/kernel.rs:15

// compute/product/kernel.rs:84-121 (pull_with) over `csr`: each row folds
// ⊗(weight, x[col]) with ⊕ in ascending column order, the first entry
// setting the sum; then Write::row.
template <class E>
Status pull(const Product& p, const Csr& csr, bool weighted, const E* x, E* y, size_t width) {
  int add = kAdd[p.semiring], mul = kMul[p.semiring];
  size_t tasks = (csr.n + ROWS_PER_TASK - 1) / ROWS_PER_TASK;
  return parallel_tasks(tasks, [&](size_t task) -> Status {
    std::vector<E> sum(width);
    uint64_t r0 = task * ROWS_PER_TASK, r1 = std::min<uint64_t>(csr.n, r0 + ROWS_PER_TASK);
    for (uint64_t row = r0; row < r1; row++) {
      bool present = false;
      for (uint64_t e = csr.off[row]; e < csr.off[row + 1]; e++) {
        double w = weighted ? csr.w[e] : 1.0;
        const E* xr = x + (size_t)csr.tgt[e] * width;
        for (size_t k = 0; k < width; k++) {
          E prod;
          Status s = times<E>(add, mul, w, xr[k], &prod);
          if (s) return s;
          if (present) {
            s = Ops<E>::apply(add, sum[k], prod, &sum[k]);
            if (s) return s;
          } else {
            sum[k] = prod;
          }
        }
        present = true;
      }
      Status s = write_row<E>(p, row, y + row * width, present ? sum.data() : nullptr, width);
      if (s) return s;
    }
    return WC_OK;
  });
}

// compute/product/kernel.rs:145-182 (push_with): y = Aᵀ ⊗ x by scattering
// rows in ascending order, then writing each row.
template <class E>
Status push(const Product& p, const Csr& csr, bool weighted, const E* x, E* y, size_t width) {
  int add = kAdd[p.semiring], mul = kMul[p.semiring];
  std::vector<E> sums(csr.n * width);
  std::vector<uint8_t> present(csr.n, 0);
  for (uint64_t row = 0; row < csr.n; row++) {
    for (uint64_t e = csr.off[row]; e < csr.off[row + 1]; e++) {
      uint64_t col = csr.tgt[e];
      double w = weighted ? csr.w[e] : 1.0;
      for (size_t k = 0; k < width; k++) {
        E prod;
        Status s = times<E>(add, mul, w, x[row * width + k], &prod);
        if (s) return s;
        E& sum = sums[col * width + k];
        if (present[col]) {
          s = Ops<E>::apply(add, sum, prod, &sum);
          if (s) return s;
        } else {
          sum = prod;
        }
      }
      present[col] = 1;
    }
  }
  for (uint64_t row = 0; row < csr.n; row++) {
    Status s = write_row<E>(p, row, y + row * width, present[row] ? &sums[row * width] : nullptr, width);
    if (s) return s;
  }
  return WC_OK;
}

// compute/product/mod.rs:181-205 + matrix.rs:126-157: pull over the forward
// CSR, or for Aᵀ over the reverse CSR, else pushed over the forward CSR.
template <class E>
Status multiply_into(const Graph& g, const Product& p, const E* x, E* y, size_t width, bool force_push) {
  bool weighted = (p.weighted != 0) && g.fwd.weighted();
  if (!p.transpose) return pull<E>(p, g.fwd, weighted, x, y, width);
  if (g.has_rev && !force_push) return pull<E>(p, g.rev, weighted, x, y, width);
  return push<E>(p, g.fwd, weighted, x, y, width);
}

// ------------------------------------------------------------------ pagerank

const size_t CHUNK_DEFAULT = 1 << 16;  // compute/reduce.rs:20
size_t g_chunk = CHUNK_DEFAULT;

struct PageRankOpts {
  double damping = 0.85;
  bool has_tol = true;
  double tol = 1e-6;
  int weighted = -1;
  uint32_t max_iter = 100;
  const double* seed = nullptr;
};

bool tombstoned(const uint64_t* words, uint64_t row) {
  return words && ((words[row >> 6] >> (row & 63)) & 1);
}

// compute/pagerank/mod.rs:96-287.
Status pagerank(const Graph& g, const uint64_t* tomb, const PageRankOpts& o, double* x_out,
                uint32_t* iterations_out, double* last_delta, double* threshold_out) {
  uint64_t n = g.fwd.n;
  uint64_t live = 0;
  for (uint64_t i = 0; i < n; i++) live += !tombstoned(tomb, i);
  double nodes = (double)live;
  double start;
  Status s = sql_float<double>(DIV, 1.0, nodes, &start);
  if (s) return s;
  std::vector<double> x(n, start);
  for (uint64_t i = 0; i < n; i++)
    if (tombstoned(tomb, i)) x[i] = 0.0;
  // out = plus_first over the forward CSR (the out-weight).
  std::vector<double> out(n, 0.0);
  Product pf;
  pf.semiring = WC_PLUS_FIRST;
  pf.weighted = o.weighted;
  if ((s = multiply_into<double>(g, pf, x.data(), out.data(), 1, false))) return s;
  // The personalisation: uniform start, or seed / sum(seed) over live rows.
  std::vector<double> shares;
  bool seeded = o.seed != nullptr;
  if (seeded) {
    size_t chunks = (n + g_chunk - 1) / g_chunk;
    double sum = 0.0;
    for (size_t c = 0; c < chunks; c++) {  // reduce.rs:137-153, 266-279
      double part = 0.0;
      for (uint64_t i = c * g_chunk; i < std::min<uint64_t>(n, (c + 1) * g_chunk); i++)
        if (!tombstoned(tomb, i)) part = part + o.seed[i];
      sum = sum + part;
    }
    double total;
    if ((s = sql_float<double>(DIV, 1.0, sum, &total))) return s;
    shares.assign(n, 0.0);
    for (uint64_t i = 0; i < n; i++)
      if (!tombstoned(tomb, i))
        if ((s = sql_float<double>(MUL, o.seed[i], total, &shares[i]))) return s;
  }
  double teleport;
  if ((s = sql_float<double>(SUB, 1.0, o.damping, &teleport))) return s;
  std::vector<double> msg(n, 0.0), y(n, 0.0);
  Product inflow;
  inflow.semiring = WC_PLUS_TIMES;
  inflow.transpose = true;
  inflow.weighted = o.weighted;
  uint32_t iterations = 0;
  size_t chunks = (n + g_chunk - 1) / g_chunk;
  std::vector<double> partial(chunks);
  double delta = 0.0, threshold = 0.0;
  while (iterations < o.max_iter) {
    iterations++;
    // spread (mod.rs:204-232)
    s = parallel_tasks(chunks, [&](size_t c) -> Status {
      double dangling = 0.0;
      for (uint64_t i = c * g_chunk; i < std::min<uint64_t>(n, (c + 1) * g_chunk); i++) {
        if (float_cmp(out[i], 0.0) > 0) {
          Status e = sql_float<double>(DIV, x[i], out[i], &msg[i]);
          if (e) return e;
        } else {
          dangling += x[i];
          msg[i] = 0.0;
        }
      }
      partial[c] = dangling;
      return WC_OK;
    });
    if (s) return s;
    double dangling = 0.0;
    for (size_t c = 0; c < chunks; c++) dangling = dangling + partial[c];
    if ((s = multiply_into<double>(g, inflow, msg.data(), y.data(), 1, false))) return s;
    // advance (mod.rs:245-282)
    s = parallel_tasks(chunks, [&](size_t c) -> Status {
      double change = 0.0;
      for (uint64_t i = c * g_chunk; i < std::min<uint64_t>(n, (c + 1) * g_chunk); i++) {
        double next = 0.0;
        if (!tombstoned(tomb, i)) {
          double p = seeded ? shares[i] : start;
          double dp, flowed, a, b;
          Status e;
          if ((e = sql_float<double>(MUL, dangling, p, &dp))) return e;
          if ((e = sql_float<double>(ADD, y[i], dp, &flowed))) return e;
          if ((e = sql_float<double>(MUL, o.damping, flowed, &a))) return e;
          if ((e = sql_float<double>(MUL, teleport, p, &b))) return e;
          if ((e = sql_float<double>(ADD, a, b, &next))) return e;
        }
        change += std::fabs(next - x[i]);
        x[i] = next;
      }
      partial[c] = change;
      return WC_OK;
    });
    if (s) return s;
    delta = 0.0;
    for (size_t c = 0; c < chunks; c++) delta = delta + partial[c];
    if (o.has_tol) {
      if ((s = sql_float<double>(MUL, nodes, o.tol, &threshold))) return s;
      if (float_cmp(delta, threshold) < 0) break;
    }
  }
  std::copy(x.begin(), x.end(), x_out);
  *iterations_out = iterations;
  if (last_delta) *last_delta = delta;
  if (threshold_out) *threshold_out = threshold;
  return WC_OK;
}

// ------------------------------------------------------------------ traversal

struct Adj {  // traversal/adjacency.rs:327-341: the rows read in a direction
  std::vector<const Csr*> rows;
  uint64_t bound(uint64_t v) const {
    uint64_t b = 0;
    for (auto* c : rows) b += c->off[v + 1] - c->off[v];
    return b;
  }
};

Adj adjacency(const Graph& g, int direction) {
  Adj a;
  if (direction == WC_OUT) a.rows = {&g.fwd};
  else if (direction == WC_IN) a.rows = {&g.rev};
  else a.rows = {&g.fwd, &g.rev};
  return a;
}

struct Visit { uint64_t node; uint32_t depth; uint64_t via; };
struct Stats { uint64_t nodes_visited = 0, edges_traversed = 0; int truncated = 0; uint32_t levels = 0, pulled = 0; };

// traversal/level.rs:88-337 (LevelSearch) with bfs.rs:63-111 (Results):
// push levels scan the sorted frontier's rows admitting unvisited nodes in
// the order reached; with `reverse`, Beamer's switch (α = 1, β = 24) may pull
// a level, admitting nodes in ascending dense id order.
Status level_search(const Graph& g, int direction, const uint64_t* starts, uint64_t nstarts,
                    uint32_t max_depth, uint64_t max_results, const uint64_t* filter,
                    bool pulling, std::vector<Visit>& visits, Stats& st) {
  const uint64_t n = g.fwd.n;
  const uint64_t ALPHA = 1, BETA = 24;
  for (uint64_t i = 0; i < nstarts; i++)
    if (starts[i] >= n) return WC_NODE_OUTSIDE_ID_SPACE;
  Adj adj = adjacency(g, direction);
  int rdir = direction == WC_OUT ? WC_IN : (direction == WC_IN ? WC_OUT : WC_BOTH);
  Adj radj = adjacency(g, rdir);
  std::vector<uint64_t> visited((n + 63) / 64, 0);
  auto is_visited = [&](uint64_t v) { return (visited[v >> 6] >> (v & 63)) & 1; };
  auto set_visited = [&](uint64_t v) { visited[v >> 6] |= 1ull << (v & 63); };
  auto in_filter = [&](uint64_t v) { return !filter || ((filter[v >> 6] >> (v & 63)) & 1); };
  std::vector<uint64_t> frontier, next;
  uint64_t emitted = 0;
  bool stop = false;
  // offer_into (level.rs:306-325) with Results::admit (bfs.rs:96-110)
  auto offer = [&](Visit v) -> bool {
    if (max_results != UINT64_MAX && emitted == max_results) {
      st.truncated = 1;
      stop = true;
      return false;
    }
    emitted++;
    st.nodes_visited++;
    set_visited(v.node);
    next.push_back(v.node);
    visits.push_back(v);
    return true;
  };
  for (uint64_t i = 0; i < nstarts && !stop; i++)
    if (!is_visited(starts[i])) offer({starts[i], 0, WC_NO_VIA});
  std::swap(frontier, next);
  next.clear();
  uint32_t depth = 0;
  while (!stop && !frontier.empty() && depth < max_depth) {
    std::sort(frontier.begin(), frontier.end());
    bool pull = false;
    if (pulling && frontier.size() * BETA > n) {  // level.rs:184-211
      uint64_t mf = 0;
      for (uint64_t v : frontier) mf += adj.bound(v);
      uint64_t limit = mf * ALPHA, mu = 0;
      pull = true;
      for (uint64_t v = 0; v < n && pull; v++)
        if (!is_visited(v)) {
          mu += radj.bound(v);
          if (mu >= limit) pull = false;
        }
    }
    uint32_t d = depth + 1;
    st.levels++;
    if (!pull) {  // level.rs:216-241
      for (uint64_t via : frontier) {
        for (auto* c : adj.rows)
          for (uint64_t e = c->off[via]; e < c->off[via + 1] && !stop; e++) {
            st.edges_traversed++;
            uint64_t v = c->tgt[e];
            if (is_visited(v) || !in_filter(v)) continue;
            offer({v, d, via});
          }
        if (stop) break;
      }
    } else {  // level.rs:246-284
      st.pulled++;
      std::vector<uint64_t> fset((n + 63) / 64, 0);
      for (uint64_t v : frontier) fset[v >> 6] |= 1ull << (v & 63);
      for (uint64_t word = 0; word < visited.size() && !stop; word++) {
        uint64_t clear = ~visited[word];
        while (clear && !stop) {
          uint64_t v = word * 64 + __builtin_ctzll(clear);
          clear &= clear - 1;
          if (v >= n) break;
          if (!in_filter(v)) continue;
          bool found = false;
          for (auto* c : radj.rows) {
            for (uint64_t e = c->off[v]; e < c->off[v + 1]; e++) {
              st.edges_traversed++;
              uint64_t via = c->tgt[e];
              if (!((fset[via >> 6] >> (via & 63)) & 1)) continue;
              offer({v, d, via});
              found = true;
              break;
            }
            if (found) break;
          }
        }
      }
    }
    std::swap(frontier, next);
    next.clear();
    depth = d;
  }
  return WC_OK;
}

// ------------------------------------------------------------------ random
// compute/random.rs:11-25: SplitMix64 finaliser and uniform(seed, stream, node).
const uint64_t GOLDEN = 0x9e3779b97f4a7c15ull;
uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
double uniform(uint64_t seed, uint64_t stream, uint64_t node) {
  uint64_t bits = mix(mix(seed ^ mix(stream * GOLDEN)) ^ (node * GOLDEN));
  return (double)(bits >> 11) / (double)(1ull << 52) - 1.0;
}

}  // namespace

// ====================================================================== C ABI

extern "C" {

typedef struct wo_graph wo_graph;

void wo_set_threads(int n) { g_threads = n; }
int wo_threads(void) { return threads(); }
void wo_set_chunk(uint64_t chunk) { g_chunk = chunk ? chunk : CHUNK_DEFAULT; }

// Builds a graph from (relation, source, target, weight) edges as the
// reference builds one (graph/csr/build/, transpose.rs); `weights` NULL:
// unweighted.  `reverse`: also build the reverse CSR.
wo_graph* wo_graph_build(uint64_t n, uint32_t relations, uint64_t count, const uint32_t* rel,
                         const uint64_t* src, const uint64_t* dst, const double* weights, int reverse) {
  std::vector<Edge> edges(count);
  for (uint64_t i = 0; i < count; i++)
    edges[i] = {rel ? rel[i] : 0u, src[i], dst[i], weights ? weights[i] : 1.0, i};
  auto* g = new Graph;
  g->fwd = build_merged(n, relations, std::move(edges), weights != nullptr);
  if (reverse) {
    g->rev = transpose(g->fwd);
    g->has_rev = true;
  }
  return (wo_graph*)g;
}

// A graph from a built CSR (offsets u64[n+1], targets, weights or NULL).
wo_graph* wo_graph_from_csr(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* tgt,
                            const double* w, int reverse) {
  auto* g = new Graph;
  g->fwd.n = n;
  g->fwd.off.assign(off, off + n + 1);
  g->fwd.tgt.assign(tgt, tgt + m);
  if (w) g->fwd.w.assign(w, w + m);
  if (reverse) {
    g->rev = transpose(g->fwd);
    g->has_rev = true;
  }
  return (wo_graph*)g;
}

void wo_graph_free(wo_graph* g) { delete (Graph*)g; }
uint64_t wo_graph_edges(const wo_graph* g) { return ((const Graph*)g)->fwd.tgt.size(); }
int wo_graph_weighted(const wo_graph* g) { return ((const Graph*)g)->fwd.weighted(); }

// Copies the CSR (and reverse CSR, if built) out; any pointer may be NULL.
void wo_graph_copy(const wo_graph* gp, uint64_t* off, uint32_t* tgt, double* w, uint64_t* roff,
                   uint32_t* rtgt, double* rw) {
  const Graph* g = (const Graph*)gp;
  if (off) std::copy(g->fwd.off.begin(), g->fwd.off.end(), off);
  if (tgt) std::copy(g->fwd.tgt.begin(), g->fwd.tgt.end(), tgt);
  if (w && g->fwd.weighted()) std::copy(g->fwd.w.begin(), g->fwd.w.end(), w);
  if (g->has_rev) {
    if (roff) std::copy(g->rev.off.begin(), g->rev.off.end(), roff);
    if (rtgt) std::copy(g->rev.tgt.begin(), g->rev.tgt.end(), rtgt);
    if (rw && g->rev.weighted()) std::copy(g->rev.w.begin(), g->rev.w.end(), rw);
  }
}

// compute/semiring.rs: apply, identity, multiply and from_weight on one
// element type, for the known-answer tests.  Values travel as 8 bytes.
int32_t wo_apply(int dtype, int op, const void* a, const void* b, void* out) {
  switch (dtype) {
    case WC_F64: return Ops<double>::apply(op, *(const double*)a, *(const double*)b, (double*)out);
    case WC_F32: return Ops<float>::apply(op, *(const float*)a, *(const float*)b, (float*)out);
    case WC_I64: return Ops<int64_t>::apply(op, *(const int64_t*)a, *(const int64_t*)b, (int64_t*)out);
    default: return Ops<uint8_t>::apply(op, *(const uint8_t*)a, *(const uint8_t*)b, (uint8_t*)out);
  }
}
int32_t wo_multiply(int dtype, int add, int mul, const void* w, const void* v, void* out) {
  switch (dtype) {
    case WC_F64: return multiply<double>(add, mul, *(const double*)w, *(const double*)v, (double*)out);
    case WC_F32: return multiply<float>(add, mul, *(const float*)w, *(const float*)v, (float*)out);
    case WC_I64: return multiply<int64_t>(add, mul, *(const int64_t*)w, *(const int64_t*)v, (int64_t*)out);
    default: return multiply<uint8_t>(add, mul, *(const uint8_t*)w, *(const uint8_t*)v, (uint8_t*)out);
  }
}
int32_t wo_from_weight(int dtype, double w, void* out) {
  switch (dtype) {
    case WC_F64: return El<double>::from_weight(w, (double*)out);
    case WC_F32: return El<float>::from_weight(w, (float*)out);
    case WC_I64: return El<int64_t>::from_weight(w, (int64_t*)out);
    default: return El<uint8_t>::from_weight(w, (uint8_t*)out);
  }
}
void wo_identity(int dtype, int monoid, void* out) {
  switch (dtype) {
    case WC_F64: *(double*)out = Ops<double>::identity(monoid); break;
    case WC_F32: *(float*)out = Ops<float>::identity(monoid); break;
    case WC_I64: *(int64_t*)out = Ops<int64_t>::identity(monoid); break;
    default: *(uint8_t*)out = Ops<uint8_t>::identity(monoid); break;
  }
}
int wo_semiring_add(int semiring) { return kAdd[semiring]; }
int wo_semiring_mul(int semiring) { return kMul[semiring]; }
// map/arithmetic.rs:49-79 on f64.
int32_t wo_float(int op, double a, double b, double* out) { return sql_float<double>((Arith)op, a, b, out); }
double wo_uniform(uint64_t seed, uint64_t stream, uint64_t node) { return uniform(seed, stream, node); }

// compute/product/mod.rs:77-110 (spmv / spmm), all relations.  `force_push`:
// multiply by Aᵀ with the push kernel even where a reverse CSR exists.
int32_t wo_product(const wo_graph* gp, int semiring, int transpose, int weighted,
                   const void* mask_values, int mask_dtype, int mask_complement, int replace,
                   int accumulate, int dtype, uint64_t width, const void* x, void* y, int force_push) {
  const Graph& g = *(const Graph*)gp;
  if (semiring < 0 || semiring > 12) return WC_UNKNOWN_SEMIRING;
  if (width == 0) return WC_ZERO_WIDTH;
  Mask mask{mask_values, mask_dtype, mask_complement != 0};
  Product p;
  p.semiring = semiring;
  p.transpose = transpose != 0;
  p.weighted = weighted;
  p.mask = mask_values ? &mask : nullptr;
  p.replace = replace != 0;
  p.accumulate = accumulate;
  switch (dtype) {
    case WC_F64: return multiply_into<double>(g, p, (const double*)x, (double*)y, width, force_push);
    case WC_F32: return multiply_into<float>(g, p, (const float*)x, (float*)y, width, force_push);
    case WC_I64: return multiply_into<int64_t>(g, p, (const int64_t*)x, (int64_t*)y, width, force_push);
    case WC_BOOL: return multiply_into<uint8_t>(g, p, (const uint8_t*)x, (uint8_t*)y, width, force_push);
  }
  return WC_DTYPE_MISMATCH;
}

// compute/pagerank/mod.rs:96-151.
int32_t wo_pagerank(const wo_graph* gp, const uint64_t* tombstones, double damping, int has_tol,
                    double tol, int weighted, uint32_t max_iter, const double* seed, double* ranks,
                    uint32_t* iterations, double* last_delta, double* threshold) {
  PageRankOpts o;
  o.damping = damping;
  o.has_tol = has_tol != 0;
  o.tol = tol;
  o.weighted = weighted;
  o.max_iter = max_iter;
  o.seed = seed;
  return pagerank(*(const Graph*)gp, tombstones, o, ranks, iterations, last_delta, threshold);
}

// traversal/level.rs:88-337 (LevelSearch::run) with bfs.rs:96-110's
// result limit: visits (node, depth, via) in the reference's order into
// `visits` (3 u64 per visit, `capacity` visits).  `pulling` lets levels be
// pulled (reachable_set's edges, with the reverse CSR); without it this is
// traversal/bfs.rs:34-79 (bfs).
int32_t wo_level_search(const wo_graph* gp, int direction, const uint64_t* starts,
                        uint64_t nstarts, uint32_t max_depth, uint64_t max_results,
                        const uint64_t* filter, int32_t pulling, uint64_t* visits,
                        uint64_t capacity, uint64_t* count, uint64_t* stats) {
  const Graph& g = *(const Graph*)gp;
  if (direction != WC_OUT && !g.has_rev) return WC_REVERSE_CSR_MISSING;
  std::vector<Visit> v;
  Stats st;
  Status s = level_search(g, direction, starts, nstarts, max_depth, max_results, filter,
                          pulling && g.has_rev, v, st);
  if (s) return s;
  *count = v.size();
  for (uint64_t i = 0; i < v.size() && i < capacity; i++) {
    visits[3 * i] = v[i].node;
    visits[3 * i + 1] = v[i].depth;
    visits[3 * i + 2] = v[i].via;
  }
  if (stats) {
    stats[0] = st.nodes_visited;
    stats[1] = st.edges_traversed;
    stats[2] = st.truncated;
    stats[3] = st.levels;
    stats[4] = st.pulled;
  }
  return WC_OK;
}

int32_t wo_bfs(const wo_graph* gp, int direction, const uint64_t* starts, uint64_t nstarts,
               uint32_t max_depth, uint64_t max_results, const uint64_t* filter, uint64_t* visits,
               uint64_t capacity, uint64_t* count, uint64_t* stats) {
  return wo_level_search(gp, direction, starts, nstarts, max_depth, max_results, filter, 0,
                         visits, capacity, count, stats);
}

// traversal/reachable.rs:79-90 (reachable_set_each): with the reverse CSR
// levels may be pulled.
int32_t wo_reachable_set(const wo_graph* gp, int direction, const uint64_t* starts, uint64_t nstarts,
                         uint32_t max_depth, uint64_t* nodes, uint64_t capacity, uint64_t* count,
                         uint64_t* stats) {
  const Graph& g = *(const Graph*)gp;
  if (direction != WC_OUT && !g.has_rev) return WC_REVERSE_CSR_MISSING;
  std::vector<Visit> v;
  Stats st;
  Status s = level_search(g, direction, starts, nstarts, max_depth, UINT64_MAX, nullptr, g.has_rev, v, st);
  if (s) return s;
  *count = v.size();
  for (uint64_t i = 0; i < v.size() && i < capacity; i++) nodes[i] = v[i].node;
  if (stats) {
    stats[0] = st.nodes_visited;
    stats[1] = st.edges_traversed;
    stats[2] = st.truncated;
    stats[3] = st.levels;
    stats[4] = st.pulled;
  }
  return WC_OK;
}

// Per-source depths of `width` plain BFS runs (out-edges, depth caps): the
// reference semantics of the batched BFS, one search per source.
// depth_out[s * n + i] = depth or 255.  edges_out[s]: edges_traversed.
int32_t wo_bfs_depths(const wo_graph* gp, const uint64_t* sources, const uint32_t* caps,
                      uint32_t width, uint8_t* depth_out, uint64_t* edges_out) {
  const Graph& g = *(const Graph*)gp;
  uint64_t n = g.fwd.n;
  return parallel_tasks(width, [&](size_t s) -> Status {
    std::vector<Visit> v;
    Stats st;
    Status e = level_search(g, WC_OUT, &sources[s], 1, caps[s], UINT64_MAX, nullptr, false, v, st);
    if (e) return e;
    uint8_t* d = depth_out + s * n;
    std::fill(d, d + n, 255);
    for (auto& x : v) d[x.node] = (uint8_t)x.depth;
    if (edges_out) edges_out[s] = st.edges_traversed;
    return WC_OK;
  });
}

// The reference's own batched shape, compute/centrality/multi_source.rs:33-160
// (SourceBatch, after Then et al., "The More the Merrier"): up to 64
// sources searched together, one bit each in a u64 word per node.  A step
// pushes each frontier node's word along its row into its neighbours' next
// words (an atomic OR less the sources that have already reached them,
// :126-150), listing a neighbour when its next word first turns non-zero;
// then each listed node takes next into seen and its frontier (:155-175).
// Frontier nodes are taken in tasks of 4,096 (centrality/mod.rs:79), in
// parallel.  With each source's depth cap applied as LevelSearch applies
// max_depth (a node at depth d is expanded for the sources whose cap is
// above d, traversal/level.rs:119-123), the depths and edges_traversed
// equal wo_bfs_depths's for every source.  Batches of 64 run in order.
int32_t wo_bfs_depths_batched64(const wo_graph* gp, const uint64_t* sources, const uint32_t* caps,
                                uint32_t width, uint8_t* depth_out, uint64_t* edges_out) {
  const Graph& g = *(const Graph*)gp;
  const uint64_t n = g.fwd.n;
  constexpr size_t kTask = 4096;
  std::vector<std::atomic<uint64_t>> seen(n), next(n);
  std::vector<uint64_t> frontier(n, 0);
  std::vector<uint64_t> current, listed(n);
  for (uint64_t i = 0; i < n; i++) {
    seen[i].store(0, std::memory_order_relaxed);
    next[i].store(0, std::memory_order_relaxed);
  }
  for (uint32_t s = 0; s < width; s++)
    if (sources[s] >= n) return WC_NODE_OUTSIDE_ID_SPACE;
  std::fill(depth_out, depth_out + (uint64_t)width * n, 255);
  for (uint32_t b0 = 0; b0 < width; b0 += 64) {
    const uint32_t bk = std::min<uint32_t>(64, width - b0);
    uint64_t edges[64] = {0};
    current.clear();
    for (uint32_t bit = 0; bit < bk; bit++) {
      const uint64_t node = sources[b0 + bit];
      if (!seen[node].load(std::memory_order_relaxed) && !frontier[node]) current.push_back(node);
      seen[node].fetch_or(1ull << bit, std::memory_order_relaxed);
      frontier[node] |= 1ull << bit;
      depth_out[(uint64_t)(b0 + bit) * n + node] = 0;
    }
    for (uint32_t d = 1; !current.empty(); d++) {
      // Sources whose cap lets them expand depth d - 1.
      uint64_t expands = 0;
      for (uint32_t bit = 0; bit < bk; bit++)
        if (caps[b0 + bit] > d - 1) expands |= 1ull << bit;
      std::atomic<size_t> count{0};
      const size_t tasks = (current.size() + kTask - 1) / kTask;
      std::vector<std::array<uint64_t, 64>> task_edges(tasks);
      parallel_tasks(tasks, [&](size_t t) -> Status {
        std::array<uint64_t, 64>& te = task_edges[t];
        te.fill(0);
        std::vector<uint64_t> mine;
        const size_t lo = t * kTask, hi = std::min(current.size(), lo + kTask);
        for (size_t q = lo; q < hi; q++) {
          const uint64_t node = current[q];
          const uint64_t word = frontier[node] & expands;
          frontier[node] = 0;
          if (!word) continue;
          const uint64_t r0 = g.fwd.off[node], r1 = g.fwd.off[node + 1];
          for (uint64_t w = word; w; w &= w - 1) te[__builtin_ctzll(w)] += r1 - r0;
          for (uint64_t e = r0; e < r1; e++) {
            const uint64_t t2 = g.fwd.tgt[e];
            const uint64_t fresh = word & ~seen[t2].load(std::memory_order_relaxed);
            if (fresh & ~next[t2].load(std::memory_order_relaxed)) {
              if (next[t2].fetch_or(fresh, std::memory_order_relaxed) == 0) mine.push_back(t2);
            }
          }
        }
        const size_t at = count.fetch_add(mine.size());
        std::copy(mine.begin(), mine.end(), listed.begin() + at);
        return WC_OK;
      });
      for (const auto& te : task_edges)
        for (uint32_t bit = 0; bit < 64; bit++) edges[bit] += te[bit];
      // Settle: each listed node takes its next word (less what it has
      // seen) into seen and its frontier, and records the depth.
      const size_t found = count.load();
      const size_t stasks = (found + kTask - 1) / kTask;
      parallel_tasks(stasks, [&](size_t t) -> Status {
        const size_t lo = t * kTask, hi = std::min(found, lo + kTask);
        for (size_t q = lo; q < hi; q++) {
          const uint64_t node = listed[q];
          const uint64_t got = next[node].exchange(0, std::memory_order_relaxed) &
                               ~seen[node].load(std::memory_order_relaxed);
          seen[node].fetch_or(got, std::memory_order_relaxed);
          frontier[node] = got;
          for (uint64_t w = got; w; w &= w - 1)
            depth_out[(uint64_t)(b0 + __builtin_ctzll(w)) * n + node] = (uint8_t)std::min(d, 255u);
        }
        return WC_OK;
      });
      current.assign(listed.begin(), listed.begin() + found);
    }
    // Clear seen for the next batch (the reference clears after each search).
    parallel_tasks((n + kTask * 16 - 1) / (kTask * 16), [&](size_t t) -> Status {
      const uint64_t lo = t * kTask * 16, hi = std::min<uint64_t>(n, lo + kTask * 16);
      for (uint64_t i = lo; i < hi; i++) seen[i].store(0, std::memory_order_relaxed);
      return WC_OK;
    });
    if (edges_out)
      for (uint32_t bit = 0; bit < bk; bit++) edges_out[b0 + bit] = edges[bit];
  }
  return WC_OK;
}

// compute_sql/library/sssp_vector.sql:14-66 over the i64 dtype: x = {source:
// 0, else the min identity}; loop spmv(x → next, min_plus, transpose,
// accumulate min) with next starting as a copy of x, counting the nodes whose
// distance fell, until none fell or max_iter.  Per source, in parallel.
int32_t wo_sssp_i64(const wo_graph* gp, const uint64_t* sources, const uint32_t* max_iter,
                    uint32_t width, int64_t* dist_out, uint32_t* iterations_out) {
  const Graph& g = *(const Graph*)gp;
  uint64_t n = g.fwd.n;
  return parallel_tasks(width, [&](size_t c) -> Status {
    std::vector<int64_t> x(n, INT64_MAX), next(n);
    if (sources[c] >= n) return WC_NODE_OUTSIDE_ID_SPACE;
    x[sources[c]] = 0;
    Product p;
    p.semiring = WC_MIN_PLUS;
    p.transpose = true;
    p.accumulate = WC_OP_MIN;
    uint32_t i = 0;
    while (i < max_iter[c]) {
      i++;
      next = x;
      // One product per source runs on this thread alone.
      int add = kAdd[p.semiring], mul = kMul[p.semiring];
      bool weighted = g.fwd.weighted();
      const Csr& csr = g.has_rev ? g.rev : g.fwd;
      if (!g.has_rev) return WC_REVERSE_CSR_MISSING;
      for (uint64_t row = 0; row < n; row++) {
        bool present = false;
        int64_t sum = 0;
        for (uint64_t e = csr.off[row]; e < csr.off[row + 1]; e++) {
          int64_t prod;
          Status st = times<int64_t>(add, mul, weighted ? csr.w[e] : 1.0, x[csr.tgt[e]], &prod);
          if (st) return st;
          if (present) Ops<int64_t>::apply(add, sum, prod, &sum);
          else sum = prod;
          present = true;
        }
        if (present) next[row] = std::min(next[row], sum);
      }
      uint64_t fell = 0;
      for (uint64_t r = 0; r < n; r++) fell += next[r] < x[r];
      x.swap(next);
      if (fell == 0) break;
    }
    std::copy(x.begin(), x.end(), dist_out + c * n);
    if (iterations_out) iterations_out[c] = i;
    return WC_OK;
  });
}

// traversal/components.rs:21-58: weakly connected components by
// union-find over the forward rows swept in ascending order, the larger
// root hung under the smaller (path halving), then every node's label set
// to its root's: the smallest dense id of its component.  Stats: every
// node visited, every forward edge traversed.
int32_t wo_components(const wo_graph* gp, uint64_t* labels, uint64_t* nodes_visited,
                      uint64_t* edges_traversed) {
  const Graph& g = *(const Graph*)gp;
  const uint64_t n = g.fwd.n;
  std::vector<uint64_t> parent(n);
  for (uint64_t i = 0; i < n; i++) parent[i] = i;
  auto root = [&](uint64_t x) {
    while (parent[x] != x) {
      const uint64_t gp2 = parent[parent[x]];
      parent[x] = gp2;
      x = gp2;
    }
    return x;
  };
  uint64_t edges = 0;
  for (uint64_t u = 0; u < n; u++)
    for (uint64_t e = g.fwd.off[u]; e < g.fwd.off[u + 1]; e++) {
      edges++;
      const uint64_t a = root(u), b = root(g.fwd.tgt[e]);
      if (a < b) parent[b] = a;
      else parent[a] = b;
    }
  for (uint64_t i = 0; i < n; i++) parent[i] = parent[parent[i]];
  for (uint64_t i = 0; i < n; i++) labels[i] = parent[i];
  *nodes_visited = n;
  *edges_traversed = edges;
  return WC_OK;
}

// compute/centrality/sources.rs:55-123 (Sources::choose): the live nodes
// the population mask selects (nonzero, flipped by `complement`), then, if
// k >= 0 is fewer, the k whose keys mix(mix(seed) ^ node·GOLDEN) are the
// smallest (the keys are distinct), ascending by id.
int32_t wo_sample_sources(uint64_t n, const uint64_t* tomb, const uint8_t* pop, int complement,
                          int64_t k, uint64_t seed, uint64_t* out, uint64_t* count) {
  std::vector<uint64_t> eligible;
  for (uint64_t u = 0; u < n; u++)
    if (!tombstoned(tomb, u) && (!pop || ((pop[u] != 0) != (complement != 0))))
      eligible.push_back(u);
  if (k >= 0 && (uint64_t)k < eligible.size()) {
    std::vector<std::pair<uint64_t, uint64_t>> keyed;
    for (uint64_t u : eligible) keyed.push_back({mix(mix(seed) ^ (u * GOLDEN)), u});
    std::sort(keyed.begin(), keyed.end());
    eligible.clear();
    for (int64_t i = 0; i < k; i++) eligible.push_back(keyed[i].second);
    std::sort(eligible.begin(), eligible.end());
  }
  std::copy(eligible.begin(), eligible.end(), out);
  *count = eligible.size();
  return WC_OK;
}

// compute/centrality/closeness.rs with the batched measures
// (centrality/mod.rs:158-190, multi_source.rs:97-116): the sources in
// batches of 64 in their order, each searched breadth-first over the
// forward rows without a depth limit; per node, per batch, per distance d
// ascending, the count c of the batch's sources first reaching it at d adds
// c to reached, c·d to the distance sum and c / d to the harmonic sum.
// Then closeness.rs:117-132 (closeness, r / total scaled by r / others
// with wf_improved) or :229-241 (harmonic, scaled by (live - 1) / others
// for a sample); tombstoned nodes 0.
int32_t wo_centrality(const wo_graph* gp, int measure, int wf_improved, const uint64_t* sources,
                      uint64_t count, const uint64_t* tomb, double* out) {
  const Graph& g = *(const Graph*)gp;
  const uint64_t n = g.fwd.n;
  std::vector<uint64_t> reached(n, 0), dsum(n, 0);
  std::vector<double> harm(n, 0.0);
  std::vector<char> is_source(n, 0);
  for (uint64_t i = 0; i < count; i++) is_source[sources[i]] = 1;
  constexpr uint64_t kBatch = 64;
  const uint64_t kFar = ~0ull;
  std::vector<std::vector<uint64_t>> dist;
  std::vector<uint64_t> queue, cnt;
  for (uint64_t b0 = 0; b0 < count; b0 += kBatch) {
    const uint64_t bk = std::min(kBatch, count - b0);
    dist.assign(bk, std::vector<uint64_t>(n, kFar));
    uint64_t deepest = 0;
    for (uint64_t j = 0; j < bk; j++) {
      std::vector<uint64_t>& d = dist[j];
      queue.assign(1, sources[b0 + j]);
      d[sources[b0 + j]] = 0;
      for (uint64_t h = 0; h < queue.size(); h++) {
        const uint64_t u = queue[h];
        for (uint64_t e = g.fwd.off[u]; e < g.fwd.off[u + 1]; e++) {
          const uint64_t t = g.fwd.tgt[e];
          if (d[t] == kFar) {
            d[t] = d[u] + 1;
            deepest = std::max(deepest, d[t]);
            queue.push_back(t);
          }
        }
      }
    }
    cnt.assign(deepest + 1, 0);
    for (uint64_t u = 0; u < n; u++) {
      for (uint64_t j = 0; j < bk; j++)
        if (dist[j][u] != kFar && dist[j][u] > 0) cnt[dist[j][u]]++;
      for (uint64_t d = 1; d <= deepest; d++) {
        if (!cnt[d]) continue;
        reached[u] += cnt[d];
        dsum[u] += cnt[d] * d;
        harm[u] = harm[u] + (double)cnt[d] / (double)d;
        cnt[d] = 0;
      }
    }
  }
  uint64_t live = 0;
  for (uint64_t u = 0; u < n; u++) live += !tombstoned(tomb, u);
  for (uint64_t u = 0; u < n; u++) {
    double v = 0.0;
    const uint64_t others = count - (uint64_t)is_source[u];
    if (tombstoned(tomb, u)) {
      v = 0.0;
    } else if (measure == 0) {
      const double r = (double)reached[u], total = (double)dsum[u];
      if (total > 0.0 && live > 1) v = wf_improved ? r / total * (r / (double)others) : r / total;
    } else if (count == live) {
      v = harm[u];
    } else if (others != 0) {
      v = harm[u] * ((double)(live - 1) / (double)others);
    }
    out[u] = v;
  }
  return WC_OK;
}

// compute/reduce.rs: elements read as f64 (bool 0 / 1), reduced in chunks
// of 65,536 (reduce.rs:20) — sums in element order from +0, max / min
// keeping the first of equal elements in SQL order — then the chunks'
// results combined in chunk order (reduce.rs:250-268).
static double elem_f64(int dtype, const void* p, uint64_t i, uint64_t len) {
  if (i >= len) return 0.0;
  switch (dtype) {
    case 0: return (double)((const float*)p)[i];
    case 1: return ((const double*)p)[i];
    case 2: return (double)((const int64_t*)p)[i];
    default: return ((const uint8_t*)p)[i] ? 1.0 : 0.0;
  }
}

// reduction: 0 sum, 1 max, 2 min, 3 l1, 4 l2, 5 nnz; values(i) yields the
// i-th element or nothing (skipped).
static bool reduce_chunks(uint64_t len, int reduction,
                          const std::function<bool(uint64_t, double*)>& values, double* result) {
  const uint64_t kChunk = 1ull << 16;
  const bool extreme = reduction == 1 || reduction == 2;
  auto pick = [&](double a, double b) {  // greatest / least: the first on a tie
    const int c = float_cmp(b, a);
    return (reduction == 1 ? c > 0 : c < 0) ? b : a;
  };
  std::vector<std::pair<bool, double>> partials;
  for (uint64_t c0 = 0; c0 < len; c0 += kChunk) {
    bool any = false;
    double acc = 0.0;
    for (uint64_t i = c0; i < std::min(len, c0 + kChunk); i++) {
      double v;
      if (!values(i, &v)) continue;
      if (extreme) {
        acc = any ? pick(acc, v) : v;
      } else {
        const double term = reduction == 3 ? std::fabs(v) : reduction == 4 ? v * v
                          : reduction == 5 ? (v != 0.0 ? 1.0 : 0.0) : v;
        acc = acc + term;
      }
      any = true;
    }
    partials.push_back({extreme ? any : true, acc});
  }
  bool any = false;
  double out = 0.0;
  for (auto& p : partials) {
    if (!p.first) continue;
    out = extreme ? (any ? pick(out, p.second) : p.second) : out + p.second;
    any = true;
  }
  if (reduction == 4) out = std::sqrt(out);
  *result = out;
  return extreme ? any : true;
}

int32_t wo_reduce(int dtype, const void* x, uint64_t n, uint64_t width, const uint64_t* tomb,
                  int reduction, double* result, int32_t* is_null) {
  const uint64_t len = n * width;
  const bool found = reduce_chunks(len, reduction, [&](uint64_t i, double* v) {
    if (tombstoned(tomb, i / width)) return false;
    *v = elem_f64(dtype, x, i, len);
    return true;
  }, result);
  *is_null = !found;
  return WC_OK;
}

// reduce.rs:175-206 (norm_diff): 0 l1, 1 l2, 2 linf of a − b, a row past
// the shorter vector's end read as zero; 0 for no elements.
int32_t wo_norm_diff(int dtype_a, const void* a, uint64_t na, int dtype_b, const void* b,
                     uint64_t nb, uint64_t width, int norm, double* result) {
  const uint64_t la = na * width, lb = nb * width, len = std::max(la, lb);
  const int reduction = norm == 0 ? 3 : norm == 1 ? 4 : 1;
  const bool found = reduce_chunks(len, reduction, [&](uint64_t i, double* v) {
    const double d = elem_f64(dtype_a, a, i, la) - elem_f64(dtype_b, b, i, lb);
    *v = norm == 2 ? std::fabs(d) : d;
    return true;
  }, result);
  if (!found) *result = 0.0;
  return WC_OK;
}

// compute/centrality/betweenness.rs with paths.rs:148-260 (unweighted):
// per source in the given order, a breadth-first search over the forward
// rows counting shortest paths (f64), then the dependencies in reverse
// search order, each row's out-neighbours in ascending order; every node's
// total gains each source's dependency in source order (the source none,
// or with endpoints the other nodes it reaches, every reached node one
// more); then betweenness.rs:113-141's rescale; tombstoned nodes 0.
int32_t wo_betweenness(const wo_graph* gp, const uint64_t* sources, uint64_t count,
                       const uint64_t* tomb, int normalized, int endpoints, int directed,
                       double* out) {
  const Graph& g = *(const Graph*)gp;
  const uint64_t n = g.fwd.n;
  std::vector<double> total(n, 0.0), dist(n, INFINITY), sigma(n, 0.0), dep(n, 0.0);
  std::vector<uint64_t> order;
  for (uint64_t q = 0; q < count; q++) {
    const uint64_t s = sources[q];
    for (uint64_t v : order) dist[v] = INFINITY, sigma[v] = 0.0, dep[v] = 0.0;
    order.assign(1, s);
    dist[s] = 0.0;
    sigma[s] = 1.0;
    for (size_t h = 0; h < order.size(); h++) {
      const uint64_t u = order[h];
      const double through = dist[u] + 1.0;
      for (uint64_t e = g.fwd.off[u]; e < g.fwd.off[u + 1]; e++) {
        const uint64_t t = g.fwd.tgt[e];
        if (dist[t] == INFINITY) {
          dist[t] = through;
          order.push_back(t);
        }
        if (dist[t] == through) sigma[t] += sigma[u];
      }
    }
    for (size_t h = order.size(); h-- > 0;) {
      const uint64_t v = order[h];
      double gained = 0.0;
      for (uint64_t e = g.fwd.off[v]; e < g.fwd.off[v + 1]; e++) {
        const uint64_t w = g.fwd.tgt[e];
        if (w != v && dist[v] + 1.0 == dist[w]) gained += sigma[v] / sigma[w] * (1.0 + dep[w]);
      }
      dep[v] = gained;
    }
    dep[s] = 0.0;
    if (endpoints) {
      for (size_t h = 1; h < order.size(); h++) dep[order[h]] += 1.0;
      dep[s] = (double)(order.size() - 1);
    }
    for (uint64_t v = 0; v < n; v++) total[v] += dep[v];
  }
  uint64_t live = 0;
  for (uint64_t v = 0; v < n; v++) live += !tombstoned(tomb, v);
  const bool every = count == live;
  const __int128 pairs = (__int128)live - (endpoints ? 0 : 1);
  double fs = 1.0, fo = 1.0;
  if (pairs >= 2) {
    const __int128 corr = directed ? 1 : 2, ks = every ? pairs : (__int128)count;
    auto factor = [&](__int128 k) {
      return normalized ? 1.0 / (double)(k * (pairs - 1)) : (double)pairs / (double)(k * corr);
    };
    fo = factor(ks);
    fs = (every || endpoints) ? fo : (ks > 1 ? factor(ks - 1) : NAN);
  }
  std::vector<char> is_source(n, 0);
  if (!every)
    for (uint64_t q = 0; q < count; q++) is_source[sources[q]] = 1;
  for (uint64_t v = 0; v < n; v++)
    out[v] = tombstoned(tomb, v) ? 0.0 : total[v] * (is_source[v] ? fs : fo);
  return WC_OK;
}

// compute/ranking.rs:15-80 (top_k) over f64 values.
int32_t wo_topk_f64(const double* x, uint64_t n, const uint64_t* tomb, uint64_t k, int descending,
                    uint64_t* nodes, double* values, uint64_t* count) {
  // better(a, b): a orders first.
  auto better = [&](uint64_t a, uint64_t b) {
    int c = descending ? float_cmp(x[b], x[a]) : float_cmp(x[a], x[b]);
    return c != 0 ? c < 0 : a < b;
  };
  std::vector<uint64_t> live;
  for (uint64_t i = 0; i < n; i++)
    if (!tombstoned(tomb, i)) live.push_back(i);
  uint64_t kept = std::min<uint64_t>(k, live.size());
  std::partial_sort(live.begin(), live.begin() + kept, live.end(), better);
  for (uint64_t i = 0; i < kept; i++) {
    nodes[i] = live[i];
    values[i] = x[live[i]];
  }
  *count = kept;
  return WC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- adjoint
// An FP64 CPU adjoint of the uniform PageRank above (no reference
// counterpart: the reference has no derivative).  At the fixed point
// x = d·(Aᵀ D⁻¹ x + (uᵀx)·p) + (1 − d)·p (D = diag(out), u the dangling
// rows, p = 1/live), a loss L = cᵀx has the adjoint λ = d·(D⁻¹Aλ + u·(pᵀλ))
// + c, solved here by the same power iteration, and
//   ∂L/∂w_ij = d · x_i / out_i · (λ_j − Σ_k (w_ik / out_i) λ_k).
// The forward solve is wo_pagerank's.
extern "C" int32_t wo_pagerank_adjoint(const wo_graph* gp, double damping, int has_tol, double tol,
                                       uint32_t max_iter, const uint64_t* targets,
                                       const uint64_t* offsets, uint32_t losses, double adjoint_tol,
                                       double* grad, double* ranks, uint32_t* iterations) {
  const Graph& g = *(const Graph*)gp;
  const uint64_t n = g.fwd.n, m = g.fwd.tgt.size();
  PageRankOpts o;
  o.damping = damping;
  o.has_tol = has_tol != 0;
  o.tol = tol;
  o.max_iter = max_iter;
  std::vector<double> x(n);
  uint32_t it = 0;
  Status s = pagerank(g, nullptr, o, x.data(), &it, nullptr, nullptr);
  if (s) return s;
  if (ranks) std::copy(x.begin(), x.end(), ranks);
  if (iterations) iterations[0] = it;
  std::vector<double> out(n, 0.0);
  for (uint64_t i = 0; i < n; i++)
    for (uint64_t e = g.fwd.off[i]; e < g.fwd.off[i + 1]; e++)
      out[i] = (e == g.fwd.off[i]) ? (g.fwd.weighted() ? g.fwd.w[e] : 1.0)
                                   : out[i] + (g.fwd.weighted() ? g.fwd.w[e] : 1.0);
  const double p = 1.0 / (double)n;
  uint32_t max_adj = 0;
  for (uint32_t c = 0; c < losses; c++) {
    std::vector<double> cvec(n, 0.0), lam(n), next(n), srow(n);
    for (uint64_t q = offsets[c]; q < offsets[c + 1]; q++) cvec[targets[q]] += 1.0;
    lam = cvec;
    uint32_t t = 0;
    for (; t < max_iter; t++) {
      double pl = 0.0;
      for (uint64_t i = 0; i < n; i++) pl += p * lam[i];
      double change = 0.0;
      for (uint64_t i = 0; i < n; i++) {
        double z = 0.0;
        for (uint64_t e = g.fwd.off[i]; e < g.fwd.off[i + 1]; e++)
          z += (g.fwd.weighted() ? g.fwd.w[e] : 1.0) * lam[g.fwd.tgt[e]];
        const double si = out[i] > 0.0 ? z / out[i] : 0.0;
        next[i] = damping * (si + (out[i] > 0.0 ? 0.0 : pl)) + cvec[i];
        change += std::fabs(next[i] - lam[i]);
      }
      lam.swap(next);
      if (change < adjoint_tol) {
        t++;
        break;
      }
    }
    max_adj = std::max(max_adj, t);
    for (uint64_t i = 0; i < n; i++) {
      double z = 0.0;
      for (uint64_t e = g.fwd.off[i]; e < g.fwd.off[i + 1]; e++)
        z += (g.fwd.weighted() ? g.fwd.w[e] : 1.0) * lam[g.fwd.tgt[e]];
      srow[i] = out[i] > 0.0 ? z / out[i] : 0.0;
    }
    for (uint64_t i = 0; i < n; i++)
      for (uint64_t e = g.fwd.off[i]; e < g.fwd.off[i + 1]; e++)
        grad[(uint64_t)c * m + e] = damping * x[i] / out[i] * (lam[g.fwd.tgt[e]] - srow[i]);
  }
  if (iterations) iterations[1] = max_adj;
  return WC_OK;
}
