// eigen.cu — wc_eigen: spectral/lanczos.rs:206-743 on the device, f64.
//
// Thick-restart Lanczos with full reorthogonalisation, as the reference runs
// it: a basis of max(2k+1, 20) vectors (at most the dimension); each step
// applies the operator to the newest vector, removes the three-term
// recurrence and makes one classical Gram–Schmidt pass against the whole
// basis (two after a restart or a random vector), then projects out the
// connected components' exact eigenvectors; when the basis is full the
// Rayleigh–Ritz pairs of H = QᵀMQ decide convergence (|β·s_last| ≤
// tol·max|θ|) or a restart onto the wanted Ritz vectors plus one per
// converged pair (clamped to a quarter..half of the rest).
//
// On the device: the operator (spectral/operator.rs:117-395: degrees, active
// nodes, D^-1/2 scaling, (A + Aᵀ)/2 unless A = Aᵀ), every O(n·basis) pass
// (projections, subtraction with the norm, rotation, combination) with
// reductions in a fixed order, and the components (min-label propagation
// with path compression; roots are each component's lowest node, which
// numbers them as spectral/components.rs does).  On the host: the dense
// symmetric eigensolve of H (≤ 41 × 41), by cyclic Jacobi rotations, where
// the reference calls nalgebra's SymmetricEigen (spectral/ritz.rs:34-52).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "bfs.h"
#include "operand.h"
#include "product.h"
#include "runtime.cuh"
#include "semiring.cuh"

namespace wc {

wc_status prepare_pull(Ctx& ctx, DevCsr& csr, int semiring, int weighted_flag, int dtype,
                       uint32_t width, PullLaunch& L);
wc_status launch_pull(const PullLaunch& L, int dtype, const void* x, void* y);

constexpr double kF64Tie = 1e-12;        // lanczos.rs:52
constexpr double kF64Breakdown = 1e-10;  // lanczos.rs:65
constexpr size_t kStepsPerBasisVector = 1000;
constexpr size_t kMinBasis = 20;
constexpr double kSymmetryTolerance = 1e-9;
constexpr uint64_t kSymmetrySeed = 0x53594d4d;
constexpr int kRedBlocks = 592;  // blocks of the fixed-order reductions

// ------------------------------------------------------------ reductions

// Σ f(i) over n, deterministic: each block a fixed share, then blocks in
// order (second kernel).
template <class F>
__global__ void sum_partial_kernel(uint32_t n, F f, double* partial) {
  __shared__ double s[32];
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += f(i);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned w = 0; w < blockDim.x / 32; w++) t += s[w];
    partial[blockIdx.x] = t;
  }
}

// out[c] = Σ_b partial[b * columns + c], b in order.  One block: the
// partials are first brought into shared memory by every thread (coalesced
// loads, all in flight at once), then each column is added up in block
// order by one thread from there, so the dependent chain of additions waits
// on shared memory rather than on L2.
constexpr uint32_t kSumFinalMaxValues = kRedBlocks * 8;  // count × columns
__global__ void __launch_bounds__(256) sum_final_kernel(const double* partial, uint32_t count,
                                                        uint32_t columns, double* out) {
  __shared__ double sp[kSumFinalMaxValues];
  // Block b combines the b-th run of count × columns partials into
  // out[b·columns ..): several projections' partials in one launch.
  partial += (size_t)blockIdx.x * count * columns;
  out += (size_t)blockIdx.x * columns;
  const uint32_t total = count * columns;
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) sp[i] = partial[i];
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < columns; c += blockDim.x) {
    double t = 0.0;
    for (uint32_t b = 0; b < count; b++) t += sp[b * columns + c];
    out[c] = t;
  }
}

// Qᵀw for vectors [j0, j0 + 8) of Q (column-major, n rows each), with an
// optional pending update w -= c·q_p first (done by the same pass).
__global__ void project_kernel(uint32_t n, const double* Q, uint32_t len, uint32_t j0, double* w,
                               int pending, double pending_c, double* partial) {
  __shared__ double s[8][8];
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; q++) acc[q] = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double wi = w[i];
    if (pending >= 0 && j0 == 0) {
      wi -= pending_c * Q[(size_t)pending * n + i];
      w[i] = wi;
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (j0 + q < len) acc[q] += wi * Q[(size_t)(j0 + q) * n + i];
  }
#pragma unroll
  for (int q = 0; q < 8; q++)
    for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < 8; q++) s[threadIdx.x >> 5][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (unsigned wv = 0; wv < blockDim.x / 32; wv++) t += s[wv][threadIdx.x];
    partial[(size_t)blockIdx.x * 8 + threadIdx.x] = t;
  }
}

// w -= Σ_j c_j q_j (j in order), with Σ w² after.
__global__ void subtract_kernel(uint32_t n, const double* Q, const double* c, uint32_t len,
                                double* w, double* partial) {
  __shared__ double s[32];
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double wi = w[i];
    for (uint32_t j = 0; j < len; j++) wi -= c[j] * Q[(size_t)j * n + i];
    w[i] = wi;
    acc += wi * wi;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned wv = 0; wv < blockDim.x / 32; wv++) t += s[wv];
    partial[blockIdx.x] = t;
  }
}

// w -= β q_{j-1}; partial dots with q_j.
__global__ void recurrence_kernel(uint32_t n, const double* qprev, const double* qj, double beta,
                                  double* w, double* partial) {
  __shared__ double s[32];
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double wi = w[i] - beta * qprev[i];
    w[i] = wi;
    acc += wi * qj[i];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned wv = 0; wv < blockDim.x / 32; wv++) t += s[wv];
    partial[blockIdx.x] = t;
  }
}

// Q'[:, l] = Σ_j V[j][l] q_j for l < kept (j in basis order), into `out`.
__global__ void rotate_kernel(uint32_t n, const double* Q, const double* V, uint32_t len,
                              uint32_t ldv, uint32_t kept, double* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double q[64];
    for (uint32_t j = 0; j < len; j++) q[j] = Q[(size_t)j * n + i];
    for (uint32_t l = 0; l < kept; l++) {
      double sum = 0.0;
      for (uint32_t j = 0; j < len; j++) sum += V[(size_t)j * ldv + l] * q[j];
      out[(size_t)l * n + i] = sum;
    }
  }
}

// ------------------------------------------------------------ operator

struct OpState {
  uint32_t n;
  int op;
  bool transpose;
  const uint8_t* active;
  const double* degrees;
  const double* scale;
};

__global__ void fill_kernel(double* x, uint32_t n, double v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

__global__ void average_kernel(double* y, const double* y2, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = (y[i] + y2[i]) / 2.0;
}

__global__ void scale_kernel(const double* x, const double* scale, double* out, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = scale[i] * x[i];
}

// operator.rs:234-262: the operator's output from y = S·(scaled) input.
__global__ void finish_apply_kernel(OpState o, const double* x, double* y) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    switch (o.op) {
      case WC_LAPLACIAN: y[i] = o.degrees[i] * x[i] - y[i]; break;
      case WC_NORMALIZED_LAPLACIAN: y[i] = x[i] - o.scale[i] * y[i]; break;
      case WC_RANDOM_WALK: y[i] = o.scale[i] * y[i]; break;
      default: break;
    }
  }
}

__global__ void measure_kernel(const double* counts, const double* degrees, uint32_t n,
                               uint8_t* active, double* scale, int normalized, DeviceError* err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool a = counts[i] > 0.0;
    active[i] = a;
    if (normalized) {
      const double d = degrees[i];
      if (a && (d != d || d <= 0.0)) raise(err, WC_NON_POSITIVE_DEGREE, i);
      scale[i] = a ? 1.0 / sqrt(d) : 0.0;
    }
  }
}

__device__ inline double uniform_dev(uint64_t seed, uint64_t stream, uint64_t node) {
  auto mix = [](uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  const uint64_t golden = 0x9e3779b97f4a7c15ull;
  const uint64_t bits = mix(mix(seed ^ mix(stream * golden)) ^ (node * golden));
  return (double)(bits >> 11) / (double)(1ull << 52) - 1.0;
}

// compute/random.rs:20-25 at active nodes, zero elsewhere.
__global__ void random_kernel(double* x, const uint8_t* active, uint32_t n, uint64_t seed,
                              uint64_t stream, int all) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = (all || active[i]) ? uniform_dev(seed, stream, i) : 0.0;
}

// ------------------------------------------------------------ components

__global__ void cc_init_kernel(uint32_t* parent, const uint8_t* active, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    parent[i] = i;
}

// Hooks the larger of an edge's two roots under the smaller.
__global__ void cc_hook_kernel(const uint32_t* off, const uint32_t* tgt, const uint8_t* active,
                               uint32_t n, uint32_t* parent, int* changed) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  bool hooked = false;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    if (!active[u]) continue;
    const uint32_t lo = off[u], hi = off[u + 1];
    for (uint32_t e = lo + lane; e < hi; e += 32) {
      const uint32_t v = tgt[e];
      if (!active[v]) continue;
      uint32_t a = parent[u], b = parent[v];
      while (a != parent[a]) a = parent[a];
      while (b != parent[b]) b = parent[b];
      if (a != b) {
        atomicMin(parent + max(a, b), min(a, b));
        hooked = true;
      }
    }
  }
  // One write of the flag a warp (every edge writing it contended on one
  // address).
  if (__any_sync(0xffffffffu, hooked) && lane == 0) *changed = 1;
}

__global__ void cc_compress_kernel(uint32_t* parent, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t r = parent[i];
    while (r != parent[r]) r = parent[r];
    parent[i] = r;
  }
}

// unit[i]: component weight (√d for the normalised operators, else 1) at
// active nodes; norms[c] += unit², per component.
__global__ void unit_kernel(uint32_t n, const uint8_t* active, const uint32_t* comp,
                            const double* degrees, int normalized, double* unit, double* norms) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double w = 0.0;
    if (active[i]) {
      w = normalized ? sqrt(degrees[i]) : 1.0;
      atomicAdd(norms + comp[i], w * w);
    }
    unit[i] = w;
  }
}

__global__ void unit_normalize_kernel(uint32_t n, const uint8_t* active, const uint32_t* comp,
                                      const double* norms, double* unit) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (active[i] && unit[i] != 0.0) unit[i] /= sqrt(norms[comp[i]]);
}

// Deflation coefficients: coef[c][0] += u·x, coef[c][1] += sign·u·x, with a
// small per-block table so a large component costs one atomic per block.
__global__ void deflate_coef_kernel(uint32_t n, const uint8_t* active, const uint32_t* comp,
                                    const uint8_t* colour, const double* unit, const double* x,
                                    double* coef) {
  __shared__ uint32_t key[64];
  __shared__ double val[64][2];
  for (uint32_t s = threadIdx.x; s < 64; s += blockDim.x) {
    key[s] = 0xffffffffu;
    val[s][0] = val[s][1] = 0.0;
  }
  __syncthreads();
  // Adds (a, b) for component c into the block's table, or into coef when
  // the table's slot holds another component.
  auto add = [&](uint32_t c, double a, double b) {
    const uint32_t slot = c & 63;
    uint32_t prev = atomicCAS(&key[slot], 0xffffffffu, c);
    if (prev == 0xffffffffu || prev == c) {
      atomicAdd(&val[slot][0], a);
      atomicAdd(&val[slot][1], b);
    } else {
      atomicAdd(coef + 2 * (size_t)c, a);
      atomicAdd(coef + 2 * (size_t)c + 1, b);
    }
  };
  // A warp takes 32 consecutive nodes a step.  When every active node among
  // them lies in one component (the common case: a large component's nodes
  // are numbered together), the warp sums them with shuffles and one lane
  // adds the sums; otherwise each active lane adds its own.
  const unsigned lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < n; i0 += stride) {
    const uint32_t i = i0 + lane;
    const bool live = i < n && active[i];
    uint32_t c = 0xffffffffu;
    double a = 0.0, b = 0.0;
    if (live) {
      c = comp[i];
      a = unit[i] * x[i];
      b = (colour && colour[i]) ? -a : a;
    }
    const unsigned lm = __ballot_sync(0xffffffffu, live);
    if (!lm) continue;
    const uint32_t c_first = __shfl_sync(0xffffffffu, c, __ffs(lm) - 1);
    if (__all_sync(0xffffffffu, !live || c == c_first)) {
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
      }
      if (lane == 0) add(c_first, a, b);
    } else if (live) {
      add(c, a, b);
    }
  }
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < 64; s += blockDim.x)
    if (key[s] != 0xffffffffu) {
      atomicAdd(coef + 2 * (size_t)key[s], val[s][0]);
      atomicAdd(coef + 2 * (size_t)key[s] + 1, val[s][1]);
    }
}

// x -= unit·(connected·coef[c][0] + alternating·sign·coef[c][1] if bipartite).
__global__ void deflate_apply_kernel(uint32_t n, const uint8_t* active, const uint32_t* comp,
                                     const uint8_t* colour, const uint8_t* bipartite,
                                     const double* unit, const double* coef, double connected,
                                     double alternating, double* x) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!active[i]) continue;
    const uint32_t c = comp[i];
    const double along = connected * coef[2 * (size_t)c];
    double across = 0.0;
    if (bipartite && bipartite[c]) {
      const double sign = (colour && colour[i]) ? -1.0 : 1.0;
      across = alternating * sign * coef[2 * (size_t)c + 1];
    }
    x[i] -= unit[i] * (along + across);
  }
}

// A known pair's vector: unit on component c (signed by colour when
// alternating), zero elsewhere.
__global__ void known_vector_kernel(uint32_t n, const uint8_t* active, const uint32_t* comp,
                                    const uint8_t* colour, const double* unit, uint32_t c,
                                    int alternating, double* x) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (active[i] && comp[i] == c) v = (alternating && colour && colour[i]) ? -unit[i] : unit[i];
    x[i] = v;
  }
}

// Settles x (lanczos.rs:726-743): the entry of largest magnitude, the
// first on ties, is found in two passes: the largest magnitude (a max is
// exact in any order), then the lowest index holding it.
__global__ void max_abs_kernel(const double* x, uint32_t n, double* partial) {
  __shared__ double s[32];
  double m = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned w = 0; w < blockDim.x / 32; w++) t = fmax(t, s[w]);
    partial[blockIdx.x] = t;
  }
}

__global__ void first_at_kernel(const double* x, uint32_t n, double m, unsigned* index) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (fabs(x[i]) == m) atomicMin(index, i);
}

__global__ void scale_vec_kernel(double* x, uint32_t n, double f) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] *= f;
}

__global__ void residual_terms_kernel(const double* x, const double* y, double value, uint32_t n,
                                      double* partial) {
  __shared__ double s[32];
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = y[i] - value * x[i];
    acc += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned w = 0; w < blockDim.x / 32; w++) t += s[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void copy_kernel(const double* a, double* b, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// ------------------------------------------------------------ host side

// Cyclic Jacobi eigen-decomposition of a symmetric n × n matrix (row-major
// a, destroyed): values in `w`, vectors as the columns of `v` (row-major).
static bool jacobi(std::vector<double>& a, size_t n, std::vector<double>& w, std::vector<double>& v) {
  v.assign(n * n, 0.0);
  for (size_t i = 0; i < n; i++) v[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (size_t p = 0; p < n; p++)
      for (size_t q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
    if (off == 0.0) break;
    for (size_t p = 0; p < n; p++)
      for (size_t q = p + 1; q < n; q++) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        const double app = a[p * n + p], aqq = a[q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (size_t k = 0; k < n; k++) {
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (size_t k = 0; k < n; k++) {
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (size_t k = 0; k < n; k++) {
          const double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (size_t i = 0; i < n; i++) {
    w[i] = a[i * n + i];
    if (!std::isfinite(w[i])) return false;
  }
  return true;
}

// ritz.rs:59-92: indexes in `which` order, the earlier first on ties; for
// Largest, runs of magnitudes within tie·max|θ| list positives first.
static std::vector<size_t> order_values(const std::vector<double>& values, int which, double tie) {
  std::vector<size_t> order(values.size());
  std::iota(order.begin(), order.end(), 0);
  auto total_cmp = [](double a, double b) {  // f64::total_cmp for non-NaN
    if (a < b) return -1;
    if (a > b) return 1;
    return std::signbit(a) == std::signbit(b) ? 0 : (std::signbit(a) ? -1 : 1);
  };
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    const double a = values[x], b = values[y];
    int c;
    if (which == WC_LARGEST) {
      c = total_cmp(std::fabs(b), std::fabs(a));
      if (c == 0) c = total_cmp(b, a);
    } else {
      c = total_cmp(a, b);
    }
    return c < 0;
  });
  if (which == WC_LARGEST) {
    double m = 0.0;
    for (double v : values) m = std::max(m, std::fabs(v));
    const double width = tie * m;
    size_t start = 0;
    while (start < order.size()) {
      const double first = std::fabs(values[order[start]]);
      size_t end = start;
      while (end < order.size() && !(first - std::fabs(values[order[end]]) > width)) end++;
      std::stable_sort(order.begin() + start, order.begin() + end,
                       [&](size_t x, size_t y) { return !(values[x] < 0.0) && values[y] < 0.0; });
      start = end;
    }
  }
  return order;
}

struct Pair {
  double value, residual;
  std::vector<double> vector;  // host copy when asked for; else empty
  bool known;
};

struct Eigensolver {
  Ctx& ctx;
  wc_version* v;
  wc_eigen_opts o;
  uint32_t n;
  bool normalized;
  OpState op;
  DevBuf *input, *output, *scratch, *scaled, *active, *degrees, *scale, *partial, *coefbuf;
  DevBuf *Q = nullptr, *Q2 = nullptr, *parent = nullptr, *comp = nullptr, *unit = nullptr,
         *colour = nullptr, *bip = nullptr, *dcoef = nullptr, *vbuf = nullptr;
  uint64_t dimension = 0, components = 0;
  bool deflating = false, nonnegative = true;
  double connected_flag = 0.0, alternating_flag = 0.0;
  bool has_connected = false, has_bipartite = false;
  double known_connected = 0.0, known_bipartite = 0.0;
  uint64_t deflated_count = 0;
  std::vector<uint8_t> bipartite_host;
  uint32_t grid;

  Eigensolver(Ctx& c, const wc_eigen_opts& opts) : ctx(c), v(c.v), o(opts) {
    n = (uint32_t)v->n;
    normalized = o.op == WC_NORMALIZED_LAPLACIAN || o.op == WC_RANDOM_WALK;
    grid = kRedBlocks;
  }

  cudaStream_t st() const { return ctx.stream; }

  wc_status sum_final(uint32_t count, uint32_t columns, double* out_host) {
    if ((uint64_t)count * columns > kSumFinalMaxValues) return WC_INVALID_ARGUMENT;
    note_launch(), sum_final_kernel<<<1, 256, 0, st()>>>(partial->as<double>(), count, columns,
                                                         coefbuf->as<double>());
    WC_CUDA(cudaMemcpyAsync(out_host, coefbuf->ptr, columns * 8, cudaMemcpyDeviceToHost, st()),
            ctx.detail);
    WC_CUDA(cudaStreamSynchronize(st()), ctx.detail);
    return WC_OK;
  }

  wc_status dot_self(const double* x, double* out) {
    auto f = [x] __device__(uint32_t i) { return x[i] * x[i]; };
    note_launch(), sum_partial_kernel<<<grid, 256, 0, st()>>>(n, f, partial->as<double>());
    return sum_final(grid, 1, out);
  }

  // y = S·x (S = A or (A + Aᵀ)/2), weighted as asked.
  wc_status multiply(const double* x, double* y, int weighted) {
    PullLaunch L;
    WC_TRY(prepare_pull(ctx, v->fwd, WC_PLUS_TIMES, weighted, WC_F64, 1, L));
    WC_TRY(launch_pull(L, WC_F64, x, y));
    if (op.transpose) {
      PullLaunch R;
      WC_TRY(prepare_pull(ctx, v->rev, WC_PLUS_TIMES, weighted, WC_F64, 1, R));
      WC_TRY(launch_pull(R, WC_F64, x, scratch->ptr));
      note_launch(), average_kernel<<<grid, 256, 0, st()>>>(y, scratch->as<double>(), n);
    }
    return WC_OK;
  }

  // output = M·x (operator.rs:234-262).
  wc_status apply(const double* x, double* out) {
    const double* src = x;
    if (normalized) {
      note_launch(), scale_kernel<<<grid, 256, 0, st()>>>(x, scale->as<double>(), scaled->as<double>(), n);
      src = scaled->as<double>();
    }
    WC_TRY(multiply(src, out, o.weighted));
    note_launch(), finish_apply_kernel<<<grid, 256, 0, st()>>>(op, x, out);
    return WC_OK;
  }

  wc_status setup() {
    const uint64_t nb = (uint64_t)n * 8;
    WC_TRY(ctx.scratch(POOL_EIG_0, nb, &input));
    WC_TRY(ctx.scratch(POOL_EIG_1, nb, &output));
    WC_TRY(ctx.scratch(POOL_EIG_2, nb, &scratch));
    WC_TRY(ctx.scratch(POOL_EIG_3, nb, &scaled));
    WC_TRY(ctx.scratch(POOL_EIG_4, n, &active));
    WC_TRY(ctx.scratch(POOL_EIG_5, nb, &degrees));
    WC_TRY(ctx.scratch(POOL_EIG_6, nb, &scale));
    WC_TRY(ctx.scratch(POOL_EIG_7, (uint64_t)grid * 8 * 8, &partial));
    WC_TRY(ctx.scratch(POOL_EIG_8, 64 * 8, &coefbuf));
    op = OpState{n, (int)o.op, o.symmetrize && !v->symmetric, active->as<uint8_t>(),
                 degrees->as<double>(), scale->as<double>()};
    // Freivalds' check when not symmetrising (operator.rs:371-395).
    if (!o.symmetrize && !v->symmetric) {
      note_launch(), random_kernel<<<grid, 256, 0, st()>>>(input->as<double>(), nullptr, n, kSymmetrySeed, 0, 1);
      PullLaunch L, R;
      WC_TRY(prepare_pull(ctx, v->fwd, WC_PLUS_TIMES, o.weighted, WC_F64, 1, L));
      WC_TRY(launch_pull(L, WC_F64, input->ptr, output->ptr));
      WC_TRY(prepare_pull(ctx, v->rev, WC_PLUS_TIMES, o.weighted, WC_F64, 1, R));
      WC_TRY(launch_pull(R, WC_F64, input->ptr, scratch->ptr));
      std::vector<double> ax(n), atx(n);
      WC_CUDA(cudaMemcpy(ax.data(), output->ptr, nb, cudaMemcpyDeviceToHost), ctx.detail);
      WC_CUDA(cudaMemcpy(atx.data(), scratch->ptr, nb, cudaMemcpyDeviceToHost), ctx.detail);
      double size = 0.0, diff = 0.0;
      bool nan = false;
      for (uint32_t i = 0; i < n; i++) {
        size = std::max(size, std::max(std::fabs(ax[i]), std::fabs(atx[i])));
        const double d = std::fabs(ax[i] - atx[i]);
        if (d != d) nan = true;
        diff = std::max(diff, d);
      }
      if (nan || diff > kSymmetryTolerance * size) return WC_NOT_SYMMETRIC;
    }
    // Active nodes and degrees (operator.rs:336-369).
    note_launch(), fill_kernel<<<grid, 256, 0, st()>>>(input->as<double>(), n, 1.0);
    WC_TRY(multiply(input->as<double>(), output->as<double>(), 0));
    WC_CUDA(cudaMemcpyAsync(scaled->ptr, output->ptr, nb, cudaMemcpyDeviceToDevice, st()), ctx.detail);
    WC_TRY(multiply(input->as<double>(), degrees->as<double>(), o.weighted));
    note_launch(), measure_kernel<<<grid, 256, 0, st()>>>(scaled->as<double>(), degrees->as<double>(), n,
                                           active->as<uint8_t>(), scale->as<double>(), normalized,
                                           v->error.as<DeviceError>());
    DeviceError e;
    WC_CUDA(cudaMemcpyAsync(&e, v->error.ptr, sizeof e, cudaMemcpyDeviceToHost, st()), ctx.detail);
    WC_CUDA(cudaStreamSynchronize(st()), ctx.detail);
    if (e.status) {
      if (ctx.detail) ctx.detail->node = e.aux;
      return (wc_status)e.status;
    }
    std::vector<uint8_t> act(n);
    WC_CUDA(cudaMemcpy(act.data(), active->ptr, n, cudaMemcpyDeviceToHost), ctx.detail);
    dimension = 0;
    for (uint8_t a : act) dimension += a;
    return WC_OK;
  }

  // The components of the active nodes, numbered by lowest node, with
  // colours and bipartiteness when the known bipartite eigenvalue is wanted.
  wc_status find_components(bool need_colours) {
    WC_TRY(ctx.scratch(POOL_EIG_9, (uint64_t)n * 4, &parent));
    WC_TRY(ctx.scratch(POOL_ADJ_0, (uint64_t)n * 4, &comp));
    DevBuf* flag;
    WC_TRY(ctx.scratch(POOL_ADJ_1, 16, &flag));
    uint32_t* par = parent->as<uint32_t>();
    note_launch(), cc_init_kernel<<<grid, 256, 0, st()>>>(par, active->as<uint8_t>(), n);
    int* changed = flag->as<int>();
    for (int round = 0; round < 1000; round++) {
      WC_CUDA(cudaMemsetAsync(changed, 0, 4, st()), ctx.detail);
      note_launch(), cc_hook_kernel<<<max_blocks(8), 256, 0, st()>>>(v->fwd.offsets.as<uint32_t>(),
                                                      v->fwd.targets.as<uint32_t>(),
                                                      active->as<uint8_t>(), n, par, changed);
      note_launch(), cc_compress_kernel<<<grid, 256, 0, st()>>>(par, n);
      int h = 0;
      WC_CUDA(cudaMemcpyAsync(&h, changed, 4, cudaMemcpyDeviceToHost, st()), ctx.detail);
      WC_CUDA(cudaStreamSynchronize(st()), ctx.detail);
      if (!h) break;
    }
    // Number the roots (active, own parent) in node order.
    std::vector<uint32_t> ph(n);
    std::vector<uint8_t> act(n);
    WC_CUDA(cudaMemcpy(ph.data(), par, (uint64_t)n * 4, cudaMemcpyDeviceToHost), ctx.detail);
    WC_CUDA(cudaMemcpy(act.data(), active->ptr, n, cudaMemcpyDeviceToHost), ctx.detail);
    std::vector<uint32_t> number(n, 0);
    components = 0;
    for (uint32_t i = 0; i < n; i++)
      if (act[i] && ph[i] == i) number[i] = (uint32_t)components++;
    std::vector<uint32_t> cm(n, 0);
    for (uint32_t i = 0; i < n; i++) cm[i] = act[i] ? number[ph[i]] : 0;
    WC_CUDA(cudaMemcpy(comp->ptr, cm.data(), (uint64_t)n * 4, cudaMemcpyHostToDevice), ctx.detail);
    colour = bip = nullptr;
    bipartite_host.assign(components, 0);
    if (need_colours) {
      // Two-colour each component from its root by BFS over both
      // directions; a component is bipartite when no edge joins equal
      // colours (a self-loop never does).
      std::vector<uint64_t> roots;
      for (uint32_t i = 0; i < n; i++)
        if (act[i] && ph[i] == i) roots.push_back(i);
      Search s;
      WC_TRY(s.run(ctx, WC_BOTH, roots.data(), roots.size(), WC_UNREACHED, nullptr, GPU_SWITCH));
      std::vector<uint32_t> depth(n);
      WC_CUDA(cudaMemcpy(depth.data(), s.depth_p, (uint64_t)n * 4, cudaMemcpyDeviceToHost), ctx.detail);
      std::vector<uint8_t> col(n, 0);
      for (uint32_t i = 0; i < n; i++) col[i] = act[i] && depth[i] != WC_UNREACHED ? (depth[i] & 1) : 0;
      std::vector<uint64_t> off(v->host_offsets);
      std::vector<uint32_t> tgt(v->m);
      WC_CUDA(cudaMemcpy(tgt.data(), v->fwd.targets.ptr, v->m * 4, cudaMemcpyDeviceToHost), ctx.detail);
      std::vector<uint8_t> odd(components, 0);
      for (uint32_t u = 0; u < n; u++) {
        if (!act[u]) continue;
        for (uint64_t e = off[u]; e < off[u + 1]; e++) {
          const uint32_t w = tgt[e];
          if (act[w] && col[w] == col[u]) odd[cm[u]] = 1;
        }
      }
      for (uint64_t c = 0; c < components; c++) bipartite_host[c] = !odd[c];
      WC_TRY(ctx.scratch(POOL_ADJ_2, n, &colour));
      WC_TRY(ctx.scratch(POOL_ADJ_3, std::max<uint64_t>(components, 1), &bip));
      WC_CUDA(cudaMemcpy(colour->ptr, col.data(), n, cudaMemcpyHostToDevice), ctx.detail);
      if (components)
        WC_CUDA(cudaMemcpy(bip->ptr, bipartite_host.data(), components, cudaMemcpyHostToDevice), ctx.detail);
    }
    return WC_OK;
  }

  // deflation.rs:87-135 and lanczos.rs:264-278.
  wc_status deflate() {
    const int op_ = o.op, which = o.which;
    if ((op_ == WC_LAPLACIAN || op_ == WC_NORMALIZED_LAPLACIAN) && which == WC_SMALLEST) {
      has_connected = true;
      known_connected = 0.0;
    } else if (op_ == WC_RANDOM_WALK && which == WC_LARGEST) {
      has_connected = has_bipartite = true;
      known_connected = 1.0;
      known_bipartite = -1.0;
    } else if (op_ == WC_NORMALIZED_LAPLACIAN && which == WC_LARGEST) {
      has_bipartite = true;
      known_bipartite = 2.0;
    } else {
      return WC_OK;
    }
    // Nonnegative: the smallest entry of each row (min_first) is >= 0 and
    // not NaN.
    {
      PullLaunch L;
      WC_TRY(prepare_pull(ctx, v->fwd, WC_MIN_FIRST, o.weighted, WC_F64, 1, L));
      WC_TRY(launch_pull(L, WC_F64, input->ptr, output->ptr));
      std::vector<double> mins(n);
      WC_CUDA(cudaMemcpy(mins.data(), output->ptr, (uint64_t)n * 8, cudaMemcpyDeviceToHost), ctx.detail);
      nonnegative = true;
      for (double m : mins)
        if (m != m || m < 0.0) nonnegative = false;
    }
    WC_TRY(find_components(has_bipartite));
    uint64_t bipartite_count = 0;
    for (uint8_t b : bipartite_host) bipartite_count += b;
    deflated_count = (has_connected ? components : 0) + (has_bipartite ? bipartite_count : 0);
    if (deflated_count == 0) return WC_OK;
    deflating = true;
    connected_flag = has_connected ? 1.0 : 0.0;
    alternating_flag = has_bipartite ? 1.0 : 0.0;
    WC_TRY(ctx.scratch(POOL_ADJ_4, (uint64_t)n * 8, &unit));
    WC_TRY(ctx.scratch(POOL_ADJ_5, std::max<uint64_t>(components, 1) * 16, &dcoef));
    WC_CUDA(cudaMemsetAsync(dcoef->ptr, 0, std::max<uint64_t>(components, 1) * 16, st()), ctx.detail);
    note_launch(), unit_kernel<<<grid, 256, 0, st()>>>(n, active->as<uint8_t>(), comp->as<uint32_t>(),
                                        degrees->as<double>(), normalized, unit->as<double>(),
                                        dcoef->as<double>());
    note_launch(), unit_normalize_kernel<<<grid, 256, 0, st()>>>(n, active->as<uint8_t>(), comp->as<uint32_t>(),
                                                  dcoef->as<double>(), unit->as<double>());
    return cuda_status(cudaGetLastError(), ctx.detail, "deflation");
  }

  // deflation.rs:174-198: x -= Σ v (v·x); returns ‖x‖.
  wc_status project_out(double* x, double* norm) {
    WC_CUDA(cudaMemsetAsync(dcoef->ptr, 0, std::max<uint64_t>(components, 1) * 16, st()), ctx.detail);
    const uint8_t* col = colour ? colour->as<uint8_t>() : nullptr;
    note_launch(), deflate_coef_kernel<<<grid, 256, 0, st()>>>(n, active->as<uint8_t>(), comp->as<uint32_t>(), col,
                                                unit->as<double>(), x, dcoef->as<double>());
    note_launch(), deflate_apply_kernel<<<grid, 256, 0, st()>>>(n, active->as<uint8_t>(), comp->as<uint32_t>(), col,
                                                 bip ? bip->as<uint8_t>() : nullptr,
                                                 unit->as<double>(), dcoef->as<double>(),
                                                 connected_flag, alternating_flag, x);
    double s;
    WC_TRY(dot_self(x, &s));
    *norm = std::sqrt(s);
    return WC_OK;
  }

  // ---------------------------------------------------------- the basis
  uint32_t size = 0, len = 0;
  uint32_t held_chunks = 1;  // projection chunks the partial and coefficient buffers hold

  double* col(uint32_t j) { return Q->as<double>() + (size_t)j * n; }

  // Qᵀw (after w -= c·q_p for pending p >= 0) into coefbuf[0 .. len) on the
  // device: every 8-column chunk's projection, then one launch combining
  // each chunk's partials in block order, then the coefficients' copy into
  // the pinned staging, all queued without a wait; subtract_projected, which
  // follows, waits once for all of it.
  wc_status project(double* w, int pending, double c) {
    if (len == 0 && pending < 0) return WC_OK;
    const uint32_t chunks = std::max<uint32_t>(1, (len + 7) / 8);
    if ((uint64_t)chunks * 8 * 8 > kStageBytes - kStagePayload) return WC_UNSUPPORTED;
    if (chunks > held_chunks) {  // grown once per solve, not charged again each step
      WC_TRY(ctx.scratch(POOL_EIG_7, (uint64_t)chunks * grid * 8 * 8, &partial));
      WC_TRY(ctx.scratch(POOL_EIG_8, (uint64_t)std::max<uint32_t>(64, chunks * 8) * 8, &coefbuf));
      held_chunks = chunks;
    }
    for (uint32_t b = 0; b < chunks; b++)
      note_launch(), project_kernel<<<grid, 256, 0, st()>>>(n, Q->as<double>(), len, 8 * b, w,
                                                            pending, c,
                                                            partial->as<double>() +
                                                                (size_t)b * grid * 8);
    note_launch(), sum_final_kernel<<<chunks, 256, 0, st()>>>(partial->as<double>(), grid, 8,
                                                              coefbuf->as<double>());
    if (len)
      WC_CUDA(cudaMemcpyAsync(v->stage_host + kStagePayload, coefbuf->ptr, len * 8,
                              cudaMemcpyDeviceToHost, st()),
              ctx.detail);
    return WC_OK;
  }

  // w -= Σ_j c_j q_j with the coefficients project left in coefbuf, then
  // ‖w‖; waits for the stream, after which `c` gets those coefficients.
  wc_status subtract_projected(double* w, std::vector<double>& c, double* norm) {
    note_launch(), subtract_kernel<<<grid, 256, 0, st()>>>(n, Q->as<double>(), coefbuf->as<double>(), len, w,
                                            partial->as<double>());
    double s;
    WC_TRY(sum_final(grid, 1, &s));
    c.assign(len, 0.0);
    if (len) std::memcpy(c.data(), v->stage_host + kStagePayload, len * 8);
    *norm = std::sqrt(s);
    return WC_OK;
  }

  // basis.rs:117-142.
  wc_status orthogonalize(double* w, bool has_previous, double previous,
                          std::vector<double>& coefficients, double* norm) {
    coefficients.assign(len, 0.0);
    int pending = -1;
    double pending_c = 0.0;
    if (has_previous && len >= 2) {
      const uint32_t j = len - 1;
      note_launch(), recurrence_kernel<<<grid, 256, 0, st()>>>(n, col(j - 1), col(j), previous, w,
                                                partial->as<double>());
      double alpha;
      WC_TRY(sum_final(grid, 1, &alpha));
      coefficients[j - 1] = previous;
      coefficients[j] = alpha;
      pending = (int)j;
      pending_c = alpha;
    } else {
      std::vector<double> first;
      WC_TRY(project(w, -1, 0.0));
      double ignored;
      WC_TRY(subtract_projected(w, first, &ignored));
      for (uint32_t j = 0; j < len; j++) coefficients[j] += first[j];
    }
    std::vector<double> correction;
    WC_TRY(project(w, pending, pending_c));
    WC_TRY(subtract_projected(w, correction, norm));
    for (uint32_t j = 0; j < len; j++) coefficients[j] += correction[j];
    return WC_OK;
  }

  wc_status push(const double* w, double norm) {
    if (len == size) return WC_OK;
    note_launch(), copy_kernel<<<grid, 256, 0, st()>>>(w, col(len), n);
    note_launch(), scale_vec_kernel<<<grid, 256, 0, st()>>>(col(len), n, 1.0 / norm);
    len++;
    return cuda_status(cudaGetLastError(), ctx.detail, "push");
  }

  // ---------------------------------------------------------- Lanczos
  std::vector<double> H;  // size × size, row-major
  bool has_prev = false;
  double prev = 0.0;
  uint64_t streams = 0, iterations = 0, max_iter = 0, wanted = 0;

  wc_status extend_randomly(bool* ok) {
    streams++;
    double* x = input->as<double>();
    note_launch(), random_kernel<<<grid, 256, 0, st()>>>(x, active->as<uint8_t>(), n, o.seed, streams - 1, 0);
    double before;
    WC_TRY(dot_self(x, &before));
    before = std::sqrt(before);
    std::vector<double> coeff;
    double norm;
    WC_TRY(orthogonalize(x, false, 0.0, coeff, &norm));
    if (deflating) WC_TRY(project_out(x, &norm));
    if (norm <= kF64Breakdown * before) {
      *ok = false;
      return WC_OK;
    }
    WC_TRY(push(x, norm));
    has_prev = false;
    *ok = true;
    return WC_OK;
  }

  // lanczos.rs:554-577: returns β or a breakdown (has_beta false).
  wc_status step(bool* has_beta, double* beta) {
    const uint32_t j = len - 1;
    double* w = output->as<double>();
    WC_TRY(apply(col(j), w));
    iterations++;
    std::vector<double> coeff;
    double norm;
    WC_TRY(orthogonalize(w, has_prev, prev, coeff, &norm));
    double b = norm;
    if (deflating) WC_TRY(project_out(w, &b));
    for (uint32_t i = 0; i < coeff.size(); i++) {
      H[(size_t)i * size + j] = coeff[i];
      H[(size_t)j * size + i] = coeff[i];
    }
    double sq = 0.0;
    for (double c : coeff) sq += c * c;
    const double before = std::sqrt(sq + b * b);
    if (!std::isfinite(b)) return WC_NOT_FINITE;
    *has_beta = b > kF64Breakdown * before;
    *beta = b;
    return WC_OK;
  }

  wc_status extend(bool has_beta, double beta, bool* ok) {
    if (has_beta) {
      WC_TRY(push(output->as<double>(), beta));
      has_prev = true;
      prev = beta;
      *ok = true;
      return WC_OK;
    }
    return extend_randomly(ok);
  }

  struct RitzPairs {
    std::vector<double> values;  // which order
    std::vector<double> vectors; // len × len, column l = pair l, row-major [i * len + l]
  };

  wc_status ritz(RitzPairs& r) {
    std::vector<double> a((size_t)len * len);
    for (uint32_t i = 0; i < len; i++)
      for (uint32_t j = 0; j < len; j++) {
        a[(size_t)i * len + j] = H[(size_t)i * size + j];
        if (!std::isfinite(a[(size_t)i * len + j])) return WC_NOT_FINITE;
      }
    std::vector<double> w, vec;
    if (!jacobi(a, len, w, vec)) return WC_NOT_FINITE;
    std::vector<size_t> ord = order_values(w, o.which, kF64Tie);
    r.values.resize(len);
    r.vectors.assign((size_t)len * len, 0.0);
    for (uint32_t l = 0; l < len; l++) {
      r.values[l] = w[ord[l]];
      for (uint32_t i = 0; i < len; i++) r.vectors[(size_t)i * len + l] = vec[(size_t)i * len + ord[l]];
    }
    return WC_OK;
  }

  // Σ_j V[j][l] q_j into `out` for one l.
  wc_status combine(const RitzPairs& r, uint32_t l, double* out) {
    std::vector<double> vl(len);
    for (uint32_t i = 0; i < len; i++) vl[i] = r.vectors[(size_t)i * len + l];
    WC_CUDA(cudaMemcpy(vbuf->ptr, vl.data(), len * 8, cudaMemcpyHostToDevice), ctx.detail);
    note_launch(), rotate_kernel<<<grid, 256, 0, st()>>>(n, Q->as<double>(), vbuf->as<double>(), len, 1, 1, out);
    return cuda_status(cudaGetLastError(), ctx.detail, "combine");
  }

  // lanczos.rs:700-743: settle (normalise, sign), residual, map.
  wc_status eigenpair(double value, double* x, Pair& p, bool keep_vector) {
    WC_TRY(settle(x));
    WC_TRY(apply(x, output->as<double>()));
    note_launch(), residual_terms_kernel<<<grid, 256, 0, st()>>>(x, output->as<double>(), value, n,
                                                  partial->as<double>());
    double s;
    WC_TRY(sum_final(grid, 1, &s));
    p.residual = std::sqrt(s);
    p.value = value;
    if (o.op == WC_RANDOM_WALK) {
      note_launch(), scale_kernel<<<grid, 256, 0, st()>>>(x, scale->as<double>(), scratch->as<double>(), n);
      note_launch(), copy_kernel<<<grid, 256, 0, st()>>>(scratch->as<double>(), x, n);
      WC_TRY(settle(x));
    }
    if (keep_vector) {
      p.vector.resize(n);
      WC_CUDA(cudaMemcpy(p.vector.data(), x, (uint64_t)n * 8, cudaMemcpyDeviceToHost), ctx.detail);
    }
    return WC_OK;
  }

  wc_status settle(double* x) {
    double s;
    WC_TRY(dot_self(x, &s));
    const double norm = std::sqrt(s);
    note_launch(), max_abs_kernel<<<grid, 256, 0, st()>>>(x, n, partial->as<double>());
    std::vector<double> part(grid);
    WC_CUDA(cudaMemcpyAsync(part.data(), partial->ptr, grid * 8, cudaMemcpyDeviceToHost, st()),
            ctx.detail);
    WC_CUDA(cudaStreamSynchronize(st()), ctx.detail);
    double m = 0.0;
    for (double q : part) m = std::max(m, q);
    double sign = 1.0;
    if (m > 0.0) {
      unsigned* idx = reinterpret_cast<unsigned*>(coefbuf->as<char>() + 8 * 60);
      WC_CUDA(cudaMemsetAsync(idx, 0xff, 4, st()), ctx.detail);
      note_launch(), first_at_kernel<<<grid, 256, 0, st()>>>(x, n, m, idx);
      unsigned at = 0;
      WC_CUDA(cudaMemcpyAsync(&at, idx, 4, cudaMemcpyDeviceToHost, st()), ctx.detail);
      WC_CUDA(cudaStreamSynchronize(st()), ctx.detail);
      double xv = 0.0;
      WC_CUDA(cudaMemcpy(&xv, x + at, 8, cudaMemcpyDeviceToHost), ctx.detail);
      sign = xv < 0 ? -1.0 : 1.0;
    }
    note_launch(), scale_vec_kernel<<<grid, 256, 0, st()>>>(x, n, sign / norm);
    return cuda_status(cudaGetLastError(), ctx.detail, "settle");
  }

  // lanczos.rs:502-545.
  wc_status run(std::vector<Pair>& found, bool* converged, bool keep) {
    H.assign((size_t)size * size, 0.0);
    WC_TRY(ctx.scratch(POOL_ADJ_6, (uint64_t)size * n * 8, &Q));
    WC_TRY(ctx.scratch(POOL_ADJ_7, (uint64_t)size * n * 8, &Q2));
    WC_TRY(ctx.scratch(POOL_ADJ_8, (uint64_t)64 * 64 * 8, &vbuf));
    WC_TRY(ctx.scratch(POOL_EIG_8, 64 * 8, &coefbuf));
    len = 0;
    bool ok;
    WC_TRY(extend_randomly(&ok));
    if (!ok) return WC_EIGENPAIR_COUNT;
    for (;;) {
      if (ctx.cancelled()) return WC_CANCELLED;
      bool has_beta;
      double beta;
      WC_TRY(step(&has_beta, &beta));
      ctx.progress("lanczos", iterations, max_iter);
      if (len < size && iterations < max_iter) {
        WC_TRY(extend(has_beta, beta, &ok));
        if (ok) continue;
        return finish(found, converged, true, keep);
      }
      RitzPairs r;
      WC_TRY(ritz(r));
      // outcome (lanczos.rs:633-650)
      double scale_ = 0.0;
      for (double v_ : r.values) scale_ = std::max(scale_, std::fabs(v_));
      const double b = has_beta ? beta : 0.0;
      uint64_t conv = 0;
      for (uint64_t l = 0; l < wanted; l++)
        if (std::fabs(b * r.vectors[(size_t)(len - 1) * len + l]) <= o.tol * scale_) conv++;
      const bool done = len == dimension - deflated_count || conv == wanted;
      if (done) return finish_with(r, found, converged, true, keep);
      if (iterations >= max_iter) return finish_with(r, found, converged, false, keep);
      // restart (lanczos.rs:658-671)
      const uint64_t free = size - wanted;
      const uint64_t lo = free / 4, hi = free / 2;
      const uint64_t extra = std::min(std::max(conv, lo), hi);
      const uint32_t kept = (uint32_t)std::min<uint64_t>(wanted + extra, size - 1);
      std::vector<double> vk((size_t)len * kept);
      for (uint32_t i = 0; i < len; i++)
        for (uint32_t l = 0; l < kept; l++) vk[(size_t)i * kept + l] = r.vectors[(size_t)i * len + l];
      WC_CUDA(cudaMemcpy(vbuf->ptr, vk.data(), vk.size() * 8, cudaMemcpyHostToDevice), ctx.detail);
      note_launch(), rotate_kernel<<<grid, 256, 0, st()>>>(n, Q->as<double>(), vbuf->as<double>(), len, kept, kept,
                                            Q2->as<double>());
      WC_CUDA(cudaMemcpyAsync(Q->ptr, Q2->ptr, (uint64_t)kept * n * 8, cudaMemcpyDeviceToDevice, st()),
              ctx.detail);
      len = kept;
      std::fill(H.begin(), H.end(), 0.0);
      for (uint32_t l = 0; l < kept; l++) H[(size_t)l * size + l] = r.values[l];
      WC_TRY(extend(has_beta, beta, &ok));
      if (!ok) return finish(found, converged, true, keep);
      has_prev = false;
    }
  }

  wc_status finish(std::vector<Pair>& found, bool* converged, bool c, bool keep) {
    RitzPairs r;
    WC_TRY(ritz(r));
    return finish_with(r, found, converged, c, keep);
  }

  wc_status finish_with(const RitzPairs& r, std::vector<Pair>& found, bool* converged, bool c,
                        bool keep) {
    *converged = c;
    for (uint64_t l = 0; l < wanted; l++) {
      double* x = input->as<double>();
      WC_TRY(combine(r, (uint32_t)l, x));
      Pair p;
      p.known = false;
      WC_TRY(eigenpair(r.values[l], x, p, keep));
      found.push_back(std::move(p));
    }
    return WC_OK;
  }
};

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_eigen(wc_version* v, const wc_call* call, const wc_eigen_opts* opts, double* values,
                   double* residuals, double* vectors, wc_eigen_stats* stats) {
  if (!v || !opts || !values || !residuals) return WC_INVALID_ARGUMENT;
  if (opts->op < WC_ADJACENCY || opts->op > WC_RANDOM_WALK || opts->which < WC_LARGEST ||
      opts->which > WC_SMALLEST)
    return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  Eigensolver es(ctx, *opts);
  WC_TRY(es.setup());
  const uint64_t k = opts->k;
  if (k == 0 || k > es.dimension) {
    if (ctx.detail) {
      ctx.detail->expected = es.dimension;
      ctx.detail->found = k;
    }
    return WC_EIGENPAIR_COUNT;
  }
  WC_TRY(es.deflate());
  if (!es.parent) WC_TRY(es.find_components(false));  // reported whether deflated or not
  // How many pairs Lanczos computes (deflation.rs:142-154).
  if (es.deflating) {
    es.wanted = es.nonnegative ? (k > es.deflated_count ? k - es.deflated_count : 0)
                               : std::min<uint64_t>(k, es.dimension - es.deflated_count);
  } else {
    es.wanted = k;
  }
  const uint64_t complement = es.dimension - (es.deflating ? es.deflated_count : 0);
  es.size = es.wanted == 0 ? 0
                           : (uint32_t)std::min<uint64_t>(complement,
                                                          std::max<uint64_t>(2 * k + 1, kMinBasis));
  es.max_iter = std::max<uint64_t>(opts->max_iter ? opts->max_iter : kStepsPerBasisVector * es.size, k);
  const bool keep = vectors != nullptr;
  std::vector<Pair> found;
  bool converged = true;
  if (es.wanted > 0) {
    if (es.size > 64) return WC_UNSUPPORTED;
    ctx.progress("lanczos", 0, es.max_iter);
    WC_TRY(es.run(found, &converged, keep));
  }
  // The components' pairs (deflation.rs:157-172), first k, in order.
  std::vector<Pair> known;
  if (es.deflating) {
    std::vector<std::pair<double, std::pair<uint64_t, int>>> kp;
    if (es.has_connected)
      for (uint64_t c = 0; c < es.components; c++) kp.push_back({es.known_connected, {c, 0}});
    if (es.has_bipartite)
      for (uint64_t c = 0; c < es.components; c++)
        if (es.bipartite_host[c]) kp.push_back({es.known_bipartite, {c, 1}});
    if (kp.size() > k) kp.resize(k);
    for (auto& q : kp) {
      double* x = es.input->as<double>();
      note_launch(), known_vector_kernel<<<es.grid, 256, 0, ctx.stream>>>(
          es.n, es.active->as<uint8_t>(), es.comp->as<uint32_t>(),
          es.colour ? es.colour->as<uint8_t>() : nullptr, es.unit->as<double>(),
          (uint32_t)q.second.first, q.second.second, x);
      Pair p;
      p.known = true;
      WC_TRY(es.eigenpair(q.first, x, p, keep));
      known.push_back(std::move(p));
    }
  }
  // merge (lanczos.rs:353-377).
  std::vector<Pair> all;
  for (auto& p : known) all.push_back(std::move(p));
  const size_t known_count = all.size();
  for (auto& p : found) all.push_back(std::move(p));
  std::vector<double> exact;
  for (size_t i = 0; i < known_count; i++)
    if (exact.empty() || exact.back() != all[i].value) exact.push_back(all[i].value);
  std::vector<double> vals;
  for (auto& p : all) vals.push_back(p.value);
  double m = 0.0;
  for (double x : vals) m = std::max(m, std::fabs(x));
  const double width = kF64Tie * m;
  std::vector<double> keys(vals);
  for (size_t i = 0; i < vals.size(); i++)
    for (double e : exact) {
      const double value = vals[i];
      const bool beyond = opts->which == WC_SMALLEST
                              ? value < e
                              : (std::fabs(value) > std::fabs(e) &&
                                 std::signbit(value) == std::signbit(e));
      if (es.nonnegative && beyond && std::fabs(value - e) <= width) {
        keys[i] = e;
        break;
      }
    }
  std::vector<size_t> ord = order_values(keys, opts->which, kF64Tie);
  if (ord.size() > k) ord.resize(k);
  uint32_t exact_count = 0;
  for (size_t q = 0; q < ord.size(); q++) {
    const Pair& p = all[ord[q]];
    values[q] = p.value;
    residuals[q] = p.residual;
    if (keep) WC_CUDA(cudaMemcpy(vectors + q * v->n, p.vector.data(), v->n * 8, cudaMemcpyDefault), ctx.detail);
    if (ord[q] < known_count) exact_count++;
  }
  if (stats) {
    stats->iterations = es.iterations;
    stats->components = es.deflating || es.components ? es.components : 0;
    stats->exact = exact_count;
    stats->converged = converged;
  }
  return ctx.finish();
}

wc_status wc_random_uniform(wc_version* v, const wc_call* call, uint64_t seed, uint64_t stream,
                            double* out) {
  if (!v || !out) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  Operand X(POOL_EIG_0);
  WC_TRY(X.output(ctx, out, v->n * 8));
  const uint32_t n = (uint32_t)v->n;
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, max_blocks(4)));
  note_launch(), random_kernel<<<grid, 256, 0, ctx.stream>>>(static_cast<double*>(X.dev), nullptr,
                                                             n, seed, stream, 1);
  WC_CUDA(cudaGetLastError(), ctx.detail);
  WC_TRY(X.out(ctx));
  return ctx.finish();
}

}  // extern "C"
