// adjoint.cu — wc_pagerank_adjoint: ∂L/∂w for every edge, for losses
// L_c = Σ_{t in T_c} x_t of the uniform PageRank x (no reference
// counterpart; its forward is compute/pagerank/mod.rs:96-287).
//
// At the fixed point x = d·(Aᵀ D⁻¹ x + (uᵀx)·p) + (1 − d)·p, with D the
// out-weights, u the dangling rows and p = 1/live, the adjoint of L = cᵀx
// solves
//     λ = d·(D⁻¹ A λ + u·(pᵀλ)) + c,
// a pull over the forward CSR (row i: Σ_j w_ij λ_j, then ÷ out_i), iterated
// like PageRank itself (a contraction by d), every loss a column of one
// SpMM.  Then, per edge i → j,
//     ∂L/∂w_ij = d · x_i / out_i · (λ_j − (D⁻¹ A λ)_i),
// the weight's direct share of rank minus its dilution of row i's others.
// The forward solve is recomputed here (wc_pagerank's kernels), never stored
// per iteration.
#include <algorithm>

#include "columns.cuh"
#include "operand.h"
#include "pagerank.h"
#include "pull32.cuh"
#include "pull_multi.cuh"

namespace wc {

constexpr uint32_t kAdjP = 32;  // losses per pass

struct AdjState {
  uint32_t n;
  uint64_t m;
  double* lam[2];      // n × P
  double* S;           // n × P: (D⁻¹Aλ)_i, of the final λ
  const double* C;     // n × P: the loss indicators (counts)
  const double* out;   // n
  const double* x;     // n, the forward ranks
  double damping, p;
  uint32_t k;
  uint32_t* running;
  uint32_t* executed;
  double* pi;          // P: pᵀλ of the current λ
  double* partials;
  unsigned* counter;
  uint32_t* iterations;  // P
  double tol;
  DeviceError* err;
};

template <int P> struct AdjEpi {
  const AdjState* s;
  int cur;
  uint32_t run_bits;
  double pi;  // this lane's column
  double delta, total;
  bool final_pass;
  __device__ void cell(uint32_t i, uint32_t c, bool present, double z) {
    const AdjState& st = *s;
    const size_t at = (size_t)i * P + c;
    const double o = st.out[i];
    const double si = (present && o > 0.0) ? z / o : 0.0;
    if (final_pass) {
      st.S[at] = si;
      return;
    }
    const double old = st.lam[cur][at];
    if (!((run_bits >> c) & 1)) {
      st.lam[cur ^ 1][at] = old;
      total += old;
      return;
    }
    const double next = st.damping * (si + (o > 0.0 ? 0.0 : pi)) + st.C[at];
    delta += fabs(next - old);
    total += next;
    st.lam[cur ^ 1][at] = next;
  }
};

template <int P>
__global__ void adj_init_kernel(AdjState s) {
  double none = 0.0, total = 0.0;
  const unsigned c = threadIdx.x % P;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / P; i < s.n;
       i += gridDim.x * blockDim.x / P) {
    const double v = s.C[(size_t)i * P + c];
    s.lam[0][(size_t)i * P + c] = v;
    total += v;
  }
  if (reduce_columns<P>(none, total, s.partials, s.counter) && threadIdx.x < P) {
    s.pi[threadIdx.x] = s.p * total;
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (uint32_t q = 0; q < s.k; q++) run |= 1u << q;
      *s.running = run;
      *s.executed = 0;
    }
    if (threadIdx.x < s.k) s.iterations[threadIdx.x] = 0;
  }
}

template <int P, class W>
__global__ void __launch_bounds__(256) adj_iter_kernel(CsrView<W> A, AdjState s, uint32_t it,
                                                       Partial<double, WC_OP_PLUS>* carry,
                                                       uint32_t max_iter) {
  const uint32_t run = *(volatile uint32_t*)s.running;
  if (!run) return;
  const unsigned c = threadIdx.x % P;
  AdjEpi<P> epi{&s, (int)(it & 1), run, s.pi[c], 0.0, 0.0, false};
  pull_multi<double, WC_PLUS_TIMES, W, P>(A, s.lam[it & 1], epi, s.err, carry);
  double delta = epi.delta, total = epi.total;
  if (reduce_columns<P>(delta, total, s.partials, s.counter)) {
    const uint32_t q = threadIdx.x;
    if (q < P && ((run >> q) & 1)) {
      s.pi[q] = s.p * total;
      s.iterations[q] = it + 1;
      if (it + 1 >= max_iter || delta < s.tol) atomicAnd(s.running, ~(1u << q));
    }
    if (q == 0) *s.executed = it + 1;
  }
}

// S = D⁻¹ A λ for the final λ (the buffer the last iteration wrote).
template <int P, class W>
__global__ void __launch_bounds__(256) adj_rows_kernel(CsrView<W> A, AdjState s,
                                                       Partial<double, WC_OP_PLUS>* carry) {
  const int cur = *s.executed & 1;
  AdjEpi<P> epi{&s, cur, 0, 0.0, 0.0, 0.0, true};
  pull_multi<double, WC_PLUS_TIMES, W, P>(A, s.lam[cur], epi, s.err, carry);
}

// The same iteration and final pass over pull32_units (cp.async gathers
// into a per-warp ring, small blocks, as many warps an SM as the registers
// allow): a lane is a loss; a loss that has stopped gathers nothing and
// keeps its λ.
struct AdjEpi32 {
  struct Row {
    double out;
  };
  const AdjState* s;
  int cur;
  uint32_t run_bits;
  double pi;
  double delta = 0.0, total = 0.0;
  bool final_pass;
  bool active;
  __device__ Row row(uint32_t i) const { return Row{s->out[i]}; }
  __device__ Row shfl(const Row& r, uint32_t src) const {
    return Row{__shfl_sync(0xffffffffu, r.out, src)};
  }
  __device__ void emit(uint32_t i, const Partial<double, WC_OP_PLUS>& acc, const Row& r) {
    const AdjState& st = *s;
    const unsigned c = threadIdx.x & 31;
    const size_t at = (size_t)i * 32 + c;
    double z = 0.0;
    if (acc.present) acc.acc.value(&z);
    const double o = r.out;
    const double si = (acc.present && o > 0.0) ? z / o : 0.0;
    if (final_pass) {
      st.S[at] = si;
      return;
    }
    const double old = st.lam[cur][at];
    if (!((run_bits >> c) & 1)) {
      st.lam[cur ^ 1][at] = old;
      total += old;
      return;
    }
    const double next = st.damping * (si + (o > 0.0 ? 0.0 : pi)) + st.C[at];
    delta += fabs(next - old);
    total += next;
    st.lam[cur ^ 1][at] = next;
  }
};

template <class W>
__global__ void __launch_bounds__(kPull32Warps * 32, 6)
    adj_iter32_kernel(CsrView<W> A, AdjState s, uint32_t it, Partial<double, WC_OP_PLUS>* carry,
                      uint32_t max_iter) {
  const uint32_t run = *(volatile uint32_t*)s.running;
  if (!run) return;
  extern __shared__ __align__(16) double adj_smem[];
  const unsigned c = threadIdx.x & 31;
  AdjEpi32 epi{&s, (int)(it & 1), run, s.pi[c]};
  epi.final_pass = false;
  epi.active = (run >> c) & 1;
  pull32_units<W>(A, s.lam[it & 1], epi, s.err, carry,
                  adj_smem + (threadIdx.x >> 5) * kPull32WarpDoubles);
  double delta = epi.delta, total = epi.total;
  if (reduce_columns<32>(delta, total, s.partials, s.counter)) {
    const uint32_t q = threadIdx.x;
    if (q < 32 && ((run >> q) & 1)) {
      s.pi[q] = s.p * total;
      s.iterations[q] = it + 1;
      if (it + 1 >= max_iter || delta < s.tol) atomicAnd(s.running, ~(1u << q));
    }
    if (q == 0) *s.executed = it + 1;
  }
}

template <class W>
__global__ void __launch_bounds__(kPull32Warps * 32, 6)
    adj_rows32_kernel(CsrView<W> A, AdjState s, Partial<double, WC_OP_PLUS>* carry) {
  extern __shared__ __align__(16) double adj_smem[];
  const int cur = *s.executed & 1;
  const unsigned c = threadIdx.x & 31;
  AdjEpi32 epi{&s, cur, 0, 0.0};
  epi.final_pass = true;
  epi.active = c < s.k;
  pull32_units<W>(A, s.lam[cur], epi, s.err, carry,
                  adj_smem + (threadIdx.x >> 5) * kPull32WarpDoubles);
}

// grad[c][e] = d · x_i / out_i · (λ_j − S_i) for e = (i → j), a warp per
// unit of the forward schedule; consecutive lanes take consecutive entries
// so each loss's row of the gradient is written coalesced.
template <int P>
__global__ void __launch_bounds__(256) adj_scatter_kernel(const uint32_t* off, const uint32_t* tgt,
                                                          const Unit* units, uint32_t unit_count,
                                                          AdjState s, double* grad) {
  __shared__ uint8_t rowof_all[8][kTileEntries];
  uint8_t* rowof = rowof_all[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const double* lam = s.lam[*s.executed & 1];
  for (uint32_t u = warp; u < unit_count; u += warps) {
    const Unit unit = units[u];
    const bool tile = (unit.c >> 31) == 0;
    uint32_t base, count, r0 = unit.a;
    if (tile) {
      const uint32_t R = unit.b - unit.a;
      uint32_t lo = 0, hi = 0;
      if (lane < R) {
        lo = off[r0 + lane];
        hi = off[r0 + lane + 1];
      }
      base = __shfl_sync(0xffffffffu, lo, 0);
      count = __shfl_sync(0xffffffffu, hi, R - 1) - base;
      for (uint32_t k = lo - base; k < hi - base; k++) rowof[k] = (uint8_t)lane;
    } else {
      base = unit.b;
      count = unit.d - unit.b;
    }
    __syncwarp();
    for (uint32_t k = lane; k < count; k += 32) {
      const uint64_t e = base + k;
      const uint32_t i = tile ? r0 + rowof[k] : r0;
      const uint32_t j = tgt[e];
      const double coef = s.damping * s.x[i] / s.out[i];
      const double* lj = lam + (size_t)j * P;
      const double* si = s.S + (size_t)i * P;
      for (uint32_t c = 0; c < s.k; c++) grad[(size_t)c * s.m + e] = coef * (lj[c] - si[c]);
    }
    __syncwarp();
  }
}

__global__ void adj_targets_kernel(const uint64_t* targets, const uint64_t* offsets, uint32_t c0,
                                   uint32_t k, double* C) {
  const uint32_t c = blockIdx.x;
  if (c >= k) return;
  for (uint64_t q = offsets[c0 + c] + threadIdx.x; q < offsets[c0 + c + 1]; q += blockDim.x)
    atomicAdd(C + (size_t)targets[q] * kAdjP + c, 1.0);
}

// The iterations' blocks: kPull32Warps warps, at most one warp a unit; six
// an SM (the kernels are held to 80 registers for it: 6% faster on R-MAT 22
// than five at 96, where the batched PPR's pull is slower at 80).
static uint32_t adjoint_grid32(const DevCsr& fwd) {
  return std::max<uint32_t>(1, std::min<uint32_t>(max_blocks(6),
                                                  (fwd.schedule.count + kPull32Warps - 1) /
                                                      kPull32Warps));
}

template <class W>
static wc_status adjoint_pass(Ctx& ctx, AdjState& s, const DevCsr& fwd, const void* weights,
                              uint32_t max_iter, Partial<double, WC_OP_PLUS>* carry, double* grad,
                              uint32_t grid) {
  CsrView<W> A{fwd.offsets.as<uint32_t>(), fwd.targets.as<uint32_t>(),
               static_cast<const W*>(weights), fwd.schedule.units.as<Unit>(), fwd.schedule.count,
               fwd.schedule.counters.as<uint32_t>(), nullptr};
  const uint32_t grid32 = adjoint_grid32(fwd);
  WC_CUDA(cudaFuncSetAttribute(adj_iter32_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kPull32Smem), ctx.detail);
  WC_CUDA(cudaFuncSetAttribute(adj_rows32_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kPull32Smem), ctx.detail);
  note_launch(), adj_init_kernel<kAdjP><<<grid, 256, 0, ctx.stream>>>(s);
  for (uint32_t it = 0; it < max_iter; it++)
    note_launch(), adj_iter32_kernel<W><<<grid32, kPull32Warps * 32, kPull32Smem, ctx.stream>>>(
        A, s, it, carry, max_iter);
  note_launch(), adj_rows32_kernel<W><<<grid32, kPull32Warps * 32, kPull32Smem, ctx.stream>>>(
      A, s, carry);
  note_launch(), adj_scatter_kernel<kAdjP><<<max_blocks(8), 256, 0, ctx.stream>>>(
      fwd.offsets.as<uint32_t>(), fwd.targets.as<uint32_t>(), fwd.schedule.units.as<Unit>(),
      fwd.schedule.count, s, grad);
  return cuda_status(cudaGetLastError(), ctx.detail, "adjoint pass");
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_pagerank_adjoint(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                              const uint64_t* loss_targets, const uint64_t* loss_offsets,
                              uint32_t losses, double adjoint_tol, double* grad_out,
                              double* ranks_out, uint32_t* iterations_out) {
  if (!v || !o || (losses && (!loss_offsets || !grad_out))) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  const uint64_t n = v->n, m = v->m;
  std::vector<uint64_t> offs(losses + 1, 0);
  if (losses)
    WC_CUDA(cudaMemcpy(offs.data(), loss_offsets, (losses + 1) * 8, cudaMemcpyDefault), ctx.detail);
  WC_TRY(ctx.begin());
  // The forward solve, recomputed.
  PageRankRun fwd;
  WC_TRY(fwd.setup(ctx, o, nullptr, nullptr));
  WC_TRY(fwd.run(ctx));
  WC_TRY(ctx.finish());
  uint32_t its = 0;
  WC_CUDA(cudaMemcpy(&its, fwd.s.iterations, 4, cudaMemcpyDeviceToHost), ctx.detail);
  if (o->max_iter == 0) its = 0;
  const double* x = fwd.s.x[its & 1];
  if (ranks_out) WC_CUDA(cudaMemcpy(ranks_out, x, n * 8, cudaMemcpyDefault), ctx.detail);
  if (losses == 0) {
    if (iterations_out) iterations_out[0] = its;
    return WC_OK;
  }
  Operand T(POOL_ADJ_0), F(POOL_ADJ_1), G(POOL_ADJ_2);
  WC_TRY(T.in(ctx, loss_targets, std::max<uint64_t>(offs[losses], 1) * 8));
  WC_TRY(F.in(ctx, loss_offsets, (losses + 1) * 8));
  WC_TRY(G.output(ctx, grad_out, (uint64_t)losses * m * 8));
  const uint32_t P = kAdjP;
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(
      max_blocks(4), (v->fwd.schedule.count + 7) / 8));
  DevBuf *lam, *Sb, *Cb, *sc, *carry, *itb;
  WC_TRY(ctx.scratch(POOL_ADJ_3, n * P * 8 * 2, &lam));
  WC_TRY(ctx.scratch(POOL_ADJ_4, n * P * 8, &Sb));
  WC_TRY(ctx.scratch(POOL_ADJ_5, n * P * 8, &Cb));
  WC_TRY(ctx.scratch(POOL_ADJ_6,
                     4096 + (uint64_t)std::max(grid, adjoint_grid32(v->fwd)) * P * 16, &sc));
  WC_TRY(ctx.scratch(POOL_ADJ_7, (uint64_t)std::max<uint32_t>(v->fwd.schedule.slots, 1) * P *
                                     sizeof(Partial<double, WC_OP_PLUS>), &carry));
  WC_TRY(ctx.scratch(POOL_ADJ_8, (uint64_t)losses * 4 + 64, &itb));
  unsigned char* scb = sc->as<unsigned char>();
  AdjState s{};
  s.n = (uint32_t)n;
  s.m = m;
  s.lam[0] = lam->as<double>();
  s.lam[1] = s.lam[0] + n * P;
  s.S = Sb->as<double>();
  s.C = Cb->as<double>();
  s.out = fwd.s.out;
  s.x = x;
  s.damping = o->damping;
  s.p = fwd.s.start;
  s.running = reinterpret_cast<uint32_t*>(scb);
  s.executed = reinterpret_cast<uint32_t*>(scb + 8);
  s.counter = reinterpret_cast<unsigned*>(scb + 16);
  s.pi = reinterpret_cast<double*>(scb + 256);
  s.partials = reinterpret_cast<double*>(scb + 4096);
  s.tol = adjoint_tol;
  s.err = v->error.as<DeviceError>();
  const bool weighted = o->weighted != 0 && v->weighted;
  for (uint32_t c0 = 0; c0 < losses; c0 += P) {
    const uint32_t k = std::min(P, losses - c0);
    s.k = k;
    s.iterations = itb->as<uint32_t>() + c0;
    WC_CUDA(cudaMemsetAsync(sc->ptr, 0, 4096, ctx.stream), ctx.detail);
    WC_CUDA(cudaMemsetAsync(Cb->ptr, 0, n * P * 8, ctx.stream), ctx.detail);
    note_launch(), adj_targets_kernel<<<k, 128, 0, ctx.stream>>>(static_cast<const uint64_t*>(T.dev),
                                                  static_cast<const uint64_t*>(F.dev), c0, k,
                                                  Cb->as<double>());
    double* g = static_cast<double*>(G.dev) + (uint64_t)c0 * m;
    auto* cp = carry->as<Partial<double, WC_OP_PLUS>>();
    if (weighted) WC_TRY(adjoint_pass<double>(ctx, s, v->fwd, v->fwd.weights.ptr, o->max_iter, cp, g, grid));
    else WC_TRY(adjoint_pass<void>(ctx, s, v->fwd, nullptr, o->max_iter, cp, g, grid));
  }
  WC_TRY(G.out(ctx));
  WC_TRY(ctx.finish());
  if (iterations_out) {
    std::vector<uint32_t> it(losses);
    WC_CUDA(cudaMemcpy(it.data(), itb->ptr, losses * 4, cudaMemcpyDeviceToHost), ctx.detail);
    iterations_out[0] = its;
    iterations_out[1] = *std::max_element(it.begin(), it.end());
  }
  return WC_OK;
}

}  // extern "C"
