// pagerank_part.cu — one rank's part of a row-partitioned PageRank (no
// reference counterpart: warren-core solves on one host).  The solve's rows
// (the locality-ordered numbering of wc_pagerank) are cut into parts of
// about equal entries at unit boundaries of the reverse CSR's schedule;
// each rank pulls its rows, and between iterations the caller exchanges
// what the next iteration reads: the parts' L1 changes and dangling ranks
// (summed) and the parts' rows of the next message vector (gathered).  Each
// iteration is wc_pagerank's own kernel over the part's units, with the stop
// test left to the caller, who has the summed change.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "operand.h"
#include "pagerank.h"
#include "pull.cuh"
#include "sqlfloat.cuh"
#include "upload.h"

namespace wc {

wc_status prepare_pull(Ctx& ctx, DevCsr& csr, int semiring, int weighted_flag, int dtype,
                       uint32_t width, PullLaunch& L);

// The parts' first units and first rows over `csr`'s schedule: units are
// taken in order and a part is closed at the first row boundary at or past
// its share of the entries; a long row's pieces stay in one part.
// The cuts are kept per (version, CSR, parts): a version never changes, and
// the schedule's units are read back from the device only the first time.
struct Cuts {
  std::vector<uint32_t> units;
  std::vector<uint64_t> rows;
};
static std::map<std::tuple<const wc_version*, const DevCsr*, uint32_t>, Cuts> g_cuts;
static std::mutex g_cuts_mu;

static wc_status compute_part_cuts(const wc_version* v, const DevCsr& csr, uint32_t parts,
                                   std::vector<uint32_t>& unit_cut,
                                   std::vector<uint64_t>& row_cut, wc_error_detail* detail);

wc_status schedule_part_cuts(const wc_version* v, const DevCsr& csr, uint32_t parts,
                             std::vector<uint32_t>& unit_cut, std::vector<uint64_t>& row_cut,
                             wc_error_detail* detail) {
  const auto key = std::make_tuple(v, &csr, parts);
  {
    std::lock_guard<std::mutex> lock(g_cuts_mu);
    auto it = g_cuts.find(key);
    if (it != g_cuts.end()) {
      unit_cut = it->second.units;
      row_cut = it->second.rows;
      return WC_OK;
    }
  }
  WC_TRY(compute_part_cuts(v, csr, parts, unit_cut, row_cut, detail));
  std::lock_guard<std::mutex> lock(g_cuts_mu);
  g_cuts[key] = Cuts{unit_cut, row_cut};
  return WC_OK;
}

static wc_status compute_part_cuts(const wc_version* v, const DevCsr& csr, uint32_t parts,
                                   std::vector<uint32_t>& unit_cut,
                                   std::vector<uint64_t>& row_cut, wc_error_detail* detail) {
  const Schedule& sc = csr.schedule;
  std::vector<Unit> units(sc.count);
  if (sc.count)
    WC_CUDA(cudaMemcpy(units.data(), sc.units.ptr, sc.count * sizeof(Unit), cudaMemcpyDeviceToHost),
            detail);
  unit_cut.assign(parts + 1, sc.count);
  row_cut.assign(parts + 1, v->n);
  unit_cut[0] = 0;
  row_cut[0] = 0;
  uint64_t seen = 0;
  uint32_t p = 1;
  for (uint32_t u = 0; u < sc.count && p < parts; u++) {
    const Unit& d = units[u];
    const bool piece = (d.c >> 31) != 0;
    const bool continues = piece && u > 0 && (units[u - 1].c >> 31) != 0 && units[u - 1].a == d.a;
    while (p < parts && !continues && seen >= (v->m * p + parts - 1) / parts) {
      unit_cut[p] = u;
      row_cut[p] = d.a;
      p++;
    }
    seen += piece ? d.d - d.b : d.c;
  }
  for (; p < parts; p++) {
    unit_cut[p] = sc.count;
    row_cut[p] = v->n;
  }
  return WC_OK;
}

static wc_status part_cuts(wc_version* v, uint32_t parts, std::vector<uint32_t>& unit_cut,
                           std::vector<uint64_t>& row_cut, wc_error_detail* detail) {
  return schedule_part_cuts(v, v->loc.csc, parts, unit_cut, row_cut, detail);
}

// The state of a part kept with the version between its calls.
struct PartSolve {
  PageRankRun run;
  uint32_t unit_begin = 0, unit_end = 0;
};

static std::map<const wc_version*, std::unique_ptr<PartSolve>> g_parts;
static std::mutex g_parts_mu;

static PartSolve* part_of(const wc_version* v) {
  std::lock_guard<std::mutex> lock(g_parts_mu);
  auto it = g_parts.find(v);
  return it == g_parts.end() ? nullptr : it->second.get();
}

void pagerank_part_forget(const wc_version* v) {
  {
    std::lock_guard<std::mutex> lock(g_parts_mu);
    g_parts.erase(v);
  }
  std::lock_guard<std::mutex> lock(g_cuts_mu);
  for (auto it = g_cuts.begin(); it != g_cuts.end();)
    it = std::get<0>(it->first) == v ? g_cuts.erase(it) : std::next(it);
}

}  // namespace wc

using namespace wc;

extern "C" {

wc_status wc_pagerank_part_rows(wc_version* v, uint32_t parts, uint64_t* row_bounds) {
  if (!v || parts == 0 || !row_bounds) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), nullptr);
  std::vector<uint32_t> uc;
  std::vector<uint64_t> rc;
  WC_TRY(part_cuts(v, parts, uc, rc, nullptr));
  std::copy(rc.begin(), rc.end(), row_bounds);
  return WC_OK;
}

wc_status wc_pagerank_part_begin(wc_version* v, const wc_call* call, const wc_pagerank_opts* o,
                                 const uint64_t* tombstones, uint32_t parts, uint32_t part,
                                 double* ranks2, double* messages2, wc_pagerank_part_info* info) {
  if (!v || !o || !ranks2 || !messages2 || !info || parts == 0 || part >= parts)
    return WC_INVALID_ARGUMENT;
  if (o->seed) return WC_UNSUPPORTED;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  if (!is_device_pointer(ranks2) || !is_device_pointer(messages2)) {
    set_message(ctx.detail, "the rank and message vectors must be device memory");
    return WC_INVALID_ARGUMENT;
  }
  WC_TRY(ctx.begin());
  auto ps = std::make_unique<PartSolve>();
  std::vector<uint32_t> uc;
  std::vector<uint64_t> rc;
  WC_TRY(part_cuts(v, parts, uc, rc, ctx.detail));
  ps->unit_begin = uc[part];
  ps->unit_end = uc[part + 1];
  PageRankRun& run = ps->run;
  WC_TRY(run.setup(ctx, o, tombstones, nullptr, true));
  // The rank and message vectors are the caller's (it exchanges their rows).
  const uint64_t n = v->n;
  run.s.x[0] = ranks2;
  run.s.x[1] = ranks2 + n;
  run.s.msg[0] = messages2;
  run.s.msg[1] = messages2 + n;
  run.s.has_tol = false;  // the caller holds the summed change
  run.s.pace = nullptr;
  run.grid = pagerank_grid(v->loc.csc);
  WC_TRY(launch_pr_init(run.s, run.grid, ctx.stream));
  WC_TRY(ctx.finish());
  double dangling0 = 0.0;
  WC_CUDA(cudaMemcpy(&dangling0, run.s.dangling, 8, cudaMemcpyDeviceToHost), ctx.detail);
  info->row_begin = rc[part];
  info->row_end = rc[part + 1];
  info->id_space = n;
  info->dangling = dangling0;
  info->threshold = run.s.threshold;
  info->live = run.live;
  std::lock_guard<std::mutex> plock(g_parts_mu);
  g_parts[v] = std::move(ps);
  return WC_OK;
}

wc_status wc_pagerank_part_step(wc_version* v, const wc_call* call, uint32_t iteration,
                                double dangling_in, double* sums) {
  if (!v || !sums) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  PartSolve* ps = part_of(v);
  if (!ps) return WC_INVALID_ARGUMENT;
  PageRankRun& run = ps->run;
  if (iteration >= run.opts.max_iter) return WC_INVALID_ARGUMENT;
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  if (ctx.cancelled()) return WC_CANCELLED;
  WC_TRY(ctx.begin());
  // This iteration's dangling rank is the parts' sum, which the caller has.
  WC_CUDA(cudaMemcpyAsync(run.s.dangling + iteration, &dangling_in, 8, cudaMemcpyHostToDevice,
                          ctx.stream), ctx.detail);
  PullLaunch L;
  WC_TRY(prepare_pull(ctx, v->loc.csc, WC_PLUS_TIMES, run.opts.weighted, WC_F64, 1, L));
  L.units += ps->unit_begin;
  L.unit_count = ps->unit_end - ps->unit_begin;
  L.hot = kPageRankHotNodes;
  if (L.unit_count) WC_TRY(launch_part_iteration(L, run.s, iteration, run.grid));
  WC_TRY(ctx.finish());
  double host[2] = {0.0, 0.0};
  if (L.unit_count) {
    WC_CUDA(cudaMemcpy(&host[0], run.s.delta + iteration, 8, cudaMemcpyDeviceToHost), ctx.detail);
    WC_CUDA(cudaMemcpy(&host[1], run.s.dangling + iteration + 1, 8, cudaMemcpyDeviceToHost),
            ctx.detail);
  }
  sums[0] = host[0];
  sums[1] = host[1];
  return WC_OK;
}

wc_status wc_pagerank_part_end(wc_version* v, const wc_call* call, uint32_t iterations,
                               double* ranks) {
  if (!v || !ranks) return WC_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lock(v->mu);
  PartSolve* ps = part_of(v);
  if (!ps) return WC_INVALID_ARGUMENT;
  WC_CUDA(cudaSetDevice(v->device), call ? call->detail : nullptr);
  Ctx ctx(v, call);
  WC_TRY(ctx.begin());
  PageRankRun& run = ps->run;
  // The caller has gathered every part's rows of x[iterations & 1].
  WC_CUDA(cudaMemcpyAsync(run.s.iterations, &iterations, 4, cudaMemcpyHostToDevice, ctx.stream),
          ctx.detail);
  WC_TRY(ctx.finish());
  const wc_status st = run.result(ctx, ranks, nullptr, nullptr);
  std::lock_guard<std::mutex> plock(g_parts_mu);
  g_parts.erase(v);
  return st;
}

}  // extern "C"
