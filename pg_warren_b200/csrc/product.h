// product.h — what a launch of the product kernels needs, independent of the
// element type, so the per-dtype translation units share one interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "runtime.cuh"

namespace wc {

// compute/product/kernel.rs:200-240 (Write::row): the mask, replace and
// accumulate of a product (accumulate < 0: overwrite).
struct WriteArgs {
  const void* mask;
  int32_t mask_dtype;
  int32_t complement;
  int32_t replace;
  int32_t accumulate;
};

enum WeightKind { WEIGHTS_NONE = 0, WEIGHTS_F64 = 1, WEIGHTS_I32 = 2 };

struct PullLaunch {
  const uint32_t* off;
  const uint32_t* tgt;
  const void* weights;
  int32_t weight_kind;
  const Unit* units;
  uint32_t unit_count;
  uint32_t* counters;
  void* carry;
  void* carry_multi;  // width > 1: 32 partials a long-row slot
  uint32_t n;
  uint32_t width;
  int32_t semiring;
  uint32_t max_blocks;
  cudaStream_t stream;
  DeviceError* err;
  wc_error_detail* detail;
  WriteArgs write;
  uint32_t hot;  // over a locality-ordered CSC: gathers of j < hot kept in L1 (0: none)
};

// Cuts `csr`'s schedule into `parts` ranges of about equal entries at unit
// boundaries (a long row's pieces in one range): unit_cut and row_cut get
// parts + 1 entries, the parts' first units and first rows.
wc_status schedule_part_cuts(const wc_version* v, const DevCsr& csr, uint32_t parts,
                             std::vector<uint32_t>& unit_cut, std::vector<uint64_t>& row_cut,
                             wc_error_detail* detail);

wc_status launch_pull_f64(const PullLaunch& L, const void* x, void* y);
wc_status launch_pull_f32(const PullLaunch& L, const void* x, void* y);
wc_status launch_pull_i64(const PullLaunch& L, const void* x, void* y);
wc_status launch_pull_bool(const PullLaunch& L, const void* x, void* y);

// The bytes of carry space a long-row schedule needs per slot (the largest
// partial accumulator: i64 plus keeps three 128-bit values).
constexpr uint64_t kCarryBytesPerSlot = 64;
// The SpMM's carry: a partial per column of a 32-column block, per slot.
constexpr uint64_t kMultiCarryBytesPerSlot = 32 * kCarryBytesPerSlot;

}  // namespace wc
