// upload.h — the steps that build a version's device copy, shared by
// wc_version_upload (host arrays) and wc_version_load_segments (stored
// segments).
#pragma once

#include <vector>

#include "runtime.cuh"

namespace wc {

// No usable sm_100 device: WC_NO_DEVICE with the reason in the detail.
wc_status wc_device_check(wc_error_detail* detail);
// The reverse CSR from the forward one, on the device (v->rev, and its
// offsets on the host).
wc_status device_reverse(wc_version* v, wc_error_detail* detail);
// Whether every weight is an i32 integer (then i32 copies of both
// orientations' weights) and the largest magnitude.
wc_status device_weight_facts(wc_version* v, wc_error_detail* detail);
// Whether the forward and reverse CSR are equal, weights included.
wc_status device_symmetric(wc_version* v, wc_error_detail* detail);
// With both orientations on the device: the weights' facts, the symmetry
// test, the row-split schedules, the locality-ordered reverse CSR, the error
// word and the mapped words.
wc_status finish_version(wc_version* v, wc_error_detail* detail);
// The row-split schedule of one orientation from its host offsets.
wc_status put_schedule(wc_version* v, DevCsr& d, const std::vector<uint64_t>& off,
                       wc_error_detail* detail);
// The reverse CSR in locality order (v->loc), after the weights' facts.
wc_status device_locality(wc_version* v, wc_error_detail* detail);
// Vectors between dense ids and the locality numbering, on `st`:
// dst[perm[i]] = src[i] (in), dst[i] = src[perm[i]] (out), and a NodeSet's
// bits renumbered (dst is cleared first).
wc_status to_locality(const wc_version* v, cudaStream_t st, const double* src, double* dst);
// A status from ctx.finish() of a solve in the locality order: a node a
// kernel reported (a row of that order) is renamed to its dense id.
wc_status locality_status(Ctx& ctx, wc_status st);
wc_status from_locality(const wc_version* v, cudaStream_t st, const double* src, double* dst);
wc_status bits_to_locality(const wc_version* v, cudaStream_t st, const uint64_t* src,
                           uint64_t* dst);

}  // namespace wc
