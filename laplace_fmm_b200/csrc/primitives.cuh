// Device-wide primitives: exclusive scan and a stable LSD radix sort.
// Written for sm_100a: warp shuffles / match_any / ballots inside the block,
// reduce-then-scan across blocks.  No library calls.
#pragma once
#include "common.cuh"

namespace lfmm {

// Scratch (in 4-byte words) that scan_exclusive_u32 needs for n elements.
size_t scan_scratch_words(size_t n);
// out[i] = sum_{j<i} in[j]; *total (device) = sum of all.  in may equal out.
void scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* scratch,
                        cudaStream_t s);

// Scratch (in 4-byte words) that radix_sort_pairs needs for n elements.
size_t radix_scratch_words(size_t n);
// Stable sort of (keys, vals) by key bits [begin_bit, end_bit).  keys_alt /
// vals_alt are ping-pong buffers of the same length.  Returns 0 when the
// result is in (keys, vals), 1 when it is in (keys_alt, vals_alt).
int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, size_t n,
                     int begin_bit, int end_bit, uint32_t* scratch, cudaStream_t s);

} // namespace lfmm
