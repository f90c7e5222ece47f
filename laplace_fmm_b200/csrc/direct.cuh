// FP64 direct-sum oracle on the device.
#pragma once
#include "context.cuh"

namespace lfmm {

// Source chunks for nt targets (1: no split), at most max_chunks.
int direct_chunks(size_t ns, size_t nt, int num_sms, size_t max_chunks);
// Enqueue with S source chunks; part: scratch of 4 * nt * S doubles (written
// before it is read; nothing needs to start at zero), unused when S == 1.
// fast: 3D 1/r from the FP64 reciprocal square root approximation refined
// by one third-order series step (the sampled checks); otherwise an FP64
// square root and divide per pair.
int direct_launch(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt,
                  const double* tgt, double* pot, double* fld, double* part, int S, bool fast = false);
// Load the 3D FP64 kernels that direct_launch may use (fast = false) into the
// current device's context now rather than at their first launch (under lazy
// module loading a first launch may allocate device memory).
int direct_preload3(Context& ctx);
// Enqueue on ctx.stream, scratch from the arena; all pointers are device pointers.
int direct_device(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* fld, bool fast = false);

// Target i (3D) against the sources of its segment [poff[seg[i]], poff[seg[i] + 1])
// only: the sampled checks of a batch of problems in one launch (FAST 1/r).
int direct_segments_device(Context& ctx, const double* src, const double* q, const uint32_t* poff,
                           const int32_t* seg, size_t m, const double* tgt, double* pot, double* fld);

} // namespace lfmm
