// FP64 direct-sum oracle on the device.
#pragma once
#include "context.cuh"

namespace lfmm {

// Enqueue on ctx.stream; all pointers are device pointers.
int direct_device(Context& ctx, int dim, size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                  double* pot, double* fld);

} // namespace lfmm
