// Internal interface between plan.cu and noalloc.cu (not part of the C ABI).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "pycusaxs_b200.h"

namespace saxs {

// Device the plan was created on.
int plan_device(const SaxsPlan *plan);

// Bytes of device scratch one frame of this plan needs when every per-frame
// buffer is carved out of caller-provided memory.
size_t single_frame_scratch_bytes(const SaxsPlan *plan);

// One frame through the plan's kernels with all per-frame buffers taken from
// `scratch` (at least single_frame_scratch_bytes, 256-byte aligned); the
// frame's histogram is written to hist_dev / nhist_dev (zeroed first).  The
// plan's accumulators are not touched.  Allocates nothing.
int forward_into_scratch(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                         unsigned char *scratch, size_t scratch_bytes, double *hist_dev,
                         double *nhist_dev, cudaStream_t st);

// Record a failure for saxs_last_error() and return `code`; clear it.
int record_error(int code, const char *msg);
void clear_error();

// Resolve (and cache) the device address of the allocation-free entry point's
// scratch array on `device`, which loads the array onto that device.  Called
// at plan creation; returns SAXS_OK or the error code (message recorded).
int noalloc_attach(int device);

}  // namespace saxs
