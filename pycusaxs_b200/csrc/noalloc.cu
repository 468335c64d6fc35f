// Allocation-free single-frame forward.
//
// Some hosts that embed this library cannot let it call cudaMalloc: an MD engine
// or application that owns every byte of device memory through its own pool and
// budget, or a per-step loop that must neither stall on the allocator nor risk
// running out of memory half-way through a long run.  saxs_forward_noalloc lets
// such a caller compute one frame's histogram with buffers it already owns: it
// passes the frame's positions and the output histogram, and every temporary
// the frame needs (sorted atoms, bin offsets, z- and y-transformed planes, the
// k-box intensities) is carved out of one fixed device array declared below.
//
// Limits and caveats, in one place:
//  * The array holds SAXS_NOALLOC_SCRATCH_BYTES (32 MiB).  It is part of this
//    module's image, so every GPU on which the module is loaded keeps those
//    32 MiB until the process exits.  Frames whose plan needs more (large grids
//    with a large q-cut) are refused with SAXS_E_RANGE and a message giving the
//    size needed.
//  * All calls share the one array, and it keeps whatever the previous call
//    left in it; the call clears the parts that accumulate.  Two calls whose
//    work overlaps on the GPU (different streams, or different host threads on
//    the same device) overwrite each other's temporaries: serialise them.
//  * The array's device address is looked up (cudaGetSymbolAddress, with the
//    device current) by saxs_plan_create, which also loads the array onto the
//    device then, at a time when the caller accepts allocations; the address is
//    cached per device.  Only if that look-up failed does the first call do it
//    (and that call should then come before any stream capture).  A device
//    reset (cudaDeviceReset) invalidates plans and the cached address alike;
//    plans created after it refresh the address.
//  * A kernel of the frame that gives up on a bounded wait, or positions that
//    hold NaN or infinity, make the call's histogram NaN: the call is
//    asynchronous and cannot return that status itself.  The plan's own status
//    word and accumulators are untouched.
//  * The call allocates nothing: no cudaMalloc, cudaFree or allocating library
//    routine is reached from it.  The plan itself is created (and allocates)
//    with saxs_plan_create beforehand, at a time when allocating is acceptable.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "pycusaxs_b200.h"
#include "scratch_forward.h"

namespace {

constexpr size_t kScratchBytes = SAXS_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The shared scratch block.  In host code this name stands for a host-side
// shadow, not a device address: kernels only ever receive the pointer that
// cudaGetSymbolAddress returned for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch block on `device` (which must be current);
// `refresh` looks it up again even when an address is cached.
int scratch_address(int device, unsigned char **out, bool refresh = false) {
  if (device < 0 || device >= kMaxDevices)
    return saxs::record_error(SAXS_E_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[device] || refresh) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      const std::string msg =
          std::string("cudaGetSymbolAddress of the scratch block failed: ") + cudaGetErrorString(e);
      return saxs::record_error(SAXS_E_CUDA, msg.c_str());
    }
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch_ptr[device]);
  return SAXS_OK;
}

}  // namespace

namespace saxs {

int noalloc_attach(int device) {
  unsigned char *p = nullptr;
  return scratch_address(device, &p, true);
}

}  // namespace saxs

extern "C" int saxs_forward_noalloc(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                                    double *hist_dev, double *nhist_dev, void *stream) {
  saxs::clear_error();
  if (!plan) return saxs::record_error(SAXS_E_INVALID, "null plan");
  const size_t need = saxs::single_frame_scratch_bytes(plan);
  if (need > kScratchBytes) {
    const std::string msg = "this plan needs " + std::to_string(need) +
                            " bytes of scratch per frame; the allocation-free entry point holds "
                            "at most " + std::to_string(kScratchBytes) +
                            " bytes (use saxs_forward instead)";
    return saxs::record_error(SAXS_E_RANGE, msg.c_str());
  }
  int prev = 0;
  cudaGetDevice(&prev);
  const int dev = saxs::plan_device(plan);
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess)
    return saxs::record_error(SAXS_E_CUDA, "cannot make the plan's device current");
  unsigned char *scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc == SAXS_OK)
    rc = saxs::forward_into_scratch(plan, xyz_dev, box_host, scratch, kScratchBytes, hist_dev,
                                    nhist_dev, static_cast<cudaStream_t>(stream));
  if (prev != dev) cudaSetDevice(prev);
  return rc;
}
