// speedy_noalloc.cu -- spd_fwd_noalloc: the plain forward for callers that cannot allocate.
//
// Some callers have no way to obtain device scratch: a foreign-function bridge (cgo, JNI, a
// ctypes stub) that only forwards the state, forcing and tendency buffers handed to it, or a
// process whose device memory is owned entirely by another runtime's pooling allocator.  This
// entry point needs no scratch argument and performs no allocation: its scratch lives in the
// fixed file-scope device array below.  The call's launch words and the instance's level-set
// state take its first 256 bytes; the rest holds up to SPD_NOALLOC_MAX_IL rows of a
// per-latitude table (the size limit of the entry point; the present kernels form each
// column's solar row themselves and leave it unused).  Every GPU that loads the library keeps
// that array (65,792 bytes) until the process exits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "speedy_column_smem.cuh"

namespace spd {
// Defined in speedy_api.cu.
int check_forward_instance(const spd_desc_t* d, const spd_inputs_t* in,
                           const spd_outputs_t* out);
Consts make_consts(const spd_desc_t* d, const spd_vgrid_t* vg, const spd_params_t* p);
int dispatch_fwd(const ConstsD& CD, int kx, const spd_inputs_t& in, const spd_outputs_t& out,
                 uint32_t* header, cudaStream_t st, cudaEvent_t marker);
}  // namespace spd

namespace {

constexpr size_t kNoallocHeader = 256;  // launch words, level-set state, padding
constexpr size_t kNoallocBytes = kNoallocHeader + (size_t)SPD_NOALLOC_MAX_IL * sizeof(spd::ZonalRow);

// The shared scratch.  In host code this name is only a host-side stand-in for the symbol;
// its device address comes from cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// Device address of g_noalloc_scratch in the current device's context.  It is looked up on
// every call (after the first call on a device, which loads the module, this is a table lookup
// in the runtime), so no address outlives the context it belongs to: after cudaDeviceReset or
// any other teardown of the primary context, the next call gets the new context's address.
int scratch_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SPD_ERR_CUDA;
  *out = p;
  return SPD_OK;
}

// The array exists once per device, so the call must run on the device whose array it uses:
// the stream's device must be the current device.
int check_stream_device(cudaStream_t st) {
  int cur = -1, sdev = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return SPD_ERR_CUDA;
  if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) return SPD_ERR_CUDA;
  return sdev == cur ? SPD_OK : SPD_ERR_STREAM_DEVICE;
}

}  // namespace

extern "C" int spd_fwd_noalloc(const spd_desc_t* desc, const spd_vgrid_t* vgrid,
                               const spd_params_t* params, const spd_inputs_t* in,
                               const spd_outputs_t* out, void* stream) {
  int rc = spd::check_forward_instance(desc, in, out);
  if (rc != SPD_OK) return rc;
  if (!vgrid || !params) return SPD_ERR_NULL;
  if (desc->il > SPD_NOALLOC_MAX_IL) return SPD_ERR_NOALLOC_LIMIT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  rc = check_stream_device(st);
  if (rc != SPD_OK) return rc;
  void* scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc != SPD_OK) return rc;
  spd::ConstsD CD;
  CD.K = spd::make_consts(desc, vgrid, params);
  CD.D = spd::derive_constants(desc, vgrid, params);
  // The array keeps the previous call's contents: the call clears the words that must start
  // at zero itself, and keeps the previous call's level set as its prediction (a prediction
  // that misses, e.g. after another instance's call, costs a second pass, never a wrong
  // result).
  return spd::dispatch_fwd(CD, desc->kx, *in, *out, static_cast<uint32_t*>(scratch), st,
                           nullptr);
}
