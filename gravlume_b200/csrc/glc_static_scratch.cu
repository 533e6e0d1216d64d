// glc_trace_static_scratch: the persistent work-queue trace for callers that cannot allocate
// device memory.
//
// Some hosts embed this library where device allocation is off limits: a renderer whose frame
// allocator owns every byte of device memory and forbids cudaMalloc/cudaFree once the frame loop
// runs (an allocation there synchronizes the device and breaks its frame pacing), or a plugin
// that runs inside another runtime's memory pool and may only touch buffers the host hands it.
// Such callers can still own their inputs and outputs, but not the scratch that glc_create
// allocates for the persistent kernel (its work-queue counter and its device job table).
//
// This entry point keeps that scratch in one file-scope __device__ array of fixed size, so it
// needs no context and allocates nothing. Every GPU that loads the library holds the array until
// the process exits. All calls on a device share it, and it keeps the last call's contents: each
// call rewrites the job table and clears the queue counter before its launch, so two calls whose
// work overlaps on the GPU (different streams without ordering between them) race on the array.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "glc_internal.h"
#include "glc_kernels.cuh"

using namespace glc;

namespace {

// Scratch size: 256 bytes for the queue counter, the rest for the job table (scenes, cameras and
// per-camera ray offsets, each section 256-byte aligned). 96 KiB holds 128 scenes and 128 cameras.
constexpr size_t kScratchBytes = 96 * 1024;
constexpr size_t kQueueBytes = 256;
constexpr int kMaxScenes = 128;
constexpr int kMaxCameras = 128;
constexpr int kMaxDevices = 64;

// In host code this name is a host-side stand-in for the device array, not a device address: the
// address each device uses comes from cudaGetSymbolAddress below.
__device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Device address of the scratch array on the current device, looked up on the first call on the
// device. A cached address is checked before use: after a cudaDeviceReset the library's module is
// loaded again and the array may live elsewhere, and then the address is looked up anew.
glc_status scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned char* ptr = g_scratch_ptr[device];
  if (ptr) {
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
    if (e != cudaSuccess || attr.type != cudaMemoryTypeDevice || attr.device != device) {
      cudaGetLastError();
      ptr = nullptr;
    }
  }
  if (!ptr) {
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_trace_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(GLC_ERR_CUDA, cudaGetErrorString(e));
    }
    g_scratch_ptr[device] = ptr;
  }
  *out = ptr;
  return GLC_OK;
}

template <int P>
glc_status launch_static(int device, const JobView& job, const glc_policy& pol, const glc_results& out,
                         cudaStream_t stream, unsigned long long* queue) {
  const unsigned block = pol.block_threads;
  if (pol.persistent == 0) {
    const unsigned long long grid = (job.total + block - 1) / block;
    if (grid > 0x7fffffffull) return set_error(GLC_ERR_CAPACITY, "too many rays for one launch");
    trace_simple_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, 0ull);
  } else {
    int per_sm = int(pol.blocks_per_sm);
    if (per_sm <= 0) {
      const cudaError_t e =
          pol.persistent == 2
              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_queue_kernel<P>, int(block), 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_persistent_kernel<P>, int(block), 0);
      if (e != cudaSuccess) return set_error(GLC_ERR_CUDA, cudaGetErrorString(e));
      if (per_sm <= 0) per_sm = 1;
    }
    int sms = 0;
    const cudaError_t ea = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (ea != cudaSuccess) return set_error(GLC_ERR_CUDA, cudaGetErrorString(ea));
    const unsigned long long warps_needed = (job.total + 31) / 32;
    unsigned long long grid = (unsigned long long)sms * per_sm;
    const unsigned long long grid_cap = (warps_needed * 32 + block - 1) / block;
    if (grid > grid_cap) grid = grid_cap < 1 ? 1 : grid_cap;
    if (pol.persistent == 2)
      trace_queue_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, queue, Handoff{nullptr, 0});
    else
      trace_persistent_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, queue, Handoff{nullptr, 0});
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(GLC_ERR_CUDA, cudaGetErrorString(e));
  return GLC_OK;
}

}  // namespace

extern "C" glc_status glc_trace_static_scratch(const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                                               int32_t n_cameras, const glc_policy* policy, const glc_results* out,
                                               void* stream) {
  if (!scenes || !cameras || !policy || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (n_scenes <= 0 || n_cameras <= 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "scenes and cameras must be non-empty");
  if (n_scenes > kMaxScenes || n_cameras > kMaxCameras)
    return set_error(GLC_ERR_CAPACITY,
                     "glc_trace_static_scratch takes at most 128 scenes and 128 cameras (96 KiB of static scratch)");
  const glc_policy& pol = *policy;
  glc_status ps = check_policy(pol);
  if (ps != GLC_OK) return ps;
  if (pol.capture_certificates || pol.escape_map)
    return set_error(GLC_ERR_INVALID_ARGUMENT,
                     "glc_trace_static_scratch has no certificate or escape-map buffers: set capture_certificates "
                     "and escape_map to 0");

  // Job table, laid out in a host buffer of the scratch's size (no allocation on either side).
  const size_t off_scenes = 0;
  const size_t off_cams = align256(sizeof(glc_scene) * size_t(n_scenes));
  const size_t off_begin = off_cams + align256(sizeof(glc_camera) * size_t(n_cameras));
  const size_t job_bytes = off_begin + align256(sizeof(unsigned long long) * size_t(n_cameras + 1));
  if (kQueueBytes + job_bytes > kScratchBytes)
    return set_error(GLC_ERR_CAPACITY, "job table exceeds the 96 KiB static scratch");
  alignas(256) static thread_local unsigned char stage[kScratchBytes];
  unsigned long long* begin = reinterpret_cast<unsigned long long*>(stage + off_begin);
  unsigned long long acc = 0;
  for (int i = 0; i < n_cameras; ++i) {
    unsigned long long n = 0;
    const glc_status s = camera_ray_count(cameras[i], scenes, n_scenes, pol, &n);
    if (s != GLC_OK) return s;
    begin[i] = acc;
    acc += n;
  }
  begin[n_cameras] = acc;
  std::memcpy(stage + off_scenes, scenes, sizeof(glc_scene) * size_t(n_scenes));
  std::memcpy(stage + off_cams, cameras, sizeof(glc_camera) * size_t(n_cameras));

  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0) {
    cudaGetLastError();
    return set_error(GLC_ERR_NO_DEVICE, "no current CUDA device");
  }
  if (device >= kMaxDevices) return set_error(GLC_ERR_CAPACITY, "device index beyond the static scratch table");
  unsigned char* scratch = nullptr;
  glc_status s = scratch_address(device, &scratch);
  if (s != GLC_OK) return s;
  if (acc == 0) return GLC_OK;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long* queue = reinterpret_cast<unsigned long long*>(scratch);
  unsigned char* job_dev = scratch + kQueueBytes;
  // The stage is pageable: the copy returns once the runtime has taken the bytes, so the next call
  // on this thread may overwrite it.
  cudaError_t e = cudaMemcpyAsync(job_dev, stage, job_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return set_error(GLC_ERR_CUDA, cudaGetErrorString(e));

  JobView job;
  job.scenes = reinterpret_cast<const glc_scene*>(job_dev + off_scenes);
  job.cams = reinterpret_cast<const glc_camera*>(job_dev + off_cams);
  job.begin = reinterpret_cast<const unsigned long long*>(job_dev + off_begin);
  job.n_cams = n_cameras;
  job.total = acc;
  job.cert_begin = nullptr;  // no certificate or escape-map buffers without a context: every ray
  job.cert = nullptr;        // is integrated
  job.emap_begin = nullptr;
  job.emap = nullptr;
  switch (pol.precision) {
    case GLC_FP32: return launch_static<kFP32>(device, job, pol, *out, st, queue);
    case GLC_MIXED: return launch_static<kMIXED>(device, job, pol, *out, st, queue);
    default: return launch_static<kFP64>(device, job, pol, *out, st, queue);
  }
}
