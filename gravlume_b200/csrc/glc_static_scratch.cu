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

// Device address of the scratch array on the current device, looked up once per device.
glc_status scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    unsigned char* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_trace_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(GLC_ERR_CUDA, cudaGetErrorString(e));
    }
    g_scratch_ptr[device] = ptr;
  }
  *out = g_scratch_ptr[device];
  return GLC_OK;
}

// Ray count of one camera under the policy's tile padding, with the checks glc_trace applies.
glc_status camera_rays(const glc_camera& c, const glc_scene* scenes, int32_t n_scenes, const glc_policy& pol,
                       unsigned long long* n) {
  if (c.scene_index < 0 || c.scene_index >= n_scenes)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "camera scene index out of range");
  if (c.kind == GLC_CAMERA_RAYLIST) {
    if (!c.ray_states && c.n_rays > 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "ray list needs states");
    if (!(c.affine_direction == 1.0 || c.affine_direction == -1.0))
      return set_error(GLC_ERR_INVALID_ARGUMENT, "affine direction must be +1 or -1");
    if ((reinterpret_cast<uintptr_t>(c.ray_states) & 15u) != 0)
      return set_error(GLC_ERR_INVALID_ARGUMENT, "ray states must be 16-byte aligned");
    *n = c.n_rays;
    return GLC_OK;
  }
  if (c.kind != GLC_CAMERA_PINHOLE && c.kind != GLC_CAMERA_EQUIRECT)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown camera kind");
  if (c.width == 0 || c.height == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "camera size must be nonzero");
  if (!(c.subpixel_x >= 0.0 && c.subpixel_x <= 1.0 && c.subpixel_y >= 0.0 && c.subpixel_y <= 1.0))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "subpixel offsets must lie in [0, 1]");
  if (c.kind == GLC_CAMERA_PINHOLE &&
      (c.width != scenes[c.scene_index].width || c.height != scenes[c.scene_index].height))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "pinhole camera size must match the scene's view");
  const unsigned long long tx = (c.width + pol.tile_w - 1) / pol.tile_w;
  const unsigned long long ty = (c.height + pol.tile_h - 1) / pol.tile_h;
  *n = tx * ty * pol.tile_w * pol.tile_h;
  return GLC_OK;
}

template <int P>
glc_status launch_static(int device, const JobView& job, const glc_policy& pol, const glc_results& out,
                         cudaStream_t stream, unsigned long long* queue) {
  const unsigned block = pol.block_threads;
  int per_sm = int(pol.blocks_per_sm);
  if (per_sm <= 0) {
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_persistent_kernel<P>, int(block), 0);
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
  trace_persistent_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, queue);
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
  if (pol.tile_w == 0 || pol.tile_h == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "tile shape must be nonzero");
  if (pol.block_threads == 0 || pol.block_threads % 32 != 0 || pol.block_threads > 128)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 up to 128");
  if (pol.precision < GLC_FP32 || pol.precision > GLC_FP64)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown precision mode");
  const double positive[] = {pol.position_rtol, pol.position_atol, pol.momentum_rtol, pol.momentum_atol,
                             pol.initial_step,  pol.minimum_step,  pol.maximum_step,  pol.safety,
                             pol.minimum_factor, pol.maximum_factor, pol.event_affine_tolerance,
                             pol.singularity_guard};
  for (double x : positive)
    if (!(x > 0.0) || !(x < 1.0e300)) return set_error(GLC_ERR_INVALID_ARGUMENT, "policy values must be positive");
  if (pol.minimum_step > pol.maximum_step || pol.maximum_accepted_steps == 0 || pol.maximum_consecutive_rejects == 0)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "inconsistent step limits");

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
    const glc_status s = camera_rays(cameras[i], scenes, n_scenes, pol, &n);
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
