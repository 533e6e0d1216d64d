// C ABI implementation: contexts, job tables, trace launches, CUDA graphs and the autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "glc_context.h"
#include "glc_internal.h"
#include "glc_certificate.cuh"
#include "glc_escape_map.cuh"
#include "glc_shadow.cuh"
#include "glc_footprint.cuh"

using namespace glc;

namespace glc {
namespace {
thread_local std::string g_last_error;
}

glc_status set_error(glc_status status, const char* message) {
  g_last_error = message ? message : "";
  return status;
}
}  // namespace glc

namespace glc {

// The reference's synthetic event-policy cases (event_policy_capture.wgsl), evaluated by the trace
// kernels' own earliest-event selection and arming test: one thread per case.
template <int kCases>
__global__ void event_policy_cases_kernel(glc_policy pol, uint32_t* out) {
  const int c = int(threadIdx.x);
  if (c >= kCases) return;
  uint32_t r[4] = {0u, 0u, 0u, 0u};
  const double tie = pol.event_tie_tolerance, band = pol.event_arming_band;
  if (c < 4) {
    int kinds[4];
    double thetas[4];
    int n = 0;
    double step = 1.0;
    if (c == 3) {
      // horizon at one half, the surface 0.75 tie tolerances before it, the escape sphere as far after
      const double off = 0.75 * tie / step;
      kinds[n] = kEvHorizon, thetas[n++] = 0.5;
      kinds[n] = kEvSurface, thetas[n++] = 0.5 - off;
      kinds[n] = kEvEscape, thetas[n++] = 0.5 + off;
    } else {
      // escape sphere at one half; the surface half a tie tolerance later (cases 0 and 1, at the
      // largest and the smallest step) or at the same fraction (case 2)
      step = c == 0 ? pol.maximum_step : pol.minimum_step;
      kinds[n] = kEvSurface, thetas[n++] = c < 2 ? 0.5 + 0.5 * tie / step : 0.5;
      kinds[n] = kEvEscape, thetas[n++] = 0.5;
    }
    uint32_t cand = 0;
    const int first = earliest_event<double>(kinds, thetas, n, step, tie, cand);
    r[0] = first >= 0 ? termination_of_event(kinds[first]) : 0u;
    r[1] = cand;
    r[2] = (cand & (cand - 1u)) != 0u ? 1u : 0u;
  } else {
    // surface arming: value 0, half the band, twice the band, and an event armed before
    const double v = c == 5 ? 0.5 * band : (c == 6 ? 2.0 * band : 0.0);
    const bool armed = c == 7 || event_clears_band<double>(kEvSurface, v, band);
    r[0] = armed ? 1u : 0u;
  }
  reinterpret_cast<uint4*>(out)[c] = make_uint4(r[0], r[1], r[2], r[3]);
}

}  // namespace glc

#define GLC_CUDA(expr)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      std::string m_ = std::string(#expr) + ": " + cudaGetErrorString(e_);                      \
      return set_error(GLC_ERR_CUDA, m_.c_str());                                               \
    }                                                                                           \
  } while (0)

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Host-side description of a job: padded ray counts per camera and the device-table layout.
struct JobLayout {
  std::vector<unsigned long long> begin;
  std::vector<unsigned long long> cert_begin;  // 16x16 certificate tiles of each image camera
  std::vector<unsigned long long> emap_begin;  // escape-map nodes of each image camera
  unsigned long long total = 0;
  size_t off_scenes = 0, off_cams = 0, off_begin = 0, off_cert_begin = 0, off_emap_begin = 0, bytes = 0;
};

// A camera's tile region (TileRegion, trace.rs:799-857): whole view ({0, 0} tiles), or a non-empty
// block of 8x8-pixel tiles inside the view's tile grid (tile_grid, trace.rs:851-856).
glc_status validate_region(const glc_camera& c) {
  if (c.tile_count[0] == 0u && c.tile_count[1] == 0u) {
    if (c.tile_origin[0] != 0u || c.tile_origin[1] != 0u)
      return set_error(GLC_ERR_INVALID_ARGUMENT, "a whole-view camera has tile origin (0, 0)");
    return GLC_OK;
  }
  if (c.kind == GLC_CAMERA_RAYLIST) return set_error(GLC_ERR_INVALID_ARGUMENT, "ray lists have no tile region");
  const uint64_t gx = (uint64_t(c.width) + kRegionTile - 1) / kRegionTile;
  const uint64_t gy = (uint64_t(c.height) + kRegionTile - 1) / kRegionTile;
  if (c.tile_count[0] == 0u || c.tile_count[1] == 0u ||
      uint64_t(c.tile_origin[0]) + c.tile_count[0] > gx || uint64_t(c.tile_origin[1]) + c.tile_count[1] > gy)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "tile region outside the view's tile grid");
  return GLC_OK;
}

bool whole_view(const glc_camera& c) { return c.tile_count[0] == 0u && c.tile_count[1] == 0u; }

}  // namespace

// Rays of one camera under the policy's tile padding (its tile region for image cameras), with
// the camera checks of every trace entry point.
glc_status glc::camera_ray_count(const glc_camera& c, const glc_scene* scenes, int32_t n_scenes,
                                 const glc_policy& pol, unsigned long long* n) {
  if (pol.tile_w == 0 || pol.tile_h == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "tile shape must be nonzero");
  if (c.scene_index < 0 || c.scene_index >= n_scenes)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "camera scene index out of range");
  const glc_status rs = validate_region(c);
  if (rs != GLC_OK) return rs;
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
  const PixelRect rc = camera_rect(c);
  const unsigned long long tx = (rc.x1 - rc.x0 + pol.tile_w - 1) / pol.tile_w;
  const unsigned long long ty = (rc.y1 - rc.y0 + pol.tile_h - 1) / pol.tile_h;
  *n = tx * ty * pol.tile_w * pol.tile_h;
  return GLC_OK;
}

namespace {

glc_status validate_job(const glc_scene* scenes, int32_t n_scenes, const glc_camera* cams, int32_t n_cams,
                        const glc_policy& pol, JobLayout& L) {
  if (!scenes || !cams || n_scenes <= 0 || n_cams <= 0)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "scenes and cameras must be non-empty");
  if (pol.tile_w == 0 || pol.tile_h == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "tile shape must be nonzero");
  L.begin.assign(size_t(n_cams) + 1, 0);
  L.cert_begin.assign(size_t(n_cams) + 1, 0);
  L.emap_begin.assign(size_t(n_cams) + 1, 0);
  unsigned long long acc = 0, tiles = 0, nodes = 0;
  for (int i = 0; i < n_cams; ++i) {
    const glc_camera& c = cams[i];
    unsigned long long n = 0;
    const glc_status cs = camera_ray_count(c, scenes, n_scenes, pol, &n);
    if (cs != GLC_OK) return cs;
    L.begin[i] = acc;
    acc += n;
    L.cert_begin[i] = tiles;
    L.emap_begin[i] = nodes;
    if (c.kind != GLC_CAMERA_RAYLIST) {
      tiles += (unsigned long long)((c.width + kCertTile - 1) / kCertTile) * ((c.height + kCertTile - 1) / kCertTile);
      nodes += (unsigned long long)map_grid_w(c.width) * map_grid_h(c.height);
    }
  }
  L.begin[n_cams] = acc;
  L.cert_begin[n_cams] = tiles;
  L.emap_begin[n_cams] = nodes;
  L.total = acc;
  L.off_scenes = 0;
  L.off_cams = align256(sizeof(glc_scene) * n_scenes);
  L.off_begin = L.off_cams + align256(sizeof(glc_camera) * n_cams);
  L.off_cert_begin = L.off_begin + align256(sizeof(unsigned long long) * (n_cams + 1));
  L.off_emap_begin = L.off_cert_begin + align256(sizeof(unsigned long long) * (n_cams + 1));
  L.bytes = L.off_emap_begin + align256(sizeof(unsigned long long) * (n_cams + 1));
  return GLC_OK;
}

void fill_staging(unsigned char* stage, const JobLayout& L, const glc_scene* scenes, int32_t n_scenes,
                  const glc_camera* cams, int32_t n_cams) {
  std::memcpy(stage + L.off_scenes, scenes, sizeof(glc_scene) * n_scenes);
  std::memcpy(stage + L.off_cams, cams, sizeof(glc_camera) * n_cams);
  std::memcpy(stage + L.off_begin, L.begin.data(), sizeof(unsigned long long) * (n_cams + 1));
  std::memcpy(stage + L.off_cert_begin, L.cert_begin.data(), sizeof(unsigned long long) * (n_cams + 1));
  std::memcpy(stage + L.off_emap_begin, L.emap_begin.data(), sizeof(unsigned long long) * (n_cams + 1));
}

JobView job_view(const unsigned char* dev, const JobLayout& L, int32_t n_cams) {
  JobView v;
  v.scenes = reinterpret_cast<const glc_scene*>(dev + L.off_scenes);
  v.cams = reinterpret_cast<const glc_camera*>(dev + L.off_cams);
  v.begin = reinterpret_cast<const unsigned long long*>(dev + L.off_begin);
  v.n_cams = n_cams;
  v.total = L.total;
  v.cert_begin = reinterpret_cast<const unsigned long long*>(dev + L.off_cert_begin);
  v.cert = nullptr;
  v.emap_begin = reinterpret_cast<const unsigned long long*>(dev + L.off_emap_begin);
  v.emap = nullptr;
  return v;
}

}  // namespace

struct glc_graph {
  glc_ctx* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned char* d_job = nullptr;
  unsigned char* h_stage = nullptr;
  unsigned long long* d_queue = nullptr;
  uint32_t* d_cert = nullptr;
  uint32_t* d_emap = nullptr;
  unsigned char* d_handoff = nullptr;
};

namespace {

template <int P>
glc_status launch_precision(glc_ctx* ctx, const JobView& job, const glc_policy& pol, const glc_results& out,
                            cudaStream_t stream, unsigned long long* queue, Handoff hv = Handoff{nullptr, 0}) {
  const unsigned block = pol.block_threads;
  if (pol.persistent) {
    int per_sm = int(pol.blocks_per_sm);
    if (per_sm <= 0) {
      if (pol.persistent == 2)
        GLC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_queue_kernel<P>, int(block), 0));
      else
        GLC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_persistent_kernel<P>, int(block), 0));
      if (per_sm <= 0) per_sm = 1;
    }
    const unsigned long long warps_needed = (job.total + 31) / 32;
    unsigned long long grid = (unsigned long long)ctx->sm_count * per_sm;
    const unsigned long long grid_cap = (warps_needed * 32 + block - 1) / block;
    if (grid > grid_cap) grid = grid_cap < 1 ? 1 : grid_cap;
    GLC_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream));
    if (pol.persistent == 2)
      trace_queue_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, queue, hv);
    else
      trace_persistent_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, queue, hv);
    ctx->stats.last_grid = unsigned(grid);
    ctx->stats.kernel_launches += 1;
  } else {
    const unsigned long long grid = (job.total + block - 1) / block;
    if (grid > 0x7fffffffull) return set_error(GLC_ERR_CAPACITY, "too many rays for one launch");
    trace_simple_kernel<P><<<unsigned(grid), block, 0, stream>>>(job, pol, out, 0ull);
    ctx->stats.last_grid = unsigned(grid);
    ctx->stats.kernel_launches += 1;
  }
  GLC_CUDA(cudaGetLastError());
  ctx->stats.last_block = block;
  ctx->stats.last_persistent = pol.persistent;
  ctx->stats.last_rays = job.total;
  return GLC_OK;
}

// MIXED as two kernels (binary32 bulk, then binary64 completion) over the hand-off records; the
// bulk kernel is the one-thread-per-ray kernel or, with `persistent`, a work-queue kernel.
bool split_mixed(const glc_policy& pol) { return pol.precision == GLC_MIXED && pol.mixed_split != 0; }

size_t handoff_bytes(unsigned long long rays) { return size_t(rays) * kHandoffWords * sizeof(uint4); }

glc_status launch_split(glc_ctx* ctx, const JobView& job, const glc_policy& pol, const glc_results& out,
                        cudaStream_t stream, unsigned char* handoff, unsigned long long* queue) {
  const unsigned block = pol.block_threads;
  const unsigned long long grid = (job.total + block - 1) / block;
  if (grid > 0x7fffffffull) return set_error(GLC_ERR_CAPACITY, "too many rays for one launch");
  const Handoff hv{reinterpret_cast<uint4*>(handoff), job.total};
  if (pol.persistent) {
    const glc_status s = launch_precision<kBULK>(ctx, job, pol, out, stream, queue, hv);
    if (s != GLC_OK) return s;
  } else {
    trace_bulk_kernel<kBULK><<<unsigned(grid), block, 0, stream>>>(job, pol, out, hv, 0ull);
    GLC_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 1;
  }
  trace_tail_kernel<kTAIL><<<unsigned(grid), block, 0, stream>>>(job, pol, out, hv, 0ull);
  GLC_CUDA(cudaGetLastError());
  if (!pol.persistent) ctx->stats.last_grid = unsigned(grid);
  ctx->stats.kernel_launches += 1;
  ctx->stats.last_block = block;
  ctx->stats.last_persistent = pol.persistent;
  ctx->stats.last_rays = job.total;
  return GLC_OK;
}

glc_status ensure_bytes(unsigned char** buf, size_t* have, size_t need) {
  if (need <= *have) return GLC_OK;
  if (*buf) GLC_CUDA(cudaFree(*buf));
  *buf = nullptr;
  *have = 0;
  GLC_CUDA(cudaMalloc(buf, need));
  *have = need;
  return GLC_OK;
}

// cert: device words for the job's certificate tiles (at least cert_tiles of them) when the policy
// asks for certificates, else unused. handoff: hand-off records for every ray of the job when the
// policy splits MIXED into two kernels (without it the one-kernel MIXED runs).
glc_status launch(glc_ctx* ctx, const JobView& job_in, const glc_policy& pol, const glc_results& out,
                  cudaStream_t stream, unsigned long long* queue, uint32_t* cert = nullptr,
                  unsigned long long cert_tiles = 0, uint32_t* emap = nullptr, unsigned long long emap_nodes = 0,
                  unsigned char* handoff = nullptr) {
  if (job_in.total == 0) return GLC_OK;
  if (pol.block_threads == 0 || pol.block_threads % 32 != 0 || pol.block_threads > 128)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 up to 128");
  JobView job = job_in;
  if (pol.capture_certificates && cert && cert_tiles > 0) {
    certify_tiles_kernel<<<unsigned((cert_tiles + 127) / 128), 128, 0, stream>>>(job, cert);
    GLC_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 1;
    job.cert = cert;
  }
  if (pol.escape_map && emap && emap_nodes > 0) {
    const unsigned grid = unsigned((emap_nodes + 127) / 128);
    switch (pol.precision) {
      case GLC_FP32: escape_map_nodes_kernel<kFP32><<<grid, 128, 0, stream>>>(job, pol, out, emap); break;
      case GLC_MIXED: escape_map_nodes_kernel<kMIXED><<<grid, 128, 0, stream>>>(job, pol, out, emap); break;
      default: escape_map_nodes_kernel<kFP64><<<grid, 128, 0, stream>>>(job, pol, out, emap); break;
    }
    GLC_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 1;
    job.emap = emap;
  }
  if (split_mixed(pol) && handoff) return launch_split(ctx, job, pol, out, stream, handoff, queue);
  switch (pol.precision) {
    case GLC_FP32: return launch_precision<kFP32>(ctx, job, pol, out, stream, queue);
    case GLC_MIXED: return launch_precision<kMIXED>(ctx, job, pol, out, stream, queue);
    case GLC_FP64: return launch_precision<kFP64>(ctx, job, pol, out, stream, queue);
    default: return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown precision mode");
  }
}

glc_status ensure_cert_capacity(uint32_t** buf, size_t* words, unsigned long long need) {
  if (need <= *words) return GLC_OK;
  if (*buf) GLC_CUDA(cudaFree(*buf));
  *buf = nullptr;
  *words = 0;
  GLC_CUDA(cudaMalloc(buf, need * sizeof(uint32_t)));
  *words = need;
  return GLC_OK;
}

glc_status validate_policy(const glc_policy& p) {
  const double v[] = {p.position_rtol, p.position_atol, p.momentum_rtol, p.momentum_atol, p.initial_step,
                      p.minimum_step,  p.maximum_step,  p.safety,        p.minimum_factor, p.maximum_factor};
  for (double x : v)
    if (!std::isfinite(x) || x <= 0.0) return set_error(GLC_ERR_INVALID_ARGUMENT, "policy values must be positive");
  if (p.minimum_step > p.maximum_step) return set_error(GLC_ERR_INVALID_ARGUMENT, "minimum step exceeds maximum step");
  if (p.maximum_consecutive_rejects == 0 || p.maximum_accepted_steps == 0)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "step and reject limits must be positive");
  if (p.precision < GLC_FP32 || p.precision > GLC_FP64) return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!(p.event_affine_tolerance > 0.0) || !(p.event_tie_tolerance >= 0.0) || !(p.event_arming_band >= 0.0) ||
      !(p.singularity_guard > 0.0))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "event tolerances must be positive");
  if (p.block_threads == 0 || p.block_threads % 32 != 0 || p.block_threads > 128)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 up to 128");
  if (p.tile_w == 0 || p.tile_h == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "tile shape must be nonzero");
  if (p.persistent > 2) return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown kernel choice (persistent 0, 1 or 2)");
  if (p.uncertain_terminals > 1 || !(p.uncertain_drift_limit > 0.0))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "uncertain_terminals is 0 or 1 with a positive drift limit");
  return GLC_OK;
}

glc_status ensure_job_capacity(glc_ctx* ctx, size_t bytes) {
  if (ctx->stage_pending) {
    GLC_CUDA(cudaEventSynchronize(ctx->stage_free));
    ctx->stage_pending = false;
  }
  if (bytes > ctx->d_job_bytes) {
    if (ctx->d_job) GLC_CUDA(cudaFree(ctx->d_job));
    ctx->d_job = nullptr;
    GLC_CUDA(cudaMalloc(&ctx->d_job, bytes));
    ctx->d_job_bytes = bytes;
  }
  if (bytes > ctx->h_stage_bytes) {
    if (ctx->h_stage) GLC_CUDA(cudaFreeHost(ctx->h_stage));
    ctx->h_stage = nullptr;
    GLC_CUDA(cudaMallocHost(&ctx->h_stage, bytes));
    ctx->h_stage_bytes = bytes;
  }
  return GLC_OK;
}

// A band of a host-buffer trace: rays [g0, g1) of the job, whose results fill slots [s0, s1).
struct Band {
  unsigned long long g0, g1, s0, s1;
};

constexpr int kMaxBands = 64;
constexpr unsigned long long kBandRays = 1ull << 19;  // split cameras of more than this many rays

// Row bands of whole tile rows for image cameras (a tile row's results are whole pixel rows, so a
// band's slots are contiguous), equal pieces for ray lists; at most 16 bands a camera.
bool plan_bands(const glc_camera* cams, int32_t n_cams, const JobLayout& L, const glc_policy& pol,
                std::vector<Band>& bands) {
  bands.clear();
  for (int c = 0; c < n_cams; ++c)
    if (!whole_view(cams[c])) return false;  // a tile region's slots are not contiguous rows
  for (int c = 0; c < n_cams; ++c) {
    const unsigned long long g = L.begin[c], rays = L.begin[c + 1] - g;
    if (rays == 0) continue;
    const unsigned long long nb = std::min<unsigned long long>(16, std::max<unsigned long long>(1, rays / kBandRays));
    if (cams[c].kind == GLC_CAMERA_RAYLIST) {
      for (unsigned long long k = 0; k < nb; ++k) {
        const unsigned long long j0 = rays * k / nb, j1 = rays * (k + 1) / nb;
        bands.push_back({g + j0, g + j1, cams[c].result_offset + j0, cams[c].result_offset + j1});
      }
    } else {
      const unsigned long long W = cams[c].width, H = cams[c].height;
      const unsigned long long tiles_x = (W + pol.tile_w - 1) / pol.tile_w, tile_rows = (H + pol.tile_h - 1) / pol.tile_h;
      const unsigned long long row_rays = tiles_x * pol.tile_w * pol.tile_h;
      const unsigned long long per = (tile_rows + nb - 1) / nb;
      for (unsigned long long r0 = 0; r0 < tile_rows; r0 += per) {
        const unsigned long long r1 = std::min(r0 + per, tile_rows);
        bands.push_back({g + r0 * row_rays, g + r1 * row_rays, cams[c].result_offset + r0 * pol.tile_h * W,
                         cams[c].result_offset + std::min(r1 * pol.tile_h, H) * W});
      }
    }
  }
  return int(bands.size()) <= kMaxBands;
}

template <int P>
void launch_band(const JobView& job, const glc_policy& pol, const glc_results& out, const Band& b, cudaStream_t st) {
  JobView jb = job;
  jb.total = b.g1;  // rays past the band's end return at once
  const unsigned long long grid = (b.g1 - b.g0 + pol.block_threads - 1) / pol.block_threads;
  trace_simple_kernel<P><<<unsigned(grid), pol.block_threads, 0, st>>>(jb, pol, out, b.g0);
}

// The two MIXED kernels on one band; the hand-off records are indexed by the job's ray index, so
// bands in flight on different streams use disjoint records.
void launch_band_split(const JobView& job, const glc_policy& pol, const glc_results& out, const Band& b,
                       cudaStream_t st, unsigned char* handoff) {
  JobView jb = job;
  jb.total = b.g1;
  const unsigned long long grid = (b.g1 - b.g0 + pol.block_threads - 1) / pol.block_threads;
  const Handoff hv{reinterpret_cast<uint4*>(handoff), job.total};
  trace_bulk_kernel<kBULK><<<unsigned(grid), pol.block_threads, 0, st>>>(jb, pol, out, hv, b.g0);
  trace_tail_kernel<kTAIL><<<unsigned(grid), pol.block_threads, 0, st>>>(jb, pol, out, hv, b.g0);
}

glc_status ensure_host_streams(glc_ctx* ctx) {
  for (cudaStream_t& c : ctx->host_compute)
    if (!c) GLC_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
  if (!ctx->host_upload) GLC_CUDA(cudaEventCreateWithFlags(&ctx->host_upload, cudaEventDisableTiming));
  if (!ctx->host_copy) GLC_CUDA(cudaStreamCreateWithFlags(&ctx->host_copy, cudaStreamNonBlocking));
  for (cudaEvent_t& e : ctx->host_band)
    if (!e) GLC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (!ctx->host_entry) GLC_CUDA(cudaEventCreateWithFlags(&ctx->host_entry, cudaEventDisableTiming));
  return GLC_OK;
}

}  // namespace

glc_status glc::check_policy(const glc_policy& p) { return validate_policy(p); }

extern "C" {

int glc_abi_version(void) { return GLC_ABI_VERSION; }

const char* glc_last_error_string(void) { return g_last_error.c_str(); }

const char* glc_status_string(glc_status s) {
  switch (s) {
    case GLC_OK: return "ok";
    case GLC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case GLC_ERR_CUDA: return "CUDA error";
    case GLC_ERR_NON_FINITE: return "non-finite input";
    case GLC_ERR_NON_POSITIVE: return "non-positive input";
    case GLC_ERR_NON_NORMALIZED: return "observer frequency not normalized";
    case GLC_ERR_EXTREMALITY_CHANGED: return "extremality changed by normalization";
    case GLC_ERR_NON_STATIONARY: return "observer is not stationary";
    case GLC_ERR_DEGENERATE_FRAME: return "degenerate observer frame";
    case GLC_ERR_SURFACE_OUTSIDE_ESCAPE: return "surface outside the escape sphere";
    case GLC_ERR_INVALID_SURFACE: return "invalid surface";
    case GLC_ERR_INVALID_VIEW: return "invalid view";
    case GLC_ERR_TIMEOUT: return "device wait timed out";
    case GLC_ERR_CAPACITY: return "capacity exceeded";
    case GLC_ERR_NO_DEVICE: return "no CUDA device";
    case GLC_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

glc_status glc_scene_pack(const glc_scene_input* input, glc_scene* out) {
  if (!input || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  return pack_scene(*input, *out);
}

glc_status glc_prograde_isco(double spin, double charge, double* out) {
  if (!out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (!std::isfinite(spin) || !std::isfinite(charge)) return set_error(GLC_ERR_NON_FINITE, "non-finite input");
  if (spin * spin + charge * charge >= 1.0) return set_error(GLC_ERR_INVALID_ARGUMENT, "ISCO needs a subextremal hole");
  *out = prograde_isco(spin, charge);
  return GLC_OK;
}

glc_status glc_policy_default(int32_t preset, int32_t precision, glc_policy* out) {
  if (!out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (precision < GLC_FP32 || precision > GLC_FP64) return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown precision");
  glc_policy p{};
  // reference-regular-v1 (crates/gravlume-reference/src/policy.rs:28-48)
  p.position_rtol = p.momentum_rtol = 2.0e-12;
  p.position_atol = p.momentum_atol = 2.0e-13;
  p.initial_step = 1.0e-3;
  p.minimum_step = 9.094947017729282e-13;
  p.maximum_step = 0.5;
  p.safety = 0.9;
  p.minimum_factor = 0.2;
  p.maximum_factor = 5.0;
  p.maximum_accepted_steps = 200000;
  p.maximum_consecutive_rejects = 64;
  p.event_affine_tolerance = 2.0e-11;
  p.event_tie_tolerance = 5.0e-11;
  p.event_arming_band = 1.28e-9;
  p.singularity_guard = 9.094947017729282e-13;
  if (preset == 1) {  // reference-strict-v1 (policy.rs:51-66)
    p.position_rtol /= 16.0;
    p.momentum_rtol /= 16.0;
    p.position_atol /= 16.0;
    p.momentum_atol /= 16.0;
    p.maximum_step = 0.25;
    p.maximum_accepted_steps *= 2;
    p.maximum_consecutive_rejects *= 2;
    p.event_affine_tolerance /= 4.0;
    p.event_tie_tolerance /= 4.0;
  } else if (preset == 2) {
    // frame policy: binary64 modes at rtol 1e-10 / atol 1e-12; binary32 stepping at a tolerance
    // its arithmetic can honour, with event tolerances scaled to its resolution
    if (precision == GLC_FP64) {
      p.position_rtol = p.momentum_rtol = 1.0e-10;
      p.position_atol = p.momentum_atol = 1.0e-12;
    } else {
      // error-controlled steps: the 0.5 M cap of the binary64 presets only multiplies far-field
      // steps (the binary32 controller is roundoff-limited well before it matters)
      p.position_rtol = p.momentum_rtol = 1.0e-6;
      p.position_atol = p.momentum_atol = 1.0e-8;
      p.maximum_step = 1.0e3;
      if (precision == GLC_MIXED) {
        // MIXED steps 0.7 times tighter than FP32, so that the truncation error of every observable
        // sits below FP32's with margin rather than by the chance of a maximum; its two-kernel form
        // still traces the 3840x2160 frame faster than the FP32 kernel at rtol 1e-6
        p.position_rtol = p.momentum_rtol = 7.0e-7;
        p.position_atol = p.momentum_atol = 7.0e-9;
      }
      if (precision == GLC_FP32) {
        p.event_affine_tolerance = 1.0e-6;
        p.event_tie_tolerance = 2.0e-6;
        p.event_arming_band = 1.0e-5;
      }
    }
  } else if (preset != 0) {
    return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown policy preset");
  }
  p.precision = precision;
  p.mixed_shell_factor = 1.2;
  p.renormalize_null = precision == GLC_MIXED ? 1u : 0u;
  // one thread per ray over 4x8 pixel tiles measured fastest for single frames; the autotuner
  // switches to the persistent work queue where ray costs vary more
  p.persistent = 0;
  p.block_threads = 128;
  p.blocks_per_sm = 0;
  p.tile_w = 4;
  p.tile_h = 8;
  p.refill_interval = 4;
  p.rays_per_grab = 64;
  p.refill_min_idle = 16;
  // MIXED carries its state as compensated binary32 pairs: about 3 % slower, and it lowers the
  // binary32 rounding floor of every observable (escape direction 6e-7 -> 2e-7 rad, g 2e-6 -> 9e-7
  // at rtol 1e-7 on the 3840x2160 frame)
  p.mixed_pair_state = precision == GLC_MIXED ? 1u : 0u;
  p.capture_certificates = 0;
  p.escape_map = 0;
  p.mixed_split = 1;
  p.uncertain_terminals = 0;
  p.uncertain_drift_limit = 0.05;
  *out = p;
  return GLC_OK;
}

glc_status glc_selftest_event_policy(const glc_policy* policy, uint32_t* out, void* stream) {
  if (!policy || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if ((reinterpret_cast<uintptr_t>(out) & 15u) != 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "out must be 16-byte aligned");
  const glc_status s = validate_policy(*policy);
  if (s != GLC_OK) return s;
  event_policy_cases_kernel<8><<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(*policy, out);
  GLC_CUDA(cudaGetLastError());
  return GLC_OK;
}

glc_status glc_flop_model(double out4[4]) {
  if (!out4) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  flop_model(out4);
  return GLC_OK;
}

glc_status glc_rhs_host(const glc_scene* scene, const double state6[6], double energy, int32_t precision,
                        double out7[7]) {
  if (!scene || !state6 || !out7) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  const LaneScene ls = make_lane_scene(*scene, 1.0);
  if (precision == GLC_FP32) {
    const KN<float> k = kn_cast<float>(ls.kn);
    float y[6], d[7], r, vr;
    for (int i = 0; i < 6; ++i) y[i] = float(state6[i]);
    kn_rhs(k, y, float(energy), d, r, vr);
    for (int i = 0; i < 7; ++i) out7[i] = d[i];
  } else {
    double r, vr;
    kn_rhs(ls.kn, state6, energy, out7, r, vr);
  }
  return GLC_OK;
}

glc_status glc_create(int32_t device, glc_ctx** out) {
  if (!out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return set_error(GLC_ERR_NO_DEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= count) return set_error(GLC_ERR_INVALID_ARGUMENT, "device index out of range");
  DeviceGuard g(device);
  glc_ctx* ctx = new glc_ctx();
  ctx->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete ctx;
    return set_error(GLC_ERR_CUDA, "cudaGetDeviceProperties failed");
  }
  ctx->sm_count = prop.multiProcessorCount;
  ctx->stats.sm_count = unsigned(prop.multiProcessorCount);
  glc_policy_default(2, GLC_MIXED, &ctx->policy);
  if (cudaMalloc(&ctx->d_queue, 256) != cudaSuccess || cudaEventCreateWithFlags(&ctx->stage_free, cudaEventDisableTiming) != cudaSuccess) {
    if (ctx->d_queue) cudaFree(ctx->d_queue);
    delete ctx;
    return set_error(GLC_ERR_CUDA, "context allocation failed");
  }
  *out = ctx;
  return GLC_OK;
}

glc_status glc_destroy(glc_ctx* ctx) {
  if (!ctx) return GLC_OK;
  DeviceGuard g(ctx->device);
  if (ctx->stage_pending) cudaEventSynchronize(ctx->stage_free);
  if (ctx->d_job) cudaFree(ctx->d_job);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->d_queue) cudaFree(ctx->d_queue);
  if (ctx->d_cert) cudaFree(ctx->d_cert);
  if (ctx->d_emap) cudaFree(ctx->d_emap);
  if (ctx->d_shadow) cudaFree(ctx->d_shadow);
  if (ctx->d_footprint) cudaFree(ctx->d_footprint);
  if (ctx->d_host_ws) cudaFree(ctx->d_host_ws);
  if (ctx->d_handoff) cudaFree(ctx->d_handoff);
  for (cudaEvent_t e : ctx->host_band)
    if (e) cudaEventDestroy(e);
  if (ctx->host_entry) cudaEventDestroy(ctx->host_entry);
  if (ctx->host_upload) cudaEventDestroy(ctx->host_upload);
  for (cudaStream_t c : ctx->host_compute)
    if (c) cudaStreamDestroy(c);
  if (ctx->host_copy) cudaStreamDestroy(ctx->host_copy);
  if (ctx->stage_free) cudaEventDestroy(ctx->stage_free);
  delete ctx;
  return GLC_OK;
}

glc_status glc_set_policy(glc_ctx* ctx, const glc_policy* policy) {
  if (!ctx || !policy) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  const glc_status s = validate_policy(*policy);
  if (s != GLC_OK) return s;
  ctx->policy = *policy;
  return GLC_OK;
}

glc_status glc_get_policy(const glc_ctx* ctx, glc_policy* out) {
  if (!ctx || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  *out = ctx->policy;
  return GLC_OK;
}

glc_status glc_get_stats(const glc_ctx* ctx, glc_launch_stats* out) {
  if (!ctx || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  *out = ctx->stats;
  return GLC_OK;
}

glc_status glc_result_slots(const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras, int32_t n_cameras,
                            uint64_t* out) {
  if (!out || !cameras || n_cameras <= 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  uint64_t m = 0;
  for (int i = 0; i < n_cameras; ++i) {
    const glc_camera& c = cameras[i];
    uint64_t n = c.kind == GLC_CAMERA_RAYLIST ? c.n_rays : uint64_t(c.width) * c.height;
    m = std::max<uint64_t>(m, c.result_offset + n);
  }
  (void)scenes;
  (void)n_scenes;
  *out = m;
  return GLC_OK;
}

glc_status glc_trace(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                     int32_t n_cameras, const glc_results* out, void* stream) {
  if (!ctx || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(ctx->device);
  JobLayout L;
  glc_status s = validate_job(scenes, n_scenes, cameras, n_cameras, ctx->policy, L);
  if (s != GLC_OK) return s;
  s = ensure_job_capacity(ctx, L.bytes);
  if (s != GLC_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  fill_staging(ctx->h_stage, L, scenes, n_scenes, cameras, n_cameras);
  GLC_CUDA(cudaMemcpyAsync(ctx->d_job, ctx->h_stage, L.bytes, cudaMemcpyHostToDevice, st));
  GLC_CUDA(cudaEventRecord(ctx->stage_free, st));
  ctx->stage_pending = true;
  const unsigned long long tiles = ctx->policy.capture_certificates ? L.cert_begin[n_cameras] : 0ull;
  if (tiles) {
    s = ensure_cert_capacity(&ctx->d_cert, &ctx->d_cert_words, tiles);
    if (s != GLC_OK) return s;
  }
  const unsigned long long nodes = ctx->policy.escape_map ? L.emap_begin[n_cameras] : 0ull;
  if (nodes) {
    s = ensure_cert_capacity(&ctx->d_emap, &ctx->d_emap_words, nodes);
    if (s != GLC_OK) return s;
  }
  if (split_mixed(ctx->policy)) {
    s = ensure_bytes(&ctx->d_handoff, &ctx->d_handoff_bytes, handoff_bytes(L.total));
    if (s != GLC_OK) return s;
  }
  return launch(ctx, job_view(ctx->d_job, L, n_cameras), ctx->policy, *out, st, ctx->d_queue, ctx->d_cert, tiles,
                ctx->d_emap, nodes, ctx->d_handoff);
}

glc_status glc_refine_shadow_edges(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes,
                                   const glc_camera* cameras, int32_t n_cameras, const glc_results* primary,
                                   float* coverage, void* stream) {
  if (!ctx || !primary || !primary->code || !coverage) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(ctx->device);
  JobLayout L;
  glc_status s = validate_job(scenes, n_scenes, cameras, n_cameras, ctx->policy, L);
  if (s != GLC_OK) return s;
  for (int i = 0; i < n_cameras; ++i)
    if (!whole_view(cameras[i]))
      return set_error(GLC_ERR_INVALID_ARGUMENT, "shadow-edge refinement takes whole-view cameras (tile_count {0, 0})");
  s = ensure_job_capacity(ctx, L.bytes);
  if (s != GLC_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  fill_staging(ctx->h_stage, L, scenes, n_scenes, cameras, n_cameras);
  GLC_CUDA(cudaMemcpyAsync(ctx->d_job, ctx->h_stage, L.bytes, cudaMemcpyHostToDevice, st));
  GLC_CUDA(cudaEventRecord(ctx->stage_free, st));
  ctx->stage_pending = true;
  const JobView job = job_view(ctx->d_job, L, n_cameras);
  // edge-list capacity: every pixel of every image camera, plus the counter word
  unsigned long long pixels = 0;
  for (int i = 0; i < n_cameras; ++i)
    if (cameras[i].kind != GLC_CAMERA_RAYLIST) pixels += (unsigned long long)cameras[i].width * cameras[i].height;
  if (pixels == 0) return GLC_OK;
  if (pixels > 0xffffffffull) return set_error(GLC_ERR_CAPACITY, "too many image pixels for one refinement");
  s = ensure_cert_capacity(&ctx->d_shadow, &ctx->d_shadow_words, 2 * pixels + 2);
  if (s != GLC_OK) return s;
  unsigned int* count = ctx->d_shadow;
  unsigned long long* list = reinterpret_cast<unsigned long long*>(ctx->d_shadow + 2);
  GLC_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned int), st));
  const uint4* code = reinterpret_cast<const uint4*>(primary->code);
  for (int i = 0; i < n_cameras; ++i) {
    if (cameras[i].kind == GLC_CAMERA_RAYLIST) continue;
    const unsigned long long np = (unsigned long long)cameras[i].width * cameras[i].height;
    shadow_classify_kernel<<<unsigned((np + 255) / 256), 256, 0, st>>>(job, i, code, coverage, list, count,
                                                                     unsigned(pixels));
    GLC_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 1;
  }
  const glc_policy& pol = ctx->policy;
  const unsigned grid = unsigned(ctx->sm_count) * 8u;
  switch (pol.precision) {
    case GLC_FP32: shadow_refine_kernel<kFP32><<<grid, 128, 0, st>>>(job, pol, list, count, unsigned(pixels), coverage); break;
    case GLC_MIXED: shadow_refine_kernel<kMIXED><<<grid, 128, 0, st>>>(job, pol, list, count, unsigned(pixels), coverage); break;
    default: shadow_refine_kernel<kFP64><<<grid, 128, 0, st>>>(job, pol, list, count, unsigned(pixels), coverage); break;
  }
  GLC_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  return GLC_OK;
}

glc_status glc_surface_footprint(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                                 int32_t n_cameras, int32_t method, const glc_results* primary, glc_footprint* out,
                                 void* stream) {
  if (!ctx || !primary || !primary->code || !out || !cameras) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (method != GLC_FOOTPRINT_QUARTER_PIXEL && method != GLC_FOOTPRINT_TANGENT)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "unknown footprint method");
  if (method == GLC_FOOTPRINT_QUARTER_PIXEL && (!primary->branch || !primary->surface))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "the quarter-pixel footprint reads the primary branch and surface arrays");
  for (int i = 0; i < n_cameras; ++i) {
    if (cameras[i].kind == GLC_CAMERA_RAYLIST)
      return set_error(GLC_ERR_INVALID_ARGUMENT, "surface footprints are defined for image cameras only");
    const double sx = cameras[i].subpixel_x, sy = cameras[i].subpixel_y;
    // footprint.rs:82-86: the centered quarter-pixel stencil must stay inside the pixel
    if (method == GLC_FOOTPRINT_QUARTER_PIXEL && !(sx >= 0.25 && sx <= 0.75 && sy >= 0.25 && sy <= 0.75))
      return set_error(GLC_ERR_INVALID_ARGUMENT, "surface footprint requires subpixel coordinates in [0.25, 0.75]");
  }
  DeviceGuard g(ctx->device);
  JobLayout L;
  glc_status s = validate_job(scenes, n_scenes, cameras, n_cameras, ctx->policy, L);
  if (s != GLC_OK) return s;
  for (int i = 0; i < n_cameras; ++i)
    if (!whole_view(cameras[i]))
      return set_error(GLC_ERR_INVALID_ARGUMENT, "surface footprints take whole-view cameras (tile_count {0, 0})");
  s = ensure_job_capacity(ctx, L.bytes);
  if (s != GLC_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  fill_staging(ctx->h_stage, L, scenes, n_scenes, cameras, n_cameras);
  GLC_CUDA(cudaMemcpyAsync(ctx->d_job, ctx->h_stage, L.bytes, cudaMemcpyHostToDevice, st));
  GLC_CUDA(cudaEventRecord(ctx->stage_free, st));
  ctx->stage_pending = true;
  const JobView job = job_view(ctx->d_job, L, n_cameras);
  unsigned long long pixels = 0;
  for (int i = 0; i < n_cameras; ++i) pixels += (unsigned long long)cameras[i].width * cameras[i].height;
  if (pixels == 0) return GLC_OK;
  if (pixels > 0xffffffffull) return set_error(GLC_ERR_CAPACITY, "too many image pixels for one footprint call");
  s = ensure_cert_capacity(&ctx->d_footprint, &ctx->d_footprint_words, 2 * pixels + 2);
  if (s != GLC_OK) return s;
  unsigned int* count = ctx->d_footprint;
  unsigned long long* list = reinterpret_cast<unsigned long long*>(ctx->d_footprint + 2);
  GLC_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned int), st));
  const uint4* code = reinterpret_cast<const uint4*>(primary->code);
  for (int i = 0; i < n_cameras; ++i) {
    const unsigned long long np = (unsigned long long)cameras[i].width * cameras[i].height;
    footprint_classify_kernel<<<unsigned((np + 255) / 256), 256, 0, st>>>(job, i, code, out, list, count,
                                                                        unsigned(pixels));
    GLC_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 1;
  }
  const glc_policy& pol = ctx->policy;
  const unsigned grid = unsigned(ctx->sm_count) * 8u;
  const unsigned cap = unsigned(pixels);
  if (method == GLC_FOOTPRINT_QUARTER_PIXEL) {
    const int4* branch = reinterpret_cast<const int4*>(primary->branch);
    const double2* surface = reinterpret_cast<const double2*>(primary->surface);
    switch (pol.precision) {
      case GLC_FP32: footprint_quarter_kernel<kFP32><<<grid, 128, 0, st>>>(job, pol, list, count, cap, code, branch, surface, out); break;
      case GLC_MIXED: footprint_quarter_kernel<kMIXED><<<grid, 128, 0, st>>>(job, pol, list, count, cap, code, branch, surface, out); break;
      default: footprint_quarter_kernel<kFP64><<<grid, 128, 0, st>>>(job, pol, list, count, cap, code, branch, surface, out); break;
    }
  } else {
    switch (pol.precision) {
      case GLC_FP32: footprint_tangent_kernel<kFP32><<<grid, 128, 0, st>>>(job, pol, list, count, cap, out); break;
      case GLC_MIXED: footprint_tangent_kernel<kMIXED><<<grid, 128, 0, st>>>(job, pol, list, count, cap, out); break;
      default: footprint_tangent_kernel<kFP64><<<grid, 128, 0, st>>>(job, pol, list, count, cap, out); break;
    }
  }
  GLC_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches += 1;
  return GLC_OK;
}

glc_status glc_trace_host(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                          int32_t n_cameras, const glc_results* host_out) {
  if (!ctx || !host_out || !cameras || n_cameras <= 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(ctx->device);
  uint64_t slots = 0;
  glc_status s = glc_result_slots(scenes, n_scenes, cameras, n_cameras, &slots);
  if (s != GLC_OK) return s;
  constexpr int kFields = 13;
  void* hfields[kFields] = {host_out->code,    host_out->branch,  host_out->escape,      host_out->surface,
                            host_out->redshift_time, host_out->event, host_out->drift_a, host_out->drift_b,
                            host_out->turning, host_out->position_xy, host_out->position_zr, host_out->intensity,
                            host_out->radiance};
  // bytes per slot of each field (radiance is RGBA16F)
  const size_t esize[kFields] = {16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 8};
  // workspace layout: ray-list states, then one array per requested field
  std::vector<size_t> state_off(size_t(n_cameras), 0);
  size_t bytes = 0;
  for (int i = 0; i < n_cameras; ++i)
    if (cameras[i].kind == GLC_CAMERA_RAYLIST && cameras[i].n_rays > 0) {
      state_off[i] = bytes;
      bytes += align256(cameras[i].n_rays * 8 * sizeof(double));
    }
  size_t field_off[kFields];
  for (int i = 0; i < kFields; ++i) {
    field_off[i] = bytes;
    if (hfields[i]) bytes += align256(slots * esize[i]);
  }
  if (bytes > ctx->d_host_ws_bytes) {
    if (ctx->d_host_ws) GLC_CUDA(cudaFree(ctx->d_host_ws));
    ctx->d_host_ws = nullptr;
    ctx->d_host_ws_bytes = 0;
    GLC_CUDA(cudaMalloc(&ctx->d_host_ws, bytes));
    ctx->d_host_ws_bytes = bytes;
  }
  glc_results dev{};
  void** dfields[kFields] = {(void**)&dev.code,    (void**)&dev.branch,  (void**)&dev.escape,  (void**)&dev.surface,
                             (void**)&dev.redshift_time, (void**)&dev.event, (void**)&dev.drift_a,
                             (void**)&dev.drift_b, (void**)&dev.turning, (void**)&dev.position_xy,
                             (void**)&dev.position_zr, (void**)&dev.intensity, (void**)&dev.radiance};
  for (int i = 0; i < kFields; ++i) *dfields[i] = hfields[i] ? ctx->d_host_ws + field_off[i] : nullptr;
  std::vector<glc_camera> cams(cameras, cameras + n_cameras);

  // One-thread-per-ray launches without the pre-passes are traced in bands on one stream while the
  // finished bands' results are copied back on another, so that the copies overlap the tracing.
  const glc_policy& pol = ctx->policy;
  JobLayout L;
  std::vector<Band> bands;
  const bool banded = pol.persistent == 0 && !pol.capture_certificates && !pol.escape_map &&
                      validate_job(scenes, n_scenes, cameras, n_cameras, pol, L) == GLC_OK &&
                      plan_bands(cameras, n_cameras, L, pol, bands) && bands.size() > 1;
  if (banded) {
    s = ensure_host_streams(ctx);
    if (s != GLC_OK) return s;
    cudaStream_t cs = ctx->host_compute[0], cs2 = ctx->host_compute[1], ps = ctx->host_copy;
    // the banded streams do not synchronize with the legacy default stream; an event recorded there
    // (which completes after all earlier work of blocking streams) orders this call after earlier
    // traces of the context, as the one-launch path on the legacy stream is ordered
    GLC_CUDA(cudaEventRecord(ctx->host_entry, nullptr));
    GLC_CUDA(cudaStreamWaitEvent(cs, ctx->host_entry, 0));
    for (int i = 0; i < n_cameras; ++i) {
      if (cams[i].kind == GLC_CAMERA_RAYLIST && cams[i].n_rays > 0) {
        unsigned char* d = ctx->d_host_ws + state_off[i];
        GLC_CUDA(cudaMemcpyAsync(d, cameras[i].ray_states, cams[i].n_rays * 8 * sizeof(double),
                                 cudaMemcpyHostToDevice, cs));
        cams[i].ray_states = reinterpret_cast<const double*>(d);
      }
    }
    s = ensure_job_capacity(ctx, L.bytes);
    if (s != GLC_OK) return s;
    const bool split = split_mixed(pol);
    if (split) {
      s = ensure_bytes(&ctx->d_handoff, &ctx->d_handoff_bytes, handoff_bytes(L.total));
      if (s != GLC_OK) return s;
    }
    fill_staging(ctx->h_stage, L, scenes, n_scenes, cams.data(), n_cameras);
    GLC_CUDA(cudaMemcpyAsync(ctx->d_job, ctx->h_stage, L.bytes, cudaMemcpyHostToDevice, cs));
    GLC_CUDA(cudaEventRecord(ctx->stage_free, cs));
    ctx->stage_pending = true;
    // bands alternate between two streams, so that one band's last warps overlap the next band
    GLC_CUDA(cudaEventRecord(ctx->host_upload, cs));
    GLC_CUDA(cudaStreamWaitEvent(cs2, ctx->host_upload, 0));
    const JobView job = job_view(ctx->d_job, L, n_cameras);
    for (size_t k = 0; k < bands.size(); ++k) {
      cudaStream_t bs = (k & 1u) ? cs2 : cs;
      if (split) {
        launch_band_split(job, pol, dev, bands[k], bs, ctx->d_handoff);
        ctx->stats.kernel_launches += 1;
      } else {
        switch (pol.precision) {
          case GLC_FP32: launch_band<kFP32>(job, pol, dev, bands[k], bs); break;
          case GLC_MIXED: launch_band<kMIXED>(job, pol, dev, bands[k], bs); break;
          default: launch_band<kFP64>(job, pol, dev, bands[k], bs); break;
        }
      }
      GLC_CUDA(cudaGetLastError());
      GLC_CUDA(cudaEventRecord(ctx->host_band[k], bs));
      ctx->stats.kernel_launches += 1;
    }
    for (size_t k = 0; k < bands.size(); ++k) {
      GLC_CUDA(cudaStreamWaitEvent(ps, ctx->host_band[k], 0));
      const Band& b = bands[k];
      for (int i = 0; i < kFields; ++i) {
        if (!hfields[i]) continue;
        GLC_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(hfields[i]) + b.s0 * esize[i],
                                 static_cast<unsigned char*>(*dfields[i]) + b.s0 * esize[i], (b.s1 - b.s0) * esize[i],
                                 cudaMemcpyDeviceToHost, ps));
      }
    }
    ctx->stats.last_block = pol.block_threads;
    ctx->stats.last_persistent = 0;
    ctx->stats.last_rays = L.total;
    GLC_CUDA(cudaStreamSynchronize(ps));
    GLC_CUDA(cudaStreamSynchronize(cs));
    GLC_CUDA(cudaStreamSynchronize(cs2));
    return GLC_OK;
  }

  for (int i = 0; i < n_cameras; ++i) {
    if (cams[i].kind == GLC_CAMERA_RAYLIST && cams[i].n_rays > 0) {
      unsigned char* d = ctx->d_host_ws + state_off[i];
      GLC_CUDA(cudaMemcpyAsync(d, cameras[i].ray_states, cams[i].n_rays * 8 * sizeof(double), cudaMemcpyHostToDevice,
                               nullptr));
      cams[i].ray_states = reinterpret_cast<const double*>(d);
    }
  }
  s = glc_trace(ctx, scenes, n_scenes, cams.data(), n_cameras, &dev, nullptr);
  if (s != GLC_OK) return s;
  bool regions = false;
  for (int i = 0; i < n_cameras; ++i) regions = regions || !whole_view(cams[i]);
  for (int i = 0; i < kFields; ++i) {
    if (!hfields[i]) continue;
    if (!regions) {
      GLC_CUDA(cudaMemcpyAsync(hfields[i], *dfields[i], slots * esize[i], cudaMemcpyDeviceToHost, nullptr));
      continue;
    }
    // tile regions: copy back each camera's traced pixels only (the rest of the host arrays, which
    // other batches fill, is left as it is)
    for (int c = 0; c < n_cameras; ++c) {
      const glc_camera& cm = cams[c];
      unsigned char* h = static_cast<unsigned char*>(hfields[i]);
      const unsigned char* d = static_cast<const unsigned char*>(*dfields[i]);
      if (cm.kind == GLC_CAMERA_RAYLIST) {
        const size_t off = cm.result_offset * esize[i];
        if (cm.n_rays) GLC_CUDA(cudaMemcpyAsync(h + off, d + off, cm.n_rays * esize[i], cudaMemcpyDeviceToHost, nullptr));
        continue;
      }
      const PixelRect rc = camera_rect(cm);
      const size_t pitch = size_t(cm.width) * esize[i];
      const size_t off = (cm.result_offset + size_t(rc.y0) * cm.width + rc.x0) * esize[i];
      GLC_CUDA(cudaMemcpy2DAsync(h + off, pitch, d + off, pitch, size_t(rc.x1 - rc.x0) * esize[i], rc.y1 - rc.y0,
                                 cudaMemcpyDeviceToHost, nullptr));
    }
  }
  GLC_CUDA(cudaStreamSynchronize(nullptr));
  return GLC_OK;
}

glc_status glc_graph_capture(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                             int32_t n_cameras, const glc_results* out, void* stream, glc_graph** graph) {
  if (!ctx || !out || !graph) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (!stream) return set_error(GLC_ERR_INVALID_ARGUMENT, "graph capture needs a non-default stream");
  *graph = nullptr;
  DeviceGuard g(ctx->device);
  JobLayout L;
  glc_status s = validate_job(scenes, n_scenes, cameras, n_cameras, ctx->policy, L);
  if (s != GLC_OK) return s;
  glc_graph* G = new glc_graph();
  G->ctx = ctx;
  auto fail = [&](glc_status st) {
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    if (G->d_job) cudaFree(G->d_job);
    if (G->h_stage) cudaFreeHost(G->h_stage);
    if (G->d_queue) cudaFree(G->d_queue);
    if (G->d_cert) cudaFree(G->d_cert);
    if (G->d_emap) cudaFree(G->d_emap);
    if (G->d_handoff) cudaFree(G->d_handoff);
    delete G;
    return st;
  };
  const unsigned long long tiles = ctx->policy.capture_certificates ? L.cert_begin[n_cameras] : 0ull;
  const unsigned long long nodes = ctx->policy.escape_map ? L.emap_begin[n_cameras] : 0ull;
  if (cudaMalloc(&G->d_job, L.bytes) != cudaSuccess || cudaMallocHost(&G->h_stage, L.bytes) != cudaSuccess ||
      cudaMalloc(&G->d_queue, 256) != cudaSuccess ||
      (tiles && cudaMalloc(&G->d_cert, tiles * sizeof(uint32_t)) != cudaSuccess) ||
      (nodes && cudaMalloc(&G->d_emap, nodes * sizeof(uint32_t)) != cudaSuccess) ||
      (split_mixed(ctx->policy) && cudaMalloc(&G->d_handoff, handoff_bytes(L.total)) != cudaSuccess))
    return fail(set_error(GLC_ERR_CUDA, "graph buffer allocation failed"));
  fill_staging(G->h_stage, L, scenes, n_scenes, cameras, n_cameras);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return fail(set_error(GLC_ERR_CUDA, "cudaStreamBeginCapture failed"));
  cudaError_t ce = cudaMemcpyAsync(G->d_job, G->h_stage, L.bytes, cudaMemcpyHostToDevice, st);
  glc_status ls = ce == cudaSuccess ? launch(ctx, job_view(G->d_job, L, n_cameras), ctx->policy, *out, st, G->d_queue,
                                           G->d_cert, tiles, G->d_emap, nodes, G->d_handoff)
                                    : set_error(GLC_ERR_CUDA, cudaGetErrorString(ce));
  cudaGraph_t gr = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(st, &gr);
  if (ls != GLC_OK) {
    if (gr) cudaGraphDestroy(gr);
    return fail(ls);
  }
  if (ee != cudaSuccess) return fail(set_error(GLC_ERR_CUDA, cudaGetErrorString(ee)));
  G->graph = gr;
  if (cudaGraphInstantiate(&G->exec, gr, 0) != cudaSuccess)
    return fail(set_error(GLC_ERR_CUDA, "cudaGraphInstantiate failed"));
  *graph = G;
  return GLC_OK;
}

glc_status glc_graph_launch(glc_graph* graph, void* stream) {
  if (!graph) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(graph->ctx->device);
  GLC_CUDA(cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream)));
  graph->ctx->stats.kernel_launches += 1;
  return GLC_OK;
}

glc_status glc_graph_destroy(glc_graph* graph) {
  if (!graph) return GLC_OK;
  DeviceGuard g(graph->ctx->device);
  cudaDeviceSynchronize();
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  if (graph->d_job) cudaFree(graph->d_job);
  if (graph->h_stage) cudaFreeHost(graph->h_stage);
  if (graph->d_queue) cudaFree(graph->d_queue);
  if (graph->d_cert) cudaFree(graph->d_cert);
  if (graph->d_emap) cudaFree(graph->d_emap);
  if (graph->d_handoff) cudaFree(graph->d_handoff);
  delete graph;
  return GLC_OK;
}

glc_status glc_autotune(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                        int32_t n_cameras, const glc_results* out, void* stream, int32_t repeats, glc_policy* policy) {
  if (!ctx || !out || !policy) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  DeviceGuard g(ctx->device);
  if (repeats < 1) repeats = 1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  GLC_CUDA(cudaEventCreate(&e0));
  GLC_CUDA(cudaEventCreate(&e1));
  const glc_policy saved = ctx->policy;
  glc_policy best = *policy;
  float best_ms = std::numeric_limits<float>::infinity();
  auto time_policy = [&](const glc_policy& cand, float& ms) -> glc_status {
    glc_status s = validate_policy(cand);
    if (s != GLC_OK) return s;
    ctx->policy = cand;
    s = glc_trace(ctx, scenes, n_scenes, cameras, n_cameras, out, stream);  // warm-up
    if (s != GLC_OK) return s;
    GLC_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < repeats; ++r) {
      s = glc_trace(ctx, scenes, n_scenes, cameras, n_cameras, out, stream);
      if (s != GLC_OK) return s;
    }
    GLC_CUDA(cudaEventRecord(e1, st));
    GLC_CUDA(cudaEventSynchronize(e1));
    GLC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    ms /= float(repeats);
    return GLC_OK;
  };
  // coordinate descent over the launch-shape knobs, starting from the caller's policy
  struct Knob {
    int which;
    std::vector<uint32_t> values;
  };
  const std::vector<std::pair<uint32_t, uint32_t>> tiles = {{8, 4}, {16, 2}, {32, 1}, {4, 8}, {8, 8}, {16, 16}};
  const std::vector<Knob> knobs = {
      {0, {0, 1, 2}},          // one thread per ray / lane-refill work queue / warp-grab work queue
      {1, {64, 96, 128}},      // block threads
      {2, {0, 1, 2, 3, 4, 5}}, // tile index
      {3, {32, 64, 128, 256}}, // rays per grab
      {4, {1, 4, 8, 16, 32}},  // refill interval
      {5, {1, 8, 16, 24, 32}}, // idle lanes that trigger a refill
  };
  glc_status s = time_policy(best, best_ms);
  for (int pass = 0; pass < 2 && s == GLC_OK; ++pass) {
    for (const Knob& k : knobs) {
      for (uint32_t v : k.values) {
        glc_policy cand = best;
        switch (k.which) {
          case 0: cand.persistent = v; break;
          case 1: cand.block_threads = v; break;
          case 2: cand.tile_w = tiles[v].first; cand.tile_h = tiles[v].second; break;
          case 3: cand.rays_per_grab = v; break;
          case 4: cand.refill_interval = v; break;
          case 5: cand.refill_min_idle = v; break;
        }
        if (!cand.persistent && k.which >= 3) continue;
        if (cand.persistent == 2 && k.which >= 4) continue;  // no lane refill in the warp-grab queue
        float ms = 0.0f;
        s = time_policy(cand, ms);
        if (s != GLC_OK) break;
        if (ms < best_ms) {
          best_ms = ms;
          best = cand;
        }
      }
      if (s != GLC_OK) break;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != GLC_OK) {
    ctx->policy = saved;
    return s;
  }
  ctx->policy = best;
  *policy = best;
  return GLC_OK;
}

}  // extern "C"
