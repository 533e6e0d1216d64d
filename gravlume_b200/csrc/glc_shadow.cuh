// Shadow-edge coverage refinement (crates/gravlume-render/src/shaders/shadow_coverage.wgsl:63-136):
// pixels of an image camera that ended in capture or escape and touch a 4-neighbour of the other
// class are re-traced with four rotated-grid subpixel samples; their coverage is the fraction of
// escaping samples.
#pragma once

#include "glc_kernels.cuh"

namespace glc {

// rotated-grid subpixel offsets of the four samples (shadow_coverage.wgsl:19-27)
__device__ __forceinline__ void shadow_sample_offset(int k, double& sx, double& sy) {
  const double ox[4] = {0.375, 0.875, 0.625, 0.125}, oy[4] = {0.125, 0.375, 0.875, 0.625};
  sx = ox[k];
  sy = oy[k];
}

__device__ __forceinline__ int shadow_branch(const uint4* code, unsigned long long slot) {
  const uint32_t t = code[slot].x & 0xFFu;
  return t == GLC_TERM_HORIZON ? 0 : (t == GLC_TERM_ESCAPE ? 1 : -1);
}

// One thread per pixel of camera `c`: primary coverage (1 escape, 0 capture, -1 otherwise) and the
// list of edge pixels (camera << 32 | pixel index) behind an atomic counter.
__global__ void shadow_classify_kernel(JobView job, int c, const uint4* code, float* coverage,
                                       unsigned long long* list, unsigned int* count, unsigned int capacity) {
  const glc_camera& cam = job.cams[c];
  const uint32_t W = cam.width, H = cam.height;
  const unsigned long long p = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (unsigned long long)W * H) return;
  const uint32_t px = uint32_t(p % W), py = uint32_t(p / W);
  const unsigned long long base = cam.result_offset;
  const int center = shadow_branch(code, base + p);
  coverage[base + p] = float(center);
  if (center < 0) return;
  const int other = 1 - center;
  bool edge = false;
  if (px > 0) edge = edge || shadow_branch(code, base + p - 1) == other;
  if (px + 1 < W) edge = edge || shadow_branch(code, base + p + 1) == other;
  if (py > 0) edge = edge || shadow_branch(code, base + p - W) == other;
  if (py + 1 < H) edge = edge || shadow_branch(code, base + p + W) == other;
  if (!edge) return;
  const unsigned int k = atomicAdd(count, 1u);
  if (k < capacity) list[k] = ((unsigned long long)c << 32) | p;
}

// Four lanes per edge pixel (one subpixel sample each), grid-stride over the device-side list. The
// stride loop runs on the warp-uniform base index, so that all 32 lanes reach the shuffles that
// add up each pixel's four samples; lanes past the list's end contribute nothing.
template <int P>
__global__ void __launch_bounds__(128, LaunchShape<P>::kMinBlocks) shadow_refine_kernel(
    JobView job, glc_policy pol, const unsigned long long* list, const unsigned int* count, unsigned int capacity,
    float* coverage) {
  using S = typename PrecTraits<P>::S;
  const unsigned FULL = 0xffffffffu;
  const unsigned int n = min(*count, capacity);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < 4ull * n;
       base += stride) {
    const unsigned long long t = base + lane;
    const int k = int(t & 3u);
    unsigned esc = 0u, bad = 0u;
    glc_camera cam;
    unsigned long long p = 0;
    if (t < 4ull * n) {
      const unsigned long long entry = list[t >> 2];
      cam = job.cams[entry >> 32];
      p = entry & 0xffffffffull;
      const uint32_t px = uint32_t(p % cam.width), py = uint32_t(p / cam.width);
      shadow_sample_offset(k, cam.subpixel_x, cam.subpixel_y);
      const glc_scene& sc = job.scenes[cam.scene_index];
      double st8[8];
      image_state(&sc, &cam, px, py, st8);
      const LaneScene ls = make_lane_scene(sc, pol.mixed_shell_factor, pol.uncertain_terminals != 0u);  // drifts only for the Uncertain gate
      Ray<P> ray;
      ray.init(ls, pol, st8, -1.0);
      RayResult<S> res;
      for (;;) {
        bool use64 = false;
        if (P == kMIXED) use64 = __any_sync(__activemask(), double(ray.r) < ls.shell_r);
        if (ray_step<P>(ray, ls, pol, res, use64)) break;
      }
      esc = res.termination == GLC_TERM_ESCAPE ? 1u : 0u;
      bad = (res.termination != GLC_TERM_ESCAPE && res.termination != GLC_TERM_HORIZON) ? 1u : 0u;
    }
    __syncwarp(FULL);
    esc += __shfl_xor_sync(FULL, esc, 1);
    bad += __shfl_xor_sync(FULL, bad, 1);
    esc += __shfl_xor_sync(FULL, esc, 2);
    bad += __shfl_xor_sync(FULL, bad, 2);
    // an edge pixel with a sample that neither escaped nor was captured keeps its primary coverage
    if (t < 4ull * n && k == 0 && bad == 0u) coverage[cam.result_offset + p] = 0.25f * float(esc);
  }
}

}  // namespace glc
