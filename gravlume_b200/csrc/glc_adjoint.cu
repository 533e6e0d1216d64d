// Discrete adjoint over the C ABI: glc_forward_ckpt (trace with per-ray checkpoints every K accepted
// steps) and glc_backward (segment replay and reverse sweeps). The per-step algebra is in
// glc_adjoint.cuh; this file holds the kernels, the tape and the host-side scene derivatives.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "glc_adjoint.cuh"
#include "glc_context.h"
#include "glc_internal.h"
#include "glc_kernels.cuh"

using namespace glc;

namespace {

template <int P>
struct RayWords {
  static_assert(std::is_trivially_copyable<Ray<P>>::value, "checkpointed rays are copied bytewise");
  static constexpr int kWords = int((sizeof(Ray<P>) + 15) / 16);
};

// One attempt with the per-ray shell decision, compiled once so that the forward pass and every
// backward replay run the identical instruction sequence (bitwise-identical step sequences).
template <int P>
__device__ __noinline__ bool adjoint_step(Ray<P>& ray, const LaneScene& ls, const glc_policy& pol,
                                          RayResult<typename PrecTraits<P>::S>& res) {
  const bool use64 = P == kMIXED && double(ray.r) < ls.shell_r;
  return ray.step(ls, pol, res, use64);
}

// Checkpoint storage: the ray object as 16-byte words. The first `cap` checkpoints of every ray
// sit in the dense region, word-major across rays (coalesced); a ray that takes more keeps the rest
// in the overflow pool, contiguously from its own base slot (sized by the rays' actual counts).
struct CkptStore {
  uint4* dense;
  uint4* pool;
  uint32_t cap;
  unsigned long long n;
};

template <int P>
__device__ __forceinline__ uint4* ckpt_word(const CkptStore& cs, uint32_t c, uint32_t base, unsigned long long gi,
                                            int w) {
  constexpr int W = RayWords<P>::kWords;
  if (c < cs.cap) return cs.dense + ((unsigned long long)c * W + w) * cs.n + gi;
  return cs.pool + ((unsigned long long)base + (c - cs.cap)) * W + w;
}

template <int P>
__device__ __forceinline__ void store_ray(const Ray<P>& ray, const CkptStore& cs, uint32_t c, uint32_t base,
                                          unsigned long long gi) {
  constexpr int W = RayWords<P>::kWords;
  uint4 buf[W];
  memcpy(buf, &ray, sizeof(Ray<P>));
#pragma unroll
  for (int w = 0; w < W; ++w) *ckpt_word<P>(cs, c, base, gi, w) = buf[w];
}

template <int P>
__device__ __forceinline__ void load_ray(Ray<P>& ray, const CkptStore& cs, uint32_t c, uint32_t base,
                                         unsigned long long gi) {
  constexpr int W = RayWords<P>::kWords;
  uint4 buf[W];
#pragma unroll
  for (int w = 0; w < W; ++w) buf[w] = *ckpt_word<P>(cs, c, base, gi, w);
  memcpy(&ray, buf, sizeof(Ray<P>));
}

// meta per ray: x checkpoints taken, y termination | status << 8 (status 1 every checkpoint stored,
// 2 waiting for its overflow slots, 0 tile padding), z accepted steps, w base slot in the overflow
// pool. counters: [0] rays over the dense capacity, [1] most accepted steps, [2] replay mismatches,
// [3] degenerate terminal events, [4] overflow slots reserved.
//
// pass 0 traces every ray, stores its first cs.cap checkpoints and reserves overflow slots for the
// rest; pass 1 (only when some ray overflowed, after the pool is sized) traces the overflowing rays
// again, bitwise identically, and stores their remaining checkpoints.
template <int P>
__global__ void __launch_bounds__(128) adjoint_forward_kernel(JobView job, glc_policy pol, glc_results out,
                                                              uint32_t K, CkptStore cs, uint4* meta,
                                                              unsigned int* counters, int pass) {
  using S = typename PrecTraits<P>::S;
  const unsigned long long gi = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= job.total) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx, shortcut;
  double rdir[3];
  uint32_t base = 0;
  if (pass == 1) {
    const uint4 m = meta[gi];
    if ((m.y >> 8) != 2u) return;
    base = m.w;
  }
  if (!ray_setup(job, pol, gi, st8, dir, slot, scene_idx, shortcut, rdir)) {
    meta[gi] = make_uint4(0, 0, 0, 0);
    return;
  }
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor);
  Ray<P> ray;
  RayResult<S> res;
  uint32_t taken = 0;
  if (pass == 0) {
    ray.init(ls, pol, st8, dir);
  } else {
    // resume from the last dense checkpoint (the stepper object at accepted step (cap - 1) K):
    // the same step function from the same object replays pass 0 bit for bit
    load_ray<P>(ray, cs, cs.cap - 1, base, gi);
    taken = cs.cap - 1;
  }
  for (;;) {
    if (ray.accepted == taken * K) {
      if (pass == 0 ? taken < cs.cap : taken >= cs.cap) store_ray<P>(ray, cs, taken, base, gi);
      ++taken;
    }
    if (adjoint_step<P>(ray, ls, pol, res)) break;
  }
  if (pass == 1) {
    meta[gi].y = res.termination | (1u << 8);
    return;
  }
  write_result<P>(out, slot, ray, res, ls);
  const bool over = taken > cs.cap;
  if (over) {
    atomicAdd(counters, 1u);
    base = atomicAdd(counters + 4, taken - cs.cap);
  }
  meta[gi] = make_uint4(taken, res.termination | ((over ? 2u : 1u) << 8), ray.accepted, base);
  atomicMax(counters + 1, ray.accepted);
}

// Adjoint of one ray: replay each checkpointed segment (recording the start state and step size of
// each attempt in the thread's scratch, K entries) and sweep it in reverse, last segment first.
template <int P>
__device__ void adjoint_backward_ray(const JobView& job, const glc_policy& pol, uint32_t K, const CkptStore& cs,
                                     const uint4* meta, double* scratch, unsigned long long stride,
                                     unsigned long long gi, const double* dl, const glc_grads& g,
                                     const double* dconst, double charge, unsigned int* counters) {
  using S = typename PrecTraits<P>::S;
  const unsigned long long n = stride;
  uint4 m = meta[gi];
  const uint32_t status = m.y >> 8;
  m.y &= 0xFFu;
  if (status == 0u) return;
  double st8[8], dir;
  unsigned long long slot;
  int scene_idx, shortcut;
  double rdir[3];
  ray_setup(job, pol, gi, st8, dir, slot, scene_idx, shortcut, rdir);
  const LaneScene ls = make_lane_scene(job.scenes[scene_idx], pol.mixed_shell_factor);
  // the reverse sweep's stage products in the forward pass's stage precision: binary32 after a
  // MIXED forward, binary64 after an FP64 one (stage points and accumulation stay binary64)
  using VR = typename std::conditional<P == kMIXED, float, double>::type;
  const KN<Dual<4, VR>> kd = kn_dual_vjp<VR>(ls.kn);
  double wobs[kObs];
  bool any = false;
  for (int k = 0; k < kObs; ++k) {
    wobs[k] = dl[slot * kObs + k];
    any = any || wobs[k] != 0.0;
  }
  double lam[6] = {0, 0, 0, 0, 0, 0}, gacc[3] = {0, 0, 0};
  const bool differentiable = status == 1u && (m.y == GLC_TERM_SURFACE || m.y == GLC_TERM_ESCAPE);
  bool ok = differentiable && any && scratch != nullptr;
  bool degenerate = false;
  double wst[7];
  step_weights(wst);
  for (int c = int(m.x) - 1; ok && c >= 0; --c) {
    Ray<P> ray;
    load_ray<P>(ray, cs, uint32_t(c), m.w, gi);
    RayResult<S> res;
    uint32_t j = 0;
    bool term = false;
    for (;;) {
      if (j >= K) {
        ok = false;
        break;
      }
      double* rec = scratch + (unsigned long long)j * 7 * n;
      for (int q = 0; q < 6; ++q) rec[q * n] = double(ray.ys(q));
      rec[6 * n] = double(ray.h);
      const uint32_t acc = ray.accepted;
      if (adjoint_step<P>(ray, ls, pol, res)) {
        term = true;
        break;
      }
      if (ray.accepted != acc) {
        ++j;
        if (ray.accepted == (uint32_t(c) + 1u) * K) break;
      }
    }
    if (!ok) break;
    const double E = double(ray.E);
    if (c == int(m.x) - 1) {
      // the replay must end where the forward pass ended
      if (!term || res.termination != m.y || ray.accepted != m.z) {
        ok = false;
        break;
      }
      const double* rec = scratch + (unsigned long long)j * 7 * n;
      double y0[6];
      for (int q = 0; q < 6; ++q) y0[q] = rec[q * n];
      if (!terminal_reverse(ls, y0, E, rec[6 * n], double(res.event_theta), double(ray.dir), m.y, wobs, lam, gacc)) {
        ok = false;
        degenerate = true;
        break;
      }
    } else if (term) {
      ok = false;
      break;
    }
    for (int jj = int(j) - 1; jj >= 0; --jj) {
      const double* rec = scratch + (unsigned long long)jj * 7 * n;
      double y0[6], l0[6];
      for (int q = 0; q < 6; ++q) y0[q] = rec[q * n];
      dp5_reverse(ls.kn, kd, y0, E, rec[6 * n], wst, lam, l0, gacc);
      for (int q = 0; q < 6; ++q) lam[q] = l0[q];
    }
  }
  if (!ok) {
    for (int q = 0; q < 6; ++q) lam[q] = 0.0;
    gacc[0] = gacc[1] = gacc[2] = 0.0;
    if (differentiable && any) atomicAdd(counters + (degenerate ? 3 : 2), 1u);
  }
  // dL/dp_t = -dL/dE (E = -p_t)
  const double gpt = -gacc[0];
  if (g.ray_momentum) {
    double2* rm = reinterpret_cast<double2*>(g.ray_momentum + 4 * slot);
    rm[0] = make_double2(gpt, lam[3]);
    rm[1] = make_double2(lam[4], lam[5]);
  }
  double pg[4] = {gacc[1], 2.0 * charge * gacc[2], 0.0, 0.0};
  const glc_camera& cam = job.cams[0];
  if (ok && dconst && cam.kind == GLC_CAMERA_PINHOLE) {
    // the initial state's dependence on (a, Q, inclination, r_obs) through the observer's tetrad
    const glc_scene& sc = job.scenes[scene_idx];
    double cv[kSceneConsts];
    gather_scene_consts(sc, cv);
    Dual<4> cd[kSceneConsts];
    for (int i = 0; i < kSceneConsts; ++i) {
      cd[i] = Dual<4>(cv[i]);
      for (int k = 0; k < 4; ++k) cd[i].d[k] = dconst[k * kSceneConsts + i];
    }
    const unsigned long long pix = slot - cam.result_offset;
    const double px = double(pix % cam.width) + cam.subpixel_x, py = double(pix / cam.width) + cam.subpixel_y;
    Dual<4> ds[8];
    pinhole_state(cd, px, py, double(cam.width), double(cam.height), ds);
    const double ls8[8] = {0.0, lam[0], lam[1], lam[2], gpt, lam[3], lam[4], lam[5]};
    for (int i = 0; i < 8; ++i)
      for (int k = 0; k < 4; ++k) pg[k] += ls8[i] * ds[i].d[k];
  }
  if (g.ray_params) {
    double2* rp = reinterpret_cast<double2*>(g.ray_params + 4 * slot);
    rp[0] = make_double2(pg[0], pg[1]);
    rp[1] = make_double2(pg[2], pg[3]);
  }
  if (g.params && ok)
    for (int k = 0; k < 4; ++k)
      if (pg[k] != 0.0) atomicAdd(g.params + k, pg[k]);
}

// One thread per ray. The replay scratch (K attempts of 7 doubles per thread) is not per ray: a
// block borrows one of n_slots scratch slots (busy flags, one per slot) for its lifetime, and
// there are as many slots as blocks that can be resident at once, so the scratch is bounded by the
// GPU's residency, not by the ray count. A block starts only once another has left, and a block
// frees its slot before it leaves, so a starting block always finds a free slot; the search is
// bounded (four rounds over the flags, long enough for a release still in flight to land), and
// should it ever fail, the block's rays get zero gradients and counters[6] records it.
template <int P>
__global__ void __launch_bounds__(128) adjoint_backward_kernel(JobView job, glc_policy pol, uint32_t K, CkptStore cs,
                                                               const uint4* meta, double* scratch, unsigned int* busy,
                                                               unsigned int n_slots, const double* dl, glc_grads g,
                                                               const double* dconst, double charge,
                                                               unsigned int* counters) {
  __shared__ unsigned int slot_s;
  if (threadIdx.x == 0) {
    unsigned int s = blockIdx.x % n_slots, found = n_slots;
    for (unsigned int it = 0; it < 4u * n_slots; ++it) {
      if (atomicCAS(busy + s, 0u, 1u) == 0u) {
        found = s;
        break;
      }
      s = s + 1u == n_slots ? 0u : s + 1u;
    }
    if (found == n_slots) atomicAdd(counters + 6, 1u);
    slot_s = found;
  }
  __syncthreads();
  const unsigned int slot = slot_s;
  const unsigned long long stride = (unsigned long long)n_slots * blockDim.x;
  double* mine = slot < n_slots ? scratch + (unsigned long long)slot * blockDim.x + threadIdx.x : nullptr;
  const unsigned long long gi = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gi < job.total) adjoint_backward_ray<P>(job, pol, K, cs, meta, mine, stride, gi, dl, g, dconst, charge, counters);
  __syncthreads();
  if (threadIdx.x == 0 && slot < n_slots) {
    __threadfence();
    atomicExch(busy + slot, 0u);
  }
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

void oblate_position(double spin, int chart, double r, double polar, double azimuth, double out[4]) {
  // KerrNewmanSpacetime::oblate_to_cartesian (crates/gravlume-domain/src/spacetime.rs:245-254)
  const double st = std::sin(polar), ct = std::cos(polar), sp = std::sin(azimuth), cp = std::cos(azimuth);
  const double cs = (chart == GLC_CHART_INGOING ? 1.0 : -1.0) * spin;
  out[0] = 0.0;
  out[1] = (cs * -sp + r * cp) * st;
  out[2] = (cs * cp + r * sp) * st;
  out[3] = r * ct;
}

// p = (a, Q, inclination, r_obs)
glc_status pack_adjoint_scene(const glc_adjoint_scene& as, const double p[4], glc_scene& out) {
  glc_scene_input in = as.input;
  in.spin = p[0];
  in.charge = p[1];
  oblate_position(p[0], in.chart, p[3], p[2], as.observer_azimuth, in.observer_txyz);
  return pack_scene(in, out);
}

}  // namespace

struct glc_tape {
  glc_ctx* ctx = nullptr;
  glc_policy pol{};
  glc_camera cam{};
  uint32_t K = 0, cap = 0, words = 0;
  unsigned long long n = 0;
  double charge = 0.0;
  unsigned char* d_job = nullptr;
  size_t off_cams = 0, off_begin = 0, off_cert = 0;
  uint4* d_ckpt = nullptr;              // dense checkpoints: cap per ray, word-major across rays
  size_t ckpt_bytes = 0, ckpt_alloc = 0;
  uint4* d_pool = nullptr;              // overflow checkpoints, sized by the rays' actual counts
  size_t pool_bytes = 0, pool_alloc = 0;
  uint4* d_meta = nullptr;
  unsigned long long meta_alloc = 0;
  double* d_dconst = nullptr;
  double* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  unsigned int* d_counters = nullptr;
  unsigned int* d_busy = nullptr;       // backward scratch slots in use (one flag per slot)
  unsigned int busy_slots = 0;
  bool pinhole = false;
  bool valid = false;  // the last forward pass into the tape completed (backward needs it)

  JobView job() const {
    JobView v;
    v.scenes = reinterpret_cast<const glc_scene*>(d_job);
    v.cams = reinterpret_cast<const glc_camera*>(d_job + off_cams);
    v.begin = reinterpret_cast<const unsigned long long*>(d_job + off_begin);
    v.cert_begin = reinterpret_cast<const unsigned long long*>(d_job + off_cert);
    v.cert = nullptr;
    v.emap_begin = nullptr;
    v.emap = nullptr;
    v.n_cams = 1;
    v.total = n;
    return v;
  }
};

namespace {

void free_tape(glc_tape* t) {
  if (!t) return;
  if (t->d_job) cudaFree(t->d_job);
  if (t->d_ckpt) cudaFree(t->d_ckpt);
  if (t->d_pool) cudaFree(t->d_pool);
  if (t->d_meta) cudaFree(t->d_meta);
  if (t->d_dconst) cudaFree(t->d_dconst);
  if (t->d_scratch) cudaFree(t->d_scratch);
  if (t->d_counters) cudaFree(t->d_counters);
  if (t->d_busy) cudaFree(t->d_busy);
  delete t;
}

glc_status cuda_status(cudaError_t e) {
  return e == cudaSuccess ? GLC_OK : set_error(GLC_ERR_CUDA, cudaGetErrorString(e));
}

constexpr int kCounters = 8;

CkptStore ckpt_store(const glc_tape* t) { return CkptStore{t->d_ckpt, t->d_pool, t->cap, t->n}; }

template <int P>
glc_status run_forward(glc_tape* t, const glc_results& out, cudaStream_t st, int pass) {
  const unsigned grid = unsigned((t->n + 127) / 128);
  glc_status s = GLC_OK;
  if (pass == 0) s = cuda_status(cudaMemsetAsync(t->d_counters, 0, kCounters * sizeof(unsigned int), st));
  if (s != GLC_OK) return s;
  adjoint_forward_kernel<P><<<grid, 128, 0, st>>>(t->job(), t->pol, out, t->K, ckpt_store(t), t->d_meta,
                                                   t->d_counters, pass);
  s = cuda_status(cudaGetLastError());
  if (s == GLC_OK) t->ctx->stats.kernel_launches += 1;
  return s;
}

glc_status forward(glc_tape* t, const glc_results& out, cudaStream_t st, int pass) {
  return t->pol.precision == GLC_MIXED ? run_forward<kMIXED>(t, out, st, pass) : run_forward<kFP64>(t, out, st, pass);
}

// A grow-only device buffer of the tape (a reused tape keeps its memory).
glc_status grow(uint4** buf, size_t* alloc, size_t need) {
  if (need <= *alloc) return GLC_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *alloc = 0;
  const glc_status s = cuda_status(cudaMalloc(buf, need));
  if (s == GLC_OK) *alloc = need;
  return s;
}

// Dense checkpoint slots for every ray: the checkpoints of the first 64 accepted steps (every ray
// takes at least its initial one); the rest go to the overflow pool.
glc_status size_checkpoints(glc_tape* t) {
  t->cap = 64 / t->K + 1;
  t->ckpt_bytes = size_t(t->cap) * t->words * 16 * t->n;
  return grow(&t->d_ckpt, &t->ckpt_alloc, t->ckpt_bytes);
}

struct DeviceScope {
  int prev = -1, want = 0;
  explicit DeviceScope(int dev) : want(dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (prev >= 0 && prev != want) cudaSetDevice(prev);
  }
};

// Validates the request and runs the forward pass into t (a new tape, or one being reused: its
// buffers are kept and grown only where this request needs more).
glc_status fill_tape(glc_tape* t, glc_ctx* ctx, const glc_adjoint_scene* as, const glc_camera* camera, int32_t K,
                     const glc_results* out, void* stream) {
  if (K < 1) return set_error(GLC_ERR_INVALID_ARGUMENT, "checkpoint interval K must be at least 1");
  const glc_policy pol = ctx->policy;
  if (pol.precision != GLC_MIXED && pol.precision != GLC_FP64)
    return set_error(GLC_ERR_UNSUPPORTED, "the adjoint runs in MIXED or FP64 precision");
  if (camera->kind != GLC_CAMERA_PINHOLE && camera->kind != GLC_CAMERA_RAYLIST)
    return set_error(GLC_ERR_UNSUPPORTED, "the adjoint takes a pinhole or ray-list camera");
  if (camera->scene_index != 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "camera must use scene 0");
  if (camera->tile_count[0] != 0u || camera->tile_count[1] != 0u)
    return set_error(GLC_ERR_INVALID_ARGUMENT, "the adjoint takes a whole-view camera (tile_count {0, 0})");
  if (!(as->observer_radius > 0.0) || !std::isfinite(as->observer_polar) || !std::isfinite(as->observer_azimuth))
    return set_error(GLC_ERR_INVALID_ARGUMENT, "observer oblate coordinates must be finite, radius positive");
  const double p0[4] = {as->input.spin, as->input.charge, as->observer_polar, as->observer_radius};
  glc_scene scene;
  glc_status s = pack_adjoint_scene(*as, p0, scene);
  if (s != GLC_OK) return s;
  unsigned long long n = 0;
  if (camera->kind == GLC_CAMERA_PINHOLE) {
    if (camera->width != scene.width || camera->height != scene.height)
      return set_error(GLC_ERR_INVALID_ARGUMENT, "pinhole camera size must match the scene's view");
    if (pol.tile_w == 0 || pol.tile_h == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "tile shape must be nonzero");
    const unsigned long long tx = (camera->width + pol.tile_w - 1) / pol.tile_w;
    const unsigned long long ty = (camera->height + pol.tile_h - 1) / pol.tile_h;
    n = tx * ty * pol.tile_w * pol.tile_h;
  } else {
    if (!camera->ray_states || (reinterpret_cast<uintptr_t>(camera->ray_states) & 15u) != 0)
      return set_error(GLC_ERR_INVALID_ARGUMENT, "ray states must be a 16-byte aligned device array");
    if (!(camera->affine_direction == 1.0 || camera->affine_direction == -1.0))
      return set_error(GLC_ERR_INVALID_ARGUMENT, "affine direction must be +1 or -1");
    n = camera->n_rays;
  }
  if (n == 0) return set_error(GLC_ERR_INVALID_ARGUMENT, "no rays");

  // scene-constant derivatives with respect to (a, Q, inclination, r_obs): central differences of
  // the host scene pack (the tetrad construction is not differentiated on the device)
  double dconst[4 * kSceneConsts] = {};
  const bool pinhole = camera->kind == GLC_CAMERA_PINHOLE;
  if (pinhole) {
    const double step[4] = {1e-6, 1e-6, 1e-6, 1e-6 * as->observer_radius};
    for (int k = 0; k < 4; ++k) {
      double pp[4], pm[4];
      std::memcpy(pp, p0, sizeof(pp));
      std::memcpy(pm, p0, sizeof(pm));
      pp[k] += step[k];
      pm[k] -= step[k];
      glc_scene sp, sm;
      s = pack_adjoint_scene(*as, pp, sp);
      if (s == GLC_OK) s = pack_adjoint_scene(*as, pm, sm);
      if (s != GLC_OK) return set_error(s, "scene derivative: a perturbed scene is invalid");
      double cp[kSceneConsts], cm[kSceneConsts];
      gather_scene_consts(sp, cp);
      gather_scene_consts(sm, cm);
      for (int i = 0; i < kSceneConsts; ++i) dconst[k * kSceneConsts + i] = (cp[i] - cm[i]) / (2.0 * step[k]);
    }
  }

  t->ctx = ctx;
  t->pol = pol;
  t->cam = *camera;
  t->K = uint32_t(K);
  t->n = n;
  t->charge = scene.charge;
  t->pinhole = pinhole;
  t->words = uint32_t(pol.precision == GLC_MIXED ? RayWords<kMIXED>::kWords : RayWords<kFP64>::kWords);
  t->off_cams = align256(sizeof(glc_scene));
  t->off_begin = t->off_cams + align256(sizeof(glc_camera));
  t->off_cert = t->off_begin + 256;
  const size_t job_bytes = t->off_cert + 256;
  alignas(16) static thread_local unsigned char host_job[4096];
  std::memset(host_job, 0, sizeof(host_job));
  std::memcpy(host_job, &scene, sizeof(glc_scene));
  std::memcpy(host_job + t->off_cams, camera, sizeof(glc_camera));
  const unsigned long long begin[2] = {0, n}, cert_begin[2] = {0, 0};
  std::memcpy(host_job + t->off_begin, begin, sizeof(begin));
  std::memcpy(host_job + t->off_cert, cert_begin, sizeof(cert_begin));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n > t->meta_alloc) {
    if (t->d_meta) cudaFree(t->d_meta);
    t->d_meta = nullptr;
    t->meta_alloc = 0;
    if (cudaMalloc(&t->d_meta, n * sizeof(uint4)) != cudaSuccess)
      return set_error(GLC_ERR_CUDA, "tape allocation failed");
    t->meta_alloc = n;
  }
  if ((!t->d_job && cudaMalloc(&t->d_job, job_bytes) != cudaSuccess) ||
      (!t->d_dconst && cudaMalloc(&t->d_dconst, sizeof(dconst)) != cudaSuccess) ||
      (!t->d_counters && cudaMalloc(&t->d_counters, kCounters * sizeof(unsigned int)) != cudaSuccess))
    return set_error(GLC_ERR_CUDA, "tape allocation failed");
  // pageable sources: both copies have consumed their bytes when they return
  if (cudaMemcpyAsync(t->d_job, host_job, job_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(t->d_dconst, dconst, sizeof(dconst), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return set_error(GLC_ERR_CUDA, "tape upload failed");
  // pass 0: every ray, its first checkpoints in the dense slots, overflow slots reserved for the rest;
  // pass 1 (when some ray overflowed): those rays again, into the pool sized by their counts
  s = size_checkpoints(t);
  if (s == GLC_OK) s = forward(t, *out, st, 0);
  if (s != GLC_OK) return s;
  unsigned int counters[kCounters];
  if (cudaMemcpyAsync(counters, t->d_counters, sizeof(counters), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return set_error(GLC_ERR_CUDA, "forward pass failed");
  t->pool_bytes = size_t(counters[4]) * t->words * 16;
  if (counters[0] > 0) {
    s = grow(&t->d_pool, &t->pool_alloc, t->pool_bytes);
    if (s == GLC_OK) s = forward(t, *out, st, 1);
    if (s != GLC_OK) return s;
  }
  return GLC_OK;
}

}  // namespace

extern "C" {

glc_status glc_forward_ckpt(glc_ctx* ctx, const glc_adjoint_scene* as, const glc_camera* camera, int32_t K,
                            const glc_results* out, void* stream, glc_tape** tape) {
  if (!ctx || !as || !camera || !out || !tape) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  *tape = nullptr;
  DeviceScope scope(ctx->device);
  glc_tape* t = new glc_tape();
  const glc_status s = fill_tape(t, ctx, as, camera, K, out, stream);
  if (s != GLC_OK) {
    free_tape(t);
    return s;
  }
  t->valid = true;
  *tape = t;
  return GLC_OK;
}

glc_status glc_forward_ckpt_into(glc_ctx* ctx, const glc_adjoint_scene* as, const glc_camera* camera, int32_t K,
                                 const glc_results* out, void* stream, glc_tape* tape) {
  if (!ctx || !as || !camera || !out || !tape) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (tape->ctx != ctx) return set_error(GLC_ERR_INVALID_ARGUMENT, "the tape belongs to another context");
  DeviceScope scope(ctx->device);
  tape->valid = false;
  const glc_status s = fill_tape(tape, ctx, as, camera, K, out, stream);
  tape->valid = s == GLC_OK;
  return s;
}

glc_status glc_backward(glc_tape* t, const double* dl, const glc_grads* out, void* stream) {
  if (!t || !dl || !out) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (!t->valid) return set_error(GLC_ERR_INVALID_ARGUMENT, "the tape's last forward pass failed; run it again");
  DeviceScope scope(t->ctx->device);
  // scratch slots: one per block that can be resident at once (the SMs times the kernel's
  // occupancy), each slot K attempts of 7 doubles for each of the block's 128 threads
  int per_sm = 0;
  glc_status s0 = cuda_status(t->pol.precision == GLC_MIXED
                                  ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_backward_kernel<kMIXED>, 128, 0)
                                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_backward_kernel<kFP64>, 128, 0));
  if (s0 != GLC_OK) return s0;
  const unsigned int n_slots = unsigned(t->ctx->sm_count * (per_sm > 0 ? per_sm : 1));
  const size_t need = size_t(t->K) * 7 * sizeof(double) * n_slots * 128;
  if (need > t->scratch_bytes) {
    if (t->d_scratch) cudaFree(t->d_scratch);
    t->d_scratch = nullptr;
    t->scratch_bytes = 0;
    if (cudaMalloc(&t->d_scratch, need) != cudaSuccess)
      return set_error(GLC_ERR_CUDA, "adjoint scratch allocation failed");
    t->scratch_bytes = need;
  }
  if (n_slots > t->busy_slots) {
    if (t->d_busy) cudaFree(t->d_busy);
    t->d_busy = nullptr;
    t->busy_slots = 0;
    if (cudaMalloc(&t->d_busy, n_slots * sizeof(unsigned int)) != cudaSuccess)
      return set_error(GLC_ERR_CUDA, "adjoint scratch allocation failed");
    t->busy_slots = n_slots;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double* dconst = t->pinhole ? t->d_dconst : nullptr;
  const unsigned long long grid = (t->n + 127) / 128;
  if (grid > 0x7fffffffull) return set_error(GLC_ERR_CAPACITY, "too many rays for one launch");
  const glc_status sm = cuda_status(cudaMemsetAsync(t->d_busy, 0, n_slots * sizeof(unsigned int), st));
  if (sm != GLC_OK) return sm;
  if (t->pol.precision == GLC_MIXED)
    adjoint_backward_kernel<kMIXED><<<unsigned(grid), 128, 0, st>>>(t->job(), t->pol, t->K, ckpt_store(t), t->d_meta,
                                                                    t->d_scratch, t->d_busy, n_slots, dl, *out, dconst,
                                                                    t->charge, t->d_counters);
  else
    adjoint_backward_kernel<kFP64><<<unsigned(grid), 128, 0, st>>>(t->job(), t->pol, t->K, ckpt_store(t), t->d_meta,
                                                                   t->d_scratch, t->d_busy, n_slots, dl, *out, dconst,
                                                                   t->charge, t->d_counters);
  const glc_status s = cuda_status(cudaGetLastError());
  if (s == GLC_OK) t->ctx->stats.kernel_launches += 1;
  return s;
}

glc_status glc_tape_info(const glc_tape* t, uint64_t* rays, uint32_t* slots, uint64_t* bytes) {
  if (!t) return set_error(GLC_ERR_INVALID_ARGUMENT, "null pointer");
  if (rays) *rays = t->n;
  if (slots) *slots = t->cap;
  if (bytes) *bytes = t->ckpt_bytes + t->pool_bytes + t->scratch_bytes + t->n * sizeof(uint4);
  return GLC_OK;
}

glc_status glc_tape_destroy(glc_tape* t) {
  if (!t) return GLC_OK;
  DeviceScope scope(t->ctx->device);
  cudaDeviceSynchronize();
  free_tape(t);
  return GLC_OK;
}

}  // extern "C"
