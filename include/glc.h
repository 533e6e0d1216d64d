/*
 * glc.h - C ABI of the B200-native Kerr-Newman null-geodesic trace (Gravlume hot path).
 *
 * Plain C: pointers, sizes and PODs only; no CUDA, C++ or torch types cross this boundary (a
 * CUDA stream is passed as `void*`). All traces are asynchronous on the caller's stream; results
 * land in caller-owned device arrays. Nothing here aborts the process: every failure is a
 * glc_status, and glc_last_error_string() describes the last one on the calling thread.
 *
 * Threading: a glc_ctx holds its own staging buffers, streams and grow-only workspaces and takes
 * no lock, so one context serves one host thread at a time (the reference drives one wgpu queue
 * per pipeline the same way). Use one context per host thread, or serialize the calls on a shared
 * one. Contexts on the same device are independent; the host-only helpers (glc_scene_pack,
 * glc_policy_default, glc_result_slots, ...) are thread-safe.
 *
 * The entry points replace the reference's trace boundary (paths are within romeoahmed/gravlume):
 *   glc_scene_pack   <- TraceUniforms::from_observation_with_surface
 *                       (crates/gravlume-render/src/trace/input.rs:45-131), with the domain
 *                       validation of PhysicalScene::new / StationaryObserverInput::build
 *                       (crates/gravlume-domain/src/scene.rs:112-143, observer.rs:67-103)
 *   glc_create       <- TracePipeline::new (crates/gravlume-render/src/trace.rs:320-327)
 *   glc_trace        <- TracePipeline::encode_batch (trace.rs:701-710) for image cameras, and
 *                       GeodesicTracer::trace / GeodesicBatch::trace_ordered
 *                       (crates/gravlume-reference/src/geodesic.rs:53-62, batch.rs:31-43) for
 *                       explicit ray lists
 *   glc_results      <- GeometricSample (src/shaders/trace_protocol.wgsl:72-83) widened to the
 *                       reference outcome (crates/gravlume-reference/src/outcome.rs:425-436)
 *   glc_policy       <- ReferencePolicy (crates/gravlume-reference/src/policy.rs:26-66)
 *                       plus the precision mode and launch shape of this implementation
 */
#ifndef GLC_H
#define GLC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GLC_ABI_VERSION 3

typedef enum glc_status {
  GLC_OK = 0,
  GLC_ERR_INVALID_ARGUMENT = 1,   /* null pointer, bad size, bad enum */
  GLC_ERR_CUDA = 2,               /* a CUDA runtime call failed (see glc_last_error_string) */
  GLC_ERR_NON_FINITE = 3,         /* GpuTraceInputError::NonFinite / ValidationIssueCode::NonFinite */
  GLC_ERR_NON_POSITIVE = 4,       /* mass, frequency or radius not positive */
  GLC_ERR_NON_NORMALIZED = 5,     /* observer frequency != 1 within 32 eps (input.rs:61-63) */
  GLC_ERR_EXTREMALITY_CHANGED = 6,/* normalization by M changed the extremality (input.rs:84-91) */
  GLC_ERR_NON_STATIONARY = 7,     /* observer needs g_tt < 0 (observer.rs:80-86) */
  GLC_ERR_DEGENERATE_FRAME = 8,   /* target/up do not define a tetrad (observer.rs:116-151) */
  GLC_ERR_SURFACE_OUTSIDE_ESCAPE = 9, /* events.rs:73-78 */
  GLC_ERR_INVALID_SURFACE = 10,   /* events.rs:66-72 */
  GLC_ERR_INVALID_VIEW = 11,      /* view.rs:349-363 */
  GLC_ERR_TIMEOUT = 12,           /* a bounded device wait ran out */
  GLC_ERR_CAPACITY = 13,          /* request exceeds a stated maximum */
  GLC_ERR_NO_DEVICE = 14,
  GLC_ERR_UNSUPPORTED = 15
} glc_status;

/* Arithmetic of the stepper. FP32: state and right-hand side in binary32. MIXED: binary64 state
 * accumulators, binary32 right-hand side and stage combination, binary64 steps inside the
 * near-hole shell, binary64 event root-finding and a binary64 null-constraint renormalisation of
 * the final momentum. FP64: binary64 throughout. */
typedef enum glc_precision { GLC_FP32 = 0, GLC_MIXED = 1, GLC_FP64 = 2 } glc_precision;

typedef enum glc_chart { GLC_CHART_INGOING = 0, GLC_CHART_OUTGOING = 1 } glc_chart;

/* Termination discriminants: 1-7 are the reference's TraceTermination
 * (crates/gravlume-render/src/trace.rs:957-967); 8 is the adaptive stepper's consecutive-reject
 * limit (ReferenceTerminal::RejectExhaustion, outcome.rs:303). */
typedef enum glc_termination {
  GLC_TERM_NONE = 0,
  GLC_TERM_HORIZON = 1,
  GLC_TERM_ESCAPE = 2,
  GLC_TERM_SINGULARITY = 3,
  GLC_TERM_STEP_EXHAUSTION = 4,
  GLC_TERM_NUMERICAL_FAILURE = 5,
  GLC_TERM_UNCERTAIN = 6,
  GLC_TERM_SURFACE = 7,
  GLC_TERM_REJECT_EXHAUSTION = 8
} glc_termination;

/* NumericalFailure kinds (outcome.rs:129-136), in bits 8..11 of glc_results.code.x. */
typedef enum glc_failure {
  GLC_FAIL_NONE = 0, GLC_FAIL_NON_FINITE = 1, GLC_FAIL_RING = 2, GLC_FAIL_CHART_BOUNDARY = 3,
  GLC_FAIL_DENOMINATOR = 4, GLC_FAIL_MINIMUM_STEP = 5
} glc_failure;

/* Physical scene, observer, view and events in the reference's terms
 * (PhysicalSceneInput scene.rs:11-36, StationaryObserverInput observer.rs:9-31,
 *  PerspectiveView view.rs:343-370, EventConfiguration events.rs:17-84,
 *  EquatorialCircularEmitter emission.rs:30-41). */
typedef struct glc_scene_input {
  double mass, spin, charge;      /* M, a = J/M, Q in geometric units */
  int32_t chart;                  /* glc_chart */
  int32_t has_surface;            /* install the equatorial Keplerian surface */
  double observer_txyz[4];        /* observer event, Cartesian Kerr-Schild */
  double target_txyz[4];          /* look-at event */
  double up_hint_xyz[3];
  double measured_frequency;      /* must be 1 (reference-v1 normalization) */
  uint32_t width, height;         /* pinhole view */
  double vertical_fov;            /* radians, in (0, pi) */
  double escape_radius;           /* > 0: escape sphere r = R (reference baseline: 200 M) */
  double surface_inner, surface_outer; /* inclusive radial interval of the surface */
  double intensity_at_six;        /* bolometric I(6 M) of the inverse-cube emitter */
  double horizon_offset;          /* capture at r = r_+ + offset (reference: 0) */
  /* surface emission and transport (EquatorialEmissionModel, SurfaceTransport: emission.rs,
   * radiation.rs of gravlume-domain) */
  int32_t emission_model;         /* 0 inverse-cube bolometric, 1 inverse-cube blackbody */
  int32_t has_slab;               /* homogeneous scalar slab in front of the surface */
  double temperature_at_six;      /* K at r = 6 M (blackbody model) */
  double slab_optical_depth;      /* tau >= 0 */
  double slab_emission;           /* integrated bolometric emission of the slab >= 0 */
  double slab_temperature;        /* K: blackbody split of the slab emission (blackbody model) */
} glc_scene_input;

/* Device-ready packed scene, normalized to M = 1 (the analogue of TraceUniforms, kept in
 * binary64). Produced by glc_scene_pack; treat as read-only. */
typedef struct glc_scene {
  double spin, charge, chart_sign, mass_scale;
  double outer_horizon;           /* r_+, or -1 without a horizon */
  double horizon_event_radius;    /* r_+ + offset */
  double escape_radius;           /* 0 when not installed */
  double surface_inner, surface_outer, intensity_at_six;
  double photon_shell_radius;     /* inner (prograde) equatorial photon orbit radius */
  double isco_prograde;           /* prograde ISCO radius (informational) */
  double observer_txyz[4];
  double four_velocity[4], image_right[4], image_up[4], arrival[4];
  double metric_covariant[16];    /* g_{mu nu} at the observer */
  double frequency;
  double tangent_half_fov;
  uint32_t width, height;
  int32_t extremality;            /* 0 subextremal, 1 extremal, 2 superextremal */
  int32_t has_horizon, has_escape, has_surface;
  int32_t emission_model;         /* 0 bolometric, 1 blackbody */
  int32_t reserved;
  double temperature_at_six;      /* K (blackbody) */
  double slab_transmittance;      /* exp(-tau), 1 without a slab */
  double slab_emission;           /* integrated bolometric emission, 0 without a slab */
  double slab_bands[3];           /* its red, green, blue band split (blackbody), else 0 */
} glc_scene;

/* Step policy: ReferencePolicy fields (policy.rs:26-66) + precision + launch shape. */
typedef struct glc_policy {
  double position_rtol, position_atol, momentum_rtol, momentum_atol;
  double initial_step, minimum_step, maximum_step;
  double safety, minimum_factor, maximum_factor;
  uint64_t maximum_accepted_steps;
  uint32_t maximum_consecutive_rejects;
  int32_t precision;              /* glc_precision */
  double event_affine_tolerance, event_tie_tolerance, event_arming_band, singularity_guard;
  double mixed_shell_factor;      /* MIXED: binary64 steps while r < factor * prograde photon orbit */
  uint32_t renormalize_null;      /* MIXED: renormalize the final momentum onto H = 0 */
  uint32_t persistent;            /* 0: one thread per ray; 1: persistent work queue with lane
                                     refill; 2: persistent work queue with warp-granular grabs */
  uint32_t block_threads;         /* threads per block (multiple of 32) */
  uint32_t blocks_per_sm;         /* persistent grid = SMs * blocks_per_sm (0 = occupancy) */
  uint32_t tile_w, tile_h;        /* pixel tile a warp's consecutive rays cover */
  uint32_t refill_interval;       /* persistent: steps between warp refills of finished lanes */
  uint32_t rays_per_grab;         /* persistent: rays a warp takes from the queue per refill (>= 32) */
  uint32_t refill_min_idle;       /* persistent: idle lanes that trigger a refill (1..32) */
  uint32_t mixed_pair_state;      /* MIXED: accumulate the state as compensated binary32 pairs */
  uint32_t capture_certificates;  /* 1: interval capture certificates on 16x16 tiles of image
                                     cameras of surface-free scenes; certified rays skip integration */
  uint32_t escape_map;            /* 1: escape-direction map (node pass on every 4th pixel, stable
                                     8x8 tiles of surface-free scenes reconstructed by interpolation) */
  uint32_t mixed_split;           /* MIXED: 1 (default) two kernels, binary32 stepping with the
                                     pair state (in the one-thread-per-ray kernel or either work
                                     queue) until a ray's first step that brackets a terminal
                                     event, crosses the surface near or on it, or enters the shell,
                                     then binary64 from a 128-byte hand-off record per ray (context
                                     memory, grow-only). The binary32 stepping takes a pericentre's
                                     turning radius as the largest root of the radial potential of
                                     the step's constants of motion rather than the root of the
                                     radial velocity on the dense output (the two differ by the
                                     constants' drift). 0: one kernel whose warps step in binary64
                                     while a lane is inside the shell */
  uint32_t uncertain_terminals;   /* 1: the replaced wgpu kernel's gate (geodesic_integration.wgsl
                                     324-330): a terminal becomes GLC_TERM_UNCERTAIN when more than
                                     one event lies within the tie tolerance of the earliest, when
                                     the terminal lies inside the bracket of a radial turning point
                                     of its step, or when a recorded invariant drift exceeds
                                     uncertain_drift_limit; 0 (default, the reference's CPU
                                     semantics): the earliest event terminates and the tied kinds
                                     are reported in the candidate bits of code.x */
  double uncertain_drift_limit;   /* drift budget of the gate (INVARIANT_DRIFT_LIMIT 0.05,
                                     crates/gravlume-render/src/trace/input.rs:13) */
} glc_policy;

typedef enum glc_camera_kind {
  GLC_CAMERA_PINHOLE = 0,         /* PerspectiveView sight plane (view.rs:408-424) */
  GLC_CAMERA_EQUIRECT = 1,        /* full-sphere longitude/latitude map in the observer frame */
  GLC_CAMERA_RAYLIST = 2          /* explicit initial states (t,x,y,z,p_t,p_x,p_y,p_z) */
} glc_camera_kind;

typedef struct glc_camera {
  int32_t kind;                   /* glc_camera_kind */
  int32_t scene_index;            /* index into the scenes array of the call */
  uint32_t width, height;         /* image size (PINHOLE: must equal the scene's view) */
  double subpixel_x, subpixel_y;  /* sample offset inside the pixel, [0, 1] */
  const double* ray_states;       /* RAYLIST: device pointer, n_rays * 8 doubles */
  uint64_t n_rays;                /* RAYLIST: number of rays (images: ignored) */
  double affine_direction;        /* RAYLIST: +1 or -1 (images trace backward, -1) */
  uint64_t result_offset;         /* first result slot of this camera */
  /* Image cameras: the batch of 8x8-pixel tiles to trace, as TileRegion { origin, workgroups }
   * (crates/gravlume-render/src/trace.rs:799-857) with TRACE_WORKGROUP_AXIS = 8. tile_count {0, 0}
   * traces the whole view. Results keep the whole view's layout (slot result_offset + y * width +
   * x), and only the batch's pixels are written, so a frame traced batch by batch equals the
   * frame traced at once. Accepted by glc_trace, glc_trace_host, glc_graph_capture and
   * glc_trace_static_scratch; the shadow-edge, footprint and adjoint passes take whole views. */
  uint32_t tile_origin[2];        /* first tile (column, row) */
  uint32_t tile_count[2];         /* tiles (columns, rows), within the view's tile grid */
} glc_camera;

/* Caller-owned device SoA, one 16-byte element per ray in each array (128-bit stores). Any
 * pointer may be NULL to skip that field. Lengths: >= max(result_offset + rays of camera).
 *   code.x  termination | failure << 8 | event candidates << 12 | (polar side + 1) << 16
 *           | flags << 20 (bit 20: shell steps taken in binary64; bit 21: null renormalized;
 *           bit 22: surface hit whose emitter observable is undefined; bit 23: escape without a
 *           direction; bit 24: capture proven by the tile's interval certificate, ray not
 *           integrated; bit 25: escape direction reconstructed from the escape-direction map)
 *   code.y  accepted steps, code.z rejected steps, code.w binary64 steps (MIXED)
 *   branch  radial turnings, equatorial crossings, azimuth winding, has turning radius
 *   escape  (polar angle, azimuth) of the unit coordinate direction at escape (NaN otherwise)
 *   surface (source radius, source azimuth) at a surface hit (NaN otherwise)
 *   redshift_time (g = nu_obs / nu_em at a surface hit or NaN, coordinate travel time)
 *   event   (normalized event residual, affine parameter at termination)
 *   drift_a (max normalized null residual, max relative energy drift)
 *   drift_b (max relative L_z drift, max relative Carter drift); when both drift arrays are NULL
 *           the invariants behind them are not evaluated at each step (they do not steer the
 *           integration), which makes the trace 10-17 % faster
 *   turning (minimum turning radius or NaN, azimuth advance)
 *   position_xy / position_zr (final x, y) / (final z, final Kerr-Schild radius)
 *   intensity / radiance: post-hit surface transport (see below) */
typedef struct glc_u32x4 { uint32_t x, y, z, w; } glc_u32x4;
typedef struct glc_i32x4 { int32_t x, y, z, w; } glc_i32x4;
typedef struct glc_f64x2 { double x, y; } glc_f64x2;
typedef struct glc_half4 { uint16_t x, y, z, w; } glc_half4; /* IEEE binary16 bit patterns */

typedef struct glc_results {
  glc_u32x4* code;
  glc_i32x4* branch;
  glc_f64x2* escape;
  glc_f64x2* surface;
  glc_f64x2* redshift_time;
  glc_f64x2* event;
  glc_f64x2* drift_a;
  glc_f64x2* drift_b;
  glc_f64x2* turning;
  glc_f64x2* position_xy;
  glc_f64x2* position_zr;
  glc_f64x2* intensity;           /* (observed bolometric intensity after the slab, emitted) at a surface hit */
  glc_half4* radiance;            /* RGBA16F, 8 bytes per ray: observed surface radiance (r, g, b, 2)
                                     at a surface hit, zero elsewhere (surface_transport.wgsl) */
} glc_results;

typedef struct glc_ctx glc_ctx;
typedef struct glc_graph glc_graph;

typedef struct glc_launch_stats {
  uint64_t kernel_launches;       /* kernels this context launched since creation */
  uint64_t last_rays;             /* rays in the last trace */
  uint32_t last_grid, last_block; /* launch shape of the last trace kernel */
  uint32_t last_persistent;       /* 1 if the last trace used the work queue */
  uint32_t sm_count;
} glc_launch_stats;

/* ---- version and errors ---------------------------------------------------------------- */
int glc_abi_version(void);
const char* glc_last_error_string(void);
const char* glc_status_string(glc_status status);

/* ---- scenes and policies (host only; no device needed) ---------------------------------- */
glc_status glc_scene_pack(const glc_scene_input* input, glc_scene* out);
/* preset: 0 reference-regular-v1, 1 reference-strict-v1, 2 frame policy of the precision mode. */
glc_status glc_policy_default(int32_t preset, int32_t precision, glc_policy* out);
/* Prograde ISCO radius of Kerr-Newman in units of M (spin, charge in units of M). */
glc_status glc_prograde_isco(double spin, double charge, double* out);
/* Algorithmic operation model of the kernel (counted from the same templated source on the host):
 * out[0] flops per right-hand-side evaluation (FMA = 2), out[1] special-function ops (rcp, sqrt,
 * rsqrt) per evaluation, out[2] flops per attempted DP5(4) step, out[3] special ops per step. */
glc_status glc_flop_model(double out4[4]);
/* Host evaluation of the device right-hand side (the same template code), for checks:
 * state = (x, y, z, p_x, p_y, p_z), energy = -p_t; out = (x', y', z', p_x', p_y', p_z', t'). */
glc_status glc_rhs_host(const glc_scene* scene, const double state6[6], double energy, int32_t precision,
                        double out7[7]);

/* ---- context ----------------------------------------------------------------------------- */
glc_status glc_create(int32_t device, glc_ctx** out);
glc_status glc_destroy(glc_ctx* ctx);
glc_status glc_set_policy(glc_ctx* ctx, const glc_policy* policy);
glc_status glc_get_policy(const glc_ctx* ctx, glc_policy* out);
glc_status glc_get_stats(const glc_ctx* ctx, glc_launch_stats* out);

/* ---- forward trace ----------------------------------------------------------------------- */
/* Number of result slots the cameras need (max over result_offset + rays). */
glc_status glc_result_slots(const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                            int32_t n_cameras, uint64_t* out);
/* Trace every camera's rays; stream-ordered and asynchronous. Scenes/cameras are host arrays
 * (copied into the context's device job table on `stream`); results are device pointers. */
glc_status glc_trace(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                     int32_t n_cameras, const glc_results* out, void* stream);
/* End-to-end convenience over host buffers: copies RAYLIST states host->device, traces, and
 * copies every non-NULL result array device->host. Synchronous. */
glc_status glc_trace_host(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                          int32_t n_cameras, const glc_results* host_out);

/* Shadow-edge coverage refinement (shadow_coverage.wgsl:63-136, classify_shadow_edges and
 * refine_shadow_edges): after a glc_trace of the same job into `primary` (its code array is read),
 * coverage[slot] is 1 for escape and 0 for capture pixels of image cameras, -1 for any other
 * class; capture/escape pixels with a 4-neighbour of the other class are re-traced with four
 * rotated-grid subpixel samples (0.375, 0.125), (0.875, 0.375), (0.625, 0.875), (0.125, 0.625) and
 * get the fraction of escaping samples, unless a sample ends another way. coverage is a device
 * float array as long as the results. Stream-ordered, no host synchronization. */
glc_status glc_refine_shadow_edges(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes,
                                   const glc_camera* cameras, int32_t n_cameras, const glc_results* primary,
                                   float* coverage, void* stream);

/* ---- surface footprint (footprint.rs:74-235) --------------------------------------------- */
/* Local source Jacobian of an image pixel that ends on the surface: rows (source radius, local
 * azimuthal arc r_c * dphi), columns (screen x, screen y), in M per image pixel (footprint.rs:30-32);
 * its singular values (major, minor; minor = |det| / major) and parity (+1, -1, 0 within
 * 64 eps |J|_F^2 of a zero determinant). 64 bytes. */
typedef struct glc_footprint {
  double jacobian[4];        /* dr/dx, dr/dy, darc/dx, darc/dy */
  double singular_values[2]; /* major, minor */
  double determinant;
  int32_t status;            /* GLC_FOOTPRINT_* */
  int32_t parity;
} glc_footprint;

#define GLC_FOOTPRINT_NO_SURFACE 0    /* center is not an unambiguous observed surface hit (CenterSurfaceUnavailable) */
#define GLC_FOOTPRINT_RESOLVED 1
#define GLC_FOOTPRINT_DISCONTINUITY 2 /* a neighbour left the surface or the center's branch key */
#define GLC_FOOTPRINT_NON_FINITE 3    /* NonFiniteJacobian */

/* QUARTER_PIXEL: the reference's estimate (surface_footprint_v1): the four neighbours a quarter
 * pixel left, right, up and down are traced, and the Jacobian is their central difference over
 * the half-pixel span; needs camera subpixels in [0.25, 0.75]. TANGENT: the exact derivative of
 * the computed trace in forward mode (two tangent channels through the ray set-up, every accepted
 * step at its frozen size and the terminal event time), one re-trace per pixel; it does not test
 * the neighbourhood and never reports DISCONTINUITY. */
#define GLC_FOOTPRINT_QUARTER_PIXEL 0
#define GLC_FOOTPRINT_TANGENT 1

/* After a glc_trace of the same job into `primary` (code, branch and surface arrays are read),
 * out[slot] (a device array as long as the results) receives the footprint of every pixel of the
 * image cameras; entries that are not RESOLVED hold NaN. Ray-list cameras are rejected.
 * Stream-ordered, no host synchronization. */
glc_status glc_surface_footprint(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                                 int32_t n_cameras, int32_t method, const glc_results* primary, glc_footprint* out,
                                 void* stream);

/* ---- CUDA graphs (per-frame replay of the job-table copy, queue reset and trace launch) ---- */
glc_status glc_graph_capture(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                             int32_t n_cameras, const glc_results* out, void* stream, glc_graph** graph);
glc_status glc_graph_launch(glc_graph* graph, void* stream);
glc_status glc_graph_destroy(glc_graph* graph);

/* ---- autotuner ----------------------------------------------------------------------------- */
/* Times candidate launch shapes (tile shape, rays per grab, refill interval, block size) on the
 * given job and writes the fastest into *policy (and the context). out may be scratch results. */
glc_status glc_autotune(glc_ctx* ctx, const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                        int32_t n_cameras, const glc_results* out, void* stream, int32_t repeats,
                        glc_policy* policy);

/* ---- discrete adjoint (forward with checkpoints, backward) --------------------------------- */
/* Gradients of per-ray observables (source radius, g, escape theta, escape phi) with respect to
 * spin a, charge Q, observer inclination, observer radius (the observer sits at fixed oblate
 * coordinates) and each ray's initial covariant momentum. The reference has no adjoint; these are
 * the forward/backward pair over the trace boundary of glc_trace (trace.rs:701-710 for images,
 * geodesic.rs:53-62 for explicit ray lists). Precision MIXED or FP64 (the context's policy). */
typedef struct glc_tape glc_tape;

typedef struct glc_adjoint_scene {
  glc_scene_input input;          /* observer_txyz is replaced by the oblate position below */
  double observer_radius;         /* oblate (Boyer-Lindquist) radius of the observer */
  double observer_polar;          /* inclination, radians */
  double observer_azimuth;
} glc_adjoint_scene;

typedef struct glc_grads {
  double* ray_momentum;           /* device, slots x 4: dL/d(p_t, p_x, p_y, p_z) at the initial state */
  double* ray_params;             /* device, slots x 4 or NULL: each ray's share of dL/d(a, Q, incl, r_obs) */
  double* params;                 /* device, 4 or NULL: dL/d(a, Q, inclination, r_obs), ADDED to (caller zeroes) */
} glc_grads;

/* Forward trace of one camera (PINHOLE of the scene's view, or RAYLIST) that also checkpoints each
 * ray's stepper state every K accepted steps into the tape (device memory owned by the tape).
 * Results as glc_trace. The MIXED shell decision is taken per ray (glc_trace takes it per warp), so
 * the backward pass can replay every segment exactly. Synchronizes the stream once (to size the
 * checkpoints). */
glc_status glc_forward_ckpt(glc_ctx* ctx, const glc_adjoint_scene* scene, const glc_camera* camera, int32_t K,
                            const glc_results* out, void* stream, glc_tape** tape);
/* The forward pass again, into a tape from glc_forward_ckpt on the same context: the tape's device
 * memory is kept and grows only where this request needs more rays or checkpoint slots, so an
 * optimization loop (forward, backward, parameter update) allocates nothing after its first
 * iteration. Earlier checkpoints are overwritten, so the earlier pass's gradients are no longer
 * available; issue it on the stream of the tape's last glc_backward (or synchronize first).
 * Synchronizes the stream once, as glc_forward_ckpt. When it fails, glc_backward rejects the tape
 * until a forward pass into it succeeds. */
glc_status glc_forward_ckpt_into(glc_ctx* ctx, const glc_adjoint_scene* scene, const glc_camera* camera, int32_t K,
                                 const glc_results* out, void* stream, glc_tape* tape);
/* Backward pass: dL_dobs is device, slots x 4 (dL/d source radius, g, escape theta, escape phi;
 * rays that end elsewhere get zero gradients). Replays each checkpointed segment and sweeps it in
 * reverse (binary64). Asynchronous on the stream. */
glc_status glc_backward(glc_tape* tape, const double* dL_dobs, const glc_grads* out, void* stream);
/* Checkpoint sizing: rays traced, checkpoint slots per ray, device bytes held by the tape. */
glc_status glc_tape_info(const glc_tape* tape, uint64_t* rays, uint32_t* slots_per_ray, uint64_t* bytes);
glc_status glc_tape_destroy(glc_tape* tape);

/* ---- test hook ----------------------------------------------------------------------------- */
/* The event-policy cases of the reference's test-only capture pipeline
 * (TracePipeline::for_event_policy_capture, crates/gravlume-render/src/gpu_capture.rs:145-150, and
 * shaders/event_policy_capture.wgsl), run on the device by the same earliest-event selection and
 * arming functions as the trace kernels, under `policy` (its tie tolerance, arming band and step
 * limits). out: 16-byte aligned device array of 8 x 4 uint32. Cases 0-3: (termination, candidate
 * bits, ambiguous, 0) of synthetic roots at fractions of the step; cases 4-7: (armed, 0, 0, 0) of
 * the surface event for a value 0, half the band, twice the band, and an already armed event.
 * Asynchronous on the stream. */
glc_status glc_selftest_event_policy(const glc_policy* policy, uint32_t* out, void* stream);

/* ---- trace without device allocation ------------------------------------------------------ */
/* No counterpart in the reference: its wgpu trace pass always allocates its own target and
 * scratch. For callers that may not allocate device memory (a host whose frame allocator owns the
 * device heap, a plugin confined to buffers its host hands it): the trace of glc_trace, without a
 * context. Its scratch (queue counter and job table) is a 96 KiB static device array, so at most
 * 128 scenes and 128 cameras (GLC_ERR_CAPACITY beyond). Runs on the current device; the first
 * call on a device looks up the array's address, so make it before any stream capture (a
 * cudaDeviceReset makes the next call look it up again). All calls share the array: calls that
 * overlap on the GPU race. Scenes, cameras and policy are host structs; results (and RAYLIST
 * states) are device pointers. The policy is checked as by glc_set_policy; `persistent` picks the
 * kernel as in glc_trace; MIXED always runs as one kernel (mixed_split is ignored: the two-kernel
 * form needs a hand-off record per ray); capture_certificates and escape_map must be 0
 * (GLC_ERR_INVALID_ARGUMENT otherwise). Tile regions are accepted. */
glc_status glc_trace_static_scratch(const glc_scene* scenes, int32_t n_scenes, const glc_camera* cameras,
                                    int32_t n_cameras, const glc_policy* policy, const glc_results* out,
                                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GLC_H */
