/*
 * bh_b200.h -- C ABI of the B200 geodesic hot path (libbh_b200.so).
 *
 * Plain pointers and sizes only; every device pointer is CUDA global memory
 * owned by the caller, every stream is a cudaStream_t passed as void*.  All
 * calls are stream-ordered and asynchronous unless the comment says
 * otherwise.  Functions return BH_OK (0) or a negative bh_status.
 *
 * State layout: a batch of n geodesic states (t, x, y, z, p_t, p_x, p_y, p_z),
 * covariant momenta, float64 -- the reference's (n, 8) row-major array
 * (blackhorizon/geodesics.py:1-16).  Trace and propagate calls also accept
 * the structure-of-arrays layout (8 planes of n doubles).
 *
 * Each entry point names the reference function it replaces
 * (MegaKruk/BlackHorizon, path within that project, file:line).
 */
#ifndef BH_B200_H
#define BH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BH_ABI_VERSION 5

typedef enum {
    BH_OK = 0,
    BH_ERR_INVALID_ARGUMENT = -1, /* bad pointer, size, tolerance or Kerr bound */
    BH_ERR_CUDA = -2,             /* a CUDA runtime call failed; see bh_last_error */
    BH_ERR_TIMEOUT = -3,          /* the trace deadline passed before every ray finished */
    BH_ERR_ESCAPE_RADIUS = -4,    /* an initial radius is >= escape_radius (tracer.py:95-99) */
    BH_ERR_WORKSPACE = -5,        /* workspace missing, too small or misaligned */
    BH_ERR_TAPE = -6              /* a ray took more accepted steps than the tape holds */
} bh_status;

/* Per-ray termination codes: blackhorizon/tracer.py:21-30 (RayStatus). */
enum {
    BH_RAY_IN_FLIGHT = 0,
    BH_RAY_CAPTURED = 1,
    BH_RAY_ESCAPED = 2,
    BH_RAY_MAX_STEPS = 3,
    BH_RAY_FAILED = 4,
    BH_RAY_DISK = 5,      /* ended on the equatorial disk (tile and real-time tracers) */
    BH_RAY_TERMINATED = 6 /* reached the interior stop radius (real-time tracer) */
};

typedef enum {
    BH_PRECISION_FP64 = 0,  /* every operation in float64 */
    BH_PRECISION_MIXED = 1  /* float32 stage arithmetic (float64 inside the
                               f64_radius band of bh_propagate), float64 state,
                               error norm, step control and termination radius */
} bh_precision;

typedef enum {
    BH_LAYOUT_AOS = 0, /* (n, 8) row-major, the reference's layout */
    BH_LAYOUT_SOA = 1  /* 8 planes of n doubles */
} bh_layout;

/* Kerr spacetime and termination radii of one scene.  capture_radius is
 * r_plus * (1 + capture_margin) (tracer.py:84); escape_radius as passed to
 * trace_rays. */
typedef struct {
    double mass;
    double spin;
    double capture_radius;
    double escape_radius;
} bh_scene;

/* A pinhole camera (camera.py:25-120) plus the scene it looks at.  The basis
 * (forward, right, up) is the one camera.py:48-66 builds on the host. */
typedef struct {
    double position[3];
    double forward[3];
    double right[3];
    double up[3];
    double fov_degrees;
    int64_t width;
    int64_t height;
    bh_scene scene;
} bh_camera;

/* Controller settings of trace_rays (tracer.py:50-61) and launch knobs. */
typedef struct {
    int64_t max_steps;     /* accepted-step budget per ray */
    double rtol, atol;
    double initial_step, max_step, min_step;
    int32_t precision;     /* bh_precision */
    int32_t layout;        /* bh_layout */
    int64_t timeout_ns;    /* device deadline for the launch; 0 = none */
    int32_t variant;       /* launch-shape variant (bh_trace_variant); -1 = default */
    int32_t blocks_per_sm; /* resident blocks per SM; 0 = occupancy maximum */
    int32_t project_every; /* Hamiltonian-constraint projection every K controller
                              iterations, 0 = off (the reference never projects) */
    int32_t flags;         /* bh_trace_flag bits; 0 for every call but bh_trace_tile */
    int32_t reserved;      /* 0 */
    /* bh_propagate, BH_PRECISION_MIXED: radius (units of M) of the float64
     * band.  An attempt runs float64 stage arithmetic for every ray of a
     * warp (rays [64 k, 64 k + 64) of the call) while one of them lies
     * between 1.01 r_+ and f64_radius;
     * elsewhere the stages run in float32.  0 = no band; < 0 = 8 u M / rtol
     * (u = 2^-24), where the float32 rounding of the curvature terms, about
     * 4 u of their relative size 2 M / r, reaches the tolerance.  Must be 0
     * for every other call.  Not in the reference (float64 throughout). */
    double f64_radius;
} bh_trace_config;

/* Bits of bh_trace_config.flags. */
typedef enum {
    /* bh_trace_tile: interior camera (offline/render.py:203-248).  The
     * scene's capture_radius is the interior stop radius; a ray ends with
     * BH_RAY_TERMINATED at r <= stop, when the norm of its spatial momentum
     * (p_x, p_y, p_z) exceeds 1e3, or at r <= 1.002 stop with a norm above
     * 50. */
    BH_TRACE_INTERIOR = 1
} bh_trace_flag;

/* Whole-launch counters of a trace or propagate call. */
typedef struct {
    int64_t iterations;    /* max attempts over rays == reference TraceResult.iterations */
    int64_t attempts;      /* attempted DP5 steps summed over rays */
    int64_t accepted;      /* accepted DP5 steps summed over rays */
    int32_t timed_out;     /* nonzero when the deadline stopped the launch */
    int32_t bad_rays;      /* rays whose initial radius is >= their escape radius */
} bh_trace_stats;

/* ------------------------------------------------------------- library */

int bh_abi_version(void);
const char *bh_status_string(int status);
/* Message of the last failure on the calling host thread ("" if none). */
const char *bh_last_error(void);

/* ---------------------------------------------------------- pointwise
 * One thread per point; float64. */

/* KerrSpacetime.geometry (blackhorizon/kerr.py:118-193).  x, y, z are read
 * with element stride `stride` (8 reads the columns of an (n,8) state).  Any
 * of grad_h (n,3) / grad_l (n,3,3, grad_l[i][j] = dl_j/dx_i) may be NULL. */
int bh_geometry(double mass, double spin, const double *x, const double *y,
                const double *z, int64_t stride, int64_t n, double *r,
                double *h, double *l, double *grad_h, double *grad_l,
                void *stream);

/* geodesic_rhs (blackhorizon/geodesics.py:42-74): (n,8) -> (n,8). */
int bh_geodesic_rhs(double mass, double spin, const double *state,
                    double *deriv, int64_t n, void *stream);

/* hamiltonian (geodesics.py:77-85): (n,8) -> (n,). */
int bh_hamiltonian(double mass, double spin, const double *state, double *out,
                   int64_t n, void *stream);

/* coordinate_velocity (geodesics.py:95-106): (n,8) -> (n,4). */
int bh_coordinate_velocity(double mass, double spin, const double *state,
                           double *out, int64_t n, void *stream);

/* null_momentum_from_velocity (geodesics.py:109-170): positions (n,3),
 * directions (n,3) -> momenta (n,4).  spin_of_ray (n,) overrides spin when
 * non-NULL. */
int bh_null_momentum(double mass, double spin, const double *spin_of_ray,
                     const double *positions, const double *directions,
                     int64_t n, int32_t past, int32_t normalize,
                     double *momenta, void *stream);

/* PinholeCamera.ray_directions + ray_origins (camera.py:96-120) followed by
 * null_momentum_from_velocity(..., "past") and build_state (geodesics.py:25-39,
 * t0 = 0): writes the (width*height, 8) initial states of a camera. */
int bh_camera_states(const bh_camera *camera, double *state, void *stream);

/* -------------------------------------------------------- integrators */

/* dormand_prince_step (blackhorizon/integrators.py:76-107) with the
 * geodesic RHS: state (n,8), h (n,) -> new_state (n,8), error (n,8). */
int bh_dp5_step(double mass, double spin, const double *state,
                const double *h, double *new_state, double *error, int64_t n,
                int32_t precision, void *stream);

/* error_ratio (integrators.py:110-117) for 8-component states. */
int bh_error_ratio(const double *state, const double *new_state,
                   const double *error, double rtol, double atol,
                   double *ratio, int64_t n, void *stream);

/* step_factor (integrators.py:120-124). */
int bh_step_factor(const double *ratio, double *factor, int64_t n,
                   void *stream);

/* The device arithmetic of the stage and controller code, point-wise, so its
 * accuracy can be checked against IEEE results: op 0 = the float64
 * reciprocal (MUFU seed, two Newton-Raphson steps), op 1 = the float64
 * reciprocal square root (likewise), op 2 = the mixed policy's step factor
 * clip(0.9 x^-0.1, 0.2, 5) of x = r^2 (float32 seed, one Newton-Raphson
 * step in float64).  No counterpart in the reference, which calls NumPy. */
int bh_device_math(int32_t op, const double *x, double *y, int64_t n, void *stream);

/* rk4_step (integrators.py:57-73) with the geodesic RHS, repeated n_steps
 * times in registers with the fixed per-ray step h (n,).  n_steps = 1 is one
 * rk4_step; the README benchmark (examples/benchmark.py:39-51) is h = 0.05,
 * 50 steps. */
int bh_rk4(double mass, double spin, const double *state, const double *h,
           double *new_state, int64_t n, int64_t n_steps, int32_t precision,
           void *stream);

/* implicit_midpoint_step (integrators.py:177-207), n_steps times: the
 * symplectic midpoint rule y1 = y0 + h f((y0 + y1) / 2) solved by
 * `iterations` fixed-point refinements of the explicit Euler half step;
 * float64.  (n, 8) in, (n, 8) out, h (n,). */
int bh_implicit_midpoint(double mass, double spin, const double *state, const double *h,
                         double *new_state, int64_t n, int32_t iterations, int64_t n_steps,
                         void *stream);

/* ------------------------------------------------------------- tracer */

/* Launch-shape variants of the trace and propagate kernels for a precision:
 * threads per block, the __launch_bounds__ minimum blocks per SM (which caps
 * registers per thread), rays per thread (2 = two rays in the halves of
 * packed float32x2 instructions, mixed precision only), and the registers
 * and resident blocks per SM of the compiled trace kernel.  The autotuner
 * times them; index -1 in bh_trace_config selects the default (here: the
 * tracer's; the propagator's mixed default is the packed 128 x 3 shape). */
int bh_trace_variant_count(int32_t precision);
int bh_trace_variant(int32_t precision, int32_t index, int32_t *block_threads,
                     int32_t *min_blocks, int32_t *rays_per_thread,
                     int32_t *registers, int32_t *max_blocks_per_sm);

/* Bytes of device workspace a trace or propagate launch needs (queue head and
 * counters), for any n; 256-byte aligned. */
size_t bh_trace_workspace_bytes(void);

/* trace_rays (blackhorizon/tracer.py:50-157) for one scene: a persistent
 * kernel, one ray per thread, state in registers, warp-aggregated refill from
 * a work queue held in `workspace`.  state0 and states may alias.  status (n,)
 * int32, steps (n,) int64 = accepted steps.  Launch counters stay in the
 * workspace until the next call; read them with bh_trace_stats_read.
 * Rays whose initial radius is >= escape_radius are counted in bad_rays and
 * make bh_trace_stats_read return BH_ERR_ESCAPE_RADIUS. */
int bh_trace(const bh_trace_config *config, const bh_scene *scene,
             const double *state0, double *states, int32_t *status,
             int64_t *steps, int64_t n, void *workspace, void *stream);

/* trace_rays for many cameras in one launch.  The pinhole ray generation of
 * bh_camera_states is fused into the refill of the persistent kernel, each
 * camera carries its own scene, and the rays of all cameras form one work
 * queue: camera c owns global rays [offset_c, offset_c + width_c*height_c),
 * offsets in table order.  bh_camera_table_upload copies the HOST camera
 * array into the workspace (which must hold
 * bh_trace_cameras_workspace_bytes(ncameras) bytes) and returns the total
 * ray count; bh_trace_cameras then resets the counters and launches, and
 * makes no host-to-device copy, so it can be captured in a CUDA graph and
 * replayed while the table stays in the workspace. */
size_t bh_trace_cameras_workspace_bytes(int32_t ncameras);
int bh_camera_table_upload(const bh_camera *cameras, int32_t ncameras,
                           void *workspace, size_t workspace_bytes,
                           int64_t *n_rays, void *stream);
int bh_trace_cameras(const bh_trace_config *config, int32_t ncameras,
                     int64_t n_rays, double *states, int32_t *status,
                     int64_t *steps, void *workspace, size_t workspace_bytes,
                     void *stream);

/* The counter reset and persistent launch of bh_trace_cameras captured once
 * into a CUDA graph (camera table already uploaded to `workspace`), then
 * replayed with one bh_graph_launch per frame; read the counters with
 * bh_trace_stats_read after each replay.  The graph keeps the pointers it was
 * captured with.  bh_graph_destroy releases it.  No counterpart in the
 * reference, which launches ~60 array kernels per RHS evaluation. */
typedef struct bh_graph bh_graph;
int bh_graph_trace_cameras(const bh_trace_config *config, int32_t ncameras,
                           int64_t n_rays, double *states, int32_t *status,
                           int64_t *steps, void *workspace,
                           size_t workspace_bytes, bh_graph **out);
int bh_graph_launch(bh_graph *graph, void *stream);
int bh_graph_destroy(bh_graph *graph);

/* bh_trace_cameras without a caller-owned workspace, for callers that cannot
 * allocate device memory (a host application that owns all GPU memory
 * through its own fixed pool, or code under a hard memory budget).  No
 * counterpart in the reference.  The launch counters, work-queue head and
 * camera table live in one static device array of the library, sized for
 * at most 256 cameras (256 + 256 x 168 = 43,264 bytes, held on every GPU that loads the library
 * until the process exits); more cameras return BH_ERR_INVALID_ARGUMENT.
 * cameras is a HOST array.  The call uploads the table, launches, then copies
 * the counters into *stats (may be NULL) and synchronises `stream`; it
 * returns what bh_trace_stats_read would.  The first call on a device looks
 * up the array's device address, so make it before any stream capture.  The
 * address is kept for the life of the process: after cudaDeviceReset (or any
 * other reset of the device's primary context) this entry point must not be
 * called again in that process, since the kept address belongs to the
 * destroyed context.
 * Every call shares the one array: calls that overlap on the GPU (on
 * different streams or host threads) race and must be serialised by the
 * caller.  Allocates nothing (no cudaMalloc / cudaFree, no heap). */
int bh_trace_cameras_noalloc(const bh_trace_config *config,
                             const bh_camera *cameras, int32_t ncameras,
                             double *states, int32_t *status, int64_t *steps,
                             bh_trace_stats *stats, void *stream);

/* Copies the counters of the last launch on `workspace` to the host and
 * synchronises `stream`.  Returns BH_ERR_TIMEOUT / BH_ERR_ESCAPE_RADIUS when
 * the launch hit its deadline or met a ray outside its escape radius, and
 * BH_ERR_INVALID_ARGUMENT when a propagate launch met a ray whose own spin
 * breaks the Kerr bound. */
int bh_trace_stats_read(const void *workspace, bh_trace_stats *out,
                        void *stream);

/* Adaptive propagation without termination: n_steps attempted DP5(4) steps
 * per ray with the accept/reject and step-size update of tracer.py:111-120.
 * spin_of_ray (n,) gives each ray its own spin when non-NULL; a ray whose spin
 * breaks the Kerr bound is traced at spin 0 and makes bh_trace_stats_read
 * return BH_ERR_INVALID_ARGUMENT.  states (n,8)
 * and h (n,) are updated in place; lam (n,), when non-NULL, accumulates the
 * affine parameter of the accepted steps in float64 (in/out); accepted (n,)
 * int64 receives accepted steps.  Uses the workspace counters like bh_trace. */
int bh_propagate(const bh_trace_config *config, double mass, double spin,
                 const double *spin_of_ray, double *states, double *h,
                 double *lam, int64_t *accepted, int64_t n, int64_t n_steps,
                 void *workspace, void *stream);

/* bh_propagate with the rays taken in the order `order` (n,) int32: launch
 * position i holds ray order[i], and every per-ray array stays indexed by
 * ray.  NULL takes the rays in their own order (bh_propagate).  Entries
 * outside [0, n) are not traced and make bh_trace_stats_read return
 * BH_ERR_INVALID_ARGUMENT.  The mixed propagator decides its float64 band per
 * warp of 64 launch positions; bh_propagate_order's order groups rays that
 * pass the hole alike, so fewer warps need the band.  No counterpart in the
 * reference, which steps every ray on its own. */
int bh_propagate_ordered(const bh_trace_config *config, double mass, double spin,
                         const double *spin_of_ray, double *states, double *h,
                         double *lam, int64_t *accepted, const int32_t *order,
                         int64_t n, int64_t n_steps, void *workspace, void *stream);

/* Device workspace bh_propagate_order needs for n rays (256-byte aligned);
 * 0 for n > 2^31 - 1, or when the sort's temporary storage cannot be sized. */
size_t bh_propagate_order_workspace_bytes(int64_t n);

/* Writes into order (n,) int32, on the device, the order in which
 * bh_propagate_ordered should take the rays of states (layout AOS (n,8) or
 * SOA (8,n)): within each segment of 16,384 consecutive rays, inward-moving
 * rays first (x.p < 0), each group by impact parameter |x × p| / |p|; equal
 * keys keep their order.  Deterministic.  A batch streamed in pieces that
 * start at multiples of 16,384 rays gets, piece by piece, the order and
 * hence the results of the single launch. */
int bh_propagate_order(const double *states, int32_t layout, int64_t n, int32_t *order,
                       void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------ adjoint */

/* bh_trace that also records, per ray, the accepted step sizes (h_tape, n x
 * capacity doubles, ray-major) and the float64 state before every
 * checkpoint_every-th accepted step (checkpoints, n x ceil(capacity /
 * checkpoint_every) x 8 doubles).  checkpoint_every in [1, 64].  A ray with
 * more than `capacity` accepted steps makes bh_trace_stats_read return
 * BH_ERR_TAPE.  No counterpart in the reference (which differentiates
 * nothing); the tape is the frozen step sequence its trace took. */
int bh_trace_tape(const bh_trace_config *config, const bh_scene *scene,
                  const double *state0, double *states, int32_t *status,
                  int64_t *steps, int64_t n, double *h_tape, double *checkpoints,
                  int64_t capacity, int32_t checkpoint_every, void *workspace,
                  void *stream);

/* Discrete adjoint of the taped accepted-step sequence: given dL/d(final
 * state) (n,8), writes dL/d(initial state) (n,8) and dL/d(spin) per ray (n,)
 * for the fifth-order DP5 map with the step sizes frozen.  Each segment of
 * checkpoint_every steps is replayed forward from its checkpoint, then swept
 * backward with the stages recomputed (BH_PRECISION_FP64: float64 stage
 * arithmetic; BH_PRECISION_MIXED: float32 stage arithmetic, float64
 * cotangents).  order (device, n, nullable): a permutation of the rays in
 * the order the threads take them; rays sorted by decreasing accepted steps
 * (zero cotangents last) keep each warp's lanes in step.  The results are
 * the same for any order.  No counterpart in the reference. */
int bh_adjoint(int32_t precision, double mass, double spin, const double *h_tape,
               const double *checkpoints, const int64_t *steps, int64_t capacity,
               int32_t checkpoint_every, const double *grad_states,
               double *grad_state0, double *grad_spin, const int64_t *order, int64_t n,
               void *stream);

/* The frozen-sequence map the adjoint differentiates: steps[i] accepted DP5
 * steps of ray i from state0 with the taped sizes, no error control.  Used
 * for finite-difference checks of the adjoint.  No counterpart in the
 * reference. */
int bh_replay(int32_t precision, double mass, double spin, const double *state0,
              const double *h_tape, const int64_t *steps, int64_t capacity,
              double *states, int64_t n, void *stream);

/* ------------------------------------------------------------ shading */

/* imaging.py:27-50 (celestial_checkerboard): RGB (n, 3) uint8 of the checker
 * cell of each unit direction (n, 3), `cells` cells over the polar angle and
 * 2 cells over the azimuth (the reference's default is 12). */
int bh_celestial_checkerboard(const double *directions, int64_t n, int32_t cells,
                              uint8_t *rgb, void *stream);

/* imaging.py:53-91 (render_image): RGB (n, 3) uint8 per traced ray.
 * Captured rays are black; escaped rays take the checkerboard colour of
 * their final spatial coordinate velocity (geodesics.py:98-106), normalised;
 * rays at the step budget are (120, 32, 32); any other status (200, 0, 200).
 * states (n, 8) AoS, 16-byte aligned; spin_of_ray (n,) or NULL for `spin`.
 * For a (height, width) frame in row-major pixel order, rgb is the image. */
int bh_render_image(double mass, double spin, const double *spin_of_ray,
                    const double *states, const int32_t *status, int64_t n,
                    int32_t cells, uint8_t *rgb, void *stream);

/* ------------------------------------------------------------ real-time */

/* Controls of the real-time shader algorithm: realtime/settings.py:70-120
 * (RenderSettings) plus the escape radius and disk of one frame. */
typedef struct {
    int64_t max_steps;       /* fixed-step budget, 1..4096 (interior: capped at 1024) */
    double step_scale;       /* step heuristic gain */
    double min_step, max_step;
    double capture_margin;   /* capture at r <= r_plus (1 + margin) */
    double momentum_bailout; /* |p| at which a ray counts as captured */
    double escape_radius;
    double disk_inner, disk_outer; /* disk_outer <= 0: no disk */
    double interior_stop;    /* > 0: interior camera, rays end at this radius */
    int32_t precision;       /* bh_precision: RK4 stage arithmetic */
    int32_t reserved;        /* 0 */
} bh_realtime_config;

/* realtime/reference.py:41-188 (trace_like_shader): fixed RK4 steps with
 * h = clip(step_scale (r - r_plus), min_step, max_step) (interior cameras:
 * a length min(max(|r - r_plus|, 0.15 r), 0.5 r)), capped at 1/max(1, |p|);
 * capture at the capture radius or when |p| >= momentum_bailout, escape at
 * escape_radius; a step crossing z = 0 is interpolated linearly and ends the
 * ray on the disk when the crossing radius is in [disk_inner, disk_outer].
 * Rays alive after the budget are BH_RAY_MAX_STEPS.  Outputs per ray
 * (device): final states (n, 8) AoS, status, and for DISK rays the crossing
 * radius, position (n, 3) and momentum (n, 4), NaN otherwise.  workspace:
 * bh_trace_workspace_bytes(); bh_trace_stats_read gives the steps taken
 * (attempts = accepted = total, iterations = the longest ray). */
int bh_trace_realtime(const bh_realtime_config *config, double mass, double spin,
                      const double *state0, double *states, int32_t *status,
                      double *hit_radius, double *hit_positions, double *hit_momenta,
                      int64_t n, void *workspace, void *stream);

/* ------------------------------------------------------------ Vaidya surrogate */

/* The charged-Vaidya/Ori mass-inflation surrogate (vaidya.py:87-135): the
 * ChargedVaidyaSpacetime fields and its shell table (advanced time v,
 * shell radius R, inflated mass m2; n_shell rows, v increasing), which
 * bh_vaidya_shell_table integrates on the host and the caller copies to
 * device memory for the device functions below. */
typedef struct {
    double mass, charge, tail_mass, tail_start, tail_power, shell_energy;
    double shell_start_v, shell_start_radius, shell_width, mass_cap;
    const double *shell_v, *shell_r, *shell_m2; /* device, n_shell rows */
    int64_t n_shell;
} bh_vaidya;

/* vaidya.py:181-237 (_integrate_shell): the shell table into HOST arrays of
 * `capacity` rows; returns the number of rows the table has (call with
 * capacity 0 to size it; at most 4,000,001), or -1. */
int64_t bh_vaidya_shell_table(const bh_vaidya *spacetime, double *v, double *r,
                              double *m2, int64_t capacity);

/* vaidya.py:285-325 (geometry_t): per point (t, x, y, z) the potential H,
 * l (n, 3), dH/dx_i = h_spatial_scale l_i, dH/dt and the radius. */
int bh_vaidya_geometry(const bh_vaidya *spacetime, const double *t, const double *x,
                       const double *y, const double *z, int64_t n, double *h,
                       double *l, double *h_spatial_scale, double *h_t,
                       double *radius, void *stream);

/* vaidya.py:260-278: mass function m(v, r) and Misner-Sharp mass
 * m - q^2/(2r); either output may be NULL. */
int bh_vaidya_mass(const bh_vaidya *spacetime, const double *v, const double *r,
                   int64_t n, double *mass, double *misner_sharp, void *stream);

/* vaidya.py:356-394 (vaidya_geodesic_rhs): d(state)/d(lambda), (n, 8). */
int bh_vaidya_rhs(const bh_vaidya *spacetime, const double *states, double *deriv,
                  int64_t n, void *stream);

/* n_steps of rk4_step (integrators.py:57-73) with the surrogate's RHS and a
 * per-ray step h (n,). */
int bh_vaidya_rk4(const bh_vaidya *spacetime, const double *states, const double *h,
                  double *out, int64_t n, int64_t n_steps, void *stream);

/* offline/inflation.py:165-240 (_trace_vaidya_tile): fixed RK4 steps of
 * clip(0.15 L, 3e-3, 0.08) (L = r - r_plus outside, r/2 inside) until the
 * terminal surface (status 1: r <= stop_radius, or r <= 1.08 stop_radius with
 * |p|^2 > 400, or |p|^2 > 1e6; Misner-Sharp mass there in end_mass), escape
 * (status 0: r >= escape_radius; unit direction of p - 2 H lp l on the t = 0
 * slice in escape_dir (n, 3)) or the budget (status 2).  Also the final
 * states and v_end = t + r of every ray.  workspace:
 * bh_trace_workspace_bytes(). */
int bh_vaidya_trace(const bh_vaidya *spacetime, const double *state0, int64_t n,
                    double escape_radius, double stop_radius, int64_t max_steps,
                    double *states, int32_t *status, double *escape_dir,
                    double *end_mass, double *v_end, void *workspace, void *stream);

/* offline/inflation.py:138-162 and 322-346 (the shading of
 * render_layer_frame): per ray of bh_vaidya_trace, status 0 takes the
 * surrogate starfield of its escape direction, status 1 the glow 0.35 +
 * 1.2 log1p(max(end_mass - mass, 0) / mass)^2 times the sheet colour (0.62,
 * 0.78, 1.0), status 2 black; each ray's radiance rounded to float32 and the
 * supersample^2 consecutive rays of a pixel averaged in float32 into hdr
 * (height, width, 3). */
int bh_inflation_radiance(double mass, const int32_t *status, const double *escape_directions,
                          const double *end_mass, int64_t width, int64_t height,
                          int32_t supersample, float *hdr, void *stream);

/* ------------------------------------------------------------ offline tile */

/* Counters of one bh_trace_tile call. */
typedef struct {
    int64_t iterations; /* max attempts over rays */
    int64_t attempts;   /* sum of attempts */
    int64_t accepted;   /* sum of accepted steps */
    int64_t crossings;  /* equatorial crossings refined */
    int64_t disk_hits;  /* rays ended on the disk */
    int32_t rounds;     /* trace + refine rounds */
    int32_t timed_out;  /* 1: rays were left BH_RAY_IN_FLIGHT at the deadline */
} bh_tile_stats;

/* Device workspace of bh_trace_tile for n rays: a 256-byte header, 1 KiB of
 * counters for ordering resumed rays, n crossing records (168 B) and two
 * arrays of n resume records (96 B each). */
size_t bh_trace_tile_workspace_bytes(int64_t n);

/* blackhorizon/offline/render.py:184-309 (_trace_tile) with the crossing
 * refinement of render.py:312-349 (_refine_crossings).  Per ray, before each
 * attempt: captured (r <= scene->capture_radius; BH_TRACE_INTERIOR in
 * config->flags selects the interior-camera rules of that flag),
 * escaped (r >= scene->escape_radius) or out of budget (steps >=
 * config->max_steps, BH_RAY_MAX_STEPS); then one DP5(4) attempt with
 * config->rtol and config->atol (the reference passes atol = rtol * 1e-3);
 * an accepted step whose z changes sign is located on the RK4 substep from
 * the pre-step state at the reference's bisection resolution (fraction
 * (L + 1/2) 2^-40 of the step), and a crossing radius in [disk_inner,
 * disk_outer] ends the ray with BH_RAY_DISK, its state left before the step.
 * disk_outer <= 0 disables crossings.  Rays in flight after 4 max_steps
 * attempts stay BH_RAY_IN_FLIGHT (render.py:223).  config->min_step is not
 * used.  Outputs per ray (device buffers): states (n, 8) in config->layout,
 * status, accepted steps, hit_positions / hit_momenta (n, 3; zero unless
 * DISK), escape_directions (n, 3; render.py:164-181, zero unless ESCAPED),
 * saturated (render.py:289-291: MAX_STEPS or steps >= floor(0.85
 * max_steps)).  The float64 refinement runs between rounds of the
 * persistent tracer, so the call synchronises `stream` once per round and
 * returns when the tile is done; stats may be NULL. */
int bh_trace_tile(const bh_trace_config *config, const bh_scene *scene,
                  double disk_inner, double disk_outer, const double *state0,
                  int64_t n, double *states, int32_t *status, int64_t *steps,
                  double *hit_positions, double *hit_momenta,
                  double *escape_directions, int8_t *saturated,
                  void *workspace, size_t workspace_bytes,
                  bh_tile_stats *stats, void *stream);

/* The real-time viewer's shading uniforms (realtime/engine.py:116-285). */
typedef struct {
    double mass, spin;
    double disk_inner, disk_outer; /* the temperature texture's radius range */
    double disk_temperature;       /* RenderSettings.disk_temperature, K */
    double disk_detail, exposure;
    double observer_lapse;         /* static lapse (exterior) or display amplification (interior) */
    double bb_log_min, bb_log_max; /* log-temperature range of the blackbody texture */
    double sky_amplification;      /* interior cameras: B of the sky shift g = B / E; 0: none */
    double sheet_radiance;         /* glow of captured / terminated rays; 0: black */
    double whiteout;               /* fraction mixed toward (0.90, 0.95, 1.0) */
    int32_t background;            /* 0 checkerboard, 1 starfield */
    int32_t temperature_size;      /* texels of the temperature texture */
    int32_t blackbody_size;        /* texels of the blackbody texture (RGB) */
    int32_t reserved;              /* 0 */
} bh_realtime_shading;

/* The pixel colours of the real-time viewer (realtime/shaders/
 * kerr_tracer.frag:205-420) from bh_trace_realtime's outputs for a
 * (height, width) frame, row 0 at the top: disk emission with the lookup
 * textures sampled linearly with repeat wrapping and the Reinhard curve, the
 * checkerboard or starfield sky by the asymptotic direction (shifted for
 * interior cameras), the blue-sheet glow, the whiteout; 8-bit unsigned
 * normalised RGB.  float32, like the shader.  states (n, 8) final states,
 * hit_positions (n, 3), hit_momenta (n, 4). */
int bh_realtime_shade(const bh_realtime_shading *shading, const int32_t *status,
                      const double *states, const double *hit_positions,
                      const double *hit_momenta, int64_t width, int64_t height,
                      const float *temperature_table, const float *blackbody_table,
                      uint8_t *rgb, void *stream);

/* ------------------------------------------------------ plunge worldline */

/* offline/infall.py:38-91 (radial_momentum): the covariant momentum
 * (p_t, p_x, p_y, p_z) = (-E, w l) of a radial infaller with conserved
 * energy E >= 0 at position[3], the future-directed inward root of the
 * timelike mass shell.  Host computation. */
int bh_radial_momentum(double mass, double spin, const double *position, double energy,
                       double *momentum);

/* offline/infall.py:94-153 (build_plunge): the plunging camera's worldline
 * from (start_radius, 0, 0) with energy E, integrated on the host by RK4 in
 * proper time with step min(step, max(0.04 r^1.5, 1e-6)), the mass shell held
 * at H = -1/2, to r <= stop_radius, the chart's edge or 2,000,000 steps.
 * Writes up to `capacity` samples (proper times taus, states (k, 8)) and
 * returns the number of samples of the whole worldline (call with capacity 0
 * to size it), or -1. */
int64_t bh_plunge_worldline(double mass, double spin, double start_radius, double energy,
                            double stop_radius, double step, int64_t capacity, double *taus,
                            double *states);

/* ---------------------------------------------------- offline camera rays */

/* A camera of the offline renderer and its supersampled pixel grid
 * (render.py:103-161, 520-599). */
typedef struct {
    double position[3];     /* Kerr-Schild camera position */
    double basis[3][3];     /* forward, right, up of a FlyCamera (pinhole mode) */
    double tetrad[4][4];    /* e0..e3 of the observer, one per row (tetrad mode) */
    double tan_half;        /* tan(fov / 2) */
    double tan_half_aspect; /* tan(fov / 2) / (width / height) */
    int64_t width, height;
    int32_t supersample;    /* supersample^2 rays per pixel */
    int32_t use_tetrad;     /* 0: pinhole basis, past-directed null momenta;
                               1: tetrad rays with unit camera frequency */
} bh_offline_camera;

/* The (width height supersample^2, 8) initial states of a frame in pixel-major
 * order (row, column, subpixel row, subpixel column), as render_hdr builds them
 * (render.py:555-599): pinhole grid directions (render.py:103-145), rotated by
 * the basis and given the past-directed null momentum at the camera
 * (geodesics.py:109-170), or taken as local tetrad directions with the traced
 * momentum -g(e0 - n.e) (frames.py:182-218); t = 0. */
int bh_offline_camera_rays(double mass, double spin, const bh_offline_camera *camera,
                           double *states, void *stream);

/* ------------------------------------------------------- offline emission */

/* Shading constants of one offline frame (offline/render.py:487-560). */
typedef struct {
    double mass, spin;
    double disk_inner;        /* ISCO: start of the temperature table, origin of the detail pattern */
    double disk_temperature;  /* OfflineSettings.disk_temperature, K */
    double disk_detail;       /* OfflineSettings.disk_detail */
    double observer_lapse;    /* frequency factor of the camera (static lapse or blue-sheet B) */
    double bb_log_min, bb_log_max; /* log-temperature range of the blackbody table */
    double sheet_rgb[3];      /* radiance of BH_RAY_TERMINATED rays (zero: black) */
    int32_t temperature_size; /* entries of the temperature table (>= 2) */
    int32_t blackbody_size;   /* rows of the blackbody table (>= 2) */
    int32_t supersample;      /* rays per pixel = supersample^2, consecutive */
    int32_t reserved;         /* 0 */
} bh_emission_config;

/* The radiance half of render_hdr (render.py:352-484, 630-680): escaped rays
 * sample the hashed HDR starfield by their escape direction (shifted by
 * observer_lapse / energy[i] when energy, the rays' initial p_t, is given:
 * tetrad cameras); BH_RAY_DISK rays take the redshifted blackbody of the
 * Novikov-Thorne disk at their hit (temperature_table on the radii
 * lut_radii, blackbody_table (blackbody_size, 3) on log temperature);
 * BH_RAY_TERMINATED rays take sheet_rgb; the rest are black.  The
 * supersample^2 rays of each pixel are averaged into hdr (height, width, 3)
 * float32.  Ray arrays are (width height supersample^2[, 3]) in pixel-major
 * order, as bh_trace_tile returns them.  float64 arithmetic in NumPy's order. */
int bh_offline_radiance(const bh_emission_config *config, const int32_t *status,
                        const double *escape_directions, const double *hit_positions,
                        const double *hit_momenta, const double *energy, int64_t width,
                        int64_t height, const float *temperature_table,
                        const double *lut_radii, const float *blackbody_table, float *hdr,
                        void *stream);

/* Device workspace of bh_develop with bloom: two float32 images. */
size_t bh_develop_workspace_bytes(int64_t width, int64_t height);

/* offline/post.py:88-106 (develop): hdr * exposure, bloom (bright pass above
 * bloom_threshold, separable Gaussian blur with edge padding by
 * blur_weights[2 radius + 1], radius <= 6000, added with bloom_strength; skipped when
 * bloom_strength <= 0), ACES filmic curve, sRGB encoding to out (height,
 * width, 3) uint8.  float32 arithmetic in NumPy's order. */
int bh_develop(const float *hdr, int64_t width, int64_t height, double exposure,
               double bloom_threshold, double bloom_strength, const double *blur_weights,
               int32_t blur_radius, uint8_t *out, void *workspace, size_t workspace_bytes,
               void *stream);

/* offline/video.py:33-43 (downsample): each factor x factor block of an 8-bit
 * (height, width, 3) image averaged and truncated to 8 bits into out
 * (height / factor, width / factor, 3); factor in [1, 256]. */
int bh_downsample(const uint8_t *image, int64_t width, int64_t height, int32_t factor,
                  uint8_t *out, void *stream);

/* Device workspace of bh_frame_bloom: three float32 images. */
size_t bh_frame_bloom_workspace_bytes(int64_t width, int64_t height);

/* offline/video.py:46-59 (frame_bloom): the 8-bit frame lifted to
 * (x / 255)^2.2, the bloom of post.py (bright pass above 0.55, separable
 * Gaussian by blur_weights[2 radius + 1]) added with `strength`, clipped and
 * sRGB-encoded into out; strength <= 0 copies the frame.  float32. */
int bh_frame_bloom(const uint8_t *image, int64_t width, int64_t height, double strength,
                   const double *blur_weights, int32_t blur_radius, uint8_t *out,
                   void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------ diagnostics */

/* Launches a vector-FMA throughput kernel of sms*8 blocks x 256 threads, each
 * running iters x 128 FMA instructions: FP64 for BH_PRECISION_FP64, packed
 * float32x2 (two FMAs per instruction) for BH_PEAK_F32X2, else FP32.  *flops
 * receives the launch's FLOP count (FMA = 2).  Timed
 * with events by the caller, it gives the CUDA-core peak that the tracer's
 * roofline fraction is quoted against.  sink: device buffer of >= 8 bytes.
 * No counterpart in the reference (a measurement aid). */
#define BH_PEAK_F32X2 2
int bh_fma_peak_launch(int32_t precision, int64_t iters, void *sink,
                       int64_t *flops, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* BH_B200_H */
