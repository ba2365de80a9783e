/*
 * bh_oracle.h -- CPU restatement of BlackHorizon's geodesic hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This header and bh_oracle.c are the oracle that
 * the parity tests, the smoke check and the CPU-baseline leg of the benchmark
 * compare the CUDA library against.  Nothing in the product path
 * (blackhorizon_b200/) may include, link or call it.
 *
 * Every function restates one reference function operation for operation
 * (same association order as the NumPy expressions, no FMA contraction) so
 * that results agree with the reference to the last bit wherever libm and
 * NumPy agree; the one known source of ulp-level difference is pow() in the
 * step-size factor (NumPy may use a SIMD pow).  Citations are to files of the
 * reference project (MegaKruk/BlackHorizon).
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Ray status codes: blackhorizon/tracer.py:21-30 (RayStatus). */
enum {
    BHO_IN_FLIGHT = 0,
    BHO_CAPTURED = 1,
    BHO_ESCAPED = 2,
    BHO_MAX_STEPS = 3,
    BHO_FAILED = 4
};

/* Kerr-Schild geometry at one point: blackhorizon/kerr.py:32-49.
 * grad_l[i][j] = d l_j / d x_i. */
typedef struct {
    double r, h;
    double l[3];
    double grad_h[3];
    double grad_l[3][3];
} bho_geometry_t;

/* Tracer controls: keyword arguments of blackhorizon/tracer.py:50-61. */
typedef struct {
    double mass, spin;
    double escape_radius;
    int64_t max_steps;
    double rtol, atol, initial_step, max_step, min_step, capture_margin;
} bho_trace_params_t;

/* kerr.py:118-193 (KerrSpacetime.geometry). */
void bho_geometry(double m, double a, double x, double y, double z,
                  int gradients, bho_geometry_t *out);

/* geodesics.py:42-74 (geodesic_rhs) for one state. */
void bho_rhs(double m, double a, const double s[8], double d[8]);

/* geodesics.py:77-85 (hamiltonian). */
double bho_hamiltonian(double m, double a, const double s[8]);

/* geodesics.py:95-106 (coordinate_velocity). */
void bho_coordinate_velocity(double m, double a, const double s[8], double v[4]);

/* geodesics.py:109-170 (null_momentum_from_velocity); past != 0 selects the
 * past-directed root. */
void bho_null_momentum(double m, double a, const double pos[3],
                       const double dir[3], int past, int normalize,
                       double p[4]);

/* integrators.py:76-107 (dormand_prince_step), autonomous form, k7 recomputed. */
void bho_dp5_step(double m, double a, const double y[8], double h,
                  double y_new[8], double err[8]);

/* integrators.py:110-117 (error_ratio) for one 8-component state. */
double bho_error_ratio(const double y[8], const double y_new[8],
                       const double err[8], double rtol, double atol);

/* integrators.py:120-124 (step_factor). */
double bho_step_factor(double ratio);

/* integrators.py:57-73 (rk4_step). */
void bho_rk4_step(double m, double a, const double y[8], double h,
                  double y_new[8]);

/* camera.py:96-113 (PinholeCamera.ray_directions) given the basis that
 * camera.py:48-66 builds; dirs is (height*width, 3), row-major from the
 * top-left pixel. */
void bho_pinhole_directions(const double forward[3], const double right[3],
                            const double up[3], double fov_degrees,
                            int64_t width, int64_t height, double *dirs);

/* tracer.py:50-157 (trace_rays) for a batch; each ray runs the reference's
 * per-iteration body until it leaves IN_FLIGHT or the batch-global cap of
 * 4*max_steps iterations.  states (n,8) is updated in place.  Returns the
 * reference's `iterations` (max attempts over rays), or -1 when an initial
 * radius is at or beyond escape_radius (the reference raises ValueError).
 * nthreads <= 0 uses one thread per online core. */
int64_t bho_trace_batch(const bho_trace_params_t *p, double *states,
                        int32_t *status, int64_t *steps, int64_t n,
                        int nthreads);

/* Lock-step adaptive propagation without termination: n_steps attempted
 * DP5(4) steps per ray with the tracer's accept/reject and step update
 * (tracer.py:111-120).  spin may be per ray (spins != NULL).  states (n,8)
 * updated in place; accepted (n,) receives accepted-step counts; h (n,) holds
 * the step size in and out. */
void bho_propagate_batch(double mass, double spin, const double *spins,
                         double *states, double *h, int64_t *accepted,
                         int64_t n, int64_t n_steps, double rtol, double atol,
                         double max_step, int nthreads);

/* Status of a ray that hit the accretion disk: tracer.py:28 (RayStatus.DISK). */
#define BHO_DISK 5

/* offline/render.py:184-309 (_trace_tile), with the
 * equatorial-disk refinement of render.py:312-349 (_refine_crossings): the
 * termination test comes before each step, the error scale uses atol =
 * rtol * 1e-3, and an accepted step whose z changes sign is bisected 40
 * times along RK4 substeps; a crossing radius in [disk_inner, disk_outer]
 * ends the ray with BHO_DISK.  disk_outer <= 0 disables the disk.
 * interior_stop > 0 selects the interior-camera mode (render.py:203-248):
 * rays end with BHO_TERMINATED at r <= interior_stop, when the spatial
 * momentum norm exceeds 1e3, or at r <= 1.002 interior_stop with a norm
 * above 50; else capture is at r_plus (1 + capture_margin).  Rays still
 * in flight after 4*max_steps iterations keep BHO_IN_FLIGHT.  Outputs per
 * ray: status, accepted steps, final state (n,8; the pre-crossing state for
 * disk hits), hit position/momentum (n,3 each, zero unless DISK), escape
 * direction (n,3, render.py:164-181, zero unless ESCAPED) and the
 * saturation flag (MAX_STEPS or steps >= int(0.85 max_steps)). */
void bho_trace_tile(const bho_trace_params_t *p, double disk_inner,
                    double disk_outer, double interior_stop, double *states,
                    int32_t *status, int64_t *steps, double *hit_pos,
                    double *hit_mom, double *escape_dir, int32_t *saturated,
                    int64_t n, int nthreads);

/* imaging.py:27-50 (celestial_checkerboard): RGB of the checker cell of each
 * unit direction (n,3), `cells` cells over the polar angle. */
void bho_celestial_checkerboard(const double *dirs, int64_t n, int cells,
                                uint8_t *rgb);

/* imaging.py:53-91 (render_image): per ray, black if captured, the
 * checkerboard colour of the final coordinate-velocity direction if
 * escaped, dark red at the step budget, magenta otherwise; rgb (n,3). */
void bho_render_image(double m, double a, const double *states,
                      const int32_t *status, int64_t n, int cells, uint8_t *rgb);

/* Controls of the real-time shader algorithm (realtime/settings.py:70-120). */
typedef struct {
    double mass, spin, escape_radius;
    int64_t max_steps;
    double step_scale, min_step, max_step, capture_margin, momentum_bailout;
    double disk_inner, disk_outer; /* disk_outer <= 0: no disk */
    double interior_stop;          /* > 0: interior camera mode */
} bho_realtime_params_t;

/* Status of a ray that reached the interior stop radius: tracer.py:29. */
#define BHO_TERMINATED 6

/* realtime/reference.py:41-188 (trace_like_shader) per ray: fixed RK4 steps
 * with the distance heuristic, momentum bail-out, linear disk crossings.
 * states (n,8) in/out (final states; DISK rays keep the crossing step's end
 * state), status (n,), hit radius (n,) and hit position (n,3) / momentum
 * (n,4) (NaN unless DISK). */
void bho_trace_realtime(const bho_realtime_params_t *p, double *states,
                        int32_t *status, double *hit_radius, double *hit_pos,
                        double *hit_mom, int64_t n, int nthreads);

/* ------------------------------------------------------------ vaidya.py */

/* The charged-Vaidya/Ori surrogate (vaidya.py:87-330): parameters and its
 * co-integrated shell table (v, R, m2). */
typedef struct {
    double mass, charge, tail_mass, tail_start, tail_power, shell_energy,
        shell_start_v, shell_start_radius, shell_width, mass_cap;
    const double *shell_v, *shell_r, *shell_m2;
    int64_t n_shell;
} bho_vaidya_t;

/* vaidya.py:181-237 (_integrate_shell): writes up to `capacity` table rows
 * and returns the row count. */
int64_t bho_vaidya_shell(const bho_vaidya_t *p, double *v, double *r, double *m2,
                         int64_t capacity);

/* vaidya.py:260-278: mass function m(v, r) and Misner-Sharp mass. */
double bho_vaidya_mass(const bho_vaidya_t *p, double v, double r);
double bho_vaidya_misner_sharp(const bho_vaidya_t *p, double v, double r);

/* vaidya.py:285-325 (geometry_t): H, l, dH/dx_i = hs l_i, dH/dt, radius. */
void bho_vaidya_geometry(const bho_vaidya_t *p, double t, double x, double y, double z,
                         double *h, double l[3], double *hs, double *ht, double *radius);

/* vaidya.py:356-394 (vaidya_geodesic_rhs). */
void bho_vaidya_rhs(const bho_vaidya_t *p, const double y[8], double out[8]);

/* n_steps of rk4_step (integrators.py:57-73) with the surrogate's RHS, fixed h. */
void bho_vaidya_rk4(const bho_vaidya_t *p, double *states, int64_t n, int64_t n_steps,
                    double h);

/* offline/inflation.py:165-240 (_trace_vaidya_tile) per ray: status 0 escaped,
 * 1 terminal surface, 2 budget; escape direction (n,3), Misner-Sharp mass at
 * the terminal point, advanced time v = t + r of the final state. */
void bho_vaidya_trace(const bho_vaidya_t *p, double *states, int64_t n,
                      double escape_radius, double stop_radius, int64_t max_steps,
                      int32_t *status, double *escape_dir, double *end_mass,
                      double *v_end, int nthreads);

/* integrate_dense (integrators.py:127-174) per ray: adaptive DP5(4) from
 * affine parameter 0 to lam_target[i], the last step cut to land on it.
 * Rays that exhaust max_attempts or underflow the step get NaN states.
 * attempts (n,) may be NULL. */
void bho_propagate_to(double mass, double spin, const double *spins,
                      double *states, const double *lam_target,
                      int64_t *attempts, int64_t n, double rtol, double atol,
                      double initial_step, double max_step,
                      int64_t max_attempts, int nthreads);

/* Fixed-step RK4 for a batch (examples/benchmark.py:39-51). */
void bho_rk4_batch(double mass, double spin, double *states, int64_t n,
                   int64_t n_steps, double h, int nthreads);

/* Batched point-wise helpers used by the parity tests. */
void bho_geometry_batch(double m, double a, const double *xyz, int64_t n,
                        double *r, double *h, double *l, double *grad_h,
                        double *grad_l);
void bho_rhs_batch(double m, double a, const double *states, int64_t n,
                   double *deriv);
void bho_dp5_batch(double m, double a, const double *states, const double *h,
                   int64_t n, double *y_new, double *err, double *ratio,
                   double rtol, double atol);
void bho_null_momentum_batch(double m, double a, const double *pos,
                             const double *dir, int64_t n, int past,
                             int normalize, double *p);

int bho_num_threads(void);

/* Shading constants of offline/render.py:487-560 for bho_offline_radiance. */
typedef struct {
    double mass, spin, disk_inner, disk_temperature, disk_detail, observer_lapse;
    double bb_log_min, bb_log_max;
    double sheet_rgb[3];
    int32_t temperature_size, blackbody_size, supersample;
} bho_emission_params_t;

/* render.py:352-419 (_starfield_hdr) per direction (n,3) -> rgb (n,3);
 * shift (n,) or NULL. */
void bho_starfield(const double *dirs, const double *shift, int64_t n, double *rgb);

/* render.py:422-484 (_disk_radiance) per hit (positions, momenta (n,3)). */
void bho_disk_radiance(const bho_emission_params_t *p, const double *pos,
                       const double *mom, int64_t n, const float *temperature,
                       const double *lut_radii, const float *bb_table, double *rgb);

/* The shading of render_hdr (render.py:630-680): per-ray radiance by status
 * (starfield with shift observer_lapse / energy[i] when energy != NULL,
 * disk, sheet_rgb for TERMINATED, else black), averaged over the
 * supersample^2 consecutive rays of each pixel into hdr (pixels, 3) float32. */
void bho_offline_radiance(const bho_emission_params_t *p, const int32_t *status,
                          const double *escape_dir, const double *hit_pos,
                          const double *hit_mom, const double *energy,
                          int64_t pixels, const float *temperature,
                          const double *lut_radii, const float *bb_table,
                          float *hdr, int nthreads);

/* The real-time viewer's shading uniforms (realtime/engine.py:235-285). */
typedef struct {
    float mass, spin, disk_inner, disk_outer, disk_temperature, disk_detail;
    float exposure, observer_lapse, bb_log_min, bb_log_max;
    float sky_amplification, sheet_radiance, whiteout;
    int32_t background, temperature_size, blackbody_size;
} bho_realtime_shading_t;

/* realtime/shaders/kerr_tracer.frag:205-420: the 8-bit pixel colour of each
 * traced ray (status, final state (n,8), hit position (n,3), hit momentum
 * (n,4)) in float32 as the shader computes it. */
void bho_realtime_shade(const bho_realtime_shading_t *p, const int32_t *status,
                        const double *states, const double *hit_pos,
                        const double *hit_mom, int64_t n, const float *temperature,
                        const float *blackbody, uint8_t *rgb);

/* offline/inflation.py:138-162, 322-346: the shading of render_layer_frame
 * (surrogate sky, layer glow, black) averaged over supersample^2 consecutive
 * rays per pixel in float32, into hdr (pixels, 3). */
void bho_inflation_radiance(double mass, const int32_t *status, const double *escape_dir,
                            const double *end_mass, int64_t pixels, int supersample,
                            float *hdr);

/* offline/post.py:88-106 (develop) on an (height, width, 3) float32 image;
 * weights (2 radius + 1) are gaussian_kernel(sigma); bloom_strength <= 0
 * skips the bloom. */
void bho_develop(const float *hdr, int64_t width, int64_t height, double exposure,
                 double bloom_threshold, double bloom_strength,
                 const double *weights, int radius, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
