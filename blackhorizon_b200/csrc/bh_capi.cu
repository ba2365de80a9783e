// bh_capi.cu -- extern "C" entry points of libbh_b200.so and the point-wise
// kernels (geometry, RHS, Hamiltonian, velocity, null momentum, camera rays,
// single DP5 / RK4 steps, error ratio, step factor).
//
// Every entry point validates its arguments on the host, launches on the
// caller's stream and returns a bh_status; nothing here allocates device
// memory.  The reference function each one replaces is cited in
// include/bh_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

static thread_local char g_last_error[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

static int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return BH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BH_ERR_CUDA;
}

static int invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

static bool kerr_ok(double mass, double spin) {
    // kerr.py:65-71: mass > 0 and |a| <= M.
    return mass > 0.0 && std::fabs(spin) <= mass && std::isfinite(mass) &&
           std::isfinite(spin);
}

static constexpr int kBlock = 256;

static unsigned grid_for(long long n) {
    long long g = (n + kBlock - 1) / kBlock;
    if (g < 1) g = 1;
    if (g > 0x7fffffffLL) g = 0x7fffffffLL;
    return (unsigned)g;
}

__device__ __forceinline__ long long tid() {
    return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}

// ------------------------------------------------------------ point-wise

__global__ void geometry_kernel(double m, double a, const double *x,
                                const double *y, const double *z,
                                long long stride, long long n, double *r,
                                double *h, double *l, double *gh, double *gl) {
    const long long i = tid();
    if (i >= n) return;
    Geometry g;
    const bool grads = gh != nullptr || gl != nullptr;
    geometry_full(m, a, x[i * stride], y[i * stride], z[i * stride], grads, g);
    if (r) r[i] = g.r;
    if (h) h[i] = g.h;
    if (l) { l[3 * i] = g.l[0]; l[3 * i + 1] = g.l[1]; l[3 * i + 2] = g.l[2]; }
    if (gh) { gh[3 * i] = g.grad_h[0]; gh[3 * i + 1] = g.grad_h[1]; gh[3 * i + 2] = g.grad_h[2]; }
    if (gl) {
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) gl[9 * i + 3 * j + k] = g.grad_l[j][k];
    }
}

__device__ __forceinline__ RayState read_state(const double *s, long long i) {
    const double *p = s + 8 * i;
    RayState y;
    y.t = p[0]; y.x = p[1]; y.y = p[2]; y.z = p[3];
    y.pt = p[4]; y.px = p[5]; y.py = p[6]; y.pz = p[7];
    return y;
}

__device__ __forceinline__ void write_state(double *s, long long i, const RayState &y) {
    double *p = s + 8 * i;
    p[0] = y.t; p[1] = y.x; p[2] = y.y; p[3] = y.z;
    p[4] = y.pt; p[5] = y.px; p[6] = y.py; p[7] = y.pz;
}

__global__ void rhs_kernel(double m, double a, const double *state,
                           double *deriv, long long n) {
    const long long i = tid();
    if (i >= n) return;
    const RayState y = read_state(state, i);
    const KerrV<double> K = make_kerr<double>(m, a);
    WStateV<double> yw;
    put_work<double>(yw, 0, y);
    const StageV<double> d = first_stage<double>(K, yw);
    double *o = deriv + 8 * i;
    o[0] = -y.pt + d.thl;
    o[1] = y.px + d.kx;
    o[2] = y.py + d.ky;
    o[3] = y.pz + d.kz;
    o[4] = 0.0;
    o[5] = d.px; o[6] = d.py; o[7] = d.pz;
}

__global__ void hamiltonian_kernel(double m, double a, const double *state,
                                   double *out, long long n) {
    const long long i = tid();
    if (i >= n) return;
    const RayState y = read_state(state, i);
    Geometry g;
    geometry_full(m, a, y.x, y.y, y.z, false, g);
    const double lp = -y.pt + (g.l[0] * y.px + g.l[1] * y.py + g.l[2] * y.pz);
    const double eta = 0.5 * (-y.pt * y.pt + (y.px * y.px + y.py * y.py + y.pz * y.pz));
    out[i] = eta - g.h * lp * lp;
}

__global__ void velocity_kernel(double m, double a, const double *state,
                                double *out, long long n) {
    const long long i = tid();
    if (i >= n) return;
    const RayState y = read_state(state, i);
    Geometry g;
    geometry_full(m, a, y.x, y.y, y.z, false, g);
    const double lp = -y.pt + (g.l[0] * y.px + g.l[1] * y.py + g.l[2] * y.pz);
    const double thl = 2.0 * g.h * lp;
    double *o = out + 4 * i;
    o[0] = -y.pt + thl;
    o[1] = y.px - thl * g.l[0];
    o[2] = y.py - thl * g.l[1];
    o[3] = y.pz - thl * g.l[2];
}

__global__ void null_momentum_kernel(double m, double a, const double *spins,
                                     const double *pos, const double *dir,
                                     long long n, int past, int normalize,
                                     double *out) {
    const long long i = tid();
    if (i >= n) return;
    const double pp[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    const double dd[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
    double p[4];
    null_momentum(m, spins ? spins[i] : a, pp, dd, past != 0, normalize != 0, p);
    double *o = out + 4 * i;
    o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; o[3] = p[3];
}

__global__ void camera_states_kernel(CameraDev c, double *state, long long n) {
    const long long i = tid();
    if (i >= n) return;
    double d[3], p[4];
    pinhole_direction(c.fwd, c.right, c.up, c.half_w, c.half_h, c.width,
                      c.height, i, d);
    null_momentum(c.mass, c.spin, c.pos, d, true, true, p);
    RayState y;
    y.t = 0.0; y.x = c.pos[0]; y.y = c.pos[1]; y.z = c.pos[2];
    y.pt = p[0]; y.px = p[1]; y.py = p[2]; y.pz = p[3];
    write_state(state, i, y);
}

template <typename V>
__global__ void dp5_kernel(double m, double a, const double *state,
                           const double *h, double *out, double *err,
                           long long n) {
    using T = VT<V>;
    const long long i = tid();
    if (i >= n) return;
    const RayState y = read_state(state, i);
    const KerrV<V> K = make_kerr<V>(T::set(m), T::set(a));
    WStateV<V> yw;
    put_work<V>(yw, 0, y);
    const StageV<V> k1 = first_stage<V>(K, yw);
    const double hh = h[i];
    AttemptV<V> at;
    dp5_attempt<V>(K, yw, T::set(hh), k1, at);
    RayState yn = y;
    commit<V>(yn, yw, at, 0, hh);
    write_state(out, i, yn);
    double *e = err + 8 * i;
    e[0] = hh * double(at.err[0]);
    e[1] = hh * double(at.err[1]);
    e[2] = hh * double(at.err[2]);
    e[3] = hh * double(at.err[3]);
    e[4] = 0.0;
    e[5] = hh * double(at.err[4]);
    e[6] = hh * double(at.err[5]);
    e[7] = hh * double(at.err[6]);
}

// error_ratio (integrators.py:110-117) of arbitrary (n,8) arrays, float64,
// NumPy's pairwise summation order.
__global__ void error_ratio_kernel(const double *s, const double *sn,
                                   const double *err, double rtol, double atol,
                                   double *out, long long n) {
    const long long i = tid();
    if (i >= n) return;
    double q[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const double sc = atol + rtol * np_max(fabs(s[8 * i + j]), fabs(sn[8 * i + j]));
        const double e = err[8 * i + j] / sc;
        q[j] = e * e;
    }
    const double sum = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
    const double r = ::sqrt(sum * 0.125);
    out[i] = isfinite(r) ? r : __longlong_as_double(0x7ff0000000000000LL);
}

__global__ void step_factor_kernel(const double *ratio, double *out, long long n) {
    const long long i = tid();
    if (i >= n) return;
    out[i] = step_factor(ratio[i]);
}

// The device arithmetic that bh_device_math exposes point-wise.
__global__ void device_math_kernel(int op, const double *x, double *out, long long n) {
    const long long i = tid();
    if (i >= n) return;
    const double v = x[i];
    out[i] = op == 0 ? rcp_f64(v) : op == 1 ? rsqrt_f64(v) : step_factor_r2(v);
}

// rk4_step (integrators.py:57-73) n_steps times with the state in registers;
// stage arithmetic in the lane type V, the state update in double.
template <typename V>
__global__ void rk4_kernel(double m, double a, const double *state,
                           const double *hs, double *out, long long n,
                           long long n_steps) {
    using T = VT<V>;
    const long long i = tid();
    if (i >= n) return;
    RayState y = read_state(state, i);
    const double h = hs[i];
    const KerrV<V> K = make_kerr<V>(T::set(m), T::set(a));
    for (long long s = 0; s < n_steps; ++s) rk4_advance<V>(K, y, h);
    write_state(out, i, y);
}

// geodesics.py:42-74 for one state, float64: d(t, x, y, z, p_t, p_x, p_y, p_z).
__device__ __forceinline__ void full_rhs(const KerrV<double> &K, const RayState &y, double d[8]) {
    WStateV<double> yw;
    put_work<double>(yw, 0, y);
    const StageV<double> s = first_stage<double>(K, yw);
    d[0] = -y.pt + s.thl;
    d[1] = y.px + s.kx;
    d[2] = y.py + s.ky;
    d[3] = y.pz + s.kz;
    d[4] = 0.0;
    d[5] = s.px;
    d[6] = s.py;
    d[7] = s.pz;
}

__device__ __forceinline__ RayState add_scaled(const RayState &y, double c, const double d[8]) {
    return RayState{y.t + c * d[0], y.x + c * d[1], y.y + c * d[2], y.z + c * d[3],
                    y.pt + c * d[4], y.px + c * d[5], y.py + c * d[6], y.pz + c * d[7]};
}

// integrators.py:177-207 (implicit_midpoint_step), n_steps times: the
// midpoint y + h/2 f(y) refined `iterations` times by y + h/2 f(midpoint),
// then y + h f(midpoint).
__global__ void midpoint_kernel(double m, double a, const double *state, const double *hs,
                                double *out, long long n, int iterations, long long n_steps) {
    const long long i = tid();
    if (i >= n) return;
    RayState y = read_state(state, i);
    const double h = hs[i];
    const KerrV<double> K = make_kerr<double>(m, a);
    double d[8];
    for (long long s = 0; s < n_steps; ++s) {
        full_rhs(K, y, d);
        RayState mid = add_scaled(y, 0.5 * h, d);
        for (int k = 0; k < iterations; ++k) {
            full_rhs(K, mid, d);
            mid = add_scaled(y, 0.5 * h, d);
        }
        full_rhs(K, mid, d);
        y = add_scaled(y, h, d);
    }
    write_state(out, i, y);
}

static CameraDev camera_dev(const bh_camera &c, long long first_ray) {
    CameraDev d;
    for (int i = 0; i < 3; ++i) {
        d.pos[i] = c.position[i];
        d.fwd[i] = c.forward[i];
        d.right[i] = c.right[i];
        d.up[i] = c.up[i];
    }
    // camera.py:102-103; math.radians(x) is x * (pi / 180).
    d.half_w = std::tan(c.fov_degrees * (M_PI / 180.0) / 2.0);
    d.half_h = d.half_w * double(c.height) / double(c.width);
    d.width = c.width;
    d.height = c.height;
    d.first_ray = first_ray;
    d.mass = c.scene.mass;
    d.spin = c.scene.spin;
    d.capture_radius = c.scene.capture_radius;
    d.escape_radius = c.scene.escape_radius;
    return d;
}

static int camera_ok(const bh_camera &c) {
    if (c.width <= 0 || c.height <= 0) return invalid("image dimensions must be positive");
    if (!(c.fov_degrees > 0.0 && c.fov_degrees < 180.0))
        return invalid("fov_degrees must be in (0, 180)");
    if (!kerr_ok(c.scene.mass, c.scene.spin))
        return invalid("Kerr bound violated or mass not positive");
    return BH_OK;
}

static int config_ok(const bh_trace_config *c) {
    if (!c) return invalid("config is NULL");
    if (c->precision != BH_PRECISION_FP64 && c->precision != BH_PRECISION_MIXED)
        return invalid("precision must be BH_PRECISION_FP64 or BH_PRECISION_MIXED");
    if (c->layout != BH_LAYOUT_AOS && c->layout != BH_LAYOUT_SOA)
        return invalid("layout must be BH_LAYOUT_AOS or BH_LAYOUT_SOA");
    if (!(c->rtol >= 0.0) || !(c->atol >= 0.0) || !(c->rtol > 0.0 || c->atol > 0.0))
        return invalid("rtol and atol must be >= 0 and not both zero");
    if (!(c->initial_step > 0.0) || !(c->max_step > 0.0) || !(c->min_step >= 0.0))
        return invalid("initial_step and max_step must be > 0, min_step >= 0");
    if (c->max_steps < 1 || c->max_steps > (1LL << 60))
        return invalid("max_steps must be in [1, 2^60]");
    if (c->timeout_ns < 0) return invalid("timeout_ns must be >= 0");
    if (c->project_every < 0) return invalid("project_every must be >= 0");
    if (c->flags != 0) return invalid("config flags are accepted by bh_trace_tile only");
    if (c->reserved != 0) return invalid("config reserved field must be 0");
    if (!(c->f64_radius == c->f64_radius)) return invalid("f64_radius must not be NaN");
    return BH_OK;
}

// Trace-family calls (everything but bh_propagate) take no float64 band.
static int trace_config_ok(const bh_trace_config *c) {
    int rc = config_ok(c);
    if (rc != BH_OK) return rc;
    if (c->f64_radius != 0.0) return invalid("f64_radius is accepted by bh_propagate only");
    return BH_OK;
}

static bool aligned(const void *p, size_t a) {
    return (reinterpret_cast<uintptr_t>(p) % a) == 0;
}

static TraceArgs base_args(const bh_trace_config *c) {
    TraceArgs a;
    std::memset(&a, 0, sizeof(a));
    a.rtol = c->rtol;
    a.atol = c->atol;
    a.initial_step = c->initial_step;
    a.max_step = c->max_step;
    a.min_step = c->min_step;
    a.max_steps = c->max_steps;
    a.max_attempts = 4 * c->max_steps;
    a.timeout_ns = c->timeout_ns;
    a.layout = c->layout;
    a.project_every = c->project_every;
    return a;
}


// trace_rays for one scene, optionally recording the accepted-step tape
// (h_tape != nullptr).
int bh_trace_with_tape(const bh_trace_config *config, const bh_scene *scene,
                       const double *state0, double *states, int32_t *status,
                       int64_t *steps, int64_t n, void *workspace, void *stream,
                       double *h_tape, double *ckpt, int64_t tape_cap, int ckpt_every) {
    int rc = trace_config_ok(config);
    if (rc != BH_OK) return rc;
    if (h_tape && config->project_every > 0)
        return invalid("a taped trace cannot project: the adjoint replays unprojected steps");
    if (!scene) return invalid("scene is NULL");
    if (!kerr_ok(scene->mass, scene->spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0) return invalid("n must be >= 0");
    if (!workspace || !aligned(workspace, 256)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    rc = cuda_status(cudaMemsetAsync(workspace, 0, sizeof(TraceWorkspace), s), "bh_trace workspace reset");
    if (rc != BH_OK || n == 0) return rc;
    if (!state0 || !states || !status || !steps) return invalid("NULL pointer argument");
    if (config->layout == BH_LAYOUT_AOS && (!aligned(state0, 16) || !aligned(states, 16)))
        return invalid("state buffers must be 16-byte aligned");
    TraceArgs a = base_args(config);
    a.state0 = state0;
    a.source = 0;
    a.mass = scene->mass;
    a.spin = scene->spin;
    a.capture_radius = scene->capture_radius;
    a.escape_radius = scene->escape_radius;
    a.states = states;
    a.status = status;
    a.steps = steps;
    a.n = n;
    a.ws = reinterpret_cast<TraceWorkspace *>(workspace);
    a.h_tape = h_tape;
    a.ckpt = ckpt;
    a.tape_cap = tape_cap;
    a.ckpt_every = ckpt_every;
    return cuda_status(launch_trace(a, config->precision, config->variant,
                                    config->blocks_per_sm, s),
                       "bh_trace launch");
}

}  // namespace bh

using namespace bh;

extern "C" {

int bh_abi_version(void) { return BH_ABI_VERSION; }

const char *bh_status_string(int status) {
    switch (status) {
        case BH_OK: return "ok";
        case BH_ERR_INVALID_ARGUMENT: return "invalid argument";
        case BH_ERR_CUDA: return "CUDA error";
        case BH_ERR_TIMEOUT: return "trace deadline exceeded";
        case BH_ERR_ESCAPE_RADIUS: return "escape_radius must exceed all initial radii";
        case BH_ERR_WORKSPACE: return "workspace missing, too small or misaligned";
        case BH_ERR_TAPE: return "a ray took more accepted steps than the tape holds";
        default: return "unknown status";
    }
}

const char *bh_last_error(void) { return g_last_error; }

int bh_geometry(double mass, double spin, const double *x, const double *y,
                const double *z, int64_t stride, int64_t n, double *r,
                double *h, double *l, double *grad_h, double *grad_l,
                void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0 || stride < 1) return invalid("n must be >= 0 and stride >= 1");
    if (n == 0) return BH_OK;
    if (!x || !y || !z) return invalid("x, y, z must not be NULL");
    geometry_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
        mass, spin, x, y, z, stride, n, r, h, l, grad_h, grad_l);
    return cuda_status(cudaGetLastError(), "bh_geometry launch");
}

int bh_geodesic_rhs(double mass, double spin, const double *state,
                    double *deriv, int64_t n, void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !deriv) return invalid("state and deriv must not be NULL");
    rhs_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(mass, spin, state, deriv, n);
    return cuda_status(cudaGetLastError(), "bh_geodesic_rhs launch");
}

int bh_hamiltonian(double mass, double spin, const double *state, double *out,
                   int64_t n, void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !out) return invalid("state and out must not be NULL");
    hamiltonian_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(mass, spin, state, out, n);
    return cuda_status(cudaGetLastError(), "bh_hamiltonian launch");
}

int bh_coordinate_velocity(double mass, double spin, const double *state,
                           double *out, int64_t n, void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !out) return invalid("state and out must not be NULL");
    velocity_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(mass, spin, state, out, n);
    return cuda_status(cudaGetLastError(), "bh_coordinate_velocity launch");
}

int bh_null_momentum(double mass, double spin, const double *spin_of_ray,
                     const double *positions, const double *directions,
                     int64_t n, int32_t past, int32_t normalize,
                     double *momenta, void *stream) {
    if (!spin_of_ray && !kerr_ok(mass, spin))
        return invalid("Kerr bound violated or mass not positive");
    if (!(mass > 0.0)) return invalid("mass must be positive");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!positions || !directions || !momenta)
        return invalid("positions, directions and momenta must not be NULL");
    null_momentum_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
        mass, spin, spin_of_ray, positions, directions, n, past, normalize, momenta);
    return cuda_status(cudaGetLastError(), "bh_null_momentum launch");
}

int bh_camera_states(const bh_camera *camera, double *state, void *stream) {
    if (!camera) return invalid("camera is NULL");
    int rc = camera_ok(*camera);
    if (rc != BH_OK) return rc;
    if (!state) return invalid("state must not be NULL");
    const long long n = camera->width * camera->height;
    camera_states_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
        camera_dev(*camera, 0), state, n);
    return cuda_status(cudaGetLastError(), "bh_camera_states launch");
}

int bh_dp5_step(double mass, double spin, const double *state,
                const double *h, double *new_state, double *error, int64_t n,
                int32_t precision, void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !h || !new_state || !error) return invalid("NULL pointer argument");
    if (precision == BH_PRECISION_FP64)
        dp5_kernel<double><<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
            mass, spin, state, h, new_state, error, n);
    else if (precision == BH_PRECISION_MIXED)
        dp5_kernel<float><<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
            mass, spin, state, h, new_state, error, n);
    else
        return invalid("unknown precision");
    return cuda_status(cudaGetLastError(), "bh_dp5_step launch");
}

int bh_error_ratio(const double *state, const double *new_state,
                   const double *error, double rtol, double atol,
                   double *ratio, int64_t n, void *stream) {
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !new_state || !error || !ratio) return invalid("NULL pointer argument");
    error_ratio_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
        state, new_state, error, rtol, atol, ratio, n);
    return cuda_status(cudaGetLastError(), "bh_error_ratio launch");
}

int bh_step_factor(const double *ratio, double *factor, int64_t n, void *stream) {
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!ratio || !factor) return invalid("NULL pointer argument");
    step_factor_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(ratio, factor, n);
    return cuda_status(cudaGetLastError(), "bh_step_factor launch");
}

int bh_device_math(int32_t op, const double *x, double *y, int64_t n, void *stream) {
    if (op < 0 || op > 2) return invalid("op must be 0 (rcp), 1 (rsqrt) or 2 (step factor of r^2)");
    if (n < 0) return invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!x || !y) return invalid("NULL pointer argument");
    device_math_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(op, x, y, n);
    return cuda_status(cudaGetLastError(), "bh_device_math launch");
}

int bh_rk4(double mass, double spin, const double *state, const double *h,
           double *new_state, int64_t n, int64_t n_steps, int32_t precision,
           void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0 || n_steps < 0) return invalid("n and n_steps must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !h || !new_state) return invalid("NULL pointer argument");
    if (precision == BH_PRECISION_FP64)
        rk4_kernel<double><<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
            mass, spin, state, h, new_state, n, n_steps);
    else if (precision == BH_PRECISION_MIXED)
        rk4_kernel<float><<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
            mass, spin, state, h, new_state, n, n_steps);
    else
        return invalid("unknown precision");
    return cuda_status(cudaGetLastError(), "bh_rk4 launch");
}

int bh_implicit_midpoint(double mass, double spin, const double *state, const double *h,
                         double *new_state, int64_t n, int32_t iterations, int64_t n_steps,
                         void *stream) {
    if (!kerr_ok(mass, spin)) return invalid("Kerr bound violated or mass not positive");
    if (n < 0 || n_steps < 0 || iterations < 0)
        return invalid("n, n_steps and iterations must be >= 0");
    if (n == 0) return BH_OK;
    if (!state || !h || !new_state) return invalid("NULL pointer argument");
    midpoint_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(
        mass, spin, state, h, new_state, n, iterations, n_steps);
    return cuda_status(cudaGetLastError(), "bh_implicit_midpoint launch");
}

int bh_trace_variant_count(int32_t precision) { return trace_variant_count(precision); }

int bh_trace_variant(int32_t precision, int32_t index, int32_t *block_threads,
                     int32_t *min_blocks, int32_t *rays_per_thread,
                     int32_t *registers, int32_t *max_blocks_per_sm) {
    if (precision != BH_PRECISION_FP64 && precision != BH_PRECISION_MIXED)
        return invalid("unknown precision");
    if (index < 0) index = trace_default_variant(precision);
    if (index >= trace_variant_count(precision)) return invalid("variant index out of range");
    const Variant v = trace_variant(precision, index);
    if (block_threads) *block_threads = v.block;
    if (min_blocks) *min_blocks = v.min_blocks;
    if (rays_per_thread) *rays_per_thread = v.rays_per_thread;
    int regs = 0, nb = 0;
    if (kernel_attributes(false, precision, index, &regs, &nb) != 0)
        return cuda_status(cudaGetLastError(), "bh_trace_variant attributes");
    if (registers) *registers = regs;
    if (max_blocks_per_sm) *max_blocks_per_sm = nb;
    return BH_OK;
}

size_t bh_trace_workspace_bytes(void) { return sizeof(TraceWorkspace); }

size_t bh_trace_cameras_workspace_bytes(int32_t ncameras) {
    if (ncameras < 0) ncameras = 0;
    const size_t bytes = sizeof(TraceWorkspace) + size_t(ncameras) * sizeof(CameraDev);
    return (bytes + 255) / 256 * 256;
}

int bh_trace(const bh_trace_config *config, const bh_scene *scene,
             const double *state0, double *states, int32_t *status,
             int64_t *steps, int64_t n, void *workspace, void *stream) {
    return bh_trace_with_tape(config, scene, state0, states, status, steps, n, workspace,
                              stream, nullptr, nullptr, 0, 1);
}

int bh_camera_table_upload(const bh_camera *cameras, int32_t ncameras,
                           void *workspace, size_t workspace_bytes,
                           int64_t *n_rays, void *stream) {
    if (ncameras < 1 || !cameras) return invalid("need at least one camera");
    if (!workspace || !aligned(workspace, 256) ||
        workspace_bytes < bh_trace_cameras_workspace_bytes(ncameras)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_cameras_workspace_bytes(ncameras)");
        return BH_ERR_WORKSPACE;
    }
    CameraDev *table = new CameraDev[ncameras];
    long long total = 0;
    for (int c = 0; c < ncameras; ++c) {
        const int rc = camera_ok(cameras[c]);
        if (rc != BH_OK) {
            delete[] table;
            return rc;
        }
        table[c] = camera_dev(cameras[c], total);
        total += cameras[c].width * cameras[c].height;
    }
    char *ws = reinterpret_cast<char *>(workspace);
    // A copy from pageable memory returns once the runtime has staged the
    // source, so the table can be freed right after.
    const int rc = cuda_status(
        cudaMemcpyAsync(ws + sizeof(TraceWorkspace), table, sizeof(CameraDev) * ncameras,
                        cudaMemcpyHostToDevice, (cudaStream_t)stream),
        "bh_camera_table_upload copy");
    delete[] table;
    if (rc == BH_OK && n_rays) *n_rays = total;
    return rc;
}

int bh_trace_cameras(const bh_trace_config *config, int32_t ncameras,
                     int64_t n_rays, double *states, int32_t *status,
                     int64_t *steps, void *workspace, size_t workspace_bytes,
                     void *stream) {
    int rc = trace_config_ok(config);
    if (rc != BH_OK) return rc;
    if (ncameras < 1) return invalid("need at least one camera");
    if (n_rays < 0) return invalid("n_rays must be >= 0");
    if (!workspace || !aligned(workspace, 256) ||
        workspace_bytes < bh_trace_cameras_workspace_bytes(ncameras)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_cameras_workspace_bytes(ncameras)");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    rc = cuda_status(cudaMemsetAsync(workspace, 0, sizeof(TraceWorkspace), s),
                     "bh_trace_cameras workspace reset");
    if (rc != BH_OK || n_rays == 0) return rc;
    if (!states || !status || !steps) return invalid("NULL pointer argument");
    if (config->layout == BH_LAYOUT_AOS && !aligned(states, 16))
        return invalid("state buffers must be 16-byte aligned");
    TraceArgs a = base_args(config);
    a.source = 1;
    a.cameras = reinterpret_cast<const CameraDev *>(
        reinterpret_cast<char *>(workspace) + sizeof(TraceWorkspace));
    a.ncameras = ncameras;
    a.states = states;
    a.status = status;
    a.steps = steps;
    a.n = n_rays;
    a.ws = reinterpret_cast<TraceWorkspace *>(workspace);
    return cuda_status(launch_trace(a, config->precision, config->variant,
                                    config->blocks_per_sm, s),
                       "bh_trace_cameras launch");
}

int bh_trace_stats_read(const void *workspace, bh_trace_stats *out, void *stream) {
    if (!workspace || !out) return invalid("NULL pointer argument");
    TraceWorkspace w;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = cuda_status(cudaMemcpyAsync(&w, workspace, sizeof(w), cudaMemcpyDeviceToHost, s),
                         "bh_trace_stats_read copy");
    if (rc != BH_OK) return rc;
    rc = cuda_status(cudaStreamSynchronize(s), "bh_trace_stats_read sync");
    if (rc != BH_OK) return rc;
    out->iterations = w.iterations;
    out->attempts = (int64_t)w.attempts;
    out->accepted = (int64_t)w.accepted;
    out->timed_out = w.timed_out;
    out->bad_rays = w.bad_rays;
    if (w.bad_rays) {
        set_error("escape_radius must exceed all initial radii (%d rays)", w.bad_rays);
        return BH_ERR_ESCAPE_RADIUS;
    }
    if (w.bad_spins) {
        set_error("Kerr bound violated: |spin| must be <= mass (%d rays)", w.bad_spins);
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (w.bad_order) {
        set_error("order is not a permutation of [0, n) (%d entries out of range)", w.bad_order);
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (w.timed_out) {
        set_error("trace deadline exceeded");
        return BH_ERR_TIMEOUT;
    }
    if (w.tape_overflow) {
        set_error("a ray took more accepted steps than the tape capacity");
        return BH_ERR_TAPE;
    }
    return BH_OK;
}

int bh_propagate(const bh_trace_config *config, double mass, double spin,
                 const double *spin_of_ray, double *states, double *h,
                 double *lam, int64_t *accepted, int64_t n, int64_t n_steps,
                 void *workspace, void *stream) {
    return bh_propagate_ordered(config, mass, spin, spin_of_ray, states, h, lam, accepted,
                                nullptr, n, n_steps, workspace, stream);
}

int bh_propagate_ordered(const bh_trace_config *config, double mass, double spin,
                         const double *spin_of_ray, double *states, double *h, double *lam,
                         int64_t *accepted, const int32_t *order, int64_t n, int64_t n_steps,
                         void *workspace, void *stream) {
    int rc = config_ok(config);
    if (rc != BH_OK) return rc;
    if (config->f64_radius != 0.0 && config->project_every > 0)
        return invalid("f64_radius and project_every cannot be combined");
    if (!(mass > 0.0)) return invalid("mass must be positive");
    if (!spin_of_ray && !kerr_ok(mass, spin)) return invalid("Kerr bound violated");
    if (n < 0 || n_steps < 0) return invalid("n and n_steps must be >= 0");
    if (!workspace || !aligned(workspace, 256)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    rc = cuda_status(cudaMemsetAsync(workspace, 0, sizeof(TraceWorkspace), s), "bh_propagate workspace reset");
    if (rc != BH_OK || n == 0) return rc;
    if (!states || !h || !accepted) return invalid("NULL pointer argument");
    if (config->layout == BH_LAYOUT_AOS && !aligned(states, 16))
        return invalid("state buffers must be 16-byte aligned");
    TraceArgs a = base_args(config);
    if (config->precision == BH_PRECISION_MIXED && config->f64_radius != 0.0) {
        // 8 u M / rtol: the radius where float32 rounding of the curvature
        // terms (about 4 u of their relative size 2 M / r) reaches rtol.
        const double radius = config->f64_radius > 0.0
                                  ? config->f64_radius
                                  : (config->rtol > 0.0 ? 8.0 * 0x1p-24 * mass / config->rtol
                                                        : 1e150);
        a.f64_r2 = fmin(radius, 1e150) * fmin(radius, 1e150);
    }
    a.state0 = states;
    a.states = states;
    a.mass = mass;
    a.spin = spin;
    a.spin_of_ray = spin_of_ray;
    a.order = order;
    a.h_io = h;
    a.lam_io = lam;
    a.steps = accepted;
    a.n = n;
    a.max_attempts = n_steps;
    a.ws = reinterpret_cast<TraceWorkspace *>(workspace);
    return cuda_status(launch_propagate(a, config->precision, config->variant,
                                        config->blocks_per_sm, s),
                       "bh_propagate launch");
}

}  // extern "C"

// ------------------------------------------------------------ CUDA graph
// A captured multi-camera trace: the counter reset and the persistent launch
// of bh_trace_cameras recorded once into a CUDA graph and replayed by
// bh_graph_launch with one call.

struct bh_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

extern "C" int bh_graph_trace_cameras(const bh_trace_config *config,
                                      int32_t ncameras, int64_t n_rays,
                                      double *states, int32_t *status,
                                      int64_t *steps, void *workspace,
                                      size_t workspace_bytes, bh_graph **out) {
    if (!out) return invalid("out is NULL");
    *out = nullptr;
    cudaStream_t cap = nullptr;
    int rc = cuda_status(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking),
                         "bh_graph_trace_cameras stream");
    if (rc != BH_OK) return rc;
    rc = cuda_status(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal),
                     "bh_graph_trace_cameras begin capture");
    if (rc != BH_OK) {
        cudaStreamDestroy(cap);
        return rc;
    }
    const int launch_rc = bh_trace_cameras(config, ncameras, n_rays, states, status, steps,
                                           workspace, workspace_bytes, cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (launch_rc != BH_OK) {
        if (graph) cudaGraphDestroy(graph);
        return launch_rc;
    }
    rc = cuda_status(end, "bh_graph_trace_cameras end capture");
    if (rc != BH_OK) return rc;
    cudaGraphExec_t exec = nullptr;
    rc = cuda_status(cudaGraphInstantiate(&exec, graph, 0), "bh_graph_trace_cameras instantiate");
    if (rc != BH_OK) {
        cudaGraphDestroy(graph);
        return rc;
    }
    *out = new bh_graph{graph, exec};
    return BH_OK;
}

extern "C" int bh_graph_launch(bh_graph *g, void *stream) {
    if (!g) return invalid("graph is NULL");
    return cuda_status(cudaGraphLaunch(g->exec, (cudaStream_t)stream), "bh_graph_launch");
}

extern "C" int bh_graph_destroy(bh_graph *g) {
    if (!g) return BH_OK;
    cudaError_t e1 = cudaGraphExecDestroy(g->exec);
    cudaError_t e2 = cudaGraphDestroy(g->graph);
    delete g;
    const int rc = cuda_status(e1, "bh_graph_destroy exec");
    return rc != BH_OK ? rc : cuda_status(e2, "bh_graph_destroy graph");
}

// ------------------------------------------------------------ no-alloc
// bh_trace_cameras_noalloc: the multi-camera trace for callers that cannot
// allocate device memory themselves -- for example a host application that
// owns every byte of GPU memory through its own fixed-size pool and hands
// this library only its output buffers, or code that runs under a hard
// memory budget where an extra cudaMalloc could fail or synchronise the
// device.  Such a caller cannot supply the workspace bh_trace_cameras needs
// (launch counters, work-queue head and camera table), so this variant keeps
// that scratch in one static device array: kNoAllocMaxCameras cameras at
// most, 256 + 256 * sizeof(CameraDev) bytes, resident on every GPU that loads
// the library until the process exits.
#include <mutex>

namespace bh {

constexpr int kNoAllocMaxCameras = 256;
constexpr size_t kNoAllocBytes =
    sizeof(TraceWorkspace) + size_t(kNoAllocMaxCameras) * sizeof(CameraDev);
constexpr int kNoAllocMaxDevices = 64;

// The scratch itself.  Host code must not use this name as a device address:
// on the host it is only a stand-in for the symbol.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device with that device current.
static int noalloc_scratch(void **out) {
    int dev = 0;
    int rc = cuda_status(cudaGetDevice(&dev), "bh_trace_cameras_noalloc device");
    if (rc != BH_OK) return rc;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return invalid("device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        rc = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                         "bh_trace_cameras_noalloc scratch address");
        if (rc != BH_OK) return rc;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return BH_OK;
}

}  // namespace bh

extern "C" int bh_trace_cameras_noalloc(const bh_trace_config *config,
                                        const bh_camera *cameras,
                                        int32_t ncameras, double *states,
                                        int32_t *status, int64_t *steps,
                                        bh_trace_stats *stats, void *stream) {
    int rc = trace_config_ok(config);
    if (rc != BH_OK) return rc;
    if (ncameras < 1 || !cameras) return invalid("need at least one camera");
    if (ncameras > kNoAllocMaxCameras) {
        set_error("bh_trace_cameras_noalloc takes at most %d cameras (got %d); "
                  "use bh_trace_cameras with a caller-owned workspace",
                  kNoAllocMaxCameras, ncameras);
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (!states || !status || !steps) return invalid("NULL pointer argument");
    if (config->layout == BH_LAYOUT_AOS && !aligned(states, 16))
        return invalid("state buffers must be 16-byte aligned");
    // The camera table is built on the host stack: no heap allocation.
    CameraDev table[kNoAllocMaxCameras];
    long long total = 0;
    for (int c = 0; c < ncameras; ++c) {
        rc = camera_ok(cameras[c]);
        if (rc != BH_OK) return rc;
        table[c] = camera_dev(cameras[c], total);
        total += cameras[c].width * cameras[c].height;
    }
    void *scratch = nullptr;
    rc = noalloc_scratch(&scratch);
    if (rc != BH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    char *base = reinterpret_cast<char *>(scratch);
    // Counters and queue head start at zero on every call; the previous
    // call's camera table is overwritten below.
    rc = cuda_status(cudaMemsetAsync(base, 0, sizeof(TraceWorkspace), s),
                     "bh_trace_cameras_noalloc reset");
    if (rc != BH_OK) return rc;
    rc = cuda_status(cudaMemcpyAsync(base + sizeof(TraceWorkspace), table,
                                     sizeof(CameraDev) * ncameras,
                                     cudaMemcpyHostToDevice, s),
                     "bh_trace_cameras_noalloc table upload");
    if (rc != BH_OK) return rc;
    TraceArgs a = base_args(config);
    a.source = 1;
    a.cameras = reinterpret_cast<const CameraDev *>(base + sizeof(TraceWorkspace));
    a.ncameras = ncameras;
    a.states = states;
    a.status = status;
    a.steps = steps;
    a.n = total;
    a.ws = reinterpret_cast<TraceWorkspace *>(base);
    rc = cuda_status(launch_trace(a, config->precision, config->variant,
                                  config->blocks_per_sm, s),
                     "bh_trace_cameras_noalloc launch");
    if (rc != BH_OK) return rc;
    bh_trace_stats local;
    return bh_trace_stats_read(scratch, stats ? stats : &local, stream);
}
