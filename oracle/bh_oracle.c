/*
 * bh_oracle.c -- CPU restatement of BlackHorizon's geodesic hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle that the CUDA library's results are
 * checked against, never part of the product.  Compile with -ffp-contract=off and without -ffast-math so each
 * expression rounds exactly like the NumPy expression it restates.  The
 * association order of every sum and product below follows the reference
 * expression left to right; NumPy reduces a 3-element axis sequentially and an
 * 8-element axis pairwise ((0+1)+(2+3))+((4+5)+(6+7)); sum3 and the sum in
 * bho_error_ratio reproduce both orders.
 */
#include "bh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* kerr.py:26 (_TINY). */
#define BHO_TINY 1e-30

/* numpy.maximum / numpy.minimum propagate NaN from either operand. */
static inline double np_max(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a >= b ? a : b;
}
static inline double np_min(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a <= b ? a : b;
}
/* numpy.clip(x, lo, hi) == minimum(maximum(x, lo), hi). */
static inline double np_clip(double x, double lo, double hi) {
    return np_min(np_max(x, lo), hi);
}
static inline double sum3(double a, double b, double c) { return (a + b) + c; }

/* ------------------------------------------------- host thread pool */

/* A minimal dynamic-schedule parallel-for over [0, n) in chunks, on plain
 * pthreads so the oracle needs no OpenMP runtime. */
typedef void (*bho_range_fn)(void *ctx, int64_t begin, int64_t end, int64_t *acc);
typedef struct {
    bho_range_fn fn;
    void *ctx;
    int64_t n, chunk;
    atomic_llong next;
    int64_t acc_max;
    pthread_mutex_t mu;
} bho_pool_t;

static void *bho_worker(void *arg) {
    bho_pool_t *pool = (bho_pool_t *)arg;
    int64_t local = 0;
    for (;;) {
        const int64_t b = (int64_t)atomic_fetch_add(&pool->next, pool->chunk);
        if (b >= pool->n) break;
        const int64_t e = b + pool->chunk < pool->n ? b + pool->chunk : pool->n;
        pool->fn(pool->ctx, b, e, &local);
    }
    pthread_mutex_lock(&pool->mu);
    if (local > pool->acc_max) pool->acc_max = local;
    pthread_mutex_unlock(&pool->mu);
    return NULL;
}

int bho_num_threads(void) {
    const long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

/* Runs fn over [0, n) on nthreads threads (<= 0: all online cores) and
 * returns the maximum of the per-thread accumulators. */
static int64_t bho_parallel_for(int64_t n, int nthreads, int64_t chunk,
                                bho_range_fn fn, void *ctx) {
    bho_pool_t pool;
    pool.fn = fn;
    pool.ctx = ctx;
    pool.n = n;
    pool.chunk = chunk > 0 ? chunk : 1;
    atomic_init(&pool.next, 0);
    pool.acc_max = 0;
    pthread_mutex_init(&pool.mu, NULL);
    if (nthreads <= 0) nthreads = bho_num_threads();
    if (nthreads > 256) nthreads = 256;
    if (nthreads == 1 || n <= pool.chunk) {
        bho_worker(&pool);
    } else {
        pthread_t tid[256];
        int started = 0;
        for (int i = 0; i < nthreads; ++i)
            if (pthread_create(&tid[i], NULL, bho_worker, &pool) == 0) ++started;
        if (started == 0) bho_worker(&pool);
        for (int i = 0; i < started; ++i) pthread_join(tid[i], NULL);
    }
    pthread_mutex_destroy(&pool.mu);
    return pool.acc_max;
}

/* ---------------------------------------------------------------- kerr.py */

void bho_geometry(double m, double a, double x, double y, double z,
                  int gradients, bho_geometry_t *o) {
    /* kerr.py:135-155 */
    const double a2 = a * a;
    const double rho2 = x * x + y * y + z * z;
    const double q = rho2 - a2;
    double s = sqrt(q * q + 4.0 * a2 * z * z);
    s = np_max(s, BHO_TINY);
    const double r2 = 0.5 * (q + s);
    const double r = sqrt(np_max(r2, BHO_TINY));
    const double r2_plus_a2 = r2 + a2;
    const double qd = np_max(r2 * r2 + a2 * z * z, BHO_TINY);
    const double h = m * r * r2 / qd;
    const double inv_r2a2 = 1.0 / np_max(r2_plus_a2, BHO_TINY);
    const double inv_r = 1.0 / r;
    const double lx = (r * x + a * y) * inv_r2a2;
    const double ly = (r * y - a * x) * inv_r2a2;
    const double lz = z * inv_r;
    o->r = r;
    o->h = h;
    o->l[0] = lx;
    o->l[1] = ly;
    o->l[2] = lz;
    if (!gradients) return;

    /* kerr.py:160-163: implicit derivative of the radius. */
    const double inv_s = 1.0 / s;
    const double r_x = x * r * inv_s;
    const double r_y = y * r * inv_s;
    const double r_z = z * r2_plus_a2 * inv_r * inv_s;

    /* kerr.py:166-171: gradient of H. */
    const double inv_qd2 = 1.0 / (qd * qd);
    const double dh_dr = m * r2 * (3.0 * a2 * z * z - r2 * r2) * inv_qd2;
    const double dh_dz_explicit = -2.0 * m * a2 * z * r * r2 * inv_qd2;
    o->grad_h[0] = dh_dr * r_x;
    o->grad_h[1] = dh_dr * r_y;
    o->grad_h[2] = dh_dr * r_z + dh_dz_explicit;

    /* kerr.py:177-191: gradients of the spatial null covector. */
    const double two_r = 2.0 * r;
    const double dlx_dx = (r_x * x + r) * inv_r2a2 - lx * two_r * r_x * inv_r2a2;
    const double dlx_dy = (r_y * x + a) * inv_r2a2 - lx * two_r * r_y * inv_r2a2;
    const double dlx_dz = r_z * x * inv_r2a2 - lx * two_r * r_z * inv_r2a2;
    const double dly_dx = (r_x * y - a) * inv_r2a2 - ly * two_r * r_x * inv_r2a2;
    const double dly_dy = (r_y * y + r) * inv_r2a2 - ly * two_r * r_y * inv_r2a2;
    const double dly_dz = r_z * y * inv_r2a2 - ly * two_r * r_z * inv_r2a2;
    const double dlz_dx = -lz * r_x * inv_r;
    const double dlz_dy = -lz * r_y * inv_r;
    const double dlz_dz = (1.0 - lz * r_z) * inv_r;
    o->grad_l[0][0] = dlx_dx; o->grad_l[0][1] = dly_dx; o->grad_l[0][2] = dlz_dx;
    o->grad_l[1][0] = dlx_dy; o->grad_l[1][1] = dly_dy; o->grad_l[1][2] = dlz_dy;
    o->grad_l[2][0] = dlx_dz; o->grad_l[2][1] = dly_dz; o->grad_l[2][2] = dlz_dz;
}

/* ----------------------------------------------------------- geodesics.py */

void bho_rhs(double m, double a, const double s[8], double d[8]) {
    /* geodesics.py:57-74 */
    bho_geometry_t g;
    bho_geometry(m, a, s[1], s[2], s[3], 1, &g);
    const double p_t = s[4];
    const double p0 = s[5], p1 = s[6], p2 = s[7];
    const double lp = -p_t + sum3(g.l[0] * p0, g.l[1] * p1, g.l[2] * p2);
    const double two_h_lp = 2.0 * g.h * lp;
    d[0] = -p_t + two_h_lp;
    d[1] = p0 - two_h_lp * g.l[0];
    d[2] = p1 - two_h_lp * g.l[1];
    d[3] = p2 - two_h_lp * g.l[2];
    d[4] = 0.0;
    const double lp2 = lp * lp;
    for (int i = 0; i < 3; ++i) {
        const double c = sum3(g.grad_l[i][0] * p0, g.grad_l[i][1] * p1,
                              g.grad_l[i][2] * p2);
        d[5 + i] = g.grad_h[i] * lp2 + two_h_lp * c;
    }
}

double bho_hamiltonian(double m, double a, const double s[8]) {
    /* geodesics.py:79-85 */
    bho_geometry_t g;
    bho_geometry(m, a, s[1], s[2], s[3], 0, &g);
    const double p_t = s[4];
    const double lp = -p_t + sum3(g.l[0] * s[5], g.l[1] * s[6], g.l[2] * s[7]);
    const double eta = 0.5 * (-p_t * p_t + sum3(s[5] * s[5], s[6] * s[6], s[7] * s[7]));
    return eta - g.h * lp * lp;
}

void bho_coordinate_velocity(double m, double a, const double s[8], double v[4]) {
    /* geodesics.py:97-106 */
    bho_geometry_t g;
    bho_geometry(m, a, s[1], s[2], s[3], 0, &g);
    const double p_t = s[4];
    const double lp = -p_t + sum3(g.l[0] * s[5], g.l[1] * s[6], g.l[2] * s[7]);
    const double two_h_lp = 2.0 * g.h * lp;
    v[0] = -p_t + two_h_lp;
    v[1] = s[5] - two_h_lp * g.l[0];
    v[2] = s[6] - two_h_lp * g.l[1];
    v[3] = s[7] - two_h_lp * g.l[2];
}

void bho_null_momentum(double m, double a, const double pos[3],
                       const double dir[3], int past, int normalize,
                       double p[4]) {
    /* geodesics.py:141-170 */
    bho_geometry_t g;
    bho_geometry(m, a, pos[0], pos[1], pos[2], 0, &g);
    const double h = g.h;
    const double l_dot_s = sum3(g.l[0] * dir[0], g.l[1] * dir[1], g.l[2] * dir[2]);
    const double s_dot_s = sum3(dir[0] * dir[0], dir[1] * dir[1], dir[2] * dir[2]);
    const double g_tt = 2.0 * h - 1.0;
    const double b_coef = 4.0 * h * l_dot_s;
    const double c_coef = s_dot_s + 2.0 * h * l_dot_s * l_dot_s;
    const double disc = b_coef * b_coef - 4.0 * g_tt * c_coef;
    const double sqrt_disc = sqrt(np_max(disc, 0.0));
    const double root_a = (-b_coef + sqrt_disc) / (2.0 * g_tt);
    const double root_b = (-b_coef - sqrt_disc) / (2.0 * g_tt);
    const double k_t = past ? np_min(root_a, root_b) : np_max(root_a, root_b);
    const double l_dot_k = k_t + l_dot_s;
    p[0] = -k_t + 2.0 * h * l_dot_k;
    for (int i = 0; i < 3; ++i) p[1 + i] = dir[i] + (2.0 * h * l_dot_k) * g.l[i];
    if (normalize) {
        const double n0 = fabs(p[0]);
        for (int i = 0; i < 4; ++i) p[i] = p[i] / n0;
    }
}

/* --------------------------------------------------------- integrators.py */

/* integrators.py:24-54 -- Dormand-Prince 5(4) tableau, autonomous form. */
#define A21 (1.0 / 5.0)
#define A31 (3.0 / 40.0)
#define A32 (9.0 / 40.0)
#define A41 (44.0 / 45.0)
#define A42 (-56.0 / 15.0)
#define A43 (32.0 / 9.0)
#define A51 (19372.0 / 6561.0)
#define A52 (-25360.0 / 2187.0)
#define A53 (64448.0 / 6561.0)
#define A54 (-212.0 / 729.0)
#define A61 (9017.0 / 3168.0)
#define A62 (-355.0 / 33.0)
#define A63 (46732.0 / 5247.0)
#define A64 (49.0 / 176.0)
#define A65 (-5103.0 / 18656.0)
#define B1 (35.0 / 384.0)
#define B3 (500.0 / 1113.0)
#define B4 (125.0 / 192.0)
#define B5 (-2187.0 / 6784.0)
#define B6 (11.0 / 84.0)
#define E1 (71.0 / 57600.0)
#define E3 (-71.0 / 16695.0)
#define E4 (71.0 / 1920.0)
#define E5 (-17253.0 / 339200.0)
#define E6 (22.0 / 525.0)
#define E7 (-1.0 / 40.0)

void bho_dp5_step(double m, double a, const double y[8], double h,
                  double y_new[8], double err[8]) {
    /* integrators.py:92-107 */
    double k1[8], k2[8], k3[8], k4[8], k5[8], k6[8], k7[8], t[8];
    int i;
    bho_rhs(m, a, y, k1);
    for (i = 0; i < 8; ++i) t[i] = y[i] + h * (A21 * k1[i]);
    bho_rhs(m, a, t, k2);
    for (i = 0; i < 8; ++i) t[i] = y[i] + h * (A31 * k1[i] + A32 * k2[i]);
    bho_rhs(m, a, t, k3);
    for (i = 0; i < 8; ++i)
        t[i] = y[i] + h * (A41 * k1[i] + A42 * k2[i] + A43 * k3[i]);
    bho_rhs(m, a, t, k4);
    for (i = 0; i < 8; ++i)
        t[i] = y[i] + h * (A51 * k1[i] + A52 * k2[i] + A53 * k3[i] + A54 * k4[i]);
    bho_rhs(m, a, t, k5);
    for (i = 0; i < 8; ++i)
        t[i] = y[i] + h * (A61 * k1[i] + A62 * k2[i] + A63 * k3[i] +
                           A64 * k4[i] + A65 * k5[i]);
    bho_rhs(m, a, t, k6);
    for (i = 0; i < 8; ++i) {
        const double inc = B1 * k1[i] + B3 * k3[i] + B4 * k4[i] + B5 * k5[i] + B6 * k6[i];
        y_new[i] = y[i] + h * inc;
    }
    bho_rhs(m, a, y_new, k7);
    for (i = 0; i < 8; ++i)
        err[i] = h * (E1 * k1[i] + E3 * k3[i] + E4 * k4[i] + E5 * k5[i] +
                      E6 * k6[i] + E7 * k7[i]);
}

double bho_error_ratio(const double y[8], const double y_new[8],
                       const double err[8], double rtol, double atol) {
    /* integrators.py:113-117 */
    double q[8];
    for (int i = 0; i < 8; ++i) {
        const double scale = atol + rtol * np_max(fabs(y[i]), fabs(y_new[i]));
        const double e = err[i] / scale;
        q[i] = e * e;
    }
    const double sum = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
    const double ratio = sqrt(sum / 8.0);
    return isfinite(ratio) ? ratio : INFINITY;
}

double bho_step_factor(double ratio) {
    /* integrators.py:122-124 */
    const double safe = np_max(ratio, 1e-16);
    return np_clip(0.9 * pow(safe, -0.2), 0.2, 5.0);
}

void bho_rk4_step(double m, double a, const double y[8], double h,
                  double y_new[8]) {
    /* integrators.py:69-73 */
    double k1[8], k2[8], k3[8], k4[8], t[8];
    int i;
    bho_rhs(m, a, y, k1);
    for (i = 0; i < 8; ++i) t[i] = y[i] + 0.5 * h * k1[i];
    bho_rhs(m, a, t, k2);
    for (i = 0; i < 8; ++i) t[i] = y[i] + 0.5 * h * k2[i];
    bho_rhs(m, a, t, k3);
    for (i = 0; i < 8; ++i) t[i] = y[i] + h * k3[i];
    bho_rhs(m, a, t, k4);
    for (i = 0; i < 8; ++i)
        y_new[i] = y[i] + (h / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
}

/* -------------------------------------------------------------- camera.py */

void bho_pinhole_directions(const double fwd[3], const double right[3],
                            const double up[3], double fov_degrees,
                            int64_t width, int64_t height, double *dirs) {
    /* camera.py:102-113; math.radians(x) is x * (pi / 180). */
    const double half_w = tan(fov_degrees * (M_PI / 180.0) / 2.0);
    const double half_h = half_w * (double)height / (double)width;
    for (int64_t row = 0; row < height; ++row) {
        const double rv = 1.0 - ((double)row + 0.5) / (double)height * 2.0;
        const double v = rv * half_h;
        for (int64_t col = 0; col < width; ++col) {
            const double cu = ((double)col + 0.5) / (double)width * 2.0 - 1.0;
            const double u = cu * half_w;
            double d[3];
            for (int i = 0; i < 3; ++i) d[i] = fwd[i] + u * right[i] + v * up[i];
            const double nrm = sqrt(sum3(d[0] * d[0], d[1] * d[1], d[2] * d[2]));
            double *o = dirs + 3 * (row * width + col);
            for (int i = 0; i < 3; ++i) o[i] = d[i] / nrm;
        }
    }
}

/* -------------------------------------------------------------- tracer.py */

static int64_t trace_one(const bho_trace_params_t *p, double capture_radius,
                         double y[8], int32_t *status_out, int64_t *steps_out) {
    /* Body of the batch loop tracer.py:103-149 for one ray: a ray that is in
     * flight at batch iteration k has made exactly k attempts, so the
     * batch-global cap 4*max_steps (tracer.py:101) is a per-ray attempt cap. */
    const int64_t max_iterations = 4 * p->max_steps;
    double h = p->initial_step;
    int64_t steps = 0;
    int32_t status = BHO_IN_FLIGHT;
    int64_t it = 0;
    while (it < max_iterations) {
        ++it;
        double y_new[8], err[8];
        bho_dp5_step(p->mass, p->spin, y, h, y_new, err);
        const double ratio = bho_error_ratio(y, y_new, err, p->rtol, p->atol);
        const int accept = ratio <= 1.0;
        if (accept) memcpy(y, y_new, sizeof(y_new));
        steps += accept;
        h = np_clip(h * bho_step_factor(ratio), 0.0, p->max_step);

        bho_geometry_t g;
        bho_geometry(p->mass, p->spin, y[1], y[2], y[3], 0, &g);
        int finite = 1;
        for (int i = 0; i < 8; ++i) finite &= isfinite(y[i]) ? 1 : 0;
        int32_t st = BHO_IN_FLIGHT;
        if (!finite) st = BHO_FAILED;
        if (finite && g.r <= capture_radius) st = BHO_CAPTURED;
        if (finite && g.r >= p->escape_radius) st = BHO_ESCAPED;
        const int in_flight = st == BHO_IN_FLIGHT;
        if (in_flight && h < p->min_step) st = BHO_FAILED;
        if (in_flight && steps >= p->max_steps) st = BHO_MAX_STEPS;
        status = st;
        if (status != BHO_IN_FLIGHT) break;
    }
    /* tracer.py:151-154 */
    if (status == BHO_IN_FLIGHT) status = BHO_MAX_STEPS;
    *status_out = status;
    *steps_out = steps;
    return it;
}

typedef struct {
    const bho_trace_params_t *p;
    double capture_radius;
    double *states;
    int32_t *status;
    int64_t *steps;
} trace_ctx_t;

static void trace_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    trace_ctx_t *c = (trace_ctx_t *)vctx;
    for (int64_t i = b; i < e; ++i) {
        const int64_t it = trace_one(c->p, c->capture_radius, c->states + 8 * i,
                                     c->status + i, c->steps + i);
        if (it > *acc) *acc = it;
    }
}

int64_t bho_trace_batch(const bho_trace_params_t *p, double *states,
                        int32_t *status, int64_t *steps, int64_t n,
                        int nthreads) {
    /* tracer.py:84 */
    const double r_plus = p->mass + sqrt(p->mass * p->mass - p->spin * p->spin);
    const double capture_radius = r_plus * (1.0 + p->capture_margin);
    /* tracer.py:95-99 */
    for (int64_t i = 0; i < n; ++i) {
        bho_geometry_t g;
        const double *s = states + 8 * i;
        bho_geometry(p->mass, p->spin, s[1], s[2], s[3], 0, &g);
        if (g.r >= p->escape_radius) return -1;
    }
    trace_ctx_t c = {p, capture_radius, states, status, steps};
    return bho_parallel_for(n, nthreads, 16, trace_range, &c);
}

typedef struct {
    double mass, spin;
    const double *spins;
    double *states, *h;
    int64_t *accepted;
    int64_t n_steps;
    double rtol, atol, max_step;
} prop_ctx_t;

static void prop_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    prop_ctx_t *c = (prop_ctx_t *)vctx;
    (void)acc;
    for (int64_t i = b; i < e; ++i) {
        const double a = c->spins ? c->spins[i] : c->spin;
        double *y = c->states + 8 * i;
        double hh = c->h[i];
        int64_t nacc = 0;
        for (int64_t k = 0; k < c->n_steps; ++k) {
            double y_new[8], err[8];
            bho_dp5_step(c->mass, a, y, hh, y_new, err);
            const double ratio = bho_error_ratio(y, y_new, err, c->rtol, c->atol);
            if (ratio <= 1.0) {
                memcpy(y, y_new, sizeof(y_new));
                ++nacc;
            }
            hh = np_clip(hh * bho_step_factor(ratio), 0.0, c->max_step);
        }
        c->h[i] = hh;
        c->accepted[i] = nacc;
    }
}

void bho_propagate_batch(double mass, double spin, const double *spins,
                         double *states, double *h, int64_t *accepted,
                         int64_t n, int64_t n_steps, double rtol, double atol,
                         double max_step, int nthreads) {
    /* The accept/reject and step update of tracer.py:111-120, without the
     * termination cascade. */
    prop_ctx_t c = {mass, spin, spins, states, h, accepted, n_steps, rtol, atol, max_step};
    bho_parallel_for(n, nthreads, 4, prop_range, &c);
}

typedef struct {
    double mass, spin;
    const double *spins, *target;
    double *states;
    int64_t *attempts;
    double rtol, atol, initial_step, max_step;
    int64_t max_attempts;
} to_ctx_t;

static void to_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    /* integrate_dense (integrators.py:155-173) for one ray: the step is cut
     * to land on the target affine parameter; a ray whose step underflows or
     * runs out of attempts gets NaN states. */
    to_ctx_t *c = (to_ctx_t *)vctx;
    (void)acc;
    for (int64_t i = b; i < e; ++i) {
        const double a = c->spins ? c->spins[i] : c->spin;
        double *y = c->states + 8 * i;
        const double total = c->target[i];
        double elapsed = 0.0, h = c->initial_step;
        int64_t k = 0;
        int ok = 1;
        while (elapsed < total) {
            if (k++ >= c->max_attempts) { ok = 0; break; }
            double rem = total - elapsed;
            if (c->max_step < h) h = c->max_step;
            if (rem < h) h = rem;
            double y_new[8], err[8];
            bho_dp5_step(c->mass, a, y, h, y_new, err);
            const double ratio = bho_error_ratio(y, y_new, err, c->rtol, c->atol);
            if (ratio <= 1.0) {
                memcpy(y, y_new, sizeof(y_new));
                elapsed += h;
            }
            h *= bho_step_factor(ratio);
            if (h < 1e-14) { ok = 0; break; }
        }
        if (!ok)
            for (int j = 0; j < 8; ++j) y[j] = NAN;
        if (c->attempts) c->attempts[i] = k;
    }
}

void bho_propagate_to(double mass, double spin, const double *spins,
                      double *states, const double *lam_target,
                      int64_t *attempts, int64_t n, double rtol, double atol,
                      double initial_step, double max_step,
                      int64_t max_attempts, int nthreads) {
    to_ctx_t c = {mass, spin, spins, lam_target, states, attempts, rtol, atol,
                  initial_step, max_step, max_attempts};
    bho_parallel_for(n, nthreads, 2, to_range, &c);
}

/* render.py:312-349 (_refine_crossings) for one ray: 40 bisections of the
 * fraction of the step at which an RK4 substep from y0 crosses z = 0. */
static int refine_crossing(double m, double a, const double y0[8], double h_full,
                           double r_in, double r_out, double y_cross[8]) {
    double low = 0.0, high = 1.0;
    for (int it = 0; it < 40; ++it) {
        const double mid = 0.5 * (low + high);
        double ym[8];
        bho_rk4_step(m, a, y0, h_full * mid, ym);
        const int same_side = ym[3] * y0[3] > 0.0;
        if (same_side) low = mid; else high = mid;
    }
    bho_rk4_step(m, a, y0, h_full * (0.5 * (low + high)), y_cross);
    bho_geometry_t g;
    bho_geometry(m, a, y_cross[1], y_cross[2], y_cross[3], 0, &g);
    return g.r >= r_in && g.r <= r_out;
}

typedef struct {
    const bho_trace_params_t *p;
    double capture_radius, r_in, r_out;
    int interior;  /* interior camera: capture_radius is the interior stop */
    double *states, *hit_pos, *hit_mom, *escape_dir;
    int32_t *status, *saturated;
    int64_t *steps;
} tile_ctx_t;

static void tile_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    tile_ctx_t *c = (tile_ctx_t *)vctx;
    const bho_trace_params_t *p = c->p;
    (void)acc;
    for (int64_t i = b; i < e; ++i) {
        double *y = c->states + 8 * i;
        double h = 0.1;  /* render.py:221 */
        int64_t steps = 0;
        int32_t status = BHO_IN_FLIGHT;
        for (int k = 0; k < 3; ++k) {
            c->hit_pos[3 * i + k] = 0.0;
            c->hit_mom[3 * i + k] = 0.0;
            c->escape_dir[3 * i + k] = 0.0;
        }
        for (int64_t it = 0; it < 4 * p->max_steps; ++it) {
            /* render.py:231-260: termination before the step. */
            bho_geometry_t g;
            bho_geometry(p->mass, p->spin, y[1], y[2], y[3], 0, &g);
            int captured = g.r <= c->capture_radius;
            if (c->interior) {
                /* render.py:234-248: a diverging spatial momentum ends the
                 * ray on the terminal surface. */
                const double pn = sqrt(sum3(y[5] * y[5], y[6] * y[6], y[7] * y[7]));
                captured = captured || pn > 1.0e3 ||
                           (g.r <= c->capture_radius * 1.002 && pn > 50.0);
            }
            const int escaped = !captured && g.r >= p->escape_radius;
            const int exhausted = steps >= p->max_steps;
            if (captured) { status = c->interior ? BHO_TERMINATED : BHO_CAPTURED; break; }
            if (escaped) { status = BHO_ESCAPED; break; }
            if (exhausted) { status = BHO_MAX_STEPS; break; }
            /* render.py:264-266 */
            double y_new[8], err[8];
            bho_dp5_step(p->mass, p->spin, y, h, y_new, err);
            const double ratio = bho_error_ratio(y, y_new, err, p->rtol, p->rtol * 1e-3);
            const int accept = ratio <= 1.0;
            /* render.py:268-281 */
            if (c->r_out > 0.0 && accept && y[3] * y_new[3] < 0.0) {
                double yc[8];
                if (refine_crossing(p->mass, p->spin, y, h, c->r_in, c->r_out, yc)) {
                    status = BHO_DISK;
                    for (int k = 0; k < 3; ++k) {
                        c->hit_pos[3 * i + k] = yc[1 + k];
                        c->hit_mom[3 * i + k] = yc[5 + k];
                    }
                }
            }
            /* render.py:283-287 */
            const int still = status == BHO_IN_FLIGHT;
            if (accept && still) {
                memcpy(y, y_new, sizeof(y_new));
                ++steps;
            }
            h = np_clip(h * bho_step_factor(ratio), 0.0, p->max_step);
            if (!still) break;
        }
        c->status[i] = status;
        c->steps[i] = steps;
        /* render.py:289-291 */
        c->saturated[i] = status == BHO_MAX_STEPS || steps >= (int64_t)(0.85 * (double)p->max_steps);
        if (status == BHO_ESCAPED) {
            /* render.py:164-181 with the ray's own p_t as the energy. */
            bho_geometry_t g;
            bho_geometry(p->mass, p->spin, y[1], y[2], y[3], 0, &g);
            const double lp = -y[4] + sum3(g.l[0] * y[5], g.l[1] * y[6], g.l[2] * y[7]);
            double d[3];
            for (int k = 0; k < 3; ++k) d[k] = y[5 + k] - 2.0 * (g.h * lp) * g.l[k];
            const double nrm = sqrt(sum3(d[0] * d[0], d[1] * d[1], d[2] * d[2]));
            for (int k = 0; k < 3; ++k) c->escape_dir[3 * i + k] = d[k] / nrm;
        }
    }
}

void bho_trace_tile(const bho_trace_params_t *p, double disk_inner,
                    double disk_outer, double interior_stop, double *states,
                    int32_t *status, int64_t *steps, double *hit_pos,
                    double *hit_mom, double *escape_dir, int32_t *saturated,
                    int64_t n, int nthreads) {
    const double r_plus = p->mass + sqrt(p->mass * p->mass - p->spin * p->spin);
    /* render.py:203-213 */
    const int interior = interior_stop > 0.0;
    tile_ctx_t c = {p, interior ? interior_stop : r_plus * (1.0 + p->capture_margin),
                    disk_inner, disk_outer, interior,
                    states, hit_pos, hit_mom, escape_dir, status, saturated, steps};
    bho_parallel_for(n, nthreads, 4, tile_range, &c);
}

typedef struct {
    double mass, spin, h;
    double *states;
    int64_t n_steps;
} rk4_ctx_t;

static void rk4_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    rk4_ctx_t *c = (rk4_ctx_t *)vctx;
    (void)acc;
    for (int64_t i = b; i < e; ++i) {
        double *y = c->states + 8 * i;
        for (int64_t k = 0; k < c->n_steps; ++k) {
            double y_new[8];
            bho_rk4_step(c->mass, c->spin, y, c->h, y_new);
            memcpy(y, y_new, sizeof(y_new));
        }
    }
}

void bho_rk4_batch(double mass, double spin, double *states, int64_t n,
                   int64_t n_steps, double h, int nthreads) {
    rk4_ctx_t c = {mass, spin, h, states, n_steps};
    bho_parallel_for(n, nthreads, 64, rk4_range, &c);
}

/* ------------------------------------------------- batched test helpers */

void bho_geometry_batch(double m, double a, const double *xyz, int64_t n,
                        double *r, double *h, double *l, double *grad_h,
                        double *grad_l) {
    for (int64_t i = 0; i < n; ++i) {
        bho_geometry_t g;
        bho_geometry(m, a, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 1, &g);
        r[i] = g.r;
        h[i] = g.h;
        for (int j = 0; j < 3; ++j) {
            l[3 * i + j] = g.l[j];
            grad_h[3 * i + j] = g.grad_h[j];
            for (int k = 0; k < 3; ++k) grad_l[9 * i + 3 * j + k] = g.grad_l[j][k];
        }
    }
}

void bho_rhs_batch(double m, double a, const double *states, int64_t n,
                   double *deriv) {
    for (int64_t i = 0; i < n; ++i) bho_rhs(m, a, states + 8 * i, deriv + 8 * i);
}

void bho_dp5_batch(double m, double a, const double *states, const double *h,
                   int64_t n, double *y_new, double *err, double *ratio,
                   double rtol, double atol) {
    for (int64_t i = 0; i < n; ++i) {
        bho_dp5_step(m, a, states + 8 * i, h[i], y_new + 8 * i, err + 8 * i);
        if (ratio)
            ratio[i] = bho_error_ratio(states + 8 * i, y_new + 8 * i,
                                       err + 8 * i, rtol, atol);
    }
}

void bho_null_momentum_batch(double m, double a, const double *pos,
                             const double *dir, int64_t n, int past,
                             int normalize, double *p) {
    for (int64_t i = 0; i < n; ++i)
        bho_null_momentum(m, a, pos + 3 * i, dir + 3 * i, past, normalize, p + 4 * i);
}

/* ------------------------------------------------------------ imaging.py */

static void checker_rgb(const double d[3], int cells, uint8_t rgb[3]) {
    /* imaging.py:38-50, NumPy's evaluation order. */
    static const uint8_t dark[3] = {24, 30, 52}, light[3] = {104, 128, 178};
    const double z = np_clip(d[2], -1.0, 1.0);
    const double theta = acos(z);
    const double phi = atan2(d[1], d[0]);
    const int64_t i_theta = (int64_t)floor(theta / M_PI * (double)cells);
    const int64_t i_phi = (int64_t)floor((phi + M_PI) / (2.0 * M_PI) * 2.0 * (double)cells);
    const uint8_t *c = ((i_theta + i_phi) % 2) ? light : dark;
    rgb[0] = c[0]; rgb[1] = c[1]; rgb[2] = c[2];
}

void bho_celestial_checkerboard(const double *dirs, int64_t n, int cells,
                                uint8_t *rgb) {
    for (int64_t i = 0; i < n; ++i) checker_rgb(dirs + 3 * i, cells, rgb + 3 * i);
}

void bho_render_image(double m, double a, const double *states,
                      const int32_t *status, int64_t n, int cells, uint8_t *rgb) {
    for (int64_t i = 0; i < n; ++i) {
        uint8_t *o = rgb + 3 * i;
        const int32_t st = status[i];
        if (st == BHO_CAPTURED) {
            o[0] = o[1] = o[2] = 0;
        } else if (st == BHO_ESCAPED) {
            /* geodesics.py:98-106: spatial coordinate velocity. */
            const double *y = states + 8 * i;
            bho_geometry_t g;
            bho_geometry(m, a, y[1], y[2], y[3], 0, &g);
            const double lp = -y[4] + sum3(g.l[0] * y[5], g.l[1] * y[6], g.l[2] * y[7]);
            const double two_h_lp = 2.0 * g.h * lp;
            double v[3];
            for (int k = 0; k < 3; ++k) v[k] = y[5 + k] - two_h_lp * g.l[k];
            double nrm = sqrt(sum3(v[0] * v[0], v[1] * v[1], v[2] * v[2]));
            if (nrm == 0.0) nrm = 1.0;
            const double d[3] = {v[0] / nrm, v[1] / nrm, v[2] / nrm};
            checker_rgb(d, cells, o);
        } else if (st == BHO_MAX_STEPS) {
            o[0] = 120; o[1] = 32; o[2] = 32;
        } else {
            o[0] = 200; o[1] = 0; o[2] = 200;
        }
    }
}

/* ------------------------------------------------------- realtime/reference.py */

typedef struct {
    const bho_realtime_params_t *p;
    double *states, *hit_radius, *hit_pos, *hit_mom;
    int32_t *status;
} realtime_ctx_t;

static void realtime_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    realtime_ctx_t *c = (realtime_ctx_t *)vctx;
    const bho_realtime_params_t *p = c->p;
    (void)acc;
    const double m = p->mass, a = p->spin;
    const double r_plus = m + sqrt(m * m - a * a);
    const int interior = p->interior_stop > 0.0;
    const double capture_radius = interior ? p->interior_stop : r_plus * (1.0 + p->capture_margin);
    const int32_t capture_status = interior ? BHO_TERMINATED : BHO_CAPTURED;
    const int64_t max_steps = interior && p->max_steps > 1024 ? 1024 : p->max_steps;
    const double bail2 = p->momentum_bailout * p->momentum_bailout;
    for (int64_t i = b; i < e; ++i) {
        double *y = c->states + 8 * i;
        int32_t st = BHO_MAX_STEPS;
        c->hit_radius[i] = NAN;
        for (int k = 0; k < 3; ++k) c->hit_pos[3 * i + k] = NAN;
        for (int k = 0; k < 4; ++k) c->hit_mom[4 * i + k] = NAN;
        for (int64_t it = 0; it < max_steps; ++it) {
            /* reference.py:107-133 */
            bho_geometry_t g;
            bho_geometry(m, a, y[1], y[2], y[3], 0, &g);
            const double r = g.r;
            const double mom2 = sum3(y[5] * y[5], y[6] * y[6], y[7] * y[7]);
            int captured = (r <= capture_radius) || (mom2 >= bail2);
            if (interior) captured = captured || ((r <= capture_radius * 1.002) && (mom2 > 2500.0));
            const int escaped = !captured && (r >= p->escape_radius);
            if (captured) { st = capture_status; break; }
            if (escaped) { st = BHO_ESCAPED; break; }
            /* reference.py:135-154 */
            double scale;
            if (!interior) scale = r - r_plus;
            else scale = np_min(np_max(fabs(r - r_plus), 0.15 * r), 0.5 * r);
            double h = np_clip(p->step_scale * scale, p->min_step, p->max_step);
            h = np_min(h, 1.0 / np_max(1.0, sqrt(mom2)));
            double y_new[8];
            bho_rk4_step(m, a, y, h, y_new);
            int hit = 0;
            /* reference.py:162-184 */
            if (p->disk_outer > 0.0 && y[3] * y_new[3] < 0.0) {
                const double t = y[3] / (y[3] - y_new[3]);
                double q[8];
                for (int k = 0; k < 8; ++k) q[k] = y[k] + t * (y_new[k] - y[k]);
                bho_geometry_t gh;
                bho_geometry(m, a, q[1], q[2], q[3], 0, &gh);
                if (gh.r >= p->disk_inner && gh.r <= p->disk_outer) {
                    hit = 1;
                    c->hit_radius[i] = gh.r;
                    for (int k = 0; k < 3; ++k) c->hit_pos[3 * i + k] = q[1 + k];
                    for (int k = 0; k < 4; ++k) c->hit_mom[4 * i + k] = q[4 + k];
                }
            }
            memcpy(y, y_new, sizeof(y_new));
            if (hit) { st = BHO_DISK; break; }
        }
        c->status[i] = st;
    }
}

void bho_trace_realtime(const bho_realtime_params_t *p, double *states,
                        int32_t *status, double *hit_radius, double *hit_pos,
                        double *hit_mom, int64_t n, int nthreads) {
    realtime_ctx_t c = {p, states, hit_radius, hit_pos, hit_mom, status};
    bho_parallel_for(n, nthreads, 4, realtime_range, &c);
}

/* ------------------------------------------------------------ vaidya.py */

/* vaidya.py:153-159 */
static double vd_m1(const bho_vaidya_t *p, double v) {
    const double vs = np_max(v, p->tail_start);
    return p->mass - p->tail_mass * pow(p->tail_start / vs, p->tail_power - 1.0);
}

/* vaidya.py:161-171 */
static double vd_rate(const bho_vaidya_t *p, double v) {
    if (!(v >= p->tail_start)) return 0.0;
    return p->tail_mass * (p->tail_power - 1.0) * pow(p->tail_start, p->tail_power - 1.0) /
           pow(np_max(v, p->tail_start), p->tail_power);
}

static double vd_f(const bho_vaidya_t *p, double m, double r) {
    return 1.0 - 2.0 * m / r + pow(p->charge, 2.0) / pow(r, 2.0);
}

int64_t bho_vaidya_shell(const bho_vaidya_t *p, double *vs, double *rs, double *m2s,
                         int64_t capacity) {
    double v = p->shell_start_v, radius = p->shell_start_radius;
    double m2 = vd_m1(p, v) + p->shell_energy;
    int64_t k = 0;
    if (k < capacity) { vs[k] = v; rs[k] = radius; m2s[k] = m2; }
    ++k;
    const double step = 0.01;
    for (int64_t it = 0; it < 4000000; ++it) {
        const double m1 = vd_m1(p, v), lum = vd_rate(p, v);
        const double f1 = vd_f(p, m1, radius), f2 = vd_f(p, m2, radius);
        if (m2 >= p->mass_cap || fabs(f1) < 1e-300) break;
        const double r_half = radius + 0.25 * step * f1;
        const double m2_half = m2 + 0.5 * step * lum * f2 / f1;
        const double v_half = v + 0.5 * step;
        const double m1_half = vd_m1(p, v_half), lum_half = vd_rate(p, v_half);
        const double f1_half = vd_f(p, m1_half, r_half), f2_half = vd_f(p, m2_half, r_half);
        radius += 0.5 * step * f1_half;
        m2 += step * lum_half * f2_half / f1_half;
        if (p->mass_cap < m2) m2 = p->mass_cap; /* Python min(m2, cap) */
        v += step;
        if (k < capacity) { vs[k] = v; rs[k] = radius; m2s[k] = m2; }
        ++k;
    }
    return k;
}

/* numpy.interp for increasing xp (NumPy's compiled interpolation). */
static double np_interp(double x, const double *xp, const double *fp, int64_t n) {
    if (isnan(x)) return x;
    if (x < xp[0]) return fp[0];
    if (x > xp[n - 1]) return fp[n - 1];
    if (x == xp[n - 1]) return fp[n - 1];
    int64_t lo = 0, hi = n - 1; /* xp[lo] <= x < xp[hi] */
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) / 2;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    if (xp[lo] == x) return fp[lo];
    const double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
    double r = slope * (x - xp[lo]) + fp[lo];
    if (isnan(r)) {
        r = slope * (x - xp[lo + 1]) + fp[lo + 1];
        if (isnan(r) && fp[lo] == fp[lo + 1]) r = fp[lo];
    }
    return r;
}

/* vaidya.py:244-269 */
double bho_vaidya_mass(const bho_vaidya_t *p, double v, double r) {
    const double shell_r = np_interp(v, p->shell_v, p->shell_r, p->n_shell);
    const double t = np_clip((shell_r - r) / p->shell_width + 0.5, 0.0, 1.0);
    const double blend = t * t * (3.0 - 2.0 * t);
    double inc = 0.0;
    if (!(v < p->shell_start_v)) {
        const double m2 = np_interp(v, p->shell_v, p->shell_m2, p->n_shell);
        inc = np_clip(m2 - vd_m1(p, v), 0.0, p->mass_cap);
    }
    return vd_m1(p, v) + blend * inc;
}

double bho_vaidya_misner_sharp(const bho_vaidya_t *p, double v, double r) {
    return bho_vaidya_mass(p, v, r) - pow(p->charge, 2.0) / (2.0 * r);
}

void bho_vaidya_geometry(const bho_vaidya_t *p, double t, double x, double y, double z,
                         double *h, double l[3], double *hs, double *ht, double *radius) {
    const double r = np_max(sqrt(sum3(x * x, y * y, z * z)), 1e-9);
    l[0] = x / r; l[1] = y / r; l[2] = z / r;
    const double v = t + r, eps = 1e-4;
    const double m0 = bho_vaidya_mass(p, v, r);
    const double m_v = (bho_vaidya_mass(p, v + eps, r) - bho_vaidya_mass(p, v - eps, r)) / (2.0 * eps);
    const double m_r = (bho_vaidya_mass(p, v, r + eps) - bho_vaidya_mass(p, v, r - eps)) / (2.0 * eps);
    const double q2 = pow(p->charge, 2.0);
    *h = m0 / r - q2 / (2.0 * pow(r, 2.0));
    const double h_v = m_v / r;
    const double h_r = m_r / r - m0 / pow(r, 2.0) + q2 / pow(r, 3.0);
    *hs = h_v + h_r;
    *ht = h_v;
    *radius = r;
}

void bho_vaidya_rhs(const bho_vaidya_t *p, const double y[8], double out[8]) {
    double h, l[3], hs, ht, r;
    bho_vaidya_geometry(p, y[0], y[1], y[2], y[3], &h, l, &hs, &ht, &r);
    const double l_dot_p = sum3(l[0] * y[5], l[1] * y[6], l[2] * y[7]);
    const double lp = -y[4] + l_dot_p;
    const double lp2 = lp * lp;
    out[0] = -y[4] + 2.0 * h * lp;
    const double c = 2.0 * h * lp;
    for (int k = 0; k < 3; ++k) out[1 + k] = y[5 + k] - c * l[k];
    out[4] = ht * lp2;
    const double g = c / r;
    for (int k = 0; k < 3; ++k)
        out[5 + k] = (hs * l[k]) * lp2 + g * (y[5 + k] - l_dot_p * l[k]);
}

static void vd_rk4_step(const bho_vaidya_t *p, const double y[8], double h, double out[8]) {
    double k1[8], k2[8], k3[8], k4[8], tmp[8];
    bho_vaidya_rhs(p, y, k1);
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + 0.5 * h * k1[i];
    bho_vaidya_rhs(p, tmp, k2);
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + 0.5 * h * k2[i];
    bho_vaidya_rhs(p, tmp, k3);
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + h * k3[i];
    bho_vaidya_rhs(p, tmp, k4);
    const double h6 = h / 6.0;
    for (int i = 0; i < 8; ++i) out[i] = y[i] + h6 * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
}

void bho_vaidya_rk4(const bho_vaidya_t *p, double *states, int64_t n, int64_t n_steps,
                    double h) {
    for (int64_t i = 0; i < n; ++i)
        for (int64_t s = 0; s < n_steps; ++s) {
            double out[8];
            vd_rk4_step(p, states + 8 * i, h, out);
            memcpy(states + 8 * i, out, sizeof(out));
        }
}

typedef struct {
    const bho_vaidya_t *p;
    double *states, *escape_dir, *end_mass, *v_end;
    double esc, stop;
    int64_t max_steps;
    int32_t *status;
} vd_trace_ctx_t;

static void vd_trace_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    vd_trace_ctx_t *c = (vd_trace_ctx_t *)vctx;
    const bho_vaidya_t *p = c->p;
    (void)acc;
    const double r_plus = p->mass + sqrt(pow(p->mass, 2.0) - pow(p->charge, 2.0));
    for (int64_t i = b; i < e; ++i) {
        double *y = c->states + 8 * i;
        int32_t st = -1;
        c->escape_dir[3 * i] = c->escape_dir[3 * i + 1] = c->escape_dir[3 * i + 2] = 0.0;
        c->end_mass[i] = 0.0;
        for (int64_t it = 0; it < c->max_steps; ++it) {
            /* inflation.py:197-232 */
            const double r = sqrt(sum3(y[1] * y[1], y[2] * y[2], y[3] * y[3]));
            const double mom2 = sum3(y[5] * y[5], y[6] * y[6], y[7] * y[7]);
            const int captured = (r <= c->stop) || ((r <= c->stop * 1.08) && (mom2 > 400.0)) ||
                                 (mom2 > 1.0e6);
            const int escaped = !captured && (r >= c->esc);
            if (captured) {
                c->end_mass[i] = bho_vaidya_misner_sharp(p, y[0] + r, r);
                st = 1;
                break;
            }
            if (escaped) {
                double h, l[3], hs, ht, rr;
                bho_vaidya_geometry(p, 0.0, y[1], y[2], y[3], &h, l, &hs, &ht, &rr);
                const double lp = -y[4] + sum3(l[0] * y[5], l[1] * y[6], l[2] * y[7]);
                double d[3];
                for (int k = 0; k < 3; ++k) d[k] = y[5 + k] - 2.0 * h * lp * l[k];
                const double nrm = sqrt(sum3(d[0] * d[0], d[1] * d[1], d[2] * d[2]));
                for (int k = 0; k < 3; ++k) c->escape_dir[3 * i + k] = d[k] / nrm;
                st = 0;
                break;
            }
            /* inflation.py:233-239 */
            const double scale = r > r_plus ? r - r_plus : 0.5 * r;
            const double hstep = np_clip(0.15 * scale, 3e-3, 0.08);
            double out[8];
            vd_rk4_step(p, y, hstep, out);
            memcpy(y, out, sizeof(out));
        }
        c->status[i] = st == -1 ? 2 : st;
        c->v_end[i] = y[0] + sqrt(sum3(y[1] * y[1], y[2] * y[2], y[3] * y[3]));
    }
}

void bho_vaidya_trace(const bho_vaidya_t *p, double *states, int64_t n,
                      double escape_radius, double stop_radius, int64_t max_steps,
                      int32_t *status, double *escape_dir, double *end_mass,
                      double *v_end, int nthreads) {
    vd_trace_ctx_t c = {p, states, escape_dir, end_mass, v_end, escape_radius, stop_radius,
                        max_steps, status};
    bho_parallel_for(n, nthreads, 2, vd_trace_range, &c);
}

/* ------------------------------------------------- offline/render.py emission */

/* render.py:368-370 */
static double hash01(double a, double b, double salt) {
    const double v = sin(a * 127.1 + b * 311.7 + salt * 74.7) * 43758.5453;
    return v - floor(v);
}

static void starfield_one(const double *d, double shift, int shifted, double *c) {
    /* render.py:366-419 */
    const double phi = atan2(d[1], d[0]);
    const double theta = acos(np_clip(d[2], -1.0, 1.0));
    static const double cells_of[2] = {160.0, 420.0}, density_of[2] = {0.10, 0.05},
                        bright_of[2] = {3.0, 0.9};
    c[0] = c[1] = c[2] = 0.0;
    for (int layer = 0; layer < 2; ++layer) {
        const double cells = cells_of[layer];
        const double cu = phi / (2.0 * M_PI) * cells;
        const double cv = theta / M_PI * cells;
        const double iu = floor(cu), iv = floor(cv);
        const int present = hash01(iu, iv, 1.0) < density_of[layer];
        const double su = iu + 0.15 + 0.7 * hash01(iu, iv, 2.0);
        const double sv = iv + 0.15 + 0.7 * hash01(iu, iv, 3.0);
        const double dist2 = (cu - su) * (cu - su) + (cv - sv) * (cv - sv);
        const double magnitude = hash01(iu, iv, 4.0);
        double amplitude = bright_of[layer] * (0.15 + pow(magnitude, 4.0));
        const double point = exp(-dist2 / 0.006);
        double warmth = hash01(iu, iv, 5.0);
        if (shifted) {
            amplitude = amplitude * pow(shift, 4.0);
            warmth = np_clip(warmth - 0.6 * log(np_max(shift, 1e-6)), 0.0, 1.0);
        }
        const double tint[3] = {0.75 + 0.35 * warmth, 0.85 + 0.10 * warmth, 1.05 - 0.35 * warmth};
        const double w = (present ? amplitude : 0.0) * point;
        for (int k = 0; k < 3; ++k) c[k] = c[k] + w * tint[k];
    }
    const double zz = d[2] / 0.30;
    const double band = 0.035 * exp(-(zz * zz));
    const double band_rgb[3] = {1.0, 0.92, 0.80};
    for (int k = 0; k < 3; ++k) {
        double b = band * band_rgb[k];
        if (shifted) {
            const double slide = np_clip(0.35 * log(np_max(shift, 1e-6)), -0.6, 0.6);
            const double tint = k == 0 ? 1.0 - slide : (k == 1 ? 1.0 : 1.0 + slide);
            b = b * pow(shift, 4.0) * tint;
        }
        c[k] = c[k] + b;
    }
}

void bho_starfield(const double *dirs, const double *shift, int64_t n, double *rgb) {
    for (int64_t i = 0; i < n; ++i)
        starfield_one(dirs + 3 * i, shift ? shift[i] : 0.0, shift != NULL, rgb + 3 * i);
}

static double interp_f32(double x, const double *xp, const float *fp, int64_t n) {
    double buf0 = fp[0], buf1;
    if (isnan(x)) return x;
    if (x < xp[0]) return buf0;
    if (x >= xp[n - 1]) return (double)fp[n - 1];
    int64_t lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    buf0 = fp[lo];
    if (xp[lo] == x) return buf0;
    buf1 = fp[lo + 1];
    const double slope = (buf1 - buf0) / (xp[lo + 1] - xp[lo]);
    return slope * (x - xp[lo]) + buf0;
}

static void disk_one(const bho_emission_params_t *p, const double *pos, const double *mom,
                     const float *temperature, const double *lut_radii, const float *bb,
                     double *c) {
    bho_geometry_t g;
    bho_geometry(p->mass, p->spin, pos[0], pos[1], pos[2], 0, &g);
    const double r = g.r;
    const double t_norm = interp_f32(r, lut_radii, temperature, p->temperature_size);
    /* emission/redshift.py:19-116 with p_t = 1 */
    const double omega = 1.0 / (pow(r, 1.5) + p->spin);
    const double v[3] = {-omega * pos[1], omega * pos[0], 0.0};
    const double ldv = 1.0 + sum3(g.l[0] * v[0], g.l[1] * v[1], g.l[2] * v[2]);
    const double norm2 = -1.0 + sum3(v[0] * v[0], v[1] * v[1], v[2] * v[2]) +
                         2.0 * g.h * ldv * ldv;
    const double u_t = 1.0 / sqrt(-norm2);
    const double u[3] = {u_t * v[0], u_t * v[1], u_t * v[2]};
    const double freq = 1.0 * u_t + sum3(mom[0] * u[0], mom[1] * u[1], mom[2] * u[2]);
    const double shift = p->observer_lapse / freq;
    const double t_obs = np_max(shift * t_norm * p->disk_temperature, 1.0);
    const double log_t = np_clip(log(t_obs), p->bb_log_min, p->bb_log_max);
    const double lut_u = (log_t - p->bb_log_min) / (p->bb_log_max - p->bb_log_min) *
                         (double)(p->blackbody_size - 1);
    const double phi = atan2(pos[1], pos[0]);
    const double detail = 1.0 + p->disk_detail * (0.18 * sin(9.0 * phi + 2.2 * r) +
                                                   0.12 * sin(23.0 * phi - 5.0 * r) +
                                                   0.15 * sin(3.5 * (r - p->disk_inner)));
    const double brightness = pow(t_obs / 6500.0, 4.0) * np_max(detail, 0.2);
    const int64_t nb = p->blackbody_size;
    for (int k = 0; k < 3; ++k) {
        double tint;
        if (isnan(lut_u)) {
            tint = lut_u;
        } else if (lut_u < 0.0) {
            tint = bb[k];
        } else if (lut_u >= (double)(nb - 1)) {
            tint = bb[3 * (nb - 1) + k];
        } else {
            const int64_t lo = (int64_t)floor(lut_u);
            const double f0 = bb[3 * lo + k];
            tint = ((double)lo == lut_u) ? f0 : (bb[3 * (lo + 1) + k] - f0) * (lut_u - (double)lo) + f0;
        }
        c[k] = tint * brightness;
    }
}

void bho_disk_radiance(const bho_emission_params_t *p, const double *pos,
                       const double *mom, int64_t n, const float *temperature,
                       const double *lut_radii, const float *bb_table, double *rgb) {
    for (int64_t i = 0; i < n; ++i)
        disk_one(p, pos + 3 * i, mom + 3 * i, temperature, lut_radii, bb_table, rgb + 3 * i);
}

typedef struct {
    const bho_emission_params_t *p;
    const int32_t *status;
    const double *escape_dir, *hit_pos, *hit_mom, *energy, *lut_radii;
    const float *temperature, *bb;
    float *hdr;
} radiance_ctx_t;

static void radiance_range(void *vctx, int64_t b, int64_t e, int64_t *acc) {
    radiance_ctx_t *c = (radiance_ctx_t *)vctx;
    const bho_emission_params_t *p = c->p;
    const int ss2 = p->supersample * p->supersample;
    (void)acc;
    for (int64_t px = b; px < e; ++px) {
        double sum[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < ss2; ++k) {
            const int64_t i = px * ss2 + k;
            double col[3] = {0.0, 0.0, 0.0};
            const int32_t st = c->status[i];
            if (st == BHO_ESCAPED) {
                const double shift = c->energy ? p->observer_lapse / c->energy[i] : 0.0;
                starfield_one(c->escape_dir + 3 * i, shift, c->energy != NULL, col);
            } else if (st == BHO_DISK) {
                disk_one(p, c->hit_pos + 3 * i, c->hit_mom + 3 * i, c->temperature,
                         c->lut_radii, c->bb, col);
            } else if (st == BHO_TERMINATED) {
                col[0] = p->sheet_rgb[0]; col[1] = p->sheet_rgb[1]; col[2] = p->sheet_rgb[2];
            }
            for (int j = 0; j < 3; ++j) sum[j] = k == 0 ? col[j] : sum[j] + col[j];
        }
        for (int j = 0; j < 3; ++j) c->hdr[3 * px + j] = (float)(sum[j] / (double)ss2);
    }
}

void bho_offline_radiance(const bho_emission_params_t *p, const int32_t *status,
                          const double *escape_dir, const double *hit_pos,
                          const double *hit_mom, const double *energy,
                          int64_t pixels, const float *temperature,
                          const double *lut_radii, const float *bb_table,
                          float *hdr, int nthreads) {
    radiance_ctx_t c = {p, status, escape_dir, hit_pos, hit_mom, energy, lut_radii,
                        temperature, bb_table, hdr};
    bho_parallel_for(pixels, nthreads, 256, radiance_range, &c);
}

/* ------------------------------------------------------ offline/post.py */

static void blur_pass(const float *src, float *dst, int64_t w, int64_t h,
                      const double *wt, int radius, int axis) {
    for (int64_t y = 0; y < h; ++y)
        for (int64_t x = 0; x < w; ++x) {
            float acc[3] = {0.0f, 0.0f, 0.0f};
            for (int t = 0; t <= 2 * radius; ++t) {
                int64_t yy = y, xx = x;
                if (axis == 0) {
                    yy = y + t - radius;
                    yy = yy < 0 ? 0 : (yy >= h ? h - 1 : yy);
                } else {
                    xx = x + t - radius;
                    xx = xx < 0 ? 0 : (xx >= w ? w - 1 : xx);
                }
                const float *s = src + 3 * (yy * w + xx);
                for (int k = 0; k < 3; ++k) acc[k] = (float)((double)acc[k] + wt[t] * (double)s[k]);
            }
            for (int k = 0; k < 3; ++k) dst[3 * (y * w + x) + k] = acc[k];
        }
}

static uint8_t develop_px(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    float m = (x * (a * x + b)) / (x * (c * x + d) + e);
    m = m < 0.0f ? 0.0f : (m > 1.0f ? 1.0f : m);
    const float enc = m <= 0.0031308f ? 12.92f * m
                                      : 1.055f * powf(m, (float)(1.0 / 2.4)) - 0.055f;
    return (uint8_t)(enc * 255.0f + 0.5f);
}

void bho_develop(const float *hdr, int64_t width, int64_t height, double exposure,
                 double bloom_threshold, double bloom_strength,
                 const double *weights, int radius, uint8_t *out) {
    const int64_t n = width * height;
    const float ex = (float)exposure;
    float *img = (float *)malloc((size_t)n * 3 * sizeof(float));
    for (int64_t i = 0; i < 3 * n; ++i) img[i] = hdr[i] * ex;
    if (bloom_strength > 0.0) {
        float *bright = (float *)malloc((size_t)n * 3 * sizeof(float));
        float *tmp = (float *)malloc((size_t)n * 3 * sizeof(float));
        const float thr = (float)bloom_threshold, st = (float)bloom_strength;
        for (int64_t i = 0; i < n; ++i) {
            const float *v = img + 3 * i;
            const float lum = 0.2126f * v[0] + 0.7152f * v[1] + 0.0722f * v[2];
            float excess = lum - thr;
            excess = excess > 0.0f ? excess : 0.0f;
            const float scale = lum > 1e-9f ? excess / (lum + 1e-9f) : 0.0f;
            for (int k = 0; k < 3; ++k) bright[3 * i + k] = v[k] * scale;
        }
        blur_pass(bright, tmp, width, height, weights, radius, 0);
        blur_pass(tmp, bright, width, height, weights, radius, 1);
        for (int64_t i = 0; i < 3 * n; ++i) img[i] = img[i] + st * bright[i];
        free(bright);
        free(tmp);
    }
    for (int64_t i = 0; i < 3 * n; ++i) out[i] = develop_px(img[i]);
    free(img);
}

/* ------------------------------------------ realtime/shaders/kerr_tracer.frag */

typedef struct { float r, h, l[3]; } geo_f_t;

static geo_f_t geo_f(float m, float a, float x, float y, float z) {
    /* kerr_tracer.frag:96-114 */
    geo_f_t g;
    const float a2 = a * a;
    const float q = (x * x + y * y + z * z) - a2;
    float s = sqrtf(q * q + 4.0f * a2 * z * z);
    s = s > 1e-12f ? s : 1e-12f;
    float r2 = 0.5f * (q + s);
    r2 = r2 > 1e-12f ? r2 : 1e-12f;
    const float r = sqrtf(r2);
    float qd = r2 * r2 + a2 * z * z;
    qd = qd > 1e-12f ? qd : 1e-12f;
    g.r = r;
    g.h = m * r * r2 / qd;
    const float inv_r2a2 = 1.0f / (r2 + a2), inv_r = 1.0f / r;
    g.l[0] = (r * x + a * y) * inv_r2a2;
    g.l[1] = (r * y - a * x) * inv_r2a2;
    g.l[2] = z * inv_r;
    return g;
}

static float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
static float fractf(float x) { return x - floorf(x); }

static float tex1d(const float *t, int n, int stride, int col, float s) {
    /* linear filtering between texel centres, repeat wrapping */
    const float u = s * (float)n - 0.5f;
    const float f = floorf(u);
    const float alpha = u - f;
    int i0 = (int)f % n;
    if (i0 < 0) i0 += n;
    const int i1 = (i0 + 1) % n;
    return (1.0f - alpha) * t[i0 * stride + col] + alpha * t[i1 * stride + col];
}

static float hash13f(float x, float y, float z) {
    /* kerr_tracer.frag:243-247 */
    x = fractf(x * 0.1031f);
    y = fractf(y * 0.1031f);
    z = fractf(z * 0.1031f);
    const float d = x * (z + 31.32f) + y * (y + 31.32f) + z * (x + 31.32f);
    x += d; y += d; z += d;
    return fractf((x + y) * z);
}

static float smoothstepf(float e0, float e1, float x) {
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

static void sky_f(int mode, const float *d, float *c) {
    /* kerr_tracer.frag:249-268 */
    const float theta = acosf(clampf(d[2], -1.0f, 1.0f));
    const float phi = atan2f(d[1], d[0]);
    if (mode == 0) {
        const float it = floorf(theta / 3.14159265f * 12.0f);
        const float ip = floorf((phi + 3.14159265f) / 6.2831853f * 2.0f * 12.0f);
        const float sum = it + ip;
        const int light = sum - 2.0f * floorf(sum * 0.5f) >= 1.0f;
        c[0] = light ? 0.408f : 0.094f;
        c[1] = light ? 0.502f : 0.118f;
        c[2] = light ? 0.698f : 0.204f;
        return;
    }
    const float star = powf(hash13f(floorf(d[0] * 220.0f), floorf(d[1] * 220.0f),
                                    floorf(d[2] * 220.0f)), 60.0f);
    const float gt = smoothstepf(0.006f, 0.0f, fabsf(fractf(theta / 0.19635f) - 0.5f) * 0.19635f);
    const float gp = smoothstepf(0.006f, 0.0f, fabsf(fractf(phi / 0.19635f) - 0.5f) * 0.19635f);
    const float g = gt > gp ? gt : gp;
    c[0] = 0.012f + star + 0.02f * g;
    c[1] = 0.014f + star + 0.03f * g;
    c[2] = 0.028f + star + 0.05f * g;
}

static void disk_f(const bho_realtime_shading_t *p, float pt, const float *pos, const float *mom,
                   const float *temperature, const float *bb, float *c) {
    /* kerr_tracer.frag:205-241 */
    const geo_f_t g = geo_f(p->mass, p->spin, pos[0], pos[1], pos[2]);
    const float omega = 1.0f / (powf(g.r, 1.5f) + p->spin);
    const float v[3] = {-omega * pos[1], omega * pos[0], 0.0f};
    const float ldv = 1.0f + (g.l[0] * v[0] + g.l[1] * v[1] + g.l[2] * v[2]);
    const float norm2 = -1.0f + (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + 2.0f * g.h * ldv * ldv;
    const float u_t = 1.0f / sqrtf(-norm2 > 1e-9f ? -norm2 : 1e-9f);
    const float nu = u_t * (pt + (mom[0] * v[0] + mom[1] * v[1] + mom[2] * v[2]));
    const float shift = p->observer_lapse / (nu > 1e-6f ? nu : 1e-6f);
    const float lut_u = clampf((g.r - p->disk_inner) / (p->disk_outer - p->disk_inner), 0.0f, 1.0f);
    const float t_obs = shift * tex1d(temperature, p->temperature_size, 1, 0, lut_u) *
                        p->disk_temperature;
    const float bb_u = clampf((logf(t_obs > 1.0f ? t_obs : 1.0f) - p->bb_log_min) /
                              (p->bb_log_max - p->bb_log_min), 0.0f, 1.0f);
    const float phi = atan2f(pos[1], pos[0]);
    const float detail = 1.0f + p->disk_detail * (0.18f * sinf(9.0f * phi + 2.2f * g.r) +
                                                  0.12f * sinf(23.0f * phi - 5.0f * g.r) +
                                                  0.15f * sinf(3.5f * (g.r - p->disk_inner)));
    const float brightness = p->exposure * powf(t_obs / 6500.0f, 4.0f) * (detail > 0.2f ? detail : 0.2f);
    for (int k = 0; k < 3; ++k) {
        const float col = tex1d(bb, p->blackbody_size, 3, k, bb_u) * brightness;
        c[k] = col / (1.0f + col);
    }
}

void bho_realtime_shade(const bho_realtime_shading_t *p, const int32_t *status,
                        const double *states, const double *hit_pos,
                        const double *hit_mom, int64_t n, const float *temperature,
                        const float *blackbody, uint8_t *rgb) {
    for (int64_t i = 0; i < n; ++i) {
        float c[3] = {0.0f, 0.0f, 0.0f};
        const int32_t st = status[i];
        if (st == BHO_DISK) {
            const float pos[3] = {(float)hit_pos[3 * i], (float)hit_pos[3 * i + 1],
                                  (float)hit_pos[3 * i + 2]};
            const float mom[3] = {(float)hit_mom[4 * i + 1], (float)hit_mom[4 * i + 2],
                                  (float)hit_mom[4 * i + 3]};
            disk_f(p, (float)hit_mom[4 * i], pos, mom, temperature, blackbody, c);
        } else if (st == BHO_ESCAPED) {
            const double *y = states + 8 * i;
            const float pos[3] = {(float)y[1], (float)y[2], (float)y[3]};
            const float pt = (float)y[4];
            const float mom[3] = {(float)y[5], (float)y[6], (float)y[7]};
            const geo_f_t g = geo_f(p->mass, p->spin, pos[0], pos[1], pos[2]);
            const float lp = -pt + (g.l[0] * mom[0] + g.l[1] * mom[1] + g.l[2] * mom[2]);
            float d[3];
            for (int k = 0; k < 3; ++k) d[k] = mom[k] - 2.0f * g.h * lp * g.l[k];
            const float inv = 1.0f / sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            for (int k = 0; k < 3; ++k) d[k] *= inv;
            sky_f(p->background, d, c);
            if (p->sky_amplification > 0.0f) {
                const float gs = p->sky_amplification / (pt > 1e-6f ? pt : 1e-6f);
                const float gain = clampf(gs * gs * gs * gs, 0.0f, 4.0e4f);
                const float slide = clampf(0.35f * logf(gs > 1e-6f ? gs : 1e-6f), -0.6f, 0.6f);
                const float t[3] = {1.0f - slide, 1.0f, 1.0f + slide};
                const float tn = 1.732f / sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
                for (int k = 0; k < 3; ++k) c[k] = c[k] * gain * (t[k] * tn);
            }
        } else if ((st == BHO_CAPTURED || st == BHO_TERMINATED) && p->sheet_radiance > 0.0f) {
            c[0] = p->sheet_radiance * 0.62f;
            c[1] = p->sheet_radiance * 0.78f;
            c[2] = p->sheet_radiance * 1.0f;
        }
        if (p->whiteout > 0.0f) {
            const float w[3] = {0.90f, 0.95f, 1.0f};
            for (int k = 0; k < 3; ++k) c[k] = c[k] * (1.0f - p->whiteout) + w[k] * p->whiteout;
        }
        for (int k = 0; k < 3; ++k) rgb[3 * i + k] = (uint8_t)lrintf(clampf(c[k], 0.0f, 1.0f) * 255.0f);
    }
}

/* ------------------------------------------ offline/inflation.py frame shading */

static double np_mod1(double x) {
    double m = fmod(x, 1.0);
    if (m != 0.0) {
        if (m < 0.0) m += 1.0;
    } else {
        m = 0.0;
    }
    return m;
}

static double sky_hash(double a, double b, double salt) {
    /* inflation.py:140-142 */
    const double h = sin(a * 12.9898 + b * 78.233 + salt * 37.719);
    return np_mod1(h * 43758.5453);
}

static void surrogate_sky(const double *d, double *c) {
    /* inflation.py:138-162 */
    const double theta = acos(np_clip(d[2], -1.0, 1.0));
    const double phi = atan2(d[1], d[0]);
    static const double cells_of[2] = {38.0, 85.0}, bright_of[2] = {1.6, 0.8};
    c[0] = c[1] = c[2] = 0.0;
    for (int layer = 0; layer < 2; ++layer) {
        const double cells = cells_of[layer];
        const double pu = phi / (2.0 * M_PI) * cells, pv = theta / M_PI * cells;
        const double iu = floor(pu), iv = floor(pv);
        const double fu = np_mod1(pu), fv = np_mod1(pv);
        const double cx = sky_hash(iu, iv, 1.0), cy = sky_hash(iu, iv, 2.0);
        const double dist2 = (fu - cx) * (fu - cx) + (fv - cy) * (fv - cy);
        const double mag = sky_hash(iu, iv, 4.0);
        const double amp = bright_of[layer] * (0.2 + pow(mag, 4.0)) * exp(-dist2 / 0.004);
        const double w = sky_hash(iu, iv, 5.0);
        const double tint[3] = {0.6 + 0.4 * w, 0.6 + 0.2 * w, 1.0 - 0.3 * w};
        for (int k = 0; k < 3; ++k) c[k] = c[k] + amp * tint[k];
    }
}

void bho_inflation_radiance(double mass, const int32_t *status, const double *escape_dir,
                            const double *end_mass, int64_t pixels, int supersample,
                            float *hdr) {
    const int ss2 = supersample * supersample;
    const float sheet[3] = {0.62f, 0.78f, 1.0f};
    for (int64_t p = 0; p < pixels; ++p) {
        float acc[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < ss2; ++k) {
            const int64_t i = p * ss2 + k;
            float c[3] = {0.0f, 0.0f, 0.0f};
            if (status[i] == 0) {
                double sky[3];
                surrogate_sky(escape_dir + 3 * i, sky);
                for (int j = 0; j < 3; ++j) c[j] = (float)sky[j];
            } else if (status[i] == 1) {
                const double excess = np_max(end_mass[i] - mass, 0.0) / mass;
                const double lg = log1p(excess);
                const double glow = 0.35 + 1.2 * (lg * lg);
                for (int j = 0; j < 3; ++j) c[j] = (float)(glow * (double)sheet[j]);
            }
            for (int j = 0; j < 3; ++j) acc[j] = k == 0 ? c[j] : acc[j] + c[j];
        }
        for (int j = 0; j < 3; ++j) hdr[3 * p + j] = acc[j] / (float)ss2;
    }
}
