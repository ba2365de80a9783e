// bh_vaidya.cu -- the charged-Vaidya/Ori mass-inflation surrogate on the
// device: its time-dependent Kerr-Schild geometry, the extended Hamiltonian
// flow and the mass-inflation renderer's tile tracer.
//
// Restates blackhorizon/vaidya.py:87-394 and offline/inflation.py:165-240.
// The spacetime is spherical, g = eta + 2 H l l with l = x / r and
//     H(v, r) = m(v, r) / r - q^2 / (2 r^2),  v = t + r,
// where m(v, r) is the Price-tail mass m1(v) outside the outgoing Ori shell
// and m1(v) plus the inflated excess m2(v) - m1(v) inside it, blended over
// the shell width.  The shell radius R(v) and m2(v) come from a table (the
// co-integrated shell ODE, vaidya.py:181-237) that the library integrates on
// the host (bh_vaidya_shell_table) and the caller keeps in device memory;
// the device interpolates it as numpy.interp does.  dH/dt and dH/dr use the
// reference's central differences (eps = 1e-4).  Because p_t is not
// conserved, the flow carries dp_t/dlambda = (dH/dt) lp^2.
#include <cmath>
#include <cstring>

#include "bh_trace_common.cuh"

namespace bh {

struct VaidyaDev {
    double mass, charge, q2, tail_mass, tail_start, tail_power, shell_start_v, shell_width,
        mass_cap;
    double tail_unit;  // tail_start / tail_start, rounded on the host
    const double *sv, *sr, *sm2;
    long long n;
};

// numpy.interp for an increasing table: end values outside, exact table
// values at nodes, slope (x - x_j) + y_j between.  vd_locate finds the
// bracket xp[lo] <= x < xp[lo + 1] of an interior x (xp[0] <= x <
// xp[n - 1]); vd_locate_near finds it from the bracket of a nearby point,
// the same index the bisection gives.  vd_interp_slope evaluates the bracket
// with its slope from vd_slope.
__device__ __forceinline__ long long vd_locate(double x, const double *xp, long long n) {
    long long lo = 0, hi = n - 1;
    while (hi - lo > 1) {  // xp[lo] <= x < xp[hi]
        const long long mid = (lo + hi) >> 1;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ long long vd_locate_near(double x, long long lo, const double *xp,
                                                    long long n) {
    for (int k = 0; k < 4; ++k) {
        if (xp[lo] > x) --lo;
        else if (xp[lo + 1] <= x) ++lo;
        else return lo;
    }
    return vd_locate(x, xp, n);
}
__device__ __forceinline__ double vd_slope(long long lo, const double *xp, const double *fp) {
    return __ddiv_rn(__dsub_rn(fp[lo + 1], fp[lo]), __dsub_rn(xp[lo + 1], xp[lo]));
}
__device__ __forceinline__ double vd_interp_slope(double x, long long lo, const double *xp,
                                                  const double *fp, double slope) {
    if (xp[lo] == x) return fp[lo];
    return __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[lo])), fp[lo]);
}

// vaidya.py:153-159: m1(v) = M - dm (v_tail / max(v, v_tail))^(p - 1).
// Before the tail (v <= v_tail) the base is v_tail / v_tail, the same
// correctly rounded quotient on the host, and it is 1 for a finite positive
// v_tail; pow(1, y) = 1 for every y (C99 F.9.4.4, as CUDA's pow).  The values
// are the reference's without the division or the pow, which the
// flythrough's rays (v below v_tail) never need.
__device__ __forceinline__ double vd_m1(const VaidyaDev &d, double v) {
    const double base = v <= d.tail_start ? d.tail_unit : d.tail_start / np_max(v, d.tail_start);
    return d.mass - d.tail_mass * (base == 1.0 ? 1.0 : ::pow(base, d.tail_power - 1.0));
}

// The v-dependent parts of m(v, r) (vaidya.py:244-269): the Price-tail mass
// m1(v), the shell radius R(v) and the inflated excess, clipped.  The two
// table columns share one bracket.  VdBracket carries a bracket and its two
// slopes to a nearby v: the search starts there (the bisection's bracket all
// the same) and the slopes, a function of the bracket alone, are reused while
// it holds.  It takes v's bracket (unchanged for v outside the table); lo = -1
// before the first look-up.
struct VdMassAt {
    double m1, shell_r, inc;
};
struct VdBracket {
    long long lo;
    double k_r, k_m2;
};
__device__ __forceinline__ VdMassAt vd_mass_at(const VaidyaDev &d, double v, VdBracket *b) {
    VdMassAt o;
    double m2;
    if (v != v) {
        o.shell_r = v;
        m2 = v;
    } else if (v < d.sv[0]) {
        o.shell_r = d.sr[0];
        m2 = d.sm2[0];
    } else if (v >= d.sv[d.n - 1]) {
        o.shell_r = d.sr[d.n - 1];
        m2 = d.sm2[d.n - 1];
    } else {
        const long long j =
            b->lo >= 0 ? vd_locate_near(v, b->lo, d.sv, d.n) : vd_locate(v, d.sv, d.n);
        if (j != b->lo) {
            b->lo = j;
            b->k_r = vd_slope(j, d.sv, d.sr);
            b->k_m2 = vd_slope(j, d.sv, d.sm2);
        }
        o.shell_r = vd_interp_slope(v, j, d.sv, d.sr, b->k_r);
        m2 = vd_interp_slope(v, j, d.sv, d.sm2, b->k_m2);
    }
    o.m1 = vd_m1(d, v);
    o.inc = 0.0;
    if (!(v < d.shell_start_v)) o.inc = np_min(np_max(m2 - o.m1, 0.0), d.mass_cap);
    return o;
}

// m(v, r) from the v-dependent parts: the blend across the shell width w.
// Correctly rounded division is monotone, so R - r >= w gives a quotient >= 1
// and R - r <= -w one <= -1: the clip's 1 and 0, taken without the division.
__device__ __forceinline__ double vd_mass_r(const VaidyaDev &d, const VdMassAt &a, double r) {
    const double dr = a.shell_r - r;
    const double t = dr >= d.shell_width    ? 1.0
                     : dr <= -d.shell_width ? 0.0
                                            : np_min(np_max(dr / d.shell_width + 0.5, 0.0), 1.0);
    const double blend = t * t * (3.0 - 2.0 * t);
    return a.m1 + blend * a.inc;
}

// vaidya.py:244-269: m(v, r).
__device__ __forceinline__ double vd_mass(const VaidyaDev &d, double v, double r) {
    VdBracket b{-1, 0.0, 0.0};
    return vd_mass_r(d, vd_mass_at(d, v, &b), r);
}

struct VaidyaGeo {
    double h, l[3], hs, ht, r, ir;
};

// vaidya.py:285-325 (geometry_t).  The reference's twelve quotients by r, r^2,
// r^3 and 2 eps (here and in vd_rhs) are products with one reciprocal 1 / r
// (rcp_f64: the MUFU seed and two Newton steps): each differs from the
// quotient by an ulp or two, and float64 division is the dearest operation of
// the RHS (the flythrough tile takes half the time; its statuses are
// unchanged).  hint (may be null): the ray's bracket from
// its previous evaluation (VdBracket), which takes v's.  A ray's v moves little
// between evaluations, so the search costs a load or two instead of a
// bisection's chain of dependent loads, and the slopes seldom change.
__device__ __forceinline__ void vd_geometry(const VaidyaDev &d, double t, double x, double y,
                                            double z, VaidyaGeo &g, VdBracket *hint = nullptr) {
    const double r = np_max(::sqrt((x * x + y * y) + z * z), 1e-9);
    const double ir = rcp_f64(r);  // r >= 1e-9: within 2 ulp of 1 / r, no slow path
    g.r = r;
    g.ir = ir;
    g.l[0] = x * ir; g.l[1] = y * ir; g.l[2] = z * ir;
    const double v = t + r, eps = 1e-4;
    // The five mass samples of the central differences need the v-dependent
    // parts at three times only, and v +- eps lie in or next to v's bracket.
    VdBracket b = hint ? *hint : VdBracket{-1, 0.0, 0.0};
    const VdMassAt a0 = vd_mass_at(d, v, &b);
    if (hint) *hint = b;
    VdBracket b_p = b, b_m = b;
    const VdMassAt ap = vd_mass_at(d, v + eps, &b_p);
    const VdMassAt am = vd_mass_at(d, v - eps, &b_m);
    const double m0 = vd_mass_r(d, a0, r);
    const double i2e = 1.0 / (2.0 * eps);
    const double m_v = (vd_mass_r(d, ap, r) - vd_mass_r(d, am, r)) * i2e;
    const double m_r = (vd_mass_r(d, a0, r + eps) - vd_mass_r(d, a0, r - eps)) * i2e;
    const double ir2 = ir * ir;
    g.h = m0 * ir - 0.5 * d.q2 * ir2;
    const double h_v = m_v * ir;
    const double h_r = m_r * ir - m0 * ir2 + d.q2 * ir2 * ir;
    g.hs = h_v + h_r;
    g.ht = h_v;
}

// vaidya.py:356-394 (vaidya_geodesic_rhs).
__device__ __forceinline__ RayState vd_rhs(const VaidyaDev &d, const RayState &y,
                                           VdBracket *hint = nullptr) {
    VaidyaGeo g;
    vd_geometry(d, y.t, y.x, y.y, y.z, g, hint);
    const double l_dot_p = (g.l[0] * y.px + g.l[1] * y.py) + g.l[2] * y.pz;
    const double lp = -y.pt + l_dot_p;
    const double lp2 = lp * lp;
    const double c = 2.0 * g.h * lp;
    const double k = c * g.ir;
    RayState o;
    o.t = -y.pt + c;
    o.x = y.px - c * g.l[0];
    o.y = y.py - c * g.l[1];
    o.z = y.pz - c * g.l[2];
    o.pt = g.ht * lp2;
    o.px = g.hs * g.l[0] * lp2 + k * (y.px - l_dot_p * g.l[0]);
    o.py = g.hs * g.l[1] * lp2 + k * (y.py - l_dot_p * g.l[1]);
    o.pz = g.hs * g.l[2] * lp2 + k * (y.pz - l_dot_p * g.l[2]);
    return o;
}

__device__ __forceinline__ RayState vd_axpy(const RayState &y, double a, const RayState &k) {
    return RayState{y.t + a * k.t, y.x + a * k.x, y.y + a * k.y, y.z + a * k.z,
                    y.pt + a * k.pt, y.px + a * k.px, y.py + a * k.py, y.pz + a * k.pz};
}

// rk4_step (integrators.py:57-73) with the surrogate's RHS, all float64.  The
// four stages run as a loop over one copy of the RHS, whose inlined code
// would otherwise be four times the instruction cache's worth; the stage
// offsets (h/2, h/2, h) and the weighted sum ((k1 + 2 k2) + 2 k3) + k4 are
// the same operations in the same order, though the compiler may fuse other
// multiply-adds than in the unrolled form (last-place differences; the
// reference, in NumPy, fuses none).
__device__ __forceinline__ void vd_rk4(const VaidyaDev &d, RayState &y, double h,
                                       VdBracket *hint = nullptr) {
    RayState k = y, acc = y;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        const RayState in = s == 0 ? y : vd_axpy(y, s == 3 ? h : 0.5 * h, k);
        k = vd_rhs(d, in, hint);
        if (s == 0) {
            acc = k;
        } else {
            const double w = s == 3 ? 1.0 : 2.0;
            acc = RayState{acc.t + w * k.t,   acc.x + w * k.x,   acc.y + w * k.y,
                           acc.z + w * k.z,   acc.pt + w * k.pt, acc.px + w * k.px,
                           acc.py + w * k.py, acc.pz + w * k.pz};
        }
    }
    const double h6 = h / 6.0;
    y.t += h6 * acc.t;
    y.x += h6 * acc.x;
    y.y += h6 * acc.y;
    y.z += h6 * acc.z;
    y.pt += h6 * acc.pt;
    y.px += h6 * acc.px;
    y.py += h6 * acc.py;
    y.pz += h6 * acc.pz;
}

__device__ __forceinline__ long long vd_tid() {
    return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}

__global__ void vd_geometry_kernel(const VaidyaDev d, const double *t, const double *x,
                                   const double *y, const double *z, long long n, double *h,
                                   double *l, double *hs, double *ht, double *r) {
    const long long i = vd_tid();
    if (i >= n) return;
    VaidyaGeo g;
    vd_geometry(d, t[i], x[i], y[i], z[i], g);
    h[i] = g.h;
    l[3 * i] = g.l[0]; l[3 * i + 1] = g.l[1]; l[3 * i + 2] = g.l[2];
    hs[i] = g.hs;
    ht[i] = g.ht;
    r[i] = g.r;
}

__global__ void vd_mass_kernel(const VaidyaDev d, const double *v, const double *r,
                               long long n, double *m, double *ms) {
    const long long i = vd_tid();
    if (i >= n) return;
    const double mm = vd_mass(d, v[i], r[i]);
    if (m) m[i] = mm;
    // vaidya.py:271-278
    if (ms) ms[i] = mm - d.q2 / (2.0 * r[i]);
}

__global__ void vd_rhs_kernel(const VaidyaDev d, const double *states, double *out, long long n) {
    const long long i = vd_tid();
    if (i >= n) return;
    RayState y;
    load_state(states, n, BH_LAYOUT_AOS, i, y);
    store_state(out, n, BH_LAYOUT_AOS, i, vd_rhs(d, y));
}

__global__ void vd_rk4_kernel(const VaidyaDev d, const double *states, const double *h,
                              double *out, long long n, long long n_steps) {
    const long long i = vd_tid();
    if (i >= n) return;
    RayState y;
    load_state(states, n, BH_LAYOUT_AOS, i, y);
    const double hi = h[i];
    for (long long s = 0; s < n_steps; ++s) vd_rk4(d, y, hi);
    store_state(out, n, BH_LAYOUT_AOS, i, y);
}

struct VaidyaTraceArgs {
    VaidyaDev d;
    const double *state0;
    long long n, max_steps;
    double escape_radius, stop_radius, r_plus;
    double *states, *escape_dir, *end_mass, *v_end;
    int32_t *status;
    TraceWorkspace *ws;
};

// offline/inflation.py:165-240 (_trace_vaidya_tile): fixed RK4 steps of
// clip(0.15 L, 3e-3, 0.08), L = r - r_plus outside the outer horizon and
// r/2 inside; status 0 escaped (direction of p - 2 H lp l on the t = 0
// slice), 1 terminal surface (r <= stop, or r <= 1.08 stop with |p|^2 > 400,
// or |p|^2 > 1e6; the Misner-Sharp mass there), 2 budget.  Persistent grid,
// idle slots refilled from the work queue.
__global__ void __launch_bounds__(128) vd_trace_kernel(const VaidyaTraceArgs a) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long long n = a.n;
    long long ray = -1, it = 0;
    VdBracket vb{-1, 0.0, 0.0};  // the ray's last table bracket (vd_geometry)
    RayState y{0.0, 10.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0};
    bool queue_open = true;
    unsigned long long my_steps = 0;
    long long my_max = 0;
    auto finish = [&](int st) {
        store_state(a.states, n, BH_LAYOUT_AOS, ray, y);
        a.status[ray] = st;
        a.v_end[ray] = y.t + ::sqrt((y.x * y.x + y.y * y.y) + y.z * y.z);
        my_steps += (unsigned long long)it;
        if (it > my_max) my_max = it;
        ray = -1;
    };
    for (;;) {
        const unsigned mask = __ballot_sync(full, ray < 0 && queue_open);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            unsigned long long base = 0;
            if (lane == leader)
                base = atomicAdd(&a.ws->queue_head, (unsigned long long)__popc(mask));
            base = __shfl_sync(full, base, leader);
            if ((mask >> lane) & 1u) {
                const long long idx = (long long)base + __popc(mask & lt_mask);
                if (idx < n) {
                    load_state(a.state0, n, BH_LAYOUT_AOS, idx, y);
                    ray = idx;
                    it = 0;
                    vb.lo = -1;
                    double *e = a.escape_dir + 3 * idx;
                    e[0] = e[1] = e[2] = 0.0;
                    a.end_mass[idx] = 0.0;
                }
            }
            if ((long long)base + __popc(mask) >= n) queue_open = false;
        }
        if (!__any_sync(full, ray >= 0 || queue_open)) break;
        bool step = false;
        double h = 0.0;
        if (ray >= 0) {
            if (it >= a.max_steps) {
                finish(2);
            } else {
                const double r = ::sqrt((y.x * y.x + y.y * y.y) + y.z * y.z);
                const double mom2 = (y.px * y.px + y.py * y.py) + y.pz * y.pz;
                const bool captured = (r <= a.stop_radius) ||
                                      ((r <= a.stop_radius * 1.08) && (mom2 > 400.0)) ||
                                      (mom2 > 1.0e6);
                if (captured) {
                    a.end_mass[ray] = vd_mass(a.d, y.t + r, r) - a.d.q2 / (2.0 * r);
                    finish(1);
                } else if (r >= a.escape_radius) {
                    VaidyaGeo g;
                    vd_geometry(a.d, 0.0, y.x, y.y, y.z, g);
                    const double lp = -y.pt + ((g.l[0] * y.px + g.l[1] * y.py) + g.l[2] * y.pz);
                    const double c = 2.0 * g.h * lp;
                    const double d0 = y.px - c * g.l[0], d1 = y.py - c * g.l[1],
                                 d2 = y.pz - c * g.l[2];
                    const double nrm = ::sqrt((d0 * d0 + d1 * d1) + d2 * d2);
                    double *e = a.escape_dir + 3 * ray;
                    e[0] = d0 / nrm; e[1] = d1 / nrm; e[2] = d2 / nrm;
                    finish(0);
                } else {
                    const double scale = r > a.r_plus ? r - a.r_plus : 0.5 * r;
                    h = np_min(np_max(0.15 * scale, 3e-3), 0.08);
                    step = true;
                }
            }
        }
        if (!step) continue;
        vd_rk4(a.d, y, h, &vb);
        ++it;
    }
    for (int off = 16; off > 0; off >>= 1) {
        my_steps += __shfl_down_sync(full, my_steps, off);
        const long long o = __shfl_down_sync(full, my_max, off);
        my_max = o > my_max ? o : my_max;
    }
    if (lane == 0) {
        atomicAdd(&a.ws->attempts, my_steps);
        atomicAdd(&a.ws->accepted, my_steps);
        atomicMax(&a.ws->iterations, my_max);
    }
}

static int vd_invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

static int vd_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return BH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BH_ERR_CUDA;
}

// Parameter checks of vaidya.py:121-135 and a usable table.
static int vd_dev(const bh_vaidya *s, VaidyaDev &d) {
    if (!s) return vd_invalid("spacetime is NULL");
    if (!(s->charge > 0.0 && s->charge < s->mass)) return vd_invalid("charge must lie in (0, mass)");
    if (!s->shell_v || !s->shell_r || !s->shell_m2 || s->n_shell < 1)
        return vd_invalid("the shell table (device, n_shell >= 1 rows) is missing");
    if (!(s->shell_width > 0.0)) return vd_invalid("shell_width must be positive");
    d.mass = s->mass;
    d.charge = s->charge;
    d.q2 = std::pow(s->charge, 2.0);
    d.tail_mass = s->tail_mass;
    d.tail_start = s->tail_start;
    d.tail_unit = s->tail_start / s->tail_start;
    d.tail_power = s->tail_power;
    d.shell_start_v = s->shell_start_v;
    d.shell_width = s->shell_width;
    d.mass_cap = s->mass_cap;
    d.sv = s->shell_v;
    d.sr = s->shell_r;
    d.sm2 = s->shell_m2;
    d.n = s->n_shell;
    return BH_OK;
}

static unsigned vd_grid(long long n) {
    const long long g = (n + 127) / 128;
    return (unsigned)(g < 1 ? 1 : g);
}

// ---- host: the shell table (vaidya.py:181-237), float64 in the
// reference's evaluation order.
static double h_m1(const bh_vaidya *p, double v) {
    const double vs = v > p->tail_start ? v : p->tail_start;
    return p->mass - p->tail_mass * std::pow(p->tail_start / vs, p->tail_power - 1.0);
}

static double h_rate(const bh_vaidya *p, double v) {
    if (!(v >= p->tail_start)) return 0.0;
    const double vs = v > p->tail_start ? v : p->tail_start;
    return p->tail_mass * (p->tail_power - 1.0) * std::pow(p->tail_start, p->tail_power - 1.0) /
           std::pow(vs, p->tail_power);
}

static double h_f(const bh_vaidya *p, double m, double r) {
    return 1.0 - 2.0 * m / r + std::pow(p->charge, 2.0) / std::pow(r, 2.0);
}

// ----------------------------------------------- the mass-inflation frame

// numpy.remainder(x, 1.0): fmod, moved into [0, 1).
__device__ __forceinline__ double mod1(double x) {
    double m = ::fmod(x, 1.0);
    if (m != 0.0) {
        if (m < 0.0) m = __dadd_rn(m, 1.0);
    } else {
        m = 0.0;
    }
    return m;
}

// offline/inflation.py:140-142: (sin(a 12.9898 + b 78.233 + salt 37.719)
// 43758.5453) mod 1.
__device__ __forceinline__ double sky_hash(double a, double b, double salt37) {
    const double h = ::sin(__dadd_rn(__dadd_rn(__dmul_rn(a, 12.9898), __dmul_rn(b, 78.233)),
                                     salt37));
    return mod1(__dmul_rn(h, 43758.5453));
}

// offline/inflation.py:138-162 (_surrogate_sky) for one unit direction,
// float64 in NumPy's operation order.
__device__ void surrogate_sky(const double *d, double c[3]) {
    const double theta = ::acos(np_min(np_max(d[2], -1.0), 1.0));
    const double phi = ::atan2(d[1], d[0]);
    c[0] = c[1] = c[2] = 0.0;
#pragma unroll
    for (int layer = 0; layer < 2; ++layer) {
        const double cells = layer == 0 ? 38.0 : 85.0;
        const double brightness = layer == 0 ? 1.6 : 0.8;
        const double pu = __dmul_rn(__ddiv_rn(phi, 2.0 * M_PI), cells);
        const double pv = __dmul_rn(__ddiv_rn(theta, M_PI), cells);
        const double iu = ::floor(pu), iv = ::floor(pv);
        const double fu = mod1(pu), fv = mod1(pv);
        const double cx = sky_hash(iu, iv, 37.719), cy = sky_hash(iu, iv, 2.0 * 37.719);
        const double du = __dsub_rn(fu, cx), dv = __dsub_rn(fv, cy);
        const double dist2 = __dadd_rn(__dmul_rn(du, du), __dmul_rn(dv, dv));
        const double mag = sky_hash(iu, iv, 4.0 * 37.719);
        const double amp = __dmul_rn(__dmul_rn(brightness, __dadd_rn(0.2, ::pow(mag, 4.0))),
                                     ::exp(__ddiv_rn(-dist2, 0.004)));
        const double warmth = sky_hash(iu, iv, 5.0 * 37.719);
        const double tint[3] = {__dadd_rn(0.6, __dmul_rn(0.4, warmth)),
                                __dadd_rn(0.6, __dmul_rn(0.2, warmth)),
                                __dsub_rn(1.0, __dmul_rn(0.3, warmth))};
#pragma unroll
        for (int k = 0; k < 3; ++k) c[k] = __dadd_rn(c[k], __dmul_rn(amp, tint[k]));
    }
}

// offline/inflation.py:322-346: escaped rays (status 0) take the surrogate
// sky, rays ended in the layer (status 1) glow by the Misner-Sharp mass
// excess, rays out of budget are black; each ray's radiance is stored as
// float32, and the supersamples of a pixel are averaged in float32.
__global__ void inflation_radiance_kernel(double mass, const int32_t *status,
                                          const double *escape_dir, const double *end_mass,
                                          long long pixels, int ss2, float *hdr) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const float sheet[3] = {0.62f, 0.78f, 1.0f};
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int k = 0; k < ss2; ++k) {
        const long long i = p * ss2 + k;
        float c[3] = {0.0f, 0.0f, 0.0f};
        if (status[i] == 0) {
            double sky[3];
            surrogate_sky(escape_dir + 3 * i, sky);
            c[0] = (float)sky[0]; c[1] = (float)sky[1]; c[2] = (float)sky[2];
        } else if (status[i] == 1) {
            const double excess = __ddiv_rn(np_max(__dsub_rn(end_mass[i], mass), 0.0), mass);
            const double lg = ::log1p(excess);
            const double glow = __dadd_rn(0.35, __dmul_rn(1.2, __dmul_rn(lg, lg)));
#pragma unroll
            for (int j = 0; j < 3; ++j) c[j] = (float)__dmul_rn(glow, (double)sheet[j]);
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[j] = k == 0 ? c[j] : __fadd_rn(acc[j], c[j]);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) hdr[3 * p + j] = __fdiv_rn(acc[j], (float)ss2);
}

}  // namespace bh

using namespace bh;

extern "C" int bh_inflation_radiance(double mass, const int32_t *status,
                                     const double *escape_directions, const double *end_mass,
                                     int64_t width, int64_t height, int32_t supersample,
                                     float *hdr, void *stream) {
    if (!(mass > 0.0) || width < 0 || height < 0 || supersample < 1)
        return vd_invalid("mass must be > 0, width and height >= 0, supersample >= 1");
    const long long pixels = (long long)width * height;
    if (pixels == 0) return BH_OK;
    if (!status || !escape_directions || !end_mass || !hdr)
        return vd_invalid("NULL pointer argument");
    inflation_radiance_kernel<<<vd_grid(pixels), 128, 0, (cudaStream_t)stream>>>(
        mass, status, escape_directions, end_mass, pixels, supersample * supersample, hdr);
    return vd_launch("bh_inflation_radiance launch");
}

extern "C" int64_t bh_vaidya_shell_table(const bh_vaidya *p, double *vs, double *rs,
                                         double *m2s, int64_t capacity) {
    if (!p || capacity < 0) return -1;
    double v = p->shell_start_v, radius = p->shell_start_radius;
    double m2 = h_m1(p, v) + p->shell_energy;
    int64_t k = 0;
    auto put = [&]() {
        if (k < capacity && vs && rs && m2s) { vs[k] = v; rs[k] = radius; m2s[k] = m2; }
        ++k;
    };
    put();
    const double step = 0.01;
    for (int64_t it = 0; it < 4000000; ++it) {
        const double m1 = h_m1(p, v), lum = h_rate(p, v);
        const double f1 = h_f(p, m1, radius), f2 = h_f(p, m2, radius);
        if (m2 >= p->mass_cap || std::fabs(f1) < 1e-300) break;
        const double r_half = radius + 0.25 * step * f1;
        const double m2_half = m2 + 0.5 * step * lum * f2 / f1;
        const double v_half = v + 0.5 * step;
        const double m1_half = h_m1(p, v_half), lum_half = h_rate(p, v_half);
        const double f1_half = h_f(p, m1_half, r_half), f2_half = h_f(p, m2_half, r_half);
        radius += 0.5 * step * f1_half;
        m2 += step * lum_half * f2_half / f1_half;
        if (p->mass_cap < m2) m2 = p->mass_cap;
        v += step;
        put();
    }
    return k;
}

extern "C" int bh_vaidya_geometry(const bh_vaidya *spacetime, const double *t, const double *x,
                                  const double *y, const double *z, int64_t n, double *h,
                                  double *l, double *h_spatial_scale, double *h_t,
                                  double *radius, void *stream) {
    VaidyaDev d;
    const int rc = vd_dev(spacetime, d);
    if (rc != BH_OK) return rc;
    if (n < 0) return vd_invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!t || !x || !y || !z || !h || !l || !h_spatial_scale || !h_t || !radius)
        return vd_invalid("NULL pointer argument");
    vd_geometry_kernel<<<vd_grid(n), 128, 0, (cudaStream_t)stream>>>(
        d, t, x, y, z, n, h, l, h_spatial_scale, h_t, radius);
    return vd_launch("bh_vaidya_geometry launch");
}

extern "C" int bh_vaidya_mass(const bh_vaidya *spacetime, const double *v, const double *r,
                              int64_t n, double *mass, double *misner_sharp, void *stream) {
    VaidyaDev d;
    const int rc = vd_dev(spacetime, d);
    if (rc != BH_OK) return rc;
    if (n < 0) return vd_invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!v || !r || (!mass && !misner_sharp)) return vd_invalid("NULL pointer argument");
    vd_mass_kernel<<<vd_grid(n), 128, 0, (cudaStream_t)stream>>>(d, v, r, n, mass, misner_sharp);
    return vd_launch("bh_vaidya_mass launch");
}

extern "C" int bh_vaidya_rhs(const bh_vaidya *spacetime, const double *states, double *deriv,
                             int64_t n, void *stream) {
    VaidyaDev d;
    const int rc = vd_dev(spacetime, d);
    if (rc != BH_OK) return rc;
    if (n < 0) return vd_invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!states || !deriv) return vd_invalid("NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(states) | reinterpret_cast<uintptr_t>(deriv)) & 15u)
        return vd_invalid("state buffers must be 16-byte aligned");
    vd_rhs_kernel<<<vd_grid(n), 128, 0, (cudaStream_t)stream>>>(d, states, deriv, n);
    return vd_launch("bh_vaidya_rhs launch");
}

extern "C" int bh_vaidya_rk4(const bh_vaidya *spacetime, const double *states, const double *h,
                             double *out, int64_t n, int64_t n_steps, void *stream) {
    VaidyaDev d;
    const int rc = vd_dev(spacetime, d);
    if (rc != BH_OK) return rc;
    if (n < 0 || n_steps < 0) return vd_invalid("n and n_steps must be >= 0");
    if (n == 0) return BH_OK;
    if (!states || !h || !out) return vd_invalid("NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(states) | reinterpret_cast<uintptr_t>(out)) & 15u)
        return vd_invalid("state buffers must be 16-byte aligned");
    vd_rk4_kernel<<<vd_grid(n), 128, 0, (cudaStream_t)stream>>>(d, states, h, out, n, n_steps);
    return vd_launch("bh_vaidya_rk4 launch");
}

extern "C" int bh_vaidya_trace(const bh_vaidya *spacetime, const double *state0, int64_t n,
                               double escape_radius, double stop_radius, int64_t max_steps,
                               double *states, int32_t *status, double *escape_dir,
                               double *end_mass, double *v_end, void *workspace, void *stream) {
    VaidyaTraceArgs a;
    const int rc = vd_dev(spacetime, a.d);
    if (rc != BH_OK) return rc;
    if (n < 0 || max_steps < 0) return vd_invalid("n and max_steps must be >= 0");
    if (!(escape_radius > 0.0) || !(stop_radius >= 0.0))
        return vd_invalid("escape_radius must be positive and stop_radius >= 0");
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(TraceWorkspace), s);
    if (e != cudaSuccess) {
        set_error("bh_vaidya_trace workspace reset: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    if (n == 0) return BH_OK;
    if (!state0 || !states || !status || !escape_dir || !end_mass || !v_end)
        return vd_invalid("NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(state0) | reinterpret_cast<uintptr_t>(states)) & 15u)
        return vd_invalid("state buffers must be 16-byte aligned");
    a.state0 = state0;
    a.n = n;
    a.max_steps = max_steps;
    a.escape_radius = escape_radius;
    a.stop_radius = stop_radius;
    a.r_plus = spacetime->mass + std::sqrt(std::pow(spacetime->mass, 2.0) -
                                           std::pow(spacetime->charge, 2.0));
    a.states = states;
    a.status = status;
    a.escape_dir = escape_dir;
    a.end_mass = end_mass;
    a.v_end = v_end;
    a.ws = reinterpret_cast<TraceWorkspace *>(workspace);
    int dev = 0, sms = 0, occ = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)vd_trace_kernel, 128, 0);
    if (e != cudaSuccess) {
        set_error("bh_vaidya_trace launch setup: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    long long blocks = (long long)sms * (occ < 1 ? 1 : occ);
    const long long need = (n + 127) / 128;
    if (blocks > need) blocks = need;
    vd_trace_kernel<<<(unsigned)blocks, 128, 0, s>>>(a);
    return vd_launch("bh_vaidya_trace launch");
}
