// bh_tile.cu -- the offline renderer's tile tracer: adaptive DP5(4) rays that
// end on the horizon, at the escape sphere, at the step budget or on the
// equatorial accretion disk.
//
// Restates _trace_tile and _refine_crossings (blackhorizon/offline/render.py:
// 184-349) for exterior cameras.  Differences from the plain tracer
// (bh_trace.cu): termination is tested before each attempt, rays still in
// flight at the attempt cap stay IN_FLIGHT, and every accepted step whose z
// changes sign is refined to the crossing point of an RK4 substep from the
// pre-step state.
//
// Scheduling.  Refining a crossing costs about ten RK4 substeps; done inside
// the tracing loop it would stall the other 31 lanes of the warp each time
// one lane crosses, and crossings are frequent (most rays cross the plane at
// least once).  Two cases:
//  - a crossing that the step's chord places clearly off the disk
//    (clear_miss) needs no refinement: the reference's refinement would
//    report a miss and the ray go on from the step's end, which it does in
//    place.  On the offline renderer's default view that is a third of all
//    crossings;
//  - for the others the tracer parks the ray: it writes a crossing record
//    and its slot takes the next ray from the work queue.  A second kernel
//    refines all parked crossings in float64, one per thread, in lock step;
//    a hit finalises the ray, and a miss (a crossing close to a disk edge)
//    writes a resume record for the next round of the tracer.
// Rounds that start with fewer than kInlineRefineBelow resumed rays refine
// their crossings in place, which ends the rounds: such a round's time is
// the latency of its longest ray, and parking again would add one such tail
// per crossing.  The host reads one counter per round.  (Claiming parked
// crossings from inside one persistent launch instead, once its queue
// drains, was measured ten times slower: every idle warp contends for the
// same claim counter.)
//
// Refinement.  The reference bisects the step fraction 40 times
// (render.py:332-339): it ends on the dyadic cell (L, L + 2^-40) with L the
// largest grid point k 2^-40 at which the substep is still on the starting
// side, and takes the cell's midpoint.  Here an Illinois (modified regula
// falsi) iteration converges on the root, the grid points on either side of
// its estimate (and, should those not close the bracket, a bisection over the
// grid points left in it) find the same L, and the crossing is the same
// substep at (L + 1/2) 2^-40: the reference's point, from about 5 RK4
// substeps instead of 41 (at most 7 on the offline renderer's default view).
#include <chrono>
#include <cmath>
#include <cstring>

#include "bh_trace_common.cuh"

namespace bh {

// Termination test before an attempt (render.py:231-260, exterior camera):
// -1 while the ray stays in flight.  r2_est: r^2 of y from the stage
// arithmetic, or NaN; see settled_radius (the interior camera's lowest radius
// threshold is 1.002 capture radii).
__device__ __forceinline__ int tile_check(const TileArgs &a, const RayState &y,
                                          long long steps, long long attempts,
                                          double r2_est) {
    // render.py:223: the loop ends after 4 max_steps iterations.
    if (attempts >= a.max_attempts) return BH_RAY_IN_FLIGHT;
    const double r = settled_radius(
        r2_est, a.interior ? a.capture_radius * 1.002 : a.capture_radius, a.escape_radius,
        a.spin, y);
    if (a.interior) {
        // render.py:234-248: diverging spatial momentum ends the ray on the
        // terminal surface.
        // Rounded as NumPy does it: ((px^2 + py^2) + pz^2), no contraction.
        const double pn = ::sqrt(__dadd_rn(__dadd_rn(__dmul_rn(y.px, y.px), __dmul_rn(y.py, y.py)),
                                           __dmul_rn(y.pz, y.pz)));
        if (r <= a.capture_radius || pn > 1.0e3 || (r <= a.capture_radius * 1.002 && pn > 50.0))
            return BH_RAY_TERMINATED;
    } else if (r <= a.capture_radius) {
        return BH_RAY_CAPTURED;
    }
    if (r >= a.escape_radius) return BH_RAY_ESCAPED;
    if (steps >= a.max_steps) return BH_RAY_MAX_STEPS;
    return -1;
}

// Writes the per-ray outputs of a finished ray.  hit: the refined crossing
// state of a disk hit, else null.  The hit buffers were zeroed before the
// rounds, and the escape directions are computed after them from the final
// states (escape_dir_kernel): both would otherwise be single-lane work inside
// the stepping loop, where the rest of the warp waits.
__device__ __forceinline__ void tile_finalize(const TileArgs &a, long long ray,
                                              const RayState &y, int st, long long steps,
                                              const RayState *hit) {
    store_state(a.states, a.n, a.layout, ray, y);
    a.status[ray] = st;
    a.steps[ray] = steps;
    // render.py:289-291
    a.saturated[ray] = (st == BH_RAY_MAX_STEPS || steps >= a.saturate_steps) ? 1 : 0;
    if (hit) {
        double *hp = a.hit_pos + 3 * ray, *hm = a.hit_mom + 3 * ray;
        hp[0] = hit->x; hp[1] = hit->y; hp[2] = hit->z;
        hm[0] = hit->px; hm[1] = hit->py; hm[2] = hit->pz;
    }
}

// Escape directions of every finished ray, one thread per ray, from the final
// states (render.py:164-181): dx = p - 2 H lp l, lp = -p_t + l.p, normalised;
// zero for rays that did not escape.
__global__ void __launch_bounds__(256) escape_dir_kernel(const TileArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        double *ed = a.escape_dir + 3 * i;
        if (a.status[i] != BH_RAY_ESCAPED) {
            ed[0] = ed[1] = ed[2] = 0.0;
            continue;
        }
        RayState y;
        load_state(a.states, a.n, a.layout, i, y);
        Geometry g;
        geometry_full(a.mass, a.spin, y.x, y.y, y.z, false, g);
        const double lp = -y.pt + ((g.l[0] * y.px + g.l[1] * y.py) + g.l[2] * y.pz);
        const double c = 2.0 * (g.h * lp);
        const double d0 = y.px - c * g.l[0], d1 = y.py - c * g.l[1], d2 = y.pz - c * g.l[2];
        const double nrm = ::sqrt((d0 * d0 + d1 * d1) + d2 * d2);
        ed[0] = d0 / nrm; ed[1] = d1 / nrm; ed[2] = d2 / nrm;
    }
}

// ------------------------------------------------------------ refinement

// rk4_step (integrators.py:57-73) from a fixed state y0 with a variable step:
// k1 = f(y0) is shared by every substep.  float64 throughout.
struct Rk4From {
    KerrV<double> K;
    WStateV<double> w;
    StageV<double> d1;
    double k1x, k1y, k1z;

    __device__ __forceinline__ Rk4From(double m, double a, const RayState &y0) {
        K = make_kerr<double>(m, a);
        put_work<double>(w, 0, y0);
        d1 = first_stage<double>(K, w);
        k1x = w.px + d1.kx; k1y = w.py + d1.ky; k1z = w.pz + d1.kz;
    }

    // The RK4 substep of size hh from y0; only z when !full.
    __device__ __forceinline__ void step(const RayState &y0, double hh, bool full,
                                         RayState &o) const {
        const double half = 0.5 * hh;
        const double e2x = half * d1.px, e2y = half * d1.py, e2z = half * d1.pz;
        const StageV<double> d2 = rhs_v<double>(K, fma(half, k1x, w.x), fma(half, k1y, w.y),
                                                fma(half, k1z, w.z), w.npt, w.px + e2x,
                                                w.py + e2y, w.pz + e2z, e2x, e2y, e2z);
        const double k2x = w.px + d2.kx, k2y = w.py + d2.ky, k2z = w.pz + d2.kz;
        const double e3x = half * d2.px, e3y = half * d2.py, e3z = half * d2.pz;
        const StageV<double> d3 = rhs_v<double>(K, fma(half, k2x, w.x), fma(half, k2y, w.y),
                                                fma(half, k2z, w.z), w.npt, w.px + e3x,
                                                w.py + e3y, w.pz + e3z, e3x, e3y, e3z);
        const double k3x = w.px + d3.kx, k3y = w.py + d3.ky, k3z = w.pz + d3.kz;
        const double e4x = hh * d3.px, e4y = hh * d3.py, e4z = hh * d3.pz;
        const StageV<double> d4 = rhs_v<double>(K, fma(hh, k3x, w.x), fma(hh, k3y, w.y),
                                                fma(hh, k3z, w.z), w.npt, w.px + e4x,
                                                w.py + e4y, w.pz + e4z, e4x, e4y, e4z);
        const double k4z = w.pz + d4.kz;
        const double h6 = hh / 6.0;
        o.z = y0.z + h6 * (k1z + 2.0 * k2z + 2.0 * k3z + k4z);
        if (!full) return;
        const double k4x = w.px + d4.kx, k4y = w.py + d4.ky;
        o.t = y0.t + h6 * (6.0 * w.npt + (d1.thl + 2.0 * d2.thl + 2.0 * d3.thl + d4.thl));
        o.x = y0.x + h6 * (k1x + 2.0 * k2x + 2.0 * k3x + k4x);
        o.y = y0.y + h6 * (k1y + 2.0 * k2y + 2.0 * k3y + k4y);
        o.pt = y0.pt;
        o.px = y0.px + h6 * (d1.px + 2.0 * d2.px + 2.0 * d3.px + d4.px);
        o.py = y0.py + h6 * (d1.py + 2.0 * d2.py + 2.0 * d3.py + d4.py);
        o.pz = y0.pz + h6 * (d1.pz + 2.0 * d2.pz + 2.0 * d3.pz + d4.pz);
    }
};

// The step fraction at which the reference's 40-step bisection ends
// (render.py:332-340), given that y0 and the accepted step lie on opposite
// sides of z = 0.
__device__ __forceinline__ double crossing_fraction(const Rk4From &rk, const RayState &y0,
                                                    double h) {
    constexpr double kCell = 0x1p-40;
    const double z0 = y0.z;
    RayState o;
    auto same_side = [&](double th, double &f) {
        rk.step(y0, h * th, false, o);
        f = o.z;
        return f * z0 > 0.0;
    };
    double f1;
    // No sign change over the whole RK4 step: every bisection test is "same
    // side" and low climbs to 1 - 2^-40.
    if (same_side(1.0, f1)) return 1.0 - 0.5 * kCell;
    // Illinois on [lo, hi]: lo on z0's side, hi not; fa, fb the (possibly
    // halved) values used for interpolation.
    double lo = 0.0, hi = 1.0, fa = z0, fb = f1, th = 0.5;
    int last = 0;
    for (int it = 0; it < 48 && hi - lo > 4.0 * kCell; ++it) {
        th = (lo * fb - hi * fa) / (fb - fa);
        if (!(th > lo && th < hi)) {
            // The secant rounds onto an end of the bracket (or that end's
            // value is exactly 0): the root lies within rounding of it.
            // Falling back to the midpoint here, as plain Illinois does, cost
            // the slowest crossing of a warp about 27 substeps instead of 6.
            th = th <= lo ? lo : hi;
            break;
        }
        double f;
        if (same_side(th, f)) {
            lo = th; fa = f;
            if (last < 0) fb *= 0.5;
            last = -1;
        } else {
            hi = th; fb = f;
            if (last > 0) fa *= 0.5;
            last = 1;
        }
    }
    // The reference tests grid points only.  Grid point kl is at or below lo
    // (on z0's side, as every point below the crossing is), kh at or above
    // hi.  The two grid points on either side of the estimate th usually
    // close the bracket; a bisection over the grid points still inside it
    // finishes any other case.
    double kl = ::floor(lo * 0x1p40), kh = ::ceil(hi * 0x1p40);
    if (kh > 0x1p40) kh = 0x1p40;
    double guess = ::floor(th * 0x1p40);
    for (int p = 0; p < 2 && kh - kl > 1.0; ++p) {
        const double km = ::fmin(::fmax(guess, kl + 1.0), kh - 1.0);
        double f;
        if (same_side(km * kCell, f)) {
            kl = km; guess = km + 1.0;
        } else {
            kh = km; guess = km - 1.0;
        }
    }
    for (int it = 0; it < 48 && kh - kl > 1.0; ++it) {
        const double km = ::floor(0.5 * (kl + kh));
        double f;
        if (same_side(km * kCell, f)) kl = km; else kh = km;
    }
    return (kl + 0.5) * kCell;
}

// Refines one crossing step (render.py:312-349): the crossing state on the
// RK4 substep at the reference's bisection point, and whether its radius is
// on the disk.
__device__ __forceinline__ bool refine_hit(double m, double a, double r_in, double r_out,
                                           const RayState &y0, double h, RayState &yc) {
    const Rk4From rk(m, a, y0);
    const double th = crossing_fraction(rk, y0, h);
    rk.step(y0, h * th, true, yc);
    const double r = ks_radius(a, yc);
    return r >= r_in && r <= r_out;
}

// Where an accepted step whose z changes sign crosses the equatorial plane,
// as far as its chord tells (render.py:268-281 refines the crossing and tests
// its radius against the disk):
//  - kClearMiss: certainly off the disk.  The reference's refinement would
//    report a miss and the ray go on from the step's end (render.py:283-287),
//    which the caller does in place;
//  - kClearHit: certainly on the disk;
//  - kNearEdge: close enough to an edge that only the refinement can tell.
// The step's path lies within (4/27)(|h v0 - d| + |h v1 - d|) of its chord,
// the bound for the cubic Hermite interpolant through the end points x0, x1
// with end velocities v0, v1 (d = x1 - x0), and 1e-6 |d| more covers the
// float32 velocities.  Twice that bound, carried into the plane through the
// chord's slope, plus 4e-6 (1 + rho) for the float32 arithmetic here (about
// 3e-7 rho), must keep the chord's crossing point clear of both disk
// edges (rho_in, rho_out: the edges' cylindrical radii in the plane,
// sqrt(r^2 + a^2)).  NaN anywhere gives kNearEdge.
constexpr int kClearMiss = 0, kClearHit = 1, kNearEdge = 2;
__device__ __forceinline__ int chord_crossing(const RayState &y0, const RayState &y1, float h,
                                              float v0x, float v0y, float v0z, float v1x,
                                              float v1y, float v1z, float rho_in,
                                              float rho_out) {
    const float dx = float(y1.x - y0.x), dy = float(y1.y - y0.y), dz = float(y1.z - y0.z);
    const float ux = fmaf(h, v0x, -dx), uy = fmaf(h, v0y, -dy), uz = fmaf(h, v0z, -dz);
    const float wx = fmaf(h, v1x, -dx), wy = fmaf(h, v1y, -dy), wz = fmaf(h, v1z, -dz);
    const float dxy2 = fmaf(dx, dx, dy * dy);
    const float dev = (4.0f / 27.0f) * (sqrtf(fmaf(ux, ux, fmaf(uy, uy, uz * uz))) +
                                        sqrtf(fmaf(wx, wx, fmaf(wy, wy, wz * wz)))) +
                      1e-6f * sqrtf(fmaf(dz, dz, dxy2));
    const float ts = float(y0.z / (y0.z - y1.z));
    const float px = fmaf(ts, dx, float(y0.x)), py = fmaf(ts, dy, float(y0.y));
    const float rho = sqrtf(fmaf(px, px, py * py));
    const float reach = 2.0f * dev * (1.0f + sqrtf(dxy2) / fabsf(dz)) + 4e-6f * (1.0f + rho);
    if (rho - reach > rho_out || rho + reach < rho_in) return kClearMiss;
    if (rho - reach >= rho_in && rho + reach <= rho_out) return kClearHit;
    return kNearEdge;
}

// INLINE = false: every crossing is parked for the refinement kernel, and
// the misses come back as the next round's resumed rays.  INLINE = true
// (the rounds that start with few resumed rays): crossings are refined in
// place, so no ray needs another round.
template <class V, int BLOCK, int MINB, bool INLINE>
__global__ void __launch_bounds__(BLOCK, MINB) tile_kernel(const TileArgs args) {
    using T = VT<V>;
    constexpr int N = T::N;
    constexpr bool F64 = sizeof(typename T::S) == 8;
    TileWorkspace *ws = args.ws;
    const int par = args.round & 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // Counters of the other parity: used next by this round's refinement
        // (n_resume) and by the next round (queue head, crossing count).
        ws->queue_head[par ^ 1] = 0;
        ws->n_cross[par ^ 1] = 0;
        ws->n_resume[par ^ 1] = 0;
        ws->n_spec[par ^ 1] = 0;
        // This round's refinement and settling claim their crossings from here.
        ws->refine_head[par] = 0;
    }
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long long n_in = args.round == 0 ? args.n : (long long)ws->n_resume[par];
    bool flush = args.flush != 0 || ws->timed_out != 0;
    const bool disk = args.disk_outer > 0.0;
    const double a2 = args.spin * args.spin;
    const float rho_in = float(::sqrt(fma(args.disk_inner, args.disk_inner, a2)));
    const float rho_out = float(::sqrt(fma(args.disk_outer, args.disk_outer, a2)));
    const unsigned long long deadline = global_timer_ns() + (unsigned long long)args.timeout_ns;
    const bool has_deadline = args.timeout_ns > 0;
    const V rt = T::set(args.rtol), at = T::set(args.atol);
    const KerrV<V> K = make_kerr<V>(T::set(args.mass), T::set(args.spin));

    extern __shared__ double bh_state_smem[];
    StateStore<V, BLOCK> ys(bh_state_smem);
    long long ray[N], steps[N], attempts[N];
    double h[N];
    WStateV<V> yw;
#pragma unroll
    for (int l = 0; l < N; ++l) {
        ray[l] = -1; steps[l] = 0; attempts[l] = 0; h[l] = args.initial_step;
        const RayState y0{0.0, 10.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0};
        ys.set(l, y0);
        put_work<V>(yw, l, y0);
    }
    StageV<V> k1 = first_stage<V>(K, yw);
    bool queue_open = true;
    int refill_waited = 0;  // iterations the warp's idle slots have waited
    // Launch counters of this thread, in shared memory: they change once per
    // ray, and in registers they cost the stepping loop five 64-bit values.
    __shared__ unsigned long long cnt[5][BLOCK];  // attempts, accepted, max, crossings, hits
#pragma unroll
    for (int k = 0; k < 5; ++k) cnt[k][threadIdx.x] = 0;
    auto finish = [&](int l, const RayState &y, int st, const RayState *hit) {
        tile_finalize(args, ray[l], y, st, steps[l], hit);
        cnt[0][threadIdx.x] += attempts[l];
        cnt[1][threadIdx.x] += steps[l];
        if ((unsigned long long)attempts[l] > cnt[2][threadIdx.x])
            cnt[2][threadIdx.x] = attempts[l];
        ray[l] = -1;
    };

    for (unsigned iter = 0;; ++iter) {
        // ---- warp-aggregated refill of the idle slots
        unsigned mask[N];
        int total = 0;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            mask[l] = __ballot_sync(full, ray[l] < 0 && queue_open);
            total += __popc(mask[l]);
        }
        bool fresh[N];
#pragma unroll
        for (int l = 0; l < N; ++l) fresh[l] = false;
        // A refill costs the warp one first-stage evaluation however many slots
        // it fills, so idle slots wait for company: at least a batch of
        // them, or a number of iterations (bh_trace_common.cuh).
        const bool do_refill =
            total && (total >= BH_TILE_REFILL_BATCH || refill_waited >= BH_TILE_REFILL_WAIT);
        refill_waited = total && !do_refill ? refill_waited + 1 : 0;
        if (do_refill) {
            unsigned any = 0;
#pragma unroll
            for (int l = 0; l < N; ++l) any |= mask[l];
            const int leader = __ffs(any) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&ws->queue_head[par], (unsigned long long)total);
            base = __shfl_sync(full, base, leader);
            int before = 0;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                if ((mask[l] >> lane) & 1u) {
                    const long long idx = (long long)base + before + __popc(mask[l] & lt_mask);
                    if (idx < n_in) {
                        RayState y0;
                        if (args.round == 0) {
                            load_state(args.state0, args.n, args.layout, idx, y0);
                            ray[l] = idx; steps[l] = 0; attempts[l] = 0;
                            h[l] = args.initial_step;
                        } else {
                            const TileResume &r = args.resume[idx];
                            y0 = RayState{r.y[0], r.y[1], r.y[2], r.y[3],
                                          r.y[4], r.y[5], r.y[6], r.y[7]};
                            ray[l] = r.ray; steps[l] = r.steps; attempts[l] = r.attempts;
                            h[l] = r.h;
                        }
                        const int st = flush ? BH_RAY_IN_FLIGHT
                                             : tile_check(args, y0, steps[l], attempts[l],
                                                          __longlong_as_double(0x7ff8000000000000LL));
                        if (st >= 0) {
                            finish(l, y0, st, nullptr);
                        } else {
                            fresh[l] = true;
                            ys.set(l, y0);
                            put_work<V>(yw, l, y0);
                        }
                    }
                }
                before += __popc(mask[l]);
            }
            if ((long long)base + total >= n_in) queue_open = false;
        }
        bool any_fresh = false;
#pragma unroll
        for (int l = 0; l < N; ++l) any_fresh |= fresh[l];
        if (any_fresh) {
            const StageV<V> f = first_stage<V>(K, yw);
            take_stage(k1, f, fresh);
        }
        bool active = false;
#pragma unroll
        for (int l = 0; l < N; ++l) active |= ray[l] >= 0;
        if (!__any_sync(full, active || queue_open)) break;

        if (active) {
            // ---- one iteration of render.py:262-287 for every slot
            V hw = T::set(0.0);
#pragma unroll
            for (int l = 0; l < N; ++l) T::put(hw, l, typename T::S(h[l]));
            AttemptV<V> a;
            dp5_attempt<V>(K, yw, hw, k1, a);
            RatioT<V> ratio[N];
            error_ratio_v<V>(yw, a, hw, rt, at, ratio, h);
            bool acc[N];
#pragma unroll
            for (int l = 0; l < N; ++l) {
                acc[l] = false;
                if (ray[l] < 0) continue;
                acc[l] = ratio[l] <= RatioT<V>(1);
                ++attempts[l];
                const double h_next =
                    next_step<F64>(h[l], ratio[l], args.max_step);
                if (acc[l]) {
                    const RayState y0 = ys.get(l);
                    RayState y1 = y0;
                    commit<V>(y1, yw, a, l, h[l]);
                    const bool crosses = disk && y0.z * y1.z < 0.0;
                    const int where =
                        crosses ? chord_crossing(y0, y1, float(h[l]),
                                                 float(y0.px) + float(T::get(k1.kx, l)),
                                                 float(y0.py) + float(T::get(k1.ky, l)),
                                                 float(y0.pz) + float(T::get(k1.kz, l)),
                                                 float(y1.px) + float(T::get(a.k7.kx, l)),
                                                 float(y1.py) + float(T::get(a.k7.ky, l)),
                                                 float(y1.pz) + float(T::get(a.k7.kz, l)),
                                                 rho_in, rho_out)
                                : kClearMiss;
                    if (crosses && where == kClearMiss) {
                        // A miss decided by the chord: the ray goes on in place.
                        ++cnt[3][threadIdx.x];
                    } else if (crosses && INLINE) {
                        // The last rounds refine in place: a parked miss would
                        // come back in yet another round.
                        RayState yc;
                        ++cnt[3][threadIdx.x];
                        if (refine_hit(args.mass, args.spin, args.disk_inner, args.disk_outer,
                                       y0, h[l], yc)) {
                            ++cnt[4][threadIdx.x];
                            finish(l, y0, BH_RAY_DISK, &yc);
                            acc[l] = false;
                            continue;
                        }
                    } else if (crosses) {
                        // render.py:268-281: a record for the refinement.  Near a
                        // disk edge the ray goes on in place, as after a miss,
                        // and the refinement overwrites its outcome should the
                        // crossing be a hit (refine_kernel, settle_kernel); else
                        // the ray is parked and its slot takes the next ray.
                        TileCrossing *rec = nullptr;
                        bool go_on = false;
                        if (where == kNearEdge) {
                            const unsigned long long k = atomicAdd(&ws->n_spec[par], 1ull);
                            if (k < (unsigned long long)args.spec_cap) {
                                rec = &args.spec[k];
                                go_on = true;
                            }
                        }
                        if (!go_on) rec = &args.cross[atomicAdd(&ws->n_cross[par], 1ull)];
                        TileCrossing &c = *rec;
                        c.y0[0] = y0.t; c.y0[1] = y0.x; c.y0[2] = y0.y; c.y0[3] = y0.z;
                        c.y0[4] = y0.pt; c.y0[5] = y0.px; c.y0[6] = y0.py; c.y0[7] = y0.pz;
                        c.y1[0] = y1.t; c.y1[1] = y1.x; c.y1[2] = y1.y; c.y1[3] = y1.z;
                        c.y1[4] = y1.pt; c.y1[5] = y1.px; c.y1[6] = y1.py; c.y1[7] = y1.pz;
                        c.h = h[l];
                        c.h_next = h_next;
                        c.steps = steps[l];
                        c.attempts = attempts[l];
                        c.ray = ray[l];
                        c.speculative = go_on ? 1 : 0;
                        c.hit = 0;
                        if (go_on) {
                            args.has_spec[ray[l]] = 1;
                        } else {
                            ray[l] = -1;
                            acc[l] = false;
                            continue;
                        }
                    }
                    ys.set(l, y1);
                    ++steps[l];
                }
                h[l] = h_next;
                int st = -1;
                if (attempts[l] >= args.max_attempts) st = BH_RAY_IN_FLIGHT;
                else if (acc[l])
                    st = tile_check(args, ys.get(l), steps[l], attempts[l],
                                    double(T::get(a.r2n, l)));
                if (st >= 0) finish(l, ys.get(l), st, nullptr);
            }
            take_stage(k1, a.k7, acc);
        }

        // ---- bounded launch time: past the deadline every ray in flight,
        // and every ray still queued, is finalised as IN_FLIGHT.
        if (has_deadline && !flush && (iter & 7u) == 0u) {
            const bool late = global_timer_ns() > deadline;
            if (__any_sync(full, late)) {
                flush = true;
#pragma unroll
                for (int l = 0; l < N; ++l)
                    if (ray[l] >= 0) finish(l, ys.get(l), BH_RAY_IN_FLIGHT, nullptr);
                if (lane == 0) atomicExch(&ws->timed_out, 1);
            }
        }
    }
    unsigned long long my_attempts = cnt[0][threadIdx.x], my_accepted = cnt[1][threadIdx.x];
    long long my_max_attempts = (long long)cnt[2][threadIdx.x];
    unsigned long long my_cross = cnt[3][threadIdx.x], my_hits = cnt[4][threadIdx.x];
    for (int off = 16; off > 0; off >>= 1) {
        my_attempts += __shfl_down_sync(full, my_attempts, off);
        my_accepted += __shfl_down_sync(full, my_accepted, off);
        my_cross += __shfl_down_sync(full, my_cross, off);
        my_hits += __shfl_down_sync(full, my_hits, off);
        const long long o = __shfl_down_sync(full, my_max_attempts, off);
        my_max_attempts = o > my_max_attempts ? o : my_max_attempts;
    }
    if (lane == 0) {
        atomicAdd(&ws->attempts, my_attempts);
        atomicAdd(&ws->accepted, my_accepted);
        atomicMax(&ws->iterations, my_max_attempts);
        if (my_cross) {
            atomicAdd(&ws->crossings, my_cross);
            atomicAdd(&ws->disk_hits, my_hits);
        }
    }
}

// The crossing records of a round: the parked ones, then the speculative ones
// (the index space of refine_kernel and settle_kernel).
__device__ __forceinline__ long long crossing_count(const TileArgs &a, int par,
                                                   long long *parked) {
    const long long nc = (long long)a.ws->n_cross[par];
    const unsigned long long ns = a.ws->n_spec[par];
    *parked = nc;
    return nc + (long long)(ns < (unsigned long long)a.spec_cap ? ns
                                                                 : (unsigned long long)a.spec_cap);
}

__device__ __forceinline__ TileCrossing &crossing_at(const TileArgs &a, long long parked,
                                                     long long i) {
    return i < parked ? a.cross[i] : a.spec[i - parked];
}

// Appends resume records for the lanes with miss set (render.py:283-287: the
// ray continues from the accepted state).  Every lane of the warp calls it.
__device__ __forceinline__ void append_resumed(const TileArgs &a, int par, bool miss,
                                               const TileCrossing *c) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(full, miss);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned long long b = 0;
    if (lane == leader) b = atomicAdd(&a.ws->n_resume[par ^ 1], (unsigned long long)__popc(m));
    b = __shfl_sync(full, b, leader);
    if (miss) {
        TileResume &r = a.resume[b + __popc(m & ((1u << lane) - 1u))];
#pragma unroll
        for (int k = 0; k < 8; ++k) r.y[k] = c->y1[k];
        r.h = c->h_next;
        r.steps = c->steps + 1;
        r.attempts = c->attempts;
        r.ray = c->ray;
    }
}

// Refines every crossing record of the round in float64, one per thread.  A
// ray without speculative records has this one record: a hit finalises it and
// a miss resumes it.  For a ray with speculative records (it went on past a
// crossing near a disk edge) the record keeps its outcome, and the ray's
// earliest hit is kept in first_hit; settle_kernel resolves those rays.
__global__ void __launch_bounds__(128) refine_kernel(const TileArgs args) {
    TileWorkspace *ws = args.ws;
    const int par = args.round & 1;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    long long parked = 0;
    const long long count = crossing_count(args, par, &parked);
    unsigned long long my_cross = 0, my_hits = 0, my_attempts = 0, my_accepted = 0;
    long long my_max = 0;
    // Warps claim 32 crossings at a time: a chunk's time is that of its
    // slowest crossing (the iteration counts differ), so a fixed split
    // would leave warps idle while others finish.
    for (;;) {
        unsigned long long chunk = 0;
        if (lane == 0) chunk = atomicAdd(&ws->refine_head[par], 1ull);
        chunk = __shfl_sync(full, chunk, 0);
        const long long base = (long long)chunk * 32;
        if (base >= count) break;
        const long long i = base + lane;
        bool miss = false;
        TileCrossing *cp = nullptr;
        if (i < count) {
            cp = &crossing_at(args, parked, i);
            TileCrossing &c = *cp;
            const RayState y0{c.y0[0], c.y0[1], c.y0[2], c.y0[3],
                              c.y0[4], c.y0[5], c.y0[6], c.y0[7]};
            RayState yc;
            ++my_cross;
            const bool hit = refine_hit(args.mass, args.spin, args.disk_inner, args.disk_outer,
                                        y0, c.h, yc);
            if (args.has_spec[c.ray]) {
                c.hit = hit ? 1 : 0;
                if (hit) {
                    c.y1[0] = yc.t; c.y1[1] = yc.x; c.y1[2] = yc.y; c.y1[3] = yc.z;
                    c.y1[4] = yc.pt; c.y1[5] = yc.px; c.y1[6] = yc.py; c.y1[7] = yc.pz;
                    atomicMin(&args.first_hit[c.ray], (unsigned long long)c.steps);
                }
            } else if (hit) {
                // render.py:278-281 and 283-286: DISK, state and steps as
                // before the step.
                tile_finalize(args, c.ray, y0, BH_RAY_DISK, c.steps, &yc);
                ++my_hits;
                my_attempts += c.attempts;
                my_accepted += c.steps;
                if (c.attempts > my_max) my_max = c.attempts;
            } else {
                miss = true;
            }
        }
        append_resumed(args, par, miss, cp);
    }
    for (int off = 16; off > 0; off >>= 1) {
        my_cross += __shfl_down_sync(full, my_cross, off);
        my_hits += __shfl_down_sync(full, my_hits, off);
        my_attempts += __shfl_down_sync(full, my_attempts, off);
        my_accepted += __shfl_down_sync(full, my_accepted, off);
        const long long o = __shfl_down_sync(full, my_max, off);
        my_max = o > my_max ? o : my_max;
    }
    if (lane == 0 && my_cross) {
        atomicAdd(&ws->crossings, my_cross);
        atomicAdd(&ws->disk_hits, my_hits);
        atomicAdd(&ws->attempts, my_attempts);
        atomicAdd(&ws->accepted, my_accepted);
        atomicMax(&ws->iterations, my_max);
    }
}

// Resolves the rays with speculative records after refine_kernel: the record
// of the ray's earliest hit finalises it as DISK (over whatever its
// continuation wrote: the reference stops at that crossing); with no hit, a
// parked record's miss resumes the ray.  The attempt counters then include
// the continuation's attempts past a crossing that proved a hit.
__global__ void __launch_bounds__(128) settle_kernel(const TileArgs args) {
    TileWorkspace *ws = args.ws;
    const int par = args.round & 1;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    long long parked = 0;
    const long long count = crossing_count(args, par, &parked);
    unsigned long long my_hits = 0, my_attempts = 0, my_accepted = 0;
    long long my_max = 0;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long warp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (long long base = warp * 32; base < count; base += warps * 32) {
        const long long i = base + lane;
        bool miss = false;
        const TileCrossing *cp = nullptr;
        if (i < count) {
            cp = &crossing_at(args, parked, i);
            const TileCrossing &c = *cp;
            if (args.has_spec[c.ray]) {
                const unsigned long long first = args.first_hit[c.ray];
                if (c.hit && (unsigned long long)c.steps == first) {
                    const RayState y0{c.y0[0], c.y0[1], c.y0[2], c.y0[3],
                                      c.y0[4], c.y0[5], c.y0[6], c.y0[7]};
                    const RayState yc{c.y1[0], c.y1[1], c.y1[2], c.y1[3],
                                      c.y1[4], c.y1[5], c.y1[6], c.y1[7]};
                    tile_finalize(args, c.ray, y0, BH_RAY_DISK, c.steps, &yc);
                    ++my_hits;
                    my_attempts += c.attempts;
                    my_accepted += c.steps;
                    if (c.attempts > my_max) my_max = c.attempts;
                } else if (!c.hit && !c.speculative && first == ~0ull) {
                    miss = true;
                }
            }
        }
        append_resumed(args, par, miss, cp);
    }
    for (int off = 16; off > 0; off >>= 1) {
        my_hits += __shfl_down_sync(full, my_hits, off);
        my_attempts += __shfl_down_sync(full, my_attempts, off);
        my_accepted += __shfl_down_sync(full, my_accepted, off);
        const long long o = __shfl_down_sync(full, my_max, off);
        my_max = o > my_max ? o : my_max;
    }
    if (lane == 0 && my_hits) {
        atomicAdd(&ws->disk_hits, my_hits);
        atomicAdd(&ws->attempts, my_attempts);
        atomicAdd(&ws->accepted, my_accepted);
        atomicMax(&ws->iterations, my_max);
    }
}

// ------------------------------------------------------------ launches

template <class V, int B, int M>
static const void *tile_fn(bool inl, size_t *smem) {
    *smem = StateStore<V, B>::shared_bytes();
    return inl ? (const void *)tile_kernel<V, B, M, true>
               : (const void *)tile_kernel<V, B, M, false>;
}

// Same launch shapes as the tracer's variants (bh_trace.cu).
static const void *tile_kernel_for(int precision, int idx, bool inl, size_t *smem) {
    if (precision == BH_PRECISION_MIXED) {
        switch (idx) {
            case 0: return tile_fn<float, 128, 3>(inl, smem);
            case 1: return tile_fn<float, 128, 4>(inl, smem);
            case 2: return tile_fn<float, 128, 5>(inl, smem);
            case 3: return tile_fn<float, 256, 2>(inl, smem);
            case 4: return tile_fn<F2, 128, 2>(inl, smem);
            case 5: return tile_fn<F2, 128, 3>(inl, smem);
            case 6: return tile_fn<F2, 64, 4>(inl, smem);
            default: return tile_fn<F2, 256, 1>(inl, smem);
        }
    }
    switch (idx) {
        case 0: return tile_fn<double, 128, 2>(inl, smem);
        case 1: return tile_fn<double, 128, 3>(inl, smem);
        case 2: return tile_fn<double, 128, 4>(inl, smem);
        default: return tile_fn<double, 256, 2>(inl, smem);
    }
}

// Measured on the offline renderer's 1280x800 supersample-2 frame (one
// round, refill batching): mixed 11.8 ms with one float ray per thread at
// 128 x 5 (96 registers), 12.3-12.4 ms at 128 x 3, 128 x 4 and 256 x 2,
// 14.5-16.3 ms packed two per thread (the parking and refill work does not
// pack); float64 24.9 ms at 256 x 2, 25.4 ms at 128 x 4, 26.4 ms at 128 x 3,
// 30.0 ms at 128 x 2.
int tile_default_variant(int precision) {
    return precision == BH_PRECISION_MIXED ? 2 : 3;
}

cudaError_t launch_tile(const TileArgs &args, int precision, int variant,
                        int blocks_per_sm, cudaStream_t stream) {
    if (variant < 0 || variant >= trace_variant_count(precision))
        variant = tile_default_variant(precision);
    const Variant v = trace_variant(precision, variant);
    size_t smem = 0;
    const void *fn = tile_kernel_for(precision, variant, args.inline_refine != 0, &smem);
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, v.block, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    TileArgs a = args;
    void *params[] = {(void *)&a};
    return cudaLaunchKernel(fn, dim3((unsigned)((long long)sms * per_sm)), dim3(v.block),
                            params, smem, stream);
}

// Resumed rays are reordered before the next round, most attempts so far
// first: rays that reach their first equatorial crossing only after many
// small steps are those winding near the photon sphere, which keep going
// longest after a miss.  Started first, they run beside the bulk of the
// round instead of after it, when the other slots would idle.  A counting
// sort by attempts (8 per bucket); the order inside a bucket does not matter,
// because every ray's result is independent of its slot.
constexpr int kResumeBuckets = 128;
// Rounds with fewer resumed rays than this refine their crossings in place.
constexpr unsigned long long kInlineRefineBelow = 65536;
struct TileResumeSort {
    unsigned count[kResumeBuckets];
    unsigned cursor[kResumeBuckets];
};
static_assert(sizeof(TileResumeSort) == 1024, "resume sort counters are 1 KiB");

__device__ __forceinline__ int resume_bucket(const TileResume &r) {
    const long long b = r.attempts >> 3;
    return (int)(b < kResumeBuckets - 1 ? b : kResumeBuckets - 1);
}

__global__ void __launch_bounds__(256) resume_count_kernel(const TileResume *in, long long n,
                                                           TileResumeSort *srt) {
    __shared__ unsigned hist[kResumeBuckets];
    for (int b = threadIdx.x; b < kResumeBuckets; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        atomicAdd(&hist[resume_bucket(in[i])], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kResumeBuckets; b += blockDim.x)
        if (hist[b]) atomicAdd(&srt->count[b], hist[b]);
}

__global__ void resume_offsets_kernel(TileResumeSort *srt) {
    if (threadIdx.x != 0) return;
    unsigned acc = 0;
    for (int b = kResumeBuckets - 1; b >= 0; --b) {
        srt->cursor[b] = acc;
        acc += srt->count[b];
    }
}

// Each block places a tile of 256 records: ranks within the tile from
// shared-memory counters, one global reservation per non-empty bucket.
__global__ void __launch_bounds__(256) resume_scatter_kernel(const TileResume *in, long long n,
                                                             TileResumeSort *srt,
                                                             TileResume *out) {
    __shared__ unsigned cnt[kResumeBuckets], base[kResumeBuckets];
    for (long long t0 = (long long)blockIdx.x * blockDim.x; t0 < n;
         t0 += (long long)gridDim.x * blockDim.x) {
        for (int b = threadIdx.x; b < kResumeBuckets; b += blockDim.x) cnt[b] = 0;
        __syncthreads();
        const long long i = t0 + threadIdx.x;
        const bool valid = i < n;
        TileResume r;
        int b = 0;
        unsigned rank = 0;
        if (valid) {
            r = in[i];
            b = resume_bucket(r);
            rank = atomicAdd(&cnt[b], 1u);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kResumeBuckets; k += blockDim.x)
            if (cnt[k]) base[k] = atomicAdd(&srt->cursor[k], cnt[k]);
        __syncthreads();
        if (valid) out[base[b] + rank] = r;
        __syncthreads();
    }
}

// Reorders in[0, n) into out (counters in srt, zeroed here).
static cudaError_t sort_resumed(const TileResume *in, long long n, TileResumeSort *srt,
                                TileResume *out, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(srt, 0, sizeof(TileResumeSort), stream);
    if (e != cudaSuccess) return e;
    const long long need = (n + 255) / 256;
    const unsigned grid = (unsigned)(need < 4LL * sms ? need : 4LL * sms);
    resume_count_kernel<<<grid, 256, 0, stream>>>(in, n, srt);
    resume_offsets_kernel<<<1, 32, 0, stream>>>(srt);
    resume_scatter_kernel<<<grid, 256, 0, stream>>>(in, n, srt, out);
    return cudaGetLastError();
}

cudaError_t launch_refine(const TileArgs &args, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, refine_kernel, 128, 0);
    if (e != cudaSuccess) return e;
    refine_kernel<<<sms * (occ > 0 ? occ : 1), 128, 0, stream>>>(args);
    settle_kernel<<<sms * 4, 128, 0, stream>>>(args);
    return cudaGetLastError();
}

static int tile_invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

static int tile_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return BH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BH_ERR_CUDA;
}

}  // namespace bh

using namespace bh;

// Speculative crossing records a tile holds; past them a crossing near a disk
// edge is parked like any other.  On the offline renderer's default view
// about one ray in 1,600 records one.
static long long spec_capacity(long long n) {
    const long long c = n / 8 + 1024;
    return c < n ? c : n;
}

// Workspace: header, resume-sort counters, parked and speculative crossing
// records, two resume arrays (the second receives the reordered records),
// each ray's first hit and speculative flag.
extern "C" size_t bh_trace_tile_workspace_bytes(int64_t n) {
    if (n < 0) n = 0;
    return sizeof(TileWorkspace) + sizeof(TileResumeSort) +
           (size_t)(n + spec_capacity(n)) * sizeof(TileCrossing) +
           (size_t)n * (2 * sizeof(TileResume) + sizeof(unsigned long long)) +
           (size_t)((n + 15) / 16 * 16);
}

extern "C" int bh_trace_tile(const bh_trace_config *config, const bh_scene *scene,
                             double disk_inner, double disk_outer, const double *state0,
                             int64_t n, double *states, int32_t *status, int64_t *steps,
                             double *hit_positions, double *hit_momenta,
                             double *escape_directions, int8_t *saturated,
                             void *workspace, size_t workspace_bytes,
                             bh_tile_stats *stats, void *stream) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!config || !scene) return tile_invalid("config and scene must not be NULL");
    const bh_trace_config &c = *config;
    if (c.precision != BH_PRECISION_FP64 && c.precision != BH_PRECISION_MIXED)
        return tile_invalid("precision must be BH_PRECISION_FP64 or BH_PRECISION_MIXED");
    if (c.layout != BH_LAYOUT_AOS && c.layout != BH_LAYOUT_SOA)
        return tile_invalid("layout must be BH_LAYOUT_AOS or BH_LAYOUT_SOA");
    if (!(c.rtol >= 0.0) || !(c.atol >= 0.0) || !(c.rtol > 0.0 || c.atol > 0.0))
        return tile_invalid("rtol and atol must be >= 0 and not both zero");
    if (!(c.initial_step > 0.0) || !(c.max_step > 0.0))
        return tile_invalid("initial_step and max_step must be > 0");
    if (c.max_steps < 1 || c.max_steps > (1LL << 60))
        return tile_invalid("max_steps must be in [1, 2^60]");
    if (c.timeout_ns < 0) return tile_invalid("timeout_ns must be >= 0");
    if (c.flags & ~BH_TRACE_INTERIOR) return tile_invalid("unknown config flags");
    if (c.reserved != 0) return tile_invalid("config reserved field must be 0");
    if (c.f64_radius != 0.0) return tile_invalid("f64_radius is accepted by bh_propagate only");
    if ((c.flags & BH_TRACE_INTERIOR) && !(scene->capture_radius > 0.0))
        return tile_invalid("an interior camera needs a stop radius > 0");
    if (!(scene->mass > 0.0) || !(std::fabs(scene->spin) <= scene->mass))
        return tile_invalid("Kerr bound violated or mass not positive");
    if (disk_outer > 0.0 && !(disk_inner >= 0.0 && disk_inner <= disk_outer))
        return tile_invalid("disk radii must satisfy 0 <= disk_inner <= disk_outer");
    if (n < 0) return tile_invalid("n must be >= 0");
    if (n == 0) return BH_OK;
    if (!state0 || !states || !status || !steps || !hit_positions || !hit_momenta ||
        !escape_directions || !saturated)
        return tile_invalid("NULL pointer argument");
    if (c.layout == BH_LAYOUT_AOS &&
        ((reinterpret_cast<uintptr_t>(state0) | reinterpret_cast<uintptr_t>(states)) & 15u))
        return tile_invalid("state buffers must be 16-byte aligned");
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) ||
        workspace_bytes < bh_trace_tile_workspace_bytes(n)) {
        set_error("workspace must be 256-byte aligned and hold bh_trace_tile_workspace_bytes(n)");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *base = static_cast<char *>(workspace);
    TileArgs a;
    std::memset(&a, 0, sizeof(a));
    a.state0 = state0;
    a.n = n;
    a.layout = c.layout;
    a.mass = scene->mass;
    a.spin = scene->spin;
    a.capture_radius = scene->capture_radius;
    a.interior = (c.flags & BH_TRACE_INTERIOR) ? 1 : 0;
    a.escape_radius = scene->escape_radius;
    a.disk_inner = disk_inner;
    a.disk_outer = disk_outer;
    a.rtol = c.rtol;
    a.atol = c.atol;
    a.initial_step = c.initial_step;
    a.max_step = c.max_step;
    a.max_steps = c.max_steps;
    a.max_attempts = 4 * c.max_steps;
    a.saturate_steps = (long long)(0.85 * (double)c.max_steps);
    a.ws = reinterpret_cast<TileWorkspace *>(base);
    TileResumeSort *resume_sort = reinterpret_cast<TileResumeSort *>(base + sizeof(TileWorkspace));
    a.cross = reinterpret_cast<TileCrossing *>(base + sizeof(TileWorkspace) +
                                               sizeof(TileResumeSort));
    a.spec_cap = spec_capacity(n);
    a.spec = a.cross + n;
    a.resume = reinterpret_cast<TileResume *>(a.spec + a.spec_cap);
    TileResume *resume_sorted = a.resume + n;
    a.first_hit = reinterpret_cast<unsigned long long *>(resume_sorted + n);
    a.has_spec = reinterpret_cast<int8_t *>(a.first_hit + n);
    a.states = states;
    a.status = status;
    a.steps = steps;
    a.hit_pos = hit_positions;
    a.hit_mom = hit_momenta;
    a.escape_dir = escape_directions;
    a.saturated = saturated;
    int rc = tile_cuda(cudaMemsetAsync(base, 0, sizeof(TileWorkspace), s), "bh_trace_tile reset");
    if (rc != BH_OK) return rc;
    rc = tile_cuda(cudaMemsetAsync(a.first_hit, 0xff, (size_t)n * sizeof(unsigned long long), s),
                   "bh_trace_tile reset");
    if (rc != BH_OK) return rc;
    rc = tile_cuda(cudaMemsetAsync(a.has_spec, 0, (size_t)n, s), "bh_trace_tile reset");
    if (rc != BH_OK) return rc;
    // Rays that end off the disk report zero hit position and momentum.
    rc = tile_cuda(cudaMemsetAsync(hit_positions, 0, (size_t)n * 3 * sizeof(double), s),
                   "bh_trace_tile hit reset");
    if (rc != BH_OK) return rc;
    rc = tile_cuda(cudaMemsetAsync(hit_momenta, 0, (size_t)n * 3 * sizeof(double), s),
                   "bh_trace_tile hit reset");
    if (rc != BH_OK) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    // Each round moves every resumed ray past at least one accepted step.
    // max_steps + 2 rounds bound the loop; past that a flush round finalises
    // whatever is left.
    const long long max_rounds = c.max_steps + 2;
    int rounds = 0;
    bool flush = false, host_late = false;
    unsigned long long entering = (unsigned long long)n;  // rays of this round
    for (long long r = 0;; ++r) {
        if (r >= max_rounds) flush = true;
        a.round = r == 0 ? 0 : (r & 1 ? 1 : 2);
        // A crossing refined in place runs about ten float64 RK4 substeps
        // for one lane while the warp's other lanes wait; parked crossings
        // are refined one per thread.  Rounds park them while many rays
        // remain and refine in place once few do, which ends the rounds.
        a.inline_refine = r > 0 && entering < kInlineRefineBelow ? 1 : 0;
        a.flush = flush ? 1 : 0;
        if (c.timeout_ns > 0) {
            const long long used = std::chrono::duration_cast<std::chrono::nanoseconds>(
                                       std::chrono::steady_clock::now() - t0).count();
            a.timeout_ns = c.timeout_ns - used;
            if (a.timeout_ns <= 0) { a.flush = 1; a.timeout_ns = 0; host_late = true; }
        }
        rc = tile_cuda(launch_tile(a, c.precision, c.variant, c.blocks_per_sm, s),
                       "bh_trace_tile launch");
        if (rc != BH_OK) return rc;
        rc = tile_cuda(launch_refine(a, s), "bh_trace_tile refinement launch");
        if (rc != BH_OK) return rc;
        ++rounds;
        // Rays resumed for the next round (written by this refinement).
        unsigned long long next = 0;
        const int np = (a.round & 1) ^ 1;
        rc = tile_cuda(cudaMemcpyAsync(&next, &a.ws->n_resume[np], sizeof(next),
                                       cudaMemcpyDeviceToHost, s),
                       "bh_trace_tile counter read");
        if (rc != BH_OK) return rc;
        rc = tile_cuda(cudaStreamSynchronize(s), "bh_trace_tile round");
        if (rc != BH_OK) return rc;
        if (next == 0 || a.flush) break;
        entering = next;
        if (r == 0 && next >= 1024 && next < (1ull << 31)) {
            rc = tile_cuda(sort_resumed(a.resume, (long long)next, resume_sort, resume_sorted, s),
                           "bh_trace_tile resume ordering");
            if (rc != BH_OK) return rc;
            a.resume = resume_sorted;
        }
    }
    {
        int dev = 0, sms = 0;
        rc = tile_cuda(cudaGetDevice(&dev), "bh_trace_tile device");
        if (rc != BH_OK) return rc;
        rc = tile_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                       "bh_trace_tile device");
        if (rc != BH_OK) return rc;
        const long long need = (n + 255) / 256;
        escape_dir_kernel<<<(unsigned)(need < 8LL * sms ? need : 8LL * sms), 256, 0, s>>>(a);
        rc = tile_cuda(cudaGetLastError(), "bh_trace_tile escape directions");
        if (rc != BH_OK) return rc;
    }
    TileWorkspace hw;
    rc = tile_cuda(cudaMemcpyAsync(&hw, a.ws, sizeof(hw), cudaMemcpyDeviceToHost, s),
                   "bh_trace_tile stats read");
    if (rc != BH_OK) return rc;
    rc = tile_cuda(cudaStreamSynchronize(s), "bh_trace_tile stats");
    if (rc != BH_OK) return rc;
    if (stats) {
        stats->iterations = hw.iterations;
        stats->attempts = (int64_t)hw.attempts;
        stats->accepted = (int64_t)hw.accepted;
        stats->crossings = (int64_t)hw.crossings;
        stats->disk_hits = (int64_t)hw.disk_hits;
        stats->rounds = rounds;
        stats->timed_out = hw.timed_out || host_late ? 1 : 0;
    }
    if (hw.timed_out || host_late) {
        set_error("bh_trace_tile: deadline passed; rays in flight were left IN_FLIGHT");
        return BH_ERR_TIMEOUT;
    }
    return BH_OK;
}
