// bh_trace.cu -- persistent adaptive tracer and lock-step propagator.
//
// trace_kernel restates the per-ray body of trace_rays (blackhorizon/
// tracer.py:100-157): one DP5(4) attempt per iteration, accept when the error
// ratio is <= 1, step update on accept and reject, then the termination
// cascade on the post-step state.  A ray in flight at batch iteration k of the
// reference has made exactly k attempts, so the batch-global cap of
// 4*max_steps iterations (tracer.py:101) becomes a per-ray attempt cap and the
// reference's `iterations` is the maximum attempt count over rays.
//
// Scheduling: N rays per thread (N = 1, or 2 in the packed float32x2 lane
// type); float64 states in registers for float64 lanes, in shared memory for
// float32 lanes (StateStore).  The grid is persistent (blocks_per_sm x SMs);
// a ray slot whose ray terminates takes the next ray from a global work queue.
// Refills are warp-aggregated: __ballot_sync collects the idle slots of the
// warp, one lane claims that many rays with a single atomicAdd and each idle
// slot takes its rank.  Every wait is bounded: each ray makes at most
// max_attempts attempts and a %globaltimer deadline ends the launch with a
// status flag.
#include <cstdio>

#include "bh_trace_common.cuh"

namespace bh {

// The scene of a ray slot: the launch's own for a state-array launch
// (cam < 0), else that of the slot's camera.  A slot keeps only the camera's
// index: four per-slot float64 values held in registers cost the stepping
// loop spills.
struct SlotScene {
    double mass, spin, capture_radius, escape_radius;
};
__device__ __forceinline__ SlotScene slot_scene(const TraceArgs &a, int cam) {
    if (cam < 0) return SlotScene{a.mass, a.spin, a.capture_radius, a.escape_radius};
    const CameraDev &c = a.cameras[cam];
    return SlotScene{c.mass, c.spin, c.capture_radius, c.escape_radius};
}

// PROJECT: every project_every controller iterations, each ray in flight is
// projected onto the null constraint in float64 (project_null) and its FSAL
// derivative recomputed; warp-uniform, so the warp pays one RHS per period.
template <class V, int BLOCK, int MINB, bool PROJECT>
__global__ void __launch_bounds__(BLOCK, MINB) trace_kernel(const TraceArgs args) {
    using T = VT<V>;
    constexpr int N = T::N;
    constexpr bool F64 = sizeof(typename T::S) == 8;
    TraceWorkspace *ws = args.ws;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long long n = args.n;
    const unsigned long long t_start = global_timer_ns();
    const bool has_deadline = args.timeout_ns > 0;
    const unsigned long long deadline = t_start + (unsigned long long)args.timeout_ns;
    const V rt = T::set(args.rtol), at = T::set(args.atol);

    extern __shared__ double bh_state_smem[];
    StateStore<V, BLOCK> ys(bh_state_smem);
    // Values that change once per ray live in shared memory, one column per
    // thread: each slot's affine parameter and the thread's launch counters
    // (attempts, accepted steps, most attempts of a ray).
    __shared__ double lam_of[N][BLOCK];
    __shared__ unsigned long long cnt[3][BLOCK];
#pragma unroll
    for (int k = 0; k < 3; ++k) cnt[k][threadIdx.x] = 0;
    long long ray[N], steps[N], attempts[N];
    int cam[N];  // the slot's camera (slot_scene)
    // r: Kerr-Schild radius of the slot's state, NaN while it lies clear of
    // both termination radii (settled_radius).
    double h[N], r[N];
    WStateV<V> yw;
    double mass0[N], spin0[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        ray[l] = -1; steps[l] = 0; attempts[l] = 0; cam[l] = -1;
        h[l] = args.initial_step; r[l] = 0.0;
        lam_of[l][threadIdx.x] = 0.0;
        mass0[l] = 1.0; spin0[l] = 0.0;
        // A benign placeholder state for idle slots (finite, far from the hole).
        const RayState y0{0.0, 10.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0};
        ys.set(l, y0);
        put_work<V>(yw, l, y0);
    }
    KerrV<V> K = make_kerr<V>(lanes_of<V>(mass0), lanes_of<V>(spin0));
    StageV<V> k1 = first_stage<V>(K, yw);
    bool queue_open = true;
    int refill_waited = 0;  // iterations the warp's idle slots have waited

    for (unsigned iter = 0;; ++iter) {
        // ---- warp-aggregated refill of the idle ray slots
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
        // Idle slots wait for company (bh_trace_common.cuh): a refill costs
        // the warp one first-stage evaluation however many slots it fills.
        const bool do_refill =
            total && (total >= BH_TRACE_REFILL_BATCH || refill_waited >= BH_TRACE_REFILL_WAIT);
        refill_waited = total && !do_refill ? refill_waited + 1 : 0;
        if (do_refill) {
            unsigned any = 0;
#pragma unroll
            for (int l = 0; l < N; ++l) any |= mask[l];
            const int leader = __ffs(any) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&ws->queue_head, (unsigned long long)total);
            base = __shfl_sync(full, base, leader);
            int before = 0;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                if ((mask[l] >> lane) & 1u) {
                    const long long idx = (long long)base + before + __popc(mask[l] & lt_mask);
                    if (idx < n) {
                        ray[l] = idx;
                        RayState y0;
                        if (args.source == 0) {
                            load_state(args.state0, n, args.layout, idx, y0);
                            cam[l] = -1;
                        } else {
                            const int c = find_camera(args.cameras, args.ncameras, idx);
                            camera_ray(args.cameras[c], idx - args.cameras[c].first_ray, y0);
                            cam[l] = c;
                        }
                        const SlotScene sc = slot_scene(args, cam[l]);
                        h[l] = args.initial_step;
                        lam_of[l][threadIdx.x] = 0.0;
                        steps[l] = 0;
                        attempts[l] = 0;
                        r[l] = ks_radius(sc.spin, y0);
                        if (r[l] >= sc.escape_radius) {
                            // tracer.py:95-99 rejects the whole call; count and skip.
                            atomicAdd(&ws->bad_rays, 1);
                            store_state(args.states, n, args.layout, idx, y0);
                            args.status[idx] = BH_RAY_FAILED;
                            args.steps[idx] = 0;
                            if (args.lam_io) args.lam_io[idx] = 0.0;
                            ray[l] = -1;
                        } else {
                            fresh[l] = true;
                            ys.set(l, y0);
                            put_work<V>(yw, l, y0);
                        }
                    }
                }
                before += __popc(mask[l]);
            }
            if ((long long)base + total >= n) queue_open = false;
        }
        bool any_fresh = false;
#pragma unroll
        for (int l = 0; l < N; ++l) any_fresh |= fresh[l];
        if (any_fresh) {
            double mass[N], spin[N];
#pragma unroll
            for (int l = 0; l < N; ++l) {
                const SlotScene sc = slot_scene(args, cam[l]);
                mass[l] = sc.mass; spin[l] = sc.spin;
            }
            K = make_kerr<V>(lanes_of<V>(mass), lanes_of<V>(spin));
            const StageV<V> f = first_stage<V>(K, yw);
            take_stage(k1, f, fresh);
        }
        bool active = false;
#pragma unroll
        for (int l = 0; l < N; ++l) active |= ray[l] >= 0;
        // Idle slots that wait for a refill batch keep the warp in the loop
        // while the queue is open.
        if (!__any_sync(full, active || queue_open)) break;

        if (active) {
            // ---- one controller iteration for every slot (tracer.py:109-149)
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
                RayState yl = ys.get(l);
                if (acc[l] && args.h_tape) {
                    // Tape of the accepted step sequence for the adjoint.
                    const long long s = steps[l];
                    if (s < args.tape_cap) {
                        args.h_tape[ray[l] * args.tape_cap + s] = h[l];
                        if (s % args.ckpt_every == 0) {
                            const long long nck = (args.tape_cap + args.ckpt_every - 1) / args.ckpt_every;
                            double *c = args.ckpt + (ray[l] * nck + s / args.ckpt_every) * 8;
                            c[0] = yl.t; c[1] = yl.x; c[2] = yl.y; c[3] = yl.z;
                            c[4] = yl.pt; c[5] = yl.px; c[6] = yl.py; c[7] = yl.pz;
                        }
                    } else {
                        atomicExch(&ws->tape_overflow, 1);
                    }
                }
                const SlotScene sc = slot_scene(args, cam[l]);
                if (acc[l]) {
                    commit<V>(yl, yw, a, l, h[l]);
                    ys.set(l, yl);
                    lam_of[l][threadIdx.x] += h[l];
                    ++steps[l];
                    r[l] = settled_radius(double(T::get(a.r2n, l)), sc.capture_radius,
                                          sc.escape_radius, sc.spin, yl);
                }
                h[l] = next_step<F64>(h[l], ratio[l], args.max_step);

                const bool finite = all_finite(yl);
                int st = BH_RAY_IN_FLIGHT;
                if (!finite) st = BH_RAY_FAILED;
                if (finite && r[l] <= sc.capture_radius) st = BH_RAY_CAPTURED;
                if (finite && r[l] >= sc.escape_radius) st = BH_RAY_ESCAPED;
                const bool in_flight = st == BH_RAY_IN_FLIGHT;
                if (in_flight && h[l] < args.min_step) st = BH_RAY_FAILED;
                if (in_flight && steps[l] >= args.max_steps) st = BH_RAY_MAX_STEPS;
                // tracer.py:151-154: rays still in flight after the cap are MAX_STEPS.
                if (st == BH_RAY_IN_FLIGHT && attempts[l] >= args.max_attempts) st = BH_RAY_MAX_STEPS;
                if (st != BH_RAY_IN_FLIGHT) {
                    // Returned states lie on the constraint too (p only: r
                    // and so the classification are unchanged).
                    if constexpr (PROJECT) project_null(sc.mass, sc.spin, yl);
                    store_state(args.states, n, args.layout, ray[l], yl);
                    args.status[ray[l]] = st;
                    args.steps[ray[l]] = steps[l];
                    if (args.lam_io) args.lam_io[ray[l]] = lam_of[l][threadIdx.x];
                    cnt[0][threadIdx.x] += attempts[l];
                    cnt[1][threadIdx.x] += steps[l];
                    if ((unsigned long long)attempts[l] > cnt[2][threadIdx.x])
                        cnt[2][threadIdx.x] = attempts[l];
                    ray[l] = -1;
                }
            }
            take_stage(k1, a.k7, acc);
            if constexpr (PROJECT) {
                if (iter % (unsigned)args.project_every == 0u) {
                    bool proj[N];
#pragma unroll
                    for (int l = 0; l < N; ++l) {
                        proj[l] = ray[l] >= 0;
                        if (proj[l]) {
                            RayState yl = ys.get(l);
                            const SlotScene sc = slot_scene(args, cam[l]);
                            project_null(sc.mass, sc.spin, yl);
                            ys.set(l, yl);
                            put_work<V>(yw, l, yl);
                        }
                    }
                    const StageV<V> f = first_stage<V>(K, yw);
                    take_stage(k1, f, proj);
                }
            }
        }

        // ---- bounded launch time
        if (has_deadline && (iter & 7u) == 0u) {
            const bool late = global_timer_ns() > deadline;
            if (__any_sync(full, late)) {
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    if (ray[l] < 0) continue;
                    store_state(args.states, n, args.layout, ray[l], ys.get(l));
                    args.status[ray[l]] = BH_RAY_IN_FLIGHT;
                    args.steps[ray[l]] = steps[l];
                    if (args.lam_io) args.lam_io[ray[l]] = lam_of[l][threadIdx.x];
                    cnt[0][threadIdx.x] += attempts[l];
                    cnt[1][threadIdx.x] += steps[l];
                }
                if (lane == 0) atomicExch(&ws->timed_out, 1);
                break;
            }
        }
    }
    // ---- launch counters: one atomic per warp
    unsigned long long my_attempts = cnt[0][threadIdx.x], my_accepted = cnt[1][threadIdx.x];
    long long my_max_attempts = (long long)cnt[2][threadIdx.x];
    for (int off = 16; off > 0; off >>= 1) {
        my_attempts += __shfl_down_sync(full, my_attempts, off);
        my_accepted += __shfl_down_sync(full, my_accepted, off);
        const long long o = __shfl_down_sync(full, my_max_attempts, off);
        my_max_attempts = o > my_max_attempts ? o : my_max_attempts;
    }
    if (lane == 0) {
        atomicAdd(&ws->attempts, my_attempts);
        atomicAdd(&ws->accepted, my_accepted);
        atomicMax(&ws->iterations, my_max_attempts);
    }
}

// One float64 DP5(4) attempt with the float64 policy's controller, for one
// ray of a mixed thread: the float64 band of propagate_kernel.  p points at
// the ray's float64 state in the block's state store and kp at its float64
// first-same-as-last derivative (7 planes after the state's 8, P doubles
// between components).  With have_k1 the stored derivative belongs to the
// current state (the previous attempt was a band attempt too); otherwise it
// is evaluated here.  The state and the derivative are updated there when the
// attempt is accepted.  Out of line: one copy of the rare path's code, apart
// from the float loop's (inlined, the headline kernel ran 6 % slower).
struct BandStep {
    double h;       // the controller's next step size
    bool accepted;
};
template <int P>
__device__ __noinline__ BandStep band_attempt(double *p, double *kp, bool have_k1, double mass, double spin, double h,
                      double rtol, double atol, double max_step) {
    RayState y{p[0], p[P], p[2 * P], p[3 * P], p[4 * P], p[5 * P], p[6 * P], p[7 * P]};
    const KerrV<double> K = make_kerr<double>(mass, spin);
    WStateV<double> w;
    put_work<double>(w, 0, y);
    StageV<double> k1;
    if (have_k1) {
        k1 = StageV<double>{kp[0], kp[P], kp[2 * P], kp[3 * P], kp[4 * P], kp[5 * P], kp[6 * P]};
    } else {
        k1 = first_stage<double>(K, w);
        kp[0] = k1.kx; kp[P] = k1.ky; kp[2 * P] = k1.kz; kp[3 * P] = k1.thl;
        kp[4 * P] = k1.px; kp[5 * P] = k1.py; kp[6 * P] = k1.pz;
    }
    AttemptV<double> a;
    dp5_attempt<double>(K, w, h, k1, a);
    double ratio[1];
    const double hl[1] = {h};
    error_ratio_v<double>(w, a, h, rtol, atol, ratio, hl);
    const bool ok = ratio[0] <= 1.0;
    if (ok) {
        commit<double>(y, w, a, 0, h);
        p[0] = y.t; p[P] = y.x; p[2 * P] = y.y; p[3 * P] = y.z;
        p[5 * P] = y.px; p[6 * P] = y.py; p[7 * P] = y.pz;
        const StageV<double> &k7 = a.k7;
        kp[0] = k7.kx; kp[P] = k7.ky; kp[2 * P] = k7.kz; kp[3 * P] = k7.thl;
        kp[4 * P] = k7.px; kp[5 * P] = k7.py; kp[6 * P] = k7.pz;
    }
    return BandStep{next_step<true>(h, ratio[0], max_step), ok};
}

// n_steps attempted DP5(4) steps per ray with the tracer's accept/reject and
// step update (tracer.py:111-120) and no termination.  Each warp claims 32
// groups of N rays at a time from the workspace's queue head, so warps that
// the scheduler runs ahead take more groups and all of them stay resident
// until the queue drains (a fixed grid-stride split left a quarter of the
// warp slots idle while the slowest warps finished).
//
// BAND (mixed lanes only): while one of the warp's rays lies between 1.01
// times the outer horizon radius and the band radius (args.f64_r2), the
// whole warp's attempt runs in float64 (band_attempt, the float64 policy's
// step); outside it the float stages run.  The test reads r^2 at each ray's current
// state from its last derivative evaluation, and is warp-uniform, so the two
// paths never diverge within a warp; the rays that share a warp are the 64
// (two per lane) of one claim, [64 k, 64 k + 64) of the launch.  Closer to
// the horizon the float stages run: the reference's tracer captures such
// rays.
template <class V, int BLOCK, int MINB, bool PROJECT, bool BAND = false>
__global__ void __launch_bounds__(BLOCK, MINB) propagate_kernel(const TraceArgs args) {
    using T = VT<V>;
    constexpr int N = T::N;
    constexpr bool F64 = sizeof(typename T::S) == 8;
    static_assert(!(BAND && F64), "the float64 band is a mixed-policy option");
    TraceWorkspace *ws = args.ws;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long n = args.n;
    const unsigned long long deadline =
        global_timer_ns() + (unsigned long long)args.timeout_ns;
    const bool has_deadline = args.timeout_ns > 0;
    const V rt = T::set(args.rtol), at = T::set(args.atol);
    unsigned long long my_attempts = 0, my_accepted = 0;
    long long my_max = 0;
    bool late = false;
    const long long groups = (n + N - 1) / N;
    extern __shared__ double bh_state_smem[];
    StateStore<V, BLOCK> ys(bh_state_smem);
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&ws->queue_head, 32ull);
        base = __shfl_sync(full, base, 0);
        if ((long long)base >= groups) break;
        const long long g = (long long)base + lane;
        // The lanes that hold a group run the same attempts in lock step;
        // the band test and the deadline are agreed among them.
        const unsigned act = __ballot_sync(full, g < groups);
        if (g < groups) {
            double h[N], lam[N], spin[N], mass[N];
            long long acc[N], src[N];
            bool valid[N];
#pragma unroll
            for (int l = 0; l < N; ++l) {
                const long long i = g * N + l;
                valid[l] = i < n;
                // A missing last ray repeats the group's first ray; its results
                // are not stored.
                src[l] = valid[l] ? i : g * N;
                if (args.order) {
                    const long long o = args.order[src[l]];
                    if (o < 0 || o >= n) {
                        // Not a permutation: counted (the stats read fails the
                        // call), and the position's own ray is traced instead.
                        if (valid[l]) atomicAdd(&ws->bad_order, 1);
                        valid[l] = false;
                    } else {
                        src[l] = o;
                    }
                }
                RayState y0;
                load_state(args.state0, n, args.layout, src[l], y0);
                ys.set(l, y0);
                spin[l] = args.spin_of_ray ? args.spin_of_ray[src[l]] : args.spin;
                mass[l] = args.mass;
                if (!(::fabs(spin[l]) <= mass[l])) {
                    // A ray's own spin outside the Kerr bound: counted (the
                    // stats read then fails the call) and traced at spin 0.
                    if (valid[l]) atomicAdd(&ws->bad_spins, 1);
                    spin[l] = 0.0;
                }
                h[l] = args.h_io[src[l]];
                lam[l] = args.lam_io ? args.lam_io[src[l]] : 0.0;
                acc[l] = 0;
            }
            const KerrV<V> K = make_kerr<V>(lanes_of<V>(mass), lanes_of<V>(spin));
            WStateV<V> yw;
#pragma unroll
            for (int l = 0; l < N; ++l) put_work<V>(yw, l, ys.get(l));
            // r2c: r^2 of each lane's current state from its last derivative
            // evaluation (BAND only).
            V r2c = T::set(0.0);
            StageV<V> k1 = first_stage_r2<V>(K, yw, BAND ? &r2c : nullptr);
            // Squared lower edge of the band per lane (BAND): 1.01 r_+.  A
            // past-directed ray that reaches the outer horizon approaches r_+
            // only asymptotically in these coordinates (the ingoing chart does
            // not cover the past horizon), so it sits just above r_+ for the
            // rest of a no-termination run; the tracers capture it at
            // r_+ (1 + margin), and below 1.01 r_+ the float stages run.
            float rp2[N];
#pragma unroll
            for (int l = 0; l < N; ++l) {
                const double rp =
                    1.01 * (mass[l] + ::sqrt(fmax(mass[l] * mass[l] - spin[l] * spin[l], 0.0)));
                rp2[l] = float(rp * rp);
            }
            const float band2 = float(args.f64_r2);
            // Whether a lane's float64 derivative in shared memory belongs to
            // its current state (BAND).
            bool band_k1[N];
#pragma unroll
            for (int l = 0; l < N; ++l) band_k1[l] = false;
            long long k = 0;
            for (; k < args.max_attempts; ++k) {
                bool in_band = false;
                if constexpr (BAND) {
                    bool mine = false;
#pragma unroll
                    for (int l = 0; l < N; ++l) {
                        const float r2l = T::get(r2c, l);
                        mine |= r2l > rp2[l] && r2l < band2;
                    }
                    in_band = __any_sync(act, mine);
                }
                if (in_band) {
#pragma unroll
                    for (int l = 0; l < N; ++l) {
                        double *slot = ys.sh + l * BLOCK + threadIdx.x;
                        const BandStep b = band_attempt<N * BLOCK>(
                            slot, slot + 8 * N * BLOCK, band_k1[l], mass[l], spin[l], h[l],
                            args.rtol, args.atol, args.max_step);
                        band_k1[l] = true;
                        if (b.accepted) {
                            lam[l] += h[l];
                            ++acc[l];
                        }
                        h[l] = b.h;
                    }
#pragma unroll
                    for (int l = 0; l < N; ++l) put_work<V>(yw, l, ys.get(l));
                    k1 = first_stage_r2<V>(K, yw, &r2c);
                } else {
                    V hw = T::set(0.0);
#pragma unroll
                    for (int l = 0; l < N; ++l) T::put(hw, l, typename T::S(h[l]));
                    AttemptV<V> a;
                    dp5_attempt<V>(K, yw, hw, k1, a);
                    RatioT<V> ratio[N];
                    error_ratio_v<V>(yw, a, hw, rt, at, ratio, h);
                    bool ok[N];
#pragma unroll
                    for (int l = 0; l < N; ++l) {
                        ok[l] = ratio[l] <= RatioT<V>(1);
                        if (ok[l]) {
                            RayState yl = ys.get(l);
                            commit<V>(yl, yw, a, l, h[l]);
                            ys.set(l, yl);
                            lam[l] += h[l];
                            ++acc[l];
                            band_k1[l] = false;
                        }
                        h[l] = next_step<F64>(h[l], ratio[l], args.max_step);
                    }
                    take_stage(k1, a.k7, ok);
                    if constexpr (BAND) take_lanes(r2c, a.r2n, ok);
                }
                if constexpr (PROJECT) {
                    if ((k + 1) % args.project_every == 0) {
                        bool proj[N];
#pragma unroll
                        for (int l = 0; l < N; ++l) {
                            proj[l] = true;
                            RayState yl = ys.get(l);
                            project_null(mass[l], spin[l], yl);
                            ys.set(l, yl);
                            put_work<V>(yw, l, yl);
                        }
                        const StageV<V> f = first_stage<V>(K, yw);
                        take_stage(k1, f, proj);
                    }
                }
                if constexpr (BAND) {
                    // Agreed among the lanes, which keep their attempts in
                    // lock step for the band test.
                    if (has_deadline && (k & 63) == 63 &&
                        __any_sync(act, global_timer_ns() > deadline)) {
                        late = true;
                        ++k;
                        break;
                    }
                } else if (has_deadline && (k & 63) == 63 && global_timer_ns() > deadline) {
                    late = true;
                    ++k;
                    break;
                }
            }
#pragma unroll
            for (int l = 0; l < N; ++l) {
                if (!valid[l]) continue;
                const long long i = src[l];
                RayState yl = ys.get(l);
                if constexpr (PROJECT) project_null(mass[l], spin[l], yl);
                store_state(args.states, n, args.layout, i, yl);
                args.h_io[i] = h[l];
                if (args.lam_io) args.lam_io[i] = lam[l];
                args.steps[i] = acc[l];
                my_attempts += (unsigned long long)k;
                my_accepted += (unsigned long long)acc[l];
            }
            if (k > my_max) my_max = k;
        }
        if (__any_sync(full, late)) break;
    }
    if (late) atomicExch(&ws->timed_out, 1);
    for (int off = 16; off > 0; off >>= 1) {
        my_attempts += __shfl_down_sync(full, my_attempts, off);
        my_accepted += __shfl_down_sync(full, my_accepted, off);
        const long long o = __shfl_down_sync(full, my_max, off);
        my_max = o > my_max ? o : my_max;
    }
    if (lane == 0) {
        atomicAdd(&ws->attempts, my_attempts);
        atomicAdd(&ws->accepted, my_accepted);
        atomicMax(&ws->iterations, my_max);
    }
}

// ---------------------------------------------------------------- variants
// (threads per block, __launch_bounds__ min blocks per SM, rays per thread).
// The register cap is 65536 / (block * min_blocks), rounded down to the
// allocation granule.  Mixed variants 4..7 run two rays per thread in packed
// float32x2 arithmetic.
static const Variant kVariantsF64[] = {{128, 2, 1}, {128, 3, 1}, {128, 4, 1}, {256, 2, 1}};
static const Variant kVariantsMixed[] = {{128, 3, 1}, {128, 4, 1}, {128, 5, 1}, {256, 2, 1},
                                         {128, 2, 2}, {128, 3, 2}, {64, 4, 2}, {256, 1, 2}};

int trace_variant_count(int precision) {
    return precision == BH_PRECISION_MIXED ? 8 : 4;
}
Variant trace_variant(int precision, int idx) {
    return precision == BH_PRECISION_MIXED ? kVariantsMixed[idx] : kVariantsF64[idx];
}
// Defaults measured on the raw-throughput and full-HD workloads: float64
// 256 x 2 for both kernels; mixed: two rays per thread (packed float32x2,
// 128 x 3) for the propagator, one ray per thread (128 x 5) for the tracer,
// whose per-ray termination and refill work does not pack.
int trace_default_variant(int precision) {
    return precision == BH_PRECISION_MIXED ? 2 : 3;
}
int propagate_default_variant(int precision) {
    return precision == BH_PRECISION_MIXED ? 5 : 3;
}

template <class V, int B, int M, bool P = false>
static const void *kfn(bool propagate, size_t *smem) {
    *smem = StateStore<V, B>::shared_bytes();
    return propagate ? (const void *)propagate_kernel<V, B, M, P>
                     : (const void *)trace_kernel<V, B, M, P>;
}

// project: the null-constraint projection is compiled for the default launch
// shapes only (the launcher switches to them); so is the float64 band of the
// mixed propagator (band).
static const void *kernel_for(bool propagate, int precision, int idx, bool project,
                              size_t *smem, bool band = false) {
    if (band && propagate && precision == BH_PRECISION_MIXED) {
        // The state store plus 7 planes of float64 band derivatives.
        *smem = StateStore<F2, 128>::shared_bytes() + size_t(7) * 2 * 128 * 8;
        return (const void *)propagate_kernel<F2, 128, 3, false, true>;
    }
    if (project) {
        if (precision != BH_PRECISION_MIXED) return kfn<double, 256, 2, true>(propagate, smem);
        return propagate ? kfn<F2, 128, 3, true>(propagate, smem)
                         : kfn<float, 128, 5, true>(propagate, smem);
    }
    if (precision == BH_PRECISION_MIXED) {
        switch (idx) {
            case 0: return kfn<float, 128, 3>(propagate, smem);
            case 1: return kfn<float, 128, 4>(propagate, smem);
            case 2: return kfn<float, 128, 5>(propagate, smem);
            case 3: return kfn<float, 256, 2>(propagate, smem);
            case 4: return kfn<F2, 128, 2>(propagate, smem);
            case 5: return kfn<F2, 128, 3>(propagate, smem);
            case 6: return kfn<F2, 64, 4>(propagate, smem);
            default: return kfn<F2, 256, 1>(propagate, smem);
        }
    }
    switch (idx) {
        case 0: return kfn<double, 128, 2>(propagate, smem);
        case 1: return kfn<double, 128, 3>(propagate, smem);
        case 2: return kfn<double, 128, 4>(propagate, smem);
        default: return kfn<double, 256, 2>(propagate, smem);
    }
}

int kernel_attributes(bool propagate, int precision, int idx, int *regs,
                      int *max_blocks) {
    size_t smem = 0;
    const void *fn = kernel_for(propagate, precision, idx, false, &smem);
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, fn);
    if (e != cudaSuccess) return -1;
    if (regs) *regs = attr.numRegs;
    if (max_blocks) {
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &nb, fn, trace_variant(precision, idx).block, smem);
        if (e != cudaSuccess) return -1;
        *max_blocks = nb;
    }
    return 0;
}

static cudaError_t launch(bool propagate, const TraceArgs &args, int precision,
                          int variant, int blocks_per_sm, cudaStream_t stream) {
    const bool project = args.project_every > 0;
    const bool band = propagate && precision == BH_PRECISION_MIXED && args.f64_r2 > 0.0;
    if (project || band || variant < 0 || variant >= trace_variant_count(precision))
        variant = propagate ? propagate_default_variant(precision)
                            : trace_default_variant(precision);
    const Variant v = trace_variant(precision, variant);
    size_t smem = 0;
    const void *fn = kernel_for(propagate, precision, variant, project, &smem, band);
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, v.block, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    const int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    long long blocks = (long long)sms * per_sm;
    if (propagate) {
        // Grid-stride: never more blocks than the ray groups need.
        const long long groups = (args.n + v.rays_per_thread - 1) / v.rays_per_thread;
        const long long need = (groups + v.block - 1) / v.block;
        if (blocks > need) blocks = need;
    }
    if (blocks < 1) blocks = 1;
    TraceArgs a = args;
    void *params[] = {(void *)&a};
    return cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(v.block), params, smem, stream);
}

cudaError_t launch_trace(const TraceArgs &args, int precision, int variant,
                         int blocks_per_sm, cudaStream_t stream) {
    return launch(false, args, precision, variant, blocks_per_sm, stream);
}

cudaError_t launch_propagate(const TraceArgs &args, int precision, int variant,
                             int blocks_per_sm, cudaStream_t stream) {
    return launch(true, args, precision, variant, blocks_per_sm, stream);
}

}  // namespace bh
