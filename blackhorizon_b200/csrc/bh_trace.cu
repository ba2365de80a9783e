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
// Scheduling: one ray per thread, state in registers.  The grid is
// persistent (blocks_per_sm x SMs); a lane whose ray terminates takes the next
// ray from a global work queue.  Refills are warp-aggregated: __ballot_sync
// collects the idle lanes, one lane claims that many rays with a single
// atomicAdd and __shfl_sync hands each idle lane its index.  Every wait is
// bounded: each ray makes at most max_attempts attempts and a %globaltimer
// deadline ends the launch with a status flag.
#include <cstdio>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void load_state(const double *base, long long n,
                                           int layout, long long i,
                                           RayState &y) {
    if (layout == BH_LAYOUT_AOS) {
        const double2 *p = reinterpret_cast<const double2 *>(base + 8 * i);
        const double2 a = p[0], b = p[1], c = p[2], d = p[3];
        y.t = a.x; y.x = a.y; y.y = b.x; y.z = b.y;
        y.pt = c.x; y.px = c.y; y.py = d.x; y.pz = d.y;
    } else {
        y.t = base[i]; y.x = base[n + i]; y.y = base[2 * n + i];
        y.z = base[3 * n + i]; y.pt = base[4 * n + i]; y.px = base[5 * n + i];
        y.py = base[6 * n + i]; y.pz = base[7 * n + i];
    }
}

__device__ __forceinline__ void store_state(double *base, long long n,
                                            int layout, long long i,
                                            const RayState &y) {
    if (layout == BH_LAYOUT_AOS) {
        double2 *p = reinterpret_cast<double2 *>(base + 8 * i);
        p[0] = make_double2(y.t, y.x);
        p[1] = make_double2(y.y, y.z);
        p[2] = make_double2(y.pt, y.px);
        p[3] = make_double2(y.py, y.pz);
    } else {
        base[i] = y.t; base[n + i] = y.x; base[2 * n + i] = y.y;
        base[3 * n + i] = y.z; base[4 * n + i] = y.pt; base[5 * n + i] = y.px;
        base[6 * n + i] = y.py; base[7 * n + i] = y.pz;
    }
}

// Camera that owns global ray index i (cameras sorted by first_ray).
__device__ __forceinline__ int find_camera(const CameraDev *cams, int ncams,
                                           long long i) {
    int lo = 0, hi = ncams - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cams[mid].first_ray <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Initial state of ray i of a camera: pinhole direction (camera.py:102-113),
// past-directed null momentum normalised to |p_t| = 1 (geodesics.py:109-170),
// t0 = 0 (geodesics.py:25-39).
__device__ __forceinline__ void camera_ray(const CameraDev &c, long long local,
                                           RayState &y) {
    double d[3], p[4];
    pinhole_direction(c.fwd, c.right, c.up, c.half_w, c.half_h, c.width,
                      c.height, local, d);
    null_momentum(c.mass, c.spin, c.pos, d, true, true, p);
    y.t = 0.0; y.x = c.pos[0]; y.y = c.pos[1]; y.z = c.pos[2];
    y.pt = p[0]; y.px = p[1]; y.py = p[2]; y.pz = p[3];
}

__device__ __forceinline__ double ks_radius(double a, const RayState &y) {
    return ::sqrt(ks_radius2(a, y.x, y.y, y.z));
}

template <typename W, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) trace_kernel(const TraceArgs args) {
    TraceWorkspace *ws = args.ws;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long n = args.n;
    const unsigned long long t_start = global_timer_ns();
    const bool has_deadline = args.timeout_ns > 0;
    const unsigned long long deadline = t_start + (unsigned long long)args.timeout_ns;

    long long ray = -1;
    RayState y;
    Stage<W> k1;
    double h = 0.0, spin = 0.0, mass = 0.0, rcap = 0.0, resc = 0.0, r = 0.0;
    long long steps = 0, attempts = 0;
    bool queue_open = true;
    unsigned long long my_attempts = 0, my_accepted = 0;
    long long my_max_attempts = 0;

    for (unsigned iter = 0;; ++iter) {
        // ---- warp-aggregated refill from the work queue
        const bool need = ray < 0 && queue_open;
        const unsigned mask = __ballot_sync(full, need);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            const int cnt = __popc(mask);
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&ws->queue_head, (unsigned long long)cnt);
            base = __shfl_sync(full, base, leader);
            if (need) {
                const long long idx = (long long)base + __popc(mask & ((1u << lane) - 1u));
                if (idx < n) {
                    ray = idx;
                    if (args.source == 0) {
                        load_state(args.state0, n, args.layout, idx, y);
                        mass = args.mass; spin = args.spin;
                        rcap = args.capture_radius; resc = args.escape_radius;
                    } else {
                        const int c = find_camera(args.cameras, args.ncameras, idx);
                        const CameraDev &cam = args.cameras[c];
                        camera_ray(cam, idx - cam.first_ray, y);
                        mass = cam.mass; spin = cam.spin;
                        rcap = cam.capture_radius; resc = cam.escape_radius;
                    }
                    h = args.initial_step;
                    steps = 0;
                    attempts = 0;
                    r = ks_radius(spin, y);
                    if (r >= resc) {
                        // tracer.py:95-99 rejects the whole call; count and skip.
                        atomicAdd(&ws->bad_rays, 1);
                        store_state(args.states, n, args.layout, idx, y);
                        args.status[idx] = BH_RAY_FAILED;
                        args.steps[idx] = 0;
                        ray = -1;
                    } else {
                        k1 = first_stage<W>(W(mass), W(spin), y);
                    }
                }
            }
            if ((long long)base + cnt >= n) queue_open = false;
        }
        const bool active = ray >= 0;
        if (!__any_sync(full, active)) break;

        if (active) {
            // ---- one controller iteration (tracer.py:109-149)
            Attempt<W> at;
            dp5_attempt<W>(W(mass), W(spin), y, h, k1, at);
            const double ratio = error_ratio<W>(y, at.y_new, at.err, args.rtol, args.atol);
            const bool accept = ratio <= 1.0;
            ++attempts;
            if (accept) {
                y = at.y_new;
                k1 = at.k7;
                ++steps;
                r = ks_radius(spin, y);
            }
            h = np_min(np_max(h * step_factor<W>(ratio), 0.0), args.max_step);

            const bool finite = all_finite(y);
            int st = BH_RAY_IN_FLIGHT;
            if (!finite) st = BH_RAY_FAILED;
            if (finite && r <= rcap) st = BH_RAY_CAPTURED;
            if (finite && r >= resc) st = BH_RAY_ESCAPED;
            const bool in_flight = st == BH_RAY_IN_FLIGHT;
            if (in_flight && h < args.min_step) st = BH_RAY_FAILED;
            if (in_flight && steps >= args.max_steps) st = BH_RAY_MAX_STEPS;
            // tracer.py:151-154: rays still in flight after the cap are MAX_STEPS.
            if (st == BH_RAY_IN_FLIGHT && attempts >= args.max_attempts) st = BH_RAY_MAX_STEPS;
            if (st != BH_RAY_IN_FLIGHT) {
                store_state(args.states, n, args.layout, ray, y);
                args.status[ray] = st;
                args.steps[ray] = steps;
                my_attempts += attempts;
                my_accepted += steps;
                if (attempts > my_max_attempts) my_max_attempts = attempts;
                ray = -1;
            }
        }

        // ---- bounded launch time
        if (has_deadline && (iter & 7u) == 0u) {
            const bool late = global_timer_ns() > deadline;
            if (__any_sync(full, late)) {
                if (ray >= 0) {
                    store_state(args.states, n, args.layout, ray, y);
                    args.status[ray] = BH_RAY_IN_FLIGHT;
                    args.steps[ray] = steps;
                    my_attempts += attempts;
                    my_accepted += steps;
                }
                if (lane == 0) atomicExch(&ws->timed_out, 1);
                break;
            }
        }
    }
    // ---- launch counters: one atomic per warp
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

// n_steps attempted DP5(4) steps per ray with the tracer's accept/reject and
// step update (tracer.py:111-120) and no termination; grid-stride over rays.
template <typename W, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) propagate_kernel(const TraceArgs args) {
    TraceWorkspace *ws = args.ws;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long n = args.n;
    const unsigned long long deadline =
        global_timer_ns() + (unsigned long long)args.timeout_ns;
    const bool has_deadline = args.timeout_ns > 0;
    unsigned long long my_attempts = 0, my_accepted = 0;
    long long my_max = 0;
    bool late = false;
    const long long stride = (long long)gridDim.x * blockDim.x;
    // The loop trip count is uniform per warp: every lane of a warp runs
    // ceil-aligned ray slots so the shuffles below see a full warp.
    const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rounds = (n + stride - 1) / stride;
    for (long long rd = 0; rd < rounds && !late; ++rd) {
        const long long i = first + rd * stride;
        const bool valid = i < n;
        if (!valid) continue;
        RayState y;
        load_state(args.state0, n, args.layout, i, y);
        const double spin = args.spin_of_ray ? args.spin_of_ray[i] : args.spin;
        const W m = W(args.mass), a = W(spin);
        double h = args.h_io[i];
        Stage<W> k1 = first_stage<W>(m, a, y);
        long long acc = 0, k = 0;
        for (; k < args.max_attempts; ++k) {
            Attempt<W> at;
            dp5_attempt<W>(m, a, y, h, k1, at);
            const double ratio = error_ratio<W>(y, at.y_new, at.err, args.rtol, args.atol);
            if (ratio <= 1.0) {
                y = at.y_new;
                k1 = at.k7;
                ++acc;
            }
            h = np_min(np_max(h * step_factor<W>(ratio), 0.0), args.max_step);
            if (has_deadline && (k & 63) == 63 && global_timer_ns() > deadline) {
                late = true;
                ++k;
                break;
            }
        }
        store_state(args.states, n, args.layout, i, y);
        args.h_io[i] = h;
        args.steps[i] = acc;
        my_attempts += (unsigned long long)k;
        my_accepted += (unsigned long long)acc;
        if (k > my_max) my_max = k;
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
// (threads per block, __launch_bounds__ min blocks per SM).  The register cap
// is 65536 / (block * min_blocks), rounded down to the allocation granule.
static const Variant kVariantsF64[] = {{128, 2}, {128, 3}, {128, 4}, {256, 2}};
static const Variant kVariantsMixed[] = {{128, 3}, {128, 4}, {128, 5}, {256, 2}};
static constexpr int kNumVariants = 4;

int trace_variant_count(int) { return kNumVariants; }
Variant trace_variant(int precision, int idx) {
    return precision == BH_PRECISION_MIXED ? kVariantsMixed[idx] : kVariantsF64[idx];
}
int trace_default_variant(int precision) {
    return precision == BH_PRECISION_MIXED ? 1 : 1;
}

template <typename W, int B, int M>
static const void *trace_fn() { return (const void *)trace_kernel<W, B, M>; }
template <typename W, int B, int M>
static const void *prop_fn() { return (const void *)propagate_kernel<W, B, M>; }

static const void *kernel_for(bool propagate, int precision, int idx) {
    if (precision == BH_PRECISION_MIXED) {
        switch (idx) {
            case 0: return propagate ? prop_fn<float, 128, 3>() : trace_fn<float, 128, 3>();
            case 1: return propagate ? prop_fn<float, 128, 4>() : trace_fn<float, 128, 4>();
            case 2: return propagate ? prop_fn<float, 128, 5>() : trace_fn<float, 128, 5>();
            default: return propagate ? prop_fn<float, 256, 2>() : trace_fn<float, 256, 2>();
        }
    }
    switch (idx) {
        case 0: return propagate ? prop_fn<double, 128, 2>() : trace_fn<double, 128, 2>();
        case 1: return propagate ? prop_fn<double, 128, 3>() : trace_fn<double, 128, 3>();
        case 2: return propagate ? prop_fn<double, 128, 4>() : trace_fn<double, 128, 4>();
        default: return propagate ? prop_fn<double, 256, 2>() : trace_fn<double, 256, 2>();
    }
}

int kernel_attributes(bool propagate, int precision, int idx, int *regs,
                      int *max_blocks) {
    const void *fn = kernel_for(propagate, precision, idx);
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, fn);
    if (e != cudaSuccess) return -1;
    if (regs) *regs = attr.numRegs;
    if (max_blocks) {
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &nb, fn, trace_variant(precision, idx).block, 0);
        if (e != cudaSuccess) return -1;
        *max_blocks = nb;
    }
    return 0;
}

static cudaError_t launch(bool propagate, const TraceArgs &args, int precision,
                          int variant, int blocks_per_sm, cudaStream_t stream) {
    if (variant < 0 || variant >= kNumVariants) variant = trace_default_variant(precision);
    const Variant v = trace_variant(precision, variant);
    const void *fn = kernel_for(propagate, precision, variant);
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, v.block, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    int per_sm = blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ;
    long long blocks = (long long)sms * per_sm;
    if (propagate) {
        // Grid-stride: never more blocks than rays need.
        const long long need = (args.n + v.block - 1) / v.block;
        if (blocks > need) blocks = need;
    }
    if (blocks < 1) blocks = 1;
    TraceArgs a = args;
    void *params[] = {(void *)&a};
    return cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(v.block), params, 0, stream);
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
