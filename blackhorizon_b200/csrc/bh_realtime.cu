// bh_realtime.cu -- the real-time renderer's fixed-step ray tracer.
//
// Restates trace_like_shader (blackhorizon/realtime/reference.py:41-188), the
// CPU mirror of the real-time fragment shader, as a persistent CUDA kernel
// that writes into device buffers.  Per iteration and ray:
//   1. termination on the current state: captured at r <= r_plus (1 +
//      margin), or when |p|^2 >= bailout^2 (past-directed rays inside the
//      shadow blueshift without bound); escaped at r >= escape_radius.
//      Interior cameras stop at interior_stop (TERMINATED), also when r <=
//      1.002 interior_stop with |p|^2 > 2500, and cap the budget at 1024;
//   2. step h = clip(step_scale * L, min_step, max_step), L = r - r_plus
//      outside (min(max(|r - r_plus|, 0.15 r), 0.5 r) for interior
//      cameras), then h <= 1 / max(1, |p|);
//   3. one classical RK4 step;
//   4. with a disk: a step whose z changes sign is interpolated linearly
//      to z = 0, and a Kerr-Schild radius there in [r_in, r_out] ends the
//      ray (DISK) with that crossing state recorded.
// Rays alive after the budget stay MAX_STEPS.  Each ray is bounded by the
// budget (<= 4096 steps), so the launch needs no deadline.
//
// Scheduling as in the tracer: a persistent grid, idle ray slots refilled
// from a work queue with one warp-aggregated atomicAdd.
#include <cmath>

#include "bh_trace_common.cuh"

namespace bh {

struct RealtimeArgs {
    const double *state0;
    long long n;
    double mass, spin, r_plus, capture_radius, escape_radius;
    double step_scale, min_step, max_step, bail2;
    double disk_inner, disk_outer;  // disk_outer <= 0: no disk
    int interior;
    int capture_status;
    long long max_steps;
    double *states;
    int32_t *status;
    double *hit_radius, *hit_pos, *hit_mom;
    TraceWorkspace *ws;
};

// Kerr-Schild radius as the reference computes it (kerr.py:135-141, with the
// _TINY clamps), float64: the interior stop lies inside |rho| < a, where the
// termination test must see the same value.
__device__ __forceinline__ double rt_radius(double a, double x, double y, double z) {
    const double a2 = a * a;
    const double q = x * x + y * y + z * z - a2;
    const double s = np_max(::sqrt(q * q + 4.0 * a2 * z * z), kTiny);
    return ::sqrt(np_max(0.5 * (q + s), kTiny));
}

// N = VT<V>::N ray slots per thread (two in the packed float32x2 lane
// type); float64 states in registers for float64 lanes and in shared memory
// for float lanes (StateStore), as in the tracer.
template <class V, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) realtime_kernel(const RealtimeArgs args) {
    using T = VT<V>;
    constexpr int N = T::N;
    TraceWorkspace *ws = args.ws;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long long n = args.n;
    const KerrV<V> K = make_kerr<V>(T::set(args.mass), T::set(args.spin));
    const bool disk = args.disk_outer > 0.0;
    // Float lanes: squared termination thresholds moved inward by 1e-3 for
    // the float32 fast path below.  An interior camera's lowest radius
    // threshold is 1.002 stop radii; above it its |p|^2 > 2500 test cannot
    // end the ray, so only the bail-out bound remains for |p|^2.
    constexpr bool kFloatLanes = sizeof(typename T::S) == 4;
    const double rt_lo = args.interior ? args.capture_radius * 1.002 : args.capture_radius;
    const float rt_lo2 = float(rt_lo * rt_lo * (1.0 + 1e-3));
    const float rt_hi2 = float(args.escape_radius * args.escape_radius * (1.0 - 1e-3));
    const float rt_bail2 = float(args.bail2 * (1.0 - 1e-3));
    extern __shared__ double bh_state_smem[];
    StateStore<V, BLOCK> ys(bh_state_smem);
    WStateV<V> yw;
    long long ray[N], it[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        ray[l] = -1; it[l] = 0;
        const RayState y0{0.0, 10.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0};
        ys.set(l, y0);
        put_work<V>(yw, l, y0);
    }
    bool queue_open = true;
    unsigned long long my_steps = 0;
    long long my_max = 0;

    auto finish = [&](int l, const RayState &y, int st, const RayState *hit, double r_hit) {
        double *o = args.states + 8 * ray[l];
        o[0] = y.t; o[1] = y.x; o[2] = y.y; o[3] = y.z;
        o[4] = y.pt; o[5] = y.px; o[6] = y.py; o[7] = y.pz;
        args.status[ray[l]] = st;
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        double *hp = args.hit_pos + 3 * ray[l], *hm = args.hit_mom + 4 * ray[l];
        if (hit) {
            args.hit_radius[ray[l]] = r_hit;
            hp[0] = hit->x; hp[1] = hit->y; hp[2] = hit->z;
            hm[0] = hit->pt; hm[1] = hit->px; hm[2] = hit->py; hm[3] = hit->pz;
        } else {
            args.hit_radius[ray[l]] = nan;
            hp[0] = hp[1] = hp[2] = nan;
            hm[0] = hm[1] = hm[2] = hm[3] = nan;
        }
        my_steps += (unsigned long long)it[l];
        if (it[l] > my_max) my_max = it[l];
        ray[l] = -1;
    };

    for (;;) {
        // ---- warp-aggregated refill of the idle slots
        unsigned mask[N];
        int total = 0;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            mask[l] = __ballot_sync(full, ray[l] < 0 && queue_open);
            total += __popc(mask[l]);
        }
        if (total) {
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
                        RayState y0;
                        load_state(args.state0, n, BH_LAYOUT_AOS, idx, y0);
                        ys.set(l, y0);
                        put_work<V>(yw, l, y0);
                        ray[l] = idx;
                        it[l] = 0;
                    }
                }
                before += __popc(mask[l]);
            }
            if ((long long)base + total >= n) queue_open = false;
        }
        bool alive = false;
#pragma unroll
        for (int l = 0; l < N; ++l) alive |= ray[l] >= 0;
        if (!__any_sync(full, alive || queue_open)) break;

        // ---- termination on the current states (reference.py:107-133)
        double h[N];
        bool step[N];
        bool any_step = false;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            h[l] = 0.0;
            step[l] = false;
            if (ray[l] < 0) continue;
            if constexpr (kFloatLanes) {
                // The radius and |p|^2 of the float32 copy of the state lie
                // within 1e-6 (r^2 + 2 a^2) and 1e-6 |p|^2 of the float64
                // values (the bounds of settled_radius); clear of every
                // threshold by 1e-3 r^2 + 1e-4 a^2 (1e-3 |p|^2), the float64
                // tests would all fail, and the step size follows from the
                // float32 values (the policy's stages are float32 anyway).
                const float a2f = T::get(K.a2, l);
                const float xf = T::get(yw.x, l), yf = T::get(yw.y, l), zf = T::get(yw.z, l);
                const float pxf = T::get(yw.px, l), pyf = T::get(yw.py, l),
                            pzf = T::get(yw.pz, l);
                const float q = fmaf(xf, xf, fmaf(yf, yf, fmaf(zf, zf, -a2f)));
                const float s2 = fmaf(q, q, 4.0f * a2f * zf * zf);
                const float r2 = 0.5f * (q + s2 * rsqrt_approx(s2));
                const float mom2 = fmaf(pxf, pxf, fmaf(pyf, pyf, pzf * pzf));
                const float slack = 1e-4f * a2f;
                if (it[l] < args.max_steps && r2 - slack > rt_lo2 && r2 + slack < rt_hi2 &&
                    mom2 < rt_bail2) {
                    const float r = r2 * rsqrt_approx(r2);
                    const float rp = float(args.r_plus);
                    const float scale = args.interior
                                            ? fminf(fmaxf(fabsf(r - rp), 0.15f * r), 0.5f * r)
                                            : r - rp;
                    const float hl = fminf(fmaxf(float(args.step_scale) * scale,
                                                 float(args.min_step)),
                                           float(args.max_step));
                    h[l] = double(fminf(hl, rcp_approx(fmaxf(1.0f, mom2 * rsqrt_approx(mom2)))));
                    step[l] = true;
                    any_step = true;
                    continue;
                }
            }
            const RayState y = ys.get(l);
            if (it[l] >= args.max_steps) {
                finish(l, y, BH_RAY_MAX_STEPS, nullptr, 0.0);
                continue;
            }
            const double r = rt_radius(args.spin, y.x, y.y, y.z);
            const double mom2 = (y.px * y.px + y.py * y.py) + y.pz * y.pz;
            bool captured = (r <= args.capture_radius) || (mom2 >= args.bail2);
            if (args.interior)
                captured = captured || ((r <= args.capture_radius * 1.002) && (mom2 > 2500.0));
            if (captured) {
                finish(l, y, args.capture_status, nullptr, 0.0);
            } else if (r >= args.escape_radius) {
                finish(l, y, BH_RAY_ESCAPED, nullptr, 0.0);
            } else {
                // reference.py:135-154
                const double scale =
                    args.interior ? np_min(np_max(::fabs(r - args.r_plus), 0.15 * r), 0.5 * r)
                                  : r - args.r_plus;
                double hl = np_min(np_max(args.step_scale * scale, args.min_step), args.max_step);
                h[l] = np_min(hl, 1.0 / np_max(1.0, ::sqrt(mom2)));
                step[l] = true;
                any_step = true;
            }
        }
        if (!any_step) continue;
        // ---- one RK4 step for every stepping slot (reference.py:155-160)
        V hw = T::set(0.0);
#pragma unroll
        for (int l = 0; l < N; ++l) T::put(hw, l, typename T::S(h[l]));
        V S[7];
        rk4_sums<V>(K, yw, hw, S);
#pragma unroll
        for (int l = 0; l < N; ++l) {
            if (!step[l]) continue;
            const RayState y0 = ys.get(l);
            RayState y = y0;
            rk4_update<V>(y, S, l, h[l]);
            ++it[l];
            ys.set(l, y);
            put_work<V>(yw, l, y);
            // ---- disk crossing (reference.py:162-184)
            if (disk && y0.z * y.z < 0.0) {
                const double t = y0.z / (y0.z - y.z);
                const RayState q{y0.t + t * (y.t - y0.t), y0.x + t * (y.x - y0.x),
                                 y0.y + t * (y.y - y0.y), y0.z + t * (y.z - y0.z),
                                 y0.pt + t * (y.pt - y0.pt), y0.px + t * (y.px - y0.px),
                                 y0.py + t * (y.py - y0.py), y0.pz + t * (y.pz - y0.pz)};
                const double r_hit = rt_radius(args.spin, q.x, q.y, q.z);
                if (r_hit >= args.disk_inner && r_hit <= args.disk_outer)
                    finish(l, y, BH_RAY_DISK, &q, r_hit);
            }
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        my_steps += __shfl_down_sync(full, my_steps, off);
        const long long o = __shfl_down_sync(full, my_max, off);
        my_max = o > my_max ? o : my_max;
    }
    if (lane == 0) {
        atomicAdd(&ws->attempts, my_steps);
        atomicAdd(&ws->accepted, my_steps);
        atomicMax(&ws->iterations, my_max);
    }
}

static int rt_invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

template <class V, int BLOCK, int MINB>
static cudaError_t launch_realtime(const RealtimeArgs &a, cudaStream_t s) {
    const void *fn = (const void *)realtime_kernel<V, BLOCK, MINB>;
    const size_t smem = StateStore<V, BLOCK>::shared_bytes();
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BLOCK, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    constexpr int kRays = BLOCK * VT<V>::N;
    long long blocks = (long long)sms * occ;
    const long long need = (a.n + kRays - 1) / kRays;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    RealtimeArgs args = a;
    void *params[] = {(void *)&args};
    return cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(BLOCK), params, smem, s);
}

}  // namespace bh

using namespace bh;

extern "C" int bh_trace_realtime(const bh_realtime_config *config, double mass, double spin,
                                 const double *state0, double *states, int32_t *status,
                                 double *hit_radius, double *hit_positions,
                                 double *hit_momenta, int64_t n, void *workspace,
                                 void *stream) {
    if (!config) return rt_invalid("config is NULL");
    const bh_realtime_config &c = *config;
    if (!(mass > 0.0) || !(std::fabs(spin) <= mass))
        return rt_invalid("Kerr bound violated or mass not positive");
    // realtime/settings.py:122-160 (validate), the ranges this kernel relies on.
    if (c.max_steps < 1 || c.max_steps > 4096) return rt_invalid("max_steps must be in [1, 4096]");
    if (!(c.step_scale > 0.0)) return rt_invalid("step_scale must be positive");
    if (!(c.min_step > 0.0 && c.min_step <= c.max_step))
        return rt_invalid("require 0 < min_step <= max_step");
    if (!(c.capture_margin >= 0.0)) return rt_invalid("capture_margin must be non-negative");
    if (!(c.momentum_bailout > 1.0)) return rt_invalid("momentum_bailout must exceed 1");
    if (!(c.escape_radius > 0.0)) return rt_invalid("escape_radius must be positive");
    if (c.disk_outer > 0.0 && !(c.disk_inner >= 0.0 && c.disk_inner <= c.disk_outer))
        return rt_invalid("disk radii must satisfy 0 <= disk_inner <= disk_outer");
    if (c.precision != BH_PRECISION_FP64 && c.precision != BH_PRECISION_MIXED)
        return rt_invalid("precision must be BH_PRECISION_FP64 or BH_PRECISION_MIXED");
    if (n < 0) return rt_invalid("n must be >= 0");
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u)) {
        set_error("workspace must be a 256-byte aligned device buffer of bh_trace_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(TraceWorkspace), s);
    if (e != cudaSuccess) {
        set_error("bh_trace_realtime workspace reset: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    if (n == 0) return BH_OK;
    if (!state0 || !states || !status || !hit_radius || !hit_positions || !hit_momenta)
        return rt_invalid("NULL pointer argument");
    if ((reinterpret_cast<uintptr_t>(state0) | reinterpret_cast<uintptr_t>(states)) & 15u)
        return rt_invalid("state buffers must be 16-byte aligned");
    RealtimeArgs a;
    a.state0 = state0;
    a.n = n;
    a.mass = mass;
    a.spin = spin;
    a.r_plus = mass + std::sqrt(mass * mass - spin * spin);
    a.interior = c.interior_stop > 0.0 ? 1 : 0;
    a.capture_radius = a.interior ? c.interior_stop : a.r_plus * (1.0 + c.capture_margin);
    a.capture_status = a.interior ? BH_RAY_TERMINATED : BH_RAY_CAPTURED;
    a.escape_radius = c.escape_radius;
    a.step_scale = c.step_scale;
    a.min_step = c.min_step;
    a.max_step = c.max_step;
    a.bail2 = c.momentum_bailout * c.momentum_bailout;
    a.disk_inner = c.disk_inner;
    a.disk_outer = c.disk_outer;
    // reference.py:99-102: interior cameras cap the budget at 1024.
    a.max_steps = a.interior && c.max_steps > 1024 ? 1024 : c.max_steps;
    a.states = states;
    a.status = status;
    a.hit_radius = hit_radius;
    a.hit_pos = hit_positions;
    a.hit_mom = hit_momenta;
    a.ws = reinterpret_cast<TraceWorkspace *>(workspace);
    // One ray per thread in both policies.  Two rays per thread in packed
    // float32x2 arithmetic were measured slower here (1.34-1.37 against 1.30
    // ms per 1280x720 frame, 128 x 2 and 128 x 3 blocks): the per-step
    // float64 state update does not pack, and the packed kernel's 138-150
    // registers leave fewer warps.
    e = c.precision == BH_PRECISION_FP64 ? launch_realtime<double, 128, 3>(a, s)
                                         : launch_realtime<float, 128, 4>(a, s);
    if (e != cudaSuccess) {
        set_error("bh_trace_realtime launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
