// bh_trace_common.cuh -- device helpers shared by the persistent tracers
// (bh_trace.cu, bh_tile.cu): state loads and stores in either layout, ray
// generation from a camera, lane selects, and the per-thread float64 state
// store.
#pragma once

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

// The radius the termination cascade compares with the capture and escape
// radii, after an accepted step.  r2_est is r^2 at the new state from the
// stage arithmetic (the FSAL evaluation, at the float32 rounding of the new
// state for float lanes).  Its error is below 1e-6 (r^2 + 2 a^2) absolute:
// rounding of the position and of q = |x|^2 - a^2 and s (which cancel in
// (q + s)/2 inside |x| < |a|), all bounded by a few units in the last place
// of |x|^2 + a^2 <= r^2 + 2 a^2.  Where the estimate lies inside both
// thresholds by 1e-3 r^2 + 1e-4 a^2 or more, the float64 tests would both
// fail, and NaN, which fails them too, stands in for the radius.  Only near
// a threshold, or for a non-finite estimate, is the float64 radius computed.
__device__ __forceinline__ double settled_radius(double r2_est, double rcap, double resc,
                                                 double a, const RayState &y) {
    const double slack = 1e-4 * (a * a);
    if (r2_est - slack > rcap * rcap * (1.0 + 1e-3) &&
        r2_est + slack < resc * resc * (1.0 - 1e-3))
        return __longlong_as_double(0x7ff8000000000000LL);
    return ks_radius(a, y);
}

// Lane-wise select of a lane-type value: dst[l] = src[l] where take[l].
template <class V>
__device__ __forceinline__ void take_lanes(V &dst, const V &src, const bool *take) {
    using T = VT<V>;
#pragma unroll
    for (int l = 0; l < T::N; ++l)
        if (take[l]) T::put(dst, l, T::get(src, l));
}

template <class V>
__device__ __forceinline__ void take_stage(StageV<V> &d, const StageV<V> &s, const bool *take) {
    take_lanes(d.kx, s.kx, take); take_lanes(d.ky, s.ky, take); take_lanes(d.kz, s.kz, take);
    take_lanes(d.thl, s.thl, take);
    take_lanes(d.px, s.px, take); take_lanes(d.py, s.py, take); take_lanes(d.pz, s.pz, take);
}

template <class V>
__device__ __forceinline__ V lanes_of(const double *v) {
    using T = VT<V>;
    V out = T::set(0.0);
#pragma unroll
    for (int l = 0; l < T::N; ++l) T::put(out, l, typename T::S(v[l]));
    return out;
}

// Where a thread keeps the float64 states of its N rays between attempts.
// float64 lanes: in registers (they coincide with the lane-type copy).
// float32 lanes: in shared memory, one plane per component, since the stages
// only read the rounded copy and the float64 state is touched on accept only;
// this frees 16 registers per ray.
template <class V, int BLOCK>
struct StateStore {
    static constexpr int N = VT<V>::N;
    static constexpr bool kShared = true;
    RayState reg[kShared ? 1 : N];
    double *sh;
    __device__ __forceinline__ explicit StateStore(double *smem) : sh(smem) {}
    __device__ __forceinline__ RayState get(int l) const {
        if constexpr (kShared) {
            const double *p = sh + l * BLOCK + threadIdx.x;
            constexpr int P = N * BLOCK;
            return RayState{p[0], p[P], p[2 * P], p[3 * P], p[4 * P], p[5 * P], p[6 * P], p[7 * P]};
        } else {
            return reg[l];
        }
    }
    __device__ __forceinline__ void set(int l, const RayState &y) {
        if constexpr (kShared) {
            double *p = sh + l * BLOCK + threadIdx.x;
            constexpr int P = N * BLOCK;
            p[0] = y.t; p[P] = y.x; p[2 * P] = y.y; p[3 * P] = y.z;
            p[4 * P] = y.pt; p[5 * P] = y.px; p[6 * P] = y.py; p[7 * P] = y.pz;
        } else {
            reg[l] = y;
        }
    }
    static constexpr size_t shared_bytes() { return kShared ? size_t(8) * N * BLOCK * 8 : 0; }
};

// Refill batching of the persistent tracers: a refill costs the warp one
// first-stage evaluation however many idle slots it fills, so idle slots wait
// for company, at least a batch of them or a number of iterations.  Measured
// (statuses unchanged in every setting):
//  - the tile tracer on the offline renderer's frame (72 attempts per ray):
//    refilling at once 12.66 / 29.91 ms (mixed / float64), batches of 2 or 1
//    iteration 12.50 / 29.20, 16 or 8 iterations 11.95 / 26.15, 32 or 16
//    iterations 11.89 / 24.89, 48 or 16 iterations 11.82 / 25.0;
//  - the tracer on the full-HD frame (222 attempts per ray): 2 or 1 iteration
//    15.74 / 38.76 ms, 16 or 8 iterations 15.67 / 36.80, 32 or 8 15.66 / 36.79.
#ifndef BH_TILE_REFILL_BATCH
#define BH_TILE_REFILL_BATCH 32
#endif
#ifndef BH_TILE_REFILL_WAIT
#define BH_TILE_REFILL_WAIT 16
#endif
#ifndef BH_TRACE_REFILL_BATCH
#define BH_TRACE_REFILL_BATCH 16
#endif
#ifndef BH_TRACE_REFILL_WAIT
#define BH_TRACE_REFILL_WAIT 8
#endif

}  // namespace bh
