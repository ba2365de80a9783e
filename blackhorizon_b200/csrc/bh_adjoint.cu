// bh_adjoint.cu -- discrete adjoint of the accepted DP5(4) step sequence and
// the frozen-sequence replay it differentiates.
//
// A traced ray is the composition of its accepted steps y_{k+1} =
// Phi(y_k; h_k, a) with the step sizes h_k the controller chose (recorded on
// the tape by bh_trace_tape).  With that sequence frozen, the cotangent of
// the final state is pulled back step by step,
//     lambda_k = (dPhi/dy_k)^T lambda_{k+1},   g_a += (dPhi/da)^T lambda_{k+1},
// so one sweep gives the gradient with respect to the initial state (hence
// camera pose and pixel coordinates) and the spin at once.  States are not
// stored per step: the tape holds one float64 checkpoint every K accepted
// steps; each segment is replayed forward from its checkpoint into a
// per-thread buffer of K states (rounded to the sweep's work type: 32 bytes
// each for the float sweep) and then swept backward, the stages of each step
// recomputed inside the vector-Jacobian product.  One ray per thread.
#include "bh_adjoint.cuh"
#include "bh_internal.h"

namespace bh {

constexpr int kMaxCheckpointEvery = 64;

__device__ __forceinline__ RayState read8(const double *p) {
    return RayState{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7]};
}

__device__ __forceinline__ void write8(double *p, const RayState &y) {
    p[0] = y.t; p[1] = y.x; p[2] = y.y; p[3] = y.z;
    p[4] = y.pt; p[5] = y.px; p[6] = y.py; p[7] = y.pz;
}

// Accepted DP5(4) steps of a frozen sequence h[0..n_steps) from y, in the
// tracer's own arithmetic (dp5_attempt + commit with lane type V).  With
// `before` non-null it writes the state before each step there, rounded to
// the sweep's work type W (all the vector-Jacobian product reads), and stops
// before the last step, whose result the caller does not use.
template <class V, typename W>
__device__ __forceinline__ RayState replay_steps(double m, double a, RayState y,
                                                 const double *h, long long n_steps,
                                                 Vec8<W> *before) {
    using T = VT<V>;
    const KerrV<V> K = make_kerr<V>(T::set(m), T::set(a));
    WStateV<V> yw;
    put_work<V>(yw, 0, y);
    StageV<V> k1 = first_stage<V>(K, yw);
    for (long long k = 0; k < n_steps; ++k) {
        if (before) {
            before[k] = to_work<W>(y);
            if (k == n_steps - 1) break;
        }
        const double hk = h[k];
        AttemptV<V> at;
        dp5_attempt<V>(K, yw, T::set(hk), k1, at);
        commit<V>(y, yw, at, 0, hk);
        k1 = at.k7;
    }
    return y;
}

// Four warps per block, three blocks per SM (a 170-register cap, which the
// float64 sweep fits without spilling).  Two-warp blocks were measured
// slower for float64.
constexpr int kAdjointBlock = 128;

template <class V, typename W>
__global__ void __launch_bounds__(kAdjointBlock, 3) adjoint_kernel(
    double m, double a, const double *h_tape, const double *ckpt,
    const int64_t *steps, long long cap, int every, const double *grad_states,
    double *grad_state0, double *grad_spin, const int64_t *order, long long n) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n) return;
    const long long i = order ? (long long)order[tid] : tid;
    const double *g = grad_states + 8 * i;
    Vec8<double> lam{g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7]};
    double ga = 0.0;
    const bool zero = lam.t == 0.0 && lam.x == 0.0 && lam.y == 0.0 && lam.z == 0.0 &&
                      lam.pt == 0.0 && lam.px == 0.0 && lam.py == 0.0 && lam.pz == 0.0;
    long long N = steps[i];
    if (N > cap) N = cap;
    if (!zero && N > 0) {
        const long long nck = (cap + every - 1) / every;
        const double *h = h_tape + i * cap;
        Vec8<W> seg_states[kMaxCheckpointEvery];
        for (long long seg = (N - 1) / every; seg >= 0; --seg) {
            const long long k0 = seg * every;
            const long long len = (N - k0 < every) ? (N - k0) : every;
            const RayState y0 = read8(ckpt + (i * nck + seg) * 8);
            replay_steps<V, W>(m, a, y0, h + k0, len, seg_states);
            // The next step's state and size are loaded before this step's
            // vector-Jacobian product, which hides their latency.
            Vec8<W> cur = seg_states[len - 1];
            double hc = h[k0 + len - 1];
            for (long long k = len - 1; k >= 0; --k) {
                Vec8<W> nxt = cur;
                double hn = hc;
                if (k > 0) {
                    nxt = seg_states[k - 1];
                    hn = h[k0 + k - 1];
                }
                dp5_step_vjp<W>(W(m), W(a), cur, hc, lam, ga);
                cur = nxt;
                hc = hn;
            }
        }
    }
    double *o = grad_state0 + 8 * i;
    o[0] = lam.t; o[1] = lam.x; o[2] = lam.y; o[3] = lam.z;
    o[4] = lam.pt; o[5] = lam.px; o[6] = lam.py; o[7] = lam.pz;
    grad_spin[i] = ga;
}

template <class V>
__global__ void __launch_bounds__(128) replay_kernel(
    double m, double a, const double *state0, const double *h_tape,
    const int64_t *steps, long long cap, double *states, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long N = steps[i];
    if (N > cap) N = cap;
    const RayState y = replay_steps<V, double>(m, a, read8(state0 + 8 * i), h_tape + i * cap,
                                               N, nullptr);
    write8(states + 8 * i, y);
}

}  // namespace bh

using namespace bh;

static unsigned grid128(long long n) {
    long long g = (n + 127) / 128;
    return (unsigned)(g < 1 ? 1 : g);
}

static unsigned grid_adjoint(long long n) {
    long long g = (n + kAdjointBlock - 1) / kAdjointBlock;
    return (unsigned)(g < 1 ? 1 : g);
}

extern "C" int bh_trace_tape(const bh_trace_config *config, const bh_scene *scene,
                             const double *state0, double *states, int32_t *status,
                             int64_t *steps, int64_t n, double *h_tape,
                             double *checkpoints, int64_t capacity,
                             int32_t checkpoint_every, void *workspace, void *stream) {
    if (!h_tape || !checkpoints) {
        set_error("h_tape and checkpoints must not be NULL");
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (capacity < 1 || checkpoint_every < 1 || checkpoint_every > kMaxCheckpointEvery) {
        set_error("capacity must be >= 1 and checkpoint_every in [1, %d]", kMaxCheckpointEvery);
        return BH_ERR_INVALID_ARGUMENT;
    }
    return bh_trace_with_tape(config, scene, state0, states, status, steps, n, workspace,
                              stream, h_tape, checkpoints, capacity, checkpoint_every);
}

extern "C" int bh_adjoint(int32_t precision, double mass, double spin,
                          const double *h_tape, const double *checkpoints,
                          const int64_t *steps, int64_t capacity,
                          int32_t checkpoint_every, const double *grad_states,
                          double *grad_state0, double *grad_spin, const int64_t *order,
                          int64_t n, void *stream) {
    if (!(mass > 0.0) || !(fabs(spin) <= mass)) {
        set_error("Kerr bound violated or mass not positive");
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (n < 0 || capacity < 1 || checkpoint_every < 1 ||
        checkpoint_every > kMaxCheckpointEvery) {
        set_error("bad size: n >= 0, capacity >= 1, checkpoint_every in [1, %d]",
                  kMaxCheckpointEvery);
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return BH_OK;
    if (!h_tape || !checkpoints || !steps || !grad_states || !grad_state0 || !grad_spin) {
        set_error("NULL pointer argument");
        return BH_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == BH_PRECISION_FP64)
        adjoint_kernel<double, double><<<grid_adjoint(n), kAdjointBlock, 0, s>>>(
            mass, spin, h_tape, checkpoints, steps, capacity, checkpoint_every, grad_states,
            grad_state0, grad_spin, order, n);
    else if (precision == BH_PRECISION_MIXED)
        adjoint_kernel<float, float><<<grid_adjoint(n), kAdjointBlock, 0, s>>>(
            mass, spin, h_tape, checkpoints, steps, capacity, checkpoint_every, grad_states,
            grad_state0, grad_spin, order, n);
    else {
        set_error("unknown precision");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("bh_adjoint launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}

extern "C" int bh_replay(int32_t precision, double mass, double spin, const double *state0,
                         const double *h_tape, const int64_t *steps, int64_t capacity,
                         double *states, int64_t n, void *stream) {
    if (!(mass > 0.0) || !(fabs(spin) <= mass)) {
        set_error("Kerr bound violated or mass not positive");
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (n < 0 || capacity < 1) {
        set_error("n must be >= 0 and capacity >= 1");
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return BH_OK;
    if (!state0 || !h_tape || !steps || !states) {
        set_error("NULL pointer argument");
        return BH_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == BH_PRECISION_FP64)
        replay_kernel<double><<<grid128(n), 128, 0, s>>>(mass, spin, state0, h_tape, steps,
                                                          capacity, states, n);
    else if (precision == BH_PRECISION_MIXED)
        replay_kernel<float><<<grid128(n), 128, 0, s>>>(mass, spin, state0, h_tape, steps,
                                                         capacity, states, n);
    else {
        set_error("unknown precision");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("bh_replay launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
