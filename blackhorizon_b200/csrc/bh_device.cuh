// bh_device.cuh -- device-side physics of the geodesic hot path (sm_100a).
//
// Kerr-Schild geometry (blackhorizon/kerr.py:118-193), the Hamiltonian
// right-hand side (blackhorizon/geodesics.py:42-74), the Dormand-Prince 5(4)
// attempt with its error norm and step controller (blackhorizon/
// integrators.py:23-124) and the termination cascade (blackhorizon/
// tracer.py:113-149), written for one ray per thread with the state in
// registers.
//
// Precision policy: the work type W is double (BH_PRECISION_FP64) or float
// (BH_PRECISION_MIXED).  The state y, its update, the error norm, the step
// size and the termination radius are always double.  W carries the stage
// arithmetic: the RHS evaluations and the stage combinations.
//
// Derivative split.  With the momentum P_i of stage i, the position
// derivative is dx/dlam = P_i - 2 H lp l and dt/dlam = -p_t + 2 H lp
// (geodesics.py:66-68).  Writing P_i = p + dP_i (p = momentum at the start of
// the step, dP_i = h * sum_j a_ij pdot_j) the stage derivative is stored as
//     kappa_i = dP_i - 2 H lp l      (position part, W)
//     thl_i   = 2 H lp               (time part, W)
//     pdot_i                          (momentum part, W)
// and the exact parts p and -p_t are added back in double: sum_j a_ij k_j =
// c_i p + sum_j a_ij kappa_j with c_i = sum_j a_ij.  Because the error
// weights sum to zero, the embedded error needs only the small W parts.  For
// W = double this is the reference arithmetic re-associated; for W = float it
// keeps float32 rounding on the small curvature terms only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bh {

// kerr.py:26 (_TINY).
constexpr double kTiny = 1e-30;

// ---------------------------------------------------------------- fast math
// Approximate float32 special functions (one MUFU instruction each, <= 2 ulp);
// float64 uses the IEEE operations.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <typename W> struct Math;
template <> struct Math<double> {
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double sqrt_(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double tiny() { return kTiny; }
};
template <> struct Math<float> {
    static __device__ __forceinline__ float rcp(float x) { return rcp_approx(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrt_approx(x); }
    static __device__ __forceinline__ float tiny() { return 1e-30f; }
};

// numpy.maximum propagates NaN (fmax would drop it).
template <typename T>
__device__ __forceinline__ T np_max(T a, T b) {
    return (a != a || b != b) ? (a + b) : (a >= b ? a : b);
}
template <typename T>
__device__ __forceinline__ T np_min(T a, T b) {
    return (a != a || b != b) ? (a + b) : (a <= b ? a : b);
}

// ------------------------------------------------------- full geometry (FP64)
// kerr.py:118-193 term by term, for the geometry/hamiltonian/velocity API.
struct Geometry {
    double r, h, l[3], grad_h[3], grad_l[3][3];
};

__device__ __forceinline__ void geometry_full(double m, double a, double x,
                                              double y, double z, bool grads,
                                              Geometry &o) {
    const double a2 = a * a;
    const double rho2 = x * x + y * y + z * z;
    const double q = rho2 - a2;
    double s = ::sqrt(q * q + 4.0 * a2 * z * z);
    s = np_max(s, kTiny);
    const double r2 = 0.5 * (q + s);
    const double r = ::sqrt(np_max(r2, kTiny));
    const double r2pa2 = r2 + a2;
    const double qd = np_max(r2 * r2 + a2 * z * z, kTiny);
    o.r = r;
    o.h = m * r * r2 / qd;
    const double inv_w = 1.0 / np_max(r2pa2, kTiny);
    const double inv_r = 1.0 / r;
    const double lx = (r * x + a * y) * inv_w;
    const double ly = (r * y - a * x) * inv_w;
    const double lz = z * inv_r;
    o.l[0] = lx; o.l[1] = ly; o.l[2] = lz;
    if (!grads) return;
    const double inv_s = 1.0 / s;
    const double r_x = x * r * inv_s, r_y = y * r * inv_s;
    const double r_z = z * r2pa2 * inv_r * inv_s;
    const double inv_qd2 = 1.0 / (qd * qd);
    const double dh_dr = m * r2 * (3.0 * a2 * z * z - r2 * r2) * inv_qd2;
    const double dh_dz = -2.0 * m * a2 * z * r * r2 * inv_qd2;
    o.grad_h[0] = dh_dr * r_x;
    o.grad_h[1] = dh_dr * r_y;
    o.grad_h[2] = dh_dr * r_z + dh_dz;
    const double two_r = 2.0 * r;
    o.grad_l[0][0] = (r_x * x + r) * inv_w - lx * two_r * r_x * inv_w;
    o.grad_l[1][0] = (r_y * x + a) * inv_w - lx * two_r * r_y * inv_w;
    o.grad_l[2][0] = r_z * x * inv_w - lx * two_r * r_z * inv_w;
    o.grad_l[0][1] = (r_x * y - a) * inv_w - ly * two_r * r_x * inv_w;
    o.grad_l[1][1] = (r_y * y + r) * inv_w - ly * two_r * r_y * inv_w;
    o.grad_l[2][1] = r_z * y * inv_w - ly * two_r * r_z * inv_w;
    o.grad_l[0][2] = -lz * r_x * inv_r;
    o.grad_l[1][2] = -lz * r_y * inv_r;
    o.grad_l[2][2] = (1.0 - lz * r_z) * inv_r;
}

// Kerr-Schild radius squared in float64, with the cancellation-free form
// r^2 = 2 a^2 z^2 / (s - q) when q < 0 (inside |rho| < |a|, where
// 0.5 (q + s) loses digits).  Used for the capture/escape tests.
__device__ __forceinline__ double ks_radius2(double a, double x, double y,
                                             double z) {
    const double a2 = a * a;
    const double a2z2 = a2 * z * z;
    const double q = x * x + y * y + z * z - a2;
    const double s = np_max(::sqrt(q * q + 4.0 * a2z2), kTiny);
    const double r2 = q >= 0.0 ? 0.5 * (q + s) : 2.0 * a2z2 / (s - q);
    return np_max(r2, kTiny);
}

// ------------------------------------------------------------ compact RHS
// Output of one RHS evaluation in the split form described at the top.
template <typename W>
struct Deriv {
    W thl;           // 2 H lp: dt/dlam = -p_t + thl
    W qx, qy, qz;    // -thl * l: dx/dlam = P + q
    W px, py, pz;    // dp/dlam
};

// geodesics.py:42-74 with kerr.py:118-193 folded in.  The 3x3 gradient of l
// is never formed: its contraction with p is
//   c_i = r_i G + (r p_x - a p_y, r p_y + a p_x, 0)_i / (r^2+a^2) + (0,0,p_z/r)_i
//   G   = (x p_x + y p_y - 2 r (l_x p_x + l_y p_y)) / (r^2+a^2) - z p_z / r^2
// and with grad H = dH/dr grad r + (0, 0, dH/dz|_r) the momentum derivative is
//   pdot_i = r_i (dH/dr lp^2 + thl G) + [thl * the explicit terms above]
// which is the reference's grad_h * lp^2 + thl * (grad_l . p) regrouped.
template <typename W>
__device__ __forceinline__ Deriv<W> rhs(W m, W a, W x, W y, W z, W pt, W px,
                                        W py, W pz) {
    using M = Math<W>;
    const W a2 = a * a;
    const W z2 = z * z;
    const W a2z2 = a2 * z2;
    const W q = x * x + y * y + z2 - a2;
    const W s = np_max(M::sqrt_(q * q + W(4) * a2z2), M::tiny());
    W r2;
    if constexpr (sizeof(W) == 8) {
        r2 = W(0.5) * (q + s);  // kerr.py:141, as the reference computes it
    } else {
        r2 = q >= W(0) ? W(0.5) * (q + s) : W(2) * a2z2 * M::rcp(s - q);
    }
    r2 = np_max(r2, M::tiny());
    const W r = M::sqrt_(r2);
    const W w = r2 + a2;
    const W qd = np_max(r2 * r2 + a2z2, M::tiny());
    const W inv_qd = M::rcp(qd);
    const W h = m * r * r2 * inv_qd;
    const W inv_w = M::rcp(np_max(w, M::tiny()));
    const W inv_r = M::rcp(r);
    const W inv_s = M::rcp(s);
    const W lx = (r * x + a * y) * inv_w;
    const W ly = (r * y - a * x) * inv_w;
    const W lz = z * inv_r;
    const W lxy = lx * px + ly * py;
    const W lp = -pt + (lxy + lz * pz);
    const W thl = W(2) * h * lp;
    Deriv<W> d;
    d.thl = thl;
    d.qx = -thl * lx;
    d.qy = -thl * ly;
    d.qz = -thl * lz;
    const W rs = r * inv_s;
    const W r_x = x * rs, r_y = y * rs;
    const W r_z = z * w * inv_r * inv_s;
    const W inv_qd2 = inv_qd * inv_qd;
    const W lp2 = lp * lp;
    const W dh_dr = m * r2 * (W(3) * a2z2 - r2 * r2) * inv_qd2;
    const W dh_dz = W(-2) * m * a2 * z * r * r2 * inv_qd2;
    const W u = x * px + y * py;
    const W g = (u - W(2) * r * lxy) * inv_w - z * pz * inv_r * inv_r;
    const W k = dh_dr * lp2 + thl * g;
    const W tw = thl * inv_w;
    d.px = r_x * k + tw * (r * px - a * py);
    d.py = r_y * k + tw * (r * py + a * px);
    d.pz = r_z * k + dh_dz * lp2 + thl * pz * inv_r;
    return d;
}

// ---------------------------------------------------------------- tableau
// integrators.py:24-54 (autonomous form); c_i = sum_j a_ij.
namespace dp {
constexpr double A21 = 1.0 / 5.0;
constexpr double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
constexpr double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
constexpr double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0,
                 A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
constexpr double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0,
                 A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                 A65 = -5103.0 / 18656.0;
constexpr double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                 B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
constexpr double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0,
                 E4 = 71.0 / 1920.0, E5 = -17253.0 / 339200.0,
                 E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;
constexpr double C2 = 1.0 / 5.0, C3 = 3.0 / 10.0, C4 = 4.0 / 5.0,
                 C5 = 8.0 / 9.0, C6 = 1.0;
}  // namespace dp

// One ray's integration state.
struct RayState {
    double t, x, y, z, pt, px, py, pz;
};

// Stage derivative in the split form: kappa (position), thl (time), pd (momentum).
template <typename W>
struct Stage {
    W kx, ky, kz, thl, px, py, pz;
};

template <typename W>
__device__ __forceinline__ Stage<W> make_stage(const Deriv<W> &d, W dpx,
                                               W dpy, W dpz) {
    Stage<W> s;
    s.kx = dpx + d.qx;
    s.ky = dpy + d.qy;
    s.kz = dpz + d.qz;
    s.thl = d.thl;
    s.px = d.px;
    s.py = d.py;
    s.pz = d.pz;
    return s;
}

// Evaluates the RHS at stage input (X = x + h (c p + S), P = p + dP).
template <typename W>
__device__ __forceinline__ Stage<W> eval_stage(W m, W a, const RayState &y,
                                               const W yw[7], double h, W hw,
                                               double c, W sx, W sy, W sz,
                                               W dpx, W dpy, W dpz) {
    W X, Y, Z;
    if constexpr (sizeof(W) == 8) {
        X = y.x + h * (c * y.px + sx);
        Y = y.y + h * (c * y.py + sy);
        Z = y.z + h * (c * y.pz + sz);
    } else {
        const W cw = W(c);
        X = yw[0] + hw * (cw * yw[4] + sx);
        Y = yw[1] + hw * (cw * yw[5] + sy);
        Z = yw[2] + hw * (cw * yw[6] + sz);
    }
    const Deriv<W> d = rhs<W>(m, a, X, Y, Z, yw[3], yw[4] + dpx, yw[5] + dpy,
                              yw[6] + dpz);
    return make_stage<W>(d, dpx, dpy, dpz);
}

#define BH_LIN2(f, c1, s1, c2, s2) (W(c1) * (s1).f + W(c2) * (s2).f)
#define BH_LIN3(f, c1, s1, c2, s2, c3, s3) (BH_LIN2(f, c1, s1, c2, s2) + W(c3) * (s3).f)
#define BH_LIN4(f, c1, s1, c2, s2, c3, s3, c4, s4) (BH_LIN3(f, c1, s1, c2, s2, c3, s3) + W(c4) * (s4).f)
#define BH_LIN5(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5) (BH_LIN4(f, c1, s1, c2, s2, c3, s3, c4, s4) + W(c5) * (s5).f)
#define BH_LIN6(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5, c6, s6) (BH_LIN5(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5) + W(c6) * (s6).f)

// Result of one DP5(4) attempt (integrators.py:76-107).
template <typename W>
struct Attempt {
    RayState y_new;
    double err[8];  // t x y z pt px py pz; err[4] == 0 (p_t is conserved)
    Stage<W> k7;    // derivative at y_new, relative to y_new's momentum
};

// One embedded Dormand-Prince 5(4) attempt from y with step h, reusing the
// first-same-as-last derivative k1 = f(y).  Identical in exact arithmetic to
// dormand_prince_step, which recomputes k1 every call.
template <typename W>
__device__ __forceinline__ void dp5_attempt(W m, W a, const RayState &y,
                                            double h, const Stage<W> &k1,
                                            Attempt<W> &out) {
    using namespace dp;
    const W yw[7] = {W(y.x), W(y.y), W(y.z), W(y.pt), W(y.px), W(y.py), W(y.pz)};
    const W hw = W(h);
    Stage<W> k2, k3, k4, k5, k6;
    {
        const W dpx = hw * (W(A21) * k1.px), dpy = hw * (W(A21) * k1.py),
                dpz = hw * (W(A21) * k1.pz);
        k2 = eval_stage<W>(m, a, y, yw, h, hw, C2, W(A21) * k1.kx,
                           W(A21) * k1.ky, W(A21) * k1.kz, dpx, dpy, dpz);
    }
    {
        const W dpx = hw * BH_LIN2(px, A31, k1, A32, k2);
        const W dpy = hw * BH_LIN2(py, A31, k1, A32, k2);
        const W dpz = hw * BH_LIN2(pz, A31, k1, A32, k2);
        k3 = eval_stage<W>(m, a, y, yw, h, hw, C3, BH_LIN2(kx, A31, k1, A32, k2),
                           BH_LIN2(ky, A31, k1, A32, k2),
                           BH_LIN2(kz, A31, k1, A32, k2), dpx, dpy, dpz);
    }
    {
        const W dpx = hw * BH_LIN3(px, A41, k1, A42, k2, A43, k3);
        const W dpy = hw * BH_LIN3(py, A41, k1, A42, k2, A43, k3);
        const W dpz = hw * BH_LIN3(pz, A41, k1, A42, k2, A43, k3);
        k4 = eval_stage<W>(m, a, y, yw, h, hw, C4,
                           BH_LIN3(kx, A41, k1, A42, k2, A43, k3),
                           BH_LIN3(ky, A41, k1, A42, k2, A43, k3),
                           BH_LIN3(kz, A41, k1, A42, k2, A43, k3), dpx, dpy, dpz);
    }
    {
        const W dpx = hw * BH_LIN4(px, A51, k1, A52, k2, A53, k3, A54, k4);
        const W dpy = hw * BH_LIN4(py, A51, k1, A52, k2, A53, k3, A54, k4);
        const W dpz = hw * BH_LIN4(pz, A51, k1, A52, k2, A53, k3, A54, k4);
        k5 = eval_stage<W>(m, a, y, yw, h, hw, C5,
                           BH_LIN4(kx, A51, k1, A52, k2, A53, k3, A54, k4),
                           BH_LIN4(ky, A51, k1, A52, k2, A53, k3, A54, k4),
                           BH_LIN4(kz, A51, k1, A52, k2, A53, k3, A54, k4), dpx,
                           dpy, dpz);
    }
    {
        const W dpx = hw * BH_LIN5(px, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5);
        const W dpy = hw * BH_LIN5(py, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5);
        const W dpz = hw * BH_LIN5(pz, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5);
        k6 = eval_stage<W>(
            m, a, y, yw, h, hw, C6,
            BH_LIN5(kx, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
            BH_LIN5(ky, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
            BH_LIN5(kz, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5), dpx, dpy,
            dpz);
    }
    // Fifth-order solution (b2 = b7 = 0).
    const W ix = BH_LIN5(kx, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W iy = BH_LIN5(ky, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W iz = BH_LIN5(kz, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W it = BH_LIN5(thl, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W ipx = BH_LIN5(px, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W ipy = BH_LIN5(py, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    const W ipz = BH_LIN5(pz, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    RayState &yn = out.y_new;
    yn.t = y.t + h * (-y.pt + double(it));
    yn.x = y.x + h * (y.px + double(ix));
    yn.y = y.y + h * (y.py + double(iy));
    yn.z = y.z + h * (y.pz + double(iz));
    yn.pt = y.pt;
    const W dpx7 = hw * ipx, dpy7 = hw * ipy, dpz7 = hw * ipz;
    yn.px = y.px + double(dpx7);
    yn.py = y.py + double(dpy7);
    yn.pz = y.pz + double(dpz7);
    // k7 = f(y_new), FSAL for the next step.  For W = float the momentum
    // increment enters the error as dP_7 (its float value), so the error
    // combination sees the same rounding as the stages.
    const Deriv<W> d7 = rhs<W>(m, a, W(yn.x), W(yn.y), W(yn.z), yw[3],
                               W(yn.px), W(yn.py), W(yn.pz));
    const Stage<W> s7 = make_stage<W>(d7, dpx7, dpy7, dpz7);
    out.k7 = make_stage<W>(d7, W(0), W(0), W(0));
    // Embedded error (e2 = 0): the exact parts p and -p_t cancel because the
    // weights e_i sum to zero.
    out.err[0] = h * double(BH_LIN6(thl, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[1] = h * double(BH_LIN6(kx, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[2] = h * double(BH_LIN6(ky, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[3] = h * double(BH_LIN6(kz, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[4] = 0.0;
    out.err[5] = h * double(BH_LIN6(px, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[6] = h * double(BH_LIN6(py, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
    out.err[7] = h * double(BH_LIN6(pz, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7));
}

#undef BH_LIN2
#undef BH_LIN3
#undef BH_LIN4
#undef BH_LIN5
#undef BH_LIN6

// k1 = f(y) in the split form (dP = 0).
template <typename W>
__device__ __forceinline__ Stage<W> first_stage(W m, W a, const RayState &y) {
    const Deriv<W> d = rhs<W>(m, a, W(y.x), W(y.y), W(y.z), W(y.pt), W(y.px),
                              W(y.py), W(y.pz));
    return make_stage<W>(d, W(0), W(0), W(0));
}

// error_ratio (integrators.py:110-117): RMS over all 8 components of
// err / (atol + rtol max(|y|, |y_new|)); non-finite -> +inf.  Accumulated in
// double; for the mixed policy the division uses a float32 reciprocal of the
// float64 scale (only ~7 digits of the ratio matter to the controller).
template <typename W>
__device__ __forceinline__ double error_ratio(const RayState &y,
                                              const RayState &yn,
                                              const double err[8], double rtol,
                                              double atol) {
    const double yv[8] = {y.t, y.x, y.y, y.z, y.pt, y.px, y.py, y.pz};
    const double nv[8] = {yn.t, yn.x, yn.y, yn.z, yn.pt, yn.px, yn.py, yn.pz};
    double q[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const double sc = atol + rtol * np_max(fabs(yv[i]), fabs(nv[i]));
        double e;
        if constexpr (sizeof(W) == 8) {
            e = err[i] / sc;
        } else {
            e = double(float(err[i]) * rcp_approx(float(sc)));
        }
        q[i] = e * e;
    }
    // NumPy's pairwise order for an 8-element mean.
    const double sum = ((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]));
    const double ratio = ::sqrt(sum * 0.125);
    return isfinite(ratio) ? ratio : __longlong_as_double(0x7ff0000000000000LL);
}

// step_factor (integrators.py:120-124): clip(0.9 max(ratio,1e-16)^-0.2, 0.2, 5).
template <typename W>
__device__ __forceinline__ double step_factor(double ratio) {
    const double safe = np_max(ratio, 1e-16);
    double f;
    if constexpr (sizeof(W) == 8) {
        f = 0.9 * ::pow(safe, -0.2);
    } else {
        // float32 power through exp2/log2; only the step heuristic uses it.
        const float sf = float(fmin(safe, 3.0e38));
        f = double(0.9f * ex2_approx(-0.2f * lg2_approx(sf)));
    }
    return np_min(np_max(f, 0.2), 5.0);
}

__device__ __forceinline__ bool all_finite(const RayState &y) {
    return isfinite(y.t) && isfinite(y.x) && isfinite(y.y) && isfinite(y.z) &&
           isfinite(y.pt) && isfinite(y.px) && isfinite(y.py) && isfinite(y.pz);
}

// --------------------------------------------------------- initial states
// null_momentum_from_velocity (geodesics.py:141-170) for one ray.
__device__ __forceinline__ void null_momentum(double m, double a,
                                              const double pos[3],
                                              const double dir[3], bool past,
                                              bool normalize, double p[4]) {
    Geometry g;
    geometry_full(m, a, pos[0], pos[1], pos[2], false, g);
    const double h = g.h;
    const double l_dot_s = g.l[0] * dir[0] + g.l[1] * dir[1] + g.l[2] * dir[2];
    const double s_dot_s = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
    const double g_tt = 2.0 * h - 1.0;
    const double b = 4.0 * h * l_dot_s;
    const double c = s_dot_s + 2.0 * h * l_dot_s * l_dot_s;
    const double disc = b * b - 4.0 * g_tt * c;
    const double sq = ::sqrt(np_max(disc, 0.0));
    const double ra = (-b + sq) / (2.0 * g_tt);
    const double rb = (-b - sq) / (2.0 * g_tt);
    const double k_t = past ? np_min(ra, rb) : np_max(ra, rb);
    const double l_dot_k = k_t + l_dot_s;
    const double f = 2.0 * h * l_dot_k;
    p[0] = -k_t + f;
    p[1] = dir[0] + f * g.l[0];
    p[2] = dir[1] + f * g.l[1];
    p[3] = dir[2] + f * g.l[2];
    if (normalize) {
        const double n0 = fabs(p[0]);
        p[0] /= n0; p[1] /= n0; p[2] /= n0; p[3] /= n0;
    }
}

// PinholeCamera.ray_directions for pixel index idx = row * width + col
// (camera.py:102-113).
__device__ __forceinline__ void pinhole_direction(
    const double fwd[3], const double right[3], const double up[3],
    double half_w, double half_h, int64_t width, int64_t height, int64_t idx,
    double d[3]) {
    const int64_t row = idx / width;
    const int64_t col = idx - row * width;
    const double u = ((double(col) + 0.5) / double(width) * 2.0 - 1.0) * half_w;
    const double v = (1.0 - (double(row) + 0.5) / double(height) * 2.0) * half_h;
    double e[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) e[i] = fwd[i] + u * right[i] + v * up[i];
    const double nrm = ::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) d[i] = e[i] / nrm;
}

}  // namespace bh
