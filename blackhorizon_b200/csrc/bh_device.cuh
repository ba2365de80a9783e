// bh_device.cuh -- device-side physics of the geodesic hot path (sm_100a).
//
// Kerr-Schild geometry (blackhorizon/kerr.py:118-193), the Hamiltonian
// right-hand side (blackhorizon/geodesics.py:42-74), the Dormand-Prince 5(4)
// attempt with its error norm and step controller (blackhorizon/
// integrators.py:23-124) and the termination cascade (blackhorizon/
// tracer.py:113-149), written for one ray per thread with the state in
// registers.
//
// Precision policy: the lane type V is double (BH_PRECISION_FP64), float
// (BH_PRECISION_MIXED, one ray per thread) or F2 (BH_PRECISION_MIXED, two
// rays per thread in the two halves of packed float32x2 instructions).  The
// state y, its update, the affine parameter, the step size with its accept
// test and the termination radius are always double, per ray.  V carries the
// stage arithmetic: the RHS evaluations, the stage combinations and the
// embedded error with its norm.
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
#include <type_traits>
#include <cuda_runtime.h>

namespace bh {

// kerr.py:26 (_TINY).
constexpr double kTiny = 1e-30;

// ---------------------------------------------------------------- fast math
// Approximate float32 special functions (one MUFU instruction each, <= 2 ulp).
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

// Reciprocal and reciprocal square root of the stage arithmetic.  float32:
// one MUFU instruction (<= 2 ulp).  float64: the MUFU seed (about 23 correct
// bits) refined by two Newton-Raphson steps on the FP64 pipe, each of which
// roughly doubles the correct bits: r <- r + r (1 - x r) for 1/x and
// r <- r (3 - x r^2) / 2 for 1/sqrt(x), the residual formed with a fused
// multiply-add.  Within 2 ulp of the correctly rounded result for normal
// inputs (bh_device_math exposes both for that check), with no IEEE slow
// path.
__device__ __forceinline__ double rcp_f64(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ double rsqrt_f64(double x) {
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    // r <- r (3 - x r^2) / 2, twice.
    double h = 0.5 * x;
    r = r * fma(-h * r, r, 1.5);
    r = r * fma(-h * r, r, 1.5);
    return r;
}

template <typename W> struct Math;
template <> struct Math<double> {
    static __device__ __forceinline__ double rcp(double x) { return rcp_f64(x); }
    static __device__ __forceinline__ double rsqrt(double x) { return rsqrt_f64(x); }
    static __device__ __forceinline__ double tiny() { return kTiny; }
    static __device__ __forceinline__ double tiny2() { return kTiny * kTiny; }
};
template <> struct Math<float> {
    static __device__ __forceinline__ float rcp(float x) { return rcp_approx(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrt_approx(x); }
    static __device__ __forceinline__ float tiny() { return 1e-30f; }
    // Smallest clamp of a squared quantity that stays a normal float.
    static __device__ __forceinline__ float tiny2() { return 1e-37f; }
};

// numpy.maximum propagates NaN (fmax would drop it).  Host code uses them too.
template <typename T>
__host__ __device__ __forceinline__ T np_max(T a, T b) {
    return (a != a || b != b) ? (a + b) : (a >= b ? a : b);
}
template <typename T>
__host__ __device__ __forceinline__ T np_min(T a, T b) {
    return (a != a || b != b) ? (a + b) : (a <= b ? a : b);
}

// ------------------------------------------------------- full geometry (FP64)
// kerr.py:118-193 term by term, for the geometry/hamiltonian/velocity API.
struct Geometry {
    double r, h, l[3], grad_h[3], grad_l[3][3];
};

__host__ __device__ __forceinline__ void geometry_full(double m, double a, double x,
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

// ------------------------------------------------------------- lane types
// F2: two rays side by side, one per half of a float2; arithmetic through the
// packed sm_100 FFMA2 / FADD2 / FMUL2 instructions (two FP32 operations per
// issue), special functions one MUFU per half.
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    return {__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)};
}
__device__ __forceinline__ F2 operator-(F2 a) {
    return {__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))};
}

// Traits of a lane type: N rays, scalar type S, broadcast, lane access and
// the handful of operations the stage arithmetic needs.
template <class V> struct VT;
template <> struct VT<double> {
    static constexpr int N = 1;
    using S = double;
    static __device__ __forceinline__ double set(double a) { return a; }
    static __device__ __forceinline__ double get(double v, int) { return v; }
    static __device__ __forceinline__ void put(double &v, int, double a) { v = a; }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }
    static __device__ __forceinline__ double max(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double abs(double a) { return ::fabs(a); }
    static __device__ __forceinline__ double rcp(double a) { return rcp_f64(a); }
    static __device__ __forceinline__ double rsqrt(double a) { return rsqrt_f64(a); }
    static __device__ __forceinline__ double tiny() { return kTiny; }
    static __device__ __forceinline__ double tiny2() { return kTiny * kTiny; }
};
template <> struct VT<float> {
    static constexpr int N = 1;
    using S = float;
    static __device__ __forceinline__ float set(double a) { return float(a); }
    static __device__ __forceinline__ float get(float v, int) { return v; }
    static __device__ __forceinline__ void put(float &v, int, float a) { v = a; }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float max(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
    static __device__ __forceinline__ float rcp(float a) { return rcp_approx(a); }
    static __device__ __forceinline__ float rsqrt(float a) { return rsqrt_approx(a); }
    static __device__ __forceinline__ float tiny() { return 1e-30f; }
    // Smallest clamp of a squared quantity that stays a normal float.
    static __device__ __forceinline__ float tiny2() { return 1e-37f; }
};
template <> struct VT<F2> {
    static constexpr int N = 2;
    using S = float;
    static __device__ __forceinline__ F2 set(double a) {
        const float f = float(a);
        return {make_float2(f, f)};
    }
    static __device__ __forceinline__ float get(F2 v, int i) { return i == 0 ? v.v.x : v.v.y; }
    static __device__ __forceinline__ void put(F2 &v, int i, float a) {
        if (i == 0) v.v.x = a; else v.v.y = a;
    }
    static __device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
    static __device__ __forceinline__ F2 max(F2 a, F2 b) {
        return {make_float2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y))};
    }
    static __device__ __forceinline__ F2 abs(F2 a) {
        return {make_float2(fabsf(a.v.x), fabsf(a.v.y))};
    }
    static __device__ __forceinline__ F2 rcp(F2 a) {
        return {make_float2(rcp_approx(a.v.x), rcp_approx(a.v.y))};
    }
    static __device__ __forceinline__ F2 rsqrt(F2 a) {
        return {make_float2(rsqrt_approx(a.v.x), rsqrt_approx(a.v.y))};
    }
    static __device__ __forceinline__ float tiny() { return 1e-30f; }
    static __device__ __forceinline__ float tiny2() { return 1e-37f; }
};

// Per-ray Kerr constants in the lane type, formed once per ray.
template <class V>
// m2, na2: the float lanes' form of the RHS; m, a2x4, a2x3, n2ma2: the
// double lanes' (each form reads only its own).
struct KerrV {
    V m, m2, a, na, a2, na2, a2x4, a2x3, n2ma2;
};
template <class V>
__device__ __forceinline__ KerrV<V> make_kerr(V m, V a) {
    using T = VT<V>;
    KerrV<V> k;
    k.m = m;
    k.m2 = m * T::set(2.0);
    k.a = a;
    k.na = -a;
    k.a2 = a * a;
    k.na2 = -k.a2;
    k.a2x4 = k.a2 * T::set(4.0);
    k.a2x3 = k.a2 * T::set(3.0);
    k.n2ma2 = (m * k.a2) * T::set(-2.0);
    return k;
}



// Stage derivative in split form (see the top of this file):
//   kx..kz = dP - 2 H lp l   (position part)   thl = 2 H lp   (time part)
//   px..pz = dp/dlambda      (momentum part)
template <class V>
struct StageV {
    V kx, ky, kz, thl, px, py, pz;
};

// The RHS of the double lanes (the float64 policy), in the operation order
// it has always had: its trajectories are pinned to the reference's end
// points within 1e-7 where the step counts agree, and near the photon sphere
// any rounding change grows past that.  See rhs_v for the regrouping.
__device__ __forceinline__ StageV<double> rhs_f64(const KerrV<double> &K, double x,
                                                  double y, double z, double npt, double px,
                                                  double py, double pz, double dpx,
                                                  double dpy, double dpz, double *r2_out) {
    const double z2 = z * z;
    const double a2z2 = K.a2 * z2;
    const double q = fma(x, x, fma(y, y, z2 - K.a2));
    const double s2 = fmax(fma(q, q, K.a2x4 * z2), kTiny * kTiny);
    const double inv_s = rsqrt_f64(s2);
    const double s = s2 * inv_s;
    const double r2 = fmax((q + s) * 0.5, kTiny);
    if (r2_out) *r2_out = r2;
    const double inv_r = rsqrt_f64(r2);
    const double r = r2 * inv_r;
    const double w = r2 + K.a2;
    const double r2sq = r2 * r2;
    const double qd = fmax(r2sq + a2z2, kTiny);
    const double inv_qd = rcp_f64(qd);
    const double inv_w = rcp_f64(w);
    const double r3 = r * r2;
    const double h = (K.m * r3) * inv_qd;
    const double lx = fma(r, x, K.a * y) * inv_w;
    const double ly = fma(r, y, K.na * x) * inv_w;
    const double lz = z * inv_r;
    const double lxy = fma(lx, px, ly * py);
    const double lzpz = lz * pz;
    const double lp = (lxy + lzpz) + npt;
    const double thl = (h + h) * lp;
    const double nthl = -thl;
    StageV<double> o;
    o.thl = thl;
    o.kx = fma(nthl, lx, dpx);
    o.ky = fma(nthl, ly, dpy);
    o.kz = fma(nthl, lz, dpz);
    const double rs = r * inv_s;
    const double r_x = x * rs, r_y = y * rs;
    const double r_z = z * (w * (inv_r * inv_s));
    const double inv_qd2 = inv_qd * inv_qd;
    const double lp2 = lp * lp;
    const double t3 = K.a2x3 * z2 - r2sq;
    const double dh_dr = ((K.m * r2) * t3) * inv_qd2;
    const double dh_dz = ((K.n2ma2 * z) * r3) * inv_qd2;
    const double u = fma(x, px, y * py);
    const double g1 = fma(r * -2.0, lxy, u);
    const double g = g1 * inv_w - lzpz * inv_r;
    const double k = fma(dh_dr, lp2, thl * g);
    const double tw = thl * inv_w;
    o.px = fma(r_x, k, tw * fma(r, px, K.na * py));
    o.py = fma(r_y, k, tw * fma(r, py, K.a * px));
    o.pz = fma(r_z, k, fma(dh_dz, lp2, (thl * pz) * inv_r));
    return o;
}

// ------------------------------------------------------------ compact RHS
// geodesics.py:42-74 with kerr.py:118-193 folded in, evaluated at position
// (x, y, z) and momentum (pt, px, py, pz); dpx..dpz is the stage's momentum
// offset dP that the position part carries.  npt = -p_t (p_t is conserved).
//
// The 3x3 gradient of l is never formed: its contraction with p is
//   c_i = r_i G + (r p_x - a p_y, r p_y + a p_x, 0)_i / (r^2+a^2) + (0,0,p_z/r)_i
//   G   = (x p_x + y p_y - 2 r (l_x p_x + l_y p_y)) / (r^2+a^2) - z p_z / r^2
// and with grad H = dH/dr grad r + (0, 0, dH/dz|_r) the momentum derivative is
//   pdot_i = r_i (dH/dr lp^2 + thl G) + [thl * the explicit terms above]
// which is the reference's grad_h * lp^2 + thl * (grad_l . p) regrouped.
// The radius uses the reference's r^2 = (q + s)/2 (kerr.py:141) for every
// lane type.  Double lanes take rhs_f64.  Float lanes regroup further:
// - the mass enters through one factor 2m/qd: thl = (2m/qd) r^3 lp, and with
//   mlp = 2m lp^2/qd^2, dH/dr lp^2 = r^2 (3a^2z^2 - r^4)/2 mlp and
//   dH/dz|_r lp^2 = -a^2 z r^3 mlp, (3a^2z^2 - r^4)/2 = 2 a^2 z^2 - qd/2;
// - the clamp constant is added to a^2 z^2, which enters s^2 and qd, instead
//   of taking maxima: both sums are non-negative, and the constant changes
//   neither unless it is within 2^24 of the sum, i.e. at the ring itself;
// - grad r is applied to k/s in one product, dr/dz = l_z (r^2+a^2)/s.
//
// r2_out, when given, receives the radius r^2 the evaluation used.
template <class V>
__device__ __forceinline__ StageV<V> rhs_v(const KerrV<V> &K, V x, V y, V z,
                                           V npt, V px, V py, V pz, V dpx,
                                           V dpy, V dpz, V *r2_out = nullptr) {
    using T = VT<V>;
    if constexpr (sizeof(typename T::S) == 8) {
        return rhs_f64(K, x, y, z, npt, px, py, pz, dpx, dpy, dpz, r2_out);
    } else {
        const V z2 = z * z;
        const V a2z2 = T::fma(K.a2, z2, T::set(T::tiny()));
        const V q = T::fma(x, x, T::fma(y, y, z2 - K.a2));
        const V s2 = T::fma(a2z2, T::set(4.0), q * q);
        const V inv_s = T::rsqrt(s2);
        const V s = s2 * inv_s;
        const V r2 = T::max(T::fma(s, T::set(0.5), q * T::set(0.5)), T::set(T::tiny()));
        if (r2_out) *r2_out = r2;
        const V inv_r = T::rsqrt(r2);
        const V r = r2 * inv_r;
        const V w = r2 + K.a2;
        const V qd = T::fma(r2, r2, a2z2);
        const V inv_qd = T::rcp(qd);
        const V inv_w = T::rcp(w);
        const V r3 = r * r2;
        const V m2i = K.m2 * inv_qd;  // 2m / qd
        const V lx = T::fma(r, x, K.a * y) * inv_w;
        const V ly = T::fma(r, y, K.na * x) * inv_w;
        const V lz = z * inv_r;
        const V lxy = T::fma(lx, px, ly * py);
        const V lp = T::fma(lz, pz, lxy) + npt;
        const V thl = (m2i * r3) * lp;  // 2 H lp
        const V nthl = -thl;
        const V tz = nthl * lz;
        StageV<V> o;
        o.thl = thl;
        o.kx = T::fma(nthl, lx, dpx);
        o.ky = T::fma(nthl, ly, dpy);
        o.kz = tz + dpz;
        const V mlp = (m2i * inv_qd) * (lp * lp);  // 2m lp^2 / qd^2
        const V t3h = T::fma(qd, T::set(-0.5), a2z2 + a2z2);
        // thl G = thl (x p_x + y p_y - 2 r (l_x p_x + l_y p_y)) / w - thl l_z p_z / r.
        const V u = T::fma(x, px, y * py);
        const V g1 = T::fma(r * T::set(-2.0), lxy, u);
        const V tw = thl * inv_w;
        const V pzr = pz * inv_r;
        const V k = T::fma(tz, pzr, T::fma(tw, g1, (r2 * t3h) * mlp));
        // grad r = (x r, y r, z w / r) / s, applied to k / s.
        const V sk = k * inv_s;
        const V rsk = r * sk;
        o.px = T::fma(x, rsk, tw * T::fma(r, px, K.na * py));
        o.py = T::fma(y, rsk, tw * T::fma(r, py, K.a * px));
        o.pz = T::fma(lz * w, sk, T::fma((K.na2 * z) * r3, mlp, thl * pzr));
        return o;
    }
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

// One ray's integration state (float64).
struct RayState {
    double t, x, y, z, pt, px, py, pz;
};

// The rays' states rounded to the lane type: RHS inputs of the stages and
// magnitudes of the error scale.  npt = -p_t.
template <class V>
struct WStateV {
    V t, x, y, z, npt, px, py, pz;
};

template <class V>
__device__ __forceinline__ void put_work(WStateV<V> &w, int l, const RayState &y) {
    using T = VT<V>;
    using S = typename T::S;
    T::put(w.t, l, S(y.t));
    T::put(w.x, l, S(y.x));
    T::put(w.y, l, S(y.y));
    T::put(w.z, l, S(y.z));
    T::put(w.npt, l, S(-y.pt));
    T::put(w.px, l, S(y.px));
    T::put(w.py, l, S(y.py));
    T::put(w.pz, l, S(y.pz));
}

// put_work after a step: p_t is conserved, so its rounded copy stays.
template <class V>
__device__ __forceinline__ void put_work_moved(WStateV<V> &w, int l, const RayState &y) {
    using T = VT<V>;
    using S = typename T::S;
    T::put(w.t, l, S(y.t));
    T::put(w.x, l, S(y.x));
    T::put(w.y, l, S(y.y));
    T::put(w.z, l, S(y.z));
    T::put(w.px, l, S(y.px));
    T::put(w.py, l, S(y.py));
    T::put(w.pz, l, S(y.pz));
}

// Result of one DP5(4) attempt (integrators.py:76-107) for every lane.  The
// float64 candidate state is not formed here: `ynw` (the candidate in the
// lane type) feeds k7 and the error norm, and commit() adds the increments
// to the float64 state once the step is accepted.
template <class V>
struct AttemptV {
    WStateV<V> ynw;  // y_new in the lane type (the next yw if accepted)
    V it, ix, iy, iz;        // sum_i b_i k_i of t, x, y, z without the exact parts
    V dpx, dpy, dpz;         // momentum increments h sum_i b_i pdot_i
    V err[7];        // sum_i e_i k_i for t x y z px py pz (the p_t error is 0)
    StageV<V> k7;    // derivative at y_new relative to y_new's momentum
    V r2n;           // Kerr-Schild r^2 at ynw, from the k7 evaluation
};

// Rounding floor of the mixed policy's error scale.  The embedded error
// h sum_i e_i k_i of float32 stage derivatives carries rounding noise of
// about u h sum_i |e_i| |k_i| (u = 2^-24 per rounding) that, unlike
// truncation error, shrinks only linearly with h, so no step size removes
// it.  Counting it as error made the controller take 2.5x the attempts of
// the float64 policy at rtol 1e-9 with no gain in accuracy.  The mixed
// policy's scale for each component is therefore the larger of atol + rtol
// max(|y|, |y_new|) and this floor, estimated from the step's own increment
// as 2 u (sum_i |e_i|) |h sum_i b_i k_i| (two roundings per term; the
// increment matches the |k_i| weighting when k varies little across the
// step and is smaller, so stricter, when it changes sign).  Where the
// tolerance is the larger, the float64 scale is unchanged.  With it the mixed
// controller takes about the float64 policy's step sequence.
constexpr double kMixedNoise =
    2.0 * (dp::E1 - dp::E3 + dp::E4 - dp::E5 + dp::E6 - dp::E7) * 0x1p-24;

#define BH_LIN2(f, c1, s1, c2, s2) (T::set(c1) * (s1).f + T::set(c2) * (s2).f)
#define BH_LIN3(f, c1, s1, c2, s2, c3, s3) (BH_LIN2(f, c1, s1, c2, s2) + T::set(c3) * (s3).f)
#define BH_LIN4(f, c1, s1, c2, s2, c3, s3, c4, s4) (BH_LIN3(f, c1, s1, c2, s2, c3, s3) + T::set(c4) * (s4).f)
#define BH_LIN5(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5) (BH_LIN4(f, c1, s1, c2, s2, c3, s3, c4, s4) + T::set(c5) * (s5).f)
#define BH_LIN6(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5, c6, s6) (BH_LIN5(f, c1, s1, c2, s2, c3, s3, c4, s4, c5, s5) + T::set(c6) * (s6).f)

// RHS at the stage input X = x + h (c p + S), P = p + dP with
// dP = h sum_j a_ij pdot_j and S = sum_j a_ij kappa_j, formed in the lane type
// from the rounded state (for V = double that is the state itself).
template <class V>
__device__ __forceinline__ StageV<V> stage_at(const KerrV<V> &K, const WStateV<V> &yw,
                                              V hw, double c, V sx, V sy, V sz,
                                              V spx, V spy, V spz) {
    using T = VT<V>;
    const V cw = T::set(c);
    const V dpx = hw * spx, dpy = hw * spy, dpz = hw * spz;
    return rhs_v<V>(K, T::fma(hw, T::fma(cw, yw.px, sx), yw.x),
                    T::fma(hw, T::fma(cw, yw.py, sy), yw.y),
                    T::fma(hw, T::fma(cw, yw.pz, sz), yw.z), yw.npt,
                    yw.px + dpx, yw.py + dpy, yw.pz + dpz, dpx, dpy, dpz);
}

// One embedded Dormand-Prince 5(4) attempt per lane from yw with step hw,
// reusing the first-same-as-last derivative k1 = f(y).  Identical in exact
// arithmetic to dormand_prince_step, which recomputes k1 every call.  The
// embedded error is h times out.err.  The time component's sums are
// accumulated as the stages are produced (it never feeds a stage input).
template <class V>
__device__ __forceinline__ void dp5_attempt(const KerrV<V> &K, const WStateV<V> &yw,
                                            V hw, const StageV<V> &k1,
                                            AttemptV<V> &out) {
    using namespace dp;
    using T = VT<V>;
    V it = T::set(B1) * k1.thl;
    V et = T::set(E1) * k1.thl;
    const StageV<V> k2 = stage_at<V>(K, yw, hw, C2, T::set(A21) * k1.kx, T::set(A21) * k1.ky,
                                     T::set(A21) * k1.kz, T::set(A21) * k1.px,
                                     T::set(A21) * k1.py, T::set(A21) * k1.pz);
    const StageV<V> k3 = stage_at<V>(
        K, yw, hw, C3, BH_LIN2(kx, A31, k1, A32, k2), BH_LIN2(ky, A31, k1, A32, k2),
        BH_LIN2(kz, A31, k1, A32, k2), BH_LIN2(px, A31, k1, A32, k2),
        BH_LIN2(py, A31, k1, A32, k2), BH_LIN2(pz, A31, k1, A32, k2));
    it = T::fma(T::set(B3), k3.thl, it);
    et = T::fma(T::set(E3), k3.thl, et);
    const StageV<V> k4 = stage_at<V>(
        K, yw, hw, C4, BH_LIN3(kx, A41, k1, A42, k2, A43, k3),
        BH_LIN3(ky, A41, k1, A42, k2, A43, k3), BH_LIN3(kz, A41, k1, A42, k2, A43, k3),
        BH_LIN3(px, A41, k1, A42, k2, A43, k3), BH_LIN3(py, A41, k1, A42, k2, A43, k3),
        BH_LIN3(pz, A41, k1, A42, k2, A43, k3));
    it = T::fma(T::set(B4), k4.thl, it);
    et = T::fma(T::set(E4), k4.thl, et);
    const StageV<V> k5 = stage_at<V>(
        K, yw, hw, C5, BH_LIN4(kx, A51, k1, A52, k2, A53, k3, A54, k4),
        BH_LIN4(ky, A51, k1, A52, k2, A53, k3, A54, k4),
        BH_LIN4(kz, A51, k1, A52, k2, A53, k3, A54, k4),
        BH_LIN4(px, A51, k1, A52, k2, A53, k3, A54, k4),
        BH_LIN4(py, A51, k1, A52, k2, A53, k3, A54, k4),
        BH_LIN4(pz, A51, k1, A52, k2, A53, k3, A54, k4));
    it = T::fma(T::set(B5), k5.thl, it);
    et = T::fma(T::set(E5), k5.thl, et);
    const StageV<V> k6 = stage_at<V>(
        K, yw, hw, C6, BH_LIN5(kx, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
        BH_LIN5(ky, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
        BH_LIN5(kz, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
        BH_LIN5(px, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
        BH_LIN5(py, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5),
        BH_LIN5(pz, A61, k1, A62, k2, A63, k3, A64, k4, A65, k5));
    it = T::fma(T::set(B6), k6.thl, it);
    et = T::fma(T::set(E6), k6.thl, et);
    // Fifth-order solution (b2 = b7 = 0).
    out.it = it;
    out.ix = BH_LIN5(kx, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    out.iy = BH_LIN5(ky, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    out.iz = BH_LIN5(kz, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    out.dpx = hw * BH_LIN5(px, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    out.dpy = hw * BH_LIN5(py, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    out.dpz = hw * BH_LIN5(pz, B1, k1, B3, k3, B4, k4, B5, k5, B6, k6);
    WStateV<V> &nw = out.ynw;
    nw.t = T::fma(hw, yw.npt + it, yw.t);
    nw.x = T::fma(hw, yw.px + out.ix, yw.x);
    nw.y = T::fma(hw, yw.py + out.iy, yw.y);
    nw.z = T::fma(hw, yw.pz + out.iz, yw.z);
    nw.npt = yw.npt;
    nw.px = yw.px + out.dpx;
    nw.py = yw.py + out.dpy;
    nw.pz = yw.pz + out.dpz;
    // k7 = f(y_new), FSAL for the next step.  Relative to this step's base
    // momentum its position part carries dP_7 = p_new - p.
    const StageV<V> s7 = rhs_v<V>(K, nw.x, nw.y, nw.z, nw.npt, nw.px, nw.py, nw.pz,
                                  out.dpx, out.dpy, out.dpz, &out.r2n);
    out.k7 = s7;
    out.k7.kx = s7.kx - out.dpx;
    out.k7.ky = s7.ky - out.dpy;
    out.k7.kz = s7.kz - out.dpz;
    // Embedded error / h (e2 = 0): the exact parts p and -p_t cancel because
    // the weights e_i sum to zero.
    out.err[0] = T::fma(T::set(E7), s7.thl, et);
    out.err[1] = BH_LIN6(kx, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
    out.err[2] = BH_LIN6(ky, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
    out.err[3] = BH_LIN6(kz, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
    out.err[4] = BH_LIN6(px, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
    out.err[5] = BH_LIN6(py, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
    out.err[6] = BH_LIN6(pz, E1, k1, E3, k3, E4, k4, E5, k5, E6, k6, E7, s7);
}

// Accepts lane l of an attempt: the float64 state advances by the attempt's
// increments (y + h (p + sum b k) for positions, y + dP for momenta) and the
// lane-type copy becomes the rounded new state.  For V = double the attempt
// already computed exactly these values in double.
template <class V>
__device__ __forceinline__ void commit(RayState &y, WStateV<V> &yw,
                                       const AttemptV<V> &a, int l, double h) {
    using T = VT<V>;
    if constexpr (T::N == 1 && sizeof(typename T::S) == 8) {
        y.t = a.ynw.t; y.x = a.ynw.x; y.y = a.ynw.y; y.z = a.ynw.z;
        y.px = a.ynw.px; y.py = a.ynw.py; y.pz = a.ynw.pz;
    } else {
        y.t = y.t + h * (-y.pt + double(T::get(a.it, l)));
        y.x = y.x + h * (y.px + double(T::get(a.ix, l)));
        y.y = y.y + h * (y.py + double(T::get(a.iy, l)));
        y.z = y.z + h * (y.pz + double(T::get(a.iz, l)));
        y.px = y.px + double(T::get(a.dpx, l));
        y.py = y.py + double(T::get(a.dpy, l));
        y.pz = y.pz + double(T::get(a.dpz, l));
    }
    put_work_moved<V>(yw, l, y);
}

#undef BH_LIN2
#undef BH_LIN3
#undef BH_LIN4
#undef BH_LIN5
#undef BH_LIN6

// k1 = f(y) in split form (dP = 0).
template <class V>
__device__ __forceinline__ StageV<V> first_stage(const KerrV<V> &K, const WStateV<V> &yw) {
    using T = VT<V>;
    const V zero = T::set(0.0);
    return rhs_v<V>(K, yw.x, yw.y, yw.z, yw.npt, yw.px, yw.py, yw.pz, zero, zero, zero);
}

// first_stage that also returns the evaluation's r^2 when r2 is not null.
template <class V>
__device__ __forceinline__ StageV<V> first_stage_r2(const KerrV<V> &K, const WStateV<V> &yw,
                                                    V *r2) {
    using T = VT<V>;
    const V zero = T::set(0.0);
    return rhs_v<V>(K, yw.x, yw.y, yw.z, yw.npt, yw.px, yw.py, yw.pz, zero, zero, zero, r2);
}

// Type of the controller's error ratio.  float64 lanes: the ratio r.  Mixed
// lanes: r^2, in float64 (BH_MIXED_NORM_F64 = 1, the default: the sum of
// squares, the accept test and the step factor in float64) or, built with
// BH_MIXED_NORM_F64 = 0, in float32 (the sum of squares in float32 and the
// factor through float32 exp2/log2; kept to measure the float64 controller
// against).
#ifndef BH_MIXED_NORM_F64
#define BH_MIXED_NORM_F64 1
#endif
template <class V>
using RatioT = typename std::conditional<sizeof(typename VT<V>::S) == 8 || BH_MIXED_NORM_F64 != 0,
                                         double, float>::type;

// error_ratio (integrators.py:110-117) per lane: RMS over all 8 components of
// h err / (atol + rtol max(|y|, |y_new|)), non-finite -> +inf, NumPy's
// pairwise summation order.  The p_t term is exactly zero (p_t is conserved)
// and is counted in the mean.  float64 policy: every operation in double.
// Mixed policy: the error is a float32 combination of float32 stage
// derivatives; its scales and quotients err_i / scale_i are float32 (the
// scale reciprocal is one MUFU instruction), each scale at least the
// rounding floor kMixedNoise |increment|.  The quotients are then converted
// once and the mean of squares h^2 sum q_i^2 / 8 is summed in float64 with
// the lane's float64 step size h (the squares of float32 values are exact in
// float64).  The value written per lane is what the controller compares with
// 1: the ratio r for the float64 policy, its square r^2 for the mixed one,
// whose accept test r^2 <= 1 decides as r <= 1 does (the square root is
// monotone) and whose step factor (next_step<false>) takes r^2 directly.
// Non-finite values become +inf.
template <class V>
__device__ __forceinline__ void error_ratio_v(const WStateV<V> &y, const AttemptV<V> &a,
                                              V hw, V rt, V at, RatioT<V> ratio[VT<V>::N],
                                              const double *hd) {
    using T = VT<V>;
    const WStateV<V> &yn = a.ynw;
    const V *err = a.err;
    const V yv[7] = {y.t, y.x, y.y, y.z, y.px, y.py, y.pz};
    const V nv[7] = {yn.t, yn.x, yn.y, yn.z, yn.px, yn.py, yn.pz};
    // Step increments without the exact parts: h sum b k for t x y z (the
    // first four carry the factor h in hn), dP for the momenta.
    const V inc[7] = {a.it, a.ix, a.iy, a.iz, a.dpx, a.dpy, a.dpz};
    const V hn = hw * T::set(kMixedNoise);
    // The floor of a position or momentum component follows the largest
    // increment of its 3-vector: a small component (p_y near zero on a
    // near-meridional orbit) is the difference of terms as large as the
    // others, and carries their rounding noise.
    V fl[7];
    if constexpr (sizeof(typename T::S) == 4) {
        const V fx = hn * T::max(T::abs(inc[1]), T::max(T::abs(inc[2]), T::abs(inc[3])));
        const V fp = T::set(kMixedNoise) *
                     T::max(T::abs(inc[4]), T::max(T::abs(inc[5]), T::abs(inc[6])));
        fl[0] = hn * T::abs(inc[0]);
        fl[1] = fl[2] = fl[3] = fx;
        fl[4] = fl[5] = fl[6] = fp;
    }
    V q[7];
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        V sc = T::fma(rt, T::max(T::abs(yv[i]), T::abs(nv[i])), at);
        if constexpr (sizeof(typename T::S) == 4) sc = T::max(sc, fl[i]);
        if constexpr (sizeof(V) == 8 && T::N == 1) {
            const V e = (hw * err[i]) / sc;
            q[i] = e * e;
        } else {
            // float lanes: q holds err / scale; the factor h goes on the sum.
            q[i] = err[i] * T::rcp(sc);
        }
    }
    if constexpr (sizeof(typename T::S) == 4 && sizeof(RatioT<V>) == 8) {
        // Components t x y z | p_t(=0) px py pz: r^2 = h^2 sum q^2 / 8 in
        // float64, the squares summed pairwise by fused multiply-adds.
#pragma unroll
        for (int l = 0; l < T::N; ++l) {
            double g[7];
#pragma unroll
            for (int i = 0; i < 7; ++i) g[i] = double(T::get(q[i], l));
            const double s01 = fma(g[1], g[1], g[0] * g[0]);
            const double s23 = fma(g[3], g[3], g[2] * g[2]);
            const double s456 = fma(g[6], g[6], fma(g[5], g[5], g[4] * g[4]));
            const double r2 = ((s01 + s23) + s456) * ((hd[l] * hd[l]) * 0.125);
            ratio[l] = isfinite(r2) ? r2 : __longlong_as_double(0x7ff0000000000000LL);
        }
    } else if constexpr (sizeof(typename T::S) == 4) {
        // Components t x y z | p_t(=0) px py pz: r^2 = h^2 sum q^2 / 8, the
        // squares summed pairwise by fused multiply-adds.
        const V s01 = T::fma(q[1], q[1], q[0] * q[0]);
        const V s23 = T::fma(q[3], q[3], q[2] * q[2]);
        const V s456 = T::fma(q[6], q[6], T::fma(q[5], q[5], q[4] * q[4]));
        const V sum = ((s01 + s23) + s456) * (hw * hw);
#pragma unroll
        for (int l = 0; l < T::N; ++l) {
            const float ms = T::get(sum, l) * 0.125f;
            ratio[l] = isfinite(ms) ? ms : __int_as_float(0x7f800000);
        }
    } else {
#pragma unroll
        for (int l = 0; l < T::N; ++l) {
            const double g[7] = {double(T::get(q[0], l)), double(T::get(q[1], l)),
                                 double(T::get(q[2], l)), double(T::get(q[3], l)),
                                 double(T::get(q[4], l)), double(T::get(q[5], l)),
                                 double(T::get(q[6], l))};
            // Components t x y z | p_t(=0) px py pz, NumPy's pairwise order.
            const double sum =
                ((g[0] + g[1]) + (g[2] + g[3])) + ((0.0 + g[4]) + (g[5] + g[6]));
            const double r = ::sqrt(sum * 0.125);
            ratio[l] = isfinite(r) ? r : __longlong_as_double(0x7ff0000000000000LL);
        }
    }
}

// Stage sums of one classical RK4 step (integrators.py:57-73) from the
// rounded state w with a step hw per lane: S = k1 + 2 k2 + 2 k3 + k4 for t,
// x, y, z, p_x, p_y, p_z, in the lane type.  The derivatives use the split
// form: dx = p + kappa, dt = -p_t + thl, dp = pdot.
template <class V>
__device__ __forceinline__ void rk4_sums(const KerrV<V> &K, const WStateV<V> &w, V hw,
                                         V S[7]) {
    using T = VT<V>;
    const V half = hw * T::set(0.5);
    const V zero = T::set(0.0);
    const StageV<V> d1 = rhs_v<V>(K, w.x, w.y, w.z, w.npt, w.px, w.py, w.pz, zero, zero, zero);
    const V k1x = w.px + d1.kx, k1y = w.py + d1.ky, k1z = w.pz + d1.kz;
    const V e2x = half * d1.px, e2y = half * d1.py, e2z = half * d1.pz;
    const StageV<V> d2 = rhs_v<V>(K, T::fma(half, k1x, w.x), T::fma(half, k1y, w.y),
                                  T::fma(half, k1z, w.z), w.npt, w.px + e2x, w.py + e2y,
                                  w.pz + e2z, e2x, e2y, e2z);
    const V k2x = w.px + d2.kx, k2y = w.py + d2.ky, k2z = w.pz + d2.kz;
    const V e3x = half * d2.px, e3y = half * d2.py, e3z = half * d2.pz;
    const StageV<V> d3 = rhs_v<V>(K, T::fma(half, k2x, w.x), T::fma(half, k2y, w.y),
                                  T::fma(half, k2z, w.z), w.npt, w.px + e3x, w.py + e3y,
                                  w.pz + e3z, e3x, e3y, e3z);
    const V k3x = w.px + d3.kx, k3y = w.py + d3.ky, k3z = w.pz + d3.kz;
    const V e4x = hw * d3.px, e4y = hw * d3.py, e4z = hw * d3.pz;
    const StageV<V> d4 = rhs_v<V>(K, T::fma(hw, k3x, w.x), T::fma(hw, k3y, w.y),
                                  T::fma(hw, k3z, w.z), w.npt, w.px + e4x, w.py + e4y,
                                  w.pz + e4z, e4x, e4y, e4z);
    const V k4x = w.px + d4.kx, k4y = w.py + d4.ky, k4z = w.pz + d4.kz;
    const V two = T::set(2.0);
    S[0] = T::set(6.0) * w.npt + (d1.thl + two * d2.thl + two * d3.thl + d4.thl);
    S[1] = k1x + two * k2x + two * k3x + k4x;
    S[2] = k1y + two * k2y + two * k3y + k4y;
    S[3] = k1z + two * k2z + two * k3z + k4z;
    S[4] = d1.px + two * d2.px + two * d3.px + d4.px;
    S[5] = d1.py + two * d2.py + two * d3.py + d4.py;
    S[6] = d1.pz + two * d2.pz + two * d3.pz + d4.pz;
}

// Lane l's float64 state after an RK4 step of size h with stage sums S.
template <class V>
__device__ __forceinline__ void rk4_update(RayState &y, const V S[7], int l, double h) {
    using T = VT<V>;
    const double h6 = h / 6.0;
    y.t += h6 * double(T::get(S[0], l));
    y.x += h6 * double(T::get(S[1], l));
    y.y += h6 * double(T::get(S[2], l));
    y.z += h6 * double(T::get(S[3], l));
    y.px += h6 * double(T::get(S[4], l));
    y.py += h6 * double(T::get(S[5], l));
    y.pz += h6 * double(T::get(S[6], l));
}

// One classical RK4 step of size h for a single ray (lane type with one
// lane): stage arithmetic in V, the state update in double.
template <class V>
__device__ __forceinline__ void rk4_advance(const KerrV<V> &K, RayState &y, double h) {
    using T = VT<V>;
    WStateV<V> w;
    put_work<V>(w, 0, y);
    V S[7];
    rk4_sums<V>(K, w, T::set(h), S);
    rk4_update<V>(y, S, 0, h);
}

// Projection onto the null constraint, float64.  The super-Hamiltonian
// H(x, p) = 1/2 (-p_t^2 + |p|^2) - H_ks lp^2 (geodesics.py:77-95) vanishes on
// null geodesics; integration error drifts it.  One Newton step along the
// spatial gradient dH/dp_i = p_i - 2 H_ks lp l_i (the coordinate velocity,
// geodesics.py:98-106) moves p back: p_i -= H v_i / |v|^2, leaving p_t, hence
// the energy, unchanged.  The residual after the step is O(H^2).  Not part of
// the reference, which never projects.
__device__ __forceinline__ void project_null(double m, double a, RayState &y) {
    Geometry g;
    geometry_full(m, a, y.x, y.y, y.z, false, g);
    const double lp = -y.pt + ((g.l[0] * y.px + g.l[1] * y.py) + g.l[2] * y.pz);
    const double ham = 0.5 * (-y.pt * y.pt + ((y.px * y.px + y.py * y.py) + y.pz * y.pz)) -
                       g.h * lp * lp;
    const double c = 2.0 * g.h * lp;
    const double vx = y.px - c * g.l[0], vy = y.py - c * g.l[1], vz = y.pz - c * g.l[2];
    const double v2 = (vx * vx + vy * vy) + vz * vz;
    if (!(v2 > 0.0)) return;
    const double s = ham / v2;
    y.px -= s * vx;
    y.py -= s * vy;
    y.pz -= s * vz;
}

// step_factor (integrators.py:120-124): clip(0.9 max(r,1e-16)^-0.2, 0.2, 5).
__device__ __forceinline__ double step_factor(double ratio) {
    const double f = 0.9 * ::pow(np_max(ratio, 1e-16), -0.2);
    return np_min(np_max(f, 0.2), 5.0);
}

// Step factor of the mixed policy from r^2, in float64:
// clip(0.9 (r^2)^-0.1, 0.2, 5), which equals step_factor(r).  y = x^-0.1 is
// one Newton-Raphson step on phi(y) = y^-10 - x, y <- y (1 + (1 - x y^10)/10),
// from the float32 seed exp2(-0.1 log2 x) (two MUFU instructions, relative
// error below 1e-6); the iteration converges quadratically with constant
// 11/2, so the result is within 1e-11 of x^-0.1 (relative).  x is clamped to
// [1e-12, 1e12] before the seed: outside [0.18^10, 4.5^10] the clip decides
// the factor, so the clamp changes no result.  r^2 is >= 0 or +inf, never NaN.
__device__ __forceinline__ double step_factor_r2(double r2) {
    const double x = fmin(fmax(r2, 1e-12), 1e12);
    const float xs = float(x);
    double y = double(ex2_approx(-0.1f * lg2_approx(xs)));
    const double y2 = y * y;
    const double y4 = y2 * y2;
    const double y10 = (y4 * y4) * y2;
    y = fma(y * 0.1, fma(-x, y10, 1.0), y);
    return fmin(fmax(0.9 * y, 0.2), 5.0);
}

// The controller's next step size (tracer.py:113-120): clip(h factor, 0,
// max_step) after accept and reject alike.  The float64 policy passes r and
// keeps the reference's forms.  The mixed policy passes r^2 (error_ratio_v):
// in float64 (RatioT = double) the factor is step_factor_r2; the float32
// controller kept for measurement takes 0.9 (r^2)^-0.1 through float32
// exp2/log2.  r^2 is >= 0 or +inf, never NaN, so the factor is finite and
// plain maxima and minima give the values NumPy's NaN-propagating ones
// would, with fewer instructions.
template <bool F64, typename R>
__device__ __forceinline__ double next_step(double h, R ratio, double max_step) {
    if constexpr (F64) {
        return np_min(np_max(h * step_factor(ratio), 0.0), max_step);
    } else if constexpr (sizeof(R) == 8) {
        return fmin(fmax(h * step_factor_r2(ratio), 0.0), max_step);
    } else {
        const float sf = fminf(fmaxf(ratio, 1e-32f), 3.0e38f);
        const double f = double(0.9f * ex2_approx(-0.1f * lg2_approx(sf)));
        return fmin(fmax(h * fmin(fmax(f, 0.2), 5.0), 0.0), max_step);
    }
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
