// bh_adjoint.cuh -- reverse-mode (vector-Jacobian) products of the geodesic
// right-hand side and of one Dormand-Prince 5(4) step with a frozen step
// size, for the discrete adjoint of the accepted step sequence.
//
// The reference differentiates nothing; it supplies the first derivatives
// grad H and grad l (kerr.py:157-191).  The adjoint needs the second
// derivatives of H and l, which are obtained here by reverse-mode
// differentiation of the RHS evaluated as the straight-line program below
// (geodesics.py:42-74 with kerr.py:118-193 folded in, the regrouped gradient
// contraction of rhs_v).  The clamps of kerr.py (_TINY) are inactive away
// from the ring singularity and are treated as the identity.  Reciprocals
// and square roots go through Math<W> (one MUFU instruction for float, the
// MUFU seed and two Newton steps for double), as in the forward stages.
//
// Work type W: double, or float for the mixed-precision adjoint; cotangents
// of the state are accumulated in double across steps either way.
#pragma once

#include "bh_device.cuh"

namespace bh {

// A state-shaped vector (t, x, y, z, p_t, p_x, p_y, p_z).
template <typename W>
struct Vec8 {
    W t, x, y, z, pt, px, py, pz;
};

template <typename W>
__device__ __forceinline__ Vec8<W> vzero() {
    return Vec8<W>{W(0), W(0), W(0), W(0), W(0), W(0), W(0), W(0)};
}

// Full derivative d(state)/d(lambda) at Y (geodesics.py:42-74).
template <typename W>
__device__ __forceinline__ Vec8<W> rhs_full(W m, W a, const Vec8<W> &Y) {
    const W x = Y.x, y = Y.y, z = Y.z, npt = -Y.pt, px = Y.px, py = Y.py, pz = Y.pz;
    const W a2 = a * a;
    const W z2 = z * z;
    const W a2z2 = a2 * z2;
    const W q = x * x + y * y + z2 - a2;
    const W s2 = q * q + W(4) * a2z2;
    const W is = Math<W>::rsqrt(s2);
    const W s = s2 * is;
    const W r2 = (q + s) * W(0.5);
    const W ir = Math<W>::rsqrt(r2);
    const W r = r2 * ir;
    const W w = r2 + a2;
    const W qd = r2 * r2 + a2z2;
    const W iq = Math<W>::rcp(qd), iw = Math<W>::rcp(w);
    const W r3 = r * r2;
    const W h = m * r3 * iq;
    const W lx = (r * x + a * y) * iw;
    const W ly = (r * y - a * x) * iw;
    const W lz = z * ir;
    const W lxy = lx * px + ly * py;
    const W lzpz = lz * pz;
    const W lp = lxy + lzpz + npt;
    const W thl = W(2) * h * lp;
    const W rs = r * is;
    const W r_x = x * rs, r_y = y * rs, r_z = z * w * ir * is;
    const W iq2 = iq * iq;
    const W lp2 = lp * lp;
    const W t3 = W(3) * a2 * z2 - r2 * r2;
    const W dh_dr = m * r2 * t3 * iq2;
    const W dh_dz = W(-2) * m * a2 * z * r3 * iq2;
    const W u = x * px + y * py;
    const W g1 = u - W(2) * r * lxy;
    const W g = g1 * iw - lzpz * ir;
    const W k = dh_dr * lp2 + thl * g;
    const W tw = thl * iw;
    Vec8<W> f;
    f.t = npt + thl;
    f.x = px - thl * lx;
    f.y = py - thl * ly;
    f.z = pz - thl * lz;
    f.pt = W(0);
    f.px = r_x * k + tw * (r * px - a * py);
    f.py = r_y * k + tw * (r * py + a * px);
    f.pz = r_z * k + dh_dz * lp2 + thl * pz * ir;
    return f;
}

// Cotangent of the RHS inputs: yb += (df/dY)^T fb and ab += (df/da)^T fb,
// the reverse sweep of rhs_full's program.
template <typename W>
__device__ __forceinline__ void rhs_vjp(W m, W a, const Vec8<W> &Y, const Vec8<W> &fb,
                                        Vec8<W> &yb, W &ab) {
    // ---- forward sweep (the intermediates of rhs_full)
    const W x = Y.x, y = Y.y, z = Y.z, npt = -Y.pt, px = Y.px, py = Y.py, pz = Y.pz;
    const W a2 = a * a;
    const W z2 = z * z;
    const W a2z2 = a2 * z2;
    const W q = x * x + y * y + z2 - a2;
    const W s2 = q * q + W(4) * a2z2;
    const W is = Math<W>::rsqrt(s2);
    const W s = s2 * is;
    const W r2 = (q + s) * W(0.5);
    const W ir = Math<W>::rsqrt(r2);
    const W r = r2 * ir;
    const W w = r2 + a2;
    const W qd = r2 * r2 + a2z2;
    const W iq = Math<W>::rcp(qd), iw = Math<W>::rcp(w);
    const W r3 = r * r2;
    const W h = m * r3 * iq;
    const W Lx = r * x + a * y, Ly = r * y - a * x;
    const W lx = Lx * iw, ly = Ly * iw, lz = z * ir;
    const W lxy = lx * px + ly * py;
    const W lzpz = lz * pz;
    const W lp = lxy + lzpz + npt;
    const W thl = W(2) * h * lp;
    const W rs = r * is;
    const W r_x = x * rs, r_y = y * rs, r_z = z * w * ir * is;
    const W iq2 = iq * iq;
    const W lp2 = lp * lp;
    const W t3 = W(3) * a2 * z2 - r2 * r2;
    const W dh_dr = m * r2 * t3 * iq2;
    const W c = W(-2) * m;
    const W dh_dz = c * a2 * z * r3 * iq2;
    const W u = x * px + y * py;
    const W g1 = u - W(2) * r * lxy;
    const W g = g1 * iw - lzpz * ir;
    const W k = dh_dr * lp2 + thl * g;
    const W tw = thl * iw;
    const W A = r * px - a * py;
    const W B = r * py + a * px;

    // ---- reverse sweep
    W x_b = 0, y_b = 0, z_b = 0, npt_b = 0, px_b = 0, py_b = 0, pz_b = 0, a_b = 0;
    W thl_b = 0, lx_b = 0, ly_b = 0, lz_b = 0, r_x_b = 0, r_y_b = 0, r_z_b = 0;
    W k_b = 0, tw_b = 0, A_b = 0, B_b = 0, dh_dz_b = 0, lp2_b = 0, ir_b = 0;
    // outputs
    npt_b += fb.t;
    thl_b += fb.t;
    px_b += fb.x; thl_b -= fb.x * lx; lx_b -= fb.x * thl;
    py_b += fb.y; thl_b -= fb.y * ly; ly_b -= fb.y * thl;
    pz_b += fb.z; thl_b -= fb.z * lz; lz_b -= fb.z * thl;
    r_x_b += fb.px * k; k_b += fb.px * r_x; tw_b += fb.px * A; A_b += fb.px * tw;
    r_y_b += fb.py * k; k_b += fb.py * r_y; tw_b += fb.py * B; B_b += fb.py * tw;
    r_z_b += fb.pz * k; k_b += fb.pz * r_z; dh_dz_b += fb.pz * lp2; lp2_b += fb.pz * dh_dz;
    thl_b += fb.pz * pz * ir; pz_b += fb.pz * thl * ir; ir_b += fb.pz * thl * pz;
    // B = r py + a px ; A = r px - a py
    W r_b = B_b * py + A_b * px;
    py_b += B_b * r - A_b * a;
    px_b += B_b * a + A_b * r;
    a_b += B_b * px - A_b * py;
    // tw = thl iw
    thl_b += tw_b * iw;
    W iw_b = tw_b * thl;
    // k = dh_dr lp2 + thl g
    const W dh_dr_b = k_b * lp2;
    lp2_b += k_b * dh_dr;
    thl_b += k_b * g;
    const W g_b = k_b * thl;
    // g = g1 iw - lzpz ir
    const W g1_b = g_b * iw;
    iw_b += g_b * g1;
    W lzpz_b = -g_b * ir;
    ir_b -= g_b * lzpz;
    // g1 = u - 2 r lxy
    const W u_b = g1_b;
    r_b -= W(2) * g1_b * lxy;
    W lxy_b = -W(2) * g1_b * r;
    // u = x px + y py
    x_b += u_b * px; px_b += u_b * x; y_b += u_b * py; py_b += u_b * y;
    // dh_dz = c a2 z r3 iq2
    W a2_b = dh_dz_b * c * z * r3 * iq2;
    z_b += dh_dz_b * c * a2 * r3 * iq2;
    W r3_b = dh_dz_b * c * a2 * z * iq2;
    W iq2_b = dh_dz_b * c * a2 * z * r3;
    // dh_dr = m r2 t3 iq2
    W r2_b = dh_dr_b * m * t3 * iq2;
    const W t3_b = dh_dr_b * m * r2 * iq2;
    iq2_b += dh_dr_b * m * r2 * t3;
    // t3 = 3 a2 z2 - r2^2
    a2_b += W(3) * t3_b * z2;
    W z2_b = W(3) * t3_b * a2;
    r2_b -= W(2) * t3_b * r2;
    // lp2 = lp^2 ; iq2 = iq^2
    W lp_b = W(2) * lp2_b * lp;
    W iq_b = W(2) * iq2_b * iq;
    // r_z = z w ir is ; r_y = y rs ; r_x = x rs ; rs = r is
    z_b += r_z_b * w * ir * is;
    W w_b = r_z_b * z * ir * is;
    ir_b += r_z_b * z * w * is;
    W is_b = r_z_b * z * w * ir;
    y_b += r_y_b * rs;
    W rs_b = r_y_b * y;
    x_b += r_x_b * rs;
    rs_b += r_x_b * x;
    r_b += rs_b * is;
    is_b += rs_b * r;
    // thl = 2 h lp
    W h_b = W(2) * thl_b * lp;
    lp_b += W(2) * thl_b * h;
    // lp = lxy + lzpz + npt
    lxy_b += lp_b;
    lzpz_b += lp_b;
    npt_b += lp_b;
    // lzpz = lz pz ; lxy = lx px + ly py
    lz_b += lzpz_b * pz;
    pz_b += lzpz_b * lz;
    lx_b += lxy_b * px; px_b += lxy_b * lx;
    ly_b += lxy_b * py; py_b += lxy_b * ly;
    // lz = z ir
    z_b += lz_b * ir;
    ir_b += lz_b * z;
    // ly = Ly iw ; lx = Lx iw
    const W Ly_b = ly_b * iw;
    iw_b += ly_b * Ly;
    const W Lx_b = lx_b * iw;
    iw_b += lx_b * Lx;
    r_b += Ly_b * y + Lx_b * x;
    y_b += Ly_b * r + Lx_b * a;
    x_b += Lx_b * r - Ly_b * a;
    a_b += Lx_b * y - Ly_b * x;
    // h = m r3 iq
    r3_b += h_b * m * iq;
    iq_b += h_b * m * r3;
    // r3 = r r2
    r_b += r3_b * r2;
    r2_b += r3_b * r;
    // reciprocals
    W s_b = -is_b * is * is;
    r_b -= ir_b * ir * ir;
    w_b -= iw_b * iw * iw;
    const W qd_b = -iq_b * iq * iq;
    // qd = r2^2 + a2z2 ; w = r2 + a2
    r2_b += W(2) * qd_b * r2;
    W a2z2_b = qd_b;
    r2_b += w_b;
    a2_b += w_b;
    // r = sqrt(r2)
    r2_b += r_b * W(0.5) * ir;
    // r2 = (q + s) / 2
    W q_b = r2_b * W(0.5);
    s_b += r2_b * W(0.5);
    // s = sqrt(q^2 + 4 a2z2)
    const W s2_b = s_b * W(0.5) * is;
    q_b += W(2) * s2_b * q;
    a2z2_b += W(4) * s2_b;
    // q = x^2 + y^2 + z2 - a2
    x_b += W(2) * q_b * x;
    y_b += W(2) * q_b * y;
    z2_b += q_b;
    a2_b -= q_b;
    // a2z2 = a2 z2 ; z2 = z^2 ; a2 = a^2
    a2_b += a2z2_b * z2;
    z2_b += a2z2_b * a2;
    z_b += W(2) * z2_b * z;
    a_b += W(2) * a2_b * a;

    yb.x += x_b; yb.y += y_b; yb.z += z_b;
    yb.pt -= npt_b;
    yb.px += px_b; yb.py += py_b; yb.pz += pz_b;
    ab += a_b;
}

namespace dpa {
// integrators.py:24-54 as arrays for the reverse sweep (b2 = 0).
__device__ constexpr double A[6][5] = {
    {0, 0, 0, 0, 0},
    {dp::A21, 0, 0, 0, 0},
    {dp::A31, dp::A32, 0, 0, 0},
    {dp::A41, dp::A42, dp::A43, 0, 0},
    {dp::A51, dp::A52, dp::A53, dp::A54, 0},
    {dp::A61, dp::A62, dp::A63, dp::A64, dp::A65}};
__device__ constexpr double B[6] = {dp::B1, 0.0, dp::B3, dp::B4, dp::B5, dp::B6};
}  // namespace dpa

template <typename W>
__device__ __forceinline__ Vec8<W> axpy(W s, const Vec8<W> &x, const Vec8<W> &y) {
    return Vec8<W>{y.t + s * x.t, y.x + s * x.x, y.y + s * x.y, y.z + s * x.z,
                   y.pt + s * x.pt, y.px + s * x.px, y.py + s * x.py, y.pz + s * x.pz};
}

// lam <- (d y_new / d y)^T lam for the fifth-order DP5 map with frozen step h
// (integrators.py:92-103 without the error estimate), and ga += (d y_new /
// d a)^T lam.  The stages are recomputed from y in W.
template <typename W>
__device__ __forceinline__ Vec8<W> to_work(const RayState &y) {
    return Vec8<W>{W(y.t), W(y.x), W(y.y), W(y.z), W(y.pt), W(y.px), W(y.py), W(y.pz)};
}

// y0: the state before the step, rounded to W.
template <typename W>
__device__ __forceinline__ void dp5_step_vjp(W m, W a, const Vec8<W> &y0, double h,
                                             Vec8<double> &lam, double &ga) {
    const W hw = W(h);
    Vec8<W> Y[6], K[6];
    Y[0] = y0;
    K[0] = rhs_full<W>(m, a, Y[0]);
    // The reverse loops are unrolled, which keeps the stage cotangents in
    // registers; float sweeps unroll the forward stage loop too, so that
    // the stage states and derivatives stay in registers as well.  The long
    // rays' sweeps are latency-bound and local-memory round trips sat on
    // their critical path: on the 256x256 frame the float sweep went from
    // 2.55 to 1.77 ms and the double one from 4.55 to 3.69 ms.  Double sweeps
    // keep the forward loop rolled: unrolled, they spilled 3 KB per thread
    // and ran 1.5x slower.
    constexpr int U = sizeof(W) == 4 ? 8 : 1;
    constexpr int UR = 8;
#pragma unroll U
    for (int i = 1; i < 6; ++i) {
        Vec8<W> acc = vzero<W>();
#pragma unroll U
        for (int j = 0; j < i; ++j) acc = axpy<W>(W(dpa::A[i][j]), K[j], acc);
        Y[i] = axpy<W>(hw, acc, Y[0]);
        K[i] = rhs_full<W>(m, a, Y[i]);
    }
    const Vec8<W> lw{W(lam.t), W(lam.x), W(lam.y), W(lam.z), W(lam.pt), W(lam.px),
                     W(lam.py), W(lam.pz)};
    Vec8<W> Kb[6];
#pragma unroll UR
    for (int j = 0; j < 6; ++j) {
        const W c = hw * W(dpa::B[j]);
        Kb[j] = Vec8<W>{c * lw.t, c * lw.x, c * lw.y, c * lw.z, c * lw.pt, c * lw.px,
                        c * lw.py, c * lw.pz};
    }
#pragma unroll UR
    for (int i = 5; i >= 0; --i) {
        Vec8<W> Yb = vzero<W>();
        W ab = W(0);
        rhs_vjp<W>(m, a, Y[i], Kb[i], Yb, ab);
        ga += double(ab);
        lam.t += double(Yb.t); lam.x += double(Yb.x); lam.y += double(Yb.y);
        lam.z += double(Yb.z); lam.pt += double(Yb.pt); lam.px += double(Yb.px);
        lam.py += double(Yb.py); lam.pz += double(Yb.pz);
#pragma unroll UR
        for (int j = 0; j < i; ++j) Kb[j] = axpy<W>(hw * W(dpa::A[i][j]), Yb, Kb[j]);
    }
}

}  // namespace bh
