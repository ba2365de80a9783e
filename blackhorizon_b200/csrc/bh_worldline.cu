// bh_worldline.cu -- the plunging camera's worldline, on the host.
//
// offline/infall.py:38-153: the doomed observer of the plunge renderer
// follows one timelike geodesic, integrated once per video and sampled every
// step.  It is a single sequential trajectory, so it runs on the host in
// float64 with the Kerr-Schild geometry shared with the device code
// (geometry_full); the camera rays of every frame then go to the device.
// - radial_momentum: the E-parameterised radial infaller p = (-E, w l),
//   the future-directed inward root of the timelike mass shell;
// - the worldline: classical RK4 (integrators.py:57-73) of Hamilton's
//   equations (geodesics.py:42-74) with the proper-time step
//   min(step, max(0.04 r^1.5, 1e-6)); after each step the momentum is
//   rescaled onto H = -1/2 when it drifts by more than 1e-9; the
//   integration stops on a non-finite state, at H >= -1e-6 (the chart's
//   edge), at r <= stop_radius or after 2,000,000 steps.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

// geodesics.py:42-74 for one state (t, x, y, z, p_t, p_x, p_y, p_z).
static void kerr_rhs(double m, double a, const double y[8], double d[8]) {
    Geometry g;
    geometry_full(m, a, y[1], y[2], y[3], true, g);
    const double lp = -y[4] + ((g.l[0] * y[5] + g.l[1] * y[6]) + g.l[2] * y[7]);
    const double thl = 2.0 * g.h * lp;
    d[0] = -y[4] + thl;
    for (int i = 0; i < 3; ++i) d[1 + i] = y[5 + i] - thl * g.l[i];
    d[4] = 0.0;
    for (int i = 0; i < 3; ++i) {
        const double c = (g.grad_l[i][0] * y[5] + g.grad_l[i][1] * y[6]) + g.grad_l[i][2] * y[7];
        d[5 + i] = g.grad_h[i] * (lp * lp) + thl * c;
    }
}

// geodesics.py:77-85
static double kerr_hamiltonian(double m, double a, const double y[8]) {
    Geometry g;
    geometry_full(m, a, y[1], y[2], y[3], false, g);
    const double lp = -y[4] + ((g.l[0] * y[5] + g.l[1] * y[6]) + g.l[2] * y[7]);
    const double eta = 0.5 * (-y[4] * y[4] + ((y[5] * y[5] + y[6] * y[6]) + y[7] * y[7]));
    return eta - g.h * lp * lp;
}

// integrators.py:57-73
static void rk4(double m, double a, double y[8], double h) {
    double k1[8], k2[8], k3[8], k4[8], t[8];
    kerr_rhs(m, a, y, k1);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + 0.5 * h * k1[i];
    kerr_rhs(m, a, t, k2);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + 0.5 * h * k2[i];
    kerr_rhs(m, a, t, k3);
    for (int i = 0; i < 8; ++i) t[i] = y[i] + h * k3[i];
    kerr_rhs(m, a, t, k4);
    for (int i = 0; i < 8; ++i)
        y[i] = y[i] + (h / 6.0) * (((k1[i] + 2.0 * k2[i]) + 2.0 * k3[i]) + k4[i]);
}

static double ks_radius_host(double m, double a, const double y[8]) {
    Geometry g;
    geometry_full(m, a, y[1], y[2], y[3], false, g);
    return g.r;
}

// infall.py:38-91: the covariant momentum (p_t, p_x, p_y, p_z); false if no
// future-directed inward root exists at the position.
static bool radial_momentum(double m, double a, const double pos[3], double energy,
                            double p[4]) {
    Geometry g;
    geometry_full(m, a, pos[0], pos[1], pos[2], false, g);
    const double p_t = -energy;
    // (1 - 2H) w^2 + 4 H p_t w + 1 - (1 + 2H) p_t^2 = 0, roots descending.
    const double A = 1.0 - 2.0 * g.h, B = 4.0 * g.h * p_t;
    const double C = 1.0 - (1.0 + 2.0 * g.h) * p_t * p_t;
    double roots[2];
    int nroots = 0;
    if (A == 0.0) {
        if (B != 0.0) roots[nroots++] = -C / B;
    } else {
        const double disc = B * B - 4.0 * A * C;
        if (disc >= 0.0) {
            const double sq = std::sqrt(disc);
            const double q = -0.5 * (B + (B >= 0.0 ? sq : -sq));
            const double r1 = q != 0.0 ? q / A : 0.0;
            const double r2 = q != 0.0 ? C / q : 0.0;
            roots[0] = r1 > r2 ? r1 : r2;
            roots[1] = r1 > r2 ? r2 : r1;
            nroots = 2;
        } else {
            roots[0] = roots[1] = -B / (2.0 * A);  // the real part of a complex pair
            nroots = 2;
        }
    }
    const double rpos = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    for (int k = 0; k < nroots; ++k) {
        const double w = roots[k];
        const double y[8] = {0.0, pos[0], pos[1], pos[2], p_t, w * g.l[0], w * g.l[1],
                             w * g.l[2]};
        if (std::fabs(kerr_hamiltonian(m, a, y) + 0.5) > 1e-9) continue;
        // frames.py:80-99: u = g^-1 p with g^-1 = eta - 2 H l^ l^.
        const double l_up = -p_t + ((g.l[0] * y[5] + g.l[1] * y[6]) + g.l[2] * y[7]);
        const double u_t = -p_t + 2.0 * g.h * l_up;
        double radial = 0.0;
        for (int i = 0; i < 3; ++i) radial += (y[5 + i] - 2.0 * g.h * l_up * g.l[i]) * pos[i];
        radial /= rpos;
        if (u_t > 0.0 && radial < 0.0) {
            p[0] = p_t;
            p[1] = y[5];
            p[2] = y[6];
            p[3] = y[7];
            return true;
        }
    }
    return false;
}

}  // namespace bh

using namespace bh;

extern "C" int bh_radial_momentum(double mass, double spin, const double *position,
                                  double energy, double *momentum) {
    if (!(mass > 0.0) || !(std::fabs(spin) <= mass) || !position || !momentum ||
        !(energy >= 0.0)) {
        set_error("invalid spacetime, energy (>= 0) or NULL pointer");
        return BH_ERR_INVALID_ARGUMENT;
    }
    if (!radial_momentum(mass, spin, position, energy, momentum)) {
        set_error("no future-directed infalling root; for E = 0 start inside the horizon");
        return BH_ERR_INVALID_ARGUMENT;
    }
    return BH_OK;
}

extern "C" int64_t bh_plunge_worldline(double mass, double spin, double start_radius,
                                       double energy, double stop_radius, double step,
                                       int64_t capacity, double *taus, double *states) {
    if (!(mass > 0.0) || !(std::fabs(spin) <= mass) || !(start_radius > 0.0) ||
        !(step > 0.0) || capacity < 0 || (capacity > 0 && (!taus || !states))) {
        set_error("invalid spacetime, start radius, step or output buffers");
        return -1;
    }
    const double pos[3] = {start_radius, 0.0, 0.0};
    double p[4];
    if (!radial_momentum(mass, spin, pos, energy, p)) {
        set_error("no future-directed infalling root; for E = 0 start inside the horizon");
        return -1;
    }
    double y[8] = {0.0, pos[0], pos[1], pos[2], p[0], p[1], p[2], p[3]};
    double tau = 0.0;
    int64_t count = 0;
    auto record = [&](double t) {
        if (count < capacity) {
            taus[count] = t;
            std::memcpy(states + 8 * count, y, sizeof(y));
        }
        ++count;
    };
    record(0.0);
    for (long long it = 0; it < 2000000; ++it) {
        const double r = ks_radius_host(mass, spin, y);
        const double h = std::fmin(step, std::fmax(0.04 * std::pow(r, 1.5), 1e-6));
        rk4(mass, spin, y, h);
        const double value = kerr_hamiltonian(mass, spin, y);
        bool finite = std::isfinite(value);
        for (int i = 0; i < 8; ++i) finite = finite && std::isfinite(y[i]);
        if (!finite || value >= -1e-6) break;
        if (std::fabs(value + 0.5) > 1e-9) {
            const double s = std::sqrt(0.5 / (-value));
            for (int i = 4; i < 8; ++i) y[i] *= s;
        }
        tau += h;
        record(tau);
        if (ks_radius_host(mass, spin, y) <= stop_radius) break;
    }
    return count;
}
