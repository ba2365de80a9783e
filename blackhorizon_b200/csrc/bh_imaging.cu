// bh_imaging.cu -- shading of traced rays into RGB pixels on the device.
//
// Restates imaging.py:27-91 (celestial_checkerboard, render_image): captured
// rays are black, escaped rays take the two-tone checker cell of their final
// propagation direction on the celestial sphere, rays at the step budget are
// dark red and every other status magenta.  Shading where the states already
// are leaves 3 bytes per pixel to copy to the host instead of the 76 of a
// state, status and step count.
//
// The direction is the spatial coordinate velocity dx/dlambda = p - 2 H lp l
// (geodesics.py:98-106), normalised.  Its combination is rounded as NumPy
// rounds it (no fused multiply-add), and the cell indices follow the
// reference's evaluation order, so a pixel can differ from the reference's
// only where the direction lies within an ulp of a cell boundary (the
// device's acos/atan2 may round differently there).
#include <cmath>
#include <cstdint>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

__device__ __forceinline__ void checker_rgb(double dx, double dy, double dz, int cells,
                                            uint8_t *o) {
    // imaging.py:38-50
    const double z = dz < -1.0 ? -1.0 : (dz > 1.0 ? 1.0 : dz);
    const double theta = ::acos(z);
    const double phi = ::atan2(dy, dx);
    const double c = (double)cells;
    const long long i_theta = (long long)::floor(__dmul_rn(__ddiv_rn(theta, M_PI), c));
    const long long i_phi = (long long)::floor(
        __dmul_rn(__dmul_rn(__ddiv_rn(__dadd_rn(phi, M_PI), 2.0 * M_PI), 2.0), c));
    const bool light = ((i_theta + i_phi) % 2) != 0;
    o[0] = light ? 104 : 24;
    o[1] = light ? 128 : 30;
    o[2] = light ? 178 : 52;
}

__global__ void checkerboard_kernel(const double *dirs, long long n, int cells, uint8_t *rgb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *d = dirs + 3 * i;
    checker_rgb(d[0], d[1], d[2], cells, rgb + 3 * i);
}

__global__ void render_kernel(double m, double a, const double *spin_of_ray,
                              const double *states, const int32_t *status, long long n,
                              int cells, uint8_t *rgb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t *o = rgb + 3 * i;
    const int st = status[i];
    if (st == BH_RAY_CAPTURED) {
        o[0] = o[1] = o[2] = 0;
    } else if (st == BH_RAY_ESCAPED) {
        // (t, x), (y, z), (p_t, p_x), (p_y, p_z)
        const double2 *p = reinterpret_cast<const double2 *>(states + 8 * i);
        const double2 tx = p[0], yz = p[1], tpx = p[2], pyz = p[3];
        const double x = tx.y, y = yz.x, z = yz.y;
        const double pt = tpx.x, px = tpx.y, py = pyz.x, pz = pyz.y;
        Geometry g;
        geometry_full(m, spin_of_ray ? spin_of_ray[i] : a, x, y, z, false, g);
        // geodesics.py:98-106 and imaging.py:79-82, in NumPy's rounding.
        const double lp = __dadd_rn(-pt, __dadd_rn(__dadd_rn(__dmul_rn(g.l[0], px),
                                                             __dmul_rn(g.l[1], py)),
                                                   __dmul_rn(g.l[2], pz)));
        const double two_h_lp = __dmul_rn(__dmul_rn(2.0, g.h), lp);
        const double vx = __dsub_rn(px, __dmul_rn(two_h_lp, g.l[0]));
        const double vy = __dsub_rn(py, __dmul_rn(two_h_lp, g.l[1]));
        const double vz = __dsub_rn(pz, __dmul_rn(two_h_lp, g.l[2]));
        double nrm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)),
                                          __dmul_rn(vz, vz)));
        if (nrm == 0.0) nrm = 1.0;
        checker_rgb(__ddiv_rn(vx, nrm), __ddiv_rn(vy, nrm), __ddiv_rn(vz, nrm), cells, o);
    } else if (st == BH_RAY_MAX_STEPS) {
        o[0] = 120; o[1] = 32; o[2] = 32;
    } else {
        o[0] = 200; o[1] = 0; o[2] = 200;
    }
}

static unsigned grid256(long long n) {
    const long long g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : g);
}

static int img_invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

static int img_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return BH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BH_ERR_CUDA;
}

}  // namespace bh

using namespace bh;

extern "C" int bh_celestial_checkerboard(const double *directions, int64_t n, int32_t cells,
                                         uint8_t *rgb, void *stream) {
    if (n < 0) return img_invalid("n must be >= 0");
    if (cells < 1) return img_invalid("cells must be >= 1");
    if (n == 0) return BH_OK;
    if (!directions || !rgb) return img_invalid("NULL pointer argument");
    checkerboard_kernel<<<grid256(n), 256, 0, (cudaStream_t)stream>>>(directions, n, cells,
                                                                      rgb);
    return img_launch("bh_celestial_checkerboard launch");
}

extern "C" int bh_render_image(double mass, double spin, const double *spin_of_ray,
                               const double *states, const int32_t *status, int64_t n,
                               int32_t cells, uint8_t *rgb, void *stream) {
    if (!(mass > 0.0) || (!spin_of_ray && !(std::fabs(spin) <= mass)))
        return img_invalid("Kerr bound violated or mass not positive");
    if (n < 0) return img_invalid("n must be >= 0");
    if (cells < 1) return img_invalid("cells must be >= 1");
    if (n == 0) return BH_OK;
    if (!states || !status || !rgb) return img_invalid("NULL pointer argument");
    if (reinterpret_cast<uintptr_t>(states) & 15u)
        return img_invalid("states must be 16-byte aligned");
    render_kernel<<<grid256(n), 256, 0, (cudaStream_t)stream>>>(mass, spin, spin_of_ray, states,
                                                                status, n, cells, rgb);
    return img_launch("bh_render_image launch");
}
