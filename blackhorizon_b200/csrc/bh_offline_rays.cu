// bh_offline_rays.cu -- initial states of an offline frame on the device.
//
// One thread per subpixel ray builds its (n, 8) state in place of the
// host-side pipeline of render_hdr (render.py:555-599):
// - the supersampled pinhole grid (render.py:103-145);
// - a pinhole camera rotates the grid by its (forward, right, up) basis
//   (render.py:148-161) and takes the past-directed null momentum at the
//   camera (geodesics.py:109-170);
// - a tetrad camera takes the momentum e0 - sum n_i e_i of the observer's
//   tetrad, negated and lowered (frames.py:63-77, 182-218).
// Sums and products keep NumPy's order and rounding (no contraction), so
// the directions equal the reference's to the last bit.
#include <cmath>
#include <cstdint>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

__global__ void offline_rays_kernel(double m, double a, const bh_offline_camera cam,
                                    long long n, double *states) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long ss = cam.supersample, ss2 = ss * ss;
    const long long p = i / ss2, k = i - p * ss2;
    const long long row = p / cam.width, col = p - row * cam.width;
    const long long sr = k / ss, sc = k - sr * ss;
    // render.py:117-125: subpixel centres (s + 0.5) / ss, u, v in [-1, 1].
    const double dss = (double)ss;
    const double px = __dadd_rn((double)col, __ddiv_rn(__dadd_rn((double)sc, 0.5), dss));
    const double py = __dadd_rn((double)row, __ddiv_rn(__dadd_rn((double)sr, 0.5), dss));
    const double u = __dsub_rn(__dmul_rn(__ddiv_rn(px, (double)cam.width), 2.0), 1.0);
    const double v = __dsub_rn(1.0, __dmul_rn(__ddiv_rn(py, (double)cam.height), 2.0));
    // render.py:134-145: (1, u tan, v tan / aspect), normalised.
    const double l1 = __dmul_rn(u, cam.tan_half), l2 = __dmul_rn(v, cam.tan_half_aspect);
    const double nrm = ::sqrt(__dadd_rn(__dadd_rn(1.0, __dmul_rn(l1, l1)), __dmul_rn(l2, l2)));
    const double d0 = __ddiv_rn(1.0, nrm), d1 = __ddiv_rn(l1, nrm), d2 = __ddiv_rn(l2, nrm);
    double mom[4];
    if (!cam.use_tetrad) {
        // render.py:148-161: local coefficients on (forward, right, up).
        double dir[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            dir[c] = __dadd_rn(__dadd_rn(__dmul_rn(d0, cam.basis[0][c]),
                                         __dmul_rn(d1, cam.basis[1][c])),
                               __dmul_rn(d2, cam.basis[2][c]));
        null_momentum(m, a, cam.position, dir, true, true, mom);
    } else {
        // frames.py:212-218 and 63-77: v = -(e0 - (n1 e1 + n2 e2 + n3 e3)),
        // lowered with g = eta + 2 H l l.
        double vec[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double spatial = __dadd_rn(__dadd_rn(__dmul_rn(d0, cam.tetrad[1][c]),
                                                       __dmul_rn(d1, cam.tetrad[2][c])),
                                             __dmul_rn(d2, cam.tetrad[3][c]));
            vec[c] = -__dsub_rn(cam.tetrad[0][c], spatial);
        }
        Geometry g;
        geometry_full(m, a, cam.position[0], cam.position[1], cam.position[2], false, g);
        const double l_v = __dadd_rn(vec[0], __dadd_rn(__dadd_rn(__dmul_rn(g.l[0], vec[1]),
                                                                 __dmul_rn(g.l[1], vec[2])),
                                                       __dmul_rn(g.l[2], vec[3])));
        const double two_h_lv = __dmul_rn(__dmul_rn(2.0, g.h), l_v);
        mom[0] = __dadd_rn(-vec[0], two_h_lv);
#pragma unroll
        for (int c = 0; c < 3; ++c) mom[1 + c] = __dadd_rn(vec[1 + c], __dmul_rn(two_h_lv, g.l[c]));
    }
    double *s = states + 8 * i;
    s[0] = 0.0;
    s[1] = cam.position[0];
    s[2] = cam.position[1];
    s[3] = cam.position[2];
    s[4] = mom[0];
    s[5] = mom[1];
    s[6] = mom[2];
    s[7] = mom[3];
}

}  // namespace bh

using namespace bh;

extern "C" int bh_offline_camera_rays(double mass, double spin, const bh_offline_camera *camera,
                                      double *states, void *stream) {
    if (!camera) {
        set_error("camera is NULL");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const bh_offline_camera &c = *camera;
    if (!(mass > 0.0) || !(std::fabs(spin) <= mass) || c.width < 0 || c.height < 0 ||
        c.supersample < 1 || (c.use_tetrad != 0 && c.use_tetrad != 1)) {
        set_error("invalid spacetime, frame size, supersample or camera mode");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const long long n = (long long)c.width * c.height * c.supersample * c.supersample;
    if (n == 0) return BH_OK;
    if (!states) {
        set_error("states is NULL");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const long long blocks = (n + 255) / 256;
    offline_rays_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(mass, spin, c, n,
                                                                            states);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("bh_offline_camera_rays launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
