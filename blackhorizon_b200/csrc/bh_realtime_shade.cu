// bh_realtime_shade.cu -- the real-time viewer's pixel colours on the device.
//
// Restates the shading of the fragment shader realtime/shaders/
// kerr_tracer.frag:205-420 on the outputs of the real-time tracer
// (bh_trace_realtime): one thread per pixel, float32 like the shader.
// - Disk hits: Novikov-Thorne emission with the circular-orbit redshift, the
//   temperature and blackbody tables sampled as the viewer's textures are
//   (linear filtering between texel centres, repeat wrapping), the detail
//   pattern and the Reinhard curve c / (1 + c).
// - Escaped rays: the two-tone checkerboard or the procedural starfield with
//   its coordinate grid, sampled by the asymptotic direction p - 2 H lp l;
//   interior cameras shift the sky by g = B / E (intensity g^4, capped at
//   4e4, and a chromatic slide).
// - Rays ended on the terminal surface glow with the blue-sheet radiance when
//   it is non-zero; every other ray is black.
// - The whiteout mixes the colour toward (0.90, 0.95, 1.0); the result is
//   stored as 8-bit unsigned normalised values, row 0 at the top.
#include <cmath>
#include <cstdint>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

struct GeoF {
    float r, h, l[3];
};

// kerr_tracer.frag:96-114 (evaluate_geometry without gradients), float32.
__device__ __forceinline__ GeoF geometry_f(float m, float a, float x, float y, float z) {
    GeoF g;
    const float a2 = a * a;
    const float rho2 = x * x + y * y + z * z;
    const float q = rho2 - a2;
    const float s = fmaxf(sqrtf(q * q + 4.0f * a2 * z * z), 1e-12f);
    const float r2 = fmaxf(0.5f * (q + s), 1e-12f);
    const float r = sqrtf(r2);
    const float qd = fmaxf(r2 * r2 + a2 * z * z, 1e-12f);
    g.r = r;
    g.h = m * r * r2 / qd;
    const float inv_r2a2 = 1.0f / (r2 + a2);
    const float inv_r = 1.0f / r;
    g.l[0] = (r * x + a * y) * inv_r2a2;
    g.l[1] = (r * y - a * x) * inv_r2a2;
    g.l[2] = z * inv_r;
    return g;
}

// A linear-filtered read of a 1-D texture of n texels at coordinate s in
// [0, 1] with repeat wrapping (the viewer's lookup textures): texel centres
// at (i + 1/2) / n.  stride/col select one channel of an (n, stride) table.
__device__ __forceinline__ float texture_1d(const float *table, int n, int stride, int col,
                                            float s) {
    const float u = s * (float)n - 0.5f;
    const float f = floorf(u);
    const float alpha = u - f;
    int i0 = (int)f % n;
    if (i0 < 0) i0 += n;
    const int i1 = (i0 + 1) % n;
    return (1.0f - alpha) * table[i0 * stride + col] + alpha * table[i1 * stride + col];
}

__device__ __forceinline__ float fract_f(float x) { return x - floorf(x); }

__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x) {
    const float t = fminf(fmaxf((x - e0) / (e1 - e0), 0.0f), 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

// kerr_tracer.frag:243-247
__device__ __forceinline__ float hash13(float x, float y, float z) {
    x = fract_f(x * 0.1031f);
    y = fract_f(y * 0.1031f);
    z = fract_f(z * 0.1031f);
    const float d = x * (z + 31.32f) + y * (y + 31.32f) + z * (x + 31.32f);
    x += d;
    y += d;
    z += d;
    return fract_f((x + y) * z);
}

// kerr_tracer.frag:249-268
__device__ void background_color(int mode, float dx, float dy, float dz, float c[3]) {
    const float theta = acosf(fminf(fmaxf(dz, -1.0f), 1.0f));
    const float phi = atan2f(dy, dx);
    if (mode == 0) {
        const float cells = 12.0f;
        const float it = floorf(theta / 3.14159265f * cells);
        const float ip = floorf((phi + 3.14159265f) / 6.2831853f * 2.0f * cells);
        const float sum = it + ip;  // GLSL mod(x, 2) = x - 2 floor(x / 2)
        const bool light = sum - 2.0f * floorf(sum * 0.5f) >= 1.0f;
        c[0] = light ? 0.408f : 0.094f;
        c[1] = light ? 0.502f : 0.118f;
        c[2] = light ? 0.698f : 0.204f;
        return;
    }
    const float star = powf(hash13(floorf(dx * 220.0f), floorf(dy * 220.0f), floorf(dz * 220.0f)),
                            60.0f);
    const float grid_t =
        smoothstep_f(0.006f, 0.0f, fabsf(fract_f(theta / 0.19635f) - 0.5f) * 0.19635f);
    const float grid_p =
        smoothstep_f(0.006f, 0.0f, fabsf(fract_f(phi / 0.19635f) - 0.5f) * 0.19635f);
    const float g = fmaxf(grid_t, grid_p);
    c[0] = 0.012f + star + 0.02f * g;
    c[1] = 0.014f + star + 0.03f * g;
    c[2] = 0.028f + star + 0.05f * g;
}

// kerr_tracer.frag:205-241, with p_t the ray's conserved energy.
__device__ void disk_emission(const RealtimeShadeArgs &s, float px_t, const float pos[3],
                              const float p[3], float c[3]) {
    const GeoF g = geometry_f(s.mass, s.spin, pos[0], pos[1], pos[2]);
    const float omega = 1.0f / (powf(g.r, 1.5f) + s.spin);
    const float v[3] = {-omega * pos[1], omega * pos[0], 0.0f};
    const float l_dot_v = 1.0f + (g.l[0] * v[0] + g.l[1] * v[1] + g.l[2] * v[2]);
    const float norm2 = -1.0f + (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) +
                        2.0f * g.h * l_dot_v * l_dot_v;
    const float u_t = rsqrtf(fmaxf(-norm2, 1e-9f));
    const float nu = u_t * (px_t + (p[0] * v[0] + p[1] * v[1] + p[2] * v[2]));
    const float shift = s.observer_lapse / fmaxf(nu, 1e-6f);
    const float lut_u =
        fminf(fmaxf((g.r - s.disk_inner) / (s.disk_outer - s.disk_inner), 0.0f), 1.0f);
    const float t_norm = texture_1d(s.temperature, s.temperature_size, 1, 0, lut_u);
    const float t_obs = shift * t_norm * s.disk_temperature;
    const float bb_u = fminf(
        fmaxf((logf(fmaxf(t_obs, 1.0f)) - s.bb_log_min) / (s.bb_log_max - s.bb_log_min), 0.0f),
        1.0f);
    const float phi = atan2f(pos[1], pos[0]);
    const float detail = 1.0f + s.disk_detail * (0.18f * sinf(9.0f * phi + 2.2f * g.r) +
                                                 0.12f * sinf(23.0f * phi - 5.0f * g.r) +
                                                 0.15f * sinf(3.5f * (g.r - s.disk_inner)));
    const float brightness = s.exposure * powf(t_obs / 6500.0f, 4.0f) * fmaxf(detail, 0.2f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float col = texture_1d(s.blackbody, s.blackbody_size, 3, k, bb_u) * brightness;
        c[k] = col / (1.0f + col);
    }
}

__device__ __forceinline__ uint8_t unorm8(float x) {
    return (uint8_t)__float2int_rn(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f);
}

__global__ void realtime_shade_kernel(const RealtimeShadeArgs s) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.pixels) return;
    const int st = s.status[i];
    float c[3] = {0.0f, 0.0f, 0.0f};
    if (st == BH_RAY_DISK) {
        const double *hp = s.hit_pos + 3 * i, *hm = s.hit_mom + 4 * i;
        const float pos[3] = {(float)hp[0], (float)hp[1], (float)hp[2]};
        const float p[3] = {(float)hm[1], (float)hm[2], (float)hm[3]};
        disk_emission(s, (float)hm[0], pos, p, c);
    } else if (st == BH_RAY_ESCAPED) {
        const double *y = s.states + 8 * i;
        const float pos[3] = {(float)y[1], (float)y[2], (float)y[3]};
        const float pt = (float)y[4];
        const float p[3] = {(float)y[5], (float)y[6], (float)y[7]};
        const GeoF g = geometry_f(s.mass, s.spin, pos[0], pos[1], pos[2]);
        const float lp = -pt + (g.l[0] * p[0] + g.l[1] * p[1] + g.l[2] * p[2]);
        float d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) d[k] = p[k] - 2.0f * g.h * lp * g.l[k];
        const float inv = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        background_color(s.background, d[0] * inv, d[1] * inv, d[2] * inv, c);
        if (s.sky_amplification > 0.0f) {
            // kerr_tracer.frag:384-400
            const float g_sky = s.sky_amplification / fmaxf(pt, 1e-6f);
            const float gain = fminf(fmaxf(g_sky * g_sky * g_sky * g_sky, 0.0f), 4.0e4f);
            const float slide = fminf(fmaxf(0.35f * logf(fmaxf(g_sky, 1e-6f)), -0.6f), 0.6f);
            const float t[3] = {1.0f - slide, 1.0f, 1.0f + slide};
            const float tn = rsqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) * 1.732f;
#pragma unroll
            for (int k = 0; k < 3; ++k) c[k] = c[k] * gain * (t[k] * tn);
        }
    } else if ((st == BH_RAY_CAPTURED || st == BH_RAY_TERMINATED) && s.sheet_radiance > 0.0f) {
        c[0] = s.sheet_radiance * 0.62f;
        c[1] = s.sheet_radiance * 0.78f;
        c[2] = s.sheet_radiance * 1.0f;
    }
    if (s.whiteout > 0.0f) {
        const float w[3] = {0.90f, 0.95f, 1.0f};
#pragma unroll
        for (int k = 0; k < 3; ++k) c[k] = c[k] * (1.0f - s.whiteout) + w[k] * s.whiteout;
    }
    uint8_t *o = s.rgb + 3 * i;
    o[0] = unorm8(c[0]);
    o[1] = unorm8(c[1]);
    o[2] = unorm8(c[2]);
}

}  // namespace bh

using namespace bh;

extern "C" int bh_realtime_shade(const bh_realtime_shading *shading, const int32_t *status,
                                 const double *states, const double *hit_positions,
                                 const double *hit_momenta, int64_t width, int64_t height,
                                 const float *temperature_table, const float *blackbody_table,
                                 uint8_t *rgb, void *stream) {
    if (!shading) {
        set_error("shading is NULL");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const bh_realtime_shading &c = *shading;
    if (!(c.mass > 0.0) || !(std::fabs(c.spin) <= c.mass) || width < 0 || height < 0 ||
        (c.background != 0 && c.background != 1) || c.temperature_size < 2 ||
        c.blackbody_size < 2 || !(c.bb_log_max > c.bb_log_min) ||
        !(c.disk_outer > c.disk_inner)) {
        set_error("invalid spacetime, frame size, background mode, tables or disk radii");
        return BH_ERR_INVALID_ARGUMENT;
    }
    const long long pixels = (long long)width * height;
    if (pixels == 0) return BH_OK;
    if (!status || !states || !hit_positions || !hit_momenta || !temperature_table ||
        !blackbody_table || !rgb) {
        set_error("NULL pointer argument");
        return BH_ERR_INVALID_ARGUMENT;
    }
    RealtimeShadeArgs a;
    a.mass = (float)c.mass;
    a.spin = (float)c.spin;
    a.disk_inner = (float)c.disk_inner;
    a.disk_outer = (float)c.disk_outer;
    a.disk_temperature = (float)c.disk_temperature;
    a.disk_detail = (float)c.disk_detail;
    a.exposure = (float)c.exposure;
    a.observer_lapse = (float)c.observer_lapse;
    a.bb_log_min = (float)c.bb_log_min;
    a.bb_log_max = (float)c.bb_log_max;
    a.sky_amplification = (float)c.sky_amplification;
    a.sheet_radiance = (float)c.sheet_radiance;
    a.whiteout = (float)c.whiteout;
    a.background = c.background;
    a.temperature_size = c.temperature_size;
    a.blackbody_size = c.blackbody_size;
    a.pixels = pixels;
    a.status = status;
    a.states = states;
    a.hit_pos = hit_positions;
    a.hit_mom = hit_momenta;
    a.temperature = temperature_table;
    a.blackbody = blackbody_table;
    a.rgb = rgb;
    const long long blocks = (pixels + 255) / 256;
    realtime_shade_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("bh_realtime_shade launch: %s", cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
