// bh_emission.cu -- the offline renderer's emission and development stages
// on the device.
//
// Radiance (render.py:352-484 and the shading part of render_hdr,
// render.py:630-680): escaped rays sample a hashed HDR starfield by their
// asymptotic direction, disk hits take a redshifted Novikov-Thorne blackbody
// (temperature and chromaticity lookup tables built on the host), rays that
// ended on the blue sheet glow, everything else is black; the supersamples
// of a pixel are averaged into a float32 HDR image.  One thread per pixel.
// Arithmetic is float64 with NumPy's operation order (no contraction), so a
// pixel differs from the reference's only by the last bits of the device's
// sin/exp/log/atan2/acos, except where a direction lies within an ulp of a
// starfield cell boundary.
//
// Development (offline/post.py:15-106): exposure, bloom (bright pass and a
// separable Gaussian blur with edge padding), the ACES filmic curve and sRGB
// encoding to 8 bits, in float32 as NumPy computes it: every blur tap
// accumulates w * x in float64 into a float32 pixel, in tap order.
#include <cmath>
#include <cstdint>

#include "bh_device.cuh"
#include "bh_internal.h"

namespace bh {

// ------------------------------------------------------------- radiance

// render.py:368-370: fract(sin(a 127.1 + b 311.7 + salt 74.7) 43758.5453).
__device__ __forceinline__ double hash01(double a, double b, double salt74) {
    const double arg = __dadd_rn(__dadd_rn(__dmul_rn(a, 127.1), __dmul_rn(b, 311.7)), salt74);
    const double v = __dmul_rn(::sin(arg), 43758.5453);
    return __dsub_rn(v, ::floor(v));
}

__device__ __forceinline__ double clip(double x, double lo, double hi) {
    return np_min(np_max(x, lo), hi);
}

// render.py:352-419 (_starfield_hdr) for one unit direction; shift > 0 is
// the per-ray frequency ratio of a tetrad camera, shift <= 0 none.
__device__ void starfield(double dx, double dy, double dz, double shift, double c[3]) {
    const double phi = ::atan2(dy, dx);
    const double theta = ::acos(clip(dz, -1.0, 1.0));
    c[0] = c[1] = c[2] = 0.0;
    const bool shifted = shift > 0.0;
    double s4 = 0.0, lnshift = 0.0;
    if (shifted) {
        s4 = ::pow(shift, 4.0);
        lnshift = ::log(np_max(shift, 1e-6));
    }
    // salt * 74.7 as Python rounds it, salts 1..5
    const double salt[5] = {74.7, 2.0 * 74.7, 3.0 * 74.7, 4.0 * 74.7, 5.0 * 74.7};
#pragma unroll
    for (int layer = 0; layer < 2; ++layer) {
        const double cells = layer == 0 ? 160.0 : 420.0;
        const double density = layer == 0 ? 0.10 : 0.05;
        const double brightness = layer == 0 ? 3.0 : 0.9;
        const double cu = __dmul_rn(__ddiv_rn(phi, 2.0 * M_PI), cells);
        const double cv = __dmul_rn(__ddiv_rn(theta, M_PI), cells);
        const double iu = ::floor(cu), iv = ::floor(cv);
        if (!(hash01(iu, iv, salt[0]) < density)) continue;  // present
        const double su = __dadd_rn(__dadd_rn(iu, 0.15), __dmul_rn(0.7, hash01(iu, iv, salt[1])));
        const double sv = __dadd_rn(__dadd_rn(iv, 0.15), __dmul_rn(0.7, hash01(iu, iv, salt[2])));
        const double du = __dsub_rn(cu, su), dv = __dsub_rn(cv, sv);
        const double dist2 = __dadd_rn(__dmul_rn(du, du), __dmul_rn(dv, dv));
        const double magnitude = hash01(iu, iv, salt[3]);
        double amplitude = __dmul_rn(brightness, __dadd_rn(0.15, ::pow(magnitude, 4.0)));
        const double point = ::exp(__ddiv_rn(-dist2, 0.006));
        double warmth = hash01(iu, iv, salt[4]);
        if (shifted) {
            amplitude = __dmul_rn(amplitude, s4);
            warmth = clip(__dsub_rn(warmth, __dmul_rn(0.6, lnshift)), 0.0, 1.0);
        }
        const double tint[3] = {__dadd_rn(0.75, __dmul_rn(0.35, warmth)),
                                __dadd_rn(0.85, __dmul_rn(0.10, warmth)),
                                __dsub_rn(1.05, __dmul_rn(0.35, warmth))};
        const double w = __dmul_rn(amplitude, point);
#pragma unroll
        for (int k = 0; k < 3; ++k) c[k] = __dadd_rn(c[k], __dmul_rn(w, tint[k]));
    }
    const double zz = __ddiv_rn(dz, 0.30);
    const double band = __dmul_rn(0.035, ::exp(-__dmul_rn(zz, zz)));
    const double band_rgb[3] = {1.0, 0.92, 0.80};
    double tint[3] = {1.0, 1.0, 1.0};
    if (shifted) {
        const double slide = clip(__dmul_rn(0.35, lnshift), -0.6, 0.6);
        tint[0] = __dsub_rn(1.0, slide);
        tint[2] = __dadd_rn(1.0, slide);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double b = __dmul_rn(band, band_rgb[k]);
        if (shifted) b = __dmul_rn(__dmul_rn(b, s4), tint[k]);
        c[k] = __dadd_rn(c[k], b);
    }
}

// numpy.interp of x on the table (xp, fp) of n points.
__device__ __forceinline__ double interp_table(double x, const double *xp, const float *fp,
                                               int n) {
    if (x != x) return x;
    if (x < xp[0]) return (double)fp[0];
    if (x >= xp[n - 1]) return (double)fp[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {  // xp[lo] <= x < xp[hi]
        const int mid = (lo + hi) >> 1;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    if (xp[lo] == x) return (double)fp[lo];
    const double f0 = fp[lo], f1 = fp[lo + 1];
    const double slope = __ddiv_rn(__dsub_rn(f1, f0), __dsub_rn(xp[lo + 1], xp[lo]));
    return __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[lo])), f0);
}

// numpy.interp on the grid 0, 1, ..., n-1 of one column of an (n, 3) table.
__device__ __forceinline__ double interp_unit(double u, const float *table, int n, int col) {
    if (u != u) return u;
    if (u < 0.0) return (double)table[col];
    if (u >= (double)(n - 1)) return (double)table[3 * (n - 1) + col];
    const int lo = (int)::floor(u);
    const double f0 = table[3 * lo + col];
    if ((double)lo == u) return f0;
    const double f1 = table[3 * (lo + 1) + col];
    const double slope = __dsub_rn(f1, f0);  // divided by xp[lo+1] - xp[lo] = 1
    return __dadd_rn(__dmul_rn(slope, __dsub_rn(u, (double)lo)), f0);
}

// render.py:422-484 (_disk_radiance) with emission/redshift.py:19-116
// (redshift_factor with p_t = 1) for one hit.
__device__ void disk_radiance(const EmissionArgs &a, const double *pos, const double *mom,
                              double c[3]) {
    Geometry g;
    geometry_full(a.mass, a.spin, pos[0], pos[1], pos[2], false, g);
    const double r = g.r;
    const double t_norm = interp_table(r, a.lut_radii, a.temperature, a.temperature_size);
    // redshift.py:19-48: circular-orbit velocity and 4-velocity.
    const double omega = __ddiv_rn(1.0, __dadd_rn(::pow(r, 1.5), a.spin));
    const double v0 = __dmul_rn(-omega, pos[1]), v1 = __dmul_rn(omega, pos[0]), v2 = 0.0;
    const double ldv = __dadd_rn(1.0, __dadd_rn(__dadd_rn(__dmul_rn(g.l[0], v0),
                                                          __dmul_rn(g.l[1], v1)),
                                                __dmul_rn(g.l[2], v2)));
    const double vv = __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)),
                                __dmul_rn(v2, v2));
    const double norm2 = __dadd_rn(__dadd_rn(-1.0, vv),
                                   __dmul_rn(__dmul_rn(__dmul_rn(2.0, g.h), ldv), ldv));
    const double u_t = __ddiv_rn(1.0, ::sqrt(-norm2));
    const double u0 = __dmul_rn(u_t, v0), u1 = __dmul_rn(u_t, v1), u2 = __dmul_rn(u_t, v2);
    // redshift.py:107-116 with traced p_t = 1.
    const double freq = __dadd_rn(__dmul_rn(1.0, u_t),
                                  __dadd_rn(__dadd_rn(__dmul_rn(mom[0], u0), __dmul_rn(mom[1], u1)),
                                            __dmul_rn(mom[2], u2)));
    const double shift = __ddiv_rn(a.observer_lapse, freq);
    const double t_obs = np_max(__dmul_rn(__dmul_rn(shift, t_norm), a.disk_temperature), 1.0);
    const double log_t = clip(::log(t_obs), a.bb_log_min, a.bb_log_max);
    const double u = __dmul_rn(__ddiv_rn(__dsub_rn(log_t, a.bb_log_min),
                                         __dsub_rn(a.bb_log_max, a.bb_log_min)),
                               (double)(a.bb_size - 1));
    const double phi = ::atan2(pos[1], pos[0]);
    const double s1 = ::sin(__dadd_rn(__dmul_rn(9.0, phi), __dmul_rn(2.2, r)));
    const double s2 = ::sin(__dsub_rn(__dmul_rn(23.0, phi), __dmul_rn(5.0, r)));
    const double s3 = ::sin(__dmul_rn(3.5, __dsub_rn(r, a.disk_inner)));
    const double detail = __dadd_rn(
        1.0, __dmul_rn(a.disk_detail, __dadd_rn(__dadd_rn(__dmul_rn(0.18, s1), __dmul_rn(0.12, s2)),
                                                __dmul_rn(0.15, s3))));
    const double brightness =
        __dmul_rn(::pow(__ddiv_rn(t_obs, 6500.0), 4.0), np_max(detail, 0.2));
#pragma unroll
    for (int k = 0; k < 3; ++k)
        c[k] = __dmul_rn(interp_unit(u, a.bb_table, a.bb_size, k), brightness);
}

// One pixel: the radiance of its supersample rays, averaged as
// radiance.reshape(h, w, ss^2, 3).mean(axis=2) (render.py:677-680).
__global__ void radiance_kernel(const EmissionArgs a) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.pixels) return;
    const int ss2 = a.supersample * a.supersample;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < ss2; ++k) {
        const long long i = p * ss2 + k;
        const int st = a.status[i];
        double c[3] = {0.0, 0.0, 0.0};
        if (st == BH_RAY_ESCAPED) {
            const double *d = a.escape_dir + 3 * i;
            // render.py:660-669: g = B / E for tetrad rays.
            const double shift = a.energy ? __ddiv_rn(a.observer_lapse, a.energy[i]) : 0.0;
            starfield(d[0], d[1], d[2], shift, c);
        } else if (st == BH_RAY_DISK) {
            disk_radiance(a, a.hit_pos + 3 * i, a.hit_mom + 3 * i, c);
        } else if (st == BH_RAY_TERMINATED) {
            c[0] = a.sheet_rgb[0]; c[1] = a.sheet_rgb[1]; c[2] = a.sheet_rgb[2];
        }
        if (k == 0) {
            acc[0] = c[0]; acc[1] = c[1]; acc[2] = c[2];
        } else {
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[j] = __dadd_rn(acc[j], c[j]);
        }
    }
    float *o = a.hdr + 3 * p;
#pragma unroll
    for (int j = 0; j < 3; ++j) o[j] = (float)__ddiv_rn(acc[j], (double)ss2);
}

// ------------------------------------------------------------ development

// post.py:47-56: scale of the bright pass; img = hdr * exposure.
__global__ void bright_kernel(const float *hdr, long long pixels, float exposure, float threshold,
                              float *bright) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    float v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] = __fmul_rn(hdr[3 * p + k], exposure);
    const float lum = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, v[0]), __fmul_rn(0.7152f, v[1])),
                                __fmul_rn(0.0722f, v[2]));
    const float excess = fmaxf(__fsub_rn(lum, threshold), 0.0f);
    const float scale = lum > 1e-9f ? __fdiv_rn(excess, __fadd_rn(lum, 1e-9f)) : 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) bright[3 * p + k] = __fmul_rn(v[k], scale);
}

// post.py:23-32: one separable pass with edge padding; each tap adds
// w * x in float64 to the float32 pixel.  axis 0 blurs along rows (y).  The
// 2 radius + 1 weights are staged in shared memory: every thread reads every
// weight.
__global__ void blur_kernel(const float *src, long long width, long long height,
                            const double *weights, int radius, int axis, float *dst) {
    extern __shared__ double w[];
    for (int t = threadIdx.x; t <= 2 * radius; t += blockDim.x) w[t] = weights[t];
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= width * height) return;
    const long long y = p / width, x = p - y * width;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int t = 0; t <= 2 * radius; ++t) {
        long long yy = y, xx = x;
        if (axis == 0) {
            yy = y + t - radius;
            yy = yy < 0 ? 0 : (yy >= height ? height - 1 : yy);
        } else {
            xx = x + t - radius;
            xx = xx < 0 ? 0 : (xx >= width ? width - 1 : xx);
        }
        const float *s = src + 3 * (yy * width + xx);
        const double wt = w[t];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            acc[k] = (float)__dadd_rn((double)acc[k], __dmul_rn(wt, (double)s[k]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[3 * p + k] = acc[k];
}

// post.py:59-85: ACES (Narkowicz 2015 fit) and the sRGB curve, float32.
// post.py:70-85 (encode_srgb): linear [0, 1] to 8 bits, float32.
__device__ __forceinline__ uint8_t srgb8(float m) {
    m = fminf(fmaxf(m, 0.0f), 1.0f);
    const float enc = m <= 0.0031308f
                          ? __fmul_rn(12.92f, m)
                          : __fsub_rn(__fmul_rn(1.055f, powf(m, (float)(1.0 / 2.4))), 0.055f);
    return (uint8_t)__fadd_rn(__fmul_rn(enc, 255.0f), 0.5f);
}

__device__ __forceinline__ uint8_t develop_channel(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    const float num = __fmul_rn(x, __fadd_rn(__fmul_rn(a, x), b));
    const float den = __fadd_rn(__fmul_rn(x, __fadd_rn(__fmul_rn(c, x), d)), e);
    return srgb8(fminf(fmaxf(__fdiv_rn(num, den), 0.0f), 1.0f));
}

// ------------------------------------------------------------ video frames

// offline/video.py:33-43 (downsample): the mean of each factor x factor block
// of an 8-bit image, truncated to 8 bits.  The float32 block sum of integers
// below 2^24 is exact in any order.
__global__ void downsample_kernel(const uint8_t *in, long long in_w, int factor,
                                  long long out_w, long long out_h, uint8_t *out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= out_w * out_h) return;
    const long long oy = p / out_w, ox = p - oy * out_w;
    float sum[3] = {0.0f, 0.0f, 0.0f};
    for (int dy = 0; dy < factor; ++dy)
        for (int dx = 0; dx < factor; ++dx) {
            const uint8_t *s = in + 3 * ((oy * factor + dy) * in_w + ox * factor + dx);
#pragma unroll
            for (int k = 0; k < 3; ++k) sum[k] += (float)s[k];
        }
    const float n = (float)(factor * factor);
#pragma unroll
    for (int k = 0; k < 3; ++k) out[3 * p + k] = (uint8_t)__fdiv_rn(sum[k], n);
}

// offline/video.py:46-59 (frame_bloom): the frame lifted to a pseudo-linear
// domain, (x / 255)^2.2 in float32.
__global__ void lift_kernel(const uint8_t *in, long long n, float *out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = powf(__fdiv_rn((float)in[i], 255.0f), 2.2f);
}

// linear + strength * blurred bright pass, clipped to [0, 1], sRGB-encoded.
__global__ void bloom_encode_kernel(const float *linear, const float *blurred, long long n,
                                    float strength, uint8_t *out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = srgb8(__fadd_rn(linear[i], __fmul_rn(strength, blurred[i])));
}

// img = hdr * exposure (+ strength * blurred bright pass), tone-mapped.
__global__ void develop_kernel(const float *hdr, const float *blurred, long long pixels,
                               float exposure, float strength, uint8_t *out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = __fmul_rn(hdr[3 * p + k], exposure);
        if (blurred) v = __fadd_rn(v, __fmul_rn(strength, blurred[3 * p + k]));
        out[3 * p + k] = develop_channel(v);
    }
}

// Largest blur radius whose weights fit the default 48 KiB of shared memory.
constexpr int kMaxBlurRadius = 6000;

static unsigned grid_of(long long n, int block) {
    const long long g = (n + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : g);
}

static int em_invalid(const char *msg) {
    set_error("%s", msg);
    return BH_ERR_INVALID_ARGUMENT;
}

static int em_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return BH_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BH_ERR_CUDA;
}

}  // namespace bh

using namespace bh;

extern "C" int bh_offline_radiance(const bh_emission_config *config, const int32_t *status,
                                   const double *escape_directions, const double *hit_positions,
                                   const double *hit_momenta, const double *energy,
                                   int64_t width, int64_t height, const float *temperature_table,
                                   const double *lut_radii, const float *blackbody_table,
                                   float *hdr, void *stream) {
    if (!config) return em_invalid("config is NULL");
    const bh_emission_config &c = *config;
    if (!(c.mass > 0.0) || !(std::fabs(c.spin) <= c.mass))
        return em_invalid("Kerr bound violated or mass not positive");
    if (c.supersample < 1) return em_invalid("supersample must be >= 1");
    if (width < 0 || height < 0) return em_invalid("width and height must be >= 0");
    if (c.temperature_size < 2 || c.blackbody_size < 2)
        return em_invalid("lookup tables need at least 2 entries");
    if (!(c.bb_log_max > c.bb_log_min)) return em_invalid("bb_log_max must exceed bb_log_min");
    const long long pixels = (long long)width * height;
    if (pixels == 0) return BH_OK;
    if (!status || !escape_directions || !hit_positions || !hit_momenta || !temperature_table ||
        !lut_radii || !blackbody_table || !hdr)
        return em_invalid("NULL pointer argument");
    EmissionArgs a;
    a.mass = c.mass;
    a.spin = c.spin;
    a.disk_inner = c.disk_inner;
    a.disk_temperature = c.disk_temperature;
    a.disk_detail = c.disk_detail;
    a.observer_lapse = c.observer_lapse;
    a.bb_log_min = c.bb_log_min;
    a.bb_log_max = c.bb_log_max;
    a.sheet_rgb[0] = c.sheet_rgb[0];
    a.sheet_rgb[1] = c.sheet_rgb[1];
    a.sheet_rgb[2] = c.sheet_rgb[2];
    a.temperature_size = c.temperature_size;
    a.bb_size = c.blackbody_size;
    a.supersample = c.supersample;
    a.pixels = pixels;
    a.status = status;
    a.escape_dir = escape_directions;
    a.hit_pos = hit_positions;
    a.hit_mom = hit_momenta;
    a.energy = energy;
    a.temperature = temperature_table;
    a.lut_radii = lut_radii;
    a.bb_table = blackbody_table;
    a.hdr = hdr;
    radiance_kernel<<<grid_of(pixels, 128), 128, 0, (cudaStream_t)stream>>>(a);
    return em_launch("bh_offline_radiance launch");
}

extern "C" size_t bh_develop_workspace_bytes(int64_t width, int64_t height) {
    if (width <= 0 || height <= 0) return 256;
    const size_t img = (size_t)width * (size_t)height * 3 * sizeof(float);
    return 2 * ((img + 255) & ~(size_t)255);
}

extern "C" int bh_develop(const float *hdr, int64_t width, int64_t height, double exposure,
                          double bloom_threshold, double bloom_strength,
                          const double *blur_weights, int32_t blur_radius, uint8_t *out,
                          void *workspace, size_t workspace_bytes, void *stream) {
    if (width < 0 || height < 0) return em_invalid("width and height must be >= 0");
    const long long pixels = (long long)width * height;
    if (pixels == 0) return BH_OK;
    if (!hdr || !out) return em_invalid("NULL pointer argument");
    const bool bloom = bloom_strength > 0.0;
    if (bloom && (!blur_weights || blur_radius < 1 || blur_radius > kMaxBlurRadius))
        return em_invalid("bloom needs blur weights and a radius in [1, 6000]");
    cudaStream_t s = (cudaStream_t)stream;
    const float ex = (float)exposure;
    if (!bloom) {
        develop_kernel<<<grid_of(pixels, 256), 256, 0, s>>>(hdr, nullptr, pixels, ex, 0.0f, out);
        return em_launch("bh_develop launch");
    }
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) ||
        workspace_bytes < bh_develop_workspace_bytes(width, height)) {
        set_error("workspace must be 256-byte aligned and hold bh_develop_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    const size_t img = ((size_t)pixels * 3 * sizeof(float) + 255) & ~(size_t)255;
    float *bright = static_cast<float *>(workspace);
    float *tmp = reinterpret_cast<float *>(static_cast<char *>(workspace) + img);
    bright_kernel<<<grid_of(pixels, 256), 256, 0, s>>>(hdr, pixels, ex, (float)bloom_threshold,
                                                       bright);
    // post.py:23-32: rows (axis 0) first, then columns; the second pass
    // writes over the bright pass, which is no longer needed.
    const size_t wbytes = (size_t)(2 * blur_radius + 1) * sizeof(double);
    blur_kernel<<<grid_of(pixels, 256), 256, wbytes, s>>>(bright, width, height, blur_weights,
                                                          blur_radius, 0, tmp);
    blur_kernel<<<grid_of(pixels, 256), 256, wbytes, s>>>(tmp, width, height, blur_weights,
                                                          blur_radius, 1, bright);
    develop_kernel<<<grid_of(pixels, 256), 256, 0, s>>>(hdr, bright, pixels, ex,
                                                        (float)bloom_strength, out);
    return em_launch("bh_develop launch");
}

extern "C" int bh_downsample(const uint8_t *image, int64_t width, int64_t height,
                             int32_t factor, uint8_t *out, void *stream) {
    if (width < 0 || height < 0 || factor < 1 || factor > 256)
        return em_invalid("width and height must be >= 0 and factor in [1, 256]");
    const long long ow = width / factor, oh = height / factor;
    if (ow * oh == 0) return BH_OK;
    if (!image || !out) return em_invalid("NULL pointer argument");
    downsample_kernel<<<grid_of(ow * oh, 256), 256, 0, (cudaStream_t)stream>>>(
        image, width, factor, ow, oh, out);
    return em_launch("bh_downsample launch");
}

extern "C" size_t bh_frame_bloom_workspace_bytes(int64_t width, int64_t height) {
    if (width <= 0 || height <= 0) return 256;
    const size_t img = (size_t)width * (size_t)height * 3 * sizeof(float);
    return 3 * ((img + 255) & ~(size_t)255);
}

extern "C" int bh_frame_bloom(const uint8_t *image, int64_t width, int64_t height,
                              double strength, const double *blur_weights, int32_t blur_radius,
                              uint8_t *out, void *workspace, size_t workspace_bytes,
                              void *stream) {
    if (width < 0 || height < 0) return em_invalid("width and height must be >= 0");
    const long long pixels = (long long)width * height;
    if (pixels == 0) return BH_OK;
    if (!image || !out) return em_invalid("NULL pointer argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (!(strength > 0.0)) {  // video.py:53-54: the frame unchanged
        const cudaError_t e =
            cudaMemcpyAsync(out, image, (size_t)pixels * 3, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) {
            set_error("bh_frame_bloom copy: %s", cudaGetErrorString(e));
            return BH_ERR_CUDA;
        }
        return BH_OK;
    }
    if (!blur_weights || blur_radius < 1 || blur_radius > kMaxBlurRadius)
        return em_invalid("bloom needs blur weights and a radius in [1, 6000]");
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) ||
        workspace_bytes < bh_frame_bloom_workspace_bytes(width, height)) {
        set_error("workspace must be 256-byte aligned and hold bh_frame_bloom_workspace_bytes()");
        return BH_ERR_WORKSPACE;
    }
    const size_t img = ((size_t)pixels * 3 * sizeof(float) + 255) & ~(size_t)255;
    float *linear = static_cast<float *>(workspace);
    float *bright = reinterpret_cast<float *>(static_cast<char *>(workspace) + img);
    float *tmp = reinterpret_cast<float *>(static_cast<char *>(workspace) + 2 * img);
    lift_kernel<<<grid_of(3 * pixels, 256), 256, 0, s>>>(image, 3 * pixels, linear);
    // post.py:40-56 with threshold 0.55, no exposure: the bright pass,
    // two blur passes (rows, then columns), added back with the strength.
    bright_kernel<<<grid_of(pixels, 256), 256, 0, s>>>(linear, pixels, 1.0f, 0.55f, bright);
    const size_t wbytes = (size_t)(2 * blur_radius + 1) * sizeof(double);
    blur_kernel<<<grid_of(pixels, 256), 256, wbytes, s>>>(bright, width, height, blur_weights,
                                                          blur_radius, 0, tmp);
    blur_kernel<<<grid_of(pixels, 256), 256, wbytes, s>>>(tmp, width, height, blur_weights,
                                                          blur_radius, 1, bright);
    bloom_encode_kernel<<<grid_of(3 * pixels, 256), 256, 0, s>>>(linear, bright, 3 * pixels,
                                                                 (float)strength, out);
    return em_launch("bh_frame_bloom launch");
}
