// bh_internal.h -- shared declarations of the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/bh_b200.h"

namespace bh {

// Device workspace of a trace / propagate launch (the first 256 bytes of the
// caller's workspace).  Zeroed by the launcher before every launch.
struct alignas(256) TraceWorkspace {
    unsigned long long queue_head;  // next unclaimed ray of the work queue
    long long iterations;           // max attempts over rays
    unsigned long long attempts;    // sum of attempts
    unsigned long long accepted;    // sum of accepted steps
    int timed_out;
    int bad_rays;
    int tape_overflow;  // rays with more accepted steps than the tape holds
    int bad_spins;      // propagate: rays whose own spin breaks the Kerr bound
    int bad_order;      // propagate: order entries outside [0, n)
};
static_assert(sizeof(TraceWorkspace) == 256, "workspace header is 256 bytes");

// Device copy of a camera: the pinhole basis plus its scene, and the first
// global ray index it owns.
struct CameraDev {
    double pos[3], fwd[3], right[3], up[3];
    double half_w, half_h;
    long long width, height;
    long long first_ray;
    double mass, spin, capture_radius, escape_radius;
};
// The camera tables' sizes (bh_trace_cameras_workspace_bytes and the static
// table of bh_trace_cameras_noalloc) are stated in bytes per camera.
static_assert(sizeof(CameraDev) == 168, "camera record is 168 bytes");

struct TraceArgs {
    // ray source: states (source == 0) or cameras (source == 1)
    const double *state0;
    const CameraDev *cameras;  // device copy (in the workspace)
    int ncameras;
    int source;
    // single-scene parameters (source == 0)
    double mass, spin, capture_radius, escape_radius;
    const double *spin_of_ray;  // propagate only; may be null
    // propagate: the ray at each launch position (bh_propagate_order); null
    // takes the rays in their own order
    const int32_t *order;
    // outputs
    double *states;
    int32_t *status;
    int64_t *steps;  // accepted steps (trace) or accepted count (propagate)
    double *h_io;    // propagate: per-ray step size in/out
    double *lam_io;  // affine parameter: propagate in/out, trace out; may be null
    long long n;
    int layout;
    // controller
    double rtol, atol, initial_step, max_step, min_step;
    long long max_steps;     // trace: accepted-step budget
    long long max_attempts;  // trace: 4 * max_steps; propagate: n_steps
    long long timeout_ns;
    int project_every;       // null-constraint projection period (iterations); 0 = off
    // Mixed propagate: squared radius of the float64 band; an attempt runs
    // float64 stage arithmetic for the whole warp while one of its rays lies
    // at r_+ < r < sqrt(f64_r2).  0 = no band.
    double f64_r2;
    TraceWorkspace *ws;
    // optional tape of the accepted steps (trace only): step sizes
    // (n x tape_cap) and float64 states before every ckpt_every-th accepted
    // step (n x ceil(tape_cap / ckpt_every) x 8)
    double *h_tape;
    double *ckpt;
    long long tape_cap;
    int ckpt_every;
};

// Launch-shape variants of the trace / propagate kernels: threads per block
// and the __launch_bounds__ minimum blocks per SM, which caps registers.
struct Variant {
    int block;
    int min_blocks;
    int rays_per_thread;
};

int trace_variant_count(int precision);
Variant trace_variant(int precision, int idx);
int trace_default_variant(int precision);
int propagate_default_variant(int precision);

// Registers and occupancy of a compiled trace (propagate = false) or propagate
// kernel variant; returns 0 on success.
int kernel_attributes(bool propagate, int precision, int idx, int *regs,
                      int *max_blocks);

cudaError_t launch_trace(const TraceArgs &args, int precision, int variant,
                         int blocks_per_sm, cudaStream_t stream);
cudaError_t launch_propagate(const TraceArgs &args, int precision, int variant,
                             int blocks_per_sm, cudaStream_t stream);

// bh_trace with an optional tape of the accepted steps (bh_capi.cu).
int bh_trace_with_tape(const bh_trace_config *config, const bh_scene *scene,
                       const double *state0, double *states, int32_t *status,
                       int64_t *steps, int64_t n, void *workspace, void *stream,
                       double *h_tape, double *ckpt, int64_t tape_cap, int ckpt_every);

// ------------------------------------------------------------ tile tracer
// A ray parked at an accepted step whose z changed sign, for refinement.
struct TileCrossing {
    double y0[8];        // state before the step
    double y1[8];        // state after the step; the refined crossing state once a hit
    double h;            // the step's size
    double h_next;       // controller step size after the step
    long long steps;     // accepted steps before the step
    long long attempts;  // attempts including the step
    long long ray;
    int speculative;     // the ray went on in place past this crossing
    int hit;             // set by the refinement for rays with speculative records
};
static_assert(sizeof(TileCrossing) == 176, "crossing record is 176 bytes");

// A ray that continues after a crossing outside the disk.
struct TileResume {
    double y[8];
    double h;
    long long steps, attempts, ray;
};
static_assert(sizeof(TileResume) == 96, "resume record is 96 bytes");

// Counters of a tile trace.  Round r uses the parity-(r & 1) queue head and
// crossing count and reads the parity-(r & 1) resume count (written by the
// refinement of round r - 1); round r's tracing kernel zeroes the other
// parity's counters before round r's refinement and round r + 1 use them.
struct alignas(256) TileWorkspace {
    unsigned long long queue_head[2];
    unsigned long long n_cross[2];
    unsigned long long n_resume[2];
    unsigned long long refine_head[2];  // chunks of 32 crossings claimed by the refinement
    unsigned long long n_spec[2];       // speculative crossing records (may pass spec_cap)
    long long iterations;  // max attempts over finalised rays
    unsigned long long attempts, accepted, crossings, disk_hits;
    int timed_out;
};
static_assert(sizeof(TileWorkspace) == 256, "tile workspace header is 256 bytes");

struct TileArgs {
    const double *state0;
    long long n;
    int layout;
    int round;  // 0: rays from state0; r > 0: resume records of parity r & 1
    int flush;  // finalise every ray in flight as IN_FLIGHT without stepping
    int interior;  // interior camera: capture_radius is the stop radius
    int inline_refine;  // refine crossings in place instead of parking them
    double mass, spin, capture_radius, escape_radius;
    double disk_inner, disk_outer;  // disk_outer <= 0: no crossing tests
    double rtol, atol, initial_step, max_step;
    long long max_steps, max_attempts, saturate_steps;
    long long timeout_ns;
    TileCrossing *cross;  // capacity n: a parked ray stops, so one per ray and round
    TileCrossing *spec;   // capacity spec_cap: crossings that the ray went on past
    long long spec_cap;
    unsigned long long *first_hit;  // per ray: fewest accepted steps of a refined hit
    int8_t *has_spec;     // per ray: a speculative record exists
    TileResume *resume;   // capacity n
    double *states;
    int32_t *status;
    int64_t *steps;
    double *hit_pos, *hit_mom, *escape_dir;
    int8_t *saturated;
    TileWorkspace *ws;
};

// Arguments of the offline radiance kernel (bh_emission.cu).
struct EmissionArgs {
    double mass, spin, disk_inner, disk_temperature, disk_detail, observer_lapse;
    double bb_log_min, bb_log_max;
    double sheet_rgb[3];
    int temperature_size, bb_size, supersample;
    long long pixels;
    const int32_t *status;
    const double *escape_dir, *hit_pos, *hit_mom, *energy;
    const float *temperature;
    const double *lut_radii;
    const float *bb_table;
    float *hdr;
};

// Arguments of the real-time shading kernel (bh_realtime_shade.cu), float32.
struct RealtimeShadeArgs {
    float mass, spin, disk_inner, disk_outer, disk_temperature, disk_detail;
    float exposure, observer_lapse, bb_log_min, bb_log_max;
    float sky_amplification, sheet_radiance, whiteout;
    int background, temperature_size, blackbody_size;
    long long pixels;
    const int32_t *status;
    const double *states, *hit_pos, *hit_mom;
    const float *temperature, *blackbody;
    uint8_t *rgb;
};

int tile_default_variant(int precision);
cudaError_t launch_tile(const TileArgs &args, int precision, int variant,
                        int blocks_per_sm, cudaStream_t stream);
cudaError_t launch_refine(const TileArgs &args, cudaStream_t stream);

// Records a message for bh_last_error on this host thread.
void set_error(const char *fmt, ...);

}  // namespace bh
