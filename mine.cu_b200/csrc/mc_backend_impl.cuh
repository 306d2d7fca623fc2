// mc_backend_impl.cuh - the environment step for one numerics mode.
//
// Included by exactly two translation units:
//   mc_fast.cu  (MC_NUMERICS_FAST=1, nvcc --use_fast_math): calls the same
//               CUDA math functions as the reference build, in the same op
//               order, so results match the reference bit for bit;
//   mc_ieee.cu  (MC_NUMERICS_FAST=0, -fmad=false): IEEE-754 ops and the trig
//               of mc_ieee_math.h, so results match the CPU checker bit for bit.
// MC_NS names the namespace so both back ends link into one library.
//
// Semantics follow the reference's src/kernels.cu; every device function
// cites the lines it restates.  Two launch forms share these functions:
//   plain : one kernel per reference kernel, in the reference's order;
//   fused : one persistent kernel per step, a warp per env.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <type_traits>
#include "mc_internal.h"
#include "mc_ieee_math.h"
#include "mc_philox.h"

#ifndef MC_NS
#error "define MC_NS before including mc_backend_impl.cuh"
#endif

namespace MC_NS {

constexpr int8_t AIR = -1, GRASS = 0, DIRT = 1, OAKLOG = 3, LEAVES = 4, BRICK = 8,
                 COBBLESTONE = 9, PLANKS = 10, BEDROCK = 12;

// Colour tables: the reference's BLOCK_COLORS / SKY_COLOR (kernels.cu:27-44)
// and the pre-rounded BLOCK_COLORS_U8 / SKY_COLOR_U8 (kernels.cu:479-495).
__constant__ float c_rgb[13][3] = {
    {0.30f, 0.65f, 0.20f}, {0.55f, 0.35f, 0.20f}, {0.50f, 0.50f, 0.50f}, {0.55f, 0.40f, 0.25f},
    {0.20f, 0.55f, 0.15f}, {0.90f, 0.85f, 0.60f}, {0.20f, 0.40f, 0.80f}, {0.85f, 0.90f, 0.95f},
    {0.70f, 0.35f, 0.30f}, {0.40f, 0.40f, 0.40f}, {0.75f, 0.60f, 0.40f}, {0.95f, 0.95f, 0.98f},
    {0.15f, 0.15f, 0.15f}};
__constant__ float c_sky[3] = {0.53f, 0.81f, 0.92f};
__constant__ uint8_t c_rgb8[13][3] = {
    {76, 166, 51}, {140, 89, 51}, {127, 127, 127}, {140, 102, 64}, {51, 140, 38},
    {229, 217, 153}, {51, 102, 204}, {217, 229, 242}, {178, 89, 76}, {102, 102, 102},
    {191, 153, 102}, {242, 242, 250}, {38, 38, 38}};
__constant__ uint8_t c_sky8[3] = {135, 206, 235};

// ---------------------------------------------------------------------------
// Numerics policy
// ---------------------------------------------------------------------------
// Arithmetic is written with explicit single-rounding ops so that the
// compiler cannot contract or reorder it differently in different contexts
// (kernel shape, basic blocks, hoisting):
//   mul/add/sub  one IEEE rounding each (never fused);
//   mad(a,b,c)   ref_fast: one fused multiply-add, exactly where the
//                reference build's compiler fuses (determined by comparing
//                outputs with the reference's kernels on millions of inputs);
//                ieee: a*b rounded, then + c rounded (the CPU checker's order).
#if MC_NUMERICS_FAST
struct N {
    static __device__ __forceinline__ float mad(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    // a/b - 1 and 1 - a/b: the build turns the division into a*(1/b) with an
    // approximate reciprocal and fuses it with the +-1
    static __device__ __forceinline__ float div_sub1(float a, float b) { return __fmaf_rn(a, __fdividef(1.0f, b), -1.0f); }
    static __device__ __forceinline__ float one_sub_div(float a, float b) { return __fmaf_rn(-a, __fdividef(1.0f, b), 1.0f); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    // a / b as the build computes it (a times the approximate reciprocal of
    // b), with the reciprocal passed in so repeated divisors share it
    static __device__ __forceinline__ float rcp_of(float b) { return __fdividef(1.0f, b); }
    static __device__ __forceinline__ float div_r(float a, float b, float rcp_b) { (void)b; return __fmul_rn(a, rcp_b); }
    static __device__ __forceinline__ float sin(float x) { return sinf(x); }
    static __device__ __forceinline__ float cos(float x) { return cosf(x); }
    static __device__ __forceinline__ float tan(float x) { return tanf(x); }
    static __device__ __forceinline__ void sincos_i(float x, float* s, float* c) { __sincosf(x, s, c); }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
};
#else
struct N {
    static __device__ __forceinline__ float mad(float a, float b, float c) { return __fadd_rn(__fmul_rn(a, b), c); }
    static __device__ __forceinline__ float div_sub1(float a, float b) { return __fsub_rn(__fdiv_rn(a, b), 1.0f); }
    static __device__ __forceinline__ float one_sub_div(float a, float b) { return __fsub_rn(1.0f, __fdiv_rn(a, b)); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float rcp_of(float b) { (void)b; return 0.0f; }
    static __device__ __forceinline__ float div_r(float a, float b, float rcp_b) { (void)rcp_b; return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sin(float x) { return mc_ieee_sinf(x); }
    static __device__ __forceinline__ float cos(float x) { return mc_ieee_cosf(x); }
    static __device__ __forceinline__ float tan(float x) { return mc_ieee_tanf(x); }
    static __device__ __forceinline__ void sincos_i(float x, float* s, float* c) { mc_ieee_sincosf(x, s, c); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float x) { return __fsqrt_rn(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return __fdiv_rn(1.0f, __fsqrt_rn(x)); }
};
#endif

// ---------------------------------------------------------------------------
// Bounds checks of the debug build (MC_CHECK_BOUNDS=1)
// ---------------------------------------------------------------------------
// In the debug build every voxel, shared-memory world, table and observation
// index is checked against its buffer before the access.  A failed check
// skips the access (a voxel read returns air) and records the first
// violation (site, index, limit) and a count in g_bounds, which
// bounds_report() reads and clears; the step kernels also set
// MC_KERR_BOUNDS in their env's error word.  Nothing traps.  The normal
// build compiles every check to nothing.
#ifndef MC_CHECK_BOUNDS
#define MC_CHECK_BOUNDS 0
#endif
#if MC_CHECK_BOUNDS
__device__ int32_t g_bounds[4];  // violations, first site (MC_SITE_*), first index, its limit
__device__ __noinline__ void bounds_fail(long long i, long long n, int site) {
    if (atomicAdd(&g_bounds[0], 1) == 0) {
        g_bounds[1] = site;
        g_bounds[2] = (int32_t)i;
        g_bounds[3] = (int32_t)n;
    }
}
__device__ __forceinline__ bool in_bounds(long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    bounds_fail(i, n, site);
    return false;
}
// A step kernel's exit: a violation anywhere is also reported in the env's error word.
__device__ __forceinline__ void bounds_to_flags(int32_t* flags) {
    if (*(volatile int32_t*)&g_bounds[0]) atomicCAS(&flags[MC_FLAG_ERROR], MC_KERR_NONE, MC_KERR_BOUNDS);
}
#else
__device__ __forceinline__ constexpr bool in_bounds(long long, long long, int) { return true; }
__device__ __forceinline__ void bounds_to_flags(int32_t*) {}
#endif

// ---------------------------------------------------------------------------
// Agent step
// ---------------------------------------------------------------------------
struct Dec {
    float fwd, strafe, dyaw, dpitch, speed;
    bool jump, brk, place;
};

// decode_actions_kernel (kernels.cu:1459-1504)
__device__ __forceinline__ Dec decode_buttons(const int8_t b[8], float l0, float l1, float sprint_mult) {
    Dec d;
    d.fwd = N::sub((float)b[0], (float)b[1]);
    d.strafe = N::sub((float)b[3], (float)b[2]);
    d.dyaw = l0;
    d.dpitch = l1;
    d.jump = (b[4] != 0);
    d.brk = (b[5] != 0);
    d.place = (b[6] != 0);
    d.speed = (b[0] && b[7]) ? sprint_mult : 1.0f;
    return d;
}

// Actions of one env group: discrete actions, or buttons + look.
struct ActionSrc {
    const uint8_t* actions;
    const int8_t* buttons;
    const float* look;
};
__device__ __forceinline__ void load_action_from(const ActionSrc& a, float look_delta, long long i, int8_t b[8],
                                                 float& l0, float& l1) {
    if (a.actions) {
        float lk[2];
        mc_discrete_to_buttons(a.actions[i], look_delta, b, lk);
        l0 = lk[0];
        l1 = lk[1];
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) b[k] = a.buttons[i * 8 + k];
        l0 = a.look[i * 2 + 0];
        l1 = a.look[i * 2 + 1];
    }
}

__device__ __forceinline__ void load_action(const mc_kp& p, long long i, int8_t b[8], float& l0, float& l1) {
    if (p.actions) {
        float lk[2];
        mc_discrete_to_buttons(p.actions[i], p.look_delta, b, lk);
        l0 = lk[0];
        l1 = lk[1];
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) b[k] = p.buttons[i * 8 + k];
        l0 = p.look[i * 2 + 0];
        l1 = p.look[i * 2 + 1];
    }
}

struct Agent {
    float x, y, z, vx, vy, vz, yaw, pitch;
    bool og;
};

__device__ __forceinline__ Agent load_agent(const mc_kp& p, long long i) {
    Agent a;
    a.x = p.positions[i * 3 + 0];
    a.y = p.positions[i * 3 + 1];
    a.z = p.positions[i * 3 + 2];
    a.vx = p.velocities[i * 3 + 0];
    a.vy = p.velocities[i * 3 + 1];
    a.vz = p.velocities[i * 3 + 2];
    a.yaw = p.yaws[i];
    a.pitch = p.pitches[i];
    a.og = p.on_ground[i] != 0;
    return a;
}

__device__ __forceinline__ void store_agent(const mc_kp& p, long long i, const Agent& a) {
    p.positions[i * 3 + 0] = a.x;
    p.positions[i * 3 + 1] = a.y;
    p.positions[i * 3 + 2] = a.z;
    p.velocities[i * 3 + 0] = a.vx;
    p.velocities[i * 3 + 1] = a.vy;
    p.velocities[i * 3 + 2] = a.vz;
    p.yaws[i] = a.yaw;
    p.pitches[i] = a.pitch;
    p.on_ground[i] = a.og ? 1 : 0;
}

// physics_kernel (kernels.cu:1511-1584): rotate, walk, gravity, clamp to the
// flat ground at world_y/4 and to [1, W-1] in x and z.  No voxel collision.
//   move_x = ((sin*fwd)*speed)*dt + ((cos*str)*walk)*dt   (the build fuses the strafe product)
//   move_z = ((cos*fwd)*speed)*dt - ((sin*str)*walk)*dt   (the build fuses the forward product)
//   vel_y += gravity*dt;  y += vel_y*dt                   (both fused)
__device__ __forceinline__ void physics(Agent& a, const Dec& d, const mc_kp& p) {
    a.yaw = N::add(a.yaw, d.dyaw);
    float new_pitch = N::add(a.pitch, d.dpitch);
    a.pitch = fminf(fmaxf(new_pitch, -1.56f), 1.56f);
    float cos_yaw = N::cos(a.yaw);
    float sin_yaw = N::sin(a.yaw);
    float fwd = d.fwd, str = d.strafe;
    float speed = N::mul(p.walk_speed, d.speed);
    float fx_ = N::mul(N::mul(N::mul(sin_yaw, fwd), speed), p.dt);
    float move_x = N::mad(N::mul(N::mul(cos_yaw, str), p.walk_speed), p.dt, fx_);
    float sz_ = N::mul(N::mul(N::mul(sin_yaw, str), p.walk_speed), p.dt);
    float move_z = N::mad(N::mul(N::mul(cos_yaw, fwd), speed), p.dt, -sz_);
    float vel_y = a.vy;
    if (d.jump && a.og) vel_y = p.jump_vel;
    vel_y = N::mad(p.gravity, p.dt, vel_y);
    float new_x = N::add(a.x, move_x);
    float new_y = N::mad(vel_y, p.dt, a.y);
    float new_z = N::add(a.z, move_z);
    float ground_y = (float)(p.wy / 4);
    if (new_y <= ground_y) {
        new_y = ground_y;
        vel_y = 0.0f;
        a.og = true;
    } else {
        a.og = false;
    }
    float margin = 1.0f;
    new_x = fminf(fmaxf(new_x, margin), N::sub((float)p.wx, margin));
    new_z = fminf(fmaxf(new_z, margin), N::sub((float)p.wz, margin));
    a.x = new_x;
    a.y = new_y;
    a.z = new_z;
    a.vy = vel_y;
}

// reset_kernel (kernels.cu:1760-1786)
__device__ __forceinline__ void reset_agent(Agent& a, const mc_kp& p) {
    a.x = p.spawn_x;
    a.y = p.spawn_y;
    a.z = p.spawn_z;
    a.vx = 0.0f;
    a.vy = 0.0f;
    a.vz = 0.0f;
    a.yaw = 0.0f;
    a.pitch = 0.0f;
    a.og = false;
}

// episode_check_kernel (kernels.cu:1954-1968) and the Python rule of
// minecu/__init__.py:363-366.
__device__ __forceinline__ bool episode_done(const mc_kp& p, int32_t cnt) {
    if (p.episode_rule == 0) return p.has_limit && cnt >= p.episode_length;
    return p.episode_length > 0 && cnt >= p.episode_length;
}

// One interact sample k of raycast_interact_kernel (kernels.cu:1621-1653):
// the point at t = 0.1 + k * 4/32 along the view direction from the eye.
struct Sample {
    int idx;  // flat in-env voxel index, valid if inb
    bool inb;
};
__device__ __forceinline__ Sample interact_sample(int k, float eye_x, float eye_y, float eye_z,
                                                  float dir_x, float dir_y, float dir_z,
                                                  int wx, int wy, int wz) {
    float reach = 4.0f;
    float t = N::mad((float)k, reach / 32.0f, 0.1f);  // k/8 is exact: same value fused or not
    float px = N::mad(dir_x, t, eye_x);
    float py = N::mad(dir_y, t, eye_y);
    float pz = N::mad(dir_z, t, eye_z);
    int vx = (int)floorf(px);
    int vy = (int)floorf(py);
    int vz = (int)floorf(pz);
    Sample s;
    s.inb = (vx >= 0 && vx < wx && vy >= 0 && vy < wy && vz >= 0 && vz < wz);
    s.idx = vy * (wx * wz) + vx * wz + vz;
    return s;
}

__device__ __forceinline__ void interact_dir(const Agent& a, float& dx, float& dy, float& dz) {
    float cos_yaw = N::cos(a.yaw);
    float sin_yaw = N::sin(a.yaw);
    float cos_pitch = N::cos(a.pitch);
    float sin_pitch = N::sin(a.pitch);
    dx = N::mul(sin_yaw, cos_pitch);
    dy = sin_pitch;
    dz = N::mul(cos_yaw, cos_pitch);
}

__device__ __forceinline__ bool reward_hit(const mc_kp& p, int8_t blk) {
    int8_t target = (int8_t)p.target_block;
    return target < 0 || blk == target;
}

// raycast_interact_kernel (kernels.cu:1591-1680), one thread per env.
// Returns the in-env index written (-1 if none); *reward as the reference.
__device__ __forceinline__ int interact_seq(int8_t* w, const Agent& a, bool brk, bool place,
                                            const mc_kp& p, float* reward) {
    *reward = 0.0f;
    if (!brk && !place) return -1;
    float dx, dy, dz;
    interact_dir(a, dx, dy, dz);
    float eye_x = a.x, eye_y = N::add(a.y, 1.6f), eye_z = a.z;
    int prev = -1;
    for (int k = 0; k < 32; ++k) {
        Sample s = interact_sample(k, eye_x, eye_y, eye_z, dx, dy, dz, p.wx, p.wy, p.wz);
        if (s.inb && in_bounds(s.idx, (long long)p.wx * p.wy * p.wz, MC_SITE_INTERACT)) {
            int8_t blk = w[s.idx];
            if (blk >= 0) {
                if (brk) {
                    if (reward_hit(p, blk)) *reward = p.reward_value;
                    w[s.idx] = AIR;
                    return s.idx;
                } else if (place && prev >= 0) {
                    w[prev] = DIRT;
                    return prev;
                }
                return -1;
            }
            prev = s.idx;
        }
    }
    return -1;
}

// The same interaction with the 32 samples spread over the 32 lanes of a
// warp: the first in-bounds solid sample is the lowest set bit of a ballot
// and the placement voxel is the highest in-bounds sample below it, which is
// exactly what the reference's sequential loop selects.  Must be called by
// all 32 lanes.  Returns the in-env index written (-1 if none), uniform
// across the warp; *mod_val gets the value written.
__device__ __forceinline__ int interact_warp(int8_t* w, const Agent& a, bool brk, bool place,
                                             const mc_kp& p, int lane, float* reward, int8_t* mod_val) {
    *reward = 0.0f;
    *mod_val = 0;
    if (!brk && !place) return -1;  // warp-uniform
    float dx, dy, dz;
    interact_dir(a, dx, dy, dz);
    Sample s = interact_sample(lane, a.x, N::add(a.y, 1.6f), a.z, dx, dy, dz, p.wx, p.wy, p.wz);
    int8_t blk = (s.inb && in_bounds(s.idx, (long long)p.wx * p.wy * p.wz, MC_SITE_INTERACT)) ? w[s.idx] : AIR;
    unsigned solid = __ballot_sync(0xffffffffu, s.inb && blk >= 0);
    unsigned inbm = __ballot_sync(0xffffffffu, s.inb);
    if (solid == 0u) return -1;
    int first = __ffs(solid) - 1;
    if (brk) {
        int8_t hb = (int8_t)__shfl_sync(0xffffffffu, (int)blk, first);
        int hidx = __shfl_sync(0xffffffffu, s.idx, first);
        if (reward_hit(p, hb)) *reward = p.reward_value;
        if (lane == first) w[s.idx] = AIR;
        *mod_val = AIR;
        return hidx;
    }
    unsigned before = inbm & ((1u << first) - 1u);
    if (before == 0u) return -1;
    int pl = 31 - __clz(before);
    int pidx = __shfl_sync(0xffffffffu, s.idx, pl);
    if (lane == pl) w[s.idx] = DIRT;
    *mod_val = DIRT;
    return pidx;
}

// ---------------------------------------------------------------------------
// Render: per-env camera constants
// ---------------------------------------------------------------------------
struct Cam {
    float eye_x, eye_y, eye_z;
    float fx, fy, fz, rx, rz, ux, uy, uz;  // forward, right (x, z), up
    float sy, cy, cp;                      // sin/cos yaw, cos pitch (TRIG ray pattern)
};

// Per-env constants of the DDA set-up: the eye's voxel and, per axis, the
// distance numerators to its upper and lower faces, (v+1) - eye and v - eye.
struct Dda0 {
    int vx, vy, vz;
    float nxp, nxm, nyp, nym, nzp, nzm;
};
__device__ __forceinline__ Dda0 dda0(const Cam& c) {
    Dda0 d;
    d.vx = (int)floorf(c.eye_x);
    d.vy = (int)floorf(c.eye_y);
    d.vz = (int)floorf(c.eye_z);
    d.nxp = N::sub((float)(d.vx + 1), c.eye_x);
    d.nxm = N::sub((float)d.vx, c.eye_x);
    d.nyp = N::sub((float)(d.vy + 1), c.eye_y);
    d.nym = N::sub((float)d.vy, c.eye_y);
    d.nzp = N::sub((float)(d.vz + 1), c.eye_z);
    d.nzm = N::sub((float)d.vz, c.eye_z);
    return d;
}

// Camera basis as the per-pixel code of render_kernel / _uint8 / _minimal /
// _fp16 / _fast computes it (kernels.cu:113-136): cosf/sinf of yaw/pitch.
// Pure function of the camera, so computing it once per env gives the bits
// every pixel of the reference computes.
__device__ __forceinline__ Cam cam_trig(float cx, float cy, float cz, float yaw, float pitch) {
    Cam c;
    c.eye_x = cx;
    c.eye_y = N::add(cy, 1.6f);
    c.eye_z = cz;
    float cos_yaw = N::cos(yaw);
    float sin_yaw = N::sin(yaw);
    float cos_pitch = N::cos(pitch);
    float sin_pitch = N::sin(pitch);
    c.fx = N::mul(sin_yaw, cos_pitch);
    c.fy = sin_pitch;
    c.fz = N::mul(cos_yaw, cos_pitch);
    c.rx = cos_yaw;
    c.rz = -sin_yaw;
    c.ux = N::mul(-sin_yaw, sin_pitch);
    c.uy = cos_pitch;
    c.uz = N::mul(-cos_yaw, sin_pitch);
    c.sy = sin_yaw;
    c.cy = cos_yaw;
    c.cp = cos_pitch;
    return c;
}

// Ray direction before normalisation, forward + u*right + v*up.  Where the
// reference computes the basis in the same kernel (TRIG: shaded, minimal,
// fp16) its compiler fuses the forward product: fma(v, up, fma(sin, cos,
// u*right)); where the basis is loaded (prebasis) it fuses u*right:
// fma(v, up, fma(u, right, forward)).
template <bool TRIG>
__device__ __forceinline__ void ray_dir(const Cam& c, float u, float v, float& x, float& y, float& z) {
    if (TRIG) {
        x = N::mad(v, c.ux, N::mad(c.sy, c.cp, N::mul(u, c.rx)));
        z = N::mad(v, c.uz, N::mad(c.cy, c.cp, N::mul(u, c.rz)));
    } else {
        x = N::mad(v, c.ux, N::mad(u, c.rx, c.fx));
        z = N::mad(v, c.uz, N::mad(u, c.rz, c.fz));
    }
    y = N::mad(v, c.uy, c.fy);
}

// |ray|^2 = fma(z, z, fma(y, y, x*x))
__device__ __forceinline__ float len2(float x, float y, float z) { return N::mad(z, z, N::mad(y, y, N::mul(x, x))); }

// precompute_camera_basis_kernel (kernels.cu:511-561), all 13 written words.
__device__ __forceinline__ void basis_compute(float cx, float cy, float cz, float yaw, float pitch,
                                              int width, int height, float fov, float out[13]) {
    float sin_yaw, cos_yaw, sin_pitch, cos_pitch;
    N::sincos_i(yaw, &sin_yaw, &cos_yaw);
    N::sincos_i(pitch, &sin_pitch, &cos_pitch);
    float fov_rad = N::mul(fov, 0.01745329f);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    float aspect = N::div((float)width, (float)height);
    out[0] = cx;
    out[1] = N::add(cy, 1.6f);
    out[2] = cz;
    out[3] = N::mul(sin_yaw, cos_pitch);
    out[4] = sin_pitch;
    out[5] = N::mul(cos_yaw, cos_pitch);
    out[6] = cos_yaw;
    out[7] = -sin_yaw;
    out[8] = N::mul(-sin_yaw, sin_pitch);
    out[9] = cos_pitch;
    out[10] = N::mul(-cos_yaw, sin_pitch);
    out[11] = N::mul(half_fov, aspect);
    out[12] = half_fov;
}

// scale_u / scale_v of precompute_camera_basis_kernel (kernels.cu:541-559);
// they do not depend on the camera.
__device__ __forceinline__ void prebasis_scales(int width, int height, float fov, float* su, float* sv) {
    float fov_rad = N::mul(fov, 0.01745329f);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    float aspect = N::div((float)width, (float)height);
    *su = N::mul(half_fov, aspect);
    *sv = half_fov;
}

__device__ __forceinline__ Cam cam_from_basis(const float* b) {
    Cam c;
    c.eye_x = b[0]; c.eye_y = b[1]; c.eye_z = b[2];
    c.fx = b[3]; c.fy = b[4]; c.fz = b[5];
    c.rx = b[6]; c.rz = b[7];
    c.ux = b[8]; c.uy = b[9]; c.uz = b[10];
    c.sy = 0.0f; c.cy = 0.0f; c.cp = 0.0f;  // unused by the prebasis ray pattern
    return c;
}

// Per-column u and per-row v of each family.  They depend only on the pixel
// coordinate and launch constants, so the fused kernel tabulates them.
// Shaded family: kernels.cu:129-134 (fov_rad = fov * 3.14159265 / 180).
__device__ __forceinline__ float u_shaded(int px, int width, int height, float fov) {
    float fov_rad = N::div(N::mul(fov, 3.14159265f), 180.0f);
    float aspect = N::div((float)width, (float)height);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    float a = N::div_sub1(N::mul(2.0f, N::add((float)px, 0.5f)), (float)width);
    return N::mul(N::mul(a, half_fov), aspect);
}
__device__ __forceinline__ float v_shaded(int py, int height, float fov) {
    float fov_rad = N::div(N::mul(fov, 3.14159265f), 180.0f);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    return N::mul(N::one_sub_div(N::mul(2.0f, N::add((float)py, 0.5f)), (float)height), half_fov);
}
// Minimal/fp16 family: kernels.cu:1029-1034 (fov_rad = fov * 0.01745329).
__device__ __forceinline__ float u_minimal(int px, int width, int height, float fov) {
    float fov_rad = N::mul(fov, 0.01745329f);
    float aspect = N::div((float)width, (float)height);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    float a = N::div_sub1(N::mul(2.0f, N::add((float)px, 0.5f)), (float)width);
    return N::mul(N::mul(a, half_fov), aspect);
}
__device__ __forceinline__ float v_minimal(int py, int height, float fov) {
    float fov_rad = N::mul(fov, 0.01745329f);
    float half_fov = N::tan(N::mul(fov_rad, 0.5f));
    return N::mul(N::one_sub_div(N::mul(2.0f, N::add((float)py, 0.5f)), (float)height), half_fov);
}
// Prebasis family: kernels.cu:616-617 (scales from the basis).
__device__ __forceinline__ float u_prebasis(int px, int width, float scale_u) {
    return N::mul(N::div_sub1(N::mul(2.0f, N::add((float)px, 0.5f)), (float)width), scale_u);
}
__device__ __forceinline__ float v_prebasis(int py, int height, float scale_v) {
    return N::mul(N::one_sub_div(N::mul(2.0f, N::add((float)py, 0.5f)), (float)height), scale_v);
}

// Voxel sources for the ray march.  at(idx, n): the voxel at idx of a world
// of n voxels (bounds-checked in the debug build).
struct VoxGlobal {
    const int8_t* w;
    __device__ __forceinline__ int8_t operator()(int idx) const { return w[idx]; }
    __device__ __forceinline__ int8_t at(int idx, int n) const {
        return in_bounds(idx, n, MC_SITE_MARCH_GLOBAL) ? w[idx] : (int8_t)-1;
    }
};
struct VoxLdg {  // read-only world (plain render kernels): the reference's __ldg path
    const int8_t* w;
    __device__ __forceinline__ int8_t operator()(int idx) const { return __ldg(w + idx); }
    __device__ __forceinline__ int8_t at(int idx, int n) const {
        return in_bounds(idx, n, MC_SITE_MARCH_GLOBAL) ? __ldg(w + idx) : (int8_t)-1;
    }
};
struct VoxShared {
    const int8_t* w;
    __device__ __forceinline__ int8_t operator()(int idx) const { return w[idx]; }
    __device__ __forceinline__ int8_t at(int idx, int n) const {
        return in_bounds(idx, n, MC_SITE_MARCH_SHARED) ? w[idx] : (int8_t)-1;
    }
};
// Either source behind one generic pointer (one call site for both), with a
// per-env flag telling whether it points into shared memory.
struct VoxEither {
    const int8_t* w;
    bool smem;
    __device__ __forceinline__ int8_t operator()(int idx) const { return w[idx]; }
    __device__ __forceinline__ int8_t at(int idx, int n) const {
        return in_bounds(idx, n, smem ? MC_SITE_MARCH_SHARED : MC_SITE_MARCH_GLOBAL) ? w[idx] : (int8_t)-1;
    }
};

struct Hit {
    int blk;    // block id, -1 for sky
    int face;   // -1 none, 0 x, 1 y, 2 z
    float t;    // entry distance of the hit voxel (shaded family only)
    int step_y; // sign of the ray's y (shaded shade rule)
};

#if MC_NUMERICS_FAST
#define MC_PTX_FTZ ".ftz"
#else
#define MC_PTX_FTZ ""
#endif

// Packed march over a world staged in shared memory (the packed form of
// shade_ray's branch-free march).  `packed` holds the voxel index in bits
// 18.. and three 6-bit in-box step counts that set bit 5 of their field when
// the ray leaves the box; p{x,y,z} move index and count of one axis.  Per
// iteration the axis of the reference's if / else-if / else choice
// (kernels.cu:239-255) is three compares whose predicates guard the index
// and distance updates directly (no selects), and the distance update comes
// after the voxel test, so at a hit tm still holds the entry distances the
// choice was made from: the caller recovers the axis and the distance t
// from them once per ray instead of carrying them through the loop.  The
// voxel is loaded before the exit test, so that one test covers both exits;
// the load of the step that leaves the box reads up to wx*wz bytes before or
// after the staged world, which the shared-memory layouts keep allocated
// (the value read there is not used).
// Returns the block hit (>= 0), or -1 when the ray left the box.
// The debug build's marches (below) also check every load address against
// `chk` (the staged world and one layer on either side: the march's own
// claim) and against the CTA's dynamic shared memory.
struct SmemRange {
    uint32_t lo, span;  // shared-memory addresses [lo, lo + span)
};
__device__ __forceinline__ SmemRange staged_range(uint32_t base, int wxz, int nvox) {
    return SmemRange{base - (uint32_t)wxz, (uint32_t)(nvox + 2 * wxz)};
}
#if MC_CHECK_BOUNDS
extern __shared__ __align__(16) uint8_t mc_dyn_smem[];
__device__ __forceinline__ SmemRange dyn_smem_range() {
    uint32_t n;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(n));
    return SmemRange{(uint32_t)__cvta_generic_to_shared(mc_dyn_smem), n};
}
// A failed check of a PTX march's load address a: which range it left.
__device__ __noinline__ void march_bounds_fail(uint32_t a, SmemRange chk, int site) {
    const SmemRange d = dyn_smem_range();
    if (a - d.lo >= d.span) bounds_fail((long long)a - d.lo, d.span, MC_SITE_MARCH_SMEM);
    else bounds_fail((long long)a - chk.lo, chk.span, site);
}
#endif

__device__ __forceinline__ int march_packed_shared(uint32_t world, int packed, int px, int py, int pz, float& tmx,
                                                   float& tmy, float& tmz, float tdx, float tdy, float tdz,
                                                   SmemRange chk = SmemRange{0u, 0u}) {
    constexpr int kGuard = (32 << 12) | (32 << 6) | 32;
    int b;
#if MC_CHECK_BOUNDS
    const SmemRange dyn = dyn_smem_range();
    uint32_t bad = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred pa, pna, pbx, pzx, pby, pzy, pz, pq, pb1, pb2;\n\t"
        ".reg .b32 ra, rc;\n\t"
        ".reg .s32 rv;\n\t"
        "MC_CMARCH_LOOP:\n\t"
        "setp.lt" MC_PTX_FTZ ".f32 pa|pna, %1, %2;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pbx|pzx, %1, %3, pa;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pby|pzy, %2, %3, pna;\n\t"
        "or.pred pz, pzx, pzy;\n\t"
        "@pbx add.s32 %4, %4, %6;\n\t"
        "@pby add.s32 %4, %4, %7;\n\t"
        "@pz add.s32 %4, %4, %8;\n\t"
        "shr.s32 ra, %4, 18;\n\t"
        "add.s32 ra, ra, %10;\n\t"
        "sub.u32 rc, ra, %15;\n\t"
        "setp.ge.u32 pb1, rc, %16;\n\t"
        "sub.u32 rc, ra, %17;\n\t"
        "setp.ge.u32 pb2, rc, %18;\n\t"
        "or.pred pb1, pb1, pb2;\n\t"
        "@pb1 mov.u32 %5, ra;\n\t"
        "@pb1 mov.s32 %0, -2;\n\t"
        "@pb1 bra MC_CMARCH_END;\n\t"
        "ld.shared.s8 rv, [ra];\n\t"
        "lop3.b32 ra, %4, rv, %9, 0xA2;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "@pq bra MC_CMARCH_DONE;\n\t"
        "@pbx add.rn" MC_PTX_FTZ ".f32 %1, %1, %11;\n\t"
        "@pby add.rn" MC_PTX_FTZ ".f32 %2, %2, %12;\n\t"
        "@pz add.rn" MC_PTX_FTZ ".f32 %3, %3, %13;\n\t"
        "bra MC_CMARCH_LOOP;\n\t"
        "MC_CMARCH_DONE:\n\t"
        "and.b32 ra, %4, %14;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "selp.b32 %0, -1, rv, pq;\n\t"
        "MC_CMARCH_END:\n\t"
        "}"
        : "=&r"(b), "+f"(tmx), "+f"(tmy), "+f"(tmz), "+r"(packed), "+r"(bad)
        : "r"(px), "r"(py), "r"(pz), "n"(kGuard | (int)0x80000000u), "r"(world), "f"(tdx), "f"(tdy), "f"(tdz),
          "n"(kGuard), "r"(chk.lo), "r"(chk.span), "r"(dyn.lo), "r"(dyn.span)
        : "memory");
    if (b == -2) {  // a load address outside its range: the load was skipped, the ray ends as sky
        march_bounds_fail(bad, chk, MC_SITE_MARCH_PACKED);
        b = -1;
    }
    return b;
#else
    (void)chk;
    asm volatile(
        "{\n\t"
        ".reg .pred pa, pna, pbx, pzx, pby, pzy, pz, pq;\n\t"
        ".reg .b32 ra;\n\t"
        ".reg .s32 rv;\n\t"
        "MC_MARCH_LOOP:\n\t"
        "setp.lt" MC_PTX_FTZ ".f32 pa|pna, %1, %2;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pbx|pzx, %1, %3, pa;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pby|pzy, %2, %3, pna;\n\t"
        "or.pred pz, pzx, pzy;\n\t"
        "@pbx add.s32 %4, %4, %5;\n\t"
        "@pby add.s32 %4, %4, %6;\n\t"
        "@pz add.s32 %4, %4, %7;\n\t"
        "shr.s32 ra, %4, 18;\n\t"
        "add.s32 ra, ra, %9;\n\t"
        "ld.shared.s8 rv, [ra];\n\t"
        // one test for both exits: a guard bit of the counts, or the sign
        // bit clear in the voxel (a block); c & (a | ~b) = lut 0xA2
        "lop3.b32 ra, %4, rv, %8, 0xA2;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "@pq bra MC_MARCH_DONE;\n\t"
        "@pbx add.rn" MC_PTX_FTZ ".f32 %1, %1, %10;\n\t"
        "@pby add.rn" MC_PTX_FTZ ".f32 %2, %2, %11;\n\t"
        "@pz add.rn" MC_PTX_FTZ ".f32 %3, %3, %12;\n\t"
        "bra MC_MARCH_LOOP;\n\t"
        "MC_MARCH_DONE:\n\t"
        "and.b32 ra, %4, %13;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "selp.b32 %0, -1, rv, pq;\n\t"
        "}"
        : "=&r"(b), "+f"(tmx), "+f"(tmy), "+f"(tmz), "+r"(packed)
        : "r"(px), "r"(py), "r"(pz), "n"(kGuard | (int)0x80000000u), "r"(world), "f"(tdx), "f"(tdy), "f"(tdz),
          "n"(kGuard)
        : "memory");
    return b;
#endif
}

// Where a ray going up from the eye's voxel (vx, vy, vz) can still meet a
// solid voxel, per quadrant q of the eye's column (bit 0: the x >= vx side,
// bit 1: the z >= vz side; each side includes the eye's own row): such a
// ray only visits voxels with y >= vy on its quadrant's sides, so once it
// is past the extreme x, the extreme z or the highest layer of the solid
// voxels there it meets none again and ends as sky, as the full march
// would.  One byte per quadrant: x = the largest x (x >= vx side) or the
// smallest (x <= vx side), z likewise, y = the highest layer + 1 (0: none).
struct UpBounds {
    uint32_t x, z, y;
};

// Bounds that cut nothing but the layers above ytop (every quadrant's x and
// z extremes at the box's faces).
__device__ __forceinline__ UpBounds up_none(int ytop) {
    return UpBounds{0xFF00FF00u, 0xFFFF0000u, (uint32_t)(min(max(ytop, -1), 254) + 1) * 0x01010101u};
}

// The highest solid layer at or above vy (-1: none), from the bounds: every
// solid voxel at or above the eye's layer lies in some quadrant.
__device__ __forceinline__ int up_top(const UpBounds& b) {
    return (int)max(max(b.y & 255u, (b.y >> 8) & 255u), max((b.y >> 16) & 255u, b.y >> 24)) - 1;
}

// In-box step counts of a march from the eye's voxel for ray sign
// combination k (bit 0: x >= 0, bit 1: y >= 0, bit 2: z >= 0): the steps
// left to each face of the box, cut for a ray going up by its quadrant's
// bounds; a count of -1 ends the ray (as sky) at its first step.
__device__ __forceinline__ void start_counts(int k, int vx, int vy, int vz, int wx, int wy, int wz,
                                             const UpBounds& ub, int& cx, int& cy, int& cz) {
    const bool px = k & 1, py = k & 2, pz = k & 4;
    cx = px ? wx - 1 - vx : vx;
    cy = py ? wy - 1 - vy : vy;
    cz = pz ? wz - 1 - vz : vz;
    if (py) {
        const int sh = 8 * ((px ? 1 : 0) | (pz ? 2 : 0));
        const int xe = (ub.x >> sh) & 255, ze = (ub.z >> sh) & 255, yt = (int)((ub.y >> sh) & 255) - 1;
        cx = max(min(cx, px ? xe - vx : vx - xe), -1);
        cz = max(min(cz, pz ? ze - vz : vz - ze), -1);
        cy = max(min(cy, yt - vy), -1);
    }
}

// Start values of march_packed_shared for an env whose eye is in voxel
// (vx, vy, vz), one per sign combination k of the ray (bit 0: x >= 0, bit 1:
// y >= 0, bit 2: z >= 0): {packed index and counts, x, y and z increments}.
// Counts from start_counts (at least -1, at most 31).
__device__ __forceinline__ int4 packed_start(int k, int vx, int vy, int vz, int wx, int wy, int wz,
                                             const UpBounds& ub) {
    const int sx = (k & 1) ? 1 : -1, sy = (k & 2) ? 1 : -1, sz = (k & 4) ? 1 : -1;
    const int wxz = wx * wz, idx = vy * wxz + vx * wz + vz;
    int cx, cy, cz;
    start_counts(k, vx, vy, vz, wx, wy, wz, ub, cx, cy, cz);
    return make_int4((idx << 18) | ((31 - cx) << 12) | ((31 - cy) << 6) | (31 - cz),
                     ((sx * wz) << 18) + (1 << 12), ((sy * wxz) << 18) + (1 << 6), (sz << 18) + 1);
}

// Counts of the split march: three 7-bit in-box step counts (z bits 0-6,
// x 7-13, y 14-20) that count up from 63 - (steps left) and set bit 6 of
// their field on leaving the box, and a 9-bit step count (bits 21-29) that
// sets its bit 8 when max_steps voxels have been stepped.  A count that
// starts at or above 64 (y of a ray going up from above `ytop`) ends the ray at
// its first step; clamping it to 126 keeps the carry out of the field.
constexpr int kSplitGuard = (1 << 6) | (1 << 13) | (1 << 20) | (1 << 29);
__device__ __forceinline__ int split_counts(int cx, int cy, int cz, int max_steps, int wx, int wy, int wz) {
    const int s0 = (max_steps > wx + wy + wz) ? 0 : 256 - max_steps;  // no ray takes more than wx+wy+wz steps
    return (63 - cz) | ((63 - cx) << 7) | ((63 - max(cy, -63)) << 14) | (s0 << 21);
}

// The march over a staged world of up to 64 voxels a side, any max_steps:
// the voxel's shared-memory address moves in one register and the counts
// (split_counts) in another, so a single mask tests every exit and the load
// needs no index arithmetic.  Axis choice, predicated updates and the
// distances left at a hit as in march_packed_shared.  Returns the block hit
// (>= 0), or -1 when the ray left the box or ran out of steps.
__device__ __forceinline__ int march_split_shared(uint32_t addr, int cnt, int dax, int day, int daz, float& tmx,
                                                  float& tmy, float& tmz, float tdx, float tdy, float tdz,
                                                  SmemRange chk = SmemRange{0u, 0u}) {
    int b;
#if MC_CHECK_BOUNDS
    const SmemRange dyn = dyn_smem_range();
    uint32_t bad = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred pa, pna, pbx, pzx, pby, pzy, pz, pq, pb1, pb2;\n\t"
        ".reg .b32 ra, rc;\n\t"
        ".reg .s32 rv;\n\t"
        "MC_CSPLIT_LOOP:\n\t"
        "setp.lt" MC_PTX_FTZ ".f32 pa|pna, %1, %2;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pbx|pzx, %1, %3, pa;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pby|pzy, %2, %3, pna;\n\t"
        "or.pred pz, pzx, pzy;\n\t"
        "@pbx add.s32 %4, %4, %7;\n\t"
        "@pby add.s32 %4, %4, %8;\n\t"
        "@pz add.s32 %4, %4, %9;\n\t"
        "@pbx add.s32 %5, %5, %10;\n\t"
        "@pby add.s32 %5, %5, %11;\n\t"
        "@pz add.s32 %5, %5, %12;\n\t"
        "sub.u32 rc, %4, %18;\n\t"
        "setp.ge.u32 pb1, rc, %19;\n\t"
        "sub.u32 rc, %4, %20;\n\t"
        "setp.ge.u32 pb2, rc, %21;\n\t"
        "or.pred pb1, pb1, pb2;\n\t"
        "@pb1 mov.u32 %6, %4;\n\t"
        "@pb1 mov.s32 %0, -2;\n\t"
        "@pb1 bra MC_CSPLIT_END;\n\t"
        "ld.shared.s8 rv, [%4];\n\t"
        "lop3.b32 ra, %5, rv, %13, 0xA2;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "@pq bra MC_CSPLIT_DONE;\n\t"
        "@pbx add.rn" MC_PTX_FTZ ".f32 %1, %1, %14;\n\t"
        "@pby add.rn" MC_PTX_FTZ ".f32 %2, %2, %15;\n\t"
        "@pz add.rn" MC_PTX_FTZ ".f32 %3, %3, %16;\n\t"
        "bra MC_CSPLIT_LOOP;\n\t"
        "MC_CSPLIT_DONE:\n\t"
        "and.b32 ra, %5, %17;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "selp.b32 %0, -1, rv, pq;\n\t"
        "MC_CSPLIT_END:\n\t"
        "}"
        : "=&r"(b), "+f"(tmx), "+f"(tmy), "+f"(tmz), "+r"(addr), "+r"(cnt), "+r"(bad)
        : "r"(dax), "r"(day), "r"(daz), "n"((1 << 7) | (1 << 21)), "n"((1 << 14) | (1 << 21)), "n"(1 | (1 << 21)),
          "n"(kSplitGuard | (int)0x80000000u), "f"(tdx), "f"(tdy), "f"(tdz), "n"(kSplitGuard), "r"(chk.lo),
          "r"(chk.span), "r"(dyn.lo), "r"(dyn.span)
        : "memory");
    if (b == -2) {
        march_bounds_fail(bad, chk, MC_SITE_MARCH_SPLIT);
        b = -1;
    }
    return b;
#else
    (void)chk;
    asm volatile(
        "{\n\t"
        ".reg .pred pa, pna, pbx, pzx, pby, pzy, pz, pq;\n\t"
        ".reg .b32 ra;\n\t"
        ".reg .s32 rv;\n\t"
        "MC_SPLIT_LOOP:\n\t"
        "setp.lt" MC_PTX_FTZ ".f32 pa|pna, %1, %2;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pbx|pzx, %1, %3, pa;\n\t"
        "setp.lt.and" MC_PTX_FTZ ".f32 pby|pzy, %2, %3, pna;\n\t"
        "or.pred pz, pzx, pzy;\n\t"
        "@pbx add.s32 %4, %4, %6;\n\t"
        "@pby add.s32 %4, %4, %7;\n\t"
        "@pz add.s32 %4, %4, %8;\n\t"
        "@pbx add.s32 %5, %5, %9;\n\t"
        "@pby add.s32 %5, %5, %10;\n\t"
        "@pz add.s32 %5, %5, %11;\n\t"
        "ld.shared.s8 rv, [%4];\n\t"
        // one test for both exits (as in march_packed_shared)
        "lop3.b32 ra, %5, rv, %12, 0xA2;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "@pq bra MC_SPLIT_DONE;\n\t"
        "@pbx add.rn" MC_PTX_FTZ ".f32 %1, %1, %13;\n\t"
        "@pby add.rn" MC_PTX_FTZ ".f32 %2, %2, %14;\n\t"
        "@pz add.rn" MC_PTX_FTZ ".f32 %3, %3, %15;\n\t"
        "bra MC_SPLIT_LOOP;\n\t"
        "MC_SPLIT_DONE:\n\t"
        "and.b32 ra, %5, %16;\n\t"
        "setp.ne.b32 pq, ra, 0;\n\t"
        "selp.b32 %0, -1, rv, pq;\n\t"
        "}"
        : "=&r"(b), "+f"(tmx), "+f"(tmy), "+f"(tmz), "+r"(addr), "+r"(cnt)
        : "r"(dax), "r"(day), "r"(daz), "n"((1 << 7) | (1 << 21)), "n"((1 << 14) | (1 << 21)), "n"(1 | (1 << 21)),
          "n"(kSplitGuard | (int)0x80000000u), "f"(tdx), "f"(tdy), "f"(tdz), "n"(kSplitGuard)
        : "memory");
    return b;
#endif
}

// March from the eye's voxel (index idx, in-box steps left cx, cy, cz) through
// a world staged at shared address `base`: the packed form where the world
// is small and every ray leaves the box before max_steps, else the split form.
__device__ __forceinline__ int march_staged(uint32_t base, int idx, int cx, int cy, int cz, int dix, int diy, int diz,
                                           int wx, int wy, int wz, int max_steps, float& tmx, float& tmy, float& tmz,
                                           float tdx, float tdy, float tdz) {
    const SmemRange chk = staged_range(base, wx * wz, wx * wy * wz);
    if (max_steps > wx + wy + wz && wx <= 31 && wy <= 31 && wz <= 31 && wx * wy * wz < 8192) {
        const int packed = (idx << 18) | ((31 - cx) << 12) | ((31 - max(cy, -32)) << 6) | (31 - cz);
        return march_packed_shared(base, packed, (dix << 18) + (1 << 12), (diy << 18) + (1 << 6), (diz << 18) + 1,
                                   tmx, tmy, tmz, tdx, tdy, tdz, chk);
    }
    return march_split_shared(base + idx, split_counts(cx, cy, cz, max_steps, wx, wy, wz), dix, diy, diz, tmx, tmy,
                              tmz, tdx, tdy, tdz, chk);
}

// Whether a march can run on the staged copy: V is a shared-memory source
// (or one flagged as such) and the world fits the counts' 64-voxel range.
template <class V>
__device__ __forceinline__ bool staged_source(const V& vox, int wx, int wy, int wz) {
    if constexpr (std::is_same<V, VoxShared>::value) {
        return wx <= 64 && wy <= 64 && wz <= 64;
    } else if constexpr (std::is_same<V, VoxEither>::value) {
        return vox.smem && wx <= 64 && wy <= 64 && wz <= 64;
    } else {
        (void)vox; (void)wx; (void)wy; (void)wz;
        return false;
    }
}
// The shared-memory address of a staged source (0 for the others, which
// staged_source turns away).
template <class V>
__device__ __forceinline__ uint32_t staged_base(const V& vox) {
    if constexpr (std::is_same<V, VoxShared>::value || std::is_same<V, VoxEither>::value) {
        return (uint32_t)__cvta_generic_to_shared(vox.w);
    } else {
        (void)vox;
        return 0u;
    }
}

// ray_intersects_aabb (kernels.cu:51-79) exit distance for a box [0, ws]^3
// given the precomputed numerators (0 - eye) and (ws - eye).
__device__ __forceinline__ float aabb_exit(float ix, float iy, float iz, float lo_x, float hi_x,
                                           float lo_y, float hi_y, float lo_z, float hi_z, float* t_entry) {
    float t1 = N::mul(lo_x, ix), t2 = N::mul(hi_x, ix);
    float t3 = N::mul(lo_y, iy), t4 = N::mul(hi_y, iy);
    float t5 = N::mul(lo_z, iz), t6 = N::mul(hi_z, iz);
    *t_entry = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
    return fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
}

// Shaded ray: ray setup, AABB early-out and DDA of render_kernel /
// render_kernel_uint8 (kernels.cu:137-269) and, with FASTG, the ground
// shortcut of render_kernel_uint8_fast (kernels.cu:1378-1405).  The
// reference's cubic box [0, ws]^3 becomes [0,wx]x[0,wy]x[0,wz], which is the
// same arithmetic when the world is cubic.  `inside` is a per-env flag: eye
// strictly inside the box and view_distance >= 0;
// then the AABB test always passes (t_entry < 0 <= view_distance) and its
// exit distance is only computed if the march leaves the world.
// With `skip_first` (a per-env fact: the eye is inside the world, its voxel
// holds air, view_distance > 0 and max_steps >= 1, and for FASTG the eye is
// at or above the ground) the first loop iteration is known to advance
// without a hit, so its tests are skipped.
//
// With `sky_exit` (per env: `inside`, no ground shortcut, and the caller does
// not need the face and distance of sky pixels, only their colour) the march stops as soon as
// the ray leaves the box: voxel coordinates move monotonically, so a ray that
// left never re-enters, and the reference, which keeps stepping until it is
// past the exit distance, also ends it as sky.  The axis is then chosen with
// selects instead of branches, and the box is tracked with per-axis counts of
// the in-box steps left.  With `vd_safe` (per env: every in-box voxel is
// entered closer than view_distance) the march has no distance test.  In
// both, `ytop` (per env: no solid voxel above this layer) ends rays going up
// once they pass it, as sky.
// VDLIM = false leaves out the branch-free march for view-limited worlds
// (those then take the reference-shaped loop), for callers whose register
// budget is better spent elsewhere.
// TAB: the caller passes `start`, the packed march's start values for the
// eight sign combinations of the ray (packed_starts), whenever the packed
// march applies to the env (nullptr otherwise).
template <bool FASTG, class V, bool VDLIM = true, bool TAB = false>
__device__ __forceinline__ Hit shade_ray(const Cam& c, const Dda0& d0, float u, float v, const V& vox, int wx, int wy,
                                         int wz, int max_steps, float vd, int gh, bool inside,
                                         bool skip_first = false, bool sky_exit = false, bool vd_safe = false,
                                         int ytop = 1 << 20, const int4* start = nullptr) {
    float ray_x, ray_y, ray_z;
    ray_dir<true>(c, u, v, ray_x, ray_y, ray_z);
    float ray_len = N::sqrt(len2(ray_x, ray_y, ray_z));
    const float rl = N::rcp_of(ray_len);
    ray_x = N::div_r(ray_x, ray_len, rl);
    ray_y = N::div_r(ray_y, ray_len, rl);
    ray_z = N::div_r(ray_z, ray_len, rl);

    float ix = (ray_x != 0.0f) ? N::div(1.0f, ray_x) : 1e30f;
    float iy = (ray_y != 0.0f) ? N::div(1.0f, ray_y) : 1e30f;
    float iz = (ray_z != 0.0f) ? N::div(1.0f, ray_z) : 1e30f;
    float lo_x = N::sub(0.0f, c.eye_x), hi_x = N::sub((float)wx, c.eye_x);
    float lo_y = N::sub(0.0f, c.eye_y), hi_y = N::sub((float)wy, c.eye_y);
    float lo_z = N::sub(0.0f, c.eye_z), hi_z = N::sub((float)wz, c.eye_z);

    Hit h;
    h.step_y = (ray_y >= 0) ? 1 : -1;
    h.blk = AIR;
    h.face = -1;
    h.t = 0.0f;
    float t_exit = 0.0f;
    bool have_exit = false;
    if (!inside) {
        float t_entry;
        t_exit = aabb_exit(ix, iy, iz, lo_x, hi_x, lo_y, hi_y, lo_z, hi_z, &t_entry);
        have_exit = true;
        if (t_exit < 0 || t_entry > t_exit || t_entry > vd) return h;  // sky
    }
    int vx = d0.vx, vy = d0.vy, vz = d0.vz;
    int sx = (ray_x >= 0) ? 1 : -1;
    int sy = h.step_y;
    int sz = (ray_z >= 0) ? 1 : -1;
    float tdx = fabsf(ix), tdy = fabsf(iy), tdz = fabsf(iz);
    float tmx = N::mul((ray_x >= 0) ? d0.nxp : d0.nxm, ix);
    float tmy = N::mul((ray_y >= 0) ? d0.nyp : d0.nym, iy);
    float tmz = N::mul((ray_z >= 0) ? d0.nzp : d0.nzm, iz);
    float t = 0.0f;
    int face = -1;
    const int wxz = wx * wz;
    const int nvox = wxz * wy;  // for the debug build's checks
    // linear voxel index kept in step with (vx, vy, vz)
    int idx = vy * wxz + vx * wz + vz;
    const int dix = sx * wz, diy = sy * wxz, diz = sz;
    int step = 0;
    if constexpr (std::is_same<V, VoxShared>::value || std::is_same<V, VoxEither>::value) {
        bool staged = true;
        if constexpr (std::is_same<V, VoxEither>::value) staged = vox.smem;
        if (!FASTG && sky_exit && staged && max_steps > 0 && wx <= 64 && wy <= 64 && wz <= 64) {
            // A staged world and the eye inside the box: the PTX marches.
            // They test view_distance once, at the hit: t never decreases
            // along the ray, so a first hit closer than view_distance is the
            // reference's hit, and a first hit at or beyond it means the
            // reference had already ended the ray as sky (its `t >= vd`
            // break); a ray that leaves the box or runs out of steps is sky
            // in both.
            int b = skip_first ? (int)AIR : (int)vox.at(idx, nvox);
            // a ray going up stops above ytop (no solid voxel lies higher): it ends as sky
            const int cx = (sx > 0) ? wx - 1 - vx : vx, cy = (sy > 0) ? min(wy - 1, ytop) - vy : vy,
                      cz = (sz > 0) ? wz - 1 - vz : vz;
            if (b < 0) {
                const uint32_t base = (uint32_t)__cvta_generic_to_shared(vox.w);
                if (TAB && start) {
                    // the env's start values for this ray's signs
                    const int4 e = start[(ray_x >= 0.0f ? 1 : 0) | (ray_y >= 0.0f ? 2 : 0) | (ray_z >= 0.0f ? 4 : 0)];
                    b = march_packed_shared(base, e.x, e.y, e.z, e.w, tmx, tmy, tmz, tdx, tdy, tdz,
                                            staged_range(base, wxz, nvox));
                } else if (vd_safe && max_steps > wx + wy + wz && wx <= 31 && wy <= 31 && wz <= 31 &&
                           wx * wy * wz < 8192) {
                    // index and in-box counts in one register (march_packed_shared)
                    const int packed = (idx << 18) | ((31 - cx) << 12) | ((31 - max(cy, -32)) << 6) | (31 - cz);
                    b = march_packed_shared(base, packed, (dix << 18) + (1 << 12), (diy << 18) + (1 << 6),
                                            (diz << 18) + 1, tmx, tmy, tmz, tdx, tdy, tdz,
                                            staged_range(base, wxz, nvox));
                } else {
                    b = march_split_shared(base + idx, split_counts(cx, cy, cz, max_steps, wx, wy, wz), dix, diy,
                                           diz, tmx, tmy, tmz, tdx, tdy, tdz, staged_range(base, wxz, nvox));
                }
                if (b >= 0) {
                    // the axis of the last step, chosen again from the same distances
                    const bool bx = tmx < tmy && tmx < tmz;
                    const bool by = !bx && tmy < tmz;
                    t = bx ? tmx : (by ? tmy : tmz);
                    face = bx ? 0 : (by ? 1 : 2);
                    if (t >= vd) b = AIR;
                }
            }
            h.blk = (b >= 0) ? b : AIR;
            h.face = face;
            h.t = t;
            return h;
        }
    }
    if (!FASTG && sky_exit && vd_safe && max_steps > 0) {
        // The same march with no distance test and no branch per axis: the
        // reference's if / else-if / else choice of axis (kernels.cu:239-255)
        // is made with selects, so lanes stepping different axes do not take
        // turns; one test per iteration ends the loop (hit, left the box, or
        // max_steps).  The eye's voxel is inside the box.
        int8_t b = AIR;
        if (!skip_first && max_steps > 0) b = vox.at(idx, nvox);
        bool lbx = false, lby = false, adv = false;
        // a ray going up stops above ytop (no solid voxel lies higher): it ends as sky
        int cx = (sx > 0) ? wx - 1 - vx : vx, cy = (sy > 0) ? min(wy - 1, ytop) - vy : vy,
            cz = (sz > 0) ? wz - 1 - vz : vz;
        if (max_steps > wx + wy + wz && wx <= 31 && wy <= 31 && wz <= 31 && wx * wy * wz < 8192) {
            // every ray leaves the box before max_steps: no step count.  The
            // voxel index and the three in-box counts share one register:
            // bits 18.. the index, three 6-bit fields below it counting up
            // from 31 - (steps left) to 32, whose bit 5 marks leaving the
            // box; one add moves both, one mask tests the exit.
            const int fx = 31 - cx, fy = 31 - max(cy, -32), fz = 31 - cz;
            int packed = (idx << 18) | (fx << 12) | (fy << 6) | fz;
            const int px = (dix << 18) + (1 << 12), py = (diy << 18) + (1 << 6), pz = (diz << 18) + 1;
            constexpr int kGuard = (32 << 12) | (32 << 6) | 32;
            while (b < 0) {
                const bool bx = tmx < tmy && tmx < tmz;
                const bool by = !bx && tmy < tmz;
                const bool bz = !bx && !by;
                t = bx ? tmx : (by ? tmy : tmz);
                // three adds (FMA pipe) instead of selecting the delta (ALU pipe,
                // the busier one); only the chosen axis keeps its sum
                const float nx = N::add(tmx, tdx), ny = N::add(tmy, tdy), nz = N::add(tmz, tdz);
                tmx = bx ? nx : tmx;
                tmy = by ? ny : tmy;
                tmz = bz ? nz : tmz;
                packed += bx ? px : (by ? py : pz);
                lbx = bx;
                lby = by;
                adv = true;
                if (packed & kGuard) break;
                b = vox.at(packed >> 18, nvox);
            }
        } else {
            while (b < 0 && max_steps > 0) {
                const bool bx = tmx < tmy && tmx < tmz;
                const bool by = !bx && tmy < tmz;
                const bool bz = !bx && !by;
                t = bx ? tmx : (by ? tmy : tmz);
                const float nx = N::add(tmx, tdx), ny = N::add(tmy, tdy), nz = N::add(tmz, tdz);
                tmx = bx ? nx : tmx;
                tmy = by ? ny : tmy;
                tmz = bz ? nz : tmz;
                cx -= bx ? 1 : 0;
                cy -= by ? 1 : 0;
                cz -= bz ? 1 : 0;
                idx += bx ? dix : (by ? diy : diz);
                lbx = bx;
                lby = by;
                adv = true;
                if ((cx | cy | cz) < 0 || ++step >= max_steps) break;
                b = vox.at(idx, nvox);
            }
        }
        if (adv) face = lbx ? 0 : (lby ? 1 : 2);
        h.blk = (b >= 0) ? (int)b : AIR;
        h.face = face;
        h.t = t;
        return h;
    }
    if (VDLIM && !FASTG && sky_exit && max_steps > 0) {
        // the same branch-free march with the distance test and the step
        // count in its single exit test (worlds whose far corners lie beyond
        // view_distance)
        int8_t b = AIR;
        if (!skip_first) b = vox.at(idx, nvox);
        bool lbx = false, lby = false, adv = false;
        // a ray going up stops above ytop (no solid voxel lies higher): it ends as sky
        int cx = (sx > 0) ? wx - 1 - vx : vx, cy = (sy > 0) ? min(wy - 1, ytop) - vy : vy,
            cz = (sz > 0) ? wz - 1 - vz : vz;
        while (b < 0) {
            const bool bx = tmx < tmy && tmx < tmz;
            const bool by = !bx && tmy < tmz;
            const bool bz = !bx && !by;
            t = bx ? tmx : (by ? tmy : tmz);
            const float nx = N::add(tmx, tdx), ny = N::add(tmy, tdy), nz = N::add(tmz, tdz);
            tmx = bx ? nx : tmx;
            tmy = by ? ny : tmy;
            tmz = bz ? nz : tmz;
            cx -= bx ? 1 : 0;
            cy -= by ? 1 : 0;
            cz -= bz ? 1 : 0;
            idx += bx ? dix : (by ? diy : diz);
            lbx = bx;
            lby = by;
            adv = true;
            if ((cx | cy | cz) < 0 || ++step >= max_steps || t >= vd) break;
            b = vox.at(idx, nvox);
        }
        if (adv) face = lbx ? 0 : (lby ? 1 : 2);
        h.blk = (b >= 0) ? (int)b : AIR;
        h.face = face;
        h.t = t;
        return h;
    }
    if (skip_first) {
        if (tmx < tmy && tmx < tmz) {
            t = tmx; tmx = N::add(tmx, tdx); vx += sx; idx += dix; face = 0;
        } else if (tmy < tmz) {
            t = tmy; tmy = N::add(tmy, tdy); vy += sy; idx += diy; face = 1;
        } else {
            t = tmz; tmz = N::add(tmz, tdz); vz += sz; idx += diz; face = 2;
        }
        step = 1;
    }
    for (; step < max_steps; ++step) {
        if (t >= vd) break;
        if (FASTG && vy < gh) {
            h.blk = (vy == gh - 1) ? GRASS : DIRT;
            break;
        }
        if ((unsigned)vx < (unsigned)wx && (unsigned)vy < (unsigned)wy && (unsigned)vz < (unsigned)wz) {
            int8_t b = vox.at(idx, nvox);
            if (b >= 0) {
                h.blk = b;
                break;
            }
        } else {
            if (!have_exit) {
                float t_entry;
                t_exit = aabb_exit(ix, iy, iz, lo_x, hi_x, lo_y, hi_y, lo_z, hi_z, &t_entry);
                have_exit = true;
            }
            if (t > t_exit) break;
        }
        if (tmx < tmy && tmx < tmz) {
            t = tmx; tmx = N::add(tmx, tdx); vx += sx; idx += dix; face = 0;
        } else if (tmy < tmz) {
            t = tmy; tmy = N::add(tmy, tdy); vy += sy; idx += diy; face = 1;
        } else {
            t = tmz; tmz = N::add(tmz, tdz); vz += sz; idx += diz; face = 2;
        }
    }
    h.face = face;
    h.t = t;
    return h;
}

// Every voxel of the box is entered closer than view_distance (with a margin
// far above the rounding of the DDA's accumulated distances), so the march's
// distance test cannot end a ray inside the box.
__device__ __forceinline__ bool box_within_view(const Cam& c, int wx, int wy, int wz, float vd) {
    const float dx = fmaxf(c.eye_x, (float)wx - c.eye_x);
    const float dy = fmaxf(c.eye_y, (float)wy - c.eye_y);
    const float dz = fmaxf(c.eye_z, (float)wz - c.eye_z);
    const float m = vd - 1.0f;
    return m > 0.0f && dx * dx + dy * dy + dz * dz < m * m;
}

__device__ __forceinline__ bool eye_inside(const Cam& c, int wx, int wy, int wz, float vd) {
    return c.eye_x > 0.0f && c.eye_x < (float)wx && c.eye_y > 0.0f && c.eye_y < (float)wy &&
           c.eye_z > 0.0f && c.eye_z < (float)wz && vd >= 0.0f;
}

// Which product each channel's c*shade*(1-fog) + sky*fog fuses in the
// reference build (measured against its kernels): float32 render_kernel
// fuses sky*fog for red only; render_kernel_uint8 for red and green;
// render_kernel_uint8_fast for red only (MC_FASTG_SKY).  Bit k = channel k.
enum { MC_COL_F32 = 0, MC_COL_U8 = 1, MC_COL_U8FAST = 2 };
#ifndef MC_FASTG_SKY
#define MC_FASTG_SKY 0x1
#endif
__device__ __forceinline__ int sky_fused_mask(int kind) {
    return kind == MC_COL_F32 ? 0x1 : (kind == MC_COL_U8 ? 0x3 : MC_FASTG_SKY);
}

// Shading and fog of the shaded family (kernels.cu:271-292, 446-469).
template <int KIND>
__device__ __forceinline__ void shade_rgb(const Hit& h, float vd, float rcp_vd, const float (*rgb)[3], const float* sky,
                                          float out[3]) {
    if (h.blk >= 0 && in_bounds(h.blk, 13, MC_SITE_TABLE)) {
        float r = rgb[h.blk][0], g = rgb[h.blk][1], b_col = rgb[h.blk][2];
        float shade = 1.0f;
        if (h.face == 0) shade = 0.8f;
        else if (h.face == 2) shade = 0.9f;
        else if (h.face == 1 && h.step_y < 0) shade = 0.6f;
        float fog = fminf(N::div_r(h.t, vd, rcp_vd), 1.0f);
        fog = N::mul(fog, fog);
        float omf = N::sub(1.0f, fog);
        const int m = sky_fused_mask(KIND);
        const float c3[3] = {r, g, b_col};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float cs = N::mul(c3[k], shade);
            out[k] = ((m >> k) & 1) ? N::mad(sky[k], fog, N::mul(cs, omf)) : N::mad(cs, omf, N::mul(sky[k], fog));
        }
    } else {
        out[0] = sky[0];
        out[1] = sky[1];
        out[2] = sky[2];
    }
}

// (uint8_t)(x * 255) for x*255 in [0, 256): adding 2^23 with round-toward-
// zero leaves trunc(x*255) in the low mantissa bits, which is the C++
// float-to-integer conversion without using the conversion unit.
__device__ __forceinline__ uint32_t to_u8(float x) {
    return __float_as_uint(__fadd_rz(N::mul(x, 255.0f), 8388608.0f)) & 0xffu;
}

// Flat ray of render_kernel_uint8_minimal / _prebasis / _smem
// (kernels.cu:1036-1097, 619-679): rsqrtf normalisation, no AABB, no fog,
// unsigned bounds test, non-cubic world.
// With `sky_exit` (per env: the eye's voxel is inside the world, and the
// caller needs only the colour of sky pixels) the march stops when the ray
// leaves the box, where the reference keeps stepping out-of-box voxels until
// max_steps: a ray that left never re-enters, so both end as sky.
// TAB: `start` holds the packed march's start values per ray sign
// combination (packed_start) whenever every ray of the env takes the packed
// march, else nullptr.
template <bool TRIG, class V, bool TAB = false>
__device__ __forceinline__ Hit flat_ray(const Cam& c, const Dda0& d0, float u, float v, const V& vox, int wx, int wy,
                                        int wz, int max_steps, bool skip_first = false, bool sky_exit = false,
                                        int ytop = 1 << 20, const int4* start = nullptr) {
    float ray_x, ray_y, ray_z;
    ray_dir<TRIG>(c, u, v, ray_x, ray_y, ray_z);
    float ray_len = N::rsqrt(len2(ray_x, ray_y, ray_z));
    ray_x = N::mul(ray_x, ray_len);
    ray_y = N::mul(ray_y, ray_len);
    ray_z = N::mul(ray_z, ray_len);
    int wxz = wx * wz;
    const int nvox = wxz * wy;  // for the debug build's checks
    int vx = d0.vx, vy = d0.vy, vz = d0.vz;
    int sx = (ray_x >= 0) ? 1 : -1;
    int sy = (ray_y >= 0) ? 1 : -1;
    int sz = (ray_z >= 0) ? 1 : -1;
    float ix = (ray_x != 0.0f) ? N::div(1.0f, ray_x) : 1e30f;
    float iy = (ray_y != 0.0f) ? N::div(1.0f, ray_y) : 1e30f;
    float iz = (ray_z != 0.0f) ? N::div(1.0f, ray_z) : 1e30f;
    float tdx = fabsf(ix), tdy = fabsf(iy), tdz = fabsf(iz);
    float tmx = N::mul((ray_x >= 0) ? d0.nxp : d0.nxm, ix);
    float tmy = N::mul((ray_y >= 0) ? d0.nyp : d0.nym, iy);
    float tmz = N::mul((ray_z >= 0) ? d0.nzp : d0.nzm, iz);
    Hit h;
    h.blk = AIR;
    h.face = -1;
    h.t = 0.0f;
    h.step_y = sy;
    int face = -1;
    int idx = vy * wxz + vx * wz + vz;
    const int dix = sx * wz, diy = sy * wxz, diz = sz;
    if (sky_exit && max_steps > 0 && staged_source(vox, wx, wy, wz)) {
        // the PTX marches over the staged world (as in shade_ray, no view distance)
        int b = skip_first ? (int)AIR : (int)vox.at(idx, nvox);
        if (b < 0) {
            // a ray going up stops above ytop (no solid voxel lies higher): it ends as sky
            const int cx = (sx > 0) ? wx - 1 - vx : vx, cy = (sy > 0) ? min(wy - 1, ytop) - vy : vy,
                      cz = (sz > 0) ? wz - 1 - vz : vz;
            if (TAB && start) {
                const int4 e = start[(ray_x >= 0.0f ? 1 : 0) | (ray_y >= 0.0f ? 2 : 0) | (ray_z >= 0.0f ? 4 : 0)];
                b = march_packed_shared(staged_base(vox), e.x, e.y, e.z, e.w, tmx, tmy, tmz, tdx, tdy, tdz,
                                        staged_range(staged_base(vox), wxz, nvox));
            } else {
                b = march_staged(staged_base(vox), idx, cx, cy, cz, dix, diy, diz, wx, wy, wz, max_steps, tmx, tmy,
                                 tmz, tdx, tdy, tdz);
            }
            if (b >= 0) {
                const bool bx = tmx < tmy && tmx < tmz;
                face = bx ? 0 : ((tmy < tmz) ? 1 : 2);
            }
        }
        h.blk = (b >= 0) ? b : AIR;
        h.face = face;
        return h;
    }
    if (sky_exit) {
        // branch-free axis choice as in shade_ray; one exit test per iteration
        int8_t b = AIR;
        int step = 0;
        if (!skip_first && max_steps > 0) b = vox.at(idx, nvox);
        while (b < 0 && max_steps > 0) {
            const bool bx = tmx < tmy && tmx < tmz;
            const bool by = !bx && tmy < tmz;
            const bool bz = !bx && !by;
            const float nx = N::add(tmx, tdx), ny = N::add(tmy, tdy), nz = N::add(tmz, tdz);
            tmx = bx ? nx : tmx;
            tmy = by ? ny : tmy;
            tmz = bz ? nz : tmz;
            vx += bx ? sx : 0;
            vy += by ? sy : 0;
            vz += bz ? sz : 0;
            idx += bx ? dix : (by ? diy : diz);
            face = bx ? 0 : (by ? 1 : 2);
            const bool out = (unsigned)vx >= (unsigned)wx || (unsigned)vy >= (unsigned)wy || (unsigned)vz >= (unsigned)wz;
            if (out || ++step >= max_steps) break;
            b = vox.at(idx, nvox);
        }
        h.blk = (b >= 0) ? (int)b : AIR;
        h.face = face;
        return h;
    }
    for (int step = 0; step < max_steps; ++step) {
        // skip_first: the eye's voxel is known to be air or outside the world
        if ((step > 0 || !skip_first) &&
            (unsigned)vx < (unsigned)wx && (unsigned)vy < (unsigned)wy && (unsigned)vz < (unsigned)wz) {
            int8_t b = vox.at(idx, nvox);
            if (b >= 0) {
                h.blk = b;
                break;
            }
        }
        if (tmx < tmy && tmx < tmz) {
            tmx = N::add(tmx, tdx); vx += sx; idx += dix; face = 0;
        } else if (tmy < tmz) {
            tmy = N::add(tmy, tdy); vy += sy; idx += diy; face = 1;
        } else {
            tmz = N::add(tmz, tdz); vz += sz; idx += diz; face = 2;
        }
    }
    h.face = face;
    return h;
}

// render_kernel_uint8_fp16 (kernels.cu:1176-1248): the DDA's t_max/t_delta
// in binary16 (inverse 65504 for a zero component).
template <class V>
__device__ __forceinline__ Hit fp16_ray(const Cam& c, const Dda0& d0, float u, float v, const V& vox, int wx, int wy,
                                        int wz, int max_steps) {
    float ray_x, ray_y, ray_z;
    ray_dir<true>(c, u, v, ray_x, ray_y, ray_z);
    float ray_len = N::rsqrt(len2(ray_x, ray_y, ray_z));
    ray_x = N::mul(ray_x, ray_len);
    ray_y = N::mul(ray_y, ray_len);
    ray_z = N::mul(ray_z, ray_len);
    int wxz = wx * wz;
    const int nvox = wxz * wy;  // for the debug build's checks
    int vx = d0.vx, vy = d0.vy, vz = d0.vz;
    int sx = (ray_x >= 0) ? 1 : -1;
    int sy = (ray_y >= 0) ? 1 : -1;
    int sz = (ray_z >= 0) ? 1 : -1;
    float ixf = (ray_x != 0.0f) ? N::div(1.0f, ray_x) : 65504.0f;
    float iyf = (ray_y != 0.0f) ? N::div(1.0f, ray_y) : 65504.0f;
    float izf = (ray_z != 0.0f) ? N::div(1.0f, ray_z) : 65504.0f;
    __half tdx = __float2half(fabsf(ixf));
    __half tdy = __float2half(fabsf(iyf));
    __half tdz = __float2half(fabsf(izf));
    __half tmx = __float2half(N::mul((ray_x >= 0) ? d0.nxp : d0.nxm, ixf));
    __half tmy = __float2half(N::mul((ray_y >= 0) ? d0.nyp : d0.nym, iyf));
    __half tmz = __float2half(N::mul((ray_z >= 0) ? d0.nzp : d0.nzm, izf));
    Hit h;
    h.blk = AIR;
    h.face = -1;
    h.t = 0.0f;
    h.step_y = sy;
    int face = -1;
    for (int step = 0; step < max_steps; ++step) {
        if ((unsigned)vx < (unsigned)wx && (unsigned)vy < (unsigned)wy && (unsigned)vz < (unsigned)wz) {
            int8_t b = vox.at(vy * wxz + vx * wz + vz, nvox);
            if (b >= 0) {
                h.blk = b;
                break;
            }
        }
        if (__hlt(tmx, tmy) && __hlt(tmx, tmz)) {
            tmx = __hadd(tmx, tdx); vx += sx; face = 0;
        } else if (__hlt(tmy, tmz)) {
            tmy = __hadd(tmy, tdy); vy += sy; face = 1;
        } else {
            tmz = __hadd(tmz, tdz); vz += sz; face = 2;
        }
    }
    h.face = face;
    return h;
}

__device__ __forceinline__ int16_t dbg_code(const Hit& h) { return (int16_t)((h.blk + 1) | ((h.face + 1) << 8)); }

// ---------------------------------------------------------------------------
// Plain form: one kernel per reference kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ void flag_any(int32_t* flags, bool v) {
    unsigned m = __ballot_sync(__activemask(), v);
    if (m && (threadIdx.x & 31) == (__ffs(m) - 1)) atomicOr(&flags[MC_FLAG_ANY_DONE], 1);
}

__global__ void k_episode_check(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    bool done = p.ext_done ? (p.do_reset[i] != 0) : episode_done(p, p.step_count[i]);
    if (!p.ext_done) p.do_reset[i] = done ? 1 : 0;
    flag_any(p.flags, done);
}

__global__ void k_decode(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    int8_t b[8];
    float l0, l1;
    load_action(p, i, b, l0, l1);
    Dec d = decode_buttons(b, l0, l1, p.sprint_mult);
    p.s_fwd[i] = d.fwd;
    p.s_strafe[i] = d.strafe;
    p.s_dyaw[i] = d.dyaw;
    p.s_dpitch[i] = d.dpitch;
    p.s_jump[i] = d.jump;
    p.s_brk[i] = d.brk;
    p.s_place[i] = d.place;
    p.s_speed[i] = d.speed;
}

__device__ __forceinline__ Dec load_dec(const mc_kp& p, long long i) {
    Dec d;
    d.fwd = p.s_fwd[i];
    d.strafe = p.s_strafe[i];
    d.dyaw = p.s_dyaw[i];
    d.dpitch = p.s_dpitch[i];
    d.jump = p.s_jump[i] != 0;
    d.brk = p.s_brk[i] != 0;
    d.place = p.s_place[i] != 0;
    d.speed = p.s_speed[i];
    return d;
}

__global__ void k_physics(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    Agent a = load_agent(p, i);
    physics(a, load_dec(p, i), p);
    p.positions[i * 3 + 0] = a.x;
    p.positions[i * 3 + 1] = a.y;
    p.positions[i * 3 + 2] = a.z;
    p.velocities[i * 3 + 1] = a.vy;
    p.yaws[i] = a.yaw;
    p.pitches[i] = a.pitch;
    p.on_ground[i] = a.og ? 1 : 0;
}

// break_only: raycast_break_kernel (kernels.cu:1687-1753), no placement.
__global__ void k_interact(mc_kp p, int break_only) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    Agent a = load_agent(p, i);
    bool brk = p.s_brk[i] != 0;
    bool place = break_only ? false : (p.s_place[i] != 0);
    float reward;
    long long wxyz = (long long)p.wx * p.wy * p.wz;
    int idx = interact_seq(p.voxels + i * wxyz, a, brk, place, p, &reward);
    p.rewards[i] = reward;
    if (p.dbg_interact) p.dbg_interact[i] = idx;
}

__global__ void k_reset(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    if (p.do_reset[i]) {
        Agent a;
        reset_agent(a, p);
        store_agent(p, i, a);
    }
}

// episode_update_kernel (kernels.cu:1971-1986) == the Python counter update
// of minecu/__init__.py:435-436.
__global__ void k_episode_update(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B || p.ext_done) return;
    p.step_count[i] = p.do_reset[i] ? 1 : p.step_count[i] + 1;
}

// update_cameras_kernel (kernels.cu:2320-2335)
__global__ void k_cameras(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    p.cameras[i * 5 + 0] = p.positions[i * 3 + 0];
    p.cameras[i * 5 + 1] = p.positions[i * 3 + 1];
    p.cameras[i * 5 + 2] = p.positions[i * 3 + 2];
    p.cameras[i * 5 + 3] = p.yaws[i];
    p.cameras[i * 5 + 4] = p.pitches[i];
}

__global__ void k_basis(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    const float* cam = p.cameras + i * 5;
    float out[13];
    basis_compute(cam[0], cam[1], cam[2], cam[3], cam[4], p.W, p.H, p.fov, out);
#pragma unroll
    for (int k = 0; k < 13; ++k) p.basis[i * 14 + k] = out[k];
}

// Shaded render, one thread per pixel over B*H*W, as render_kernel /
// render_kernel_uint8 / render_kernel_uint8_fast (1-D grid, 128 threads).
template <bool FASTG, bool F32>
__global__ void __launch_bounds__(128) k_render_shaded(mc_kp p) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long hw = (long long)p.H * p.W;
    if (idx >= (long long)p.B * hw) return;
    long long b = idx / hw;
    int pix = (int)(idx - b * hw);
    int py = pix / p.W, px = pix - py * p.W;
    const float* cam = p.cameras + b * 5;
    Cam c = cam_trig(__ldg(cam + 0), __ldg(cam + 1), __ldg(cam + 2), __ldg(cam + 3), __ldg(cam + 4));
    bool inside = eye_inside(c, p.wx, p.wy, p.wz, p.vd);
    float u = u_shaded(px, p.W, p.H, p.fov);
    float v = v_shaded(py, p.H, p.fov);
    VoxLdg vox{p.voxels + b * (long long)p.wx * p.wy * p.wz};
    Hit h = shade_ray<FASTG>(c, dda0(c), u, v, vox, p.wx, p.wy, p.wz, p.max_steps, p.vd, p.gh, inside);
    float rgb[3];
    shade_rgb<F32 ? MC_COL_F32 : (FASTG ? MC_COL_U8FAST : MC_COL_U8)>(h, p.vd, N::rcp_of(p.vd), c_rgb, c_sky, rgb);
    if (F32) {
        float* o = (float*)p.obs + idx * 3;
        o[0] = rgb[0]; o[1] = rgb[1]; o[2] = rgb[2];
    } else {
        uint8_t* o = (uint8_t*)p.obs + idx * 3;
        o[0] = (uint8_t)to_u8(rgb[0]); o[1] = (uint8_t)to_u8(rgb[1]); o[2] = (uint8_t)to_u8(rgb[2]);
    }
    if (p.dbg_pixel) p.dbg_pixel[idx] = dbg_code(h);
}

// Flat render, one thread per pixel over B*H*W (minimal / fp16: per-pixel
// trig; prebasis: reads the [B,14] basis).  The reference launches the
// prebasis kernel on a 2-D grid (pixel blocks, env), which caps B at 65535;
// the per-pixel work is the same.
template <int FAM>
__global__ void __launch_bounds__(128) k_render_flat(mc_kp p) {
    long long hw = (long long)p.H * p.W;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)p.B * hw) return;
    long long b = idx / hw;
    int pix = (int)(idx - b * hw);
    int py = pix / p.W, px = pix - py * p.W;
    Cam c;
    float u, v;
    if (FAM == MC_FAM_PREBASIS) {
        const float* bs = p.basis + b * 14;
        float bb[13];
#pragma unroll
        for (int k = 0; k < 13; ++k) bb[k] = __ldg(bs + k);
        c = cam_from_basis(bb);
        u = u_prebasis(px, p.W, bb[11]);
        v = v_prebasis(py, p.H, bb[12]);
    } else {
        const float* cam = p.cameras + b * 5;
        c = cam_trig(__ldg(cam + 0), __ldg(cam + 1), __ldg(cam + 2), __ldg(cam + 3), __ldg(cam + 4));
        u = u_minimal(px, p.W, p.H, p.fov);
        v = v_minimal(py, p.H, p.fov);
    }
    long long wxyz = (long long)p.wx * p.wy * p.wz;
    VoxLdg vox{p.voxels + b * wxyz};
    Hit h;
    const Dda0 d0 = dda0(c);
    if (FAM == MC_FAM_FP16) h = fp16_ray(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps);
    else if (FAM == MC_FAM_PREBASIS) h = flat_ray<false>(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps);
    else h = flat_ray<true>(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps);
    long long o = (b * hw + pix);
    uint8_t* out = (uint8_t*)p.obs + o * 3;
    const uint8_t* col = (h.blk >= 0 && in_bounds(h.blk, 13, MC_SITE_TABLE)) ? c_rgb8[h.blk] : c_sky8;
    out[0] = col[0]; out[1] = col[1]; out[2] = col[2];
    if (p.dbg_pixel) p.dbg_pixel[o] = dbg_code(h);
}

// render_kernel_uint8_coalesced (kernels.cu:709-826): prebasis semantics over
// a [Y, X, Z, B] voxel layout, a warp = one pixel across 32 envs.
__global__ void __launch_bounds__(128) k_render_coalesced(const int8_t* vox, const float* basis, uint8_t* out,
                                                          int B, int ws, int W, int H, int max_steps) {
    int pix = blockIdx.x;
    int b = blockIdx.y * blockDim.x + threadIdx.x;
    if (pix >= H * W || b >= B) return;
    int py = pix / W, px = pix - py * W;
    float bb[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) bb[k] = __ldg(basis + (long long)b * 14 + k);
    Cam c = cam_from_basis(bb);
    float u = u_prebasis(px, W, bb[11]);
    float v = v_prebasis(py, H, bb[12]);
    struct VoxYXZB {
        const int8_t* v;
        int B, b, ws;
        __device__ __forceinline__ int8_t operator()(int idx) const {
            // idx = y*ws*ws + x*ws + z  ->  [y][x][z][b]
            return __ldg(v + (long long)idx * B + b);
        }
        __device__ __forceinline__ int8_t at(int idx, int n) const {
            return in_bounds(idx, n, MC_SITE_MARCH_GLOBAL) ? (*this)(idx) : (int8_t)-1;
        }
    } acc{vox, B, b, ws};
    Hit h = flat_ray<false>(c, dda0(c), u, v, acc, ws, ws, ws, max_steps);
    const uint8_t* col = (h.blk >= 0 && in_bounds(h.blk, 13, MC_SITE_TABLE)) ? c_rgb8[h.blk] : c_sky8;
    uint8_t* o = out + ((long long)b * H * W + pix) * 3;
    o[0] = col[0]; o[1] = col[1]; o[2] = col[2];
}

// ---------------------------------------------------------------------------
// Fused form: one persistent kernel per step, one warp per env
// ---------------------------------------------------------------------------
// Shared memory layout (per CTA): u/v tables, colour tables, then per warp a
// pixel staging buffer, an mbarrier and (stage=1) one world.  A warp marches
// one tile of tile_w x (32/tile_w) pixels per iteration (nearby rays have
// similar lengths, which keeps the lanes of the DDA loop together) and
// stages a band of 32/tile_w full image rows, written out contiguously.
struct FusedLayout {
    int W, H;
    int tile_w, tile_h;
    int stage_bytes;   // staging bytes per warp (one band of rows)
    int world_bytes;   // world bytes per warp (0 when not staged)
    int warp_bytes;    // total per warp (16-aligned)
    int head_bytes;    // tables (16-aligned)
    int pad_bytes;     // allocated after the last warp's world
};

__host__ __device__ inline int mc_align16(int x) { return (x + 15) & ~15; }

// Tables of the per-warp kernel's common-case render loop, at the start of
// its shared memory: per block and shade code the colour times the shade
// (13 x 4 float4), then per block the flat colour packed as r | g << 8 | b << 16.
constexpr int kShadeTableBytes = 13 * 4 * 16;
constexpr int kFastTableBytes = MC_FAST_TABLE_BYTES;
static_assert(kFastTableBytes == kShadeTableBytes + 64, "fast tables");

__host__ __device__ inline FusedLayout fused_layout(int W, int H, int wxyz, int wxz, int obs_f32, int stage,
                                                   int tile_w) {
    FusedLayout L;
    L.W = W;
    L.H = H;
    L.tile_w = tile_w;
    L.tile_h = 32 / tile_w;
    L.stage_bytes = mc_align16(W * L.tile_h * 3 * (obs_f32 ? 4 : 1));
    L.world_bytes = stage ? mc_align16(wxyz) : 0;
    L.warp_bytes = 16 + 128 + L.stage_bytes + L.world_bytes;  // 16: mbarrier, 128: packed_start table
    L.head_bytes = kFastTableBytes + mc_align16((W + H) * 4 + 13 * 3 * 4 + 16 + 13 * 3 + 3);
    // the march reads up to wx*wz bytes on either side of a staged world:
    // keep that much allocated before the first world and after the last
    L.pad_bytes = stage ? mc_align16(wxz) : 0;
    const int before = L.head_bytes + 16 + 128 + L.stage_bytes;
    if (before < L.pad_bytes) L.head_bytes += mc_align16(L.pad_bytes - before);
    return L;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Bounded wait on an mbarrier phase; returns false on timeout.  polls: 0 =
// MC_WAIT_POLLS_DEFAULT, n > 0 = n polls, < 0 = none (the timeout path's test).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, int polls = 0) {
    const int limit = polls == 0 ? MC_WAIT_POLLS_DEFAULT : (polls < 0 ? 0 : polls);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Write `bytes` of a repeating 48-byte pattern (p0 p1 p2) to dst, lanes
// strided.  dst must be 16-byte aligned and bytes a multiple of 16.
__device__ __forceinline__ void fill_pattern16(uint8_t* dst, int bytes, uint4 p0, uint4 p1, uint4 p2, int lane) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    int n = bytes >> 4;
    int m = lane % 3;  // (lane + 32 k) mod 3 advances by 2 per iteration
    for (int k = lane; k < n; k += 32) {
        d[k] = (m == 0) ? p0 : ((m == 1) ? p1 : p2);
        m = (m + 2 >= 3) ? m - 1 : m + 2;
    }
}

// Next env for this warp: claimed from a device counter (dynamic schedule,
// balances the uneven per-env work) or by static striding.
__device__ __forceinline__ long long next_env(const mc_kp& p, long long cur, long long total_warps, int lane) {
    if (!p.sched_dynamic) return cur + total_warps;
    unsigned v = 0;
    if (lane == 0) v = atomicAdd(reinterpret_cast<unsigned*>(&p.flags[MC_FLAG_WORK]), 1u);
    return (long long)__shfl_sync(0xffffffffu, v, 0);
}

// Per-warp view of the shared-memory tables and buffers used by one env.
struct FusedCtx {
    const float* s_u;            // per-column u of the env's image
    const float* s_v;            // per-row v
    const float (*s_rgb)[3];
    const float* s_sky;
    const uint8_t (*s_rgb8)[3];
    const uint8_t* s_sky8;
    uint8_t* stage;              // staging band of this warp
    int8_t* sworld;              // staged world of this warp
    uint32_t mbar_a;             // mbarrier of this warp
    float rcp_vd;                // reciprocal of the env's view distance
    const float4* s_cs;          // colour x shade table of the common-case loop (fast_band)
    const uint32_t* s_rgbp;      // packed flat colours
    int4* sstart;                // this warp's table of march start values (8 entries)
};

// The common-case loop's tables: colour x shade per block and shade code
// (0 x face, 1 z face, 2 y face stepping down, 3 y face stepping up, as in
// shade_rgb) and the flat colours packed r | g << 8 | b << 16.
__device__ __forceinline__ void build_fast_tables(float4* s_cs, uint32_t* s_rgbp) {
    for (int k = threadIdx.x; k < 13 * 4; k += blockDim.x) {
        const int blk = k >> 2, code = k & 3;
        const float shade = code == 0 ? 0.8f : (code == 1 ? 0.9f : (code == 2 ? 0.6f : 1.0f));
        s_cs[k] = make_float4(N::mul(c_rgb[blk][0], shade), N::mul(c_rgb[blk][1], shade),
                              N::mul(c_rgb[blk][2], shade), 0.0f);
    }
    for (int k = threadIdx.x; k < 13; k += blockDim.x)
        s_rgbp[k] = (uint32_t)c_rgb8[k][0] | ((uint32_t)c_rgb8[k][1] << 8) | ((uint32_t)c_rgb8[k][2] << 16);
}

// Shared colour tables: 13*3 + 4 floats, 13*3 + 3 bytes.
constexpr int kColourTableBytes = 13 * 3 * 4 + 16 + 13 * 3 + 3;
static_assert(kColourTableBytes <= MC_COLOUR_TABLE_BYTES, "colour tables");

__device__ __forceinline__ void load_colour_tables(uint8_t* base, FusedCtx& cx) {
    float (*s_rgb)[3] = reinterpret_cast<float (*)[3]>(base);
    float* s_sky = reinterpret_cast<float*>(s_rgb + 13);
    uint8_t (*s_rgb8)[3] = reinterpret_cast<uint8_t (*)[3]>(s_sky + 4);
    uint8_t* s_sky8 = reinterpret_cast<uint8_t*>(s_rgb8 + 13);
    for (int k = threadIdx.x; k < 39; k += blockDim.x) {
        s_rgb[k / 3][k % 3] = c_rgb[k / 3][k % 3];
        s_rgb8[k / 3][k % 3] = c_rgb8[k / 3][k % 3];
    }
    if (threadIdx.x < 3) {
        s_sky[threadIdx.x] = c_sky[threadIdx.x];
        s_sky8[threadIdx.x] = c_sky8[threadIdx.x];
    }
    cx.s_rgb = s_rgb;
    cx.s_sky = s_sky;
    cx.s_rgb8 = s_rgb8;
    cx.s_sky8 = s_sky8;
}

// u/v tables of one image size (threads of the CTA cooperate).
template <int FAM>
__device__ __forceinline__ void build_uv_tables(const mc_kp& p, float* s_u, float* s_v) {
    const int W = p.W, H = p.H;
    float pb_su = 0.0f, pb_sv = 0.0f;
    if (FAM == MC_FAM_PREBASIS) prebasis_scales(W, H, p.fov, &pb_su, &pb_sv);
    for (int k = threadIdx.x; k < W; k += blockDim.x) {
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) s_u[k] = u_shaded(k, W, H, p.fov);
        else if (FAM == MC_FAM_MINIMAL || FAM == MC_FAM_FP16) s_u[k] = u_minimal(k, W, H, p.fov);
        else s_u[k] = u_prebasis(k, W, pb_su);
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) s_v[k] = v_shaded(k, H, p.fov);
        else if (FAM == MC_FAM_MINIMAL || FAM == MC_FAM_FP16) s_v[k] = v_minimal(k, H, p.fov);
        else s_v[k] = v_prebasis(k, H, pb_sv);
    }
}

// The parameters a ray needs.
struct RayPar {
    int wx, wy, wz, max_steps, gh;
    float vd;
};
__device__ __forceinline__ RayPar ray_par(const mc_kp& p) {
    RayPar r;
    r.wx = p.wx;
    r.wy = p.wy;
    r.wz = p.wz;
    r.max_steps = p.max_steps;
    r.gh = p.gh;
    r.vd = p.vd;
    return r;
}

// One pixel's ray through one of the two voxel sources.
// VDLIM = false: view-limited worlds take the reference-shaped loop (fewer registers).
template <int FAM, class V, bool VDLIM = true>
__device__ __forceinline__ Hit march_pixel(const RayPar& p, const Cam& c, const Dda0& d0, float u, float v,
                                           const V& vox, bool inside, bool skip_first, bool sky_exit = false,
                                           bool vd_safe = false, int ytop = 1 << 20) {
    if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST)
        return shade_ray<FAM == MC_FAM_SHADED_FAST, V, VDLIM>(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps, p.vd,
                                                              p.gh, inside, skip_first, sky_exit, vd_safe, ytop);
    if (FAM == MC_FAM_FP16) return fp16_ray(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps);
    return flat_ray<FAM != MC_FAM_PREBASIS>(c, d0, u, v, vox, p.wx, p.wy, p.wz, p.max_steps, skip_first, sky_exit,
                                              ytop);
}

__device__ __forceinline__ void mbar_init_warp(uint32_t mbar_a, int lane) {
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// Last warp of a dynamically scheduled launch resets the work counters.
__device__ __forceinline__ void finish_dynamic(int32_t* flags, long long total_warps) {
    __threadfence();
    unsigned prev = atomicAdd(reinterpret_cast<unsigned*>(&flags[MC_FLAG_WARPS_DONE]), 1u);
    if (prev == (unsigned)(total_warps - 1)) {
        flags[MC_FLAG_WORK] = 0;
        flags[MC_FLAG_WARPS_DONE] = 0;
        __threadfence();
    }
}

// Highest layer of a staged world holding a solid voxel (solid = byte >= 0,
// sign bit clear), found by one warp; -1 for an empty world; wy - 1 when the
// layer size is not a multiple of 16 bytes (not measured).
__device__ __forceinline__ int staged_top_layer(const int8_t* world, int wx, int wy, int wz, int lane) {
    const int layer = wx * wz;
    if (layer & 15) return wy - 1;
    const uint4* w4 = reinterpret_cast<const uint4*>(world);
    const int n16 = (layer * wy) >> 4, per_layer = layer >> 4;
    int top = -1;
    for (int k = n16 - 1 - lane; k >= 0; k -= 32) {
        const uint4 q = w4[k];
        if ((~q.x | ~q.y | ~q.z | ~q.w) & 0x80808080u) {
            top = k / per_layer;
            break;  // this lane's remaining chunks lie in lower layers
        }
    }
    return __reduce_max_sync(0xffffffffu, top);
}

// Solid voxels (byte >= 0) of 16 consecutive bytes as a 16-bit mask: per
// 32-bit word the four sign bits (7, 15, 23, 31) of ~w, multiplied by
// 1 + 2^7 + 2^14 + 2^21, land on bits 28..31 with no carries.
__device__ __forceinline__ uint32_t solid_mask16(uint4 q) {
    auto four = [](uint32_t w) { return ((~w & 0x80808080u) * 0x00204081u) >> 28; };
    return four(q.x) | (four(q.y) << 4) | (four(q.z) << 8) | (four(q.w) << 12);
}

// Whether staged_up_bounds can scan a world of this shape: whole 16-byte
// chunks per row of z, at most 64 voxels a side.
__host__ __device__ __forceinline__ bool up_scan_shape(int wx, int wy, int wz) {
    return (wz & 15) == 0 && wz <= 64 && wx <= 64 && wy <= 64;
}

// One warp scans the rows (y >= vy, x) of a staged world (up_scan_shape;
// the eye's voxel inside the box) for the bounds of every quadrant.  Each
// lane keeps one x (two in worlds wider than 32): G = 32 / wx groups of wx
// lanes sweep every G-th layer, so per row a lane only ORs the row's solid
// z mask into its column's union and notes the highest layers with a solid
// voxel at z >= vz and at z <= vz; the column's x side and the z extremes
// are settled once, after the sweep.  With nw > 1 warps sharing the scan,
// warp w of them sweeps the layers of groups w*G .. w*G+G-1 of nw*G, and
// the result is the warp's part of the bounds (combined by team_up_bounds).
template <typename M>
struct UpPart {
    int xa0, xa1, xa2, xa3;  // x extremes of q0 (x-, z-), q1 (x+, z-), q2 (x-, z+), q3 (x+, z+)
    int ya0, ya1, ya2, ya3;  // highest layer + 1
    M mp, mm;                // solid z masks of the x >= vx / x <= vx columns
};

template <typename M>
__device__ __forceinline__ UpPart<M> staged_up_part(const int8_t* world, int wx, int wy, int wz, int vx, int vy,
                                                    int vz, int lane, int w = 0, int nw = 1) {
    const int cpr = wz >> 4;                              // 16-byte chunks per row
    constexpr int kBits = 8 * sizeof(M);
    const M zpm = ~M(0) << vz;                            // z >= vz
    const M zmm = (vz + 1 < kBits) ? ((M(1) << (vz + 1)) - 1) : ~M(0);  // z <= vz
    const int G = wx <= 32 ? 32 / wx : 1, g = wx <= 32 ? lane / wx : 0;
    int xa0 = 255, xa1 = 0, xa2 = 255, xa3 = 0;
    int ya0 = 0, ya1 = 0, ya2 = 0, ya3 = 0;
    M mp = 0, mm = 0;
    for (int x = wx <= 32 ? lane - g * wx : lane; g < G && x < wx; x += 32) {
        M mu = 0;
        int yp = 0, ym = 0;  // highest layer + 1 with a solid voxel at z >= vz / z <= vz
        for (int y = vy + w * G + g; y < wy; y += G * nw) {
            const int r = y * wx + x;
            const uint4* row = reinterpret_cast<const uint4*>(world + r * wz);
            M m = 0;
            for (int k = 0; k < cpr; ++k) {
                const uint4 q = in_bounds((long long)r * cpr + k, (long long)wx * wy * cpr, MC_SITE_SCAN)
                                    ? row[k] : make_uint4(~0u, ~0u, ~0u, ~0u);
                m |= M(solid_mask16(q)) << (16 * k);
            }
            mu |= m;
            yp = (m & zpm) ? y + 1 : yp;
            ym = (m & zmm) ? y + 1 : ym;
        }
        if (x >= vx) {
            mp |= mu;
            if (yp) { xa3 = max(xa3, x); ya3 = max(ya3, yp); }
            if (ym) { xa1 = max(xa1, x); ya1 = max(ya1, ym); }
        }
        if (x <= vx) {
            mm |= mu;
            if (yp) { xa2 = min(xa2, x); ya2 = max(ya2, yp); }
            if (ym) { xa0 = min(xa0, x); ya0 = max(ya0, ym); }
        }
    }
    constexpr unsigned F = 0xffffffffu;
    auto or_all = [](M v) -> M {
        if (sizeof(M) == 8)
            return M(__reduce_or_sync(F, (unsigned)v)) | (M(__reduce_or_sync(F, (unsigned)(v >> 16 >> 16))) << 16 << 16);
        return M(__reduce_or_sync(F, (unsigned)v));
    };
    UpPart<M> r;
    r.mp = or_all(mp);
    r.mm = or_all(mm);
    r.xa0 = __reduce_min_sync(F, xa0);
    r.xa1 = __reduce_max_sync(F, xa1);
    r.xa2 = __reduce_min_sync(F, xa2);
    r.xa3 = __reduce_max_sync(F, xa3);
    r.ya0 = __reduce_max_sync(F, ya0);
    r.ya1 = __reduce_max_sync(F, ya1);
    r.ya2 = __reduce_max_sync(F, ya2);
    r.ya3 = __reduce_max_sync(F, ya3);
    return r;
}

// The bounds from the (combined) parts.  z extremes: over a side's solid
// voxels the largest z is the z >= vz quadrant's extreme whenever that
// quadrant holds any (else its y byte is 0 and the value is not used), the
// smallest z likewise.
template <typename M>
__device__ __forceinline__ UpBounds up_bounds_of(const UpPart<M>& r) {
    constexpr int kBits = 8 * sizeof(M);
    auto hi = [](M v) { return kBits - 1 - (sizeof(M) == 8 ? __clzll((long long)v) : __clz((int)v)); };
    auto lo = [](M v) { return (sizeof(M) == 8 ? __ffsll((long long)v) : __ffs((int)v)) - 1; };
    UpBounds b;
    b.x = (unsigned)r.xa0 | ((unsigned)r.xa1 << 8) | ((unsigned)r.xa2 << 16) | ((unsigned)r.xa3 << 24);
    b.z = ((unsigned)lo(r.mm) & 255u) | (((unsigned)lo(r.mp) & 255u) << 8) | (((unsigned)hi(r.mm) & 255u) << 16) |
          (((unsigned)hi(r.mp) & 255u) << 24);
    b.y = (unsigned)r.ya0 | ((unsigned)r.ya1 << 8) | ((unsigned)r.ya2 << 16) | ((unsigned)r.ya3 << 24);
    return b;
}

__device__ __forceinline__ UpBounds staged_up_bounds(const int8_t* world, int wx, int wy, int wz, int vx, int vy,
                                                     int vz, int lane) {
    return wz > 32 ? up_bounds_of(staged_up_part<unsigned long long>(world, wx, wy, wz, vx, vy, vz, lane))
                   : up_bounds_of(staged_up_part<uint32_t>(world, wx, wy, wz, vx, vy, vz, lane));
}

// ---------------------------------------------------------------------------
// Fused step, one warp per env (one env group per launch)
// ---------------------------------------------------------------------------
// The per-env body below does what agent_step + fill_env + render_env of the
// team kernel do, written out in one piece: built from those helpers, the
// same kernel needed spill slots at its 64-register budget (4 CTAs of 8 warps
// per SM) and ran 8% slower on B=32768, 16^3, 32x32, so it keeps its own
// copy; the parity tests hold the two kernels to the same bits.
// The common-case render of one band of an env's image (both step
// kernels): the world is staged, the eye is inside the box with air in its
// voxel (every ray starts one DDA step in, and ends as sky when it leaves
// the box), no debug output is asked for, and the image is a whole number of
// tile_w x (32/tile_w) tiles.  Every ray's march start values come from a
// per-env table of the eight ray sign combinations (packed_start for the
// packed march, split_start for the split march).  Every per-env fact is
// settled before the loop, so the per-ray code has no branch but the
// march's: the same operations in the same order as shade_ray / flat_ray
// and shade_rgb (the bits are identical), with the shading done for every
// lane and the sky colour selected afterwards, the colour times the face's
// shade read from s_cs (built with the same N::mul), and the band address
// stepped incrementally.  The band goes to `stage`, then to `dst` with
// 16-byte stores.
struct FastEnv {
    const int4* start;  // per sign combination: packed (index|counts, dx, dy, dz) or split (counts, dax, day, daz)
    uint32_t base;      // staged world (packed) / the eye voxel's address in it (split)
    SmemRange chk;      // the staged world +- one layer (debug build)
    float vd, rcp_vd;
};

template <int FAM, bool F32, bool SPLIT>
__device__ __forceinline__ void fast_band(const Cam& c, const Dda0& d0, const FastEnv& fe, int W, int TW, int row0,
                                          int lane, const float* s_u, const float* s_v, const float4* s_cs,
                                          const uint32_t* s_rgbp, uint8_t* stage, uint8_t* dst) {
    constexpr bool SHADED = FAM == MC_FAM_SHADED;
    constexpr bool TRIG = FAM != MC_FAM_PREBASIS;
    constexpr int bpp = 3 * (F32 ? 4 : 1);
    constexpr int m = F32 ? 0x1 : 0x3;  // sky_fused_mask of the float32 / uint8 shaded kernels
    const float sky0 = 0.53f, sky1 = 0.81f, sky2 = 0.92f;  // SKY_COLOR (c_sky)
    const int TH = 32 / TW;
    const int lx = lane % TW, ly = lane / TW;
    const float v = s_v[row0 + ly];
    const float yraw = N::mad(v, c.uy, c.fy);
    uint8_t* sp = stage + (ly * W + lx) * bpp;
    for (int tx0 = 0; tx0 < W; tx0 += TW, sp += TW * bpp) {
        const float u = s_u[tx0 + lx];
        float x, y = yraw, z;
        if (TRIG) {
            x = N::mad(v, c.ux, N::mad(c.sy, c.cp, N::mul(u, c.rx)));
            z = N::mad(v, c.uz, N::mad(c.cy, c.cp, N::mul(u, c.rz)));
        } else {
            x = N::mad(v, c.ux, N::mad(u, c.rx, c.fx));
            z = N::mad(v, c.uz, N::mad(u, c.rz, c.fz));
        }
        if (SHADED) {
            const float len = N::sqrt(len2(x, y, z));
            const float rl = N::rcp_of(len);
            x = N::div_r(x, len, rl);
            y = N::div_r(y, len, rl);
            z = N::div_r(z, len, rl);
        } else {
            const float rs = N::rsqrt(len2(x, y, z));
            x = N::mul(x, rs);
            y = N::mul(y, rs);
            z = N::mul(z, rs);
        }
        const float ix = (x != 0.0f) ? N::div(1.0f, x) : 1e30f;
        const float iy = (y != 0.0f) ? N::div(1.0f, y) : 1e30f;
        const float iz = (z != 0.0f) ? N::div(1.0f, z) : 1e30f;
        const bool xp = x >= 0.0f, yp = y >= 0.0f, zp = z >= 0.0f;
        float tmx = N::mul(xp ? d0.nxp : d0.nxm, ix);
        float tmy = N::mul(yp ? d0.nyp : d0.nym, iy);
        float tmz = N::mul(zp ? d0.nzp : d0.nzm, iz);
        const int4 e = fe.start[(xp ? 1 : 0) | (yp ? 2 : 0) | (zp ? 4 : 0)];
        const int b = SPLIT ? march_split_shared(fe.base, e.x, e.y, e.z, e.w, tmx, tmy, tmz, fabsf(ix), fabsf(iy),
                                                 fabsf(iz), fe.chk)
                            : march_packed_shared(fe.base, e.x, e.y, e.z, e.w, tmx, tmy, tmz, fabsf(ix), fabsf(iy),
                                                  fabsf(iz), fe.chk);
        if (SHADED) {
            // the axis of the last step, chosen again from the same distances
            const bool bx = tmx < tmy && tmx < tmz;
            const bool by = !bx && tmy < tmz;
            const float t = bx ? tmx : (by ? tmy : tmz);
            const bool hit = b >= 0 && !(t >= fe.vd);
            const int code = bx ? 0 : (by ? (yp ? 3 : 2) : 1);
            const float4 cs = s_cs[(b >= 0 ? b : 0) * 4 + code];
            float fog = fminf(N::div_r(t, fe.vd, fe.rcp_vd), 1.0f);
            fog = N::mul(fog, fog);
            const float omf = N::sub(1.0f, fog);
            const float c0 = (m & 1) ? N::mad(sky0, fog, N::mul(cs.x, omf)) : N::mad(cs.x, omf, N::mul(sky0, fog));
            const float c1 = (m & 2) ? N::mad(sky1, fog, N::mul(cs.y, omf)) : N::mad(cs.y, omf, N::mul(sky1, fog));
            const float c2 = (m & 4) ? N::mad(sky2, fog, N::mul(cs.z, omf)) : N::mad(cs.z, omf, N::mul(sky2, fog));
            const float o0 = hit ? c0 : sky0, o1 = hit ? c1 : sky1, o2 = hit ? c2 : sky2;
            if (F32) {
                float* sf = reinterpret_cast<float*>(sp);
                sf[0] = o0;
                sf[1] = o1;
                sf[2] = o2;
            } else {
                sp[0] = (uint8_t)to_u8(o0);
                sp[1] = (uint8_t)to_u8(o1);
                sp[2] = (uint8_t)to_u8(o2);
            }
        } else {
            // SKY_COLOR_U8 (135, 206, 235) packed
            const uint32_t col = b >= 0 ? s_rgbp[b] : (135u | (206u << 8) | (235u << 16));
            sp[0] = (uint8_t)col;
            sp[1] = (uint8_t)(col >> 8);
            sp[2] = (uint8_t)(col >> 16);
        }
    }
    __syncwarp();
    // copy the band (rows row0 .. row0+TH-1) out with 16-byte stores
    const uint4* s4 = reinterpret_cast<const uint4*>(stage);
    uint4* d4 = reinterpret_cast<uint4*>(dst);
    for (int k = lane; k < ((W * TH * bpp) >> 4); k += 32) d4[k] = s4[k];
    __syncwarp();
}

// Start values of march_split_shared for an env whose eye is in voxel (vx,
// vy, vz), one per sign combination k of the ray (as packed_start): {counts,
// x, y and z address steps}; the start address is the eye voxel's.
__device__ __forceinline__ int4 split_start(int k, int vx, int vy, int vz, int wx, int wy, int wz,
                                            const UpBounds& ub, int max_steps) {
    const int sx = (k & 1) ? 1 : -1, sy = (k & 2) ? 1 : -1, sz = (k & 4) ? 1 : -1;
    int cx, cy, cz;
    start_counts(k, vx, vy, vz, wx, wy, wz, ub, cx, cy, cz);
    return make_int4(split_counts(cx, cy, cz, max_steps, wx, wy, wz), sx * wz, sy * wx * wz, sz);
}

// Whether an env takes the common-case loop, and which march: 0 no, 1
// packed, 2 split.  `eye_air_inside`: the eye is strictly inside the box
// (view distance > 0 for the shaded family) and its voxel holds air.
template <int FAM>
__device__ __forceinline__ int fast_kind(bool staged, bool eye_air_inside, bool dbg, bool vd_safe, int max_steps,
                                         int wx, int wy, int wz, int W, int H, int TW, int bpp, bool vec_ok) {
    if (!(FAM == MC_FAM_SHADED || FAM == MC_FAM_MINIMAL || FAM == MC_FAM_PREBASIS)) return 0;
    if (!staged || !eye_air_inside || dbg || max_steps <= 0 || wx > 64 || wy > 64 || wz > 64) return 0;
    if (W % TW || H % (32 / TW) || !vec_ok || ((W * (32 / TW) * bpp) & 15)) return 0;
    const bool packed = (FAM == MC_FAM_SHADED ? vd_safe : true) && max_steps > wx + wy + wz && wx <= 31 &&
                        wy <= 31 && wz <= 31 && wx * wy * wz < 8192;
    return packed ? 1 : 2;
}

// The per-env start table (8 lanes write, the warp reads).
__device__ __forceinline__ void build_fast_start(int4* sstart, int kind, const Dda0& d0, int wx, int wy, int wz,
                                                 const UpBounds& ub, int max_steps, int lane) {
    if (lane < 8)
        sstart[lane] = kind == 1 ? packed_start(lane, d0.vx, d0.vy, d0.vz, wx, wy, wz, ub)
                                 : split_start(lane, d0.vx, d0.vy, d0.vz, wx, wy, wz, ub, max_steps);
    __syncwarp();
}

// Per-env facts of a render (EnvRender::bits).
// MC_ER_TSCAN: the up bounds are scanned by the whole team after its barrier.
enum { MC_ER_DONE = 1, MC_ER_BURIED = 2, MC_ER_INSIDE = 4, MC_ER_SKIP = 8, MC_ER_STAGED = 16, MC_ER_TSCAN = 32 };

// The rest of a per-warp launch for a warp whose bulk copy timed out
// (defined after render_env): env e, already stepped, then `claimed` (the
// env a depth-2 warp has already claimed, or -1 for none), then every env
// the warp claims after them, rendered from the worlds in global memory.
// Called after the main loop and out of line, so the staged path keeps its
// registers.  Returns whether any of those envs was done.
template <int FAM, bool F32>
__device__ __noinline__ bool fused_finish_from_global(const mc_kp& p, long long e, long long claimed,
                                                      long long total_warps, int tile_w, int lane, FusedCtx cx);

#ifndef MC_FUSED_MIN_BLOCKS
#define MC_FUSED_MIN_BLOCKS 4
#endif
// DEPTH: 0 worlds read from global memory, 1 staged, 2 staged with the next
// env claimed ahead and its world prefetched into L2.
template <int FAM, bool F32, int DEPTH>
__global__ void __launch_bounds__(256, MC_FUSED_MIN_BLOCKS) k_step_fused(const __grid_constant__ mc_kp p, int tile_w) {
    constexpr bool STAGE = DEPTH > 0;
    constexpr bool prefetch = DEPTH == 2;
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int W = p.W, H = p.H;
    const int HW = W * H;
    const int wxz = p.wx * p.wz;
    const int wxyz = wxz * p.wy;
    FusedLayout L = fused_layout(W, H, wxyz, p.wx * p.wz, F32, STAGE, tile_w);

    // --- tables -------------------------------------------------------------
    float4* s_cs = reinterpret_cast<float4*>(smem);                           // [13][4]
    uint32_t* s_rgbp = reinterpret_cast<uint32_t*>(smem + kShadeTableBytes);  // [13]
    build_fast_tables(s_cs, s_rgbp);
    float* s_u = reinterpret_cast<float*>(smem + kFastTableBytes);
    float* s_v = s_u + W;
    float (*s_rgb)[3] = reinterpret_cast<float (*)[3]>(s_v + H);
    float* s_sky = reinterpret_cast<float*>(s_rgb + 13);
    uint8_t (*s_rgb8)[3] = reinterpret_cast<uint8_t (*)[3]>(s_sky + 4);
    uint8_t* s_sky8 = reinterpret_cast<uint8_t*>(s_rgb8 + 13);
    float pb_su = 0.0f, pb_sv = 0.0f;
    if (FAM == MC_FAM_PREBASIS) prebasis_scales(W, H, p.fov, &pb_su, &pb_sv);
    for (int k = threadIdx.x; k < W; k += blockDim.x) {
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) s_u[k] = u_shaded(k, W, H, p.fov);
        else if (FAM == MC_FAM_MINIMAL || FAM == MC_FAM_FP16) s_u[k] = u_minimal(k, W, H, p.fov);
        else s_u[k] = u_prebasis(k, W, pb_su);
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) s_v[k] = v_shaded(k, H, p.fov);
        else if (FAM == MC_FAM_MINIMAL || FAM == MC_FAM_FP16) s_v[k] = v_minimal(k, H, p.fov);
        else s_v[k] = v_prebasis(k, H, pb_sv);
    }
    for (int k = threadIdx.x; k < 39; k += blockDim.x) {
        s_rgb[k / 3][k % 3] = c_rgb[k / 3][k % 3];
        s_rgb8[k / 3][k % 3] = c_rgb8[k / 3][k % 3];
    }
    if (threadIdx.x < 3) {
        s_sky[threadIdx.x] = c_sky[threadIdx.x];
        s_sky8[threadIdx.x] = c_sky8[threadIdx.x];
    }
    uint8_t* wbase = smem + L.head_bytes + warp * L.warp_bytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(wbase);
    int4* sstart = reinterpret_cast<int4*>(wbase + 16);
    uint8_t* stage = wbase + 16 + 128;
    int8_t* sworld = reinterpret_cast<int8_t*>(wbase + 16 + 128 + L.stage_bytes);
    uint32_t mbar_a = smem_u32(mbar);
    if (STAGE && lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0;
    bool no_stage = false;        // a copy timed out: this warp renders from global memory from now on
    bool pending = false;         // ... and that copy may still be in flight
    uint32_t pending_phase = 0;   // its phase, waited for before the warp leaves
    // The kernel runs at its 64-register budget: values that would stay live
    // across the env loop are recomputed where they are used (1 / vd, the
    // env sizes) or not kept at all (the any-done flag goes straight to the
    // flag word), and env indices are 32-bit (fewer spills, measured faster).

    const int obs_env_bytes = HW * 3 * (F32 ? 4 : 1);
    const int total_warps = gridDim.x * nwarps;
    const int first = p.sched_dynamic ? (int)next_env(p, 0, total_warps, lane) : blockIdx.x * nwarps + warp;
    int e = first;
    // staging depth 2 (prefetch): the warp claims its next env one ahead and,
    // while it steps and renders this one, prefetches that env's world (and
    // the state the step reads) into L2, so the next bulk copy reads L2
    int ahead = (prefetch && e < p.B) ? (int)next_env(p, e, total_warps, lane) : p.B;
    auto advance = [&]() -> int {
        if (!prefetch) return (int)next_env(p, e, total_warps, lane);
        const int r = ahead;
        ahead = r < p.B ? (int)next_env(p, r, total_warps, lane) : r;
        return r;
    };
    for (; e < p.B; e = advance()) {
        if (prefetch && ahead < p.B) {
            if (lane == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p.voxels + ahead * (long long)wxyz),
                             "r"(wxyz)
                             : "memory");
            const void* st = lane == 1 ? (const void*)(p.positions + ahead * 3)
                           : lane == 2 ? (const void*)(p.velocities + ahead * 3)
                           : lane == 3 ? (const void*)(p.yaws + ahead)
                           : lane == 4 ? (const void*)(p.pitches + ahead)
                           : lane == 5 ? (const void*)(p.on_ground + ahead)
                           : lane == 6 && p.actions ? (const void*)(p.actions + ahead)
                                                    : nullptr;
            if (st) asm volatile("prefetch.global.L2 [%0];" ::"l"(st));
        }
        // ---- agent step (every lane computes the same values) --------------
        int8_t btn[8];
        float l0, l1;
        load_action(p, e, btn, l0, l1);
        Dec d = decode_buttons(btn, l0, l1, p.sprint_mult);
        int32_t cnt = p.ext_done ? 0 : p.step_count[e];
        bool done = p.ext_done ? (p.do_reset[e] != 0) : episode_done(p, cnt);
        Agent a = load_agent(p, e);
        physics(a, d, p);
        int8_t* gw = p.voxels + e * (long long)wxyz;
        float reward;
        int8_t mod_val;
        int mod_idx = interact_warp(gw, a, d.brk, d.place, p, lane, &reward, &mod_val);
        if (done) reset_agent(a, p);
        if (done && lane == 0) atomicOr(&p.flags[MC_FLAG_ANY_DONE], 1);  // rare: no per-warp accumulator
        if (lane == 0) {
            store_agent(p, e, a);
            if (!p.ext_done) {
                p.step_count[e] = done ? 1 : cnt + 1;
                p.do_reset[e] = done ? 1 : 0;
            }
            p.rewards[e] = reward;
            if (p.res_rewards) {
                p.res_rewards[e] = reward;
                p.res_dones[e] = done ? 1 : 0;
            }
            p.cameras[e * 5 + 0] = a.x;
            p.cameras[e * 5 + 1] = a.y;
            p.cameras[e * 5 + 2] = a.z;
            p.cameras[e * 5 + 3] = a.yaw;
            p.cameras[e * 5 + 4] = a.pitch;
            if (p.dbg_interact) p.dbg_interact[e] = mod_idx;
        }
        // ---- per-env render constants -------------------------------------
        Cam c;
        float bas[13];
        if (FAM == MC_FAM_PREBASIS) {
            basis_compute(a.x, a.y, a.z, a.yaw, a.pitch, W, H, p.fov, bas);
            c = cam_from_basis(bas);
            if (p.basis && lane == 0) {
#pragma unroll
                for (int k = 0; k < 13; ++k) p.basis[e * 14 + k] = bas[k];
            }
        } else {
            c = cam_trig(a.x, a.y, a.z, a.yaw, a.pitch);
        }
        // Every ray starts in the eye's voxel.  If the first DDA step already
        // hits (the eye is inside a solid voxel, or below ground for the
        // ground-shortcut family), every pixel of the env gets the same
        // colour, so the env is filled without marching.
        const int ex = (int)floorf(c.eye_x), ey = (int)floorf(c.eye_y), ez = (int)floorf(c.eye_z);
        bool eye_inb = (unsigned)ex < (unsigned)p.wx && (unsigned)ey < (unsigned)p.wy && (unsigned)ez < (unsigned)p.wz;
        int eye_idx = ey * wxz + ex * p.wz + ez;
        int8_t eye_blk = AIR;
        __syncwarp();
        if (eye_inb && in_bounds(eye_idx, wxyz, MC_SITE_EYE)) eye_blk = gw[eye_idx];
        bool inside = false;
        bool buried;
        int fill_blk = eye_blk;
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
            inside = eye_inside(c, p.wx, p.wy, p.wz, p.vd);
            bool start_hit = eye_blk >= 0;
            if (FAM == MC_FAM_SHADED_FAST && ey < p.gh) {
                start_hit = true;
                fill_blk = (ey == p.gh - 1) ? GRASS : DIRT;
            }
            buried = inside && p.vd > 0.0f && p.max_steps > 0 && start_hit;
        } else {
            buried = p.max_steps > 0 && eye_inb && eye_blk >= 0;
        }
        // not buried: the first DDA step of every ray tests the eye voxel and
        // advances; when that test is known to fail, rays start advanced
        bool skip_first;
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST)
            skip_first = inside && p.vd > 0.0f && p.max_steps > 0 && eye_blk < 0 &&
                         !(FAM == MC_FAM_SHADED_FAST && ey < p.gh);
        else
            skip_first = p.max_steps > 0 && !(eye_inb && eye_blk >= 0);
        uint8_t* oenv = (uint8_t*)p.obs + (long long)e * obs_env_bytes;
        const bool vec_ok = ((obs_env_bytes & 15) == 0) && ((((uintptr_t)oenv) & 15) == 0);
        if (buried) {
            Hit h;
            h.blk = fill_blk;
            h.face = -1;
            h.t = 0.0f;
            h.step_y = 1;
            uint8_t bytes[12];
            if (F32 || FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
                float rgb[3];
                shade_rgb<F32 ? MC_COL_F32 : (FAM == MC_FAM_SHADED_FAST ? MC_COL_U8FAST : MC_COL_U8)>(
                    h, p.vd, N::rcp_of(p.vd), s_rgb, s_sky, rgb);
                if (F32) {
                    // pattern period 12 bytes
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        uint32_t w32 = __float_as_uint(rgb[k]);
                        bytes[4 * k + 0] = (uint8_t)(w32);
                        bytes[4 * k + 1] = (uint8_t)(w32 >> 8);
                        bytes[4 * k + 2] = (uint8_t)(w32 >> 16);
                        bytes[4 * k + 3] = (uint8_t)(w32 >> 24);
                    }
                } else {
                    bytes[0] = (uint8_t)to_u8(rgb[0]);
                    bytes[1] = (uint8_t)to_u8(rgb[1]);
                    bytes[2] = (uint8_t)to_u8(rgb[2]);
                }
            } else {
                bytes[0] = s_rgb8[fill_blk][0];
                bytes[1] = s_rgb8[fill_blk][1];
                bytes[2] = s_rgb8[fill_blk][2];
            }
            const int period = F32 ? 12 : 3;
            if (vec_ok) {
                uint32_t w[12];
#pragma unroll
                for (int k = 0; k < 12; ++k) {
                    w[k] = (uint32_t)bytes[(4 * k + 0) % period] | ((uint32_t)bytes[(4 * k + 1) % period] << 8) |
                           ((uint32_t)bytes[(4 * k + 2) % period] << 16) | ((uint32_t)bytes[(4 * k + 3) % period] << 24);
                }
                fill_pattern16(oenv, (int)obs_env_bytes, make_uint4(w[0], w[1], w[2], w[3]),
                               make_uint4(w[4], w[5], w[6], w[7]), make_uint4(w[8], w[9], w[10], w[11]), lane);
            } else {
                for (int k = lane; k < obs_env_bytes; k += 32) oenv[k] = bytes[k % period];
            }
            if (p.dbg_pixel) {
                int16_t code = dbg_code(h);
                for (int k = lane; k < HW; k += 32) p.dbg_pixel[(long long)e * HW + k] = code;
            }
            continue;
        }
        // ---- stage the world into shared memory ----------------------------
        const int8_t* wsrc = gw;
        int ytop = p.wy - 1;  // highest layer with a solid voxel (all layers unless measured)
        UpBounds ub = up_none(ytop);
        if (STAGE) {
#if MC_CHECK_BOUNDS
            {
                const SmemRange dyn = dyn_smem_range();
                const long long off = (long long)smem_u32(sworld) - dyn.lo;
                if (!in_bounds(off, dyn.span, MC_SITE_STAGE) || !in_bounds(off + wxyz - 1, dyn.span, MC_SITE_STAGE)) {
                    no_stage = true;  // no copy issued: render from global memory
                    break;
                }
            }
#endif
            if (lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_a), "r"(wxyz)
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_u32(sworld)),
                    "l"(gw), "r"(wxyz), "r"(mbar_a)
                    : "memory");
            }
            if (!mbar_wait(mbar_a, phase, p.wait_polls)) {
                if (lane == 0) atomicExch(&p.flags[MC_FLAG_ERROR], MC_KERR_TMA_TIMEOUT);
                no_stage = true;  // the copy may still land in this warp's buffer: never read it again
                pending = true;
                pending_phase = phase;
                break;            // env e and the rest: fused_finish_from_global below
            }
            phase ^= 1u;
            // the interaction may have written after the copy read the byte
            if (lane == 0 && mod_idx >= 0 && in_bounds(mod_idx, wxyz, MC_SITE_PATCH)) sworld[mod_idx] = mod_val;
            __syncwarp();
            wsrc = sworld;
            if (eye_inb && up_scan_shape(p.wx, p.wy, p.wz)) {
                ub = staged_up_bounds(sworld, p.wx, p.wy, p.wz, ex, ey, ez, lane);
                ytop = up_top(ub);  // the same cut for rays going up from the eye
            } else {
                ytop = staged_top_layer(sworld, p.wx, p.wy, p.wz, lane);
                ub = up_none(ytop);
            }
        }
        // ---- march every pixel ---------------------------------------------
        const Dda0 d0 = dda0(c);
        // per-env facts that let the march stop early (debug output needs the
        // reference's face and distance of sky pixels too)
        const bool sky_exit = (FAM == MC_FAM_SHADED) ? (inside && p.vd > 0.0f && !p.dbg_pixel)
                                                     : (eye_inb && !p.dbg_pixel);
        const bool vd_safe = sky_exit && box_within_view(c, p.wx, p.wy, p.wz, p.vd);
        // where every ray takes the packed march, its start values per sign
        // combination, built once for the env
        const int4* start = nullptr;
        const bool flat_fam = FAM == MC_FAM_MINIMAL || FAM == MC_FAM_PREBASIS;
        if (STAGE && (FAM == MC_FAM_SHADED ? vd_safe : (flat_fam && sky_exit)) &&
            p.max_steps > p.wx + p.wy + p.wz && p.wx <= 31 && p.wy <= 31 && p.wz <= 31 && wxyz < 8192) {
            if (lane < 8) sstart[lane] = packed_start(lane, d0.vx, d0.vy, d0.vz, p.wx, p.wy, p.wz, ub);
            __syncwarp();
            start = sstart;
        }
        const int TW = L.tile_w, TH = L.tile_h;
        if constexpr (STAGE && (FAM == MC_FAM_SHADED || FAM == MC_FAM_MINIMAL || FAM == MC_FAM_PREBASIS)) {
            // the common case (fast_band): staged world, eye inside with air in
            // its voxel, no debug output, whole tiles
            const int fk = fast_kind<FAM>(true, sky_exit && skip_first, p.dbg_pixel != nullptr, vd_safe,
                                          p.max_steps, p.wx, p.wy, p.wz, W, H, TW, 3 * (F32 ? 4 : 1), vec_ok);
            if (fk) {
                if (fk == 2 || !start) build_fast_start(sstart, fk, d0, p.wx, p.wy, p.wz, ub, p.max_steps, lane);
                const uint32_t wb = smem_u32(sworld);
                FastEnv fe;
                fe.start = sstart;
                fe.base = fk == 1 ? wb : wb + (uint32_t)(d0.vy * wxz + d0.vx * p.wz + d0.vz);
                fe.chk = staged_range(wb, wxz, wxyz);
                fe.vd = p.vd;
                fe.rcp_vd = N::rcp_of(p.vd);
                for (int row0 = 0; row0 < H; row0 += TH) {
                    uint8_t* dst = oenv + (long long)row0 * W * (3 * (F32 ? 4 : 1));
                    if (fk == 1)
                        fast_band<FAM, F32, false>(c, d0, fe, W, TW, row0, lane, s_u, s_v, s_cs, s_rgbp, stage, dst);
                    else
                        fast_band<FAM, F32, true>(c, d0, fe, W, TW, row0, lane, s_u, s_v, s_cs, s_rgbp, stage, dst);
                }
                continue;
            }
        }
        const int lx = lane % TW, ly = lane / TW;
        const int bpp = 3 * (F32 ? 4 : 1);  // bytes per pixel
        for (int row0 = 0; row0 < H; row0 += TH) {
            const int py = row0 + ly;
            const float v = (py < H && in_bounds(py, H, MC_SITE_TABLE)) ? s_v[py] : 0.0f;
            for (int tx0 = 0; tx0 < W; tx0 += TW) {
                const int px = tx0 + lx;
                if (px < W && py < H && in_bounds(px, W, MC_SITE_TABLE)) {
                    Hit h;
                    const float u = s_u[px];
                    if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
                        // the one-warp-per-env kernel keeps its 64-register budget: the
                        // branch-free march only where the whole box is within view
                        if (STAGE) h = shade_ray<FAM == MC_FAM_SHADED_FAST, VoxShared, false, true>(c, d0, u, v, VoxShared{wsrc}, p.wx, p.wy, p.wz, p.max_steps, p.vd, p.gh, inside, skip_first, sky_exit, vd_safe, ytop, start);
                        else h = shade_ray<FAM == MC_FAM_SHADED_FAST, VoxGlobal, false>(c, d0, u, v, VoxGlobal{wsrc}, p.wx, p.wy, p.wz, p.max_steps, p.vd, p.gh, inside, skip_first, sky_exit, vd_safe);
                    } else if (FAM == MC_FAM_FP16) {
                        if (STAGE) h = fp16_ray(c, d0, u, v, VoxShared{wsrc}, p.wx, p.wy, p.wz, p.max_steps);
                        else h = fp16_ray(c, d0, u, v, VoxGlobal{wsrc}, p.wx, p.wy, p.wz, p.max_steps);
                    } else {
                        constexpr bool TRIG = (FAM != MC_FAM_PREBASIS);
                        if (STAGE) h = flat_ray<TRIG, VoxShared, true>(c, d0, u, v, VoxShared{wsrc}, p.wx, p.wy, p.wz, p.max_steps, skip_first, sky_exit, ytop, start);
                        else h = flat_ray<TRIG>(c, d0, u, v, VoxGlobal{wsrc}, p.wx, p.wy, p.wz, p.max_steps, skip_first, sky_exit);
                    }
                    const int so = ly * W + px;  // pixel within the staged band
                    if (!in_bounds((long long)(so + 1) * bpp - 1, L.stage_bytes, MC_SITE_BAND)) continue;
                    if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
                        float rgb[3];
                        shade_rgb<F32 ? MC_COL_F32 : (FAM == MC_FAM_SHADED_FAST ? MC_COL_U8FAST : MC_COL_U8)>(
                            h, p.vd, N::rcp_of(p.vd), s_rgb, s_sky, rgb);
                        if (F32) {
                            float* sf = reinterpret_cast<float*>(stage) + so * 3;
                            sf[0] = rgb[0]; sf[1] = rgb[1]; sf[2] = rgb[2];
                        } else {
                            uint8_t* sb = stage + so * 3;
                            sb[0] = (uint8_t)to_u8(rgb[0]);
                            sb[1] = (uint8_t)to_u8(rgb[1]);
                            sb[2] = (uint8_t)to_u8(rgb[2]);
                        }
                    } else {
                        const uint8_t* col = (h.blk >= 0 && in_bounds(h.blk, 13, MC_SITE_TABLE)) ? s_rgb8[h.blk] : s_sky8;
                        uint8_t* sb = stage + so * 3;
                        sb[0] = col[0]; sb[1] = col[1]; sb[2] = col[2];
                    }
                    if (p.dbg_pixel && in_bounds(py * W + px, HW, MC_SITE_DEBUG))
                        p.dbg_pixel[(long long)e * HW + py * W + px] = dbg_code(h);
                }
            }
            __syncwarp();
            // copy the band (rows row0 .. row0+TH-1) out
            const int nbytes = min(TH, H - row0) * W * bpp;
            uint8_t* dst = oenv + (long long)row0 * W * bpp;
            if (!in_bounds((long long)row0 * W * bpp + nbytes - 1, obs_env_bytes, MC_SITE_COPY_OUT) ||
                !in_bounds(nbytes - 1, L.stage_bytes, MC_SITE_BAND)) {
                __syncwarp();
                continue;
            }
            if (vec_ok && (nbytes & 15) == 0 && (((long long)row0 * W * bpp) & 15) == 0) {
                const uint4* s4 = reinterpret_cast<const uint4*>(stage);
                uint4* d4 = reinterpret_cast<uint4*>(dst);
                for (int k = lane; k < (nbytes >> 4); k += 32) d4[k] = s4[k];
            } else {
                for (int k = lane; k < nbytes; k += 32) dst[k] = stage[k];
            }
            __syncwarp();
        }
    }
    if (STAGE && no_stage) {
        FusedCtx cx;
        cx.s_u = s_u;
        cx.s_v = s_v;
        cx.s_rgb = s_rgb;
        cx.s_sky = s_sky;
        cx.s_rgb8 = s_rgb8;
        cx.s_sky8 = s_sky8;
        cx.stage = stage;
        cx.rcp_vd = N::rcp_of(p.vd);
        if (fused_finish_from_global<FAM, F32>(p, e, prefetch ? ahead : -1, total_warps, tile_w, lane, cx) && lane == 0)
            atomicOr(&p.flags[MC_FLAG_ANY_DONE], 1);
        // the timed-out copy may still be in flight: let it land (bounded, with
        // the default budget) before this warp's part of shared memory can be released
        if (pending) mbar_wait(mbar_a, pending_phase);
    }
    // No CTA barrier here: warps leave as soon as their last env is done.
    if (lane == 0) {
        bounds_to_flags(p.flags);
        if (p.sched_dynamic) {
            // every claim of this warp has returned (the last one >= B); the
            // last warp to get here resets the counters for the next launch
            __threadfence();
            unsigned prev = atomicAdd(reinterpret_cast<unsigned*>(&p.flags[MC_FLAG_WARPS_DONE]), 1u);
            if (prev == (unsigned)(total_warps - 1)) {
                p.flags[MC_FLAG_WORK] = 0;
                p.flags[MC_FLAG_WARPS_DONE] = 0;
                __threadfence();
            }
        }
    }
}


// ---------------------------------------------------------------------------
// Team kernel: env groups of any size, stepped by teams of warps
// ---------------------------------------------------------------------------
// A CTA of warps_per_cta warps is split into teams of team_warps warps.  A
// team claims one work unit at a time from a device counter:
//  * a cooperative group's unit is ONE env: the team's first warp steps the
//    agent, then all warps of the team march row bands of its image (bands
//    claimed from a shared counter), reading the world from one shared-memory
//    copy per team when staged.  Big images over big worlds then keep an
//    SM's L1 and shared memory on few worlds, like a per-pixel kernel;
//  * a per-warp group's unit is team_warps envs, one per warp, each stepped
//    and rendered by its warp alone.
// Units are ordered by decreasing per-env cost across groups, so the most
// expensive envs are claimed first and do not straggle at the end.

// What the render of one env needs from its agent step.
struct EnvRender {
    Cam c;
    int bits;      // MC_ER_*
    int fill_blk;  // block of the uniform fill of a buried camera
    int mod_idx;   // voxel index the interaction wrote, -1 if none
    int mod_val;
    int ytop;      // no solid voxel above this layer (wy - 1 unless measured)
    UpBounds ub;   // bounds of the rays going up (up_none(ytop) unless measured)
};

// Whether the eye's voxel lies in the box.
__device__ __forceinline__ bool eye_in_box(const Cam& c, int wx, int wy, int wz) {
    const int ex = (int)floorf(c.eye_x), ey = (int)floorf(c.eye_y), ez = (int)floorf(c.eye_z);
    return (unsigned)ex < (unsigned)wx && (unsigned)ey < (unsigned)wy && (unsigned)ez < (unsigned)wz;
}

// Measure a staged world for the rays going up: per quadrant of the eye's
// column when the eye's voxel lies in the box, else the top layer only.
__device__ __forceinline__ void measure_staged(EnvRender& r, const int8_t* world, int wx, int wy, int wz, int lane) {
    const int ex = (int)floorf(r.c.eye_x), ey = (int)floorf(r.c.eye_y), ez = (int)floorf(r.c.eye_z);
    if (eye_in_box(r.c, wx, wy, wz) && up_scan_shape(wx, wy, wz)) {
        r.ub = staged_up_bounds(world, wx, wy, wz, ex, ey, ez, lane);
        r.ytop = up_top(r.ub);
    } else {
        r.ytop = staged_top_layer(world, wx, wy, wz, lane);
        r.ub = up_none(r.ytop);
    }
}


// Barrier of one team (named barrier `bar`, nthreads threads).
__device__ __forceinline__ void team_sync(int bar, int nthreads) {
    if (nthreads == 32)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nthreads) : "memory");
}

struct TeamShared {
    unsigned unit[2];  // claimed units, alternating slots
    int band_ctr;      // next row band of the cooperative env
    int pad;
    EnvRender r;       // the cooperative env
    // the cooperative env's up bounds, combined over the team's warps (UpPart)
    int uxa[4], uya[4];
    unsigned long long ump, umm;
};
static_assert(sizeof(TeamShared) <= MC_TEAM_HEAD_BYTES, "team head");

// Reset the team's up-bound words (the stepping warp's lane 0, before the
// barrier that publishes the env).
__device__ __forceinline__ void team_up_reset(TeamShared* ts) {
    ts->uxa[0] = 255; ts->uxa[1] = 0; ts->uxa[2] = 255; ts->uxa[3] = 0;
    ts->uya[0] = ts->uya[1] = ts->uya[2] = ts->uya[3] = 0;
    ts->ump = ts->umm = 0ull;
}

// The up bounds of a cooperative env, scanned by all nw warps of its team
// (warp w sweeps its share of the layers, staged_up_part) and combined in
// the team's shared words with shared-memory atomics, so every warp holds
// the same bounds after the team barrier.  Called by every warp of the team.
template <typename M>
__device__ __forceinline__ UpBounds team_up_bounds_t(const int8_t* world, int wx, int wy, int wz, int vx, int vy,
                                                     int vz, int lane, int w, int nw, TeamShared* ts, int bar) {
    const UpPart<M> r = staged_up_part<M>(world, wx, wy, wz, vx, vy, vz, lane, w, nw);
    if (lane == 0) {
        atomicMin(&ts->uxa[0], r.xa0);
        atomicMax(&ts->uxa[1], r.xa1);
        atomicMin(&ts->uxa[2], r.xa2);
        atomicMax(&ts->uxa[3], r.xa3);
        atomicMax(&ts->uya[0], r.ya0);
        atomicMax(&ts->uya[1], r.ya1);
        atomicMax(&ts->uya[2], r.ya2);
        atomicMax(&ts->uya[3], r.ya3);
        atomicOr(&ts->ump, (unsigned long long)r.mp);
        atomicOr(&ts->umm, (unsigned long long)r.mm);
    }
    team_sync(bar, nw * 32);
    UpPart<M> t;
    t.xa0 = ts->uxa[0];
    t.xa1 = ts->uxa[1];
    t.xa2 = ts->uxa[2];
    t.xa3 = ts->uxa[3];
    t.ya0 = ts->uya[0];
    t.ya1 = ts->uya[1];
    t.ya2 = ts->uya[2];
    t.ya3 = ts->uya[3];
    t.mp = (M)ts->ump;
    t.mm = (M)ts->umm;
    return up_bounds_of(t);
}
__device__ __forceinline__ UpBounds team_up_bounds(const int8_t* world, int wx, int wy, int wz, int vx, int vy, int vz,
                                                   int lane, int w, int nw, TeamShared* ts, int bar) {
    return wz > 32 ? team_up_bounds_t<unsigned long long>(world, wx, wy, wz, vx, vy, vz, lane, w, nw, ts, bar)
                   : team_up_bounds_t<uint32_t>(world, wx, wy, wz, vx, vy, vz, lane, w, nw, ts, bar);
}

// Decode, episode rule, physics, interaction, reset, counters and camera of
// env e, run by one whole warp: every lane computes the same values, lane 0
// writes the state.
template <int FAM>
__device__ __forceinline__ EnvRender agent_step(const mc_kp& p, const ActionSrc& act, long long e, int lane) {
    const int wxz = p.wx * p.wz;
    const int wxyz = wxz * p.wy;
    int8_t btn[8];
    float l0, l1;
    load_action_from(act, p.look_delta, e, btn, l0, l1);
    Dec d = decode_buttons(btn, l0, l1, p.sprint_mult);
    int32_t cnt = p.ext_done ? 0 : p.step_count[e];
    bool done = p.ext_done ? (p.do_reset[e] != 0) : episode_done(p, cnt);
    Agent a = load_agent(p, e);
    physics(a, d, p);
    int8_t* gw = p.voxels + e * (long long)wxyz;
    float reward;
    int8_t mod_val;
    int mod_idx = interact_warp(gw, a, d.brk, d.place, p, lane, &reward, &mod_val);
    if (done) reset_agent(a, p);
    if (lane == 0) {
        store_agent(p, e, a);
        if (!p.ext_done) {
            p.step_count[e] = done ? 1 : cnt + 1;
            p.do_reset[e] = done ? 1 : 0;
        }
        p.rewards[e] = reward;
        if (p.res_rewards) {
            p.res_rewards[e] = reward;
            p.res_dones[e] = done ? 1 : 0;
        }
        p.cameras[e * 5 + 0] = a.x;
        p.cameras[e * 5 + 1] = a.y;
        p.cameras[e * 5 + 2] = a.z;
        p.cameras[e * 5 + 3] = a.yaw;
        p.cameras[e * 5 + 4] = a.pitch;
        if (p.dbg_interact) p.dbg_interact[e] = mod_idx;
    }
    EnvRender r;
    if (FAM == MC_FAM_PREBASIS) {
        float bas[13];
        basis_compute(a.x, a.y, a.z, a.yaw, a.pitch, p.W, p.H, p.fov, bas);
        r.c = cam_from_basis(bas);
        if (p.basis && lane == 0) {
#pragma unroll
            for (int k = 0; k < 13; ++k) p.basis[e * 14 + k] = bas[k];
        }
    } else {
        r.c = cam_trig(a.x, a.y, a.z, a.yaw, a.pitch);
    }
    // Every ray starts in the eye's voxel.  If the first DDA step already
    // hits (the eye is inside a solid voxel, or below ground for the
    // ground-shortcut family), every pixel of the env gets the same colour.
    const Cam& c = r.c;
    const int ex = (int)floorf(c.eye_x), ey = (int)floorf(c.eye_y), ez = (int)floorf(c.eye_z);
    bool eye_inb = (unsigned)ex < (unsigned)p.wx && (unsigned)ey < (unsigned)p.wy && (unsigned)ez < (unsigned)p.wz;
    int8_t eye_blk = AIR;
    __syncwarp();
    if (eye_inb && in_bounds(ey * wxz + ex * p.wz + ez, wxyz, MC_SITE_EYE)) eye_blk = gw[ey * wxz + ex * p.wz + ez];
    bool inside = false, buried, skip_first;
    int fill_blk = eye_blk;
    if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
        inside = eye_inside(c, p.wx, p.wy, p.wz, p.vd);
        bool start_hit = eye_blk >= 0;
        if (FAM == MC_FAM_SHADED_FAST && ey < p.gh) {
            start_hit = true;
            fill_blk = (ey == p.gh - 1) ? GRASS : DIRT;
        }
        buried = inside && p.vd > 0.0f && p.max_steps > 0 && start_hit;
        // not buried: the first DDA step of every ray tests the eye voxel
        // and advances; when that test is known to fail, rays start advanced
        skip_first = inside && p.vd > 0.0f && p.max_steps > 0 && eye_blk < 0 &&
                     !(FAM == MC_FAM_SHADED_FAST && ey < p.gh);
    } else {
        buried = p.max_steps > 0 && eye_inb && eye_blk >= 0;
        skip_first = p.max_steps > 0 && !(eye_inb && eye_blk >= 0);
    }
    r.bits = (done ? MC_ER_DONE : 0) | (buried ? MC_ER_BURIED : 0) | (inside ? MC_ER_INSIDE : 0) |
             (skip_first ? MC_ER_SKIP : 0);
    r.fill_blk = fill_blk;
    r.mod_idx = mod_idx;
    r.mod_val = mod_val;
    r.ytop = p.wy - 1;
    r.ub = up_none(r.ytop);
    return r;
}

// Repeating 48-byte pattern written with 16-byte stores by nt threads.
__device__ __forceinline__ void fill_pattern16_n(uint8_t* dst, int bytes, uint4 p0, uint4 p1, uint4 p2, int t,
                                                 int nt) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    const int n = bytes >> 4, adv = nt % 3;
    int m = t % 3;
    for (int k = t; k < n; k += nt) {
        d[k] = (m == 0) ? p0 : ((m == 1) ? p1 : p2);
        m += adv;
        if (m >= 3) m -= 3;
    }
}

// The uniform observation of a buried camera, written by nt threads.
template <int FAM, bool F32>
__device__ __forceinline__ void fill_env(const mc_kp& p, long long e, const EnvRender& r, const FusedCtx& cx, int t,
                                         int nt) {
    const int HW = p.W * p.H;
    const long long obs_env_bytes = (long long)HW * 3 * (F32 ? 4 : 1);
    uint8_t* oenv = (uint8_t*)p.obs + e * obs_env_bytes;
    const bool vec_ok = ((obs_env_bytes & 15) == 0) && ((((uintptr_t)oenv) & 15) == 0);
    Hit h;
    h.blk = r.fill_blk;
    h.face = -1;
    h.t = 0.0f;
    h.step_y = 1;
    uint8_t bytes[12];
    if (F32 || FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
        float rgb[3];
        shade_rgb<F32 ? MC_COL_F32 : (FAM == MC_FAM_SHADED_FAST ? MC_COL_U8FAST : MC_COL_U8)>(h, p.vd, cx.rcp_vd,
                                                                                              cx.s_rgb, cx.s_sky, rgb);
        if (F32) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                uint32_t w32 = __float_as_uint(rgb[k]);
                bytes[4 * k + 0] = (uint8_t)(w32);
                bytes[4 * k + 1] = (uint8_t)(w32 >> 8);
                bytes[4 * k + 2] = (uint8_t)(w32 >> 16);
                bytes[4 * k + 3] = (uint8_t)(w32 >> 24);
            }
        } else {
            bytes[0] = (uint8_t)to_u8(rgb[0]);
            bytes[1] = (uint8_t)to_u8(rgb[1]);
            bytes[2] = (uint8_t)to_u8(rgb[2]);
        }
    } else {
        bytes[0] = cx.s_rgb8[r.fill_blk][0];
        bytes[1] = cx.s_rgb8[r.fill_blk][1];
        bytes[2] = cx.s_rgb8[r.fill_blk][2];
    }
    const int period = F32 ? 12 : 3;
    if (vec_ok) {
        uint32_t w[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            w[k] = (uint32_t)bytes[(4 * k + 0) % period] | ((uint32_t)bytes[(4 * k + 1) % period] << 8) |
                   ((uint32_t)bytes[(4 * k + 2) % period] << 16) | ((uint32_t)bytes[(4 * k + 3) % period] << 24);
        }
        fill_pattern16_n(oenv, (int)obs_env_bytes, make_uint4(w[0], w[1], w[2], w[3]),
                         make_uint4(w[4], w[5], w[6], w[7]), make_uint4(w[8], w[9], w[10], w[11]), t, nt);
    } else {
        for (long long k = t; k < obs_env_bytes; k += nt) oenv[k] = bytes[k % period];
    }
    if (p.dbg_pixel) {
        int16_t code = dbg_code(h);
        for (int k = t; k < HW; k += nt) p.dbg_pixel[(long long)e * HW + k] = code;
    }
}

// March row bands of env e's image with one warp: every band when band_ctr is
// null, else the bands this warp claims from the team's shared counter.
template <int FAM, bool F32, class V, bool VDLIM = true>
__device__ __forceinline__ void render_env(const mc_kp& p, long long e, const EnvRender& r, const FusedCtx& cx,
                                           const V& vox, int tile_w, int lane, int* band_ctr) {
    // parameters in registers: p may live in shared memory, which the band
    // stores below would otherwise force to be re-read per pixel
    const int W = p.W, H = p.H;
    const RayPar rp = ray_par(p);
    int16_t* const dbg_pixel = p.dbg_pixel;
    const float vd = p.vd;
    const long long obs_env_bytes = (long long)W * H * 3 * (F32 ? 4 : 1);
    uint8_t* oenv = (uint8_t*)p.obs + e * obs_env_bytes;
    const bool vec_ok = ((obs_env_bytes & 15) == 0) && ((((uintptr_t)oenv) & 15) == 0);
    const bool inside = (r.bits & MC_ER_INSIDE) != 0, skip_first = (r.bits & MC_ER_SKIP) != 0;
    // per-env facts that let the march stop early (see shade_ray / flat_ray)
    const bool eye_inb = (unsigned)(int)floorf(r.c.eye_x) < (unsigned)rp.wx &&
                         (unsigned)(int)floorf(r.c.eye_y) < (unsigned)rp.wy &&
                         (unsigned)(int)floorf(r.c.eye_z) < (unsigned)rp.wz;
    const bool sky_exit = (FAM == MC_FAM_SHADED) ? (inside && rp.vd > 0.0f && !dbg_pixel) : (eye_inb && !dbg_pixel);
    const bool vd_safe = sky_exit && box_within_view(r.c, rp.wx, rp.wy, rp.wz, rp.vd);
    const Dda0 d0 = dda0(r.c);
    const int TW = tile_w, TH = 32 / tile_w;
    const int lx = lane % TW, ly = lane / TW;
    const int bpp = 3 * (F32 ? 4 : 1);
    const int nbands = (H + TH - 1) / TH;
    auto claim = [&]() -> int {
        int v = 0;
        if (lane == 0) v = atomicAdd(band_ctr, 1);
        return __shfl_sync(0xffffffffu, v, 0);
    };
    if constexpr (std::is_same<V, VoxEither>::value &&
                  (FAM == MC_FAM_SHADED || FAM == MC_FAM_MINIMAL || FAM == MC_FAM_PREBASIS)) {
        // the common case (fast_band): staged world, eye inside with air in
        // its voxel, no debug output, whole tiles
        const int fk = fast_kind<FAM>(vox.smem, sky_exit && skip_first, dbg_pixel != nullptr, vd_safe, rp.max_steps,
                                      rp.wx, rp.wy, rp.wz, W, H, TW, bpp, vec_ok);
        if (fk) {
            build_fast_start(cx.sstart, fk, d0, rp.wx, rp.wy, rp.wz, r.ub, rp.max_steps, lane);
            const uint32_t wb = staged_base(vox);
            const int wxz = rp.wx * rp.wz;
            FastEnv fe;
            fe.start = cx.sstart;
            fe.base = fk == 1 ? wb : wb + (uint32_t)(d0.vy * wxz + d0.vx * rp.wz + d0.vz);
            fe.chk = staged_range(wb, wxz, wxz * rp.wy);
            fe.vd = vd;
            fe.rcp_vd = cx.rcp_vd;
            for (int b = band_ctr ? claim() : 0; b < nbands; b = band_ctr ? claim() : b + 1) {
                const int row0 = b * TH;
                uint8_t* dst = oenv + (long long)row0 * W * bpp;
                if (fk == 1)
                    fast_band<FAM, F32, false>(r.c, d0, fe, W, TW, row0, lane, cx.s_u, cx.s_v, cx.s_cs, cx.s_rgbp,
                                               cx.stage, dst);
                else
                    fast_band<FAM, F32, true>(r.c, d0, fe, W, TW, row0, lane, cx.s_u, cx.s_v, cx.s_cs, cx.s_rgbp,
                                              cx.stage, dst);
            }
            return;
        }
    }
    for (int b = band_ctr ? claim() : 0; b < nbands; b = band_ctr ? claim() : b + 1) {
        const int row0 = b * TH;
        const int py = row0 + ly;
        const float v = (py < H && in_bounds(py, H, MC_SITE_TABLE)) ? cx.s_v[py] : 0.0f;
        for (int tx0 = 0; tx0 < W; tx0 += TW) {
            const int px = tx0 + lx;
            if (px < W && py < H && in_bounds(px, W, MC_SITE_TABLE)) {
                const float u = cx.s_u[px];
                Hit h = march_pixel<FAM, V, VDLIM>(rp, r.c, d0, u, v, vox, inside, skip_first, sky_exit, vd_safe,
                                                   r.ytop);
                const int so = ly * W + px;  // pixel within the staged band
                if (!in_bounds((long long)(so + 1) * bpp - 1, (long long)TH * W * bpp, MC_SITE_BAND)) continue;
                if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
                    float rgb[3];
                    shade_rgb<F32 ? MC_COL_F32 : (FAM == MC_FAM_SHADED_FAST ? MC_COL_U8FAST : MC_COL_U8)>(
                        h, vd, cx.rcp_vd, cx.s_rgb, cx.s_sky, rgb);
                    if (F32) {
                        float* sf = reinterpret_cast<float*>(cx.stage) + so * 3;
                        sf[0] = rgb[0];
                        sf[1] = rgb[1];
                        sf[2] = rgb[2];
                    } else {
                        uint8_t* sb = cx.stage + so * 3;
                        sb[0] = (uint8_t)to_u8(rgb[0]);
                        sb[1] = (uint8_t)to_u8(rgb[1]);
                        sb[2] = (uint8_t)to_u8(rgb[2]);
                    }
                } else {
                    const uint8_t* col = (h.blk >= 0 && in_bounds(h.blk, 13, MC_SITE_TABLE)) ? cx.s_rgb8[h.blk] : cx.s_sky8;
                    uint8_t* sb = cx.stage + so * 3;
                    sb[0] = col[0];
                    sb[1] = col[1];
                    sb[2] = col[2];
                }
                if (dbg_pixel && in_bounds(py * W + px, W * H, MC_SITE_DEBUG))
                    dbg_pixel[e * W * H + py * W + px] = dbg_code(h);
            }
        }
        __syncwarp();
        // copy the band (rows row0 .. row0+TH-1) out
        const int nbytes = min(TH, H - row0) * W * bpp;
        uint8_t* dst = oenv + (long long)row0 * W * bpp;
        if (!in_bounds((long long)row0 * W * bpp + nbytes - 1, obs_env_bytes, MC_SITE_COPY_OUT)) {
            __syncwarp();
            continue;
        }
        if (vec_ok && (nbytes & 15) == 0 && (((long long)row0 * W * bpp) & 15) == 0) {
            const uint4* s4 = reinterpret_cast<const uint4*>(cx.stage);
            uint4* d4 = reinterpret_cast<uint4*>(dst);
            for (int k = lane; k < (nbytes >> 4); k += 32) d4[k] = s4[k];
        } else {
            for (int k = lane; k < nbytes; k += 32) dst[k] = cx.stage[k];
        }
        __syncwarp();
    }
}

template <int FAM, bool F32>
__device__ __noinline__ bool fused_finish_from_global(const mc_kp& p, long long e, long long claimed,
                                                      long long total_warps, int tile_w, int lane, FusedCtx cx) {
    const long long wxyz = (long long)p.wx * p.wy * p.wz;
    if (e < p.B) {
        // env e was stepped and found not buried: its camera, as stored by the
        // step, gives the same render constants bit for bit
        EnvRender r;
        const float* cam = p.cameras + e * 5;
        __syncwarp();
        if (FAM == MC_FAM_PREBASIS) {
            float bas[13];
            basis_compute(cam[0], cam[1], cam[2], cam[3], cam[4], p.W, p.H, p.fov, bas);
            r.c = cam_from_basis(bas);
        } else {
            r.c = cam_trig(cam[0], cam[1], cam[2], cam[3], cam[4]);
        }
        const int ey = (int)floorf(r.c.eye_y);
        bool inside = false, skip_first;
        if (FAM == MC_FAM_SHADED || FAM == MC_FAM_SHADED_FAST) {
            inside = eye_inside(r.c, p.wx, p.wy, p.wz, p.vd);
            skip_first = inside && p.vd > 0.0f && p.max_steps > 0 && !(FAM == MC_FAM_SHADED_FAST && ey < p.gh);
        } else {
            skip_first = p.max_steps > 0;  // not buried: the eye's voxel holds air or lies outside the world
        }
        r.bits = (inside ? MC_ER_INSIDE : 0) | (skip_first ? MC_ER_SKIP : 0);
        r.fill_blk = AIR;
        r.mod_idx = -1;
        r.mod_val = 0;
        r.ytop = p.wy - 1;
        r.ub = up_none(r.ytop);
        render_env<FAM, F32, VoxGlobal, false>(p, e, r, cx, VoxGlobal{p.voxels + e * wxyz}, tile_w, lane, nullptr);
        // a depth-2 warp's next env is the one it claimed already
        e = claimed >= 0 ? claimed : next_env(p, e, total_warps, lane);
    }
    bool any_done = false;
    const ActionSrc act{p.actions, p.buttons, p.look};
    for (; e < p.B; e = next_env(p, e, total_warps, lane)) {
        EnvRender r = agent_step<FAM>(p, act, e, lane);
        any_done |= (r.bits & MC_ER_DONE) != 0;
        if (r.bits & MC_ER_BURIED)
            fill_env<FAM, F32>(p, e, r, cx, lane, 32);
        else
            render_env<FAM, F32, VoxGlobal, false>(p, e, r, cx, VoxGlobal{p.voxels + e * wxyz}, tile_w, lane,
                                                   nullptr);
    }
    return any_done;
}

// Start the bulk copy of one world into shared memory (lane 0 issues it).
__device__ __forceinline__ void issue_world_copy(uint32_t mbar_a, int8_t* dst, const int8_t* src, int bytes, int lane) {
    if (lane == 0) {
        // generic-proxy reads of the previous world must precede the copy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_a), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(dst)),
            "l"(src), "r"(bytes), "r"(mbar_a)
            : "memory");
    }
}

// Bulk copy of one world into shared memory, waited for with a bound.
__device__ __forceinline__ bool stage_world(uint32_t mbar_a, uint32_t& phase, int8_t* dst, const int8_t* src,
                                            int bytes, int lane, int polls) {
    issue_world_copy(mbar_a, dst, src, bytes, lane);
    const bool ok = mbar_wait(mbar_a, phase, polls);
    phase ^= 1u;
    return ok;
}

#ifndef MC_TEAM_MIN_BLOCKS
#define MC_TEAM_MIN_BLOCKS 3  // 80 registers: the render path without spills
#endif
template <int FAM, bool F32>
__global__ void __launch_bounds__(256, MC_TEAM_MIN_BLOCKS) k_step_team(const __grid_constant__ mc_ragged_kp rk) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int TWN = rk.team_warps;
    const int team = warp / TWN, wt = warp % TWN;
    const int teams_per_cta = nwarps / TWN;
    const int G = rk.ngroups;
    // layout: colour tables | u/v tables | teams | warps; the groups'
    // parameter blocks stay in the kernel's parameter space
    FusedCtx cx;
    load_colour_tables(smem, cx);
    build_fast_tables(reinterpret_cast<float4*>(smem + MC_COLOUR_TABLE_BYTES),
                      reinterpret_cast<uint32_t*>(smem + MC_COLOUR_TABLE_BYTES + kShadeTableBytes));
    cx.s_cs = reinterpret_cast<const float4*>(smem + MC_COLOUR_TABLE_BYTES);
    cx.s_rgbp = reinterpret_cast<const uint32_t*>(smem + MC_COLOUR_TABLE_BYTES + kShadeTableBytes);
    float* tables = reinterpret_cast<float*>(smem + rk.tables_off);
    for (int g = 0; g < G; ++g)
        build_uv_tables<FAM>(rk.groups[g], tables + rk.uv_off[g], tables + rk.uv_off[g] + rk.groups[g].W);
    TeamShared* ts = reinterpret_cast<TeamShared*>(smem + rk.teams_off + team * rk.team_bytes);
    int8_t* tworld = reinterpret_cast<int8_t*>(ts) + MC_TEAM_HEAD_BYTES;
    uint8_t* wbase = smem + rk.warps_off + warp * rk.warp_bytes;
    cx.mbar_a = smem_u32(wbase);
    cx.sstart = reinterpret_cast<int4*>(wbase + 16);
    cx.stage = wbase + 16 + 128;
    if (rk.stage_mask) mbar_init_warp(cx.mbar_a, lane);
    const bool claimer = (wt == 0 && lane == 0);
    const long long total_teams = (long long)gridDim.x * teams_per_cta;
    const long long my_team = (long long)blockIdx.x * teams_per_cta + team;
    const unsigned total_units = (unsigned)rk.ustart[G];
    auto claim = [&](int k) -> unsigned {
        if (rk.sched_dynamic) return atomicAdd(reinterpret_cast<unsigned*>(&rk.flags[MC_FLAG_WORK]), 1u);
        const long long u = my_team + (long long)k * total_teams;
        return u < (long long)total_units ? (unsigned)u : total_units;
    };
    if (claimer) ts->unit[0] = claim(0);
    __syncthreads();
    const int bar = 1 + team, nthr = TWN * 32;
    uint32_t phase = 0;
    bool warp_no_stage = false;   // a copy of this warp timed out: it renders from global memory from now on
    uint32_t pending_phase = 0;   // that copy's phase, waited for before the warp leaves
    for (int k = 0;; ++k) {
        const unsigned u = ts->unit[k & 1];
        if (u >= total_units) break;
        int vg = 0;
        while (vg + 1 < G && (long long)u >= rk.ustart[vg + 1]) ++vg;
        const int g = rk.order[vg];
        const mc_kp& p = rk.groups[g];
        cx.s_u = tables + rk.uv_off[g];
        cx.s_v = cx.s_u + p.W;
        cx.rcp_vd = N::rcp_of(p.vd);
        const long long local = (long long)u - rk.ustart[vg];
        const int wxyz = p.wx * p.wy * p.wz;
        const bool coop = (rk.coop_mask >> g) & 1;
        // coop: warp 0 steps the env and the team renders it; else each warp
        // steps and renders its own env of the unit
        const long long e = coop ? local : local * TWN + wt;
        const bool stepper = coop ? (wt == 0) : (e < p.B);
        const int8_t* gw = p.voxels + e * (long long)wxyz;
        int8_t* world = coop ? tworld : tworld + wt * rk.slot_bytes;
        EnvRender r;
        bool staged = false;
        if (stepper) {
            const long long s0 = rk.start[g];
            const ActionSrc act{rk.actions ? rk.actions + s0 : nullptr, rk.actions ? nullptr : rk.buttons + 8 * s0,
                                rk.actions ? nullptr : rk.look + 2 * s0};
            // the world's bulk copy starts before the agent step, which it
            // overlaps (the voxel the interaction changes is patched in after it
            // lands); a buried env's copy is waited for and not used
            bool copying = ((rk.stage_mask >> g) & 1) && !warp_no_stage;
#if MC_CHECK_BOUNDS
            if (copying) {
                const SmemRange dyn = dyn_smem_range();
                const long long off = (long long)smem_u32(world) - dyn.lo;
                if (!in_bounds(off, dyn.span, MC_SITE_STAGE) || !in_bounds(off + wxyz - 1, dyn.span, MC_SITE_STAGE))
                    copying = false;  // no copy issued: render from global memory
            }
#endif
            if (copying) issue_world_copy(cx.mbar_a, world, gw, wxyz, lane);
            r = agent_step<FAM>(p, act, e, lane);
            if (lane == 0) {
                // rare: set as the env ends (a per-team mask of groups would
                // stay live across the loop and spill)
                if (r.bits & MC_ER_DONE) atomicOr(&p.flags[MC_FLAG_ANY_DONE], 1);
                if (rk.rewards_cat) {
                    rk.rewards_cat[rk.start[g] + e] = p.rewards[e];
                    rk.dones_cat[rk.start[g] + e] = (uint8_t)(r.bits & MC_ER_DONE);
                }
            }
            staged = copying && !(r.bits & MC_ER_BURIED);
            if (copying) {
                const uint32_t ph = phase;
                const bool landed = mbar_wait(cx.mbar_a, phase, p.wait_polls);
                phase ^= 1u;
                if (!landed) {
                    if (lane == 0) atomicExch(&p.flags[MC_FLAG_ERROR], MC_KERR_TMA_TIMEOUT);
                    warp_no_stage = true;  // the copy may still land: render from global memory from now on
                    pending_phase = ph;
                    staged = false;
                } else if (staged) {
                    // the interaction may have written after the copy read the byte
                    if (lane == 0 && r.mod_idx >= 0 && in_bounds(r.mod_idx, wxyz, MC_SITE_PATCH))
                        world[r.mod_idx] = (int8_t)r.mod_val;
                    __syncwarp();
                    if (coop && TWN > 1 && eye_in_box(r.c, p.wx, p.wy, p.wz) && up_scan_shape(p.wx, p.wy, p.wz))
                        r.bits |= MC_ER_TSCAN;  // the whole team scans, after the barrier
                    else
                        measure_staged(r, world, p.wx, p.wy, p.wz, lane);
                }
            }
            if (coop && lane == 0) {
                r.bits |= staged ? MC_ER_STAGED : 0;
                ts->r = r;
                ts->band_ctr = 0;
                if (r.bits & MC_ER_TSCAN) team_up_reset(ts);
            }
            __syncwarp();
        }
        if (coop) {
            team_sync(bar, nthr);
            r = ts->r;
            staged = (r.bits & MC_ER_STAGED) != 0;
            if (r.bits & MC_ER_TSCAN) {  // team-uniform
                r.ub = team_up_bounds(world, p.wx, p.wy, p.wz, (int)floorf(r.c.eye_x), (int)floorf(r.c.eye_y),
                                      (int)floorf(r.c.eye_z), lane, wt, TWN, ts, bar);
                r.ytop = up_top(r.ub);
            }
        }
        if (coop || stepper) {
            if (r.bits & MC_ER_BURIED)
                fill_env<FAM, F32>(p, e, r, cx, coop ? wt * 32 + lane : lane, coop ? nthr : 32);
            else
                render_env<FAM, F32>(p, e, r, cx, VoxEither{staged ? world : gw, staged}, rk.tile_w[g], lane,
                                     coop ? &ts->band_ctr : nullptr);
        }
        if (claimer) ts->unit[(k + 1) & 1] = claim(k + 1);
        team_sync(bar, nthr);
    }
    // a timed-out copy may still be in flight: let it land (bounded) before
    // this warp's part of shared memory can be released
    if (warp_no_stage) mbar_wait(cx.mbar_a, pending_phase);
    if (lane == 0) {
        for (int g = 0; g < G; ++g) bounds_to_flags(rk.groups[g].flags);
    }
    if (claimer && rk.sched_dynamic) finish_dynamic(rk.flags, total_teams);
}

// ---------------------------------------------------------------------------
// Team kernel with staging depth 2
// ---------------------------------------------------------------------------
// The same work as k_step_team, pipelined one unit deep: each team holds two
// claimed units.  Before a team renders unit k, the warp(s) that step unit
// k+1 run its agent step and start its world's bulk copy into the second
// world buffer (and the second mbarrier) of their slot, so the copy and the
// agent step overlap the render of unit k; the copy is waited for only when
// unit k+1 is rendered.  The env's render constants wait in a per-warp
// shared-memory stash between the two.
static_assert(sizeof(EnvRender) <= MC_ENV_STASH_BYTES, "env stash");

template <int FAM, bool F32>
__global__ void __launch_bounds__(256, MC_TEAM_MIN_BLOCKS) k_step_team2(const __grid_constant__ mc_ragged_kp rk) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int TWN = rk.team_warps;
    const int team = warp / TWN, wt = warp % TWN;
    const int teams_per_cta = nwarps / TWN;
    const int G = rk.ngroups;
    FusedCtx cx;
    load_colour_tables(smem, cx);
    build_fast_tables(reinterpret_cast<float4*>(smem + MC_COLOUR_TABLE_BYTES),
                      reinterpret_cast<uint32_t*>(smem + MC_COLOUR_TABLE_BYTES + kShadeTableBytes));
    cx.s_cs = reinterpret_cast<const float4*>(smem + MC_COLOUR_TABLE_BYTES);
    cx.s_rgbp = reinterpret_cast<const uint32_t*>(smem + MC_COLOUR_TABLE_BYTES + kShadeTableBytes);
    float* tables = reinterpret_cast<float*>(smem + rk.tables_off);
    for (int g = 0; g < G; ++g)
        build_uv_tables<FAM>(rk.groups[g], tables + rk.uv_off[g], tables + rk.uv_off[g] + rk.groups[g].W);
    TeamShared* ts = reinterpret_cast<TeamShared*>(smem + rk.teams_off + team * rk.team_bytes);
    int8_t* tworld = reinterpret_cast<int8_t*>(ts) + MC_TEAM_HEAD_BYTES;
    uint8_t* wbase = smem + rk.warps_off + warp * rk.warp_bytes;
    const uint32_t mbar0 = smem_u32(wbase);  // depth slot d's mbarrier at mbar0 + 8 d
    cx.sstart = reinterpret_cast<int4*>(wbase + 16);
    EnvRender* stash = reinterpret_cast<EnvRender*>(wbase + 16 + 128);  // depth slot d's env at + 96 d
    cx.stage = wbase + 16 + 128 + 2 * MC_ENV_STASH_BYTES;
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0 + 8) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const bool claimer = (wt == 0 && lane == 0);
    const long long total_teams = (long long)gridDim.x * teams_per_cta;
    const long long my_team = (long long)blockIdx.x * teams_per_cta + team;
    const unsigned total_units = (unsigned)rk.ustart[G];
    auto claim = [&](int k) -> unsigned {
        if (rk.sched_dynamic) return atomicAdd(reinterpret_cast<unsigned*>(&rk.flags[MC_FLAG_WORK]), 1u);
        const long long u = my_team + (long long)k * total_teams;
        return u < (long long)total_units ? (unsigned)u : total_units;
    };
    if (claimer) {
        ts->unit[0] = claim(0);
        ts->unit[1] = claim(1);
    }
    __syncthreads();
    const int bar = 1 + team, nthr = TWN * 32;
    uint32_t phases = 0;          // bit d: parity of depth slot d's next wait
    bool warp_no_stage = false;   // a copy of this warp timed out: no more copies, render from global memory
    uint32_t pending = 0;         // bit d: a timed-out copy into slot d may still be in flight
    uint32_t pending_phases = 0;  // bit d: its parity

    // Where unit u lies: its group, env, and whether this warp steps it.
    struct Unit {
        int g;
        long long e;
        bool coop, stepper;
    };
    auto locate = [&](unsigned u) -> Unit {
        int vg = 0;
        while (vg + 1 < G && (long long)u >= rk.ustart[vg + 1]) ++vg;
        Unit t;
        t.g = rk.order[vg];
        const long long local = (long long)u - rk.ustart[vg];
        t.coop = (rk.coop_mask >> t.g) & 1;
        t.e = t.coop ? local : local * TWN + wt;
        t.stepper = t.coop ? (wt == 0) : (t.e < rk.groups[t.g].B);
        return t;
    };
    auto slot_world = [&](int d, bool coop) -> int8_t* {
        return tworld + d * rk.world_stride + (coop ? 0 : wt * rk.slot_bytes);
    };
    // The stepper of unit u steps its env and starts its world's copy into depth slot d.
    auto prepare = [&](unsigned u, int d) {
        const Unit t = locate(u);
        if (!t.stepper) return;
        const mc_kp& p = rk.groups[t.g];
        const int wxyz = p.wx * p.wy * p.wz;
        const long long s0 = rk.start[t.g];
        const ActionSrc act{rk.actions ? rk.actions + s0 : nullptr, rk.actions ? nullptr : rk.buttons + 8 * s0,
                            rk.actions ? nullptr : rk.look + 2 * s0};
        EnvRender r = agent_step<FAM>(p, act, t.e, lane);
        if (lane == 0) {
            if (r.bits & MC_ER_DONE) atomicOr(&p.flags[MC_FLAG_ANY_DONE], 1);  // rare: set as the env ends
            if (rk.rewards_cat) {
                rk.rewards_cat[s0 + t.e] = p.rewards[t.e];
                rk.dones_cat[s0 + t.e] = (uint8_t)(r.bits & MC_ER_DONE);
            }
        }
        bool staged = ((rk.stage_mask >> t.g) & 1) && !(r.bits & MC_ER_BURIED) && !warp_no_stage;
        int8_t* world = slot_world(d, t.coop);
#if MC_CHECK_BOUNDS
        if (staged) {
            const SmemRange dyn = dyn_smem_range();
            const long long off = (long long)smem_u32(world) - dyn.lo;
            if (!in_bounds(off, dyn.span, MC_SITE_STAGE) || !in_bounds(off + wxyz - 1, dyn.span, MC_SITE_STAGE))
                staged = false;  // no copy issued: render from global memory
        }
#endif
        if (staged && lane == 0) {
            const uint32_t mb = mbar0 + 8 * d;
            // generic-proxy reads of the slot's previous world must precede the copy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(wxyz) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(world)),
                "l"(p.voxels + t.e * (long long)wxyz), "r"(wxyz), "r"(mb)
                : "memory");
        }
        r.bits |= staged ? MC_ER_STAGED : 0;
        if (lane == 0) stash[d] = r;
        __syncwarp();
    };
    // The stepper of unit u (slot d): wait for the world, patch and measure it.
    auto finish = [&](const Unit& t, int d) {
        const mc_kp& p = rk.groups[t.g];
        const int wxyz = p.wx * p.wy * p.wz;
        EnvRender r = stash[d];
        if (r.bits & MC_ER_STAGED) {
            int8_t* world = slot_world(d, t.coop);
            const uint32_t ph = (phases >> d) & 1u;
            if (mbar_wait(mbar0 + 8 * d, ph, p.wait_polls)) {
                // the interaction may have written after the copy read the byte
                if (lane == 0 && r.mod_idx >= 0 && in_bounds(r.mod_idx, wxyz, MC_SITE_PATCH))
                    world[r.mod_idx] = (int8_t)r.mod_val;
                __syncwarp();
                measure_staged(r, world, p.wx, p.wy, p.wz, lane);
            } else {
                if (lane == 0) atomicExch(&p.flags[MC_FLAG_ERROR], MC_KERR_TMA_TIMEOUT);
                warp_no_stage = true;  // the copy may still land: render from global memory from now on
                pending |= 1u << d;
                pending_phases = (pending_phases & ~(1u << d)) | (ph << d);
                r.bits &= ~MC_ER_STAGED;
            }
            phases ^= 1u << d;
        }
        if (lane == 0) {
            if (t.coop) {
                ts->r = r;
                ts->band_ctr = 0;
            } else {
                stash[d] = r;
            }
        }
        __syncwarp();
    };

    if (ts->unit[0] < total_units) prepare(ts->unit[0], 0);
    for (int k = 0;; ++k) {
        const int d = k & 1;
        const unsigned u = ts->unit[d];
        if (u >= total_units) break;
        const Unit t = locate(u);
        if (t.stepper) finish(t, d);
        if (t.coop) team_sync(bar, nthr);
        // step the next unit and start its copy, then render this one
        const unsigned u1 = ts->unit[d ^ 1];
        if (u1 < total_units) prepare(u1, d ^ 1);
        const mc_kp& p = rk.groups[t.g];
        if (t.coop || t.stepper) {
            const EnvRender r = t.coop ? ts->r : stash[d];
            cx.s_u = tables + rk.uv_off[t.g];
            cx.s_v = cx.s_u + p.W;
            cx.rcp_vd = N::rcp_of(p.vd);
            const bool staged = (r.bits & MC_ER_STAGED) != 0;
            const int8_t* gw = p.voxels + t.e * (long long)p.wx * p.wy * p.wz;
            if (r.bits & MC_ER_BURIED)
                fill_env<FAM, F32>(p, t.e, r, cx, t.coop ? wt * 32 + lane : lane, t.coop ? nthr : 32);
            else
                render_env<FAM, F32>(p, t.e, r, cx, VoxEither{staged ? slot_world(d, t.coop) : gw, staged},
                                     rk.tile_w[t.g], lane, t.coop ? &ts->band_ctr : nullptr);
        }
        if (claimer) ts->unit[d] = claim(k + 2);
        team_sync(bar, nthr);
    }
    // timed-out copies may still be in flight: let them land (bounded)
    // before this warp's part of shared memory can be released
    for (int d = 0; d < 2; ++d)
        if ((pending >> d) & 1u) mbar_wait(mbar0 + 8 * d, (pending_phases >> d) & 1u);
    if (lane == 0) {
        for (int g = 0; g < G; ++g) bounds_to_flags(rk.groups[g].flags);
    }
    if (claimer && rk.sched_dynamic) finish_dynamic(rk.flags, total_teams);
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline int grid_1d(long long n, int bs) { return (int)((n + bs - 1) / bs); }

static int render_launch(const mc_kp* p, int family, cudaStream_t s) {
    long long total = (long long)p->B * p->H * p->W;
    if (total == 0) return 0;
    switch (family) {
        case MC_FAM_SHADED:
            if (p->obs_f32) k_render_shaded<false, true><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            else k_render_shaded<false, false><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            break;
        case MC_FAM_SHADED_FAST:
            k_render_shaded<true, false><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            break;
        case MC_FAM_MINIMAL:
            k_render_flat<MC_FAM_MINIMAL><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            break;
        case MC_FAM_FP16:
            k_render_flat<MC_FAM_FP16><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            break;
        case MC_FAM_PREBASIS:
            k_render_flat<MC_FAM_PREBASIS><<<grid_1d(total, 128), 128, 0, s>>>(*p);
            break;
        default:
            return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

// The reference's step kernel sequence (kernels.cu:2457-2494, 2909-2991):
// episode check, decode, physics, interact, reset, counter, cameras,
// (basis), render.  World regeneration is launched by the caller.
static int step_plain(const mc_kp* p, cudaStream_t s) {
    if (p->B == 0) return 0;
    int gb = grid_1d(p->B, 256);
    k_episode_check<<<gb, 256, 0, s>>>(*p);
    k_decode<<<gb, 256, 0, s>>>(*p);
    k_physics<<<gb, 256, 0, s>>>(*p);
    k_interact<<<gb, 256, 0, s>>>(*p, 0);
    k_reset<<<gb, 256, 0, s>>>(*p);
    k_episode_update<<<gb, 256, 0, s>>>(*p);
    k_cameras<<<gb, 256, 0, s>>>(*p);
    if (p->family == MC_FAM_PREBASIS) k_basis<<<gb, 256, 0, s>>>(*p);
    int rc = (int)cudaGetLastError();
    if (rc) return rc;
    return render_launch(p, p->family, s);
}

static size_t fused_smem(const mc_kp* p, const mc_fused_cfg* cfg) {
    int wxyz = p->wx * p->wy * p->wz;
    FusedLayout L = fused_layout(p->W, p->H, wxyz, p->wx * p->wz, p->obs_f32, cfg->stage, cfg->tile_w);
    return (size_t)L.head_bytes + (size_t)cfg->warps_per_cta * L.warp_bytes + (size_t)L.pad_bytes;
}

template <int FAM, bool F32, int DEPTH>
static int launch_fused_t(const mc_kp* p, const mc_fused_cfg* cfg, int num_sms, cudaStream_t s) {
    auto kern = k_step_fused<FAM, F32, DEPTH>;
    size_t smem = fused_smem(p, cfg);
    static size_t attr_set = 0;  // per instantiation
    if (smem > 48 * 1024 && smem > attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        attr_set = smem;
    }
    int threads = 32 * cfg->warps_per_cta;
    long long ctas_needed = ((long long)p->B + cfg->warps_per_cta - 1) / cfg->warps_per_cta;
    long long grid = (long long)num_sms * (cfg->ctas_per_sm > 0 ? cfg->ctas_per_sm : 1);
    if (grid > ctas_needed) grid = ctas_needed;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, threads, smem, s>>>(*p, cfg->tile_w);
    return (int)cudaGetLastError();
}

template <int FAM, bool F32>
static int launch_fused_f(const mc_kp* p, const mc_fused_cfg* cfg, int num_sms, cudaStream_t s) {
    if (cfg->stage == 2) return launch_fused_t<FAM, F32, 2>(p, cfg, num_sms, s);
    return cfg->stage ? launch_fused_t<FAM, F32, 1>(p, cfg, num_sms, s) : launch_fused_t<FAM, F32, 0>(p, cfg, num_sms, s);
}

template <int FAM, bool F32>
static int launch_team_t(const mc_ragged_kp* rk, int warps_per_cta, int ctas_per_sm, int num_sms, cudaStream_t s) {
    const bool deep = rk->depth == 2;
    auto kern = deep ? k_step_team2<FAM, F32> : k_step_team<FAM, F32>;
    size_t smem = (size_t)rk->warps_off + (size_t)warps_per_cta * rk->warp_bytes + (size_t)rk->tail_bytes;
    static size_t attr_set[2] = {0, 0};  // per kernel of this instantiation
    if (smem > 48 * 1024 && smem > attr_set[deep]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        attr_set[deep] = smem;
    }
    const int teams_per_cta = warps_per_cta / rk->team_warps;
    long long ctas_needed = (rk->ustart[rk->ngroups] + teams_per_cta - 1) / teams_per_cta;
    long long grid = (long long)num_sms * (ctas_per_sm > 0 ? ctas_per_sm : 1);
    if (grid > ctas_needed) grid = ctas_needed;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, 32 * warps_per_cta, smem, s>>>(*rk);
    return (int)cudaGetLastError();
}

static int step_team(const mc_ragged_kp* rk, int family, int obs_f32, int warps_per_cta, int ctas_per_sm,
                     int num_sms, cudaStream_t s) {
    if (rk->ustart[rk->ngroups] == 0) return 0;
    switch (family) {
        case MC_FAM_SHADED:
            return obs_f32 ? launch_team_t<MC_FAM_SHADED, true>(rk, warps_per_cta, ctas_per_sm, num_sms, s)
                           : launch_team_t<MC_FAM_SHADED, false>(rk, warps_per_cta, ctas_per_sm, num_sms, s);
        case MC_FAM_SHADED_FAST: return launch_team_t<MC_FAM_SHADED_FAST, false>(rk, warps_per_cta, ctas_per_sm, num_sms, s);
        case MC_FAM_MINIMAL: return launch_team_t<MC_FAM_MINIMAL, false>(rk, warps_per_cta, ctas_per_sm, num_sms, s);
        case MC_FAM_FP16: return launch_team_t<MC_FAM_FP16, false>(rk, warps_per_cta, ctas_per_sm, num_sms, s);
        case MC_FAM_PREBASIS: return launch_team_t<MC_FAM_PREBASIS, false>(rk, warps_per_cta, ctas_per_sm, num_sms, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

static int step_fused(const mc_kp* p, const mc_fused_cfg* cfg, int num_sms, cudaStream_t s) {
    if (p->B == 0) return 0;
    switch (p->family) {
        case MC_FAM_SHADED:
            return p->obs_f32 ? launch_fused_f<MC_FAM_SHADED, true>(p, cfg, num_sms, s)
                              : launch_fused_f<MC_FAM_SHADED, false>(p, cfg, num_sms, s);
        case MC_FAM_SHADED_FAST: return launch_fused_f<MC_FAM_SHADED_FAST, false>(p, cfg, num_sms, s);
        case MC_FAM_MINIMAL: return launch_fused_f<MC_FAM_MINIMAL, false>(p, cfg, num_sms, s);
        case MC_FAM_FP16: return launch_fused_f<MC_FAM_FP16, false>(p, cfg, num_sms, s);
        case MC_FAM_PREBASIS: return launch_fused_f<MC_FAM_PREBASIS, false>(p, cfg, num_sms, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

#if MC_CHECK_BOUNDS
// One failed check with no memory access behind it: shows that a violation
// reaches the record (the checks themselves cannot be made to fail on
// purpose without an out-of-range access to skip).
__global__ void k_bounds_selftest() {
    if (threadIdx.x == 0) (void)in_bounds(-1, 1, 0);
}
#endif
static int bounds_selftest(cudaStream_t s) {
#if MC_CHECK_BOUNDS
    k_bounds_selftest<<<1, 32, 0, s>>>();
    return (int)cudaGetLastError();
#else
    (void)s;
    return -1;
#endif
}

// The debug build's bounds-check record: out = {violations, first site,
// first index, its limit}, then cleared.  -1 (and out untouched) in the
// normal build, which checks nothing.
static int bounds_report(int32_t out[4], cudaStream_t s) {
#if MC_CHECK_BOUNDS
    int32_t h[4];
    cudaError_t e = cudaMemcpyFromSymbolAsync(h, g_bounds, sizeof(h), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return (int)e;
    const int32_t zero[4] = {0, 0, 0, 0};
    e = cudaMemcpyToSymbolAsync(g_bounds, zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return (int)e;
    for (int i = 0; i < 4; ++i) out[i] = h[i];
    return 0;
#else
    (void)out;
    (void)s;
    return -1;
#endif
}

static int basis_launch(const mc_kp* p, cudaStream_t s) {
    if (p->B == 0) return 0;
    k_basis<<<grid_1d(p->B, 256), 256, 0, s>>>(*p);
    return (int)cudaGetLastError();
}
static int decode_launch(const mc_kp* p, cudaStream_t s) {
    if (p->B == 0) return 0;
    k_decode<<<grid_1d(p->B, 256), 256, 0, s>>>(*p);
    return (int)cudaGetLastError();
}
static int physics_launch(const mc_kp* p, cudaStream_t s) {
    if (p->B == 0) return 0;
    k_physics<<<grid_1d(p->B, 256), 256, 0, s>>>(*p);
    return (int)cudaGetLastError();
}
static int interact_launch(const mc_kp* p, int break_only, cudaStream_t s) {
    if (p->B == 0) return 0;
    k_interact<<<grid_1d(p->B, 256), 256, 0, s>>>(*p, break_only);
    return (int)cudaGetLastError();
}
static int coalesced_launch(const int8_t* vox, const float* basis, uint8_t* out, int B, int ws, int W, int H,
                            int max_steps, cudaStream_t s) {
    if (B == 0 || W * H == 0) return 0;
    dim3 g(W * H, (B + 127) / 128);
    k_render_coalesced<<<g, 128, 0, s>>>(vox, basis, out, B, ws, W, H, max_steps);
    return (int)cudaGetLastError();
}

}  // namespace MC_NS
