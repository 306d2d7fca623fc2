// mc_runtime.cu - host runtime and C-ABI of libminecu_b200.so.
//
// Owns what the reference keeps in Python or in process-global statics:
// the env handle (minecu/__init__.py MineEnv), the world template and its
// regeneration (minecu/__init__.py:258-268, 356-359, 439-442), masked
// reset (minecu/__init__.py:270-302), CUDA-graph capture of fused rollouts
// (the reference's StepGraphState, src/kernels.cu:2338-2382, which keys its
// graph on 3 of the ~20 pointers it bakes in; here the cache key is every
// pointer the graph uses), and argument checking (the reference checks only
// device/dtype of a few tensors, src/bindings.cpp:223-228).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/minecu_b200.h"
#include "mc_env_impl.h"
#include "mc_internal.h"
#include "mc_philox.h"

#ifndef MC_CHECK_BOUNDS
#define MC_CHECK_BOUNDS 0
#endif
#define MC_CHECK_BOUNDS_BUILD MC_CHECK_BOUNDS

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local char g_err[512];

static int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

static int cuda_fail(cudaError_t e, const char* what) {
    return fail(MC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define MC_CK(call)                                            \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);    \
    } while (0)

static int backend_rc(int rc, const char* what) {
    if (rc == 0) return MC_OK;
    return cuda_fail((cudaError_t)rc, what);
}

int mc_set_error(int code, const char* msg) { return fail(code, "%s", msg); }

int mc_fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int mc_cuda_fail(cudaError_t e, const char* what) { return cuda_fail(e, what); }

extern "C" int mc_abi_version(void) { return MC_ABI_VERSION; }
extern "C" const char* mc_last_error(void) { return g_err; }

// ---------------------------------------------------------------------------
// numerics-independent kernels
// ---------------------------------------------------------------------------
namespace {

constexpr int8_t AIR = -1, GRASS = 0, DIRT = 1, OAKLOG = 3, LEAVES = 4, BRICK = 8, COBBLESTONE = 9,
                 PLANKS = 10, BEDROCK = 12;

// generate_world_kernel (kernels.cu:1793-1828): y=0 bedrock, 1 <= y < gh-1
// dirt, y = gh-1 grass, air above.  One thread per (env, y, x) row of z.
__global__ void k_generate_world(int8_t* vox, long long rows, int wx, int wy, int wz, int gh) {
    long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int y = (int)((r / wx) % wy);
    int8_t blk = AIR;
    if (y == 0) blk = BEDROCK;
    else if (y < gh - 1) blk = DIRT;
    else if (y == gh - 1) blk = GRASS;
    int8_t* row = vox + r * wz;
    for (int z = 0; z < wz; ++z) row[z] = blk;
}

// place_tree_kernel (kernels.cu:1831-1865)
__global__ void k_place_tree(int8_t* vox, int B, int wx, int wy, int wz, int tx, int tz, int gh) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    long long wxz = (long long)wx * wz, wxyz = wxz * wy;
    for (int dy = 0; dy < 3; ++dy) {
        int y = gh + dy;
        if (y < wy) vox[b * wxyz + y * wxz + (long long)tx * wz + tz] = OAKLOG;
    }
    int ly = gh + 3;
    if (ly < wy) vox[b * wxyz + ly * wxz + (long long)tx * wz + tz] = LEAVES;
}

// place_house_kernel (kernels.cu:1868-1946)
__device__ __forceinline__ void house_set(int8_t* w, int wx, int wy, int wz, int hx, int hz, int gh, int dy, int dx,
                                          int dz, int8_t blk) {
    int vx = hx + dx, vy = gh + dy, vz = hz + dz;
    if (vx >= 0 && vx < wx && vy >= 0 && vy < wy && vz >= 0 && vz < wz)
        w[(long long)vy * wx * wz + (long long)vx * wz + vz] = blk;
}

__global__ void k_place_house(int8_t* vox, int B, int wx, int wy, int wz, int hx, int hz, int gh) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int W = 5, D = 4, H = 4;
    int8_t* w = vox + (long long)b * wx * wy * wz;
    for (int dx = 0; dx < W; ++dx)
        for (int dz = 0; dz < D; ++dz) house_set(w, wx, wy, wz, hx, hz, gh, 0, dx, dz, COBBLESTONE);
    for (int dy = 1; dy <= 3; ++dy) {
        for (int dx = 0; dx < W; ++dx) {
            if (dx == 2 && dy <= 2) continue;  // door
            house_set(w, wx, wy, wz, hx, hz, gh, dy, dx, 0, PLANKS);
        }
        for (int dx = 0; dx < W; ++dx) house_set(w, wx, wy, wz, hx, hz, gh, dy, dx, D - 1, PLANKS);
        for (int dz = 1; dz < D - 1; ++dz) house_set(w, wx, wy, wz, hx, hz, gh, dy, 0, dz, PLANKS);
        for (int dz = 1; dz < D - 1; ++dz) house_set(w, wx, wy, wz, hx, hz, gh, dy, W - 1, dz, PLANKS);
    }
    for (int dy = 1; dy <= 3; ++dy) {
        house_set(w, wx, wy, wz, hx, hz, gh, dy, 0, 0, OAKLOG);
        house_set(w, wx, wy, wz, hx, hz, gh, dy, W - 1, 0, OAKLOG);
        house_set(w, wx, wy, wz, hx, hz, gh, dy, 0, D - 1, OAKLOG);
        house_set(w, wx, wy, wz, hx, hz, gh, dy, W - 1, D - 1, OAKLOG);
    }
    for (int dx = 0; dx < W; ++dx)
        for (int dz = 0; dz < D; ++dz) house_set(w, wx, wy, wz, hx, hz, gh, H, dx, dz, BRICK);
}

// Regenerate every world from the template (generate + tree + house give the
// same bytes for every env, so one generated world is broadcast).  With
// `conditional`, nothing is written unless flags[ANY_DONE] is set.  The last
// CTA to finish clears the flag for the next step; every CTA reads the flag
// before it arrives on the counter, so no CTA can see the cleared value.
__global__ void k_regen(int8_t* vox, const int8_t* tmpl, int B, int wxyz, int32_t* flags, int conditional) {
    __shared__ int go;
    if (threadIdx.x == 0) go = conditional ? (*(volatile int32_t*)&flags[MC_FLAG_ANY_DONE] != 0) : 1;
    __syncthreads();
    // The flag was set before this launch and only its last CTA clears it,
    // after every CTA has read it: all CTAs read the same value, so when it
    // is clear none of them has anything to write, count or clear.
    if (!go) return;
    {
        // 16-byte stores only when every world starts on a 16-byte boundary
        // (a voxels view may start at any byte offset)
        if ((wxyz & 15) == 0 && ((((uintptr_t)vox) | ((uintptr_t)tmpl)) & 15) == 0) {
            const int n16 = wxyz >> 4;
            const uint4* t4 = reinterpret_cast<const uint4*>(tmpl);
            for (long long b = blockIdx.x; b < B; b += gridDim.x) {
                uint4* d4 = reinterpret_cast<uint4*>(vox + b * (long long)wxyz);
                for (int k = threadIdx.x; k < n16; k += blockDim.x) d4[k] = __ldg(t4 + k);
            }
        } else {
            for (long long b = blockIdx.x; b < B; b += gridDim.x) {
                int8_t* d = vox + b * (long long)wxyz;
                for (int k = threadIdx.x; k < wxyz; k += blockDim.x) d[k] = tmpl[k];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned prev = atomicAdd(reinterpret_cast<unsigned*>(&flags[MC_FLAG_REGEN_CTR]), 1u);
        if (prev == gridDim.x - 1) {
            flags[MC_FLAG_ANY_DONE] = 0;
            flags[MC_FLAG_REGEN_CTR] = 0;
            __threadfence();
        }
    }
}

// MineEnv.reset(mask) steps 1-3 (minecu/__init__.py:286-294): do_reset =
// mask (or all), reset_kernel on those envs (kernels.cu:1760-1786),
// step_count = 0 there; and the `mask.any()` test as a device flag.
__global__ void k_reset_masked(mc_kp p, const uint8_t* mask) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool m = false;
    if (i < p.B) {
        m = mask ? (mask[i] != 0) : true;
        p.do_reset[i] = m ? 1 : 0;
        if (m) {
            p.positions[i * 3 + 0] = p.spawn_x;
            p.positions[i * 3 + 1] = p.spawn_y;
            p.positions[i * 3 + 2] = p.spawn_z;
            p.velocities[i * 3 + 0] = 0.0f;
            p.velocities[i * 3 + 1] = 0.0f;
            p.velocities[i * 3 + 2] = 0.0f;
            p.yaws[i] = 0.0f;
            p.pitches[i] = 0.0f;
            p.on_ground[i] = 0;
            p.step_count[i] = 0;
        }
    }
    unsigned any = __ballot_sync(0xffffffffu, m);
    if (any && (threadIdx.x & 31) == 0) atomicOr(&p.flags[MC_FLAG_ANY_DONE], 1);
}

// reset_kernel (kernels.cu:1760-1786) as the stand-alone _C.reset
__global__ void k_reset_agents(float* pos, float* vel, float* yaw, float* pitch, uint8_t* og, const uint8_t* dr,
                               int B, float sx, float sy, float sz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B || !dr[i]) return;
    pos[i * 3 + 0] = sx;
    pos[i * 3 + 1] = sy;
    pos[i * 3 + 2] = sz;
    vel[i * 3 + 0] = 0.0f;
    vel[i * 3 + 1] = 0.0f;
    vel[i * 3 + 2] = 0.0f;
    yaw[i] = 0.0f;
    pitch[i] = 0.0f;
    og[i] = 0;
}

// update_cameras_kernel (kernels.cu:2320-2335)
__global__ void k_cameras_rt(mc_kp p) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.B) return;
    p.cameras[i * 5 + 0] = p.positions[i * 3 + 0];
    p.cameras[i * 5 + 1] = p.positions[i * 3 + 1];
    p.cameras[i * 5 + 2] = p.positions[i * 3 + 2];
    p.cameras[i * 5 + 3] = p.yaws[i];
    p.cameras[i * 5 + 4] = p.pitches[i];
}

__global__ void k_philox(uint8_t* actions, int B, int K, int env_offset, int step0, uint64_t seed, int break_half) {
    long long n = (long long)B * K;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int k = (int)(i / B), b = (int)(i - (long long)k * B);
        actions[i] = mc_action_draw(seed, (uint32_t)(env_offset + b), (uint32_t)(step0 + k), break_half);
    }
}

__global__ void k_discrete(const uint8_t* a, int B, float ld, int8_t* btn, float* look) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    int8_t b[8];
    float l[2];
    mc_discrete_to_buttons(a[i], ld, b, l);
    for (int k = 0; k < 8; ++k) btn[(long long)i * 8 + k] = b[k];
    look[(long long)i * 2 + 0] = l[0];
    look[(long long)i * 2 + 1] = l[1];
}

inline int blocks(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

int mc_launch_reset_agents(const mc_kp* p, const uint8_t* mask, cudaStream_t s) {
    if (p->B == 0) return 0;
    k_reset_masked<<<blocks(p->B, 256), 256, 0, s>>>(*p, mask);
    return (int)cudaGetLastError();
}

// Per-env regeneration (MC_REGEN_PER_ENV): the world of every env whose
// do_reset is set this step is copied from the template, the others are left
// alone; the all-world rule's flag is cleared unused.  The rule of the
// reference's unused masked kernels (src/kernels.cu:1988-2069), except that
// the template also holds the house, as every world does at the start.
__global__ void k_regen_masked(int8_t* vox, const int8_t* tmpl, const uint8_t* do_reset, int B, int wxyz,
                               int32_t* flags) {
    if (blockIdx.x == 0 && threadIdx.x == 0) flags[MC_FLAG_ANY_DONE] = 0;
    for (long long b = blockIdx.x; b < B; b += gridDim.x) {
        if (!do_reset[b]) continue;  // the same value for every thread of the CTA
        if ((wxyz & 15) == 0 && ((((uintptr_t)vox) | ((uintptr_t)tmpl)) & 15) == 0) {
            uint4* d4 = reinterpret_cast<uint4*>(vox + b * (long long)wxyz);
            const uint4* t4 = reinterpret_cast<const uint4*>(tmpl);
            for (int k = threadIdx.x; k < (wxyz >> 4); k += blockDim.x) d4[k] = __ldg(t4 + k);
        } else {
            int8_t* d = vox + b * (long long)wxyz;
            for (int k = threadIdx.x; k < wxyz; k += blockDim.x) d[k] = tmpl[k];
        }
    }
}

int mc_launch_regen(const mc_kp* p, int conditional, cudaStream_t s) {
    int wxyz = p->wx * p->wy * p->wz;
    if (conditional && p->regen_per_env) {
        const int grid = p->B < 1184 ? (p->B > 0 ? p->B : 1) : 1184;
        k_regen_masked<<<grid, 256, 0, s>>>(p->voxels, p->world_template, p->do_reset, p->B, wxyz, p->flags);
        return (int)cudaGetLastError();
    }
    int grid = p->B < 1184 ? (p->B > 0 ? p->B : 1) : 1184;  // 148 SMs x 8
    k_regen<<<grid, 256, 0, s>>>(p->voxels, p->world_template, p->B, wxyz, p->flags, conditional);
    return (int)cudaGetLastError();
}

// The conditional regeneration of several env groups in one launch (a
// ragged step, a server launch): each group whose any-done flag its step set
// gets its worlds back (every world under the all-world rule, the worlds of
// its done envs under the per-env rule), as mc_launch_regen would for that
// group alone; one launch instead of one per group.
namespace {
struct RegenGroups {
    int8_t* vox[MC_MAX_GROUPS];
    const int8_t* tmpl[MC_MAX_GROUPS];
    const uint8_t* do_reset[MC_MAX_GROUPS];
    int32_t* flags[MC_MAX_GROUPS];
    int B[MC_MAX_GROUPS];
    int wxyz[MC_MAX_GROUPS];
    int per_env[MC_MAX_GROUPS];
    int G;
    int32_t* ctr;  // finished CTAs of the launch (cleared by the last one)
};

__global__ void k_regen_groups(const __grid_constant__ RegenGroups rg) {
    __shared__ int go[MC_MAX_GROUPS];
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (threadIdx.x < rg.G) {
        go[threadIdx.x] = *(volatile int32_t*)&rg.flags[threadIdx.x][MC_FLAG_ANY_DONE] != 0;
        if (go[threadIdx.x]) atomicOr(&any, 1);
    }
    __syncthreads();
    // The flags were set before this launch and only its last CTA clears
    // them: every CTA reads the same values, so when none is set none of them
    // has anything to write, count or clear.
    if (!any) return;
    for (int g = 0; g < rg.G; ++g) {
        if (!go[g]) continue;
        const int wxyz = rg.wxyz[g];
        const bool vec = (wxyz & 15) == 0 && ((((uintptr_t)rg.vox[g]) | ((uintptr_t)rg.tmpl[g])) & 15) == 0;
        for (long long b = blockIdx.x; b < rg.B[g]; b += gridDim.x) {
            if (rg.per_env[g] && !rg.do_reset[g][b]) continue;  // the same for every thread of the CTA
            int8_t* d = rg.vox[g] + b * (long long)wxyz;
            if (vec) {
                uint4* d4 = reinterpret_cast<uint4*>(d);
                const uint4* t4 = reinterpret_cast<const uint4*>(rg.tmpl[g]);
                for (int k = threadIdx.x; k < (wxyz >> 4); k += blockDim.x) d4[k] = __ldg(t4 + k);
            } else {
                for (int k = threadIdx.x; k < wxyz; k += blockDim.x) d[k] = rg.tmpl[g][k];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(reinterpret_cast<unsigned*>(rg.ctr), 1u);
        if (prev == gridDim.x - 1) {
            for (int g = 0; g < rg.G; ++g)
                if (go[g]) rg.flags[g][MC_FLAG_ANY_DONE] = 0;
            *rg.ctr = 0;
            __threadfence();
        }
    }
}
}  // namespace

int mc_launch_regen_groups(const mc_kp* const* kps, int G, int32_t* ctr, cudaStream_t s) {
    RegenGroups rg{};
    for (int g = 0; g < G; ++g) {
        const mc_kp& k = *kps[g];
        if (k.B == 0 || !dones_possible(k)) continue;
        const int i = rg.G++;
        rg.vox[i] = k.voxels;
        rg.tmpl[i] = k.world_template;
        rg.do_reset[i] = k.do_reset;
        rg.flags[i] = k.flags;
        rg.B[i] = k.B;
        rg.wxyz[i] = k.wx * k.wy * k.wz;
        rg.per_env[i] = k.regen_per_env;
    }
    if (rg.G == 0) return 0;
    rg.ctr = ctr;
    k_regen_groups<<<1184, 256, 0, s>>>(rg);  // 148 SMs x 8
    return (int)cudaGetLastError();
}

namespace {
__global__ void k_flag_from_byte(int32_t* flags, const uint8_t* flag) {
    flags[MC_FLAG_ANY_DONE] = *flag ? 1 : 0;
}
}  // namespace

// Regeneration conditional on a device byte (copied into the any-done word,
// which the last CTA of k_regen clears).
int mc_launch_regen_if(const mc_kp* p, const uint8_t* flag, cudaStream_t s) {
    k_flag_from_byte<<<1, 1, 0, s>>>(p->flags, flag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return mc_launch_regen(p, 1, s);
}

// ---------------------------------------------------------------------------
// configuration
// ---------------------------------------------------------------------------
static int family_of(int obs_mode) {
    switch (obs_mode) {
        case MC_OBS_FLOAT32:
        case MC_OBS_UINT8: return MC_FAM_SHADED;
        case MC_OBS_UINT8_FAST: return MC_FAM_SHADED_FAST;
        case MC_OBS_UINT8_MINIMAL: return MC_FAM_MINIMAL;
        case MC_OBS_UINT8_FP16: return MC_FAM_FP16;
        case MC_OBS_UINT8_PREBASIS:
        case MC_OBS_UINT8_PREBASIS_FULL:
        case MC_OBS_UINT8_SMEM: return MC_FAM_PREBASIS;
        default: return -1;
    }
}

static const mc_backend* backend_of(int numerics) {
    if (numerics == MC_NUMERICS_REF_FAST) return mc_backend_fast();
    if (numerics == MC_NUMERICS_IEEE) return mc_backend_ieee();
    return nullptr;
}

static int check_config(const mc_env_config* c) {
    if (!c) return fail(MC_ERR_INVALID, "config is NULL");
    if (c->batch_size < 0) return fail(MC_ERR_INVALID, "batch_size %d < 0", c->batch_size);
    if (c->world_x < 1 || c->world_y < 1 || c->world_z < 1)
        return fail(MC_ERR_INVALID, "world dims must be >= 1 (got %d,%d,%d)", c->world_x, c->world_y, c->world_z);
    long long wxyz = (long long)c->world_x * c->world_y * c->world_z;
    if (wxyz > (1LL << 30)) return fail(MC_ERR_INVALID, "world too large (%lld voxels)", wxyz);
    if (c->render_width < 1 || c->render_height < 1 || (long long)c->render_width * c->render_height > (1 << 24))
        return fail(MC_ERR_INVALID, "render size %dx%d out of range", c->render_width, c->render_height);
    if (family_of(c->obs_mode) < 0) return fail(MC_ERR_INVALID, "unknown obs_mode %d", c->obs_mode);
    if (!backend_of(c->numerics)) return fail(MC_ERR_INVALID, "unknown numerics %d", c->numerics);
    if (c->target_block < -128 || c->target_block > 127)
        return fail(MC_ERR_INVALID, "target_block %d outside int8", c->target_block);
    return MC_OK;
}

// MineEnv's spawn, tree and house positions (minecu/__init__.py:195-206).
struct Placement {
    float sx, sy, sz;
    int tx, tz, hx, hz;
};
static Placement placement_of(const mc_env_config* c) {
    Placement p;
    p.sx = (float)(c->world_x / 2.0);
    p.sy = (float)(c->ground_height + 2);
    p.sz = (float)(c->world_z / 2.0);
    if (c->spawn_override) {
        p.sx = c->spawn_x;
        p.sy = c->spawn_y;
        p.sz = c->spawn_z;
    }
    p.tx = (int)(c->world_x / 2.0);
    p.tz = (int)(c->world_z / 2.0) + 2;
    p.hx = (int)(c->world_x / 2.0) + 6;
    p.hz = (int)(c->world_z / 2.0) - 2;
    return p;
}

static void fill_kp(mc_kp* k, const mc_env_config* c, const mc_env_state* s) {
    memset(k, 0, sizeof(*k));
    Placement pl = placement_of(c);
    k->B = c->batch_size;
    k->wx = c->world_x;
    k->wy = c->world_y;
    k->wz = c->world_z;
    k->W = c->render_width;
    k->H = c->render_height;
    k->max_steps = c->max_steps;
    k->vd = c->view_distance;
    k->fov = c->fov_degrees;
    k->dt = c->dt;
    k->gravity = c->gravity;
    k->walk_speed = c->walk_speed;
    k->sprint_mult = c->sprint_mult;
    k->jump_vel = c->jump_vel;
    k->gh = c->ground_height;
    k->target_block = c->target_block;
    k->reward_value = c->reward_value;
    k->spawn_x = pl.sx;
    k->spawn_y = pl.sy;
    k->spawn_z = pl.sz;
    k->episode_rule = (c->obs_mode == MC_OBS_UINT8_PREBASIS_FULL) ? 1 : 0;
    k->ext_done = 0;
    k->has_limit = c->has_episode_limit;
    k->episode_length = c->episode_length;
    k->family = family_of(c->obs_mode);
    k->obs_f32 = (c->obs_mode == MC_OBS_FLOAT32);
    k->look_delta = c->look_delta;
    if (s) {
        k->voxels = s->voxels;
        k->positions = s->positions;
        k->velocities = s->velocities;
        k->yaws = s->yaws;
        k->pitches = s->pitches;
        k->on_ground = s->on_ground;
        k->step_count = s->step_count;
        k->do_reset = s->do_reset;
        k->cameras = s->cameras;
        k->basis = s->basis;
        k->obs = s->obs;
        k->rewards = s->rewards;
        k->dbg_interact = s->dbg_interact;
        k->dbg_pixel = s->dbg_pixel;
    }
}

// need_count = false: the stateless steps of every mode but prebasis_full,
// whose episode counter is the caller's and is never read or written
static int check_state(const mc_env_config* c, const mc_env_state* s, bool need_count = true) {
    if (!s) return fail(MC_ERR_INVALID, "state is NULL");
    if (c->batch_size == 0) return MC_OK;
    const void* cnt = (need_count || s->step_count) ? (const void*)s->step_count : (const void*)s->voxels;
    const void* req[] = {s->voxels, s->positions, s->velocities, s->yaws, s->pitches, s->on_ground,
                         cnt, s->do_reset, s->cameras, s->obs, s->rewards};
    const char* names[] = {"voxels", "positions", "velocities", "yaws", "pitches", "on_ground",
                           "step_count", "do_reset", "cameras", "obs", "rewards"};
    for (int i = 0; i < 11; ++i)
        if (!req[i]) return fail(MC_ERR_INVALID, "state.%s is NULL", names[i]);
    if (((uintptr_t)s->positions | (uintptr_t)s->velocities | (uintptr_t)s->yaws | (uintptr_t)s->pitches |
         (uintptr_t)s->cameras | (uintptr_t)s->rewards | (uintptr_t)s->step_count) & 3)
        return fail(MC_ERR_INVALID, "float/int32 state buffers must be 4-byte aligned");
    if (family_of(c->obs_mode) == MC_FAM_PREBASIS && c->obs_mode != MC_OBS_UINT8_SMEM && !s->basis)
        return fail(MC_ERR_INVALID, "prebasis modes need state.basis [B,14]");
    return MC_OK;
}

// ---------------------------------------------------------------------------
// env handle
// ---------------------------------------------------------------------------
bool dones_possible(const mc_kp& k) {
    if (k.ext_done) return false;
    if (k.episode_rule == 0) return k.has_limit != 0;
    return k.episode_length > 0;
}

static inline int align16i(long long x) { return (int)((x + 15) & ~15LL); }

void team_layout(const mc_kp* const* kps, int G, const int* stage, const int* tile_w, const int* coop,
                        int team_warps, int warps_per_cta, mc_ragged_kp* rk) {
    *rk = mc_ragged_kp{};
    rk->ngroups = G;
    rk->team_warps = team_warps;
    rk->sched_dynamic = 1;
    const int bpp = 3 * (kps[0]->obs_f32 ? 4 : 1);
    long long start = 0;
    int uv = 0, band = 16, coop_world = 0, slot = 0, pad = 0, depth = 0;
    for (int g = 0; g < G; ++g) {
        const mc_kp& k = *kps[g];
        const long long wxyz = (long long)k.wx * k.wy * k.wz;
        rk->groups[g] = k;
        rk->start[g] = start;
        start += k.B;
        rk->uv_off[g] = uv;
        uv += k.W + k.H;
        rk->tile_w[g] = tile_w[g];
        band = std::max(band, align16i((long long)k.W * (32 / tile_w[g]) * bpp));
        if (coop[g]) rk->coop_mask |= 1 << g;
        if (stage[g]) {
            rk->stage_mask |= 1 << g;
            depth = std::max(depth, stage[g]);  // the launch stages every staged group at the largest depth asked
            pad = std::max(pad, align16i((long long)k.wx * k.wz));
            if (coop[g])
                coop_world = std::max(coop_world, align16i(wxyz));
            else
                slot = std::max(slot, align16i(wxyz));
        }
    }
    rk->start[G] = start;
    // visit the groups with the most expensive envs first (pixels x world extent)
    std::vector<int> order(G);
    for (int g = 0; g < G; ++g) order[g] = g;
    auto cost = [&](int g) {
        const mc_kp& k = *kps[g];
        return (double)k.W * k.H * (k.wx + k.wy + k.wz);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    rk->ustart[0] = 0;
    for (int v = 0; v < G; ++v) {
        const int g = order[v];
        rk->order[v] = g;
        const long long B = kps[g]->B;
        rk->ustart[v + 1] = rk->ustart[v] + (coop[g] ? B : (B + team_warps - 1) / team_warps);
    }
    rk->slot_bytes = slot;
    rk->tables_off = MC_COLOUR_TABLE_BYTES + MC_FAST_TABLE_BYTES;
    rk->teams_off = rk->tables_off + align16i((long long)uv * 4);
    // the march reads up to one world layer (wx*wz bytes) on either side of a
    // staged world: worlds that follow one another are farther apart than
    // that, so only the first needs bytes before it and the last bytes after
    if (rk->teams_off + MC_TEAM_HEAD_BYTES < pad) rk->teams_off += align16i(pad - rk->teams_off - MC_TEAM_HEAD_BYTES);
    rk->depth = depth;
    rk->world_stride = std::max(coop_world, team_warps * slot);
    rk->team_bytes = MC_TEAM_HEAD_BYTES + std::max(depth, 1) * rk->world_stride;
    rk->warps_off = rk->teams_off + (warps_per_cta / team_warps) * rk->team_bytes;
    // per warp: two mbarriers, a table of march start values, [depth 2: two env stashes], one band
    rk->warp_bytes = 16 + 128 + (depth == 2 ? 2 * MC_ENV_STASH_BYTES : 0) + band;
    const int after = warps_per_cta * rk->warp_bytes;
    rk->tail_bytes = after < pad ? pad - after : 0;
}

long long team_smem(const mc_ragged_kp& rk, int warps_per_cta) {
    return (long long)rk.warps_off + (long long)warps_per_cta * rk.warp_bytes + rk.tail_bytes;
}

int team_validate(const mc_kp* const* kps, int G, const int* stage, const int* tile_w, const int* coop,
                         int team_warps, int warps_per_cta, int ctas_per_sm) {
    if (warps_per_cta < 1 || warps_per_cta > 8) return fail(MC_ERR_INVALID, "warps_per_cta must be 1..8");
    if (team_warps != 1 && team_warps != 2 && team_warps != 4 && team_warps != 8)
        return fail(MC_ERR_INVALID, "team_warps must be 1, 2, 4 or 8");
    if (warps_per_cta % team_warps) return fail(MC_ERR_INVALID, "team_warps must divide warps_per_cta");
    if (ctas_per_sm < 1 || ctas_per_sm > 32) return fail(MC_ERR_INVALID, "ctas_per_sm out of range");
    for (int g = 0; g < G; ++g) {
        const int tw = tile_w[g];
        if (tw != 4 && tw != 8 && tw != 16 && tw != 32)
            return fail(MC_ERR_INVALID, "group %d: tile_w must be 4, 8, 16 or 32", g);
        if (stage[g] < 0 || stage[g] > 2 || (coop[g] != 0 && coop[g] != 1))
            return fail(MC_ERR_INVALID, "group %d: stage (staging depth) must be 0, 1 or 2 and coop 0 or 1", g);
        if (stage[g]) {
            const mc_kp& k = *kps[g];
            if (((long long)k.wx * k.wy * k.wz) & 15)
                return fail(MC_ERR_INVALID, "group %d: stage needs world bytes %% 16 == 0", g);
            if (((uintptr_t)k.voxels) & 15) return fail(MC_ERR_INVALID, "group %d: stage needs 16-byte aligned voxels", g);
        }
    }
    mc_ragged_kp rk;
    team_layout(kps, G, stage, tile_w, coop, team_warps, warps_per_cta, &rk);
    if (rk.ustart[G] >= (1LL << 31)) return fail(MC_ERR_INVALID, "more than 2^31 work units");
    const long long smem = team_smem(rk, warps_per_cta);
    if (smem > 227 * 1024) return fail(MC_ERR_INVALID, "team kernel shared memory %lld > 227 KB", smem);
    return MC_OK;
}

static bool team_mode(const mc_fused_cfg& f) { return f.team_warps > 1 || f.coop; }

static int validate_fused_kp(const mc_env_config* cfg, const mc_kp* kp, const mc_backend* be,
                             const mc_fused_cfg* f) {
    if (team_mode(*f)) {
        const mc_kp* kps[1] = {kp};
        return team_validate(kps, 1, &f->stage, &f->tile_w, &f->coop, f->team_warps, f->warps_per_cta,
                             f->ctas_per_sm);
    }
    if (f->team_warps != 1) return fail(MC_ERR_INVALID, "team_warps must be 1 without coop");
    if (f->stage < 0 || f->stage > 2)
        return fail(MC_ERR_INVALID, "stage (staging depth) must be 0, 1 or 2");
    if (f->warps_per_cta != 4 && f->warps_per_cta != 8)
        return fail(MC_ERR_INVALID, "warps_per_cta must be 4 or 8");
    if (f->tile_w != 4 && f->tile_w != 8 && f->tile_w != 16 && f->tile_w != 32)
        return fail(MC_ERR_INVALID, "tile_w must be 4, 8, 16 or 32");
    if (f->ctas_per_sm < 1 || f->ctas_per_sm > 32) return fail(MC_ERR_INVALID, "ctas_per_sm out of range");
    int wxyz = cfg->world_x * cfg->world_y * cfg->world_z;
    if (f->stage && (wxyz & 15)) return fail(MC_ERR_INVALID, "stage needs world bytes %% 16 == 0");
    mc_kp k = *kp;
    size_t smem = be->fused_smem_bytes(&k, f);
    if (smem > 227 * 1024) return fail(MC_ERR_INVALID, "fused shared memory %zu > 227 KB", smem);
    return MC_OK;
}

static int validate_fused(const mc_env* e, const mc_fused_cfg* f) {
    return validate_fused_kp(&e->cfg, &e->kp, e->be, f);
}

// The default launch shape of an env (a pure function of its configuration,
// the voxels' alignment and the SM count).  Small worlds: one warp per env,
// world staged in shared memory.  Big worlds, or big images over too few
// envs to give every resident warp (SMs x 32) two envs: teams of 4 warps
// render each env together from one staged copy of its world.  (16^3
// worlds, 64x64 images: teams take 0.166 ms/step at B=4096, where one warp
// per env takes 0.206; one warp per env takes 0.492 ms/step at B=16384,
// where teams take 0.587.)  A shape whose shared memory does not fit falls
// back to the team shape (whose per-warp image band is half as tall), then
// to one team per CTA, then to unstaged worlds.  The autotuner (minecu/autotune.py) refines the
// shape per configuration.
static mc_fused_cfg default_launch(const mc_env_config* cfg, const mc_kp* kp, const mc_backend* be, int num_sms) {
    const int wxyz = cfg->world_x * cfg->world_y * cfg->world_z;
    const bool aligned = (wxyz & 15) == 0 && !(((uintptr_t)kp->voxels) & 15);
    const bool few_envs = (long long)cfg->batch_size < 2LL * num_sms * 32;
    const bool big = (cfg->render_width * cfg->render_height >= 64 * 64 && few_envs) || wxyz > 8192;
    auto team_shape = [&](mc_fused_cfg& f) {
        f.warps_per_cta = 8;
        f.stage = (wxyz <= 32768 && aligned) ? 1 : 0;
        f.ctas_per_sm = 3;
        f.tile_w = 8;
        f.team_warps = 4;
        f.coop = 1;
    };
    mc_fused_cfg f;
    if (big) {
        team_shape(f);
    } else {
        f.warps_per_cta = 8;
        f.stage = (wxyz <= 8192 && aligned) ? 1 : 0;
        f.ctas_per_sm = 4;
        f.tile_w = 4;
        f.team_warps = 1;
        f.coop = 0;
    }
    const std::string saved = mc_last_error();  // probing shapes must not replace the caller's message
    if (!big && validate_fused_kp(cfg, kp, be, &f) != MC_OK) team_shape(f);  // e.g. wide float32 images
    if (validate_fused_kp(cfg, kp, be, &f) != MC_OK) f.warps_per_cta = 4;    // one team per CTA
    if (validate_fused_kp(cfg, kp, be, &f) != MC_OK) f.stage = 0;  // e.g. a world too big for a team's copy
    mc_set_error(MC_OK, saved.c_str());
    return f;
}

static void default_fused(mc_env* e) { e->fcfg = default_launch(&e->cfg, &e->kp, e->be, e->num_sms); }

extern "C" int mc_default_fused_config(const mc_env_config* cfg, int32_t num_sms, int32_t voxels_aligned,
                                       mc_fused_config* out, int64_t* smem_bytes) {
    if (!out) return fail(MC_ERR_INVALID, "out is NULL");
    int rc = check_config(cfg);
    if (rc) return rc;
    if (num_sms < 1) return fail(MC_ERR_INVALID, "num_sms must be >= 1");
    mc_kp k;
    fill_kp(&k, cfg, nullptr);
    k.voxels = voxels_aligned ? nullptr : reinterpret_cast<int8_t*>((uintptr_t)1);
    const mc_backend* be = backend_of(cfg->numerics);
    mc_fused_cfg f = default_launch(cfg, &k, be, num_sms);
    rc = validate_fused_kp(cfg, &k, be, &f);
    if (rc) return rc;
    *out = mc_fused_config{f.stage, f.warps_per_cta, f.ctas_per_sm, f.tile_w, f.team_warps, f.coop};
    if (smem_bytes) {
        if (team_mode(f)) {
            const mc_kp* kps[1] = {&k};
            mc_ragged_kp rk;
            team_layout(kps, 1, &f.stage, &f.tile_w, &f.coop, f.team_warps, f.warps_per_cta, &rk);
            *smem_bytes = team_smem(rk, f.warps_per_cta);
        } else {
            *smem_bytes = (int64_t)be->fused_smem_bytes(&k, &f);
        }
    }
    return MC_OK;
}

static void drop_graphs(mc_env* e) {
    for (auto& g : e->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
}

extern "C" int mc_env_create(const mc_env_config* cfg, const mc_env_state* state, mc_env** out) {
    if (!out) return fail(MC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = check_config(cfg);
    if (rc) return rc;
    rc = check_state(cfg, state);
    if (rc) return rc;
    Placement pl = placement_of(cfg);
    if (pl.tx < 0 || pl.tx >= cfg->world_x || pl.tz < 0 || pl.tz >= cfg->world_z)
        return fail(MC_ERR_INVALID,
                    "tree at (%d,%d) outside the %dx%d world (world_z must be >= 5); the reference writes out of "
                    "bounds here",
                    pl.tx, pl.tz, cfg->world_x, cfg->world_z);
    mc_env* e = new mc_env();
    e->cfg = *cfg;
    e->st = *state;
    e->be = backend_of(cfg->numerics);
    fill_kp(&e->kp, cfg, state);
    cudaError_t ce = cudaGetDevice(&e->device);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device);
    long long wxyz = (long long)cfg->world_x * cfg->world_y * cfg->world_z;
    if (ce == cudaSuccess) ce = cudaMalloc(&e->flags, MC_FLAG_WORDS * sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaMemset(e->flags, 0, MC_FLAG_WORDS * sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaMalloc(&e->tmpl, (size_t)((wxyz + 15) & ~15LL));
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) {
        // the template world: generate + tree + house on one env
        k_generate_world<<<blocks((long long)cfg->world_y * cfg->world_x, 128), 128, 0, e->cap_stream>>>(
            e->tmpl, (long long)cfg->world_y * cfg->world_x, cfg->world_x, cfg->world_y, cfg->world_z,
            cfg->ground_height);
        k_place_tree<<<1, 32, 0, e->cap_stream>>>(e->tmpl, 1, cfg->world_x, cfg->world_y, cfg->world_z, pl.tx, pl.tz,
                                                   cfg->ground_height);
        k_place_house<<<1, 32, 0, e->cap_stream>>>(e->tmpl, 1, cfg->world_x, cfg->world_y, cfg->world_z, pl.hx,
                                                    pl.hz, cfg->ground_height);
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->cap_stream);
    }
    if (ce != cudaSuccess) {
        int r = cuda_fail(ce, "mc_env_create");
        mc_env_destroy(e);
        return r;
    }
    e->kp.flags = e->flags;
    e->kp.world_template = e->tmpl;
    e->kp.sched_dynamic = 1;  // the handle's flag block is used by one launch at a time
    default_fused(e);
    *out = e;
    return MC_OK;
}

static void hostio_free(HostIO** ph) {
    HostIO* h = *ph;
    if (!h) return;
    for (int i = 0; i < 2; ++i) {
        if (h->d_act[i]) cudaFree(h->d_act[i]);
        if (h->d_res[i]) cudaFree(h->d_res[i]);
        for (cudaEvent_t ev : {h->act_ready[i], h->act_free[i], h->res_ready[i], h->res_free[i]})
            if (ev) cudaEventDestroy(ev);
    }
    if (h->up) cudaStreamDestroy(h->up);
    if (h->down) cudaStreamDestroy(h->down);
    delete h;
    *ph = nullptr;
}

// Wait for the copies in flight into or out of the caller's host buffers, then free.
static void hostio_close(HostIO** ph) {
    if (!*ph) return;
    if ((*ph)->up) cudaStreamSynchronize((*ph)->up);
    if ((*ph)->down) cudaStreamSynchronize((*ph)->down);
    hostio_free(ph);
}

extern "C" int mc_env_destroy(mc_env* e) {
    if (!e) return MC_OK;
    hostio_close(&e->hio);
    drop_graphs(e);
    if (e->flags) cudaFree(e->flags);
    if (e->tmpl) cudaFree(e->tmpl);
    if (e->scratch) cudaFree(e->scratch);
    if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
    delete e;
    return MC_OK;
}

extern "C" int mc_env_set_state(mc_env* e, const mc_env_state* s) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    int rc = check_state(&e->cfg, s);
    if (rc) return rc;
    e->st = *s;
    int32_t* flags = e->kp.flags;
    const int8_t* tmpl = e->kp.world_template;
    const int polls = e->kp.wait_polls;
    fill_kp(&e->kp, &e->cfg, s);
    e->kp.flags = flags;
    e->kp.world_template = tmpl;
    e->kp.wait_polls = polls;
    e->kp.regen_per_env = e->regen_mode == MC_REGEN_PER_ENV;
    e->kp.sched_dynamic = 1;
    drop_graphs(e);
    return MC_OK;
}

static int ensure_scratch(mc_env* e) {
    if (e->scratch || e->cfg.batch_size == 0) return MC_OK;
    size_t B = (size_t)e->cfg.batch_size;
    MC_CK(cudaMalloc(&e->scratch, B * (5 * 4 + 3) + 64));
    uint8_t* p = e->scratch;
    e->kp.s_fwd = (float*)p; p += B * 4;
    e->kp.s_strafe = (float*)p; p += B * 4;
    e->kp.s_dyaw = (float*)p; p += B * 4;
    e->kp.s_dpitch = (float*)p; p += B * 4;
    e->kp.s_speed = (float*)p; p += B * 4;
    e->kp.s_jump = p; p += B;
    e->kp.s_brk = p; p += B;
    e->kp.s_place = p;
    return MC_OK;
}

extern "C" int mc_env_generate_world(mc_env* e, void* stream) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (e->cfg.batch_size == 0) return MC_OK;
    return backend_rc(mc_launch_regen(&e->kp, 0, (cudaStream_t)stream), "regen");
}

static int render_obs(mc_env* e, cudaStream_t s) {
    mc_kp k = e->kp;
    if (k.B == 0) return MC_OK;
    k_cameras_rt<<<blocks(k.B, 256), 256, 0, s>>>(k);
    MC_CK(cudaGetLastError());
    // MineEnv._render always uses the shaded kernel: float32 for "float32",
    // render_uint8 for every uint8 mode (minecu/__init__.py:455-464).
    return backend_rc(e->be->render(&k, MC_FAM_SHADED, s), "render");
}

extern "C" int mc_env_reset(mc_env* e, const uint8_t* mask, void* stream) {
    NvtxRange nvtx("mc_env_reset");
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    if (e->cfg.batch_size == 0) return MC_OK;
    int rc = backend_rc(mc_launch_reset_agents(&e->kp, mask, s), "reset");
    if (rc) return rc;
    rc = backend_rc(mc_launch_regen(&e->kp, 1, s), "regen");
    if (rc) return rc;
    return render_obs(e, s);
}

// res_rewards / res_dones: where the per-warp fused kernel also writes every
// env's reward and done (the host-buffer step's read-back buffer); the other
// launch forms ignore them.
static int do_step(mc_env* e, const int8_t* buttons, const float* look, const uint8_t* actions, int form,
                   cudaStream_t s, float* res_rewards = nullptr, uint8_t* res_dones = nullptr) {
    if (e->cfg.batch_size == 0) return MC_OK;
    mc_kp k = e->kp;
    k.buttons = buttons;
    k.look = look;
    k.actions = actions;
    int rc;
    if (form == MC_FORM_PLAIN) {
        rc = ensure_scratch(e);
        if (rc) return rc;
        k = e->kp;
        k.buttons = buttons;
        k.look = look;
        k.actions = actions;
        rc = backend_rc(e->be->step_plain(&k, s), "step_plain");
    } else if (form == MC_FORM_FUSED && team_mode(e->fcfg)) {
        const mc_fused_cfg& f = e->fcfg;
        const mc_kp* kps[1] = {&e->kp};
        mc_ragged_kp rk;
        team_layout(kps, 1, &f.stage, &f.tile_w, &f.coop, f.team_warps, f.warps_per_cta, &rk);
        rk.flags = e->flags;
        rk.actions = actions;
        rk.buttons = buttons;
        rk.look = look;
        rc = backend_rc(e->be->step_team(&rk, k.family, k.obs_f32, f.warps_per_cta, f.ctas_per_sm, e->num_sms, s),
                        "step_team");
    } else if (form == MC_FORM_FUSED) {
        k.res_rewards = res_rewards;
        k.res_dones = res_dones;
        rc = backend_rc(e->be->step_fused(&k, &e->fcfg, e->num_sms, s), "step_fused");
    } else {
        return fail(MC_ERR_INVALID, "unknown form %d", form);
    }
    if (rc) return rc;
    if (dones_possible(k)) return backend_rc(mc_launch_regen(&k, 1, s), "regen");
    return MC_OK;
}

extern "C" int mc_env_step(mc_env* e, const int8_t* buttons, const float* look, int form, void* stream) {
    NvtxRange nvtx("mc_env_step");
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (e->cfg.batch_size && (!buttons || !look)) return fail(MC_ERR_INVALID, "buttons/look are NULL");
    if (((uintptr_t)look) & 3) return fail(MC_ERR_INVALID, "look must be 4-byte aligned");
    return do_step(e, buttons, look, nullptr, form, (cudaStream_t)stream);
}

extern "C" int mc_env_step_discrete(mc_env* e, const uint8_t* actions, int form, void* stream) {
    NvtxRange nvtx("mc_env_step_discrete");
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (e->cfg.batch_size && !actions) return fail(MC_ERR_INVALID, "actions is NULL");
    return do_step(e, nullptr, nullptr, actions, form, (cudaStream_t)stream);
}

namespace {
// rewards (float[B]) and dones (byte[B]) of the step just run, copied into
// one block so that one buffer pair per step goes back to the host
__global__ void k_results_snapshot(const float* rewards, const uint8_t* dones, long long B, uint8_t* out) {
    float* r = reinterpret_cast<float*>(out);
    uint8_t* d = out + 4 * B;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < B; i += (long long)gridDim.x * blockDim.x) {
        r[i] = rewards[i];
        d[i] = dones[i];
    }
}
}  // namespace

static int hostio_init(HostIO** ph, long long batch) {
    if (*ph) return MC_OK;
    HostIO* h = new HostIO();
    *ph = h;
    const size_t B = (size_t)batch;
    cudaError_t ce = cudaStreamCreateWithFlags(&h->up, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&h->down, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && ce == cudaSuccess; ++i) {
        ce = cudaMalloc(&h->d_act[i], B + 16);
        if (ce == cudaSuccess) ce = cudaMalloc(&h->d_res[i], 5 * B + 16);
        for (cudaEvent_t* ev : {&h->act_ready[i], &h->act_free[i], &h->res_ready[i], &h->res_free[i]})
            if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    if (ce != cudaSuccess) {
        int rc = cuda_fail(ce, "host-buffer step: set-up");
        hostio_free(ph);
        return rc;
    }
    return MC_OK;
}

// Upload of call k's actions into action buffer i (= k mod 2) once the step
// two calls back is done reading it; stream s waits for the upload.
static int hostio_upload(HostIO* h, int i, const uint8_t* host_actions, long long B, cudaStream_t s) {
    MC_CK(cudaStreamWaitEvent(h->up, h->act_free[i], 0));
    MC_CK(cudaMemcpyAsync(h->d_act[i], host_actions, (size_t)B, cudaMemcpyHostToDevice, h->up));
    MC_CK(cudaEventRecord(h->act_ready[i], h->up));
    MC_CK(cudaStreamWaitEvent(s, h->act_ready[i], 0));
    return MC_OK;
}

// Read-back of result buffer i (rewards then dones, written on stream s)
// while the next step runs; ends the call.
static int hostio_readback(HostIO* h, int i, float* host_rewards, uint8_t* host_dones, long long B, cudaStream_t s) {
    MC_CK(cudaEventRecord(h->res_ready[i], s));
    MC_CK(cudaStreamWaitEvent(h->down, h->res_ready[i], 0));
    MC_CK(cudaMemcpyAsync(host_rewards, h->d_res[i], (size_t)B * 4, cudaMemcpyDeviceToHost, h->down));
    MC_CK(cudaMemcpyAsync(host_dones, h->d_res[i] + 4 * B, (size_t)B, cudaMemcpyDeviceToHost, h->down));
    MC_CK(cudaEventRecord(h->res_free[i], h->down));
    h->calls++;
    return MC_OK;
}

static int hostio_join(const HostIO* h, cudaStream_t s) {
    if (!h || h->calls == 0) return MC_OK;
    // the read-back stream runs in call order: its last event covers every copy
    MC_CK(cudaStreamWaitEvent(s, h->res_free[(h->calls - 1) & 1], 0));
    return MC_OK;
}

extern "C" int mc_env_step_host(mc_env* e, const uint8_t* host_actions, float* host_rewards, uint8_t* host_dones,
                                int form, void* stream) {
    NvtxRange nvtx("mc_env_step_host");
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    const long long B = e->cfg.batch_size;
    if (B == 0) return MC_OK;
    if (!host_actions || !host_rewards || !host_dones) return fail(MC_ERR_INVALID, "host buffers are NULL");
    if (form != MC_FORM_PLAIN && form != MC_FORM_FUSED) return fail(MC_ERR_INVALID, "unknown form %d", form);
    int rc = hostio_init(&e->hio, B);
    if (rc) return rc;
    HostIO* h = e->hio;
    cudaStream_t s = (cudaStream_t)stream;
    const int i = (int)(h->calls & 1);
    rc = hostio_upload(h, i, host_actions, B, s);
    if (rc) return rc;
    // results go into this call's buffer once the read-back two calls back
    // is done with it; the per-warp fused kernel writes them there itself,
    // the other forms through a copy kernel after the step
    MC_CK(cudaStreamWaitEvent(s, h->res_free[i], 0));
    const bool direct = form == MC_FORM_FUSED && !team_mode(e->fcfg);
    float* res_rew = reinterpret_cast<float*>(h->d_res[i]);
    uint8_t* res_done = h->d_res[i] + 4 * B;
    rc = do_step(e, nullptr, nullptr, h->d_act[i], form, s, direct ? res_rew : nullptr, direct ? res_done : nullptr);
    if (rc) return rc;
    MC_CK(cudaEventRecord(h->act_free[i], s));
    if (!direct) {
        const int grid = (int)std::min<long long>((B + 255) / 256, (long long)e->num_sms * 4);
        k_results_snapshot<<<grid, 256, 0, s>>>(e->st.rewards, e->st.do_reset, B, h->d_res[i]);
        MC_CK(cudaGetLastError());
    }
    return hostio_readback(h, i, host_rewards, host_dones, B, s);
}

extern "C" int mc_env_host_join(mc_env* e, void* stream) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    return hostio_join(e->hio, (cudaStream_t)stream);
}

extern "C" int mc_env_set_regen_mode(mc_env* e, int32_t mode) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (mode != MC_REGEN_ALL && mode != MC_REGEN_PER_ENV) return fail(MC_ERR_INVALID, "unknown regen mode %d", mode);
    e->regen_mode = mode;
    e->kp.regen_per_env = mode == MC_REGEN_PER_ENV;
    drop_graphs(e);  // captured steps hold the old rule
    return MC_OK;
}

extern "C" int mc_env_set_wait_limit(mc_env* e, int32_t polls) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    e->kp.wait_polls = polls < 0 ? 0 : (polls == 0 ? -1 : polls);
    drop_graphs(e);  // captured steps hold the old budget
    return MC_OK;
}

extern "C" int mc_env_get_regen_mode(const mc_env* e) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    return e->regen_mode;
}

extern "C" int mc_env_regenerate_if(mc_env* e, const uint8_t* flag, void* stream) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (!flag) return fail(MC_ERR_INVALID, "flag is NULL");
    if (e->cfg.batch_size == 0) return MC_OK;
    return backend_rc(mc_launch_regen_if(&e->kp, flag, (cudaStream_t)stream), "regen");
}

extern "C" int mc_env_render(mc_env* e, void* stream) {
    NvtxRange nvtx("mc_env_render");
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    return render_obs(e, (cudaStream_t)stream);
}

static bool same_fcfg(const mc_fused_cfg& a, const mc_fused_cfg& b) {
    return a.stage == b.stage && a.warps_per_cta == b.warps_per_cta && a.ctas_per_sm == b.ctas_per_sm &&
           a.tile_w == b.tile_w && a.team_warps == b.team_warps && a.coop == b.coop;
}

static int rollout_graph(mc_env* e, const uint8_t* actions, int32_t K, float* rewards_out, uint8_t* dones_out,
                         RolloutGraph** out) {
    *out = nullptr;
    RolloutGraph* hit = nullptr;
    for (auto& g : e->graphs)
        if (g.actions == actions && g.K == K && g.rewards_out == rewards_out && g.dones_out == dones_out &&
            same_fcfg(g.fcfg, e->fcfg))
            hit = &g;
    if (!hit) {
        // capture K fused steps (+ conditional regeneration and output copies)
        long long B = e->cfg.batch_size;
        cudaGraph_t graph = nullptr;
        MC_CK(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
        int rc = MC_OK;
        for (int k = 0; k < K && rc == MC_OK; ++k) {
            rc = do_step(e, nullptr, nullptr, actions + (long long)k * B, MC_FORM_FUSED, e->cap_stream);
            if (rc == MC_OK && rewards_out) {
                cudaError_t ce = cudaMemcpyAsync(rewards_out + (long long)k * B, e->kp.rewards, B * sizeof(float),
                                                 cudaMemcpyDeviceToDevice, e->cap_stream);
                if (ce) rc = cuda_fail(ce, "rollout copy");
            }
            if (rc == MC_OK && dones_out) {
                cudaError_t ce = cudaMemcpyAsync(dones_out + (long long)k * B, e->kp.do_reset, B,
                                                 cudaMemcpyDeviceToDevice, e->cap_stream);
                if (ce) rc = cuda_fail(ce, "rollout copy");
            }
        }
        cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        RolloutGraph g;
        ce = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
        g.actions = actions;
        g.K = K;
        g.rewards_out = rewards_out;
        g.dones_out = dones_out;
        g.fcfg = e->fcfg;
        if (e->graphs.size() >= 8) {
            cudaGraphExecDestroy(e->graphs.front().exec);
            e->graphs.erase(e->graphs.begin());
        }
        e->graphs.push_back(g);
        hit = &e->graphs.back();
    }
    *out = hit;
    return MC_OK;
}

static int rollout_args(mc_env* e, const uint8_t* actions, int32_t K) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    if (K < 0) return fail(MC_ERR_INVALID, "K < 0");
    if (K > 0 && e->cfg.batch_size > 0 && !actions) return fail(MC_ERR_INVALID, "actions is NULL");
    return MC_OK;
}

extern "C" int mc_env_rollout_prepare(mc_env* e, const uint8_t* actions, int32_t K, float* rewards_out,
                                      uint8_t* dones_out) {
    int rc = rollout_args(e, actions, K);
    if (rc || K == 0 || e->cfg.batch_size == 0) return rc;
    RolloutGraph* g;
    return rollout_graph(e, actions, K, rewards_out, dones_out, &g);
}

extern "C" int mc_env_rollout(mc_env* e, const uint8_t* actions, int32_t K, float* rewards_out, uint8_t* dones_out,
                              void* stream) {
    NvtxRange nvtx("mc_env_rollout");
    int rc = rollout_args(e, actions, K);
    if (rc || K == 0 || e->cfg.batch_size == 0) return rc;
    RolloutGraph* g;
    rc = rollout_graph(e, actions, K, rewards_out, dones_out, &g);
    if (rc) return rc;
    MC_CK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return MC_OK;
}

extern "C" int mc_env_set_fused_config(mc_env* e, const mc_fused_config* c) {
    if (!e || !c) return fail(MC_ERR_INVALID, "NULL argument");
    mc_fused_cfg f{c->stage, c->warps_per_cta, c->ctas_per_sm, c->tile_w, c->team_warps, c->coop};
    int rc = validate_fused(e, &f);
    if (rc) return rc;
    e->fcfg = f;
    return MC_OK;
}

extern "C" int mc_env_get_fused_config(const mc_env* e, mc_fused_config* c) {
    if (!e || !c) return fail(MC_ERR_INVALID, "NULL argument");
    c->stage = e->fcfg.stage;
    c->warps_per_cta = e->fcfg.warps_per_cta;
    c->ctas_per_sm = e->fcfg.ctas_per_sm;
    c->tile_w = e->fcfg.tile_w;
    c->team_warps = e->fcfg.team_warps;
    c->coop = e->fcfg.coop;
    return MC_OK;
}

extern "C" int64_t mc_env_fused_smem_bytes(const mc_env* e) {
    if (!e) return -1;
    if (team_mode(e->fcfg)) {
        const mc_fused_cfg& f = e->fcfg;
        const mc_kp* kps[1] = {&e->kp};
        mc_ragged_kp rk;
        team_layout(kps, 1, &f.stage, &f.tile_w, &f.coop, f.team_warps, f.warps_per_cta, &rk);
        return team_smem(rk, f.warps_per_cta);
    }
    mc_kp k = e->kp;
    return (int64_t)e->be->fused_smem_bytes(&k, &e->fcfg);
}

extern "C" int mc_debug_bounds_report(int32_t numerics, int32_t* out, void* stream) {
    if (!out) return fail(MC_ERR_INVALID, "out is NULL");
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics %d", numerics);
    const int rc = be->bounds_report(out, (cudaStream_t)stream);
    if (rc < 0) return fail(MC_ERR_UNSUPPORTED, "not the bounds-checked build (libminecu_b200_checked.so)");
    return backend_rc(rc, "bounds report");
}

extern "C" int mc_debug_bounds_selftest(int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics %d", numerics);
    const int rc = be->bounds_selftest((cudaStream_t)stream);
    if (rc < 0) return fail(MC_ERR_UNSUPPORTED, "not the bounds-checked build (libminecu_b200_checked.so)");
    return backend_rc(rc, "bounds self-test");
}

extern "C" int mc_build_checks_bounds(void) { return MC_CHECK_BOUNDS_BUILD; }

extern "C" int mc_env_check_error(mc_env* e, void* stream) {
    if (!e) return fail(MC_ERR_INVALID, "env is NULL");
    int32_t h[MC_FLAG_WORDS];
    cudaStream_t s = (cudaStream_t)stream;
    MC_CK(cudaMemcpyAsync(h, e->flags, sizeof(h), cudaMemcpyDeviceToHost, s));
    MC_CK(cudaStreamSynchronize(s));
    if (h[MC_FLAG_ERROR] != MC_KERR_NONE) {
        int code = h[MC_FLAG_ERROR];
        int32_t zero = 0;
        MC_CK(cudaMemcpyAsync(e->flags + MC_FLAG_ERROR, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
        MC_CK(cudaStreamSynchronize(s));
        return fail(MC_ERR_KERNEL, "kernel error %d (%s)", code,
                    code == MC_KERR_TMA_TIMEOUT ? "bulk copy wait timed out"
                                                : (code == MC_KERR_BOUNDS ? "index out of bounds (debug build)"
                                                                          : "unknown"));
    }
    return MC_OK;
}

// ---------------------------------------------------------------------------
// ragged handle: several env handles stepped by one launch
// ---------------------------------------------------------------------------
struct RaggedGraph {
    cudaGraphExec_t exec = nullptr;
    const uint8_t* actions = nullptr;
    int K = 0;
    long long version = 0;  // config/kp version it was captured with
};

static_assert(MC_RAGGED_MAX_GROUPS == MC_MAX_GROUPS, "group limit");

struct mc_ragged {
    std::vector<mc_env*> envs;  // borrowed
    const mc_backend* be = nullptr;
    int family = 0, obs_f32 = 0;
    int device = 0, num_sms = 0;
    mc_ragged_config cfg{};
    std::vector<mc_kp> uploaded;  // group parameter blocks the cached graphs were captured with
    int32_t* flags = nullptr;     // the launch's work counter
    mc_ragged_kp rk{};
    long long version = 1;
    cudaStream_t cap_stream = nullptr;
    std::vector<RaggedGraph> graphs;
    HostIO* hio = nullptr;  // mc_ragged_step_host buffers
};

static long long ragged_wxyz(const mc_env* e) {
    return (long long)e->cfg.world_x * e->cfg.world_y * e->cfg.world_z;
}

static void ragged_kps(const mc_ragged* r, std::vector<const mc_kp*>* kps) {
    kps->clear();
    for (auto* e : r->envs) kps->push_back(&e->kp);
}

static void ragged_layout(const mc_ragged* r, const mc_ragged_config* c, mc_ragged_kp* rk) {
    std::vector<const mc_kp*> kps;
    ragged_kps(r, &kps);
    team_layout(kps.data(), (int)kps.size(), c->stage, c->tile_w, c->coop, c->team_warps, c->warps_per_cta, rk);
    rk->flags = r->flags;
}

static int ragged_validate(const mc_ragged* r, const mc_ragged_config* c) {
    std::vector<const mc_kp*> kps;
    ragged_kps(r, &kps);
    return team_validate(kps.data(), (int)kps.size(), c->stage, c->tile_w, c->coop, c->team_warps, c->warps_per_cta,
                         c->ctas_per_sm);
}

static void ragged_default_config(mc_ragged* r) {
    // teams of 8 warps; groups with big images or big worlds render each env
    // as a team, small ones one env per warp; small worlds are staged
    r->cfg = mc_ragged_config{};
    r->cfg.warps_per_cta = 8;
    r->cfg.ctas_per_sm = 4;
    r->cfg.team_warps = 4;
    for (size_t g = 0; g < r->envs.size(); ++g) {
        const mc_env* e = r->envs[g];
        const long long wxyz = ragged_wxyz(e);
        const bool big = (long long)e->cfg.render_width * e->cfg.render_height >= 64 * 64 || wxyz > 8192;
        r->cfg.coop[g] = big ? 1 : 0;
        r->cfg.stage[g] = (wxyz <= (big ? 32768 : 4096) && (wxyz & 15) == 0 && !(((uintptr_t)e->kp.voxels) & 15));
        r->cfg.tile_w[g] = big ? 8 : 4;
    }
}

static void ragged_drop_graphs(mc_ragged* r) {
    for (auto& g : r->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    r->graphs.clear();
}

// The launch copies the groups' parameter blocks by value; when one of them
// changed (an env handle was re-pointed), cached graphs hold stale copies.
static int ragged_sync_groups(mc_ragged* r, bool capturing) {
    bool same = r->uploaded.size() == r->envs.size();
    for (size_t g = 0; same && g < r->envs.size(); ++g)
        same = memcmp(&r->uploaded[g], &r->envs[g]->kp, sizeof(mc_kp)) == 0;
    if (same) return MC_OK;
    if (capturing) return fail(MC_ERR_INVALID, "a group was re-pointed; step once outside capture first");
    r->uploaded.clear();
    for (auto* e : r->envs) r->uploaded.push_back(e->kp);
    ++r->version;
    ragged_drop_graphs(r);
    return MC_OK;
}

extern "C" int mc_ragged_create(mc_env* const* groups, int32_t ngroups, mc_ragged** out) {
    if (!out) return fail(MC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!groups || ngroups < 1 || ngroups > MC_RAGGED_MAX_GROUPS)
        return fail(MC_ERR_INVALID, "ngroups must be 1..%d", MC_RAGGED_MAX_GROUPS);
    long long total = 0;
    for (int g = 0; g < ngroups; ++g) {
        const mc_env* e = groups[g];
        if (!e) return fail(MC_ERR_INVALID, "group %d is NULL", g);
        for (int h = 0; h < g; ++h)
            if (groups[h] == e) return fail(MC_ERR_INVALID, "group %d repeats group %d", g, h);
        if (e->device != groups[0]->device) return fail(MC_ERR_INVALID, "group %d is on another device", g);
        if (e->cfg.numerics != groups[0]->cfg.numerics) return fail(MC_ERR_INVALID, "group %d: other numerics", g);
        if (e->kp.family != groups[0]->kp.family || e->kp.obs_f32 != groups[0]->kp.obs_f32)
            return fail(MC_ERR_INVALID, "group %d: another observation kind (obs_mode)", g);
        total += e->cfg.batch_size;
    }
    if (total > (1LL << 30)) return fail(MC_ERR_INVALID, "more than 2^30 envs in one ragged handle");
    int dev = -1;
    MC_CK(cudaGetDevice(&dev));
    if (dev != groups[0]->device) return fail(MC_ERR_INVALID, "the groups live on device %d, current is %d",
                                              groups[0]->device, dev);
    mc_ragged* r = new mc_ragged();
    r->envs.assign(groups, groups + ngroups);
    r->be = groups[0]->be;
    r->family = groups[0]->kp.family;
    r->obs_f32 = groups[0]->kp.obs_f32;
    r->device = dev;
    r->num_sms = groups[0]->num_sms;
    cudaError_t ce = cudaMalloc(&r->flags, MC_FLAG_WORDS * sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaMemset(r->flags, 0, MC_FLAG_WORDS * sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&r->cap_stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        int rc = cuda_fail(ce, "mc_ragged_create");
        mc_ragged_destroy(r);
        return rc;
    }
    ragged_default_config(r);
    if (ragged_validate(r, &r->cfg) != MC_OK) {  // e.g. unaligned voxels: no staging
        for (int g = 0; g < ngroups; ++g) r->cfg.stage[g] = 0;
    }
    ragged_sync_groups(r, false);
    *out = r;
    return MC_OK;
}

extern "C" int mc_ragged_destroy(mc_ragged* r) {
    if (!r) return MC_OK;
    hostio_close(&r->hio);
    ragged_drop_graphs(r);
    if (r->flags) cudaFree(r->flags);
    if (r->cap_stream) cudaStreamDestroy(r->cap_stream);
    delete r;
    return MC_OK;
}

extern "C" int mc_ragged_set_config(mc_ragged* r, const mc_ragged_config* c) {
    if (!r || !c) return fail(MC_ERR_INVALID, "NULL argument");
    int rc = ragged_validate(r, c);
    if (rc) return rc;
    r->cfg = *c;
    for (size_t g = r->envs.size(); g < MC_RAGGED_MAX_GROUPS; ++g) r->cfg.stage[g] = r->cfg.tile_w[g] = r->cfg.coop[g] = 0;
    ++r->version;
    return MC_OK;
}

extern "C" int mc_ragged_get_config(const mc_ragged* r, mc_ragged_config* c) {
    if (!r || !c) return fail(MC_ERR_INVALID, "NULL argument");
    *c = r->cfg;
    return MC_OK;
}

extern "C" int64_t mc_ragged_total_envs(const mc_ragged* r) {
    if (!r) return -1;
    long long t = 0;
    for (auto* e : r->envs) t += e->cfg.batch_size;
    return t;
}

extern "C" int64_t mc_ragged_smem_bytes(const mc_ragged* r) {
    if (!r) return -1;
    mc_ragged_kp rk;
    ragged_layout(r, &r->cfg, &rk);
    return team_smem(rk, r->cfg.warps_per_cta);
}

static int ragged_do_step(mc_ragged* r, const int8_t* buttons, const float* look, const uint8_t* actions,
                          cudaStream_t s, bool capturing, float* rewards_cat = nullptr,
                          uint8_t* dones_cat = nullptr) {
    int rc = ragged_sync_groups(r, capturing);
    if (rc) return rc;
    mc_ragged_kp rk;
    ragged_layout(r, &r->cfg, &rk);
    rk.rewards_cat = rewards_cat;  // every env's reward and done also at its index in the batch
    rk.dones_cat = dones_cat;
    rk.actions = actions;
    rk.buttons = buttons;
    rk.look = look;
    rc = backend_rc(r->be->step_team(&rk, r->family, r->obs_f32, r->cfg.warps_per_cta, r->cfg.ctas_per_sm,
                                     r->num_sms, s),
                    "step_team");
    if (rc) return rc;
    std::vector<const mc_kp*> kps;
    for (auto* e : r->envs) kps.push_back(&e->kp);
    return backend_rc(mc_launch_regen_groups(kps.data(), (int)kps.size(), r->flags + MC_FLAG_REGEN_CTR, s),
                      "regen");
}

extern "C" int mc_ragged_step(mc_ragged* r, const int8_t* buttons, const float* look, void* stream) {
    NvtxRange nvtx("mc_ragged_step");
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    if (mc_ragged_total_envs(r) > 0 && (!buttons || !look)) return fail(MC_ERR_INVALID, "buttons/look are NULL");
    if (((uintptr_t)look) & 3) return fail(MC_ERR_INVALID, "look must be 4-byte aligned");
    return ragged_do_step(r, buttons, look, nullptr, (cudaStream_t)stream, false);
}

extern "C" int mc_ragged_step_discrete(mc_ragged* r, const uint8_t* actions, void* stream) {
    NvtxRange nvtx("mc_ragged_step_discrete");
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    if (mc_ragged_total_envs(r) > 0 && !actions) return fail(MC_ERR_INVALID, "actions is NULL");
    return ragged_do_step(r, nullptr, nullptr, actions, (cudaStream_t)stream, false);
}

extern "C" int mc_ragged_step_host(mc_ragged* r, const uint8_t* host_actions, float* host_rewards,
                                   uint8_t* host_dones, void* stream) {
    NvtxRange nvtx("mc_ragged_step_host");
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    const long long B = mc_ragged_total_envs(r);
    if (B == 0) return MC_OK;
    if (!host_actions || !host_rewards || !host_dones) return fail(MC_ERR_INVALID, "host buffers are NULL");
    int rc = hostio_init(&r->hio, B);
    if (rc) return rc;
    HostIO* h = r->hio;
    cudaStream_t s = (cudaStream_t)stream;
    const int i = (int)(h->calls & 1);
    rc = hostio_upload(h, i, host_actions, B, s);
    if (rc) return rc;
    // the team kernel writes the results straight into this call's buffer,
    // once the read-back two calls back is done with it
    MC_CK(cudaStreamWaitEvent(s, h->res_free[i], 0));
    rc = ragged_do_step(r, nullptr, nullptr, h->d_act[i], s, false, reinterpret_cast<float*>(h->d_res[i]),
                        h->d_res[i] + 4 * B);
    if (rc) return rc;
    MC_CK(cudaEventRecord(h->act_free[i], s));
    return hostio_readback(h, i, host_rewards, host_dones, B, s);
}

extern "C" int mc_ragged_host_join(mc_ragged* r, void* stream) {
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    return hostio_join(r->hio, (cudaStream_t)stream);
}

static int ragged_graph(mc_ragged* r, const uint8_t* actions, int32_t K, RaggedGraph** out) {
    *out = nullptr;
    int rc = ragged_sync_groups(r, false);
    if (rc) return rc;
    for (auto& g : r->graphs)
        if (g.actions == actions && g.K == K && g.version == r->version) {
            *out = &g;
            return MC_OK;
        }
    const long long total = mc_ragged_total_envs(r);
    cudaGraph_t graph = nullptr;
    MC_CK(cudaStreamBeginCapture(r->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K && rc == MC_OK; ++k)
        rc = ragged_do_step(r, nullptr, nullptr, actions + (long long)k * total, r->cap_stream, true);
    cudaError_t ce = cudaStreamEndCapture(r->cap_stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    RaggedGraph g;
    ce = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    g.actions = actions;
    g.K = K;
    g.version = r->version;
    if (r->graphs.size() >= 8) {
        cudaGraphExecDestroy(r->graphs.front().exec);
        r->graphs.erase(r->graphs.begin());
    }
    r->graphs.push_back(g);
    *out = &r->graphs.back();
    return MC_OK;
}

extern "C" int mc_ragged_rollout_prepare(mc_ragged* r, const uint8_t* actions, int32_t K) {
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    if (K < 0) return fail(MC_ERR_INVALID, "K < 0");
    if (K == 0 || mc_ragged_total_envs(r) == 0) return MC_OK;
    if (!actions) return fail(MC_ERR_INVALID, "actions is NULL");
    RaggedGraph* g;
    return ragged_graph(r, actions, K, &g);
}

extern "C" int mc_ragged_rollout(mc_ragged* r, const uint8_t* actions, int32_t K, void* stream) {
    NvtxRange nvtx("mc_ragged_rollout");
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    if (K < 0) return fail(MC_ERR_INVALID, "K < 0");
    if (K == 0 || mc_ragged_total_envs(r) == 0) return MC_OK;
    if (!actions) return fail(MC_ERR_INVALID, "actions is NULL");
    RaggedGraph* g;
    int rc = ragged_graph(r, actions, K, &g);
    if (rc) return rc;
    MC_CK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return MC_OK;
}

extern "C" int mc_ragged_check_error(mc_ragged* r, void* stream) {
    if (!r) return fail(MC_ERR_INVALID, "ragged handle is NULL");
    for (auto* e : r->envs) {
        int rc = mc_env_check_error(e, stream);
        if (rc) return rc;
    }
    return MC_OK;
}

// ---------------------------------------------------------------------------
// stateless entry points (the reference's _C functions)
// ---------------------------------------------------------------------------
static int32_t* stateless_flags() {
    // one flag block per device for the stand-alone entry points; the any-done
    // flag they set is never read (their callers regenerate from Python)
    static int32_t* per_dev[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!per_dev[dev]) {
        int32_t* p = nullptr;
        if (cudaMalloc(&p, MC_FLAG_WORDS * sizeof(int32_t)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, MC_FLAG_WORDS * sizeof(int32_t));
        per_dev[dev] = p;
    }
    return per_dev[dev];
}

extern "C" int mc_generate_world(int8_t* vox, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t gh, uint32_t seed,
                                 void* stream) {
    (void)seed;  // unused by the reference's generator too (kernels.cu:1800)
    if (B < 0 || wx < 1 || wy < 1 || wz < 1) return fail(MC_ERR_INVALID, "bad world dims");
    if (B == 0) return MC_OK;
    if (!vox) return fail(MC_ERR_INVALID, "voxels is NULL");
    long long rows = (long long)B * wy * wx;
    k_generate_world<<<blocks(rows, 128), 128, 0, (cudaStream_t)stream>>>(vox, rows, wx, wy, wz, gh);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_place_tree(int8_t* vox, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t tx, int32_t tz,
                             int32_t gh, void* stream) {
    if (B < 0 || wx < 1 || wy < 1 || wz < 1) return fail(MC_ERR_INVALID, "bad world dims");
    if (tx < 0 || tx >= wx || tz < 0 || tz >= wz)
        return fail(MC_ERR_INVALID, "tree at (%d,%d) outside the world; the reference writes out of bounds here", tx,
                    tz);
    if (B == 0) return MC_OK;
    if (!vox) return fail(MC_ERR_INVALID, "voxels is NULL");
    k_place_tree<<<blocks(B, 256), 256, 0, (cudaStream_t)stream>>>(vox, B, wx, wy, wz, tx, tz, gh);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_place_house(int8_t* vox, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t hx, int32_t hz,
                              int32_t gh, void* stream) {
    if (B < 0 || wx < 1 || wy < 1 || wz < 1) return fail(MC_ERR_INVALID, "bad world dims");
    if (B == 0) return MC_OK;
    if (!vox) return fail(MC_ERR_INVALID, "voxels is NULL");
    k_place_house<<<blocks(B, 256), 256, 0, (cudaStream_t)stream>>>(vox, B, wx, wy, wz, hx, hz, gh);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_reset_agents(float* pos, float* vel, float* yaw, float* pitch, uint8_t* og, const uint8_t* dr,
                               int32_t B, float sx, float sy, float sz, void* stream) {
    if (B < 0) return fail(MC_ERR_INVALID, "B < 0");
    if (B == 0) return MC_OK;
    if (!pos || !vel || !yaw || !pitch || !og || !dr) return fail(MC_ERR_INVALID, "NULL buffer");
    k_reset_agents<<<blocks(B, 256), 256, 0, (cudaStream_t)stream>>>(pos, vel, yaw, pitch, og, dr, B, sx, sy, sz);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_render(const mc_env_config* cfg, const mc_env_state* st, int32_t shaded, void* stream) {
    int rc = check_config(cfg);
    if (rc) return rc;
    if (!st || (cfg->batch_size && (!st->voxels || !st->obs))) return fail(MC_ERR_INVALID, "NULL buffer");
    mc_kp k;
    fill_kp(&k, cfg, st);
    int fam = shaded ? (cfg->obs_mode == MC_OBS_UINT8_FAST ? MC_FAM_SHADED_FAST : MC_FAM_SHADED) : k.family;
    if (fam == MC_FAM_PREBASIS ? !st->basis : !st->cameras) return fail(MC_ERR_INVALID, "cameras/basis is NULL");
    return backend_rc(backend_of(cfg->numerics)->render(&k, fam, (cudaStream_t)stream), "render");
}

extern "C" int mc_precompute_camera_basis(const float* cameras, float* basis, int32_t B, int32_t W, int32_t H,
                                          float fov, int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics");
    if (B < 0 || W < 1 || H < 1) return fail(MC_ERR_INVALID, "bad sizes");
    if (B == 0) return MC_OK;
    if (!cameras || !basis) return fail(MC_ERR_INVALID, "NULL buffer");
    mc_kp k;
    memset(&k, 0, sizeof(k));
    k.B = B;
    k.W = W;
    k.H = H;
    k.fov = fov;
    k.cameras = (float*)cameras;
    k.basis = basis;
    return backend_rc(be->basis(&k, (cudaStream_t)stream), "basis");
}

extern "C" int mc_render_uint8_prebasis(const int8_t* vox, const float* basis, uint8_t* out, int32_t B, int32_t wx,
                                        int32_t wy, int32_t wz, int32_t W, int32_t H, int32_t max_steps,
                                        int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics");
    if (B < 0 || W < 1 || H < 1 || wx < 1 || wy < 1 || wz < 1) return fail(MC_ERR_INVALID, "bad sizes");
    if (B == 0) return MC_OK;
    if (!vox || !basis || !out) return fail(MC_ERR_INVALID, "NULL buffer");
    mc_kp k;
    memset(&k, 0, sizeof(k));
    k.B = B;
    k.wx = wx;
    k.wy = wy;
    k.wz = wz;
    k.W = W;
    k.H = H;
    k.max_steps = max_steps;
    k.voxels = (int8_t*)vox;
    k.basis = (float*)basis;
    k.obs = out;
    k.family = MC_FAM_PREBASIS;
    return backend_rc(be->render(&k, MC_FAM_PREBASIS, (cudaStream_t)stream), "render_prebasis");
}

extern "C" int mc_render_uint8_coalesced(const int8_t* vox, const float* basis, uint8_t* out, int32_t B, int32_t ws,
                                         int32_t W, int32_t H, int32_t max_steps, int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics");
    if (B < 0 || W < 1 || H < 1 || ws < 1) return fail(MC_ERR_INVALID, "bad sizes");
    if (B == 0) return MC_OK;
    if (!vox || !basis || !out) return fail(MC_ERR_INVALID, "NULL buffer");
    return backend_rc(be->render_coalesced(vox, basis, out, B, ws, W, H, max_steps, (cudaStream_t)stream),
                      "render_coalesced");
}

extern "C" int mc_step_stateless(const mc_env_config* cfg, const mc_env_state* st, const int8_t* buttons,
                                 const float* look, const mc_decode_buffers* dec, int32_t form, void* stream) {
    int rc = check_config(cfg);
    if (rc) return rc;
    rc = check_state(cfg, st, cfg->obs_mode == MC_OBS_UINT8_PREBASIS_FULL);
    if (rc) return rc;
    if (cfg->batch_size == 0) return MC_OK;
    if (!buttons || !look) return fail(MC_ERR_INVALID, "buttons/look are NULL");
    mc_kp k;
    fill_kp(&k, cfg, st);
    k.ext_done = (cfg->obs_mode == MC_OBS_UINT8_PREBASIS_FULL) ? 0 : 1;
    k.buttons = buttons;
    k.look = look;
    k.flags = stateless_flags();
    if (!k.flags) return fail(MC_ERR_CUDA, "flag buffer allocation failed");
    const mc_backend* be = backend_of(cfg->numerics);
    if (form == MC_FORM_PLAIN) {
        if (!dec || !dec->forward_in || !dec->strafe_in || !dec->delta_yaw_in || !dec->delta_pitch_in ||
            !dec->jump_in || !dec->do_break || !dec->do_place || !dec->speed_mult)
            return fail(MC_ERR_INVALID, "the plain form needs the 8 decode buffers");
        k.s_fwd = dec->forward_in;
        k.s_strafe = dec->strafe_in;
        k.s_dyaw = dec->delta_yaw_in;
        k.s_dpitch = dec->delta_pitch_in;
        k.s_jump = dec->jump_in;
        k.s_brk = dec->do_break;
        k.s_place = dec->do_place;
        k.s_speed = dec->speed_mult;
        return backend_rc(be->step_plain(&k, (cudaStream_t)stream), "step_plain");
    }
    if (form == MC_FORM_FUSED) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        mc_fused_cfg f;
        int wxyz = cfg->world_x * cfg->world_y * cfg->world_z;
        f.stage = (wxyz <= 8192 && (wxyz & 15) == 0) ? 1 : 0;
        f.warps_per_cta = 8;
        f.ctas_per_sm = 4;
        f.tile_w = 4;
        f.team_warps = 1;
        f.coop = 0;
        return backend_rc(be->step_fused(&k, &f, sms, (cudaStream_t)stream), "step_fused");
    }
    return fail(MC_ERR_INVALID, "unknown form %d", form);
}

extern "C" int mc_physics(float* pos, float* vel, float* yaw, float* pitch, uint8_t* og, const float* fwd,
                          const float* strafe, const float* dyaw, const float* dpitch, const uint8_t* jump,
                          const float* speed, int32_t B, int32_t ws, float dt, float gravity, float walk_speed,
                          float jump_vel, int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics");
    if (B < 0 || ws < 1) return fail(MC_ERR_INVALID, "bad sizes");
    if (B == 0) return MC_OK;
    mc_kp k;
    memset(&k, 0, sizeof(k));
    k.B = B;
    k.wx = k.wy = k.wz = ws;  // cubic, as launch_physics (kernels.cu:2244-2249)
    k.dt = dt;
    k.gravity = gravity;
    k.walk_speed = walk_speed;
    k.jump_vel = jump_vel;
    k.positions = pos;
    k.velocities = vel;
    k.yaws = yaw;
    k.pitches = pitch;
    k.on_ground = og;
    k.s_fwd = (float*)fwd;
    k.s_strafe = (float*)strafe;
    k.s_dyaw = (float*)dyaw;
    k.s_dpitch = (float*)dpitch;
    k.s_jump = (uint8_t*)jump;
    k.s_speed = (float*)speed;
    // physics reads brk/place only through load_dec; point them at jump (unused)
    k.s_brk = (uint8_t*)jump;
    k.s_place = (uint8_t*)jump;
    return backend_rc(be->physics(&k, (cudaStream_t)stream), "physics");
}

extern "C" int mc_raycast_break(int8_t* vox, const float* pos, const float* yaw, const float* pitch,
                                const uint8_t* do_break, float* rewards, int32_t B, int32_t ws, int32_t target_block,
                                float reward_value, int32_t numerics, void* stream) {
    const mc_backend* be = backend_of(numerics);
    if (!be) return fail(MC_ERR_INVALID, "unknown numerics");
    if (B < 0 || ws < 1) return fail(MC_ERR_INVALID, "bad sizes");
    if (target_block < -128 || target_block > 127) return fail(MC_ERR_INVALID, "target_block outside int8");
    if (B == 0) return MC_OK;
    mc_kp k;
    memset(&k, 0, sizeof(k));
    k.B = B;
    k.wx = k.wy = k.wz = ws;
    k.voxels = vox;
    k.positions = (float*)pos;
    k.yaws = (float*)yaw;
    k.pitches = (float*)pitch;
    k.s_brk = (uint8_t*)do_break;
    k.s_place = (uint8_t*)do_break;
    k.rewards = rewards;
    k.target_block = target_block;
    k.reward_value = reward_value;
    // load_agent reads velocities and on_ground; the break kernel only uses
    // position and view, so point those reads at valid memory
    k.velocities = (float*)pos;
    k.on_ground = (uint8_t*)do_break;
    return backend_rc(be->interact(&k, 1, (cudaStream_t)stream), "raycast_break");
}

namespace {
// obs / 255 for every channel value; a thread converts 4 pixels at a time
// when every env's pixel count is a multiple of 4 (then 12 bytes of input are
// 4-byte aligned and each output plane segment is a float4), else 1 pixel.
template <bool NCHW, int PX>
__global__ void k_obs_to_policy(const uint8_t* __restrict__ obs, float* __restrict__ out, long long B, int HW) {
    const long long groups = B * (HW / PX);
    for (long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < groups;
         gi += (long long)gridDim.x * blockDim.x) {
        const long long b = gi / (HW / PX);
        const int p0 = (int)(gi - b * (HW / PX)) * PX;
        const long long pix = b * HW + p0;
        float v[3 * PX];
        if (PX == 4) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(obs + pix * 3);
            const uint32_t w0 = src[0], w1 = src[1], w2 = src[2];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[k] = __fdiv_rn((float)((w0 >> (8 * k)) & 0xff), 255.0f);
                v[4 + k] = __fdiv_rn((float)((w1 >> (8 * k)) & 0xff), 255.0f);
                v[8 + k] = __fdiv_rn((float)((w2 >> (8 * k)) & 0xff), 255.0f);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3 * PX; ++k) v[k] = __fdiv_rn((float)obs[pix * 3 + k], 255.0f);
        }
        if (NCHW) {
            // v holds PX pixels' RGB interleaved: channel c of pixel k is v[3k + c]
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float* plane = out + (b * 3 + c) * (long long)HW + p0;
                if (PX == 4)
                    *reinterpret_cast<float4*>(plane) = make_float4(v[c], v[3 + c], v[6 + c], v[9 + c]);
                else
                    plane[0] = v[c];
            }
        } else {
            float* dst = out + pix * 3;
            if (PX == 4) {
                float4* d4 = reinterpret_cast<float4*>(dst);
                d4[0] = make_float4(v[0], v[1], v[2], v[3]);
                d4[1] = make_float4(v[4], v[5], v[6], v[7]);
                d4[2] = make_float4(v[8], v[9], v[10], v[11]);
            } else {
                dst[0] = v[0];
                dst[1] = v[1];
                dst[2] = v[2];
            }
        }
    }
}
}  // namespace

extern "C" int mc_obs_to_policy(const uint8_t* obs, float* out, int64_t B, int32_t H, int32_t W, int32_t layout,
                                void* stream) {
    if (B < 0 || H < 0 || W < 0) return fail(MC_ERR_INVALID, "bad sizes");
    if (layout != MC_POLICY_NCHW && layout != MC_POLICY_NHWC) return fail(MC_ERR_INVALID, "unknown layout %d", layout);
    const long long HW = (long long)H * W;
    if (B == 0 || HW == 0) return MC_OK;
    if (HW > (1LL << 30)) return fail(MC_ERR_INVALID, "image too large");
    if (!obs || !out) return fail(MC_ERR_INVALID, "NULL buffer");
    const bool vec = (HW % 4) == 0 && (((uintptr_t)obs) & 3) == 0 && (((uintptr_t)out) & 15) == 0;
    const long long groups = B * (vec ? HW / 4 : HW);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::min<long long>((groups + 255) / 256, (long long)sms * 16);
    cudaStream_t s = (cudaStream_t)stream;
    if (layout == MC_POLICY_NCHW) {
        if (vec) k_obs_to_policy<true, 4><<<grid, 256, 0, s>>>(obs, out, B, (int)HW);
        else k_obs_to_policy<true, 1><<<grid, 256, 0, s>>>(obs, out, B, (int)HW);
    } else {
        if (vec) k_obs_to_policy<false, 4><<<grid, 256, 0, s>>>(obs, out, B, (int)HW);
        else k_obs_to_policy<false, 1><<<grid, 256, 0, s>>>(obs, out, B, (int)HW);
    }
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_philox_actions(uint8_t* actions, int32_t B, int32_t K, int32_t env_offset, int32_t step0,
                                 uint64_t seed, int32_t break_half, void* stream) {
    if (B < 0 || K < 0) return fail(MC_ERR_INVALID, "bad sizes");
    long long n = (long long)B * K;
    if (n == 0) return MC_OK;
    if (!actions) return fail(MC_ERR_INVALID, "actions is NULL");
    int grid = (int)((n + 255) / 256);
    if (grid > 148 * 32) grid = 148 * 32;
    k_philox<<<grid, 256, 0, (cudaStream_t)stream>>>(actions, B, K, env_offset, step0, seed, break_half);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

extern "C" int mc_discrete_to_buttons(const uint8_t* actions, int32_t B, float look_delta, int8_t* buttons,
                                      float* look, void* stream) {
    if (B < 0) return fail(MC_ERR_INVALID, "B < 0");
    if (B == 0) return MC_OK;
    if (!actions || !buttons || !look) return fail(MC_ERR_INVALID, "NULL buffer");
    k_discrete<<<blocks(B, 256), 256, 0, (cudaStream_t)stream>>>(actions, B, look_delta, buttons, look);
    MC_CK(cudaGetLastError());
    return MC_OK;
}

int mc_step_stateless_with_flags(const mc_env_config* cfg, const mc_env_state* st, const int8_t* buttons,
                                 const float* look, const mc_decode_buffers* dec, int32_t* flags, int form,
                                 void* stream) {
    int rc = check_config(cfg);
    if (rc) return rc;
    rc = check_state(cfg, st, cfg->obs_mode == MC_OBS_UINT8_PREBASIS_FULL);
    if (rc) return rc;
    if (cfg->batch_size == 0) return MC_OK;
    if (!buttons || !look) return fail(MC_ERR_INVALID, "buttons/look are NULL");
    if (form != MC_FORM_PLAIN || !dec || !flags) return fail(MC_ERR_INVALID, "plain form with decode buffers and flags");
    mc_kp k;
    fill_kp(&k, cfg, st);
    k.ext_done = (cfg->obs_mode == MC_OBS_UINT8_PREBASIS_FULL) ? 0 : 1;
    k.buttons = buttons;
    k.look = look;
    k.flags = flags;
    k.s_fwd = dec->forward_in;
    k.s_strafe = dec->strafe_in;
    k.s_dyaw = dec->delta_yaw_in;
    k.s_dpitch = dec->delta_pitch_in;
    k.s_jump = dec->jump_in;
    k.s_brk = dec->do_break;
    k.s_place = dec->do_place;
    k.s_speed = dec->speed_mult;
    return backend_rc(backend_of(cfg->numerics)->step_plain(&k, (cudaStream_t)stream), "step_plain");
}
