// mc_internal.h - parameter blocks shared by the host runtime and the two
// numerics back ends (mc_fast.cu, mc_ieee.cu).  Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Render families: one per reference render kernel.
enum {
    MC_FAM_SHADED = 0,       // render_kernel / render_kernel_uint8 (kernels.cu:87-470)
    MC_FAM_SHADED_FAST = 1,  // render_kernel_uint8_fast (kernels.cu:1268-1442)
    MC_FAM_MINIMAL = 2,      // render_kernel_uint8_minimal (kernels.cu:985-1119)
    MC_FAM_FP16 = 3,         // render_kernel_uint8_fp16 (kernels.cu:1127-1260)
    MC_FAM_PREBASIS = 4,     // render_kernel_uint8_prebasis / _smem (kernels.cu:568-700, 835-982)
};

// Device flag words owned by an env handle.
enum {
    MC_FLAG_ANY_DONE = 0,    // set by a step when any env is done
    MC_FLAG_REGEN_CTR = 1,   // CTAs of the regeneration kernel that finished
    MC_FLAG_ERROR = 2,       // MC_KERR_* recorded by a kernel
    MC_FLAG_WORK = 3,        // next env to claim (fused kernel, dynamic schedule)
    MC_FLAG_WARPS_DONE = 4,  // warps of the fused kernel that finished
    MC_FLAG_WORDS = 8
};

// Error codes a kernel can record in flags[MC_FLAG_ERROR] (never a trap).
enum { MC_KERR_NONE = 0, MC_KERR_TMA_TIMEOUT = 1, MC_KERR_BOUNDS = 2 };

// Places the debug build checks an index (the first violation's site is
// reported by mc_debug_bounds_report).
enum {
    MC_SITE_INTERACT = 1,      // interaction samples: world voxel read/write
    MC_SITE_EYE = 2,           // the eye's voxel
    MC_SITE_MARCH_GLOBAL = 3,  // march over a world in global memory
    MC_SITE_MARCH_SHARED = 4,  // march over a staged world (C++ loops)
    MC_SITE_MARCH_PACKED = 5,  // PTX packed march: load address vs the staged world +- one layer
    MC_SITE_MARCH_SPLIT = 6,   // PTX split march: the same
    MC_SITE_MARCH_SMEM = 7,    // PTX marches: load address vs the CTA's dynamic shared memory
    MC_SITE_BAND = 8,          // a pixel's bytes in the shared-memory band
    MC_SITE_COPY_OUT = 9,      // a band's bytes in the env's observation
    MC_SITE_DEBUG = 10,        // per-pixel debug code
    MC_SITE_PATCH = 11,        // the interaction's voxel patched into the staged world
    MC_SITE_TABLE = 12,        // u/v tables, colour tables
    MC_SITE_STAGE = 13,        // a bulk copy's destination vs the CTA's dynamic shared memory
    MC_SITE_SCAN = 14,         // a staged world's rows read by the up-bounds scan
};

// Polls of an mbarrier before a bulk-copy wait gives up (each poll is one
// try_wait, which itself blocks for a short hardware-defined time).
#define MC_WAIT_POLLS_DEFAULT (1 << 22)

// Everything one step launch needs, passed to kernels by value.
struct mc_kp {
    // sizes
    int B, wx, wy, wz, W, H;
    // parameters (MineEnv.__init__, minecu/__init__.py:141-165)
    int max_steps;
    float vd, fov, dt, gravity, walk_speed, sprint_mult, jump_vel;
    int gh;
    int target_block;  // int8 semantics
    float reward_value;
    float spawn_x, spawn_y, spawn_z;
    int episode_rule;  // 0: python rule (has_limit && cnt >= L); 1: kernel rule (L > 0 && cnt >= L)
    int ext_done;      // 1: do_reset is an input and step_count is not touched (the reference's
                       //    _C.step* entry points, whose episode logic runs in Python)
    int sched_dynamic; // fused kernel: 1 = warps claim envs from flags[MC_FLAG_WORK] (needs a
                       // flag block no other launch uses concurrently); 0 = static striding
    int has_limit, episode_length;
    int family;   // MC_FAM_*
    int obs_f32;  // float32 obs (else uint8)
    float look_delta;  // discrete-action look step (radians)
    int regen_per_env; // MC_REGEN_PER_ENV: a done (or reset) env regenerates only its own world
    int wait_polls;    // bounded waits on a bulk copy: 0 = MC_WAIT_POLLS_DEFAULT polls, n > 0 = n polls,
                       // < 0 = give up at once (a test of the timeout path)
    // state (device, borrowed from the caller)
    int8_t* voxels;
    float* positions;
    float* velocities;
    float* yaws;
    float* pitches;
    uint8_t* on_ground;
    int32_t* step_count;
    uint8_t* do_reset;
    float* cameras;
    float* basis;  // [B,14] for the prebasis family, else may be null
    void* obs;
    float* rewards;
    int32_t* dbg_interact;  // optional
    int16_t* dbg_pixel;     // optional
    // actions: either buttons+look, or discrete actions
    const int8_t* buttons;
    const float* look;
    const uint8_t* actions;
    // plain-form decode scratch (the reference's 8 decode buffers)
    float* s_fwd;
    float* s_strafe;
    float* s_dyaw;
    float* s_dpitch;
    uint8_t* s_jump;
    uint8_t* s_brk;
    uint8_t* s_place;
    float* s_speed;
    int32_t* flags;               // MC_FLAG_* words
    const int8_t* world_template; // one generated world (wx*wy*wz bytes)
    // optional (per-warp fused kernel only): every env's reward and done also
    // written here, in env order (the host-buffer step's read-back buffer)
    float* res_rewards;
    uint8_t* res_dones;
};

// Launch shape of the fused step kernel (chosen by the autotuner).
struct mc_fused_cfg {
    int stage;          // 1: copy each rendered world into shared memory with a bulk copy; 0: read voxels from L1/L2
    int warps_per_cta;  // 4 or 8
    int ctas_per_sm;    // persistent grid = SMs * ctas_per_sm
    int tile_w;         // march tiles of tile_w x (32/tile_w) pixels (4, 8, 16 or 32)
    int team_warps;     // 1 with coop = 0: the per-warp kernel; else the team kernel with teams of this many warps
    int coop;           // team kernel: 1 = a team renders each env together
};

// Several env groups stepped by one launch of the team kernel (k_step_team).
enum { MC_MAX_GROUPS = 16 };
enum { MC_COLOUR_TABLE_BYTES = 224 };  // shared colour tables of the fused kernels (16-aligned)
// the common-case render loop's tables (colour x shade: 13 x 4 float4; packed
// flat colours: 13 uint32 padded to 64 bytes), after the colour tables
enum { MC_FAST_TABLE_BYTES = 13 * 4 * 16 + 64 };
enum { MC_TEAM_HEAD_BYTES = 256 };     // per-team shared words ahead of the team's world buffer
enum { MC_ENV_STASH_BYTES = 96 };      // one env's render constants, kept in shared memory (depth 2)
struct mc_ragged_kp {
    mc_kp groups[MC_MAX_GROUPS];    // the groups' parameter blocks (kernel parameter space)
    // optional: every env's reward and done flag also written at its global
    // index (one contiguous read-back for a batch of jobs)
    float* rewards_cat;
    uint8_t* dones_cat;
    // actions of all groups, concatenated in group order: discrete actions, or buttons + look
    const uint8_t* actions;
    const int8_t* buttons;
    const float* look;
    int32_t* flags;                      // work counter of the launch
    long long start[MC_MAX_GROUPS + 1];  // first global env index of each group; start[ngroups] = total
    int ngroups;
    // work units: groups visited in `order` (most expensive envs first);
    // ustart[v] = first unit of the v-th visited group, ustart[ngroups] = total units
    int order[MC_MAX_GROUPS];
    long long ustart[MC_MAX_GROUPS + 1];
    int team_warps;                 // warps per team
    int coop_mask;                  // bit g: a whole team renders each env of group g
    int stage_mask;                 // bit g: group g's worlds are bulk-copied into shared memory
    int tile_w[MC_MAX_GROUPS];
    int uv_off[MC_MAX_GROUPS];      // float offset of each group's u table (v follows)
    int sched_dynamic;              // 1: teams claim units from flags[MC_FLAG_WORK]
    // shared-memory layout (bytes): colour tables at 0, then
    int tables_off, teams_off, warps_off;
    int team_bytes;                 // MC_TEAM_HEAD_BYTES + max(depth, 1) x world_stride
    int slot_bytes;                 // world slot of one warp of a per-warp staged group
    int depth;                      // staging depth: 0 none, 1 one world buffer per stepper, 2 two (the
                                    // next unit's world is copied while the current one renders)
    int world_stride;               // bytes of one depth slot of a team's world region
    int warp_bytes;                 // 16 (two mbarriers) + 128 (march start values) [+ depth 2: two env
                                    // stashes] + one band of observation bytes
    int tail_bytes;                 // allocated after the warps: the march may read one world layer past the last world
};

// One numerics back end (ref_fast or ieee).
struct mc_backend {
    const char* name;
    int (*step_plain)(const mc_kp* p, cudaStream_t s);
    int (*step_fused)(const mc_kp* p, const mc_fused_cfg* cfg, int num_sms, cudaStream_t s);
    // shaded (f32/u8) or flat render of every env from p->cameras (or p->basis)
    int (*render)(const mc_kp* p, int family, cudaStream_t s);
    // stand-alone kernels of the reference's _C module
    int (*basis)(const mc_kp* p, cudaStream_t s);
    int (*decode)(const mc_kp* p, cudaStream_t s);
    int (*physics)(const mc_kp* p, cudaStream_t s);
    int (*interact)(const mc_kp* p, int break_only, cudaStream_t s);
    int (*render_coalesced)(const int8_t* vox_yxzb, const float* basis, uint8_t* out, int B, int ws,
                            int W, int H, int max_steps, cudaStream_t s);
    size_t (*fused_smem_bytes)(const mc_kp* p, const mc_fused_cfg* cfg);
    // the team kernel over rk's groups: grid = SMs x ctas_per_sm (at most one unit per team)
    int (*step_team)(const mc_ragged_kp* rk, int family, int obs_f32, int warps_per_cta, int ctas_per_sm,
                     int num_sms, cudaStream_t s);
    // debug build (MC_CHECK_BOUNDS=1): read and clear the bounds-check record; -1 in the normal build
    int (*bounds_report)(int32_t out[4], cudaStream_t s);
    // debug build: one failed check at site 0 with no access behind it; -1 in the normal build
    int (*bounds_selftest)(cudaStream_t s);
};

extern "C" const mc_backend* mc_backend_fast();
extern "C" const mc_backend* mc_backend_ieee();

// numerics-independent kernels (mc_runtime.cu)
int mc_launch_reset_agents(const mc_kp* p, const uint8_t* mask, cudaStream_t s);
int mc_launch_regen(const mc_kp* p, int conditional, cudaStream_t s);
int mc_launch_regen_if(const mc_kp* p, const uint8_t* flag, cudaStream_t s);
// The conditional regeneration of up to MC_MAX_GROUPS groups in one launch
// (groups that cannot end an episode are skipped; no launch when none can);
// ctr is a counter word no other launch uses concurrently.
int mc_launch_regen_groups(const mc_kp* const* kps, int G, int32_t* ctr, cudaStream_t s);

// Record an error message for mc_last_error() and return `code`.
int mc_set_error(int code, const char* msg);
// mc_step_stateless with the flag words supplied by the caller (no lazy
// allocation of the per-device flag block).
struct mc_env_config;
struct mc_env_state;
struct mc_decode_buffers;
int mc_step_stateless_with_flags(const mc_env_config* cfg, const mc_env_state* st, const int8_t* buttons,
                                 const float* look, const mc_decode_buffers* dec, int32_t* flags, int form,
                                 void* stream);
