/*
 * minecu_b200.h - C-ABI of libminecu_b200.so, the B200 implementation of
 * mine.cu's environment step.
 *
 * The reference exposes its step as `extern "C"` launchers in
 * src/kernels.cu:2076-3245 (launch_step*, launch_render*, launch_generate_world,
 * ...) bound by pybind11 in src/bindings.cpp.  Those take raw device
 * pointers, run on the legacy default stream, return void and keep
 * process-global CUDA-graph state.  The entry points below take the same
 * pointers and sizes, plus an explicit CUDA stream (`void*` holding a
 * cudaStream_t, NULL = legacy default stream) and return an int status
 * (MC_OK or a negative MC_ERR_*; mc_last_error() gives the message).
 *
 * Ownership: the caller owns every state buffer (as the reference's
 * MineEnv owns its torch tensors, minecu/__init__.py:214-256); the library
 * borrows the pointers and writes in place.  An mc_env handle owns only
 * small internal buffers (flag words, decode scratch, one template world).
 *
 * Threading: a handle may be used by one host thread at a time.  Different
 * handles are independent (the reference's graph cache is process-global per
 * mode, src/kernels.cu:2376-2382; here it is per handle).
 */
#ifndef MINECU_B200_H
#define MINECU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC_ABI_VERSION 2

/* status codes */
#define MC_OK 0
#define MC_ERR_INVALID (-1)     /* bad argument (size, pointer, alignment) */
#define MC_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define MC_ERR_KERNEL (-3)      /* a kernel recorded an error (bounded wait expired) */
#define MC_ERR_UNSUPPORTED (-4) /* configuration not supported by this build */
#define MC_ERR_BUDGET (-5)      /* env server: admission would exceed the HBM budget */
#define MC_ERR_TIMEOUT (-6)     /* env server: the wait ended before the request completed */
#define MC_ERR_BUSY (-7)        /* env server: the job still has requests queued or running */

/* numerics modes */
#define MC_NUMERICS_REF_FAST 0 /* same fast-math CUDA calls and op order as the reference build */
#define MC_NUMERICS_IEEE 1     /* IEEE-754 ops, bit-identical to the CPU checker */

/* observation modes = MineEnv(obs_dtype=...) (minecu/__init__.py:162-169) */
#define MC_OBS_FLOAT32 0
#define MC_OBS_UINT8 1
#define MC_OBS_UINT8_MINIMAL 2
#define MC_OBS_UINT8_FP16 3
#define MC_OBS_UINT8_PREBASIS 4
#define MC_OBS_UINT8_PREBASIS_FULL 5
#define MC_OBS_UINT8_SMEM 6
#define MC_OBS_UINT8_FAST 7

/* step forms */
#define MC_FORM_PLAIN 0 /* one kernel per reference kernel, in the reference's order */
#define MC_FORM_FUSED 1 /* one persistent kernel per step */

/* Constructor arguments of MineEnv (minecu/__init__.py:141-165). */
typedef struct mc_env_config {
    int32_t batch_size;
    int32_t world_x, world_y, world_z;
    int32_t render_width, render_height;
    int32_t max_steps;
    float view_distance;
    float fov_degrees;
    float dt;
    float gravity;
    float walk_speed;
    float sprint_mult;
    float jump_vel;
    int32_t ground_height;
    int32_t target_block; /* -128..127, int8 semantics as the reference */
    float reward_value;
    int32_t has_episode_limit; /* 0 = episode_length None */
    int32_t episode_length;
    int32_t obs_mode;  /* MC_OBS_* */
    int32_t numerics;  /* MC_NUMERICS_* */
    float look_delta;  /* radians per discrete look action */
    /* 0: spawn at (world_x/2, ground_height+2, world_z/2) as MineEnv does
     * (minecu/__init__.py:195-198); 1: use spawn_x/y/z, as the reference's
     * launchers take them (src/kernels.cu:2497-2520) */
    int32_t spawn_override;
    float spawn_x, spawn_y, spawn_z;
} mc_env_config;

/* State buffers (device pointers), the MineEnv attributes of
 * minecu/__init__.py:214-256.  dbg_* are optional debug outputs the
 * reference keeps internal: the voxel index the interaction touched per env
 * (-1 none) and per pixel (hit_block + 1) | ((hit_face + 1) << 8). */
typedef struct mc_env_state {
    int8_t* voxels;      /* [B, Y, X, Z] */
    float* positions;    /* [B, 3] */
    float* velocities;   /* [B, 3] */
    float* yaws;         /* [B] */
    float* pitches;      /* [B] */
    uint8_t* on_ground;  /* [B] (torch.bool) */
    int32_t* step_count; /* [B] */
    uint8_t* do_reset;   /* [B] (torch.bool) */
    float* cameras;      /* [B, 5] */
    float* basis;        /* [B, 14] for the prebasis modes, else NULL */
    void* obs;           /* [B, H, W, 3] uint8 or float32 */
    float* rewards;      /* [B] */
    int32_t* dbg_interact; /* [B] or NULL */
    int16_t* dbg_pixel;    /* [B, H, W] or NULL */
} mc_env_state;

typedef struct mc_env mc_env;

/* Launch shape of the fused kernel (see mc_env_set_fused_config). */
typedef struct mc_fused_config {
    int32_t stage;         /* 1: bulk-copy each marched world into shared memory */
    int32_t warps_per_cta; /* 1..8 warps per CTA */
    int32_t ctas_per_sm;   /* persistent grid = SMs x ctas_per_sm */
    int32_t tile_w;        /* a warp marches tiles of tile_w x (32/tile_w) pixels: 4, 8, 16 or 32 */
    int32_t team_warps;    /* 1: one warp steps and renders each env (4 or 8 warps per CTA);
                              1, 2, 4 or 8 with coop = 1: a team of that many warps renders each env */
    int32_t coop;          /* 1: the team shares one env (its image bands and one staged world) */
} mc_fused_config;

/* ---- library ---------------------------------------------------------- */
int mc_abi_version(void);
/* Message of the last failed call on this host thread. */
const char* mc_last_error(void);

/* ---- env handle: MineEnv (minecu/__init__.py:65-479) ------------------ */
/* Replaces MineEnv.__init__'s native half (minecu/__init__.py:141-212). */
int mc_env_create(const mc_env_config* cfg, const mc_env_state* state, mc_env** out);
int mc_env_destroy(mc_env* env);
/* Re-point the borrowed state buffers (same sizes). */
int mc_env_set_state(mc_env* env, const mc_env_state* state);
/* MineEnv._generate_world (minecu/__init__.py:258-268): every world. */
int mc_env_generate_world(mc_env* env, void* stream);
/* MineEnv.reset(mask) (minecu/__init__.py:270-302); mask = device bool[B]
 * or NULL for all.  No host synchronisation: the "any env reset" test of
 * the reference (mask.any()) runs on the device. */
int mc_env_reset(mc_env* env, const uint8_t* mask, void* stream);
/* MineEnv.step(buttons int8[B,8], look float32[B,2]) (minecu/__init__.py:304-444),
 * including the all-world regeneration when any env is done. */
int mc_env_step(mc_env* env, const int8_t* buttons, const float* look, int form, void* stream);
/* The discrete form step(actions) of docs/environment.md:5-17: actions
 * uint8[B] in 0..10, look step = config.look_delta. */
int mc_env_step_discrete(mc_env* env, const uint8_t* actions, int form, void* stream);
/* The discrete step with host buffers: the reference's step(actions) as a
 * caller with a host-side policy drives it (minecu/__init__.py:304-444; its
 * rewards and dones are then copied back to the host).  actions uint8[B]
 * are read from host memory, rewards float32[B] and dones uint8[B] written
 * to host memory.  The copies run on the env's own upload and read-back
 * streams and overlap the device steps of the neighbouring calls: the
 * actions of call k+1 go up while step k runs, the results of step k come
 * back while step k+1 runs.  Host buffers must be pinned (cudaHostAlloc or
 * cudaHostRegister) and must stay untouched until the results of the call
 * are known to be in host memory: after mc_env_host_join(env, s) on stream
 * s, once s reaches that point.  The first call allocates the env's two
 * action and two result buffers (B * 6 bytes each pair). */
int mc_env_step_host(mc_env* env, const uint8_t* host_actions, float* host_rewards, uint8_t* host_dones, int form,
                     void* stream);
/* Make `stream` wait, on the device, for every copy issued by the
 * mc_env_step_host calls so far (their host results are complete when the
 * stream reaches this point). */
int mc_env_host_join(mc_env* env, void* stream);
/* MineEnv.get_obs / _render (minecu/__init__.py:446-472). */
int mc_env_render(mc_env* env, void* stream);
/* Regenerate every world of the env when the device byte *flag is non-zero,
 * without a host synchronisation: the reference's "any env done -> every
 * world regenerated" rule (minecu/__init__.py:356-358, 439-441) across the
 * shards of a batch split over several GPUs, with *flag the all-reduced
 * any-done byte. */
int mc_env_regenerate_if(mc_env* env, const uint8_t* flag, void* stream);
/* Which worlds a step's dones (and reset(mask)) regenerate.  MC_REGEN_ALL,
 * the default: every world when any env is done or reset, the reference's
 * rule (minecu/__init__.py:290-300, 356-358, 439-441).  MC_REGEN_PER_ENV
 * (opt-in): only the worlds of the envs done or reset; the other envs keep
 * their worlds.  The reference has this only as unused masked kernels
 * (src/kernels.cu:1988-2069), which also leave out the house; here a
 * regenerated world is the start world, house included.  Setting the mode
 * drops the env's cached rollout graphs. */
#define MC_REGEN_ALL 0
#define MC_REGEN_PER_ENV 1
int mc_env_set_regen_mode(mc_env* env, int32_t mode);
/* The mode, or a negative status. */
int mc_env_get_regen_mode(const mc_env* env);
/* Budget of the fused kernels' bounded waits for a bulk copy of a world into
 * shared memory: polls > 0 polls, 0 = give up at once (makes every wait run
 * out, to test the timeout path), < 0 = the default (2^22 polls).  A wait
 * that runs out records a timeout in the error word (mc_env_check_error)
 * and the warp renders that env and every later one from global memory, so
 * the results stay the same.  No counterpart in the reference, which has no
 * bulk copies. */
int mc_env_set_wait_limit(mc_env* env, int32_t polls);
/* K fused steps of discrete actions actions[K,B] captured once in a CUDA
 * graph and replayed; rewards_out / dones_out ([K,B], optional) receive each
 * step's rewards and dones.  The graph is cached per (actions, outputs, K). */
int mc_env_rollout(mc_env* env, const uint8_t* actions, int32_t K, float* rewards_out, uint8_t* dones_out,
                   void* stream);
/* Capture (and cache) the rollout graph without running it. */
int mc_env_rollout_prepare(mc_env* env, const uint8_t* actions, int32_t K, float* rewards_out, uint8_t* dones_out);
int mc_env_set_fused_config(mc_env* env, const mc_fused_config* cfg);
int mc_env_get_fused_config(const mc_env* env, mc_fused_config* cfg);
/* Reads and clears the device error word (synchronises the stream). */
int mc_env_check_error(mc_env* env, void* stream);

/* ---- debug build (no counterpart in the reference, which checks no
 * index: src/kernels.cu:2087-2091) -------------------------------------
 * libminecu_b200_checked.so is this library compiled with every voxel,
 * shared-memory world, table and observation index checked against its
 * buffer before the access (including the ray march's load one step past
 * the staged world, which must stay within the layer of padding kept around
 * it); a failed check skips the access and is recorded, never trapped, and
 * the step kernels also set the env's error word (mc_env_check_error).
 * mc_build_checks_bounds() is 1 there, 0 in libminecu_b200.so.
 * mc_debug_bounds_report reads and clears the record of one numerics back
 * end: out[0] violations, out[1] first site, out[2] its index, out[3] the
 * limit it broke; MC_ERR_UNSUPPORTED in the normal build.
 * mc_debug_bounds_selftest records one violation at site 0 with no memory
 * access behind it, to show that a violation reaches the record. */
int mc_build_checks_bounds(void);
int mc_debug_bounds_report(int32_t numerics, int32_t* out, void* stream);
int mc_debug_bounds_selftest(int32_t numerics, void* stream);
/* Bytes of dynamic shared memory the fused kernel uses per CTA. */
int64_t mc_env_fused_smem_bytes(const mc_env* env);
/* The launch shape mc_env_create would choose for this configuration on a
 * GPU with num_sms SMs (voxels_aligned: the voxels start on a 16-byte
 * boundary), and the dynamic shared memory it uses per CTA (smem_bytes may
 * be NULL).  Needs no GPU.  No counterpart in the reference, whose launch
 * shapes are fixed per kernel (src/kernels.cu:2457-2494). */
int mc_default_fused_config(const mc_env_config* cfg, int32_t num_sms, int32_t voxels_aligned, mc_fused_config* out,
                            int64_t* smem_bytes);

/* ---- ragged batches: several env handles stepped by one launch ---------
 * No counterpart in the reference, which runs one world size and one
 * resolution per MineEnv (minecu/__init__.py:141-212) and one kernel
 * sequence per step.  A ragged handle borrows up to MC_RAGGED_MAX_GROUPS env
 * handles ("groups": different world sizes, resolutions, parameters; same
 * numerics and the same observation kind) and steps all of them with one
 * persistent fused launch, then regenerates the worlds of each group in
 * which an env was done, exactly as mc_env_step would.  Every group's
 * results are identical to stepping that env handle alone with the fused
 * form.  Actions are concatenated in group order (sum of batch sizes). */
#define MC_RAGGED_MAX_GROUPS 16
typedef struct mc_ragged mc_ragged;
typedef struct mc_ragged_config {
    int32_t warps_per_cta; /* 1..8 warps per CTA */
    int32_t ctas_per_sm;   /* persistent grid = SMs x ctas_per_sm */
    int32_t team_warps;    /* warps per team (1, 2, 4, 8; divides warps_per_cta) */
    int32_t stage[MC_RAGGED_MAX_GROUPS];  /* per group: 1 = bulk-copy each marched world into shared memory */
    int32_t tile_w[MC_RAGGED_MAX_GROUPS]; /* per group: pixel tile tile_w x (32/tile_w), 4/8/16/32 */
    int32_t coop[MC_RAGGED_MAX_GROUPS];   /* per group: 1 = a whole team renders each env; 0 = one warp per env */
} mc_ragged_config;
/* The env handles must outlive the ragged handle; re-pointing one of them
 * (mc_env_set_state) is picked up at the next step. */
int mc_ragged_create(mc_env* const* groups, int32_t ngroups, mc_ragged** out);
int mc_ragged_destroy(mc_ragged* r);
int mc_ragged_set_config(mc_ragged* r, const mc_ragged_config* cfg);
int mc_ragged_get_config(const mc_ragged* r, mc_ragged_config* cfg);
/* Total envs over the groups, and the dynamic shared memory per CTA. */
int64_t mc_ragged_total_envs(const mc_ragged* r);
int64_t mc_ragged_smem_bytes(const mc_ragged* r);
/* One step of every group: buttons int8[total,8] + look float32[total,2]. */
int mc_ragged_step(mc_ragged* r, const int8_t* buttons, const float* look, void* stream);
/* One step of every group: discrete actions uint8[total]. */
int mc_ragged_step_discrete(mc_ragged* r, const uint8_t* actions, void* stream);
/* The discrete step of every group with host buffers, as mc_env_step_host:
 * actions uint8[total] from pinned host memory, every env's reward
 * float32[total] and done uint8[total] (concatenated in group order) to
 * pinned host memory, the copies overlapping the neighbouring steps; the
 * launch writes the results straight into the read-back buffer.  Results
 * are in host memory once a stream given to mc_ragged_host_join reaches
 * that point. */
int mc_ragged_step_host(mc_ragged* r, const uint8_t* host_actions, float* host_rewards, uint8_t* host_dones,
                        void* stream);
int mc_ragged_host_join(mc_ragged* r, void* stream);
/* K steps of actions uint8[K,total] in one CUDA graph (cached per actions, K and config). */
int mc_ragged_rollout(mc_ragged* r, const uint8_t* actions, int32_t K, void* stream);
int mc_ragged_rollout_prepare(mc_ragged* r, const uint8_t* actions, int32_t K);
/* Reads and clears the device error words of the launch and of every group. */
int mc_ragged_check_error(mc_ragged* r, void* stream);

/* ---- env server: many client jobs on one device ----------------------
 * No counterpart in the reference (one Python MineEnv per process, stepped
 * by its owner).  A server owns the device state of many jobs (each job is
 * one env configuration: batch, world, resolution, ...), admitted against
 * an HBM budget, and serves step/reset requests from client threads.  A
 * launcher thread takes the oldest queued request of every job with work
 * and runs them together: resets as MineEnv.reset, steps as one launch of
 * the team kernel over the jobs (groups of up to MC_RAGGED_MAX_GROUPS), with
 * one actions upload and one rewards/dones read-back per launch.  A job's
 * requests run in submission order; each step's results equal
 * mc_env_step_discrete with the fused form on that job alone.  With
 * batching = 0 the server runs one request at a time, in arrival order, with
 * the plain form (the one-job-at-a-time loop the batching is compared to).
 * Latency = request submission to results in host memory. */
#define MC_REQ_STEP 0
#define MC_REQ_RESET 1
typedef struct mc_server mc_server;
typedef struct mc_server_config {
    int64_t hbm_budget_bytes;   /* admission budget for the jobs' device state (mc_server_job_bytes) */
    int32_t numerics;           /* MC_NUMERICS_*, shared by every job */
    int32_t batching;           /* 1: batch one request per job into team launches; 0: one request at a time */
    int32_t max_inflight;       /* launches queued on the device at once, 1..4 */
    int32_t max_envs_per_launch;/* cap on the envs of one step launch (0: 1 << 20) */
} mc_server_config;
typedef struct mc_server_stats {
    int64_t step_requests;      /* completed since create / mc_server_reset_stats */
    int64_t reset_requests;
    int64_t env_steps;
    int64_t launches;           /* step launches */
    double elapsed_s;           /* since create / reset */
    double env_steps_per_s;     /* env_steps / elapsed_s */
    double p50_us, p90_us, p99_us, max_us, mean_us; /* step latency */
    double reset_p50_us, reset_p99_us;
    double mean_jobs_per_launch;
    int32_t jobs;               /* admitted now */
    int64_t bytes_admitted;
} mc_server_stats;
int mc_server_create(const mc_server_config* cfg, mc_server** out);
/* Stops the threads after the requests already queued have run. */
int mc_server_destroy(mc_server* s);
/* Step requests of one job a batching launch may run (1..8, default 1): a
 * launch takes the oldest request of every job with work (round 0), then
 * the next queued request of those jobs (round 1), and so on while the
 * launch's envs stay within max_envs_per_launch; the rounds run one after
 * another (a team launch each), so a burst of one job's requests waits for
 * one launch instead of one launch per request.  No reference counterpart. */
int mc_server_set_rounds(mc_server* s, int32_t rounds);
/* Device bytes one job of this configuration is charged at admission. */
int64_t mc_server_job_bytes(const mc_env_config* cfg);
/* Allocate and generate a job's worlds and spawn its agents (as MineEnv(...)
 * followed by reset()); MC_ERR_BUDGET if it does not fit. */
int mc_server_admit(mc_server* s, const mc_env_config* cfg, int32_t* job);
/* Free a job; MC_ERR_BUSY while it has requests queued or running. */
int mc_server_release(mc_server* s, int32_t job);
/* The job's device state (observations, rewards, ... as MineEnv tensors). */
int mc_server_job_state(mc_server* s, int32_t job, mc_env_state* out);
/* Queue a request: MC_REQ_STEP with host actions uint8[batch] (copied), or
 * MC_REQ_RESET (actions unused).  The ticket is passed to mc_server_wait. */
int mc_server_submit(mc_server* s, int32_t job, int32_t kind, const uint8_t* actions, int64_t* ticket);
/* Wait for a request; rewards float[batch] and dones uint8[batch] (host,
 * optional) receive a step's results.  timeout_us < 0 waits for ever;
 * MC_ERR_TIMEOUT leaves the ticket valid. */
int mc_server_wait(mc_server* s, int64_t ticket, float* rewards, uint8_t* dones, int64_t timeout_us);
int mc_server_get_stats(mc_server* s, mc_server_stats* out);
int mc_server_reset_stats(mc_server* s);
/* Load generator: one client thread per entry, each issuing requests for
 * its job for `seconds` - open loop with Poisson arrivals at rate_hz, or
 * closed loop (the next request when the last one completed) - with a reset
 * every episode_steps steps and uniform discrete actions from Philox
 * (seed, job env, step).  Waits for every issued request, then fills `out`
 * with the latencies of the requests issued in the window and the env-steps
 * completed in it. */
typedef struct mc_load_job {
    int32_t job;
    double rate_hz;             /* open loop: mean requests per second */
    int32_t episode_steps;      /* steps between reset requests (0: none) */
    uint32_t seed;
} mc_load_job;
typedef struct mc_load_config {
    double seconds;
    int32_t closed_loop;
    int32_t njobs;
    const mc_load_job* jobs;
} mc_load_config;
int mc_server_drive(mc_server* s, const mc_load_config* cfg, mc_server_stats* out);

/* ---- stateless kernels: the reference's _C functions ------------------ */
/* generate_world_kernel (src/kernels.cu:1793-1828) via launch_generate_world
 * (src/kernels.cu:2281-2290); the seed is unused, as in the reference. */
int mc_generate_world(int8_t* voxels, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t ground_height,
                      uint32_t seed, void* stream);
/* launch_place_tree (src/kernels.cu:2292-2301) */
int mc_place_tree(int8_t* voxels, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t tree_x, int32_t tree_z,
                  int32_t ground_height, void* stream);
/* launch_place_house (src/kernels.cu:2303-2312) */
int mc_place_house(int8_t* voxels, int32_t B, int32_t wx, int32_t wy, int32_t wz, int32_t house_x,
                   int32_t house_z, int32_t ground_height, void* stream);
/* launch_reset (src/kernels.cu:2268-2279) */
int mc_reset_agents(float* positions, float* velocities, float* yaws, float* pitches, uint8_t* on_ground,
                    const uint8_t* do_reset, int32_t B, float spawn_x, float spawn_y, float spawn_z, void* stream);
/* launch_render / launch_render_uint8 / _minimal / _fp16 / _fast
 * (src/kernels.cu:2078-2160): render every env of `state` from
 * state->cameras with the render family of cfg->obs_mode (shaded for
 * float32/uint8/uint8_fast, flat otherwise). */
int mc_render(const mc_env_config* cfg, const mc_env_state* state, int32_t shaded, void* stream);
/* launch_precompute_camera_basis (src/kernels.cu:2162-2170) */
int mc_precompute_camera_basis(const float* cameras, float* basis, int32_t B, int32_t width, int32_t height,
                               float fov_degrees, int32_t numerics, void* stream);
/* launch_render_uint8_prebasis (src/kernels.cu:2172-2190), non-cubic */
int mc_render_uint8_prebasis(const int8_t* voxels, const float* basis, uint8_t* out, int32_t B, int32_t wx,
                             int32_t wy, int32_t wz, int32_t width, int32_t height, int32_t max_steps,
                             int32_t numerics, void* stream);
/* launch_render_uint8_coalesced (src/kernels.cu:2212-2232): [Y,X,Z,B] voxels */
int mc_render_uint8_coalesced(const int8_t* voxels_yxzb, const float* basis, uint8_t* out, int32_t B,
                              int32_t world_size, int32_t width, int32_t height, int32_t max_steps,
                              int32_t numerics, void* stream);
/* The reference's 8 action-decode buffers (MineEnv.forward_in ...,
 * minecu/__init__.py:242-250), written by decode_actions_kernel. */
typedef struct mc_decode_buffers {
    float* forward_in;
    float* strafe_in;
    float* delta_yaw_in;
    float* delta_pitch_in;
    uint8_t* jump_in;
    uint8_t* do_break;
    uint8_t* do_place;
    float* speed_mult;
} mc_decode_buffers;

/* One step of the reference's _C.step / step_uint8 / _minimal / _fp16 /
 * _fast / _prebasis / _prebasis_full / _smem (launch_step*,
 * src/kernels.cu:2497-3243): kernels only, no world regeneration.  For
 * every mode but prebasis_full, do_reset is an input and step_count is not
 * touched and may be NULL (their episode logic runs in Python,
 * minecu/__init__.py:363-366, 435-436); for prebasis_full the episode check
 * and counter update run in the step.  The plain form writes the decode
 * buffers as the reference does (dec must be non-NULL); the fused form keeps
 * them in registers. */
int mc_step_stateless(const mc_env_config* cfg, const mc_env_state* state, const int8_t* buttons,
                      const float* look, const mc_decode_buffers* dec, int32_t form, void* stream);
/* launch_physics (src/kernels.cu:2234-2250) from the 8 decode inputs */
int mc_physics(float* positions, float* velocities, float* yaws, float* pitches, uint8_t* on_ground,
               const float* forward_in, const float* strafe_in, const float* delta_yaw_in,
               const float* delta_pitch_in, const uint8_t* jump_in, const float* speed_mult, int32_t B,
               int32_t world_size, float dt, float gravity, float walk_speed, float jump_vel, int32_t numerics,
               void* stream);
/* launch_raycast_break (src/kernels.cu:2252-2266) */
int mc_raycast_break(int8_t* voxels, const float* positions, const float* yaws, const float* pitches,
                     const uint8_t* do_break, float* rewards, int32_t B, int32_t world_size, int32_t target_block,
                     float reward_value, int32_t numerics, void* stream);

/* ---- allocation-free step (no counterpart in the reference) -----------
 * For callers that cannot allocate device memory (fixed memory budgets,
 * allocators owned by another runtime): the plain step of
 * mc_step_stateless(..., MC_FORM_PLAIN), with its action-decode scratch and
 * flag words in a static device array inside the library instead of caller
 * buffers or lazy allocations.  At most MC_NOALLOC_MAX_ENVS envs per call
 * (larger batches are rejected with MC_ERR_INVALID); the array (about
 * 1.5 MB) stays on every GPU that loads the library until exit.  The first
 * call on a device looks up the array's address: make it before any stream
 * capture; the address is kept, so cudaDeviceReset while the library is
 * loaded is not supported.  Calls share the array, so calls that overlap on
 * the GPU race. */
#define MC_NOALLOC_MAX_ENVS 65536
int mc_step_plain_noalloc(const mc_env_config* cfg, const mc_env_state* state, const int8_t* buttons,
                          const float* look, void* stream);

/* ---- synthetic action stream (no reference counterpart: the benchmark's
 *      seeded Philox4x32-10 actions, docs/environment.md:5-17 table) ----- */
int mc_philox_actions(uint8_t* actions, int32_t B, int32_t K, int32_t env_offset, int32_t step0, uint64_t seed,
                      int32_t break_half, void* stream);
int mc_discrete_to_buttons(const uint8_t* actions, int32_t B, float look_delta, int8_t* buttons, float* look,
                           void* stream);

/* ---- policy input: a uint8 observation as float32 in [0, 1] -----------
 * The conversion a policy applies to the reference's observations before
 * its first layer (examples/train_wood.py:51-56 permutes NHWC to NCHW), done
 * in one pass: out = obs / 255 (IEEE division, correctly rounded) for every
 * channel value of the uint8 [B,H,W,3] observation, written as float32
 * [B,3,H,W] (MC_POLICY_NCHW) or [B,H,W,3] (MC_POLICY_NHWC).  No counterpart
 * in the reference, whose observations are float32 by default. */
#define MC_POLICY_NCHW 0
#define MC_POLICY_NHWC 1
int mc_obs_to_policy(const uint8_t* obs, float* out, int64_t B, int32_t H, int32_t W, int32_t layout, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MINECU_B200_H */
