/*
 * mc_oracle.h - TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of mine.cu's environment step (reference files
 * src/kernels.cu and minecu/__init__.py), used as the checker for the CUDA
 * product path.  Only the tests, the smoke check and bench.py's CPU
 * baseline leg may load it; the product never does.
 *
 * Numerics: the "ieee" mode of the product (IEEE-754 single precision, no
 * fused multiply-add, correctly rounded / and sqrt, trig from
 * mc_ieee_math.h).  The reference itself is built with --use_fast_math, so
 * this oracle reproduces the reference's algorithm and op order exactly but
 * not the hardware-approximate bits of its sin/cos/tan/sqrt/div; the GPU
 * "ref_fast" mode is compared with the reference's own CUDA build instead.
 */
#ifndef MC_ORACLE_H
#define MC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Render families (one per reference render kernel) */
enum {
    ORC_RENDER_SHADED = 0,   /* render_kernel / render_kernel_uint8 (kernels.cu:87-470) */
    ORC_RENDER_SHADED_FAST,  /* render_kernel_uint8_fast (kernels.cu:1268-1442) */
    ORC_RENDER_MINIMAL,      /* render_kernel_uint8_minimal (kernels.cu:985-1119) */
    ORC_RENDER_FP16,         /* render_kernel_uint8_fp16 (kernels.cu:1127-1260) */
    ORC_RENDER_PREBASIS      /* render_kernel_uint8_prebasis / _smem (kernels.cu:568-700, 835-982) */
};

typedef struct orc_cfg {
    int B, wx, wy, wz;          /* batch, world dims ([B, Y, X, Z] layout) */
    int width, height;          /* render resolution */
    int max_steps;
    float view_distance, fov_degrees;
    float dt, gravity, walk_speed, sprint_mult, jump_vel;
    int ground_height;
    int target_block;
    float reward_value;
    float spawn_x, spawn_y, spawn_z;
    int tree_x, tree_z, house_x, house_z;
    int episode_rule;           /* 0: python rule (done = has_limit && cnt >= L), 1: kernel rule (L > 0 && cnt >= L) */
    int has_limit, episode_length;
    int render;                 /* ORC_RENDER_* used by step() */
    int obs_f32;                /* 1: float32 obs, 0: uint8 obs */
    int regen_per_env;          /* 1: a done or reset env regenerates only its own world (the
                                   build's opt-in MC_REGEN_PER_ENV); 0: every world, the reference's rule */
} orc_cfg;

typedef struct orc_state {
    int8_t* voxels;      /* [B, wy, wx, wz] */
    float* positions;    /* [B, 3] */
    float* velocities;   /* [B, 3] */
    float* yaws;         /* [B] */
    float* pitches;      /* [B] */
    uint8_t* on_ground;  /* [B] */
    int32_t* step_count; /* [B] */
    uint8_t* do_reset;   /* [B] */
    float* cameras;      /* [B, 5] */
    float* basis;        /* [B, 14] or NULL */
    void* obs;           /* [B, H, W, 3] uint8 or float32 */
    float* rewards;      /* [B] */
    int32_t* dbg_interact; /* [B] flat in-env voxel index touched by interact, -1 if none; may be NULL */
    int16_t* dbg_pixel;    /* [B, H, W] (hit_block + 1) | ((hit_face + 1) << 8); may be NULL */
} orc_state;

/* world generation (kernels.cu:1793-1946), all envs */
void orc_generate_world(int8_t* vox, int B, int wx, int wy, int wz, int ground_height);
void orc_place_tree(int8_t* vox, int B, int wx, int wy, int wz, int tree_x, int tree_z, int ground_height);
void orc_place_house(int8_t* vox, int B, int wx, int wy, int wz, int house_x, int house_z, int ground_height);

/* MineEnv.reset(mask) (minecu/__init__.py:270-302); mask may be NULL (= all) */
void orc_env_reset(const orc_cfg* c, orc_state* s, const uint8_t* mask, int threads);
/* MineEnv.step(buttons, look) (minecu/__init__.py:304-444). Returns number of done envs. */
int orc_env_step(const orc_cfg* c, orc_state* s, const int8_t* buttons, const float* look, int threads);
/* MineEnv._render (minecu/__init__.py:446-466): shaded render of the current pose */
void orc_env_render(const orc_cfg* c, orc_state* s, int threads);
/* Stand-alone render of one family from a camera buffer, for kernel-level tests. */
void orc_render(const orc_cfg* c, int family, int obs_f32, const int8_t* vox, const float* cameras,
                void* obs, int16_t* dbg_pixel, int threads);

/* Philox4x32-10 action stream + discrete adapter (shared with the product). */
void orc_philox_actions(uint8_t* actions, int B, int env_offset, int step, uint64_t seed, int break_half);
void orc_discrete_to_buttons(const uint8_t* actions, int B, float look_delta, int8_t* buttons, float* look);

/* IEEE trig exported for tests */
float orc_sinf(float x);
float orc_cosf(float x);
float orc_tanf(float x);

#ifdef __cplusplus
}
#endif
#endif
