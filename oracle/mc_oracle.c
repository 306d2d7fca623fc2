/*
 * mc_oracle.c - TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A scalar CPU restatement of mine.cu's environment step.  Every function
 * cites the reference lines (src/kernels.cu, minecu/__init__.py) whose
 * semantics and op order it follows.  Envs are independent, so OpenMP runs
 * envs in parallel; each env's work is the reference's per-thread code.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp).
 * Numerics: IEEE single precision; trig from mc_ieee_math.h (shared with the
 * product's "ieee" numerics mode so both give the same bits).
 */
#include "mc_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../mine.cu_b200/csrc/mc_ieee_math.h"
#include "../mine.cu_b200/csrc/mc_philox.h"

/* Block ids (kernels.cu:11-24) */
enum { AIR = -1, GRASS = 0, DIRT = 1, STONE = 2, OAKLOG = 3, LEAVES = 4, SAND = 5,
       WATER = 6, GLASS = 7, BRICK = 8, COBBLESTONE = 9, PLANKS = 10, SNOW = 11, BEDROCK = 12 };

/* Float colours (kernels.cu:27-41) and sky (kernels.cu:44). */
static const float BC[13][3] = {
    {0.30f, 0.65f, 0.20f}, {0.55f, 0.35f, 0.20f}, {0.50f, 0.50f, 0.50f}, {0.55f, 0.40f, 0.25f},
    {0.20f, 0.55f, 0.15f}, {0.90f, 0.85f, 0.60f}, {0.20f, 0.40f, 0.80f}, {0.85f, 0.90f, 0.95f},
    {0.70f, 0.35f, 0.30f}, {0.40f, 0.40f, 0.40f}, {0.75f, 0.60f, 0.40f}, {0.95f, 0.95f, 0.98f},
    {0.15f, 0.15f, 0.15f}};
static const float SKY[3] = {0.53f, 0.81f, 0.92f};
/* Pre-rounded uint8 colours used by the flat render kernels (kernels.cu:479-495). */
static const uint8_t BC8[13][3] = {
    {76, 166, 51}, {140, 89, 51}, {127, 127, 127}, {140, 102, 64}, {51, 140, 38},
    {229, 217, 153}, {51, 102, 204}, {217, 229, 242}, {178, 89, 76}, {102, 102, 102},
    {191, 153, 102}, {242, 242, 250}, {38, 38, 38}};
static const uint8_t SKY8[3] = {135, 206, 235};

float orc_sinf(float x) { return mc_ieee_sinf(x); }
float orc_cosf(float x) { return mc_ieee_cosf(x); }
float orc_tanf(float x) { return mc_ieee_tanf(x); }
/* The Philox4x32-10 block function of the action stream, for known-answer tests. */
void orc_philox4x32_10(uint32_t* ctr, uint32_t k0, uint32_t k1) { mc_philox4x32_10(ctr, k0, k1); }

static void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

/* ------------------------------------------------------------------ */
/* World generation                                                    */
/* ------------------------------------------------------------------ */

/* generate_world_kernel (kernels.cu:1793-1828); the seed is unused there. */
void orc_generate_world(int8_t* vox, int B, int wx, int wy, int wz, int gh) {
    long long wxyz = (long long)wx * wy * wz;
    for (long long b = 0; b < B; ++b) {
        int8_t* w = vox + b * wxyz;
        for (int y = 0; y < wy; ++y) {
            int8_t blk = AIR;
            if (y == 0) blk = BEDROCK;
            else if (y < gh - 1) blk = DIRT;
            else if (y == gh - 1) blk = GRASS;
            memset(w + (long long)y * wx * wz, blk, (size_t)wx * wz);
        }
    }
}

/* place_tree_kernel (kernels.cu:1831-1865): 3 OAKLOG at y = gh..gh+2 and
 * LEAVES at gh+3, clipped only in y. */
void orc_place_tree(int8_t* vox, int B, int wx, int wy, int wz, int tx, int tz, int gh) {
    long long wxyz = (long long)wx * wy * wz;
    long long wxz = (long long)wx * wz;
    for (long long b = 0; b < B; ++b) {
        for (int dy = 0; dy < 3; ++dy) {
            int y = gh + dy;
            if (y < wy) vox[b * wxyz + y * wxz + (long long)tx * wz + tz] = OAKLOG;
        }
        int ly = gh + 3;
        if (ly < wy) vox[b * wxyz + ly * wxz + (long long)tx * wz + tz] = LEAVES;
    }
}

/* place_house_kernel (kernels.cu:1868-1946): 5 (X) x 4 (Z) x 4 (Y) house,
 * cobblestone floor, plank walls with a 1x2 door at dx=2 on the z=0 wall,
 * oak-log corner pillars, brick roof; every voxel clipped to the world. */
static void house_set(int8_t* w, int wx, int wy, int wz, int hx, int hz, int gh,
                      int dy, int dx, int dz, int8_t blk) {
    int vx = hx + dx, vy = gh + dy, vz = hz + dz;
    if (vx >= 0 && vx < wx && vy >= 0 && vy < wy && vz >= 0 && vz < wz)
        w[(long long)vy * wx * wz + (long long)vx * wz + vz] = blk;
}

void orc_place_house(int8_t* vox, int B, int wx, int wy, int wz, int hx, int hz, int gh) {
    const int W = 5, D = 4, H = 4;
    long long wxyz = (long long)wx * wy * wz;
    for (long long b = 0; b < B; ++b) {
        int8_t* w = vox + b * wxyz;
        for (int dx = 0; dx < W; ++dx)
            for (int dz = 0; dz < D; ++dz) house_set(w, wx, wy, wz, hx, hz, gh, 0, dx, dz, COBBLESTONE);
        for (int dy = 1; dy <= 3; ++dy) {
            for (int dx = 0; dx < W; ++dx) {
                if (dx == 2 && dy <= 2) continue;
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
}

/* MineEnv._generate_world (minecu/__init__.py:258-268) */
static void regen_all(const orc_cfg* c, orc_state* s) {
    orc_generate_world(s->voxels, c->B, c->wx, c->wy, c->wz, c->ground_height);
    orc_place_tree(s->voxels, c->B, c->wx, c->wy, c->wz, c->tree_x, c->tree_z, c->ground_height);
    orc_place_house(s->voxels, c->B, c->wx, c->wy, c->wz, c->house_x, c->house_z, c->ground_height);
}

/* The per-env rule (regen_per_env): the same three generators on the world
 * of each env whose do_reset is set, the others untouched. */
static void regen_flagged(const orc_cfg* c, orc_state* s) {
    const long long wxyz = (long long)c->wx * c->wy * c->wz;
    for (long long i = 0; i < c->B; ++i) {
        if (!s->do_reset[i]) continue;
        int8_t* w = s->voxels + i * wxyz;
        orc_generate_world(w, 1, c->wx, c->wy, c->wz, c->ground_height);
        orc_place_tree(w, 1, c->wx, c->wy, c->wz, c->tree_x, c->tree_z, c->ground_height);
        orc_place_house(w, 1, c->wx, c->wy, c->wz, c->house_x, c->house_z, c->ground_height);
    }
}

/* ------------------------------------------------------------------ */
/* Render                                                              */
/* ------------------------------------------------------------------ */

typedef struct {
    float eye_x, eye_y, eye_z;
    float fx, fy, fz, rx, rz, ux, uy, uz;
} cam_basis;

/* Per-pixel camera basis of the shaded/minimal/fp16 kernels
 * (kernels.cu:113-136, 323-341, 1017-1032, 1158-1172). */
static void basis_trig(const float* cam, cam_basis* k) {
    float yaw = cam[3], pitch = cam[4];
    k->eye_x = cam[0];
    k->eye_y = cam[1] + 1.6f;
    k->eye_z = cam[2];
    float cy = mc_ieee_cosf(yaw), sy = mc_ieee_sinf(yaw);
    float cp = mc_ieee_cosf(pitch), sp = mc_ieee_sinf(pitch);
    k->fx = sy * cp; k->fy = sp; k->fz = cy * cp;
    k->rx = cy; k->rz = -sy;
    k->ux = -sy * sp; k->uy = cp; k->uz = -cy * sp;
}

/* precompute_camera_basis_kernel (kernels.cu:511-561) */
static void basis_pre(const float* cam, int width, int height, float fov, float* out14) {
    float sy, cy, sp, cp;
    mc_ieee_sincosf(cam[3], &sy, &cy);
    mc_ieee_sincosf(cam[4], &sp, &cp);
    float fov_rad = fov * 0.01745329f;
    float half_fov = mc_ieee_tanf(fov_rad * 0.5f);
    float aspect = (float)width / (float)height;
    out14[0] = cam[0];
    out14[1] = cam[1] + 1.6f;
    out14[2] = cam[2];
    out14[3] = sy * cp;
    out14[4] = sp;
    out14[5] = cy * cp;
    out14[6] = cy;
    out14[7] = -sy;
    out14[8] = -sy * sp;
    out14[9] = cp;
    out14[10] = -cy * sp;
    out14[11] = half_fov * aspect;
    out14[12] = half_fov;
    out14[13] = 0.0f; /* padding; the reference never writes it */
}

static int16_t dbg_code(int blk, int face) { return (int16_t)((blk + 1) | ((face + 1) << 8)); }

/* ray_intersects_aabb (kernels.cu:51-79) against [0,wx]x[0,wy]x[0,wz]
 * (the reference's [0, ws]^3 for a cubic world) */
static int aabb(float ox, float oy, float oz, float dx, float dy, float dz, float fwx, float fwy, float fwz,
                float* t_entry, float* t_exit) {
    float idx = (dx != 0.0f) ? 1.0f / dx : 1e30f;
    float idy = (dy != 0.0f) ? 1.0f / dy : 1e30f;
    float idz = (dz != 0.0f) ? 1.0f / dz : 1e30f;
    float t1 = (0.0f - ox) * idx, t2 = (fwx - ox) * idx;
    float t3 = (0.0f - oy) * idy, t4 = (fwy - oy) * idy;
    float t5 = (0.0f - oz) * idz, t6 = (fwz - oz) * idz;
    float tmin = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
    float tmax = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
    *t_entry = tmin;
    *t_exit = tmax;
    if (tmax < 0 || tmin > tmax) return 0;
    return 1;
}

static void put_rgb(void* obs, int obs_f32, long long pix, const float rgb[3]) {
    if (obs_f32) {
        float* o = (float*)obs + pix * 3;
        o[0] = rgb[0]; o[1] = rgb[1]; o[2] = rgb[2];
    } else {
        uint8_t* o = (uint8_t*)obs + pix * 3;
        o[0] = (uint8_t)(rgb[0] * 255.0f);
        o[1] = (uint8_t)(rgb[1] * 255.0f);
        o[2] = (uint8_t)(rgb[2] * 255.0f);
    }
}

static void put_rgb8(void* obs, long long pix, const uint8_t rgb[3]) {
    uint8_t* o = (uint8_t*)obs + pix * 3;
    o[0] = rgb[0]; o[1] = rgb[1]; o[2] = rgb[2];
}

/* render_kernel (kernels.cu:87-293), render_kernel_uint8 (kernels.cu:300-470)
 * and, with fast_ground, render_kernel_uint8_fast (kernels.cu:1268-1442).
 * One pixel.  The reference's cubic world of size ws is generalised to
 * wx x wy x wz; a cubic world gives the reference's arithmetic. */
static void shade_pixel(const cam_basis* k, const int8_t* w, int wx, int wy, int wz, int width, int height,
                        int px, int py, int max_steps, float vd, float fov, int fast_ground, int gh,
                        void* obs, int obs_f32, long long pix, int16_t* dbg) {
    float fov_rad = fov * 3.14159265f / 180.0f;
    float aspect = (float)width / (float)height;
    float half_fov = mc_ieee_tanf(fov_rad * 0.5f);
    float u = (2.0f * ((float)px + 0.5f) / (float)width - 1.0f) * half_fov * aspect;
    float v = (1.0f - 2.0f * ((float)py + 0.5f) / (float)height) * half_fov;
    float ray_x = k->fx + u * k->rx + v * k->ux;
    float ray_y = k->fy + v * k->uy;
    float ray_z = k->fz + u * k->rz + v * k->uz;
    float ray_len = sqrtf(ray_x * ray_x + ray_y * ray_y + ray_z * ray_z);
    ray_x = ray_x / ray_len;
    ray_y = ray_y / ray_len;
    ray_z = ray_z / ray_len;

    float t_entry, t_exit;
    int hits = aabb(k->eye_x, k->eye_y, k->eye_z, ray_x, ray_y, ray_z, (float)wx, (float)wy, (float)wz,
                    &t_entry, &t_exit);
    if (!hits || t_entry > vd) {
        put_rgb(obs, obs_f32, pix, SKY);
        if (dbg) dbg[pix] = dbg_code(AIR, -1);
        return;
    }
    long long wxz = (long long)wx * wz;
    int vx = (int)floorf(k->eye_x), vy = (int)floorf(k->eye_y), vz = (int)floorf(k->eye_z);
    int sx = (ray_x >= 0) ? 1 : -1, sy = (ray_y >= 0) ? 1 : -1, sz = (ray_z >= 0) ? 1 : -1;
    float ix = (ray_x != 0.0f) ? 1.0f / ray_x : 1e30f;
    float iy = (ray_y != 0.0f) ? 1.0f / ray_y : 1e30f;
    float iz = (ray_z != 0.0f) ? 1.0f / ray_z : 1e30f;
    float tdx = fabsf(ix), tdy = fabsf(iy), tdz = fabsf(iz);
    float tmx = (ray_x >= 0) ? ((float)(vx + 1) - k->eye_x) * ix : ((float)vx - k->eye_x) * ix;
    float tmy = (ray_y >= 0) ? ((float)(vy + 1) - k->eye_y) * iy : ((float)vy - k->eye_y) * iy;
    float tmz = (ray_z >= 0) ? ((float)(vz + 1) - k->eye_z) * iz : ((float)vz - k->eye_z) * iz;
    float t = 0.0f;
    int face = -1;
    int blk = AIR;
    /* the reference unrolls this loop 4x with `step >= max_steps` checks,
     * which visits exactly max_steps voxels (kernels.cu:220-269) */
    for (int step = 0; step < max_steps; ++step) {
        if (t >= vd) break;
        if (fast_ground && vy < gh) { blk = (vy == gh - 1) ? GRASS : DIRT; break; }
        if (vx >= 0 && vx < wx && vy >= 0 && vy < wy && vz >= 0 && vz < wz) {
            int8_t b = w[vy * wxz + (long long)vx * wz + vz];
            if (b >= 0) { blk = b; break; }
        } else if (t > t_exit) {
            break;
        }
        if (tmx < tmy && tmx < tmz) { t = tmx; tmx += tdx; vx += sx; face = 0; }
        else if (tmy < tmz) { t = tmy; tmy += tdy; vy += sy; face = 1; }
        else { t = tmz; tmz += tdz; vz += sz; face = 2; }
    }
    if (dbg) dbg[pix] = dbg_code(blk, face);
    if (blk >= 0) {
        float shade = 1.0f;
        if (face == 0) shade = 0.8f;
        else if (face == 2) shade = 0.9f;
        else if (face == 1 && sy < 0) shade = 0.6f;
        float fog = fminf(t / vd, 1.0f);
        fog = fog * fog;
        float rgb[3];
        for (int ch = 0; ch < 3; ++ch) rgb[ch] = BC[blk][ch] * shade * (1.0f - fog) + SKY[ch] * fog;
        put_rgb(obs, obs_f32, pix, rgb);
    } else {
        put_rgb(obs, obs_f32, pix, SKY);
    }
}

/* IEEE binary16 helpers for render_kernel_uint8_fp16. */
static uint16_t half_from_double(double x) {
    /* round-to-nearest-even conversion of a double to binary16 */
    uint16_t sign = 0;
    if (x != x) return 0x7e00;
    if (x < 0 || (x == 0 && 1.0 / x < 0)) { sign = 0x8000; x = -x; }
    if (x >= 65520.0) return sign | 0x7c00;
    if (x < 5.9604644775390625e-08 * 0.5) { /* below half the smallest subnormal (or exactly half: ties to even 0) */
        return sign;
    }
    int e;
    double m = frexp(x, &e); /* x = m * 2^e, m in [0.5, 1) */
    int exp = e - 1;         /* x = (2m) * 2^exp */
    if (exp < -14) {
        /* subnormal: value = n * 2^-24 */
        double n = x / 5.9604644775390625e-08;
        double fl = floor(n);
        double diff = n - fl;
        long long ni = (long long)fl;
        if (diff > 0.5 || (diff == 0.5 && (ni & 1))) ni++;
        return sign | (uint16_t)ni; /* ni may reach 1024 = smallest normal, encoded correctly */
    }
    double frac = (2.0 * m - 1.0) * 1024.0; /* 10-bit mantissa */
    double fl = floor(frac);
    double diff = frac - fl;
    long long mi = (long long)fl;
    if (diff > 0.5 || (diff == 0.5 && (mi & 1))) mi++;
    int be = exp + 15;
    if (mi == 1024) { mi = 0; be++; }
    if (be >= 31) return sign | 0x7c00;
    return sign | (uint16_t)(be << 10) | (uint16_t)mi;
}

static double half_to_double(uint16_t h) {
    int s = h >> 15, e = (h >> 10) & 31, m = h & 1023;
    double v;
    if (e == 0) v = ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexp(1.0 + m / 1024.0, e - 15);
    return s ? -v : v;
}

static uint16_t hadd(uint16_t a, uint16_t b) { return half_from_double(half_to_double(a) + half_to_double(b)); }
static int hlt(uint16_t a, uint16_t b) { return half_to_double(a) < half_to_double(b); }

/* render_kernel_uint8_minimal (kernels.cu:985-1119), render_kernel_uint8_fp16
 * (kernels.cu:1127-1260) and render_kernel_uint8_prebasis/_smem
 * (kernels.cu:568-700, 835-982): flat colours, no AABB or fog. */
static void flat_pixel(int family, const float* bas, const cam_basis* k, const int8_t* w,
                       int wx, int wy, int wz, int width, int height, int px, int py, int max_steps,
                       float fov, uint8_t* obs, long long pix, int16_t* dbg) {
    float eye_x, eye_y, eye_z, fx, fy, fz, rx, rz, ux, uy, uz, u, v;
    if (family == ORC_RENDER_PREBASIS) {
        eye_x = bas[0]; eye_y = bas[1]; eye_z = bas[2];
        fx = bas[3]; fy = bas[4]; fz = bas[5]; rx = bas[6]; rz = bas[7];
        ux = bas[8]; uy = bas[9]; uz = bas[10];
        u = (2.0f * ((float)px + 0.5f) / (float)width - 1.0f) * bas[11];
        v = (1.0f - 2.0f * ((float)py + 0.5f) / (float)height) * bas[12];
    } else {
        eye_x = k->eye_x; eye_y = k->eye_y; eye_z = k->eye_z;
        fx = k->fx; fy = k->fy; fz = k->fz; rx = k->rx; rz = k->rz;
        ux = k->ux; uy = k->uy; uz = k->uz;
        float fov_rad = fov * 0.01745329f;
        float aspect = (float)width / (float)height;
        float half_fov = mc_ieee_tanf(fov_rad * 0.5f);
        u = (2.0f * ((float)px + 0.5f) / (float)width - 1.0f) * half_fov * aspect;
        v = (1.0f - 2.0f * ((float)py + 0.5f) / (float)height) * half_fov;
    }
    float ray_x = fx + u * rx + v * ux;
    float ray_y = fy + v * uy;
    float ray_z = fz + u * rz + v * uz;
    /* rsqrtf in the reference; "ieee" numerics define it as 1/sqrt */
    float ray_len = 1.0f / sqrtf(ray_x * ray_x + ray_y * ray_y + ray_z * ray_z);
    ray_x = ray_x * ray_len;
    ray_y = ray_y * ray_len;
    ray_z = ray_z * ray_len;
    long long wxz = (long long)wx * wz;
    int vx = (int)floorf(eye_x), vy = (int)floorf(eye_y), vz = (int)floorf(eye_z);
    int sx = (ray_x >= 0) ? 1 : -1, sy = (ray_y >= 0) ? 1 : -1, sz = (ray_z >= 0) ? 1 : -1;
    int blk = AIR;
    int face = -1;
    if (family == ORC_RENDER_FP16) {
        float ixf = (ray_x != 0.0f) ? 1.0f / ray_x : 65504.0f;
        float iyf = (ray_y != 0.0f) ? 1.0f / ray_y : 65504.0f;
        float izf = (ray_z != 0.0f) ? 1.0f / ray_z : 65504.0f;
        uint16_t tdx = half_from_double(fabsf(ixf)), tdy = half_from_double(fabsf(iyf)), tdz = half_from_double(fabsf(izf));
        uint16_t tmx = half_from_double((ray_x >= 0) ? ((float)(vx + 1) - eye_x) * ixf : ((float)vx - eye_x) * ixf);
        uint16_t tmy = half_from_double((ray_y >= 0) ? ((float)(vy + 1) - eye_y) * iyf : ((float)vy - eye_y) * iyf);
        uint16_t tmz = half_from_double((ray_z >= 0) ? ((float)(vz + 1) - eye_z) * izf : ((float)vz - eye_z) * izf);
        for (int step = 0; step < max_steps; ++step) {
            if ((unsigned)vx < (unsigned)wx && (unsigned)vy < (unsigned)wy && (unsigned)vz < (unsigned)wz) {
                int8_t b = w[vy * wxz + (long long)vx * wz + vz];
                if (b >= 0) { blk = b; break; }
            }
            if (hlt(tmx, tmy) && hlt(tmx, tmz)) { tmx = hadd(tmx, tdx); vx += sx; face = 0; }
            else if (hlt(tmy, tmz)) { tmy = hadd(tmy, tdy); vy += sy; face = 1; }
            else { tmz = hadd(tmz, tdz); vz += sz; face = 2; }
        }
    } else {
        float ix = (ray_x != 0.0f) ? 1.0f / ray_x : 1e30f;
        float iy = (ray_y != 0.0f) ? 1.0f / ray_y : 1e30f;
        float iz = (ray_z != 0.0f) ? 1.0f / ray_z : 1e30f;
        float tdx = fabsf(ix), tdy = fabsf(iy), tdz = fabsf(iz);
        float tmx = (ray_x >= 0) ? ((float)(vx + 1) - eye_x) * ix : ((float)vx - eye_x) * ix;
        float tmy = (ray_y >= 0) ? ((float)(vy + 1) - eye_y) * iy : ((float)vy - eye_y) * iy;
        float tmz = (ray_z >= 0) ? ((float)(vz + 1) - eye_z) * iz : ((float)vz - eye_z) * iz;
        for (int step = 0; step < max_steps; ++step) {
            if ((unsigned)vx < (unsigned)wx && (unsigned)vy < (unsigned)wy && (unsigned)vz < (unsigned)wz) {
                int8_t b = w[vy * wxz + (long long)vx * wz + vz];
                if (b >= 0) { blk = b; break; }
            }
            if (tmx < tmy && tmx < tmz) { tmx += tdx; vx += sx; face = 0; }
            else if (tmy < tmz) { tmy += tdy; vy += sy; face = 1; }
            else { tmz += tdz; vz += sz; face = 2; }
        }
    }
    if (dbg) dbg[pix] = dbg_code(blk, face);
    if (blk >= 0) put_rgb8(obs, pix, BC8[blk]);
    else put_rgb8(obs, pix, SKY8);
}

static void render_env(const orc_cfg* c, int family, int obs_f32, const int8_t* vox_all,
                       const float* cameras, const float* basis_in, long long b, void* obs, int16_t* dbg) {
    long long wxyz = (long long)c->wx * c->wy * c->wz;
    const int8_t* w = vox_all + b * wxyz;
    const float* cam = cameras + b * 5;
    cam_basis k;
    basis_trig(cam, &k);
    float bas[14];
    if (family == ORC_RENDER_PREBASIS) {
        if (basis_in) memcpy(bas, basis_in + b * 14, sizeof(bas));
        else basis_pre(cam, c->width, c->height, c->fov_degrees, bas);
    }
    long long hw = (long long)c->width * c->height;
    for (int py = 0; py < c->height; ++py) {
        for (int px = 0; px < c->width; ++px) {
            long long pix = b * hw + (long long)py * c->width + px;
            if (family == ORC_RENDER_SHADED || family == ORC_RENDER_SHADED_FAST) {
                shade_pixel(&k, w, c->wx, c->wy, c->wz, c->width, c->height, px, py, c->max_steps, c->view_distance,
                            c->fov_degrees, family == ORC_RENDER_SHADED_FAST, c->ground_height,
                            obs, obs_f32, pix, dbg);
            } else {
                flat_pixel(family, bas, &k, w, c->wx, c->wy, c->wz, c->width, c->height, px, py,
                           c->max_steps, c->fov_degrees, (uint8_t*)obs, pix, dbg);
            }
        }
    }
}

void orc_render(const orc_cfg* c, int family, int obs_f32, const int8_t* vox, const float* cameras,
                void* obs, int16_t* dbg_pixel, int threads) {
    set_threads(threads);
    long long b;
#pragma omp parallel for schedule(dynamic, 16)
    for (b = 0; b < c->B; ++b) render_env(c, family, obs_f32, vox, cameras, NULL, b, obs, dbg_pixel);
}

/* ------------------------------------------------------------------ */
/* Agent step                                                          */
/* ------------------------------------------------------------------ */

/* decode_actions_kernel (kernels.cu:1459-1504) + physics_kernel
 * (kernels.cu:1511-1584) for one env. */
static void physics_env(const orc_cfg* c, orc_state* s, long long i, const int8_t* btn, const float* look) {
    int8_t fwd = btn[0], back = btn[1], left = btn[2], right = btn[3];
    int8_t jump = btn[4], sprint = btn[7];
    float forward_in = (float)fwd - (float)back;
    float strafe_in = (float)right - (float)left;
    float dyaw = look[0], dpitch = look[1];
    int jump_in = (jump != 0);
    float speed_mult = (fwd && sprint) ? c->sprint_mult : 1.0f;

    s->yaws[i] = s->yaws[i] + dyaw;
    float new_pitch = s->pitches[i] + dpitch;
    s->pitches[i] = fminf(fmaxf(new_pitch, -1.56f), 1.56f);
    float cos_yaw = mc_ieee_cosf(s->yaws[i]);
    float sin_yaw = mc_ieee_sinf(s->yaws[i]);
    float speed = c->walk_speed * speed_mult;
    float move_x = sin_yaw * forward_in * speed * c->dt + cos_yaw * strafe_in * c->walk_speed * c->dt;
    float move_z = cos_yaw * forward_in * speed * c->dt - sin_yaw * strafe_in * c->walk_speed * c->dt;
    float vel_y = s->velocities[i * 3 + 1];
    if (jump_in && s->on_ground[i]) vel_y = c->jump_vel;
    vel_y = vel_y + c->gravity * c->dt;
    float new_x = s->positions[i * 3 + 0] + move_x;
    float new_y = s->positions[i * 3 + 1] + vel_y * c->dt;
    float new_z = s->positions[i * 3 + 2] + move_z;
    float ground_y = (float)(c->wy / 4);
    if (new_y <= ground_y) {
        new_y = ground_y;
        vel_y = 0.0f;
        s->on_ground[i] = 1;
    } else {
        s->on_ground[i] = 0;
    }
    float margin = 1.0f;
    new_x = fminf(fmaxf(new_x, margin), (float)c->wx - margin);
    new_z = fminf(fmaxf(new_z, margin), (float)c->wz - margin);
    s->positions[i * 3 + 0] = new_x;
    s->positions[i * 3 + 1] = new_y;
    s->positions[i * 3 + 2] = new_z;
    s->velocities[i * 3 + 1] = vel_y;
}

/* raycast_interact_kernel (kernels.cu:1591-1680): 32 point samples at
 * t = 0.1 + k * 4/32 from the eye; the first in-bounds solid sample is
 * broken (reward if it is the target) or, failing a break request, DIRT is
 * placed at the last in-bounds air sample before it. */
static void interact_env(const orc_cfg* c, orc_state* s, long long i, const int8_t* btn) {
    s->rewards[i] = 0.0f;
    if (s->dbg_interact) s->dbg_interact[i] = -1;
    int wants_break = (btn[5] != 0), wants_place = (btn[6] != 0);
    if (!wants_break && !wants_place) return;
    float yaw = s->yaws[i], pitch = s->pitches[i];
    float cos_yaw = mc_ieee_cosf(yaw), sin_yaw = mc_ieee_sinf(yaw);
    float cos_pitch = mc_ieee_cosf(pitch), sin_pitch = mc_ieee_sinf(pitch);
    float dir_x = sin_yaw * cos_pitch, dir_y = sin_pitch, dir_z = cos_yaw * cos_pitch;
    float eye_x = s->positions[i * 3 + 0];
    float eye_y = s->positions[i * 3 + 1] + 1.6f;
    float eye_z = s->positions[i * 3 + 2];
    float reach = 4.0f;
    int wx = c->wx, wy = c->wy, wz = c->wz;
    long long wxz = (long long)wx * wz, wxyz = (long long)wx * wy * wz;
    int8_t* w = s->voxels + i * wxyz;
    int pvx = -1, pvy = -1, pvz = -1;
    for (int step = 0; step < 32; ++step) {
        float t = 0.1f + (float)step * (reach / 32.0f);
        float px = eye_x + dir_x * t;
        float py = eye_y + dir_y * t;
        float pz = eye_z + dir_z * t;
        int vx = (int)floorf(px), vy = (int)floorf(py), vz = (int)floorf(pz);
        if (vx >= 0 && vx < wx && vy >= 0 && vy < wy && vz >= 0 && vz < wz) {
            long long idx = vy * wxz + (long long)vx * wz + vz;
            int8_t blk = w[idx];
            if (blk >= 0) {
                if (wants_break) {
                    if ((int8_t)c->target_block < 0 || blk == (int8_t)c->target_block) s->rewards[i] = c->reward_value;
                    w[idx] = AIR;
                    if (s->dbg_interact) s->dbg_interact[i] = (int32_t)idx;
                } else if (wants_place && pvx >= 0) {
                    long long pidx = pvy * wxz + (long long)pvx * wz + pvz;
                    w[pidx] = DIRT;
                    if (s->dbg_interact) s->dbg_interact[i] = (int32_t)pidx;
                }
                return;
            }
            pvx = vx; pvy = vy; pvz = vz;
        }
    }
}

/* reset_kernel (kernels.cu:1760-1786) */
static void reset_agent(const orc_cfg* c, orc_state* s, long long i) {
    s->positions[i * 3 + 0] = c->spawn_x;
    s->positions[i * 3 + 1] = c->spawn_y;
    s->positions[i * 3 + 2] = c->spawn_z;
    s->velocities[i * 3 + 0] = 0.0f;
    s->velocities[i * 3 + 1] = 0.0f;
    s->velocities[i * 3 + 2] = 0.0f;
    s->yaws[i] = 0.0f;
    s->pitches[i] = 0.0f;
    s->on_ground[i] = 0;
}

/* update_cameras_kernel (kernels.cu:2320-2335) */
static void update_camera(orc_state* s, long long i) {
    s->cameras[i * 5 + 0] = s->positions[i * 3 + 0];
    s->cameras[i * 5 + 1] = s->positions[i * 3 + 1];
    s->cameras[i * 5 + 2] = s->positions[i * 3 + 2];
    s->cameras[i * 5 + 3] = s->yaws[i];
    s->cameras[i * 5 + 4] = s->pitches[i];
}

/* MineEnv.step (minecu/__init__.py:304-444), kernel order of
 * launch_step*_kernels (kernels.cu:2457-2494, 2909-2991):
 * episode check -> decode -> physics -> interact -> reset -> counter ->
 * cameras -> (basis) -> render; then, if any env is done, every world is
 * regenerated (minecu/__init__.py:356-359, 439-442). */
int orc_env_step(const orc_cfg* c, orc_state* s, const int8_t* buttons, const float* look, int threads) {
    set_threads(threads);
    int any_done = 0;
    long long i;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : any_done)
    for (i = 0; i < c->B; ++i) {
        int done;
        if (c->episode_rule == 0) done = c->has_limit && s->step_count[i] >= c->episode_length;
        else done = (c->episode_length > 0) && s->step_count[i] >= c->episode_length;
        s->do_reset[i] = (uint8_t)done;
        physics_env(c, s, i, buttons + i * 8, look + i * 2);
        interact_env(c, s, i, buttons + i * 8);
        if (done) reset_agent(c, s, i);
        s->step_count[i] = done ? 1 : s->step_count[i] + 1;
        update_camera(s, i);
        if (c->render == ORC_RENDER_PREBASIS && s->basis)
            basis_pre(s->cameras + i * 5, c->width, c->height, c->fov_degrees, s->basis + i * 14);
        render_env(c, c->render, c->obs_f32, s->voxels, s->cameras, s->basis, i, s->obs, s->dbg_pixel);
        any_done |= done;
    }
    int n_done = 0;
    for (i = 0; i < c->B; ++i) n_done += s->do_reset[i];
    if (c->regen_per_env) regen_flagged(c, s);
    else if (any_done) regen_all(c, s);
    return n_done;
}

/* MineEnv._render (minecu/__init__.py:446-466): cameras from the pose, then
 * the shaded kernel (float32 obs, or uint8 for every uint8 mode). */
void orc_env_render(const orc_cfg* c, orc_state* s, int threads) {
    set_threads(threads);
    long long i;
    for (i = 0; i < c->B; ++i) update_camera(s, i);
#pragma omp parallel for schedule(dynamic, 16)
    for (i = 0; i < c->B; ++i)
        render_env(c, ORC_RENDER_SHADED, c->obs_f32, s->voxels, s->cameras, NULL, i, s->obs, s->dbg_pixel);
}

/* MineEnv.reset(mask) (minecu/__init__.py:270-302) */
void orc_env_reset(const orc_cfg* c, orc_state* s, const uint8_t* mask, int threads) {
    int any = 0;
    for (long long i = 0; i < c->B; ++i) {
        s->do_reset[i] = mask ? (mask[i] != 0) : 1;
        any |= s->do_reset[i];
    }
    for (long long i = 0; i < c->B; ++i) {
        if (s->do_reset[i]) {
            reset_agent(c, s, i);
            s->step_count[i] = 0;
        }
    }
    if (c->regen_per_env) regen_flagged(c, s);
    else if (mask == NULL || any) regen_all(c, s);
    orc_env_render(c, s, threads);
}

/* ------------------------------------------------------------------ */
/* Actions                                                             */
/* ------------------------------------------------------------------ */

void orc_philox_actions(uint8_t* actions, int B, int env_offset, int step, uint64_t seed, int break_half) {
    for (int i = 0; i < B; ++i)
        actions[i] = mc_action_draw(seed, (uint32_t)(env_offset + i), (uint32_t)step, break_half);
}

void orc_discrete_to_buttons(const uint8_t* actions, int B, float look_delta, int8_t* buttons, float* look) {
    for (int i = 0; i < B; ++i) mc_discrete_to_buttons(actions[i], look_delta, buttons + i * 8, look + i * 2);
}
