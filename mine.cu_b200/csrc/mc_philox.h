/*
 * mc_philox.h - seeded action stream shared by the CUDA path and the CPU
 * checker, so that both step the same synthetic workload.
 *
 * Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11): a counter-based
 * generator, so action (env, step) is a pure function of the seed and needs
 * no generator state.  Counter = (global env index, step, 0, 0), key =
 * (seed low 32 bits, seed high 32 bits).
 *
 * Discrete actions follow the 11-action table of the reference's
 * docs/environment.md:5-17 (0 no-op, 1 forward, 2 back, 3 strafe left,
 * 4 strafe right, 5 jump, 6 break, 7 look left, 8 look right, 9 look up,
 * 10 look down).  An action is floor(x0 * 11 / 2^32).  With break_half set,
 * the top bit of x1 forces action 6 (break) on about half of the draws.
 */
#ifndef MC_PHILOX_H
#define MC_PHILOX_H
#include <stdint.h>

#ifdef __CUDACC__
#define MC_PHX_HD static __host__ __device__ __forceinline__
#else
#define MC_PHX_HD static inline
#endif

#define MC_ACTION_DIM 11

MC_PHX_HD void mc_philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * ctr[0];
        uint64_t p1 = (uint64_t)M1 * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += W0; k1 += W1;
    }
}

MC_PHX_HD uint8_t mc_action_draw(uint64_t seed, uint32_t env, uint32_t step, int break_half) {
    uint32_t c[4] = {env, step, 0u, 0u};
    mc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    if (break_half && (c[1] >> 31)) return 6;
    return (uint8_t)(((uint64_t)c[0] * MC_ACTION_DIM) >> 32);
}

/* Discrete action -> 8 multi-hot buttons + 2 look deltas (radians).
 * Unknown actions (>= 11) are no-ops. */
MC_PHX_HD void mc_discrete_to_buttons(uint8_t a, float look_delta, int8_t btn[8], float look[2]) {
    for (int i = 0; i < 8; ++i) btn[i] = 0;
    look[0] = 0.0f; look[1] = 0.0f;
    switch (a) {
        case 1: btn[0] = 1; break;            /* forward */
        case 2: btn[1] = 1; break;            /* backward */
        case 3: btn[2] = 1; break;            /* strafe left */
        case 4: btn[3] = 1; break;            /* strafe right */
        case 5: btn[4] = 1; break;            /* jump */
        case 6: btn[5] = 1; break;            /* break */
        case 7: look[0] = look_delta; break;  /* look left  (+yaw) */
        case 8: look[0] = -look_delta; break; /* look right (-yaw) */
        case 9: look[1] = look_delta; break;  /* look up    (+pitch) */
        case 10: look[1] = -look_delta; break;/* look down  (-pitch) */
        default: break;                       /* 0 and unknown: no-op */
    }
}

#endif /* MC_PHILOX_H */
