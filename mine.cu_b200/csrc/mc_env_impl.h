// mc_env_impl.h - the env handle's internals and the runtime helpers shared
// by mc_runtime.cu (env and ragged handles) and mc_server.cu (env server).
// Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/minecu_b200.h"
#include "mc_internal.h"

#define MC_HIDDEN __attribute__((visibility("hidden")))

// NVTX range over a host phase (header-only NVTX3: a no-op unless a
// profiler that collects NVTX is attached).
#include <nvtx3/nvToolsExt.h>
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct RolloutGraph {
    cudaGraphExec_t exec = nullptr;
    const uint8_t* actions = nullptr;
    float* rewards_out = nullptr;
    uint8_t* dones_out = nullptr;
    int K = 0;
    mc_fused_cfg fcfg{};
    mc_kp kp{};
};

// Double-buffered host I/O of mc_env_step_host (allocated on first use).
struct HostIO {
    cudaStream_t up = nullptr, down = nullptr;  // action uploads, result read-backs
    uint8_t* d_act[2] = {nullptr, nullptr};     // B bytes each
    uint8_t* d_res[2] = {nullptr, nullptr};     // rewards (4B bytes) then dones (B bytes)
    cudaEvent_t act_ready[2] = {nullptr, nullptr}, act_free[2] = {nullptr, nullptr};
    cudaEvent_t res_ready[2] = {nullptr, nullptr}, res_free[2] = {nullptr, nullptr};
    long long calls = 0;
};

struct mc_env {
    mc_env_config cfg;
    mc_env_state st;
    mc_kp kp;
    const mc_backend* be;
    int device;
    int num_sms;
    mc_fused_cfg fcfg;
    int32_t* flags;
    int8_t* tmpl;
    uint8_t* scratch;  // plain-form decode buffers
    cudaStream_t cap_stream;
    std::vector<RolloutGraph> graphs;
    HostIO* hio;
    int regen_mode;  // MC_REGEN_ALL (the reference's rule) or MC_REGEN_PER_ENV
};

// Record a formatted message for mc_last_error() and return `code`.
MC_HIDDEN int mc_fail(int code, const char* fmt, ...);
// MC_ERR_CUDA with the CUDA error string.
MC_HIDDEN int mc_cuda_fail(cudaError_t e, const char* what);

// Whether a step of these parameters can end an episode (and so regenerate worlds).
MC_HIDDEN bool dones_possible(const mc_kp& k);

// Launch description of the team kernel over G groups (host copies of their
// parameter blocks, copied into the launch's parameter block); flags and
// actions are left to the caller.
MC_HIDDEN void team_layout(const mc_kp* const* kps, int G, const int* stage, const int* tile_w, const int* coop,
                           int team_warps, int warps_per_cta, mc_ragged_kp* rk);
// Dynamic shared memory of that launch per CTA.
MC_HIDDEN long long team_smem(const mc_ragged_kp& rk, int warps_per_cta);
// MC_OK, or MC_ERR_INVALID with a message when the team launch is not possible.
MC_HIDDEN int team_validate(const mc_kp* const* kps, int G, const int* stage, const int* tile_w, const int* coop,
                            int team_warps, int warps_per_cta, int ctas_per_sm);
