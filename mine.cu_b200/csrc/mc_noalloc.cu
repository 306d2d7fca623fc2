// mc_noalloc.cu - the plain environment step without any device allocation.
//
// Some callers cannot allocate device memory at all: a host that hands the
// library pre-allocated buffers under a fixed memory budget, a process whose
// allocator is owned by another runtime, or code running where cudaMalloc is
// not allowed.  mc_env_create and the reference-style stateless entry points
// allocate small device buffers (flag words, decode scratch) on first use;
// mc_step_plain_noalloc does not.  Its scratch (the 8 action-decode arrays of
// the plain step and its flag words) lives in the file-scope array below,
// sized for MC_NOALLOC_MAX_ENVS envs (about 1.5 MB), which every GPU that
// loads the library holds until the process exits.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture.  The address is kept for the life of the
// process, so cudaDeviceReset on a device while the library is loaded is
// not supported (the kept address would no longer name the array).  Every
// call shares the one array, so calls that overlap on the GPU (different
// streams, or different host threads on the same device) race on it.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/minecu_b200.h"
#include "mc_internal.h"

namespace {

constexpr size_t kFlagBytes = 256;  // MC_FLAG_WORDS ints, padded to the array alignment
constexpr size_t kPerEnv = 5 * sizeof(float) + 3;  // fwd, strafe, dyaw, dpitch, speed + jump, brk, place
constexpr size_t kScratchBytes = kFlagBytes + ((size_t)MC_NOALLOC_MAX_ENVS * kPerEnv + 255) / 256 * 256;
static_assert(kFlagBytes >= MC_FLAG_WORDS * sizeof(int32_t), "the flag words must fit in front of the scratch");
static_assert(kFlagBytes % 16 == 0, "the decode arrays after the flag words stay 16-byte aligned");

static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

uint8_t* g_scratch_addr[64] = {nullptr};
std::mutex g_scratch_mu;

int noalloc_fail(int code, const char* msg) { return mc_set_error(code, msg); }

// Device address of the scratch array on the current device (set-up once per device).
int scratch_on_current_device(uint8_t** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return noalloc_fail(MC_ERR_CUDA, "mc_step_plain_noalloc: no current CUDA device");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(MC_ERR_CUDA, "mc_step_plain_noalloc: cudaGetSymbolAddress failed");
        g_scratch_addr[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return MC_OK;
}

}  // namespace

extern "C" int mc_step_plain_noalloc(const mc_env_config* cfg, const mc_env_state* st, const int8_t* buttons,
                                     const float* look, void* stream) {
    if (!cfg || !st) return noalloc_fail(MC_ERR_INVALID, "mc_step_plain_noalloc: NULL config or state");
    if (cfg->batch_size < 0 || cfg->batch_size > MC_NOALLOC_MAX_ENVS)
        return noalloc_fail(MC_ERR_INVALID,
                            "mc_step_plain_noalloc: batch_size outside 0..MC_NOALLOC_MAX_ENVS (65536); "
                            "use mc_step_stateless for larger batches");
    if (cfg->batch_size == 0) return MC_OK;
    uint8_t* base = nullptr;
    int rc = scratch_on_current_device(&base);
    if (rc) return rc;
    // the flag words must start at zero for every call
    cudaError_t e = cudaMemsetAsync(base, 0, kFlagBytes, (cudaStream_t)stream);
    if (e != cudaSuccess) return noalloc_fail(MC_ERR_CUDA, "mc_step_plain_noalloc: clearing the flag words failed");
    const size_t B = (size_t)cfg->batch_size;
    uint8_t* q = base + kFlagBytes;
    mc_decode_buffers d;
    d.forward_in = (float*)q; q += B * 4;
    d.strafe_in = (float*)q; q += B * 4;
    d.delta_yaw_in = (float*)q; q += B * 4;
    d.delta_pitch_in = (float*)q; q += B * 4;
    d.speed_mult = (float*)q; q += B * 4;
    d.jump_in = q; q += B;
    d.do_break = q; q += B;
    d.do_place = q;
    return mc_step_stateless_with_flags(cfg, st, buttons, look, &d, (int32_t*)base, MC_FORM_PLAIN, stream);
}
