// mc_fast.cu - the "ref_fast" numerics back end.
// Built with --use_fast_math: the same CUDA math calls (sinf/cosf/tanf/__sincosf,
// "/", sqrtf, rsqrtf) and op order as the reference build (setup.py:19), so
// results equal the reference's bit for bit.
#define MC_NUMERICS_FAST 1
#define MC_NS mc_fast
#include "mc_backend_impl.cuh"

namespace mc_fast {
static int render_entry(const mc_kp* p, int family, cudaStream_t s) { return render_launch(p, family, s); }
static const mc_backend g_backend = {
    "ref_fast",
    step_plain,
    step_fused,
    render_entry,
    basis_launch,
    decode_launch,
    physics_launch,
    interact_launch,
    coalesced_launch,
    fused_smem,
    step_team,
    bounds_report,
    bounds_selftest,
};
}  // namespace mc_fast

extern "C" const mc_backend* mc_backend_fast() { return &mc_fast::g_backend; }
