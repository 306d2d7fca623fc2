// mc_ieee.cu - the "ieee" numerics back end.
// Built with -fmad=false and IEEE division/sqrt: every op is a single
// IEEE-754 rounding and trig comes from mc_ieee_math.h, so results equal the
// CPU checker (oracle/mc_oracle.c) bit for bit.
#define MC_NUMERICS_FAST 0
#define MC_NS mc_ieee
#include "mc_backend_impl.cuh"

namespace mc_ieee {
static int render_entry(const mc_kp* p, int family, cudaStream_t s) { return render_launch(p, family, s); }
static const mc_backend g_backend = {
    "ieee",
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
}  // namespace mc_ieee

extern "C" const mc_backend* mc_backend_ieee() { return &mc_ieee::g_backend; }
