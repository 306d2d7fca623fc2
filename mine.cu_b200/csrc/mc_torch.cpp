// mc_torch.cpp - the torch extension minecu._C.
//
// Keeps the reference module's function names, argument order and defaults
// (src/bindings.cpp:985-1269) so that code written against the reference's
// minecu._C runs unchanged, and adds the handle API used by minecu.MineEnv.
// Every function turns tensors into raw pointers, checks device, dtype,
// shape and contiguity (the reference checks only a few device/dtype
// properties, src/bindings.cpp:223-228, 453-457), and calls the C-ABI of
// libminecu_b200.so on torch's current CUDA stream.
#include <torch/extension.h>

#include <vector>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include <cstdint>
#include <string>

#include "../../include/minecu_b200.h"

namespace {

void ck(int rc, const char* what) {
    TORCH_CHECK(rc == MC_OK, what, " failed (", rc, "): ", mc_last_error());
}

void* cur_stream() { return (void*)at::cuda::getCurrentCUDAStream().stream(); }

void need(const torch::Tensor& t, const char* name, at::ScalarType dt) {
    TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
    TORCH_CHECK(t.scalar_type() == dt, name, " must be ", c10::toString(dt), ", got ", c10::toString(t.scalar_type()));
    TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
}

void need_shape(const torch::Tensor& t, const char* name, std::initializer_list<int64_t> shape) {
    TORCH_CHECK(t.dim() == (int64_t)shape.size(), name, " must have ", shape.size(), " dims, got ", t.dim());
    int i = 0;
    for (int64_t s : shape) {
        TORCH_CHECK(s < 0 || t.size(i) == s, name, " dim ", i, " must be ", s, ", got ", t.size(i));
        ++i;
    }
}

template <class T>
T* ptr(const torch::Tensor& t) { return t.numel() ? reinterpret_cast<T*>(t.data_ptr()) : nullptr; }

template <class T>
T* opt_ptr(const c10::optional<torch::Tensor>& t) {
    return (t.has_value() && t->defined() && t->numel()) ? reinterpret_cast<T*>(t->data_ptr()) : nullptr;
}

// ---------------------------------------------------------------------------
// the reference's pybind functions
// ---------------------------------------------------------------------------
struct StepTensors {
    torch::Tensor voxels, positions, velocities, yaws, pitches, on_ground, buttons, look, do_reset;
    torch::Tensor forward_in, strafe_in, delta_yaw_in, delta_pitch_in, jump_in, do_break, do_place, speed_mult;
    torch::Tensor cameras, obs_buffer, rewards;
};

mc_env_config step_config(const StepTensors& T, int obs_mode, int width, int height, int max_steps, float vd,
                          float fov, float dt, float gravity, float walk_speed, float sprint_mult, float jump_vel,
                          int target_block, float reward_value, int episode_length) {
    mc_env_config c{};
    c.batch_size = (int32_t)T.voxels.size(0);
    c.world_y = (int32_t)T.voxels.size(1);
    c.world_x = (int32_t)T.voxels.size(2);
    c.world_z = (int32_t)T.voxels.size(3);
    c.render_width = width;
    c.render_height = height;
    c.max_steps = max_steps;
    c.view_distance = vd;
    c.fov_degrees = fov;
    c.dt = dt;
    c.gravity = gravity;
    c.walk_speed = walk_speed;
    c.sprint_mult = sprint_mult;
    c.jump_vel = jump_vel;
    c.ground_height = 0;
    c.target_block = target_block;
    c.reward_value = reward_value;
    c.has_episode_limit = episode_length > 0;
    c.episode_length = episode_length;
    c.obs_mode = obs_mode;
    c.numerics = MC_NUMERICS_REF_FAST;
    c.look_delta = 0.0f;
    return c;
}

void check_step_tensors(const StepTensors& T, bool f32_obs, int width, int height) {
    need(T.voxels, "voxels", at::kChar);
    TORCH_CHECK(T.voxels.dim() == 4, "voxels must be [B, Y, X, Z]");
    int64_t B = T.voxels.size(0);
    need(T.positions, "positions", at::kFloat);
    need_shape(T.positions, "positions", {B, 3});
    need(T.velocities, "velocities", at::kFloat);
    need_shape(T.velocities, "velocities", {B, 3});
    need(T.yaws, "yaws", at::kFloat);
    need_shape(T.yaws, "yaws", {B});
    need(T.pitches, "pitches", at::kFloat);
    need_shape(T.pitches, "pitches", {B});
    need(T.on_ground, "on_ground", at::kBool);
    need_shape(T.on_ground, "on_ground", {B});
    need(T.buttons, "buttons", at::kChar);
    need_shape(T.buttons, "buttons", {B, 8});
    need(T.look, "look", at::kFloat);
    need_shape(T.look, "look", {B, 2});
    need(T.do_reset, "do_reset", at::kBool);
    need_shape(T.do_reset, "do_reset", {B});
    need(T.cameras, "cameras", at::kFloat);
    need_shape(T.cameras, "cameras", {B, 5});
    need(T.obs_buffer, "obs_buffer", f32_obs ? at::kFloat : at::kByte);
    need_shape(T.obs_buffer, "obs_buffer", {B, height, width, 3});
    need(T.rewards, "rewards", at::kFloat);
    need_shape(T.rewards, "rewards", {B});
    const char* fn[] = {"forward_in", "strafe_in", "delta_yaw_in", "delta_pitch_in", "speed_mult"};
    const torch::Tensor* ft[] = {&T.forward_in, &T.strafe_in, &T.delta_yaw_in, &T.delta_pitch_in, &T.speed_mult};
    for (int i = 0; i < 5; ++i) {
        need(*ft[i], fn[i], at::kFloat);
        need_shape(*ft[i], fn[i], {B});
    }
    const char* bn[] = {"jump_in", "do_break", "do_place"};
    const torch::Tensor* bt[] = {&T.jump_in, &T.do_break, &T.do_place};
    for (int i = 0; i < 3; ++i) {
        need(*bt[i], bn[i], at::kBool);
        need_shape(*bt[i], bn[i], {B});
    }
}

void run_step(const StepTensors& T, int obs_mode, torch::Tensor* basis, torch::Tensor* step_count, int width,
              int height, int max_steps, float vd, float fov, float dt, float gravity, float walk_speed,
              float sprint_mult, float jump_vel, int target_block, float reward_value, float spawn_x, float spawn_y,
              float spawn_z, int episode_length, int ground_height = 0) {
    bool f32 = obs_mode == MC_OBS_FLOAT32;
    check_step_tensors(T, f32, width, height);
    c10::cuda::CUDAGuard g(T.voxels.device());
    mc_env_config c = step_config(T, obs_mode, width, height, max_steps, vd, fov, dt, gravity, walk_speed,
                                  sprint_mult, jump_vel, target_block, reward_value, episode_length);
    c.spawn_override = 1;
    c.spawn_x = spawn_x;
    c.spawn_y = spawn_y;
    c.spawn_z = spawn_z;
    c.ground_height = ground_height;
    mc_env_state s{};
    s.voxels = ptr<int8_t>(T.voxels);
    s.positions = ptr<float>(T.positions);
    s.velocities = ptr<float>(T.velocities);
    s.yaws = ptr<float>(T.yaws);
    s.pitches = ptr<float>(T.pitches);
    s.on_ground = ptr<uint8_t>(T.on_ground);
    s.do_reset = ptr<uint8_t>(T.do_reset);
    s.cameras = ptr<float>(T.cameras);
    s.obs = T.obs_buffer.data_ptr();
    s.rewards = ptr<float>(T.rewards);
    if (step_count) {
        need(*step_count, "step_count", at::kInt);
        need_shape(*step_count, "step_count", {T.voxels.size(0)});
        s.step_count = ptr<int32_t>(*step_count);
    }  // else NULL: these modes' episode counter lives in Python and the step never touches it
    if (basis) {
        need(*basis, "basis", at::kFloat);
        need_shape(*basis, "basis", {T.voxels.size(0), 14});
        s.basis = ptr<float>(*basis);
    }
    mc_decode_buffers d{ptr<float>(T.forward_in),   ptr<float>(T.strafe_in),  ptr<float>(T.delta_yaw_in),
                        ptr<float>(T.delta_pitch_in), ptr<uint8_t>(T.jump_in), ptr<uint8_t>(T.do_break),
                        ptr<uint8_t>(T.do_place),   ptr<float>(T.speed_mult)};
    ck(mc_step_stateless(&c, &s, ptr<int8_t>(T.buttons), ptr<float>(T.look), &d, MC_FORM_PLAIN, cur_stream()),
       "step");
}

#define STEP_ARGS                                                                                                  \
    torch::Tensor voxels, torch::Tensor positions, torch::Tensor velocities, torch::Tensor yaws,                  \
        torch::Tensor pitches, torch::Tensor on_ground, torch::Tensor buttons, torch::Tensor look,                \
        torch::Tensor do_reset, torch::Tensor forward_in, torch::Tensor strafe_in, torch::Tensor delta_yaw_in,    \
        torch::Tensor delta_pitch_in, torch::Tensor jump_in, torch::Tensor do_break, torch::Tensor do_place,      \
        torch::Tensor speed_mult, torch::Tensor cameras
#define STEP_TAIL                                                                                                  \
    torch::Tensor obs_buffer, torch::Tensor rewards, int width, int height, int max_steps, float view_distance,   \
        float fov_degrees, float dt, float gravity, float walk_speed, float sprint_mult, float jump_vel,          \
        int target_block, float reward_value, float spawn_x, float spawn_y, float spawn_z
#define STEP_T                                                                                                     \
    StepTensors T{voxels,     positions, velocities,   yaws,           pitches,  on_ground, buttons,              \
                  look,       do_reset,  forward_in,   strafe_in,      delta_yaw_in, delta_pitch_in, jump_in,      \
                  do_break,   do_place,  speed_mult,   cameras,        obs_buffer, rewards}
#define STEP_PARAMS                                                                                                \
    width, height, max_steps, view_distance, fov_degrees, dt, gravity, walk_speed, sprint_mult, jump_vel,        \
        target_block, reward_value, spawn_x, spawn_y, spawn_z

void py_step(STEP_ARGS, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_FLOAT32, nullptr, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8(STEP_ARGS, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_UINT8, nullptr, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8_fast(STEP_ARGS, STEP_TAIL, int ground_height) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_FAST, nullptr, nullptr, STEP_PARAMS, 0, ground_height);
}
void py_step_uint8_minimal(STEP_ARGS, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_MINIMAL, nullptr, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8_fp16(STEP_ARGS, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_FP16, nullptr, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8_prebasis(STEP_ARGS, torch::Tensor basis, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_PREBASIS, &basis, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8_smem(STEP_ARGS, torch::Tensor basis, STEP_TAIL) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_SMEM, &basis, nullptr, STEP_PARAMS, 0);
}
void py_step_uint8_prebasis_full(torch::Tensor voxels, torch::Tensor positions, torch::Tensor velocities,
                                 torch::Tensor yaws, torch::Tensor pitches, torch::Tensor on_ground,
                                 torch::Tensor buttons, torch::Tensor look, torch::Tensor do_reset,
                                 torch::Tensor step_count, torch::Tensor forward_in, torch::Tensor strafe_in,
                                 torch::Tensor delta_yaw_in, torch::Tensor delta_pitch_in, torch::Tensor jump_in,
                                 torch::Tensor do_break, torch::Tensor do_place, torch::Tensor speed_mult,
                                 torch::Tensor cameras, torch::Tensor basis, STEP_TAIL, int episode_length) {
    STEP_T;
    run_step(T, MC_OBS_UINT8_PREBASIS_FULL, &basis, &step_count, STEP_PARAMS, episode_length);
}

mc_env_config render_config(const torch::Tensor& voxels, const torch::Tensor& output, int obs_mode, int max_steps,
                            float vd, float fov) {
    need(voxels, "voxels", at::kChar);
    TORCH_CHECK(voxels.dim() == 4, "voxels must be [B, Y, X, Z]");
    TORCH_CHECK(output.dim() == 4 && output.size(3) == 3, "output must be [B, H, W, 3]");
    TORCH_CHECK(output.size(0) == voxels.size(0), "batch mismatch");
    mc_env_config c{};
    c.batch_size = (int32_t)voxels.size(0);
    c.world_y = (int32_t)voxels.size(1);
    c.world_x = (int32_t)voxels.size(2);
    c.world_z = (int32_t)voxels.size(3);
    c.render_height = (int32_t)output.size(1);
    c.render_width = (int32_t)output.size(2);
    c.max_steps = max_steps;
    c.view_distance = vd;
    c.fov_degrees = fov;
    c.obs_mode = obs_mode;
    c.numerics = MC_NUMERICS_REF_FAST;
    return c;
}

void py_render_any(torch::Tensor voxels, torch::Tensor cameras, torch::Tensor output, int max_steps, float vd,
                   float fov, bool f32) {
    mc_env_config c = render_config(voxels, output, f32 ? MC_OBS_FLOAT32 : MC_OBS_UINT8, max_steps, vd, fov);
    need(output, "output", f32 ? at::kFloat : at::kByte);
    need(cameras, "cameras", at::kFloat);
    need_shape(cameras, "cameras", {voxels.size(0), 5});
    c10::cuda::CUDAGuard g(voxels.device());
    mc_env_state s{};
    s.voxels = ptr<int8_t>(voxels);
    s.cameras = ptr<float>(cameras);
    s.obs = output.data_ptr();
    ck(mc_render(&c, &s, 1, cur_stream()), "render");
}

void py_render(torch::Tensor voxels, torch::Tensor cameras, torch::Tensor output, int max_steps, float vd, float fov) {
    py_render_any(voxels, cameras, output, max_steps, vd, fov, true);
}
void py_render_uint8(torch::Tensor voxels, torch::Tensor cameras, torch::Tensor output, int max_steps, float vd,
                     float fov) {
    py_render_any(voxels, cameras, output, max_steps, vd, fov, false);
}

void py_physics(torch::Tensor positions, torch::Tensor velocities, torch::Tensor yaws, torch::Tensor pitches,
                torch::Tensor on_ground, torch::Tensor forward_in, torch::Tensor strafe_in, torch::Tensor delta_yaw_in,
                torch::Tensor delta_pitch_in, torch::Tensor jump_in, torch::Tensor speed_mult, int world_size,
                float dt, float gravity, float walk_speed, float jump_vel) {
    need(positions, "positions", at::kFloat);
    int64_t B = positions.size(0);
    need(on_ground, "on_ground", at::kBool);
    need(jump_in, "jump_in", at::kBool);
    c10::cuda::CUDAGuard g(positions.device());
    ck(mc_physics(ptr<float>(positions), ptr<float>(velocities), ptr<float>(yaws), ptr<float>(pitches),
                  ptr<uint8_t>(on_ground), ptr<float>(forward_in), ptr<float>(strafe_in), ptr<float>(delta_yaw_in),
                  ptr<float>(delta_pitch_in), ptr<uint8_t>(jump_in), ptr<float>(speed_mult), (int32_t)B, world_size,
                  dt, gravity, walk_speed, jump_vel, MC_NUMERICS_REF_FAST, cur_stream()),
       "physics");
}

void py_raycast_break(torch::Tensor voxels, torch::Tensor positions, torch::Tensor yaws, torch::Tensor pitches,
                      torch::Tensor do_break, torch::Tensor rewards, int target_block, float reward_value) {
    need(voxels, "voxels", at::kChar);
    need(do_break, "do_break", at::kBool);
    c10::cuda::CUDAGuard g(voxels.device());
    TORCH_CHECK(voxels.size(1) == voxels.size(2) && voxels.size(2) == voxels.size(3),
                "raycast_break takes a cubic world (as launch_raycast_break)");
    ck(mc_raycast_break(ptr<int8_t>(voxels), ptr<float>(positions), ptr<float>(yaws), ptr<float>(pitches),
                        ptr<uint8_t>(do_break), ptr<float>(rewards), (int32_t)voxels.size(0), (int32_t)voxels.size(1),
                        target_block, reward_value, MC_NUMERICS_REF_FAST, cur_stream()),
       "raycast_break");
}

void py_reset(torch::Tensor positions, torch::Tensor velocities, torch::Tensor yaws, torch::Tensor pitches,
              torch::Tensor on_ground, torch::Tensor do_reset, float spawn_x, float spawn_y, float spawn_z) {
    need(do_reset, "do_reset", at::kBool);
    need(on_ground, "on_ground", at::kBool);
    c10::cuda::CUDAGuard g(positions.device());
    ck(mc_reset_agents(ptr<float>(positions), ptr<float>(velocities), ptr<float>(yaws), ptr<float>(pitches),
                       ptr<uint8_t>(on_ground), ptr<uint8_t>(do_reset), (int32_t)positions.size(0), spawn_x, spawn_y,
                       spawn_z, cur_stream()),
       "reset");
}

void py_generate_world(torch::Tensor voxels, int ground_height, unsigned int seed) {
    need(voxels, "voxels", at::kChar);
    c10::cuda::CUDAGuard g(voxels.device());
    ck(mc_generate_world(ptr<int8_t>(voxels), (int32_t)voxels.size(0), (int32_t)voxels.size(2),
                         (int32_t)voxels.size(1), (int32_t)voxels.size(3), ground_height, seed, cur_stream()),
       "generate_world");
}

void py_place_tree(torch::Tensor voxels, int tree_x, int tree_z, int ground_height) {
    need(voxels, "voxels", at::kChar);
    c10::cuda::CUDAGuard g(voxels.device());
    ck(mc_place_tree(ptr<int8_t>(voxels), (int32_t)voxels.size(0), (int32_t)voxels.size(2), (int32_t)voxels.size(1),
                     (int32_t)voxels.size(3), tree_x, tree_z, ground_height, cur_stream()),
       "place_tree");
}

void py_place_house(torch::Tensor voxels, int house_x, int house_z, int ground_height) {
    need(voxels, "voxels", at::kChar);
    c10::cuda::CUDAGuard g(voxels.device());
    ck(mc_place_house(ptr<int8_t>(voxels), (int32_t)voxels.size(0), (int32_t)voxels.size(2), (int32_t)voxels.size(1),
                      (int32_t)voxels.size(3), house_x, house_z, ground_height, cur_stream()),
       "place_house");
}

void py_precompute_camera_basis(torch::Tensor cameras, torch::Tensor basis, int width, int height, float fov) {
    need(cameras, "cameras", at::kFloat);
    need(basis, "basis", at::kFloat);
    c10::cuda::CUDAGuard g(cameras.device());
    ck(mc_precompute_camera_basis(ptr<float>(cameras), ptr<float>(basis), (int32_t)cameras.size(0), width, height, fov,
                                  MC_NUMERICS_REF_FAST, cur_stream()),
       "precompute_camera_basis");
}

void py_render_uint8_prebasis(torch::Tensor voxels, torch::Tensor basis, torch::Tensor output, int max_steps) {
    need(voxels, "voxels", at::kChar);
    need(basis, "basis", at::kFloat);
    need(output, "output", at::kByte);
    c10::cuda::CUDAGuard g(voxels.device());
    // the reference passes world_size = voxels.size(1) for all three axes
    // (src/bindings.cpp:938-960); a cubic world gives the same arithmetic
    ck(mc_render_uint8_prebasis(ptr<int8_t>(voxels), ptr<float>(basis), ptr<uint8_t>(output), (int32_t)voxels.size(0),
                                (int32_t)voxels.size(2), (int32_t)voxels.size(1), (int32_t)voxels.size(3),
                                (int32_t)output.size(2), (int32_t)output.size(1), max_steps, MC_NUMERICS_REF_FAST,
                                cur_stream()),
       "render_uint8_prebasis");
}

void py_render_uint8_coalesced(torch::Tensor voxels, torch::Tensor basis, torch::Tensor output, int max_steps) {
    need(voxels, "voxels", at::kChar);
    need(basis, "basis", at::kFloat);
    need(output, "output", at::kByte);
    TORCH_CHECK(voxels.dim() == 4, "voxels must be [Y, X, Z, B]");
    c10::cuda::CUDAGuard g(voxels.device());
    ck(mc_render_uint8_coalesced(ptr<int8_t>(voxels), ptr<float>(basis), ptr<uint8_t>(output),
                                 (int32_t)voxels.size(3), (int32_t)voxels.size(0), (int32_t)output.size(2),
                                 (int32_t)output.size(1), max_steps, MC_NUMERICS_REF_FAST, cur_stream()),
       "render_uint8_coalesced");
}

// ---------------------------------------------------------------------------
// handle API used by minecu.MineEnv
// ---------------------------------------------------------------------------
struct Env {
    mc_env* h = nullptr;
    ~Env() {
        if (h) mc_env_destroy(h);
    }
};

mc_env_state state_of(const py::dict& st) {
    auto T = [&](const char* k) -> torch::Tensor { return st[k].cast<torch::Tensor>(); };
    auto P = [&](const char* k) -> void* {
        if (!st.contains(k) || st[k].is_none()) return nullptr;
        torch::Tensor t = st[k].cast<torch::Tensor>();
        TORCH_CHECK(t.is_cuda() && t.is_contiguous(), k, " must be a contiguous CUDA tensor");
        return t.numel() ? t.data_ptr() : nullptr;
    };
    (void)T;
    mc_env_state s{};
    s.voxels = (int8_t*)P("voxels");
    s.positions = (float*)P("positions");
    s.velocities = (float*)P("velocities");
    s.yaws = (float*)P("yaws");
    s.pitches = (float*)P("pitches");
    s.on_ground = (uint8_t*)P("on_ground");
    s.step_count = (int32_t*)P("step_count");
    s.do_reset = (uint8_t*)P("do_reset");
    s.cameras = (float*)P("cameras");
    s.basis = (float*)P("basis");
    s.obs = P("obs_buffer");
    s.rewards = (float*)P("rewards");
    s.dbg_interact = (int32_t*)P("dbg_interact");
    s.dbg_pixel = (int16_t*)P("dbg_pixel");
    return s;
}

mc_env_config config_of(const py::dict& d) {
    mc_env_config c{};
    auto I = [&](const char* k) { return d[k].cast<int32_t>(); };
    auto F = [&](const char* k) { return d[k].cast<float>(); };
    c.batch_size = I("batch_size");
    c.world_x = I("world_x");
    c.world_y = I("world_y");
    c.world_z = I("world_z");
    c.render_width = I("render_width");
    c.render_height = I("render_height");
    c.max_steps = I("max_steps");
    c.view_distance = F("view_distance");
    c.fov_degrees = F("fov_degrees");
    c.dt = F("dt");
    c.gravity = F("gravity");
    c.walk_speed = F("walk_speed");
    c.sprint_mult = F("sprint_mult");
    c.jump_vel = F("jump_vel");
    c.ground_height = I("ground_height");
    c.target_block = I("target_block");
    c.reward_value = F("reward_value");
    c.has_episode_limit = I("has_episode_limit");
    c.episode_length = I("episode_length");
    c.obs_mode = I("obs_mode");
    c.numerics = I("numerics");
    c.look_delta = F("look_delta");
    return c;
}

std::shared_ptr<Env> env_create(py::dict cfg, py::dict state) {
    auto e = std::make_shared<Env>();
    mc_env_config c = config_of(cfg);
    mc_env_state s = state_of(state);
    ck(mc_env_create(&c, &s, &e->h), "env_create");
    return e;
}

void env_set_state(std::shared_ptr<Env> e, py::dict state) {
    mc_env_state s = state_of(state);
    ck(mc_env_set_state(e->h, &s), "env_set_state");
}

void env_generate_world(std::shared_ptr<Env> e) { ck(mc_env_generate_world(e->h, cur_stream()), "generate_world"); }

void env_reset(std::shared_ptr<Env> e, c10::optional<torch::Tensor> mask) {
    const uint8_t* m = nullptr;
    if (mask.has_value() && mask->defined()) {
        need(*mask, "mask", at::kBool);
        m = ptr<uint8_t>(*mask);
    }
    ck(mc_env_reset(e->h, m, cur_stream()), "reset");
}

void env_step(std::shared_ptr<Env> e, torch::Tensor buttons, torch::Tensor look, int form) {
    need(buttons, "buttons", at::kChar);
    need(look, "look", at::kFloat);
    ck(mc_env_step(e->h, ptr<int8_t>(buttons), ptr<float>(look), form, cur_stream()), "step");
}

void env_step_discrete(std::shared_ptr<Env> e, torch::Tensor actions, int form) {
    need(actions, "actions", at::kByte);
    ck(mc_env_step_discrete(e->h, ptr<uint8_t>(actions), form, cur_stream()), "step");
}

// Host tensors of mc_env_step_host: pinned CPU memory, contiguous, n entries.
void need_pinned(const torch::Tensor& t, const char* name, std::initializer_list<at::ScalarType> dts, int64_t n) {
    TORCH_CHECK(!t.is_cuda(), name, " must be a host (CPU) tensor");
    bool ok = false;
    for (auto dt : dts) ok |= t.scalar_type() == dt;
    TORCH_CHECK(ok, name, " has dtype ", c10::toString(t.scalar_type()), ", which this call does not take");
    TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
    TORCH_CHECK(t.numel() == n, name, " must have ", n, " entries, got ", t.numel());
    TORCH_CHECK(t.is_pinned(), name, " must be in pinned memory (tensor.pin_memory())");
}

void env_step_host(std::shared_ptr<Env> e, torch::Tensor actions, torch::Tensor rewards, torch::Tensor dones,
                   int64_t batch, int form) {
    need_pinned(actions, "actions", {at::kByte}, batch);
    need_pinned(rewards, "rewards_out", {at::kFloat}, batch);
    need_pinned(dones, "dones_out", {at::kBool, at::kByte}, batch);
    ck(mc_env_step_host(e->h, static_cast<const uint8_t*>(actions.data_ptr()), rewards.data_ptr<float>(),
                        static_cast<uint8_t*>(dones.data_ptr()), form, cur_stream()),
       "step_host");
}

void env_host_join(std::shared_ptr<Env> e) { ck(mc_env_host_join(e->h, cur_stream()), "host_join"); }

void obs_to_policy(torch::Tensor obs, torch::Tensor out, int64_t layout) {
    need(obs, "obs", at::kByte);
    need(out, "out", at::kFloat);
    TORCH_CHECK(obs.dim() == 4 && obs.size(3) == 3, "obs must be uint8 [B, H, W, 3]");
    TORCH_CHECK(out.numel() == obs.numel(), "out must have as many elements as obs");
    TORCH_CHECK(out.device() == obs.device(), "obs and out must be on the same device");
    ck(mc_obs_to_policy(obs.data_ptr<uint8_t>(), out.data_ptr<float>(), obs.size(0), (int32_t)obs.size(1),
                        (int32_t)obs.size(2), (int32_t)layout, cur_stream()),
       "obs_to_policy");
}

void env_render(std::shared_ptr<Env> e) { ck(mc_env_render(e->h, cur_stream()), "render"); }

void env_set_regen_mode(std::shared_ptr<Env> e, int mode) { ck(mc_env_set_regen_mode(e->h, mode), "set_regen_mode"); }
void env_set_wait_limit(std::shared_ptr<Env> e, int polls) { ck(mc_env_set_wait_limit(e->h, polls), "set_wait_limit"); }

void env_regenerate_if(std::shared_ptr<Env> e, torch::Tensor flag) {
    TORCH_CHECK(flag.is_cuda() && flag.numel() >= 1 && flag.element_size() == 1,
                "flag must be a one-byte CUDA tensor (uint8 or bool)");
    ck(mc_env_regenerate_if(e->h, static_cast<const uint8_t*>(flag.data_ptr()), cur_stream()), "regenerate_if");
}

void env_rollout(std::shared_ptr<Env> e, torch::Tensor actions, c10::optional<torch::Tensor> rewards_out,
                 c10::optional<torch::Tensor> dones_out) {
    need(actions, "actions", at::kByte);
    TORCH_CHECK(actions.dim() == 2, "actions must be [K, B]");
    ck(mc_env_rollout(e->h, ptr<uint8_t>(actions), (int32_t)actions.size(0), opt_ptr<float>(rewards_out),
                      opt_ptr<uint8_t>(dones_out), cur_stream()),
       "rollout");
}

void env_rollout_prepare(std::shared_ptr<Env> e, torch::Tensor actions, c10::optional<torch::Tensor> rewards_out,
                         c10::optional<torch::Tensor> dones_out) {
    need(actions, "actions", at::kByte);
    TORCH_CHECK(actions.dim() == 2, "actions must be [K, B]");
    ck(mc_env_rollout_prepare(e->h, ptr<uint8_t>(actions), (int32_t)actions.size(0), opt_ptr<float>(rewards_out),
                              opt_ptr<uint8_t>(dones_out)),
       "rollout_prepare");
}

void env_set_fused(std::shared_ptr<Env> e, int stage, int warps_per_cta, int ctas_per_sm, int tile_w, int team_warps,
                   int coop) {
    mc_fused_config f{stage, warps_per_cta, ctas_per_sm, tile_w, team_warps, coop};
    ck(mc_env_set_fused_config(e->h, &f), "set_fused_config");
}

py::dict env_get_fused(std::shared_ptr<Env> e) {
    mc_fused_config f{};
    ck(mc_env_get_fused_config(e->h, &f), "get_fused_config");
    py::dict d;
    d["stage"] = f.stage;
    d["warps_per_cta"] = f.warps_per_cta;
    d["ctas_per_sm"] = f.ctas_per_sm;
    d["tile_w"] = f.tile_w;
    d["team_warps"] = f.team_warps;
    d["coop"] = f.coop;
    d["smem_bytes"] = mc_env_fused_smem_bytes(e->h);
    return d;
}

void env_check_error(std::shared_ptr<Env> e) { ck(mc_env_check_error(e->h, cur_stream()), "check_error"); }

// ragged handle: several Env handles stepped by one launch
struct Ragged {
    mc_ragged* h = nullptr;
    std::vector<std::shared_ptr<Env>> groups;  // keeps the borrowed env handles alive
    ~Ragged() {
        if (h) mc_ragged_destroy(h);
    }
};

std::shared_ptr<Ragged> ragged_create(std::vector<std::shared_ptr<Env>> groups) {
    auto r = std::make_shared<Ragged>();
    std::vector<mc_env*> hs;
    for (auto& g : groups) {
        TORCH_CHECK(g && g->h, "ragged_create: a group is not a live env handle");
        hs.push_back(g->h);
    }
    r->groups = groups;
    ck(mc_ragged_create(hs.data(), (int32_t)hs.size(), &r->h), "ragged_create");
    return r;
}

void ragged_set_config(std::shared_ptr<Ragged> r, int warps_per_cta, int ctas_per_sm, int team_warps,
                       std::vector<int> stage, std::vector<int> tile_w, std::vector<int> coop) {
    const size_t G = r->groups.size();
    TORCH_CHECK(stage.size() == G && tile_w.size() == G && coop.size() == G,
                "one stage, one tile_w and one coop per group");
    mc_ragged_config c{};
    c.warps_per_cta = warps_per_cta;
    c.ctas_per_sm = ctas_per_sm;
    c.team_warps = team_warps;
    for (size_t g = 0; g < G; ++g) {
        c.stage[g] = stage[g];
        c.tile_w[g] = tile_w[g];
        c.coop[g] = coop[g];
    }
    ck(mc_ragged_set_config(r->h, &c), "ragged_set_config");
}

py::dict ragged_get_config(std::shared_ptr<Ragged> r) {
    mc_ragged_config c{};
    ck(mc_ragged_get_config(r->h, &c), "ragged_get_config");
    std::vector<int> st, tw, co;
    for (size_t g = 0; g < r->groups.size(); ++g) {
        st.push_back(c.stage[g]);
        tw.push_back(c.tile_w[g]);
        co.push_back(c.coop[g]);
    }
    py::dict d;
    d["warps_per_cta"] = c.warps_per_cta;
    d["ctas_per_sm"] = c.ctas_per_sm;
    d["team_warps"] = c.team_warps;
    d["stage"] = st;
    d["tile_w"] = tw;
    d["coop"] = co;
    d["smem_bytes"] = mc_ragged_smem_bytes(r->h);
    return d;
}

int64_t ragged_total_envs(std::shared_ptr<Ragged> r) { return mc_ragged_total_envs(r->h); }

void ragged_step(std::shared_ptr<Ragged> r, torch::Tensor buttons, torch::Tensor look) {
    need(buttons, "buttons", at::kChar);
    need(look, "look", at::kFloat);
    const int64_t n = mc_ragged_total_envs(r->h);
    TORCH_CHECK(buttons.numel() == n * 8 && look.numel() == n * 2, "buttons [total,8], look [total,2]");
    ck(mc_ragged_step(r->h, ptr<int8_t>(buttons), ptr<float>(look), cur_stream()), "ragged_step");
}

void ragged_step_discrete(std::shared_ptr<Ragged> r, torch::Tensor actions) {
    need(actions, "actions", at::kByte);
    TORCH_CHECK(actions.numel() == mc_ragged_total_envs(r->h), "actions must hold one action per env");
    ck(mc_ragged_step_discrete(r->h, ptr<uint8_t>(actions), cur_stream()), "ragged_step");
}

void ragged_step_host(std::shared_ptr<Ragged> r, torch::Tensor actions, torch::Tensor rewards, torch::Tensor dones) {
    const int64_t n = mc_ragged_total_envs(r->h);
    need_pinned(actions, "actions", {at::kByte}, n);
    need_pinned(rewards, "rewards_out", {at::kFloat}, n);
    need_pinned(dones, "dones_out", {at::kBool, at::kByte}, n);
    ck(mc_ragged_step_host(r->h, static_cast<const uint8_t*>(actions.data_ptr()), rewards.data_ptr<float>(),
                           static_cast<uint8_t*>(dones.data_ptr()), cur_stream()),
       "ragged_step_host");
}

void ragged_host_join(std::shared_ptr<Ragged> r) { ck(mc_ragged_host_join(r->h, cur_stream()), "ragged_host_join"); }

void ragged_rollout(std::shared_ptr<Ragged> r, torch::Tensor actions, bool prepare_only) {
    need(actions, "actions", at::kByte);
    TORCH_CHECK(actions.dim() == 2 && actions.size(1) == mc_ragged_total_envs(r->h), "actions must be [K, total]");
    if (prepare_only)
        ck(mc_ragged_rollout_prepare(r->h, ptr<uint8_t>(actions), (int32_t)actions.size(0)), "ragged_rollout_prepare");
    else
        ck(mc_ragged_rollout(r->h, ptr<uint8_t>(actions), (int32_t)actions.size(0), cur_stream()), "ragged_rollout");
}

void ragged_check_error(std::shared_ptr<Ragged> r) { ck(mc_ragged_check_error(r->h, cur_stream()), "check_error"); }

void philox_actions(torch::Tensor out, int env_offset, int step0, uint64_t seed, bool break_half) {
    need(out, "out", at::kByte);
    TORCH_CHECK(out.dim() == 2, "out must be [K, B]");
    ck(mc_philox_actions(ptr<uint8_t>(out), (int32_t)out.size(1), (int32_t)out.size(0), env_offset, step0, seed,
                         break_half ? 1 : 0, cur_stream()),
       "philox_actions");
}

void discrete_to_buttons(torch::Tensor actions, double look_delta, torch::Tensor buttons, torch::Tensor look) {
    need(actions, "actions", at::kByte);
    need(buttons, "buttons", at::kChar);
    need(look, "look", at::kFloat);
    ck(mc_discrete_to_buttons(ptr<uint8_t>(actions), (int32_t)actions.numel(), (float)look_delta,
                              ptr<int8_t>(buttons), ptr<float>(look), cur_stream()),
       "discrete_to_buttons");
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.doc() = "mine.cu environment step on B200 (torch bindings of libminecu_b200.so)";
    m.attr("ABI_VERSION") = mc_abi_version();

    // ---- the reference module's functions (src/bindings.cpp:985-1269) ----
    m.def("render", &py_render, py::arg("voxels"), py::arg("cameras"), py::arg("output"), py::arg("max_steps") = 64,
          py::arg("view_distance") = 32.0f, py::arg("fov_degrees") = 70.0f);
    m.def("render_uint8", &py_render_uint8, py::arg("voxels"), py::arg("cameras"), py::arg("output"),
          py::arg("max_steps") = 64, py::arg("view_distance") = 32.0f, py::arg("fov_degrees") = 70.0f);
    m.def("physics", &py_physics, py::arg("positions"), py::arg("velocities"), py::arg("yaws"), py::arg("pitches"),
          py::arg("on_ground"), py::arg("forward_in"), py::arg("strafe_in"), py::arg("delta_yaw_in"),
          py::arg("delta_pitch_in"), py::arg("jump_in"), py::arg("speed_mult"), py::arg("world_size"),
          py::arg("dt") = 0.05f, py::arg("gravity") = -20.0f, py::arg("walk_speed") = 4.0f,
          py::arg("jump_vel") = 8.0f);
    m.def("raycast_break", &py_raycast_break, py::arg("voxels"), py::arg("positions"), py::arg("yaws"),
          py::arg("pitches"), py::arg("do_break"), py::arg("rewards"), py::arg("target_block") = -1,
          py::arg("reward_value") = 1.0f);
    m.def("reset", &py_reset, py::arg("positions"), py::arg("velocities"), py::arg("yaws"), py::arg("pitches"),
          py::arg("on_ground"), py::arg("do_reset"), py::arg("spawn_x"), py::arg("spawn_y"), py::arg("spawn_z"));
    m.def("generate_world", &py_generate_world, py::arg("voxels"), py::arg("ground_height"), py::arg("seed") = 42);
    m.def("place_tree", &py_place_tree, py::arg("voxels"), py::arg("tree_x"), py::arg("tree_z"),
          py::arg("ground_height"));
    m.def("place_house", &py_place_house, py::arg("voxels"), py::arg("house_x"), py::arg("house_z"),
          py::arg("ground_height"));
#define STEP_PYARGS                                                                                                \
    py::arg("voxels"), py::arg("positions"), py::arg("velocities"), py::arg("yaws"), py::arg("pitches"),          \
        py::arg("on_ground"), py::arg("buttons"), py::arg("look"), py::arg("do_reset")
#define STEP_PYDEC                                                                                                 \
    py::arg("forward_in"), py::arg("strafe_in"), py::arg("delta_yaw_in"), py::arg("delta_pitch_in"),              \
        py::arg("jump_in"), py::arg("do_break"), py::arg("do_place"), py::arg("speed_mult"), py::arg("cameras")
#define STEP_PYTAIL                                                                                                \
    py::arg("obs_buffer"), py::arg("rewards"), py::arg("width"), py::arg("height"), py::arg("max_steps") = 64,    \
        py::arg("view_distance") = 32.0f, py::arg("fov_degrees") = 70.0f, py::arg("dt") = 0.05f,                  \
        py::arg("gravity") = -20.0f, py::arg("walk_speed") = 4.0f, py::arg("sprint_mult") = 1.5f,                 \
        py::arg("jump_vel") = 8.0f, py::arg("target_block") = -1, py::arg("reward_value") = 1.0f,                 \
        py::arg("spawn_x") = 16.0f, py::arg("spawn_y") = 9.0f, py::arg("spawn_z") = 16.0f
    m.def("step", &py_step, STEP_PYARGS, STEP_PYDEC, STEP_PYTAIL);
    m.def("step_uint8", &py_step_uint8, STEP_PYARGS, STEP_PYDEC, STEP_PYTAIL);
    m.def("step_uint8_fast", &py_step_uint8_fast, STEP_PYARGS, STEP_PYDEC, STEP_PYTAIL,
          py::arg("ground_height") = 8);
    m.def("step_uint8_minimal", &py_step_uint8_minimal, STEP_PYARGS, STEP_PYDEC, STEP_PYTAIL);
    m.def("step_uint8_fp16", &py_step_uint8_fp16, STEP_PYARGS, STEP_PYDEC, STEP_PYTAIL);
    m.def("step_uint8_prebasis", &py_step_uint8_prebasis, STEP_PYARGS, STEP_PYDEC, py::arg("basis"), STEP_PYTAIL);
    m.def("step_uint8_smem", &py_step_uint8_smem, STEP_PYARGS, STEP_PYDEC, py::arg("basis"), STEP_PYTAIL);
    m.def("step_uint8_prebasis_full", &py_step_uint8_prebasis_full, STEP_PYARGS, py::arg("step_count"),
          STEP_PYDEC, py::arg("basis"), STEP_PYTAIL, py::arg("episode_length") = 0);
    m.def("precompute_camera_basis", &py_precompute_camera_basis, py::arg("cameras"), py::arg("basis"),
          py::arg("width"), py::arg("height"), py::arg("fov_degrees") = 70.0f);
    m.def("render_uint8_prebasis", &py_render_uint8_prebasis, py::arg("voxels"), py::arg("basis"),
          py::arg("output"), py::arg("max_steps") = 64);
    m.def("render_uint8_coalesced", &py_render_uint8_coalesced, py::arg("voxels"), py::arg("basis"),
          py::arg("output"), py::arg("max_steps") = 64);

    // ---- handle API --------------------------------------------------------
    py::class_<Env, std::shared_ptr<Env>>(m, "Env");
    m.def("env_create", &env_create);
    m.def("env_set_state", &env_set_state);
    m.def("env_generate_world", &env_generate_world);
    m.def("env_reset", &env_reset, py::arg("env"), py::arg("mask") = py::none());
    m.def("env_step", &env_step);
    m.def("env_step_discrete", &env_step_discrete);
    m.def("env_step_host", &env_step_host);
    m.def("env_host_join", &env_host_join);
    m.def("obs_to_policy", &obs_to_policy);
    m.def("env_render", &env_render);
    m.def("env_set_regen_mode", &env_set_regen_mode);
    m.def("env_set_wait_limit", &env_set_wait_limit);
    m.def("env_regenerate_if", &env_regenerate_if);
    m.def("env_rollout", &env_rollout, py::arg("env"), py::arg("actions"), py::arg("rewards_out") = py::none(),
          py::arg("dones_out") = py::none());
    m.def("env_rollout_prepare", &env_rollout_prepare, py::arg("env"), py::arg("actions"),
          py::arg("rewards_out") = py::none(), py::arg("dones_out") = py::none());
    m.def("env_set_fused", &env_set_fused);
    m.def("env_get_fused", &env_get_fused);
    m.def("env_check_error", &env_check_error);
    py::class_<Ragged, std::shared_ptr<Ragged>>(m, "Ragged");
    m.def("ragged_create", &ragged_create);
    m.def("ragged_set_config", &ragged_set_config);
    m.def("ragged_step_host", &ragged_step_host);
    m.def("ragged_host_join", &ragged_host_join);
    m.def("ragged_get_config", &ragged_get_config);
    m.def("ragged_total_envs", &ragged_total_envs);
    m.def("ragged_step", &ragged_step);
    m.def("ragged_step_discrete", &ragged_step_discrete);
    m.def("ragged_rollout", &ragged_rollout, py::arg("ragged"), py::arg("actions"), py::arg("prepare_only") = false);
    m.def("ragged_check_error", &ragged_check_error);
    m.def("philox_actions", &philox_actions, py::arg("out"), py::arg("env_offset"), py::arg("step0"),
          py::arg("seed"), py::arg("break_half") = false);
    m.def("discrete_to_buttons", &discrete_to_buttons);
}
