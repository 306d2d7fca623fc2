// mc_server.cu - the env server: many client jobs stepped on one device.
//
// Jobs (env configurations) are admitted against an HBM budget; their state
// lives in one device block each (from the device's stream-ordered memory
// pool) and stays resident until released.  Client threads queue step and
// reset requests (mc_server_submit) and wait for them (mc_server_wait).
//
// Two threads run the device:
//  * the launcher takes, for every job with queued work, its oldest request
//    (up to MC_RAGGED_MAX_GROUPS step requests of one render family per
//    launch, oldest jobs first) and enqueues on the server stream: resets
//    (MineEnv.reset), one upload of all step actions, one team-kernel launch
//    over the stepping jobs (each job one group), the conditional world
//    regenerations, one read-back of all rewards and dones, an event;
//  * the completer waits for those events in launch order, hands the
//    results to the requests and records their latency (submission to
//    results in host memory).
// Both threads poll (the launcher its queue for a while before sleeping, the
// completer its event) instead of blocking, which keeps thread wake-ups out
// of the request latency at the cost of two busy host cores under load.
// Up to max_inflight launches are queued on the device at once, so the host
// work of the next launch overlaps the current one; the actions upload and
// the results read-back run on their own streams, so they overlap the
// neighbouring launches' kernels instead of queueing between them.  A job's requests run in
// submission order (one stream).  With batching = 0 the launcher takes one
// request at a time (oldest first) and steps with the plain form: the
// one-job-at-a-time loop the batched server is compared with.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <random>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/minecu_b200.h"
#include "mc_env_impl.h"
#include "mc_internal.h"
#include "mc_philox.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kMaxSlots = 4;
constexpr long long kDefaultCap = 1LL << 20;
constexpr int64_t kJobOverhead = 4096;  // flag words and handle-side allocations
constexpr int kSpin = 20000;            // launcher polls before sleeping on the condition variable

struct Job;

struct Req {
    int64_t ticket = 0;
    Job* job = nullptr;
    int job_id = -1;
    int kind = MC_REQ_STEP;
    std::vector<uint8_t> actions;
    Clock::time_point t_submit, t_done;
    std::vector<float> rewards;
    std::vector<uint8_t> dones;
    bool done = false;
    bool detached = false;  // nobody waits: freed at completion
    int status = MC_OK;
};

struct Job {
    bool live = false;
    bool reserved = false;   // slot in use (admission in progress, live, or release in progress)
    mc_env_config cfg{};
    mc_env* env = nullptr;
    void* block = nullptr;
    int64_t bytes = 0;
    mc_env_state st{};
    std::deque<Req*> queue;  // not launched yet
    int inflight = 0;        // launched, not completed
};

struct Slot {
    cudaEvent_t ev = nullptr;     // recorded after the read-back: the launch is complete
    cudaEvent_t ev_up = nullptr;  // actions uploaded
    cudaEvent_t ev_k = nullptr;   // device work of the launch done
    uint8_t* h_act = nullptr;  // pinned
    uint8_t* d_act = nullptr;
    uint8_t* h_res = nullptr;  // pinned: rewards (cap floats), then dones (cap bytes)
    uint8_t* d_res = nullptr;
    std::vector<Req*> reqs;
    std::vector<int> round;       // round of each request (a job's r-th request of the launch runs in round r)
    std::vector<long long> offs;  // env offset of each step request in the launch
    long long total = 0;          // envs of the step launch: rewards at [0, 4 total), dones after them
    bool step_launch = false;
    bool busy = false;
};

struct Rec {  // one completed request
    float lat_us;
    double t_submit, t_done;  // seconds since the statistics epoch
    int32_t envs;
    int8_t kind;
};

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

bool is_prebasis(int obs_mode) {
    return obs_mode == MC_OBS_UINT8_PREBASIS || obs_mode == MC_OBS_UINT8_PREBASIS_FULL ||
           obs_mode == MC_OBS_UINT8_SMEM;
}

int family_of_mode(int obs_mode) {
    switch (obs_mode) {
        case MC_OBS_FLOAT32:
        case MC_OBS_UINT8: return MC_FAM_SHADED;
        case MC_OBS_UINT8_FAST: return MC_FAM_SHADED_FAST;
        case MC_OBS_UINT8_MINIMAL: return MC_FAM_MINIMAL;
        case MC_OBS_UINT8_FP16: return MC_FAM_FP16;
        default: return MC_FAM_PREBASIS;
    }
}

// Offsets of the state tensors in a job's block (each 256-byte aligned).
struct JobLayout {
    size_t voxels, positions, velocities, yaws, pitches, on_ground, step_count, do_reset, cameras, basis, obs,
        rewards, total;
};

JobLayout job_layout(const mc_env_config* c) {
    const size_t B = (size_t)c->batch_size;
    const size_t wxyz = (size_t)c->world_x * c->world_y * c->world_z;
    const size_t px = (size_t)c->render_width * c->render_height * 3 * (c->obs_mode == MC_OBS_FLOAT32 ? 4 : 1);
    JobLayout L{};
    size_t o = 0;
    auto take = [&](size_t n) {
        size_t r = o;
        o += al256(n);
        return r;
    };
    L.voxels = take(B * wxyz);
    L.positions = take(B * 12);
    L.velocities = take(B * 12);
    L.yaws = take(B * 4);
    L.pitches = take(B * 4);
    L.on_ground = take(B);
    L.step_count = take(B * 4);
    L.do_reset = take(B);
    L.cameras = take(B * 20);
    L.basis = is_prebasis(c->obs_mode) ? take(B * 56) : (size_t)-1;
    L.obs = take(B * px);
    L.rewards = take(B * 4);
    L.total = o;
    return L;
}

int64_t job_bytes(const mc_env_config* c) {
    const size_t wxyz = (size_t)c->world_x * c->world_y * c->world_z;
    return (int64_t)(job_layout(c).total + al256(wxyz) + kJobOverhead);
}

double percentile(std::vector<float>& v, double q) {
    if (v.empty()) return 0.0;
    size_t k = (size_t)std::min<double>((double)v.size() - 1, q * (double)(v.size() - 1) + 0.5);
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

struct mc_server {
    mc_server_config cfg{};
    int device = 0;
    int num_sms = 0;
    const mc_backend* be = nullptr;
    long long cap = 0;
    int rounds = 1;  // step requests of one job per launch (mc_server_set_rounds)
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_slot, cv_flight;
    std::vector<std::unique_ptr<Job>> jobs;
    int64_t used = 0;
    std::unordered_map<int64_t, Req*> tickets;
    int64_t next_ticket = 1;
    int pending = 0;  // requests queued or in flight
    std::atomic<int> queued{0};  // requests queued, not launched (read without the lock by the launcher's spin)
    std::atomic<bool> stopping{false};
    bool stop = false, launcher_done = false;
    std::thread launcher, completer;
    cudaStream_t stream = nullptr, admit_stream = nullptr;
    cudaStream_t up = nullptr, down = nullptr;  // actions uploads, results read-backs
    int32_t* flags = nullptr;  // work counter of the team launches
    Slot slots[kMaxSlots];
    int nslots = 0;
    std::deque<int> flight;  // busy slots in launch order
    // statistics
    Clock::time_point epoch;
    std::vector<Rec> recs;
    int64_t launches = 0, jobs_in_launches = 0;
};

namespace {

bool has_queued(const mc_server* s) {
    for (auto& j : s->jobs)
        if (j->live && !j->queue.empty()) return true;
    return false;
}

int free_slot(const mc_server* s) {
    for (int i = 0; i < s->nslots; ++i)
        if (!s->slots[i].busy) return i;
    return -1;
}

// Requests of the next launch (called with the lock held), with the round
// each runs in.  Round 0 takes the oldest request of every job with work (up
// to 16 step requests of one render family, oldest first, within the env
// cap); round r > 0 takes the next queued request of the jobs that had one in
// round r - 1, while the envs of the whole launch stay within the cap.  A
// burst of one job's requests so runs in one launch (its steps one after
// another, a team launch per round) instead of one launch per request.
std::vector<Req*> take_batch(mc_server* s, std::vector<int>* rounds) {
    std::vector<Job*> cand;
    for (auto& j : s->jobs)
        if (j->live && !j->queue.empty()) cand.push_back(j.get());
    std::sort(cand.begin(), cand.end(),
              [](const Job* a, const Job* b) { return a->queue.front()->t_submit < b->queue.front()->t_submit; });
    std::vector<Req*> out;
    if (!s->cfg.batching) {
        if (!cand.empty()) out.push_back(cand[0]->queue.front());
    } else {
        int steps = 0, fam = -1, f32 = -1;
        long long envs = 0;
        for (Job* j : cand) {
            Req* r = j->queue.front();
            if (r->kind == MC_REQ_STEP) {
                const int jf = family_of_mode(j->cfg.obs_mode), jf32 = j->cfg.obs_mode == MC_OBS_FLOAT32;
                if (steps == MC_RAGGED_MAX_GROUPS || (fam >= 0 && (jf != fam || jf32 != f32))) continue;
                if (steps > 0 && envs + j->cfg.batch_size > s->cap) continue;
                fam = jf;
                f32 = jf32;
                envs += j->cfg.batch_size;
                ++steps;
            }
            out.push_back(r);
        }
    }
    rounds->assign(out.size(), 0);
    if (s->cfg.batching && s->rounds > 1) {
        long long envs = 0;
        int fam = -1, f32 = -1;  // every round's team launch renders one family
        for (Req* r : out)
            if (r->kind == MC_REQ_STEP) {
                envs += r->job->cfg.batch_size;
                fam = family_of_mode(r->job->cfg.obs_mode);
                f32 = r->job->cfg.obs_mode == MC_OBS_FLOAT32;
            }
        std::vector<Job*> prev;
        for (Req* r : out) prev.push_back(r->job);
        for (int rd = 1; rd < s->rounds && !prev.empty(); ++rd) {
            std::vector<Job*> next;
            int steps = 0;
            for (Job* j : prev) {
                if ((int)j->queue.size() <= rd) continue;
                Req* r = j->queue[rd];
                if (r->kind == MC_REQ_STEP) {
                    const int jf = family_of_mode(j->cfg.obs_mode), jf32 = j->cfg.obs_mode == MC_OBS_FLOAT32;
                    if (steps == MC_RAGGED_MAX_GROUPS || (fam >= 0 && (jf != fam || jf32 != f32))) continue;
                    if (envs + j->cfg.batch_size > s->cap) continue;
                    fam = jf;
                    f32 = jf32;
                    envs += j->cfg.batch_size;
                    ++steps;
                }
                out.push_back(r);
                rounds->push_back(rd);
                next.push_back(j);
            }
            prev.swap(next);
        }
    }
    for (Req* r : out) {
        r->job->queue.pop_front();
        r->job->inflight++;
    }
    s->queued -= (int)out.size();
    return out;
}

// Enqueue the device work of one launch on the server stream (no lock held;
// the jobs of `reqs` cannot be released while they are in flight).
int run_round(mc_server* s, Slot& sl, const std::vector<Req*>& reqs, const std::vector<size_t>& steps,
              cudaStream_t st);

int run_batch(mc_server* s, Slot& sl, const std::vector<Req*>& reqs) {
    cudaStream_t st = s->stream;
    sl.offs.assign(reqs.size(), -1);
    sl.step_launch = false;
    int rc = MC_OK;
    int nrounds = 1;
    for (int rd : sl.round) nrounds = std::max(nrounds, rd + 1);
    // step requests round by round, each round's in launch order: their envs'
    // actions and results are contiguous per round
    std::vector<size_t> steps;
    std::vector<size_t> round_first(nrounds + 1, 0);
    for (int rd = 0; rd < nrounds; ++rd) {
        round_first[rd] = steps.size();
        for (size_t i = 0; i < reqs.size(); ++i)
            if (sl.round[i] == rd && reqs[i]->kind == MC_REQ_STEP) steps.push_back(i);
    }
    round_first[nrounds] = steps.size();
    long long off = 0;
    for (size_t i : steps) {
        Req* r = reqs[i];
        memcpy(sl.h_act + off, r->actions.data(), r->actions.size());
        sl.offs[i] = off;
        off += r->job->cfg.batch_size;
    }
    sl.total = off;
    if (!steps.empty()) {
        sl.step_launch = true;
        cudaError_t ce = cudaMemcpyAsync(sl.d_act, sl.h_act, (size_t)off, cudaMemcpyHostToDevice, s->up);
        if (ce == cudaSuccess) ce = cudaEventRecord(sl.ev_up, s->up);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, sl.ev_up, 0);
        if (ce != cudaSuccess) return mc_cuda_fail(ce, "server: actions upload");
    }
    for (int rd = 0; rd < nrounds && rc == MC_OK; ++rd) {
        for (size_t i = 0; i < reqs.size(); ++i)
            if (sl.round[i] == rd && reqs[i]->kind == MC_REQ_RESET && rc == MC_OK)
                rc = mc_env_reset(reqs[i]->job->env, nullptr, st);
        if (rc != MC_OK || round_first[rd] == round_first[rd + 1]) continue;
        const std::vector<size_t> rsteps(steps.begin() + round_first[rd], steps.begin() + round_first[rd + 1]);
        rc = run_round(s, sl, reqs, rsteps, st);
    }
    return rc;
}

// One round's step requests (at most one per job, one render family) as one
// team launch plus the conditional regenerations.
int run_round(mc_server* s, Slot& sl, const std::vector<Req*>& reqs, const std::vector<size_t>& steps,
              cudaStream_t st) {
    int rc = MC_OK;
    cudaError_t ce = cudaSuccess;
    {
        const long long first = sl.offs[steps[0]];
        // rewards then dones, contiguous over the launch: one read-back
        float* d_rew = reinterpret_cast<float*>(sl.d_res) + first;
        uint8_t* d_done = sl.d_res + sl.total * 4 + first;
        uint8_t* d_act = sl.d_act + first;
        if (s->cfg.batching) {
            const int G = (int)steps.size();
            std::vector<const mc_kp*> kps(G);
            int stage[MC_MAX_GROUPS], tile_w[MC_MAX_GROUPS], coop[MC_MAX_GROUPS];
            bool any_coop = false;
            for (int g = 0; g < G; ++g) {
                const mc_env* e = reqs[steps[g]]->job->env;
                kps[g] = &e->kp;
                stage[g] = e->fcfg.stage;
                tile_w[g] = e->fcfg.tile_w;
                coop[g] = e->fcfg.coop;
                any_coop |= coop[g] != 0;
            }
            const int team = any_coop ? 4 : 1, cps = any_coop ? 3 : 4;
            if (team_validate(kps.data(), G, stage, tile_w, coop, team, 8, cps) != MC_OK)
                for (int g = 0; g < G; ++g) stage[g] = 0;  // the staged worlds do not fit together
            mc_ragged_kp rk;
            team_layout(kps.data(), G, stage, tile_w, coop, team, 8, &rk);
            rk.flags = s->flags;
            rk.actions = d_act;
            rk.rewards_cat = d_rew;
            rk.dones_cat = d_done;
            const mc_kp& k0 = *kps[0];
            rc = s->be->step_team(&rk, k0.family, k0.obs_f32, 8, cps, s->num_sms, st);
            if (rc) return mc_cuda_fail((cudaError_t)rc, "server: step launch");
            rc = mc_launch_regen_groups(kps.data(), G, s->flags + MC_FLAG_REGEN_CTR, st);
            if (rc) return mc_cuda_fail((cudaError_t)rc, "server: regeneration");
        } else {
            Req* r = reqs[steps[0]];
            rc = mc_env_step_discrete(r->job->env, d_act, MC_FORM_PLAIN, st);
            if (rc) return rc;
            const long long B = r->job->cfg.batch_size;
            ce = cudaMemcpyAsync(d_rew, r->job->st.rewards, B * 4, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(d_done, r->job->st.do_reset, B, cudaMemcpyDeviceToDevice, st);
            if (ce != cudaSuccess) return mc_cuda_fail(ce, "server: result gather");
        }
    }
    return rc;
}

// After the device work of a launch: its results read-back on the read-back
// stream, then the event the completer waits for.
int finish_batch(mc_server* s, Slot& sl, bool readback) {
    cudaError_t ce = cudaEventRecord(sl.ev_k, s->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s->down, sl.ev_k, 0);
    if (ce == cudaSuccess && readback)
        ce = cudaMemcpyAsync(sl.h_res, sl.d_res, (size_t)sl.total * 5, cudaMemcpyDeviceToHost, s->down);
    if (ce == cudaSuccess) ce = cudaEventRecord(sl.ev, s->down);
    return ce == cudaSuccess ? MC_OK : mc_cuda_fail(ce, "server: results read-back");
}

void launcher_main(mc_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Req*> reqs;
        int si;
        // poll for work for a while before sleeping: a thread woken through
        // the condition variable adds tens of microseconds to a request
        for (int i = 0; i < kSpin && s->queued.load(std::memory_order_relaxed) == 0 &&
                        !s->stopping.load(std::memory_order_relaxed);
             ++i)
            std::this_thread::yield();
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || has_queued(s); });
            if (!has_queued(s)) {
                s->launcher_done = true;
                s->cv_flight.notify_all();
                return;
            }
            s->cv_slot.wait(lk, [&] { return free_slot(s) >= 0; });
            si = free_slot(s);
            s->slots[si].busy = true;
            reqs = take_batch(s, &s->slots[si].round);
        }
        Slot& sl = s->slots[si];
        NvtxRange nvtx("mc_server launch");
        int rc = run_batch(s, sl, reqs);
        const int rc_fin = finish_batch(s, sl, rc == MC_OK && sl.step_launch);
        if (rc == MC_OK) rc = rc_fin;
        for (Req* r : reqs)
            if (rc != MC_OK) r->status = rc;
        std::lock_guard<std::mutex> lk(s->mu);
        sl.reqs = reqs;
        s->flight.push_back(si);
        s->cv_flight.notify_one();
    }
}

void completer_main(mc_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        int si;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_flight.wait(lk, [&] { return !s->flight.empty() || s->launcher_done; });
            if (s->flight.empty()) return;
            si = s->flight.front();
        }
        Slot& sl = s->slots[si];
        // poll the event rather than block on it (lower completion latency)
        cudaError_t ce;
        while ((ce = cudaEventQuery(sl.ev)) == cudaErrorNotReady) std::this_thread::yield();
        const Clock::time_point t = Clock::now();
        NvtxRange nvtx("mc_server complete");
        std::lock_guard<std::mutex> lk(s->mu);
        int nsteps = 0;
        for (size_t i = 0; i < sl.reqs.size(); ++i) {
            Req* r = sl.reqs[i];
            if (ce != cudaSuccess && r->status == MC_OK) r->status = MC_ERR_CUDA;
            const long long B = r->job->cfg.batch_size;
            if (r->kind == MC_REQ_STEP) {
                ++nsteps;
                if (!r->detached && r->status == MC_OK) {
                    const float* rew = reinterpret_cast<const float*>(sl.h_res) + sl.offs[i];
                    const uint8_t* dn = sl.h_res + sl.total * 4 + sl.offs[i];
                    r->rewards.assign(rew, rew + B);
                    r->dones.assign(dn, dn + B);
                }
            }
            r->job->inflight--;
            s->pending--;
            r->t_done = t;
            r->done = true;
            Rec rec;
            rec.lat_us = (float)std::chrono::duration<double, std::micro>(t - r->t_submit).count();
            rec.t_submit = std::chrono::duration<double>(r->t_submit - s->epoch).count();
            rec.t_done = std::chrono::duration<double>(t - s->epoch).count();
            rec.envs = r->kind == MC_REQ_STEP ? (int32_t)B : 0;
            rec.kind = (int8_t)r->kind;
            if (r->status == MC_OK) s->recs.push_back(rec);
            if (r->detached) delete r;
        }
        if (sl.step_launch) {
            s->launches++;
            s->jobs_in_launches += nsteps;
        }
        sl.reqs.clear();
        sl.busy = false;
        s->flight.pop_front();
        s->cv_done.notify_all();
        s->cv_slot.notify_one();
        s->cv_work.notify_one();
    }
}

Job* live_job(mc_server* s, int32_t job) {
    if (job < 0 || job >= (int32_t)s->jobs.size() || !s->jobs[job]->live) return nullptr;
    return s->jobs[job].get();
}

int submit_impl(mc_server* s, int32_t job, int32_t kind, const uint8_t* actions, bool detached, int64_t* ticket) {
    if (kind != MC_REQ_STEP && kind != MC_REQ_RESET) return mc_fail(MC_ERR_INVALID, "server: unknown request kind %d", kind);
    Req* r = new Req();
    r->kind = kind;
    r->detached = detached;
    r->job_id = job;
    std::lock_guard<std::mutex> lk(s->mu);
    Job* j = live_job(s, job);
    if (!j) {
        delete r;
        return mc_fail(MC_ERR_INVALID, "server: job %d is not admitted", job);
    }
    if (kind == MC_REQ_STEP) {
        if (!actions) {
            delete r;
            return mc_fail(MC_ERR_INVALID, "server: step request without actions");
        }
        r->actions.assign(actions, actions + j->cfg.batch_size);
    }
    r->job = j;
    r->t_submit = Clock::now();
    r->ticket = s->next_ticket++;
    if (!detached) s->tickets[r->ticket] = r;
    if (ticket) *ticket = detached ? 0 : r->ticket;
    j->queue.push_back(r);
    s->pending++;
    s->queued++;
    s->cv_work.notify_one();
    return MC_OK;
}

void fill_stats(mc_server* s, double t_begin, double t_end, bool window, mc_server_stats* out) {
    std::vector<float> lat, rlat;
    int64_t env_steps = 0, n_step = 0, n_reset = 0;
    double sum = 0.0, mx = 0.0;
    for (const Rec& r : s->recs) {
        if (window && (r.t_submit < t_begin || r.t_submit > t_end)) continue;
        if (r.kind == MC_REQ_STEP) {
            lat.push_back(r.lat_us);
            sum += r.lat_us;
            mx = std::max(mx, (double)r.lat_us);
            ++n_step;
            if (!window || r.t_done <= t_end) env_steps += r.envs;
        } else {
            rlat.push_back(r.lat_us);
            ++n_reset;
        }
    }
    *out = mc_server_stats{};
    out->step_requests = n_step;
    out->reset_requests = n_reset;
    out->env_steps = env_steps;
    out->launches = s->launches;
    out->elapsed_s = window ? (t_end - t_begin) : std::chrono::duration<double>(Clock::now() - s->epoch).count();
    out->env_steps_per_s = out->elapsed_s > 0 ? env_steps / out->elapsed_s : 0.0;
    out->p50_us = percentile(lat, 0.50);
    out->p90_us = percentile(lat, 0.90);
    out->p99_us = percentile(lat, 0.99);
    out->max_us = mx;
    out->mean_us = n_step ? sum / n_step : 0.0;
    out->reset_p50_us = percentile(rlat, 0.50);
    out->reset_p99_us = percentile(rlat, 0.99);
    out->mean_jobs_per_launch = s->launches ? (double)s->jobs_in_launches / s->launches : 0.0;
    int32_t live = 0;
    for (auto& j : s->jobs) live += j->live;
    out->jobs = live;
    out->bytes_admitted = s->used;
}

}  // namespace

extern "C" int64_t mc_server_job_bytes(const mc_env_config* cfg) {
    if (!cfg || cfg->batch_size < 0 || cfg->world_x <= 0 || cfg->world_y <= 0 || cfg->world_z <= 0 ||
        cfg->render_width <= 0 || cfg->render_height <= 0)
        return -1;
    return job_bytes(cfg);
}

extern "C" int mc_server_create(const mc_server_config* cfg, mc_server** out) {
    if (!out) return mc_fail(MC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!cfg) return mc_fail(MC_ERR_INVALID, "server config is NULL");
    if (cfg->hbm_budget_bytes <= 0) return mc_fail(MC_ERR_INVALID, "hbm_budget_bytes must be > 0");
    if (cfg->numerics != MC_NUMERICS_REF_FAST && cfg->numerics != MC_NUMERICS_IEEE)
        return mc_fail(MC_ERR_INVALID, "unknown numerics %d", cfg->numerics);
    if (cfg->max_inflight < 1 || cfg->max_inflight > kMaxSlots)
        return mc_fail(MC_ERR_INVALID, "max_inflight must be 1..%d", kMaxSlots);
    if (cfg->max_envs_per_launch < 0) return mc_fail(MC_ERR_INVALID, "max_envs_per_launch < 0");
    mc_server* s = new mc_server();
    s->cfg = *cfg;
    s->cap = cfg->max_envs_per_launch ? cfg->max_envs_per_launch : kDefaultCap;
    s->be = cfg->numerics == MC_NUMERICS_REF_FAST ? mc_backend_fast() : mc_backend_ieee();
    s->nslots = cfg->max_inflight;
    s->epoch = Clock::now();
    cudaError_t ce = cudaGetDevice(&s->device);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->admit_stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMalloc(&s->flags, MC_FLAG_WORDS * sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaMemset(s->flags, 0, MC_FLAG_WORDS * sizeof(int32_t));
    for (int i = 0; i < s->nslots && ce == cudaSuccess; ++i) {
        Slot& sl = s->slots[i];
        ce = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&sl.ev_up, cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&sl.ev_k, cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaMallocHost(&sl.h_act, (size_t)s->cap);
        if (ce == cudaSuccess) ce = cudaMalloc(&sl.d_act, (size_t)s->cap);
        if (ce == cudaSuccess) ce = cudaMallocHost(&sl.h_res, (size_t)s->cap * 5);
        if (ce == cudaSuccess) ce = cudaMalloc(&sl.d_res, (size_t)s->cap * 5);
    }
    if (ce != cudaSuccess) {
        int rc = mc_cuda_fail(ce, "mc_server_create");
        s->launcher_done = true;
        mc_server_destroy(s);
        return rc;
    }
    s->launcher = std::thread(launcher_main, s);
    s->completer = std::thread(completer_main, s);
    *out = s;
    return MC_OK;
}

extern "C" int mc_server_set_rounds(mc_server* s, int32_t rounds) {
    if (!s) return mc_fail(MC_ERR_INVALID, "server is NULL");
    if (rounds < 1 || rounds > 8) return mc_fail(MC_ERR_INVALID, "rounds must be 1..8");
    std::lock_guard<std::mutex> lk(s->mu);
    s->rounds = rounds;
    return MC_OK;
}

extern "C" int mc_server_destroy(mc_server* s) {
    if (!s) return MC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->stopping = true;
        s->cv_work.notify_all();
        s->cv_flight.notify_all();
    }
    if (s->launcher.joinable()) s->launcher.join();
    if (s->completer.joinable()) s->completer.join();
    cudaSetDevice(s->device);
    // the launcher ran every queued request before it stopped; the tickets
    // left hold completed requests nobody waited for
    for (auto& j : s->jobs) {
        if (j->env) mc_env_destroy(j->env);
        if (j->block) cudaFree(j->block);
    }
    for (auto& kv : s->tickets) delete kv.second;
    for (int i = 0; i < s->nslots; ++i) {
        Slot& sl = s->slots[i];
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.ev_up) cudaEventDestroy(sl.ev_up);
        if (sl.ev_k) cudaEventDestroy(sl.ev_k);
        if (sl.h_act) cudaFreeHost(sl.h_act);
        if (sl.d_act) cudaFree(sl.d_act);
        if (sl.h_res) cudaFreeHost(sl.h_res);
        if (sl.d_res) cudaFree(sl.d_res);
    }
    if (s->flags) cudaFree(s->flags);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->up) cudaStreamDestroy(s->up);
    if (s->down) cudaStreamDestroy(s->down);
    if (s->admit_stream) cudaStreamDestroy(s->admit_stream);
    delete s;
    return MC_OK;
}

extern "C" int mc_server_admit(mc_server* s, const mc_env_config* cfg, int32_t* job) {
    if (!s || !cfg || !job) return mc_fail(MC_ERR_INVALID, "NULL argument");
    *job = -1;
    if (cfg->numerics != s->cfg.numerics)
        return mc_fail(MC_ERR_INVALID, "job numerics %d differs from the server's %d", cfg->numerics, s->cfg.numerics);
    const int64_t bytes = mc_server_job_bytes(cfg);
    if (bytes < 0) return mc_fail(MC_ERR_INVALID, "invalid job configuration");
    if (cfg->batch_size > s->cap)
        return mc_fail(MC_ERR_INVALID, "batch_size %d above max_envs_per_launch %lld", cfg->batch_size, s->cap);
    int32_t id;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->used + bytes > s->cfg.hbm_budget_bytes)
            return mc_fail(MC_ERR_BUDGET, "job needs %lld bytes; %lld of the %lld-byte budget are in use",
                           (long long)bytes, (long long)s->used, (long long)s->cfg.hbm_budget_bytes);
        s->used += bytes;  // reserved
        id = -1;
        for (size_t i = 0; i < s->jobs.size(); ++i)
            if (!s->jobs[i]->reserved) {
                id = (int32_t)i;
                break;
            }
        if (id < 0) {
            s->jobs.emplace_back(new Job());
            id = (int32_t)s->jobs.size() - 1;
        }
        s->jobs[id]->reserved = true;
    }
    cudaSetDevice(s->device);
    auto unreserve = [&](int rc) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->used -= bytes;
        s->jobs[id]->reserved = false;
        return rc;
    };
    const JobLayout L = job_layout(cfg);
    void* block = nullptr;
    cudaError_t ce = cudaMallocAsync(&block, L.total, s->admit_stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(block, 0, L.total, s->admit_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->admit_stream);
    if (ce != cudaSuccess) {
        if (block) cudaFree(block);
        return unreserve(mc_cuda_fail(ce, "mc_server_admit: allocation"));
    }
    uint8_t* b = static_cast<uint8_t*>(block);
    mc_env_state st{};
    st.voxels = reinterpret_cast<int8_t*>(b + L.voxels);
    st.positions = reinterpret_cast<float*>(b + L.positions);
    st.velocities = reinterpret_cast<float*>(b + L.velocities);
    st.yaws = reinterpret_cast<float*>(b + L.yaws);
    st.pitches = reinterpret_cast<float*>(b + L.pitches);
    st.on_ground = b + L.on_ground;
    st.step_count = reinterpret_cast<int32_t*>(b + L.step_count);
    st.do_reset = b + L.do_reset;
    st.cameras = reinterpret_cast<float*>(b + L.cameras);
    st.basis = L.basis == (size_t)-1 ? nullptr : reinterpret_cast<float*>(b + L.basis);
    st.obs = b + L.obs;
    st.rewards = reinterpret_cast<float*>(b + L.rewards);
    mc_env* env = nullptr;
    int rc = mc_env_create(cfg, &st, &env);
    if (rc == MC_OK) rc = mc_env_generate_world(env, s->admit_stream);
    if (rc == MC_OK) rc = mc_env_reset(env, nullptr, s->admit_stream);
    if (rc == MC_OK) {
        ce = cudaStreamSynchronize(s->admit_stream);
        if (ce != cudaSuccess) rc = mc_cuda_fail(ce, "mc_server_admit: world generation");
    }
    if (rc != MC_OK) {
        if (env) mc_env_destroy(env);
        cudaFree(block);
        return unreserve(rc);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    Job& j = *s->jobs[id];
    j.cfg = *cfg;
    j.env = env;
    j.block = block;
    j.bytes = bytes;
    j.st = st;
    j.inflight = 0;
    j.live = true;
    *job = id;
    return MC_OK;
}

extern "C" int mc_server_release(mc_server* s, int32_t job) {
    if (!s) return mc_fail(MC_ERR_INVALID, "server is NULL");
    mc_env* env;
    void* block;
    int64_t bytes;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        Job* j = live_job(s, job);
        if (!j) return mc_fail(MC_ERR_INVALID, "server: job %d is not admitted", job);
        if (!j->queue.empty() || j->inflight)
            return mc_fail(MC_ERR_BUSY, "server: job %d has %zu queued and %d running requests", job, j->queue.size(),
                           j->inflight);
        // completed requests nobody waited for
        for (auto it = s->tickets.begin(); it != s->tickets.end();) {
            if (it->second->job_id == job) {
                delete it->second;
                it = s->tickets.erase(it);
            } else {
                ++it;
            }
        }
        j->live = false;
        env = j->env;
        block = j->block;
        bytes = j->bytes;
    }
    cudaSetDevice(s->device);
    mc_env_destroy(env);
    cudaError_t ce = cudaFreeAsync(block, s->admit_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->admit_stream);
    std::lock_guard<std::mutex> lk(s->mu);
    Job& j = *s->jobs[job];
    j.env = nullptr;
    j.block = nullptr;
    j.reserved = false;
    s->used -= bytes;
    if (ce != cudaSuccess) return mc_cuda_fail(ce, "mc_server_release");
    return MC_OK;
}

extern "C" int mc_server_job_state(mc_server* s, int32_t job, mc_env_state* out) {
    if (!s || !out) return mc_fail(MC_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    Job* j = live_job(s, job);
    if (!j) return mc_fail(MC_ERR_INVALID, "server: job %d is not admitted", job);
    *out = j->st;
    return MC_OK;
}

extern "C" int mc_server_submit(mc_server* s, int32_t job, int32_t kind, const uint8_t* actions, int64_t* ticket) {
    if (!s || !ticket) return mc_fail(MC_ERR_INVALID, "NULL argument");
    return submit_impl(s, job, kind, actions, false, ticket);
}

extern "C" int mc_server_wait(mc_server* s, int64_t ticket, float* rewards, uint8_t* dones, int64_t timeout_us) {
    if (!s) return mc_fail(MC_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return mc_fail(MC_ERR_INVALID, "server: unknown ticket %lld", (long long)ticket);
    Req* r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready)) {
        return mc_fail(MC_ERR_TIMEOUT, "server: ticket %lld not complete after %lld us", (long long)ticket,
                       (long long)timeout_us);
    }
    if (r->kind == MC_REQ_STEP && r->status == MC_OK) {
        if (rewards) memcpy(rewards, r->rewards.data(), r->rewards.size() * sizeof(float));
        if (dones) memcpy(dones, r->dones.data(), r->dones.size());
    }
    const int status = r->status;
    s->tickets.erase(it);
    delete r;
    if (status != MC_OK) return mc_fail(status, "server: request failed on the device");
    return MC_OK;
}

extern "C" int mc_server_get_stats(mc_server* s, mc_server_stats* out) {
    if (!s || !out) return mc_fail(MC_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    fill_stats(s, 0.0, 0.0, false, out);
    return MC_OK;
}

extern "C" int mc_server_reset_stats(mc_server* s) {
    if (!s) return mc_fail(MC_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    s->recs.clear();
    s->launches = 0;
    s->jobs_in_launches = 0;
    s->epoch = Clock::now();
    return MC_OK;
}

extern "C" int mc_server_drive(mc_server* s, const mc_load_config* cfg, mc_server_stats* out) {
    if (!s || !cfg || !out) return mc_fail(MC_ERR_INVALID, "NULL argument");
    if (cfg->seconds <= 0 || cfg->njobs < 1 || !cfg->jobs) return mc_fail(MC_ERR_INVALID, "empty load");
    std::vector<int32_t> batch(cfg->njobs);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int i = 0; i < cfg->njobs; ++i) {
            Job* j = live_job(s, cfg->jobs[i].job);
            if (!j) return mc_fail(MC_ERR_INVALID, "load job %d: job %d is not admitted", i, cfg->jobs[i].job);
            if (!cfg->closed_loop && !(cfg->jobs[i].rate_hz > 0))
                return mc_fail(MC_ERR_INVALID, "load job %d: rate_hz must be > 0", i);
            batch[i] = j->cfg.batch_size;
        }
    }
    mc_server_reset_stats(s);
    const Clock::time_point t_begin = Clock::now();
    const Clock::time_point t_end = t_begin + std::chrono::duration_cast<Clock::duration>(
                                                  std::chrono::duration<double>(cfg->seconds));
    std::vector<int> errors(cfg->njobs, MC_OK);
    std::vector<std::thread> clients;
    for (int i = 0; i < cfg->njobs; ++i) {
        clients.emplace_back([&, i] {
            const mc_load_job& lj = cfg->jobs[i];
            std::mt19937_64 rng(((uint64_t)lj.seed << 20) ^ (uint64_t)i);
            std::exponential_distribution<double> gap(cfg->closed_loop ? 1.0 : lj.rate_hz);
            std::vector<uint8_t> acts(batch[i]);
            Clock::time_point next = t_begin;
            for (int64_t n = 0;; ++n) {
                if (!cfg->closed_loop) {
                    next += std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(gap(rng)));
                    if (next >= t_end) break;
                    std::this_thread::sleep_until(next);
                } else if (Clock::now() >= t_end) {
                    break;
                }
                const bool reset = lj.episode_steps > 0 && n % ((int64_t)lj.episode_steps + 1) == 0;
                if (!reset)
                    for (int e = 0; e < batch[i]; ++e)
                        acts[e] = (uint8_t)mc_action_draw(lj.seed, (uint32_t)e, (uint32_t)n, false);
                int64_t ticket = 0;
                int rc = submit_impl(s, lj.job, reset ? MC_REQ_RESET : MC_REQ_STEP, acts.data(), !cfg->closed_loop,
                                     &ticket);
                if (rc == MC_OK && cfg->closed_loop) rc = mc_server_wait(s, ticket, nullptr, nullptr, -1);
                if (rc != MC_OK) {
                    errors[i] = rc;
                    break;
                }
            }
        });
    }
    for (auto& t : clients) t.join();
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->pending == 0; });
        const double b = std::chrono::duration<double>(t_begin - s->epoch).count();
        const double e = std::chrono::duration<double>(t_end - s->epoch).count();
        fill_stats(s, b, e, true, out);
    }
    for (int i = 0; i < cfg->njobs; ++i)
        if (errors[i] != MC_OK) return mc_fail(errors[i], "load job %d stopped on an error", i);
    return MC_OK;
}
