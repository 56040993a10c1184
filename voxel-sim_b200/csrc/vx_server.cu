// vx_server.cu — the served form: host threads that keep scenes resident in
// pools, admit new requests at round boundaries as slots and memory free up,
// and step every resident scene of a pool together (include/vxcorot.h).
//
// With several lanes, requests are routed by size: each lane has its own pool,
// stream and thread, and steps only scenes up to its REV bound. A round lasts
// as long as its largest scene needs, so a small scene in its own lane runs
// short rounds, concurrently on the GPU with the long rounds of the large
// scenes, instead of waiting for them; the lanes of smaller scenes get higher
// stream priorities. A scene's result does not depend on its lane (pool slots
// keep per-scene scalars).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vx_internal.h"
#include "vx_kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// A request owns a copy of its scene until the pool has it.
struct Request {
    uint64_t ticket = 0;
    uint32_t n = 0;
    std::vector<double> pos, rot, target;
    std::vector<uint8_t> kin, tmask;
    std::vector<float> mass, fib, ani, solid, therm, dT, form, plas, dmg;
    std::vector<uint32_t> mat, nbr;
    std::vector<vx_material> mats;
    vx_request_plan plan{};
    int state = 0;  // 0 queued, 1 resident, 2 finished
    uint32_t lane = 0;
    uint32_t slot = 0;
    vx_request_result res{};
    std::vector<double> final_pos;
    Clock::time_point submitted, admitted;

    vx_scene_desc desc() const {
        vx_scene_desc d{};
        d.n = n;
        d.position = pos.data();
        d.rotation = rot.empty() ? nullptr : rot.data();
        d.kinematic = kin.data();
        d.mass = mass.data();
        d.material = mat.data();
        d.materials = mats.data();
        d.material_count = (uint32_t)mats.size();
        d.fiber = fib.data();
        d.anisotropy = ani.data();
        d.solid_fraction = solid.empty() ? nullptr : solid.data();
        d.thermal_strength = therm.empty() ? nullptr : therm.data();
        d.thermal_delta = dT.empty() ? nullptr : dT.data();
        d.neighbor = nbr.data();
        d.formation_offset = form.empty() ? nullptr : form.data();
        d.plastic_strain = plas.empty() ? nullptr : plas.data();
        d.damage = dmg.empty() ? nullptr : dmg.data();
        return d;
    }
};

template <typename T>
std::vector<T> copy_of(const T* p, size_t count) {
    return p ? std::vector<T>(p, p + count) : std::vector<T>();
}

}  // namespace

// One pool with its own thread; its queue and slots are guarded by the
// server's mutex.
struct Lane {
    vx_pool* pool = nullptr;
    uint64_t max_scene_revs = 0;  // largest scene routed here (the last lane: no bound)
    uint64_t pool_revs = 0, pool_bytes = 0;
    uint32_t max_slots = 0;
    std::thread worker;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> slots;
};

struct vx_server {
    vx_ctx* ctx = nullptr;
    int device = 0;
    vx_server_config cfg{};
    uint64_t pool_revs = 0, pool_bytes = 0;
    std::vector<std::unique_ptr<Lane>> lanes;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
    uint64_t next_ticket = 1;
    // statistics (under mu)
    uint64_t submitted = 0, completed = 0, failed = 0, rounds = 0, scene_steps = 0, solves = 0;
    double busy_s = 0.0, worst_residual = 0.0;
    uint64_t not_converged = 0;
    std::vector<float> latency_ms;
    Clock::time_point start = Clock::now();

    void run(Lane& L);
    void finish(Lane& L, const std::shared_ptr<Request>& r, int32_t status, bool download);
};

// Ends a resident request: final positions, slot freed, waiter woken.
void vx_server::finish(Lane& L, const std::shared_ptr<Request>& r, int32_t status, bool download) {
    if (download && r->n) {
        r->final_pos.assign(3 * (size_t)r->n, 0.0);
        if (vx_pool_get_positions(L.pool, r->slot, r->final_pos.data()) != VX_OK && status == VX_OK)
            status = VX_CUDA_ERROR;
    }
    vx_pool_remove(L.pool, r->slot);
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> g(mu);
    L.slots[r->slot].reset();
    if (status == VX_OK && r->res.status != VX_OK) status = r->res.status;
    r->res.status = status;
    r->res.run_s = seconds(r->admitted, now);
    r->state = 2;
    if (status == VX_OK || status == VX_NOT_CONVERGED) ++completed;
    else ++failed;
    cv_done.notify_all();
}

void vx_server::run(Lane& L) {
    cudaSetDevice(device);
    const uint32_t S = L.max_slots;
    vx_pool* pool = L.pool;
    std::deque<std::shared_ptr<Request>>& queue = L.queue;
    std::vector<std::shared_ptr<Request>>& slots = L.slots;
    std::vector<uint8_t> enabled(S);
    std::vector<double> delta(3 * (size_t)S);
    std::vector<vx_step_stats> st(S);
    for (;;) {
        std::vector<std::shared_ptr<Request>> admit;
        {
            std::unique_lock<std::mutex> lk(mu);
            auto resident = [&] {
                return std::any_of(slots.begin(), slots.end(), [](const std::shared_ptr<Request>& p) { return (bool)p; });
            };
            while (!stop && queue.empty() && !resident()) cv_work.wait_for(lk, std::chrono::milliseconds(50));
            if (stop) return;
            size_t free_slots = std::count(slots.begin(), slots.end(), nullptr);
            while (!queue.empty() && admit.size() < free_slots) {
                admit.push_back(queue.front());
                queue.pop_front();
            }
        }
        // admission in arrival order; the first scene that does not fit ends it
        for (size_t k = 0; k < admit.size(); ++k) {
            const std::shared_ptr<Request>& r = admit[k];
            const vx_scene_desc d = r->desc();
            uint32_t slot = 0;
            int32_t st_add = vx_pool_add(pool, &d, &slot);
            if (st_add == VX_OOM) {
                std::lock_guard<std::mutex> g(mu);
                for (size_t j = admit.size(); j-- > k;) queue.push_front(admit[j]);
                break;
            }
            const bool added = st_add == VX_OK;
            if (added && !r->tmask.empty())
                st_add = vx_pool_set_targets(pool, slot, r->tmask.data(), r->target.empty() ? nullptr : r->target.data());
            if (st_add != VX_OK && added) vx_pool_remove(pool, slot);
            std::lock_guard<std::mutex> g(mu);
            if (st_add != VX_OK) {
                r->res.status = st_add;
                r->state = 2;
                ++failed;
                cv_done.notify_all();
                continue;
            }
            r->slot = slot;
            r->state = 1;
            r->admitted = Clock::now();
            r->res.queued_s = seconds(r->submitted, r->admitted);
            // host copies are no longer needed once the pool holds the scene
            r->pos = {};
            r->rot = {};
            r->nbr = {};
            slots[slot] = r;
        }
        std::vector<std::shared_ptr<Request>> res(S);
        {
            std::lock_guard<std::mutex> g(mu);
            res = slots;
        }
        bool any = false;
        for (uint32_t k = 0; k < S; ++k) {
            enabled[k] = res[k] ? 1 : 0;
            any = any || enabled[k];
            for (int a = 0; a < 3; ++a)
                delta[3 * (size_t)k + a] = res[k] ? res[k]->plan.target_velocity[a] * cfg.step.fixed_dt : 0.0;
        }
        if (!any) continue;
        const Clock::time_point t0 = Clock::now();
        int32_t rs = vx_pool_advance_targets(pool, enabled.data(), delta.data());
        if (rs == VX_OK || rs == VX_NOT_CONVERGED) rs = vx_pool_step(pool, enabled.data(), &cfg.step, st.data());
        const Clock::time_point t1 = Clock::now();
        const float ms = (float)(1000.0 * seconds(t0, t1));
        const bool fatal = !(rs == VX_OK || rs == VX_NOT_CONVERGED);
        std::vector<std::shared_ptr<Request>> done;
        {
            std::lock_guard<std::mutex> g(mu);
            ++rounds;
            busy_s += seconds(t0, t1);
            for (uint32_t k = 0; k < S; ++k) {
                const std::shared_ptr<Request>& r = res[k];
                if (!r) continue;
                if (fatal) {
                    done.push_back(r);
                    continue;
                }
                r->res.steps_done += 1;
                r->res.passes += st[k].passes;
                r->res.pcg_iterations += st[k].pcg_iterations;
                r->res.worst_residual = std::max(r->res.worst_residual, st[k].residual);
                if (!st[k].converged) {
                    r->res.status = VX_NOT_CONVERGED;
                    ++not_converged;
                }
                worst_residual = std::max(worst_residual, st[k].residual);
                ++scene_steps;
                solves += st[k].passes;
                latency_ms.push_back(ms);
                if (r->res.steps_done >= r->plan.steps) done.push_back(r);
            }
        }
        for (const auto& r : done) finish(L, r, fatal ? rs : VX_OK, !fatal);
    }
}

extern "C" {

int32_t vx_server_create(vx_ctx* ctx, const vx_server_config* cfg, vx_server** out) {
    vx::clear_error();
    if (!ctx || !cfg || !out || cfg->max_slots == 0) {
        vx::set_error("vx_server_create: null argument or zero slots");
        return VX_BAD_INPUT;
    }
    if (cfg->step.pass.precision != VX_PRECISION_MIXED || !(cfg->step.fixed_dt > 0.0) || cfg->step.substeps == 0 ||
        cfg->step.corotation_iterations == 0) {
        vx::set_error("vx_server_create: the step must be a VX_PRECISION_MIXED step with fixed_dt > 0");
        return VX_BAD_INPUT;
    }
    cudaSetDevice(ctx->device);
    uint64_t revs = cfg->max_revs;
    if (revs == 0) {
        if (!(cfg->hbm_fraction > 0.0 && cfg->hbm_fraction <= 1.0)) {
            vx::set_error("vx_server_create: hbm_fraction must be in (0, 1] when max_revs is 0");
            return VX_BAD_INPUT;
        }
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            vx::set_error("vx_server_create: cudaMemGetInfo failed");
            return VX_CUDA_ERROR;
        }
        const double budget = std::min(cfg->hbm_fraction * (double)total_b, 0.95 * (double)free_b);
        const uint64_t probe = 1ull << 20;
        double per_rev = (double)vx_pool_footprint_bytes(probe, cfg->max_slots) / (double)probe;
        // the contact stage's buffers scale with the pool's REV capacity too
        if (cfg->step.contact) per_rev += (double)vx::contact_state_bytes((uint32_t)probe) / (double)probe;
        revs = (uint64_t)(budget / per_rev) / 256 * 256;
        if (revs > 0x7FFFFF00ull) revs = 0x7FFFFF00ull;
    }
    // lanes: the REV budget and the slots split by scene size
    const uint32_t nl = std::min<uint32_t>(std::max<uint32_t>(cfg->lanes, 1u), 4u);
    const uint64_t default_bounds[3] = {1ull << 14, 1ull << 17, 1ull << 20};
    std::vector<uint64_t> bound(nl, ~0ull), lane_revs(nl, 0);
    std::vector<uint32_t> lane_slots(nl, cfg->max_slots / nl);
    lane_slots[nl - 1] += cfg->max_slots % nl;
    uint64_t given = 0;
    for (uint32_t k = 0; k + 1 < nl; ++k) {
        bound[k] = cfg->lane_max_revs[k] ? cfg->lane_max_revs[k] : default_bounds[k];
        if (lane_slots[k] == 0 || (k > 0 && bound[k] <= bound[k - 1])) {
            vx::set_error("vx_server_create: %u lanes need at least as many slots and increasing REV bounds", nl);
            return VX_BAD_INPUT;
        }
        // room for a full set of the lane's largest scenes, at most a quarter of the budget
        lane_revs[k] = std::min<uint64_t>((uint64_t)lane_slots[k] * ((bound[k] + 255) / 256 * 256), revs / 4) / 256 * 256;
        given += lane_revs[k];
    }
    if (given >= revs) {
        vx::set_error("vx_server_create: a pool of %llu REVs is too small for %u lanes", (unsigned long long)revs, nl);
        return VX_BAD_INPUT;
    }
    lane_revs[nl - 1] = (revs - given) / 256 * 256;
    vx_server* s = new (std::nothrow) vx_server();
    if (!s) return VX_OOM;
    s->ctx = ctx;
    s->device = ctx->device;
    s->cfg = *cfg;
    for (uint32_t k = 0; k < nl; ++k) {
        auto L = std::make_unique<Lane>();
        L->max_scene_revs = bound[k];
        L->max_slots = lane_slots[k];
        L->pool_revs = lane_revs[k];
        L->pool_bytes = vx_pool_footprint_bytes(lane_revs[k], lane_slots[k]);
        int32_t r = vx_pool_create(ctx, lane_revs[k], lane_slots[k], &L->pool);
        if (r == VX_OK && nl > 1) {
            // the lane of the smallest scenes runs first when the lanes share the GPU
            int least = 0, greatest = 0;
            cudaDeviceGetStreamPriorityRange(&least, &greatest);
            const int prio = std::max(greatest, std::min(least, greatest + (int)k * (least - greatest) / (int)(nl - 1)));
            r = vx::pool_stream_priority(L->pool, prio);
            if (r != VX_OK) vx_pool_destroy(L->pool);
        }
        if (r != VX_OK) {
            for (auto& M : s->lanes) vx_pool_destroy(M->pool);
            delete s;
            return r;
        }
        L->slots.assign(lane_slots[k], nullptr);
        s->pool_revs += L->pool_revs;
        s->pool_bytes += L->pool_bytes;
        s->lanes.push_back(std::move(L));
    }
    for (auto& L : s->lanes) {
        Lane* lp = L.get();
        L->worker = std::thread([s, lp] { s->run(*lp); });
    }
    *out = s;
    return VX_OK;
}

int32_t vx_server_submit(vx_server* s, const vx_scene_desc* d, const uint8_t* mask, const double* target,
                         const vx_request_plan* plan, uint64_t* out_ticket) {
    vx::clear_error();
    if (!s || !d || !plan || !out_ticket || plan->steps == 0 || d->n == 0 || !d->position || !d->kinematic ||
        !d->mass || !d->material || !d->materials || !d->fiber || !d->anisotropy || !d->neighbor) {
        vx::set_error("vx_server_submit: null argument, empty scene or zero steps");
        return VX_BAD_INPUT;
    }
    for (int a = 0; a < 3; ++a)
        if (!std::isfinite(plan->target_velocity[a])) {
            vx::set_error("vx_server_submit: non-finite target velocity");
            return VX_NONFINITE;
        }
    uint32_t lane = 0;
    while (lane + 1 < s->lanes.size() && d->n > s->lanes[lane]->max_scene_revs) ++lane;
    const uint64_t need = (d->n + 255ull) / 256 * 256;
    if (need > s->lanes[lane]->pool_revs) {
        vx::set_error("vx_server_submit: scene of %u REVs exceeds the capacity of its lane's pool, %llu REVs", d->n,
                      (unsigned long long)s->lanes[lane]->pool_revs);
        return VX_OOM;
    }
    auto r = std::make_shared<Request>();
    const size_t n = d->n;
    r->n = d->n;
    r->pos = copy_of(d->position, 3 * n);
    r->rot = copy_of(d->rotation, 4 * n);
    r->kin = copy_of(d->kinematic, n);
    r->mass = copy_of(d->mass, n);
    r->mat = copy_of(d->material, n);
    r->mats = copy_of(d->materials, d->material_count);
    r->fib = copy_of(d->fiber, 3 * n);
    r->ani = copy_of(d->anisotropy, n);
    r->solid = copy_of(d->solid_fraction, n);
    r->therm = copy_of(d->thermal_strength, n);
    r->dT = copy_of(d->thermal_delta, n);
    r->nbr = copy_of(d->neighbor, 3 * n);
    r->form = copy_of(d->formation_offset, 9 * n);
    r->plas = copy_of(d->plastic_strain, 9 * n);
    r->dmg = copy_of(d->damage, 3 * n);
    r->tmask = copy_of(mask, n);
    r->target = copy_of(target, 3 * n);
    r->plan = *plan;
    r->lane = lane;
    r->res.n = d->n;
    r->res.status = VX_OK;
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    r->ticket = s->next_ticket++;
    s->live[r->ticket] = r;
    s->lanes[lane]->queue.push_back(r);
    ++s->submitted;
    *out_ticket = r->ticket;
    s->cv_work.notify_all();
    return VX_OK;
}

int32_t vx_server_wait(vx_server* s, uint64_t ticket, double timeout_s, vx_request_result* out, double* positions) {
    vx::clear_error();
    if (!s) return VX_BAD_INPUT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
        vx::set_error("vx_server_wait: unknown ticket %llu", (unsigned long long)ticket);
        return VX_BAD_INPUT;
    }
    std::shared_ptr<Request> r = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(std::max(0.0, timeout_s)));
    while (r->state != 2)
        if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && r->state != 2) {
            vx::set_error("vx_server_wait: request %llu still %s", (unsigned long long)ticket,
                          r->state == 0 ? "queued" : "running");
            return VX_TIMEOUT;
        }
    if (out) *out = r->res;
    if (positions && !r->final_pos.empty()) std::memcpy(positions, r->final_pos.data(), r->final_pos.size() * 8);
    s->live.erase(it);
    return VX_OK;
}

int32_t vx_server_get_stats(vx_server* s, vx_server_stats* out) {
    vx::clear_error();
    if (!s || !out) return VX_BAD_INPUT;
    std::lock_guard<std::mutex> g(s->mu);
    vx_server_stats o{};
    o.submitted = s->submitted;
    o.completed = s->completed;
    o.failed = s->failed;
    for (const auto& L : s->lanes) {
        o.resident += (uint32_t)std::count_if(L->slots.begin(), L->slots.end(),
                                              [](const std::shared_ptr<Request>& p) { return (bool)p; });
        o.queued += (uint32_t)L->queue.size();
    }
    o.rounds = s->rounds;
    o.scene_steps = s->scene_steps;
    o.solves = s->solves;
    o.elapsed_s = seconds(s->start, Clock::now());
    o.busy_s = s->busy_s;
    if (!s->latency_ms.empty()) {
        std::vector<float> v = s->latency_ms;
        auto pct = [&](double q) {
            size_t k = (size_t)std::min<double>((double)v.size() - 1, std::floor(q * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return (double)v[k];
        };
        o.p50_step_ms = pct(0.50);
        o.p99_step_ms = pct(0.99);
        o.max_step_ms = *std::max_element(v.begin(), v.end());
    }
    o.pool_revs = s->pool_revs;
    o.pool_bytes = s->pool_bytes;
    o.worst_residual = s->worst_residual;
    o.not_converged = s->not_converged;
    *out = o;
    return VX_OK;
}

int32_t vx_server_destroy(vx_server* s) {
    if (!s) return VX_BAD_INPUT;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (auto& L : s->lanes)
        if (L->worker.joinable()) L->worker.join();
    for (auto& L : s->lanes)
        if (L->pool) vx_pool_destroy(L->pool);
    delete s;
    return VX_OK;
}

}  // extern "C"
