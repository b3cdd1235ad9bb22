// Serving loop over a multi-scene batch: requests (scene + substep count)
// are admitted in arrival order while their device footprint fits, advanced
// together, and retired as soon as their own substep count is reached.
// Included at the end of slosh_b200.cu after batch.cuh.
//
// Footprint accounting.  The batch is allocated once from the HBM budget:
// 70 % as particle pool (280 bytes a particle: two copies of the 128-byte
// particle state and of the original-index plane, the sort key, the
// permutation and the cell slot) and up to 30 % as block
// capacity (8756 bytes a block: hash slots, per-cell counts, cursors and order,
// neighbour ranks, the P2G partial tile, nodes and the collision caches).  A
// request's footprint is n * 280 + blocks * 8756 with blocks estimated as
// 2.5 n / 512 + 64 (8 particles per cell fill 512 per block; the factor
// covers the +1 neighbour blocks and partly filled blocks).  Admission needs
// the pool's free particles, the estimated blocks and a free scene slot.
//
// Steps.  A batched step advances every in-flight scene by the smallest
// remaining substep count (at most tick_substeps), so every request gets
// exactly its own number of substeps and leaves the batch right after its
// last one.  Admission has two phases: while a tick runs on the GPU, queued
// requests are staged (their records copied into the batch's upload
// buffer); between ticks the staged scenes are activated (converted into
// the pool) and join the next tick.
#pragma once

#include <condition_variable>
#include <deque>
#include <thread>

struct slosh_server {
    slosh_server_config cfg{};
    slosh_batch *batch = nullptr;
    uint32_t pool_particles = 0, pool_blocks = 0;
    uint64_t pool_bytes = 0;
    struct Req {
        uint64_t id = 0;
        slosh_request r{};
        double submit_s = 0, admit_s = 0;
        uint32_t slot = 0, remaining = 0, blocks = 0;
        uint64_t bytes = 0;
    };
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv, idle_cv;
    bool stop = false;
    std::deque<Req> queue;
    std::vector<Req> staging;  // staged in the batch, joining at the next activation
    std::vector<Req> flight;
    std::deque<slosh_completion> done;
    uint64_t next_id = 1, submitted = 0, admitted = 0, completed = 0, work = 0, in_flight_bytes = 0;
    uint32_t blocks_in_flight = 0, max_seen = 0;
    double busy = 0.0;
    std::tuple<int, uint32_t, int> tuned_key{-1, 0u, -1};  // the mix the launch shape was tuned for
    slosh_tuning tuning{};  // the batch's launch shape, copied under the lock after tuning
    std::chrono::steady_clock::time_point t0;
    std::string last_error;
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

constexpr uint64_t POOL_BYTES_PER_PARTICLE = 280;
constexpr uint64_t POOL_BYTES_PER_BLOCK = 8756;
constexpr uint32_t AUTOTUNE_SUBSTEPS = 20;  // 10 candidates x (1 warm-up + 1 timed)

uint32_t request_blocks(uint32_t n) { return (uint32_t)(2.5 * (double)n / 512.0) + 64u; }

void retire(slosh_server *s, slosh_server::Req &q, int status, uint32_t done_substeps) {
    slosh_completion c{};
    c.id = q.id;
    c.status = status;
    c.n = q.r.n;
    c.substeps = done_substeps;
    c.submit_s = q.submit_s;
    c.admit_s = q.admit_s;
    c.done_s = s->now();
    s->done.push_back(c);
    s->completed += 1;
    s->in_flight_bytes -= q.bytes;
    s->blocks_in_flight -= q.blocks;
}

// Stages queued requests, in arrival order, while they fit.  Called both
// between ticks and while a tick runs: staging only copies records into the
// batch's upload buffer.
void stage_pending(slosh_server *s, std::unique_lock<std::mutex> &lk) {
    slosh_batch *b = s->batch;
    while (!s->queue.empty()) {
        const slosh_server::Req &q = s->queue.front();
        uint32_t free_slots = 0;
        for (const auto &sl : b->slots) free_slots += sl.used ? 0u : 1u;
        const size_t active = s->flight.size() + s->staging.size();
        const bool fits = (s->cfg.max_in_flight == 0 || active < s->cfg.max_in_flight) && free_slots > 0 &&
                          (uint64_t)b->n_storage + b->staged_n + q.r.n <= s->pool_particles &&
                          (uint64_t)b->up_used + q.r.n <= b->up_cap &&
                          (uint64_t)s->blocks_in_flight + q.blocks <= s->pool_blocks;
        if (!fits) return;
        slosh_server::Req r = q;
        s->queue.pop_front();
        lk.unlock();
        uint32_t slot = 0;
        RecordScan scan;
        int st = batch_validate(b, &r.r.desc, r.r.particles, r.r.n, r.r.bodies, r.r.n_bodies, scan);
        if (st == SLOSH_OK)
            st = batch_stage(b, &r.r.desc, r.r.particles, r.r.n, r.r.bodies, r.r.n_bodies, scan, &slot);
        lk.lock();
        s->admitted += 1;
        s->in_flight_bytes += r.bytes;
        s->blocks_in_flight += r.blocks;
        r.admit_s = s->now();
        if (st != SLOSH_OK) {
            s->last_error = b->c.last_error;
            retire(s, r, st, 0);
            continue;
        }
        r.slot = slot;
        r.remaining = r.r.substeps;
        s->staging.push_back(r);
    }
}

void server_loop(slosh_server *s) {
    cudaSetDevice(s->cfg.device);
    slosh_batch *b = s->batch;
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        stage_pending(s, lk);
        if (s->flight.empty() && s->staging.empty()) {
            if (!b->dropped.empty()) {
                // retired scenes hold pool space and slots until a substep compacts them
                lk.unlock();
                slosh_batch_step(b, 1, nullptr);
                slosh_batch_sync(b, nullptr);
                lk.lock();
                continue;
            }
            if (s->queue.empty()) s->idle_cv.notify_all();
            s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            continue;
        }
        // activation: the staged scenes join the batch (no tick in flight)
        if (!s->staging.empty()) {
            lk.unlock();
            const int st = batch_activate(b, b->c.stream);
            lk.lock();
            for (auto &r : s->staging) {
                if (st == SLOSH_OK) {
                    s->flight.push_back(r);
                } else {
                    s->last_error = b->c.last_error;
                    retire(s, r, st, 0);
                }
            }
            s->staging.clear();
            s->max_seen = std::max<uint32_t>(s->max_seen, (uint32_t)s->flight.size());
            if (s->flight.empty()) continue;
        }
        uint32_t tick = std::max<uint32_t>(s->cfg.tick_substeps, 1u);
        for (const auto &r : s->flight) tick = std::min(tick, r.remaining);
        // the launch shape is tuned again whenever the in-flight mix moves to
        // another (dim, material mix, particle-count bucket): a bucket seen
        // before takes its cached shape at once
        const auto mix = tune_key(b);
        const bool tune = s->cfg.autotune && tick >= AUTOTUNE_SUBSTEPS && mix != s->tuned_key;
        lk.unlock();
        const double ta = s->now();
        int st = SLOSH_OK;
        uint32_t ran = 0;
        if (tune) {
            // times each launch shape on real substeps of the in-flight
            // scenes (or applies a cached shape without stepping)
            st = batch_autotune(b, 1, nullptr, &ran);
        }
        if (st == SLOSH_OK && ran == 0) st = slosh_batch_step(b, tick, nullptr);
        else if (ran) tick = ran;
        lk.lock();
        // while the tick runs on the GPU: copy the next requests' records up
        if (st == SLOSH_OK) stage_pending(s, lk);
        lk.unlock();
        if (st == SLOSH_OK) st = slosh_batch_sync(b, nullptr);
        const double tb = s->now();
        lk.lock();
        if (tune) {
            s->tuned_key = mix;
            s->tuning = b->tune;
        }
        s->busy += tb - ta;
        if (st != SLOSH_OK) {
            s->last_error = b->c.last_error;
            for (auto &r : s->flight) {
                retire(s, r, st, r.r.substeps - r.remaining);
                lk.unlock();
                slosh_batch_remove_scene(b, r.slot);
                lk.lock();
            }
            s->flight.clear();
            continue;
        }
        for (auto &r : s->flight) {
            r.remaining -= tick;
            s->work += (uint64_t)r.r.n * tick;
        }
        for (size_t k = 0; k < s->flight.size();) {
            slosh_server::Req &r = s->flight[k];
            if (r.remaining != 0) {
                ++k;
                continue;
            }
            lk.unlock();
            int st2 = r.r.out_positions
                          ? slosh_batch_download_positions(b, r.slot, r.r.out_positions, r.r.n, nullptr)
                          : SLOSH_OK;
            const int st3 = slosh_batch_remove_scene(b, r.slot);
            if (st2 == SLOSH_OK) st2 = st3;
            lk.lock();
            retire(s, r, st2, r.r.substeps);
            s->flight.erase(s->flight.begin() + (long)k);
        }
        if (s->flight.empty() && s->queue.empty() && s->staging.empty() && b->dropped.empty())
            s->idle_cv.notify_all();
    }
}

}  // namespace

extern "C" {

int slosh_server_create(const slosh_server_config *cfg, slosh_server **out) {
    if (!cfg || !out) return SLOSH_E_INVALID;
    *out = nullptr;
    if ((cfg->dim != 2 && cfg->dim != 3) || cfg->hbm_budget_bytes < (64ull << 20) || cfg->max_scenes == 0 ||
        cfg->max_scenes > MAX_SCENES)
        return SLOSH_E_INVALID;
    slosh_server *s = new slosh_server();
    s->cfg = *cfg;
    const double budget = (double)cfg->hbm_budget_bytes;
    // upload buffer for staged records: a quarter of the pool, at most 4 M records
    const double pool0 = std::min<double>(0.7 * budget / POOL_BYTES_PER_PARTICLE, 2147483648.0);
    const uint32_t up_records = (uint32_t)std::min<double>(pool0 / 4.0, 4194304.0);
    s->pool_particles = (uint32_t)((0.7 * budget - (double)up_records * sizeof(slosh_particle)) /
                                   POOL_BYTES_PER_PARTICLE);
    uint32_t blocks = 1;
    while ((double)blocks * 2.0 * POOL_BYTES_PER_BLOCK <= 0.3 * budget && blocks < (1u << 24)) blocks <<= 1;
    s->pool_blocks = blocks;
    s->pool_bytes = (uint64_t)s->pool_particles * POOL_BYTES_PER_PARTICLE + (uint64_t)blocks * POOL_BYTES_PER_BLOCK +
                    (uint64_t)up_records * sizeof(slosh_particle);
    slosh_batch_config bc{};
    bc.dim = cfg->dim;
    bc.max_particles = s->pool_particles;
    bc.grid_capacity = s->pool_blocks;
    bc.max_scenes = cfg->max_scenes;
    bc.max_bodies = std::max<uint32_t>(cfg->max_bodies, 16u);
    bc.device = cfg->device;
    int st = slosh_batch_create(&bc, &s->batch);
    if (st == SLOSH_OK) st = batch_reserve_upload(s->batch, up_records);
    if (st == SLOSH_OK) {
        // downloads of completed scenes go through the batch's record staging
        slosh_ctx *c = &s->batch->c;
        st = dalloc(c, &c->staging, up_records);
        if (st == SLOSH_OK) s->batch->staging_cap = up_records;
    }
    if (st != SLOSH_OK) {
        if (s->batch) slosh_batch_destroy(s->batch);
        delete s;
        return st;
    }
    s->tuning = s->batch->tune;
    s->t0 = std::chrono::steady_clock::now();
    s->worker = std::thread(server_loop, s);
    *out = s;
    return SLOSH_OK;
}

void slosh_server_destroy(slosh_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    slosh_batch_destroy(s->batch);
    delete s;
}

int slosh_server_submit(slosh_server *s, const slosh_request *req, uint64_t *id) {
    if (!s || !req || !req->particles || req->n == 0 || (!req->bodies && req->n_bodies)) return SLOSH_E_INVALID;
    slosh_server::Req q;
    q.r = *req;
    q.blocks = request_blocks(req->n);
    q.bytes = (uint64_t)req->n * POOL_BYTES_PER_PARTICLE + (uint64_t)q.blocks * POOL_BYTES_PER_BLOCK;
    std::lock_guard<std::mutex> lk(s->mu);
    if (req->n > s->pool_particles || q.blocks > s->pool_blocks || req->n > s->batch->up_cap) {
        s->last_error = "request larger than the budget's particle pool or block capacity";
        return SLOSH_E_CAPACITY;
    }
    q.id = s->next_id++;
    q.submit_s = s->now();
    s->queue.push_back(q);
    s->submitted += 1;
    if (id) *id = q.id;
    s->cv.notify_one();
    return SLOSH_OK;
}

int slosh_server_poll(slosh_server *s, slosh_completion *out, uint32_t cap, uint32_t *n_out) {
    if (!s || (!out && cap) || !n_out) return SLOSH_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    uint32_t k = 0;
    while (k < cap && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n_out = k;
    return SLOSH_OK;
}

int slosh_server_wait_idle(slosh_server *s, double timeout_s) {
    if (!s) return SLOSH_E_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->idle_cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                        [&] { return s->queue.empty() && s->flight.empty() && s->staging.empty(); });
    if (!ok) {
        s->last_error = "timeout waiting for the queue to drain";
        return SLOSH_E_STATE;
    }
    return SLOSH_OK;
}

int slosh_server_get_stats(slosh_server *s, slosh_server_stats *out) {
    if (!s || !out) return SLOSH_E_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->particle_substeps = s->work;
    out->in_flight_bytes = s->in_flight_bytes;
    out->pool_bytes = s->pool_bytes;
    out->busy_s = s->busy;
    out->now_s = s->now();
    out->in_flight = (uint32_t)(s->flight.size() + s->staging.size());
    out->queued = (uint32_t)s->queue.size();
    out->max_in_flight_seen = s->max_seen;
    out->tuning = s->tuning;
    return SLOSH_OK;
}

int slosh_server_last_error(const slosh_server *s, char *buf, size_t len) {
    if (!s || !buf || len == 0) return SLOSH_E_INVALID;
    std::snprintf(buf, len, "%s", s->last_error.c_str());
    return SLOSH_OK;
}

}  // extern "C"
