// Commitment server: continuous batching of MSM requests over resident base
// tables (one per curve); and a pool of such servers, one per GPU, that
// routes whole requests to replicas by queue depth and free HBM.
//
// The reference has no concurrent or persistent batching: its "async" batch
// runs MSMs one after another (Sources/zkMetal/MSM/MultiMSM.swift:175-238).
// Here a request (curve, n scalars over a prefix of that curve's table) is
// queued by zkmsm_server_submit.  W worker threads each own an Engine (its
// own CUDA stream and resident scratch).  A free worker takes the oldest
// pending request's curve and admits, in arrival order, every pending
// request of that curve that fits the batch limits and the HBM budget, runs
// them as one batch, and hands the results back.  Requests that arrive while
// batches are on the GPU wait only for the next free worker, and batches of
// different workers overlap on the device.  Admission charges each request
// an estimate of the device memory it needs; a request larger than the whole
// budget is refused with ZKMETAL_ERR_BUSY at submit time.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <unordered_map>

#include "../../include/zkmsm.h"
#include "engine.cuh"

namespace zkmsm {


namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    int curve;
    int fmt;
    uint32_t n;
    const uint8_t* scalars;  // caller keeps it valid until the request completes
    uint64_t bytes;          // admission charge
    Clock::time_point t_submit, t_start, t_done;
    int status = 1;          // 1 pending, 2 running, 0 done ok, < 0 error
    uint8_t result[3 * 48];
};

// batches of at most this many points run on a worker's high-priority stream
constexpr uint64_t SMALL_BATCH_POINTS = 1ull << 20;

struct Server {
    TableView tables[2];
    bool has_table[2] = {false, false};
    uint64_t budget, in_use = 0;
    uint64_t max_batch_points;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> all;
    std::atomic<uint64_t> next_id{1};
    bool stop = false;
    std::vector<std::thread> workers;
    // points of requests submitted and not yet finished (pending or running):
    // the queue depth a replica pool routes by
    uint64_t queued_points = 0;
    // stats
    uint64_t batches = 0, completed = 0, failed = 0, max_batch = 0;
    std::vector<double> latencies_ms;
    int device = 0;
    const Clock::time_point t_created = Clock::now();
    // host-side fault injection for tests: fail the next k batches
    std::atomic<int> inject_failures{0};

    static uint64_t estimate(int curve, uint32_t n) {
        // scalars + sorted entries (2 halves x up to 8 windows x 8 B) + buckets
        // and partial sums; generous so admission errs on the safe side
        const uint64_t per_point = 32 + 2 * 8 * 8 + (curve == ZKMSM_BN254 ? 64 : 96);
        return (uint64_t)n * per_point + (64ull << 20);
    }

    void worker_main(int w) {
        cudaSetDevice(device);
        std::unique_ptr<Engine> eng;
        try {
            eng.reset(new Engine());
        } catch (...) {
            return;
        }
        uint32_t* d_scalars = nullptr;
        size_t d_cap = 0;
        // Size the workspace now for the batch shapes that set its high-water
        // marks (full-table requests up to the batch limit; sizes doubling
        // from 2^10 points to the table size, repeated up to the limit), so
        // that serving rarely has to grow it: a growth while the other
        // workers' batches ran has held up every batch on the device, once
        // for 3.5 s.
        try {
            for (int c = 0; c < 2; c++) {
                if (!has_table[c]) continue;
                const TableView& tv = tables[c];
                const uint64_t T = std::min<uint64_t>(tv.n, max_batch_points), M = max_batch_points;
                std::vector<std::vector<uint32_t>> shapes(2);
                for (uint64_t s = 0; T && s + T <= M; s += T) shapes[0].push_back((uint32_t)T);
                for (uint64_t s = 0, added = 1; added && T;) {
                    added = 0;
                    for (uint64_t n = std::min<uint64_t>(1024, T); n <= T && s + n <= M; n *= 2, added++) {
                        shapes[1].push_back((uint32_t)n);
                        s += n;
                    }
                }
                for (auto& counts : shapes) {
                    if (counts.empty()) continue;
                    std::vector<uint32_t> boffs(counts.size(), 0);
                    if (c == 0)
                        eng->ensure_workspace<Bn254>(eng->transient_plan<Bn254>(counts, boffs, 1, tv.shifts));
                    else
                        eng->ensure_workspace<Bls381>(eng->transient_plan<Bls381>(counts, boffs, 1, tv.shifts));
                }
            }
            const uint64_t want = max_batch_points * 36;
            if (cudaMallocAsync(reinterpret_cast<void**>(&d_scalars), want, eng->stream) == cudaSuccess) d_cap = want;
            else d_scalars = nullptr;
            cudaStreamSynchronize(eng->stream);
        } catch (...) {
        }
        cudaGetLastError();
        // small batches run on a high-priority stream: their blocks get SMs
        // as soon as blocks of other workers' large batches finish, instead
        // of queueing behind whole kernels
        cudaStream_t own = eng->stream, hi = nullptr;
        {
            int lo_pri = 0, hi_pri = 0;
            if (cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri) != cudaSuccess ||
                cudaStreamCreateWithPriority(&hi, cudaStreamNonBlocking, hi_pri) != cudaSuccess) {
                cudaGetLastError();
                hi = nullptr;
            }
        }
        for (;;) {
            std::vector<std::shared_ptr<Request>> batch;
            uint64_t charged = 0;
            int curve = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !pending.empty(); });
                if (stop && pending.empty()) break;
                curve = pending.front()->curve;
                const int fmt0 = pending.front()->fmt;
                uint64_t pts = 0;
                for (auto it = pending.begin(); it != pending.end();) {
                    auto& r = *it;
                    if (r->curve != curve || r->fmt != fmt0) {
                        ++it;
                        continue;
                    }
                    bool first = batch.empty();
                    bool fits_mem = in_use + charged + r->bytes <= budget;
                    bool fits_pts = pts + r->n <= max_batch_points;
                    // the oldest request runs once memory frees up; later ones only if they fit
                    if (!(fits_mem && (fits_pts || first))) {
                        if (first) break;  // wait for memory
                        ++it;
                        continue;
                    }
                    pts += r->n;
                    charged += r->bytes;
                    r->status = 2;
                    r->t_start = Clock::now();
                    batch.push_back(r);
                    it = pending.erase(it);
                }
                if (batch.empty()) {
                    // nothing admissible now: wait for a completion to release memory
                    cv_done.wait_for(lk, std::chrono::milliseconds(5));
                    continue;
                }
                in_use += charged;
            }
            // run the batch outside the lock
            int st = ZKMETAL_SUCCESS;
            std::vector<uint8_t> out;
#ifdef ZKMSM_SERVER_TRACE
            const auto t_b0 = Clock::now();
#endif
            try {
                if (inject_failures.load() > 0 && inject_failures.fetch_sub(1) > 0)
                    throw std::runtime_error("injected batch failure");
                const TableView& tv = tables[curve];
                std::vector<uint32_t> counts, boffs;
                uint64_t total = 0;
                for (auto& r : batch) {
                    counts.push_back(r->n);
                    boffs.push_back(0);
                    total += r->n;
                }
                // the previous batch has completed on whichever stream it used
                eng->stream = (hi && total <= SMALL_BATCH_POINTS) ? hi : own;
                if (total * 32 > d_cap) {  // grows geometrically, in stream order (no device-wide wait)
                    const uint64_t want = std::max<uint64_t>(total * 36, d_cap + d_cap / 2);
                    if (d_scalars) ZK_CUDA(cudaFreeAsync(d_scalars, eng->stream));
                    d_scalars = nullptr;
                    d_cap = 0;
                    ZK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_scalars), want, eng->stream));
                    d_cap = want;
                }
                // one host-to-device copy per request into the batch's scalar array
                uint64_t off = 0;
                int fmt = batch[0]->fmt;
                for (auto& r : batch) {
                    ZK_CUDA(cudaMemcpyAsync(reinterpret_cast<uint8_t*>(d_scalars) + off * 32, r->scalars,
                                            (size_t)r->n * 32, cudaMemcpyHostToDevice, eng->stream));
                    off += r->n;
                    if (r->fmt != fmt) fmt = -1;
                }
                if (fmt < 0) throw std::runtime_error("mixed scalar formats in one batch");
                int fb = curve == ZKMSM_BN254 ? 32 : 48;
                out.resize(batch.size() * 3 * fb);
                if (curve == ZKMSM_BN254) {
                    Plan& pl = eng->transient_plan<Bn254>(counts, boffs, fmt, tv.shifts);
                    eng->run_device<Bn254>(pl, tv.points, tv.phi, d_scalars, out.data());
                } else {
                    Plan& pl = eng->transient_plan<Bls381>(counts, boffs, fmt, tv.shifts);
                    eng->run_device<Bls381>(pl, tv.points, tv.phi, d_scalars, out.data());
                }
                for (size_t i = 0; i < batch.size(); i++) memcpy(batch[i]->result, out.data() + i * 3 * fb, 3 * fb);
#ifdef ZKMSM_SERVER_TRACE
                {
                    const auto t_b1 = Clock::now();
                    double oldest = 0;
                    for (auto& r : batch)
                        oldest = std::max(oldest, std::chrono::duration<double, std::milli>(t_b0 - r->t_submit).count());
                    const DevBuf* ws[] = {&eng->w_counts, &eng->w_cursor, &eng->w_ents, &eng->w_ents2,
                                          &eng->w_thist, &eng->w_buckets, &eng->w_cnt, &eng->w_pkeys[0],
                                          &eng->w_pkeys[1], &eng->w_pvals[0], &eng->w_pvals[1], &eng->w_redS[0],
                                          &eng->w_redS[1], &eng->w_redW[0], &eng->w_redW[1], &eng->w_tiles};
                    uint64_t wsb = d_cap;
                    for (const DevBuf* b : ws) wsb += b->cap;
                    uint64_t pool_res = 0, pool_used = 0;
                    cudaMemPool_t pool;
                    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
                        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &pool_res);
                        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &pool_used);
                    }
                    fprintf(stderr,
                            "trace t %.3f worker %d curve %d reqs %zu points %llu run %.2f ms oldest wait %.2f ms "
                            "growths %llu ws_mb %llu pool_res_mb %llu pool_used_mb %llu\n",
                            std::chrono::duration<double>(t_b0 - t_created).count(), w, curve,
                            batch.size(), (unsigned long long)total,
                            std::chrono::duration<double, std::milli>(t_b1 - t_b0).count(), oldest,
                            (unsigned long long)eng->workspace_growths, (unsigned long long)(wsb >> 20),
                            (unsigned long long)(pool_res >> 20), (unsigned long long)(pool_used >> 20));
                }
#endif
            } catch (const CudaError& e) {
                set_error(std::string("server batch: ") + e.where + ": " + cudaGetErrorString(e.code));
                cudaGetLastError();
                st = ZKMETAL_ERR_GPU_ERROR;
            } catch (const std::exception& e) {
                set_error(std::string("server batch: ") + e.what());
                st = ZKMETAL_ERR_GPU_ERROR;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                auto now = Clock::now();
                for (auto& r : batch) {
                    r->t_done = now;
                    r->status = st;
                    queued_points -= r->n;
                    if (st == ZKMETAL_SUCCESS) {
                        completed++;
                        latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
                    } else {
                        failed++;
                    }
                }
                in_use -= charged;
                batches++;
                max_batch = std::max<uint64_t>(max_batch, batch.size());
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        eng->stream = own;
        if (d_scalars) cudaFree(d_scalars);
        if (hi) cudaStreamDestroy(hi);
        (void)w;
    }
};

// A pool of servers, one per GPU (each with its own resident tables): whole
// requests are routed to one replica, with no collective and no data moving
// between GPUs.
struct Pool {
    std::vector<Server*> reps;
    std::mutex mu;
    std::unordered_map<uint64_t, std::pair<uint32_t, uint64_t>> ids;  // pool id -> (replica, server id)
    uint64_t next_id = 1;
    std::vector<uint64_t> routed;
    uint32_t rr = 0;  // first replica of the tie order, advanced per request
};

}  // namespace
}  // namespace zkmsm

using namespace zkmsm;

extern "C" {

int zkmsm_route_pick(const ZkMsmReplicaLoad* loads, uint32_t n_replicas, uint32_t request_points,
                     uint64_t request_bytes, uint32_t first) {
    if (!loads || n_replicas == 0) return -1;
    int best = -1;
    bool best_room = false;
    double best_depth = 0;
    uint64_t best_free = 0;
    // replicas in cyclic order from `first`: on a full tie the earliest wins,
    // so a caller that advances `first` spreads ties over the replicas
    for (uint32_t k = 0; k < n_replicas; k++) {
        const uint32_t i = (first + k) % n_replicas;
        const ZkMsmReplicaLoad& l = loads[i];
        if (!l.has_table || request_points > l.table_points || request_bytes > l.budget_bytes) continue;
        const double speed = l.relative_speed > 0 ? l.relative_speed : 1.0;
        const double depth = (double)(l.queued_points + request_points) / speed;
        const uint64_t free_b = l.budget_bytes > l.in_use_bytes ? l.budget_bytes - l.in_use_bytes : 0;
        const bool room = free_b >= request_bytes;
        // a replica with room for the request now beats one without; then the
        // shallower queue (in points, scaled by speed); between replicas that
        // all lack room, equal queues go to the one with more free memory
        bool better = best < 0 || (room && !best_room) ||
                      (room == best_room &&
                       (depth < best_depth || (depth == best_depth && !room && free_b > best_free)));
        if (better) {
            best = (int)i;
            best_room = room;
            best_depth = depth;
            best_free = free_b;
        }
    }
    return best;
}

ZkMetalStatus zkmsm_pool_create(const ZkMsmServer* servers, uint32_t n_servers, ZkMsmPool* out) {
    if (!servers || !out || n_servers == 0 || n_servers > 64) return ZKMETAL_ERR_INVALID_INPUT;
    std::unique_ptr<Pool> p(new Pool());
    for (uint32_t i = 0; i < n_servers; i++) {
        if (!servers[i]) return ZKMETAL_ERR_INVALID_INPUT;
        p->reps.push_back(static_cast<Server*>(servers[i]));
    }
    p->routed.assign(n_servers, 0);
    *out = p.release();
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_pool_submit(ZkMsmPool pool, int curve, const void* scalars, int scalar_fmt, uint32_t n_points,
                                uint64_t* request_id) {
    if (!pool || !request_id || (curve != ZKMSM_BN254 && curve != ZKMSM_BLS12_381)) return ZKMETAL_ERR_INVALID_INPUT;
    Pool& p = *static_cast<Pool*>(pool);
    const uint32_t R = (uint32_t)p.reps.size();
    std::vector<ZkMsmReplicaLoad> loads(R);
    for (uint32_t i = 0; i < R; i++) {
        Server& s = *p.reps[i];
        std::lock_guard<std::mutex> lk(s.mu);
        loads[i].has_table = s.has_table[curve] ? 1 : 0;
        loads[i].table_points = s.has_table[curve] ? s.tables[curve].n : 0;
        loads[i].queued_points = s.queued_points;
        loads[i].budget_bytes = s.budget;
        loads[i].in_use_bytes = s.in_use;
        loads[i].relative_speed = 1.0;
    }
    const uint64_t bytes = Server::estimate(curve, n_points);
    uint32_t first;
    {
        std::lock_guard<std::mutex> lk(p.mu);
        first = p.rr++ % R;
    }
    // the best replica first; on refusal (e.g. the budget changed) the next best
    for (uint32_t tries = 0; tries < R; tries++) {
        const int pick = zkmsm_route_pick(loads.data(), R, n_points, bytes, first);
        if (pick < 0) break;
        uint64_t sid = 0;
        const ZkMetalStatus st = zkmsm_server_submit(p.reps[pick], curve, scalars, scalar_fmt, n_points, &sid);
        if (st == ZKMETAL_SUCCESS) {
            std::lock_guard<std::mutex> lk(p.mu);
            const uint64_t id = p.next_id++;
            p.ids[id] = {(uint32_t)pick, sid};
            p.routed[pick]++;
            *request_id = id;
            return ZKMETAL_SUCCESS;
        }
        if (st != ZKMETAL_ERR_BUSY) return st;
        loads[pick].has_table = 0;
    }
    set_error("no replica can take the request (no table for the curve, table too short, or over every budget)");
    return ZKMETAL_ERR_BUSY;
}

ZkMetalStatus zkmsm_pool_wait(ZkMsmPool pool, uint64_t request_id, int timeout_ms, uint8_t* result,
                              double* latency_ms) {
    if (!pool) return ZKMETAL_ERR_INVALID_INPUT;
    Pool& p = *static_cast<Pool*>(pool);
    std::pair<uint32_t, uint64_t> where;
    {
        std::lock_guard<std::mutex> lk(p.mu);
        auto it = p.ids.find(request_id);
        if (it == p.ids.end()) return ZKMETAL_ERR_INVALID_INPUT;
        where = it->second;
    }
    const ZkMetalStatus st = zkmsm_server_wait(p.reps[where.first], where.second, timeout_ms, result, latency_ms);
    if (st != ZKMETAL_ERR_BUSY || timeout_ms < 0) {
        std::lock_guard<std::mutex> lk(p.mu);
        p.ids.erase(request_id);
    }
    return st;
}

ZkMetalStatus zkmsm_pool_stats(ZkMsmPool pool, char* buf, uint64_t buflen) {
    if (!pool || !buf || !buflen) return ZKMETAL_ERR_INVALID_INPUT;
    Pool& p = *static_cast<Pool*>(pool);
    std::string js = "{\"replicas\":[";
    for (size_t i = 0; i < p.reps.size(); i++) {
        char tmp[1024];
        if (zkmsm_server_stats(p.reps[i], tmp, sizeof tmp) != ZKMETAL_SUCCESS) return ZKMETAL_ERR_INVALID_INPUT;
        uint64_t routed;
        {
            std::lock_guard<std::mutex> lk(p.mu);
            routed = p.routed[i];
        }
        std::string one(tmp);
        one.insert(1, "\"routed\":" + std::to_string(routed) + ",\"device\":" + std::to_string(p.reps[i]->device) +
                              ",");
        js += (i ? "," : "") + one;
    }
    js += "]}";
    if (js.size() + 1 > buflen) return ZKMETAL_ERR_INVALID_INPUT;
    memcpy(buf, js.c_str(), js.size() + 1);
    return ZKMETAL_SUCCESS;
}

void zkmsm_pool_destroy(ZkMsmPool pool) { delete static_cast<Pool*>(pool); }

ZkMetalStatus zkmsm_server_create(ZkMsmTable bn254_table, ZkMsmTable bls12_381_table, uint64_t hbm_budget_bytes,
                                  int workers, uint64_t max_batch_points, ZkMsmServer* out) {
    if (!out || (!bn254_table && !bls12_381_table) || workers < 1 || workers > 16) return ZKMETAL_ERR_INVALID_INPUT;
    std::unique_ptr<Server> s(new Server());
    if (bn254_table) {
        if (!table_view(bn254_table, &s->tables[0]) || s->tables[0].curve != ZKMSM_BN254)
            return ZKMETAL_ERR_INVALID_INPUT;
        s->has_table[0] = true;
    }
    if (bls12_381_table) {
        if (!table_view(bls12_381_table, &s->tables[1]) || s->tables[1].curve != ZKMSM_BLS12_381)
            return ZKMETAL_ERR_INVALID_INPUT;
        s->has_table[1] = true;
    }
    cudaGetDevice(&s->device);
    s->max_batch_points = max_batch_points ? max_batch_points : (1ull << 24);
    // Reserve workspace memory in the device's memory pool.  Engines grow
    // their workspaces through the stream-ordered allocator; a growth that
    // has to map new physical memory (gigabytes for a large batch of many
    // medium MSMs) held up the other workers' batches for a few hundred
    // milliseconds.  Memory reserved once and kept by the pool is handed out
    // without mapping.  A worker's workspace for a full batch of small and
    // medium MSMs over window-shift tables (one sorted entry per window per
    // point, two entry arrays, scalars) reaches about 480 B per batch point.
    {
        size_t fr = 0, tot = 0;
        cudaMemPool_t pool;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
            const uint64_t want =
                    std::min<uint64_t>((uint64_t)workers * s->max_batch_points * 512 + (1ull << 30), fr / 4);
            uint64_t thr = 0;
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            if (thr < want) {
                thr = want;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            }
            void* p = nullptr;
            if (cudaMallocAsync(&p, want, 0) == cudaSuccess) {
                cudaFreeAsync(p, 0);
                cudaStreamSynchronize(0);
            }
        }
        cudaGetLastError();
    }
    if (hbm_budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return ZKMETAL_ERR_GPU_ERROR;
        hbm_budget_bytes = fr / 10 * 7;  // leave room for the engines' own growth
    }
    s->budget = hbm_budget_bytes;
    Server* sp = s.get();
    for (int w = 0; w < workers; w++) s->workers.emplace_back([sp, w] { sp->worker_main(w); });
    *out = s.release();
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_server_submit(ZkMsmServer server, int curve, const void* scalars, int scalar_fmt,
                                  uint32_t n_points, uint64_t* request_id) {
    if (!server || !scalars || !request_id || n_points == 0) return ZKMETAL_ERR_INVALID_INPUT;
    if (curve != ZKMSM_BN254 && curve != ZKMSM_BLS12_381) return ZKMETAL_ERR_INVALID_INPUT;
    if (scalar_fmt != ZKMSM_SCALAR_INT && scalar_fmt != ZKMSM_SCALAR_MONT) return ZKMETAL_ERR_INVALID_INPUT;
    Server& s = *static_cast<Server*>(server);
    if (!s.has_table[curve] || n_points > s.tables[curve].n) return ZKMETAL_ERR_INVALID_INPUT;
    auto r = std::make_shared<Request>();
    r->curve = curve;
    r->fmt = scalar_fmt;
    r->n = n_points;
    r->scalars = static_cast<const uint8_t*>(scalars);
    r->bytes = Server::estimate(curve, n_points);
    if (r->bytes > s.budget) {
        set_error("request needs more device memory than the server's budget");
        return ZKMETAL_ERR_BUSY;
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s.mu);
        if (s.stop) return ZKMETAL_ERR_BUSY;
        r->id = s.next_id++;
        s.all[r->id] = r;
        s.pending.push_back(r);
        s.queued_points += n_points;
    }
    s.cv_work.notify_one();
    *request_id = r->id;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_server_cancel(ZkMsmServer server, uint64_t request_id) {
    if (!server) return ZKMETAL_ERR_INVALID_INPUT;
    Server& s = *static_cast<Server*>(server);
    std::lock_guard<std::mutex> lk(s.mu);
    auto it = s.all.find(request_id);
    if (it == s.all.end()) return ZKMETAL_ERR_INVALID_INPUT;
    auto& r = it->second;
    if (r->status != 1) return ZKMETAL_ERR_BUSY;  // already running or done
    s.pending.erase(std::remove(s.pending.begin(), s.pending.end(), r), s.pending.end());
    s.queued_points -= r->n;
    r->status = ZKMETAL_ERR_BUSY;
    r->t_done = Clock::now();
    s.cv_done.notify_all();
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_server_wait(ZkMsmServer server, uint64_t request_id, int timeout_ms, uint8_t* result,
                                double* latency_ms) {
    if (!server) return ZKMETAL_ERR_INVALID_INPUT;
    Server& s = *static_cast<Server*>(server);
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.all.find(request_id);
    if (it == s.all.end()) return ZKMETAL_ERR_INVALID_INPUT;
    auto r = it->second;
    auto done = [&] { return r->status <= 0; };
    if (timeout_ms < 0) s.cv_done.wait(lk, done);
    else if (!s.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return ZKMETAL_ERR_BUSY;
    int st = r->status;
    if (st == ZKMETAL_SUCCESS && result) memcpy(result, r->result, 3 * (r->curve == ZKMSM_BN254 ? 32 : 48));
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    s.all.erase(it);
    return st;
}

ZkMetalStatus zkmsm_server_stats(ZkMsmServer server, char* buf, uint64_t buflen) {
    if (!server || !buf || !buflen) return ZKMETAL_ERR_INVALID_INPUT;
    Server& s = *static_cast<Server*>(server);
    std::lock_guard<std::mutex> lk(s.mu);
    std::vector<double> v = s.latencies_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
    char tmp[512];
    snprintf(tmp, sizeof tmp,
             "{\"completed\":%llu,\"failed\":%llu,\"batches\":%llu,\"max_batch\":%llu,\"pending\":%zu,"
             "\"p50_ms\":%.3f,\"p99_ms\":%.3f,\"max_ms\":%.3f,\"budget_bytes\":%llu,\"in_use_bytes\":%llu}",
             (unsigned long long)s.completed, (unsigned long long)s.failed, (unsigned long long)s.batches,
             (unsigned long long)s.max_batch, s.pending.size(), pct(0.5), pct(0.99), v.empty() ? 0.0 : v.back(),
             (unsigned long long)s.budget, (unsigned long long)s.in_use);
    size_t k = std::min<size_t>(strlen(tmp), buflen - 1);
    memcpy(buf, tmp, k);
    buf[k] = 0;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_server_inject_failures(ZkMsmServer server, int batches) {
    if (!server || batches < 0) return ZKMETAL_ERR_INVALID_INPUT;
    static_cast<Server*>(server)->inject_failures.store(batches);
    return ZKMETAL_SUCCESS;
}

void zkmsm_server_destroy(ZkMsmServer server) {
    if (!server) return;
    Server* s = static_cast<Server*>(server);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    delete s;
}

}  // extern "C"
