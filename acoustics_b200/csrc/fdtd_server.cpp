// fdtd_server.cpp — continuous batching of submitted solves on one GPU.
//
// Submitters (any host thread) append deep copies of their scenes to a queue.
// One worker thread owns an fdtd_batch and loops:
//   admit   while the queue head's device bytes fit the budget and a member
//           slot is free: hand it to the preparer thread, which creates its
//           solver (allocates, classifies, first step) beside the batched steps;
//   place   members the preparer has finished join the batch;
//   step    fdtd_batch_step(chunk) over all running members;
//   retire  finished members: copy their series out, release the slot and its
//           device bytes, wake waiters.
// Admission is in arrival order (no overtaking), so a large request at the
// head waits for memory instead of being starved by smaller ones.  With
// preemption on, a head that does not fit may evict running members with much
// more work left (their state and rows move to host memory, fdtd_batch_member_
// snapshot) and they queue again right behind it; re-admitted, they continue
// from the snapshot (fdtd_batch_add_snapshot).  A cancelled request leaves the
// queue, or its member is released after the chunk in progress.  Latency is
// measured on the host clock from submit to the retirement of the request.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

namespace {

using Clock = std::chrono::steady_clock;

// a scene with its arrays owned
struct SceneCopy {
    fdtd_scene_desc d{};
    std::vector<fdtd_object_desc> objs;
    std::vector<fdtd_plane_desc> planes;
    std::vector<fdtd_gaussian_source_desc> srcs;
    std::vector<double> lis;
    std::vector<fdtd_mesh_desc> meshes;
    std::vector<std::vector<double>> mverts;
    std::vector<std::vector<int32_t>> mtris;
    std::vector<fdtd_keyframe_track> tracks;
    std::vector<std::vector<double>> tframes;
    void take(const fdtd_scene_desc& s) {
        d = s;
        objs.assign(s.objects, s.objects + std::max(0, s.n_objects));
        planes.assign(s.constraints, s.constraints + std::max(0, s.n_constraints));
        srcs.assign(s.sources, s.sources + std::max(0, s.n_sources));
        lis.assign(s.listeners, s.listeners + 3 * (size_t)std::max(0, s.n_listeners));
        const int nm = s.meshes ? std::max(0, s.n_meshes) : 0;
        meshes.assign(s.meshes, s.meshes + nm);
        mverts.resize(nm);
        mtris.resize(nm);
        for (int m = 0; m < nm; ++m) {
            const fdtd_mesh_desc& M = s.meshes[m];
            mverts[m].assign(M.vertices, M.vertices + 3 * (size_t)std::max(0, M.n_vertices));
            mtris[m].assign(M.triangles, M.triangles + 3 * (size_t)std::max(0, M.n_triangles));
            meshes[m].vertices = mverts[m].data();
            meshes[m].triangles = mtris[m].data();
        }
        d.objects = objs.empty() ? nullptr : objs.data();
        d.constraints = planes.empty() ? nullptr : planes.data();
        d.sources = srcs.empty() ? nullptr : srcs.data();
        d.listeners = lis.empty() ? nullptr : lis.data();
        d.meshes = meshes.empty() ? nullptr : meshes.data();
        d.n_meshes = nm;
        const int nt = s.tracks ? std::max(0, s.n_tracks) : 0;
        tracks.assign(s.tracks, s.tracks + nt);
        tframes.resize(nt);
        for (int k = 0; k < nt; ++k) {
            const fdtd_keyframe_track& T = s.tracks[k];
            if (T.frames && T.n_frames > 0) tframes[k].assign(T.frames, T.frames + 7 * (size_t)T.n_frames);
            tracks[k].frames = tframes[k].empty() ? nullptr : tframes[k].data();
        }
        d.tracks = tracks.empty() ? nullptr : tracks.data();
        d.n_tracks = nt;
    }
};

struct Request {
    int64_t id = 0;
    SceneCopy scene;
    int32_t steps = 0;
    int64_t bytes = 0;
    double cells = 0;
    int32_t state = FDTD_REQ_QUEUED;
    int32_t status = FDTD_OK;
    int32_t member = -1;
    int64_t steps_done = 0;
    int32_t n_listeners = 0;
    std::vector<double> out;
    Clock::time_point t_submit, t_done;
    std::string err;
    bool cancel = false;            // cancellation asked while running
    std::vector<char> snap;         // evicted: the member's state ...
    std::vector<double> rows;       // ... and its listener rows so far
    int64_t evicted_steps = -1;     // steps done when evicted (-1: never)
    fdtd::PreparedMember prep;      // made by the preparer thread
    fdtd_status prep_status = FDTD_OK;
    std::string prep_err;
    bool in_prep = false;           // handed to the preparer, not yet placed (it reads snap and rows)
};

}  // namespace

struct fdtd_server {
    fdtd_options opt{};
    fdtd_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::map<int32_t, int64_t> running;  // member -> request
    int64_t next_id = 1;
    int64_t used_bytes = 0;
    bool stop = false;
    std::thread worker;
    std::thread preparer;
    std::condition_variable cv_prep;
    std::deque<int64_t> to_prepare;      // admitted, waiting for the preparer
    std::vector<int64_t> prepared;       // made, waiting to join the batch
    int64_t preparing = 0;               // admitted and not yet placed
    fdtd_batch* batch = nullptr;
    std::string create_err;
    bool ready = false, failed_start = false;
    // statistics
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, evictions = 0, peak_members = 0, peak_bytes = 0;
    std::vector<double> latencies;
    double cell_steps_done = 0;
    bool have_first = false;
    Clock::time_point t_first, t_last;
};

namespace {

void finish(fdtd_server* S, Request& r, int32_t state, int32_t status, const std::string& err) {
    r.state = state;
    r.status = status;
    r.err = err;
    r.t_done = Clock::now();
    if (state == FDTD_REQ_DONE) {
        S->completed++;
        S->latencies.push_back(std::chrono::duration<double>(r.t_done - r.t_submit).count());
        S->cell_steps_done += r.cells * r.steps;
        S->t_last = r.t_done;
    } else if (state == FDTD_REQ_CANCELLED) {
        S->cancelled++;
    } else {
        S->failed++;
    }
    if (!r.in_prep) {  // (the worker drops them when the preparer is done with them)
        r.snap.clear();
        r.snap.shrink_to_fit();
        r.rows.clear();
        r.rows.shrink_to_fit();
    }
}

// Members to evict so that `need` more bytes fit: running members whose
// remaining cell-steps exceed twice the head's, most remaining work first.
// Returns an empty list when evicting them all would not make room.  (Lock held.)
std::vector<int32_t> eviction_plan(fdtd_server* S, const Request& head) {
    std::vector<std::pair<double, int32_t>> cand;
    for (const auto& mr : S->running) {
        const Request& r = *S->reqs[mr.second];
        if (r.cancel) continue;
        const double left = r.cells * (double)(r.steps - r.steps_done);
        if (left > 2.0 * head.cells * head.steps) cand.push_back({left, mr.first});
    }
    std::sort(cand.begin(), cand.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<int32_t> out;
    int64_t used = S->used_bytes;
    for (const auto& c : cand) {
        if (used + head.bytes <= S->cfg.hbm_budget_bytes) break;
        out.push_back(c.second);
        used -= S->reqs[S->running[c.second]]->bytes;
    }
    if (used + head.bytes > S->cfg.hbm_budget_bytes) out.clear();
    return out;
}

// Move member m to host memory and queue its request again behind the head.
void evict(fdtd_server* S, int32_t m) {
    int64_t id;
    {
        std::lock_guard<std::mutex> g(S->mu);
        id = S->running[m];
    }
    Request* r = S->reqs[id].get();  // the worker owns running requests' members
    int64_t done = 0, total = 0, bytes = 0;
    int32_t nl = 0, mst = 0;
    fdtd_status st = fdtd_batch_member_info(S->batch, m, &done, &total, &nl, &mst);
    std::vector<double> rows((size_t)done * nl);
    std::vector<char> snap;
    if (st == FDTD_OK && mst == FDTD_OK && !rows.empty()) st = fdtd_batch_output(S->batch, m, rows.data(), (int64_t)rows.size());
    if (st == FDTD_OK && mst == FDTD_OK) st = fdtd_batch_member_snapshot(S->batch, m, nullptr, &bytes);
    if (st == FDTD_OK && mst == FDTD_OK) {
        snap.resize((size_t)bytes);
        st = fdtd_batch_member_snapshot(S->batch, m, snap.data(), &bytes);
    }
    const std::string err = st != FDTD_OK ? fdtd_last_error() : "";
    fdtd_batch_release(S->batch, m);
    std::lock_guard<std::mutex> g(S->mu);
    S->running.erase(m);
    S->used_bytes -= r->bytes;
    r->member = -1;
    if (st != FDTD_OK || mst != FDTD_OK) {
        finish(S, *r, FDTD_REQ_FAILED, st != FDTD_OK ? st : mst, err.empty() ? "device-side error flag set" : err);
        S->cv_done.notify_all();
        return;
    }
    r->snap.swap(snap);
    r->rows.swap(rows);
    r->steps_done = done;
    r->evicted_steps = done;
    r->state = FDTD_REQ_QUEUED;
    S->queue.insert(S->queue.empty() ? S->queue.end() : S->queue.begin() + 1, id);
    S->evictions++;
}

// Members are made on this thread while the worker steps the batch: a
// request's solver creation and first step no longer stall every running solve.
void preparer_main(fdtd_server* S) {
    cudaSetDevice(S->opt.device);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_prep.wait(lk, [&] { return S->stop || !S->to_prepare.empty(); });
            if (S->stop) return;
            r = S->reqs[S->to_prepare.front()].get();
            S->to_prepare.pop_front();
        }
        // the request's scene and snapshot are not touched by other threads meanwhile
        fdtd::PreparedMember pm;
        std::string err;
        const bool resumed = r->evicted_steps >= 0;
        const fdtd_status st =
            fdtd::batch_prepare(S->opt, &r->scene.d, r->steps, resumed ? r->snap.data() : nullptr,
                                resumed ? (int64_t)r->snap.size() : 0, resumed && !r->rows.empty() ? r->rows.data() : nullptr,
                                resumed ? r->evicted_steps : 0, &pm, &err);
        std::lock_guard<std::mutex> g(S->mu);
        r->prep = std::move(pm);
        r->prep_status = st;
        r->prep_err = err;
        S->prepared.push_back(r->id);
        S->cv_work.notify_all();
    }
}

// The queue head can be handed to the preparer now.  (Lock held.)
bool admissible(const fdtd_server* S) {
    if (S->queue.empty() || (int64_t)S->running.size() + S->preparing >= S->cfg.max_members) return false;
    const Request& r = *S->reqs.at(S->queue.front());
    return S->used_bytes + r.bytes <= S->cfg.hbm_budget_bytes;
}

void worker_main(fdtd_server* S) {
    cudaSetDevice(S->opt.device);
    {
        fdtd_batch* b = nullptr;
        fdtd_status st = fdtd_batch_create(0, nullptr, nullptr, &S->opt, &b);
        std::lock_guard<std::mutex> g(S->mu);
        if (st != FDTD_OK) {
            S->create_err = fdtd_last_error();
            S->failed_start = true;
        } else {
            S->batch = b;
        }
        S->ready = true;
        S->cv_done.notify_all();
        if (st != FDTD_OK) return;
    }
    const int chunk = S->cfg.chunk_steps > 0 ? S->cfg.chunk_steps : std::max(S->opt.graph_steps, 32);
    for (;;) {
        // ---- admit: queue heads go to the preparer ----
        std::vector<int64_t> place;
        std::vector<int32_t> victims;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || !S->prepared.empty() || !S->running.empty() || admissible(S); });
            if (S->stop) break;
            bool handed = false;
            while (admissible(S)) {
                const int64_t id = S->queue.front();
                S->queue.pop_front();
                S->used_bytes += S->reqs[id]->bytes;
                S->reqs[id]->in_prep = true;
                S->preparing++;
                S->to_prepare.push_back(id);
                handed = true;
            }
            if (handed) S->cv_prep.notify_one();
            S->peak_bytes = std::max(S->peak_bytes, S->used_bytes);
            // a head that does not fit: evict only when nothing is on its way in
            if (S->cfg.preempt && !S->queue.empty() && S->preparing == 0 && S->prepared.empty() &&
                S->used_bytes + S->reqs[S->queue.front()]->bytes > S->cfg.hbm_budget_bytes)
                victims = eviction_plan(S, *S->reqs[S->queue.front()]);
            place.swap(S->prepared);
        }
        if (!victims.empty()) {
            for (int32_t m : victims) evict(S, m);
            continue;  // admit the head now
        }
        // ---- place the members the preparer made ----
        for (int64_t id : place) {
            std::lock_guard<std::mutex> g(S->mu);
            Request* r = S->reqs[id].get();
            S->preparing--;
            r->in_prep = false;
            if (r->state == FDTD_REQ_CANCELLED) {  // cancelled while it was being prepared
                if (r->prep.s) fdtd_solver_destroy(r->prep.s);
                r->prep.s = nullptr;
                S->used_bytes -= r->bytes;
                r->snap.clear();
                r->snap.shrink_to_fit();
                r->rows.clear();
                r->rows.shrink_to_fit();
                continue;
            }
            if (r->prep_status != FDTD_OK) {
                S->used_bytes -= r->bytes;
                finish(S, *r, FDTD_REQ_FAILED, r->prep_status, r->prep_err);
                S->cv_done.notify_all();
                continue;
            }
            const int32_t m = fdtd::batch_place(S->batch, std::move(r->prep));
            r->snap.clear();
            r->snap.shrink_to_fit();
            r->rows.clear();
            r->rows.shrink_to_fit();
            r->member = m;
            r->state = FDTD_REQ_RUNNING;
            r->n_listeners = r->scene.d.n_listeners;
            S->running[m] = r->id;
            S->peak_members = std::max<int64_t>(S->peak_members, (int64_t)S->running.size());
        }
        // ---- step ----
        bool any_running;
        {
            std::lock_guard<std::mutex> g(S->mu);
            any_running = !S->running.empty();
        }
        if (!any_running) continue;
        int32_t n_active = 0;
        fdtd_status st = fdtd_batch_step(S->batch, chunk, &n_active);
        // ---- retire ----
        std::vector<std::pair<int32_t, int64_t>> members;
        {
            std::lock_guard<std::mutex> g(S->mu);
            members.assign(S->running.begin(), S->running.end());
        }
        for (auto& mr : members) {
            int64_t done = 0, total = 0;
            int32_t nl = 0, mst = 0;
            fdtd_batch_member_info(S->batch, mr.first, &done, &total, &nl, &mst);
            bool cancelled;
            {
                std::lock_guard<std::mutex> g(S->mu);
                cancelled = S->reqs[mr.second]->cancel;
            }
            if (cancelled) {
                fdtd_batch_release(S->batch, mr.first);
                std::lock_guard<std::mutex> g(S->mu);
                Request& r = *S->reqs[mr.second];
                r.steps_done = done;
                S->running.erase(mr.first);
                S->used_bytes -= r.bytes;
                finish(S, r, FDTD_REQ_CANCELLED, FDTD_ERR_CANCELLED, "request cancelled");
                S->cv_done.notify_all();
                continue;
            }
            const bool ok = st == FDTD_OK && mst == FDTD_OK;
            const bool finished = !ok || done >= total;
            std::vector<double> out;
            if (finished) {
                if (ok) {
                    out.resize((size_t)done * nl);
                    fdtd_batch_output(S->batch, mr.first, out.data(), (int64_t)out.size());
                }
                fdtd_batch_release(S->batch, mr.first);  // also stops a member that failed mid-run
            }
            std::lock_guard<std::mutex> g(S->mu);
            Request& r = *S->reqs[mr.second];
            r.steps_done = done;
            if (!finished) continue;
            S->running.erase(mr.first);
            S->used_bytes -= r.bytes;
            if (st != FDTD_OK) finish(S, r, FDTD_REQ_FAILED, st, fdtd_last_error());
            else if (mst != FDTD_OK) finish(S, r, FDTD_REQ_FAILED, mst, "device-side error flag set");
            else {
                r.out.swap(out);
                finish(S, r, FDTD_REQ_DONE, FDTD_OK, "");
            }
            S->cv_done.notify_all();
        }
        if (st != FDTD_OK) {
            // the batch is in an unknown state: fail every queued request and stop
            std::lock_guard<std::mutex> g(S->mu);
            for (int64_t id : S->queue) finish(S, *S->reqs[id], FDTD_REQ_FAILED, st, "server stopped after a failed step");
            S->queue.clear();
            S->stop = true;
            S->cv_prep.notify_all();
            S->cv_done.notify_all();
            break;
        }
    }
}

Request* find(fdtd_server* S, int64_t id) {
    auto it = S->reqs.find(id);
    return it == S->reqs.end() ? nullptr : it->second.get();
}

double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

fdtd_status fdtd_server_create(const fdtd_options* options, const fdtd_server_config* config, fdtd_server** out) {
    if (!out) return FDTD_ERR_INVALID_ARG;
    *out = nullptr;
    std::unique_ptr<fdtd_server> S(new fdtd_server());
    if (options) S->opt = *options;
    if (config) S->cfg = *config;
    if (S->cfg.max_members <= 0) S->cfg.max_members = 256;
    if (S->cfg.hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(S->opt.device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            fdtd::set_error(nullptr, "fdtd_server_create: no CUDA device");
            return FDTD_ERR_CUDA;
        }
        S->cfg.hbm_budget_bytes = (int64_t)(0.9 * (double)fr);
    }
    fdtd_server* raw = S.get();
    S->worker = std::thread(worker_main, raw);
    S->preparer = std::thread(preparer_main, raw);
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [&] { return S->ready; });
    }
    if (S->failed_start) {
        S->worker.join();
        {
            std::lock_guard<std::mutex> g(S->mu);
            S->stop = true;
            S->cv_prep.notify_all();
        }
        S->preparer.join();
        fdtd::set_error(nullptr, S->create_err);
        return FDTD_ERR_CUDA;
    }
    *out = S.release();
    return FDTD_OK;
}

fdtd_status fdtd_server_submit(fdtd_server* S, const fdtd_scene_desc* scene, int32_t steps, int64_t* request) {
    if (!S || !scene || steps < 1) return (fdtd::set_error(nullptr, "fdtd_server_submit: invalid arguments"), FDTD_ERR_INVALID_ARG);
    const int64_t bytes = fdtd_scene_device_bytes(scene, &S->opt);
    if (bytes < 0) return FDTD_ERR_INVALID_ARG;
    if (bytes > S->cfg.hbm_budget_bytes) {
        fdtd::set_error(nullptr, "scene needs " + std::to_string(bytes) + " device bytes, more than the budget");
        return FDTD_ERR_INVALID_ARG;
    }
    std::unique_ptr<Request> r(new Request());
    r->scene.take(*scene);
    r->steps = steps;
    r->bytes = bytes;
    r->cells = (double)scene->divisions[0] * scene->divisions[1] * scene->divisions[2];
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) return (fdtd::set_error(nullptr, "server stopped"), FDTD_ERR_BUSY);
    r->id = S->next_id++;
    if (!S->have_first) {
        S->have_first = true;
        S->t_first = r->t_submit;
    }
    if (request) *request = r->id;
    S->queue.push_back(r->id);
    S->reqs[r->id] = std::move(r);
    S->submitted++;
    S->cv_work.notify_all();
    return FDTD_OK;
}

fdtd_status fdtd_server_poll(fdtd_server* S, int64_t id, int32_t* state, int64_t* steps_done, int32_t* status) {
    if (!S) return FDTD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    Request* r = find(S, id);
    if (!r) return (fdtd::set_error(nullptr, "unknown request"), FDTD_ERR_INVALID_ARG);
    if (state) *state = r->state;
    if (steps_done) *steps_done = r->steps_done;
    if (status) *status = r->status;
    return FDTD_OK;
}

fdtd_status fdtd_server_wait(fdtd_server* S, int64_t id, double timeout_s) {
    if (!S) return FDTD_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    if (!find(S, id)) return (fdtd::set_error(nullptr, "unknown request"), FDTD_ERR_INVALID_ARG);
    auto pred = [&] {
        Request* r = find(S, id);
        return !r || r->state == FDTD_REQ_DONE || r->state == FDTD_REQ_FAILED || r->state == FDTD_REQ_CANCELLED;
    };
    if (timeout_s < 0) S->cv_done.wait(lk, pred);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return (fdtd::set_error(nullptr, "wait timed out"), FDTD_ERR_TIMEOUT);
    Request* r = find(S, id);
    return r && (r->state == FDTD_REQ_FAILED || r->state == FDTD_REQ_CANCELLED) ? r->status : FDTD_OK;
}

fdtd_status fdtd_server_result(fdtd_server* S, int64_t id, double* out, int64_t count, int64_t* steps,
                               int32_t* n_listeners, double* latency_s) {
    if (!S) return FDTD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    Request* r = find(S, id);
    if (!r) return (fdtd::set_error(nullptr, "unknown request"), FDTD_ERR_INVALID_ARG);
    if (r->state == FDTD_REQ_FAILED || r->state == FDTD_REQ_CANCELLED) {
        fdtd::set_error(nullptr, r->err);
        return r->status;
    }
    if (r->state != FDTD_REQ_DONE) return (fdtd::set_error(nullptr, "request not finished"), FDTD_ERR_BUSY);
    if (steps) *steps = r->steps_done;
    if (n_listeners) *n_listeners = r->n_listeners;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (!out) return FDTD_OK;  // size query
    if (count < (int64_t)r->out.size())
        return (fdtd::set_error(nullptr, "output buffer too small"), FDTD_ERR_INVALID_ARG);
    if (!r->out.empty()) std::memcpy(out, r->out.data(), r->out.size() * sizeof(double));
    S->reqs.erase(id);
    return FDTD_OK;
}

fdtd_status fdtd_server_drain(fdtd_server* S, double timeout_s) {
    if (!S) return FDTD_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto pred = [&] { return S->stop || (S->queue.empty() && S->running.empty()); };
    if (timeout_s < 0) S->cv_done.wait(lk, pred);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return (fdtd::set_error(nullptr, "drain timed out"), FDTD_ERR_TIMEOUT);
    return FDTD_OK;
}

fdtd_status fdtd_server_stats_get(fdtd_server* S, fdtd_server_stats* st) {
    if (!S || !st) return FDTD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->failed = S->failed;
    st->queued = (int64_t)S->queue.size();
    st->running = (int64_t)S->running.size();
    st->peak_members = S->peak_members;
    st->peak_device_bytes = S->peak_bytes;
    st->device_bytes_in_use = S->used_bytes;
    st->cancelled = S->cancelled;
    st->evictions = S->evictions;
    st->p50_latency_s = pct(S->latencies, 0.50);
    st->p99_latency_s = pct(S->latencies, 0.99);
    double sum = 0;
    for (double v : S->latencies) sum += v;
    st->mean_latency_s = S->latencies.empty() ? 0.0 : sum / S->latencies.size();
    if (S->completed > 0) {
        st->span_s = std::chrono::duration<double>(S->t_last - S->t_first).count();
        if (st->span_s > 0) {
            st->solves_per_s = S->completed / st->span_s;
            st->cell_steps_per_s = S->cell_steps_done / st->span_s;
        }
    }
    return FDTD_OK;
}

fdtd_status fdtd_server_cancel(fdtd_server* S, int64_t id) {
    if (!S) return FDTD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    Request* r = find(S, id);
    if (!r) return (fdtd::set_error(nullptr, "unknown request"), FDTD_ERR_INVALID_ARG);
    if (r->state == FDTD_REQ_QUEUED) {
        auto it = std::find(S->queue.begin(), S->queue.end(), id);
        if (it != S->queue.end()) S->queue.erase(it);
        finish(S, *r, FDTD_REQ_CANCELLED, FDTD_ERR_CANCELLED, "request cancelled");
        S->cv_done.notify_all();
        S->cv_work.notify_all();
        return FDTD_OK;
    }
    if (r->state == FDTD_REQ_RUNNING) {
        r->cancel = true;  // the worker releases the member after the chunk in progress
        S->cv_work.notify_all();
        return FDTD_OK;
    }
    return (fdtd::set_error(nullptr, "request already finished"), FDTD_ERR_INVALID_ARG);
}

const char* fdtd_server_request_error(fdtd_server* S, int64_t id) {
    if (!S) return "";
    std::lock_guard<std::mutex> g(S->mu);
    Request* r = find(S, id);
    return r ? r->err.c_str() : "";
}

fdtd_status fdtd_server_destroy(fdtd_server* S) {
    if (!S) return FDTD_OK;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
        S->cv_prep.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    if (S->preparer.joinable()) S->preparer.join();
    // members made but never placed
    for (auto& kv : S->reqs)
        if (kv.second->prep.s) {
            fdtd_solver_destroy(kv.second->prep.s);
            kv.second->prep.s = nullptr;
        }
    if (S->batch) {
        cudaSetDevice(S->opt.device);
        fdtd_batch_destroy(S->batch);
    }
    delete S;
    return FDTD_OK;
}

}  // extern "C"
