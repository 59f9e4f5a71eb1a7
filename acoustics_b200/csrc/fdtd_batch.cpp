// fdtd_batch.cpp — many independent static solves stepped together.
//
// Each member is a complete fdtd_solver (own device arrays, classification,
// ghost list, sources, listeners).  Its first step runs through the solver's
// own path (it classifies the cells); afterwards every step of all active
// members is one call of launch_batch_*: shell and interior kernels over tile
// tables of all members, then batched ghost-list, source, listener
// and advance kernels (fdtd_batch.cuh).  Members finish at their own step
// counts and leave the tables; a captured graph of graph_steps batched steps is
// replayed while the membership is unchanged.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_device.cuh"
#include "fdtd_internal.hpp"
#include "fdtd_launch.hpp"

using namespace fdtd;

namespace fdtd {
void build_shell_boxes(fdtd_solver* s, int xs);
int shell_planes(const fdtd_solver* s, int tile_y);
}

namespace {

struct Member {
    fdtd_solver* s = nullptr;
    int64_t total = 0;
    int64_t done = 0;
    bool active = false;
    bool released = false;  // slot free for a later fdtd_batch_add
    fdtd_status status = FDTD_OK;
    int L = 0;
    std::vector<double> rows;
    int64_t tiles = 0;      // interior + shell tiles of the member in the current tables
};

}  // namespace

struct fdtd_batch {
    fdtd_options opt{};
    int precision = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr, stream3 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_ghost = nullptr;
    // listener rows of a step run on stream4 beside the next step; the advance of
    // the next step (and with it every later kernel) waits on ev_lis[table of the step]
    cudaStream_t stream4 = nullptr;
    cudaEvent_t ev_step = nullptr, ev_lis[2] = {nullptr, nullptr}, ev_lis_join = nullptr;
    bool lis_pending[2] = {false, false};
    // the interior arguments in the kernel's parameter bank, one table per step
    // parity (BatchIntParams<T>); empty when more members have interior tiles
    // than the table holds (the tile table path then)
    std::vector<char> int_params[2];
    int int_ctas = 0;
    std::vector<Member> members;
    // device tables
    void* d_descs = nullptr;
    size_t desc_cap = 0;
    BatchTile* d_int = nullptr;
    size_t int_cap = 0;
    BatchTile* d_shell = nullptr;
    size_t shell_cap = 0;
    ListenerRef* d_refs = nullptr;
    size_t refs_cap = 0;
    BatchLaunch L{};
    size_t table_bytes = 0;  // one descriptor table (the second, at this offset, has every parity flipped)
    int flip = 0;            // table of the next step
    bool dirty = true;
    int64_t table_tiles = 0;  // tiles in the current tables (finished members' included until the next rebuild)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // G steps starting at table 0 / 1
    long long launches = 0, last_launches = 0, graph_launches = 0;
    std::string err;
};

namespace {

fdtd_status batch_fail(fdtd_batch* b, fdtd_status st, const std::string& m) {
    fdtd::set_error(nullptr, m);
    if (b) b->err = m;
    return st;
}

fdtd_status batch_cuda_fail(fdtd_batch* b, cudaError_t e, const char* what) {
    return batch_fail(b, e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA,
                      std::string("CUDA: ") + cudaGetErrorString(e) + " at " + what);
}

}  // namespace

#define BATCH_TRY(b, expr)                                             \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) return batch_cuda_fail((b), _e, #expr); \
    } while (0)

namespace {

template <typename T>
void fill_desc(BatchDesc<T>& d, fdtd_solver* s, bool active, int64_t total, bool halted) {
    std::memset(&d, 0, sizeof(d));
    d.a[0] = make_kargs<T>(s->dP, s->hP, 0);
    d.a[1] = make_kargs<T>(s->dP, s->hP, 1);
    d.P = s->dP;
    d.interior = s->region.interior;
    d.src_region = s->region.src_region;
    d.shell = s->shell;
    d.ring = s->d_lis;
    d.ring_cap = s->lis_cap_steps;
    d.n_lis = s->L;
    d.cur = s->cur;
    d.active = active ? 1 : 0;
    d.has_src = s->hP.n_src > 0 ? 1 : 0;
    d.ghost_cap = s->region.ghost_cap;
    d.total = total;
    d.halted = halted ? 1 : 0;
}

template <typename T>
size_t desc_bytes() {
    return sizeof(BatchDesc<T>);
}

template <typename T>
fdtd_status grow(fdtd_batch* b, T** ptr, size_t* cap, size_t need) {
    if (need <= *cap) return FDTD_OK;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    const size_t n = std::max<size_t>(need, 64);
    BATCH_TRY(b, cudaMalloc((void**)ptr, n * sizeof(T)));
    *cap = n;
    return FDTD_OK;
}

// Interior entries of the parameter-bank table: (descriptor index, unit tiles, x tiles).
struct IntEntry {
    int m, tu, tx;
};

template <typename T>
int fill_int_params(std::vector<char>& buf, const char* table, size_t dsz, const std::vector<IntEntry>& list) {
    buf.assign(sizeof(BatchIntParams<T>), 0);
    BatchIntParams<T>& P = *reinterpret_cast<BatchIntParams<T>*>(buf.data());
    P.n = (int)list.size();
    int ctas = 0;
    for (size_t i = 0; i < list.size(); ++i) {
        const BatchDesc<T>& d = *reinterpret_cast<const BatchDesc<T>*>(table + (size_t)list[i].m * dsz);
        const KArgs<T>& A = d.a[d.cur];
        BatchIntMember<T>& M = P.m[i];
        M.pc = A.pc;
        M.pn = A.pn;
        M.dinc = A.dinc;
        M.cls = A.cls;
        M.sx = A.sx;
        M.sy = A.sy;
        M.c2k2 = A.c2k2;
        M.lap_scale = A.lap_scale;
        M.kcalp = A.kcalp;
        M.box = d.interior;
        M.tu = list[i].tu;
        M.member = list[i].m;
        P.first[i] = ctas;
        ctas += list[i].tu * list[i].tx;
    }
    P.first[list.size()] = ctas;
    return ctas;
}

// Rebuild descriptors and tile tables after a membership change.
fdtd_status rebuild(fdtd_batch* b) {
    const bool f64 = b->precision == FDTD_PRECISION_FP64;
    const int xb = (b->opt.x_chunk == 4 || b->opt.x_chunk == 8) ? b->opt.x_chunk : 2;
    const int xs = b->opt.tile_y > 0 ? std::min(b->opt.tile_y, 256) : FDTD_SHELL_PLANES;
    const size_t dsz = f64 ? desc_bytes<double>() : desc_bytes<float>();
    const size_t nm = b->members.size();
    const size_t tbytes = std::max<size_t>(nm, 1) * dsz;
    std::vector<char> descs(2 * tbytes, 0);
    std::vector<BatchTile> it, st, st_full;
    std::vector<IntEntry> int_list;
    std::vector<ListenerRef> refs;
    int max_ghost = 0, max_src = 0, max_solid = 0;
    for (size_t m = 0; m < nm; ++m) {
        Member& mb = b->members[m];
        if (!mb.s) continue;
        const int xs_m = shell_planes(mb.s, b->opt.tile_y);
        if (mb.s->shell.xs != xs_m) build_shell_boxes(mb.s, xs_m);
        mb.s->region.shell = mb.s->shell;
        for (int par = 0; par < 2; ++par) {
            char* dst = &descs[par * tbytes + m * dsz];
            if (f64) {
                fill_desc<double>(*reinterpret_cast<BatchDesc<double>*>(dst), mb.s, mb.active, mb.total, mb.done >= mb.total);
                reinterpret_cast<BatchDesc<double>*>(dst)->cur ^= par;
            } else {
                fill_desc<float>(*reinterpret_cast<BatchDesc<float>*>(dst), mb.s, mb.active, mb.total, mb.done >= mb.total);
                reinterpret_cast<BatchDesc<float>*>(dst)->cur ^= par;
            }
        }
        mb.tiles = 0;
        if (!mb.active) continue;
        const size_t tiles0 = it.size() + st.size() + st_full.size();
        const Box3& I = mb.s->region.interior;
        const int nx = I.hi[0] - I.lo[0], ny = I.hi[1] - I.lo[1], nz = I.hi[2] - I.lo[2];
        if (nx > 0 && ny > 0 && nz > 0) {
            const int tu = interior_unit_tiles(I, f64 ? 2 : 4), tx = (nx + xb - 1) / xb;
            for (int x = 0; x < tx; ++x)
                for (int u = 0; u < tu; ++u) it.push_back({(int)m, 0, u, 0, x});
            if (tu > 0 && tx > 0) int_list.push_back({(int)m, tu, tx});
        }
        const ShellBoxes& B = mb.s->shell;
        // members with the reduced PML state come first in the shell table
        std::vector<BatchTile>& tab = mb.s->region.red ? st : st_full;
        for (int bx = 0; bx < B.n; ++bx)
            for (int x = 0; x < B.tx[bx]; ++x)
                for (int u = 0; u < B.tu[bx]; ++u) tab.push_back({(int)m, bx, u, 0, x});
        mb.tiles = (int64_t)(it.size() + st.size() + st_full.size() - tiles0);
        for (int li = 0; li < mb.s->L; ++li) refs.push_back({(int)m, li});
        max_ghost = std::max(max_ghost, (mb.s->region.ghost_cap + 127) / 128);
        max_solid = std::max(max_solid, (mb.s->n_solid_pml + 255) / 256);
        if (mb.s->hP.n_src > 0) {
            const Box3& r = mb.s->region.src_region;
            const long long cells = (long long)(r.hi[0] - r.lo[0]) * (r.hi[1] - r.lo[1]) * (r.hi[2] - r.lo[2]);
            max_src = std::max<int>(max_src, (int)std::min<long long>((cells + 255) / 256, 64));
        }
    }
    const int n_shell_red = (int)st.size();
    st.insert(st.end(), st_full.begin(), st_full.end());
    fdtd_status st_ = FDTD_OK;
    char* dd = static_cast<char*>(b->d_descs);
    if (b->desc_cap < descs.size()) {
        if (b->d_descs) cudaFree(b->d_descs);
        b->d_descs = nullptr;
        b->desc_cap = 0;
        BATCH_TRY(b, cudaMalloc(&b->d_descs, descs.size() * 2));
        b->desc_cap = descs.size() * 2;
        dd = static_cast<char*>(b->d_descs);
    }
    if ((st_ = grow(b, &b->d_int, &b->int_cap, it.size())) != FDTD_OK) return st_;
    if ((st_ = grow(b, &b->d_shell, &b->shell_cap, st.size())) != FDTD_OK) return st_;
    if ((st_ = grow(b, &b->d_refs, &b->refs_cap, refs.size())) != FDTD_OK) return st_;
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    BATCH_TRY(b, cudaMemcpy(dd, descs.data(), descs.size(), cudaMemcpyHostToDevice));
    if (!it.empty()) BATCH_TRY(b, cudaMemcpy(b->d_int, it.data(), it.size() * sizeof(BatchTile), cudaMemcpyHostToDevice));
    if (!st.empty()) BATCH_TRY(b, cudaMemcpy(b->d_shell, st.data(), st.size() * sizeof(BatchTile), cudaMemcpyHostToDevice));
    if (!refs.empty())
        BATCH_TRY(b, cudaMemcpy(b->d_refs, refs.data(), refs.size() * sizeof(ListenerRef), cudaMemcpyHostToDevice));
    BatchLaunch& L = b->L;
    L.descs = b->d_descs;
    b->table_bytes = tbytes;
    b->flip = 0;
    L.int_tiles = b->d_int;
    L.n_int = (int)it.size();
    b->int_ctas = 0;
    for (int par = 0; par < 2; ++par) b->int_params[par].clear();
    if (!int_list.empty() && int_list.size() <= (size_t)BATCH_PARAM_MEMBERS)
        for (int par = 0; par < 2; ++par)
            b->int_ctas = f64 ? fill_int_params<double>(b->int_params[par], &descs[par * tbytes], dsz, int_list)
                              : fill_int_params<float>(b->int_params[par], &descs[par * tbytes], dsz, int_list);
    b->table_tiles = (int64_t)(it.size() + st.size());
    L.shell_tiles = b->d_shell;
    L.n_shell = (int)st.size();
    L.n_shell_red = b->precision == FDTD_PRECISION_FP64 ? 0 : n_shell_red;
    L.refs = b->d_refs;
    L.n_refs = (int)refs.size();
    L.n_members = (int)nm;
    L.xb = xb;
    L.xs = xs;
    L.ghost_blocks = std::min(max_ghost, 32);
    L.src_blocks = max_src;
    L.solid_blocks = std::min(max_solid, 64);
    for (int i = 0; i < 2; ++i)
        if (b->graph[i]) {
            cudaGraphExecDestroy(b->graph[i]);
            b->graph[i] = nullptr;
        }
    b->dirty = false;
    return FDTD_OK;
}

fdtd_status enqueue(fdtd_batch* b) {
    int l = 0;
    BatchLaunch L = b->L;
    const int p = b->flip;  // table of this step
    L.descs = static_cast<char*>(b->d_descs) + p * b->table_bytes;
    L.int_params = b->int_params[p].empty() ? nullptr : b->int_params[p].data();
    L.int_ctas = b->int_ctas;
    L.descs_other = static_cast<char*>(b->d_descs) + (p ^ 1) * b->table_bytes;
    b->flip ^= 1;
    const StepStreams SS{b->stream, b->stream2, b->stream3, b->ev_fork, b->ev_join, b->ev_ghost};
    cudaError_t e = b->precision == FDTD_PRECISION_FP64
                        ? launch_batch_fp64(L, SS, &l)
                        : launch_batch_fp32(L, SS, &l);
    // listener rows of this step beside the next step
    const bool rows = L.n_refs > 0;
    if (e == cudaSuccess && rows) e = cudaEventRecord(b->ev_step, b->stream);
    if (e == cudaSuccess && rows) e = cudaStreamWaitEvent(b->stream4, b->ev_step, 0);
    if (e == cudaSuccess && rows) e = launch_batch_listeners_any(b->precision, L, b->stream4, &l);
    if (e == cudaSuccess && rows) e = cudaEventRecord(b->ev_lis[p], b->stream4);
    // the rows of the step before read the pressure the next step overwrites and
    // the table this step's advance marks halted members in
    if (e == cudaSuccess && b->lis_pending[p ^ 1]) {
        e = cudaStreamWaitEvent(b->stream, b->ev_lis[p ^ 1], 0);
        b->lis_pending[p ^ 1] = false;
    }
    if (rows) b->lis_pending[p] = true;
    if (e == cudaSuccess) e = launch_batch_advance_any(b->precision, L, b->stream, &l);
    b->launches += l;
    if (e != cudaSuccess) return batch_fail(b, FDTD_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

// Make the batch stream wait for every listener launch on stream4.
fdtd_status join_listeners(fdtd_batch* b) {
    if (!b->lis_pending[0] && !b->lis_pending[1]) return FDTD_OK;
    BATCH_TRY(b, cudaEventRecord(b->ev_lis_join, b->stream4));
    BATCH_TRY(b, cudaStreamWaitEvent(b->stream, b->ev_lis_join, 0));
    b->lis_pending[0] = b->lis_pending[1] = false;
    return FDTD_OK;
}

// Capture n (even) steps starting at the current table into graph[flip].
fdtd_status capture(fdtd_batch* b, int n) {
    cudaGraph_t g = nullptr;
    const int f0 = b->flip;
    fdtd_status st = join_listeners(b);  // no dependency on work outside the capture
    if (st != FDTD_OK) return st;
    BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long l0 = b->launches;
    for (int i = 0; i < n && st == FDTD_OK; ++i) st = enqueue(b);
    if (st == FDTD_OK) st = join_listeners(b);  // the graph ends with every row written
    b->lis_pending[0] = b->lis_pending[1] = false;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->graph_launches = b->launches - l0;
    b->launches = l0;
    b->flip = f0;  // capturing launched nothing
    if (st != FDTD_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return batch_fail(b, FDTD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph[f0], g, 0);
    cudaGraphDestroy(g);
    if (e == cudaSuccess) e = cudaGraphUpload(b->graph[f0], b->stream);  // device-side setup now
    if (e != cudaSuccess) return batch_fail(b, FDTD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

// Copy listener rows of steps [first, first+count) of a member from its ring.
fdtd_status collect_rows(fdtd_batch* b, Member& mb, int64_t first, int64_t count) {
    if (mb.L == 0 || count <= 0) return FDTD_OK;
    const int cap = mb.s->lis_cap_steps;
    const size_t old = mb.rows.size();
    mb.rows.resize(old + (size_t)count * mb.L);
    int64_t k = 0;
    while (k < count) {
        const int64_t pos = (first + k) % cap;
        const int64_t run = std::min<int64_t>(count - k, cap - pos);
        BATCH_TRY(b, cudaMemcpyAsync(mb.rows.data() + old + (size_t)k * mb.L, mb.s->d_lis + (size_t)pos * mb.L,
                                     (size_t)run * mb.L * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        k += run;
    }
    return FDTD_OK;
}

}  // namespace

extern "C" {

fdtd_status fdtd_batch_create(int32_t n, const fdtd_scene_desc* scenes, const int32_t* steps,
                              const fdtd_options* options, fdtd_batch** out) {
    if (!out || n < 0 || (n > 0 && (!scenes || !steps)))
        return batch_fail(nullptr, FDTD_ERR_INVALID_ARG, "fdtd_batch_create: invalid arguments");
    *out = nullptr;
    std::unique_ptr<fdtd_batch> b(new fdtd_batch());
    if (options) b->opt = *options;
    if (b->opt.kernel != FDTD_KERNEL_FUSED)
        return batch_fail(nullptr, FDTD_ERR_INVALID_ARG, "batches use the fused kernel path");
    if (b->opt.graph_steps < 0 || (b->opt.graph_steps % 2) != 0 || b->opt.graph_steps > 256)
        return batch_fail(nullptr, FDTD_ERR_INVALID_ARG, "graph_steps must be an even number in [0, 256]");
    b->precision = b->opt.precision;
    BATCH_TRY(nullptr, cudaSetDevice(b->opt.device));
    BATCH_TRY(nullptr, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BATCH_TRY(nullptr, cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking));
    BATCH_TRY(nullptr, cudaStreamCreateWithFlags(&b->stream3, cudaStreamNonBlocking));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_ghost, cudaEventDisableTiming));
    if (b->precision == FDTD_PRECISION_FP32_COMPENSATED) BATCH_TRY(nullptr, prepare_fp32_kernels());
    else BATCH_TRY(nullptr, prepare_fp64_kernels());
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    BATCH_TRY(nullptr, cudaStreamCreateWithFlags(&b->stream4, cudaStreamNonBlocking));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_step, cudaEventDisableTiming));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_lis[0], cudaEventDisableTiming));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_lis[1], cudaEventDisableTiming));
    BATCH_TRY(nullptr, cudaEventCreateWithFlags(&b->ev_lis_join, cudaEventDisableTiming));
    for (int i = 0; i < n; ++i) {
        int32_t id;
        fdtd_status st = fdtd_batch_add(b.get(), &scenes[i], steps[i], &id);
        if (st != FDTD_OK) {
            fdtd_batch_destroy(b.release());
            return st;
        }
    }
    *out = b.release();
    return FDTD_OK;
}

namespace {
// the slot of a new member: the first released one, else a new one
int32_t place_member(fdtd_batch* b, Member&& mb) {
    size_t slot = b->members.size();
    for (size_t i = 0; i < b->members.size(); ++i)
        if (b->members[i].released) {
            slot = i;
            break;
        }
    if (slot == b->members.size()) b->members.push_back(std::move(mb));
    else b->members[slot] = std::move(mb);
    b->dirty = true;
    return (int32_t)slot;
}
}  // namespace

fdtd_status fdtd_batch_member_snapshot(fdtd_batch* b, int32_t member, void* buffer, int64_t* bytes) {
    if (!b || !bytes || member < 0 || member >= (int32_t)b->members.size() || b->members[member].released ||
        !b->members[member].s)
        return batch_fail(b, FDTD_ERR_INVALID_ARG, "fdtd_batch_member_snapshot: no such member");
    fdtd_solver* s = b->members[member].s;
    if (buffer) {
        BATCH_TRY(b, cudaSetDevice(b->opt.device));
        BATCH_TRY(b, cudaStreamSynchronize(b->stream));  // the member's batched steps are done
    }
    const fdtd_status st = fdtd_solver_snapshot(s, buffer, bytes);
    if (st != FDTD_OK) return batch_fail(b, st, fdtd_solver_last_error(s));
    return FDTD_OK;
}

}  // extern "C"

namespace fdtd {

fdtd_status batch_prepare(const fdtd_options& batch_opt, const fdtd_scene_desc* scene, int32_t steps_total,
                          const void* snapshot, int64_t snapshot_bytes, const double* rows, int64_t steps_done,
                          PreparedMember* out, std::string* err) {
    auto fail = [&](fdtd_status code, const std::string& m, fdtd_solver* s) {
        if (s) fdtd_solver_destroy(s);
        *err = m;
        return code;
    };
    if (!scene || !out || steps_total < 0 || steps_done < 0 || steps_done > steps_total)
        return fail(FDTD_ERR_INVALID_ARG, "batch member: invalid arguments", nullptr);
    if (scene->boundary_handling != FDTD_BOUNDARY_RASTERIZE)
        return fail(FDTD_ERR_UNSUPPORTED, "batched members use RASTERIZE boundaries", nullptr);
    if (scene->air_viscosity_alpha != 0.0)
        return fail(FDTD_ERR_UNSUPPORTED, "batched members have no air viscosity", nullptr);
    if (snapshot && scene->n_listeners > 0 && steps_done > 0 && !rows)
        return fail(FDTD_ERR_INVALID_ARG, "batch member: rows missing", nullptr);
    fdtd_options o = batch_opt;
    o.graph_steps = 0;
    o.shell_staging = FDTD_SHELL_STAGING_RING;  // the batch kernels stage per thread
    fdtd_solver* s = nullptr;
    fdtd_status st = fdtd_solver_create(scene, &o, &s);
    if (st != FDTD_OK) return fail(st, fdtd_last_error(), nullptr);
    if (s->moving) return fail(FDTD_ERR_UNSUPPORTED, "moving bodies are stepped by fdtd_solver, not in batches", s);
    if (!s->eng.empty()) return fail(FDTD_ERR_UNSUPPORTED, "batched members have a PML on every side", s);
    PreparedMember pm;
    pm.s = s;
    pm.total = steps_total;
    if (snapshot) {
        st = fdtd_solver_restore(s, snapshot, snapshot_bytes);
        if (st != FDTD_OK) return fail(st, fdtd_solver_last_error(s), s);
        if (s->step_index != steps_done) return fail(FDTD_ERR_INVALID_ARG, "snapshot step differs from steps_done", s);
        pm.done = steps_done;
        if (s->L > 0 && steps_done > 0) pm.rows.assign(rows, rows + (size_t)steps_done * s->L);
    } else if (steps_total > 0) {
        // the first step classifies the cells (MAC_Grid::classifyCells_FAST)
        pm.rows.resize(s->L);
        st = fdtd_solver_step(s, 1, s->L ? pm.rows.data() : nullptr);
        if (st < 0) return fail(st, fdtd_solver_last_error(s), s);
        pm.done = 1;
    }
    *out = std::move(pm);
    return FDTD_OK;
}

int32_t batch_place(fdtd_batch* b, PreparedMember&& pm) {
    Member mb;
    mb.s = pm.s;
    mb.total = pm.total;
    mb.done = pm.done;
    mb.L = pm.s->L;
    mb.rows = std::move(pm.rows);
    mb.active = mb.done < mb.total;
    pm.s = nullptr;
    return place_member(b, std::move(mb));
}

}  // namespace fdtd

extern "C" {

fdtd_status fdtd_batch_add_snapshot(fdtd_batch* b, const fdtd_scene_desc* scene, int32_t steps_total,
                                    const void* snapshot, int64_t bytes, const double* rows, int64_t steps_done,
                                    int32_t* member) {
    if (!b || !scene || !snapshot) return batch_fail(b, FDTD_ERR_INVALID_ARG, "fdtd_batch_add_snapshot: invalid arguments");
    fdtd::PreparedMember pm;
    std::string err;
    const fdtd_status st = fdtd::batch_prepare(b->opt, scene, steps_total, snapshot, bytes, rows, steps_done, &pm, &err);
    if (st != FDTD_OK) return batch_fail(b, st, err);
    const int32_t slot = fdtd::batch_place(b, std::move(pm));
    if (member) *member = slot;
    return FDTD_OK;
}

fdtd_status fdtd_batch_add(fdtd_batch* b, const fdtd_scene_desc* scene, int32_t steps, int32_t* member) {
    if (!b || !scene || steps < 0) return batch_fail(b, FDTD_ERR_INVALID_ARG, "fdtd_batch_add: invalid arguments");
    fdtd::PreparedMember pm;
    std::string err;
    const fdtd_status st = fdtd::batch_prepare(b->opt, scene, steps, nullptr, 0, nullptr, 0, &pm, &err);
    if (st != FDTD_OK) return batch_fail(b, st, err);
    const int32_t slot = fdtd::batch_place(b, std::move(pm));
    if (member) *member = slot;
    return FDTD_OK;
}

fdtd_status fdtd_batch_step(fdtd_batch* b, int32_t n_steps, int32_t* n_active) {
    if (!b || n_steps < 0) return batch_fail(b, FDTD_ERR_INVALID_ARG, "fdtd_batch_step: invalid arguments");
    BATCH_TRY(b, cudaSetDevice(b->opt.device));
    const long long l0 = b->launches;
    int64_t left = n_steps;
    const int G = b->opt.graph_steps;
    while (left > 0) {
        // members stop on the device at their own last step (k_batch_advance), so a
        // chunk runs until the longest member finishes, within the listener rings
        int64_t chunk = left, longest = 0;
        bool any = false;
        for (auto& mb : b->members)
            if (mb.active) {
                any = true;
                longest = std::max<int64_t>(longest, mb.total - mb.done);
                chunk = std::min<int64_t>(chunk, mb.s->lis_cap_steps);
            }
        if (!any) break;
        chunk = std::min(chunk, longest);
        if (b->dirty) {
            fdtd_status st = rebuild(b);
            if (st != FDTD_OK) return st;
        }
        if (G > 0 && chunk >= G) {
            chunk = (chunk / G) * G;
            if (!b->graph[b->flip]) {
                fdtd_status st = capture(b, G);
                if (st != FDTD_OK) return st;
            }
            for (int64_t i = 0; i < chunk / G; ++i) {
                // G is even: the graph leaves the table parity as it found it
                BATCH_TRY(b, cudaGraphLaunch(b->graph[b->flip], b->stream));
                b->launches += b->graph_launches;
            }
        } else {
            for (int64_t i = 0; i < chunk; ++i) {
                fdtd_status st = enqueue(b);
                if (st != FDTD_OK) return st;
            }
        }
        // rows, host mirrors, retirement
        fdtd_status jst = join_listeners(b);
        if (jst != FDTD_OK) return jst;
        std::vector<int> errs(b->members.size(), 0);
        for (size_t m = 0; m < b->members.size(); ++m) {
            Member& mb = b->members[m];
            if (!mb.active) continue;
            fdtd_status st = collect_rows(b, mb, mb.done, std::min<int64_t>(chunk, mb.total - mb.done));
            if (st != FDTD_OK) return st;
            BATCH_TRY(b, cudaMemcpyAsync(&errs[m], mb.s->hP.dev_error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        }
        BATCH_TRY(b, cudaStreamSynchronize(b->stream));
        int64_t idle_tiles = 0;
        for (size_t m = 0; m < b->members.size(); ++m) {
            Member& mb = b->members[m];
            if (!mb.active) {
                idle_tiles += mb.tiles;
                continue;
            }
            fdtd_solver* s = mb.s;
            const int64_t n = std::min<int64_t>(chunk, mb.total - mb.done);
            s->cur ^= (int)(n & 1);
            s->step_index += n;
            for (int64_t i = 0; i < n; ++i) s->time += s->k;
            mb.done += n;
            if (errs[m] & 1) mb.status = FDTD_ERR_NUMERIC;
            if (mb.done >= mb.total) {
                mb.active = false;
                idle_tiles += mb.tiles;
            }
        }
        // new tables (and graphs) only once a quarter of the tiles belong to finished members
        if (idle_tiles * 4 > b->table_tiles) b->dirty = true;
        left -= chunk;
    }
    b->last_launches = b->launches - l0;
    if (n_active) {
        int a = 0;
        for (auto& mb : b->members) a += mb.active ? 1 : 0;
        *n_active = a;
    }
    return FDTD_OK;
}

fdtd_status fdtd_batch_run(fdtd_batch* b) {
    if (!b) return FDTD_ERR_INVALID_ARG;
    int32_t active = 1;
    while (active > 0) {
        fdtd_status st = fdtd_batch_step(b, 1 << 20, &active);
        if (st != FDTD_OK) return st;
    }
    return FDTD_OK;
}

fdtd_status fdtd_batch_member_info(fdtd_batch* b, int32_t member, int64_t* steps_done, int64_t* steps_total,
                                   int32_t* n_listeners, int32_t* status) {
    if (!b || member < 0 || member >= (int32_t)b->members.size() || b->members[member].released)
        return batch_fail(b, FDTD_ERR_INVALID_ARG, "no such member (out of range or released)");
    const Member& mb = b->members[member];
    if (steps_done) *steps_done = mb.done;
    if (steps_total) *steps_total = mb.total;
    if (n_listeners) *n_listeners = mb.L;
    if (status) *status = mb.status;
    return FDTD_OK;
}

fdtd_status fdtd_batch_output(fdtd_batch* b, int32_t member, double* out, int64_t count) {
    if (!b || member < 0 || member >= (int32_t)b->members.size() || b->members[member].released)
        return batch_fail(b, FDTD_ERR_INVALID_ARG, "no such member (out of range or released)");
    const Member& mb = b->members[member];
    if (count < (int64_t)mb.rows.size() || (!out && !mb.rows.empty()))
        return batch_fail(b, FDTD_ERR_INVALID_ARG, "output buffer smaller than steps_done * n_listeners");
    if (!mb.rows.empty()) std::memcpy(out, mb.rows.data(), mb.rows.size() * sizeof(double));
    return FDTD_OK;
}

fdtd_status fdtd_batch_release(fdtd_batch* b, int32_t member) {
    if (!b || member < 0 || member >= (int32_t)b->members.size())
        return batch_fail(b, FDTD_ERR_INVALID_ARG, "member index out of range");
    Member& mb = b->members[member];
    if (mb.released) return FDTD_OK;
    if (mb.s) {
        BATCH_TRY(b, cudaStreamSynchronize(b->stream));
        fdtd_solver_destroy(mb.s);
        mb.s = nullptr;
    }
    mb = Member();
    mb.released = true;
    b->dirty = true;
    return FDTD_OK;
}

fdtd_status fdtd_batch_destroy(fdtd_batch* b) {
    if (!b) return FDTD_OK;
    cudaSetDevice(b->opt.device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->stream4) cudaStreamSynchronize(b->stream4);
    for (int i = 0; i < 2; ++i)
        if (b->graph[i]) cudaGraphExecDestroy(b->graph[i]);
    for (auto& mb : b->members)
        if (mb.s) fdtd_solver_destroy(mb.s);
    if (b->d_descs) cudaFree(b->d_descs);
    if (b->d_int) cudaFree(b->d_int);
    if (b->d_shell) cudaFree(b->d_shell);
    if (b->d_refs) cudaFree(b->d_refs);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->ev_ghost) cudaEventDestroy(b->ev_ghost);
    for (cudaEvent_t ev : {b->ev_step, b->ev_lis[0], b->ev_lis[1], b->ev_lis_join})
        if (ev) cudaEventDestroy(ev);
    if (b->stream4) cudaStreamDestroy(b->stream4);
    if (b->stream2) cudaStreamDestroy(b->stream2);
    if (b->stream3) cudaStreamDestroy(b->stream3);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FDTD_OK;
}

void* fdtd_batch_stream(fdtd_batch* b) { return b ? (void*)b->stream : nullptr; }
int64_t fdtd_batch_last_launch_count(fdtd_batch* b) { return b ? b->last_launches : 0; }

int64_t fdtd_batch_device_bytes(fdtd_batch* b) {
    if (!b) return 0;
    int64_t t = 0;
    for (auto& mb : b->members)
        if (mb.s) t += (int64_t)mb.s->arena_bytes;
    return t;
}

}  // extern "C"
