// fdtd_api.cpp — the C-ABI of include/fdtd_c.h: solver lifecycle, the
// host-side FP64 geometry (computed with the reference's own expressions and
// operation order, -ffp-contract=off), classification driver, step loop with
// CUDA graphs, read-back, snapshot/restore.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_device.cuh"
#include "fdtd_geometry.cuh"
#include "fdtd_internal.hpp"
#include "fdtd_launch.hpp"

using namespace fdtd;

namespace {
thread_local std::string g_last_error;
// fdtd_debug_inject_failure: which allocation fails next, and after how many more calls
std::atomic<int> g_inject_what{FDTD_INJECT_NONE};
std::atomic<int> g_inject_after{0};
const double EPS = 1e-10;                  // src/config.h:45
const double GAUSSIAN_CHECK_BOUND = 2.0;   // Wavesolver_ConstantsAndTypes.h:77
}  // namespace

namespace fdtd {
bool inject_failure(int what) {
    if (g_inject_what.load() != what) return false;
    if (g_inject_after.fetch_sub(1) != 0) return false;
    g_inject_what.store(FDTD_INJECT_NONE);
    return true;
}

void set_error(fdtd_solver* s, const std::string& msg) {
    g_last_error = msg;
    if (s) s->err = msg;
}
}  // namespace fdtd

#define CUDA_TRY(s, expr)                                                                         \
    do {                                                                                          \
        cudaError_t _e = (expr);                                                                  \
        if (_e != cudaSuccess) {                                                                  \
            set_error((s), std::string("CUDA: ") + cudaGetErrorString(_e) + " at " #expr);       \
            return _e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA;                \
        }                                                                                         \
    } while (0)

// ---------------------------------------------------------------------------
// Host geometry (FP64, reference expressions)
// ---------------------------------------------------------------------------
namespace fdtd {

// MAC_Grid::PML_absorptionCoefficient, quadratic profile (MAC_Grid.cpp:4064-4101),
// along axis d for boundary preset `preset` (0: PML on every side; 1: on the
// low sides and +y; 2: on +z only); pow(x,2) written as x*x (the compiler
// folds it identically without fast-math).
static double absorption(double x, double mn, double mx, double w, double S, int preset, int d) {
    const double hMin = x - mn, hMax = mx - x;
    const double a2 = w * w;
    const double distMin = w - hMin, distMax = w - hMax;
    if (preset == 0) {
        if (hMin <= w) return S * (distMin * distMin) / a2;
        if (hMax <= w) return S * (distMax * distMax) / a2;
    } else if (preset == 1) {
        if (hMin <= w) return S * (distMin * distMin) / a2;
        if (d == 1 && hMax <= w) return S * (distMax * distMax) / a2;
    } else if (preset == 2) {
        if (d != 2 || hMin <= w) return 0.0;
        if (hMax <= w) return S * (distMax * distMax) / a2;
    }
    return 0.0;
}

// Arena blocks of destroyed solvers, kept per device for the next solver:
// cudaFree of a block of a few hundred MB synchronises the device and was
// measured to take from a few ms to half a second, which a server creating and
// destroying solves, or a caller timing whole solves, would pay every time.  A
// block serves a request of at least half its size; when cudaMalloc fails, the
// blocks kept for that device are freed and the allocation is tried again.
namespace {
struct KeptArena {
    int device;
    void* ptr;
    size_t bytes;
};
std::mutex g_arena_mu;
std::vector<KeptArena> g_arenas;  // oldest first
// kept blocks per process: at most this many and this many bytes (a destroy that
// pushes past a limit frees the oldest blocks, which is where cudaFree's cost
// returns, so the limits sit above what a server's or a benchmark's churn keeps)
constexpr size_t ARENAS_KEPT = 256;
constexpr size_t ARENAS_KEPT_BYTES = (size_t)16 << 30;

void free_kept(int device) {
    std::vector<KeptArena> drop;
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        std::vector<KeptArena> keep;
        for (const auto& a : g_arenas) (device < 0 || a.device == device ? drop : keep).push_back(a);
        g_arenas.swap(keep);
    }
    int cur = -1;
    cudaGetDevice(&cur);
    for (const auto& a : drop) {
        cudaSetDevice(a.device);
        cudaFree(a.ptr);
    }
    if (cur >= 0) cudaSetDevice(cur);
}
}  // namespace

cudaError_t arena_acquire(int device, size_t bytes, void** ptr, size_t* block_bytes) {
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        int best = -1;
        for (int i = 0; i < (int)g_arenas.size(); ++i) {
            const KeptArena& a = g_arenas[i];
            if (a.device != device || a.bytes < bytes || a.bytes / 2 > bytes) continue;
            if (best < 0 || a.bytes < g_arenas[best].bytes) best = i;
        }
        if (best >= 0) {
            *ptr = g_arenas[best].ptr;
            *block_bytes = g_arenas[best].bytes;
            g_arenas.erase(g_arenas.begin() + best);
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        free_kept(device);
        e = cudaMalloc(ptr, bytes);
    }
    if (e == cudaSuccess) *block_bytes = bytes;
    return e;
}

void arena_release(int device, void* ptr, size_t block_bytes) {
    if (!ptr) return;
    std::vector<KeptArena> drop;
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        g_arenas.push_back({device, ptr, block_bytes});
        size_t total = 0;
        for (const auto& a : g_arenas) total += a.bytes;
        while (g_arenas.size() > 1 && (g_arenas.size() > ARENAS_KEPT || total > ARENAS_KEPT_BYTES)) {
            total -= g_arenas.front().bytes;
            drop.push_back(g_arenas.front());
            g_arenas.erase(g_arenas.begin());
        }
    }
    if (!drop.empty()) {
        int cur = -1;
        cudaGetDevice(&cur);
        for (const auto& a : drop) {
            cudaSetDevice(a.device);
            cudaFree(a.ptr);
        }
        if (cur >= 0) cudaSetDevice(cur);
    }
}

// one dimension of MAC_Grid::InsidePML (MAC_Grid.cpp:4027-4062)
static bool inside_pml_1d(double x, double mn, double mx, double w, int preset, int d) {
    const double pmlWidth = w + 1E-12;
    const double hMin = x - mn, hMax = mx - x;
    if (preset == 0) return hMin <= pmlWidth || hMax <= pmlWidth;
    if (preset == 1) return hMin <= pmlWidth || (d == 1 && hMax <= pmlWidth);
    if (preset == 2) return d == 2 && hMax <= pmlWidth;
    return false;
}

void host_object_pose(HostObject& o, double t) {
    if (o.d.motion == FDTD_MOTION_KEYFRAMED && o.kf) {
        // FDTD_Objects::AnimateObjects -> SetRigidBodyTransform: rotation R * R0, centre to the frame's
        double R[9];
        keyframe_pose(o.kf, o.kf_n, o.kf_step, t, o.c, R);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                o.d.rotation[i * 3 + j] =
                    R[i * 3 + 0] * o.R0[0 * 3 + j] + R[i * 3 + 1] * o.R0[1 * 3 + j] + R[i * 3 + 2] * o.R0[2 * 3 + j];
        if (o.d.shape == FDTD_SHAPE_MESH && o.mv) mesh_extent(o.mv, (size_t)o.mv_n, o.d.rotation, o.mlo, o.mhi);
        return;
    }
    for (int a = 0; a < 3; ++a) {
        if (o.d.motion == FDTD_MOTION_BALLISTIC)
            o.c[a] = o.d.center[a] + o.d.velocity[a] * t + 0.5 * o.d.gravity[a] * t * t;
        else
            o.c[a] = o.d.center[a];
    }
}

static void half_extent(const HostObject& o, double e[3]) {
    for (int i = 0; i < 3; ++i) {
        if (o.d.shape == FDTD_SHAPE_SPHERE) { e[i] = o.d.size[0]; continue; }
        double s = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double rij = o.d.rotation[i * 3 + j];
            if (o.d.shape == FDTD_SHAPE_BOX) s = s + std::fabs(rij) * o.d.size[j];
            else s = s + (rij * o.d.size[j]) * (rij * o.d.size[j]);
        }
        e[i] = (o.d.shape == FDTD_SHAPE_BOX) ? s : std::sqrt(s);
    }
}

// FDTD_RigidObject::UpdateBoundingBox (FDTD_RigidObject.cpp:190-226) with the
// BoundingBox::Update / Union arithmetic of FDTD_MovableObject.h:81-99
void host_update_bbox(HostObject& o) {
    for (int d = 0; d < 3; ++d) { o.umin[d] = o.bmin[d]; o.umax[d] = o.bmax[d]; }
    if (o.d.shape == FDTD_SHAPE_MESH) {
        for (int d = 0; d < 3; ++d) { o.bmin[d] = o.c[d] + o.mlo[d]; o.bmax[d] = o.c[d] + o.mhi[d]; }
    } else {
        double e[3];
        half_extent(o, e);
        for (int d = 0; d < 3; ++d) { o.bmin[d] = o.c[d] - e[d]; o.bmax[d] = o.c[d] + e[d]; }
    }
    for (int d = 0; d < 3; ++d) {
        o.umin[d] = std::min(o.bmin[d], o.umin[d]);
        o.umax[d] = std::max(o.bmax[d], o.umax[d]);
    }
}

HostObject make_host_object(const fdtd_scene_desc* sc, int i) {
    HostObject h;
    h.d = sc->objects[i];
    for (int k = 0; k < 9; ++k) h.R0[k] = h.d.rotation[k];
    if (h.d.shape == FDTD_SHAPE_MESH) {
        const fdtd_mesh_desc& m = sc->meshes[h.d.mesh];
        mesh_extent(m.vertices, (size_t)m.n_vertices, h.d.rotation, h.mlo, h.mhi);
        h.mv = m.vertices;
        h.mv_n = m.n_vertices;
    }
    if (h.d.motion == FDTD_MOTION_KEYFRAMED)
        for (int k = 0; k < sc->n_tracks; ++k)
            if (sc->tracks[k].object == i) {
                h.kf = sc->tracks[k].frames;
                h.kf_n = sc->tracks[k].n_frames;
                h.kf_step = sc->tracks[k].step;
            }
    return h;
}

void host_reset_union(HostObject& o) {
    for (int d = 0; d < 3; ++d) { o.umin[d] = o.bmin[d]; o.umax[d] = o.bmax[d]; }
}

static void to_dev_object(const HostObject& o, DevObject& d) {
    std::memset(&d, 0, sizeof(d));
    d.shape = o.d.shape;
    d.accel_kind = o.d.accel_kind;
    d.motion = o.d.motion;
    for (int i = 0; i < 3; ++i) {
        d.c[i] = o.c[i];
        d.size[i] = o.d.size[i];
        d.bmin[i] = o.bmin[i];
        d.bmax[i] = o.bmax[i];
        d.bdim[i] = o.bmax[i] - o.bmin[i];
        d.bcen[i] = (o.bmax[i] + o.bmin[i]) / 2.0;
        d.dir[i] = o.d.accel_dir[i];
    }
    for (int i = 0; i < 9; ++i) d.R[i] = o.d.rotation[i];
    d.amp = o.d.accel_amplitude;
    d.t0 = o.d.accel_t0;
    d.tau = o.d.accel_tau;
    d.mesh = o.mview;
}

void to_dev_objects(fdtd_solver* s) {
    for (size_t i = 0; i < s->objs.size(); ++i) to_dev_object(s->objs[i], s->hP.obj[i]);
}

// ScalarField::GetIterationBox (ScalarField.cpp:288-314), clamped to the grid
static void iteration_box(const fdtd_solver* s, double mn[3], double mx[3], int start[3], int range[3]) {
    auto inside = [&](const double* x) {
        return x[0] >= s->bmin[0] && x[1] >= s->bmin[1] && x[2] >= s->bmin[2] && x[0] <= s->bmax[0] &&
               x[1] <= s->bmax[1] && x[2] <= s->bmax[2];
    };
    const double imn[3] = {mn[0], mn[1], mn[2]}, imx[3] = {mx[0], mx[1], mx[2]};
    if (!inside(imn)) for (int d = 0; d < 3; ++d) mn[d] = std::max(s->bmin[d], mn[d]);
    if (!inside(imx)) for (int d = 0; d < 3; ++d) mx[d] = std::min(s->bmax[d], mx[d]);
    for (int d = 0; d < 3; ++d) {
        start[d] = (int)std::floor((mn[d] - s->bmin[d]) / s->h);
        const int end = (int)std::ceil((mx[d] - s->bmin[d]) / s->h);
        range[d] = std::max(end - start[d], 1);
        if (start[d] < 0) { range[d] += start[d]; start[d] = 0; }
        if (start[d] + range[d] > s->N[d]) range[d] = s->N[d] - start[d];
        if (range[d] < 0) range[d] = 0;
    }
}

// The object and constraint boxes that classifyCells_FAST iterates (MAC_Grid.cpp:3510-3551)
void classification_boxes(const fdtd_solver* s, ClsBoxes& B) {
    B.n = 0;
    B.first[0] = 0;
    B.ufirst[0] = 0;
    auto push = [&](const int st[3], const int rg[3]) {
        for (int d = 0; d < 3; ++d) {
            B.lo[B.n][d] = st[d];
            B.rg[B.n][d] = rg[d];
        }
        const bool empty = rg[0] <= 0 || rg[1] <= 0 || rg[2] <= 0;
        B.first[B.n + 1] = B.first[B.n] + (empty ? 0 : (long long)rg[0] * rg[1] * rg[2]);
        // units reached: rows lo-1 .. lo+rg (clipped), chunks holding cells lo2-1 .. lo2+rg2
        long long units = 0;
        if (!empty) {
            for (int d = 0; d < 2; ++d) {
                const int a = std::max(0, st[d] - 1), b = std::min(s->N[d] - 1, st[d] + rg[d]);
                B.u0[B.n][d] = a;
                B.un[B.n][d] = std::max(0, b - a + 1);
            }
            const int ka = std::max(0, st[2] - 1), kb = std::min(s->N[2] - 1, st[2] + rg[2]);
            B.u0[B.n][2] = ka / CLS_CHUNK;
            B.un[B.n][2] = kb >= ka ? kb / CLS_CHUNK - ka / CLS_CHUNK + 1 : 0;
            units = (long long)B.un[B.n][0] * B.un[B.n][1] * B.un[B.n][2];
        } else {
            for (int d = 0; d < 3; ++d) B.u0[B.n][d] = B.un[B.n][d] = 0;
        }
        B.ufirst[B.n + 1] = B.ufirst[B.n] + units;
        ++B.n;
    };
    for (const auto& o : s->objs) {
        double mn[3] = {o.umin[0], o.umin[1], o.umin[2]}, mx[3] = {o.umax[0], o.umax[1], o.umax[2]};
        for (const auto& pl : s->planes) {
            if (pl.normal_sign > 0) mn[pl.normal_dir] = std::max(mn[pl.normal_dir], pl.height);
            else mx[pl.normal_dir] = std::min(mx[pl.normal_dir], pl.height);
        }
        int st[3], rg[3];
        iteration_box(s, mn, mx, st, rg);
        push(st, rg);
    }
    for (const auto& pl : s->planes) {
        const double NEG_INF = std::numeric_limits<double>::lowest(), POS_INF = std::numeric_limits<double>::max();
        double mn[3] = {NEG_INF, NEG_INF, NEG_INF}, mx[3] = {POS_INF, POS_INF, POS_INF};
        if (pl.normal_sign > 0) mx[pl.normal_dir] = pl.height;
        else mn[pl.normal_dir] = pl.height;
        int st[3], rg[3];
        iteration_box(s, mn, mx, st, rg);
        push(st, rg);
    }
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
namespace {

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Carver {
    size_t off = 0;
    std::vector<std::pair<void**, size_t>> req;
    void add(void** p, size_t bytes) {
        req.push_back({p, off});
        off += align256(bytes);
    }
};

fdtd_status upload_params(fdtd_solver* s) {
    CUDA_TRY(s, fdtd::counted_copyAsync(s, s->dP, &s->hP, sizeof(SolveParams), cudaMemcpyHostToDevice, s->stream));
    return FDTD_OK;
}

fdtd_status run_classification(fdtd_solver* s) {
    ClsBoxes& B = s->hP.boxes;
    classification_boxes(s, B);
    CUDA_TRY(s, fdtd::counted_copyAsync(s, &s->dP->boxes, &B, sizeof(ClsBoxes), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, launch_classify(s->dP, s->N, B, false, s->stream));
    s->cls_boxes_current = true;
    s->launches += B.ufirst[B.n] > 0 ? 3 : 2;
    return FDTD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// create / reset
// ---------------------------------------------------------------------------
namespace fdtd {

// Whether a solve keeps the reduced PML state (k_pml_shell_red): FP32 fused
// solves of static scenes with no solid PML cell, or of moving bodies that stay
// two cells clear of the PML at every step until end_time, the five-box shell, and, along
// every axis, unit decay factors on both faces of every cell outside that axis'
// PML (the condition under which the plain axes of a PML cell telescope into one
// leapfrog increment exactly).
bool use_reduced_pml(const fdtd_solver* s, bool no_solid_pml) {
    if (s->precision != FDTD_PRECISION_FP32_COMPENSATED || s->opt.kernel != FDTD_KERNEL_FUSED) return false;
    if (s->opt.pml_state != FDTD_PML_STATE_AUTO || !no_solid_pml) return false;
    // moving bodies only when they stay clear of the PML until end_time
    if (s->moving && !moving_clear_of_pml(const_cast<fdtd_solver*>(s))) return false;
    if (!s->shell.xy_slabs || s->shell.zbox < 0 || !s->eng.empty()) return false;
    for (int d = 0; d < 3; ++d) {
        const auto& T = s->tab[d];
        for (int i = 0; i < s->N[d]; ++i) {
            if (T.pml_cell[i]) continue;
            if (i == 0 || i + 1 >= s->N[d]) return false;
            if (T.pupd[i] != 1.0 || T.vupd[i] != 1.0 || T.vupd[i + 1] != 1.0) return false;
            if (T.vgrad[i] != T.vgrad[i + 1] || T.pdiv[i] != -1.0 * s->rho * s->c * s->c / (1.0 / s->k)) return false;
        }
    }
    return true;
}

// x planes per PML-shell thread: tile_y when given, else the default of the
// solve's PML state.
int shell_planes(const fdtd_solver* s, int tile_y) {
    if (tile_y > 0) return std::min(tile_y, 256);
    return s->region.red ? FDTD_SHELL_RED_PLANES : FDTD_SHELL_PLANES;
}

// PML shell boxes for a given number of x planes per thread (xs).
void build_shell_boxes(fdtd_solver* s, int xs) {
    ShellBoxes& B = s->shell;
    std::memset(&B, 0, sizeof(B));
    B.xs = xs;
    B.zbox = -1;
    const int V = shell_vz(s->precision == FDTD_PRECISION_FP64 ? 8 : 4);  // z cells per vector group
    B.vz = V;
    const int* N = s->N;
    const int* lo = s->interior.lo;
    const int* hi = s->interior.hi;
    auto groups = [&](int z0, int z1) { return z1 > z0 ? (z1 - 1) / V - z0 / V + 1 : 0; };
    auto add = [&](int x0, int x1, int y0, int y1, int za0, int za1, int zb0, int zb1, bool zp = false) {
        const int nz = (za1 - za0) + (zb1 - zb0);
        if (x1 <= x0 || y1 <= y0 || nz <= 0) return;
        const int b = B.n;
        B.zp[b] = zp ? 1 : 0;
        B.x0[b] = x0; B.nx[b] = x1 - x0;
        B.y0[b] = y0; B.ny[b] = y1 - y0;
        B.za[b] = za0; B.zae[b] = za1; B.zb[b] = zb0; B.zbe[b] = zb1;
        B.gl[b] = groups(za0, za1);
        B.ng[b] = B.gl[b] + groups(zb0, zb1);
        B.tu[b] = (B.ny[b] * B.ng[b] + 255) / 256;
        B.tx[b] = (B.nx[b] + xs - 1) / xs;
        B.block_first[b + 1] = B.block_first[b] + B.tu[b] * B.tx[b];
        B.cells += (long long)B.nx[b] * B.ny[b] * nz;
        ++B.n;
    };
    if (hi[0] <= lo[0] || hi[1] <= lo[1] || hi[2] <= lo[2]) {
        add(0, N[0], 0, N[1], 0, N[2], N[2], N[2]);  // every cell is a PML cell
        return;
    }
    // FP32: each x / y slab as two boxes, the vector groups that hold a z-PML
    // cell and those that are whole and outside the z PML, so the reduced-state
    // kernel runs the plain-z columns of a CTA on one specialised path (shell
    // 52.0 -> 48.9 us at 256^3, 22.8 -> 20.5 us at 192^3); short rows keep one
    // box (more boxes of few units leave partial tiles: a batch of 48-160 cell
    // grids lost 1.4 %)
    const int zs0 = (lo[2] + V - 1) / V * V, zs1 = hi[2] / V * V;
    const bool split = s->precision != FDTD_PRECISION_FP64 && zs1 - zs0 >= 128;
    auto slab = [&](int x0, int x1, int y0, int y1) {
        if (split) {
            add(x0, x1, y0, y1, 0, zs0, zs1, N[2]);
            add(x0, x1, y0, y1, zs0, zs1, zs1, zs1, true);
        } else {
            add(x0, x1, y0, y1, 0, N[2], N[2], N[2]);
        }
    };
    slab(0, lo[0], 0, N[1]);
    slab(hi[0], N[0], 0, N[1]);
    slab(lo[0], hi[0], 0, lo[1]);
    slab(lo[0], hi[0], hi[1], N[1]);
    B.xy_slabs = lo[0] > 0 && hi[0] < N[0] && lo[1] > 0 && hi[1] < N[1] && (lo[2] > 0 || hi[2] < N[2]);
    add(lo[0], hi[0], lo[1], hi[1], 0, lo[2], hi[2], N[2]);
    if (B.n > 0 && B.x0[B.n - 1] == lo[0] && B.y0[B.n - 1] == lo[1] && B.zb[B.n - 1] == hi[2]) {
        B.zbox = B.n - 1;
        B.zrw = (B.ng[B.zbox] + 1) * V;
    }
}

// The cells of the Engquist-Majda branch of MAC_Grid::PML_pressureUpdateCollocated
// (MAC_Grid.cpp:515-533): non-PML cells with a boundary normal at offset 1 and
// none at offset 0 (ScalarField::boundaryCellNormal, ScalarField.h:202-213).
// They exist where a side has no PML (presets 1 and 2) or the PML is under
// 1.5 cells; non-PML cells on the domain edge itself are never updated.
static void build_engquist(fdtd_solver* s) {
    s->eng.clear();
    const int* N = s->N;
    const long long stride[3] = {s->SX, s->SY, 1};
    auto normal = [&](const int* ijk, int off, int* n) {
        for (int d = 0; d < 3; ++d) n[d] = ijk[d] == off ? -1 : (ijk[d] == N[d] - 1 - off ? 1 : 0);
    };
    auto is_pml = [&](const int* a) {
        return s->tab[0].pml_cell[a[0]] || s->tab[1].pml_cell[a[1]] || s->tab[2].pml_cell[a[2]];
    };
    auto edge1 = [&](int d, int i) { return i == 1 || i == N[d] - 2; };
    for (int i = 0; i < N[0]; ++i)
        for (int j = 0; j < N[1]; ++j) {
            const bool all_z = edge1(0, i) || edge1(1, j);
            for (int l = 0; l < N[2]; ++l) {
                if (!all_z && l != 1 && l != N[2] - 2) continue;
                const int ijk[3] = {i, j, l};
                if (is_pml(ijk)) continue;
                int n0[3], n1[3];
                normal(ijk, 0, n0);
                if (n0[0] || n0[1] || n0[2]) continue;
                normal(ijk, 1, n1);
                const int btype = std::abs(n1[0]) + std::abs(n1[1]) + std::abs(n1[2]);
                if (btype == 0) continue;
                EngCell e{};
                e.c = (unsigned)(i * s->SX + j * s->SY + l);
                e.flags = btype;
                // axis order: the reference's di, dj, dk of each type
                int di = 0, dj = 1, dk = 2;
                if (btype == 1) {
                    while (n1[di] == 0) ++di;
                    dj = (di + 1) % 3;
                    dk = (di + 2) % 3;
                } else if (btype == 2) {
                    while (n1[di] == 0) ++di;
                    dj = di + 1;
                    while (n1[dj] == 0) ++dj;
                    dk = dj != di + 1 ? (di + 1) % 3 : (di + 2) % 3;
                }
                const int ax[3] = {di, dj, dk};
                // offset of the cell displaced by (u, v, w) along (di, dj, dk)
                auto off = [&](int u, int v, int w, bool* pml) {
                    int a[3] = {i, j, l};
                    const int du[3] = {u, v, w};
                    long long o = 0;
                    for (int q = 0; q < 3; ++q) {
                        const int d = ax[q];
                        a[d] += du[q];
                        o += (long long)du[q] * stride[d];
                    }
                    if (pml) *pml = is_pml(a);
                    return (int)o;
                };
                const int ni = n1[di], nj = n1[dj], nk = n1[dk];
                // tangential neighbours clamped to the grid as the reference clamps them
                auto clampd = [&](int q, int sgn) {
                    const int d = ax[q], v = ijk[d] + sgn;
                    return std::min(std::max(v, 0), N[d] - 1) - ijk[d];
                };
                bool px[4] = {false, false, false, false};
                if (btype == 1) {
                    e.o[0] = off(ni, 0, 0, &px[0]);
                    e.o[1] = off(-ni, 0, 0, nullptr);
                    e.o[2] = off(0, clampd(1, 1), 0, nullptr);
                    e.o[3] = off(0, clampd(1, -1), 0, nullptr);
                    e.o[4] = off(0, 0, clampd(2, 1), nullptr);
                    e.o[5] = off(0, 0, clampd(2, -1), nullptr);
                } else if (btype == 2) {
                    e.o[0] = off(ni, 0, 0, &px[0]);
                    e.o[1] = off(0, nj, 0, &px[1]);
                    e.o[2] = off(ni, nj, 0, &px[3]);
                    e.o[3] = off(-ni, 0, 0, nullptr);
                    e.o[4] = off(0, -nj, 0, nullptr);
                    e.o[5] = off(0, 0, clampd(2, 1), nullptr);
                    e.o[6] = off(0, 0, clampd(2, -1), nullptr);
                } else {
                    e.o[0] = off(ni, 0, 0, &px[0]);
                    e.o[1] = off(0, nj, 0, &px[1]);
                    e.o[2] = off(0, 0, nk, &px[2]);
                    e.o[3] = off(-ni, 0, 0, nullptr);
                    e.o[4] = off(0, -nj, 0, nullptr);
                    e.o[5] = off(0, 0, -nk, nullptr);
                    e.o[6] = off(ni, nj, nk, &px[3]);
                }
                for (int q = 0; q < 4; ++q)
                    if (px[q]) e.flags |= 16 << q;
                s->eng.push_back(e);
            }
        }
}

// Cells the interior kernel updates: the non-PML box less the cells on the
// domain edge (never updated) and one cell inside it (the Engquist cells).
static Box3 update_box(const fdtd_solver* s) {
    Box3 b = s->interior;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = std::max(b.lo[d], 2);
        b.hi[d] = std::min(b.hi[d], s->N[d] - 2);
    }
    if (b.lo[0] >= b.hi[0] || b.lo[1] >= b.hi[1] || b.lo[2] >= b.hi[2])
        for (int d = 0; d < 3; ++d) b.lo[d] = b.hi[d] = 0;
    return b;
}

fdtd_status solver_init_geometry(fdtd_solver* s, const fdtd_scene_desc* sc) {
    s->h = sc->cell_size;
    s->c = sc->sound_speed;
    s->rho = sc->density;
    s->k = sc->time_step;
    s->end_time = sc->end_time;
    s->preset = sc->boundary_condition_preset;
    // BoundingBox(cellSize, divisions, center) (BoundingBox.h:89-99) -> ScalarField (ScalarField.cpp:29-50)
    for (int d = 0; d < 3; ++d) {
        const double mn = sc->domain_center[d] - s->h * (double)sc->divisions[d] / 2.0;
        const double mx = sc->domain_center[d] + s->h * (double)sc->divisions[d] / 2.0;
        s->N[d] = (int)std::ceil(((mx - mn) - EPS) / s->h);
        s->bmin[d] = mn;
        s->bmax[d] = s->bmin[d];
        s->bmax[d] += s->h * (double)s->N[d];
    }
    s->ncell = (long long)s->N[0] * s->N[1] * s->N[2];
    // padded layout shared by cells and the three face grids: rows of Nz+1
    // rounded up to 8 elements, Ny+1 rows per plane, Nx+1 planes
    s->SY = ((long long)s->N[2] + 1 + 7) / 8 * 8;
    s->SX = ((long long)s->N[1] + 1) * s->SY;
    s->np = ((long long)s->N[0] + 1) * s->SX;
    const double w = sc->pml_width * s->h;  // setPMLBoundaryWidth (MAC_Grid.cpp:146-150)
    const double S = sc->pml_strength;
    s->pml_strength = S;
    const double one_over_k = 1.0 / s->k;
    for (int d = 0; d < 3; ++d) {
        const int n = s->N[d];
        auto& T = s->tab[d];
        T.pml_cell.assign(n, 0);
        T.pml_face.assign(n + 1, 0);
        T.cpos.assign(n, 0.0);
        T.csig.assign(n, 0.0);
        T.fpos.assign(n + 1, 0.0);
        T.pupd.assign(n, 0.0);
        T.pdiv.assign(n, 0.0);
        T.vupd.assign(n + 1, 0.0);
        T.vgrad.assign(n + 1, 0.0);
        for (int i = 0; i < n; ++i) {
            double p = s->bmin[d];
            p += (0.5 + (double)i) * s->h;  // ScalarField::cellPosition (ScalarField.cpp:131-140)
            T.cpos[i] = p;
            T.pml_cell[i] = inside_pml_1d(p, s->bmin[d], s->bmax[d], w, s->preset, d);
            const double sigma = absorption(p, s->bmin[d], s->bmax[d], w, S, s->preset, d);
            T.csig[i] = sigma;
            const double directional = one_over_k + sigma / 2.0;           // MAC_Grid.h:550-553
            T.pupd[i] = (1.0 / s->k - sigma / 2.0) / directional;          // MAC_Grid.h:558-561
            T.pdiv[i] = (-1.0 * s->rho * s->c * s->c / directional);       // MAC_Grid.h:566-569
        }
        const double vmin = s->bmin[d] - s->h / 2.0;  // MAC_Grid.cpp:103-113
        for (int i = 0; i <= n; ++i) {
            double p = vmin;
            p += (0.5 + (double)i) * s->h;
            T.fpos[i] = p;
            T.pml_face[i] = inside_pml_1d(p, s->bmin[d], s->bmax[d], w, s->preset, d);
            const double sigma = absorption(p, s->bmin[d], s->bmax[d], w, S, s->preset, d);
            double u = 1.0 / s->k - sigma / 2.0;  // MAC_Grid.h:530-536
            u /= 1.0 / s->k + sigma / 2.0;
            T.vupd[i] = u;
            double g = 1.0 / s->k + sigma / 2.0;  // MAC_Grid.h:541-547
            g *= s->rho * s->h;
            T.vgrad[i] = -1.0 / g;
        }
    }
    // PML / interior counts
    long long inner = 1;
    for (int d = 0; d < 3; ++d) {
        long long m = 0;
        for (int i = 0; i < s->N[d]; ++i) m += s->tab[d].pml_cell[i] ? 0 : 1;
        inner *= m;
    }
    s->n_interior = inner;
    s->n_pml = s->ncell - inner;
    // non-PML box and the PML shell as six disjoint slabs (x slabs full, y slabs
    // inside the x range, z slabs inside the x and y ranges)
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = 0;
        while (lo[d] < s->N[d] && s->tab[d].pml_cell[lo[d]]) ++lo[d];
        hi[d] = s->N[d];
        while (hi[d] > lo[d] && s->tab[d].pml_cell[hi[d] - 1]) --hi[d];
        s->interior.lo[d] = lo[d];
        s->interior.hi[d] = hi[d];
    }
    const int* N = s->N;
    if (lo[0] >= hi[0] || lo[1] >= hi[1] || lo[2] >= hi[2])
        for (int d = 0; d < 3; ++d) s->interior.lo[d] = s->interior.hi[d] = 0;
    build_shell_boxes(s, FDTD_SHELL_PLANES);
    build_engquist(s);
    (void)N;
    return FDTD_OK;
}

}  // namespace fdtd

static fdtd_status validate_scene(const fdtd_scene_desc* sc) {
    if (!sc) return (set_error(nullptr, "scene is NULL"), FDTD_ERR_INVALID_ARG);
    if (!(sc->cell_size > 0) || !(sc->time_step > 0) || !(sc->sound_speed > 0) || !(sc->density > 0))
        return (set_error(nullptr, "cell_size, time_step, sound_speed and density must be positive"), FDTD_ERR_INVALID_ARG);
    for (int d = 0; d < 3; ++d)
        if (sc->divisions[d] < 4 || sc->divisions[d] > 4096)
            return (set_error(nullptr, "divisions must lie in [4, 4096]"), FDTD_ERR_INVALID_ARG);
    if ((long long)sc->divisions[0] * sc->divisions[1] * sc->divisions[2] >= (1LL << 31))
        return (set_error(nullptr, "grid has 2^31 cells or more (flat index is int32, as ScalarField)"), FDTD_ERR_INVALID_ARG);
    if (sc->boundary_condition_preset < 0 || sc->boundary_condition_preset > 2)
        return (set_error(nullptr, "boundary_condition_preset must be 0, 1 or 2"), FDTD_ERR_INVALID_ARG);
    if (!(sc->pml_width >= 0.0)) return (set_error(nullptr, "PML_width must be non-negative"), FDTD_ERR_INVALID_ARG);
    if (!(sc->air_viscosity_alpha >= 0.0))
        return (set_error(nullptr, "air_viscosity_alpha must be non-negative"), FDTD_ERR_INVALID_ARG);
    if (sc->n_objects < 0 || sc->n_objects > FDTD_MAX_OBJECTS)
        return (set_error(nullptr, "too many objects (max " + std::to_string(FDTD_MAX_OBJECTS) + ")"), FDTD_ERR_INVALID_ARG);
    if (sc->n_sources < 0 || sc->n_sources > FDTD_MAX_SOURCES)
        return (set_error(nullptr, "too many pressure sources (max " + std::to_string(FDTD_MAX_SOURCES) + ")"), FDTD_ERR_INVALID_ARG);
    if (sc->n_constraints < 0 || sc->n_constraints > 4)
        return (set_error(nullptr, "too many plane constraints (max 4)"), FDTD_ERR_INVALID_ARG);
    if (sc->n_listeners < 0 || (sc->n_listeners > 0 && !sc->listeners))
        return (set_error(nullptr, "listener array missing"), FDTD_ERR_INVALID_ARG);
    if ((sc->n_objects > 0 && !sc->objects) || (sc->n_sources > 0 && !sc->sources) ||
        (sc->n_constraints > 0 && !sc->constraints))
        return (set_error(nullptr, "scene array missing"), FDTD_ERR_INVALID_ARG);
    if (sc->n_meshes < 0 || (sc->n_meshes > 0 && !sc->meshes))
        return (set_error(nullptr, "scene mesh array missing"), FDTD_ERR_INVALID_ARG);
    if (sc->n_tracks < 0 || (sc->n_tracks > 0 && !sc->tracks))
        return (set_error(nullptr, "scene keyframe-track array missing"), FDTD_ERR_INVALID_ARG);
    for (int k = 0; k < sc->n_tracks; ++k)
        if (sc->tracks[k].object < 0 || sc->tracks[k].object >= sc->n_objects ||
            sc->objects[sc->tracks[k].object].motion != FDTD_MOTION_KEYFRAMED)
            return (set_error(nullptr, "keyframe track of an object that is not keyframed"), FDTD_ERR_INVALID_ARG);
    for (int i = 0; i < sc->n_objects; ++i) {
        const auto& o = sc->objects[i];
        if (o.shape < 0 || o.shape > FDTD_SHAPE_MESH) return (set_error(nullptr, "unknown object shape"), FDTD_ERR_INVALID_ARG);
        if (o.shape == FDTD_SHAPE_MESH) {
            if (o.mesh < 0 || o.mesh >= sc->n_meshes)
                return (set_error(nullptr, "object mesh index out of range"), FDTD_ERR_INVALID_ARG);
            MeshHost m;
            std::string err;
            if (!build_mesh(sc->meshes[o.mesh], m, err)) return (set_error(nullptr, err), FDTD_ERR_GEOMETRY);

        }
        if (o.accel_kind == FDTD_ACCEL_GAUSSIAN_PULSATION && o.shape != FDTD_SHAPE_SPHERE)
            return (set_error(nullptr, "pulsating acceleration is defined for spheres only"), FDTD_ERR_UNSUPPORTED);
        if (o.motion != FDTD_MOTION_STATIC && o.shape == FDTD_SHAPE_ELLIPSOID)
            return (set_error(nullptr, "moving ellipsoids are not supported (no closest-point query)"), FDTD_ERR_UNSUPPORTED);
        if (o.motion < FDTD_MOTION_STATIC || o.motion > FDTD_MOTION_KEYFRAMED)
            return (set_error(nullptr, "unknown object motion"), FDTD_ERR_INVALID_ARG);
        if (o.motion == FDTD_MOTION_KEYFRAMED) {
            int found = 0;
            for (int k = 0; k < sc->n_tracks; ++k)
                if (sc->tracks && sc->tracks[k].object == i) {
                    const fdtd_keyframe_track& t = sc->tracks[k];
                    if (t.n_frames < 1 || !t.frames || !(t.step > 0))
                        return (set_error(nullptr, "keyframe track needs frames and a positive step"), FDTD_ERR_INVALID_ARG);
                    for (long long q = 0; q < 7LL * t.n_frames; ++q)
                        if (!std::isfinite(t.frames[q]))
                            return (set_error(nullptr, "keyframe track has a non-finite value"), FDTD_ERR_INVALID_ARG);
                    ++found;
                }
            if (found != 1)
                return (set_error(nullptr, "a keyframed object needs exactly one keyframe track"), FDTD_ERR_INVALID_ARG);
        }
        if (o.accel_kind != FDTD_ACCEL_NONE && !(o.accel_tau > 0))
            return (set_error(nullptr, "accel_tau must be positive"), FDTD_ERR_INVALID_ARG);
        for (int d = 0; d < 3; ++d)
            if (o.shape != FDTD_SHAPE_MESH && (o.shape != FDTD_SHAPE_SPHERE || d == 0) && !(o.size[d] > 0))
                return (set_error(nullptr, "object size must be positive"), FDTD_ERR_INVALID_ARG);
    }
    for (int i = 0; i < sc->n_sources; ++i)
        if (!(sc->sources[i].width_time > 0)) return (set_error(nullptr, "source_width_time must be positive"), FDTD_ERR_INVALID_ARG);
    if (sc->boundary_handling != FDTD_BOUNDARY_RASTERIZE && sc->boundary_handling != FDTD_BOUNDARY_FULLY_COUPLED)
        return (set_error(nullptr, "unknown boundary_handling"), FDTD_ERR_INVALID_ARG);
    if (sc->boundary_handling == FDTD_BOUNDARY_FULLY_COUPLED)
        for (int i = 0; i < sc->n_objects; ++i)
            if (sc->objects[i].shape == FDTD_SHAPE_ELLIPSOID)
                return (set_error(nullptr, "FULLY_COUPLED boundaries need a closest-point query (spheres, boxes, meshes)"),
                        FDTD_ERR_UNSUPPORTED);
    return FDTD_OK;
}

// Bounding box of the Gaussian source supports (cells whose centre may lie
// strictly inside a source's box) clipped to the interior kernel's box.
static Box3 source_region(const fdtd_solver* s) {
    Box3 r{};
    const Box3 U = update_box(s);  // the Engquist cells add their sources themselves
    bool any = false;
    for (const auto& g : s->sources) {
        for (int d = 0; d < 3; ++d) {
            const double a = (g.position[d] - 2.0 * g.width_space - s->bmin[d]) / s->h - 0.5;
            const double b = (g.position[d] + 2.0 * g.width_space - s->bmin[d]) / s->h - 0.5;
            const int lo = std::max(U.lo[d], (int)std::floor(a));
            const int hi = std::min(U.hi[d], (int)std::ceil(b) + 1);
            if (!any) { r.lo[d] = lo; r.hi[d] = hi; }
            else { r.lo[d] = std::min(r.lo[d], lo); r.hi[d] = std::max(r.hi[d], hi); }
        }
        any = true;
    }
    for (int d = 0; d < 3; ++d)
        if (!any || r.hi[d] < r.lo[d]) r.hi[d] = r.lo[d];
    return r;
}

// Offsets of every device array of a solver inside its one arena allocation;
// needs the geometry (solver_init_geometry) and the listener list.
static void carve_arena(fdtd_solver* s, const fdtd_scene_desc* sc, const fdtd_options& o, Carver& cv) {
    const size_t w = s->precision == FDTD_PRECISION_FP64 ? 8 : 4;
    const long long n = s->np;  // every array uses the padded layout
    const int* N = s->N;
    SolveParams& P = s->hP;
    std::memset(&P, 0, sizeof(P));
    cv.add((void**)&s->dP, sizeof(SolveParams));
    cv.add((void**)&P.cls, n);
    cv.add((void**)&P.gobj, n);
    if (!s->eng.empty()) {
        cv.add((void**)&P.eng, s->eng.size() * sizeof(EngCell));
        cv.add((void**)&P.eng_buf, s->eng.size() * ENG_BUF * 8);
    }
    cv.add(&P.p[0], n * w);
    cv.add(&P.p[1], n * w);
    if (s->precision != FDTD_PRECISION_FP64) cv.add((void**)&P.dinc, n * 4);
    for (int d = 0; d < 3; ++d) cv.add(&P.pd[d], n * w);
    for (int d = 0; d < 3; ++d) {
        s->vcount[d] = (long long)(N[0] + (d == 0)) * (N[1] + (d == 1)) * (N[2] + (d == 2));  // dense face count
        cv.add(&P.v[0][d], n * w);
        if (o.kernel != FDTD_KERNEL_PHASED) cv.add(&P.v[1][d], n * w);  // double-buffered faces
    }
    if (o.kernel == FDTD_KERNEL_PHASED) cv.add((void**)&s->d_lap, n * 8);
    if (sc->air_viscosity_alpha > 0.0) {  // Laplacians of this and the previous step
        cv.add(&P.lapv[0], n * w);
        cv.add(&P.lapv[1], n * w);
    }
    // per-axis spatial factors of the sources
    s->region.src_region = source_region(s);
    if (!s->sources.empty())
        for (int d = 0; d < 3; ++d) cv.add((void**)&P.src_ax[d], s->sources.size() * (size_t)N[d] * 8);
    // compact storage of the z-slab box (region-split path)
    const ShellBoxes& SB = s->shell;
    if (o.kernel == FDTD_KERNEL_FUSED && SB.zbox >= 0) {
        P.zcount = (long long)SB.nx[SB.zbox] * SB.ny[SB.zbox] * SB.zrw;
        for (int d = 0; d < 3; ++d) {
            cv.add(&P.zpd[d], P.zcount * w);
            cv.add(&P.zv[0][d], P.zcount * w);
            cv.add(&P.zv[1][d], P.zcount * w);
        }
    }
    cv.add((void**)&P.consts, 2 * sizeof(StepConsts));
    cv.add((void**)&P.dev_error, 16);
    cv.add((void**)&s->d_status, 16);
    cv.add((void**)&P.listeners, std::max<size_t>(1, s->listeners.size()) * 8);
    cv.add((void**)&P.lis_rows, (size_t)std::max(1, s->L) * 64 * sizeof(LisRow));
    cv.add((void**)&P.lis_plan, (size_t)std::max(1, s->L) * sizeof(LisPlan));
    for (int d = 0; d < 3; ++d) {
        cv.add((void**)&P.pml_cell[d], N[d]);
        cv.add((void**)&P.pml_face[d], N[d] + 1);
        cv.add((void**)&P.cpos[d], N[d] * 8);
        cv.add((void**)&P.fpos[d], (N[d] + 1) * 8);
        cv.add((void**)&P.pupd[d], N[d] * 8);
        cv.add((void**)&P.pdiv[d], N[d] * 8);
        cv.add((void**)&P.vupd[d], (N[d] + 1) * 8);
        cv.add((void**)&P.vgrad[d], (N[d] + 1) * 8);
        cv.add((void**)&P.pupd_f[d], N[d] * 4);
        cv.add((void**)&P.pdiv_f[d], N[d] * 4);
        cv.add((void**)&P.vupd_f[d], (N[d] + 1) * 4);
        cv.add((void**)&P.vgrad_f[d], (N[d] + 1) * 4);
        // N+8 entries: z-vector groups of the shell kernel read up to 7 past N (zeros)
        cv.add((void**)&P.axflag[d], N[d] + 8);
        cv.add((void**)&P.coef_d[d], (N[d] + 8) * sizeof(AxisCoef<double>));
        cv.add((void**)&P.coef_f[d], (N[d] + 8) * sizeof(AxisCoef<float>));
    }
    s->lis_cap_steps = std::max(256, o.graph_steps);
    cv.add((void**)&s->d_lis, (size_t)s->lis_cap_steps * std::max(1, s->L) * 8);
    // ghost-neighbour list: at most 6 bulk neighbours per solid cell; solid cells lie
    // in the object boxes (dilated by 2 cells, and by the travel of moving bodies)
    {
        double cells = 4096;
        for (int i = 0; i < sc->n_objects; ++i) {
            HostObject tmp = make_host_object(sc, i);
            host_object_pose(tmp, sc->start_time);
            host_update_bbox(tmp);
            double vol = 1.0;
            for (int d = 0; d < 3; ++d) {
                double ext = (tmp.bmax[d] - tmp.bmin[d]) / s->h + 4.0;
                if (tmp.d.motion != FDTD_MOTION_STATIC) ext *= 2.0;
                vol *= std::min(ext, (double)N[d]);
            }
            cells += 6.0 * vol;
        }
        cells += 2.0 * sc->n_constraints * ((double)N[0] * N[1] + (double)N[1] * N[2] + (double)N[0] * N[2]);
        s->region.ghost_cap = (int)std::min<double>(cells, (double)n);
        cv.add((void**)&s->d_ghost_list, (size_t)s->region.ghost_cap * 4);
        cv.add((void**)&s->d_ghost_count, 16);
        // fresh cells were solid the step before: fewer than the solid cells of the boxes
        P.fresh_cap = s->moving ? s->region.ghost_cap : 0;
        cv.add((void**)&P.fresh_list, (size_t)std::max(1, P.fresh_cap) * 4);
    }
}

extern "C" {

int32_t fdtd_abi_version(void) { return FDTD_ABI_VERSION; }

const char* fdtd_last_error(void) { return g_last_error.c_str(); }

fdtd_status fdtd_device_count(int32_t* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        set_error(nullptr, cudaGetErrorString(e));
        return FDTD_ERR_CUDA;
    }
    *count = n;
    return FDTD_OK;
}

fdtd_status fdtd_debug_inject_failure(int32_t what, int32_t after) {
    if (what < FDTD_INJECT_NONE || what > FDTD_INJECT_HOST_ALLOC || after < 0)
        return (set_error(nullptr, "fdtd_debug_inject_failure: invalid arguments"), FDTD_ERR_INVALID_ARG);
    g_inject_what.store(FDTD_INJECT_NONE);
    g_inject_after.store(after);
    g_inject_what.store(what);
    return FDTD_OK;
}

fdtd_status fdtd_gaussian_source_defaults(fdtd_gaussian_source_desc* src, double sound_speed) {
    if (!src) return FDTD_ERR_INVALID_ARG;
    // ImpulseResponseParser.cpp:660-663
    if (src->width_space <= 0) src->width_space = sound_speed * src->width_time;
    if (src->normalize_constant == 0)
        src->normalize_constant = 1.0 / std::pow(std::sqrt(2.0 * M_PI) * src->width_space, 3);
    return FDTD_OK;
}

fdtd_status fdtd_solver_create(const fdtd_scene_desc* sc, const fdtd_options* opt, fdtd_solver** out) {
    if (!out) return (set_error(nullptr, "out is NULL"), FDTD_ERR_INVALID_ARG);
    *out = nullptr;
    fdtd_status st = validate_scene(sc);
    if (st != FDTD_OK) return st;
    fdtd_options o{};
    if (opt) o = *opt;
    if (o.precision != FDTD_PRECISION_FP64 && o.precision != FDTD_PRECISION_FP32_COMPENSATED)
        return (set_error(nullptr, "unknown precision"), FDTD_ERR_INVALID_ARG);
    if (o.kernel != FDTD_KERNEL_FUSED && o.kernel != FDTD_KERNEL_PHASED)
        return (set_error(nullptr, "unknown kernel path"), FDTD_ERR_INVALID_ARG);
    if (o.kernel == FDTD_KERNEL_PHASED && o.precision != FDTD_PRECISION_FP64)
        return (set_error(nullptr, "the phased kernel path is FP64 only"), FDTD_ERR_INVALID_ARG);
    if (o.graph_steps < 0 || (o.graph_steps % 2) != 0)
        return (set_error(nullptr, "graph_steps must be a non-negative even number"), FDTD_ERR_INVALID_ARG);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return (set_error(nullptr, "no CUDA device visible"), FDTD_ERR_CUDA);
    if (o.device < 0 || o.device >= ndev) return (set_error(nullptr, "device ordinal out of range"), FDTD_ERR_INVALID_ARG);

    if (sc->boundary_handling == FDTD_BOUNDARY_FULLY_COUPLED && o.kernel != FDTD_KERNEL_FUSED)
        return (set_error(nullptr, "FULLY_COUPLED boundaries run on the fused kernels"), FDTD_ERR_UNSUPPORTED);
    std::unique_ptr<fdtd_solver> s(new fdtd_solver());
    // a failure below releases what was created so far (streams, events, memory)
    struct Release {
        std::unique_ptr<fdtd_solver>& s;
        ~Release() {
            if (s) fdtd_solver_destroy(s.release());
        }
    } release{s};
    s->opt = o;
    s->precision = o.precision;
    s->boundary_handling = sc->boundary_handling;
    CUDA_TRY(nullptr, cudaSetDevice(o.device));
    bool any_moving = false;
    for (int i = 0; i < sc->n_objects; ++i) any_moving = any_moving || sc->objects[i].motion != FDTD_MOTION_STATIC;
    if (any_moving) {
        // moving bodies: the classification on the solver stream goes before the
        // blocks of the PML shell that runs beside it on stream5
        int least = 0, greatest = 0;
        CUDA_TRY(nullptr, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_TRY(nullptr, cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, greatest));
    } else {
        CUDA_TRY(nullptr, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    }
    {
        // moving bodies: the interior and ghost-list CTAs go before the remaining
        // CTAs of the shell that started beside the classification (FP64 moving
        // step 0.356 -> 0.344 ms; FP32 unchanged)
        int least = 0, greatest = 0;
        CUDA_TRY(nullptr, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int pr = any_moving ? greatest : least;
        CUDA_TRY(nullptr, cudaStreamCreateWithPriority(&s->stream2, cudaStreamNonBlocking, pr));
        CUDA_TRY(nullptr, cudaStreamCreateWithPriority(&s->stream3, cudaStreamNonBlocking, pr));
    }
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_ghost, cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaStreamCreateWithFlags(&s->stream4, cudaStreamNonBlocking));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_step, cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_lis[0], cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_lis[1], cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_lis_join, cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaStreamCreateWithFlags(&s->stream5, cudaStreamNonBlocking));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_sfork, cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_sdone, cudaEventDisableTiming));
    if (s->precision == FDTD_PRECISION_FP32_COMPENSATED) CUDA_TRY(nullptr, prepare_fp32_kernels());
    else CUDA_TRY(nullptr, prepare_fp64_kernels());
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(nullptr, cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    solver_init_geometry(s.get(), sc);
    if (!s->eng.empty() && o.kernel == FDTD_KERNEL_PHASED) {
        set_error(nullptr, "the phased kernel path needs a PML of 1.5 cells or more on every side");
        return FDTD_ERR_UNSUPPORTED;
    }
    if (s->np >= (1LL << 31)) {
        set_error(nullptr, "grid too large: cell indices are 32-bit (padded cells >= 2^31)");
        return FDTD_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < sc->n_objects; ++i) {
        HostObject h = make_host_object(sc, i);
        s->objs.push_back(h);
        if (h.d.motion != FDTD_MOTION_STATIC) s->moving = true;
    }
    // meshes of the objects: hierarchy and pseudo-normals (validated above)
    s->meshes.resize(sc->n_meshes);
    for (int i = 0; i < sc->n_objects; ++i) {
        const int m = sc->objects[i].shape == FDTD_SHAPE_MESH ? sc->objects[i].mesh : -1;
        if (m < 0 || !s->meshes[m].tris.empty()) continue;
        std::string err;
        if (!build_mesh(sc->meshes[m], s->meshes[m], err)) {
            set_error(nullptr, err);
            return FDTD_ERR_GEOMETRY;
        }
    }
    // keyframe tracks and mesh vertices the objects read after creation: solver-owned copies
    s->kf_store.resize(s->objs.size());
    for (size_t i = 0; i < s->objs.size(); ++i) {
        HostObject& o = s->objs[i];
        if (o.kf) {
            s->kf_store[i].assign(o.kf, o.kf + 7 * (size_t)o.kf_n);
            o.kf = s->kf_store[i].data();
        }
        if (o.d.shape == FDTD_SHAPE_MESH) {
            o.mv = s->meshes[o.d.mesh].vertices.data();
            o.mv_n = (int)(s->meshes[o.d.mesh].vertices.size() / 3);
        }
    }
    for (int i = 0; i < sc->n_constraints; ++i) s->planes.push_back(sc->constraints[i]);
    for (int i = 0; i < sc->n_sources; ++i) {
        fdtd_gaussian_source_desc g = sc->sources[i];
        fdtd_gaussian_source_defaults(&g, s->c);
        s->sources.push_back(g);
    }
    s->listeners.assign(sc->listeners, sc->listeners + 3 * (size_t)sc->n_listeners);
    s->L = sc->n_listeners;
    s->start_time = sc->start_time;

    // ---- device arena ----
    Carver cv;
    carve_arena(s.get(), sc, o, cv);
    const long long n = s->ncell;
    const int* N = s->N;
    SolveParams& P = s->hP;
    void* base = nullptr;
    size_t block = 0;
    cudaError_t e = inject_failure(FDTD_INJECT_DEVICE_ALLOC) ? cudaErrorMemoryAllocation
                                                             : arena_acquire(o.device, cv.off, &base, &block);
    if (e != cudaSuccess) {
        set_error(nullptr, std::string("cudaMalloc of ") + std::to_string(cv.off) + " bytes failed: " + cudaGetErrorString(e));
        return FDTD_ERR_OOM;
    }
    s->arena = base;
    s->arena_block = block;
    s->arena_bytes = cv.off;
    for (auto& r : cv.req) *r.first = (char*)base + r.second;
    const long long ncell = s->ncell;
    // meshes: hierarchy and triangles, one device allocation each
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        const MeshHost& M = s->meshes[m];
        if (M.tris.empty()) continue;
        const size_t nb = M.nodes.size() * sizeof(MeshNode), tb = M.tris.size() * sizeof(MeshTri);
        void* d = nullptr;
        CUDA_TRY(nullptr, cudaMalloc(&d, nb + tb));
        s->mesh_alloc.push_back(d);
        s->arena_bytes += nb + tb;
        CUDA_TRY(nullptr, fdtd::counted_copy(s.get(), d, M.nodes.data(), nb, cudaMemcpyHostToDevice));
        CUDA_TRY(nullptr, fdtd::counted_copy(s.get(), (char*)d + nb, M.tris.data(), tb, cudaMemcpyHostToDevice));
        const MeshView v{(const MeshNode*)d, (const MeshTri*)((char*)d + nb), (int)M.nodes.size(), (int)M.tris.size()};
        for (auto& o : s->objs)
            if (o.d.shape == FDTD_SHAPE_MESH && o.d.mesh == (int)m) o.mview = v;
    }

    // ---- constants ----
    for (int d = 0; d < 3; ++d) {
        P.N[d] = N[d];
        P.bmin[d] = s->bmin[d];
        for (int e2 = 0; e2 < 3; ++e2) P.vN[d][e2] = N[e2] + (d == e2 ? 1 : 0);
        P.vcount[d] = s->vcount[d];
    }
    P.ncell = ncell;
    P.SX = s->SX;
    P.SY = s->SY;
    P.np = s->np;
    P.h = s->h;
    P.inv_h = 1.0 / s->h;
    P.rho = s->rho;
    P.c = s->c;
    P.k = s->k;
    P.c2k2 = (s->c * s->k) * (s->c * s->k);
    P.kcalp = s->c * sc->air_viscosity_alpha * s->k;  // MAC_Grid.cpp:486
    P.visc = sc->air_viscosity_alpha > 0.0 ? 1 : 0;
    P.lap_scale = 1.0 / (s->h * s->h);
    P.q = 0.75 * s->h;
    P.quarter_h = 0.25 * s->h;
    P.n_obj = (int)s->objs.size();
    P.n_plane = (int)s->planes.size();
    P.n_src = (int)s->sources.size();
    P.n_lis = s->L;
    P.precision = s->precision;
    P.ghost_list = s->d_ghost_list;
    P.ghost_count = s->d_ghost_count;
    P.ghost_cap = s->region.ghost_cap;
    P.fresh_count = s->d_ghost_count + 1;
    s->region.interior = update_box(s.get());
    P.eng_n = (int)s->eng.size();
    P.eng_lambda = s->c * s->k / s->h;  // MAC_Grid.cpp:488
    if (P.eng_n > 0)
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.eng, s->eng.data(), s->eng.size() * sizeof(EngCell),
                                             cudaMemcpyHostToDevice));
    s->region.shell = s->shell;
    s->region.sources = 0;
    for (int i = 0; i < P.n_plane; ++i) {
        P.plane[i].dir = s->planes[i].normal_dir;
        P.plane[i].sign = s->planes[i].normal_sign;
        P.plane[i].height = s->planes[i].height;
    }
    for (int i = 0; i < P.n_src; ++i) {
        const auto& g = s->sources[i];
        DevSource& D = P.src[i];
        // GaussianPressureSource bbox (GaussianPressureSource.h:34-37) and centroid (FDTD_MovableObject.h:54-58)
        for (int d = 0; d < 3; ++d) {
            D.bmin[d] = g.position[d] - g.width_space * GAUSSIAN_CHECK_BOUND;
            D.bmax[d] = g.position[d] + g.width_space * GAUSSIAN_CHECK_BOUND;
            D.cen[d] = (D.bmax[d] + D.bmin[d]) / 2.0;
        }
        D.denom = 2.0 * g.width_space * g.width_space;
        D.t0 = g.offset_time;
        D.wt = g.width_time;
        D.scale = 1. / 3.6836 * g.normalize_constant;
    }
    // Gaussian sources (GaussianPressureSource.cpp:6-30): zero outside the box
    // x_s +- 2 sigma_s (strict, per axis), exp(-|x - x_s|^2 / 2 sigma_s^2) * scale
    // inside, the product of one factor per axis
    if (!s->sources.empty())
        for (int d = 0; d < 3; ++d) {
            std::vector<double> g(s->sources.size() * (size_t)N[d], 0.0);
            for (size_t i = 0; i < s->sources.size(); ++i) {
                const DevSource& S = P.src[i];
                for (int x = 0; x < N[d]; ++x) {
                    const double px = s->tab[d].cpos[x];
                    if (!(px < S.bmax[d] && px > S.bmin[d])) continue;
                    double v = std::exp(-((px - S.cen[d]) * (px - S.cen[d])) / S.denom);
                    if (d == 0) v *= S.scale;
                    g[i * N[d] + x] = v;
                }
            }
            CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.src_ax[d], g.data(), g.size() * 8, cudaMemcpyHostToDevice));
        }
    // tables
    for (int d = 0; d < 3; ++d) {
        auto& T = s->tab[d];
        std::vector<float> f1(T.pupd.begin(), T.pupd.end()), f2(T.pdiv.begin(), T.pdiv.end());
        std::vector<float> f3(T.vupd.begin(), T.vupd.end()), f4(T.vgrad.begin(), T.vgrad.end());
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pml_cell[d], T.pml_cell.data(), N[d], cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pml_face[d], T.pml_face.data(), N[d] + 1, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.cpos[d], T.cpos.data(), N[d] * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.fpos[d], T.fpos.data(), (N[d] + 1) * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pupd[d], T.pupd.data(), N[d] * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pdiv[d], T.pdiv.data(), N[d] * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.vupd[d], T.vupd.data(), (N[d] + 1) * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.vgrad[d], T.vgrad.data(), (N[d] + 1) * 8, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pupd_f[d], f1.data(), N[d] * 4, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.pdiv_f[d], f2.data(), N[d] * 4, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.vupd_f[d], f3.data(), (N[d] + 1) * 4, cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.vgrad_f[d], f4.data(), (N[d] + 1) * 4, cudaMemcpyHostToDevice));
        // packed flags and coefficient quads of the shell kernel
        std::vector<uint8_t> fl(N[d] + 8, 0);
        std::vector<AxisCoef<double>> cd(N[d] + 8, AxisCoef<double>{0.0, 0.0, 0.0, 0.0});
        std::vector<AxisCoef<float>> cf(N[d] + 8, AxisCoef<float>{0.0f, 0.0f, 0.0f, 0.0f});
        for (int i = 0; i <= N[d]; ++i) {
            uint8_t f = 0;
            if (i < N[d]) {
                if (T.pml_cell[i]) f |= AXF_PML;
                if (i > 0 && T.pml_face[i]) f |= AXF_FACE_LO;
                if (i + 1 < N[d] && T.pml_face[i + 1]) f |= AXF_FACE_HI;
                if (i + 1 < N[d] && T.pml_cell[i + 1]) f |= AXF_NEXT_PML;
                if (i > 0) f |= AXF_HAS_LO;
                if (i + 1 < N[d]) f |= AXF_HAS_HI;
            }
            fl[i] = f;
            cd[i].vupd = T.vupd[i];
            cd[i].vgrad = T.vgrad[i];
            cd[i].pupd = i < N[d] ? T.pupd[i] : 0.0;
            cd[i].pdiv = i < N[d] ? T.pdiv[i] : 0.0;
            cf[i].vupd = (float)cd[i].vupd;
            cf[i].vgrad = (float)cd[i].vgrad;
            cf[i].pupd = (float)cd[i].pupd;
            cf[i].pdiv = (float)cd[i].pdiv;
        }
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.axflag[d], fl.data(), fl.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.coef_d[d], cd.data(), cd.size() * sizeof(cd[0]), cudaMemcpyHostToDevice));
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.coef_f[d], cf.data(), cf.size() * sizeof(cf[0]), cudaMemcpyHostToDevice));
    }
    if (s->L > 0)
        CUDA_TRY(s.get(), fdtd::counted_copy(s.get(), (void*)P.listeners, s->listeners.data(), s->listeners.size() * 8, cudaMemcpyHostToDevice));
    CUDA_TRY(s.get(), inject_failure(FDTD_INJECT_HOST_ALLOC)
                          ? cudaErrorMemoryAllocation
                          : cudaMallocHost((void**)&s->h_lis_stage, (size_t)s->lis_cap_steps * std::max(1, s->L) * 8));
    s->xb = (o.x_chunk == 2 || o.x_chunk == 4 || o.x_chunk == 8) ? o.x_chunk : 2;
    s->region.xb = s->xb;
    // tile_y: x planes each PML-shell thread marches over
    if (o.kernel == FDTD_KERNEL_FUSED && o.tile_y > 0) build_shell_boxes(s.get(), std::min(o.tile_y, 256));
    s->region.shell = s->shell;
    st = fdtd_solver_reset(s.get(), sc->start_time);
    if (st != FDTD_OK) return st;
    *out = s.release();
    return FDTD_OK;
}

void fdtd_release_cached_memory(int32_t device) { fdtd::free_kept(device); }

fdtd_status fdtd_solver_destroy(fdtd_solver* s) {
    if (!s) return FDTD_OK;
    cudaSetDevice(s->opt.device);
    // (also releases a solver whose creation failed part way: null handles are skipped)
    for (cudaStream_t st : {s->stream, s->stream2, s->stream3, s->stream4, s->stream5})
        if (st) cudaStreamSynchronize(st);
    for (int i = 0; i < 4; ++i)
        if (s->graph_exec[i]) cudaGraphExecDestroy(s->graph_exec[i]);
    free_fully_coupled(s);
    free_shell_tma(s);
    for (void* p : s->mesh_alloc) cudaFree(p);
    if (s->d_solid_pml) cudaFree(s->d_solid_pml);
    if (s->arena) arena_release(s->opt.device, s->arena, s->arena_block);
    if (s->h_lis_stage) cudaFreeHost(s->h_lis_stage);
    for (cudaEvent_t ev : {s->ev_fork, s->ev_join, s->ev_ghost, s->ev_step, s->ev_lis[0], s->ev_lis[1], s->ev_lis_join,
                           s->ev_sfork, s->ev_sdone})
        if (ev) cudaEventDestroy(ev);
    for (cudaStream_t st : {s->stream2, s->stream3, s->stream4, s->stream5, s->stream})
        if (st) cudaStreamDestroy(st);
    delete s;
    return FDTD_OK;
}

// PML_WaveSolver::Reinitialize_PML_WaveSolver(true, t0) (PML_WaveSolver.cpp:102-146)
// + FDTD_AcousticSimulator::ResetStartTime (FDTD_AcousticSimulator.cpp:458-523)
fdtd_status fdtd_solver_reset(fdtd_solver* s, double t0) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    SolveParams& P = s->hP;
    const size_t w = s->precision == FDTD_PRECISION_FP64 ? 8 : 4;
    // zero all state (fields, velocities, split pressures, flags; padding included)
    const long long np = s->np;
    CUDA_TRY(s, cudaMemsetAsync(P.p[0], 0, np * w, s->stream));
    CUDA_TRY(s, cudaMemsetAsync(P.p[1], 0, np * w, s->stream));
    if (P.dinc) CUDA_TRY(s, cudaMemsetAsync(P.dinc, 0, np * 4, s->stream));
    for (int b = 0; b < 2; ++b)
        if (P.lapv[b]) CUDA_TRY(s, cudaMemsetAsync(P.lapv[b], 0, np * w, s->stream));
    for (int d = 0; d < 3; ++d) {
        CUDA_TRY(s, cudaMemsetAsync(P.pd[d], 0, np * w, s->stream));
        CUDA_TRY(s, cudaMemsetAsync(P.v[0][d], 0, np * w, s->stream));
        if (P.v[1][d]) CUDA_TRY(s, cudaMemsetAsync(P.v[1][d], 0, np * w, s->stream));
        if (P.zcount > 0) {
            CUDA_TRY(s, cudaMemsetAsync(P.zpd[d], 0, P.zcount * w, s->stream));
            CUDA_TRY(s, cudaMemsetAsync(P.zv[0][d], 0, P.zcount * w, s->stream));
            CUDA_TRY(s, cudaMemsetAsync(P.zv[1][d], 0, P.zcount * w, s->stream));
        }
    }
    // initFieldRasterized: every cell bulk with valid history (MAC_Grid.cpp:2459-2470, :4170-4180)
    CUDA_TRY(s, cudaMemsetAsync(P.cls, CLS_BULK | CLS_VALID, np, s->stream));
    if (P.eng_buf) CUDA_TRY(s, cudaMemsetAsync(P.eng_buf, 0, s->eng.size() * ENG_BUF * 8, s->stream));
    CUDA_TRY(s, cudaMemsetAsync(P.gobj, GOBJ_NONE, np, s->stream));
    CUDA_TRY(s, cudaMemsetAsync(P.consts, 0, 2 * sizeof(StepConsts), s->stream));
    CUDA_TRY(s, cudaMemsetAsync(P.dev_error, 0, sizeof(int), s->stream));
    CUDA_TRY(s, cudaMemsetAsync(s->d_status, 0, 16, s->stream));
    s->time = t0;
    s->state_time = t0;
    s->step_index = 0;
    s->cur = 0;
    for (auto& o : s->objs) {
        host_object_pose(o, t0);
        host_update_bbox(o);
        host_reset_union(o);
    }
    for (size_t i = 0; i < s->objs.size(); ++i) to_dev_object(s->objs[i], P.obj[i]);
    s->n_solid_pml = 0;
    P.solid_pml = nullptr;
    P.n_solid_pml = 0;
    P.lis_ready = 0;  // the first step classifies and rebuilds the listener fits
    fdtd_status st = upload_params(s);
    if (st != FDTD_OK) return st;
    CUDA_TRY(s, launch_consts_init(s->dP, t0, s->stream));
    s->launches = 0;
    st = run_classification(s);
    if (st != FDTD_OK) return st;
    // ResetCellHistory(true): every cell has a valid history after reset (the
    // classification kernels keep it in bit 6; set it on all cells), and the
    // solid cells inside the PML, re-zeroed every step of a static scene
    int* d_count = s->d_status + 3;
    int n_solid = 0;
    CUDA_TRY(s, cudaMemsetAsync(d_count, 0, sizeof(int), s->stream));
    CUDA_TRY(s, launch_cls_history(s->dP, s->ncell, d_count, nullptr, 0, s->stream));
    CUDA_TRY(s, fdtd::counted_copyAsync(s, &n_solid, d_count, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->d_solid_pml) {
        cudaFree(s->d_solid_pml);
        s->d_solid_pml = nullptr;
    }
    if (n_solid > 0 && !s->moving) {
        CUDA_TRY(s, cudaMalloc((void**)&s->d_solid_pml, (size_t)n_solid * sizeof(int)));
        CUDA_TRY(s, cudaMemsetAsync(d_count, 0, sizeof(int), s->stream));
        CUDA_TRY(s, launch_cls_history(s->dP, s->ncell, d_count, s->d_solid_pml, n_solid, s->stream));
        P.solid_pml = s->d_solid_pml;
        P.n_solid_pml = n_solid;
        s->n_solid_pml = P.n_solid_pml;
    }
    CUDA_TRY(s, cudaMemsetAsync(d_count, 0, sizeof(int), s->stream));
    if (s->boundary_handling == FDTD_BOUNDARY_FULLY_COUPLED) {
        st = build_fully_coupled(s);
        if (st != FDTD_OK) return st;
    }
    s->region.fc = P.fc_n > 0 ? 1 : 0;
    s->region.red = use_reduced_pml(s, n_solid == 0) ? 1 : 0;
    // reduced state: the TMA-staged shell kernel where it applies (tiles and
    // tensor maps of this solve), else the per-thread cp.async kernel
    free_shell_tma(s);
    // (moving scenes run the shell beside the per-step classification on a
    // low-priority stream: a persistent kernel would hold every SM the
    // classification chain needs, so they keep the per-thread kernel)
    if (s->region.red && s->opt.shell_staging == FDTD_SHELL_STAGING_TMA && !s->moving) {
        st = build_shell_tma(s);
        if (st != FDTD_OK && st != FDTD_ERR_UNSUPPORTED) return st;
        if (st == FDTD_ERR_UNSUPPORTED) s->err.clear();
    }
    // default x planes per shell thread of the state in effect (tile_y overrides)
    if (s->opt.kernel == FDTD_KERNEL_FUSED) {
        const int xs = shell_planes(s, s->opt.tile_y);
        if (s->shell.xs != xs) build_shell_boxes(s, xs);
        s->region.shell = s->shell;
    }
    st = upload_params(s);
    if (st != FDTD_OK) return st;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    for (int i = 0; i < 4; ++i) {
        if (s->graph_exec[i]) cudaGraphExecDestroy(s->graph_exec[i]);
        s->graph_exec[i] = nullptr;
    }
    return FDTD_OK;
}

fdtd_status fdtd_scene_info(const fdtd_scene_desc* sc, const fdtd_options* opt, fdtd_solver_info* info) {
    if (!info) return (set_error(nullptr, "info is NULL"), FDTD_ERR_INVALID_ARG);
    fdtd_status st = validate_scene(sc);
    if (st != FDTD_OK) return st;
    fdtd_options o{};
    if (opt) o = *opt;
    fdtd_solver s;
    s.opt = o;
    s.precision = o.precision;
    solver_init_geometry(&s, sc);
    for (int i = 0; i < sc->n_sources; ++i) {
        fdtd_gaussian_source_desc g = sc->sources[i];
        fdtd_gaussian_source_defaults(&g, s.c);
        s.sources.push_back(g);
    }
    s.listeners.assign(sc->listeners, sc->listeners + 3 * (size_t)sc->n_listeners);
    s.L = sc->n_listeners;
    Carver cv;
    carve_arena(&s, sc, o, cv);
    std::memset(info, 0, sizeof(*info));
    for (int d = 0; d < 3; ++d) info->divisions[d] = s.N[d];
    info->n_listeners = s.L;
    info->n_cells = s.ncell;
    info->n_pml_cells = s.n_pml;
    info->n_interior_cells = s.n_interior;
    info->device_bytes = (int64_t)cv.off;
    // meshes: triangles plus a hierarchy of at most two nodes per triangle
    std::vector<char> counted(std::max(0, sc->n_meshes), 0);
    for (int i = 0; i < sc->n_objects; ++i) {
        const int m = sc->objects[i].shape == FDTD_SHAPE_MESH ? sc->objects[i].mesh : -1;
        if (m < 0 || counted[m]) continue;
        counted[m] = 1;
        info->device_bytes += (int64_t)sc->meshes[m].n_triangles * (int64_t)(sizeof(MeshTri) + 2 * sizeof(MeshNode));
    }
    info->time = sc->start_time;
    info->time_step = s.k;
    const double w = s.precision == FDTD_PRECISION_FP64 ? 8.0 : 4.0;
    info->algorithmic_bytes_per_step = w * (3.0 * (double)s.n_interior + 14.0 * (double)s.n_pml);
    return FDTD_OK;
}

int64_t fdtd_scene_device_bytes(const fdtd_scene_desc* sc, const fdtd_options* opt) {
    fdtd_solver_info info;
    if (fdtd_scene_info(sc, opt, &info) != FDTD_OK) return -1;
    return info.device_bytes;
}

}  // extern "C"
