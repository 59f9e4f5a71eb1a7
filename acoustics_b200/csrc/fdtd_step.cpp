// fdtd_step.cpp — the step loop (SimWorld::StepWorld -> RunForSteps(1) ->
// PML_WaveSolver::stepSystem -> FetchPressureData, SimWorld.cpp:507-600), CUDA
// graph capture of static scenes, read-back and snapshot/restore.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_device.cuh"
#include "fdtd_internal.hpp"
#include "fdtd_launch.hpp"

using namespace fdtd;

#define CUDA_TRY(s, expr)                                                                   \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) {                                                            \
            set_error((s), std::string("CUDA: ") + cudaGetErrorString(_e) + " at " #expr); \
            return _e == cudaErrorMemoryAllocation ? FDTD_ERR_OOM : FDTD_ERR_CUDA;          \
        }                                                                                   \
    } while (0)

namespace {

// Classification over the boxes already in s->hP.boxes.
void classification_launches(fdtd_solver* s, fdtd_status& st, const ClsBoxes* prev) {
    const ClsBoxes& B = s->hP.boxes;
    // pageable source: the copy is staged before the call returns
    cudaError_t e = fdtd::counted_copyAsync(s, &s->dP->boxes, &B, sizeof(ClsBoxes), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = launch_classify(s->dP, s->N, B, s->moving, s->stream, prev);
    s->launches += B.ufirst[B.n] > 0 ? 3 : 2;
    if (e != cudaSuccess) {
        set_error(s, std::string("classification launch: ") + cudaGetErrorString(e));
        st = FDTD_ERR_CUDA;
    }
}

// Every box with cells lies inside the non-PML box, two cells from its faces.
// The classification writes pressures only at solid cells (in the boxes of
// this step) and fresh cells (in those of the step before); the shell kernel
// reads and writes the PML cells and reads one cell beyond them.
bool boxes_clear_of_shell(const fdtd_solver* s, const ClsBoxes& B) {
    for (int b = 0; b < B.n; ++b) {
        if (B.first[b + 1] == B.first[b]) continue;
        for (int d = 0; d < 3; ++d)
            if (B.lo[b][d] < s->interior.lo[d] + 2 || B.lo[b][d] + B.rg[b][d] > s->interior.hi[d] - 2) return false;
    }
    return true;
}

// True when a Gaussian source may contribute at a step starting at time t:
// exp(-u^2/2) underflows to zero for |u| > 38.6 (GaussianPressureSource.cpp:21-24).
bool sources_active(const fdtd_solver* s, double t) {
    const double ts = t + 0.5 * s->k;
    for (const auto& g : s->sources)
        if (std::fabs((ts - g.offset_time) / g.width_time) < 40.0) return true;
    return false;
}

// Sources active at any step of [t, t + n k)
bool sources_active_window(const fdtd_solver* s, double t, int n) {
    for (const auto& g : s->sources) {
        const double a = (t + 0.5 * s->k - g.offset_time) / g.width_time;
        const double b = (t + (n - 0.5) * s->k - g.offset_time) / g.width_time;
        if (b > -40.0 && a < 40.0) return true;
    }
    return false;
}

// The Laplacian array of the phased path: with air viscosity the one of the
// step's parity (the previous step's stays for the update), else the single one.
double* phased_lap(const fdtd_solver* s, int cur) {
    return s->hP.visc ? (double*)s->hP.lapv[cur] : s->d_lap;
}

StepStreams step_streams(const fdtd_solver* s) {
    return StepStreams{s->stream, s->stream2, s->stream3, s->ev_fork, s->ev_join, s->ev_ghost};
}

// Listener rows of static scenes run on stream4 beside the next step.  Not for
// moving bodies or solid cells inside the PML: the next step's classification /
// prologue rewrites cells of the pressure they read.
// True when no listener stencil (the cells its MLS may read, two cells around
// them) meets a classification box: the classification of the next step writes
// flags and pressures only inside its boxes, its fresh cells lie in the boxes of
// this step.
bool listeners_clear_of(const fdtd_solver* s, const ClsBoxes& B) {
    for (int l = 0; l < s->L; ++l) {
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            const double diff = (s->listeners[3 * (size_t)l + d] - s->bmin[d]) - s->h / 2.0;
            const int a0 = std::min(std::max((int)(diff / s->h), 0), s->N[d] - 1);
            lo[d] = a0 - 2;
            hi[d] = a0 + 4;
        }
        for (int b = 0; b < B.n; ++b) {
            if (B.first[b + 1] == B.first[b]) continue;
            bool meet = true;
            for (int d = 0; d < 3; ++d) meet = meet && lo[d] < B.lo[b][d] + B.rg[b][d] && B.lo[b][d] < hi[d];
            if (meet) return false;
        }
    }
    return true;
}

// The listener rows of a step run on stream4 beside the next step: static
// scenes after their first step, moving scenes while every listener stencil is
// clear of this step's classification boxes (the next step waits for them if
// its own boxes reach a stencil).  Not with Engquist cells (the step after
// writes the exterior cells of the pressure they read) or solids in the PML
// (re-zeroed at the start of every step).
bool listeners_aside(const fdtd_solver* s, bool classify) {
    if (!s->stream4 || s->n_solid_pml != 0 || !s->eng.empty()) return false;
    return s->moving ? listeners_clear_of(s, s->hP.boxes) : !classify;
}

// Make the solver stream wait for every listener launch on stream4.
fdtd_status join_listeners(fdtd_solver* s) {
    if (!s->lis_pending[0] && !s->lis_pending[1]) return FDTD_OK;
    CUDA_TRY(s, cudaEventRecord(s->ev_lis_join, s->stream4));
    CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_lis_join, 0));
    s->lis_pending[0] = s->lis_pending[1] = false;
    return FDTD_OK;
}

// Enqueue one time step with the pressure parity `cur`; listener row to dev_row.
fdtd_status enqueue_step(fdtd_solver* s, int cur, double* dev_row, bool classify, bool src) {
    s->region.sources = src ? 1 : 0;
    fdtd_status st = FDTD_OK;
    // this step writes the pressure slot the listeners of the step before last read
    if (s->lis_pending[cur]) {
        CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_lis[cur], 0));
        s->lis_pending[cur] = false;
    }
    const bool fused = s->opt.kernel == FDTD_KERNEL_FUSED;
    bool shell_ahead = false;
    if (classify) {
        // MAC_Grid::classifyCells_FAST + InterpolateFreshPressureCell (PML_WaveSolver.cpp:807-812)
        const ClsBoxes prev = s->hP.boxes;
        classification_boxes(s, s->hP.boxes);
        // the rows of the step before still being read beside this step: this
        // step's classification must not write under a listener stencil first
        if (s->lis_pending[cur ^ 1] && !listeners_clear_of(s, s->hP.boxes)) {
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_lis[cur ^ 1], 0));
            s->lis_pending[cur ^ 1] = false;
        }
        if (s->moving && s->region.red && !boxes_clear_of_shell(s, s->hP.boxes)) {
            // past the end time the bodies were checked for: the reduced PML state no longer holds
            set_error(s, "a moving body came within two cells of the PML of a reduced-state solve (past its end_time)");
            return FDTD_ERR_UNSUPPORTED;
        }
        // Moving bodies clear of the PML: the shell kernel reads nothing the
        // classification writes, so it starts first, on stream5, beside it.
        shell_ahead = s->moving && fused && s->cls_boxes_current && s->n_solid_pml == 0 && !s->hP.visc &&
                      s->eng.empty() &&
                      s->stream5 && s->interior.hi[0] > s->interior.lo[0] && boxes_clear_of_shell(s, prev) &&
                      boxes_clear_of_shell(s, s->hP.boxes);
        if (shell_ahead) {
            RegionLaunch R = s->region;
            R.skip |= 1 | 4;  // the shell only
            R.sources = 0;
            R.fc = 0;
            const StepStreams S5{s->stream5, nullptr, nullptr, s->ev_fork, s->ev_join, s->ev_ghost};
            CUDA_TRY(s, cudaEventRecord(s->ev_sfork, s->stream));
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream5, s->ev_sfork, 0));
            int l = 0;
            if (s->precision == FDTD_PRECISION_FP64)
                CUDA_TRY(s, launch_step_regions_fp64(s->dP, s->hP, R, cur, S5, &l));
            else
                CUDA_TRY(s, launch_step_regions_fp32(s->dP, s->hP, R, cur, S5, &l));
            s->launches += l;
            s->overlapped_steps++;
            CUDA_TRY(s, cudaEventRecord(s->ev_sdone, s->stream5));
        }
        // moving bodies after a classification of the step before: only the units
        // its boxes reached can hold flags other than the defaults
        classification_launches(s, st, (s->moving && s->cls_boxes_current) ? &prev : nullptr);
        s->cls_boxes_current = true;
        if (st != FDTD_OK) return st;
        if (s->moving) {
            CUDA_TRY(s, launch_fresh_cells(s->dP, s->precision, cur, s->ncell, s->d_status, s->stream));
            s->launches++;
            if (s->boundary_handling == FDTD_BOUNDARY_FULLY_COUPLED) {
                // the coupled rows of this step's ghost faces (host build from the new flags)
                st = build_fully_coupled(s);
                if (st != FDTD_OK) return st;
                s->region.fc = s->hP.fc_n > 0 ? 1 : 0;
                CUDA_TRY(s, fdtd::counted_copyAsync(s, s->dP, &s->hP, sizeof(SolveParams), cudaMemcpyHostToDevice,
                                                    s->stream));
            }
        }
        if (!s->moving && s->L > 0) {
            // static classification: the listener fits become fixed weights
            CUDA_TRY(s, launch_listener_prep(s->dP, s->precision, cur ^ 1, s->L, s->stream));
            s->launches += 2;
            s->hP.lis_ready = 1;  // host mirror of the flag the prep sets (later uploads keep it)
        }
    }
    // the region-split path advances the step constants inside its shell kernel;
    // the prologue then only runs to re-zero solid cells inside the PML, or to
    // advance the constants of a grid without PML cells
    RegionLaunch R = s->region;
    if (shell_ahead) R.skip |= 2;
    const bool no_shell = R.shell.block_first[R.shell.n] == 0;
    const int advance = (!fused || no_shell) ? 1 : 0;
    if (s->precision == FDTD_PRECISION_FP64) {
        if (advance || s->n_solid_pml > 0) {
            CUDA_TRY(s, launch_prologue_fp64(s->dP, cur, advance, s->n_solid_pml, s->stream));
            s->launches++;
        }
        int l = 0;
        if (s->opt.kernel == FDTD_KERNEL_PHASED) {
            CUDA_TRY(s, launch_phased_fp64(s->dP, s->N, cur, phased_lap(s, cur), s->stream, &l));
        } else {
            CUDA_TRY(s, launch_step_regions_fp64(s->dP, s->hP, R, cur, step_streams(s), &l));
        }
        s->launches += l;
    } else {
        if (advance || s->n_solid_pml > 0) {
            CUDA_TRY(s, launch_prologue_fp32(s->dP, cur, advance, s->n_solid_pml, s->stream));
            s->launches++;
        }
        int l = 0;
        CUDA_TRY(s, launch_step_regions_fp32(s->dP, s->hP, R, cur, step_streams(s), &l));
        s->launches += l;
    }
    if (shell_ahead) CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_sdone, 0));
    if (s->L > 0 && dev_row) {
        // the phased path keeps p^{n+1} in the same slot as the fused one
        if (listeners_aside(s, classify)) {
            CUDA_TRY(s, cudaEventRecord(s->ev_step, s->stream));
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream4, s->ev_step, 0));
            CUDA_TRY(s, launch_listeners(s->dP, s->precision, cur ^ 1, s->L, dev_row, s->stream4));
            CUDA_TRY(s, cudaEventRecord(s->ev_lis[cur], s->stream4));
            s->lis_pending[cur] = true;
        } else {
            CUDA_TRY(s, launch_listeners(s->dP, s->precision, cur ^ 1, s->L, dev_row, s->stream));
        }
        s->launches++;
    }
    return FDTD_OK;
}

// Host bookkeeping after a step: parity, clock mirror, object animation
// (SimWorld::UpdateObjectState(t + dt), SimWorld.cpp:596-600).
fdtd_status after_step(fdtd_solver* s) {
    s->cur ^= 1;
    s->step_index++;
    s->time += s->k;
    if (s->moving) {
        s->state_time += s->k;
        for (size_t i = 0; i < s->objs.size(); ++i) {
            auto& o = s->objs[i];
            if (o.d.motion == FDTD_MOTION_STATIC) continue;
            host_object_pose(o, s->state_time);
            host_update_bbox(o);
        }
        to_dev_objects(s);
        CUDA_TRY(s, fdtd::counted_copyAsync(s, &s->dP->obj[0], &s->hP.obj[0], sizeof(DevObject) * s->objs.size(),
                                    cudaMemcpyHostToDevice, s->stream));
    }
    return FDTD_OK;
}

fdtd_status check_device_errors(fdtd_solver* s) {
    int dev_error = 0;
    int status[4] = {0, 0, 0, 0};
    CUDA_TRY(s, fdtd::counted_copyAsync(s, &dev_error, s->hP.dev_error, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, fdtd::counted_copyAsync(s, status, s->d_status, sizeof(status), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    int ghosts = 0;
    CUDA_TRY(s, fdtd::counted_copy(s, &ghosts, s->d_ghost_count, sizeof(int), cudaMemcpyDeviceToHost));
    if (ghosts > s->region.ghost_cap) {
        set_error(s, "ghost-neighbour list overflow (" + std::to_string(ghosts) + " > " +
                         std::to_string(s->region.ghost_cap) + ")");
        return FDTD_ERR_OOM;
    }
    if (status[0] == 2) {
        set_error(s, "fresh cell inside an object (MAC_Grid.cpp:2050-2053)");
        return FDTD_ERR_GEOMETRY;
    }
    if (dev_error & 1) {
        set_error(s, "listener sample not finite, or a degenerate listener stencil (no cell or rank-deficient MLS)");
        return FDTD_ERR_NUMERIC;
    }
    if (dev_error & fdtd::DEV_ERR_ENGQUIST) {
        set_error(s, "a solid cell reaches the stencil of an Engquist-Majda boundary cell (the ghost-pressure forms of "
                     "MAC_Grid.cpp:533-920 are not built): keep bodies and constraints three cells from sides without PML");
        return FDTD_ERR_UNSUPPORTED;
    }
    if (dev_error & fdtd::FDTD_DEV_ERR_TMA_TIMEOUT) {
        set_error(s, "a tensor copy of the PML-shell kernel did not complete within its bounded wait");
        return FDTD_ERR_TIMEOUT;
    }
    return FDTD_OK;
}

// Capture `n` steps starting at parity `cur` into a graph (static scenes only).
fdtd_status capture_graph(fdtd_solver* s, int cur, int n, bool src, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    fdtd_status st = join_listeners(s);  // no dependency on work outside the capture
    if (st != FDTD_OK) return st;
    CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int c = cur;
    for (int i = 0; i < n && st == FDTD_OK; ++i) {
        st = enqueue_step(s, c, s->d_lis + (size_t)i * s->L, false, src);
        c ^= 1;
    }
    if (st == FDTD_OK) st = join_listeners(s);  // the graph ends with every row written
    s->lis_pending[0] = s->lis_pending[1] = false;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st != FDTD_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) {
        set_error(s, std::string("graph capture: ") + cudaGetErrorString(e));
        return FDTD_ERR_CUDA;
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    // the graph's device-side setup now, not at its first launch
    if (e == cudaSuccess) e = cudaGraphUpload(*out, s->stream);
    if (e != cudaSuccess) {
        set_error(s, std::string("graph instantiate: ") + cudaGetErrorString(e));
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

// Run n steps; listener rows land in the device ring d_lis (chunks of at most
// lis_cap_steps) and are passed to `sink(first_step, count)` after each chunk.
// Static scenes replay captured graphs of graph_steps steps once the first
// step (which classifies) has run.
template <typename Sink>
fdtd_status run_steps(fdtd_solver* s, int n, Sink sink) {
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    const long long launches0 = s->launches;
    const int G = s->opt.graph_steps;
    int done = 0;
    while (done < n) {
        const int remaining = n - done;
        const bool classify_now = s->moving || s->step_index == 0;
        if (!classify_now && G > 0 && remaining >= G) {
            const bool src = sources_active_window(s, s->time, G);
            const int key = s->cur + (src ? 2 : 0);
            if (!s->graph_exec[key]) {
                const long long l0 = s->launches;
                fdtd_status st = capture_graph(s, s->cur, G, src, &s->graph_exec[key]);
                if (st != FDTD_OK) return st;
                s->graph_launches_per_exec = s->launches - l0;
                s->launches = l0;
            }
            CUDA_TRY(s, cudaGraphLaunch(s->graph_exec[key], s->stream));
            s->launches += s->graph_launches_per_exec;
            for (int q = 0; q < G; ++q) {
                fdtd_status st = after_step(s);
                if (st != FDTD_OK) return st;
            }
            fdtd_status st = sink(done, G);
            if (st != FDTD_OK) return st;
            done += G;
            continue;
        }
        int m = std::min(remaining, s->lis_cap_steps);
        if (G > 0 && !s->moving && classify_now) m = 1;
        for (int i = 0; i < m; ++i) {
            const bool classify = s->moving || s->step_index == 0;
            fdtd_status st = enqueue_step(s, s->cur, s->d_lis + (size_t)i * s->L, classify, sources_active(s, s->time));
            if (st != FDTD_OK) return st;
            st = after_step(s);
            if (st != FDTD_OK) return st;
        }
        fdtd_status st = join_listeners(s);
        if (st != FDTD_OK) return st;
        st = sink(done, m);
        if (st != FDTD_OK) return st;
        done += m;
    }
    s->last_launches = s->launches - launches0;
    return FDTD_OK;
}

// FDTD_CELL_* bits of cell (i, j, k) from its classification and ghost-object bytes.
uint8_t cell_flags(const fdtd_solver* s, uint8_t code, uint8_t gobj, int i, int j, int k) {
    const bool bulk = code & CLS_BULK;
    uint8_t f = 0;
    if (bulk) f |= FDTD_CELL_BULK;
    if (!bulk && (code & CLS_MASK)) f |= FDTD_CELL_GHOST;
    if (code & CLS_VALID) f |= FDTD_CELL_VALID_HISTORY;
    if (s->tab[0].pml_cell[i] || s->tab[1].pml_cell[j] || s->tab[2].pml_cell[k]) f |= FDTD_CELL_PML;
    if (!bulk && (gobj & GOBJ_CONSTRAINT)) f |= FDTD_CELL_CONSTRAINT;
    return f;
}

}  // namespace

extern "C" {

fdtd_status fdtd_solver_step(fdtd_solver* s, int32_t n_steps, double* listener_out) {
    if (!s || n_steps < 0) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    const int L = s->L;
    // rows of consecutive chunks gather in the pinned staging buffer (copies in
    // stream order, before the next chunk rewrites the device ring); the host
    // waits only when the buffer is full and at the end
    int staged = 0, staged_first = 0;
    auto flush = [&]() -> fdtd_status {
        if (staged == 0) return FDTD_OK;
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        std::memcpy(listener_out + (size_t)staged_first * L, s->h_lis_stage, (size_t)staged * L * 8);
        staged = 0;
        return FDTD_OK;
    };
    fdtd_status st = run_steps(s, n_steps, [&](int first, int count) -> fdtd_status {
        if (listener_out && L > 0) {
            if (staged + count > s->lis_cap_steps) {
                const fdtd_status f = flush();
                if (f != FDTD_OK) return f;
            }
            if (staged == 0) staged_first = first;
            CUDA_TRY(s, fdtd::counted_copyAsync(s, s->h_lis_stage + (size_t)staged * L, s->d_lis, (size_t)count * L * 8,
                                        cudaMemcpyDeviceToHost, s->stream));
            staged += count;
        }
        return FDTD_OK;
    });
    if (st != FDTD_OK) return st;
    st = flush();
    if (st != FDTD_OK) return st;
    st = check_device_errors(s);
    if (st != FDTD_OK) return st;
    if (s->end_time > 0.0 && s->time >= s->end_time) return FDTD_END_OF_TIME;
    return FDTD_OK;
}

fdtd_status fdtd_solver_step_device(fdtd_solver* s, int32_t n_steps, void* device_listener_out) {
    if (!s || n_steps < 0) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    const int L = s->L;
    double* out = (double*)device_listener_out;
    fdtd_status st = run_steps(s, n_steps, [&](int first, int count) -> fdtd_status {
        if (out && L > 0)
            CUDA_TRY(s, fdtd::counted_copyAsync(s, out + (size_t)first * L, s->d_lis, (size_t)count * L * 8,
                                        cudaMemcpyDeviceToDevice, s->stream));
        return FDTD_OK;
    });
    return st;
}

fdtd_status fdtd_solver_fetch_listeners(fdtd_solver* s, double* out) {
    if (!s || (!out && s->L > 0)) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    if (s->L == 0) return FDTD_OK;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    CUDA_TRY(s, launch_listeners(s->dP, s->precision, s->cur, s->L, s->d_lis, s->stream));
    CUDA_TRY(s, fdtd::counted_copyAsync(s, out, s->d_lis, (size_t)s->L * 8, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return FDTD_OK;
}

fdtd_status fdtd_solver_time_kernel(fdtd_solver* s, int32_t which, int32_t n_launches, float* elapsed_ms) {
    if (!s || n_launches <= 0 || !elapsed_ms || which < 0 || which > 4)
        return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    if (which > 0 && s->opt.kernel != FDTD_KERNEL_FUSED)
        return (set_error(s, "single-kernel timing needs the region-split (fused) path"), FDTD_ERR_INVALID_ARG);
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    cudaEvent_t e0, e1;
    CUDA_TRY(s, cudaEventCreate(&e0));
    CUDA_TRY(s, cudaEventCreate(&e1));
    RegionLaunch R = s->region;
    R.sources = 0;
    if (which == 1) R.skip = 2 | 4;
    if (which == 2) R.skip = 1 | 4;
    if (which == 3) R.skip = 1 | 2;
    // the launches are captured into a graph and the graph is timed: device time
    // only, whatever the host's launch rate (a step forks to three streams)
    fdtd_status jst = join_listeners(s);
    if (jst != FDTD_OK) return jst;
    CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int c = s->cur;
    for (int i = 0; i < n_launches; ++i) {
        cudaError_t e;
        if (which == 4) {
            e = launch_listeners(s->dP, s->precision, c, s->L, s->d_lis, s->stream);
        } else if (s->precision == FDTD_PRECISION_FP64) {
            if (s->opt.kernel == FDTD_KERNEL_PHASED) e = launch_phased_fp64(s->dP, s->N, c, phased_lap(s, c), s->stream, nullptr);
            else e = launch_step_regions_fp64(s->dP, s->hP, R, c, step_streams(s), nullptr);
        } else {
            e = launch_step_regions_fp32(s->dP, s->hP, R, c, step_streams(s), nullptr);
        }
        if (e != cudaSuccess) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s->stream, &g);
            if (g) cudaGraphDestroy(g);
            set_error(s, std::string("stencil launch: ") + cudaGetErrorString(e));
            return FDTD_ERR_CUDA;
        }
        if (which != 4) c ^= 1;
    }
    cudaGraph_t g = nullptr;
    CUDA_TRY(s, cudaStreamEndCapture(s->stream, &g));
    cudaGraphExec_t x = nullptr;
    cudaError_t ge = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (ge != cudaSuccess) {
        set_error(s, std::string("stencil graph: ") + cudaGetErrorString(ge));
        return FDTD_ERR_CUDA;
    }
    // one untimed replay, one timed: 2 n launches, so the parity comes back
    ge = cudaGraphLaunch(x, s->stream);
    if (ge == cudaSuccess) ge = cudaEventRecord(e0, s->stream);
    if (ge == cudaSuccess) ge = cudaGraphLaunch(x, s->stream);
    if (ge == cudaSuccess) ge = cudaEventRecord(e1, s->stream);
    if (ge == cudaSuccess) ge = cudaEventSynchronize(e1);
    if (ge == cudaSuccess) ge = cudaEventElapsedTime(elapsed_ms, e0, e1);
    cudaGraphExecDestroy(x);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ge != cudaSuccess) {
        set_error(s, std::string("stencil timing: ") + cudaGetErrorString(ge));
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

fdtd_status fdtd_solver_time_stencil(fdtd_solver* s, int32_t n_launches, float* elapsed_ms) {
    return fdtd_solver_time_kernel(s, 0, n_launches, elapsed_ms);
}

fdtd_status fdtd_solver_synchronize(fdtd_solver* s) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return FDTD_OK;
}

void* fdtd_solver_stream(fdtd_solver* s) { return s ? (void*)s->stream : nullptr; }

const char* fdtd_solver_last_error(fdtd_solver* s) { return s ? s->err.c_str() : ""; }

int64_t fdtd_solver_last_launch_count(fdtd_solver* s) { return s ? s->last_launches : 0; }

int64_t fdtd_solver_overlapped_steps(fdtd_solver* s) { return s ? s->overlapped_steps : 0; }

int32_t fdtd_solver_shell_staging(fdtd_solver* s) {
    if (!s || !s->region.red) return -1;
    return s->region.tma ? FDTD_SHELL_STAGING_TMA : FDTD_SHELL_STAGING_RING;
}

fdtd_status fdtd_solver_transfer_bytes(fdtd_solver* s, int64_t* host_to_device, int64_t* device_to_host) {
    if (!s || !host_to_device || !device_to_host) return (set_error(s, "invalid arguments"), FDTD_ERR_INVALID_ARG);
    *host_to_device = s->bytes_h2d;
    *device_to_host = s->bytes_d2h;
    return FDTD_OK;
}

fdtd_status fdtd_solver_prepare_graphs(fdtd_solver* s) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    const int G = s->opt.graph_steps;
    if (G <= 0 || s->moving || s->step_index == 0) return FDTD_OK;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    const bool src = sources_active_window(s, s->time, G);
    const int key = s->cur + (src ? 2 : 0);
    if (s->graph_exec[key]) return FDTD_OK;
    const long long l0 = s->launches;
    fdtd_status st = capture_graph(s, s->cur, G, src, &s->graph_exec[key]);
    if (st != FDTD_OK) return st;
    s->graph_launches_per_exec = s->launches - l0;
    s->launches = l0;
    return FDTD_OK;
}

int32_t fdtd_solver_pml_state(fdtd_solver* s) {
    return (s && s->region.red) ? FDTD_PML_STATE_AUTO : FDTD_PML_STATE_FULL;
}

fdtd_status fdtd_solver_info_get(fdtd_solver* s, fdtd_solver_info* info) {
    if (!s || !info) return FDTD_ERR_INVALID_ARG;
    std::memset(info, 0, sizeof(*info));
    for (int d = 0; d < 3; ++d) info->divisions[d] = s->N[d];
    info->n_listeners = s->L;
    info->n_cells = s->ncell;
    info->n_pml_cells = s->n_pml;
    info->n_interior_cells = s->n_interior;
    info->device_bytes = (int64_t)s->arena_bytes;
    info->step_index = s->step_index;
    info->time = s->time;
    info->time_step = s->k;
    const double w = s->precision == FDTD_PRECISION_FP64 ? 8.0 : 4.0;
    info->algorithmic_bytes_per_step = w * (3.0 * (double)s->n_interior + 14.0 * (double)s->n_pml);
    return FDTD_OK;
}

fdtd_status fdtd_solver_get_classification(fdtd_solver* s, uint8_t* flags, fdtd_ghost_face* faces, int64_t* n_faces) {
    if (!s) return FDTD_ERR_INVALID_ARG;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    std::vector<uint8_t> pcls(s->np), pgobj(s->np);
    CUDA_TRY(s, fdtd::counted_copyAsync(s, pcls.data(), s->hP.cls, s->np, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, fdtd::counted_copyAsync(s, pgobj.data(), s->hP.gobj, s->np, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    // dense (reference) order and indices
    std::vector<uint8_t> cls(s->ncell), gobj(s->ncell);
    {
        long long c = 0;
        for (int i = 0; i < s->N[0]; ++i)
            for (int j = 0; j < s->N[1]; ++j)
                for (int k = 0; k < s->N[2]; ++k, ++c) {
                    cls[c] = pcls[i * s->SX + j * s->SY + k];
                    gobj[c] = pgobj[i * s->SX + j * s->SY + k];
                }
    }
    const long long sx = (long long)s->N[1] * s->N[2];
    int64_t count = 0;
    const int64_t cap = (faces && n_faces) ? *n_faces : 0;
    for (long long c = 0; c < s->ncell; ++c) {
        const uint8_t code = cls[c];
        const bool bulk = code & CLS_BULK;
        const unsigned mask = code & CLS_MASK;
        const int i = (int)(c / sx), j = (int)((c / s->N[2]) % s->N[1]), k = (int)(c % s->N[2]);
        if (flags) flags[c] = cell_flags(s, code, gobj[c], i, j, k);
        if (bulk || !mask) continue;
        // faces in key order: neighbour flat index ascending (-x, -y, -z, +z, +y, +x)
        static const int od[6] = {0, 1, 2, 2, 1, 0};
        static const int os[6] = {-1, -1, -1, +1, +1, +1};
        const long long strides[3] = {sx, s->N[2], 1};
        for (int f = 0; f < 6; ++f) {
            if (!((mask >> (2 * od[f] + (os[f] > 0))) & 1u)) continue;
            if (count < cap) {
                fdtd_ghost_face& g = faces[count];
                std::memset(&g, 0, sizeof(g));
                g.owner_cell = (int32_t)c;
                g.neighbour_cell = (int32_t)(c + os[f] * strides[od[f]]);
                g.topology = os[f] * (od[f] + 1);
                g.type = (gobj[c] & GOBJ_CONSTRAINT) ? 1 : 0;
                const int o = gobj[c] & 0x7F;
                g.boundary_object = (o == GOBJ_NONE) ? -1 : o;
                g.key = szudzik(g.owner_cell, g.neighbour_cell);
            }
            ++count;
        }
    }
    if (n_faces) *n_faces = count;
    return FDTD_OK;
}

}  // extern "C"

namespace {

// Index into the compact z-slab arrays of the PML state (ShellBoxes::zbox) of
// the split pressure of cell (x, y, z) (dface < 0) or of its low face along
// dface; -1 when that element lives in the padded arrays.
long long zslab_index(const fdtd_solver* s, int dface, int x, int y, int z) {
    const ShellBoxes& B = s->shell;
    const int b = B.zbox, V = B.vz;
    if (s->hP.zcount <= 0 || b < 0) return -1;
    if (x < B.x0[b] || x >= B.x0[b] + B.nx[b] || y < B.y0[b] || y >= B.y0[b] + B.ny[b]) return -1;
    if (dface != 2 && z >= s->N[2]) return -1;
    auto slot = [&](int zz) -> long long {  // compact slot of the cell (or its low face) zz in the row
        if (zz >= B.za[b] && zz < B.zae[b]) return (long long)(zz / V - B.za[b] / V) * V + zz % V;
        if (zz >= B.zb[b] && zz < B.zbe[b]) return (long long)(B.gl[b] + zz / V - B.zb[b] / V) * V + zz % V;
        return -1;
    };
    long long q = slot(z);
    if (dface == 2 && q < 0 && z == B.zae[b] && z > 0) {
        // boundary face after the first range: high face of its last cell
        const long long qc = slot(z - 1);
        q = ((z - 1) % V != V - 1) ? qc + 1 : (long long)B.ng[b] * V;
    }
    if (q < 0) return -1;
    return ((long long)(x - B.x0[b]) * B.ny[b] + (y - B.y0[b])) * B.zrw + q;
}

// Field `which` between the device layout (padded arrays, the compact z-slab
// arrays of the PML state) and a dense host array in the reference's flat order
// (cells, or faces of one orientation).  to_device: dense -> device.  FP32
// PRESSURE_PREV is p^n - d (d the compensated increment); writing it sets d from
// the p^n already on the device, so write PRESSURE first.
fdtd_status field_transfer(fdtd_solver* s, int32_t which, double* dense, int64_t count, bool to_device) {
    if (!s || !dense) return FDTD_ERR_INVALID_ARG;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    const SolveParams& P = s->hP;
    const bool f64 = s->precision == FDTD_PRECISION_FP64;
    const size_t w = f64 ? 8 : 4;
    void* src = nullptr;
    long long n = s->ncell;
    int vbuf = s->opt.kernel == FDTD_KERNEL_PHASED ? 0 : s->cur;
    switch (which) {
        case FDTD_FIELD_PRESSURE: src = P.p[s->cur]; break;
        case FDTD_FIELD_PRESSURE_PREV: src = f64 ? P.p[s->cur ^ 1] : P.p[s->cur]; break;
        case FDTD_FIELD_PML_PX: case FDTD_FIELD_PML_PY: case FDTD_FIELD_PML_PZ: src = P.pd[which - FDTD_FIELD_PML_PX]; break;
        case FDTD_FIELD_VX: case FDTD_FIELD_VY: case FDTD_FIELD_VZ:
            src = P.v[vbuf][which - FDTD_FIELD_VX];
            n = s->vcount[which - FDTD_FIELD_VX];
            break;
        default: return (set_error(s, "unknown field"), FDTD_ERR_INVALID_ARG);
    }
    if (count != n) return (set_error(s, "count does not match the field size"), FDTD_ERR_INVALID_ARG);
    if (s->region.red && which >= FDTD_FIELD_PML_PX)
        return (set_error(s, "this FP32 solve keeps the reduced PML state (no split pressures or face velocities "
                             "along axes without absorption); create it with pml_state = FDTD_PML_STATE_FULL to "
                             "access them"),
                FDTD_ERR_UNSUPPORTED);
    // extent of the requested grid (cells, or faces of one orientation)
    int ext[3] = {s->N[0], s->N[1], s->N[2]};
    if (which >= FDTD_FIELD_VX) ext[which - FDTD_FIELD_VX] += 1;
    const long long np = s->np;
    std::vector<char> raw(np * w);
    std::vector<float> inc;
    CUDA_TRY(s, fdtd::counted_copyAsync(s, raw.data(), src, np * w, cudaMemcpyDeviceToHost, s->stream));
    const bool fp32_prev = !f64 && which == FDTD_FIELD_PRESSURE_PREV;
    if (fp32_prev) {
        inc.resize(np);
        CUDA_TRY(s, fdtd::counted_copyAsync(s, inc.data(), P.dinc, np * 4, cudaMemcpyDeviceToHost, s->stream));
    }
    // the z-slab box keeps its PML state in compact arrays (ShellBoxes)
    const ShellBoxes& B = s->shell;
    const bool zc = P.zcount > 0 && which >= FDTD_FIELD_PML_PX;
    std::vector<char> zraw;
    void* zsrc = nullptr;
    if (zc) {
        zsrc = which <= FDTD_FIELD_PML_PZ ? P.zpd[which - FDTD_FIELD_PML_PX] : P.zv[vbuf][which - FDTD_FIELD_VX];
        zraw.resize(P.zcount * w);
        CUDA_TRY(s, fdtd::counted_copyAsync(s, zraw.data(), zsrc, P.zcount * w, cudaMemcpyDeviceToHost, s->stream));
    }
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    // every (padded grid index, compact index) pair of the z-slab box
    auto for_compact = [&](auto&& fn) {
        const int b = B.zbox;
        const int dface = which >= FDTD_FIELD_VX ? which - FDTD_FIELD_VX : -1;
        for (int x = B.x0[b]; x < B.x0[b] + B.nx[b]; ++x)
            for (int y = B.y0[b]; y < B.y0[b] + B.ny[b]; ++y)
                for (int z = 0; z <= s->N[2]; ++z) {
                    const long long q = zslab_index(s, dface, x, y, z);
                    if (q >= 0) fn(x * s->SX + y * s->SY + z, q);
                }
    };
    double* r64 = (double*)raw.data();
    float* r32 = (float*)raw.data();
    if (!to_device) {
        if (zc) for_compact([&](long long c, long long q) { std::memcpy(raw.data() + c * w, zraw.data() + q * w, w); });
        long long o = 0;
        for (int i = 0; i < ext[0]; ++i)
            for (int j = 0; j < ext[1]; ++j)
                for (int k = 0; k < ext[2]; ++k, ++o) {
                    const long long c = i * s->SX + j * s->SY + k;
                    if (f64) dense[o] = r64[c];
                    else dense[o] = fp32_prev ? (double)r32[c] - (double)inc[c] : (double)r32[c];
                }
        return FDTD_OK;
    }
    long long o = 0;
    for (int i = 0; i < ext[0]; ++i)
        for (int j = 0; j < ext[1]; ++j)
            for (int k = 0; k < ext[2]; ++k, ++o) {
                const long long c = i * s->SX + j * s->SY + k;
                if (f64) r64[c] = dense[o];
                else if (fp32_prev) inc[c] = (float)((double)r32[c] - dense[o]);
                else r32[c] = (float)dense[o];
            }
    if (fp32_prev) {
        CUDA_TRY(s, fdtd::counted_copyAsync(s, P.dinc, inc.data(), np * 4, cudaMemcpyHostToDevice, s->stream));
    } else {
        if (zc) for_compact([&](long long c, long long q) { std::memcpy(zraw.data() + q * w, raw.data() + c * w, w); });
        CUDA_TRY(s, fdtd::counted_copyAsync(s, src, raw.data(), np * w, cudaMemcpyHostToDevice, s->stream));
        if (zc) CUDA_TRY(s, fdtd::counted_copyAsync(s, zsrc, zraw.data(), P.zcount * w, cudaMemcpyHostToDevice, s->stream));
    }
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return FDTD_OK;
}

// Device address of element (x, y, z) of a split pressure or face-velocity
// field, where field_transfer finds it; null when the solve does not hold it
// (the reduced PML state).
const void* field_element(const fdtd_solver* s, int which, int x, int y, int z) {
    const SolveParams& P = s->hP;
    if (s->region.red) return nullptr;
    const size_t w = s->precision == FDTD_PRECISION_FP64 ? 8 : 4;
    const int vbuf = s->opt.kernel == FDTD_KERNEL_PHASED ? 0 : s->cur;
    const int dface = which >= FDTD_FIELD_VX ? which - FDTD_FIELD_VX : -1;
    const void* base = dface < 0 ? P.pd[which - FDTD_FIELD_PML_PX] : P.v[vbuf][dface];
    if (!base) return nullptr;
    const long long q = zslab_index(s, dface, x, y, z);
    if (q >= 0) {
        const void* zb = dface < 0 ? P.zpd[which - FDTD_FIELD_PML_PX] : P.zv[vbuf][dface];
        return (const char*)zb + q * (long long)w;
    }
    return (const char*)base + (x * s->SX + y * s->SY + z) * (long long)w;
}

// MAC_Grid::GetCell (MAC_Grid.cpp:4182-4258) + the stored Laplacian of
// PML_WaveSolver::FetchCell (PML_WaveSolver.cpp:439-447) for the cells of
// dense indices `cells`: the device gathers (k_fetch_cells), the host fills
// the geometry and PressureCellType (MAC_Grid.cpp:3977-3997).
fdtd_status fetch_cells(fdtd_solver* s, const std::vector<long long>& cells, fdtd_cell* out) {
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    const int n = (int)cells.size();
    if (n == 0) return FDTD_OK;
    std::vector<FetchReq> req(n);
    for (int q = 0; q < n; ++q) {
        int ijk[3];
        const long long t = cells[q];
        ijk[0] = (int)(t / ((long long)s->N[1] * s->N[2]));
        ijk[1] = (int)((t / s->N[2]) % s->N[1]);
        ijk[2] = (int)(t % s->N[2]);
        FetchReq& R = req[q];
        R.c = ijk[0] * s->SX + ijk[1] * s->SY + ijk[2];
        for (int d = 0; d < 3; ++d) {
            int up[3] = {ijk[0], ijk[1], ijk[2]};
            up[d] += 1;  // the upper face index never exceeds N[d] (MAC_Grid.cpp:4247-4249)
            R.a[d] = field_element(s, FDTD_FIELD_PML_PX + d, ijk[0], ijk[1], ijk[2]);
            R.a[3 + 2 * d] = field_element(s, FDTD_FIELD_VX + d, ijk[0], ijk[1], ijk[2]);
            R.a[4 + 2 * d] = field_element(s, FDTD_FIELD_VX + d, up[0], up[1], up[2]);
        }
    }
    const size_t req_bytes = (size_t)n * sizeof(FetchReq), val_bytes = (size_t)n * sizeof(FetchVal);
    std::vector<FetchVal> vals(n);
    void* dbuf = nullptr;
    CUDA_TRY(s, cudaMallocAsync(&dbuf, req_bytes + val_bytes, s->stream));
    FetchReq* dreq = (FetchReq*)dbuf;
    FetchVal* dval = (FetchVal*)((char*)dbuf + req_bytes);
    cudaError_t e = fdtd::counted_copyAsync(s, dreq, req.data(), req_bytes, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess)
        e = launch_fetch_cells(s->dP, s->precision == FDTD_PRECISION_FP64, s->cur, dreq, dval, n, s->stream);
    if (e == cudaSuccess) {
        ++s->launches;
        e = fdtd::counted_copyAsync(s, vals.data(), dval, val_bytes, cudaMemcpyDeviceToHost, s->stream);
    }
    const cudaError_t ef = cudaFreeAsync(dbuf, s->stream);
    if (e == cudaSuccess) e = ef;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    CUDA_TRY(s, e);
    // the Laplacian kept for the next step: the phased path keeps the reference's
    // (every cell, every step); the fused kernels keep it on the non-PML cells of
    // a static scene (its other cells stay zero)
    const bool visc = s->hP.visc != 0;
    const bool phased = s->opt.kernel == FDTD_KERNEL_PHASED;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int q = 0; q < n; ++q) {
        const long long t = cells[q];
        const FetchVal& v = vals[q];
        fdtd_cell& C = out[q];
        std::memset(&C, 0, sizeof(C));
        C.index = (int32_t)t;
        C.indices[0] = (int32_t)(t / ((long long)s->N[1] * s->N[2]));
        C.indices[1] = (int32_t)((t / s->N[2]) % s->N[1]);
        C.indices[2] = (int32_t)(t % s->N[2]);
        const int i = C.indices[0], j = C.indices[1], k = C.indices[2];
        const uint8_t f = cell_flags(s, (uint8_t)v.cls, (uint8_t)v.gobj, i, j, k);
        int32_t flags = f;
        const bool pml = f & FDTD_CELL_PML;
        if (pml) {
            double m = std::numeric_limits<double>::min();
            m = std::max(m, s->tab[0].csig[i]);
            m = std::max(m, s->tab[1].csig[j]);
            m = std::max(m, s->tab[2].csig[k]);
            C.r_identity = -0.5 * m / s->pml_strength;
        } else if (f & FDTD_CELL_BULK) {
            C.r_identity = 0.5;
        } else if (!(f & FDTD_CELL_GHOST)) {
            C.r_identity = 1.0;
        } else {
            C.r_identity = -1.0;
            C.n_gc_value = 6;
        }
        const double cp[3] = {s->tab[0].cpos[i], s->tab[1].cpos[j], s->tab[2].cpos[k]};
        for (int d = 0; d < 3; ++d) {
            C.centroid[d] = cp[d];
            C.lower_corner[d] = cp[d] - s->h / 2.0;
            C.upper_corner[d] = cp[d] + s->h / 2.0;
        }
        // ghost faces toward bulk neighbours; they hold zero until the first step computes them
        const unsigned faces = C.n_gc_value ? (unsigned)(v.cls & CLS_MASK) : 0u;
        for (int g = 0; g < 6; ++g)
            C.gc_value[g] = ((faces >> g) & 1u) ? (s->step_index == 0 ? 0.0 : v.gc[g]) : -1.0;
        for (int d = 0; d < 3; ++d) C.p_directional[d] = v.pdir[d];
        C.p_full = v.p;
        C.vx[0] = v.v[0], C.vx[1] = v.v[1];
        C.vy[0] = v.v[2], C.vy[1] = v.v[3];
        C.vz[0] = v.v[4], C.vz[1] = v.v[5];
        if (!s->region.red) flags |= FDTD_CELLINFO_PML_STATE;
        C.h = s->h;
        if (s->step_index == 0) {
            C.laplacian = 0.0;
            flags |= FDTD_CELLINFO_LAPLACIAN;
        } else if (visc && (phased || (!s->moving && !pml))) {
            C.laplacian = v.lap;
            flags |= FDTD_CELLINFO_LAPLACIAN;
        } else {
            C.laplacian = nan;
        }
        C.flags = flags;
    }
    return FDTD_OK;
}

}  // namespace

extern "C" {

fdtd_status fdtd_solver_get_field(fdtd_solver* s, int32_t which, double* out, int64_t count) {
    // the read-back stages the field in host memory
    if (s && fdtd::inject_failure(FDTD_INJECT_HOST_ALLOC))
        return (set_error(s, "host staging buffer of the field read-back: allocation failed"), FDTD_ERR_OOM);
    return field_transfer(s, which, out, count, false);
}

fdtd_status fdtd_solver_set_field(fdtd_solver* s, int32_t which, const double* in, int64_t count) {
    return field_transfer(s, which, const_cast<double*>(in), count, true);
}

fdtd_status fdtd_solver_domain(fdtd_solver* s, double min_bound[3], double max_bound[3]) {
    if (!s || !min_bound || !max_bound) return FDTD_ERR_INVALID_ARG;
    for (int d = 0; d < 3; ++d) {
        min_bound[d] = s->bmin[d];
        max_bound[d] = s->bmax[d];
    }
    return FDTD_OK;
}

fdtd_status fdtd_solver_fetch_cell(fdtd_solver* s, int64_t cell_index, fdtd_cell* out) {
    if (!s || !out) return FDTD_ERR_INVALID_ARG;
    if (cell_index < 0 || cell_index >= s->ncell)
        return (set_error(s, "cell_index out of range"), FDTD_ERR_INVALID_ARG);
    return fetch_cells(s, std::vector<long long>{cell_index}, out);
}

fdtd_status fdtd_solver_sample_slice(fdtd_solver* s, int32_t dim, double offset, fdtd_cell* out, int64_t capacity,
                                     int64_t* count) {
    if (!s || !count) return FDTD_ERR_INVALID_ARG;
    if (dim < 0 || dim > 2) return (set_error(s, "dim must be 0, 1 or 2"), FDTD_ERR_INVALID_ARG);
    const int d1 = (dim + 1) % 3, d2 = (dim + 2) % 3;
    const int64_t n = (int64_t)s->N[d1] * s->N[d2];
    *count = n;
    if (!out) return FDTD_OK;
    if (capacity < n) return (set_error(s, "capacity below the slice's cell count"), FDTD_ERR_INVALID_ARG);
    // the face grid along dim starts half a cell below the cells (MAC_Grid.cpp:103-113)
    const double lower = s->bmin[dim] - s->h / 2.0;
    const double r = (offset - lower) / s->h;
    if (!(r > -1.0) || !(r < 2147483647.0))
        return (set_error(s, "offset outside the grid along dim"), FDTD_ERR_INVALID_ARG);
    const int k = std::min((int)r, s->N[dim] - 1);
    std::vector<long long> cells((size_t)n);
    size_t c = 0;
    for (int a = 0; a < s->N[d1]; ++a)
        for (int b = 0; b < s->N[d2]; ++b) {
            int idx[3];
            idx[dim] = k;
            idx[d1] = a;
            idx[d2] = b;
            cells[c++] = ((long long)idx[0] * s->N[1] + idx[1]) * s->N[2] + idx[2];
        }
    return fetch_cells(s, cells, out);
}

// ---------------------------------------------------------------------------
// snapshot / restore (FDTD_AcousticSimulator::_SaveSimulationSnapshot, :381-415)
// ---------------------------------------------------------------------------
namespace {
struct SnapHeader {
    uint64_t magic;
    int64_t ncell;
    int32_t precision, kernel, cur, n_obj;
    int64_t step_index;
    double time, state_time;
};
const uint64_t SNAP_MAGIC = 0x314e53445446ULL;  // "FTDSN1"

std::vector<std::pair<void*, size_t>> snap_regions(fdtd_solver* s) {
    const SolveParams& P = s->hP;
    const size_t w = s->precision == FDTD_PRECISION_FP64 ? 8 : 4;
    std::vector<std::pair<void*, size_t>> r;
    const size_t np = (size_t)s->np;  // the padded arrays as they are
    r.push_back({P.p[0], np * w});
    r.push_back({P.p[1], np * w});
    if (P.dinc) r.push_back({P.dinc, np * 4});
    for (int d = 0; d < 3; ++d) r.push_back({P.pd[d], np * w});
    for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 3; ++d)
            if (P.v[b][d]) r.push_back({P.v[b][d], np * w});
    r.push_back({P.cls, np});
    r.push_back({P.gobj, np});
    if (P.zcount > 0)
        for (int d = 0; d < 3; ++d) {
            r.push_back({P.zpd[d], (size_t)P.zcount * w});
            r.push_back({P.zv[0][d], (size_t)P.zcount * w});
            r.push_back({P.zv[1][d], (size_t)P.zcount * w});
        }
    for (int b = 0; b < 2; ++b)
        if (P.lapv[b]) r.push_back({P.lapv[b], np * (s->precision == FDTD_PRECISION_FP64 ? 8 : 4)});
    if (P.eng_buf) r.push_back({P.eng_buf, s->eng.size() * ENG_BUF * 8});
    r.push_back({P.consts, 2 * sizeof(StepConsts)});
    r.push_back({P.dev_error, sizeof(int)});
    return r;
}
}  // namespace

}  // extern "C"

namespace fdtd {
// Moving bodies that stay two cells clear of the PML at every step of
// [start_time, end_time]: the per-step classification boxes of the whole run,
// posed and unioned as the step driver does, are checked on the host.  Then no
// PML cell is ever solid or next to a solid, and the reduced PML state is exact.
bool moving_clear_of_pml(fdtd_solver* s) {
    if (!s->moving || !(s->end_time > s->start_time) || !(s->k > 0)) return false;
    const double nsteps = std::ceil((s->end_time - s->start_time) / s->k) + 2.0;
    if (nsteps > 2.0e7) return false;
    std::vector<HostObject> objs = s->objs;
    double t = s->start_time;
    for (auto& o : objs) {
        host_object_pose(o, t);
        host_update_bbox(o);
        host_reset_union(o);
    }
    bool clear = true;
    std::swap(s->objs, objs);  // classification_boxes reads s->objs
    ClsBoxes B;
    for (long long i = 0; i <= (long long)nsteps && clear; ++i) {
        if (i > 0) {
            t += s->k;
            for (auto& o : s->objs) {
                if (o.d.motion == FDTD_MOTION_STATIC) continue;
                host_object_pose(o, t);
                host_update_bbox(o);
            }
        }
        classification_boxes(s, B);
        clear = boxes_clear_of_shell(s, B);
    }
    std::swap(s->objs, objs);
    return clear;
}

// Listener plans (fixed MLS weights) of a static solve from its current
// classification, as its first step builds them; used after a restore.
fdtd_status rebuild_listener_plans(fdtd_solver* s) {
    if (s->moving || s->L <= 0) return FDTD_OK;
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    CUDA_TRY(s, launch_listener_prep(s->dP, s->precision, s->cur, s->L, s->stream));
    s->hP.lis_ready = 1;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return FDTD_OK;
}
}  // namespace fdtd

extern "C" {

fdtd_status fdtd_solver_snapshot(fdtd_solver* s, void* buffer, int64_t* bytes) {
    if (!s || !bytes) return FDTD_ERR_INVALID_ARG;
    auto regs = snap_regions(s);
    size_t total = sizeof(SnapHeader) + s->objs.size() * sizeof(HostObject);
    for (auto& r : regs) total += r.second;
    if (!buffer) {
        *bytes = (int64_t)total;
        return FDTD_OK;
    }
    if (*bytes < (int64_t)total) return (set_error(s, "snapshot buffer too small"), FDTD_ERR_INVALID_ARG);
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    SnapHeader h{SNAP_MAGIC, s->ncell, s->precision, s->opt.kernel, s->cur, (int32_t)s->objs.size(),
                 s->step_index, s->time, s->state_time};
    char* p = (char*)buffer;
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    std::memcpy(p, s->objs.data(), s->objs.size() * sizeof(HostObject));
    p += s->objs.size() * sizeof(HostObject);
    for (auto& r : regs) {
        CUDA_TRY(s, fdtd::counted_copyAsync(s, p, r.first, r.second, cudaMemcpyDeviceToHost, s->stream));
        p += r.second;
    }
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    *bytes = (int64_t)total;
    return FDTD_OK;
}

fdtd_status fdtd_solver_restore(fdtd_solver* s, const void* buffer, int64_t bytes) {
    if (!s || !buffer) return FDTD_ERR_INVALID_ARG;
    SnapHeader h;
    if (bytes < (int64_t)sizeof(h)) return (set_error(s, "snapshot truncated"), FDTD_ERR_INVALID_ARG);
    std::memcpy(&h, buffer, sizeof(h));
    if (h.magic != SNAP_MAGIC || h.ncell != s->ncell || h.precision != s->precision || h.kernel != s->opt.kernel ||
        h.n_obj != (int32_t)s->objs.size())
        return (set_error(s, "snapshot does not match this solver"), FDTD_ERR_INVALID_ARG);
    auto regs = snap_regions(s);
    size_t total = sizeof(SnapHeader) + s->objs.size() * sizeof(HostObject);
    for (auto& r : regs) total += r.second;
    if (bytes < (int64_t)total) return (set_error(s, "snapshot truncated"), FDTD_ERR_INVALID_ARG);
    CUDA_TRY(s, cudaSetDevice(s->opt.device));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    const char* p = (const char*)buffer + sizeof(h);
    // the pose state comes from the snapshot; what points into this solver's own
    // storage (device meshes, keyframe tracks, mesh vertices) stays this solver's
    const std::vector<HostObject> own = s->objs;
    std::memcpy(s->objs.data(), p, s->objs.size() * sizeof(HostObject));
    for (size_t i = 0; i < s->objs.size(); ++i) {
        s->objs[i].mview = own[i].mview;
        s->objs[i].kf = own[i].kf;
        s->objs[i].mv = own[i].mv;
    }
    p += s->objs.size() * sizeof(HostObject);
    for (auto& r : regs) {
        CUDA_TRY(s, fdtd::counted_copy(s, r.first, p, r.second, cudaMemcpyHostToDevice));
        p += r.second;
    }
    s->cur = h.cur;
    s->step_index = h.step_index;
    s->time = h.time;
    s->state_time = h.state_time;
    s->cls_boxes_current = false;  // the flags came from the snapshot, not from hP.boxes
    to_dev_objects(s);
    CUDA_TRY(s, fdtd::counted_copy(s, s->dP, &s->hP, sizeof(SolveParams), cudaMemcpyHostToDevice));
    // the fixed listener weights of the restored classification (a first step
    // classifies and derives them itself)
    if (s->step_index > 0) return rebuild_listener_plans(s);
    return FDTD_OK;
}

}  // extern "C"
