// fdtd_internal.hpp — host-side state of one solver handle.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

#include "../../include/fdtd_c.h"
#include "fdtd_device.cuh"
#include "fdtd_tma.hpp"

namespace fdtd {

struct HostObject {
    fdtd_object_desc d;
    double c[3] = {0, 0, 0};
    double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};  // _bboxWorld
    double umin[3] = {0, 0, 0}, umax[3] = {0, 0, 0};  // _bboxWorldUnion2Steps
    double mlo[3] = {0, 0, 0}, mhi[3] = {0, 0, 0};    // mesh: extent of rotation * v about the centre
    MeshView mview{};                                 // mesh: device hierarchy and triangles
    // FDTD_MOTION_KEYFRAMED: the track (solver-owned frames) and the rest rotation it turns
    const double* kf = nullptr;
    int kf_n = 0;
    double kf_step = 0;
    double R0[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    // meshes: object-frame vertices (solver-owned) for the extent of a turned mesh
    const double* mv = nullptr;
    int mv_n = 0;
};

// A validated mesh with its pseudo-normals and hierarchy (fdtd_mesh.cpp).
struct MeshHost {
    std::vector<MeshNode> nodes;
    std::vector<MeshTri> tris;  // leaf order
    std::vector<double> vertices;
};
bool build_mesh(const fdtd_mesh_desc& md, MeshHost& out, std::string& err);
void mesh_extent(const double* verts, size_t nv, const double R[9], double lo[3], double hi[3]);
// A host object of scene object i at rest (mesh extent set; pose and box not yet).
HostObject make_host_object(const fdtd_scene_desc* sc, int i);
bool read_obj(const char* path, double scale, std::vector<double>& verts, std::vector<int32_t>& tris, std::string& err);

struct AxisTables {
    std::vector<uint8_t> pml_cell, pml_face;
    std::vector<double> cpos, fpos, pupd, pdiv, vupd, vgrad;
    std::vector<double> csig;  // absorption coefficient at the cell centres
};

void host_object_pose(HostObject& o, double t);
// keyframed pose at time t: centre and the rotation that turns the rest pose (fdtd_kinematics.cpp)
void keyframe_pose(const double* frames, int n, double step, double t, double com[3], double R[9]);
bool read_kinematics(const char* path, std::vector<double>& frames, std::string& err);
void host_update_bbox(HostObject& o);
void host_reset_union(HostObject& o);

}  // namespace fdtd

struct fdtd_solver {
    fdtd_options opt{};
    int precision = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;   // second stream: interior kernel concurrent with the shell
    cudaStream_t stream3 = nullptr;   // third stream: ghost-cell list beside the interior
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_ghost = nullptr;
    // listener rows of step n run on stream4 beside step n+1; step n+2, which
    // overwrites the pressure they read, waits on ev_lis[parity of step n]
    cudaStream_t stream4 = nullptr;
    cudaEvent_t ev_step = nullptr, ev_lis[2] = {nullptr, nullptr}, ev_lis_join = nullptr;
    bool lis_pending[2] = {false, false};
    // moving bodies clear of the PML: the shell kernel of a step runs on stream5
    // beside that step's classification
    cudaStream_t stream5 = nullptr;
    cudaEvent_t ev_sfork = nullptr, ev_sdone = nullptr;
    // hP.boxes are the boxes of the classification the cell flags hold (the
    // solid cells lie in them); cleared when the flags are loaded from elsewhere
    bool cls_boxes_current = false;
    long long overlapped_steps = 0;
    // geometry
    double h = 0, c = 0, rho = 0, k = 0, end_time = 0, start_time = 0;
    double pml_strength = 0;
    int N[3] = {0, 0, 0};
    long long ncell = 0, n_pml = 0, n_interior = 0;
    long long SX = 0, SY = 0, np = 0;  // padded strides and elements per device array
    long long vcount[3] = {0, 0, 0};
    double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
    fdtd::AxisTables tab[3];
    std::vector<fdtd::HostObject> objs;
    std::vector<fdtd::MeshHost> meshes;     // the scene's meshes (those objects use)
    std::vector<std::vector<double>> kf_store;  // keyframe tracks of the objects (empty: none)
    std::vector<void*> mesh_alloc;          // their device copies
    std::vector<fdtd_plane_desc> planes;
    std::vector<fdtd_gaussian_source_desc> sources;
    std::vector<double> listeners;
    int L = 0;
    bool moving = false;
    int preset = 0;                 // boundary_condition_preset
    std::vector<fdtd::EngCell> eng;  // Engquist-Majda cells (sides without PML)
    int boundary_handling = 0;              // FDTD_BOUNDARY_*
    std::vector<void*> fc_alloc;            // device arrays of the FULLY_COUPLED rows
    long long fc_immersed = 0, fc_fallback = 0;
    // device
    fdtd::SolveParams hP{};
    fdtd::SolveParams* dP = nullptr;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    size_t arena_block = 0;         // bytes of the device block holding the arena (>= its carve)
    int* d_solid_pml = nullptr;
    int n_solid_pml = 0;
    double* d_lap = nullptr;
    int* d_status = nullptr;
    double* d_lis = nullptr;
    double* h_lis_stage = nullptr;
    int lis_cap_steps = 0;
    int xb = 4;                       // planes per thread of the interior kernel
    fdtd::Box3 interior{};            // non-PML box
    fdtd::ShellBoxes shell{};         // PML shell boxes
    fdtd::RegionLaunch region{};      // launch description of the region-split step
    int* d_ghost_list = nullptr;
    int* d_ghost_count = nullptr;
    // stepping state
    int cur = 0;
    long long step_index = 0;
    double time = 0.0;        // simulation time of the next step (host mirror of the device clock)
    double state_time = 0.0;  // SimWorld::_state.time for object animation
    bool classified_after_first_step = false;
    cudaGraphExec_t graph_exec[4] = {nullptr, nullptr, nullptr, nullptr};  // [parity + 2*sources]
    long long launches = 0;
    long long last_launches = 0;
    long long graph_launches_per_exec = 0;
    fdtd::TmaStep* tma = nullptr;     // tiles and tensor maps of the TMA-staged shell (reduced state)
    // bytes this handle copied between host and device memory since creation
    long long bytes_h2d = 0, bytes_d2h = 0;
    std::string err;
};

namespace fdtd {
// Host<->device copies of a solver handle, added to its transfer totals
// (fdtd_solver_transfer_bytes); s may be NULL.
inline void count_transfer(fdtd_solver* s, size_t n, cudaMemcpyKind kind) {
    if (!s) return;
    if (kind == cudaMemcpyHostToDevice) s->bytes_h2d += (long long)n;
    else if (kind == cudaMemcpyDeviceToHost) s->bytes_d2h += (long long)n;
}
inline cudaError_t counted_copy(fdtd_solver* s, void* dst, const void* src, size_t n, cudaMemcpyKind kind) {
    count_transfer(s, n, kind);
    return cudaMemcpy(dst, src, n, kind);
}
inline cudaError_t counted_copyAsync(fdtd_solver* s, void* dst, const void* src, size_t n, cudaMemcpyKind kind,
                                     cudaStream_t stream) {
    count_transfer(s, n, kind);
    return cudaMemcpyAsync(dst, src, n, kind, stream);
}
void set_error(fdtd_solver* s, const std::string& msg);
// moving bodies two cells clear of the PML through [start_time, end_time]
bool moving_clear_of_pml(fdtd_solver* s);
// A batch member made outside the batch: its solver created and its first step
// run (or its snapshot restored), ready to be placed between two batched steps
// (fdtd_batch.cpp).  batch_prepare touches no batch state, so a server prepares
// members on another host thread while its batch steps.
struct PreparedMember {
    fdtd_solver* s = nullptr;
    int64_t total = 0, done = 0;
    std::vector<double> rows;
};
fdtd_status batch_prepare(const fdtd_options& batch_opt, const fdtd_scene_desc* scene, int32_t steps_total,
                          const void* snapshot, int64_t snapshot_bytes, const double* rows, int64_t steps_done,
                          PreparedMember* out, std::string* err);
int32_t batch_place(fdtd_batch* b, PreparedMember&& pm);
// Device blocks for solver arenas, kept after a solver is destroyed for the next
// one on the same device (fdtd_api.cpp)
cudaError_t arena_acquire(int device, size_t bytes, void** ptr, size_t* block_bytes);
void arena_release(int device, void* ptr, size_t block_bytes);
// listener plans of a static solve from its current classification (after a restore)
fdtd_status rebuild_listener_plans(fdtd_solver* s);
// fdtd_debug_inject_failure: true when this allocation of kind `what` is to fail
bool inject_failure(int what);
// TMA-staged PML shell (fdtd_tma.cpp)
bool tma_encoder_available();
fdtd_status build_shell_tma(fdtd_solver* s);
void free_shell_tma(fdtd_solver* s);
fdtd_status solver_init_geometry(fdtd_solver* s, const fdtd_scene_desc* sc);
void classification_boxes(const fdtd_solver* s, ClsBoxes& B);
void to_dev_objects(fdtd_solver* s);
fdtd_status build_fully_coupled(fdtd_solver* s);
void free_fully_coupled(fdtd_solver* s);
}  // namespace fdtd
