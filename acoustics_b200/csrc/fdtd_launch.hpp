// fdtd_launch.hpp — host-callable launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "fdtd_device.cuh"

namespace fdtd {

// Streams of one step.  The step is enqueued on s and ends on s; in between the
// ghost-cell list runs on s3 (launched first: a few latency-bound CTAs next to
// the interior's), the interior and then the sources on s2, the PML shell on s.
// s2 / s3 may be null (everything on s).
struct StepStreams {
    cudaStream_t s, s2, s3;
    cudaEvent_t fork, join, ghost;
};

// region-split step: PML shell, interior, ghost-neighbour list and (while active) sources
cudaError_t launch_step_regions_fp64(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                                     const StepStreams& S, int* launches);
cudaError_t launch_step_regions_fp32(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                                     const StepStreams& S, int* launches);

// batched step of many members (fdtd_batch.cuh)
cudaError_t launch_batch_fp64(const BatchLaunch& L, const StepStreams& S, int* launches);
cudaError_t launch_batch_fp32(const BatchLaunch& L, const StepStreams& S, int* launches);
// listener rows / advance of a batched step, for either field type (FP64 unit)
cudaError_t launch_batch_listeners_any(int precision, const BatchLaunch& L, cudaStream_t s, int* launches);
cudaError_t launch_batch_advance_any(int precision, const BatchLaunch& L, cudaStream_t s, int* launches);

// fdtd_fp64.cu (compiled with -fmad=false)
cudaError_t launch_prologue_fp64(const SolveParams* dP, int cur, int advance, int n_solid_pml, cudaStream_t s);
cudaError_t launch_listener_prep(SolveParams* dP, int precision, int newp, int n_lis, cudaStream_t s);
cudaError_t launch_consts_init(const SolveParams* dP, double t0, cudaStream_t s);
cudaError_t launch_listeners(const SolveParams* dP, int precision, int newp, int n_lis, double* out_row,
                             cudaStream_t s);
// cell classification over the boxes B (a copy of dP->boxes): the box solid
// test, the sweep over the units no box reaches and the one over those it does
// (3 launches; the last only when some box has cells).  With `prev` (the boxes
// of the classification before, when every cell outside them is known to hold
// the default flags) the first sweep visits only the units those reached.
cudaError_t launch_classify(const SolveParams* dP, const int N[3], const ClsBoxes& B, bool collect_fresh,
                            cudaStream_t s, const ClsBoxes* prev = nullptr);
cudaError_t launch_cls_history(const SolveParams* dP, long long ncell, int* count, int* list, int cap, cudaStream_t s);
cudaError_t launch_fresh_cells(const SolveParams* dP, int precision, int cur, long long ncell, int* d_status,
                               cudaStream_t s);

// plain FP64 path, one kernel per reference phase
cudaError_t launch_phased_fp64(const SolveParams* dP, const int N[3], int cur, double* lap, cudaStream_t s,
                               int* launches);

// fdtd_fetch.cu: cell read-back (FetchCell / SampleAxisAlignedSlice).  A request
// is a padded cell index and the element addresses of its split pressures
// (a[0..2]) and of its lower (a[3+2d]) and upper (a[4+2d]) face velocities,
// null where the solve does not hold them.
struct FetchReq {
    long long c;
    const void* a[9];
};
struct FetchVal {
    double p, p_prev;   // p^{n+1} (current) and p^n
    double pdir[3];
    double v[6];        // lower / upper face along x, y, z
    double gc[6];       // ghost-face pressures of the last step toward -x,+x,-y,+y,-z,+z; -1: none
    double lap;         // the Laplacian kept for the next step (air viscosity), else NaN
    int cls, gobj;      // classification byte and ghost-object byte
};
cudaError_t launch_fetch_cells(const SolveParams* dP, bool fp64, int cur, const FetchReq* req, FetchVal* out, int n,
                               cudaStream_t s);

// fdtd_fp32.cu
cudaError_t prepare_fp32_kernels();
// fdtd_fp64.cu: shared-memory limits of the FP64 kernels that stage loads
cudaError_t prepare_fp64_kernels();
cudaError_t launch_prologue_fp32(const SolveParams* dP, int cur, int advance, int n_solid_pml, cudaStream_t s);

}  // namespace fdtd
