// fdtd_stencil.cuh — per-cell update formulas shared by the step kernels:
// PML face velocity (MAC_Grid.cpp:461-479), PML split-field pressure
// (MAC_Grid.cpp:496-508), the Gaussian pressure sources
// (GaussianPressureSource.cpp:6-30), the step prologue and the step-constant
// initialisation.
//
// Precision variants of the leapfrog (fdtd_hot.cuh, fdtd_region.cuh):
//   double, in-place leapfrog: p^{n+1} overwrites p^{n-1} (each cell reads only
//     its own p^{n-1}); bit-faithful to the reference operation order when the
//     translation unit is compiled with -fmad=false.
//   float, compensated: the increment d = p^n - p^{n-1} is stored, and
//     d^{n+1} = d^n + (ck)^2 lap + k src, p^{n+1} = p^n + d^{n+1}, so that the
//     leapfrog's rounding error does not integrate twice.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_geometry.cuh"

namespace fdtd {

template <typename T>
struct Coef;
template <>
struct Coef<double> {
    __device__ static const double* pupd(const SolveParams& P, int d) { return P.pupd[d]; }
    __device__ static const double* pdiv(const SolveParams& P, int d) { return P.pdiv[d]; }
    __device__ static const double* vupd(const SolveParams& P, int d) { return P.vupd[d]; }
    __device__ static const double* vgrad(const SolveParams& P, int d) { return P.vgrad[d]; }
};
template <>
struct Coef<float> {
    __device__ static const float* pupd(const SolveParams& P, int d) { return P.pupd_f[d]; }
    __device__ static const float* pdiv(const SolveParams& P, int d) { return P.pdiv_f[d]; }
    __device__ static const float* vupd(const SolveParams& P, int d) { return P.vupd_f[d]; }
    __device__ static const float* vgrad(const SolveParams& P, int d) { return P.vgrad_f[d]; }
};

// v <- v*upd + grad*pR - grad*pL   (MAC_Grid.cpp:471-474).  FP64: the reference's
// roundings in its order (the unit is compiled without FMA contraction).  FP32:
// two explicit FMAs, so the result does not depend on how the compiler
// contracts a given instantiation (every device unit is built with -fmad=false).
template <typename T>
__device__ __forceinline__ T vel_update(T v, T upd, T grad, T pR, T pL) {
    if constexpr (sizeof(T) == 4) {
        return fmaf(-grad, pL, fmaf(grad, pR, v * upd));
    } else {
        T r = v * upd;
        r = r + grad * pR;
        r = r - grad * pL;
        return r;
    }
}

// p_d <- p_d*upd + div*vR/h - div*vL/h   (MAC_Grid.cpp:500-505); FP32 as above
template <typename T>
__device__ __forceinline__ T pd_update(T pd, T upd, T div, T vR, T vL, T inv_h) {
    if constexpr (sizeof(T) == 4) {
        const float dv = div * inv_h;
        return fmaf(-dv, vL, fmaf(dv, vR, pd * upd));
    } else {
        T r = pd * upd;
        r = r + div * vR * inv_h;
        r = r - div * vL * inv_h;
        return r;
    }
}

// Sum of the Gaussian pressure sources at a cell centre (GaussianPressureSource.cpp:6-30,
// FDTD_Objects.cpp:356-367); the time factor comes precomputed from the prologue.
static __device__ __noinline__ double source_sum(const SolveParams& P, const StepConsts& sc, double x, double y,
                                          double z) {
    double sum = 0;
    for (int s = 0; s < P.n_src; ++s) {
        const DevSource& S = P.src[s];
        double v = 0.0;
        if (x < S.bmax[0] && x > S.bmin[0] && y < S.bmax[1] && y > S.bmin[1] && z < S.bmax[2] && z > S.bmin[2]) {
            v = (x - S.cen[0]) * (x - S.cen[0]) + (y - S.cen[1]) * (y - S.cen[1]) + (z - S.cen[2]) * (z - S.cen[2]);
            v = -v / S.denom;
            v = exp(v);
            v *= sc.src_tf[s];
            v *= S.scale;
        }
        sum += v;
    }
    return sum;
}

// Step prologue: advances the step constants (PML_WaveSolver.cpp:825
// _currentTime += _timeStep) and re-zeroes solid cells inside the PML, which
// classifyCells_FAST zeroes at the start of every step (MAC_Grid.cpp:3796-3798).
template <typename T>
__global__ void k_prologue(const SolveParams* __restrict__ Pp, int cur, int advance) {
    const SolveParams& P = *Pp;
    if (advance && blockIdx.x == 0 && threadIdx.x == 0) advance_consts(P, cur);
    T* p0 = (T*)P.p[0];
    T* p1 = (T*)P.p[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_solid_pml; i += gridDim.x * blockDim.x) {
        const int c = P.solid_pml[i];
        p0[c] = (T)0;
        p1[c] = (T)0;
        if (P.dinc) P.dinc[c] = 0.0f;
    }
}

// consts[0] <- the constants of the first step at time t0.
static __global__ void k_consts_init(const SolveParams* __restrict__ Pp, double t0) {
    const SolveParams& P = *Pp;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.consts[1].t = t0 - P.k;
        P.consts[1].step = -1;
        advance_consts(P, 1);
        P.consts[0].t = t0;
        P.consts[0].step = 0;
    }
}

}  // namespace fdtd
