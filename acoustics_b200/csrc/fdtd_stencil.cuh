// fdtd_stencil.cuh — the fused step kernel: PML face-velocity update, PML
// split-field pressure update, ghost-aware Laplacian, interior leapfrog and the
// Gaussian pressure sources of one time step, in one pass over the grid.
//
// It fuses these reference phases of PML_WaveSolver::stepCollocated
// (PML_WaveSolver.cpp:775-826):
//   PML_pressureUpdateGhostCells   MAC_Grid.cpp:1131-1441 (RASTERIZE, evaluated where used)
//   PML_velocityUpdateCollocated   MAC_Grid.cpp:461-479
//   pressureFieldLaplacianGhostCell MAC_Grid.cpp:187-299
//   PML_pressureUpdateCollocated   MAC_Grid.cpp:481-946
//
// Grid mapping (2.5D streaming): a CTA of 32 x BY threads owns a 32-wide z
// strip of BY y rows and marches along x, the slowest axis, over x_chunk
// planes.  Each thread keeps p(x-1), p(x), p(x+1) of its column in registers,
// takes z neighbours from its warp with shuffles and y neighbours from the
// L1-resident rows of the CTA.  The x face velocity of the right face of
// plane x is the left face of plane x+1 and is carried in a register.
//
// Precision variants:
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

template <typename T, int BY>
__global__ void __launch_bounds__(32 * BY) k_step_fused(const SolveParams* __restrict__ Pp, int cur, int xchunk) {
    const SolveParams& P = *Pp;
    const int lane = threadIdx.x;
    const int z = blockIdx.x * 32 + lane;
    const int y = blockIdx.y * BY + threadIdx.y;
    const int Nx = P.N[0], Ny = P.N[1], Nz = P.N[2];
    const bool active = (y < Ny) && (z < Nz);
    const int zc = z < Nz ? z : Nz - 1;  // inactive lanes shadow a valid column for shuffles
    const int yc = y < Ny ? y : Ny - 1;
    const int x0 = blockIdx.z * xchunk;
    const int x1 = min(x0 + xchunk, Nx);
    if (x0 >= Nx) return;
    const long long sx = (long long)Ny * Nz;
    const int sy = Nz;
    const T* __restrict__ pc = (const T*)P.p[cur];
    T* __restrict__ pn = (T*)P.p[cur ^ 1];
    T* __restrict__ pdx = (T*)P.pd[0];
    T* __restrict__ pdy = (T*)P.pd[1];
    T* __restrict__ pdz = (T*)P.pd[2];
    const T* __restrict__ vox = (const T*)P.v[cur][0];
    const T* __restrict__ voy = (const T*)P.v[cur][1];
    const T* __restrict__ voz = (const T*)P.v[cur][2];
    T* __restrict__ vnx = (T*)P.v[cur ^ 1][0];
    T* __restrict__ vny = (T*)P.v[cur ^ 1][1];
    T* __restrict__ vnz = (T*)P.v[cur ^ 1][2];
    const uint8_t* __restrict__ cls = P.cls;
    const StepConsts sc = P.consts[cur];
    const T inv_h = (T)P.inv_h;
    const T c2k2 = (T)P.c2k2;
    const T lap_scale = (T)P.lap_scale;
    const bool pmly = P.pml_cell[1][yc] != 0;
    const bool pmlz = P.pml_cell[2][zc] != 0;
    const bool pfy_l = (yc > 0) && (P.pml_face[1][yc] != 0);
    const bool pfz_l = (zc > 0) && (P.pml_face[2][zc] != 0);
    const bool pfy_r = (yc + 1 < Ny) && (P.pml_face[1][yc + 1] != 0);
    const bool pfz_r = (zc + 1 < Nz) && (P.pml_face[2][zc + 1] != 0);
    const T vupd_y = Coef<T>::vupd(P, 1)[yc], vgrad_y = Coef<T>::vgrad(P, 1)[yc];
    const T vupd_z = Coef<T>::vupd(P, 2)[zc], vgrad_z = Coef<T>::vgrad(P, 2)[zc];
    const T vupd_yr = Coef<T>::vupd(P, 1)[yc + 1], vgrad_yr = Coef<T>::vgrad(P, 1)[yc + 1];
    const T vupd_zr = Coef<T>::vupd(P, 2)[zc + 1], vgrad_zr = Coef<T>::vgrad(P, 2)[zc + 1];
    const T pupd_y = Coef<T>::pupd(P, 1)[yc], pdiv_y = Coef<T>::pdiv(P, 1)[yc];
    const T pupd_z = Coef<T>::pupd(P, 2)[zc], pdiv_z = Coef<T>::pdiv(P, 2)[zc];
    const double cy = P.cpos[1][yc], cz = P.cpos[2][zc];
    bool any_src = false;
    for (int s = 0; s < P.n_src; ++s) any_src |= (sc.src_tf[s] != 0.0);

    // face-velocity flat indices at plane x0
    const long long fy_stride_x = (long long)(Ny + 1) * Nz;
    const long long fz_stride_x = (long long)Ny * (Nz + 1);
    long long c = (long long)x0 * sx + (long long)yc * sy + zc;
    long long fy = (long long)x0 * fy_stride_x + (long long)yc * Nz + zc;
    long long fz = (long long)x0 * fz_stride_x + (long long)yc * (Nz + 1) + zc;

    T p_xm = x0 > 0 ? pc[c - sx] : pc[c];
    T p_0 = pc[c];
    // x face velocity of the left face of plane x0 (new value), carried along x
    T vx_left = vox[c];
    if ((x0 > 0) && (P.pml_face[0][x0] != 0 || pmly || pmlz))
        vx_left = vel_update<T>(vx_left, Coef<T>::vupd(P, 0)[x0], Coef<T>::vgrad(P, 0)[x0], p_0, p_xm);
    for (int x = x0; x < x1; ++x) {
        const T p_xp = (x + 1 < Nx) ? pc[c + sx] : p_0;
        const bool pmlx = P.pml_cell[0][x] != 0;
        const bool pml = pmlx || pmly || pmlz;
        // z neighbours from the warp, edges from memory
        T p_zm = __shfl_up_sync(0xffffffffu, p_0, 1);
        T p_zp = __shfl_down_sync(0xffffffffu, p_0, 1);
        if (lane == 0) p_zm = zc > 0 ? pc[c - 1] : p_0;
        if (lane == 31 || z + 1 >= Nz) p_zp = (zc + 1 < Nz) ? pc[c + 1] : p_0;
        if (zc == 0) p_zm = p_0;
        const T p_ym = yc > 0 ? pc[c - sy] : p_0;
        const T p_yp = yc + 1 < Ny ? pc[c + sy] : p_0;
        // a face lies in the PML when InsidePML holds at its position (MAC_Grid.cpp:2631-2633);
        // faces at index 0 and N_d are the rigid outer wall and never change (:2568-2575)
        const bool fxl = (x > 0) && (P.pml_face[0][x] != 0 || pmly || pmlz);
        const bool fxr = (x + 1 < Nx) && (P.pml_face[0][x + 1] != 0 || pmly || pmlz);
        const bool fyl = (yc > 0) && (pfy_l || pmlx || pmlz);
        const bool fyr = (yc + 1 < Ny) && (pfy_r || pmlx || pmlz);
        const bool fzl = (zc > 0) && (pfz_l || pmlx || pmly);
        const bool fzr = (zc + 1 < Nz) && (pfz_r || pmlx || pmly);
        if (active) {
            // ---- face velocities owned by this cell (left faces), MAC_Grid.cpp:461-479 ----
            T vy_l = 0, vz_l = 0;
            if (fyl || pml) vy_l = voy[fy];
            if (fzl || pml) vz_l = voz[fz];
            if (fyl) {
                vy_l = vel_update<T>(vy_l, vupd_y, vgrad_y, p_0, p_ym);
                vny[fy] = vy_l;
            }
            if (fzl) {
                vz_l = vel_update<T>(vz_l, vupd_z, vgrad_z, p_0, p_zm);
                vnz[fz] = vz_l;
            }
            if (fxl) vnx[c] = vx_left;
            // right x face (the next plane's left face), new value carried in a register
            T vx_r = vox[c + sx];
            if (fxr) vx_r = vel_update<T>(vx_r, Coef<T>::vupd(P, 0)[x + 1], Coef<T>::vgrad(P, 0)[x + 1], p_xp, p_0);

            if (pml) {
                // ---- split-field PML pressure, MAC_Grid.cpp:496-508 ----
                T vy_r = voy[fy + Nz];
                T vz_r = voz[fz + 1];
                if (fyr) vy_r = vel_update<T>(vy_r, vupd_yr, vgrad_yr, p_yp, p_0);
                if (fzr) vz_r = vel_update<T>(vz_r, vupd_zr, vgrad_zr, p_zp, p_0);
                const T ax = pd_update<T>(pdx[c], Coef<T>::pupd(P, 0)[x], Coef<T>::pdiv(P, 0)[x], vx_r, vx_left, inv_h);
                const T ay = pd_update<T>(pdy[c], pupd_y, pdiv_y, vy_r, vy_l, inv_h);
                const T az = pd_update<T>(pdz[c], pupd_z, pdiv_z, vz_r, vz_l, inv_h);
                pdx[c] = ax;
                pdy[c] = ay;
                pdz[c] = az;
                pn[c] = ax + ay + az;
            } else {
                const uint8_t code = cls[c];
                if (code & CLS_BULK) {
                    // ---- ghost-aware Laplacian, MAC_Grid.cpp:267-297 ----
                    const unsigned mask = code & CLS_MASK;
                    T lap = 0.0;
                    int surrounded = 0;
                    if (mask == 0) {
                        lap = lap + (p_xp + p_xm - (T)2.0 * p_0);
                        lap = lap + (p_yp + p_ym - (T)2.0 * p_0);
                        lap = lap + (p_zp + p_zm - (T)2.0 * p_0);
                    } else {
                        const T nbp[3] = {p_xp, p_yp, p_zp};
                        const T nbm[3] = {p_xm, p_ym, p_zm};
                        const long long strides[3] = {sx, (long long)sy, 1};
                        const int idx[3] = {x, yc, zc};
                        for (int d = 0; d < 3; ++d) {
                            const bool gn = (mask >> (2 * d)) & 1u;
                            const bool gp = (mask >> (2 * d + 1)) & 1u;
                            T gpv = 0, gnv = 0;
                            if (gp || gn) {
                                double own[3] = {P.cpos[0][x], cy, cz};
                                if (gp) {
                                    own[d] = P.cpos[d][idx[d] + 1];
                                    gpv = (T)ghost_pressure(P, P.gobj[c + strides[d]], own, d, -1, (double)p_0, sc.t);
                                }
                                if (gn) {
                                    own[d] = P.cpos[d][idx[d] - 1];
                                    gnv = (T)ghost_pressure(P, P.gobj[c - strides[d]], own, d, +1, (double)p_0, sc.t);
                                }
                            }
                            if (gp && gn) {
                                lap = lap + (gpv + gnv - (T)2.0 * p_0) / (T)(9.0 / 16.0);
                                ++surrounded;
                            } else if (gp) {
                                lap = lap + (gpv + (T)0.75 * nbm[d] - (T)(7.0 / 4.0) * p_0) / (T)(21.0 / 32.0);
                            } else if (gn) {
                                lap = lap + ((T)0.75 * nbp[d] + gnv - (T)(7.0 / 4.0) * p_0) / (T)(21.0 / 32.0);
                            } else {
                                lap = lap + (nbp[d] + nbm[d] - (T)2.0 * p_0);
                            }
                        }
                    }
                    lap = lap * lap_scale;
                    const bool cavity = (surrounded > 1) && (code & CLS_VALID);
                    double src = 0.0;
                    if (any_src) src = source_sum(P, sc, P.cpos[0][x], cy, cz);
                    if constexpr (sizeof(T) == 8) {
                        // ---- leapfrog, MAC_Grid.cpp:921-944 ----
                        T pnext;
                        if (cavity) {
                            pnext = p_0;
                        } else {
                            pnext = (T)2.0 * p_0 - pn[c] + lap * c2k2;
                        }
                        if (P.n_src > 0) pnext += src * P.k;
                        pn[c] = pnext;
                    } else {
                        // ---- compensated increment form ----
                        float d = P.dinc[c];
                        if (cavity) {
                            d = 0.0f;
                        } else {
                            d = d + lap * c2k2;
                        }
                        if (any_src) d = d + (float)(src * P.k);
                        P.dinc[c] = d;
                        pn[c] = p_0 + d;
                    }
                }
            }
            vx_left = vx_r;
        }
        // advance the column
        p_xm = p_0;
        p_0 = p_xp;
        c += sx;
        fy += fy_stride_x;
        fz += fz_stride_x;
    }
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
