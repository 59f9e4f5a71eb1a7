// fdtd_region.cuh — the step split by region, one lean kernel per region:
//
//   k_interior   non-PML cells, box [lo, hi): ghost-aware Laplacian, leapfrog /
//                compensated increment, Gaussian sources
//                (MAC_Grid.cpp:187-299 + :921-944).  Only pressure words move:
//                p^n (neighbours from the CTA's rows), p^{n-1} or the increment,
//                p^{n+1}, plus one classification byte.
//   k_pml_shell  the six slab boxes of the PML shell: face velocities
//                (MAC_Grid.cpp:461-479) and split-field pressures (:496-508).
//
// Face ownership: a PML face is written by the cell to its right; the one face
// layer whose right cell is not a PML cell (x = W h on the low side) is written
// by its left (PML) cell, so the interior kernel never touches velocities.
//
// Cells next to a solid (a compact list built by the classification) and the
// Gaussian sources while they are active have kernels of their own, so the
// interior kernel is a pure 7-point leapfrog.
//
// Interior mapping: a CTA of 32 (z) x 8 (y) threads, each thread owns XB
// consecutive x planes of one (y, z) column.  All loads of the XB planes
// (p^n at XB+2 planes, y neighbours, p^{n-1}/increment, classification) are
// issued before any arithmetic so that every thread keeps ~5*XB independent
// HBM requests in flight; z neighbours come from the warp with shuffles.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_coupled.cuh"
#include "fdtd_geometry.cuh"
#include "fdtd_stencil.cuh"

namespace fdtd {

// Ghost-aware Laplacian of one bulk cell with at least one solid neighbour
// (MAC_Grid.cpp:267-297); returns the unscaled sum and the number of axes with
// ghost cells on both sides.
template <typename T>
__device__ __noinline__ T ghost_laplacian(const SolveParams& P, long long c, const int idx[3], unsigned mask, T p0,
                                          const T nbp[3], const T nbm[3], double t, int par, int* surrounded) {
    const long long strides[3] = {P.SX, P.SY, 1};
    T lap = 0.0;
    int s = 0;
    for (int d = 0; d < 3; ++d) {
        const bool gn = (mask >> (2 * d)) & 1u;
        const bool gp = (mask >> (2 * d + 1)) & 1u;
        T gpv = 0, gnv = 0;
        if (gp || gn) {
            double own[3] = {P.cpos[0][idx[0]], P.cpos[1][idx[1]], P.cpos[2][idx[2]]};
            // FULLY_COUPLED: the solved ghost pressures of this step; RASTERIZE: pg
            if (gp) {
                own[d] = P.cpos[d][idx[d] + 1];
                gpv = P.fc_rows ? (T)fc_ghost(P, par, c + strides[d], 2 * d, (double)p0)
                                : (T)ghost_pressure(P, P.gobj[c + strides[d]], own, d, -1, (double)p0, t);
            }
            if (gn) {
                own[d] = P.cpos[d][idx[d] - 1];
                gnv = P.fc_rows ? (T)fc_ghost(P, par, c - strides[d], 2 * d + 1, (double)p0)
                                : (T)ghost_pressure(P, P.gobj[c - strides[d]], own, d, +1, (double)p0, t);
            }
        }
        if (gp && gn) {
            lap = lap + (gpv + gnv - (T)2.0 * p0) / (T)(9.0 / 16.0);
            ++s;
        } else if (gp) {
            lap = lap + (gpv + (T)0.75 * nbm[d] - (T)(7.0 / 4.0) * p0) / (T)(21.0 / 32.0);
        } else if (gn) {
            lap = lap + ((T)0.75 * nbp[d] + gnv - (T)(7.0 / 4.0) * p0) / (T)(21.0 / 32.0);
        } else {
            lap = lap + (nbp[d] + nbm[d] - (T)2.0 * p0);
        }
    }
    *surrounded = s;
    return lap;
}

// Full update of one non-PML bulk cell next to a solid (ghost-aware Laplacian,
// cavity freeze), everything re-read from memory.  Sources are added by
// k_sources afterwards, as the reference adds them after the update
// (MAC_Grid.cpp:938-944).
template <typename T>
__device__ __forceinline__ void ghost_cells_body(const SolveParams& P, int cur, int bid, int nblocks) {
    const int n = *P.ghost_count;
    const long long sx = P.SX, sy = P.SY;
    const T* __restrict__ pc = (const T*)P.p[cur];
    T* __restrict__ pn = (T*)P.p[cur ^ 1];
    const double t = P.consts[cur].t;
    for (int g = bid * blockDim.x + threadIdx.x; g < n && g < P.ghost_cap; g += nblocks * blockDim.x) {
        const long long c = P.ghost_list[g];
        int x, y, z;
        cell_ijk(P, c, x, y, z);
        const uint8_t code = P.cls[c];
        const T p0 = pc[c];
        const T nbp[3] = {pc[c + sx], pc[c + sy], pc[c + 1]};
        const T nbm[3] = {pc[c - sx], pc[c - sy], pc[c - 1]};
        const int idx[3] = {x, y, z};
        int surrounded = 0;
        T lap = ghost_laplacian<T>(P, c, idx, code & CLS_MASK, p0, nbp, nbm, t, cur, &surrounded);
        lap = lap * (T)P.lap_scale;
        const bool cavity = (surrounded > 1) && (code & CLS_VALID);
        // air viscosity on cells with a valid history (MAC_Grid.cpp:926-930)
        const bool visc = P.visc && (code & CLS_VALID);
        T lapl = 0;
        if (P.visc) {
            lapl = ((const T*)P.lapv[cur ^ 1])[c];
            ((T*)P.lapv[cur])[c] = lap;
        }
        if constexpr (sizeof(T) == 8) {
            if (cavity) pn[c] = p0;
            else if (visc) pn[c] = (T)2.0 * p0 - pn[c] - lapl * (T)P.kcalp + lap * (T)(P.c2k2 + P.kcalp);
            else pn[c] = (T)2.0 * p0 - pn[c] + lap * (T)P.c2k2;
        } else {
            float d = cavity ? 0.0f : P.dinc[c] + (float)(lap * (T)P.c2k2);
            if (!cavity && visc) d = fmaf((float)P.kcalp, (float)(lap - lapl), d);
            P.dinc[c] = d;
            pn[c] = p0 + d;
        }
    }
}

// pNext += k * sum_s G_s(x, t + k/2) over the bounding box of the source
// supports clipped to the non-PML box (GaussianPressureSource.cpp:6-30), with
// G_s = (product of the per-axis spatial factors) * (time factor of the step).
template <typename T>
__device__ __forceinline__ void sources_body(const SolveParams& P, int cur, const Box3& region, int bid, int nblocks) {
    const StepConsts& sc = P.consts[cur];
    bool any_src = false;
    for (int s = 0; s < P.n_src; ++s) any_src |= (sc.src_tf[s] != 0.0);
    if (!any_src) return;
    const int nx = region.hi[0] - region.lo[0], ny = region.hi[1] - region.lo[1], nz = region.hi[2] - region.lo[2];
    const long long total = (long long)nx * ny * nz;
    const T* __restrict__ pc = (const T*)P.p[cur];
    T* __restrict__ pn = (T*)P.p[cur ^ 1];
    for (long long t = bid * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)nblocks * blockDim.x) {
        const int z = region.lo[2] + (int)(t % nz);
        const int y = region.lo[1] + (int)((t / nz) % ny);
        const int x = region.lo[0] + (int)(t / ((long long)nz * ny));
        const long long c = cidx(P, x, y, z);
        if (!(P.cls[c] & CLS_BULK)) continue;
        const double src = source_term(P, cur, x, y, z);
        if constexpr (sizeof(T) == 8) {
            pn[c] += src * P.k;
        } else {
            const float d = P.dinc[c] + (float)(src * P.k);
            P.dinc[c] = d;
            pn[c] = pc[c] + d;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(128) k_ghost_cells(const SolveParams* __restrict__ Pp, int cur) {
    ghost_cells_body<T>(*Pp, cur, blockIdx.x, gridDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_sources(const SolveParams* __restrict__ Pp, int cur, Box3 region) {
    sources_body<T>(*Pp, cur, region, blockIdx.x, gridDim.x);
}

}  // namespace fdtd
