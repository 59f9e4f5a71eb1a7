// fdtd_fp64.cu — FP64 step kernels, cell classification, listener sampling and
// fresh-cell interpolation.  Compiled with -fmad=false: every product and sum
// is rounded on its own, in the order the reference writes it, which keeps the
// FP64 path and the classification bit-reproducible against a CPU build of the
// same expressions.
#include <cuda_runtime.h>

#include "fdtd_device.cuh"
#include "fdtd_geometry.cuh"
#include "fdtd_launch.hpp"
#include "fdtd_listeners.cuh"
#include "fdtd_stencil.cuh"

namespace fdtd {

// ---------------------------------------------------------------------------
// Cell classification (MAC_Grid::classifyCells_FAST, MAC_Grid.cpp:3455-3891)
// ---------------------------------------------------------------------------

// validHistory <- isBulk; isBulk <- true (MAC_Grid.cpp:3464-3472)
__global__ void k_cls_reset(const SolveParams* __restrict__ Pp, long long n) {
    const SolveParams& P = *Pp;
    uint8_t* cls = P.cls;
    if (blockIdx.x == 0 && threadIdx.x == 0) *P.ghost_count = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        dense_ijk(P, t, i, j, k);
        const long long c = cidx(P, i, j, k);
        const uint8_t code = cls[c];
        cls[c] = CLS_BULK | ((code & CLS_BULK) ? CLS_VALID : 0);
    }
}

// Solid test over one object / constraint iteration box (MAC_Grid.cpp:3608-3653)
// and zeroing of the pressure buffers at solid cells (MAC_Grid.cpp:3796-3798).
__global__ void k_cls_solid(const SolveParams* __restrict__ Pp, int s0, int s1, int s2, int r0, int r1, int r2) {
    const SolveParams& P = *Pp;
    const long long total = (long long)r0 * r1 * r2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = s0 + (int)(t / ((long long)r1 * r2));
        const int j = s1 + (int)((t / r2) % r1);
        const int k = s2 + (int)(t % r2);
        const long long c = cidx(P, i, j, k);
        const double pos[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]};
        int type = 0;
        if (!is_fluid(P, pos, type)) {
            P.cls[c] = P.cls[c] & (uint8_t)~CLS_BULK;
            P.gobj[c] = type ? GOBJ_CONSTRAINT : 0;
            if (P.precision == 0) {
                ((double*)P.p[0])[c] = 0.0;
                ((double*)P.p[1])[c] = 0.0;
            } else {
                ((float*)P.p[0])[c] = 0.0f;
                ((float*)P.p[1])[c] = 0.0f;
                P.dinc[c] = 0.0f;
            }
        }
    }
}

// Neighbour masks: for a solid cell the directions of its bulk neighbours (one
// ghost face each, MakeGhostCell MAC_Grid.cpp:4310-4340) and its closest
// object (LowestObjectDistance, MAC_Grid.cpp:3810-3814); for a bulk cell the
// directions of its solid (ghost) neighbours, read by the Laplacian.
__global__ void k_cls_ghost(const SolveParams* __restrict__ Pp, long long n) {
    const SolveParams& P = *Pp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        dense_ijk(P, t, i, j, k);
        const long long c = cidx(P, i, j, k);
        const int idx[3] = {i, j, k};
        const long long strides[3] = {P.SX, P.SY, 1};
        const uint8_t code = P.cls[c];
        const bool bulk = code & CLS_BULK;
        unsigned mask = 0;
        for (int d = 0; d < 3; ++d) {
            if (idx[d] > 0) {
                const bool nb = P.cls[c - strides[d]] & CLS_BULK;
                if (bulk != nb) mask |= 1u << (2 * d);
            }
            if (idx[d] + 1 < P.N[d]) {
                const bool nb = P.cls[c + strides[d]] & CLS_BULK;
                if (bulk != nb) mask |= 1u << (2 * d + 1);
            }
        }
        if (!bulk) {
            const double pos[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]};
            const int o = lowest_object(P, pos);
            P.gobj[c] = (P.gobj[c] & GOBJ_CONSTRAINT) | (uint8_t)(o < 0 ? GOBJ_NONE : o);
        } else if (mask && !(P.pml_cell[0][i] || P.pml_cell[1][j] || P.pml_cell[2][k])) {
            // non-PML bulk cell next to a solid: updated by k_ghost_cells
            const int slot = atomicAdd(P.ghost_count, 1);
            if (slot < P.ghost_cap) P.ghost_list[slot] = (int)c;
        }
        P.cls[c] = (uint8_t)((code & (CLS_BULK | CLS_VALID)) | mask);
    }
}

// Listener sampling: fdtd_listeners.cuh (one warp per listener)

// ---------------------------------------------------------------------------
// Fresh-cell interpolation (MAC_Grid::InterpolateFreshPressureCell, MLS branch,
// MAC_Grid.cpp:1993-2254): a cell that is bulk now but was solid before gets
// p = p_MLS(image point) + rho (a . n) |s| in p^{n-1} and p^n.
// ---------------------------------------------------------------------------
template <typename T>
__device__ double fresh_value(const SolveParams& P, const T* __restrict__ pa, const T* __restrict__ pb, bool diff,
                              long long c, double t, int* status) {
    // value of buffer "a" (or a - b when diff) at cell n
    auto val = [&](long long n) -> double { return diff ? (double)pa[n] - (double)pb[n] : (double)pa[n]; };
    int i, j, k;
    cell_ijk(P, c, i, j, k);
    const double cp[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]};
    double distance = DBL_MAX;
    const int oid = lowest_object(P, cp, &distance);
    if (oid < 0 || distance < DISTANCE_TOLERANCE) {
        *status = 2;
        return 0.0;
    }
    const DevObject& o = P.obj[oid];
    double image[3], bp[3], nrm[3], travelled;
    reflect_against_boundary(o, cp, image, bp, nrm, travelled);
    int cells[8];
    const int nc = enclosing_neighbours(P, image, cells);
    double A[8 * 4], b[8];
    int kept[8];
    int nk = 0;
    for (int q = 0; q < nc; ++q) {
        const int n = cells[q];
        if (!(P.cls[n] & CLS_VALID)) continue;
        int ni, nj, nn;
        cell_ijk(P, n, ni, nj, nn);
        const double np_[3] = {P.cpos[0][ni], P.cpos[1][nj], P.cpos[2][nn]};
        mls_row(image, np_, val(n), &A[nk * 4], b[nk]);
        kept[nk++] = n;
    }
    if (nk < 4) {
        if (nk != 0) {
            double md = DBL_MAX;
            int mid = -1;
            for (int q = 0; q < nk; ++q) {
                const int n = kept[q];
                int ni, nj, nn;
                cell_ijk(P, n, ni, nj, nn);
                const double dx = image[0] - P.cpos[0][ni], dy = image[1] - P.cpos[1][nj], dz = image[2] - P.cpos[2][nn];
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 < md) { md = d2; mid = n; }
            }
            return val(mid);
        }
        const int idx[3] = {i, j, k};
        const long long strides[3] = {P.SX, P.SY, 1};
        for (int d = 0; d < 3; ++d)
            for (int s = 1; s >= -1; s -= 2) {
                if (idx[d] + s < 0 || idx[d] + s >= P.N[d]) continue;
                const long long n = c + s * strides[d];
                if (P.cls[n] & CLS_BULK) return val(n);
            }
        return 0.0;
    }
    double c0 = 0.0;
    if (!householder_ls4(A, b, nk, c0)) c0 = 0.0;
    double acc[3];
    boundary_accel(o, bp, t, acc);
    const double an = acc[0] * nrm[0] + acc[1] * nrm[1] + acc[2] * nrm[2];
    return c0 + P.rho * an * fabs(travelled);
}

template <typename T>
__global__ void k_fresh_cells(const SolveParams* __restrict__ Pp, int cur, long long n, int* status) {
    const SolveParams& P = *Pp;
    const double t = P.consts[cur].t;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        dense_ijk(P, q, i, j, k);
        const long long c = cidx(P, i, j, k);
        const uint8_t code = P.cls[c];
        if (!(code & CLS_BULK) || (code & CLS_VALID)) continue;
        int st = 0;
        if (sizeof(T) == 8) {
            double* pl = (double*)P.p[cur ^ 1];
            double* pc = (double*)P.p[cur];
            const double vl = fresh_value<double>(P, pl, pl, false, c, t, &st);
            const double vc = fresh_value<double>(P, pc, pc, false, c, t, &st);
            pl[c] = vl;
            pc[c] = vc;
        } else {
            // FP32 keeps p^n and the increment; p^{n-1} = p^n - d
            float* pc = (float*)P.p[cur];
            const double vc = fresh_value<float>(P, pc, pc, false, c, t, &st);
            const double vl = fresh_value<float>(P, pc, P.dinc, true, c, t, &st);
            pc[c] = (float)vc;
            P.dinc[c] = (float)(vc - vl);
        }
        if (st) atomicMax(status, st);
    }
}

// ---------------------------------------------------------------------------
// Plain FP64 path: one kernel per reference phase over full-grid arrays, as
// PML_WaveSolver::stepCollocated sequences them (PML_WaveSolver.cpp:800-823).
// ---------------------------------------------------------------------------
__global__ void k_phase_velocity(const SolveParams* __restrict__ Pp, int cur, int dim) {
    const SolveParams& P = *Pp;
    const int* vN = P.vN[dim];
    const long long total = (long long)vN[0] * vN[1] * vN[2];
    const double* p = (const double*)P.p[cur];
    double* v = (double*)P.v[0][dim];
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total; f += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(f / ((long long)vN[1] * vN[2]));
        const int j = (int)((f / vN[2]) % vN[1]);
        const int k = (int)(f % vN[2]);
        int a[3] = {i, j, k};
        if (a[dim] == 0 || a[dim] == vN[dim] - 1) continue;
        bool inpml = P.pml_face[dim][a[dim]] != 0;
        for (int d = 0; d < 3; ++d)
            if (d != dim) inpml = inpml || P.pml_cell[d][a[d]] != 0;
        if (!inpml) continue;
        const long long pr = cidx(P, a[0], a[1], a[2]);  // also the face index
        const long long pl = pr - (dim == 0 ? P.SX : (dim == 1 ? P.SY : 1));
        v[pr] = vel_update<double>(v[pr], P.vupd[dim][a[dim]], P.vgrad[dim][a[dim]], p[pr], p[pl]);
    }
}

__global__ void k_phase_laplacian(const SolveParams* __restrict__ Pp, int cur, double* __restrict__ lap) {
    const SolveParams& P = *Pp;
    const double* p = (const double*)P.p[cur];
    const double t = P.consts[cur].t;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.ncell; q += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        dense_ijk(P, q, idx[0], idx[1], idx[2]);
        const long long c = cidx(P, idx[0], idx[1], idx[2]);
        const uint8_t code = P.cls[c];
        if (!(code & CLS_BULK)) { lap[c] = 0.0; continue; }
        const long long strides[3] = {P.SX, P.SY, 1};
        const unsigned mask = code & CLS_MASK;
        double L = 0.0;
        int surrounded = 0;
        const double p0 = p[c];
        for (int d = 0; d < 3; ++d) {
            const double pp = idx[d] + 1 < P.N[d] ? p[c + strides[d]] : p0;
            const double pm = idx[d] > 0 ? p[c - strides[d]] : p0;
            const bool gn = (mask >> (2 * d)) & 1u, gp = (mask >> (2 * d + 1)) & 1u;
            double own[3] = {P.cpos[0][idx[0]], P.cpos[1][idx[1]], P.cpos[2][idx[2]]};
            double gpv = 0, gnv = 0;
            if (gp) {
                own[d] = P.cpos[d][idx[d] + 1];
                gpv = ghost_pressure(P, P.gobj[c + strides[d]], own, d, -1, p0, t);
            }
            if (gn) {
                own[d] = P.cpos[d][idx[d] - 1];
                gnv = ghost_pressure(P, P.gobj[c - strides[d]], own, d, +1, p0, t);
            }
            if (gp && gn) {
                L += (gpv + gnv - 2.0 * p0) / (9.0 / 16.0);
                ++surrounded;
            } else if (gp) {
                L += (gpv + 0.75 * pm - (7.0 / 4.0) * p0) / (21.0 / 32.0);
            } else if (gn) {
                L += (0.75 * pp + gnv - (7.0 / 4.0) * p0) / (21.0 / 32.0);
            } else {
                L += (pp + pm - 2.0 * p0);
            }
        }
        L *= P.lap_scale;
        (void)surrounded;  // the pressure phase re-derives the cavity flag from the mask
        lap[c] = L;
    }
}

__global__ void k_phase_pressure(const SolveParams* __restrict__ Pp, int cur, const double* __restrict__ lap) {
    const SolveParams& P = *Pp;
    const double* pc = (const double*)P.p[cur];
    double* pn = (double*)P.p[cur ^ 1];
    const StepConsts sc = P.consts[cur];
    bool any_src = false;
    for (int s = 0; s < P.n_src; ++s) any_src |= (sc.src_tf[s] != 0.0);
    const double* v0 = (const double*)P.v[0][0];
    const double* v1 = (const double*)P.v[0][1];
    const double* v2 = (const double*)P.v[0][2];
    double* pd0 = (double*)P.pd[0];
    double* pd1 = (double*)P.pd[1];
    double* pd2 = (double*)P.pd[2];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P.ncell; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        dense_ijk(P, q, i, j, k);
        const long long c = cidx(P, i, j, k);  // the cell and its three low faces
        const bool pml = P.pml_cell[0][i] || P.pml_cell[1][j] || P.pml_cell[2][k];
        if (pml) {
            const double a = pd_update<double>(pd0[c], P.pupd[0][i], P.pdiv[0][i], v0[c + P.SX], v0[c], P.inv_h);
            const double b = pd_update<double>(pd1[c], P.pupd[1][j], P.pdiv[1][j], v1[c + P.SY], v1[c], P.inv_h);
            const double d = pd_update<double>(pd2[c], P.pupd[2][k], P.pdiv[2][k], v2[c + 1], v2[c], P.inv_h);
            pd0[c] = a;
            pd1[c] = b;
            pd2[c] = d;
            pn[c] = a + b + d;
            continue;
        }
        const uint8_t code = P.cls[c];
        if (!(code & CLS_BULK)) continue;
        const unsigned mask = code & CLS_MASK;
        int surrounded = 0;
        for (int dd = 0; dd < 3; ++dd)
            if (((mask >> (2 * dd)) & 3u) == 3u) ++surrounded;
        double pnext;
        if (surrounded > 1 && (code & CLS_VALID)) pnext = pc[c];
        else if (P.visc && (code & CLS_VALID))  // air viscosity (MAC_Grid.cpp:926-930)
            pnext = 2.0 * pc[c] - pn[c] - ((const double*)P.lapv[cur ^ 1])[c] * P.kcalp + lap[c] * (P.c2k2 + P.kcalp);
        else pnext = 2.0 * pc[c] - pn[c] + lap[c] * P.c2k2;
        if (P.n_src > 0) {
            double src = 0.0;
            if (any_src) src = source_sum(P, sc, P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]);
            pnext += src * P.k;
        }
        pn[c] = pnext;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g > 148LL * 16) g = 148LL * 16;
    if (g < 1) g = 1;
    return (int)g;
}

cudaError_t launch_prologue_fp64(const SolveParams* dP, int cur, int advance, int n_solid_pml, cudaStream_t s) {
    const int blocks = n_solid_pml > 0 ? grid_for(n_solid_pml, 256) : 1;
    k_prologue<double><<<blocks, 256, 0, s>>>(dP, cur, advance);
    return cudaGetLastError();
}

// Spatial factor of each Gaussian source over the source region
// (GaussianPressureSource.cpp:6-30 without the time factor), once per reset:
// the per-step source update is then one multiply-add per source and cell.
__global__ void k_source_factors(const SolveParams* __restrict__ Pp, Box3 r) {
    const SolveParams& P = *Pp;
    const int nx = r.hi[0] - r.lo[0], ny = r.hi[1] - r.lo[1], nz = r.hi[2] - r.lo[2];
    const long long R = (long long)nx * ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < R * P.n_src;
         t += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(t / R);
        const long long q = t - s * R;
        const int z = r.lo[2] + (int)(q % nz);
        const int y = r.lo[1] + (int)((q / nz) % ny);
        const int x = r.lo[0] + (int)(q / ((long long)nz * ny));
        const double px = P.cpos[0][x], py = P.cpos[1][y], pz = P.cpos[2][z];
        const DevSource& S = P.src[s];
        double v = 0.0;
        if (px < S.bmax[0] && px > S.bmin[0] && py < S.bmax[1] && py > S.bmin[1] && pz < S.bmax[2] && pz > S.bmin[2]) {
            v = (px - S.cen[0]) * (px - S.cen[0]) + (py - S.cen[1]) * (py - S.cen[1]) + (pz - S.cen[2]) * (pz - S.cen[2]);
            v = -v / S.denom;
            v = exp(v);
            v *= S.scale;
        }
        P.src_g[t] = v;
    }
}

cudaError_t launch_source_factors(const SolveParams* dP, Box3 region, int n_src, long long cells, cudaStream_t s) {
    if (cells <= 0 || n_src <= 0) return cudaSuccess;
    k_source_factors<<<grid_for(cells * n_src, 256), 256, 0, s>>>(dP, region);
    return cudaGetLastError();
}

cudaError_t launch_consts_init(const SolveParams* dP, double t0, cudaStream_t s) {
    k_consts_init<<<1, 32, 0, s>>>(dP, t0);
    return cudaGetLastError();
}

cudaError_t launch_listeners(const SolveParams* dP, int precision, int newp, int n_lis, double* out_row,
                             cudaStream_t s) {
    if (n_lis <= 0) return cudaSuccess;
    const int warps_per_block = 4;
    const int grid = (n_lis + warps_per_block - 1) / warps_per_block;
    if (precision == 0) k_listeners_warp<double><<<grid, 32 * warps_per_block, 0, s>>>(dP, newp, out_row);
    else k_listeners_warp<float><<<grid, 32 * warps_per_block, 0, s>>>(dP, newp, out_row);
    return cudaGetLastError();
}

// listener fit plans from the current classification (static scenes, once)
__global__ void k_set_lis_ready(SolveParams* __restrict__ Pp) { Pp->lis_ready = 1; }

cudaError_t launch_listener_prep(SolveParams* dP, int precision, int newp, int n_lis, cudaStream_t s) {
    if (n_lis <= 0) return cudaSuccess;
    const int grid = (n_lis + 3) / 4;
    if (precision == 0) k_listener_prep<double><<<grid, 128, 0, s>>>(dP, newp);
    else k_listener_prep<float><<<grid, 128, 0, s>>>(dP, newp);
    k_set_lis_ready<<<1, 1, 0, s>>>(dP);
    return cudaGetLastError();
}

cudaError_t launch_cls_reset(const SolveParams* dP, long long ncell, cudaStream_t s) {
    k_cls_reset<<<grid_for(ncell, 256), 256, 0, s>>>(dP, ncell);
    return cudaGetLastError();
}

cudaError_t launch_cls_solid(const SolveParams* dP, const int start[3], const int range[3], cudaStream_t s) {
    const long long total = (long long)range[0] * range[1] * range[2];
    if (total <= 0) return cudaSuccess;
    k_cls_solid<<<grid_for(total, 128), 128, 0, s>>>(dP, start[0], start[1], start[2], range[0], range[1], range[2]);
    return cudaGetLastError();
}

// ResetCellHistory(true) after the classification of a reset: every cell gets a
// valid history (bit 6).  Also counts the solid cells inside the PML into
// *count and, when `list` is given, writes their padded indices (in no fixed
// order: they are only re-zeroed each step).
__global__ void k_cls_history(const SolveParams* __restrict__ Pp, long long n, int* count, int* list, int cap) {
    const SolveParams& P = *Pp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        dense_ijk(P, t, i, j, k);
        const long long c = cidx(P, i, j, k);
        const uint8_t code = P.cls[c];
        if (!list) P.cls[c] = code | CLS_VALID;
        if (!(code & CLS_BULK) && (P.pml_cell[0][i] || P.pml_cell[1][j] || P.pml_cell[2][k])) {
            const int slot = atomicAdd(count, 1);
            if (list && slot < cap) list[slot] = (int)c;
        }
    }
}

cudaError_t launch_cls_history(const SolveParams* dP, long long ncell, int* count, int* list, int cap, cudaStream_t s) {
    k_cls_history<<<grid_for(ncell, 256), 256, 0, s>>>(dP, ncell, count, list, cap);
    return cudaGetLastError();
}

cudaError_t launch_cls_ghost(const SolveParams* dP, long long ncell, cudaStream_t s) {
    k_cls_ghost<<<grid_for(ncell, 256), 256, 0, s>>>(dP, ncell);
    return cudaGetLastError();
}

cudaError_t launch_fresh_cells(const SolveParams* dP, int precision, int cur, long long ncell, int* d_status,
                               cudaStream_t s) {
    if (precision == 0) k_fresh_cells<double><<<grid_for(ncell, 256), 256, 0, s>>>(dP, cur, ncell, d_status);
    else k_fresh_cells<float><<<grid_for(ncell, 256), 256, 0, s>>>(dP, cur, ncell, d_status);
    return cudaGetLastError();
}

cudaError_t launch_phased_fp64(const SolveParams* dP, const int N[3], int cur, double* lap, cudaStream_t s,
                               int* launches) {
    const long long n = (long long)N[0] * N[1] * N[2];
    for (int d = 0; d < 3; ++d) {
        const long long nf = n + (long long)(d == 0 ? N[1] * N[2] : d == 1 ? N[0] * N[2] : N[0] * N[1]);
        k_phase_velocity<<<grid_for(nf, 256), 256, 0, s>>>(dP, cur, d);
    }
    k_phase_laplacian<<<grid_for(n, 256), 256, 0, s>>>(dP, cur, lap);
    k_phase_pressure<<<grid_for(n, 256), 256, 0, s>>>(dP, cur, lap);
    if (launches) *launches += 5;
    return cudaGetLastError();
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// region-split step, FP64
// ---------------------------------------------------------------------------
#include "fdtd_hot.cuh"
namespace fdtd {
cudaError_t launch_step_regions_fp64(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                                     const StepStreams& S, int* launches) {
    return launch_regions<double>(dP, hP, R, cur, S, launches);
}
}  // namespace fdtd

// ---------------------------------------------------------------------------
// batched step, FP64
// ---------------------------------------------------------------------------
#include "fdtd_batch.cuh"
namespace fdtd {
cudaError_t launch_batch_fp64(const BatchLaunch& L, const StepStreams& S, int* launches) {
    return launch_batch<double>(L, S, launches);
}
cudaError_t launch_batch_tail_any(int precision, const BatchLaunch& L, cudaStream_t s, int* launches) {
    return precision == 0 ? launch_batch_tail<double>(L, s, launches) : launch_batch_tail<float>(L, s, launches);
}
}  // namespace fdtd
