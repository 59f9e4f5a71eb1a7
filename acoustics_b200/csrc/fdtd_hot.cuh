// fdtd_hot.cuh — the two bandwidth kernels of a step and their launcher.
//
//   k_interior   non-PML bulk cells without a solid neighbour: 7-point
//                Laplacian and leapfrog (MAC_Grid.cpp:267-287, :921-935).
//                FP64: p^{n+1} = 2p^n - p^{n-1} + (ck)^2 lap, written over p^{n-1}.
//                FP32: d <- d + (ck)^2 lap, p^{n+1} = p^n + d (compensated).
//   k_pml_shell  PML cells: face velocities (MAC_Grid.cpp:461-479) and
//                split-field pressures (MAC_Grid.cpp:496-508).
//
// Both take their pointers and scalars by value (KArgs): the kernels issue no
// loads to fetch parameters.  They touch disjoint cells and read only p^n, so
// the launcher runs them concurrently on two streams; cells next to a solid
// (k_ghost_cells) and active sources (k_sources) follow on the first stream.
//
// Interior mapping: a CTA of 32 (z) x 8 (y) threads, each thread owns XB
// consecutive x planes of one (y, z) column; every load of those planes is
// issued before the arithmetic; z neighbours come from the warp by shuffles.
//
// Shell mapping: five boxes (two x slabs, two y slabs, the merged pair of z
// slabs whose z index jumps from the low slab to the high one so warps stay
// full); a CTA of 32 x 8 threads owns one tile of one box and XS x planes,
// decoded once per CTA from a prefix table; offsets are 32-bit.
// Face ownership: a face is written by the cell to its right, or by its left
// cell when the right one is not a PML cell (the x = W h layer on the low side),
// so the interior kernel never touches velocities.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_region.cuh"
#include "fdtd_stencil.cuh"

#ifndef FDTD_SHELL_MINB
#define FDTD_SHELL_MINB 4
#endif

namespace fdtd {

// One interior tile: 32 z x 8 y columns, XB x planes, starting at tile
// coordinates (tz, ty, tx) of the box.  Every thread of the CTA must call it
// (z neighbours are exchanged by warp shuffles).
template <typename T, int XB>
__device__ __forceinline__ void interior_tile(const KArgs<T>& A, const Box3& box, int tz, int ty, int tx) {
    constexpr bool COMP = sizeof(T) == 4;
    const int lane = threadIdx.x;
    const int z = box.lo[2] + tz * 32 + lane;
    const int y = box.lo[1] + ty * 8 + threadIdx.y;
    const int x0 = box.lo[0] + tx * XB;
    const bool active = (z < box.hi[2]) && (y < box.hi[1]);
    const int zc = min(z, box.hi[2] - 1);
    const int yc = min(y, box.hi[1] - 1);
    const int nx = min(XB, box.hi[0] - x0);
    const int Nz = A.N2;
    const int sx = (int)A.sx;
    const unsigned off = (unsigned)x0 * A.sx + (unsigned)yc * Nz + zc;
    const T* __restrict__ pc = A.pc + off;
    T* __restrict__ pn = A.pn + off;
    float* __restrict__ dinc = A.dinc + off;
    const uint8_t* __restrict__ cls = A.cls + off;

    T pcol[XB + 2];
    T ym[XB], yp[XB], prev[XB];
    uint8_t code[XB];
    pcol[0] = pc[-sx];
#pragma unroll
    for (int i = 0; i < XB + 1; ++i)
        if (i <= nx) pcol[i + 1] = pc[i * sx];
#pragma unroll
    for (int i = 0; i < XB; ++i) {
        if (i < nx) {
            ym[i] = pc[i * sx - Nz];
            yp[i] = pc[i * sx + Nz];
            if constexpr (COMP) prev[i] = (T)dinc[i * sx];
            else prev[i] = pn[i * sx];
            code[i] = cls[i * sx];
        }
    }
#pragma unroll
    for (int i = 0; i < XB; ++i) {
        if (i >= nx) break;
        const T p0 = pcol[i + 1];
        T zm = __shfl_up_sync(0xffffffffu, p0, 1);
        T zp = __shfl_down_sync(0xffffffffu, p0, 1);
        if (lane == 0) zm = pc[i * sx - 1];
        if (lane == 31 || z + 1 >= box.hi[2]) zp = pc[i * sx + 1];
        // solid cells are left untouched; cells next to a solid go to k_ghost_cells
        if (!active || (code[i] & (CLS_BULK | CLS_MASK)) != CLS_BULK) continue;
        T lap = 0.0;
        lap = lap + (pcol[i + 2] + pcol[i] - (T)2.0 * p0);
        lap = lap + (yp[i] + ym[i] - (T)2.0 * p0);
        lap = lap + (zp + zm - (T)2.0 * p0);
        lap = lap * A.lap_scale;
        if constexpr (!COMP) {
            pn[i * sx] = (T)2.0 * p0 - prev[i] + lap * A.c2k2;
        } else {
            const float d = (float)prev[i] + (float)(lap * A.c2k2);
            dinc[i * sx] = d;
            pn[i * sx] = p0 + d;
        }
    }
}

template <typename T, int XB>
__global__ void __launch_bounds__(256) k_interior(const KArgs<T> A, Box3 box) {
    interior_tile<T, XB>(A, box, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One PML-shell tile of box b at tile coordinates (tz, ty, tx).
template <typename T, int XS>
__device__ __forceinline__ void shell_tile(const KArgs<T>& A, const ShellBoxes& B, int b, int tz, int ty, int tx) {
    const int zz = tz * 32 + threadIdx.x;
    const int yy = ty * 8 + threadIdx.y;
    if (zz >= B.nz[b] || yy >= B.ny[b]) return;
    const int z = zz < B.nza[b] ? B.z0a[b] + zz : B.z0b[b] + (zz - B.nza[b]);
    const int y = B.y0[b] + yy;
    const int xbeg = B.x0[b] + tx * XS;
    const int xend = min(xbeg + XS, B.x0[b] + B.nx[b]);
    const int N0 = A.N0, N1 = A.N1, N2 = A.N2;
    const unsigned sy1 = (unsigned)(N1 + 1) * N2;  // x stride of the y-face grid
    const unsigned sz2 = (unsigned)N1 * (N2 + 1);  // x stride of the z-face grid
    const bool pmly = A.pml_cell[1][y] != 0;
    const bool pmlz = A.pml_cell[2][z] != 0;

#pragma unroll
    for (int i = 0; i < XS; ++i) {
        const int x = xbeg + i;
        if (x >= xend) break;
        const unsigned c = (unsigned)x * A.sx + (unsigned)y * N2 + z;
        const unsigned fy = (unsigned)x * sy1 + (unsigned)y * N2 + z;
        const unsigned fz = (unsigned)x * sz2 + (unsigned)y * (N2 + 1) + z;
        const bool pmlx = A.pml_cell[0][x] != 0;
        // faces inside the PML (InsidePML at the face position, MAC_Grid.cpp:2631-2633),
        // outer faces excluded (:2568-2575)
        const bool fxl = x > 0 && (A.pml_face[0][x] != 0 || pmly || pmlz);
        const bool fxr = x + 1 < N0 && (A.pml_face[0][x + 1] != 0 || pmly || pmlz);
        const bool fyl = y > 0 && (A.pml_face[1][y] != 0 || pmlx || pmlz);
        const bool fyr = y + 1 < N1 && (A.pml_face[1][y + 1] != 0 || pmlx || pmlz);
        const bool fzl = z > 0 && (A.pml_face[2][z] != 0 || pmlx || pmly);
        const bool fzr = z + 1 < N2 && (A.pml_face[2][z + 1] != 0 || pmlx || pmly);
        // ---- loads ----
        const T p0 = A.pc[c];
        const T pxm = fxl ? A.pc[c - A.sx] : p0;
        const T pxp = fxr ? A.pc[c + A.sx] : p0;
        const T pym = fyl ? A.pc[c - N2] : p0;
        const T pyp = fyr ? A.pc[c + N2] : p0;
        const T pzm = fzl ? A.pc[c - 1] : p0;
        const T pzp = fzr ? A.pc[c + 1] : p0;
        T vxl = A.vo[0][c], vxr = A.vo[0][c + A.sx];
        T vyl = A.vo[1][fy], vyr = A.vo[1][fy + N2];
        T vzl = A.vo[2][fz], vzr = A.vo[2][fz + 1];
        const T ax0 = A.pd[0][c], ay0 = A.pd[1][c], az0 = A.pd[2][c];
        // ---- face velocities ----
        if (fxl) {
            vxl = vel_update<T>(vxl, A.vupd[0][x], A.vgrad[0][x], p0, pxm);
            A.vn[0][c] = vxl;
        }
        if (fxr) {
            vxr = vel_update<T>(vxr, A.vupd[0][x + 1], A.vgrad[0][x + 1], pxp, p0);
            if (!(A.pml_cell[0][x + 1] != 0 || pmly || pmlz)) A.vn[0][c + A.sx] = vxr;
        }
        if (fyl) {
            vyl = vel_update<T>(vyl, A.vupd[1][y], A.vgrad[1][y], p0, pym);
            A.vn[1][fy] = vyl;
        }
        if (fyr) {
            vyr = vel_update<T>(vyr, A.vupd[1][y + 1], A.vgrad[1][y + 1], pyp, p0);
            if (!(A.pml_cell[1][y + 1] != 0 || pmlx || pmlz)) A.vn[1][fy + N2] = vyr;
        }
        if (fzl) {
            vzl = vel_update<T>(vzl, A.vupd[2][z], A.vgrad[2][z], p0, pzm);
            A.vn[2][fz] = vzl;
        }
        if (fzr) {
            vzr = vel_update<T>(vzr, A.vupd[2][z + 1], A.vgrad[2][z + 1], pzp, p0);
            if (!(A.pml_cell[2][z + 1] != 0 || pmlx || pmly)) A.vn[2][fz + 1] = vzr;
        }
        // ---- split-field pressures ----
        const T ax = pd_update<T>(ax0, A.pupd[0][x], A.pdiv[0][x], vxr, vxl, A.inv_h);
        const T ay = pd_update<T>(ay0, A.pupd[1][y], A.pdiv[1][y], vyr, vyl, A.inv_h);
        const T az = pd_update<T>(az0, A.pupd[2][z], A.pdiv[2][z], vzr, vzl, A.inv_h);
        A.pd[0][c] = ax;
        A.pd[1][c] = ay;
        A.pd[2][c] = az;
        A.pn[c] = ax + ay + az;
    }
}

// CTA -> (box, tile) through the prefix table of the shell boxes
__device__ __forceinline__ void shell_decode(const ShellBoxes& B, int blk, int& b, int& tz, int& ty, int& tx) {
    b = 0;
#pragma unroll
    for (int q = 1; q < 5; ++q)
        if (q < B.n && blk >= B.block_first[q]) b = q;
    int local = blk - B.block_first[b];
    tz = local % B.tz[b];
    local /= B.tz[b];
    ty = local % B.ty[b];
    tx = local / B.ty[b];
}

template <typename T, int XS>
__global__ void __launch_bounds__(256, FDTD_SHELL_MINB) k_pml_shell(const KArgs<T> A, const ShellBoxes B) {
    if (A.advance && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) advance_consts(*A.P, A.cur);
    int b, tz, ty, tx;
    shell_decode(B, blockIdx.x, b, tz, ty, tx);
    shell_tile<T, XS>(A, B, b, tz, ty, tx);
}

// Host side: one region-split step.  The shell kernel runs on s, the interior
// kernel on s2 (forked and joined with the two events), then the ghost-cell
// list and the sources on s.
template <typename T>
cudaError_t launch_regions(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                           cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join, int* launches) {
    int l = 0;
    const KArgs<T> A = make_kargs<T>(const_cast<SolveParams*>(dP), hP, cur);
    const Box3& b = R.interior;
    const int nx = b.hi[0] - b.lo[0], ny = b.hi[1] - b.lo[1], nz = b.hi[2] - b.lo[2];
    const bool has_interior = nx > 0 && ny > 0 && nz > 0;
    const bool concurrent = has_interior && s2 != nullptr;
    cudaError_t e = cudaSuccess;
    if (concurrent) {
        e = cudaEventRecord(fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
        if (e != cudaSuccess) return e;
    }
    if (has_interior) {
        cudaStream_t si = concurrent ? s2 : s;
        dim3 block(32, 8);
        const int xb = (R.xb == 2 || R.xb == 8) ? R.xb : 4;
        dim3 grid((nz + 31) / 32, (ny + 7) / 8, (nx + xb - 1) / xb);
        if (xb == 2) k_interior<T, 2><<<grid, block, 0, si>>>(A, b);
        else if (xb == 8) k_interior<T, 8><<<grid, block, 0, si>>>(A, b);
        else k_interior<T, 4><<<grid, block, 0, si>>>(A, b);
        ++l;
    }
    const int nblk = R.shell.block_first[R.shell.n];
    if (nblk > 0) {
        if (R.shell.xs == 2) k_pml_shell<T, 2><<<nblk, dim3(32, 8), 0, s>>>(A, R.shell);
        else k_pml_shell<T, 1><<<nblk, dim3(32, 8), 0, s>>>(A, R.shell);
        ++l;
    }
    if (R.ghost_cap > 0) {
        // cells next to a solid: disjoint from the interior and shell cells
        const int blocks = (R.ghost_cap + 127) / 128 < 1184 ? (R.ghost_cap + 127) / 128 : 1184;
        k_ghost_cells<T><<<blocks, 128, 0, concurrent ? s2 : s>>>(dP, cur);
        ++l;
    }
    if (concurrent) {
        e = cudaEventRecord(join, s2);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
        if (e != cudaSuccess) return e;
    }
    if (R.sources) {
        const Box3& r = R.src_region;
        const long long total = (long long)(r.hi[0] - r.lo[0]) * (r.hi[1] - r.lo[1]) * (r.hi[2] - r.lo[2]);
        if (total > 0) {
            const long long g = (total + 255) / 256;
            k_sources<T><<<(unsigned)(g < 148 * 16 ? g : 148 * 16), 256, 0, s>>>(dP, cur, r);
            ++l;
        }
    }
    if (launches) *launches += l;
    return cudaGetLastError();
}

}  // namespace fdtd
