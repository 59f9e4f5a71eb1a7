// fdtd_shell.cuh — the PML shell kernel and the host launcher of a region-split
// step.
//
// The shell is covered by five boxes: the two x slabs (full y-z planes), the two
// y slabs inside the x range, and the pair of z slabs inside the x and y ranges
// merged into one box whose z index jumps from the low slab to the high one, so
// that every warp is full (a 16-cell slab would otherwise leave half a warp idle).
// A CTA of 32 (z) x 8 (y) threads owns one tile of one box and XS consecutive x
// planes; the tile is decoded once per CTA from a prefix table, all offsets are
// 32-bit, and every load of a cell (p^n and its six neighbours, the six face
// velocities of the old buffer, the three split pressures) is issued before its
// arithmetic.
//
// Per PML cell (MAC_Grid.cpp:461-479, :496-508):
//   v_f <- v_f*upd + grad*(p_right - p_left)   for the owned faces (left faces,
//          and the right face when the right neighbour is not a PML cell)
//   p_d <- p_d*upd_d + div_d*(v_d(right) - v_d(left))/h,  p^{n+1} = p_x+p_y+p_z
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_region.cuh"
#include "fdtd_stencil.cuh"

namespace fdtd {

template <typename T, int XS>
__global__ void __launch_bounds__(256) k_pml_shell(const SolveParams* __restrict__ Pp, int cur, ShellBoxes B) {
    const SolveParams& P = *Pp;
    // ---- CTA -> (box, tile) ----
    const int blk = blockIdx.x;
    int b = 0;
#pragma unroll
    for (int q = 1; q < 5; ++q)
        if (q < B.n && blk >= B.block_first[q]) b = q;
    int local = blk - B.block_first[b];
    const int tz = local % B.tz[b];
    local /= B.tz[b];
    const int ty = local % B.ty[b];
    const int tx = local / B.ty[b];
    const int zz = tz * 32 + threadIdx.x;
    const int yy = ty * 8 + threadIdx.y;
    if (zz >= B.nz[b] || yy >= B.ny[b]) return;
    const int z = zz < B.nza[b] ? B.z0a[b] + zz : B.z0b[b] + (zz - B.nza[b]);
    const int y = B.y0[b] + yy;
    const int xbeg = B.x0[b] + tx * XS;
    const int xend = min(xbeg + XS, B.x0[b] + B.nx[b]);

    const int N0 = P.N[0], N1 = P.N[1], N2 = P.N[2];
    const unsigned sx = (unsigned)N1 * N2;
    const unsigned sy1 = (unsigned)(N1 + 1) * N2;   // x stride of the y-face grid
    const unsigned sz2 = (unsigned)N1 * (N2 + 1);   // x stride of the z-face grid
    const T* __restrict__ pc = (const T*)P.p[cur];
    T* __restrict__ pn = (T*)P.p[cur ^ 1];
    const T* __restrict__ vox = (const T*)P.v[cur][0];
    const T* __restrict__ voy = (const T*)P.v[cur][1];
    const T* __restrict__ voz = (const T*)P.v[cur][2];
    T* __restrict__ vnx = (T*)P.v[cur ^ 1][0];
    T* __restrict__ vny = (T*)P.v[cur ^ 1][1];
    T* __restrict__ vnz = (T*)P.v[cur ^ 1][2];
    T* __restrict__ pdx = (T*)P.pd[0];
    T* __restrict__ pdy = (T*)P.pd[1];
    T* __restrict__ pdz = (T*)P.pd[2];
    const T inv_h = (T)P.inv_h;

    // per-column (y, z) quantities
    const bool pmly = P.pml_cell[1][y] != 0;
    const bool pmlz = P.pml_cell[2][z] != 0;
    const bool pfy_l = y > 0 && P.pml_face[1][y] != 0;
    const bool pfy_r = y + 1 < N1 && P.pml_face[1][y + 1] != 0;
    const bool pfz_l = z > 0 && P.pml_face[2][z] != 0;
    const bool pfz_r = z + 1 < N2 && P.pml_face[2][z + 1] != 0;
    const bool pml_yr = y + 1 < N1 && P.pml_cell[1][y + 1] != 0;
    const bool pml_zr = z + 1 < N2 && P.pml_cell[2][z + 1] != 0;
    const T vupd_y = Coef<T>::vupd(P, 1)[y], vgrad_y = Coef<T>::vgrad(P, 1)[y];
    const T vupd_yr = Coef<T>::vupd(P, 1)[y + 1], vgrad_yr = Coef<T>::vgrad(P, 1)[y + 1];
    const T vupd_z = Coef<T>::vupd(P, 2)[z], vgrad_z = Coef<T>::vgrad(P, 2)[z];
    const T vupd_zr = Coef<T>::vupd(P, 2)[z + 1], vgrad_zr = Coef<T>::vgrad(P, 2)[z + 1];
    const T pupd_y = Coef<T>::pupd(P, 1)[y], pdiv_y = Coef<T>::pdiv(P, 1)[y];
    const T pupd_z = Coef<T>::pupd(P, 2)[z], pdiv_z = Coef<T>::pdiv(P, 2)[z];

#pragma unroll
    for (int i = 0; i < XS; ++i) {
        const int x = xbeg + i;
        if (x >= xend) break;
        const unsigned c = (unsigned)x * sx + (unsigned)y * N2 + z;
        const unsigned fy = (unsigned)x * sy1 + (unsigned)y * N2 + z;
        const unsigned fz = (unsigned)x * sz2 + (unsigned)y * (N2 + 1) + z;
        const bool pmlx = P.pml_cell[0][x] != 0;
        // face predicates: InsidePML at the face position, outer faces excluded
        const bool fxl = x > 0 && (P.pml_face[0][x] != 0 || pmly || pmlz);
        const bool fxr = x + 1 < N0 && (P.pml_face[0][x + 1] != 0 || pmly || pmlz);
        const bool fyl = pfy_l || (y > 0 && (pmlx || pmlz));
        const bool fyr = pfy_r || (y + 1 < N1 && (pmlx || pmlz));
        const bool fzl = pfz_l || (z > 0 && (pmlx || pmly));
        const bool fzr = pfz_r || (z + 1 < N2 && (pmlx || pmly));
        // ---- loads ----
        const T p0 = pc[c];
        const T pxm = fxl ? pc[c - sx] : p0;
        const T pxp = fxr ? pc[c + sx] : p0;
        const T pym = fyl ? pc[c - N2] : p0;
        const T pyp = fyr ? pc[c + N2] : p0;
        const T pzm = fzl ? pc[c - 1] : p0;
        const T pzp = fzr ? pc[c + 1] : p0;
        T vxl = vox[c], vxr = vox[c + sx];
        T vyl = voy[fy], vyr = voy[fy + N2];
        T vzl = voz[fz], vzr = voz[fz + 1];
        const T ax0 = pdx[c], ay0 = pdy[c], az0 = pdz[c];
        // ---- face velocities ----
        if (fxl) {
            vxl = vel_update<T>(vxl, Coef<T>::vupd(P, 0)[x], Coef<T>::vgrad(P, 0)[x], p0, pxm);
            vnx[c] = vxl;
        }
        if (fxr) {
            vxr = vel_update<T>(vxr, Coef<T>::vupd(P, 0)[x + 1], Coef<T>::vgrad(P, 0)[x + 1], pxp, p0);
            if (!(P.pml_cell[0][x + 1] != 0 || pmly || pmlz)) vnx[c + sx] = vxr;
        }
        if (fyl) {
            vyl = vel_update<T>(vyl, vupd_y, vgrad_y, p0, pym);
            vny[fy] = vyl;
        }
        if (fyr) {
            vyr = vel_update<T>(vyr, vupd_yr, vgrad_yr, pyp, p0);
            if (!(pml_yr || pmlx || pmlz)) vny[fy + N2] = vyr;
        }
        if (fzl) {
            vzl = vel_update<T>(vzl, vupd_z, vgrad_z, p0, pzm);
            vnz[fz] = vzl;
        }
        if (fzr) {
            vzr = vel_update<T>(vzr, vupd_zr, vgrad_zr, pzp, p0);
            if (!(pml_zr || pmlx || pmly)) vnz[fz + 1] = vzr;
        }
        // ---- split-field pressures ----
        const T ax = pd_update<T>(ax0, Coef<T>::pupd(P, 0)[x], Coef<T>::pdiv(P, 0)[x], vxr, vxl, inv_h);
        const T ay = pd_update<T>(ay0, pupd_y, pdiv_y, vyr, vyl, inv_h);
        const T az = pd_update<T>(az0, pupd_z, pdiv_z, vzr, vzl, inv_h);
        pdx[c] = ax;
        pdy[c] = ay;
        pdz[c] = az;
        pn[c] = ax + ay + az;
    }
}

// Host side: one region-split step on stream s.
template <typename T>
cudaError_t launch_regions(const SolveParams* dP, const RegionLaunch& R, int cur, cudaStream_t s, int* launches) {
    int l = 0;
    const int nblk = R.shell.block_first[R.shell.n];
    if (nblk > 0) {
        if (R.shell.xs == 2) k_pml_shell<T, 2><<<nblk, dim3(32, 8), 0, s>>>(dP, cur, R.shell);
        else k_pml_shell<T, 1><<<nblk, dim3(32, 8), 0, s>>>(dP, cur, R.shell);
        ++l;
    }
    const Box3& b = R.interior;
    const int nx = b.hi[0] - b.lo[0], ny = b.hi[1] - b.lo[1], nz = b.hi[2] - b.lo[2];
    if (nx > 0 && ny > 0 && nz > 0) {
        dim3 block(32, 8);
        const int xb = (R.xb == 2 || R.xb == 8) ? R.xb : 4;
        dim3 grid((nz + 31) / 32, (ny + 7) / 8, (nx + xb - 1) / xb);
        if (xb == 2) k_interior<T, 2><<<grid, block, 0, s>>>(dP, cur, b);
        else if (xb == 8) k_interior<T, 8><<<grid, block, 0, s>>>(dP, cur, b);
        else k_interior<T, 4><<<grid, block, 0, s>>>(dP, cur, b);
        ++l;
    }
    if (R.ghost_cap > 0) {
        const int blocks = (R.ghost_cap + 127) / 128 < 1184 ? (R.ghost_cap + 127) / 128 : 1184;
        k_ghost_cells<T><<<blocks, 128, 0, s>>>(dP, cur);
        ++l;
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
