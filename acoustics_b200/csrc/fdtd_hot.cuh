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

// resident CTAs of 256 threads the shell kernels are compiled for (register
// budget per thread): FP32 64 / 80 / 128, FP64 80 / 128 / 255 for 1 / 2 / 4 x planes
__host__ __device__ constexpr int shell_min_blocks(int xs, int word) {
    return word == 4 ? (xs == 1 ? 4 : (xs == 2 ? 3 : 2)) : (xs == 1 ? 3 : (xs == 2 ? 2 : 1));
}

namespace fdtd {

// 16-byte vector of T (4 floats or 2 doubles) for aligned z-vector accesses
template <typename T>
struct alignas(16) Vec16 {
    T e[16 / sizeof(T)];
};
template <typename T>
__device__ __forceinline__ Vec16<T> ldv(const T* p) {
    return *reinterpret_cast<const Vec16<T>*>(p);
}
template <typename T>
__device__ __forceinline__ void stv(T* p, const Vec16<T>& v) {
    *reinterpret_cast<Vec16<T>*>(p) = v;
}

// One interior tile: 32 z-vector groups (128 FP32 / 64 FP64 cells) x 8 y rows
// x XB x planes, at tile coordinates (tz, ty, tx) of the box.  Every access is
// a 16-byte vector load or store (classification bytes: one 4- or 2-byte
// word), z neighbours across vectors come from the adjacent lane by shuffles
// and at the strip edges from memory.  Cells of a group outside the box or not
// plain bulk are masked (scalar stores for partial groups).  Every thread of
// the CTA must call it.
template <typename T, int XB>
__device__ __forceinline__ void interior_tile(const KArgs<T>& A, const Box3& box, int tz, int ty, int tx) {
    constexpr bool COMP = sizeof(T) == 4;
    constexpr int V = 16 / (int)sizeof(T);
    using VT = Vec16<T>;
    const int lane = threadIdx.x;
    const int zg0 = box.lo[2] / V * V;
    const int zlast = (box.hi[2] - 1) / V * V;
    const int zv = zg0 + (tz * 32 + lane) * V;
    const int y = box.lo[1] + ty * 8 + threadIdx.y;
    const int x0 = box.lo[0] + tx * XB;
    const bool lane_on = (zv <= zlast) && (y < box.hi[1]);
    const int zc = min(zv, zlast);  // inactive lanes shadow a valid group for the shuffles
    const int yc = min(y, box.hi[1] - 1);
    const int nx = min(XB, box.hi[0] - x0);
    // signed strides: offsets below are formed relative to the tile's first cell
    // and may be negative (pc[i*sx - 1] at i = 0)
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned off = (unsigned)x0 * A.sx + (unsigned)yc * A.sy + zc;
    const T* __restrict__ pc = A.pc + off;
    T* __restrict__ pn = A.pn + off;
    float* __restrict__ dinc = A.dinc + off;
    const uint8_t* __restrict__ cls = A.cls + off;
    // the z+V neighbour comes from memory where the next lane does not hold it
    const bool zp_mem = (lane == 31) || (zv + V > zlast);

    VT pcol[XB + 2], ym[XB], yp[XB], prev[XB];
    uint32_t code[XB];
    T zme[XB], zpe[XB];
    pcol[0] = ldv(pc - sx);
#pragma unroll
    for (int i = 0; i < XB + 1; ++i)
        if (i <= nx) pcol[i + 1] = ldv(pc + i * sx);
#pragma unroll
    for (int i = 0; i < XB; ++i) {
        if (i < nx) {
            ym[i] = ldv(pc + i * sx - sy);
            yp[i] = ldv(pc + i * sx + sy);
            if constexpr (COMP) {
                const Vec16<float> d = ldv(dinc + i * sx);
#pragma unroll
                for (int e = 0; e < V; ++e) prev[i].e[e] = d.e[e];
            } else {
                prev[i] = ldv(pn + i * sx);
            }
            if constexpr (V == 4) code[i] = *reinterpret_cast<const uint32_t*>(cls + i * sx);
            else code[i] = *reinterpret_cast<const uint16_t*>(cls + i * sx);
            zme[i] = (lane == 0) ? pc[i * sx - 1] : (T)0;
            zpe[i] = zp_mem ? pc[i * sx + V] : (T)0;
        }
    }
#pragma unroll
    for (int i = 0; i < XB; ++i) {
        if (i >= nx) break;
        const VT& c0 = pcol[i + 1];
        const T left = __shfl_up_sync(0xffffffffu, c0.e[V - 1], 1);
        const T right = __shfl_down_sync(0xffffffffu, c0.e[0], 1);
        const T zm_edge = lane == 0 ? zme[i] : left;
        const T zp_edge = zp_mem ? zpe[i] : right;
        VT outp, outd;
        unsigned act = 0;
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const T p0 = c0.e[e];
            const T zm = e > 0 ? c0.e[e - 1] : zm_edge;
            const T zp = e < V - 1 ? c0.e[e + 1] : zp_edge;
            const int z = zc + e;
            const uint8_t cb = (uint8_t)(code[i] >> (8 * e));
            // solid cells are left untouched; cells next to a solid go to k_ghost_cells
            const bool on = lane_on && z >= box.lo[2] && z < box.hi[2] && (cb & (CLS_BULK | CLS_MASK)) == CLS_BULK;
            act |= (on ? 1u : 0u) << e;
            T lap = 0.0;
            lap = lap + (pcol[i + 2].e[e] + pcol[i].e[e] - (T)2.0 * p0);
            lap = lap + (yp[i].e[e] + ym[i].e[e] - (T)2.0 * p0);
            lap = lap + (zp + zm - (T)2.0 * p0);
            lap = lap * A.lap_scale;
            if constexpr (!COMP) {
                outp.e[e] = (T)2.0 * p0 - prev[i].e[e] + lap * A.c2k2;
            } else {
                const float d = fmaf(lap, A.c2k2, prev[i].e[e]);
                outd.e[e] = d;
                outp.e[e] = p0 + d;
            }
        }
        if (act == (1u << V) - 1u) {
            stv(pn + i * sx, outp);
            if constexpr (COMP) stv(dinc + i * sx, outd);
        } else if (act) {
#pragma unroll
            for (int e = 0; e < V; ++e)
                if ((act >> e) & 1u) {
                    pn[i * sx + e] = outp.e[e];
                    if constexpr (COMP) dinc[i * sx + e] = outd.e[e];
                }
        }
    }
}

template <typename T, int XB>
__global__ void __launch_bounds__(256) k_interior(const KArgs<T> A, Box3 box) {
    interior_tile<T, XB>(A, box, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One PML-shell tile of box b at tile coordinates (tz, ty, tx): XS x planes of
// one (y, z) column per thread.  Every global load of the XS planes (pressure
// and its six neighbours, six face velocities, three split pressures) is
// issued before the first use, with neighbour offsets clamped at the domain
// edge instead of branched on, so a thread keeps ~13*XS independent loads in
// flight; the face flags and coefficients come from the packed per-axis
// tables (L1-resident).  Arithmetic order per cell is unchanged.
template <typename T, int XS>
__device__ __forceinline__ void shell_tile(const KArgs<T>& A, const ShellBoxes& B, int b, int tz, int ty, int tx) {
    const int zz = tz * 32 + threadIdx.x;
    const int yy = ty * 8 + threadIdx.y;
    if (zz >= B.nz[b] || yy >= B.ny[b]) return;
    const int z = zz < B.nza[b] ? B.z0a[b] + zz : B.z0b[b] + (zz - B.nza[b]);
    const int y = B.y0[b] + yy;
    const int xbeg = B.x0[b] + tx * XS;
    const int nxh = min(XS, B.x0[b] + B.nx[b] - xbeg);
    const unsigned sx = A.sx, sy = A.sy;
    const unsigned c0 = (unsigned)xbeg * sx + (unsigned)y * sy + z;  // cell and its three low faces
    const uint8_t gy = __ldg(A.axflag[1] + y), gz = __ldg(A.axflag[2] + z);
    const bool pmly = gy & AXF_PML, pmlz = gz & AXF_PML;
    const unsigned oym = (gy & AXF_HAS_LO) ? sy : 0u, oyp = (gy & AXF_HAS_HI) ? sy : 0u;
    const unsigned ozm = (gz & AXF_HAS_LO) ? 1u : 0u, ozp = (gz & AXF_HAS_HI) ? 1u : 0u;

    // ---- loads of all XS planes ----
    T p0v[XS], xm[XS], xp[XS], ym[XS], yp[XS], zm[XS], zp[XS];
    T vxl[XS], vxr[XS], vyl[XS], vyr[XS], vzl[XS], vzr[XS], a0[XS], a1[XS], a2[XS];
    uint8_t gx[XS];
#pragma unroll
    for (int i = 0; i < XS; ++i) {
        if (i < nxh) {
            const int x = xbeg + i;
            const unsigned c = c0 + i * sx;
            gx[i] = __ldg(A.axflag[0] + x);
            p0v[i] = A.pc[c];
            xm[i] = A.pc[c - (x > 0 ? sx : 0u)];
            xp[i] = A.pc[c + (x + 1 < A.N0 ? sx : 0u)];
            ym[i] = A.pc[c - oym];
            yp[i] = A.pc[c + oyp];
            zm[i] = A.pc[c - ozm];
            zp[i] = A.pc[c + ozp];
            vxl[i] = A.vo[0][c];
            vxr[i] = A.vo[0][c + sx];
            vyl[i] = A.vo[1][c];
            vyr[i] = A.vo[1][c + sy];
            vzl[i] = A.vo[2][c];
            vzr[i] = A.vo[2][c + 1];
            a0[i] = A.pd[0][c];
            a1[i] = A.pd[1][c];
            a2[i] = A.pd[2][c];
        }
    }
    const AxisCoef<T> cyl = A.coef[1][y], cyr = A.coef[1][y + 1];
    const AxisCoef<T> czl = A.coef[2][z], czr = A.coef[2][z + 1];

    // ---- face velocities, split pressures, pressure ----
#pragma unroll
    for (int i = 0; i < XS; ++i) {
        if (i >= nxh) break;
        const int x = xbeg + i;
        const unsigned c = c0 + i * sx;
        const uint8_t g = gx[i];
        const bool pmlx = g & AXF_PML;
        // faces inside the PML (InsidePML at the face position, MAC_Grid.cpp:2631-2633),
        // outer faces excluded (:2568-2575); a high face is written here only when the
        // cell beyond it is not a PML cell
        const bool oyz = pmly || pmlz, oxz = pmlx || pmlz, oxy = pmlx || pmly;
        const bool fxl = (g & AXF_FACE_LO) || ((g & AXF_HAS_LO) && oyz);
        const bool fxr = (g & AXF_FACE_HI) || ((g & AXF_HAS_HI) && oyz);
        const bool fyl = (gy & AXF_FACE_LO) || ((gy & AXF_HAS_LO) && oxz);
        const bool fyr = (gy & AXF_FACE_HI) || ((gy & AXF_HAS_HI) && oxz);
        const bool fzl = (gz & AXF_FACE_LO) || ((gz & AXF_HAS_LO) && oxy);
        const bool fzr = (gz & AXF_FACE_HI) || ((gz & AXF_HAS_HI) && oxy);
        const T p0 = p0v[i];
        T vxl_ = vxl[i], vxr_ = vxr[i];
        T vyl_ = vyl[i], vyr_ = vyr[i], vzl_ = vzl[i], vzr_ = vzr[i];
        const AxisCoef<T> cxl = A.coef[0][x], cxr = A.coef[0][x + 1];
        if (fxl) {
            vxl_ = vel_update<T>(vxl_, cxl.vupd, cxl.vgrad, p0, xm[i]);
            A.vn[0][c] = vxl_;
        }
        if (fxr) {
            vxr_ = vel_update<T>(vxr_, cxr.vupd, cxr.vgrad, xp[i], p0);
            if (!((g & AXF_NEXT_PML) || oyz)) A.vn[0][c + sx] = vxr_;
        }
        if (fyl) {
            vyl_ = vel_update<T>(vyl_, cyl.vupd, cyl.vgrad, p0, ym[i]);
            A.vn[1][c] = vyl_;
        }
        if (fyr) {
            vyr_ = vel_update<T>(vyr_, cyr.vupd, cyr.vgrad, yp[i], p0);
            if (!((gy & AXF_NEXT_PML) || oxz)) A.vn[1][c + sy] = vyr_;
        }
        if (fzl) {
            vzl_ = vel_update<T>(vzl_, czl.vupd, czl.vgrad, p0, zm[i]);
            A.vn[2][c] = vzl_;
        }
        if (fzr) {
            vzr_ = vel_update<T>(vzr_, czr.vupd, czr.vgrad, zp[i], p0);
            if (!((gz & AXF_NEXT_PML) || oxy)) A.vn[2][c + 1] = vzr_;
        }
        const T ax = pd_update<T>(a0[i], cxl.pupd, cxl.pdiv, vxr_, vxl_, A.inv_h);
        const T ay = pd_update<T>(a1[i], cyl.pupd, cyl.pdiv, vyr_, vyl_, A.inv_h);
        const T az = pd_update<T>(a2[i], czl.pupd, czl.pdiv, vzr_, vzl_, A.inv_h);
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
__global__ void __launch_bounds__(256, shell_min_blocks(XS, sizeof(T))) k_pml_shell(const KArgs<T> A, const ShellBoxes B) {
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
    const bool has_interior = nx > 0 && ny > 0 && nz > 0 && !(R.skip & 1);
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
        const int xb = (R.xb == 4 || R.xb == 8) ? R.xb : 2;
        dim3 grid(interior_strips_z(b, 16 / (int)sizeof(T)), (ny + 7) / 8, (nx + xb - 1) / xb);
        if (xb == 2) k_interior<T, 2><<<grid, block, 0, si>>>(A, b);
        else if (xb == 8) k_interior<T, 8><<<grid, block, 0, si>>>(A, b);
        else k_interior<T, 4><<<grid, block, 0, si>>>(A, b);
        ++l;
    }
    const int nblk = (R.skip & 2) ? 0 : R.shell.block_first[R.shell.n];
    if (nblk > 0) {
        if (R.shell.xs == 2) k_pml_shell<T, 2><<<nblk, dim3(32, 8), 0, s>>>(A, R.shell);
        else if (R.shell.xs == 4) k_pml_shell<T, 4><<<nblk, dim3(32, 8), 0, s>>>(A, R.shell);
        else k_pml_shell<T, 1><<<nblk, dim3(32, 8), 0, s>>>(A, R.shell);
        ++l;
    }
    if (R.ghost_cap > 0 && !(R.skip & 4)) {
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
