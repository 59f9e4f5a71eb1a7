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
// Interior mapping: a CTA of 256 threads owns 256 consecutive (row, z-group)
// units of the non-PML box, each thread XB consecutive x planes of its unit;
// every load of those planes is issued before the arithmetic; z neighbours come
// from the warp by shuffles.
//
// Shell mapping: five boxes (two x slabs, two y slabs, the merged pair of z
// slabs); a thread owns one z-vector group of one row and marches along x; a
// CTA of 256 threads owns 256 consecutive (row, group) units of one box, decoded
// once per CTA from a prefix table; offsets are 32-bit.
// Face ownership: a face is written by the cell to its right, or by its left
// cell when the right one is not a PML cell (the x = W h layer on the low side),
// so the interior kernel never touches velocities.
#pragma once
#include <algorithm>

#include "fdtd_device.cuh"
#include "fdtd_region.cuh"
#include "fdtd_stencil.cuh"

// resident CTAs of 256 threads the shell kernels are compiled for: 2 (128
// registers per thread) in FP32, 1 (255) in FP64 by default
#ifndef FDTD_SHELL_MINB_F32
#define FDTD_SHELL_MINB_F32 2
#endif
#ifndef FDTD_SHELL_MINB_F64
#define FDTD_SHELL_MINB_F64 1
#endif
// 1: a shell thread issues the loads of its next x plane before computing the
// current one (two planes of registers); 0: one plane at a time, more warps
#ifndef FDTD_SHELL_PREFETCH
#define FDTD_SHELL_PREFETCH 1
#endif
__host__ __device__ constexpr int shell_min_blocks(int word) {
    return word == 4 ? FDTD_SHELL_MINB_F32 : FDTD_SHELL_MINB_F64;
}

namespace fdtd {

// Vector of V consecutive z cells (aligned to its size) for z-vector accesses;
// Vec16<T> is the 16-byte one (4 floats or 2 doubles)
template <typename T, int V>
struct alignas(sizeof(T) * V) Vec {
    T e[V];
};
template <typename T>
using Vec16 = Vec<T, 16 / sizeof(T)>;
template <typename T, int V = 16 / sizeof(T)>
__device__ __forceinline__ Vec<T, V> ldv(const T* p) {
    return *reinterpret_cast<const Vec<T, V>*>(p);
}
template <typename T, int V>
__device__ __forceinline__ void stv(T* p, const Vec<T, V>& v) {
    *reinterpret_cast<Vec<T, V>*>(p) = v;
}

// One interior tile: 256 consecutive (row, z-group) units of the box (one per
// thread; a z group is a 16-byte vector of V = 4 FP32 / 2 FP64 cells starting
// at a multiple of V) x XB x planes, at unit tile tu and plane tile tx.  Units
// are packed densely across rows, so narrow boxes leave no lane idle.  Every
// access is a 16-byte vector load or store (classification bytes: one 4- or
// 2-byte word); the z neighbour across vectors comes from the adjacent lane by a
// shuffle when that lane holds the neighbouring group of the same row, else
// from memory.  Cells of a group outside the box or not plain bulk are masked
// (scalar stores for partial groups).  Every thread of the CTA must call it.
template <typename T, int XB, bool VISC = false, typename AT = KArgs<T>>
__device__ __forceinline__ void interior_tile(const AT& A, const Box3& box, int tu, int tx) {
    constexpr bool COMP = sizeof(T) == 4;
    constexpr int V = 16 / (int)sizeof(T);
    using VT = Vec16<T>;
    const int lane = threadIdx.x;
    const int ng = interior_groups_z(box, V);
    const int ny = box.hi[1] - box.lo[1];
    const int u = tu * 256 + threadIdx.x + 32 * threadIdx.y;
    int row = u / ng, g = u - row * ng;
    const bool lane_on = row < ny;
    if (!lane_on) {  // inactive lanes shadow the box's last unit for the shuffles
        row = ny - 1;
        g = ng - 1;
    }
    const int zc = box.lo[2] / V * V + g * V;
    const int yc = box.lo[1] + row;
    const int x0 = box.lo[0] + tx * XB;
    const int nx = min(XB, box.hi[0] - x0);
    // signed strides: offsets below are formed relative to the tile's first cell
    // and may be negative (pc[i*sx - 1] at i = 0)
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned off = (unsigned)x0 * A.sx + (unsigned)yc * A.sy + zc;
    const T* __restrict__ pc = A.pc + off;
    T* __restrict__ pn = A.pn + off;
    float* __restrict__ dinc = A.dinc + off;
    const uint8_t* __restrict__ cls = A.cls + off;
    // z neighbours from memory where the adjacent lane does not hold them
    const bool zm_mem = (lane == 0) || (g == 0);
    const bool zp_mem = (lane == 31) || (g == ng - 1);

    VT pcol[XB + 2], ym[XB], yp[XB], prev[XB], lapl[XB];
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
            if constexpr (VISC) lapl[i] = ldv(A.lapl + off + i * sx);
            zme[i] = zm_mem ? pc[i * sx - 1] : (T)0;
            zpe[i] = zp_mem ? pc[i * sx + V] : (T)0;
        }
    }
#pragma unroll
    for (int i = 0; i < XB; ++i) {
        if (i >= nx) break;
        const VT& c0 = pcol[i + 1];
        const T left = __shfl_up_sync(0xffffffffu, c0.e[V - 1], 1);
        const T right = __shfl_down_sync(0xffffffffu, c0.e[0], 1);
        const T zm_edge = zm_mem ? zme[i] : left;
        const T zp_edge = zp_mem ? zpe[i] : right;
        VT outp, outd, outl;
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
            // air viscosity on cells with a valid history (MAC_Grid.cpp:926-930)
            const bool visc = VISC && (cb & CLS_VALID);
            if constexpr (!COMP) {
                if (visc) outp.e[e] = (T)2.0 * p0 - prev[i].e[e] - lapl[i].e[e] * A.kcalp + lap * (A.c2k2 + A.kcalp);
                else outp.e[e] = (T)2.0 * p0 - prev[i].e[e] + lap * A.c2k2;
            } else {
                float d = fmaf(lap, A.c2k2, prev[i].e[e]);
                if (visc) d = fmaf(A.kcalp, lap - lapl[i].e[e], d);
                outd.e[e] = d;
                outp.e[e] = p0 + d;
            }
            outl.e[e] = lap;
        }
        if (act == (1u << V) - 1u) {
            stv(pn + i * sx, outp);
            if constexpr (COMP) stv(dinc + i * sx, outd);
            if constexpr (VISC) stv(A.lapc + off + i * sx, outl);
        } else if (act) {
#pragma unroll
            for (int e = 0; e < V; ++e)
                if ((act >> e) & 1u) {
                    pn[i * sx + e] = outp.e[e];
                    if constexpr (COMP) dinc[i * sx + e] = outd.e[e];
                    if constexpr (VISC) A.lapc[off + i * sx + e] = outl.e[e];
                }
        }
    }
}

template <typename T, int XB, bool VISC = false>
__global__ void __launch_bounds__(256) k_interior(const KArgs<T> A, Box3 box) {
    interior_tile<T, XB, VISC>(A, box, blockIdx.x, blockIdx.y);
}

// Masked store of a z vector: one vector store when every cell is selected,
// else the selected cells one by one.
template <typename T, int V>
__device__ __forceinline__ void st_masked(T* p, const Vec<T, V>& v, unsigned m) {
    if (m == (1u << V) - 1u) {
        stv(p, v);
    } else if (m) {
#pragma unroll
        for (int e = 0; e < V; ++e)
            if ((m >> e) & 1u) p[e] = v.e[e];
    }
}

// V-bit mask of bit k of each of V flag bytes
template <int V>
__device__ __forceinline__ unsigned flag_mask(const uint8_t (&f)[V], int k) {
    unsigned m = 0;
#pragma unroll
    for (int e = 0; e < V; ++e) m |= ((f[e] >> k) & 1u) << e;
    return m;
}

// Where a shell column keeps its split pressures and face velocities: the grid
// arrays (CMP = false: offsets equal the cell offsets, strides the grid's), or
// the compact arrays of the z-slab box (CMP = true, ShellBoxes).  The choice is
// a template parameter, so the array pointers stay kernel parameters instead of
// registers.
template <typename T, bool CMP>
__device__ __forceinline__ T* sh_pd(const KArgs<T>& A, int d) {
    return CMP ? A.zpd[d] : A.pd[d];
}
template <typename T, bool CMP>
__device__ __forceinline__ const T* sh_vo(const KArgs<T>& A, int d) {
    return CMP ? A.zvo[d] : A.vo[d];
}
template <typename T, bool CMP>
__device__ __forceinline__ T* sh_vn(const KArgs<T>& A, int d) {
    return CMP ? A.zvn[d] : A.vn[d];
}

// Per-thread asynchronous copies (cp.async) into shared memory, for the rings
// of staged shell loads: a thread reads back only what it copied, so no barrier.
__device__ __forceinline__ int threadIdx_lin() { return threadIdx.x + 32 * threadIdx.y; }
template <int BYTES>
__device__ __forceinline__ void cpa(unsigned saddr, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(saddr), "l"(g), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// x planes of the full-state shell whose loads a thread keeps in flight through
// a shared-memory ring; 0: the register prefetch of FDTD_SHELL_PREFETCH.
#ifndef FDTD_SHELL_F64_STAGES
#define FDTD_SHELL_F64_STAGES 3
#endif
#ifndef FDTD_SHELL_F32_STAGES
#define FDTD_SHELL_F32_STAGES 0
#endif
template <typename T>
__host__ __device__ constexpr int shell_full_stages() {
    return sizeof(T) == 8 ? FDTD_SHELL_F64_STAGES : FDTD_SHELL_F32_STAGES;
}
// one stage: ten vector fields and three scalar fields, each over the CTA's 256 threads
template <typename T>
__host__ __device__ constexpr int shell_stage_bytes() {
    return 256 * (10 * (int)sizeof(T) * shell_vz(sizeof(T)) + 3 * (int)sizeof(T));
}
template <typename T>
__host__ __device__ constexpr int shell_smem_bytes() {
    return shell_full_stages<T>() * shell_stage_bytes<T>();
}

// Strides and edge flags of the compact storage (CMP only).
struct ShellStore {
    int sx, sy;         // plane and row strides of that storage
    bool y_hi_grid;     // this row reads its high y face from the grid
    bool y_lo_grid;     // this row also writes its low y faces to the grid
    int spare;          // offset (from the group) of the spare high-z-face slot, 0: next slot
};

// Loads of one x plane of a shell column (everything but p(x-1), p(x) and the
// low x face, which the previous plane carries).
template <typename T, int V>
struct ShellPlane {
    Vec<T, V> pp, ym, yp, vxr, vyl, vyr, vzl, a0, a1, a2;
    T zme, zpe, vze;
    AxisCoef<T> cxr;
    uint8_t g;
};

// The loads of shell_load as asynchronous copies into ring stage `st` (the
// shared address of this thread's vector slot 0 of the stage): vector field f at
// st + f * 256 * VB, scalar field k at this thread's word of the scalar arrays.
template <typename T, int V, bool CMP>
__device__ __forceinline__ void shell_stage(const KArgs<T>& A, const ShellStore& S, unsigned st, int x,
                                            bool last_plane, unsigned c, unsigned q, int oym, int oyp, int ozm) {
    constexpr int W = (int)sizeof(T), VB = W * V;
    constexpr unsigned FV = 256 * VB, FS = 256 * W, S0 = 10 * FV;
    const unsigned sc = st + S0 - (unsigned)((VB - W) * threadIdx_lin());  // scalar field 0 of this thread
    const int sx = (int)A.sx, sy = (int)A.sy;
    const T* pc = A.pc + c;
    cpa<VB>(st + 0 * FV, pc + (x + 1 < A.N0 ? sx : 0));
    cpa<VB>(st + 1 * FV, pc - oym);
    cpa<VB>(st + 2 * FV, pc + oyp);
    cpa<W>(sc + 0 * FS, pc - ozm);
    cpa<W>(sc + 1 * FS, pc + V);
    if constexpr (CMP) {
        cpa<VB>(st + 3 * FV, last_plane ? A.vo[0] + c + sx : A.zvo[0] + q + S.sx);
        cpa<VB>(st + 4 * FV, A.zvo[1] + q);
        cpa<VB>(st + 5 * FV, S.y_hi_grid ? A.vo[1] + c + sy : A.zvo[1] + q + S.sy);
        cpa<VB>(st + 6 * FV, A.zvo[2] + q);
        cpa<W>(sc + 2 * FS, A.zvo[2] + q + (S.spare ? S.spare : V));
    } else {
        cpa<VB>(st + 3 * FV, A.vo[0] + c + sx);
        cpa<VB>(st + 4 * FV, A.vo[1] + c);
        cpa<VB>(st + 5 * FV, A.vo[1] + c + sy);
        cpa<VB>(st + 6 * FV, A.vo[2] + c);
        cpa<W>(sc + 2 * FS, A.vo[2] + c + V);
    }
    cpa<VB>(st + 7 * FV, sh_pd<T, CMP>(A, 0) + q);
    cpa<VB>(st + 8 * FV, sh_pd<T, CMP>(A, 1) + q);
    cpa<VB>(st + 9 * FV, sh_pd<T, CMP>(A, 2) + q);
}

// Read back a completed stage (`sp`: generic pointer to this thread's vector slot 0).
template <typename T, int V>
__device__ __forceinline__ void shell_unstage(const KArgs<T>& A, ShellPlane<T, V>& L, const char* sp, int x) {
    constexpr int W = (int)sizeof(T), VB = W * V;
    constexpr int FV = 256 * VB, FS = 256 * W, S0 = 10 * FV;
    using VT = Vec<T, V>;
    const char* sc = sp + S0 - (VB - W) * threadIdx_lin();
    L.g = __ldg(A.axflag[0] + x);
    L.cxr = A.coef[0][x + 1];
    L.pp = *reinterpret_cast<const VT*>(sp + 0 * FV);
    L.ym = *reinterpret_cast<const VT*>(sp + 1 * FV);
    L.yp = *reinterpret_cast<const VT*>(sp + 2 * FV);
    L.zme = *reinterpret_cast<const T*>(sc + 0 * FS);
    L.zpe = *reinterpret_cast<const T*>(sc + 1 * FS);
    L.vxr = *reinterpret_cast<const VT*>(sp + 3 * FV);
    L.vyl = *reinterpret_cast<const VT*>(sp + 4 * FV);
    L.vyr = *reinterpret_cast<const VT*>(sp + 5 * FV);
    L.vzl = *reinterpret_cast<const VT*>(sp + 6 * FV);
    L.vze = *reinterpret_cast<const T*>(sc + 2 * FS);
    L.a0 = *reinterpret_cast<const VT*>(sp + 7 * FV);
    L.a1 = *reinterpret_cast<const VT*>(sp + 8 * FV);
    L.a2 = *reinterpret_cast<const VT*>(sp + 9 * FV);
}

template <typename T, int V, bool CMP>
__device__ __forceinline__ void shell_load(const KArgs<T>& A, const ShellStore& S, ShellPlane<T, V>& L, int x,
                                           bool last_plane, unsigned c, unsigned q, int oym, int oyp, int ozm) {
    const int sx = (int)A.sx, sy = (int)A.sy;
    const T* pc = A.pc + c;
    L.g = __ldg(A.axflag[0] + x);
    L.cxr = A.coef[0][x + 1];
    L.pp = ldv<T, V>(pc + (x + 1 < A.N0 ? sx : 0));
    L.ym = ldv<T, V>(pc - oym);
    L.yp = ldv<T, V>(pc + oyp);
    L.zme = pc[-ozm];
    L.zpe = pc[V];
    if constexpr (CMP) {
        L.vxr = last_plane ? ldv<T, V>(A.vo[0] + c + sx) : ldv<T, V>(A.zvo[0] + q + S.sx);
        L.vyl = ldv<T, V>(A.zvo[1] + q);
        L.vyr = S.y_hi_grid ? ldv<T, V>(A.vo[1] + c + sy) : ldv<T, V>(A.zvo[1] + q + S.sy);
        L.vzl = ldv<T, V>(A.zvo[2] + q);
        L.vze = A.zvo[2][q + (S.spare ? S.spare : V)];
    } else {
        L.vxr = ldv<T, V>(A.vo[0] + c + sx);
        L.vyl = ldv<T, V>(A.vo[1] + c);
        L.vyr = ldv<T, V>(A.vo[1] + c + sy);
        L.vzl = ldv<T, V>(A.vo[2] + c);
        L.vze = A.vo[2][c + V];
    }
    L.a0 = ldv<T, V>(sh_pd<T, CMP>(A, 0) + q);
    L.a1 = ldv<T, V>(sh_pd<T, CMP>(A, 1) + q);
    L.a2 = ldv<T, V>(sh_pd<T, CMP>(A, 2) + q);
}

// One PML-shell tile: unit tile tu (256 consecutive (row, z-group) units of box
// b, one per thread) by x tile tx.  A thread owns one z group (a vector of
// shell_vz cells starting at a multiple of its width; cells outside the
// group's z range are masked) of one row and marches along x over B.xs planes:
// p(x-1), p(x) and the low x face velocity are carried in registers, and (with
// FDTD_SHELL_PREFETCH) the loads of plane x+1 are issued before plane x is
// computed and stored.  Face flags (MAC_Grid.cpp:2568-2575, :2631-2633) are
// V-bit masks from the packed per-axis tables; the arithmetic per cell is the
// reference's, in its order.  CMP: box b is the z-slab pair with compact storage.
template <typename T, bool CMP>
__device__ __forceinline__ void shell_tile_impl(const KArgs<T>& A, const ShellBoxes& B, int b, int tu, int tx) {
    constexpr int V = shell_vz(sizeof(T));
    constexpr unsigned ALL = (1u << V) - 1u;
    using VT = Vec<T, V>;
    const int u = tu * 256 + threadIdx.x + 32 * threadIdx.y;
    const int ng = B.ng[b];
    if (u >= B.ny[b] * ng) return;
    const int yl = u / ng;
    const int gi = u - yl * ng;
    const int y = B.y0[b] + yl;
    // the group and its cells belong to the range they were enumerated from (a
    // low and a high group may share a vector when the ranges are close)
    const bool first = gi < B.gl[b];
    const int zg = first ? (B.za[b] / V + gi) * V : (B.zb[b] / V + (gi - B.gl[b])) * V;
    const int zr0 = first ? B.za[b] : B.zb[b], zr1 = first ? B.zae[b] : B.zbe[b];
    unsigned inbox = 0;
#pragma unroll
    for (int e = 0; e < V; ++e) inbox |= (zg + e >= zr0 && zg + e < zr1 ? 1u : 0u) << e;
    const int x0 = B.x0[b] + tx * B.xs;
    const int x1 = min(x0 + B.xs, B.x0[b] + B.nx[b]);
    const int xend = B.x0[b] + B.nx[b];
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned c0 = (unsigned)x0 * A.sx + (unsigned)y * A.sy + zg;  // cell and its three low faces

    ShellStore S;
    unsigned q0;
    if constexpr (CMP) {
        S.sy = B.zrw;
        S.sx = B.ny[b] * B.zrw;
        q0 = (unsigned)(x0 - B.x0[b]) * S.sx + (unsigned)yl * S.sy + gi * V;
        const bool last_group = first ? (gi == B.gl[b] - 1) : (gi == ng - 1);
        S.spare = last_group ? (ng - gi) * V + (first ? 0 : 1) : 0;
        S.y_hi_grid = (y + 1 == B.y0[b] + B.ny[b]);
        S.y_lo_grid = (yl == 0);
    } else {
        S.sx = sx;
        S.sy = sy;
        q0 = c0;
        S.spare = 0;
        S.y_hi_grid = S.y_lo_grid = false;
    }

    const uint8_t gy = __ldg(A.axflag[1] + y);
    uint8_t gz[V];
#pragma unroll
    for (int e = 0; e < V; ++e) gz[e] = __ldg(A.axflag[2] + zg + e);
    const unsigned zpml = flag_mask<V>(gz, 0), zflo = flag_mask<V>(gz, 1), zfhi = flag_mask<V>(gz, 2);
    const unsigned znext = flag_mask<V>(gz, 3), zhlo = flag_mask<V>(gz, 4), zhhi = flag_mask<V>(gz, 5);
    const unsigned mpy = (gy & AXF_PML) ? ALL : 0u;
    const int oym = (gy & AXF_HAS_LO) ? sy : 0, oyp = (gy & AXF_HAS_HI) ? sy : 0;
    const int ozm = zg > 0 ? 1 : 0;
    const AxisCoef<T> cyl = A.coef[1][y], cyr = A.coef[1][y + 1];
    AxisCoef<T> cz[V + 1];
#pragma unroll
    for (int e = 0; e <= V; ++e) cz[e] = A.coef[2][zg + e];

    // carried along x
    VT pm = ldv<T, V>(A.pc + c0 - (x0 > 0 ? sx : 0));
    VT p0 = ldv<T, V>(A.pc + c0);
    VT vxl = ldv<T, V>(sh_vo<T, CMP>(A, 0) + q0);
    AxisCoef<T> cxl = A.coef[0][x0];
    ShellPlane<T, V> cur, nxt;
    constexpr int NS = shell_full_stages<T>();
    constexpr bool PF = NS == 0 && FDTD_SHELL_PREFETCH;
    extern __shared__ __align__(16) char full_ring[];
    char* const sp0 = full_ring + threadIdx_lin() * (int)sizeof(T) * V;
    const unsigned ss0 = (unsigned)__cvta_generic_to_shared(sp0);
    if constexpr (NS > 0) {
#pragma unroll
        for (int k = 0; k < NS - 1; ++k) {
            if (x0 + k < x1)
                shell_stage<T, V, CMP>(A, S, ss0 + k * shell_stage_bytes<T>(), x0 + k, x0 + k + 1 == xend,
                                       c0 + (unsigned)k * A.sx, q0 + (unsigned)(k * S.sx), oym, oyp, ozm);
            cpa_commit();
        }
    } else if constexpr (PF) {
        shell_load<T, V, CMP>(A, S, cur, x0, x0 + 1 == xend, c0, q0, oym, oyp, ozm);
    }
    int ring = 0;  // stage of plane x
#pragma unroll 1
    for (int x = x0; x < x1; ++x) {
        const unsigned c = c0 + (unsigned)(x - x0) * A.sx;
        const unsigned q = CMP ? q0 + (unsigned)(x - x0) * S.sx : c;
        if constexpr (NS > 0) {
            // the stage of plane x + NS - 1 is the one plane x - 1 was read from
            const int st = ring == 0 ? NS - 1 : ring - 1;
            if (x + NS - 1 < x1)
                shell_stage<T, V, CMP>(A, S, ss0 + st * shell_stage_bytes<T>(), x + NS - 1, x + NS == xend,
                                       c + (unsigned)(NS - 1) * A.sx, q + (unsigned)((NS - 1) * S.sx), oym, oyp,
                                       ozm);
            cpa_commit();
            cpa_wait<NS - 1>();
            shell_unstage<T, V>(A, cur, sp0 + ring * shell_stage_bytes<T>(), x);
            ring = ring == NS - 1 ? 0 : ring + 1;
        } else if constexpr (PF) {
            if (x + 1 < x1) shell_load<T, V, CMP>(A, S, nxt, x + 1, x + 2 == xend, c + sx, q + S.sx, oym, oyp, ozm);
        } else {
            shell_load<T, V, CMP>(A, S, cur, x, x + 1 == xend, c, q, oym, oyp, ozm);
        }
        const uint8_t g = cur.g;
        const unsigned mpx = (g & AXF_PML) ? ALL : 0u;
        const unsigned oyz = mpy | zpml, oxz = mpx | zpml, oxy = mpx | mpy;
        // faces inside the PML, outer faces excluded; a high face is written by
        // this cell only when the cell beyond it is not a PML cell
        const unsigned fxl = ((g & AXF_FACE_LO) ? ALL : 0u) | ((g & AXF_HAS_LO) ? oyz : 0u);
        const unsigned fxr = ((g & AXF_FACE_HI) ? ALL : 0u) | ((g & AXF_HAS_HI) ? oyz : 0u);
        const unsigned fyl = ((gy & AXF_FACE_LO) ? ALL : 0u) | ((gy & AXF_HAS_LO) ? oxz : 0u);
        const unsigned fyr = ((gy & AXF_FACE_HI) ? ALL : 0u) | ((gy & AXF_HAS_HI) ? oxz : 0u);
        const unsigned fzl = zflo | (zhlo & oxy);
        const unsigned fzr = zfhi | (zhhi & oxy);
        const unsigned m_xl = inbox & fxl;
        const unsigned m_xr = inbox & fxr & ~(((g & AXF_NEXT_PML) ? ALL : 0u) | oyz);
        const unsigned m_yl = inbox & fyl;
        const unsigned m_yr = inbox & fyr & ~(((gy & AXF_NEXT_PML) ? ALL : 0u) | oxz);
        const unsigned m_zl = inbox & fzl;
        const unsigned m_zr = inbox & fzr & ~(znext | oxy);
        const AxisCoef<T> cxr = cur.cxr;
        VT nxl, nxr, nyl, nyr, nzl, ax, ay, az, pn;
        T nzr[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const T pz = p0.e[e];
            const T pzm = e > 0 ? p0.e[e - 1] : cur.zme;
            const T pzp = e < V - 1 ? p0.e[e + 1] : cur.zpe;
            const T vx_l0 = vxl.e[e], vx_r0 = cur.vxr.e[e], vy_l0 = cur.vyl.e[e], vy_r0 = cur.vyr.e[e];
            const T vz_l0 = cur.vzl.e[e], vz_r0 = e < V - 1 ? cur.vzl.e[e + 1] : cur.vze;
            const T vx_l = ((fxl >> e) & 1u) ? vel_update<T>(vx_l0, cxl.vupd, cxl.vgrad, pz, pm.e[e]) : vx_l0;
            const T vx_r = ((fxr >> e) & 1u) ? vel_update<T>(vx_r0, cxr.vupd, cxr.vgrad, cur.pp.e[e], pz) : vx_r0;
            const T vy_l = ((fyl >> e) & 1u) ? vel_update<T>(vy_l0, cyl.vupd, cyl.vgrad, pz, cur.ym.e[e]) : vy_l0;
            const T vy_r = ((fyr >> e) & 1u) ? vel_update<T>(vy_r0, cyr.vupd, cyr.vgrad, cur.yp.e[e], pz) : vy_r0;
            const T vz_l = ((fzl >> e) & 1u) ? vel_update<T>(vz_l0, cz[e].vupd, cz[e].vgrad, pz, pzm) : vz_l0;
            const T vz_r = ((fzr >> e) & 1u) ? vel_update<T>(vz_r0, cz[e + 1].vupd, cz[e + 1].vgrad, pzp, pz) : vz_r0;
            nxl.e[e] = vx_l;
            nxr.e[e] = vx_r;
            nyl.e[e] = vy_l;
            nyr.e[e] = vy_r;
            nzl.e[e] = vz_l;
            nzr[e] = vz_r;
            ax.e[e] = pd_update<T>(cur.a0.e[e], cxl.pupd, cxl.pdiv, vx_r, vx_l, A.inv_h);
            ay.e[e] = pd_update<T>(cur.a1.e[e], cyl.pupd, cyl.pdiv, vy_r, vy_l, A.inv_h);
            az.e[e] = pd_update<T>(cur.a2.e[e], cz[e].pupd, cz[e].pdiv, vz_r, vz_l, A.inv_h);
            pn.e[e] = ax.e[e] + ay.e[e] + az.e[e];
        }
        st_masked<T, V>(sh_vn<T, CMP>(A, 0) + q, nxl, m_xl);
        st_masked<T, V>(sh_vn<T, CMP>(A, 1) + q, nyl, m_yl);
        st_masked<T, V>(sh_vn<T, CMP>(A, 2) + q, nzl, m_zl);
        if constexpr (CMP) {
            // low x / y faces shared with the x / y slabs, high faces owned by them
            if (x == B.x0[b]) st_masked<T, V>(A.vn[0] + c, nxl, m_xl);
            if (S.y_lo_grid) st_masked<T, V>(A.vn[1] + c, nyl, m_yl);
            st_masked<T, V>(x + 1 == xend ? A.vn[0] + c + sx : A.zvn[0] + q + S.sx, nxr, m_xr);
            st_masked<T, V>(S.y_hi_grid ? A.vn[1] + c + sy : A.zvn[1] + q + S.sy, nyr, m_yr);
        } else {
            st_masked<T, V>(A.vn[0] + c + sx, nxr, m_xr);
            st_masked<T, V>(A.vn[1] + c + sy, nyr, m_yr);
        }
        if (m_zr) {
            T* vz = sh_vn<T, CMP>(A, 2);
#pragma unroll
            for (int e = 0; e < V; ++e)
                if ((m_zr >> e) & 1u) vz[q + ((e == V - 1 && S.spare) ? S.spare : e + 1)] = nzr[e];
        }
        st_masked<T, V>(sh_pd<T, CMP>(A, 0) + q, ax, inbox);
        st_masked<T, V>(sh_pd<T, CMP>(A, 1) + q, ay, inbox);
        st_masked<T, V>(sh_pd<T, CMP>(A, 2) + q, az, inbox);
        st_masked<T, V>(A.pn + c, pn, inbox);
        // carry to plane x+1
        pm = p0;
        p0 = cur.pp;
        vxl = cur.vxr;
        cxl = cxr;
        if constexpr (PF) cur = nxt;
    }
    if constexpr (NS > 0) cpa_wait<0>();  // no copy outlives the thread
}

template <typename T>
__device__ __forceinline__ void shell_tile(const KArgs<T>& A, const ShellBoxes& B, int b, int tu, int tx) {
    if (b == B.zbox) shell_tile_impl<T, true>(A, B, b, tu, tx);
    else shell_tile_impl<T, false>(A, B, b, tu, tx);
}

// CTA -> (box, unit tile, plane tile) through the prefix table of the shell boxes
__device__ __forceinline__ void shell_decode(const ShellBoxes& B, int blk, int& b, int& tu, int& tx) {
    b = 0;
#pragma unroll
    for (int q = 1; q < SHELL_MAX_BOXES; ++q)
        if (q < B.n && blk >= B.block_first[q]) b = q;
    const int local = blk - B.block_first[b];
    tu = local % B.tu[b];
    tx = local / B.tu[b];
}

template <typename T>
__global__ void __launch_bounds__(256, shell_min_blocks(sizeof(T))) k_pml_shell(const KArgs<T> A, const ShellBoxes B) {
    if (A.advance && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) advance_consts(*A.P, A.cur);
    int b, tu, tx;
    shell_decode(B, blockIdx.x, b, tu, tx);
    shell_tile<T>(A, B, b, tu, tx);
}

}  // namespace fdtd

#include "fdtd_engquist.cuh"
#include "fdtd_shell_red.cuh"
#include "fdtd_shell_tma.cuh"

namespace fdtd {

// Host side: one region-split step (streams: StepStreams).  Launch order: the
// ghost-cell list (s3), the interior (s2), the shell (s) (FP64: the shell before
// the interior), then the sources (s2, after the interior and the ghost list,
// whose cells they add to).
#ifndef FDTD_SHELL_FIRST_F64
#define FDTD_SHELL_FIRST_F64 1
#endif
template <typename T>
cudaError_t launch_regions(const SolveParams* dP, const SolveParams& hP, const RegionLaunch& R, int cur,
                           const StepStreams& S, int* launches) {
    int l = 0;
    const KArgs<T> A = make_kargs<T>(const_cast<SolveParams*>(dP), hP, cur);
    const Box3& b = R.interior;
    const int nx = b.hi[0] - b.lo[0], ny = b.hi[1] - b.lo[1], nz = b.hi[2] - b.lo[2];
    const bool has_interior = nx > 0 && ny > 0 && nz > 0 && !(R.skip & 1);
    const bool has_ghost = R.ghost_cap > 0 && !(R.skip & 4);
    const bool split = has_interior && S.s2 != nullptr;
    const bool gside = split && (has_ghost || R.fc) && S.s3 != nullptr;
    const cudaStream_t si = split ? S.s2 : S.s;
    cudaError_t e = cudaSuccess;
    const unsigned eng_blocks = hP.eng_n > 0 ? (unsigned)std::min((hP.eng_n + 127) / 128, 148 * 8) : 0u;
    if (eng_blocks) {
        // Engquist cells read p^{n-1} of their stencils: before any kernel writes p^{n+1}
        k_engquist_predict<T><<<eng_blocks, 128, 0, S.s>>>(dP, cur);
        ++l;
    }
    if (split) {
        e = cudaEventRecord(S.fork, S.s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(S.s2, S.fork, 0);
        if (e == cudaSuccess && gside) e = cudaStreamWaitEvent(S.s3, S.fork, 0);
        if (e != cudaSuccess) return e;
    }
    if (R.fc) {
        // FULLY_COUPLED: this step's ghost pressures, before the cells that read them
        k_fc_rhs<T><<<64, 256, 0, gside ? S.s3 : si>>>(dP, cur);
        k_fc_solve<<<1, 1024, 0, gside ? S.s3 : si>>>(dP, cur);
        l += 2;
    }
    if (has_ghost) {
        // cells next to a solid: disjoint from the interior and shell cells
        const int blocks = (R.ghost_cap + 127) / 128 < 1184 ? (R.ghost_cap + 127) / 128 : 1184;
        k_ghost_cells<T><<<blocks, 128, 0, gside ? S.s3 : si>>>(dP, cur);
        ++l;
    }
    if (gside && (e = cudaEventRecord(S.ghost, S.s3)) != cudaSuccess) return e;
    // FP64: the shell first.  A shell CTA (188 registers, the 141 KB ring) takes
    // one per SM and leaves the registers of one interior CTA beside it, which
    // the interior's CTAs, dispatched after, fill; FP32 CTAs of the two kernels
    // do not fit one SM together, and the interior goes first.
    constexpr bool shell_first = sizeof(T) == 8 && FDTD_SHELL_FIRST_F64;
    auto launch_interior = [&]() {
        if (has_interior) {
            dim3 block(32, 8);
            const int xb = (!hP.visc && (R.xb == 4 || R.xb == 8)) ? R.xb : 2;
            dim3 grid(interior_unit_tiles(b, 16 / (int)sizeof(T)), (nx + xb - 1) / xb);
            if (hP.visc) k_interior<T, 2, true><<<grid, block, 0, si>>>(A, b);
            else if (xb == 2) k_interior<T, 2><<<grid, block, 0, si>>>(A, b);
            else if (xb == 8) k_interior<T, 8><<<grid, block, 0, si>>>(A, b);
            else k_interior<T, 4><<<grid, block, 0, si>>>(A, b);
            ++l;
        }
    };
    if (!shell_first) launch_interior();
    const int nblk = (R.skip & 2) ? 0 : R.shell.block_first[R.shell.n];
    if (nblk > 0) {
        if constexpr (sizeof(T) == 4) {
            if (R.red && R.tma)
                k_pml_shell_tma<float><<<R.tma->grid, TMA_BLOCK, tma_smem_bytes(R.tma->launch), S.s>>>(
                    A, R.tma->launch, R.tma->d_tiles, R.tma->d_cta_first, R.tma->d_maps, hP.dev_error);
            else if (R.red) k_pml_shell_red<float><<<nblk, dim3(32, 8), red_smem_bytes(), S.s>>>(A, R.shell);
            else k_pml_shell<T><<<nblk, dim3(32, 8), shell_smem_bytes<T>(), S.s>>>(A, R.shell);
        } else {
            k_pml_shell<T><<<nblk, dim3(32, 8), shell_smem_bytes<T>(), S.s>>>(A, R.shell);
        }
        ++l;
    }
    if (shell_first) launch_interior();
    if (gside && (e = cudaStreamWaitEvent(S.s2, S.ghost, 0)) != cudaSuccess) return e;
    if (R.sources) {
        // source cells are non-PML cells: after the interior and ghost updates of
        // their cells, concurrent with the shell
        const Box3& r = R.src_region;
        const long long total = (long long)(r.hi[0] - r.lo[0]) * (r.hi[1] - r.lo[1]) * (r.hi[2] - r.lo[2]);
        if (total > 0) {
            const long long g = (total + 255) / 256;
            k_sources<T><<<(unsigned)(g < 148 * 16 ? g : 148 * 16), 256, 0, si>>>(dP, cur, r);
            ++l;
        }
    }
    if (split) {
        e = cudaEventRecord(S.join, S.s2);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(S.s, S.join, 0);
        if (e != cudaSuccess) return e;
    }
    if (eng_blocks) {
        // after every kernel that reads p^n: the exterior values go into both buffers
        k_engquist_commit<T><<<eng_blocks, 128, 0, S.s>>>(dP, cur);
        ++l;
    }
    if (launches) *launches += l;
    return cudaGetLastError();
}

}  // namespace fdtd
