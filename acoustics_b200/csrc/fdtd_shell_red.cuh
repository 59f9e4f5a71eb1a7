// fdtd_shell_red.cuh — PML-shell tile of FP32 solves on the reduced PML state.
//
// Take a PML cell c and an axis d along which c lies outside the PML: the
// absorption is zero at c and at both of its d faces, and neither face is an
// outer wall.  The reference updates that axis with unit decay factors,
//   v_d <- v_d + g0 (p[right] - p[left])          on both d faces (MAC_Grid.cpp:461-479)
//   p_d <- p_d + D0 (v_d[hi] - v_d[lo]) / h                       (MAC_Grid.cpp:496-508)
// with g0 = -k/(rho h) and D0 = -rho c^2 k.  Differencing two steps, the face
// velocities cancel:
//   p_d^{n+1} - p_d^n = (p_d^n - p_d^{n-1}) + (ck/h)^2 (p[c+e_d] - 2 p[c] + p[c-e_d]),
// which is the interior's leapfrog.  Summed over the plain axes P(c) of the
// cell it needs one increment q = sum_{d in P} (p_d^n - p_d^{n-1}) per cell
// instead of |P| split pressures and 2|P| face velocities.  The absorbing axes
// A(c) keep the reference's split form, and the plain part of p^n is what the
// absorbing split pressures leave of it:
//   q       <- q + (ck/h)^2 sum_{d in P} (p[c+e_d] - 2 p[c] + p[c-e_d])
//   p^{n+1}  = sum_{d in A} p_d^{n+1} + (p^n - sum_{d in A} p_d^n) + q
// In exact arithmetic this is the reference's step; in FP32 it differs by
// rounding.  Face velocities are kept only along absorbing axes; such a face is
// written by the cell to its right when that cell absorbs along the axis, else
// by its left cell.  A slab cell (one absorbing axis) then moves 8 words per
// step instead of 14.
//
// Storage (the arrays of the full state, fewer of them touched): q lives in the
// split-pressure array of the cell's first plain axis.
//   x slabs   a0 = p_x;  a1 = p_y (row inside the y PML) or q;  a2 = p_z (z-PML cell) or q (when a1 = p_y)
//   y slabs   a0 = q;    a1 = p_y;  a2 = p_z (z-PML cell)
//   z slabs   a0 = q;    a2 = p_z   (compact arrays of the z-slab pair)
// The host uses this state only where it is exact: FP32 static scenes with no
// solid cell inside the PML and zero absorption on every face of a cell outside
// the PML along that face's axis.
// Included by fdtd_hot.cuh after the tile primitives (Vec, ldv, st_masked,
// flag_mask, shell_decode) and before the launcher.
#pragma once

#ifndef FDTD_SHELL_RED_MINB
#define FDTD_SHELL_RED_MINB 2
#endif
#ifndef FDTD_SHELL_RED_PREFETCH
#define FDTD_SHELL_RED_PREFETCH 1
#endif
// x planes whose loads a thread keeps in flight through a shared-memory ring
// (cp.async); 0: the register prefetch of FDTD_SHELL_RED_PREFETCH instead
#ifndef FDTD_SHELL_RED_STAGES
#define FDTD_SHELL_RED_STAGES 3
#endif

namespace fdtd {

// Shared-memory ring of the staged loads: per stage, RED_NVEC vector fields
// (pp, ym, yp, vxr, vyl, vyr, vzl, a0, a1, a2) and RED_NSCA scalar fields (zme,
// zpe, vze), each an array over the CTA's 256 threads, so a thread's slots are
// consecutive words of its own (no bank conflict, no barrier: every thread
// reads back only what it copied).
constexpr int RED_NVEC = 10, RED_NSCA = 3;
__host__ __device__ constexpr int red_stage_bytes() { return 256 * (RED_NVEC * 4 * shell_vz(4) + RED_NSCA * 4); }
__host__ __device__ constexpr int red_smem_bytes() {
    return FDTD_SHELL_RED_STAGES > 0 ? FDTD_SHELL_RED_STAGES * red_stage_bytes() : 0;
}

// Loads of one x plane of a reduced-state shell column.
template <int V>
struct RedPlane {
    Vec<float, V> pp, ym, yp, vxr, vyl, vyr, vzl, a0, a1, a2;
    float zme, zpe, vze;
    AxisCoef<float> cxr;
    uint8_t g;
};

// KIND 0: x slab (x absorbing; y absorbing when EY), 1: y slab, 2: z-slab pair.
template <int KIND, bool EY>
__device__ __forceinline__ void red_load(const KArgs<float>& A, RedPlane<shell_vz(4)>& L, int x, unsigned c,
                                         unsigned q, int spare, unsigned ezm, int oym, int oyp, int ozm) {
    constexpr int V = shell_vz(4);
    constexpr bool CMP = KIND == 2;
    const int sx = (int)A.sx, sy = (int)A.sy;
    const float* pc = A.pc + c;
    L.pp = ldv<float, V>(pc + (x + 1 < A.N0 ? sx : 0));
    L.ym = ldv<float, V>(pc - oym);
    L.yp = ldv<float, V>(pc + oyp);
    L.zme = pc[-ozm];
    L.zpe = pc[V];
    if constexpr (KIND == 0) {
        L.g = __ldg(A.axflag[0] + x);
        L.cxr = A.coef[0][x + 1];
        L.vxr = ldv<float, V>(A.vo[0] + c + sx);
    }
    if constexpr (EY) {
        L.vyl = ldv<float, V>(A.vo[1] + c);
        L.vyr = ldv<float, V>(A.vo[1] + c + sy);
    }
    if (ezm) {
        const float* vz = CMP ? A.zvo[2] : A.vo[2];
        L.vzl = ldv<float, V>(vz + q);
        L.vze = vz[q + (spare ? spare : V)];
    }
    float* const* pd = CMP ? A.zpd : A.pd;
    L.a0 = ldv<float, V>(pd[0] + q);
    if constexpr (KIND != 2) L.a1 = ldv<float, V>(pd[1] + q);
    if ((KIND == 0 && EY) || ezm) L.a2 = ldv<float, V>(pd[2] + q);
}

// The loads of red_load as asynchronous copies into ring stage `st` (a shared
// address of this thread's slot 0 of the stage).
template <int KIND, bool EY>
__device__ __forceinline__ void red_stage(const KArgs<float>& A, unsigned st, int x, unsigned c, unsigned q, int spare,
                                          unsigned ezm, int oym, int oyp, int ozm) {
    constexpr int V = shell_vz(4);
    constexpr int VB = 4 * V;
    constexpr unsigned FV = 256 * VB, FS = 256 * 4, S0 = RED_NVEC * FV;
    constexpr bool CMP = KIND == 2;
    const int sx = (int)A.sx, sy = (int)A.sy;
    const float* pc = A.pc + c;
    cpa<VB>(st + 0 * FV, pc + (x + 1 < A.N0 ? sx : 0));
    cpa<VB>(st + 1 * FV, pc - oym);
    cpa<VB>(st + 2 * FV, pc + oyp);
    cpa<4>(st + S0 + 0 * FS - (VB - 4) * threadIdx_lin(), pc - ozm);
    cpa<4>(st + S0 + 1 * FS - (VB - 4) * threadIdx_lin(), pc + V);
    if constexpr (KIND == 0) cpa<VB>(st + 3 * FV, A.vo[0] + c + sx);
    if constexpr (EY) {
        cpa<VB>(st + 4 * FV, A.vo[1] + c);
        cpa<VB>(st + 5 * FV, A.vo[1] + c + sy);
    }
    if (ezm) {
        const float* vz = CMP ? A.zvo[2] : A.vo[2];
        cpa<VB>(st + 6 * FV, vz + q);
        cpa<4>(st + S0 + 2 * FS - (VB - 4) * threadIdx_lin(), vz + q + (spare ? spare : V));
    }
    float* const* pd = CMP ? A.zpd : A.pd;
    cpa<VB>(st + 7 * FV, pd[0] + q);
    if constexpr (KIND != 2) cpa<VB>(st + 8 * FV, pd[1] + q);
    if ((KIND == 0 && EY) || ezm) cpa<VB>(st + 9 * FV, pd[2] + q);
}

// Read back a completed stage (`sp`: generic pointer to this thread's slot 0).
template <int KIND, bool EY>
__device__ __forceinline__ void red_unstage(const KArgs<float>& A, RedPlane<shell_vz(4)>& L, const char* sp, int x,
                                            unsigned ezm) {
    constexpr int V = shell_vz(4);
    constexpr int VB = 4 * V;
    constexpr int FV = 256 * VB, FS = 256 * 4, S0 = RED_NVEC * FV;
    using VT = Vec<float, V>;
    const int sfix = (VB - 4) * threadIdx_lin();
    L.pp = *reinterpret_cast<const VT*>(sp + 0 * FV);
    L.ym = *reinterpret_cast<const VT*>(sp + 1 * FV);
    L.yp = *reinterpret_cast<const VT*>(sp + 2 * FV);
    L.zme = *reinterpret_cast<const float*>(sp + S0 + 0 * FS - sfix);
    L.zpe = *reinterpret_cast<const float*>(sp + S0 + 1 * FS - sfix);
    if constexpr (KIND == 0) {
        L.g = __ldg(A.axflag[0] + x);
        L.cxr = A.coef[0][x + 1];
        L.vxr = *reinterpret_cast<const VT*>(sp + 3 * FV);
    }
    if constexpr (EY) {
        L.vyl = *reinterpret_cast<const VT*>(sp + 4 * FV);
        L.vyr = *reinterpret_cast<const VT*>(sp + 5 * FV);
    }
    if (ezm) {
        L.vzl = *reinterpret_cast<const VT*>(sp + 6 * FV);
        L.vze = *reinterpret_cast<const float*>(sp + S0 + 2 * FS - sfix);
    }
    L.a0 = *reinterpret_cast<const VT*>(sp + 7 * FV);
    if constexpr (KIND != 2) L.a1 = *reinterpret_cast<const VT*>(sp + 8 * FV);
    if ((KIND == 0 && EY) || ezm) L.a2 = *reinterpret_cast<const VT*>(sp + 9 * FV);
}

// ZP: every group of box b is whole, in the box and outside the z PML (every
// per-cell z mask is then known: all cells in, none absorbing along z).
template <int KIND, bool EY, bool PF, bool ZP = false>
__device__ __forceinline__ void shell_tile_red_impl(const KArgs<float>& A, const ShellBoxes& B, int b, int u, int tx) {
    using T = float;
    constexpr bool CMP = KIND == 2;
    constexpr bool EX = KIND == 0;
    constexpr int V = shell_vz(4);
    constexpr unsigned ALL = (1u << V) - 1u;
    using VT = Vec<T, V>;
    const int ng = B.ng[b];
    const int yl = u / ng;
    const int gi = u - yl * ng;
    const int y = B.y0[b] + yl;
    const bool first = gi < B.gl[b];
    const int zg = first ? (B.za[b] / V + gi) * V : (B.zb[b] / V + (gi - B.gl[b])) * V;
    const int zr0 = first ? B.za[b] : B.zb[b], zr1 = first ? B.zae[b] : B.zbe[b];
    unsigned inbox = 0;
#pragma unroll
    for (int e = 0; e < V; ++e) inbox |= (zg + e >= zr0 && zg + e < zr1 ? 1u : 0u) << e;
    if constexpr (ZP) inbox = ALL;
    const int x0 = B.x0[b] + tx * B.xs;
    const int x1 = min(x0 + B.xs, B.x0[b] + B.nx[b]);
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned c0 = (unsigned)x0 * A.sx + (unsigned)y * A.sy + zg;
    int csx = sx, spare = 0;
    unsigned q0 = c0;
    if constexpr (CMP) {
        csx = B.ny[b] * B.zrw;
        q0 = (unsigned)(x0 - B.x0[b]) * csx + (unsigned)yl * B.zrw + gi * V;
        const bool last_group = first ? (gi == B.gl[b] - 1) : (gi == ng - 1);
        spare = last_group ? (ng - gi) * V + (first ? 0 : 1) : 0;
    }

    const uint8_t gy = __ldg(A.axflag[1] + y);
    uint8_t gz[V];
#pragma unroll
    for (int e = 0; e < V; ++e) gz[e] = ZP ? (uint8_t)0 : __ldg(A.axflag[2] + zg + e);
    const unsigned zpml = flag_mask<V>(gz, 0), zflo = flag_mask<V>(gz, 1), zfhi = flag_mask<V>(gz, 2);
    const unsigned znext = flag_mask<V>(gz, 3), zhlo = flag_mask<V>(gz, 4), zhhi = flag_mask<V>(gz, 5);
    const unsigned ezm = zpml & inbox;  // cells absorbing along z
    const unsigned mpy = (gy & AXF_PML) ? ALL : 0u;
    const int oym = (gy & AXF_HAS_LO) ? sy : 0, oyp = (gy & AXF_HAS_HI) ? sy : 0;
    const int ozm = zg > 0 ? 1 : 0;
    // faces the reference updates (inside the PML, outer walls excluded), as in shell_tile_impl
    const unsigned mpx = EX ? ALL : 0u;
    const unsigned fyl = ((gy & AXF_FACE_LO) ? ALL : 0u) | ((gy & AXF_HAS_LO) ? (mpx | zpml) : 0u);
    const unsigned fyr = ((gy & AXF_FACE_HI) ? ALL : 0u) | ((gy & AXF_HAS_HI) ? (mpx | zpml) : 0u);
    const unsigned fzl = zflo | (zhlo & (mpx | mpy));
    const unsigned fzr = zfhi | (zhhi & (mpx | mpy));
    // faces this cell writes: its low face along an absorbing axis, its high face
    // when the next cell does not absorb along that axis
    const unsigned m_yl = EY ? inbox & fyl : 0u;
    const unsigned m_yr = EY ? inbox & fyr & ((gy & AXF_NEXT_PML) ? 0u : ALL) : 0u;
    const unsigned m_zl = ezm & fzl;
    const unsigned m_zr = ezm & fzr & ~znext;
    const unsigned m_a1 = KIND == 2 ? 0u : inbox;
    const unsigned m_a2 = (KIND == 0 && EY) ? inbox : ezm;
    AxisCoef<T> cyl, cyr;
    if constexpr (EY) {
        cyl = A.coef[1][y];
        cyr = A.coef[1][y + 1];
    }
    AxisCoef<T> cz[V + 1];
    if (ezm) {
#pragma unroll
        for (int e = 0; e <= V; ++e) cz[e] = A.coef[2][zg + e];
    }
    const float ls = A.lap_scale, c2k2 = A.c2k2, inv_h = A.inv_h;

    // carried along x
    VT pm = ldv<T, V>(A.pc + c0 - (x0 > 0 ? sx : 0));
    VT p0 = ldv<T, V>(A.pc + c0);
    VT vxl;
    AxisCoef<T> cxl;
    if constexpr (EX) {
        vxl = ldv<T, V>(A.vo[0] + c0);
        cxl = A.coef[0][x0];
    }
    RedPlane<V> cur, nxt;
    constexpr int NS = FDTD_SHELL_RED_STAGES;
    extern __shared__ __align__(16) char red_ring[];
    // this thread's slot 0 of stage 0 (vector fields are VB bytes per thread,
    // scalar fields 4: red_stage/red_unstage correct the scalar offsets)
    const int tl = threadIdx_lin();
    char* const sp0 = red_ring + tl * 4 * V;
    const unsigned ss0 = (unsigned)__cvta_generic_to_shared(sp0);
    if constexpr (NS > 0) {
#pragma unroll
        for (int k = 0; k < NS - 1; ++k) {
            if (x0 + k < x1)
                red_stage<KIND, EY>(A, ss0 + k * red_stage_bytes(), x0 + k, c0 + (unsigned)k * A.sx,
                                    q0 + (unsigned)(k * csx), spare, ezm, oym, oyp, ozm);
            cpa_commit();
        }
    } else if constexpr (PF) {
        red_load<KIND, EY>(A, cur, x0, c0, q0, spare, ezm, oym, oyp, ozm);
    }
    float* const* pdst = CMP ? A.zpd : A.pd;
    T* const vzn = CMP ? A.zvn[2] : A.vn[2];
    int ring = 0;  // stage of plane x
#pragma unroll 1
    for (int x = x0; x < x1; ++x) {
        const unsigned c = c0 + (unsigned)(x - x0) * A.sx;
        const unsigned q = CMP ? q0 + (unsigned)(x - x0) * csx : c;
        if constexpr (NS > 0) {
            // the stage of plane x + NS - 1 is the one plane x - 1 was read from
            const int st = ring == 0 ? NS - 1 : ring - 1;
            if (x + NS - 1 < x1)
                red_stage<KIND, EY>(A, ss0 + st * red_stage_bytes(), x + NS - 1, c + (unsigned)(NS - 1) * A.sx,
                                    q + (unsigned)((NS - 1) * csx), spare, ezm, oym, oyp, ozm);
            cpa_commit();
            cpa_wait<NS - 1>();
            red_unstage<KIND, EY>(A, cur, sp0 + ring * red_stage_bytes(), x, ezm);
            ring = ring == NS - 1 ? 0 : ring + 1;
        } else if constexpr (PF) {
            if (x + 1 < x1) red_load<KIND, EY>(A, nxt, x + 1, c + sx, q + csx, spare, ezm, oym, oyp, ozm);
        } else {
            red_load<KIND, EY>(A, cur, x, c, q, spare, ezm, oym, oyp, ozm);
        }
        unsigned fxl = 0, fxr = 0, m_xl = 0, m_xr = 0;
        if constexpr (EX) {
            const uint8_t g = cur.g;
            const unsigned oyz = mpy | zpml;
            fxl = ((g & AXF_FACE_LO) ? ALL : 0u) | ((g & AXF_HAS_LO) ? oyz : 0u);
            fxr = ((g & AXF_FACE_HI) ? ALL : 0u) | ((g & AXF_HAS_HI) ? oyz : 0u);
            m_xl = inbox & fxl;
            m_xr = inbox & fxr & ((g & AXF_NEXT_PML) ? 0u : ALL);
        }
        VT nxl, nxr, nyl, nyr, nzl, o0, o1, o2, pn;
        T nzr[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const T pz = p0.e[e];
            const T pzm = e > 0 ? p0.e[e - 1] : cur.zme;
            const T pzp = e < V - 1 ? p0.e[e + 1] : cur.zpe;
            const bool ez = (ezm >> e) & 1u;
            T lap = 0.0f, sn = 0.0f, so = 0.0f;
            if constexpr (EX) {
                const T l0 = vxl.e[e], r0 = cur.vxr.e[e];
                const T vl = ((fxl >> e) & 1u) ? vel_update<T>(l0, cxl.vupd, cxl.vgrad, pz, pm.e[e]) : l0;
                const T vr = ((fxr >> e) & 1u) ? vel_update<T>(r0, cur.cxr.vupd, cur.cxr.vgrad, cur.pp.e[e], pz) : r0;
                nxl.e[e] = vl;
                nxr.e[e] = vr;
                const T a = pd_update<T>(cur.a0.e[e], cxl.pupd, cxl.pdiv, vr, vl, inv_h);
                o0.e[e] = a;
                sn = a;
                so = cur.a0.e[e];
            } else {
                lap = lap + (cur.pp.e[e] + pm.e[e] - 2.0f * pz);
            }
            if constexpr (EY) {
                const T l0 = cur.vyl.e[e], r0 = cur.vyr.e[e];
                const T vl = ((fyl >> e) & 1u) ? vel_update<T>(l0, cyl.vupd, cyl.vgrad, pz, cur.ym.e[e]) : l0;
                const T vr = ((fyr >> e) & 1u) ? vel_update<T>(r0, cyr.vupd, cyr.vgrad, cur.yp.e[e], pz) : r0;
                nyl.e[e] = vl;
                nyr.e[e] = vr;
                const T a = pd_update<T>(cur.a1.e[e], cyl.pupd, cyl.pdiv, vr, vl, inv_h);
                o1.e[e] = a;
                sn = sn + a;
                so = so + cur.a1.e[e];
            } else {
                lap = lap + (cur.yp.e[e] + cur.ym.e[e] - 2.0f * pz);
            }
            T az = 0.0f;
            if (ez) {
                const T l0 = cur.vzl.e[e], r0 = e < V - 1 ? cur.vzl.e[e + 1] : cur.vze;
                const T vl = ((fzl >> e) & 1u) ? vel_update<T>(l0, cz[e].vupd, cz[e].vgrad, pz, pzm) : l0;
                const T vr = ((fzr >> e) & 1u) ? vel_update<T>(r0, cz[e + 1].vupd, cz[e + 1].vgrad, pzp, pz) : r0;
                nzl.e[e] = vl;
                nzr[e] = vr;
                az = pd_update<T>(cur.a2.e[e], cz[e].pupd, cz[e].pdiv, vr, vl, inv_h);
                sn = sn + az;
                so = so + cur.a2.e[e];
            } else {
                nzl.e[e] = 0.0f;
                nzr[e] = 0.0f;
                lap = lap + (pzp + pzm - 2.0f * pz);
            }
            // the increment of the plain axes (none for a corner cell)
            const T qold = EX ? (EY ? cur.a2.e[e] : cur.a1.e[e]) : cur.a0.e[e];
            const T qn = fmaf(lap * ls, c2k2, qold);
            const bool plain = !(EX && EY && ez);
            pn.e[e] = (sn + (pz - so)) + (plain ? qn : 0.0f);
            if constexpr (!EX) o0.e[e] = qn;
            if constexpr (EX && !EY) o1.e[e] = qn;
            o2.e[e] = ez ? az : qn;
        }
        if constexpr (EX) {
            st_masked<T, V>(A.vn[0] + c, nxl, m_xl);
            st_masked<T, V>(A.vn[0] + c + sx, nxr, m_xr);
        }
        if constexpr (EY) {
            st_masked<T, V>(A.vn[1] + c, nyl, m_yl);
            st_masked<T, V>(A.vn[1] + c + sy, nyr, m_yr);
        }
        st_masked<T, V>(vzn + q, nzl, m_zl);
        if (m_zr) {
#pragma unroll
            for (int e = 0; e < V; ++e)
                if ((m_zr >> e) & 1u) vzn[q + ((e == V - 1 && spare) ? spare : e + 1)] = nzr[e];
        }
        st_masked<T, V>(pdst[0] + q, o0, inbox);
        if constexpr (KIND != 2) st_masked<T, V>(pdst[1] + q, o1, m_a1);
        st_masked<T, V>(pdst[2] + q, o2, m_a2);
        st_masked<T, V>(A.pn + c, pn, inbox);
        // carry to plane x+1
        pm = p0;
        p0 = cur.pp;
        if constexpr (EX) {
            vxl = cur.vxr;
            cxl = cur.cxr;
        }
        if constexpr (NS == 0 && PF) cur = nxt;
    }
    if constexpr (NS > 0) cpa_wait<0>();  // no copy outlives the thread
}

// Box kind: the z-slab pair is B.zbox; an x slab absorbs along x on its first
// plane; otherwise a y slab.  Uniform per CTA except EY (per row).
__device__ __forceinline__ void shell_tile_red(const KArgs<float>& A, const ShellBoxes& B, int b, int tu, int tx) {
    const int u = tu * 256 + threadIdx.x + 32 * threadIdx.y;
    if (u >= B.ny[b] * B.ng[b]) return;
    // columns with two absorbing axes hold more state per plane: they load one
    // plane at a time (PF_EY), the others issue the next plane's loads first
    constexpr bool PF = FDTD_SHELL_RED_PREFETCH != 0, PF_EY = FDTD_SHELL_RED_PREFETCH == 2;
    // (B.zp is uniform per CTA: the plain-z boxes take their own path without divergence)
    if (b == B.zbox) {
        shell_tile_red_impl<2, false, PF>(A, B, b, u, tx);
    } else if (__ldg(A.axflag[0] + B.x0[b]) & AXF_PML) {
        const int y = B.y0[b] + u / B.ng[b];
        if (__ldg(A.axflag[1] + y) & AXF_PML) {
            if (B.zp[b]) shell_tile_red_impl<0, true, PF_EY, true>(A, B, b, u, tx);
            else shell_tile_red_impl<0, true, PF_EY>(A, B, b, u, tx);
        } else {
            if (B.zp[b]) shell_tile_red_impl<0, false, PF, true>(A, B, b, u, tx);
            else shell_tile_red_impl<0, false, PF>(A, B, b, u, tx);
        }
    } else if (B.zp[b]) {
        shell_tile_red_impl<1, true, PF_EY, true>(A, B, b, u, tx);
    } else {
        shell_tile_red_impl<1, true, PF_EY>(A, B, b, u, tx);
    }
}

// (a template so that every translation unit may include it; instantiated for float only)
template <typename T>
__global__ void __launch_bounds__(256, FDTD_SHELL_RED_MINB) k_pml_shell_red(const KArgs<T> A, const ShellBoxes B) {
    static_assert(sizeof(T) == 4, "the reduced PML state is an FP32 path");
    if (A.advance && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) advance_consts(*A.P, A.cur);
    int b, tu, tx;
    shell_decode(B, blockIdx.x, b, tu, tx);
    shell_tile_red(A, B, b, tu, tx);
}

}  // namespace fdtd
