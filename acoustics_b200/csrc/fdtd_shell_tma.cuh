// fdtd_shell_tma.cuh — PML shell of FP32 solves on the reduced PML state with
// tensor-memory-accelerator (TMA) staging of every load.
//
// The arithmetic per cell is that of shell_tile_red_impl (fdtd_shell_red.cuh),
// in the same order, so the two kernels give the same bits; what changes is how
// the operands reach the threads.  A CTA of 128 threads owns one tile of the
// shell: TY rows x TZ cells of a (y, z) window, four consecutive z cells per
// thread, and marches along x over the tile's planes.  Per x plane one thread
// issues 3-D bulk tensor copies (cp.async.bulk.tensor, this GPU's memory only,
// no multicast) of every array the tile reads into one stage of a 4-stage
// shared-memory ring, completed on that stage's mbarrier:
//   P   p^n with a one-cell halo in y and a four-cell halo in z (z stays a
//       multiple of 4: the copy's innermost coordinate is 16-byte aligned;
//       halo cells outside the grid read as zeros and are never used)
//   VX  x faces of the plane (x slabs), VY the TY+1 y faces of its rows,
//   VZ  the TZ+4 z faces of its rows, A0..A2 the reduced split state.
// At plane x the threads read P of x-1, x, x+1 and the faces of x and x+1 from
// the ring: no per-thread address, clamp or predicate work for loads, each p
// value crosses L2 -> SM about 1.4 times instead of 5.  Results are stored
// from registers with 16-byte vector stores.  All storage is the grid's
// (the z slabs too: a tile window reads their 16-cell rows as 3-D boxes).
//
// Tiles (host side, build_tma_tiles): x slabs and y slabs in TZ0 x TY0 = 64 x 8
// windows, z slabs in TZ1 x TY1 windows (TZ1 = the slab width rounded up to a
// power of two, TY1 = 512 / TZ1); each tile covers at most 16 x planes.
// Every wait on an mbarrier is bounded: after about a second without
// completion the kernel records FDTD_DEV_ERR_TMA_TIMEOUT, waits (bounded) for
// its copies still in flight and returns.
#pragma once

#include "fdtd_tma.hpp"

namespace fdtd {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false after ~2^22 polls (each poll may suspend the thread for a
// while inside try_wait), about a second
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// Copies of ring stage j (plane x0 - 1 + j): P always; the x faces of planes
// x0..x0+nx (x slabs); the other arrays of planes x0..x0+nx-1.
__device__ __forceinline__ void tma_issue_stage(const TmaMaps& M, const TmaShape& S, int sh, const TmaTile& T,
                                                uint32_t stage, uint32_t bar, int j) {
    const int xs = T.x0 - 1 + j;
    const bool state = j >= 1 && j <= T.nx;
    const bool vx = T.kind == 0 && j >= 1 && j <= T.nx + 1;
    const bool vy = state && (T.flags & TT_VY);
    const bool vz = state && (T.flags & TT_VZ);
    const bool a1 = state && T.kind != 2;
    const bool a2 = state && (T.flags & TT_A2);
    uint32_t bytes = S.bytes[TB_P];
    if (vx) bytes += S.bytes[TB_VX];
    if (vy) bytes += S.bytes[TB_VY];
    if (vz) bytes += S.bytes[TB_VZ];
    if (state) bytes += S.bytes[TB_A0];
    if (a1) bytes += S.bytes[TB_A1];
    if (a2) bytes += S.bytes[TB_A2];
    mbar_expect_tx(bar, bytes);
    const CUtensorMap* m = M.m[sh];
    tma_load_3d(stage + S.off[TB_P], &m[TB_P], T.z0 - 4, T.y0 - 1, xs, bar);
    if (vx) tma_load_3d(stage + S.off[TB_VX], &m[TB_VX], T.z0, T.y0, xs, bar);
    if (vy) tma_load_3d(stage + S.off[TB_VY], &m[TB_VY], T.z0, T.y0, xs, bar);
    if (vz) tma_load_3d(stage + S.off[TB_VZ], &m[TB_VZ], T.z0, T.y0, xs, bar);
    if (state) tma_load_3d(stage + S.off[TB_A0], &m[TB_A0], T.z0, T.y0, xs, bar);
    if (a1) tma_load_3d(stage + S.off[TB_A1], &m[TB_A1], T.z0, T.y0, xs, bar);
    if (a2) tma_load_3d(stage + S.off[TB_A2], &m[TB_A2], T.z0, T.y0, xs, bar);
}

template <int V>
__device__ __forceinline__ Vec<float, V> lds(const unsigned char* base, int elem) {
    return *reinterpret_cast<const Vec<float, V>*>(base + 4 * elem);
}

// One plane of one thread's four cells.  KIND / EY as in shell_tile_red_impl;
// sM, s0, sP: the ring stages of planes x-1, x, x+1.
template <int KIND, bool EY>
__device__ __forceinline__ void tma_plane(const KArgs<float>& A, const TmaShape& S, const unsigned char* sM,
                                          const unsigned char* s0, const unsigned char* sP, int x, int y, int r,
                                          int zc, int lz, unsigned inbox, uint8_t gy, const unsigned (&zm)[6],
                                          const AxisCoef<float> (&cz)[5], const AxisCoef<float>& cyl,
                                          const AxisCoef<float>& cyr) {
    using T = float;
    constexpr int V = 4;
    constexpr unsigned ALL = 0xFu;
    constexpr bool EX = KIND == 0;
    using VT = Vec<T, V>;
    const int tz = S.tz;
    const int pw = tz + 8;                       // P row width
    const int pc = (r + 1) * pw + lz + 4;        // this thread's cells in P
    const unsigned zpml = zm[0], zflo = zm[1], zfhi = zm[2], znext = zm[3], zhlo = zm[4], zhhi = zm[5];
    const unsigned ezm = zpml & inbox;
    const unsigned mpy = (gy & AXF_PML) ? ALL : 0u;
    const unsigned mpx = EX ? ALL : 0u;
    const unsigned fyl = ((gy & AXF_FACE_LO) ? ALL : 0u) | ((gy & AXF_HAS_LO) ? (mpx | zpml) : 0u);
    const unsigned fyr = ((gy & AXF_FACE_HI) ? ALL : 0u) | ((gy & AXF_HAS_HI) ? (mpx | zpml) : 0u);
    const unsigned fzl = zflo | (zhlo & (mpx | mpy));
    const unsigned fzr = zfhi | (zhhi & (mpx | mpy));
    const unsigned m_yl = EY ? inbox & fyl : 0u;
    const unsigned m_yr = EY ? inbox & fyr & ((gy & AXF_NEXT_PML) ? 0u : ALL) : 0u;
    const unsigned m_zl = ezm & fzl;
    const unsigned m_zr = ezm & fzr & ~znext;
    const unsigned m_a1 = KIND == 2 ? 0u : inbox;
    const unsigned m_a2 = (KIND == 0 && EY) ? inbox : ezm;

    const unsigned char* P0 = s0 + S.off[TB_P];
    const VT p0 = lds<V>(P0, pc);
    const VT pm = lds<V>(sM + S.off[TB_P], pc);
    const VT pp = lds<V>(sP + S.off[TB_P], pc);
    const VT ym = lds<V>(P0, pc - pw);
    const VT yp = lds<V>(P0, pc + pw);
    const T zme = *reinterpret_cast<const T*>(P0 + 4 * (pc - 1));
    const T zpe = *reinterpret_cast<const T*>(P0 + 4 * (pc + V));
    const int ai = r * tz + lz;                 // this thread's cells in the TZ-wide buffers
    VT vxl, vxr, vyl, vyr, vzl, a0, a1, a2;
    T vze = 0.0f;
    AxisCoef<T> cxl, cxr;
    uint8_t g = 0;
    if constexpr (EX) {
        vxl = lds<V>(s0 + S.off[TB_VX], ai);
        vxr = lds<V>(sP + S.off[TB_VX], ai);
        g = __ldg(A.axflag[0] + x);
        cxl = A.coef[0][x];
        cxr = A.coef[0][x + 1];
    }
    if constexpr (EY) {
        vyl = lds<V>(s0 + S.off[TB_VY], ai);
        vyr = lds<V>(s0 + S.off[TB_VY], ai + tz);
    }
    if (ezm) {
        const int zi = r * (tz + 4) + lz;
        vzl = lds<V>(s0 + S.off[TB_VZ], zi);
        vze = *reinterpret_cast<const T*>(s0 + S.off[TB_VZ] + 4 * (zi + V));
    }
    a0 = lds<V>(s0 + S.off[TB_A0], ai);
    if constexpr (KIND != 2) a1 = lds<V>(s0 + S.off[TB_A1], ai);
    if ((KIND == 0 && EY) || ezm) a2 = lds<V>(s0 + S.off[TB_A2], ai);

    unsigned fxl = 0, fxr = 0, m_xl = 0, m_xr = 0;
    if constexpr (EX) {
        const unsigned oyz = mpy | zpml;
        fxl = ((g & AXF_FACE_LO) ? ALL : 0u) | ((g & AXF_HAS_LO) ? oyz : 0u);
        fxr = ((g & AXF_FACE_HI) ? ALL : 0u) | ((g & AXF_HAS_HI) ? oyz : 0u);
        m_xl = inbox & fxl;
        m_xr = inbox & fxr & ((g & AXF_NEXT_PML) ? 0u : ALL);
    }
    const float ls = A.lap_scale, c2k2 = A.c2k2, inv_h = A.inv_h;
    VT nxl, nxr, nyl, nyr, nzl, o0, o1, o2, pn;
    T nzr[V];
#pragma unroll
    for (int e = 0; e < V; ++e) {
        const T pz = p0.e[e];
        const T pzm = e > 0 ? p0.e[e - 1] : zme;
        const T pzp = e < V - 1 ? p0.e[e + 1] : zpe;
        const bool ez = (ezm >> e) & 1u;
        T lap = 0.0f, sn = 0.0f, so = 0.0f;
        if constexpr (EX) {
            const T l0 = vxl.e[e], r0 = vxr.e[e];
            const T vl = ((fxl >> e) & 1u) ? vel_update<T>(l0, cxl.vupd, cxl.vgrad, pz, pm.e[e]) : l0;
            const T vr = ((fxr >> e) & 1u) ? vel_update<T>(r0, cxr.vupd, cxr.vgrad, pp.e[e], pz) : r0;
            nxl.e[e] = vl;
            nxr.e[e] = vr;
            const T a = pd_update<T>(a0.e[e], cxl.pupd, cxl.pdiv, vr, vl, inv_h);
            o0.e[e] = a;
            sn = a;
            so = a0.e[e];
        } else {
            lap = lap + (pp.e[e] + pm.e[e] - 2.0f * pz);
        }
        if constexpr (EY) {
            const T l0 = vyl.e[e], r0 = vyr.e[e];
            const T vl = ((fyl >> e) & 1u) ? vel_update<T>(l0, cyl.vupd, cyl.vgrad, pz, ym.e[e]) : l0;
            const T vr = ((fyr >> e) & 1u) ? vel_update<T>(r0, cyr.vupd, cyr.vgrad, yp.e[e], pz) : r0;
            nyl.e[e] = vl;
            nyr.e[e] = vr;
            const T a = pd_update<T>(a1.e[e], cyl.pupd, cyl.pdiv, vr, vl, inv_h);
            o1.e[e] = a;
            sn = sn + a;
            so = so + a1.e[e];
        } else {
            lap = lap + (yp.e[e] + ym.e[e] - 2.0f * pz);
        }
        T az = 0.0f;
        if (ez) {
            const T l0 = vzl.e[e], r0 = e < V - 1 ? vzl.e[e + 1] : vze;
            const T vl = ((fzl >> e) & 1u) ? vel_update<T>(l0, cz[e].vupd, cz[e].vgrad, pz, pzm) : l0;
            const T vr = ((fzr >> e) & 1u) ? vel_update<T>(r0, cz[e + 1].vupd, cz[e + 1].vgrad, pzp, pz) : r0;
            nzl.e[e] = vl;
            nzr[e] = vr;
            az = pd_update<T>(a2.e[e], cz[e].pupd, cz[e].pdiv, vr, vl, inv_h);
            sn = sn + az;
            so = so + a2.e[e];
        } else {
            nzl.e[e] = 0.0f;
            nzr[e] = 0.0f;
            lap = lap + (pzp + pzm - 2.0f * pz);
        }
        const T qold = EX ? (EY ? a2.e[e] : a1.e[e]) : a0.e[e];
        const T qn = fmaf(lap * ls, c2k2, qold);
        const bool plain = !(EX && EY && ez);
        pn.e[e] = (sn + (pz - so)) + (plain ? qn : 0.0f);
        if constexpr (!EX) o0.e[e] = qn;
        if constexpr (EX && !EY) o1.e[e] = qn;
        o2.e[e] = ez ? az : qn;
    }
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned c = (unsigned)x * A.sx + (unsigned)y * A.sy + zc;
    if constexpr (EX) {
        st_masked<T, V>(A.vn[0] + c, nxl, m_xl);
        st_masked<T, V>(A.vn[0] + c + sx, nxr, m_xr);
    }
    if constexpr (EY) {
        st_masked<T, V>(A.vn[1] + c, nyl, m_yl);
        st_masked<T, V>(A.vn[1] + c + sy, nyr, m_yr);
    }
    st_masked<T, V>(A.vn[2] + c, nzl, m_zl);
    if (m_zr) {
#pragma unroll
        for (int e = 0; e < V; ++e)
            if ((m_zr >> e) & 1u) A.vn[2][c + e + 1] = nzr[e];
    }
    st_masked<T, V>(A.pd[0] + c, o0, inbox);
    if constexpr (KIND != 2) st_masked<T, V>(A.pd[1] + c, o1, m_a1);
    st_masked<T, V>(A.pd[2] + c, o2, m_a2);
    st_masked<T, V>(A.pn + c, pn, inbox);
}

// (a template so that every translation unit may include it; instantiated for float only)
template <typename TT>
__global__ void __launch_bounds__(TMA_THREADS, 3)
    k_pml_shell_tma(const KArgs<TT> A, const __grid_constant__ TmaMaps M, const TmaLaunch Lc,
                    const TmaTile* __restrict__ tiles, int* __restrict__ dev_error) {
    static_assert(sizeof(TT) == 4, "the reduced PML state is an FP32 path");
    // the ring: TMA_STAGES stages of Lc.stage_bytes, then one mbarrier per stage
    extern __shared__ __align__(128) unsigned char tma_ring[];
    uint64_t* full = reinterpret_cast<uint64_t*>(tma_ring + TMA_STAGES * Lc.stage_bytes);
    if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) advance_consts(*A.P, A.cur);
    const TmaTile T = tiles[blockIdx.x];
    const int sh = T.kind == 2 ? 1 : 0;
    const TmaShape& S = Lc.shape[sh];
    const int tid = threadIdx.x;
    const uint32_t ring = smem_u32(tma_ring);
    // tensor copies land on 128-byte boundaries (every buffer size is a multiple of 128)
    if (ring & 127u) {
        if (tid == 0) atomicOr(dev_error, FDTD_DEV_ERR_TMA_TIMEOUT);
        return;
    }
    const int nst = T.nx + 2;  // stages of the tile (planes x0-1 .. x0+nx)
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < TMA_STAGES; ++s) mbar_init(smem_u32(&full[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0)
        for (int j = 0; j < TMA_STAGES && j < nst; ++j)
            tma_issue_stage(M, S, sh, T, ring + j * Lc.stage_bytes, smem_u32(&full[j]), j);

    // this thread's cells: row r of the window, z group lz .. lz+3
    const int gpr = S.tz / 4;
    const int r = tid / gpr;
    const int lz = (tid - r * gpr) * 4;
    const int zc = T.z0 + lz;
    const int y = T.y0 + (r < T.ny ? r : T.ny - 1);
    const bool row_on = r < T.ny && r < S.ty;
    unsigned inbox = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) inbox |= (row_on && zc + e >= T.zlo && zc + e < T.zhi ? 1u : 0u) << e;
    const uint8_t gy = __ldg(A.axflag[1] + y);
    unsigned zm[6];
    {
        uint8_t gz[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) gz[e] = zc + e < A.N2 ? __ldg(A.axflag[2] + zc + e) : (uint8_t)0;
#pragma unroll
        for (int k = 0; k < 6; ++k) zm[k] = flag_mask<4>(gz, k);
    }
    AxisCoef<float> cz[5];
    if (zm[0] & inbox) {
#pragma unroll
        for (int e = 0; e <= 4; ++e) cz[e] = A.coef[2][zc + e];
    }
    AxisCoef<float> cyl{}, cyr{};
    const bool ey = T.kind == 1 || (T.kind == 0 && (gy & AXF_PML));
    if (ey) {
        cyl = A.coef[1][y];
        cyr = A.coef[1][y + 1];
    }

    // stages 0..waited-1 have arrived; 0..issued-1 were issued
    bool ok = true;
    int waited = 0;
    for (int j = 0; j < 2 && j < nst; ++j) {
        if (ok) ok = mbar_wait(smem_u32(&full[j]), 0);
        if (ok) waited = j + 1;
    }
    int issued = nst < TMA_STAGES ? nst : TMA_STAGES;
    bool fail = false;
    for (int i = 0; i < T.nx; ++i) {
        const int jn = i + 2;  // stage of plane x+1
        if (ok && jn < nst) {
            ok = mbar_wait(smem_u32(&full[jn % TMA_STAGES]), (jn / TMA_STAGES) & 1);
            if (ok) waited = jn + 1;
        }
        const int x = T.x0 + i;
        const unsigned char* sM = tma_ring + (i % TMA_STAGES) * Lc.stage_bytes;
        const unsigned char* s0 = tma_ring + ((i + 1) % TMA_STAGES) * Lc.stage_bytes;
        const unsigned char* sP = tma_ring + (jn % TMA_STAGES) * Lc.stage_bytes;
        // (after a failed wait the plane is computed from whatever the stage
        // holds, in bounds, and the solve reports the error)
        if (inbox) {
            if (T.kind == 2) tma_plane<2, false>(A, S, sM, s0, sP, x, y, r, zc, lz, inbox, gy, zm, cz, cyl, cyr);
            else if (T.kind == 1) tma_plane<1, true>(A, S, sM, s0, sP, x, y, r, zc, lz, inbox, gy, zm, cz, cyl, cyr);
            else if (ey) tma_plane<0, true>(A, S, sM, s0, sP, x, y, r, zc, lz, inbox, gy, zm, cz, cyl, cyr);
            else tma_plane<0, false>(A, S, sM, s0, sP, x, y, r, zc, lz, inbox, gy, zm, cz, cyl, cyr);
        }
        // every thread is done with the stage of plane x-1 (and all waits held)
        if (__syncthreads_or(!ok)) {
            fail = true;
            break;
        }
        const int jf = i + TMA_STAGES;
        if (jf < nst) {
            if (tid == 0)
                tma_issue_stage(M, S, sh, T, ring + (jf % TMA_STAGES) * Lc.stage_bytes,
                                smem_u32(&full[jf % TMA_STAGES]), jf);
            issued = jf + 1;
        }
    }
    if (fail && tid == 0) {
        atomicOr(dev_error, FDTD_DEV_ERR_TMA_TIMEOUT);
        // wait (bounded) for the copies this CTA still has in flight
        for (int j = waited; j < issued; ++j) (void)mbar_wait(smem_u32(&full[j % TMA_STAGES]), (j / TMA_STAGES) & 1);
    }
}

}  // namespace fdtd
