// fdtd_shell_tma.cuh — PML shell of FP32 solves on the reduced PML state with
// tensor-memory-accelerator (TMA) staging of every load.
//
// The arithmetic per cell is that of shell_tile_red_impl (fdtd_shell_red.cuh),
// in the same order, so the two kernels give the same bits; what changes is how
// the work is cut and how the operands reach the threads.
//
// Tiles.  The shell is cut by absorbing axes: every tile holds cells that
// absorb along the same axes (x only, y only, z only, the three edges' pairs,
// the corners), so the update of a tile is one of seven specialised bodies
// with no per-cell axis tests, and a tile stages only the arrays its axes use.
// A CTA of 128 threads owns one tile: ty rows x tz cells of a (y, z) window
// (four consecutive z cells per thread), marching along x over at most 16
// planes.  Window shapes follow the extents of the tile class (a z-PML window
// is as wide as the z slab, y-slab tiles as high as the y slab), so the copies
// carry few cells outside the shell.
//
// Staging.  The kernel is persistent: a CTA walks a list of tiles (balanced on
// the host by their bytes).  A producer warp issues, per x plane, 3-D bulk
// tensor copies (cp.async.bulk.tensor, tensor maps in device memory describing
// this GPU's arrays, no multicast) of every array the tile reads into one stage
// of a TMA_STAGES-deep shared-memory ring, completed on the stage's "full"
// mbarrier; the stage sequence runs on across tiles, so the ring never drains
// between them.  Four consumer warps compute; each releases a stage on its
// "empty" mbarrier when done with it, and the producer refills it then.
//   P   p^n with a one-cell halo in y and a four-cell halo in z (z stays a
//       multiple of 4: the copy's innermost coordinate is 16-byte aligned;
//       halo cells outside the grid read as zeros and are never used)
//   VX  x faces of the plane, VY the ty+1 y faces of its rows, VZ the tz+4 z
//       faces of its rows, A0..A2 the reduced split state.
// At plane x the threads read P of x-1, x, x+1 and the faces of x and x+1 from
// the ring and store their results from registers with 16-byte vector stores.
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
// bounded wait: false after 2^22 polls (each poll may suspend the thread for a
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
// x0..x0+nx (tiles absorbing along x); the other arrays of planes x0..x0+nx-1.
__device__ __forceinline__ void tma_issue_stage(const CUtensorMap* m, const TmaShape& S, const TmaTile& T,
                                                uint32_t stage, uint32_t bar, int j) {
    const int xs = T.x0 - 1 + j;
    const bool ex = T.cls & TC_X, ey = T.cls & TC_Y, ez = T.cls & TC_Z;
    const bool state = j >= 1 && j <= T.nx;
    const bool vx = ex && j >= 1 && j <= T.nx + 1;
    const bool vy = state && ey;
    const bool vz = state && ez;
    const bool a1 = state && (ex || ey);
    const bool a2 = state && (ez || (ex && ey));
    uint32_t bytes = S.bytes[TB_P];
    if (vx) bytes += S.bytes[TB_VX];
    if (vy) bytes += S.bytes[TB_VY];
    if (vz) bytes += S.bytes[TB_VZ];
    if (state) bytes += S.bytes[TB_A0];
    if (a1) bytes += S.bytes[TB_A1];
    if (a2) bytes += S.bytes[TB_A2];
    mbar_expect_tx(bar, bytes);
    tma_load_3d(stage + S.off[TB_P], &m[TB_P], T.z0 - 4, T.y0 - 1, xs, bar);
    if (vx) tma_load_3d(stage + S.off[TB_VX], &m[TB_VX], T.z0, T.y0, xs, bar);
    if (vy) tma_load_3d(stage + S.off[TB_VY], &m[TB_VY], T.z0, T.y0, xs, bar);
    if (vz) tma_load_3d(stage + S.off[TB_VZ], &m[TB_VZ], T.z0, T.y0, xs, bar);
    if (state) tma_load_3d(stage + S.off[TB_A0], &m[TB_A0], T.z0, T.y0, xs, bar);
    if (a1) tma_load_3d(stage + S.off[TB_A1], &m[TB_A1], T.z0, T.y0, xs, bar);
    if (a2) tma_load_3d(stage + S.off[TB_A2], &m[TB_A2], T.z0, T.y0, xs, bar);
}

__device__ __forceinline__ Vec<float, 4> lds4(const unsigned char* base, int elem) {
    return *reinterpret_cast<const Vec<float, 4>*>(base + 4 * elem);
}
__device__ __forceinline__ float lds1(const unsigned char* base, int elem) {
    return *reinterpret_cast<const float*>(base + 4 * elem);
}

// Per-thread constants of a tile: its cells and their flags and coefficients.
struct TmaThread {
    int r, lz, zc, y;
    unsigned inbox;              // cells of the box among the four
    uint8_t gy;                  // y flags of the row
    unsigned zm[6];              // z flag bits of the four cells (flag_mask)
    AxisCoef<float> cz[5];       // z coefficients of the cells and the next face (EZ)
    AxisCoef<float> cyl, cyr;    // y coefficients of the row (EY)
};

// One plane of one thread's four cells, for a tile absorbing along EX / EY / EZ.
// sM, s0, sP: the ring stages of planes x-1, x, x+1.
template <bool EX, bool EY, bool EZ>
__device__ __forceinline__ void tma_plane(const KArgs<float>& A, const TmaShape& S, const unsigned char* sM,
                                          const unsigned char* s0, const unsigned char* sP, int x,
                                          const TmaThread& H) {
    using T = float;
    constexpr int V = 4;
    constexpr unsigned ALL = 0xFu;
    using VT = Vec<T, V>;
    const int tz = S.tz;
    const int pw = tz + 8;                      // P row width
    const int pc = (H.r + 1) * pw + H.lz + 4;   // this thread's cells in P
    const unsigned inbox = H.inbox;
    // masks of the face rules (as in shell_tile_red_impl; the axis sets are the tile's)
    const unsigned zpml = EZ ? ALL : 0u;
    const unsigned mpx = EX ? ALL : 0u, mpy = EY ? ALL : 0u;
    const unsigned ezm = EZ ? inbox : 0u;

    const unsigned char* P0 = s0 + S.off[TB_P];
    const VT p0 = lds4(P0, pc);
    const VT pm = lds4(sM + S.off[TB_P], pc);
    const VT pp = lds4(sP + S.off[TB_P], pc);
    const VT ym = lds4(P0, pc - pw);
    const VT yp = lds4(P0, pc + pw);
    const T zme = lds1(P0, pc - 1);
    const T zpe = lds1(P0, pc + V);
    const int ai = H.r * tz + H.lz;             // this thread's cells in the tz-wide buffers
    VT vxl, vxr, vyl, vyr, vzl, a0, a1, a2;
    T vze = 0.0f;
    AxisCoef<T> cxl, cxr;
    unsigned fxl = 0, fxr = 0, m_xl = 0, m_xr = 0;
    if constexpr (EX) {
        vxl = lds4(s0 + S.off[TB_VX], ai);
        vxr = lds4(sP + S.off[TB_VX], ai);
        const uint8_t g = __ldg(A.axflag[0] + x);
        cxl = A.coef[0][x];
        cxr = A.coef[0][x + 1];
        const unsigned oyz = mpy | zpml;
        fxl = ((g & AXF_FACE_LO) ? ALL : 0u) | ((g & AXF_HAS_LO) ? oyz : 0u);
        fxr = ((g & AXF_FACE_HI) ? ALL : 0u) | ((g & AXF_HAS_HI) ? oyz : 0u);
        m_xl = inbox & fxl;
        m_xr = inbox & fxr & ((g & AXF_NEXT_PML) ? 0u : ALL);
    }
    unsigned fyl = 0, fyr = 0, m_yl = 0, m_yr = 0;
    if constexpr (EY) {
        vyl = lds4(s0 + S.off[TB_VY], ai);
        vyr = lds4(s0 + S.off[TB_VY], ai + tz);
        const uint8_t gy = H.gy;
        fyl = ((gy & AXF_FACE_LO) ? ALL : 0u) | ((gy & AXF_HAS_LO) ? (mpx | zpml) : 0u);
        fyr = ((gy & AXF_FACE_HI) ? ALL : 0u) | ((gy & AXF_HAS_HI) ? (mpx | zpml) : 0u);
        m_yl = inbox & fyl;
        m_yr = inbox & fyr & ((gy & AXF_NEXT_PML) ? 0u : ALL);
    }
    unsigned fzl = 0, fzr = 0, m_zl = 0, m_zr = 0;
    if constexpr (EZ) {
        const int zi = H.r * (tz + 4) + H.lz;
        vzl = lds4(s0 + S.off[TB_VZ], zi);
        vze = lds1(s0 + S.off[TB_VZ], zi + V);
        fzl = H.zm[1] | (H.zm[4] & (mpx | mpy));
        fzr = H.zm[2] | (H.zm[5] & (mpx | mpy));
        m_zl = ezm & fzl;
        m_zr = ezm & fzr & ~H.zm[3];
    }
    a0 = lds4(s0 + S.off[TB_A0], ai);
    if constexpr (EX || EY) a1 = lds4(s0 + S.off[TB_A1], ai);
    if constexpr (EZ || (EX && EY)) a2 = lds4(s0 + S.off[TB_A2], ai);

    const float ls = A.lap_scale, c2k2 = A.c2k2, inv_h = A.inv_h;
    VT nxl, nxr, nyl, nyr, nzl, o0, o1, o2, pn;
    T nzr[V];
#pragma unroll
    for (int e = 0; e < V; ++e) {
        const T pz = p0.e[e];
        const T pzm = e > 0 ? p0.e[e - 1] : zme;
        const T pzp = e < V - 1 ? p0.e[e + 1] : zpe;
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
            const T vl = ((fyl >> e) & 1u) ? vel_update<T>(l0, H.cyl.vupd, H.cyl.vgrad, pz, ym.e[e]) : l0;
            const T vr = ((fyr >> e) & 1u) ? vel_update<T>(r0, H.cyr.vupd, H.cyr.vgrad, yp.e[e], pz) : r0;
            nyl.e[e] = vl;
            nyr.e[e] = vr;
            const T a = pd_update<T>(a1.e[e], H.cyl.pupd, H.cyl.pdiv, vr, vl, inv_h);
            o1.e[e] = a;
            sn = sn + a;
            so = so + a1.e[e];
        } else {
            lap = lap + (yp.e[e] + ym.e[e] - 2.0f * pz);
        }
        T az = 0.0f;
        if constexpr (EZ) {
            const T l0 = vzl.e[e], r0 = e < V - 1 ? vzl.e[e + 1] : vze;
            const T vl = ((fzl >> e) & 1u) ? vel_update<T>(l0, H.cz[e].vupd, H.cz[e].vgrad, pz, pzm) : l0;
            const T vr = ((fzr >> e) & 1u) ? vel_update<T>(r0, H.cz[e + 1].vupd, H.cz[e + 1].vgrad, pzp, pz) : r0;
            nzl.e[e] = vl;
            nzr[e] = vr;
            az = pd_update<T>(a2.e[e], H.cz[e].pupd, H.cz[e].pdiv, vr, vl, inv_h);
            sn = sn + az;
            so = so + a2.e[e];
        } else {
            lap = lap + (pzp + pzm - 2.0f * pz);
        }
        if constexpr (EX && EY && EZ) {
            // a corner cell has no plain axis
            pn.e[e] = (sn + (pz - so)) + 0.0f;
            o2.e[e] = az;
        } else {
            // the increment of the plain axes
            const T qold = EX ? (EY ? a2.e[e] : a1.e[e]) : a0.e[e];
            const T qn = fmaf(lap * ls, c2k2, qold);
            pn.e[e] = (sn + (pz - so)) + qn;
            if constexpr (!EX) o0.e[e] = qn;
            if constexpr (EX && !EY) o1.e[e] = qn;
            o2.e[e] = EZ ? az : qn;
        }
    }
    const int sx = (int)A.sx, sy = (int)A.sy;
    const unsigned c = (unsigned)x * A.sx + (unsigned)H.y * A.sy + H.zc;
    if constexpr (EX) {
        st_masked<T, V>(A.vn[0] + c, nxl, m_xl);
        st_masked<T, V>(A.vn[0] + c + sx, nxr, m_xr);
    }
    if constexpr (EY) {
        st_masked<T, V>(A.vn[1] + c, nyl, m_yl);
        st_masked<T, V>(A.vn[1] + c + sy, nyr, m_yr);
    }
    if constexpr (EZ) {
        st_masked<T, V>(A.vn[2] + c, nzl, m_zl);
        if (m_zr) {
#pragma unroll
            for (int e = 0; e < V; ++e)
                if ((m_zr >> e) & 1u) A.vn[2][c + e + 1] = nzr[e];
        }
    }
    st_masked<T, V>(A.pd[0] + c, o0, inbox);
    if constexpr (EX || EY) st_masked<T, V>(A.pd[1] + c, o1, inbox);
    if constexpr (EZ || (EX && EY)) st_masked<T, V>(A.pd[2] + c, o2, inbox);
    st_masked<T, V>(A.pn + c, pn, inbox);
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// Consumer side of one tile: its planes, reading the stages g0 .. g0+nx+1 of
// the CTA's global stage sequence; every consumer warp releases each stage once
// it no longer needs it.  False when a stage did not arrive within its bounded wait.
template <bool EX, bool EY, bool EZ>
__device__ __forceinline__ bool tma_tile(const KArgs<float>& A, const TmaShape& S, const TmaTile& T,
                                         unsigned char* ring, int stage_bytes, uint64_t* full, uint64_t* empty,
                                         const TmaThread& H, int g0) {
    const bool lead = (threadIdx.x & 31) == 0;
    auto slot = [&](int g) { return g % TMA_STAGES; };
    auto wait_full = [&](int g) { return mbar_wait(smem_u32(&full[slot(g)]), (g / TMA_STAGES) & 1); };
    auto release = [&](int g) {
        __syncwarp();
        if (lead) mbar_arrive(smem_u32(&empty[slot(g)]));
    };
    if (!wait_full(g0) || !wait_full(g0 + 1)) return false;
    for (int i = 0; i < T.nx; ++i) {
        const int g = g0 + i;  // stage of plane x-1
        if (!wait_full(g + 2)) return false;
        if (H.inbox)
            tma_plane<EX, EY, EZ>(A, S, ring + slot(g) * stage_bytes, ring + slot(g + 1) * stage_bytes,
                                  ring + slot(g + 2) * stage_bytes, T.x0 + i, H);
        release(g);  // plane x-1 is no longer read
    }
    release(g0 + T.nx);
    release(g0 + T.nx + 1);
    return true;
}

// Persistent kernel: CTA b processes tiles cta_first[b] .. cta_first[b+1]-1 (a
// balanced assignment made on the host).  Warps 0-3 compute; warp 4 (one
// lane) issues the stages of the CTA's tiles in sequence, running ahead of the
// computation by up to TMA_STAGES stages (a stage is refilled once every
// consumer warp has released it).
// (a template so that every translation unit may include it; instantiated for float only)
template <typename TT>
__global__ void __launch_bounds__(TMA_BLOCK, 3)
    k_pml_shell_tma(const KArgs<TT> A, const TmaLaunch Lc, const TmaTile* __restrict__ tiles,
                    const int* __restrict__ cta_first, const CUtensorMap* __restrict__ maps,
                    int* __restrict__ dev_error) {
    static_assert(sizeof(TT) == 4, "the reduced PML state is an FP32 path");
    // the ring: TMA_STAGES stages of Lc.stage_bytes, then the full and the empty mbarriers
    extern __shared__ __align__(128) unsigned char tma_ring[];
    uint64_t* full = reinterpret_cast<uint64_t*>(tma_ring + TMA_STAGES * Lc.stage_bytes);
    uint64_t* empty = full + TMA_STAGES;
    if (A.advance && blockIdx.x == 0 && threadIdx.x == 0) advance_consts(*A.P, A.cur);
    const int tid = threadIdx.x;
    const uint32_t ring = smem_u32(tma_ring);
    // tensor copies land on 128-byte boundaries (every buffer size is a multiple of 128)
    if (ring & 127u) {
        if (tid == 0) atomicOr(dev_error, FDTD_DEV_ERR_TMA_TIMEOUT);
        return;
    }
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < TMA_STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), TMA_THREADS / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();
    const int t_begin = cta_first[blockIdx.x], t_end = cta_first[blockIdx.x + 1];

    if (tid >= TMA_THREADS) {
        // ---- producer: one lane issues every stage of the CTA's tiles ----
        if (tid != TMA_THREADS) return;
        int g = 0;
        bool ok = true;
        for (int t = t_begin; t < t_end && ok; ++t) {
            const TmaTile T = tiles[t];
            const TmaShape& S = Lc.shape[T.shape];
            const CUtensorMap* m = maps + ((size_t)A.cur * Lc.nshape + T.shape) * TB_N;
            for (int j = 0; j < T.nx + 2 && ok; ++j, ++g) {
                const int sl = g % TMA_STAGES;
                // the slot's previous stage (g - TMA_STAGES) has been released by every consumer warp
                if (g >= TMA_STAGES) ok = mbar_wait(smem_u32(&empty[sl]), (g / TMA_STAGES - 1) & 1);
                if (ok) tma_issue_stage(m, S, T, ring + sl * Lc.stage_bytes, smem_u32(&full[sl]), j);
            }
        }
        if (!ok) atomicOr(dev_error, FDTD_DEV_ERR_TMA_TIMEOUT);
        // no copy outlives the CTA: wait (bounded) for the last stages issued
        for (int k = g - 1; k >= 0 && k >= g - TMA_STAGES; --k)
            (void)mbar_wait(smem_u32(&full[k % TMA_STAGES]), (k / TMA_STAGES) & 1);
        return;
    }

    // ---- consumers ----
    int g0 = 0;
    for (int t = t_begin; t < t_end; ++t) {
        const TmaTile T = tiles[t];
        const TmaShape& S = Lc.shape[T.shape];
        // this thread's cells: row r of the window, z group lz .. lz+3
        TmaThread H;
        const int gpr = S.tz / 4;
        H.r = tid / gpr;
        H.lz = (tid - H.r * gpr) * 4;
        H.zc = T.z0 + H.lz;
        const bool row_on = H.r < T.ny;
        H.y = T.y0 + (row_on ? H.r : T.ny - 1);
        H.inbox = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) H.inbox |= (row_on && H.zc + e >= T.zlo && H.zc + e < T.zhi ? 1u : 0u) << e;
        H.gy = __ldg(A.axflag[1] + H.y);
        {
            uint8_t gz[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) gz[e] = H.zc + e < A.N2 ? __ldg(A.axflag[2] + H.zc + e) : (uint8_t)0;
#pragma unroll
            for (int k = 0; k < 6; ++k) H.zm[k] = flag_mask<4>(gz, k);
        }
        if ((T.cls & TC_Z) && H.inbox) {
#pragma unroll
            for (int e = 0; e <= 4; ++e) H.cz[e] = A.coef[2][H.zc + e];
        }
        if (T.cls & TC_Y) {
            H.cyl = A.coef[1][H.y];
            H.cyr = A.coef[1][H.y + 1];
        }
        unsigned char* R = tma_ring;
        const int sb = Lc.stage_bytes;
        bool done;
        switch (T.cls) {
            case TC_X: done = tma_tile<true, false, false>(A, S, T, R, sb, full, empty, H, g0); break;
            case TC_Y: done = tma_tile<false, true, false>(A, S, T, R, sb, full, empty, H, g0); break;
            case TC_Z: done = tma_tile<false, false, true>(A, S, T, R, sb, full, empty, H, g0); break;
            case TC_X | TC_Y: done = tma_tile<true, true, false>(A, S, T, R, sb, full, empty, H, g0); break;
            case TC_X | TC_Z: done = tma_tile<true, false, true>(A, S, T, R, sb, full, empty, H, g0); break;
            case TC_Y | TC_Z: done = tma_tile<false, true, true>(A, S, T, R, sb, full, empty, H, g0); break;
            default: done = tma_tile<true, true, true>(A, S, T, R, sb, full, empty, H, g0); break;
        }
        if (!done) {
            // a stage never arrived: record it and leave (the producer's own
            // bounded waits end, and it waits for its copies in flight)
            if ((tid & 31) == 0) atomicOr(dev_error, FDTD_DEV_ERR_TMA_TIMEOUT);
            return;
        }
        g0 += T.nx + 2;
    }
}

}  // namespace fdtd
