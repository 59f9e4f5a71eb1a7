// fdtd_fp64.cu — FP64 step kernels, cell classification, listener sampling and
// fresh-cell interpolation.  Compiled with -fmad=false: every product and sum
// is rounded on its own, in the order the reference writes it, which keeps the
// FP64 path and the classification bit-reproducible against a CPU build of the
// same expressions.
#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "fdtd_device.cuh"
#include "fdtd_geometry.cuh"
#include "fdtd_launch.hpp"
#include "fdtd_listeners.cuh"
#include "fdtd_stencil.cuh"

namespace fdtd {

// ---------------------------------------------------------------------------
// Cell classification (MAC_Grid::classifyCells_FAST, MAC_Grid.cpp:3455-3891)
// ---------------------------------------------------------------------------

// A classification is two launches.  k_cls_boxes visits the cells of the
// iteration boxes (each cell once) and makes their new bulk / valid bits, the
// solid test of MAC_Grid.cpp:3608-3653 with the zeroing of solid pressures
// (MAC_Grid.cpp:3796-3798).  k_cls_sweep then visits every cell as "quads":
// four cells of one z row, read and written as one 32-bit word (rows start at
// multiples of 8 bytes, and a quad never reaches past its row's padding), one
// quad per thread.  A cell outside every box is bulk with
// validHistory <- isBulk (MAC_Grid.cpp:3464-3472); only quads within one cell
// of a box look further (neighbour masks, closest objects, lists).
struct ClsQuad {
    int i, j, k0, nk;
    long long c0;
};

// bytes of a quad word that are cells (the rest is row padding, left as it was)
__device__ __forceinline__ uint32_t quad_cells(int nk) { return nk >= 4 ? 0xFFFFFFFFu : (1u << (8 * nk)) - 1u; }

constexpr uint32_t QUAD_BULK = 0x01010101u * CLS_BULK;
constexpr uint32_t QUAD_VALID = 0x01010101u * CLS_VALID;

__device__ __forceinline__ bool in_box(const ClsBoxes& B, int b, int i, int j, int k) {
    return i >= B.lo[b][0] && i < B.lo[b][0] + B.rg[b][0] && j >= B.lo[b][1] && j < B.lo[b][1] + B.rg[b][1] &&
           k >= B.lo[b][2] && k < B.lo[b][2] + B.rg[b][2];
}

// 0xFF at the bytes of cells k0 .. k0+3 of row (i, j) that lie in some box
__device__ uint32_t box_bytes(const ClsBoxes& B, int i, int j, int k0) {
    uint32_t m = 0;
    for (int b = 0; b < B.n; ++b) {
        if (i < B.lo[b][0] || i >= B.lo[b][0] + B.rg[b][0] || j < B.lo[b][1] || j >= B.lo[b][1] + B.rg[b][1]) continue;
        const int lo = max(k0, B.lo[b][2]) - k0, hi = min(k0 + 4, B.lo[b][2] + B.rg[b][2]) - k0;
        if (hi > lo) m |= (hi >= 4 ? 0xFFFFFFFFu : (1u << (8 * hi)) - 1u) & ~((1u << (8 * lo)) - 1u);
    }
    return m;
}

// some box reaches a cell of the quad or one of its six neighbours
__device__ __forceinline__ bool quad_near(const ClsBoxes& B, const ClsQuad& q) {
    for (int b = 0; b < B.n; ++b) {
        if (B.rg[b][0] <= 0 || B.rg[b][1] <= 0 || B.rg[b][2] <= 0) continue;
        if (q.i + 1 >= B.lo[b][0] && q.i - 1 < B.lo[b][0] + B.rg[b][0] && q.j + 1 >= B.lo[b][1] &&
            q.j - 1 < B.lo[b][1] + B.rg[b][1] && q.k0 + q.nk >= B.lo[b][2] && q.k0 - 1 < B.lo[b][2] + B.rg[b][2])
            return true;
    }
    return false;
}

// Solid test of the box cells, each cell once (in its first box).  Also
// empties the ghost-neighbour and fresh-cell lists the sweep fills.
__global__ void __launch_bounds__(128) k_cls_boxes(const SolveParams* __restrict__ Pp) {
    const SolveParams& P = *Pp;
    const ClsBoxes& B = P.boxes;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *P.ghost_count = 0;
        *P.fresh_count = 0;
    }
    const long long total = B.first[B.n];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int b = 0;
        while (t >= B.first[b + 1]) ++b;
        const long long r = t - B.first[b];
        const int r1 = B.rg[b][1], r2 = B.rg[b][2];
        const int i = B.lo[b][0] + (int)(r / ((long long)r1 * r2));
        const int j = B.lo[b][1] + (int)((r / r2) % r1);
        const int k = B.lo[b][2] + (int)(r % r2);
        bool dup = false;
        for (int e = 0; e < b; ++e) dup = dup || in_box(B, e, i, j, k);
        if (dup) continue;
        const long long c = cidx(P, i, j, k);
        const double pos[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]};
        int type = 0;
        const bool fluid = is_fluid(P, pos, type);
        const uint8_t old = P.cls[c];
        P.cls[c] = (uint8_t)((fluid ? CLS_BULK : 0) | ((old & CLS_BULK) ? CLS_VALID : 0) | (old & CLS_MASK));
        if (!fluid) {
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

// The cells of a quad that need more than their mask: ghost cells (closest
// object), non-PML bulk cells with a solid neighbour (ghost-neighbour list) and
// fresh cells (fresh-cell list); `sel` has the bulk bit set at those bytes,
// `code` the quad's new bulk / valid bits.  The list slots of the lanes that
// call it together are taken with one atomic per list (an atomic per cell on
// one counter serialises thousands of cells a step); the lists are unordered.
__device__ __noinline__ void cls_cells(const SolveParams& P, const ClsQuad q, uint32_t sel, uint32_t code,
                                       uint32_t listed, uint32_t fresh) {
    namespace cg = cooperative_groups;
    uint32_t to_list = 0, to_fresh = 0;  // bytes (bulk bit) of this quad's cells for each list
    while (sel) {
        const int m = (__ffs(sel) - 1) >> 3;
        sel &= ~(0xFFu << (8 * m));
        const int k = q.k0 + m;
        const long long c = q.c0 + m;
        if (!((code >> (8 * m)) & CLS_BULK)) {
            const double pos[3] = {P.cpos[0][q.i], P.cpos[1][q.j], P.cpos[2][k]};
            const int o = lowest_object(P, pos);
            P.gobj[c] = (P.gobj[c] & GOBJ_CONSTRAINT) | (uint8_t)(o < 0 ? GOBJ_NONE : o);
            continue;
        }
        // non-PML bulk cells next to a solid: updated by k_ghost_cells
        if (((listed >> (8 * m)) & CLS_BULK) && !(P.pml_cell[0][q.i] || P.pml_cell[1][q.j] || P.pml_cell[2][k]))
            to_list |= (uint32_t)CLS_BULK << (8 * m);
        if ((fresh >> (8 * m)) & CLS_BULK) to_fresh |= (uint32_t)CLS_BULK << (8 * m);
    }
    const cg::coalesced_group g = cg::coalesced_threads();
    const int nl = __popc(to_list), nf = __popc(to_fresh);
    const int pl = cg::exclusive_scan(g, nl), pf = cg::exclusive_scan(g, nf);
    const int tl = g.shfl(pl + nl, g.size() - 1), tf = g.shfl(pf + nf, g.size() - 1);
    int bl = 0, bf = 0;
    if (g.thread_rank() == 0) {
        if (tl) bl = atomicAdd(P.ghost_count, tl);
        if (tf) bf = atomicAdd(P.fresh_count, tf);
    }
    int sl = g.shfl(bl, 0) + pl, sf = g.shfl(bf, 0) + pf;
    while (to_list) {
        const int m = (__ffs(to_list) - 1) >> 3;
        to_list &= ~(0xFFu << (8 * m));
        if (sl < P.ghost_cap) P.ghost_list[sl] = (int)(q.c0 + m);
        ++sl;
    }
    while (to_fresh) {
        const int m = (__ffs(to_fresh) - 1) >> 3;
        to_fresh &= ~(0xFFu << (8 * m));
        if (sf < P.fresh_cap) P.fresh_list[sf] = (int)(q.c0 + m);
        ++sf;
    }
}

// New bulk bits of the quad of row (i, j) at k0: from memory in the boxes
// (written by k_cls_boxes and not changed by the sweep), bulk elsewhere.
__device__ __forceinline__ uint32_t quad_bulk(const SolveParams& P, const ClsBoxes& B, int i, int j, int k0) {
    const uint32_t m = box_bytes(B, i, j, k0);
    const uint32_t w = m ? *(const uint32_t*)(P.cls + (long long)i * P.SX + (long long)j * P.SY + k0) : 0u;
    return (w & m & QUAD_BULK) | (QUAD_BULK & ~m);
}

// Quads within one cell of a box.  Neighbour masks: for a solid cell the
// directions of its bulk neighbours (one ghost face each, MakeGhostCell
// MAC_Grid.cpp:4310-4340) and, where it has one, its closest object
// (LowestObjectDistance, MAC_Grid.cpp:3810-3814; only ghost faces read it);
// for a bulk cell the directions of its solid (ghost) neighbours, read by the
// Laplacian.  Mask bit 2d + (s > 0) is set where the
// neighbour in direction s along axis d exists and differs in bulk-ness; the
// four cells are compared at once, byte by byte of the words.
__device__ __noinline__ void cls_sweep_near(const SolveParams& P, const ClsQuad q, uint32_t own, int collect_fresh) {
    const ClsBoxes& B = P.boxes;
    const uint32_t cells = quad_cells(q.nk);
    const uint32_t inb = box_bytes(B, q.i, q.j, q.k0);
    const uint32_t reset = QUAD_BULK | ((own & QUAD_BULK) >> 1);  // CLS_VALID is CLS_BULK >> 1
    const uint32_t base = (own & inb & (QUAD_BULK | QUAD_VALID)) | (reset & ~inb);
    // a missing neighbour reads as the cell itself (no difference, no face)
    const uint32_t xm = q.i > 0 ? quad_bulk(P, B, q.i - 1, q.j, q.k0) : base;
    const uint32_t xp = q.i + 1 < P.N[0] ? quad_bulk(P, B, q.i + 1, q.j, q.k0) : base;
    const uint32_t ym = q.j > 0 ? quad_bulk(P, B, q.i, q.j - 1, q.k0) : base;
    const uint32_t yp = q.j + 1 < P.N[1] ? quad_bulk(P, B, q.i, q.j + 1, q.k0) : base;
    uint32_t zlo = base & 0xFFu, zhi = base >> 24;
    if (q.k0 > 0) {
        bool in = false;
        for (int b = 0; b < B.n; ++b) in = in || in_box(B, b, q.i, q.j, q.k0 - 1);
        zlo = in ? (P.cls[q.c0 - 1] & CLS_BULK) : CLS_BULK;
    }
    if (q.k0 + 4 < P.N[2]) {
        bool in = false;
        for (int b = 0; b < B.n; ++b) in = in || in_box(B, b, q.i, q.j, q.k0 + 4);
        zhi = in ? (P.cls[q.c0 + 4] & CLS_BULK) : CLS_BULK;
    }
    const uint32_t zm = (base << 8) | zlo;
    const uint32_t zp = (base >> 8) | (zhi << 24);
    uint32_t mask = (((base ^ xm) & QUAD_BULK) >> 7) | (((base ^ xp) & QUAD_BULK) >> 6) |
                    (((base ^ ym) & QUAD_BULK) >> 5) | (((base ^ yp) & QUAD_BULK) >> 4) |
                    (((base ^ zm) & QUAD_BULK) >> 3) | (((base ^ zp) & QUAD_BULK) >> 2);
    // a quad that ends inside its word: the last cell's +z neighbour is padding
    if (q.nk < 4) mask &= ~(0x20u << (8 * (q.nk - 1)));
    const uint32_t bulk = base & QUAD_BULK & cells;
    // cells with a nonzero mask (a 6-bit byte plus 0x3F carries into bit 6)
    const uint32_t masked = ((mask + 0x3F3F3F3Fu) & 0x40404040u) << 1;
    // ghost cells: the solid cells whose closest object is read (ghost faces);
    // k_cls_boxes has reset the object of every solid cell of this step
    const uint32_t ghost = ~base & QUAD_BULK & cells & masked;
    const uint32_t listed = bulk & masked;
    const uint32_t fresh = collect_fresh ? bulk & ~((base & QUAD_VALID) << 1) : 0u;
    const uint32_t sel = ghost | listed | fresh;
    if (sel) cls_cells(P, q, sel, base, listed, fresh);
    const uint32_t out = ((base | mask) & cells) | (own & ~cells);
    if (out != own) *(uint32_t*)(P.cls + q.c0) = out;
}

// One quad of the sweep with its word `own`.
__device__ __forceinline__ void cls_sweep_quad(const SolveParams& P, const ClsQuad& q, uint32_t own, int collect_fresh) {
    if (quad_near(P.boxes, q)) {
        cls_sweep_near(P, q, own, collect_fresh);
        return;
    }
    // no solid cell within one cell: bulk, history from the last step, no mask
    const uint32_t cells = quad_cells(q.nk);
    const uint32_t out = ((QUAD_BULK | ((own & QUAD_BULK) >> 1)) & cells) | (own & ~cells);
    if (out != own) {
        *(uint32_t*)(P.cls + q.c0) = out;
        const uint32_t fresh = collect_fresh ? ~own & QUAD_BULK & cells : 0u;
        if (fresh) cls_cells(P, q, fresh, out, 0u, fresh);
    }
}

// Box b reaches unit (i, j, ch): a cell of it, or a neighbour of one, is in the box.
__device__ __forceinline__ bool unit_in(const ClsBoxes& B, int b, int i, int j, int ch) {
    return i >= B.u0[b][0] && i < B.u0[b][0] + B.un[b][0] && j >= B.u0[b][1] && j < B.u0[b][1] + B.un[b][1] &&
           ch >= B.u0[b][2] && ch < B.u0[b][2] + B.un[b][2];
}

// Units no box reaches: bulk cells with the history of the last step and no
// mask; the cells that were solid the step before are fresh.  A warp takes
// CLS_UNITS consecutive units (256 cells of a z row each) and loads all of them
// first, 8 bytes a lane (rows start at multiples of 8 bytes and a lane's 8 bytes
// stay inside its row's padding).  Units some box reaches are left to k_cls_near.
constexpr int CLS_UNITS = 8;

__global__ void __launch_bounds__(256) k_cls_sweep(const SolveParams* __restrict__ Pp, int nunits, int chunks,
                                                   int collect_fresh) {
    const SolveParams& P = *Pp;
    const ClsBoxes& B = P.boxes;
    const int lane = threadIdx.x & 31;
    const int first = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * CLS_UNITS;
    if (first >= nunits) return;  // whole warps
    const int N1 = P.N[1], N2 = P.N[2];
    const long long SX = P.SX, SY = P.SY;
    // lane r < CLS_UNITS tests unit first + r against the boxes
    bool lane_near = false;
    if (lane < CLS_UNITS && first + lane < nunits) {
        const int u = first + lane;
        const int row = u / chunks;
        const int i = row / N1, j = row - (row / N1) * N1;
        for (int b = 0; b < B.n && !lane_near; ++b) lane_near = unit_in(B, b, i, j, u - row * chunks);
    }
    const unsigned near_units = __ballot_sync(0xffffffffu, lane_near);
    // the warp's first unit; later ones step through chunks, then rows
    const int row0 = first / chunks;
    const int i0 = row0 / N1, j0 = row0 - i0 * N1, ch0 = first - row0 * chunks;
    const int nu = min(CLS_UNITS, nunits - first);
    uint2 d[CLS_UNITS];
    {
        int i = i0, j = j0, ch = ch0;
#pragma unroll
        for (int r = 0; r < CLS_UNITS; ++r) {
            d[r] = make_uint2(0u, 0u);
            const int k0 = ch * CLS_CHUNK + lane * 8;
            if (r < nu && !((near_units >> r) & 1u) && k0 < N2)
                d[r] = *(const uint2*)(P.cls + i * SX + j * SY + k0);
            if (++ch == chunks) {
                ch = 0;
                if (++j == N1) {
                    j = 0;
                    ++i;
                }
            }
        }
    }
    const unsigned long long bulk8 = 0x0101010101010101ull * CLS_BULK;
    int i = i0, j = j0, ch = ch0;
#pragma unroll
    for (int r = 0; r < CLS_UNITS; ++r) {
        const int k0 = ch * CLS_CHUNK + lane * 8;
        const int ci = i, cj = j;
        if (++ch == chunks) {
            ch = 0;
            if (++j == N1) {
                j = 0;
                ++i;
            }
        }
        if (r >= nu || ((near_units >> r) & 1u) || k0 >= N2) continue;
        const unsigned long long w = ((unsigned long long)d[r].y << 32) | d[r].x;
        const int nk = min(8, N2 - k0);
        const unsigned long long cells = nk >= 8 ? ~0ull : (1ull << (8 * nk)) - 1ull;
        const unsigned long long out = ((bulk8 | ((w & bulk8) >> 1)) & cells) | (w & ~cells);
        if (out == w) continue;
        const long long c = ci * SX + cj * SY + k0;
        *(uint2*)(P.cls + c) = make_uint2((uint32_t)out, (uint32_t)(out >> 32));
        unsigned long long fresh = collect_fresh ? ~w & bulk8 & cells : 0ull;
        while (fresh) {
            const int m = (__ffsll((long long)fresh) - 1) >> 3;
            fresh &= ~(0xFFull << (8 * m));
            const int slot = atomicAdd(P.fresh_count, 1);
            if (slot < P.fresh_cap) P.fresh_list[slot] = (int)(c + m);
        }
    }
}

// The sweep of a moving-body step restricted to the units the boxes of the
// step before reached: every cell outside them already holds bulk, a valid
// history and no mask (the boxes are unions of a body's bounds over two steps,
// so the solid, masked and fresh cells of the step before all lie in units they
// reach), so the full sweep would write nothing there.  One warp per unit,
// every unit once; units a box of this step reaches are left to k_cls_near.
__global__ void __launch_bounds__(256) k_cls_sweep_prev(const SolveParams* __restrict__ Pp, const ClsBoxes prev,
                                                        int collect_fresh) {
    const SolveParams& P = *Pp;
    const ClsBoxes& B = P.boxes;
    const int lane = threadIdx.x & 31;
    const long long total = prev.ufirst[prev.n];
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const unsigned long long bulk8 = 0x0101010101010101ull * CLS_BULK;
    for (long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; t < total; t += nwarps) {
        int b = 0;
        while (t >= prev.ufirst[b + 1]) ++b;
        const long long r = t - prev.ufirst[b];
        const int nj = prev.un[b][1], nc = prev.un[b][2];
        const int i = prev.u0[b][0] + (int)(r / ((long long)nj * nc));
        const int j = prev.u0[b][1] + (int)((r / nc) % nj);
        const int ch = prev.u0[b][2] + (int)(r % nc);
        bool skip = false;
        for (int e = 0; e < b && !skip; ++e) skip = unit_in(prev, e, i, j, ch);
        for (int e = 0; e < B.n && !skip; ++e) skip = unit_in(B, e, i, j, ch);
        if (skip) continue;
        const int k0 = ch * CLS_CHUNK + lane * 8;
        if (k0 >= P.N[2]) continue;
        const long long c = (long long)i * P.SX + (long long)j * P.SY + k0;
        const uint2 d = *(const uint2*)(P.cls + c);
        const unsigned long long w = ((unsigned long long)d.y << 32) | d.x;
        const int nk = min(8, P.N[2] - k0);
        const unsigned long long cells = nk >= 8 ? ~0ull : (1ull << (8 * nk)) - 1ull;
        const unsigned long long out = ((bulk8 | ((w & bulk8) >> 1)) & cells) | (w & ~cells);
        if (out == w) continue;
        *(uint2*)(P.cls + c) = make_uint2((uint32_t)out, (uint32_t)(out >> 32));
        unsigned long long fresh = collect_fresh ? ~w & bulk8 & cells : 0ull;
        while (fresh) {
            const int m = (__ffsll((long long)fresh) - 1) >> 3;
            fresh &= ~(0xFFull << (8 * m));
            const int slot = atomicAdd(P.fresh_count, 1);
            if (slot < P.fresh_cap) P.fresh_list[slot] = (int)(c + m);
        }
    }
}

// Units some box reaches, one warp each, every unit once (in the first box
// that reaches it); a lane takes two quads.
__global__ void __launch_bounds__(256) k_cls_near(const SolveParams* __restrict__ Pp, int collect_fresh) {
    const SolveParams& P = *Pp;
    const ClsBoxes& B = P.boxes;
    const int lane = threadIdx.x & 31;
    // two warps per unit, a quad per lane: the few units of a step spread over
    // twice the warps, each walking half the chain
    const long long total = 2 * B.ufirst[B.n];
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long th = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; th < total; th += nwarps) {
        const long long t = th >> 1;
        const int half = (int)(th & 1);
        int b = 0;
        while (t >= B.ufirst[b + 1]) ++b;
        const long long r = t - B.ufirst[b];
        const int nj = B.un[b][1], nc = B.un[b][2];
        const int i = B.u0[b][0] + (int)(r / ((long long)nj * nc));
        const int j = B.u0[b][1] + (int)((r / nc) % nj);
        const int ch = B.u0[b][2] + (int)(r % nc);
        bool dup = false;
        for (int e = 0; e < b && !dup; ++e) dup = unit_in(B, e, i, j, ch);
        if (dup) continue;
        const int k0 = ch * CLS_CHUNK + lane * 8 + 4 * half;
        if (k0 >= P.N[2]) continue;
        ClsQuad q;
        q.i = i;
        q.j = j;
        q.k0 = k0;
        q.nk = min(4, P.N[2] - k0);
        q.c0 = (long long)i * P.SX + (long long)j * P.SY + k0;
        cls_sweep_quad(P, q, *(const uint32_t*)(P.cls + q.c0), collect_fresh);
    }
}

// Listener sampling: fdtd_listeners.cuh (one warp per listener)

// ---------------------------------------------------------------------------
// Fresh-cell interpolation (MAC_Grid::InterpolateFreshPressureCell, MLS branch,
// MAC_Grid.cpp:1993-2254): a cell that is bulk now but was solid before gets
// p = p_MLS(image point) + rho (a . n) |s| in p^{n-1} and p^n.
// ---------------------------------------------------------------------------
// Out of line: the few fresh cells of a step run this once per launch, and one
// copy of the code misses the instruction cache less than several inlined ones.
template <typename T>
__device__ __noinline__ double fresh_value(const SolveParams& P, const T* __restrict__ pa, const T* __restrict__ pb,
                                           bool diff, long long c, double t, int* status) {
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
    // the flags, values and positions of the stencil cells, loaded together
    // (one round trip to memory instead of one per cell)
    uint8_t code[8];
    double vals[8], npos[8][3];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (q >= nc) break;
        const int n = cells[q];
        int ni, nj, nn;
        cell_ijk(P, n, ni, nj, nn);
        code[q] = P.cls[n];
        vals[q] = val(n);
        npos[q][0] = P.cpos[0][ni];
        npos[q][1] = P.cpos[1][nj];
        npos[q][2] = P.cpos[2][nn];
    }
    // the MLS rows of the stencil cells with a valid history, in a fixed block of
    // 8 (rows of the other cells zero), kept in registers
    double A[8][4], b[8];
    unsigned keptm = 0;
    int nk = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const bool kq = q < nc && (code[q] & CLS_VALID);
        if (kq) {
            mls_row(image, npos[q], vals[q], A[q], b[q]);
            keptm |= 1u << q;
            ++nk;
        } else {
            A[q][0] = A[q][1] = A[q][2] = A[q][3] = 0.0;
            b[q] = 0.0;
        }
    }
    if (nk < 4) {
        if (nk != 0) {
            double md = DBL_MAX;
            int mid = -1;
            for (int q = 0; q < 8; ++q) {
                if (!((keptm >> q) & 1u)) continue;
                const double dx = image[0] - npos[q][0], dy = image[1] - npos[q][1], dz = image[2] - npos[q][2];
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 < md) { md = d2; mid = q; }
            }
            return vals[mid];
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
    if (!householder_ls4_rows8(A, b, nk, c0)) c0 = 0.0;
    double acc[3];
    boundary_accel(o, bp, t, acc);
    const double an = acc[0] * nrm[0] + acc[1] * nrm[1] + acc[2] * nrm[2];
    return c0 + P.rho * an * fabs(travelled);
}

template <typename T>
__device__ __forceinline__ void fresh_cell(const SolveParams& P, int cur, long long c, double t, int* st) {
    if (sizeof(T) == 8) {
        double* pl = (double*)P.p[cur ^ 1];
        double* pc = (double*)P.p[cur];
        const double vl = fresh_value<double>(P, pl, pl, false, c, t, st);
        const double vc = fresh_value<double>(P, pc, pc, false, c, t, st);
        pl[c] = vl;
        pc[c] = vc;
    } else {
        // FP32 keeps p^n and the increment; p^{n-1} = p^n - d
        float* pc = (float*)P.p[cur];
        const double vc = fresh_value<float>(P, pc, pc, false, c, t, st);
        const double vl = fresh_value<float>(P, pc, P.dinc, true, c, t, st);
        pc[c] = (float)vc;
        P.dinc[c] = (float)(vc - vl);
    }
}

// The fresh value of one cell computed by a half-warp: lane q < 8 of the half
// holds the MLS row of stencil cell q (bits of q = x, y, z of the 2x2x2
// enclosing cells; a cell repeated at the domain edge keeps its first lane), so
// the eight rows, their weights and the Householder updates run in parallel.
// Every reduction adds the lanes' terms in row order from zero, and zero rows
// add nothing, so the result is bit-equal to householder_ls4_rows8 over the
// same rows.  All 32 lanes must call it with the same cell (both halves take
// the same branches: they share the image point and the stencil flags).
template <typename T>
__device__ __noinline__ double fresh_value_half(const SolveParams& P, const T* __restrict__ pa,
                                                const T* __restrict__ pb, bool diff, long long c, double t,
                                                int* status) {
    const int q = threadIdx.x & 15;
    const int base = threadIdx.x & 16;  // first lane of this half
    auto sum_rows = [&](double x, int from) {
        double acc = 0.0;
        for (int i = from; i < 8; ++i) acc += __shfl_sync(0xffffffffu, x, base + i);
        return acc;
    };
    auto from_row = [&](double x, int i) { return __shfl_sync(0xffffffffu, x, base + i); };
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
    // enclosing cells of the image point (enclosing_neighbours)
    int a0[3], a1[3];
    for (int d = 0; d < 3; ++d) {
        double df = image[d] - P.bmin[d];
        df -= P.h / 2.0;
        int i0 = (int)(df / P.h);
        i0 = i0 < 0 ? 0 : i0;
        i0 = i0 > P.N[d] - 1 ? P.N[d] - 1 : i0;
        a0[d] = i0;
        a1[d] = (df < 0.0 ? 0 : (i0 + 1 < P.N[d] - 1 ? i0 + 1 : P.N[d] - 1));
    }
    const int bx = (q >> 2) & 1, by = (q >> 1) & 1, bz = q & 1;
    const bool in_stencil = q < 8 && !(bx && a1[0] == a0[0]) && !(by && a1[1] == a0[1]) && !(bz && a1[2] == a0[2]);
    const int ni = bx ? a1[0] : a0[0], nj = by ? a1[1] : a0[1], nn = bz ? a1[2] : a0[2];
    double Ar[4] = {0.0, 0.0, 0.0, 0.0}, br = 0.0, vq = 0.0, pq[3] = {0.0, 0.0, 0.0};
    bool valid = false;
    if (in_stencil) {
        const long long n = cidx(P, ni, nj, nn);
        valid = (P.cls[n] & CLS_VALID) != 0;
        vq = diff ? (double)pa[n] - (double)pb[n] : (double)pa[n];
        pq[0] = P.cpos[0][ni];
        pq[1] = P.cpos[1][nj];
        pq[2] = P.cpos[2][nn];
        if (valid) mls_row(image, pq, vq, Ar, br);
    }
    const unsigned kept = (__ballot_sync(0xffffffffu, valid) >> base) & 0xffu;
    const int nk = __popc(kept);
    if (nk < 4) {
        if (nk != 0) {
            // the valid stencil cell nearest the image point (first in row order on ties)
            double md = DBL_MAX;
            int mid = -1;
            for (int r = 0; r < 8; ++r) {
                const double dx = image[0] - from_row(pq[0], r), dy = image[1] - from_row(pq[1], r),
                             dz = image[2] - from_row(pq[2], r);
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (((kept >> r) & 1u) && d2 < md) {
                    md = d2;
                    mid = r;
                }
            }
            double vm = 0.0;
            for (int r = 0; r < 8; ++r) {
                const double v = from_row(vq, r);
                if (r == mid) vm = v;
            }
            return vm;
        }
        const int idx[3] = {i, j, k};
        const long long strides[3] = {P.SX, P.SY, 1};
        for (int d = 0; d < 3; ++d)
            for (int s = 1; s >= -1; s -= 2) {
                if (idx[d] + s < 0 || idx[d] + s >= P.N[d]) continue;
                const long long n = c + s * strides[d];
                if (P.cls[n] & CLS_BULK) return diff ? (double)pa[n] - (double)pb[n] : (double)pa[n];
            }
        return 0.0;
    }
    // Householder QR of the 8 x 4 block, one row per lane (householder_ls4_rows8)
    double R[4][4];
    bool ok = true;
#pragma unroll
    for (int jc = 0; jc < 4; ++jc) {
        const double s = sum_rows(q >= jc && q < 8 ? Ar[jc] * Ar[jc] : 0.0, jc);
        const double norm = sqrt(s);
        if (!(norm > 0.0)) {
            ok = false;
            break;
        }
        const double x0 = from_row(Ar[jc], jc);
        const double alpha = x0 > 0.0 ? -norm : norm;
        if (q == jc) Ar[jc] = x0 - alpha;
        const double vnorm2 = sum_rows(q >= jc && q < 8 ? Ar[jc] * Ar[jc] : 0.0, jc);
#pragma unroll
        for (int cc = jc + 1; cc < 4; ++cc) {
            const double dot = sum_rows(q >= jc && q < 8 ? Ar[jc] * Ar[cc] : 0.0, jc);
            const double f = 2.0 * dot / vnorm2;
            if (q >= jc && q < 8) Ar[cc] -= f * Ar[jc];
        }
        {
            const double dot = sum_rows(q >= jc && q < 8 ? Ar[jc] * br : 0.0, jc);
            const double f = 2.0 * dot / vnorm2;
            if (q >= jc && q < 8) br -= f * Ar[jc];
        }
        R[jc][jc] = alpha;
#pragma unroll
        for (int cc = jc + 1; cc < 4; ++cc) R[jc][cc] = from_row(Ar[cc], jc);
    }
    double c0 = 0.0;
    if (ok) {
        const double rmax = dmax(dmax(fabs(R[0][0]), fabs(R[1][1])), dmax(fabs(R[2][2]), fabs(R[3][3])));
#pragma unroll
        for (int jc = 0; jc < 4; ++jc)
            if (fabs(R[jc][jc]) <= (double)(nk > 4 ? nk : 4) * 2.220446049250313e-16 * rmax) ok = false;
    }
    if (ok) {
        double bq[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) bq[r] = from_row(br, r);
        double x[4];
#pragma unroll
        for (int jc = 3; jc >= 0; --jc) {
            double s2 = bq[jc];
#pragma unroll
            for (int cc = jc + 1; cc < 4; ++cc) s2 -= R[jc][cc] * x[cc];
            x[jc] = s2 / R[jc][jc];
        }
        c0 = x[0];
    }
    double acc[3];
    boundary_accel(o, bp, t, acc);
    const double an = acc[0] * nrm[0] + acc[1] * nrm[1] + acc[2] * nrm[2];
    return c0 + P.rho * an * fabs(travelled);
}

// Fresh cells of the classification just made, from the list the ghost sweep
// filled, one warp per cell: the half-warp 16 w + q makes the value of buffer w
// (p^n for w = 0, p^{n-1} for w = 1).  A list that overflowed is replaced by a
// sweep over every cell, a thread per cell.  Each fresh value reads only cells
// with a valid history, never another fresh cell, so the order does not matter.
template <typename T>
__global__ void __launch_bounds__(128) k_fresh_cells(const SolveParams* __restrict__ Pp, int cur, long long n,
                                                     int* status) {
    const SolveParams& P = *Pp;
    const double t = P.consts[cur].t;
    const int count = *P.fresh_count;
    int st = 0;
    if (count > P.fresh_cap) {
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
             q += (long long)gridDim.x * blockDim.x) {
            int i, j, k;
            dense_ijk(P, q, i, j, k);
            const long long c = cidx(P, i, j, k);
            const uint8_t code = P.cls[c];
            if (!(code & CLS_BULK) || (code & CLS_VALID)) continue;
            fresh_cell<T>(P, cur, c, t, &st);
        }
        if (st) atomicMax(status, st);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int w = lane >> 4;
    for (int f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < count; f += (gridDim.x * blockDim.x) >> 5) {
        const long long c = P.fresh_list[f];
        double v;
        if (sizeof(T) == 8) {
            const double* buf = (const double*)P.p[cur ^ w];
            v = fresh_value_half<double>(P, buf, buf, false, c, t, &st);
        } else {
            const float* pc = (const float*)P.p[cur];
            v = w ? fresh_value_half<float>(P, pc, P.dinc, true, c, t, &st)
                  : fresh_value_half<float>(P, pc, pc, false, c, t, &st);
        }
        const double other = __shfl_xor_sync(0xffffffffu, v, 16);
        if ((lane & 15) != 0) continue;
        if (sizeof(T) == 8) {
            ((double*)P.p[cur ^ w])[c] = v;
        } else if (w == 0) {
            // FP32 keeps p^n and the increment; p^{n-1} = p^n - d
            ((float*)P.p[cur])[c] = (float)v;
            P.dinc[c] = (float)(v - other);
        }
    }
    if (st) atomicMax(status, st);
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

cudaError_t launch_classify(const SolveParams* dP, const int N[3], const ClsBoxes& B, bool collect_fresh,
                            cudaStream_t s, const ClsBoxes* prev) {
    k_cls_boxes<<<grid_for(B.first[B.n], 128), 128, 0, s>>>(dP);
    if (prev) {
        const long long units = prev->ufirst[prev->n];
        if (units > 0)
            k_cls_sweep_prev<<<(unsigned)std::min<long long>((units + 7) / 8, 148 * 16), 256, 0, s>>>(
                dP, *prev, collect_fresh ? 1 : 0);
    } else {
        const int chunks = (N[2] + CLS_CHUNK - 1) / CLS_CHUNK;
        const int nunits = N[0] * N[1] * chunks;
        const int warps = (nunits + CLS_UNITS - 1) / CLS_UNITS;
        k_cls_sweep<<<(warps + 7) / 8, 256, 0, s>>>(dP, nunits, chunks, collect_fresh ? 1 : 0);
    }
    if (B.ufirst[B.n] > 0) k_cls_near<<<grid_for((2 * B.ufirst[B.n] + 7) / 8, 1), 256, 0, s>>>(dP, collect_fresh ? 1 : 0);
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

cudaError_t launch_fresh_cells(const SolveParams* dP, int precision, int cur, long long ncell, int* d_status,
                               cudaStream_t s) {
    // the list, a warp per cell (a few thousand cells a step at most)
    const int grid = 4 * 148;
    if (precision == 0) k_fresh_cells<double><<<grid, 128, 0, s>>>(dP, cur, ncell, d_status);
    else k_fresh_cells<float><<<grid, 128, 0, s>>>(dP, cur, ncell, d_status);
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
cudaError_t prepare_fp64_kernels() {
    // the full-state shell's ring of staged loads
    cudaError_t e = cudaSuccess;
    if (shell_smem_bytes<double>() > 0) {
        e = cudaFuncSetAttribute(k_pml_shell<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 shell_smem_bytes<double>());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_batch_shell<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     shell_smem_bytes<double>());
    }
    return e;
}
cudaError_t launch_batch_listeners_any(int precision, const BatchLaunch& L, cudaStream_t s, int* launches) {
    return precision == 0 ? launch_batch_listeners<double>(L, s, launches) : launch_batch_listeners<float>(L, s, launches);
}
cudaError_t launch_batch_advance_any(int precision, const BatchLaunch& L, cudaStream_t s, int* launches) {
    return precision == 0 ? launch_batch_advance<double>(L, s, launches) : launch_batch_advance<float>(L, s, launches);
}
}  // namespace fdtd
