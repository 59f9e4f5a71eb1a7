// fdtd_batch.cuh — one step of many independent solves of uneven sizes in a
// fixed number of launches, whatever the number of solves.
//
// Every member keeps its own device state (the arrays of its fdtd_solver); a
// descriptor per member holds its kernel arguments for both buffer parities,
// its boxes, its listener ring and its parity in that table.  Because the step
// constants live on the device, a captured graph of an even number of batched
// steps replays for any step index.
//
// Per step:  k_batch_ghost (third stream)  ||  k_batch_interior (second stream)
//            ||  k_batch_shell_red / k_batch_shell (PML tiles of the members with
//            the reduced / full PML state), then k_batch_sources (second
//            stream, after the ghost list), then k_batch_advance; the listener
//            rows (k_batch_listeners) on a fourth stream beside the next step.
// The descriptors come in two tables, one per step parity (every member's
// parity flips each step), so consecutive steps alternate tables and no kernel
// flips parities on the device.
// The shell kernels run one CTA per entry of a tile table that lists the tiles
// of every member (sorted by member); the interior kernel finds its members'
// arguments in its parameter bank (up to BATCH_PARAM_MEMBERS members, else a
// tile table too).  Both call the same tile functions as the single-solve kernels.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_hot.cuh"
#include "fdtd_listeners.cuh"
#include "fdtd_region.cuh"

namespace fdtd {

#ifndef FDTD_BATCH_INT_TILES
#define FDTD_BATCH_INT_TILES 4
#endif

// The tile-table interior (more members than the parameter-bank table holds):
// FDTD_BATCH_INT_TILES consecutive tiles per CTA.  The tiles are sorted by
// member, so a CTA copies its member's arguments into registers once for the
// tiles that share it: only the first waits on the chain tile -> descriptor ->
// arguments before its data loads can issue.
#ifndef FDTD_BATCH_INT_MINB
#define FDTD_BATCH_INT_MINB 3
#endif
template <typename T, int XB>
__global__ void __launch_bounds__(256, XB == 2 ? FDTD_BATCH_INT_MINB : 1) k_batch_interior(const BatchDesc<T>* __restrict__ D,
                                                                         const BatchTile* __restrict__ tiles,
                                                                         int n_tiles) {
    constexpr int K = FDTD_BATCH_INT_TILES;
    int m = -1;
    bool halted = true;
    KArgs<T> A;
    Box3 box;
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
        const int t = blockIdx.x * K + k;
        if (t >= n_tiles) break;  // uniform per CTA
        const BatchTile tile = tiles[t];
        if (tile.m != m) {
            m = tile.m;
            const BatchDesc<T>& d = D[m];
            halted = d.halted != 0;
            A = d.a[d.cur];
            box = d.interior;
        }
        if (!halted) interior_tile<T, XB>(A, box, tile.tz, tile.tx);
    }
}

// One CTA per interior tile, its member found by a binary search of the
// parameter-bank table from blockIdx alone (warp-uniform, like its arguments);
// a member's CTAs enumerate its tiles as the tile table does (x tile outer).
template <typename T, int XB>
__global__ void __launch_bounds__(256, XB == 2 ? 4 : 1)
    k_batch_interior_p(const __grid_constant__ BatchIntParams<T> P, const BatchDesc<T>* __restrict__ D) {
    const int blk = (int)blockIdx.x;
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.first[mid] <= blk) lo = mid;
        else hi = mid - 1;
    }
    const BatchIntMember<T>& M = P.m[lo];
    if (D[M.member].halted) return;
    const int local = blk - P.first[lo];
    interior_tile<T, XB>(M, M.box, local % M.tu, local / M.tu);
}

// One CTA per shell tile of the tables (all members in one launch).  The
// member's arguments are read through references into its descriptor in global
// memory (L1-resident after the first warp), so a CTA starts without a barrier.

template <typename T>
__global__ void __launch_bounds__(256, shell_min_blocks(sizeof(T))) k_batch_shell(const BatchDesc<T>* __restrict__ D,
                                                                      const BatchTile* __restrict__ tiles) {
    const BatchTile tile = tiles[blockIdx.x];
    const BatchDesc<T>& d = D[tile.m];
    if (d.halted) return;
    shell_tile<T>(d.a[d.cur], d.shell, tile.box, tile.tz, tile.tx);
}

// Shell tiles of members that keep the reduced PML state (FP32 only).
template <typename T>
__global__ void __launch_bounds__(256, FDTD_SHELL_RED_MINB) k_batch_shell_red(const BatchDesc<T>* __restrict__ D,
                                                                      const BatchTile* __restrict__ tiles) {
    static_assert(sizeof(T) == 4, "the reduced PML state is an FP32 path");
    const BatchTile tile = tiles[blockIdx.x];
    const BatchDesc<T>& d = D[tile.m];
    if (d.halted) return;
    const KArgs<float> A = d.a[d.cur];  // in registers: the plane loop reads them every plane
    shell_tile_red(A, d.shell, tile.box, tile.tz, tile.tx);
}

// grid (solid_blocks, members): re-zero the solid cells inside the PML of the
// members that have some (the PML update writes every PML cell; classification
// zeroes solid cells in every buffer at the start of a step, MAC_Grid.cpp:3566-3600)
template <typename T>
__global__ void __launch_bounds__(256) k_batch_solid_pml(const BatchDesc<T>* __restrict__ D) {
    const BatchDesc<T>& d = D[blockIdx.y];
    if (!d.active || d.halted) return;
    const SolveParams& P = *d.P;
    T* p0 = (T*)P.p[0];
    T* p1 = (T*)P.p[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_solid_pml; i += gridDim.x * blockDim.x) {
        const int c = P.solid_pml[i];
        p0[c] = (T)0;
        p1[c] = (T)0;
        if (P.dinc) P.dinc[c] = 0.0f;
    }
}

// grid (ghost_blocks, members)
template <typename T>
__global__ void __launch_bounds__(128) k_batch_ghost(const BatchDesc<T>* __restrict__ D) {
    const BatchDesc<T>& d = D[blockIdx.y];
    if (!d.active || d.halted || d.ghost_cap == 0) return;
    ghost_cells_body<T>(*d.P, d.cur, blockIdx.x, gridDim.x);
}

// grid (src_blocks, members)
template <typename T>
__global__ void __launch_bounds__(256) k_batch_sources(const BatchDesc<T>* __restrict__ D) {
    const BatchDesc<T>& d = D[blockIdx.y];
    if (!d.active || d.halted || !d.has_src) return;
    // a source whose time factor underflowed to zero adds nothing (the single-solve
    // path skips the launch then); the whole block leaves together
    const StepConsts& c = d.P->consts[d.cur];
    bool any = false;
    for (int s = 0; s < d.P->n_src; ++s) any |= c.src_tf[s] != 0.0;
    if (!any) return;
    sources_body<T>(*d.P, d.cur, d.src_region, blockIdx.x, gridDim.x);
}

// one warp per (member, listener)
template <typename T>
__global__ void __launch_bounds__(128) k_batch_listeners(const BatchDesc<T>* __restrict__ D,
                                                         const ListenerRef* __restrict__ refs, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= n) return;
    const ListenerRef r = refs[w];
    const BatchDesc<T>& d = D[r.m];
    if (!d.active || d.halted) return;
    const long long step = d.P->consts[d.cur].step;
    double* row = d.ring + (size_t)(step % d.ring_cap) * d.n_lis;
    if (d.P->lis_ready) listener_plan<T>(*d.P, d.cur ^ 1, r.li, row);
    else listener_body<T>(*d.P, d.cur ^ 1, r.li, row);
    flag_nonfinite(*d.P, row, r.li);
}

template <typename T>
cudaError_t launch_batch(const BatchLaunch& L, const StepStreams& S, int* launches) {
    BatchDesc<T>* D = static_cast<BatchDesc<T>*>(L.descs);
    int l = 0;
    if (L.solid_blocks > 0) {
        k_batch_solid_pml<T><<<dim3(L.solid_blocks, L.n_members), 256, 0, S.s>>>(D);
        ++l;
    }
    const bool gside = L.ghost_blocks > 0 && S.s3 != nullptr;
    cudaError_t e = cudaEventRecord(S.fork, S.s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S.s2, S.fork, 0);
    if (e == cudaSuccess && gside) e = cudaStreamWaitEvent(S.s3, S.fork, 0);
    if (e != cudaSuccess) return e;
    if (L.ghost_blocks > 0) {
        // first: a few latency-bound CTAs that run beside the interior's
        k_batch_ghost<T><<<dim3(L.ghost_blocks, L.n_members), 128, 0, gside ? S.s3 : S.s2>>>(D);
        ++l;
        if (gside && (e = cudaEventRecord(S.ghost, S.s3)) != cudaSuccess) return e;
    }
    if (L.int_params && L.int_ctas > 0) {
        const dim3 block(32, 8);
        const BatchIntParams<T>& P = *static_cast<const BatchIntParams<T>*>(L.int_params);
        if (L.xb == 2) k_batch_interior_p<T, 2><<<L.int_ctas, block, 0, S.s2>>>(P, D);
        else if (L.xb == 8) k_batch_interior_p<T, 8><<<L.int_ctas, block, 0, S.s2>>>(P, D);
        else k_batch_interior_p<T, 4><<<L.int_ctas, block, 0, S.s2>>>(P, D);
        ++l;
    } else if (L.n_int > 0) {
        const dim3 block(32, 8);
        const unsigned grid = (unsigned)((L.n_int + FDTD_BATCH_INT_TILES - 1) / FDTD_BATCH_INT_TILES);
        if (L.xb == 2) k_batch_interior<T, 2><<<grid, block, 0, S.s2>>>(D, L.int_tiles, L.n_int);
        else if (L.xb == 8) k_batch_interior<T, 8><<<grid, block, 0, S.s2>>>(D, L.int_tiles, L.n_int);
        else k_batch_interior<T, 4><<<grid, block, 0, S.s2>>>(D, L.int_tiles, L.n_int);
        ++l;
    }
    int n_red = 0;
    if constexpr (sizeof(T) == 4) {
        n_red = L.n_shell_red;
        if (n_red > 0) {
            k_batch_shell_red<float><<<n_red, dim3(32, 8), red_smem_bytes(), S.s>>>(D, L.shell_tiles);
            ++l;
        }
    }
    if (L.n_shell > n_red) {
        k_batch_shell<T><<<L.n_shell - n_red, dim3(32, 8), shell_smem_bytes<T>(), S.s>>>(D, L.shell_tiles + n_red);
        ++l;
    }
    if (gside && (e = cudaStreamWaitEvent(S.s2, S.ghost, 0)) != cudaSuccess) return e;
    if (L.src_blocks > 0) {
        // source cells are non-PML cells: ordered after the interior and ghost updates
        // of their cells, concurrent with the shell
        k_batch_sources<T><<<dim3(L.src_blocks, L.n_members), 256, 0, S.s2>>>(D);
        ++l;
    }
    e = cudaEventRecord(S.join, S.s2);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S.s, S.join, 0);
    if (e != cudaSuccess) return e;
    if (launches) *launches += l;
    return cudaGetLastError();
}

// Last kernel of a batched step, one thread per member: write the member's
// constants of the next step (consts[cur ^ 1]) and, after its last step, mark
// it halted, so its kernels leave at once from the next step on (the tables
// alternate every step, a halted member's state no longer does).  The flag goes
// into the next step's table D2 first and into this step's table D one step
// later, by this kernel of the next step: the listener rows of this step, which
// run beside the next step and read D, still see the member running.  (That
// kernel of the next step waits for them.)  Members retire without a new tile
// table or graph.
template <typename T>
__global__ void __launch_bounds__(128) k_batch_advance(BatchDesc<T>* __restrict__ D, BatchDesc<T>* __restrict__ D2,
                                                       int n) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const BatchDesc<T>& d = D[m];
    if (!d.active) return;
    if (d.halted) {
        D2[m].halted = 1;
        return;
    }
    const long long step = d.P->consts[d.cur].step;
    advance_consts(*d.P, d.cur);
    if (step + 1 >= d.total) D2[m].halted = 1;
}

// Listener rows of a batched step.  Instantiated in the FP64 translation unit
// for both field types, like the single-solve listener kernel, so the
// double-precision MLS arithmetic is compiled the same way (no FMA
// contraction) and batch rows equal single-solve rows bit for bit.
template <typename T>
cudaError_t launch_batch_listeners(const BatchLaunch& L, cudaStream_t s, int* launches) {
    BatchDesc<T>* D = static_cast<BatchDesc<T>*>(L.descs);
    if (L.n_refs > 0) {
        k_batch_listeners<T><<<(L.n_refs * 32 + 127) / 128, 128, 0, s>>>(D, L.refs, L.n_refs);
        if (launches) *launches += 1;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_batch_advance(const BatchLaunch& L, cudaStream_t s, int* launches) {
    BatchDesc<T>* D = static_cast<BatchDesc<T>*>(L.descs);
    if (L.n_members > 0) {
        k_batch_advance<T><<<(L.n_members + 127) / 128, 128, 0, s>>>(D, static_cast<BatchDesc<T>*>(L.descs_other),
                                                                      L.n_members);
        if (launches) *launches += 1;
    }
    return cudaGetLastError();
}

}  // namespace fdtd
