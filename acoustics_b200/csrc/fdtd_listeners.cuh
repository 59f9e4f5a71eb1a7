// fdtd_listeners.cuh — listener sampling, one warp per listener
// (PML_WaveSolver::FetchScalarData, PML_WaveSolver.cpp:210-317, with the order-1
// MLS of MLSModeInterpolator::lookup, MLSModeInterpolator.hpp:282-431).
//
// Lanes 0..7 read the (up to) eight enclosing cells; a warp scan turns their
// point counts (0 for NaN, 1 for a bulk or plain solid cell, one per ghost face
// for a ghost cell) into the row index of every MLS sample, so lane j builds
// rows j and j+32.  The weighted least-squares fit is a Householder QR whose
// column norms and dot products are warp reductions; its solution is the unique
// minimiser for a full-rank stencil, as with the reference's JacobiSVD.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_coupled.cuh"
#include "fdtd_geometry.cuh"

namespace fdtd {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The k-th (0-based) set direction of a ghost mask in key order
// (-x, -y, -z, +z, +y, +x) as (dim, sign).
__device__ __forceinline__ void kth_face(unsigned mask, int k, int& d, int& s) {
    const int od[6] = {0, 1, 2, 2, 1, 0};
    const int os[6] = {-1, -1, -1, +1, +1, +1};
    d = 0;
    s = -1;
    int seen = 0;
    for (int f = 0; f < 6; ++f) {
        if ((mask >> (2 * od[f] + (os[f] > 0 ? 1 : 0))) & 1u) {
            if (seen == k) { d = od[f]; s = os[f]; return; }
            ++seen;
        }
    }
}

template <typename T>
__device__ void build_row(const SolveParams& P, const T* __restrict__ pold, double t, int par, const double pt[3],
                          int cell, uint8_t code, double v, int k, double A[4], double& b) {
    int i, j, kk;
    cell_ijk(P, cell, i, j, kk);
    const double cp[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][kk]};
    const unsigned mask = code & CLS_MASK;
    if ((code & CLS_BULK) || mask == 0) {
        mls_row(pt, cp, v, A, b);
        return;
    }
    int d, s;
    kth_face(mask, k, d, s);
    const long long strides[3] = {P.SX, P.SY, 1};
    const long long nbr = cell + s * strides[d];
    const double pg = P.fc_rows ? fc_ghost(P, par, cell, 2 * d + (s > 0 ? 1 : 0), (double)pold[nbr])
                                : ghost_pressure(P, P.gobj[cell], cp, d, s, (double)pold[nbr], t);
    double fp[3] = {cp[0], cp[1], cp[2]};
    fp[d] += (s > 0 ? 1.0 : -1.0) * 0.25 * P.h;
    mls_row(pt, fp, pg, A, b);
}

// Listener li of solve P into out_row[li]; called by a whole warp.  With PREP
// the same fit is built from the classification alone and, instead of a value,
// its plan is written: the weight of every sample row in the fitted value at
// the listener (x0 = e0' R^-1 Q' b = (Q [R^-T e0; 0])' b, b_r = w_r value_r).
template <typename T, bool PREP = false>
__device__ void listener_body(const SolveParams& P, int newp, int li, double* __restrict__ out_row) {
    const int lane = threadIdx.x & 31;
    const T* __restrict__ pnew = (const T*)P.p[newp];
    const T* __restrict__ pold = (const T*)P.p[newp ^ 1];
    const double t = P.consts[newp ^ 1].t;
    const double pt[3] = {P.listeners[3 * li], P.listeners[3 * li + 1], P.listeners[3 * li + 2]};
    int cells[8];
    const int nc = enclosing_neighbours(P, pt, cells);

    // ---- per-cell value, class and point count (lanes 0..nc-1) ----
    int cellq = lane < nc ? cells[lane < 8 ? lane : 0] : 0;
    double v = 0.0;
    uint8_t code = 0;
    if (lane < nc) {
        v = (double)pnew[cellq];
        code = P.cls[cellq];
    }
    const bool kept = lane < nc && !isnan(v);
    int cnt = 0;
    if (kept) cnt = ((code & CLS_BULK) || !(code & CLS_MASK)) ? 1 : __popc(code & CLS_MASK);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += n;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(0xffffffffu, incl, nc - 1);
    const unsigned keptmask = __ballot_sync(0xffffffffu, kept);
    const int nk = __popc(keptmask);
    if constexpr (PREP) {
        if (lane < 8) P.lis_plan[li].cells[lane] = lane < nc ? cellq : 0;
        if (lane == 0) {
            P.lis_plan[li].nc = nc;
            P.lis_plan[li].n = 0;
        }
    }
    if (nk == 0) {
        if (lane == 0) {
            if constexpr (PREP) {
                P.lis_plan[li].mode = 2;
            } else {
                out_row[li] = 0.0;
                atomicOr(P.dev_error, 1);
            }
        }
        return;
    }
    if (nk < 4) {  // nearest kept cell centre (PML_WaveSolver.cpp:294-309)
        double d2 = DBL_MAX;
        if (kept) {
            int i, j, k;
            cell_ijk(P, cellq, i, j, k);
            const double dx = P.cpos[0][i] - pt[0], dy = P.cpos[1][j] - pt[1], dz = P.cpos[2][k] - pt[2];
            d2 = dx * dx + dy * dy + dz * dz;
        }
        // first minimum in ascending cell order (strict <)
        double best = DBL_MAX;
        int bl = -1;
        for (int q = 0; q < nc; ++q) {
            const double dq = __shfl_sync(0xffffffffu, d2, q);
            if (dq < best) { best = dq; bl = q; }
        }
        const double val = __shfl_sync(0xffffffffu, v, bl < 0 ? 0 : bl);
        if constexpr (PREP) {
            const int cb = __shfl_sync(0xffffffffu, cellq, bl < 0 ? 0 : bl);
            if (lane == 0) {
                P.lis_plan[li].mode = 1;
                P.lis_plan[li].cell = cb;
            }
        } else {
            if (lane == 0) out_row[li] = val;
        }
        return;
    }

    // ---- rows: lane j owns sample rows j and j + 32 ----
    double A0[4] = {0, 0, 0, 0}, A1[4] = {0, 0, 0, 0};
    double b0 = 0.0, b1 = 0.0;
    const bool has0 = lane < total, has1 = lane + 32 < total;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int r = lane + 32 * half;
        // owner cell q: excl[q] <= r < excl[q] + cnt[q]
        int owner = 0, first = 0;
        for (int q = 0; q < nc; ++q) {
            const int eq = __shfl_sync(0xffffffffu, excl, q);
            const int cq = __shfl_sync(0xffffffffu, cnt, q);
            if (cq > 0 && r >= eq && r < eq + cq) { owner = q; first = eq; }
        }
        const double vq = __shfl_sync(0xffffffffu, v, owner);
        const int codeq = __shfl_sync(0xffffffffu, (int)code, owner);
        const int cellqq = __shfl_sync(0xffffffffu, cellq, owner);
        if (half == 0 && has0) build_row<T>(P, pold, t, newp ^ 1, pt, cellqq, (uint8_t)codeq, vq, r - first, A0, b0);
        if (half == 1 && has1) build_row<T>(P, pold, t, newp ^ 1, pt, cellqq, (uint8_t)codeq, vq, r - first, A1, b1);
        if constexpr (PREP) {
            if ((half == 0 && has0) || (half == 1 && has1)) {
                // row source: the cell value, or the ghost face it stands for
                int kind = 0;
                const unsigned mask = (unsigned)codeq & CLS_MASK;
                if (!(codeq & CLS_BULK) && mask != 0) {
                    int dd, ss;
                    kth_face(mask, r - first, dd, ss);
                    kind = 1 + 2 * dd + (ss > 0 ? 1 : 0);
                }
                LisRow& row = P.lis_rows[(size_t)li * 64 + r];
                row.cell = cellqq;
                row.kind = kind;
                row.w = half == 0 ? A0[0] : A1[0];  // the row weight (first column)
            }
        }
    }

    // ---- Householder QR, warp-parallel ----
    double R[4][4];
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const bool a0 = has0 && lane >= j;          // row index lane >= j
        const bool a1 = has1;                        // rows >= 32 are always >= j
        double s = (a0 ? A0[j] * A0[j] : 0.0) + (a1 ? A1[j] * A1[j] : 0.0);
        s = warp_sum(s);
        const double norm = sqrt(s);
        if (!(norm > 0.0)) ok = false;
        const double x0 = __shfl_sync(0xffffffffu, A0[j], j);
        const double alpha = x0 > 0.0 ? -norm : norm;
        if (lane == j) A0[j] = x0 - alpha;
        double vn = (a0 ? A0[j] * A0[j] : 0.0) + (a1 ? A1[j] * A1[j] : 0.0);
        vn = warp_sum(vn);
#pragma unroll
        for (int cc = j + 1; cc < 4; ++cc) {
            double dot = (a0 ? A0[j] * A0[cc] : 0.0) + (a1 ? A1[j] * A1[cc] : 0.0);
            dot = warp_sum(dot);
            const double f = 2.0 * dot / vn;
            if (a0) A0[cc] -= f * A0[j];
            if (a1) A1[cc] -= f * A1[j];
        }
        {
            double dot = (a0 ? A0[j] * b0 : 0.0) + (a1 ? A1[j] * b1 : 0.0);
            dot = warp_sum(dot);
            const double f = 2.0 * dot / vn;
            if (a0) b0 -= f * A0[j];
            if (a1) b1 -= f * A1[j];
        }
        R[j][j] = alpha;
#pragma unroll
        for (int cc = j + 1; cc < 4; ++cc) R[j][cc] = __shfl_sync(0xffffffffu, A0[cc], j);
    }
    if constexpr (PREP) {
        const double rmax = dmax(dmax(fabs(R[0][0]), fabs(R[1][1])), dmax(fabs(R[2][2]), fabs(R[3][3])));
        for (int j = 0; j < 4; ++j)
            if (fabs(R[j][j]) <= (double)(total > 4 ? total : 4) * 2.220446049250313e-16 * rmax) ok = false;
        if (!ok) {
            if (lane == 0) P.lis_plan[li].mode = 2;
            return;
        }
        // u = R^-T e0, then y = H0 H1 H2 H3 [u; 0] (reflectors in reverse order)
        double u[4];
        u[0] = 1.0 / R[0][0];
        u[1] = -(R[0][1] * u[0]) / R[1][1];
        u[2] = -(R[0][2] * u[0] + R[1][2] * u[1]) / R[2][2];
        u[3] = -(R[0][3] * u[0] + R[1][3] * u[1] + R[2][3] * u[2]) / R[3][3];
        double y0 = lane < 4 ? u[lane] : 0.0, y1 = 0.0;
#pragma unroll
        for (int j = 3; j >= 0; --j) {
            const bool a0 = has0 && lane >= j;
            const bool a1 = has1;
            const double vv = warp_sum((a0 ? A0[j] * A0[j] : 0.0) + (a1 ? A1[j] * A1[j] : 0.0));
            const double dot = warp_sum((a0 ? A0[j] * y0 : 0.0) + (a1 ? A1[j] * y1 : 0.0));
            const double f = 2.0 * dot / vv;
            if (a0) y0 -= f * A0[j];
            if (a1) y1 -= f * A1[j];
        }
        if (has0) P.lis_rows[(size_t)li * 64 + lane].w *= y0;
        if (has1) P.lis_rows[(size_t)li * 64 + lane + 32].w *= y1;
        if (lane == 0) {
            P.lis_plan[li].mode = 0;
            P.lis_plan[li].n = total;
        }
        return;
    }
    double bt[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) bt[j] = __shfl_sync(0xffffffffu, b0, j);
    if (lane != 0) return;
    const double rmax = dmax(dmax(fabs(R[0][0]), fabs(R[1][1])), dmax(fabs(R[2][2]), fabs(R[3][3])));
    for (int j = 0; j < 4; ++j)
        if (fabs(R[j][j]) <= (double)(total > 4 ? total : 4) * 2.220446049250313e-16 * rmax) ok = false;
    double x[4];
    for (int j = 3; j >= 0; --j) {
        double s = bt[j];
        for (int cc = j + 1; cc < 4; ++cc) s -= R[j][cc] * x[cc];
        x[j] = s / R[j][j];
    }
    out_row[li] = ok ? x[0] : 0.0;
    if (!ok) atomicOr(P.dev_error, 1);
}

// FDTD_ERR_NUMERIC for a listener sample that is not finite (lane 0 wrote it).
__device__ __forceinline__ void flag_nonfinite(const SolveParams& P, const double* out_row, int li) {
    if ((threadIdx.x & 31) == 0 && !isfinite(out_row[li])) atomicOr(P.dev_error, 1);
}

// Listener li from its plan: sum_r w_r value_r as a warp reduction.  A NaN
// among the enclosing cells (which the full fit drops) falls back to it.
template <typename T>
__device__ __forceinline__ void listener_plan(const SolveParams& P, int newp, int li, double* __restrict__ out_row) {
    const int lane = threadIdx.x & 31;
    const LisPlan& pl = P.lis_plan[li];
    const T* __restrict__ pnew = (const T*)P.p[newp];
    const int nc = pl.nc;
    const double vc = lane < nc ? (double)pnew[pl.cells[lane < 8 ? lane : 0]] : 0.0;
    if (__ballot_sync(0xffffffffu, lane < nc && isnan(vc))) {
        listener_body<T>(P, newp, li, out_row);
        return;
    }
    if (pl.mode == 1) {
        if (lane == 0) out_row[li] = (double)pnew[pl.cell];
        return;
    }
    if (pl.mode == 2) {
        if (lane == 0) {
            out_row[li] = 0.0;
            atomicOr(P.dev_error, 1);
        }
        return;
    }
    const T* __restrict__ pold = (const T*)P.p[newp ^ 1];
    const double t = P.consts[newp ^ 1].t;
    double acc = 0.0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int r = lane + 32 * half;
        if (r >= pl.n) continue;
        const LisRow row = P.lis_rows[(size_t)li * 64 + r];
        double val;
        if (row.kind == 0) {
            val = (double)pnew[row.cell];
        } else {
            const int d = (row.kind - 1) >> 1, sgn = ((row.kind - 1) & 1) ? 1 : -1;
            int i, j, k;
            cell_ijk(P, row.cell, i, j, k);
            const double cp[3] = {P.cpos[0][i], P.cpos[1][j], P.cpos[2][k]};
            const long long strides[3] = {P.SX, P.SY, 1};
            const double pn = (double)pold[row.cell + sgn * strides[d]];
            val = P.fc_rows ? fc_ghost(P, newp ^ 1, row.cell, 2 * d + (sgn > 0 ? 1 : 0), pn)
                            : ghost_pressure(P, P.gobj[row.cell], cp, d, sgn, pn, t);
        }
        acc += row.w * val;
    }
    acc = warp_sum(acc);
    if (lane == 0) out_row[li] = acc;
}

// Plans of every listener from the current classification (one warp each)
template <typename T>
__global__ void __launch_bounds__(128) k_listener_prep(const SolveParams* __restrict__ Pp, int newp) {
    const int li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (li >= Pp->n_lis) return;
    listener_body<T, true>(*Pp, newp, li, nullptr);
}

template <typename T>
__global__ void __launch_bounds__(128) k_listeners_warp(const SolveParams* __restrict__ Pp, int newp,
                                                        double* __restrict__ out_row) {
    const int li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (li >= Pp->n_lis) return;  // the whole warp leaves together
    if (Pp->lis_ready) listener_plan<T>(*Pp, newp, li, out_row);
    else listener_body<T>(*Pp, newp, li, out_row);
    flag_nonfinite(*Pp, out_row, li);
}

}  // namespace fdtd
