// fdtd_coupled.cuh — per-step part of the FULLY_COUPLED ghost cells
// (MAC_Grid::PML_pressureUpdateGhostCells, MAC_Grid.cpp:1131-1425): the
// right-hand side of the fixed sparse system of a static scene (rows built by
// fdtd_coupled.cpp) and its solution by BiCGSTAB with the diagonal
// preconditioner and a tolerance of one machine epsilon relative to the
// right-hand side, the reference's solver and settings (MAC_Grid.cpp:1409-1412),
// in one CTA.  The ghost pressures of a step land in fc_x[parity]; the
// ghost-cell Laplacian and the listeners of that step read them there.
#pragma once
#include "fdtd_device.cuh"
#include "fdtd_geometry.cuh"

namespace fdtd {

// Row of the ghost face of solid cell `owner` towards direction f = 2 dim +
// (sign > 0); -1 when the cell has no ghost face there.
FDTD_HD int fc_row(const SolveParams& P, long long owner, int f) {
    const int e = P.fc_idx[owner];
    if (e < 0 || !((e >> f) & 1)) return -1;
    int below = 0;
    for (int q = 0; q < f; ++q) below += (e >> q) & 1;
    return (e >> 6) + below;
}

// Ghost pressure of that face in the step of parity `par` (fallback when the
// cell has no face there, which classification rules out).
FDTD_HD double fc_ghost(const SolveParams& P, int par, long long owner, int f, double fallback) {
    const int r = fc_row(P, owner, f);
    return r < 0 ? fallback : P.fc_x[(size_t)par * P.fc_n + r];
}

template <typename T>
__global__ void __launch_bounds__(256) k_fc_rhs(const SolveParams* __restrict__ Pp, int cur) {
    const SolveParams& P = *Pp;
    const T* __restrict__ p = (const T*)P.p[cur];
    const double t = P.consts[cur].t;
    for (int ri = blockIdx.x * blockDim.x + threadIdx.x; ri < P.fc_n; ri += gridDim.x * blockDim.x) {
        const FcRow& R = P.fc_rows[ri];
        const double p_neig = (double)p[R.nbr];
        double b = p_neig;
        if (R.kind != 1) {
            double a[3];
            boundary_accel(P.obj[R.obj], R.bp, t, a);
            double g[3];
            for (int i = 0; i < 3; ++i) g[i] = a[i] * (-P.rho);
            double n[3] = {0.0, 0.0, 0.0};
            n[R.dim] = (R.sign > 0 ? 1.0 : -1.0);
            const double g_nr = g[0] * n[0] + g[1] * n[1] + g[2] * n[2];
            const double pg = p_neig - 0.75 * P.h * g_nr;
            if (R.kind == 0) {
                b = pg;
            } else if (R.kind == 3) {
                b = -pg;
            } else {
                const double g_ne = g[0] * R.ne[0] + g[1] * R.ne[1] + g[2] * R.ne[2];
                b = -(g_ne * R.fdw);
                for (int q = 0; q < 8; ++q)
                    if (R.cell[q] >= 0) b -= R.w[q] * (double)p[R.cell[q]];
                if (R.si >= 0) b -= R.w[R.si] * (g_ne * P.h);
            }
        }
        P.fc_b[ri] = b;
    }
}

// Sum over the CTA (1024 threads) of one value per thread.
__device__ __forceinline__ double fc_block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    return red[32];
}

// diagonal of row r: +1 (kinds 0, 1) or -1 (kinds 2, 3); the preconditioner is its inverse
__device__ __forceinline__ double fc_diag(const FcRow& R) { return R.kind <= 1 ? 1.0 : -1.0; }

// out = A (D^-1 in), D the diagonal
__device__ __forceinline__ void fc_apply_precond(const SolveParams& P, const double* in, double* out) {
    for (int r = threadIdx.x; r < P.fc_n; r += blockDim.x) {
        const FcRow& R = P.fc_rows[r];
        double y = in[r];  // diag * (in / diag)
        if (R.kind == 2)
            for (int q = 0; q < 8; ++q)
                if (R.unk[q] >= 0) y += R.w[q] * (in[R.unk[q]] / fc_diag(P.fc_rows[R.unk[q]]));
        out[r] = y;
    }
}

// One CTA of 1024 threads.  BiCGSTAB from x = 0 with the right preconditioned
// update of the reference's solver; stops once |r|^2 <= eps^2 |b|^2 or after
// fc_maxit iterations (status: iterations, or -iterations when not converged).
static __global__ void __launch_bounds__(1024) k_fc_solve(const SolveParams* __restrict__ Pp, int cur) {
    const SolveParams& P = *Pp;
    __shared__ double red[33];
    const int n = P.fc_n;
    double* x = P.fc_x + (size_t)cur * n;
    double* r = P.fc_work;
    double* r0 = r + n;
    double* pv = r0 + n;
    double* v = pv + n;
    double* sv = v + n;
    double* tv = sv + n;
    const double* b = P.fc_b;
    double bb = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        x[i] = 0.0;
        r[i] = b[i];
        r0[i] = b[i];
        pv[i] = 0.0;
        v[i] = 0.0;
        bb += b[i] * b[i];
    }
    const double rhs2 = fc_block_sum(bb, red);
    if (rhs2 == 0.0) {
        if (threadIdx.x == 0) P.fc_status[0] = 0;
        return;
    }
    const double eps = 2.220446049250313e-16;
    const double tol2 = eps * eps * rhs2;
    double r0_sq = rhs2, rr = rhs2;
    double rho = 1.0, alpha = 1.0, w = 1.0;
    int it = 0, restarts = 0;
    while (rr > tol2 && it < P.fc_maxit) {
        const double rho_old = rho;
        double part = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) part += r0[i] * r[i];
        rho = fc_block_sum(part, red);
        if (fabs(rho) < eps * eps * r0_sq) {
            // the basis became orthogonal to r0: restart from the current residual
            __syncthreads();
            part = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const FcRow& R = P.fc_rows[i];
                double ax = fc_diag(R) * x[i];
                if (R.kind == 2)
                    for (int q = 0; q < 8; ++q)
                        if (R.unk[q] >= 0) ax += R.w[q] * x[R.unk[q]];
                r[i] = b[i] - ax;
                r0[i] = r[i];
                part += r[i] * r[i];
            }
            rho = r0_sq = fc_block_sum(part, red);
            if (restarts++ == 0) it = 0;
        }
        const double beta = (rho / rho_old) * (alpha / w);
        for (int i = threadIdx.x; i < n; i += blockDim.x) pv[i] = r[i] + beta * (pv[i] - w * v[i]);
        __syncthreads();
        fc_apply_precond(P, pv, v);  // v = A y, y = D^-1 p
        __syncthreads();
        part = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) part += r0[i] * v[i];
        alpha = rho / fc_block_sum(part, red);
        for (int i = threadIdx.x; i < n; i += blockDim.x) sv[i] = r[i] - alpha * v[i];
        __syncthreads();
        fc_apply_precond(P, sv, tv);  // t = A z, z = D^-1 s
        __syncthreads();
        double tt = 0.0, ts = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            tt += tv[i] * tv[i];
            ts += tv[i] * sv[i];
        }
        const double tt_all = fc_block_sum(tt, red);
        const double ts_all = fc_block_sum(ts, red);
        w = tt_all > 0.0 ? ts_all / tt_all : 0.0;
        part = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double dinv = 1.0 / fc_diag(P.fc_rows[i]);
            x[i] += alpha * (pv[i] * dinv) + w * (sv[i] * dinv);
            r[i] = sv[i] - w * tv[i];
            part += r[i] * r[i];
        }
        rr = fc_block_sum(part, red);
        ++it;
    }
    if (threadIdx.x == 0) P.fc_status[0] = rr > tol2 ? -it : it;
}

}  // namespace fdtd
