// fdtd_engquist.cuh — the Engquist-Majda absorbing update of the non-PML cells
// one cell inside the domain edge (MAC_Grid::PML_pressureUpdateCollocated,
// MAC_Grid.cpp:515-920).  It is live where a side has no PML: the wall presets
// 1 and 2 (MAC_Grid.cpp:4027-4101), or a PML under 1.5 cells.
//
// Per cell the reference extrapolates the pressure of its exterior
// neighbour(s) on the domain edge, writes them into the CURRENT pressure buffer
// (zero at the diagonal exterior cell of an edge or corner) and takes a
// six-point leapfrog step with them; faces use the second-order form, edges and
// corners the first-order one.  With three rotating buffers, the edge cells of
// the buffer that is current at step n hold the values written at step n-3
// until this step's update overwrites them, and the values of step n-2 once it
// becomes the next pressure.  Two kernels reproduce that on two buffers:
//
//   k_engquist_predict  (first in the step, before any kernel writes p^{n+1}):
//       reads p^n and p^{n-1} of the stencil (p^{n-1} of an exterior cell is the
//       value extrapolated at step n-1), stores p^{n+1} (+ sources) and this
//       step's exterior values in the cell's buffer entry;
//   k_engquist_commit   (last in the step, after every kernel that reads p^n):
//       writes p^{n+1} of the cell (FP32: the increment too), the exterior
//       values of step n into p^n and those of step n-2 into p^{n+1} (not where
//       an exterior cell is a PML cell: its p^{n+1} comes from the PML update),
//       and shifts the cell's history of exterior values.
//
// A solid cell in a stencil needs the ghost-pressure forms, which are not
// built: the predict kernel flags DEV_ERR_ENGQUIST and the step fails.
#pragma once

namespace fdtd {

template <typename T>
__global__ void __launch_bounds__(128) k_engquist_predict(const SolveParams* __restrict__ Pp, int cur) {
    const SolveParams& P = *Pp;
    const T* __restrict__ pc = (const T*)P.p[cur];
    const T* __restrict__ pl = (const T*)P.p[cur ^ 1];  // p^{n-1}: nothing has written p^{n+1} yet
    const double lambda = P.eng_lambda;
    const double lambda2 = lambda * lambda;
    const StepConsts& sc = P.consts[cur];
    bool any_src = false;
    for (int q = 0; q < P.n_src; ++q) any_src |= (sc.src_tf[q] != 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.eng_n; i += gridDim.x * blockDim.x) {
        const EngCell e = P.eng[i];
        double* b = P.eng_buf + (size_t)i * ENG_BUF;
        const long long c = e.c;
        if ((P.cls[c] & (CLS_BULK | CLS_MASK)) != CLS_BULK) {
            atomicOr(P.dev_error, DEV_ERR_ENGQUIST);
            continue;
        }
        const int type = e.flags & 3;
        const double pC = (double)pc[c], pL = (double)pl[c];
        double pn, x0 = 0.0, x1 = 0.0, x2 = 0.0;
        if (type == 1) {
            // face, second order (MAC_Grid.cpp:547-646)
            const double pl_ii_p = (double)pl[c + e.o[0]];
            const double p_ii_n = (double)pc[c + e.o[1]], pl_ii_n = (double)pl[c + e.o[1]];
            const double p_jj_p = (double)pc[c + e.o[2]], p_jj_n = (double)pc[c + e.o[3]];
            const double p_kk_p = (double)pc[c + e.o[4]], p_kk_n = (double)pc[c + e.o[5]];
            double p1 = (2. / lambda2 + 4. / lambda - 6. - 4. * lambda) * pC - (1. / lambda2 + 2. / lambda) * pL +
                        pl_ii_p - pl_ii_n + 2. * p_ii_n + (lambda + 1.) * (p_jj_p + p_jj_n + p_kk_p + p_kk_n);
            p1 *= (lambda2 / (1. + 2. * lambda));
            x0 = pl_ii_p + p_ii_n - pl_ii_n - 2. / lambda * (p1 + pL - 2. * pC) +
                 lambda * (p_jj_p + p_jj_n + p_kk_p + p_kk_n - 4. * pC);
            pn = 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_p + p_jj_n + p_kk_p + p_kk_n + x0 - 6. * pC);
        } else if (type == 2) {
            // edge, first order (MAC_Grid.cpp:648-767)
            const double p_ii_n = (double)pc[c + e.o[3]], p_jj_n = (double)pc[c + e.o[4]];
            const double p_kk_p = (double)pc[c + e.o[5]], p_kk_n = (double)pc[c + e.o[6]];
            double p1 = (2. / lambda2 - 6.) * pC + (2.0 * lambda - 1.0) / lambda2 * pL + 2. * p_ii_n + 2. * p_jj_n +
                        p_kk_p + p_kk_n;
            p1 *= (lambda2 / (1. + 2. * lambda));
            x0 = (pL - p1) / lambda + p_ii_n;
            x1 = (pL - p1) / lambda + p_jj_n;
            pn = 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_n + p_kk_p + p_kk_n + x0 + x1 - 6. * pC);
        } else {
            // corner, first order (MAC_Grid.cpp:768-913)
            const double p_ii_n = (double)pc[c + e.o[3]], p_jj_n = (double)pc[c + e.o[4]];
            const double p_kk_n = (double)pc[c + e.o[5]];
            double p1 = (2. / lambda2 - 6.) * pC + (3.0 * lambda - 1.0) / lambda2 * pL + 2. * p_ii_n + 2. * p_jj_n +
                        2. * p_kk_n;
            p1 *= (lambda2 / (1. + 3. * lambda));
            x0 = (pL - p1) / lambda + p_ii_n;
            x1 = (pL - p1) / lambda + p_jj_n;
            x2 = (pL - p1) / lambda + p_kk_n;
            pn = 2.0 * pC - pL + lambda2 * (p_ii_n + p_jj_n + p_kk_n + x0 + x1 + x2 - 6. * pC);
        }
        if (any_src) {
            // MAC_Grid.cpp:938-944: the source term of non-PML cells
            int x, y, z;
            cell_ijk(P, c, x, y, z);
            pn += source_term(P, cur, x, y, z) * P.k;
        }
        b[0] = pn;
        b[1] = x0;
        b[2] = x1;
        b[3] = x2;
    }
}

template <typename T>
__global__ void __launch_bounds__(128) k_engquist_commit(const SolveParams* __restrict__ Pp, int cur) {
    const SolveParams& P = *Pp;
    T* __restrict__ pc = (T*)P.p[cur];
    T* __restrict__ pn = (T*)P.p[cur ^ 1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.eng_n; i += gridDim.x * blockDim.x) {
        const EngCell e = P.eng[i];
        double* b = P.eng_buf + (size_t)i * ENG_BUF;
        const long long c = e.c;
        if constexpr (sizeof(T) == 8) {
            pn[c] = b[0];
        } else {
            // the compensated form: the increment is p^{n+1} - p^n
            const float d = (float)(b[0] - (double)pc[c]);
            P.dinc[c] = d;
            pn[c] = pc[c] + d;
        }
        const int type = e.flags & 3;
        for (int q = 0; q < type; ++q) {
            const long long x = c + e.o[q];
            pc[x] = (T)b[1 + q];
            if (!(e.flags & (16 << q))) pn[x] = (T)b[7 + q];
            b[7 + q] = b[4 + q];
            b[4 + q] = b[1 + q];
        }
        if (type >= 2) {
            const long long x = c + e.o[type == 2 ? 2 : 6];
            pc[x] = (T)0.0;
            if (!(e.flags & (16 << 3))) pn[x] = (T)0.0;
        }
    }
}

}  // namespace fdtd
