"""Independent vectorised numpy restatement of the reference's collocated FDTD
step, used to pin the C++ oracle on small grids (test infrastructure only).

It follows the same reference functions as the oracle but shares no code with
it: PML_WaveSolver::stepCollocated (PML_WaveSolver.cpp:775-826) with
MAC_Grid::classifyCells_FAST (MAC_Grid.cpp:3455-3891, spheres only, no
constraints), PML_pressureUpdateGhostCells in RASTERIZE mode with no boundary
acceleration (ghost pressure = neighbour pressure, MAC_Grid.cpp:1254-1281),
PML_velocityUpdateCollocated (:461-479), pressureFieldLaplacianGhostCell
(:187-299), PML_pressureUpdateCollocated (:481-946) with its Engquist-Majda
branch for sides without PML (:533-920; boundary presets of :4027-4101) over
three rotating pressure buffers, and the Gaussian pressure source
(GaussianPressureSource.cpp:6-30).  Listeners are sampled with the
order-1 weighted least squares of MLSModeInterpolator::lookup through
numpy.linalg.lstsq.
"""
from __future__ import annotations

import math

import numpy as np


class NumpyFDTD:
    def __init__(self, scene):
        sc = scene
        self.h = h = sc.cell_size
        self.c, self.rho, self.k = sc.sound_speed, sc.density, sc.time_step
        N = [int(n) for n in sc.divisions]
        self.N = N
        mn = np.array([sc.domain_center[d] - h * float(N[d]) / 2.0 for d in range(3)])
        mx0 = np.array([sc.domain_center[d] + h * float(N[d]) / 2.0 for d in range(3)])
        for d in range(3):
            assert math.ceil(((mx0[d] - mn[d]) - 1e-10) / h) == N[d]
        mx = mn + h * np.asarray(N, dtype=np.float64)
        self.mn, self.mx = mn, mx
        self.cpos = [mn[d] + (0.5 + np.arange(N[d])) * h for d in range(3)]
        self.fpos = [(mn[d] - h / 2.0) + (0.5 + np.arange(N[d] + 1)) * h for d in range(3)]
        W = sc.pml_width * h
        S = sc.pml_strength

        preset = int(getattr(sc, "boundary_condition_preset", 0))
        self.preset = preset
        # sides that absorb, per axis (low, high): preset 0 all; 1 the low sides
        # and +y; 2 +z only (MAC_Grid.cpp:4027-4101)
        sides = {0: [(True, True)] * 3, 1: [(True, False), (True, True), (True, False)],
                 2: [(False, False), (False, False), (False, True)]}[preset]

        def sigma(x, d):
            hmin, hmax = x - mn[d], mx[d] - x
            out = np.zeros_like(x)
            lo = (hmin <= W) & sides[d][0]
            if preset == 2:  # the reference tests the low side first and returns 0 there
                hi = (hmin > W) & (hmax <= W) & sides[d][1]
            else:
                hi = (~(hmin <= W) if preset == 0 else ~lo) & (hmax <= W) & sides[d][1]
            with np.errstate(invalid="ignore", divide="ignore"):  # W = 0: 0/0 on the outer faces, as the reference
                out[lo] = S * ((W - hmin[lo]) ** 2) / (W * W)
                out[hi] = S * ((W - hmax[hi]) ** 2) / (W * W)
            return out

        def inside(x, d):
            return (((x - mn[d]) <= W + 1e-12) & sides[d][0]) | (((mx[d] - x) <= W + 1e-12) & sides[d][1])

        k = self.k
        self.pml_c = [inside(self.cpos[d], d) for d in range(3)]
        self.pml_f = [inside(self.fpos[d], d) for d in range(3)]
        sc_ = [sigma(self.cpos[d], d) for d in range(3)]
        sf_ = [sigma(self.fpos[d], d) for d in range(3)]
        self.pupd = [(1.0 / k - s / 2.0) / (1.0 / k + s / 2.0) for s in sc_]
        self.pdiv = [(-1.0 * self.rho * self.c * self.c) / (1.0 / k + s / 2.0) for s in sc_]
        self.vupd = [(1.0 / k - s / 2.0) / (1.0 / k + s / 2.0) for s in sf_]
        self.vgrad = [-1.0 / ((1.0 / k + s / 2.0) * (self.rho * h)) for s in sf_]
        X, Y, Z = np.meshgrid(*self.cpos, indexing="ij")
        self.X, self.Y, self.Z = X, Y, Z
        px, py, pz = np.meshgrid(*self.pml_c, indexing="ij")
        self.is_pml = px | py | pz
        # spheres: solid if centre or a +-h/4 sample is strictly inside (distance < 0)
        solid = np.zeros(N, dtype=bool)
        for o in sc.objects:
            assert o.shape == 0 and o.accel_kind == 0 and o.motion == 0
            c0 = np.asarray(o.center, dtype=np.float64)
            r = float(o.size[0])
            bmin, bmax = c0 - r, c0 + r
            dim, cen = bmax - bmin, (bmax + bmin) / 2.0

            def dist(x, y, z):
                inb = ((x < cen[0] + dim[0] * 1.1) & (x > cen[0] - dim[0] * 1.1) & (y < cen[1] + dim[1] * 1.1) &
                       (y > cen[1] - dim[1] * 1.1) & (z < cen[2] + dim[2] * 1.1) & (z > cen[2] - dim[2] * 1.1))
                d = np.sqrt((x - c0[0]) ** 2 + (y - c0[1]) ** 2 + (z - c0[2]) ** 2) - r
                return np.where(inb, d, np.finfo(np.float64).max)

            s = dist(X, Y, Z) < 0
            for ax in range(3):
                for sg in (1.0, -1.0):
                    P = [X, Y, Z]
                    P[ax] = P[ax] + sg * 0.25 * h
                    s |= dist(*P) < 0
            solid |= s
        self.bulk = ~solid
        # ghost-neighbour masks of bulk cells
        self.ghost_nb = {}
        for d in range(3):
            for sgn in (-1, 1):
                nb = np.zeros(N, dtype=bool)
                sl_dst = [slice(None)] * 3
                sl_src = [slice(None)] * 3
                if sgn > 0:
                    sl_dst[d], sl_src[d] = slice(0, N[d] - 1), slice(1, N[d])
                else:
                    sl_dst[d], sl_src[d] = slice(1, N[d]), slice(0, N[d] - 1)
                nb[tuple(sl_dst)] = solid[tuple(sl_src)]
                self.ghost_nb[(d, sgn)] = nb & self.bulk
        self.srcs = []
        for g in sc.sources:
            ws = g.width_space if g.width_space > 0 else self.c * g.width_time
            C = g.normalize_constant if g.normalize_constant != 0 else 1.0 / (math.sqrt(2.0 * math.pi) * ws) ** 3
            lo = np.asarray(g.position) - ws * 2.0
            hi = np.asarray(g.position) + ws * 2.0
            self.srcs.append((lo, hi, (hi + lo) / 2.0, ws, g.width_time, g.offset_time, C))
        self.p_prev = np.zeros(N)
        self.p_cur = np.zeros(N)
        self.p_spare = np.zeros(N)  # the third rotating buffer: the next pressure is written into it
        # boundary normals at offset 0 and 1 (ScalarField::boundaryCellNormal)
        idx = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")

        def normal(off):
            return np.stack([np.where(idx[d] == off, -1, np.where(idx[d] == N[d] - 1 - off, 1, 0)) for d in range(3)])

        self.idx = idx
        self.nml0, self.nml1 = normal(0), normal(1)
        edge0 = (self.nml0 != 0).any(axis=0)
        self.eng = self.bulk & ~self.is_pml & ~edge0 & (self.nml1 != 0).any(axis=0)
        self.edge0 = edge0
        self.pd = [np.zeros(N) for _ in range(3)]
        self.v = [np.zeros([N[e] + (1 if e == d else 0) for e in range(3)]) for d in range(3)]
        self.t = 0.0
        self.listeners = None if sc.listeners is None else np.asarray(sc.listeners, dtype=np.float64).reshape(-1, 3)

    def _shift(self, a, d, s):
        """a at index i+s along d, clamped to self at the domain edge."""
        out = a.copy()
        n = a.shape[d]
        dst = [slice(None)] * 3
        src = [slice(None)] * 3
        if s > 0:
            dst[d], src[d] = slice(0, n - 1), slice(1, n)
        else:
            dst[d], src[d] = slice(1, n), slice(0, n - 1)
        out[tuple(dst)] = a[tuple(src)]
        return out

    def step(self):
        N, h, k = self.N, self.h, self.k
        p = self.p_cur
        # velocities on PML faces (not the outer faces)
        for d in range(3):
            v = self.v[d]
            shape = v.shape
            pm = [self.pml_c[e] if e != d else self.pml_f[d] for e in range(3)]
            grids = np.meshgrid(*pm, indexing="ij")
            face_pml = grids[0] | grids[1] | grids[2]
            idx = [slice(None)] * 3
            idx[d] = slice(1, shape[d] - 1)
            idx = tuple(idx)
            sl_r = [slice(None)] * 3
            sl_l = [slice(None)] * 3
            sl_r[d] = slice(1, N[d])
            sl_l[d] = slice(0, N[d] - 1)
            pr, pl = p[tuple(sl_r)], p[tuple(sl_l)]
            shp = [1, 1, 1]
            shp[d] = shape[d] - 2
            upd = self.vupd[d][1:-1].reshape(shp)
            grad = self.vgrad[d][1:-1].reshape(shp)
            newv = v[idx] * upd
            newv = newv + grad * pr
            newv = newv - grad * pl
            m = face_pml[idx]
            v[idx] = np.where(m, newv, v[idx])
        # Laplacian with ghost faces (pg = p of the bulk cell itself)
        lap = np.zeros(N)
        surrounded = np.zeros(N, dtype=int)
        for d in range(3):
            pp = self._shift(p, d, +1)
            pn = self._shift(p, d, -1)
            gp = self.ghost_nb[(d, 1)]
            gn = self.ghost_nb[(d, -1)]
            both = gp & gn
            term = np.where(both, (p + p - 2.0 * p) / (9.0 / 16.0),
                            np.where(gp, (p + 0.75 * pn - (7.0 / 4.0) * p) / (21.0 / 32.0),
                                     np.where(gn, (0.75 * pp + p - (7.0 / 4.0) * p) / (21.0 / 32.0),
                                              pp + pn - 2.0 * p)))
            lap = lap + term
            surrounded += both
        lap = lap * (1.0 / (h * h))
        lap[~self.bulk] = 0.0
        c2k2 = (self.c * k) * (self.c * k)
        new = self.p_spare  # keeps its values where nothing writes (non-PML cells on the edge)
        interior = self.bulk & ~self.is_pml & ~self.edge0 & ~self.eng
        upd = 2.0 * p - self.p_prev + lap * c2k2
        cav = interior & (surrounded > 1)
        upd = np.where(cav, p, upd)
        if self.srcs:
            ts = self.t + 0.5 * k
            src = np.zeros(N)
            for lo, hi, cen, ws, wt, t0, C in self.srcs:
                inb = ((self.X < hi[0]) & (self.X > lo[0]) & (self.Y < hi[1]) & (self.Y > lo[1]) & (self.Z < hi[2]) &
                       (self.Z > lo[2]))
                val = (self.X - cen[0]) ** 2 + (self.Y - cen[1]) ** 2 + (self.Z - cen[2]) ** 2
                val = np.exp(-val / (2.0 * ws * ws))
                u = (ts - t0) / wt
                val = val * math.exp(-(u * u) / 2.0)
                val = val * (1.0 / 3.6836 * C)
                src = src + np.where(inb, val, 0.0)
            upd = upd + src * k
        new[interior] = upd[interior]
        if self.eng.any():
            e_new = self._engquist(p, self.p_prev)
            if self.srcs:
                e_new = e_new + (src * k)[self.eng]
            new[self.eng] = e_new
        # PML split pressures
        for d in range(3):
            shp = [1, 1, 1]
            shp[d] = N[d]
            sl_r = [slice(None)] * 3
            sl_l = [slice(None)] * 3
            sl_r[d] = slice(1, N[d] + 1)
            sl_l[d] = slice(0, N[d])
            vr, vl = self.v[d][tuple(sl_r)], self.v[d][tuple(sl_l)]
            div = self.pdiv[d].reshape(shp)
            a = self.pd[d] * self.pupd[d].reshape(shp)
            a = a + div * vr * (1.0 / h)
            a = a - div * vl * (1.0 / h)
            self.pd[d] = np.where(self.is_pml, a, self.pd[d])
        pml_sum = self.pd[0] + self.pd[1] + self.pd[2]
        new[self.is_pml] = pml_sum[self.is_pml]
        new[~self.bulk & ~self.is_pml] = 0.0
        self.p_spare, self.p_prev, self.p_cur = self.p_prev, p, new
        self.t += k
        return self.sample()

    def _engquist(self, pc, pl):
        """MAC_Grid.cpp:533-920 over every Engquist cell at once: p^{n+1} of the
        cells; the exterior values (zero on the diagonal) go into pc in place."""
        N = self.N
        lam = self.c * self.k / self.h
        lam2 = lam * lam
        cells = np.nonzero(self.eng)
        m = len(cells[0])
        X = np.stack(cells)                       # (3, m) coordinates
        nml = self.nml1[:, cells[0], cells[1], cells[2]]
        btype = np.abs(nml).sum(axis=0)
        out = np.zeros(m)
        writes = []

        def at(a, C):
            return a[C[0], C[1], C[2]]

        for t in (1, 2, 3):
            sel = np.nonzero(btype == t)[0]
            if len(sel) == 0:
                continue
            n = nml[:, sel]
            r = np.arange(len(sel))
            nz = np.abs(n) > 0
            if t == 1:
                di = np.argmax(nz, axis=0)
                dj, dk = (di + 1) % 3, (di + 2) % 3
            elif t == 2:
                di = np.argmax(nz, axis=0)
                dk = np.argmin(nz, axis=0)
                dj = 3 - di - dk
            else:
                di, dj, dk = np.zeros(len(sel), int), np.ones(len(sel), int), np.full(len(sel), 2)

            def shift(axis, amount, clamp=False):
                C = X[:, sel].copy()
                C[axis, r] = C[axis, r] + amount
                if clamp:
                    C[axis, r] = np.clip(C[axis, r], 0, np.asarray(N)[axis] - 1)
                return C

            ni, nj, nk = n[di, r], n[dj, r], n[dk, r]
            C0 = X[:, sel]
            pC, pL = at(pc, C0), at(pl, C0)
            if t == 1:
                Cip = shift(di, ni)
                pl_ii_p = at(pl, Cip)
                Cin = shift(di, -ni)
                p_ii_n, pl_ii_n = at(pc, Cin), at(pl, Cin)
                p_jj_p, p_jj_n = at(pc, shift(dj, 1, True)), at(pc, shift(dj, -1, True))
                p_kk_p, p_kk_n = at(pc, shift(dk, 1, True)), at(pc, shift(dk, -1, True))
                p1 = ((2. / lam2 + 4. / lam - 6. - 4. * lam) * pC - (1. / lam2 + 2. / lam) * pL + pl_ii_p - pl_ii_n
                      + 2. * p_ii_n + (lam + 1.) * (p_jj_p + p_jj_n + p_kk_p + p_kk_n))
                p1 = p1 * (lam2 / (1. + 2. * lam))
                x0 = (pl_ii_p + p_ii_n - pl_ii_n - 2. / lam * (p1 + pL - 2. * pC)
                      + lam * (p_jj_p + p_jj_n + p_kk_p + p_kk_n - 4. * pC))
                out[sel] = 2.0 * pC - pL + lam2 * (p_ii_n + p_jj_p + p_jj_n + p_kk_p + p_kk_n + x0 - 6. * pC)
                writes.append((Cip, x0))
            elif t == 2:
                p_ii_n, p_jj_n = at(pc, shift(di, -ni)), at(pc, shift(dj, -nj))
                p_kk_p, p_kk_n = at(pc, shift(dk, 1, True)), at(pc, shift(dk, -1, True))
                p1 = (2. / lam2 - 6.) * pC + (2.0 * lam - 1.0) / lam2 * pL + 2. * p_ii_n + 2. * p_jj_n + p_kk_p + p_kk_n
                p1 = p1 * (lam2 / (1. + 2. * lam))
                x0 = (pL - p1) / lam + p_ii_n
                x1 = (pL - p1) / lam + p_jj_n
                out[sel] = 2.0 * pC - pL + lam2 * (p_ii_n + p_jj_n + p_kk_p + p_kk_n + x0 + x1 - 6. * pC)
                Cd = shift(di, ni)
                Cd[dj, r] = Cd[dj, r] + nj
                writes += [(shift(di, ni), x0), (shift(dj, nj), x1), (Cd, np.zeros(len(sel)))]
            else:
                p_ii_n, p_jj_n, p_kk_n = at(pc, shift(0, -ni)), at(pc, shift(1, -nj)), at(pc, shift(2, -nk))
                p1 = (2. / lam2 - 6.) * pC + (3.0 * lam - 1.0) / lam2 * pL + 2. * p_ii_n + 2. * p_jj_n + 2. * p_kk_n
                p1 = p1 * (lam2 / (1. + 3. * lam))
                x0 = (pL - p1) / lam + p_ii_n
                x1 = (pL - p1) / lam + p_jj_n
                x2 = (pL - p1) / lam + p_kk_n
                out[sel] = 2.0 * pC - pL + lam2 * (p_ii_n + p_jj_n + p_kk_n + x0 + x1 + x2 - 6. * pC)
                Cd = X[:, sel] + n
                writes += [(shift(0, ni), x0), (shift(1, nj), x1), (shift(2, nk), x2), (Cd, np.zeros(len(sel)))]
        for C, v in writes:
            pc[C[0], C[1], C[2]] = v
        return out

    def sample(self):
        if self.listeners is None:
            return np.zeros(0)
        out = []
        N, h = self.N, self.h
        for pt in self.listeners:
            idx = []
            for d in range(3):
                diff = (pt[d] - self.mn[d]) - h / 2.0
                i0 = min(max(int(diff / h), 0), N[d] - 1)
                i1 = 0 if diff < 0 else min(i0 + 1, N[d] - 1)
                idx.append(sorted({i0, i1}))
            pts, vals = [], []
            for i in idx[0]:
                for j in idx[1]:
                    for kk in idx[2]:
                        assert self.bulk[i, j, kk], "listener stencil touches a solid cell"
                        pts.append([self.cpos[0][i], self.cpos[1][j], self.cpos[2][kk]])
                        vals.append(self.p_cur[i, j, kk])
            P = np.asarray(pts) - pt
            w = np.exp(-(P ** 2).sum(axis=1) / (2.0 * 0.018 * 0.018))
            A = np.column_stack([np.ones(len(P)), P]) * w[:, None]
            b = np.asarray(vals) * w
            c, *_ = np.linalg.lstsq(A, b, rcond=None)
            out.append(c[0])
        return np.asarray(out)
