"""Generates tests/golden/golden_s2M3.npz with a pure-Python loop restatement.

This is a second restatement of the reference, written independently of the C
oracle (oracle/dgv_oracle.c), loop for loop after the Fortran:

  grid and nodes ......... miscset.f90:433-470 (uniform mesh), 882-937, 1112-1183
  canonical cell ......... dgvtools_mod.f90:300-338, 1175-1247
  shift tables ........... miscset.f90:1202-1311
  Q (APlus) .............. collision_mod.f90:143-229
  mixed terms ............ collision_mod.f90:244-332
  spatial operator ....... spat_oper_mod.f90:28-68 (run_mode 0)
  RK2 / RK4 .............. time_integr_mod.f90:47-60, 86-104
  AB2 start-up + steps ... time_integr_mod.f90:443-569, 314-364
  moments / Maxwellian ... dgvtools_mod.f90:1437-1458, distributions_mod.f90:83-95

Gauss-Legendre nodes come from numpy.polynomial.legendre.leggauss.  The
A-arrays are the seeded synthetic records (prefilter of dgvtools_mod.f90:527 +
exact sphere/cell support, value w*w*|g|/8*u with u from splitmix64), also
restated here.  Grid: s=2 nodes per cell per axis, M=3 cells, [-3,3]^3 (N=216).

Run:  python tests/golden/make_golden.py      (about a minute)
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
S, M, L = 2, 3, 3.0
SEED = 20240611
KAPPA = 1.0
DT = 0.01
MASK64 = (1 << 64) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def synth_value(seed, p, i2, i3, w2, w3, dsph):
    k = (p << 48) ^ (i2 << 24) ^ i3
    h = splitmix64(k ^ splitmix64(seed))
    u = float(h >> 11) * (1.0 / 9007199254740992.0)
    u = 2.0 * u - 1.0
    return w2 * w3 * (dsph / 8.0) * u


class Grid:
    def __init__(self, s, m, lo, hi):
        self.s, self.M = s, m
        self.g = [lo + (hi - lo) / float(m) * float(i) for i in range(m + 1)]
        xg, wg = np.polynomial.legendre.leggauss(s)
        self.cells = []  # (lu, ru, lv, rv, lw, rw, ugi, vgi, wgi)
        for iu in range(m):
            for iv in range(m):
                for iw in range(m):
                    self.cells.append((self.g[iu], self.g[iu + 1], self.g[iv], self.g[iv + 1],
                                       self.g[iw], self.g[iw + 1], iu, iv, iw))
        self.u, self.v, self.w, self.wt, self.pc, self.ui, self.vi, self.wi = ([] for _ in range(8))
        for ic, (lu, ru, lv, rv, lw, rw, *_r) in enumerate(self.cells):
            for iu in range(s):
                uu = xg[iu] * (ru - lu) / 2.0 + (ru + lu) / 2.0
                qu = wg[iu]
                for iv in range(s):
                    vv = xg[iv] * (rv - lv) / 2.0 + (rv + lv) / 2.0
                    qv = wg[iv]
                    for iw in range(s):
                        ww = xg[iw] * (rw - lw) / 2.0 + (rw + lw) / 2.0
                        qw = wg[iw]
                        self.u.append(uu); self.v.append(vv); self.w.append(ww)
                        self.wt.append(qu * qv * qw * (ru - lu) * (rv - lv) * (rw - lw) / 8.0)
                        self.pc.append(ic); self.ui.append(iu); self.vi.append(iv); self.wi.append(iw)
        self.N = len(self.u)
        self.P = s ** 3
        self.ccell = self.find_cell(0.0, 0.0, 0.0)

    def find_cell(self, u, v, w):
        eps = 10e-11

        def axis(x):
            g = self.g
            if x < g[0] - eps or x > g[-1] + eps:
                return 0
            i = 1
            while x >= g[i - 1] - eps and i < len(g):
                i += 1
            return i
        ui, vi, wi = axis(u), axis(v), axis(w)
        return (ui - 2) * self.M * self.M + (vi - 2) * self.M + (wi - 2)


def synth_records(G, seed):
    cc = G.cells[G.ccell]
    uu, vv, ww = (cc[0], cc[1]), (cc[2], cc[3]), (cc[4], cc[5])
    dphi = math.sqrt((uu[1] - uu[0]) * (uu[1] - uu[0]) + (vv[1] - vv[0]) * (vv[1] - vv[0]) +
                     (ww[1] - ww[0]) * (ww[1] - ww[0]))
    lo, hi = (uu[0], vv[0], ww[0]), (uu[1], vv[1], ww[1])
    pairs = []
    for i2 in range(G.N):
        for i3 in range(i2 + 1, G.N):
            a, b, c = G.u[i2] - G.u[i3], G.v[i2] - G.v[i3], G.w[i2] - G.w[i3]
            dsph = math.sqrt(a * a + b * b + c * c)
            p = G.u[i2] + G.u[i3] - uu[0] - uu[1]
            q = G.v[i2] + G.v[i3] - vv[0] - vv[1]
            r = G.w[i2] + G.w[i3] - ww[0] - ww[1]
            dist2 = math.sqrt(p * p + q * q + r * r)
            if dist2 > dsph + dphi or dist2 + dphi < dsph:
                continue
            m = ((G.u[i2] + G.u[i3]) / 2.0, (G.v[i2] + G.v[i3]) / 2.0, (G.w[i2] + G.w[i3]) / 2.0)
            dmin = dmax = 0.0
            for k in range(3):
                aa, bb = lo[k] - m[k], m[k] - hi[k]
                t = aa if aa > 0.0 else (bb if bb > 0.0 else 0.0)
                dmin += t * t
                fa, fb = abs(m[k] - lo[k]), abs(m[k] - hi[k])
                fm = fa if fa > fb else fb
                dmax += fm * fm
            rad = dsph / 2.0
            if not (rad * rad >= dmin and rad * rad <= dmax):
                continue
            pairs.append((i2, i3, dsph))
    capphi = [0] * G.N
    A, xi, xi1 = [], [], []
    for p in range(G.P):
        capphi[G.ccell * G.P + p] = len(pairs)
        for i2, i3, dsph in pairs:
            A.append(synth_value(seed, p, i2, i3, G.wt[i2], G.wt[i3], dsph))
            xi.append(i2 + 1)
            xi1.append(i3 + 1)
    return capphi, A, xi, xi1


class RefState:
    """Module state after SetCellsUGINdsSftArrs; 1-based record indices."""

    def __init__(self, G, capphi, A, xi, xi1):
        self.G, self.capphi, self.A, self.xi, self.xi1 = G, capphi, A, xi, xi1
        cc = G.cells[G.ccell]
        self.dui, self.dvi, self.dwi, self.phican, self.Ashift = [], [], [], [], []
        pre = [0]
        for k in capphi:
            pre.append(pre[-1] + k)
        for iphi in range(G.N):
            pcl = G.cells[G.pc[iphi]]
            self.dui.append(pcl[6] - cc[6]); self.dvi.append(pcl[7] - cc[7]); self.dwi.append(pcl[8] - cc[8])
            ph = G.ccell * G.P + G.ui[iphi] * G.s * G.s + G.vi[iphi] * G.s + G.wi[iphi]
            self.phican.append(ph)
            self.Ashift.append(pre[ph])

    def _shift(self, k, du, dv, dw):
        G = self.G
        c = G.cells[G.pc[k]]
        iu, iv, iw = c[6] + du, c[7] + dv, c[8] + dw
        if not (0 <= iu < G.M and 0 <= iv < G.M and 0 <= iw < G.M):
            return -1
        return (iu * G.M * G.M + iv * G.M + iw) * G.P + G.ui[k] * G.s * G.s + G.vi[k] * G.s + G.wi[k]

    def _loop(self, iphi):
        sh, cap = self.Ashift[iphi], self.capphi[self.phican[iphi]]
        du, dv, dw = self.dui[iphi], self.dvi[iphi], self.dwi[iphi]
        for j in range(sh, sh + cap):
            a = self._shift(self.xi[j] - 1, du, dv, dw)
            if a < 0:
                continue
            b = self._shift(self.xi1[j] - 1, du, dv, dw)
            if b < 0:
                continue
            yield a, b, self.A[j]

    def aplus(self, f):
        fc = np.zeros(self.G.N)
        for iphi in range(self.G.N):
            acc = 0.0
            for a, b, Aj in self._loop(iphi):
                acc = acc + 2 * f[a] * f[b] * Aj
            fc[iphi] = acc / self.G.wt[iphi]
        return fc

    def mixed(self, f, fm):
        fc = np.zeros(self.G.N)
        for iphi in range(self.G.N):
            acc = 0.0
            for a, b, Aj in self._loop(iphi):
                acc = acc + (fm[a] * f[b] + f[a] * fm[b]) * Aj
            fc[iphi] = 2 * acc / self.G.wt[iphi]
        return fc

    def spatial(self, f, dt):
        return self.aplus(f) * (KAPPA * dt)

    def rk2(self, f, dt):
        frhs1 = self.spatial(f, dt)
        ft2 = self.spatial(f + frhs1 * 2 / 3.0, dt)
        f = f + frhs1 / 4.0 + ft2 * 3.0 / 4
        return f, frhs1 / dt

    def rk4(self, f, dt):
        frhs1 = self.spatial(f, dt)
        ft2 = self.spatial(f + frhs1 / 2.0, dt)
        ft3 = self.spatial(f + frhs1 / 4.0 + ft2 / 4.0, dt)
        ft2 = self.spatial(f - ft2 + ft3 * 2, dt)
        f = f + frhs1 / 6.0 + ft3 * 2 / 3.0 + ft2 / 6.0
        return f, frhs1 / dt

    def moments(self, f):
        G = self.G
        wt, u, v, w = (np.array(x) for x in (G.wt, G.u, G.v, G.w))
        n = sum(f[i] * wt[i] for i in range(G.N))
        ub = sum(f[i] * wt[i] * u[i] for i in range(G.N)) / n
        vb = sum(f[i] * wt[i] * v[i] for i in range(G.N)) / n
        wb = sum(f[i] * wt[i] * w[i] for i in range(G.N)) / n
        t = sum(f[i] * wt[i] * ((u[i] - ub) ** 2 + (v[i] - vb) ** 2 + (w[i] - wb) ** 2) for i in range(G.N))
        return np.array([n, ub, vb, wb, t / n / 3.0 * 2.0])


def maxwellian(G, T, u0, v0, w0, n):
    beta = math.sqrt(math.pi * T) * (math.pi * T)
    return np.array([n * math.exp(-((G.u[i] - u0) ** 2 + (G.v[i] - v0) ** 2 + (G.w[i] - w0) ** 2) /
                                  max(T, 0.0000001)) / beta for i in range(G.N)])


def main(out=os.path.join(HERE, "golden_s2M3.npz")):
    G = Grid(S, M, -L, L)
    capphi, A, xi, xi1 = synth_records(G, SEED)
    st = RefState(G, capphi, A, xi, xi1)
    f0 = maxwellian(G, 0.6, 0.8, 0.0, 0.0, 0.5) + maxwellian(G, 0.6, -0.8, 0.1, 0.0, 0.5)
    fm = maxwellian(G, 0.7, 0.0, 0.0, 0.0, 1.0)
    q0 = st.aplus(f0)
    mixed = st.mixed(f0 - fm, fm)
    f_rk2 = f0.copy()
    rk2_traj = []
    for _ in range(3):
        f_rk2, r = st.rk2(f_rk2, DT)
        rk2_traj.append(f_rk2.copy())
    f_rk4, _ = st.rk4(f0.copy(), DT)
    # AB2: PrepareMTS_SH_DGV (one RK2 step filling frhs1), then two MTS steps
    f_ab, frhs1 = st.rk2(f0.copy(), DT)
    ab_traj = []
    for _ in range(2):
        frhs2 = frhs1
        fc = st.spatial(f_ab, DT)
        f_ab = f_ab + fc * 3.0 / 2.0 - DT * frhs2 / 2.0
        frhs1 = fc / DT
        ab_traj.append(f_ab.copy())
    np.savez_compressed(
        out, s=S, M=M, L=L, seed=SEED, kappa=KAPPA, dt=DT,
        nodes_u=np.array(G.u), nodes_v=np.array(G.v), nodes_w=np.array(G.w), nodes_gwts=np.array(G.wt),
        ccell=G.ccell, capphi=np.array(capphi, np.int32), A=np.array(A), A_xi=np.array(xi, np.int32),
        A_xi1=np.array(xi1, np.int32), Ashift=np.array(st.Ashift, np.int64),
        dui=np.array(st.dui, np.int32), phican=np.array(st.phican, np.int32),
        f0=f0, fm=fm, q0=q0, mixed=mixed, rk2_traj=np.array(rk2_traj), rk4_1=f_rk4,
        ab2_traj=np.array(ab_traj), moments0=st.moments(f0))
    print("wrote", out, "records", len(A))


if __name__ == "__main__":
    main()
