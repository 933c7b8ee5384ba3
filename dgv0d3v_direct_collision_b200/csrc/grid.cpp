// grid.cpp -- uniform velocity grid, nodes and weights of the nodal-DG
// discretisation.  Restates SetDGblzmGnodes / SetDGVblzmmesh /
// Set3DCellsR_DGVblzm / SetNodesDGV (miscset.f90:29-208, 210-470, 544-597,
// 882-937, 1112-1183) for a single uniform grid, and the canonical-cell search
// FindCellContainsPoint_DGV + finduiviwi (dgvtools_mod.f90:300-338, 1175-1247).
// Compiled with -ffp-contract=off: the expressions keep the reference's
// operation order so node coordinates are reproducible bit for bit.
#include <cmath>

#include "dgv_internal.h"

namespace dgv {

// Gauss-Legendre nodes (ascending) and weights on [-1,1]: Newton iteration on
// the three-term Legendre recurrence from Chebyshev-like initial guesses.
static void gauss_legendre(int n, double *x, double *w)
{
    const double pi = 3.141592653589793238462643;
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }
    int half = (n + 1) / 2;
    for (int i = 0; i < half; i++) {
        double z = std::cos(pi * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1; p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; k++) {
            double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1; p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
        w[n - 1 - i] = w[i];
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// index (1-based) of the right end point of the interval holding x, 0 if off
// the grid; `bound` is the array size the reference's loop compares with
static int find_axis(const std::vector<double> &g, int bound, double x)
{
    const double eps = 10e-11;
    int npts = (int)g.size();
    if (x < g[0] - eps || x > g[npts - 1] + eps) return 0;
    int i = 1;
    while (x >= g[i - 1] - eps && i < bound) i++;
    return i;
}

int build_grid(const dgv_grid_desc &d, Grid &g, std::string &err)
{
    if (d.su < 1 || d.sv < 1 || d.sw < 1 || d.Mu < 1 || d.Mv < 1 || d.Mw < 1) {
        err = "grid: node and cell counts must be positive";
        return DGV_EINVAL;
    }
    if (d.su * d.sv * d.sw > 255) {
        err = "grid: at most 255 nodes per cell";
        return DGV_EUNSUP;
    }
    if (d.Mu > 127 || d.Mv > 127 || d.Mw > 127) {
        err = "grid: at most 127 cells per axis";
        return DGV_EUNSUP;
    }
    if (!(d.u_R > d.u_L) || !(d.v_R > d.v_L) || !(d.w_R > d.w_L)) {
        err = "grid: empty velocity box";
        return DGV_EINVAL;
    }
    g.d = d;
    g.P = d.su * d.sv * d.sw;
    g.Nc = d.Mu * d.Mv * d.Mw;
    g.N = (long long)g.P * g.Nc;
    auto mesh = [](int M, double L, double R, std::vector<double> &out) {
        out.resize(M + 1);
        for (int i = 0; i <= M; i++) out[i] = L + (R - L) / (double)M * (double)i;
    };
    mesh(d.Mu, d.u_L, d.u_R, g.gu);
    mesh(d.Mv, d.v_L, d.v_R, g.gv);
    mesh(d.Mw, d.w_L, d.w_R, g.gw);
    g.xu.resize(d.su); g.wu.resize(d.su); gauss_legendre(d.su, g.xu.data(), g.wu.data());
    g.xv.resize(d.sv); g.wv.resize(d.sv); gauss_legendre(d.sv, g.xv.data(), g.wv.data());
    g.xw.resize(d.sw); g.ww.resize(d.sw); gauss_legendre(d.sw, g.xw.data(), g.ww.data());
    int Nc = g.Nc;
    g.lu.resize(Nc); g.ru.resize(Nc); g.lv.resize(Nc); g.rv.resize(Nc); g.lw.resize(Nc); g.rw.resize(Nc);
    int m = 0;
    for (int iu = 0; iu < d.Mu; iu++)
        for (int iv = 0; iv < d.Mv; iv++)
            for (int iw = 0; iw < d.Mw; iw++, m++) {
                g.lu[m] = g.gu[iu]; g.ru[m] = g.gu[iu + 1];
                g.lv[m] = g.gv[iv]; g.rv[m] = g.gv[iv + 1];
                g.lw[m] = g.gw[iw]; g.rw[m] = g.gw[iw + 1];
            }
    long long N = g.N;
    g.nu.resize(N); g.nv.resize(N); g.nw.resize(N); g.nwt.resize(N);
    long long j = 0;
    for (int ic = 0; ic < Nc; ic++)
        for (int iu = 0; iu < d.su; iu++) {
            double ru = g.xu[iu] * (g.ru[ic] - g.lu[ic]) / 2.0 + (g.ru[ic] + g.lu[ic]) / 2.0;
            double qu = g.wu[iu];
            for (int iv = 0; iv < d.sv; iv++) {
                double rv = g.xv[iv] * (g.rv[ic] - g.lv[ic]) / 2.0 + (g.rv[ic] + g.lv[ic]) / 2.0;
                double qv = g.wv[iv];
                for (int iw = 0; iw < d.sw; iw++, j++) {
                    double rw = g.xw[iw] * (g.rw[ic] - g.lw[ic]) / 2.0 + (g.rw[ic] + g.lw[ic]) / 2.0;
                    double qw = g.ww[iw];
                    g.nu[j] = ru; g.nv[j] = rv; g.nw[j] = rw;
                    g.nwt[j] = qu * qv * qw * (g.ru[ic] - g.lu[ic]) * (g.rv[ic] - g.lv[ic]) *
                               (g.rw[ic] - g.lw[ic]) / 8.0;
                }
            }
        }
    // canonical cell: the one containing v = 0; the v search is bounded by
    // size(grids_u) as in the reference
    int ui = find_axis(g.gu, d.Mu + 1, 0.0);
    int vi = find_axis(g.gv, d.Mu + 1, 0.0);
    int wi = find_axis(g.gw, d.Mw + 1, 0.0);
    if (ui * vi * wi == 0) {
        err = "grid: v = 0 is not inside the velocity box (no canonical cell)";
        return DGV_EINVAL;
    }
    g.ccu = ui - 2; g.ccv = vi - 2; g.ccw = wi - 2;
    if (g.ccv >= d.Mv) {
        err = "grid: canonical-cell search left the v grid";
        return DGV_EINVAL;
    }
    g.ccell = (g.ccu * d.Mv + g.ccv) * d.Mw + g.ccw;
    return DGV_OK;
}

}  // namespace dgv
