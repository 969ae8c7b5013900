// Host check of the hand-derived vector-Jacobian products of gral_b200/csrc/adj_level.cuh: for
// random level configurations, inputs and cotangents, the VJP (in double) must equal the central
// difference of the forward row along random directions.  Prints one line per component and
// exits non-zero on a mismatch.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "adj_level.cuh"

using namespace gral::adj;

namespace {

LevelConst random_level(std::mt19937_64 &rng, int &k) {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    LevelConst c{};
    c.KK = (int)(u(rng) * 6);
    const int ks[] = {c.KK + 1, c.KK + 2, c.KK + 3, c.KK + 7, c.KK + 12};
    k = ks[(int)(u(rng) * 5)];
    c.k = k;
    c.kad = c.KK + 1 + (int)(u(rng) * 8);
    c.wlo = c.KK + 1 - (int)(u(rng) * 3);
    c.whi = c.KK + 1 + (int)(u(rng) * 3);
    c.dz = (float)(1.0 + 2.0 * u(rng));
    c.dxk = 2.0f;
    c.dyk = (float)(2.0 + u(rng));
    c.dxdz = c.dxk * c.dz;
    c.dydz = c.dyk * c.dz;
    c.area = c.dxk * c.dyk;
    c.ap0 = (float)(1.0 + 10.0 * u(rng));
    c.vishmin = (u(rng) < 0.5) ? 0.0f : 0.01f;
    c.cor = 1.0e-4f;
    c.geo = (float)(2.0 * u(rng) - 1.0);
    c.hokK = (float)(2.0 * c.KK);
    c.hok = c.hokK + (float)(c.k - c.KK) * c.dz;
    c.cov = (u(rng) < 0.3) ? (float)u(rng) : 0.0f;
    c.help_t = 0.2f;
    c.help_o = 0.15f;
    uint32_t fl = 0;
    if (u(rng) < 0.5) fl |= LF_VEG;
    if (u(rng) < 0.5) fl |= LF_CUTKLT1;
    if (u(rng) < 0.5) fl |= LF_Z0GE;
    if (u(rng) < 0.2) fl |= LF_BS;
    if (u(rng) < 0.2) fl |= LF_BN;
    if (u(rng) < 0.2) fl |= LF_BW;
    if (u(rng) < 0.2) fl |= LF_BE;
    c.fl = fl;
    return c;
}

template <class F, class G>
int check(const char *name, int n, F row, G vjp, std::mt19937_64 &rng) {
    std::normal_distribution<double> nd(0.0, 1.0);
    int bad = 0;
    double worst = 0.0;
    for (int trial = 0; trial < 4000; ++trial) {
        int k = 0;
        const LevelConst c = random_level(rng, k);
        std::vector<double> x(n), v(n), g(n, 0.0), xp(n), xm(n);
        for (int q = 0; q < n; ++q) x[q] = 1.5 * nd(rng);
        x[0] = 2.0 * nd(rng);
        double l[4];
        for (double &z : l) z = nd(rng);
        vjp(c, x.data(), l, g.data());
        for (int dir = 0; dir < 3; ++dir) {
            for (int q = 0; q < n; ++q) v[q] = nd(rng);
            const double h = 1e-6;
            for (int q = 0; q < n; ++q) { xp[q] = x[q] + h * v[q]; xm[q] = x[q] - h * v[q]; }
            double op[8], om[8];
            row(c, xp.data(), op);
            row(c, xm.data(), om);
            double fd = 0.0, ad = 0.0, scale = 0.0;
            for (int r = 0; r < 4; ++r) fd += l[r] * (op[r] - om[r]) / (2 * h);
            // the neighbour coefficients are dD/dn: check them against differences of D
            double o0[8];
            row(c, x.data(), o0);
            for (int r = 0; r < 4; ++r) {
                const int q = n - 4 + r;
                std::vector<double> yp(x), ym(x);
                yp[q] += h; ym[q] -= h;
                double a1[8], a2[8];
                row(c, yp.data(), a1);
                row(c, ym.data(), a2);
                const double want = (a1[3] - a2[3]) / (2 * h);
                if (std::fabs(want - o0[4 + r]) > 1e-6 * (1.0 + std::fabs(want))) {
                    if (bad < 5) std::printf("%s neighbour coefficient %d: %.12g vs %.12g\n", name, r, o0[4 + r], want);
                    ++bad;
                }
            }
            for (int q = 0; q < n; ++q) { ad += g[q] * v[q]; scale += std::fabs(g[q] * v[q]); }
            const double err = std::fabs(fd - ad) / std::max(scale, 1e-12);
            worst = std::max(worst, err);
            if (err > 1e-5) {
                if (bad < 5)
                    std::printf("%s mismatch: trial %d k=%d KK=%d kad=%d fl=%x fd=%.12g ad=%.12g\n", name, trial, c.k,
                                c.KK, c.kad, c.fl, fd, ad);
                ++bad;
            }
        }
    }
    std::printf("%s: worst relative difference %.3g, %d mismatches\n", name, worst, bad);
    return bad;
}

}  // namespace

int main() {
    std::mt19937_64 rng(12345);
    int bad = 0;
    bad += check("U", U_COUNT, [](const LevelConst &c, const double *x, double *o) { u_row(c, x, o); },
                 [](const LevelConst &c, const double *x, const double *l, double *g) { u_row_vjp(c, x, l, g); }, rng);
    bad += check("V", V_COUNT, [](const LevelConst &c, const double *x, double *o) { v_row(c, x, o); },
                 [](const LevelConst &c, const double *x, const double *l, double *g) { v_row_vjp(c, x, l, g); }, rng);
    bad += check("W", W_COUNT, [](const LevelConst &c, const double *x, double *o) { w_row(c, x, o); },
                 [](const LevelConst &c, const double *x, const double *l, double *g) { w_row_vjp(c, x, l, g); }, rng);
    return bad ? 1 : 0;
}
