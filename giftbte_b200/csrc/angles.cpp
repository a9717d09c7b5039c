// Angular quadrature, as GiftBTE's BTEAngle (src/BTEAngle/BTEAngle.cpp:11-190):
//   method 1 (CADOM): uniform midpoint rule; 2D material: 4*nphi in-plane
//     directions of weight 2pi/(4 nphi); 3D: 8*ntheta*nphi directions with
//     the solid-angle weight 2|sin th| sin(dth/2) dphi.
//   method 2 (Gauss): Gauss-Legendre in phi on [0, pi/2] mirrored into four
//     quadrants (2D), times Gauss-Legendre in cos(theta) on [-1, 0] mirrored
//     to [0, 1] (3D).
// The modal weight used by the solver is weight / SolidAngle
// (StaticBTESynthetic.cpp:610). Gauss nodes come from Newton iteration on the
// Legendre polynomial started at the Chebyshev points, stopped at 2^-52
// (src/utility/utility.cpp:116-172).
#include <cmath>
#include <vector>

#include "gbte_internal.h"

namespace gbte {
namespace {

void gauss_legendre(double a, double b, int n, std::vector<double> &x, std::vector<double> &w) {
    const int N = n - 1, N1 = n, N2 = n + 1;
    std::vector<double> y(N1), yprev(N1, 2.0), dP(N1);
    std::vector<double> Lm(N2);
    for (int i = 0; i < N1; i++) y[i] = std::cos((2 * (N - i) + 1) * M_PI / (2 * N + 2));
    auto moved = [&]() {
        double r = 0;
        for (int i = 0; i < N1; i++) r = std::fmax(std::fabs(y[i] - yprev[i]), r);
        return r;
    };
    std::vector<double> Pn(N1), Pn1(N1);
    while (moved() > std::pow(2.0, -52)) {
        for (int i = 0; i < N1; i++) {
            // three-term recurrence up to P_{N+1}
            Lm[0] = 1;
            Lm[1] = y[i];
            for (int j = 2; j < N2; j++) Lm[j] = ((2 * j - 1) * y[i] * Lm[j - 1] - (j - 1) * Lm[j - 2]) / j;
            Pn[i] = Lm[N1 - 1];
            Pn1[i] = Lm[N2 - 1];
        }
        for (int i = 0; i < N1; i++) {
            dP[i] = N2 * (Pn[i] - y[i] * Pn1[i]) / (1 - y[i] * y[i]);
            yprev[i] = y[i];
            y[i] = yprev[i] - Pn1[i] / dP[i];
        }
    }
    x.resize(N1);
    w.resize(N1);
    for (int i = 0; i < N1; i++) {
        x[i] = (a * (1 - y[i]) + b * (1 + y[i])) / 2;
        w[i] = (b - a) / ((1 - y[i] * y[i]) * dP[i] * dP[i]) * N2 / N1 * N2 / N1;
    }
}

}  // namespace

Error explicit_angles(int n, const double *xyz, const double *weight, double solid, Angles &A) {
    A = Angles();
    if (n <= 0 || !xyz || !weight) return {-1, "explicit angles: need num_directions > 0, direction_xyz and weight"};
    if (!(solid > 0)) return {-1, "explicit angles: solid_angle must be positive"};
    A.nd = n;
    A.solid = solid;
    for (int d = 0; d < n; d++) {
        A.sx.push_back(xyz[3 * d]);
        A.sy.push_back(xyz[3 * d + 1]);
        A.sz.push_back(xyz[3 * d + 2]);
        A.w.push_back(weight[d] / solid);
    }
    return {0, ""};
}

Error make_angles(int method, int ntheta, int nphi, int dm, Angles &A) {
    A = Angles();
    if (nphi <= 0 || (dm == 3 && ntheta <= 0)) return {-1, "Ntheta/Nphi must be positive"};
    if (dm != 2 && dm != 3) return {-1, "MaterialDimension must be 2 or 3"};
    std::vector<double> wt;
    auto push = [&](double x, double y, double z, double w) {
        A.sx.push_back(x);
        A.sy.push_back(y);
        A.sz.push_back(z);
        wt.push_back(w);
    };
    if (method == 1) {
        if (dm == 2) {
            A.solid = 2 * M_PI;
            int n = 4 * nphi;
            double dphi = 0.5 * M_PI / nphi, phi = 0.5 * dphi;
            for (int i = 0; i < n; i++) {
                if (i > 0) phi = phi + dphi;
                push(std::cos(phi), std::sin(phi), 0, A.solid / n);
            }
        } else {
            A.solid = 4 * M_PI;
            double dth = 0.5 * M_PI / ntheta, dphi = 0.5 * M_PI / nphi;
            std::vector<double> th(2 * ntheta), ph(4 * nphi);
            th[0] = 0.5 * dth;
            ph[0] = 0.5 * dphi;
            for (int i = 1; i < 2 * ntheta; i++) th[i] = th[i - 1] + dth;
            for (int i = 1; i < 4 * nphi; i++) ph[i] = ph[i - 1] + dphi;
            for (int t = 0; t < 2 * ntheta; t++)
                for (int p = 0; p < 4 * nphi; p++)
                    push(std::sin(th[t]) * std::cos(ph[p]), std::sin(th[t]) * std::sin(ph[p]), std::cos(th[t]),
                         2. * std::fabs(std::sin(th[t])) * std::sin(0.5 * dth) * dphi);
        }
    } else {
        std::vector<double> gx, gw;
        gauss_legendre(0, M_PI / 2, nphi, gx, gw);
        // in-plane cosines/sines mirrored into four quadrants
        std::vector<double> cp, sp, wp;
        for (int i = 0; i < nphi; i++) {
            cp.push_back(std::cos(gx[i]));
            wp.push_back(gw[i]);
            sp.push_back(std::pow(1 - cp[i] * cp[i], 0.5));
        }
        for (int i = nphi - 1; i >= 0; i--) {
            cp.push_back(-std::cos(gx[i]));
            wp.push_back(gw[i]);
            sp.push_back(std::pow(1 - cp[i] * cp[i], 0.5));
        }
        for (int i = 0; i < nphi; i++) {
            cp.push_back(-std::cos(gx[i]));
            wp.push_back(gw[i]);
            sp.push_back(-std::pow(1 - cp[i] * cp[i], 0.5));
        }
        for (int i = nphi - 1; i >= 0; i--) {
            cp.push_back(std::cos(gx[i]));
            wp.push_back(gw[i]);
            sp.push_back(-std::pow(1 - cp[i] * cp[i], 0.5));
        }
        if (dm == 2) {
            A.solid = 2 * M_PI;
            for (int i = 0; i < 4 * nphi; i++) push(cp[i], sp[i], 0, wp[i]);
        } else {
            A.solid = 4 * M_PI;
            std::vector<double> tx, tw;
            gauss_legendre(-1, 0, ntheta, tx, tw);
            std::vector<double> ct, st, wt_;
            for (int i = 0; i < ntheta; i++) {
                ct.push_back(-tx[i]);
                wt_.push_back(tw[i]);
                st.push_back(std::pow(1 - ct[i] * ct[i], 0.5));
            }
            for (int i = ntheta - 1; i >= 0; i--) {
                ct.push_back(tx[i]);
                wt_.push_back(tw[i]);
                st.push_back(std::pow(1 - ct[i] * ct[i], 0.5));
            }
            for (int t = 0; t < 2 * ntheta; t++)
                for (int p = 0; p < 4 * nphi; p++) push(st[t] * cp[p], st[t] * sp[p], ct[t], wt_[t] * wp[p]);
        }
    }
    A.nd = (int)A.sx.size();
    A.w.resize(A.nd);
    for (int d = 0; d < A.nd; d++) A.w[d] = wt[d] / A.solid;
    return {0, ""};
}

}  // namespace gbte
