// ORACLE — test infrastructure, never shipped and never on the product path.
//
// A sequential FP64 CPU restatement of GiftBTE's steady synthetic-accelerated
// source iteration (Order=2, IterativeScheme=Synthetic, MatrixSolver=LU),
// written from the reference's behaviour so that the CUDA implementation can
// be checked against it on the same inputs. It re-derives, in its own
// data layout:
//   * mesh topology and geometry       src/BTEMesh/BTEMesh.cpp:600-844 (2D),
//                                      :845-1023 (boundaries, periodic pairs,
//                                      face list), Distribute.cpp:150-197
//                                      (undefined boundaries -> type 1, T=0)
//   * angular quadrature               src/BTEAngle/BTEAngle.cpp:11-190,
//                                      src/utility/utility.cpp:116-172
//   * the solver                       src/StaticBTESynthetic/
//                                      StaticBTESyntheticSolver.cpp:12-247 and
//                                      StaticBTESynthetic.cpp (functions cited
//                                      at each routine below)
// The transport solve A d = R (an Eigen SparseLU in the reference) is done
// exactly by forward substitution in upwind topological order, with
// Gauss-Seidel to machine precision on any cyclic remainder. The macro
// (Fourier) system is solved exactly by a reverse-Cuthill-McKee-ordered
// banded LU. Pinned against the compiled reference (oracle/_ref/BTE_CPU) on
// 2D decks by tests/test_oracle_pin.py. The 3D branch follows the
// dimension-generic formulas of the reference; the reference's own 3D mesh
// code is stripped from its public release, so 3D parity is unpinned.
// Two extensions without a reference counterpart, each reducing to the
// reference at its neutral value: a per-cell scattering multiplier s_c (the
// transport uses tau / s_c in cell c; s_c = 1 is the reference) and the
// partially specular wall, type 6 with value p (p = 0 and p = 1 become the
// reference's types 2 and 3).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <vector>

namespace {

struct V3 {
    double x = 0, y = 0, z = 0;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double dist(V3 a, V3 b) {
    return std::sqrt(std::pow(a.x - b.x, 2) + std::pow(a.y - b.y, 2) + std::pow(a.z - b.z, 2));
}

struct Face {
    std::vector<int> v;
    double area = 0;
    V3 n, c;
    int neighbor = -1, bound = -1, index = -1;
};
struct Cell {
    std::vector<int> v;
    std::vector<Face> f;
    double vol = 0;
    V3 c;
    int region = 0, matter = 0;
    double heat = 0;
};
struct Bnd {
    int tag = 0, bc = -1, type = 0, connect = -1;
    double T = 0;
    std::vector<int> cell, face;
};

bool has(const std::vector<int> &a, int x) { return std::find(a.begin(), a.end(), x) != a.end(); }

double heron(V3 a, V3 b, V3 c) {  // get_tri_area, utility.cpp:88-95
    double la = dist(a, b), lb = dist(b, c), lc = dist(a, c);
    double p = (la + lb + lc) / 2;
    return std::sqrt(p * (p - la) * (p - lb) * (p - lc));
}

// Gauss-Legendre nodes/weights on [a,b] (utility.cpp:116-172), Newton on P_N.
std::vector<double> gauss_points(double a, double b, int N) {
    N = N - 1;
    int N1 = N + 1, N2 = N + 2;
    std::vector<double> y(N1), y0(N1, 2.0), Lp(N1), g;
    std::vector<std::vector<double>> L(N1, std::vector<double>(N2));
    for (int i = 0; i < N1; i++) {
        L[i][0] = 1;
        y[i] = std::cos((2 * (N - i) + 1) * M_PI / (2 * N + 2));
    }
    auto margin = [&]() {
        double r = 0;
        for (int i = 0; i < N1; i++) r = std::max(std::fabs(y[i] - y0[i]), r);
        return r;
    };
    while (margin() > std::pow(2, -52)) {
        for (int i = 0; i < N1; i++) L[i][1] = y[i];
        for (int j = 2; j < N1 + 1; j++)
            for (int i = 0; i < N1; i++) L[i][j] = ((2 * j - 1) * y[i] * L[i][j - 1] - (j - 1) * L[i][j - 2]) / j;
        for (int i = 0; i < N1; i++) {
            Lp[i] = (N2) * (L[i][N1 - 1] - y[i] * L[i][N2 - 1]) / (1 - y[i] * y[i]);
            y0[i] = y[i];
            y[i] = y0[i] - L[i][N2 - 1] / Lp[i];
        }
    }
    for (int i = 0; i < N1; i++) {
        g.push_back((a * (1 - y[i]) + b * (1 + y[i])) / 2);
        g.push_back((b - a) / ((1 - y[i] * y[i]) * Lp[i] * Lp[i]) * N2 / N1 * N2 / N1);
    }
    return g;
}

// BTEAngle.cpp:11-190
void make_angles(int method, int ntheta, int nphi, int dm, std::vector<V3> &dir, std::vector<double> &w,
                 double &solid) {
    dir.clear();
    w.clear();
    if (method == 1) {
        if (dm == 2) {
            solid = 2 * M_PI;
            int n = 4 * nphi;
            double dphi = 0.5 * M_PI / nphi;
            std::vector<double> phi(n);
            phi[0] = 0.5 * dphi;
            for (int i = 1; i < n; i++) phi[i] = phi[i - 1] + dphi;
            for (int i = 0; i < n; i++) {
                w.push_back(solid / n);
                dir.push_back({std::cos(phi[i]), std::sin(phi[i]), 0});
            }
        } else {
            solid = 4 * M_PI;
            double dth = 0.5 * M_PI / ntheta, dphi = 0.5 * M_PI / nphi;
            std::vector<double> th(2 * ntheta), phi(4 * nphi);
            th[0] = 0.5 * dth;
            phi[0] = 0.5 * dphi;
            for (int i = 1; i < 2 * ntheta; i++) th[i] = th[i - 1] + dth;
            for (int i = 1; i < 4 * nphi; i++) phi[i] = phi[i - 1] + dphi;
            for (int t = 0; t < 2 * ntheta; t++)
                for (int p = 0; p < 4 * nphi; p++) {
                    w.push_back(2. * std::fabs(std::sin(th[t])) * std::sin(0.5 * dth) * dphi);
                    dir.push_back({std::sin(th[t]) * std::cos(phi[p]), std::sin(th[t]) * std::sin(phi[p]),
                                   std::cos(th[t])});
                }
        }
    } else {
        if (dm == 2) {
            solid = 2 * M_PI;
            std::vector<double> cs, sn, W;
            std::vector<double> g = gauss_points(0, M_PI / 2, nphi);
            for (int i = 0; i < nphi; i++) {
                cs.push_back(std::cos(g[2 * i]));
                W.push_back(g[2 * i + 1]);
                sn.push_back(std::pow(1 - cs[i] * cs[i], 0.5));
            }
            for (int i = nphi - 1; i >= 0; i--) {
                cs.push_back(-std::cos(g[2 * i]));
                W.push_back(g[2 * i + 1]);
                sn.push_back(std::pow(1 - cs[i] * cs[i], 0.5));
            }
            for (int i = 0; i < nphi; i++) {
                cs.push_back(-std::cos(g[2 * i]));
                W.push_back(g[2 * i + 1]);
                sn.push_back(-std::pow(1 - cs[i] * cs[i], 0.5));
            }
            for (int i = nphi - 1; i >= 0; i--) {
                cs.push_back(std::cos(g[2 * i]));
                W.push_back(g[2 * i + 1]);
                sn.push_back(-std::pow(1 - cs[i] * cs[i], 0.5));
            }
            for (int i = 0; i < 4 * nphi; i++) {
                w.push_back(W[i]);
                dir.push_back({cs[i], sn[i], 0});
            }
        } else {
            solid = 4 * M_PI;
            std::vector<double> ct, cp, st, sp, W, Wp;
            std::vector<double> g = gauss_points(-1, 0, ntheta), gp = gauss_points(0, M_PI / 2, nphi);
            for (int i = 0; i < ntheta; i++) {
                ct.push_back(-g[2 * i]);
                W.push_back(g[2 * i + 1]);
                st.push_back(std::pow(1 - ct[i] * ct[i], 0.5));
            }
            for (int i = ntheta - 1; i >= 0; i--) {
                ct.push_back(g[2 * i]);
                W.push_back(g[2 * i + 1]);
                st.push_back(std::pow(1 - ct[i] * ct[i], 0.5));
            }
            for (int i = 0; i < nphi; i++) {
                cp.push_back(std::cos(gp[2 * i]));
                Wp.push_back(gp[2 * i + 1]);
                sp.push_back(std::pow(1 - cp[i] * cp[i], 0.5));
            }
            for (int i = nphi - 1; i >= 0; i--) {
                cp.push_back(-std::cos(gp[2 * i]));
                Wp.push_back(gp[2 * i + 1]);
                sp.push_back(std::pow(1 - cp[i] * cp[i], 0.5));
            }
            for (int i = 0; i < nphi; i++) {
                cp.push_back(-std::cos(gp[2 * i]));
                Wp.push_back(gp[2 * i + 1]);
                sp.push_back(-std::pow(1 - cp[i] * cp[i], 0.5));
            }
            for (int i = nphi - 1; i >= 0; i--) {
                cp.push_back(std::cos(gp[2 * i]));
                Wp.push_back(gp[2 * i + 1]);
                sp.push_back(-std::pow(1 - cp[i] * cp[i], 0.5));
            }
            for (int t = 0; t < 2 * ntheta; t++)
                for (int p = 0; p < 4 * nphi; p++) {
                    w.push_back(W[t] * Wp[p]);
                    dir.push_back({st[t] * cp[p], st[t] * sp[p], ct[t]});
                }
        }
    }
}

// (J^T J)^-1 J^T for a k x dim J (utility.cpp:401-549); out[r][j].
void lsq_pinv(const std::vector<std::vector<double>> &J, int dim, std::vector<std::vector<double>> &out) {
    int k = (int)J.size();
    out.assign(3, std::vector<double>(k, 0.0));
    double M[3][3] = {{0}};
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++)
            for (int r = 0; r < k; r++) M[i][j] += J[r][i] * J[r][j];
    double Ni[3][3] = {{0}};
    if (dim == 2) {
        double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        Ni[0][0] = M[1][1] / det;
        Ni[0][1] = -M[0][1] / det;
        Ni[1][1] = M[0][0] / det;
        Ni[1][0] = -M[1][0] / det;
    } else {
        double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) +
                     M[0][1] * (M[1][2] * M[2][0] - M[1][0] * M[2][2]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        Ni[0][0] = 1.0 / det * (M[1][1] * M[2][2] - M[1][2] * M[2][1]);
        Ni[1][0] = 1.0 / det * (M[0][2] * M[2][1] - M[0][1] * M[2][2]);
        Ni[2][0] = 1.0 / det * (M[0][1] * M[1][2] - M[0][2] * M[1][1]);
        Ni[0][1] = 1.0 / det * (M[1][2] * M[2][0] - M[1][0] * M[2][2]);
        Ni[1][1] = 1.0 / det * (M[0][0] * M[2][2] - M[0][2] * M[2][0]);
        Ni[2][1] = 1.0 / det * (M[1][0] * M[0][2] - M[0][0] * M[1][2]);
        Ni[0][2] = 1.0 / det * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        Ni[1][2] = 1.0 / det * (M[0][1] * M[2][0] - M[0][0] * M[2][1]);
        Ni[2][2] = 1.0 / det * (M[0][0] * M[1][1] - M[1][0] * M[0][1]);
    }
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < k; j++) {
            double s = 0;
            for (int q = 0; q < dim; q++) s += Ni[i][q] * J[j][q];
            out[i][j] = s;
        }
}

// Banded LU without pivoting on a reverse-Cuthill-McKee ordering. The macro
// matrix is a weakly diagonally dominant M-matrix, so no pivoting is needed.
struct BandLU {
    int n = 0, bw = 0;
    std::vector<int> perm, iperm;
    std::vector<double> a;  // row-major band: a[i*(2bw+1) + (j-i+bw)]
    double &at(int i, int j) { return a[(size_t)i * (2 * bw + 1) + (j - i + bw)]; }
    void factor(int N, const std::vector<std::vector<std::pair<int, double>>> &rows) {
        n = N;
        // RCM from a minimum-degree start
        std::vector<std::vector<int>> adj(n);
        for (int i = 0; i < n; i++)
            for (auto &e : rows[i])
                if (e.first != i) {
                    adj[i].push_back(e.first);
                    adj[e.first].push_back(i);
                }
        for (auto &l : adj) {
            std::sort(l.begin(), l.end());
            l.erase(std::unique(l.begin(), l.end()), l.end());
        }
        std::vector<int> order;
        std::vector<char> seen(n, 0);
        while ((int)order.size() < n) {
            int s = -1;
            for (int i = 0; i < n; i++)
                if (!seen[i] && (s < 0 || adj[i].size() < adj[s].size())) s = i;
            std::queue<int> q;
            q.push(s);
            seen[s] = 1;
            while (!q.empty()) {
                int u = q.front();
                q.pop();
                order.push_back(u);
                std::vector<int> nb;
                for (int x : adj[u])
                    if (!seen[x]) nb.push_back(x);
                std::sort(nb.begin(), nb.end(), [&](int a1, int b1) { return adj[a1].size() < adj[b1].size(); });
                for (int x : nb) {
                    seen[x] = 1;
                    q.push(x);
                }
            }
        }
        std::reverse(order.begin(), order.end());
        perm = order;  // new -> old
        iperm.assign(n, 0);
        for (int i = 0; i < n; i++) iperm[perm[i]] = i;
        bw = 0;
        for (int i = 0; i < n; i++)
            for (auto &e : rows[i]) bw = std::max(bw, std::abs(iperm[i] - iperm[e.first]));
        a.assign((size_t)n * (2 * bw + 1), 0.0);
        for (int i = 0; i < n; i++)
            for (auto &e : rows[i]) at(iperm[i], iperm[e.first]) += e.second;
        for (int k = 0; k < n; k++) {
            double piv = at(k, k);
            int hi = std::min(n - 1, k + bw);
            for (int i = k + 1; i <= hi; i++) {
                double &lik = at(i, k);
                if (lik == 0) continue;
                lik /= piv;
                for (int j = k + 1; j <= hi; j++) at(i, j) -= lik * at(k, j);
            }
        }
    }
    void solve(const std::vector<double> &b, std::vector<double> &x) {
        std::vector<double> y(n);
        for (int i = 0; i < n; i++) y[i] = b[perm[i]];
        for (int i = 0; i < n; i++) {
            int lo = std::max(0, i - bw);
            double s = y[i];
            for (int j = lo; j < i; j++) s -= at(i, j) * y[j];
            y[i] = s;
        }
        for (int i = n - 1; i >= 0; i--) {
            int hi = std::min(n - 1, i + bw);
            double s = y[i];
            for (int j = i + 1; j <= hi; j++) s -= at(i, j) * y[j];
            y[i] = s / at(i, i);
        }
        x.assign(n, 0);
        for (int i = 0; i < n; i++) x[perm[i]] = y[i];
    }
};

struct Oracle {
    int dim = 2, nmat = 1, nb = 1, nd = 1, nc = 0, nn = 0;
    double Lx = 1;
    std::vector<V3> node;
    std::vector<std::vector<int>> node_cells;
    std::vector<Cell> cell;
    std::vector<Bnd> bnd;
    // face list (BTEMesh.cpp:987-1021)
    std::vector<int> fb;                        // Boundindex
    std::vector<std::array<int, 2>> fcell, fface;
    // bands, angles
    std::vector<double> vg, tau, C, lat, hr;    // [mat*nb + b]
    std::vector<double> kappa, capb;
    std::vector<V3> dir;
    std::vector<double> mw;                     // weight / SolidAngle
    // solver state
    std::vector<std::vector<int>> nbr;          // elementNeighborList
    std::vector<std::vector<std::vector<double>>> cellW;  // CellMatrix[c][3][k]
    std::vector<std::vector<std::vector<double>>> faceW;  // FaceMatrix[f][3][nv]
    std::vector<std::vector<double>> e;         // [p][nc], p = d*nb + b
    std::vector<double> ebound;                 // [b][d][ib][2]
    std::vector<double> T, Told, Tlat, Tband, E, qx, qy, qz, qxo, qyo, qzo, ReMacro, heat;
    std::vector<double> tsc;                    // 1 / s_c: per-cell relaxation-time scale (extension, 1 = reference)
    int order = 2;                              // 1: solve_firstorder (zero face gradients)
    bool sequential = false;                    // IterativeScheme=Sequential: no macro correction
    std::vector<std::array<double, 2>> bTmacro;
    double errOld = 0, errOldq = 0, err = 0, errq = 0;
    int errInc = 0;
    double inner_last = 0;
    int use_limiter = 0;
    BandLU macroLU;

    V3 v(int m, int b, int d) const {
        double s = vg[m * nb + b];
        return {s * dir[d].x, s * dir[d].y, s * dir[d].z};
    }
    double &eb(int b, int d, int ib, int ic) { return ebound[(((size_t)b * nd + d) * bnd.size() + ib) * 2 + ic]; }
    int P() const { return nb * nd; }
};

// ---------------------------------------------------------------- mesh ----
// BTEMesh::setMeshParams (BTEMesh.cpp:668-842) for 2D; tets for 3D.
int build_mesh(Oracle &o, int dim, int nn, const double *xyz, int nc, const int *cptr, const int *cverts,
               const int *creg, int nbe, const int *bptr, const int *bverts, const int *btag, int nbc,
               const int *bc_tag, const int *bc_type, const double *bc_val, const int *reg_mat, int nreg) {
    o.dim = dim;
    o.nn = nn;
    o.nc = nc;
    o.node.resize(nn);
    for (int i = 0; i < nn; i++) o.node[i] = {xyz[3 * i], xyz[3 * i + 1], dim == 2 ? 0.0 : xyz[3 * i + 2]};
    o.cell.assign(nc, Cell());
    for (int i = 0; i < nc; i++) {
        Cell &c = o.cell[i];
        c.v.assign(cverts + cptr[i], cverts + cptr[i + 1]);
        c.region = creg[i];
        if (c.region < 0 || c.region >= nreg) return -1;
        c.matter = reg_mat[c.region];
    }
    for (int i = 0; i < nc; i++) {
        Cell &c = o.cell[i];
        auto &N = o.node;
        if (dim == 2) {
            if (c.v.size() == 3) {
                c.vol = heron(N[c.v[0]], N[c.v[1]], N[c.v[2]]);
                c.c = {((N[c.v[0]].x + N[c.v[1]].x) + N[c.v[2]].x) / 3, ((N[c.v[0]].y + N[c.v[1]].y) + N[c.v[2]].y) / 3,
                       ((N[c.v[0]].z + N[c.v[1]].z) + N[c.v[2]].z) / 3};
                c.f.resize(3);
                for (int j = 0; j < 3; j++) c.f[j].v = {c.v[(j + 1) % 3], c.v[(j + 2) % 3]};
            } else if (c.v.size() == 4) {
                c.vol = heron(N[c.v[0]], N[c.v[1]], N[c.v[2]]) + heron(N[c.v[1]], N[c.v[2]], N[c.v[3]]);
                c.c = {((N[c.v[0]].x + N[c.v[1]].x) + N[c.v[2]].x + N[c.v[3]].x) / 4,
                       ((N[c.v[0]].y + N[c.v[1]].y) + N[c.v[2]].y + N[c.v[3]].y) / 4,
                       ((N[c.v[0]].z + N[c.v[1]].z) + N[c.v[2]].z + N[c.v[3]].z) / 4};
                c.f.resize(4);
                c.f[0].v = {c.v[0], c.v[1]};
                c.f[1].v = {c.v[1], c.v[3]};
                c.f[2].v = {c.v[3], c.v[2]};
                c.f[3].v = {c.v[2], c.v[0]};
            } else
                return -1;
            for (auto &f : c.f) {
                V3 a0 = N[f.v[0]], a1 = N[f.v[1]];
                f.area = dist(a0, a1);
                f.c = {(a0.x + a1.x) / 2, (a0.y + a1.y) / 2, (a0.z + a1.z) / 2};
                V3 a = sub(a0, a1);
                a = {a.x / f.area, a.y / f.area, a.z / f.area};
                f.n = {a.y, -a.x, 0};
                if (dot(sub(c.c, f.c), f.n) > 0) f.n = {-f.n.x, -f.n.y, f.n.z};
            }
        } else {
            if (c.v.size() != 4) return -1;
            V3 p[4];
            for (int k = 0; k < 4; k++) p[k] = N[c.v[k]];
            V3 a = sub(p[1], p[0]), b = sub(p[2], p[0]), d = sub(p[3], p[0]);
            double det = a.x * (b.y * d.z - b.z * d.y) - a.y * (b.x * d.z - b.z * d.x) + a.z * (b.x * d.y - b.y * d.x);
            c.vol = std::fabs(det) / 6.0;
            c.c = {(p[0].x + p[1].x + p[2].x + p[3].x) / 4, (p[0].y + p[1].y + p[2].y + p[3].y) / 4,
                   (p[0].z + p[1].z + p[2].z + p[3].z) / 4};
            c.f.resize(4);
            for (int j = 0; j < 4; j++) {
                Face &f = c.f[j];
                f.v = {c.v[(j + 1) % 4], c.v[(j + 2) % 4], c.v[(j + 3) % 4]};
                V3 q0 = N[f.v[0]], q1 = N[f.v[1]], q2 = N[f.v[2]];
                f.area = heron(q0, q1, q2);
                f.c = {(q0.x + q1.x + q2.x) / 3, (q0.y + q1.y + q2.y) / 3, (q0.z + q1.z + q2.z) / 3};
                V3 u = sub(q1, q0), w = sub(q2, q0);
                V3 cr = {u.y * w.z - u.z * w.y, u.z * w.x - u.x * w.z, u.x * w.y - u.y * w.x};
                double l = std::sqrt(dot(cr, cr));
                f.n = {cr.x / l, cr.y / l, cr.z / l};
                if (dot(sub(c.c, f.c), f.n) > 0) f.n = {-f.n.x, -f.n.y, -f.n.z};
            }
        }
    }
    o.node_cells.assign(nn, {});
    for (int i = 0; i < nc; i++)
        for (int vtx : o.cell[i].v) o.node_cells[vtx].push_back(i);
    for (int i = 0; i < nc; i++)
        for (auto &f : o.cell[i].f) {
            f.neighbor = -1;
            for (int k : o.node_cells[f.v[0]]) {
                if (k == i) continue;
                bool all = true;
                for (int vv : f.v) all = all && has(o.cell[k].v, vv);
                if (all) f.neighbor = k;
            }
            f.bound = -1;
        }
    // boundary elements -> (cell, face) sides (BTEMesh.cpp:812-833)
    struct RawB {
        int tag;
        std::vector<int> cells, faces;
    };
    std::vector<RawB> raw(nbe);
    for (int i = 0; i < nbe; i++) {
        std::vector<int> bv(bverts + bptr[i], bverts + bptr[i + 1]);
        raw[i].tag = btag[i];
        for (int idx : o.node_cells[bv[0]]) {
            for (int k = 0; k < (int)o.cell[idx].f.size(); k++) {
                const auto &fv = o.cell[idx].f[k].v;
                bool all = true;
                for (int x : bv) all = all && has(fv, x);
                if (all) {
                    raw[i].cells.push_back(idx);
                    raw[i].faces.push_back(k);
                }
            }
        }
    }
    // BCs + undefined boundaries (Distribute.cpp:150-197)
    std::vector<int> tags(bc_tag, bc_tag + nbc), types(bc_type, bc_type + nbc);
    std::vector<double> vals(bc_val, bc_val + nbc);
    std::vector<int> nodefine;
    for (auto &r : raw) {
        bool set = has(tags, r.tag) || r.cells.size() == 2;
        if (!set && !has(nodefine, r.tag)) nodefine.push_back(r.tag);
    }
    for (int t : nodefine) {
        tags.push_back(t);
        types.push_back(1);
        vals.push_back(0.0);
    }
    // setMeshParams1 (BTEMesh.cpp:845-866)
    o.bnd.clear();
    for (auto &r : raw)
        for (int j = 0; j < (int)tags.size(); j++)
            if (r.tag == tags[j]) {
                Bnd b;
                b.tag = r.tag;
                b.bc = j;
                b.cell = r.cells;
                b.face = r.faces;
                b.type = types[j];
                b.T = vals[j];
                // extension: partially specular wall (type 6, value = p); its
                // ends are the reference's diffuse and specular walls
                if (b.type == 6) {
                    if (!(b.T >= 0 && b.T <= 1)) return -4;
                    if (b.T == 0) b.type = 2;
                    else if (b.T == 1) b.type = 3;
                }
                o.bnd.push_back(b);
            }
    for (int i = 0; i < (int)o.bnd.size(); i++)
        for (int j = 0; j < (int)o.bnd[i].cell.size(); j++) o.cell[o.bnd[i].cell[j]].f[o.bnd[i].face[j]].bound = i;
    for (auto &c : o.cell)
        for (auto &f : c.f)
            if (f.bound == -1 && f.neighbor == -1) return -2;
    // periodic pairing by nearest face centre (BTEMesh.cpp:903-925)
    for (auto &b : o.bnd) {
        b.connect = -1;
        if (types[b.bc] < 0) {
            double best = 1000;
            for (int j = 0; j < (int)o.bnd.size(); j++) {
                if (tags[b.bc] == -types[o.bnd[j].bc]) {
                    double d1 = dist(o.cell[b.cell[0]].f[b.face[0]].c, o.cell[o.bnd[j].cell[0]].f[o.bnd[j].face[0]].c);
                    if (d1 < best) {
                        best = d1;
                        b.connect = j;
                    }
                }
            }
            if (b.connect < 0) return -3;
        }
    }
    // face list (BTEMesh.cpp:987-1021)
    std::vector<std::vector<int>> isin(nc);
    for (int i = 0; i < nc; i++) isin[i].assign(o.cell[i].f.size(), 1);
    o.fb.clear();
    o.fcell.clear();
    o.fface.clear();
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < (int)o.cell[i].f.size(); j++) {
            if (!isin[i][j]) continue;
            std::array<int, 2> fc = {i, -1}, ff = {j, -1};
            int idx = (int)o.fb.size();
            o.cell[i].f[j].index = idx;
            if (o.cell[i].f[j].bound == -1) {
                int nbc_ = o.cell[i].f[j].neighbor;
                fc[1] = nbc_;
                for (int k = 0; k < (int)o.cell[nbc_].f.size(); k++)
                    if (o.cell[nbc_].f[k].neighbor == i) {
                        ff[1] = k;
                        isin[nbc_][k] = 0;
                        o.cell[nbc_].f[k].index = idx;
                    }
            }
            o.fb.push_back(o.cell[i].f[j].bound);
            o.fcell.push_back(fc);
            o.fface.push_back(ff);
        }
    return 0;
}

// ------------------------------------------------------------- solver -----
// _get_CellMatrix_larger (StaticBTESynthetic.cpp:967-1025) + neighbour lists (:453-465)
void setup_lsq(Oracle &o) {
    o.nbr.assign(o.nc, {});
    for (int i = 0; i < o.nc; i++)
        for (int vtx : o.cell[i].v)
            for (int k : o.node_cells[vtx])
                if (!has(o.nbr[i], k) && o.cell[k].matter == o.cell[i].matter && k != i) o.nbr[i].push_back(k);
    o.cellW.assign(o.nc, {});
    for (int i = 0; i < o.nc; i++) {
        int k = (int)o.nbr[i].size();
        std::vector<std::vector<double>> J(k, std::vector<double>(o.dim));
        for (int j = 0; j < k; j++) {
            J[j][0] = 1.0 / o.Lx * (o.cell[o.nbr[i][j]].c.x - o.cell[i].c.x);
            J[j][1] = 1.0 / o.Lx * (o.cell[o.nbr[i][j]].c.y - o.cell[i].c.y);
            if (o.dim == 3) J[j][2] = 1.0 / o.Lx * (o.cell[o.nbr[i][j]].c.z - o.cell[i].c.z);
        }
        bool ok = (o.dim == 2) ? (k > 2) : (k > 3);
        if (ok)
            lsq_pinv(J, o.dim, o.cellW[i]);
        else
            o.cellW[i].assign(3, std::vector<double>(k, 0.0));
    }
    // _get_face_matrix (StaticBTESynthetic.cpp:1617-1649), 3D only
    o.faceW.assign(o.fb.size(), {});
    if (o.dim == 3)
        for (size_t f = 0; f < o.fb.size(); f++) {
            const Face &F = o.cell[o.fcell[f][0]].f[o.fface[f][0]];
            int nv = (int)F.v.size();
            std::vector<std::vector<double>> J(nv, std::vector<double>(3));
            J[0] = {F.n.x, F.n.y, F.n.z};
            for (int m = 0; m < nv - 1; m++) {
                V3 a = o.node[F.v[m + 1]], b = o.node[F.v[m]];
                J[m + 1] = {1.0 / o.Lx * (a.x - b.x), 1.0 / o.Lx * (a.y - b.y), 1.0 / o.Lx * (a.z - b.z)};
            }
            lsq_pinv(J, 3, o.faceW[f]);
        }
}

// _get_gradient_larger (StaticBTESynthetic.cpp:1243-1424); limiter optional
void gradient(const Oracle &o, const std::vector<double> &e, int b, int d, std::vector<V3> &g, std::vector<double> &lim) {
    g.assign(o.nc, V3());
    lim.assign(o.nc, 1.0);
    if (o.order == 1) return;  // solve_firstorder: gradients stay zero (StaticBTESyntheticSolver.cpp:530-535)
    for (int i = 0; i < o.nc; i++) {
        int k = (int)o.nbr[i].size();
        if (k < 3) continue;
        V3 s;
        for (int m = 0; m < k; m++) {
            double d1 = 1.0 / o.Lx * (e[o.nbr[i][m]] - e[i]);
            s.x += o.cellW[i][0][m] * d1;
            s.y += o.cellW[i][1][m] * d1;
            if (o.dim == 3) s.z += o.cellW[i][2][m] * d1;
        }
        if (std::isnan(s.x) || std::isnan(s.y) || std::isnan(s.z)) s = V3();
        g[i] = s;
    }
    if (o.use_limiter == 1) {
        Oracle &oo = const_cast<Oracle &>(o);
        for (int i = 0; i < o.nc; i++) {
            const Cell &c = o.cell[i];
            double mx = e[i], mn = e[i];
            V3 vv = o.v(c.matter, b, d);
            for (int j = 0; j < (int)c.f.size(); j++) {
                const Face &f = c.f[j];
                if (f.bound == -1) {
                    mx = std::max(mx, e[f.neighbor]);
                    mn = std::min(mn, e[f.neighbor]);
                } else if (o.bnd[f.bound].type != 3 && dot(vv, f.n) < 0) {
                    double x = oo.eb(b, d, f.bound, 0);
                    mx = std::max(mx, x);
                    mn = std::min(mn, x);
                }
            }
            for (int j = 0; j < (int)c.f.size(); j++) {
                V3 a = sub(c.f[j].c, c.c);
                double gd = dot(g[i], a);
                if (gd * lim[i] + e[i] < mn) {
                    double y = (mn - e[i]) / gd;
                    lim[i] = (y * y + 2 * y) / (y * y + y + 2);
                }
                if (gd * lim[i] + e[i] > mx) {
                    double y = (mx - e[i]) / gd;
                    lim[i] = (y * y + 2 * y) / (y * y + y + 2);
                }
            }
        }
    }
}

struct PairWork {
    std::vector<V3> g;
    std::vector<double> lim, R, eV;
    std::vector<V3> gf;  // face gradients [2*nf]
};

// one (band, direction): gradient, _get_Re, exact solve, _get_bound_ee,
// _set_vertex_energydensity, _get_face_gradient, _get_non_fourier
void bte_pair(Oracle &o, int b, int d, PairWork &w, std::vector<double> &remacro_acc) {
    const int nc = o.nc;
    int p = d * o.nb + b;
    std::vector<double> &e = o.e[p];
    gradient(o, e, b, d, w.g, w.lim);
    // _get_Re (StaticBTESynthetic.cpp:1427-1500)
    w.R.assign(nc, 0.0);
    for (int ie = 0; ie < nc; ie++) {
        const Cell &c = o.cell[ie];
        int m = c.matter;
        V3 vv = o.v(m, b, d);
        double t = o.tau[m * o.nb + b] * o.tsc[ie];
        for (const Face &f : c.f) {
            double dp = dot(vv, f.n);
            double temp = t * f.area / c.vol * dp;
            if (dp >= 0) {
                V3 a = sub(f.c, c.c);
                w.R[ie] -= temp * (e[ie] + dot(a, w.g[ie]) * w.lim[ie]);
            } else if (f.bound == -1) {
                int nbc = f.neighbor;
                V3 a = sub(f.c, o.cell[nbc].c);
                w.R[ie] -= temp * (e[nbc] + dot(a, w.g[nbc]) * w.lim[nbc]);
            }
        }
        w.R[ie] += o.Told[ie] * o.C[m * o.nb + b];
        w.R[ie] += c.heat * o.hr[m * o.nb + b] * t;
        w.R[ie] -= e[ie];
    }
    for (int ib = 0; ib < (int)o.bnd.size(); ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
            int ie = o.bnd[ib].cell[ic];
            const Cell &c = o.cell[ie];
            const Face &f = c.f[o.bnd[ib].face[ic]];
            V3 vv = o.v(c.matter, b, d);
            double dp = dot(vv, f.n);
            if (dp < 0) {
                double temp = o.tau[c.matter * o.nb + b] * o.tsc[ie] * f.area / c.vol * dp;
                w.R[ie] -= temp * o.eb(b, d, ib, ic);
            }
        }
    // exact solve of the first-order upwind system (_get_coefficient :784-840)
    {
        std::vector<double> diag(nc, 1.0);
        std::vector<std::vector<std::pair<int, double>>> low(nc);
        std::vector<int> indeg(nc, 0);
        std::vector<std::vector<int>> outs(nc);
        for (int ie = 0; ie < nc; ie++) {
            const Cell &c = o.cell[ie];
            V3 vv = o.v(c.matter, b, d);
            double t = o.tau[c.matter * o.nb + b] * o.tsc[ie];
            double vd = 0;
            for (const Face &f : c.f) {
                double dp = dot(vv, f.n);
                double temp = t * f.area / c.vol * dp;
                if (dp >= 0)
                    vd += temp;
                else if (f.bound == -1) {
                    low[ie].push_back({f.neighbor, temp});
                    indeg[ie]++;
                    outs[f.neighbor].push_back(ie);
                }
            }
            diag[ie] = vd + 1.0;
        }
        std::vector<double> x(nc, 0.0);
        std::vector<char> done(nc, 0);
        std::queue<int> q;
        for (int i = 0; i < nc; i++)
            if (indeg[i] == 0) q.push(i);
        int ndone = 0;
        while (!q.empty()) {
            int i = q.front();
            q.pop();
            double s = w.R[i];
            for (auto &l : low[i]) s -= l.second * x[l.first];
            x[i] = s / diag[i];
            done[i] = 1;
            ndone++;
            for (int k : outs[i])
                if (--indeg[k] == 0) q.push(k);
        }
        if (ndone < nc) {  // cyclic remainder: Gauss-Seidel to machine precision
            for (int it = 0; it < 100000; it++) {
                double ch = 0, mag = 0;
                for (int i = 0; i < nc; i++) {
                    if (done[i]) continue;
                    double s = w.R[i];
                    for (auto &l : low[i]) s -= l.second * x[l.first];
                    double xn = s / diag[i];
                    ch = std::max(ch, std::fabs(xn - x[i]));
                    mag = std::max(mag, std::fabs(xn));
                    x[i] = xn;
                }
                if (ch <= 1e-17 * mag) break;
            }
        }
        for (int i = 0; i < nc; i++) e[i] = x[i] + e[i];
    }
    // _get_bound_ee (:1502-1539): outgoing with the pre-solve gradient
    for (int ib = 0; ib < (int)o.bnd.size(); ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
            int ie = o.bnd[ib].cell[ic];
            const Cell &c = o.cell[ie];
            const Face &f = c.f[o.bnd[ib].face[ic]];
            if (dot(o.v(c.matter, b, d), f.n) >= 0) {
                V3 a = sub(f.c, c.c);
                o.eb(b, d, ib, ic) = e[ie] + dot(a, w.g[ie]) * w.lim[ie];
            }
        }
    // _set_vertex_energydensity (:1541-1616)
    const int M = o.nmat;
    std::vector<double> tmp(o.nn * M, 0.0), rn(o.nn * M, 0.0);
    for (int i = 0; i < nc; i++)
        for (int vtx : o.cell[i].v) {
            double ds = dist(o.node[vtx], o.cell[i].c);
            tmp[vtx * M + o.cell[i].matter] += e[i] / ds;
            rn[vtx * M + o.cell[i].matter] += 1.0 / ds;
        }
    for (int ib = 0; ib < (int)o.bnd.size(); ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
            int i = o.bnd[ib].cell[ic];
            for (int vtx : o.cell[i].f[o.bnd[ib].face[ic]].v) {
                tmp[vtx * M + o.cell[i].matter] = 0;
                rn[vtx * M + o.cell[i].matter] = 0;
            }
        }
    for (int ib = 0; ib < (int)o.bnd.size(); ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
            int i = o.bnd[ib].cell[ic];
            const Face &f = o.cell[i].f[o.bnd[ib].face[ic]];
            for (int vtx : f.v) {
                double ds = dist(o.node[vtx], f.c);
                tmp[vtx * M + o.cell[i].matter] += o.eb(b, d, ib, ic) / ds;
                rn[vtx * M + o.cell[i].matter] += 1.0 / ds;
            }
        }
    w.eV.assign(o.nn * M, 0.0);
    for (int i = 0; i < o.nn * M; i++) {
        w.eV[i] = tmp[i] / rn[i];
        if (std::isnan(w.eV[i])) w.eV[i] = 0;
    }
    // _get_face_gradient (:1651-1781)
    const int nf = (int)o.fb.size();
    w.gf.assign(2 * nf, V3());
    auto tang = [&](const Face &F, int f, int slotm, bool bug) {
        V3 t;
        if (o.dim == 2) {
            int v0 = F.v[0], v1 = F.v[1];
            double mX = o.node[v1].x - o.node[v0].x, mY = o.node[v1].y - o.node[v0].y;
            double e1 = bug ? w.eV[v1] : w.eV[v1 * M + slotm], e0 = bug ? w.eV[v0] : w.eV[v0 * M + slotm];
            t.x = (e1 - e0) / (mX * mX + mY * mY) * mX;
            t.y = (e1 - e0) / (mX * mX + mY * mY) * mY;
        } else {
            int nv = (int)F.v.size();
            std::vector<double> d1(nv, 0.0);
            for (int m = 0; m < nv - 1; m++) {
                double e1 = bug ? w.eV[F.v[m + 1]] : w.eV[F.v[m + 1] * M + slotm];
                double e0 = bug ? w.eV[F.v[m]] : w.eV[F.v[m] * M + slotm];
                d1[m + 1] = 1.0 / o.Lx * (e1 - e0);
            }
            for (int m = 0; m < nv; m++) {
                t.x += o.faceW[f][0][m] * d1[m];
                t.y += o.faceW[f][1][m] * d1[m];
                t.z += o.faceW[f][2][m] * d1[m];
            }
        }
        return t;
    };
    for (int f = 0; f < nf; f++) {
        if (o.fb[f] == -1) {
            int i = o.fcell[f][0], j = o.fface[f][0], i2 = o.fcell[f][1];
            const Face &F = o.cell[i].f[j];
            V3 a = sub(o.cell[i2].c, o.cell[i].c);
            double gn = (e[i2] - e[i]) * dot(a, F.n) / dot(a, a);
            V3 t = tang(F, f, o.cell[i].matter, false);
            V3 gg = {gn * F.n.x + t.x, gn * F.n.y + t.y, gn * F.n.z + t.z};
            w.gf[2 * f] = gg;
            w.gf[2 * f + 1] = gg;
        } else if (o.bnd[o.fb[f]].type != 3) {
            for (int icell = 0; icell < 2; icell++) {
                int ie = o.fcell[f][icell];
                if (ie < 0) continue;
                int jf = o.fface[f][icell];
                int ibcell = 0;
                const Bnd &B = o.bnd[o.fb[f]];
                for (int ik = 0; ik < 2; ik++)
                    if (ik < (int)B.cell.size() ? B.cell[ik] == ie : -1 == ie) ibcell = ik;
                const Face &F = o.cell[ie].f[jf];
                V3 a = sub(F.c, o.cell[ie].c);
                double eface = o.eb(b, d, o.fb[f], ibcell);
                double gn = (eface - e[ie]) * dot(a, F.n) / dot(a, a);
                V3 t = tang(F, f, 0, true);
                w.gf[2 * f + icell] = {gn * F.n.x + t.x, gn * F.n.y + t.y, gn * F.n.z + t.z};
            }
        }
    }
    // _get_non_fourier (:1883-1937)
    auto add_nf = [&](int ie, const Face &F, double area, V3 gg) {
        int m = o.cell[ie].matter;
        if (!(o.hr[m * o.nb + b] > 0)) return;
        V3 vv = o.v(m, b, d);
        double mwt = o.mw[d];
        remacro_acc[ie] -= mwt * area * o.tau[m * o.nb + b] * dot(vv, gg) * dot(vv, F.n);
        remacro_acc[ie] += o.kappa[m] * mwt * area * o.lat[m * o.nb + b] / o.C[m * o.nb + b] * dot(F.n, gg);
    };
    for (int f = 0; f < nf; f++) {
        if (o.fb[f] == -1) {
            int i = o.fcell[f][0], j = o.fface[f][0], i2 = o.fcell[f][1], j2 = o.fface[f][1];
            double area = o.cell[i].f[j].area;
            add_nf(i, o.cell[i].f[j], area, w.gf[2 * f]);
            add_nf(i2, o.cell[i2].f[j2], area, w.gf[2 * f + 1]);
        } else if (o.bnd[o.fb[f]].type != 3) {
            for (int icell = 0; icell < 2; icell++) {
                int ie = o.fcell[f][icell];
                if (ie < 0) continue;
                const Face &F = o.cell[ie].f[o.fface[f][icell]];
                add_nf(ie, F, F.area, w.gf[2 * f + icell]);
            }
        }
    }
}

// _set_bound_ee_1 (StaticBTESynthetic.cpp:2083-2232), sequential in-place
void set_bound_ee_1(Oracle &o) {
    for (int d = 0; d < o.nd; d++)
        for (int b = 0; b < o.nb; b++)
            for (int ib = 0; ib < (int)o.bnd.size(); ib++) {
                const Bnd &B = o.bnd[ib];
                for (int ic = 0; ic < (int)B.cell.size() && ic < 2; ic++) {
                    int ie = B.cell[ic];
                    const Cell &c = o.cell[ie];
                    int m = c.matter;
                    const Face &f = c.f[B.face[ic]];
                    if (o.hr[m * o.nb + b] == 0) continue;
                    double dp = dot(o.v(m, b, d), f.n);
                    if (!(dp < 0)) continue;
                    double e;
                    if (B.type == 1) {
                        e = o.C[m * o.nb + b] * B.T;
                    } else if (B.type == 2) {
                        double s1 = 0, s2 = 0;
                        for (int k = 0; k < o.nd; k++) {
                            double d1 = dot(o.v(m, b, k), f.n);
                            if (d1 >= 0) {
                                s1 += o.eb(b, k, ib, ic) * (d1 * o.mw[k]);
                                s2 += (d1 * o.mw[k]);
                            }
                        }
                        e = s1 / s2;
                    } else if (B.type == 3) {
                        double d1 = dot(o.dir[d], f.n);
                        V3 r = {o.dir[d].x - f.n.x * d1 * 2, o.dir[d].y - f.n.y * d1 * 2, o.dir[d].z - f.n.z * d1 * 2};
                        double close = 1;
                        int nf = -1;
                        for (int k = 0; k < o.nd; k++) {
                            double l = std::sqrt(std::pow(r.x - o.dir[k].x, 2) + std::pow(r.y - o.dir[k].y, 2) +
                                                 std::pow(r.z - o.dir[k].z, 2));
                            if (l < close) {
                                nf = k;
                                close = l;
                            }
                        }
                        e = o.eb(b, nf, ib, ic);
                    } else if (B.type == 6) {
                        // extension: p x (outgoing direction nearest the
                        // mirror image) + (1 - p) x the diffuse value
                        double s1 = 0, s2 = 0;
                        for (int k = 0; k < o.nd; k++) {
                            double d1 = dot(o.v(m, b, k), f.n);
                            if (d1 >= 0) {
                                s1 += o.eb(b, k, ib, ic) * (d1 * o.mw[k]);
                                s2 += (d1 * o.mw[k]);
                            }
                        }
                        double d1 = dot(o.dir[d], f.n);
                        V3 r = {o.dir[d].x - f.n.x * d1 * 2, o.dir[d].y - f.n.y * d1 * 2, o.dir[d].z - f.n.z * d1 * 2};
                        double close = 1e300;
                        int nf = -1;
                        for (int k = 0; k < o.nd; k++) {
                            if (dot(o.dir[k], f.n) < 0) continue;
                            double l = std::pow(r.x - o.dir[k].x, 2) + std::pow(r.y - o.dir[k].y, 2) +
                                       std::pow(r.z - o.dir[k].z, 2);
                            if (l < close) {
                                nf = k;
                                close = l;
                            }
                        }
                        e = B.T * o.eb(b, nf, ib, ic) + (1.0 - B.T) * (s1 / s2);
                    } else if (B.type < 0) {
                        e = o.eb(b, d, B.connect, ic) + o.C[m * o.nb + b] * (B.T - o.bnd[B.connect].T);
                    } else {
                        e = o.eb(b, d, ib, ic);
                    }
                    o.eb(b, d, ib, ic) = e;
                }
            }
}

// _set_macro_boundary_condition (:2234-2274)
void macro_bc(Oracle &o) {
    int nbnd = (int)o.bnd.size();
    o.bTmacro.assign(nbnd, {0.0, 0.0});
    for (int ib = 0; ib < nbnd; ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
            int m = o.cell[o.bnd[ib].cell[ic]].matter;
            double s = 0;
            for (int b = 0; b < o.nb; b++)
                for (int d = 0; d < o.nd; d++)
                    s += o.lat[m * o.nb + b] * o.eb(b, d, ib, ic) / o.C[m * o.nb + b] * o.mw[d];
            o.bTmacro[ib][ic] = s;
        }
    for (int ib = 0; ib < nbnd; ib++)
        for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++)
            if (o.bnd[ib].type < 0 && o.bnd[ib].T > 0) {
                o.bTmacro[ib][ic] = o.bnd[ib].T / 2;
                o.bTmacro[o.bnd[ib].connect][ic] = -o.bnd[ib].T / 2;
            }
}

// _get_coefficient_macro (:842-884)
void macro_matrix(Oracle &o) {
    std::vector<std::vector<std::pair<int, double>>> rows(o.nc);
    for (int ie = 0; ie < o.nc; ie++) {
        const Cell &c = o.cell[ie];
        double diag = 0;
        for (const Face &f : c.f) {
            double temp = o.kappa[c.matter] * f.area;
            if (f.bound == -1) {
                V3 a = sub(o.cell[f.neighbor].c, c.c);
                temp = temp / dot(f.n, a);
                diag += -temp;
                rows[ie].push_back({f.neighbor, temp});
            } else if (o.bnd[f.bound].type != 3) {
                V3 a = sub(f.c, c.c);
                temp = temp / dot(f.n, a);
                diag += -temp;
            }
        }
        rows[ie].push_back({ie, diag});
    }
    o.macroLU.factor(o.nc, rows);
}

// _marco_solution (:2692-2734) with _set_vertex_temperature (:2276-2305)
// and _get_Re_macro (:2307-2407)
void macro_solution(Oracle &o) {
    const int M = o.nmat;
    double internal = 1000;
    std::vector<double> T1(o.nc), rhs(o.nc), sol;
    while (internal > 1e-6) {
        T1 = o.T;
        std::vector<double> tmp(o.nn * M, 0.0), rn(o.nn * M, 0.0), TV(o.nn * M, 0.0);
        for (int i = 0; i < o.nc; i++)
            for (int vtx : o.cell[i].v) {
                double ds = dist(o.node[vtx], o.cell[i].c);
                tmp[vtx * M + o.cell[i].matter] += o.T[i] / ds;
                rn[vtx * M + o.cell[i].matter] += 1.0 / ds;
            }
        for (int i = 0; i < o.nn * M; i++) TV[i] = tmp[i] / rn[i];
        for (int ie = 0; ie < o.nc; ie++) {
            const Cell &c = o.cell[ie];
            double r = o.ReMacro[ie] - c.heat * c.vol;
            for (int j = 0; j < (int)c.f.size(); j++) {
                const Face &f = c.f[j];
                V3 a;
                if (f.bound >= 0) {
                    if (o.bnd[f.bound].type != 3) {
                        const Bnd &B = o.bnd[f.bound];
                        for (int ic = 0; ic < 2; ic++) {
                            int bc_cell = ic < (int)B.cell.size() ? B.cell[ic] : -1;
                            if (bc_cell == ie) {
                                double temp = o.kappa[c.matter] * f.area;
                                a = sub(f.c, c.c);
                                temp = temp / dot(f.n, a);
                                r += -temp * o.bTmacro[f.bound][ic];
                            }
                        }
                    }
                } else {
                    a = sub(o.cell[f.neighbor].c, c.c);
                }
                double an = dot(a, f.n);
                V3 a2 = {f.n.x - a.x / an, f.n.y - a.y / an, f.n.z - a.z / an};
                V3 gT;
                if (o.dim == 2) {
                    int v0 = f.v[0], v1 = f.v[1];
                    double gx = o.node[v1].x - o.node[v0].x, gy = o.node[v1].y - o.node[v0].y;
                    double dT = TV[v1 * M + c.matter] - TV[v0 * M + c.matter];
                    gT = {dT / (gx * gx + gy * gy) * gx, dT / (gx * gx + gy * gy) * gy, 0};
                } else {
                    // 3D: the reference accumulates onto the face-offset vector
                    // (ax += ... at :2368-2370); reproduced as written.
                    int fi = f.index;
                    int i1 = o.fcell[fi][0], j1 = o.fface[fi][0];
                    const Face &F1 = o.cell[i1].f[j1];
                    int nv = (int)F1.v.size();
                    std::vector<double> d1(nv, 0.0);
                    for (int m = 0; m < nv - 1; m++)
                        d1[m + 1] = 1.0 / o.Lx *
                                    (TV[F1.v[m + 1] * M + o.cell[i1].matter] - TV[F1.v[m] * M + o.cell[i1].matter]);
                    gT = a;
                    for (int m = 0; m < nv; m++) {
                        gT.x += o.faceW[fi][0][m] * d1[m];
                        gT.y += o.faceW[fi][1][m] * d1[m];
                        gT.z += o.faceW[fi][2][m] * d1[m];
                    }
                }
                if (f.bound >= 0) {
                    if (o.bnd[f.bound].type != 3) r -= o.kappa[c.matter] * f.area * dot(a2, gT);
                } else
                    r -= o.kappa[c.matter] * f.area * dot(a2, gT);
            }
            rhs[ie] = r;
        }
        o.macroLU.solve(rhs, sol);
        internal = 0;
        for (int i = 0; i < o.nc; i++) {
            o.T[i] = sol[i];
            internal += std::pow(T1[i] - o.T[i], 2);
        }
        internal = internal / o.nc;
        o.inner_last = internal;
    }
}

// _get_magin_check_error (:2565-2611)
bool margins(Oracle &o, double elT, double elq) {
    double Tmax = 0, e1 = 0;
    for (int i = 0; i < o.nc; i++) Tmax = std::max(Tmax, std::fabs(o.T[i]));
    for (int i = 0; i < o.nc; i++) e1 += std::sqrt(std::pow(o.T[i] - o.Told[i], 2));
    o.err = e1 / o.nc / Tmax;
    double hmax = 0, e2 = 0;
    for (int i = 0; i < o.nc; i++) {
        double h = std::sqrt(std::pow(o.qx[i], 2) + std::pow(o.qy[i], 2) + std::pow(o.qz[i], 2));
        double h1 = std::sqrt(std::pow(o.qxo[i], 2) + std::pow(o.qyo[i], 2) + std::pow(o.qzo[i], 2));
        hmax = std::max(hmax, h);
        e2 += std::fabs(h - h1);
    }
    o.errq = e2 / o.nc / hmax;
    if ((o.err > o.errOld && o.errq > o.errOldq) || std::isnan(o.err) || std::isnan(o.errq) || std::isinf(o.err) ||
        std::isinf(o.errq))
        o.errInc++;
    else
        o.errInc = 0;
    o.errOld = o.err;
    o.errOldq = o.errq;
    return o.err <= elT && o.errq <= elq;
}

}  // namespace

extern "C" {

// Runs the full restated solve. Arrays follow the C-ABI mesh view of the
// product (node coordinates already scaled to metres). Angles are generated
// from (angle_method, ntheta, nphi, material_dim) as BTEAngle does. Returns
// 0 on success, <0 on a mesh/topology error.
int oracle_solve(int dim, int nn, const double *xyz, int nc, const int *cptr, const int *cverts, const int *creg,
                 int nbe, const int *bptr, const int *bverts, const int *btag, int nbc, const int *bc_tag,
                 const int *bc_type, const double *bc_val, int nmat, int nband, const double *v, const double *tau,
                 const double *C, const double *lat, const double *hr, const int *reg_mat, int nreg, int material_dim,
                 int angle_method, int ntheta, int nphi, double Lx, const double *cell_heat, const double *T0,
                 const double *q0, int max_iter, double errT, double errq, int use_limiter, double *out_Tlat,
                 double *out_E, double *out_q, double *out_Tband, int *out_iters, double *out_err,
                 const double *cell_scatter, int order, int sequential) {
    Oracle o;
    o.nmat = nmat;
    o.nb = nband;
    o.Lx = Lx;
    o.use_limiter = use_limiter;
    int rc = build_mesh(o, dim, nn, xyz, nc, cptr, cverts, creg, nbe, bptr, bverts, btag, nbc, bc_tag, bc_type, bc_val,
                        reg_mat, nreg);
    if (rc) return rc;
    for (int i = 0; i < nc; i++) o.cell[i].heat = cell_heat ? cell_heat[i] : 0.0;
    o.order = order == 1 ? 1 : 2;
    o.sequential = sequential != 0;
    o.tsc.assign(nc, 1.0);
    if (cell_scatter)
        for (int i = 0; i < nc; i++) o.tsc[i] = 1.0 / cell_scatter[i];
    o.vg.assign(v, v + nmat * nband);
    o.tau.assign(tau, tau + nmat * nband);
    o.C.assign(C, C + nmat * nband);
    o.lat.assign(lat, lat + nmat * nband);
    o.hr.assign(hr, hr + nmat * nband);
    o.kappa.assign(nmat, 0.0);
    o.capb.assign(nmat, 0.0);
    for (int m = 0; m < nmat; m++)
        for (int b = 0; b < nband; b++) {  // BTEBand.cpp:791-803
            double k = C[m * nband + b] * v[m * nband + b] * v[m * nband + b] * tau[m * nband + b];
            o.kappa[m] += (material_dim == 2) ? k / 2 : k / 3;
            o.capb[m] += C[m * nband + b];
        }
    std::vector<double> w;
    double solid = 0;
    make_angles(angle_method, ntheta, nphi, material_dim, o.dir, w, solid);
    o.nd = (int)o.dir.size();
    o.mw.resize(o.nd);
    for (int d = 0; d < o.nd; d++) o.mw[d] = w[d] / solid;

    setup_lsq(o);
    macro_matrix(o);
    const int P = o.P();
    o.T.assign(T0, T0 + nc);
    o.Told = o.T;
    o.qx.assign(nc, 0);
    o.qy.assign(nc, 0);
    o.qz.assign(nc, 0);
    if (q0)
        for (int i = 0; i < nc; i++) {
            o.qx[i] = q0[3 * i];
            o.qy[i] = q0[3 * i + 1];
            o.qz[i] = q0[3 * i + 2];
        }
    o.ebound.assign((size_t)nband * o.nd * o.bnd.size() * 2, 0.0);
    o.e.assign(P, std::vector<double>(nc));
    // _set_initial (:765-782)
    for (int d = 0; d < o.nd; d++)
        for (int b = 0; b < nband; b++)
            for (int i = 0; i < nc; i++) o.e[d * nband + b][i] = o.T[i] * o.C[o.cell[i].matter * nband + b];
    // initial outgoing boundary values (StaticBTESyntheticSolver.cpp:47-61)
    for (int d = 0; d < o.nd; d++)
        for (int b = 0; b < nband; b++) {
            std::vector<V3> g;
            std::vector<double> lim;
            gradient(o, o.e[d * nband + b], b, d, g, lim);
            for (int ib = 0; ib < (int)o.bnd.size(); ib++)
                for (int ic = 0; ic < (int)o.bnd[ib].cell.size() && ic < 2; ic++) {
                    int ie = o.bnd[ib].cell[ic];
                    const Face &f = o.cell[ie].f[o.bnd[ib].face[ic]];
                    if (dot(o.v(o.cell[ie].matter, b, d), f.n) >= 0)
                        o.eb(b, d, ib, ic) = o.e[d * nband + b][ie] + dot(sub(f.c, o.cell[ie].c), g[ie]) * lim[ie];
                }
        }
    set_bound_ee_1(o);

    int nt = 0, iters = 0;
    for (nt = 0; nt < max_iter; ++nt) {
        // copy() (:2655-2690)
        o.Told = o.T;
        o.qxo = o.qx;
        o.qyo = o.qy;
        o.qzo = o.qz;
        std::vector<double> Tacc(nc, 0.0), Eacc(nc, 0.0), qxa(nc, 0.0), qya(nc, 0.0), qza(nc, 0.0),
            Tb(nband * nc, 0.0), RM(nc, 0.0);
        // all (b,d) pairs are independent within an iteration (Jacobi)
        int nthr = std::max(1, std::min<int>(P, (int)std::thread::hardware_concurrency()));
        std::vector<std::vector<double>> RMt(nthr, std::vector<double>(nc, 0.0));
        {
            std::vector<std::thread> pool;
            for (int t = 0; t < nthr; t++)
                pool.emplace_back([&, t]() {
                    PairWork w;
                    for (int p = t; p < P; p += nthr) bte_pair(o, p % nband, p / nband, w, RMt[t]);
                });
            for (auto &th : pool) th.join();
        }
        for (int t = 0; t < nthr; t++)
            for (int i = 0; i < nc; i++) RM[i] += RMt[t][i];
        // moments (:2487-2520), in (d, b) order
        for (int d = 0; d < o.nd; d++)
            for (int b = 0; b < nband; b++) {
                const std::vector<double> &e = o.e[d * nband + b];
                for (int i = 0; i < nc; i++) {
                    int m = o.cell[i].matter;
                    double mwt = o.mw[d];
                    double Cb = o.C[m * nband + b];
                    Tacc[i] += o.lat[m * nband + b] * e[i] * mwt / Cb;
                    Tb[b * nc + i] += e[i] * mwt / Cb;
                    Eacc[i] += e[i] * mwt / o.capb[m];
                    V3 vv = o.v(m, b, d);
                    qxa[i] += vv.x * mwt * e[i];
                    qya[i] += vv.y * mwt * e[i];
                    qza[i] += vv.z * mwt * e[i];
                }
            }
        o.T = Tacc;
        o.Tlat = Tacc;
        o.E = Eacc;
        o.qx = qxa;
        o.qy = qya;
        o.qz = qza;
        o.Tband = Tb;
        o.ReMacro = RM;
        set_bound_ee_1(o);
        if (!o.sequential) {  // solve_DOM (StaticBTESyntheticSolver.cpp:968-1179) keeps T_lat
            macro_bc(o);
            macro_solution(o);
        }
        iters = nt + 1;
        bool stop = margins(o, errT, errq);
        if (stop || o.errInc >= 10) break;
    }
    for (int i = 0; i < nc; i++) {
        out_Tlat[i] = o.T[i];
        out_E[i] = o.E[i];
        out_q[3 * i] = o.qx[i];
        out_q[3 * i + 1] = o.qy[i];
        out_q[3 * i + 2] = o.qz[i];
    }
    if (out_Tband)
        for (int i = 0; i < nband * nc; i++) out_Tband[i] = o.Tband[i];
    if (out_iters) *out_iters = iters;
    if (out_err) {
        out_err[0] = o.err;
        out_err[1] = o.errq;
    }
    return 0;
}

}  // extern "C"
