// Mesh flattening: raw cells/boundary elements + BC table -> FlatMesh.
//
// Topology semantics follow GiftBTE's BTEMesh (src/BTEMesh/BTEMesh.cpp):
//   * 2D cell geometry, face vertex order and outward normals :668-772
//     (triangles: face j = (v[j+1], v[j+2]); COMSOL quads: v0-v1, v1-v3,
//     v3-v2, v2-v0; area by Heron's formula as get_tri_area)
//   * face neighbour = last other cell around the face's first vertex that
//     holds all face vertices :782-806
//   * boundary element -> (cell, face) sides :808-834
//   * boundaries kept in mesh order when their tag is in the BC table;
//     tags that are in no BC row become isothermal at 0 K unless the element
//     has two cells (Distribute.cpp:150-197)
//   * periodic partner = nearest face centre among boundaries whose type
//     names this tag :903-925
//   * global face list in cell/face order :987-1021
// 3D tetrahedra (stripped from the reference's public release) use face j =
// the three vertices other than vertex j, area by Heron, outward normal.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <unordered_map>

#include "gbte_internal.h"

namespace gbte {
namespace {

inline double sq(double x) { return x * x; }
inline double dist3(double ax, double ay, double az, double bx, double by, double bz) {
    return std::sqrt(std::pow(ax - bx, 2) + std::pow(ay - by, 2) + std::pow(az - bz, 2));
}
double heron(const double *a, const double *b, const double *c) {
    double la = dist3(a[0], a[1], a[2], b[0], b[1], b[2]);
    double lb = dist3(b[0], b[1], b[2], c[0], c[1], c[2]);
    double lc = dist3(a[0], a[1], a[2], c[0], c[1], c[2]);
    double p = (la + lb + lc) / 2;
    return std::sqrt(p * (p - la) * (p - lb) * (p - lc));
}

// (J^T J)^-1 J^T for k rows of dimension dim -> out[r*k + j], r < 3
void lsq_pinv(const std::vector<double> &J, int k, int dim, std::vector<double> &out) {
    out.assign(3 * (size_t)k, 0.0);
    double M[3][3] = {{0}}, N[3][3] = {{0}};
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++)
            for (int r = 0; r < k; r++) M[i][j] += J[r * 3 + i] * J[r * 3 + j];
    if (dim == 2) {
        double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        N[0][0] = M[1][1] / det;
        N[0][1] = -M[0][1] / det;
        N[1][1] = M[0][0] / det;
        N[1][0] = -M[1][0] / det;
    } else {
        double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) + M[0][1] * (M[1][2] * M[2][0] - M[1][0] * M[2][2]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        N[0][0] = 1.0 / det * (M[1][1] * M[2][2] - M[1][2] * M[2][1]);
        N[1][0] = 1.0 / det * (M[0][2] * M[2][1] - M[0][1] * M[2][2]);
        N[2][0] = 1.0 / det * (M[0][1] * M[1][2] - M[0][2] * M[1][1]);
        N[0][1] = 1.0 / det * (M[1][2] * M[2][0] - M[1][0] * M[2][2]);
        N[1][1] = 1.0 / det * (M[0][0] * M[2][2] - M[0][2] * M[2][0]);
        N[2][1] = 1.0 / det * (M[1][0] * M[0][2] - M[0][0] * M[1][2]);
        N[0][2] = 1.0 / det * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        N[1][2] = 1.0 / det * (M[0][1] * M[2][0] - M[0][0] * M[2][1]);
        N[2][2] = 1.0 / det * (M[0][0] * M[1][1] - M[1][0] * M[0][1]);
    }
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < k; j++) {
            double s = 0;
            for (int q = 0; q < dim; q++) s += N[i][q] * J[j * 3 + q];
            out[i * (size_t)k + j] = s;
        }
}

// f(lo, hi) over contiguous ranges of [0, n) on up to 64 of the host's
// threads (one range when n is small); f must only write entries owned by
// its range.
template <typename F>
void for_ranges(int n, F &&f, int max_threads = 64) {
    const int hw = std::min(max_threads, (int)std::max(1u, std::thread::hardware_concurrency()));
    const int nth = std::max(1, std::min(hw, n / 4096 + 1));
    if (nth == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; t++)
        pool.emplace_back([&f, n, nth, t]() { f((int)((long long)n * t / nth), (int)((long long)n * (t + 1) / nth)); });
    for (auto &th : pool) th.join();
}

}  // namespace

Error build_flat_mesh(const RawMesh &raw, const BCs &bcs, const Bands &bands, FlatMesh &m) {
    const int dim = raw.dim, nc = raw.nc(), nn = raw.nn(), nbe = raw.nbe();
    if (dim != 2 && dim != 3) return {-1, "dimension must be 2 or 3"};
    if (nc <= 0 || nn <= 0) return {-1, "empty mesh"};
    m = FlatMesh();
    m.dim = dim;
    m.nc = nc;
    m.nn = nn;
    m.nmat = bands.nmat;
    m.Lx = raw.Lx;
    m.node_x.resize(nn);
    m.node_y.resize(nn);
    m.node_z.resize(nn);
    for (int i = 0; i < nn; i++) {
        m.node_x[i] = raw.xyz[3 * i];
        m.node_y[i] = raw.xyz[3 * i + 1];
        m.node_z[i] = dim == 2 ? 0.0 : raw.xyz[3 * i + 2];
    }
    auto P = [&](int v, double *p) {
        p[0] = m.node_x[v];
        p[1] = m.node_y[v];
        p[2] = m.node_z[v];
    };
    m.cptr = raw.cptr;
    m.cverts = raw.cverts;
    if (raw.comp_ptr.empty()) {
        m.comp_ptr = {0, nc};
    } else {
        m.comp_ptr = raw.comp_ptr;
        if (m.comp_ptr.front() != 0 || m.comp_ptr.back() != nc) return {-1, "component ranges must cover the cells"};
        for (size_t k = 0; k + 1 < m.comp_ptr.size(); k++)
            if (m.comp_ptr[k + 1] <= m.comp_ptr[k]) return {-1, "component ranges must be non-empty and increasing"};
    }
    m.matter.resize(nc);
    m.vol.resize(nc);
    m.cx.resize(nc);
    m.cy.resize(nc);
    m.cz.resize(nc);
    m.cf_ptr.assign(nc + 1, 0);
    for (int c = 0; c < nc; c++) {
        int r = raw.creg[c];
        if (r < 0 || r >= (int)bands.region_material.size())
            return {-1, "cell region " + std::to_string(r) + " has no material (GeometryMaterialType)"};
        m.matter[c] = bands.region_material[r];
        int nv = raw.cptr[c + 1] - raw.cptr[c];
        int nfc = (dim == 2) ? nv : 4;
        if (dim == 2 && nv != 3 && nv != 4) return {-1, "2D cells must be triangles or quads"};
        if (dim == 3 && nv != 4) return {-8, "3D cells must be tetrahedra"};
        m.cf_ptr[c + 1] = m.cf_ptr[c] + nfc;
    }
    const int ncf = m.cf_ptr[nc];
    m.cf_area.resize(ncf);
    m.cf_nx.resize(ncf);
    m.cf_ny.resize(ncf);
    m.cf_nz.resize(ncf);
    m.cf_fx.resize(ncf);
    m.cf_fy.resize(ncf);
    m.cf_fz.resize(ncf);
    m.cf_nbr.assign(ncf, -1);
    m.cf_bside.assign(ncf, -1);
    m.cf_bound.assign(ncf, -1);
    m.cf_face.assign(ncf, -1);
    m.cf_v.assign(3 * (size_t)ncf, -1);
    for (int c = 0; c < nc; c++) {
        const int *v = &raw.cverts[raw.cptr[c]];
        int nv = raw.cptr[c + 1] - raw.cptr[c];
        double p[4][3];
        for (int k = 0; k < std::min(nv, 4); k++) P(v[k], p[k]);
        int k0 = m.cf_ptr[c];
        if (dim == 2) {
            if (nv == 3) {
                m.vol[c] = heron(p[0], p[1], p[2]);
                m.cx[c] = ((p[0][0] + p[1][0]) + p[2][0]) / 3;
                m.cy[c] = ((p[0][1] + p[1][1]) + p[2][1]) / 3;
                m.cz[c] = ((p[0][2] + p[1][2]) + p[2][2]) / 3;
                for (int j = 0; j < 3; j++) {
                    m.cf_v[3 * (k0 + j)] = v[(j + 1) % 3];
                    m.cf_v[3 * (k0 + j) + 1] = v[(j + 2) % 3];
                }
            } else {
                m.vol[c] = heron(p[0], p[1], p[2]) + heron(p[1], p[2], p[3]);
                m.cx[c] = ((p[0][0] + p[1][0]) + p[2][0] + p[3][0]) / 4;
                m.cy[c] = ((p[0][1] + p[1][1]) + p[2][1] + p[3][1]) / 4;
                m.cz[c] = ((p[0][2] + p[1][2]) + p[2][2] + p[3][2]) / 4;
                const int qf[4][2] = {{0, 1}, {1, 3}, {3, 2}, {2, 0}};
                for (int j = 0; j < 4; j++) {
                    m.cf_v[3 * (k0 + j)] = v[qf[j][0]];
                    m.cf_v[3 * (k0 + j) + 1] = v[qf[j][1]];
                }
            }
            for (int j = 0; j < nv; j++) {
                int k = k0 + j;
                double a0[3], a1[3];
                P(m.cf_v[3 * k], a0);
                P(m.cf_v[3 * k + 1], a1);
                double area = dist3(a0[0], a0[1], a0[2], a1[0], a1[1], a1[2]);
                m.cf_area[k] = area;
                m.cf_fx[k] = (a0[0] + a1[0]) / 2;
                m.cf_fy[k] = (a0[1] + a1[1]) / 2;
                m.cf_fz[k] = (a0[2] + a1[2]) / 2;
                double ax = (a0[0] - a1[0]) / area, ay = (a0[1] - a1[1]) / area;
                double nx = ay, ny = -ax;
                double dx = m.cx[c] - m.cf_fx[k], dy = m.cy[c] - m.cf_fy[k], dz = m.cz[c] - m.cf_fz[k];
                if (dx * nx + dy * ny + dz * 0.0 > 0) {
                    nx = -nx;
                    ny = -ny;
                }
                m.cf_nx[k] = nx;
                m.cf_ny[k] = ny;
                m.cf_nz[k] = 0;
            }
        } else {
            double a[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
            double b[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
            double d[3] = {p[3][0] - p[0][0], p[3][1] - p[0][1], p[3][2] - p[0][2]};
            double det = a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0]) + a[2] * (b[0] * d[1] - b[1] * d[0]);
            m.vol[c] = std::fabs(det) / 6.0;
            m.cx[c] = (p[0][0] + p[1][0] + p[2][0] + p[3][0]) / 4;
            m.cy[c] = (p[0][1] + p[1][1] + p[2][1] + p[3][1]) / 4;
            m.cz[c] = (p[0][2] + p[1][2] + p[2][2] + p[3][2]) / 4;
            for (int j = 0; j < 4; j++) {
                int k = k0 + j;
                int fv[3] = {v[(j + 1) % 4], v[(j + 2) % 4], v[(j + 3) % 4]};
                double q[3][3];
                for (int t = 0; t < 3; t++) {
                    m.cf_v[3 * k + t] = fv[t];
                    P(fv[t], q[t]);
                }
                m.cf_area[k] = heron(q[0], q[1], q[2]);
                m.cf_fx[k] = (q[0][0] + q[1][0] + q[2][0]) / 3;
                m.cf_fy[k] = (q[0][1] + q[1][1] + q[2][1]) / 3;
                m.cf_fz[k] = (q[0][2] + q[1][2] + q[2][2]) / 3;
                double u[3] = {q[1][0] - q[0][0], q[1][1] - q[0][1], q[1][2] - q[0][2]};
                double w[3] = {q[2][0] - q[0][0], q[2][1] - q[0][1], q[2][2] - q[0][2]};
                double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
                double l = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
                double nx = cr[0] / l, ny = cr[1] / l, nz = cr[2] / l;
                if ((m.cx[c] - m.cf_fx[k]) * nx + (m.cy[c] - m.cf_fy[k]) * ny + (m.cz[c] - m.cf_fz[k]) * nz > 0) {
                    nx = -nx;
                    ny = -ny;
                    nz = -nz;
                }
                m.cf_nx[k] = nx;
                m.cf_ny[k] = ny;
                m.cf_nz[k] = nz;
            }
        }
    }
    // node -> cells (in cell order)
    std::vector<int> nc_ptr(nn + 1, 0), nc_idx;
    for (int c = 0; c < nc; c++)
        for (int q = raw.cptr[c]; q < raw.cptr[c + 1]; q++) {
            int vtx = raw.cverts[q];
            if (vtx < 0 || vtx >= nn) return {-1, "cell vertex index out of range"};
            nc_ptr[vtx + 1]++;
        }
    for (int i = 0; i < nn; i++) nc_ptr[i + 1] += nc_ptr[i];
    nc_idx.resize(nc_ptr[nn]);
    {
        std::vector<int> fill(nc_ptr.begin(), nc_ptr.end() - 1);
        for (int c = 0; c < nc; c++)
            for (int q = raw.cptr[c]; q < raw.cptr[c + 1]; q++) nc_idx[fill[raw.cverts[q]]++] = c;
    }
    auto cell_has = [&](int c, int vtx) {
        for (int q = raw.cptr[c]; q < raw.cptr[c + 1]; q++)
            if (raw.cverts[q] == vtx) return true;
        return false;
    };
    const int fnv = (dim == 2) ? 2 : 3;
    // face neighbours (each cell writes its own faces' entries)
    for_ranges(nc, [&](int lo, int hi) {
        for (int c = lo; c < hi; c++)
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++) {
                int v0 = m.cf_v[3 * k];
                for (int q = nc_ptr[v0]; q < nc_ptr[v0 + 1]; q++) {
                    int o = nc_idx[q];
                    if (o == c) continue;
                    bool all = true;
                    for (int t = 0; t < fnv; t++) all = all && cell_has(o, m.cf_v[3 * k + t]);
                    if (all) m.cf_nbr[k] = o;
                }
            }
    });
    // boundary elements -> sides
    std::vector<std::vector<std::pair<int, int>>> bsides(nbe);
    for (int i = 0; i < nbe; i++) {
        int nv = raw.bptr[i + 1] - raw.bptr[i];
        if (nv != fnv) return {-1, "boundary element vertex count does not match the dimension"};
        const int *bv = &raw.bverts[raw.bptr[i]];
        for (int t = 0; t < nv; t++)
            if (bv[t] < 0 || bv[t] >= nn) return {-1, "boundary vertex index out of range"};
        for (int q = nc_ptr[bv[0]]; q < nc_ptr[bv[0] + 1]; q++) {
            int c = nc_idx[q];
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++) {
                bool all = true;
                for (int t = 0; t < nv; t++) {
                    bool in = false;
                    for (int u = 0; u < fnv; u++) in = in || m.cf_v[3 * k + u] == bv[t];
                    all = all && in;
                }
                if (all) bsides[i].push_back({c, k - m.cf_ptr[c]});
            }
        }
    }
    // BC rows + undefined tags
    std::vector<int> tags = bcs.tag, types = bcs.type;
    std::vector<double> vals = bcs.value;
    std::vector<int> nodefine;
    for (int i = 0; i < nbe; i++) {
        int t = raw.btag[i];
        bool set = std::find(tags.begin(), tags.end(), t) != tags.end() || bsides[i].size() == 2;
        if (!set && std::find(nodefine.begin(), nodefine.end(), t) == nodefine.end()) nodefine.push_back(t);
    }
    for (int t : nodefine) {
        tags.push_back(t);
        types.push_back(1);
        vals.push_back(0.0);
    }
    std::vector<int> b_row;
    std::vector<std::vector<std::pair<int, int>>> b_sides;
    for (int i = 0; i < nbe; i++)
        for (int j = 0; j < (int)tags.size(); j++)
            if (raw.btag[i] == tags[j]) {
                if (bsides[i].size() > 2) return {-7, "boundary element shared by more than two cells"};
                b_row.push_back(j);
                b_sides.push_back(bsides[i]);
            }
    const int nbd = (int)b_row.size();
    m.b_type.resize(nbd);
    m.b_T.resize(nbd);
    m.b_tag.resize(nbd);
    m.b_connect.assign(nbd, -1);
    m.bs_cell.assign(2 * nbd, -1);
    m.bs_cf.assign(2 * nbd, -1);
    for (int ib = 0; ib < nbd; ib++) {
        m.b_type[ib] = types[b_row[ib]];
        m.b_T[ib] = vals[b_row[ib]];
        if (m.b_type[ib] == 6) {
            // partially specular wall, value = specularity p: the ends of the
            // range are the diffuse (2) and specular (3) walls themselves
            if (!(m.b_T[ib] >= 0 && m.b_T[ib] <= 1))
                return {-1, "partially specular wall (type 6): the specularity must lie in [0, 1]"};
            if (m.b_T[ib] == 0) m.b_type[ib] = 2;
            else if (m.b_T[ib] == 1) m.b_type[ib] = 3;
        }
        m.b_tag[ib] = tags[b_row[ib]];
        for (int ic = 0; ic < (int)b_sides[ib].size(); ic++) {
            int c = b_sides[ib][ic].first, k = m.cf_ptr[c] + b_sides[ib][ic].second;
            m.bs_cell[2 * ib + ic] = c;
            m.bs_cf[2 * ib + ic] = k;
            m.cf_bound[k] = ib;
            m.cf_bside[k] = 2 * ib + ic;
        }
    }
    for (int k = 0; k < ncf; k++)
        if (m.cf_bound[k] < 0 && m.cf_nbr[k] < 0) return {-7, "a face is neither an interior face nor on a boundary in the BC table"};
    // interface walls (type 5): each side's transmissivity is the table row
    // of its cell's material (BTEMesh.cpp:495-510)
    for (int ib = 0; ib < nbd; ib++) {
        if (m.b_type[ib] != 5) continue;
        if (m.bs_cell[2 * ib] < 0 || m.bs_cell[2 * ib + 1] < 0)
            return {-7, "an interface wall (type 5) needs a cell on each side"};
        if (bcs.trans.empty()) return {-1, "an interface wall (type 5) needs the transmissivity table"};
        if (m.bs_trans.empty()) m.bs_trans.assign((size_t)2 * nbd * bands.nb, 0.0);
        for (int ic = 0; ic < 2; ic++) {
            const int mt = m.matter[m.bs_cell[2 * ib + ic]];
            const double *row = &bcs.trans[((size_t)b_row[ib] * bands.nmat + mt) * bands.nb];
            std::copy(row, row + bands.nb, m.bs_trans.begin() + (size_t)(2 * ib + ic) * bands.nb);
        }
    }
    for (int k = 0; k < ncf; k++)
        if (m.cf_bound[k] >= 0) m.cf_nbr[k] = m.cf_nbr[k];  // boundary faces keep their neighbour for the face list
    // periodic partners: candidates are the boundaries whose type names this
    // tag, in boundary order (the first nearest one wins)
    std::unordered_map<int, std::vector<int>> naming;
    for (int j = 0; j < nbd; j++)
        if (types[b_row[j]] < 0) naming[-types[b_row[j]]].push_back(j);
    for (int ib = 0; ib < nbd; ib++) {
        if (types[b_row[ib]] >= 0) continue;
        double best = 1000;
        int k0 = m.bs_cf[2 * ib];
        if (k0 < 0) return {-7, "periodic boundary without a cell"};
        auto cand = naming.find(tags[b_row[ib]]);
        if (cand == naming.end()) return {-7, "periodic boundary tag " + std::to_string(tags[b_row[ib]]) + " has no partner"};
        for (int j : cand->second) {
            int k1 = m.bs_cf[2 * j];
            if (k1 < 0) continue;
            double d1 = dist3(m.cf_fx[k0], m.cf_fy[k0], m.cf_fz[k0], m.cf_fx[k1], m.cf_fy[k1], m.cf_fz[k1]);
            if (d1 < best) {
                best = d1;
                m.b_connect[ib] = j;
            }
        }
        if (m.b_connect[ib] < 0) return {-7, "periodic boundary tag " + std::to_string(tags[b_row[ib]]) + " has no partner"};
    }
    // global face list
    {
        std::vector<char> done(ncf, 0);
        for (int c = 0; c < nc; c++)
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++) {
                if (done[k]) continue;
                int f = (int)m.f_cell0.size();
                m.cf_face[k] = f;
                done[k] = 1;
                int c1 = -1, k1 = -1;
                if (m.cf_bound[k] == -1) {
                    int o = m.cf_nbr[k];
                    c1 = o;
                    for (int q = m.cf_ptr[o]; q < m.cf_ptr[o + 1]; q++)
                        if (m.cf_nbr[q] == c && m.cf_bound[q] == -1) {
                            k1 = q;
                            done[q] = 1;
                            m.cf_face[q] = f;
                        }
                }
                m.f_cell0.push_back(c);
                m.f_cf0.push_back(k);
                m.f_cell1.push_back(c1);
                m.f_cf1.push_back(k1);
                m.f_bound.push_back(m.cf_bound[k]);
            }
    }
    // vertex-neighbour LSQ stencil: every cell around each of the cell's
    // vertices, in vertex order then node-to-cell order, once each, same
    // material only. Two passes over ranges of cells (count, then fill and
    // weigh), each thread with its own mark array.
    m.nbr_ptr.assign(nc + 1, 0);
    {
        auto stencil = [&](int c, std::vector<int> &mark, int *out) {
            int k = 0;
            for (int q = raw.cptr[c]; q < raw.cptr[c + 1]; q++) {
                int vtx = raw.cverts[q];
                for (int t = nc_ptr[vtx]; t < nc_ptr[vtx + 1]; t++) {
                    int o = nc_idx[t];
                    if (o != c && mark[o] != c && m.matter[o] == m.matter[c]) {
                        mark[o] = c;
                        if (out) out[k] = o;
                        k++;
                    }
                }
            }
            return k;
        };
        for_ranges(nc, [&](int lo, int hi) {
            std::vector<int> mark(nc, -1);
            for (int c = lo; c < hi; c++) m.nbr_ptr[c + 1] = stencil(c, mark, nullptr);
        });
        for (int c = 0; c < nc; c++) m.nbr_ptr[c + 1] += m.nbr_ptr[c];
        m.nbr_idx.resize(m.nbr_ptr[nc]);
        m.lsq_w.assign(3 * (size_t)m.nbr_ptr[nc], 0.0);
        for_ranges(nc, [&](int lo, int hi) {
            std::vector<int> mark(nc, -1);
            std::vector<double> J, W;
            for (int c = lo; c < hi; c++) {
                int *lst = m.nbr_idx.data() + m.nbr_ptr[c];
                const int k = stencil(c, mark, lst);
                if (k < 3) continue;  // zero gradient (StaticBTESynthetic.cpp:1290)
                J.assign(3 * (size_t)k, 0.0);
                for (int j = 0; j < k; j++) {
                    int o = lst[j];
                    J[3 * j] = 1.0 / m.Lx * (m.cx[o] - m.cx[c]);
                    J[3 * j + 1] = 1.0 / m.Lx * (m.cy[o] - m.cy[c]);
                    J[3 * j + 2] = dim == 3 ? 1.0 / m.Lx * (m.cz[o] - m.cz[c]) : 0.0;
                }
                lsq_pinv(J, k, dim, W);
                bool bad = false;
                for (double x : W) bad = bad || !std::isfinite(x);
                if (bad) continue;  // singular stencil: the reference's NaN check zeroes the gradient
                for (int j = 0; j < k; j++)
                    for (int r = 0; r < dim; r++)
                        m.lsq_w[3 * (size_t)(m.nbr_ptr[c] + j) + r] = W[r * (size_t)k + j] / m.Lx;
            }
        });
    }
    // 3D face tangential LSQ
    if (dim == 3) {
        const int nf = m.nf();
        m.face_w.assign(9 * (size_t)nf, 0.0);
        std::vector<double> J(9), W;
        for (int f = 0; f < nf; f++) {
            int k = m.f_cf0[f];
            J[0] = m.cf_nx[k];
            J[1] = m.cf_ny[k];
            J[2] = m.cf_nz[k];
            for (int t = 0; t < 2; t++) {
                int a = m.cf_v[3 * k + t + 1], b = m.cf_v[3 * k + t];
                J[3 * (t + 1)] = 1.0 / m.Lx * (m.node_x[a] - m.node_x[b]);
                J[3 * (t + 1) + 1] = 1.0 / m.Lx * (m.node_y[a] - m.node_y[b]);
                J[3 * (t + 1) + 2] = 1.0 / m.Lx * (m.node_z[a] - m.node_z[b]);
            }
            lsq_pinv(J, 3, 3, W);
            for (int i = 0; i < 9; i++) m.face_w[9 * (size_t)f + i] = W[i];
        }
    }
    // node-slot interpolation weights
    const int M = m.nmat, nslot = nn * M;
    {
        std::vector<std::vector<std::pair<int, double>>> ev(nslot), tv(nslot);
        for (int c = 0; c < nc; c++)
            for (int q = raw.cptr[c]; q < raw.cptr[c + 1]; q++) {
                int vtx = raw.cverts[q];
                double ds = dist3(m.node_x[vtx], m.node_y[vtx], m.node_z[vtx], m.cx[c], m.cy[c], m.cz[c]);
                ev[vtx * M + m.matter[c]].push_back({c, 1.0 / ds});
                tv[vtx * M + m.matter[c]].push_back({c, 1.0 / ds});
            }
        for (int s = 0; s < 2 * nbd; s++) {
            int c = m.bs_cell[s];
            if (c < 0) continue;
            int k = m.bs_cf[s];
            for (int t = 0; t < fnv; t++) ev[m.cf_v[3 * k + t] * M + m.matter[c]].clear();
        }
        for (int s = 0; s < 2 * nbd; s++) {
            int c = m.bs_cell[s];
            if (c < 0) continue;
            int k = m.bs_cf[s];
            for (int t = 0; t < fnv; t++) {
                int vtx = m.cf_v[3 * k + t];
                double ds = dist3(m.node_x[vtx], m.node_y[vtx], m.node_z[vtx], m.cf_fx[k], m.cf_fy[k], m.cf_fz[k]);
                ev[vtx * M + m.matter[c]].push_back({-1 - s, 1.0 / ds});
            }
        }
        auto pack = [&](std::vector<std::vector<std::pair<int, double>>> &lst, std::vector<int> &ptr, std::vector<int> &src,
                        std::vector<double> &w) {
            ptr.assign(nslot + 1, 0);
            for (int i = 0; i < nslot; i++) ptr[i + 1] = ptr[i] + (int)lst[i].size();
            src.resize(ptr[nslot]);
            w.resize(ptr[nslot]);
            for (int i = 0; i < nslot; i++) {
                double tot = 0;
                for (auto &e : lst[i]) tot += e.second;
                for (size_t j = 0; j < lst[i].size(); j++) {
                    src[ptr[i] + j] = lst[i][j].first;
                    w[ptr[i] + j] = lst[i][j].second / tot;
                }
            }
        };
        pack(ev, m.nv_ptr, m.nv_src, m.nv_w);
        pack(tv, m.nt_ptr, m.nt_src, m.nt_w);
    }
    return {0, ""};
}

// Upwind level schedule per direction (Kahn's algorithm). Cell c depends on
// interior neighbour o across face k when s_d . n_k < 0. Faces that close a
// cycle (possible on distorted 3D tetrahedra) are lagged: the sweep treats
// the neighbour's correction as zero, which changes only the convergence
// rate of the defect correction, not its fixed point.
void build_schedule(const FlatMesh &m, const Angles &a, Schedule &s, int nthreads) {
    const int nc = m.nc, nd = a.nd, ncomp = std::max(1, m.ncomp());
    s.ncomp = ncomp;
    s.lvl_cells.assign((size_t)nd * nc, 0);
    std::vector<std::vector<int>> dir_ptr((size_t)nd * ncomp);
    std::vector<std::vector<uint8_t>> dir_lag(nd);
    std::vector<int> dir_lagged(nd, 0);
    auto work = [&](int d) {
        std::vector<int> indeg(nc, 0), level(nc, 0);
        std::vector<uint8_t> lag(nc, 0);
        std::vector<int> out_ptr(nc + 1, 0), out_idx;
        for (int c = 0; c < nc; c++)
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++) {
                if (m.cf_bound[k] != -1) continue;
                double dp = a.sx[d] * m.cf_nx[k] + a.sy[d] * m.cf_ny[k] + a.sz[d] * m.cf_nz[k];
                if (dp < 0) {
                    indeg[c]++;
                    out_ptr[m.cf_nbr[k] + 1]++;
                }
            }
        for (int c = 0; c < nc; c++) out_ptr[c + 1] += out_ptr[c];
        out_idx.resize(out_ptr[nc]);
        {
            std::vector<int> fill(out_ptr.begin(), out_ptr.end() - 1);
            for (int c = 0; c < nc; c++)
                for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++) {
                    if (m.cf_bound[k] != -1) continue;
                    double dp = a.sx[d] * m.cf_nx[k] + a.sy[d] * m.cf_ny[k] + a.sz[d] * m.cf_nz[k];
                    if (dp < 0) out_idx[fill[m.cf_nbr[k]]++] = c;
                }
        }
        std::vector<int> order;
        order.reserve(nc);
        std::vector<char> done(nc, 0);
        std::vector<int> frontier;
        for (int c = 0; c < nc; c++)
            if (indeg[c] == 0) frontier.push_back(c);
        int next_seed = 0, lagged = 0;
        while ((int)order.size() < nc) {
            if (frontier.empty()) {
                // cycle: lag every not-yet-swept upwind face of the lowest pending cell
                while (done[next_seed] || indeg[next_seed] == 0) next_seed++;
                int c = next_seed;
                int j = 0, lvl = 0;
                for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++, j++) {
                    if (m.cf_bound[k] != -1) continue;
                    double dp = a.sx[d] * m.cf_nx[k] + a.sy[d] * m.cf_ny[k] + a.sz[d] * m.cf_nz[k];
                    if (!(dp < 0)) continue;
                    if (done[m.cf_nbr[k]])
                        lvl = std::max(lvl, level[m.cf_nbr[k]] + 1);
                    else {
                        lag[c] |= (uint8_t)(1u << j);
                        lagged++;
                        indeg[c]--;
                    }
                }
                level[c] = lvl;
                frontier.push_back(c);
                continue;
            }
            std::vector<int> nxt;
            for (int c : frontier) {
                done[c] = 1;
                order.push_back(c);
                for (int q = out_ptr[c]; q < out_ptr[c + 1]; q++) {
                    int o = out_idx[q];
                    if (done[o]) continue;
                    level[o] = std::max(level[o], level[c] + 1);
                    if (--indeg[o] == 0) nxt.push_back(o);
                }
            }
            frontier.swap(nxt);
        }
        // group by component, then by level (stable within a level): the
        // cells of component k take positions comp_ptr[k] .. comp_ptr[k+1]
        int *dst = &s.lvl_cells[(size_t)d * nc];
        std::vector<int> comp_of(nc);
        for (int k = 0; k < ncomp; k++)
            for (int c = m.comp_ptr[k]; c < m.comp_ptr[k + 1]; c++) comp_of[c] = k;
        std::vector<std::vector<int>> fills(ncomp);
        for (int k = 0; k < ncomp; k++) {
            int nl = 0;
            for (int c = m.comp_ptr[k]; c < m.comp_ptr[k + 1]; c++) nl = std::max(nl, level[c] + 1);
            std::vector<int> cnt(nl + 1, 0);
            for (int c = m.comp_ptr[k]; c < m.comp_ptr[k + 1]; c++) cnt[level[c] + 1]++;
            cnt[0] = m.comp_ptr[k];
            for (int l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
            fills[k].assign(cnt.begin(), cnt.end() - 1);
            dir_ptr[(size_t)d * ncomp + k] = cnt;
        }
        for (int c : order) dst[fills[comp_of[c]][level[c]]++] = c;
        dir_lag[d] = lag;
        dir_lagged[d] = lagged;
    };
    nthreads = std::max(1, std::min(nthreads, nd));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
        pool.emplace_back([&, t]() {
            for (int d = t; d < nd; d += nthreads) work(d);
        });
    for (auto &th : pool) th.join();
    s.dir_lvl_off.assign((size_t)nd * ncomp + 1, 0);
    s.lvl_ptr.clear();
    s.max_levels = 0;
    s.lagged_faces = 0;
    for (size_t e = 0; e < (size_t)nd * ncomp; e++) {
        s.dir_lvl_off[e] = (int)s.lvl_ptr.size();
        s.lvl_ptr.insert(s.lvl_ptr.end(), dir_ptr[e].begin(), dir_ptr[e].end());
        s.max_levels = std::max(s.max_levels, (int)dir_ptr[e].size() - 1);
    }
    for (int d = 0; d < nd; d++) s.lagged_faces += dir_lagged[d];
    s.dir_lvl_off[(size_t)nd * ncomp] = (int)s.lvl_ptr.size();
    if (s.lagged_faces > 0) {
        s.lag.assign((size_t)nd * nc, 0);
        for (int d = 0; d < nd; d++) std::copy(dir_lag[d].begin(), dir_lag[d].end(), s.lag.begin() + (size_t)d * nc);
    } else
        s.lag.clear();
}

Error build_sweep_plan(const FlatMesh &m, const Angles &a, const Schedule &s, int min_ring, int far_cap,
                       SweepPlan &out) {
    const int nc = m.nc, nd = a.nd, ncomp = s.ncomp;
    out = SweepPlan{};
    for (size_t e = 0; e < (size_t)nd * ncomp; e++)
        for (int k = s.dir_lvl_off[e]; k + 1 < s.dir_lvl_off[e + 1]; k++)
            out.max_width = std::max(out.max_width, s.lvl_ptr[k + 1] - s.lvl_ptr[k]);
    int ring = 1;
    while (ring < std::max(min_ring, out.max_width)) ring *= 2;
    out.ring = ring;
    const size_t N = (size_t)nd * nc;
    // left uninitialised here: work(d) writes every entry of direction d's
    // ranges (and clears np and a past each position's neighbours first)
    out.np.resize(4 * N);
    out.a.resize(4 * N);
    out.sig.resize(N);
    out.nin.resize(N);
    out.cell.resize(N);
    out.far_w.resize(N);
    HostArray<int> np_far(4 * N);  // np with far references encoded as slots
    std::vector<int> dir_slots(nd, 0);
    std::vector<long long> dir_refs(nd, 0);
    std::vector<std::string> dir_err(nd);
    auto work = [&](int d) {
        const int *lc = &s.lvl_cells[(size_t)d * nc];
        // level (within its component) and level end of every position
        std::vector<int> po(nc), lev(nc), lend(nc), last_read(nc, -1);
        for (int k = 0; k < ncomp; k++) {
            const size_t e = (size_t)d * ncomp + k;
            const int *lp = &s.lvl_ptr[s.dir_lvl_off[e]];
            const int nl = s.dir_lvl_off[e + 1] - s.dir_lvl_off[e] - 1;
            for (int l = 0; l < nl; l++)
                for (int pos = lp[l]; pos < lp[l + 1]; pos++) {
                    po[lc[pos]] = pos;
                    lev[pos] = l;
                    lend[pos] = lp[l + 1];
                }
        }
        const size_t P0 = (size_t)d * nc;
        std::fill(out.np.begin() + 4 * P0, out.np.begin() + 4 * (P0 + nc), 0);
        std::fill(out.a.begin() + 4 * P0, out.a.begin() + 4 * (P0 + nc), 0.0);
        for (int pos = 0; pos < nc; pos++) {
            const size_t P = P0 + pos;
            const int c = lc[pos];
            out.cell[P] = c;
            const unsigned lm = s.lag.empty() ? 0u : s.lag[P0 + c];
            double sig = 0;
            int j = 0, nin = 0;
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++, j++) {
                const double dpn = a.sx[d] * m.cf_nx[k] + a.sy[d] * m.cf_ny[k] + a.sz[d] * m.cf_nz[k];
                const double av = m.cf_area[k] / m.vol[c] * dpn;
                if (dpn >= 0)
                    sig += av;
                else if (m.cf_bound[k] < 0 && !((lm >> j) & 1u)) {
                    if (nin >= 4) {
                        dir_err[d] = "a cell has more than four upwind neighbours";
                        return;
                    }
                    const int q = po[m.cf_nbr[k]];
                    out.np[4 * P + nin] = q;
                    out.a[4 * P + nin] = av;
                    if (q < lend[pos] - ring) {
                        last_read[q] = std::max(last_read[q], lev[pos]);
                        dir_refs[d]++;
                    }
                    nin++;
                }
            }
            out.sig[P] = sig;
            out.nin[P] = nin;
        }
        // far slots, per component (one sweep CTA walks one component): a
        // slot is taken at its writer's level and free again from the level
        // after its last reader's
        std::vector<int> slot(nc, -1);
        int maxslots = 0;
        for (int k = 0; k < ncomp; k++) {
            const size_t e = (size_t)d * ncomp + k;
            const int *lp = &s.lvl_ptr[s.dir_lvl_off[e]];
            const int nl = s.dir_lvl_off[e + 1] - s.dir_lvl_off[e] - 1;
            std::vector<int> freel;
            std::vector<std::vector<int>> release(nl + 1);
            int nslots = 0;
            for (int l = 0; l < nl; l++) {
                for (int sl : release[l]) freel.push_back(sl);
                for (int pos = lp[l]; pos < lp[l + 1]; pos++) {
                    if (last_read[pos] < 0) continue;
                    int sl;
                    if (!freel.empty()) {
                        sl = freel.back();
                        freel.pop_back();
                    } else {
                        sl = nslots++;
                    }
                    slot[pos] = sl;
                    release[last_read[pos] + 1].push_back(sl);
                }
            }
            maxslots = std::max(maxslots, nslots);
        }
        dir_slots[d] = maxslots;
        for (int pos = 0; pos < nc; pos++) {
            const size_t P = P0 + pos;
            for (int jj = 0; jj < 4; jj++) {
                const int q = out.np[4 * P + jj];
                np_far[4 * P + jj] = (jj < out.nin[P] && q < lend[pos] - ring) ? -(1 + slot[q]) : q;
            }
        }
        for (int pos = 0; pos < nc; pos++) out.far_w[P0 + pos] = slot[pos];
    };
    const int nthreads = std::max(1, std::min((int)std::max(1u, std::thread::hardware_concurrency()), nd));
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++)
        pool.emplace_back([&, t]() {
            for (int d = t; d < nd; d += nthreads) work(d);
        });
    for (auto &th : pool) th.join();
    for (int d = 0; d < nd; d++)
        if (!dir_err[d].empty()) return {-8, dir_err[d]};
    for (int d = 0; d < nd; d++) {
        out.far_slots = std::max(out.far_slots, dir_slots[d]);
        out.far_refs += dir_refs[d];
    }
    out.far_enabled = far_cap > 0 && out.far_slots <= far_cap;
    if (out.far_enabled)
        out.np.swap(np_far);
    else
        std::fill(out.far_w.begin(), out.far_w.end(), -1);
    return {0, ""};
}

void locality_order(const RawMesh &raw, std::vector<int> &perm) {
    const int nc = raw.nc();
    std::vector<double> c(3 * (size_t)nc, 0.0);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < nc; i++) {
        const int n = raw.cptr[i + 1] - raw.cptr[i];
        for (int k = raw.cptr[i]; k < raw.cptr[i + 1]; k++)
            for (int a = 0; a < 3; a++) c[3 * (size_t)i + a] += raw.xyz[3 * (size_t)raw.cverts[k] + a] / n;
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], c[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], c[3 * (size_t)i + a]);
        }
    }
    // Morton code of the centre quantised to 21 bits per axis
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<uint64_t> key(nc);
    for (int i = 0; i < nc; i++) {
        uint64_t q[3];
        for (int a = 0; a < 3; a++) {
            const double span = hi[a] - lo[a];
            const double t = span > 0 ? (c[3 * (size_t)i + a] - lo[a]) / span : 0.0;
            q[a] = (uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
        }
        key[i] = spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2;
    }
    perm.resize(nc);
    const std::vector<int> cp = raw.comp_ptr.empty() ? std::vector<int>{0, nc} : raw.comp_ptr;
    for (size_t k = 0; k + 1 < cp.size(); k++) {
        for (int i = cp[k]; i < cp[k + 1]; i++) perm[i] = i;
        std::stable_sort(perm.begin() + cp[k], perm.begin() + cp[k + 1],
                         [&](int a, int b) { return key[a] < key[b]; });
    }
}

void scatter_rows(const std::vector<int> &perm, double *const *cols, int ncols, int w) {
    const size_t nc = perm.size();
    if (nc == 0 || ncols <= 0 || w <= 0) return;
    const size_t len = nc * (size_t)w;
    auto one = [&](double *a, std::vector<double> &tmp, size_t k0, size_t k1) {
        for (size_t k = k0; k < k1; k++)
            for (int j = 0; j < w; j++) a[(size_t)perm[k] * w + j] = tmp[k * w + j];
    };
    const int hw = std::min(64, (int)std::max(1u, std::thread::hardware_concurrency()));
    if (ncols >= 4 && hw > 1 && nc >= 4096) {
        // whole columns per thread, each thread with its own copy buffer
        // (at most 16: the scatter is bound by memory, not by threads)
        const int nth = std::min(std::min(hw, 16), ncols);
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; t++)
            pool.emplace_back([&, t]() {
                std::vector<double> tmp(len);
                for (int c = t; c < ncols; c += nth) {
                    std::copy(cols[c], cols[c] + len, tmp.begin());
                    one(cols[c], tmp, 0, nc);
                }
            });
        for (auto &th : pool) th.join();
        return;
    }
    // few columns: ranges of rows per thread (perm is a permutation, so the
    // ranges write disjoint rows)
    std::vector<double> tmp(len);
    for (int c = 0; c < ncols; c++) {
        double *a = cols[c];
        for_ranges((int)nc, [&](int lo, int hi) {
            std::copy(a + (size_t)lo * w, a + (size_t)hi * w, tmp.begin() + (size_t)lo * w);
        });
        for_ranges((int)nc, [&](int lo, int hi) { one(a, tmp, lo, hi); });
    }
}

void reorder_cells(RawMesh &raw, const std::vector<int> &perm) {
    const int nc = raw.nc();
    std::vector<int> cptr(1, 0), cverts, creg(nc);
    cverts.reserve(raw.cverts.size());
    for (int k = 0; k < nc; k++) {
        const int c = perm[k];
        for (int j = raw.cptr[c]; j < raw.cptr[c + 1]; j++) cverts.push_back(raw.cverts[j]);
        cptr.push_back((int)cverts.size());
        creg[k] = raw.creg[c];
    }
    raw.cptr.swap(cptr);
    raw.cverts.swap(cverts);
    raw.creg.swap(creg);
}

Error make_union(const std::vector<RawMesh> &meshes, const std::vector<BCs> &bcs, RawMesh &out, BCs &out_bcs) {
    const int n = (int)meshes.size();
    if (n <= 0 || (int)bcs.size() != n) return {-1, "a batch needs at least one geometry and one BC table each"};
    for (int k = 0; k < n; k++)
        if (!bcs[k].trans.empty()) return {-8, "interface walls (type 5) are not supported in a batched solve"};
    int span = 1;  // tags of geometry k are shifted by k * span
    for (int k = 0; k < n; k++) {
        for (int t : meshes[k].btag) span = std::max(span, t + 1);
        for (int t : bcs[k].tag) span = std::max(span, t + 1);
        for (int t : bcs[k].type)
            if (t < 0) span = std::max(span, -t + 1);
    }
    out = RawMesh();
    out_bcs = BCs();
    out.dim = meshes[0].dim;
    out.Lx = meshes[0].Lx;
    out.Ly = meshes[0].Ly;
    out.Lz = meshes[0].Lz;
    out.cptr.assign(1, 0);
    out.bptr.assign(1, 0);
    out.comp_ptr.assign(1, 0);
    int node0 = 0;
    for (int k = 0; k < n; k++) {
        const RawMesh &m = meshes[k];
        if (m.dim != out.dim) return {-1, "the geometries of a batch must have one dimension"};
        if (m.Lx != out.Lx) return {-1, "the geometries of a batch must share ScaleX (it scales the LSQ stencils)"};
        if ((long long)out.nc() + m.nc() > 0x7fffffff / 2) return {-1, "batch too large"};
        out.xyz.insert(out.xyz.end(), m.xyz.begin(), m.xyz.end());
        for (int c = 0; c < m.nc(); c++) out.cptr.push_back(out.cptr.back() + (m.cptr[c + 1] - m.cptr[c]));
        for (int v : m.cverts) out.cverts.push_back(v + node0);
        out.creg.insert(out.creg.end(), m.creg.begin(), m.creg.end());
        for (int e = 0; e < m.nbe(); e++) out.bptr.push_back(out.bptr.back() + (m.bptr[e + 1] - m.bptr[e]));
        for (int v : m.bverts) out.bverts.push_back(v + node0);
        for (int t : m.btag) out.btag.push_back(t + k * span);
        for (size_t i = 0; i < bcs[k].tag.size(); i++) {
            const int ty = bcs[k].type[i];
            out_bcs.tag.push_back(bcs[k].tag[i] + k * span);
            out_bcs.type.push_back(ty < 0 ? -(-ty + k * span) : ty);
            out_bcs.value.push_back(bcs[k].value[i]);
        }
        out.comp_ptr.push_back(out.nc());
        node0 += m.nn();
    }
    return {0, ""};
}

// The union of block blk (cells c0 .. c1 - 1): its own cells, then the
// other cells that `nbr(k)` names for its entries k in [k0, k1), ascending.
// mark[] holds, per cell, the last block that listed it (blocks of one
// thread are visited in increasing order).
template <typename Nbr>
static void block_halo(int blk, int c0, int c1, int k0, int k1, Nbr &&nbr, std::vector<int> &mark,
                       std::vector<int> &halo) {
    for (int c = c0; c < c1; c++) mark[c] = blk;
    halo.clear();
    for (int k = k0; k < k1; k++) {
        const int j = nbr(k);
        if (j >= 0 && mark[j] != blk) {
            mark[j] = blk;
            halo.push_back(j);
        }
    }
    std::sort(halo.begin(), halo.end());
}

Error build_grad_tiles(const FlatMesh &m, int B, GradTiles &out) {
    out = GradTiles();
    if (B < 1 || B > 1024) return {-1, "gradient tile size out of range"};
    const int nc = m.nc;
    out.B = B;
    out.nblk = (nc + B - 1) / B;
    const int nblk = out.nblk;
    out.loc.resize(m.nbr_idx.size());
    auto nbr = [&](int q) { return m.nbr_idx[q]; };
    // union sizes per block, then the unions and local indices; blocks are
    // independent, so ranges of blocks run on the host's threads, each
    // thread with its own mark and slot arrays
    std::vector<int> nu(nblk);
    for_ranges(nblk, [&](int lo, int hi) {
        std::vector<int> mark(nc, -1), halo;
        for (int blk = lo; blk < hi; blk++) {
            const int c0 = blk * B, c1 = std::min(nc, c0 + B);
            block_halo(blk, c0, c1, m.nbr_ptr[c0], m.nbr_ptr[c1], nbr, mark, halo);
            nu[blk] = (c1 - c0) + (int)halo.size();
        }
    }, 16);
    out.ptr.assign(nblk + 1, 0);
    for (int blk = 0; blk < nblk; blk++) {
        if (nu[blk] > 65535) return {-8, "gradient tile union exceeds 16-bit local indices"};
        const int c0 = blk * B, c1 = std::min(nc, c0 + B);
        out.ptr[blk + 1] = out.ptr[blk] + nu[blk];
        out.umax = std::max(out.umax, nu[blk]);
        out.qmax = std::max(out.qmax, m.nbr_ptr[c1] - m.nbr_ptr[c0]);
    }
    out.cells.resize(out.ptr[nblk]);
    for_ranges(nblk, [&](int lo, int hi) {
        std::vector<int> mark(nc, -1), slot(nc, 0), halo;
        for (int blk = lo; blk < hi; blk++) {
            const int c0 = blk * B, c1 = std::min(nc, c0 + B);
            block_halo(blk, c0, c1, m.nbr_ptr[c0], m.nbr_ptr[c1], nbr, mark, halo);
            int *cl = out.cells.data() + out.ptr[blk];
            for (int c = c0; c < c1; c++) {
                slot[c] = c - c0;
                cl[c - c0] = c;
            }
            for (size_t h = 0; h < halo.size(); h++) {
                slot[halo[h]] = (c1 - c0) + (int)h;
                cl[(c1 - c0) + h] = halo[h];
            }
            for (int q = m.nbr_ptr[c0]; q < m.nbr_ptr[c1]; q++) out.loc[q] = (unsigned short)slot[m.nbr_idx[q]];
        }
    }, 16);
    return {0, ""};
}

Error build_face_tiles(const FlatMesh &m, int B, FaceTiles &out) {
    out = FaceTiles();
    if (B < 1 || B > 1024) return {-1, "residual tile size out of range"};
    const int nc = m.nc;
    out.B = B;
    out.nblk = (nc + B - 1) / B;
    const int nblk = out.nblk;
    out.floc.assign(m.cf_ptr[nc], 0xFFFF);
    auto nbr = [&](int k) { return m.cf_bound[k] >= 0 ? -1 : m.cf_nbr[k]; };
    // as build_grad_tiles: union sizes, then unions and face-slot indices
    std::vector<int> nu(nblk);
    for_ranges(nblk, [&](int lo, int hi) {
        std::vector<int> mark(nc, -1), halo;
        for (int blk = lo; blk < hi; blk++) {
            const int c0 = blk * B, c1 = std::min(nc, c0 + B);
            block_halo(blk, c0, c1, m.cf_ptr[c0], m.cf_ptr[c1], nbr, mark, halo);
            nu[blk] = (c1 - c0) + (int)halo.size();
        }
    }, 16);
    out.ptr.assign(nblk + 1, 0);
    for (int blk = 0; blk < nblk; blk++) {
        if (nu[blk] > 65535) return {-8, "residual tile union exceeds 16-bit local indices"};
        out.ptr[blk + 1] = out.ptr[blk] + nu[blk];
        out.umax = std::max(out.umax, nu[blk]);
    }
    out.cells.resize(out.ptr[nblk]);
    for_ranges(nblk, [&](int lo, int hi) {
        std::vector<int> mark(nc, -1), slot(nc, 0), halo;
        for (int blk = lo; blk < hi; blk++) {
            const int c0 = blk * B, c1 = std::min(nc, c0 + B);
            block_halo(blk, c0, c1, m.cf_ptr[c0], m.cf_ptr[c1], nbr, mark, halo);
            int *cl = out.cells.data() + out.ptr[blk];
            for (int c = c0; c < c1; c++) {
                slot[c] = c - c0;
                cl[c - c0] = c;
            }
            for (size_t h = 0; h < halo.size(); h++) {
                slot[halo[h]] = (c1 - c0) + (int)h;
                cl[(c1 - c0) + h] = halo[h];
            }
            for (int k = m.cf_ptr[c0]; k < m.cf_ptr[c1]; k++)
                if (m.cf_bound[k] < 0) out.floc[k] = (unsigned short)slot[m.cf_nbr[k]];
        }
    }, 16);
    return {0, ""};
}

}  // namespace gbte

namespace gbte {

bool index_checks_enabled() {
#ifdef GBTE_DEBUG
    return true;
#else
    const char *v = std::getenv("GBTE_DEBUG");
    return v && *v && std::strcmp(v, "0") != 0;
#endif
}

namespace {

// Range checks over index arrays; the first failure is kept.
struct IndexCheck {
    long long n = 0;
    std::string err;
    bool ok() const { return err.empty(); }
    void fail(const std::string &what) {
        if (err.empty()) err = what;
    }
    void size(const char *name, size_t got, size_t want) {
        if (got != want)
            fail(std::string(name) + ": " + std::to_string(got) + " entries, expected " + std::to_string(want));
    }
    void value(const char *name, size_t i, long long v, long long lo, long long hi) {
        n++;
        if (v < lo || v >= hi)
            fail(std::string(name) + "[" + std::to_string(i) + "] = " + std::to_string(v) + " outside [" +
                 std::to_string(lo) + ", " + std::to_string(hi) + ")");
    }
    void range(const char *name, const std::vector<int> &v, long long lo, long long hi) {
        for (size_t i = 0; i < v.size() && ok(); i++) value(name, i, v[i], lo, hi);
    }
    // CSR offsets of `rows` rows over `total` entries
    void offsets(const char *name, const std::vector<int> &p, size_t rows, long long total) {
        size(name, p.size(), rows + 1);
        if (!ok()) return;
        if (p[0] != 0 || p[rows] != total) fail(std::string(name) + ": offsets do not span the entries");
        for (size_t i = 0; i < rows && ok(); i++) {
            n++;
            if (p[i + 1] < p[i]) fail(std::string(name) + "[" + std::to_string(i + 1) + "] decreases");
        }
    }
};

}  // namespace

Error check_indices(const FlatMesh &m, int nb, const Schedule &s, int nd, const SweepPlan &sp, long long &checked) {
    IndexCheck c;
    const int nc = m.nc, nn = m.nn, ncf = m.ncf(), nf = m.nf(), nbd = m.nbd(), nbs = m.nbs();
    const size_t nslot = (size_t)nn * m.nmat;
    // cells and cell faces
    c.offsets("cf_ptr", m.cf_ptr, nc, ncf);
    c.size("matter", m.matter.size(), nc);
    c.range("matter", m.matter, 0, m.nmat);
    c.size("cf_nbr", m.cf_nbr.size(), ncf);
    c.size("cf_bound", m.cf_bound.size(), ncf);
    c.size("cf_bside", m.cf_bside.size(), ncf);
    c.size("cf_face", m.cf_face.size(), ncf);
    c.size("cf_v", m.cf_v.size(), 3 * (size_t)ncf);
    c.range("cf_bound", m.cf_bound, -1, nbd);
    c.range("cf_face", m.cf_face, 0, nf);
    for (int cc = 0; cc < nc && c.ok(); cc++)
        for (int k = m.cf_ptr[cc]; k < m.cf_ptr[cc + 1] && c.ok(); k++) {
            if (m.cf_bound[k] < 0) {
                c.value("cf_nbr", k, m.cf_nbr[k], 0, nc);
            } else {
                c.value("cf_bside", k, m.cf_bside[k], 0, nbs);
                if (c.ok() && (m.bs_cf[m.cf_bside[k]] != k || m.bs_cell[m.cf_bside[k]] != cc))
                    c.fail("cf_bside[" + std::to_string(k) + "] names a wall side of another cell face");
            }
            for (int t = 0; t < m.dim && c.ok(); t++) c.value("cf_v", 3 * (size_t)k + t, m.cf_v[3 * (size_t)k + t], 0, nn);
        }
    // global faces
    c.range("f_cell0", m.f_cell0, 0, nc);
    c.range("f_cf0", m.f_cf0, 0, ncf);
    c.range("f_cell1", m.f_cell1, -1, nc);
    c.range("f_cf1", m.f_cf1, -1, ncf);
    c.range("f_bound", m.f_bound, -1, nbd);
    if (m.dim == 3) c.size("face_w", m.face_w.size(), 9 * (size_t)nf);
    // least-squares stencil
    c.offsets("nbr_ptr", m.nbr_ptr, nc, (long long)m.nbr_idx.size());
    c.range("nbr_idx", m.nbr_idx, 0, nc);
    c.size("lsq_w", m.lsq_w.size(), 3 * m.nbr_idx.size());
    // walls
    c.size("b_connect", m.b_connect.size(), nbd);
    for (int ib = 0; ib < nbd && c.ok(); ib++)
        if (m.b_type[ib] < 0) c.value("b_connect", ib, m.b_connect[ib], 0, nbd);
    c.size("bs_cell", m.bs_cell.size(), nbs);
    c.size("bs_cf", m.bs_cf.size(), nbs);
    c.range("bs_cell", m.bs_cell, -1, nc);
    c.range("bs_cf", m.bs_cf, -1, ncf);
    if (!m.bs_trans.empty()) c.size("bs_trans", m.bs_trans.size(), (size_t)nbs * nb);
    // node slots
    c.offsets("nv_ptr", m.nv_ptr, nslot, (long long)m.nv_src.size());
    c.range("nv_src", m.nv_src, -(long long)nbs, nc);
    c.size("nv_w", m.nv_w.size(), m.nv_src.size());
    c.offsets("nt_ptr", m.nt_ptr, nslot, (long long)m.nt_src.size());
    c.range("nt_src", m.nt_src, 0, nc);
    c.size("nt_w", m.nt_w.size(), m.nt_src.size());
    c.size("node_x", m.node_x.size(), nn);
    c.offsets("comp_ptr", m.comp_ptr, m.ncomp() < 0 ? 0 : m.ncomp(), nc);
    // schedule: every direction's level order is a permutation of the cells
    c.size("lvl_cells", s.lvl_cells.size(), (size_t)nd * nc);
    c.size("dir_lvl_off", s.dir_lvl_off.size(), (size_t)nd * s.ncomp + 1);
    if (!s.lag.empty()) c.size("lag", s.lag.size(), (size_t)nd * nc);
    std::vector<int> seen(nc, -1);
    for (int d = 0; d < nd && c.ok(); d++)
        for (int pos = 0; pos < nc && c.ok(); pos++) {
            const int cell = s.lvl_cells[(size_t)d * nc + pos];
            c.value("lvl_cells", (size_t)d * nc + pos, cell, 0, nc);
            if (c.ok() && seen[cell] == d) c.fail("lvl_cells: direction " + std::to_string(d) + " visits a cell twice");
            if (c.ok()) seen[cell] = d;
        }
    for (size_t e = 0; e + 1 < s.dir_lvl_off.size() && c.ok(); e++) {
        c.value("dir_lvl_off", e, s.dir_lvl_off[e], 0, (long long)s.lvl_ptr.size());
        for (int l = s.dir_lvl_off[e]; l < s.dir_lvl_off[e + 1] && c.ok(); l++) {
            c.value("lvl_ptr", l, s.lvl_ptr[l], 0, (long long)nc + 1);
            if (c.ok() && l + 1 < s.dir_lvl_off[e + 1] && s.lvl_ptr[l + 1] < s.lvl_ptr[l])
                c.fail("lvl_ptr[" + std::to_string(l + 1) + "] decreases");
        }
    }
    // sweep records: upwind neighbours are earlier positions or far slots
    const size_t np = (size_t)nd * nc;
    c.size("sweep cell", sp.cell.size(), np);
    c.size("sweep nin", sp.nin.size(), np);
    c.size("sweep np", sp.np.size(), 4 * np);
    c.size("sweep far_w", sp.far_w.size(), np);
    for (size_t P = 0; P < np && c.ok(); P++) {
        const int pos = (int)(P % nc);
        c.value("sweep cell", P, sp.cell[P], 0, nc);
        c.value("sweep nin", P, sp.nin[P], 0, 5);
        c.value("sweep far_w", P, sp.far_w[P], -1, sp.far_enabled ? sp.far_slots : 0);
        for (int j = 0; j < sp.nin[P] && c.ok(); j++) {
            const int q = sp.np[4 * P + j];
            if (q >= 0)
                c.value("sweep np", 4 * P + j, q, 0, pos);
            else
                c.value("sweep np (far slot)", 4 * P + j, -1 - (long long)q, 0, sp.far_enabled ? sp.far_slots : 0);
        }
    }
    checked = c.n;
    if (!c.ok()) return {-7, "index check: " + c.err};
    return {0, ""};
}

Error check_tiles(const FlatMesh &m, const GradTiles *g, const FaceTiles *f, long long &checked) {
    IndexCheck c;
    const int nc = m.nc;
    auto tile = [&](const char *name, int B, int nblk, int umax, const std::vector<int> &ptr,
                    const std::vector<int> &cells) {
        c.size(name, (size_t)nblk, (size_t)((nc + B - 1) / std::max(1, B)));
        c.offsets(name, ptr, nblk, (long long)cells.size());
        c.range(name, cells, 0, nc);
        for (int b = 0; b < nblk && c.ok(); b++) {
            c.value(name, b, ptr[b + 1] - ptr[b], 0, (long long)umax + 1);
            // a block's union starts with its own cells in order
            for (int i = 0; i < std::min(B, nc - b * B) && c.ok(); i++)
                if (cells[ptr[b] + i] != b * B + i) c.fail(std::string(name) + ": block does not start with its cells");
        }
    };
    if (g) {
        tile("gradient tile", g->B, g->nblk, g->umax, g->ptr, g->cells);
        c.size("gradient tile loc", g->loc.size(), m.nbr_idx.size());
        for (int cc = 0; cc < nc && c.ok(); cc++) {
            const int b = cc / g->B, base = g->ptr[b], u = g->ptr[b + 1] - base;
            for (int q = m.nbr_ptr[cc]; q < m.nbr_ptr[cc + 1] && c.ok(); q++) {
                c.value("gradient tile loc", q, g->loc[q], 0, u);
                if (c.ok() && g->cells[base + g->loc[q]] != m.nbr_idx[q])
                    c.fail("gradient tile loc[" + std::to_string(q) + "] names another cell");
            }
        }
    }
    if (f) {
        tile("residual tile", f->B, f->nblk, f->umax, f->ptr, f->cells);
        c.size("residual tile floc", f->floc.size(), (size_t)m.ncf());
        for (int cc = 0; cc < nc && c.ok(); cc++) {
            const int b = cc / f->B, base = f->ptr[b], u = f->ptr[b + 1] - base;
            for (int k = m.cf_ptr[cc]; k < m.cf_ptr[cc + 1] && c.ok(); k++) {
                if (m.cf_bound[k] >= 0) {
                    if (f->floc[k] != 0xFFFF) c.fail("residual tile floc[" + std::to_string(k) + "] set on a wall");
                    continue;
                }
                c.value("residual tile floc", k, f->floc[k], 0, u);
                if (c.ok() && f->cells[base + f->floc[k]] != m.cf_nbr[k])
                    c.fail("residual tile floc[" + std::to_string(k) + "] names another cell");
            }
        }
    }
    checked = c.n;
    if (!c.ok()) return {-7, "index check: " + c.err};
    return {0, ""};
}

}  // namespace gbte
