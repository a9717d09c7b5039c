// Deck reader: the reference's input files, parsed with the same keyword
// semantics (a line that contains a keyword and no '!' is followed by its
// value as the next whitespace-separated token; src/BTEMain.cpp:87-315,
// src/BTEBand/BTEBand.cpp:14-79,740-836,
// src/BTEBoundaryCondition/BTEBoundaryCondition.cpp:8-31,
// src/BTEMesh/ReadinMesh.cpp:228-534, src/BTEMesh/BTEMesh.cpp:1056-1107).
// Relative file names are resolved against the deck directory, which plays
// the role of the reference's working directory. Failures return an Error
// instead of exiting.
#include <cmath>
#include <fstream>
#include <sstream>

#include "gbte_internal.h"

namespace gbte {
namespace {

bool has_kw(const std::string &line, const char *kw) {
    return line.find(kw) != std::string::npos && line.find('!') == std::string::npos;
}

std::string resolve(const std::string &root, const std::string &p) {
    if (p.empty() || p[0] == '/') return p;
    return root + "/" + p;
}

bool has_word(const std::string &line, const char *w) { return line.find(w) != std::string::npos; }

int leading_int(const std::string &s) {
    std::istringstream ss(s);
    int v = 0;
    ss >> v;
    return v;
}

Error read_comsol(std::ifstream &in, int dim, double Lx, double Ly, RawMesh &m) {
    if (dim != 2) return {-8, "COMSOL meshes are read in 2D only"};
    std::string s;
    std::getline(in, s);
    if (!has_word(s, "COMSOL")) return {-2, "mesh file format error (no COMSOL header)"};
    int sdim = -1;
    while (std::getline(in, s))
        if (has_word(s, "# sdim")) {
            sdim = leading_int(s);
            break;
        }
    if (sdim != dim) return {-2, "COMSOL sdim does not match GeometryDimension"};
    int nn = -1;
    while (std::getline(in, s))
        if (has_word(s, "# number of mesh")) {
            nn = leading_int(s);
            break;
        }
    if (nn <= 0) return {-2, "COMSOL: no mesh vertices"};
    for (int i = 0; i < 3; i++) std::getline(in, s);
    m.xyz.assign(3 * (size_t)nn, 0.0);
    for (int i = 0; i < nn; i++) {
        double x, y;
        if (!(in >> x >> y)) return {-2, "COMSOL: truncated vertex block"};
        m.xyz[3 * i] = x * Lx;
        m.xyz[3 * i + 1] = y * Ly;
    }
    int ntypes = 0;
    while (std::getline(in, s))
        if (has_word(s, "# number of element types")) {
            ntypes = leading_int(s);
            break;
        }
    std::vector<std::vector<int>> cells, bels;
    std::vector<int> creg, btag;
    while (ntypes-- > 0) {
        int nv = -1;
        while (std::getline(in, s))
            if (has_word(s, "# number of vertices per element") || has_word(s, "# number of nodes per element")) {
                nv = leading_int(s);
                break;
            }
        if (nv != 2 && nv != 3 && nv != 4) continue;  // vertex elements are skipped
        int ne = 0;
        while (std::getline(in, s))
            if (has_word(s, "# number of elements")) {
                ne = leading_int(s);
                break;
            }
        std::getline(in, s);
        std::vector<std::vector<int>> el(ne, std::vector<int>(nv));
        for (int i = 0; i < ne; i++)
            for (int k = 0; k < nv; k++)
                if (!(in >> el[i][k])) return {-2, "COMSOL: truncated element block"};
        for (int i = 0; i < 4; i++) std::getline(in, s);
        std::vector<int> ent(ne);
        for (int i = 0; i < ne; i++)
            if (!(in >> ent[i])) return {-2, "COMSOL: truncated entity block"};
        if (nv == 2) {
            for (int i = 0; i < ne; i++) {
                bels.push_back(el[i]);
                btag.push_back(ent[i] + 1);
            }
        } else {
            for (int i = 0; i < ne; i++) {
                cells.push_back(el[i]);
                creg.push_back(ent[i] - 1);
            }
        }
    }
    m.cptr.assign(1, 0);
    for (auto &c : cells) {
        m.cverts.insert(m.cverts.end(), c.begin(), c.end());
        m.cptr.push_back((int)m.cverts.size());
    }
    m.creg = creg;
    m.bptr.assign(1, 0);
    for (auto &b : bels) {
        m.bverts.insert(m.bverts.end(), b.begin(), b.end());
        m.bptr.push_back((int)m.bverts.size());
    }
    m.btag = btag;
    return {0, ""};
}

// gmsh MSH 4.1 ASCII. 2D: line elements (type 1) are boundary elements tagged
// by their entity tag, triangles (2) and quads (3, read as a0 a1 a3 a2) are
// cells in region (entity tag - 1). 3D (not in the reference's public
// release): triangles (2) are boundary elements, tetrahedra (4) are cells.
Error read_msh(std::ifstream &in, int dim, double Lx, double Ly, double Lz, RawMesh &m) {
    std::string s;
    std::getline(in, s);
    if (!has_word(s, "MeshFormat")) return {-2, "mesh file format error (no $MeshFormat)"};
    int nblock = 0, nn = 0;
    bool got_nodes = false;
    while (std::getline(in, s))
        if (has_word(s, "Nodes")) {
            long long mn, mx;
            in >> nblock >> nn >> mn >> mx;
            std::getline(in, s);
            m.xyz.assign(3 * (size_t)nn, 0.0);
            for (int b = 0; b < nblock; b++) {
                int edim, etag, para, cnt;
                in >> edim >> etag >> para >> cnt;
                std::vector<long long> tag(cnt);
                for (int j = 0; j < cnt; j++) in >> tag[j];
                for (int j = 0; j < cnt; j++) {
                    double x, y, z;
                    in >> x >> y >> z;
                    if (tag[j] < 1 || tag[j] > nn) return {-2, "MSH: node tag out of range"};
                    m.xyz[3 * (tag[j] - 1)] = x * Lx;
                    m.xyz[3 * (tag[j] - 1) + 1] = y * Ly;
                    m.xyz[3 * (tag[j] - 1) + 2] = dim == 3 ? z * Lz : 0.0;
                }
            }
            got_nodes = true;
            break;
        }
    if (!got_nodes || !in) return {-2, "MSH: no $Nodes section"};
    m.cptr.assign(1, 0);
    m.bptr.assign(1, 0);
    while (std::getline(in, s))
        if (has_word(s, "Elements")) {
            long long ne, mn, mx;
            in >> nblock >> ne >> mn >> mx;
            std::getline(in, s);
            for (int b = 0; b < nblock; b++) {
                int edim, etag, type, cnt;
                in >> edim >> etag >> type >> cnt;
                std::getline(in, s);
                for (int j = 0; j < cnt; j++) {
                    long long lt;
                    if (dim == 2 && type == 1) {
                        int a0, a1;
                        in >> lt >> a0 >> a1;
                        m.bverts.push_back(a0 - 1);
                        m.bverts.push_back(a1 - 1);
                        m.bptr.push_back((int)m.bverts.size());
                        m.btag.push_back(etag);
                    } else if (dim == 2 && type == 2) {
                        int a[3];
                        in >> lt >> a[0] >> a[1] >> a[2];
                        for (int k = 0; k < 3; k++) m.cverts.push_back(a[k] - 1);
                        m.cptr.push_back((int)m.cverts.size());
                        m.creg.push_back(etag - 1);
                    } else if (dim == 2 && type == 3) {
                        int a[4];
                        in >> lt >> a[0] >> a[1] >> a[3] >> a[2];
                        for (int k = 0; k < 4; k++) m.cverts.push_back(a[k] - 1);
                        m.cptr.push_back((int)m.cverts.size());
                        m.creg.push_back(etag - 1);
                    } else if (dim == 3 && type == 2) {
                        int a[3];
                        in >> lt >> a[0] >> a[1] >> a[2];
                        for (int k = 0; k < 3; k++) m.bverts.push_back(a[k] - 1);
                        m.bptr.push_back((int)m.bverts.size());
                        m.btag.push_back(etag);
                    } else if (dim == 3 && type == 4) {
                        int a[4];
                        in >> lt >> a[0] >> a[1] >> a[2] >> a[3];
                        for (int k = 0; k < 4; k++) m.cverts.push_back(a[k] - 1);
                        m.cptr.push_back((int)m.cverts.size());
                        m.creg.push_back(etag - 1);
                    } else {
                        std::getline(in, s);
                    }
                    if (dim == 2 && edim == 3) return {-2, "MSH: three-dimensional element in a 2D mesh"};
                }
            }
            break;
        }
    if (m.cptr.size() < 2) return {-2, "MSH: no cells"};
    return {0, ""};
}

}  // namespace

Error read_deck(const std::string &root, Deck &D) {
    D = Deck();
    const std::string in = root + "/input/";
    std::string str;
    // CONTROL
    {
        std::ifstream f(in + "CONTROL");
        if (!f.is_open()) return {-2, "need input/CONTROL"};
        std::string state = "Steady";
        while (std::getline(f, str)) {
            if (has_kw(str, "State")) f >> state;
            if (has_kw(str, "Order")) f >> D.order;
            if (has_kw(str, "IterativeScheme")) f >> D.method;
            if (has_kw(str, "MatrixSolver")) f >> D.matrix;
            if (has_kw(str, "Tref")) f >> D.tref;
            if (has_kw(str, "MaxNumIter")) f >> D.max_iter;
            if (has_kw(str, "ResidualTemp")) f >> D.err_temp;
            if (has_kw(str, "ResidualFlux")) f >> D.err_flux;
            if (has_kw(str, "InitialTemperatureFile")) return {-8, "InitialTemperatureFile is not supported"};
        }
        if (state != "Steady") return {-8, "only State=Steady is implemented"};
    }
    // GEOMETRY
    int gdim = -1;
    double Lx = 1, Ly = 1, Lz = 1;
    std::string bcfile, meshtype, meshfile, heattype, heatfile;
    {
        std::ifstream f(in + "GEOMETRY");
        if (!f.is_open()) return {-2, "need input/GEOMETRY"};
        while (std::getline(f, str)) {
            if (has_kw(str, "GeometryDimension")) f >> gdim;
            if (has_kw(str, "ScaleX")) f >> Lx;
            if (has_kw(str, "ScaleY")) f >> Ly;
            if (has_kw(str, "ScaleZ")) f >> Lz;
            if (has_kw(str, "UniformHeat")) f >> D.uniform_heat;
            if (has_kw(str, "BCFile")) f >> bcfile;
            if (has_kw(str, "MeshType")) f >> meshtype;
            if (has_kw(str, "MeshFile")) f >> meshfile;
            if (has_kw(str, "HeatType")) f >> heattype;
            if (has_kw(str, "HeatFile")) f >> heatfile;
        }
    }
    if (gdim != 2 && gdim != 3) return {-1, "GeometryDimension must be 2 or 3"};
    // PHONON: angles
    int mdim = 3;
    {
        std::ifstream f(in + "PHONON");
        if (!f.is_open()) return {-2, "need input/PHONON"};
        while (std::getline(f, str)) {
            if (has_kw(str, "MaterialDimension")) f >> mdim;
            if (has_kw(str, "Angle_method")) f >> D.angle_method;
            if (has_kw(str, "Ntheta")) f >> D.n_theta;
            if (has_kw(str, "Nphi")) f >> D.n_phi;
        }
    }
    // PHONON: bands (DATABASE or inline tables)
    Bands &B = D.bands;
    B.material_dim = mdim;
    {
        std::ifstream f(in + "PHONON");
        int nmat = 0, nb = 0;
        while (std::getline(f, str)) {
            if (has_kw(str, "MaterialNumber")) f >> nmat;
            if (has_kw(str, "BandNumber")) f >> nb;
        }
        if (nmat <= 0 || nb <= 0) return {-2, "PHONON: provide MaterialNumber and BandNumber"};
        B.nmat = nmat;
        B.nb = nb;
        B.v.assign(nmat * nb, 0);
        B.tau = B.C = B.lat = B.hr = B.v;
        std::ifstream g(in + "PHONON");
        for (int i = 0; i < nmat; i++) {
            bool got = false;
            while (std::getline(g, str)) {
                if (!has_word(str, "MaterialFile")) continue;
                if (!has_word(str, "DATABASE")) return {-8, "only DATABASE material files are supported"};
                std::string file;
                g >> file;
                std::ifstream t(resolve(root, file));
                if (!t.is_open()) return {-2, "DATABASE band file not open: " + file};
                for (int j = 0; j < nb; j++)
                    if (!(t >> B.v[i * nb + j] >> B.tau[i * nb + j] >> B.C[i * nb + j] >> B.lat[i * nb + j] >> B.hr[i * nb + j]))
                        return {-2, "DATABASE band file too short: " + file};
                got = true;
                break;
            }
            if (!got) return {-2, "PHONON: missing MaterialFile entry"};
        }
        while (std::getline(g, str))
            if (has_word(str, "GeometryMaterialType")) {
                while (std::getline(g, str)) {
                    if (str.length() <= 1) break;
                    std::istringstream ss(str);
                    int a, b;
                    if (!(ss >> a >> b)) break;
                    if (std::abs(b) > 100) break;
                    B.region_material.push_back(b - 1);
                }
            }
        if (B.region_material.empty()) return {-2, "PHONON: missing GeometryMaterialType"};
        for (int mtl : B.region_material)
            if (mtl < 0 || mtl >= nmat) return {-2, "PHONON: GeometryMaterialType names an unknown material"};
    }
    // BC table
    {
        std::ifstream f(resolve(root, bcfile));
        if (!f.is_open()) return {-2, "BC file not open: " + bcfile};
        int num = 0;
        f >> num;
        for (int i = 0; i < 3; i++) std::getline(f, str);
        std::vector<std::vector<double>> rows;  // transmissivity per row, [nmat * nb]
        bool any5 = false;
        for (int i = 0; i < num; i++) {
            int idx, type;
            double val;
            if (!(f >> idx >> type)) return {-2, "BC file truncated"};
            if (type == 4) return {-8, "BC type 4 has no steady-state branch in the reference solver"};
            f >> val;
            std::vector<double> tr((size_t)B.nmat * B.nb, 0.0);
            if (type == 5) {
                // interface wall: value, then the transmissivity file
                // (BTEBoundaryCondition.cpp:22-35): blocks that start at a
                // line naming "matter" (its first token the 0-based
                // material), one value per line, ended by a short line
                std::string tfile;
                f >> tfile;
                std::ifstream tf(resolve(root, tfile));
                if (!tf.is_open()) return {-2, "interface file not open: " + tfile};
                std::string line;
                while (std::getline(tf, line)) {
                    size_t at = line.find("matter");
                    if (at == std::string::npos || at == 0) continue;
                    const int mt = std::atoi(line.substr(0, line.find(' ')).c_str());
                    if (mt < 0 || mt >= B.nmat) return {-2, "interface file names an unknown material: " + tfile};
                    int b = 0;
                    while (std::getline(tf, line)) {
                        if (line.length() <= 1) break;
                        if (b < B.nb) tr[(size_t)mt * B.nb + b] = std::atof(line.c_str());
                        b++;
                    }
                    if (b != B.nb) return {-2, "interface file: band count differs from the band table: " + tfile};
                }
                any5 = true;
            }
            std::getline(f, str);
            D.bcs.tag.push_back(idx);
            D.bcs.type.push_back(type);
            D.bcs.value.push_back(val);
            rows.push_back(tr);
        }
        if (any5)
            for (auto &r : rows) D.bcs.trans.insert(D.bcs.trans.end(), r.begin(), r.end());
    }
    // mesh
    {
        std::ifstream f(resolve(root, meshfile));
        if (!f.is_open()) return {-2, "mesh file not open: " + meshfile};
        D.mesh.dim = gdim;
        D.mesh.Lx = Lx;
        D.mesh.Ly = Ly;
        D.mesh.Lz = Lz;
        Error e;
        if (meshtype == "COMSOL")
            e = read_comsol(f, gdim, Lx, Ly, D.mesh);
        else if (meshtype == "MSH")
            e = read_msh(f, gdim, Lx, Ly, Lz, D.mesh);
        else
            return {-8, "unsupported MeshType " + meshtype};
        if (e.code) return e;
    }
    // heat source per cell (BTEMesh.cpp:1056-1104)
    const int nc = D.mesh.nc();
    D.cell_heat.assign(nc, D.uniform_heat);
    if (!heatfile.empty()) {
        std::ifstream f(resolve(root, heatfile));
        if (f.is_open() && heattype == "REGION") {
            int nr = 0;
            f >> nr;
            std::getline(f, str);
            std::vector<int> idx(nr);
            std::vector<double> q(nr);
            for (int i = 0; i < nr; i++) f >> idx[i] >> q[i];
            for (int c = 0; c < nc; c++) {
                int r = D.mesh.creg[c];
                if (r < 0 || r >= nr) return {-2, "heat file does not cover every region"};
                D.cell_heat[c] = q[r];
            }
        } else if (f.is_open() && heattype == "COORDINATE") {
            return {-8, "HeatType COORDINATE is not supported"};
        }
    }
    return {0, ""};
}

}  // namespace gbte
