// Deck reader: the reference's input files, parsed with the same keyword
// semantics (a line that contains a keyword and no '!' is followed by its
// value as the next whitespace-separated token; src/BTEMain.cpp:87-315,
// src/BTEBand/BTEBand.cpp:14-79,740-836,
// src/BTEBoundaryCondition/BTEBoundaryCondition.cpp:8-31,
// src/BTEMesh/ReadinMesh.cpp:228-534, src/BTEMesh/BTEMesh.cpp:1056-1107).
// Relative file names are resolved against the deck directory, which plays
// the role of the reference's working directory. Failures return an Error
// instead of exiting.
#include <algorithm>
#include <cmath>
#include <cstdlib>
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

// ---- band tables from first-principles mode lists (BTEBand.cpp:81-737) ----
//
// Both readers reduce a list of phonon modes (capacity C, |v|, kappa
// contribution k), in the order the files give them, to nb bands of equal
// mode count: with m = (number of modes) / nb (integer division), mode j goes
// to band min(j / m, nb - 1), so the last band takes the remainder. Per band
// the sums run in mode order: v = sum C v / sum C, C = sum C,
// tau = sum k / C / v / v, then lattice_ratio = (C / tau) / sum_b (C / tau)
// and heat_ratio = C / sum_b C (BTEBand.cpp:568-613, :691-724).
struct Mode {
    double C, v, k;
};

Error bin_modes(const std::vector<Mode> &modes, int nb, double *v, double *tau, double *C, double *lat,
                double *hr, const std::string &what) {
    const int n = (int)modes.size();
    const int per = n / nb;
    std::vector<double> sC(nb, 0.0), sCv(nb, 0.0), sk(nb, 0.0);
    for (int j = 0; j < n; j++) {
        const int b = per > 0 ? std::min(j / per, nb - 1) : nb - 1;
        sC[b] += modes[j].C;
        sCv[b] += modes[j].C * modes[j].v;
        sk[b] += modes[j].k;
    }
    double sumL = 0, sumheat = 0;
    for (int b = 0; b < nb; b++) {
        v[b] = sCv[b] / sC[b];
        C[b] = sC[b];
        tau[b] = sk[b] / C[b] / v[b] / v[b];
        sumL += C[b] / tau[b];
        sumheat += C[b];
    }
    for (int b = 0; b < nb; b++) {
        lat[b] = C[b] / tau[b] / sumL;
        hr[b] = C[b] / sumheat;
        if (!std::isfinite(v[b]) || !std::isfinite(tau[b]) || !std::isfinite(lat[b]))
            return {-2, what + ": band " + std::to_string(b + 1) + " has no modes with a finite capacity"};
    }
    return {0, ""};
}

// whitespace-separated numbers of one line (NaN and inf as strtod reads them)
std::vector<double> numbers(const std::string &line) {
    std::vector<double> out;
    const char *p = line.c_str();
    while (*p) {
        while (*p == ' ' || *p == '\t' || *p == '\r') p++;
        if (!*p) break;
        char *end = nullptr;
        const double x = std::strtod(p, &end);
        if (end == p) break;
        out.push_back(x);
        p = end;
    }
    return out;
}

// rows of numbers until the first line of at most one character
std::vector<std::vector<double>> number_rows(std::ifstream &f) {
    std::vector<std::vector<double>> rows;
    std::string line;
    while (std::getline(f, line)) {
        if (line.length() <= 1) break;
        rows.push_back(numbers(line));
    }
    return rows;
}

// ALAMODE lifetime file (BTEBand.cpp:629-731): after the "Phonon lifetime"
// line, "# kpoint range k0 k1" and "# mode range b0 b1", a header line, then
// one line per (k-point, branch): ik, is, frequency [cm^-1], lifetime [ps],
// |v| [m/s], MFP, multiplicity and the nine per-mode conductivity tensor
// entries xx .. zz. kappa = (xx + yy + zz) multiplicity,
// C = kappa / v / v / tau (0 where tau or v is 0). `key_len` is the length of
// the PHONON line that named the file: the reference accepts the
// "Phonon lifetime" line only where the phrase starts before that column.
Error read_alamode(const std::string &path, int nb, size_t key_len, double *v, double *tau, double *C,
                   double *lat, double *hr) {
    std::ifstream f(path);
    if (!f.is_open()) return {-2, "ALAMODE band file not open: " + path};
    std::string line;
    while (std::getline(f, line)) {
        const size_t at = line.find("Phonon lifetime");
        if (!(at > 0 && at < key_len)) continue;
        std::string w1, w2, w3;
        long k0 = 0, k1 = -1, b0 = 0, b1 = -1;
        if (!(f >> w1 >> w2 >> w3 >> k0 >> k1 >> w1 >> w2 >> w3 >> b0 >> b1))
            return {-2, "ALAMODE: missing kpoint/mode ranges: " + path};
        std::getline(f, line);
        std::getline(f, line);
        const long n = (b1 - b0 + 1) * (k1 - k0 + 1);
        if (n <= 0) return {-2, "ALAMODE: empty mode range: " + path};
        std::vector<Mode> modes((size_t)n);
        for (long j = 0; j < n; j++) {
            double iq, ib, freq, t, vel, mfp, mult, k[9];
            if (!(f >> iq >> ib >> freq >> t >> vel >> mfp >> mult)) return {-2, "ALAMODE: truncated mode list: " + path};
            for (double &x : k)
                if (!(f >> x)) return {-2, "ALAMODE: truncated mode list: " + path};
            Mode &m = modes[(size_t)j];
            t *= 1e-12;
            m.v = vel;
            m.k = (k[0] + k[4] + k[8]) * mult;
            m.C = (t == 0 || vel == 0) ? 0.0 : m.k / vel / vel / t;
        }
        return bin_modes(modes, nb, v, tau, C, lat, hr, "ALAMODE " + path);
    }
    return {-2, "ALAMODE: no \"Phonon lifetime\" section: " + path};
}

// ShengBTE output directory (BTEBand.cpp:81-617): CONTROL gives lfactor
// [nm], the three lattice vectors and T; BTE.omega the frequencies [rad/ps]
// per irreducible q-point (row) and branch (column); BTE.qpoints_full the
// full grid (second column: the irreducible q-point, 1-based); BTE.w_final
// and BTE.v one row per (branch, irreducible q-point), branch-major: the
// scattering rate [1/ps] in column 2 and the group velocity [km/s]. Per
// full-grid mode: C = (1/V) kB x^2 e^x / (e^x - 1)^2 / Nq with
// x = hbar omega / (kB T), tau = 1 / w, kappa = C v^2 tau, taken branch by
// branch over the full grid, skipping modes whose kappa is NaN or negative.
// As in the reference: V is formed with lattvec(1,2) in place of
// lattvec(2,1) in one term of the determinant, kB = 1.38062e-23 and
// hbar = 1.05459e-34, and T comes from the last CONTROL line holding an
// upper-case T past its first column and neither TRUE nor True.
Error read_shengbte(const std::string &dir, int nb, double *v, double *tau, double *C, double *lat, double *hr) {
    std::ifstream ctl(dir + "/CONTROL");
    if (!ctl.is_open()) return {-2, "ShengBTE CONTROL file not open: " + dir};
    double lf = 1.0, T = 0, a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    std::string line;
    auto after_eq = [](const std::string &l) { return l.substr(l.find('=') + 1); };
    while (std::getline(ctl, line)) {
        const size_t at_lf = line.find("lfactor");
        if (at_lf > 0 && at_lf != std::string::npos) lf = std::strtod(after_eq(line).c_str(), nullptr);
        for (int r = 0; r < 3; r++) {
            const std::string key = "lattvec(:," + std::to_string(r + 1) + ")";
            const size_t at = line.find(key);
            if (at > 0 && at != std::string::npos) {
                const std::vector<double> x = numbers(after_eq(line));
                for (int c = 0; c < 3 && c < (int)x.size(); c++) a[r][c] = x[c];
            }
        }
        const size_t at_t = line.find('T');
        if (at_t > 0 && at_t != std::string::npos) {
            const std::string rest = after_eq(line);
            if (rest.find("TRUE") == std::string::npos && rest.find("True") == std::string::npos)
                T = std::strtod(rest.c_str(), nullptr);
        }
    }
    double V = (a[0][0] * a[1][1] * a[2][2] + a[1][0] * a[2][1] * a[0][2] + a[0][1] * a[1][2] * a[2][0] -
                a[0][2] * a[1][1] * a[2][0] - a[0][1] * a[0][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1]) *
               lf * lf * lf;
    V = std::fabs(V) * 1e-27;
    if (!(T > 0) || !(V > 0)) return {-2, "ShengBTE CONTROL: no temperature or cell volume: " + dir};
    std::vector<std::vector<double>> om, qf, wf, vf;
    for (auto &p : {std::make_pair("/BTE.omega", &om), std::make_pair("/BTE.qpoints_full", &qf),
                    std::make_pair("/BTE.w_final", &wf), std::make_pair("/BTE.v", &vf)}) {
        std::ifstream g(dir + p.first);
        if (!g.is_open()) return {-2, std::string("ShengBTE file not open: ") + dir + p.first};
        *p.second = number_rows(g);
    }
    const int nirr = (int)om.size(), nq = (int)qf.size();
    if (nirr == 0 || nq == 0) return {-2, "ShengBTE: empty BTE.omega or BTE.qpoints_full: " + dir};
    const int nbr = (int)om.back().size();  // branches: the count of the last row
    const double kb = 1.38062e-23, hbar = 1.05459e-34;
    std::vector<Mode> modes;
    for (int br = 0; br < nbr; br++)
        for (int q = 0; q < nq; q++) {
            if (qf[q].size() < 2) return {-2, "ShengBTE: short BTE.qpoints_full row: " + dir};
            const int irr = (int)qf[q][1] - 1;
            const size_t row = (size_t)br * nirr + irr;
            if (irr < 0 || irr >= nirr || (int)om[irr].size() <= br || row >= wf.size() || row >= vf.size() ||
                wf[row].size() < 2 || vf[row].size() < 3)
                return {-2, "ShengBTE: q-point or branch outside the files: " + dir};
            const double w = om[irr][br] * 1e12;
            const double t = 1 / wf[row][1] * 1e-12;
            const double vel = std::pow(std::pow(vf[row][0] * 1000, 2) + std::pow(vf[row][1] * 1000, 2) +
                                            std::pow(vf[row][2] * 1000, 2),
                                        0.5);
            const double x = hbar * w / kb / T;
            const double cap = 1 / V * kb * x * x * std::exp(x) / std::pow(std::exp(x) - 1, 2);
            const double k = cap / nq * vel * vel * t;
            if (std::isnan(k) || !(k >= 0)) continue;
            modes.push_back({cap / nq, vel, k});
        }
    if (modes.empty()) return {-2, "ShengBTE: no mode with a finite conductivity: " + dir};
    return bin_modes(modes, nb, v, tau, C, lat, hr, "ShengBTE " + dir);
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
            if (has_kw(str, "TimeStep")) f >> D.time_step;
            if (has_kw(str, "TotalTime")) f >> D.total_time;
            if (has_kw(str, "InitialTemperatureFile")) return {-8, "InitialTemperatureFile is not supported"};
        }
        if (state != "Steady" && state != "Transient") return {-8, "State must be Steady or Transient"};
        D.transient = state == "Transient";
        if (D.transient && (D.time_step == -1 || D.total_time == -1))
            return {-2, "provide TimeStep and TotalTime for the transient solver"};
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
                // the source named on the line, in the reference's order of
                // tests: DATABASE, ShengBTE, ALAMODE (BTEBand.cpp:60-81, :629)
                const size_t at_db = str.find("DATABASE"), at_sh = str.find("ShengBTE"), at_al = str.find("ALAMODE");
                std::string file;
                g >> file;
                double *bv = &B.v[i * nb], *bt = &B.tau[i * nb], *bc = &B.C[i * nb], *bl = &B.lat[i * nb],
                       *bh = &B.hr[i * nb];
                if (at_db > 0 && at_db != std::string::npos) {
                    std::ifstream t(resolve(root, file));
                    if (!t.is_open()) return {-2, "DATABASE band file not open: " + file};
                    for (int j = 0; j < nb; j++)
                        if (!(t >> bv[j] >> bt[j] >> bc[j] >> bl[j] >> bh[j]))
                            return {-2, "DATABASE band file too short: " + file};
                } else if (at_sh > 0 && at_sh != std::string::npos) {
                    Error e = read_shengbte(resolve(root, file), nb, bv, bt, bc, bl, bh);
                    if (e.code) return e;
                } else if (at_al > 0 && at_al != std::string::npos) {
                    Error e = read_alamode(resolve(root, file), nb, str.length(), bv, bt, bc, bl, bh);
                    if (e.code) return e;
                } else {
                    return {-8, "MaterialFile: unknown source (DATABASE, ShengBTE or ALAMODE)"};
                }
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
                    // the reference warns and goes on, reading past the end of
                    // its table for the missing bands; here the deck is refused
                    if (b != B.nb)
                        return {-2, "interface file " + tfile + ": material " + std::to_string(mt) + " lists " +
                                        std::to_string(b) + " transmissivities for " + std::to_string(B.nb) + " bands"};
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
