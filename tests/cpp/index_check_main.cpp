// Host-only driver of the index checks (built by tests/test_abi.py with g++
// from the library's host sources): reads a deck directory, builds the
// flattened mesh, schedule, sweep records and tiles exactly as the solver
// does, checks them (expects a pass), then plants one bad entry per array
// kind and expects each to be caught. Prints one line per case and exits 0
// when every case behaved.
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "gbte_internal.h"

using namespace gbte;

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    Deck D;
    Error e = read_deck(argv[1], D);
    if (e.code) {
        std::printf("read_deck: %s\n", e.msg.c_str());
        return 2;
    }
    D.bands.kappa.assign(D.bands.nmat, 1.0);
    D.bands.capb.assign(D.bands.nmat, 1.0);
    FlatMesh fm;
    if ((e = build_flat_mesh(D.mesh, D.bcs, D.bands, fm)).code) {
        std::printf("build_flat_mesh: %s\n", e.msg.c_str());
        return 2;
    }
    Angles ang;
    if ((e = make_angles(D.angle_method, D.n_theta, D.n_phi, D.bands.material_dim, ang)).code) return 2;
    Schedule sch;
    build_schedule(fm, ang, sch, 2);
    SweepPlan sp;
    if ((e = build_sweep_plan(fm, ang, sch, kSweepMinRing, kSweepFarCap, sp)).code) return 2;
    GradTiles gt;
    FaceTiles ft;
    if (build_grad_tiles(fm, 64, gt).code || build_face_tiles(fm, 64, ft).code) return 2;

    int bad = 0;
    auto run = [&](const char *name, bool expect_pass, const std::function<Error(long long &)> &f) {
        long long n = 0;
        Error r = f(n);
        const bool passed = r.code == 0;
        std::printf("%s: %s (%lld entries) %s\n", name, passed ? "pass" : "caught", n, r.msg.c_str());
        if (passed != expect_pass || (!passed && r.code != -7)) bad++;
    };
    auto mesh_check = [&](const FlatMesh &m, const Schedule &s, const SweepPlan &p) {
        return [&m, &s, &p, &ang, &D](long long &n) { return check_indices(m, D.bands.nb, s, ang.nd, p, n); };
    };
    run("built", true, mesh_check(fm, sch, sp));
    run("tiles", true, [&](long long &n) { return check_tiles(fm, &gt, &ft, n); });
    {
        FlatMesh m = fm;
        for (size_t k = 0; k < m.cf_bound.size(); k++)
            if (m.cf_bound[k] < 0) {
                m.cf_nbr[k] = m.nc;
                break;
            }
        run("cf_nbr past the cells", false, mesh_check(m, sch, sp));
    }
    {
        FlatMesh m = fm;
        m.nv_ptr[1] = m.nv_ptr[2] + 1;
        run("nv_ptr decreasing", false, mesh_check(m, sch, sp));
    }
    {
        FlatMesh m = fm;
        m.nbr_idx.back() = -1;
        run("nbr_idx negative", false, mesh_check(m, sch, sp));
    }
    {
        FlatMesh m = fm;
        m.nv_src[0] = -1 - m.nbs();
        run("nv_src past the wall sides", false, mesh_check(m, sch, sp));
    }
    {
        Schedule s = sch;
        s.lvl_cells[1] = s.lvl_cells[0];
        run("level order visits a cell twice", false, mesh_check(fm, s, sp));
    }
    {
        SweepPlan p = sp;
        for (size_t P = 0; P < p.nin.size(); P++)
            if (p.nin[P] > 0 && p.np[4 * P] >= 0) {
                p.np[4 * P] = (int)(P % fm.nc);  // its own position: not upwind
                break;
            }
        run("sweep record reads a later position", false, mesh_check(fm, sch, p));
    }
    {
        GradTiles t = gt;
        t.loc[0] = (unsigned short)(t.ptr[1] - t.ptr[0]);
        run("gradient tile index past its union", false, [&](long long &n) { return check_tiles(fm, &t, nullptr, n); });
    }
    {
        FaceTiles t = ft;
        for (size_t k = 0; k < t.floc.size(); k++)
            if (fm.cf_bound[k] < 0) {
                t.floc[k] = (unsigned short)(t.floc[k] == 0 ? 1 : 0);
                break;
            }
        run("residual tile names another cell", false, [&](long long &n) { return check_tiles(fm, nullptr, &t, n); });
    }
    std::printf("%s\n", bad ? "FAILED" : "OK");
    return bad ? 1 : 0;
}
