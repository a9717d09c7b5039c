// Host check of the sweep plan's on-chip addressing (test program).
//
// Reads a deck directory, builds the flattened mesh, the per-direction level
// schedule and the sweep plan with the given smallest ring (1: the ring is
// as small as the widest level allows, so many upwind reads fall outside it)
// and runs, per direction and for random residuals, two sweeps of
// d_c = (R_c - kb sum_j a_j d_j) / (1 + kb sig_c):
//   direct: every correction kept by position;
//   plan:   only a ring of the plan's size and the far slots, addressed
//           exactly as the device sweep does (np >= lo: ring, np < 0: far
//           slot), each level reading all its operands before any of its
//           cells writes (the device's level-parallel order).
// With a copies argument > 1 the check runs on a batch of that many copies
// of the deck (disjoint union, one level list per copy and direction).
// Prints "far_refs <n> far_slots <n> ring <n> max_abs_diff <x>" and exits 1
// if the sweeps differ or a far reference found neither ring nor slot.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "gbte_internal.h"

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s deck_dir min_ring [perturb|plain] [copies]\n", argv[0]);
        return 2;
    }
    gbte::Deck deck;
    gbte::Error e = gbte::read_deck(argv[1], deck);
    if (e.code) {
        std::fprintf(stderr, "read_deck: %s\n", e.msg.c_str());
        return 2;
    }
    gbte::Angles ang;
    e = gbte::make_angles(deck.angle_method, deck.n_theta, deck.n_phi, deck.bands.material_dim, ang);
    if (e.code) return std::fprintf(stderr, "angles: %s\n", e.msg.c_str()), 2;
    // optional: a batch of `copies` copies of the deck (disjoint union)
    const int copies = argc > 4 ? std::atoi(argv[4]) : 1;
    gbte::RawMesh raw = deck.mesh;
    gbte::BCs bcs = deck.bcs;
    if (copies > 1) {
        std::vector<gbte::RawMesh> ms(copies, deck.mesh);
        std::vector<gbte::BCs> bs(copies, deck.bcs);
        e = gbte::make_union(ms, bs, raw, bcs);
        if (e.code) return std::fprintf(stderr, "union: %s\n", e.msg.c_str()), 2;
    }
    gbte::FlatMesh fm;
    e = gbte::build_flat_mesh(raw, bcs, deck.bands, fm);
    if (e.code) return std::fprintf(stderr, "mesh: %s\n", e.msg.c_str()), 2;
    gbte::Schedule sch;
    gbte::build_schedule(fm, ang, sch, 4);
    gbte::SweepPlan sp;
    e = gbte::build_sweep_plan(fm, ang, sch, std::atoi(argv[2]), 1 << 20, sp);
    if (e.code) return std::fprintf(stderr, "plan: %s\n", e.msg.c_str()), 2;
    if (!sp.far_enabled) return std::fprintf(stderr, "far slots not enabled\n"), 1;
    if (fm.ncomp() != copies || sch.ncomp != copies) return std::fprintf(stderr, "components lost\n"), 1;
    if (argc > 3 && std::string(argv[3]) == "perturb" && sp.far_slots > 1) {
        // plant one wrong far slot in the plan (the check must then fail)
        for (size_t k = 0; k < sp.np.size(); k++)
            if (sp.np[k] < 0) {
                sp.np[k] = -1 - ((-1 - sp.np[k] + 1) % sp.far_slots);
                break;
            }
    }
    const int nc = fm.nc, nd = ang.nd, ring = sp.ring, mask = ring - 1;
    std::mt19937 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    double maxdiff = 0;
    bool bad = false;
    const double kb = 0.7;
    for (int e = 0; e < nd * sch.ncomp; e++) {
        const int d = e / sch.ncomp;
        const int *lp = &sch.lvl_ptr[sch.dir_lvl_off[e]];
        const int nl = sch.dir_lvl_off[e + 1] - sch.dir_lvl_off[e] - 1;
        const size_t P0 = (size_t)d * nc;
        std::vector<double> R(nc), direct(nc), ringv(ring, NAN), far(std::max(1, sp.far_slots), NAN), lvl(nc);
        for (int i = 0; i < nc; i++) R[i] = U(rng);
        // direct sweep: the upwind neighbours taken from the mesh (same
        // faces and order as the plan), corrections kept by position
        std::vector<int> posof(nc);
        for (int pos = 0; pos < nc; pos++) posof[sp.cell[P0 + pos]] = pos;
        for (int l = 0; l < nl; l++)
            for (int pos = lp[l]; pos < lp[l + 1]; pos++) {
                const size_t P = P0 + pos;
                const int c = sp.cell[P];
                double sum = 0;
                int j = 0, jj = 0;
                const unsigned lm = sch.lag.empty() ? 0u : sch.lag[P0 + c];
                for (int k = fm.cf_ptr[c]; k < fm.cf_ptr[c + 1]; k++, j++) {
                    const double dpn = ang.sx[d] * fm.cf_nx[k] + ang.sy[d] * fm.cf_ny[k] + ang.sz[d] * fm.cf_nz[k];
                    if (dpn >= 0 || fm.cf_bound[k] >= 0 || ((lm >> j) & 1u)) continue;
                    sum += sp.a[4 * P + jj] * direct[posof[fm.cf_nbr[k]]];
                    jj++;
                }
                direct[pos] = (R[pos] - kb * sum) / (1.0 + kb * sp.sig[P]);
            }
        // plan sweep, level-parallel: all reads of a level, then its writes
        for (int l = 0; l < nl; l++) {
            const int c0 = lp[l], c1 = lp[l + 1], lo = c1 - ring;
            for (int pos = c0; pos < c1; pos++) {
                const size_t P = P0 + pos;
                double sum = 0;
                for (int j = 0; j < sp.nin[P]; j++) {
                    const int q = sp.np[4 * P + j];
                    double v;
                    if (q >= lo)
                        v = ringv[q & mask];
                    else if (q < 0)
                        v = far[-1 - q];
                    else {
                        bad = true;  // a far reference without a slot
                        v = NAN;
                    }
                    sum += sp.a[4 * P + j] * v;
                }
                lvl[pos] = (R[pos] - kb * sum) / (1.0 + kb * sp.sig[P]);
            }
            for (int pos = c0; pos < c1; pos++) {
                ringv[pos & mask] = lvl[pos];
                const int fw = sp.far_w[P0 + pos];
                if (fw >= 0) far[fw] = lvl[pos];
            }
        }
        for (int pos = 0; pos < nc; pos++) {
            const double df = std::fabs(lvl[pos] - direct[pos]);
            if (!(df <= maxdiff)) maxdiff = std::isnan(df) ? INFINITY : df;
        }
    }
    std::printf("far_refs %lld far_slots %d ring %d max_abs_diff %.3e\n", sp.far_refs, sp.far_slots, ring, maxdiff);
    return (bad || maxdiff != 0.0) ? 1 : 0;
}
