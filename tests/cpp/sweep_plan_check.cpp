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
// With a fifth argument "morton" the cells are first renumbered by the
// library's locality order; the check then also requires that order to be a
// permutation inside each copy, and the renumbered mesh to keep the volume,
// faces and boundary sides of the original. It prints the median index gap
// between face neighbours before and after ("gap_before", "gap_after").
// Prints "far_refs <n> far_slots <n> ring <n> max_abs_diff <x>" and exits 1
// if the sweeps differ or a far reference found neither ring nor slot.
#include <cmath>
#include <cstdio>
#include <algorithm>
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
    // median index gap between interior face neighbours
    auto gap = [](const gbte::FlatMesh &m) {
        std::vector<int> g;
        for (int c = 0; c < m.nc; c++)
            for (int k = m.cf_ptr[c]; k < m.cf_ptr[c + 1]; k++)
                if (m.cf_nbr[k] >= 0) g.push_back(std::abs(m.cf_nbr[k] - c));
        if (g.empty()) return 0;
        std::nth_element(g.begin(), g.begin() + g.size() / 2, g.end());
        return g[g.size() / 2];
    };
    gbte::FlatMesh fm;
    if (argc > 5 && std::string(argv[5]) == "morton") {
        gbte::FlatMesh f0;
        e = gbte::build_flat_mesh(raw, bcs, deck.bands, f0);
        if (e.code) return std::fprintf(stderr, "mesh: %s\n", e.msg.c_str()), 2;
        std::vector<int> perm;
        gbte::locality_order(raw, perm);
        const std::vector<int> cp = raw.comp_ptr.empty() ? std::vector<int>{0, raw.nc()} : raw.comp_ptr;
        std::vector<char> seen(raw.nc(), 0);
        for (size_t q = 0; q + 1 < cp.size(); q++)
            for (int k = cp[q]; k < cp[q + 1]; k++) {
                const int c = perm[k];
                if (c < cp[q] || c >= cp[q + 1] || seen[c]) return std::fprintf(stderr, "not a permutation\n"), 1;
                seen[c] = 1;
            }
        gbte::reorder_cells(raw, perm);
        e = gbte::build_flat_mesh(raw, bcs, deck.bands, fm);
        if (e.code) return std::fprintf(stderr, "mesh: %s\n", e.msg.c_str()), 2;
        double v0 = 0, v1 = 0, dv = 0;
        for (int k = 0; k < fm.nc; k++) {
            v0 += f0.vol[perm[k]];
            v1 += fm.vol[k];
            dv = std::max(dv, std::fabs(fm.vol[k] - f0.vol[perm[k]]));
        }
        if (fm.nf() != f0.nf() || fm.nbd() != f0.nbd() || dv > 1e-12 * std::fabs(v0) / fm.nc ||
            std::fabs(v1 - v0) > 1e-12 * std::fabs(v0))
            return std::fprintf(stderr, "renumbered mesh differs\n"), 1;
        for (int b = 0; b < fm.nbd(); b++) {
            const int s0 = f0.bs_cell[2 * b] >= 0 ? perm[fm.bs_cell[2 * b]] : -1;
            const int s1 = f0.bs_cell[2 * b + 1] >= 0 ? perm[fm.bs_cell[2 * b + 1]] : -1;
            const bool same = (s0 == f0.bs_cell[2 * b] && s1 == f0.bs_cell[2 * b + 1]) ||
                              (s0 == f0.bs_cell[2 * b + 1] && s1 == f0.bs_cell[2 * b]);
            if (f0.b_type[b] != fm.b_type[b] || !same) return std::fprintf(stderr, "boundary sides differ\n"), 1;
        }
        std::printf("gap_before %d gap_after %d ", gap(f0), gap(fm));
    } else {
        e = gbte::build_flat_mesh(raw, bcs, deck.bands, fm);
        if (e.code) return std::fprintf(stderr, "mesh: %s\n", e.msg.c_str()), 2;
    }
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
