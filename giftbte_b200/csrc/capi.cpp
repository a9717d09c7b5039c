// C ABI of the B200 solver (include/giftbte.h). Converts the plain-pointer
// views into host structures, builds the flat mesh and the device solver,
// and maps every failure to a status code plus a per-handle message; nothing
// here exits the process or lets an exception cross the boundary.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <memory>
#include <new>
#include <string>
#include <thread>

#include "../../include/giftbte.h"
#include "gbte_internal.h"
#include "solver.cuh"

struct gbte_handle {
    gbte::Solver solver;
    gbte::FlatMesh *mesh() { return &solver.mesh; }
    std::string err;
    double setup_ms = 0;
    // cell order: internal cell k is the caller's cell perm[k]; empty = same order
    std::vector<int> perm;
    std::vector<int> bc_tags;  // tags of the boundary table's rows, in its order
    // caller's array of nc rows of w values -> internal order
    std::vector<double> to_internal(const double *user, int w) const {
        const size_t nc = perm.size();
        std::vector<double> v(nc * w);
        for (size_t k = 0; k < nc; k++)
            for (int j = 0; j < w; j++) v[k * w + j] = user[(size_t)perm[k] * w + j];
        return v;
    }
    // internal array of nc rows of w values -> caller's order, in place
    void to_user(double *a, int w) const {
        double *cols[1] = {a};
        gbte::scatter_rows(perm, cols, 1, w);
    }
};

namespace {

thread_local std::string g_create_error;

int fail(gbte_handle *h, const gbte::Error &e) {
    if (h) h->err = e.msg;
    g_create_error = e.msg;
    return e.code;
}

int status_of(int code) {
    switch (code) {
    case 0: return GBTE_OK;
    case 1: return GBTE_ERR_NOT_CONVERGED;
    case -1: return GBTE_ERR_ARG;
    case -2: return GBTE_ERR_IO;
    case -3: return GBTE_ERR_CUDA;
    case -4: return GBTE_ERR_DIVERGED;
    case -5: return GBTE_ERR_TIMEOUT;
    case -6: return GBTE_ERR_NOMEM;
    case -7: return GBTE_ERR_MESH;
    case -8: return GBTE_ERR_UNSUPPORTED;
    case -9: return GBTE_ERR_EXCHANGE;
    default: return GBTE_ERR_ARG;
    }
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// kappa_bulk / capacity_bulk and the band-table checks of BTEBand.cpp:791-819
int finish_bands(gbte::Bands &bands) {
    bands.kappa.assign(bands.nmat, 0.0);
    bands.capb.assign(bands.nmat, 0.0);
    for (int m = 0; m < bands.nmat; m++) {  // BTEBand.cpp:791-819
        double sl = 0, sh = 0;
        for (int b = 0; b < bands.nb; b++) {
            int i = m * bands.nb + b;
            double k = bands.C[i] * bands.v[i] * bands.v[i] * bands.tau[i];
            bands.kappa[m] += (bands.material_dim == 2) ? k / 2 : k / 3;
            bands.capb[m] += bands.C[i];
            sl += bands.lat[i];
            sh += bands.hr[i];
        }
        if (std::isnan(bands.kappa[m])) return fail(nullptr, {-1, "mistake in phonon properties, nan"}), GBTE_ERR_ARG;
        if (std::fabs(sl - 1.0) > 1e-6)
            return fail(nullptr, {-1, "lattice ratios of a material do not sum to 1"}), GBTE_ERR_ARG;
        for (int b = 0; b < bands.nb; b++)
            if (!(bands.C[m * bands.nb + b] > 0) || !(bands.v[m * bands.nb + b] > 0) || !(bands.tau[m * bands.nb + b] > 0))
                return fail(nullptr, {-1, "band heat capacity, group velocity and relaxation time must be positive"}),
                       GBTE_ERR_ARG;
    }
    return GBTE_OK;
}

// Cells are renumbered inside the library along a Morton curve of their
// centres (per geometry of a batch) unless options.cell_order = 1: upwind and
// stencil neighbours then sit close in memory, so the gathers of the sweep,
// the gradient and the residual hit fewer distinct lines. Every cell array of
// the ABI is mapped back to the caller's order.
int create_common(const gbte::RawMesh &raw_in, const gbte::Bands &bands_in, const gbte::BCs &bcs, const gbte_angle_spec &as,
                  const gbte_options &opt, const std::vector<double> &cell_heat, gbte_handle **out) {
    double t0 = now_ms();
    std::unique_ptr<gbte_handle> h(new (std::nothrow) gbte_handle());
    if (!h) {
        g_create_error = "host allocation failed";
        return GBTE_ERR_NOMEM;
    }
    gbte::Bands bands = bands_in;
    int brc = finish_bands(bands);
    if (brc != GBTE_OK) return brc;
    gbte::Angles ang;
    gbte::Error e = as.method == 0 ? gbte::explicit_angles(as.num_directions, as.direction_xyz, as.weight,
                                                           as.solid_angle, ang)
                                   : gbte::make_angles(as.method, as.n_theta, as.n_phi, bands.material_dim, ang);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    if (opt.cell_order != 0 && opt.cell_order != 1)
        return fail(nullptr, {-1, "cell_order must be 0 (automatic) or 1 (caller's order)"}), GBTE_ERR_ARG;
    std::vector<double> scatter;
    if (opt.cell_scatter) scatter.assign(opt.cell_scatter, opt.cell_scatter + raw_in.nc());
    const gbte::RawMesh *rp = &raw_in;
    gbte::RawMesh reordered;
    std::vector<double> heat = cell_heat;
    if (opt.cell_order == 0) {
        gbte::locality_order(raw_in, h->perm);
        reordered = raw_in;
        gbte::reorder_cells(reordered, h->perm);
        rp = &reordered;
        if (!heat.empty()) heat = h->to_internal(cell_heat.data(), 1);
        if (!scatter.empty()) scatter = h->to_internal(scatter.data(), 1);
    }
    const gbte::RawMesh &raw = *rp;
    gbte::FlatMesh fm;
    e = gbte::build_flat_mesh(raw, bcs, bands, fm);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    gbte::SolverConfig cfg;
    cfg.precision = opt.precision;
    cfg.use_limiter = opt.use_limiter;
    cfg.max_iter = opt.max_iter;
    cfg.err_temp = opt.err_temp;
    cfg.err_flux = opt.err_flux;
    cfg.macro_rtol = opt.macro_rtol > 0 ? opt.macro_rtol : 1e-13;
    cfg.verbose = opt.verbose;
    cfg.profile = opt.profile;
    cfg.sweep_bands = opt.sweep_bands;
    cfg.sweep_far_slots = opt.sweep_far_slots;
    cfg.direction_batch = opt.direction_batch;
    cfg.cell_scatter = scatter;
    if (opt.order != 0 && opt.order != 1 && opt.order != 2)
        return fail(nullptr, {-1, "order must be 1 or 2 (0 = 2)"}), GBTE_ERR_ARG;
    if (opt.scheme != 0 && opt.scheme != 1)
        return fail(nullptr, {-1, "scheme must be 0 (Synthetic) or 1 (Sequential)"}), GBTE_ERR_ARG;
    cfg.order = opt.order == 1 ? 1 : 2;
    cfg.sequential = opt.scheme == 1;
    cfg.macro_exact = opt.macro_exact != 0;
    if (opt.sweep_vector != 0 && opt.sweep_vector != 1 && opt.sweep_vector != 2 && opt.sweep_vector != 4)
        return fail(nullptr, {-1, "sweep_vector must be 0 (automatic), 1, 2 or 4"}), GBTE_ERR_ARG;
    cfg.sweep_vector = opt.sweep_vector;
    if (opt.sweep_kernel < 0 || opt.sweep_kernel > 3)
        return fail(nullptr, {-1, "sweep_kernel must be 0 (automatic), 1 (block), 2 (warp) or 3 (wide)"}),
               GBTE_ERR_ARG;
    cfg.sweep_kernel = opt.sweep_kernel;
    if (opt.gradient_dirs < 0 || opt.gradient_dirs > 10 || opt.gradient_dirs == 3)
        return fail(nullptr, {-1, "gradient_dirs must be 0 (automatic), 1, 2, 4, 5, 6, 7, 8, 9 or 10"}), GBTE_ERR_ARG;
    cfg.gradient_dirs = opt.gradient_dirs;
    if (opt.residual_form != 0 && opt.residual_form != 1 && (opt.residual_form < 5 || opt.residual_form > 8))
        return fail(nullptr, {-1, "residual_form must be 0 (automatic), 1, 5, 6, 7 or 8"}), GBTE_ERR_ARG;
    cfg.residual_form = opt.residual_form;
    if (opt.adjoint_history < -1 || opt.adjoint_history > 8)
        return fail(nullptr, {-1, "adjoint_history must be -1 (plain), 0 (default) or 1..8"}), GBTE_ERR_ARG;
    cfg.adjoint_anderson = opt.adjoint_history == 0 ? 6 : opt.adjoint_history < 0 ? 0 : opt.adjoint_history;
    cfg.device = opt.device;
    cfg.stream = (cudaStream_t)opt.stream;
    if (opt.precision != GBTE_FP64 && opt.precision != GBTE_FP32_MIXED)
        return fail(nullptr, {-1, "precision must be GBTE_FP64 or GBTE_FP32_MIXED"}), GBTE_ERR_ARG;
    e = h->solver.init(fm, bands, ang, heat, cfg);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    h->bc_tags = bcs.tag;
    h->setup_ms = now_ms() - t0;
    *out = h.release();
    return GBTE_OK;
}

}  // namespace

extern "C" {

size_t gbte_options_size(void) { return sizeof(gbte_options); }

void gbte_default_options(gbte_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = GBTE_FP64;
    o->max_iter = 10000;
    o->err_temp = 1e-6;
    o->err_flux = 1e-4;
    o->macro_rtol = 1e-13;
}

static int convert_views(const gbte_mesh_view *mv, const gbte_band_table *bt, const gbte_bc_table *bc,
                         gbte::RawMesh &raw, gbte::Bands &B, gbte::BCs &bcs) {
    if (mv->num_nodes <= 0 || mv->num_cells <= 0 || !mv->node_xyz || !mv->cell_ptr || !mv->cell_verts ||
        !mv->cell_region || (mv->num_boundary_elements > 0 && (!mv->belem_ptr || !mv->belem_verts || !mv->belem_tag)))
        return fail(nullptr, {-1, "incomplete mesh view"}), GBTE_ERR_ARG;
    if (bt->num_materials <= 0 || bt->num_bands <= 0 || !bt->group_velocity || !bt->relaxation_time ||
        !bt->heat_capacity || !bt->lattice_ratio || !bt->heat_ratio || bt->num_regions <= 0 || !bt->region_material)
        return fail(nullptr, {-1, "incomplete band table"}), GBTE_ERR_ARG;
    if (bc->num < 0 || (bc->num > 0 && (!bc->tag || !bc->type || !bc->value)))
        return fail(nullptr, {-1, "incomplete BC table"}), GBTE_ERR_ARG;
    raw.dim = mv->dimension;
    raw.xyz.assign(mv->node_xyz, mv->node_xyz + 3 * (size_t)mv->num_nodes);
    raw.cptr.assign(mv->cell_ptr, mv->cell_ptr + mv->num_cells + 1);
    if (raw.cptr[0] != 0) return fail(nullptr, {-1, "cell_ptr must start at 0"}), GBTE_ERR_ARG;
    for (int i = 0; i < mv->num_cells; i++)
        if (raw.cptr[i + 1] < raw.cptr[i]) return fail(nullptr, {-1, "cell_ptr must be non-decreasing"}), GBTE_ERR_ARG;
    raw.cverts.assign(mv->cell_verts, mv->cell_verts + raw.cptr.back());
    raw.creg.assign(mv->cell_region, mv->cell_region + mv->num_cells);
    raw.bptr.assign(1, 0);
    if (mv->num_boundary_elements > 0) {
        raw.bptr.assign(mv->belem_ptr, mv->belem_ptr + mv->num_boundary_elements + 1);
        if (raw.bptr[0] != 0) return fail(nullptr, {-1, "belem_ptr must start at 0"}), GBTE_ERR_ARG;
        for (int i = 0; i < mv->num_boundary_elements; i++)
            if (raw.bptr[i + 1] < raw.bptr[i]) return fail(nullptr, {-1, "belem_ptr must be non-decreasing"}), GBTE_ERR_ARG;
        raw.bverts.assign(mv->belem_verts, mv->belem_verts + raw.bptr.back());
        raw.btag.assign(mv->belem_tag, mv->belem_tag + mv->num_boundary_elements);
    }
    raw.Lx = mv->scale_x > 0 ? mv->scale_x : 1.0;
    raw.Ly = mv->scale_y;
    raw.Lz = mv->scale_z;
    B.nmat = bt->num_materials;
    B.nb = bt->num_bands;
    B.material_dim = bt->material_dimension;
    size_t n = (size_t)B.nmat * B.nb;
    B.v.assign(bt->group_velocity, bt->group_velocity + n);
    B.tau.assign(bt->relaxation_time, bt->relaxation_time + n);
    B.C.assign(bt->heat_capacity, bt->heat_capacity + n);
    B.lat.assign(bt->lattice_ratio, bt->lattice_ratio + n);
    B.hr.assign(bt->heat_ratio, bt->heat_ratio + n);
    B.region_material.assign(bt->region_material, bt->region_material + bt->num_regions);
    for (int r : B.region_material)
        if (r < 0 || r >= B.nmat) return fail(nullptr, {-1, "region_material out of range"}), GBTE_ERR_ARG;
    bool any5 = false;
    for (int i = 0; i < bc->num; i++) {
        bcs.tag.push_back(bc->tag[i]);
        bcs.type.push_back(bc->type[i]);
        bcs.value.push_back(bc->value[i]);
        if (bc->type[i] == 4)
            return fail(nullptr, {-8, "BC type 4 has no steady-state branch in the reference solver"}), GBTE_ERR_UNSUPPORTED;
        any5 = any5 || bc->type[i] == 5;
    }
    if (any5) {
        if (!bc->transmissivity)
            return fail(nullptr, {-1, "a type-5 interface row needs the transmissivity table"}), GBTE_ERR_ARG;
        bcs.trans.assign(bc->transmissivity, bc->transmissivity + (size_t)bc->num * B.nmat * B.nb);
    }
    return GBTE_OK;
}

// host-only build of everything gbte_create would put on the device
static int inspect_common(const gbte::RawMesh &raw_in, const gbte::Bands &bands_in, const gbte::BCs &bcs,
                          const gbte_angle_spec &as, gbte_deck_info *info) {
    gbte::Bands bands = bands_in;
    int brc = finish_bands(bands);
    if (brc != GBTE_OK) return brc;
    gbte::Angles ang;
    gbte::Error e = as.method == 0 ? gbte::explicit_angles(as.num_directions, as.direction_xyz, as.weight,
                                                           as.solid_angle, ang)
                                   : gbte::make_angles(as.method, as.n_theta, as.n_phi, bands.material_dim, ang);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    // the cell order gbte_create uses by default
    std::vector<int> perm;
    gbte::locality_order(raw_in, perm);
    gbte::RawMesh raw = raw_in;
    gbte::reorder_cells(raw, perm);
    gbte::FlatMesh fm;
    e = gbte::build_flat_mesh(raw, bcs, bands, fm);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    gbte::Schedule sch;
    gbte::build_schedule(fm, ang, sch, (int)std::max(1u, std::thread::hardware_concurrency()));
    std::memset(info, 0, sizeof(*info));
    info->dimension = fm.dim;
    info->num_nodes = fm.nn;
    info->num_cells = fm.nc;
    info->num_faces = fm.nf();
    info->num_boundaries = fm.nbd();
    info->num_boundary_sides = fm.nbs();
    info->num_bands = bands.nb;
    info->num_directions = ang.nd;
    info->num_materials = bands.nmat;
    info->max_levels = sch.max_levels;
    info->lagged_faces = sch.lagged_faces;
    info->kappa_bulk = bands.kappa[0];
    info->capacity_bulk = bands.capb[0];
    for (double v : fm.vol) info->total_volume += v;
    gbte::SweepPlan sp;
    e = gbte::build_sweep_plan(fm, ang, sch, gbte::kSweepMinRing, gbte::kSweepFarCap, sp);
    if (e.code) return fail(nullptr, e), status_of(e.code);
    info->max_level_width = sp.max_width;
    info->sweep_ring = sp.ring;
    info->far_slots = sp.far_slots;
    info->far_refs = sp.far_refs;
    if (gbte::index_checks_enabled()) {
        e = gbte::check_indices(fm, bands.nb, sch, ang.nd, sp, info->index_entries_checked);
        if (e.code) return fail(nullptr, e), status_of(e.code);
        // the tiles the solver would build for the shared-memory gradient
        // and residual forms
        for (int B : {fm.dim == 3 ? 32 : 64, fm.dim == 3 ? 64 : 128}) {
            gbte::GradTiles gt;
            gbte::FaceTiles ft;
            long long n = 0;
            if (gbte::build_grad_tiles(fm, B, gt).code == 0) {
                e = gbte::check_tiles(fm, &gt, nullptr, n);
                if (e.code) return fail(nullptr, e), status_of(e.code);
                info->index_entries_checked += n;
            }
            if (gbte::build_face_tiles(fm, B, ft).code == 0) {
                e = gbte::check_tiles(fm, nullptr, &ft, n);
                if (e.code) return fail(nullptr, e), status_of(e.code);
                info->index_entries_checked += n;
            }
        }
    }
    return GBTE_OK;
}

int gbte_inspect_mesh(const gbte_mesh_view *mv, const gbte_band_table *bt, const gbte_bc_table *bc,
                      const gbte_angle_spec *as, gbte_deck_info *info) {
    try {
        if (!mv || !bt || !bc || !as || !info) return fail(nullptr, {-1, "null argument"}), GBTE_ERR_ARG;
        gbte::RawMesh raw;
        gbte::Bands B;
        gbte::BCs bcs;
        int rc = convert_views(mv, bt, bc, raw, B, bcs);
        if (rc != GBTE_OK) return rc;
        return inspect_common(raw, B, bcs, *as, info);
    } catch (const std::exception &ex) {
        g_create_error = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_inspect_deck(const char *dir, gbte_deck_info *info) {
    try {
        if (!dir || !info) return fail(nullptr, {-1, "null argument"}), GBTE_ERR_ARG;
        gbte::Deck deck;
        gbte::Error e = gbte::read_deck(dir, deck);
        if (e.code) return fail(nullptr, e), status_of(e.code);
        gbte_angle_spec as{deck.angle_method, deck.n_theta, deck.n_phi};
        int rc = inspect_common(deck.mesh, deck.bands, deck.bcs, as, info);
        if (rc == GBTE_OK) {
            info->max_iter_or_zero = deck.max_iter;
            info->err_temp = deck.err_temp;
            info->err_flux = deck.err_flux;
            info->transient = deck.transient ? 1 : 0;
            info->time_step = deck.time_step;
            info->total_time = deck.total_time;
        }
        return rc;
    } catch (const std::exception &ex) {
        g_create_error = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_create(const gbte_mesh_view *mv, const gbte_band_table *bt, const gbte_bc_table *bc, const gbte_angle_spec *as,
                const gbte_options *opt, gbte_handle **out) {
    try {
        if (!mv || !bt || !bc || !as || !opt || !out) return fail(nullptr, {-1, "null argument"}), GBTE_ERR_ARG;
        *out = nullptr;
        gbte::RawMesh raw;
        gbte::Bands B;
        gbte::BCs bcs;
        int rc = convert_views(mv, bt, bc, raw, B, bcs);
        if (rc != GBTE_OK) return rc;
        std::vector<double> heat;
        if (opt->cell_heat) heat.assign(opt->cell_heat, opt->cell_heat + mv->num_cells);
        return create_common(raw, B, bcs, *as, *opt, heat, out);
    } catch (const std::bad_alloc &) {
        g_create_error = "host allocation failed";
        return GBTE_ERR_NOMEM;
    } catch (const std::exception &ex) {
        g_create_error = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_batch_create(int num, const gbte_mesh_view *meshes, const gbte_band_table *bt, const gbte_bc_table *bcs,
                      const gbte_angle_spec *as, const gbte_options *opt, gbte_handle **out) {
    try {
        if (num <= 0 || !meshes || !bt || !bcs || !as || !opt || !out)
            return fail(nullptr, {-1, "null argument or empty batch"}), GBTE_ERR_ARG;
        *out = nullptr;
        std::vector<gbte::RawMesh> raws(num);
        std::vector<gbte::BCs> tables(num);
        gbte::Bands B;
        long long total = 0;
        for (int k = 0; k < num; k++) {
            gbte::Bands Bk;
            int rc = convert_views(&meshes[k], bt, &bcs[k], raws[k], Bk, tables[k]);
            if (rc != GBTE_OK) return rc;
            if (k == 0) B = Bk;
            total += meshes[k].num_cells;
        }
        gbte::RawMesh raw;
        gbte::BCs all;
        gbte::Error e = gbte::make_union(raws, tables, raw, all);
        if (e.code) return fail(nullptr, e), status_of(e.code);
        std::vector<double> heat;
        if (opt->cell_heat) heat.assign(opt->cell_heat, opt->cell_heat + total);
        return create_common(raw, B, all, *as, *opt, heat, out);
    } catch (const std::bad_alloc &) {
        g_create_error = "host allocation failed";
        return GBTE_ERR_NOMEM;
    } catch (const std::exception &ex) {
        g_create_error = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_batch_geometries(gbte_handle *h, int *num, int *cell_offsets) {
    if (!h) return GBTE_ERR_ARG;
    const std::vector<int> &cp = h->solver.mesh.comp_ptr;
    const int n = cp.empty() ? 1 : (int)cp.size() - 1;
    if (num) *num = n;
    if (cell_offsets) {
        if (cp.empty()) {
            cell_offsets[0] = 0;
            cell_offsets[1] = h->solver.mesh.nc;
        } else {
            for (int k = 0; k <= n; k++) cell_offsets[k] = cp[k];
        }
    }
    return GBTE_OK;
}

int gbte_create_from_deck(const char *dir, const gbte_options *opt_in, gbte_handle **out) {
    try {
        if (!dir || !out) return fail(nullptr, {-1, "null argument"}), GBTE_ERR_ARG;
        *out = nullptr;
        gbte_options opt;
        if (opt_in)
            opt = *opt_in;
        else
            gbte_default_options(&opt);
        gbte::Deck deck;
        gbte::Error e = gbte::read_deck(dir, deck);
        if (e.code) return fail(nullptr, e), status_of(e.code);
        if (deck.order == "2limit")
            opt.use_limiter = 1;
        else if (deck.order == "1")
            opt.order = 1;
        else if (deck.order == "2")
            opt.order = 2;
        else
            return fail(nullptr, {-8, "Order must be 1, 2 or 2limit"}), GBTE_ERR_UNSUPPORTED;
        if (deck.method == "Sequential")
            opt.scheme = 1;
        else if (deck.method != "Synthetic")
            return fail(nullptr, {-8, "IterativeScheme must be Synthetic or Sequential"}), GBTE_ERR_UNSUPPORTED;
        opt.max_iter = deck.max_iter;
        opt.err_temp = deck.err_temp;
        opt.err_flux = deck.err_flux;
        gbte_angle_spec as{deck.angle_method, deck.n_theta, deck.n_phi};
        int rc = create_common(deck.mesh, deck.bands, deck.bcs, as, opt, deck.cell_heat, out);
        if (rc == GBTE_OK) {
            // Tref as the initial temperature; gbte_fourier_initial / gbte_set_initial may replace it
            std::vector<double> T0(deck.mesh.nc(), deck.tref);
            gbte::Error e2 = (*out)->solver.set_initial(T0.data(), nullptr, nullptr);
            if (e2.code) {
                delete *out;
                *out = nullptr;
                return fail(nullptr, e2), status_of(e2.code);
            }
        }
        return rc;
    } catch (const std::bad_alloc &) {
        g_create_error = "host allocation failed";
        return GBTE_ERR_NOMEM;
    } catch (const std::exception &ex) {
        g_create_error = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_set_initial(gbte_handle *h, const double *T0, const double *q0, const double *bth) {
    if (!h) return GBTE_ERR_ARG;
    try {
        gbte::Error e;
        if (h->perm.empty() || !T0) {
            e = h->solver.set_initial(T0, q0, bth);
        } else {
            std::vector<double> T = h->to_internal(T0, 1), q;
            if (q0) q = h->to_internal(q0, 3);
            e = h->solver.set_initial(T.data(), q0 ? q.data() : nullptr, bth);
        }
        if (e.code) return fail(h, e), status_of(e.code);
        return GBTE_OK;
    } catch (const std::exception &ex) {
        h->err = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_fourier_initial(gbte_handle *h) {
    if (!h) return GBTE_ERR_ARG;
    gbte::Error e = h->solver.fourier_initial();
    if (e.code) return fail(h, e), status_of(e.code);
    return GBTE_OK;
}

int gbte_fourier_initial_noalloc(gbte_handle *h) {
    if (!h) return GBTE_ERR_ARG;
    gbte::Error e = h->solver.fourier_initial_noalloc();
    if (e.code) return fail(h, e), status_of(e.code);
    return GBTE_OK;
}

int gbte_solve(gbte_handle *h, gbte_stats *st) {
    if (!h) return GBTE_ERR_ARG;
    try {
        gbte::SolveStats s;
        gbte::Error e = h->solver.solve(s);
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->iterations = s.iterations;
            st->err_temp = s.err_temp;
            st->err_flux = s.err_flux;
            st->solve_ms = s.solve_ms;
            st->setup_ms = h->setup_ms;
            st->transport_ms = s.transport_ms;
            st->macro_ms = s.macro_ms;
            st->macro_cg_iterations = s.cg_iterations;
            st->updates = s.updates;
            st->num_directions = h->solver.ang.nd;
            st->num_bands = h->solver.bands.nb;
            st->num_cells = h->solver.mesh.nc;
            st->max_levels = h->solver.sched.max_levels;
            st->lagged_faces = h->solver.sched.lagged_faces;
            st->inner_iterations = s.inner_iterations;
            st->kernel_launches = s.launches;
            const int fixed = h->solver.cfg.sweep_bands;
            st->sweep_bands = (fixed >= 1 && fixed <= 32) ? fixed : h->solver.tuned_sweep_bands_;
            st->direction_batch = h->solver.ndb_;
            st->sweep_stage_levels = h->solver.tuned_sweep_look_;
            st->sweep_vector = h->solver.last_sweep_vb_;
            st->sweep_threads = h->solver.last_sweep_threads_;
            st->sweep_kernel = h->solver.last_sweep_warp_ == 1 ? 2 : h->solver.last_sweep_warp_ == 2 ? 3 : 1;
            st->gradient_dirs = h->solver.last_grad_dirs_;
            st->residual_form = h->solver.last_res_form_;
            for (int k = 0; k < GBTE_NUM_KERNELS && k < gbte::K_NUM; k++) {
                st->kernel_ms[k] = s.kernel_ms[k];
                st->kernel_count[k] = s.kernel_count[k];
            }
        }
        if (e.code) {
            if (e.code > 0) {
                h->err = e.msg;
                return status_of(e.code);
            }
            return fail(h, e), status_of(e.code);
        }
        return GBTE_OK;
    } catch (const std::exception &ex) {
        h->err = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_solve_with(gbte_handle *h, int max_iter, double err_temp, double err_flux, gbte_stats *st) {
    if (!h) return GBTE_ERR_ARG;
    if (max_iter < 0 || !(err_temp >= 0) || !(err_flux >= 0)) return fail(h, {-1, "invalid solve limits"}), GBTE_ERR_ARG;
    gbte::SolverConfig saved = h->solver.cfg;
    h->solver.cfg.max_iter = max_iter;
    h->solver.cfg.err_temp = err_temp;
    h->solver.cfg.err_flux = err_flux;
    int rc = gbte_solve(h, st);
    h->solver.cfg.max_iter = saved.max_iter;
    h->solver.cfg.err_temp = saved.err_temp;
    h->solver.cfg.err_flux = saved.err_flux;
    return rc;
}

int gbte_get_fields(gbte_handle *h, double *TE, double *TL, double *q, double *TB) {
    if (!h) return GBTE_ERR_ARG;
    gbte::Error e = h->solver.get_fields(TE, TL, q, TB);
    if (e.code) return fail(h, e), status_of(e.code);
    if (!h->perm.empty()) {
        // the one-value columns (E, T and each band's temperature) together
        const size_t nc = h->perm.size();
        std::vector<double *> cols;
        if (TE) cols.push_back(TE);
        if (TL) cols.push_back(TL);
        if (TB)
            for (int b = 0; b < h->solver.bands.nb; b++) cols.push_back(TB + (size_t)b * nc);
        gbte::scatter_rows(h->perm, cols.data(), (int)cols.size(), 1);
        if (q) h->to_user(q, 3);
    }
    return GBTE_OK;
}

int gbte_get_sizes(gbte_handle *h, int *nc, int *nb, int *nd, int *nbs) {
    if (!h) return GBTE_ERR_ARG;
    if (nc) *nc = h->solver.mesh.nc;
    if (nb) *nb = h->solver.bands.nb;
    if (nd) *nd = h->solver.ang.nd;
    if (nbs) *nbs = h->solver.mesh.nbs();
    return GBTE_OK;
}

int gbte_get_geometry(gbte_handle *h, double *centers, double *volumes) {
    if (!h) return GBTE_ERR_ARG;
    const gbte::FlatMesh &m = h->solver.mesh;
    for (int k = 0; k < m.nc; k++) {
        const int c = h->perm.empty() ? k : h->perm[k];
        if (centers) {
            centers[3 * c] = m.cx[k];
            centers[3 * c + 1] = m.cy[k];
            centers[3 * c + 2] = m.cz[k];
        }
        if (volumes) volumes[c] = m.vol[k];
    }
    return GBTE_OK;
}

int gbte_write_outputs(gbte_handle *h, const char *dir) {
    if (!h || !dir) return GBTE_ERR_ARG;
    const gbte::FlatMesh &m = h->solver.mesh;
    const int nc = m.nc, nb = h->solver.bands.nb;
    std::vector<double> TE(nc), TL(nc), q(3 * (size_t)nc), TB((size_t)nb * nc);
    int rc = gbte_get_fields(h, TE.data(), TL.data(), q.data(), TB.data());
    if (rc != GBTE_OK) return rc;
    // files list cells in the caller's order: row i is internal cell at[i]
    std::vector<int> at(nc);
    for (int k = 0; k < nc; k++) at[h->perm.empty() ? k : h->perm[k]] = k;
    std::vector<double> cx(nc), cy(nc), cz(nc);
    for (int i = 0; i < nc; i++) {
        cx[i] = m.cx[at[i]];
        cy[i] = m.cy[at[i]];
        cz[i] = m.cz[at[i]];
    }
    std::string d(dir);
    auto open = [&](const char *name, std::ofstream &f) {
        f.open(d + "/" + name);
        f << std::setprecision(17);
        return f.is_open();
    };
    std::ofstream f;
    // TempLattice.dat / Tempband.dat / Temperature.dat / HeatFlux.dat (StaticBTESynthetic.cpp:2613-2653)
    if (!open("TempLattice.dat", f)) return fail(h, {-2, "cannot write TempLattice.dat"}), GBTE_ERR_IO;
    for (int i = 0; i < nc; i++) f << cx[i] << " " << cy[i] << " " << cz[i] << " " << TL[i] << "\n";
    f.close();
    if (!open("Tempband.dat", f)) return fail(h, {-2, "cannot write Tempband.dat"}), GBTE_ERR_IO;
    for (int j = 0; j < nb; j++)
        for (int i = 0; i < nc; i++)
            f << j + 1 << " " << cx[i] << " " << cy[i] << " " << cz[i] << " " << TB[(size_t)j * nc + i] << "\n";
    f.close();
    if (!open("Temperature.dat", f)) return fail(h, {-2, "cannot write Temperature.dat"}), GBTE_ERR_IO;
    for (int i = 0; i < nc; i++) f << cx[i] << " " << cy[i] << " " << cz[i] << " " << TE[i] << "\n";
    f.close();
    if (!open("HeatFlux.dat", f)) return fail(h, {-2, "cannot write HeatFlux.dat"}), GBTE_ERR_IO;
    for (int i = 0; i < nc; i++) {
        double v[6] = {cx[i], cy[i], cz[i], q[3 * i], q[3 * i + 1], q[3 * i + 2]};
        for (double x : v) f << " " << std::setw(24) << x;
        f << "\n";
    }
    f.close();
    // Result.vtk (Solution.cpp:163-220): legacy ASCII, nodes divided by the scales
    if (!open("Result.vtk", f)) return fail(h, {-2, "cannot write Result.vtk"}), GBTE_ERR_IO;
    f << "# vtk DataFile Version 2.0\nRESULT\nASCII\nDATASET UNSTRUCTURED_GRID\n";
    f << "POINTS " << m.nn << " float\n";
    for (int i = 0; i < m.nn; i++) f << m.node_x[i] / m.Lx << " " << m.node_y[i] / m.Lx << " " << m.node_z[i] / m.Lx << "\n";
    size_t total = 0;
    for (int c = 0; c < nc; c++) total += m.cptr[c + 1] - m.cptr[c] + 1;
    f << "\nCELLS " << nc << " " << total << "\n";
    for (int i = 0; i < nc; i++) {
        const int c = at[i];
        f << m.cptr[c + 1] - m.cptr[c];
        for (int k = m.cptr[c]; k < m.cptr[c + 1]; k++) f << " " << m.cverts[k];
        f << "\n";
    }
    f << "\nCELL_TYPES " << nc << "\n";
    for (int i = 0; i < nc; i++) {
        const int c = at[i];
        int nv = m.cptr[c + 1] - m.cptr[c];
        f << (m.dim == 2 ? (nv == 4 ? 8 : 5) : 10) << "\n";
    }
    f << "\nCELL_DATA " << nc << "\nSCALARS Temperature float 1\nLOOKUP_TABLE default\n";
    for (int c = 0; c < nc; c++) f << TE[c] << "\n";
    f << "VECTORS HeatFLux float\n";
    for (int c = 0; c < nc; c++) f << q[3 * c] << " " << q[3 * c + 1] << " " << q[3 * c + 2] << "\n";
    f.close();
    return GBTE_OK;
}

int gbte_transient_solve(gbte_handle *h, double time_step, double total_time, double err_temp, double err_flux,
                         int probe_cell, double *probe_history, long long history_len, gbte_transient_stats *st) {
    if (!h) return GBTE_ERR_ARG;
    try {
        const int nc = h->solver.mesh.nc;
        if (probe_cell < 0 || probe_cell >= nc) return fail(h, {-1, "probe_cell out of range"}), GBTE_ERR_ARG;
        if (history_len < 0 || !(err_temp >= 0) || !(err_flux >= 0))
            return fail(h, {-1, "invalid transient limits"}), GBTE_ERR_ARG;
        // internal indices of the caller's cells: the probe, and the cells
        // numbered like the walls (the start's specular walls read them)
        int probe = probe_cell;
        std::vector<int> wall_cell;
        if (!h->perm.empty()) {
            std::vector<int> inv(nc);
            for (int k = 0; k < nc; k++) inv[h->perm[k]] = k;
            probe = inv[probe_cell];
            wall_cell.assign(h->solver.mesh.nbd(), -1);
            for (int ib = 0; ib < (int)wall_cell.size() && ib < nc; ib++) wall_cell[ib] = inv[ib];
        }
        gbte::TransientStats ts;
        gbte::Error e = h->solver.transient(time_step, total_time, err_temp, err_flux, probe,
                                            history_len > 0 ? probe_history : nullptr, history_len, wall_cell, ts);
        if (e.code) return fail(h, e), status_of(e.code);
        if (st) {
            st->steps = ts.steps;
            st->updates = ts.updates;
            st->err_temp = ts.err_temp;
            st->err_flux = ts.err_flux;
            st->solve_ms = ts.ms;
        }
        return GBTE_OK;
    } catch (const std::bad_alloc &) {
        h->err = "host allocation failed";
        return GBTE_ERR_NOMEM;
    } catch (const std::exception &ex) {
        h->err = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_vjp(gbte_handle *h, const double *T_bar, const double *q_bar, int max_iter, double tol, double *grad_tau,
             double *grad_scatter, double *grad_specularity, gbte_vjp_stats *st) {
    if (!h) return GBTE_ERR_ARG;
    try {
        const gbte::FlatMesh &m = h->solver.mesh;
        std::vector<double> Tb, qb, gc(grad_scatter ? m.nc : 0), gb(m.nbd());
        if (!h->perm.empty()) {
            if (T_bar) Tb = h->to_internal(T_bar, 1), T_bar = Tb.data();
            if (q_bar) qb = h->to_internal(q_bar, 3), q_bar = qb.data();
        }
        gbte::VjpStats vs;
        gbte::Error e = h->solver.vjp(T_bar, q_bar, max_iter, tol, grad_tau, grad_scatter ? gc.data() : nullptr,
                                      gb.data(), vs);
        if (e.code) return fail(h, e), status_of(e.code);
        if (grad_scatter) {
            std::memcpy(grad_scatter, gc.data(), gc.size() * sizeof(double));
            if (!h->perm.empty()) h->to_user(grad_scatter, 1);
        }
        if (grad_specularity) {
            for (size_t r = 0; r < h->bc_tags.size(); r++) grad_specularity[r] = 0;
            for (int ib = 0; ib < m.nbd(); ib++)
                for (size_t r = 0; r < h->bc_tags.size(); r++)
                    if (h->bc_tags[r] == m.b_tag[ib]) grad_specularity[r] += gb[ib];
        }
        if (st) {
            st->iterations = vs.iterations;
            st->picard_steps = vs.picard_steps;
            st->change = vs.change;
            st->vjp_ms = vs.ms;
            st->residual = vs.residual;
        }
        return GBTE_OK;
    } catch (const std::bad_alloc &) {
        h->err = "host allocation failed";
        return GBTE_ERR_NOMEM;
    } catch (const std::exception &ex) {
        h->err = ex.what();
        return GBTE_ERR_ARG;
    }
}

int gbte_set_direction_shard(gbte_handle *h, int dir_begin, int dir_count, gbte_exchange_fn exchange, void *user) {
    if (!h) return GBTE_ERR_ARG;
    gbte::Error e = h->solver.set_shard(dir_begin, dir_count, exchange, user);
    if (e.code) return fail(h, e), status_of(e.code);
    return GBTE_OK;
}

int gbte_set_profile(gbte_handle *h, int on) {
    if (!h) return GBTE_ERR_ARG;
    h->solver.cfg.profile = on ? 1 : 0;
    return GBTE_OK;
}

const char *gbte_kernel_name(int i) { return gbte::kernel_name(i); }

const char *gbte_last_error(const gbte_handle *h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

const char *gbte_status_string(int s) {
    switch (s) {
    case GBTE_OK: return "ok";
    case GBTE_ERR_ARG: return "invalid argument";
    case GBTE_ERR_IO: return "input/output error";
    case GBTE_ERR_CUDA: return "CUDA error";
    case GBTE_ERR_DIVERGED: return "diverged";
    case GBTE_ERR_TIMEOUT: return "device wait timed out";
    case GBTE_ERR_NOMEM: return "out of memory";
    case GBTE_ERR_MESH: return "mesh topology error";
    case GBTE_ERR_UNSUPPORTED: return "unsupported input";
    case GBTE_ERR_EXCHANGE: return "direction shard exchange failed";
    case GBTE_ERR_NOT_CONVERGED: return "not converged within max_iter";
    default: return "unknown status";
    }
}

int gbte_destroy(gbte_handle *h) {
    delete h;
    return GBTE_OK;
}

}  // extern "C"
