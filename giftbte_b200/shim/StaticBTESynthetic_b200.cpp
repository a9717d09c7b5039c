// The B200 drop-in StaticBTESynthetic (see StaticBTESynthetic/StaticBTESynthetic.h):
// flattens the reference's mesh, band, boundary-condition and angle objects
// into the C ABI's views once, and runs each solve variant on the device.
#include "StaticBTESynthetic/StaticBTESynthetic.h"

#include <cmath>
#include <cstdlib>
#include <iostream>

#include "giftbte.h"

namespace {

[[noreturn]] void stop(const char *what, int rc, const gbte_handle *h) {
    // the reference reports errors on cout and exits
    std::cout << "B200 solver: " << what << " failed (" << gbte_status_string(rc) << "): " << gbte_last_error(h)
              << std::endl;
    std::exit(1);
}

}  // namespace

StaticBTESynthetic::StaticBTESynthetic(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles,
                                       int num_proc, int world_rank) {
    if (gbte_options_size() != sizeof(gbte_options)) {
        std::cout << "B200 solver: libgiftbte_b200 was built from another giftbte.h (options of "
                  << gbte_options_size() << " bytes, this class expects " << sizeof(gbte_options)
                  << "); rebuild the drop-in" << std::endl;
        std::exit(1);
    }
    // the reference's constructor reads the same objects
    // (src/StaticBTESynthetic/StaticBTESynthetic.cpp:224-626)
    dimension = mesh->Dimension;
    numCell = (int)mesh->Elements.size();
    numBand = (int)bands->bands.size();
    numDirection = (int)angles->direction.size();
    numBound = (int)mesh->Boundaries.size();
    worldRank = world_rank;
    numProc = num_proc;
    scale_[0] = mesh->L_x, scale_[1] = mesh->L_y, scale_[2] = mesh->L_z;

    node_xyz_.reserve(3 * mesh->Nodes.size());
    for (const Point &p : mesh->Nodes) node_xyz_.insert(node_xyz_.end(), {p.x, p.y, p.z});
    cell_ptr_.assign(1, 0);
    for (const Cell &c : mesh->Elements) {
        cell_verts_.insert(cell_verts_.end(), c.vertexes.begin(), c.vertexes.end());
        cell_ptr_.push_back((int)cell_verts_.size());
        cell_region_.push_back(c.index);  // 0-based region (BTEMesh.cpp:694)
        cell_heat_.push_back(c.heat_source);
    }
    // boundary elements in the reference's boundary order, each as the face
    // it sits on, tagged with its BC file index (after setMeshParams1,
    // Boundary::index is the position in the BC list, BTEMesh.cpp:412-421)
    belem_ptr_.assign(1, 0);
    for (const Boundary &b : mesh->Boundaries) {
        const Face &f = mesh->Elements[b.cellindex[0]].faces[b.faceindex[0]];
        belem_verts_.insert(belem_verts_.end(), f.vertexes.begin(), f.vertexes.end());
        belem_ptr_.push_back((int)belem_verts_.size());
        belem_tag_.push_back(bcs->boundaryConditions[b.index].index);
    }
    // bands, material-major; regions map to materials through geo_matter_index
    num_materials_ = numBand > 0 ? (int)bands->bands[0].group_velocity.size() : 1;
    bool any5 = false;
    for (const BoundaryCondition &bc : bcs->boundaryConditions) {
        bc_tag_.push_back(bc.index);
        bc_type_.push_back(bc.type);
        bc_value_.push_back(bc.temperature);
        any5 = any5 || bc.type == 5;
    }
    // interface walls: each row's transmissivity per material and band, from
    // the blocks the reference read from the interface file
    if (any5) {
        const size_t row = (size_t)num_materials_ * numBand;
        bc_trans_.assign(bcs->boundaryConditions.size() * row, 0.0);
        for (size_t i = 0; i < bcs->boundaryConditions.size(); i++)
            for (const transcoeff &t : bcs->boundaryConditions[i].matter_trans)
                for (int b = 0; b < numBand && b < (int)t.trans.size(); b++)
                    if (t.matter >= 0 && t.matter < num_materials_)
                        bc_trans_[i * row + (size_t)t.matter * numBand + b] = t.trans[b];
    }
    for (int m = 0; m < num_materials_; m++)
        for (const Band &b : bands->bands) {
            band_v_.push_back(b.group_velocity[m]);
            band_tau_.push_back(b.relaxation_time[m]);
            band_C_.push_back(b.heat_capacity[m]);
            band_lat_.push_back(b.lattice_ratio[m]);
            band_hr_.push_back(b.heat_ratio[m]);
        }
    region_material_ = bands->geo_matter_index;
    // the quadrature as the angle object holds it; its solid angle tells the
    // material dimension (2 pi: 2D, 4 pi: 3D; BTEAngle.cpp:11-190)
    for (int d = 0; d < numDirection; d++) {
        dir_xyz_.insert(dir_xyz_.end(), {angles->direction[d].x, angles->direction[d].y, angles->direction[d].z});
        dir_w_.push_back(angles->weight[d]);
    }
    solid_angle_ = angles->SolidAngle;
    material_dimension_ = std::fabs(solid_angle_ - 2 * M_PI) < 1e-9 ? 2 : 3;

    temperature = new double[numCell]();
    heatFluxXGlobal = new double[numCell]();
    heatFluxYGlobal = new double[numCell]();
    heatFluxZGlobal = new double[numCell]();
    totalEnergy = new double[numCell]();
    temperatureband = new double[(size_t)numCell * numBand]();
    boundaryThermal = new double[numBound];
    for (int i = 0; i < numBound; i++) boundaryThermal[i] = mesh->Boundaries[i].Temperature;
}

StaticBTESynthetic::~StaticBTESynthetic() {
    if (h_) gbte_destroy(h_);
    delete[] temperature;
    delete[] heatFluxXGlobal;
    delete[] heatFluxYGlobal;
    delete[] heatFluxZGlobal;
    delete[] totalEnergy;
    delete[] temperatureband;
    delete[] boundaryThermal;
}

void StaticBTESynthetic::run(int order, int sequential, int Use_Backup, int max_iter, int use_limiter,
                             double error_temp_limit, double error_flux_limit) {
    if (Use_Backup != 0) {
        std::cout << "B200 solver: Use_Backup restarts are not supported" << std::endl;
        std::exit(1);
    }
    if (h_ && (h_order_ != order || h_sequential_ != sequential || h_limiter_ != use_limiter)) {
        gbte_destroy(h_);
        h_ = nullptr;
    }
    if (!h_) {
        gbte_mesh_view mv{};
        mv.dimension = dimension;
        mv.num_nodes = (int)(node_xyz_.size() / 3);
        mv.num_cells = numCell;
        mv.num_boundary_elements = numBound;
        mv.node_xyz = node_xyz_.data();
        mv.cell_ptr = cell_ptr_.data();
        mv.cell_verts = cell_verts_.data();
        mv.cell_region = cell_region_.data();
        mv.belem_ptr = belem_ptr_.data();
        mv.belem_verts = belem_verts_.data();
        mv.belem_tag = belem_tag_.data();
        mv.scale_x = scale_[0], mv.scale_y = scale_[1], mv.scale_z = scale_[2];
        gbte_band_table bt{};
        bt.num_materials = num_materials_;
        bt.num_bands = numBand;
        bt.group_velocity = band_v_.data();
        bt.relaxation_time = band_tau_.data();
        bt.heat_capacity = band_C_.data();
        bt.lattice_ratio = band_lat_.data();
        bt.heat_ratio = band_hr_.data();
        bt.num_regions = (int)region_material_.size();
        bt.region_material = region_material_.data();
        bt.material_dimension = material_dimension_;
        gbte_bc_table bc{};
        bc.num = (int)bc_tag_.size();
        bc.tag = bc_tag_.data();
        bc.type = bc_type_.data();
        bc.value = bc_value_.data();
        bc.transmissivity = bc_trans_.empty() ? nullptr : bc_trans_.data();
        gbte_angle_spec as{};
        as.method = 0;
        as.num_directions = numDirection;
        as.direction_xyz = dir_xyz_.data();
        as.weight = dir_w_.data();
        as.solid_angle = solid_angle_;
        gbte_options opt;
        gbte_default_options(&opt);
        opt.precision = GBTE_FP64;
        opt.use_limiter = use_limiter;
        opt.order = order;
        opt.scheme = sequential;
        opt.cell_heat = cell_heat_.data();
        // the reference solves the macro system exactly (sparse LU) in every
        // Picard step, so a fixed number of outer iterations follows its
        // iterates only with exact macro solves
        opt.macro_exact = 1;
        opt.verbose = worldRank == 0 ? 1 : 0;
        // one GPU per rank; every rank holds every direction (the results
        // are the same on all ranks, so no exchange is needed)
        int ndev = 1;
        const char *dev = std::getenv("GIFTBTE_DEVICES");
        if (dev) ndev = std::max(1, std::atoi(dev));
        opt.device = worldRank % ndev;
        const int rc = gbte_create(&mv, &bt, &bc, &as, &opt, &h_);
        if (rc != GBTE_OK) stop("gbte_create", rc, nullptr);
        h_order_ = order, h_sequential_ = sequential, h_limiter_ = use_limiter;
    }
    std::vector<double> q0(3 * (size_t)numCell);
    for (int i = 0; i < numCell; i++)
        q0[3 * i] = heatFluxXGlobal[i], q0[3 * i + 1] = heatFluxYGlobal[i], q0[3 * i + 2] = heatFluxZGlobal[i];
    int rc = gbte_set_initial(h_, temperature, q0.data(), boundaryThermal);
    if (rc != GBTE_OK) stop("gbte_set_initial", rc, h_);
    // the reference's loop stops at max_iter or at the margins; both end a
    // solve normally here
    rc = gbte_solve_with(h_, max_iter, error_temp_limit, error_flux_limit, nullptr);
    if (rc != GBTE_OK && rc != GBTE_ERR_NOT_CONVERGED) stop("gbte_solve", rc, h_);
    rc = gbte_get_fields(h_, totalEnergy, temperature, q0.data(), temperatureband);
    if (rc != GBTE_OK) stop("gbte_get_fields", rc, h_);
    for (int i = 0; i < numCell; i++)
        heatFluxXGlobal[i] = q0[3 * i], heatFluxYGlobal[i] = q0[3 * i + 1], heatFluxZGlobal[i] = q0[3 * i + 2];
    // the solver's own result files, as its _print_out writes them
    // (StaticBTESynthetic.cpp:2613-2653); SolutionAll::_print_out then
    // writes Temperature.dat, HeatFlux.dat and Result.vtk from the arrays
    if (worldRank == 0) {
        rc = gbte_write_outputs(h_, ".");
        if (rc != GBTE_OK) stop("gbte_write_outputs", rc, h_);
    }
}

void StaticBTESynthetic::solve(int b, int n, int lim, double et, double ef) { run(2, 0, b, n, lim, et, ef); }
void StaticBTESynthetic::solve_Iterative(int b, int n, int lim, double et, double ef) { run(2, 0, b, n, lim, et, ef); }
void StaticBTESynthetic::solve_firstorder(int b, int n, int lim, double et, double ef) { run(1, 0, b, n, 0, et, ef); }
void StaticBTESynthetic::solve_firstorder_Iterative(int b, int n, int lim, double et, double ef) {
    run(1, 0, b, n, 0, et, ef);
}
void StaticBTESynthetic::solve_DOM(int b, int n, int lim, double et, double ef) { run(2, 1, b, n, lim, et, ef); }
void StaticBTESynthetic::solve_DOM_Iterative(int b, int n, int lim, double et, double ef) {
    run(2, 1, b, n, lim, et, ef);
}
void StaticBTESynthetic::solve_DOM_firstorder(int b, int n, int lim, double et, double ef) {
    run(1, 1, b, n, 0, et, ef);
}
void StaticBTESynthetic::solve_DOM_firstorder_Iterative(int b, int n, int lim, double et, double ef) {
    run(1, 1, b, n, 0, et, ef);
}
