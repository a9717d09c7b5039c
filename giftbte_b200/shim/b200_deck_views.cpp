// The reference's objects flattened into the C ABI's views (see
// b200_deck_views.h), shared by the B200 drop-in solver classes.
#include "b200_deck_views.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <iostream>

void b200_check_library() {
    if (gbte_options_size() != sizeof(gbte_options)) {
        std::cout << "B200 solver: libgiftbte_b200 was built from another giftbte.h (options of "
                  << gbte_options_size() << " bytes, this drop-in expects " << sizeof(gbte_options)
                  << "); rebuild the drop-in" << std::endl;
        std::exit(1);
    }
}

void b200_stop(const char *what, int rc, const gbte_handle *h) {
    std::cout << "B200 solver: " << what << " failed (" << gbte_status_string(rc) << "): " << gbte_last_error(h)
              << std::endl;
    std::exit(1);
}

int b200_device(int world_rank) {
    int ndev = 1;
    const char *dev = std::getenv("GIFTBTE_DEVICES");
    if (dev) ndev = std::max(1, std::atoi(dev));
    return world_rank % ndev;
}

void B200DeckViews::fill(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles) {
    dimension = mesh->Dimension;
    numCell = (int)mesh->Elements.size();
    numBand = (int)bands->bands.size();
    numDirection = (int)angles->direction.size();
    numBound = (int)mesh->Boundaries.size();
    scale_[0] = mesh->L_x, scale_[1] = mesh->L_y, scale_[2] = mesh->L_z;

    node_xyz_.reserve(3 * mesh->Nodes.size());
    for (const Point &p : mesh->Nodes) node_xyz_.insert(node_xyz_.end(), {p.x, p.y, p.z});
    cell_ptr_.assign(1, 0);
    for (const Cell &c : mesh->Elements) {
        cell_verts_.insert(cell_verts_.end(), c.vertexes.begin(), c.vertexes.end());
        cell_ptr_.push_back((int)cell_verts_.size());
        cell_region_.push_back(c.index);  // 0-based region (BTEMesh.cpp:694)
        cell_heat.push_back(c.heat_source);
        center_x.push_back(c.center.x);
        center_y.push_back(c.center.y);
        center_z.push_back(c.center.z);
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
        boundary_thermal.push_back(b.Temperature);
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
}

int B200DeckViews::create(const gbte_options &opt_in, gbte_handle **out) const {
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
    gbte_options opt = opt_in;
    opt.cell_heat = cell_heat.data();
    return gbte_create(&mv, &bt, &bc, &as, &opt, out);
}
