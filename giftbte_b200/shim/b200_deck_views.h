// The reference's mesh, band, boundary-condition and angle objects
// flattened once into the C ABI's views (include/giftbte.h), for the B200
// drop-in classes that replace GiftBTE's solver classes (StaticBTESynthetic,
// Transient). The views point into this object's vectors, so it must
// outlive the handles made from it only while gbte_create runs (the library
// copies what it keeps).
#ifndef GIFTBTE_B200_DECK_VIEWS_H
#define GIFTBTE_B200_DECK_VIEWS_H
#include <string>
#include <vector>

#include "BTEAngle/BTEAngle.h"
#include "BTEBand/BTEBand.h"
#include "BTEBoundaryCondition/BTEBoundaryCondition.h"
#include "BTEMesh/BTEMesh.h"
#include "giftbte.h"

struct B200DeckViews {
    int dimension = 0, numCell = 0, numBand = 0, numDirection = 0, numBound = 0;
    // cell centres and the wall temperatures the reference's objects hold
    std::vector<double> center_x, center_y, center_z, boundary_thermal, cell_heat;

    // reads the objects the reference's solver constructors read
    // (src/StaticBTESynthetic/StaticBTESynthetic.cpp:224-626,
    // src/TransientBTE/transient.cpp:178-585)
    void fill(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles);
    // gbte_create over the views with the given options
    int create(const gbte_options &opt, gbte_handle **out) const;

private:
    std::vector<double> node_xyz_, band_v_, band_tau_, band_C_, band_lat_, band_hr_;
    std::vector<double> dir_xyz_, dir_w_, bc_value_, bc_trans_;
    std::vector<int> cell_ptr_, cell_verts_, cell_region_, belem_ptr_, belem_verts_, belem_tag_;
    std::vector<int> region_material_, bc_tag_, bc_type_;
    double scale_[3] = {1, 1, 1};
    double solid_angle_ = 0;
    int num_materials_ = 1, material_dimension_ = 2;
};

// The library's options struct must be the one this drop-in was compiled
// with; the reference reports errors on cout and exits, and so do these.
void b200_check_library();
[[noreturn]] void b200_stop(const char *what, int rc, const gbte_handle *h);
// the device of this rank: rank % GIFTBTE_DEVICES (default one GPU)
int b200_device(int world_rank);

#endif  // GIFTBTE_B200_DECK_VIEWS_H
