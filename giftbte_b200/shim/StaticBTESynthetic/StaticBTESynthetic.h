// B200 drop-in for GiftBTE's steady solver class.
//
// Put this directory ahead of GiftBTE's includes/ on the include path and
// link StaticBTESynthetic_b200.cpp and libgiftbte_b200 in place of
// src/StaticBTESynthetic/*.cpp: the reference's SolutionAll::_BTE_Solver
// (src/Solution/Solution.cpp:262-414) then compiles unchanged against this
// class and runs its steady solve on the GPU through the C ABI of
// include/giftbte.h. The class keeps the reference's interface
// (includes/StaticBTESynthetic/StaticBTESynthetic.h:177,221-235): the same
// constructor, the eight solve variants, and the public arrays the caller
// writes before a solve (temperature, heatFlux{X,Y,Z}Global,
// boundaryThermal) and reads after it (totalEnergy, temperature,
// heatFlux{X,Y,Z}Global, temperatureband). Everything else of the reference
// class (its LU factors, per-band work arrays, the MPI decomposition) has
// no counterpart: the device holds the state.
#ifndef STATICBTESOLVER_STATICBTESYNTHETIC_H
#define STATICBTESOLVER_STATICBTESYNTHETIC_H
#include <memory>
#include <string>
#include <unordered_set>
#include <vector>

#include "BTEAngle/BTEAngle.h"
#include "BTEBand/BTEBand.h"
#include "BTEBoundaryCondition/BTEBoundaryCondition.h"
#include "BTEMesh/BTEMesh.h"
#include "utility/utility.h"

// the reference header provides these to the files that include it
#include "Eigen/Sparse"
#include "Eigen/SparseLU"
typedef Eigen::Triplet<double> Tri;

#include "b200_deck_views.h"

class StaticBTESynthetic {
public:
    int dimension = 0;
    int numCell = 0;
    int numBand = 0;
    int numDirection = 0;
    int numBound = 0;
    int worldRank = 0;
    int numProc = 1;

    // written by the caller before a solve (initial field, previous-iterate
    // flux, boundary temperatures; the constructor fills them like the
    // reference: zeros and each boundary's BC value)
    double *temperature = nullptr;
    double *heatFluxXGlobal = nullptr;
    double *heatFluxYGlobal = nullptr;
    double *heatFluxZGlobal = nullptr;
    double *boundaryThermal = nullptr;
    // results after a solve (temperature is overwritten with the lattice
    // temperature, as the reference does)
    double *totalEnergy = nullptr;
    double *temperatureband = nullptr;  // [numBand * numCell], band-major
    // declared so that SolutionAll::_get_solver (a function the reference
    // never calls) still compiles; not populated
    double ***energyDensity = nullptr;
    double *ebound = nullptr;
    double *boundaryTemp = nullptr;
    double *boundaryFlux = nullptr;

    StaticBTESynthetic(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles, int num_proc,
                       int world_rank);

    // Order=2 Synthetic (LU / BICGSTAB: the sweep solves the transport
    // systems exactly either way); USE_limiter = 1 is Order=2limit
    void solve(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit, double error_flux_limit);
    void solve_Iterative(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                         double error_flux_limit);
    // Order=1 Synthetic
    void solve_firstorder(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                          double error_flux_limit);
    void solve_firstorder_Iterative(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                                    double error_flux_limit);
    // Order=2 Sequential
    void solve_DOM(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit, double error_flux_limit);
    void solve_DOM_Iterative(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                             double error_flux_limit);
    // Order=1 Sequential
    void solve_DOM_firstorder(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                              double error_flux_limit);
    void solve_DOM_firstorder_Iterative(int Use_Backup, int max_iter, int USE_limiter, double error_temp_limit,
                                        double error_flux_limit);

    StaticBTESynthetic(const StaticBTESynthetic &solver) = delete;
    ~StaticBTESynthetic();

private:
    void run(int order, int sequential, int Use_Backup, int max_iter, int use_limiter, double error_temp_limit,
             double error_flux_limit);
    // the reference's objects flattened into the C ABI's views (kept for
    // the handle, which is created by the first solve: the variant's order,
    // scheme and limiter are options of gbte_create)
    B200DeckViews views_;
    gbte_handle *h_ = nullptr;
    int h_order_ = 0, h_sequential_ = 0, h_limiter_ = 0;
};

#endif  // STATICBTESOLVER_STATICBTESYNTHETIC_H
