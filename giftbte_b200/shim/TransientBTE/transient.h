// B200 drop-in for GiftBTE's explicit transient solver class.
//
// Put the shim directory ahead of GiftBTE's includes/ on the include path and
// link transient_b200.cpp, b200_deck_views.cpp and libgiftbte_b200 in place
// of src/TransientBTE/*.cpp: the reference's
// SolutionAll::_Transient_BTE_Solver (src/Solution/Solution.cpp:500-520) then
// compiles unchanged against this class and runs State=Transient on the GPU
// through gbte_transient_solve (include/giftbte.h). The class keeps the
// reference's interface as its caller uses it
// (includes/TransientBTE/transient.h:169-206): the constructor, solve, and
// the arrays read after it (temperature, heatFlux{X,Y,Z}Global). It writes
// the reference's result files: TTG.dat (time and the temperature of cell 0
// after every step), Tempcell.dat, Tempcell1.dat, HeatSource.dat and
// HeatFlux.dat (transient.cpp:865-889).
#ifndef STATICBTESOLVER_TRANSIENT_H
#define STATICBTESOLVER_TRANSIENT_H
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

class Transient {
public:
    int dimension = 0;
    int numCell = 0;
    int numBand = 0;
    int numDirection = 0;
    int numBound = 0;
    int worldRank = 0;
    int numProc = 1;
    // the caller writes the steady start here before solve (the reference's
    // solve replaces it with its grating start); results after solve
    double *temperature = nullptr;
    double *heatFluxXGlobal = nullptr;
    double *heatFluxYGlobal = nullptr;
    double *heatFluxZGlobal = nullptr;

    Transient(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles, int num_proc,
              int world_rank, double deltaT, double totalT, int use_TDTR, double pulse_time,
              double repetition_frequency, double modulation_frequency, double xy_r);

    void solve(int Use_Backup, double error_temp_limit, double error_flux_limit, double deltaT, double totalT,
               int use_TDTR, double pulse_time, double repetition_frequency, double modulation_frequency,
               double xy_r);
    // an empty function in the reference (TransientSolver.cpp:304-307)
    void solve_first_order(int Use_Backup, int Use_Limiter, double error_temp_limit, double error_flux_limit,
                           double deltaT, double totalT);

    Transient(const Transient &) = delete;
    ~Transient();

private:
    B200DeckViews views_;
};

#endif  // STATICBTESOLVER_TRANSIENT_H
