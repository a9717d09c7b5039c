// The B200 drop-in StaticBTESynthetic (see StaticBTESynthetic/StaticBTESynthetic.h):
// flattens the reference's mesh, band, boundary-condition and angle objects
// into the C ABI's views once, and runs each solve variant on the device.
#include "StaticBTESynthetic/StaticBTESynthetic.h"

#include <cmath>
#include <cstdlib>
#include <iostream>

#include "giftbte.h"

StaticBTESynthetic::StaticBTESynthetic(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles,
                                       int num_proc, int world_rank) {
    b200_check_library();
    // the reference's constructor reads the same objects
    // (src/StaticBTESynthetic/StaticBTESynthetic.cpp:224-626)
    views_.fill(mesh, bcs, bands, angles);
    dimension = views_.dimension;
    numCell = views_.numCell;
    numBand = views_.numBand;
    numDirection = views_.numDirection;
    numBound = views_.numBound;
    worldRank = world_rank;
    numProc = num_proc;
    temperature = new double[numCell]();
    heatFluxXGlobal = new double[numCell]();
    heatFluxYGlobal = new double[numCell]();
    heatFluxZGlobal = new double[numCell]();
    totalEnergy = new double[numCell]();
    temperatureband = new double[(size_t)numCell * numBand]();
    boundaryThermal = new double[numBound];
    for (int i = 0; i < numBound; i++) boundaryThermal[i] = views_.boundary_thermal[i];
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
        gbte_options opt;
        gbte_default_options(&opt);
        opt.precision = GBTE_FP64;
        opt.use_limiter = use_limiter;
        opt.order = order;
        opt.scheme = sequential;
        // the reference solves the macro system exactly (sparse LU) in every
        // Picard step, so a fixed number of outer iterations follows its
        // iterates only with exact macro solves
        opt.macro_exact = 1;
        opt.verbose = worldRank == 0 ? 1 : 0;
        // one GPU per rank; every rank holds every direction (the results
        // are the same on all ranks, so no exchange is needed)
        opt.device = b200_device(worldRank);
        const int rc = views_.create(opt, &h_);
        if (rc != GBTE_OK) b200_stop("gbte_create", rc, nullptr);
        h_order_ = order, h_sequential_ = sequential, h_limiter_ = use_limiter;
    }
    std::vector<double> q0(3 * (size_t)numCell);
    for (int i = 0; i < numCell; i++)
        q0[3 * i] = heatFluxXGlobal[i], q0[3 * i + 1] = heatFluxYGlobal[i], q0[3 * i + 2] = heatFluxZGlobal[i];
    int rc = gbte_set_initial(h_, temperature, q0.data(), boundaryThermal);
    if (rc != GBTE_OK) b200_stop("gbte_set_initial", rc, h_);
    // the reference's loop stops at max_iter or at the margins; both end a
    // solve normally here
    rc = gbte_solve_with(h_, max_iter, error_temp_limit, error_flux_limit, nullptr);
    if (rc != GBTE_OK && rc != GBTE_ERR_NOT_CONVERGED) b200_stop("gbte_solve", rc, h_);
    rc = gbte_get_fields(h_, totalEnergy, temperature, q0.data(), temperatureband);
    if (rc != GBTE_OK) b200_stop("gbte_get_fields", rc, h_);
    for (int i = 0; i < numCell; i++)
        heatFluxXGlobal[i] = q0[3 * i], heatFluxYGlobal[i] = q0[3 * i + 1], heatFluxZGlobal[i] = q0[3 * i + 2];
    // the solver's own result files, as its _print_out writes them
    // (StaticBTESynthetic.cpp:2613-2653); SolutionAll::_print_out then
    // writes Temperature.dat, HeatFlux.dat and Result.vtk from the arrays
    if (worldRank == 0) {
        rc = gbte_write_outputs(h_, ".");
        if (rc != GBTE_OK) b200_stop("gbte_write_outputs", rc, h_);
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
