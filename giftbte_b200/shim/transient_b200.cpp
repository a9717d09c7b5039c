// The B200 drop-in Transient (see TransientBTE/transient.h): flattens the
// reference's objects into the C ABI's views and runs the explicit
// transient solve on the device.
#include "TransientBTE/transient.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "giftbte.h"

Transient::Transient(BTEMesh *mesh, BTEBoundaryCondition *bcs, BTEBand *bands, BTEAngle *angles, int num_proc,
                     int world_rank, double, double, int, double, double, double, double) {
    b200_check_library();
    // the objects the reference's constructor reads (transient.cpp:178-585)
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
}

Transient::~Transient() {
    delete[] temperature;
    delete[] heatFluxXGlobal;
    delete[] heatFluxYGlobal;
    delete[] heatFluxZGlobal;
}

void Transient::solve_first_order(int, int, double, double, double, double) {}

void Transient::solve(int Use_Backup, double error_temp_limit, double error_flux_limit, double deltaT,
                      double totalT, int use_TDTR, double, double, double, double) {
    if (Use_Backup != 0) {
        std::cout << "B200 solver: Use_Backup restarts are not supported" << std::endl;
        std::exit(1);
    }
    if (use_TDTR == 1) {
        std::cout << "B200 solver: the TDTR pulse source is not built" << std::endl;
        std::exit(1);
    }
    gbte_options opt;
    gbte_default_options(&opt);
    opt.precision = GBTE_FP64;
    opt.order = 2;
    opt.verbose = worldRank == 0 ? 1 : 0;
    opt.device = b200_device(worldRank);
    gbte_handle *h = nullptr;
    int rc = views_.create(opt, &h);
    if (rc != GBTE_OK) b200_stop("gbte_create", rc, nullptr);
    // the steps the reference takes: the integers below totalT / deltaT;
    // TTG.dat keeps the first 2^26 of them
    const long long steps = (long long)std::ceil(totalT / deltaT);
    const long long kept = std::min(steps, 1LL << 26);
    std::vector<double> ttg((size_t)kept, 0.0);
    gbte_transient_stats st{};
    rc = gbte_transient_solve(h, deltaT, totalT, error_temp_limit, error_flux_limit, 0, ttg.data(), kept, &st);
    if (rc != GBTE_OK) b200_stop("gbte_transient_solve", rc, h);
    std::vector<double> q(3 * (size_t)numCell);
    rc = gbte_get_fields(h, nullptr, temperature, q.data(), nullptr);
    if (rc != GBTE_OK) b200_stop("gbte_get_fields", rc, h);
    gbte_destroy(h);
    for (int i = 0; i < numCell; i++)
        heatFluxXGlobal[i] = q[3 * i], heatFluxYGlobal[i] = q[3 * i + 1], heatFluxZGlobal[i] = q[3 * i + 2];
    if (worldRank != 0) return;
    // the reference's result files (TransientSolver.cpp:147, :216;
    // transient.cpp:865-889); Tempcell1.dat holds an array the reference
    // never fills, written as zeros here
    const std::vector<double> &x = views_.center_x, &y = views_.center_y, &z = views_.center_z;
    std::ofstream ttgf("TTG.dat");
    for (long long n = 0; n < std::min(st.steps, kept); n++)
        ttgf << (n + 1) * deltaT << " " << ttg[(size_t)n] << std::endl;
    std::ofstream t0("Tempcell.dat"), t1("Tempcell1.dat"), hs("HeatSource.dat"), hf("HeatFlux.dat");
    for (int i = 0; i < numCell; i++) {
        t0 << x[i] << " " << y[i] << " " << z[i] << " " << temperature[i] << std::endl;
        t1 << x[i] << " " << y[i] << " " << z[i] << " " << 0.0 << std::endl;
        hs << x[i] << " " << y[i] << " " << z[i] << " " << views_.cell_heat[i] << std::endl;
        hf << std::setw(15) << x[i] << std::setw(15) << y[i] << std::setw(15) << z[i] << std::setw(15)
           << heatFluxXGlobal[i] << std::setw(15) << heatFluxYGlobal[i] << std::setw(15) << heatFluxZGlobal[i]
           << std::endl;
    }
}
