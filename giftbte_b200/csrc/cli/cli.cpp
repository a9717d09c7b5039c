// giftbte_cli: command-line drop-in for the reference's BTE_CPU main
// (src/BTEMain.cpp) on the steady synthetic path. Reads input/CONTROL,
// input/GEOMETRY, input/PHONON and the files they name from the working
// directory (or from the directory given as the first argument), solves on
// one GPU and writes Temperature.dat, TempLattice.dat, HeatFlux.dat,
// Tempband.dat and Result.vtk next to input/.
//   giftbte_cli [deck_dir] [--fp32] [--device N] [--quiet]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "giftbte.h"

int main(int argc, char **argv) {
    std::string dir = ".";
    gbte_options opt;
    gbte_default_options(&opt);
    opt.verbose = 1;
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--fp32"))
            opt.precision = GBTE_FP32_MIXED;
        else if (!std::strcmp(argv[i], "--quiet"))
            opt.verbose = 0;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            opt.device = std::atoi(argv[++i]);
        else
            dir = argv[i];
    }
    gbte_handle *h = nullptr;
    int rc = gbte_create_from_deck(dir.c_str(), &opt, &h);
    if (rc != GBTE_OK) {
        std::fprintf(stderr, "Error: %s (%s)\n", gbte_last_error(nullptr), gbte_status_string(rc));
        return 1;
    }
    int frc = gbte_fourier_initial(h);
    if (frc != GBTE_OK && frc != GBTE_ERR_UNSUPPORTED) {
        std::fprintf(stderr, "Error: %s\n", gbte_last_error(h));
        gbte_destroy(h);
        return 1;
    }
    gbte_stats st;
    rc = gbte_solve(h, &st);
    if (rc != GBTE_OK && rc != GBTE_ERR_NOT_CONVERGED) {
        std::fprintf(stderr, "Error: %s (%s)\n", gbte_last_error(h), gbte_status_string(rc));
        gbte_destroy(h);
        return 1;
    }
    std::printf("iterations %d  margins T %.3e q %.3e  solve %.3f ms  (%.3e band*dir*cell updates/s)\n", st.iterations,
                st.err_temp, st.err_flux, st.solve_ms, st.updates / (st.solve_ms * 1e-3));
    rc = gbte_write_outputs(h, dir.c_str());
    gbte_destroy(h);
    return rc == GBTE_OK ? 0 : 1;
}
