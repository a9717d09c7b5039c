// Host-only driver of gbte::scatter_rows (built by tests/test_abi.py with
// g++ from the library's host sources): random permutations, one to many
// columns of rows of 1 or 3 values, so both the column-per-thread and the
// row-range paths run; each result must equal the plain serial scatter
// a[perm[k]] = old a[k]. Prints one line per case and "OK" when all match.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "gbte_internal.h"

int main() {
    std::mt19937 rng(7);
    int bad = 0;
    for (int nc : {1, 5, 4096 + 17, 100003})
        for (int ncols : {1, 3, 4, 45})
            for (int w : {1, 3}) {
                std::vector<int> perm(nc);
                for (int k = 0; k < nc; k++) perm[k] = k;
                std::shuffle(perm.begin(), perm.end(), rng);
                std::vector<std::vector<double>> got(ncols), want(ncols);
                std::vector<double *> cols(ncols);
                for (int c = 0; c < ncols; c++) {
                    got[c].resize((size_t)nc * w);
                    for (auto &x : got[c]) x = std::uniform_real_distribution<double>(-1, 1)(rng);
                    want[c].assign(got[c].size(), 0.0);
                    for (int k = 0; k < nc; k++)
                        for (int j = 0; j < w; j++) want[c][(size_t)perm[k] * w + j] = got[c][(size_t)k * w + j];
                    cols[c] = got[c].data();
                }
                gbte::scatter_rows(perm, cols.data(), ncols, w);
                bool ok = true;
                for (int c = 0; c < ncols; c++) ok = ok && got[c] == want[c];
                std::printf("nc %d cols %d w %d: %s\n", nc, ncols, w, ok ? "match" : "DIFFER");
                bad += !ok;
            }
    std::printf("%s\n", bad ? "FAIL" : "OK");
    return bad ? 1 : 0;
}
