// Toeplitz reconstruction path (placeholder until the gridding / FFT engine lands).
#include "../../include/impatient_b200.h"

#include <cstdio>

extern "C" imp_status imp_toeplitz_dir_cli(const char *, const char *, int, int, float, int,
                                           int, int, float, float, float, int, int,
                                           const char *, int) {
    std::fprintf(stderr, "\nError: the Toeplitz path is not built yet.\n");
    return IMP_ERR_UNSUPPORTED;
}
