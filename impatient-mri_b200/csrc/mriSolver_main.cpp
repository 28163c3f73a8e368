// mriSolver executable: the reference's command line (main.cpp:103) over the C-ABI.
#include "../../include/impatient_b200.h"

int main(int argc, char **argv) { return imp_mrisolver_main(argc, argv); }
