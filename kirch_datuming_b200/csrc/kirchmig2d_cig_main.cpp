// Drop-in executable for the reference tool kirchmig2d_cig (adj=1).
#include <stdlib.h>

#include "../../include/kcig.h"

int main(int argc, char **argv) { return kcig_run_cli(argc, argv) == KCIG_OK ? EXIT_SUCCESS : EXIT_FAILURE; }
