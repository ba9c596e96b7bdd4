// Drop-in executable for the reference tool kirchmig2d (adj=1).
#include <stdlib.h>

#include "../../include/kcig.h"

int main(int argc, char **argv) { return kcig_run_kirchmig2d_cli(argc, argv) == KCIG_OK ? EXIT_SUCCESS : EXIT_FAILURE; }
