// Drop-in executable for the reference tool eikods2d (2-D velocity files).
#include <stdlib.h>

#include "../../include/kcig.h"

int main(int argc, char **argv) { return kcig_run_eikods_cli(argc, argv) == KCIG_OK ? EXIT_SUCCESS : EXIT_FAILURE; }
