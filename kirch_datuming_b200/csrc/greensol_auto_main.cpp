// Drop-in executable for the reference tool greensol_auto.
#include <stdlib.h>

#include "../../include/kcig.h"

int main(int argc, char **argv) { return kcig_run_greensol_auto_cli(argc, argv) == KCIG_OK ? EXIT_SUCCESS : EXIT_FAILURE; }
