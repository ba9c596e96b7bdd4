// Drop-in executable for the reference tool layercom_cig (ADCIG stitching).
#include <stdlib.h>

#include "../../include/kcig.h"

int main(int argc, char **argv) { return kcig_run_layercom_cig_cli(argc, argv) == KCIG_OK ? EXIT_SUCCESS : EXIT_FAILURE; }
