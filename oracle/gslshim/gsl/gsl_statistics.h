/* GSL-API shim header (oracle test infrastructure); declarations in ../gsl_shim.h */
#include "../gsl_shim.h"
