/* Empty stand-in: the oracle replaces the PARDISO driver with its own dense solver. */
#include "mkl_types.h"
