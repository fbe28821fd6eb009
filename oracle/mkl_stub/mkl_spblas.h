/* Empty stand-in: no sparse BLAS routine is called by the compiled oracle sources. */
#include "mkl_types.h"
