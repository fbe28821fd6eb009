// bem3_lib.cu -- single translation unit of the CUDA library (the kernels share __constant__
// tables, so they are compiled together rather than with relocatable device code).
#include "assemble.cu"
#include "self_interior.cu"
#include "capi.cu"
#include "solve.cu"
#include "field.cu"
#include "force.cu"
#include "solve_dtn.cu"
#include "context.cu"
#include "batch.cu"
#include "mesh.cu"
