// Compiles the reference's cudaFluidStep.cu with the MC slope limiter, the choice the reference
// makes with its SLOPEFUNC define (gpuclass/cudaFluidStep.cu:129-135).  The limiter header is
// read first so that its functions keep their own names; afterwards the name of the default
// (Ospre) slope limiter is mapped to the MC limiter for the kernels that use it.
#include "limiter_functions.h"
#define slopeLimiter_Ospre slopeLimiter_MC
#include "cudaFluidStep.cu"
