// Single translation unit for the prover: one copy of each __constant__
// table, no relocatable device code needed. (lde_noalloc.cu is separate.)
#include "capi_stage.cuh"
#include "capi_prove.cuh"
#include "capi_server.cuh"
#include "capi_verify.cuh"
#include "capi_tune.cuh"
