// Single translation unit for the whole library: one copy of each
// __constant__ table, no relocatable device code needed.
#include "capi_stage.cuh"
#include "capi_prove.cuh"
