// Single translation unit for the whole library: one copy of the
// __constant__ Poseidon2 table, no relocatable device code needed.
#include "capi_stage.cuh"
