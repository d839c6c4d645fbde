// Multimode evaluation round instance: Nt = 2^6, 2 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(6, 1, 1)
