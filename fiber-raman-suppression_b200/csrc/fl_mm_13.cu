// Multimode evaluation round instance: Nt = 2^13, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(13, 4, 1)
