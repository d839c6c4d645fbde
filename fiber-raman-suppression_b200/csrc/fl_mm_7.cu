// Multimode evaluation round instance: Nt = 2^7, 4 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(7, 2, 1)
