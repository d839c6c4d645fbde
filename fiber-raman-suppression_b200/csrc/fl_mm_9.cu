// Multimode evaluation round instance: Nt = 2^9, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(9, 4, 1)
