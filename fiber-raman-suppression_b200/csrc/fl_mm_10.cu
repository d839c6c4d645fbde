// Multimode evaluation round instance: Nt = 2^10, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(10, 4, 1)
