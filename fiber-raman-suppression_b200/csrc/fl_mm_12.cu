// Multimode evaluation round instance: Nt = 2^12, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(12, 4, 1)
