// Multimode evaluation round instance: Nt = 2^8, 8 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(8, 3, 1)
