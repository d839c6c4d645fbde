// Multimode evaluation round instance: Nt = 2^14, 32 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(14, 5, 1)
