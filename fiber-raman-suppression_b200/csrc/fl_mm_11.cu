// Multimode evaluation round instance: Nt = 2^11, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(11, 4, 1)
