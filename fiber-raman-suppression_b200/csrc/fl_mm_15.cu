// Multimode evaluation round instance: Nt = 2^15 over a cluster of 4 CTAs per
// transform, 16 elements per thread.
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE(15, 4, 4)
