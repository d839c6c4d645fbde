// Multimode evaluation round instance: Nt = 2^14, FP32 transforms on one CTA
// (32 elements per thread), FP64 transforms over a cluster of 2 CTAs (16 per
// thread: 2^14 FP64 values do not fit one CTA's registers).
#include "fl_mm_inst.cuh"
FL_MM_INSTANCE2(14, 5, 1, 4, 2)
