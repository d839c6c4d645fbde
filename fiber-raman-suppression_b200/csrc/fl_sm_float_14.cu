// Single-mode stepper instance: float, Nt = 2^14, 32 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, 14, 5)
