// Single-mode stepper instance: float, Nt = 2^12, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, 12, 4)
