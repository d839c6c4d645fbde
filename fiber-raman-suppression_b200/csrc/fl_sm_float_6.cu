// Single-mode stepper instance: float, Nt = 2^6, 2 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, 6, 1)
