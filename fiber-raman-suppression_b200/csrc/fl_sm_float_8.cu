// Single-mode stepper instance: float, Nt = 2^8, 8 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, 8, 3)
