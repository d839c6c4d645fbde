// Single-mode stepper instance: float, Nt = 2^7, 4 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, 7, 2)
