// Single-mode stepper instance: double, Nt = 2^6, 2 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, 6, 1)
