// Single-mode stepper instance: double, Nt = 2^8, 8 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, 8, 3)
