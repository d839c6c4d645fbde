// Single-mode stepper instance: double, Nt = 2^12, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, 12, 4)
