// Single-mode stepper instance: FP64 throughout, Nt = 2^13, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, double, double, 13, 4)
