// Single-mode stepper instance: FP64 throughout, Nt = 2^8, 8 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, double, double, 8, 3)
