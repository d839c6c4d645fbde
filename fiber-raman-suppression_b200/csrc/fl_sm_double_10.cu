// Single-mode stepper instance: FP64 throughout, Nt = 2^10, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, double, double, 10, 4)
