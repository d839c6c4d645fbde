// Single-mode stepper instance: FP64 throughout, Nt = 2^11, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, double, double, 11, 4)
