// Single-mode stepper instance: double, Nt = 2^10, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, 10, 4)
