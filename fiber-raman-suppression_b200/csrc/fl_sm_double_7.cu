// Single-mode stepper instance: double, Nt = 2^7, 4 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(double, 7, 2)
