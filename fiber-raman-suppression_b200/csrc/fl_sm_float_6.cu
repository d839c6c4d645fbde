// Single-mode stepper instance: FP32 forward / FP64 adjoint, Nt = 2^6, 2 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, float, double, 6, 1)
