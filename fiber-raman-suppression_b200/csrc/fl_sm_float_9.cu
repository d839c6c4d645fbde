// Single-mode stepper instance: FP32 forward / FP64 adjoint, Nt = 2^9, 16 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, float, double, 9, 4)
