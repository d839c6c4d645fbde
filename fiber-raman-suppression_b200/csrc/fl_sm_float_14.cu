// Single-mode stepper instance: FP32 forward / FP64 adjoint, Nt = 2^14, 32 elements per thread.
#include "fl_sm_inst.cuh"
FL_SM_INSTANCE(float, float, double, 14, 5)
