// Reference harness stand-in for the CUDA samples' helper_cuda.h: errors are
// recorded, never fatal.
#pragma once
#include <cuda_runtime.h>
void ref_emu_check(int code, const char *what);
#define checkCudaErrors(val) ref_emu_check((int)(val), #val)
#define getLastCudaError(msg) ((void)0)
