// Reference GPU harness stand-in for the CUDA samples' helper_cuda.h: a failed
// call is recorded (count and first message), never fatal.
#pragma once
#include <cuda_runtime.h>
void refgpu_check(int code, const char *what, const char *file, int line);
#define checkCudaErrors(val) refgpu_check((int)(val), #val, __FILE__, __LINE__)
#define getLastCudaError(msg) refgpu_check((int)cudaGetLastError(), msg, __FILE__, __LINE__)
