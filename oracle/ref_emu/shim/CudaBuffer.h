// The reference includes "CudaBuffer.h"; the file is cudaBuffer.h (case-insensitive on its platform).
#include "cudaBuffer.h"
