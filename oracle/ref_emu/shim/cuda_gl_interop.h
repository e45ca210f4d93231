// Reference harness stand-in for cuda_gl_interop.h (no graphics stack here):
// GL buffer/texture names map to host arrays registered by the harness.
#pragma once
#include <cuda_runtime.h>
#include "GL/freeglut.h"
#define GL_TEXTURE_2D 0x0DE1
cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource **res, GLuint buffer, unsigned int flags);
cudaError_t cudaGraphicsGLRegisterImage(cudaGraphicsResource **res, GLuint image, GLenum target, unsigned int flags);
