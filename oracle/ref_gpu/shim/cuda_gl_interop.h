// Reference GPU harness stand-in for cuda_gl_interop.h (no graphics stack): the
// two GL registration calls the reference makes are renamed to harness
// functions that look the GL name up in the harness's buffer registry.
#pragma once
#include <cuda_runtime.h>
#include "GL/freeglut.h"
#define GL_TEXTURE_2D 0x0DE1
#define cudaGraphicsGLRegisterBuffer refgpu_gl_register_buffer
#define cudaGraphicsGLRegisterImage refgpu_gl_register_image
cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource **res, GLuint buffer, unsigned int flags);
cudaError_t cudaGraphicsGLRegisterImage(cudaGraphicsResource **res, GLuint image, GLenum target, unsigned int flags);
