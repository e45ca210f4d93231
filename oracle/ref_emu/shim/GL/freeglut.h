// Reference harness stand-in for GL/freeglut.h: GL scalar types only.
#pragma once
typedef unsigned int GLuint;
typedef unsigned int GLenum;
typedef int GLint;
typedef float GLfloat;
