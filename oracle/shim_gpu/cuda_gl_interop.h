/* Stand-in for <cuda_gl_interop.h> in the GPU build of the reference harness: the
 * reference's include/renderers/renderer.h includes it only for the cudaGraphicsResource
 * type, which <cuda_runtime.h> already declares. No OpenGL header or library is involved;
 * the harness never registers or maps graphics resources. */
#pragma once
#include <cuda_runtime.h>
