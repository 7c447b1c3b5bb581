/*
 * ref_shim.h -- force-included (g++ -include) ahead of the reference's own ksw_extend2
 * source lines when oracle/build_ref.sh compiles them as host C++.  Test infrastructure
 * only: it maps the CUDA qualifier away and routes the device bump arena calls
 * (CUDAKernelMalloc / CUDAKernelCalloc, bwa/src/gmem_alloc.h:22-23) to a host bump arena
 * that ref_wrap.cpp resets before every call.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#define __device__
void *g3r_arena_take(void *arena, size_t bytes, int zero);
#define CUDAKernelMalloc(arena, size, align) g3r_arena_take((arena), (size_t)(size), 0)
#define CUDAKernelCalloc(arena, num, size, align) g3r_arena_take((arena), (size_t)(num) * (size_t)(size), 1)
