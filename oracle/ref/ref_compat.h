/*
 * ref_compat.h — forced include for building the reference harness (test infrastructure).
 *
 * methods_cuda.cu:814 reads `dirvectors[dim].v[i]` through a `curandDirectionVectors32_t*`,
 * but cuRAND declares that type as `unsigned int[32]` (no member `v`), so the file does not
 * compile as shipped.  Instead of editing or copying the reference, this header is included
 * first: it pulls in the cuRAND headers under their real names, then makes the name the
 * reference uses denote a struct with the member `v` and the same size and layout (128 bytes),
 * and adapts the one host API that takes the array type.
 */
#pragma once
#include <curand.h>
#include <curand_kernel.h>

typedef curandDirectionVectors32_t mcqref_dv32_array;
struct mcqref_dv32 { unsigned int v[32]; };
static_assert(sizeof(mcqref_dv32) == sizeof(mcqref_dv32_array), "layout");
#define curandDirectionVectors32_t mcqref_dv32
#define curandGetDirectionVectors32(ptr, set) \
    curandGetDirectionVectors32(reinterpret_cast<mcqref_dv32_array**>(ptr), (set))
