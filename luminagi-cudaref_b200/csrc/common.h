// common.h -- error plumbing shared by the library's translation units.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "lumina.h"

namespace lg
{
// Records a thread-local message for lg_last_error() and returns `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

// Sizes and layout checks tying the C ABI records to the C++ drop-in structs.
static_assert(sizeof(lg_triangle) == 100, "lg_triangle layout");
static_assert(sizeof(lg_bvh_node) == 40, "lg_bvh_node layout");
static_assert(sizeof(lg_point_light) == 32, "lg_point_light layout");
static_assert(sizeof(lg_dir_light) == 28, "lg_dir_light layout");
}  // namespace lg

#define LG_TRY_CUDA(expr)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (expr);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return ::lg::set_error(LG_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #expr,        \
                                   cudaGetErrorString(e_));                                        \
    } while (0)

#define LG_TRY(expr)                                                                               \
    do {                                                                                           \
        int rc_ = (expr);                                                                          \
        if (rc_ != LG_OK) return rc_;                                                              \
    } while (0)
