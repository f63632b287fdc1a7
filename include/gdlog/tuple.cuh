// gdlog/tuple.cuh — tuple and hook types of the drop-in C++ API.
//
// Same names and meanings as the reference's include/tuple.cuh:5-25:
// columns are unsigned 64-bit, a tuple is a pointer to its first column,
// and user callbacks are __device__ functions whose addresses the program
// fetches with cudaMemcpyFromSymbol (test/tc.cu:126-130).
#pragma once

#include <cstdint>

using u64 = unsigned long long;
using u32 = unsigned long;  // the reference's (misnamed) 64-bit column type

using column_type = u32;
using tuple_type = column_type *;
using tuple_size_t = u64;

typedef void (*tuple_generator_hook)(tuple_type, tuple_type, tuple_type);
typedef void (*tuple_copy_hook)(tuple_type, tuple_type);
typedef bool (*tuple_predicate)(tuple_type);

static_assert(sizeof(column_type) == 8, "column_type must be 64-bit (LP64)");
