/*
 * Host stand-in for the TI header <c7x_scalable.h> (test infrastructure only,
 * see c7x.h).  Provides the vector type names and the max_simd trait that
 * src/common/DSPLIB_types.h references; a 256-bit vector (C7504) is assumed.
 */
#ifndef ORACLE_SHIM_C7X_SCALABLE_H_
#define ORACLE_SHIM_C7X_SCALABLE_H_

#include <stddef.h>
#include <stdint.h>

namespace c7x {
struct uchar_vec { uint8_t s[32]; };
struct ushort_vec { uint16_t s[16]; };
template <typename T> struct max_simd { static constexpr size_t value = 32 / sizeof(T); };
}

#endif
