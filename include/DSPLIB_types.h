/*
 * Common types of the DSPLIB C API (status codes, function style, handle).
 *
 * Drop-in replacement for src/common/DSPLIB_types.h of the reference: status
 * values (DSPLIB_types.h:174-194), the handle type (:196) and the function
 * styles (:199-204) keep their numeric values.
 *
 * DSPLIB_MMA_SIZE_* name the panel width that callers pass in
 * DSPLIB_fir_InitArgs.MMA_SIZE; on this library it only fixes the padded
 * filter-buffer layout used when enableMMA = 1 (2*MMA_SIZE leading zeros,
 * see DSPLIB_fir_getSizes).  The values are those of a 256-bit MMA device.
 */
#ifndef COMMON_DSPLIB_TYPES_H_
#define COMMON_DSPLIB_TYPES_H_

#include <inttypes.h>
#include <stddef.h>
#include <stdint.h>

#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef double DSPLIB_D64;
typedef float DSPLIB_F32;

typedef enum {
   DSPLIB_SUCCESS = 0,
   DSPLIB_ERR_FAILURE = 1,
   DSPLIB_ERR_INVALID_VALUE = 2,
   DSPLIB_ERR_INVALID_TYPE = 3,
   DSPLIB_ERR_INVALID_DIMENSION = 4,
   DSPLIB_ERR_NULL_POINTER = 5,
   DSPLIB_ERR_NOT_IMPLEMENTED = 6,
   DSPLIB_ERR_NOT_EQUAL_WIDTH_STRIDE = 7,
   DSPLIB_ERR_NOT_ALIGNED_PTRS_STRIDES = 8,
   DSPLIB_ERR_NOT_ALIGNED_WIDTHS = 9,
   DSPLIB_ERR_BUFFER_TOO_SMALL = 10,
   DSPLIB_ERR_INVALID_ACTIVATION = 11,
   DSPLIB_ERR_INVALID_SHIFT = 12,
   DSPLIB_ERROR_MAX = 13,
   DSPLIB_ERR_INVALID_MMA_FLAG = 14,
} DSPLIB_STATUS_NAME;

typedef DSPLIB_STATUS_NAME DSPLIB_STATUS;

typedef void *DSPLIB_kernelHandle;

typedef enum {
   DSPLIB_FUNCTION_NATC = 0,
   DSPLIB_FUNCTION_OPTIMIZED,
   DSPLIB_FUNCTION_MAX = 128
} DSPLIB_FUNCTION_STYLE;

#define DSPLIB_PARAM_SIZE 128

#define DSPLIB_min(x, y) (((x) < (y)) ? (x) : (y))
#define DSPLIB_max(x, y) (((x) < (y)) ? (y) : (x))
#define DSPLIB_ceilingDiv(x, y) (((x) + (y) -1) / (y))

#define DSPLIB_MMA_SIZE_8_BIT 32
#define DSPLIB_MMA_SIZE_16_BIT 16
#define DSPLIB_MMA_SIZE_32_BIT 8

#ifdef __cplusplus
}
#endif

#endif /* COMMON_DSPLIB_TYPES_H_ */
