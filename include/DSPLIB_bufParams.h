/*
 * Buffer descriptors and element types of the DSPLIB C API.
 *
 * Drop-in replacement for src/common/DSPLIB_bufParams.h of the reference:
 * the enum values (DSPLIB_bufParams.h:22-48), the descriptor field order
 * (:77-85) and DSPLIB_sizeof (:135) must be identical so that existing callers
 * compile and link unchanged.
 */
#ifndef DSPLIB_BUFPARAMS_H_
#define DSPLIB_BUFPARAMS_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum _DSPLIB_data_type_e {
   DSPLIB_INT8 = 0,
   DSPLIB_INT16 = 1,
   DSPLIB_INT32 = 2,
   DSPLIB_INT64 = 3,
   DSPLIB_INT128 = 4,
   DSPLIB_UINT8 = 5,
   DSPLIB_UINT16 = 6,
   DSPLIB_UINT24 = 7,
   DSPLIB_UINT32 = 8,
   DSPLIB_UINT64 = 9,
   DSPLIB_UINT128 = 10,
   DSPLIB_FLOAT16 = 11,
   DSPLIB_FLOAT32 = 12,
   DSPLIB_FLOAT64 = 13,
   DSPLIB_CINT16 = 14,
   DSPLIB_CINT32 = 15,
   DSPLIB_CINT64 = 16,
   DSPLIB_CFLOAT32 = 17,
   DSPLIB_CFLOAT64 = 18,
} DSPLIB_data_type_e;

#define DSPLIB_ISSIGNED(type) ((type) < DSPLIB_UINT8 || (type) > DSPLIB_UINT128)

typedef enum _DSPLIB_dimension_e {
   DSPLIB_2D = 0,
   DSPLIB_3D = 1,
   DSPLIB_4D = 2,
   DSPLIB_5D = 3,
   DSPLIB_6D = 4
} DSPLIB_dimension_e;

/** One-dimensional buffer: element type and length. */
typedef struct {
   uint32_t data_type; /**< DSPLIB_data_type_e */
   uint32_t dim_x;     /**< elements */
} DSPLIB_bufParams1D_t;

/** Two-dimensional buffer: rows of dim_x elements, stride_y BYTES apart. */
typedef struct {
   uint32_t data_type; /**< DSPLIB_data_type_e */
   uint32_t dim_x;     /**< elements per row */
   uint32_t dim_y;     /**< rows */
   int32_t stride_y;   /**< bytes between rows */
} DSPLIB_bufParams2D_t;

typedef struct {
   uint32_t data_type;
   uint32_t dim_x;
   uint32_t dim_y;
   int32_t stride_y;
   uint32_t dim_z;
   int32_t stride_z;
} DSPLIB_bufParams3D_t;

typedef struct {
   uint32_t data_type;
   uint32_t dim_0;
   uint32_t dim_1;
   int32_t stride_1;
   uint32_t dim_2;
   int32_t stride_2;
   uint32_t dim_3;
   int32_t stride_3;
   uint32_t dim_4;
   int32_t stride_4;
   uint32_t dim_5;
   int32_t stride_5;
   uint32_t dimension;
} DSPLIB_bufParamsND_t;

/** Bytes per element of a DSPLIB_data_type_e (1 for unknown types, as the reference). */
static inline int32_t DSPLIB_sizeof(uint32_t type)
{
   switch (type) {
   case DSPLIB_INT8:
   case DSPLIB_UINT8: return 1;
   case DSPLIB_INT16:
   case DSPLIB_UINT16:
   case DSPLIB_FLOAT16: return 2;
   case DSPLIB_UINT24: return 3;
   case DSPLIB_INT32:
   case DSPLIB_UINT32:
   case DSPLIB_FLOAT32:
   case DSPLIB_CINT16: return 4;
   case DSPLIB_INT64:
   case DSPLIB_UINT64:
   case DSPLIB_FLOAT64:
   case DSPLIB_CFLOAT32:
   case DSPLIB_CINT32: return 8;
   case DSPLIB_INT128:
   case DSPLIB_UINT128:
   case DSPLIB_CFLOAT64:
   case DSPLIB_CINT64: return 16;
   default: return 1;
   }
}

#ifdef __cplusplus
}
#endif

#endif /* DSPLIB_BUFPARAMS_H_ */
