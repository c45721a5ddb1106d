/*
 * Host stand-in for the TI C7x compiler header <c7x.h>.
 *
 * Test infrastructure only: it lets the reference's natural-C (_cn) sources
 * for DSPLIB_fir and DSPLIB_cascadeBiquad compile with g++ on x86 so that they
 * can serve as the parity oracle.  It declares only what those sources and the
 * headers they include touch: opaque streaming-engine / MMA register structs
 * (never dereferenced by the _cn code), the MMA panel width macro and the two
 * 64-bit shift intrinsics used by DSPLIB_int128_t.  TI's own host-emulation
 * package (which would normally provide this header) is not installed.
 */
#ifndef ORACLE_SHIM_C7X_H_
#define ORACLE_SHIM_C7X_H_

#include <stdint.h>

/* Opaque hardware templates: sized like the real ones (64-byte parameter
 * blocks), contents unused by the natural-C kernels. */
typedef struct { uint64_t w[8]; } __SE_TEMPLATE_v1;
typedef struct { uint64_t w[8]; } __SA_TEMPLATE_v1;
typedef struct { uint64_t w[8]; } __HWA_CONFIG_REG_v1;
typedef struct { uint64_t w[8]; } __HWA_OFFSET_REG;

#define SE_PARAM_SIZE 64

/* MMA panel width in elements for a C7504-class (256-bit MMAv2) device:
 * 32 bytes of A-matrix columns. */
#define __MMA_A_COLS(eltsize) (32 / (eltsize))

static inline uint64_t __shift_left(uint64_t v, uint32_t s) { return v << s; }
static inline uint64_t __shift_right(uint64_t v, uint32_t s) { return v >> s; }

#endif
