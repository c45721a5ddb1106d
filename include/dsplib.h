/* Umbrella header, as src/dsplib.h of the reference (:19 biquad, :28 FIR, :11 addNCh, :24 deinterleave, :29 fltoq15, :31 interleave, :53 q15tofl). */
#ifndef DSPLIB_H_
#define DSPLIB_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"
#include "DSPLIB_addNCh.h"
#include "DSPLIB_cascadeBiquad.h"
#include "DSPLIB_deinterleave.h"
#include "DSPLIB_fir.h"
#include "DSPLIB_fltoq15.h"
#include "DSPLIB_interleave.h"
#include "DSPLIB_q15tofl.h"
#include "dsplib_gpu.h"

#endif
