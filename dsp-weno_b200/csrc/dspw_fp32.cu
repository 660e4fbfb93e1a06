// FP32 form: FP32 state, fluxes and reconstruction; DSP-WENO layers as BF16
// tensor-core MMA with FP32 accumulation.  Compiled with FMA contraction.
#define DSPW_T float
#include "dspw_precision.inc"
