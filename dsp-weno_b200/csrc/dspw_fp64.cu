// FP64 plain form.  Compiled with --fmad=false so every multiply and add rounds
// separately, as in the reference's x86-64 build.
#define DSPW_T double
#include "dspw_precision.inc"
