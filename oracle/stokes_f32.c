/* FP32 instantiation of the Stokes oracle.  TEST INFRASTRUCTURE ONLY. */
#include "fi_oracle.h"
#define REAL float
#define SUF _f32
#include "stokes_impl.h"
