/* FP64 instantiation of the Stokes oracle.  TEST INFRASTRUCTURE ONLY. */
#include "fi_oracle.h"
#define REAL double
#define SUF _f64
#include "stokes_impl.h"
