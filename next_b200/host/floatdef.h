// Precision of the host-side SoA lanes, as the reference selects it
// (include/floatdef.h:8-18).  The device path computes in FP64 state with
// either FP64 or FP32-mixed interactions whatever `real` is; NEXT_FP32 only
// narrows the host arrays.  FP64 is the default (the reference's only
// compiling precision).
#pragma once
#if defined(NEXT_FP32)
using real = float;
#else
using real = double;
#endif
