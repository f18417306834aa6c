// Precision of the host-side SoA lanes, selected as the reference selects it
// (include/floatdef.h:8-18): NEXT_FP64 gives double and takes precedence,
// NEXT_FP32 gives float.  Where neither is defined (the reference refuses to
// compile then) this build defaults to double, the reference's only
// compiling precision.  The device path computes in FP64 state with either
// FP64 or FP32-mixed interactions whatever `real` is; NEXT_FP32 only narrows
// the host arrays.
#pragma once
#if defined(NEXT_FP64)
using real = double;
#elif defined(NEXT_FP32)
using real = float;
#else
using real = double;
#endif
