// variant.h - the build variant of an engine translation unit.
//
// The engine templates are compiled more than once with different
// arithmetic (FP64 bit-for-bit with the reference, FP64 fast, FP32).  Each
// translation unit names its variant before including the engine, and every
// engine symbol then lives in lare::<variant> (an inline namespace), so that
// host launch stubs and kernels of two variants never share a mangled name
// and the linker cannot merge one variant's code into another's.
//
//   LARE_VARIANT  inline namespace of this unit (default: base)
//   LARE_FAST     1: the unit is not bound to the reference's exact
//                 arithmetic, so quotients may be formed from shared or
//                 approximate reciprocals (fast_rcp / fdiv in common.cuh)
#pragma once

#ifndef LARE_VARIANT
#define LARE_VARIANT base
#endif
#ifndef LARE_FAST
#define LARE_FAST 0
#endif

#define LARE_BEGIN \
  namespace lare { \
  inline namespace LARE_VARIANT {
#define LARE_END \
  } \
  }
