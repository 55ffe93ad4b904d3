// Device index checks of the bounds-check build.
//
// Compiled with -DJC_BOUNDS_CHECK (build.py --bounds-check, which writes
// libjc_layout_bc.so), JC_IN_BOUNDS(i, lim, err) tests i < lim where a kernel
// is about to index memory through a value it loaded (a neighbour id, a body
// index, a tree node index, a sort destination). A failed check records
// JC_ERR_BOUNDS in the given device error word (first error wins) and the
// caller skips the access; nothing traps. In the normal build the macro is the
// constant `true` and costs nothing.
#pragma once

#include <cstdint>

#include "../../include/jc_layout.h"

namespace jc {

__device__ __forceinline__ bool bounds_ok(bool ok, uint32_t* err) {
  if (!ok && err) atomicCAS(err, 0u, (uint32_t)JC_ERR_BOUNDS);
  return ok;
}

}  // namespace jc

#ifdef JC_BOUNDS_CHECK
#define JC_IN_BOUNDS(i, lim, err) (::jc::bounds_ok((uint64_t)(i) < (uint64_t)(lim), (err)))
#define JC_BOUNDS_BUILD 1
#else
#define JC_IN_BOUNDS(i, lim, err) true
#define JC_BOUNDS_BUILD 0
#endif
