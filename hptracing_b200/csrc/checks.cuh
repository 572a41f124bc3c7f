// Device index guards. The library is built with -DHPT_DEVICE_CHECKS: every
// index a kernel dereferences is range-checked first; a failing check
// records its site and value in the error word (first failure wins), the
// access is skipped, and the host call returns HPT_ERR_INVALID_SCENE naming
// the site. Compiling without the define removes the guards (experiments
// only: that configuration is not shipped).
#pragma once

#include "device_types.h"
#include "dmath.cuh"

namespace hpt {

HPT_HD void record_fault(DevErr* e, int site, long long value) {
  if (!e) return;
#ifdef __CUDA_ARCH__
  if (atomicCAS(reinterpret_cast<int*>(&e->site), 0, site) == 0) e->value = value;
  atomicOr(&e->flags, 2u);
#else
  if (e->site == 0) {
    e->site = site;
    e->value = value;
  }
  e->flags |= 2u;
#endif
}

}  // namespace hpt

// Used as a statement: HPT_DCHECK(err, cond, site, value, on_fail);
// on_fail may be `continue` / `break` / `return ...` of the enclosing code.
#ifdef HPT_DEVICE_CHECKS
#define HPT_DCHECK(err, cond, site, value, on_fail)              \
  if (!(cond)) {                                                 \
    ::hpt::record_fault((err), (site), (long long)(value));      \
    on_fail;                                                     \
  } else                                                         \
    (void)0
#else
#define HPT_DCHECK(err, cond, site, value, on_fail) (void)0
#endif
