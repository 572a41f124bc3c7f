// Optional device self-checks. Built with -DHPT_DEVICE_CHECKS, every index
// the kernels dereference is range-checked first; a failing check records
// its site and value in the error word (first failure wins) and the access
// is skipped. Normal builds compile the checks away.
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
