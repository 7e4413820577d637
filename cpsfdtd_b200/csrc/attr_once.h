// attr_once.h -- a per-device "set once" flag for kernel attributes (host
// code, no CUDA types).
//
// cudaFuncSetAttribute (the dynamic shared-memory size and carveout a kernel
// needs before a launch above 48 KiB) applies to the current device only, so
// the flag is kept per device: bit d of `done` says the attribute is set on
// device d.  Threads may race to set it; the attribute call is idempotent, so
// the race only repeats it.  A failed call leaves the bit clear (the next
// launch retries) and its error is returned to the caller.  Devices 64 and up
// have no bit and are set on every call.
//
//   get_device(int *dev) -> int  (0 on success)   e.g. cudaGetDevice
//   apply() -> int               (0 on success)   e.g. cudaFuncSetAttribute
#pragma once

#include <stdint.h>

#include <atomic>

namespace cps {

template <typename GetDevice, typename Apply>
int attr_once_per_device(std::atomic<uint64_t> &done, GetDevice &&get_device, Apply &&apply)
{
    int dev = 0;
    const int e = get_device(&dev);
    if (e != 0) return e;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t{1} << dev) : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return 0;
    const int r = apply();
    if (r == 0 && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return r;
}

}  // namespace cps
