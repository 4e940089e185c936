// hb_once.h -- "once per device" for per-device CUDA settings.
//
// A kernel's dynamic shared-memory limit (cudaFuncSetAttribute) belongs to the
// kernel on one device: a process that drives two GPUs must set it on each.
// PerDeviceOnce runs a setter the first time a (device, key) pair is seen and
// remembers it only when the setter succeeded.  Plain C++ (no CUDA types), so
// that a CPU test can drive it with a fake setter.
#pragma once

#include <mutex>
#include <set>
#include <utility>

namespace hb {

class PerDeviceOnce {
 public:
  // Runs set() unless (dev, key) already succeeded; returns set()'s code (0 =
  // success) or 0 when nothing had to be done.
  template <typename Set>
  int run(int dev, const void *key, Set set) {
    std::lock_guard<std::mutex> lock(mu_);
    const auto k = std::make_pair(dev, key);
    if (done_.count(k)) return 0;
    const int rc = set();
    if (rc == 0) done_.insert(k);
    return rc;
  }
  size_t size() {
    std::lock_guard<std::mutex> lock(mu_);
    return done_.size();
  }

 private:
  std::mutex mu_;
  std::set<std::pair<int, const void *>> done_;
};

}  // namespace hb
