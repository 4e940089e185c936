// CPU driver of csrc/hb_once.h: the per-device "set once" cache of kernel
// attributes, with a fake setter that counts calls per (device, kernel).
#include <map>
#include <utility>

#include "hb_once.h"

namespace {
hb::PerDeviceOnce g_once;
std::map<std::pair<int, const void *>, int> g_calls;
int g_fail_next = 0;
}  // namespace

extern "C" {
// Runs the cache for (dev, key); the fake setter fails (returns -2) when a
// failure was armed with once_fail_next.  Returns the cache's result.
int once_run(int dev, long key) {
  const void *k = reinterpret_cast<const void *>(key);
  return g_once.run(dev, k, [&]() -> int {
    g_calls[{dev, k}]++;
    if (g_fail_next) {
      g_fail_next = 0;
      return -2;
    }
    return 0;
  });
}
int once_calls(int dev, long key) {
  const auto it = g_calls.find({dev, reinterpret_cast<const void *>(key)});
  return it == g_calls.end() ? 0 : it->second;
}
void once_fail_next() { g_fail_next = 1; }
int once_size() { return (int)g_once.size(); }
}
