// Error reporting and small shared helpers of the C-ABI (include/drb.h).
#include "drb_internal.h"

#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

namespace drb
{
namespace
{
thread_local std::string g_last_error;
}

void set_last_error (const char *msg) { g_last_error = msg ? msg : ""; }

namespace
{
std::atomic<unsigned long long> g_launches{ 0 };
}

int check_launch (const char *what)
{
  ++g_launches;
  const cudaError_t e = cudaGetLastError ();
  if (e == cudaSuccess) return DRB_OK;
  char buf[512];
  std::snprintf (buf, sizeof (buf), "%s: %s", what, cudaGetErrorString (e));
  set_last_error (buf);
  return status_from (e);
}

// The scratch of every entry point comes from the device's default
// stream-ordered pool.  With the pool's default release threshold (0) the
// memory goes back to the driver at every synchronisation, and the next
// call maps it again; calls that synchronise (drb_locate_host, the build)
// would pay that each time.  Keep it reserved instead, once per device.
void keep_pool_reserved ()
{
  static std::atomic<unsigned long long> done{ 0 };
  int dev = 0;
  if (cudaGetDevice (&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  const unsigned long long bit = 1ull << dev;
  if (done.load (std::memory_order_relaxed) & bit) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool (&pool, dev) == cudaSuccess)
  {
    unsigned long long threshold = ~0ull;
    cudaMemPoolSetAttribute (pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  done.fetch_or (bit);
}

// SM count of the current device, looked up once per device ordinal, so
// persistent grids are sized for the device they launch on.
int sm_count ()
{
  static std::atomic<int> cached[64] = {};
  int dev = 0;
  if (cudaGetDevice (&dev) != cudaSuccess) dev = 0;
  if (dev < 0 || dev >= 64)
  {
    int v = 0;
    cudaDeviceGetAttribute (&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }
  int c = cached[dev].load (std::memory_order_relaxed);
  if (c == 0)
  {
    int v = 0;
    cudaDeviceGetAttribute (&v, cudaDevAttrMultiProcessorCount, dev);
    c = v > 0 ? v : 148;
    cached[dev].store (c, std::memory_order_relaxed);
  }
  return c;
}

} // namespace drb

extern "C" const char *drb_last_error (void) { return drb::g_last_error.c_str (); }

extern "C" int drb_version (void) { return 1; }

extern "C" unsigned long long drb_kernel_launches (void) { return drb::g_launches.load (); }
