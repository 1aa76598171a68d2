// Allocation-free batched point location.
//
// Some callers of this library cannot allocate device memory at the time they
// locate points: hosts whose device memory is owned by another allocator (a
// simulation code's pool, an in-situ framework) that forbids side
// allocations, or real-time paths where cudaMalloc's implicit
// synchronisation is not acceptable.  drb_locate_batched needs scratch
// memory (query Morton codes, the sort's ping-pong buffers and histograms,
// the work-queue counter) and obtains it with cudaMallocAsync.  This entry
// point runs the same computation with all of that scratch in one
// file-scope device array of fixed size instead, so it never allocates.
//
// Limits and sharing:
//   - at most kNoAllocMaxQueries queries per call (larger calls are rejected
//     with DRB_ERR_INVALID_ARG and a message);
//   - the array (about 20 MB) is part of this library's device code and stays
//     allocated on every device where it has been loaded, until the process
//     exits;
//   - every call on a device uses the same array: calls whose GPU work can
//     overlap (different streams without ordering, or several host threads)
//     race on it and must be serialised by the caller;
//   - the work-queue counter is cleared on the stream at every call; the
//     other buffers are fully overwritten before they are read.
#include "drb_internal.h"

#include <cstdio>
#include <mutex>

namespace drb
{
namespace
{

constexpr int kNoAllocMaxQueries = 1 << 20;
constexpr size_t kAlign = 256;

constexpr size_t align_up (size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kQBytes = align_up (sizeof (int) * (size_t)kNoAllocMaxQueries);
constexpr size_t kHeadOff = 0;
constexpr size_t kCodesOff = kHeadOff + kAlign;
constexpr size_t kIotaOff = kCodesOff + kQBytes;
constexpr size_t kOrderOff = kIotaOff + kQBytes;
// cell counts of the query order (2^21 Morton cells), then the block sums
// of their scan
constexpr size_t kCellInts = 1u << 21;
constexpr size_t kHistOff = kOrderOff + kQBytes;
constexpr size_t kScanOff = kHistOff + align_up (sizeof (int) * kCellInts);
constexpr size_t kScanInts = 4096;
constexpr size_t kScratchBytes = kScanOff + align_up (sizeof (int) * kScanInts);

// The scratch itself.  Host code must not use this name as an address: on
// the host it is only a stand-in for the symbol; the device address comes
// from cudaGetSymbolAddress below.
static __device__ __align__ (256) unsigned char g_locate_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char *g_dev_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (with that device current) and cached.
int scratch_for_current_device (unsigned char **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice (&dev);
  if (e != cudaSuccess)
  {
    set_last_error (cudaGetErrorString (e));
    return status_from (e);
  }
  if (dev < 0 || dev >= kMaxDevices)
  {
    set_last_error ("locate_batched_noalloc: device ordinal out of range");
    return DRB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock (g_mutex);
  if (!g_dev_ptr[dev])
  {
    void *p = nullptr;
    e = cudaGetSymbolAddress (&p, g_locate_scratch);
    if (e != cudaSuccess || !p)
    {
      char buf[256];
      std::snprintf (buf, sizeof (buf), "locate_batched_noalloc: cudaGetSymbolAddress: %s",
                     cudaGetErrorString (e));
      set_last_error (buf);
      return e != cudaSuccess ? status_from (e) : DRB_ERR_CUDA;
    }
    g_dev_ptr[dev] = static_cast<unsigned char *> (p);
  }
  *out = g_dev_ptr[dev];
  return DRB_OK;
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_noalloc_max_queries (void) { return kNoAllocMaxQueries; }

extern "C" int drb_locate_batched_noalloc (const drb_mesh *mesh, const drb_bvh *bvh,
                                           const float *pts, int n, const drb_newton_opts *opts,
                                           const drb_locate_config *cfg, int *cell, float *ref,
                                           drb_query_stats stats, void *stream)
{
  if (n > kNoAllocMaxQueries)
  {
    char buf[200];
    std::snprintf (buf, sizeof (buf),
                   "locate_batched_noalloc: %d queries exceed the fixed scratch capacity of %d "
                   "queries per call; split the call or use drb_locate_batched",
                   n, kNoAllocMaxQueries);
    set_last_error (buf);
    return DRB_ERR_INVALID_ARG;
  }
  if (n < 0)
  {
    set_last_error ("locate_batched_noalloc: negative query count");
    return DRB_ERR_INVALID_ARG;
  }
  unsigned char *base = nullptr;
  int st = scratch_for_current_device (&base);
  if (st) return st;
  LocateWorkspace ws{};
  ws.head = reinterpret_cast<int *> (base + kHeadOff);
  ws.codes = reinterpret_cast<unsigned *> (base + kCodesOff);
  ws.iota = reinterpret_cast<int *> (base + kIotaOff);
  ws.order = reinterpret_cast<int *> (base + kOrderOff);
  ws.hist = reinterpret_cast<int *> (base + kHistOff);
  ws.radix.scan_tmp = reinterpret_cast<int *> (base + kScanOff);
  if ((size_t)query_cell_count () != kCellInts || scan_ws_ints ((int)kCellInts) > (int)kScanInts)
  {
    set_last_error ("locate_batched_noalloc: scratch layout does not match the query order");
    return DRB_ERR_UNSUPPORTED;
  }
  return locate_batched_ws (mesh, bvh, pts, n, opts, cfg, ws, cell, ref, stats,
                            (cudaStream_t)stream);
}
