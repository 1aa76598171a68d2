// Point location from and to host memory, with the copies overlapped.
//
// Mesh::locate takes an Array<Vec3> that may live on the host
// (unstructured_mesh.cpp:124-148 reads it through get_device_ptr, one
// synchronous copy in, one out).  Here the batch is cut into chunks that
// cycle through three streams: while one chunk's Location records go back
// to the host, the next chunk is Morton-sorted and located and the one after
// it is copied in, so both copy engines and the SMs work at the same time.
// Each stream owns its device buffers, and stream order keeps a chunk from
// overwriting buffers that an earlier chunk on the same stream still uses.
// Host buffers should be page-locked; with pageable memory the result is
// the same but the copies do not overlap.  The call returns when the
// results are in host memory.
#include "drb_internal.h"

namespace drb
{
namespace
{

constexpr int kLanes = 3;
constexpr int kDefaultChunk = 1 << 21;

struct Lane
{
  cudaStream_t s = nullptr;
  cudaEvent_t ready = nullptr;
  float *pts = nullptr;
  int *cell = nullptr;
  float *ref = nullptr;
  LocateWorkspace ws{};
};

// Streams and device buffers of the lanes, allocated from the device's
// stream-ordered pool; false (and the error set) if anything failed.
bool open_lanes (Lane (&lane)[kLanes], int chunk, cudaEvent_t start, cudaError_t &e)
{
  const int cells = query_cell_count ();
  const int scan_ints = scan_ws_ints (cells);
  const size_t q = (size_t)chunk;
  for (int l = 0; l < kLanes && e == cudaSuccess; ++l)
  {
    e = cudaStreamCreateWithFlags (&lane[l].s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags (&lane[l].ready, cudaEventDisableTiming);
    // work queued on the caller's stream before this call comes first
    if (e == cudaSuccess) e = cudaStreamWaitEvent (lane[l].s, start, 0);
    void *p[9] = {};
    const size_t bytes[9] = { 3 * q * sizeof (float), q * sizeof (int), 3 * q * sizeof (float),
                              sizeof (int), q * sizeof (unsigned), q * sizeof (int),
                              q * sizeof (int), sizeof (int) * (size_t)cells,
                              sizeof (int) * (size_t)scan_ints };
    for (int b = 0; b < 9 && e == cudaSuccess; ++b) e = cudaMallocAsync (&p[b], bytes[b], lane[l].s);
    lane[l].pts = (float *)p[0];
    lane[l].cell = (int *)p[1];
    lane[l].ref = (float *)p[2];
    lane[l].ws.head = (int *)p[3];
    lane[l].ws.codes = (unsigned *)p[4];
    lane[l].ws.iota = (int *)p[5];
    lane[l].ws.order = (int *)p[6];
    lane[l].ws.hist = (int *)p[7];
    lane[l].ws.radix.scan_tmp = (int *)p[8];
  }
  if (e != cudaSuccess) set_last_error (cudaGetErrorString (e));
  return e == cudaSuccess;
}

// Free the lanes' buffers in stream order, make the caller's stream wait for
// them, then wait on the host; returns the first error met.
int close_lanes (Lane (&lane)[kLanes], cudaStream_t caller, int st)
{
  for (int l = 0; l < kLanes; ++l)
  {
    if (!lane[l].s) continue;
    void *bufs[9] = { lane[l].pts, lane[l].cell, lane[l].ref, lane[l].ws.head, lane[l].ws.codes,
                      lane[l].ws.iota, lane[l].ws.order, lane[l].ws.hist,
                      lane[l].ws.radix.scan_tmp };
    for (void *b : bufs)
      if (b) cudaFreeAsync (b, lane[l].s);
    if (lane[l].ready)
    {
      cudaEventRecord (lane[l].ready, lane[l].s);
      cudaStreamWaitEvent (caller, lane[l].ready, 0);
    }
  }
  for (int l = 0; l < kLanes; ++l)
  {
    if (!lane[l].s) continue;
    const cudaError_t se = cudaStreamSynchronize (lane[l].s);
    if (se != cudaSuccess && st == DRB_OK)
    {
      set_last_error (cudaGetErrorString (se));
      st = status_from (se);
    }
    if (lane[l].ready) cudaEventDestroy (lane[l].ready);
    cudaStreamDestroy (lane[l].s);
  }
  return st;
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_locate_host (const drb_mesh *mesh, const drb_bvh *bvh, const float *host_pts,
                                int n, const drb_newton_opts *opts, const drb_locate_config *cfg,
                                int chunk, int *host_cell, float *host_ref, void *stream)
{
  if (!mesh || !bvh || !opts || n < 0 || (n > 0 && (!host_pts || !host_cell || !host_ref)))
  {
    set_last_error ("locate_host: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  keep_pool_reserved ();
  if (chunk <= 0) chunk = kDefaultChunk;
  if (chunk > n) chunk = n;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaEvent_t start = nullptr;
  cudaError_t e = cudaEventCreateWithFlags (&start, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord (start, caller);
  Lane lane[kLanes];
  int st = DRB_OK;
  if (e != cudaSuccess)
  {
    set_last_error (cudaGetErrorString (e));
    st = status_from (e);
  }
  else if (!open_lanes (lane, chunk, start, e))
  {
    st = status_from (e);
  }
  drb_locate_config c = cfg ? *cfg : drb_locate_config{ 128, 0, 64, 1, 0 };
  c.sort_queries = 1; // the workspace path sorts each chunk
  for (long long off = 0, k = 0; off < n && st == DRB_OK; off += chunk, ++k)
  {
    Lane &L = lane[k % kLanes];
    const int m = (int)((n - off) < chunk ? (n - off) : chunk);
    e = cudaMemcpyAsync (L.pts, host_pts + 3 * off, sizeof (float) * 3 * (size_t)m,
                         cudaMemcpyHostToDevice, L.s);
    if (e == cudaSuccess)
    {
      st = locate_batched_ws (mesh, bvh, L.pts, m, opts, &c, L.ws, L.cell, L.ref,
                              drb_query_stats{ nullptr, nullptr, nullptr }, L.s);
      if (st) break;
      e = cudaMemcpyAsync (host_cell + off, L.cell, sizeof (int) * (size_t)m,
                           cudaMemcpyDeviceToHost, L.s);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync (host_ref + 3 * off, L.ref, sizeof (float) * 3 * (size_t)m,
                           cudaMemcpyDeviceToHost, L.s);
    if (e != cudaSuccess)
    {
      set_last_error (cudaGetErrorString (e));
      st = status_from (e);
    }
  }
  st = close_lanes (lane, caller, st);
  if (start) cudaEventDestroy (start);
  return st;
}
