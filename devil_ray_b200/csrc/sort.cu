// Stable LSD radix sort of (uint32 key, int32 value) pairs and an int32
// exclusive scan, hand-written for sm_100a.  Replaces the host std::sort of
// the reference's LBVH build (linear_bvh_builder.cpp:120-135) and the RAJA
// exclusive_scan of its compactions (array_utils.hpp:171-270).
//
// Sort pass (8-bit digit):
//   hist_kernel     per-tile digit histogram in shared memory, written
//                   digit-major so one exclusive scan gives every tile's
//                   global base per digit
//   scan            exclusive_scan_i32 over 256 x tiles counts
//   scatter_kernel  per tile, items ranked in original order: rounds of one
//                   item per thread; within a warp __match_any_sync gives the
//                   peers with the same digit, per-warp counts are prefixed
//                   across warps in shared memory, so equal keys keep their
//                   input order (stability), which makes the result
//                   deterministic run to run.
#include "drb_common.cuh"
#include "drb_internal.h"

namespace drb
{
namespace
{
constexpr int kSortBlock = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kSortWarps = kSortBlock / kWarp;
constexpr int kRadix = 256;

__global__ void __launch_bounds__ (kSortBlock)
hist_kernel (const unsigned *__restrict__ keys, int n, int shift, int ntiles, int *__restrict__ counts)
{
  __shared__ int hist[kRadix];
  hist[threadIdx.x] = 0;
  __syncthreads ();
  const long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j)
  {
    const long long idx = base + (long long)j * kSortBlock + threadIdx.x;
    if (idx < n) atomicAdd (&hist[(keys[idx] >> shift) & 0xffu], 1);
  }
  __syncthreads ();
  counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__ (kSortBlock)
scatter_kernel (const unsigned *__restrict__ keys_in, const int *__restrict__ vals_in,
                unsigned *__restrict__ keys_out, int *__restrict__ vals_out, int n, int shift,
                int ntiles, const int *__restrict__ offsets)
{
  __shared__ int base_off[kRadix];
  __shared__ int running[kRadix];
  __shared__ int wcnt[kSortWarps][kRadix];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  base_off[tid] = offsets[(size_t)tid * ntiles + blockIdx.x];
  running[tid] = 0;
  const unsigned lt_mask = (1u << lane) - 1u;
  const long long base = (long long)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j)
  {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) wcnt[w][tid] = 0;
    const long long idx = base + (long long)j * kSortBlock + tid;
    const bool valid = idx < n;
    unsigned key = 0;
    int val = 0;
    int digit = kRadix; // sentinel groups the invalid lanes together
    if (valid)
    {
      key = keys_in[idx];
      val = vals_in[idx];
      digit = (key >> shift) & 0xffu;
    }
    const unsigned peers = __match_any_sync (0xffffffffu, digit);
    const int rank = __popc (peers & lt_mask);
    const int leader = __ffs (peers) - 1;
    __syncthreads ();
    if (valid && lane == leader) wcnt[warp][digit] = __popc (peers);
    __syncthreads ();
    {
      int acc = running[tid];
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w)
      {
        const int t = wcnt[w][tid];
        wcnt[w][tid] = acc;
        acc += t;
      }
      running[tid] = acc;
    }
    __syncthreads ();
    if (valid)
    {
      const int pos = base_off[digit] + wcnt[warp][digit] + rank;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads ();
  }
}

// ---- exclusive scan (three phases, recursive on the block sums) ----
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

DRB_D int block_exclusive_scan (int v, int *total)
{
  __shared__ int warp_sums[kScanBlock / kWarp];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    const int y = __shfl_up_sync (0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads ();
  if (warp == 0)
  {
    int s = (lane < kScanBlock / kWarp) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
      const int y = __shfl_up_sync (0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanBlock / kWarp) warp_sums[lane] = s;
  }
  __syncthreads ();
  const int warp_prefix = (warp > 0) ? warp_sums[warp - 1] : 0;
  if (total) *total = warp_sums[kScanBlock / kWarp - 1];
  __syncthreads ();
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__ (kScanBlock)
scan_reduce_kernel (const int *__restrict__ in, int n, int *__restrict__ block_sums)
{
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) s += in[base + j];
  int total;
  block_exclusive_scan (s, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__ (kScanBlock)
scan_apply_kernel (const int *in, int *out, int n, const int *__restrict__ block_offsets,
                   int *d_total, int nblocks)
{
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
  {
    v[j] = (base + j < n) ? in[base + j] : 0;
    s += v[j];
  }
  int total;
  int prefix = block_exclusive_scan (s, &total);
  prefix += block_offsets ? block_offsets[blockIdx.x] : 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
  {
    if (base + j < n) out[base + j] = prefix;
    prefix += v[j];
  }
  if (d_total && blockIdx.x == nblocks - 1 && threadIdx.x == kScanBlock - 1) *d_total = prefix;
}

} // namespace

int exclusive_scan_i32 (const int *in, int *out, int n, int *d_total, cudaStream_t s)
{
  if (n <= 0)
  {
    if (d_total) cudaMemsetAsync (d_total, 0, sizeof (int), s);
    return DRB_OK;
  }
  const int nblocks = div_up (n, kScanTile);
  if (nblocks == 1)
  {
    scan_apply_kernel<<<1, kScanBlock, 0, s>>> (in, out, n, nullptr, d_total, 1);
    return check_launch ("scan_apply_kernel");
  }
  Scratch scr (s);
  int *sums = scr.alloc<int> (nblocks);
  if (!sums) return status_from (scr.err);
  scan_reduce_kernel<<<nblocks, kScanBlock, 0, s>>> (in, n, sums);
  int st = check_launch ("scan_reduce_kernel");
  if (st) return st;
  st = exclusive_scan_i32 (sums, sums, nblocks, nullptr, s);
  if (st) return st;
  scan_apply_kernel<<<nblocks, kScanBlock, 0, s>>> (in, out, n, sums, d_total, nblocks);
  return check_launch ("scan_apply_kernel");
}

int radix_sort_pairs (const unsigned *keys_in, const int *vals_in, unsigned *keys_out,
                      int *vals_out, int n, int bits, cudaStream_t s)
{
  if (n <= 0) return DRB_OK;
  const int ntiles = div_up (n, kSortTile);
  const int passes = (bits + 7) / 8;
  Scratch scr (s);
  int *counts = scr.alloc<int> ((size_t)kRadix * ntiles);
  unsigned *kbuf = scr.alloc<unsigned> (n);
  int *vbuf = scr.alloc<int> (n);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  // Ping-pong so that the last pass lands in keys_out/vals_out.
  const unsigned *ksrc = keys_in;
  const int *vsrc = vals_in;
  for (int p = 0; p < passes; ++p)
  {
    const bool last = (p == passes - 1);
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    unsigned *kdst = to_out ? keys_out : kbuf;
    int *vdst = to_out ? vals_out : vbuf;
    (void)last;
    hist_kernel<<<ntiles, kSortBlock, 0, s>>> (ksrc, n, 8 * p, ntiles, counts);
    int st = check_launch ("hist_kernel");
    if (st) return st;
    st = exclusive_scan_i32 (counts, counts, kRadix * ntiles, nullptr, s);
    if (st) return st;
    scatter_kernel<<<ntiles, kSortBlock, 0, s>>> (ksrc, vsrc, kdst, vdst, n, 8 * p, ntiles, counts);
    st = check_launch ("scatter_kernel");
    if (st) return st;
    ksrc = kdst;
    vsrc = vdst;
  }
  return DRB_OK;
}

// ---- variants over a caller-provided workspace (no allocation) ----

int scan_ws_ints (int n)
{
  int total = 0;
  while (n > kScanTile)
  {
    n = div_up (n, kScanTile);
    total += n;
  }
  return total + 1;
}

int exclusive_scan_i32_ws (const int *in, int *out, int n, int *d_total, int *tmp, cudaStream_t s)
{
  if (n <= 0)
  {
    if (d_total) cudaMemsetAsync (d_total, 0, sizeof (int), s);
    return DRB_OK;
  }
  const int nblocks = div_up (n, kScanTile);
  if (nblocks == 1)
  {
    scan_apply_kernel<<<1, kScanBlock, 0, s>>> (in, out, n, nullptr, d_total, 1);
    return check_launch ("scan_apply_kernel");
  }
  int *sums = tmp;
  scan_reduce_kernel<<<nblocks, kScanBlock, 0, s>>> (in, n, sums);
  int st = check_launch ("scan_reduce_kernel");
  if (st) return st;
  st = exclusive_scan_i32_ws (sums, sums, nblocks, nullptr, tmp + nblocks, s);
  if (st) return st;
  scan_apply_kernel<<<nblocks, kScanBlock, 0, s>>> (in, out, n, sums, d_total, nblocks);
  return check_launch ("scan_apply_kernel");
}

long long radix_ws_counts (int n) { return (long long)kRadix * div_up (n, kSortTile); }

int radix_sort_pairs_ws (const unsigned *keys_in, const int *vals_in, unsigned *keys_out,
                         int *vals_out, int n, int bits, const RadixWorkspace &ws, cudaStream_t s)
{
  if (n <= 0) return DRB_OK;
  const int ntiles = div_up (n, kSortTile);
  const int passes = (bits + 7) / 8;
  const unsigned *ksrc = keys_in;
  const int *vsrc = vals_in;
  for (int p = 0; p < passes; ++p)
  {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    unsigned *kdst = to_out ? keys_out : ws.kbuf;
    int *vdst = to_out ? vals_out : ws.vbuf;
    hist_kernel<<<ntiles, kSortBlock, 0, s>>> (ksrc, n, 8 * p, ntiles, ws.counts);
    int st = check_launch ("hist_kernel");
    if (st) return st;
    st = exclusive_scan_i32_ws (ws.counts, ws.counts, kRadix * ntiles, nullptr, ws.scan_tmp, s);
    if (st) return st;
    scatter_kernel<<<ntiles, kSortBlock, 0, s>>> (ksrc, vsrc, kdst, vdst, n, 8 * p, ntiles, ws.counts);
    st = check_launch ("scatter_kernel");
    if (st) return st;
    ksrc = kdst;
    vsrc = vdst;
  }
  return DRB_OK;
}

} // namespace drb

extern "C" int drb_radix_sort_pairs (const unsigned *keys_in, const int *vals_in,
                                     unsigned *keys_out, int *vals_out, int n, int bits,
                                     void *stream)
{
  if (n < 0 || bits < 1 || bits > 32 ||
      (n > 0 && (!keys_in || !vals_in || !keys_out || !vals_out)))
  {
    drb::set_last_error ("radix_sort_pairs: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n > 0 && (keys_in == keys_out || vals_in == vals_out))
  {
    drb::set_last_error ("radix_sort_pairs: in-place sort is not supported");
    return DRB_ERR_INVALID_ARG;
  }
  return drb::radix_sort_pairs (keys_in, vals_in, keys_out, vals_out, n, bits,
                                (cudaStream_t)stream);
}
