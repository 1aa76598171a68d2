// Internal host-side declarations shared by the CUDA translation units of
// libdrb.  Not part of the public C-ABI (include/drb.h is).
#pragma once

#include "../../include/drb.h"
#include <cuda_runtime.h>
#include <cstddef>

namespace drb
{

// Keep the device's default memory pool reserved across synchronisations.
void keep_pool_reserved ();

// Stream-ordered scratch allocation; all scratch is freed before a public
// entry point returns (stream-ordered, so no synchronisation is implied).
struct Scratch
{
  cudaStream_t stream;
  void *ptrs[32];
  int n = 0;
  cudaError_t err = cudaSuccess;
  explicit Scratch (cudaStream_t s) : stream (s) { keep_pool_reserved (); }
  template <typename T> T *alloc (size_t count)
  {
    if (err != cudaSuccess || n >= 32) return nullptr;
    void *p = nullptr;
    err = cudaMallocAsync (&p, count * sizeof (T) + 16, stream);
    if (err != cudaSuccess) return nullptr;
    ptrs[n++] = p;
    return static_cast<T *> (p);
  }
  ~Scratch ()
  {
    for (int i = 0; i < n; ++i) cudaFreeAsync (ptrs[i], stream);
  }
};

inline int status_from (cudaError_t e)
{
  if (e == cudaSuccess) return DRB_OK;
  if (e == cudaErrorMemoryAllocation) return DRB_ERR_OOM;
  return DRB_ERR_CUDA;
}

void set_last_error (const char *msg);
int check_launch (const char *what);

// radix sort of (key, value) pairs on the low `bits` bits of the keys
int radix_sort_pairs (const unsigned *keys_in, const int *vals_in, unsigned *keys_out,
                      int *vals_out, int n, int bits, cudaStream_t stream);
// exclusive prefix sum of n int32 values (in may equal out); total -> *d_total if non-null
int exclusive_scan_i32 (const int *in, int *out, int n, int *d_total, cudaStream_t stream);

inline int div_up (long long a, long long b) { return (int)((a + b - 1) / b); }

// Workspace of the allocation-free radix sort (sizes from radix_ws_counts
// and scan_ws_ints; kbuf/vbuf hold n elements).
struct RadixWorkspace
{
  unsigned *kbuf;
  int *vbuf;
  int *counts;
  int *scan_tmp;
};
long long radix_ws_counts (int n);
int scan_ws_ints (int n);
int exclusive_scan_i32_ws (const int *in, int *out, int n, int *d_total, int *tmp, cudaStream_t s);
int radix_sort_pairs_ws (const unsigned *keys_in, const int *vals_in, unsigned *keys_out,
                         int *vals_out, int n, int bits, const RadixWorkspace &ws, cudaStream_t s);
// Batched locate with every scratch buffer supplied by the caller.
struct LocateWorkspace
{
  int *head;
  unsigned *codes;
  unsigned *codes_sorted;
  int *iota;
  int *order;
  RadixWorkspace radix;
  int *hist; // query_cell_count() cell counts of the query order
};
// Cells of the query order (counting sort over Morton cells).
int query_cell_count ();
int locate_batched_ws (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                       const drb_newton_opts *opts, const drb_locate_config *cfg,
                       const LocateWorkspace &ws, int *cell, float *ref, drb_query_stats stats,
                       cudaStream_t s);

int sm_count ();

// Dofs per element of a mesh of either shape (drb_elem_dofs).
int mesh_nd (const drb_mesh *m);

} // namespace drb
