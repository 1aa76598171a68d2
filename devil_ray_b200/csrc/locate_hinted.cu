// Two-phase point location for the learned initial guess.
//
//   first_candidate_kernel  traverse each query (in Morton order) to its first
//                           candidate leaf in the reference's traversal order
//                           (device_mesh.hpp:248-318) without solving; the
//                           (query, element) pairs feed the guess network.
//                           With grid lists the first leaf comes from the
//                           query's cell (first_grid_candidate_kernel).
//   locate_hinted_kernel    persistent warps as in drb_locate_batched; a query
//                           first solves in its first candidate from the given
//                           guess (element-centre fallback), and only if that
//                           fails resumes the traversal from the root, skipping
//                           the already-tried first leaf.  Results equal
//                           drb_locate with DRB_GUESS_GIVEN: the same candidates
//                           are tried in the same order with the same guesses.
#include "drb_common.cuh"
#include "drb_internal.h"
#include "locate.cuh"

namespace drb
{
namespace
{

template <bool WIDE>
__global__ void first_candidate_kernel (const float4 *__restrict__ nodes, const float4 *__restrict__ wide,
                                        const int *__restrict__ leaf_nodes,
                                        const float *__restrict__ pts, const int *__restrict__ order,
                                        int n, int *__restrict__ first_leaf, int *__restrict__ first_elem)
{
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n) return;
  const int qi = order ? order[pos] : pos;
  const float pt[3] = { pts[3 * (size_t)qi], pts[3 * (size_t)qi + 1], pts[3 * (size_t)qi + 2] };
  int todo[TraversalStack<WIDE>::kDepth];
  int sp = 0, cur = 0, visited = 0;
  todo[0] = kBarrier;
  const int leaf = next_leaf<WIDE> (nodes, wide, pt, todo, sp, cur, visited);
  first_leaf[qi] = leaf;
  if (first_elem) first_elem[qi] = leaf >= 0 ? __ldg (leaf_nodes + leaf) : -1;
}

// First candidate from the point's grid cell: the first listed leaf whose
// box holds the point, which is the traversal's first leaf (the lists hold
// the traversal's candidates in its order).
__global__ void first_grid_candidate_kernel (GridLists gl, const int *__restrict__ leaf_nodes,
                                             const float *__restrict__ pts,
                                             const int *__restrict__ order, int n,
                                             int *__restrict__ first_leaf, int *__restrict__ first_elem)
{
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n) return;
  const int qi = order ? order[pos] : pos;
  const float pt[3] = { pts[3 * (size_t)qi], pts[3 * (size_t)qi + 1], pts[3 * (size_t)qi + 2] };
  const int c = grid_cell (gl.dims, gl.origin, gl.inv, pt);
  int cur = __ldg (gl.start + c), visited = 0;
  const int leaf = next_grid_leaf (gl, pt, cur, __ldg (gl.start + c + 1), visited);
  first_leaf[qi] = leaf;
  if (first_elem) first_elem[qi] = leaf >= 0 ? __ldg (leaf_nodes + leaf) : -1;
}

template <int P, bool REG, bool WIDE>
__global__ void locate_hinted_kernel (LocateParams lp, const float *__restrict__ pts,
                                      const int *__restrict__ order, const int *__restrict__ hint,
                                      int n, int chunk, int *__restrict__ queue_head,
                                      int *__restrict__ cell, float *__restrict__ ref,
                                      int *__restrict__ it_out, int *__restrict__ ca_out,
                                      int *__restrict__ nd_out)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int pool_next = 0, pool_end = 0;
  bool exhausted = false;
  int qi = -1;
  float pt[3] = { 0.f, 0.f, 0.f };
  int todo[TraversalStack<WIDE>::kDepth];
  int sp = 0, cur = kBarrier, skip = -1;
  int iters = 0, cands = 0, nodes = 0;
  int pending = -1; // leaf to solve next (the hinted first candidate)
  bool first = true;
  while (true)
  {
    unsigned need = __ballot_sync (FULL, qi < 0);
    while (need != 0u && !exhausted)
    {
      if (pool_next >= pool_end)
      {
        int base = 0;
        if (lane == 0) base = atomicAdd (queue_head, chunk);
        base = __shfl_sync (FULL, base, 0);
        if (base >= n)
        {
          exhausted = true;
          break;
        }
        pool_next = base;
        pool_end = min (base + chunk, n);
      }
      const int avail = pool_end - pool_next;
      const int rank = __popc (need & lt);
      if (qi < 0 && rank < avail)
      {
        const int pos = pool_next + rank;
        qi = order ? __ldg (order + pos) : pos;
        pt[0] = __ldg (pts + 3 * (size_t)qi);
        pt[1] = __ldg (pts + 3 * (size_t)qi + 1);
        pt[2] = __ldg (pts + 3 * (size_t)qi + 2);
        iters = cands = nodes = 0;
        first = true;
        pending = __ldg (hint + qi);
        skip = pending;
        sp = 0;
        todo[0] = kBarrier;
        cur = (pending >= 0) ? 0 : kBarrier; // no candidate at all: not found
      }
      pool_next += min (__popc (need), avail);
      need = __ballot_sync (FULL, qi < 0);
    }
    if (__ballot_sync (FULL, qi >= 0) == 0u) break;

    int leaf = -1;
    bool from_hint = false;
    if (qi >= 0)
    {
      if (pending >= 0)
      {
        leaf = pending;
        pending = -1;
        from_hint = true;
      }
      else
      {
        // the first leaf met from the root is the hinted one: skip it once
        leaf = next_leaf<WIDE> (lp.nodes, lp.wide, pt, todo, sp, cur, nodes);
        if (leaf >= 0 && leaf == skip)
        {
          cur = todo[sp];
          --sp;
          leaf = next_leaf<WIDE> (lp.nodes, lp.wide, pt, todo, sp, cur, nodes);
        }
        skip = -1;
      }
    }
    if (qi >= 0)
    {
      bool done = false;
      int found_el = -1;
      float x[3] = { -1.f, -1.f, -1.f };
      if (leaf >= 0)
      {
        const int el = __ldg (lp.leaf_nodes + leaf);
        ++cands;
        const bool found = solve_candidate<P, REG> (lp, leaf, el, qi, first, pt, x, iters);
        first = false;
        if (found)
        {
          found_el = el;
          done = true;
        }
        else if (!from_hint)
        {
          cur = todo[sp];
          --sp;
        }
      }
      else
      {
        done = true;
      }
      if (done)
      {
        cell[qi] = found_el;
        if (found_el < 0) x[0] = x[1] = x[2] = -1.f;
        ref[3 * (size_t)qi] = x[0];
        ref[3 * (size_t)qi + 1] = x[1];
        ref[3 * (size_t)qi + 2] = x[2];
        if (it_out) it_out[qi] = iters;
        if (ca_out) ca_out[qi] = cands;
        if (nd_out) nd_out[qi] = nodes;
        qi = -1;
      }
    }
  }
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_first_candidates (const drb_bvh *bvh, const float *pts, int n, const int *order,
                                     int *first_leaf, int *first_elem, void *stream)
{
  if (!bvh || n < 0 || (n > 0 && (!pts || !first_leaf)))
  {
    set_last_error ("first_candidates: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  const GridLists gl = grid_lists (bvh);
  if (gl.start)
    first_grid_candidate_kernel<<<div_up (n, 128), 128, 0, (cudaStream_t)stream>>> (
    gl, bvh->leaf_nodes, pts, order, n, first_leaf, first_elem);
  else if (bvh->wide_nodes)
    first_candidate_kernel<true><<<div_up (n, 128), 128, 0, (cudaStream_t)stream>>> (
    (const float4 *)bvh->inner_nodes, (const float4 *)bvh->wide_nodes, bvh->leaf_nodes, pts, order,
    n, first_leaf, first_elem);
  else
    first_candidate_kernel<false><<<div_up (n, 128), 128, 0, (cudaStream_t)stream>>> (
    (const float4 *)bvh->inner_nodes, nullptr, bvh->leaf_nodes, pts, order, n, first_leaf,
    first_elem);
  return check_launch ("first_candidate_kernel");
}

extern "C" int drb_locate_hinted (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                                  const int *order, const int *first_leaf,
                                  const drb_newton_opts *opts, const drb_locate_config *cfg_in,
                                  int *cell, float *ref, drb_query_stats stats, void *stream)
{
  if (!mesh || !bvh || !opts || n < 0 || (n > 0 && (!pts || !cell || !ref || !first_leaf)))
  {
    set_last_error ("locate_hinted: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (mesh->dim != 3 || mesh->ncomp != 3 || mesh->order < 1 || mesh->order > 3 ||
      mesh->shape != DRB_SHAPE_TENSOR)
  {
    set_last_error ("locate_hinted: needs a hex geometry mesh of order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  if ((opts->guess_mode == DRB_GUESS_GIVEN && !opts->guess) || opts->max_steps < 0 || !(opts->tol > 0.f))
  {
    set_last_error ("locate_hinted: bad Newton options");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  drb_locate_config cfg;
  if (cfg_in) cfg = *cfg_in;
  else
  {
    cfg.block = 128;
    cfg.blocks_per_sm = 0;
    cfg.chunk = 64;
    cfg.sort_queries = 1;
    cfg.reg_elements = 0;
  }
  if (cfg.block < 32 || cfg.block > 1024 || (cfg.block % 32) || cfg.chunk < 1)
  {
    set_last_error ("locate_hinted: bad launch configuration");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  int *head = scr.alloc<int> (1);
  if (!head) return status_from (scr.err);
  cudaMemsetAsync (head, 0, sizeof (int), s);
  LocateParams lp;
  lp.nodes = (const float4 *)bvh->inner_nodes;
  lp.wide = (const float4 *)bvh->wide_nodes;
  lp.leaf_nodes = bvh->leaf_nodes;
  lp.aabb_ids = bvh->aabb_ids;
  lp.ref_boxes = bvh->ref_boxes;
  lp.packed = mesh->packed;
  lp.ctrl_idx = mesh->ctrl_idx;
  lp.xyz = mesh->values;
  lp.stride = packed_stride ((mesh->order + 1) * (mesh->order + 1) * (mesh->order + 1), 3);
  lp.tol = opts->tol;
  lp.max_steps = opts->max_steps;
  lp.guess_mode = opts->guess_mode;
  lp.guess = opts->guess;
  lp.leaf_maps = (const float4 *)bvh->leaf_maps;
  int nb = 0;
  const bool reg = cfg.reg_elements == 1 && mesh->order <= 2; // the register row mode
  const bool wide = lp.wide != nullptr;
#define DRB_HFN(W) (mesh->order == 1 ? (reg ? (const void *)locate_hinted_kernel<1, true, W> : (const void *)locate_hinted_kernel<1, false, W>) \
                   : mesh->order == 2 ? (reg ? (const void *)locate_hinted_kernel<2, true, W> : (const void *)locate_hinted_kernel<2, false, W>) \
                                      : (const void *)locate_hinted_kernel<3, false, W>)
  const void *fn = wide ? DRB_HFN (true) : DRB_HFN (false);
#undef DRB_HFN
  cudaOccupancyMaxActiveBlocksPerMultiprocessor (&nb, fn, cfg.block, 0);
  if (nb < 1) nb = 1;
  const int bps = cfg.blocks_per_sm > 0 ? min (cfg.blocks_per_sm, nb) : nb;
  long long blocks = (long long)bps * sm_count ();
  const long long need = ((long long)n + cfg.block - 1) / cfg.block;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
#define DRB_HINT(P, R, W)                                                                              \
  locate_hinted_kernel<P, R, W><<<(unsigned)blocks, cfg.block, 0, s>>> (lp, pts, order, first_leaf, n, \
                                                                        cfg.chunk, head, cell, ref,    \
                                                                        stats.iters, stats.candidates, \
                                                                        stats.nodes)
  if (wide)
  {
    if (mesh->order == 1) { if (reg) DRB_HINT (1, true, true); else DRB_HINT (1, false, true); }
    else if (mesh->order == 2) { if (reg) DRB_HINT (2, true, true); else DRB_HINT (2, false, true); }
    else DRB_HINT (3, false, true);
  }
  else
  {
    if (mesh->order == 1) { if (reg) DRB_HINT (1, true, false); else DRB_HINT (1, false, false); }
    else if (mesh->order == 2) { if (reg) DRB_HINT (2, true, false); else DRB_HINT (2, false, false); }
    else DRB_HINT (3, false, false);
  }
#undef DRB_HINT
  return check_launch ("locate_hinted_kernel");
}
