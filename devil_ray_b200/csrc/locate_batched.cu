// Persistent, batched point location.
//
// The reference launches one thread per point in input order
// (data_model/unstructured_mesh.cpp:137-148): warps mix points from
// unrelated parts of the mesh, and every lane waits for the slowest lane's
// traversal and Newton iterations.  This path instead
//   1. orders the queries by Morton cell (up to 7 bits per axis over the
//      BVH bounds, a counting sort), so a warp's lanes follow nearly the
//      same BVH path and hit the same few elements (L1/L2 reuse);
//   2. runs a persistent kernel, grid sized to the resident capacity of the
//      148 SMs, whose warps pop chunks of sorted queries from a global atomic
//      queue;
//   3. inside a warp, lanes that finish a query are refilled immediately from
//      the warp's chunk by ballot ranking (warp-ballot compaction), and
//      traversal and Newton are separated into phases so the Newton solves of
//      a warp run converged (traverse until every busy lane holds a
//      candidate leaf or has finished, then solve together).
// Results are identical to the plain kernel's: every query follows the same
// traversal order and per-candidate solves.  The queue holds no waits (only
// atomicAdd pops), so nothing in the kernel can spin.
#include "drb_common.cuh"
#include "drb_internal.h"
#include "locate.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>

namespace drb
{
namespace
{

// Query order by counting sort into Morton cells over the BVH bounds: 7 bits
// per axis for 16M queries (2^21 cells, one cell an eighth of an element of
// a 64^3 mesh), fewer for smaller batches so that a cell holds about eight
// queries (cell_bits: 3..7), which keeps the cell scan proportional to the
// batch.  The persistent kernel needs spatially coherent warps, not a
// sorted sequence, so the order inside a cell is whatever the atomics give:
// one counting pass, a scan of the cell counts and one scatter replace the
// four passes of a 30-bit radix sort.  Every query's result is independent
// of the order.
constexpr int kCellBits = 7;
constexpr int kCells = 1 << (3 * kCellBits);

int cell_bits (int n)
{
  int bits = 3;
  while (bits < kCellBits && (8ll << (3 * bits)) < (long long)n) ++bits;
  return bits;
}

// Grid of the query order: origin and inverse extents of the BVH bounds,
// bits per axis.
struct CellFrame
{
  float lo[3], sc[3];
  int bits;
};

// Morton code (x in the lowest bit) of the cell of a point; NaN queries go
// to cell 0.
DRB_D unsigned point_cell (float px, float py, float pz, const CellFrame &f)
{
  const float p[3] = { px, py, pz };
  unsigned e[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    float t = (p[k] - f.lo[k]) * f.sc[k];
    t = fminf (fmaxf (t * (float)(1 << f.bits), 0.f), (float)((1 << f.bits) - 1));
    unsigned x = (t == t) ? (unsigned)t : 0u;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    e[k] = x;
  }
  return (e[2] << 2) | (e[1] << 1) | e[0];
}

__global__ void cell_count_kernel (const float *__restrict__ pts, int n, float x0, float y0,
                                   float z0, float sx, float sy, float sz,
                                   int bits, unsigned *__restrict__ cell_of,
                                   int *__restrict__ rank, int *__restrict__ hist)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CellFrame f{ { x0, y0, z0 }, { sx, sy, sz }, bits };
  const unsigned c = point_cell (pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2], f);
  cell_of[i] = c;
  rank[i] = atomicAdd (hist + c, 1);
}

// order[pos] = i and, when pos_of is set, pos_of[i] = pos (written in input
// order, so the inverse permutation costs a coalesced store).
__global__ void cell_scatter_kernel (const unsigned *__restrict__ cell_of, const int *__restrict__ rank,
                                     const int *__restrict__ offset, int n, int *__restrict__ order,
                                     int *__restrict__ pos_of)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pos = __ldg (offset + cell_of[i]) + rank[i];
  order[pos] = i;
  if (pos_of) pos_of[i] = pos;
}

// ------------------------------------------------------- staged queries --
//
// Query records in processing order, (x, y, z, input index as int bits), for
// the staged modes (drb_locate_config.sort_queries 2 and 3): the locate
// kernel then reads its queries as consecutive 16-byte records.  They are
// gathered through the index order (random reads, coalesced writes);
// scattering the records themselves would write 16 bytes at random into an
// array larger than L2, a DRAM read-modify-write per record.
__global__ void stage_gather_kernel (const float *__restrict__ pts, const int *__restrict__ order,
                                     int n, float4 *__restrict__ staged)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = __ldg (order + k);
  const float x = __ldg (pts + 3 * (size_t)i), y = __ldg (pts + 3 * (size_t)i + 1),
              z = __ldg (pts + 3 * (size_t)i + 2);
  staged[k] = make_float4 (x, y, z, __int_as_float (i));
}

// Results back to input order: query i's record (cell as int bits, then the
// reference point) sits at its processing position pos_of[i].
__global__ void unstage_kernel (const int *__restrict__ pos_of, const float4 *__restrict__ res, int n,
                                int *__restrict__ cell, float *__restrict__ ref)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 r = __ldg (res + __ldg (pos_of + i));
  cell[i] = __float_as_int (r.x);
  ref[3 * (size_t)i] = r.y;
  ref[3 * (size_t)i + 1] = r.z;
  ref[3 * (size_t)i + 2] = r.w;
}

// The BVH bounds as the cell grid's origin and inverse extents.
void order_frame (const drb_bvh *bvh, float (&lo)[3], float (&sc)[3])
{
  const float *b = bvh->bounds;
  for (int k = 0; k < 3; ++k)
  {
    const float ext = b[2 * k + 1] - b[2 * k];
    sc[k] = (ext > 0.f && std::isfinite (ext)) ? 1.f / ext : 0.f;
    lo[k] = std::isfinite (b[2 * k]) ? b[2 * k] : 0.f;
  }
}

// Cell of every query, its rank inside the cell, and the cells' start
// offsets (exclusive scan of the counts, in hist): cell_of and rank hold n
// values, hist kCells, scan_tmp scan_ws_ints(kCells) (enough for every
// batch size).  Query i's processing position is hist[cell_of[i]] + rank[i].
int cell_positions (const drb_bvh *bvh, const float *pts, int n, unsigned *cell_of, int *rank,
                    int *hist, int *scan_tmp, cudaStream_t s)
{
  float lo[3], sc[3];
  order_frame (bvh, lo, sc);
  const int bits = cell_bits (n);
  const int cells = 1 << (3 * bits);
  cudaError_t e = cudaMemsetAsync (hist, 0, sizeof (int) * cells, s);
  if (e != cudaSuccess)
  {
    set_last_error (cudaGetErrorString (e));
    return status_from (e);
  }
  cell_count_kernel<<<div_up (n, 256), 256, 0, s>>> (pts, n, lo[0], lo[1], lo[2], sc[0], sc[1],
                                                      sc[2], bits, cell_of, rank, hist);
  int st = check_launch ("cell_count_kernel");
  if (st) return st;
  return exclusive_scan_i32_ws (hist, hist, cells, nullptr, scan_tmp, s);
}

// order[0..n) over caller buffers (as cell_positions).
int cell_order (const drb_bvh *bvh, const float *pts, int n, int *order, unsigned *cell_of,
                int *rank, int *hist, int *scan_tmp, cudaStream_t s, int *pos_of = nullptr)
{
  int st = cell_positions (bvh, pts, n, cell_of, rank, hist, scan_tmp, s);
  if (st) return st;
  cell_scatter_kernel<<<div_up (n, 256), 256, 0, s>>> (cell_of, rank, hist, n, order, pos_of);
  return check_launch ("cell_scatter_kernel");
}

// The queries staged in processing order: staged[k] = (x, y, z, input
// index bits) of the k-th query in Morton-cell order (the order inside a
// cell is unspecified); order, cell_of, rank, hist and scan_tmp as
// cell_order's; pos_of (optional): each query's processing position.
int cell_stage (const drb_bvh *bvh, const float *pts, int n, float4 *staged, int *order,
                unsigned *cell_of, int *rank, int *hist, int *scan_tmp, int *pos_of, cudaStream_t s)
{
  int st = cell_order (bvh, pts, n, order, cell_of, rank, hist, scan_tmp, s, pos_of);
  if (st) return st;
  stage_gather_kernel<<<div_up (n, 256), 256, 0, s>>> (pts, order, n, staged);
  return check_launch ("stage_gather_kernel");
}

int unstage (const int *pos_of, const float4 *res, int n, int *cell, float *ref, cudaStream_t s)
{
  unstage_kernel<<<div_up (n, 256), 256, 0, s>>> (pos_of, res, n, cell, ref);
  return check_launch ("unstage_kernel");
}

// Element-row modes of the candidate solves (drb_locate_config.reg_elements)
enum RowMode
{
  kRowsL1 = 0,     // control points read through L1 on every Newton step
  kRowsReg = 1,    // the row copied into registers (orders 1-2)
  kRowsShared = 2  // the distinct rows of a warp's candidates staged in shared memory
};

// Shared-memory row stride (floats): the packed row plus one, odd, so 32
// lanes reading the same column of different rows hit 32 different banks.
template <int P> constexpr int smem_row_stride ()
{
  return packed_stride ((P + 1) * (P + 1) * (P + 1), 3) + 1;
}
template <int P> constexpr size_t smem_rows_bytes_per_warp ()
{
  return sizeof (float) * 32 * (size_t)smem_row_stride<P> ();
}

// Staged queries (staged != NULL): the queries are read from staged[pos],
// already in processing order with the input index in w, so a warp reads
// its queries as one contiguous block (`order` and `pts` are unused).  With
// res == NULL the results go to cell/ref at the input index (scattered
// writes, which the kernel's latency-bound loop absorbs); with res set they
// go to res[pos] as (cell as int bits, reference point), contiguous, for a
// separate pass to put back.  Statistics always go to the input index.
// TRAV: 0 binary tree, 1 4-wide tree, 2 grid candidate lists.
template <int P, int MODE, int TRAV, int S>
DRB_D void persistent_body (const LocateParams &lp, const float *__restrict__ pts,
                                            const int *__restrict__ order, int n, int chunk,
                                            int *__restrict__ queue_head, int *__restrict__ cell,
                                            float *__restrict__ ref, int *__restrict__ it_out,
                                            int *__restrict__ ca_out, int *__restrict__ nd_out,
                                            const float4 *__restrict__ staged,
                                            float4 *__restrict__ res, const GridLists &gl)
{
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  extern __shared__ float s_rows[]; // kRowsShared: 32 row slots per warp
  float *warp_rows = s_rows + (size_t)(threadIdx.x >> 5) * 32 * smem_row_stride<P> ();
  int pool_next = 0, pool_end = 0; // warp-uniform
  bool exhausted = false;          // warp-uniform
  int qi = -1;
  float pt[3] = { 0.f, 0.f, 0.f };
  constexpr bool WIDE = TRAV == 1, GRID = TRAV == 2;
  int todo[GRID ? 1 : TraversalStack<WIDE>::kDepth];
  int sp = 0, cur = kBarrier;
  int iters = 0, cands = 0, nodes = 0;
  bool first = true;
  // The last three elements whose solve failed for this query.  With a guess
  // that does not depend on the leaf (zero, element centre, or a given
  // guess whose centre fallback also ran) a repeat of one of them fails
  // again the same way, so its solve is skipped.  Simplex kinds only: the
  // sub-boxes of a tet or triangle overlap heavily (a query lies in about
  // 20 tet sub-boxes of 3.6 distinct tets), those of a hex barely (1.3
  // boxes of 1.04 hexes), where the check would only cost registers.
  constexpr bool kSkipRepeats = (S == kSimplex || S == kTri2D);
  const bool leaf_free_guess = kSkipRepeats && lp.guess_mode != DRB_GUESS_SUBREF_CENTER &&
                               lp.guess_mode != DRB_GUESS_SUBBOX_LINEAR;
  int failed0 = -1, failed1 = -1, failed2 = -1;

  while (true)
  {
    // ---- refill idle lanes from the warp's chunk (ballot ranking) ----
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
        if (staged)
        {
          // qi: the processing position when the results are staged (the
          // guess mode is then never DRB_GUESS_GIVEN), else the input index
          const float4 v = __ldg (staged + pos);
          qi = res ? pos : __float_as_int (v.w);
          pt[0] = v.x;
          pt[1] = v.y;
          pt[2] = v.z;
        }
        else
        {
          qi = order ? __ldg (order + pos) : pos;
          pt[0] = __ldg (pts + 3 * (size_t)qi);
          pt[1] = __ldg (pts + 3 * (size_t)qi + 1);
          pt[2] = __ldg (pts + 3 * (size_t)qi + 2);
        }
        sp = 0;
        todo[0] = kBarrier;
        cur = 0;
        if constexpr (GRID)
        {
          // grid lists: cur walks the cell's entries up to sp
          const int c = grid_cell (gl.dims, gl.origin, gl.inv, pt);
          cur = __ldg (gl.start + c);
          sp = __ldg (gl.start + c + 1);
        }
        iters = cands = nodes = 0;
        first = true;
        failed0 = failed1 = failed2 = -1;
      }
      pool_next += min (__popc (need), avail);
      need = __ballot_sync (FULL, qi < 0);
    }
    if (__ballot_sync (FULL, qi >= 0) == 0u) break;

    // ---- traversal phase: advance to the next candidate leaf ----
    // Simplex kinds: a candidate that the repeat or hull filter rejects
    // needs no solve, so the lane moves straight on to the next candidate
    // here instead of sitting out the warp's solves of this iteration.
    int leaf = -1;
    if (qi >= 0)
    {
      while (true)
      {
        if constexpr (GRID) leaf = next_grid_leaf (gl, pt, cur, sp, nodes);
        else leaf = next_leaf<WIDE> (lp.nodes, lp.wide, pt, todo, sp, cur, nodes);
        if (!kSkipRepeats || leaf < 0) break;
        const int e = __ldg (lp.leaf_nodes + leaf);
        const bool repeat = leaf_free_guess && (e == failed0 || e == failed1 || e == failed2);
        if (!repeat && !(S == kSimplex && lp.hull && hull_rejects (lp, e, pt))) break;
        ++cands;
        first = false;
        if (!repeat)
        {
          failed2 = failed1;
          failed1 = failed0;
          failed0 = e;
        }
        if constexpr (!GRID)
        {
          cur = todo[sp];
          --sp;
        }
      }
    }

    // ---- candidate phase: converged Newton solves ----
    int el = -1;
    if (qi >= 0 && leaf >= 0) el = __ldg (lp.leaf_nodes + leaf);
    const float *my_row = nullptr;
    if (MODE == kRowsShared)
    {
      // lanes with the same element share one slot; the warp loads each
      // distinct row once with float4 reads and stores it at odd stride
      constexpr int S = smem_row_stride<P> ();
      constexpr int F4 = (S - 1) / 4;
      const bool has = el >= 0;
      const unsigned same = __match_any_sync (FULL, has ? el : -1 - lane);
      const int leader = __ffs (same) - 1;
      const unsigned leaders = __ballot_sync (FULL, has && leader == lane);
      const int slot = __popc (leaders & ((1u << leader) - 1u));
      __syncwarp ();
      unsigned todo_rows = leaders;
      int r = 0;
      while (todo_rows)
      {
        const int src = __ffs (todo_rows) - 1;
        todo_rows &= todo_rows - 1u;
        const int e = __shfl_sync (FULL, el, src);
        for (int q = lane; q < F4; q += 32)
        {
          const float4 v = __ldg (reinterpret_cast<const float4 *> (lp.packed + (size_t)e * lp.stride) + q);
          float *d = warp_rows + r * S + 4 * q;
          d[0] = v.x;
          d[1] = v.y;
          d[2] = v.z;
          d[3] = v.w;
        }
        ++r;
      }
      __syncwarp ();
      if (has) my_row = warp_rows + slot * S;
    }
    if (qi >= 0)
    {
      bool done = false;
      int found_el = -1;
      float x[3] = { -1.f, -1.f, -1.f };
      if (leaf >= 0)
      {
        ++cands;
        // (the simplex filters ran in the traversal phase)
        const bool found = (MODE == kRowsShared)
                           ? solve_candidate_smem<P> (lp, leaf, my_row, qi, first, pt, x, iters)
                           : solve_candidate<P, MODE == kRowsReg, S> (lp, leaf, el, qi, first, pt, x, iters);
        first = false;
        if (found)
        {
          found_el = el;
          done = true;
        }
        else
        {
          if (kSkipRepeats)
          {
            failed2 = failed1;
            failed1 = failed0;
            failed0 = el;
          }
          if constexpr (!GRID)
          {
            cur = todo[sp];
            --sp;
          }
        }
      }
      else
      {
        done = true; // traversal exhausted: not found
      }
      if (done)
      {
        if (found_el < 0) x[0] = x[1] = x[2] = -1.f;
        int q = qi;
        if (res)
        {
          res[qi] = make_float4 (__int_as_float (found_el), x[0], x[1], x[2]);
          if (it_out || ca_out || nd_out) q = __float_as_int (__ldg (&staged[qi].w));
        }
        else
        {
          cell[qi] = found_el;
          ref[3 * (size_t)qi] = x[0];
          ref[3 * (size_t)qi + 1] = x[1];
          ref[3 * (size_t)qi + 2] = x[2];
        }
        if (it_out) it_out[q] = iters;
        if (ca_out) ca_out[q] = cands;
        if (nd_out) nd_out[q] = nodes;
        qi = -1;
      }
    }
  }
}

#define DRB_PERSISTENT_ARGS                                                                   \
  LocateParams lp, const float *__restrict__ pts, const int *__restrict__ order, int n, int chunk, \
      int *__restrict__ queue_head, int *__restrict__ cell, float *__restrict__ ref,              \
      int *__restrict__ it_out, int *__restrict__ ca_out, int *__restrict__ nd_out,               \
      const float4 *__restrict__ staged, float4 *__restrict__ res, GridLists gl
template <int P, int MODE, int TRAV, int S = kTensor>
__global__ void locate_persistent_kernel (DRB_PERSISTENT_ARGS)
{
  persistent_body<P, MODE, TRAV, S> (lp, pts, order, n, chunk, queue_head, cell, ref, it_out, ca_out,
                                     nd_out, staged, res, gl);
}
// The grid scan with L1 rows at orders 1-2, held to 80 registers (the
// compiler's choice of 89 at order 2 costs a quarter of the resident warps;
// measured 9 % faster at 80, slower at 72, where it spills).
template <int P, int MODE, int TRAV, int S = kTensor>
__global__ void __maxnreg__ (80) locate_persistent_kernel_r80 (DRB_PERSISTENT_ARGS)
{
  persistent_body<P, MODE, TRAV, S> (lp, pts, order, n, chunk, queue_head, cell, ref, it_out, ca_out,
                                     nd_out, staged, res, gl);
}
#undef DRB_PERSISTENT_ARGS

template <int P, int MODE, int TRAV> constexpr bool capped_kernel ()
{
  return TRAV == 2 && MODE == kRowsL1 && P <= 2;
}

// Tets run the L1 and register row modes (shared rows are tensor-only).
template <int P, int W, int S> const void *persistent_fn_pw (int mode)
{
  if (S == kTensor && mode == kRowsShared) return (const void *)locate_persistent_kernel<P, kRowsShared, W>;
  if (mode == kRowsReg && P <= 2) return (const void *)locate_persistent_kernel<P, kRowsReg, W, S>;
  if constexpr (capped_kernel<P, kRowsL1, W> ())
    return (const void *)locate_persistent_kernel_r80<P, kRowsL1, W, S>;
  else
    return (const void *)locate_persistent_kernel<P, kRowsL1, W, S>;
}

template <int P, int S> const void *persistent_fn_p (int mode, int trav)
{
  return trav == 2 ? persistent_fn_pw<P, 2, S> (mode) : trav == 1 ? persistent_fn_pw<P, 1, S> (mode)
                                                      : persistent_fn_pw<P, 0, S> (mode);
}

template <int S> const void *persistent_fn_s (int order, int mode, int trav)
{
  if (order == 1) return persistent_fn_p<1, S> (mode, trav);
  if (order == 2) return persistent_fn_p<2, S> (mode, trav);
  return persistent_fn_p<3, S> (mode, trav);
}

const void *persistent_fn (const drb_mesh *mesh, int mode, int trav)
{
  if (mesh->shape == DRB_SHAPE_SIMPLEX && mesh->dim == 2) return persistent_fn_s<kTri2D> (mesh->order, mode, trav);
  if (mesh->shape == DRB_SHAPE_SIMPLEX) return persistent_fn_s<kSimplex> (mesh->order, mode, trav);
  if (mesh->dim == 2) return persistent_fn_s<kQuad2D> (mesh->order, mode, trav);
  return persistent_fn_s<kTensor> (mesh->order, mode, trav);
}

// Row mode actually used: registers only for orders 1-2, shared rows only
// for hexes with a packed element copy.
int effective_mode (const drb_mesh *mesh, int requested)
{
  if (requested == kRowsReg && mesh->order <= 2) return kRowsReg;
  if (requested == kRowsShared && mesh->packed && mesh->shape == DRB_SHAPE_TENSOR && mesh->dim == 3)
    return kRowsShared;
  return kRowsL1;
}

size_t dynamic_smem (int order, int mode, int block)
{
  if (mode != kRowsShared) return 0;
  const size_t per_warp = order == 1 ? smem_rows_bytes_per_warp<1> ()
                          : order == 2 ? smem_rows_bytes_per_warp<2> () : smem_rows_bytes_per_warp<3> ();
  return per_warp * (size_t)(block / 32);
}

// Query records of a staged launch (both NULL: unstaged).
struct Staging
{
  const float4 *staged = nullptr;
  float4 *res = nullptr;
};

template <int P, int W, int S>
void launch_pw (int mode, dim3 grid, int block, size_t smem, cudaStream_t s, const LocateParams &lp,
                const GridLists &gl, const float *pts, const int *ord, int n, int chunk, int *head, int *cell, float *ref,
                drb_query_stats st, Staging sg)
{
#define DRB_LP(K, M, SS) K<P, M, W, SS><<<grid, block, smem, s>>> (lp, pts, ord, n, chunk, head, cell, ref, st.iters, st.candidates, st.nodes, sg.staged, sg.res, gl)
  if (S == kTensor && mode == kRowsShared) DRB_LP (locate_persistent_kernel, kRowsShared, kTensor);
  else if (mode == kRowsReg && P <= 2) DRB_LP (locate_persistent_kernel, P <= 2 ? kRowsReg : kRowsL1, S);
  else if constexpr (capped_kernel<P, kRowsL1, W> ()) DRB_LP (locate_persistent_kernel_r80, kRowsL1, S);
  else DRB_LP (locate_persistent_kernel, kRowsL1, S);
#undef DRB_LP
}

template <int S>
void launch_s (int order, int trav, int mode, dim3 grid, int block, size_t smem, cudaStream_t s,
               const LocateParams &lp, const GridLists &gl, const float *pts, const int *ord, int n,
               int chunk, int *head, int *cell, float *ref, drb_query_stats st, Staging sg)
{
#define DRB_LT(P, T) launch_pw<P, T, S> (mode, grid, block, smem, s, lp, gl, pts, ord, n, chunk, head, cell, ref, st, sg)
#define DRB_LO(P) { if (trav == 2) DRB_LT (P, 2); else if (trav == 1) DRB_LT (P, 1); else DRB_LT (P, 0); }
  if (order == 1) DRB_LO (1)
  else if (order == 2) DRB_LO (2)
  else DRB_LO (3)
#undef DRB_LO
#undef DRB_LT
}

// Traversal of the batched kernels: grid lists, else the 4-wide tree, else
// the binary tree.
int traversal_kind (const LocateParams &lp, const GridLists &gl)
{
  return gl.start ? 2 : lp.wide ? 1 : 0;
}

int launch_persistent (const drb_mesh *mesh, int mode, dim3 grid, int block, cudaStream_t s,
                       const LocateParams &lp, const GridLists &gl, const float *pts, const int *ord, int n, int chunk,
                       int *head, int *cell, float *ref, drb_query_stats st, Staging sg = Staging ())
{
  const int order = mesh->order;
  const size_t smem = dynamic_smem (order, mode, block);
  const int trav = traversal_kind (lp, gl);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute (persistent_fn (mesh, mode, trav), cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)smem);
  if (mesh->shape == DRB_SHAPE_SIMPLEX && mesh->dim == 2)
    launch_s<kTri2D> (order, trav, mode, grid, block, smem, s, lp, gl, pts, ord, n, chunk, head, cell, ref, st, sg);
  else if (mesh->shape == DRB_SHAPE_SIMPLEX)
    launch_s<kSimplex> (order, trav, mode, grid, block, smem, s, lp, gl, pts, ord, n, chunk, head, cell, ref, st, sg);
  else if (mesh->dim == 2)
    launch_s<kQuad2D> (order, trav, mode, grid, block, smem, s, lp, gl, pts, ord, n, chunk, head, cell, ref, st, sg);
  else
    launch_s<kTensor> (order, trav, mode, grid, block, smem, s, lp, gl, pts, ord, n, chunk, head, cell, ref, st, sg);
  return check_launch ("locate_persistent_kernel");
}

int resident_blocks (const drb_mesh *mesh, int mode, int trav, int block)
{
  const size_t smem = dynamic_smem (mesh->order, mode, block);
  const void *fn = persistent_fn (mesh, mode, trav);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute (fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor (&nb, fn, block, smem);
  return nb > 0 ? nb : 1;
}

LocateParams make_params (const drb_mesh *mesh, const drb_bvh *bvh, const drb_newton_opts *opts)
{
  LocateParams lp;
  lp.nodes = (const float4 *)bvh->inner_nodes;
  lp.wide = (const float4 *)bvh->wide_nodes;
  lp.leaf_nodes = bvh->leaf_nodes;
  lp.aabb_ids = bvh->aabb_ids;
  lp.ref_boxes = bvh->ref_boxes;
  lp.packed = mesh->packed;
  lp.ctrl_idx = mesh->ctrl_idx;
  lp.xyz = mesh->values;
  lp.stride = packed_stride (mesh_nd (mesh), 3);
  lp.tol = opts->tol;
  lp.max_steps = opts->max_steps;
  lp.guess_mode = opts->guess_mode;
  lp.guess = opts->guess;
  lp.hull = (mesh->shape == DRB_SHAPE_SIMPLEX && mesh->dim == 3) ? (const float4 *)mesh->hull_planes
                                                                   : nullptr;
  lp.leaf_maps = mesh->dim == 3 ? (const float4 *)bvh->leaf_maps : nullptr;
  return lp;
}

int check_args (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                const drb_newton_opts *opts, const int *cell, const float *ref)
{
  if (!mesh || !bvh || !opts || n < 0 || (n > 0 && (!pts || !cell || !ref)))
  {
    set_last_error ("locate_batched: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (mesh->ncomp != 3 || mesh->order < 1 || mesh->order > 3 ||
      !((mesh->dim == 3 || mesh->dim == 2) &&
        (mesh->shape == DRB_SHAPE_TENSOR || mesh->shape == DRB_SHAPE_SIMPLEX)))
  {
    set_last_error ("locate_batched: needs a hex, tet, quad or triangle geometry mesh of order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  if (opts->guess_mode == DRB_GUESS_GIVEN && !opts->guess)
  {
    set_last_error ("locate_batched: DRB_GUESS_GIVEN needs a guess array");
    return DRB_ERR_INVALID_ARG;
  }
  if (opts->max_steps < 0 || !(opts->tol > 0.f))
  {
    set_last_error ("locate_batched: tol must be > 0 and max_steps >= 0");
    return DRB_ERR_INVALID_ARG;
  }
  return DRB_OK;
}

drb_locate_config default_config (int order)
{
  drb_locate_config c;
  c.block = 128;
  c.blocks_per_sm = 0; // 0 = all resident blocks
  c.chunk = 64;
  c.sort_queries = 1;
  c.reg_elements = 0;
  (void)order;
  return c;
}

} // namespace

// Morton order of the queries over the BVH bounds (device int32 order[n]).
int query_cell_count () { return kCells; }

int query_morton_order (const drb_bvh *bvh, const float *pts, int n, int *order, cudaStream_t s)
{
  Scratch scr (s);
  unsigned *cell_of = scr.alloc<unsigned> (n);
  int *rank = scr.alloc<int> (n);
  int *hist = scr.alloc<int> (kCells);
  int *tmp = scr.alloc<int> (scan_ws_ints (kCells));
  if (scr.err != cudaSuccess) return status_from (scr.err);
  return cell_order (bvh, pts, n, order, cell_of, rank, hist, tmp, s);
}

int check_config (const drb_locate_config &cfg)
{
  if (cfg.block < 32 || cfg.block > 1024 || (cfg.block % 32) || cfg.chunk < 1)
  {
    set_last_error ("locate_batched: block must be a multiple of 32 in [32,1024], chunk >= 1");
    return DRB_ERR_INVALID_ARG;
  }
  return DRB_OK;
}

// Persistent grid of a launch: the resident blocks of the configured shape
// on every SM (or cfg.blocks_per_sm of them), no more than the queries fill.
int persistent_blocks (const drb_mesh *mesh, const drb_bvh *bvh, const drb_locate_config &cfg,
                       int mode, int n)
{
  const int per_sm = resident_blocks (mesh, mode, grid_lists (bvh).start ? 2
                                                 : bvh->wide_nodes ? 1 : 0, cfg.block);
  const int bps = (cfg.blocks_per_sm > 0) ? min (cfg.blocks_per_sm, per_sm) : per_sm;
  const long long warps_needed = ((long long)n + 31) / 32;
  long long blocks = (long long)bps * sm_count ();
  const long long blocks_needed = (warps_needed * 32 + cfg.block - 1) / cfg.block;
  if (blocks > blocks_needed) blocks = blocks_needed;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// The persistent kernel over staged query records (head: the queue counter,
// cleared here on the stream): results to res in the staged order, or with
// res NULL to cell/ref at the input index.
int locate_staged_launch (const drb_mesh *mesh, const drb_bvh *bvh, const float4 *staged, int n,
                          const drb_newton_opts *opts, const drb_locate_config &cfg, int *head,
                          float4 *res, int *cell, float *ref, drb_query_stats stats,
                          cudaStream_t s)
{
  cudaError_t e = cudaMemsetAsync (head, 0, sizeof (int), s);
  if (e != cudaSuccess) return status_from (e);
  const int mode = effective_mode (mesh, cfg.reg_elements);
  const int blocks = persistent_blocks (mesh, bvh, cfg, mode, n);
  const LocateParams lp = make_params (mesh, bvh, opts);
  Staging sg;
  sg.staged = staged;
  sg.res = res;
  return launch_persistent (mesh, mode, dim3 ((unsigned)blocks), cfg.block, s, lp, grid_lists (bvh),
                            nullptr, nullptr, n, cfg.chunk, head, cell, ref, stats, sg);
}

// Sorted, staged batch over caller buffers: stage the queries in Morton-cell
// order and locate them; with res set (sort_queries 3) the results are
// staged too and put back in input order by a separate pass.
int locate_staged_batch (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                         const drb_newton_opts *opts, const drb_locate_config &cfg, int *order,
                         unsigned *cell_of, int *rank, int *hist, int *scan_tmp, int *pos_of,
                         int *head, float4 *staged, float4 *res, int *cell, float *ref,
                         drb_query_stats stats, cudaStream_t s)
{
  int st = cell_stage (bvh, pts, n, staged, order, cell_of, rank, hist, scan_tmp,
                       res ? pos_of : nullptr, s);
  if (st) return st;
  st = locate_staged_launch (mesh, bvh, staged, n, opts, cfg, head, res, cell, ref, stats, s);
  if (st || !res) return st;
  return unstage (pos_of, res, n, cell, ref, s);
}

// Query order modes (drb_locate_config.sort_queries).
constexpr int kSortIndexed = 1;       // Morton order; queries read through the order
constexpr int kSortStaged = 2;        // query records staged, results in place
constexpr int kSortStagedResults = 3; // results staged too, put back in a pass

int locate_batched_impl (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                         const drb_newton_opts *opts, const drb_locate_config *cfg_in,
                         const int *order_in, int *cell, float *ref, drb_query_stats stats,
                         cudaStream_t s)
{
  int st = check_args (mesh, bvh, pts, n, opts, cell, ref);
  if (st) return st;
  if (n == 0) return DRB_OK;
  const drb_locate_config cfg = cfg_in ? *cfg_in : default_config (mesh->order);
  if ((st = check_config (cfg))) return st;
  Scratch scr (s);
  int *head = scr.alloc<int> (1);
  if (!order_in && cfg.sort_queries >= kSortStaged)
  {
    // staged: query records read in processing order; results written in
    // place, or staged as well (not with given guesses, which are indexed
    // by the input order)
    const bool stage_res = cfg.sort_queries == kSortStagedResults &&
                           opts->guess_mode != DRB_GUESS_GIVEN;
    int *ord = scr.alloc<int> (n);
    unsigned *cell_of = scr.alloc<unsigned> (n);
    int *rank = scr.alloc<int> (n);
    int *hist = scr.alloc<int> (kCells);
    int *tmp = scr.alloc<int> (scan_ws_ints (kCells));
    float4 *staged = scr.alloc<float4> (n);
    float4 *res = stage_res ? scr.alloc<float4> (n) : nullptr;
    int *pos_of = stage_res ? scr.alloc<int> (n) : nullptr;
    if (scr.err != cudaSuccess) return status_from (scr.err);
    return locate_staged_batch (mesh, bvh, pts, n, opts, cfg, ord, cell_of, rank, hist, tmp,
                                pos_of, head, staged, res, cell, ref, stats, s);
  }
  const int *ord = order_in;
  if (!ord && cfg.sort_queries)
  {
    int *o = scr.alloc<int> (n);
    if (!o) return status_from (scr.err);
    st = query_morton_order (bvh, pts, n, o, s);
    if (st) return st;
    ord = o;
  }
  if (scr.err != cudaSuccess) return status_from (scr.err);
  cudaMemsetAsync (head, 0, sizeof (int), s);
  const int mode = effective_mode (mesh, cfg.reg_elements);
  const int blocks = persistent_blocks (mesh, bvh, cfg, mode, n);
  const LocateParams lp = make_params (mesh, bvh, opts);
  return launch_persistent (mesh, mode, dim3 ((unsigned)blocks), cfg.block, s, lp, grid_lists (bvh),
                            pts, ord, n,
                            cfg.chunk, head, cell, ref, stats);
}

// Same as locate_batched_impl with sorting (queries read through the index
// order), but over caller-provided workspace.
int locate_batched_ws (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                       const drb_newton_opts *opts, const drb_locate_config *cfg_in,
                       const LocateWorkspace &ws, int *cell, float *ref, drb_query_stats stats,
                       cudaStream_t s)
{
  int st = check_args (mesh, bvh, pts, n, opts, cell, ref);
  if (st) return st;
  if (n == 0) return DRB_OK;
  const drb_locate_config cfg = cfg_in ? *cfg_in : default_config (mesh->order);
  if ((st = check_config (cfg))) return st;
  const int *ord = nullptr;
  if (cfg.sort_queries)
  {
    st = cell_order (bvh, pts, n, ws.order, ws.codes, ws.iota, ws.hist, ws.radix.scan_tmp, s);
    if (st) return st;
    ord = ws.order;
  }
  cudaError_t e = cudaMemsetAsync (ws.head, 0, sizeof (int), s);
  if (e != cudaSuccess) return status_from (e);
  const int mode = effective_mode (mesh, cfg.reg_elements);
  const int blocks = persistent_blocks (mesh, bvh, cfg, mode, n);
  const LocateParams lp = make_params (mesh, bvh, opts);
  return launch_persistent (mesh, mode, dim3 ((unsigned)blocks), cfg.block, s, lp, grid_lists (bvh),
                            pts, ord, n,
                            cfg.chunk, ws.head, cell, ref, stats);
}

} // namespace drb

using namespace drb;

extern "C" int drb_locate_batched (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts,
                                   int n, const drb_newton_opts *opts,
                                   const drb_locate_config *cfg, int *cell, float *ref,
                                   drb_query_stats stats, void *stream)
{
  return locate_batched_impl (mesh, bvh, pts, n, opts, cfg, nullptr, cell, ref, stats,
                              (cudaStream_t)stream);
}

extern "C" int drb_query_order (const drb_bvh *bvh, const float *pts, int n, int *order,
                                void *stream)
{
  if (!bvh || n < 0 || (n > 0 && (!pts || !order)))
  {
    set_last_error ("query_order: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  return query_morton_order (bvh, pts, n, order, (cudaStream_t)stream);
}

extern "C" int drb_locate_ordered (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts,
                                   int n, const int *order, const drb_newton_opts *opts,
                                   const drb_locate_config *cfg, int *cell, float *ref,
                                   drb_query_stats stats, void *stream)
{
  if (!order && n > 0)
  {
    set_last_error ("locate_ordered: order is NULL");
    return DRB_ERR_INVALID_ARG;
  }
  return locate_batched_impl (mesh, bvh, pts, n, opts, cfg, order, cell, ref, stats,
                              (cudaStream_t)stream);
}

extern "C" int drb_query_stage (const drb_bvh *bvh, const float *pts, int n, float *staged,
                                void *stream)
{
  if (!bvh || n < 0 || (n > 0 && (!pts || !staged)))
  {
    set_last_error ("query_stage: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  if (reinterpret_cast<uintptr_t> (staged) % 16)
  {
    set_last_error ("query_stage: staged must be 16-byte aligned");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  int *ord = scr.alloc<int> (n);
  unsigned *cell_of = scr.alloc<unsigned> (n);
  int *rank = scr.alloc<int> (n);
  int *hist = scr.alloc<int> (kCells);
  int *tmp = scr.alloc<int> (scan_ws_ints (kCells));
  if (scr.err != cudaSuccess) return status_from (scr.err);
  return cell_stage (bvh, pts, n, reinterpret_cast<float4 *> (staged), ord, cell_of, rank, hist,
                     tmp, nullptr, s);
}

extern "C" int drb_locate_staged (const drb_mesh *mesh, const drb_bvh *bvh, const float *staged,
                                  int n, const drb_newton_opts *opts, const drb_locate_config *cfg_in,
                                  float *res, int *cell, float *ref, drb_query_stats stats,
                                  void *stream)
{
  const bool to_res = res != nullptr;
  int st = check_args (mesh, bvh, staged, n, opts, to_res ? (const int *)res : cell,
                       to_res ? res : ref);
  if (st) return st;
  if (to_res && opts->guess_mode == DRB_GUESS_GIVEN)
  {
    set_last_error ("locate_staged: DRB_GUESS_GIVEN needs the results at the input index "
                    "(res NULL)");
    return DRB_ERR_INVALID_ARG;
  }
  if ((reinterpret_cast<uintptr_t> (staged) | reinterpret_cast<uintptr_t> (res)) % 16)
  {
    set_last_error ("locate_staged: staged and res must be 16-byte aligned");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  const drb_locate_config cfg = cfg_in ? *cfg_in : default_config (mesh->order);
  if ((st = check_config (cfg))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  int *head = scr.alloc<int> (1);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  return locate_staged_launch (mesh, bvh, reinterpret_cast<const float4 *> (staged), n, opts, cfg,
                               head, reinterpret_cast<float4 *> (res), cell, ref, stats, s);
}

// Autotuner: times every (block, blocks/SM, chunk) candidate on the given
// sample with CUDA events and returns the fastest.  The sample is located
// in Morton order once; each candidate runs twice and the second run counts.
extern "C" int drb_locate_tune (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                                const drb_newton_opts *opts, drb_locate_config *best,
                                float *best_ms, void *stream)
{
  int st = check_args (mesh, bvh, pts, n, opts, (const int *)1, (const float *)1);
  if (st) return st;
  if (!best || n <= 0)
  {
    set_last_error ("locate_tune: best is NULL or the sample is empty");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  // the kernel as drb_locate_batched runs it by default: the sample in
  // Morton-cell order once, read through that order
  int *ord = scr.alloc<int> (n);
  int *cell = scr.alloc<int> (n);
  float *ref = scr.alloc<float> ((size_t)3 * n);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  st = query_morton_order (bvh, pts, n, ord, s);
  if (st) return st;
  const int blocks[] = { 64, 128, 256 };
  const int per_sm[] = { 0, 4, 2 };
  const int chunks[] = { 32, 64, 128, 256 };
  cudaEvent_t e0, e1;
  cudaEventCreate (&e0);
  cudaEventCreate (&e1);
  float best_t = 1e30f;
  drb_locate_config bc = default_config (mesh->order);
  const int modes[] = { kRowsL1, kRowsReg, kRowsShared };
  for (int rg : modes)
  if (effective_mode (mesh, rg) == rg)
  for (int b : blocks)
    for (int ps : per_sm)
      for (int c : chunks)
      {
        drb_locate_config cfg;
        cfg.block = b;
        cfg.blocks_per_sm = ps;
        cfg.chunk = c;
        cfg.sort_queries = 1;
        cfg.reg_elements = rg;
        float t = 0.f;
        for (int rep = 0; rep < 2 && st == DRB_OK; ++rep)
        {
          cudaEventRecord (e0, s);
          st = locate_batched_impl (mesh, bvh, pts, n, opts, &cfg, ord, cell, ref,
                                    drb_query_stats{ nullptr, nullptr, nullptr }, s);
          cudaEventRecord (e1, s);
          cudaEventSynchronize (e1);
          cudaEventElapsedTime (&t, e0, e1);
        }
        if (st) break;
        if (t < best_t)
        {
          best_t = t;
          bc = cfg;
        }
      }
  cudaEventDestroy (e0);
  cudaEventDestroy (e1);
  if (st) return st;
  *best = bc;
  if (best_ms) *best_ms = best_t;
  return DRB_OK;
}
