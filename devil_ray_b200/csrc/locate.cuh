// Device pieces shared by the point-location kernels (plain, persistent)
// and the volume renderer: node tests, the per-candidate guess and the
// per-element Newton dispatch.
#pragma once

#include "drb_common.cuh"
#include "newton.cuh"
#include "simplex.cuh"
#include "../../include/drb.h"

namespace drb
{

// Point-in-box tests of both children of an inner node (device_mesh.hpp:262-318).
DRB_D void node_point_test (const float4 *__restrict__ nodes, int node, const float (&p)[3],
                            bool &in_left, bool &in_right)
{
  const float4 a = __ldg (nodes + node + 0);
  const float4 b = __ldg (nodes + node + 1);
  const float4 c = __ldg (nodes + node + 2);
  in_left = !(p[0] < a.x || p[1] < a.y || p[2] < a.z || p[0] > a.w || p[1] > b.x || p[2] > b.y);
  in_right = !(p[0] < b.z || p[1] < b.w || p[2] < c.x || p[0] > c.y || p[1] > c.z || p[2] > c.w);
}

// The whole 64-byte node record in one go: boxes and child ids are issued
// together, so a visit costs one dependent round trip instead of two.
DRB_D void node_point_test_kids (const float4 *__restrict__ nodes, int node, const float (&p)[3],
                                 bool &in_left, bool &in_right, int &l, int &r)
{
  const float4 a = __ldg (nodes + node + 0);
  const float4 b = __ldg (nodes + node + 1);
  const float4 c = __ldg (nodes + node + 2);
  const float4 d = __ldg (nodes + node + 3);
  in_left = !(p[0] < a.x || p[1] < a.y || p[2] < a.z || p[0] > a.w || p[1] > b.x || p[2] > b.y);
  in_right = !(p[0] < b.z || p[1] < b.w || p[2] < c.x || p[0] > c.y || p[1] > c.z || p[2] > c.w);
  l = __float_as_int (d.x);
  r = __float_as_int (d.y);
}

// The four child boxes of a wide node (drb_bvh_widen) against a point, with
// the binary node test's comparisons: bit c set when child c holds p.
DRB_D unsigned wide_node_test (const float4 *__restrict__ wide, int w, const float (&p)[3],
                               int4 &kids)
{
  const float4 *q = wide + 8 * (size_t)w;
  const float4 lx = __ldg (q), ly = __ldg (q + 1), lz = __ldg (q + 2);
  const float4 hx = __ldg (q + 3), hy = __ldg (q + 4), hz = __ldg (q + 5);
  const float4 kk = __ldg (q + 6);
  kids = make_int4 (__float_as_int (kk.x), __float_as_int (kk.y), __float_as_int (kk.z),
                    __float_as_int (kk.w));
  unsigned m = 0u;
  m |= !(p[0] < lx.x || p[1] < ly.x || p[2] < lz.x || p[0] > hx.x || p[1] > hy.x || p[2] > hz.x) ? 1u : 0u;
  m |= !(p[0] < lx.y || p[1] < ly.y || p[2] < lz.y || p[0] > hx.y || p[1] > hy.y || p[2] > hz.y) ? 2u : 0u;
  m |= !(p[0] < lx.z || p[1] < ly.z || p[2] < lz.z || p[0] > hx.z || p[1] > hy.z || p[2] > hz.z) ? 4u : 0u;
  m |= !(p[0] < lx.w || p[1] < ly.w || p[2] < lz.w || p[0] > hx.w || p[1] > hy.w || p[2] > hz.w) ? 8u : 0u;
  return m;
}

template <bool WIDE> struct TraversalStack
{
  static constexpr int kDepth = WIDE ? kWideStack : kStackDepth;
};

// Advance a traversal to its next candidate leaf (left-first DFS, as
// device_mesh.hpp:262-318): returns the leaf, or -1 when the tree is
// exhausted.  After a candidate the caller resumes with cur = todo[sp--].
// WIDE walks the 4-wide tree (lowest hit child first, the other hits
// pushed highest first), else the binary nodes.
template <bool WIDE>
DRB_D int next_leaf (const float4 *__restrict__ nodes, const float4 *__restrict__ wide,
                     const float (&pt)[3], int (&todo)[TraversalStack<WIDE>::kDepth], int &sp,
                     int &cur, int &visited)
{
  constexpr int D = TraversalStack<WIDE>::kDepth;
  while (cur != kBarrier)
  {
    if (cur > -1)
    {
      ++visited;
      if (WIDE)
      {
        int4 k;
        const unsigned m = wide_node_test (wide, cur, pt, k);
        if (m == 0u)
        {
          cur = todo[sp];
          --sp;
        }
        else
        {
          const int f = __ffs (m) - 1;
          if ((m & 8u) && f != 3 && sp < D - 1) todo[++sp] = k.w;
          if ((m & 4u) && f != 2 && sp < D - 1) todo[++sp] = k.z;
          if ((m & 2u) && f != 1 && sp < D - 1) todo[++sp] = k.y;
          cur = f == 0 ? k.x : f == 1 ? k.y : f == 2 ? k.z : k.w;
        }
      }
      else
      {
        bool in_l, in_r;
        int l, r;
        node_point_test_kids (nodes, cur, pt, in_l, in_r, l, r);
        if (!in_l && !in_r)
        {
          cur = todo[sp];
          --sp;
        }
        else
        {
          cur = in_l ? l : r;
          if (in_l && in_r && sp < D - 1) todo[++sp] = r;
        }
      }
    }
    else
    {
      return -cur - 1;
    }
  }
  return -1;
}

struct LocateParams
{
  const float4 *nodes;
  const float4 *wide = nullptr; // 4-wide tree or NULL
  const int *leaf_nodes;
  const int *aabb_ids;
  const float *ref_boxes;
  const float *packed;
  const int *ctrl_idx;
  const float *xyz;
  int stride;
  float tol;
  int max_steps;
  int guess_mode;
  const float *guess;
  const float4 *hull = nullptr; // tet hull planes (drb_tet_hull_planes) or NULL
  const float4 *leaf_maps = nullptr; // per-leaf linear maps (drb_bvh_leaf_maps) or NULL
};

// Uniform-grid candidate lists of a BVH (drb_bvh_grid_build); a separate
// kernel argument, so the tree-walking kernels carry none of it.
struct GridLists
{
  const int *start = nullptr;
  const int *entries = nullptr;  // leaf indices, cell by cell
  const float4 *boxes = nullptr; // per leaf: lo.xyz + element bits, hi.xyz + 0
  int dims[3] = { 1, 1, 1 };
  float origin[3] = { 0.f, 0.f, 0.f };
  float inv[3] = { 0.f, 0.f, 0.f };
};

// Grid lists of a BVH, or empty ones (start null) when it has none.
inline GridLists grid_lists (const drb_bvh *bvh)
{
  GridLists gl;
  if (bvh->grid_start && bvh->grid_entries && bvh->grid_boxes)
  {
    gl.start = bvh->grid_start;
    gl.entries = bvh->grid_entries;
    gl.boxes = (const float4 *)bvh->grid_boxes;
    for (int d = 0; d < 3; ++d)
    {
      gl.dims[d] = bvh->grid_dims[d];
      gl.origin[d] = bvh->grid_origin[d];
      gl.inv[d] = bvh->grid_inv[d];
    }
  }
  return gl;
}

// Cell coordinate of x along one grid axis: floor((x - o) * inv) clamped to
// [0, g - 1].  Monotone in x, so every point of a box [lo, hi] falls in a
// cell between those of lo and hi; the grid build files each leaf under
// that range with this same function.  NaN maps to 0.
DRB_D int grid_axis (float x, float o, float inv, int g)
{
  float v = __fmul_rn (__fsub_rn (x, o), inv);
  v = fminf (fmaxf (v, 0.f), (float)(g - 1));
  return __float2int_rd (v);
}

DRB_D int grid_cell (const int (&dims)[3], const float (&o)[3], const float (&inv)[3],
                     const float (&p)[3])
{
  const int cx = grid_axis (p[0], o[0], inv[0], dims[0]);
  const int cy = grid_axis (p[1], o[1], inv[1], dims[1]);
  const int cz = grid_axis (p[2], o[2], inv[2], dims[2]);
  return (cz * dims[1] + cy) * dims[0] + cx;
}

// Next candidate leaf of a point from its grid cell's list: the entries
// hold every leaf whose box overlaps the cell, in leaf order; each leaf's
// box (the same floats as in its parent's node) is in gl.boxes.  A leaf is
// reached by the left-first traversal exactly when its own box holds the
// point (refit makes every ancestor's box contain it), and that traversal
// meets leaves in index order (each Karras node covers a contiguous range,
// left before right), so this scan yields the traversal's candidates in
// the traversal's order.  cur and end index the entries; -1 when done.
DRB_D int next_grid_leaf (const GridLists &gl, const float (&p)[3], int &cur, int end,
                          int &visited)
{
  while (cur < end)
  {
    const int k = __ldg (gl.entries + cur);
    const float4 a = __ldg (gl.boxes + 2 * (size_t)k);
    const float4 b = __ldg (gl.boxes + 2 * (size_t)k + 1);
    ++cur;
    ++visited;
    if (!(p[0] < a.x || p[1] < a.y || p[2] < a.z || p[0] > b.x || p[1] > b.y || p[2] > b.z))
      return k;
  }
  return -1;
}

// Candidate filter of the batched locate (drb_tet_hull_planes): true when
// the query lies more than kHullMargin * tol * D outside one of the tet's
// hull planes, where no Newton solve can be accepted.
constexpr float kHullMargin = 128.f;
DRB_D bool hull_rejects (const LocateParams &lp, int el, const float (&pt)[3])
{
  const float4 *h = lp.hull + 5 * (size_t)el;
  const float margin = kHullMargin * lp.tol * __ldg (h + 4).x;
  bool out = false;
#pragma unroll
  for (int f = 0; f < 4; ++f)
  {
    const float4 q = __ldg (h + f);
    out |= q.x * pt[0] + q.y * pt[1] + q.z * pt[2] - q.w > margin;
  }
  return out;
}

// Element kinds of the locate templates: drb_shape for volume elements,
// plus the quads of 2D meshes (tensor shape, dim 2).
constexpr int kTensor = DRB_SHAPE_TENSOR;
constexpr int kSimplex = DRB_SHAPE_SIMPLEX;
constexpr int kQuad2D = 2;
constexpr int kTri2D = 3;

// Dofs of an order-P element of kind S, and its reference centre
// coordinate (hex (0.5,0.5,0.5), tet centroid (0.25,0.25,0.25)).
template <int S, int P> constexpr int shape_dofs ()
{
  return S == kSimplex ? tet_dofs<P> () : S == kQuad2D ? (P + 1) * (P + 1)
         : S == kTri2D ? tri_dofs<P> () : (P + 1) * (P + 1) * (P + 1);
}
template <int S> constexpr float shape_centre ()
{
  return S == kSimplex ? 0.25f : S == kTri2D ? (float)(1.0 / 3) : 0.5f;
}

// Tet Newton solve (simplex counterpart of the tensor path below).
template <int P, bool REG>
DRB_D bool solve_in_tet (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                         int &steps, LU3 &lu)
{
  constexpr int ND = tet_dofs<P> ();
  if (lp.packed)
  {
    const float *row = lp.packed + (size_t)el * lp.stride;
    float t[3];
    local_target<ND> (row, pt, t);
    if (REG && P <= 2)
    {
      RegCP<3 * ND> r;
      load_reg_tet<P> (r, row);
      return tet_newton<P> (r, t, x, lp.tol, lp.max_steps, steps, lu);
    }
    PackedCP cp{ row };
    return tet_newton<P> (cp, t, x, lp.tol, lp.max_steps, steps, lu);
  }
  IndirectCP cp{ lp.ctrl_idx + (size_t)el * ND, lp.xyz, 3 };
  return tet_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps, lu);
}

// Quad of a 2D mesh (LocateHack<2>): quad_newton on the packed row.
template <int P, bool REG>
DRB_D bool solve_in_quad (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                          int &steps, LU3 &lu)
{
  constexpr int ND = (P + 1) * (P + 1);
  if (lp.packed)
  {
    const float *row = lp.packed + (size_t)el * lp.stride;
    float t[3];
    local_target<ND> (row, pt, t);
    if (REG)
    {
      RegCP<3 * ND> r;
      load_reg_rows<3 * ND> (r, row);
      return quad_newton<P> (r, t, x, lp.tol, lp.max_steps, steps, lu);
    }
    PackedCP cp{ row };
    return quad_newton<P> (cp, t, x, lp.tol, lp.max_steps, steps, lu);
  }
  IndirectCP cp{ lp.ctrl_idx + (size_t)el * ND, lp.xyz, 3 };
  return quad_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps, lu);
}

// Triangle of a 2D mesh (LocateHack<2>): tri_newton on the packed row.
template <int P, bool REG>
DRB_D bool solve_in_tri (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                         int &steps, LU3 &lu)
{
  constexpr int ND = tri_dofs<P> ();
  if (lp.packed)
  {
    const float *row = lp.packed + (size_t)el * lp.stride;
    float t[3];
    local_target<ND> (row, pt, t);
    if (REG)
    {
      RegCP<3 * ND> r;
      load_reg_rows<3 * ND> (r, row);
      return tri_newton<P> (r, t, x, lp.tol, lp.max_steps, steps, lu);
    }
    PackedCP cp{ row };
    return tri_newton<P> (cp, t, x, lp.tol, lp.max_steps, steps, lu);
  }
  IndirectCP cp{ lp.ctrl_idx + (size_t)el * ND, lp.xyz, 3 };
  return tri_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps, lu);
}

// Newton solve of one point in one element, choosing register-resident or
// L1-read control points by order.
template <int P, bool REG = (P <= 2), int S = kTensor>
DRB_D bool solve_in_element (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                             int &steps, LU3 &lu)
{
  if (S == kSimplex) return solve_in_tet<P, REG> (lp, el, pt, x, steps, lu);
  if (S == kQuad2D) return solve_in_quad<P, REG> (lp, el, pt, x, steps, lu);
  if (S == kTri2D) return solve_in_tri<P, REG> (lp, el, pt, x, steps, lu);
  constexpr int ND = (P + 1) * (P + 1) * (P + 1);
  if (lp.packed)
  {
    // packed rows are relative to the element's first control point
    const float *row = lp.packed + (size_t)el * lp.stride;
    float t[3];
    local_target<ND> (row, pt, t);
    if (REG && P <= 2)
    {
      RegCP<3 * ND> r;
      load_reg_cp<P> (r, row);
      return hex_newton<P> (r, t, x, lp.tol, lp.max_steps, steps, lu);
    }
    PackedCP cp{ row };
    return hex_newton<P> (cp, t, x, lp.tol, lp.max_steps, steps, lu);
  }
  IndirectCP cp{ lp.ctrl_idx + (size_t)el * ND, lp.xyz, 3 };
  return hex_newton<P> (cp, pt, x, lp.tol, lp.max_steps, steps, lu);
}

template <int P, bool REG = (P <= 2)>
DRB_D bool solve_in_element (const LocateParams &lp, int el, const float (&pt)[3], float (&x)[3],
                             int &steps)
{
  LU3 lu;
  return solve_in_element<P, REG> (lp, el, pt, x, steps, lu);
}

// Element rows staged in shared memory by the warp (locate_persistent_kernel
// with shared rows): a packed geometry row (relative coordinates, then the
// origin) at a lane-group slot; reads are plain shared-memory loads.
struct SmemCP
{
  // volatile: read on every use, so the row stays in shared memory instead
  // of being hoisted into 81+ registers across the Newton steps
  const volatile float *p;
  DRB_D float operator() (int i, int k) const { return p[3 * i + k]; }
};

// Newton solve of one point in the element whose packed row is in shared
// memory (same arithmetic as the packed path of solve_in_element).
template <int P>
DRB_D bool solve_in_smem_row (const LocateParams &lp, const float *row, const float (&pt)[3],
                              float (&x)[3], int &steps)
{
  constexpr int ND = (P + 1) * (P + 1) * (P + 1);
  float t[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) t[d] = __fsub_rn (pt[d], row[packed_origin (ND) + d]);
  SmemCP cp{ row };
  return hex_newton<P> (cp, t, x, lp.tol, lp.max_steps, steps);
}

// Initial guess of a candidate leaf's Newton solve (drb_guess_mode).
template <int S = kTensor>
DRB_D void candidate_guess (const LocateParams &lp, int leaf, long long qi, bool first,
                            const float (&pt)[3], float (&x)[3], bool &given)
{
  given = false;
  if (lp.guess_mode == DRB_GUESS_ZERO)
  {
    x[0] = x[1] = x[2] = 0.f;
  }
  else if (lp.guess_mode == DRB_GUESS_SUBBOX_LINEAR && (S == kTensor || S == kSimplex) &&
           lp.leaf_maps)
  {
    // the element map linearised at the leaf's sub-box centre (a tet's:
    // its sub-simplex centroid) c:
    // x = c + J(c)^-1 (p - X(c)); record (c, X(c), J^-1 row-major, 0)
    const float4 *m = lp.leaf_maps + 4 * (size_t)leaf;
    const float4 a = __ldg (m), b = __ldg (m + 1), c = __ldg (m + 2), d = __ldg (m + 3);
    const float r0 = pt[0] - a.w, r1 = pt[1] - b.x, r2 = pt[2] - b.y;
    x[0] = a.x + (b.z * r0 + b.w * r1 + c.x * r2);
    x[1] = a.y + (c.y * r0 + c.z * r1 + c.w * r2);
    x[2] = a.z + (d.x * r0 + d.y * r1 + d.z * r2);
  }
  else if ((lp.guess_mode == DRB_GUESS_SUBREF_CENTER || lp.guess_mode == DRB_GUESS_SUBBOX_LINEAR) &&
           S == kSimplex)
  {
    // subref_center<Simplex> (data_model/subref.hpp:39-48): the origin
    // vertex plus the three axis vertices, times 1/4
    const float *rb = lp.ref_boxes + 12 * (size_t)__ldg (lp.aabb_ids + leaf);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      float sum = __fadd_rn (rb[9 + d], rb[d]);
      sum = __fadd_rn (sum, rb[3 + d]);
      sum = __fadd_rn (sum, rb[6 + d]);
      x[d] = __fmul_rn (sum, 0.25f);
    }
  }
  else if ((lp.guess_mode == DRB_GUESS_SUBREF_CENTER || lp.guess_mode == DRB_GUESS_SUBBOX_LINEAR) &&
           S == kTri2D)
  {
    // subref_center<Simplex> in 2D: origin, then the axis vertices, times 1/3
    const float *rb = lp.ref_boxes + 6 * (size_t)__ldg (lp.aabb_ids + leaf);
#pragma unroll
    for (int d = 0; d < 2; ++d)
      x[d] = __fmul_rn (__fadd_rn (__fadd_rn (rb[4 + d], rb[d]), rb[2 + d]), (float)(1.0 / 3));
    x[2] = 0.f;
  }
  else if ((lp.guess_mode == DRB_GUESS_SUBREF_CENTER || lp.guess_mode == DRB_GUESS_SUBBOX_LINEAR) &&
           S == kQuad2D)
  {
    // SubRef<2,Tensor>: low (u, v), then high (u, v)
    const float *rb = lp.ref_boxes + 4 * (size_t)__ldg (lp.aabb_ids + leaf);
    x[0] = (rb[0] + rb[2]) * 0.5f;
    x[1] = (rb[1] + rb[3]) * 0.5f;
    x[2] = 0.f;
  }
  else if (lp.guess_mode == DRB_GUESS_SUBREF_CENTER || lp.guess_mode == DRB_GUESS_SUBBOX_LINEAR)
  {
    const float *rb = lp.ref_boxes + 6 * (size_t)__ldg (lp.aabb_ids + leaf);
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = (rb[d] + rb[3 + d]) * 0.5f;
  }
  else if (lp.guess_mode == DRB_GUESS_GIVEN && first)
  {
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = lp.guess[3 * (size_t)qi + d];
    given = true;
  }
  else
  {
    x[0] = x[1] = x[2] = shape_centre<S> ();
  }
}

// Newton in one candidate element with the guess-mode fallback: a given
// guess whose solve does not converge within the step budget is retried
// from the element centre.  A guessed solve that converged (it stopped
// before the budget) to a point outside the element has shown that the
// point is not in it, so it is not retried.
template <int P, bool REG = (P <= 2), int S = kTensor>
DRB_D bool solve_candidate (const LocateParams &lp, int leaf, int el, long long qi, bool first,
                            const float (&pt)[3], float (&x)[3], int &iters, LU3 &lu)
{
  bool given;
  candidate_guess<S> (lp, leaf, qi, first, pt, x, given);
  int steps = 0;
  bool found = solve_in_element<P, REG, S> (lp, el, pt, x, steps, lu);
  iters += steps;
  if (!found && given && steps >= lp.max_steps)
  {
    x[0] = x[1] = x[2] = shape_centre<S> ();
    found = solve_in_element<P, REG, S> (lp, el, pt, x, steps, lu);
    iters += steps;
  }
  return found;
}

template <int P, bool REG = (P <= 2), int S = kTensor>
DRB_D bool solve_candidate (const LocateParams &lp, int leaf, int el, long long qi, bool first,
                            const float (&pt)[3], float (&x)[3], int &iters)
{
  LU3 lu;
  return solve_candidate<P, REG, S> (lp, leaf, el, qi, first, pt, x, iters, lu);
}

// solve_candidate on a shared-memory row (same guess and fallback rule).
template <int P>
DRB_D bool solve_candidate_smem (const LocateParams &lp, int leaf, const float *row, long long qi,
                                 bool first, const float (&pt)[3], float (&x)[3], int &iters)
{
  bool given;
  candidate_guess<kTensor> (lp, leaf, qi, first, pt, x, given);
  int steps = 0;
  bool found = solve_in_smem_row<P> (lp, row, pt, x, steps);
  iters += steps;
  if (!found && given && steps >= lp.max_steps)
  {
    x[0] = x[1] = x[2] = 0.5f;
    found = solve_in_smem_row<P> (lp, row, pt, x, steps);
    iters += steps;
  }
  return found;
}

// Full point location of one query (DeviceMesh::locate, device_mesh.hpp:248-354):
// traversal left child first, first converged+inside candidate wins.
template <int P, bool WIDE = false, int S = kTensor>
DRB_D int locate_point (const LocateParams &lp, int qi, const float (&pt)[3], float (&out_ref)[3],
                        int &iters, int &cands, int &nodes, LU3 &lu)
{
  // depth is bounded by the tree height; the binary stack of 64 covers 2^63
  // leaves of a balanced tree and the reference uses the same fixed stack
  int todo[TraversalStack<WIDE>::kDepth];
  int current = 0;
  int sp = 0;
  todo[sp] = kBarrier;
  bool first_candidate = true;
  while (true)
  {
    const int leaf = next_leaf<WIDE> (lp.nodes, lp.wide, pt, todo, sp, current, nodes);
    if (leaf < 0) break;
    const int el = __ldg (lp.leaf_nodes + leaf);
    ++cands;
    float x[3];
    const bool found = solve_candidate<P, (P <= 2), S> (lp, leaf, el, qi, first_candidate, pt, x, iters, lu);
    first_candidate = false;
    if (found)
    {
      out_ref[0] = x[0];
      out_ref[1] = x[1];
      out_ref[2] = x[2];
      return el;
    }
    current = todo[sp];
    --sp;
  }
  return -1;
}

template <int P, bool WIDE = false, int S = kTensor>
DRB_D int locate_point (const LocateParams &lp, int qi, const float (&pt)[3], float (&out_ref)[3],
                        int &iters, int &cands, int &nodes)
{
  LU3 lu;
  return locate_point<P, WIDE, S> (lp, qi, pt, out_ref, iters, cands, nodes, lu);
}

} // namespace drb
