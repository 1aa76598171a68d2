// CPU restatement of the reference's point-location algorithm: test oracle.
//
// Test infrastructure only (see drb_oracle.h).  Each function cites the
// reference code it restates.  Element evaluation uses the closed-form
// tensor Bernstein basis B_i^p(t) = C(p,i) t^i (1-t)^(p-i) and its
// derivative p (B_{i-1}^{p-1} - B_i^{p-1}), the same polynomial the
// reference evaluates with its Horner/lower-order scheme
// (data_model/pos_tensor_element.tcc:99-232); run in double it is the FP64
// reference point for error statements, run in float it restates the
// reference's FP32 Newton.
#include "drb_oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace
{

template <typename T> void basis (int p, T t, T *b, T *d)
{
  // B_i^p via binomials and powers; derivative via order p-1 basis.
  std::vector<T> lower (p + 1, T (0));
  auto bern = [] (int q, int i, T x) -> T {
    if (i < 0 || i > q) return T (0);
    double c = 1.0;
    for (int k = 1; k <= i; ++k) c = c * (q - i + k) / k;
    T v = T (c);
    for (int k = 0; k < i; ++k) v *= x;
    for (int k = 0; k < q - i; ++k) v *= (T (1) - x);
    return v;
  };
  for (int i = 0; i <= p; ++i)
  {
    b[i] = bern (p, i, t);
    d[i] = (p == 0) ? T (0) : T (p) * (bern (p - 1, i - 1, t) - bern (p - 1, i, t));
  }
}

// Element_impl<3,ncomp,Tensor,P>::eval_d: value and d/du, d/dv, d/dw.
template <typename T, typename CP>
void hex_eval_d (int p, int ncomp, const CP &cp, const T *r, T *X, T *J)
{
  T bu[16], du[16], bv[16], dv[16], bw[16], dw[16];
  basis<T> (p, r[0], bu, du);
  basis<T> (p, r[1], bv, dv);
  basis<T> (p, r[2], bw, dw);
  for (int k = 0; k < ncomp; ++k)
  {
    X[k] = 0;
    J[k] = J[ncomp + k] = J[2 * ncomp + k] = 0;
  }
  int i = 0;
  for (int c = 0; c <= p; ++c)
    for (int b = 0; b <= p; ++b)
      for (int a = 0; a <= p; ++a, ++i)
        for (int k = 0; k < ncomp; ++k)
        {
          const T q = cp (i, k);
          X[k] += q * bu[a] * bv[b] * bw[c];
          J[k] += q * du[a] * bv[b] * bw[c];
          J[ncomp + k] += q * bu[a] * dv[b] * bw[c];
          J[2 * ncomp + k] += q * bu[a] * bv[b] * dw[c];
        }
}

// MatrixLUPFactor / MatrixLUPSolve (matrix.hpp:221-373): partial pivoting,
// Crout form with unit-diagonal U.
template <typename T> bool lup_solve3 (T A[3][3], const T *bvec, T *x)
{
  int perm[3] = { 0, 1, 2 };
  bool valid = true;
  const T eps = sizeof (T) == 4 ? T (1e-4) : T (1e-8);
  for (int t = 0; t < 3; ++t)
  {
    int mr = t;
    T mv = std::fabs (A[t][t]);
    for (int r = t + 1; r < 3; ++r)
      if (mv < std::fabs (A[r][t]))
      {
        mv = std::fabs (A[r][t]);
        mr = r;
      }
    if (mv < eps) valid = false;
    if (mr != t)
    {
      for (int c = 0; c < 3; ++c) std::swap (A[mr][c], A[t][c]);
      std::swap (perm[mr], perm[t]);
    }
    for (int c = t + 1; c < 3; ++c) A[t][c] /= A[t][t];
    for (int r = t + 1; r < 3; ++r)
      for (int c = t + 1; c < 3; ++c) A[r][c] -= A[r][t] * A[t][c];
  }
  T y[3];
  for (int r = 0; r < 3; ++r)
  {
    y[r] = bvec[perm[r]];
    for (int c = 0; c < r; ++c) y[r] -= A[r][c] * y[c];
    y[r] /= A[r][r];
  }
  for (int r = 2; r >= 0; --r)
  {
    x[r] = y[r];
    for (int c = r + 1; c < 3; ++c) x[r] -= A[r][c] * x[c];
  }
  return valid;
}

template <typename T> T maxabs3 (T a, T b, T c)
{
  // Vec::Normlinf (vec.hpp:229-238), fmax-based like the reference
  T m = std::fmax (-a, a);
  m = std::fmax (m, std::fmax (-b, b));
  m = std::fmax (m, std::fmax (-c, c));
  return m;
}

// Control points of one element.  With an origin o (local frame), the value
// is the FP32 difference P_i - o, as the packed element rows of the CUDA
// path hold them (origin = the element's first control point).
struct ElemCP
{
  const int *idx;
  const float *xyz;
  const float *o = nullptr;
  double operator() (int i, int k) const
  {
    const float v = xyz[3 * (size_t)idx[i] + k];
    return o ? (double)(float)(v - o[k]) : (double)v;
  }
};

// eval_inverse_local + IterativeMethod::solve (data_model/element.hpp:435-486,
// newton_solver.hpp:60-74), tol and max_steps as parameters; accept iff
// converged and is_inside(x, tol) (pos_tensor_element.tcc:49-61).
template <typename T, typename CPT> void tet_eval_d (int p, int ncomp, const CPT &cp, const T *r, T *X, T *J);
template <typename T> bool inside_simplex (const T *x, T eps);

template <typename T>
bool newton (int p, const ElemCP &cp, const T *target, T *x, T tol, int max_steps, int &steps,
             bool simplex = false)
{
  struct CPT
  {
    const ElemCP &c;
    T operator() (int i, int k) const { return T (c (i, k)); }
  } cpt{ cp };
  T prev[3] = { x[0], x[1], x[2] };
  bool conv = false;
  steps = 0;
  while (steps < max_steps && !conv)
  {
    for (int d = 0; d < 3; ++d) x[d] = std::fmin (T (1), std::fmax (x[d], T (0)));
    T X[3], J[9];
    if (simplex) tet_eval_d<T> (p, 3, cpt, x, X, J);
    else hex_eval_d<T> (p, 3, cpt, x, X, J);
    T A[3][3], dy[3], dx[3];
    for (int r = 0; r < 3; ++r)
    {
      dy[r] = target[r] - X[r];
      for (int c = 0; c < 3; ++c) A[r][c] = J[3 * c + r];
    }
    lup_solve3<T> (A, dy, dx);
    for (int d = 0; d < 3; ++d) x[d] += dx[d];
    ++steps;
    conv = maxabs3 (x[0] - prev[0], x[1] - prev[1], x[2] - prev[2]) < tol;
    for (int d = 0; d < 3; ++d) prev[d] = x[d];
  }
  if (!conv) return false;
  if (simplex) return inside_simplex<T> (x, tol);
  T mn = 2, mx = -1;
  for (int d = 0; d < 3; ++d)
  {
    mn = std::fmin (x[d], mn);
    mx = std::fmax (x[d], mx);
  }
  return mn >= T (0) - tol && mx <= T (1) + tol;
}

template <typename T>
int locate_one (int p, const int *ctrl_idx, const float *xyz, const float *nodes, const int *leaf_nodes,
                const int *aabb_ids, const float *ref_boxes, const float *pt, float tol,
                int max_steps, int guess_mode, const float *guess, int local_frame, float *out_ref,
                int &iters, int &cands, bool simplex = false)
{
  // DeviceMesh::locate (device_mesh.hpp:248-354)
  const int nd = simplex ? (p + 1) * (p + 2) * (p + 3) / 6 : (p + 1) * (p + 1) * (p + 1);
  const T centre = simplex ? T (0.25) : T (0.5);
  int todo[64];
  int cur = 0, sp = 0;
  todo[0] = -2000000000;
  bool first = true;
  while (cur != -2000000000)
  {
    if (cur > -1)
    {
      const float *a = nodes + 4 * (size_t)cur;
      const bool in_l = !(pt[0] < a[0] || pt[1] < a[1] || pt[2] < a[2] || pt[0] > a[3] ||
                          pt[1] > a[4] || pt[2] > a[5]);
      const bool in_r = !(pt[0] < a[6] || pt[1] < a[7] || pt[2] < a[8] || pt[0] > a[9] ||
                          pt[1] > a[10] || pt[2] > a[11]);
      if (!in_l && !in_r)
      {
        cur = todo[sp--];
      }
      else
      {
        int l, r;
        std::memcpy (&l, a + 12, 4);
        std::memcpy (&r, a + 13, 4);
        cur = in_l ? l : r;
        if (in_l && in_r && sp < 63) todo[++sp] = r;
      }
    }
    else
    {
      const int leaf = -cur - 1;
      const int el = leaf_nodes[leaf];
      ++cands;
      T x[3];
      bool given = false;
      if (guess_mode == 0) x[0] = x[1] = x[2] = 0;
      else if (guess_mode == 2 && simplex)
      {
        // subref_center<Simplex> (subref.hpp:39-48)
        const float *rb = ref_boxes + 12 * (size_t)aabb_ids[leaf];
        for (int d = 0; d < 3; ++d)
        {
          float sum = rb[9 + d];
          sum += rb[d];
          sum += rb[3 + d];
          sum += rb[6 + d];
          x[d] = T (sum * 0.25f);
        }
      }
      else if (guess_mode == 2)
      {
        const float *rb = ref_boxes + 6 * (size_t)aabb_ids[leaf];
        for (int d = 0; d < 3; ++d) x[d] = (T (rb[d]) + T (rb[3 + d])) * T (0.5);
      }
      else if (guess_mode == 3 && first)
      {
        for (int d = 0; d < 3; ++d) x[d] = guess[d];
        given = true;
      }
      else x[0] = x[1] = x[2] = centre;
      first = false;
      ElemCP cp{ ctrl_idx + (size_t)el * nd, xyz };
      T tgt[3] = { pt[0], pt[1], pt[2] };
      if (local_frame)
      {
        // the target relative to the first control point, in FP32
        cp.o = xyz + 3 * (size_t)ctrl_idx[(size_t)el * nd];
        for (int d = 0; d < 3; ++d) tgt[d] = T ((float)(pt[d] - cp.o[d]));
      }
      int steps = 0;
      bool found = newton<T> (p, cp, tgt, x, T (tol), max_steps, steps, simplex);
      iters += steps;
      // the centre retry only after a guessed solve that used its whole
      // step budget (one that converged outside the element has shown the
      // point is not in it)
      if (!found && given && steps >= max_steps)
      {
        x[0] = x[1] = x[2] = centre;
        found = newton<T> (p, cp, tgt, x, T (tol), max_steps, steps, simplex);
        iters += steps;
      }
      if (found)
      {
        for (int d = 0; d < 3; ++d) out_ref[d] = (float)x[d];
        return el;
      }
      cur = todo[sp--];
    }
  }
  return -1;
}

} // namespace

extern "C" void orc_hex_eval_d (int p, int ncomp, const double *cp, int n, const double *ref,
                                double *X, double *J)
{
  struct CPD
  {
    const double *c;
    int nc;
    double operator() (int i, int k) const { return c[nc * i + k]; }
  } f{ cp, ncomp };
  for (int q = 0; q < n; ++q) hex_eval_d<double> (p, ncomp, f, ref + 3 * q, X + ncomp * q, J + 3 * ncomp * q);
}

extern "C" void orc_locate (int p, int n_elem, const int *ctrl_idx, const float *xyz, int n_inner,
                            const float *inner_nodes, const int *leaf_nodes, const int *aabb_ids,
                            const float *ref_boxes, int n, const float *pts, float tol,
                            int max_steps, int guess_mode, const float *guess, int use_double,
                            int local_frame, int *cell, float *ref, int *iters, int *cands)
{
  (void)n_elem;
  (void)n_inner;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i)
  {
    float r[3] = { -1.f, -1.f, -1.f };
    int it = 0, ca = 0;
    const float *g = guess ? guess + 3 * (size_t)i : nullptr;
    int c = use_double
            ? locate_one<double> (p, ctrl_idx, xyz, inner_nodes, leaf_nodes, aabb_ids, ref_boxes,
                                  pts + 3 * (size_t)i, tol, max_steps, guess_mode, g, local_frame, r, it, ca)
            : locate_one<float> (p, ctrl_idx, xyz, inner_nodes, leaf_nodes, aabb_ids, ref_boxes,
                                 pts + 3 * (size_t)i, tol, max_steps, guess_mode, g, local_frame, r, it, ca);
    cell[i] = c;
    if (c < 0) r[0] = r[1] = r[2] = -1.f;
    for (int d = 0; d < 3; ++d) ref[3 * (size_t)i + d] = r[d];
    if (iters) iters[i] = it;
    if (cands) cands[i] = ca;
  }
}

extern "C" void orc_newton_fp64 (int p, const int *ctrl_idx, const float *xyz, int n,
                                 const int *elem, const float *pts, double *ref_out, int *ok)
{
  const int nd = (p + 1) * (p + 1) * (p + 1);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i)
  {
    double x[3] = { 0.5, 0.5, 0.5 };
    int steps = 0;
    const double tgt[3] = { pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2] };
    bool conv = false;
    if (elem[i] >= 0)
    {
      ElemCP cp{ ctrl_idx + (size_t)elem[i] * nd, xyz };
      // converge without the inside test: the element is given
      newton<double> (p, cp, tgt, x, 1e-13, 60, steps);
      conv = steps < 60;
    }
    for (int d = 0; d < 3; ++d) ref_out[3 * (size_t)i + d] = x[d];
    ok[i] = conv ? 1 : 0;
  }
}

// ---- simplex (tet) elements ---------------------------------------------

namespace
{

// Layered dof index of multi-index (i, j, k) in an order-p tet: the nodes of
// the k layers below, of the j rows below in layer k, then i (the order the
// general-order evaluator walks, elem_ops.hpp:945-1030).
int tet_index (int i, int j, int k, int p)
{
  int base = 0;
  for (int q = 0; q < k; ++q) base += (p - q + 1) * (p - q + 2) / 2;
  for (int q = 0; q < j; ++q) base += p - k - q + 1;
  return base + i;
}

// The reference's cartesian_to_tet_idx (elem_ops.hpp:32-47) with e = p + 1,
// whose in-layer term does not shrink with the layer.
int tet_index_reference (int i, int j, int k, int p)
{
  const int e = p + 1;
  return (((-1 - e) * 3 + k) * k + (3 * e + 6) * e + 2) * k / 6 + (2 * e + 1 - j) * j / 2 + i;
}

double factorial (int n) { return n <= 1 ? 1.0 : n * factorial (n - 1); }

float box_measure (const float *b)
{
  const float l0 = b[1] - b[0], l1 = b[3] - b[2], l2 = b[5] - b[4];
  float vol = 1.f * l0 * l1 * l2;
  if (vol == 0.f) vol = 2.f * l0 * l1 + 2.f * l1 * l2 + 2.f * l2 * l0;
  return vol;
}

void hull (const float *cps, int nd, float *b)
{
  for (int k = 0; k < 3; ++k)
  {
    b[2 * k] = INFINITY;
    b[2 * k + 1] = -INFINITY;
  }
  for (int i = 0; i < nd; ++i)
    for (int k = 0; k < 3; ++k)
    {
      b[2 * k] = std::fmin (b[2 * k], cps[3 * i + k]);
      b[2 * k + 1] = std::fmax (b[2 * k + 1], cps[3 * i + k]);
    }
}

void scale_range (float &mn, float &mx, float s)
{
  if (mn > mx) return;
  const float c = 0.5f * (mn + mx);
  const float delta = s * 0.5f * (mx - mn);
  mn = std::fmin (mn, c - delta);
  mx = std::fmax (mx, c + delta);
}

// split_inplace<3,Simplex> (elem_ops.hpp:1270-1311) at factor 0.5, with the
// dof index chosen by `ref_index`.
void tet_split (float *cps, int p, int v0, int v1, bool ref_index)
{
  const int avail = 0xf & ~(1 << v0) & ~(1 << v1);
  const int v2 = (avail & 1) ? 0 : (avail & 2) ? 1 : (avail & 4) ? 2 : 3;
  const int v3 = 6 - v0 - v1 - v2;
  int b[4];
  for (b[v3] = 0; b[v3] < p; ++b[v3])
    for (b[v2] = 0; b[v2] < p - b[v3]; ++b[v2])
    {
      const int gph = b[v2] + b[v3];
      for (int nu = p - gph; nu >= 1; --nu)
        for (b[v0] = p - gph; b[v0] > p - gph - nu; --b[v0])
        {
          b[v1] = p - gph - b[v0];
          int bl[4];
          bl[v0] = b[v0] - 1;
          bl[v1] = b[v1] + 1;
          bl[v2] = b[v2];
          bl[v3] = b[v3];
          const int r = ref_index ? tet_index_reference (b[0], b[1], b[2], p) : tet_index (b[0], b[1], b[2], p);
          const int l = ref_index ? tet_index_reference (bl[0], bl[1], bl[2], p) : tet_index (bl[0], bl[1], bl[2], p);
          for (int k = 0; k < 3; ++k) cps[3 * r + k] = cps[3 * r + k] * 0.5f + cps[3 * l + k] * 0.5f;
        }
    }
}

// Closed-form Bernstein simplex value and u, v, w derivatives (the
// polynomial of Element_impl<3,ncomp,Simplex,General>::eval_d,
// elem_ops.hpp:901-1030); J holds the d/du, d/dv, d/dw blocks.
template <typename T, typename CPT> void tet_eval_d (int p, int ncomp, const CPT &cp, const T *r, T *X, T *J)
{
  const T u = r[0], v = r[1], w = r[2];
  const T t = T (1) - u - v - w;
  for (int c = 0; c < ncomp; ++c) X[c] = J[c] = J[ncomp + c] = J[2 * ncomp + c] = T (0);
  auto pw = [] (T a, int e) {
    T q = T (1);
    for (int z = 0; z < e; ++z) q *= a;
    return q;
  };
  for (int k = 0; k <= p; ++k)
    for (int j = 0; j <= p - k; ++j)
      for (int i = 0; i <= p - k - j; ++i)
      {
        const int l = p - i - j - k;
        const T m = T (factorial (p) / (factorial (i) * factorial (j) * factorial (k) * factorial (l)));
        const T B = m * pw (u, i) * pw (v, j) * pw (w, k) * pw (t, l);
        const T tl1 = l ? T (l) * pw (t, l - 1) : T (0);
        const T du = m * ((i ? T (i) * pw (u, i - 1) : T (0)) * pw (t, l) - tl1 * pw (u, i)) * pw (v, j) * pw (w, k);
        const T dv = m * ((j ? T (j) * pw (v, j - 1) : T (0)) * pw (t, l) - tl1 * pw (v, j)) * pw (u, i) * pw (w, k);
        const T dw = m * ((k ? T (k) * pw (w, k - 1) : T (0)) * pw (t, l) - tl1 * pw (w, k)) * pw (u, i) * pw (v, j);
        const int idx = tet_index (i, j, k, p);
        for (int c = 0; c < ncomp; ++c)
        {
          const T q = cp (idx, c);
          X[c] += B * q;
          J[c] += du * q;
          J[ncomp + c] += dv * q;
          J[2 * ncomp + c] += dw * q;
        }
      }
}

// TriRefSpace<3>::is_inside(ref, eps) (pos_simplex_element.tcc:493-505).
template <typename T> bool inside_simplex (const T *x, T eps)
{
  T mn = T (2), t = T (1);
  for (int d = 0; d < 3; ++d)
  {
    mn = std::fmin (x[d], mn);
    t -= x[d];
  }
  mn = std::fmin (t, mn);
  return mn >= T (0) - eps;
}

} // namespace

extern "C" void orc_locate_tet (int p, const int *ctrl_idx, const float *xyz, const float *inner_nodes,
                                const int *leaf_nodes, const int *aabb_ids, const float *ref_boxes,
                                int n, const float *pts, float tol, int max_steps, int guess_mode,
                                const float *guess, int use_double, int local_frame, int *cell,
                                float *ref, int *iters, int *cands)
{
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i)
  {
    float r[3] = { -1.f, -1.f, -1.f };
    int it = 0, ca = 0;
    const float *g = guess ? guess + 3 * (size_t)i : nullptr;
    int c = use_double
            ? locate_one<double> (p, ctrl_idx, xyz, inner_nodes, leaf_nodes, aabb_ids, ref_boxes,
                                  pts + 3 * (size_t)i, tol, max_steps, guess_mode, g, local_frame, r, it, ca, true)
            : locate_one<float> (p, ctrl_idx, xyz, inner_nodes, leaf_nodes, aabb_ids, ref_boxes,
                                 pts + 3 * (size_t)i, tol, max_steps, guess_mode, g, local_frame, r, it, ca, true);
    cell[i] = c;
    if (c < 0) r[0] = r[1] = r[2] = -1.f;
    for (int d = 0; d < 3; ++d) ref[3 * (size_t)i + d] = r[d];
    if (iters) iters[i] = it;
    if (cands) cands[i] = ca;
  }
}

extern "C" void orc_tet_subboxes (int p, int n_elem, const int *ctrl_idx, const float *xyz,
                                  int reference_index, float *aabbs6, float *ref12)
{
  const int nd = (p + 1) * (p + 2) * (p + 3) / 6;
  // boxes are contiguous, nd dofs each, as in the reference's scratch
  // (mesh_utils.cpp:548-551); the reference index reaches dof nd at order 3,
  // i.e. dof 0 of the next box, and one spare dof follows the last box
  const int slot = nd;
  constexpr int NB = 33;
#pragma omp parallel for schedule(static)
  for (int el = 0; el < n_elem; ++el)
  {
    std::vector<float> cps ((size_t)NB * slot * 3 + 3, 0.f);
    float boxes[NB][6], refs[NB][12];
    for (int i = 0; i < nd; ++i)
      for (int k = 0; k < 3; ++k) cps[3 * i + k] = xyz[3 * (size_t)ctrl_idx[(size_t)el * nd + i] + k];
    hull (cps.data (), nd, boxes[0]);
    const float universe[12] = { 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0 };
    std::memcpy (refs[0], universe, sizeof (universe));
    for (int count = 1; count < NB; ++count)
    {
      int max_id = 0;
      float max_m = box_measure (boxes[0]);
      for (int b = 1; b < count; ++b)
      {
        const float m = box_measure (boxes[b]);
        if (m > max_m)
        {
          max_id = b;
          max_m = m;
        }
      }
      // pick_binary_split<Simplex> (mesh_utils.cpp:455-480)
      const float *rm = refs[max_id];
      int dv = 0, tv = 1;
      float max_l2 = 0.f;
      for (int a = 0; a < 3; ++a)
        for (int b = a + 1; b < 4; ++b)
        {
          float l2 = 0.f;
          for (int k = 0; k < 3; ++k)
          {
            const float e = rm[3 * a + k] - rm[3 * b + k];
            l2 += e * e;
          }
          if (l2 > max_l2)
          {
            dv = a;
            tv = b;
            max_l2 = l2;
          }
        }
      // split_subref<Simplex> (ref_space.hpp:133-146)
      float sp[3];
      for (int k = 0; k < 3; ++k) sp[k] = refs[max_id][3 * tv + k] * 0.5f + refs[max_id][3 * dv + k] * 0.5f;
      std::memcpy (refs[count], refs[max_id], sizeof (refs[0]));
      for (int k = 0; k < 3; ++k)
      {
        refs[max_id][3 * dv + k] = sp[k];
        refs[count][3 * tv + k] = sp[k];
      }
      float *mother = cps.data () + (size_t)max_id * slot * 3;
      float *dghter = cps.data () + (size_t)count * slot * 3;
      std::memcpy (dghter, mother, sizeof (float) * nd * 3);
      tet_split (mother, p, dv, tv, reference_index != 0);
      tet_split (dghter, p, tv, dv, reference_index != 0);
      hull (mother, nd, boxes[max_id]);
      hull (dghter, nd, boxes[count]);
    }
    const float s = (float)1.000001;
    for (int b = 0; b < NB; ++b)
    {
      float bx[6];
      std::memcpy (bx, boxes[b], sizeof (bx));
      for (int k = 0; k < 3; ++k) scale_range (bx[2 * k], bx[2 * k + 1], s);
      std::memcpy (aabbs6 + 6 * ((size_t)el * NB + b), bx, sizeof (bx));
      std::memcpy (ref12 + 12 * ((size_t)el * NB + b), refs[b], sizeof (refs[b]));
    }
  }
}

// Closed-form Bernstein simplex: X = sum_b C_b p!/(i! j! k! l!) u^i v^j w^k t^l
// with t = 1 - u - v - w, and its u, v, w derivatives, in double.
extern "C" void orc_tet_eval_d (int p, int ncomp, const double *cp, int n, const double *ref,
                                double *X, double *J)
{
  for (int q = 0; q < n; ++q)
  {
    const double u = ref[3 * q], v = ref[3 * q + 1], w = ref[3 * q + 2];
    const double t = 1.0 - u - v - w;
    double *x = X + ncomp * q;
    double *jj = J + 3 * ncomp * q;
    for (int c = 0; c < ncomp; ++c) x[c] = jj[c] = jj[ncomp + c] = jj[2 * ncomp + c] = 0.0;
    auto pw = [] (double a, int e) {
      double r = 1.0;
      for (int z = 0; z < e; ++z) r *= a;
      return r;
    };
    for (int k = 0; k <= p; ++k)
      for (int j = 0; j <= p - k; ++j)
        for (int i = 0; i <= p - k - j; ++i)
        {
          const int l = p - i - j - k;
          const double m = factorial (p) / (factorial (i) * factorial (j) * factorial (k) * factorial (l));
          const double B = m * pw (u, i) * pw (v, j) * pw (w, k) * pw (t, l);
          // dB/du = m (i u^(i-1) ... t^l - l u^i ... t^(l-1))
          const double du = m * ((i ? i * pw (u, i - 1) : 0.0) * pw (t, l) - (l ? l * pw (t, l - 1) : 0.0) * pw (u, i)) * pw (v, j) * pw (w, k);
          const double dv = m * ((j ? j * pw (v, j - 1) : 0.0) * pw (t, l) - (l ? l * pw (t, l - 1) : 0.0) * pw (v, j)) * pw (u, i) * pw (w, k);
          const double dw = m * ((k ? k * pw (w, k - 1) : 0.0) * pw (t, l) - (l ? l * pw (t, l - 1) : 0.0) * pw (w, k)) * pw (u, i) * pw (v, j);
          const int idx = tet_index (i, j, k, p);
          for (int c = 0; c < ncomp; ++c)
          {
            const double cv = cp[ncomp * idx + c];
            x[c] += B * cv;
            jj[c] += du * cv;
            jj[ncomp + c] += dv * cv;
            jj[2 * ncomp + c] += dw * cv;
          }
        }
  }
}
