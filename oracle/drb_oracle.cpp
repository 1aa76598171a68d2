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
template <typename T>
bool newton (int p, const ElemCP &cp, const T *target, T *x, T tol, int max_steps, int &steps)
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
    hex_eval_d<T> (p, 3, cpt, x, X, J);
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
                int &iters, int &cands)
{
  // DeviceMesh::locate (device_mesh.hpp:248-354)
  const int nd = (p + 1) * (p + 1) * (p + 1);
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
      else x[0] = x[1] = x[2] = T (0.5);
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
      bool found = newton<T> (p, cp, tgt, x, T (tol), max_steps, steps);
      iters += steps;
      if (!found && given)
      {
        x[0] = x[1] = x[2] = T (0.5);
        found = newton<T> (p, cp, tgt, x, T (tol), max_steps, steps);
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
