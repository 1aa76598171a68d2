// Simplex (tetrahedral) Bernstein elements of order 1-3: evaluation with
// derivatives, the reference-space inside test and the Newton inversion.
//
// Reference semantics:
//   - dof order: multi-index (i, j, k) of u, v, w with the fourth index
//     l = p - i - j - k of t = 1 - u - v - w implicit; i fastest, then j,
//     then k (elem_ops.hpp:19-47, cartesian_to_tet_idx).  Vertex (0,0,0) is
//     node 0, u = 1 is node p, v = 1 node (p+1)(p+2)/2 - 1, w = 1 the last.
//   - evaluation, Element_impl<3,ncomp,Simplex,General>::eval_d
//     (elem_ops.hpp:901-1010): the same polynomial, written here as one de
//     Casteljau step over the order p-1 basis, which gives the position and
//     the three derivatives from one pass over the dofs.  The reference's
//     fixed-order Linear specialisation (elem_ops.hpp:785-815) writes all
//     three derivatives into out_deriv[0] and leaves C[3] out of them; the
//     general-order path, which the reference also instantiates
//     (TetMesh = UnstructuredMesh<Tet3>), is the one restated.
//   - is_inside (pos_simplex_element.tcc:479-491): the smallest of u, v, w
//     and 1 - u - v - w (subtracted in that order) must be >= -eps.
//   - the Newton stepper is the tensor one (element.hpp:435-486): clamp each
//     coordinate to [0, 1], solve J dx = target - X(x), converged when the
//     change is below tol, accepted if converged and inside.
#pragma once

#include "bernstein.cuh"
#include "drb_common.cuh"
#include "newton.cuh"

namespace drb
{

DRB_HD constexpr int tet_dofs (int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
template <int P> constexpr int tet_dofs () { return (P + 1) * (P + 2) * (P + 3) / 6; }

// Position of multi-index (i, j, k) in an order-p element's dof list: the
// nodes of the k layers below, the j rows below in layer k, then i.
DRB_HD constexpr int tet_index (int i, int j, int k, int p)
{
  int base = 0;
  for (int q = 0; q < k; ++q) base += (p - q + 1) * (p - q + 2) / 2;
  for (int q = 0; q < j; ++q) base += p - k - q + 1;
  return base + i;
}

DRB_HD constexpr int factorial (int n) { return n <= 1 ? 1 : n * factorial (n - 1); }

// Multinomial coefficient n! / (i! j! k! l!) with l = n - i - j - k.
DRB_HD constexpr float multinomial (int n, int i, int j, int k)
{
  return (float)(factorial (n) / (factorial (i) * factorial (j) * factorial (k) *
                                  factorial (n - i - j - k)));
}

// X(u,v,w) and its derivatives for an order-P tet, cp(i, k) = component k of
// dof i.  With B the order P-1 basis over (u, v, w, t):
//   X     = sum_a B_a(u,v,w,t) (u C[a+e_u] + v C[a+e_v] + w C[a+e_w] + t C[a+e_t])
//   dX/du = P sum_a B_a (C[a+e_u] - C[a+e_t])   (likewise v, w)
template <int P, int NC, class CP>
DRB_D void tet_eval_d (const CP &cp, float u, float v, float w, float (&X)[NC], float (&Ju)[NC],
                       float (&Jv)[NC], float (&Jw)[NC])
{
  const float t = 1.f - (u + v + w);
  float pu[P], pv[P], pw[P], pt[P];
  pu[0] = pv[0] = pw[0] = pt[0] = 1.f;
#pragma unroll
  for (int q = 1; q < P; ++q)
  {
    pu[q] = pu[q - 1] * u;
    pv[q] = pv[q - 1] * v;
    pw[q] = pw[q - 1] * w;
    pt[q] = pt[q - 1] * t;
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) X[c] = Ju[c] = Jv[c] = Jw[c] = 0.f;
#pragma unroll
  for (int k = 0; k < P; ++k)
#pragma unroll
    for (int j = 0; j < P - k; ++j)
#pragma unroll
      for (int i = 0; i < P - k - j; ++i)
      {
        const int l = P - 1 - i - j - k;
        const float B = multinomial (P - 1, i, j, k) * pu[i] * pv[j] * pw[k] * pt[l];
        const int it = tet_index (i, j, k, P);
        const int iu = tet_index (i + 1, j, k, P);
        const int iv = tet_index (i, j + 1, k, P);
        const int iw = tet_index (i, j, k + 1, P);
#pragma unroll
        for (int c = 0; c < NC; ++c)
        {
          const float ct = cp (it, c), cu = cp (iu, c), cv = cp (iv, c), cw = cp (iw, c);
          X[c] += B * (u * cu + v * cv + w * cw + t * ct);
          Ju[c] += B * (cu - ct);
          Jv[c] += B * (cv - ct);
          Jw[c] += B * (cw - ct);
        }
      }
#pragma unroll
  for (int c = 0; c < NC; ++c)
  {
    Ju[c] *= (float)P;
    Jv[c] *= (float)P;
    Jw[c] *= (float)P;
  }
}

// ---- triangles (the faces of tets) ----
DRB_HD constexpr int tri_dofs (int p) { return (p + 1) * (p + 2) / 2; }
template <int P> constexpr int tri_dofs () { return (P + 1) * (P + 2) / 2; }

// Position of multi-index (i, j) in an order-p triangle's dof list: i
// fastest, then j (cartesian_to_tri_idx, elem_ops.hpp:19-30).
DRB_HD constexpr int tri_index (int i, int j, int p) { return (2 * p + 3 - j) * j / 2 + i; }

// X(u,v) and its derivatives for an order-P triangle, with t = 1 - u - v
// and B the order P-1 basis: X = sum_a B_a (u C[a+e_u] + v C[a+e_v] +
// t C[a+e_t]), dX/du = P sum_a B_a (C[a+e_u] - C[a+e_t]), likewise v
// (Element_impl<2,ncomp,Simplex,*>::eval_d, elem_ops.hpp:700-780,
// pos_simplex_element.tcc:510-600).
template <int P, int NC, class CP>
DRB_D void tri_eval_d (const CP &cp, float u, float v, float (&X)[NC], float (&Ju)[NC],
                       float (&Jv)[NC])
{
  const float t = 1.f - (u + v);
  float pu[P], pv[P], pt[P];
  pu[0] = pv[0] = pt[0] = 1.f;
#pragma unroll
  for (int q = 1; q < P; ++q)
  {
    pu[q] = pu[q - 1] * u;
    pv[q] = pv[q - 1] * v;
    pt[q] = pt[q - 1] * t;
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) X[c] = Ju[c] = Jv[c] = 0.f;
#pragma unroll
  for (int j = 0; j < P; ++j)
#pragma unroll
    for (int i = 0; i < P - j; ++i)
    {
      const int l = P - 1 - i - j;
      const float B = multinomial (P - 1, i, j, 0) * pu[i] * pv[j] * pt[l];
      const int it = tri_index (i, j, P);
      const int iu = tri_index (i + 1, j, P);
      const int iv = tri_index (i, j + 1, P);
#pragma unroll
      for (int c = 0; c < NC; ++c)
      {
        const float ct = cp (it, c), cu = cp (iu, c), cv = cp (iv, c);
        X[c] += B * (u * cu + v * cv + t * ct);
        Ju[c] += B * (cu - ct);
        Jv[c] += B * (cv - ct);
      }
    }
#pragma unroll
  for (int c = 0; c < NC; ++c)
  {
    Ju[c] *= (float)P;
    Jv[c] *= (float)P;
  }
}

// TriRefSpace<2>::is_inside (pos_simplex_element.tcc:479-491), eps =
// epsilon<Float>() = 1e-4 when called without one.
DRB_D bool is_inside_tri (float u, float v, float eps)
{
  float mn = fminf (u, 2.f);
  float t = __fsub_rn (1.f, u);
  mn = fminf (v, mn);
  t = __fsub_rn (t, v);
  mn = fminf (t, mn);
  return mn >= 0.f - eps;
}

// LocateHack<2> (data_model/device_mesh.hpp:166-238) on a triangle of a 2D
// mesh: the quad_newton iteration with the triangle's evaluation and
// TriRefSpace<2>::is_inside(ref, tol).
template <int P, class CP>
DRB_D bool tri_newton (const CP &cp, const float (&target)[3], float (&x)[3], float tol,
                       int max_steps, int &steps, LU3 &lu)
{
  float prev[3] = { x[0], x[1], x[2] };
  bool converged = false;
  steps = 0;
  while (steps < max_steps && !converged)
  {
    x[0] = fminf (1.f, fmaxf (x[0], 0.f));
    x[1] = fminf (1.f, fmaxf (x[1], 0.f));
    float X[3], Ju[3], Jv[3];
    tri_eval_d<P, 3> (cp, x[0], x[1], X, Ju, Jv);
    float dy[3], J[3][3], dx[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
    {
      dy[r] = target[r] - X[r];
      J[r][0] = Ju[r];
      J[r][1] = Jv[r];
      J[r][2] = (r == 2) ? 1.f : 0.f;
    }
    lu.factor (J);
    lu.solve (dy, dx);
    x[0] += dx[0];
    x[1] += dx[1];
    ++steps;
    converged = step_change2 (x, prev) < tol;
  }
  x[2] = -1.f;
  return converged && is_inside_tri (x[0], x[1], tol);
}

// TriRefSpace<3>::is_inside(ref, eps) (pos_simplex_element.tcc:493-505).
DRB_D bool is_inside_simplex (const float (&x)[3], float eps)
{
  float mn = 2.f;
  float t = 1.f;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    mn = fminf (x[d], mn);
    t = __fsub_rn (t, x[d]);
  }
  mn = fminf (t, mn);
  return mn >= 0.f - eps;
}

template <int P, class CP>
DRB_D void tet_step (const CP &cp, const float (&target)[3], float (&x)[3], LU3 &lu)
{
#pragma unroll
  for (int d = 0; d < 3; ++d) x[d] = fminf (1.f, fmaxf (x[d], 0.f));
  float X[3], Ju[3], Jv[3], Jw[3];
  tet_eval_d<P, 3> (cp, x[0], x[1], x[2], X, Ju, Jv, Jw);
  float dy[3], J[3][3], dx[3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
  {
    dy[r] = target[r] - X[r];
    J[r][0] = Ju[r];
    J[r][1] = Jv[r];
    J[r][2] = Jw[r];
  }
  lu.factor (J);
  lu.solve (dy, dx);
#pragma unroll
  for (int d = 0; d < 3; ++d) x[d] += dx[d];
}

template <int P, class CP>
DRB_D bool tet_newton (const CP &cp, const float (&target)[3], float (&x)[3], float tol,
                       int max_steps, int &steps, LU3 &lu)
{
  float prev[3] = { x[0], x[1], x[2] };
  bool converged = false;
  steps = 0;
  while (steps < max_steps && !converged)
  {
    tet_step<P> (cp, target, x, lu);
    ++steps;
    converged = step_change3 (x, prev) < tol;
  }
  return converged && is_inside_simplex (x, tol);
}

// Register-resident tet row (orders 1-2: 12 or 30 floats of a packed row).
template <int P> DRB_D void load_reg_tet (RegCP<3 * tet_dofs<P> ()> &r, const float *p)
{
  constexpr int N = 3 * tet_dofs<P> ();
  const float4 *p4 = reinterpret_cast<const float4 *> (p);
#pragma unroll
  for (int q = 0; q < N / 4; ++q)
  {
    const float4 t = __ldg (p4 + q);
    r.v[4 * q] = t.x;
    r.v[4 * q + 1] = t.y;
    r.v[4 * q + 2] = t.z;
    r.v[4 * q + 3] = t.w;
  }
#pragma unroll
  for (int q = (N / 4) * 4; q < N; ++q) r.v[q] = __ldg (p + q);
}

} // namespace drb
