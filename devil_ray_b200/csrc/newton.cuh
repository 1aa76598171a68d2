// Newton inversion of tensor Bernstein elements and BVH point queries.
//
//   hex_newton   InvertibleElement_impl::eval_inverse_local with
//                IterativeMethod::solve (data_model/element.hpp:435-486,
//                newton_solver.hpp:33-74): clamp x to [0,1], eval_d, LUP-solve
//                J dx = target - X(x), x += dx; converged when the inf-norm of
//                the change from the previous (unclamped) iterate is < tol;
//                accept only if converged and is_inside(x, tol)
//                (pos_tensor_element.tcc:49-61).  tol and max_steps are
//                parameters (the reference fixes 1e-4 and 20).
//   Element access goes through a functor cp(i, k) so the same solver runs on
//   register-resident control points (orders 1-2) or L1-resident packed rows.
#pragma once

#include "bernstein.cuh"
#include "drb_common.cuh"

namespace drb
{

DRB_D bool is_inside_ref (const float (&x)[3], float eps)
{
  float mn = 2.f, mx = -1.f;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    mn = fminf (x[d], mn);
    mx = fmaxf (x[d], mx);
  }
  return (mn >= 0.f - eps) && (mx <= 1.f + eps);
}

// Vec::Normlinf (vec.hpp:229-238): fmaxf-based, so a NaN component is skipped.
DRB_D float norm_linf3 (float a, float b, float c)
{
  float m = fmaxf (-a, a);
  m = fmaxf (m, fmaxf (-b, b));
  m = fmaxf (m, fmaxf (-c, c));
  return m;
}

// lu receives the factorised Jacobian of the last step, taken within tol
// (in reference space) of the returned x when the solve converged: the
// volume renderer reuses it for the world-space gradient and for the next
// sample's predictor instead of evaluating the geometry again.
// One step of the hex iteration: clamp x to [0,1]^3, evaluate, LUP-solve
// J dx = target - X(x), x += dx.  hex_newton loops over it; the step-wise
// locate kernel calls it once per round, so both run the same arithmetic.
template <int P, class CP>
DRB_D void hex_step (const CP &cp, const float (&target)[3], float (&x)[3], LU3 &lu)
{
#pragma unroll
  for (int d = 0; d < 3; ++d) x[d] = fminf (1.f, fmaxf (x[d], 0.f));
  float X[3], Ju[3], Jv[3], Jw[3];
  hex_eval_d<P, 3> (cp, x[0], x[1], x[2], X, Ju, Jv, Jw);
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

// Change of the iterate from prev (inf-norm over 3 coordinates), then prev = x.
DRB_D float step_change3 (const float (&x)[3], float (&prev)[3])
{
  const float res = norm_linf3 (x[0] - prev[0], x[1] - prev[1], x[2] - prev[2]);
#pragma unroll
  for (int d = 0; d < 3; ++d) prev[d] = x[d];
  return res;
}

template <int P, class CP>
DRB_D bool hex_newton (const CP &cp, const float (&target)[3], float (&x)[3], float tol,
                       int max_steps, int &steps, LU3 &lu)
{
  float prev[3] = { x[0], x[1], x[2] };
  bool converged = false;
  steps = 0;
  while (steps < max_steps && !converged)
  {
    hex_step<P> (cp, target, x, lu);
    ++steps;
    converged = step_change3 (x, prev) < tol;
  }
  return converged && is_inside_ref (x, tol);
}

template <int P, class CP>
DRB_D bool hex_newton (const CP &cp, const float (&target)[3], float (&x)[3], float tol,
                       int max_steps, int &steps)
{
  LU3 lu;
  return hex_newton<P> (cp, target, x, tol, max_steps, steps, lu);
}

// LocateHack<2>::eval_inverse (data_model/device_mesh.hpp:166-238): a quad
// of a 2D mesh in 3D space with z ignored.  The 3x3 Jacobian is
// [dX/du, dX/dv, e_z]; only the u and v of the LUP solution step x;
// converged when the inf-norm of that 2D step is below tol, accepted if
// converged and inside [0,1]^2 within tol (QuadRefSpace<2>::is_inside,
// pos_tensor_element.tcc:49-61).  x[2] is left at -1, as the reference
// leaves the third coordinate of a 2D Location.
template <int P, class CP>
DRB_D void quad_step (const CP &cp, const float (&target)[3], float (&x)[3], LU3 &lu)
{
  x[0] = fminf (1.f, fmaxf (x[0], 0.f));
  x[1] = fminf (1.f, fmaxf (x[1], 0.f));
  float X[3], Ju[3], Jv[3];
  quad_eval_d<P, 3> (cp, x[0], x[1], X, Ju, Jv);
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
}

// Change over the two reference coordinates of a quad, then prev = x.
DRB_D float step_change2 (const float (&x)[3], float (&prev)[3])
{
  const float a = x[0] - prev[0], b = x[1] - prev[1];
  prev[0] = x[0];
  prev[1] = x[1];
  return fmaxf (fmaxf (-a, a), fmaxf (-b, b));
}

DRB_D bool quad_inside (const float (&x)[3], float tol)
{
  const float mn = fminf (fminf (x[0], 2.f), x[1]);
  const float mx = fmaxf (fmaxf (x[0], -1.f), x[1]);
  return mn >= 0.f - tol && mx <= 1.f + tol;
}

template <int P, class CP>
DRB_D bool quad_newton (const CP &cp, const float (&target)[3], float (&x)[3], float tol,
                        int max_steps, int &steps, LU3 &lu)
{
  float prev[3] = { x[0], x[1], x[2] };
  bool converged = false;
  steps = 0;
  while (steps < max_steps && !converged)
  {
    quad_step<P> (cp, target, x, lu);
    ++steps;
    converged = step_change2 (x, prev) < tol;
  }
  x[2] = -1.f;
  return converged && quad_inside (x, tol);
}

// Control points of one element read through the packed element-major copy.
struct PackedCP
{
  const float *__restrict__ p;
  DRB_D float operator() (int i, int k) const { return __ldg (p + 3 * i + k); }
};

// Order-3 rows of a packed element: 12 floats at 48-byte offsets of a
// 16-byte aligned row, so three float4 loads instead of twelve scalar ones.
template <> DRB_D void cp_row<3, 3, PackedCP> (const PackedCP &cp, int i0, float (&v)[12])
{
  const float4 *q = reinterpret_cast<const float4 *> (cp.p + 3 * i0);
  const float4 a = __ldg (q), b = __ldg (q + 1), c = __ldg (q + 2);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  v[8] = c.x; v[9] = c.y; v[10] = c.z; v[11] = c.w;
}

// Order-2 rows: 9 floats at 36-byte offsets.  The offset modulo 16 bytes
// is known once the caller's loops are unrolled, and picks the widest
// aligned loads that cover the row (3 or 4 loads instead of 9).
template <> DRB_D void cp_row<2, 3, PackedCP> (const PackedCP &cp, int i0, float (&v)[9])
{
  const float *q = cp.p + 3 * i0;
  const int mis = (3 * i0) & 3; // floats past a 16-byte boundary
  if (mis == 0)
  {
    const float4 a = __ldg (reinterpret_cast<const float4 *> (q));
    const float4 b = __ldg (reinterpret_cast<const float4 *> (q + 4));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    v[8] = __ldg (q + 8);
  }
  else if (mis == 1)
  {
    v[0] = __ldg (q);
    const float2 a = __ldg (reinterpret_cast<const float2 *> (q + 1));
    const float4 b = __ldg (reinterpret_cast<const float4 *> (q + 3));
    const float2 c = __ldg (reinterpret_cast<const float2 *> (q + 7));
    v[1] = a.x; v[2] = a.y;
    v[3] = b.x; v[4] = b.y; v[5] = b.z; v[6] = b.w;
    v[7] = c.x; v[8] = c.y;
  }
  else if (mis == 2)
  {
    const float2 a = __ldg (reinterpret_cast<const float2 *> (q));
    const float4 b = __ldg (reinterpret_cast<const float4 *> (q + 2));
    const float2 c = __ldg (reinterpret_cast<const float2 *> (q + 6));
    v[0] = a.x; v[1] = a.y;
    v[2] = b.x; v[3] = b.y; v[4] = b.z; v[5] = b.w;
    v[6] = c.x; v[7] = c.y;
    v[8] = __ldg (q + 8);
  }
  else
  {
    v[0] = __ldg (q);
    const float4 a = __ldg (reinterpret_cast<const float4 *> (q + 1));
    const float4 b = __ldg (reinterpret_cast<const float4 *> (q + 5));
    v[1] = a.x; v[2] = a.y; v[3] = a.z; v[4] = a.w;
    v[5] = b.x; v[6] = b.y; v[7] = b.z; v[8] = b.w;
  }
}

// pt - O for a packed geometry row with ND control points (O stored at
// packed_origin(ND)); t is the Newton target in the row's frame.
template <int ND> DRB_D void local_target (const float *__restrict__ row, const float (&pt)[3], float (&t)[3])
{
#pragma unroll
  for (int d = 0; d < 3; ++d) t[d] = __fsub_rn (pt[d], __ldg (row + packed_origin (ND) + d));
}

// X + O: a position evaluated from a packed geometry row, in world space.
template <int ND> DRB_D void to_world (const float *__restrict__ row, float (&X)[3])
{
#pragma unroll
  for (int d = 0; d < 3; ++d) X[d] = __fadd_rn (X[d], __ldg (row + packed_origin (ND) + d));
}

// Control points of one element read through the reference's double
// indirection val[ctrl_idx[e*nd+i]] (data_model/dof_access.hpp:23-54).
struct IndirectCP
{
  const int *__restrict__ idx;
  const float *__restrict__ val;
  int ncomp;
  DRB_D float operator() (int i, int k) const
  {
    return __ldg (val + (size_t)ncomp * __ldg (idx + i) + k);
  }
};

// Register-resident copy of an element (orders 1-2: 24 or 81 floats).
template <int N> struct RegCP
{
  float v[N];
  DRB_D float operator() (int i, int k) const { return v[3 * i + k]; }
};

// The first N floats of a packed row (16-byte aligned) into registers.
template <int N> DRB_D void load_reg_rows (RegCP<N> &r, const float *p)
{
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

template <int P> DRB_D void load_reg_cp (RegCP<3 * (P + 1) * (P + 1) * (P + 1)> &r, const float *p)
{
  constexpr int N = 3 * (P + 1) * (P + 1) * (P + 1);
  // packed rows start on a float4 boundary (drb_packed_stride)
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
