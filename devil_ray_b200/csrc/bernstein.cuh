// Tensor-product Bernstein elements (hex: dim 3, quad: dim 2) of order 1-3
// and the 3x3 LUP solve used by every Newton step.
//
// Reference semantics:
//   - element evaluation with derivatives, Element_impl<dim,ncomp,Tensor,P>::eval_d
//     (data_model/pos_tensor_element.tcc:99-232 general order, :474-499 P1 hex,
//      :610-704 P2 hex, :373-578 P1/P2 quad)
//   - dof order lexicographic, u fastest (pos_tensor_element.tcc:159-180)
//   - LUP factor/solve with partial pivoting, singular when the pivot is
//     below epsilon<float>() = 1e-4 (matrix.hpp:221-373, math.hpp:25)
//
// The evaluation here is sum-factorised (contract u, then v, then w) instead
// of the reference's term-by-term sums: the same polynomial, about half the
// FP32 operations, and FMA-contracted.  Results agree with the reference to
// FP32 rounding; Newton results are compared within the reference-space
// tolerance, not bitwise.
#pragma once

#include "drb_common.cuh"

namespace drb
{

// 1D Bernstein basis of order P and its derivative at t.
template <int P> struct Basis1D;

template <> struct Basis1D<1>
{
  DRB_D static void eval (float t, float (&b)[2], float (&d)[2])
  {
    b[0] = 1.f - t;
    b[1] = t;
    d[0] = -1.f;
    d[1] = 1.f;
  }
};

template <> struct Basis1D<2>
{
  DRB_D static void eval (float t, float (&b)[3], float (&d)[3])
  {
    const float s = 1.f - t;
    b[0] = s * s;
    b[1] = 2.f * t * s;
    b[2] = t * t;
    d[0] = -2.f * s;
    d[1] = 2.f - 4.f * t;
    d[2] = 2.f * t;
  }
};

template <> struct Basis1D<3>
{
  DRB_D static void eval (float t, float (&b)[4], float (&d)[4])
  {
    const float s = 1.f - t;
    const float ts = t * s;
    b[0] = s * s * s;
    b[1] = 3.f * ts * s;
    b[2] = 3.f * ts * t;
    b[3] = t * t * t;
    d[0] = -3.f * s * s;
    d[1] = 3.f * s * s - 6.f * ts;
    d[2] = 6.f * ts - 3.f * t * t;
    d[3] = 3.f * t * t;
  }
};

template <int P> constexpr int hex_dofs () { return (P + 1) * (P + 1) * (P + 1); }
template <int P> constexpr int quad_dofs () { return (P + 1) * (P + 1); }
// Packed element rows (drb_pack_elements), one per element, padded to a
// multiple of 4 floats so every row starts on a 16-byte boundary.
//   geometry (ncomp 3): control points relative to the element's first
//     control point O (P_i - O, rounded once in FP32), then O itself at
//     float offset 3 nd.  Newton then works on X(r) - O and pt - O, whose
//     magnitudes are the element size instead of the domain size, so its
//     rounding noise in reference space no longer grows with the element
//     count (with absolute coordinates a 128^3 mesh in [0,1]^3 sits at
//     about 2e-5, above a 1e-5 tolerance).
//   scalar fields (ncomp 1): the values.
DRB_HD constexpr int packed_stride (int nd, int ncomp)
{
  return ncomp == 3 ? ((3 * nd + 3 + 3) / 4) * 4 : ((nd * ncomp + 3) / 4) * 4;
}
DRB_HD constexpr int packed_origin (int nd) { return 3 * nd; }

// One u-row of control points: components of points i0 .. i0 + P, point
// major.  Element accessors whose rows are 16-byte aligned overload this
// with vector loads (PackedCP at order 3, the volume's field rows).
template <int P, int NC, class CP>
DRB_D void cp_row (const CP &cp, int i0, float (&v)[(P + 1) * NC])
{
#pragma unroll
  for (int a = 0; a <= P; ++a)
#pragma unroll
    for (int k = 0; k < NC; ++k) v[a * NC + k] = cp (i0 + a, k);
}

// Hex element: value X and the three columns dX/du, dX/dv, dX/dw.
// `cp(i, k)` returns component k of control point i.
template <int P, int NC, class CP>
DRB_D void hex_eval_d (const CP &cp, float u, float v, float w, float (&X)[NC],
                       float (&Ju)[NC], float (&Jv)[NC], float (&Jw)[NC])
{
  float bu[P + 1], du[P + 1], bv[P + 1], dv[P + 1], bw[P + 1], dw[P + 1];
  Basis1D<P>::eval (u, bu, du);
  Basis1D<P>::eval (v, bv, dv);
  Basis1D<P>::eval (w, bw, dw);
#pragma unroll
  for (int k = 0; k < NC; ++k) X[k] = Ju[k] = Jv[k] = Jw[k] = 0.f;
#pragma unroll
  for (int c = 0; c <= P; ++c)
  {
    float pv[NC], pu[NC], pdv[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) pv[k] = pu[k] = pdv[k] = 0.f;
#pragma unroll
    for (int b = 0; b <= P; ++b)
    {
      float s[NC], sd[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) s[k] = sd[k] = 0.f;
      float row[(P + 1) * NC];
      cp_row<P, NC> (cp, (c * (P + 1) + b) * (P + 1), row);
#pragma unroll
      for (int a = 0; a <= P; ++a)
      {
#pragma unroll
        for (int k = 0; k < NC; ++k)
        {
          const float q = row[a * NC + k];
          s[k] = fmaf (q, bu[a], s[k]);
          sd[k] = fmaf (q, du[a], sd[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < NC; ++k)
      {
        pv[k] = fmaf (s[k], bv[b], pv[k]);
        pu[k] = fmaf (sd[k], bv[b], pu[k]);
        pdv[k] = fmaf (s[k], dv[b], pdv[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k)
    {
      X[k] = fmaf (pv[k], bw[c], X[k]);
      Ju[k] = fmaf (pu[k], bw[c], Ju[k]);
      Jv[k] = fmaf (pdv[k], bw[c], Jv[k]);
      Jw[k] = fmaf (pv[k], dw[c], Jw[k]);
    }
  }
}

// Hex element value only (no derivatives).
template <int P, int NC, class CP>
DRB_D void hex_eval (const CP &cp, float u, float v, float w, float (&X)[NC])
{
  float bu[P + 1], du[P + 1], bv[P + 1], dv[P + 1], bw[P + 1], dw[P + 1];
  Basis1D<P>::eval (u, bu, du);
  Basis1D<P>::eval (v, bv, dv);
  Basis1D<P>::eval (w, bw, dw);
#pragma unroll
  for (int k = 0; k < NC; ++k) X[k] = 0.f;
#pragma unroll
  for (int c = 0; c <= P; ++c)
  {
    float pv[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) pv[k] = 0.f;
#pragma unroll
    for (int b = 0; b <= P; ++b)
    {
      float s[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) s[k] = 0.f;
#pragma unroll
      for (int a = 0; a <= P; ++a)
      {
        const int i = (c * (P + 1) + b) * (P + 1) + a;
#pragma unroll
        for (int k = 0; k < NC; ++k) s[k] = fmaf (cp (i, k), bu[a], s[k]);
      }
#pragma unroll
      for (int k = 0; k < NC; ++k) pv[k] = fmaf (s[k], bv[b], pv[k]);
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) X[k] = fmaf (pv[k], bw[c], X[k]);
  }
}

// Quad element embedded in 3D (NC = 3) or a scalar on a quad (NC = 1).
template <int P, int NC, class CP>
DRB_D void quad_eval_d (const CP &cp, float u, float v, float (&X)[NC], float (&Ju)[NC],
                        float (&Jv)[NC])
{
  float bu[P + 1], du[P + 1], bv[P + 1], dv[P + 1];
  Basis1D<P>::eval (u, bu, du);
  Basis1D<P>::eval (v, bv, dv);
#pragma unroll
  for (int k = 0; k < NC; ++k) X[k] = Ju[k] = Jv[k] = 0.f;
#pragma unroll
  for (int b = 0; b <= P; ++b)
  {
    float s[NC], sd[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) s[k] = sd[k] = 0.f;
    float row[(P + 1) * NC];
    cp_row<P, NC> (cp, b * (P + 1), row);
#pragma unroll
    for (int a = 0; a <= P; ++a)
    {
#pragma unroll
      for (int k = 0; k < NC; ++k)
      {
        const float q = row[a * NC + k];
        s[k] = fmaf (q, bu[a], s[k]);
        sd[k] = fmaf (q, du[a], sd[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k)
    {
      X[k] = fmaf (s[k], bv[b], X[k]);
      Ju[k] = fmaf (sd[k], bv[b], Ju[k]);
      Jv[k] = fmaf (s[k], dv[b], Jv[k]);
    }
  }
}

// 3x3 LUP factorisation + solve (matrix.hpp:221-373, matrix_mult_inv :461-477).
// A is row-major a[r][c].  Returns false when a pivot is below 1e-4; like the
// reference's Newton stepper, callers still use the solution.
struct LU3
{
  float a[3][3];
  int perm[3];
  bool valid;

  DRB_D void factor (const float (&m)[3][3])
  {
#pragma unroll
    for (int r = 0; r < 3; ++r)
    {
#pragma unroll
      for (int c = 0; c < 3; ++c) a[r][c] = m[r][c];
      perm[r] = r;
    }
    valid = true;
#pragma unroll
    for (int t = 0; t < 3; ++t)
    {
      // pivot search (MatrixLUPFactorFindPivot)
      int max_row = t;
      float max_val = fabsf (a[t][t]);
#pragma unroll
      for (int r = t + 1; r < 3; ++r)
      {
        const float cv = fabsf (a[r][t]);
        if (max_val < cv)
        {
          max_val = cv;
          max_row = r;
        }
      }
      if (max_val < kEpsilon) valid = false;
      if (max_row != t)
      {
#pragma unroll
        for (int r = t + 1; r < 3; ++r)
        {
          if (r == max_row)
          {
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
              const float tmp = a[r][c];
              a[r][c] = a[t][c];
              a[t][c] = tmp;
            }
            const int tp = perm[r];
            perm[r] = perm[t];
            perm[t] = tp;
          }
        }
      }
      // upper-triangle elements (MatrixLUPFactorFindUpperTriangleElements)
#pragma unroll
      for (int c = t + 1; c < 3; ++c) a[t][c] = a[t][c] / a[t][t];
#pragma unroll
      for (int r = t + 1; r < 3; ++r)
#pragma unroll
        for (int c = t + 1; c < 3; ++c) a[r][c] -= a[r][t] * a[t][c];
    }
  }

  DRB_D void solve (const float (&b)[3], float (&x)[3]) const
  {
    float y[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
    {
      const int pr = perm[r];
      y[r] = pr == 0 ? b[0] : (pr == 1 ? b[1] : b[2]);
#pragma unroll
      for (int c = 0; c < r; ++c) y[r] -= a[r][c] * y[c];
      y[r] = y[r] / a[r][r];
    }
#pragma unroll
    for (int r = 2; r >= 0; --r)
    {
      x[r] = y[r];
#pragma unroll
      for (int c = r + 1; c < 3; ++c) x[r] -= a[r][c] * x[c];
    }
  }
};

} // namespace drb
