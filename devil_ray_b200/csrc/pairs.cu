// Per-(element, point) kernels used to generate and check the learned guess:
//   map_points_kernel    physical point X_e(r) of reference points r
//                        (Element::eval, pos_tensor_element.tcc:99-232)
//   newton_pairs_kernel  Newton inversion of each point in a given element
//                        (eval_inverse_local, data_model/element.hpp:435-486)
//                        from the element centre or a given guess; the
//                        labels of the training set are these solutions.
#include "drb_common.cuh"
#include "drb_internal.h"
#include "newton.cuh"
#include "simplex.cuh"

namespace drb
{
namespace
{

// K: 0 hex, 1 tet, 2 quad of a 2D mesh
template <int P, int K>
__global__ void map_points_kernel (const float *__restrict__ packed, int stride,
                                   const int *__restrict__ elem, const float *__restrict__ ref,
                                   int n, float *__restrict__ pts)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = elem[i];
  float X[3] = { NAN, NAN, NAN };
  if (e >= 0)
  {
    const float *row = packed + (size_t)e * stride;
    PackedCP cp{ row };
    const float u = ref[3 * (size_t)i], v = ref[3 * (size_t)i + 1], w = ref[3 * (size_t)i + 2];
    if (K == 1)
    {
      float Ju[3], Jv[3], Jw[3];
      tet_eval_d<P, 3> (cp, u, v, w, X, Ju, Jv, Jw);
      to_world<tet_dofs<P> ()> (row, X);
    }
    else if (K == 2)
    {
      float Ju[3], Jv[3];
      quad_eval_d<P, 3> (cp, u, v, X, Ju, Jv);
      to_world<(P + 1) * (P + 1)> (row, X);
    }
    else if (K == 3)
    {
      float Ju[3], Jv[3];
      tri_eval_d<P, 3> (cp, u, v, X, Ju, Jv);
      to_world<tri_dofs<P> ()> (row, X);
    }
    else
    {
      hex_eval<P, 3> (cp, u, v, w, X);
      to_world<(P + 1) * (P + 1) * (P + 1)> (row, X);
    }
  }
  pts[3 * (size_t)i] = X[0];
  pts[3 * (size_t)i + 1] = X[1];
  pts[3 * (size_t)i + 2] = X[2];
}

template <int P>
__global__ void newton_pairs_kernel (const float *__restrict__ packed, int stride,
                                     const int *__restrict__ elem, const float *__restrict__ pts,
                                     int n, float tol, int max_steps,
                                     const float *__restrict__ guess, float *__restrict__ ref,
                                     int *__restrict__ found, int *__restrict__ iters)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = elem[i];
  float x[3] = { 0.5f, 0.5f, 0.5f };
  if (guess)
  {
    x[0] = guess[3 * (size_t)i];
    x[1] = guess[3 * (size_t)i + 1];
    x[2] = guess[3 * (size_t)i + 2];
  }
  int steps = 0;
  bool ok = false;
  if (e >= 0)
  {
    const float pw[3] = { pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2] };
    const float *row = packed + (size_t)e * stride;
    float pt[3];
    local_target<(P + 1) * (P + 1) * (P + 1)> (row, pw, pt);
    if (P <= 2)
    {
      RegCP<3 * (P + 1) * (P + 1) * (P + 1)> r;
      load_reg_cp<P> (r, row);
      ok = hex_newton<P> (r, pt, x, tol, max_steps, steps);
    }
    else
    {
      PackedCP cp{ row };
      ok = hex_newton<P> (cp, pt, x, tol, max_steps, steps);
    }
  }
  ref[3 * (size_t)i] = x[0];
  ref[3 * (size_t)i + 1] = x[1];
  ref[3 * (size_t)i + 2] = x[2];
  if (found) found[i] = ok ? 1 : 0;
  if (iters) iters[i] = steps;
}

// UnstructuredField::eval at located points (unstructured_field.cpp:214-245):
// value of the scalar field at (cell, ref); cell -1 -> empty value.
template <int P, int K>
__global__ void field_eval_kernel (const float *__restrict__ packed, int stride,
                                   const int *__restrict__ cell, const float *__restrict__ ref,
                                   int n, float empty, float *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = cell[i];
  float v = empty;
  if (e >= 0)
  {
    struct F
    {
      const float *p;
      DRB_D float operator() (int q, int) const { return __ldg (p + q); }
    } cp{ packed + (size_t)e * stride };
    float X[1];
    const float u = ref[3 * (size_t)i], vv = ref[3 * (size_t)i + 1], w = ref[3 * (size_t)i + 2];
    if (K == 1)
    {
      float Ju[1], Jv[1], Jw[1];
      tet_eval_d<P, 1> (cp, u, vv, w, X, Ju, Jv, Jw);
    }
    else if (K == 2)
    {
      float Ju[1], Jv[1];
      quad_eval_d<P, 1> (cp, u, vv, X, Ju, Jv);
    }
    else if (K == 3)
    {
      float Ju[1], Jv[1];
      tri_eval_d<P, 1> (cp, u, vv, X, Ju, Jv);
    }
    else
    {
      hex_eval<P, 1> (cp, u, vv, w, X);
    }
    v = X[0];
  }
  out[i] = v;
}

int check_pairs (const drb_mesh *m, int n, bool any_kind = false)
{
  if (!m || !m->packed || m->ncomp != 3 || m->order < 1 || m->order > 3 || n < 0 ||
      (m->dim != 3 && !(any_kind && m->dim == 2)))
  {
    set_last_error ("pairs: needs a packed hex geometry mesh of order 1..3");
    return DRB_ERR_INVALID_ARG;
  }
  if (m->shape != DRB_SHAPE_TENSOR && !(any_kind && m->shape == DRB_SHAPE_SIMPLEX))
  {
    set_last_error ("pairs: element shape not supported here");
    return DRB_ERR_UNSUPPORTED;
  }
  return DRB_OK;
}

// 0 hex, 1 tet, 2 quad, 3 triangle (the K of the kernels above)
int kind_of (const drb_mesh *m)
{
  if (m->shape == DRB_SHAPE_SIMPLEX) return m->dim == 2 ? 3 : 1;
  return m->dim == 2 ? 2 : 0;
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_map_points (const drb_mesh *mesh, const int *elem, const float *ref, int n,
                               float *pts, void *stream)
{
  int st = check_pairs (mesh, n, true);
  if (st) return st;
  if (n == 0) return DRB_OK;
  if (!elem || !ref || !pts)
  {
    set_last_error ("map_points: NULL array");
    return DRB_ERR_INVALID_ARG;
  }
  const int stride = packed_stride (mesh_nd (mesh), 3);
  cudaStream_t s = (cudaStream_t)stream;
  const int b = div_up (n, 256);
#define DRB_MP(P, K) map_points_kernel<P, K><<<b, 256, 0, s>>> (mesh->packed, stride, elem, ref, n, pts)
#define DRB_MPK(K) (mesh->order == 1 ? DRB_MP (1, K) : mesh->order == 2 ? DRB_MP (2, K) : DRB_MP (3, K))
  const int kind = kind_of (mesh);
  if (kind == 1) DRB_MPK (1);
  else if (kind == 2) DRB_MPK (2);
  else if (kind == 3) DRB_MPK (3);
  else DRB_MPK (0);
#undef DRB_MPK
#undef DRB_MP
  return check_launch ("map_points_kernel");
}

extern "C" int drb_newton_pairs (const drb_mesh *mesh, const int *elem, const float *pts, int n,
                                 float tol, int max_steps, const float *guess, float *ref,
                                 int *found, int *iters, void *stream)
{
  int st = check_pairs (mesh, n);
  if (st) return st;
  if (n == 0) return DRB_OK;
  if (!elem || !pts || !ref || !(tol > 0.f) || max_steps < 0)
  {
    set_last_error ("newton_pairs: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  const int nd = (mesh->order + 1) * (mesh->order + 1) * (mesh->order + 1);
  const int stride = packed_stride (nd, 3);
  cudaStream_t s = (cudaStream_t)stream;
  const int b = div_up (n, 128);
  if (mesh->order == 1)
    newton_pairs_kernel<1><<<b, 128, 0, s>>> (mesh->packed, stride, elem, pts, n, tol, max_steps, guess, ref, found, iters);
  else if (mesh->order == 2)
    newton_pairs_kernel<2><<<b, 128, 0, s>>> (mesh->packed, stride, elem, pts, n, tol, max_steps, guess, ref, found, iters);
  else
    newton_pairs_kernel<3><<<b, 128, 0, s>>> (mesh->packed, stride, elem, pts, n, tol, max_steps, guess, ref, found, iters);
  return check_launch ("newton_pairs_kernel");
}

extern "C" int drb_field_eval (const drb_mesh *field, const int *cell, const float *ref, int n,
                               float empty_value, float *values, void *stream)
{
  if (!field || !field->packed || field->ncomp != 1 || field->order < 1 || field->order > 3 ||
      n < 0 || (n > 0 && (!cell || !ref || !values)) ||
      !((field->dim == 3 || field->dim == 2) &&
        (field->shape == DRB_SHAPE_TENSOR || field->shape == DRB_SHAPE_SIMPLEX)))
  {
    set_last_error ("field_eval: needs a packed scalar hex, tet or quad field of order 1..3");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  const int stride = packed_stride (mesh_nd (field), 1);
  cudaStream_t s = (cudaStream_t)stream;
  const int b = div_up (n, 256);
#define DRB_FE(P, K) field_eval_kernel<P, K><<<b, 256, 0, s>>> (field->packed, stride, cell, ref, n, empty_value, values)
#define DRB_FEK(K) (field->order == 1 ? DRB_FE (1, K) : field->order == 2 ? DRB_FE (2, K) : DRB_FE (3, K))
  const int kind = kind_of (field);
  if (kind == 1) DRB_FEK (1);
  else if (kind == 2) DRB_FEK (2);
  else if (kind == 3) DRB_FEK (3);
  else DRB_FEK (0);
#undef DRB_FEK
#undef DRB_FE
  return check_launch ("field_eval_kernel");
}
