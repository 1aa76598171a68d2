/* CPU restatement of the reference's point-location algorithm (test oracle).
 *
 * Test infrastructure: only tests/, __graft_entry__.smoke() and the bench's
 * CPU-baseline leg load this library; the product never does.
 *
 * Parity of this restatement is pinned two ways: against the known answers
 * of the reference's t_dray_external_evals test fixture (iota control values,
 * orders 1-5) and against the reference itself (oracle/_ref, built from its
 * sources) on the same meshes and points.
 */
#ifndef DRB_ORACLE_H
#define DRB_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Tensor Bernstein hex eval with derivatives at n reference points, order p
 * (any p >= 0), ncomp components; cp = (p+1)^3 * ncomp values of one element
 * (u fastest).  X: n*ncomp, J: n*3*ncomp (d/du, d/dv, d/dw blocks).  double. */
void orc_hex_eval_d (int p, int ncomp, const double *cp, int n, const double *ref, double *X,
                     double *J);

/* Point location over a given BVH in the reference layout, with the
 * reference's traversal order.  use_double selects the FP64 Newton.
 * guess_mode as drb_guess_mode; guess (n*3) for mode 3.  local_frame != 0
 * evaluates each candidate relative to its first control point in FP32, as
 * the CUDA path's packed rows do (the reference uses absolute coordinates).
 * OpenMP over points. */
void orc_locate (int p, int n_elem, const int *ctrl_idx, const float *xyz, int n_inner,
                 const float *inner_nodes, const int *leaf_nodes, const int *aabb_ids,
                 const float *ref_boxes, int n, const float *pts, float tol, int max_steps,
                 int guess_mode, const float *guess, int use_double, int local_frame,
                 int *cell, float *ref, int *iters, int *cands);

/* FP64 Newton solve of each (point, element) pair from the element centre
 * to tol 1e-13, up to 60 steps; ref_out = the FP64 solution (n*3), ok[i] = 1
 * when converged. */
void orc_newton_fp64 (int p, const int *ctrl_idx, const float *xyz, int n, const int *elem,
                      const float *pts, double *ref_out, int *ok);

/* Per-tet sub-boxes of construct_bvh (mesh_utils.cpp:514-677) for order-p
 * tets: 33 per element, aabbs6 (scaled by 1.000001) and ref12 (the
 * reference sub-simplex: u, v, w axis vertices, then the origin), element
 * major.  reference_index != 0 linearises the split's dof multi-indices with
 * the reference's cartesian_to_tet_idx (elem_ops.hpp:32-47), which for
 * orders >= 2 addresses other dofs than the evaluators' layout; 0 uses that
 * layout.  float arithmetic in the reference's operation order. */
void orc_tet_subboxes (int p, int n_elem, const int *ctrl_idx, const float *xyz,
                       int reference_index, float *aabbs6, float *ref12);

/* Bernstein tet eval with derivatives at n reference points, order p (any
 * p >= 0), ncomp components; cp = (p+1)(p+2)(p+3)/6 * ncomp values of one
 * element in the reference's dof order.  X: n*ncomp, J: n*3*ncomp.  double. */
void orc_tet_eval_d (int p, int ncomp, const double *cp, int n, const double *ref, double *X,
                     double *J);

/* orc_locate for order-p tets: simplex evaluation, inside test and
 * sub-simplex centre guess (ref_boxes 12 floats per sub-box), element centre
 * (0.25,0.25,0.25). */
void orc_locate_tet (int p, const int *ctrl_idx, const float *xyz, const float *inner_nodes,
                     const int *leaf_nodes, const int *aabb_ids, const float *ref_boxes, int n,
                     const float *pts, float tol, int max_steps, int guess_mode, const float *guess,
                     int use_double, int local_frame, int *cell, float *ref, int *iters, int *cands);

#ifdef __cplusplus
}
#endif
#endif
