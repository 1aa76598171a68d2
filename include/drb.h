/*
 * drb.h - C-ABI of the B200-native (sm_100a) ray-element hot path.
 *
 * Plain C types, device pointers and sizes; no C++ or torch types.  Every
 * entry point takes a cudaStream_t (as void*, NULL = legacy default stream),
 * enqueues its work on it and returns a drb_status.  Buffers named "device"
 * must be device-accessible; "host" buffers are read or written on the host
 * after the stream has been synchronised by the call where noted.
 *
 * Each entry point names the reference interface (Devil Ray, src/dray/...)
 * whose behaviour it replaces.
 */
#ifndef DRB_H
#define DRB_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference throws dray::DRayError (error.hpp:41-49) on
 * host-side misuse and only prints device errors (error_check.hpp:17-28);
 * here every failure is returned, with a message in drb_last_error(). */
enum drb_status
{
  DRB_OK = 0,
  DRB_ERR_INVALID_ARG = 1,
  DRB_ERR_OOM = 2,
  DRB_ERR_CUDA = 3,
  DRB_ERR_QUEUE_GIVEUP = 4, /* a bounded device-side wait ran out */
  DRB_ERR_UNSUPPORTED = 5
};

/* Initial guess for the per-candidate Newton solve of point location. */
enum drb_guess_mode
{
  /* (0,0,0): the reference as compiled with zero-initialised locals; its
   * DeviceMesh::locate passes use_init_guess=true with an uninitialised
   * guess (data_model/device_mesh.hpp:327-334). */
  DRB_GUESS_ZERO = 0,
  /* element centre: (0.5,0.5,0.5) for tensor elements, the centroid
   * (0.25,0.25,0.25) for tets; the plain GPU path. */
  DRB_GUESS_ELEM_CENTER = 1,
  /* centre of the candidate leaf's reference sub-box, the reference's
   * intended guess (device_mesh.hpp:161-162). */
  DRB_GUESS_SUBREF_CENTER = 2,
  /* the element map linearised at the candidate leaf's reference sub-box
   * centre c (a tet's: its sub-simplex centroid): x0 = c + J(c)^-1 (p - X(c)),
   * from the per-leaf maps of drb_bvh_leaf_maps (3D meshes; without them,
   * and on 2D meshes, as DRB_GUESS_SUBREF_CENTER).
   * No reference counterpart: the reference's guess is its sub-box centre. */
  DRB_GUESS_SUBBOX_LINEAR = 4,
  /* caller-provided guess per point for its first candidate element (e.g.
   * the learned guess), element centre for later candidates and as the
   * fallback when the guessed solve does not converge within max_steps (a
   * guessed solve that converged outside the element is not retried). */
  DRB_GUESS_GIVEN = 3
};

/* Element shape of a drb_mesh (ElemType, data_model/elem_attr.hpp). */
enum drb_shape
{
  DRB_SHAPE_TENSOR = 0,  /* hex (dim 3), quad (dim 2): (order+1)^dim dofs */
  DRB_SHAPE_SIMPLEX = 1  /* tet (dim 3): (order+1)(order+2)(order+3)/6 dofs in
                            the reference's order (i fastest, then j, then k;
                            elem_ops.hpp:901-1030); triangle (dim 2):
                            (order+1)(order+2)/2 dofs, i fastest */
};

/* A Bernstein mesh or field: GridFunction<ncomp> of the reference
 * (data_model/grid_function.hpp:19-30).  dim 3 = hex or tet, dim 2 = quad;
 * shape (drb_shape) selects tensor or simplex elements.  Tet meshes are
 * accepted by drb_pack_elements, drb_elem_subboxes, drb_lbvh_build,
 * drb_bvh_widen, drb_locate, drb_locate_batched (and its ordered, host and
 * allocation-free forms, and drb_locate_tune), drb_field_eval,
 * drb_map_points, the volume renderer (drb_volume_integrate,
 * drb_volume_render, with a tet scalar field) and drb_mesh_boundary, whose
 * triangle faces (dim 2, simplex) drb_surface_intersect and
 * drb_surface_shade render; the hex-only face-neighbour table and the
 * learned guess return DRB_ERR_UNSUPPORTED for them.  2D quad and triangle
 * meshes (dim 2) are located by the same locate entry points and evaluated
 * by drb_field_eval and drb_map_points, besides their use as surfaces. */
typedef struct drb_mesh
{
  int dim;               /* 3 hex or tet, 2 quad or triangle */
  int order;             /* polynomial order 1..3 */
  int ncomp;             /* 3 geometry, 1 scalar field */
  int n_elem;
  int n_ctrl;
  const int *ctrl_idx;   /* device int32[n_elem * drb_elem_dofs()] */
  const float *values;   /* device float[n_ctrl * ncomp] */
  const float *packed;   /* optional device float[n_elem * drb_packed_stride_shape()]:
                            element-major copy made by drb_pack_elements(), or NULL */
  const int *face_neighbors; /* optional device int32[6 * n_elem] of a hex or
                            int32[4 * n_elem] of a tet geometry mesh
                            (drb_mesh_face_neighbors), or NULL */
  int shape;             /* drb_shape; 0 (tensor) when zero-initialised */
  const float *hull_planes; /* optional device float[20 * n_elem] of a tet geometry
                            mesh (drb_tet_hull_planes), or NULL */
} drb_mesh;

/* Bounding planes of each tet of a geometry mesh (no reference counterpart):
 * four outward unit normals n_f with offsets d_f such that n_f . x <= d_f on
 * the whole element (the vertex tet's face planes pushed out to the farthest
 * control point; Bernstein elements lie in their control points' hull), then
 * (D, 0, 0, 0) with D the diagonal of the control points' box; 20 floats per
 * tet.  With drb_mesh.hull_planes set, the batched locate skips the Newton
 * solve of a candidate tet whose planes put the query more than 128 tol D
 * outside: such a solve cannot be accepted, so the results are those of the
 * unfiltered solve. */
int drb_tet_hull_planes (const drb_mesh *mesh, float *planes, void *stream);

/* Face neighbours of a hex or tet mesh (no reference counterpart; faces
 * are matched by their corner control points, as MeshBoundary matches them,
 * mesh_utils.cpp:98-398): for a hex, neighbors[6 e + f] is the element
 * across face f of element e (f = u0, u1, v0, v1, w0, w1); for a tet,
 * neighbors[4 e + f] with f = u=0, v=0, w=0, u+v+w=1; -1 on the boundary.
 * The volume march uses it (through drb_mesh.face_neighbors) to step into
 * the next element across the face a ray leaves by before searching the
 * BVH. */
int drb_mesh_face_neighbors (const drb_mesh *mesh, int *neighbors, void *stream);

/* Linear BVH in the reference's layout (bvh.hpp:16-37, device_bvh.hpp:15-28). */
typedef struct drb_bvh
{
  int n_inner;           /* n_leaf - 1 */
  int n_leaf;
  float *inner_nodes;    /* device float[16 * n_inner]: 4 x float4 per node */
  int *leaf_nodes;       /* device int32[n_leaf]: element id per sorted leaf */
  int *aabb_ids;         /* device int32[n_leaf]: sub-box id per sorted leaf */
  float *ref_boxes;      /* device float[n_leaf * drb_ref_box_floats()]: reference
                            sub-box per sub-box id (tensor: low then high corner;
                            simplex: u, v, w axis vertices, then the origin) */
  float bounds[6];       /* host: xmin,xmax,ymin,ymax,zmin,zmax (filled by the build) */
  /* Optional 4-wide collapse of the same tree for the batched kernels
   * (drb_bvh_widen); NULL: they traverse the binary nodes. */
  float *wide_nodes;     /* device float[32 * n_wide]: 8 x float4 per node */
  int n_wide;
  int wide_depth;        /* wide levels (root = 1) */
  /* Optional per-leaf linear maps for DRB_GUESS_SUBBOX_LINEAR
   * (drb_bvh_leaf_maps); NULL: that guess falls back to the sub-box centre. */
  float *leaf_maps;      /* device float[16 * n_leaf] */
  /* Optional uniform-grid candidate lists for the batched kernels
   * (drb_bvh_grid_size + drb_bvh_grid_build); NULL: they traverse the tree.
   * Cell (cx, cy, cz) is (cz * dims[1] + cy) * dims[0] + cx, with
   * c = clamp(floor((x - origin) * inv), 0, dims - 1) per axis. */
  int *grid_start;       /* device int32[n_cells + 1]: list of cell c = entries
                            [grid_start[c], grid_start[c + 1]) */
  int *grid_entries;     /* device int32[n_entries]: sorted leaf indices */
  float *grid_boxes;     /* device float[8 * n_leaf]: per sorted leaf its box low
                            corner, its element id (int bits), its high corner,
                            0 (the floats of its parent's node record) */
  int grid_dims[3];
  float grid_origin[3];
  float grid_inv[3];     /* cells per unit length (0 on a flat axis) */
} drb_bvh;

/* Uniform-grid candidate lists over a built BVH's leaves (no reference
 * counterpart; the reference traverses its binary nodes,
 * device_mesh.hpp:262-318).  Each cell lists every leaf whose box overlaps
 * it, in leaf order; the leaves' boxes sit in a table beside.  A leaf is a
 * traversal candidate exactly when its box holds the point, and the
 * left-first traversal meets candidates in leaf order, so a batched locate
 * that scans the point's cell visits the same candidates in the same order
 * as the traversal: results are identical (the statistics' node count then
 * counts entries tested).  Points with a NaN coordinate scan cell 0.
 *
 * drb_bvh_grid_size picks the grid (cells about cell_scale times the mean
 * leaf extent on each axis, at most 2^28 cells), writes grid_dims,
 * grid_origin and grid_inv into *bvh and returns the number of entries in
 * *n_entries; it synchronises the stream.  The caller allocates
 * int32[n_cells + 1], int32[n_entries] and float[8 * n_leaf], sets
 * grid_start, grid_entries and grid_boxes, and calls drb_bvh_grid_build
 * (stream-ordered scratch of about 12 bytes per entry and 32 per leaf).
 * Needs at least two leaves and fewer than 2^31 entries. */
int drb_bvh_grid_size (drb_bvh *bvh, float cell_scale, long long *n_entries, void *stream);
int drb_bvh_grid_build (const drb_bvh *bvh, void *stream);

/* Per-leaf linearisation of a hex or tet mesh's element maps for
 * DRB_GUESS_SUBBOX_LINEAR: for sorted leaf k with element e and reference
 * sub-box centre c (tets: the mean of the sub-simplex's four vertices),
 * maps[16 k ..] = (c, X_e(c), J_e(c)^-1 row-major, 0),
 * X in absolute coordinates.  A leaf whose Jacobian is singular gets a zero
 * inverse (the guess is then c).  No reference counterpart. */
int drb_bvh_leaf_maps (const drb_mesh *mesh, const drb_bvh *bvh, float *maps, void *stream);

/* 4-wide traversal tree of a built BVH (no reference counterpart: the
 * reference traverses the binary nodes, device_mesh.hpp:262-318).  Every
 * binary inner node at even depth becomes a 128-byte node holding its up to
 * four grandchildren (children where those are leaves) in left-to-right
 * order: child boxes as SoA float4 lo x/y/z, hi x/y/z (copied bit for bit),
 * child codes (wide index >= 0, leaf -(leaf+1), empty INT_MIN), count.
 * Locate over it tries the same candidates in the same order as over the
 * binary tree.  With wide_nodes NULL it only fills bvh->n_wide and
 * bvh->wide_depth; otherwise it writes up to capacity nodes and sets
 * bvh->wide_nodes.  Synchronises the stream (reads the node count). */
int drb_bvh_widen (drb_bvh *bvh, float *wide_nodes, int capacity, void *stream);

/* Newton options.  The reference hard-codes tol 1e-4 and 20 steps for
 * volume elements (data_model/element.hpp:474-475), 1e-4 and 10 steps for
 * ray-face solves (face_intersection.hpp:153-154). */
typedef struct drb_newton_opts
{
  float tol;             /* reference-space step tolerance, also is_inside eps */
  int max_steps;
  int guess_mode;        /* enum drb_guess_mode */
  const float *guess;    /* device float[3*n] for DRB_GUESS_GIVEN, else NULL */
} drb_newton_opts;

/* Per-query statistics (utils/appstats.hpp:18-63 counts the same things). */
typedef struct drb_query_stats
{
  int *iters;            /* device int32[n]: Newton iterations summed over candidates, or NULL */
  int *candidates;       /* device int32[n]: leaves whose box held the query, or NULL */
  int *nodes;            /* device int32[n]: inner BVH nodes visited, or NULL */
} drb_query_stats;

const char *drb_last_error (void);
int drb_version (void);
/* Number of kernels this library has launched in the process (all threads). */
unsigned long long drb_kernel_launches (void);

/* Floats per element in a packed element-major copy, padded to a multiple
 * of 4 so each row is 16-byte aligned: geometry (ncomp 3) 3 nd + 3 (the
 * origin), scalar fields nd. */
int drb_packed_stride (int dim, int order, int ncomp);

/* Dofs per element and packed-row stride for any shape (drb_shape);
 * drb_packed_stride is the tensor case.  -1 for unsupported arguments. */
int drb_elem_dofs (int shape, int dim, int order);
int drb_packed_stride_shape (int shape, int dim, int order, int ncomp);

/* Floats per reference sub-box: SubRef<dim,Tensor> 2 dim,
 * SubRef<dim,Simplex> dim (dim + 1) (data_model/subref.hpp:26-35). */
int drb_ref_box_floats (int shape, int dim);

/* Gather the element control points into an element-major array
 * (replaces the double indirection val[ctrl_idx[e*nd+i]] of SharedDofPtr,
 * data_model/dof_access.hpp:23-54).  Geometry rows hold P_i - P_0 (FP32)
 * followed by P_0, the element's first control point: the Newton solves
 * run in that local frame, where FP32 rounding is relative to the element
 * size rather than to the domain.  Scalar rows hold the values. */
int drb_pack_elements (const drb_mesh *mesh, float *packed, void *stream);

/* Sizes of the BVH over a mesh's sub-boxes: 33 per hex or tet, 17 per quad
 * (construct_bvh, data_model/mesh_utils.cpp:527-531). */
int drb_bvh_sizes (int dim, int n_elem, int *n_inner, int *n_leaf);

/* Per-element sub-box split (the forall of detail::construct_bvh,
 * data_model/mesh_utils.cpp:557-670): 32 (hex) / 16 (quad) de Casteljau
 * splits of the largest box, convex-hull AABBs scaled by 1.000001.
 * Outputs per sub-box (element-major, e*(splits+1)+i): aabbs6 device
 * float[6*n], prim_ids device int32[n], ref_boxes device
 * float[drb_ref_box_floats()*n]; bounds6 device float[6] receives the
 * reduction of linear_bvh_builder.cpp:19-58.  Tets split the longest edge of
 * the reference sub-simplex (mesh_utils.cpp:455-480, elem_ops.hpp:1270-1311)
 * with the dof layout of the element evaluators; at order 1 the boxes are
 * bit-identical to the reference's, at orders 2-3 the reference's split
 * indexes the wrong dofs (cartesian_to_tet_idx, elem_ops.hpp:32-47) and its
 * boxes differ. */
int drb_elem_subboxes (const drb_mesh *mesh, float *aabbs6, int *prim_ids, float *ref_boxes,
                       float *bounds6, void *stream);

/* 30-bit Morton codes of AABB centroids (get_mcodes + morton_3d,
 * linear_bvh_builder.cpp:60-90, morton_codes.hpp:39-53). */
int drb_morton_codes (const float *aabbs6, int n, const float *bounds6, unsigned *codes,
                      void *stream);

/* Stable LSD radix sort of (key, value) pairs on the low `bits` key bits
 * (replaces the host std::sort of sort_mcodes, linear_bvh_builder.cpp:120-135). */
int drb_radix_sort_pairs (const unsigned *keys_in, const int *vals_in, unsigned *keys_out,
                          int *vals_out, int n, int bits, void *stream);

/* Full BVH over a mesh: detail::construct_bvh + LinearBVHBuilder::construct
 * (mesh_utils.cpp:514-677, linear_bvh_builder.cpp:399-518).  bvh arrays are
 * caller-allocated with drb_bvh_sizes(); sorted_codes (device uint32[n_leaf])
 * optionally receives the sorted Morton codes.  Synchronises the stream to
 * fill bvh->bounds. */
int drb_lbvh_build (const drb_mesh *mesh, drb_bvh *bvh, unsigned *sorted_codes, void *stream);

/* Point location: Mesh::locate (data_model/unstructured_mesh.cpp:124-148,
 * DeviceMesh::locate device_mesh.hpp:248-354).  One thread per point, BVH
 * traversal left child first, first leaf whose Newton solve converges and is
 * inside wins.  pts device float[3n]; cell device int32[n] (-1 = not found);
 * ref device float[3n] (-1 for misses).  Hex, tet and 2D quad meshes; a quad
 * mesh is located as LocateHack<2> does (device_mesh.hpp:166-238): z is
 * ignored and the third reference coordinate stays -1. */
int drb_locate (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                const drb_newton_opts *opts, int *cell, float *ref, drb_query_stats stats,
                void *stream);

/* Launch shape of the persistent point-location kernel (chosen by
 * drb_locate_tune; no counterpart in the reference, which launches one
 * thread per point in 128-thread blocks, policies.hpp:17-21). */
typedef struct drb_locate_config
{
  int block;             /* threads per block, multiple of 32 */
  int blocks_per_sm;     /* resident blocks per SM, 0 = as many as fit */
  int chunk;             /* queries a warp pops from the global queue at once */
  int sort_queries;      /* 0 = process the queries in input order; 1 =
                            in Morton-cell order, each query read through
                            that order and its result written at its input
                            index (the fastest end to end); 2 = as 1 but
                            the query records staged in that order first
                            (a gather pass; one coalesced read per warp in
                            the kernel); 3 = as 2 with the results also
                            staged contiguously and put back in input order
                            by a separate pass (not with DRB_GUESS_GIVEN,
                            which then runs as 2) */
  int reg_elements;      /* where a candidate's control points are read from
                            during its Newton solve: 0 = through L1 on every
                            step; 1 = registers (orders <= 2; fewer loads,
                            more registers); 2 = shared memory: the warp
                            stages each distinct element row of its lanes'
                            candidates once (packed hex meshes; falls back
                            to 0) */
} drb_locate_config;

/* Batched point location, same results as drb_locate (same traversal order
 * and per-candidate solves per point): queries Morton-sorted, persistent
 * warps popping chunks from a global atomic queue, idle lanes refilled by
 * ballot ranking, Newton solves of a warp run converged.  cfg NULL = default.
 * Replaces UnstructuredMesh::locate (data_model/unstructured_mesh.cpp:124-148). */
int drb_locate_batched (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                        const drb_newton_opts *opts, const drb_locate_config *cfg, int *cell,
                        float *ref, drb_query_stats stats, void *stream);

/* drb_locate_batched without any device allocation, for callers that cannot
 * allocate when they locate points: a host application whose device memory
 * is owned by its own allocator or pool (a simulation code, an in-situ
 * framework) that forbids side allocations, or a latency-critical path where
 * cudaMalloc's implicit synchronisation is not acceptable.  No
 * counterpart in the reference.  All scratch lives in one fixed array of
 * about 20 MB inside the library's device code, which stays allocated on each
 * device where it is loaded until the process exits.  At most
 * drb_noalloc_max_queries() (1,048,576) queries per call; more is rejected
 * with DRB_ERR_INVALID_ARG.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  All calls share the array: calls whose GPU
 * work may overlap race and must be serialised by the caller.  Results equal
 * drb_locate_batched's. */
int drb_locate_batched_noalloc (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts,
                                int n, const drb_newton_opts *opts,
                                const drb_locate_config *cfg, int *cell, float *ref,
                                drb_query_stats stats, void *stream);
/* Largest query count drb_locate_batched_noalloc accepts per call. */
int drb_noalloc_max_queries (void);

/* Morton-cell order of query points over the BVH bounds: device int32
 * order[n], a permutation of 0..n-1 that lists the queries cell by cell
 * along a Morton curve of 2^21 cells (7 bits per axis); inside a cell the
 * order is unspecified.  No reference counterpart (it never reorders). */
int drb_query_order (const drb_bvh *bvh, const float *pts, int n, int *order, void *stream);

/* drb_locate_batched with a caller-supplied processing order (e.g. from
 * drb_query_order, reused across calls on the same queries). */
int drb_locate_ordered (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                        const int *order, const drb_newton_opts *opts,
                        const drb_locate_config *cfg, int *cell, float *ref,
                        drb_query_stats stats, void *stream);

/* Query records in processing order: staged[4 * k .. 4 * k + 3] = (x, y, z,
 * input index as int32 bits) of the k-th query of the Morton-cell order
 * (drb_query_order's order, with the same unspecified order inside a cell).
 * staged: device float[4n], 16-byte aligned.  drb_locate_batched stages its
 * queries this way internally, so the kernel reads and writes consecutive
 * records.  No reference counterpart (it never reorders). */
int drb_query_stage (const drb_bvh *bvh, const float *pts, int n, float *staged, void *stream);

/* The persistent locate kernel of drb_locate_batched on staged records
 * (drb_query_stage).  res non-NULL: res[4 * k .. 4 * k + 3] = (cell as int32
 * bits, r, s, t) of staged query k, in the staged order (not for
 * DRB_GUESS_GIVEN); res NULL: cell[i] and ref[3 * i ..] at each query's input
 * index i, as drb_locate_batched writes them.  Statistics, when requested, go
 * to the input index.  staged and res 16-byte aligned.  Replaces the forall
 * body of UnstructuredMesh::locate (data_model/unstructured_mesh.cpp:137-148)
 * for callers that keep their queries in processing order. */
int drb_locate_staged (const drb_mesh *mesh, const drb_bvh *bvh, const float *staged, int n,
                       const drb_newton_opts *opts, const drb_locate_config *cfg, float *res,
                       int *cell, float *ref, drb_query_stats stats, void *stream);

/* UnstructuredMesh::locate (unstructured_mesh.cpp:124-148) on points that
 * live in host memory: host_pts float[3n] in, host_cell int32[n] and
 * host_ref float[3n] out.  The batch is cut into chunks (chunk <= 0: 2M
 * points) that cycle through three internal streams, so the copies in, the
 * batched locate (drb_locate_batched, Morton order per chunk) and the
 * copies out of consecutive chunks overlap.  Results equal
 * drb_locate_batched's.  Host buffers should be page-locked for the copies
 * to overlap.  Work already queued on stream runs first; the call returns
 * when the results are in host memory. */
int drb_locate_host (const drb_mesh *mesh, const drb_bvh *bvh, const float *host_pts, int n,
                     const drb_newton_opts *opts, const drb_locate_config *cfg, int chunk,
                     int *host_cell, float *host_ref, void *stream);

/* Autotuner of the persistent kernel: times every candidate launch shape on
 * a query sample (CUDA events, synchronous) and returns the fastest in
 * *best and its time in *best_ms (may be NULL).  No reference counterpart. */
int drb_locate_tune (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                     const drb_newton_opts *opts, drb_locate_config *best, float *best_ms,
                     void *stream);

/* ------------------------------------------------------------ rendering */

/* Ray records are dray::Ray (ray.hpp:20-27): dir[3], near, orig[3], far,
 * int32 pixel_id = 36 bytes.  Partials are dray::VolumePartial
 * (rendering/volume_partial.hpp): int32 pixel, depth, rgba = 24 bytes.
 * Point lights are dray::PointLight (rendering/point_light.hpp): pos, amb,
 * diff, spec (3 floats each), spec_pow = 52 bytes. */

/* Camera state of dray::Camera (rendering/camera.hpp:18-118). */
typedef struct drb_camera
{
  int width, height;
  float pos[3];
  float look_at[3];
  float up[3];
  float fov_y;            /* degrees; fov_x follows from the aspect (camera.cpp:132-163) */
  float zoom;             /* 1 = none */
} drb_camera;

/* Per-ray counters of the renderers (device int32[n] each, or NULL). */
typedef struct drb_ray_stats
{
  int *samples;           /* volume: samples that located (Newton-resolved) */
  int *iters;             /* Newton iterations */
  int *candidates;        /* candidate elements tried */
} drb_ray_stats;

/* Volume::integrate options (rendering/volume.hpp:19-59). */
typedef struct drb_volume_opts
{
  int samples;            /* Volume::samples: steps over the bounds diagonal */
  int use_lighting;       /* Blinn-Phong from the field gradient */
  float tol;              /* Newton tolerance (reference: 1e-4) */
  int max_steps;          /* Newton steps (reference: 20) */
  int guess_mode;         /* drb_guess_mode for full locates */
  int coherent;           /* 1: try the previous sample's element first,
                             from r + J^-1 dx (the previous sample's point
                             and factorised Jacobian); 2: as 1, from
                             r_{k-1} + 2 J^-1 dx when the two previous
                             samples lie in the same element */
  float bounds[6];        /* Collection::bounds of the data (sample distance) */
  int cull;               /* 1: rays are raw camera rays; the march applies the
                             slab test of remove_missed_rays itself (no
                             compaction, no host synchronisation) */
} drb_volume_opts;

/* Camera::create_rays / gen_perspective (rendering/camera.cpp:219-483):
 * width*height rays, pixel id j*width+i.  rays: device dray::Ray[w*h]. */
int drb_camera_rays (const drb_camera *cam, void *rays, void *stream);

/* Surface::draw_mesh (rendering/surface.cpp:25-111, 522-550): for every
 * ray whose hit is valid, the mesh-line colour line_color4 with its alpha
 * scaled by the smoothed distance of the hit's reference point to the
 * nearest face edge (line_thickness in reference units, sub_res >= 1 lines
 * per unit) is blended over fb_rgba at the ray's pixel.  rays/hits: device
 * dray::Ray / dray::RayHit [n]. */
int drb_surface_mesh_lines (const void *rays, const void *hits, int n, const float *line_color4,
                            float line_thickness, float sub_res, float *fb_rgba, void *stream);

/* Volume partials ordered by pixel id, then depth (stable): the single-rank
 * order the reference's partial compositor works in before blending each
 * pixel front to back (rendering/renderer.cpp:323-335).  Needed when the
 * partials of several domains are concatenated.  sorted must not alias
 * partials. */
int drb_sort_partials (const void *partials, int n, void *sorted, void *stream);

/* Camera::elevate and Camera::azimuth (rendering/camera.cpp:516-555): turn
 * the view about the camera's right axis (by -degrees) or its up axis and
 * keep the distance to look_at; updates cam->pos (host only). */
int drb_camera_elevate (drb_camera *cam, float degrees);
int drb_camera_azimuth (drb_camera *cam, float degrees);

/* Camera::reset_to_bounds (rendering/camera.cpp:485-514): bounds6 = (xmin,
 * xmax, ymin, ymax, zmin, zmax), padded by the given fractions of each
 * extent; look_at becomes their centre, pos one diagonal away along the
 * current view direction, fov_y 60 (host only). */
int drb_camera_reset_to_bounds (drb_camera *cam, const float *bounds6, double xpad, double ypad,
                                double zpad);

/* detail::default_light (rendering/renderer.cpp:141-159) on the host:
 * light13 = pos[3], amb[3], diff[3], spec[3], spec_pow (PointLight defaults). */
int drb_default_light (const drb_camera *cam, float *light13);

/* remove_missed_rays (ray.cpp:102-115): keep rays hitting bounds6 scaled by
 * 1.001, in order, with near/far set by calc_ray_start (ray.cpp:183-241).
 * Synchronises the stream to return *n_active. */
int drb_cull_rays (const void *rays, int n, const float *bounds6, void *active_rays,
                   int *n_active, void *stream);

/* Range of a scalar field's control values (get_range,
 * data_model/unstructured_field.cpp:35-80): range2 device float[2]. */
int drb_field_range (const drb_mesh *field, float *range2, void *stream);

/* ColorTable::sample after correct_opacity(opacity_factor)
 * (color_table.cpp:152-323); host arrays, no GPU.  rgb_pts n x (pos,r,g,b),
 * alpha_pts n x (pos,a); opacity_factor <= 0 skips the correction. */
int drb_color_table_sample (int n_rgb, const float *rgb_pts, int n_alpha, const float *alpha_pts,
                            int smooth, int n_samples, float alpha_scale, float opacity_factor,
                            float *rgba);

/* Volume::integrate (rendering/volume.cpp:71-228, 324-348) over culled
 * rays: partials compacted in ray then depth order (device
 * dray::VolumePartial[5*n_rays] capacity); *n_partials returned after a
 * stream synchronise.  tf: device float4[tf_size] (opacity corrected);
 * range2: host float[2] scalar range; lights: device PointLight[n_lights].
 * Hex or tet (dispatch_3d, dispatcher.hpp:209-219) mesh and field of one
 * shape and order; tet samples are located through the BVH whenever the
 * previous sample's element does not hold them (no face table). */
int drb_volume_integrate (const drb_mesh *mesh, const drb_mesh *field, const drb_bvh *bvh,
                          const void *active_rays, int n_rays, const drb_volume_opts *opts,
                          const float *tf, int tf_size, const float *range2, const void *lights,
                          int n_lights, void *partials, int *n_partials, drb_ray_stats stats,
                          void *stream);

/* Volume::integrate fused with the compositing of Volume::save
 * (volume.cpp:369-416): writes the composited colour of every pixel with a
 * partial into fb_rgba (device float4[w*h], cleared by the caller) and the
 * first partial's depth into fb_depth (may be NULL).  No partial buffer. */
int drb_volume_render (const drb_mesh *mesh, const drb_mesh *field, const drb_bvh *bvh,
                       const void *active_rays, int n_rays, const drb_volume_opts *opts,
                       const float *tf, int tf_size, const float *range2, const void *lights,
                       int n_lights, float *fb_rgba, float *fb_depth, drb_ray_stats stats,
                       void *stream);

/* Volume::save compositing of partials sorted by pixel then depth. */
int drb_composite_partials (const void *partials, int n, float *fb_rgba, void *stream);

/* Renderer's partials_to_framebuffer (rendering/renderer.cpp:98-139) after
 * compositing each pixel's partials (sorted by pixel then depth); blend_over
 * puts the volume in front of the framebuffer's current (surface) colour. */
int drb_partials_to_framebuffer (const void *partials, int n, float *fb_rgba, float *fb_depth,
                                 int blend_over, void *stream);

/* Framebuffer::clear / composite_background (rendering/framebuffer.cpp:126-162).
 * color4/bg4 are host float[4]; NULL = (0,0,0,0) / white. */
int drb_framebuffer_clear (float *rgba, float *depth, int n_pixels, const float *color4,
                           void *stream);
int drb_framebuffer_composite_background (float *rgba, int n_pixels, const float *bg4,
                                          void *stream);

/* MeshBoundary::execute (filters/mesh_boundary.cpp:339-361, 205-236) for a
 * hex mesh: the boundary quads in the reference's order (sorted face corner
 * tuples), each as (p+1)^2 indices into the unchanged value arrays.
 * field_ctrl_idx (optional) is the scalar field's ctrl_idx, mapped to
 * face_field_idx the same way; elid_faceid (optional) receives (element,
 * face id 0..5) pairs.  Outputs need capacity 6*n_elem faces; *n_faces is
 * returned after a stream synchronise (call once with NULL outputs to size).
 * For a tet mesh the faces are triangles, (p+1)(p+2)/2 indices each (the
 * triangle dof order of cartesian_to_tri_idx), face ids 0..3, capacity
 * 4*n_elem; the face mesh is then a dim-2 simplex mesh. */
int drb_mesh_boundary (const drb_mesh *hex, const int *field_ctrl_idx, int *face_ctrl_idx,
                       int *face_field_idx, int *elid_faceid, int *n_faces, void *stream);

/* Surface::nearest_hit (rendering/surface.cpp:304-437, 497-520) over a quad
 * mesh and its BVH: ordered traversal, ray-face Newton per candidate
 * (face_intersection.hpp:96-173; reference tol 1e-4, 10 steps).  hits:
 * device dray::RayHit[n] (int32 idx, dist, ref[3] = 20 bytes). */
int drb_surface_intersect (const drb_mesh *faces, const drb_bvh *bvh, const void *rays, int n,
                           float tol, int max_steps, void *hits, drb_ray_stats stats,
                           void *stream);

/* Traceable::fragments + Traceable::shade (rendering/traceable.cpp:49-147,
 * 242-387) for quad faces, fused: fragments (optional device float[4n]:
 * scalar, normal) and, for hits, the shaded colour and depth into the
 * framebuffer (device float4/float [w*h], indexed by the ray's pixel id).
 * With fb_rgba NULL only the fragments are computed and rays may be NULL. */
int drb_surface_shade (const drb_mesh *faces, const drb_mesh *face_field, const void *rays,
                       const void *hits, int n, const float *tf, int tf_size,
                       const float *range2, const void *lights, int n_lights, int use_lighting,
                       float *fragments, float *fb_rgba, float *fb_depth, void *stream);

/* The writes of ScalarRenderer::render (rendering/scalar_renderer.cpp:
 * 296-365) for the rays that hit: depths[pid] = dist and zone_ids[pid] =
 * hit_idx + zone_offset (each optional), and scalars[pid] = the fragment's
 * scalar (frags4: {scalar, normal} per ray from drb_surface_shade) when
 * scalars is given.  pid is the ray's pixel id. */
int drb_scalar_buffer_write (const void *rays, const void *hits, const float *frags4, int n,
                             int zone_offset, float *depths, int *zone_ids, float *scalars,
                             void *stream);

/* ray_max (ray.cpp:243-259): far = hit distance for rays that hit. */
int drb_ray_max (void *rays, const void *hits, int n, void *stream);

/* -------------------------------------------- learned initial guess --
 * No counterpart in the reference.  A small MLP (the (P+1)^3 control points
 * x 3 + point x 3 inputs -> 128 -> 128 -> 3, GELU) predicts the reference
 * coordinates of a point in an order-P hex candidate element: 84 inputs at
 * order 2, 195 at order 3.  `order` selects the network; the mesh's order
 * does where a mesh is passed.  Parameters: one fp32 vector of
 * drb_mlp_param_count(order) floats (W1 [128 x inputs], b1, W2 [128 x
 * 128], b2, W3 [3 x 128], b3); bf16 tensor-core operands:
 * drb_mlp_bf16_count(order) values written by drb_mlp_prepare.  Feature
 * rows are drb_mlp_input_width(order) wide (inputs padded to 16: 96 at
 * order 2, 208 at order 3).  Tensor-core kernels report a bounded-wait
 * timeout through *err (device int32).  Counts are -1 for an order outside
 * 1..3. */
int drb_mlp_param_count (int order);
int drb_mlp_bf16_count (int order);
int drb_mlp_input_width (int order);
long long drb_mlp_workspace_bytes (int order, int n_pad);
int drb_mlp_prepare (int order, const float *params, void *wbf16, void *stream);
/* features of (element, point) pairs: X device bf16 [n_pad x input width] */
int drb_mlp_features (const drb_mesh *mesh, const int *elem, const float *pts, int n, int n_pad,
                      void *X, void *stream);
/* forward: y device float[3n]; n_pad multiple of 128 */
int drb_mlp_forward (int order, const float *params, const void *wbf16, const void *X, int n,
                     int n_pad, float *y, void *workspace, int *err, void *stream);
/* one training step: masked MSE against target (device float[3n], weight
 * optional device float[n]); grad (device float[param_count]) and *loss */
int drb_mlp_train_step (int order, const float *params, const void *wbf16, const void *X,
                        const float *target, const float *weight, int n, int n_pad, float *grad,
                        float *loss, void *workspace, int *err, void *stream);
int drb_mlp_adam (int order, float *params, const float *grad, float *m, float *v, float lr,
                  float beta1, float beta2, float eps, int step, void *stream);
/* fused tensor-core inference: guess device float[3n] for the pairs
 * (elem[q], pts[q]); rows are visited in the order order[0..n) when given
 * (the Morton order of drb_query_order keeps a tile's elements together in
 * L1), else 0..n-1.  Results do not depend on the order. */
int drb_mlp_guess (const float *params, const void *wbf16, const drb_mesh *mesh,
                   const int *elem, const float *pts, const int *order, int n, float *guess,
                   int *err, void *stream);

/* UnstructuredField::eval at located points (data_model/unstructured_field.cpp:
 * 214-245): values[i] = f(cell[i], ref[i]), empty_value where cell is -1. */
int drb_field_eval (const drb_mesh *field, const int *cell, const float *ref, int n,
                    float empty_value, float *values, void *stream);

/* Lineout::create_points (queries/lineout.cpp:98-140): samples + 2 evenly
 * spaced points per line from start to end inclusive, bit-identical to the
 * reference's (same operations in the same order).  starts, ends: device
 * float[3 n_lines]; points: device float[3 n_lines (samples + 2)]. */
int drb_lineout_points (const float *starts, const float *ends, int n_lines, int samples,
                        float *points, void *stream);

/* Physical points X_e(r) (Element::eval, pos_tensor_element.tcc:99-232;
 * tets elem_ops.hpp:901-1030). */
int drb_map_points (const drb_mesh *mesh, const int *elem, const float *ref, int n, float *pts,
                    void *stream);
/* Newton in a given element per point (eval_inverse_local,
 * data_model/element.hpp:435-486): guess NULL = element centre. */
int drb_newton_pairs (const drb_mesh *mesh, const int *elem, const float *pts, int n, float tol,
                      int max_steps, const float *guess, float *ref, int *found, int *iters,
                      void *stream);
/* First candidate leaf (and element) of each query in the traversal order of
 * DeviceMesh::locate (device_mesh.hpp:248-318); -1 when there is none.  With
 * grid lists (drb_bvh_grid_build) the leaf comes from the query's cell: the
 * same leaf. */
int drb_first_candidates (const drb_bvh *bvh, const float *pts, int n, const int *order,
                          int *first_leaf, int *first_elem, void *stream);
/* Persistent locate that starts at each query's first candidate (guess from
 * opts, element-centre fallback) and resumes the traversal only when that
 * fails; results equal drb_locate with the same options. */
int drb_locate_hinted (const drb_mesh *mesh, const drb_bvh *bvh, const float *pts, int n,
                       const int *order, const int *first_leaf, const drb_newton_opts *opts,
                       const drb_locate_config *cfg, int *cell, float *ref,
                       drb_query_stats stats, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DRB_H */
