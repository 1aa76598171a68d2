// Test oracle: a thin extern "C" driver over the reference's own C++ classes
// (Devil Ray, compiled from its sources against the host-only shims in
// oracle/shims).  It is test infrastructure: tests, smoke() and the bench's
// CPU-baseline leg call it to obtain the reference's results; the product
// never links it.
//
// Every entry point drives the reference through its public API:
//   UnstructuredMesh<E>(GridFunction<3>, order)        data_model/unstructured_mesh.cpp:34
//   UnstructuredMesh::get_bvh / get_ref_aabbs           data_model/unstructured_mesh.cpp:23, .hpp:109
//   UnstructuredMesh::locate                            data_model/unstructured_mesh.cpp:124
//   get_mcodes / reduce (LBVH internals, non-static)    linear_bvh_builder.cpp:19,60
//   Camera::create_rays                                 rendering/camera.cpp:219
//   Volume::integrate + the host compositing loop of
//   Volume::save                                        rendering/volume.cpp:324,369
//   MeshBoundary::execute                               filters/mesh_boundary.cpp:339
//   Surface::nearest_hit / fragments / shade            rendering/surface.cpp:497, traceable.cpp
//   Framebuffer::clear / composite_background           rendering/framebuffer.cpp:126,146
#include <dray/queries/lineout.hpp>
#include <dray/aabb.hpp>
#include <dray/array.hpp>
#include <dray/bvh.hpp>
#include <dray/color_map.hpp>
#include <dray/color_table.hpp>
#include <dray/data_model/collection.hpp>
#include <dray/data_model/element.hpp>
#include <dray/data_model/dof_access.hpp>
#include <dray/data_model/data_set.hpp>
#include <dray/data_model/grid_function.hpp>
#include <dray/data_model/unstructured_field.hpp>
#include <dray/data_model/unstructured_mesh.hpp>
#include <dray/filters/mesh_boundary.hpp>
#include <dray/location.hpp>
#include <dray/ray.hpp>
#include <dray/ray_hit.hpp>
#include <dray/rendering/camera.hpp>
#include <dray/rendering/colors.hpp>
#include <dray/rendering/fragment.hpp>
#include <dray/rendering/framebuffer.hpp>
#include <dray/rendering/point_light.hpp>
#include <dray/rendering/renderer.hpp>
#include <dray/rendering/surface.hpp>
#include <dray/rendering/volume.hpp>
#include <dray/rendering/volume_partial.hpp>

#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace dray
{
// Free functions of linear_bvh_builder.cpp (external linkage there).
AABB<> reduce (const Array<AABB<>> &aabbs);
Array<uint32> get_mcodes (Array<AABB<>> &aabbs, const AABB<> &bounds);
} // namespace dray

using namespace dray;

namespace
{
struct RefMesh
{
  int order = 0;
  std::shared_ptr<Mesh> mesh;
  Collection collection;
  bool has_field = false;
};

GridFunction<3> make_gf3 (int n_el, int nd, const int *idx, int n_ctrl, const float *xyz)
{
  GridFunction<3> gf;
  gf.resize (n_el, nd, n_ctrl);
  std::memcpy (gf.m_ctrl_idx.get_host_ptr (), idx, sizeof (int) * (size_t)n_el * nd);
  std::memcpy ((void *)gf.m_values.get_host_ptr (), xyz, sizeof (float) * 3 * (size_t)n_ctrl);
  return gf;
}

GridFunction<1> make_gf1 (int n_el, int nd, const int *idx, int n_ctrl, const float *vals)
{
  GridFunction<1> gf;
  gf.resize (n_el, nd, n_ctrl);
  std::memcpy (gf.m_ctrl_idx.get_host_ptr (), idx, sizeof (int) * (size_t)n_el * nd);
  std::memcpy ((void *)gf.m_values.get_host_ptr (), vals, sizeof (float) * (size_t)n_ctrl);
  return gf;
}

std::shared_ptr<Mesh> make_hex_mesh (int order, const GridFunction<3> &gf)
{
  if (order == 1) return std::make_shared<HexMesh_P1> (gf, 1);
  if (order == 2) return std::make_shared<HexMesh_P2> (gf, 2);
  return std::make_shared<HexMesh> (gf, order);
}

std::shared_ptr<Field> make_hex_field (int order, const GridFunction<1> &gf, const char *name)
{
  if (order == 1)
    return std::make_shared<UnstructuredField<HexScalar_P1>> (gf, 1, name);
  if (order == 2)
    return std::make_shared<UnstructuredField<HexScalar_P2>> (gf, 2, name);
  return std::make_shared<UnstructuredField<HexScalar>> (gf, order, name);
}

// Tet meshes: the fixed-order specialisations (TetMesh_P1/_P2) when
// `fixed`, else the general-order TetMesh (UnstructuredMesh<Tet3>).
std::shared_ptr<Mesh> make_tet_mesh (int order, int fixed, const GridFunction<3> &gf)
{
  if (fixed && order == 1) return std::make_shared<TetMesh_P1> (gf, 1);
  if (fixed && order == 2) return std::make_shared<TetMesh_P2> (gf, 2);
  return std::make_shared<TetMesh> (gf, order);
}

std::shared_ptr<Field> make_tet_field (int order, int fixed, const GridFunction<1> &gf,
                                       const char *name)
{
  if (fixed && order == 1)
    return std::make_shared<UnstructuredField<TetScalar_P1>> (gf, 1, name);
  if (fixed && order == 2)
    return std::make_shared<UnstructuredField<TetScalar_P2>> (gf, 2, name);
  return std::make_shared<UnstructuredField<TetScalar>> (gf, order, name);
}

template <typename MeshT> BVH bvh_of (Mesh *m)
{
  return dynamic_cast<MeshT *> (m)->get_bvh ();
}

BVH get_bvh_any (Mesh *m)
{
  if (auto *p = dynamic_cast<HexMesh_P1 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<HexMesh_P2 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<HexMesh *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<QuadMesh_P1 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<QuadMesh_P2 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<QuadMesh *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TetMesh_P1 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TetMesh_P2 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TetMesh *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TriMesh_P1 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TriMesh_P2 *> (m)) return p->get_bvh ();
  if (auto *p = dynamic_cast<TriMesh *> (m)) return p->get_bvh ();
  throw std::runtime_error ("unsupported mesh type");
}

// Reference boxes are SubRef<dim,Tensor>: two corners of dim floats.
int copy_ref_boxes (Mesh *m, float *out)
{
  if (auto *p = dynamic_cast<HexMesh_P1 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  if (auto *p = dynamic_cast<HexMesh_P2 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  if (auto *p = dynamic_cast<HexMesh *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  if (auto *p = dynamic_cast<QuadMesh_P1 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 16); return 2; }
  if (auto *p = dynamic_cast<QuadMesh_P2 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 16); return 2; }
  if (auto *p = dynamic_cast<QuadMesh *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 16); return 2; }
  // SubRef<3,Simplex>: four vertices (u, v, w axis vertices, then the origin)
  if (auto *p = dynamic_cast<TetMesh_P1 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 48); return 4; }
  if (auto *p = dynamic_cast<TetMesh_P2 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 48); return 4; }
  if (auto *p = dynamic_cast<TetMesh *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 48); return 4; }
  // SubRef<2,Simplex>: three vertices of two floats
  if (auto *p = dynamic_cast<TriMesh_P1 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  if (auto *p = dynamic_cast<TriMesh_P2 *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  if (auto *p = dynamic_cast<TriMesh *> (m))
  { auto a = p->get_ref_aabbs (); std::memcpy (out, (const void *)a.get_host_ptr_const (), a.size () * 24); return 3; }
  return 0;
}

thread_local std::string g_err;

ColorTable make_table (int n_rgb, const float *rgb_pts, int n_alpha, const float *alpha_pts)
{
  // rgb_pts: n_rgb x (pos, r, g, b); alpha_pts: n_alpha x (pos, a)
  ColorTable t;
  t.set_smooth (true);
  for (int i = 0; i < n_rgb; ++i)
    t.add_point (rgb_pts[4 * i], make_vec3f (rgb_pts[4 * i + 1], rgb_pts[4 * i + 2], rgb_pts[4 * i + 3]));
  for (int i = 0; i < n_alpha; ++i) t.add_alpha (alpha_pts[2 * i], alpha_pts[2 * i + 1]);
  return t;
}

void setup_camera (Camera &cam, int w, int h, const float *cam9, float fov)
{
  cam.set_width (w);
  cam.set_height (h);
  cam.set_pos (make_vec3f (cam9[0], cam9[1], cam9[2]));
  cam.set_look_at (make_vec3f (cam9[3], cam9[4], cam9[5]));
  cam.set_up (make_vec3f (cam9[6], cam9[7], cam9[8]));
  cam.set_fov (fov);
}

Array<PointLight> make_lights (int n, const float *l13)
{
  // l13: n x (pos3, amb3, diff3, spec3, spec_pow)
  Array<PointLight> lights;
  lights.resize (n);
  PointLight *lp = lights.get_host_ptr ();
  for (int i = 0; i < n; ++i)
  {
    const float *s = l13 + 13 * i;
    lp[i].m_pos = make_vec3f (s[0], s[1], s[2]);
    lp[i].m_amb = make_vec3f (s[3], s[4], s[5]);
    lp[i].m_diff = make_vec3f (s[6], s[7], s[8]);
    lp[i].m_spec = make_vec3f (s[9], s[10], s[11]);
    lp[i].m_spec_pow = s[12];
  }
  return lights;
}
} // namespace

extern "C" {

const char *ref_last_error () { return g_err.c_str (); }

int ref_num_threads ()
{
#ifdef _OPENMP
  return omp_get_max_threads ();
#else
  return 1;
#endif
}

void ref_set_num_threads (int n)
{
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads (n);
#else
  (void)n;
#endif
}

// Create a hex mesh of polynomial order `order` (element type chosen as the
// reference's dispatcher does: fixed-order P1/P2 specialisations, General
// otherwise) plus an optional scalar field named "f" on the same layout.
void *ref_hex_create (int order, int n_el, const int *ctrl_idx, int n_ctrl, const float *xyz,
                      const int *field_idx, int n_field_ctrl, const float *field_vals)
{
  try
  {
    const int nd = (order + 1) * (order + 1) * (order + 1);
    RefMesh *r = new RefMesh ();
    r->order = order;
    r->mesh = make_hex_mesh (order, make_gf3 (n_el, nd, ctrl_idx, n_ctrl, xyz));
    DataSet ds (r->mesh);
    if (field_vals != nullptr)
    {
      ds.add_field (make_hex_field (order, make_gf1 (n_el, nd, field_idx, n_field_ctrl, field_vals), "f"));
      r->has_field = true;
    }
    r->collection.add_domain (ds);
    return r;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return nullptr;
  }
}

// Create a tet mesh (and optional scalar field "f") of polynomial order
// `order`; `fixed` picks the fixed-order P1/P2 element types, otherwise the
// general-order ones.
void *ref_tet_create (int order, int fixed, int n_el, const int *ctrl_idx, int n_ctrl,
                      const float *xyz, const int *field_idx, int n_field_ctrl,
                      const float *field_vals)
{
  try
  {
    const int nd = (order + 1) * (order + 2) * (order + 3) / 6;
    RefMesh *r = new RefMesh ();
    r->order = order;
    r->mesh = make_tet_mesh (order, fixed, make_gf3 (n_el, nd, ctrl_idx, n_ctrl, xyz));
    DataSet ds (r->mesh);
    if (field_vals != nullptr)
    {
      ds.add_field (make_tet_field (order, fixed, make_gf1 (n_el, nd, field_idx, n_field_ctrl, field_vals), "f"));
      r->has_field = true;
    }
    r->collection.add_domain (ds);
    return r;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return nullptr;
  }
}

// Create a quad (2D) mesh and optional scalar field "f": QuadMesh_P1/P2
// for orders 1-2, QuadMesh (general order) otherwise, as the dispatcher
// picks them.
void *ref_quad_create (int order, int n_el, const int *ctrl_idx, int n_ctrl, const float *xyz,
                       const int *field_idx, int n_field_ctrl, const float *field_vals)
{
  try
  {
    const int nd = (order + 1) * (order + 1);
    RefMesh *r = new RefMesh ();
    r->order = order;
    GridFunction<3> gf = make_gf3 (n_el, nd, ctrl_idx, n_ctrl, xyz);
    if (order == 1) r->mesh = std::make_shared<QuadMesh_P1> (gf, 1);
    else if (order == 2) r->mesh = std::make_shared<QuadMesh_P2> (gf, 2);
    else r->mesh = std::make_shared<QuadMesh> (gf, order);
    DataSet ds (r->mesh);
    if (field_vals != nullptr)
    {
      GridFunction<1> ff = make_gf1 (n_el, nd, field_idx, n_field_ctrl, field_vals);
      std::shared_ptr<Field> f;
      if (order == 1) f = std::make_shared<UnstructuredField<QuadScalar_P1>> (ff, 1, "f");
      else if (order == 2) f = std::make_shared<UnstructuredField<QuadScalar_P2>> (ff, 2, "f");
      else f = std::make_shared<UnstructuredField<QuadScalar>> (ff, order, "f");
      ds.add_field (f);
      r->has_field = true;
    }
    r->collection.add_domain (ds);
    return r;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return nullptr;
  }
}

// Create a triangle (2D) mesh and optional scalar field "f": TriMesh_P1/P2
// for orders 1-2, TriMesh (general order) otherwise.
void *ref_tri_create (int order, int n_el, const int *ctrl_idx, int n_ctrl, const float *xyz,
                      const int *field_idx, int n_field_ctrl, const float *field_vals)
{
  try
  {
    const int nd = (order + 1) * (order + 2) / 2;
    RefMesh *r = new RefMesh ();
    r->order = order;
    GridFunction<3> gf = make_gf3 (n_el, nd, ctrl_idx, n_ctrl, xyz);
    if (order == 1) r->mesh = std::make_shared<TriMesh_P1> (gf, 1);
    else if (order == 2) r->mesh = std::make_shared<TriMesh_P2> (gf, 2);
    else r->mesh = std::make_shared<TriMesh> (gf, order);
    DataSet ds (r->mesh);
    if (field_vals != nullptr)
    {
      GridFunction<1> ff = make_gf1 (n_el, nd, field_idx, n_field_ctrl, field_vals);
      std::shared_ptr<Field> f;
      if (order == 1) f = std::make_shared<UnstructuredField<TriScalar_P1>> (ff, 1, "f");
      else if (order == 2) f = std::make_shared<UnstructuredField<TriScalar_P2>> (ff, 2, "f");
      else f = std::make_shared<UnstructuredField<TriScalar>> (ff, order, "f");
      ds.add_field (f);
      r->has_field = true;
    }
    r->collection.add_domain (ds);
    return r;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return nullptr;
  }
}

void ref_free (void *h) { delete static_cast<RefMesh *> (h); }

// Builds (if needed) the mesh BVH and reports its sizes.
int ref_bvh_sizes (void *h, int *n_inner, int *n_leaf)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    BVH b = get_bvh_any (r->mesh.get ());
    *n_inner = (int)b.m_inner_nodes.size () / 4;
    *n_leaf = (int)b.m_leaf_nodes.size ();
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Copies the BVH: inner nodes (16 floats each), leaf prim ids, aabb ids
// (sort permutation), bounds (xmin,xmax,ymin,ymax,zmin,zmax) and the
// per-sub-box reference boxes (2*dim floats each, original sub-box order).
int ref_bvh_copy (void *h, float *inner, int *leaf_nodes, int *aabb_ids, float *bounds6,
                  float *ref_boxes)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    BVH b = get_bvh_any (r->mesh.get ());
    std::memcpy (inner, (const void *)b.m_inner_nodes.get_host_ptr_const (),
                 sizeof (float) * 4 * b.m_inner_nodes.size ());
    std::memcpy (leaf_nodes, b.m_leaf_nodes.get_host_ptr_const (), sizeof (int) * b.m_leaf_nodes.size ());
    std::memcpy (aabb_ids, b.m_aabb_ids.get_host_ptr_const (), sizeof (int) * b.m_aabb_ids.size ());
    for (int d = 0; d < 3; ++d)
    {
      bounds6[2 * d] = b.m_bounds.m_ranges[d].min ();
      bounds6[2 * d + 1] = b.m_bounds.m_ranges[d].max ();
    }
    if (ref_boxes) copy_ref_boxes (r->mesh.get (), ref_boxes);
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Reference Morton codes and scene bounds for a list of AABBs given as
// (xmin,xmax,ymin,ymax,zmin,zmax) records.
void ref_morton (int n, const float *aabbs6, unsigned *codes, float *bounds6)
{
  Array<AABB<>> boxes;
  boxes.resize (n);
  std::memcpy ((void *)boxes.get_host_ptr (), aabbs6, sizeof (float) * 6 * (size_t)n);
  AABB<> bounds = reduce (boxes);
  Array<uint32> m = get_mcodes (boxes, bounds);
  std::memcpy (codes, m.get_host_ptr_const (), sizeof (unsigned) * (size_t)n);
  for (int d = 0; d < 3; ++d)
  {
    bounds6[2 * d] = bounds.m_ranges[d].min ();
    bounds6[2 * d + 1] = bounds.m_ranges[d].max ();
  }
}

// Mesh::locate: cell id (-1 = not found) and reference coordinates.
int ref_locate (void *h, int n, const float *pts, int *cell, float *ref3)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    Array<Vec<Float, 3>> p;
    p.resize (n);
    std::memcpy ((void *)p.get_host_ptr (), pts, sizeof (float) * 3 * (size_t)n);
    Array<Location> loc = r->mesh->locate (p);
    const Location *lp = loc.get_host_ptr_const ();
    for (int i = 0; i < n; ++i)
    {
      cell[i] = lp[i].m_cell_id;
      ref3[3 * i] = lp[i].m_ref_pt[0];
      ref3[3 * i + 1] = lp[i].m_ref_pt[1];
      ref3[3 * i + 2] = lp[i].m_ref_pt[2];
    }
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Camera::create_rays: rays as (dir3, near, orig3, far, pixel_id) = 9 words.
// Camera moves through the reference's Camera: optional reset_to_bounds
// (bounds6 = xmin,xmax,ymin,ymax,zmin,zmax; pads3 as doubles), then elevate
// and azimuth; out9 = position, look_at, up, *out_fov = field of view.
int ref_camera_move (int w, int h, const float *cam9, float fov, const float *bounds6,
                     const double *pads3, float elevate_deg, float azimuth_deg, float *out9,
                     float *out_fov)
{
  try
  {
    Camera cam;
    setup_camera (cam, w, h, cam9, fov);
    if (bounds6)
    {
      AABB<> b;
      for (int d = 0; d < 3; ++d)
      {
        b.m_ranges[d].include (bounds6[2 * d]);
        b.m_ranges[d].include (bounds6[2 * d + 1]);
      }
      cam.reset_to_bounds (b, pads3[0], pads3[1], pads3[2]);
    }
    if (elevate_deg != 0.f) cam.elevate (elevate_deg);
    if (azimuth_deg != 0.f) cam.azimuth (azimuth_deg);
    const Vec<float32, 3> p = cam.get_pos (), l = cam.get_look_at (), u = cam.get_up ();
    for (int i = 0; i < 3; ++i)
    {
      out9[i] = p[i];
      out9[3 + i] = l[i];
      out9[6 + i] = u[i];
    }
    *out_fov = cam.get_fov ();
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

int ref_camera_rays (int w, int h, const float *cam9, float fov, float *rays9)
{
  try
  {
    Camera cam;
    setup_camera (cam, w, h, cam9, fov);
    Array<Ray> rays;
    cam.create_rays (rays);
    std::memcpy (rays9, (const void *)rays.get_host_ptr_const (), sizeof (Ray) * (size_t)rays.size ());
    return rays.size ();
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Volume::integrate over camera rays, then the host compositing of
// Volume::save and Framebuffer::composite_background (white background).
// Outputs the partial count and, when rgba/partials are non-null, the
// composited image (w*h*4 floats) and the raw partials (6 words each:
// pixel, depth, r, g, b, a).
int ref_volume (void *h, int w, int hgt, const float *cam9, float fov, int samples,
                int use_lighting, int tf_samples, int n_rgb, const float *rgb_pts, int n_alpha,
                const float *alpha_pts, int n_lights, const float *lights13, float *rgba,
                float *partials6, int max_partials)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    Camera cam;
    setup_camera (cam, w, hgt, cam9, fov);
    Array<Ray> rays;
    cam.create_rays (rays);
    Volume vol (r->collection);
    vol.field ("f");
    vol.samples (samples);
    vol.use_lighting (use_lighting != 0);
    ColorMap &cmap = vol.color_map ();
    cmap.samples (tf_samples);
    cmap.color_table (make_table (n_rgb, rgb_pts, n_alpha, alpha_pts));
    Array<PointLight> lights = make_lights (n_lights, lights13);
    Array<VolumePartial> partials = vol.integrate (rays, lights);

    const int size = partials.size ();
    const VolumePartial *pp = partials.get_host_ptr_const ();
    if (partials6)
    {
      for (int i = 0; i < size && i < max_partials; ++i)
      {
        partials6[6 * i] = (float)pp[i].m_pixel_id;
        partials6[6 * i + 1] = pp[i].m_depth;
        for (int c = 0; c < 4; ++c) partials6[6 * i + 2 + c] = pp[i].m_color[c];
      }
    }
    if (rgba)
    {
      Framebuffer fb (w, hgt);
      fb.clear ();
      Vec<float32, 4> *color_ptr = fb.colors ().get_host_ptr ();
      if (size > 0)
      {
        Vec<float32, 4> color = pp[0].m_color;
        int32 current_pixel = -1;
        for (int i = 0; i < size; ++i)
        {
          VolumePartial p = pp[i];
          if (current_pixel != p.m_pixel_id)
          {
            if (current_pixel != -1) color_ptr[current_pixel] = color;
            color = p.m_color;
            current_pixel = p.m_pixel_id;
          }
          else
          {
            pre_mult_alpha_blend_host (color, p.m_color);
          }
          if (i == size - 1) color_ptr[current_pixel] = color;
        }
      }
      fb.composite_background ();
      std::memcpy (rgba, (const void *)fb.colors ().get_host_ptr_const (), sizeof (float) * 4 * (size_t)w * hgt);
    }
    return size;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

} // extern "C" (reopened below)

// Installs a BVH built elsewhere (the same record layout: inner nodes of
// 16 floats, leaf element ids, leaf sub-box ids, bounds, and one SubRef
// reference box of 6 floats per sub-box) into a hex mesh, in place of the
// lazy UnstructuredMesh::get_bvh build.  The reference's own build cannot
// run at the 128^3 order-3 size: its split scratch holds
// num_els * 33 * (p+1)^3 control points, 53 GB there, indexed by int32
// (data_model/mesh_utils.cpp:552-569).  The fields are protected; member
// pointers taken through a derived type reach them.
template <typename MeshT> struct BvhAccess : MeshT
{
  static void install (Mesh *m, const BVH &b, const float *ref6, int n_leaf)
  {
    MeshT *mesh = dynamic_cast<MeshT *> (m);
    if (!mesh) throw std::runtime_error ("set_bvh: not this mesh type");
    mesh->*(&BvhAccess::m_bvh) = b;
    Array<SubRef<3, ElemType::Tensor>> &ra = mesh->*(&BvhAccess::m_ref_aabbs);
    ra.resize (n_leaf);
    std::memcpy ((void *)ra.get_host_ptr (), ref6, sizeof (float) * 6 * (size_t)n_leaf);
    mesh->*(&BvhAccess::m_is_constructed) = true;
  }
};

extern "C" {

int ref_hex_set_bvh (void *h, int n_inner, const float *inner, int n_leaf, const int *leaf_nodes,
                     const int *aabb_ids, const float *bounds6, const float *ref6)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    BVH b;
    b.m_inner_nodes.resize ((size_t)4 * n_inner);
    std::memcpy ((void *)b.m_inner_nodes.get_host_ptr (), inner, sizeof (float) * 16 * (size_t)n_inner);
    b.m_leaf_nodes.resize (n_leaf);
    std::memcpy (b.m_leaf_nodes.get_host_ptr (), leaf_nodes, sizeof (int) * (size_t)n_leaf);
    b.m_aabb_ids.resize (n_leaf);
    std::memcpy (b.m_aabb_ids.get_host_ptr (), aabb_ids, sizeof (int) * (size_t)n_leaf);
    for (int d = 0; d < 3; ++d)
    {
      b.m_bounds.m_ranges[d].reset ();
      b.m_bounds.m_ranges[d].include (bounds6[2 * d]);
      b.m_bounds.m_ranges[d].include (bounds6[2 * d + 1]);
    }
    Mesh *m = r->mesh.get ();
    if (dynamic_cast<HexMesh_P1 *> (m)) BvhAccess<HexMesh_P1>::install (m, b, ref6, n_leaf);
    else if (dynamic_cast<HexMesh_P2 *> (m)) BvhAccess<HexMesh_P2>::install (m, b, ref6, n_leaf);
    else BvhAccess<HexMesh>::install (m, b, ref6, n_leaf);
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Volume::integrate on given rays (the reference's 36-byte Ray records:
// dir, near, orig, far, pixel id), e.g. a tile of a camera's rays; the
// partials as (pixel, depth, r, g, b, a) records.  Returns their count.
int ref_volume_rays (void *h, int n_rays, const float *rays9, int samples, int use_lighting,
                     int tf_samples, int n_rgb, const float *rgb_pts, int n_alpha,
                     const float *alpha_pts, int n_lights, const float *lights13,
                     float *partials6, int max_partials)
{
  try
  {
    static_assert (sizeof (Ray) == 36, "Ray record");
    RefMesh *r = static_cast<RefMesh *> (h);
    Array<Ray> rays;
    rays.resize (n_rays);
    std::memcpy ((void *)rays.get_host_ptr (), rays9, sizeof (float) * 9 * (size_t)n_rays);
    Volume vol (r->collection);
    vol.field ("f");
    vol.samples (samples);
    vol.use_lighting (use_lighting != 0);
    ColorMap &cmap = vol.color_map ();
    cmap.samples (tf_samples);
    cmap.color_table (make_table (n_rgb, rgb_pts, n_alpha, alpha_pts));
    Array<PointLight> lights = make_lights (n_lights, lights13);
    Array<VolumePartial> partials = vol.integrate (rays, lights);
    const int size = partials.size ();
    const VolumePartial *pp = partials.get_host_ptr_const ();
    if (partials6)
      for (int i = 0; i < size && i < max_partials; ++i)
      {
        partials6[6 * i] = (float)pp[i].m_pixel_id;
        partials6[6 * i + 1] = pp[i].m_depth;
        for (int c = 0; c < 4; ++c) partials6[6 * i + 2 + c] = pp[i].m_color[c];
      }
    return size;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Renderer::render (rendering/renderer.cpp:229-363) over a collection of
// n_dom hex-mesh domains (arrays concatenated: orders, n_elem and n_ctrl per
// domain; their control indices, coordinates and field "f" values one after
// the other), with an optional boundary Surface (MeshBoundary of domains
// surf_first .. surf_first + surf_count - 1; mesh lines when draw_mesh), an
// optional Volume of the whole collection, and the camera
// moved by reset_to_bounds(collection bounds, pads3) when pads3 is given,
// then elevate and azimuth.  Colour bars off.  Writes the framebuffer's
// colours and depths; with save_prefix set, also <prefix>.png and
// <prefix>_depth.png through Framebuffer::save / save_depth.
int ref_render_scene (int n_dom, const int *orders, const int *n_elems, const int *n_ctrls,
                      const int *ctrl_idx, const float *xyz, const float *field, int w, int h,
                      const float *cam9, float fov, const double *pads3, float elevate_deg,
                      float azimuth_deg, int surface, int surf_first, int surf_count,
                      int draw_mesh, float line_thickness,
                      int volume, int samples, int use_lighting, int tf_samples, int n_rgb,
                      const float *rgb_pts, int n_alpha, const float *alpha_pts, float *rgba,
                      float *depth, const char *save_prefix)
{
  try
  {
    Collection col;
    size_t oi = 0, oc = 0;
    for (int d = 0; d < n_dom; ++d)
    {
      const int nd = (orders[d] + 1) * (orders[d] + 1) * (orders[d] + 1);
      GridFunction<3> gf = make_gf3 (n_elems[d], nd, ctrl_idx + oi, n_ctrls[d], xyz + 3 * oc);
      GridFunction<1> ff = make_gf1 (n_elems[d], nd, ctrl_idx + oi, n_ctrls[d], field + oc);
      DataSet ds (make_hex_mesh (orders[d], gf));
      ds.add_field (make_hex_field (orders[d], ff, "f"));
      col.add_domain (ds);
      oi += (size_t)n_elems[d] * nd;
      oc += (size_t)n_ctrls[d];
    }
    Camera cam;
    setup_camera (cam, w, h, cam9, fov);
    if (pads3) cam.reset_to_bounds (col.bounds (), pads3[0], pads3[1], pads3[2]);
    if (elevate_deg != 0.f) cam.elevate (elevate_deg);
    if (azimuth_deg != 0.f) cam.azimuth (azimuth_deg);
    ColorTable table = make_table (n_rgb, rgb_pts, n_alpha, alpha_pts);
    Renderer renderer;
    renderer.color_bar (false);
    renderer.use_lighting (use_lighting != 0);
    Collection faces;
    if (surface)
    {
      Collection part;
      for (int d = surf_first; d < surf_first + surf_count; ++d) part.add_domain (col.domain (d));
      MeshBoundary boundary;
      faces = boundary.execute (part);
      std::shared_ptr<Surface> surf = std::make_shared<Surface> (faces);
      surf->field ("f");
      surf->color_map ().color_table (table);
      surf->draw_mesh (draw_mesh != 0);
      if (draw_mesh) surf->line_thickness (line_thickness);
      renderer.add (surf);
    }
    if (volume)
    {
      std::shared_ptr<Volume> vol = std::make_shared<Volume> (col);
      vol->field ("f");
      vol->samples (samples);
      vol->use_lighting (use_lighting != 0);
      vol->color_map ().samples (tf_samples);
      vol->color_map ().color_table (table);
      renderer.volume (vol);
    }
    Framebuffer fb = renderer.render (cam);
    std::memcpy (rgba, (const void *)fb.colors ().get_host_ptr_const (),
                 sizeof (float) * 4 * (size_t)w * h);
    std::memcpy (depth, fb.depths ().get_host_ptr_const (), sizeof (float) * (size_t)w * h);
    if (save_prefix)
    {
      fb.save (std::string (save_prefix));
      fb.save_depth (std::string (save_prefix) + "_depth");
    }
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// MeshBoundary::execute: number of boundary faces and their (element,
// face-id) pairs are not exposed by the reference, so this returns the
// boundary quad mesh's control-index array (n_faces * (p+1)^2 ints).
int ref_boundary (void *h, int *face_ctrl_idx, int max_faces)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    MeshBoundary mb;
    Collection out = mb.execute (r->collection);
    DataSet ds = out.domain (0);
    Mesh *m = ds.mesh ();
    GridFunction<3> gf;
    if (auto *p = dynamic_cast<QuadMesh_P1 *> (m)) gf = p->get_dof_data ();
    else if (auto *p = dynamic_cast<QuadMesh_P2 *> (m)) gf = p->get_dof_data ();
    else if (auto *p = dynamic_cast<QuadMesh *> (m)) gf = p->get_dof_data ();
    else if (auto *p = dynamic_cast<TriMesh_P1 *> (m)) gf = p->get_dof_data ();
    else if (auto *p = dynamic_cast<TriMesh_P2 *> (m)) gf = p->get_dof_data ();
    else if (auto *p = dynamic_cast<TriMesh *> (m)) gf = p->get_dof_data ();
    else throw std::runtime_error ("boundary: unexpected mesh type");
    const int nf = gf.get_num_elem ();
    if (face_ctrl_idx && nf <= max_faces)
      std::memcpy (face_ctrl_idx, gf.m_ctrl_idx.get_host_ptr_const (), sizeof (int) * (size_t)gf.m_ctrl_idx.size ());
    return nf;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Surface render of the mesh boundary: MeshBoundary -> Surface::nearest_hit
// -> fragments -> shade (lit) into a cleared framebuffer.  Outputs hits
// (idx, dist, ref u, ref v per ray) and the framebuffer (w*h*4 floats +
// w*h depths) before background compositing.
int ref_surface (void *h, int w, int hgt, const float *cam9, float fov, int tf_samples,
                 int n_rgb, const float *rgb_pts, int n_alpha, const float *alpha_pts,
                 int n_lights, const float *lights13, int *hit_idx, float *hit_dist,
                 float *hit_ref2, float *rgba, float *depth)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    MeshBoundary mb;
    Collection faces = mb.execute (r->collection);
    Camera cam;
    setup_camera (cam, w, hgt, cam9, fov);
    Array<Ray> rays;
    cam.create_rays (rays);
    Surface surf (faces);
    surf.field ("f");
    ColorMap &cmap = surf.color_map ();
    cmap.samples (tf_samples);
    cmap.color_table (make_table (n_rgb, rgb_pts, n_alpha, alpha_pts));
    Array<RayHit> hits = surf.nearest_hit (rays);
    Array<Fragment> frags = surf.fragments (hits);
    Framebuffer fb (w, hgt);
    fb.clear ();
    if (n_lights > 0)
    {
      Array<PointLight> lights = make_lights (n_lights, lights13);
      surf.shade (rays, hits, frags, lights, fb);
    }
    else
    {
      surf.shade (rays, hits, frags, fb);
    }
    const RayHit *hp = hits.get_host_ptr_const ();
    const int n = hits.size ();
    for (int i = 0; i < n; ++i)
    {
      if (hit_idx) hit_idx[i] = hp[i].m_hit_idx;
      if (hit_dist) hit_dist[i] = hp[i].m_dist;
      if (hit_ref2)
      {
        hit_ref2[2 * i] = hp[i].m_ref_pt[0];
        hit_ref2[2 * i + 1] = hp[i].m_ref_pt[1];
      }
    }
    if (rgba)
      std::memcpy (rgba, (const void *)fb.colors ().get_host_ptr_const (), sizeof (float) * 4 * (size_t)w * hgt);
    if (depth)
      std::memcpy (depth, fb.depths ().get_host_ptr_const (), sizeof (float) * (size_t)w * hgt);
    return n;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Element<3,1,Tensor,P>::eval_d of one scalar hex element with control
// values `vals` ((p+1)^3, u fastest) at n reference points; fixed != 0 uses
// the fixed-order specialisation (orders 1 and 2), else Order::General.
// This is how the reference's own t_dray_external_evals test drives it.
// The per-pixel writes of ScalarRenderer::render (rendering/scalar_renderer.cpp
// :296-365) on the boundary surface and field "f", driven through the same
// public calls (Surface::nearest_hit, Traceable::fragments): depth and
// scalar start at NaN and zone ids at -1 (ScalarBuffer's clear values).
int ref_scalar_render (void *h, int w, int hgt, const float *cam9, float fov, float *depth,
                       int *zone_id, float *scalar)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    MeshBoundary mb;
    Collection faces = mb.execute (r->collection);
    Camera cam;
    setup_camera (cam, w, hgt, cam9, fov);
    Array<Ray> rays;
    cam.create_rays (rays);
    Surface surf (faces);
    surf.field ("f");
    Array<RayHit> hits = surf.nearest_hit (rays);
    Array<Fragment> frags = surf.fragments (hits);
    const int npix = w * hgt;
    for (int i = 0; i < npix; ++i)
    {
      depth[i] = nan<Float> ();
      scalar[i] = nan<Float> ();
      zone_id[i] = -1;
    }
    const RayHit *hp = hits.get_host_ptr_const ();
    const Ray *rp = rays.get_host_ptr_const ();
    const Fragment *fp = frags.get_host_ptr_const ();
    for (int i = 0; i < (int)hits.size (); ++i)
    {
      if (hp[i].m_hit_idx > -1)
      {
        const int pid = rp[i].m_pixel_id;
        depth[pid] = hp[i].m_dist;
        zone_id[pid] = hp[i].m_hit_idx;
        scalar[pid] = fp[i].m_scalar;
      }
    }
    return npix;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Lineout::execute (queries/lineout.cpp:114-205) on field "f": points
// float[3 * n_lines * (samples + 2)], values float[n_lines * (samples + 2)].
int ref_lineout (void *h, int n_lines, const float *starts, const float *ends, int samples,
                 float empty, float *points, float *values)
{
  try
  {
    RefMesh *r = static_cast<RefMesh *> (h);
    Lineout lo;
    lo.samples (samples);
    lo.empty_val (empty);
    lo.add_var ("f");
    for (int l = 0; l < n_lines; ++l)
    {
      Vec<Float, 3> a, b;
      for (int k = 0; k < 3; ++k)
      {
        a[k] = starts[3 * l + k];
        b[k] = ends[3 * l + k];
      }
      lo.add_line (a, b);
    }
    Lineout::Result res = lo.execute (r->collection);
    const int n = (int)res.m_points.size ();
    std::memcpy (points, (const void *)res.m_points.get_host_ptr_const (), sizeof (float) * 3 * (size_t)n);
    std::memcpy (values, (const void *)res.m_values[0].get_host_ptr_const (), sizeof (float) * (size_t)n);
    return n;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

int ref_eval_hex_scalar (int p, int fixed, const float *vals, int n, const float *ref3,
                         float *out_val, float *out_d3)
{
  try
  {
    const int nd = (p + 1) * (p + 1) * (p + 1);
    std::vector<int32> ids (nd);
    std::vector<Vec<Float, 1>> data (nd);
    for (int i = 0; i < nd; ++i)
    {
      ids[i] = i;
      data[i][0] = vals[i];
    }
    ReadDofPtr<Vec<Float, 1>> rdp;
    rdp.m_offset_ptr = ids.data ();
    rdp.m_dof_ptr = data.data ();
    for (int q = 0; q < n; ++q)
    {
      Vec<Float, 3> r = { { ref3[3 * q], ref3[3 * q + 1], ref3[3 * q + 2] } };
      Vec<Vec<Float, 1>, 3> d;
      Vec<Float, 1> v;
      if (fixed && p == 1)
        v = Element<3, 1, ElemType::Tensor, Order::Linear>::create (0, rdp, p).eval_d (r, d);
      else if (fixed && p == 2)
        v = Element<3, 1, ElemType::Tensor, Order::Quadratic>::create (0, rdp, p).eval_d (r, d);
      else
        v = Element<3, 1, ElemType::Tensor, Order::General>::create (0, rdp, p).eval_d (r, d);
      out_val[q] = v[0];
      for (int k = 0; k < 3; ++k) out_d3[3 * q + k] = d[k][0];
    }
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

// Element<3,1,Simplex,*>::eval_d of one tet scalar element (dofs in the
// reference's order) at n reference points.
int ref_eval_tet_scalar (int p, int fixed, const float *vals, int n, const float *ref3,
                         float *out_val, float *out_d3)
{
  try
  {
    const int nd = (p + 1) * (p + 2) * (p + 3) / 6;
    std::vector<int32> ids (nd);
    std::vector<Vec<Float, 1>> data (nd);
    for (int i = 0; i < nd; ++i)
    {
      ids[i] = i;
      data[i][0] = vals[i];
    }
    ReadDofPtr<Vec<Float, 1>> rdp;
    rdp.m_offset_ptr = ids.data ();
    rdp.m_dof_ptr = data.data ();
    for (int q = 0; q < n; ++q)
    {
      Vec<Float, 3> r = { { ref3[3 * q], ref3[3 * q + 1], ref3[3 * q + 2] } };
      Vec<Vec<Float, 1>, 3> d;
      d = Vec<Float, 1>{ { 0.f } };
      Vec<Float, 1> v;
      if (fixed && p == 1)
        v = Element<3, 1, ElemType::Simplex, Order::Linear>::create (0, rdp, p).eval_d (r, d);
      else if (fixed && p == 2)
        v = Element<3, 1, ElemType::Simplex, Order::Quadratic>::create (0, rdp, p).eval_d (r, d);
      else
        v = Element<3, 1, ElemType::Simplex, Order::General>::create (0, rdp, p).eval_d (r, d);
      out_val[q] = v[0];
      for (int k = 0; k < 3; ++k) out_d3[3 * q + k] = d[k][0];
    }
    return 0;
  }
  catch (const std::exception &e)
  {
    g_err = e.what ();
    return -1;
  }
}

} // extern "C"
