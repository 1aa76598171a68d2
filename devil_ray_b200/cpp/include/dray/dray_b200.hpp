// C++ host interface of the B200 ray-element path, mirroring the classes of
// Devil Ray that sit on it (names, argument meaning, error behaviour), over
// the C-ABI of include/drb.h:
//
//   Vec, Range, AABB                         vec.hpp, range.hpp, aabb.hpp
//   GridFunction                             data_model/grid_function.hpp:19-50
//   Element tags, UnstructuredMesh,
//   UnstructuredField, Mesh, Field           data_model/unstructured_mesh.hpp,
//                                            unstructured_field.hpp, mesh.hpp, field.hpp
//   DataSet, Collection                      data_model/data_set.hpp, collection.hpp
//   Location, Ray, RayHit, Fragment,
//   VolumePartial, PointLight                location.hpp, ray.hpp, ray_hit.hpp,
//                                            rendering/{fragment,volume_partial,point_light}.hpp
//   ColorTable, ColorMap                     color_table.hpp, color_map.hpp
//   Camera, Framebuffer                      rendering/camera.hpp, framebuffer.hpp
//   Volume, Traceable, Surface, Renderer     rendering/{volume,traceable,surface,renderer}.hpp
//   MeshBoundary, PointLocation              filters/mesh_boundary.hpp, queries/point_location.hpp
//
// Only tensor (hex / quad) elements of order 1-3 are supported; other element
// types are outside this path and raise DRayError.
#pragma once

#include <cmath>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "array.hpp"

struct drb_bvh;
struct drb_mesh;

namespace dray
{

template <typename T, int32 S> struct Vec
{
  T m_data[S];
  T &operator[] (int32 i) { return m_data[i]; }
  const T &operator[] (int32 i) const { return m_data[i]; }
};
using Vec3f = Vec<float32, 3>;
using Vec4f = Vec<float32, 4>;
inline Vec3f make_vec3f (float32 x, float32 y, float32 z) { return { { x, y, z } }; }
inline Vec4f make_vec4f (float32 x, float32 y, float32 z, float32 w) { return { { x, y, z, w } }; }

class Range
{
  Float m_min = INFINITY, m_max = -INFINITY;
  public:
  void include (Float v)
  {
    m_min = fminf (m_min, v);
    m_max = fmaxf (m_max, v);
  }
  bool is_empty () const { return m_min > m_max; }
  Float min () const { return m_min; }
  Float max () const { return m_max; }
  Float length () const { return m_max - m_min; }
};

template <int32 dim = 3> struct AABB
{
  Range m_ranges[dim];
  bool is_empty () const
  {
    for (int d = 0; d < dim; ++d)
      if (!m_ranges[d].is_empty ()) return false;
    return true;
  }
};

// element tags (data_model/element.hpp)
enum ElemType { Tensor = 0, Simplex = 1 };
namespace Order
{
enum { General = -1, Constant = 0, Linear = 1, Quadratic = 2 };
}
template <int32 dim, int32 ncomp, ElemType etype, int32 P = Order::General> struct Element
{
  static constexpr int32 get_dim () { return dim; }
  static constexpr int32 get_ncomp () { return ncomp; }
  static constexpr ElemType get_etype () { return etype; }
  static constexpr int32 get_P () { return P; }
};
using Hex3 = Element<3, 3, Tensor, Order::General>;
using Hex_P1 = Element<3, 3, Tensor, Order::Linear>;
using Hex_P2 = Element<3, 3, Tensor, Order::Quadratic>;
using Quad3 = Element<2, 3, Tensor, Order::General>;
using Quad_P1 = Element<2, 3, Tensor, Order::Linear>;
using Quad_P2 = Element<2, 3, Tensor, Order::Quadratic>;
using HexScalar = Element<3, 1, Tensor, Order::General>;
using HexScalar_P1 = Element<3, 1, Tensor, Order::Linear>;
using HexScalar_P2 = Element<3, 1, Tensor, Order::Quadratic>;
using QuadScalar = Element<2, 1, Tensor, Order::General>;
using QuadScalar_P1 = Element<2, 1, Tensor, Order::Linear>;
using QuadScalar_P2 = Element<2, 1, Tensor, Order::Quadratic>;
// Tets (data_model/unstructured_mesh.hpp:121-124, unstructured_field.hpp:95-98).
// The fixed-order Linear type evaluates like the general one here: the
// reference's Tet_P1 eval_d leaves two derivatives unset (elem_ops.hpp:785-815).
using Tet3 = Element<3, 3, Simplex, Order::General>;
using Tet_P1 = Element<3, 3, Simplex, Order::Linear>;
using Tet_P2 = Element<3, 3, Simplex, Order::Quadratic>;
using TetScalar = Element<3, 1, Simplex, Order::General>;
using TetScalar_P1 = Element<3, 1, Simplex, Order::Linear>;
using TetScalar_P2 = Element<3, 1, Simplex, Order::Quadratic>;
// Triangles: the boundary faces of tet meshes (unstructured_mesh.hpp:129-131).
using Tri3 = Element<2, 3, Simplex, Order::General>;
using Tri_P1 = Element<2, 3, Simplex, Order::Linear>;
using Tri_P2 = Element<2, 3, Simplex, Order::Quadratic>;
using TriScalar = Element<2, 1, Simplex, Order::General>;
using TriScalar_P1 = Element<2, 1, Simplex, Order::Linear>;
using TriScalar_P2 = Element<2, 1, Simplex, Order::Quadratic>;

template <int32 PhysDim> struct GridFunction
{
  Array<int32> m_ctrl_idx;
  Array<Vec<Float, PhysDim>> m_values;
  int32 m_el_dofs = 0;
  int32 m_size_el = 0;
  int32 m_size_ctrl = 0;
  void resize (int32 size_el, int32 el_dofs, int32 size_ctrl)
  {
    m_el_dofs = el_dofs;
    m_size_el = size_el;
    m_size_ctrl = size_ctrl;
    m_ctrl_idx.resize ((size_t)size_el * el_dofs);
    m_values.resize (size_ctrl);
  }
  int32 get_num_elem () const { return m_size_el; }
};

struct Location
{
  int32 m_cell_id;
  Vec<Float, 3> m_ref_pt;
};
struct Ray
{
  Vec<Float, 3> m_dir;
  Float m_near;
  Vec<Float, 3> m_orig;
  Float m_far;
  int32 m_pixel_id;
};
struct RayHit
{
  int32 m_hit_idx;
  Float m_dist;
  Vec<Float, 3> m_ref_pt;
};
struct Fragment
{
  float32 m_scalar;
  Vec<float32, 3> m_normal;
};
struct VolumePartial
{
  int32 m_pixel_id;
  float32 m_depth;
  Vec<float32, 4> m_color;
};
struct PointLight
{
  Vec<float32, 3> m_pos = { { 0.f, 0.f, 0.f } };
  Vec<float32, 3> m_amb = { { 0.4f, 0.4f, 0.4f } };
  Vec<float32, 3> m_diff = { { 0.75f, 0.75f, 0.75f } };
  Vec<float32, 3> m_spec = { { 0.8f, 0.8f, 0.8f } };
  float32 m_spec_pow = 15.f;
};

// Newton settings of point location; the reference hard-codes tol 1e-4 and
// 20 steps (data_model/element.hpp:474-475).  guess_mode is drb_guess_mode.
struct LocateSettings
{
  Float tol = 1e-4f;
  int32 max_steps = 20;
  int32 guess_mode = 1; // element centre
};

class Mesh
{
  protected:
  std::string m_name;
  public:
  virtual ~Mesh () {}
  std::string name () const { return m_name; }
  void name (const std::string &n) { m_name = n; }
  virtual std::string type_name () const = 0;
  virtual int32 cells () const = 0;
  virtual int32 order () const = 0;
  virtual int32 dims () const = 0;
  virtual AABB<3> bounds () = 0;
  virtual Array<Location> locate (Array<Vec<Float, 3>> &wpoints) = 0;
};

// Device state shared by meshes and fields of one element layout.
struct DeviceGeometry;

class Field
{
  protected:
  std::string m_name;
  public:
  virtual ~Field () {}
  std::string name () const { return m_name; }
  void name (const std::string &n) { m_name = n; }
  virtual std::vector<Range> range () const = 0;
  virtual int32 order () const = 0;
  virtual int32 components () const = 0;
  virtual std::string type_name () const = 0;
  virtual void eval (const Array<Location> locs, Array<Float> &values) = 0;
};

// Non-template core of UnstructuredMesh (dim 3 hex or tet, dim 2 quad).
class ElementMesh : public Mesh
{
  protected:
  GridFunction<3> m_dof_data;
  int32 m_poly_order;
  int32 m_dim;
  ElemType m_etype;
  std::shared_ptr<DeviceGeometry> m_dev;
  public:
  LocateSettings m_locate;
  ElementMesh (const GridFunction<3> &dof, int32 order, int32 dim, ElemType etype = Tensor);
  ElemType etype () const { return m_etype; }
  ~ElementMesh () override;
  int32 cells () const override { return m_dof_data.get_num_elem (); }
  int32 order () const override { return m_poly_order; }
  int32 dims () const override { return m_dim; }
  AABB<3> bounds () override;
  Array<Location> locate (Array<Vec<Float, 3>> &wpoints) override;
  GridFunction<3> get_dof_data () { return m_dof_data; }
  // device handles for the C-ABI (BVH built lazily, like get_bvh())
  const drb_mesh *device_mesh ();
  const drb_bvh *device_bvh ();
};

template <class ElemT> class UnstructuredMesh : public ElementMesh
{
  static_assert (ElemT::get_dim () == 2 || ElemT::get_dim () == 3, "2D or 3D elements");
  static_assert (ElemT::get_ncomp () == 3, "meshes have 3 components");
  public:
  UnstructuredMesh (const GridFunction<3> &dof, int32 order)
  : ElementMesh (dof, order, ElemT::get_dim (), ElemT::get_etype ())
  {
    if (ElemT::get_P () != Order::General && ElemT::get_P () != order)
      DRAY_ERROR ("Fixed order mismatch. Poly order " << order << " template " << ElemT::get_P ());
  }
  std::string type_name () const override
  {
    const char *n = ElemT::get_etype () == Simplex ? (ElemT::get_dim () == 3 ? "Tet" : "Tri")
                    : ElemT::get_dim () == 3                ? "Hex"
                                                            : "Quad";
    return std::string (n) + "_P" + std::to_string (m_poly_order);
  }
};
using HexMesh = UnstructuredMesh<Hex3>;
using HexMesh_P1 = UnstructuredMesh<Hex_P1>;
using HexMesh_P2 = UnstructuredMesh<Hex_P2>;
using QuadMesh = UnstructuredMesh<Quad3>;
using QuadMesh_P1 = UnstructuredMesh<Quad_P1>;
using QuadMesh_P2 = UnstructuredMesh<Quad_P2>;
using TetMesh = UnstructuredMesh<Tet3>;
using TetMesh_P1 = UnstructuredMesh<Tet_P1>;
using TetMesh_P2 = UnstructuredMesh<Tet_P2>;
using TriMesh = UnstructuredMesh<Tri3>;
using TriMesh_P1 = UnstructuredMesh<Tri_P1>;
using TriMesh_P2 = UnstructuredMesh<Tri_P2>;

class ElementField : public Field
{
  protected:
  GridFunction<1> m_dof_data;
  int32 m_poly_order;
  int32 m_dim;
  ElemType m_etype;
  std::shared_ptr<DeviceGeometry> m_dev;
  mutable std::vector<Range> m_range;
  public:
  ElementField (const GridFunction<1> &dof, int32 order, int32 dim, const std::string &name,
                ElemType etype = Tensor);
  ~ElementField () override;
  std::vector<Range> range () const override;
  int32 order () const override { return m_poly_order; }
  int32 components () const override { return 1; }
  void eval (const Array<Location> locs, Array<Float> &values) override;
  GridFunction<1> get_dof_data () { return m_dof_data; }
  const drb_mesh *device_field ();
};

template <class ElemT> class UnstructuredField : public ElementField
{
  static_assert (ElemT::get_ncomp () == 1, "only scalar fields are on this path");
  public:
  UnstructuredField (const GridFunction<1> &dof, int32 order, const std::string &name = "")
  : ElementField (dof, order, ElemT::get_dim (), name, ElemT::get_etype ())
  {
  }
  std::string type_name () const override
  {
    const char *n = ElemT::get_etype () == Simplex ? (ElemT::get_dim () == 3 ? "TetScalar" : "TriScalar")
                    : ElemT::get_dim () == 3                ? "HexScalar"
                                                            : "QuadScalar";
    return std::string (n) + "_P" + std::to_string (m_poly_order);
  }
};

class DataSet
{
  std::vector<std::shared_ptr<Mesh>> m_meshes;
  std::vector<std::shared_ptr<Field>> m_fields;
  public:
  DataSet () {}
  explicit DataSet (std::shared_ptr<Mesh> m) { m_meshes.push_back (m); }
  void add_mesh (std::shared_ptr<Mesh> m) { m_meshes.push_back (m); }
  Mesh *mesh (int32 i = 0) { return m_meshes.at (i).get (); }
  std::shared_ptr<Mesh> mesh_shared (int32 i = 0) { return m_meshes.at (i); }
  int32 number_of_meshes () const { return (int32)m_meshes.size (); }
  void add_field (std::shared_ptr<Field> f) { m_fields.push_back (f); }
  int32 number_of_fields () const { return (int32)m_fields.size (); }
  bool has_field (const std::string &n) const;
  Field *field (const std::string &n);
  Field *field (int32 i) { return m_fields.at (i).get (); }
  std::shared_ptr<Field> field_shared (const std::string &n);
};

class Collection
{
  std::vector<DataSet> m_domains;
  public:
  void add_domain (const DataSet &d) { m_domains.push_back (d); }
  DataSet domain (int32 i) { return m_domains.at (i); }
  int32 local_size () const { return (int32)m_domains.size (); }
  int32 size () const { return local_size (); }
  AABB<3> bounds ();
  Range range (const std::string &field_name);
  bool has_field (const std::string &field_name)
  {
    for (auto &d : m_domains)
      if (d.has_field (field_name)) return true;
    return false;
  }
};

class ColorTable
{
  std::vector<Vec<float32, 4>> m_rgb;   // (pos, r, g, b)
  std::vector<Vec<float32, 2>> m_alpha; // (pos, a)
  bool m_smooth = true;
  public:
  ColorTable () {}
  void add_point (float32 pos, const Vec3f &c) { m_rgb.push_back ({ { pos, c[0], c[1], c[2] } }); }
  void add_alpha (float32 pos, float32 a) { m_alpha.push_back ({ { pos, a } }); }
  void set_smooth (bool s) { m_smooth = s; }
  void clear () { m_rgb.clear (); m_alpha.clear (); }
  // ColorTable::sample after correct_opacity(factor) (factor <= 0: none)
  std::vector<float32> sample (int32 n, float32 alpha_scale = 1.f, float32 opacity_factor = 0.f) const;
};

class ColorMap
{
  ColorTable m_table;
  int32 m_samples = 1024;
  Range m_range;
  public:
  void color_table (const ColorTable &t) { m_table = t; }
  ColorTable color_table () const { return m_table; }
  void samples (int32 n) { m_samples = n; }
  int32 samples () const { return m_samples; }
  void scalar_range (const Range &r) { m_range = r; }
  Range scalar_range () const { return m_range; }
  bool range_set () const { return !m_range.is_empty (); }
};

class Camera
{
  int32 m_width = 500, m_height = 500;
  float32 m_fov_y = 30.f, m_zoom = 1.f;
  Vec3f m_pos = { { 0.f, 0.f, 0.f } }, m_look_at = { { 0.f, 0.f, -1.f } }, m_up = { { 0.f, 1.f, 0.f } };
  public:
  void set_width (const int32 &w);
  void set_height (const int32 &h);
  int32 get_width () const { return m_width; }
  int32 get_height () const { return m_height; }
  void set_fov (const float32 &degrees);
  float32 get_fov () const { return m_fov_y; }
  void set_zoom (const float32 z);
  void set_pos (const Vec3f &p) { m_pos = p; }
  void set_look_at (const Vec3f &p) { m_look_at = p; }
  void set_up (const Vec3f &u) { m_up = u; }
  Vec3f get_pos () const { return m_pos; }
  Vec3f get_look_at () const { return m_look_at; }
  Vec3f get_up () const { return m_up; }
  void create_rays (Array<Ray> &rays);
  // the bounds are accepted and, as in the reference, not used
  void create_rays (Array<Ray> &rays, AABB<> bounds);
  // Camera::reset_to_bounds / elevate / azimuth (rendering/camera.cpp:485-555)
  void reset_to_bounds (const AABB<> bounds, const float64 xpad = 0., const float64 ypad = 0.,
                        const float64 zpad = 0.);
  void elevate (const float32 degrees);
  void azimuth (const float32 degrees);
};

class Framebuffer
{
  Array<Vec<float32, 4>> m_colors;
  Array<float32> m_depths;
  int32 m_width, m_height;
  Vec4f m_bg_color = { { 1.f, 1.f, 1.f, 1.f } };
  public:
  Framebuffer (int32 width = 1024, int32 height = 1024);
  int32 width () const { return m_width; }
  int32 height () const { return m_height; }
  void clear ();
  void clear (const Vec4f &color);
  void composite_background ();
  void background_color (const Vec4f &c) { m_bg_color = c; }
  Array<Vec<float32, 4>> colors () const { return m_colors; }
  Array<float32> depths () const { return m_depths; }
  // Framebuffer::save / save_depth (rendering/framebuffer.cpp:45-105):
  // <name>.png, 8-bit RGBA, first image row at the top (the framebuffer's
  // last row); the depth image is the finite depths scaled to [0, 1] as grey
  void save (const std::string name);
  void save_depth (const std::string name);
};

// Default point light above the camera (detail::default_light,
// rendering/renderer.cpp:141-159).
PointLight default_light (Camera &camera);

class Volume
{
  Collection m_collection;
  std::string m_field;
  int32 m_samples = 100;
  bool m_use_lighting = true;
  ColorMap m_color_map;
  int32 m_active_domain = 0;
  public:
  explicit Volume (Collection &c);
  // the domain integrate() works on (volume.hpp:36-38)
  void active_domain (int32 domain_index);
  int32 active_domain () const { return m_active_domain; }
  int32 num_domains () const { return m_collection.local_size (); }
  void field (const std::string f) { m_field = f; }
  std::string field () const { return m_field; }
  void samples (int32 n) { m_samples = n; }
  void use_lighting (bool on) { m_use_lighting = on; }
  ColorMap &color_map () { return m_color_map; }
  LocateSettings m_locate;
  bool m_coherent = false; // try the previous sample's element first
  Array<VolumePartial> integrate (Array<Ray> &rays, Array<PointLight> &lights);
  // Volume::save without the PNG: partials composited over white
  static Framebuffer composite (Array<VolumePartial> partials, int32 width, int32 height);
  // Volume::save (rendering/volume.cpp:369-416): composite, then <name>.png
  static void save (const std::string name, Array<VolumePartial> partials, const int32 width,
                    const int32 height);
};

class Traceable
{
  protected:
  Collection m_collection;
  std::string m_field_name;
  ColorMap m_color_map;
  int32 m_active_domain = 0;
  public:
  explicit Traceable (Collection &c) : m_collection (c) {}
  virtual ~Traceable () {}
  // the domain nearest_hit/fragments/shade work on (traceable.hpp:63-65)
  void active_domain (int32 domain_index);
  int32 active_domain () const { return m_active_domain; }
  int32 num_domains () const { return m_collection.local_size (); }
  void field (const std::string &f) { m_field_name = f; }
  std::string field () const { return m_field_name; }
  ColorMap &color_map () { return m_color_map; }
  virtual Array<RayHit> nearest_hit (Array<Ray> &rays) = 0;
  virtual Array<Fragment> fragments (Array<RayHit> &hits);
  virtual void shade (const Array<Ray> &rays, const Array<RayHit> &hits,
                      const Array<Fragment> &fragments, const Array<PointLight> &lights,
                      Framebuffer &fb);
  virtual void shade (const Array<Ray> &rays, const Array<RayHit> &hits,
                      const Array<Fragment> &fragments, Framebuffer &fb);
  protected:
  void shade_impl (const Array<Ray> *rays, const Array<RayHit> &hits, const Array<PointLight> *lights,
                   Framebuffer *fb, Array<Fragment> *frags);
};

class Surface : public Traceable
{
  bool m_draw_mesh = false;
  float32 m_line_thickness = 0.05f;
  float32 m_sub_res = 1.f;
  Vec4f m_line_color = { { 0.f, 0.f, 0.f, 1.f } };
  void draw_mesh (const Array<Ray> &rays, const Array<RayHit> &hits, Framebuffer &fb);
  public:
  explicit Surface (Collection &c) : Traceable (c) {}
  Array<RayHit> nearest_hit (Array<Ray> &rays) override;
  // mesh lines over the shaded faces (rendering/surface.cpp:507-627)
  void draw_mesh (bool on) { m_draw_mesh = on; }
  void line_thickness (const float32 thickness);
  void line_color (const Vec4f &color) { m_line_color = color; }
  void mesh_sub_res (float32 sub_res);
  void shade (const Array<Ray> &rays, const Array<RayHit> &hits, const Array<Fragment> &fragments,
              const Array<PointLight> &lights, Framebuffer &fb) override;
  void shade (const Array<Ray> &rays, const Array<RayHit> &hits, const Array<Fragment> &fragments,
              Framebuffer &fb) override;
};

class MeshBoundary
{
  public:
  Collection execute (Collection &collection);
};

class PointLocation
{
  Float m_empty_val = 0.f;
  std::vector<std::string> m_vars;
  public:
  struct Result
  {
    Array<Vec<Float, 3>> m_points;
    std::vector<Array<Float>> m_values;
    std::vector<std::string> m_vars;
    Float m_empty_val;
  };
  void empty_val (const Float v) { m_empty_val = v; }
  void add_var (const std::string v) { m_vars.push_back (v); }
  Result execute (Collection &collection, Array<Vec<Float, 3>> &points);
};

// ScalarBuffer (rendering/scalar_buffer.hpp): per-pixel depth, zone id and
// one plane per field, cleared to the clear value (zone ids to -1).
class ScalarBuffer
{
  public:
  int32 m_width = 0, m_height = 0;
  Float m_clear_value = 0.f;
  Array<Float> m_depths;
  Array<int32> m_zone_ids;
  std::map<std::string, Array<Float>> m_scalars;
  ScalarBuffer () {}
  ScalarBuffer (int32 width, int32 height, Float clear_value);
  bool has_field (const std::string name) { return m_scalars.find (name) != m_scalars.end (); }
  void add_field (const std::string name);
  int32 size () const { return m_width * m_height; }
};

// ScalarRenderer (rendering/scalar_renderer.hpp), one domain: the nearest
// hit of each ray, its depth and zone id, and each named field's value at
// the hit, per pixel.
class ScalarRenderer
{
  std::shared_ptr<Traceable> m_traceable;
  std::vector<std::string> m_field_names;
  public:
  ScalarRenderer () {}
  explicit ScalarRenderer (std::shared_ptr<Traceable> traceable) : m_traceable (traceable) {}
  void set (std::shared_ptr<Traceable> traceable) { m_traceable = traceable; }
  void field_names (const std::vector<std::string> &names) { m_field_names = names; }
  ScalarBuffer render (Camera &camera);
  void render (Array<Ray> &rays, ScalarBuffer &scalar_buffer);
};

// Lineout (queries/lineout.hpp): field values at samples + 2 evenly spaced
// points along each line, start and end included.
class Lineout
{
  int32 m_samples = 100;
  Float m_empty_val = 0.f;
  std::vector<Vec<Float, 3>> m_starts, m_ends;
  std::vector<std::string> m_vars;
  public:
  struct Result
  {
    Array<Vec<Float, 3>> m_points;
    int32 m_points_per_line;
    std::vector<Array<Float>> m_values;
    std::vector<std::string> m_vars;
    Float m_empty_val;
  };
  int32 samples () const { return m_samples; }
  void samples (int32 samples);
  void empty_val (const Float val) { m_empty_val = val; }
  void add_line (const Vec<Float, 3> start, const Vec<Float, 3> end)
  {
    m_starts.push_back (start);
    m_ends.push_back (end);
  }
  void add_var (const std::string var) { m_vars.push_back (var); }
  Result execute (Collection &collection);
  Array<Vec<Float, 3>> create_points ();
};

class Renderer
{
  std::vector<std::shared_ptr<Traceable>> m_traceables;
  std::shared_ptr<Volume> m_volume;
  std::vector<PointLight> m_lights;
  bool m_use_lighting = true;
  bool m_color_bar = false;
  public:
  // Colour bars, triad and world annotations draw text and are not on this
  // path: asking for them raises DRayError (the reference draws colour bars
  // by default; renderer.cpp:166-169).
  void color_bar (bool on);
  void triad (bool on);
  void world_annotations (bool on);
  void add (std::shared_ptr<Traceable> t) { m_traceables.push_back (t); }
  void volume (std::shared_ptr<Volume> v) { m_volume = v; }
  void add_light (const PointLight &l) { m_lights.push_back (l); }
  void use_lighting (bool on) { m_use_lighting = on; }
  Framebuffer render (Camera &camera);
};

} // namespace dray
