// Implementation of the C++ host interface (include/dray/dray_b200.hpp)
// over the C-ABI of include/drb.h.  Every compute step is a libdrb call on
// the legacy default stream; host synchronisation happens only where the
// reference's API returns host-visible results.
#include "dray/dray_b200.hpp"

#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <fstream>
#include <limits>

#include "drb.h"

namespace dray
{

namespace
{
void drb_check (int st, const char *what)
{
  if (st != DRB_OK)
  {
    std::ostringstream os;
    os << what << " failed (status " << st << "): " << drb_last_error ();
    throw DRayError (os.str ());
  }
}

template <typename T> struct DevBuf
{
  T *p = nullptr;
  size_t n = 0;
  void alloc (size_t count)
  {
    release ();
    n = count;
    if (count) cuda_check (cudaMalloc ((void **)&p, sizeof (T) * count), "cudaMalloc");
  }
  void release ()
  {
    if (p) cudaFree (p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf () { release (); }
};

int32 nd_of (int32 dim, int32 order, ElemType etype)
{
  return drb_elem_dofs (etype == Simplex ? DRB_SHAPE_SIMPLEX : DRB_SHAPE_TENSOR, dim, order);
}

int shape_of (ElemType etype) { return etype == Simplex ? DRB_SHAPE_SIMPLEX : DRB_SHAPE_TENSOR; }
} // namespace

// Device copies, packed element rows and (for meshes) the lazily built BVH.
struct DeviceGeometry
{
  drb_mesh mesh{};
  DevBuf<float> packed;
  bool has_bvh = false;
  drb_bvh bvh{};
  DevBuf<float> inner, refb, wide, hull;
  DevBuf<int32> leaf, ids, nbr;
};

// ------------------------------------------------------------ meshes --

ElementMesh::ElementMesh (const GridFunction<3> &dof, int32 order, int32 dim, ElemType etype)
: m_dof_data (dof), m_poly_order (order), m_dim (dim), m_etype (etype),
  m_dev (std::make_shared<DeviceGeometry> ())
{
  if (order < 1 || order > 3) DRAY_ERROR ("polynomial order " << order << " is outside 1..3");
  if (dof.m_el_dofs != nd_of (dim, order, etype))
    DRAY_ERROR ("GridFunction has " << dof.m_el_dofs << " dofs per element, order " << order
                                    << " needs " << nd_of (dim, order, etype));
}

ElementMesh::~ElementMesh () {}

const drb_mesh *ElementMesh::device_mesh ()
{
  DeviceGeometry &g = *m_dev;
  if (!g.mesh.ctrl_idx || g.mesh.n_elem != cells ())
  {
    g.mesh.dim = m_dim;
    g.mesh.shape = shape_of (m_etype);
    g.mesh.order = m_poly_order;
    g.mesh.ncomp = 3;
    g.mesh.n_elem = cells ();
    g.mesh.n_ctrl = (int)m_dof_data.m_values.size ();
    g.mesh.ctrl_idx = m_dof_data.m_ctrl_idx.get_device_ptr_const ();
    g.mesh.values = (const float *)m_dof_data.m_values.get_device_ptr_const ();
    const int stride = drb_packed_stride_shape (g.mesh.shape, m_dim, m_poly_order, 3);
    g.packed.alloc ((size_t)std::max (cells (), 1) * stride);
    g.mesh.packed = nullptr;
    drb_check (drb_pack_elements (&g.mesh, g.packed.p, nullptr), "drb_pack_elements");
    g.mesh.packed = g.packed.p;
  }
  return &g.mesh;
}

const drb_bvh *ElementMesh::device_bvh ()
{
  DeviceGeometry &g = *m_dev;
  device_mesh ();
  if (!g.has_bvh)
  {
    int ni = 0, nl = 0;
    drb_check (drb_bvh_sizes (m_dim, cells (), &ni, &nl), "drb_bvh_sizes");
    g.inner.alloc ((size_t)16 * ni);
    g.leaf.alloc (nl);
    g.ids.alloc (nl);
    g.refb.alloc ((size_t)drb_ref_box_floats (g.mesh.shape, m_dim) * nl);
    g.bvh.n_inner = ni;
    g.bvh.n_leaf = nl;
    g.bvh.inner_nodes = g.inner.p;
    g.bvh.leaf_nodes = g.leaf.p;
    g.bvh.aabb_ids = g.ids.p;
    g.bvh.ref_boxes = g.refb.p;
    drb_check (drb_lbvh_build (&g.mesh, &g.bvh, nullptr, nullptr), "drb_lbvh_build");
    {
      // 4-wide traversal tree for the batched locate and the volume march
      drb_check (drb_bvh_widen (&g.bvh, nullptr, 0, nullptr), "drb_bvh_widen");
      g.wide.alloc ((size_t)32 * g.bvh.n_wide);
      drb_check (drb_bvh_widen (&g.bvh, g.wide.p, g.bvh.n_wide, nullptr), "drb_bvh_widen");
    }
    if (m_etype == Simplex && m_dim == 3)
    {
      // bounding planes: the batched locate's candidate filter for tets
      g.hull.alloc ((size_t)20 * std::max (cells (), 1));
      drb_check (drb_tet_hull_planes (&g.mesh, g.hull.p, nullptr), "drb_tet_hull_planes");
      g.mesh.hull_planes = g.hull.p;
    }
    if (m_dim == 3)
    {
      // face neighbours: the volume march steps across faces with them
      g.nbr.alloc ((size_t)(m_etype == Simplex ? 4 : 6) * std::max (cells (), 1));
      drb_check (drb_mesh_face_neighbors (&g.mesh, g.nbr.p, nullptr), "drb_mesh_face_neighbors");
      g.mesh.face_neighbors = g.nbr.p;
    }
    g.has_bvh = true;
  }
  return &g.bvh;
}

AABB<3> ElementMesh::bounds ()
{
  const drb_bvh *b = device_bvh ();
  AABB<3> r;
  for (int d = 0; d < 3; ++d)
  {
    if (b->bounds[2 * d] <= b->bounds[2 * d + 1])
    {
      r.m_ranges[d].include (b->bounds[2 * d]);
      r.m_ranges[d].include (b->bounds[2 * d + 1]);
    }
  }
  return r;
}

Array<Location> ElementMesh::locate (Array<Vec<Float, 3>> &wpoints)
{
  const int n = (int)wpoints.size ();
  Array<Location> out;
  out.resize (n);
  if (n == 0) return out;
  const drb_bvh *b = device_bvh ();
  DevBuf<int32> cell;
  DevBuf<float> ref;
  cell.alloc (n);
  ref.alloc ((size_t)3 * n);
  drb_newton_opts opts{ m_locate.tol, m_locate.max_steps, m_locate.guess_mode, nullptr };
  drb_check (drb_locate_batched (device_mesh (), b, (const float *)wpoints.get_device_ptr_const (), n,
                                 &opts, nullptr, cell.p, ref.p, drb_query_stats{}, nullptr),
             "drb_locate_batched");
  std::vector<int32> hc (n);
  std::vector<float> hr ((size_t)3 * n);
  cuda_check (cudaMemcpy (hc.data (), cell.p, sizeof (int32) * n, cudaMemcpyDeviceToHost), "copy");
  cuda_check (cudaMemcpy (hr.data (), ref.p, sizeof (float) * 3 * n, cudaMemcpyDeviceToHost), "copy");
  Location *lp = out.get_host_ptr ();
  for (int i = 0; i < n; ++i)
  {
    lp[i].m_cell_id = hc[i];
    for (int k = 0; k < 3; ++k) lp[i].m_ref_pt[k] = hr[3 * (size_t)i + k];
  }
  return out;
}

// ------------------------------------------------------------ fields --

ElementField::ElementField (const GridFunction<1> &dof, int32 order, int32 dim, const std::string &name,
                            ElemType etype)
: m_dof_data (dof), m_poly_order (order), m_dim (dim), m_etype (etype),
  m_dev (std::make_shared<DeviceGeometry> ())
{
  m_name = name;
  if (order < 1 || order > 3) DRAY_ERROR ("polynomial order " << order << " is outside 1..3");
}

ElementField::~ElementField () {}

const drb_mesh *ElementField::device_field ()
{
  DeviceGeometry &g = *m_dev;
  if (!g.mesh.ctrl_idx)
  {
    g.mesh.dim = m_dim;
    g.mesh.shape = shape_of (m_etype);
    g.mesh.order = m_poly_order;
    g.mesh.ncomp = 1;
    g.mesh.n_elem = m_dof_data.get_num_elem ();
    g.mesh.n_ctrl = (int)m_dof_data.m_values.size ();
    g.mesh.ctrl_idx = m_dof_data.m_ctrl_idx.get_device_ptr_const ();
    g.mesh.values = (const float *)m_dof_data.m_values.get_device_ptr_const ();
    const int stride = drb_packed_stride_shape (g.mesh.shape, m_dim, m_poly_order, 1);
    g.packed.alloc ((size_t)std::max (g.mesh.n_elem, 1) * stride);
    drb_check (drb_pack_elements (&g.mesh, g.packed.p, nullptr), "drb_pack_elements");
    g.mesh.packed = g.packed.p;
  }
  return &g.mesh;
}

std::vector<Range> ElementField::range () const
{
  if (m_range.empty ())
  {
    float r[2];
    DevBuf<float> d;
    d.alloc (2);
    drb_check (drb_field_range (const_cast<ElementField *> (this)->device_field (), d.p, nullptr),
               "drb_field_range");
    cuda_check (cudaMemcpy (r, d.p, sizeof (r), cudaMemcpyDeviceToHost), "copy");
    Range rr;
    if (r[0] <= r[1])
    {
      rr.include (r[0]);
      rr.include (r[1]);
    }
    m_range.push_back (rr);
  }
  return m_range;
}

void ElementField::eval (const Array<Location> locs, Array<Float> &values)
{
  const int n = (int)locs.size ();
  values.resize (n);
  if (n == 0) return;
  // split Location records into cell ids and reference points on the device
  std::vector<int32> cell (n);
  std::vector<float> ref ((size_t)3 * n);
  const Location *lp = locs.get_host_ptr_const ();
  for (int i = 0; i < n; ++i)
  {
    cell[i] = lp[i].m_cell_id;
    for (int k = 0; k < 3; ++k) ref[3 * (size_t)i + k] = lp[i].m_ref_pt[k];
  }
  Array<int32> dcell (cell.data (), n);
  Array<float> dref (ref.data (), (size_t)3 * n);
  drb_check (drb_field_eval (device_field (), dcell.get_device_ptr_const (),
                             dref.get_device_ptr_const (), n, 0.f, values.get_device_ptr (), nullptr),
             "drb_field_eval");
}

// --------------------------------------------------------- collection --

bool DataSet::has_field (const std::string &n) const
{
  for (auto &f : m_fields)
    if (f->name () == n) return true;
  return false;
}

Field *DataSet::field (const std::string &n) { return field_shared (n).get (); }

std::shared_ptr<Field> DataSet::field_shared (const std::string &n)
{
  for (auto &f : m_fields)
    if (f->name () == n) return f;
  DRAY_ERROR ("No field named '" << n << "'");
}

AABB<3> Collection::bounds ()
{
  AABB<3> r;
  for (auto &d : m_domains)
  {
    AABB<3> b = d.mesh ()->bounds ();
    for (int k = 0; k < 3; ++k)
      if (!b.m_ranges[k].is_empty ())
      {
        r.m_ranges[k].include (b.m_ranges[k].min ());
        r.m_ranges[k].include (b.m_ranges[k].max ());
      }
  }
  return r;
}

Range Collection::range (const std::string &field_name)
{
  Range r;
  for (auto &d : m_domains)
    if (d.has_field (field_name))
    {
      Range fr = d.field (field_name)->range ()[0];
      if (!fr.is_empty ())
      {
        r.include (fr.min ());
        r.include (fr.max ());
      }
    }
  return r;
}

// ------------------------------------------------------------ colours --

std::vector<float32> ColorTable::sample (int32 n, float32 alpha_scale, float32 opacity_factor) const
{
  std::vector<float32> out ((size_t)4 * n);
  std::vector<float32> rgb, al;
  for (auto &v : m_rgb)
    for (int k = 0; k < 4; ++k) rgb.push_back (v[k]);
  for (auto &v : m_alpha)
    for (int k = 0; k < 2; ++k) al.push_back (v[k]);
  drb_check (drb_color_table_sample ((int)m_rgb.size (), rgb.empty () ? nullptr : rgb.data (),
                                     (int)m_alpha.size (), al.empty () ? nullptr : al.data (),
                                     m_smooth ? 1 : 0, n, alpha_scale, opacity_factor, out.data ()),
             "drb_color_table_sample");
  return out;
}

// ------------------------------------------------------------- camera --

void Camera::set_width (const int32 &w)
{
  if (w <= 0) DRAY_ERROR ("Camera width must be greater than zero.");
  m_width = w;
}
void Camera::set_height (const int32 &h)
{
  if (h <= 0) DRAY_ERROR ("Camera height must be greater than zero.");
  m_height = h;
}
void Camera::set_fov (const float32 &d)
{
  if (d <= 0) DRAY_ERROR ("Camera feild of view must be greater than zero.");
  if (d > 180) DRAY_ERROR ("Camera feild of view must be less than 180.");
  m_fov_y = d;
}
void Camera::set_zoom (const float32 z)
{
  if (z <= 0) DRAY_ERROR ("Zoom must be greater than 0");
  m_zoom = z;
}

static drb_camera to_drb (const Camera &c)
{
  drb_camera d{};
  d.width = c.get_width ();
  d.height = c.get_height ();
  for (int k = 0; k < 3; ++k)
  {
    d.pos[k] = c.get_pos ()[k];
    d.look_at[k] = c.get_look_at ()[k];
    d.up[k] = c.get_up ()[k];
  }
  d.fov_y = c.get_fov ();
  d.zoom = 1.f;
  return d;
}

void Camera::create_rays (Array<Ray> &rays)
{
  rays.resize ((size_t)m_width * m_height);
  drb_camera d = to_drb (*this);
  d.zoom = m_zoom;
  drb_check (drb_camera_rays (&d, rays.get_device_ptr (), nullptr), "drb_camera_rays");
}

void Camera::create_rays (Array<Ray> &rays, AABB<> bounds)
{
  (void)bounds; // create_rays_imp ignores them (camera.cpp:219-242)
  create_rays (rays);
}

void Camera::reset_to_bounds (const AABB<> bounds, const float64 xpad, const float64 ypad,
                              const float64 zpad)
{
  drb_camera d = to_drb (*this);
  float b6[6];
  for (int k = 0; k < 3; ++k)
  {
    b6[2 * k] = bounds.m_ranges[k].min ();
    b6[2 * k + 1] = bounds.m_ranges[k].max ();
  }
  drb_check (drb_camera_reset_to_bounds (&d, b6, xpad, ypad, zpad), "drb_camera_reset_to_bounds");
  m_pos = make_vec3f (d.pos[0], d.pos[1], d.pos[2]);
  m_look_at = make_vec3f (d.look_at[0], d.look_at[1], d.look_at[2]);
  set_fov (d.fov_y);
}

void Camera::elevate (const float32 degrees)
{
  drb_camera d = to_drb (*this);
  drb_check (drb_camera_elevate (&d, degrees), "drb_camera_elevate");
  m_pos = make_vec3f (d.pos[0], d.pos[1], d.pos[2]);
}

void Camera::azimuth (const float32 degrees)
{
  drb_camera d = to_drb (*this);
  drb_check (drb_camera_azimuth (&d, degrees), "drb_camera_azimuth");
  m_pos = make_vec3f (d.pos[0], d.pos[1], d.pos[2]);
}

PointLight default_light (Camera &camera)
{
  drb_camera d = to_drb (camera);
  float l[13];
  drb_check (drb_default_light (&d, l), "drb_default_light");
  PointLight p;
  for (int k = 0; k < 3; ++k)
  {
    p.m_pos[k] = l[k];
    p.m_amb[k] = l[3 + k];
    p.m_diff[k] = l[6 + k];
    p.m_spec[k] = l[9 + k];
  }
  p.m_spec_pow = l[12];
  return p;
}

// -------------------------------------------------------- framebuffer --

Framebuffer::Framebuffer (int32 w, int32 h) : m_width (w), m_height (h)
{
  m_colors.resize ((size_t)w * h);
  m_depths.resize ((size_t)w * h);
  clear ();
}

void Framebuffer::clear () { clear (make_vec4f (0.f, 0.f, 0.f, 0.f)); }

void Framebuffer::clear (const Vec4f &c)
{
  float col[4] = { c[0], c[1], c[2], c[3] };
  drb_check (drb_framebuffer_clear ((float *)m_colors.get_device_ptr (), m_depths.get_device_ptr (),
                                    m_width * m_height, col, nullptr),
             "drb_framebuffer_clear");
}

void Framebuffer::composite_background ()
{
  float bg[4] = { m_bg_color[0], m_bg_color[1], m_bg_color[2], m_bg_color[3] };
  drb_check (drb_framebuffer_composite_background ((float *)m_colors.get_device_ptr (),
                                                   m_width * m_height, bg, nullptr),
             "drb_framebuffer_composite_background");
}

// PNG file of 8-bit RGBA rows (top row first): signature, IHDR, one zlib
// IDAT of filter-0 scanlines, IEND, each chunk with its CRC-32.
static void write_png (const std::string &path, const std::vector<unsigned char> &rgba, int w,
                       int h)
{
  std::vector<unsigned char> raw ((size_t)h * (1 + 4 * (size_t)w));
  for (int y = 0; y < h; ++y)
  {
    unsigned char *row = raw.data () + (size_t)y * (1 + 4 * (size_t)w);
    row[0] = 0; // filter: none
    std::memcpy (row + 1, rgba.data () + (size_t)y * 4 * w, 4 * (size_t)w);
  }
  uLongf zlen = compressBound ((uLong)raw.size ());
  std::vector<unsigned char> z (zlen);
  if (compress2 (z.data (), &zlen, raw.data (), (uLong)raw.size (), 6) != Z_OK)
    DRAY_ERROR ("png: compression failed");
  z.resize (zlen);
  std::ofstream f (path, std::ios::binary);
  if (!f) DRAY_ERROR ("png: cannot open '" << path << "'");
  auto be32 = [&] (uint32_t v) {
    const unsigned char b[4] = { (unsigned char)(v >> 24), (unsigned char)(v >> 16),
                                 (unsigned char)(v >> 8), (unsigned char)v };
    f.write ((const char *)b, 4);
  };
  auto chunk = [&] (const char *type, const unsigned char *data, size_t len) {
    be32 ((uint32_t)len);
    f.write (type, 4);
    if (len) f.write ((const char *)data, len);
    uLong c = crc32 (0L, (const Bytef *)type, 4);
    if (len) c = crc32 (c, data, (uInt)len);
    be32 ((uint32_t)c);
  };
  const unsigned char sig[8] = { 0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n' };
  f.write ((const char *)sig, 8);
  unsigned char ihdr[13] = { (unsigned char)(w >> 24), (unsigned char)(w >> 16),
                             (unsigned char)(w >> 8),  (unsigned char)w,
                             (unsigned char)(h >> 24), (unsigned char)(h >> 16),
                             (unsigned char)(h >> 8),  (unsigned char)h,
                             8, 6, 0, 0, 0 }; // 8-bit RGBA, deflate, no interlace
  chunk ("IHDR", ihdr, 13);
  chunk ("IDAT", z.data (), z.size ());
  chunk ("IEND", nullptr, 0);
  if (!f) DRAY_ERROR ("png: write failed for '" << path << "'");
}

// PNGEncoder::encode (utils/png_encoder.cpp:61-97): 255 * value truncated
// to 8 bits, framebuffer rows flipped so its last row comes first.
static std::vector<unsigned char> to_rgba8 (const float *rgba, int w, int h)
{
  std::vector<unsigned char> out ((size_t)4 * w * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x)
      for (int c = 0; c < 4; ++c)
      {
        float v = rgba[((size_t)y * w + x) * 4 + c] * 255.f;
        v = v < 0.f ? 0.f : v > 255.f ? 255.f : v; // out-of-range colours saturate
        out[((size_t)(h - y - 1) * w + x) * 4 + c] = (unsigned char)v;
      }
  return out;
}

void Framebuffer::save (const std::string name)
{
  write_png (name + ".png", to_rgba8 ((const float *)m_colors.get_host_ptr_const (), m_width,
                                      m_height),
             m_width, m_height);
}

void Framebuffer::save_depth (const std::string name)
{
  // finite depths scaled to [0, 1] as grey, infinite ones black, alpha 1
  // (framebuffer.cpp:54-105)
  const size_t n = (size_t)m_width * m_height;
  const float *d = m_depths.get_host_ptr_const ();
  float lo = std::numeric_limits<float>::infinity (), hi = -lo;
  for (size_t i = 0; i < n; ++i)
    if (d[i] != std::numeric_limits<float>::infinity ())
    {
      lo = std::min (lo, d[i]);
      hi = std::max (hi, d[i]);
    }
  const float len = hi - lo;
  std::vector<float> g (4 * n);
  for (size_t i = 0; i < n; ++i)
  {
    const float v = d[i] != std::numeric_limits<float>::infinity () ? (d[i] - lo) / len : 0.f;
    g[4 * i] = g[4 * i + 1] = g[4 * i + 2] = v;
    g[4 * i + 3] = 1.f;
  }
  write_png (name + ".png", to_rgba8 (g.data (), m_width, m_height), m_width, m_height);
}

// ------------------------------------------------------------- volume --

Volume::Volume (Collection &c) : m_collection (c)
{
  // Volume() adds two alpha points to its default table (volume.cpp:274-282)
  ColorTable t = m_color_map.color_table ();
  t.add_alpha (0.1f, 0.f);
  t.add_alpha (1.0f, 0.7f);
  m_color_map.color_table (t);
}

static ElementMesh *as_tensor_mesh (Mesh *m)
{
  ElementMesh *t = dynamic_cast<ElementMesh *> (m);
  if (!t) DRAY_ERROR ("mesh type is not a tensor mesh of this path");
  return t;
}
static ElementField *as_tensor_field (Field *f)
{
  ElementField *t = dynamic_cast<ElementField *> (f);
  if (!t) DRAY_ERROR ("field type is not a scalar tensor field of this path");
  return t;
}

void Volume::active_domain (int32 domain_index)
{
  if (domain_index < 0 || domain_index >= num_domains ())
    DRAY_ERROR ("Volume: domain " << domain_index << " of " << num_domains ());
  m_active_domain = domain_index;
}

void Traceable::active_domain (int32 domain_index)
{
  if (domain_index < 0 || domain_index >= num_domains ())
    DRAY_ERROR ("Traceable: domain " << domain_index << " of " << num_domains ());
  m_active_domain = domain_index;
}

Array<VolumePartial> Volume::integrate (Array<Ray> &rays, Array<PointLight> &lights)
{
  if (m_field == "") DRAY_ERROR ("Field never set");
  DataSet ds = m_collection.domain (m_active_domain);
  ElementMesh *mesh = as_tensor_mesh (ds.mesh ());
  ElementField *field = as_tensor_field (ds.field (m_field));
  Range r = m_color_map.range_set () ? m_color_map.scalar_range () : m_collection.range (m_field);
  const AABB<3> bounds = m_collection.bounds ();
  const drb_bvh *bvh = mesh->device_bvh ();
  // remove_missed_rays against the mesh bounds
  const int n = (int)rays.size ();
  Array<Ray> active;
  active.resize (n);
  int n_active = 0;
  drb_check (drb_cull_rays (rays.get_device_ptr_const (), n, bvh->bounds, active.get_device_ptr (),
                            &n_active, nullptr),
             "drb_cull_rays");
  // opacity-corrected table sampled at the default 1024 entries (volume.cpp:81-87)
  std::vector<float32> tf = m_color_map.color_table ().sample (1024, 1.f, 10.f / m_samples);
  Array<Vec4f> tfa ((const Vec4f *)tf.data (), 1024);
  drb_volume_opts o{};
  o.samples = m_samples;
  o.use_lighting = m_use_lighting ? 1 : 0;
  o.tol = m_locate.tol;
  o.max_steps = m_locate.max_steps;
  o.guess_mode = m_locate.guess_mode;
  o.coherent = m_coherent ? 1 : 0;
  for (int d = 0; d < 3; ++d)
  {
    o.bounds[2 * d] = bounds.m_ranges[d].min ();
    o.bounds[2 * d + 1] = bounds.m_ranges[d].max ();
  }
  o.cull = 0;
  float range2[2] = { r.min (), r.max () };
  Array<VolumePartial> out;
  out.resize ((size_t)5 * std::max (n_active, 1));
  int np = 0;
  drb_check (drb_volume_integrate (mesh->device_mesh (), field->device_field (), bvh,
                                   active.get_device_ptr_const (), n_active, &o,
                                   (const float *)tfa.get_device_ptr_const (), 1024, range2,
                                   lights.get_device_ptr_const (), (int)lights.size (),
                                   out.get_device_ptr (), &np, drb_ray_stats{}, nullptr),
             "drb_volume_integrate");
  Array<VolumePartial> res;
  res.resize (np);
  if (np)
    cuda_check (cudaMemcpy (res.get_device_ptr (), out.get_device_ptr_const (),
                            sizeof (VolumePartial) * np, cudaMemcpyDeviceToDevice),
                "copy");
  return res;
}

void Volume::save (const std::string name, Array<VolumePartial> partials, const int32 w,
                   const int32 h)
{
  composite (partials, w, h).save (name);
}

Framebuffer Volume::composite (Array<VolumePartial> partials, int32 w, int32 h)
{
  Framebuffer fb (w, h);
  Array<Vec<float32, 4>> c = fb.colors ();
  drb_check (drb_composite_partials (partials.get_device_ptr_const (), (int)partials.size (),
                                     (float *)c.get_device_ptr (), nullptr),
             "drb_composite_partials");
  fb.composite_background ();
  return fb;
}

// ------------------------------------------------------------ surfaces --

Array<RayHit> Surface::nearest_hit (Array<Ray> &rays)
{
  DataSet ds = m_collection.domain (m_active_domain);
  ElementMesh *faces = as_tensor_mesh (ds.mesh ());
  if (faces->dims () != 2) DRAY_ERROR ("Surface needs a quad (boundary) mesh");
  Array<RayHit> hits;
  hits.resize (rays.size ());
  // face_intersection.hpp:153-154: tol 1e-4, 10 steps
  drb_check (drb_surface_intersect (faces->device_mesh (), faces->device_bvh (),
                                    rays.get_device_ptr_const (), (int)rays.size (), 1e-4f, 10,
                                    hits.get_device_ptr (), drb_ray_stats{}, nullptr),
             "drb_surface_intersect");
  return hits;
}

void Traceable::shade_impl (const Array<Ray> *rays, const Array<RayHit> &hits,
                            const Array<PointLight> *lights, Framebuffer *fb, Array<Fragment> *frags)
{
  DataSet ds = m_collection.domain (m_active_domain);
  ElementMesh *faces = as_tensor_mesh (ds.mesh ());
  ElementField *field = as_tensor_field (ds.field (m_field_name));
  Range r = m_color_map.range_set () ? m_color_map.scalar_range () : m_collection.range (m_field_name);
  std::vector<float32> tf = m_color_map.color_table ().sample (m_color_map.samples ());
  Array<Vec4f> tfa ((const Vec4f *)tf.data (), m_color_map.samples ());
  float range2[2] = { r.min (), r.max () };
  Array<Fragment> local;
  Array<Fragment> &fr = frags ? *frags : local;
  fr.resize (hits.size ());
  Array<Vec<float32, 4>> colors;
  Array<float32> depths;
  if (fb)
  {
    colors = fb->colors ();
    depths = fb->depths ();
  }
  drb_check (drb_surface_shade (faces->device_mesh (), field->device_field (),
                                rays ? rays->get_device_ptr_const () : nullptr,
                                hits.get_device_ptr_const (), (int)hits.size (),
                                (const float *)tfa.get_device_ptr_const (), m_color_map.samples (),
                                range2, lights ? lights->get_device_ptr_const () : nullptr,
                                lights ? (int)lights->size () : 0, lights ? 1 : 0,
                                (float *)fr.get_device_ptr (),
                                fb ? (float *)colors.get_device_ptr () : nullptr,
                                fb ? depths.get_device_ptr () : nullptr, nullptr),
             "drb_surface_shade");
}

Array<Fragment> Traceable::fragments (Array<RayHit> &hits)
{
  // get_fragments (traceable.cpp:49-147): field value and surface normal
  Array<Fragment> frags;
  shade_impl (nullptr, hits, nullptr, nullptr, &frags);
  return frags;
}

void Traceable::shade (const Array<Ray> &rays, const Array<RayHit> &hits, const Array<Fragment> &,
                       const Array<PointLight> &lights, Framebuffer &fb)
{
  shade_impl (&rays, hits, &lights, &fb, nullptr);
}

void Traceable::shade (const Array<Ray> &rays, const Array<RayHit> &hits, const Array<Fragment> &,
                       Framebuffer &fb)
{
  shade_impl (&rays, hits, nullptr, &fb, nullptr);
}

void Surface::line_thickness (const float32 thickness)
{
  if (thickness <= 0.f) DRAY_ERROR ("Cannot have 0 thickness");
  m_line_thickness = thickness;
}

void Surface::mesh_sub_res (float32 sub_res)
{
  if (sub_res < 1.f) DRAY_ERROR ("Sub resolution is a number greater than 1");
  m_sub_res = sub_res;
}

void Surface::draw_mesh (const Array<Ray> &rays, const Array<RayHit> &hits, Framebuffer &fb)
{
  const float lc[4] = { m_line_color[0], m_line_color[1], m_line_color[2], m_line_color[3] };
  Array<Vec<float32, 4>> c = fb.colors ();
  drb_check (drb_surface_mesh_lines (rays.get_device_ptr_const (), hits.get_device_ptr_const (),
                                     (int)hits.size (), lc, m_line_thickness, m_sub_res,
                                     (float *)c.get_device_ptr (), nullptr),
             "drb_surface_mesh_lines");
}

void Surface::shade (const Array<Ray> &rays, const Array<RayHit> &hits,
                     const Array<Fragment> &fragments, const Array<PointLight> &lights,
                     Framebuffer &fb)
{
  Traceable::shade (rays, hits, fragments, lights, fb);
  if (m_draw_mesh) draw_mesh (rays, hits, fb);
}

void Surface::shade (const Array<Ray> &rays, const Array<RayHit> &hits,
                     const Array<Fragment> &fragments, Framebuffer &fb)
{
  Traceable::shade (rays, hits, fragments, fb);
  if (m_draw_mesh) draw_mesh (rays, hits, fb);
}

// ------------------------------------------------------------ filters --

Collection MeshBoundary::execute (Collection &collection)
{
  Collection res;
  for (int32 i = 0; i < collection.local_size (); ++i)
  {
    DataSet ds = collection.domain (i);
    ElementMesh *hex = dynamic_cast<ElementMesh *> (ds.mesh ());
    if (!hex || hex->dims () != 3)
    {
      res.add_domain (ds);
      continue;
    }
    const drb_mesh *dm = hex->device_mesh ();
    int nf = 0;
    drb_check (drb_mesh_boundary (dm, nullptr, nullptr, nullptr, nullptr, &nf, nullptr),
               "drb_mesh_boundary");
    const int p = hex->order ();
    const bool tets = hex->etype () == Simplex;
    const int fd = tets ? (p + 1) * (p + 2) / 2 : (p + 1) * (p + 1);
    GridFunction<3> fg;
    GridFunction<3> vol = hex->get_dof_data ();
    fg.m_values = vol.m_values; // the quads index the volume's value array
    fg.m_el_dofs = fd;
    fg.m_size_el = nf;
    fg.m_size_ctrl = vol.m_size_ctrl;
    fg.m_ctrl_idx.resize ((size_t)nf * fd);
    std::vector<std::shared_ptr<Field>> fields;
    std::vector<GridFunction<1>> fgs;
    // one pass per scalar field (the dof mapping is identical for all)
    DataSet out;
    int32 *fi = fg.m_ctrl_idx.get_device_ptr ();
    drb_check (drb_mesh_boundary (dm, nullptr, fi, nullptr, nullptr, &nf, nullptr), "drb_mesh_boundary");
    std::shared_ptr<Mesh> qm;
    if (tets)
    {
      // a tet mesh's boundary is triangles (mesh_boundary.cpp:102-185)
      if (p == 1) qm = std::make_shared<TriMesh_P1> (fg, 1);
      else if (p == 2) qm = std::make_shared<TriMesh_P2> (fg, 2);
      else qm = std::make_shared<TriMesh> (fg, p);
    }
    else if (p == 1) qm = std::make_shared<QuadMesh_P1> (fg, 1);
    else if (p == 2) qm = std::make_shared<QuadMesh_P2> (fg, 2);
    else qm = std::make_shared<QuadMesh> (fg, p);
    out.add_mesh (qm);
    for (int32 k = 0; k < ds.number_of_fields (); ++k)
    {
      ElementField *f = dynamic_cast<ElementField *> (ds.field (k));
      if (!f || f->order () != p) continue;
      GridFunction<1> vf = f->get_dof_data ();
      GridFunction<1> ff;
      ff.m_values = vf.m_values;
      ff.m_el_dofs = fd;
      ff.m_size_el = nf;
      ff.m_size_ctrl = vf.m_size_ctrl;
      ff.m_ctrl_idx.resize ((size_t)nf * fd);
      drb_check (drb_mesh_boundary (dm, vf.m_ctrl_idx.get_device_ptr_const (),
                                    fg.m_ctrl_idx.get_device_ptr (), ff.m_ctrl_idx.get_device_ptr (),
                                    nullptr, &nf, nullptr),
                 "drb_mesh_boundary");
      std::shared_ptr<Field> qf;
      if (tets && p == 1) qf = std::make_shared<UnstructuredField<TriScalar_P1>> (ff, 1, f->name ());
      else if (tets && p == 2) qf = std::make_shared<UnstructuredField<TriScalar_P2>> (ff, 2, f->name ());
      else if (tets) qf = std::make_shared<UnstructuredField<TriScalar>> (ff, p, f->name ());
      else if (p == 1) qf = std::make_shared<UnstructuredField<QuadScalar_P1>> (ff, 1, f->name ());
      else if (p == 2) qf = std::make_shared<UnstructuredField<QuadScalar_P2>> (ff, 2, f->name ());
      else qf = std::make_shared<UnstructuredField<QuadScalar>> (ff, p, f->name ());
      out.add_field (qf);
    }
    res.add_domain (out);
  }
  return res;
}

PointLocation::Result PointLocation::execute (Collection &collection, Array<Vec<Float, 3>> &points)
{
  // queries/point_location.cpp:178-287, single domain per rank
  Result r;
  r.m_points = points;
  r.m_vars = m_vars;
  r.m_empty_val = m_empty_val;
  const int n = (int)points.size ();
  for (size_t v = 0; v < m_vars.size (); ++v)
  {
    Array<Float> a;
    a.resize (n);
    Float *ap = a.get_host_ptr ();
    for (int i = 0; i < n; ++i) ap[i] = m_empty_val;
    r.m_values.push_back (a);
  }
  for (int32 d = 0; d < collection.local_size (); ++d)
  {
    DataSet ds = collection.domain (d);
    Array<Location> locs = ds.mesh ()->locate (points);
    const Location *lp = locs.get_host_ptr_const ();
    for (size_t v = 0; v < m_vars.size (); ++v)
    {
      if (!ds.has_field (m_vars[v])) continue;
      Array<Float> vals;
      ds.field (m_vars[v])->eval (locs, vals);
      const Float *vp = vals.get_host_ptr_const ();
      Float *out = r.m_values[v].get_host_ptr ();
      for (int i = 0; i < n; ++i)
        if (lp[i].m_cell_id != -1) out[i] = vp[i];
    }
  }
  return r;
}

// ------------------------------------------------------------ renderer --

// ------------------------------------------------------- ScalarRenderer --

ScalarBuffer::ScalarBuffer (int32 width, int32 height, Float clear_value)
: m_width (width), m_height (height), m_clear_value (clear_value)
{
  m_depths.resize ((size_t)width * height);
  m_zone_ids.resize ((size_t)width * height);
  Float *d = m_depths.get_host_ptr ();
  int32 *z = m_zone_ids.get_host_ptr ();
  for (int32 i = 0; i < width * height; ++i)
  {
    d[i] = clear_value;
    z[i] = -1;
  }
}

void ScalarBuffer::add_field (const std::string name)
{
  Array<Float> a;
  a.resize ((size_t)m_width * m_height);
  Float *p = a.get_host_ptr ();
  for (int32 i = 0; i < m_width * m_height; ++i) p[i] = m_clear_value;
  m_scalars[name] = a;
}

ScalarBuffer ScalarRenderer::render (Camera &camera)
{
  // rendering/scalar_renderer.cpp:446-462
  if (!m_traceable) DRAY_ERROR ("ScalarRenderer: traceable never set");
  Array<Ray> rays;
  camera.create_rays (rays);
  ScalarBuffer buffer (camera.get_width (), camera.get_height (),
                       std::numeric_limits<Float>::quiet_NaN ());
  render (rays, buffer);
  return buffer;
}

void ScalarRenderer::render (Array<Ray> &rays, ScalarBuffer &buffer)
{
  // rendering/scalar_renderer.cpp:296-365, one domain (zone offset 0)
  if (!m_traceable) DRAY_ERROR ("ScalarRenderer: traceable never set");
  Array<RayHit> hits = m_traceable->nearest_hit (rays);
  const int n = (int)rays.size ();
  drb_check (drb_scalar_buffer_write (rays.get_device_ptr_const (), hits.get_device_ptr_const (),
                                      nullptr, n, 0, buffer.m_depths.get_device_ptr (),
                                      buffer.m_zone_ids.get_device_ptr (), nullptr, nullptr),
             "drb_scalar_buffer_write");
  const std::string saved = m_traceable->field ();
  for (const std::string &name : m_field_names)
  {
    m_traceable->field (name);
    Array<Fragment> frags;
    try
    {
      frags = m_traceable->fragments (hits);
    }
    catch (const DRayError &)
    {
      continue; // a field this surface does not carry
    }
    if (!buffer.has_field (name)) buffer.add_field (name);
    drb_check (drb_scalar_buffer_write (rays.get_device_ptr_const (), hits.get_device_ptr_const (),
                                        (const float *)frags.get_device_ptr_const (), n, 0, nullptr,
                                        nullptr, buffer.m_scalars[name].get_device_ptr (), nullptr),
               "drb_scalar_buffer_write");
  }
  m_traceable->field (saved);
  drb_check (drb_ray_max (rays.get_device_ptr (), hits.get_device_ptr_const (), n, nullptr),
             "drb_ray_max");
}

// ------------------------------------------------------------ Lineout --

void Lineout::samples (int32 samples)
{
  if (samples < 1) DRAY_ERROR ("Number of samples must be positive");
  m_samples = samples;
}

Array<Vec<Float, 3>> Lineout::create_points ()
{
  // queries/lineout.cpp:98-140, on the device (drb_lineout_points)
  const int32 n = (int32)m_starts.size ();
  Array<Vec<Float, 3>> starts, ends, points;
  starts.resize (n);
  ends.resize (n);
  Vec<Float, 3> *sp = starts.get_host_ptr ();
  Vec<Float, 3> *ep = ends.get_host_ptr ();
  for (int32 i = 0; i < n; ++i)
  {
    sp[i] = m_starts[i];
    ep[i] = m_ends[i];
  }
  points.resize ((size_t)n * (m_samples + 2));
  drb_check (drb_lineout_points ((const float *)starts.get_device_ptr_const (),
                                 (const float *)ends.get_device_ptr_const (), n, m_samples,
                                 (float *)points.get_device_ptr (), nullptr),
             "drb_lineout_points");
  return points;
}

Lineout::Result Lineout::execute (Collection &collection)
{
  // queries/lineout.cpp:114-205
  if (m_vars.empty ()) DRAY_ERROR ("Lineout: must specify at least 1 variables:");
  if (m_starts.empty ()) DRAY_ERROR ("Lineout: must specify at least 1 line:");
  PointLocation locator;
  int32 valid = 0;
  for (const std::string &v : m_vars)
    if (collection.has_field (v))
    {
      locator.add_var (v);
      ++valid;
    }
  if (valid == 0) DRAY_ERROR ("Lineout: must specify at least one valid field.");
  locator.empty_val (m_empty_val);
  Array<Vec<Float, 3>> points = create_points ();
  PointLocation::Result lres = locator.execute (collection, points);
  Result res;
  res.m_points = points;
  res.m_points_per_line = m_samples + 2;
  res.m_vars = m_vars;
  res.m_values = lres.m_values;
  res.m_empty_val = m_empty_val;
  return res;
}

void Renderer::color_bar (bool on)
{
  if (on) DRAY_ERROR ("colour bars draw text, which is not on this path");
  m_color_bar = on;
}
void Renderer::triad (bool on)
{
  if (on) DRAY_ERROR ("the triad annotation is not on this path");
}
void Renderer::world_annotations (bool on)
{
  if (on) DRAY_ERROR ("world annotations are not on this path");
}

Framebuffer Renderer::render (Camera &camera)
{
  // Renderer::render (rendering/renderer.cpp:229-363): every domain of
  // every surface shades and shortens the rays to its hits (ray_max), so a
  // later domain only wins where it is closer; then the volume's partials
  // of all domains, ordered by pixel and depth, are blended per pixel and
  // composited in front of the surfaces (partials_to_framebuffer).
  Array<Ray> rays;
  camera.create_rays (rays);
  Framebuffer fb (camera.get_width (), camera.get_height ());
  std::vector<PointLight> lv = m_lights;
  if (lv.empty ()) lv.push_back (default_light (camera));
  Array<PointLight> lights (lv.data (), lv.size ());
  for (auto &t : m_traceables)
  {
    for (int32 d = 0; d < t->num_domains (); ++d)
    {
      t->active_domain (d);
      Array<RayHit> hits = t->nearest_hit (rays);
      Array<Fragment> frags;
      if (m_use_lighting) t->shade (rays, hits, frags, lights, fb);
      else t->shade (rays, hits, frags, fb);
      drb_check (drb_ray_max (rays.get_device_ptr (), hits.get_device_ptr_const (),
                              (int)rays.size (), nullptr),
                 "drb_ray_max");
    }
  }
  if (m_volume)
  {
    std::vector<Array<VolumePartial>> per_domain;
    size_t total = 0;
    for (int32 d = 0; d < m_volume->num_domains (); ++d)
    {
      m_volume->active_domain (d);
      per_domain.push_back (m_volume->integrate (rays, lights));
      total += per_domain.back ().size ();
    }
    Array<VolumePartial> parts;
    if (per_domain.size () == 1)
      parts = per_domain[0];
    else
    {
      Array<VolumePartial> all;
      all.resize (total);
      size_t off = 0;
      for (auto &p : per_domain)
      {
        if (p.size ())
          cuda_check (cudaMemcpy (all.get_device_ptr () + off, p.get_device_ptr_const (),
                                  sizeof (VolumePartial) * p.size (), cudaMemcpyDeviceToDevice),
                      "copy partials");
        off += p.size ();
      }
      parts.resize (total);
      drb_check (drb_sort_partials (all.get_device_ptr_const (), (int)total,
                                    parts.get_device_ptr (), nullptr),
                 "drb_sort_partials");
    }
    Array<Vec<float32, 4>> c = fb.colors ();
    Array<float32> dep = fb.depths ();
    drb_check (drb_partials_to_framebuffer (parts.get_device_ptr_const (), (int)parts.size (),
                                            (float *)c.get_device_ptr (), dep.get_device_ptr (),
                                            m_traceables.empty () ? 0 : 1, nullptr),
               "drb_partials_to_framebuffer");
  }
  return fb;
}

} // namespace dray
