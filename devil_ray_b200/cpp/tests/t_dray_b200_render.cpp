// Drives the C++ host interface's rendering classes the way a Devil Ray
// user does: a Collection of several hex-mesh domains, a camera placed with
// reset_to_bounds / elevate / azimuth, a boundary Surface with mesh lines
// and a Volume handed to a Renderer (the surface may cover a subset of the
// domains, so that a volume in front of it shows), the framebuffer saved as
// PNG images, and a Volume::save of one domain's partials.  Inputs and outputs are raw binary
// files so the Python test (tests/test_cpp_facade_gpu.py) can compare each
// result with the same calls made on the reference.
//
//   t_dray_b200_render <dir>
//     reads  <dir>/scene.bin   int32 n_dom; per domain int32 order, n_elem, n_ctrl,
//                              int32 ctrl_idx[n_elem*nd], float xyz[3 n_ctrl],
//                              float field[n_ctrl];
//                              int32 w, h; float cam9[9], fov; int32 has_pads;
//                              double pads[3]; float elevate, azimuth;
//                              int32 surface, surf_first, surf_count, draw_mesh;
//                              float line_thickness;
//                              int32 volume, samples, lighting, tf_samples;
//                              int32 n_rgb; float rgb[4 n_rgb]; int32 n_alpha;
//                              float alpha[2 n_alpha]
//     writes <dir>/render.bin  float rgba[4wh]; float depth[wh]  (Renderer::render)
//            <dir>/camera.bin  float pos[3], look_at[3], fov       (after the moves)
//            <dir>/render.png, <dir>/render_depth.png  (Framebuffer::save, save_depth)
//            <dir>/volume.png  (Volume::save of domain 0's partials on the camera's rays)
#include <dray/dray_b200.hpp>

#include <fstream>
#include <iostream>
#include <vector>

using namespace dray;

namespace
{
template <typename T> void rd (std::ifstream &f, T *p, size_t n)
{
  f.read (reinterpret_cast<char *> (p), sizeof (T) * n);
  if (!f) throw std::runtime_error ("short read");
}
template <typename T> T rd1 (std::ifstream &f)
{
  T v;
  rd (f, &v, 1);
  return v;
}
template <typename T> void wr (std::ofstream &f, const T *p, size_t n)
{
  f.write (reinterpret_cast<const char *> (p), sizeof (T) * n);
}

std::shared_ptr<Mesh> hex_mesh (const GridFunction<3> &gf, int32 order)
{
  if (order == 1) return std::make_shared<HexMesh_P1> (gf, order);
  if (order == 2) return std::make_shared<HexMesh_P2> (gf, order);
  return std::make_shared<HexMesh> (gf, order);
}
std::shared_ptr<Field> hex_field (const GridFunction<1> &gf, int32 order)
{
  if (order == 1) return std::make_shared<UnstructuredField<HexScalar_P1>> (gf, order, "f");
  if (order == 2) return std::make_shared<UnstructuredField<HexScalar_P2>> (gf, order, "f");
  return std::make_shared<UnstructuredField<HexScalar>> (gf, order, "f");
}
} // namespace

int main (int argc, char **argv)
{
  if (argc < 2)
  {
    std::cerr << "usage: t_dray_b200_render <dir>\n";
    return 2;
  }
  const std::string dir = argv[1];
  try
  {
    std::ifstream f (dir + "/scene.bin", std::ios::binary);
    const int32 n_dom = rd1<int32> (f);
    Collection col;
    for (int32 d = 0; d < n_dom; ++d)
    {
      const int32 order = rd1<int32> (f), n_elem = rd1<int32> (f), n_ctrl = rd1<int32> (f);
      const int32 nd = (order + 1) * (order + 1) * (order + 1);
      GridFunction<3> gf;
      gf.resize (n_elem, nd, n_ctrl);
      rd (f, gf.m_ctrl_idx.get_host_ptr (), (size_t)n_elem * nd);
      rd (f, (float *)gf.m_values.get_host_ptr (), (size_t)3 * n_ctrl);
      GridFunction<1> ff;
      ff.resize (n_elem, nd, n_ctrl);
      std::memcpy (ff.m_ctrl_idx.get_host_ptr (), gf.m_ctrl_idx.get_host_ptr_const (),
                   sizeof (int32) * (size_t)n_elem * nd);
      rd (f, (float *)ff.m_values.get_host_ptr (), (size_t)n_ctrl);
      DataSet ds (hex_mesh (gf, order));
      ds.add_field (hex_field (ff, order));
      col.add_domain (ds);
    }
    const int32 w = rd1<int32> (f), h = rd1<int32> (f);
    float cam9[9];
    rd (f, cam9, 9);
    const float fov = rd1<float> (f);
    const int32 has_pads = rd1<int32> (f);
    double pads[3];
    rd (f, pads, 3);
    const float elevate = rd1<float> (f), azimuth = rd1<float> (f);
    const int32 surface = rd1<int32> (f), surf_first = rd1<int32> (f);
    const int32 surf_count = rd1<int32> (f), draw_mesh = rd1<int32> (f);
    const float thickness = rd1<float> (f);
    const int32 volume = rd1<int32> (f), samples = rd1<int32> (f), lighting = rd1<int32> (f);
    const int32 tf_samples = rd1<int32> (f);
    ColorTable table;
    const int32 n_rgb = rd1<int32> (f);
    for (int32 i = 0; i < n_rgb; ++i)
    {
      float p[4];
      rd (f, p, 4);
      table.add_point (p[0], make_vec3f (p[1], p[2], p[3]));
    }
    const int32 n_alpha = rd1<int32> (f);
    for (int32 i = 0; i < n_alpha; ++i)
    {
      float p[2];
      rd (f, p, 2);
      table.add_alpha (p[0], p[1]);
    }

    Camera cam;
    cam.set_width (w);
    cam.set_height (h);
    cam.set_pos (make_vec3f (cam9[0], cam9[1], cam9[2]));
    cam.set_look_at (make_vec3f (cam9[3], cam9[4], cam9[5]));
    cam.set_up (make_vec3f (cam9[6], cam9[7], cam9[8]));
    cam.set_fov (fov);
    if (has_pads) cam.reset_to_bounds (col.bounds (), pads[0], pads[1], pads[2]);
    if (elevate != 0.f) cam.elevate (elevate);
    if (azimuth != 0.f) cam.azimuth (azimuth);

    Renderer renderer;
    renderer.use_lighting (lighting != 0);
    std::shared_ptr<Volume> vol;
    if (surface)
    {
      Collection part;
      for (int32 d = surf_first; d < surf_first + surf_count; ++d) part.add_domain (col.domain (d));
      MeshBoundary boundary;
      Collection faces = boundary.execute (part);
      if (faces.local_size () != surf_count) throw std::runtime_error ("boundary domain count");
      auto surf = std::make_shared<Surface> (faces);
      surf->field ("f");
      surf->color_map ().color_table (table);
      surf->draw_mesh (draw_mesh != 0);
      if (draw_mesh) surf->line_thickness (thickness);
      if (surf->num_domains () != surf_count) throw std::runtime_error ("surface domain count");
      renderer.add (surf);
    }
    if (volume)
    {
      vol = std::make_shared<Volume> (col);
      vol->field ("f");
      vol->samples (samples);
      vol->use_lighting (lighting != 0);
      vol->color_map ().samples (tf_samples);
      vol->color_map ().color_table (table);
      renderer.volume (vol);
    }
    // annotations are off this path: asking for one is an error
    bool refused = false;
    try
    {
      renderer.color_bar (true);
    }
    catch (const DRayError &)
    {
      refused = true;
    }
    if (!refused) throw std::runtime_error ("color_bar(true) was accepted");

    Framebuffer fb = renderer.render (cam);
    {
      std::ofstream o (dir + "/render.bin", std::ios::binary);
      wr (o, (const float *)fb.colors ().get_host_ptr_const (), (size_t)4 * w * h);
      wr (o, fb.depths ().get_host_ptr_const (), (size_t)w * h);
      std::ofstream c (dir + "/camera.bin", std::ios::binary);
      const Vec3f p = cam.get_pos (), l = cam.get_look_at ();
      const float cf[7] = { p[0], p[1], p[2], l[0], l[1], l[2], cam.get_fov () };
      wr (c, cf, 7);
    }
    fb.save (dir + "/render");
    fb.save_depth (dir + "/render_depth");
    if (vol)
    {
      vol->active_domain (0);
      Array<Ray> rays;
      cam.create_rays (rays, col.bounds ());
      Array<PointLight> lights;
      lights.resize (1);
      lights.get_host_ptr ()[0] = default_light (cam);
      Array<VolumePartial> parts = vol->integrate (rays, lights);
      Volume::save (dir + "/volume", parts, w, h);
    }
  }
  catch (const std::exception &e)
  {
    std::cerr << "error: " << e.what () << "\n";
    return 1;
  }
  std::cout << "ok\n";
  return 0;
}
