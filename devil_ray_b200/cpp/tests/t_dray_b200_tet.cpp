// Drives the C++ host interface with a tet mesh the way a Devil Ray user
// does: UnstructuredMesh<Tet*> and UnstructuredField<TetScalar*> in a
// DataSet/Collection, Mesh::locate, PointLocation, Volume::integrate, and
// MeshBoundary + Surface on the tets' triangle faces.
// Raw binary inputs and
// outputs, compared with the reference oracle by tests/test_tet_gpu.py.
//
//   t_dray_b200_tet <dir>
//     reads  <dir>/mesh.bin     int32 order, n_elem, n_ctrl; int32 ctrl_idx[n_elem*nd];
//                               float xyz[3*n_ctrl]; float field[n_ctrl]
//                               (nd = (order+1)(order+2)(order+3)/6)
//            <dir>/points.bin   int32 n; float pts[3n]
//            <dir>/render.bin   (optional) int32 w, h, samples; float cam9[9], fov;
//                               float light13[13]; int32 n_rgb; float rgb[4 n_rgb];
//                               int32 n_alpha; float alpha[2 n_alpha]
//     writes <dir>/locate.bin   int32 cell[n]; float ref[3n]
//            <dir>/pointloc.bin float value[n]
//            <dir>/volume.bin   float rgba[4wh]  (Volume::integrate + save
//                               compositing, when render.bin is given)
//            <dir>/surface.bin  float rgba[4wh]; float depth[wh]  (MeshBoundary +
//                               Surface, when render.bin is given)
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
template <typename T> void wr (std::ofstream &f, const T *p, size_t n)
{
  f.write (reinterpret_cast<const char *> (p), sizeof (T) * n);
}
} // namespace

int main (int argc, char **argv)
{
  if (argc < 2)
  {
    std::cerr << "usage: t_dray_b200_tet <dir>\n";
    return 2;
  }
  const std::string dir = argv[1];
  try
  {
    std::ifstream fm (dir + "/mesh.bin", std::ios::binary);
    int32 hdr[3];
    rd (fm, hdr, 3);
    const int32 order = hdr[0], n_elem = hdr[1], n_ctrl = hdr[2];
    const int32 nd = (order + 1) * (order + 2) * (order + 3) / 6;
    GridFunction<3> gf;
    gf.resize (n_elem, nd, n_ctrl);
    rd (fm, gf.m_ctrl_idx.get_host_ptr (), (size_t)n_elem * nd);
    rd (fm, (float *)gf.m_values.get_host_ptr (), (size_t)3 * n_ctrl);
    GridFunction<1> ff;
    ff.resize (n_elem, nd, n_ctrl);
    std::memcpy (ff.m_ctrl_idx.get_host_ptr (), gf.m_ctrl_idx.get_host_ptr_const (),
                 sizeof (int32) * n_elem * nd);
    rd (fm, (float *)ff.m_values.get_host_ptr (), (size_t)n_ctrl);

    std::shared_ptr<Mesh> mesh;
    std::shared_ptr<Field> field;
    if (order == 1)
    {
      mesh = std::make_shared<TetMesh_P1> (gf, 1);
      field = std::make_shared<UnstructuredField<TetScalar_P1>> (ff, 1, "f");
    }
    else if (order == 2)
    {
      mesh = std::make_shared<TetMesh_P2> (gf, 2);
      field = std::make_shared<UnstructuredField<TetScalar_P2>> (ff, 2, "f");
    }
    else
    {
      mesh = std::make_shared<TetMesh> (gf, order);
      field = std::make_shared<UnstructuredField<TetScalar>> (ff, order, "f");
    }
    if (mesh->type_name ().rfind ("Tet_P", 0) != 0) throw std::runtime_error ("type name");
    DataSet ds (mesh);
    ds.add_field (field);
    Collection col;
    col.add_domain (ds);

    std::ifstream fp (dir + "/points.bin", std::ios::binary);
    int32 n = 0;
    rd (fp, &n, 1);
    Array<Vec<Float, 3>> pts;
    pts.resize (n);
    rd (fp, (float *)pts.get_host_ptr (), (size_t)3 * n);
    static_cast<ElementMesh *> (mesh.get ())->m_locate.guess_mode = 0;
    Array<Location> locs = mesh->locate (pts);
    {
      std::ofstream fo (dir + "/locate.bin", std::ios::binary);
      const Location *lp = locs.get_host_ptr_const ();
      std::vector<int32> c (n);
      std::vector<float> r ((size_t)3 * n);
      for (int i = 0; i < n; ++i)
      {
        c[i] = lp[i].m_cell_id;
        for (int k = 0; k < 3; ++k) r[3 * (size_t)i + k] = lp[i].m_ref_pt[k];
      }
      wr (fo, c.data (), n);
      wr (fo, r.data (), r.size ());
    }
    PointLocation pl;
    pl.add_var ("f");
    pl.empty_val (-1e30f);
    PointLocation::Result res = pl.execute (col, pts);
    {
      std::ofstream fo (dir + "/pointloc.bin", std::ios::binary);
      wr (fo, res.m_values[0].get_host_ptr_const (), (size_t)n);
    }

    // Volume::integrate over the tet mesh (dispatch_3d's TetMesh case)
    std::ifstream fr (dir + "/render.bin", std::ios::binary);
    if (fr)
    {
      int32 whs[3];
      rd (fr, whs, 3);
      float cam9[9], fov, light13[13];
      rd (fr, cam9, 9);
      rd (fr, &fov, 1);
      rd (fr, light13, 13);
      int32 nrgb = 0, nal = 0;
      rd (fr, &nrgb, 1);
      std::vector<float> rgb ((size_t)4 * nrgb);
      rd (fr, rgb.data (), rgb.size ());
      rd (fr, &nal, 1);
      std::vector<float> al ((size_t)2 * nal);
      rd (fr, al.data (), al.size ());
      ColorTable table;
      for (int i = 0; i < nrgb; ++i)
        table.add_point (rgb[4 * i], make_vec3f (rgb[4 * i + 1], rgb[4 * i + 2], rgb[4 * i + 3]));
      for (int i = 0; i < nal; ++i) table.add_alpha (al[2 * i], al[2 * i + 1]);
      Camera cam;
      cam.set_width (whs[0]);
      cam.set_height (whs[1]);
      cam.set_pos (make_vec3f (cam9[0], cam9[1], cam9[2]));
      cam.set_look_at (make_vec3f (cam9[3], cam9[4], cam9[5]));
      cam.set_up (make_vec3f (cam9[6], cam9[7], cam9[8]));
      cam.set_fov (fov);
      PointLight light;
      for (int k = 0; k < 3; ++k)
      {
        light.m_pos[k] = light13[k];
        light.m_amb[k] = light13[3 + k];
        light.m_diff[k] = light13[6 + k];
        light.m_spec[k] = light13[9 + k];
      }
      light.m_spec_pow = light13[12];
      Array<PointLight> lights (&light, 1);
      Array<Ray> rays;
      cam.create_rays (rays);
      Volume vol (col);
      vol.field ("f");
      vol.samples (whs[2]);
      vol.use_lighting (true);
      vol.color_map ().color_table (table);
      vol.m_locate.guess_mode = 0;
      Array<VolumePartial> parts = vol.integrate (rays, lights);
      if (parts.size () == 0) throw std::runtime_error ("no partials");
      Framebuffer fb = Volume::composite (parts, whs[0], whs[1]);
      std::ofstream fo (dir + "/volume.bin", std::ios::binary);
      wr (fo, (const float *)fb.colors ().get_host_ptr_const (), (size_t)4 * whs[0] * whs[1]);

      // MeshBoundary (triangle faces) + Surface
      MeshBoundary mb;
      Collection faces = mb.execute (col);
      if (faces.domain (0).mesh ()->type_name ().rfind ("Tri_P", 0) != 0)
        throw std::runtime_error ("boundary type " + faces.domain (0).mesh ()->type_name ());
      Surface surf (faces);
      surf.field ("f");
      surf.color_map ().color_table (table);
      surf.color_map ().samples (1024);
      Array<Ray> srays;
      cam.create_rays (srays);
      Array<RayHit> hits = surf.nearest_hit (srays);
      Array<Fragment> frags = surf.fragments (hits);
      Framebuffer sfb (whs[0], whs[1]);
      surf.shade (srays, hits, frags, lights, sfb);
      std::ofstream fs (dir + "/surface.bin", std::ios::binary);
      wr (fs, (const float *)sfb.colors ().get_host_ptr_const (), (size_t)4 * whs[0] * whs[1]);
      wr (fs, sfb.depths ().get_host_ptr_const (), (size_t)whs[0] * whs[1]);
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
