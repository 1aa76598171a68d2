// Drives the C++ host interface with a tet mesh the way a Devil Ray user
// does: UnstructuredMesh<Tet*> and UnstructuredField<TetScalar*> in a
// DataSet/Collection, Mesh::locate and PointLocation.  Raw binary inputs and
// outputs, compared with the reference oracle by tests/test_tet_gpu.py.
//
//   t_dray_b200_tet <dir>
//     reads  <dir>/mesh.bin     int32 order, n_elem, n_ctrl; int32 ctrl_idx[n_elem*nd];
//                               float xyz[3*n_ctrl]; float field[n_ctrl]
//                               (nd = (order+1)(order+2)(order+3)/6)
//            <dir>/points.bin   int32 n; float pts[3n]
//     writes <dir>/locate.bin   int32 cell[n]; float ref[3n]
//            <dir>/pointloc.bin float value[n]
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
  }
  catch (const std::exception &e)
  {
    std::cerr << "error: " << e.what () << "\n";
    return 1;
  }
  std::cout << "ok\n";
  return 0;
}
