// Stand-in for APComp's volume-partial compositor (a third-party library,
// not in the reference tree).  Devil Ray's Renderer::render hands it one
// vector of partials per rank (rendering/renderer.cpp:323-335); with one rank
// it reduces to ordering each pixel's partials front to back and blending
// them.  This shim does that with the reference's own premultiplied
// front-to-back blend, the one Volume::save uses (rendering/colors.hpp:45-53,
// rendering/volume.cpp:369-416), so the Renderer path and Volume::save agree.
// APComp's own arithmetic is not reproduced: parity at this boundary is
// pinned to Volume::save, not to APComp.
#ifndef ORACLE_SHIM_APCOMP_PARTIAL_COMPOSITOR_HPP
#define ORACLE_SHIM_APCOMP_PARTIAL_COMPOSITOR_HPP
#include <algorithm>
#include <vector>

namespace apcomp
{

template <typename FloatType> struct VolumePartial
{
  int m_pixel_id;
  FloatType m_depth;
  FloatType m_pixel[3];
  FloatType m_alpha;
};

template <typename PartialType> class PartialCompositor
{
  public:
  // One output partial per pixel, in pixel order: the pixel's partials
  // blended front to back; its depth is the front partial's.
  void composite (std::vector<std::vector<PartialType>> &in, std::vector<PartialType> &out)
  {
    std::vector<PartialType> all;
    for (auto &v : in) all.insert (all.end (), v.begin (), v.end ());
    std::stable_sort (all.begin (), all.end (), [] (const PartialType &a, const PartialType &b) {
      return a.m_pixel_id != b.m_pixel_id ? a.m_pixel_id < b.m_pixel_id : a.m_depth < b.m_depth;
    });
    out.clear ();
    for (size_t i = 0; i < all.size ();)
    {
      PartialType acc = all[i];
      size_t j = i + 1;
      for (; j < all.size () && all[j].m_pixel_id == acc.m_pixel_id; ++j)
      {
        const float a = 1.f - acc.m_alpha;
        acc.m_pixel[0] = acc.m_pixel[0] + all[j].m_pixel[0] * a;
        acc.m_pixel[1] = acc.m_pixel[1] + all[j].m_pixel[1] * a;
        acc.m_pixel[2] = acc.m_pixel[2] + all[j].m_pixel[2] * a;
        acc.m_alpha = acc.m_alpha + all[j].m_alpha * a;
      }
      out.push_back (acc);
      i = j;
    }
  }
};

} // namespace apcomp
#endif
