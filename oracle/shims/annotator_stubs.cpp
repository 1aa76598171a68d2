// Link stand-ins for Devil Ray's screen and world annotators (colour bars,
// triad, axes and text: rendering/screen_annotator.cpp, world_annotator.cpp),
// which Renderer::render calls only when those options are on.  Their
// sources need fonts and Conduit's fmt, which the oracle build does not
// have; the parity tests turn the options off, so any call here is a test
// set-up error and throws.
#include <dray/rendering/screen_annotator.hpp>
#include <dray/rendering/world_annotator.hpp>

#include <stdexcept>

namespace dray
{
static void not_in_oracle (const char *what)
{
  throw std::runtime_error (std::string (what) + " is not built into the oracle; "
                            "turn the annotation off");
}

ScreenAnnotator::ScreenAnnotator () : m_max_color_bars (2) {}
void ScreenAnnotator::max_color_bars (int max_bars) { m_max_color_bars = max_bars; }
void ScreenAnnotator::draw_color_bars (Framebuffer &, const std::vector<std::string> &,
                                       std::vector<ColorMap> &)
{
  not_in_oracle ("ScreenAnnotator::draw_color_bars");
}
void ScreenAnnotator::draw_triad (Framebuffer &, Vec<float32, 2>, float32, Camera &)
{
  not_in_oracle ("ScreenAnnotator::draw_triad");
}

WorldAnnotator::WorldAnnotator (AABB<3> bounds) : m_bounds (bounds) {}
void WorldAnnotator::add_axes (const Camera &) { not_in_oracle ("WorldAnnotator::add_axes"); }
void WorldAnnotator::add_bounding_box () { not_in_oracle ("WorldAnnotator::add_bounding_box"); }
void WorldAnnotator::render (Framebuffer &, Array<Ray> &, const Camera &)
{
  not_in_oracle ("WorldAnnotator::render");
}
} // namespace dray
