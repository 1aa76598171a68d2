// Lineout sample points (Lineout::create_points, queries/lineout.cpp:98-140):
// samples + 2 points per line, from start to end inclusive, evenly spaced.
// The arithmetic is the reference's, with every operation rounded
// explicitly in its order (no contraction), so the points are bit-identical:
//   dir = end - start; step = |dir| / (samples + 1); dir /= |dir|;
//   point = start + (step * k) * dir.
// The values at the points come from point location and field evaluation
// (PointLocation::execute), as in the reference.
#include "drb_common.cuh"
#include "drb_internal.h"

namespace drb
{
namespace
{

__global__ void lineout_points_kernel (const float *__restrict__ starts, const float *__restrict__ ends,
                                       int n_lines, int per_line, float *__restrict__ points)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)n_lines * per_line) return;
  const int line = (int)(i / per_line);
  const int k = (int)(i - (long long)line * per_line);
  float a[3], d[3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
  {
    a[c] = starts[3 * (size_t)line + c];
    d[c] = __fsub_rn (ends[3 * (size_t)line + c], a[c]);
  }
  // Vec::magnitude: sum of squares in component order, then sqrtf
  float m2 = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) m2 = __fadd_rn (m2, __fmul_rn (d[c], d[c]));
  const float mag = __fsqrt_rn (m2);
  const float step = __fdiv_rn (mag, (float)(per_line - 1));
  const float s = __fmul_rn (step, (float)k);
#pragma unroll
  for (int c = 0; c < 3; ++c)
    points[3 * (size_t)i + c] = __fadd_rn (a[c], __fmul_rn (s, __fdiv_rn (d[c], mag)));
}

} // namespace
} // namespace drb

using namespace drb;

extern "C" int drb_lineout_points (const float *starts, const float *ends, int n_lines,
                                   int samples, float *points, void *stream)
{
  if (n_lines < 0 || samples < 1 || (n_lines > 0 && (!starts || !ends || !points)))
  {
    set_last_error ("lineout_points: needs samples >= 1 and start, end and point arrays");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_lines == 0) return DRB_OK;
  const int per_line = samples + 2;
  const long long total = (long long)n_lines * per_line;
  lineout_points_kernel<<<div_up (total, 256), 256, 0, (cudaStream_t)stream>>> (starts, ends, n_lines,
                                                                                 per_line, points);
  return check_launch ("lineout_points_kernel");
}
