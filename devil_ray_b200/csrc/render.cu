// Camera rays, ray culling, transfer functions, volume integration and
// compositing (the reference's rendering/ layer on the hot path).
//
//   camera_rays_kernel      Camera::gen_perspective (rendering/camera.cpp:402-483);
//                           host part of the set-up (set_fov, basis, deltas)
//                           in host float arithmetic, per-ray part with
//                           explicitly rounded ops: rays are bit-exact
//   cull_kernel + scan      mark_active / index_flags / gather / calc_ray_start
//                           (ray.cpp:102-241), stable compaction
//   volume_kernel           integrate_partials (rendering/volume.cpp:71-228):
//                           fixed-step march, locate per sample, <=5 segments,
//                           alpha cut 0.95, Blinn-Phong from the field gradient
//                           (rendering/volume_shader.hpp:40-167), front-to-back
//                           blend (rendering/colors.hpp:15-23).  Persistent
//                           warps pop rays from a global queue.  Optional
//                           coherent mode: a sample first tries the previous
//                           sample's element from the previous reference point,
//                           and falls back to the full BVH locate.
//   composite kernels       Volume::save / Framebuffer::composite_background
//                           (volume.cpp:369-416, framebuffer.cpp:126-162)
#include "bernstein.cuh"
#include "drb_common.cuh"
#include "drb_internal.h"
#include "locate.cuh"

#include <cmath>
#include <cstring>
#include <vector>

namespace drb
{

// ---------------------------------------------------------------- camera --

struct HostVec3
{
  float v[3];
};

static float h_mag (const float *a)
{
  float s = 0.f;
  for (int i = 0; i < 3; ++i) s += a[i] * a[i];
  return sqrtf (s);
}
static void h_normalize (float *a)
{
  const float m = h_mag (a);
  for (int i = 0; i < 3; ++i) a[i] /= m;
}
static void h_cross (const float *a, const float *b, float *r)
{
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

struct CamSetup
{
  float nlook[3], dx[3], dy[3], pos[3];
  int w, h;
};

// Camera::set_fov + create_rays_imp + the host part of gen_perspective.
static int camera_setup (const drb_camera *cam, CamSetup &cs)
{
  if (!cam || cam->width <= 0 || cam->height <= 0)
  {
    set_last_error ("camera: width and height must be > 0");
    return DRB_ERR_INVALID_ARG;
  }
  if (!(cam->fov_y > 0.f) || cam->fov_y > 180.f)
  {
    set_last_error ("camera: field of view must be in (0, 180]");
    return DRB_ERR_INVALID_ARG;
  }
  const float pi_f = (float)3.14159265358979323846264338327950288;
  // set_fov (camera.cpp:132-163)
  const float fov_y = cam->fov_y;
  const float fov_y_rad = (fov_y * pi_f) / 180.0f;
  const float vertical = tanf (0.5f * fov_y_rad);
  const float aspect = float (cam->width) / float (cam->height);
  const float horizontal = aspect * vertical;
  const float fov_x_rad = 2.0f * atanf (horizontal);
  const float fov_x = 180.0f * (fov_x_rad / pi_f);
  // set_up normalises the up vector (camera.cpp:172-176)
  float up[3] = { cam->up[0], cam->up[1], cam->up[2] };
  h_normalize (up);
  float look[3];
  for (int i = 0; i < 3; ++i) look[i] = cam->look_at[i] - cam->pos[i];
  // gen_perspective (camera.cpp:402-455)
  const float thx = tanf ((fov_x * pi_f / 180.f) * .5f);
  const float thy = tanf ((fov_y * pi_f / 180.f) * .5f);
  float ruf[3], ru[3], rvf[3], rv[3];
  h_cross (look, up, ruf);
  for (int i = 0; i < 3; ++i) ru[i] = ruf[i];
  h_normalize (ru);
  h_cross (ruf, look, rvf);
  for (int i = 0; i < 3; ++i) rv[i] = rvf[i];
  h_normalize (rv);
  const float sx = 2 * thx / (float)cam->width;
  const float sy = 2 * thy / (float)cam->height;
  const float zoom = cam->zoom > 0.f ? cam->zoom : 1.f;
  for (int i = 0; i < 3; ++i)
  {
    cs.dx[i] = ru[i] * sx;
    cs.dy[i] = rv[i] * sy;
    if (cam->zoom > 0.f)
    {
      cs.dx[i] = cs.dx[i] / zoom;
      cs.dy[i] = cs.dy[i] / zoom;
    }
    cs.nlook[i] = look[i];
    cs.pos[i] = cam->pos[i];
  }
  h_normalize (cs.nlook);
  cs.w = cam->width;
  cs.h = cam->height;
  return DRB_OK;
}

// Rotation of v about the unit-length-normalised axis by `degrees`
// (Rodrigues' formula as the 4x4 matrix of transform_3d.hpp:126-157,
// applied with a zero w: transform_3d.hpp:54-60).  Single precision in the
// reference's operation order, so camera moves match it bit for bit.
static void h_rotate (float degrees, const float *axis_in, float *v)
{
  const float pi_180 = 0.01745329251994329547437168059786927f;
  const float rad = pi_180 * degrees;
  float a[3] = { axis_in[0], axis_in[1], axis_in[2] };
  h_normalize (a);
  const float sn = sinf (rad);
  const float cs = cosf (rad);
  float m[3][4];
  m[0][0] = a[0] * a[0] * (1 - cs) + cs;
  m[0][1] = a[0] * a[1] * (1 - cs) - a[2] * sn;
  m[0][2] = a[0] * a[2] * (1 - cs) + a[1] * sn;
  m[1][0] = a[1] * a[0] * (1 - cs) + a[2] * sn;
  m[1][1] = a[1] * a[1] * (1 - cs) + cs;
  m[1][2] = a[1] * a[2] * (1 - cs) - a[0] * sn;
  m[2][0] = a[2] * a[0] * (1 - cs) - a[1] * sn;
  m[2][1] = a[2] * a[1] * (1 - cs) + a[0] * sn;
  m[2][2] = a[2] * a[2] * (1 - cs) + cs;
  m[0][3] = m[1][3] = m[2][3] = 0.f;
  const float hv[4] = { v[0], v[1], v[2], 0.f };
  for (int r = 0; r < 3; ++r)
  {
    float acc = 0.f;
    for (int c = 0; c < 4; ++c) acc += m[r][c] * hv[c];
    v[r] = acc;
  }
}

// Camera::elevate / azimuth (rendering/camera.cpp:516-555): turn the view
// direction about the camera's right (elevate, by -degrees) or up (azimuth)
// axis and put the camera back at the same distance from look_at.
static int camera_turn (drb_camera *cam, float degrees, bool about_right)
{
  if (!cam)
  {
    set_last_error ("camera: NULL camera");
    return DRB_ERR_INVALID_ARG;
  }
  float up[3] = { cam->up[0], cam->up[1], cam->up[2] };
  h_normalize (up); // the reference stores its up vector normalised
  float look[3];
  for (int i = 0; i < 3; ++i) look[i] = cam->look_at[i] - cam->pos[i];
  const float distance = h_mag (look);
  float right[3], vup[3];
  h_cross (look, up, right);
  h_cross (right, look, vup);
  h_normalize (look);
  h_normalize (right);
  h_normalize (vup);
  if (about_right) h_rotate (-degrees, right, look);
  else h_rotate (degrees, vup, look);
  for (int i = 0; i < 3; ++i) cam->pos[i] = cam->look_at[i] - look[i] * distance;
  return DRB_OK;
}

__global__ void camera_rays_kernel (CamSetup cs, Ray *__restrict__ rays)
{
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)cs.w * cs.h) return;
  const int i = (int)(idx % cs.w);
  const int j = (int)(idx / cs.w);
  // (2 i - w) / 2 and (2 j - w) / 2: the reference uses the width for both
  // (camera.cpp:469-470)
  const float si = __fdiv_rn (__fsub_rn (__fmul_rn (2.f, (float)i), (float)cs.w), 2.0f);
  const float sj = __fdiv_rn (__fsub_rn (__fmul_rn (2.f, (float)j), (float)cs.w), 2.0f);
  float d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    d[k] = __fadd_rn (__fadd_rn (cs.nlook[k], __fmul_rn (cs.dx[k], si)), __fmul_rn (cs.dy[k], sj));
    if (d[k] == 0.f) d[k] = __fadd_rn (d[k], 0.0000001f);
  }
  const float m2 = __fadd_rn (__fadd_rn (__fmul_rn (d[0], d[0]), __fmul_rn (d[1], d[1])),
                              __fmul_rn (d[2], d[2]));
  const float mag = __fsqrt_rn (m2);
  Ray r;
  r.dir = make3 (__fdiv_rn (d[0], mag), __fdiv_rn (d[1], mag), __fdiv_rn (d[2], mag));
  r.near_t = 0.f;
  r.orig = make3 (cs.pos[0], cs.pos[1], cs.pos[2]);
  r.far_t = INFINITY;
  r.pixel_id = j * cs.w + i;
  rays[idx] = r;
}

// ------------------------------------------------------------ ray culling --

struct CullBox
{
  float mn[3], mx[3];
};

// slab test of ray.cpp:132-176 / 190-235, explicit rounding
DRB_D bool slab (const Ray &r, const CullBox &b, float &tmin, float &tmax)
{
  const float inv[3] = { rcp_safe (r.dir.x), rcp_safe (r.dir.y), rcp_safe (r.dir.z) };
  const float o[3] = { r.orig.x, r.orig.y, r.orig.z };
  float lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    const float od = __fmul_rn (o[k], inv[k]);
    lo[k] = __fsub_rn (__fmul_rn (b.mn[k], inv[k]), od);
    hi[k] = __fsub_rn (__fmul_rn (b.mx[k], inv[k]), od);
  }
  float min_dist = fmaxf (fmaxf (fmaxf (fminf (lo[1], hi[1]), fminf (lo[0], hi[0])), fminf (lo[2], hi[2])), r.near_t);
  float max_dist = fminf (fminf (fmaxf (lo[1], hi[1]), fmaxf (lo[0], hi[0])), fmaxf (lo[2], hi[2]));
  max_dist = fminf (max_dist, r.far_t);
  tmin = min_dist;
  tmax = max_dist;
  return max_dist > min_dist;
}

__global__ void cull_flags_kernel (const Ray *__restrict__ rays, int n, CullBox b, int *__restrict__ flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float t0, t1;
  flags[i] = slab (rays[i], b, t0, t1) ? 1 : 0;
}

__global__ void cull_gather_kernel (const Ray *__restrict__ rays, int n, CullBox b,
                                    const int *__restrict__ flags, const int *__restrict__ offs,
                                    Ray *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  Ray r = rays[i];
  float t0, t1;
  slab (r, b, t0, t1);
  r.near_t = t0;
  r.far_t = t1;
  out[offs[i]] = r;
}

static CullBox cull_box (const float *bounds6)
{
  // AABB::scale(1.001f) about the centre (ray.cpp:120-121, range.hpp:162-172)
  CullBox b;
  const float s = 1.001f;
  for (int k = 0; k < 3; ++k)
  {
    float mn = bounds6[2 * k], mx = bounds6[2 * k + 1];
    if (!(mn > mx))
    {
      const float c = 0.5f * (mn + mx);
      const float delta = s * 0.5f * (mx - mn);
      mn = fminf (mn, c - delta);
      mx = fmaxf (mx, c + delta);
    }
    b.mn[k] = mn;
    b.mx[k] = mx;
  }
  return b;
}

// ---------------------------------------------------------- field range --

__global__ void range_kernel (const float *__restrict__ v, long long n, unsigned *__restrict__ ord)
{
  float mn = INFINITY, mx = -INFINITY;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
  {
    mn = fminf (mn, v[i]);
    mx = fmaxf (mx, v[i]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
  {
    mn = fminf (mn, __shfl_xor_sync (0xffffffffu, mn, o));
    mx = fmaxf (mx, __shfl_xor_sync (0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0 && mn <= mx)
  {
    atomicMin (ord, float_to_ordered (mn));
    atomicMax (ord + 1, float_to_ordered (mx));
  }
}

__global__ void range_init_kernel (unsigned *ord)
{
  ord[0] = float_to_ordered (INFINITY);
  ord[1] = float_to_ordered (-INFINITY);
}

__global__ void range_finish_kernel (const unsigned *ord, float *out)
{
  out[0] = ordered_to_float (ord[0]);
  out[1] = ordered_to_float (ord[1]);
}

// ------------------------------------------------------------- volume --

struct VolumeParams
{
  LocateParams lp;            // geometry + BVH + Newton options
  const float *field_packed;  // packed scalar rows (stride fstride) or NULL
  const int *field_idx;
  const float *field_vals;
  int fstride;
  const float4 *tf;           // transfer function (opacity corrected)
  int tf_size;
  float fmin, fmax, inv_range;
  const PointLight *lights;
  int n_lights;
  int use_lighting;
  int coherent;
  int quadratic_predictor;    // coherent mode 2: r_{k-1} + 2 J^-1 dx
  float sample_dist;
  int cull;
  CullBox box;
  const int *nbr;             // face neighbours (6 per element) or NULL
};

template <int P> struct FieldCP
{
  const float *__restrict__ row;
  DRB_D float operator() (int i, int) const { return __ldg (row + i); }
};
// Order-3 scalar rows: 4 values at 16-byte offsets, one float4 load.
template <> DRB_D void cp_row<3, 1, FieldCP<3>> (const FieldCP<3> &cp, int i0, float (&v)[4])
{
  const float4 a = __ldg (reinterpret_cast<const float4 *> (cp.row + i0));
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}

template <int P> struct FieldIndCP
{
  const int *__restrict__ idx;
  const float *__restrict__ val;
  DRB_D float operator() (int i, int) const { return __ldg (val + __ldg (idx + i)); }
};

// DeviceColorMap::color (device_color_map.hpp:61-78), linear scale
DRB_D float4 colormap (const VolumeParams &vp, float s)
{
  s = clampf (s, vp.fmin, vp.fmax);
  const float normalized = (s - vp.fmin) * vp.inv_range;
  int idx = (int)(normalized * float (vp.tf_size - 1));
  idx = min (max (idx, 0), vp.tf_size - 1);
  return __ldg (vp.tf + idx);
}

template <int P, int S = kTensor>
DRB_D void field_eval_d (const VolumeParams &vp, int el, const float (&r)[3], float &f, float (&g)[3])
{
  constexpr int ND = shape_dofs<S, P> ();
  float X[1], Ju[1], Jv[1], Jw[1];
  if (vp.field_packed)
  {
    FieldCP<P> cp{ vp.field_packed + (size_t)el * vp.fstride };
    if (S == kSimplex) tet_eval_d<P, 1> (cp, r[0], r[1], r[2], X, Ju, Jv, Jw);
    else hex_eval_d<P, 1> (cp, r[0], r[1], r[2], X, Ju, Jv, Jw);
  }
  else
  {
    FieldIndCP<P> cp{ vp.field_idx + (size_t)el * ND, vp.field_vals };
    if (S == kSimplex) tet_eval_d<P, 1> (cp, r[0], r[1], r[2], X, Ju, Jv, Jw);
    else hex_eval_d<P, 1> (cp, r[0], r[1], r[2], X, Ju, Jv, Jw);
  }
  f = X[0];
  g[0] = Ju[0];
  g[1] = Jv[0];
  g[2] = Jw[0];
}

// VolumeShader::color / shaded_color (volume_shader.hpp:40-167).  The
// geometry Jacobian is not evaluated again: lu is the factorised Jacobian of
// the located sample's last Newton step, taken within tol of ref, and the
// world position is the sample point itself (the solve's target).
template <int P, int S = kTensor>
DRB_D float4 shade_sample (const VolumeParams &vp, int el, const float (&r)[3], const Ray &ray,
                           const LU3 &lu, const float (&wpos)[3])
{
  float f, gref[3];
  field_eval_d<P, S> (vp, el, r, f, gref);
  const float4 c = colormap (vp, f);
  if (!vp.use_lighting) return c;
  float4 acc = make_float4 (0.f, 0.f, 0.f, 0.f);
  if (!(c.w > 0.01f)) return acc;
  // matrix_inverse via LUP (matrix.hpp:430-456); gradient = gref * J^-1
  float inv[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
  {
    float e[3] = { 0.f, 0.f, 0.f };
    e[c] = 1.f;
    float col[3];
    lu.solve (e, col);
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) inv[rr][c] = col[rr];
  }
  Vec3 g;
  g.x = gref[0] * inv[0][0] + gref[1] * inv[1][0] + gref[2] * inv[2][0];
  g.y = gref[0] * inv[0][1] + gref[1] * inv[1][1] + gref[2] * inv[2][1];
  g.z = gref[0] * inv[0][2] + gref[1] * inv[1][2] + gref[2] * inv[2][2];
  {
    const float m = sqrtf (dot (g, g));
    g = make3 (g.x / m, g.y / m, g.z / m);
  }
  const Vec3 view = make3 (-ray.dir.x, -ray.dir.y, -ray.dir.z);
  const Vec3 wp = make3 (wpos[0], wpos[1], wpos[2]);
  for (int l = 0; l < vp.n_lights; ++l)
  {
    const PointLight L = vp.lights[l];
    Vec3 ld = make3 (L.pos[0] - wp.x, L.pos[1] - wp.y, L.pos[2] - wp.z);
    {
      const float m = sqrtf (dot (ld, ld));
      ld = make3 (ld.x / m, ld.y / m, ld.z / m);
    }
    if (dot (ld, g) < 0.f) g = make3 (-g.x, -g.y, -g.z);
    const float diffuse = clampf (dot (ld, g), 0.f, 1.f);
    float sc[4] = { L.amb[0] * c.x, L.amb[1] * c.y, L.amb[2] * c.z, c.w };
    const float cc[3] = { c.x, c.y, c.z };
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] += diffuse * L.diff[k] * cc[k];
    Vec3 hv = 0.5f * (view + ld);
    {
      const float m = sqrtf (dot (hv, hv));
      hv = make3 (hv.x / m, hv.y / m, hv.z / m);
    }
    if (dot (g, hv) < 0.f) g = make3 (-g.x, -g.y, -g.z);
    const float doth = clampf (dot (g, hv), 0.f, 1.f);
    const float intensity = powf (doth, L.spec_pow);
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] += intensity * L.spec[k] * cc[k];
    acc.x = clampf (acc.x + sc[0], 0.f, 1.f);
    acc.y = clampf (acc.y + sc[1], 0.f, 1.f);
    acc.z = clampf (acc.z + sc[2], 0.f, 1.f);
    acc.w = acc.w + sc[3];
  }
  return acc;
}

DRB_D void blend (float4 &front, const float4 &back)
{
  const float alpha = back.w * (1.f - front.w);
  front.x = front.x + back.x * alpha;
  front.y = front.y + back.y * alpha;
  front.z = front.z + back.z * alpha;
  front.w = alpha + front.w;
}

// A predicted reference point outside the previous element means the sample
// has left it.  With a face table the march steps across the exit face at
// once (margin 0: the face walk comes back if the prediction was off);
// without one, whose next stop is the BVH, a prediction within this margin
// is solved in the previous element first.
constexpr float kCoherentMargin = 0.1f;

// Face by which a reference point outside [0,1]^3 leaves the element (the
// axis with the largest excursion; faces u0, u1, v0, v1, w0, w1), -1 inside.
// Tets: the most negative of u, v, w and 1 - u - v - w (faces u=0, v=0,
// w=0, u+v+w=1).
template <int S = kTensor>
DRB_D int exit_face (const float (&x)[3])
{
  if (S == kSimplex)
  {
    int f = -1;
    float worst = 0.f;
    const float t = 1.f - (x[0] + x[1] + x[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      if (-x[d] > worst)
      {
        worst = -x[d];
        f = d;
      }
    }
    if (-t > worst) f = 3;
    return f;
  }
  int f = -1;
  float worst = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    if (-x[d] > worst)
    {
      worst = -x[d];
      f = 2 * d;
    }
    if (x[d] - 1.f > worst)
    {
      worst = x[d] - 1.f;
      f = 2 * d + 1;
    }
  }
  return f;
}

// The element across face f, and the guess carried over into its frame
// (hexes: the structured-lattice case, the same axes shifted by one; tets,
// whose neighbours' frames are unrelated: the neighbour's centroid).
template <int S = kTensor>
DRB_D int step_across (const VolumeParams &vp, int el, int f, float (&x)[3])
{
  if (f < 0 || !vp.nbr) return -1;
  if (S == kSimplex)
  {
    const int nb = __ldg (vp.nbr + 4 * (size_t)el + f);
    if (nb >= 0) x[0] = x[1] = x[2] = 0.25f;
    return nb;
  }
  const int nb = __ldg (vp.nbr + 6 * (size_t)el + f);
  if (nb >= 0) x[f >> 1] += (f & 1) ? -1.f : 1.f;
  return nb;
}

// Locate one sample.  Coherent mode first tries the previous sample's
// element, starting from a predictor step r_prev + J^-1 (pt - pt_prev) with
// the previous solve's Jacobian (lu), so that the solve usually converges in
// two steps.  When the prediction (or that solve) leaves the element, the
// element across the exit face is tried (face-neighbour table), and from its
// solve the next one, up to face_steps<S>() elements (a ray passing near an
// edge or a corner of a hex crosses two or three faces between samples; the
// six tets of a cube are thinner).  Tets take the neighbour's centroid as
// the first guess.  Then, or in plain mode, the BVH candidates in the
// reference's order; the same acceptance rule throughout.  All candidates
// go through one Newton call site, which keeps the kernel's code small.  On
// success lu holds the located solve's Jacobian.
template <int S> constexpr int face_steps () { return S == kSimplex ? 6 : 3; }
template <int P, bool WIDE, int S = kTensor>
DRB_D int locate_sample (const VolumeParams &vp, const float (&pt)[3], const float (&step)[3],
                         int prev_el, const float (&prev_ref)[3], bool prev2_ok,
                         const float (&prev2_ref)[3], LU3 &lu, float (&ref)[3], int &iters,
                         int &cands, int &nodes)
{
  int todo[TraversalStack<WIDE>::kDepth];
  int sp = 0, cur = 0;
  todo[0] = kBarrier;
  int el = -1, leaf = -1;
  int crossed = 0; // face steps taken by this sample
  float x[3];
  if (vp.coherent && prev_el >= 0)
  {
    // predictor along the ray: r + J^-1 dx from the previous sample's
    // factorised Jacobian, or, when the two previous samples lie in the same
    // element, r_{k-1} + 2 J_k^-1 dx, which is exact where the reference
    // point moves quadratically in the ray parameter
    float dr[3];
    lu.solve (step, dr);
    if (prev2_ok)
    {
      x[0] = prev2_ref[0] + 2.f * dr[0];
      x[1] = prev2_ref[1] + 2.f * dr[1];
      x[2] = prev2_ref[2] + 2.f * dr[2];
    }
    else
    {
      x[0] = prev_ref[0] + dr[0];
      x[1] = prev_ref[1] + dr[1];
      x[2] = prev_ref[2] + dr[2];
    }
    const float margin = vp.nbr ? 0.f : kCoherentMargin;
    if (S == kSimplex ? is_inside_simplex (x, margin) : is_inside_ref (x, margin))
    {
      el = prev_el;
    }
    else
    {
      el = step_across<S> (vp, prev_el, exit_face<S> (x), x);
      crossed = 1;
    }
  }
  while (true)
  {
    if (el < 0)
    {
      leaf = next_leaf<WIDE> (vp.lp.nodes, vp.lp.wide, pt, todo, sp, cur, nodes);
      if (leaf < 0) return -1;
      el = __ldg (vp.lp.leaf_nodes + leaf);
      bool given;
      candidate_guess<S> (vp.lp, leaf, 0, false, pt, x, given);
    }
    int steps = 0;
    ++cands;
    // order 2 and 3 rows are read through L1: keeping 81+ values in
    // registers would halve the resident warps of this kernel
    const bool found = solve_in_element<P, (P == 1), S> (vp.lp, el, pt, x, steps, lu);
    iters += steps;
    if (found)
    {
      ref[0] = x[0];
      ref[1] = x[1];
      ref[2] = x[2];
      return el;
    }
    if (leaf < 0 && crossed < face_steps<S> ())
    {
      // the solve ended outside its element: step across its exit face
      ++crossed;
      el = step_across<S> (vp, el, exit_face<S> (x), x);
      if (el >= 0) continue;
    }
    el = -1;
    if (leaf >= 0)
    {
      cur = todo[sp];
      --sp;
    }
  }
}

// One ray's march (integrate_partials, volume.cpp:71-228) as a state that
// advances one sample at a time, so a lane whose ray ends takes the next
// ray at once instead of idling until the warp's longest ray ends.
struct RayMarch
{
  Ray ray;
  int i;              // ray index, -1: lane idle
  float distance;     // position of the next sample
  int segment;        // partials written so far (at most 5)
  bool in_seg;        // inside a run of located samples
  float seg_depth;
  float4 color;       // the current segment's blend
  float4 pixel;       // partials composited front to back (Volume::save)
  float first_depth;
  int prev_el;
  float prev_ref[3];
  bool prev2_ok;      // the sample before prev was in prev_el too
  float prev2_ref[3];
  int n_samples, iters, cands, nodes;
};

// End of a run of located samples: write the partial and composite it
// behind the earlier ones (Volume::save order).
DRB_D void end_segment (RayMarch &s, VolumePartial *__restrict__ partials)
{
  constexpr int kMaxSegments = 5;
  if (partials)
  {
    VolumePartial part;
    part.pixel_id = s.ray.pixel_id;
    part.depth = s.seg_depth;
    part.color[0] = s.color.x;
    part.color[1] = s.color.y;
    part.color[2] = s.color.z;
    part.color[3] = s.color.w;
    partials[(size_t)kMaxSegments * s.i + s.segment] = part;
  }
  if (s.segment == 0)
  {
    s.pixel = s.color;
    s.first_depth = s.seg_depth;
  }
  else
  {
    const float a = 1.f - s.pixel.w;
    s.pixel.x = s.pixel.x + s.color.x * a;
    s.pixel.y = s.pixel.y + s.color.y * a;
    s.pixel.z = s.pixel.z + s.color.z * a;
    s.pixel.w = s.pixel.w + s.color.w * a;
  }
  ++s.segment;
  s.in_seg = false;
}

DRB_D void finish_ray (RayMarch &s, float4 *__restrict__ fb_color, float *__restrict__ fb_depth,
                       int *__restrict__ ray_samples, int *__restrict__ ray_iters,
                       int *__restrict__ ray_cands)
{
  if (fb_color && s.segment > 0)
  {
    fb_color[s.ray.pixel_id] = s.pixel;
    if (fb_depth) fb_depth[s.ray.pixel_id] = s.first_depth;
  }
  if (ray_samples) ray_samples[s.i] = s.n_samples;
  if (ray_iters) ray_iters[s.i] = s.iters;
  if (ray_cands) ray_cands[s.i] = s.cands;
  s.i = -1;
}

// Persistent march: warps pop chunks of rays from a global queue and keep
// every lane on a ray (ballot refill, as the batched locate does with
// queries).  Each loop iteration advances every busy lane by one sample:
// locate (coherent or full), shade, blend, and the segment and ray
// termination rules of integrate_partials: a segment ends at the first
// sample not located, at the ray's far distance or when its alpha reaches
// 0.95; the ray ends after 5 segments, at far, or when alpha exceeds 0.95.
// Partials go to slot 5 i + segment of ray i and the framebuffer pixel gets
// their front-to-back composite, so the processing order changes nothing.
template <int P, bool WIDE, int S>
__global__ void __launch_bounds__ (128)
volume_kernel (VolumeParams vp, const Ray *__restrict__ rays, int n_rays, int *__restrict__ queue,
               VolumePartial *__restrict__ partials, float4 *__restrict__ fb_color,
               float *__restrict__ fb_depth, int *__restrict__ ray_samples,
               int *__restrict__ ray_iters, int *__restrict__ ray_cands)
{
  constexpr int kMaxSegments = 5; // volume.cpp:110
  constexpr int kChunk = 32;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int pool_next = 0, pool_end = 0; // warp-uniform
  bool exhausted = false;          // warp-uniform
  RayMarch s;
  s.i = -1;
  LU3 lu;
  float step[3] = { 0.f, 0.f, 0.f };
  while (true)
  {
    // ---- give idle lanes the next rays of the warp's chunk ----
    unsigned need = __ballot_sync (FULL, s.i < 0);
    while (need != 0u && !exhausted)
    {
      if (pool_next >= pool_end)
      {
        int base = 0;
        if (lane == 0) base = atomicAdd (queue, kChunk);
        base = __shfl_sync (FULL, base, 0);
        if (base >= n_rays)
        {
          exhausted = true;
          break;
        }
        pool_next = base;
        pool_end = min (base + kChunk, n_rays);
      }
      const int avail = pool_end - pool_next;
      const int rank = __popc (need & lt);
      if (s.i < 0 && rank < avail)
      {
        s.i = pool_next + rank;
        s.ray = rays[s.i];
        bool live = true;
        if (vp.cull)
        {
          // mark_active + calc_ray_start (ray.cpp:117-241) on the raw ray
          float t0, t1;
          live = slab (s.ray, vp.box, t0, t1);
          s.ray.near_t = t0;
          s.ray.far_t = t1;
        }
        s.distance = s.ray.near_t + vp.sample_dist;
        s.segment = 0;
        s.in_seg = false;
        s.color = make_float4 (0.f, 0.f, 0.f, 0.f);
        s.pixel = make_float4 (0.f, 0.f, 0.f, 0.f);
        s.first_depth = INFINITY;
        s.seg_depth = 0.f;
        s.prev_el = -1;
        s.prev_ref[0] = s.prev_ref[1] = s.prev_ref[2] = 0.5f;
        s.prev2_ok = false;
        s.prev2_ref[0] = s.prev2_ref[1] = s.prev2_ref[2] = 0.5f;
        s.n_samples = s.iters = s.cands = s.nodes = 0;
        step[0] = s.ray.dir.x * vp.sample_dist;
        step[1] = s.ray.dir.y * vp.sample_dist;
        step[2] = s.ray.dir.z * vp.sample_dist;
        if (!live || !(s.distance < s.ray.far_t))
          finish_ray (s, fb_color, fb_depth, ray_samples, ray_iters, ray_cands);
      }
      pool_next += min (__popc (need), avail);
      need = __ballot_sync (FULL, s.i < 0);
    }
    if (__ballot_sync (FULL, s.i >= 0) == 0u) break;
    if (s.i < 0) continue;

    // ---- one sample of this lane's ray ----
    const float pt[3] = { s.ray.orig.x + s.distance * s.ray.dir.x,
                          s.ray.orig.y + s.distance * s.ray.dir.y,
                          s.ray.orig.z + s.distance * s.ray.dir.z };
    float ref[3];
    const int el = locate_sample<P, WIDE, S> (vp, pt, step, s.prev_el, s.prev_ref, s.prev2_ok,
                                              s.prev2_ref, lu, ref, s.iters, s.cands, s.nodes);
    bool done = false;
    if (el >= 0)
    {
      if (!s.in_seg)
      {
        s.in_seg = true;
        s.seg_depth = s.distance;
        s.color = make_float4 (0.f, 0.f, 0.f, 0.f);
      }
      ++s.n_samples;
      const float4 sc = shade_sample<P, S> (vp, el, ref, s.ray, lu, pt);
      blend (s.color, sc);
      s.prev2_ok = vp.quadratic_predictor && el == s.prev_el;
      s.prev2_ref[0] = s.prev_ref[0];
      s.prev2_ref[1] = s.prev_ref[1];
      s.prev2_ref[2] = s.prev_ref[2];
      s.prev_el = el;
      s.prev_ref[0] = ref[0];
      s.prev_ref[1] = ref[1];
      s.prev_ref[2] = ref[2];
      s.distance += vp.sample_dist;
      if (!(s.distance < s.ray.far_t) || !(s.color.w < 0.95f))
      {
        const float alpha = s.color.w;
        end_segment (s, partials);
        done = !(s.distance < s.ray.far_t) || alpha > 0.95f || s.segment == kMaxSegments;
      }
    }
    else
    {
      s.prev_el = -1;
      s.prev2_ok = false;
      if (s.in_seg)
      {
        end_segment (s, partials);
        done = s.segment == kMaxSegments;
      }
      s.distance += vp.sample_dist;
      if (!(s.distance < s.ray.far_t)) done = true;
    }
    if (done) finish_ray (s, fb_color, fb_depth, ray_samples, ray_iters, ray_cands);
  }
}

__global__ void init_partials_kernel (VolumePartial *p, long long n)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  VolumePartial v;
  v.pixel_id = -1;
  v.depth = INFINITY;
  v.color[0] = v.color[1] = v.color[2] = v.color[3] = 0.f;
  p[i] = v;
}

__global__ void partial_flags_kernel (const VolumePartial *p, int n, int *flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flags[i] = (p[i].depth == INFINITY) ? 0 : 1;
}

__global__ void partial_gather_kernel (const VolumePartial *p, int n, const int *flags,
                                       const int *offs, VolumePartial *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flags[i]) out[offs[i]] = p[i];
}

// Volume::save compositing over partials sorted by pixel then depth
__global__ void composite_partials_kernel (const VolumePartial *p, int n, float4 *fb)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pix = p[i].pixel_id;
  if (i > 0 && p[i - 1].pixel_id == pix) return; // not the first of its run
  float4 c = make_float4 (p[i].color[0], p[i].color[1], p[i].color[2], p[i].color[3]);
  for (int k = i + 1; k < n && p[k].pixel_id == pix; ++k)
  {
    const float a = 1.f - c.w;
    c.x = c.x + p[k].color[0] * a;
    c.y = c.y + p[k].color[1] * a;
    c.z = c.z + p[k].color[2] * a;
    c.w = c.w + p[k].color[3] * a;
  }
  fb[pix] = c;
}

// partials_to_framebuffer (rendering/renderer.cpp:98-139) after the
// per-pixel composite of partials sorted by pixel then depth; with blend the
// volume is composited in front of what the framebuffer holds (surfaces).
__global__ void partials_to_fb_kernel (const VolumePartial *p, int n, float4 *fb, float *depth,
                                       int blend_over)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pix = p[i].pixel_id;
  if (i > 0 && p[i - 1].pixel_id == pix) return;
  float4 c = make_float4 (p[i].color[0], p[i].color[1], p[i].color[2], p[i].color[3]);
  for (int k = i + 1; k < n && p[k].pixel_id == pix; ++k)
  {
    const float a = 1.f - c.w;
    c.x = c.x + p[k].color[0] * a;
    c.y = c.y + p[k].color[1] * a;
    c.z = c.z + p[k].color[2] * a;
    c.w = c.w + p[k].color[3] * a;
  }
  if (blend_over)
  {
    const float4 f = fb[pix];
    const float op = 1.f - c.w;
    c = make_float4 (c.x + op * f.x, c.y + op * f.y, c.z + op * f.z, c.w + op * f.w);
  }
  fb[pix] = c;
  if (depth) depth[pix] = p[i].depth;
}

__global__ void fb_clear_kernel (float4 *c, float *d, int n, float4 v)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  c[i] = v;
  if (d) d[i] = INFINITY;
}

__global__ void fb_background_kernel (float4 *c, int n, float4 bg)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = c[i];
  if (v.w < 1.f)
  {
    // blend_pre_alpha (colors.hpp:25-33)
    const float a = 1.f - v.w;
    v.x = v.x + bg.x * a;
    v.y = v.y + bg.y * a;
    v.z = v.z + bg.z * a;
    v.w = v.w + bg.w * a;
    c[i] = v;
  }
}

template <int P, bool WIDE, int S>
int launch_volume_w (const VolumeParams &vp, const Ray *rays, int n, int *queue,
                     VolumePartial *partials, float4 *fb, float *depth, const drb_ray_stats &st,
                     cudaStream_t s)
{
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor (&nb, volume_kernel<P, WIDE, S>, 128, 0);
  if (nb < 1) nb = 1;
  long long blocks = (long long)nb * sm_count ();
  const long long need = ((long long)n + 127) / 128;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  volume_kernel<P, WIDE, S><<<(unsigned)blocks, 128, 0, s>>> (vp, rays, n, queue, partials, fb, depth,
                                                              st.samples, st.iters, st.candidates);
  return check_launch ("volume_kernel");
}

// full locates of the march walk the 4-wide tree when the BVH has one
template <int P, int S>
int launch_volume_s (const VolumeParams &vp, const Ray *rays, int n, int *queue,
                     VolumePartial *partials, float4 *fb, float *depth, const drb_ray_stats &st,
                     cudaStream_t s)
{
  if (vp.lp.wide) return launch_volume_w<P, true, S> (vp, rays, n, queue, partials, fb, depth, st, s);
  return launch_volume_w<P, false, S> (vp, rays, n, queue, partials, fb, depth, st, s);
}

int launch_volume (const drb_mesh *mesh, const VolumeParams &vp, const Ray *rays, int n,
                   int *queue, VolumePartial *partials, float4 *fb, float *depth,
                   const drb_ray_stats &st, cudaStream_t s)
{
#define DRB_LV(P, S) launch_volume_s<P, S> (vp, rays, n, queue, partials, fb, depth, st, s)
  if (mesh->shape == DRB_SHAPE_SIMPLEX)
    return mesh->order == 1 ? DRB_LV (1, kSimplex) : mesh->order == 2 ? DRB_LV (2, kSimplex) : DRB_LV (3, kSimplex);
  return mesh->order == 1 ? DRB_LV (1, kTensor) : mesh->order == 2 ? DRB_LV (2, kTensor) : DRB_LV (3, kTensor);
#undef DRB_LV
}

} // namespace drb

using namespace drb;

// ------------------------------------------------------------- C-ABI --

extern "C" int drb_camera_rays (const drb_camera *cam, void *rays, void *stream)
{
  CamSetup cs;
  int st = camera_setup (cam, cs);
  if (st) return st;
  if (!rays)
  {
    set_last_error ("camera_rays: rays is NULL");
    return DRB_ERR_INVALID_ARG;
  }
  const long long n = (long long)cs.w * cs.h;
  camera_rays_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (cs, (Ray *)rays);
  return check_launch ("camera_rays_kernel");
}

// detail::default_light (rendering/renderer.cpp:141-159): a point light
// above the camera; host float arithmetic.  light13 = pos3, amb3, diff3,
// spec3, spec_pow with the PointLight defaults (rendering/point_light.hpp).
extern "C" int drb_default_light (const drb_camera *cam, float *light13)
{
  if (!cam || !light13)
  {
    set_last_error ("default_light: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  float up[3] = { cam->up[0], cam->up[1], cam->up[2] };
  h_normalize (up); // Camera::set_up
  h_normalize (up); // default_light normalises again
  float look[3];
  for (int i = 0; i < 3; ++i) look[i] = cam->look_at[i] - cam->pos[i];
  const float mag = h_mag (look);
  float right[3], mup[3];
  h_cross (look, up, right);
  h_normalize (right);
  h_cross (right, look, mup);
  h_normalize (mup);
  for (int i = 0; i < 3; ++i) light13[i] = cam->pos[i] + .1f * mag * mup[i];
  const float amb = 0.4f, diff = 0.75f, spec = 0.8f;
  for (int i = 0; i < 3; ++i)
  {
    light13[3 + i] = amb;
    light13[6 + i] = diff;
    light13[9 + i] = spec;
  }
  light13[12] = 15.f;
  return DRB_OK;
}

extern "C" int drb_cull_rays (const void *rays, int n, const float *bounds6, void *active_rays,
                              int *n_active, void *stream)
{
  if (n < 0 || (n > 0 && (!rays || !bounds6 || !active_rays || !n_active)))
  {
    set_last_error ("cull_rays: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0)
  {
    *n_active = 0;
    return DRB_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const CullBox b = cull_box (bounds6);
  Scratch scr (s);
  int *flags = scr.alloc<int> (n);
  int *offs = scr.alloc<int> (n);
  int *total = scr.alloc<int> (1);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  cull_flags_kernel<<<div_up (n, 256), 256, 0, s>>> ((const Ray *)rays, n, b, flags);
  int st = check_launch ("cull_flags_kernel");
  if (st) return st;
  st = exclusive_scan_i32 (flags, offs, n, total, s);
  if (st) return st;
  cull_gather_kernel<<<div_up (n, 256), 256, 0, s>>> ((const Ray *)rays, n, b, flags, offs, (Ray *)active_rays);
  st = check_launch ("cull_gather_kernel");
  if (st) return st;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync (&h, total, sizeof (int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  if (e != cudaSuccess) return status_from (e);
  *n_active = h;
  return DRB_OK;
}

extern "C" int drb_field_range (const drb_mesh *field, float *range2, void *stream)
{
  if (!field || !range2 || field->ncomp != 1 || field->n_ctrl < 0 || (field->n_ctrl > 0 && !field->values))
  {
    set_last_error ("field_range: needs a scalar field");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  unsigned *ord = scr.alloc<unsigned> (2);
  if (!ord) return status_from (scr.err);
  range_init_kernel<<<1, 1, 0, s>>> (ord);
  int st = check_launch ("range_init_kernel");
  if (st) return st;
  if (field->n_ctrl > 0)
  {
    const int blocks = min (div_up (field->n_ctrl, 256), sm_count () * 8);
    range_kernel<<<blocks, 256, 0, s>>> (field->values, field->n_ctrl, ord);
    if ((st = check_launch ("range_kernel"))) return st;
  }
  range_finish_kernel<<<1, 1, 0, s>>> (ord, range2);
  return check_launch ("range_finish_kernel");
}

// ColorTable::sample with correct_opacity (color_table.cpp:152-323): host.
extern "C" int drb_color_table_sample (int n_rgb, const float *rgb_pts, int n_alpha,
                                       const float *alpha_pts, int smooth, int n_samples,
                                       float alpha_scale, float opacity_factor, float *rgba)
{
  if (n_samples < 1 || !rgba || n_rgb < 0 || n_alpha < 0 || (n_rgb > 0 && !rgb_pts) ||
      (n_alpha > 0 && !alpha_pts))
  {
    set_last_error ("color_table_sample: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  std::vector<float> apos (n_alpha), aval (n_alpha);
  for (int i = 0; i < n_alpha; ++i)
  {
    apos[i] = alpha_pts[2 * i];
    aval[i] = alpha_pts[2 * i + 1];
    if (opacity_factor > 0.f) aval[i] = 1.f - powf ((1.f - aval[i]), opacity_factor);
  }
  for (int i = 0; i < n_samples; ++i)
  {
    const float scalar = n_samples > 1 ? static_cast<float> (i) / static_cast<float> (n_samples - 1) : 0.f;
    float c[4] = { 0.5f, 0.5f, 0.5f, 1.f };
    // map_rgb
    if (n_rgb > 0)
    {
      if (n_rgb == 1 || scalar <= rgb_pts[0])
      {
        for (int k = 0; k < 3; ++k) c[k] = rgb_pts[1 + k];
        c[3] = 1.f;
      }
      else if (scalar >= rgb_pts[4 * (n_rgb - 1)])
      {
        for (int k = 0; k < 3; ++k) c[k] = rgb_pts[4 * (n_rgb - 1) + 1 + k];
        c[3] = 1.f;
      }
      else
      {
        int second;
        for (second = 1; second < n_rgb - 1; ++second)
          if (scalar < rgb_pts[4 * second]) break;
        const int first = second - 1;
        const float seg = rgb_pts[4 * second] - rgb_pts[4 * first];
        const float alpha = (seg == 0.f) ? .5f : (scalar - rgb_pts[4 * first]) / seg;
        for (int k = 0; k < 3; ++k)
        {
          const float a = rgb_pts[4 * first + 1 + k], b = rgb_pts[4 * second + 1 + k];
          c[k] = smooth ? (a * (1.0f - alpha) + b * alpha) : (alpha < .5 ? a : b);
        }
        c[3] = smooth ? (1.f * (1.0f - alpha) + 1.f * alpha) : 1.f;
      }
    }
    // map_alpha
    float av = 1.f;
    if (n_alpha > 0)
    {
      if (n_alpha == 1 || scalar <= apos[0]) av = aval[0];
      else if (scalar >= apos[n_alpha - 1]) av = aval[n_alpha - 1];
      else
      {
        int second;
        for (second = 1; second < n_alpha - 1; ++second)
          if (scalar < apos[second]) break;
        const int first = second - 1;
        const float seg = apos[second] - apos[first];
        const float alpha = (seg == 0.f) ? .5f : (scalar - apos[first]) / seg;
        av = smooth ? (aval[first] * (1.f - alpha) + aval[second] * alpha)
                    : (alpha < .5 ? aval[first] : aval[second]);
      }
    }
    c[3] = av * alpha_scale;
    for (int k = 0; k < 4; ++k) rgba[4 * i + k] = c[k];
  }
  return DRB_OK;
}

static int volume_common (const drb_mesh *mesh, const drb_mesh *field, const drb_bvh *bvh,
                          const void *active_rays, int n_rays, const drb_volume_opts *o,
                          const float *tf, int tf_size, const float *range2,
                          const void *lights, int n_lights, VolumeParams &vp)
{
  if (!mesh || !field || !bvh || !o || n_rays < 0 || (n_rays > 0 && !active_rays) || !tf ||
      tf_size < 1 || !range2 || n_lights < 0 || (n_lights > 0 && !lights))
  {
    set_last_error ("volume: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (mesh->dim != 3 || mesh->ncomp != 3 || field->dim != 3 || field->ncomp != 1 ||
      mesh->order != field->order || mesh->n_elem != field->n_elem || mesh->order < 1 ||
      mesh->order > 3 || mesh->shape != field->shape ||
      (mesh->shape != DRB_SHAPE_TENSOR && mesh->shape != DRB_SHAPE_SIMPLEX))
  {
    set_last_error ("volume: needs a hex (or tet) mesh and a scalar field of the same shape and "
                    "order 1..3");
    return DRB_ERR_UNSUPPORTED;
  }
  if (o->samples < 1 || !(o->tol > 0.f) || o->max_steps < 0)
  {
    set_last_error ("volume: samples >= 1, tol > 0, max_steps >= 0 required");
    return DRB_ERR_INVALID_ARG;
  }
  drb_newton_opts no;
  no.tol = o->tol;
  no.max_steps = o->max_steps;
  no.guess_mode = o->guess_mode == DRB_GUESS_GIVEN ? DRB_GUESS_ELEM_CENTER : o->guess_mode;
  no.guess = nullptr;
  LocateParams &lp = vp.lp;
  lp.nodes = (const float4 *)bvh->inner_nodes;
  lp.wide = (const float4 *)bvh->wide_nodes;
  lp.leaf_nodes = bvh->leaf_nodes;
  lp.aabb_ids = bvh->aabb_ids;
  lp.ref_boxes = bvh->ref_boxes;
  lp.packed = mesh->packed;
  lp.ctrl_idx = mesh->ctrl_idx;
  lp.xyz = mesh->values;
  const int nd = mesh_nd (mesh);
  lp.stride = packed_stride (nd, 3);
  lp.tol = no.tol;
  lp.max_steps = no.max_steps;
  lp.guess_mode = no.guess_mode;
  lp.guess = nullptr;
  lp.leaf_maps = mesh->dim == 3 ? (const float4 *)bvh->leaf_maps : nullptr;
  vp.field_packed = field->packed;
  vp.field_idx = field->ctrl_idx;
  vp.field_vals = field->values;
  vp.fstride = packed_stride (nd, 1);
  vp.nbr = mesh->face_neighbors;
  vp.tf = (const float4 *)tf;
  vp.tf_size = tf_size;
  // DeviceColorMap: range of the field's control values, rcp_safe(length)
  vp.fmin = range2[0];
  vp.fmax = range2[1];
  {
    float len = vp.fmax - vp.fmin;
    float g = (fabsf (len) < 1e-8f) ? (std::signbit (len) ? -1e-8f : 1e-8f) : len;
    vp.inv_range = 1.0f / g;
  }
  vp.lights = (const PointLight *)lights;
  vp.n_lights = n_lights;
  vp.use_lighting = o->use_lighting;
  vp.coherent = o->coherent != 0;
  vp.quadratic_predictor = o->coherent == 2;
  vp.cull = o->cull;
  vp.box = cull_box (bvh->bounds);
  // sample distance: |bounds diagonal| / samples (volume.cpp:89-91)
  const float *b = o->bounds;
  float dd[3] = { b[1] - b[0], b[3] - b[2], b[5] - b[4] };
  const float mag = h_mag (dd);
  vp.sample_dist = mag / float (o->samples);
  return DRB_OK;
}

extern "C" int drb_volume_integrate (const drb_mesh *mesh, const drb_mesh *field,
                                     const drb_bvh *bvh, const void *active_rays, int n_rays,
                                     const drb_volume_opts *opts, const float *tf, int tf_size,
                                     const float *range2, const void *lights, int n_lights,
                                     void *partials, int *n_partials, drb_ray_stats stats,
                                     void *stream)
{
  VolumeParams vp;
  int st = volume_common (mesh, field, bvh, active_rays, n_rays, opts, tf, tf_size, range2,
                          lights, n_lights, vp);
  if (st) return st;
  if (!partials || !n_partials)
  {
    set_last_error ("volume_integrate: partials and n_partials are required");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_rays == 0)
  {
    *n_partials = 0;
    return DRB_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long long np = 5ll * n_rays;
  if (np >= (1ll << 31))
  {
    set_last_error ("volume_integrate: too many rays for int32 partial indices");
    return DRB_ERR_INVALID_ARG;
  }
  Scratch scr (s);
  VolumePartial *raw = scr.alloc<VolumePartial> (np);
  int *flags = scr.alloc<int> (np);
  int *offs = scr.alloc<int> (np);
  int *total = scr.alloc<int> (1);
  int *queue = scr.alloc<int> (1);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  init_partials_kernel<<<div_up (np, 256), 256, 0, s>>> (raw, np);
  if ((st = check_launch ("init_partials_kernel"))) return st;
  cudaMemsetAsync (queue, 0, sizeof (int), s);
  const Ray *rays = (const Ray *)active_rays;
  st = launch_volume (mesh, vp, rays, n_rays, queue, raw, nullptr, nullptr, stats, s);
  if (st) return st;
  // compact_partials (volume.cpp:42-67)
  partial_flags_kernel<<<div_up (np, 256), 256, 0, s>>> (raw, (int)np, flags);
  if ((st = check_launch ("partial_flags_kernel"))) return st;
  if ((st = exclusive_scan_i32 (flags, offs, (int)np, total, s))) return st;
  partial_gather_kernel<<<div_up (np, 256), 256, 0, s>>> (raw, (int)np, flags, offs, (VolumePartial *)partials);
  if ((st = check_launch ("partial_gather_kernel"))) return st;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync (&h, total, sizeof (int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  if (e != cudaSuccess) return status_from (e);
  *n_partials = h;
  return DRB_OK;
}

extern "C" int drb_volume_render (const drb_mesh *mesh, const drb_mesh *field, const drb_bvh *bvh,
                                  const void *active_rays, int n_rays,
                                  const drb_volume_opts *opts, const float *tf, int tf_size,
                                  const float *range2, const void *lights, int n_lights,
                                  float *fb_rgba, float *fb_depth, drb_ray_stats stats,
                                  void *stream)
{
  VolumeParams vp;
  int st = volume_common (mesh, field, bvh, active_rays, n_rays, opts, tf, tf_size, range2,
                          lights, n_lights, vp);
  if (st) return st;
  if (!fb_rgba)
  {
    set_last_error ("volume_render: fb_rgba is required");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_rays == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  int *queue = scr.alloc<int> (1);
  if (!queue) return status_from (scr.err);
  cudaMemsetAsync (queue, 0, sizeof (int), s);
  const Ray *rays = (const Ray *)active_rays;
  float4 *fb = (float4 *)fb_rgba;
  st = launch_volume (mesh, vp, rays, n_rays, queue, nullptr, fb, fb_depth, stats, s);
  return st;
}

extern "C" int drb_composite_partials (const void *partials, int n, float *fb_rgba, void *stream)
{
  if (n < 0 || (n > 0 && (!partials || !fb_rgba)))
  {
    set_last_error ("composite_partials: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  composite_partials_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (
  (const VolumePartial *)partials, n, (float4 *)fb_rgba);
  return check_launch ("composite_partials_kernel");
}

extern "C" int drb_framebuffer_clear (float *rgba, float *depth, int n_pixels, const float *color4,
                                      void *stream)
{
  if (n_pixels < 0 || (n_pixels > 0 && !rgba))
  {
    set_last_error ("framebuffer_clear: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_pixels == 0) return DRB_OK;
  const float4 c = color4 ? make_float4 (color4[0], color4[1], color4[2], color4[3])
                          : make_float4 (0.f, 0.f, 0.f, 0.f);
  fb_clear_kernel<<<div_up (n_pixels, 256), 256, 0, (cudaStream_t)stream>>> ((float4 *)rgba, depth, n_pixels, c);
  return check_launch ("fb_clear_kernel");
}

extern "C" int drb_framebuffer_composite_background (float *rgba, int n_pixels,
                                                     const float *bg4, void *stream)
{
  if (n_pixels < 0 || (n_pixels > 0 && !rgba))
  {
    set_last_error ("framebuffer_composite_background: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_pixels == 0) return DRB_OK;
  const float4 c = bg4 ? make_float4 (bg4[0], bg4[1], bg4[2], bg4[3]) : make_float4 (1.f, 1.f, 1.f, 1.f);
  fb_background_kernel<<<div_up (n_pixels, 256), 256, 0, (cudaStream_t)stream>>> ((float4 *)rgba, n_pixels, c);
  return check_launch ("fb_background_kernel");
}

extern "C" int drb_partials_to_framebuffer (const void *partials, int n, float *fb_rgba,
                                            float *fb_depth, int blend_over, void *stream)
{
  if (n < 0 || (n > 0 && (!partials || !fb_rgba)))
  {
    set_last_error ("partials_to_framebuffer: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  partials_to_fb_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (
  (const VolumePartial *)partials, n, (float4 *)fb_rgba, fb_depth, blend_over);
  return check_launch ("partials_to_fb_kernel");
}

extern "C" int drb_camera_elevate (drb_camera *cam, float degrees)
{
  return drb::camera_turn (cam, degrees, true);
}

extern "C" int drb_camera_azimuth (drb_camera *cam, float degrees)
{
  return drb::camera_turn (cam, degrees, false);
}

// Camera::reset_to_bounds (rendering/camera.cpp:485-514): pad the bounds
// by a fraction of each extent, look at their centre from the current
// direction at one diagonal's distance, field of view 60 degrees.  The pads
// are double and the padded bounds single precision, as in the reference.
extern "C" int drb_camera_reset_to_bounds (drb_camera *cam, const float *bounds6, double xpad,
                                           double ypad, double zpad)
{
  if (!cam || !bounds6)
  {
    set_last_error ("camera_reset_to_bounds: NULL camera or bounds");
    return DRB_ERR_INVALID_ARG;
  }
  const double pads[3] = { xpad, ypad, zpad };
  float lo[3], hi[3], center[3], extent[3];
  for (int d = 0; d < 3; ++d)
  {
    const float bmin = bounds6[2 * d], bmax = bounds6[2 * d + 1];
    if (!(bmin <= bmax))
    {
      set_last_error ("camera_reset_to_bounds: empty bounds");
      return DRB_ERR_INVALID_ARG;
    }
    const double pad = pads[d] * (bmax - bmin);
    const float a = (float)(bmax + pad), b = (float)(bmin - pad);
    lo[d] = fminf (INFINITY, a);
    hi[d] = fmaxf (-INFINITY, a);
    lo[d] = fminf (lo[d], b);
    hi[d] = fmaxf (hi[d], b);
    center[d] = 0.5f * (lo[d] + hi[d]);
    extent[d] = hi[d] - lo[d];
  }
  float dir[3];
  for (int i = 0; i < 3; ++i) dir[i] = cam->pos[i] - cam->look_at[i];
  drb::h_normalize (dir);
  const float diagonal = drb::h_mag (extent);
  for (int i = 0; i < 3; ++i)
  {
    cam->look_at[i] = center[i];
    cam->pos[i] = center[i] + dir[i] * diagonal * 1.0f;
  }
  cam->fov_y = 60.0f;
  return DRB_OK;
}

// ------------------------------------------------------------ mesh lines --

namespace drb
{
namespace
{

// Surface::draw_mesh (rendering/surface.cpp:25-111, 522-550): a line colour
// whose alpha falls off with the distance of the hit's reference point to
// the nearest face edge (second-nearest of the three coordinates, cubic
// smoothstep over `rcp`), blended over the pixel's colour.  The reference
// rounds through double in its shader; the same steps are taken here with
// explicitly rounded operations so no multiply-add is fused.
__device__ float edge_term (float p)
{
  // 0.5 - |p - 0.5| in double, on the fractional part inside [0, 1]
  const double d = p;
  return (float)(d < 0.0 ? 0.0 : d > 1.0 ? 0.0 : __dsub_rn (0.5, fabs (__dsub_rn (d, 0.5))));
}

__global__ void mesh_lines_kernel (const Ray *__restrict__ rays, const RayHit *__restrict__ hits,
                                   int n, float4 line, float rcp, int grid_res,
                                   float4 *__restrict__ fb)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RayHit h = hits[i];
  if (h.hit_idx == -1) return;
  float d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    float p = __fmul_rn ((float)grid_res, h.ref[k]);
    p = __fsub_rn (p, floorf (p));
    d[k] = edge_term (p);
  }
  const float min2 = d[0] < d[1] ? d[0] : d[1];
  const float max2 = d[0] < d[1] ? d[1] : d[0];
  float edge = d[2] < min2 ? min2 : max2 < d[2] ? max2 : d[2];
  edge = __fmul_rn (edge, rcp);
  const double x = fminf (edge, 1.0f);
  const float w = (float)__dadd_rn (__dmul_rn (__dmul_rn (__dsub_rn (__dmul_rn (2.0, x), 3.0), x), x), 1.0);
  float4 f = make_float4 (line.x, line.y, line.z, __fmul_rn (line.w, w));
  const int pix = rays[i].pixel_id;
  const float4 b = fb[pix];
  // blend (rendering/colors.hpp:15-23): front over back
  const float a = __fmul_rn (b.w, __fsub_rn (1.f, f.w));
  f.x = __fadd_rn (f.x, __fmul_rn (b.x, a));
  f.y = __fadd_rn (f.y, __fmul_rn (b.y, a));
  f.z = __fadd_rn (f.z, __fmul_rn (b.z, a));
  f.w = __fadd_rn (a, f.w);
  fb[pix] = f;
}

// Order-preserving unsigned key of a float (negative values flipped).
__global__ void partial_depth_keys_kernel (const VolumePartial *__restrict__ p, int n,
                                           unsigned *__restrict__ key, int *__restrict__ idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned b = __float_as_uint (p[i].depth);
  key[i] = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  idx[i] = i;
}

__global__ void partial_pixel_keys_kernel (const VolumePartial *__restrict__ p, const int *__restrict__ idx,
                                           int n, unsigned *__restrict__ key)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = (unsigned)p[idx[i]].pixel_id;
}

__global__ void partial_order_gather_kernel (const VolumePartial *__restrict__ p, const int *__restrict__ idx,
                                       int n, VolumePartial *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = p[idx[i]];
}

} // namespace
} // namespace drb

extern "C" int drb_surface_mesh_lines (const void *rays, const void *hits, int n,
                                       const float *line_color4, float line_thickness,
                                       float sub_res, float *fb_rgba, void *stream)
{
  if (n < 0 || (n > 0 && (!rays || !hits || !fb_rgba || !line_color4)))
  {
    set_last_error ("surface_mesh_lines: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (!(line_thickness > 0.f) || !(sub_res >= 1.f))
  {
    set_last_error ("surface_mesh_lines: thickness must be > 0 and sub resolution >= 1");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  // ShadeMeshLines::set_uniforms (surface.cpp:34-40): the reciprocal in
  // double times the integer grid resolution, stored as float
  const int grid_res = (int)sub_res;
  const float rcp = (float)((line_thickness > 0.0 ? 1.0 / (double)line_thickness : 0.05) * grid_res);
  const float4 line = make_float4 (line_color4[0], line_color4[1], line_color4[2], line_color4[3]);
  drb::mesh_lines_kernel<<<div_up (n, 256), 256, 0, (cudaStream_t)stream>>> (
  (const drb::Ray *)rays, (const drb::RayHit *)hits, n, line, rcp, grid_res, (float4 *)fb_rgba);
  return check_launch ("mesh_lines_kernel");
}

extern "C" int drb_sort_partials (const void *partials, int n, void *sorted, void *stream)
{
  if (n < 0 || (n > 0 && (!partials || !sorted)))
  {
    set_last_error ("sort_partials: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  if (partials == sorted)
  {
    set_last_error ("sort_partials: the output may not alias the input");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  Scratch scr (s);
  unsigned *k0 = scr.alloc<unsigned> (n);
  unsigned *k1 = scr.alloc<unsigned> (n);
  int *i0 = scr.alloc<int> (n);
  int *i1 = scr.alloc<int> (n);
  if (scr.err != cudaSuccess) return status_from (scr.err);
  const VolumePartial *p = (const VolumePartial *)partials;
  // stable by depth, then stable by pixel: (pixel, depth) order
  drb::partial_depth_keys_kernel<<<div_up (n, 256), 256, 0, s>>> (p, n, k0, i0);
  int st = check_launch ("partial_depth_keys_kernel");
  if (st) return st;
  if ((st = radix_sort_pairs (k0, i0, k1, i1, n, 32, s))) return st;
  drb::partial_pixel_keys_kernel<<<div_up (n, 256), 256, 0, s>>> (p, i1, n, k0);
  if ((st = check_launch ("partial_pixel_keys_kernel"))) return st;
  if ((st = radix_sort_pairs (k0, i1, k1, i0, n, 32, s))) return st;
  drb::partial_order_gather_kernel<<<div_up (n, 256), 256, 0, s>>> (p, i0, n, (VolumePartial *)sorted);
  return check_launch ("partial_order_gather_kernel");
}
