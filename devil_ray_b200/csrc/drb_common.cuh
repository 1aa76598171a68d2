// Common device-side definitions for the B200 ray-element hot path.
//
// Data layouts kept identical to Devil Ray's so that the C-ABI is a drop-in
// for its device structures:
//   - mesh geometry: GridFunction<3> = ctrl_idx int32[n_elem*nd] +
//     values float3[n_ctrl]           (data_model/grid_function.hpp:19-30)
//   - dofs lexicographic, u fastest, then v, then w
//                                     (data_model/pos_tensor_element.tcc:159-180)
//   - BVH inner node = 4 x float4: left box, right box, child ids as int bits;
//     inner child = 4*node, leaf = -(i+1)   (bvh.hpp:16-37, linear_bvh_builder.cpp:319-397)
//   - AABB = (xmin,xmax,ymin,ymax,zmin,zmax) (aabb.hpp:23-27, range.hpp)
//   - Location = {int32 cell, float ref[3]}  (location.hpp:16-20)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define DRB_HD __host__ __device__ __forceinline__
#define DRB_D __device__ __forceinline__

namespace drb
{

constexpr int kWarp = 32;
constexpr int kStackDepth = 64;          // device_mesh.hpp:255 (int32 todo[64])
constexpr int kBarrier = -2000000000;     // device_mesh.hpp:259
// 4-wide traversal (drb_bvh_widen): stack bound 3 per wide level, checked
// against the tree depth when the wide tree is built; empty child slot code
constexpr int kWideStack = 96;
constexpr int kWideEmpty = (int)0x80000000;
constexpr float kEpsilon = 1e-4f;         // math.hpp:25 DRAY_EPSILON_32

struct Vec3
{
  float x, y, z;
};

DRB_HD Vec3 make3 (float x, float y, float z) { return Vec3{ x, y, z }; }
DRB_HD Vec3 operator+ (Vec3 a, Vec3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
DRB_HD Vec3 operator- (Vec3 a, Vec3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
DRB_HD Vec3 operator* (Vec3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
DRB_HD Vec3 operator* (float s, Vec3 a) { return { a.x * s, a.y * s, a.z * s }; }
DRB_HD float dot (Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DRB_HD Vec3 cross (Vec3 a, Vec3 b)
{
  return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
DRB_D float comp (const Vec3 &v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
DRB_D void set_comp (Vec3 &v, int i, float s)
{
  if (i == 0) v.x = s;
  else if (i == 1) v.y = s;
  else v.z = s;
}

// Vec::normalize divides by sqrt(dot) (vec.hpp); rsqrt keeps it on the SFU.
DRB_D Vec3 normalized (Vec3 v)
{
  float inv = rsqrtf (dot (v, v));
  return v * inv;
}

// math.hpp:212-220 rcp_safe: clamp |f| < 1e-8 away from zero, keep the sign.
DRB_D float rcp_safe (float f)
{
  float g = (fabsf (f) < 1e-8f) ? (signbit (f) ? -1e-8f : 1e-8f) : f;
  return 1.0f / g;
}

DRB_D float clampf (float v, float lo, float hi) { return fminf (fmaxf (v, lo), hi); }

// Order-preserving float <-> uint mapping for atomicMin/Max on floats.
DRB_D unsigned int float_to_ordered (float f)
{
  unsigned int u = __float_as_uint (f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
DRB_D float ordered_to_float (unsigned int u)
{
  u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return __uint_as_float (u);
}

struct Ray
{
  // ray.hpp:20-27: dir, near, orig, far, pixel_id (36 bytes)
  Vec3 dir;
  float near_t;
  Vec3 orig;
  float far_t;
  int pixel_id;
};
static_assert (sizeof (Ray) == 36, "Ray layout must match dray::Ray");

struct Location
{
  int cell;
  float ref[3];
};
static_assert (sizeof (Location) == 16, "Location layout must match dray::Location");

struct RayHit
{
  // ray_hit.hpp:16-28
  int hit_idx;
  float dist;
  float ref[3];
};
static_assert (sizeof (RayHit) == 20, "RayHit layout must match dray::RayHit");

struct VolumePartial
{
  // rendering/volume_partial.hpp: pixel, depth, rgba
  int pixel_id;
  float depth;
  float color[4];
};
static_assert (sizeof (VolumePartial) == 24, "VolumePartial layout");

struct PointLight
{
  // rendering/point_light.hpp
  float pos[3];
  float amb[3];
  float diff[3];
  float spec[3];
  float spec_pow;
};
static_assert (sizeof (PointLight) == 52, "PointLight layout");

} // namespace drb
