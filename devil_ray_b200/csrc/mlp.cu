// Learned initial guess for the Newton inversion: a small MLP
// (3 (P+1)^3 + 3 -> 128 -> 128 -> 3, GELU) mapping an order-P hex element's
// control points plus a physical point to a reference-space guess: 84
// inputs at order 2 (27 control points), 195 at order 3 (64).  No counterpart
// in the reference; it feeds DRB_GUESS_GIVEN, with plain Newton from the
// element centre as the fallback whenever the guessed solve fails.
//
// Tensor-core kernels (tcgen05 / UMMA, BF16 operands, FP32 accumulation in
// tensor memory):
//   gemm_kernel       D = A * B^T for A [M x K], B [N x K] (both K-major
//                     bf16), one 128-row tile per CTA, K in chunks of 64,
//                     optional split-K; fused epilogues: +bias & GELU
//                     (storing the pre-activation), x GELU'(Z), fp32 store or
//                     fp32 atomic accumulation (weight gradients)
//   mlp_guess_kernel  fused inference: per tile of 128 (point, element)
//                     pairs, features are built in shared memory, two UMMA
//                     GEMMs run with the weights resident in shared memory,
//                     the 128 -> 3 head runs on the CUDA cores
// Every mbarrier wait is bounded; on timeout the kernel records an error
// flag, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <cstdio>

#include "bernstein.cuh"
#include "drb_common.cuh"
#include "drb_internal.h"
#include "umma.cuh"

namespace drb
{
namespace mlp
{

constexpr int kHid = 128;
constexpr int kOut = 3;

// Dimensions and parameter layout of the network for order-P hex elements.
// Inputs: the (P+1)^3 control points' 3 coordinates, then the point; K
// padded to a multiple of 16 for the UMMA K steps.  Parameters, in one fp32
// vector: W1 [128 x kIn], b1, W2 [128 x 128], b2, W3 [3 x 128], b3.  bf16
// operand copies: W1 [128 x kInPad], W2, W2^T.
template <int P> struct Net
{
  static constexpr int kNd = (P + 1) * (P + 1) * (P + 1);
  static constexpr int kCoords = 3 * kNd;
  static constexpr int kIn = kCoords + 3;
  static constexpr int kInPad = (kIn + 15) / 16 * 16;
  static constexpr int kW1 = 0;
  static constexpr int kB1 = kW1 + kHid * kIn;
  static constexpr int kW2 = kB1 + kHid;
  static constexpr int kB2 = kW2 + kHid * kHid;
  static constexpr int kW3 = kB2 + kHid;
  static constexpr int kB3 = kW3 + kOut * kHid;
  static constexpr int kParams = kB3 + kOut;
  static constexpr int kBW1 = 0;
  static constexpr int kBW2 = kBW1 + kHid * kInPad;
  static constexpr int kBW2T = kBW2 + kHid * kHid;
  static constexpr int kBf16 = kBW2T + kHid * kHid;
  // packed geometry rows: kCoords relative coordinates, then the origin
  static constexpr int kRowF4 = packed_stride (kNd, 3) / 4;
  // activation tile width: the layer-1 input, then the layer-2 input in
  // the same bytes
  static constexpr int kActW = kInPad > kHid ? kInPad : kHid;
  // 128-row tiles in flight per CTA in the fused inference (shared memory:
  // W1, W2 and one activation tile per group within 227 KB)
  static constexpr int kGroups = kActW > kHid ? 2 : 4;
};
static_assert (Net<2>::kIn == 84 && Net<2>::kInPad == 96 && Net<3>::kIn == 195 &&
               Net<3>::kInPad == 208, "network input widths");
static_assert (packed_origin (27) == 81 && packed_origin (64) == 192,
               "geometry rows: relative coordinates, then the origin");

constexpr uint32_t kWaitTries = 1u << 22;

// tanh on the special-function unit (PTX tanh.approx.f32, relative error
// about 2^-11): one instruction instead of a libm-style evaluation, and
// well below the bf16 rounding the activations go through.
DRB_D float tanh_sfu (float x)
{
  float y;
  asm ("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
DRB_D float gelu (float x)
{
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.f + tanh_sfu (u));
}
DRB_D float gelu_grad (float x)
{
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float t = tanh_sfu (u);
  const float du = 0.7978845608028654f * (1.f + 3.f * 0.044715f * x * x);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * du;
}

// Features of one (element, point) pair: control points and point relative
// to the centre of the element's control-point box, scaled by its largest
// half-extent.  (P+1)^3 x 3 control coordinates, then the point, then zeros.
// The packed row holds the relative coordinates, then the origin O, 16-byte
// aligned, so it is read as float4.

// Centre and inverse largest half-extent of the control-point box.
template <int P> DRB_D void pair_frame (const float *__restrict__ row, float (&c)[3], float &inv)
{
  const float4 *r4 = reinterpret_cast<const float4 *> (row);
  float mn[3] = { INFINITY, INFINITY, INFINITY }, mx[3] = { -INFINITY, -INFINITY, -INFINITY };
#pragma unroll
  for (int j = 0; j < Net<P>::kRowF4; ++j)
  {
    const float4 v4 = __ldg (r4 + j);
    const float v[4] = { v4.x, v4.y, v4.z, v4.w };
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      const int q = 4 * j + t;
      if (q < Net<P>::kCoords)
      {
        mn[q % 3] = fminf (mn[q % 3], v[t]);
        mx[q % 3] = fmaxf (mx[q % 3], v[t]);
      }
    }
  }
  float h = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k)
  {
    c[k] = 0.5f * (mn[k] + mx[k]);
    h = fmaxf (h, 0.5f * (mx[k] - mn[k]));
  }
  inv = h > 0.f ? 1.f / h : 0.f;
}

// Features [8 k8, 8 k8 + 8) of one pair as eight packed bf16.  The point
// enters in the row's frame, pt - O (O follows the coordinates in the row).
template <int P>
DRB_D uint4 pair_features8 (const float *__restrict__ row, const float (&pt)[3], const float (&c)[3],
                            float inv, int k8)
{
  constexpr int RF = 4 * Net<P>::kRowF4;
  const int f0 = 8 * k8;
  const float4 z4 = make_float4 (0.f, 0.f, 0.f, 0.f);
  const float4 a = f0 < RF ? __ldg (reinterpret_cast<const float4 *> (row) + 2 * k8) : z4;
  const float4 b = f0 + 4 < RF ? __ldg (reinterpret_cast<const float4 *> (row) + 2 * k8 + 1) : z4;
  float v[8] = { a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w };
#pragma unroll
  for (int t = 0; t < 8; ++t)
  {
    const int q = f0 + t;
    if (q >= Net<P>::kIn) v[t] = 0.f;
    else if (q >= Net<P>::kCoords) v[t] = __fsub_rn (pt[q - Net<P>::kCoords], v[t]);
  }
#pragma unroll
  for (int t = 0; t < 8; ++t)
  {
    const int q = f0 + t;
    if (q < Net<P>::kIn) v[t] = (v[t] - c[q % 3]) * inv;
  }
  uint4 out;
  __nv_bfloat162 p0 = __floats2bfloat162_rn (v[0], v[1]), p1 = __floats2bfloat162_rn (v[2], v[3]);
  __nv_bfloat162 p2 = __floats2bfloat162_rn (v[4], v[5]), p3 = __floats2bfloat162_rn (v[6], v[7]);
  out.x = *reinterpret_cast<uint32_t *> (&p0);
  out.y = *reinterpret_cast<uint32_t *> (&p1);
  out.z = *reinterpret_cast<uint32_t *> (&p2);
  out.w = *reinterpret_cast<uint32_t *> (&p3);
  return out;
}

// ------------------------------------------------------------ prepare --

template <int P>
__global__ void prepare_kernel (const float *__restrict__ p, __nv_bfloat16 *__restrict__ wb)
{
  using N = Net<P>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < kHid * N::kInPad)
  {
    const int r = t / N::kInPad, k = t - r * N::kInPad;
    wb[N::kBW1 + t] = __float2bfloat16_rn (k < N::kIn ? p[N::kW1 + r * N::kIn + k] : 0.f);
  }
  if (t < kHid * kHid)
  {
    const int r = t / kHid, k = t - r * kHid;
    wb[N::kBW2 + t] = __float2bfloat16_rn (p[N::kW2 + t]);
    wb[N::kBW2T + t] = __float2bfloat16_rn (p[N::kW2 + k * kHid + r]);
  }
}

// ----------------------------------------------------------- features --

template <int P>
__global__ void features_kernel (const float *__restrict__ packed, int stride,
                                 const int *__restrict__ elem, const float *__restrict__ pts, int n,
                                 int n_pad, __nv_bfloat16 *__restrict__ X)
{
  using N = Net<P>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pad) return;
  const int e = i < n ? elem[i] : -1;
  uint4 *dst = reinterpret_cast<uint4 *> (X + (size_t)i * N::kInPad);
  if (e < 0)
  {
#pragma unroll
    for (int k8 = 0; k8 < N::kInPad / 8; ++k8) dst[k8] = make_uint4 (0u, 0u, 0u, 0u);
    return;
  }
  const float *row = packed + (size_t)e * stride;
  const float pt[3] = { pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2] };
  float c[3], inv;
  pair_frame<P> (row, c, inv);
#pragma unroll
  for (int k8 = 0; k8 < N::kInPad / 8; ++k8) dst[k8] = pair_features8<P> (row, pt, c, inv, k8);
}

// --------------------------------------------------------------- GEMM --

enum Epilogue
{
  EPI_STORE = 0,     // C[r, c] = D (+ bias[c])                 fp32
  EPI_BIAS_GELU = 1, // Z[r, c] = D + bias[c], H = bf16(gelu(Z))
  EPI_GELU_GRAD = 2, // H[r, c] = bf16(D * gelu'(Z[r, c]))
  EPI_ATOMIC = 3,    // atomicAdd(C[r * ldc + c], D) for c < ncols
  EPI_ATOMIC_T = 4   // atomicAdd(C[c * ldc + r], D) for r < ncols (transposed)
};

struct GemmArgs
{
  const __nv_bfloat16 *A; // [M x K]
  const __nv_bfloat16 *B; // [N x K]
  int M, N, K;
  int k_split;             // K elements per split (multiple of 64)
  const float *bias;
  float *C;                // fp32 output / pre-activation Z
  __nv_bfloat16 *H;        // bf16 output
  const float *Zin;        // pre-activation for EPI_GELU_GRAD
  int ldc, ncols;          // for EPI_ATOMIC
  int *err;
};

constexpr int kKC = 64;       // K per chunk
constexpr int kGemmN = 128;   // max N handled (TMEM columns)

template <int EPI>
__global__ void __launch_bounds__ (128) gemm_kernel (GemmArgs g)
{
  extern __shared__ __align__ (1024) unsigned char smem[];
  unsigned char *sA = smem;                       // 128 x 64 bf16 = 16 KB
  unsigned char *sB = smem + 128 * kKC * 2;       // N x 64 bf16 <= 16 KB
  __shared__ __align__ (8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  const int kbeg = blockIdx.y * g.k_split;
  const int kend = min (g.K, kbeg + g.k_split);
  if (warp == 0) umma::tmem_alloc (&tmem_base, kGemmN);
  if (tid == 0) umma::mbar_init (&mbar, 1);
  umma::fence_before_sync ();
  __syncthreads ();
  umma::fence_after_sync ();
  const uint32_t tbase = tmem_base;
  const uint32_t idesc = umma::idesc_bf16_f32 (128, g.N);
  uint32_t phase = 0;
  bool ok = true;
  int chunks = 0;
  for (int k0 = kbeg; k0 < kend; k0 += kKC)
  {
    // cooperative 16-byte loads into the interleaved layout
    for (int v = tid; v < 128 * (kKC / 8); v += 128)
    {
      const int r = v / (kKC / 8), j = v - r * (kKC / 8);
      const int k = k0 + 8 * j;
      uint4 val = make_uint4 (0, 0, 0, 0);
      if (m0 + r < g.M && k < kend)
        val = *reinterpret_cast<const uint4 *> (g.A + (size_t)(m0 + r) * g.K + k);
      *reinterpret_cast<uint4 *> (sA + umma::tile_offset (r, 8 * j, kKC)) = val;
    }
    for (int v = tid; v < g.N * (kKC / 8); v += 128)
    {
      const int r = v / (kKC / 8), j = v - r * (kKC / 8);
      const int k = k0 + 8 * j;
      uint4 val = make_uint4 (0, 0, 0, 0);
      if (k < kend) val = *reinterpret_cast<const uint4 *> (g.B + (size_t)r * g.K + k);
      *reinterpret_cast<uint4 *> (sB + umma::tile_offset (r, 8 * j, kKC)) = val;
    }
    umma::fence_async_smem ();
    __syncthreads ();
    if (tid == 0)
    {
      umma::fence_after_sync ();
      const uint32_t a0 = umma::smem_addr (sA), b0 = umma::smem_addr (sB);
#pragma unroll
      for (int kk = 0; kk < kKC / 16; ++kk)
      {
        const uint64_t ad = umma::desc_kmajor (a0 + kk * 256, 128, (kKC / 8) * 128);
        const uint64_t bd = umma::desc_kmajor (b0 + kk * 256, 128, (kKC / 8) * 128);
        umma::mma_bf16 (tbase, ad, bd, idesc, (chunks > 0 || kk > 0) ? 1u : 0u);
      }
      umma::mma_commit (&mbar);
    }
    ok = umma::mbar_wait (&mbar, phase, kWaitTries) && ok;
    phase ^= 1u;
    ++chunks;
    umma::fence_after_sync ();
    __syncthreads ();
    if (!__syncthreads_and (ok)) break;
  }
  ok = __syncthreads_and (ok) != 0; // CTA-uniform before the warp-collective loads
  if (!ok && tid == 0 && g.err) atomicExch (g.err, 1);
  // epilogue: thread t owns accumulator row t (TMEM lane t)
  const int r = m0 + tid;
  if (ok && chunks > 0)
  {
    for (int c0 = 0; c0 < g.N; c0 += 32)
    {
      float d[32];
      umma::tmem_ld32 (tbase + ((uint32_t)(warp * 32) << 16) + c0, d);
      if (r >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 32; ++j)
      {
        const int c = c0 + j;
        if (c >= g.N) break;
        if (EPI == EPI_STORE)
          g.C[(size_t)r * g.N + c] = d[j] + (g.bias ? g.bias[c] : 0.f);
        else if (EPI == EPI_BIAS_GELU)
        {
          const float z = d[j] + g.bias[c];
          g.C[(size_t)r * g.N + c] = z;
          g.H[(size_t)r * g.N + c] = __float2bfloat16_rn (gelu (z));
        }
        else if (EPI == EPI_GELU_GRAD)
          g.H[(size_t)r * g.N + c] = __float2bfloat16_rn (d[j] * gelu_grad (g.Zin[(size_t)r * g.N + c]));
        else if (EPI == EPI_ATOMIC)
        {
          if (c < g.ncols) atomicAdd (g.C + (size_t)r * g.ldc + c, d[j]);
        }
        else if (r < g.ncols)
          atomicAdd (g.C + (size_t)c * g.ldc + r, d[j]);
      }
    }
  }
  umma::fence_before_sync ();
  __syncthreads ();
  if (warp == 0) umma::tmem_dealloc (tbase, kGemmN);
}

// ------------------------------------------------------- head / losses --

// y = W3 gelu(Z2) + b3; masked MSE; dY; grads of W3, b3; dZ2 = (W3^T dY) x
// gelu'(Z2) as bf16; db2.  One block of 128 threads per 128 rows, in two
// coalesced phases: a warp per row for the head and dY (Z2 rows read as
// float4, the 3 dot products reduced by shuffles), then a thread per column
// over the block's rows for dZ2 and the weight-gradient column sums, so the
// block adds one partial per parameter to the global gradient.
template <int P>
__global__ void __launch_bounds__ (128)
head_kernel (const float *__restrict__ p, const float *__restrict__ Z2, const float *__restrict__ target,
             const float *__restrict__ weight, int n, int n_pad, float inv_count, float *__restrict__ y_out,
             float *__restrict__ grad, __nv_bfloat16 *__restrict__ dZ2, float *__restrict__ loss)
{
  constexpr int kW3 = Net<P>::kW3, kB3 = Net<P>::kB3, kB2 = Net<P>::kB2;
  __shared__ float s_w3[kOut * kHid];
  __shared__ float s_dy[128][kOut];
  __shared__ float s_loss;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int q = tid; q < kOut * kHid; q += blockDim.x) s_w3[q] = p[kW3 + q];
  if (tid == 0) s_loss = 0.f;
  __syncthreads ();
  const int r0 = blockIdx.x * 128;
  const int rows = min (128, n_pad - r0);
  const float b3[kOut] = { p[kB3], p[kB3 + 1], p[kB3 + 2] };
  // phase 1: head and dY, a warp per row, lane l holds columns [4 l, 4 l + 4)
  for (int rr = warp; rr < rows; rr += 4)
  {
    const int i = r0 + rr;
    const float4 z4 = *reinterpret_cast<const float4 *> (Z2 + (size_t)i * kHid + 4 * lane);
    const float z[4] = { z4.x, z4.y, z4.z, z4.w };
    float y[kOut] = { 0.f, 0.f, 0.f };
#pragma unroll
    for (int t = 0; t < 4; ++t)
    {
      const float h = gelu (z[t]);
#pragma unroll
      for (int o = 0; o < kOut; ++o) y[o] = fmaf (s_w3[o * kHid + 4 * lane + t], h, y[o]);
    }
#pragma unroll
    for (int o = 0; o < kOut; ++o)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) y[o] += __shfl_xor_sync (0xffffffffu, y[o], off);
    if (lane == 0)
    {
      const float w = (i < n && weight) ? weight[i] : (i < n ? 1.f : 0.f);
      float l = 0.f;
#pragma unroll
      for (int o = 0; o < kOut; ++o)
      {
        const float yo = y[o] + b3[o];
        const float e = (i < n && target) ? (yo - target[3 * (size_t)i + o]) : 0.f;
        l += w * e * e;
        s_dy[rr][o] = 2.f * w * e * inv_count;
        if (y_out && i < n) y_out[3 * (size_t)i + o] = yo;
      }
      if (grad) atomicAdd (&s_loss, l * inv_count);
    }
  }
  if (!grad) return;
  __syncthreads ();
  // phase 2: thread c owns column c of the block's rows
  const int c = tid;
  float gw3[kOut] = { 0.f, 0.f, 0.f };
  float db2 = 0.f;
  const float w3c[kOut] = { s_w3[c], s_w3[kHid + c], s_w3[2 * kHid + c] };
  for (int rr = 0; rr < rows; ++rr)
  {
    const size_t at = (size_t)(r0 + rr) * kHid + c;
    const float z = Z2[at];
    const float h = gelu (z);
    float dh = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; ++o)
    {
      const float dy = s_dy[rr][o];
      gw3[o] = fmaf (dy, h, gw3[o]);
      dh = fmaf (w3c[o], dy, dh);
    }
    const float dz = dh * gelu_grad (z);
    dZ2[at] = __float2bfloat16_rn (dz);
    db2 += dz;
  }
#pragma unroll
  for (int o = 0; o < kOut; ++o) atomicAdd (grad + kW3 + o * kHid + c, gw3[o]);
  atomicAdd (grad + kB2 + c, db2);
  if (tid < kOut)
  {
    float gb = 0.f;
    for (int rr = 0; rr < rows; ++rr) gb += s_dy[rr][tid];
    atomicAdd (grad + kB3 + tid, gb);
  }
  if (tid == 0 && loss) atomicAdd (loss, s_loss);
}

// column sums of a bf16 [rows x 128] matrix into grad[off + c]
__global__ void colsum_kernel (const __nv_bfloat16 *__restrict__ M, int rows, float *__restrict__ out)
{
  __shared__ float s[kHid];
  if (threadIdx.x < kHid) s[threadIdx.x] = 0.f;
  __syncthreads ();
  const int c = threadIdx.x & (kHid - 1);
  float acc = 0.f;
  for (int r = blockIdx.x * (blockDim.x / kHid) + threadIdx.x / kHid; r < rows;
       r += gridDim.x * (blockDim.x / kHid))
    acc += __bfloat162float (M[(size_t)r * kHid + c]);
  atomicAdd (&s[c], acc);
  __syncthreads ();
  if (threadIdx.x < kHid) atomicAdd (out + threadIdx.x, s[threadIdx.x]);
}

// bf16 transpose [rows x cols] -> [cols x rows]
__global__ void transpose_kernel (const __nv_bfloat16 *__restrict__ in, int rows, int cols,
                                  __nv_bfloat16 *__restrict__ out)
{
  __shared__ __nv_bfloat16 t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y)
  {
    const int r = by + j, c = bx + threadIdx.x;
    t[j][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : __float2bfloat16_rn (0.f);
  }
  __syncthreads ();
  for (int j = threadIdx.y; j < 32; j += blockDim.y)
  {
    const int c = bx + j, r = by + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)c * rows + r] = t[threadIdx.x][j];
  }
}

__global__ void adam_kernel (float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                             float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                             float c1, float c2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf (vi * c2) + eps);
}

// ------------------------------------------------------ fused inference --

struct GuessArgs
{
  const float *params;
  const __nv_bfloat16 *wb;
  const float *packed;
  int stride;
  const int *elem;
  const float *pts;
  const int *order;
  int n;
  float *guess;
  int *err;
};

// Fused inference keeps Net<P>::kGroups 128-row tiles in flight per CTA
// (four at orders 1-2, two at order 3, whose 208-wide layer-1 input needs
// wider tiles), one per warpgroup, with the bf16 weights resident once per
// CTA.  Each warpgroup owns one activation tile (the layer-1 input, then
// the 128-wide layer-2 input in the same bytes) and 128 TMEM columns (D1,
// then D2 in the same columns), and synchronises only with itself (named
// barrier 1 + g), so one group's gathers and epilogues overlap the others'
// MMAs.
template <int P> constexpr size_t guess_w1_bytes () { return (size_t)kHid * Net<P>::kInPad * 2; }
constexpr size_t guess_w2_bytes () { return (size_t)kHid * kHid * 2; }
template <int P> constexpr size_t guess_act_bytes () { return (size_t)128 * Net<P>::kActW * 2; }
template <int P> constexpr size_t guess_smem ()
{
  return guess_w1_bytes<P> () + guess_w2_bytes () + Net<P>::kGroups * guess_act_bytes<P> ();
}
static_assert (guess_smem<3> () <= 227 * 1024 && guess_smem<2> () <= 227 * 1024 &&
               guess_smem<1> () <= 227 * 1024, "fused inference fits in shared memory");

DRB_D void group_sync (int g)
{
  asm volatile ("bar.sync %0, %1;" ::"r"(1 + g), "r"(128) : "memory");
}
// AND of a predicate over the 128 threads of warpgroup g.
DRB_D bool group_and (int g, bool v)
{
  uint32_t r;
  asm volatile ("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
                "bar.red.and.pred p, %2, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(r)
                : "r"((uint32_t)v), "r"(1 + g)
                : "memory");
  return r != 0;
}

template <int P>
__global__ void __launch_bounds__ (128 * Net<P>::kGroups, 1) mlp_guess_kernel (GuessArgs a)
{
  using N = Net<P>;
  constexpr int kGuessGroups = N::kGroups;
  constexpr int kGuessThreads = 128 * kGuessGroups;
  constexpr int kInPad = N::kInPad;
  constexpr size_t kGuessW1 = guess_w1_bytes<P> ();
  constexpr size_t kGuessW2 = guess_w2_bytes ();
  constexpr size_t kGuessAct = guess_act_bytes<P> ();
  extern __shared__ __align__ (1024) unsigned char smem[];
  unsigned char *sW1 = smem;                     // 128 x 96
  unsigned char *sW2 = sW1 + kGuessW1;           // 128 x 128
  __shared__ float s_b1[kHid], s_b2[kHid], s_w3[kOut * kHid], s_b3[kOut];
  __shared__ __align__ (8) uint64_t mbar[kGuessGroups];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int g = warp >> 2;              // warpgroup = tile slot
  const int row = tid & 127;            // row of the tile = TMEM lane
  unsigned char *sAct = sW2 + kGuessW2 + (size_t)g * kGuessAct;
  for (int v = tid; v < kHid * (kInPad / 8); v += kGuessThreads)
  {
    const int r = v / (kInPad / 8), j = v - r * (kInPad / 8);
    *reinterpret_cast<uint4 *> (sW1 + umma::tile_offset (r, 8 * j, kInPad)) =
    *reinterpret_cast<const uint4 *> (a.wb + N::kBW1 + (size_t)r * kInPad + 8 * j);
  }
  for (int v = tid; v < kHid * (kHid / 8); v += kGuessThreads)
  {
    const int r = v / (kHid / 8), j = v - r * (kHid / 8);
    *reinterpret_cast<uint4 *> (sW2 + umma::tile_offset (r, 8 * j, kHid)) =
    *reinterpret_cast<const uint4 *> (a.wb + N::kBW2 + (size_t)r * kHid + 8 * j);
  }
  for (int q = tid; q < kHid; q += kGuessThreads)
  {
    s_b1[q] = a.params[N::kB1 + q];
    s_b2[q] = a.params[N::kB2 + q];
  }
  for (int q = tid; q < kOut * kHid; q += kGuessThreads) s_w3[q] = a.params[N::kW3 + q];
  if (tid < kOut) s_b3[tid] = a.params[N::kB3 + tid];
  if (warp == 0) umma::tmem_alloc (&tmem_base, kGuessGroups * kHid);
  if (tid < kGuessGroups) umma::mbar_init (&mbar[tid], 1);
  umma::fence_before_sync ();
  __syncthreads ();
  umma::fence_after_sync ();
  // warp w reads TMEM lanes [32 (w % 4), +32); its group's columns start at 128 g
  const uint32_t tacc = tmem_base + (uint32_t)(g * kHid) + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t tmma = tmem_base + (uint32_t)(g * kHid);
  const uint32_t idesc = umma::idesc_bf16_f32 (128, kHid);
  uint32_t phase = 0;
  bool ok = true;
  const int tiles = (a.n + 127) / 128;
  for (int tile = blockIdx.x * kGuessGroups + g; tile < tiles; tile += gridDim.x * kGuessGroups)
  {
    const int i = tile * 128 + row;
    const int q = i < a.n ? (a.order ? __ldg (a.order + i) : i) : -1;
    const int e = q >= 0 ? __ldg (a.elem + q) : -1;
    float pt[3] = { 0.f, 0.f, 0.f };
    // layer-1 input row: features in the 96-wide interleaved layout
    if (e >= 0)
    {
      pt[0] = __ldg (a.pts + 3 * (size_t)q);
      pt[1] = __ldg (a.pts + 3 * (size_t)q + 1);
      pt[2] = __ldg (a.pts + 3 * (size_t)q + 2);
      const float *er = a.packed + (size_t)e * a.stride;
      float c[3], inv;
      pair_frame<P> (er, c, inv);
#pragma unroll
      for (int k8 = 0; k8 < kInPad / 8; ++k8)
        *reinterpret_cast<uint4 *> (sAct + umma::tile_offset (row, 8 * k8, kInPad)) =
        pair_features8<P> (er, pt, c, inv, k8);
    }
    else
    {
#pragma unroll
      for (int k8 = 0; k8 < kInPad / 8; ++k8)
        *reinterpret_cast<uint4 *> (sAct + umma::tile_offset (row, 8 * k8, kInPad)) =
        make_uint4 (0u, 0u, 0u, 0u);
    }
    umma::fence_async_smem ();
    group_sync (g);
    if (row == 0)
    {
      umma::fence_after_sync ();
      const uint32_t a0 = umma::smem_addr (sAct), b0 = umma::smem_addr (sW1);
#pragma unroll
      for (int kk = 0; kk < kInPad / 16; ++kk)
        umma::mma_bf16 (tmma, umma::desc_kmajor (a0 + kk * 256, 128, (kInPad / 8) * 128),
                        umma::desc_kmajor (b0 + kk * 256, 128, (kInPad / 8) * 128), idesc,
                        kk > 0 ? 1u : 0u);
      umma::mma_commit (&mbar[g]);
    }
    ok = group_and (g, umma::mbar_wait (&mbar[g], phase, kWaitTries));
    phase ^= 1u;
    umma::fence_after_sync ();
    if (!ok) break;
    // layer-1 epilogue: GELU(D1 + b1) as bf16 -> layer-2 input (same bytes)
#pragma unroll 1
    for (int c0 = 0; c0 < kHid; c0 += 32)
    {
      float d[32];
      umma::tmem_ld32 (tacc + c0, d);
#pragma unroll
      for (int k8 = 0; k8 < 4; ++k8)
      {
        uint4 o;
        uint32_t *ow = reinterpret_cast<uint32_t *> (&o);
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
          const int cc = 8 * k8 + 2 * j;
          __nv_bfloat162 h2 = __floats2bfloat162_rn (gelu (d[cc] + s_b1[c0 + cc]),
                                                     gelu (d[cc + 1] + s_b1[c0 + cc + 1]));
          ow[j] = *reinterpret_cast<uint32_t *> (&h2);
        }
        *reinterpret_cast<uint4 *> (sAct + umma::tile_offset (row, c0 + 8 * k8, kHid)) = o;
      }
    }
    umma::fence_async_smem ();
    umma::fence_before_sync ();
    group_sync (g);
    if (row == 0)
    {
      umma::fence_after_sync ();
      const uint32_t a0 = umma::smem_addr (sAct), b0 = umma::smem_addr (sW2);
#pragma unroll
      for (int kk = 0; kk < kHid / 16; ++kk)
        umma::mma_bf16 (tmma, umma::desc_kmajor (a0 + kk * 256, 128, (kHid / 8) * 128),
                        umma::desc_kmajor (b0 + kk * 256, 128, (kHid / 8) * 128), idesc,
                        kk > 0 ? 1u : 0u);
      umma::mma_commit (&mbar[g]);
    }
    ok = group_and (g, umma::mbar_wait (&mbar[g], phase, kWaitTries));
    phase ^= 1u;
    umma::fence_after_sync ();
    if (!ok) break;
    // layer-2 epilogue + 128 -> 3 head on the CUDA cores
    float y[kOut] = { s_b3[0], s_b3[1], s_b3[2] };
#pragma unroll 1
    for (int c0 = 0; c0 < kHid; c0 += 32)
    {
      float d[32];
      umma::tmem_ld32 (tacc + c0, d);
#pragma unroll
      for (int j = 0; j < 32; ++j)
      {
        const float h = gelu (d[j] + s_b2[c0 + j]);
#pragma unroll
        for (int o = 0; o < kOut; ++o) y[o] = fmaf (s_w3[o * kHid + c0 + j], h, y[o]);
      }
    }
    if (q >= 0)
    {
#pragma unroll
      for (int o = 0; o < kOut; ++o)
        a.guess[3 * (size_t)q + o] = (e >= 0) ? fminf (1.f, fmaxf (0.f, y[o])) : 0.5f;
    }
    // D2 and the activation tile are reused by the next tile of this group
    umma::fence_before_sync ();
    group_sync (g);
  }
  if (!ok && row == 0 && a.err) atomicExch (a.err, 1);
  umma::fence_before_sync ();
  __syncthreads ();
  if (warp == 0) umma::tmem_dealloc (tmem_base, kGuessGroups * kHid);
}

template <int EPI> int launch_gemm (const GemmArgs &g, cudaStream_t s)
{
  const size_t smem = (size_t)128 * kKC * 2 + (size_t)kGemmN * kKC * 2;
  // at most 4 CTAs per SM so that their TMEM (128 columns each) always fits
  const size_t smem_req = smem < 48 * 1024 ? 48 * 1024 : smem;
  cudaFuncSetAttribute (gemm_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_req);
  dim3 grid ((unsigned)div_up (g.M, 128), (unsigned)div_up (g.K, g.k_split));
  gemm_kernel<EPI><<<grid, 128, smem_req, s>>> (g);
  return check_launch ("gemm_kernel");
}

} // namespace mlp
} // namespace drb

using namespace drb;
using namespace drb::mlp;

namespace
{

bool mlp_order_ok (int order)
{
  if (order >= 1 && order <= 3) return true;
  set_last_error ("mlp: the network is defined for hex orders 1..3");
  return false;
}

template <int P> int prepare_p (const float *params, void *wbf16, cudaStream_t s)
{
  const int n = kHid * (Net<P>::kInPad > kHid ? Net<P>::kInPad : kHid);
  prepare_kernel<P><<<div_up (n, 256), 256, 0, s>>> (params, (__nv_bfloat16 *)wbf16);
  return check_launch ("prepare_kernel");
}

template <int P>
int features_p (const drb_mesh *mesh, const int *elem, const float *pts, int n, int n_pad, void *X,
                cudaStream_t s)
{
  features_kernel<P><<<div_up (n_pad, 128), 128, 0, s>>> (
  mesh->packed, packed_stride (Net<P>::kNd, 3), elem, pts, n, n_pad, (__nv_bfloat16 *)X);
  return check_launch ("features_kernel");
}

template <int P> long long workspace_p (int n_pad)
{
  const long long r = n_pad;
  return r * kHid * 4 * 2 + r * kHid * 2 * 4 + r * kHid * 2 * 3 + r * Net<P>::kInPad * 2 + 4096;
}

// The two layers of the forward pass into Z1/H1 and Z2/H2.
template <int P>
int forward_layers (const float *params, const __nv_bfloat16 *wb, const void *X, int n_pad,
                    float *Z1, __nv_bfloat16 *H1, float *Z2, __nv_bfloat16 *H2, int *err,
                    cudaStream_t s)
{
  using N = Net<P>;
  GemmArgs g{};
  g.A = (const __nv_bfloat16 *)X;
  g.B = wb + N::kBW1;
  g.M = n_pad;
  g.N = kHid;
  g.K = N::kInPad;
  g.k_split = ((N::kInPad + kKC - 1) / kKC) * kKC;
  g.bias = params + N::kB1;
  g.C = Z1;
  g.H = H1;
  g.err = err;
  int st = launch_gemm<EPI_BIAS_GELU> (g, s);
  if (st) return st;
  g.A = H1;
  g.B = wb + N::kBW2;
  g.K = kHid;
  g.k_split = kHid;
  g.bias = params + N::kB2;
  g.C = Z2;
  g.H = H2;
  return launch_gemm<EPI_BIAS_GELU> (g, s);
}

template <int P>
int forward_p (const float *params, const void *wbf16, const void *X, int n, int n_pad, float *y,
               void *workspace, int *err, cudaStream_t s)
{
  unsigned char *w = (unsigned char *)workspace;
  float *Z1 = (float *)w;
  float *Z2 = Z1 + (size_t)n_pad * kHid;
  __nv_bfloat16 *H1 = (__nv_bfloat16 *)(Z2 + (size_t)n_pad * kHid);
  __nv_bfloat16 *H2 = H1 + (size_t)n_pad * kHid;
  int st = forward_layers<P> (params, (const __nv_bfloat16 *)wbf16, X, n_pad, Z1, H1, Z2, H2, err, s);
  if (st) return st;
  head_kernel<P><<<div_up (n_pad, 128), 128, 0, s>>> (params, Z2, nullptr, nullptr, n, n_pad, 0.f, y,
                                                      nullptr, nullptr, nullptr);
  return check_launch ("head_kernel");
}

template <int P>
int train_step_p (const float *params, const void *wbf16, const void *X, const float *target,
                  const float *weight, int n, int n_pad, float *grad, float *loss, void *workspace,
                  int *err, cudaStream_t s)
{
  using N = Net<P>;
  unsigned char *w = (unsigned char *)workspace;
  const size_t R = (size_t)n_pad;
  float *Z1 = (float *)w;
  float *Z2 = Z1 + R * kHid;
  __nv_bfloat16 *H1 = (__nv_bfloat16 *)(Z2 + R * kHid);
  __nv_bfloat16 *H2 = H1 + R * kHid;
  __nv_bfloat16 *dZ2 = H2 + R * kHid;
  __nv_bfloat16 *dZ1 = dZ2 + R * kHid;
  __nv_bfloat16 *dZ2T = dZ1 + R * kHid;
  __nv_bfloat16 *H1T = dZ2T + R * kHid;
  __nv_bfloat16 *dZ1T = H1T + R * kHid;
  __nv_bfloat16 *XT = dZ1T + R * kHid;
  const __nv_bfloat16 *wb = (const __nv_bfloat16 *)wbf16;
  cudaMemsetAsync (grad, 0, sizeof (float) * N::kParams, s);
  if (loss) cudaMemsetAsync (loss, 0, sizeof (float), s);
  int st = forward_layers<P> (params, wb, X, n_pad, Z1, H1, Z2, H2, err, s);
  if (st) return st;
  // head, loss, dW3, db3, dZ2, db2
  head_kernel<P><<<div_up (n_pad, 128), 128, 0, s>>> (params, Z2, target, weight, n, n_pad,
                                                      1.f / (float)n, nullptr, grad, dZ2, loss);
  if ((st = check_launch ("head_kernel"))) return st;
  // dZ1 = (dZ2 W2) x gelu'(Z1): B operand is W2^T
  GemmArgs b{};
  b.A = dZ2;
  b.B = wb + N::kBW2T;
  b.M = n_pad;
  b.N = kHid;
  b.K = kHid;
  b.k_split = kHid;
  b.Zin = Z1;
  b.H = dZ1;
  b.err = err;
  if ((st = launch_gemm<EPI_GELU_GRAD> (b, s))) return st;
  colsum_kernel<<<min (div_up (n_pad, 2), 1024), 256, 0, s>>> (dZ1, n_pad, grad + N::kB1);
  if ((st = check_launch ("colsum_kernel"))) return st;
  // transposes for the weight gradients (K = batch)
  dim3 tb (32, 8);
  transpose_kernel<<<dim3 (kHid / 32, div_up (n_pad, 32)), tb, 0, s>>> (dZ2, n_pad, kHid, dZ2T);
  transpose_kernel<<<dim3 (kHid / 32, div_up (n_pad, 32)), tb, 0, s>>> (H1, n_pad, kHid, H1T);
  transpose_kernel<<<dim3 (kHid / 32, div_up (n_pad, 32)), tb, 0, s>>> (dZ1, n_pad, kHid, dZ1T);
  transpose_kernel<<<dim3 (div_up (N::kInPad, 32), div_up (n_pad, 32)), tb, 0, s>>> (
  (const __nv_bfloat16 *)X, n_pad, N::kInPad, XT);
  if ((st = check_launch ("transpose_kernel"))) return st;
  const int ksplit = n_pad <= 1024 ? ((n_pad + kKC - 1) / kKC) * kKC : 1024;
  // dW2 = dZ2^T H1
  GemmArgs d2{};
  d2.A = dZ2T;
  d2.B = H1T;
  d2.M = kHid;
  d2.N = kHid;
  d2.K = n_pad;
  d2.k_split = ksplit;
  d2.C = grad + N::kW2;
  d2.ldc = kHid;
  d2.ncols = kHid;
  d2.err = err;
  if ((st = launch_gemm<EPI_ATOMIC> (d2, s))) return st;
  GemmArgs d1{};
  d1.K = n_pad;
  d1.k_split = ksplit;
  d1.C = grad + N::kW1;
  d1.ldc = N::kIn;
  d1.ncols = N::kIn;
  d1.err = err;
  if (N::kInPad <= kGemmN)
  {
    // dW1 = dZ1^T X (the first kIn of kInPad columns)
    d1.A = dZ1T;
    d1.B = XT;
    d1.M = kHid;
    d1.N = N::kInPad;
    return launch_gemm<EPI_ATOMIC> (d1, s);
  }
  // wider inputs: dW1^T = X^T dZ1, rows of the input dimension in 128-row
  // tiles, stored transposed (the first kIn rows)
  d1.A = XT;
  d1.B = dZ1T;
  d1.M = N::kInPad;
  d1.N = kHid;
  return launch_gemm<EPI_ATOMIC_T> (d1, s);
}

template <int P>
int guess_p (const float *params, const void *wbf16, const drb_mesh *mesh, const int *elem,
             const float *pts, const int *order, int n, float *guess, int *err, cudaStream_t s)
{
  GuessArgs a;
  a.params = params;
  a.wb = (const __nv_bfloat16 *)wbf16;
  a.packed = mesh->packed;
  a.stride = packed_stride (Net<P>::kNd, 3);
  a.elem = elem;
  a.pts = pts;
  a.order = order;
  a.n = n;
  a.guess = guess;
  a.err = err;
  constexpr size_t smem = guess_smem<P> ();
  cudaFuncSetAttribute (mlp_guess_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int tiles = div_up (n, 128);
  const int grid = min (div_up (tiles, Net<P>::kGroups), sm_count ());
  mlp_guess_kernel<P><<<grid, 128 * Net<P>::kGroups, smem, s>>> (a);
  return check_launch ("mlp_guess_kernel");
}

bool mesh_ok (const drb_mesh *mesh, const char *what)
{
  if (mesh && mesh->packed && mesh->dim == 3 && mesh->order >= 1 && mesh->order <= 3 &&
      mesh->ncomp == 3 && mesh->shape == DRB_SHAPE_TENSOR)
    return true;
  char buf[160];
  std::snprintf (buf, sizeof (buf), "%s: needs a packed hex geometry mesh of order 1..3", what);
  set_last_error (buf);
  return false;
}

} // namespace

extern "C" int drb_mlp_param_count (int order)
{
  return !mlp_order_ok (order) ? -1 : order == 1 ? Net<1>::kParams : order == 2 ? Net<2>::kParams
                                                                                  : Net<3>::kParams;
}
extern "C" int drb_mlp_bf16_count (int order)
{
  return !mlp_order_ok (order) ? -1 : order == 1 ? Net<1>::kBf16 : order == 2 ? Net<2>::kBf16
                                                                                : Net<3>::kBf16;
}
extern "C" int drb_mlp_input_width (int order)
{
  return !mlp_order_ok (order) ? -1 : order == 1 ? Net<1>::kInPad : order == 2 ? Net<2>::kInPad
                                                                                 : Net<3>::kInPad;
}

extern "C" int drb_mlp_prepare (int order, const float *params, void *wbf16, void *stream)
{
  if (!mlp_order_ok (order)) return DRB_ERR_INVALID_ARG;
  if (!params || !wbf16)
  {
    set_last_error ("mlp_prepare: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  return order == 1 ? prepare_p<1> (params, wbf16, s) : order == 2 ? prepare_p<2> (params, wbf16, s)
                                                                   : prepare_p<3> (params, wbf16, s);
}

extern "C" int drb_mlp_features (const drb_mesh *mesh, const int *elem, const float *pts, int n,
                                 int n_pad, void *X, void *stream)
{
  if (!mesh_ok (mesh, "mlp_features")) return DRB_ERR_INVALID_ARG;
  if (n < 0 || n_pad < n || (n_pad > 0 && !X) || (n > 0 && (!elem || !pts)))
  {
    set_last_error ("mlp_features: bad arguments (n <= n_pad)");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_pad == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int o = mesh->order;
  return o == 1 ? features_p<1> (mesh, elem, pts, n, n_pad, X, s)
         : o == 2 ? features_p<2> (mesh, elem, pts, n, n_pad, X, s)
                  : features_p<3> (mesh, elem, pts, n, n_pad, X, s);
}

// Workspace of one training step over n_pad rows (multiple of 128):
// Z1, Z2 fp32 [n_pad x 128]; H1, H2, dZ2, dZ1 bf16 [n_pad x 128];
// transposes dZ2T, H1T, dZ1T bf16 [128 x n_pad], XT bf16 [kInPad x n_pad].
extern "C" long long drb_mlp_workspace_bytes (int order, int n_pad)
{
  if (!mlp_order_ok (order) || n_pad < 0) return -1;
  return order == 1 ? workspace_p<1> (n_pad) : order == 2 ? workspace_p<2> (n_pad)
                                                          : workspace_p<3> (n_pad);
}

extern "C" int drb_mlp_forward (int order, const float *params, const void *wbf16, const void *X,
                                int n, int n_pad, float *y, void *workspace, int *err,
                                void *stream)
{
  if (!mlp_order_ok (order)) return DRB_ERR_INVALID_ARG;
  if (!params || !wbf16 || !X || !y || !workspace || n < 0 || n_pad < n || (n_pad % 128))
  {
    set_last_error ("mlp_forward: bad arguments (n_pad must be a multiple of 128 and >= n)");
    return DRB_ERR_INVALID_ARG;
  }
  if (n_pad == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return order == 1 ? forward_p<1> (params, wbf16, X, n, n_pad, y, workspace, err, s)
         : order == 2 ? forward_p<2> (params, wbf16, X, n, n_pad, y, workspace, err, s)
                      : forward_p<3> (params, wbf16, X, n, n_pad, y, workspace, err, s);
}

extern "C" int drb_mlp_train_step (int order, const float *params, const void *wbf16, const void *X,
                                   const float *target, const float *weight, int n, int n_pad,
                                   float *grad, float *loss, void *workspace, int *err,
                                   void *stream)
{
  if (!mlp_order_ok (order)) return DRB_ERR_INVALID_ARG;
  if (!params || !wbf16 || !X || !target || !grad || !workspace || n < 1 || n_pad < n ||
      (n_pad % 128))
  {
    set_last_error ("mlp_train_step: bad arguments (n_pad must be a multiple of 128 and >= n)");
    return DRB_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  return order == 1 ? train_step_p<1> (params, wbf16, X, target, weight, n, n_pad, grad, loss,
                                       workspace, err, s)
         : order == 2 ? train_step_p<2> (params, wbf16, X, target, weight, n, n_pad, grad, loss,
                                         workspace, err, s)
                      : train_step_p<3> (params, wbf16, X, target, weight, n, n_pad, grad, loss,
                                         workspace, err, s);
}

extern "C" int drb_mlp_adam (int order, float *params, const float *grad, float *m, float *v,
                             float lr, float beta1, float beta2, float eps, int step, void *stream)
{
  if (!mlp_order_ok (order)) return DRB_ERR_INVALID_ARG;
  if (!params || !grad || !m || !v || step < 1)
  {
    set_last_error ("mlp_adam: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  const int np = drb_mlp_param_count (order);
  const float c1 = 1.f / (1.f - powf (beta1, (float)step));
  const float c2 = 1.f / (1.f - powf (beta2, (float)step));
  adam_kernel<<<div_up (np, 256), 256, 0, (cudaStream_t)stream>>> (params, grad, m, v, np, lr, beta1,
                                                                   beta2, eps, c1, c2);
  return check_launch ("adam_kernel");
}

extern "C" int drb_mlp_guess (const float *params, const void *wbf16, const drb_mesh *mesh,
                              const int *elem, const float *pts, const int *order, int n,
                              float *guess, int *err, void *stream)
{
  if (!mesh_ok (mesh, "mlp_guess")) return DRB_ERR_INVALID_ARG;
  if (!params || !wbf16 || n < 0 || (n > 0 && (!elem || !pts || !guess)))
  {
    set_last_error ("mlp_guess: bad arguments");
    return DRB_ERR_INVALID_ARG;
  }
  if (n == 0) return DRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int o = mesh->order;
  return o == 1 ? guess_p<1> (params, wbf16, mesh, elem, pts, order, n, guess, err, s)
         : o == 2 ? guess_p<2> (params, wbf16, mesh, elem, pts, order, n, guess, err, s)
                  : guess_p<3> (params, wbf16, mesh, elem, pts, order, n, guess, err, s);
}
