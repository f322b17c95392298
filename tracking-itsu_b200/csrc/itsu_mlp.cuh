// itsu_mlp.cuh - the learned tracklet-pair prefilter: pair features and the 8-64-64-1 MLP.
//
// The prefilter scores the tracklet pairs that pass the cell cuts of Tracker.cxx:161-216 before
// they become cells; a pair is dropped when its logit is below the model's threshold. Its 8
// features are the pair's dphi, dz and dtanL (the cut variables of Tracker.cxx:161-171), the
// curvature of each tracklet's circle through the primary vertex (the reference Tracklet,
// Tracklet.h:33-36, has none: this build defines them), the pair's DCA to the vertex (Tracker.cxx:
// 203-210), the inner layer index and the first cluster's radius. The network is 8 -> 64 -> 64 ->
// 1 with GELU (tanh form, Hendrycks & Gimpel 2016) and a sigmoid output, BF16 weights and
// activations, FP32 accumulation and biases. It runs on the tensor cores as warp MMAs
// (mma.sync m16n8k16, BF16 in, FP32 accumulate) over 32 pairs at a time; each layer's FP32
// accumulators are re-packed in registers as the next layer's BF16 A operand. Thresholding the
// logit is thresholding the sigmoid output at sigmoid(threshold).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace itsu {

constexpr int kMlpIn = 8;

// Parameter count and offsets of the trainable parameters of an 8 -> H -> H -> 1 network in its
// flat FP32 master array (w1 [H][8], b1, w2 [H][H], b2, w3 [H], b3: the C ABI model order).
template <int H>
struct MlpShape {
  static_assert(H % 16 == 0 && H >= 16 && H <= 64, "hidden width: whole 16-wide MMA tiles");
  static constexpr int kHidden = H;
  static constexpr int kParams = H * kMlpIn + H + H * H + H + H + 1;
  static constexpr int kOffW1 = 0;
  static constexpr int kOffB1 = kOffW1 + H * kMlpIn;
  static constexpr int kOffW2 = kOffB1 + H;
  static constexpr int kOffB2 = kOffW2 + H * H;
  static constexpr int kOffW3 = kOffB2 + H;
  static constexpr int kOffB3 = kOffW3 + H;
  // row pitch (BF16 elements) of the [out][in] W2 / W3 operands and of hidden-activation rows:
  // H + 8, so that the 8 rows one fragment load touches fall in distinct banks
  static constexpr int kHidPitch = H + 8;
};

// The pair prefilter's network (8 -> 64 -> 64 -> 1, GELU).
constexpr int kMlpHidden = 64;
constexpr int kMlpParams = MlpShape<kMlpHidden>::kParams;
constexpr int kOffW1 = MlpShape<kMlpHidden>::kOffW1;
constexpr int kOffB1 = MlpShape<kMlpHidden>::kOffB1;
constexpr int kOffW2 = MlpShape<kMlpHidden>::kOffW2;
constexpr int kOffB2 = MlpShape<kMlpHidden>::kOffB2;
constexpr int kOffW3 = MlpShape<kMlpHidden>::kOffW3;
constexpr int kOffB3 = MlpShape<kMlpHidden>::kOffB3;
static_assert(kOffB3 + 1 == kMlpParams, "parameter layout");
// The tracklet gate's network (8 -> 16 -> 16 -> 1, ReLU).
constexpr int kGateHidden = 16;
constexpr int kGateParams = MlpShape<kGateHidden>::kParams;

// Row pitches (in BF16 elements) of the shared-memory operands, padded so that the 8 rows one
// MMA fragment load touches fall in distinct banks.
constexpr int kRowPitch = 24;  // feature rows and W1 rows (16 used)
constexpr int kHidPitch = MlpShape<kMlpHidden>::kHidPitch;  // the pair network's W2 / W3 / hidden rows
constexpr int kSmpPitch = 40;  // transposed [unit][sample] operands (32 used)

// A network as the device keeps it in global memory.
template <int H>
struct MlpDeviceT {
  __nv_bfloat16 w1[H][kMlpIn];  // [out][in]
  __nv_bfloat16 w2[H][H];       // [out][in]
  __nv_bfloat16 w3[H];
  float b1[H];
  float b2[H];
  float b3;
  float threshold;
  float mean[kMlpIn];
  float inv_std[kMlpIn];
  float window[6];     // the tracklet gate's per-layer |dphi| window (the pair prefilter: pi, unused)
  float dz_window[6];  // and its |dz| window (the pair prefilter: infinity, unused)
  uint32_t mlp_layers; // the gate: bit l, the network scores inner layer l (the pair prefilter: unused)
};

// A network staged in shared memory in MMA-friendly, zero-padded form.
template <int H>
struct __align__(16) MlpSmemT {
  static constexpr int kPitch = MlpShape<H>::kHidPitch;
  __nv_bfloat16 w1[H][kRowPitch];  // columns 8.. are zero (the first MMA has K = 16)
  __nv_bfloat16 w2[H][kPitch];
  __nv_bfloat16 w3[8][kPitch];     // row 0 holds the output weights, rows 1..7 are zero (N = 8)
  float b1[H];
  float b2[H];
  float b3;
  float threshold;
  float mean[kMlpIn];
  float inv_std[kMlpIn];
  uint32_t layers;  // the gate: the inner layers the network scores (bit l)
};

using MlpSmem = MlpSmemT<kMlpHidden>;
using GateSmem = MlpSmemT<kGateHidden>;

// Block-cooperative copy of a network into shared memory (the caller synchronises the block).
template <int H>
__device__ __forceinline__ void load_mlp(MlpSmemT<H> &s, const MlpDeviceT<H> &g)
{
  constexpr int P = MlpSmemT<H>::kPitch;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  for (int i = threadIdx.x; i < H * kRowPitch; i += blockDim.x) {
    const int r = i / kRowPitch, c = i % kRowPitch;
    s.w1[r][c] = c < kMlpIn ? g.w1[r][c] : zero;
  }
  for (int i = threadIdx.x; i < H * P; i += blockDim.x) {
    const int r = i / P, c = i % P;
    s.w2[r][c] = c < H ? g.w2[r][c] : zero;
  }
  for (int i = threadIdx.x; i < 8 * P; i += blockDim.x) {
    const int r = i / P, c = i % P;
    s.w3[r][c] = (r == 0 && c < H) ? g.w3[c] : zero;
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.b1[i] = g.b1[i];
    s.b2[i] = g.b2[i];
  }
  for (int i = threadIdx.x; i < kMlpIn; i += blockDim.x) {
    s.mean[i] = g.mean[i];
    s.inv_std[i] = g.inv_std[i];
  }
  if (threadIdx.x == 0) {
    s.b3 = g.b3;
    s.threshold = g.threshold;
    s.layers = g.mlp_layers;
  }
}

constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float tanh_approx(float x)
{
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float gelu(float x)
{
  const float u = kGeluC * (x + kGeluA * (x * x * x));
  return 0.5f * x * (1.0f + tanh_approx(u));
}

__device__ __forceinline__ float gelu_grad(float x)
{
  const float x2 = x * x;
  const float th = tanh_approx(kGeluC * (x + kGeluA * (x2 * x)));
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * kGeluC * (1.0f + 3.0f * kGeluA * x2);
}

// Signed curvature (1/R) of the circle through three points of the transverse plane; 0 when
// they are collinear or coincide.
__device__ __forceinline__ float circle_curvature(float ax, float ay, float bx, float by, float cx, float cy)
{
  const float ux = bx - ax, uy = by - ay, vx = cx - ax, vy = cy - ay, wx = cx - bx, wy = cy - by;
  const float cross = ux * vy - uy * vx;
  const float d = sqrtf((ux * ux + uy * uy) * (vx * vx + vy * vy) * (wx * wx + wy * wy));
  return d > 0.0f ? 2.0f * cross / d : 0.0f;
}

// The 8 raw features of a pair (t1 from cluster c1 to c2, t2 from c2 to c3; c = (x, y, z, r)).
__device__ __forceinline__ void pair_features(int layer, float t1_tan_lambda, float t1_phi, float t2_tan_lambda, float t2_phi,
                                              float4 c1, float4 c2, float4 c3, float vx, float vy, float vz, float dca,
                                              float f[kMlpIn])
{
  const float delta_phi = fabsf(t1_phi - t2_phi);
  f[0] = fminf(delta_phi, fabsf(delta_phi - 6.28318530717958647692f));
  f[1] = fabsf(-(0.5f * (t1_tan_lambda + t2_tan_lambda)) * c1.w + c1.z - vz);
  f[2] = fabsf(t1_tan_lambda - t2_tan_lambda);
  f[3] = circle_curvature(vx, vy, c1.x, c1.y, c2.x, c2.y);
  f[4] = circle_curvature(vx, vy, c2.x, c2.y, c3.x, c3.y);
  f[5] = dca;
  f[6] = (float)layer;
  f[7] = c1.w;
}

// Standardised features as one BF16 row of the first MMA's A operand (columns 8..15 zero).
__device__ __forceinline__ void feature_row(const float *mean, const float *inv_std, const float f[kMlpIn],
                                            __nv_bfloat16 *row)
{
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) {
    row[k] = __float2bfloat16_rn((f[k] - mean[k]) * inv_std[k]);
  }
#pragma unroll
  for (int k = kMlpIn; k < 16; ++k) {
    row[k] = __float2bfloat16_rn(0.0f);
  }
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// D += A * B for one m16n8k16 tile (A row-major 16x16, B column-major 16x8, BF16; D FP32).
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Fragment layout of m16n8k16 (g = lane / 4, t = lane % 4): A registers hold (row g, k 2t..2t+1),
// (row g+8, k 2t..), (row g, k 2t+8..), (row g+8, k 2t+8..); B registers hold (k 2t..2t+1, col g)
// and (k 2t+8.., col g); D holds (row g, col 2t), (row g, col 2t+1), (row g+8, col 2t), (row g+8,
// col 2t+1).

// Hidden-layer activation: GELU (the pair prefilter) or ReLU (the tracklet gate, which scores
// every tracklet: its activation must be cheap).
template <bool kRelu>
__device__ __forceinline__ float act(float x)
{
  if constexpr (kRelu) {
    return fmaxf(x, 0.0f);
  } else {
    return gelu(x);
  }
}

template <bool kRelu>
__device__ __forceinline__ float act_grad(float x)
{
  if constexpr (kRelu) {
    return x > 0.0f ? 1.0f : 0.0f;
  } else {
    return gelu_grad(x);
  }
}

// Where the training pass keeps a 32-sample tile's intermediate values.
template <int H>
struct MlpTraceT {
  float (*a1)[H + 1];               // [sample][unit] layer-1 pre-activations
  float (*a2)[H + 1];               // [sample][unit] layer-2 pre-activations
  __nv_bfloat16 (*h1t)[kSmpPitch];  // [unit][sample] layer-1 activations (BF16, as the next MMA sees them)
};
using MlpTrace = MlpTraceT<kMlpHidden>;

// Forward pass of rows 16 mt .. 16 mt + 15 of a 32-row tile; returns the logits of rows g and
// g + 8 of the tile in lo / hi (valid in lanes with t == 0). All lanes of the warp take part.
template <bool kTrace, int H, bool kRelu>
__device__ __forceinline__ void mlp_forward_m16(const MlpSmemT<H> &m, const __nv_bfloat16 (*rows)[kRowPitch], int mt, float &lo,
                                                float &hi, const MlpTraceT<H> *trace)
{
  constexpr int NT = H / 8, KT = H / 16;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = mt * 16 + g, r1 = r0 + 8;
  uint32_t a[4];
  a[0] = ld32(&rows[r0][2 * t]);
  a[1] = ld32(&rows[r1][2 * t]);
  a[2] = ld32(&rows[r0][2 * t + 8]);
  a[3] = ld32(&rows[r1][2 * t + 8]);
  // layer 1: [16 x 16] x [16 x H] -> activation -> BF16 A fragments of layer 2 (hk[kk] covers k 16kk..)
  uint32_t hk[KT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma_bf16(c, a, ld32(&m.w1[nt * 8 + g][2 * t]), ld32(&m.w1[nt * 8 + g][2 * t + 8]));
    const int col = nt * 8 + 2 * t;
    c[0] += m.b1[col];
    c[1] += m.b1[col + 1];
    c[2] += m.b1[col];
    c[3] += m.b1[col + 1];
    const uint32_t top = pack_bf16(act<kRelu>(c[0]), act<kRelu>(c[1]));
    const uint32_t bottom = pack_bf16(act<kRelu>(c[2]), act<kRelu>(c[3]));
    hk[nt >> 1][(nt & 1) * 2 + 0] = top;
    hk[nt >> 1][(nt & 1) * 2 + 1] = bottom;
    if constexpr (kTrace) {
      trace->a1[r0][col] = c[0];
      trace->a1[r0][col + 1] = c[1];
      trace->a1[r1][col] = c[2];
      trace->a1[r1][col + 1] = c[3];
      const __nv_bfloat162 tv = *reinterpret_cast<const __nv_bfloat162 *>(&top);
      const __nv_bfloat162 bv = *reinterpret_cast<const __nv_bfloat162 *>(&bottom);
      trace->h1t[col][r0] = tv.x;
      trace->h1t[col + 1][r0] = tv.y;
      trace->h1t[col][r1] = bv.x;
      trace->h1t[col + 1][r1] = bv.y;
    }
  }
  // layer 2: [16 x H] x [H x H]
  float h2[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    h2[nt][0] = h2[nt][1] = h2[nt][2] = h2[nt][3] = 0.0f;
  }
#pragma unroll
  for (int kk = 0; kk < KT; ++kk) {
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      mma_bf16(h2[nt], hk[kk], ld32(&m.w2[nt * 8 + g][16 * kk + 2 * t]), ld32(&m.w2[nt * 8 + g][16 * kk + 2 * t + 8]));
    }
  }
  // layer 3: [16 x H] x [H x 8], column 0 real
  float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int kk = 0; kk < KT; ++kk) {
    uint32_t ak[4];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int nt = 2 * kk + half;
      const int col = nt * 8 + 2 * t;
      const float v0 = h2[nt][0] + m.b2[col], v1 = h2[nt][1] + m.b2[col + 1];
      const float v2 = h2[nt][2] + m.b2[col], v3 = h2[nt][3] + m.b2[col + 1];
      if constexpr (kTrace) {
        trace->a2[r0][col] = v0;
        trace->a2[r0][col + 1] = v1;
        trace->a2[r1][col] = v2;
        trace->a2[r1][col + 1] = v3;
      }
      ak[half * 2 + 0] = pack_bf16(act<kRelu>(v0), act<kRelu>(v1));
      ak[half * 2 + 1] = pack_bf16(act<kRelu>(v2), act<kRelu>(v3));
    }
    mma_bf16(o, ak, ld32(&m.w3[g][16 * kk + 2 * t]), ld32(&m.w3[g][16 * kk + 2 * t + 8]));
  }
  lo = o[0] + m.b3;
  hi = o[2] + m.b3;
}

template <class T>
struct NoDeduce {
  using type = T;
};

// Logits of the 32 rows of a tile; lane l gets row l's. All lanes of the warp take part.
template <bool kTrace, int H = kMlpHidden, bool kRelu = false>
__device__ __forceinline__ float mlp_logits_warp(const MlpSmemT<H> &m, const __nv_bfloat16 (*rows)[kRowPitch],
                                                 const typename NoDeduce<MlpTraceT<H>>::type *trace)
{
  const int lane = threadIdx.x & 31;
  float mine = 0.0f;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    float lo, hi;
    mlp_forward_m16<kTrace, H, kRelu>(m, rows, mt, lo, hi, trace);
    // row r of this m-tile sits in lane 4 (r mod 8), in lo for r < 8 and hi otherwise
    const int src = (lane & 7) << 2;
    lo = __shfl_sync(0xffffffffu, lo, src);
    hi = __shfl_sync(0xffffffffu, hi, src);
    if ((lane >> 4) == mt) {
      mine = (lane & 8) ? hi : lo;
    }
  }
  return mine;
}

// The tracklet gate's 8 raw features of the tracklet from inner cluster c1 to outer cluster c2
// (c = (x, y, z, r), phi the clusters' azimuths about the vertex, as the clustering computed
// them): |dphi| and dphi (wrapped to [-pi, pi]), the tracklet cut's dz (Tracker.cxx:93-95) and its
// absolute value, the signed curvature of the circle through the vertex and both clusters, the
// inner layer, the inner cluster's radius and its slope from the vertex. The gate scores every
// tracklet, so its features use the hardware's fast division and reciprocal square root
// (__fdividef, rsqrtf: a few units in the last place); the export and the gate pass run this same
// code, so training and inference see the same values. What depends on the inner cluster alone
// is computed once per inner cluster (GateInner).
struct GateInner {
  float ux, uy, uu;   // the inner cluster relative to the vertex, and its squared length
  float z1, r1, phi1;
  float tan_lambda;   // slope from the vertex
  float vx, vy;
  int layer;
};

__device__ __forceinline__ GateInner gate_inner(int layer, float4 c1, float phi1, float vx, float vy, float vz)
{
  GateInner g;
  g.ux = c1.x - vx;
  g.uy = c1.y - vy;
  g.uu = g.ux * g.ux + g.uy * g.uy;
  g.z1 = c1.z;
  g.r1 = c1.w;
  g.phi1 = phi1;
  g.tan_lambda = __fdividef(c1.z - vz, c1.w);
  g.vx = vx;
  g.vy = vy;
  g.layer = layer;
  return g;
}

__device__ __forceinline__ void gate_features(const GateInner &g, float4 c2, float phi2, float f[kMlpIn])
{
  constexpr float kPiF = 3.14159265358979323846f, kTwoPiF = 6.28318530717958647692f;
  float dphi = g.phi1 - phi2;
  dphi = dphi > kPiF ? dphi - kTwoPiF : (dphi < -kPiF ? dphi + kTwoPiF : dphi);
  const float dz = g.tan_lambda * (c2.w - g.r1) + g.z1 - c2.z;
  // curvature of the circle through the vertex and both clusters: 2 (u x w) / (|u| |w| |w - u|)
  const float wx = c2.x - g.vx, wy = c2.y - g.vy, dx = wx - g.ux, dy = wy - g.uy;
  const float prod = g.uu * (wx * wx + wy * wy) * (dx * dx + dy * dy);
  f[0] = fabsf(dphi);
  f[1] = dz;
  f[2] = fabsf(dz);
  f[3] = prod > 0.0f ? 2.0f * (g.ux * wy - g.uy * wx) * rsqrtf(prod) : 0.0f;
  f[4] = (float)g.layer;
  f[5] = g.r1;
  f[6] = g.tan_lambda;
  f[7] = dphi;
}

// The cascade's first stage for one inner cluster: its per-layer windows on |dphi| and |dz| (the
// gate's features 0 and 2, with the same arithmetic: the slope by the fast division of
// gate_inner).
struct GateWindow {
  float dphi, dz;
  float phi1, z1, r1, tan_lambda;
};

__device__ __forceinline__ GateWindow gate_window(const MlpDeviceT<kGateHidden> &m, int layer, float4 c1, float phi1, float vz)
{
  GateWindow w;
  w.dphi = m.window[layer];
  w.dz = m.dz_window[layer];
  w.phi1 = phi1;
  w.z1 = c1.z;
  w.r1 = c1.w;
  w.tan_lambda = __fdividef(c1.z - vz, c1.w);
  return w;
}

__device__ __forceinline__ bool gate_window_pass(const GateWindow &w, float4 c2, float phi2)
{
  constexpr float kPiF = 3.14159265358979323846f, kTwoPiF = 6.28318530717958647692f;
  float dphi = w.phi1 - phi2;
  dphi = dphi > kPiF ? dphi - kTwoPiF : (dphi < -kPiF ? dphi + kTwoPiF : dphi);
  const float dz = w.tan_lambda * (c2.w - w.r1) + w.z1 - c2.z;
  return fabsf(dphi) <= w.dphi && fabsf(dz) <= w.dz;
}

__device__ __forceinline__ void tracklet_features(int layer, float4 c1, float phi1, float4 c2, float phi2, float vx, float vy,
                                                  float vz, float f[kMlpIn])
{
  gate_features(gate_inner(layer, c1, phi1, vx, vy, vz), c2, phi2, f);
}

// The tracklet gate's network in registers: at 16 hidden units the whole network is 17 values
// per lane, each lane holding its MMA fragments and the biases of its output columns, so the gate
// pass reads no weights from memory per tile. The operands are those of mlp_forward_m16 (the k 8..15
// halves of layer 1's operands are zero there), so the logits are the same, bit for bit.
struct GateRegs {
  uint32_t w1[2];     // layer 1 B fragment (k 2t, 2t+1; column g) per n-tile
  uint32_t w2[2][2];  // layer 2 B fragments per n-tile
  uint32_t w3[2];     // layer 3 B fragments (column 0 real)
  float b1[2][2], b2[2][2];  // biases of the lane's output columns 2t, 2t+1 per n-tile
  float b3;
};

__device__ __forceinline__ GateRegs gate_regs(const MlpSmemT<kGateHidden> &m)
{
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  GateRegs r;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    r.w1[nt] = ld32(&m.w1[nt * 8 + g][2 * t]);
    r.w2[nt][0] = ld32(&m.w2[nt * 8 + g][2 * t]);
    r.w2[nt][1] = ld32(&m.w2[nt * 8 + g][2 * t + 8]);
    r.b1[nt][0] = m.b1[nt * 8 + 2 * t];
    r.b1[nt][1] = m.b1[nt * 8 + 2 * t + 1];
    r.b2[nt][0] = m.b2[nt * 8 + 2 * t];
    r.b2[nt][1] = m.b2[nt * 8 + 2 * t + 1];
  }
  r.w3[0] = ld32(&m.w3[g][2 * t]);
  r.w3[1] = ld32(&m.w3[g][2 * t + 8]);
  r.b3 = m.b3;
  return r;
}

// Logits of rows 16 mt + g (lo) and 16 mt + g + 8 (hi) of a 32-row tile whose rows hold the 8
// standardised BF16 features (valid in lanes with t == 0). All lanes of the warp take part.
__device__ __forceinline__ void gate_forward_m16(const GateRegs &R, const __nv_bfloat16 (*rows)[kMlpIn], int mt, float &lo,
                                                 float &hi)
{
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t a[4] = {ld32(&rows[mt * 16 + g][2 * t]), ld32(&rows[mt * 16 + g + 8][2 * t]), 0u, 0u};
  uint32_t hk[4];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    mma_bf16(c, a, R.w1[nt], 0u);
    hk[nt * 2 + 0] = pack_bf16(act<true>(c[0] + R.b1[nt][0]), act<true>(c[1] + R.b1[nt][1]));
    hk[nt * 2 + 1] = pack_bf16(act<true>(c[2] + R.b1[nt][0]), act<true>(c[3] + R.b1[nt][1]));
  }
  float h2[2][4];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    h2[nt][0] = h2[nt][1] = h2[nt][2] = h2[nt][3] = 0.0f;
    mma_bf16(h2[nt], hk, R.w2[nt][0], R.w2[nt][1]);
  }
  uint32_t ak[4];
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    ak[nt * 2 + 0] = pack_bf16(act<true>(h2[nt][0] + R.b2[nt][0]), act<true>(h2[nt][1] + R.b2[nt][1]));
    ak[nt * 2 + 1] = pack_bf16(act<true>(h2[nt][2] + R.b2[nt][0]), act<true>(h2[nt][3] + R.b2[nt][1]));
  }
  float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  mma_bf16(o, ak, R.w3[0], R.w3[1]);
  lo = o[0] + R.b3;
  hi = o[2] + R.b3;
}

// The 8 standardised BF16 features of one row (as feature_row rounds them), packed in 16 bytes.
__device__ __forceinline__ uint4 gate_row(const float *mean, const float *inv_std, const float f[kMlpIn])
{
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    w[k] = pack_bf16((f[2 * k] - mean[2 * k]) * inv_std[2 * k], (f[2 * k + 1] - mean[2 * k + 1]) * inv_std[2 * k + 1]);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

}  // namespace itsu
