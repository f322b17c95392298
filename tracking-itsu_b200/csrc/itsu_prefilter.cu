// itsu_prefilter.cu - the learned prefilter's training-side kernels: sample export, scoring,
// minibatch gradients and the Adam step.
//
// Inference lives in the cell stage (k_cells_prefilter, itsu_kernels.cu: each cell entry's
// features, the three layers and the threshold in one pass, no feature rows in memory); the
// scorer here runs the same device code (pair_features, mlp_logits_warp) on exported feature
// rows, so that the two give the same logit for the same pair. Training is binary cross-entropy on the sigmoid output with
// the forward pass exactly as inference computes it (BF16 inputs, weights and activations, FP32
// accumulation) and the backward pass on the tensor cores too: the gradients with respect to the
// pre-activations are rounded to BF16 for the three backward MMAs (dW2, dh1, dW1), accumulated in
// FP32, and applied to FP32 master weights (the BF16 rounding of the forward pass is passed
// straight through).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "itsu_device.cuh"
#include "itsu_internal.h"
#include "itsu_mlp.cuh"

namespace itsu {
namespace {

constexpr int kTrainWarps = 4;
constexpr int kMaxGradBlocks = 64;  // per-block gradient partials the Adam step reduces

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// ---- publish: FP32 master -> device model ----

// The FP32 master of an 8 -> H -> H -> 1 network (itsu_prefilter_model / itsu_gate_model): the
// trainable parameters in MlpShape<H> order, then mean[8], inv_std[8] and the logit threshold.
template <int H>
__device__ __forceinline__ void publish_param(MlpDeviceT<H> *model, int i, float w)
{
  using S = MlpShape<H>;
  if (i < S::kOffB1) {
    model->w1[i / kMlpIn][i % kMlpIn] = __float2bfloat16_rn(w);
  } else if (i < S::kOffW2) {
    model->b1[i - S::kOffB1] = w;
  } else if (i < S::kOffB2) {
    model->w2[(i - S::kOffW2) / H][(i - S::kOffW2) % H] = __float2bfloat16_rn(w);
  } else if (i < S::kOffW3) {
    model->b2[i - S::kOffB2] = w;
  } else if (i < S::kOffB3) {
    model->w3[i - S::kOffW3] = __float2bfloat16_rn(w);
  } else {
    model->b3 = w;
  }
}

// window: the gate's per-layer |dphi| window in the master (null for the pair prefilter: pi).
template <int H>
__global__ void k_mlp_publish(const float *master, const float *window, const float *dz_window, const int32_t *mlp_layers,
                              MlpDeviceT<H> *model)
{
  constexpr int P = MlpShape<H>::kParams;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    publish_param<H>(model, i, master[i]);
  }
  for (int i = threadIdx.x; i < kMlpIn; i += blockDim.x) {
    model->mean[i] = master[P + i];
    model->inv_std[i] = master[P + kMlpIn + i];
  }
  for (int i = threadIdx.x; i < 6; i += blockDim.x) {
    model->window[i] = window ? window[i] : 3.14159265358979323846f;
    model->dz_window[i] = dz_window ? dz_window[i] : HUGE_VALF;
  }
  if (threadIdx.x == 0) {
    model->threshold = master[P + 2 * kMlpIn];
    model->mlp_layers = mlp_layers ? (uint32_t)*mlp_layers : 0x3fu;
  }
}

// ---- export: one sample per cell, road membership and road keys ----

__global__ void k_export_cells(Arena a, itsu_prefilter_samples out)
{
  const int64_t n = a.status->total[kCells];
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    if (out.labels) {
      out.labels[c] = 0;
    }
    if (!out.features) {
      continue;
    }
    const int sid = a.cell_seg_id[c];
    const int e = sid / ITSU_CELL_LAYERS, layer = sid % ITSU_CELL_LAYERS;
    const itsu_cell cell = a.cells[c];
    const int32_t *ts = a.trk_seg + e * ITSU_TRACKLET_LAYERS;
    const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
    const itsu_tracklet t1 = a.tracklets[ts[layer] + cell.first_tracklet];
    const itsu_tracklet t2 = a.tracklets[ts[layer + 1] + cell.second_tracklet];
    const float4 c1 = a.xyzr[lo[layer] + cell.first_cluster];
    const float4 c2 = a.xyzr[lo[layer + 1] + cell.second_cluster];
    const float4 c3 = a.xyzr[lo[layer + 2] + cell.third_cluster];
    const float vx = a.vtx[3 * e], vy = a.vtx[3 * e + 1], vz = a.vtx[3 * e + 2];
    float3 normal;
    float curvature, dca;
    cell_geometry(layer, c1, c2, c3, vx, vy, normal, curvature, dca);
    float f[kMlpIn];
    pair_features(layer, t1.tan_lambda, t1.phi, t2.tan_lambda, t2.phi, c1, c2, c3, vx, vy, vz, dca, f);
    float4 *dst = reinterpret_cast<float4 *>(out.features + c * kMlpIn);
    dst[0] = make_float4(f[0], f[1], f[2], f[3]);
    dst[1] = make_float4(f[4], f[5], f[6], f[7]);
  }
}

__global__ void k_export_roads(Arena a, itsu_prefilter_samples out)
{
  const int64_t n = a.status->total[kRoads];
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    // event of the road: last e with road_seg[e] <= r
    int lo_e = 0, hi_e = a.n_events - 1;
    while (lo_e < hi_e) {
      const int mid = (lo_e + hi_e + 1) >> 1;
      if (a.road_seg[mid] <= r) {
        lo_e = mid;
      } else {
        hi_e = mid - 1;
      }
    }
    const int e = lo_e;
    const itsu_road road = a.roads[r];
    const int32_t *cs = a.cell_seg + e * ITSU_CELL_LAYERS;
    int32_t key[ITSU_LAYERS];
    for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
      const int64_t gc = cs[l] + road.cell_ids[l];
      if (out.labels) {
        out.labels[gc] = 1;
      }
      if (out.road_cells) {
        out.road_cells[r * ITSU_CELL_LAYERS + l] = (int32_t)gc;
      }
      const itsu_cell cell = a.cells[gc];
      if (l == 0) {
        key[0] = cell.first_cluster;
        key[1] = cell.second_cluster;
      }
      key[l + 2] = cell.third_cluster;
    }
    if (out.road_keys) {
      int32_t *k = out.road_keys + r * 8;
      k[0] = e;
      for (int l = 0; l < ITSU_LAYERS; ++l) {
        k[l + 1] = key[l];
      }
    }
    if (out.road_fake) {
      out.road_fake[r] = road.is_fake;
    }
  }
}

// ---- gate export: one sample per tracklet, on-road labels ----

__global__ void k_export_tracklets(Arena a, itsu_gate_samples out)
{
  const int64_t n = a.status->total[kTracklets];
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    if (out.labels) {
      out.labels[k] = 0;
    }
    if (!out.features) {
      continue;
    }
    const int sid = a.trk_seg_id[k];
    const int e = sid / ITSU_TRACKLET_LAYERS, layer = sid % ITSU_TRACKLET_LAYERS;
    const itsu_tracklet t = a.tracklets[k];
    const int32_t *lo = a.layer_off + e * ITSU_LAYERS;
    const int64_t i1 = lo[layer] + t.first_cluster, i2 = lo[layer + 1] + t.second_cluster;
    float f[kMlpIn];
    tracklet_features(layer, a.xyzr[i1], a.phi[i1], a.xyzr[i2], a.phi[i2], a.vtx[3 * e], a.vtx[3 * e + 1], a.vtx[3 * e + 2], f);
    float4 *dst = reinterpret_cast<float4 *>(out.features + k * kMlpIn);
    dst[0] = make_float4(f[0], f[1], f[2], f[3]);
    dst[1] = make_float4(f[4], f[5], f[6], f[7]);
  }
}

// Marks the two tracklets of every cell of every road (after k_export_tracklets cleared them) and
// lists each road's tracklets, layers 0..5 (-1 where the road has no cell).
__global__ void k_export_tracklet_labels(Arena a, itsu_gate_samples out)
{
  const int64_t n = a.status->total[kRoads];
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    int lo_e = 0, hi_e = a.n_events - 1;  // the road's event: last e with road_seg[e] <= r
    while (lo_e < hi_e) {
      const int mid = (lo_e + hi_e + 1) >> 1;
      if (a.road_seg[mid] <= r) {
        lo_e = mid;
      } else {
        hi_e = mid - 1;
      }
    }
    const itsu_road road = a.roads[r];
    const int32_t *cs = a.cell_seg + lo_e * ITSU_CELL_LAYERS;
    const int32_t *ts = a.trk_seg + lo_e * ITSU_TRACKLET_LAYERS;
    int32_t rows[ITSU_TRACKLET_LAYERS];
    for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
      rows[l] = -1;
    }
    for (int l = 0; l < ITSU_CELL_LAYERS; ++l) {
      if (road.cell_ids[l] < 0) {
        continue;
      }
      const itsu_cell cell = a.cells[cs[l] + road.cell_ids[l]];
      rows[l] = ts[l] + cell.first_tracklet;
      rows[l + 1] = ts[l + 1] + cell.second_tracklet;
    }
    for (int l = 0; l < ITSU_TRACKLET_LAYERS; ++l) {
      if (out.labels && rows[l] >= 0) {
        out.labels[rows[l]] = 1;
      }
      if (out.road_tracklets) {
        out.road_tracklets[r * ITSU_TRACKLET_LAYERS + l] = rows[l];
      }
    }
  }
}

// ---- scoring ----

constexpr int kScoreThreads = 256;

template <int H, bool kRelu>
__global__ void __launch_bounds__(kScoreThreads) k_mlp_score(const MlpDeviceT<H> *model, const float *features, int64_t n,
                                                            float *logits)
{
  __shared__ MlpSmemT<H> mlp;
  __shared__ __align__(16) __nv_bfloat16 rows[kScoreThreads / 32][32][kRowPitch];
  load_mlp(mlp, *model);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t tiles = (n + 31) / 32;
  for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; tile < tiles; tile += (int64_t)gridDim.x * (blockDim.x >> 5)) {
    const int64_t row = tile * 32 + lane;
    float f[kMlpIn];
    for (int k = 0; k < kMlpIn; ++k) {
      f[k] = row < n ? features[row * kMlpIn + k] : mlp.mean[k];
    }
    feature_row(mlp.mean, mlp.inv_std, f, rows[warp][lane]);
    __syncwarp();
    const float logit = mlp_logits_warp<false, H, kRelu>(mlp, rows[warp], nullptr);
    if (row < n) {
      logits[row] = logit;
    }
    __syncwarp();
  }
}

// ---- training: minibatch gradient ----

// One warp's 32-sample tile of the training pass of an 8 -> H -> H -> 1 network.
template <int H>
struct TrainWarp {
  static constexpr int kPitch = MlpShape<H>::kHidPitch;
  __nv_bfloat16 x[32][kRowPitch];     // standardised inputs [sample][feature] (A of layer 1)
  __nv_bfloat16 xt[8][kSmpPitch];     // the same, [feature][sample] (B of dW1)
  float a1[32][H + 1];                // layer-1 pre-activations, then dL/da1
  float a2[32][H + 1];                // layer-2 pre-activations, then dL/da2
  __nv_bfloat16 h1t[H][kSmpPitch];    // layer-1 activations [unit][sample] (B of dW2)
  __nv_bfloat16 d2[32][kPitch];       // dL/da2 [sample][unit] (A of dh1)
  __nv_bfloat16 d2t[H][kSmpPitch];    // dL/da2 [unit][sample] (A of dW2)
  __nv_bfloat16 d1t[H][kSmpPitch];    // dL/da1 [unit][sample] (A of dW1)
  float dz[32];                       // dL/dlogit
};

template <int H>
struct __align__(16) TrainBlock {
  MlpSmemT<H> mlp;
  __nv_bfloat16 w2t[H][MlpShape<H>::kHidPitch];  // W2 transposed [in][out] (B of dh1)
  float grad[MlpShape<H>::kParams];
  TrainWarp<H> warps[kTrainWarps];
};

template <int H, bool kRelu>
__global__ void __launch_bounds__(kTrainWarps * 32) k_mlp_gradient(const MlpDeviceT<H> *model, const float *features,
                                                                   const uint8_t *labels, int64_t n, int32_t batch,
                                                                   int32_t sequential, uint64_t seed, int64_t step,
                                                                   float pos_weight, float *grad_partials, float *loss)
{
  using S = MlpShape<H>;
  constexpr int NT = H / 8, KT = H / 16, P = S::kHidPitch;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainBlock<H> &B = *reinterpret_cast<TrainBlock<H> *>(smem_raw);
  load_mlp(B.mlp, *model);
  for (int i = threadIdx.x; i < H * P; i += blockDim.x) {
    const int r = i / P, c = i % P;
    B.w2t[r][c] = c < H ? model->w2[c][r] : __float2bfloat16_rn(0.0f);
  }
  for (int i = threadIdx.x; i < S::kParams; i += blockDim.x) {
    B.grad[i] = 0.0f;
  }
  __syncthreads();
  const MlpSmemT<H> &M = B.mlp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  TrainWarp<H> &W = B.warps[warp];
  const float inv_batch = 1.0f / (float)batch;
  const int64_t tiles = (batch + 31) / 32;
  for (int64_t tile = (int64_t)blockIdx.x * kTrainWarps + warp; tile < tiles; tile += (int64_t)gridDim.x * kTrainWarps) {
    // 1. the tile's samples
    const int64_t k = tile * 32 + lane;
    const bool valid = k < batch;
    float f[kMlpIn];
    float y = 0.0f;
    if (valid) {
      const int64_t idx = sequential ? k : (int64_t)(splitmix64(seed + (uint64_t)step * 0x632BE59BD9B4E019ull + (uint64_t)k) % (uint64_t)n);
      const float4 *src = reinterpret_cast<const float4 *>(features + idx * kMlpIn);
      const float4 u = src[0], v = src[1];
      f[0] = u.x, f[1] = u.y, f[2] = u.z, f[3] = u.w, f[4] = v.x, f[5] = v.y, f[6] = v.z, f[7] = v.w;
      y = labels[idx] ? 1.0f : 0.0f;
    } else {
      for (int q = 0; q < kMlpIn; ++q) {
        f[q] = M.mean[q];
      }
    }
    feature_row(M.mean, M.inv_std, f, W.x[lane]);
    for (int q = 0; q < kMlpIn; ++q) {
      W.xt[q][lane] = W.x[lane][q];
    }
    __syncwarp();
    // 2. forward, keeping the pre-activations and the layer-1 activations
    const MlpTraceT<H> trace{W.a1, W.a2, W.h1t};
    const float z = mlp_logits_warp<true, H, kRelu>(M, W.x, &trace);
    // 3. loss and dL/dz: weighted binary cross-entropy of sigmoid(z), averaged over the batch
    const float wgt = valid ? (y > 0.0f ? pos_weight : 1.0f) : 0.0f;
    const float prob = 1.0f / (1.0f + expf(-z));
    W.dz[lane] = wgt * (prob - y) * inv_batch;
    float l = wgt * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)))) * inv_batch;
    float dzsum = W.dz[lane];
    for (int o = 16; o > 0; o >>= 1) {
      l += __shfl_xor_sync(0xffffffffu, l, o);
      dzsum += __shfl_xor_sync(0xffffffffu, dzsum, o);
    }
    if (lane == 0) {
      atomicAdd(loss, l);
      atomicAdd(&B.grad[S::kOffB3], dzsum);
    }
    __syncwarp();
    // 4. dW3 (lane owns units lane and lane + 32)
    for (int jj = lane; jj < H; jj += 32) {
      float acc = 0.0f;
      for (int s2 = 0; s2 < 32; ++s2) {
        acc += W.dz[s2] * bf16r(act<kRelu>(W.a2[s2][jj]));
      }
      atomicAdd(&B.grad[S::kOffW3 + jj], acc);
    }
    __syncwarp();
    // 5. dL/da2 (lane owns sample lane)
    {
      const float dz = W.dz[lane];
      for (int j = 0; j < H; ++j) {
        const float d = dz * __bfloat162float(M.w3[0][j]) * act_grad<kRelu>(W.a2[lane][j]);
        W.a2[lane][j] = d;
        const __nv_bfloat16 db = __float2bfloat16_rn(d);
        W.d2[lane][j] = db;
        W.d2t[j][lane] = db;
      }
    }
    __syncwarp();
    for (int jj = lane; jj < H; jj += 32) {
      float acc = 0.0f;
      for (int s2 = 0; s2 < 32; ++s2) {
        acc += W.a2[s2][jj];
      }
      atomicAdd(&B.grad[S::kOffB2 + jj], acc);
    }
    // 6. dW2 = dL/da2^T h1: [H j x 32 s] x [32 s x H i]
    for (int mt = 0; mt < KT; ++mt) {
      float acc[NT][4];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
      }
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        uint32_t a[4];
        a[0] = ld32(&W.d2t[16 * mt + g][16 * kk + 2 * t]);
        a[1] = ld32(&W.d2t[16 * mt + g + 8][16 * kk + 2 * t]);
        a[2] = ld32(&W.d2t[16 * mt + g][16 * kk + 2 * t + 8]);
        a[3] = ld32(&W.d2t[16 * mt + g + 8][16 * kk + 2 * t + 8]);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          mma_bf16(acc[nt], a, ld32(&W.h1t[nt * 8 + g][16 * kk + 2 * t]), ld32(&W.h1t[nt * 8 + g][16 * kk + 2 * t + 8]));
        }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        float *row0 = &B.grad[S::kOffW2 + (16 * mt + g) * H + nt * 8 + 2 * t];
        float *row1 = row0 + 8 * H;
        atomicAdd(row0, acc[nt][0]);
        atomicAdd(row0 + 1, acc[nt][1]);
        atomicAdd(row1, acc[nt][2]);
        atomicAdd(row1 + 1, acc[nt][3]);
      }
    }
    // 7. dL/da1 = (dL/da2 W2) * act'(a1): [32 s x H j] x [H j x H i]
    for (int mt = 0; mt < 2; ++mt) {
      float acc[NT][4];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
      }
#pragma unroll
      for (int kk = 0; kk < KT; ++kk) {
        uint32_t a[4];
        a[0] = ld32(&W.d2[16 * mt + g][16 * kk + 2 * t]);
        a[1] = ld32(&W.d2[16 * mt + g + 8][16 * kk + 2 * t]);
        a[2] = ld32(&W.d2[16 * mt + g][16 * kk + 2 * t + 8]);
        a[3] = ld32(&W.d2[16 * mt + g + 8][16 * kk + 2 * t + 8]);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          mma_bf16(acc[nt], a, ld32(&B.w2t[nt * 8 + g][16 * kk + 2 * t]), ld32(&B.w2t[nt * 8 + g][16 * kk + 2 * t + 8]));
        }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int s2 = 16 * mt + g + (q >> 1) * 8, i = nt * 8 + 2 * t + (q & 1);
          const float d = acc[nt][q] * act_grad<kRelu>(W.a1[s2][i]);
          W.a1[s2][i] = d;
          W.d1t[i][s2] = __float2bfloat16_rn(d);
        }
      }
    }
    __syncwarp();
    for (int jj = lane; jj < H; jj += 32) {
      float acc = 0.0f;
      for (int s2 = 0; s2 < 32; ++s2) {
        acc += W.a1[s2][jj];
      }
      atomicAdd(&B.grad[S::kOffB1 + jj], acc);
    }
    // 8. dW1 = dL/da1^T x: [H i x 32 s] x [32 s x 8 f]
    for (int mt = 0; mt < KT; ++mt) {
      float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        uint32_t a[4];
        a[0] = ld32(&W.d1t[16 * mt + g][16 * kk + 2 * t]);
        a[1] = ld32(&W.d1t[16 * mt + g + 8][16 * kk + 2 * t]);
        a[2] = ld32(&W.d1t[16 * mt + g][16 * kk + 2 * t + 8]);
        a[3] = ld32(&W.d1t[16 * mt + g + 8][16 * kk + 2 * t + 8]);
        mma_bf16(acc, a, ld32(&W.xt[g][16 * kk + 2 * t]), ld32(&W.xt[g][16 * kk + 2 * t + 8]));
      }
      float *row0 = &B.grad[S::kOffW1 + (16 * mt + g) * kMlpIn + 2 * t];
      float *row1 = row0 + 8 * kMlpIn;
      atomicAdd(row0, acc[0]);
      atomicAdd(row0 + 1, acc[1]);
      atomicAdd(row1, acc[2]);
      atomicAdd(row1 + 1, acc[3]);
    }
    __syncwarp();
  }
  __syncthreads();
  float *out = grad_partials + (int64_t)blockIdx.x * S::kParams;
  for (int i = threadIdx.x; i < S::kParams; i += blockDim.x) {
    out[i] = B.grad[i];
  }
}

// ---- Adam ----

template <int H>
__global__ void k_mlp_adam(float *master, const float *grad_partials, int blocks, float *m, float *v, float lr, float beta1,
                           float beta2, float eps, float weight_decay, float bias1, float bias2, MlpDeviceT<H> *model)
{
  using S = MlpShape<H>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S::kParams) {
    return;
  }
  float gsum = 0.0f;
  for (int b = 0; b < blocks; ++b) {
    gsum += grad_partials[(int64_t)b * S::kParams + i];
  }
  const float mm = beta1 * m[i] + (1.0f - beta1) * gsum;
  const float vv = beta2 * v[i] + (1.0f - beta2) * gsum * gsum;
  m[i] = mm;
  v[i] = vv;
  float w = master[i];
  const bool is_weight = i < S::kOffB1 || (i >= S::kOffW2 && i < S::kOffB2) || (i >= S::kOffW3 && i < S::kOffB3);
  if (is_weight) {
    w -= lr * weight_decay * w;
  }
  w -= lr * (mm / bias1) / (sqrtf(vv / bias2) + eps);
  master[i] = w;
  publish_param<H>(model, i, w);
}

int gradient_blocks(int32_t batch)
{
  const int64_t tiles = ((int64_t)batch + 31) / 32;
  const int64_t blocks = (tiles + kTrainWarps - 1) / kTrainWarps;
  return (int)(blocks < kMaxGradBlocks ? (blocks > 0 ? blocks : 1) : kMaxGradBlocks);
}

}  // namespace

namespace {

template <int H, bool kRelu>
void score_net(const MlpDeviceT<H> *model, const float *features, int64_t n, float *logits, int num_sms, cudaStream_t stream)
{
  const int64_t tiles = (n + 31) / 32;
  int64_t blocks = (tiles + kScoreThreads / 32 - 1) / (kScoreThreads / 32);
  if (blocks > (int64_t)num_sms * 8) {
    blocks = (int64_t)num_sms * 8;
  }
  if (blocks > 0) {
    k_mlp_score<H, kRelu><<<(unsigned)blocks, kScoreThreads, 0, stream>>>(model, features, n, logits);
  }
}

template <int H, bool kRelu>
void gradient_net(const MlpDeviceT<H> *model, const float *features, const uint8_t *labels, int64_t n, int32_t batch, bool sequential,
                  uint64_t seed, int64_t step, float pos_weight, float *grad_partials, float *loss, cudaStream_t stream)
{
  // per device and cheap: set before every launch (training runs outside graph capture)
  cudaFuncSetAttribute(k_mlp_gradient<H, kRelu>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainBlock<H>));
  k_mlp_gradient<H, kRelu><<<gradient_blocks(batch), kTrainWarps * 32, sizeof(TrainBlock<H>), stream>>>(
      model, features, labels, n, batch, sequential ? 1 : 0, seed, step, pos_weight, grad_partials, loss);
}

}  // namespace

static_assert(sizeof(itsu_prefilter_model) == sizeof(float) * (kMlpParams + 2 * kMlpIn + 1), "pair model layout");
static_assert(sizeof(itsu_gate_model) == sizeof(float) * (kGateParams + 2 * kMlpIn + 1 + 2 * ITSU_TRACKLET_LAYERS + 1), "gate model layout");

size_t mlp_device_bytes() { return sizeof(MlpDevice); }
size_t gate_device_bytes() { return sizeof(GateDevice); }
int mlp_gradient_blocks(int32_t batch) { return gradient_blocks(batch); }
int mlp_max_gradient_blocks() { return kMaxGradBlocks; }

void launch_mlp_publish(const itsu_prefilter_model *master, MlpDevice *model, cudaStream_t stream)
{
  k_mlp_publish<kMlpHidden><<<1, 512, 0, stream>>>(&master->w1[0][0], nullptr, nullptr, nullptr, model);
}

void launch_mlp_publish(const itsu_gate_model *master, GateDevice *model, cudaStream_t stream)
{
  k_mlp_publish<kGateHidden><<<1, 512, 0, stream>>>(&master->w1[0][0], &master->dphi_window[0], &master->dz_window[0],
                                                     &master->mlp_layers, model);
}

void launch_prefilter_export(const Arena &a, const itsu_prefilter_samples &out, int num_sms, cudaStream_t stream)
{
  k_export_cells<<<num_sms * 8, 256, 0, stream>>>(a, out);
  k_export_roads<<<num_sms * 4, 256, 0, stream>>>(a, out);
}

void launch_gate_export(const Arena &a, const itsu_gate_samples &out, int num_sms, cudaStream_t stream)
{
  k_export_tracklets<<<num_sms * 8, 256, 0, stream>>>(a, out);
  if (out.labels || out.road_tracklets) {
    k_export_tracklet_labels<<<num_sms * 4, 256, 0, stream>>>(a, out);
  }
}

void launch_mlp_score(const MlpDevice *model, const float *features, int64_t n, float *logits, int num_sms, cudaStream_t stream)
{
  score_net<kMlpHidden, false>(model, features, n, logits, num_sms, stream);
}

void launch_mlp_score(const GateDevice *model, const float *features, int64_t n, float *logits, int num_sms, cudaStream_t stream)
{
  score_net<kGateHidden, true>(model, features, n, logits, num_sms, stream);
}

void launch_mlp_gradient(const MlpDevice *model, const float *features, const uint8_t *labels, int64_t n, int32_t batch,
                         bool sequential, uint64_t seed, int64_t step, float pos_weight, float *grad_partials, float *loss,
                         cudaStream_t stream)
{
  gradient_net<kMlpHidden, false>(model, features, labels, n, batch, sequential, seed, step, pos_weight, grad_partials, loss, stream);
}

void launch_mlp_gradient(const GateDevice *model, const float *features, const uint8_t *labels, int64_t n, int32_t batch,
                         bool sequential, uint64_t seed, int64_t step, float pos_weight, float *grad_partials, float *loss,
                         cudaStream_t stream)
{
  gradient_net<kGateHidden, true>(model, features, labels, n, batch, sequential, seed, step, pos_weight, grad_partials, loss, stream);
}

void launch_mlp_adam(itsu_prefilter_model *master, const float *grad_partials, int blocks, float *m, float *v, float lr,
                     float beta1, float beta2, float eps, float weight_decay, float bias1, float bias2, MlpDevice *model,
                     cudaStream_t stream)
{
  k_mlp_adam<kMlpHidden><<<(kMlpParams + 255) / 256, 256, 0, stream>>>(&master->w1[0][0], grad_partials, blocks, m, v, lr,
                                                                       beta1, beta2, eps, weight_decay, bias1, bias2, model);
}

void launch_mlp_adam(itsu_gate_model *master, const float *grad_partials, int blocks, float *m, float *v, float lr, float beta1,
                     float beta2, float eps, float weight_decay, float bias1, float bias2, GateDevice *model, cudaStream_t stream)
{
  k_mlp_adam<kGateHidden><<<(kGateParams + 255) / 256, 256, 0, stream>>>(&master->w1[0][0], grad_partials, blocks, m, v, lr,
                                                                         beta1, beta2, eps, weight_decay, bias1, bias2, model);
}

}  // namespace itsu
