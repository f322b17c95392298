// itsu_device.cuh - device-side arithmetic of the ITS CA track finder.
//
// Every expression below is the reference's, term for term and in the reference's evaluation
// order, in binary32. This translation unit is compiled with -fmad=false (no FMA contraction),
// IEEE division and square root (nvcc's defaults without --use_fast_math) and no flush-to-zero,
// which is exactly the arithmetic of the reference's x86-64 -O3 build. The azimuth uses the
// correctly rounded itsu_atan2f that the oracle also uses.
#pragma once

#include <cstdint>

#include "itsu.h"
#include "itsu_atan2f.h"

namespace itsu {

// ---- Constants (include/ITSReconstruction/CA/Constants.h:31-92) ----
constexpr float kPi = 3.14159265359f;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kFloatMinThreshold = 1e-20f;
constexpr int kZBins = 20;
constexpr int kPhiBins = 20;
constexpr int kTableBins = kZBins * kPhiBins;  // 400
constexpr int kTableSize = kTableBins + 1;     // 401
constexpr float kInversePhiBinSize = kPhiBins / kTwoPi;  // int / float: binary32 division
constexpr float kCellMaxDeltaTanLambda = 0.025f;
constexpr float kCellMaxDeltaPhi = 0.14f;
constexpr float kZCoordinateCut = 0.5f;
constexpr float kPhiCoordinateCut = 0.3f;
constexpr int kCellsMinLevel = 5;
// The wrap-around half of the reference's azimuth cuts, |delta_phi - 2pi| < cut in binary32, for a
// binary32 delta_phi = |phi1 - phi2| in [0, kTwoPi] (both azimuths normalised to [0, kTwoPi], or
// both atan2 results in [-pi, pi]): for delta_phi >= kPi the subtraction is exact (Sterbenz), so
// the test is delta_phi > kTwoPi - cut in real arithmetic, i.e. delta_phi greater than the largest
// binary32 value not above kTwoPi - cut; below kPi both forms are false. One compare instead of a
// subtraction and a compare; tests/test_phi_wrap.py checks every binary32 delta_phi in
// [kPi, kTwoPi] and a sample below.
constexpr float kPhiWrapTracklet = 0x1.7eec82p+2f;  // largest binary32 <= kTwoPi - kPhiCoordinateCut
constexpr float kPhiWrapCell = 0x1.8929f2p+2f;      // largest binary32 <= kTwoPi - kCellMaxDeltaPhi

struct LayerConstants {
  float z_half[7];           // LayersZCoordinate
  float r[7];                // LayersRCoordinate
  float inv_z_bin[7];        // InverseZBinSize: 0.5 * ZBins / Zhalf in double, stored as float
  float trk_max_dz[6];       // TrackletMaxDeltaZThreshold
  float cell_max_dz[5];      // CellMaxDeltaZThreshold
  float cell_max_dca[5];     // CellMaxDistanceOfClosestApproachThreshold
  float nb_max_normal[4];    // NeighbourCellMaxNormalVectorsDelta
  float nb_max_curv[4];      // NeighbourCellMaxCurvaturesDelta
};

__constant__ const LayerConstants kC = {
    {16.333f, 16.333f, 16.333f, 42.140f, 42.140f, 73.745f, 73.745f},
    {2.33959f, 3.14076f, 3.91924f, 19.6213f, 24.5597f, 34.388f, 39.3329f},
    {(float)(0.5 * kZBins / (double)16.333f), (float)(0.5 * kZBins / (double)16.333f),
     (float)(0.5 * kZBins / (double)16.333f), (float)(0.5 * kZBins / (double)42.140f),
     (float)(0.5 * kZBins / (double)42.140f), (float)(0.5 * kZBins / (double)73.745f),
     (float)(0.5 * kZBins / (double)73.745f)},
    {0.1f, 0.1f, 0.3f, 0.3f, 0.3f, 0.3f},
    {0.2f, 0.4f, 0.5f, 0.6f, 3.0f},
    {0.05f, 0.04f, 0.05f, 0.2f, 0.4f},
    {0.002f, 0.009f, 0.002f, 0.005f},
    {0.008f, 0.0025f, 0.003f, 0.0035f},
};

// IndexTableUtils.h:47-51: truncating conversion of (z + Zhalf) * invZ
__device__ __forceinline__ int z_bin_index(int layer, float z) { return (int)((z + kC.z_half[layer]) * kC.inv_z_bin[layer]); }
// IndexTableUtils.h:53-56
__device__ __forceinline__ int phi_bin_index(float phi) { return (int)(phi * kInversePhiBinSize); }
// IndexTableUtils.h:58-62
__device__ __forceinline__ int bin_index(int z_index, int phi_index) { return min(phi_index * kPhiBins + z_index, kTableBins); }
// MathUtils.h:47-51
__device__ __forceinline__ float normalized_phi(float phi)
{
  return (phi < 0) ? phi + kTwoPi : (phi > kTwoPi) ? phi - kTwoPi : phi;
}

// Cluster.cxx:35-45 with MathUtils.h:37-45.
struct Transformed {
  float phi, r;
  int bin;
};
__device__ __forceinline__ Transformed transform_cluster(int layer, float x, float y, float z, float vx, float vy)
{
  const float dx = x - vx;
  const float dy = y - vy;
  Transformed t;
  t.phi = normalized_phi(itsu_atan2f(-dy, -dx) + kPi);
  t.r = sqrtf(dx * dx + dy * dy);
  t.bin = bin_index(z_bin_index(layer, z), phi_bin_index(t.phi));
  return t;
}

// TrackingUtils.cxx:30-48 getBinsRect: {zMin, phiMin, zMax, phiMax}; all zero means empty.
__device__ __forceinline__ int4 bins_rect(float phi, int layer, float dir_z)
{
  const float z_min = dir_z - 2 * kZCoordinateCut;
  const float phi_min = phi - kPhiCoordinateCut;
  const float z_max = dir_z + 2 * kZCoordinateCut;
  const float phi_max = phi + kPhiCoordinateCut;
  if (z_max < -kC.z_half[layer + 1] || z_min > kC.z_half[layer + 1] || z_min > z_max) {
    return make_int4(0, 0, 0, 0);
  }
  return make_int4(max(0, z_bin_index(layer + 1, z_min)), phi_bin_index(normalized_phi(phi_min)),
                   min(kZBins - 1, z_bin_index(layer + 1, z_max)), phi_bin_index(normalized_phi(phi_max)));
}

// Tracker.cxx:93-100: the tracklet cut for candidate (r2, z2, phi2) of inner cluster (r1, z1, phi1).
__device__ __forceinline__ bool tracklet_cut(int layer, float tan_lambda, float r1, float z1, float phi1, float r2, float z2,
                                             float phi2)
{
  const float delta_z = fabsf(tan_lambda * (r2 - r1) + z1 - z2);
  const float delta_phi = fabsf(phi1 - phi2);
  return delta_z < kC.trk_max_dz[layer] && (delta_phi < kPhiCoordinateCut || delta_phi > kPhiWrapTracklet);
}

// Tracker.cxx:161-173: the cheap cell cuts, which need only the two tracklets and the first
// cluster (c = (x, y, z, r)); most pairs stop here. Every term is evaluated (no early exit: the
// terms are pure, so the result is the reference's short-circuit one) so that a loop over
// outgoing tracklets runs without branches; max_dz is the layer's CellMaxDeltaZThreshold.
__device__ __forceinline__ bool cell_precut_dz(float t1_tan_lambda, float t1_phi, float t2_tan_lambda, float t2_phi, float4 c1,
                                               float vz, float max_dz)
{
  const float delta_tan_lambda = fabsf(t1_tan_lambda - t2_tan_lambda);
  const float delta_phi = fabsf(t1_phi - t2_phi);
  const float average_tan_lambda = 0.5f * (t1_tan_lambda + t2_tan_lambda);
  const float dir_z = -average_tan_lambda * c1.w + c1.z;
  const float delta_z = fabsf(dir_z - vz);
  return (delta_tan_lambda < kCellMaxDeltaTanLambda) &
         ((delta_phi < kCellMaxDeltaPhi) | (delta_phi > kPhiWrapCell)) & (delta_z < max_dz);
}

__device__ __forceinline__ bool cell_precut(int layer, float t1_tan_lambda, float t1_phi, float t2_tan_lambda, float t2_phi,
                                            float4 c1, float vz)
{
  return cell_precut_dz(t1_tan_lambda, t1_phi, t2_tan_lambda, t2_phi, c1, vz, kC.cell_max_dz[layer]);
}

// Tracker.cxx:175-216: circle-plane normal, radius and DCA of the three clusters. Returns false
// when the pair is rejected; otherwise fills the unit normal and curvature. dca_out receives the
// DCA whenever it is computed (-1 when the clusters give no plane).
__device__ __forceinline__ bool cell_geometry(int layer, float4 c1, float4 c2, float4 c3, float vx, float vy, float3 &normal,
                                              float &curvature, float &dca_out)
{
  dca_out = -1.0f;
  const float r1sq = c1.w * c1.w;
  const float r2sq = c2.w * c2.w;
  const float r3sq = c3.w * c3.w;
  const float d1x = c2.x - c1.x, d1y = c2.y - c1.y, d1z = r2sq - r1sq;
  const float d2x = c3.x - c1.x, d2y = c3.y - c1.y, d2z = r3sq - r1sq;
  // MathUtils.h:53-60 crossProduct
  const float nx = (d1y * d2z) - (d1z * d2y);
  const float ny = (d1z * d2x) - (d1x * d2z);
  const float nz = (d1x * d2y) - (d1y * d2x);
  const float norm = sqrtf(nx * nx + ny * ny + nz * nz);
  if (norm < kFloatMinThreshold || fabsf(nz) < kFloatMinThreshold) {
    return false;
  }
  const float inv = 1.0f / norm;
  const float unx = nx * inv, uny = ny * inv, unz = nz * inv;
  // Tracker.cxx:200-202, with the reference's grouping of the y term
  const float plane_d = -unx * (c2.x - vx) - (uny * c2.y - vy) - unz * r2sq;
  const float nzsq = unz * unz;
  const float radius = sqrtf((1.0f - nzsq - 4.0f * plane_d * unz) / (4.0f * nzsq));
  const float ccx = -0.5f * unx / unz;
  const float ccy = -0.5f * uny / unz;
  const float dca = fabsf(radius - sqrtf(ccx * ccx + ccy * ccy));
  dca_out = dca;
  if (dca > kC.cell_max_dca[layer]) {
    return false;
  }
  normal = make_float3(unx, uny, unz);
  curvature = 1.0f / radius;
  return true;
}

__device__ __forceinline__ bool cell_geometry(int layer, float4 c1, float4 c2, float4 c3, float vx, float vy, float3 &normal,
                                              float &curvature)
{
  float dca;
  return cell_geometry(layer, c1, c2, c3, vx, vy, normal, curvature, dca);
}

// Tracker.cxx:448-459: neighbour cut between a cell and a next-layer cell.
__device__ __forceinline__ bool neighbour_cut(int layer, float3 n1, float k1, float3 n2, float k2)
{
  const float dx = n1.x - n2.x, dy = n1.y - n2.y, dz = n1.z - n2.z;
  const float delta_normal = (dx * dx) + (dy * dy) + (dz * dz);
  const float delta_curvature = fabsf(k1 - k2);
  return delta_normal < kC.nb_max_normal[layer] && delta_curvature < kC.nb_max_curv[layer];
}

}  // namespace itsu
