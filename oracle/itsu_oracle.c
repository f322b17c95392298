/*
 * itsu_oracle.c - CPU restatement of the reference tracker's hot path (plain C99).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. The product library never links or
 * calls this file. Each function names the reference lines it follows; the expressions are
 * written in the reference's order, in binary32, and the file is compiled without FMA
 * contraction (-ffp-contract=off), like the reference's own -O3 x86-64 build.
 *
 * Patches relative to the literal reference (all memory-safety or determinism fixes; none
 * changes a computed value of a well-defined run):
 *   P1  candidate loop bound: also stop at the end of the layer (Tracker.cxx:88; the reference's
 *       own GPU kernel guards the same bound, Tracker.cu:87).
 *   P2  cells lookup table of layer L sized to the tracklets of layer L (Tracker.cxx:221-224
 *       writes past the coefficient-sized table of PrimaryVertexContext.cxx:70-73).
 *   P3  stable sort by bin (PrimaryVertexContext.cxx:52): ties keep input order.
 *   P4  correctly rounded atan2f (include/itsu_atan2f.h) in place of the C library's.
 *   P5  a phi row's upper index-table bin is clamped to 400 (Tracker.cxx:84-86): a window edge
 *       that normalises to exactly 2*pi has phi bin 20 and reads past the 401-entry table.
 */
#include "itsu_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/itsu_atan2f.h"

/* ---- Constants (include/ITSReconstruction/CA/Constants.h:31-92) ---- */
static const float kPi = 3.14159265359f;
static const float kTwoPi = 2.0f * 3.14159265359f;
static const float kFloatMinThreshold = 1e-20f;
static const float kLayersZ[7] = {16.333f, 16.333f, 16.333f, 42.140f, 42.140f, 73.745f, 73.745f};
static const float kLayersR[7] = {2.33959f, 3.14076f, 3.91924f, 19.6213f, 24.5597f, 34.388f, 39.3329f};
static const float kTrackletMaxDeltaZ[6] = {0.1f, 0.1f, 0.3f, 0.3f, 0.3f, 0.3f};
static const float kCellMaxDeltaTanLambda = 0.025f;
static const float kCellMaxDeltaZ[5] = {0.2f, 0.4f, 0.5f, 0.6f, 3.0f};
static const float kCellMaxDCA[5] = {0.05f, 0.04f, 0.05f, 0.2f, 0.4f};
static const float kCellMaxDeltaPhi = 0.14f;
static const float kZCoordinateCut = 0.5f;
static const float kPhiCoordinateCut = 0.3f;
static const float kNeighbourMaxNormalDelta[4] = {0.002f, 0.009f, 0.002f, 0.005f};
static const float kNeighbourMaxCurvatureDelta[4] = {0.008f, 0.0025f, 0.003f, 0.0035f};
enum { kZBins = 20, kPhiBins = 20, kTableBins = kZBins * kPhiBins, kCellsPerRoad = 5, kCellsMinLevel = 5 };

/* Constants.h:79: PhiBins / TwoPi in binary32 */
static float inverse_phi_bin_size(void) { return (float)kPhiBins / kTwoPi; }
/* Constants.h:80-84: 0.5 * ZBins / LayersZ[L] evaluated in double, stored as float */
static float inverse_z_bin_size(int layer) { return (float)(0.5 * kZBins / (double)kLayersZ[layer]); }

/* ---- growable arrays ---- */
typedef struct {
  char *data;
  int64_t size, cap;
  size_t elem;
} vec;

static int vec_push(vec *v, const void *item)
{
  if (v->size == v->cap) {
    int64_t ncap = v->cap ? v->cap * 2 : 64;
    char *nd = (char *)realloc(v->data, (size_t)ncap * v->elem);
    if (!nd) {
      return -1;
    }
    v->data = nd;
    v->cap = ncap;
  }
  memcpy(v->data + (size_t)v->size * v->elem, item, v->elem);
  v->size++;
  return 0;
}

struct oracle_result {
  float pv[3];
  int32_t n[ITSU_LAYERS];
  itsu_cluster *clusters[ITSU_LAYERS];
  int32_t index_tables[ITSU_TRACKLET_LAYERS][ITSU_INDEX_TABLE_SIZE];
  vec tracklets[ITSU_TRACKLET_LAYERS];
  int32_t *trk_lookup[ITSU_CELL_LAYERS];
  int64_t trk_lookup_size[ITSU_CELL_LAYERS];
  vec cells[ITSU_CELL_LAYERS];
  int32_t *cell_lookup[ITSU_NEIGHBOUR_LAYERS];
  int64_t cell_lookup_size[ITSU_NEIGHBOUR_LAYERS];
  vec nb_lists[ITSU_NEIGHBOUR_LAYERS]; /* (next cell, cell) pairs in push order */
  int32_t *nb_offsets[ITSU_NEIGHBOUR_LAYERS];
  int32_t *nb_flat[ITSU_NEIGHBOUR_LAYERS];
  int64_t nb_count[ITSU_NEIGHBOUR_LAYERS];
  vec roads;
  int failed;
};

/* ---- per-vertex cluster transform ---- */

/* IndexTableUtils.h:47-51 getZBinIndex: truncating conversion of (z + Zhalf) * invZ */
static int z_bin_index(int layer, float z) { return (int)((z + kLayersZ[layer]) * inverse_z_bin_size(layer)); }
/* IndexTableUtils.h:53-56 getPhiBinIndex */
static int phi_bin_index(float phi) { return (int)(phi * inverse_phi_bin_size()); }
/* IndexTableUtils.h:58-62 getBinIndex */
static int bin_index(int z_index, int phi_index)
{
  int b = phi_index * kPhiBins + z_index;
  return b < kTableBins ? b : kTableBins;
}
/* MathUtils.h:47-51 getNormalizedPhiCoordinate */
static float normalized_phi(float phi)
{
  return (phi < 0) ? phi + kTwoPi : (phi > kTwoPi) ? phi - kTwoPi : phi;
}

float oracle_atan2f(float y, float x) { return itsu_atan2f(y, x); }
void oracle_atan2f_n(const float *y, const float *x, float *out, int64_t n)
{
  for (int64_t i = 0; i < n; ++i) out[i] = itsu_atan2f(y[i], x[i]);
}

/* Cluster.cxx:35-45 with MathUtils.h:37-45: vertex-relative phi and r, then the bin. */
void oracle_transform_cluster(int layer, const float vertex[3], const itsu_cluster *raw, itsu_cluster *out)
{
  const float dx = raw->x - vertex[0];
  const float dy = raw->y - vertex[1];
  *out = *raw;
  out->phi = normalized_phi(itsu_atan2f(-dy, -dx) + kPi);
  out->r = sqrtf(dx * dx + dy * dy);
  out->bin = bin_index(z_bin_index(layer, out->z), phi_bin_index(out->phi));
}

/* Stable merge sort of clusters by bin (P3 form of PrimaryVertexContext.cxx:52-54). */
static void stable_sort_by_bin(itsu_cluster *a, itsu_cluster *tmp, int64_t n)
{
  int64_t width, i;
  itsu_cluster *src = a, *dst = tmp;
  for (width = 1; width < n; width *= 2) {
    for (i = 0; i < n; i += 2 * width) {
      int64_t lo = i, mid = i + width < n ? i + width : n, hi = i + 2 * width < n ? i + 2 * width : n;
      int64_t p = lo, q = mid, k = lo;
      while (p < mid && q < hi) {
        dst[k++] = (src[q].bin < src[p].bin) ? src[q++] : src[p++];
      }
      while (p < mid) {
        dst[k++] = src[p++];
      }
      while (q < hi) {
        dst[k++] = src[q++];
      }
    }
    {
      itsu_cluster *t = src;
      src = dst;
      dst = t;
    }
  }
  if (src != a) {
    memcpy(a, src, (size_t)n * sizeof(itsu_cluster));
  }
}

/* PrimaryVertexContext::initialize (PrimaryVertexContext.cxx:31-142), CPU branch. */
static void initialize(oracle_result *res, const itsu_cluster *const layers[ITSU_LAYERS])
{
  int layer;
  for (layer = 0; layer < ITSU_LAYERS; ++layer) {
    const int32_t n = res->n[layer];
    int32_t i;
    itsu_cluster *tmp;
    res->clusters[layer] = (itsu_cluster *)malloc(sizeof(itsu_cluster) * (size_t)(n > 0 ? n : 1));
    tmp = (itsu_cluster *)malloc(sizeof(itsu_cluster) * (size_t)(n > 0 ? n : 1));
    if (!res->clusters[layer] || !tmp) {
      free(tmp);
      res->failed = 1;
      return;
    }
    /* :46-50 per-vertex transform of every cluster */
    for (i = 0; i < n; ++i) {
      oracle_transform_cluster(layer, res->pv, &layers[layer][i], &res->clusters[layer][i]);
    }
    /* :52-54 sort by bin (stable: P3) */
    stable_sort_by_bin(res->clusters[layer], tmp, n);
    free(tmp);
    /* :90-119 index table of layer L >= 1: first sorted index of each bin */
    if (layer > 0) {
      int32_t *table = res->index_tables[layer - 1];
      int previous = 0, b;
      table[0] = 0;
      for (i = 0; i < n; ++i) {
        const int current = res->clusters[layer][i].bin;
        if (current > previous) {
          for (b = previous + 1; b <= current; ++b) {
            table[b] = i;
          }
          previous = current;
        }
      }
      for (b = previous + 1; b <= kTableBins; ++b) {
        table[b] = n;
      }
    }
  }
  /* :136-138 tracklets lookup table L (clusters of layer L+1), all unused */
  for (layer = 0; layer < ITSU_CELL_LAYERS; ++layer) {
    int64_t i, size = res->n[layer + 1];
    res->trk_lookup_size[layer] = size;
    res->trk_lookup[layer] = (int32_t *)malloc(sizeof(int32_t) * (size_t)(size > 0 ? size : 1));
    if (!res->trk_lookup[layer]) {
      res->failed = 1;
      return;
    }
    for (i = 0; i < size; ++i) {
      res->trk_lookup[layer][i] = ITSU_UNUSED_INDEX;
    }
  }
}

/* TrackingUtils.cxx:30-48 getBinsRect: {zMin, phiMin, zMax, phiMax}, all zero when empty. */
static void bins_rect(const itsu_cluster *c, int layer, float dir_z, int rect[4])
{
  const float z_min = dir_z - 2 * kZCoordinateCut;
  const float phi_min = c->phi - kPhiCoordinateCut;
  const float z_max = dir_z + 2 * kZCoordinateCut;
  const float phi_max = c->phi + kPhiCoordinateCut;
  int zb;
  if (z_max < -kLayersZ[layer + 1] || z_min > kLayersZ[layer + 1] || z_min > z_max) {
    rect[0] = rect[1] = rect[2] = rect[3] = 0;
    return;
  }
  zb = z_bin_index(layer + 1, z_min);
  rect[0] = zb > 0 ? zb : 0;
  rect[1] = phi_bin_index(normalized_phi(phi_min));
  zb = z_bin_index(layer + 1, z_max);
  rect[2] = zb < kZBins - 1 ? zb : kZBins - 1;
  rect[3] = phi_bin_index(normalized_phi(phi_max));
}

/* TrackerTraits<false>::computeLayerTracklets (Tracker.cxx:45-117) with P1 and P5. */
static void compute_tracklets(oracle_result *res)
{
  int layer;
  for (layer = 0; layer < ITSU_TRACKLET_LAYERS; ++layer) {
    const int32_t n = res->n[layer], n_next = res->n[layer + 1];
    const int32_t *table = res->index_tables[layer];
    int32_t i;
    if (n == 0 || n_next == 0) {
      return; /* :49-52 */
    }
    for (i = 0; i < n; ++i) {
      const itsu_cluster *cur = &res->clusters[layer][i];
      const float tan_lambda = (cur->z - res->pv[2]) / cur->r;
      const float dir_z = tan_lambda * (kLayersR[layer + 1] - cur->r) + cur->z;
      int rect[4], phi_bins, phi_bin, phi_count;
      bins_rect(cur, layer, dir_z, rect);
      if (rect[0] == 0 && rect[1] == 0 && rect[2] == 0 && rect[3] == 0) {
        continue;
      }
      phi_bins = rect[3] - rect[1] + 1;
      if (phi_bins < 0) {
        phi_bins += kPhiBins;
      }
      for (phi_bin = rect[1], phi_count = 0; phi_count < phi_bins;
           phi_bin = (phi_bin + 1 == kPhiBins) ? 0 : phi_bin + 1, phi_count++) {
        const int first_bin = bin_index(rect[0], phi_bin);
        int max_bin = first_bin + rect[2] - rect[0] + 1;
        int32_t first_row, max_row, j;
        if (max_bin > kTableBins) {
          max_bin = kTableBins; /* P5 */
        }
        first_row = table[first_bin];
        max_row = table[max_bin];
        for (j = first_row; j <= max_row && j < n_next; ++j) { /* P1 */
          const itsu_cluster *next = &res->clusters[layer + 1][j];
          const float delta_z = fabsf(tan_lambda * (next->r - cur->r) + cur->z - next->z);
          const float delta_phi = fabsf(cur->phi - next->phi);
          if (delta_z < kTrackletMaxDeltaZ[layer] &&
              (delta_phi < kPhiCoordinateCut || fabsf(delta_phi - kTwoPi) < kPhiCoordinateCut)) {
            itsu_tracklet t;
            if (layer > 0 && res->trk_lookup[layer - 1][i] == ITSU_UNUSED_INDEX) {
              res->trk_lookup[layer - 1][i] = (int32_t)res->tracklets[layer].size;
            }
            /* Tracklet.cxx:32-40 */
            t.first_cluster = i;
            t.second_cluster = j;
            t.tan_lambda = (cur->z - next->z) / (cur->r - next->r);
            t.phi = itsu_atan2f(cur->y - next->y, cur->x - next->x);
            if (vec_push(&res->tracklets[layer], &t)) {
              res->failed = 1;
              return;
            }
          }
        }
      }
    }
  }
}

/* TrackerTraits<false>::computeLayerCells (Tracker.cxx:120-235) with P2. */
static void compute_cells(oracle_result *res)
{
  int layer;
  for (layer = 0; layer < ITSU_CELL_LAYERS; ++layer) {
    const vec *trk = &res->tracklets[layer], *trk_next = &res->tracklets[layer + 1];
    const int32_t n_trk = (int32_t)trk->size, n_next = (int32_t)trk_next->size;
    int32_t it;
    if (n_next == 0 || n_trk == 0) {
      return; /* :124-128 */
    }
    if (layer > 0) { /* P2: one lookup entry per tracklet of this layer */
      int32_t k;
      res->cell_lookup_size[layer - 1] = n_trk;
      res->cell_lookup[layer - 1] = (int32_t *)malloc(sizeof(int32_t) * (size_t)n_trk);
      if (!res->cell_lookup[layer - 1]) {
        res->failed = 1;
        return;
      }
      for (k = 0; k < n_trk; ++k) {
        res->cell_lookup[layer - 1][k] = ITSU_UNUSED_INDEX;
      }
    }
    for (it = 0; it < n_trk; ++it) {
      const itsu_tracklet *cur = &((const itsu_tracklet *)trk->data)[it];
      const int32_t next_cluster = cur->second_cluster;
      const int32_t next_first = res->trk_lookup[layer][next_cluster];
      const itsu_cluster *c1, *c2;
      float r1sq, r2sq, d1x, d1y, d1z;
      int32_t jt;
      if (next_first == ITSU_UNUSED_INDEX) {
        continue;
      }
      c1 = &res->clusters[layer][cur->first_cluster];
      c2 = &res->clusters[layer + 1][cur->second_cluster];
      r1sq = c1->r * c1->r;
      r2sq = c2->r * c2->r;
      d1x = c2->x - c1->x;
      d1y = c2->y - c1->y;
      d1z = r2sq - r1sq;
      for (jt = next_first;
           jt < n_next && ((const itsu_tracklet *)trk_next->data)[jt].first_cluster == next_cluster; ++jt) {
        const itsu_tracklet *nxt = &((const itsu_tracklet *)trk_next->data)[jt];
        const float delta_tan_lambda = fabsf(cur->tan_lambda - nxt->tan_lambda);
        const float delta_phi = fabsf(cur->phi - nxt->phi);
        if (delta_tan_lambda < kCellMaxDeltaTanLambda &&
            (delta_phi < kCellMaxDeltaPhi || fabsf(delta_phi - kTwoPi) < kCellMaxDeltaPhi)) {
          const float avg_tan_lambda = 0.5f * (cur->tan_lambda + nxt->tan_lambda);
          const float dir_z = -avg_tan_lambda * c1->r + c1->z;
          const float delta_z = fabsf(dir_z - res->pv[2]);
          if (delta_z < kCellMaxDeltaZ[layer]) {
            const itsu_cluster *c3 = &res->clusters[layer + 2][nxt->second_cluster];
            const float r3sq = c3->r * c3->r;
            const float d2x = c3->x - c1->x, d2y = c3->y - c1->y, d2z = r3sq - r1sq;
            /* MathUtils.h:53-60 crossProduct */
            const float nx = (d1y * d2z) - (d1z * d2y);
            const float ny = (d1z * d2x) - (d1x * d2z);
            const float nz = (d1x * d2y) - (d1y * d2x);
            const float norm = sqrtf(nx * nx + ny * ny + nz * nz);
            float inv, unx, uny, unz, plane_d, nzsq, radius, ccx, ccy, dca;
            if (norm < kFloatMinThreshold || fabsf(nz) < kFloatMinThreshold) {
              continue;
            }
            inv = 1.0f / norm;
            unx = nx * inv;
            uny = ny * inv;
            unz = nz * inv;
            /* :200-202, including the reference's grouping of the y term */
            plane_d = -unx * (c2->x - res->pv[0]) - (uny * c2->y - res->pv[1]) - unz * r2sq;
            nzsq = unz * unz;
            radius = sqrtf((1.0f - nzsq - 4.0f * plane_d * unz) / (4.0f * nzsq));
            ccx = -0.5f * unx / unz;
            ccy = -0.5f * uny / unz;
            dca = fabsf(radius - sqrtf(ccx * ccx + ccy * ccy));
            if (dca > kCellMaxDCA[layer]) {
              continue;
            }
            {
              itsu_cell cell;
              if (layer > 0 && res->cell_lookup[layer - 1][it] == ITSU_UNUSED_INDEX) {
                res->cell_lookup[layer - 1][it] = (int32_t)res->cells[layer].size;
              }
              /* Cell.cxx:24-32 */
              cell.first_cluster = cur->first_cluster;
              cell.second_cluster = nxt->first_cluster;
              cell.third_cluster = nxt->second_cluster;
              cell.first_tracklet = it;
              cell.second_tracklet = jt;
              cell.nx = unx;
              cell.ny = uny;
              cell.nz = unz;
              cell.curvature = 1.0f / radius;
              cell.level = 1;
              if (vec_push(&res->cells[layer], &cell)) {
                res->failed = 1;
                return;
              }
            }
          }
        }
      }
    }
  }
}

/* Tracker<IsGPU>::findCellsNeighbours (Tracker.cxx:417-474). Neighbour lists are kept as
 * (next cell, cell) pairs in push order and turned into a CSR afterwards. */
static void find_neighbours(oracle_result *res)
{
  int layer;
  for (layer = 0; layer < ITSU_NEIGHBOUR_LAYERS; ++layer) {
    vec *cells = &res->cells[layer], *next_cells = &res->cells[layer + 1];
    const int32_t n_cells = (int32_t)cells->size, n_next = (int32_t)next_cells->size;
    int32_t ic;
    if (n_next == 0 || res->cell_lookup_size[layer] == 0) {
      continue; /* :421-425 */
    }
    for (ic = 0; ic < n_cells; ++ic) {
      const itsu_cell *cur = &((const itsu_cell *)cells->data)[ic];
      const int32_t next_trk = cur->second_tracklet;
      const int32_t next_first = res->cell_lookup[layer][next_trk];
      itsu_cell *nc = (itsu_cell *)next_cells->data;
      int32_t jc;
      if (next_first == ITSU_UNUSED_INDEX || nc[next_first].first_tracklet != next_trk) {
        continue;
      }
      for (jc = next_first; jc < n_next && nc[jc].first_tracklet == next_trk; ++jc) {
        const float dx = cur->nx - nc[jc].nx, dy = cur->ny - nc[jc].ny, dz = cur->nz - nc[jc].nz;
        const float delta_normal = (dx * dx) + (dy * dy) + (dz * dz);
        const float delta_curvature = fabsf(cur->curvature - nc[jc].curvature);
        if (delta_normal < kNeighbourMaxNormalDelta[layer] && delta_curvature < kNeighbourMaxCurvatureDelta[layer]) {
          int32_t pair[2];
          pair[0] = jc;
          pair[1] = ic;
          if (vec_push(&res->nb_lists[layer], pair)) {
            res->failed = 1;
            return;
          }
          if (cur->level >= nc[jc].level) {
            nc[jc].level = cur->level + 1;
          }
        }
      }
    }
  }
  /* CSR over the cells of layer L+1; each row keeps push order (ascending cell index). */
  for (layer = 0; layer < ITSU_NEIGHBOUR_LAYERS; ++layer) {
    const int64_t rows = res->cells[layer + 1].size, nnz = res->nb_lists[layer].size;
    const int32_t *pairs = (const int32_t *)res->nb_lists[layer].data;
    int32_t *cursor;
    int64_t k;
    res->nb_offsets[layer] = (int32_t *)calloc((size_t)rows + 1, sizeof(int32_t));
    res->nb_flat[layer] = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    cursor = (int32_t *)calloc((size_t)rows + 1, sizeof(int32_t));
    if (!res->nb_offsets[layer] || !res->nb_flat[layer] || !cursor) {
      free(cursor);
      res->failed = 1;
      return;
    }
    for (k = 0; k < nnz; ++k) {
      res->nb_offsets[layer][pairs[2 * k] + 1]++;
    }
    for (k = 0; k < rows; ++k) {
      res->nb_offsets[layer][k + 1] += res->nb_offsets[layer][k];
    }
    for (k = 0; k < nnz; ++k) {
      const int32_t row = pairs[2 * k];
      res->nb_flat[layer][res->nb_offsets[layer][row] + cursor[row]++] = pairs[2 * k + 1];
    }
    res->nb_count[layer] = nnz;
    free(cursor);
  }
}

/* Road::Road(layer, cell) and Road::addCell (Road.cxx:24-50) */
static void road_init(itsu_road *road, int layer, int32_t cell)
{
  int k;
  memset(road, 0, sizeof *road);
  for (k = 0; k < ITSU_CELL_LAYERS; ++k) {
    road->cell_ids[k] = ITSU_UNUSED_INDEX;
  }
  road->size = 1;
  road->cell_ids[layer] = cell;
}

static void road_add_cell(itsu_road *road, int layer, int32_t cell)
{
  if (road->cell_ids[layer] == ITSU_UNUSED_INDEX) {
    road->size++;
  }
  road->cell_ids[layer] = cell;
}

/* Tracker<IsGPU>::traverseCellsTree (Tracker.cxx:532-571) */
static void traverse_cells_tree(oracle_result *res, int32_t cell_id, int layer)
{
  const itsu_cell *cell = &((const itsu_cell *)res->cells[layer].data)[cell_id];
  const int level = cell->level;
  road_add_cell(&((itsu_road *)res->roads.data)[res->roads.size - 1], layer, cell_id);
  if (layer > 0) {
    const int32_t *offs = res->nb_offsets[layer - 1];
    const int32_t begin = offs[cell_id], end = offs[cell_id + 1];
    int first_valid = 1;
    int32_t k;
    for (k = begin; k < end; ++k) {
      const int32_t nb = res->nb_flat[layer - 1][k];
      if (level - 1 != ((const itsu_cell *)res->cells[layer - 1].data)[nb].level) {
        continue;
      }
      if (first_valid) {
        first_valid = 0;
      } else {
        itsu_road copy = ((itsu_road *)res->roads.data)[res->roads.size - 1];
        if (vec_push(&res->roads, &copy)) {
          res->failed = 1;
          return;
        }
      }
      traverse_cells_tree(res, nb, layer - 1);
    }
  }
}

/* Tracker<IsGPU>::findTracks (Tracker.cxx:477-529) */
static void find_tracks(oracle_result *res)
{
  int level;
  for (level = kCellsPerRoad; level >= kCellsMinLevel; --level) {
    const int minimum_level = level - 1;
    int layer;
    for (layer = kCellsPerRoad - 1; layer >= minimum_level; --layer) {
      const int32_t n_cells = (int32_t)res->cells[layer].size;
      int32_t ic;
      for (ic = 0; ic < n_cells; ++ic) {
        const itsu_cell *cur = &((const itsu_cell *)res->cells[layer].data)[ic];
        itsu_road road;
        int first_valid = 1;
        int32_t k, begin, end;
        if (cur->level != level) {
          continue;
        }
        road_init(&road, layer, ic);
        if (vec_push(&res->roads, &road)) {
          res->failed = 1;
          return;
        }
        begin = res->nb_offsets[layer - 1][ic];
        end = res->nb_offsets[layer - 1][ic + 1];
        for (k = begin; k < end; ++k) {
          const int32_t nb = res->nb_flat[layer - 1][k];
          if (level - 1 != ((const itsu_cell *)res->cells[layer - 1].data)[nb].level) {
            continue;
          }
          if (first_valid) {
            first_valid = 0;
          } else {
            road_init(&road, layer, ic);
            if (vec_push(&res->roads, &road)) {
              res->failed = 1;
              return;
            }
          }
          traverse_cells_tree(res, nb, layer - 1);
        }
      }
    }
  }
}

/* Tracker<IsGPU>::computeMontecarloLabels (Tracker.cxx:574-652): Moore's voting. */
static void compute_labels(oracle_result *res)
{
  int64_t ir;
  for (ir = 0; ir < res->roads.size; ++ir) {
    itsu_road *road = &((itsu_road *)res->roads.data)[ir];
    int max_value = ITSU_UNUSED_INDEX, count = 0, fake = 0, first = 1, ic;
    for (ic = 0; ic < kCellsPerRoad; ++ic) {
      const int32_t cell_index = road->cell_ids[ic];
      const itsu_cell *cell;
      int current;
      if (cell_index == ITSU_UNUSED_INDEX) {
        if (first) {
          continue;
        }
        break;
      }
      cell = &((const itsu_cell *)res->cells[ic].data)[cell_index];
      if (first) {
        int second;
        max_value = res->clusters[ic][cell->first_cluster].mc_id;
        count = 1;
        second = res->clusters[ic + 1][cell->second_cluster].mc_id;
        if (second == max_value) {
          ++count;
        } else {
          max_value = second;
          count = 1;
          fake = 1;
        }
        first = 0;
      }
      current = res->clusters[ic + 2][cell->third_cluster].mc_id;
      if (current == max_value) {
        ++count;
      } else {
        --count;
        fake = 1;
      }
      if (count == 0) {
        max_value = current;
        count = 1;
      }
    }
    road->label = max_value;
    road->is_fake = (uint8_t)fake;
  }
}

oracle_result *oracle_run_vertex(const itsu_cluster *const layers[ITSU_LAYERS], const int32_t counts[ITSU_LAYERS],
                                 const float vertex[3])
{
  oracle_result *res = (oracle_result *)calloc(1, sizeof(oracle_result));
  int k;
  if (!res) {
    return NULL;
  }
  res->pv[0] = vertex[0];
  res->pv[1] = vertex[1];
  res->pv[2] = vertex[2];
  for (k = 0; k < ITSU_LAYERS; ++k) {
    res->n[k] = counts[k];
  }
  for (k = 0; k < ITSU_TRACKLET_LAYERS; ++k) {
    res->tracklets[k].elem = sizeof(itsu_tracklet);
  }
  for (k = 0; k < ITSU_CELL_LAYERS; ++k) {
    res->cells[k].elem = sizeof(itsu_cell);
  }
  for (k = 0; k < ITSU_NEIGHBOUR_LAYERS; ++k) {
    res->nb_lists[k].elem = 2 * sizeof(int32_t);
  }
  res->roads.elem = sizeof(itsu_road);
  initialize(res, layers);
  if (!res->failed) compute_tracklets(res);
  if (!res->failed) compute_cells(res);
  if (!res->failed) find_neighbours(res);
  if (!res->failed) find_tracks(res);
  if (!res->failed) compute_labels(res);
  if (res->failed) {
    oracle_free(res);
    return NULL;
  }
  return res;
}

int64_t oracle_size(const oracle_result *res, int kind, int layer)
{
  switch (kind) {
  case ORACLE_CLUSTERS: return res->n[layer];
  case ORACLE_INDEX_TABLE: return ITSU_INDEX_TABLE_SIZE;
  case ORACLE_TRACKLETS: return res->tracklets[layer].size;
  case ORACLE_TRACKLETS_LOOKUP: return res->trk_lookup_size[layer];
  case ORACLE_CELLS: return res->cells[layer].size;
  case ORACLE_CELLS_LOOKUP: return res->cell_lookup_size[layer];
  case ORACLE_NEIGHBOUR_OFFSETS: return res->cells[layer + 1].size + 1;
  case ORACLE_NEIGHBOURS: return res->nb_count[layer];
  case ORACLE_ROADS: return res->roads.size;
  default: return -1;
  }
}

const void *oracle_data(const oracle_result *res, int kind, int layer)
{
  switch (kind) {
  case ORACLE_CLUSTERS: return res->clusters[layer];
  case ORACLE_INDEX_TABLE: return res->index_tables[layer];
  case ORACLE_TRACKLETS: return res->tracklets[layer].data;
  case ORACLE_TRACKLETS_LOOKUP: return res->trk_lookup[layer];
  case ORACLE_CELLS: return res->cells[layer].data;
  case ORACLE_CELLS_LOOKUP: return res->cell_lookup[layer];
  case ORACLE_NEIGHBOUR_OFFSETS: return res->nb_offsets[layer];
  case ORACLE_NEIGHBOURS: return res->nb_flat[layer];
  case ORACLE_ROADS: return res->roads.data;
  default: return NULL;
  }
}

void oracle_free(oracle_result *res)
{
  int k;
  if (!res) {
    return;
  }
  for (k = 0; k < ITSU_LAYERS; ++k) free(res->clusters[k]);
  for (k = 0; k < ITSU_TRACKLET_LAYERS; ++k) free(res->tracklets[k].data);
  for (k = 0; k < ITSU_CELL_LAYERS; ++k) {
    free(res->trk_lookup[k]);
    free(res->cells[k].data);
  }
  for (k = 0; k < ITSU_NEIGHBOUR_LAYERS; ++k) {
    free(res->cell_lookup[k]);
    free(res->nb_lists[k].data);
    free(res->nb_offsets[k]);
    free(res->nb_flat[k]);
  }
  free(res->roads.data);
  free(res);
}

int64_t oracle_run_batch(const itsu_cluster *clusters, const int32_t *layer_offsets, const float *vertices,
                         int32_t n_events)
{
  int64_t roads = 0;
  int32_t e;
  for (e = 0; e < n_events; ++e) {
    const itsu_cluster *layers[ITSU_LAYERS];
    int32_t counts[ITSU_LAYERS];
    oracle_result *res;
    int k;
    for (k = 0; k < ITSU_LAYERS; ++k) {
      layers[k] = clusters + layer_offsets[e * ITSU_LAYERS + k];
      counts[k] = layer_offsets[e * ITSU_LAYERS + k + 1] - layer_offsets[e * ITSU_LAYERS + k];
    }
    res = oracle_run_vertex(layers, counts, vertices + 3 * e);
    if (!res) {
      return -1;
    }
    roads += res->roads.size;
    oracle_free(res);
  }
  return roads;
}

/* ---- road report: IOUtils::writeRoadsReport (IOUtils.cxx:125-170), classification part ----
 * Per event, the labels map's ids (first entry per id, as unordered_map::emplace) are sorted for
 * lookup; the roads of the event's vertices are walked in order: a road whose label is not in
 * the map is skipped (:146-149); a fake one is reported fake (:153-155); otherwise the first road
 * of its label is correct and later ones are duplicates (:159-166). */
static int cmp_i32(const void *a, const void *b)
{
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

static int64_t find_sorted(const int32_t *ids, int64_t n, int32_t key)
{
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (ids[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return (lo < n && ids[lo] == key) ? lo : -1;
}

int oracle_roads_report(const itsu_road *roads, const int32_t *run_offsets, const int32_t *run_event, int32_t n_runs,
                        const itsu_label *labels, const int32_t *label_offsets, int32_t n_events, uint8_t *road_class,
                        itsu_report_counts *counts)
{
  int32_t e, r = 0;
  for (e = 0; e < n_events; ++e) {
    const int64_t l0 = label_offsets[e], nl = label_offsets[e + 1] - label_offsets[e];
    int32_t *ids = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nl > 0 ? nl : 1));
    unsigned char *found = NULL;
    int64_t n_ids = 0, k;
    itsu_report_counts c = {0, 0, 0, 0};
    if (!ids) return -1;
    for (k = 0; k < nl; ++k) ids[k] = labels[l0 + k].mc_id;
    qsort(ids, (size_t)nl, sizeof(int32_t), cmp_i32);
    for (k = 0; k < nl; ++k) {
      if (n_ids == 0 || ids[n_ids - 1] != ids[k]) ids[n_ids++] = ids[k];
    }
    found = (unsigned char *)calloc((size_t)(n_ids > 0 ? n_ids : 1), 1);
    if (!found) {
      free(ids);
      return -1;
    }
    c.labels = (int32_t)n_ids;
    /* the event's runs: consecutive, run_event non-decreasing (NULL: run r is event r) */
    for (; r < n_runs && (run_event ? run_event[r] : r) == e; ++r) {
      int64_t i;
      for (i = run_offsets[r]; i < run_offsets[r + 1]; ++i) {
        const int64_t slot = find_sorted(ids, n_ids, roads[i].label);
        uint8_t cls = ITSU_ROAD_UNREPORTED;
        if (slot >= 0) {
          if (roads[i].is_fake) {
            cls = ITSU_ROAD_FAKE;
            ++c.fake;
          } else if (found[slot]) {
            cls = ITSU_ROAD_DUPLICATE;
            ++c.duplicate;
          } else {
            cls = ITSU_ROAD_CORRECT;
            ++c.correct;
            found[slot] = 1;
          }
        }
        if (road_class) road_class[i] = cls;
      }
    }
    if (counts) counts[e] = c;
    free(found);
    free(ids);
  }
  return 0;
}
