/*
 * CPU restatement of fastfusion's depth-fusion hot path: the oracle.
 * ORACLE INFRASTRUCTURE ONLY -- see ff_port.h for what it restates and who may
 * load it.  Built with -frounding-math -ffp-contract=off so that every float
 * operation is a single IEEE operation in the current rounding mode.
 */
#define _GNU_SOURCE
#include "ff_port.h"
#include "ff_port_internal.h"

#include <fenv.h>
#include <xmmintrin.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BRANCHINIT FFP_BRANCHINIT
#define MAXLEAFNUMBER 10000000u /* reference definitions.h:159 */
#define BL 8                    /* BRICKLENGTH, definitions.h:234 */
#define DIST_W_EPS 0.005f       /* DISTANCEWEIGHTEPSILON, definitions.h:252 */
#define WEIGHT_FACTOR 3.0f      /* definitions.h:255 */
#define COLOR_MUL 256.0f        /* COLOR_MULTIPLICATOR, definitions.h:58 */

struct ffp_map {
  float scale, threshold;
  int color;
  uint16_t n, bandwidth;
  float offset[3];
  uint32_t *tree;
  uint32_t branches_used, branches_total;
  uint32_t leaves_used, leaves_total;
  uint16_t *leaf_pos; /* 3 per leaf */
  uint16_t *leaf_scale;
  uint32_t *leaf_parent;
  uint32_t parent_cap;
  uint32_t *queue_index;
  uint32_t *queue;
  uint32_t nqueued;
  float *dist, *wgt;
  uint16_t *col; /* 3 per voxel: R, G, B (the reference's colortype3 x, y, z) */
  double *dist64, *wgt64; /* update mode 3 (FP64 oracle) */
  int img_w, img_h;
  float *pxp, *pyp;
  int box_min[3], box_max[3];
  int frames;
  int meshing_ok;
  int grows;
  int branch_overflow;
  int rz_exact;
  int fp16; /* SDF and weight stored rounded to half precision (ffp_set_storage_fp16) */
  const float *conf; /* per-pixel confidence of the next frames (learned weight), or NULL */
  /* mesh of the last ffp_update_meshes */
  ffp_cell *cells;
  int64_t ncells;
  ffp_mesh_result mesh;
};

/* ---------------------------------------------------------------- helpers */

/* x86 float->int32 conversion under round-toward-zero, as _mm256_cvtps_epi32
 * does under MXCSR=RZ: truncation, and 0x80000000 for NaN or out of range. */
static int cvt_rz(float f) {
  if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT_MIN;
  return (int)f;
}

/* Reciprocal of the update.  Mode 1 (the defined target): exact division in
 * the current rounding mode.  Mode 2: the host CPU's approximate RCPPS, the
 * instruction the reference executes (_mm256_rcp_ps); its low bits are CPU
 * specific, so this mode exists only to check the restatement against the
 * compiled reference on the same machine. */
static int g_rcp_mode = 1;
static float recip(float x) {
  if (g_rcp_mode == 2) return _mm_cvtss_f32(_mm_rcp_ss(_mm_set_ss(x)));
  return 1.0f / x;
}

/* ------------------------------------------------------------------ setup */

ffp_map *ffp_create(float scale, float threshold, int color, uint32_t leaves_total, uint32_t branches_total) {
  ffp_map *m = (ffp_map *)calloc(1, sizeof(ffp_map));
  m->scale = scale;
  m->threshold = threshold;
  m->color = color;
  /* _bandwidth(_distanceThreshold / _scale*BANDWIDTHFACTOR), geometryfusion_mipmap_cpu.cpp:425 */
  m->bandwidth = (uint16_t)(double)(threshold / scale * 1.0);
  m->leaves_total = leaves_total;
  m->branches_total = branches_total;
  m->tree = (uint32_t *)malloc(sizeof(uint32_t) * branches_total);
  for (uint32_t i = 0; i < branches_total; i++) m->tree[i] = BRANCHINIT;
  m->branches_used = 16;
  m->leaf_pos = (uint16_t *)calloc((size_t)leaves_total * 3, sizeof(uint16_t));
  m->leaf_scale = (uint16_t *)calloc(leaves_total, sizeof(uint16_t));
  m->parent_cap = leaves_total;
  m->leaf_parent = (uint32_t *)malloc(sizeof(uint32_t) * leaves_total);
  m->queue_index = (uint32_t *)malloc(sizeof(uint32_t) * leaves_total);
  m->queue = (uint32_t *)malloc(sizeof(uint32_t) * leaves_total);
  m->dist = (float *)calloc((size_t)leaves_total * 512, sizeof(float));
  m->wgt = (float *)calloc((size_t)leaves_total * 512, sizeof(float));
  m->col = (uint16_t *)calloc((size_t)leaves_total * 512 * 3, sizeof(uint16_t));
  m->meshing_ok = 1;
  m->rz_exact = 1;
  return m;
}

void ffp_destroy(ffp_map *m) {
  if (!m) return;
  free(m->tree);
  free(m->leaf_pos);
  free(m->leaf_scale);
  free(m->leaf_parent);
  free(m->queue_index);
  free(m->queue);
  free(m->dist);
  free(m->wgt);
  free(m->col);
  free(m->dist64);
  free(m->wgt64);
  free(m->pxp);
  free(m->pyp);
  free(m->cells);
  free(m->mesh.xyz);
  free(m->mesh.rgb);
  free(m->mesh.faces);
  free(m->mesh.cell_v);
  free(m);
}

/* Learned weight: the update's weight increment of every voxel is multiplied
 * by conf[pixel] (W x H floats of the frames that follow; NULL = the
 * reference's weight).  The array is borrowed, not copied. */
void ffp_set_confidence(ffp_map *m, const float *conf) { m->conf = conf; }

void ffp_set_update_mode(ffp_map *m, int mode) {
  m->rz_exact = mode;
  if (mode == 3 && !m->dist64) {
    m->dist64 = (double *)calloc((size_t)m->leaves_total * 512, sizeof(double));
    m->wgt64 = (double *)calloc((size_t)m->leaves_total * 512, sizeof(double));
  }
}

/* FP16 storage of SDF and weight (no counterpart in the reference, whose
 * pool is float): after each update the stored value is the nearest binary16
 * value (ties to even, overflow to infinity, subnormals kept), held here as
 * the float it converts back to.  Done with integer operations, so the
 * rounding does not depend on the floating-point rounding mode the update
 * runs in (round-toward-zero). */
void ffp_set_storage_fp16(ffp_map *m, int on) { m->fp16 = on != 0; }

static float round_to_half(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  const uint32_t sign = u & 0x80000000u, a = u & 0x7fffffffu;
  uint32_t r;
  if (a >= 0x7f800000u) {
    r = u; /* infinity or NaN */
  } else if (a >= 0x477ff000u) {
    r = sign | 0x7f800000u; /* at or above 65520: infinity */
  } else if (a <= 0x33000000u) {
    r = sign; /* at or below 2^-25: zero (2^-25 ties to the even zero) */
  } else {
    const int e = (int)(a >> 23) - 127;
    if (e >= -14) {
      /* normal binary16: keep 10 mantissa bits, round to nearest even */
      const uint32_t lsb = (a >> 13) & 1u;
      r = sign | ((a + 0xfffu + lsb) & ~0x1fffu);
    } else {
      /* subnormal binary16: a multiple of 2^-24 */
      const uint32_t mant = (a & 0x7fffffu) | 0x800000u;
      const int sh = -(e + 1);
      uint32_t q = mant >> sh;
      const uint32_t rem = mant & ((1u << sh) - 1u), half = 1u << (sh - 1);
      if (rem > half || (rem == half && (q & 1u))) q++;
      float v = (float)q * 5.9604644775390625e-08f; /* exact: q <= 1024 */
      memcpy(&r, &v, 4);
      r |= sign;
    }
  }
  float out;
  memcpy(&out, &r, 4);
  return out;
}

float ffp_half_round(float f) { return round_to_half(f); }

/* Float camera parameters, the reference's camPamsFloat (definitions.h:71-88),
 * built in double and rounded once to float. */
typedef struct {
  float r[9];
  float t[3];
  float fx, fy, cx, cy;
} campams;

/* p: world -> voxel grid (geometryfusion_mipmap_cpu.cpp:1617-1625). */
static campams cam_world_to_grid(const ffp_map *m, const double *K, const double *R, const double *t) {
  campams p;
  for (int i = 0; i < 9; i++) p.r[i] = (float)(R[i] / (double)m->scale);
  for (int i = 0; i < 3; i++) p.t[i] = (float)((t[i] - (double)m->offset[i]) / (double)m->scale);
  p.fx = (float)K[0];
  p.fy = (float)K[1];
  p.cx = (float)K[2];
  p.cy = (float)K[3];
  return p;
}

/* pInv: world (offset folded in) -> camera (geometryfusion_mipmap_cpu.cpp:1771-1793),
 * with the extrinsic inverse [R^T | -R^T t] (camerautils.cpp:153-161). */
static campams cam_grid_to_camera(const ffp_map *m, const double *K, const double *R, const double *t) {
  campams q;
  double r2[9], t2[3];
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) r2[r * 3 + c] = R[c * 3 + r];
    double s = R[0 * 3 + r] * t[0] + R[1 * 3 + r] * t[1];
    s = s + R[2 * 3 + r] * t[2];
    t2[r] = -s;
  }
  for (int i = 0; i < 9; i++) q.r[i] = (float)r2[i];
  for (int r = 0; r < 3; r++) {
    double v = r2[r * 3 + 0] * (double)m->offset[0] + r2[r * 3 + 1] * (double)m->offset[1];
    v = v + r2[r * 3 + 2] * (double)m->offset[2];
    v = v + t2[r];
    q.t[r] = (float)v;
  }
  q.fx = (float)K[0];
  q.fy = (float)K[1];
  q.cx = (float)K[2];
  q.cy = (float)K[3];
  return q;
}

/* -------------------------------------------------- first-frame volume */

/* computeBoundingboxIntCPU(ushort), geometryfusion_mipmap_cpu.cpp:1270-1303 */
static void first_frame_bbox(const campams *p, const uint16_t *depth, float scaling, float maxcam, int w, int h,
                             int bw, int *mn, int *mx) {
  for (int y = 0; y < h; y++) {
    for (int x = 0; x < w; x++) {
      float pz = (float)depth[y * w + x] * scaling;
      if (pz > 0.0f && pz < maxcam) {
        float px = ((float)x - p->cx) / p->fx * pz;
        float py = ((float)y - p->cy) / p->fy * pz;
        int v[3];
        for (int r = 0; r < 3; r++) v[r] = (int)(p->r[r * 3 + 0] * px + p->r[r * 3 + 1] * py + p->r[r * 3 + 2] * pz + p->t[r]);
        for (int r = 0; r < 3; r++) {
          if (mn[r] > v[r] - bw) mn[r] = v[r] - bw;
          if (mx[r] < v[r] + bw) mx[r] = v[r] + bw;
        }
      }
    }
  }
}

/* setInitialVolume, geometryfusion_mipmap_cpu.cpp:1186-1233 */
static int set_initial_volume(ffp_map *m, const int *mn, const int *mx) {
  if (mn[0] >= mx[0] || mn[1] >= mx[1] || mn[2] >= mx[2]) return 0;
  uint16_t hi[3];
  for (int r = 0; r < 3; r++) hi[r] = (uint16_t)(mx[r] - mn[r]);
  uint16_t high = hi[0] > hi[1] ? hi[0] : hi[1];
  if (hi[2] > high) high = hi[2];
  uint16_t n;
  for (n = 2 * BL; n <= high; n = (uint16_t)(n * 2)) {
  }
  m->n = n;
  for (int r = 0; r < 3; r++) m->offset[r] = (float)(mn[r] - ((int)n - (int)hi[r]) / 2) * m->scale;
  return 1;
}

/* ------------------------------------------------------------ traversal */

static void queue_leaf(ffp_map *m, uint32_t leaf) {
  if (m->queue_index[leaf] >= m->nqueued) {
    m->queue_index[leaf] = m->nqueued;
    m->queue[m->nqueued++] = leaf;
  }
}

/* queryPointDepthSingle_func_subtree + addLeaf, traversal_functions.cpp:185-211, 308-395 */
static void query_point(ffp_map *m, uint16_t x, uint16_t y, uint16_t z, uint16_t target) {
  uint16_t o[3] = {0, 0, 0};
  uint16_t half = m->n >> 1;
  uint32_t branch = 0;
  uint32_t pl = BRANCHINIT;
  while ((uint16_t)(half >> 1) >= target) {
    uint32_t co = (x >= o[0] + half) * 1 + (y >= o[1] + half) * 2 + (z >= o[2] + half) * 4;
    uint32_t ptr = branch + co + 8;
    uint32_t child = m->tree[ptr];
    uint32_t leaf = m->tree[ptr - 8];
    if (leaf < m->leaves_total) {
      pl = leaf;
      queue_leaf(m, leaf);
    }
    if (child == BRANCHINIT) {
      /* the reference writes past its tree array here when it is full
       * (traversal_functions.cpp:345-354); the restatement stops instead */
      if (m->branches_used + 16 > m->branches_total) {
        m->branch_overflow = 1;
        return;
      }
      m->tree[ptr] = child = m->branches_used;
      m->branches_used += 16;
    }
    o[0] = (uint16_t)(o[0] + half * ((co & 1) != 0));
    o[1] = (uint16_t)(o[1] + half * ((co & 2) != 0));
    o[2] = (uint16_t)(o[2] + half * ((co & 4) != 0));
    branch = child;
    half >>= 1;
  }
  uint32_t co = (x >= o[0] + half) * 1 + (y >= o[1] + half) * 2 + (z >= o[2] + half) * 4;
  uint32_t ptr = branch + co;
  uint32_t child = m->tree[ptr];
  if (child >= BRANCHINIT) {
    m->tree[ptr] = child = m->leaves_used;
    if (child < m->leaves_total) {
      m->leaf_pos[3 * child + 0] = (uint16_t)(o[0] + half * ((co & 1) != 0));
      m->leaf_pos[3 * child + 1] = (uint16_t)(o[1] + half * ((co & 2) != 0));
      m->leaf_pos[3 * child + 2] = (uint16_t)(o[2] + half * ((co & 4) != 0));
      m->leaf_scale[child] = (uint16_t)(half / BL);
      m->leaf_parent[child] = pl;
    }
    m->leaves_used++;
  }
  if (child < m->leaves_total) queue_leaf(m, child);
}

/* leafScaleFunc with SCALE_LINEAR, REFERENCE_DEPTH 1 (inline_functions.hpp:128-145) */
static uint16_t leaf_scale_target(float depth) {
  float factor = depth / 1.0f;
  if (factor < 1.0f) factor = 1.0f;
  return (uint16_t)floorf(factor * (float)BL);
}

/* transformLoopSimPrecalculatedNeg_subtree(ushort), traversal_wrapper_functions.cpp:576-694 */
static void traverse(ffp_map *m, const campams *p, const uint16_t *depth, float scaling, float maxcam) {
  int W = m->img_w, H = m->img_h;
  float *qx = (float *)malloc(sizeof(float) * 3 * W);
  float *qy = (float *)malloc(sizeof(float) * 3 * H);
  for (int x = 0; x < W; x++)
    for (int r = 0; r < 3; r++) qx[3 * x + r] = p->r[r * 3 + 0] * m->pxp[x];
  for (int y = 0; y < H; y++)
    for (int r = 0; r < 3; r++) qy[3 * y + r] = p->r[r * 3 + 1] * m->pyp[y] + p->r[r * 3 + 2];
  int *col = (int *)malloc(sizeof(int) * 3 * W);
  for (int i = 0; i < 3 * W; i++) col[i] = -1;
  int n = m->n, bw = m->bandwidth;
  for (int y = 0; y < H; y++) {
    int row[3] = {-1, -1, -1};
    for (int x = 0; x < W; x++) {
      float d = (float)depth[y * W + x];
      int v[3], k[3];
      for (int r = 0; r < 3; r++) {
        v[r] = (int)((qx[3 * x + r] + qy[3 * y + r]) * d * scaling + p->t[r]);
        k[r] = v[r] & -8;
      }
      float ds = d * scaling;
      int valid = ds > 0.0f && ds < maxcam;
      if (valid && (k[0] != col[3 * x] || k[1] != col[3 * x + 1] || k[2] != col[3 * x + 2]) &&
          (k[0] != row[0] || k[1] != row[1] || k[2] != row[2])) {
        for (int r = 0; r < 3; r++) col[3 * x + r] = row[r] = k[r];
        for (int r = 0; r < 3; r++) {
          int lo = v[r] - bw, hi = v[r] + bw;
          if (lo < 0 && m->box_min[r] > lo) m->box_min[r] = lo;
          if (hi >= n && m->box_max[r] < hi) m->box_max[r] = hi;
        }
        if (v[0] >= 0 && (uint16_t)v[0] < n && v[1] >= 0 && (uint16_t)v[1] < n && v[2] >= 0 &&
            (uint16_t)v[2] < n)
          query_point(m, (uint16_t)v[0], (uint16_t)v[1], (uint16_t)v[2], leaf_scale_target(ds));
      } else {
        for (int r = 0; r < 3; r++) col[3 * x + r] = row[r] = -1;
      }
    }
  }
  free(qx);
  free(qy);
  free(col);
}

/* ----------------------------------------------------------------- grow */

static uint16_t highest_pow2(uint16_t in) {
  uint16_t r = 1;
  while (r * 2 <= in) r = (uint16_t)(r * 2);
  return r;
}

/* grow(), geometryfusion_mipmap_cpu.cpp:3071-3319 */
static int grow(ffp_map *m) {
  int n = m->n;
  uint16_t pl_[3], mi_[3];
  for (int r = 0; r < 3; r++) {
    pl_[r] = (uint16_t)((m->box_max[r] >= n) * ((m->box_max[r] - n) / n + 1));
    mi_[r] = (uint16_t)((m->box_min[r] < 0) * ((-m->box_min[r]) / n + 1));
  }
  for (int r = 0; r < 3; r++) {
    uint16_t cut = pl_[r] & mi_[r];
    if (cut) {
      if (mi_[r] > pl_[r])
        mi_[r] = (uint16_t)(2 * highest_pow2(mi_[r]) + (mi_[r] & (uint16_t)~cut));
      else
        pl_[r] = (uint16_t)(2 * highest_pow2(pl_[r]) + (pl_[r] & (uint16_t)~cut));
    }
  }
  uint16_t levels = highest_pow2(mi_[0]);
  for (int r = 0; r < 3; r++) {
    if (levels < highest_pow2(pl_[r])) levels = highest_pow2(pl_[r]);
    if (levels < highest_pow2(mi_[r])) levels = highest_pow2(mi_[r]);
  }
  uint32_t shift = (uint32_t)levels * 16;
  if (shift > m->branches_total - m->branches_used) return 0;
  /* shiftBranchesMipMap: every child-branch pointer moves by `shift` */
  for (uint32_t b = 0; b < m->branches_used; b += 16)
    for (int c = 8; c < 16; c++)
      if (m->tree[b + c] != BRANCHINIT) m->tree[b + c] += shift;
  memmove(m->tree + shift, m->tree, sizeof(uint32_t) * m->branches_used);
  for (uint32_t i = 0; i < shift; i++) m->tree[i] = BRANCHINIT;
  m->branches_used += shift;
  uint16_t add[3] = {0, 0, 0};
  uint32_t index = (uint32_t)(levels - 1) * 16;
  for (uint16_t level = 0; level < levels; level++) {
    unsigned dec = 1u << level;
    uint32_t co = 0;
    for (int r = 0; r < 3; r++) {
      if ((mi_[r] & dec) || (!(pl_[r] & dec) && (pl_[r] > mi_[r]))) {
        add[r] = (uint16_t)(add[r] + m->n);
        co += 1u << r;
      }
    }
    m->tree[index + co + 8] = index + 16;
    m->n = (uint16_t)(m->n * 2);
    index -= 16;
  }
  for (int r = 0; r < 3; r++) m->offset[r] -= (float)add[r] * m->scale;
  for (uint32_t i = 0; i < m->leaves_used; i++)
    for (int r = 0; r < 3; r++) m->leaf_pos[3 * i + r] = (uint16_t)(m->leaf_pos[3 * i + r] + add[r]);
  m->grows++;
  return 1;
}

/* --------------------------------------------------------------- update */

/* update8AddLoopAVXSingleInteger, update_functions.cpp:1187-1444, one brick.
 * All arithmetic in the caller's rounding mode (round-toward-zero). */
static void update_brick(ffp_map *m, const campams *q, const uint16_t *depth, const uint8_t *rgb, float scaling,
                         float maxcam, uint32_t brick) {
  const float *M = q->r;
  const float m14 = q->t[0], m24 = q->t[1], m34 = q->t[2];
  const int W = m->img_w, H = m->img_h;
  const uint16_t *o = m->leaf_pos + 3 * brick;
  const float ls = (float)m->leaf_scale[brick];
  const float scale = m->scale;
  float fls = ls * scale;
  float ox = (M[0] * (float)o[0] + M[1] * (float)o[1] + M[2] * (float)o[2]) * scale + m14;
  float oy = (M[3] * (float)o[0] + M[4] * (float)o[1] + M[5] * (float)o[2]) * scale + m24;
  float oz = (M[6] * (float)o[0] + M[7] * (float)o[1] + M[8] * (float)o[2]) * scale + m34;
  float d11 = M[0] * fls, d21 = M[3] * fls, d31 = M[6] * fls;
  float d12 = M[1] * fls, d22 = M[4] * fls, d32 = M[7] * fls;
  float d13 = M[2] * fls, d23 = M[5] * fls, d33 = M[8] * fls;
  float kx[8], ky[8], kz[8];
  static const float kmul[8] = {0.0f, 1.0f, 2.0f, 3.0f, 4.0f, 5.0f, 6.0f, 7.0f};
  kx[0] = ky[0] = kz[0] = 0.0f;
  kx[1] = d11;
  ky[1] = d21;
  kz[1] = d31;
  for (int k = 2; k < 8; k++) {
    kx[k] = kmul[k] * d11;
    ky[k] = kmul[k] * d21;
    kz[k] = kmul[k] * d31;
  }
  const float thrD = m->threshold * ls;
  const float thrW = WEIGHT_FACTOR * m->threshold * ls;
  const float fallRcp = recip(thrW - DIST_W_EPS);
  const float colMax = 255.0f * COLOR_MUL;
  float pzx = ox, pzy = oy, pzz = oz;
  size_t idx = (size_t)brick * 512;
  for (int z = 0; z < 8; z++, pzx += d13, pzy += d23, pzz += d33) {
    float pyx = pzx, pyy = pzy, pyz = pzz;
    for (int y = 0; y < 8; y++, pyx += d12, pyy += d22, pyz += d32) {
      for (int k = 0; k < 8; k++, idx++) {
        float px = pyx + kx[k], py = pyy + ky[k], pz = pyz + kz[k];
        float len = sqrtf(px * px + py * py + pz * pz);
        float rc = recip(pz);
        int imx = cvt_rz(q->cx + q->fx * (px * rc));
        int imy = cvt_rz(q->cy + q->fy * (py * rc));
        int cy = imy < H - 1 ? imy : H - 1;
        cy = cy > 0 ? cy : 0;
        int cx = imx < W - 1 ? imx : W - 1;
        cx = cx > 0 ? cx : 0;
        int ii = W * cy + cx;
        float h = scaling * (float)depth[ii];
        float dInc = len - (len * rc) * h;
        int mask = pz > 0.0f && imy < H && imy > -1 && imx < W && imx > -1 && h < maxcam;
        float front = dInc < DIST_W_EPS ? 1.0f : 0.0f;
        float back = (dInc >= DIST_W_EPS && dInc < thrW) ? 1.0f : 0.0f;
        float fall = (thrW - dInc) * fallRcp;
        float wInc = mask ? front + fall * back : 0.0f;
        if (m->conf) wInc = wInc * m->conf[ii];
        float wAcc = m->wgt[idx], dAcc = m->dist[idx];
        float wNew = wAcc + wInc;
        float factor = recip(wNew + (wNew <= 0.0f ? 1.0f : 0.0f));
        float lo = -1.0f * thrD;
        float tr = dInc < thrD ? dInc : thrD;
        tr = tr > lo ? tr : lo;
        float add = mask ? tr * wInc : 0.0f;
        m->dist[idx] = (dAcc * wAcc + add) * factor;
        m->wgt[idx] = wNew;
        if (m->fp16) {
          m->dist[idx] = round_to_half(m->dist[idx]);
          m->wgt[idx] = round_to_half(wNew);
        }
        if (m->color) {
          const uint8_t *px8 = rgb + 3 * (size_t)ii;
          float inc[3] = {(float)px8[2] * COLOR_MUL, (float)px8[1] * COLOR_MUL, (float)px8[0] * COLOR_MUL};
          for (int c = 0; c < 3; c++) {
            float acc = (float)m->col[3 * idx + c];
            float v = (acc * wAcc + inc[c] * wInc) * factor;
            v = v < colMax ? v : colMax;
            m->col[3 * idx + c] = (uint16_t)(int)v;
          }
        }
      }
    }
  }
}

/* The same update in double precision (update mode 3): voxel positions from
 * the double pose and the map offset, exact reciprocals, round-to-nearest;
 * pixel selection and masks as in the reference (truncating conversion). */
static int cvt_trunc64(double f) {
  if (!(f > -2147483649.0 && f < 2147483648.0)) return (int)0x80000000;
  return (int)f;
}

static void update_brick64(ffp_map *m, const double *r2, const double *t2, const double *K, const uint16_t *depth,
                           double scaling, double maxcam, uint32_t brick) {
  const int W = m->img_w, H = m->img_h;
  const uint16_t *o = m->leaf_pos + 3 * brick;
  const double ls = (double)m->leaf_scale[brick];
  const double scale = (double)m->scale;
  const double thr = (double)m->threshold;
  const double thrD = thr * ls, thrW = (double)WEIGHT_FACTOR * thr * ls;
  const double eps = (double)DIST_W_EPS;
  size_t idx = (size_t)brick * 512;
  for (int z = 0; z < 8; z++)
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++, idx++) {
        const double g[3] = {(double)o[0] + x * ls, (double)o[1] + y * ls, (double)o[2] + z * ls};
        double p[3];
        for (int r = 0; r < 3; r++) {
          double v = t2[r];
          for (int c = 0; c < 3; c++) v += r2[r * 3 + c] * ((double)m->offset[c] + g[c] * scale);
          p[r] = v;
        }
        const double len = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        const double rc = 1.0 / p[2];
        const int imx = cvt_trunc64(K[2] + K[0] * (p[0] * rc));
        const int imy = cvt_trunc64(K[3] + K[1] * (p[1] * rc));
        int cy = imy < H - 1 ? imy : H - 1;
        cy = cy > 0 ? cy : 0;
        int cx = imx < W - 1 ? imx : W - 1;
        cx = cx > 0 ? cx : 0;
        const double h = scaling * (double)depth[W * cy + cx];
        const double dInc = len - (len * rc) * h;
        const int mask = p[2] > 0.0 && imy < H && imy > -1 && imx < W && imx > -1 && h < maxcam;
        const double front = dInc < eps ? 1.0 : 0.0;
        const double back = (dInc >= eps && dInc < thrW) ? 1.0 : 0.0;
        const double fall = (thrW - dInc) / (thrW - eps);
        const double wInc = mask ? front + fall * back : 0.0;
        const double wAcc = m->wgt64[idx], dAcc = m->dist64[idx];
        const double wNew = wAcc + wInc;
        double tr = dInc < thrD ? dInc : thrD;
        tr = tr > -thrD ? tr : -thrD;
        const double add = mask ? tr * wInc : 0.0;
        m->dist64[idx] = (dAcc * wAcc + add) / (wNew + (wNew <= 0.0 ? 1.0 : 0.0));
        m->wgt64[idx] = wNew;
      }
}

void ffp_bricks64(const ffp_map *m, int64_t n, double *dist, double *wgt) {
  if (!m->dist64) return;
  memcpy(dist, m->dist64, sizeof(double) * 512 * (size_t)n);
  memcpy(wgt, m->wgt64, sizeof(double) * 512 * (size_t)n);
}

/* ---------------------------------------------------------------- addMap */

int ffp_add_map(ffp_map *m, const uint16_t *depth, const uint8_t *bgr, int w, int h, const double *K,
                const double *R, const double *t, float scaling, float maxcam) {
  campams p = cam_world_to_grid(m, K, R, t);
  for (uint32_t i = 0; i < m->leaves_total; i++) m->queue_index[i] = MAXLEAFNUMBER;
  m->nqueued = 0;
  if (!m->n) {
    int mn[3] = {1000000, 1000000, 1000000}, mx[3] = {-1000000, -1000000, -1000000};
    first_frame_bbox(&p, depth, scaling, maxcam, w, h, m->bandwidth, mn, mx);
    set_initial_volume(m, mn, mx);
    p = cam_world_to_grid(m, K, R, t);
  }
  if (m->img_w != w || m->img_h != h) {
    m->img_w = w;
    m->img_h = h;
    free(m->pxp);
    free(m->pyp);
    m->pxp = (float *)malloc(sizeof(float) * w);
    m->pyp = (float *)malloc(sizeof(float) * h);
    for (int x = 0; x < w; x++) m->pxp[x] = ((float)x - p.cx) / p.fx;
    for (int y = 0; y < h; y++) m->pyp[y] = ((float)y - p.cy) / p.fy;
  }
  for (int r = 0; r < 3; r++) {
    m->box_min[r] = 0;
    m->box_max[r] = m->n - 1;
  }
  /* the voxel->camera parameters are taken before any grow() of this frame */
  campams q = cam_grid_to_camera(m, K, R, t);
  traverse(m, &p, depth, scaling, maxcam);
  if (m->leaves_used < m->leaves_total && m->branches_used < m->branches_total &&
      (m->box_min[0] < 0 || m->box_min[1] < 0 || m->box_min[2] < 0 || m->box_max[0] >= m->n ||
       m->box_max[1] >= m->n || m->box_max[2] >= m->n))
    grow(m);
  int saved = fegetround();
  if (m->rz_exact == 3) {
    /* FP64 oracle: the extrinsic inverse [R^T | -R^T t] in double */
    double r2[9], t2[3];
    for (int r = 0; r < 3; r++) {
      for (int c = 0; c < 3; c++) r2[r * 3 + c] = R[c * 3 + r];
      t2[r] = -(R[0 * 3 + r] * t[0] + R[1 * 3 + r] * t[1] + R[2 * 3 + r] * t[2]);
    }
    fesetround(FE_TONEAREST);
    for (uint32_t i = 0; i < m->nqueued; i++)
      update_brick64(m, r2, t2, K, depth, (double)scaling, (double)maxcam, m->queue[i]);
  } else {
    fesetround(m->rz_exact ? FE_TOWARDZERO : FE_TONEAREST);
    g_rcp_mode = m->rz_exact == 2 ? 2 : 1;
    for (uint32_t i = 0; i < m->nqueued; i++) update_brick(m, &q, depth, bgr, scaling, maxcam, m->queue[i]);
  }
  fesetround(saved);
  if (m->branch_overflow || m->leaves_used > m->leaves_total) m->meshing_ok = 0;
  m->frames++;
  return (int)m->nqueued;
}

/* ------------------------------------------------------------- accessors */

void ffp_state(const ffp_map *m, int64_t *ints, float *offset) {
  ints[0] = m->n;
  ints[1] = m->leaves_used;
  ints[2] = m->branches_used;
  ints[3] = m->nqueued;
  ints[4] = m->leaves_total;
  ints[5] = m->branches_total;
  ints[6] = m->frames;
  ints[7] = m->bandwidth;
  ints[8] = m->meshing_ok;
  ints[9] = m->grows;
  for (int r = 0; r < 3; r++) offset[r] = m->offset[r];
}

void ffp_leaves(const ffp_map *m, uint16_t *pos, uint16_t *scale, uint32_t *parent) {
  uint32_t n = m->leaves_used < m->leaves_total ? m->leaves_used : m->leaves_total;
  memcpy(pos, m->leaf_pos, sizeof(uint16_t) * 3 * n);
  memcpy(scale, m->leaf_scale, sizeof(uint16_t) * n);
  memcpy(parent, m->leaf_parent, sizeof(uint32_t) * n);
}

void ffp_queue(const ffp_map *m, uint32_t *q) { memcpy(q, m->queue, sizeof(uint32_t) * m->nqueued); }

void ffp_tree(const ffp_map *m, uint32_t *tree) { memcpy(tree, m->tree, sizeof(uint32_t) * m->branches_used); }

void ffp_bricks(const ffp_map *m, int64_t n, float *dist, float *wgt, uint16_t *col) {
  memcpy(dist, m->dist, sizeof(float) * 512 * n);
  memcpy(wgt, m->wgt, sizeof(float) * 512 * n);
  memcpy(col, m->col, sizeof(uint16_t) * 512 * 3 * n);
}

void ffp_set_bricks(ffp_map *m, int64_t n, const float *dist, const float *wgt, const uint16_t *col) {
  memcpy(m->dist, dist, sizeof(float) * 512 * n);
  memcpy(m->wgt, wgt, sizeof(float) * 512 * n);
  memcpy(m->col, col, sizeof(uint16_t) * 512 * 3 * n);
}

/* -------------------------------------------------------------- meshing */

/* updateMeshes() with every cell re-meshed from the current voxel data; the
 * cells come in ascending (type, quirk, size, origin) order. */
int64_t ffp_update_meshes(ffp_map *m) {
  free(m->cells);
  free(m->mesh.xyz);
  free(m->mesh.rgb);
  free(m->mesh.faces);
  free(m->mesh.cell_v);
  memset(&m->mesh, 0, sizeof(m->mesh));
  m->cells = NULL;
  m->ncells = 0;
  if (!m->n || !m->meshing_ok) return 0;
  m->ncells = ffp_enumerate_cells(m->tree, m->n, m->leaves_total, &m->cells);
  ffp_mesh_src src;
  src.pos = m->leaf_pos;
  src.scale_of = m->leaf_scale;
  src.parent = m->leaf_parent;
  src.dist = m->dist;
  src.wgt = m->wgt;
  src.col = m->col;
  src.leaves_used = m->leaves_used < m->leaves_total ? m->leaves_used : m->leaves_total;
  for (int r = 0; r < 3; r++) src.offset[r] = m->offset[r];
  src.scale = m->scale;
  ffp_mesh_cells(&src, m->cells, m->ncells, &m->mesh);
  return m->ncells;
}

void ffp_mesh_counts(const ffp_map *m, int64_t *ncells, int64_t *nv, int64_t *nf) {
  *ncells = m->ncells;
  *nv = m->mesh.nv;
  *nf = m->mesh.nf;
}

/* cells: 14 int32 each (type, quirk, ox, oy, oz, size, L0..L7); ranges: 4 int64 each */
void ffp_mesh_copy(const ffp_map *m, int32_t *cells, int64_t *ranges, float *xyz, uint8_t *rgb, uint32_t *faces) {
  for (int64_t i = 0; i < m->ncells; i++) {
    const ffp_cell *e = &m->cells[i];
    int32_t *o = cells + 14 * i;
    o[0] = e->type;
    o[1] = e->quirk;
    o[2] = e->o[0];
    o[3] = e->o[1];
    o[4] = e->o[2];
    o[5] = e->size;
    for (int k = 0; k < 8; k++) o[6 + k] = (int32_t)e->L[k];
  }
  if (m->ncells) memcpy(ranges, m->mesh.cell_v, sizeof(int64_t) * 4 * m->ncells);
  if (m->mesh.nv) {
    memcpy(xyz, m->mesh.xyz, sizeof(float) * 3 * m->mesh.nv);
    memcpy(rgb, m->mesh.rgb, 3 * m->mesh.nv);
  }
  if (m->mesh.nf) memcpy(faces, m->mesh.faces, sizeof(uint32_t) * 3 * m->mesh.nf);
}

/* Replace the whole state (octree, leaf table, bricks) -- e.g. with the
 * compiled reference's, so that meshing can be compared on identical input. */
int ffp_set_state(ffp_map *m, uint32_t n, const float *offset, const uint32_t *tree, uint32_t branches_used,
                  const uint16_t *pos, const uint16_t *scale, const uint32_t *parent, uint32_t leaves_used,
                  const float *dist, const float *wgt, const uint16_t *col) {
  if (branches_used > m->branches_total || leaves_used > m->leaves_total) return -1;
  for (uint32_t i = 0; i < m->branches_total; i++) m->tree[i] = i < branches_used ? tree[i] : BRANCHINIT;
  m->branches_used = branches_used;
  memcpy(m->leaf_pos, pos, sizeof(uint16_t) * 3 * leaves_used);
  memcpy(m->leaf_scale, scale, sizeof(uint16_t) * leaves_used);
  memcpy(m->leaf_parent, parent, sizeof(uint32_t) * leaves_used);
  memcpy(m->dist, dist, sizeof(float) * 512 * (size_t)leaves_used);
  memcpy(m->wgt, wgt, sizeof(float) * 512 * (size_t)leaves_used);
  memcpy(m->col, col, sizeof(uint16_t) * 3 * 512 * (size_t)leaves_used);
  m->leaves_used = leaves_used;
  m->n = (uint16_t)n;
  for (int r = 0; r < 3; r++) m->offset[r] = offset[r];
  m->meshing_ok = 1;
  return 0;
}
