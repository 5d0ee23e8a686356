/*
 * CPU restatement of the reference's incremental marching cubes: the oracle
 * for the meshing stage.  ORACLE INFRASTRUCTURE ONLY (see ff_port.h).
 *
 * Mesh cells.  The reference keeps, per octree slot, lists of "mesh cells"
 * (MeshCell, treeandbrick_incremental.hpp:71-93) that it splits incrementally
 * as branches are created (meshcelltraversalSplitReferenced.hpp:6-790,
 * 2568-5950, 9123-9289).  The cells are the dual cells of the octree of
 * branch slots: one interior cell per unsubdivided slot, one wall per pair of
 * face-adjacent unsubdivided slots, one edge cell per four slots around an
 * edge, one corner cell per eight slots around a vertex, each as large as
 * the smallest slot it touches.  A cell side refers to the finest leaf at or
 * above its slot (lastLeaf).  This file enumerates those cells directly from
 * the octree with the recursive cell/face/edge/vertex traversal; the result is
 * the reference's cell set, cell for cell.
 *
 * Per-cell meshing restates addBrickInterior_indexed_incremental_optimized,
 * addBrickWallX/Y/Z_, addBrickEdgeX/Y/Z_ and addBrickMiddle_indexed_incremental
 * (mesh_interleaved_meshcell.cpp:9-635, 641-2687) with MarchingCubes::
 * getCubeIndex / VertexInterp (mesh.hpp:259-290, mesh.cpp:1266-1340,
 * 1931-2010): round-to-nearest float sampling in the reference's operation
 * order, double-precision vertex interpolation, per-cell vertex de-duplication
 * by (lattice point, axis), and the reference's vertex and face orders.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ff_port.h"
#include "ff_port_internal.h"

#define BRANCHINIT FFP_BRANCHINIT

/* Marching-cubes triangle table of the published method (Lorensen & Cline;
 * the public-domain table of P. Bourke / C. Bloyd that the reference uses):
 * per cube case, the number of triangles in bits 60-63 and up to 15 cube
 * edge numbers, 4 bits each from bit 0.  Edges: 0:(0,1) 1:(1,2) 2:(2,3)
 * 3:(3,0) 4:(4,5) 5:(5,6) 6:(6,7) 7:(7,4) 8:(0,4) 9:(1,5) 10:(2,6) 11:(3,7)
 * over the cube corners (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),
 * (1,1,1),(0,1,1). */
const unsigned long long ffp_mc_tri[256] = {
    0x0000000000000000ull, 0x1000000000000380ull, 0x1000000000000910ull, 0x2000000000189381ull,
    0x1000000000000a21ull, 0x2000000000a21380ull, 0x2000000000920a29ull, 0x300000089a8a2382ull,
    0x10000000000002b3ull, 0x20000000000b82b0ull, 0x2000000000b32091ull, 0x3000000b89b912b1ull,
    0x20000000003ab1a3ull, 0x3000000ab8a801a0ull, 0x30000009ab9b3093ull, 0x2000000000b8aa89ull,
    0x1000000000000874ull, 0x2000000000437034ull, 0x2000000000748910ull, 0x3000000137174914ull,
    0x2000000000748a21ull, 0x3000000a21403743ull, 0x3000000748209a29ull, 0x40004973727929a2ull,
    0x20000000002b3748ull, 0x300000040242b74bull, 0x3000000b32748109ull, 0x40001292b9b49b74ull,
    0x3000000487ab31a3ull, 0x40004b7401b41ab1ull, 0x400030bab9b09874ull, 0x3000000ab99b4b74ull,
    0x1000000000000459ull, 0x2000000000380459ull, 0x2000000000051450ull, 0x3000000513538458ull,
    0x2000000000459a21ull, 0x3000000594a21803ull, 0x3000000204245a25ull, 0x40008434535235a2ull,
    0x2000000000b32459ull, 0x3000000594b802b0ull, 0x3000000b32510450ull, 0x4000584b82852512ull,
    0x300000045931ab3aull, 0x4000ab81a8180594ull, 0x400030bab5b05045ull, 0x3000000b8aa85845ull,
    0x2000000000975879ull, 0x3000000375359039ull, 0x3000000751710870ull, 0x2000000000753351ull,
    0x300000021a759879ull, 0x400037503505921aull, 0x400025a758528208ull, 0x30000007533525a2ull,
    0x30000002b3987597ull, 0x4000b72029279759ull, 0x4000751871810b32ull, 0x300000051771b12bull,
    0x4000b3a31a758859ull, 0x50aba010b7905075ull, 0x507570805a30b0abull, 0x20000000005b75abull,
    0x100000000000056aull, 0x20000000006a5380ull, 0x20000000006a5109ull, 0x30000006a5891381ull,
    0x2000000000162561ull, 0x3000000803621561ull, 0x3000000620609569ull, 0x4000823625285895ull,
    0x200000000056ab32ull, 0x300000056a02b80bull, 0x30000006a5b32910ull, 0x4000b892b92916a5ull,
    0x3000000315356b36ull, 0x40006b51505b0b80ull, 0x40009505606306b3ull, 0x300000089bb96956ull,
    0x20000000008746a5ull, 0x3000000a56374034ull, 0x30000007486a5091ull, 0x400049737179156aull,
    0x3000000874156216ull, 0x4000743403625521ull, 0x4000620560509748ull, 0x5962695923497937ull,
    0x300000056a4872b3ull, 0x4000b720242746a5ull, 0x40006a5b32874910ull, 0x56a54b7b492b9129ull,
    0x40006b51535b3748ull, 0x5b404b7b016b5b15ull, 0x574836b630560950ull, 0x40009b7974b96956ull,
    0x2000000000a4694aull, 0x3000000380a946a4ull, 0x300000004606a10aull, 0x4000a16468618138ull,
    0x3000000462421941ull, 0x4000462942921803ull, 0x2000000000624420ull, 0x3000000624428238ull,
    0x300000032b46a94aull, 0x40006a4a94b82280ull, 0x4000a164606102b3ull, 0x51b8b12184a16146ull,
    0x400036b319639469ull, 0x514641916b0181b8ull, 0x30000004600636b3ull, 0x200000000086b846ull,
    0x3000000a98a876a7ull, 0x4000a76a907a0370ull, 0x40000818717a176aull, 0x300000037117a76aull,
    0x4000768981861621ull, 0x5937390976192962ull, 0x3000000206607087ull, 0x2000000000276237ull,
    0x400076898a86ab32ull, 0x57a9a76790b72702ull, 0x5b32a767a1871081ull, 0x400017616a71b12bull,
    0x563136b619768698ull, 0x200000000076b190ull, 0x400006b0b3607087ull, 0x10000000000006b7ull,
    0x1000000000000b67ull, 0x200000000067b803ull, 0x200000000067b910ull, 0x300000067b138918ull,
    0x20000000007b621aull, 0x30000007b6803a21ull, 0x30000007b69a2092ull, 0x400089a38a3a27b6ull,
    0x2000000000726327ull, 0x3000000026067807ull, 0x3000000910732672ull, 0x4000678891681261ull,
    0x300000073171a67aull, 0x4000801781a7167aull, 0x40007a69a0a70730ull, 0x30000009a88a7a67ull,
    0x200000000068b486ull, 0x3000000640603b63ull, 0x3000000109648b68ull, 0x400063b139369649ull,
    0x30000001a28b6486ull, 0x4000640b60b03a21ull, 0x40009a2920b648b4ull, 0x536463b34923a39aull,
    0x3000000264248328ull, 0x2000000000264240ull, 0x4000834642432091ull, 0x3000000642241491ull,
    0x40001a6648168318ull, 0x300000040660a01aull, 0x539a9303a6834364ull, 0x20000000004a649aull,
    0x2000000000b67594ull, 0x300000067b594380ull, 0x3000000b67045105ull, 0x400051345343867bull,
    0x3000000b6721a459ull, 0x4000594380a217b6ull, 0x4000204a24a45b67ull, 0x567b25a523453843ull,
    0x3000000945267327ull, 0x4000786260680459ull, 0x4000045051673263ull, 0x5851584812786826ull,
    0x400073167161a459ull, 0x5459078701671a61ull, 0x5a737a6a305a4a04ull, 0x4000a84a458a7a67ull,
    0x300000098b9b6596ull, 0x4000590650360b63ull, 0x4000b65510b508b0ull, 0x30000001355363b6ull,
    0x400065b8b9b59a21ull, 0x5a21965690b603b0ull, 0x552025a50865b58bull, 0x400035a3a25363b6ull,
    0x4000283265825985ull, 0x3000000260069659ull, 0x5826283865081851ull, 0x2000000000612651ull,
    0x5698965683a61631ull, 0x400006505960a01aull, 0x2000000000a65830ull, 0x100000000000065aull,
    0x2000000000b57a5bull, 0x300000003857ba5bull, 0x3000000091ba57b5ull, 0x40001381897ba57aull,
    0x300000015717b21bull, 0x4000b27571721380ull, 0x40007b2209729579ull, 0x5289823295b27257ull,
    0x3000000573532a52ull, 0x400052a578258028ull, 0x40002a37353a5109ull, 0x525752a278129289ull,
    0x2000000000573531ull, 0x3000000571170780ull, 0x3000000735539309ull, 0x2000000000795789ull,
    0x30000008ba8a5485ull, 0x400003bba50b5405ull, 0x400054aba8a48910ull, 0x541314943b54a4baull,
    0x40008548b2582152ull, 0x5b151b2b543b0b40ull, 0x558b8545b2950520ull, 0x20000000003b2549ull,
    0x4000483543253a52ull, 0x30000000244252a5ull, 0x5910854583a532a3ull, 0x40002492914252a5ull,
    0x3000000153358548ull, 0x2000000000501540ull, 0x4000530509358548ull, 0x1000000000000549ull,
    0x3000000ba9b947b4ull, 0x4000ba97b9794380ull, 0x4000b470414b1ba1ull, 0x54bab474a1843413ull,
    0x4000219b294b97b4ull, 0x53801b2b197b9479ull, 0x300000004224b47bull, 0x400042343824b47bull,
    0x4000947732972a92ull, 0x570207872a4797a9ull, 0x5a040a1a472a3a73ull, 0x20000000004782a1ull,
    0x3000000317714194ull, 0x4000178180714194ull, 0x2000000000347304ull, 0x1000000000000784ull,
    0x20000000008ba8a9ull, 0x3000000a9bb93903ull, 0x3000000ba88a0a10ull, 0x2000000000a3ba13ull,
    0x30000008b99b1b21ull, 0x40009b2921b93903ull, 0x2000000000b08b20ull, 0x1000000000000b23ull,
    0x300000098aa82832ull, 0x20000000002902a9ull, 0x40008a1810a82832ull, 0x10000000000002a1ull,
    0x2000000000819831ull, 0x1000000000000190ull, 0x1000000000000830ull, 0x0000000000000000ull,
};

static const int EDGE_A[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
static const int EDGE_B[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
/* edge -> (corner offset (dx,dy,dz), axis) of the lattice edge it lies on */
static const int EDGE_SLOT[12][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {0, 1, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {1, 0, 1, 1},
                                    {0, 1, 1, 0}, {0, 0, 1, 1}, {0, 0, 0, 2}, {1, 0, 0, 2}, {1, 1, 0, 2}, {0, 1, 0, 2}};

int ffp_mc_ntri(int c) { return (int)(ffp_mc_tri[c] >> 60); }
int ffp_mc_edge(int c, int k) { return (int)((ffp_mc_tri[c] >> (4 * k)) & 15u); }

/* ---------------------------------------------------------------------------
 * Dual-cell enumeration
 * ------------------------------------------------------------------------- */

typedef struct {
  uint32_t S; /* tree entry of the slot (its leaf); child branch at S+8 */
  int o[3];
  int size;
  uint32_t la; /* finest leaf at or above */
} slot_t;

typedef struct {
  const uint32_t *tree;
  uint32_t leaves_total;
  ffp_cell *cells;
  int64_t n, cap;
} enum_ctx;

static int is_sub(const enum_ctx *c, const slot_t *s) { return c->tree[s->S + 8] < BRANCHINIT; }

static slot_t child_of(const enum_ctx *c, const slot_t *s, int co) {
  slot_t r;
  uint32_t sub = c->tree[s->S + 8];
  int h = s->size / 2;
  r.S = sub + (uint32_t)co;
  r.o[0] = s->o[0] + h * (co & 1);
  r.o[1] = s->o[1] + h * ((co >> 1) & 1);
  r.o[2] = s->o[2] + h * ((co >> 2) & 1);
  r.size = h;
  uint32_t lf = c->tree[r.S];
  r.la = lf < c->leaves_total ? lf : s->la;
  return r;
}

static slot_t ch(const enum_ctx *c, const slot_t *s, int co) { return is_sub(c, s) ? child_of(c, s, co) : *s; }

static void emit(enum_ctx *c, int type, const int *o, int size, const uint32_t *L, int nl) {
  for (int k = 0; k < nl; k++)
    if (L[k] >= BRANCHINIT) return; /* never meshed: some side has no leaf */
  if (c->n == c->cap) {
    c->cap = c->cap ? 2 * c->cap : 4096;
    c->cells = (ffp_cell *)realloc(c->cells, sizeof(ffp_cell) * c->cap);
  }
  ffp_cell *e = &c->cells[c->n++];
  e->type = type;
  e->quirk = 0;
  for (int r = 0; r < 3; r++) e->o[r] = o[r];
  e->size = size;
  for (int k = 0; k < 8; k++) e->L[k] = k < nl ? L[k] : BRANCHINIT;
}

static void vert_proc(enum_ctx *c, const slot_t *S8) {
  int any = 0;
  for (int j = 0; j < 8; j++) any |= is_sub(c, &S8[j]);
  if (any) {
    slot_t T[8];
    for (int j = 0; j < 8; j++) T[j] = ch(c, &S8[j], 7 - j);
    vert_proc(c, T);
    return;
  }
  /* the vertex is a corner of the smallest slot around it */
  int size = S8[0].size, small = 0;
  for (int j = 1; j < 8; j++)
    if (S8[j].size < size) size = S8[j].size, small = j;
  int o[3];
  for (int r = 0; r < 3; r++) o[r] = S8[small].o[r] + (((small >> r) & 1) ? 0 : size) - size;
  uint32_t L[8];
  for (int j = 0; j < 8; j++) L[j] = S8[j].la;
  emit(c, 7, o, size, L, 8);
}

/* the two axes other than e, ascending */
static void others(int e, int *p, int *q) {
  *p = e == 0 ? 1 : 0;
  *q = e == 2 ? 1 : 2;
}

/* S4: slots around an edge along axis e, ordered (p-,q-), (p+,q-), (p-,q+), (p+,q+) */
static void edge_proc(enum_ctx *c, const slot_t *S4, int e) {
  int any = 0;
  for (int j = 0; j < 4; j++) any |= is_sub(c, &S4[j]);
  int p, q;
  others(e, &p, &q);
  if (!any) {
    int size = S4[0].size, small = 0;
    for (int j = 1; j < 4; j++)
      if (S4[j].size < size) size = S4[j].size, small = j;
    /* the edge line runs along a side of the smallest slot */
    int o[3];
    o[e] = S4[small].o[e];
    o[p] = S4[small].o[p] + ((small & 1) ? 0 : size) - size;
    o[q] = S4[small].o[q] + ((small & 2) ? 0 : size) - size;
    uint32_t L[4] = {S4[0].la, S4[1].la, S4[2].la, S4[3].la};
    emit(c, 4 + e, o, size, L, 4);
    return;
  }
  for (int half = 0; half < 2; half++) {
    slot_t T[4];
    for (int j = 0; j < 4; j++) {
      int k = ((j & 1) ? 0 : (1 << p)) | (((j >> 1) & 1) ? 0 : (1 << q)) | (half ? (1 << e) : 0);
      T[j] = ch(c, &S4[j], k);
    }
    edge_proc(c, T, e);
  }
  slot_t S8[8];
  for (int j = 0; j < 8; j++) {
    int pj = (j >> p) & 1, qj = (j >> q) & 1, ej = (j >> e) & 1;
    /* across the edge line: the half of the slot next to the line; along
     * the edge: the half on the vertex's own side of the midpoint */
    int k = (pj ? 0 : (1 << p)) | (qj ? 0 : (1 << q)) | (ej ? (1 << e) : 0);
    S8[j] = ch(c, &S4[pj | (qj << 1)], k);
  }
  vert_proc(c, S8);
}

static void face_proc(enum_ctx *c, const slot_t *A, const slot_t *B, int ax) {
  if (!is_sub(c, A) && !is_sub(c, B)) {
    int size = A->size < B->size ? A->size : B->size;
    const slot_t *small = A->size <= B->size ? A : B;
    int o[3] = {small->o[0], small->o[1], small->o[2]};
    o[ax] = B->o[ax] - size;
    uint32_t L[2] = {A->la, B->la};
    emit(c, 1 + ax, o, size, L, 2);
    return;
  }
  int bit = 1 << ax, u, v;
  others(ax, &u, &v);
  for (int qd = 0; qd < 4; qd++) {
    int k = ((qd & 1) ? (1 << u) : 0) | ((qd & 2) ? (1 << v) : 0);
    slot_t a = ch(c, A, k | bit), b = ch(c, B, k);
    face_proc(c, &a, &b, ax);
  }
  /* the four edges in the face plane: along u (at v mid) and along v (at u mid) */
  for (int t = 0; t < 2; t++) {
    int e = t == 0 ? u : v;
    int other = t == 0 ? v : u;
    int p, q;
    others(e, &p, &q);
    for (int half = 0; half < 2; half++) {
      slot_t S4[4];
      for (int j = 0; j < 4; j++) {
        int side[3] = {0, 0, 0};
        side[p] = j & 1;
        side[q] = (j >> 1) & 1;
        int k = (half ? (1 << e) : 0) | (side[other] ? (1 << other) : 0);
        S4[j] = side[ax] ? ch(c, B, k) : ch(c, A, k | bit);
      }
      edge_proc(c, S4, e);
    }
  }
  slot_t S8[8];
  for (int j = 0; j < 8; j++) {
    int k = j & ~bit;
    S8[j] = ((j >> ax) & 1) ? ch(c, B, k) : ch(c, A, k | bit);
  }
  vert_proc(c, S8);
}

static void cell_children(enum_ctx *c, const slot_t *C) {
  static const int FX[4][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}};
  static const int FY[4][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}};
  static const int FZ[4][2] = {{0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int j = 0; j < 8; j++) {
    if (is_sub(c, &C[j])) {
      slot_t T[8];
      for (int k = 0; k < 8; k++) T[k] = child_of(c, &C[j], k);
      cell_children(c, T);
    } else {
      uint32_t L[1] = {C[j].la};
      emit(c, 0, C[j].o, C[j].size, L, 1);
    }
  }
  for (int i = 0; i < 4; i++) face_proc(c, &C[FX[i][0]], &C[FX[i][1]], 0);
  for (int i = 0; i < 4; i++) face_proc(c, &C[FY[i][0]], &C[FY[i][1]], 1);
  for (int i = 0; i < 4; i++) face_proc(c, &C[FZ[i][0]], &C[FZ[i][1]], 2);
  for (int x = 0; x < 2; x++) {
    slot_t S4[4] = {C[x], C[x | 2], C[x | 4], C[x | 6]};
    edge_proc(c, S4, 0);
  }
  for (int y = 0; y < 4; y += 2) {
    slot_t S4[4] = {C[y], C[y | 1], C[y | 4], C[y | 5]};
    edge_proc(c, S4, 1);
  }
  for (int z = 0; z < 8; z += 4) {
    slot_t S4[4] = {C[z], C[z | 1], C[z | 2], C[z | 3]};
    edge_proc(c, S4, 2);
  }
  vert_proc(c, C);
}

static uint64_t cell_key(const ffp_cell *e) {
  int lsz = 0;
  while ((1 << lsz) < e->size) lsz++;
  return ((uint64_t)e->type << 54) | ((uint64_t)e->quirk << 53) | ((uint64_t)lsz << 48) |
         ((uint64_t)(uint16_t)e->o[0] << 32) | ((uint64_t)(uint16_t)e->o[1] << 16) | (uint64_t)(uint16_t)e->o[2];
}

static int cmp_cell(const void *a, const void *b) {
  uint64_t ka = cell_key((const ffp_cell *)a), kb = cell_key((const ffp_cell *)b);
  return ka < kb ? -1 : ka > kb;
}

int64_t ffp_enumerate_cells(const uint32_t *tree, uint32_t n, uint32_t leaves_total, ffp_cell **out) {
  enum_ctx c = {tree, leaves_total, NULL, 0, 0};
  if (n >= 16) {
    slot_t C[8];
    int h = (int)n / 2;
    for (int co = 0; co < 8; co++) {
      C[co].S = (uint32_t)co;
      C[co].o[0] = h * (co & 1);
      C[co].o[1] = h * ((co >> 1) & 1);
      C[co].o[2] = h * ((co >> 2) & 1);
      C[co].size = h;
      C[co].la = tree[co] < leaves_total ? tree[co] : BRANCHINIT;
    }
    cell_children(&c, C);
  }
  qsort(c.cells, (size_t)c.n, sizeof(ffp_cell), cmp_cell);
  *out = c.cells;
  return c.n;
}

/* ---------------------------------------------------------------------------
 * Per-cell marching cubes
 * ------------------------------------------------------------------------- */

typedef struct {
  float d, w;
  uint16_t c[3];
} sample_t;

/* MarchingCubes::VertexInterp(Vertex3f, Vertex3f, double, double), mesh.cpp:1266-1315 */
static void vinterp(const float *p1, const float *p2, double v1, double v2, float *out) {
  if (fabs(0.0 - v1) < 1e-40) {
    memcpy(out, p1, 12);
    return;
  }
  if (fabs(0.0 - v2) < 1e-40) {
    memcpy(out, p2, 12);
    return;
  }
  if (fabs(v1 - v2) < 1e-40) {
    memcpy(out, p1, 12);
    return;
  }
  double mu = (0.0 - v1) / (v2 - v1);
  for (int r = 0; r < 3; r++) {
    double dd = (double)p2[r] - (double)p1[r];
    out[r] = (float)((double)p1[r] + mu * dd);
  }
}

/* MarchingCubes::VertexInterp(VertexColor, ...), mesh.cpp:1317-1340 */
static void cinterp(const uint16_t *c1, const uint16_t *c2, float v1, float v2, uint16_t *out) {
  if (fabsf(0.0f - v1) < 1e-40) {
    memcpy(out, c1, 6);
    return;
  }
  if (fabsf(0.0f - v2) < 1e-40) {
    memcpy(out, c2, 6);
    return;
  }
  if (fabsf(v1 - v2) < 1e-40) {
    memcpy(out, c1, 6);
    return;
  }
  float mu = (0.0f - v1) / (v2 - v1);
  for (int r = 0; r < 3; r++) {
    float p = (float)c1[r] + mu * ((float)c2[r] - (float)c1[r]);
    out[r] = p <= 65280.0f ? (p >= 0.0f ? (uint16_t)p : 0) : 65280;
  }
}

static int cube_case(const sample_t *s, int idx) {
  static const int off[8] = {0, 1, 9, 8, 64, 65, 73, 72};
  for (int k = 0; k < 8; k++)
    if (s[idx + off[k]].w == 0.0f) return 0;
  int ci = 0;
  for (int k = 0; k < 8; k++)
    if (s[idx + off[k]].d < 0.0f) ci |= 1 << k;
  return ci;
}

/* voxel index of (lx,ly,lz) in a leaf, with the reference's uint16 wrap */
static size_t vox_index(const ffp_mesh_src *m, uint32_t leaf, uint16_t lx, uint16_t ly, uint16_t lz) {
  size_t i = (size_t)leaf * 512 + ((size_t)lz * 8 + ly) * 8 + lx;
  size_t lim = (size_t)m->leaves_used * 512;
  return i < lim ? i : lim - 1; /* the reference would read past its pool here */
}

static void sample_corner_voxel(const ffp_mesh_src *m, uint32_t leaf, size_t vi, sample_t *s) {
  (void)leaf;
  s->d = m->dist[vi];
  s->w += m->wgt[vi];
  for (int r = 0; r < 3; r++) s->c[r] = m->col[3 * vi + r];
}

typedef struct {
  float *xyz;
  uint8_t *rgb;
  uint32_t *faces;
  int64_t nv, nf, capv, capf;
} mesh_buf;

static void push_vertex(mesh_buf *b, const float *p, const uint16_t *c) {
  if (b->nv == b->capv) {
    b->capv = b->capv ? 2 * b->capv : 65536;
    b->xyz = (float *)realloc(b->xyz, sizeof(float) * 3 * b->capv);
    b->rgb = (uint8_t *)realloc(b->rgb, 3 * b->capv);
  }
  memcpy(b->xyz + 3 * b->nv, p, 12);
  for (int r = 0; r < 3; r++) b->rgb[3 * b->nv + r] = (uint8_t)(c[r] / 256);
  b->nv++;
}

static void push_face(mesh_buf *b, uint32_t a, uint32_t c, uint32_t d) {
  if (b->nf == b->capf) {
    b->capf = b->capf ? 2 * b->capf : 65536;
    b->faces = (uint32_t *)realloc(b->faces, sizeof(uint32_t) * 3 * b->capf);
  }
  b->faces[3 * b->nf] = a;
  b->faces[3 * b->nf + 1] = c;
  b->faces[3 * b->nf + 2] = d;
  b->nf++;
}

/* addBrickMiddle_indexed_incremental (mesh_interleaved_meshcell.cpp:2480-2687) */
static void mesh_corner(const ffp_mesh_src *m, const ffp_cell *e, mesh_buf *b) {
  const uint32_t *L = e->L;
  int stretch = m->scale_of[L[0]];
  for (int i = 1; i < 7; i++)
    if (stretch < m->scale_of[L[i]]) stretch = m->scale_of[L[i]];
  if (stretch > e->size) return;
  sample_t s[8];
  for (int i = 0; i < 8; i++) {
    int p[3];
    for (int r = 0; r < 3; r++) p[r] = ((i >> r) & 1) ? e->o[r] + e->size : e->o[r] + e->size - stretch;
    s[i].w = 0.0f;
    s[i].d = 0.0f;
    s[i].c[0] = s[i].c[1] = s[i].c[2] = 0;
    for (uint32_t leaf = L[i]; leaf < BRANCHINIT && s[i].w <= 0.0f; leaf = m->parent[leaf]) {
      const uint16_t *lo = m->pos + 3 * (size_t)leaf;
      int ls = m->scale_of[leaf];
      uint16_t l[3];
      for (int r = 0; r < 3; r++) l[r] = (uint16_t)(((int)(uint16_t)p[r] - (int)lo[r]) / ls);
      sample_corner_voxel(m, leaf, vox_index(m, leaf, l[0], l[1], l[2]), &s[i]);
    }
  }
  /* cube corners in marching-cubes order from the sample bits (x, y, z) */
  static const int mcv[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  float val[8], wv[8];
  const uint16_t *cv[8];
  for (int k = 0; k < 8; k++) {
    val[k] = s[mcv[k]].d;
    wv[k] = s[mcv[k]].w;
    cv[k] = s[mcv[k]].c;
  }
  int ci = 0, zero = 0;
  for (int k = 0; k < 8; k++) zero |= wv[k] == 0.0f;
  if (!zero)
    for (int k = 0; k < 8; k++)
      if (val[k] < 0.0f) ci |= 1 << k;
  float ox = m->offset[0] + (float)(e->o[0] + e->size - stretch) * m->scale;
  float oy = m->offset[1] + (float)(e->o[1] + e->size - stretch) * m->scale;
  float oz = m->offset[2] + (float)(e->o[2] + e->size - stretch) * m->scale;
  float sx = m->scale * (float)stretch;
  float P[8][3];
  for (int k = 0; k < 8; k++) {
    int bx = (k == 1 || k == 2 || k == 5 || k == 6), by = (k == 2 || k == 3 || k == 6 || k == 7), bz = k >= 4;
    P[k][0] = ox + (float)bx * sx;
    P[k][1] = oy + (float)by * sx;
    P[k][2] = oz + (float)bz * sx;
  }
  float vl[12][3];
  uint16_t cl[12][3];
  for (int ed = 0; ed < 12; ed++) {
    int a = EDGE_A[ed], c = EDGE_B[ed];
    if (((ci >> a) & 1) != ((ci >> c) & 1)) {
      vinterp(P[a], P[c], val[a], val[c], vl[ed]);
      cinterp(cv[a], cv[c], val[a], val[c], cl[ed]);
    }
  }
  int nt = ffp_mc_ntri(ci);
  for (int t = 0; t < nt; t++) {
    int e0 = ffp_mc_edge(ci, 3 * t), e1 = ffp_mc_edge(ci, 3 * t + 1), e2 = ffp_mc_edge(ci, 3 * t + 2);
    const float *v0 = vl[e0], *v1 = vl[e1], *v2 = vl[e2];
    int deg = (v0[0] == v1[0] && v0[1] == v1[1] && v0[2] == v1[2]) ||
              (v2[0] == v1[0] && v2[1] == v1[1] && v2[2] == v1[2]) ||
              (v0[0] == v2[0] && v0[1] == v2[1] && v0[2] == v2[2]);
    if (deg) continue;
    uint32_t base = (uint32_t)b->nv;
    push_vertex(b, v0, cl[e0]);
    push_vertex(b, v1, cl[e1]);
    push_vertex(b, v2, cl[e2]);
    push_face(b, base, base + 1, base + 2);
  }
}

/* Roles of the three axes of a cell type: 0 = lattice of spacing sizeMin,
 * 1 = the two samples either side of the shared boundary. */
static const int ROLE[7][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};

/* Interior, walls and edges: sample lattice, cube cases, vertices, faces. */
static void mesh_lattice(const ffp_mesh_src *m, const ffp_cell *e, mesh_buf *b) {
  const int t = e->type;
  const uint32_t *L = e->L;
  const int size = e->size;
  int sizeMin, stretch = 0;
  if (t == 0) {
    sizeMin = m->scale_of[L[0]];
    if (sizeMin > size) return;
    if (size / sizeMin > 8) return;
  } else if (t <= 3) {
    int a = m->scale_of[L[0]], c = m->scale_of[L[1]];
    sizeMin = a < c ? a : c;
    stretch = a;
    if (stretch > size) return;
  } else {
    int s0 = m->scale_of[L[0]], s1 = m->scale_of[L[1]], s2 = m->scale_of[L[2]], s3 = m->scale_of[L[3]];
    stretch = s0 > s1 ? s0 : s1;
    if (s2 > stretch) stretch = s2;
    int a = s0 < s1 ? s0 : s1, c = s2 < s3 ? s2 : s3;
    sizeMin = a < c ? a : c;
    if (stretch > size) return;
  }
  const int *role = ROLE[t];
  int cnt[3];
  for (int r = 0; r < 3; r++) cnt[r] = role[r] ? 2 : (size + sizeMin - 1) / sizeMin;
  /* integer sample coordinates along each axis */
  int pos[3][8];
  for (int r = 0; r < 3; r++)
    for (int k = 0; k < cnt[r]; k++)
      pos[r][k] = role[r] ? (k ? e->o[r] + size : e->o[r] + size - stretch) : e->o[r] + k * sizeMin;
  if (t == 0) {
    /* the interior cell must lie inside its leaf (mesh_interleaved_meshcell.cpp:65-71) */
    const uint16_t *lo = m->pos + 3 * (size_t)L[0];
    int ext = m->scale_of[L[0]] * 8;
    for (int r = 0; r < 3; r++)
      if (e->o[r] + size > lo[r] + ext || e->o[r] < lo[r]) return;
  }
  sample_t s[512];
  memset(s, 0, sizeof(s));
  for (int bz = 0; bz < cnt[2]; bz++)
    for (int by = 0; by < cnt[1]; by++)
      for (int bx = 0; bx < cnt[0]; bx++) {
        const int idx = (bz * 8 + by) * 8 + bx;
        const int bb[3] = {bx, by, bz};
        uint32_t first;
        if (t == 0)
          first = L[0];
        else if (t <= 3)
          first = L[bb[t - 1]];
        else {
          int p, q;
          others(t - 4, &p, &q);
          first = L[bb[p] + 2 * bb[q]];
        }
        sample_t *sp = &s[idx];
        sp->w = 0.0f;
        for (uint32_t leaf = first; leaf < BRANCHINIT && sp->w <= 0.0f; leaf = m->parent[leaf]) {
          const uint16_t *lo = m->pos + 3 * (size_t)leaf;
          const int ls = m->scale_of[leaf];
          if (t == 0) {
            int ext = ls * 8;
            for (int r = 0; r < 3; r++)
              if (e->o[r] + size > lo[r] + ext || e->o[r] < lo[r]) return;
          }
          uint16_t ll[3], lh[3];
          float rr[3];
          for (int r = 0; r < 3; r++) {
            const int p = pos[r][bb[r]];
            ll[r] = (uint16_t)((p - (int)lo[r]) / ls);
            if (role[r]) {
              lh[r] = ll[r];
              rr[r] = 0.0f;
            } else {
              uint16_t rem = (uint16_t)((p - (int)lo[r]) % ls);
              rr[r] = (float)rem / (float)ls;
              lh[r] = (uint16_t)(ll[r] + (rr[r] > 0.0 && ll[r] < 7));
            }
          }
          if (t == 0) {
            /* trilinear, summed as the reference's SSE code does (:144-230) */
            const float rx = rr[0], ry = rr[1], rz = rr[2];
            const float rxn = 1.0f - rx, ryn = 1.0f - ry, rzn = 1.0f - rz;
            const float f[8] = {rzn * ryn * rxn, rzn * ryn * rx, rzn * ry * rxn, rzn * ry * rx,
                                rz * ryn * rxn,  rz * ryn * rx,  rz * ry * rxn,  rz * ry * rx};
            size_t vi[8];
            for (int k = 0; k < 8; k++)
              vi[k] = vox_index(m, leaf, (k & 1) ? lh[0] : ll[0], (k & 2) ? lh[1] : ll[1], (k & 4) ? lh[2] : ll[2]);
            float df[8], cf[3][8];
            for (int k = 0; k < 8; k++) {
              df[k] = m->dist[vi[k]];
              for (int r = 0; r < 3; r++) cf[r][k] = (float)m->col[3 * vi[k] + r];
            }
            sp->w += m->wgt[vi[0]];
            sp->d = ((f[0] * df[0] + f[4] * df[4]) + (f[1] * df[1] + f[5] * df[5])) +
                    ((f[2] * df[2] + f[6] * df[6]) + (f[3] * df[3] + f[7] * df[7]));
            for (int r = 0; r < 3; r++) {
              float v = ((f[0] * cf[r][0] + f[4] * cf[r][4]) + (f[1] * cf[r][1] + f[5] * cf[r][5])) +
                        ((f[2] * cf[r][2] + f[6] * cf[r][6]) + (f[3] * cf[r][3] + f[7] * cf[r][7]));
              sp->c[r] = (uint16_t)(int)v;
            }
          } else if (t <= 3) {
            /* bilinear over the two lattice axes a (low) and c (high) */
            int a = -1, c = -1;
            for (int r = 0; r < 3; r++)
              if (!role[r]) {
                if (a < 0) a = r; else c = r;
              }
            const float ra = rr[a], rc = rr[c], ran = 1.0f - ra, rcn = 1.0f - rc;
            size_t vi[4];
            for (int k = 0; k < 4; k++) {
              uint16_t l3[3] = {ll[0], ll[1], ll[2]};
              l3[a] = (k & 1) ? lh[a] : ll[a];
              l3[c] = (k & 2) ? lh[c] : ll[c];
              vi[k] = vox_index(m, leaf, l3[0], l3[1], l3[2]);
            }
            float wf[4], df[4], cf[3][4];
            for (int k = 0; k < 4; k++) {
              wf[k] = m->wgt[vi[k]];
              df[k] = m->dist[vi[k]];
              for (int r = 0; r < 3; r++) cf[r][k] = (float)m->col[3 * vi[k] + r];
            }
            sp->w += rcn * ran * wf[0] + rcn * ra * wf[1] + rc * ran * wf[2] + rc * ra * wf[3];
            sp->d = rcn * ran * df[0] + rcn * ra * df[1] + rc * ran * df[2] + rc * ra * df[3];
            for (int r = 0; r < 3; r++) {
              float v = rcn * ran * cf[r][0] + rcn * ra * cf[r][1] + rc * ran * cf[r][2] + rc * ra * cf[r][3];
              sp->c[r] = (uint16_t)(int)v;
            }
          } else {
            /* linear along the edge axis, weight = max of the two */
            const int a = t - 4;
            const float ra = rr[a];
            uint16_t l3[3] = {ll[0], ll[1], ll[2]};
            const size_t v0 = vox_index(m, leaf, l3[0], l3[1], l3[2]);
            l3[a] = lh[a];
            const size_t v1 = vox_index(m, leaf, l3[0], l3[1], l3[2]);
            const float w0 = m->wgt[v0], w1 = m->wgt[v1];
            sp->w += w0 > w1 ? w0 : w1;
            sp->d = (1.0f - ra) * m->dist[v0] + ra * m->dist[v1];
            for (int r = 0; r < 3; r++) {
              float v = (1.0f - ra) * (float)m->col[3 * v0 + r] + ra * (float)m->col[3 * v1 + r];
              sp->c[r] = (uint16_t)(int)v;
            }
          }
        }
      }
  /* cubes: case per cube, and which (lattice point, axis) edges carry a vertex */
  int ncube[3];
  for (int r = 0; r < 3; r++) ncube[r] = cnt[r] - 1;
  unsigned char caseOf[512];
  unsigned char edgeSet[512 * 3];
  memset(caseOf, 0, sizeof(caseOf));
  memset(edgeSet, 0, sizeof(edgeSet));
  for (int bz = 0; bz < ncube[2]; bz++)
    for (int by = 0; by < ncube[1]; by++)
      for (int bx = 0; bx < ncube[0]; bx++) {
        int idx = (bz * 8 + by) * 8 + bx;
        int ci = cube_case(s, idx);
        caseOf[idx] = (unsigned char)ci;
        int nt = ffp_mc_ntri(ci);
        for (int k = 0; k < 3 * nt; k++) {
          const int *es = EDGE_SLOT[ffp_mc_edge(ci, k)];
          edgeSet[3 * (idx + es[0] + 8 * es[1] + 64 * es[2]) + es[3]] = 1;
        }
      }
  /* vertices in the reference's loop order of this cell type */
  uint32_t vidx[512 * 3];
  int order[3]; /* outer .. inner axis */
  switch (t) {
    case 0: case 1: order[0] = 2; order[1] = 1; order[2] = 0; break;
    case 2: order[0] = 2; order[1] = 0; order[2] = 1; break;
    case 3: order[0] = 1; order[1] = 0; order[2] = 2; break;
    case 4: order[0] = 0; order[1] = 2; order[2] = 1; break;
    case 5: order[0] = 1; order[1] = 2; order[2] = 0; break;
    default: order[0] = 2; order[1] = 1; order[2] = 0; break;
  }
  float P0[3];
  uint32_t base = (uint32_t)b->nv;
  for (int i0 = 0; i0 < cnt[order[0]]; i0++)
    for (int i1 = 0; i1 < cnt[order[1]]; i1++)
      for (int i2 = 0; i2 < cnt[order[2]]; i2++) {
        int bb[3];
        bb[order[0]] = i0;
        bb[order[1]] = i1;
        bb[order[2]] = i2;
        const int idx = (bb[2] * 8 + bb[1]) * 8 + bb[0];
        for (int r = 0; r < 3; r++) P0[r] = m->offset[r] + (float)pos[r][bb[r]] * m->scale;
        for (int a = 0; a < 3; a++) {
          if (!edgeSet[3 * idx + a]) continue;
          const int step = a == 0 ? 1 : (a == 1 ? 8 : 64);
          float P1[3] = {P0[0], P0[1], P0[2]};
          int q2 = pos[a][bb[a]] + (role[a] ? stretch : sizeMin);
          P1[a] = m->offset[a] + (float)q2 * m->scale;
          float v[3];
          uint16_t col[3];
          vinterp(P0, P1, s[idx].d, s[idx + step].d, v);
          cinterp(s[idx].c, s[idx + step].c, s[idx].d, s[idx + step].d, col);
          vidx[3 * idx + a] = (uint32_t)b->nv;
          push_vertex(b, v, col);
        }
      }
  (void)base;
  /* faces, cube by cube in the same z, y, x nesting as the vertex loop */
  for (int i0 = 0; i0 < (order[0] < 3 ? ncube[order[0]] : 1); i0++)
    for (int i1 = 0; i1 < ncube[order[1]]; i1++)
      for (int i2 = 0; i2 < ncube[order[2]]; i2++) {
        int bb[3];
        bb[order[0]] = i0;
        bb[order[1]] = i1;
        bb[order[2]] = i2;
        const int idx = (bb[2] * 8 + bb[1]) * 8 + bb[0];
        const int ci = caseOf[idx];
        const int nt = ffp_mc_ntri(ci);
        for (int tt = 0; tt < nt; tt++) {
          uint32_t f3[3];
          for (int k = 0; k < 3; k++) {
            const int *es = EDGE_SLOT[ffp_mc_edge(ci, 3 * tt + k)];
            f3[k] = vidx[3 * (idx + es[0] + 8 * es[1] + 64 * es[2]) + es[3]];
          }
          push_face(b, f3[0], f3[1], f3[2]);
        }
      }
}

void ffp_mesh_cells(const ffp_mesh_src *m, const ffp_cell *cells, int64_t ncell, ffp_mesh_result *res) {
  mesh_buf b = {NULL, NULL, NULL, 0, 0, 0, 0};
  res->cell_v = (int64_t *)malloc(sizeof(int64_t) * 4 * (ncell ? ncell : 1));
  for (int64_t i = 0; i < ncell; i++) {
    int64_t v0 = b.nv, f0 = b.nf;
    if (cells[i].type == 7)
      mesh_corner(m, &cells[i], &b);
    else
      mesh_lattice(m, &cells[i], &b);
    res->cell_v[4 * i + 0] = v0;
    res->cell_v[4 * i + 1] = b.nv - v0;
    res->cell_v[4 * i + 2] = f0;
    res->cell_v[4 * i + 3] = b.nf - f0;
  }
  res->xyz = b.xyz;
  res->rgb = b.rgb;
  res->faces = b.faces;
  res->nv = b.nv;
  res->nf = b.nf;
}
