// Incremental marching cubes on the GPU.
//
// Cells.  The reference meshes "mesh cells" that it maintains incrementally
// per octree slot (MeshCell, treeandbrick_incremental.hpp:71-93;
// meshcelltraversalSplitReferenced.hpp).  They are the dual cells of the
// octree of branch slots: one interior cell per unsubdivided slot, one wall
// per pair of face-adjacent unsubdivided slots, one edge cell per four slots
// around an edge, one corner cell per eight slots around a vertex, each the
// size of the smallest slot it touches; each side refers to the finest leaf
// at or above its slot.  Here they are generated from the octree by a
// level-synchronous cell/face/edge/vertex traversal (one kernel per octree
// level, work queues in HBM) -- the reference's cell set, cell for cell --
// then sorted by (type, size, origin, leaves) so that the output order is
// deterministic.
//
// Meshing.  A warp per interior/wall/edge cell gathers the cell's lattice of
// samples (falling back along the parent-leaf chain where the weight is zero),
// classifies the cubes, flags the lattice edges that carry a vertex, then
// emits vertices and faces with warp prefix sums in the reference's per-type
// loop orders (mesh_interleaved_meshcell.cpp:9-2478); a thread per corner
// cell runs the reference's non-indexed single-cube path (:2480-2687).  A
// count pass, an exclusive scan over cells and an emit pass write the
// interleaved mesh without atomics, so it is identical run to run.
// Incremental: a cell whose leaves (and their parent chains) were not updated
// since the previous mesh, and whose leaves did not change, copies its old
// vertices and faces instead of being re-meshed.
#include <algorithm>
#include <cstddef>
#include <mutex>
#include <string>
#include <vector>

#include "ff_mesh.h"
#include "ff_sort.h"

namespace ffb {

// ---------------------------------------------------------------------------
// Marching-cubes triangle table of the published method (Lorensen & Cline;
// the public-domain table of P. Bourke / C. Bloyd, as used by the reference):
// per cube case, the triangle count in bits 60-63 and up to 15 cube-edge
// numbers, 4 bits each from bit 0.  Edges: 0:(0,1) 1:(1,2) 2:(2,3) 3:(3,0)
// 4:(4,5) 5:(5,6) 6:(6,7) 7:(7,4) 8:(0,4) 9:(1,5) 10:(2,6) 11:(3,7) over the
// corners (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1).
// ---------------------------------------------------------------------------
__constant__ unsigned long long c_mc_tri[256] = {
#include "ff_mc_table.inc"
};

// edge -> lattice edge it lies on: corner offset (dx,dy,dz) and axis
__constant__ uint8_t c_edge_slot[12][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {0, 1, 0, 0}, {0, 0, 0, 1},
                                           {0, 0, 1, 0}, {1, 0, 1, 1}, {0, 1, 1, 0}, {0, 0, 1, 1},
                                           {0, 0, 0, 2}, {1, 0, 0, 2}, {1, 1, 0, 2}, {0, 1, 0, 2}};
__constant__ uint8_t c_edge_a[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
__constant__ uint8_t c_edge_b[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};

// The tables as the meshing kernels read them: from shared memory, since
// the lanes of a warp index them by different cube cases.
struct McTab {
  unsigned long long tri[256];
  uint32_t slot[12];  // c_edge_slot packed: dx | dy << 8 | dz << 16 | axis << 24
};

// Copy the tables into the block's shared memory (all threads of the block).
__device__ __forceinline__ void load_mc(McTab &T) {
  for (int i = threadIdx.x; i < 256; i += blockDim.x) T.tri[i] = c_mc_tri[i];
  for (int i = threadIdx.x; i < 12; i += blockDim.x)
    T.slot[i] = (uint32_t)c_edge_slot[i][0] | ((uint32_t)c_edge_slot[i][1] << 8) |
                ((uint32_t)c_edge_slot[i][2] << 16) | ((uint32_t)c_edge_slot[i][3] << 24);
  __syncthreads();
}
__device__ __forceinline__ int mc_ntri(const McTab &T, int c) { return (int)(T.tri[c] >> 60); }
__device__ __forceinline__ int mc_edge(const McTab &T, int c, int k) { return (int)((T.tri[c] >> (4 * k)) & 15ull); }
// flat lattice-edge slot (3 * voxel index + axis) of a cube edge, relative to the cube's voxel index
__device__ __forceinline__ int mc_slot(const McTab &T, int e) {
  const uint32_t v = T.slot[e];
  return 3 * ((int)(v & 255u) + 8 * (int)((v >> 8) & 255u) + 64 * (int)((v >> 16) & 255u)) + (int)(v >> 24);
}

// ---------------------------------------------------------------------------
// Cell generation
// ---------------------------------------------------------------------------

struct __align__(16) Slot {
  uint32_t S;   // tree entry of the slot's leaf; child branch at S + 8
  uint32_t la;  // finest leaf at or above the slot (BRANCHINIT if none)
  uint16_t o[3];
  uint16_t size;
};

struct Cell {
  uint8_t type, quirk;
  uint16_t size;
  uint16_t o[3];
  uint16_t pad;
  uint32_t L[8];
};
static_assert(sizeof(Cell) == 44, "mesh cell layout");
static_assert(sizeof(Slot) == 16, "traversal slot layout");

// Work items of the traversal.  Faces and edges are queued per axis (the
// queue gives the axis), so the lanes of a warp expand items of one kind and
// axis: the item functions are specialised by axis, and a warp whose lanes
// held several kinds would run them one after the other.
struct FaceItem {
  Slot a, b;
};
struct EdgeItem {
  Slot s[4];
};
struct VertItem {
  Slot s[8];
};

// the queues of a level: cells, faces of axis 0-2, edges of axis 0-2, vertices
constexpr int QK = 8;
constexpr int QK_CELL = 0, QK_FACE = 1, QK_EDGE = 4, QK_VERT = 7;

struct GenQueues {
  Slot *cellq[2];
  FaceItem *faceq[2];  // three regions of cap_face items, one per axis
  EdgeItem *edgeq[2];  // three regions of cap_edge items, one per axis
  VertItem *vertq[2];
  uint32_t *lvl;  // [level][QK]: item count of each queue of each level
  uint32_t cap_cell, cap_face, cap_edge, cap_vert;
  Cell *cells;
  uint32_t *n_cells;
  uint32_t cap_cells;
  uint32_t *error;
  uint32_t *n_corners;
};

// counter words of the generation (see MeshImpl::d_count)
constexpr int LEVEL_COUNTS = 32;
constexpr int MAX_GEN_LEVELS = 48;
constexpr int COUNT_WORDS = LEVEL_COUNTS + QK * (MAX_GEN_LEVELS + 1) + 30;
// host mirror only: 3 uint64 + 2 uint32 read back per update, then the emit
// pass's sample count (uint64)
constexpr int HOST_TOTALS = COUNT_WORDS - 10;
static_assert(HOST_TOTALS % 2 == 0, "the host totals are read as uint64");

struct GenCtx {
  const uint32_t *tree;
  uint32_t leaves_max;
  // Incremental generation (incr != 0): only items with a slot that changed
  // since the previous update are expanded or emit cells; the cells of the
  // other items are kept from the previous list.  A slot changed if it lies
  // in a branch allocated since (entry index >= prev_branches), if its
  // finest leaf at or above is new (index >= prev_leaves), if it was
  // subdivided since (child branch index >= prev_branches), or if a branch
  // or leaf was created in its subtree since (branch stamp > since).
  const uint32_t *bstamp;
  uint32_t since, prev_leaves, prev_branches;
  int incr;
  // incremental, while the top levels are traversed again to refill their
  // cache: every item is expanded, but only changed items emit cells
  int expand_all;
};

// Queue reads bypass L1: in the one-launch traversal a block reads the items
// that other blocks wrote during the previous level, into a buffer whose
// lines its SM may still hold from two levels before.
__device__ __forceinline__ Slot ld_slot(const Slot *p) {
  const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(p));
  Slot s;
  s.S = v.x;
  s.la = v.y;
  s.o[0] = (uint16_t)(v.z & 0xffffu);
  s.o[1] = (uint16_t)(v.z >> 16);
  s.o[2] = (uint16_t)(v.w & 0xffffu);
  s.size = (uint16_t)(v.w >> 16);
  return s;
}

// the octree is read-only while the mesh is built: reads go through the
// read-only data cache
__device__ __forceinline__ uint32_t tree_at(const GenCtx &g, uint32_t i) { return __ldg(g.tree + i); }

__device__ __forceinline__ bool is_sub(const GenCtx &g, const Slot &s) { return tree_at(g, s.S + 8) < PENDING; }

__device__ __forceinline__ Slot child_of(const GenCtx &g, const Slot &s, int co) {
  Slot r;
  const uint32_t sub = tree_at(g, s.S + 8);
  const uint16_t h = s.size >> 1;
  r.S = sub + (uint32_t)co;
  r.o[0] = (uint16_t)(s.o[0] + h * (co & 1));
  r.o[1] = (uint16_t)(s.o[1] + h * ((co >> 1) & 1));
  r.o[2] = (uint16_t)(s.o[2] + h * ((co >> 2) & 1));
  r.size = h;
  const uint32_t lf = tree_at(g, r.S);
  r.la = lf < g.leaves_max ? lf : s.la;
  return r;
}

__device__ __forceinline__ Slot ch(const GenCtx &g, const Slot &s, int co) { return is_sub(g, s) ? child_of(g, s, co) : s; }

__device__ __forceinline__ bool slot_changed(const GenCtx &g, const Slot &s) {
  if (!g.incr) return true;
  // a slot of a branch allocated since: it did not exist (its cells are new
  // even where it inherits an old leaf)
  if (s.S >= g.prev_branches) return true;
  if (s.la < g.leaves_max && s.la >= g.prev_leaves) return true;
  const uint32_t c = tree_at(g, s.S + 8);
  if (c >= PENDING) return false;
  if (c >= g.prev_branches) return true;
  return __ldg(g.bstamp + (c >> 4)) > g.since;
}

__device__ __forceinline__ void others(int e, int &p, int &q) {
  p = e == 0 ? 1 : 0;
  q = e == 2 ? 1 : 2;
}

// Slots for every active lane of a warp: n[k] entries of counter ctr[k]
// (0 <= n[k] < 16, per lane).  All lanes of a launch push into the same
// counters (the next level's queues and the cell list), so each counter takes
// one atomic per warp, and the K atomics are independent: their latencies
// overlap instead of adding up.
template <int K>
__device__ __forceinline__ void claim_multi(uint32_t *const (&ctr)[K], const uint32_t (&n)[K], uint32_t (&base)[K]) {
  const unsigned mask = __activemask();
  const unsigned lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int leader = __ffs(mask) - 1;
  uint32_t tot[K], got[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    uint32_t pre = 0, t = 0;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const unsigned bal = __ballot_sync(mask, (n[k] >> b) & 1u);
      pre += (uint32_t)__popc(bal & below) << b;
      t += (uint32_t)__popc(bal) << b;
    }
    base[k] = pre;
    tot[k] = t;
    got[k] = 0;
  }
  if ((int)lane == leader) {
#pragma unroll
    for (int k = 0; k < K; k++)
      if (tot[k]) got[k] = atomicAdd(ctr[k], tot[k]);
  }
#pragma unroll
  for (int k = 0; k < K; k++) base[k] += __shfl_sync(mask, got[k], leader);
}

// One slot of *ctr for the calling lane: one atomic per group of active lanes
// that push to the same counter.
__device__ __forceinline__ uint32_t claim(uint32_t *ctr) {
  const unsigned mask = __activemask();
  const unsigned peers = __match_any_sync(mask, (unsigned long long)(uintptr_t)ctr);
  const int leader = __ffs(peers) - 1;
  const unsigned lane = threadIdx.x & 31;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

// a cell with a side without a leaf is never meshed
template <int N>
__device__ __forceinline__ bool all_leaves(const uint32_t (&L)[N]) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < N; k++) ok &= L[k] < BRANCHINIT;
  return ok;
}

// Store a cell at a claimed position of the list.
template <int N>
__device__ __forceinline__ void store_cell(const GenQueues &Q, uint32_t i, int type, const int *o, int size,
                                           const uint32_t (&L)[N]) {
  if (i >= Q.cap_cells) {
    atomicOr(Q.error, ERR_CELL_OVERFLOW);
    return;
  }
  Cell c;
  c.type = (uint8_t)type;
  c.quirk = 0;
  c.size = (uint16_t)size;
  for (int r = 0; r < 3; r++) c.o[r] = (uint16_t)o[r];
  c.pad = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) c.L[k] = k < N ? L[k] : BRANCHINIT;
  Q.cells[i] = c;
}

// Store an item at a claimed position of a queue, unless past its end.
template <typename T>
__device__ __forceinline__ void put(T *q, uint32_t i, uint32_t cap, const T &v, uint32_t *error) {
  if (i >= cap) {
    atomicOr(error, ERR_CELL_OVERFLOW);
    return;
  }
  q[i] = v;
}

// Every item is a pure function of its slots, so an item found while
// expanding another is queued for the next launch rather than expanded by the
// same thread: each thread does a bounded amount of work (a few independent
// tree reads, one set of queue claims) and the levels run wide.
struct Out {
  Slot *cellq;
  FaceItem *faceq;  // axis regions of Q.cap_face items
  EdgeItem *edgeq;  // axis regions of Q.cap_edge items
  VertItem *vertq;
  uint32_t *count;  // the next level's QK counters
};

__device__ __forceinline__ void put_face(const GenQueues &Q, const Out &O, int ax, uint32_t i, const Slot &a,
                                         const Slot &b) {
  FaceItem f;
  f.a = a;
  f.b = b;
  if (i >= Q.cap_face) {
    atomicOr(Q.error, ERR_CELL_OVERFLOW);
    return;
  }
  O.faceq[(size_t)ax * Q.cap_face + i] = f;
}
__device__ __forceinline__ void put_edge(const GenQueues &Q, const Out &O, int ax, uint32_t i, const Slot *S4) {
  EdgeItem it;
  for (int j = 0; j < 4; j++) it.s[j] = S4[j];
  if (i >= Q.cap_edge) {
    atomicOr(Q.error, ERR_CELL_OVERFLOW);
    return;
  }
  O.edgeq[(size_t)ax * Q.cap_edge + i] = it;
}
__device__ __forceinline__ void put_vert(const GenQueues &Q, const Out &O, uint32_t i, const Slot *S8) {
  VertItem v;
  for (int j = 0; j < 8; j++) v.s[j] = S8[j];
  put(O.vertq, i, Q.cap_vert, v, Q.error);
}

// The item functions are templated on their axis and fully unrolled, so every
// slot array index is a compile-time constant and the slots stay in registers.
//
// A slot that is not subdivided and has no leaf at or above it is empty
// space: it stays itself in every descendant of an item that holds it, and a
// cell with a side without a leaf is never meshed, so such an item is
// dropped without expanding it (the meshed cells are the same).
__device__ __forceinline__ bool dead_slot(const Slot &s, bool sub) { return !sub && s.la >= BRANCHINIT; }

__device__ __forceinline__ void vert_item(const GenCtx &g, const GenQueues &Q, const Out &O, const Slot (&S8)[8],
                                          bool emit) {
  bool any = false, dead = false;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const bool sub = is_sub(g, S8[j]);
    any |= sub;
    dead |= dead_slot(S8[j], sub);
  }
  if (dead) return;
  uint32_t L[8];
#pragma unroll
  for (int j = 0; j < 8; j++) L[j] = S8[j].la;
  const bool em = !any && emit && all_leaves(L);
  Slot C[8];
  if (any) {
#pragma unroll
    for (int j = 0; j < 8; j++) C[j] = ch(g, S8[j], 7 - j);
  }
  uint32_t *const ctr[3] = {O.count + QK_VERT, Q.n_cells, Q.n_corners};
  const uint32_t n[3] = {any ? 1u : 0u, em ? 1u : 0u, em ? 1u : 0u};
  uint32_t at[3];
  claim_multi(ctr, n, at);
  if (any) {
    put_vert(Q, O, at[0], C);
    return;
  }
  if (!em) return;
  // the vertex is a corner of the smallest slot around it
  int size = S8[0].size, small = 0;
#pragma unroll
  for (int j = 1; j < 8; j++)
    if (S8[j].size < size) size = S8[j].size, small = j;
  int o[3] = {0, 0, 0};
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j == small) {
#pragma unroll
      for (int r = 0; r < 3; r++) o[r] = (int)S8[j].o[r] + (((j >> r) & 1) ? 0 : size) - size;
    }
  store_cell(Q, at[1], 7, o, size, L);
}

template <int E>
__device__ __forceinline__ void edge_item(const GenCtx &g, const GenQueues &Q, const Out &O, const Slot (&S4)[4],
                                          bool emit) {
  constexpr int P = E == 0 ? 1 : 0, Qx = E == 2 ? 1 : 2;  // the two axes across the edge line
  bool any = false, dead = false;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const bool sub = is_sub(g, S4[j]);
    any |= sub;
    dead |= dead_slot(S4[j], sub);
  }
  if (dead) return;
  const uint32_t L[4] = {S4[0].la, S4[1].la, S4[2].la, S4[3].la};
  const bool em = !any && emit && all_leaves(L);
  uint32_t *const ctr[3] = {O.count + QK_EDGE + E, O.count + QK_VERT, Q.n_cells};
  const uint32_t n[3] = {any ? 2u : 0u, any ? 1u : 0u, em ? 1u : 0u};
  uint32_t at[3];
  claim_multi(ctr, n, at);
  if (!any) {
    if (!em) return;
    // the edge line runs along a side of the smallest slot
    int size = S4[0].size, small = 0;
#pragma unroll
    for (int j = 1; j < 4; j++)
      if (S4[j].size < size) size = S4[j].size, small = j;
    int o[3] = {0, 0, 0};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (j == small) {
        o[E] = S4[j].o[E];
        o[P] = (int)S4[j].o[P] + ((j & 1) ? 0 : size) - size;
        o[Qx] = (int)S4[j].o[Qx] + ((j & 2) ? 0 : size) - size;
      }
    store_cell(Q, at[2], 4 + E, o, size, L);
    return;
  }
#pragma unroll
  for (int half = 0; half < 2; half++) {
    Slot H[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = ((j & 1) ? 0 : (1 << P)) | (((j >> 1) & 1) ? 0 : (1 << Qx)) | (half ? (1 << E) : 0);
      H[j] = ch(g, S4[j], k);
    }
    put_edge(Q, O, E, at[0] + half, H);
  }
  Slot S8[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    // across the edge line: the half of the slot next to the line; along the
    // edge: the half on the vertex's own side of the midpoint
    const int pj = (j >> P) & 1, qj = (j >> Qx) & 1, ej = (j >> E) & 1;
    const int k = (pj ? 0 : (1 << P)) | (qj ? 0 : (1 << Qx)) | (ej ? (1 << E) : 0);
    S8[j] = ch(g, S4[pj | (qj << 1)], k);
  }
  put_vert(Q, O, at[1], S8);
}

template <int AX>
__device__ __forceinline__ void face_item(const GenCtx &g, const GenQueues &Q, const Out &O, const Slot &A,
                                          const Slot &B, bool emit) {
  const bool sa = is_sub(g, A), sb = is_sub(g, B);
  if (dead_slot(A, sa) || dead_slot(B, sb)) return;
  constexpr int U = AX == 0 ? 1 : 0, V = AX == 2 ? 1 : 2;
  const bool leafy = !sa && !sb;
  const uint32_t L[2] = {A.la, B.la};
  const bool em = leafy && emit && all_leaves(L);
  uint32_t *const ctr[5] = {O.count + QK_FACE + AX, O.count + QK_EDGE + U, O.count + QK_EDGE + V, O.count + QK_VERT,
                            Q.n_cells};
  const uint32_t n[5] = {leafy ? 0u : 4u, leafy ? 0u : 2u, leafy ? 0u : 2u, leafy ? 0u : 1u, em ? 1u : 0u};
  uint32_t at[5];
  claim_multi(ctr, n, at);
  if (leafy) {
    if (!em) return;
    const int size = min((int)A.size, (int)B.size);
    const bool a_small = A.size <= B.size;
    int o[3] = {a_small ? A.o[0] : B.o[0], a_small ? A.o[1] : B.o[1], a_small ? A.o[2] : B.o[2]};
    o[AX] = (int)B.o[AX] - size;
    store_cell(Q, at[4], 1 + AX, o, size, L);
    return;
  }
  constexpr int bit = 1 << AX;
  // the two sides' halves next to the face: A's children on its +ax side, B's
  // on its -ax side (a slot that is not subdivided stands for all of them)
  Slot a[8], b[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    if (k & bit) continue;
    a[k] = ch(g, A, k | bit);
    b[k] = ch(g, B, k);
  }
#pragma unroll
  for (int qd = 0; qd < 4; qd++) {
    const int k = ((qd & 1) ? (1 << U) : 0) | ((qd & 2) ? (1 << V) : 0);
    put_face(Q, O, AX, at[0] + qd, a[k], b[k]);
  }
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int e = t == 0 ? U : V;
    const int other = t == 0 ? V : U;
    const int p = e == 0 ? 1 : 0, q = e == 2 ? 1 : 2;
#pragma unroll
    for (int half = 0; half < 2; half++) {
      Slot S4[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        int side[3] = {0, 0, 0};
        side[p] = j & 1;
        side[q] = (j >> 1) & 1;
        const int k = (half ? (1 << e) : 0) | (side[other] ? (1 << other) : 0);
        S4[j] = side[AX] ? b[k] : a[k];
      }
      put_edge(Q, O, e, at[1 + t] + half, S4);
    }
  }
  Slot S8[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int k = j & ~bit;
    S8[j] = ((j >> AX) & 1) ? b[k] : a[k];
  }
  put_vert(Q, O, at[3], S8);
}

// one subdivided slot: its children, their 12 faces, 6 edges and centre
__device__ __forceinline__ void cell_item(const GenCtx &g, const GenQueues &Q, const Out &O, const Slot (&C)[8]) {
  uint32_t sub = 0, em = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    if (is_sub(g, C[j])) sub |= 1u << j;
    else if (C[j].la < BRANCHINIT && slot_changed(g, C[j])) em |= 1u << j;
  }
  uint32_t *const ctr[9] = {O.count + QK_CELL,     Q.n_cells,             O.count + QK_FACE, O.count + QK_FACE + 1,
                            O.count + QK_FACE + 2, O.count + QK_EDGE,     O.count + QK_EDGE + 1,
                            O.count + QK_EDGE + 2, O.count + QK_VERT};
  const uint32_t n[9] = {(uint32_t)__popc(sub), (uint32_t)__popc(em), 4, 4, 4, 2, 2, 2, 1};
  uint32_t at[9];
  claim_multi(ctr, n, at);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const uint32_t below = (1u << j) - 1u;
    if (sub >> j & 1u) {
      put(O.cellq, at[0] + (uint32_t)__popc(sub & below), Q.cap_cell, C[j], Q.error);
    } else if (em >> j & 1u) {
      const int o[3] = {C[j].o[0], C[j].o[1], C[j].o[2]};
      const uint32_t L[1] = {C[j].la};
      store_cell(Q, at[1] + (uint32_t)__popc(em & below), 0, o, C[j].size, L);
    }
  }
  constexpr int F[3][4][2] = {{{0, 1}, {2, 3}, {4, 5}, {6, 7}}, {{0, 2}, {1, 3}, {4, 6}, {5, 7}},
                              {{0, 4}, {1, 5}, {2, 6}, {3, 7}}};
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int i = 0; i < 4; i++) put_face(Q, O, ax, at[2 + ax] + i, C[F[ax][i][0]], C[F[ax][i][1]]);
#pragma unroll
  for (int x = 0; x < 2; x++) {
    Slot S4[4] = {C[x], C[x | 2], C[x | 4], C[x | 6]};
    put_edge(Q, O, 0, at[5] + x, S4);
  }
#pragma unroll
  for (int y = 0; y < 4; y += 2) {
    Slot S4[4] = {C[y], C[y | 1], C[y | 4], C[y | 5]};
    put_edge(Q, O, 1, at[6] + y / 2, S4);
  }
#pragma unroll
  for (int z = 0; z < 8; z += 4) {
    Slot S4[4] = {C[z], C[z | 1], C[z | 2], C[z | 3]};
    put_edge(Q, O, 2, at[7] + z / 4, S4);
  }
  put_vert(Q, O, at[8], C);
}

template <int AX>
__device__ __forceinline__ void face_at(const GenCtx &g, const GenQueues &Q, const Out &O, int cur, uint32_t j) {
  const FaceItem *f = Q.faceq[cur] + (size_t)AX * Q.cap_face + j;
  const Slot a = ld_slot(&f->a), b = ld_slot(&f->b);
  const bool changed = slot_changed(g, a) || slot_changed(g, b);
  if (!changed && !g.expand_all) return;
  face_item<AX>(g, Q, O, a, b, changed);
}

template <int E>
__device__ __forceinline__ void edge_at(const GenCtx &g, const GenQueues &Q, const Out &O, int cur, uint32_t j) {
  const EdgeItem *e = Q.edgeq[cur] + (size_t)E * Q.cap_edge + j;
  Slot S4[4];
  bool changed = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    S4[k] = ld_slot(&e->s[k]);
    changed |= slot_changed(g, S4[k]);
  }
  if (!changed && !g.expand_all) return;
  edge_item<E>(g, Q, O, S4, changed);
}

// Items of level `lv` (queue buffer lv & 1, counters lvl + QK lv) expand into
// level lv + 1 or emit cells.  Level 0 is the root: the volume's 8 octants.
// The queues' threads are laid out one after the other, each queue's padded
// to whole warps, so that the lanes of a warp run the same item function.
__device__ __forceinline__ void gen_level(const GenCtx &g, const GenQueues &Q, int lv, uint32_t n) {
  const int cur = lv & 1, nb = cur ^ 1;
  const bool root = lv == 0;
  const uint32_t *cnt = Q.lvl + QK * lv;
  Out O{Q.cellq[nb], Q.faceq[nb], Q.edgeq[nb], Q.vertq[nb], Q.lvl + QK * (lv + 1)};
  uint32_t c[QK], e[QK];
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < QK; k++) {
    const uint32_t cap = k == QK_CELL ? Q.cap_cell : (k < QK_EDGE ? Q.cap_face : (k < QK_VERT ? Q.cap_edge : Q.cap_vert));
    c[k] = root ? (k == QK_CELL ? 1u : 0u) : min(__ldcg(cnt + k), cap);
    acc += (c[k] + 31u) & ~31u;
    e[k] = acc;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < e[QK - 1]; i += gridDim.x * blockDim.x) {
    if (i < e[0]) {
      if (i >= c[0]) continue;
      Slot C[8];
      if (root) {
        const uint16_t h = (uint16_t)(n >> 1);
        for (int co = 0; co < 8; co++) {
          C[co].S = (uint32_t)co;
          C[co].o[0] = (uint16_t)(h * (co & 1));
          C[co].o[1] = (uint16_t)(h * ((co >> 1) & 1));
          C[co].o[2] = (uint16_t)(h * ((co >> 2) & 1));
          C[co].size = h;
          const uint32_t lf = tree_at(g, co);
          C[co].la = lf < g.leaves_max ? lf : BRANCHINIT;
        }
      } else {
        const Slot s = ld_slot(Q.cellq[cur] + i);
        if (!g.expand_all && !slot_changed(g, s)) continue;
        for (int co = 0; co < 8; co++) C[co] = child_of(g, s, co);
      }
      cell_item(g, Q, O, C);
    } else if (i < e[1]) {
      if (i - e[0] < c[1]) face_at<0>(g, Q, O, cur, i - e[0]);
    } else if (i < e[2]) {
      if (i - e[1] < c[2]) face_at<1>(g, Q, O, cur, i - e[1]);
    } else if (i < e[3]) {
      if (i - e[2] < c[3]) face_at<2>(g, Q, O, cur, i - e[2]);
    } else if (i < e[4]) {
      if (i - e[3] < c[4]) edge_at<0>(g, Q, O, cur, i - e[3]);
    } else if (i < e[5]) {
      if (i - e[4] < c[5]) edge_at<1>(g, Q, O, cur, i - e[4]);
    } else if (i < e[6]) {
      if (i - e[5] < c[6]) edge_at<2>(g, Q, O, cur, i - e[5]);
    } else if (i - e[6] < c[7]) {
      const VertItem *v = Q.vertq[cur] + (i - e[6]);
      Slot S8[8];
      bool changed = false;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        S8[j] = ld_slot(&v->s[j]);
        changed |= slot_changed(g, S8[j]);
      }
      if (!changed && !g.expand_all) continue;
      vert_item(g, Q, O, S8, changed);
    }
  }
}

// The items of traversal level MESH_TOP_LEVELS, kept from one update to the
// next: the levels above it hold few items, each a long chain of dependent
// tree reads, and they produce the same items until a frame creates a branch
// or a leaf that close to the root.
struct TopCache {
  Slot *cellq;
  FaceItem *faceq;  // axis regions of cap[1] items
  EdgeItem *edgeq;  // axis regions of cap[2] items
  VertItem *vertq;
  uint32_t cap[4];  // cells, faces and edges per axis, vertices
  uint32_t *count;  // the QK queues' items; [QK]: 1 if they did not fit
};

// n items of `words` 16-byte words each, read past L1 (see ld_slot)
__device__ __forceinline__ void copy_items(void *dst, const void *src, uint32_t n, int words, uint32_t t0,
                                           uint32_t stride) {
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  const uint4 *q = reinterpret_cast<const uint4 *>(src);
  const size_t total = (size_t)n * (size_t)words;
  for (size_t i = t0; i < total; i += stride) d[i] = __ldcg(q + i);
}

// Keep level lv's items (complete once level lv - 1 has run), every thread of
// the grid taking part.
__device__ void save_top(const GenQueues &Q, int lv, const TopCache &T) {
  const uint32_t *cp = Q.lvl + QK * lv;
  uint32_t c[QK];
  for (int k = 0; k < QK; k++) c[k] = __ldcg(cp + k);
  const int b = lv & 1;
  bool fits = c[0] <= T.cap[0] && c[0] <= Q.cap_cell && c[7] <= T.cap[3] && c[7] <= Q.cap_vert;
  for (int k = 0; k < 3; k++) {
    fits &= c[QK_FACE + k] <= T.cap[1] && c[QK_FACE + k] <= Q.cap_face;
    fits &= c[QK_EDGE + k] <= T.cap[2] && c[QK_EDGE + k] <= Q.cap_edge;
  }
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (t0 == 0) {
    for (int k = 0; k < QK; k++) T.count[k] = c[k];
    T.count[QK] = fits ? 0u : 1u;
  }
  if (!fits) return;
  copy_items(T.cellq, Q.cellq[b], c[0], 1, t0, stride);
  for (int k = 0; k < 3; k++) {
    copy_items(T.faceq + (size_t)k * T.cap[1], Q.faceq[b] + (size_t)k * Q.cap_face, c[QK_FACE + k], 2, t0, stride);
    copy_items(T.edgeq + (size_t)k * T.cap[2], Q.edgeq[b] + (size_t)k * Q.cap_edge, c[QK_EDGE + k], 4, t0, stride);
  }
  copy_items(T.vertq, Q.vertq[b], c[7], 8, t0, stride);
}

// (the cache's counts fit the queues: the queues only grow while it is valid)
__global__ void k_load_top(GenQueues Q, int lv, TopCache T) {
  pdl_enter();
  const int b = lv & 1;
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (t0 == 0) {
    uint32_t *c = Q.lvl + QK * lv;
    for (int k = 0; k < QK; k++) c[k] = T.count[k];
  }
  for (uint32_t i = t0; i < T.count[0]; i += stride) Q.cellq[b][i] = T.cellq[i];
  for (int k = 0; k < 3; k++) {
    for (uint32_t i = t0; i < T.count[QK_FACE + k]; i += stride)
      Q.faceq[b][(size_t)k * Q.cap_face + i] = T.faceq[(size_t)k * T.cap[1] + i];
    for (uint32_t i = t0; i < T.count[QK_EDGE + k]; i += stride)
      Q.edgeq[b][(size_t)k * Q.cap_edge + i] = T.edgeq[(size_t)k * T.cap[2] + i];
  }
  for (uint32_t i = t0; i < T.count[7]; i += stride) Q.vertq[b][i] = T.vertq[i];
}

// One launch runs the traversal levels [lv0, lv_end): a grid barrier between
// two levels (bounded: it gives up after spin_limit polls and sets
// ERR_CELL_TIMEOUT), the top levels' items kept when level save_level is
// complete, and an early end at the first level without items.  Each level
// is a handful of microseconds of dependent tree reads and queue claims, so
// one launch per level would cost as much again in launch gaps.
struct GenRun {
  int lv0, lv_end;
  int incr;
  int save_level;  // level whose items are kept (TopCache), -1: none
  uint32_t *bar;   // grid barrier: arrivals, generation (zero at the first launch)
  uint32_t spin_limit;
};

constexpr int GEN_THREADS = 128;

__global__ void __launch_bounds__(GEN_THREADS, 4) k_gen_levels(GenCtx g, GenQueues Q, GenRun R, uint32_t n,
                                                               TopCache T) {
  for (int lv = R.lv0; lv < R.lv_end; lv++) {
    g.expand_all = (R.incr && lv < MESH_TOP_LEVELS) ? 1 : 0;
    gen_level(g, Q, lv, n);
    grid_barrier_bounded(R.bar, gridDim.x, Q.error, ERR_CELL_TIMEOUT, R.spin_limit);
    if (__ldcg(Q.error) & ERR_CELL_TIMEOUT) return;
    if (lv + 1 == R.save_level) save_top(Q, lv + 1, T);
    // every block reads the same counts after the barrier
    const uint32_t *c = Q.lvl + QK * (lv + 1);
    uint32_t any = 0;
    for (int k = 0; k < QK; k++) any |= __ldcg(c + k);
    if (!any) {
      // the levels below are empty too: so is the one to keep
      if (R.save_level > lv + 1) save_top(Q, R.save_level, T);
      return;
    }
  }
}

// Blocks of the one-launch traversal for levels of about `items` items:
// one block per SM at least (the barrier's cost grows with the blocks), as
// many as are resident at once at most (the grid must be co-resident);
// 0 if the device cannot be queried.
static int gen_blocks(size_t items) {
  static int sms = 0, most = 0;
  if (!most) {
    int per_sm = 0, n = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gen_levels, GEN_THREADS, 0) != cudaSuccess ||
        per_sm < 1 || n < 1)
      return 0;
    sms = n;
    most = std::min(per_sm, 4) * n;
  }
  const size_t want = (items + GEN_THREADS - 1) / GEN_THREADS;
  return (int)std::max<size_t>(sms, std::min<size_t>(want, most));
}

// Sort key of a cell: (type, log2 size, origin x, y, z), the order of the
// mesh; B bits per origin coordinate (origins lie inside the volume, below
// 2^B), so the radix sort runs over 3B + 7 bits only.
__device__ __forceinline__ uint64_t cell_key(const Cell &c, int B) {
  int lsz = 0;
  while ((1 << lsz) < c.size) lsz++;
  return ((uint64_t)c.type << (3 * B + 4)) | ((uint64_t)lsz << (3 * B)) | ((uint64_t)c.o[0] << (2 * B)) |
         ((uint64_t)c.o[1] << B) | (uint64_t)c.o[2];
}

__global__ void k_cell_keys(const Cell *cells, uint32_t n, int B, uint64_t *keys, uint32_t *error) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Cell c = cells[i];
  const uint32_t lim = 1u << B;
  if (c.o[0] >= lim || c.o[1] >= lim || c.o[2] >= lim) atomicOr(error, ERR_CELL_KEY);
  keys[i] = cell_key(c, B);
}

__global__ void k_gather_cells(const Cell *in, const uint32_t *order, uint32_t n, Cell *out) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[order[i]];
}

// ---------------------------------------------------------------------------
// Incremental cell list: the previous update's cells whose item did not
// change are kept; the traversal (pruned to changed items) adds the rest.
// ---------------------------------------------------------------------------

// Did the slot that held point p in the previous update's octree change?  The
// previous octree is this one without the branches allocated since
// (index >= prev_branches; a child slot, once set, never changes), so the
// descent stops where the previous one stopped: at the slot that was not
// subdivided.  It changed if it is subdivided now or if its finest leaf at or
// above is new.  Most of the octree is unchanged: the descent ends early at
// a branch whose subtree gained nothing (its stamp) while the leaves on the
// path so far are old, since every leaf further down is old then too.
__device__ __forceinline__ bool side_changed(const GenCtx &g, uint32_t n, const int (&p)[3]) {
  uint32_t branch = 0, la = BRANCHINIT, half = n >> 1;
  uint32_t ox = 0, oy = 0, oz = 0;
  for (int lvl = 0; lvl < 32 && half; lvl++) {
    const uint32_t co = ((uint32_t)p[0] >= ox + half) * 1u + ((uint32_t)p[1] >= oy + half) * 2u +
                        ((uint32_t)p[2] >= oz + half) * 4u;
    const uint32_t S = branch + co;
    const uint32_t lf = tree_at(g, S);
    if (lf < g.leaves_max) la = lf;
    const uint32_t c = tree_at(g, S + 8);
    if (c >= PENDING) return la < g.leaves_max && la >= g.prev_leaves;
    if (c >= g.prev_branches) return true;
    // nothing created below since, and no new leaf on the path so far: the
    // slot and its finest leaf are as they were
    if (__ldg(g.bstamp + (c >> 4)) <= g.since && !(la < g.leaves_max && la >= g.prev_leaves)) return false;
    ox += half * ((co & 1) != 0);
    oy += half * ((co & 2) != 0);
    oz += half * ((co & 4) != 0);
    branch = c;
    half >>= 1;
  }
  return true;  // deeper than any octree: treat as changed
}

// A point inside side k of a cell (the sides in the order of Cell::L):
// interior cell: its slot; wall across axis a: the slot before and after the
// plane o[a] + size; edge along axis e: the four slots around the line
// (o[p] + size, o[q] + size), bit 0 of k the +p side, bit 1 the +q side;
// corner: the eight slots around the vertex o + size, bit r of k the +r side.
__device__ __forceinline__ void side_point(const Cell &c, int k, int (&p)[3]) {
  const int sz = c.size;
  for (int r = 0; r < 3; r++) p[r] = c.o[r];
  if (c.type == 0) return;
  if (c.type <= 3) {
    const int a = c.type - 1;
    p[a] = c.o[a] + sz - (k == 0 ? 1 : 0);
    return;
  }
  if (c.type <= 6) {
    const int e = c.type - 4;
    const int pa = e == 0 ? 1 : 0, qa = e == 2 ? 1 : 2;
    p[pa] = c.o[pa] + sz - ((k & 1) ? 0 : 1);
    p[qa] = c.o[qa] + sz - ((k & 2) ? 0 : 1);
    return;
  }
  for (int r = 0; r < 3; r++) p[r] = c.o[r] + sz - (((k >> r) & 1) ? 0 : 1);
}

constexpr int KEEP_THREADS = 256, KEEP_SCAN_THREADS = 1024;

// Block-wide exclusive prefix of one value per thread (KEEP_THREADS threads);
// the block's total in *total.
__device__ __forceinline__ uint32_t block_scan_keep(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sum[KEEP_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += u;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int j = 0; j < KEEP_THREADS / 32; j++) {
    const uint32_t t = warp_sum[j];
    if (j < w) before += t;
    all += t;
  }
  *total = all;
  return before + x - v;
}

// keep[i] = 1 if previous cell i is kept; per tile of KEEP_THREADS cells, the
// number kept (tile_sum).
__global__ void __launch_bounds__(KEEP_THREADS) k_keep_cells(GenCtx g, uint32_t n, const Cell *__restrict__ old_cells,
                                                            uint32_t n_old, uint32_t *keep, uint32_t *tile_sum) {
  pdl_enter();
  const uint32_t i = blockIdx.x * KEEP_THREADS + threadIdx.x;
  uint32_t k = 0;
  if (i < n_old) {
    const Cell c = old_cells[i];
    const int nl = c.type == 0 ? 1 : (c.type <= 3 ? 2 : (c.type <= 6 ? 4 : 8));
    bool changed = false;
    for (int s = 0; s < nl && !changed; s++) {
      int p[3];
      side_point(c, s, p);
      changed = side_changed(g, n, p);
    }
    k = changed ? 0u : 1u;
    keep[i] = k;
  }
  uint32_t total;
  (void)block_scan_keep(k, &total);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in one block (any number of tiles, in
// chunks of the block size).
__global__ void __launch_bounds__(KEEP_SCAN_THREADS) k_keep_tile_scan(uint32_t *tile_sum, uint32_t ntiles) {
  pdl_enter();
  __shared__ uint32_t warp_sum[KEEP_SCAN_THREADS / 32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t base = 0; base < ntiles; base += KEEP_SCAN_THREADS) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < ntiles ? tile_sum[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (int j = 0; j < KEEP_SCAN_THREADS / 32; j++) {
      const uint32_t t = warp_sum[j];
      if (j < w) before += t;
      all += t;
    }
    const uint32_t c0 = carry;
    if (i < ntiles) tile_sum[i] = c0 + before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) carry = c0 + all;
    __syncthreads();
  }
}

// keep[] becomes the exclusive prefix of the kept flags, with the total at
// keep[n_old]; counts[0] = cells kept, counts[1] = cells kept before the
// previous list's first corner cell.
__global__ void __launch_bounds__(KEEP_THREADS) k_keep_apply(uint32_t *keep, uint32_t n_old, const uint32_t *tile_sum,
                                                            uint32_t ntiles, uint32_t first_corner_old,
                                                            uint32_t *counts) {
  pdl_enter();
  const uint32_t i = blockIdx.x * KEEP_THREADS + threadIdx.x;
  const uint32_t k = i < n_old ? keep[i] : 0u;
  uint32_t total;
  const uint32_t ex = block_scan_keep(k, &total) + tile_sum[blockIdx.x];
  if (i < n_old) keep[i] = ex;
  if (i == first_corner_old) counts[1] = ex;
  if (blockIdx.x == ntiles - 1 && threadIdx.x == 0) {
    keep[n_old] = tile_sum[blockIdx.x] + total;
    counts[0] = tile_sum[blockIdx.x] + total;
    if (first_corner_old >= n_old) counts[1] = tile_sum[blockIdx.x] + total;
  }
}

// first index in keys[0, n) whose key is >= key (strict: > key)
__device__ __forceinline__ uint32_t key_bound(const uint64_t *keys, uint32_t n, uint64_t key, bool strict) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint64_t k = keys[mid];
    if (k < key || (strict && k == key)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Merge the kept previous cells (sorted, keep_scan their exclusive prefix)
// with the new cells (sorted keys, order into raw): a stable merge with the
// kept cells first among equal keys, so every position of the output is
// written exactly once.  Equal keys (which the cell geometry rules out) are
// reported with ERR_CELL_MERGE.
__global__ void k_merge_cells(const Cell *__restrict__ old_cells, const uint64_t *__restrict__ old_keys,
                              const uint32_t *__restrict__ keep_scan, uint32_t n_old, const Cell *__restrict__ raw,
                              const uint64_t *__restrict__ new_keys, const uint32_t *__restrict__ new_order,
                              uint32_t n_new, Cell *out, uint64_t *out_keys, uint32_t *error) {
  pdl_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_old) {
    const uint32_t ks = keep_scan[i];
    if (keep_scan[i + 1] == ks) return;  // not kept
    const uint64_t key = old_keys[i];
    const uint32_t lb = key_bound(new_keys, n_new, key, false);
    if (lb < n_new && new_keys[lb] == key) atomicOr(error, ERR_CELL_MERGE);
    out[ks + lb] = old_cells[i];
    out_keys[ks + lb] = key;
  } else if (i < n_old + n_new) {
    const uint32_t j = i - n_old;
    const uint64_t key = new_keys[j];
    if (j > 0 && new_keys[j - 1] == key) atomicOr(error, ERR_CELL_MERGE);
    const uint32_t ub = key_bound(old_keys, n_old, key, true);
    const uint32_t pos = j + keep_scan[ub];
    out[pos] = raw[new_order[j]];
    out_keys[pos] = key;
  }
}

// ---------------------------------------------------------------------------
// Per-cell marching cubes
// ---------------------------------------------------------------------------

struct VoxSrc {
  const ushort4 *leaf;
  const uint32_t *parent;
  const float *sdf, *wgt;
  const __half *sdf16, *wgt16;
  const uint16_t *col;  // [leaf][3][512]
  int fp16;
  uint32_t leaves_used;
  float offset[3];
  float scale;
  unsigned long long *samples;  // count pass: voxel samples read (profiling)
  // a part of a sharded map meshes the cells it owns (ff_set_shard)
  uint32_t shard, shards;
  int32_t shift[3];
};

// Whether this part meshes cell c: a hash of its origin, size and type in
// coordinates that grow() does not move (every part has every cell; each
// cell is meshed by exactly one part).
__device__ __forceinline__ bool owns_cell(const VoxSrc &m, const Cell &c) {
  if (m.shards <= 1) return true;
  return shard_hash(c.o[0], c.o[1], c.o[2], c.size, 1u + c.type, m.shift) % m.shards == m.shard;
}

__device__ __forceinline__ size_t vox_index(const VoxSrc &m, uint32_t leaf, uint16_t lx, uint16_t ly, uint16_t lz) {
  // the reference computes the index in uint16 voxel coordinates and may
  // step outside the brick (never outside the pool here)
  size_t i = (size_t)leaf * 512 + ((size_t)lz * 8 + ly) * 8 + lx;
  size_t lim = (size_t)m.leaves_used * 512;
  return i < lim ? i : lim - 1;
}
__device__ __forceinline__ float vd(const VoxSrc &m, size_t i) { return m.fp16 ? __half2float(m.sdf16[i]) : m.sdf[i]; }
__device__ __forceinline__ float vw(const VoxSrc &m, size_t i) { return m.fp16 ? __half2float(m.wgt16[i]) : m.wgt[i]; }
__device__ __forceinline__ uint16_t vc(const VoxSrc &m, size_t i, int c) {
  return m.col[(i >> 9) * 1536 + c * 512 + (i & 511)];
}

// A sample's colour channel, or 0 without a read when the pass needs no
// colour (the count pass: only SDF and weight decide the cube cases).
template <bool COLOR>
__device__ __forceinline__ uint16_t vcs(const VoxSrc &m, size_t i, int c) {
  return COLOR ? vc(m, i, c) : (uint16_t)0;
}

// MarchingCubes::VertexInterp(Vertex3f, Vertex3f, double, double), mesh.cpp:1266-1315
__device__ void vinterp(const float *p1, const float *p2, double v1, double v2, float *out) {
  if (fabs(__dsub_rn(0.0, v1)) < 1e-40) {
    out[0] = p1[0], out[1] = p1[1], out[2] = p1[2];
    return;
  }
  if (fabs(__dsub_rn(0.0, v2)) < 1e-40) {
    out[0] = p2[0], out[1] = p2[1], out[2] = p2[2];
    return;
  }
  if (fabs(__dsub_rn(v1, v2)) < 1e-40) {
    out[0] = p1[0], out[1] = p1[1], out[2] = p1[2];
    return;
  }
  const double mu = __ddiv_rn(__dsub_rn(0.0, v1), __dsub_rn(v2, v1));
#pragma unroll
  for (int r = 0; r < 3; r++)
    out[r] = __double2float_rn(__dadd_rn((double)p1[r], __dmul_rn(mu, __dsub_rn((double)p2[r], (double)p1[r]))));
}

// MarchingCubes::VertexInterp(VertexColor, ...), mesh.cpp:1317-1340
__device__ void cinterp(const uint16_t *c1, const uint16_t *c2, float v1, float v2, uint16_t *out) {
  if ((double)fabsf(__fsub_rn(0.0f, v1)) < 1e-40) {
    out[0] = c1[0], out[1] = c1[1], out[2] = c1[2];
    return;
  }
  if ((double)fabsf(__fsub_rn(0.0f, v2)) < 1e-40) {
    out[0] = c2[0], out[1] = c2[1], out[2] = c2[2];
    return;
  }
  if ((double)fabsf(__fsub_rn(v1, v2)) < 1e-40) {
    out[0] = c1[0], out[1] = c1[1], out[2] = c1[2];
    return;
  }
  const float mu = __fdiv_rn(__fsub_rn(0.0f, v1), __fsub_rn(v2, v1));
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float p = __fadd_rn((float)c1[r], __fmul_rn(mu, __fsub_rn((float)c2[r], (float)c1[r])));
    out[r] = p <= 65280.0f ? (p >= 0.0f ? (uint16_t)__float2int_rz(p) : (uint16_t)0) : (uint16_t)65280;
  }
}

struct Sample {
  float d, w;
  uint16_t c[3];
  uint16_t pad;
};

// axis roles per type: 0 = lattice of spacing sizeMin, 1 = the two samples
// either side of the shared boundary
__constant__ uint8_t c_role[7][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
// loop nesting of the reference's vertex/face loops, outer to inner axis
__constant__ uint8_t c_order[7][3] = {{2, 1, 0}, {2, 1, 0}, {2, 0, 1}, {1, 0, 2}, {0, 2, 1}, {1, 2, 0}, {2, 1, 0}};

struct CellGeom {
  int type, size, sizeMin, stretch;
  int cnt[3];
  int o[3];
  bool empty;
};

__device__ CellGeom cell_geom(const VoxSrc &m, const Cell &c) {
  CellGeom G;
  G.type = c.type;
  G.size = c.size;
  G.stretch = 0;
  G.empty = false;
  for (int r = 0; r < 3; r++) G.o[r] = c.o[r];
  const int t = c.type;
  if (t == 0) {
    G.sizeMin = m.leaf[c.L[0]].w;
    if (G.sizeMin > G.size || G.size / G.sizeMin > 8) G.empty = true;
    const ushort4 lo = m.leaf[c.L[0]];
    const int ext = lo.w * 8;
    if (G.o[0] + G.size > lo.x + ext || G.o[0] < lo.x || G.o[1] + G.size > lo.y + ext || G.o[1] < lo.y ||
        G.o[2] + G.size > lo.z + ext || G.o[2] < lo.z)
      G.empty = true;
  } else if (t <= 3) {
    const int a = m.leaf[c.L[0]].w, b = m.leaf[c.L[1]].w;
    G.sizeMin = min(a, b);
    G.stretch = a;
    if (G.stretch > G.size) G.empty = true;
  } else {
    const int s0 = m.leaf[c.L[0]].w, s1 = m.leaf[c.L[1]].w, s2 = m.leaf[c.L[2]].w, s3 = m.leaf[c.L[3]].w;
    G.stretch = max(max(s0, s1), s2);
    G.sizeMin = min(min(s0, s1), min(s2, s3));
    if (G.stretch > G.size) G.empty = true;
  }
  if (G.sizeMin <= 0) G.empty = true;
  for (int r = 0; r < 3; r++) G.cnt[r] = c_role[t][r] ? 2 : (G.empty ? 1 : (G.size + G.sizeMin - 1) / G.sizeMin);
  for (int r = 0; r < 3; r++)
    if (G.cnt[r] > 8) G.empty = true;  // a lattice never exceeds one brick
  return G;
}

__device__ __forceinline__ int sample_pos(const CellGeom &G, int r, int b) {
  return c_role[G.type][r] ? (b ? G.o[r] + G.size : G.o[r] + G.size - G.stretch) : G.o[r] + b * G.sizeMin;
}

// One lattice sample of an interior/wall/edge cell; returns false when the
// interior cell does not fit in a leaf of its chain (the reference then
// leaves the cell's mesh empty).
template <bool COLOR>
__device__ bool lattice_sample(const VoxSrc &m, const Cell &c, const CellGeom &G, int bx, int by, int bz, Sample &s) {
  const int t = G.type;
  const int bb[3] = {bx, by, bz};
  uint32_t first;
  if (t == 0)
    first = c.L[0];
  else if (t <= 3)
    first = c.L[bb[t - 1]];
  else {
    int p, q;
    others(t - 4, p, q);
    first = c.L[bb[p] + 2 * bb[q]];
  }
  s.w = 0.0f;
  s.d = 0.0f;
  s.c[0] = s.c[1] = s.c[2] = 0;
  int guard = 0;
  // (the parent is read only when the walk goes on: most samples settle at
  // their first leaf)
  for (uint32_t leaf = first; leaf < BRANCHINIT && s.w <= 0.0f && guard < 64;
       leaf = s.w <= 0.0f ? m.parent[leaf] : BRANCHINIT, guard++) {
    if (leaf >= m.leaves_used) break;
    const ushort4 lo4 = m.leaf[leaf];
    const int lo[3] = {lo4.x, lo4.y, lo4.z};
    const int ls = lo4.w;
    if (t == 0) {
      const int ext = ls * 8;
      for (int r = 0; r < 3; r++)
        if (G.o[r] + G.size > lo[r] + ext || G.o[r] < lo[r]) return false;
    }
    uint16_t ll[3], lh[3];
    float rr[3];
    // leaf scales are powers of two: divide by shifting (same truncating
    // quotient and remainder as / and %), and rem / ls is exact
    const bool pow2 = ls > 0 && (ls & (ls - 1)) == 0;
    const int sh = __ffs(ls) - 1;
    const float inv_ls = __int_as_float((127 - sh) << 23);
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const int p = sample_pos(G, r, bb[r]);
      const int num = p - lo[r];
      int q, rm;
      if (pow2) {
        const int mag = num < 0 ? -num : num;
        q = num < 0 ? -(mag >> sh) : (mag >> sh);
        rm = num < 0 ? -(mag & (ls - 1)) : (mag & (ls - 1));
      } else {
        q = num / ls;
        rm = num % ls;
      }
      ll[r] = (uint16_t)q;
      if (c_role[t][r]) {
        lh[r] = ll[r];
        rr[r] = 0.0f;
      } else {
        const uint16_t rem = (uint16_t)rm;
        rr[r] = pow2 ? __fmul_rn((float)rem, inv_ls) : __fdiv_rn((float)rem, (float)ls);
        lh[r] = (uint16_t)(ll[r] + (rr[r] > 0.0f && ll[r] < 7));
      }
    }
    if (t == 0 && rr[0] == 0.0f && rr[1] == 0.0f && rr[2] == 0.0f) {
      // on the leaf's lattice the weights are (1, 0, ..., 0) and the
      // trilinear sums reduce to the voxel itself (finite values)
      const size_t v0 = vox_index(m, leaf, ll[0], ll[1], ll[2]);
      const float d0 = vd(m, v0);
      if (isfinite(d0)) {
        s.w = __fadd_rn(s.w, vw(m, v0));
        s.d = d0;
#pragma unroll
        for (int r = 0; r < 3; r++) s.c[r] = vcs<COLOR>(m, v0, r);
        continue;
      }
    }
    if (t == 0) {
      // trilinear, summed as the reference's SSE code (mesh_interleaved_meshcell.cpp:144-230)
      const float rx = rr[0], ry = rr[1], rz = rr[2];
      const float rxn = __fsub_rn(1.0f, rx), ryn = __fsub_rn(1.0f, ry), rzn = __fsub_rn(1.0f, rz);
      const float f[8] = {__fmul_rn(__fmul_rn(rzn, ryn), rxn), __fmul_rn(__fmul_rn(rzn, ryn), rx),
                          __fmul_rn(__fmul_rn(rzn, ry), rxn),  __fmul_rn(__fmul_rn(rzn, ry), rx),
                          __fmul_rn(__fmul_rn(rz, ryn), rxn),  __fmul_rn(__fmul_rn(rz, ryn), rx),
                          __fmul_rn(__fmul_rn(rz, ry), rxn),   __fmul_rn(__fmul_rn(rz, ry), rx)};
      size_t vi[8];
#pragma unroll
      for (int k = 0; k < 8; k++)
        vi[k] = vox_index(m, leaf, (k & 1) ? lh[0] : ll[0], (k & 2) ? lh[1] : ll[1], (k & 4) ? lh[2] : ll[2]);
      // a sample on the leaf's own lattice reads one voxel 8 times: load it once
      const bool on_lattice = lh[0] == ll[0] && lh[1] == ll[1] && lh[2] == ll[2];
      float df[8];
      float cf3[3][8];
      if (on_lattice) {
        const float d0 = vd(m, vi[0]);
        const float c0 = (float)vcs<COLOR>(m, vi[0], 0), c1 = (float)vcs<COLOR>(m, vi[0], 1), c2 = (float)vcs<COLOR>(m, vi[0], 2);
#pragma unroll
        for (int k = 0; k < 8; k++) df[k] = d0, cf3[0][k] = c0, cf3[1][k] = c1, cf3[2][k] = c2;
      } else {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          df[k] = vd(m, vi[k]);
          cf3[0][k] = (float)vcs<COLOR>(m, vi[k], 0);
          cf3[1][k] = (float)vcs<COLOR>(m, vi[k], 1);
          cf3[2][k] = (float)vcs<COLOR>(m, vi[k], 2);
        }
      }
      s.w = __fadd_rn(s.w, vw(m, vi[0]));
      s.d = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f[0], df[0]), __fmul_rn(f[4], df[4])),
                                __fadd_rn(__fmul_rn(f[1], df[1]), __fmul_rn(f[5], df[5]))),
                      __fadd_rn(__fadd_rn(__fmul_rn(f[2], df[2]), __fmul_rn(f[6], df[6])),
                                __fadd_rn(__fmul_rn(f[3], df[3]), __fmul_rn(f[7], df[7]))));
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float *cf = cf3[r];
        const float v = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f[0], cf[0]), __fmul_rn(f[4], cf[4])),
                                            __fadd_rn(__fmul_rn(f[1], cf[1]), __fmul_rn(f[5], cf[5]))),
                                  __fadd_rn(__fadd_rn(__fmul_rn(f[2], cf[2]), __fmul_rn(f[6], cf[6])),
                                            __fadd_rn(__fmul_rn(f[3], cf[3]), __fmul_rn(f[7], cf[7]))));
        s.c[r] = (uint16_t)__float2int_rz(v);
      }
    } else if (t <= 3) {
      // bilinear over the two lattice axes a < b (addBrickWallX/Y/Z)
      const int a = t == 1 ? 1 : 0, b = t == 3 ? 1 : 2;
      const float ra = rr[a], rb = rr[b], ran = __fsub_rn(1.0f, ra), rbn = __fsub_rn(1.0f, rb);
      if (ra == 0.0f && rb == 0.0f) {
        // weights (1, 0, 0, 0): the sums reduce to the voxel itself (finite values)
        const size_t v0 = vox_index(m, leaf, ll[0], ll[1], ll[2]);
        const float w0 = vw(m, v0), d0 = vd(m, v0);
        if (isfinite(w0) && isfinite(d0)) {
          s.w = __fadd_rn(s.w, w0);
          s.d = d0;
#pragma unroll
          for (int r = 0; r < 3; r++) s.c[r] = vcs<COLOR>(m, v0, r);
          continue;
        }
      }
      const float f[4] = {__fmul_rn(rbn, ran), __fmul_rn(rbn, ra), __fmul_rn(rb, ran), __fmul_rn(rb, ra)};
      size_t vi[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint16_t l3[3] = {ll[0], ll[1], ll[2]};
        l3[a] = (k & 1) ? lh[a] : ll[a];
        l3[b] = (k & 2) ? lh[b] : ll[b];
        vi[k] = vox_index(m, leaf, l3[0], l3[1], l3[2]);
      }
      float wf[4], df[4], cf3[3][4];
      if (lh[a] == ll[a] && lh[b] == ll[b]) {
        // on the leaf's own lattice: one voxel
        const float w0 = vw(m, vi[0]), d0 = vd(m, vi[0]);
        const float c0 = (float)vcs<COLOR>(m, vi[0], 0), c1 = (float)vcs<COLOR>(m, vi[0], 1), c2 = (float)vcs<COLOR>(m, vi[0], 2);
#pragma unroll
        for (int k = 0; k < 4; k++) wf[k] = w0, df[k] = d0, cf3[0][k] = c0, cf3[1][k] = c1, cf3[2][k] = c2;
      } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          wf[k] = vw(m, vi[k]);
          df[k] = vd(m, vi[k]);
          cf3[0][k] = (float)vcs<COLOR>(m, vi[k], 0);
          cf3[1][k] = (float)vcs<COLOR>(m, vi[k], 1);
          cf3[2][k] = (float)vcs<COLOR>(m, vi[k], 2);
        }
      }
      const float wsum = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f[0], wf[0]), __fmul_rn(f[1], wf[1])),
                                             __fmul_rn(f[2], wf[2])),
                                   __fmul_rn(f[3], wf[3]));
      s.w = __fadd_rn(s.w, wsum);
      s.d = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f[0], df[0]), __fmul_rn(f[1], df[1])), __fmul_rn(f[2], df[2])),
                      __fmul_rn(f[3], df[3]));
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float *cf = cf3[r];
        const float v = __fadd_rn(
            __fadd_rn(__fadd_rn(__fmul_rn(f[0], cf[0]), __fmul_rn(f[1], cf[1])), __fmul_rn(f[2], cf[2])),
            __fmul_rn(f[3], cf[3]));
        s.c[r] = (uint16_t)__float2int_rz(v);
      }
    } else {
      // linear along the edge axis, weight = max of the two (addBrickEdgeX/Y/Z)
      const int a = t - 4;
      const float ra = rr[a], ran = __fsub_rn(1.0f, ra);
      uint16_t l3[3] = {ll[0], ll[1], ll[2]};
      const size_t v0 = vox_index(m, leaf, l3[0], l3[1], l3[2]);
      l3[a] = lh[a];
      const size_t v1 = vox_index(m, leaf, l3[0], l3[1], l3[2]);
      const float w0 = vw(m, v0), w1 = vw(m, v1);
      s.w = __fadd_rn(s.w, w0 < w1 ? w1 : w0);
      s.d = __fadd_rn(__fmul_rn(ran, vd(m, v0)), __fmul_rn(ra, vd(m, v1)));
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float v = __fadd_rn(__fmul_rn(ran, (float)vcs<COLOR>(m, v0, r)), __fmul_rn(ra, (float)vcs<COLOR>(m, v1, r)));
        s.c[r] = (uint16_t)__float2int_rz(v);
      }
    }
  }
  return true;
}

// An interior cell that is its leaf's whole brick: sample k (< 512) is
// voxel k of the brick (lattice_sample's first step reads that one voxel).
__device__ __forceinline__ bool brick_cell(const VoxSrc &m, const Cell &c, const CellGeom &G, uint32_t &leaf) {
  if (G.type != 0) return false;
  const uint32_t l0 = c.L[0];
  if (l0 >= BRANCHINIT || l0 >= m.leaves_used) return false;
  const ushort4 a = m.leaf[l0];
  const int ls = a.w;
  if (ls <= 0 || (ls & (ls - 1)) != 0 || G.sizeMin != ls || G.size != 8 * ls) return false;
  if (G.o[0] != a.x || G.o[1] != a.y || G.o[2] != a.z) return false;
  leaf = l0;
  return true;
}

// Per-warp shared scratch of one lattice cell.  Only the zero test of a
// sample's weight is needed after sampling; colours and vertex numbers are
// used by the emit pass alone, so the count pass's scratch stops before them
// (more warps per SM).
// Edge flags are bytes: plain stores, where bits would need atomics.
struct WarpScratch {
  float sd[512];           // SDF of each lattice sample
  uint8_t wzero[512];      // the sample's weight is zero
  uint8_t cube_case[512];  // marching-cubes case of each cube
  uint8_t edge_set[512 * 3];  // lattice-edge slots (3 per voxel) that carry a vertex
  uint16_t sc[512 * 3];    // emit pass: colour (R, G, B) of each sample
  uint16_t vidx[512 * 3];  // emit pass: the vertex number of each such slot
  uint16_t vlist[512 * 3];  // emit pass: the vertex-carrying slots in vertex order
};
constexpr size_t SCRATCH_COUNT_BYTES = offsetof(WarpScratch, sc);
constexpr size_t SCRATCH_EMIT_BYTES = sizeof(WarpScratch);
static_assert(SCRATCH_COUNT_BYTES % 16 == 0 && SCRATCH_EMIT_BYTES % 16 == 0, "scratch alignment");

__device__ __forceinline__ int edge_bit(const WarpScratch &W, int slot) { return W.edge_set[slot]; }

constexpr int MESH_WARPS = 4;

// Output of the count pass / input of the emit pass, per cell.
struct CellOut {
  uint32_t nv, nf;
};

// A position k < 512 of a lattice of extents n0 (fastest) x n1 x n2 split
// into its three coordinates.  The quotients are products with ceil(2^16 / d)
// shifted right by 16, exact while k (d - 1) < 2^16 (k < 512, d <= 64 here):
// the extents vary per cell, and a division by a value known only at run
// time costs a long instruction sequence per lattice position.
struct Lat3 {
  uint32_t n0, n1, m0, m01;  // extents, multipliers for n0 and n0 n1
};
__device__ __forceinline__ uint32_t quot_mul(uint32_t d) { return d ? (65536u + d - 1u) / d : 0u; }
__device__ __forceinline__ Lat3 lat3(int n0, int n1) {
  Lat3 L;
  L.n0 = (uint32_t)n0;
  L.n1 = (uint32_t)n1;
  L.m0 = quot_mul(L.n0);
  L.m01 = quot_mul(L.n0 * L.n1);
  return L;
}
__device__ __forceinline__ void split3(const Lat3 &L, int k, int &c0, int &c1, int &c2) {
  const uint32_t q0 = ((uint32_t)k * L.m0) >> 16;   // k / n0
  const uint32_t q01 = ((uint32_t)k * L.m01) >> 16;  // k / (n0 n1) = (k / n0) / n1
  c0 = k - (int)(q0 * L.n0);
  c1 = (int)(q0 - q01 * L.n1);
  c2 = (int)q01;
}

// lattice-order position k -> lattice index, for the cell type's loop nesting
// (L: the extents in that nesting, fastest first)
__device__ __forceinline__ int lattice_idx(const CellGeom &G, int k, const Lat3 &L, int &b0, int &b1, int &b2) {
  const uint8_t *ord = c_order[G.type];
  int i0, i1, i2;
  split3(L, k, i2, i1, i0);
  int bb[3];
  bb[ord[0]] = i0;
  bb[ord[1]] = i1;
  bb[ord[2]] = i2;
  b0 = bb[0];
  b1 = bb[1];
  b2 = bb[2];
  return (bb[2] * 8 + bb[1]) * 8 + bb[0];
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int &total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

// emit = false: count vertices/faces of each cell into out[]; emit = true:
// write them at vbase/fbase.
// The next cell for this warp (work: a counter that starts at zero).
__device__ __forceinline__ uint32_t next_cell(uint32_t *work, int lane) {
  uint32_t v = 0;
  if (lane == 0) v = atomicAdd(work, 1u);
  return __shfl_sync(0xffffffffu, v, 0);
}

// (register caps: the count pass's 4.6 KB of scratch per warp leaves room
// for 8 blocks per SM at 64 registers; the emit pass's 13.5 KB for 4)
template <bool EMIT>
__global__ void __launch_bounds__(32 * MESH_WARPS, EMIT ? 4 : 8) k_mesh_lattice(VoxSrc m, const Cell *__restrict__ cells,
                                                                  uint32_t first, uint32_t ncell,
                                                                  const uint32_t *__restrict__ list, const uint32_t *list_n, CellOut *out,
                                                                  const uint64_t *vbase, const uint64_t *fbase,
                                                                  float *xyz, uint8_t *rgb, uint32_t *faces,
                                                                  uint32_t *work, uint8_t *__restrict__ cases) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ McTab T;
  pdl_trigger();
  load_mc(T);  // (constant tables: before the wait for the kernel ahead)
  pdl_wait();
  WarpScratch &W = *reinterpret_cast<WarpScratch *>(smem_raw + (size_t)(threadIdx.x >> 5) *
                                                                      (EMIT ? SCRATCH_EMIT_BYTES : SCRATCH_COUNT_BYTES));
  const int lane = threadIdx.x & 31;
  // the dirty cells: a list of ids, or all cells of [first, first + ncell).
  // Emit: warps take the next cell from a shared counter (cells differ in
  // cost); count: a fixed stride (its cells are cheap next to the fetch).
  const uint32_t n = list ? *list_n : ncell;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t ci = EMIT ? next_cell(work, lane) : gw; ci < n; ci = EMIT ? next_cell(work, lane) : ci + nw) {
    const uint32_t cid = list ? list[ci] : first + ci;
    // emit: a cell that the count pass found without vertices writes nothing
    if (EMIT && out[cid].nv == 0) continue;
    const Cell c = cells[cid];
    if (!owns_cell(m, c)) {
      // another part meshes it
      if (!EMIT && lane == 0) out[cid] = CellOut{0u, 0u};
      continue;
    }
    const CellGeom G = cell_geom(m, c);
    if (G.empty) {
      if (!EMIT && lane == 0) out[cid] = CellOut{0u, 0u};
      continue;
    }
    const int n3[3] = {G.cnt[0], G.cnt[1], G.cnt[2]};
    const int nsamp = n3[0] * n3[1] * n3[2];
    const int nc3[3] = {n3[0] - 1, n3[1] - 1, n3[2] - 1};
    const int ncube = nc3[0] * nc3[1] * nc3[2];
    // (the lattices of samples and cubes are split by Lat3s made just
    // before each loop: in memory order, or in the cell type's loop nesting)
    const uint8_t *ord = c_order[G.type];
    // the count pass's marching-cubes case of every cube of this cell
    uint4 *const cell_cases = reinterpret_cast<uint4 *>(cases + (size_t)ci * 512);
    if (EMIT) {
      // Only the samples at the ends of lattice edges that carry a vertex
      // are read: the edge slots follow from the stored cube cases, and the
      // samples are the same function of the volume as in the count pass
      // (which found every sample of this cell inside its leaves).
      reinterpret_cast<uint4 *>(W.cube_case)[lane] = cell_cases[lane];
      for (int k = lane; k < 384; k += 32) reinterpret_cast<uint32_t *>(W.edge_set)[k] = 0;
      for (int k = lane; k < 128; k += 32) reinterpret_cast<uint32_t *>(W.wzero)[k] = 0;  // "needed" flags
      __syncwarp();
      const Lat3 Lc = lat3(nc3[0], nc3[1]);
      for (int k = lane; k < ncube; k += 32) {
        int bx, by, bz;
        split3(Lc, k, bx, by, bz);
        const int idx = (bz * 8 + by) * 8 + bx;
        const int ci8 = W.cube_case[idx];
        const int nt = mc_ntri(T, ci8);
        for (int q = 0; q < 3 * nt; q++) {
          const int slot = 3 * idx + mc_slot(T, mc_edge(T, ci8, q));
          const int si = slot / 3, a = slot - 3 * si;
          W.edge_set[slot] = 1;
          W.wzero[si] = 1;
          W.wzero[si + (a == 0 ? 1 : (a == 1 ? 8 : 64))] = 1;
        }
      }
      __syncwarp();
      // compact list of the needed sample indices (in vidx, free until the
      // vertex loop below)
      uint16_t *need = W.vidx;
      int nneed = 0;
      for (int k0 = 0; k0 < 512; k0 += 32) {
        const bool nd = W.wzero[k0 + lane] != 0;
        const unsigned b = __ballot_sync(0xffffffffu, nd);
        if (nd) need[nneed + __popc(b & ((1u << lane) - 1u))] = (uint16_t)(k0 + lane);
        nneed += __popc(b);
      }
      __syncwarp();
      if (lane == 0) atomicAdd(m.samples, (unsigned long long)nneed);
      for (int k = lane; k < nneed; k += 32) {
        const int si = need[k];
        Sample s;
        lattice_sample<true>(m, c, G, si & 7, (si >> 3) & 7, si >> 6, s);
        W.sd[si] = s.d;
        W.sc[3 * si] = s.c[0];
        W.sc[3 * si + 1] = s.c[1];
        W.sc[3 * si + 2] = s.c[2];
      }
      __syncwarp();
    } else {
      bool fit = true;
      const Lat3 Ls = lat3(n3[0], n3[1]);
      uint32_t bl;
      if (brick_cell(m, c, G, bl)) {
        // the brick's voxels in order; a sample that its voxel does not
        // settle (no weight, or not finite) takes the general path
        const size_t vb0 = (size_t)bl * 512;
        for (int k = lane; k < 512; k += 32) {
          const float d0 = vd(m, vb0 + k), w0 = vw(m, vb0 + k);
          if (isfinite(d0)) {
            const float w = __fadd_rn(0.0f, w0);
            if (!(w <= 0.0f)) {
              W.sd[k] = d0;
              W.wzero[k] = 0;
              continue;
            }
          }
          Sample s;
          fit &= lattice_sample<false>(m, c, G, k & 7, (k >> 3) & 7, k >> 6, s);
          W.sd[k] = s.d;
          W.wzero[k] = s.w == 0.0f;
        }
      } else
      for (int k = lane; k < nsamp; k += 32) {
        int bx, by, bz;
        split3(Ls, k, bx, by, bz);
        Sample s;
        fit &= lattice_sample<false>(m, c, G, bx, by, bz, s);  // (no colour: the count pass needs none)
        const int si = (bz * 8 + by) * 8 + bx;
        W.sd[si] = s.d;
        W.wzero[si] = s.w == 0.0f;
      }
      for (int k = lane; k < 384; k += 32) reinterpret_cast<uint32_t *>(W.edge_set)[k] = 0;
      fit = __all_sync(0xffffffffu, fit);
      __syncwarp();
      if (lane == 0) atomicAdd(m.samples, (unsigned long long)nsamp);
      if (!fit) {
        if (lane == 0) out[cid] = CellOut{0u, 0u};
        continue;
      }
      uint32_t tri = 0;  // this lane's cubes' triangles
      const Lat3 Lc = lat3(nc3[0], nc3[1]);
      for (int k = lane; k < ncube; k += 32) {
        int bx, by, bz;
        split3(Lc, k, bx, by, bz);
        const int idx = (bz * 8 + by) * 8 + bx;
        const int off[8] = {0, 1, 9, 8, 64, 65, 73, 72};
        bool zero = false;
        int ci8 = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
          zero |= W.wzero[idx + off[q]] != 0;
          if (W.sd[idx + off[q]] < 0.0f) ci8 |= 1 << q;
        }
        if (zero) ci8 = 0;
        W.cube_case[idx] = (uint8_t)ci8;
        const int nt = mc_ntri(T, ci8);
        tri += (uint32_t)nt;
        for (int q = 0; q < 3 * nt; q++) {
          const int slot = 3 * idx + mc_slot(T, mc_edge(T, ci8, q));
          W.edge_set[slot] = 1;  // lanes that set the same slot store the same byte
        }
      }
      __syncwarp();
      // kept for the emit pass (entries of cubes outside the lattice unused)
      cell_cases[lane] = reinterpret_cast<const uint4 *>(W.cube_case)[lane];
      // The counts need no order: a vertex per edge slot that carries one
      // (every such slot lies at a lattice sample, and the flags outside the
      // lattice are clear), a face per triangle of the lattice's cubes.
      uint32_t verts = 0;
      for (int k = lane; k < 384; k += 32) verts += (uint32_t)__popc(reinterpret_cast<const uint32_t *>(W.edge_set)[k]);
      verts = __reduce_add_sync(0xffffffffu, verts);
      tri = __reduce_add_sync(0xffffffffu, tri);
      if (lane == 0) out[cid] = CellOut{verts, tri};
      __syncwarp();
      continue;
    }
    // (the emit pass from here) vertices, in the reference's loop order of
    // this cell type: the slots that carry one listed in that order first
    // (a warp scan per 32 samples), then one lane per vertex
    uint32_t vrun = 0;
    const uint64_t vb = EMIT ? vbase[cid] : 0;
    const Lat3 Lso = lat3(n3[ord[2]], n3[ord[1]]);
    for (int k0 = 0; k0 < nsamp; k0 += 32) {
      const int k = k0 + lane;
      int b0 = 0, b1 = 0, b2 = 0, idx = 0, cntv = 0;
      if (k < nsamp) {
        idx = lattice_idx(G, k, Lso, b0, b1, b2);
        cntv = edge_bit(W, 3 * idx) + edge_bit(W, 3 * idx + 1) + edge_bit(W, 3 * idx + 2);
      }
      int tot;
      const int ex = warp_excl_scan(cntv, lane, tot);
      uint32_t at = vrun + (uint32_t)ex;
      for (int a = 0; a < 3 && cntv; a++)
        if (edge_bit(W, 3 * idx + a)) W.vlist[at++] = (uint16_t)(3 * idx + a);
      vrun += (uint32_t)tot;
    }
    __syncwarp();
    for (uint32_t q = lane; q < vrun; q += 32) {
      const int slot = W.vlist[q];
      const int idx = slot / 3, a = slot - 3 * idx;
      const int bb[3] = {idx & 7, (idx >> 3) & 7, idx >> 6};
      float P0[3];
#pragma unroll
      for (int r = 0; r < 3; r++) P0[r] = __fadd_rn(m.offset[r], __fmul_rn((float)sample_pos(G, r, bb[r]), m.scale));
      const int step = a == 0 ? 1 : (a == 1 ? 8 : 64);
      float P1[3] = {P0[0], P0[1], P0[2]};
      const int q2 = sample_pos(G, a, bb[a]) + (c_role[G.type][a] ? G.stretch : G.sizeMin);
      P1[a] = __fadd_rn(m.offset[a], __fmul_rn((float)q2, m.scale));
      float v[3];
      uint16_t col[3];
      const float d0 = W.sd[idx], d1 = W.sd[idx + step];
      vinterp(P0, P1, (double)d0, (double)d1, v);
      cinterp(&W.sc[3 * idx], &W.sc[3 * (idx + step)], d0, d1, col);
      const uint64_t gi = vb + q;
      xyz[3 * gi] = v[0];
      xyz[3 * gi + 1] = v[1];
      xyz[3 * gi + 2] = v[2];
      rgb[3 * gi] = (uint8_t)(col[0] / 256);
      rgb[3 * gi + 1] = (uint8_t)(col[1] / 256);
      rgb[3 * gi + 2] = (uint8_t)(col[2] / 256);
      W.vidx[slot] = (uint16_t)q;
    }
    __syncwarp();
    // faces, cube by cube in the same nesting
    uint32_t frun = 0;
    const uint64_t fb = EMIT ? fbase[cid] : 0;
    const Lat3 Lco = lat3(nc3[ord[2]], nc3[ord[1]]);
    for (int k0 = 0; k0 < ncube; k0 += 32) {
      const int k = k0 + lane;
      int idx = 0, nt = 0, ci8 = 0;
      if (k < ncube) {
        int b0, b1, b2;
        idx = lattice_idx(G, k, Lco, b0, b1, b2);
        ci8 = W.cube_case[idx];
        nt = mc_ntri(T, ci8);
      }
      int tot;
      int ex = warp_excl_scan(nt, lane, tot);
      if (EMIT) {
        for (int t = 0; t < nt; t++) {
          const uint64_t gf = fb + frun + (uint32_t)ex + t;
#pragma unroll
          for (int q = 0; q < 3; q++)
            faces[3 * gf + q] = (uint32_t)(vb + W.vidx[3 * idx + mc_slot(T, mc_edge(T, ci8, 3 * t + q))]);
        }
      }
      frun += (uint32_t)tot;
    }
    __syncwarp();
  }
}

// addBrickMiddle_indexed_incremental: eight lanes per corner cell, one per
// sample (the samples' parent-leaf walks are chains of dependent loads: in
// one thread they would run one after the other), then the cell's first lane
// runs the single-cube marching cubes on the gathered samples.
constexpr int CORNER_LANES = 8;

template <bool EMIT>
__global__ void k_mesh_corner(VoxSrc m, const Cell *__restrict__ cells, uint32_t first, uint32_t ncell,
                              const uint32_t *__restrict__ list, const uint32_t *list_n, CellOut *out,
                              const uint64_t *vbase, const uint64_t *fbase, float *xyz, uint8_t *rgb,
                              uint32_t *faces) {
  __shared__ McTab T;
  pdl_trigger();
  load_mc(T);  // (constant tables: before the wait for the kernel ahead)
  pdl_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = t / CORNER_LANES;
  const int k = (int)(t % CORNER_LANES);  // this lane's sample
  const unsigned gmask = 0xffu << (threadIdx.x & 24u);
  if (i >= (list ? *list_n : ncell)) return;
  const uint32_t cid = list ? list[i] : first + i;
  const Cell c = cells[cid];
  if (!owns_cell(m, c)) {
    if (!EMIT && k == 0) out[cid] = CellOut{0u, 0u};
    return;
  }
  // the largest leaf scale of sides 0-6
  int stretch = k < 7 ? (int)m.leaf[c.L[k]].w : 0;
#pragma unroll
  for (int o = 1; o < CORNER_LANES; o <<= 1) stretch = max(stretch, __shfl_xor_sync(gmask, stretch, o, CORNER_LANES));
  if (stretch > c.size) {
    if (!EMIT && k == 0) out[cid] = CellOut{0u, 0u};
    return;
  }
  {
    const unsigned act = __activemask();
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(act) - 1)) atomicAdd(m.samples, (unsigned long long)__popc(act));
  }
  float dk = 0.0f, wk = 0.0f;
  uint16_t ck[3] = {0, 0, 0};
  {
    int p[3];
    for (int r = 0; r < 3; r++) p[r] = ((k >> r) & 1) ? c.o[r] + c.size : c.o[r] + c.size - stretch;
    int guard = 0;
    for (uint32_t leaf = c.L[k]; leaf < BRANCHINIT && wk <= 0.0f && guard < 64;
         leaf = wk <= 0.0f ? m.parent[leaf] : BRANCHINIT, guard++) {
      if (leaf >= m.leaves_used) break;
      const ushort4 lo = m.leaf[leaf];
      const int ls = lo.w;
      const uint16_t lx = (uint16_t)(((int)(uint16_t)p[0] - (int)lo.x) / ls);
      const uint16_t ly = (uint16_t)(((int)(uint16_t)p[1] - (int)lo.y) / ls);
      const uint16_t lz = (uint16_t)(((int)(uint16_t)p[2] - (int)lo.z) / ls);
      const size_t vi = vox_index(m, leaf, lx, ly, lz);
      wk = __fadd_rn(wk, vw(m, vi));
      dk = vd(m, vi);
      for (int r = 0; r < 3; r++) ck[r] = vcs<EMIT>(m, vi, r);  // (the count pass needs no colour)
    }
  }
  // every lane of the cell gets all eight samples
  float d[8], w[8];
  uint16_t col[8][3];
  const uint32_t ck01 = (uint32_t)ck[0] | ((uint32_t)ck[1] << 16);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    d[j] = __shfl_sync(gmask, dk, j, CORNER_LANES);
    w[j] = __shfl_sync(gmask, wk, j, CORNER_LANES);
    const uint32_t a01 = __shfl_sync(gmask, ck01, j, CORNER_LANES);
    const uint32_t a2 = __shfl_sync(gmask, (uint32_t)ck[2], j, CORNER_LANES);
    col[j][0] = (uint16_t)(a01 & 0xffffu);
    col[j][1] = (uint16_t)(a01 >> 16);
    col[j][2] = (uint16_t)a2;
  }
  if (k != 0) return;
  const int mcv[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  float val[8];
  bool zero = false;
  int ci8 = 0;
  for (int k = 0; k < 8; k++) {
    val[k] = d[mcv[k]];
    zero |= w[mcv[k]] == 0.0f;
    if (val[k] < 0.0f) ci8 |= 1 << k;
  }
  if (zero) ci8 = 0;
  const float sx = __fmul_rn(m.scale, (float)stretch);
  float O[3];
  for (int r = 0; r < 3; r++) O[r] = __fadd_rn(m.offset[r], __fmul_rn((float)(c.o[r] + c.size - stretch), m.scale));
  float P[8][3];
  for (int k = 0; k < 8; k++) {
    const int bx = (k == 1 || k == 2 || k == 5 || k == 6), by = (k == 2 || k == 3 || k == 6 || k == 7), bz = k >= 4;
    P[k][0] = __fadd_rn(O[0], __fmul_rn((float)bx, sx));
    P[k][1] = __fadd_rn(O[1], __fmul_rn((float)by, sx));
    P[k][2] = __fadd_rn(O[2], __fmul_rn((float)bz, sx));
  }
  float vl[12][3];
  uint16_t cl[12][3];
  for (int e = 0; e < 12; e++) {
    const int a = c_edge_a[e], b = c_edge_b[e];
    if (((ci8 >> a) & 1) != ((ci8 >> b) & 1)) {
      vinterp(P[a], P[b], (double)val[a], (double)val[b], vl[e]);
      if (EMIT) cinterp(col[mcv[a]], col[mcv[b]], val[a], val[b], cl[e]);
    }
  }
  const int nt = mc_ntri(T, ci8);
  uint32_t kept = 0;
  const uint64_t vb = EMIT ? vbase[cid] : 0, fb = EMIT ? fbase[cid] : 0;
  for (int t = 0; t < nt; t++) {
    const int e0 = mc_edge(T, ci8, 3 * t), e1 = mc_edge(T, ci8, 3 * t + 1), e2 = mc_edge(T, ci8, 3 * t + 2);
    const float *v0 = vl[e0], *v1 = vl[e1], *v2 = vl[e2];
    const bool deg = (v0[0] == v1[0] && v0[1] == v1[1] && v0[2] == v1[2]) ||
                     (v2[0] == v1[0] && v2[1] == v1[1] && v2[2] == v1[2]) ||
                     (v0[0] == v2[0] && v0[1] == v2[1] && v0[2] == v2[2]);
    if (deg) continue;
    if (EMIT) {
      const int es[3] = {e0, e1, e2};
      for (int q = 0; q < 3; q++) {
        const uint64_t gi = vb + 3 * kept + q;
        for (int r = 0; r < 3; r++) {
          xyz[3 * gi + r] = vl[es[q]][r];
          rgb[3 * gi + r] = (uint8_t)(cl[es[q]][r] / 256);
        }
        faces[3 * (fb + kept) + q] = (uint32_t)gi;
      }
    }
    kept++;
  }
  if (!EMIT) out[cid] = CellOut{3 * kept, kept};
}

// ---------------------------------------------------------------------------
// Incremental bookkeeping
// ---------------------------------------------------------------------------

// a cell is dirty if it is new, its leaves changed, or a leaf on any of its
// parent chains was updated since the previous mesh
__global__ void k_mark_dirty(const Cell *cells, uint32_t n, const Cell *old_cells, uint32_t n_old,
                             const uint64_t *old_keys, const uint32_t *stamp, const uint32_t *parent,
                             uint32_t leaves_used, uint32_t since, uint8_t *dirty, int32_t *old_index,
                             uint32_t *n_dirty, uint32_t first_corner, uint32_t *list, uint32_t *n_list, int B) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Cell c = cells[i];
  const uint64_t key = cell_key(c, B);
  int32_t found = -1;
  uint32_t lo = 0, hi = n_old;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (old_keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  for (uint32_t j = lo; j < n_old && old_keys[j] == key; j++) {
    bool same = true;
    for (int k = 0; k < 8; k++) same &= old_cells[j].L[k] == c.L[k];
    if (same) {
      found = (int32_t)j;
      break;
    }
  }
  bool d = found < 0;
  const int nl = c.type == 0 ? 1 : (c.type <= 3 ? 2 : (c.type <= 6 ? 4 : 8));
  for (int k = 0; k < nl && !d; k++) {
    int guard = 0;
    for (uint32_t leaf = c.L[k]; leaf < leaves_used && guard < 64; leaf = parent[leaf], guard++)
      if (stamp[leaf] > since) {
        d = true;
        break;
      }
  }
  dirty[i] = d ? 1 : 0;
  old_index[i] = found;
  if (d) {
    atomicAdd(n_dirty, 1u);
    // lattice cells listed from the front, corner cells from first_corner
    if (i < first_corner) list[claim(n_list)] = i;
    else list[first_corner + claim(n_list + 1)] = i;
  }
}

// ---------------------------------------------------------------------------
// Exclusive scans of the cells' vertex and face counts (both at once): the
// mesh offsets of every cell, and the totals at index n.  Three launches: the
// sums of tiles of 4096 cells, a scan of the tile sums in one block, then
// each tile's scan from its offset.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 1024, SCAN_PER_THREAD = 4, SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

// Exclusive prefix over the block of each thread's pair (a, b); the block's
// totals in *ta, *tb.  Every thread of the 1024-thread block calls it.
__device__ __forceinline__ void block_scan2(uint64_t a, uint64_t b, uint64_t &pa, uint64_t &pb, uint64_t *ta,
                                            uint64_t *tb) {
  __shared__ uint64_t wa[32], wb[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t ia = a, ib = b;  // inclusive within the warp
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t ua = __shfl_up_sync(0xffffffffu, ia, o), ub = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) ia += ua, ib += ub;
  }
  if (lane == 31) wa[w] = ia, wb[w] = ib;
  __syncthreads();
  if (w == 0) {
    uint64_t xa = wa[lane], xb = wb[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t ua = __shfl_up_sync(0xffffffffu, xa, o), ub = __shfl_up_sync(0xffffffffu, xb, o);
      if (lane >= o) xa += ua, xb += ub;
    }
    wa[lane] = xa;  // inclusive over warps
    wb[lane] = xb;
  }
  __syncthreads();
  pa = (w ? wa[w - 1] : 0ull) + ia - a;
  pb = (w ? wb[w - 1] : 0ull) + ib - b;
  if (ta) *ta = wa[31];
  if (tb) *tb = wb[31];
  __syncthreads();  // (wa/wb reused by the next call)
}

__global__ void __launch_bounds__(SCAN_THREADS) k_count_tile_sums(const CellOut *__restrict__ out, uint32_t n,
                                                                  uint64_t *tile_v, uint64_t *tile_f) {
  pdl_enter();
  const uint32_t i0 = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER_THREAD;
  uint64_t a = 0, b = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++)
    if (i0 + k < n) a += out[i0 + k].nv, b += out[i0 + k].nf;
  uint64_t pa, pb, ta, tb;
  block_scan2(a, b, pa, pb, &ta, &tb);
  if (threadIdx.x == 0) {
    tile_v[blockIdx.x] = ta;
    tile_f[blockIdx.x] = tb;
  }
}

// One block: tile sums -> exclusive tile offsets (in place), totals to
// vbase[n] and fbase[n].
__global__ void __launch_bounds__(SCAN_THREADS) k_count_tile_scan(uint64_t *tile_v, uint64_t *tile_f, uint32_t ntiles,
                                                                  uint64_t *vbase, uint64_t *fbase, uint32_t n) {
  pdl_enter();
  __shared__ uint64_t carry_v, carry_f;
  if (threadIdx.x == 0) carry_v = carry_f = 0;
  __syncthreads();
  for (uint32_t c0 = 0; c0 < ntiles; c0 += SCAN_THREADS) {
    const uint32_t i = c0 + threadIdx.x;
    const uint64_t a = i < ntiles ? tile_v[i] : 0ull, b = i < ntiles ? tile_f[i] : 0ull;
    uint64_t pa, pb, ta, tb;
    block_scan2(a, b, pa, pb, &ta, &tb);
    if (i < ntiles) {
      tile_v[i] = carry_v + pa;
      tile_f[i] = carry_f + pb;
    }
    __syncthreads();
    if (threadIdx.x == 0) carry_v += ta, carry_f += tb;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    vbase[n] = carry_v;
    fbase[n] = carry_f;
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_count_tile_apply(const CellOut *__restrict__ out, uint32_t n,
                                                                   const uint64_t *tile_v, const uint64_t *tile_f,
                                                                   uint64_t *vbase, uint64_t *fbase) {
  pdl_enter();
  const uint32_t i0 = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER_THREAD;
  uint32_t cv[SCAN_PER_THREAD], cf[SCAN_PER_THREAD];
  uint64_t a = 0, b = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    const bool in = i0 + k < n;
    cv[k] = in ? out[i0 + k].nv : 0u;
    cf[k] = in ? out[i0 + k].nf : 0u;
    a += cv[k];
    b += cf[k];
  }
  uint64_t pa, pb;
  block_scan2(a, b, pa, pb, nullptr, nullptr);
  uint64_t ov = tile_v[blockIdx.x] + pa, of = tile_f[blockIdx.x] + pb;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    if (i0 + k < n) {
      vbase[i0 + k] = ov;
      fbase[i0 + k] = of;
    }
    ov += cv[k];
    of += cf[k];
  }
}

// clean cells copy their previous vertices and faces (faces re-based)
__global__ void k_copy_clean(const uint8_t *dirty, const int32_t *old_index, uint32_t n, const CellOut *out,
                             const uint64_t *vbase, const uint64_t *fbase, const uint64_t *old_vbase,
                             const uint64_t *old_fbase, const float *old_xyz, const uint8_t *old_rgb,
                             const uint32_t *old_faces, float *xyz, uint8_t *rgb, uint32_t *faces) {
  pdl_enter();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < n; i += nwarps) {
    if (dirty[i]) continue;
    const int32_t j = old_index[i];
    const uint64_t nv = out[i].nv, nf = out[i].nf;
    const uint64_t v0 = vbase[i], f0 = fbase[i], ov0 = old_vbase[j], of0 = old_fbase[j];
    for (uint64_t k = lane; k < 3 * nv; k += 32) {
      xyz[3 * v0 + k] = old_xyz[3 * ov0 + k];
      rgb[3 * v0 + k] = old_rgb[3 * ov0 + k];
    }
    for (uint64_t k = lane; k < 3 * nf; k += 32) faces[3 * f0 + k] = (uint32_t)(old_faces[3 * of0 + k] - ov0 + v0);
  }
}

__global__ void k_fill_counts_from_old(const uint8_t *dirty, const int32_t *old_index, uint32_t n,
                                       const CellOut *old_out, CellOut *out) {
  pdl_enter();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || dirty[i]) return;
  out[i] = old_out[old_index[i]];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// The mesher's buffers come from one stream-ordered pool per device that
// keeps freed memory (release threshold: never), so regrowing a buffer as the
// map grows neither synchronises nor returns memory to the driver.
static cudaError_t pool_of_current_device(cudaMemPool_t &pool) {
  static cudaMemPool_t pools[64] = {};
  static std::atomic<unsigned long long> made{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!(made.load() & (1ull << dev))) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep_all = ~0ull;
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep_all);
    if (e != cudaSuccess) return e;
    pools[dev] = p;
    made.fetch_or(1ull << dev);
  }
  pool = pools[dev];
  return cudaSuccess;
}

static cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool;
  cudaError_t e = pool_of_current_device(pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

template <typename T>
static cudaError_t grow_buf(T *&p, size_t &cap, size_t need, cudaStream_t s) {
  if (need <= cap && p) return cudaSuccess;
  size_t ncap = std::max<size_t>(2 * need, 4096);
  void *q = nullptr;
  cudaError_t e = pool_alloc(&q, sizeof(T) * ncap, s);
  if (e != cudaSuccess) return e;
  if (p) {
    e = cudaFreeAsync(p, s);
    if (e != cudaSuccess) return e;
  }
  p = (T *)q;
  cap = ncap;
  return cudaSuccess;
}

struct MeshImpl {
  // generation queues
  Slot *cellq[2] = {nullptr, nullptr};
  FaceItem *faceq[2] = {nullptr, nullptr};
  EdgeItem *edgeq[2] = {nullptr, nullptr};
  VertItem *vertq[2] = {nullptr, nullptr};
  size_t cap_cellq[2] = {0, 0}, cap_faceq[2] = {0, 0}, cap_edgeq[2] = {0, 0}, cap_vertq[2] = {0, 0};
  uint32_t n_corners = 0;
  // last update's largest level of each kind of queue (faces and edges: of
  // one axis), and its cell count
  size_t peak[5] = {0, 0, 0, 0, 0};
  int key_bits = 0;                   // bits per origin coordinate of old_keys / keys
  // words 8 n_cells, 9 error, 10 n_dirty, 11 n_corners, 12-13 samples;
  // from LEVEL_COUNTS: QK item counters per generation level
  uint32_t *d_count = nullptr;
  uint32_t *h_count = nullptr;
  // cells: unsorted, sorted (current), previous
  Cell *raw = nullptr, *cells = nullptr, *old_cells = nullptr;
  size_t cap_raw = 0, cap_cells = 0, cap_old = 0;
  uint64_t *keys = nullptr, *keys_sorted = nullptr, *old_keys = nullptr;
  size_t cap_keys = 0, cap_keys2 = 0, cap_oldkeys = 0;
  uint32_t *vals = nullptr, *vals_sorted = nullptr;
  size_t cap_vals = 0, cap_vals2 = 0;
  void *sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  uint32_t n_old = 0;
  // per-cell counts and offsets: current and previous
  CellOut *out = nullptr, *old_out = nullptr;
  size_t cap_out = 0, cap_oldout = 0;
  // nv/nf: the count scan's tile sums (vertices, faces) of 4096-cell tiles
  uint64_t *nv = nullptr, *nf = nullptr, *vbase = nullptr, *fbase = nullptr, *old_vbase = nullptr,
           *old_fbase = nullptr;
  size_t cap_nv = 0, cap_nf = 0, cap_vb = 0, cap_fb = 0, cap_ovb = 0, cap_ofb = 0;
  uint8_t *dirty = nullptr;
  size_t cap_dirty = 0;
  int32_t *old_index = nullptr;
  size_t cap_oi = 0;
  uint32_t *dlist = nullptr;  // dirty cell ids: lattice cells, then (from first_corner) corner cells
  size_t cap_dlist = 0;
  uint8_t *cases = nullptr;  // count pass -> emit pass: 512 cube cases per dirty lattice cell
  size_t cap_cases = 0;
  void *scan_tmp = nullptr;
  size_t scan_tmp_bytes = 0;
  // previous mesh (the current output moves here before the next update)
  float *old_xyz = nullptr;
  uint8_t *old_rgb = nullptr;
  uint32_t *old_faces = nullptr;
  size_t cap_oxyz = 0, cap_orgb = 0, cap_ofaces = 0;
  size_t cap_xyz = 0, cap_rgb = 0, cap_faces = 0;
  uint32_t since = 0;
  // incremental cell list: the previous update's leaf and branch counts and
  // growth count; per previous cell its kept flag, then their prefix; merged
  // keys; the last update's generated and kept cell counts
  uint32_t prev_leaves = 0, prev_branches = 0, grows = 0;
  uint32_t *keep = nullptr, *keep_tiles = nullptr;
  size_t cap_keep = 0, cap_keep_tiles = 0;
  uint64_t *mkeys = nullptr;
  size_t cap_mkeys = 0;
  uint32_t n_new = 0, n_kept = 0;
  bool redo_full = false;  // the last incremental list was inconsistent: regenerate every cell
  // the traversal's level-MESH_TOP_LEVELS items (TopCache), their count and
  // fit flag (device, pinned mirror), and whether they are current
  Slot *top_cellq = nullptr;
  FaceItem *top_faceq = nullptr;
  EdgeItem *top_edgeq = nullptr;
  VertItem *top_vertq = nullptr;
  size_t cap_top[4] = {0, 0, 0, 0};
  uint32_t *d_top_count = nullptr, *h_top_count = nullptr;
  bool top_valid = false;
  uint32_t gen_start_level = 0;  // the last update's first traversed level (statistics)
};

static MeshImpl &impl(MeshState &m) {
  if (!m.impl) m.impl = new MeshImpl();
  return *reinterpret_cast<MeshImpl *>(m.impl);
}

#define MCK(call)                                                              \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      err = std::string("meshing: ") + #call + ": " + cudaGetErrorString(e_);  \
      return 2;                                                                \
    }                                                                          \
  } while (0)

// Generate, sort and store the mesh cells of the current octree.
// Bits per origin coordinate in the cell keys of a volume of side n (a
// power of two): a cell's origin is the low corner of a slot inside the
// volume, so below n (k_cell_keys reports one that is not).
static int key_bits_for(uint32_t n) {
  int b = 1;
  while ((1u << b) < n) b++;
  return std::min(b, 16);
}

// Cell words of the counter array (d_count) used by the incremental list:
// cells kept, and kept before the previous list's first corner cell.
constexpr int KEPT_WORD = 20;
// d_count words 24, 25: the grid barrier of the one-launch traversal
constexpr int GEN_BARRIER_WORD = 24;

static int generate_cells(MeshImpl &I, const MeshInputs &in, bool incr, cudaStream_t s, uint32_t &ncells,
                          std::string &err) {
  const int key_bits = key_bits_for(in.n);
  const uint32_t n_old = incr ? I.n_old : 0u;
  // programmatic dependent launches, unless the stage profile is on
  const bool pdl = !in.prof->on;
  const uint32_t first_corner_old = n_old - std::min(I.n_corners, n_old);
  const uint32_t keep_tiles = (n_old + KEEP_THREADS - 1) / KEEP_THREADS;
  if (incr) {
    MCK(grow_buf(I.keep, I.cap_keep, (size_t)n_old + 1, s));
    MCK(grow_buf(I.keep_tiles, I.cap_keep_tiles, std::max<size_t>(keep_tiles, 1), s));
  }
  // queue sizes (faces and edges: per axis): a first guess from the octree
  // size, then the previous update's peaks with headroom (the map grows
  // slowly between updates)
  const uint32_t slots = std::max<uint32_t>(in.branches_used / 2, 64);
  size_t want[5] = {(size_t)slots * 2 + 4096, (size_t)slots * 2 + 4096, (size_t)slots * 2 + 4096,
                    (size_t)slots * 2 + 4096, (size_t)slots * 16 + 4096};
  for (int k = 0; k < 5; k++) want[k] = std::max<size_t>(want[k], I.peak[k] + I.peak[k] / 4 + 1024);
  for (int attempt = 0; attempt < 6; attempt++) {
    for (int b = 0; b < 2; b++) {
      MCK(grow_buf(I.cellq[b], I.cap_cellq[b], want[0], s));
      MCK(grow_buf(I.faceq[b], I.cap_faceq[b], 3 * want[1], s));
      MCK(grow_buf(I.edgeq[b], I.cap_edgeq[b], 3 * want[2], s));
      MCK(grow_buf(I.vertq[b], I.cap_vertq[b], want[3], s));
    }
    MCK(grow_buf(I.raw, I.cap_raw, want[4], s));
    if (!I.d_count) {
      MCK(pool_alloc((void **)&I.d_count, COUNT_WORDS * sizeof(uint32_t), s));
      MCK(cudaMallocHost((void **)&I.h_count, COUNT_WORDS * sizeof(uint32_t)));
    }
    MCK(cudaMemsetAsync(I.d_count, 0, COUNT_WORDS * sizeof(uint32_t), s));
    GenQueues Q;
    for (int b = 0; b < 2; b++) {
      Q.cellq[b] = I.cellq[b];
      Q.faceq[b] = I.faceq[b];
      Q.edgeq[b] = I.edgeq[b];
      Q.vertq[b] = I.vertq[b];
    }
    Q.lvl = I.d_count + LEVEL_COUNTS;
    Q.cap_cell = (uint32_t)std::min(I.cap_cellq[0], I.cap_cellq[1]);
    Q.cap_face = (uint32_t)(std::min(I.cap_faceq[0], I.cap_faceq[1]) / 3);
    Q.cap_edge = (uint32_t)(std::min(I.cap_edgeq[0], I.cap_edgeq[1]) / 3);
    Q.cap_vert = (uint32_t)std::min(I.cap_vertq[0], I.cap_vertq[1]);
    Q.cells = I.raw;
    Q.n_cells = I.d_count + 8;
    Q.cap_cells = (uint32_t)I.cap_raw;
    Q.error = I.d_count + 9;
    Q.n_corners = I.d_count + 11;
    GenCtx g;
    g.tree = in.tree;
    g.leaves_max = in.leaves_max;
    g.bstamp = in.bstamp;
    g.since = I.since;
    g.prev_leaves = I.prev_leaves;
    g.prev_branches = I.prev_branches;
    g.incr = incr ? 1 : 0;
    g.expand_all = 0;  // (set per level by the traversal)
    if (incr) {
      // the previous cells whose sides did not change, and their positions
      // among the kept (words KEPT_WORD, KEPT_WORD + 1: kept, kept before the
      // first corner cell)
      // (the scan and the apply: programmatic dependents of the kernel before)
      note_launch(3);
      k_keep_cells<<<keep_tiles, KEEP_THREADS, 0, s>>>(g, in.n, I.old_cells, n_old, I.keep, I.keep_tiles);
      MCK(launch_pdl(pdl, k_keep_tile_scan, dim3(1), dim3(KEEP_SCAN_THREADS), 0, s, I.keep_tiles, keep_tiles));
      MCK(launch_pdl(pdl, k_keep_apply, dim3(keep_tiles), dim3(KEEP_THREADS), 0, s, I.keep, n_old,
                     (const uint32_t *)I.keep_tiles, keep_tiles, first_corner_old, I.d_count + KEPT_WORD));
    }
    // The top levels: an incremental update whose frames created nothing
    // near the root starts from the kept level-MESH_TOP_LEVELS items;
    // otherwise the top levels run (in an incremental update expanding every
    // item, so that the whole level is there to keep, but emitting only the
    // changed items' cells) and their output is kept for the next updates.
    constexpr int LC = MESH_TOP_LEVELS;
    if (!I.d_top_count) {
      MCK(pool_alloc((void **)&I.d_top_count, (QK + 1) * sizeof(uint32_t), s));
      MCK(cudaMallocHost((void **)&I.h_top_count, (QK + 1) * sizeof(uint32_t)));
      I.h_top_count[QK] = 1;
    }
    TopCache T;
    T.cellq = I.top_cellq;
    T.faceq = I.top_faceq;
    T.edgeq = I.top_edgeq;
    T.vertq = I.top_vertq;
    for (int k = 0; k < 4; k++) T.cap[k] = (uint32_t)(k == 1 || k == 2 ? I.cap_top[k] / 3 : I.cap_top[k]);
    T.count = I.d_top_count;
    const bool use_top = incr && I.top_valid && !in.top_changed;
    const int lv0 = use_top ? LC : 0;
    if (!use_top) {
      // room for the level's items: as much as the queues hold, at most the
      // 8^LC cell items and 27^LC items of each other kind the level can have
      size_t most = 1, cells_most = 1;
      for (int k = 0; k < LC; k++) most *= 27, cells_most *= 8;
      MCK(grow_buf(I.top_cellq, I.cap_top[0], std::min(want[0], cells_most), s));
      MCK(grow_buf(I.top_faceq, I.cap_top[1], 3 * std::min(want[1], most), s));
      MCK(grow_buf(I.top_edgeq, I.cap_top[2], 3 * std::min(want[2], most), s));
      MCK(grow_buf(I.top_vertq, I.cap_top[3], std::min(want[3], most), s));
      T.cellq = I.top_cellq;
      T.faceq = I.top_faceq;
      T.edgeq = I.top_edgeq;
      T.vertq = I.top_vertq;
      for (int k = 0; k < 4; k++) T.cap[k] = (uint32_t)(k == 1 || k == 2 ? I.cap_top[k] / 3 : I.cap_top[k]);
    }
    I.gen_start_level = (uint32_t)lv0;
    if (use_top) {
      note_launch(1);
      // (after the keep test's last kernel: a programmatic dependent)
      MCK(launch_pdl(pdl, k_load_top, dim3(148 * 2), dim3(256), 0, s, Q, (int)LC, T));
    }
    // An item of level l holds slots of depth l at most, and it expands only
    // if one of them is subdivided, so the last level with items is the
    // depth of the finest slots (size 8, the finest leaf's brick): the first
    // batch runs the levels down to it, and further ones only run if items
    // are left all the same.
    int depth = 1;
    for (uint32_t h = in.n; h > 8; h >>= 1) depth++;
    int lv = lv0, batch = std::max(depth - lv0, 1);
    bool leftover = true;
    while (leftover && lv < MAX_GEN_LEVELS) {
      const int end = std::min(lv + batch, MAX_GEN_LEVELS);
      // the widest level of the last update (an incremental update's levels
      // hold few items), or as many blocks as fit for a full generation
      const size_t widest = incr ? I.peak[0] + 3 * I.peak[1] + 3 * I.peak[2] + I.peak[3] : SIZE_MAX / 2;
      const int blocks = gen_blocks(widest);
      if (!blocks) {
        err = "meshing: no resident blocks for the cell generation";
        return 2;
      }
      GenRun R;
      R.lv0 = lv;
      R.lv_end = end;
      R.incr = incr ? 1 : 0;
      // level LC's items are complete once level LC - 1 has run: keep them
      R.save_level = (!use_top && lv < LC && LC <= end) ? LC : -1;
      R.bar = I.d_count + GEN_BARRIER_WORD;
      R.spin_limit = in.spin_limit;
      void *args[] = {&g, &Q, &R, (void *)&in.n, &T};
      note_launch(1);
      MCK(cudaLaunchCooperativeKernel((const void *)k_gen_levels, dim3(blocks), dim3(GEN_THREADS), args, 0, s));
      lv = end;
      MCK(cudaGetLastError());
      MCK(cudaMemcpyAsync(I.h_count, I.d_count, COUNT_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      if (!use_top)
        MCK(cudaMemcpyAsync(I.h_top_count, I.d_top_count, (QK + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      MCK(cudaStreamSynchronize(s));
      const uint32_t *cl = I.h_count + LEVEL_COUNTS + QK * lv;
      leftover = false;
      for (int k = 0; k < QK; k++) leftover |= cl[k] != 0;
      if (I.h_count[9] & (ERR_CELL_OVERFLOW | ERR_CELL_TIMEOUT)) break;
      batch = 2;
    }
    if (I.h_count[9] & ERR_CELL_TIMEOUT) {
      // the traversal stopped part way: nothing of this update is used (the
      // previous list and state stay as they were); the top-level items are
      // traversed again next time
      I.top_valid = false;
      err = "meshing: a grid barrier of the cell generation gave up (spin limit)";
      return 5;
    }
    const bool overflow = (I.h_count[9] & ERR_CELL_OVERFLOW) != 0;
    const uint32_t *hc = I.h_count;
    if (!use_top) {
      // kept if it fitted; else the cache grows to the level's size and is
      // filled by the next update that traverses the top levels
      I.top_valid = !overflow && I.h_top_count[QK] == 0 && lv > LC;
      if (!I.top_valid && !overflow) {
        const uint32_t *cl = hc + LEVEL_COUNTS + QK * LC;
        const size_t nf = std::max({cl[QK_FACE], cl[QK_FACE + 1], cl[QK_FACE + 2]});
        const size_t ne = std::max({cl[QK_EDGE], cl[QK_EDGE + 1], cl[QK_EDGE + 2]});
        MCK(grow_buf(I.top_cellq, I.cap_top[0], (size_t)cl[QK_CELL] + cl[QK_CELL] / 4 + 256, s));
        MCK(grow_buf(I.top_faceq, I.cap_top[1], 3 * (nf + nf / 4 + 256), s));
        MCK(grow_buf(I.top_edgeq, I.cap_top[2], 3 * (ne + ne / 4 + 256), s));
        MCK(grow_buf(I.top_vertq, I.cap_top[3], (size_t)cl[QK_VERT] + cl[QK_VERT] / 4 + 256, s));
      }
    }
    if (overflow) {
      for (int k = 0; k < 5; k++) want[k] *= 2;
      continue;
    }
    for (int k = 0; k < 5; k++) I.peak[k] = 0;
    // (queue k's kind: cells, faces, edges, vertices)
    for (int l = 0; l <= lv; l++)
      for (int k = 0; k < QK; k++) {
        const int kind = k == QK_CELL ? 0 : (k < QK_EDGE ? 1 : (k < QK_VERT ? 2 : 3));
        I.peak[kind] = std::max<size_t>(I.peak[kind], hc[LEVEL_COUNTS + QK * l + k]);
      }
    I.peak[4] = hc[8];
    if (leftover) {
      err = "meshing: cell generation did not finish within the level limit";
      return 6;
    }
    const uint32_t n_kept = incr ? hc[KEPT_WORD] : 0u;
    const uint32_t kept_corners = incr ? n_kept - hc[KEPT_WORD + 1] : 0u;
    I.n_new = hc[8];
    I.n_kept = n_kept;
    ncells = n_kept + I.n_new;
    I.n_corners = hc[11] + kept_corners;
    break;
  }
  if (I.h_count[9] & ERR_CELL_OVERFLOW) {
    err = "meshing: cell queues overflow";
    return 4;
  }
  // sort the generated cells by key: deterministic order and a stable
  // identity across updates; with a kept list, merge the two
  const uint32_t n_new = I.n_new;
  MCK(grow_buf(I.keys, I.cap_keys, n_new, s));
  MCK(grow_buf(I.keys_sorted, I.cap_keys2, std::max(n_new, ncells), s));
  MCK(grow_buf(I.vals_sorted, I.cap_vals2, n_new, s));
  MCK(grow_buf(I.cells, I.cap_cells, ncells, s));
  if (incr) MCK(grow_buf(I.mkeys, I.cap_mkeys, ncells, s));
  // (keys, sort and merge follow one another on the stream: the sort and the
  // merge or gather are programmatic dependents of the kernel before them)
  if (n_new) {
    const int end_bit = 3 * key_bits + 7;
    const size_t bytes = argsort_temp_bytes(n_new);
    if (bytes > I.sort_tmp_bytes) {
      if (I.sort_tmp) MCK(cudaFreeAsync(I.sort_tmp, s));
      I.sort_tmp = nullptr;
      MCK(pool_alloc(&I.sort_tmp, bytes, s));
      I.sort_tmp_bytes = bytes;
    }
    note_launch(1);
    k_cell_keys<<<(n_new + 255) / 256, 256, 0, s>>>(I.raw, n_new, key_bits, I.keys, I.d_count + 9);
    unsigned sort_launches = 0;
    MCK(argsort_u64(I.keys, n_new, end_bit, I.keys_sorted, I.vals_sorted, I.sort_tmp, I.sort_tmp_bytes, s,
                    &sort_launches, pdl));
    note_launch(sort_launches);
  }
  if (!incr) {
    if (n_new) {
      note_launch(1);
      MCK(launch_pdl(pdl, k_gather_cells, dim3((n_new + 255) / 256), dim3(256), 0, s, (const Cell *)I.raw,
                     (const uint32_t *)I.vals_sorted, n_new, I.cells));
    }
  } else if (ncells) {
    // kept and new cells merged in key order; the merged keys replace the
    // sorted ones
    note_launch(1);
    MCK(launch_pdl(pdl && n_new > 0, k_merge_cells, dim3((n_old + n_new + 255) / 256), dim3(256), 0, s,
                   (const Cell *)I.old_cells, (const uint64_t *)I.old_keys, (const uint32_t *)I.keep, n_old,
                   (const Cell *)I.raw, (const uint64_t *)I.keys_sorted, (const uint32_t *)I.vals_sorted, n_new,
                   I.cells, I.mkeys, I.d_count + 9));
    std::swap(I.mkeys, I.keys_sorted);
    std::swap(I.cap_mkeys, I.cap_keys2);
  }
  return 0;
}

// Reserve pool memory once (allocate and free a block): later buffer growth
// is served from it instead of fresh driver allocations.
static cudaError_t reserve_pool(size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev & 63]) return cudaSuccess;
  void *p = nullptr;
  e = pool_alloc(&p, bytes, s);
  if (e != cudaSuccess) return e;
  e = cudaFreeAsync(p, s);
  if (e == cudaSuccess) done[dev & 63] = true;
  return e;
}

int mesh_update(MeshState &M, const MeshInputs &in, cudaStream_t s, std::string &err) {
  // about 2 KB of mesher memory per brick of capacity, at most 512 MB
  MCK(reserve_pool(std::min<size_t>((size_t)in.leaves_max * 2048, (size_t)512 << 20), s));
  MeshImpl &I = impl(M);
  uint32_t ncells = 0;
  Prof &P = *in.prof;
  int pi = P.begin(ST_MESH_CELLS, s);
  // the previous list can be kept where the octree did not change: not after
  // a growth (every cell moves) or a change of the key layout
  const bool incr_cells = M.valid && I.n_old > 0 && I.key_bits == key_bits_for(in.n) && !in.full_cells &&
                          I.grows == in.grows && !I.redo_full;
  const uint32_t n_old_cells = incr_cells ? I.n_old : 0u;
  int rc = generate_cells(I, in, incr_cells, s, ncells, err);
  if (rc) return rc;
  // sizeof(Cell) = 44 B per cell read or written: the previous list read by the keep test,
  // the new cells written by the traversal and read by the gather or merge,
  // the kept cells read by the merge, the list written
  P.end(pi, (double)sizeof(Cell) * ((double)n_old_cells + 2.0 * I.n_new + I.n_kept + ncells), s);
  VoxSrc vs;
  vs.leaf = in.leaf;
  vs.parent = in.parent;
  vs.sdf = in.sdf;
  vs.wgt = in.wgt;
  vs.sdf16 = in.sdf16;
  vs.wgt16 = in.wgt16;
  vs.col = in.col;
  vs.fp16 = in.storage == 1;
  vs.leaves_used = in.leaves_used;
  for (int r = 0; r < 3; r++) vs.offset[r] = in.offset[r];
  vs.scale = in.scale;
  vs.shard = in.shard;
  vs.shards = in.shards;
  for (int r = 0; r < 3; r++) vs.shift[r] = in.shift[r];
  // d_count words 12-13 hold the sample counter (8-byte aligned)
  vs.samples = reinterpret_cast<unsigned long long *>(I.d_count + 12);
  MCK(cudaMemsetAsync(I.d_count + 12, 0, 2 * sizeof(uint32_t), s));

  MCK(grow_buf(I.out, I.cap_out, ncells, s));
  MCK(grow_buf(I.dirty, I.cap_dirty, ncells, s));
  MCK(grow_buf(I.old_index, I.cap_oi, ncells, s));
  MCK(grow_buf(I.vbase, I.cap_vb, ncells + 1, s));
  MCK(grow_buf(I.fbase, I.cap_fb, ncells + 1, s));
  MCK(grow_buf(I.dlist, I.cap_dlist, ncells, s));
  // the previous update's keys are comparable only with the same key layout
  const int kb = key_bits_for(in.n);
  const bool incremental = M.valid && I.n_old > 0 && I.key_bits == kb;
  // the sorted cell list holds interiors, walls, edges, then corners (type is
  // the key's top field)
  const uint32_t first_corner = ncells - std::min(I.n_corners, ncells);
  // buffers of the count pass and the scans, ahead of the kernels (nothing
  // but kernels between them on the stream)
  const uint32_t ntiles = (ncells + SCAN_TILE - 1) / SCAN_TILE;
  MCK(grow_buf(I.cases, I.cap_cases, (size_t)first_corner * 512, s));
  MCK(grow_buf(I.nv, I.cap_nv, std::max<uint32_t>(ntiles, 1), s));  // tile sums of the vertex counts
  MCK(grow_buf(I.nf, I.cap_nf, std::max<uint32_t>(ntiles, 1), s));  // and of the face counts
  // programmatic dependent launches, unless the stage profile's events lie
  // between the kernels
  const bool pdl = !P.on;
  // dirty cells: all on the first update, otherwise those whose inputs changed
  MCK(cudaMemsetAsync(I.d_count + 10, 0, sizeof(uint32_t), s));
  MCK(cudaMemsetAsync(I.d_count + 14, 0, 2 * sizeof(uint32_t), s));
  if (ncells) {
    if (incremental) {
      note_launch(2);
      k_mark_dirty<<<(ncells + 255) / 256, 256, 0, s>>>(I.cells, ncells, I.old_cells, I.n_old, I.old_keys, in.stamp,
                                                        in.parent, in.leaves_used, I.since, I.dirty, I.old_index,
                                                        I.d_count + 10, first_corner, I.dlist, I.d_count + 14,
                                                        kb);
      MCK(launch_pdl(pdl, k_fill_counts_from_old, dim3((ncells + 255) / 256), dim3(256), 0, s, I.dirty, I.old_index,
                     ncells, I.old_out, I.out));
    } else {
      MCK(cudaMemsetAsync(I.dirty, 1, ncells, s));
    }
  }
  const size_t smem_count = SCRATCH_COUNT_BYTES * MESH_WARPS, smem_emit = SCRATCH_EMIT_BYTES * MESH_WARPS;
  static std::atomic<unsigned long long> attr_devices{0};
  int dev = 0;
  MCK(cudaGetDevice(&dev));
  const unsigned long long dbit = 1ull << (dev & 63);
  if (!(attr_devices.load() & dbit)) {
    MCK(cudaFuncSetAttribute(k_mesh_lattice<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_count));
    MCK(cudaFuncSetAttribute(k_mesh_lattice<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_emit));
    attr_devices.fetch_or(dbit);
  }
  const uint32_t *lat_list = incremental ? I.dlist : nullptr;
  const uint32_t *cor_list = incremental ? I.dlist + first_corner : nullptr;
  pi = P.begin(ST_MESH_COUNT, s);
  const int lat_blocks = std::max(1, std::min<int>(148 * 8, (int)((first_corner + MESH_WARPS - 1) / MESH_WARPS)));
  note_launch((first_corner ? 1 : 0) + (ncells > first_corner ? 1 : 0) + (ncells ? 1 : 0));
  // (the kernels from here to the totals' copy follow one another on the
  // stream: each after the first is a programmatic dependent of the one
  // before; the dirty marking is one when the volume's cells were kept)
  bool chained = pdl && incremental && ncells;
  if (first_corner) {
    MCK(launch_pdl(chained, k_mesh_lattice<false>, dim3(lat_blocks), dim3(32 * MESH_WARPS), smem_count, s, vs,
                   (const Cell *)I.cells, 0u, first_corner, lat_list, (const uint32_t *)(I.d_count + 14), I.out,
                   (const uint64_t *)nullptr, (const uint64_t *)nullptr, (float *)nullptr, (uint8_t *)nullptr,
                   (uint32_t *)nullptr, I.d_count + 16, I.cases));
    chained = pdl;
  }
  if (ncells > first_corner) {
    MCK(launch_pdl(chained, k_mesh_corner<false>, dim3(((ncells - first_corner) * CORNER_LANES + 127) / 128),
                   dim3(128), 0, s, vs, (const Cell *)I.cells, first_corner, ncells - first_corner, cor_list,
                   (const uint32_t *)(I.d_count + 15), I.out, (const uint64_t *)nullptr, (const uint64_t *)nullptr,
                   (float *)nullptr, (uint8_t *)nullptr, (uint32_t *)nullptr));
    chained = pdl;
  }
  const int pi_count = pi;
  P.end(pi_count, 0.0, s);
  MCK(cudaGetLastError());
  // exclusive scans of vertex and face counts -> per-cell bases (totals at ncells)
  {
    note_launch(ntiles ? 3 : 1);
    if (ntiles) {
      MCK(launch_pdl(chained, k_count_tile_sums, dim3(ntiles), dim3(SCAN_THREADS), 0, s, (const CellOut *)I.out,
                     ncells, I.nv, I.nf));
      chained = pdl;
    }
    MCK(launch_pdl(chained, k_count_tile_scan, dim3(1), dim3(SCAN_THREADS), 0, s, I.nv, I.nf, ntiles, I.vbase,
                   I.fbase, ncells));
    if (ntiles)
      MCK(launch_pdl(pdl, k_count_tile_apply, dim3(ntiles), dim3(SCAN_THREADS), 0, s, (const CellOut *)I.out, ncells,
                     (const uint64_t *)I.nv, (const uint64_t *)I.nf, I.vbase, I.fbase));
  }
  // totals, dirty count and samples through the pinned counter mirror
  uint64_t *h_tot = reinterpret_cast<uint64_t *>(I.h_count + HOST_TOTALS);
  MCK(cudaMemcpyAsync(h_tot + 0, I.vbase + ncells, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(h_tot + 1, I.fbase + ncells, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(h_tot + 2, I.d_count + 12, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(I.h_count + HOST_TOTALS + 6, I.d_count + 10, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(I.h_count + HOST_TOTALS + 7, I.d_count + 9, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  MCK(cudaStreamSynchronize(s));
  if (I.h_count[HOST_TOTALS + 7] & ERR_CELL_KEY) {
    mesh_invalidate(M);
    err = "meshing: a mesh cell lies outside the volume";
    return 6;
  }
  if (I.h_count[HOST_TOTALS + 7] & ERR_CELL_MERGE) {
    // the kept and the new cells overlap: build this update from the whole
    // octree instead (every cell generated and meshed again)
    if (!incr_cells) {
      mesh_invalidate(M);
      err = "meshing: two mesh cells share a sort key";
      return 6;
    }
    mesh_invalidate(M);
    I.redo_full = true;
    rc = mesh_update(M, in, s, err);
    I.redo_full = false;
    return rc;
  }
  const uint64_t tot[2] = {h_tot[0], h_tot[1]};
  const unsigned long long nsamples = h_tot[2];
  const uint32_t ndirty = incremental ? I.h_count[HOST_TOTALS + 6] : ncells;
  // count pass: SDF and weight of every sample of the dirty cells (the emit
  // pass reads colour as well: sample_bytes)
  const double sample_bytes = vs.fp16 ? 10.0 : 14.0;
  P.set_bytes(pi_count, (double)nsamples * (vs.fp16 ? 4.0 : 8.0));
  // the previous output becomes the copy source; the new output is written fresh
  std::swap(I.old_xyz, M.d_xyz);
  std::swap(I.cap_oxyz, I.cap_xyz);
  std::swap(I.old_rgb, M.d_rgb);
  std::swap(I.cap_orgb, I.cap_rgb);
  std::swap(I.old_faces, M.d_faces);
  std::swap(I.cap_ofaces, I.cap_faces);
  MCK(grow_buf(M.d_xyz, I.cap_xyz, 3 * tot[0] + 3, s));
  MCK(grow_buf(M.d_rgb, I.cap_rgb, 3 * tot[0] + 3, s));
  MCK(grow_buf(M.d_faces, I.cap_faces, 3 * tot[1] + 3, s));
  // the emit pass counts the samples it reads in d_count words 18-19
  vs.samples = reinterpret_cast<unsigned long long *>(I.d_count + 18);
  pi = P.begin(ST_MESH_EMIT, s);
  note_launch((first_corner ? 1 : 0) + (ncells > first_corner ? 1 : 0) + (incremental && ncells ? 1 : 0));
  // (the emit kernels after the first: programmatic dependents of the one
  // before)
  chained = false;
  if (first_corner) {
    k_mesh_lattice<true><<<lat_blocks, 32 * MESH_WARPS, smem_emit, s>>>(vs, I.cells, 0, first_corner, lat_list,
                                                                   I.d_count + 14, I.out, I.vbase, I.fbase, M.d_xyz,
                                                                   M.d_rgb, M.d_faces, I.d_count + 17, I.cases);
    chained = pdl;
  }
  if (ncells > first_corner) {
    MCK(launch_pdl(chained, k_mesh_corner<true>, dim3(((ncells - first_corner) * CORNER_LANES + 127) / 128),
                   dim3(128), 0, s, vs, (const Cell *)I.cells, first_corner, ncells - first_corner, cor_list,
                   (const uint32_t *)(I.d_count + 15), I.out, (const uint64_t *)I.vbase, (const uint64_t *)I.fbase,
                   M.d_xyz, M.d_rgb, M.d_faces));
    chained = pdl;
  }
  if (incremental && ncells)
    MCK(launch_pdl(chained, k_copy_clean, dim3(148 * 8), dim3(256), 0, s, (const uint8_t *)I.dirty,
                   (const int32_t *)I.old_index, ncells, (const CellOut *)I.out, (const uint64_t *)I.vbase,
                   (const uint64_t *)I.fbase, (const uint64_t *)I.old_vbase, (const uint64_t *)I.old_fbase,
                   (const float *)I.old_xyz, (const uint8_t *)I.old_rgb, (const uint32_t *)I.old_faces, M.d_xyz,
                   M.d_rgb, M.d_faces));
  // emit pass: the samples it reads (the ends of vertex-carrying lattice
  // edges, corner cells' 8) and the whole mesh written (xyz 12 B + rgb 3 B
  // per vertex, 12 B per face); the sample count arrives with the final sync
  const int pi_emit = pi;
  P.end(pi_emit, 0.0, s);
  MCK(cudaGetLastError());
  uint64_t *h_emit = reinterpret_cast<uint64_t *>(I.h_count + HOST_TOTALS + 8);
  if (P.on) MCK(cudaMemcpyAsync(h_emit, I.d_count + 18, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  // keep this update's cells, counts and bases for the next one
  std::swap(I.cells, I.old_cells);
  std::swap(I.cap_cells, I.cap_old);
  std::swap(I.keys_sorted, I.old_keys);
  std::swap(I.cap_keys2, I.cap_oldkeys);
  std::swap(I.out, I.old_out);
  std::swap(I.cap_out, I.cap_oldout);
  std::swap(I.vbase, I.old_vbase);
  std::swap(I.cap_vb, I.cap_ovb);
  std::swap(I.fbase, I.old_fbase);
  std::swap(I.cap_fb, I.cap_ofb);
  I.n_old = ncells;
  I.key_bits = kb;
  I.since = in.frame;
  I.prev_leaves = in.leaves_used;
  I.prev_branches = in.branches_used;
  I.grows = in.grows;
  // The emit pass may still run when this returns: everything that reads the
  // mesh or the volume later is ordered after it on this stream.  With the
  // stage profile on, wait for its sample count (the stage's bytes).
  if (P.on) {
    MCK(cudaStreamSynchronize(s));
    P.set_bytes(pi_emit, (double)*h_emit * sample_bytes + (double)tot[0] * 15 + (double)tot[1] * 12);
  }
  M.n_vertices = tot[0];
  M.n_faces = tot[1];
  M.n_cells = ncells;
  M.n_dirty = ndirty;
  M.n_generated = I.n_new;
  M.top_kept = I.gen_start_level > 0;
  M.valid = true;
  return 0;
}

int mesh_copy_out(MeshState &M, float *xyz, uint8_t *rgb, uint32_t *faces, cudaStream_t s, std::string &err) {
  if (M.n_vertices) {
    MCK(cudaMemcpyAsync(xyz, M.d_xyz, sizeof(float) * 3 * M.n_vertices, cudaMemcpyDeviceToHost, s));
    MCK(cudaMemcpyAsync(rgb, M.d_rgb, 3 * M.n_vertices, cudaMemcpyDeviceToHost, s));
  }
  if (M.n_faces) MCK(cudaMemcpyAsync(faces, M.d_faces, sizeof(uint32_t) * 3 * M.n_faces, cudaMemcpyDeviceToHost, s));
  MCK(cudaStreamSynchronize(s));
  return 0;
}

__global__ void k_export_cells(const Cell *cells, const CellOut *out, const uint64_t *vbase, const uint64_t *fbase,
                               uint32_t n, int32_t *rows, int64_t *ranges) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Cell c = cells[i];
  int32_t *r = rows + 14 * (size_t)i;
  r[0] = c.type;
  r[1] = c.quirk;
  r[2] = c.o[0];
  r[3] = c.o[1];
  r[4] = c.o[2];
  r[5] = c.size;
  for (int k = 0; k < 8; k++) r[6 + k] = (int32_t)c.L[k];
  int64_t *g = ranges + 4 * (size_t)i;
  g[0] = (int64_t)vbase[i];
  g[1] = out[i].nv;
  g[2] = (int64_t)fbase[i];
  g[3] = out[i].nf;
}

int mesh_copy_cells(MeshState &M, int32_t *rows, int64_t *ranges, cudaStream_t s, std::string &err) {
  if (!M.impl || !M.valid || !M.n_cells) return 0;
  MeshImpl &I = impl(M);
  const uint32_t n = (uint32_t)M.n_cells;
  int32_t *d_rows = nullptr;
  int64_t *d_ranges = nullptr;
  MCK(cudaMallocAsync((void **)&d_rows, sizeof(int32_t) * 14 * n, s));
  MCK(cudaMallocAsync((void **)&d_ranges, sizeof(int64_t) * 4 * n, s));
  // after an update the current cells, counts and bases are the "old" set
  note_launch();
  k_export_cells<<<(n + 255) / 256, 256, 0, s>>>(I.old_cells, I.old_out, I.old_vbase, I.old_fbase, n, d_rows,
                                                 d_ranges);
  MCK(cudaMemcpyAsync(rows, d_rows, sizeof(int32_t) * 14 * n, cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(ranges, d_ranges, sizeof(int64_t) * 4 * n, cudaMemcpyDeviceToHost, s));
  MCK(cudaFreeAsync(d_rows, s));
  MCK(cudaFreeAsync(d_ranges, s));
  MCK(cudaStreamSynchronize(s));
  return 0;
}

// ---------------------------------------------------------------------------
// Cell export without allocation
//
// For callers that must not allocate device memory during the call (a fixed
// memory budget, an allocator they do not control, code that runs where
// cudaMalloc is not allowed): the export kernel's staging area is this
// file-scope device array instead of stream-ordered allocations.  It is
// shared by every call in the process, on every handle.
// ---------------------------------------------------------------------------
constexpr uint32_t NOALLOC_MAX_CELLS = 65536;
constexpr size_t NOALLOC_RANGES_BYTES = sizeof(int64_t) * 4 * NOALLOC_MAX_CELLS;
constexpr size_t NOALLOC_ROWS_BYTES = sizeof(int32_t) * 14 * NOALLOC_MAX_CELLS;
static __device__ __align__(256) unsigned char g_export_scratch[NOALLOC_RANGES_BYTES + NOALLOC_ROWS_BYTES];

// The array's device address on the current device, looked up at every call
// with the map's device current (in host code the symbol names a host-side
// stand-in, never the device memory itself).  The lookup is cheap, and a
// cached address would go stale with a new primary context (after
// cudaDeviceReset, say).
static cudaError_t export_scratch_address(unsigned char **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_export_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned char *>(p);
  return cudaSuccess;
}

int mesh_copy_cells_noalloc(MeshState &M, int32_t *rows, int64_t *ranges, cudaStream_t s, std::string &err) {
  if (!M.impl || !M.valid || !M.n_cells) return 0;
  const uint32_t n = (uint32_t)M.n_cells;
  if (n > NOALLOC_MAX_CELLS) {
    err = "ff_get_mesh_cells_noalloc: the mesh has " + std::to_string(n) + " cells, more than the " +
          std::to_string(NOALLOC_MAX_CELLS) + " its fixed device buffer holds (use ff_get_mesh_cells)";
    return 1;  // FF_ERR_BAD_ARG
  }
  unsigned char *base = nullptr;
  MCK(export_scratch_address(&base));
  // every word copied back is written by this call's kernel first, so the
  // previous call's contents need no clearing
  int64_t *d_ranges = reinterpret_cast<int64_t *>(base);
  int32_t *d_rows = reinterpret_cast<int32_t *>(base + NOALLOC_RANGES_BYTES);
  MeshImpl &I = impl(M);
  note_launch();
  k_export_cells<<<(n + 255) / 256, 256, 0, s>>>(I.old_cells, I.old_out, I.old_vbase, I.old_fbase, n, d_rows,
                                                 d_ranges);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(rows, d_rows, sizeof(int32_t) * 14 * n, cudaMemcpyDeviceToHost, s));
  MCK(cudaMemcpyAsync(ranges, d_ranges, sizeof(int64_t) * 4 * n, cudaMemcpyDeviceToHost, s));
  MCK(cudaStreamSynchronize(s));
  return 0;
}

void mesh_free(MeshState &M) {
  if (M.impl) {
    MeshImpl &I = impl(M);
    void *ptrs[] = {I.cellq[0], I.cellq[1], I.faceq[0], I.faceq[1], I.edgeq[0], I.edgeq[1], I.vertq[0],
                    I.vertq[1], I.d_count, I.raw, I.cells, I.old_cells, I.keys, I.keys_sorted, I.old_keys,
                    I.vals, I.vals_sorted, I.sort_tmp, I.out, I.old_out, I.nv, I.nf, I.vbase, I.fbase,
                    I.old_vbase, I.old_fbase, I.dirty, I.old_index, I.scan_tmp, I.old_xyz, I.old_rgb,
                    I.old_faces, I.dlist, I.cases, I.keep, I.keep_tiles, I.mkeys, I.top_cellq, I.top_faceq,
                    I.top_edgeq, I.top_vertq, I.d_top_count};
    for (void *p : ptrs)
      if (p) cudaFreeAsync(p, 0);
    if (I.h_count) cudaFreeHost(I.h_count);
    if (I.h_top_count) cudaFreeHost(I.h_top_count);
    delete &I;
    M.impl = nullptr;
  }
  if (M.d_xyz) cudaFreeAsync(M.d_xyz, 0);
  if (M.d_rgb) cudaFreeAsync(M.d_rgb, 0);
  if (M.d_faces) cudaFreeAsync(M.d_faces, 0);
  cudaStreamSynchronize(0);
  M.d_xyz = nullptr;
  M.d_rgb = nullptr;
  M.d_faces = nullptr;
}

void mesh_next_outputs(MeshState &M, const void **xyz, const void **rgb, const void **faces) {
  if (!M.impl) {
    *xyz = *rgb = *faces = nullptr;
    return;
  }
  MeshImpl &I = impl(M);
  *xyz = I.old_xyz;
  *rgb = I.old_rgb;
  *faces = I.old_faces;
}

void mesh_invalidate(MeshState &M) {
  M.valid = false;
  if (M.impl) {
    impl(M).n_old = 0;
    impl(M).top_valid = false;
  }
}

void mesh_note_frame(MeshState &) {}

cudaError_t prewarm_mesh_kernels() {
  const void *fns[] = {(const void *)k_gen_levels,         (const void *)k_cell_keys,
                       (const void *)k_gather_cells,       (const void *)k_mesh_lattice<false>,
                       (const void *)k_mesh_lattice<true>, (const void *)k_mesh_corner<false>,
                       (const void *)k_mesh_corner<true>,  (const void *)k_mark_dirty,
                       (const void *)k_count_tile_sums,    (const void *)k_copy_clean,
                       (const void *)k_count_tile_scan,    (const void *)k_count_tile_apply,
                       (const void *)k_fill_counts_from_old, (const void *)k_export_cells,
                       (const void *)k_keep_cells,         (const void *)k_keep_tile_scan,
                       (const void *)k_keep_apply,         (const void *)k_merge_cells,
                       (const void *)k_load_top};
  for (const void *f : fns) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return prewarm_sort_kernels();
}

}  // namespace ffb
