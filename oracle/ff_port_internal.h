/* Internal interface between the traversal/update restatement (ff_port.c) and
 * the meshing restatement (ff_port_mesh.c).  ORACLE INFRASTRUCTURE ONLY. */
#ifndef FF_PORT_INTERNAL_H
#define FF_PORT_INTERNAL_H
#include <stdint.h>

typedef struct {
  int type;  /* 0 interior, 1-3 wall x/y/z, 4-6 edge x/y/z, 7 corner */
  int quirk; /* always 0; kept so that rows keep their layout */
  int o[3];
  int size;
  uint32_t L[8]; /* lastLeaf of each side */
} ffp_cell;

typedef struct {
  const uint16_t *pos; /* 3 per leaf */
  const uint16_t *scale_of;
  const uint32_t *parent;
  const float *dist, *wgt;
  const uint16_t *col; /* 3 per voxel */
  uint32_t leaves_used;
  float offset[3];
  float scale;
} ffp_mesh_src;

typedef struct {
  float *xyz;
  uint8_t *rgb;
  uint32_t *faces;
  int64_t nv, nf;
  int64_t *cell_v; /* per cell: first vertex, vertex count, first face, face count */
} ffp_mesh_result;

int64_t ffp_enumerate_cells(const uint32_t *tree, uint32_t n, uint32_t leaves_total, ffp_cell **out);
void ffp_mesh_cells(const ffp_mesh_src *m, const ffp_cell *cells, int64_t ncell, ffp_mesh_result *res);
extern const unsigned long long ffp_mc_tri[256];
#endif
