/* octlb_forest.h -- host forest builder and flattener (C ABI).
 *
 * p4est owns the mesh in the reference (src/mesh/forest/octree_forest.cpp,
 * src/mesh/topology/face_pair_list.cpp).  p4est is not part of this build, so
 * this module provides the same contract for the forests the hot path runs
 * on: a brick of root trees (optionally periodic), recursive refinement by
 * level or by box, 2:1 face balance, and the flattened FacePairList lists
 * that octlb_gpu_create consumes:
 *   same-level faces   one entry per direction of every same-level pair
 *                      (FaceCallback, face_pair_list.cpp:207-270)
 *   coarse-fine faces  one entry per hanging face, coarse side's face as the
 *                      normal, the four fine leaves in Morton order, bounds
 *                      of both sides (face_pair_list.cpp:272-335)
 *   tree boundary      one entry per outer leaf face (face_pair_list.cpp:179-200)
 * Leaves are numbered in Morton order inside each tree, trees x-fastest.
 * Coarse-fine faces are listed grouped by coarse level.
 * A caller that owns a real p4est forest can skip this module and fill
 * octlb_tables from its FacePairList directly. */
#ifndef OCTLB_FOREST_H_
#define OCTLB_FOREST_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct octlb_forest octlb_forest;

/* Brick of bx*by*bz unit trees mapped onto domain {xmin,ymin,zmin,xmax,ymax,zmax};
 * px/py/pz = 1 makes that axis periodic (p8est_connectivity_new_brick). */
octlb_forest* octlb_forest_new(int bx, int by, int bz, int px, int py, int pz,
                               const double domain[6]);
void octlb_forest_free(octlb_forest* f);
/* Refine every leaf coarser than `level` until it reaches `level`. */
int octlb_forest_refine_uniform(octlb_forest* f, int level);
/* Refine, recursively up to `level`, every leaf whose box overlaps `box`
 * with positive volume (OctreeForest::refine with a bounds criterion). */
int octlb_forest_refine_box(octlb_forest* f, const double box[6], int level);
/* 2:1 balance across faces (p8est_balance, P8EST_CONNECT_FACE). */
int octlb_forest_balance(octlb_forest* f);
/* Order the leaves and build the face lists.  Returns the leaf count. */
int octlb_forest_build(octlb_forest* f);

int octlb_forest_num_leaves(const octlb_forest* f);
/* levels[n], bounds[n][6] */
int octlb_forest_leaves(const octlb_forest* f, int* levels, double* bounds);
int octlb_forest_num_same_level(const octlb_forest* f);
int octlb_forest_same_level(const octlb_forest* f, int* out /* [n][3] */);
int octlb_forest_num_coarse_fine(const octlb_forest* f);
int octlb_forest_coarse_fine(const octlb_forest* f, int* out /* [n][8] */, double* bounds /* [n][30] */);
int octlb_forest_num_tree_boundary(const octlb_forest* f);
int octlb_forest_tree_boundary(const octlb_forest* f, int* out /* [n][2] */);

#ifdef __cplusplus
}
#endif
#endif
