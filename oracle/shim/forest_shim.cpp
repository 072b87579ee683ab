// Host stand-in for the two p4est-backed classes the reference's hot path
// needs (OctreeForest, FacePairList), used ONLY to link the reference's own
// lattice / coupler / time-loop code into the test oracle (oracle/_ref).
//
// The forest is not built here: a caller injects the leaves (level, bounds)
// and the face lists that p4est's iterate pass would have produced
// (src/mesh/topology/face_pair_list.cpp:176-390 emits one SameLevelFace per
// direction of a same-rank pair, one CoarseFineFace per hanging face, and one
// TreeBoundaryFace per outer face).  The same flattened lists feed the GPU
// path, so both sides see identical topology.
//
// Test infrastructure: nothing in the product links this file.
#include <stdexcept>
#include <vector>

#include "src/mesh/forest/octree_forest.h"
#include "src/mesh/topology/face_pair_list.h"

namespace octlb {

struct OctreeForest::Impl {
  MPI_Comm comm = MPI_COMM_WORLD;
  BoundingBox domain{};
  std::vector<int> levels;
  std::vector<BoundingBox> bounds;
  std::vector<SameLevelFace> same_level;
  std::vector<CoarseFineFace> coarse_fine;
  std::vector<TreeBoundaryFace> tree_boundary;
};

// Befriended by OctreeForest (octree_forest.h:16); gives the shim access to
// the injected data.
struct MeshForestAccess {
  static void CopyFaces(const OctreeForest& f, std::vector<SameLevelFace>* sl,
                        std::vector<CoarseFineFace>* cf,
                        std::vector<TreeBoundaryFace>* tb) {
    *sl = f.impl_->same_level;
    *cf = f.impl_->coarse_fine;
    *tb = f.impl_->tree_boundary;
  }
  static void Inject(OctreeForest& f, const std::vector<int>& levels,
                     const std::vector<BoundingBox>& bounds,
                     const std::vector<SameLevelFace>& sl,
                     const std::vector<CoarseFineFace>& cf,
                     const std::vector<TreeBoundaryFace>& tb) {
    f.impl_->levels = levels;
    f.impl_->bounds = bounds;
    f.impl_->same_level = sl;
    f.impl_->coarse_fine = cf;
    f.impl_->tree_boundary = tb;
  }
};

OctreeForest::OctreeForest(MPI_Comm comm, BoundingBox domain, int, int, int)
    : impl_(std::make_unique<Impl>()) {
  impl_->comm = comm;
  impl_->domain = domain;
}
OctreeForest::~OctreeForest() = default;
OctreeForest::OctreeForest(OctreeForest&&) noexcept = default;
OctreeForest& OctreeForest::operator=(OctreeForest&&) noexcept = default;

void OctreeForest::refine(std::function<bool(OctantId)>, int) {
  throw std::logic_error("oracle forest shim: refine is not available");
}
void OctreeForest::refine(std::function<bool(const BoundingBox&, int)>, int) {
  throw std::logic_error("oracle forest shim: refine is not available");
}
void OctreeForest::balance() {}
void OctreeForest::partition(std::function<int(OctantId)>) {}
void OctreeForest::RebuildGhost() {}
void OctreeForest::RebuildGhostLayer(Impl*) {}
MPI_Comm OctreeForest::comm() const { return impl_->comm; }

label OctreeForest::local_num_octants() const {
  return static_cast<label>(impl_->levels.size());
}
BoundingBox OctreeForest::quadrant_bounds(OctantId id) const {
  if (id < 0 || id >= local_num_octants()) throw std::out_of_range("OctantId");
  return impl_->bounds[static_cast<std::size_t>(id)];
}
int OctreeForest::quadrant_level(OctantId id) const {
  if (id < 0 || id >= local_num_octants()) throw std::out_of_range("OctantId");
  return impl_->levels[static_cast<std::size_t>(id)];
}

FacePairList::FacePairList(const OctreeForest& forest) { rebuild(forest); }

void FacePairList::rebuild(const OctreeForest& forest) {
  MeshForestAccess::CopyFaces(forest, &same_level_, &coarse_fine_, &tree_boundary_);
  cross_rank_edges_.clear();
}
const std::vector<SameLevelFace>& FacePairList::same_level_faces() const { return same_level_; }
const std::vector<CoarseFineFace>& FacePairList::coarse_fine_faces() const { return coarse_fine_; }
const std::vector<TreeBoundaryFace>& FacePairList::tree_boundary_faces() const { return tree_boundary_; }
const std::vector<CrossRankEdge>& FacePairList::cross_rank_edges() const { return cross_rank_edges_; }

// Injection entry used by the oracle C API (ref_capi.cpp).
void OracleForestInject(OctreeForest& forest, const std::vector<int>& levels,
                        const std::vector<BoundingBox>& bounds,
                        const std::vector<SameLevelFace>& sl,
                        const std::vector<CoarseFineFace>& cf,
                        const std::vector<TreeBoundaryFace>& tb) {
  MeshForestAccess::Inject(forest, levels, bounds, sl, cf, tb);
}

}  // namespace octlb
