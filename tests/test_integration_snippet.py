"""The reference-side binding of the boundary,
compiled and checked on the host.  The flattening function between the
`flatten:begin` / `flatten:end` markers is written out verbatim, compiled
against the reference's own OctreeForest / FacePairList headers (the oracle's
host stand-in for their p4est-backed parts, oracle/shim/forest_shim.cpp), and
run on the lists of the library's forest builder (include/octlb_forest.h)
injected as the reference's SameLevelFace / CoarseFineFace / TreeBoundaryFace
records: the octlb_tables arrays it fills must equal the builder's lists --
the field mapping of every record (FaceDir numbering, the four fine slots,
the bounds order) agrees with what octlb_gpu_create reads.  Forests: a
three-level channel with a refined cylinder region, and the two-level
cavity."""
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#include "flatten.hpp"
#include "octlb_forest.h"

namespace octlb {
void OracleForestInject(OctreeForest& forest, const std::vector<int>& levels, const std::vector<BoundingBox>& bounds,
                        const std::vector<SameLevelFace>& sl, const std::vector<CoarseFineFace>& cf,
                        const std::vector<TreeBoundaryFace>& tb);
}

static int check(const char* what, const std::vector<int>& a, const int* b, size_t nb) {
  if (a.size() != nb) { std::printf("%s: %zu vs %zu\n", what, a.size(), nb); return 1; }
  for (size_t k = 0; k < nb; ++k)
    if (a[k] != b[k]) { std::printf("%s[%zu]: %d vs %d\n", what, k, a[k], b[k]); return 1; }
  return 0;
}
static int check(const char* what, const std::vector<double>& a, const double* b, size_t nb) {
  if (a.size() != nb) { std::printf("%s: %zu vs %zu\n", what, a.size(), nb); return 1; }
  for (size_t k = 0; k < nb; ++k)
    if (a[k] != b[k]) { std::printf("%s[%zu]: %g vs %g\n", what, k, a[k], b[k]); return 1; }
  return 0;
}

static int run(octlb_forest* f, int n) {
  using namespace octlb;
  const int nl = octlb_forest_build(f);
  std::vector<int> lv(nl), sl(3 * octlb_forest_num_same_level(f)), cf(8 * octlb_forest_num_coarse_fine(f)),
      tb(2 * octlb_forest_num_tree_boundary(f));
  std::vector<double> bd(6 * nl), cfb(30 * octlb_forest_num_coarse_fine(f));
  octlb_forest_leaves(f, lv.data(), bd.data());
  octlb_forest_same_level(f, sl.data());
  octlb_forest_coarse_fine(f, cf.data(), cfb.data());
  octlb_forest_tree_boundary(f, tb.data());
  // the builder's lists as the reference's records
  std::vector<BoundingBox> bx;
  for (int i = 0; i < nl; ++i)
    bx.push_back({bd[6 * i], bd[6 * i + 1], bd[6 * i + 2], bd[6 * i + 3], bd[6 * i + 4], bd[6 * i + 5]});
  std::vector<SameLevelFace> slv;
  for (size_t k = 0; k < sl.size(); k += 3) slv.push_back({sl[k], FaceDir(sl[k + 1]), sl[k + 2], 0, 0});
  std::vector<CoarseFineFace> cfv;
  for (size_t k = 0; k < cf.size() / 8; ++k) {
    CoarseFineFace c{};
    c.coarse_id = cf[8 * k];
    for (int s = 0; s < 4; ++s) c.fine_ids[s] = cf[8 * k + 1 + s];
    c.normal = FaceDir(cf[8 * k + 5]);
    c.coarse_level = cf[8 * k + 6];
    c.fine_level = cf[8 * k + 7];
    const double* b = &cfb[30 * k];
    c.coarse_bounds = {b[0], b[1], b[2], b[3], b[4], b[5]};
    for (int s = 0; s < 4; ++s)
      c.fine_bounds[s] = {b[6 + 6 * s], b[7 + 6 * s], b[8 + 6 * s], b[9 + 6 * s], b[10 + 6 * s], b[11 + 6 * s]};
    cfv.push_back(c);
  }
  std::vector<TreeBoundaryFace> tbv;
  for (size_t k = 0; k < tb.size(); k += 2) tbv.push_back({tb[k], FaceDir(tb[k + 1])});
  OctreeForest forest(MPI_COMM_WORLD, BoundingBox{0, 0, 0, 1, 1, 1}, 1, 1, 1);
  OracleForestInject(forest, lv, bx, slv, cfv, tbv);
  const FacePairList pairs(forest);
  std::vector<uint8_t> kinds(static_cast<size_t>(nl) * n * n * n, 0);
  FlatTables flat;
  FlattenForest(forest, pairs, n, kinds.data(), flat);
  const octlb_tables& t = flat.t;
  int bad = 0;
  bad |= t.n != n || t.n_blocks != nl || t.kinds != kinds.data();
  bad |= check("levels", flat.levels, lv.data(), lv.size());
  bad |= check("bounds", flat.bounds, bd.data(), bd.size());
  bad |= check("same_level", flat.same_level, sl.data(), sl.size());
  bad |= check("coarse_fine", flat.coarse_fine, cf.data(), cf.size());
  bad |= check("coarse_fine_bounds", flat.coarse_fine_bounds, cfb.data(), cfb.size());
  bad |= check("tree_boundary", flat.tree_boundary, tb.data(), tb.size());
  bad |= t.n_same_level * 3 != int(sl.size()) || t.n_coarse_fine * 8 != int(cf.size()) ||
         t.n_tree_boundary * 2 != int(tb.size()) || t.tree_boundary_spec == nullptr;
  std::printf("leaves %d same-level %zu coarse-fine %zu tree-boundary %zu: %s\n", nl, sl.size() / 3, cf.size() / 8,
              tb.size() / 2, bad ? "MISMATCH" : "ok");
  octlb_forest_free(f);
  return bad;
}

int main() {
  const double channel[6] = {0, 0, 0, 4, 1, 1}, unit[6] = {0, 0, 0, 1, 1, 1};
  octlb_forest* a = octlb_forest_new(4, 1, 1, 0, 0, 1, channel);
  octlb_forest_refine_uniform(a, 1);
  const double near1[6] = {0.5, 0.25, 0, 1.5, 0.75, 1}, near2[6] = {0.75, 0.375, 0, 1.25, 0.625, 1};
  octlb_forest_refine_box(a, near1, 2);
  octlb_forest_refine_box(a, near2, 3);
  octlb_forest_balance(a);
  octlb_forest* b = octlb_forest_new(1, 1, 1, 0, 0, 0, unit);
  octlb_forest_refine_uniform(b, 3);
  const double band[6] = {0, 0.875, 0, 1, 1, 1};
  octlb_forest_refine_box(b, band, 4);
  octlb_forest_balance(b);
  return run(a, 8) | run(b, 8);
}
'''


def reference_tree():
    sys.path.insert(0, ROOT)
    import __graft_entry__
    tree = os.environ.get("OCTLB_REFERENCE", __graft_entry__.REFERENCE_TREE)
    return tree if os.path.isdir(os.path.join(tree, "src", "mesh", "topology")) else None


def test_flattening_snippet_compiles_and_matches_the_forest_builder(ob, tmp_path):
    ref = reference_tree()
    if ref is None:
        pytest.skip("the reference sources are not mounted")
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"<!-- flatten:begin -->\s*```cpp\n(.*?)```\s*<!-- flatten:end -->", doc, re.S)
    assert m, "INTEGRATION.md has no flatten block"
    (tmp_path / "flatten.hpp").write_text("#pragma once\n" + m.group(1))
    (tmp_path / "main.cpp").write_text(HARNESS)
    exe = tmp_path / "snippet"
    lib_dir = os.path.join(ROOT, "octlb_b200")
    cmd = ["g++", "-std=c++20", "-O1", "-I", str(tmp_path), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "oracle", "shim"), "-I", ref, "-I", os.path.join(ref, "src", "solver", "lbm"),
           str(tmp_path / "main.cpp"), os.path.join(ROOT, "oracle", "shim", "forest_shim.cpp"),
           "-o", str(exe), "-L", lib_dir, "-loctlb_b200", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 2
