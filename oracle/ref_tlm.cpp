// Tangent-linear FP64 build of the reference path.  TEST INFRASTRUCTURE ONLY:
// the checker of the GPU adjoint; the product never links it.
//
// The reference's own hot-path sources (BlockLattice, LevelCoupler,
// BouzidiLinkData, GhostSchedule, TimeLoop, MomentumExchangeDrag) and the
// restated pieces of ref_capi.cpp are compiled here with their floating type
// replaced by octlb_tlm::Dual (oracle/tlm_dual.h): a value and kDirs
// directional derivatives.  Running the reference's TimeLoop on duals is
// forward-mode differentiation of the reference itself: the value part is the
// reference's trajectory and each derivative part the tangent-linear model
// along one seeded parameter direction.
//
// Seeds (tlm_set_seeds, before ref_sim_new): a derivative of omega per
// direction (d omega / d tau = -omega^2 for tau) and a relative derivative of
// every tree-boundary wall velocity (1 / u_max for the inlet velocity scale);
// tlm_sim_set_body_force seeds the body force along given directions.
// tlm_sim_drag returns the momentum-exchange force with its derivatives.
//
// Every standard header (and the vendored OpenLB scalar helpers, which spell
// `long double`) is included before the replacement so that only the
// reference and oracle sources see it.
#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <optional>
#include <ostream>
#include <set>
#include <source_location>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <typeindex>
#include <unordered_set>
#include <utility>
#include <variant>
#include <vector>

#include "tlm_dual.h"

// The vendored OpenLB scalar helpers spell `long double` overloads: they are
// compiled with the plain floating type and serve the dual through their
// generic templates.
#include "core/platform/platform.h"
#include "core/baseType.h"
#include "utilities/omath.h"
#include "utilities/aDiff.h"

using f64 = double;
namespace {
double g_omega_seed[octlb_tlm::kDirs] = {};
double g_wall_seed[octlb_tlm::kDirs] = {};
}  // namespace
inline f64 to_f64(const octlb_tlm::Dual& x) { return x.v; }
inline octlb_tlm::Dual seed_omega(f64 omega) {
  octlb_tlm::Dual r(omega);
  for (int k = 0; k < octlb_tlm::kDirs; ++k) r.d[k] = g_omega_seed[k];
  return r;
}
inline octlb_tlm::Dual seed_wall(f64 u) {
  octlb_tlm::Dual r(u);
  for (int k = 0; k < octlb_tlm::kDirs; ++k) r.d[k] = u * g_wall_seed[k];
  return r;
}

#define OCTLB_REF_TLM 1
#define double octlb_tlm::Dual

#include "src/solver/lbm/block_lattice.cpp"
#include "src/solver/lbm/level_coupler.cpp"
#include "src/solver/lbm/bouzidi_link_data.cpp"
#include "src/mesh/geometry/material_field.cpp"
#include "src/mesh/geometry/triangle_soup.cpp"
#include "shim/forest_shim.cpp"
#include "ref_capi.cpp"

#undef double

extern "C" {

int tlm_dirs() { return octlb_tlm::kDirs; }

// Seeds for the next ref_sim_new: omega_seed[k] = d omega along direction k;
// wall_seed[k] = d u_w / u_w along direction k for every wall velocity.
void tlm_set_seeds(const double* omega_seed, const double* wall_seed) {
  for (int k = 0; k < octlb_tlm::kDirs; ++k) {
    g_omega_seed[k] = omega_seed ? omega_seed[k] : 0.0;
    g_wall_seed[k] = wall_seed ? wall_seed[k] : 0.0;
  }
}

// Body force F [oct][n^3][3] (null = zero) with derivative dirs[k] along
// direction k ([kDirs][oct][n^3][3]; null rows = 0).
void tlm_sim_set_body_force(void* h, const double* force, const double* dirs, int ndirs) {
  auto* s = static_cast<Sim*>(h);
  const std::size_t m = static_cast<std::size_t>(s->blocks->size()) * s->n * s->n * s->n * 3;
  std::vector<octlb_tlm::Dual> f(m);
  for (std::size_t c = 0; c < m; ++c) {
    f[c].v = force ? force[c] : 0.0;
    for (int k = 0; k < ndirs && k < octlb_tlm::kDirs; ++k) f[c].d[k] = dirs[static_cast<std::size_t>(k) * m + c];
  }
  static_cast<RestatedBoundary*>(s->bc.get())->set_force(s->loop.get(), f.data());
}

// Momentum-exchange force (as ref_sim_drag) and its derivatives:
// out[3], dout[3][kDirs].
void tlm_sim_drag(void* h, const uint8_t* mask, double* out, double* dout) {
  const std::array<octlb_tlm::Dual, 3> f = SimDrag(static_cast<Sim*>(h), mask);
  for (int a = 0; a < 3; ++a) {
    out[a] = f[a].v;
    for (int k = 0; k < octlb_tlm::kDirs; ++k) dout[a * octlb_tlm::kDirs + k] = f[a].d[k];
  }
}

}  // extern "C"
