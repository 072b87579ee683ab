// octlb_gpu_time_loop.hpp -- header-only C++ adapter over the C ABI with the
// reference TimeLoop's method names (src/solver/lbm/time_loop/time_loop.h:47-121)
// so a case driver (examples/cavity3d, examples/cylinder3d) can swap its
// TimeLoop for the GPU context with the same calls:
//
//   TimeLoop loop(forest, blocks, ghosts, coupler, domain_bc, omega);   // reference
//   octlb::GpuTimeLoop loop(tables, params, init_pops);                 // this path
//   loop.set_snapshot_post_collide(true);
//   loop.advance_one();
//   loop.counters();  loop.max_level();
//   auto f = loop.force_on_fluid();     // MomentumExchangeDrag::force_on_fluid_if
//   octlb::GpuTimeLoop cav(tables, params, init_pops, true);   // use_const_rho_bgk
//   cav.average_rho();                  // TimeLoop::average_rho
//
// cavity3d's TimeLoop around a ConcreteDomainBoundaryHandler
// (cavity3d_case.h:148-197) takes the handler's face specs:
//
//   octlb::GpuDomainBc bc;              // CavityBoundarySpecs
//   for (int f = 0; f < 6; ++f) bc.types[f] = OCTLB_FD_VELOCITY;
//   bc.u_wall[3 * 3 + 0] = u_lid;       // y+ face
//   octlb::GpuTimeLoop cav(tables, params, nullptr, true, &bc);
//   loop.write_vtk("out", "cylinder3d", it);   // AmrVtkWriter::WriteTimestep + WriteVtmAndPvd
//
// Errors surface as std::runtime_error, the reference's convention
// (block_lattice.cpp:35-36, level_coupler.cpp:72-74).
#ifndef OCTLB_GPU_TIME_LOOP_HPP_
#define OCTLB_GPU_TIME_LOOP_HPP_

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "octlb_gpu.h"

namespace octlb {

// The DomainBcSpec list of a ConcreteDomainBoundaryHandler, one entry per
// face in FaceDir order (x-, x+, y-, y+, z-, z+): type (OCTLB_FD_*), wall
// velocity, target density, inlet field.
struct GpuDomainBc {
  int types[6] = {OCTLB_FD_NO_SLIP, OCTLB_FD_NO_SLIP, OCTLB_FD_NO_SLIP,
                  OCTLB_FD_NO_SLIP, OCTLB_FD_NO_SLIP, OCTLB_FD_NO_SLIP};
  double u_wall[18] = {};
  double rho_target[6] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
  octlb_fd_inlet inlets[6] = {};
};

struct GpuTimeLoopCounters {
  std::vector<int> collide;
  std::vector<int> stream;
};

class GpuTimeLoop {
 public:
  // use_const_rho_bgk: the TimeLoop constructor argument (time_loop.h:47-54).
  // domain_bc: the finite-difference domain conditions of a
  // ConcreteDomainBoundaryHandler; the face cells of the tables' kinds are
  // stamped with the faces' kinds first (bc::StampTreeBoundaryCells).
  GpuTimeLoop(const octlb_tables& tables, const octlb_params& params,
              const double* init_pops = nullptr, bool use_const_rho_bgk = false,
              const GpuDomainBc* domain_bc = nullptr) {
    octlb_tables t = tables;
    std::vector<uint8_t> kinds;
    int rc = OCTLB_OK;
    if (domain_bc) {
      kinds.resize(static_cast<size_t>(tables.n_blocks) * tables.n * tables.n * tables.n);
      rc = octlb_fd_stamp_kinds(&tables, domain_bc->types, kinds.data());
      t.kinds = kinds.data();
    }
    if (rc == OCTLB_OK) rc = octlb_gpu_create(&t, &params, init_pops, &ctx_);
    if (rc == OCTLB_OK && use_const_rho_bgk) rc = octlb_gpu_set_const_rho(ctx_, 1);
    if (rc == OCTLB_OK && domain_bc)
      rc = octlb_gpu_set_fd_boundary_inlets(ctx_, domain_bc->types, domain_bc->u_wall, domain_bc->rho_target,
                                            domain_bc->inlets);
    if (rc != OCTLB_OK) {
      const std::string msg = ctx_ ? octlb_gpu_last_error(ctx_) : "invalid tables or face specs";
      octlb_gpu_destroy(ctx_);
      ctx_ = nullptr;
      throw std::runtime_error("GpuTimeLoop: " + msg);
    }
  }
  ~GpuTimeLoop() { octlb_gpu_destroy(ctx_); }
  GpuTimeLoop(const GpuTimeLoop&) = delete;
  GpuTimeLoop& operator=(const GpuTimeLoop&) = delete;

  void advance_one() { check(octlb_gpu_advance(ctx_, 1)); }
  void advance(int n) { check(octlb_gpu_advance(ctx_, n)); }
  void synchronize() { check(octlb_gpu_synchronize(ctx_)); }

  int max_level() const { return octlb_gpu_max_level(ctx_); }
  GpuTimeLoopCounters counters() const {
    GpuTimeLoopCounters c;
    c.collide.assign(32, 0);
    c.stream.assign(32, 0);
    const int n = octlb_gpu_counters(ctx_, c.collide.data(), c.stream.data(), 32);
    c.collide.resize(n > 0 ? n : 0);
    c.stream.resize(n > 0 ? n : 0);
    return c;
  }
  // The momentum exchange always reads the post-collide state the step
  // consumed, so the snapshot switch costs nothing and is kept for API parity.
  void set_snapshot_post_collide(bool on) { snapshot_ = on; }
  bool snapshot_post_collide() const { return snapshot_; }

  std::array<double, 3> force_on_fluid() {
    std::array<double, 3> f{};
    check(octlb_gpu_force(ctx_, f.data()));
    return f;
  }
  // Cd = 2 (-F . e) / (rho u^2 A)  (drag_postprocessor.h:159-165)
  double drag_coefficient(double rho, double u, double area, std::array<double, 3> flow_dir) {
    const auto f = force_on_fluid();
    const double fdot = f[0] * flow_dir[0] + f[1] * flow_dir[1] + f[2] * flow_dir[2];
    return 2.0 * (-fdot) / (rho * u * u * area);
  }
  double total_mass() {
    double a[4];
    check(octlb_gpu_audit(ctx_, a));
    return a[0];
  }
  // TimeLoop::average_rho() (time_loop.h:87-88): 1 without ConstRhoBGK
  double average_rho() {
    double a = 1.0;
    check(octlb_gpu_average_rho(ctx_, &a));
    return a;
  }
  // One .vts per block (base_r<rank>_oct<id>_T<step>.vts), the step's .vtm and
  // its .pvd entry, as AmrVtkWriter::WriteTimestep + WriteVtmAndPvd
  void write_vtk(const std::string& output_dir, const std::string& base_name, int step,
                 int fields = OCTLB_VTK_VELOCITY | OCTLB_VTK_PRESSURE, int rank = 0, bool write_index = true) {
    check(octlb_gpu_write_vtk(ctx_, output_dir.c_str(), base_name.c_str(), step, rank, fields, write_index ? 1 : 0));
  }
  octlb_ctx* handle() { return ctx_; }

 private:
  void check(int rc) const {
    if (rc != OCTLB_OK) throw std::runtime_error(std::string("GpuTimeLoop: ") + octlb_gpu_last_error(ctx_));
  }
  octlb_ctx* ctx_ = nullptr;
  bool snapshot_ = false;
};

}  // namespace octlb

#endif  // OCTLB_GPU_TIME_LOOP_HPP_
