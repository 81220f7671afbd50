// dmdgpu_reference.hpp -- the reference-side adapters over the C ABI of
// dmdgpu.h, for a maintainer of DMD to add to its C++ tree.
//
// Header-only C++20.  It includes the reference's own headers
// (force/force_component.h, sim/simulation_config.h, core/cell.h,
// core/error.h), so it compiles only with the reference's src/ directory on
// the include path; the library itself (libdmdgpu.so) has no C++ in its
// interface.
//
//   dmdgpu_ref::SystemView        SimulationConfig (src/sim/simulation_config.h:27-84)
//                                 -> dmdgpu_system, the term sets concatenated
//   dmdgpu_ref::GpuForceComponent ForceComponent (src/force/force_component.h:9-21)
//                                 over dmdgpu_component_compute: accumulates forces
//                                 and energy like every reference component
//   dmdgpu_ref::GpuSimulationEngine the run loop of SimulationEngine
//                                 (src/sim/simulation_engine.h:16-76) on the device
//
// Status codes 1..5 of the library are ForceError's values
// (src/core/error.h:6-12); the adapters rethrow them as ForceException.
#pragma once

#include <cstdint>
#include <span>
#include <string>
#include <utility>
#include <vector>

#include "core/cell.h"
#include "core/error.h"
#include "force/force_component.h"
#include "sim/simulation_config.h"
#include "dmdgpu.h"

namespace dmdgpu_ref {

inline ForceError force_error(int rc) {
    return static_cast<ForceError>((rc >= 1 && rc <= 5 ? rc : 5) - 1);
}

// SimulationConfig -> dmdgpu_system.  The reference keeps its bonded terms as
// vectors of parameter sets; the library takes one set per kind, so the sets
// are concatenated here (the view owns the concatenated arrays).
class SystemView {
  public:
    explicit SystemView(const SimulationConfig& cfg) {
        const auto n = static_cast<int32_t>(cfg.masses.size());
        s_.n_atoms = n;
        s_.box_size = cfg.box_size;
        s_.masses = cfg.masses.data();
        q_ = cfg.charges.empty() ? std::vector<double>(cfg.masses.size(), 0.0) : cfg.charges;
        s_.charges = q_.data();
        s_.pos_x = cfg.pos_x.data();
        s_.pos_y = cfg.pos_y.data();
        s_.pos_z = cfg.pos_z.data();
        if (!cfg.vel_x.empty()) {
            s_.vel_x = cfg.vel_x.data();
            s_.vel_y = cfg.vel_y.data();
            s_.vel_z = cfg.vel_z.data();
        }
        types_.assign(cfg.atom_types.begin(), cfg.atom_types.end());
        s_.atom_types = types_.empty() ? nullptr : types_.data();
        s_.use_lj = cfg.use_lj ? 1 : 0;
        s_.lj_n_types = static_cast<int32_t>(cfg.lj.n_types);
        s_.lj_sigma = cfg.lj.sigma.data();
        s_.lj_epsilon = cfg.lj.epsilon.data();
        s_.lj_cutoff = cfg.lj_cutoff;
        for (const auto& b : cfg.bonds) {
            append(bi_, b.i); append(bj_, b.j); append(bk_, b.k); append(br_, b.r0);
        }
        s_.n_bonds = static_cast<int32_t>(bi_.size());
        s_.bond_i = bi_.data(); s_.bond_j = bj_.data(); s_.bond_k = bk_.data(); s_.bond_r0 = br_.data();
        for (const auto& a : cfg.angles) {
            append(ai_, a.i); append(aj_, a.j); append(ak_, a.k); append(akt_, a.k_theta); append(at0_, a.theta0);
        }
        s_.n_angles = static_cast<int32_t>(ai_.size());
        s_.angle_i = ai_.data(); s_.angle_j = aj_.data(); s_.angle_k = ak_.data();
        s_.angle_k_theta = akt_.data(); s_.angle_theta0 = at0_.data();
        for (const auto& d : cfg.dihedrals) {
            append(di_, d.i); append(dj_, d.j); append(dk_, d.k); append(dl_, d.l);
            append(dn_, d.periodicity); append(dkp_, d.k_phi); append(dp0_, d.phi0);
        }
        s_.n_dihedrals = static_cast<int32_t>(di_.size());
        s_.dihedral_i = di_.data(); s_.dihedral_j = dj_.data(); s_.dihedral_k = dk_.data();
        s_.dihedral_l = dl_.data(); s_.dihedral_periodicity = dn_.data();
        s_.dihedral_k_phi = dkp_.data(); s_.dihedral_phi0 = dp0_.data();
        for (const auto& m : cfg.impropers) {
            append(ii_, m.i); append(ij_, m.j); append(ik_, m.k); append(il_, m.l);
            append(ikp_, m.k_phi); append(ip0_, m.phi0);
        }
        s_.n_impropers = static_cast<int32_t>(ii_.size());
        s_.improper_i = ii_.data(); s_.improper_j = ij_.data(); s_.improper_k = ik_.data();
        s_.improper_l = il_.data(); s_.improper_k_phi = ikp_.data(); s_.improper_phi0 = ip0_.data();
        s_.coulomb_type = cfg.coulomb_type == "pme" ? DMDGPU_COULOMB_PME : DMDGPU_COULOMB_CUTOFF;
        s_.coulomb_cutoff = cfg.coulomb_cutoff;
        s_.ewald_coeff = cfg.ewald_coeff;
        s_.pme_grid_spacing = cfg.pme_grid_spacing;
        s_.pme_order = cfg.pme_order;
        ei_.assign(cfg.excl_i.begin(), cfg.excl_i.end());
        ej_.assign(cfg.excl_j.begin(), cfg.excl_j.end());
        s_.n_excl = static_cast<int32_t>(ei_.size());
        s_.excl_i = ei_.data();
        s_.excl_j = ej_.data();
        s_.dt = cfg.dt;
        s_.n_steps = cfg.n_steps;
        s_.gen_vel = cfg.gen_vel ? 1 : 0;
        s_.seed = cfg.seed;
        s_.init_temperature = cfg.init_temperature;
        s_.thermostat_type = code(cfg.thermostat.type, {"none", "berendsen", "nose-hoover", "andersen"});
        s_.thermo_temperature = cfg.thermostat.temperature;
        s_.thermo_tau = cfg.thermostat.tau;
        s_.thermo_frequency = cfg.thermostat.frequency;
        s_.barostat_type = code(cfg.barostat.type, {"none", "berendsen", "andersen"});
        s_.baro_pressure = cfg.barostat.pressure;
        s_.baro_tau = cfg.barostat.tau;
        s_.baro_compressibility = cfg.barostat.compressibility;
        s_.checkpoint_interval = cfg.checkpoint_interval;
        s_.checkpoint_path = cfg.checkpoint_path.c_str();
        if (cfg.constraint_type == "shake" && !cfg.constraint_i.empty()) {
            ci_.assign(cfg.constraint_i.begin(), cfg.constraint_i.end());
            cj_.assign(cfg.constraint_j.begin(), cfg.constraint_j.end());
            s_.constraint_type = 1;
            s_.n_constraints = static_cast<int32_t>(ci_.size());
            s_.constraint_i = ci_.data();
            s_.constraint_j = cj_.data();
            s_.constraint_dist = cfg.constraint_dist.data();
            s_.constraint_tolerance = cfg.constraint_tolerance;
        }
    }
    SystemView(const SystemView&) = delete;
    SystemView& operator=(const SystemView&) = delete;
    const dmdgpu_system* get() const { return &s_; }

  private:
    template <typename T, typename U>
    static void append(std::vector<T>& dst, const std::vector<U>& src) {
        dst.insert(dst.end(), src.begin(), src.end());
    }
    static int32_t code(const std::string& v, std::initializer_list<const char*> names) {
        int32_t k = 0;
        for (const char* nm : names) {
            if (v == nm) return k;
            ++k;
        }
        throw ForceException(ForceError::ParmError, "dmdgpu", "unknown type '" + v + "'");
    }
    dmdgpu_system s_{};
    std::vector<double> q_;
    std::vector<int32_t> types_, bi_, bj_, ai_, aj_, ak_, di_, dj_, dk_, dl_, dn_, ii_, ij_, ik_, il_,
        ei_, ej_, ci_, cj_;
    std::vector<double> bk_, br_, akt_, at0_, dkp_, dp0_, ikp_, ip0_;
};

// One context per adapter; options: DMDGPU_PROFILE_*, DMDGPU_PRECISION_*.
inline dmdgpu_ctx* open_context(const SimulationConfig& cfg, int profile, int precision, int device = 0) {
    SystemView v(cfg);
    dmdgpu_options o{};
    o.profile = profile;
    o.precision = precision;
    o.skin = 0.1;
    o.device = device;
    o.rng_seed = 0x5EED;
    o.nb_form = DMDGPU_NB_AUTO;
    dmdgpu_ctx* ctx = nullptr;
    const int rc = dmdgpu_create(v.get(), &o, &ctx);
    if (rc) {
        std::string msg = ctx ? dmdgpu_last_error(ctx) : "dmdgpu_create failed";
        dmdgpu_destroy(ctx);
        throw ForceException(force_error(rc), "dmdgpu", msg);
    }
    return ctx;
}

// ForceComponent over the device: component ids 0 LJ, 1 bond, 2 angle,
// 3 dihedral, 4 real-space Ewald, 5 PME, 6 exclusion, 7 improper.  Forces and
// energy are added to the caller's (the ForceEngine contract).  Every call
// copies positions in and forces out, so this is for parity tests and single
// points, not for MD steps (GpuSimulationEngine runs those on the device).
class GpuForceComponent : public ForceComponent {
  public:
    GpuForceComponent(const SimulationConfig& cfg, int component, std::string name,
                      int profile = DMDGPU_PROFILE_REF, int precision = DMDGPU_PRECISION_FP64)
        : ctx_(open_context(cfg, profile, precision)), which_(component), name_(std::move(name)) {}
    ~GpuForceComponent() override { dmdgpu_destroy(ctx_); }
    GpuForceComponent(const GpuForceComponent&) = delete;
    GpuForceComponent& operator=(const GpuForceComponent&) = delete;

    std::string name() const override { return name_; }

    void compute(std::span<const double> pos_x, std::span<const double> pos_y,
                 std::span<const double> pos_z, const Cell& cell, std::span<double> forces_x,
                 std::span<double> forces_y, std::span<double> forces_z, double& energy_out) override {
        const int rc = dmdgpu_component_compute(ctx_, which_, pos_x.data(), pos_y.data(), pos_z.data(),
                                                cell.matrix[0], forces_x.data(), forces_y.data(),
                                                forces_z.data(), &energy_out);
        if (rc) throw ForceException(force_error(rc), name_.c_str(), dmdgpu_last_error(ctx_));
    }

  private:
    dmdgpu_ctx* ctx_;
    int which_;
    std::string name_;
};

// The run loop on the device: step / run / run_n advance the device state in
// one call each; state is read back on demand.
class GpuSimulationEngine {
  public:
    explicit GpuSimulationEngine(const SimulationConfig& cfg, int profile = DMDGPU_PROFILE_PHYS,
                                 int precision = DMDGPU_PRECISION_MIXED, int device = 0)
        : ctx_(open_context(cfg, profile, precision, device)), n_(cfg.masses.size()) {}
    ~GpuSimulationEngine() { dmdgpu_destroy(ctx_); }
    GpuSimulationEngine(const GpuSimulationEngine&) = delete;
    GpuSimulationEngine& operator=(const GpuSimulationEngine&) = delete;

    void step() { check(dmdgpu_step(ctx_, 1)); }
    void run() { check(dmdgpu_run(ctx_)); }
    void run_n(int n) { check(dmdgpu_step(ctx_, n)); }
    long long current_step() {
        dmdgpu_scalars s{};
        check(dmdgpu_get_scalars(ctx_, &s));
        return s.step;
    }
    double potential_energy() {
        dmdgpu_scalars s{};
        check(dmdgpu_get_scalars(ctx_, &s));
        return s.potential_energy;
    }
    // which: 0 positions, 1 velocities, 2 forces (SoA, n_atoms each)
    void state(int which, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z) {
        x.resize(n_);
        y.resize(n_);
        z.resize(n_);
        check(dmdgpu_get_state(ctx_, which, x.data(), y.data(), z.data()));
    }
    void save_checkpoint(const std::string& path) { check(dmdgpu_save_checkpoint(ctx_, path.c_str())); }
    void load_checkpoint(const std::string& path) { check(dmdgpu_load_checkpoint(ctx_, path.c_str())); }

  private:
    void check(int rc) {
        if (rc) throw ForceException(force_error(rc), "dmdgpu", dmdgpu_last_error(ctx_));
    }
    dmdgpu_ctx* ctx_;
    size_t n_;
};

}  // namespace dmdgpu_ref
