// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// A thin extern "C" driver around the reference DMD engine's own, unmodified
// C++ classes, compiled from their sources in place by oracle/Makefile into
// oracle/_ref/libdmdref.so.  Only the test-suite, the smoke check and the CPU
// baseline leg of bench.py load it; nothing in the product links it.
//
// Buildable reference translation units (g++ 13, -std=c++20, no FMA
// contraction, which is what the reference's own CMake build produces on
// x86-64): src/core/*, src/force/*, src/integrate/*, src/thermostat/*,
// src/barostat/*, src/sim/checkpoint.cpp.  src/force/coulomb_pme.cpp includes
// <fftw3.h>; FFTW3 is not installed, so it is compiled against shims/fftw3.h
// (the same API over this repo's FFT, FFTW's in-place layout kept).
// Unbuildable here: src/sim/simulation_engine.cpp (includes trajectory/h5md_writer.h -> HDF5),
// src/trajectory/* (HDF5).  The engine step sequence of
// src/sim/simulation_engine.cpp:53-86 and the factory of :147-203 are
// therefore restated below (a dozen lines) on top of the reference's own
// ForceEngine / Integrator / Thermostat / Barostat objects.
//
// The pair list of LennardJones / CoulombDirect is private in the reference;
// it is read here (for pair-set parity) by compiling the headers with
// `private` mapped to `public`.  That changes no layout or code.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <span>
#include <string>
#include <vector>

#define private public
#include "core/cell.h"
#include "core/constants.h"
#include "core/system_data.h"
#include "force/force_engine.h"
#include "force/force_component.h"
#include "force/lennard_jones.h"
#include "force/coulomb_direct.h"
#include "force/coulomb_exclusion.h"
#include "force/coulomb_pme.h"
#include "force/harmonic_bond.h"
#include "force/harmonic_angle.h"
#include "force/periodic_dihedral.h"
#include "force/harmonic_improper.h"
#include "integrate/integrator.h"
#include "integrate/constraints.h"
#include "thermostat/thermostat.h"
#include "thermostat/berendsen.h"
#include "thermostat/nose_hoover.h"
#include "thermostat/andersen.h"
#include "barostat/barostat.h"
#include "barostat/berendsen_barostat.h"
#include "barostat/andersen_barostat.h"
#include "sim/checkpoint.h"
#undef private

namespace {

std::vector<double> vec(const double* p, int n) { return std::vector<double>(p, p + n); }
std::vector<int> veci(const int* p, int n) { return std::vector<int>(p, p + n); }

}  // namespace

extern "C" {

// ---- integrate/constraints: the reference's SHAKE / RATTLE on arrays --------
void ref_shake(int n, int nc, const int* ci, const int* cj, const double* dist, double tol,
               double L, const double* m, double* x, double* y, double* z) {
    SystemData sys(static_cast<size_t>(n));
    sys.masses = vec(m, n);
    sys.pos_x = vec(x, n);
    sys.pos_y = vec(y, n);
    sys.pos_z = vec(z, n);
    ConstraintsParams p;
    p.i = veci(ci, nc);
    p.j = veci(cj, nc);
    p.distance_target = vec(dist, nc);
    p.tolerance = tol;
    Constraints c(std::move(p));
    Cell cell(L, L, L);
    c.apply(sys, cell);
    std::copy(sys.pos_x.begin(), sys.pos_x.end(), x);
    std::copy(sys.pos_y.begin(), sys.pos_y.end(), y);
    std::copy(sys.pos_z.begin(), sys.pos_z.end(), z);
}

void ref_rattle(int n, int nc, const int* ci, const int* cj, const double* dist, double tol,
                double L, const double* m, const double* x, const double* y, const double* z,
                double* vx, double* vy, double* vz) {
    SystemData sys(static_cast<size_t>(n));
    sys.masses = vec(m, n);
    sys.pos_x = vec(x, n);
    sys.pos_y = vec(y, n);
    sys.pos_z = vec(z, n);
    sys.vel_x = vec(vx, n);
    sys.vel_y = vec(vy, n);
    sys.vel_z = vec(vz, n);
    ConstraintsParams p;
    p.i = veci(ci, nc);
    p.j = veci(cj, nc);
    p.distance_target = vec(dist, nc);
    p.tolerance = tol;
    Constraints c(std::move(p));
    Cell cell(L, L, L);
    c.apply_rattle(sys, cell);
    std::copy(sys.vel_x.begin(), sys.vel_x.end(), vx);
    std::copy(sys.vel_y.begin(), sys.vel_y.end(), vy);
    std::copy(sys.vel_z.begin(), sys.vel_z.end(), vz);
}

// ---- core/cell ----------------------------------------------------------
void ref_min_image(double L, double dx, double dy, double dz, double* out) {
    Cell c(L, L, L);
    c.minimum_image(dx, dy, dz, out[0], out[1], out[2]);
}
void ref_wrap(double L, double* xyz) {
    Cell c(L, L, L);
    c.wrap(xyz[0], xyz[1], xyz[2]);
}

// ---- LennardJones: rebuild (O(N^2)) + one compute --------------------------
// Returns the number of pairs; copies up to cap pairs into pi/pj.
long ref_lj(int n, const double* x, const double* y, const double* z, double L,
            const int* types, int n_types, const double* sigma, const double* eps,
            double rc, double* fx, double* fy, double* fz, double* energy,
            int* pi, int* pj, long cap) {
    LennardJonesParams p;
    p.n_types = static_cast<size_t>(n_types);
    p.sigma = vec(sigma, n_types * n_types);
    p.epsilon = vec(eps, n_types * n_types);
    LennardJones lj(std::move(p), rc);
    lj.set_atom_types(std::span<const int>(types, n));
    Cell cell(L, L, L);
    std::span<const double> sx(x, n), sy(y, n), sz(z, n);
    lj.rebuild_pair_list(sx, sy, sz, cell);
    lj.compute(sx, sy, sz, cell, std::span<double>(fx, n), std::span<double>(fy, n),
               std::span<double>(fz, n), *energy);
    long np = static_cast<long>(lj.pairs_i_.size());
    for (long k = 0; k < np && k < cap; ++k) {
        pi[k] = lj.pairs_i_[k];
        pj[k] = lj.pairs_j_[k];
    }
    return np;
}

// ---- CoulombDirect with an explicitly built list (unit-test usage) --------
void ref_coulomb_direct(int n, const double* x, const double* y, const double* z, double L,
                        const double* q, double rc, double alpha, double* fx, double* fy,
                        double* fz, double* energy) {
    CoulombDirectParams p;
    p.cutoff = rc;
    p.ewald_coefficient = alpha;
    CoulombDirect c(p);
    c.set_charges(std::span<const double>(q, n));
    Cell cell(L, L, L);
    std::span<const double> sx(x, n), sy(y, n), sz(z, n);
    c.rebuild_pair_list(sx, sy, sz, cell);
    c.compute(sx, sy, sz, cell, std::span<double>(fx, n), std::span<double>(fy, n),
              std::span<double>(fz, n), *energy);
}

// ---- CoulombPME (reciprocal part + self energy) on a cubic K^3 mesh ------
void ref_pme(int n, const double* x, const double* y, const double* z, double L, const double* q,
             int K, double rc, double alpha, int order, double* fx, double* fy, double* fz,
             double* energy) {
    PMEParams p;
    p.cutoff = rc;
    p.ewald_coefficient = alpha;
    p.spline_order = order;
    p.nx = p.ny = p.nz = K;
    CoulombPME c(p);
    c.set_charges(std::span<const double>(q, n));
    Cell cell(L, L, L);
    c.compute(std::span<const double>(x, n), std::span<const double>(y, n),
              std::span<const double>(z, n), cell, std::span<double>(fx, n),
              std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

void ref_exclusion(int n, const double* x, const double* y, const double* z, double L,
                   const double* q, int ne, const int* ei, const int* ej, double* fx,
                   double* fy, double* fz, double* energy) {
    CoulombExclusion c;
    c.set_charges(std::span<const double>(q, n));
    c.set_exclusions(std::span<const int>(ei, ne), std::span<const int>(ej, ne));
    Cell cell(L, L, L);
    c.compute(std::span<const double>(x, n), std::span<const double>(y, n),
              std::span<const double>(z, n), cell, std::span<double>(fx, n),
              std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

void ref_bond(int n, const double* x, const double* y, const double* z, double L, int nb,
              const int* bi, const int* bj, const double* k, const double* r0, double* fx,
              double* fy, double* fz, double* energy) {
    HarmonicBondParams p;
    p.n = nb;
    p.i = veci(bi, nb);
    p.j = veci(bj, nb);
    p.k = vec(k, nb);
    p.r0 = vec(r0, nb);
    HarmonicBond b(std::move(p));
    Cell cell(L, L, L);
    b.compute(std::span<const double>(x, n), std::span<const double>(y, n),
              std::span<const double>(z, n), cell, std::span<double>(fx, n),
              std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

void ref_angle(int n, const double* x, const double* y, const double* z, double L, int na,
               const int* ai, const int* aj, const int* ak, const double* kt, const double* t0,
               double* fx, double* fy, double* fz, double* energy) {
    HarmonicAngleParams p;
    p.n = na;
    p.i = veci(ai, na);
    p.j = veci(aj, na);
    p.k = veci(ak, na);
    p.k_theta = vec(kt, na);
    p.theta0 = vec(t0, na);
    HarmonicAngle a(std::move(p));
    Cell cell(L, L, L);
    a.compute(std::span<const double>(x, n), std::span<const double>(y, n),
              std::span<const double>(z, n), cell, std::span<double>(fx, n),
              std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

void ref_dihedral(int n, const double* x, const double* y, const double* z, double L, int nd,
                  const int* di, const int* dj, const int* dk, const int* dl, const int* per,
                  const double* kphi, const double* phi0, double* fx, double* fy, double* fz,
                  double* energy) {
    PeriodicDihedralParams p;
    p.n = nd;
    p.i = veci(di, nd);
    p.j = veci(dj, nd);
    p.k = veci(dk, nd);
    p.l = veci(dl, nd);
    p.periodicity = veci(per, nd);
    p.k_phi = vec(kphi, nd);
    p.phi0 = vec(phi0, nd);
    PeriodicDihedral d(std::move(p));
    Cell cell(L, L, L);
    d.compute(std::span<const double>(x, n), std::span<const double>(y, n),
              std::span<const double>(z, n), cell, std::span<double>(fx, n),
              std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

void ref_improper(int n, const double* x, const double* y, const double* z, double L, int ni,
                  const int* ii, const int* ij, const int* ik, const int* il, const double* kphi,
                  const double* phi0, double* fx, double* fy, double* fz, double* energy) {
    ImproperParams p;
    p.n = ni;
    p.i = veci(ii, ni);
    p.j = veci(ij, ni);
    p.k = veci(ik, ni);
    p.l = veci(il, ni);
    p.k_phi = vec(kphi, ni);
    p.phi0 = vec(phi0, ni);
    HarmonicImproper im(std::move(p));
    Cell cell(L, L, L);
    im.compute(std::span<const double>(x, n), std::span<const double>(y, n),
               std::span<const double>(z, n), cell, std::span<double>(fx, n),
               std::span<double>(fy, n), std::span<double>(fz, n), *energy);
}

// ---- thermostat / barostat helpers ---------------------------------------
double ref_kinetic_energy(int n, const double* m, const double* vx, const double* vy,
                          const double* vz) {
    SystemData s(n);
    s.masses = vec(m, n);
    s.vel_x = vec(vx, n);
    s.vel_y = vec(vy, n);
    s.vel_z = vec(vz, n);
    return kinetic_energy(s);
}
double ref_temperature(double ekin, int n) { return temperature(ekin, static_cast<size_t>(n)); }

// ---- engine: the reference's components driven in SimulationEngine::step order ----
struct RefEngine {
    std::unique_ptr<ForceEngine> fe;
    std::unique_ptr<Thermostat> thermo;
    std::unique_ptr<Barostat> baro;
    std::unique_ptr<Constraints> cons;
    LennardJones* lj{nullptr};
    Integrator integ;
    Cell cell;
    SystemData sys;
    double dt{0.002};
    int step{0};
    double time{0.0};
};

struct ref_run_desc {
    int n_atoms;
    double box;
    const double *mass, *charge, *x, *y, *z, *vx, *vy, *vz;
    const int* types;
    int use_lj, n_types;
    const double *lj_sigma, *lj_eps;
    double lj_cutoff;
    int n_bonds;
    const int *bond_i, *bond_j;
    const double *bond_k, *bond_r0;
    int n_angles;
    const int *ang_i, *ang_j, *ang_k;
    const double *ang_kt, *ang_t0;
    int n_dih;
    const int *dih_i, *dih_j, *dih_k, *dih_l, *dih_n;
    const double *dih_kphi, *dih_phi0;
    int n_imp;
    const int *imp_i, *imp_j, *imp_k, *imp_l;
    const double *imp_kphi, *imp_phi0;
    int n_excl;
    const int *excl_i, *excl_j;
    int coulomb_type;  // 0 = cutoff/direct, 1 = pme
    double coul_cutoff, ewald;
    double pme_spacing;
    int pme_order;
    double dt;
    int thermostat;  // 0 none 1 berendsen 2 nose-hoover 3 andersen
    double t_temp, t_tau, t_freq;
    int barostat;  // 0 none 1 berendsen
    double b_pressure, b_tau, b_compress;
    int gen_vel, seed;
    double init_temperature;
    int n_cons;  // SHAKE / RATTLE distance constraints (0: none)
    const int *cons_i, *cons_j;
    const double* cons_dist;
    double cons_tol;
};

void* ref_engine_create(const ref_run_desc* d) {
    auto* e = new RefEngine();
    const int n = d->n_atoms;
    e->fe = std::make_unique<ForceEngine>();
    // component insertion order of build_force_engine (simulation_engine.cpp:147-203)
    if (d->use_lj) {
        LennardJonesParams p;
        p.n_types = static_cast<size_t>(d->n_types);
        p.sigma = vec(d->lj_sigma, d->n_types * d->n_types);
        p.epsilon = vec(d->lj_eps, d->n_types * d->n_types);
        auto lj = std::make_unique<LennardJones>(std::move(p), d->lj_cutoff);
        e->lj = lj.get();
        e->fe->add_component(std::move(lj));
    }
    if (d->n_bonds > 0) {
        HarmonicBondParams p;
        p.n = d->n_bonds;
        p.i = veci(d->bond_i, d->n_bonds);
        p.j = veci(d->bond_j, d->n_bonds);
        p.k = vec(d->bond_k, d->n_bonds);
        p.r0 = vec(d->bond_r0, d->n_bonds);
        e->fe->add_component(std::make_unique<HarmonicBond>(std::move(p)));
    }
    if (d->n_angles > 0) {
        HarmonicAngleParams p;
        p.n = d->n_angles;
        p.i = veci(d->ang_i, d->n_angles);
        p.j = veci(d->ang_j, d->n_angles);
        p.k = veci(d->ang_k, d->n_angles);
        p.k_theta = vec(d->ang_kt, d->n_angles);
        p.theta0 = vec(d->ang_t0, d->n_angles);
        e->fe->add_component(std::make_unique<HarmonicAngle>(std::move(p)));
    }
    if (d->n_dih > 0) {
        PeriodicDihedralParams p;
        p.n = d->n_dih;
        p.i = veci(d->dih_i, d->n_dih);
        p.j = veci(d->dih_j, d->n_dih);
        p.k = veci(d->dih_k, d->n_dih);
        p.l = veci(d->dih_l, d->n_dih);
        p.periodicity = veci(d->dih_n, d->n_dih);
        p.k_phi = vec(d->dih_kphi, d->n_dih);
        p.phi0 = vec(d->dih_phi0, d->n_dih);
        e->fe->add_component(std::make_unique<PeriodicDihedral>(std::move(p)));
    }
    if (d->n_imp > 0) {
        ImproperParams p;
        p.n = d->n_imp;
        p.i = veci(d->imp_i, d->n_imp);
        p.j = veci(d->imp_j, d->n_imp);
        p.k = veci(d->imp_k, d->n_imp);
        p.l = veci(d->imp_l, d->n_imp);
        p.k_phi = vec(d->imp_kphi, d->n_imp);
        p.phi0 = vec(d->imp_phi0, d->n_imp);
        e->fe->add_component(std::make_unique<HarmonicImproper>(std::move(p)));
    }
    CoulombDirect* cd = nullptr;
    CoulombExclusion* ce = nullptr;
    CoulombPME* cp = nullptr;
    {
        CoulombDirectParams p;
        p.cutoff = d->coul_cutoff;
        p.ewald_coefficient = d->ewald;
        auto c = std::make_unique<CoulombDirect>(p);
        cd = c.get();
        e->fe->add_component(std::move(c));
    }
    if (d->coulomb_type == 1) {
        // pme branch of build_force_engine (simulation_engine.cpp:173-190):
        // direct, PME, then the exclusion correction (always added)
        PMEParams p;
        p.cutoff = d->coul_cutoff;
        p.ewald_coefficient = d->ewald;
        p.spline_order = d->pme_order;
        p.nx = std::max(8, static_cast<int>(d->box / d->pme_spacing + 0.5));
        p.ny = p.nx;
        p.nz = p.nx;
        auto c = std::make_unique<CoulombPME>(p);
        cp = c.get();
        e->fe->add_component(std::move(c));
    }
    if (d->coulomb_type == 1 || d->n_excl > 0) {
        auto c = std::make_unique<CoulombExclusion>();
        c->set_exclusions(std::span<const int>(d->excl_i, d->n_excl),
                          std::span<const int>(d->excl_j, d->n_excl));
        ce = c.get();
        e->fe->add_component(std::move(c));
    }
    if (d->thermostat == 1) {
        BerendsenParams p;
        p.temperature = d->t_temp;
        p.tau = d->t_tau;
        e->thermo = std::make_unique<BerendsenThermostat>(p);
    } else if (d->thermostat == 2) {
        NoseHooverParams p;
        p.temperature = d->t_temp;
        p.tau = d->t_tau;
        e->thermo = std::make_unique<NoseHooverThermostat>(p, static_cast<size_t>(n));
    } else if (d->thermostat == 3) {
        AndersenParams p;
        p.temperature = d->t_temp;
        p.frequency = d->t_freq;
        e->thermo = std::make_unique<AndersenThermostat>(p);
    }
    if (d->barostat == 1) {
        BerendsenBarostatParams p;
        p.pressure = d->b_pressure;
        p.tau = d->b_tau;
        p.compressibility = d->b_compress;
        e->baro = std::make_unique<BerendsenBarostat>(p);
    } else if (d->barostat == 2) {  // build_barostat (simulation_engine.cpp:239-243)
        AndersenBarostatParams p;
        p.pressure = d->b_pressure;
        p.tau = d->b_tau;
        e->baro = std::make_unique<AndersenBarostat>(p, static_cast<size_t>(n));
    }
    e->cell = Cell(d->box, d->box, d->box);
    e->dt = d->dt;
    e->sys = SystemData(static_cast<size_t>(n));
    auto& s = e->sys;
    s.masses = vec(d->mass, n);
    s.charges = vec(d->charge, n);
    s.pos_x = vec(d->x, n);
    s.pos_y = vec(d->y, n);
    s.pos_z = vec(d->z, n);
    if (d->vx) {
        s.vel_x = vec(d->vx, n);
        s.vel_y = vec(d->vy, n);
        s.vel_z = vec(d->vz, n);
    }
    s.atom_types = d->types ? veci(d->types, n) : std::vector<int>(n, 0);
    if (e->lj) e->lj->set_atom_types(s.atom_types);
    if (cd) cd->set_charges(s.charges);
    if (cp) cp->set_charges(s.charges);
    if (ce) ce->set_charges(s.charges);
    if (d->gen_vel && n > 0) {
        // Maxwell-Boltzmann generation as in build_simulation (simulation_engine.cpp:339-383)
        std::mt19937 rng(d->seed);
        std::normal_distribution<double> normal(0.0, 1.0);
        double kBT = dmd_constants::KB * d->init_temperature;
        for (int i = 0; i < n; ++i) {
            double sg = std::sqrt(kBT / s.masses[i]);
            s.vel_x[i] = normal(rng) * sg;
            s.vel_y[i] = normal(rng) * sg;
            s.vel_z[i] = normal(rng) * sg;
        }
        double cx = 0, cy = 0, cz = 0, tm = 0;
        for (int i = 0; i < n; ++i) {
            cx += s.masses[i] * s.vel_x[i];
            cy += s.masses[i] * s.vel_y[i];
            cz += s.masses[i] * s.vel_z[i];
            tm += s.masses[i];
        }
        cx /= tm;
        cy /= tm;
        cz /= tm;
        for (int i = 0; i < n; ++i) {
            s.vel_x[i] -= cx;
            s.vel_y[i] -= cy;
            s.vel_z[i] -= cz;
        }
        if (d->init_temperature > 0) {
            double ek = 0;
            for (int i = 0; i < n; ++i)
                ek += 0.5 * s.masses[i] *
                      (s.vel_x[i] * s.vel_x[i] + s.vel_y[i] * s.vel_y[i] +
                       s.vel_z[i] * s.vel_z[i]);
            double ta = temperature(ek, s.n_atoms);
            double lam = std::sqrt(d->init_temperature / ta);
            for (int i = 0; i < n; ++i) {
                s.vel_x[i] *= lam;
                s.vel_y[i] *= lam;
                s.vel_z[i] *= lam;
            }
        }
    }
    if (d->n_cons > 0) {  // build_simulation (simulation_engine.cpp:293-300)
        ConstraintsParams cp;
        cp.i = veci(d->cons_i, d->n_cons);
        cp.j = veci(d->cons_j, d->n_cons);
        cp.distance_target = vec(d->cons_dist, d->n_cons);
        cp.tolerance = d->cons_tol;
        e->cons = std::make_unique<Constraints>(std::move(cp));
    }
    return e;
}

// SimulationEngine::step (simulation_engine.cpp:53-86), restated on the reference objects.
void ref_engine_step(void* h, int nsteps) {
    auto* e = static_cast<RefEngine*>(h);
    auto& s = e->sys;
    for (int it = 0; it < nsteps; ++it) {
        s.step = e->step;
        s.time = e->time;
        s.forces_x.assign(s.n_atoms, 0.0);
        s.forces_y.assign(s.n_atoms, 0.0);
        s.forces_z.assign(s.n_atoms, 0.0);
        s.potential_energy = 0.0;
        e->fe->compute(s, e->cell);
        e->integ.half_kick(s, e->dt);
        e->integ.advance(s, e->dt);
        if (e->cons) e->cons->apply(s, e->cell);
        s.forces_x.assign(s.n_atoms, 0.0);
        s.forces_y.assign(s.n_atoms, 0.0);
        s.forces_z.assign(s.n_atoms, 0.0);
        s.potential_energy = 0.0;
        e->fe->compute(s, e->cell);
        e->integ.half_kick(s, e->dt);
        if (e->cons) e->cons->apply_rattle(s, e->cell);
        if (e->thermo) e->thermo->apply(s, e->dt);
        if (e->baro) e->baro->apply(s, e->cell, e->dt);
        ++e->step;
        s.step = e->step;
        e->time += e->dt;
    }
}

// which: 0 pos, 1 vel, 2 forces
void ref_engine_get(void* h, int which, double* x, double* y, double* z) {
    auto* e = static_cast<RefEngine*>(h);
    auto& s = e->sys;
    const std::vector<double>* v[3];
    if (which == 0) { v[0] = &s.pos_x; v[1] = &s.pos_y; v[2] = &s.pos_z; }
    else if (which == 1) { v[0] = &s.vel_x; v[1] = &s.vel_y; v[2] = &s.vel_z; }
    else { v[0] = &s.forces_x; v[1] = &s.forces_y; v[2] = &s.forces_z; }
    std::memcpy(x, v[0]->data(), s.n_atoms * sizeof(double));
    std::memcpy(y, v[1]->data(), s.n_atoms * sizeof(double));
    std::memcpy(z, v[2]->data(), s.n_atoms * sizeof(double));
}

// out: [potential_energy, box, time, step, lj_step_since_rebuild, zeta]
void ref_engine_scalars(void* h, double* out) {
    auto* e = static_cast<RefEngine*>(h);
    out[0] = e->sys.potential_energy;
    out[1] = e->cell.matrix[0];
    out[2] = e->time;
    out[3] = e->step;
    out[4] = e->lj ? e->lj->step_since_rebuild() : 0;
    auto* nh = dynamic_cast<NoseHooverThermostat*>(e->thermo.get());
    out[5] = nh ? nh->zeta() : 0.0;
}

void ref_engine_save_checkpoint(void* h, const char* path) {
    auto* e = static_cast<RefEngine*>(h);
    checkpoint::save(path, e->sys, e->lj ? e->lj->step_since_rebuild() : 0);
}

void ref_engine_destroy(void* h) { delete static_cast<RefEngine*>(h); }

}  // extern "C"
