// adapter_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own force components (LennardJones, HarmonicBond,
// HarmonicAngle, PeriodicDihedral, compiled unmodified from its src/) and
// include/dmdgpu_reference.hpp's GpuForceComponent for the same component ids
// side by side on one system, so a test can hold the adapter a maintainer
// would add to the reference to the reference's own classes.  Built by
// oracle/Makefile (target `adapter`) against libdmdgpu.so.
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

#include "core/cell.h"
#include "dmdgpu_reference.hpp"
#include "force/harmonic_angle.h"
#include "force/harmonic_bond.h"
#include "force/lennard_jones.h"
#include "force/periodic_dihedral.h"

extern "C" int adapter_check(int n, double box, const double* mass, const double* q, const double* x,
                             const double* y, const double* z, const int* types, int n_types,
                             const double* sigma, const double* eps, double lj_cutoff, int nb,
                             const int* bi, const int* bj, const double* bk, const double* br, int na,
                             const int* ai, const int* aj, const int* ak, const double* akt,
                             const double* at0, int nd, const int* di, const int* dj, const int* dk,
                             const int* dl, const int* dn, const double* dkp, const double* dp0,
                             int precision, double* f_ref, double* e_ref, double* f_gpu, double* e_gpu,
                             char* err, int err_len) {
    try {
        SimulationConfig cfg;
        cfg.box_size = box;
        cfg.masses.assign(mass, mass + n);
        cfg.charges.assign(q, q + n);
        cfg.pos_x.assign(x, x + n);
        cfg.pos_y.assign(y, y + n);
        cfg.pos_z.assign(z, z + n);
        cfg.atom_types.assign(types, types + n);
        cfg.use_lj = true;
        cfg.lj.n_types = static_cast<size_t>(n_types);
        cfg.lj.sigma.assign(sigma, sigma + n_types * n_types);
        cfg.lj.epsilon.assign(eps, eps + n_types * n_types);
        cfg.lj_cutoff = lj_cutoff;
        HarmonicBondParams b;
        b.n = nb;
        b.i.assign(bi, bi + nb);
        b.j.assign(bj, bj + nb);
        b.k.assign(bk, bk + nb);
        b.r0.assign(br, br + nb);
        HarmonicAngleParams a;
        a.n = na;
        a.i.assign(ai, ai + na);
        a.j.assign(aj, aj + na);
        a.k.assign(ak, ak + na);
        a.k_theta.assign(akt, akt + na);
        a.theta0.assign(at0, at0 + na);
        PeriodicDihedralParams d;
        d.n = nd;
        d.i.assign(di, di + nd);
        d.j.assign(dj, dj + nd);
        d.k.assign(dk, dk + nd);
        d.l.assign(dl, dl + nd);
        d.periodicity.assign(dn, dn + nd);
        d.k_phi.assign(dkp, dkp + nd);
        d.phi0.assign(dp0, dp0 + nd);
        if (nb) cfg.bonds.push_back(b);
        if (na) cfg.angles.push_back(a);
        if (nd) cfg.dihedrals.push_back(d);

        auto lj = std::make_unique<LennardJones>(cfg.lj, lj_cutoff);
        lj->set_atom_types(cfg.atom_types);
        std::unique_ptr<ForceComponent> ref[4] = {std::move(lj), std::make_unique<HarmonicBond>(b),
                                                   std::make_unique<HarmonicAngle>(a),
                                                   std::make_unique<PeriodicDihedral>(d)};
        const char* names[4] = {"lj", "bond", "angle", "dihedral"};
        const Cell cell(box, box, box);
        for (int c = 0; c < 4; ++c) {
            dmdgpu_ref::GpuForceComponent gpu(cfg, c, names[c], DMDGPU_PROFILE_REF, precision);
            double* fr = f_ref + 3LL * n * c;
            double* fg = f_gpu + 3LL * n * c;
            std::memset(fr, 0, sizeof(double) * 3 * n);
            std::memset(fg, 0, sizeof(double) * 3 * n);
            e_ref[c] = 0.0;
            e_gpu[c] = 0.0;
            ref[c]->compute(cfg.pos_x, cfg.pos_y, cfg.pos_z, cell, std::span<double>(fr, n),
                            std::span<double>(fr + n, n), std::span<double>(fr + 2 * n, n), e_ref[c]);
            gpu.compute(cfg.pos_x, cfg.pos_y, cfg.pos_z, cell, std::span<double>(fg, n),
                        std::span<double>(fg + n, n), std::span<double>(fg + 2 * n, n), e_gpu[c]);
        }
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), static_cast<size_t>(err_len - 1));
            err[err_len - 1] = '\0';
        }
        return 1;
    }
    return 0;
}
