// dmd_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// An FP64 CPU restatement of the DMD reference's per-step force-and-integrate
// path, written for this repository as the checker of the CUDA path.  Only
// tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it
// (through oracle/oracle.py); the product never links or calls it.
//
// Two semantic profiles share this file:
//   profile 0 "ref"  -- the reference's formulas operation for operation,
//                       quirks included (its LJ list has no skin and is rebuilt
//                       every 10 force evaluations; its real-space Ewald list is
//                       never built; exclusion force sign; angle force sign;
//                       dihedral force formula; PME grid indexing, 1/N and
//                       sinc^(2p) factors).
//   profile 1 "phys" -- gradient-consistent forces on the same inputs: shared
//                       cutoff list with exclusions, erfc real space, textbook
//                       SPME, analytic bonded gradients, atomic virial.
// Each function cites the reference file:line it restates.
//
// Parity pinning: the ref profile is checked bit-for-bit against the
// reference's own classes compiled from source (oracle/_ref/libdmdref.so) for
// every component except PME (its translation unit needs FFTW3 and cannot be
// built here); PME is pinned to the reference's known-answer tests
// (tests/unit/force/test_coulomb_pme.cpp) and, in the phys profile, to a direct
// Ewald sum.  The FFT used here is self-written (mixed radix) and is checked
// against numpy.fft by the CPU tests.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <unordered_set>
#include <vector>

#include "fft.h"

namespace {

constexpr double KB = 0.008314462618;   // src/core/constants.h:6
constexpr double KE = 138.935456;       // src/force/coulomb_pme.h:45, coulomb_direct.cpp:49-51
constexpr double PI = 3.14159265358979323846;
constexpr double BAR = 0.0602214086;    // kJ mol^-1 nm^-3 per bar (berendsen_barostat.cpp:60)

// Cell::minimum_image, orthorhombic branch (src/core/cell.cpp:26-38)
inline void min_image(double L, double& dx, double& dy, double& dz) {
    double inv = 1.0 / L;
    dx = dx - std::round(dx * inv) * L;
    dy = dy - std::round(dy * inv) * L;
    dz = dz - std::round(dz * inv) * L;
}

// ---- exact pair enumeration ------------------------------------------------
// All i<j whose minimum-image r2 (reference expression, lennard_jones.cpp:27-39)
// is < rc2, in (i, j) lexicographic order -- identical to the reference's
// O(N^2) double loop.  Cells on wrapped coordinates only prune the search.
void pairs_within(int n, const double* x, const double* y, const double* z, double L,
                  double rc, std::vector<int>& pi, std::vector<int>& pj) {
    pi.clear();
    pj.clear();
    const double rc2 = rc * rc;
    int nc = static_cast<int>(std::floor(L / (rc * (1.0 + 1e-9))));
    if (nc < 3 || n < 256) {
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) {
                double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
                min_image(L, dx, dy, dz);
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rc2) {
                    pi.push_back(i);
                    pj.push_back(j);
                }
            }
        return;
    }
    const double cs = L / nc;
    std::vector<int> cell(n), head(nc * nc * nc, -1), next(n, -1);
    auto ci = [&](double v) {
        double w = v - std::floor(v / L) * L;
        int c = static_cast<int>(w / cs);
        return std::min(std::max(c, 0), nc - 1);
    };
    for (int i = n - 1; i >= 0; --i) {
        int c = (ci(z[i]) * nc + ci(y[i])) * nc + ci(x[i]);
        cell[i] = c;
        next[i] = head[c];
        head[c] = i;
    }
    std::vector<std::pair<int, int>> out;
    std::vector<int> nb;
    for (int i = 0; i < n; ++i) {
        int c = cell[i];
        int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
        nb.clear();
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int nx_ = (cx + dx + nc) % nc, ny_ = (cy + dy + nc) % nc,
                        nz_ = (cz + dz + nc) % nc;
                    nb.push_back((nz_ * nc + ny_) * nc + nx_);
                }
        std::sort(nb.begin(), nb.end());
        nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
        for (int cc : nb)
            for (int j = head[cc]; j >= 0; j = next[j]) {
                if (j <= i) continue;
                double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
                min_image(L, dx, dy, dz);
                double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rc2) out.emplace_back(i, j);
            }
    }
    std::sort(out.begin(), out.end());
    pi.resize(out.size());
    pj.resize(out.size());
    for (size_t k = 0; k < out.size(); ++k) {
        pi[k] = out[k].first;
        pj[k] = out[k].second;
    }
}

// ---- FFT (fft.h: the same transform the FFTW-API shim gives the reference) --
// FFTW-style in-place r2c on a padded K^3 buffer: real row (z,y) at
// buf[(z*K+y)*P + x], x < K, P = 2(K/2+1); the half spectrum overwrites it.
void r2c_inplace(std::vector<double>& buf, int K) {
    dmd_fft::r2c3d(buf.data(), 2 * (K / 2 + 1), buf.data(), K, K, K);
}

// Unnormalised c2r in place; padding doubles of each output row are set to
// zero (FFTW leaves them unspecified; this build defines them as zero).
void c2r_inplace(std::vector<double>& buf, int K) {
    dmd_fft::c2r3d(buf.data(), buf.data(), 2 * (K / 2 + 1), K, K, K);
}

// CoulombPME::theta4 / dtheta4 (src/force/coulomb_pme.cpp:50-69)
double theta4(double u) {
    double a = std::abs(u);
    if (a >= 2.0) return 0.0;
    if (a >= 1.0) {
        double t = 2.0 - a;
        return t * t * t / 6.0;
    }
    return (4.0 - 6.0 * a * a + 3.0 * a * a * a) / 6.0;
}
double dtheta4(double u) {
    double a = std::abs(u);
    if (a >= 2.0) return 0.0;
    double s = (u >= 0.0) ? 1.0 : -1.0;
    if (a >= 1.0) {
        double t = 2.0 - a;
        return -s * t * t / 2.0;
    }
    return s * (9.0 * a * a - 12.0 * a) / 6.0;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), used by the phys Andersen thermostat.
void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
        uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
        uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n1 = static_cast<uint32_t>(p1);
        uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c[3] ^ k1;
        uint32_t n3 = static_cast<uint32_t>(p0);
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

}  // namespace

extern "C" {

struct orc_system {
    int n_atoms;
    double box;
    const double* q;
    const int* type;
    int n_types;
    const double *lj_sigma, *lj_eps;
    int use_lj;
    double lj_cutoff;
    int coulomb_type;  // 0 cutoff/direct, 1 pme
    double coul_cutoff, ewald;
    int pme_K, pme_order;
    int n_excl;
    const int *excl_i, *excl_j;
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
    int profile;  // 0 ref, 1 phys
};

struct orc_energy {
    double lj, coul_real, coul_recip, coul_self, coul_excl, bond, angle, dihedral, improper, total,
        virial;
};

// ---- exported small helpers (pinned against the reference's unit tests) ----
void orc_min_image(double L, double dx, double dy, double dz, double* out) {
    min_image(L, dx, dy, dz);
    out[0] = dx; out[1] = dy; out[2] = dz;
}
double orc_theta4(double u) { return theta4(u); }
double orc_dtheta4(double u) { return dtheta4(u); }
// CoulombPME::calc_self_energy (coulomb_pme.cpp:71-75)
double orc_self_energy(double alpha, const double* q, int n, double k_e) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += q[i] * q[i];
    return -k_e * alpha / std::sqrt(M_PI) * s;
}
void orc_philox(uint32_t* c, uint32_t k0, uint32_t k1) { philox(c, k0, k1); }

// ---- distance constraints (src/integrate/constraints.cpp) ------------------
// Constraints::apply (constraints.cpp:9-47): SHAKE as Gauss-Seidel sweeps over
// the constraints in their order; each constraint whose |r^2 - d^2| exceeds
// the tolerance moves both atoms along the current (minimum-image) bond
// vector by lambda = (r^2 - d^2) / (2 d^2 (1/m_i + 1/m_j)), weighted by the
// inverse masses; at most 100 sweeps, stopping after the first sweep whose
// largest error (measured before each correction) is below the tolerance.
// Positions in place; returns the number of sweeps.
int orc_shake(int nc, const int* ci, const int* cj, const double* dist, double tol, double L,
              const double* m, double* x, double* y, double* z) {
    int it = 0;
    while (it < 100) {
        ++it;
        double worst = 0.0;
        for (int c = 0; c < nc; ++c) {
            const int a = ci[c], b = cj[c];
            double dx = x[b] - x[a], dy = y[b] - y[a], dz = z[b] - z[a];
            min_image(L, dx, dy, dz);
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double d2 = dist[c] * dist[c];
            const double err = r2 - d2;
            worst = std::max(worst, std::abs(err));
            if (!(std::abs(err) > tol)) continue;
            const double wa = 1.0 / m[a], wb = 1.0 / m[b];
            const double lam = err / (2.0 * d2 * (wa + wb));
            x[a] += lam * dx * wa;
            y[a] += lam * dy * wa;
            z[a] += lam * dz * wa;
            x[b] -= lam * dx * wb;
            y[b] -= lam * dy * wb;
            z[b] -= lam * dz * wb;
        }
        if (worst < tol) break;
    }
    return it;
}

// Constraints::apply_rattle (constraints.cpp:49-91): the velocity half, the
// same sweeps on r.v (relative velocity along the bond), lambda = r.v / (r^2
// (1/m_i + 1/m_j)).  Velocities in place; returns the number of sweeps.
int orc_rattle(int nc, const int* ci, const int* cj, double tol, double L, const double* m,
               const double* x, const double* y, const double* z, double* vx, double* vy,
               double* vz) {
    int it = 0;
    while (it < 100) {
        ++it;
        double worst = 0.0;
        for (int c = 0; c < nc; ++c) {
            const int a = ci[c], b = cj[c];
            double dx = x[b] - x[a], dy = y[b] - y[a], dz = z[b] - z[a];
            min_image(L, dx, dy, dz);
            const double rv = dx * (vx[b] - vx[a]) + dy * (vy[b] - vy[a]) + dz * (vz[b] - vz[a]);
            const double r2 = dx * dx + dy * dy + dz * dz;
            worst = std::max(worst, std::abs(rv));
            if (!(std::abs(rv) > tol)) continue;
            const double wa = 1.0 / m[a], wb = 1.0 / m[b];
            const double lam = rv / (r2 * (wa + wb));
            vx[a] += lam * dx * wa;
            vy[a] += lam * dy * wa;
            vz[a] += lam * dz * wa;
            vx[b] -= lam * dx * wb;
            vy[b] -= lam * dy * wb;
            vz[b] -= lam * dz * wb;
        }
        if (worst < tol) break;
    }
    return it;
}

// 3-D r2c of a K^3 real array (natural layout) -> K*K*(K/2+1) complex (interleaved)
void orc_rfft3(int K, const double* in, double* out) {
    const int P = 2 * (K / 2 + 1);
    std::vector<double> buf(static_cast<size_t>(K) * K * P, 0.0);
    for (size_t r = 0; r < static_cast<size_t>(K) * K; ++r)
        for (int x = 0; x < K; ++x) buf[r * P + x] = in[r * K + x];
    r2c_inplace(buf, K);
    std::memcpy(out, buf.data(), sizeof(double) * K * K * (K / 2 + 1) * 2);
}

// pair list handle ---------------------------------------------------------
struct orc_pairs { std::vector<int> i, j; };
void* orc_pairs_build(int n, const double* x, const double* y, const double* z, double L,
                      double rc) {
    auto* p = new orc_pairs();
    pairs_within(n, x, y, z, L, rc, p->i, p->j);
    return p;
}
long orc_pairs_count(void* h) { return static_cast<long>(static_cast<orc_pairs*>(h)->i.size()); }
void orc_pairs_copy(void* h, int* pi, int* pj) {
    auto* p = static_cast<orc_pairs*>(h);
    std::copy(p->i.begin(), p->i.end(), pi);
    std::copy(p->j.begin(), p->j.end(), pj);
}
void orc_pairs_free(void* h) { delete static_cast<orc_pairs*>(h); }

}  // extern "C"

namespace {

using Sys = orc_system;

// LennardJones::compute over a given list (lennard_jones.cpp:43-92); the r2 recheck
// against the cutoff uses the current positions.
void lj_ref(const Sys& s, const double* x, const double* y, const double* z, double L,
            const std::vector<int>& pi, const std::vector<int>& pj, double* fx, double* fy,
            double* fz, double& eout) {
    const double rc2 = s.lj_cutoff * s.lj_cutoff;
    double energy = 0.0;
    for (size_t p = 0; p < pi.size(); ++p) {
        int i = pi[p], j = pj[p];
        double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
        min_image(L, dx, dy, dz);
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= rc2) continue;
        int ti = s.type[i], tj = s.type[j];
        double eps = s.lj_eps[ti * s.n_types + tj];
        double sig = s.lj_sigma[ti * s.n_types + tj];
        double sig2 = sig * sig;
        double sig6 = sig2 * sig2 * sig2;
        double r6 = r2 * r2 * r2;
        double sr6 = sig6 / r6;
        double f = 24.0 * eps * (2.0 * sr6 * sr6 - sr6) / r2;
        fx[i] -= f * dx; fy[i] -= f * dy; fz[i] -= f * dz;
        fx[j] += f * dx; fy[j] += f * dy; fz[j] += f * dz;
        energy += 4.0 * eps * (sr6 * sr6 - sr6);
    }
    eout += energy;
}

// HarmonicBond::compute (harmonic_bond.cpp:12-47); identical in both profiles.
void bonds(const Sys& s, const double* x, const double* y, const double* z, double L,
           double* fx, double* fy, double* fz, double& eout, double& vir) {
    double energy = 0.0;
    for (int n = 0; n < s.n_bonds; ++n) {
        int ai = s.bond_i[n], aj = s.bond_j[n];
        double dx = x[aj] - x[ai], dy = y[aj] - y[ai], dz = z[aj] - z[ai];
        min_image(L, dx, dy, dz);
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = std::sqrt(r2);
        double dr = r - s.bond_r0[n];
        double f = -s.bond_k[n] * dr / r;
        double gx = f * dx, gy = f * dy, gz = f * dz;
        fx[ai] -= gx; fy[ai] -= gy; fz[ai] -= gz;
        fx[aj] += gx; fy[aj] += gy; fz[aj] += gz;
        energy += 0.5 * s.bond_k[n] * dr * dr;
        vir += f * r2;
    }
    eout += energy;
}

// HarmonicAngle::compute (harmonic_angle.cpp:10-63).  The reference's force is the
// negative of -grad(E) (sign quirk); phys flips it.
void angles(const Sys& s, const double* x, const double* y, const double* z, double L,
            double* fx, double* fy, double* fz, double& eout, double& vir) {
    const double sg = (s.profile == 0) ? 1.0 : -1.0;
    double energy = 0.0;
    for (int n = 0; n < s.n_angles; ++n) {
        int ai = s.ang_i[n], aj = s.ang_j[n], ak = s.ang_k[n];
        double dx_ij = x[ai] - x[aj], dy_ij = y[ai] - y[aj], dz_ij = z[ai] - z[aj];
        min_image(L, dx_ij, dy_ij, dz_ij);
        double dx_kj = x[ak] - x[aj], dy_kj = y[ak] - y[aj], dz_kj = z[ak] - z[aj];
        min_image(L, dx_kj, dy_kj, dz_kj);
        double r_ij2 = dx_ij * dx_ij + dy_ij * dy_ij + dz_ij * dz_ij;
        double r_kj2 = dx_kj * dx_kj + dy_kj * dy_kj + dz_kj * dz_kj;
        double r_ij = std::sqrt(r_ij2);
        double r_kj = std::sqrt(r_kj2);
        double dot = dx_ij * dx_kj + dy_ij * dy_kj + dz_ij * dz_kj;
        double c = dot / (r_ij * r_kj);
        c = std::max(-1.0, std::min(1.0, c));
        double theta = std::acos(c);
        double dth = theta - s.ang_t0[n];
        double f = -s.ang_kt[n] * dth / std::sqrt(1.0 - c * c);
        double fx_ij = f * (dx_kj / (r_ij * r_kj) - c * dx_ij / r_ij2);
        double fy_ij = f * (dy_kj / (r_ij * r_kj) - c * dy_ij / r_ij2);
        double fz_ij = f * (dz_kj / (r_ij * r_kj) - c * dz_ij / r_ij2);
        double fx_kj = f * (dx_ij / (r_ij * r_kj) - c * dx_kj / r_kj2);
        double fy_kj = f * (dy_ij / (r_ij * r_kj) - c * dy_kj / r_kj2);
        double fz_kj = f * (dz_ij / (r_ij * r_kj) - c * dz_kj / r_kj2);
        if (sg < 0) {
            fx_ij = -fx_ij; fy_ij = -fy_ij; fz_ij = -fz_ij;
            fx_kj = -fx_kj; fy_kj = -fy_kj; fz_kj = -fz_kj;
        }
        fx[ai] += fx_ij; fy[ai] += fy_ij; fz[ai] += fz_ij;
        fx[aj] -= fx_ij + fx_kj; fy[aj] -= fy_ij + fy_kj; fz[aj] -= fz_ij + fz_kj;
        fx[ak] += fx_kj; fy[ak] += fy_kj; fz[ak] += fz_kj;
        energy += 0.5 * s.ang_kt[n] * dth * dth;
        vir += dx_ij * fx_ij + dy_ij * fy_ij + dz_ij * fz_ij + dx_kj * fx_kj + dy_kj * fy_kj +
               dz_kj * fz_kj;
    }
    eout += energy;
}

// PeriodicDihedral::compute (periodic_dihedral.cpp:10-137) and, with IMP,
// HarmonicImproper::compute (harmonic_improper.cpp:10-130): the same plane
// geometry and angle; E = k (1 + cos(n phi - phi0)) or k/2 (chi - chi0)^2.
// ref: the reference's gradient vectors times -dE/dangle; phys: the analytic
// gradient of the same energy.
template <bool IMP>
void torsions(const Sys& s, const double* x, const double* y, const double* z, double L,
              double* fx, double* fy, double* fz, double& eout, double& vir) {
    double energy = 0.0;
    const int nt = IMP ? s.n_imp : s.n_dih;
    for (int n = 0; n < nt; ++n) {
        int ai = IMP ? s.imp_i[n] : s.dih_i[n], aj = IMP ? s.imp_j[n] : s.dih_j[n];
        int ak = IMP ? s.imp_k[n] : s.dih_k[n], al = IMP ? s.imp_l[n] : s.dih_l[n];
        double ba_x = x[ai] - x[aj], ba_y = y[ai] - y[aj], ba_z = z[ai] - z[aj];
        min_image(L, ba_x, ba_y, ba_z);
        double bc_x = x[ak] - x[aj], bc_y = y[ak] - y[aj], bc_z = z[ak] - z[aj];
        min_image(L, bc_x, bc_y, bc_z);
        double dc_x = x[ak] - x[al], dc_y = y[ak] - y[al], dc_z = z[ak] - z[al];
        min_image(L, dc_x, dc_y, dc_z);
        double n1_x = ba_y * bc_z - ba_z * bc_y;
        double n1_y = ba_z * bc_x - ba_x * bc_z;
        double n1_z = ba_x * bc_y - ba_y * bc_x;
        double n2_x = bc_y * dc_z - bc_z * dc_y;
        double n2_y = bc_z * dc_x - bc_x * dc_z;
        double n2_z = bc_x * dc_y - bc_y * dc_x;
        double n1_sq = n1_x * n1_x + n1_y * n1_y + n1_z * n1_z;
        double n2_sq = n2_x * n2_x + n2_y * n2_y + n2_z * n2_z;
        double bc_sq = bc_x * bc_x + bc_y * bc_y + bc_z * bc_z;
        if (n1_sq < 1e-30 || n2_sq < 1e-30 || bc_sq < 1e-30) continue;
        double n1_norm = std::sqrt(n1_sq);
        double n2_norm = std::sqrt(n2_sq);
        double bc_norm = std::sqrt(bc_sq);
        double dot = n1_x * n2_x + n1_y * n2_y + n1_z * n2_z;
        double cos_phi = dot / (n1_norm * n2_norm);
        cos_phi = std::max(-1.0, std::min(1.0, cos_phi));
        double triple = bc_x * (n1_y * n2_z - n1_z * n2_y) + bc_y * (n1_z * n2_x - n1_x * n2_z) +
                        bc_z * (n1_x * n2_y - n1_y * n2_x);
        double sin_phi = triple / (bc_norm * n1_norm * n2_norm);
        sin_phi = std::max(-1.0, std::min(1.0, sin_phi));
        double phi = std::atan2(sin_phi, cos_phi);
        int p = IMP ? 0 : s.dih_n[n];
        double k = IMP ? s.imp_kphi[n] : s.dih_kphi[n];
        double phi0 = IMP ? s.imp_phi0[n] : s.dih_phi0[n];
        double dchi = phi - phi0;
        if (IMP) energy += 0.5 * k * dchi * dchi;
        else energy += k * (1.0 + std::cos(p * phi - phi0));
        if (s.profile == 0) {
            double pref = IMP ? -k * dchi : k * p * std::sin(p * phi - phi0);
            if (std::abs(pref) < 1e-30) continue;
            double gi_x = (bc_y * n1_z - bc_z * n1_y) / n1_sq;
            double gi_y = (bc_z * n1_x - bc_x * n1_z) / n1_sq;
            double gi_z = (bc_x * n1_y - bc_y * n1_x) / n1_sq;
            double gl_x = -(bc_y * n2_z - bc_z * n2_y) / n2_sq;
            double gl_y = -(bc_z * n2_x - bc_x * n2_z) / n2_sq;
            double gl_z = -(bc_x * n2_y - bc_y * n2_x) / n2_sq;
            double n1xba_x = n1_y * ba_z - n1_z * ba_y;
            double n1xba_y = n1_z * ba_x - n1_x * ba_z;
            double n1xba_z = n1_x * ba_y - n1_y * ba_x;
            double dcxn2_x = dc_y * n2_z - dc_z * n2_y;
            double dcxn2_y = dc_z * n2_x - dc_x * n2_z;
            double dcxn2_z = dc_x * n2_y - dc_y * n2_x;
            double gj_x = n1xba_x / n1_sq + dcxn2_x / n2_sq - gi_x;
            double gj_y = n1xba_y / n1_sq + dcxn2_y / n2_sq - gi_y;
            double gj_z = n1xba_z / n1_sq + dcxn2_z / n2_sq - gi_z;
            double bxn2_x = (bc_y * n2_z - bc_z * n2_y) / n2_sq;
            double bxn2_y = (bc_z * n2_x - bc_x * n2_z) / n2_sq;
            double bxn2_z = (bc_x * n2_y - bc_y * n2_x) / n2_sq;
            double gk_x = bxn2_x - n1xba_x / n1_sq - dcxn2_x / n2_sq;
            double gk_y = bxn2_y - n1xba_y / n1_sq - dcxn2_y / n2_sq;
            double gk_z = bxn2_z - n1xba_z / n1_sq - dcxn2_z / n2_sq;
            fx[ai] += pref * gi_x; fy[ai] += pref * gi_y; fz[ai] += pref * gi_z;
            fx[aj] += pref * gj_x; fy[aj] += pref * gj_y; fz[aj] += pref * gj_z;
            fx[ak] += pref * gk_x; fy[ak] += pref * gk_y; fz[ak] += pref * gk_z;
            fx[al] += pref * gl_x; fy[al] += pref * gl_y; fz[al] += pref * gl_z;
            vir += ba_x * pref * gi_x + ba_y * pref * gi_y + ba_z * pref * gi_z +
                   bc_x * pref * gk_x + bc_y * pref * gk_y + bc_z * pref * gk_z +
                   (bc_x - dc_x) * pref * gl_x + (bc_y - dc_y) * pref * gl_y +
                   (bc_z - dc_z) * pref * gl_z;
        } else {
            // dE/dphi = -k p sin(p phi - phi0); phi is the IUPAC angle of
            // m = r_ij x r_kj and n = r_kj x r_kl (r_ij = ba, r_kj = bc, r_kl = dc).
            double ddphi = IMP ? k * dchi : -k * p * std::sin(p * phi - phi0);
            double f_i_x = -ddphi * bc_norm / n1_sq * n1_x;
            double f_i_y = -ddphi * bc_norm / n1_sq * n1_y;
            double f_i_z = -ddphi * bc_norm / n1_sq * n1_z;
            double f_l_x = ddphi * bc_norm / n2_sq * n2_x;
            double f_l_y = ddphi * bc_norm / n2_sq * n2_y;
            double f_l_z = ddphi * bc_norm / n2_sq * n2_z;
            double pp = (ba_x * bc_x + ba_y * bc_y + ba_z * bc_z) / bc_sq;
            double qq = (dc_x * bc_x + dc_y * bc_y + dc_z * bc_z) / bc_sq;
            double sv_x = pp * f_i_x - qq * f_l_x;
            double sv_y = pp * f_i_y - qq * f_l_y;
            double sv_z = pp * f_i_z - qq * f_l_z;
            double f_j_x = f_i_x - sv_x, f_j_y = f_i_y - sv_y, f_j_z = f_i_z - sv_z;
            double f_k_x = f_l_x + sv_x, f_k_y = f_l_y + sv_y, f_k_z = f_l_z + sv_z;
            fx[ai] += f_i_x; fy[ai] += f_i_y; fz[ai] += f_i_z;
            fx[aj] -= f_j_x; fy[aj] -= f_j_y; fz[aj] -= f_j_z;
            fx[ak] -= f_k_x; fy[ak] -= f_k_y; fz[ak] -= f_k_z;
            fx[al] += f_l_x; fy[al] += f_l_y; fz[al] += f_l_z;
            vir += ba_x * f_i_x + ba_y * f_i_y + ba_z * f_i_z - bc_x * f_k_x - bc_y * f_k_y -
                   bc_z * f_k_z + (bc_x - dc_x) * f_l_x + (bc_y - dc_y) * f_l_y +
                   (bc_z - dc_z) * f_l_z;
        }
    }
    eout += energy;
}
void dihedrals(const Sys& s, const double* x, const double* y, const double* z, double L,
               double* fx, double* fy, double* fz, double& eout, double& vir) {
    torsions<false>(s, x, y, z, L, fx, fy, fz, eout, vir);
}
void impropers(const Sys& s, const double* x, const double* y, const double* z, double L,
               double* fx, double* fy, double* fz, double& eout, double& vir) {
    torsions<true>(s, x, y, z, L, fx, fy, fz, eout, vir);
}

// CoulombExclusion::compute (coulomb_exclusion.cpp:16-56).  ref: E -= k q q / r with
// the repulsive Coulomb force (sign quirk).  phys: -k q q erf(a r)/r and its gradient.
void exclusions(const Sys& s, const double* x, const double* y, const double* z, double L,
                double* fx, double* fy, double* fz, double& eout, double& vir) {
    const double k_e = 138.935456;
    double energy = 0.0;
    const double a = s.ewald;
    for (int p = 0; p < s.n_excl; ++p) {
        int i = s.excl_i[p], j = s.excl_j[p];
        double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
        min_image(L, dx, dy, dz);
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = std::sqrt(r2);
        double qiqj = s.q[i] * s.q[j];
        if (s.profile == 0) {
            double f = k_e * qiqj / (r2 * r);
            fx[i] -= f * dx; fy[i] -= f * dy; fz[i] -= f * dz;
            fx[j] += f * dx; fy[j] += f * dy; fz[j] += f * dz;
            energy += k_e * qiqj / r;
            vir += f * r2;
        } else {
            double erf_ar = std::erf(a * r);
            double g = 2.0 * a / std::sqrt(PI) * std::exp(-a * a * r2);
            double f = k_e * qiqj * (g / r2 - erf_ar / (r2 * r));
            fx[i] -= f * dx; fy[i] -= f * dy; fz[i] -= f * dz;
            fx[j] += f * dx; fy[j] += f * dy; fz[j] += f * dz;
            energy += k_e * qiqj * erf_ar / r;
            vir += f * r2;
        }
    }
    eout -= energy;
}

// phys non-bonded: LJ (lennard_jones.cpp formula) + erfc real space
// (coulomb_direct.cpp:68-83 formula) over all non-excluded pairs within the cutoffs.
void nonbonded_phys(const Sys& s, const double* x, const double* y, const double* z, double L,
                    double* fx, double* fy, double* fz, double& e_lj, double& e_c, double& vir) {
    const bool coul = true;
    const double rcl = s.use_lj ? s.lj_cutoff : 0.0;
    const double rcc = coul ? s.coul_cutoff : 0.0;
    const double rmax = std::max(rcl, rcc);
    if (rmax <= 0.0) return;
    std::unordered_set<uint64_t> ex;
    for (int p = 0; p < s.n_excl; ++p) {
        uint64_t a = static_cast<uint32_t>(std::min(s.excl_i[p], s.excl_j[p]));
        uint64_t b = static_cast<uint32_t>(std::max(s.excl_i[p], s.excl_j[p]));
        ex.insert((a << 32) | b);
    }
    std::vector<int> pi, pj;
    pairs_within(s.n_atoms, x, y, z, L, rmax, pi, pj);
    const double rcl2 = rcl * rcl, rcc2 = rcc * rcc, a = s.ewald;
    const double k_e = 138.935456;
    double el = 0.0, ec = 0.0;
    for (size_t p = 0; p < pi.size(); ++p) {
        int i = pi[p], j = pj[p];
        if (!ex.empty() && ex.count((static_cast<uint64_t>(i) << 32) | static_cast<uint32_t>(j)))
            continue;
        double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
        min_image(L, dx, dy, dz);
        double r2 = dx * dx + dy * dy + dz * dz;
        double f = 0.0;
        if (s.use_lj && r2 < rcl2) {
            int ti = s.type[i], tj = s.type[j];
            double eps = s.lj_eps[ti * s.n_types + tj];
            double sig = s.lj_sigma[ti * s.n_types + tj];
            double sig2 = sig * sig;
            double sig6 = sig2 * sig2 * sig2;
            double r6 = r2 * r2 * r2;
            double sr6 = sig6 / r6;
            f += 24.0 * eps * (2.0 * sr6 * sr6 - sr6) / r2;
            el += 4.0 * eps * (sr6 * sr6 - sr6);
        }
        double qq = s.q[i] * s.q[j];
        if (coul && r2 < rcc2 && qq != 0.0) {
            double r = std::sqrt(r2);
            double erfc_ar = std::erfc(a * r);
            f += k_e * qq * (erfc_ar / (r2 * r) + 2.0 * a * std::exp(-a * a * r2) / (std::sqrt(PI) * r2));
            ec += k_e * qq * erfc_ar / r;
        }
        fx[i] -= f * dx; fy[i] -= f * dy; fz[i] -= f * dz;
        fx[j] += f * dx; fy[j] += f * dy; fz[j] += f * dz;
        vir += f * r2;
    }
    e_lj += el;
    e_c += ec;
}

// CoulombPME (coulomb_pme.cpp:79-318).  ref reproduces its grid indexing (unpadded
// index into FFTW's padded in-place buffer), the 1/N factor on the potential and the
// multiplied sinc^(2p) factor; phys is textbook SPME (padded layout, no 1/N,
// B-spline moduli 1/(2/3 + cos(2 pi m/K)/3)^2 divided out) plus the reciprocal virial.
void pme(const Sys& s, const double* x, const double* y, const double* z, double L, double* fx,
         double* fy, double* fz, double& e_rec, double& e_self, double& vir) {
    const int K = s.pme_K, H = K / 2 + 1, P = 2 * H;
    const bool ref = (s.profile == 0);
    const int n = s.n_atoms;
    std::vector<double> grid(static_cast<size_t>(K) * K * P, 0.0);
    auto gidx = [&](int gz, int gy, int gx) -> size_t {
        return ref ? static_cast<size_t>(gz) * K * K + static_cast<size_t>(gy) * K + gx
                   : (static_cast<size_t>(gz) * K + gy) * P + gx;
    };
    // spread_charges (:79-136)
    for (int i = 0; i < n; ++i) {
        double q = s.q[i];
        if (q == 0.0) continue;
        double frx = x[i] / L, fry = y[i] / L, frz = z[i] / L;
        frx -= std::floor(frx);
        fry -= std::floor(fry);
        frz -= std::floor(frz);
        double ux = frx * K, uy = fry * K, uz = frz * K;
        int m0x = static_cast<int>(std::floor(ux)) - 1;
        int m0y = static_cast<int>(std::floor(uy)) - 1;
        int m0z = static_cast<int>(std::floor(uz)) - 1;
        double wx[4], wy[4], wz[4];
        for (int d = 0; d < 4; ++d) {
            wx[d] = theta4(ux - (m0x + d));
            wy[d] = theta4(uy - (m0y + d));
            wz[d] = theta4(uz - (m0z + d));
        }
        for (int iz = 0; iz < 4; ++iz) {
            int gz = (m0z + iz) % K;
            if (gz < 0) gz += K;
            double w_z = wz[iz];
            for (int iy = 0; iy < 4; ++iy) {
                int gy = (m0y + iy) % K;
                if (gy < 0) gy += K;
                double w_yz = wy[iy] * w_z;
                for (int ix = 0; ix < 4; ++ix) {
                    int gx = (m0x + ix) % K;
                    if (gx < 0) gx += K;
                    grid[gidx(gz, gy, gx)] += q * wx[ix] * w_yz;
                }
            }
        }
    }
    // compute_reciprocal_energy_and_potential (:143-201)
    r2c_inplace(grid, K);
    const double alpha = s.ewald;
    const double V = L * (L * L)  /* Cell::volume of a diagonal cell (cell.cpp:19-24) */;
    const double k_e = 138.935456;
    auto bref = [&](int m) -> double {
        if (m == 0) return 1.0;
        double t = M_PI * std::abs(m) / K;
        return std::pow(std::sin(t) / t, 2 * s.pme_order);
    };
    auto bphys = [&](int m) -> double {
        double c = 2.0 / 3.0 + std::cos(2.0 * PI * m / K) / 3.0;
        return 1.0 / (c * c);
    };
    double energy = 0.0, wrec = 0.0;
    for (int kz = 0; kz < K; ++kz) {
        int mz = (kz <= K / 2) ? kz : kz - K;
        for (int ky = 0; ky < K; ++ky) {
            int my = (ky <= K / 2) ? ky : ky - K;
            size_t row = (static_cast<size_t>(kz) * K + ky) * H;
            for (int kx = 0; kx <= K / 2; ++kx) {
                int mx = kx;
                if (mx == 0 && my == 0 && mz == 0) {
                    if (!ref) { grid[row * 2] = 0.0; grid[row * 2 + 1] = 0.0; }
                    continue;
                }
                double w = (kx == 0 || (K % 2 == 0 && kx == K / 2)) ? 1.0 : 2.0;
                double msq = (static_cast<double>(mx) * mx) / (L * L) +
                             (static_cast<double>(my) * my) / (L * L) +
                             (static_cast<double>(mz) * mz) / (L * L);
                double k2 = 4.0 * M_PI * M_PI * msq;
                double B = ref ? bref(mx) * bref(my) * bref(mz) : bphys(mx) * bphys(my) * bphys(mz);
                double green = 4.0 * M_PI * k_e / V * std::exp(-k2 / (4.0 * alpha * alpha)) * B / k2;
                size_t idx = (row + kx) * 2;
                double re = grid[idx], im = grid[idx + 1];
                double ek = 0.5 * w * green * (re * re + im * im);
                energy += ek;
                wrec += ek * (1.0 - k2 / (2.0 * alpha * alpha));
                grid[idx] = re * green;
                grid[idx + 1] = im * green;
            }
        }
    }
    c2r_inplace(grid, K);
    if (ref) {
        double norm = 1.0 / (static_cast<double>(K) * K * K);
        for (size_t i = 0; i < static_cast<size_t>(K) * K * K; ++i) grid[i] *= norm;
    }
    // interpolate_forces (:205-283)
    const double fac = static_cast<double>(K) / L;
    for (int i = 0; i < n; ++i) {
        double q = s.q[i];
        if (q == 0.0) continue;
        double frx = x[i] / L, fry = y[i] / L, frz = z[i] / L;
        frx -= std::floor(frx);
        fry -= std::floor(fry);
        frz -= std::floor(frz);
        double ux = frx * K, uy = fry * K, uz = frz * K;
        int m0x = static_cast<int>(std::floor(ux)) - 1;
        int m0y = static_cast<int>(std::floor(uy)) - 1;
        int m0z = static_cast<int>(std::floor(uz)) - 1;
        double wx[4], wy[4], wz[4], dwx[4], dwy[4], dwz[4];
        for (int d = 0; d < 4; ++d) {
            wx[d] = theta4(ux - (m0x + d));
            wy[d] = theta4(uy - (m0y + d));
            wz[d] = theta4(uz - (m0z + d));
            dwx[d] = dtheta4(ux - (m0x + d));
            dwy[d] = dtheta4(uy - (m0y + d));
            dwz[d] = dtheta4(uz - (m0z + d));
        }
        double gx_ = 0.0, gy_ = 0.0, gz_ = 0.0;
        for (int iz = 0; iz < 4; ++iz) {
            int gz = (m0z + iz) % K;
            if (gz < 0) gz += K;
            double w_z = wz[iz], dw_z = dwz[iz];
            for (int iy = 0; iy < 4; ++iy) {
                int gy = (m0y + iy) % K;
                if (gy < 0) gy += K;
                double w_y = wy[iy], dw_y = dwy[iy];
                for (int ix = 0; ix < 4; ++ix) {
                    int gx = (m0x + ix) % K;
                    if (gx < 0) gx += K;
                    double phi = grid[gidx(gz, gy, gx)];
                    gx_ += phi * dwx[ix] * w_y * w_z;
                    gy_ += phi * wx[ix] * dw_y * w_z;
                    gz_ += phi * wx[ix] * w_y * dw_z;
                }
            }
        }
        fx[i] -= q * fac * gx_;
        fy[i] -= q * fac * gy_;
        fz[i] -= q * fac * gz_;
    }
    double sq = 0.0;
    for (int i = 0; i < n; ++i) sq += s.q[i] * s.q[i];
    e_rec += energy;
    e_self += -k_e * alpha / std::sqrt(M_PI) * sq;
    vir += wrec;
}

bool has_coulomb_excl(const Sys& s) {
    return s.coulomb_type == 1 || s.n_excl > 0;
}

// ForceEngine::compute for the component list of build_force_engine
// (simulation_engine.cpp:147-203), order LJ, bonds, angles, dihedrals,
// CoulombDirect, [PME], [Exclusion].  lj_list (ref only) is the LJ pair list in use.
void eval_forces(const Sys& s, const double* x, const double* y, const double* z, double L,
                 const std::vector<int>* lpi, const std::vector<int>* lpj, double* fx,
                 double* fy, double* fz, orc_energy& e) {
    double pe = 0.0;  // the reference accumulates one running potential_energy
    e = orc_energy{};
    if (s.profile == 0) {
        if (s.use_lj) {
            double t = 0.0;
            lj_ref(s, x, y, z, L, *lpi, *lpj, fx, fy, fz, t);
            e.lj = t;
            pe += t;
        }
        double v = 0.0, t = 0.0;
        if (s.n_bonds) { t = 0.0; bonds(s, x, y, z, L, fx, fy, fz, t, v); e.bond = t; pe += t; }
        if (s.n_angles) { t = 0.0; angles(s, x, y, z, L, fx, fy, fz, t, v); e.angle = t; pe += t; }
        if (s.n_dih) { t = 0.0; dihedrals(s, x, y, z, L, fx, fy, fz, t, v); e.dihedral = t; pe += t; }
        if (s.n_imp) { t = 0.0; impropers(s, x, y, z, L, fx, fy, fz, t, v); e.improper = t; pe += t; }
        // CoulombDirect: list never built in engine runs -> contributes 0 (Q1)
        if (s.coulomb_type == 1) {
            double er = 0.0, es = 0.0;
            pme(s, x, y, z, L, fx, fy, fz, er, es, v);
            e.coul_recip = er;
            e.coul_self = es;
            pe += er + es;
        }
        if (has_coulomb_excl(s)) {
            t = 0.0;
            exclusions(s, x, y, z, L, fx, fy, fz, t, v);
            e.coul_excl = t;
            pe += t;
        }
        e.total = pe;
        e.virial = 0.0;  // ref virial is sum r.F over absolute positions (barostat.cpp:6-14)
        return;
    }
    double vir = 0.0;
    nonbonded_phys(s, x, y, z, L, fx, fy, fz, e.lj, e.coul_real, vir);
    bonds(s, x, y, z, L, fx, fy, fz, e.bond, vir);
    angles(s, x, y, z, L, fx, fy, fz, e.angle, vir);
    dihedrals(s, x, y, z, L, fx, fy, fz, e.dihedral, vir);
    impropers(s, x, y, z, L, fx, fy, fz, e.improper, vir);
    if (s.coulomb_type == 1) pme(s, x, y, z, L, fx, fy, fz, e.coul_recip, e.coul_self, vir);
    if (has_coulomb_excl(s)) exclusions(s, x, y, z, L, fx, fy, fz, e.coul_excl, vir);
    e.total = e.lj + e.coul_real + e.coul_recip + e.coul_self + e.coul_excl + e.bond + e.angle +
              e.dihedral + e.improper;
    e.virial = vir;
}

}  // namespace

extern "C" {

// Single-point forces (accumulated into f*) and energy terms at positions x,y,z.
// In the ref profile the LJ list is a fresh rebuild at these positions (what the
// reference does on its first compute() call).
void orc_forces(const orc_system* s, const double* x, const double* y, const double* z,
                double* fx, double* fy, double* fz, orc_energy* e) {
    std::vector<int> pi, pj;
    if (s->profile == 0 && s->use_lj) pairs_within(s->n_atoms, x, y, z, s->box, s->lj_cutoff, pi, pj);
    eval_forces(*s, x, y, z, s->box, &pi, &pj, fx, fy, fz, *e);
}

// Per-component entry points (ForceComponent::compute contract: accumulate).
void orc_component(const orc_system* s, int which, const double* x, const double* y,
                   const double* z, double* fx, double* fy, double* fz, double* energy,
                   double* virial) {
    double v = 0.0;
    const double L = s->box;
    switch (which) {
        case 0: {  // LJ (ref: fresh list; phys: nonbonded without charges)
            if (s->profile == 0) {
                std::vector<int> pi, pj;
                pairs_within(s->n_atoms, x, y, z, L, s->lj_cutoff, pi, pj);
                lj_ref(*s, x, y, z, L, pi, pj, fx, fy, fz, *energy);
            } else {
                double ec = 0.0;
                orc_system t = *s;
                t.coul_cutoff = 0.0;
                nonbonded_phys(t, x, y, z, L, fx, fy, fz, *energy, ec, v);
            }
            break;
        }
        case 1: bonds(*s, x, y, z, L, fx, fy, fz, *energy, v); break;
        case 2: angles(*s, x, y, z, L, fx, fy, fz, *energy, v); break;
        case 3: dihedrals(*s, x, y, z, L, fx, fy, fz, *energy, v); break;
        case 4: {  // real-space Coulomb (phys) -- zero in ref engine runs
            if (s->profile == 1) {
                double el = 0.0;
                orc_system t = *s;
                t.use_lj = 0;
                nonbonded_phys(t, x, y, z, L, fx, fy, fz, el, *energy, v);
            }
            break;
        }
        case 5: {
            double es = 0.0;
            pme(*s, x, y, z, L, fx, fy, fz, *energy, es, v);
            *energy += es;
            break;
        }
        case 6: exclusions(*s, x, y, z, L, fx, fy, fz, *energy, v); break;
        case 7: impropers(*s, x, y, z, L, fx, fy, fz, *energy, v); break;
        default: break;
    }
    if (virial) *virial += v;
}

// ---- engine ----------------------------------------------------------------
struct orc_run {
    double dt;
    const double *mass, *x, *y, *z, *vx, *vy, *vz;
    int gen_vel, seed;
    double init_temperature;
    int thermostat;  // 0 none 1 berendsen 2 nose-hoover 3 andersen
    double t_temp, t_tau, t_freq;
    int barostat;    // 0 none 1 berendsen
    double b_pressure, b_tau, b_compress;
    uint64_t rng_seed;  // phys Andersen (Philox key)
    int brute_list;     // ref profile: rebuild the LJ list with the reference's O(N^2) loop
    int n_cons;         // SHAKE / RATTLE distance constraints (0: none)
    const int *cons_i, *cons_j;
    const double* cons_dist;
    double cons_tol;
};

struct OrcEngine {
    orc_system s;
    // owned copies of every array referenced by s
    std::vector<double> q, lj_sigma, lj_eps, bond_k, bond_r0, ang_kt, ang_t0, dih_kphi, dih_phi0, imp_kphi,
        imp_phi0;
    std::vector<int> imp_i, imp_j, imp_k, imp_l;
    std::vector<int> type, excl_i, excl_j, bond_i, bond_j, ang_i, ang_j, ang_k, dih_i, dih_j,
        dih_k, dih_l, dih_n;
    std::vector<double> m, x, y, z, vx, vy, vz, fx, fy, fz;
    std::vector<int> lpi, lpj;
    int lj_counter{10};
    double L, dt, time{0.0};
    long step{0};
    orc_run run;
    double zeta{0.0};
    unsigned int andersen_seed{42};
    orc_energy e{};
    bool have_forces{false};
    double pscale{1.0};  // phys: barostat scale chosen at the end of a step, applied with the next drift
    double eps_dot{0.0};   // Andersen barostat: piston velocity (strain rate)
    double piston_W{1.0};  // and piston mass
    std::vector<int> cons_i, cons_j;  // distance constraints, in the order they are swept
    std::vector<double> cons_d;
    double cons_tol{1e-6};
};

void* orc_engine_create(const orc_system* s, const orc_run* r) {
    auto* E = new OrcEngine();
    const int n = s->n_atoms;
    auto cpd = [](std::vector<double>& v, const double* p, size_t c) { v.assign(p ? p : nullptr, p ? p + c : nullptr); };
    auto cpi = [](std::vector<int>& v, const int* p, size_t c) { v.assign(p ? p : nullptr, p ? p + c : nullptr); };
    E->s = *s;
    const size_t nt2 = static_cast<size_t>(s->n_types) * s->n_types;
    cpd(E->q, s->q, n); E->s.q = E->q.data();
    cpi(E->type, s->type, n); E->s.type = E->type.data();
    cpd(E->lj_sigma, s->lj_sigma, nt2); E->s.lj_sigma = E->lj_sigma.data();
    cpd(E->lj_eps, s->lj_eps, nt2); E->s.lj_eps = E->lj_eps.data();
    cpi(E->excl_i, s->excl_i, s->n_excl); E->s.excl_i = E->excl_i.data();
    cpi(E->excl_j, s->excl_j, s->n_excl); E->s.excl_j = E->excl_j.data();
    cpi(E->bond_i, s->bond_i, s->n_bonds); E->s.bond_i = E->bond_i.data();
    cpi(E->bond_j, s->bond_j, s->n_bonds); E->s.bond_j = E->bond_j.data();
    cpd(E->bond_k, s->bond_k, s->n_bonds); E->s.bond_k = E->bond_k.data();
    cpd(E->bond_r0, s->bond_r0, s->n_bonds); E->s.bond_r0 = E->bond_r0.data();
    cpi(E->ang_i, s->ang_i, s->n_angles); E->s.ang_i = E->ang_i.data();
    cpi(E->ang_j, s->ang_j, s->n_angles); E->s.ang_j = E->ang_j.data();
    cpi(E->ang_k, s->ang_k, s->n_angles); E->s.ang_k = E->ang_k.data();
    cpd(E->ang_kt, s->ang_kt, s->n_angles); E->s.ang_kt = E->ang_kt.data();
    cpd(E->ang_t0, s->ang_t0, s->n_angles); E->s.ang_t0 = E->ang_t0.data();
    cpi(E->dih_i, s->dih_i, s->n_dih); E->s.dih_i = E->dih_i.data();
    cpi(E->dih_j, s->dih_j, s->n_dih); E->s.dih_j = E->dih_j.data();
    cpi(E->dih_k, s->dih_k, s->n_dih); E->s.dih_k = E->dih_k.data();
    cpi(E->dih_l, s->dih_l, s->n_dih); E->s.dih_l = E->dih_l.data();
    cpi(E->dih_n, s->dih_n, s->n_dih); E->s.dih_n = E->dih_n.data();
    cpd(E->dih_kphi, s->dih_kphi, s->n_dih); E->s.dih_kphi = E->dih_kphi.data();
    cpd(E->dih_phi0, s->dih_phi0, s->n_dih); E->s.dih_phi0 = E->dih_phi0.data();
    cpi(E->imp_i, s->imp_i, s->n_imp); E->s.imp_i = E->imp_i.data();
    cpi(E->imp_j, s->imp_j, s->n_imp); E->s.imp_j = E->imp_j.data();
    cpi(E->imp_k, s->imp_k, s->n_imp); E->s.imp_k = E->imp_k.data();
    cpi(E->imp_l, s->imp_l, s->n_imp); E->s.imp_l = E->imp_l.data();
    cpd(E->imp_kphi, s->imp_kphi, s->n_imp); E->s.imp_kphi = E->imp_kphi.data();
    cpd(E->imp_phi0, s->imp_phi0, s->n_imp); E->s.imp_phi0 = E->imp_phi0.data();
    E->run = *r;
    E->L = s->box;
    E->dt = r->dt;
    cpd(E->m, r->mass, n);
    cpd(E->x, r->x, n); cpd(E->y, r->y, n); cpd(E->z, r->z, n);
    if (r->vx) { cpd(E->vx, r->vx, n); cpd(E->vy, r->vy, n); cpd(E->vz, r->vz, n); }
    else { E->vx.assign(n, 0.0); E->vy.assign(n, 0.0); E->vz.assign(n, 0.0); }
    E->fx.assign(n, 0.0); E->fy.assign(n, 0.0); E->fz.assign(n, 0.0);
    if (r->gen_vel && n > 0) {  // build_simulation (simulation_engine.cpp:339-383)
        std::mt19937 rng(r->seed);
        std::normal_distribution<double> normal(0.0, 1.0);
        double kBT = KB * r->init_temperature;
        for (int i = 0; i < n; ++i) {
            double sg = std::sqrt(kBT / E->m[i]);
            E->vx[i] = normal(rng) * sg;
            E->vy[i] = normal(rng) * sg;
            E->vz[i] = normal(rng) * sg;
        }
        double cx = 0, cy = 0, cz = 0, tm = 0;
        for (int i = 0; i < n; ++i) {
            cx += E->m[i] * E->vx[i]; cy += E->m[i] * E->vy[i]; cz += E->m[i] * E->vz[i];
            tm += E->m[i];
        }
        cx /= tm; cy /= tm; cz /= tm;
        for (int i = 0; i < n; ++i) { E->vx[i] -= cx; E->vy[i] -= cy; E->vz[i] -= cz; }
        if (r->init_temperature > 0) {
            double ek = 0;
            for (int i = 0; i < n; ++i)
                ek += 0.5 * E->m[i] * (E->vx[i] * E->vx[i] + E->vy[i] * E->vy[i] + E->vz[i] * E->vz[i]);
            double ta = (n < 2) ? 0.0 : 2.0 * ek / ((3.0 * n - 3.0) * KB);
            double lam = std::sqrt(r->init_temperature / ta);
            for (int i = 0; i < n; ++i) { E->vx[i] *= lam; E->vy[i] *= lam; E->vz[i] *= lam; }
        }
    }
    {  // AndersenBarostat's piston mass (andersen_barostat.cpp:8-14)
        double dof = 3.0 * static_cast<double>(n) - 3.0;
        if (dof < 1.0) dof = 1.0;
        E->piston_W = dof * KB * r->b_pressure * r->b_tau * r->b_tau;
    }
    if (r->n_cons > 0) {  // constraint_type "shake" with pairs (simulation_engine.cpp:294-300)
        cpi(E->cons_i, r->cons_i, r->n_cons);
        cpi(E->cons_j, r->cons_j, r->n_cons);
        cpd(E->cons_d, r->cons_dist, r->n_cons);
        E->cons_tol = r->cons_tol;
    }
    return E;
}

}  // extern "C"

namespace {

double kinetic(const OrcEngine* E) {  // thermostat.cpp:6-15
    double ek = 0.0;
    const size_t n = E->m.size();
    for (size_t i = 0; i < n; ++i)
        ek += 0.5 * E->m[i] * (E->vx[i] * E->vx[i] + E->vy[i] * E->vy[i] + E->vz[i] * E->vz[i]);
    return ek;
}
double temp_of(double ek, size_t n) {  // thermostat.cpp:17-21
    if (n < 2) return 0.0;
    double dof = 3.0 * static_cast<double>(n) - 3.0;
    return 2.0 * ek / (dof * KB);
}

void eng_compute(OrcEngine* E) {
    const int n = E->s.n_atoms;
    std::fill(E->fx.begin(), E->fx.end(), 0.0);
    std::fill(E->fy.begin(), E->fy.end(), 0.0);
    std::fill(E->fz.begin(), E->fz.end(), 0.0);
    if (E->s.profile == 0 && E->s.use_lj) {
        // LennardJones::compute rebuild cadence (lennard_jones.cpp:53-55, :91)
        if (E->lj_counter >= 10) {
            if (E->run.brute_list) {
                // LennardJones::rebuild_pair_list (lennard_jones.cpp:18-41), O(N^2)
                E->lpi.clear();
                E->lpj.clear();
                const double rc2 = E->s.lj_cutoff * E->s.lj_cutoff;
                const double* x = E->x.data();
                const double* y = E->y.data();
                const double* z = E->z.data();
                for (int i = 0; i < n; ++i)
                    for (int j = i + 1; j < n; ++j) {
                        double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
                        min_image(E->L, dx, dy, dz);
                        if (dx * dx + dy * dy + dz * dz < rc2) {
                            E->lpi.push_back(i);
                            E->lpj.push_back(j);
                        }
                    }
            } else {
                pairs_within(n, E->x.data(), E->y.data(), E->z.data(), E->L, E->s.lj_cutoff, E->lpi, E->lpj);
            }
            E->lj_counter = 0;
        }
    }
    E->s.box = E->L;
    eval_forces(E->s, E->x.data(), E->y.data(), E->z.data(), E->L, &E->lpi, &E->lpj,
                E->fx.data(), E->fy.data(), E->fz.data(), E->e);
    if (E->s.profile == 0 && E->s.use_lj) ++E->lj_counter;
    E->have_forces = true;
}

void eng_half_kick(OrcEngine* E) {  // integrator.cpp:4-12
    double half_dt = 0.5 * E->dt;
    for (size_t i = 0; i < E->m.size(); ++i) {
        double inv_mass = 1.0 / E->m[i];
        E->vx[i] += E->fx[i] * inv_mass * half_dt;
        E->vy[i] += E->fy[i] * inv_mass * half_dt;
        E->vz[i] += E->fz[i] * inv_mass * half_dt;
    }
}
void eng_advance(OrcEngine* E) {  // integrator.cpp:14-20
    for (size_t i = 0; i < E->m.size(); ++i) {
        E->x[i] += E->vx[i] * E->dt;
        E->y[i] += E->vy[i] * E->dt;
        E->z[i] += E->vz[i] * E->dt;
    }
}

void eng_thermostat(OrcEngine* E) {
    const orc_run& r = E->run;
    const size_t n = E->m.size();
    const double dt = E->dt;
    if (r.thermostat == 1) {  // berendsen.cpp:13-28
        if (r.t_tau <= 0.0) return;
        double ek = kinetic(E);
        if (ek <= 0.0) return;
        double T = temp_of(ek, n);
        double lam = std::sqrt(1.0 + dt / r.t_tau * (r.t_temp / T - 1.0));
        if (lam <= 0.0) return;
        for (size_t i = 0; i < n; ++i) { E->vx[i] *= lam; E->vy[i] *= lam; E->vz[i] *= lam; }
    } else if (r.thermostat == 2) {  // nose_hoover.cpp:6-32
        double dof = 3.0 * static_cast<double>(n) - 3.0;
        if (dof < 1.0) dof = 1.0;
        double Q = dof * KB * r.t_temp * r.t_tau * r.t_tau;
        double ek = kinetic(E);
        double T = temp_of(ek, n);
        E->zeta += 0.5 * dt * KB * (T - r.t_temp) / Q;
        double sc = std::exp(-E->zeta * 0.5 * dt);
        for (size_t i = 0; i < n; ++i) { E->vx[i] *= sc; E->vy[i] *= sc; E->vz[i] *= sc; }
    } else if (r.thermostat == 3) {
        double prob = r.t_freq * dt;
        if (prob <= 0.0) return;
        if (E->s.profile == 0) {  // andersen.cpp:14-32
            std::mt19937_64 rng(E->andersen_seed);
            std::uniform_real_distribution<double> uni(0.0, 1.0);
            std::normal_distribution<double> nd(0.0, 1.0);
            for (size_t i = 0; i < n; ++i) {
                if (uni(rng) < prob) {
                    double sg = std::sqrt(KB * r.t_temp / E->m[i]);
                    E->vx[i] = nd(rng) * sg;
                    E->vy[i] = nd(rng) * sg;
                    E->vz[i] = nd(rng) * sg;
                }
            }
            ++E->andersen_seed;
        } else {
            // counter-based: (atom, call index) -> Philox4x32-10 -> uniform + Box-Muller
            const uint32_t k0 = static_cast<uint32_t>(r.rng_seed), k1 = static_cast<uint32_t>(r.rng_seed >> 32);
            const uint64_t call = E->andersen_seed - 42u;
            for (size_t i = 0; i < n; ++i) {
                uint32_t c[4] = {static_cast<uint32_t>(i), static_cast<uint32_t>(call),
                                 static_cast<uint32_t>(call >> 32), 0x414E4400u};
                philox(c, k0, k1);
                double u = c[0] * 2.3283064365386963e-10;
                if (u < prob) {
                    double sg = std::sqrt(KB * r.t_temp / E->m[i]);
                    double u1 = (c[1] + 1.0) * 2.3283064365386963e-10;
                    double u2 = c[2] * 2.3283064365386963e-10;
                    double rr = std::sqrt(-2.0 * std::log(u1));
                    uint32_t d[4] = {static_cast<uint32_t>(i), static_cast<uint32_t>(call),
                                     static_cast<uint32_t>(call >> 32), 0x414E4401u};
                    philox(d, k0, k1);
                    double u3 = (d[0] + 1.0) * 2.3283064365386963e-10;
                    double u4 = d[1] * 2.3283064365386963e-10;
                    E->vx[i] = rr * std::cos(2.0 * PI * u2) * sg;
                    E->vy[i] = rr * std::sin(2.0 * PI * u2) * sg;
                    E->vz[i] = std::sqrt(-2.0 * std::log(u3)) * std::cos(2.0 * PI * u4) * sg;
                }
            }
            ++E->andersen_seed;
        }
    }
}

// AndersenBarostat::apply (andersen_barostat.cpp:20-45), REF profile: the
// piston velocity takes half a step of 3V (P - P0) / W (P from the reference's
// virial and kinetic energy, P0 as given: the reference's units), positions and
// box scale by exp(eps_dot dt), then the second half step with the same forcing.
void eng_andersen_barostat(OrcEngine* E) {
    const orc_run& r = E->run;
    const size_t n = E->m.size();
    const double L = E->L;
    const double volume = L * (L * L);
    if (volume <= 0.0) return;
    const double ek = kinetic(E);
    double w = 0.0;
    for (size_t i = 0; i < n; ++i)  // barostat.cpp:6-14
        w += E->x[i] * E->fx[i] + E->y[i] * E->fy[i] + E->z[i] * E->fz[i];
    const double P = (2.0 * ek + w) / (3.0 * volume);
    const double forcing = 3.0 * volume * (P - r.b_pressure) / E->piston_W;
    E->eps_dot = E->eps_dot + 0.5 * E->dt * forcing;
    const double sc = std::exp(E->eps_dot * E->dt);
    for (size_t i = 0; i < n; ++i) { E->x[i] *= sc; E->y[i] *= sc; E->z[i] *= sc; }
    E->L *= sc;
    E->eps_dot = E->eps_dot + 0.5 * E->dt * forcing;
}

void eng_barostat(OrcEngine* E) {  // berendsen_barostat.cpp:14-66
    const orc_run& r = E->run;
    if (r.barostat == 2 && E->s.profile == 0) {
        eng_andersen_barostat(E);
        return;
    }
    if (r.barostat != 1) return;
    if (r.b_tau <= 0.0) return;
    const size_t n = E->m.size();
    double L = E->L;
    double volume = L * (L * L)  /* Cell::volume of a diagonal cell (cell.cpp:19-24) */;
    if (volume <= 0.0) return;
    double ek = kinetic(E);
    double w = 0.0;
    if (E->s.profile == 0) {
        for (size_t i = 0; i < n; ++i)  // barostat.cpp:6-14
            w += E->x[i] * E->fx[i] + E->y[i] * E->fy[i] + E->z[i] * E->fz[i];
    } else {
        w = E->e.virial;
    }
    double P = (volume <= 0.0) ? 0.0 : (2.0 * ek + w) / (3.0 * volume);
    double mu;
    if (E->s.profile == 0) {
        double beta_internal = r.b_compress / BAR;
        mu = 1.0 - (E->dt / r.b_tau) * beta_internal * (r.b_pressure - P);
    } else {
        mu = 1.0 - (E->dt / r.b_tau) * r.b_compress * (r.b_pressure - P / BAR);
    }
    if (mu <= 0.0) mu = 0.0;
    double sc = std::cbrt(mu);
    if (E->s.profile == 1) {  // phys: applied with the next step's drift (eng_apply_pending_scale)
        E->pscale = sc;
        return;
    }
    for (size_t i = 0; i < n; ++i) { E->x[i] *= sc; E->y[i] *= sc; E->z[i] *= sc; }
    E->L *= sc;
}

// phys correction of Q13 with a barostat: the reference scales positions and box
// at the end of a step and evaluates forces twice in the next one; here the
// scale waits for the next drift, so the first kick of a step uses the forces of
// the previous evaluation and the single evaluation of the step sees the scaled
// positions.
void eng_apply_pending_scale(OrcEngine* E) {
    if (E->pscale == 1.0) return;
    const double sc = E->pscale;
    for (size_t i = 0; i < E->m.size(); ++i) { E->x[i] *= sc; E->y[i] *= sc; E->z[i] *= sc; }
    E->L *= sc;
    E->pscale = 1.0;
}

// After the drift (simulation_engine.cpp:67): SHAKE on the new positions.
// phys: the displacement SHAKE makes is also given to the half-step velocities
// (v += dx / dt), so that positions and velocities stay consistent.
void eng_shake(OrcEngine* E) {
    if (E->cons_i.empty()) return;
    const int n = static_cast<int>(E->x.size());
    const bool phys = E->s.profile == 1;
    std::vector<double> x0, y0, z0;
    if (phys) {
        x0 = E->x;
        y0 = E->y;
        z0 = E->z;
    }
    orc_shake(static_cast<int>(E->cons_i.size()), E->cons_i.data(), E->cons_j.data(), E->cons_d.data(),
              E->cons_tol, E->L, E->m.data(), E->x.data(), E->y.data(), E->z.data());
    if (phys)
        for (int i = 0; i < n; ++i) {
            E->vx[i] += (E->x[i] - x0[i]) / E->dt;
            E->vy[i] += (E->y[i] - y0[i]) / E->dt;
            E->vz[i] += (E->z[i] - z0[i]) / E->dt;
        }
}

// After the second half kick (simulation_engine.cpp:78): RATTLE on the velocities.
void eng_rattle(OrcEngine* E) {
    if (E->cons_i.empty()) return;
    orc_rattle(static_cast<int>(E->cons_i.size()), E->cons_i.data(), E->cons_j.data(), E->cons_tol,
               E->L, E->m.data(), E->x.data(), E->y.data(), E->z.data(), E->vx.data(), E->vy.data(),
               E->vz.data());
}

}  // namespace

extern "C" {

// SimulationEngine::step (simulation_engine.cpp:53-86).  The phys profile skips the
// first evaluation when it would repeat the previous step's second one, which does
// not change any result because phys forces depend on positions only; with a
// barostat it applies the pending scale before the drift (eng_apply_pending_scale).
void orc_engine_step(void* h, int nsteps) {
    auto* E = static_cast<OrcEngine*>(h);
    for (int it = 0; it < nsteps; ++it) {
        bool skip = (E->s.profile == 1) && E->have_forces;
        if (!skip) eng_compute(E);
        eng_half_kick(E);
        if (E->s.profile == 1) eng_apply_pending_scale(E);
        eng_advance(E);
        eng_shake(E);
        eng_compute(E);
        eng_half_kick(E);
        eng_rattle(E);
        eng_thermostat(E);
        eng_barostat(E);
        ++E->step;
        E->time += E->dt;
    }
}

void orc_engine_get(void* h, int which, double* x, double* y, double* z) {
    auto* E = static_cast<OrcEngine*>(h);
    const std::vector<double>* v[3];
    if (which == 0) { v[0] = &E->x; v[1] = &E->y; v[2] = &E->z; }
    else if (which == 1) { v[0] = &E->vx; v[1] = &E->vy; v[2] = &E->vz; }
    else { v[0] = &E->fx; v[1] = &E->fy; v[2] = &E->fz; }
    std::memcpy(x, v[0]->data(), v[0]->size() * sizeof(double));
    std::memcpy(y, v[1]->data(), v[1]->size() * sizeof(double));
    std::memcpy(z, v[2]->data(), v[2]->size() * sizeof(double));
}

// out: [PE, box, time, step, lj_counter, zeta, KE, andersen_calls]
void orc_engine_scalars(void* h, double* out) {
    auto* E = static_cast<OrcEngine*>(h);
    out[0] = E->e.total;
    out[1] = E->L;
    out[2] = E->time;
    out[3] = static_cast<double>(E->step);
    out[4] = E->lj_counter;
    out[5] = E->zeta;
    out[6] = kinetic(E);
    out[7] = E->andersen_seed - 42.0;
}

void orc_engine_energy(void* h, orc_energy* e) { *e = static_cast<OrcEngine*>(h)->e; }

void orc_engine_destroy(void* h) { delete static_cast<OrcEngine*>(h); }

}  // extern "C"
