// k_integrate.cu -- Velocity Verlet with fused thermostat / barostat bookkeeping.
//
// Reference sequence (SimulationEngine::step, src/sim/simulation_engine.cpp:53-86):
//   compute; half_kick; advance; compute; half_kick; thermostat; barostat.
// Device form (per step, every replica of the batch in the same launches):
//   [eval #1]           only where the first evaluation would differ from the
//                       previous step's second one (REF barostat moved the atoms,
//                       no forces yet, or the REF list cadence rebuilds now)
//   k_kick_drift        pending thermostat scale, half kick, PHYS pending
//                       barostat scale, drift, clear forces, write the sorted
//                       FP32/FP64 mirror, skin check (replicas with step < target)
//   [eval #2]           (its k_eval_begin marks the replicas that advance and
//                       scales the PHYS box to match the drift)
//   k_kick2             half kick (+ Andersen), per-tile KE / virial partials
//   k_replica_update    closes eval #2, KE, thermostat (Berendsen / Nose-Hoover
//                       scale, applied lazily in the next kick), Berendsen
//                       barostat factor (REF: applied now; PHYS: pending for the
//                       next drift)
//   k_apply_scale       REF barostat position scaling (only when a barostat exists)
// PHYS therefore evaluates forces once per step with or without a barostat:
// the first kick of a step uses the forces of the previous evaluation and the
// scaling is applied with the drift, so every evaluation sees the positions
// the next kick is for.
// Integration arithmetic is FP64 with the reference's operation order
// (src/integrate/integrator.cpp:4-20) and no FMA contraction.
#include "device.cuh"
#include "launch.h"

namespace dmd {

namespace {

__global__ void k_eval_begin(Dev d, int pass) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) {
        *d.nb_work = 0;
        if (d.nb_work_mi) *d.nb_work_mi = 0;
        d.grid_bar[0] = 0;  // arrivals (the generation word keeps counting)
    }
    if (r >= d.n_rep) return;
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    const bool ref_lj = !(R.flags & F_PHYS) && (R.flags & F_LJ);
    // which replicas advance this step (the host may have moved the targets)
    if (pass != PASS_SINGLE) s->active = (s->step < s->target_step) ? 1 : 0;
    // REF: the barostat scale of the previous step has been applied; PHYS keeps
    // its pending scale for k_kick_drift (positions) and the second pass (box),
    // so an evaluation before the drift sees the unscaled pair.
    if (pass == PASS_FIRST && !(R.flags & F_PHYS)) s->pscale = 1.0;
    int ev;
    if (pass == PASS_FIRST) {
        ev = s->active && ((R.barostat != 0 && !(R.flags & F_PHYS)) || !s->have_forces ||
                           (ref_lj && s->lj_counter >= 10));
        // LennardJones::compute advances its counter on every call (lennard_jones.cpp:91)
        if (s->active && !ev && ref_lj) s->lj_counter += 1;
    } else if (pass == PASS_SECOND) {
        ev = s->active;
        // consumed by k_kick_drift; a replica that has reached its target keeps
        // its pending thermostat scale for the next read of its velocities
        if (s->active) s->vscale = 1.0;
        if (s->active && (R.flags & F_PHYS) && s->pscale != 1.0) {
            // the box follows the positions k_kick_drift has just scaled
            s->L *= s->pscale;
            s->invL = 1.0 / s->L;
            s->pscale = 1.0;
        }
    } else {
        ev = 1;
    }
    s->eval = ev;
    s->green_ok = (s->green_L == s->L) ? 1 : 0;
    // Pair energies and the pair virial are needed by single-point evaluations,
    // by the evaluation that ends a run (its energies are what the host reads) and,
    // with the PHYS barostat, every step (its pressure uses the atomic virial).
    // Eval #1 never needs them: eval #2 of the same step overwrites its sums.
    s->want_e = (pass == PASS_SINGLE) ||
                (pass == PASS_SECOND && (s->step + 1 >= s->target_step || ((R.flags & F_PHYS) && R.barostat)));
    if (ev) {
        for (int k = 0; k < N_EACC; ++k) s->e_acc[k] = 0;
        s->e_recip = 0.0;
        s->vir_recip = 0.0;
        if (ref_lj && s->lj_counter >= 10) s->rebuild = 1;
    }
}

__global__ void k_eval_end(Dev d) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= d.n_rep) return;
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    if (!s->eval) return;
    if (!(R.flags & F_PHYS) && (R.flags & F_LJ)) s->lj_counter += 1;
    s->have_forces = 1;
    if (R.flags & F_PME) s->green_L = s->L;  // the influence kernel has filled the cache
}

__global__ void k_clear_forces(Dev d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.n_slots) {
        int r = d.tile_rep[i >> 5];
        if (d.st[r].eval) {
            d.fnx[i] = 0;
            d.fny[i] = 0;
            d.fnz[i] = 0;
        }
    }
    if (i < d.n_atoms) {
        int r = d.atom_rep[i];
        if (d.st[r].eval) {
            d.fbx[i] = 0;
            d.fby[i] = 0;
            d.fbz[i] = 0;
        }
    }
}

__device__ __forceinline__ void write_mirror(const Dev& d, int slot, int a, double x, double y, double z,
                                             double L) {
    if (d.xq32) {
        const int t = slot >> 5;
        d.xq32[slot] = make_float4(static_cast<float>((x - d.imgx[a] * L) - d.tcx[t]),
                                   static_cast<float>((y - d.imgy[a] * L) - d.tcy[t]),
                                   static_cast<float>((z - d.imgz[a] * L) - d.tcz[t]),
                                   static_cast<float>(d.q[a]));
    }
    if (d.xq64) d.xq64[slot] = make_double4(x, y, z, d.q[a]);
}

__device__ __forceinline__ void skin_check(const Dev& d, RepState* s, const Rep& R, int a, double x,
                                           double y, double z) {
    if (!(R.flags & F_PHYS)) return;
    const double dx = x - d.xr[a], dy = y - d.yr[a], dz = z - d.zr[a];
    if (dx * dx + dy * dy + dz * dz > R.half_skin2) s->rebuild = 1;
}

// Integrator::half_kick + advance (integrator.cpp:4-20), with the pending
// thermostat scale of the previous step applied first.  PHYS with a barostat:
// the pending position scale s (1 otherwise, an exact multiply) is applied
// before the drift, x <- s x + v dt, and the mirror is written for the box
// s L that k_eval_begin stores next.
// One thread per atom in reference order: the FP64 state, masses and bonded
// forces are read and written coalesced; only the pair forces and the mirror
// are addressed through the atom's slot.
__global__ void k_kick_drift(Dev d) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= d.n_atoms) return;
    const int r = d.atom_rep[a];
    RepState* s = d.st + r;
    if (!(s->step < s->target_step)) return;  // runs before this step's k_eval_begin
    const int slot = d.slot_of_atom[a];
    const Rep& R = d.rep[r];
    const double dt = R.dt, half_dt = 0.5 * dt;
    const double inv_mass = 1.0 / d.mass[a];
    const double lam = s->vscale;
    const double fx = from_fix(d.fnx[slot] + d.fbx[a], FSCALE);
    const double fy = from_fix(d.fny[slot] + d.fby[a], FSCALE);
    const double fz = from_fix(d.fnz[slot] + d.fbz[a], FSCALE);
    double vx = __dmul_rn(d.vx[a], lam), vy = __dmul_rn(d.vy[a], lam), vz = __dmul_rn(d.vz[a], lam);
    vx = __dadd_rn(vx, __dmul_rn(__dmul_rn(fx, inv_mass), half_dt));
    vy = __dadd_rn(vy, __dmul_rn(__dmul_rn(fy, inv_mass), half_dt));
    vz = __dadd_rn(vz, __dmul_rn(__dmul_rn(fz, inv_mass), half_dt));
    const double sc = s->pscale;
    const double x = __dadd_rn(__dmul_rn(d.x[a], sc), __dmul_rn(vx, dt));
    const double y = __dadd_rn(__dmul_rn(d.y[a], sc), __dmul_rn(vy, dt));
    const double z = __dadd_rn(__dmul_rn(d.z[a], sc), __dmul_rn(vz, dt));
    d.vx[a] = vx;
    d.vy[a] = vy;
    d.vz[a] = vz;
    d.x[a] = x;
    d.y[a] = y;
    d.z[a] = z;
    d.fnx[slot] = 0;
    d.fny[slot] = 0;
    d.fnz[slot] = 0;
    d.fbx[a] = 0;
    d.fby[a] = 0;
    d.fbz[a] = 0;
    write_mirror(d, slot, a, x, y, z, s->L * sc);
    skin_check(d, s, R, a, x, y, z);
}

// Philox4x32-10 (Salmon et al., SC'11) for the PHYS Andersen thermostat.
__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Second half kick, optional Andersen collisions, per-tile KE and r.F partials.
__global__ void k_kick2(Dev d, int andersen_ref, int andersen_phys) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int t = slot >> 5;
    const int r = (t < d.n_tiles) ? d.tile_rep[t] : 0;
    RepState* s = d.st + r;
    double ke = 0.0, w = 0.0;
    if (slot < d.n_slots && s->active) {
        const int a = d.atom_of_slot[slot];
        if (a >= 0) {
            const Rep& R = d.rep[r];
            const double half_dt = 0.5 * R.dt;
            const double m = d.mass[a];
            const double inv_mass = 1.0 / m;
            const double fx = from_fix(d.fnx[slot] + d.fbx[a], FSCALE);
            const double fy = from_fix(d.fny[slot] + d.fby[a], FSCALE);
            const double fz = from_fix(d.fnz[slot] + d.fbz[a], FSCALE);
            double vx = __dadd_rn(d.vx[a], __dmul_rn(__dmul_rn(fx, inv_mass), half_dt));
            double vy = __dadd_rn(d.vy[a], __dmul_rn(__dmul_rn(fy, inv_mass), half_dt));
            double vz = __dadd_rn(d.vz[a], __dmul_rn(__dmul_rn(fz, inv_mass), half_dt));
            if (R.thermostat == 3 && R.t_freq * R.dt > 0.0) {
                if (andersen_ref && d.and_flag && d.and_flag[a]) {
                    vx = d.and_v[3 * a];
                    vy = d.and_v[3 * a + 1];
                    vz = d.and_v[3 * a + 2];
                } else if (andersen_phys && (R.flags & F_PHYS)) {
                    const uint32_t call = static_cast<uint32_t>(s->andersen_calls);
                    const uint32_t callh = static_cast<uint32_t>(s->andersen_calls >> 32);
                    const uint32_t li = static_cast<uint32_t>(a - R.atom_begin);
                    uint32_t c[4] = {li, call, callh, 0x414E4400u};
                    philox(c, R.key0, R.key1);
                    const double u = c[0] * 2.3283064365386963e-10;
                    if (u < R.t_freq * R.dt) {
                        const double sg = sqrt(KB * R.t_temp / m);
                        const double u1 = (c[1] + 1.0) * 2.3283064365386963e-10;
                        const double u2 = c[2] * 2.3283064365386963e-10;
                        const double rr = sqrt(-2.0 * log(u1));
                        uint32_t e[4] = {li, call, callh, 0x414E4401u};
                        philox(e, R.key0, R.key1);
                        const double u3 = (e[0] + 1.0) * 2.3283064365386963e-10;
                        const double u4 = e[1] * 2.3283064365386963e-10;
                        vx = rr * cos(2.0 * PI * u2) * sg;
                        vy = rr * sin(2.0 * PI * u2) * sg;
                        vz = sqrt(-2.0 * log(u3)) * cos(2.0 * PI * u4) * sg;
                    }
                }
            }
            d.vx[a] = vx;
            d.vy[a] = vy;
            d.vz[a] = vz;
            // kinetic_energy (thermostat.cpp:6-15) and virial (barostat.cpp:6-14) terms
            ke = __dmul_rn(__dmul_rn(0.5, m),
                           __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz)));
            w = __dadd_rn(__dadd_rn(__dmul_rn(d.x[a], fx), __dmul_rn(d.y[a], fy)), __dmul_rn(d.z[a], fz));
        }
    }
    ke = warp_sum_d(ke);
    w = warp_sum_d(w);
    if (lane == 0 && t < d.n_tiles) {
        d.tile_ke[t] = ke;
        d.tile_vir[t] = w;
    }
}

// Constraints::apply (src/integrate/constraints.cpp:9-47) after the drift: one
// thread per group of constraints that share atoms (a molecule), its
// constraints swept in their given order until the group's largest
// |r^2 - d^2| (measured before each correction) is below the tolerance, at
// most 100 sweeps.  Groups share no atoms, so this is the reference's
// Gauss-Seidel sweep over all constraints, group by group.  The FP64
// operations follow the reference's order; the moved atoms' mirror entries
// are written again.  PHYS: the box is the drifted frame's (L times the
// pending barostat scale), and SHAKE's displacement is also given to the
// half-step velocities (v += dx / dt).
__global__ void k_shake(Dev d) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= d.n_cgroups) return;
    const int r = d.cgroup_rep[g];
    RepState* s = d.st + r;
    if (!(s->step < s->target_step)) return;  // the replicas k_kick_drift moved
    const Rep& R = d.rep[r];
    const bool phys = (R.flags & F_PHYS) != 0;
    const double L = phys ? s->L * s->pscale : s->L, inv = 1.0 / L, tol = R.cons_tol;
    const int c0 = d.cgroup_begin[g], c1 = d.cgroup_begin[g + 1];
    const int q0 = d.cgroup_atom_begin[g], q1 = d.cgroup_atom_begin[g + 1];
    const int na = d.n_atoms;
    if (phys)
        for (int q = q0; q < q1; ++q) {
            const int a = d.cgroup_atoms[q];
            d.cons_x0[a] = d.x[a];
            d.cons_x0[na + a] = d.y[a];
            d.cons_x0[2 * na + a] = d.z[a];
        }
    for (int it = 0; it < 100; ++it) {
        double worst = 0.0;
        for (int c = c0; c < c1; ++c) {
            const int a = d.cons_ij[c].x, b = d.cons_ij[c].y;
            double dx = __dsub_rn(d.x[b], d.x[a]), dy = __dsub_rn(d.y[b], d.y[a]), dz = __dsub_rn(d.z[b], d.z[a]);
            dx = __dsub_rn(dx, __dmul_rn(round(__dmul_rn(dx, inv)), L));
            dy = __dsub_rn(dy, __dmul_rn(round(__dmul_rn(dy, inv)), L));
            dz = __dsub_rn(dz, __dmul_rn(round(__dmul_rn(dz, inv)), L));
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double d2 = __dmul_rn(d.cons_d[c], d.cons_d[c]);
            const double err = __dsub_rn(r2, d2);
            if (fabs(err) > worst) worst = fabs(err);
            if (fabs(err) > tol) {
                const double wa = 1.0 / d.mass[a], wb = 1.0 / d.mass[b];
                const double lam = err / __dmul_rn(__dmul_rn(2.0, d2), __dadd_rn(wa, wb));
                d.x[a] = __dadd_rn(d.x[a], __dmul_rn(__dmul_rn(lam, dx), wa));
                d.y[a] = __dadd_rn(d.y[a], __dmul_rn(__dmul_rn(lam, dy), wa));
                d.z[a] = __dadd_rn(d.z[a], __dmul_rn(__dmul_rn(lam, dz), wa));
                d.x[b] = __dsub_rn(d.x[b], __dmul_rn(__dmul_rn(lam, dx), wb));
                d.y[b] = __dsub_rn(d.y[b], __dmul_rn(__dmul_rn(lam, dy), wb));
                d.z[b] = __dsub_rn(d.z[b], __dmul_rn(__dmul_rn(lam, dz), wb));
            }
        }
        if (worst < tol) break;
    }
    for (int q = q0; q < q1; ++q) {
        const int a = d.cgroup_atoms[q];
        const double x = d.x[a], y = d.y[a], z = d.z[a];
        if (phys) {
            d.vx[a] = __dadd_rn(d.vx[a], __dsub_rn(x, d.cons_x0[a]) / R.dt);
            d.vy[a] = __dadd_rn(d.vy[a], __dsub_rn(y, d.cons_x0[na + a]) / R.dt);
            d.vz[a] = __dadd_rn(d.vz[a], __dsub_rn(z, d.cons_x0[2 * na + a]) / R.dt);
        }
        write_mirror(d, d.slot_of_atom[a], a, x, y, z, L);
        skin_check(d, s, R, a, x, y, z);
    }
}

// Constraints::apply_rattle (constraints.cpp:49-91), after the second half
// kick: the same group sweeps on r.v, lambda = r.v / (r^2 (1/m_i + 1/m_j)).
__global__ void k_rattle(Dev d) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= d.n_cgroups) return;
    const int r = d.cgroup_rep[g];
    RepState* s = d.st + r;
    if (!s->active) return;
    const Rep& R = d.rep[r];
    const double L = s->L, inv = 1.0 / L, tol = R.cons_tol;
    const int c0 = d.cgroup_begin[g], c1 = d.cgroup_begin[g + 1];
    for (int it = 0; it < 100; ++it) {
        double worst = 0.0;
        for (int c = c0; c < c1; ++c) {
            const int a = d.cons_ij[c].x, b = d.cons_ij[c].y;
            double dx = __dsub_rn(d.x[b], d.x[a]), dy = __dsub_rn(d.y[b], d.y[a]), dz = __dsub_rn(d.z[b], d.z[a]);
            dx = __dsub_rn(dx, __dmul_rn(round(__dmul_rn(dx, inv)), L));
            dy = __dsub_rn(dy, __dmul_rn(round(__dmul_rn(dy, inv)), L));
            dz = __dsub_rn(dz, __dmul_rn(round(__dmul_rn(dz, inv)), L));
            const double dvx = __dsub_rn(d.vx[b], d.vx[a]), dvy = __dsub_rn(d.vy[b], d.vy[a]),
                         dvz = __dsub_rn(d.vz[b], d.vz[a]);
            const double rv = __dadd_rn(__dadd_rn(__dmul_rn(dx, dvx), __dmul_rn(dy, dvy)), __dmul_rn(dz, dvz));
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double e = fabs(rv);
            if (e > worst) worst = e;
            if (e > tol) {
                const double wa = 1.0 / d.mass[a], wb = 1.0 / d.mass[b];
                const double lam = rv / __dmul_rn(r2, __dadd_rn(wa, wb));
                d.vx[a] = __dadd_rn(d.vx[a], __dmul_rn(__dmul_rn(lam, dx), wa));
                d.vy[a] = __dadd_rn(d.vy[a], __dmul_rn(__dmul_rn(lam, dy), wa));
                d.vz[a] = __dadd_rn(d.vz[a], __dmul_rn(__dmul_rn(lam, dz), wa));
                d.vx[b] = __dsub_rn(d.vx[b], __dmul_rn(__dmul_rn(lam, dx), wb));
                d.vy[b] = __dsub_rn(d.vy[b], __dmul_rn(__dmul_rn(lam, dy), wb));
                d.vz[b] = __dsub_rn(d.vz[b], __dmul_rn(__dmul_rn(lam, dz), wb));
            }
        }
        if (worst < tol) break;
    }
}

// Per-tile kinetic-energy partials again after RATTLE (the thermostat reads the
// constrained velocities; same expression and order as k_kick2's).
__global__ void k_tile_ke(Dev d) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int t = slot >> 5;
    const int r = (t < d.n_tiles) ? d.tile_rep[t] : 0;
    double ke = 0.0;
    if (slot < d.n_slots && d.st[r].active) {
        const int a = d.atom_of_slot[slot];
        if (a >= 0) {
            const double m = d.mass[a], vx = d.vx[a], vy = d.vy[a], vz = d.vz[a];
            ke = __dmul_rn(__dmul_rn(0.5, m),
                           __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz)));
        }
    }
    ke = warp_sum_d(ke);
    if (lane == 0 && t < d.n_tiles) d.tile_ke[t] = ke;
}

__device__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

// PME energy / virial partial sums of replica r (fixed order).
__device__ void reduce_pme(const Dev& d, int r, double* sh) {
    const Rep& R = d.rep[r];
    double e = 0.0, v = 0.0;
    if (R.flags & F_PME) {
        for (int b = threadIdx.x; b < R.pme_blocks; b += blockDim.x) {
            e += d.pme_part[2 * (R.pme_block_begin + b)];
            v += d.pme_part[2 * (R.pme_block_begin + b) + 1];
        }
    }
    e = block_sum(e, sh);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        d.st[r].e_recip = e;
        d.st[r].vir_recip = v;
    }
}

__global__ void k_energy_reduce(Dev d) {
    __shared__ double sh[256];
    const int r = blockIdx.x;
    if (!d.st[r].eval) return;
    reduce_pme(d, r, sh);
}

// Four block-wide sums at once in a fixed order: lane sums by shuffles, then
// the block's warps in order by warp 0 (blockDim.x = 256).
__device__ void block_sum4(double v[4], double (*sh)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum_d(v[k]);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int k = 0; k < 4; ++k) sh[w][k] = v[k];
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < 4; ++k) {
            double x = (lane < nw) ? sh[lane][k] : 0.0;
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
            v[k] = x;
        }
    }
}

// Thermostat (berendsen.cpp:13-28, nose_hoover.cpp:6-32) and Berendsen barostat
// (berendsen_barostat.cpp:14-66); one block per replica.  Tile partials of KE
// and r.F and the PME blocks' energy / virial partials are summed together.
__global__ void k_replica_update(Dev d) {
    __shared__ double sh[8][4];
    const int r = blockIdx.x;
    RepState* s = d.st + r;
    if (!s->active) return;
    const Rep& R = d.rep[r];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = R.tile_begin + threadIdx.x; t < R.tile_begin + R.n_tiles; t += blockDim.x) {
        v[0] += d.tile_ke[t];
        v[1] += d.tile_vir[t];
    }
    if (R.flags & F_PME) {
        for (int b = threadIdx.x; b < R.pme_blocks; b += blockDim.x) {
            v[2] += d.pme_part[2 * (R.pme_block_begin + b)];
            v[3] += d.pme_part[2 * (R.pme_block_begin + b) + 1];
        }
    }
    block_sum4(v, sh);
    if (threadIdx.x != 0) return;
    // one thread from here: the replica's records are copied to registers at
    // once (independent loads) and written back at the end, instead of a chain
    // of dependent global reads and writes
    RepState st = *s;
    const Rep Rr = R;
    const double ke = v[0], w = v[1];
    st.e_recip = v[2];
    st.vir_recip = v[3];
    // end of the step's second evaluation (k_eval_end's work, at the box it used)
    if (st.eval) {
        if (!(Rr.flags & F_PHYS) && (Rr.flags & F_LJ)) st.lj_counter += 1;
        st.have_forces = 1;
        if (Rr.flags & F_PME) st.green_L = st.L;
    }
    const double n = static_cast<double>(Rr.n_atoms);
    const double dt = Rr.dt;
    auto temp = [&](double ek) { return Rr.n_atoms < 2 ? 0.0 : 2.0 * ek / ((3.0 * n - 3.0) * KB); };
    double lam = 1.0;
    if (Rr.thermostat == 1) {
        if (Rr.t_tau > 0.0 && ke > 0.0) {
            const double T = temp(ke);
            const double l = sqrt(1.0 + dt / Rr.t_tau * (Rr.t_temp / T - 1.0));
            if (!(l <= 0.0)) lam = l;
        }
    } else if (Rr.thermostat == 2) {
        const double T = temp(ke);
        st.zeta += 0.5 * dt * KB * (T - Rr.t_temp) / Rr.nh_Q;
        lam = exp(-st.zeta * 0.5 * dt);
    } else if (Rr.thermostat == 3) {
        if (Rr.t_freq * dt > 0.0) st.andersen_calls += 1;
    }
    st.vscale = lam;
    const double ke_after = ke * lam * lam;
    st.ke = ke_after;
    const double L = st.L;
    const double V = L * (L * L);
    double W;
    if (Rr.flags & F_PHYS) W = from_fix(st.e_acc[E_VIR], ESCALE) + st.vir_recip;
    else W = w;
    st.virial = W;
    st.pressure = (V <= 0.0) ? 0.0 : (2.0 * ke_after + W) / (3.0 * V);
    if (Rr.barostat == 2 && V > 0.0) {
        // AndersenBarostat::apply (andersen_barostat.cpp:20-45), ref profile: half a
        // step of piston velocity from 3V (P - P0) / W (P0 in the reference's units),
        // positions and box scale by exp(eps_dot dt) (positions in k_apply_scale),
        // then the second half step with the same forcing
        const double forcing = 3.0 * V * (st.pressure - Rr.b_pressure) / Rr.piston_W;
        st.eps_dot = st.eps_dot + 0.5 * dt * forcing;
        const double sc = exp(st.eps_dot * dt);
        st.pscale = sc;
        st.L = L * sc;
        st.invL = 1.0 / st.L;
        st.eps_dot = st.eps_dot + 0.5 * dt * forcing;
    }
    if (Rr.barostat == 1 && Rr.b_tau > 0.0 && V > 0.0) {
        double mu;
        if (Rr.flags & F_PHYS) mu = 1.0 - (dt / Rr.b_tau) * Rr.b_compress * (Rr.b_pressure - st.pressure / BAR);
        else mu = 1.0 - (dt / Rr.b_tau) * (Rr.b_compress / BAR) * (Rr.b_pressure - st.pressure);
        if (mu <= 0.0) mu = 0.0;
        const double sc = cbrt(mu);
        st.pscale = sc;
        if (!(Rr.flags & F_PHYS)) {  // REF: positions and box scale now (k_apply_scale)
            st.L = L * sc;
            st.invL = 1.0 / st.L;
        }
    }
    st.step += 1;
    st.time += dt;
    *s = st;
}

// BerendsenBarostat position scaling (berendsen_barostat.cpp:60-65).
__global__ void k_apply_scale(Dev d) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= d.n_slots) return;
    const int r = d.tile_rep[slot >> 5];
    RepState* s = d.st + r;
    if (!s->active || s->pscale == 1.0) return;
    const int a = d.atom_of_slot[slot];
    if (a < 0) return;
    const double sc = s->pscale;
    const double x = d.x[a] * sc, y = d.y[a] * sc, z = d.z[a] * sc;
    d.x[a] = x;
    d.y[a] = y;
    d.z[a] = z;
    write_mirror(d, slot, a, x, y, z, s->L);
    skin_check(d, s, d.rep[r], a, x, y, z);
}

__global__ void k_finalize_v(Dev d) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= d.n_atoms) return;
    const double lam = d.st[d.atom_rep[a]].vscale;
    if (lam == 1.0) return;
    d.vx[a] = __dmul_rn(d.vx[a], lam);
    d.vy[a] = __dmul_rn(d.vy[a], lam);
    d.vz[a] = __dmul_rn(d.vz[a], lam);
}

// One replica's frame into a device staging buffer, without changing any
// state: [step, time, box, x[n], y[n], z[n], vx[n], vy[n], vz[n]], the
// velocities with the pending thermostat scale applied as k_finalize_v would.
__global__ void k_frame_snapshot(Dev d, int r, double* out) {
    const Rep& R = d.rep[r];
    const RepState& s = d.st[r];
    const int n = R.n_atoms;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        out[0] = static_cast<double>(s.step);
        out[1] = s.time;
        out[2] = s.L;
    }
    if (i >= n) return;
    const int a = R.atom_begin + i;
    const double lam = s.vscale;
    double* o = out + 3;
    o[i] = d.x[a];
    o[n + i] = d.y[a];
    o[2 * n + i] = d.z[a];
    o[3 * n + i] = lam == 1.0 ? d.vx[a] : __dmul_rn(d.vx[a], lam);
    o[4 * n + i] = lam == 1.0 ? d.vy[a] : __dmul_rn(d.vy[a], lam);
    o[5 * n + i] = lam == 1.0 ? d.vz[a] : __dmul_rn(d.vz[a], lam);
}

__global__ void k_finalize_reset(Dev d) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < d.n_rep) d.st[r].vscale = 1.0;
}

__global__ void k_write_mirror(Dev d) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= d.n_slots) return;
    const int a = d.atom_of_slot[slot];
    if (a < 0) return;
    const int r = d.tile_rep[slot >> 5];
    write_mirror(d, slot, a, d.x[a], d.y[a], d.z[a], d.st[r].L);
}

}  // namespace

void launch_eval_begin(const Dev& d, int pass, cudaStream_t st, long long* n) {
    k_eval_begin<<<(d.n_rep + 127) / 128, 128, 0, st>>>(d, pass);
    ++*n;
}
void launch_clear_forces(const Dev& d, cudaStream_t st, long long* n) {
    const int m = d.n_slots > d.n_atoms ? d.n_slots : d.n_atoms;
    k_clear_forces<<<(m + 255) / 256, 256, 0, st>>>(d);
    ++*n;
}
void launch_eval_end(const Dev& d, cudaStream_t st, long long* n) {
    k_eval_end<<<(d.n_rep + 127) / 128, 128, 0, st>>>(d);
    ++*n;
}
void launch_kick_drift(const Dev& d, bool, cudaStream_t st, long long* n) {
    k_kick_drift<<<(d.n_atoms + 255) / 256, 256, 0, st>>>(d);
    ++*n;
}
void launch_kick2(const Dev& d, bool andersen_ref, bool andersen_phys, cudaStream_t st, long long* n) {
    k_kick2<<<(d.n_slots + 255) / 256, 256, 0, st>>>(d, andersen_ref ? 1 : 0, andersen_phys ? 1 : 0);
    ++*n;
}
void launch_shake(const Dev& d, cudaStream_t st, long long* n) {
    k_shake<<<(d.n_cgroups + 127) / 128, 128, 0, st>>>(d);
    ++*n;
}
void launch_rattle(const Dev& d, cudaStream_t st, long long* n) {
    k_rattle<<<(d.n_cgroups + 127) / 128, 128, 0, st>>>(d);
    k_tile_ke<<<(d.n_slots + 255) / 256, 256, 0, st>>>(d);
    *n += 2;
}
void launch_replica_update(const Dev& d, cudaStream_t st, long long* n) {
    k_replica_update<<<d.n_rep, 256, 0, st>>>(d);
    ++*n;
}
void launch_apply_scale(const Dev& d, bool, cudaStream_t st, long long* n) {
    k_apply_scale<<<(d.n_slots + 255) / 256, 256, 0, st>>>(d);
    ++*n;
}
void launch_finalize_velocities(const Dev& d, cudaStream_t st, long long* n) {
    k_finalize_v<<<(d.n_atoms + 255) / 256, 256, 0, st>>>(d);
    k_finalize_reset<<<(d.n_rep + 127) / 128, 128, 0, st>>>(d);
    *n += 2;
}
void launch_frame_snapshot(const Dev& d, int r, int n_atoms, double* out, cudaStream_t st, long long* n) {
    k_frame_snapshot<<<(n_atoms + 255) / 256, 256, 0, st>>>(d, r, out);
    ++*n;
}
void launch_energy_reduce(const Dev& d, cudaStream_t st, long long* n) {
    k_energy_reduce<<<d.n_rep, 256, 0, st>>>(d);
    ++*n;
}
void launch_write_mirror(const Dev& d, bool, cudaStream_t st, long long* n) {
    k_write_mirror<<<(d.n_slots + 255) / 256, 256, 0, st>>>(d);
    ++*n;
}

}  // namespace dmd
