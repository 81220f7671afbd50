// k_forces.cu -- bonded terms, exclusion correction and SPME kernels.
//
// Bonded: one thread per term; the bond vectors are formed in FP64 with the
// reference's minimum image, then the term is evaluated in `real` (FP32 in the
// mixed path).  REF formulas follow src/force/harmonic_bond.cpp:12-47,
// harmonic_angle.cpp:10-63 (force sign quirk kept), periodic_dihedral.cpp:10-137
// and harmonic_improper.cpp:10-130 (the reference's gradient vectors); PHYS
// uses -grad E.
//
// SPME (src/force/coulomb_pme.cpp): spread (order-4 B-spline, int64 fixed-point
// atomics onto the mesh), convert (fixed -> real, REF reinterprets the
// reference's unpadded-index grid through FFTW's padded in-place layout),
// cuFFT R2C, influence multiply + energy/virial, cuFFT C2R, gather.
#include "device.cuh"
#include "launch.h"

namespace dmd {

namespace {

// Energy/virial of one work item, reduced over lanes that share a replica.
__device__ __forceinline__ void add_energy(const Dev& d, int r, int term, long long e, long long v,
                                           bool valid) {
    const unsigned grp = __match_any_sync(FULL, valid ? r : -1);
    const int leader = __ffs(grp) - 1;
    long long es = 0, vs = 0;
    // sum within the group in lane order (integer: order does not matter)
    for (unsigned g = grp; g; g &= g - 1) {
        const int l = __ffs(g) - 1;
        es += __shfl_sync(grp, e, l);
        vs += __shfl_sync(grp, v, l);
    }
    if (valid && (threadIdx.x & 31) == leader) {
        if (es) fix_add(&d.st[r].e_acc[term], es);
        if (vs) fix_add(&d.st[r].e_acc[E_VIR], vs);
    }
}

template <typename T>
__device__ __forceinline__ void add_force(const Dev& d, int a, T fx, T fy, T fz, RepState* s) {
    fix_add(d.fbx + a, to_fix(fx, FSCALE, s));
    fix_add(d.fby + a, to_fix(fy, FSCALE, s));
    fix_add(d.fbz + a, to_fix(fz, FSCALE, s));
}

template <typename T, bool PHYS>
__device__ __forceinline__ void do_bond(const Dev& d, int n) {
    const bool in = n < d.n_bonds;
    int r = 0;
    long long ef = 0, vf = 0;
    bool valid = false;
    if (in) {
        const int2 ij = d.bond_ij[n];
        r = d.atom_rep[ij.x];
        RepState* s = d.st + r;
        if (s->eval) {
            valid = true;
            const double L = s->L, invL = s->invL;
            const double2 kr = d.bond_kr[n];
            const double ddx = mi_ref(__dsub_rn(d.x[ij.y], d.x[ij.x]), L, invL);
            const double ddy = mi_ref(__dsub_rn(d.y[ij.y], d.y[ij.x]), L, invL);
            const double ddz = mi_ref(__dsub_rn(d.z[ij.y], d.z[ij.x]), L, invL);
            // bond length and its deviation in FP64 (stiff bonds: r - r0 << r)
            const double rd = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            const T dx = (T)ddx, dy = (T)ddy, dz = (T)ddz;
            const T rr = (T)rd;
            const T r2 = (T)(rd * rd);
            const T dr = (T)(rd - kr.y);
            const T f = -(T)kr.x * dr / rr;
            add_force(d, ij.x, -f * dx, -f * dy, -f * dz, s);
            add_force(d, ij.y, f * dx, f * dy, f * dz, s);
            ef = to_fix(T(0.5) * (T)kr.x * dr * dr, ESCALE, s);
            vf = PHYS ? to_fix(f * r2, ESCALE, s) : 0;
        }
    }
    add_energy(d, r, E_BOND, ef, vf, valid);
}

template <typename T, bool PHYS>
__device__ __forceinline__ void do_angle(const Dev& d, int n) {
    int r = 0;
    long long ef = 0, vf = 0;
    bool valid = false;
    if (n < d.n_angles) {
        const int4 t = d.ang_ijk[n];
        r = d.atom_rep[t.x];
        RepState* s = d.st + r;
        if (s->eval) {
            valid = true;
            const double L = s->L, invL = s->invL;
            const double2 kt = d.ang_kt[n];
            const T x1 = (T)mi_ref(__dsub_rn(d.x[t.x], d.x[t.y]), L, invL);
            const T y1 = (T)mi_ref(__dsub_rn(d.y[t.x], d.y[t.y]), L, invL);
            const T z1 = (T)mi_ref(__dsub_rn(d.z[t.x], d.z[t.y]), L, invL);
            const T x2 = (T)mi_ref(__dsub_rn(d.x[t.z], d.x[t.y]), L, invL);
            const T y2 = (T)mi_ref(__dsub_rn(d.y[t.z], d.y[t.y]), L, invL);
            const T z2 = (T)mi_ref(__dsub_rn(d.z[t.z], d.z[t.y]), L, invL);
            const T r12 = x1 * x1 + y1 * y1 + z1 * z1;
            const T r22 = x2 * x2 + y2 * y2 + z2 * z2;
            const T ra = sqrt(r12), rb = sqrt(r22);
            T c = (x1 * x2 + y1 * y2 + z1 * z2) / (ra * rb);
            c = fmax(T(-1), fmin(T(1), c));
            const T th = acos(c);
            const T dth = th - (T)kt.y;
            // reference: f = -k dth / sin(theta); PHYS flips the sign (true -grad E)
            T f = -(T)kt.x * dth / sqrt(T(1) - c * c);
            if (PHYS) f = -f;
            const T iab = T(1) / (ra * rb);
            const T fx1 = f * (x2 * iab - c * x1 / r12), fy1 = f * (y2 * iab - c * y1 / r12),
                    fz1 = f * (z2 * iab - c * z1 / r12);
            const T fx2 = f * (x1 * iab - c * x2 / r22), fy2 = f * (y1 * iab - c * y2 / r22),
                    fz2 = f * (z1 * iab - c * z2 / r22);
            add_force(d, t.x, fx1, fy1, fz1, s);
            add_force(d, t.y, -(fx1 + fx2), -(fy1 + fy2), -(fz1 + fz2), s);
            add_force(d, t.z, fx2, fy2, fz2, s);
            ef = to_fix(T(0.5) * (T)kt.x * dth * dth, ESCALE, s);
            vf = PHYS ? to_fix(x1 * fx1 + y1 * fy1 + z1 * fz1 + x2 * fx2 + y2 * fy2 + z2 * fz2, ESCALE, s)
                      : 0;
        }
    }
    add_energy(d, r, E_ANGLE, ef, vf, valid);
}

// Torsions: PeriodicDihedral (periodic_dihedral.cpp:10-137) and, with IMP,
// HarmonicImproper (harmonic_improper.cpp:10-130).  Both measure the angle
// between the planes (i, j, k) and (j, k, l) as atan2 of the same clamped sine
// and cosine; the dihedral's energy is k (1 + cos(n phi - phi0)), the
// improper's k/2 (chi - chi0)^2 (chi - chi0 not wrapped, as in the reference).
// REF forces are the reference's gradient vectors times -dE/dangle; PHYS
// forces are -grad E.
template <typename T, bool PHYS, bool IMP>
__device__ __forceinline__ void do_torsion(const Dev& d, int n) {
    int r = 0;
    long long ef = 0, vf = 0;
    bool valid = false;
    if (n < (IMP ? d.n_imp : d.n_dih)) {
        const int4 q = IMP ? d.imp_ijkl[n] : d.dih_ijkl[n];
        r = d.atom_rep[q.x];
        RepState* s = d.st + r;
        if (s->eval) {
            valid = true;
            const double L = s->L, invL = s->invL;
            const T bax = (T)mi_ref(__dsub_rn(d.x[q.x], d.x[q.y]), L, invL);
            const T bay = (T)mi_ref(__dsub_rn(d.y[q.x], d.y[q.y]), L, invL);
            const T baz = (T)mi_ref(__dsub_rn(d.z[q.x], d.z[q.y]), L, invL);
            const T bcx = (T)mi_ref(__dsub_rn(d.x[q.z], d.x[q.y]), L, invL);
            const T bcy = (T)mi_ref(__dsub_rn(d.y[q.z], d.y[q.y]), L, invL);
            const T bcz = (T)mi_ref(__dsub_rn(d.z[q.z], d.z[q.y]), L, invL);
            const T dcx = (T)mi_ref(__dsub_rn(d.x[q.z], d.x[q.w]), L, invL);
            const T dcy = (T)mi_ref(__dsub_rn(d.y[q.z], d.y[q.w]), L, invL);
            const T dcz = (T)mi_ref(__dsub_rn(d.z[q.z], d.z[q.w]), L, invL);
            const T n1x = bay * bcz - baz * bcy, n1y = baz * bcx - bax * bcz, n1z = bax * bcy - bay * bcx;
            const T n2x = bcy * dcz - bcz * dcy, n2y = bcz * dcx - bcx * dcz, n2z = bcx * dcy - bcy * dcx;
            const T n1s = n1x * n1x + n1y * n1y + n1z * n1z;
            const T n2s = n2x * n2x + n2y * n2y + n2z * n2z;
            const T bcs = bcx * bcx + bcy * bcy + bcz * bcz;
            const T tiny = sizeof(T) == 8 ? T(1e-30) : T(1e-30);
            if (!(n1s < tiny || n2s < tiny || bcs < tiny)) {
                const T n1n = sqrt(n1s), n2n = sqrt(n2s), bcn = sqrt(bcs);
                T cph = (n1x * n2x + n1y * n2y + n1z * n2z) / (n1n * n2n);
                cph = fmax(T(-1), fmin(T(1), cph));
                const T trip = bcx * (n1y * n2z - n1z * n2y) + bcy * (n1z * n2x - n1x * n2z) +
                               bcz * (n1x * n2y - n1y * n2x);
                T sph = trip / (bcn * n1n * n2n);
                sph = fmax(T(-1), fmin(T(1), sph));
                const T phi = atan2(sph, cph);
                const int p = IMP ? 0 : d.dih_n[n];
                const double2 kp = IMP ? d.imp_kp[n] : d.dih_kp[n];
                const T k = (T)kp.x, phi0 = (T)kp.y;
                const T dphi = phi - phi0;                           // improper
                const T ncos = IMP ? T(0) : (T)(p * phi - phi0);    // dihedral
                ef = to_fix(IMP ? T(0.5) * k * dphi * dphi : k * (T(1) + cos(ncos)), ESCALE, s);
                if (!PHYS) {
                    const T pref = IMP ? -k * dphi : k * p * sin(ncos);
                    if (fabs(pref) >= tiny) {
                        const T gix = (bcy * n1z - bcz * n1y) / n1s, giy = (bcz * n1x - bcx * n1z) / n1s,
                                giz = (bcx * n1y - bcy * n1x) / n1s;
                        const T glx = -(bcy * n2z - bcz * n2y) / n2s, gly = -(bcz * n2x - bcx * n2z) / n2s,
                                glz = -(bcx * n2y - bcy * n2x) / n2s;
                        const T ax = n1y * baz - n1z * bay, ay = n1z * bax - n1x * baz, az = n1x * bay - n1y * bax;
                        const T cx = dcy * n2z - dcz * n2y, cy = dcz * n2x - dcx * n2z, cz = dcx * n2y - dcy * n2x;
                        const T gjx = ax / n1s + cx / n2s - gix, gjy = ay / n1s + cy / n2s - giy,
                                gjz = az / n1s + cz / n2s - giz;
                        const T bx = (bcy * n2z - bcz * n2y) / n2s, by = (bcz * n2x - bcx * n2z) / n2s,
                                bz = (bcx * n2y - bcy * n2x) / n2s;
                        const T gkx = bx - ax / n1s - cx / n2s, gky = by - ay / n1s - cy / n2s,
                                gkz = bz - az / n1s - cz / n2s;
                        add_force(d, q.x, pref * gix, pref * giy, pref * giz, s);
                        add_force(d, q.y, pref * gjx, pref * gjy, pref * gjz, s);
                        add_force(d, q.z, pref * gkx, pref * gky, pref * gkz, s);
                        add_force(d, q.w, pref * glx, pref * gly, pref * glz, s);
                    }
                } else {
                    const T dd = IMP ? k * dphi : -k * p * sin(ncos);  // dE/dphi
                    const T fix_ = -dd * bcn / n1s * n1x, fiy_ = -dd * bcn / n1s * n1y, fiz_ = -dd * bcn / n1s * n1z;
                    const T flx = dd * bcn / n2s * n2x, fly = dd * bcn / n2s * n2y, flz = dd * bcn / n2s * n2z;
                    const T pp = (bax * bcx + bay * bcy + baz * bcz) / bcs;
                    const T qq = (dcx * bcx + dcy * bcy + dcz * bcz) / bcs;
                    const T svx = pp * fix_ - qq * flx, svy = pp * fiy_ - qq * fly, svz = pp * fiz_ - qq * flz;
                    const T fjx = fix_ - svx, fjy = fiy_ - svy, fjz = fiz_ - svz;
                    const T fkx = flx + svx, fky = fly + svy, fkz = flz + svz;
                    add_force(d, q.x, fix_, fiy_, fiz_, s);
                    add_force(d, q.y, -fjx, -fjy, -fjz, s);
                    add_force(d, q.z, -fkx, -fky, -fkz, s);
                    add_force(d, q.w, flx, fly, flz, s);
                    vf = to_fix(bax * fix_ + bay * fiy_ + baz * fiz_ - bcx * fkx - bcy * fky - bcz * fkz +
                                    (bcx - dcx) * flx + (bcy - dcy) * fly + (bcz - dcz) * flz,
                                ESCALE, s);
                }
            }
        }
    }
    add_energy(d, r, IMP ? E_IMP : E_DIH, ef, vf, valid);
}

// CoulombExclusion (coulomb_exclusion.cpp:16-56).  REF: E -= k q q / r with the
// repulsive-Coulomb force; PHYS: E -= k q q erf(a r)/r with its gradient.
// Evaluated in FP64 in both precisions: like the Ewald self term, this O(N)
// correction is large (~1e2 kJ/mol per pair) and cancels against the
// reciprocal sum, so FP32 rounding here would dominate the total-energy error.
template <typename T, bool PHYS>
__device__ __forceinline__ void do_exclusion(const Dev& d, int n) {
    int r = 0;
    long long ef = 0, vf = 0;
    bool valid = false;
    if (n < d.n_excl) {
        const int2 p = d.excl[n];
        r = d.atom_rep[p.x];
        RepState* s = d.st + r;
        const Rep& R = d.rep[r];
        if (s->eval && (R.flags & F_EXCL)) {
            valid = true;
            const double L = s->L, invL = s->invL;
            const T dx = (T)mi_ref(__dsub_rn(d.x[p.y], d.x[p.x]), L, invL);
            const T dy = (T)mi_ref(__dsub_rn(d.y[p.y], d.y[p.x]), L, invL);
            const T dz = (T)mi_ref(__dsub_rn(d.z[p.y], d.z[p.x]), L, invL);
            const T r2 = dx * dx + dy * dy + dz * dz;
            const T rr = sqrt(r2);
            const T qq = (T)(KE * d.q[p.x] * d.q[p.y]);
            T f, e;
            if (!PHYS) {
                f = qq / (r2 * rr);
                e = qq / rr;
            } else {
                const T a = (T)R.alpha;
                const T erf_ar = erf(a * rr);
                const T g = T(1.1283791670955125739) * a * exp(-a * a * r2);
                f = qq * (g / r2 - erf_ar / (r2 * rr));
                e = qq * erf_ar / rr;
            }
            add_force(d, p.x, -f * dx, -f * dy, -f * dz, s);
            add_force(d, p.y, f * dx, f * dy, f * dz, s);
            ef = to_fix(-e, ESCALE, s);
            vf = PHYS ? to_fix(f * r2, ESCALE, s) : 0;
        }
    }
    add_energy(d, r, E_CEXCL, ef, vf, valid);
}

// Fractional mesh coordinate as in spread_charges (coulomb_pme.cpp:93-112): the
// position is divided by L, wrapped with floor, scaled by K; FP64.
__device__ __forceinline__ int wrap_mesh(int g, int K) {
    g += (g < 0) ? K : 0;
    return g - ((g >= K) ? K : 0);
}

// The first stencil index m0 always lies in [-1, K - 1] (u = K when f - floor(f)
// rounds up to 1): a coordinate that is not finite (a NaN or infinite
// position) gives m0 = -1 and a non-finite u (its weights are then NaN and the
// caller flags the status word), so no float-to-integer conversion of a
// non-finite value ever becomes an index.  Returns whether u is finite.
__device__ __forceinline__ bool mesh_coord(double x, double invL, int K, int& m0, double& u) {
    double f = x * invL;
    f -= floor(f);
    u = f * K;
    const double fl = floor(u);
    const bool ok = fl >= 0.0 && fl <= static_cast<double>(K);
    m0 = ok ? static_cast<int>(fl) - 1 : -1;
    return ok;
}

// 16 threads per atom: thread (iy, ix) = (sub >> 2, sub & 3) adds the atom's
// 4 mesh points along z at (x, y).  A warp instruction then covers 4
// consecutive x of 8 rows, so the L2 sees a few contiguous sectors per
// instruction instead of 32 scattered ones.  Each contribution is rounded to
// the fixed-point mesh on its own; the integer sums do not depend on order.
template <typename T>
__global__ void k_pme_spread(Dev d) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int a = static_cast<int>(t >> 4);
    if (a >= d.n_atoms) return;
    const int r = d.atom_rep[a];
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    if (!s->eval || !(R.flags & F_PME)) return;
    const double q = d.q[a];
    if (q == 0.0) return;
    const int K = R.pme_K;
    const int ix = threadIdx.x & 3, iy = (threadIdx.x >> 2) & 3;
    int m0[3];
    double u[3];
    const bool fin = mesh_coord(d.x[a], s->invL, K, m0[0], u[0]) & mesh_coord(d.y[a], s->invL, K, m0[1], u[1]) &
                     mesh_coord(d.z[a], s->invL, K, m0[2], u[2]);
    if (!fin && (threadIdx.x & 15) == 0) set_status(s, ST_NAN);
    const T wx = theta4<T>((T)(u[0] - (m0[0] + ix)));
    const T wy = theta4<T>((T)(u[1] - (m0[1] + iy)));
    long long* mesh = d.mesh_fix + R.mesh_fix_off;
    const T qt = (T)q;
    const T qwx = qt * wx;
    // m0 + j lies in [-1, K + 2]: one conditional wrap per index.  grid_[gz*ny*nx +
    // gy*nx + gx] (coulomb_pme.cpp:131); the REF buffer is K*K*2(K/2+1) long, the
    // PHYS one K^3: the index is the same.
    const int gx = wrap_mesh(m0[0] + ix, K), gy = wrap_mesh(m0[1] + iy, K);
#pragma unroll
    for (int iz = 0; iz < 4; ++iz) {
        const T wz = theta4<T>((T)(u[2] - (m0[2] + iz)));
        const int gz = wrap_mesh(m0[2] + iz, K);
        const long long idx = (static_cast<long long>(gz) * K + gy) * K + gx;
        fix_add(mesh + idx, __double2ll_rn(static_cast<double>(qwx * (wy * wz)) * MSCALE));
    }
}

// Fixed-point mesh -> real FFT input (K^3, natural layout); clears the fixed mesh.
// REF: the FFT reads FFTW's padded in-place rows, i.e. element (z,y,x) of the real
// array is fixed[(z*K + y)*P + x] with P = 2(K/2+1).
// Each block converts 1,024 points of one replica's mesh (the block -> replica
// table is built at packing), four consecutive points per thread: 16-byte loads
// and stores where the group lies inside a PHYS mesh.  Replicas that do not
// evaluate this pass hold a zero mesh, so converting it is harmless and no
// per-replica test delays the loads.
template <typename T>
__global__ void k_pme_convert(Dev d) {
    const int r = d.conv_block_rep[blockIdx.x];
    const Rep& R = d.rep[r];
    const int loc0 = 1024 * (blockIdx.x - R.conv_block_begin) + 4 * threadIdx.x;
    if (loc0 >= R.mesh_fix_n) return;
    long long* fix = d.mesh_fix + R.mesh_fix_off;
    T* real = reinterpret_cast<T*>(d.mesh_real) + R.mesh_real_off;
    if ((R.flags & F_PHYS) && loc0 + 4 <= R.mesh_fix_n) {
        longlong2* src = reinterpret_cast<longlong2*>(fix + loc0);
        const longlong2 a = src[0], b = src[1];
        src[0] = make_longlong2(0, 0);
        src[1] = make_longlong2(0, 0);
        const T v0 = static_cast<T>(static_cast<double>(a.x) * (1.0 / MSCALE));
        const T v1 = static_cast<T>(static_cast<double>(a.y) * (1.0 / MSCALE));
        const T v2 = static_cast<T>(static_cast<double>(b.x) * (1.0 / MSCALE));
        const T v3 = static_cast<T>(static_cast<double>(b.y) * (1.0 / MSCALE));
        if (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(real + loc0) = make_float4(v0, v1, v2, v3);
        } else {
            reinterpret_cast<double2*>(real + loc0)[0] = make_double2(v0, v1);
            reinterpret_cast<double2*>(real + loc0)[1] = make_double2(v2, v3);
        }
        return;
    }
    const int K = R.pme_K;
    for (int j = 0; j < 4 && loc0 + j < R.mesh_fix_n; ++j) {
        const int loc = loc0 + j;  // meshes are < 2^31 points
        const long long v = fix[loc];
        fix[loc] = 0;
        const T val = static_cast<T>(static_cast<double>(v) * (1.0 / MSCALE));
        if (R.flags & F_PHYS) {
            real[loc] = val;  // natural layout, same index
        } else {
            const int pitch = 2 * (K / 2 + 1);
            const int row = loc / pitch;
            const int col = loc - row * pitch;
            if (col < K) real[static_cast<long long>(row) * K + col] = val;
        }
    }
}

// Green's function multiply and reciprocal energy/virial
// (compute_reciprocal_energy_and_potential, coulomb_pme.cpp:143-201).
// The influence function G depends only on the box, alpha and K: it is cached
// (rounded to T) and recomputed only when the box edge changed (barostat, state
// load).  Energy and virial sums are formed only when this evaluation's
// energies are read.
template <typename T>
__global__ void k_pme_influence(Dev d) {
    const int r = d.pme_block_rep[blockIdx.x];
    const Rep& R = d.rep[r];
    RepState* s = d.st + r;
    if (!s->eval) return;  // uniform over the block
    const int lb = blockIdx.x - R.pme_block_begin;
    const int K = R.pme_K, H = K / 2 + 1;
    const int nc = K * K * H;
    const int e = lb * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x);
    const bool want_e = s->want_e != 0;
    double en = 0.0, vr = 0.0;
    if (e < nc) {
        using C2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
        C2* cm = reinterpret_cast<C2*>(d.mesh_cplx) + R.mesh_cplx_off;
        T* gc = reinterpret_cast<T*>(d.pme_green) + R.mesh_cplx_off;
        const int kx = e % H;
        const int ky = (e / H) % K;
        const int kz = e / (H * K);
        const int mx = kx, my = (ky <= K / 2) ? ky : ky - K, mz = (kz <= K / 2) ? kz : kz - K;
        if (mx == 0 && my == 0 && mz == 0) {
            if (R.flags & F_PHYS) cm[e] = C2{0, 0};
        } else {
            const double L = s->L;
            double k2 = 0.0;
            if (!s->green_ok || want_e) {
                const double msq = (static_cast<double>(mx) * mx) / (L * L) +
                                   (static_cast<double>(my) * my) / (L * L) +
                                   (static_cast<double>(mz) * mz) / (L * L);
                k2 = 4.0 * PI * PI * msq;
            }
            T green;
            if (s->green_ok) {
                green = gc[e];
            } else {
                const double V = L * (L * L);
                const double* b = d.bsp + R.bsp_off;
                const double B = b[kx] * b[ky] * b[kz];
                green = static_cast<T>(4.0 * PI * KE / V * exp(-k2 / (4.0 * R.alpha * R.alpha)) * B / k2);
                gc[e] = green;
            }
            const C2 z = cm[e];
            if (want_e) {
                const double w = (kx == 0 || (K % 2 == 0 && kx == K / 2)) ? 1.0 : 2.0;
                const double re = z.x, im = z.y;
                const double ek = 0.5 * w * static_cast<double>(green) * (re * re + im * im);
                en = ek;
                vr = ek * (1.0 - k2 / (2.0 * R.alpha * R.alpha));
            }
            cm[e] = C2{z.x * green, z.y * green};
        }
    }
    if (!want_e) return;  // uniform over the block
    // deterministic block reduction (fixed tree)
    __shared__ double se[256], sv[256];
    se[threadIdx.x] = en;
    sv[threadIdx.x] = vr;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            se[threadIdx.x] += se[threadIdx.x + o];
            sv[threadIdx.x] += sv[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.pme_part[2 * blockIdx.x] = se[0];
        d.pme_part[2 * blockIdx.x + 1] = sv[0];
    }
}

// interpolate_forces (coulomb_pme.cpp:205-283).  REF reads the potential with
// the unpadded index from FFTW's padded buffer (padding reads as zero) and
// scales it by 1/N (:303-306); PHYS reads the natural layout, unscaled.
// 4 threads per atom: thread iz sums its (y, x) slice of the 4x4x4 stencil,
// rows of 4 adjacent x at a time, then the atom's 4 lanes reduce in a fixed
// order.  The x and y weights are computed once per thread.
template <typename T>
__global__ void k_pme_gather(Dev d) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int a = static_cast<int>(t >> 2);
    // every condition below is uniform over the atom's 4 lanes
    if (a >= d.n_atoms) return;
    const int r = d.atom_rep[a];
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    if (!s->eval || !(R.flags & F_PME)) return;
    const double q = d.q[a];
    if (q == 0.0) return;
    const int K = R.pme_K;
    const bool phys = (R.flags & F_PHYS) != 0;
    const int P = 2 * (K / 2 + 1);
    const double norm = 1.0 / (static_cast<double>(K) * K * K);
    const int iz = threadIdx.x & 3;
    int m0[3];
    double u[3];
    mesh_coord(d.x[a], s->invL, K, m0[0], u[0]);
    mesh_coord(d.y[a], s->invL, K, m0[1], u[1]);
    mesh_coord(d.z[a], s->invL, K, m0[2], u[2]);
    T wx[4], dwx[4], wy[4], dwy[4];
    int xs[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const T tx = (T)(u[0] - (m0[0] + j)), ty = (T)(u[1] - (m0[1] + j));
        wx[j] = theta4<T>(tx);
        dwx[j] = dtheta4<T>(tx);
        wy[j] = theta4<T>(ty);
        dwy[j] = dtheta4<T>(ty);
        xs[j] = wrap_mesh(m0[0] + j, K);
    }
    const T tz = (T)(u[2] - (m0[2] + iz));
    const T wz = theta4<T>(tz), dwz = dtheta4<T>(tz);
    const T* real = reinterpret_cast<const T*>(d.mesh_real) + R.mesh_real_off;
    const int z = wrap_mesh(m0[2] + iz, K);
    T gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int iy = 0; iy < 4; ++iy) {
        const int y = wrap_mesh(m0[1] + iy, K);
        const int row = (z * K + y) * K;
        T sd = 0, sw = 0;  // the row's sums of phi * dtheta_x and phi * theta_x
#pragma unroll
        for (int ix = 0; ix < 4; ++ix) {
            const int lin = row + xs[ix];
            T phi;
            if (phys) {
                phi = real[lin];
            } else {
                const int rr = lin / P;
                const int col = lin - rr * P;
                phi = (col < K) ? (T)(static_cast<double>(real[rr * K + col]) * norm) : T(0);
            }
            sd += phi * dwx[ix];
            sw += phi * wx[ix];
        }
        gx += sd * wy[iy];
        gy += sw * dwy[iy];
        gz += sw * wy[iy];
    }
    gx *= wz;
    gy *= wz;
    gz *= dwz;
    const unsigned grp = 0xFu << (threadIdx.x & 28);
#pragma unroll
    for (int o = 2; o > 0; o >>= 1) {
        gx += __shfl_xor_sync(grp, gx, o);
        gy += __shfl_xor_sync(grp, gy, o);
        gz += __shfl_xor_sync(grp, gz, o);
    }
    if (iz == 0) {
        const T fac = (T)(static_cast<double>(K) * s->invL);
        const T qt = (T)q;
        add_force(d, a, -qt * fac * gx, -qt * fac * gy, -qt * fac * gz, s);
    }
}

// One launch for every bonded-type term: blocks [0, nb) bonds, then angles,
// dihedrals, impropers and exclusion pairs (exclusions always in FP64, see
// do_exclusion).
template <typename T, bool PHYS>
__global__ void k_bonded(Dev d, int nb, int na, int nd, int ni) {
    int b = blockIdx.x;
    if (b < nb) { do_bond<T, PHYS>(d, b * blockDim.x + threadIdx.x); return; }
    b -= nb;
    if (b < na) { do_angle<T, PHYS>(d, b * blockDim.x + threadIdx.x); return; }
    b -= na;
    if (b < nd) { do_torsion<T, PHYS, false>(d, b * blockDim.x + threadIdx.x); return; }
    b -= nd;
    if (b < ni) { do_torsion<T, PHYS, true>(d, b * blockDim.x + threadIdx.x); return; }
    b -= ni;
    do_exclusion<double, PHYS>(d, b * blockDim.x + threadIdx.x);
}

}  // namespace

void launch_bonded(const Dev& d, bool fp64, bool phys, cudaStream_t st, long long* nlaunch) {
    const int T = 256;
    const int nb = (d.n_bonds + T - 1) / T, na = (d.n_angles + T - 1) / T, nd = (d.n_dih + T - 1) / T,
              ni = (d.n_imp + T - 1) / T, ne = (d.n_excl + T - 1) / T;
    const int g = nb + na + nd + ni + ne;
    if (g == 0) return;
    if (fp64) {
        if (phys) k_bonded<double, true><<<g, T, 0, st>>>(d, nb, na, nd, ni);
        else k_bonded<double, false><<<g, T, 0, st>>>(d, nb, na, nd, ni);
    } else {
        if (phys) k_bonded<float, true><<<g, T, 0, st>>>(d, nb, na, nd, ni);
        else k_bonded<float, false><<<g, T, 0, st>>>(d, nb, na, nd, ni);
    }
    ++*nlaunch;
}

void launch_pme_spread(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch) {
    const int T = 256, g = static_cast<int>((16LL * d.n_atoms + T - 1) / T);
    if (fp64) k_pme_spread<double><<<g, T, 0, st>>>(d);
    else k_pme_spread<float><<<g, T, 0, st>>>(d);
    ++*nlaunch;
}

void launch_pme_convert(const Dev& d, bool fp64, int n_blocks, cudaStream_t st, long long* nlaunch) {
    if (n_blocks <= 0) return;
    if (fp64) k_pme_convert<double><<<n_blocks, 256, 0, st>>>(d);
    else k_pme_convert<float><<<n_blocks, 256, 0, st>>>(d);
    ++*nlaunch;
}

void launch_pme_influence(const Dev& d, bool fp64, int n_blocks, cudaStream_t st, long long* nlaunch) {
    if (fp64) k_pme_influence<double><<<n_blocks, 256, 0, st>>>(d);
    else k_pme_influence<float><<<n_blocks, 256, 0, st>>>(d);
    ++*nlaunch;
}

void launch_pme_gather(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch) {
    const int T = 256, g = static_cast<int>((4LL * d.n_atoms + T - 1) / T);
    if (fp64) k_pme_gather<double><<<g, T, 0, st>>>(d);
    else k_pme_gather<float><<<g, T, 0, st>>>(d);
    ++*nlaunch;
}

}  // namespace dmd
