// k_nonbonded.cu -- Lennard-Jones + real-space Ewald pair forces over the chunk list.
//
// Replaces LennardJones::compute (src/force/lennard_jones.cpp:43-92) and
// CoulombDirect::compute (src/force/coulomb_direct.cpp:38-86).  One warp per
// chunk: lane i holds i-atom i of the tile; the chunk's 32 j atoms are staged
// in shared memory and visited in a rotated order ((lane + k) & 31) so every
// lane touches a different j at each of the 32 steps; the j forces rotate with
// warp shuffles and are flushed once per chunk, i forces once per chunk.
// Forces go to int64 fixed point (deterministic), energies/virial to per-lane
// int64 accumulators flushed per warp.
//
// Precision
//  * mixed: tile-local FP32 coordinates (|x| < ~1 nm) plus the FP64 tile-center
//    offset rounded once per j, FP32 arithmetic; a pair whose r^2 lies within
//    1e-5 relative of a cutoff is re-tested with the FP64 reference expression,
//    so the interacting set is exactly the reference's.
//  * fp64: unwrapped FP64 coordinates with the reference's minimum image and
//    LJ operation order, no FMA contraction in the per-pair force.
#include "device.cuh"
#include "launch.h"

namespace dmd {

namespace {

constexpr float TWO_OVER_SQRTPI_F = 1.1283791670955126f;
constexpr double TWO_OVER_SQRTPI = 1.1283791670955125739;

struct Acc {
    long long lj, c, v;
};

// erfc(x) for x >= 0 given e = exp(-x*x): Abramowitz & Stegun, Handbook of
// Mathematical Functions, eq. 7.1.26 (absolute error <= 1.5e-7).
__device__ __forceinline__ float erfc_as(float x, float e) {
    const float t = __fdividef(1.0f, fmaf(0.3275911f, x, 1.0f));
    const float p = fmaf(fmaf(fmaf(fmaf(1.061405429f, t, -1.453152027f), t, 1.421413741f), t,
                              -0.284496736f), t, 0.254829592f);
    return t * p * e;
}

__device__ __forceinline__ void flush_acc(const Dev& d, int r, Acc& acc) {
    long long lj = warp_sum_ll(acc.lj), c = warp_sum_ll(acc.c), v = warp_sum_ll(acc.v);
    if ((threadIdx.x & 31) == 0 && r >= 0) {
        if (lj) fix_add(&d.st[r].e_acc[E_LJ], lj);
        if (c) fix_add(&d.st[r].e_acc[E_CREAL], c);
        if (v) fix_add(&d.st[r].e_acc[E_VIR], v);
    }
    acc.lj = acc.c = acc.v = 0;
}

// Exact reference membership of (ai, aj) for cutoff^2 rc2.
__device__ __forceinline__ bool exact_inside(const Dev& d, int ai, int aj, double L, double invL,
                                             double rc2) {
    double dx = mi_ref(__dsub_rn(d.x[aj], d.x[ai]), L, invL);
    double dy = mi_ref(__dsub_rn(d.y[aj], d.y[ai]), L, invL);
    double dz = mi_ref(__dsub_rn(d.z[aj], d.z[ai]), L, invL);
    return r2_ref(dx, dy, dz) < rc2;
}

template <bool PHYS>
__global__ void __launch_bounds__(256) k_nb_f32(Dev d) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    __shared__ float4 s_xj[8][32];
    __shared__ int s_tj[8][32];
    __shared__ int s_aj[8][32];
    __shared__ uint32_t s_mk[8][32];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int total = d.chunk_prefix[d.n_rep];
    Acc acc{0, 0, 0};
    int cur = -1;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += nw) {
        const int r = chunk_replica(d.chunk_prefix, d.n_rep, w);
        if (r != cur) {
            flush_acc(d, cur, acc);
            cur = r;
        }
        RepState* s = d.st + r;
        if (!s->eval) continue;
        const Rep& R = d.rep[r];
        const int c = R.chunk_begin + (w - d.chunk_prefix[r]);
        const double L = s->L, invL = s->invL;
        const int I = d.chunk_itile[c];
        const int si = 32 * I + lane;
        const float4 xi = d.xq32[si];
        const int ti = d.type_s[si];
        const uint32_t e = d.chunk_j[32 * c + lane];
        const uint32_t mk = d.chunk_mask[32 * c + lane];
        const int js = static_cast<int>(e & 0x03FFFFFFu);
        float4 xj = make_float4(1e6f, 1e6f, 1e6f, 0.f);
        int tj = 0, aj = -1;
        if (mk) {
            xj = d.xq32[js];
            tj = d.type_s[js];
            aj = d.atom_of_slot[js];
            const int J = js >> 5;
            const int mx = static_cast<int>((e >> 26) & 3u) - 1;
            const int my = static_cast<int>((e >> 28) & 3u) - 1;
            const int mz = static_cast<int>((e >> 30) & 3u) - 1;
            xj.x += static_cast<float>(d.tcx[J] - d.tcx[I] + mx * L);
            xj.y += static_cast<float>(d.tcy[J] - d.tcy[I] + my * L);
            xj.z += static_cast<float>(d.tcz[J] - d.tcz[I] + mz * L);
        }
        s_xj[wib][lane] = xj;
        s_tj[wib][lane] = tj;
        s_aj[wib][lane] = aj;
        s_mk[wib][lane] = mk;
        __syncwarp();
        const int ai = d.atom_of_slot[si];
        const bool has_lj = (R.flags & F_LJ) != 0;
        const bool has_c = PHYS && (R.flags & F_COUL_REAL) != 0;
        // a term that is absent gets a cutoff of 0 so its test is always false
        const float rl2 = has_lj ? static_cast<float>(R.rc_lj2) : 0.f;
        const float rcc2 = has_c ? static_cast<float>(R.rc_c2) : 0.f;
        const float bl_lo = rl2 * (1.f - 1e-5f), bl_hi = rl2 * (1.f + 1e-5f);
        const float bc_lo = rcc2 * (1.f - 1e-5f), bc_hi = rcc2 * (1.f + 1e-5f);
        const float alpha = static_cast<float>(R.alpha);
        const float a2l2e = -alpha * alpha * 1.4426950408889634f;  // -alpha^2 log2(e)
        const float keqi = static_cast<float>(KE) * xi.w;
        const float2* lj = d.lj32 + R.lj_off + ti * R.n_types;
        float fix = 0.f, fiy = 0.f, fiz = 0.f;
        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
        float el = 0.f, ec = 0.f, vir = 0.f;
#pragma unroll 2
        for (int k = 0; k < 32; ++k) {
            const int src = (lane + k) & 31;
            const uint32_t m = s_mk[wib][src];
            if ((m >> lane) & 1u) {
                const float4 pj = s_xj[wib][src];
                const float dx = pj.x - xi.x, dy = pj.y - xi.y, dz = pj.z - xi.z;
                const float r2 = dx * dx + dy * dy + dz * dz;
                bool in_l = r2 < rl2;
                bool in_c = r2 < rcc2;
                if ((r2 > bl_lo && r2 < bl_hi) || (r2 > bc_lo && r2 < bc_hi)) {
                    // within 1e-5 of a cutoff: the reference's FP64 test decides
                    const int aj2 = s_aj[wib][src];
                    if (has_lj) in_l = exact_inside(d, ai, aj2, L, invL, R.rc_lj2);
                    if (has_c) in_c = exact_inside(d, ai, aj2, L, invL, R.rc_c2);
                }
                float f = 0.f;
                const float rinv = rsqrtf(r2);
                const float ir2 = rinv * rinv;
                if (in_l) {
                    const float2 p = lj[s_tj[wib][src]];
                    const float ir6 = ir2 * ir2 * ir2;
                    const float c12 = p.y * ir6;
                    f += (12.f * c12 - 6.f * p.x) * ir6 * ir2;
                    el += (c12 - p.x) * ir6;
                }
                if (in_c) {
                    const float qq = keqi * pj.w;
                    const float ar = alpha * (r2 * rinv);
                    const float ex = exp2f(a2l2e * r2);
                    const float erfc_ar = erfc_as(ar, ex);
                    f += qq * (erfc_ar * rinv + TWO_OVER_SQRTPI_F * alpha * ex) * ir2;
                    ec += qq * erfc_ar * rinv;
                }
                vir += f * r2;
                fix -= f * dx;
                fiy -= f * dy;
                fiz -= f * dz;
                fjx += f * dx;
                fjy += f * dy;
                fjz += f * dz;
            }
            fjx = __shfl_sync(FULL, fjx, (lane + 1) & 31);
            fjy = __shfl_sync(FULL, fjy, (lane + 1) & 31);
            fjz = __shfl_sync(FULL, fjz, (lane + 1) & 31);
        }
        // after 32 rotations lane l again holds the forces of entry l
        if (ai >= 0) {
            fix_add(d.fnx + si, to_fix(fix, FSCALE, s));
            fix_add(d.fny + si, to_fix(fiy, FSCALE, s));
            fix_add(d.fnz + si, to_fix(fiz, FSCALE, s));
        }
        if (mk) {
            fix_add(d.fnx + js, to_fix(fjx, FSCALE, s));
            fix_add(d.fny + js, to_fix(fjy, FSCALE, s));
            fix_add(d.fnz + js, to_fix(fjz, FSCALE, s));
        }
        acc.lj += to_fix(el, ESCALE, s);
        acc.c += to_fix(ec, ESCALE, s);
        acc.v += to_fix(vir, ESCALE, s);
        __syncwarp();
    }
    flush_acc(d, cur, acc);
}

template <bool PHYS>
__global__ void __launch_bounds__(256) k_nb_f64(Dev d) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    __shared__ double4 s_xj[8][32];
    __shared__ int s_tj[8][32];
    __shared__ uint32_t s_mk[8][32];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int total = d.chunk_prefix[d.n_rep];
    Acc acc{0, 0, 0};
    int cur = -1;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += nw) {
        const int r = chunk_replica(d.chunk_prefix, d.n_rep, w);
        if (r != cur) {
            flush_acc(d, cur, acc);
            cur = r;
        }
        RepState* s = d.st + r;
        if (!s->eval) continue;
        const Rep& R = d.rep[r];
        const int c = R.chunk_begin + (w - d.chunk_prefix[r]);
        const double L = s->L, invL = s->invL;
        const int I = d.chunk_itile[c];
        const int si = 32 * I + lane;
        const double4 xi = d.xq64[si];
        const int ti = d.type_s[si];
        const uint32_t e = d.chunk_j[32 * c + lane];
        const uint32_t mk = d.chunk_mask[32 * c + lane];
        const int js = static_cast<int>(e & 0x03FFFFFFu);
        double4 xj = make_double4(0, 0, 0, 0);
        int tj = 0;
        if (mk) {
            xj = d.xq64[js];
            tj = d.type_s[js];
        }
        s_xj[wib][lane] = xj;
        s_tj[wib][lane] = tj;
        s_mk[wib][lane] = mk;
        __syncwarp();
        const bool has_lj = (R.flags & F_LJ) != 0;
        const bool has_c = PHYS && (R.flags & F_COUL_REAL) != 0;
        const double rl2 = R.rc_lj2, rcc2 = R.rc_c2, alpha = R.alpha;
        const double2* lj = d.lj64 + R.lj_off + ti * R.n_types;
        double fix = 0, fiy = 0, fiz = 0, fjx = 0, fjy = 0, fjz = 0;
        double el = 0, ec = 0, vir = 0;
        for (int k = 0; k < 32; ++k) {
            const int src = (lane + k) & 31;
            const uint32_t m = s_mk[wib][src];
            if ((m >> lane) & 1u) {
                const double4 pj = s_xj[wib][src];
                const double dx = mi_ref(__dsub_rn(pj.x, xi.x), L, invL);
                const double dy = mi_ref(__dsub_rn(pj.y, xi.y), L, invL);
                const double dz = mi_ref(__dsub_rn(pj.z, xi.z), L, invL);
                const double r2 = r2_ref(dx, dy, dz);
                double f = 0.0;
                if (has_lj && r2 < rl2) {
                    // 24 eps (2 sr6^2 - sr6) / r2 and 4 eps (sr6^2 - sr6), reference order
                    const double2 p = lj[s_tj[wib][src]];
                    const double r6 = __dmul_rn(__dmul_rn(r2, r2), r2);
                    const double sr6 = __ddiv_rn(p.y, r6);
                    f = __ddiv_rn(__dmul_rn(__dmul_rn(24.0, p.x),
                                            __dsub_rn(__dmul_rn(__dmul_rn(2.0, sr6), sr6), sr6)), r2);
                    el += __dmul_rn(__dmul_rn(4.0, p.x), __dsub_rn(__dmul_rn(sr6, sr6), sr6));
                }
                if (has_c && r2 < rcc2) {
                    const double qq = KE * xi.w * pj.w;
                    const double r = sqrt(r2);
                    const double erfc_ar = erfc(alpha * r);
                    f += qq * (erfc_ar / (r2 * r) + 2.0 * alpha * exp(-alpha * alpha * r2) /
                                                        (1.7724538509055160273 * r2));
                    ec += qq * erfc_ar / r;
                }
                vir += f * r2;
                fix -= f * dx;
                fiy -= f * dy;
                fiz -= f * dz;
                fjx += f * dx;
                fjy += f * dy;
                fjz += f * dz;
            }
            fjx = __shfl_sync(FULL, fjx, (lane + 1) & 31);
            fjy = __shfl_sync(FULL, fjy, (lane + 1) & 31);
            fjz = __shfl_sync(FULL, fjz, (lane + 1) & 31);
        }
        if (d.atom_of_slot[si] >= 0) {
            fix_add(d.fnx + si, to_fix(fix, FSCALE, s));
            fix_add(d.fny + si, to_fix(fiy, FSCALE, s));
            fix_add(d.fnz + si, to_fix(fiz, FSCALE, s));
        }
        if (mk) {
            fix_add(d.fnx + js, to_fix(fjx, FSCALE, s));
            fix_add(d.fny + js, to_fix(fjy, FSCALE, s));
            fix_add(d.fnz + js, to_fix(fjz, FSCALE, s));
        }
        acc.lj += to_fix(el, ESCALE, s);
        acc.c += to_fix(ec, ESCALE, s);
        acc.v += to_fix(vir, ESCALE, s);
        __syncwarp();
    }
    flush_acc(d, cur, acc);
}

}  // namespace

void launch_nonbonded(const Dev& d, bool fp64, bool phys, int n_sm, cudaStream_t st,
                      long long* nlaunch) {
    const int blocks = n_sm * 8;
    if (fp64) {
        if (phys) k_nb_f64<true><<<blocks, 256, 0, st>>>(d);
        else k_nb_f64<false><<<blocks, 256, 0, st>>>(d);
    } else {
        if (phys) k_nb_f32<true><<<blocks, 256, 0, st>>>(d);
        else k_nb_f32<false><<<blocks, 256, 0, st>>>(d);
    }
    *nlaunch += 1;
}

}  // namespace dmd
