// k_nonbonded.cu -- Lennard-Jones + real-space Ewald pair forces over the chunk list.
//
// Replaces LennardJones::compute (src/force/lennard_jones.cpp:43-92) and
// CoulombDirect::compute (src/force/coulomb_direct.cpp:38-86).  One warp per
// chunk: lane i holds i-atom i of the tile; the chunk's 32 j atoms are staged
// in shared memory and visited in a rotated order ((lane + k) & 31) so every
// lane touches a different j at each of the 32 steps; the j forces rotate with
// warp shuffles and are flushed once per chunk, i forces once per chunk.  The
// chunk's 32 masks are transposed in registers into each lane's visiting order.
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
#include <algorithm>

#include "device.cuh"
#include "launch.h"

namespace dmd {

namespace {

constexpr float TWO_OVER_SQRTPI_F = 1.1283791670955126f;
constexpr double TWO_OVER_SQRTPI = 1.1283791670955125739;

struct Acc {
    long long lj, c, v;
};

// Single-instruction approximations (PTX .approx forms, flush-to-zero).
__device__ __forceinline__ float rsqrt_ap(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_ap(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ap(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// erfc(x) for x >= 0 given e = exp(-x*x): Abramowitz & Stegun, Handbook of
// Mathematical Functions, eq. 7.1.26 (absolute error <= 1.5e-7).
__device__ __forceinline__ float erfc_as(float x, float e) {
    const float t = rcp_ap(fmaf(0.3275911f, x, 1.0f));
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

// Rotated transpose of the chunk's masks: entry j's mask has bit i set when
// (i, j) interacts; lane l receives the bits it visits, bit k = (l, entry (l+k)&31).
// Butterfly transpose of the 32x32 bit matrix over five shuffle stages, then a
// rotation by the lane index.
__device__ __forceinline__ uint32_t rotated_columns(uint32_t x, int lane) {
    const uint32_t m[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int w = 16 >> s;
        const uint32_t y = __shfl_xor_sync(FULL, x, w);
        x = (lane & w) ? ((x & ~m[s]) | ((y >> w) & m[s])) : ((x & m[s]) | ((y << w) & ~m[s]));
    }
    return __funnelshift_r(x, x, lane);
}

// Per-warp staging of one chunk's 32 j entries.  Coordinates and LJ columns are
// stored twice (entry l at l and l + 32) so round k of lane l reads index l + k
// with an immediate offset instead of (l + k) & 31.
struct ChunkStage {
    float4 xq[64];
    int tj[64];
    int js[32];
    int aj[32];
};

// Force of one pair over r (f: F_j = f (r_j - r_i)) and its energy terms.
// c12f/c6f are the force-scaled LJ coefficients (12 c12, 6 c6) and qq the
// Coulomb prefactor, each already zero when the term does not apply.
template <bool PHYS>
__device__ __forceinline__ float pair_f(float r2, float c6f, float c12f, float qq, float alpha,
                                        float a2l2e, float c2a, float& ir6, float& rinv,
                                        float& erfc_ar) {
    rinv = rsqrt_ap(r2);
    const float ir2 = rinv * rinv;
    ir6 = ir2 * ir2 * ir2;
    float fr = ir6 * fmaf(c12f, ir6, -c6f);
    if (PHYS) {
        const float ex = ex2_ap(a2l2e * r2);
        erfc_ar = erfc_as(alpha * (r2 * rinv), ex);
        fr = fmaf(qq, fmaf(erfc_ar, rinv, c2a * ex), fr);
    }
    return fr * ir2;
}

// One chunk (an i-tile against 32 j entries) for one warp.  Lane l owns i atom l
// and j entry l; in round k it pairs its i atom with entry (l+k)&31 and passes the
// j forces it accumulated on to lane l-1, so after 32 rounds they are back home.
// The loop is branch-free: a pair that is masked out or outside a cutoff gets
// zero coefficients.  Pairs whose FP32 r^2 lies within 1e-5 (relative) of a
// cutoff are left out of the loop and redone afterwards with the FP64 reference
// membership test, so the interacting set is exactly the reference's.
//
// PHYS = false evaluates LJ only (the REF profile, and PHYS replicas without
// charges); SAME = true is the PHYS form whose LJ and Coulomb cutoffs are equal
// (one band test, one cutoff test per pair).  MI = true (boxes narrower than
// twice the list cutoff) takes the minimum image of every pair at every
// evaluation, as the reference does (Cell::minimum_image, cell.cpp:26-38): in
// such a box the nearest image of a listed pair can change between list
// builds, so the image frozen at the build is not enough.
template <bool PHYS, bool SAME, bool ENERGY, bool MI>
__device__ __forceinline__ void nb_chunk(const Dev& d, const Rep& R, RepState* s, int c, int lane,
                                         ChunkStage& S, const float4* lj_tab, Acc& acc) {
    const double L = s->L;
    const float Lf = static_cast<float>(L), iLf = static_cast<float>(s->invL);
    const int I = d.chunk_itile[c];
    const int si = 32 * I + lane;
    const float4 xi = d.xq32[si];
    const int ti = d.type_s[si];
    const int ai = d.atom_of_slot[si];  // loaded with the chunk's other inputs, used at its end
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
    S.xq[lane] = xj;
    S.xq[lane + 32] = xj;
    S.tj[lane] = tj;
    S.tj[lane + 32] = tj;
    S.js[lane] = js;
    S.aj[lane] = aj;
    uint32_t rm = rotated_columns(mk, lane);
    __syncwarp();
    const bool has_lj = (R.flags & F_LJ) != 0;
    const bool has_c = PHYS && (R.flags & F_COUL_REAL) != 0;
    // an absent term gets a cutoff (and band) at r^2 = 0, so its tests are false
    const float rl2 = has_lj ? static_cast<float>(R.rc_lj2) : 0.f;
    const float rcc2 = has_c ? static_cast<float>(R.rc_c2) : 0.f;
    const float wl = rl2 * 1e-5f, wc = rcc2 * 1e-5f;
    const float alpha = static_cast<float>(R.alpha);
    const float a2l2e = -alpha * alpha * 1.4426950408889634f;  // -alpha^2 log2(e)
    const float c2a = TWO_OVER_SQRTPI_F * alpha;
    const float keqi = static_cast<float>(KE) * xi.w;
    const float4* lj = lj_tab + R.lj_off + ti * R.n_types;
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float fjx = 0.f, fjy = 0.f, fjz = 0.f;
    float el = 0.f, ec = 0.f, vir = 0.f;
    uint32_t band = 0;
    const int src_lane = (lane + 1) & 31;
#pragma unroll 1
    for (int kk = 0; kk < 32; kk += 8) {
        const float4* px = S.xq + lane + kk;
        const int* pt = S.tj + lane + kk;
        uint32_t b8 = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const bool bit = (rm >> u) & 1u;
            const float4 pj = px[u];
            const float4 p = lj[pt[u]];
            float dx = pj.x - xi.x, dy = pj.y - xi.y, dz = pj.z - xi.z;
            if (MI) {
                dx = fmaf(-Lf, rintf(dx * iLf), dx);
                dy = fmaf(-Lf, rintf(dy * iLf), dy);
                dz = fmaf(-Lf, rintf(dz * iLf), dz);
            }
            const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (!ENERGY && (!PHYS || SAME)) {
                // one cutoff: evaluate with the table coefficients and keep the
                // force only for interacting pairs (a masked self pair of a
                // diagonal chunk gives a non-finite f, which the select drops)
                const bool near = bit & (fabsf(d2 - rl2) < wl);
                const bool in = bit & !near & (d2 < rl2);
                b8 |= static_cast<uint32_t>(near) << u;
                float ir6, rinv, erfc_ar;
                const float fa = pair_f<PHYS>(d2, p.z, p.w, keqi * pj.w, alpha, a2l2e, c2a, ir6, rinv, erfc_ar);
                const float f = in ? fa : 0.f;
                fix = fmaf(-f, dx, fix);
                fiy = fmaf(-f, dy, fiy);
                fiz = fmaf(-f, dz, fiz);
                fjx = fmaf(f, dx, fjx);
                fjy = fmaf(f, dy, fjy);
                fjz = fmaf(f, dz, fjz);
                fjx = __shfl_sync(FULL, fjx, src_lane);
                fjy = __shfl_sync(FULL, fjy, src_lane);
                fjz = __shfl_sync(FULL, fjz, src_lane);
                continue;
            }
            const float r2 = fmaxf(d2, 1e-6f);
            bool near, in_l, in_c;
            if (!PHYS || SAME) {
                near = bit & (fabsf(r2 - rl2) < wl);
                in_l = bit & !near & (r2 < rl2);
                in_c = in_l;
            } else {
                near = bit & ((fabsf(r2 - rl2) < wl) | (fabsf(r2 - rcc2) < wc));
                const bool use = bit & !near;
                in_l = use & (r2 < rl2);
                in_c = use & (r2 < rcc2);
            }
            b8 |= static_cast<uint32_t>(near) << u;
            const float c6f = in_l ? p.z : 0.f, c12f = in_l ? p.w : 0.f;
            const float qq = (PHYS && in_c) ? keqi * pj.w : 0.f;
            float ir6, rinv, erfc_ar;
            const float f = pair_f<PHYS>(r2, c6f, c12f, qq, alpha, a2l2e, c2a, ir6, rinv, erfc_ar);
            if (ENERGY) {
                const float c6 = in_l ? p.x : 0.f, c12 = in_l ? p.y : 0.f;
                el = fmaf(ir6, fmaf(c12, ir6, -c6), el);
                if (PHYS) ec = fmaf(qq * erfc_ar, rinv, ec);
                vir = fmaf(f, r2, vir);
            }
            fix = fmaf(-f, dx, fix);
            fiy = fmaf(-f, dy, fiy);
            fiz = fmaf(-f, dz, fiz);
            fjx = fmaf(f, dx, fjx);
            fjy = fmaf(f, dy, fjy);
            fjz = fmaf(f, dz, fjz);
            fjx = __shfl_sync(FULL, fjx, src_lane);
            fjy = __shfl_sync(FULL, fjy, src_lane);
            fjz = __shfl_sync(FULL, fjz, src_lane);
        }
        band |= b8 << kk;
        rm >>= 8;
    }
    // after 32 rounds lane l holds the forces of entry l again
    while (band) {  // pairs at a cutoff (rare): FP64 reference membership
        const int k = __ffs(band) - 1;
        band &= band - 1;
        const int src = (lane + k) & 31;
        const float4 pj = S.xq[src];
        const float4 p = lj[S.tj[src]];
        const int aj2 = S.aj[src];
        const bool in_l = has_lj && exact_inside(d, ai, aj2, L, s->invL, R.rc_lj2);
        const bool in_c = has_c && exact_inside(d, ai, aj2, L, s->invL, R.rc_c2);
        float dx = pj.x - xi.x, dy = pj.y - xi.y, dz = pj.z - xi.z;
        if (MI) {
            dx = fmaf(-Lf, rintf(dx * iLf), dx);
            dy = fmaf(-Lf, rintf(dy * iLf), dy);
            dz = fmaf(-Lf, rintf(dz * iLf), dz);
        }
        const float r2 = fmaxf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)), 1e-6f);
        const float qq = (PHYS && in_c) ? keqi * pj.w : 0.f;
        float ir6, rinv, erfc_ar;
        const float f = pair_f<PHYS>(r2, in_l ? p.z : 0.f, in_l ? p.w : 0.f, qq, alpha, a2l2e, c2a, ir6,
                                     rinv, erfc_ar);
        if (ENERGY) {
            el = fmaf(ir6, fmaf(in_l ? p.y : 0.f, ir6, in_l ? -p.x : 0.f), el);
            if (PHYS) ec = fmaf(qq * erfc_ar, rinv, ec);
            vir = fmaf(f, r2, vir);
        }
        fix = fmaf(-f, dx, fix);
        fiy = fmaf(-f, dy, fiy);
        fiz = fmaf(-f, dz, fiz);
        const int js2 = S.js[src];
        fix_add(d.fnx + js2, to_fix(f * dx, FSCALE, s));
        fix_add(d.fny + js2, to_fix(f * dy, FSCALE, s));
        fix_add(d.fnz + js2, to_fix(f * dz, FSCALE, s));
    }
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
    if (ENERGY) {
        acc.lj += to_fix(el, ESCALE, s);
        acc.c += to_fix(ec, ESCALE, s);
        acc.v += to_fix(vir, ESCALE, s);
    }
    __syncwarp();
}

// LJ table entries staged in shared memory per block (larger tables are read
// from global memory).
constexpr int LJ_SMEM = 512;

// LJS: the LJ table fits LJ_SMEM and is staged in shared memory (a compile-time
// choice, so the table loads are shared-memory loads).  MIK: the kernel for the
// replicas whose box is narrower than twice their list cutoff (minimum image
// per evaluation); launched, with its own work counter, only when the table
// has such replicas (d.mi_split), in which case the main kernel leaves them to
// it -- so their forms do not weigh on the main kernel's registers.
// 80 registers (3 blocks of 256 threads per SM) with the real-space Ewald
// forms; the LJ-only instantiation (PHYS = false: the REF profile, and PHYS
// tables without real-space Coulomb) fits 64 (4 blocks per SM).
template <bool PHYS, bool LJS, bool MIK>
__global__ void __launch_bounds__(256, PHYS ? 3 : 4) k_nb_f32(Dev d) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    __shared__ ChunkStage s_stage[8];
    __shared__ float4 s_lj[LJS ? LJ_SMEM : 1];
    if (LJS)
        for (int k = threadIdx.x; k < d.n_lj; k += blockDim.x) s_lj[k] = d.lj32[k];
    __syncthreads();
    const float4* lj_tab = LJS ? s_lj : d.lj32;
    const int total = d.chunk_prefix[d.n_rep];
    Acc acc{0, 0, 0};
    int cur = -1;
    // chunks are taken one per warp from a counter, so warps on SMs shared with
    // the concurrent PME kernels simply take fewer
    int* counter = MIK ? d.nb_work_mi : d.nb_work;
    for (;;) {
        int w = 0;
        if (lane == 0) w = atomicAdd(counter, 1);
        w = __shfl_sync(FULL, w, 0);
        if (w >= total) break;
        const int r = chunk_replica(d.chunk_prefix, d.n_rep, w);
        if (r != cur) {
            flush_acc(d, cur, acc);
            cur = r;
        }
        RepState* s = d.st + r;
        const Rep& R = d.rep[r];
        // box narrower than twice the list cutoff: minimum image per evaluation
        // (d.mi_split is set whenever a replica's box is, or under a barostat
        // may become, that narrow)
        const bool mi = 4.0 * R.rc_list2 > s->L * s->L;
        if (!s->eval || MIK != (mi && d.mi_split)) {
            // a replica this kernel skips: move the counter past its chunks.
            // The minimum-image kernel evaluates few replicas of a table, so it
            // moves the counter straight to the next one it evaluates (lanes
            // test 32 replicas at a time) instead of one replica per claim.
            int next = r + 1;
            if (MIK) {
                next = d.n_rep;
                for (int b = r + 1; b < d.n_rep; b += 32) {
                    const int q = b + lane;
                    bool take = false;
                    if (q < d.n_rep) {
                        const RepState* sq = d.st + q;
                        take = sq->eval && 4.0 * d.rep[q].rc_list2 > sq->L * sq->L;
                    }
                    const unsigned m = __ballot_sync(FULL, take);
                    if (m) {
                        next = b + __ffs(m) - 1;
                        break;
                    }
                }
            }
            if (lane == 0) atomicMax(counter, d.chunk_prefix[next]);
            continue;
        }
        const int c = R.chunk_begin + (w - d.chunk_prefix[r]);
        // warp-uniform choice of the pair form for this replica
        const bool coul = PHYS && (R.flags & F_COUL_REAL);
        const bool same = coul && (R.flags & F_LJ) && R.rc_lj2 == R.rc_c2;
        if (MIK) {
            if (!coul) {
                if (s->want_e) nb_chunk<false, false, true, true>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
                else nb_chunk<false, false, false, true>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            } else {
                if (s->want_e) nb_chunk<PHYS, false, true, true>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
                else nb_chunk<PHYS, false, false, true>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            }
        } else if (s->want_e) {
            if (!coul) nb_chunk<false, false, true, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            else if (same) nb_chunk<true, true, true, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            else nb_chunk<true, false, true, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
        } else {
            if (!coul) nb_chunk<false, false, false, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            else if (same) nb_chunk<true, true, false, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
            else nb_chunk<true, false, false, false>(d, R, s, c, lane, s_stage[wib], lj_tab, acc);
        }
    }
    flush_acc(d, cur, acc);
}

// ---- 8-atom i-cluster form -------------------------------------------------
// One warp per i-cluster (8 consecutive slots of a tile), over the cluster's
// rows of 32 j entries.  Lane l owns j entry l of the row: it brings that j
// atom into the i-tile frame once per row, visits the 8 cluster atoms in turn
// (their coordinates are warp-uniform shared-memory broadcasts) and keeps the
// j force in registers, flushed once per row.  Each lane also keeps its own
// partial i forces for the 8 atoms (24 registers) over all the cluster's rows;
// at the end a butterfly reduce-scatter sums them across the warp in a fixed
// order.  No shuffle per pair, and because a cluster's entries are the j atoms
// within the list cutoff of its 8 atoms (not of a whole 32-atom tile), far
// fewer of the evaluated lane pairs are empty.  Masked and out-of-cutoff pairs
// get zero force by a select, as in the 32-wide form; pairs within 1e-5
// (relative) of a cutoff are redone with the FP64 reference membership test
// and added by fixed-point atomics of their own.
struct ClusterStage {
    float4 xi[8];   // x, y, z (tile frame), KE q
    int row[8];     // LJ table row of each cluster atom
    int ai[8];      // atom index (-1: padding slot)
};

// Butterfly reduce-scatter of v[0..7] over the warp: afterwards every lane
// holds the warp sum of v[i] for i = 4 b4 + 2 b3 + b2 (b = lane bits).
__device__ __forceinline__ float reduce8(const float (&v)[8], int lane) {
    float w4[4], w2[2];
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float send = h16 ? v[j] : v[j + 4];
        const float keep = h16 ? v[j + 4] : v[j];
        w4[j] = keep + __shfl_xor_sync(FULL, send, 16);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float send = h8 ? w4[j] : w4[j + 2];
        const float keep = h8 ? w4[j + 2] : w4[j];
        w2[j] = keep + __shfl_xor_sync(FULL, send, 8);
    }
    const float send = h4 ? w2[0] : w2[1];
    float t = (h4 ? w2[1] : w2[0]) + __shfl_xor_sync(FULL, send, 4);
    t += __shfl_xor_sync(FULL, t, 2);
    t += __shfl_xor_sync(FULL, t, 1);
    return t;
}

template <bool PHYS, bool SAME, bool ENERGY>
__device__ __forceinline__ void nb_cluster(const Dev& d, const Rep& R, RepState* s, int cl, int2 job,
                                           int lane, ClusterStage& S, const float4* lj_tab, Acc& acc) {
    const double L = s->L;
    const int I = cl >> 2;
    const int s0 = 32 * I + 8 * (cl & 3);
    if (lane < 8) {
        const int si = s0 + lane;
        const float4 x = d.xq32[si];
        S.xi[lane] = make_float4(x.x, x.y, x.z, static_cast<float>(KE) * x.w);
        S.row[lane] = R.lj_off + d.type_s[si] * R.n_types;
        S.ai[lane] = d.atom_of_slot[si];
    }
    __syncwarp();
    const double tIx = d.tcx[I], tIy = d.tcy[I], tIz = d.tcz[I];
    const bool has_lj = (R.flags & F_LJ) != 0;
    const bool has_c = PHYS && (R.flags & F_COUL_REAL) != 0;
    const float rl2 = has_lj ? static_cast<float>(R.rc_lj2) : 0.f;
    const float rcc2 = has_c ? static_cast<float>(R.rc_c2) : 0.f;
    const float wl = rl2 * 1e-5f, wc = rcc2 * 1e-5f;
    const float alpha = static_cast<float>(R.alpha);
    const float a2l2e = -alpha * alpha * 1.4426950408889634f;
    const float c2a = TWO_OVER_SQRTPI_F * alpha;
    float fix[8], fiy[8], fiz[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) fix[i] = fiy[i] = fiz[i] = 0.f;
    float el = 0.f, ec = 0.f, vir = 0.f;
#pragma unroll 1
    for (int k = 0; k < job.y; ++k) {
        const long long g = job.x + k;
        const uint32_t e = d.cl_j[32 * g + lane];
        const uint32_t m8 = d.cl_m[32 * g + lane];
        const int js = static_cast<int>(e & 0x03FFFFFFu);
        float4 xj = make_float4(1e6f, 1e6f, 1e6f, 0.f);
        int tj = 0;
        if (m8) {
            xj = d.xq32[js];
            tj = d.type_s[js];
            const int J = js >> 5;
            const int mx = static_cast<int>((e >> 26) & 3u) - 1;
            const int my = static_cast<int>((e >> 28) & 3u) - 1;
            const int mz = static_cast<int>((e >> 30) & 3u) - 1;
            xj.x += static_cast<float>(d.tcx[J] - tIx + mx * L);
            xj.y += static_cast<float>(d.tcy[J] - tIy + my * L);
            xj.z += static_cast<float>(d.tcz[J] - tIz + mz * L);
        }
        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
        uint32_t band = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float4 xi = S.xi[i];
            const float4 p = lj_tab[S.row[i] + tj];
            const bool bit = (m8 >> i) & 1u;
            const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            float f;
            if (!ENERGY && (!PHYS || SAME)) {
                const bool near = bit & (fabsf(d2 - rl2) < wl);
                const bool in = bit & !near & (d2 < rl2);
                band |= static_cast<uint32_t>(near) << i;
                float ir6, rinv, erfc_ar;
                const float fa = pair_f<PHYS>(d2, p.z, p.w, xi.w * xj.w, alpha, a2l2e, c2a, ir6, rinv, erfc_ar);
                f = in ? fa : 0.f;
            } else {
                const float r2 = fmaxf(d2, 1e-6f);
                bool near, in_l, in_c;
                if (!PHYS || SAME) {
                    near = bit & (fabsf(r2 - rl2) < wl);
                    in_l = bit & !near & (r2 < rl2);
                    in_c = in_l;
                } else {
                    near = bit & ((fabsf(r2 - rl2) < wl) | (fabsf(r2 - rcc2) < wc));
                    const bool use = bit & !near;
                    in_l = use & (r2 < rl2);
                    in_c = use & (r2 < rcc2);
                }
                band |= static_cast<uint32_t>(near) << i;
                const float qq = (PHYS && in_c) ? xi.w * xj.w : 0.f;
                float ir6, rinv, erfc_ar;
                f = pair_f<PHYS>(r2, in_l ? p.z : 0.f, in_l ? p.w : 0.f, qq, alpha, a2l2e, c2a, ir6, rinv,
                                 erfc_ar);
                if (ENERGY) {
                    el = fmaf(ir6, fmaf(in_l ? p.y : 0.f, ir6, in_l ? -p.x : 0.f), el);
                    if (PHYS) ec = fmaf(qq * erfc_ar, rinv, ec);
                    vir = fmaf(f, r2, vir);
                }
            }
            fix[i] = fmaf(-f, dx, fix[i]);
            fiy[i] = fmaf(-f, dy, fiy[i]);
            fiz[i] = fmaf(-f, dz, fiz[i]);
            fjx = fmaf(f, dx, fjx);
            fjy = fmaf(f, dy, fjy);
            fjz = fmaf(f, dz, fjz);
        }
        if (__any_sync(FULL, band != 0)) {  // pairs at a cutoff (rare): FP64 reference membership
            const int aj = band ? d.atom_of_slot[js] : -1;
            while (band) {
                const int i = __ffs(band) - 1;
                band &= band - 1;
                const float4 xi = S.xi[i];
                const float4 p = lj_tab[S.row[i] + tj];
                const int ai = S.ai[i];
                const bool in_l = has_lj && exact_inside(d, ai, aj, L, s->invL, R.rc_lj2);
                const bool in_c = has_c && exact_inside(d, ai, aj, L, s->invL, R.rc_c2);
                const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                const float r2 = fmaxf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)), 1e-6f);
                const float qq = (PHYS && in_c) ? xi.w * xj.w : 0.f;
                float ir6, rinv, erfc_ar;
                const float f = pair_f<PHYS>(r2, in_l ? p.z : 0.f, in_l ? p.w : 0.f, qq, alpha, a2l2e, c2a,
                                             ir6, rinv, erfc_ar);
                if (ENERGY) {
                    el = fmaf(ir6, fmaf(in_l ? p.y : 0.f, ir6, in_l ? -p.x : 0.f), el);
                    if (PHYS) ec = fmaf(qq * erfc_ar, rinv, ec);
                    vir = fmaf(f, r2, vir);
                }
                const int si = s0 + i;
                fix_add(d.fnx + si, to_fix(-f * dx, FSCALE, s));
                fix_add(d.fny + si, to_fix(-f * dy, FSCALE, s));
                fix_add(d.fnz + si, to_fix(-f * dz, FSCALE, s));
                fjx = fmaf(f, dx, fjx);
                fjy = fmaf(f, dy, fjy);
                fjz = fmaf(f, dz, fjz);
            }
        }
        if (m8) {
            fix_add(d.fnx + js, to_fix(fjx, FSCALE, s));
            fix_add(d.fny + js, to_fix(fjy, FSCALE, s));
            fix_add(d.fnz + js, to_fix(fjz, FSCALE, s));
        }
    }
    const float rx = reduce8(fix, lane), ry = reduce8(fiy, lane), rz = reduce8(fiz, lane);
    if ((lane & 3) == 0) {
        const int i = ((lane >> 2) & 1) | ((lane >> 2) & 2) | ((lane >> 2) & 4);
        if (S.ai[i] >= 0) {
            const int si = s0 + i;
            fix_add(d.fnx + si, to_fix(rx, FSCALE, s));
            fix_add(d.fny + si, to_fix(ry, FSCALE, s));
            fix_add(d.fnz + si, to_fix(rz, FSCALE, s));
        }
    }
    if (ENERGY) {
        acc.lj += to_fix(el, ESCALE, s);
        acc.c += to_fix(ec, ESCALE, s);
        acc.v += to_fix(vir, ESCALE, s);
    }
    __syncwarp();
}

// Persistent over i-clusters (4 per tile, every replica), taken one per warp
// from a counter.  The cluster's 8 atoms stay in registers across its rows
// (up to 128 registers per thread: 2 blocks of 256 threads per SM).
template <bool PHYS, bool LJS>
__global__ void __launch_bounds__(256, 2) k_nb8_f32(Dev d) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    __shared__ ClusterStage s_stage[8];
    __shared__ float4 s_lj[LJS ? LJ_SMEM : 1];
    if (LJS)
        for (int k = threadIdx.x; k < d.n_lj; k += blockDim.x) s_lj[k] = d.lj32[k];
    __syncthreads();
    const float4* lj_tab = LJS ? s_lj : d.lj32;
    const int total = 4 * d.n_tiles;
    Acc acc{0, 0, 0};
    int cur = -1;
    for (;;) {
        int w = 0;
        if (lane == 0) w = atomicAdd(d.nb_work, 1);
        w = __shfl_sync(FULL, w, 0);
        if (w >= total) break;
        const int r = d.tile_rep[w >> 2];
        RepState* s = d.st + r;
        if (!s->eval) continue;
        // narrow-box replicas are left to the minimum-image chunk kernel
        if (d.mi_split && 4.0 * d.rep[r].rc_list2 > s->L * s->L) continue;
        const int2 job = d.cl_job[w];
        if (job.y == 0) continue;
        if (r != cur) {
            flush_acc(d, cur, acc);
            cur = r;
        }
        const Rep& R = d.rep[r];
        const bool coul = PHYS && (R.flags & F_COUL_REAL);
        const bool same = coul && (R.flags & F_LJ) && R.rc_lj2 == R.rc_c2;
        if (s->want_e) {
            if (!coul) nb_cluster<false, false, true>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
            else if (same) nb_cluster<true, true, true>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
            else nb_cluster<true, false, true>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
        } else {
            if (!coul) nb_cluster<false, false, false>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
            else if (same) nb_cluster<true, true, false>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
            else nb_cluster<true, false, false>(d, R, s, w, job, lane, s_stage[wib], lj_tab, acc);
        }
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

namespace {
const void* const kNbKernels[] = {
    reinterpret_cast<const void*>(k_nb_f32<true, true, false>),
    reinterpret_cast<const void*>(k_nb_f32<true, false, false>),
    reinterpret_cast<const void*>(k_nb_f32<false, true, false>),
    reinterpret_cast<const void*>(k_nb_f32<false, false, false>),
    reinterpret_cast<const void*>(k_nb_f32<true, true, true>),
    reinterpret_cast<const void*>(k_nb_f32<true, false, true>),
    reinterpret_cast<const void*>(k_nb_f32<false, true, true>),
    reinterpret_cast<const void*>(k_nb_f32<false, false, true>),
    reinterpret_cast<const void*>(k_nb8_f32<true, true>),
    reinterpret_cast<const void*>(k_nb8_f32<true, false>),
    reinterpret_cast<const void*>(k_nb8_f32<false, true>),
    reinterpret_cast<const void*>(k_nb8_f32<false, false>),
    reinterpret_cast<const void*>(k_nb_f64<true>),
    reinterpret_cast<const void*>(k_nb_f64<false>)};
}  // namespace

bool is_nonbonded_kernel(const void* f) {
    for (const void* p : kNbKernels)
        if (p == f) return true;
    return false;
}

// The persistent pair kernel holds its SMs for the whole force evaluation.
// With the default carveout the SMs it runs on are configured with little
// more shared memory than its own blocks use, and the PME chain's cuFFT
// kernels (4-16 KB of shared memory per block) cannot start beside it: on
// water 30k they waited ~24 us for its last blocks.  A carveout of 60 % of the
// unified L1 / shared memory as shared memory leaves room for them; the SPME
// chain then runs during the pair kernel (step period 140 -> 128 us).
void configure_nonbonded_kernels() {
    for (const void* k : kNbKernels)
        if (cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 60) != cudaSuccess)
            cudaGetLastError();
}

void launch_nonbonded(const Dev& d, bool fp64, bool phys, int n_sm, int blocks_per_sm, int form,
                      cudaStream_t st, long long* nlaunch) {
    if (fp64) {
        if (phys) k_nb_f64<true><<<n_sm * 8, 256, 0, st>>>(d);
        else k_nb_f64<false><<<n_sm * 8, 256, 0, st>>>(d);
    } else {
        const bool ljs = d.n_lj <= LJ_SMEM;
        // a table without real-space Coulomb runs the LJ-only instantiation
        // (its replicas take the same LJ form in either)
        phys = phys && d.any_coul;
        const int max_bps = phys ? 3 : 4;
        // persistent: up to the blocks per SM its registers allow (2 for the
        // cluster form, 3 for the chunk form, 4 for its LJ-only instantiation);
        // fewer leave room on every SM for the bonded / PME kernels alongside
        const int bps = std::max(blocks_per_sm, 1);
        if (form == NB_CLUSTER8 && d.cl_j) {
            const int g = n_sm * std::min(bps, 2);
            if (phys) {
                if (ljs) k_nb8_f32<true, true><<<g, 256, 0, st>>>(d);
                else k_nb8_f32<true, false><<<g, 256, 0, st>>>(d);
            } else {
                if (ljs) k_nb8_f32<false, true><<<g, 256, 0, st>>>(d);
                else k_nb8_f32<false, false><<<g, 256, 0, st>>>(d);
            }
        } else {
            const int g = n_sm * std::min(bps, max_bps);
            if (phys) {
                if (ljs) k_nb_f32<true, true, false><<<g, 256, 0, st>>>(d);
                else k_nb_f32<true, false, false><<<g, 256, 0, st>>>(d);
            } else {
                if (ljs) k_nb_f32<false, true, false><<<g, 256, 0, st>>>(d);
                else k_nb_f32<false, false, false><<<g, 256, 0, st>>>(d);
            }
        }
        if (d.mi_split) {  // narrow-box replicas: their own kernel on the same stream
            const int g = n_sm * std::min(bps, max_bps);
            if (phys) {
                if (ljs) k_nb_f32<true, true, true><<<g, 256, 0, st>>>(d);
                else k_nb_f32<true, false, true><<<g, 256, 0, st>>>(d);
            } else {
                if (ljs) k_nb_f32<false, true, true><<<g, 256, 0, st>>>(d);
                else k_nb_f32<false, false, true><<<g, 256, 0, st>>>(d);
            }
            *nlaunch += 1;
        }
    }
    *nlaunch += 1;
}

}  // namespace dmd
