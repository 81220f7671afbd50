// k_list.cu -- spatial sort and Verlet pair-list build (rebuild-time kernels).
//
// The pair list replaces LennardJones::rebuild_pair_list
// (src/force/lennard_jones.cpp:18-41): an O(N^2) loop over i<j that keeps
// pairs with minimum-image r^2 < rc^2.  Here atoms are counting-sorted into
// columns (x-y) and thin z slabs visited in a snake order, so that 32
// consecutive atoms form a compact tile; for every i-tile a list of "chunks"
// is built: 32 j atoms, each with a 32-bit mask over the i-tile's lanes.  A
// pair is tested in FP32 on tile-local coordinates; pairs within 1e-5 relative
// of the cutoff are decided with the reference's own FP64 expression
// (d - round(d/L) L, r2 summed left to right, strict <), so the pair set is
// identical to the reference's.  Only replicas whose `rebuild` flag is set do
// any work; the kernels are cheap no-ops otherwise.
#include "device.cuh"
#include "launch.h"

namespace dmd {

// R1: voxel of every atom (wrapped coordinates), frozen periodic image.
__device__ __forceinline__ void bin_atom(const Dev& d, int a) {
    int r = d.atom_rep[a];
    RepState* s = d.st + r;
    if (!s->rebuild) return;
    const Rep& R = d.rep[r];
    const double L = s->L;
    double p[3] = {d.x[a], d.y[a], d.z[a]};
    int im[3], v[3];
    for (int k = 0; k < 3; ++k) {
        const int nk = (k < 2) ? R.nvx : R.nvz;
        double f = floor(p[k] / L);
        im[k] = static_cast<int>(f);
        double w = p[k] - f * L;
        int c = static_cast<int>(w / L * nk);
        v[k] = min(max(c, 0), nk - 1);
    }
    d.imgx[a] = im[0];
    d.imgy[a] = im[1];
    d.imgz[a] = im[2];
    int vox = (v[0] * R.nvx + v[1]) * R.nvz + v[2];
    int bin = R.bin_begin + d.vox_rank[R.bin_begin + vox];
    d.atom_bin[a] = bin;
    atomicAdd(d.bin_count + bin, 1);
}

// R2: exclusive scan of one replica's bin counts by one block (NT_B threads):
// contiguous bin ranges per thread, warp-shuffle scan of the thread sums.
constexpr int NT_R = 128;
__device__ __forceinline__ void bin_scan_replica(const Dev& d, int r) {
    __shared__ int s_warp[NT_R / 32];
    const Rep& R = d.rep[r];
    const int nb = R.nvx * R.nvx * R.nvz;
    const int per = (nb + NT_R - 1) / NT_R;
    const int b0 = R.bin_begin + min(static_cast<int>(threadIdx.x) * per, nb);
    const int b1 = min(b0 + per, R.bin_begin + nb);
    int local = 0;
    for (int b = b0; b < b1; ++b) local += d.bin_count[b];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    int off = 0;
    for (int k = 0; k < w; ++k) off += s_warp[k];
    int run = off + incl - local + 32 * R.tile_begin;
    for (int b = b0; b < b1; ++b) {
        d.bin_start[b] = run;
        run += d.bin_count[b];
    }
    __syncthreads();
}

// R3: scatter atoms to their bin ranges (order within a bin fixed by R4).
__device__ __forceinline__ void bin_scatter_atom(const Dev& d, int a) {
    if (!d.st[d.atom_rep[a]].rebuild) return;
    int b = d.atom_bin[a];
    int pos = d.bin_start[b] + atomicAdd(d.bin_fill + b, 1);
    d.sort_buf[pos] = a;
}

// R4: order each bin by atom index (deterministic slot order) and reset its
// counters.  One warp per bin: every member's rank is the number of smaller
// atom indices in the bin (indices are distinct), and it is written straight
// to its slot in atom_of_slot.
__device__ __forceinline__ void bin_sort_warp(const Dev& d, const int* bin_rep, int b, int lane) {
    if (!d.st[bin_rep[b]].rebuild) return;
    const int n = d.bin_count[b];
    const int* p = d.sort_buf + d.bin_start[b];
    int* out = d.atom_of_slot + d.bin_start[b];
    for (int base = 0; base < n; base += 32) {
        const int v = (base + lane < n) ? p[base + lane] : 0x7fffffff;
        int rank = 0;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int w = (c0 + lane < n) ? p[c0 + lane] : 0x7fffffff;
#pragma unroll 8
            for (int k = 0; k < 32; ++k) rank += (__shfl_sync(FULL, w, k) < v) ? 1 : 0;
        }
        if (base + lane < n) out[rank] = v;
    }
    __syncwarp();
    if (lane == 0) {
        d.bin_count[b] = 0;
        d.bin_fill[b] = 0;
    }
}

// R5: tiles -- slot<->atom maps, reference positions, bounding boxes, mirror.
__device__ __forceinline__ void tile_warp(const Dev& d, int t, int lane) {
    const int r = d.tile_rep[t];
    RepState* s = d.st + r;
    if (!s->rebuild) return;
    const Rep& R = d.rep[r];
    const double L = s->L;
    const int slot = 32 * t + lane;
    const int local = slot - 32 * R.tile_begin;
    const int a = (local < R.n_atoms) ? d.atom_of_slot[slot] : -1;  // ordered by R4
    d.atom_of_slot[slot] = a;
    double w[3] = {0.0, 0.0, 0.0};
    double xa = 0, ya = 0, za = 0, qa = 0;
    if (a >= 0) {
        d.slot_of_atom[a] = slot;
        d.type_s[slot] = d.type[a];
        xa = d.x[a];
        ya = d.y[a];
        za = d.z[a];
        qa = d.q[a];
        d.xr[a] = xa;
        d.yr[a] = ya;
        d.zr[a] = za;
        w[0] = xa - d.imgx[a] * L;
        w[1] = ya - d.imgy[a] * L;
        w[2] = za - d.imgz[a] * L;
    } else {
        d.type_s[slot] = 0;
    }
    double c[3];
    float h[3];
    for (int k = 0; k < 3; ++k) {
        double lo = warp_min_d(a >= 0 ? w[k] : 1e300);
        double hi = warp_max_d(a >= 0 ? w[k] : -1e300);
        c[k] = 0.5 * (lo + hi);
        h[k] = static_cast<float>(0.5 * (hi - lo)) * 1.000001f + 1e-6f;
    }
    if (lane == 0) {
        d.tcx[t] = c[0];
        d.tcy[t] = c[1];
        d.tcz[t] = c[2];
        d.thx[t] = h[0];
        d.thy[t] = h[1];
        d.thz[t] = h[2];
    }
    // build-frame FP32 coordinates (the mixed-precision mirror itself when it exists)
    d.xl32[slot] = (a >= 0) ? make_float4(static_cast<float>(w[0] - c[0]), static_cast<float>(w[1] - c[1]),
                                          static_cast<float>(w[2] - c[2]), static_cast<float>(qa))
                            : make_float4(0.f, 0.f, 0.f, 0.f);
    if (d.xq64) d.xq64[slot] = make_double4(xa, ya, za, qa);
}

// Entry encoding: bits 0..25 j slot, 26..31 image shift (mx+1, my+1, mz+1), 2 bits each.
//
// R6: chunk list.  A block of BW warps per i-tile, in batches of up to MAXC
// candidate j-tiles (J >= I, same replica, conservative bounding-box test,
// enumerated in tile order):
//  1. enumerate the batch's candidates into shared memory;
//  2. stage their j atoms in the i-tile's frame (all threads, independent loads);
//  3. per candidate (round-robin over warps), lane = i atom: one ballot per j
//     atom gives that j's 32-bit mask.  A candidate whose two tiles need more
//     than one periodic image (small boxes) takes the general per-pair path;
//  4. compact the non-empty entries in order and write whole chunks with one
//     counter update per batch; fewer than 32 left over carry to the next batch.
// Per pair: FP32 on tile-local coordinates, the reference's FP64 expression
// within 1e-5 of the cutoff; PHYS drops excluded pairs.
constexpr int BW = 4;
constexpr int NT_B = 32 * BW;
constexpr int MAXC = 48;
constexpr float FAR = 1e18f;  // coordinate of padding atoms: r^2 overflows to +inf
constexpr int ONE_IMAGE = 1 << 6;

// The reference's minimum-image r^2 < rc2 test in FP64 (src/core/pbc.h semantics).
__device__ __forceinline__ bool ref_member(const Dev& d, int ai, int aj, double L, double invL, double rc2) {
    double ex = __dsub_rn(d.x[aj], d.x[ai]), ey = __dsub_rn(d.y[aj], d.y[ai]), ez = __dsub_rn(d.z[aj], d.z[ai]);
    ex = __dsub_rn(ex, __dmul_rn(round(__dmul_rn(ex, invL)), L));
    ey = __dsub_rn(ey, __dmul_rn(round(__dmul_rn(ey, invL)), L));
    ez = __dsub_rn(ez, __dmul_rn(round(__dmul_rn(ez, invL)), L));
    return r2_ref(ex, ey, ez) < rc2;
}

__device__ __forceinline__ void build_tile(const Dev& d, int I) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    __shared__ float s_lx[32], s_ly[32], s_lz[32];
    __shared__ int s_a[32];
    __shared__ uint32_t s_e[BW][64], s_m[BW][64];   // general path: per-warp entry buffers
    __shared__ int s_left[BW];
    __shared__ int s_cand[MAXC], s_cinfo[MAXC];
    __shared__ float4 s_coff[MAXC];                  // j-tile frame -> i-tile frame (FP32)
    __shared__ float4 s_jx[MAXC * 32];               // staged j atoms (w = atom index bits);
                                                     // reused for compaction
    __shared__ uint32_t s_je[MAXC * 32];             // staged j entry words
    __shared__ uint32_t s_msk[MAXC * 32];
    __shared__ uint32_t s_carry_e[32], s_carry_m[32];
    __shared__ int s_wcnt[4][BW];
    __shared__ int s_jnext, s_c0;
    const int r = d.tile_rep[I];
    RepState* s = d.st + r;
    if (!s->rebuild) return;
    const Rep& R = d.rep[r];
    const double L = s->L, invL = s->invL;
    const float Lf = static_cast<float>(L), hLf = 0.5f * Lf;
    const bool phys = (R.flags & F_PHYS) != 0;
    const double rc2 = R.rc_list2;
    const float rc2_lo = static_cast<float>(rc2 * (1.0 - 1e-5));
    const float rc2_hi = static_cast<float>(rc2 * (1.0 + 1e-5));
    const double bb_rc2 = rc2 * (1.0 + 1e-6) + 1e-9;
    const double cIx = d.tcx[I], cIy = d.tcy[I], cIz = d.tcz[I];
    if (wib == 0) {
        const int a = d.atom_of_slot[32 * I + lane];
        const float4 p = d.xl32[32 * I + lane];
        s_a[lane] = a;
        s_lx[lane] = p.x;
        s_ly[lane] = p.y;
        s_lz[lane] = p.z;
    }
    __syncthreads();
    const float hIx = d.thx[I], hIy = d.thy[I], hIz = d.thz[I];
    const int t_end = R.tile_begin + R.n_tiles;
    // this lane's i atom and (PHYS) its exclusion partners, sorted ascending
    const int ai = s_a[lane];
    // a padding i lane sits far away (+FAR), padding j atoms at -FAR: no pair
    const float lix = ai >= 0 ? s_lx[lane] : FAR, liy = ai >= 0 ? s_ly[lane] : FAR,
                liz = ai >= 0 ? s_lz[lane] : FAR;
    int iex[8];
    // exclusion partners span [i_lo, i_lo + i_span]; an empty set never matches
    int i_e0 = 0, i_e1 = 0, i_lo = 0x7fffffff, i_span = 0;
    if (phys && ai >= 0) {
        i_e0 = d.ex_start[ai];
        i_e1 = d.ex_start[ai + 1];
        if (i_e1 > i_e0) {
            i_lo = d.ex_list[i_e0];
            i_span = d.ex_list[i_e1 - 1] - i_lo;
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) iex[k] = (i_e0 + k < i_e1) ? d.ex_list[i_e0 + k] : -1;

    // ---- general path (several periodic images per tile pair) ----------------
    int nbuf = 0;  // entries buffered in s_e/s_m[wib] (warp-uniform)
    auto flush_chunk = [&](const uint32_t* be, const uint32_t* bm, int count) {
        int c = 0;
        if (lane == 0) c = atomicAdd(&s->n_chunks, 1);
        c = __shfl_sync(FULL, c, 0);
        if (c >= R.chunk_cap) {
            if (lane == 0) set_status(s, ST_CAPACITY);
            return;
        }
        const int g = R.chunk_begin + c;
        if (lane == 0) d.chunk_itile[g] = I;
        d.chunk_j[32 * g + lane] = lane < count ? be[lane] : 0u;
        d.chunk_mask[32 * g + lane] = lane < count ? bm[lane] : 0u;
    };
    auto push = [&](uint32_t e, uint32_t m) {
        const uint32_t has = __ballot_sync(FULL, m != 0);
        const int pos = nbuf + __popc(has & ((1u << lane) - 1));
        if (m) {
            s_e[wib][pos] = e;
            s_m[wib][pos] = m;
        }
        nbuf += __popc(has);
        __syncwarp();
        if (nbuf >= 32) {
            flush_chunk(s_e[wib], s_m[wib], 32);
            __syncwarp();
            if (lane < nbuf - 32) {
                s_e[wib][lane] = s_e[wib][lane + 32];
                s_m[wib][lane] = s_m[wib][lane + 32];
            }
            nbuf -= 32;
            __syncwarp();
        }
    };
    // One candidate tile J, lane = j atom: each j is tested against every i,
    // and every periodic image code found becomes its own entry.
    auto general_candidate = [&](int J) {
        const int js = 32 * J + lane;
        const int aj = d.atom_of_slot[js];
        const double ddx = d.tcx[J] - cIx, ddy = d.tcy[J] - cIy, ddz = d.tcz[J] - cIz;
        const double rx0 = round(ddx * invL), ry0 = round(ddy * invL), rz0 = round(ddz * invL);
        float jx = 0.f, jy = 0.f, jz = 0.f;
        int ex[8];
        int nex = 0, e0 = 0, e1 = 0;
        if (aj >= 0) {
            jx = static_cast<float>((d.x[aj] - d.imgx[aj] * L) - cIx - rx0 * L);
            jy = static_cast<float>((d.y[aj] - d.imgy[aj] * L) - cIy - ry0 * L);
            jz = static_cast<float>((d.z[aj] - d.imgz[aj] * L) - cIz - rz0 * L);
            e0 = d.ex_start[aj];
            e1 = d.ex_start[aj + 1];
            if (phys) nex = e1 - e0;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) ex[k] = (k < nex) ? d.ex_list[e0 + k] : -1;
        uint32_t todo = 0;
        if (aj >= 0) todo = (J == I) ? ((1u << lane) - 1u) : 0xffffffffu;
        while (__any_sync(FULL, todo != 0)) {
            uint32_t bits = 0, rest = 0, code0 = 0xffffffffu;
            for (uint32_t t = todo; t; t &= t - 1) {
                const int i = __ffs(t) - 1;
                const int a_i = s_a[i];
                if (a_i < 0) continue;
                float dx = jx - s_lx[i], dy = jy - s_ly[i], dz = jz - s_lz[i];
                int sx = 0, sy = 0, sz = 0;
                if (dx > hLf) { dx -= Lf; sx = 1; } else if (dx < -hLf) { dx += Lf; sx = -1; }
                if (dy > hLf) { dy -= Lf; sy = 1; } else if (dy < -hLf) { dy += Lf; sy = -1; }
                if (dz > hLf) { dz -= Lf; sz = 1; } else if (dz < -hLf) { dz += Lf; sz = -1; }
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 >= rc2_hi) continue;
                int mx, my, mz;
                if (r2 > rc2_lo) {
                    // borderline: the reference's FP64 expression decides
                    double ex_ = __dsub_rn(d.x[aj], d.x[a_i]), ey = __dsub_rn(d.y[aj], d.y[a_i]),
                           ez = __dsub_rn(d.z[aj], d.z[a_i]);
                    const double qx = round(__dmul_rn(ex_, invL)), qy = round(__dmul_rn(ey, invL)),
                                 qz = round(__dmul_rn(ez, invL));
                    ex_ = __dsub_rn(ex_, __dmul_rn(qx, L));
                    ey = __dsub_rn(ey, __dmul_rn(qy, L));
                    ez = __dsub_rn(ez, __dmul_rn(qz, L));
                    if (!(r2_ref(ex_, ey, ez) < rc2)) continue;
                    mx = d.imgx[aj] - d.imgx[a_i] - static_cast<int>(qx);
                    my = d.imgy[aj] - d.imgy[a_i] - static_cast<int>(qy);
                    mz = d.imgz[aj] - d.imgz[a_i] - static_cast<int>(qz);
                } else {
                    // displacement = w_j - w_i - (r0 + s) L
                    mx = -static_cast<int>(rx0) - sx;
                    my = -static_cast<int>(ry0) - sy;
                    mz = -static_cast<int>(rz0) - sz;
                }
                if (phys) {
                    bool excluded = false;
                    if (nex <= 8) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) excluded |= (ex[k] == a_i);
                    } else {
                        for (int e = e0; e < e1; ++e) excluded |= (d.ex_list[e] == a_i);
                    }
                    if (excluded) continue;
                }
                const uint32_t code = static_cast<uint32_t>((mx + 1) | ((my + 1) << 2) | ((mz + 1) << 4));
                if (code0 == 0xffffffffu) code0 = code;
                if (code == code0) bits |= 1u << i;
                else rest |= 1u << i;
            }
            push(static_cast<uint32_t>(js) | ((bits ? code0 : 0u) << 26), bits);
            todo = rest;
        }
    };

    int carry_n = 0;
    int J_next = I;
    while (J_next < t_end) {
        // 1. candidates of this batch, in tile order (4 tiles per thread per round)
        if (tid == 0) s_jnext = t_end;
        int nc = 0;
        int J0 = J_next;
        while (J0 < t_end && nc < MAXC) {
            bool cand[4];
            int info[4];
            float4 off[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int J = J0 + u * NT_B + tid;
                cand[u] = false;
                info[u] = 0;
                off[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (J >= t_end) continue;
                double dx = d.tcx[J] - cIx, dy = d.tcy[J] - cIy, dz = d.tcz[J] - cIz;
                const double rx0 = round(dx * invL), ry0 = round(dy * invL), rz0 = round(dz * invL);
                dx -= L * rx0;
                dy -= L * ry0;
                dz -= L * rz0;
                const double ex = (double)(hIx + d.thx[J]), ey = (double)(hIy + d.thy[J]),
                             ez = (double)(hIz + d.thz[J]);
                const double gx = fmax(fabs(dx) - ex, 0.0), gy = fmax(fabs(dy) - ey, 0.0),
                             gz = fmax(fabs(dz) - ez, 0.0);
                cand[u] = gx * gx + gy * gy + gz * gz <= bb_rc2;
                // one periodic image serves every pair of the two tiles when their
                // extents around the centre displacement stay inside half a box
                const double hL = 0.5 * L;
                const bool one = fabs(dx) + ex < hL && fabs(dy) + ey < hL && fabs(dz) + ez < hL;
                info[u] = (static_cast<int>(rx0) + 1) | ((static_cast<int>(ry0) + 1) << 2) |
                          ((static_cast<int>(rz0) + 1) << 4) | (one ? ONE_IMAGE : 0);
                off[u] = make_float4(static_cast<float>(dx), static_cast<float>(dy), static_cast<float>(dz), 0.f);
            }
            uint32_t bal[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                bal[u] = __ballot_sync(FULL, cand[u]);
                if (lane == 0) s_wcnt[u][wib] = __popc(bal[u]);
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int before = nc, tot = 0;
#pragma unroll
                for (int w = 0; w < BW; ++w) {
                    before += (w < wib) ? s_wcnt[u][w] : 0;
                    tot += s_wcnt[u][w];
                }
                const int rank = before + __popc(bal[u] & ((1u << lane) - 1u));
                if (cand[u]) {
                    if (rank < MAXC) {
                        s_cand[rank] = J0 + u * NT_B + tid;
                        s_cinfo[rank] = info[u];
                        s_coff[rank] = off[u];
                    } else if (rank == MAXC) {
                        s_jnext = J0 + u * NT_B + tid;  // first candidate left for the next batch
                    }
                }
                nc += tot;
            }
            J0 += 4 * NT_B;
            __syncthreads();
        }
        J_next = (nc > MAXC) ? s_jnext : J0;
        if (nc > MAXC) nc = MAXC;
        // 2. stage, in order, the j atoms of single-image candidates that lie
        //    within the list cutoff of the i-tile's box (i-tile frame, FP32)
        int nj = 0;
        for (int e0 = 0; e0 < nc * 32; e0 += 4 * NT_B) {
            float4 pj[4];
            uint32_t ent[4];
            bool keep[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int idx = e0 + u * NT_B + tid;
                keep[u] = false;
                ent[u] = 0u;
                pj[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (idx >= nc * 32) continue;
                const int k = idx >> 5, info = s_cinfo[k];
                if (!(info & ONE_IMAGE)) continue;
                const int js = 32 * s_cand[k] + (idx & 31);
                const int aj = d.atom_of_slot[js];
                if (aj < 0) continue;
                const float4 p = d.xl32[js];
                const float4 o = s_coff[k];
                pj[u] = make_float4(p.x + o.x, p.y + o.y, p.z + o.z, __int_as_float(aj));
                const float gx = fmaxf(fabsf(pj[u].x) - hIx, 0.f), gy = fmaxf(fabsf(pj[u].y) - hIy, 0.f),
                            gz = fmaxf(fabsf(pj[u].z) - hIz, 0.f);
                keep[u] = gx * gx + gy * gy + gz * gz <= rc2_hi * 1.0001f + 1e-6f;
                const uint32_t code = static_cast<uint32_t>((2 - (info & 3)) | ((2 - ((info >> 2) & 3)) << 2) |
                                                            ((2 - ((info >> 4) & 3)) << 4));
                ent[u] = static_cast<uint32_t>(js) | (code << 26);
            }
            uint32_t bal[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                bal[u] = __ballot_sync(FULL, keep[u]);
                if (lane == 0) s_wcnt[u][wib] = __popc(bal[u]);
            }
            __syncthreads();
            int run = nj;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int before = run, tot = 0;
#pragma unroll
                for (int w = 0; w < BW; ++w) {
                    before += (w < wib) ? s_wcnt[u][w] : 0;
                    tot += s_wcnt[u][w];
                }
                if (keep[u]) {
                    const int pos = before + __popc(bal[u] & ((1u << lane) - 1u));
                    s_jx[pos] = pj[u];
                    s_je[pos] = ent[u];
                }
                run += tot;
            }
            nj = run;
            __syncthreads();
        }
        const int ngroups = (nj + 31) >> 5;
        for (int idx = nj + tid; idx < 32 * ngroups; idx += NT_B) {
            s_jx[idx] = make_float4(-FAR, -FAR, -FAR, __int_as_float(-1));
            s_je[idx] = 0u;
        }
        __syncthreads();
        // 3. masks, 32 staged j atoms per warp pass; lane = i atom, one ballot per
        //    j.  Pairs at the cutoff band or among the i atom's exclusion partners
        //    are settled after the pass (rare): FP64 reference test, exclusions.
        for (int g = wib; g < ngroups; g += BW) {
            const float4* pjs = s_jx + 32 * g;
            uint32_t rare = 0;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const float4 pj = pjs[j];
                const int a2 = __float_as_int(pj.w);
                const float dx = pj.x - lix, dy = pj.y - liy, dz = pj.z - liz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const bool exr = static_cast<unsigned>(a2 - i_lo) <= static_cast<unsigned>(i_span);
                const bool in = (r2 < rc2_lo) & !exr;
                rare |= static_cast<uint32_t>((r2 < rc2_hi) & ((r2 >= rc2_lo) | exr)) << j;
                const uint32_t m = __ballot_sync(FULL, in);
                if (lane == 0) s_msk[32 * g + j] = m;
            }
            __syncwarp();
            while (rare) {
                const int j = __ffs(rare) - 1;
                rare &= rare - 1;
                const float4 pj = pjs[j];
                const int a2 = __float_as_int(pj.w);
                const float dx = pj.x - lix, dy = pj.y - liy, dz = pj.z - liz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                bool in = (r2 < rc2_lo) || ref_member(d, ai, a2, L, invL, rc2);
                if (in && static_cast<unsigned>(a2 - i_lo) <= static_cast<unsigned>(i_span)) {
                    if (i_e1 - i_e0 <= 8) {
#pragma unroll
                        for (int q = 0; q < 8; ++q) in &= (iex[q] != a2);
                    } else {
                        for (int e = i_e0; e < i_e1; ++e) in &= (d.ex_list[e] != a2);
                    }
                }
                if (in) atomicOr(&s_msk[32 * g + j], 1u << lane);
            }
        }
        // general path for candidates that need several periodic images
        for (int k = wib; k < nc; k += BW)
            if (!(s_cinfo[k] & ONE_IMAGE)) general_candidate(s_cand[k]);
        __syncthreads();
        // 4. ordered compaction of the non-empty entries (s_jx reused), whole chunks out
        uint32_t* s_oe = reinterpret_cast<uint32_t*>(s_jx);
        uint32_t* s_om = s_oe + (MAXC * 32 + 32);
        if (tid < carry_n) {
            s_oe[tid] = s_carry_e[tid];
            s_om[tid] = s_carry_m[tid];
        }
        int base = carry_n;
        for (int e0 = 0; e0 < nj; e0 += NT_B) {
            const int idx = e0 + tid;
            uint32_t m = 0u, e = 0u;
            if (idx < nj) {
                m = s_msk[idx];
                e = s_je[idx];
                // within the i-tile itself only pairs i < j
                const int js = static_cast<int>(e & 0x03FFFFFFu);
                if ((js >> 5) == I) m &= (1u << (js & 31)) - 1u;
            }
            const uint32_t b = __ballot_sync(FULL, m != 0u);
            if (lane == 0) s_wcnt[0][wib] = __popc(b);
            __syncthreads();
            int before = base, tot = 0;
#pragma unroll
            for (int w = 0; w < BW; ++w) {
                before += (w < wib) ? s_wcnt[0][w] : 0;
                tot += s_wcnt[0][w];
            }
            if (m) {
                const int pos = before + __popc(b & ((1u << lane) - 1u));
                s_oe[pos] = e;
                s_om[pos] = m;
            }
            base += tot;
            __syncthreads();
        }
        const int nfull = base >> 5;
        if (nfull > 0) {
            if (tid == 0) {
                const int c0 = atomicAdd(&s->n_chunks, nfull);
                s_c0 = c0;
                if (c0 + nfull > R.chunk_cap) set_status(s, ST_CAPACITY);
            }
            __syncthreads();
            const int c0 = s_c0;
            for (int idx = tid; idx < nfull * 32; idx += NT_B) {
                const int c = c0 + (idx >> 5);
                if (c >= R.chunk_cap) continue;
                const int g = R.chunk_begin + c;
                if ((idx & 31) == 0) d.chunk_itile[g] = I;
                d.chunk_j[32 * g + (idx & 31)] = s_oe[idx];
                d.chunk_mask[32 * g + (idx & 31)] = s_om[idx];
            }
        }
        carry_n = base - 32 * nfull;
        if (tid < carry_n) {
            s_carry_e[tid] = s_oe[32 * nfull + tid];
            s_carry_m[tid] = s_om[32 * nfull + tid];
        }
        __syncthreads();
    }
    // merge the carry and the general path's leftovers: warp 0 flushes them
    if (lane == 0) s_left[wib] = nbuf;
    __syncthreads();
    if (wib == 0) {
        for (int w = 1; w < BW; ++w) {
            const int nl = s_left[w];
            for (int base = 0; base < nl; base += 32) {
                const bool mine = base + lane < nl;
                push(mine ? s_e[w][base + lane] : 0u, mine ? s_m[w][base + lane] : 0u);
            }
        }
        push(lane < carry_n ? s_carry_e[lane] : 0u, lane < carry_n ? s_carry_m[lane] : 0u);
        if (nbuf > 0) flush_chunk(s_e[0], s_m[0], nbuf);
    }
}

// R7: close the rebuild -- capacity check, counters, flat chunk numbering --
// by one warp: each lane takes a contiguous run of replicas, a warp scan
// places the runs.
__device__ __forceinline__ void rebuild_finish(const Dev& d, int lane) {
    const int n = d.n_rep;
    const int per = (n + 31) >> 5;
    const int r0 = min(lane * per, n), r1 = min(r0 + per, n);
    int sum = 0;
    for (int r = r0; r < r1; ++r) {
        RepState* s = d.st + r;
        if (s->rebuild) {
            if (s->n_chunks > d.rep[r].chunk_cap) {
                s->status |= ST_CAPACITY;
                s->n_chunks = d.rep[r].chunk_cap;
            }
            s->rebuild = 0;
            s->lj_counter = 0;
            s->list_builds += 1;
            s->L_build = s->L;
        }
        sum += s->n_chunks;
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    int run = incl - sum;
    for (int r = r0; r < r1; ++r) {
        d.chunk_prefix[r] = run;
        run += d.st[r].n_chunks;
    }
    if (lane == 31) d.chunk_prefix[n] = incl;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier over the co-resident blocks of the cooperative launch:
// bar[0] counts arrivals, bar[1] is the generation.  A wait gives up after one
// second, records ST_TIMEOUT and returns false (the caller leaves the kernel).
__device__ bool grid_barrier(const Dev& d) {
    __shared__ int ok;
    unsigned* bar = d.grid_bar;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned gen = ld_acquire(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            bar[0] = 0;
            __threadfence();
            st_release(bar + 1, gen + 1);
        } else {
            const unsigned long long t0 = global_ns();
            while (ld_acquire(bar + 1) == gen) {
                if (global_ns() - t0 > 1000000000ull) {
                    atomicOr(&d.st[0].status, ST_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

// The whole rebuild as one cooperative launch: R0 decides (all blocks read the
// same flags, so a step without a rebuild leaves at once), then R1..R7 with a
// grid barrier between phases.  Only replicas whose `rebuild` flag is set are
// touched.
__global__ void __launch_bounds__(NT_B, 4) k_rebuild(Dev d, const int* bin_rep) {
    int any = 0;
    for (int r = 0; r < d.n_rep; ++r) any |= d.st[r].rebuild;
    if (!any) return;
    const int tid = threadIdx.x, lane = tid & 31;
    const int gthreads = gridDim.x * NT_B;
    const int gtid = blockIdx.x * NT_B + tid;
    const int gwarp = gtid >> 5, nwarps = gthreads >> 5;
    // R0: chunk counters of the replicas that rebuild, work counter of R6 and
    // the prefixes of the rebuilding replicas' atoms, sort cells and tiles (the
    // later phases visit only those)
    if (gtid == 0) *d.build_work = 0;
    for (int r = gtid; r < d.n_rep; r += gthreads)
        if (d.st[r].rebuild) d.st[r].n_chunks = 0;
    if (blockIdx.x == 0 && tid < 96) {  // warps 0, 1, 2: atoms, sort cells, tiles
        const int kind = tid >> 5;
        int* pre = d.build_prefix + kind * (d.n_rep + 1);
        int run = 0;
        for (int base = 0; base < d.n_rep; base += 32) {
            const int r = base + lane;
            int v = 0;
            if (r < d.n_rep && d.st[r].rebuild) {
                const Rep& R = d.rep[r];
                v = kind == 0 ? R.n_atoms : (kind == 1 ? R.nvx * R.nvx * R.nvz : R.n_tiles);
            }
            int incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            if (r < d.n_rep) pre[r] = run + incl - v;
            run += __shfl_sync(FULL, incl, 31);
        }
        if (lane == 0) pre[d.n_rep] = run;
    }
    if (!grid_barrier(d)) return;
    // the phases below visit only the rebuilding replicas' atoms, cells and tiles
    const int* pa = d.build_prefix;
    const int* pb = pa + d.n_rep + 1;
    const int* pt = pb + d.n_rep + 1;
    const int n_a = pa[d.n_rep], n_b = pb[d.n_rep], n_t = pt[d.n_rep];
    for (int w = gtid; w < n_a; w += gthreads) {
        const int r = chunk_replica(pa, d.n_rep, w);
        bin_atom(d, d.rep[r].atom_begin + (w - pa[r]));
    }
    if (!grid_barrier(d)) return;
    for (int r = blockIdx.x; r < d.n_rep; r += gridDim.x)
        if (d.st[r].rebuild) bin_scan_replica(d, r);
    if (!grid_barrier(d)) return;
    for (int w = gtid; w < n_a; w += gthreads) {
        const int r = chunk_replica(pa, d.n_rep, w);
        bin_scatter_atom(d, d.rep[r].atom_begin + (w - pa[r]));
    }
    if (!grid_barrier(d)) return;
    for (int w = gwarp; w < n_b; w += nwarps) {
        const int r = chunk_replica(pb, d.n_rep, w);
        bin_sort_warp(d, bin_rep, d.rep[r].bin_begin + (w - pb[r]), lane);
    }
    if (!grid_barrier(d)) return;
    for (int w = gwarp; w < n_t; w += nwarps) {
        const int r = chunk_replica(pt, d.n_rep, w);
        tile_warp(d, d.rep[r].tile_begin + (w - pt[r]), lane);
    }
    if (!grid_barrier(d)) return;
    // R6: the rebuilding replicas' i-tiles taken one at a time from a counter
    // (their costs differ)
    __shared__ int s_tile;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(d.build_work, 1);
        __syncthreads();
        const int w = s_tile;
        __syncthreads();
        if (w >= n_t) break;
        const int r = chunk_replica(pt, d.n_rep, w);
        build_tile(d, d.rep[r].tile_begin + (w - pt[r]));
    }
    if (!grid_barrier(d)) return;
    if (gtid < 32) rebuild_finish(d, lane);
}

void launch_rebuild(const Dev& d, const int* bin_rep, int n_sm, cudaStream_t st, long long* nlaunch) {
    static int per_sm = 0;  // co-resident blocks per SM (same on every device of one kind)
    if (per_sm == 0) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_rebuild, NT_B, 0);
        per_sm = n < 1 ? 1 : (n > 4 ? 4 : n);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(n_sm * per_sm));
    cfg.blockDim = dim3(NT_B);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_rebuild, d, bin_rep);
    *nlaunch += 1;
}

}  // namespace dmd
