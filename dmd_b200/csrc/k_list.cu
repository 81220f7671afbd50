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
    // a position that is not finite is reported and binned as image 0, cell 0:
    // every float-to-integer conversion below takes a clamped, finite value
    if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]))) set_status(s, ST_NAN);
    for (int k = 0; k < 3; ++k) {
        const int nk = (k < 2) ? R.nvx : R.nvz;
        double f = floor(p[k] / L);
        im[k] = fabs(f) < 1e9 ? static_cast<int>(f) : 0;
        double w = p[k] - f * L;
        const double cw = w / L * nk;
        v[k] = cw >= 0.0 ? (cw < nk ? static_cast<int>(cw) : nk - 1) : 0;
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
    if (d.tile_nch && lane == 0) {  // chunk counters of the i-cluster regrouping
        d.tile_nch[t] = 0;
        d.tile_fill[t] = 0;
    }
}

// Entry encoding: bits 0..25 j slot, 26..31 image shift (mx+1, my+1, mz+1), 2 bits each.
//
// R6: chunk list, one block of BW warps per i-tile (lane = i atom), tiles taken
// from a counter.  Two builders, chosen per replica by its tile count alone (so
// a replica's chunks do not depend on what else is in the table):
//
// Plain scan (replicas below CELL_TILES tiles), in batches of up to MAXC
// candidate j-tiles (J >= I, same replica, conservative bounding-box test,
// enumerated in tile order over every later tile):
//  1. enumerate the batch's candidates into shared memory;
//  2. stage their j atoms in the i-tile's frame (all threads, independent loads);
//  3. per candidate (round-robin over warps), lane = i atom: one ballot per j
//     atom gives that j's 32-bit mask.  A candidate whose two tiles need more
//     than one periodic image (small boxes) takes the general per-pair path;
//  4. compact the non-empty entries in order and write whole chunks with one
//     counter update per batch; fewer than 32 left over carry to the next batch.
//
// Cell ranges (larger replicas), where the scan over every later tile would
// dominate:
//  1. candidate j-tiles (J >= I, same replica): the tiles that hold the atoms
//     of the sort grid's columns and z slabs within list-cutoff reach of the
//     i-tile's bounding box, as ranges of tiles in slot order (every tile
//     once); boxes too small for that scan every later tile.  Warp w takes
//     the w-th quarter of the candidate indices; a conservative bounding-box
//     test keeps the candidates;
//  2. the j atoms of up to GRP candidates are loaded together, brought into
//     the i-tile's frame (FP32) and those within the list cutoff of the
//     i-tile's box are staged in order;
//  3. per 32 staged j atoms, one ballot per j gives that j's 32-bit mask over
//     the i lanes; a candidate whose two tiles need more than one periodic
//     image (small boxes) takes the general per-pair path instead;
//  4. each warp appends its non-empty entries in order and writes whole chunks
//     (reserved OUTCAP / 32 at a time); the fewer than 32 left in each warp
//     are then chained in warp order and written by warp 0.  The chunks of an
//     i-tile (and their number, that of one stream) depend on the replica
//     alone, not on the block or launch shape that built them.
// Per pair: FP32 on tile-local coordinates, the reference's FP64 expression
// within 1e-5 of the cutoff; PHYS drops excluded pairs.
constexpr int BW = 4;
constexpr int NT_B = 32 * BW;
constexpr int MAXC = 48;        // plain scan: candidates per batch
constexpr int CELL_TILES = 2048;  // replicas with at least this many tiles use cell ranges
constexpr int MAXR = 128;       // cell ranges: column z-runs per i-tile before the plain scan takes over
constexpr int OUTCAP = 256;     // cell ranges: entries buffered per warp before chunks are reserved
constexpr int GRP = 4;          // cell ranges: candidate j-tiles whose atoms are loaded together
constexpr int STAGE = 32 * GRP + 64;  // staged j atoms: < 32 left over + one load group + padding
constexpr float FAR = 1e18f;  // coordinate of padding atoms: r^2 overflows to +inf
constexpr int ONE_IMAGE = 1 << 6;

// Per-warp scratch of the cell-range builder.
struct TileScratch {
    float4 jx[STAGE];          // staged j atoms in the i-tile frame (w = atom index bits)
    uint32_t je[STAGE];        // their entry words
    uint32_t msk[32];          // masks of one group of 32 staged j atoms
    uint32_t oe[OUTCAP + 32];  // entries waiting to be written as chunks
    uint32_t om[OUTCAP + 32];
    int r0[MAXR];              // candidate tile ranges: first tile
    int rp[MAXR + 1];          // exclusive prefix of the range lengths
    int ia[32];                // i atoms and their tile-local coordinates (general path)
    float ilx[32], ily[32], ilz[32];
    int nr, total;             // ranges and candidate indices (warp 0's copy is used)
    int nleft;                 // entries left after this warp's whole chunks
};

// The reference's minimum-image r^2 < rc2 test in FP64 (src/core/pbc.h semantics).
__device__ __forceinline__ bool ref_member(const Dev& d, int ai, int aj, double L, double invL, double rc2) {
    double ex = __dsub_rn(d.x[aj], d.x[ai]), ey = __dsub_rn(d.y[aj], d.y[ai]), ez = __dsub_rn(d.z[aj], d.z[ai]);
    ex = __dsub_rn(ex, __dmul_rn(round(__dmul_rn(ex, invL)), L));
    ey = __dsub_rn(ey, __dmul_rn(round(__dmul_rn(ey, invL)), L));
    ez = __dsub_rn(ez, __dmul_rn(round(__dmul_rn(ez, invL)), L));
    return r2_ref(ex, ey, ez) < rc2;
}

// Block scratch of the plain-scan builder.
struct ScanScratch {
    float lx[32], ly[32], lz[32];
    int a[32];
    uint32_t e[BW][64], m[BW][64];  // general path: per-warp entry buffers
    int left[BW];
    int cand[MAXC], cinfo[MAXC];
    float4 coff[MAXC];              // j-tile frame -> i-tile frame (FP32)
    float4 jx[MAXC * 32];           // staged j atoms (w = atom index bits); reused for compaction
    uint32_t je[MAXC * 32];         // staged j entry words
    uint32_t msk[MAXC * 32];
    uint32_t carry_e[32], carry_m[32];
    int wcnt[4][BW];
    int jnext, c0;
};

__device__ __forceinline__ void build_tile_scan(const Dev& d, int I, ScanScratch& O) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wib = tid >> 5;
    float(&s_lx)[32] = O.lx;
    float(&s_ly)[32] = O.ly;
    float(&s_lz)[32] = O.lz;
    int(&s_a)[32] = O.a;
    uint32_t(&s_e)[BW][64] = O.e;
    uint32_t(&s_m)[BW][64] = O.m;
    int(&s_left)[BW] = O.left;
    int(&s_cand)[MAXC] = O.cand;
    int(&s_cinfo)[MAXC] = O.cinfo;
    float4(&s_coff)[MAXC] = O.coff;
    float4(&s_jx)[MAXC * 32] = O.jx;
    uint32_t(&s_je)[MAXC * 32] = O.je;
    uint32_t(&s_msk)[MAXC * 32] = O.msk;
    uint32_t(&s_carry_e)[32] = O.carry_e;
    uint32_t(&s_carry_m)[32] = O.carry_m;
    int(&s_wcnt)[4][BW] = O.wcnt;
    int& s_jnext = O.jnext;
    int& s_c0 = O.c0;
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

__device__ __forceinline__ int mod_n(int a, int n) {
    const int m = a % n;
    return m < 0 ? m + n : m;
}

// Sort-grid cells [lo, lo + cnt) (modulo n) along one axis that hold every
// wrapped coordinate within `span` of c; cnt == n: all of them.  The cell
// index is R1's expression (w / L * n), which is monotonic in w.
__device__ __forceinline__ void cell_reach(double c, double span, double L, int n, int& lo, int& cnt) {
    const double fa = floor((c - span) / L * n), fb = floor((c + span) / L * n);
    lo = 0;
    cnt = n;
    // every cell when the reach covers the axis (or the coordinates are not finite)
    if (!(fb - fa + 3.0 < n) || !(fabs(fa) < 1e8) || !(fabs(fb) < 1e8)) return;
    int a = static_cast<int>(fa), b = static_cast<int>(fb);
    // R1 clamps a wrapped coordinate that rounds up to L into the last cell and
    // one just below 0 into the first
    if (mod_n(a, n) == 0) a -= 1;
    if (mod_n(b, n) == n - 1) b += 1;
    if (b - a + 1 < n) {
        lo = mod_n(a, n);
        cnt = b - a + 1;
    }
}

// k-th smallest value of the cyclic interval [lo, lo + cnt) modulo n.
__device__ __forceinline__ int nth_ascending(int lo, int cnt, int n, int k) {
    const int w = lo + cnt - n;  // values that wrapped to 0 .. w-1
    return (w > 0) ? (k < w ? k : lo + (k - w)) : lo + k;
}

__device__ __forceinline__ void build_tile_cells(const Dev& d, int I, TileScratch* SS) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    TileScratch& S = SS[wib];
    TileScratch& S0 = SS[0];
    const uint32_t lt = (1u << lane) - 1u;
    const int r = d.tile_rep[I];
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    const double L = s->L, invL = s->invL;
    const float Lf = static_cast<float>(L), hLf = 0.5f * Lf;
    const bool phys = (R.flags & F_PHYS) != 0;
    const double rc2 = R.rc_list2;
    const float rc2_lo = static_cast<float>(rc2 * (1.0 - 1e-5));
    const float rc2_hi = static_cast<float>(rc2 * (1.0 + 1e-5));
    const double bb_rc2 = rc2 * (1.0 + 1e-6) + 1e-9;
    const double cIx = d.tcx[I], cIy = d.tcy[I], cIz = d.tcz[I];
    const float hIx = d.thx[I], hIy = d.thy[I], hIz = d.thz[I];
    const int t_end = R.tile_begin + R.n_tiles;

    // this lane's i atom; a padding i lane sits far away (+FAR), padding j atoms at -FAR
    const int ai = d.atom_of_slot[32 * I + lane];
    const float4 pi = d.xl32[32 * I + lane];
    const float lix = ai >= 0 ? pi.x : FAR, liy = ai >= 0 ? pi.y : FAR, liz = ai >= 0 ? pi.z : FAR;
    S.ia[lane] = ai;
    S.ilx[lane] = pi.x;
    S.ily[lane] = pi.y;
    S.ilz[lane] = pi.z;
    // (PHYS) exclusion partners, sorted ascending, spanning [i_lo, i_lo + i_span];
    // an empty set never matches
    int i_e0 = 0, i_e1 = 0, i_lo = 0x7fffffff, i_span = 0;
    if (phys && ai >= 0) {
        i_e0 = d.ex_start[ai];
        i_e1 = d.ex_start[ai + 1];
        if (i_e1 > i_e0) {
            i_lo = d.ex_list[i_e0];
            i_span = d.ex_list[i_e1 - 1] - i_lo;
        }
    }

    // ---- 1a. candidate tile ranges (warp 0) ---------------------------------
    if (wib == 0) {
        int nr, total;
        const double rc_m = sqrt(rc2) * (1.0 + 1e-4) + 1e-6 * L;
        const int nvx = R.nvx, nvz = R.nvz;
        int xlo, xc, ylo, yc, zlo, zc;
        cell_reach(cIx, static_cast<double>(hIx) + rc_m, L, nvx, xlo, xc);
        cell_reach(cIy, static_cast<double>(hIy) + rc_m, L, nvx, ylo, yc);
        cell_reach(cIz, static_cast<double>(hIz) + rc_m, L, nvz, zlo, zc);
        const int ncol = xc * yc;
        if ((xc == nvx && yc == nvx && zc == nvz) || 2 * ncol > MAXR) {
            nr = 1;
            total = t_end - I;
            if (lane == 0) {
                S.r0[0] = I;
                S.rp[0] = 0;
                S.rp[1] = total;
            }
        } else {
            // range q = 2 * (column k) + run: columns in ascending column index
            // (x-major, y in the snake direction of its x row), the one or two z
            // runs of each column in ascending bin order
            nr = 2 * ncol;
            const int B = R.bin_begin;
            const int nb = nvx * nvx * nvz;
            const int slot_end = 32 * R.tile_begin + R.n_atoms;
            const int wz = zlo + zc - nvz;  // > 0: the z interval wraps
            int t0[4], t1[4];
            int lmax = I - 1;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = 4 * lane + u;
                t0[u] = I;  // empty: [I, I - 1]
                t1[u] = I - 1;
                if (q >= nr) continue;
                const int kcol = q >> 1, run = q & 1;
                const int ix = nth_ascending(xlo, xc, nvx, kcol / yc);
                const int ky = kcol % yc;
                const int iy = nth_ascending(ylo, yc, nvx, (ix & 1) ? yc - 1 - ky : ky);
                const int col = ix * nvx + ((ix & 1) ? nvx - 1 - iy : iy);
                // z runs as cell intervals [a0, a1], [b0, b1] (b empty unless wrapped)
                int a0, a1, b0 = 1, b1 = 0;
                if (wz > 0) {
                    a0 = 0;
                    a1 = wz - 1;
                    b0 = zlo;
                    b1 = nvz - 1;
                } else {
                    a0 = zlo;
                    a1 = zlo + zc - 1;
                }
                // bin offsets within the column (odd columns run top-down)
                if (col & 1) {
                    const int na0 = nvz - 1 - a1, na1 = nvz - 1 - a0;
                    const int nb0 = nvz - 1 - b1, nb1 = nvz - 1 - b0;
                    a0 = na0;
                    a1 = na1;
                    b0 = nb0;
                    b1 = nb1;
                    if (wz > 0) {  // ascending: b's offsets come first
                        int t = a0;
                        a0 = b0;
                        b0 = t;
                        t = a1;
                        a1 = b1;
                        b1 = t;
                    }
                }
                const int o0 = run ? b0 : a0, o1 = run ? b1 : a1;
                if (o1 < o0) continue;
                const int g0 = B + col * nvz + o0, g1 = B + col * nvz + o1;
                const int s_lo = d.bin_start[g0];
                const int s_hi = (g1 + 1 < B + nb) ? d.bin_start[g1 + 1] : slot_end;
                if (s_hi <= s_lo) continue;
                t0[u] = max(s_lo >> 5, I);
                t1[u] = (s_hi - 1) >> 5;
                lmax = max(lmax, t1[u]);
            }
            // ranges are disjoint in slots and ascending, so consecutive ones share at
            // most an end tile: start each after the largest tile of those before it
            int prev = lmax;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, prev, o);
                if (lane >= o) prev = max(prev, v);
            }
            prev = __shfl_up_sync(FULL, prev, 1);
            if (lane == 0) prev = I - 1;
            int len[4], lsum = 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                t0[u] = max(t0[u], prev + 1);
                len[u] = max(t1[u] - t0[u] + 1, 0);
                prev = max(prev, t1[u]);
                lsum += len[u];
            }
            int incl = lsum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            int run_v = incl - lsum;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = 4 * lane + u;
                if (q < nr) {
                    S.r0[q] = t0[u];
                    S.rp[q] = run_v;
                }
                run_v += len[u];
            }
            total = __shfl_sync(FULL, incl, 31);
            if (lane == 0) S.rp[nr] = total;
        }
        if (lane == 0) {
            S.nr = nr;
            S.total = total;
        }
    }
    __syncthreads();
    const int nr = S0.nr, total = S0.total;
    // this warp's quarter of the candidate indices
    const int v_beg = static_cast<int>(static_cast<long long>(total) * wib / BW);
    const int v_end = static_cast<int>(static_cast<long long>(total) * (wib + 1) / BW);

    // ---- output: ordered entries, written as whole chunks reserved in bulk ---
    int no = 0;  // entries waiting in S.oe / S.om (warp-uniform)
    auto write_chunks = [&](int count) {
        const int k = (count + 31) >> 5;
        int c0 = 0;
        if (lane == 0) c0 = atomicAdd(&s->n_chunks, k);
        c0 = __shfl_sync(FULL, c0, 0);
        if (c0 + k > R.chunk_cap && lane == 0) set_status(s, ST_CAPACITY);
        for (int q = 0; q < k && c0 + q < R.chunk_cap; ++q) {
            const int g = R.chunk_begin + c0 + q;
            const int idx = 32 * q + lane;
            if (lane == 0) d.chunk_itile[g] = I;
            d.chunk_j[32 * g + lane] = idx < count ? S.oe[idx] : 0u;
            d.chunk_mask[32 * g + lane] = idx < count ? S.om[idx] : 0u;
        }
    };
    auto emit = [&](uint32_t e, uint32_t m) {
        const uint32_t has = __ballot_sync(FULL, m != 0u);
        const int pos = no + __popc(has & lt);
        if (m) {
            S.oe[pos] = e;
            S.om[pos] = m;
        }
        no += __popc(has);
        __syncwarp();
        if (no >= OUTCAP) {
            write_chunks(OUTCAP);
            __syncwarp();
            if (lane < no - OUTCAP) {
                S.oe[lane] = S.oe[lane + OUTCAP];
                S.om[lane] = S.om[lane + OUTCAP];
            }
            no -= OUTCAP;
            __syncwarp();
        }
    };

    // ---- 3. masks of `count` (<= 32) staged j atoms from `base` (lane = i atom)
    int ns = 0, s0 = 0;  // staged j atoms S.jx[s0, s0 + ns) (warp-uniform)
    auto mask_group = [&](int base, int count) {
        if (lane >= count) {
            S.jx[base + lane] = make_float4(-FAR, -FAR, -FAR, __int_as_float(-1));
            S.je[base + lane] = 0u;
        }
        __syncwarp();
        const float4* pjs = S.jx + base;
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
            if (lane == 0) S.msk[j] = m;
        }
        __syncwarp();
        // pairs at the cutoff band or among the i atom's exclusion partners (rare):
        // the FP64 reference test, then the exclusions
        while (rare) {
            const int j = __ffs(rare) - 1;
            rare &= rare - 1;
            const float4 pj = pjs[j];
            const int a2 = __float_as_int(pj.w);
            const float dx = pj.x - lix, dy = pj.y - liy, dz = pj.z - liz;
            const float r2 = dx * dx + dy * dy + dz * dz;
            bool in = (r2 < rc2_lo) || ref_member(d, ai, a2, L, invL, rc2);
            if (in && static_cast<unsigned>(a2 - i_lo) <= static_cast<unsigned>(i_span))
                for (int e = i_e0; e < i_e1; ++e) in &= (d.ex_list[e] != a2);
            if (in) atomicOr(&S.msk[j], 1u << lane);
        }
        __syncwarp();
        // lane = staged j: within the i-tile itself only pairs i < j
        uint32_t m = S.msk[lane];
        const uint32_t e = S.je[base + lane];
        const int js = static_cast<int>(e & 0x03FFFFFFu);
        if (lane >= count) m = 0u;
        if ((js >> 5) == I) m &= (1u << (js & 31)) - 1u;
        __syncwarp();
        emit(e, m);
    };

    // ---- general path: one candidate with several periodic images, lane = j --
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
        if (aj >= 0) todo = (J == I) ? lt : 0xffffffffu;
        while (__any_sync(FULL, todo != 0)) {
            uint32_t bits = 0, rest = 0, code0 = 0xffffffffu;
            for (uint32_t t = todo; t; t &= t - 1) {
                const int i = __ffs(t) - 1;
                const int a_i = S.ia[i];
                if (a_i < 0) continue;
                float dx = jx - S.ilx[i], dy = jy - S.ily[i], dz = jz - S.ilz[i];
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
            emit(static_cast<uint32_t>(js) | ((bits ? code0 : 0u) << 26), bits);
            todo = rest;
        }
    };

    // ---- 1b/2. candidates in tile order --------------------------------------
    // One step per pass, each kind of work at one place in the code: a mask
    // group when 32 atoms are staged (or fewer before a general candidate and at
    // the end), the next 32 candidate indices, a general candidate, or the
    // atoms of up to GRP one-image candidates.
    const double hL = 0.5 * L;
    int v0 = v_beg;
    uint32_t cm = 0, gm = 0;  // candidates of the current 32 indices not yet taken; general ones
    int J = 0, info = 0;      // this lane's candidate among them
    float4 off = make_float4(0.f, 0.f, 0.f, 0.f);
    for (;;) {
        const bool at_end = cm == 0u && v0 >= v_end;
        const bool next_general = cm != 0u && ((gm >> (__ffs(cm) - 1)) & 1u);
        if (ns >= 32 || (ns > 0 && (at_end || next_general))) {
            const int cnt = min(ns, 32);
            mask_group(s0, cnt);
            s0 += cnt;
            ns -= cnt;
            continue;
        }
        if (at_end) break;
        if (cm == 0u) {
            const int v = v0 + lane;
            v0 += 32;
            bool cand = false;
            if (v < v_end) {
                // the range holding v: the last one whose prefix is <= v
                int lo = 0, hi = nr - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (S0.rp[mid] <= v) lo = mid;
                    else hi = mid - 1;
                }
                J = S0.r0[lo] + (v - S0.rp[lo]);
                double dx = d.tcx[J] - cIx, dy = d.tcy[J] - cIy, dz = d.tcz[J] - cIz;
                const double rx0 = round(dx * invL), ry0 = round(dy * invL), rz0 = round(dz * invL);
                dx -= L * rx0;
                dy -= L * ry0;
                dz -= L * rz0;
                const double ex = (double)(hIx + d.thx[J]), ey = (double)(hIy + d.thy[J]),
                             ez = (double)(hIz + d.thz[J]);
                const double gx = fmax(fabs(dx) - ex, 0.0), gy = fmax(fabs(dy) - ey, 0.0),
                             gz = fmax(fabs(dz) - ez, 0.0);
                cand = gx * gx + gy * gy + gz * gz <= bb_rc2;
                // one periodic image serves every pair of the two tiles when their
                // extents around the centre displacement stay inside half a box
                const bool one = fabs(dx) + ex < hL && fabs(dy) + ey < hL && fabs(dz) + ez < hL;
                info = (static_cast<int>(rx0) + 1) | ((static_cast<int>(ry0) + 1) << 2) |
                       ((static_cast<int>(rz0) + 1) << 4) | (one ? ONE_IMAGE : 0);
                off = make_float4(static_cast<float>(dx), static_cast<float>(dy), static_cast<float>(dz), 0.f);
            }
            cm = __ballot_sync(FULL, cand);
            gm = __ballot_sync(FULL, cand && !(info & ONE_IMAGE));
            continue;
        }
        if (next_general) {
            const int k = __ffs(cm) - 1;
            cm &= cm - 1;
            general_candidate(__shfl_sync(FULL, J, k));
            continue;
        }
        // up to GRP one-image candidates before the next general one, in order;
        // the fewer than 32 atoms left staged move to the front first
        if (s0 > 0) {
            float4 pk = make_float4(0.f, 0.f, 0.f, 0.f);
            uint32_t ek = 0u;
            if (lane < ns) {
                pk = S.jx[s0 + lane];
                ek = S.je[s0 + lane];
            }
            __syncwarp();
            if (lane < ns) {
                S.jx[lane] = pk;
                S.je[lane] = ek;
            }
            s0 = 0;
            __syncwarp();
        }
        const uint32_t gpend = gm & cm;  // general candidates not yet taken (none is lowest)
        const uint32_t avail = gpend ? (cm & ((gpend & (0u - gpend)) - 1u)) : cm;
        uint32_t take = avail;
        int kk[GRP], aj[GRP];
        float4 pg[GRP];
#pragma unroll
        for (int u = 0; u < GRP; ++u) {
            kk[u] = take ? __ffs(take) - 1 : -1;
            take &= take - 1;
            const int Jk = __shfl_sync(FULL, J, kk[u] & 31);
            aj[u] = -1;
            pg[u] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (kk[u] >= 0) {
                aj[u] = d.atom_of_slot[32 * Jk + lane];
                pg[u] = d.xl32[32 * Jk + lane];
            }
        }
        cm &= ~(avail & ~take);  // the candidates taken
#pragma unroll
        for (int u = 0; u < GRP; ++u) {
            const int k = kk[u] & 31;
            const int Jk = __shfl_sync(FULL, J, k);
            const int ik = __shfl_sync(FULL, info, k);
            const float ox = __shfl_sync(FULL, off.x, k), oy = __shfl_sync(FULL, off.y, k),
                        oz = __shfl_sync(FULL, off.z, k);
            bool keep = false;
            float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
            if (kk[u] >= 0 && aj[u] >= 0) {
                pj = make_float4(pg[u].x + ox, pg[u].y + oy, pg[u].z + oz, __int_as_float(aj[u]));
                const float gx = fmaxf(fabsf(pj.x) - hIx, 0.f), gy = fmaxf(fabsf(pj.y) - hIy, 0.f),
                            gz = fmaxf(fabsf(pj.z) - hIz, 0.f);
                keep = gx * gx + gy * gy + gz * gz <= rc2_hi * 1.0001f + 1e-6f;
            }
            const uint32_t code = static_cast<uint32_t>((2 - (ik & 3)) | ((2 - ((ik >> 2) & 3)) << 2) |
                                                        ((2 - ((ik >> 4) & 3)) << 4));
            const uint32_t kb = __ballot_sync(FULL, keep);
            if (keep) {
                const int pos = ns + __popc(kb & lt);
                S.jx[pos] = pj;
                S.je[pos] = static_cast<uint32_t>(32 * Jk + lane) | (code << 26);
            }
            ns += __popc(kb);
        }
        __syncwarp();
    }
    // whole chunks of this warp; the rest (< 32) moves to the front
    const int whole = no & ~31;
    if (whole > 0) {
        write_chunks(whole);
        __syncwarp();
        uint32_t e = 0u, m = 0u;
        if (lane < no - whole) {
            e = S.oe[whole + lane];
            m = S.om[whole + lane];
        }
        __syncwarp();
        if (lane < no - whole) {
            S.oe[lane] = e;
            S.om[lane] = m;
        }
        no -= whole;
    }
    if (lane == 0) S.nleft = no;
    __syncthreads();
    if (wib == 0) {
        // the leftovers of the other warps, in warp order, after warp 0's own
        for (int w = 1; w < BW; ++w) {
            const int nl = SS[w].nleft;
            emit(lane < nl ? SS[w].oe[lane] : 0u, lane < nl ? SS[w].om[lane] : 0u);
        }
        if (no > 0) write_chunks(no);
    }
    __syncthreads();
}

// R6 block scratch: one builder runs at a time.
// R11 per-warp staging of one i-cluster row (fewer than 32 entries carried
// plus one chunk's 32).
constexpr int CL_STAGE = 64;
struct ClusterScratch {
    uint32_t e[BW][CL_STAGE];
    uint8_t m[BW][CL_STAGE];
};

union BuildScratch {
    ScanScratch scan;
    TileScratch cells[BW];
    ClusterScratch cl;  // R11, after the list build is complete
};

// R7: close the rebuild -- capacity check, counters, flat chunk numbering --
// by one warp: each lane takes a contiguous run of replicas, a warp scan
// places the runs.  With the i-cluster regrouping to follow (d.cl_j), it also
// numbers the rebuilding replicas' chunks (build_prefix[3]) and leaves their
// `rebuild` flags for the regrouping's closing phase to clear.
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ void rebuild_finish(const Dev& d, int lane) {
    const int n = d.n_rep;
    const int per = (n + 31) >> 5;
    const int r0 = min(lane * per, n), r1 = min(r0 + per, n);
    const bool regroup = d.cl_j != nullptr;
    int sum = 0, sum_rb = 0;
    for (int r = r0; r < r1; ++r) {
        RepState* s = d.st + r;
        if (s->rebuild) {
            if (s->n_chunks > d.rep[r].chunk_cap) {
                s->status |= ST_CAPACITY;
                s->n_chunks = d.rep[r].chunk_cap;
            }
            if (!regroup) s->rebuild = 0;
            s->lj_counter = 0;
            s->list_builds += 1;
            s->L_build = s->L;
            sum_rb += s->n_chunks;
        }
        sum += s->n_chunks;
    }
    const int incl = warp_incl_scan(sum, lane);
    int run = incl - sum;
    for (int r = r0; r < r1; ++r) {
        d.chunk_prefix[r] = run;
        run += d.st[r].n_chunks;
    }
    if (lane == 31) d.chunk_prefix[n] = incl;
    if (regroup) {
        int* pc = d.build_prefix + 3 * (n + 1);
        const int incl_rb = warp_incl_scan(sum_rb, lane);
        int run_rb = incl_rb - sum_rb;
        for (int r = r0; r < r1; ++r) {
            pc[r] = run_rb;
            if (d.st[r].rebuild) run_rb += d.st[r].n_chunks;
        }
        if (lane == 31) pc[n] = incl_rb;
    }
}

// ---- i-cluster regrouping (R8 .. R12, mixed precision only) -----------------
// The pair list of every rebuilt replica regrouped by 8-atom i-cluster: for
// i-tile I and k = 0..3, cluster 4 I + k holds the entries of I's chunks whose
// mask has a bit among lanes 8k .. 8k+7, with those 8 bits as the entry's
// mask, packed 32 to a row.  The pair set is the same bit for bit; the
// cluster's j atoms are those within the list cutoff of its 8 atoms rather
// than of all 32, so far fewer of the (i, j) lane pairs a row evaluates are
// empty.  The order is canonical -- a tile's chunks sorted by their first
// entry word (unique within a tile), entries in lane order -- so the rows do
// not depend on the order in which the builders allocated the chunks.

// R9: exclusive scan of one replica's per-tile chunk counts into tile_c0 (the
// tile's first position in chunk_order), by one block.
__device__ __forceinline__ void tile_scan_replica(const Dev& d, int r) {
    __shared__ int s_warp[NT_B / 32];
    const Rep& R = d.rep[r];
    const int nt = R.n_tiles;
    const int per = (nt + NT_B - 1) / NT_B;
    const int t0 = R.tile_begin + min(static_cast<int>(threadIdx.x) * per, nt);
    const int t1 = min(t0 + per, R.tile_begin + nt);
    int local = 0;
    for (int t = t0; t < t1; ++t) local += d.tile_nch[t];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int incl = warp_incl_scan(local, lane);
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    int off = 0;
    for (int k = 0; k < w; ++k) off += s_warp[k];
    int run = R.chunk_begin + off + incl - local;
    for (int t = t0; t < t1; ++t) {
        d.tile_c0[t] = run;
        run += d.tile_nch[t];
    }
    __syncthreads();
}

// R11a: one warp per rebuilt i-tile puts its chunks in canonical order: rank
// by (first entry word, then position) -- the first entry words of a tile's
// chunks are distinct, so the order does not depend on how the builders
// allocated them.
__device__ __forceinline__ void sort_tile_chunks(const Dev& d, int t, int lane) {
    const int n = d.tile_nch[t];
    const int c0 = d.tile_c0[t];
    const int* ids = d.chunk_order + c0;
    int* sorted = d.chunk_sorted + c0;
    for (int base = 0; base < n; base += 32) {
        const int mine = base + lane;
        const int id = mine < n ? ids[mine] : -1;
        const uint32_t key = id >= 0 ? d.chunk_j[32LL * id] : 0xffffffffu;
        int rank = 0;
        for (int b2 = 0; b2 < n; b2 += 32) {
            const int other = b2 + lane;
            const uint32_t ok = other < n ? d.chunk_j[32LL * ids[other]] : 0xffffffffu;
            for (int k = 0; k < 32 && b2 + k < n; ++k) {
                const uint32_t kk = __shfl_sync(FULL, ok, k);
                rank += (kk < key || (kk == key && b2 + k < mine)) ? 1 : 0;
            }
        }
        if (id >= 0) sorted[rank] = id;
    }
}

// R11b: one warp per i-cluster (cluster 4 t + q of a rebuilt tile t) streams
// the tile's chunks in canonical order and packs the entries with a bit among
// lanes 8q .. 8q+7 into 32-entry rows.  It reserves the most rows the cluster
// can need (one per chunk plus a partial one; 4 (chunks + tiles) in all, the
// capacity) and records the rows it wrote.  The next chunk's ids, entries and
// masks are loaded while the current one is packed.
__device__ __forceinline__ void cluster_rows(const Dev& d, int cl, int lane, uint32_t* se, uint8_t* sm) {
    const int t = cl >> 2, q = cl & 3;
    const int r = d.tile_rep[t];
    RepState* s = d.st + r;
    const Rep& R = d.rep[r];
    const int n = d.tile_nch[t];
    const int* sorted = d.chunk_sorted + d.tile_c0[t];
    int base = 0;
    if (lane == 0) base = atomicAdd(&s->n_cl, n + 1);
    base = __shfl_sync(FULL, base, 0);
    if (base + n + 1 > R.cl_cap) {  // cannot happen with cl_cap = 4 chunk_cap + 4 n_tiles
        if (lane == 0) {
            set_status(s, ST_CAPACITY);
            d.cl_job[cl] = make_int2(0, 0);
        }
        return;
    }
    const int first = R.cl_begin + base;
    int g = first;
    int fill = 0;
    int ids = n > 0 ? sorted[min(lane, n - 1)] : 0;  // ids of chunks 32 b .. 32 b + 31
    long long c = __shfl_sync(FULL, ids, 0);
    uint32_t e = n > 0 ? d.chunk_j[32 * c + lane] : 0u;
    uint32_t m = n > 0 ? d.chunk_mask[32 * c + lane] : 0u;
    for (int k = 0; k < n; ++k) {
        // next chunk's data, in flight while this one is packed
        const int k1 = k + 1;
        if ((k1 & 31) == 0 && k1 < n) ids = sorted[min(k1 + lane, n - 1)];
        uint32_t e1 = 0u, m1 = 0u;
        if (k1 < n) {
            const long long c1 = __shfl_sync(FULL, ids, k1 & 31);
            e1 = d.chunk_j[32 * c1 + lane];
            m1 = d.chunk_mask[32 * c1 + lane];
        }
        const uint32_t m8 = (m >> (8 * q)) & 0xffu;
        const uint32_t has = __ballot_sync(FULL, m8 != 0);
        const int pos = fill + __popc(has & ((1u << lane) - 1u));
        if (m8) {
            se[pos] = e;
            sm[pos] = static_cast<uint8_t>(m8);
        }
        fill += __popc(has);
        __syncwarp();
        if (fill >= 32) {
            d.cl_j[32LL * g + lane] = se[lane];
            d.cl_m[32LL * g + lane] = sm[lane];
            ++g;
            const uint32_t te = se[lane + 32];
            const uint8_t tm = sm[lane + 32];
            __syncwarp();
            se[lane] = te;
            sm[lane] = tm;
            fill -= 32;
            __syncwarp();
        }
        e = e1;
        m = m1;
    }
    if (fill > 0) {
        d.cl_j[32LL * g + lane] = lane < fill ? se[lane] : 0u;
        d.cl_m[32LL * g + lane] = lane < fill ? sm[lane] : static_cast<uint8_t>(0);
        ++g;
    }
    __syncwarp();
    if (lane == 0) d.cl_job[cl] = make_int2(first, g - first);
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
// second (d.bar_limit_ns when set), records ST_TIMEOUT and returns false (the
// caller leaves the kernel).
__device__ bool grid_barrier(const Dev& d) {
    __shared__ int ok;
    unsigned* bar = d.grid_bar;
    const unsigned long long limit = d.bar_limit_ns ? d.bar_limit_ns : 1000000000ull;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned gen = ld_acquire(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1 + d.bar_extra) {
            bar[0] = 0;
            __threadfence();
            st_release(bar + 1, gen + 1);
        } else {
            const unsigned long long t0 = global_ns();
            while (ld_acquire(bar + 1) == gen) {
                if (global_ns() - t0 > limit) {
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
        if (d.st[r].rebuild) {
            d.st[r].n_chunks = 0;
            d.st[r].n_cl = 0;
        }
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
    // R6: the rebuilding replicas' i-tiles, one per block, taken from a counter
    // (their costs differ)
    __shared__ BuildScratch s_scr;
    __shared__ int s_tile;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(d.build_work, 1);
        __syncthreads();
        const int w = s_tile;
        __syncthreads();
        if (w >= n_t) break;
        const int r = chunk_replica(pt, d.n_rep, w);
        const int I = d.rep[r].tile_begin + (w - pt[r]);
        if (d.rep[r].n_tiles >= CELL_TILES) build_tile_cells(d, I, s_scr.cells);
        else build_tile_scan(d, I, s_scr.scan);
    }
    if (!grid_barrier(d)) return;
    if (gtid < 32) rebuild_finish(d, lane);
    if (!d.cl_j) return;  // FP64 tables keep the chunk list only
    if (!grid_barrier(d)) return;
    // R8: chunks per rebuilt i-tile
    const int* pc = pt + (d.n_rep + 1);  // build_prefix[3] (pa, pb, pt, pc), written by R7
    const int n_c = pc[d.n_rep];
    for (int w = gtid; w < n_c; w += gthreads) {
        const int r = chunk_replica(pc, d.n_rep, w);
        atomicAdd(d.tile_nch + d.chunk_itile[d.rep[r].chunk_begin + (w - pc[r])], 1);
    }
    if (!grid_barrier(d)) return;
    // R9: each tile's first position in chunk_order
    for (int r = blockIdx.x; r < d.n_rep; r += gridDim.x)
        if (d.st[r].rebuild) tile_scan_replica(d, r);
    if (!grid_barrier(d)) return;
    // R10: chunk ids grouped by tile (order within a tile fixed by R11)
    for (int w = gtid; w < n_c; w += gthreads) {
        const int r = chunk_replica(pc, d.n_rep, w);
        const int c = d.rep[r].chunk_begin + (w - pc[r]);
        const int I = d.chunk_itile[c];
        d.chunk_order[d.tile_c0[I] + atomicAdd(d.tile_fill + I, 1)] = c;
    }
    if (!grid_barrier(d)) return;
    // R11a: canonical chunk order of every rebuilt tile
    for (int w = gwarp; w < n_t; w += nwarps) {
        const int r = chunk_replica(pt, d.n_rep, w);
        sort_tile_chunks(d, d.rep[r].tile_begin + (w - pt[r]), lane);
    }
    if (!grid_barrier(d)) return;
    // R11b: the rows of every cluster of the rebuilt tiles
    const int wib = tid >> 5;
    for (int w = gwarp; w < 4 * n_t; w += nwarps) {
        const int r = chunk_replica(pt, d.n_rep, w >> 2);
        const int t = d.rep[r].tile_begin + ((w >> 2) - pt[r]);
        cluster_rows(d, 4 * t + (w & 3), lane, s_scr.cl.e[wib], s_scr.cl.m[wib]);
    }
    if (!grid_barrier(d)) return;
    // R12: the rebuild is complete
    for (int r = gtid; r < d.n_rep; r += gthreads)
        if (d.st[r].rebuild) d.st[r].rebuild = 0;
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
