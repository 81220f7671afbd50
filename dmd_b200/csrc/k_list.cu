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
__global__ void k_bin_atoms(Dev d) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= d.n_atoms) return;
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

// R2: exclusive scan of bin counts per replica (one block per replica).
__global__ void k_bin_scan(Dev d) {
    int r = blockIdx.x;
    if (!d.st[r].rebuild) return;
    const Rep& R = d.rep[r];
    const int nb = R.nvx * R.nvx * R.nvz;
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b0 = R.bin_begin + threadIdx.x * per;
    const int b1 = min(b0 + per, R.bin_begin + nb);
    int local = 0;
    for (int b = b0; b < b1; ++b) local += d.bin_count[b];
    __shared__ int sh[1024];
    sh[threadIdx.x] = local;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        int v = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += v;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - local + 32 * R.tile_begin;
    for (int b = b0; b < b1; ++b) {
        d.bin_start[b] = run;
        run += d.bin_count[b];
    }
}

// R3: scatter atoms to their bin ranges (order within a bin fixed by R4).
__global__ void k_bin_scatter(Dev d) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= d.n_atoms) return;
    if (!d.st[d.atom_rep[a]].rebuild) return;
    int b = d.atom_bin[a];
    int pos = d.bin_start[b] + atomicAdd(d.bin_fill + b, 1);
    d.sort_buf[pos] = a;
}

// R4: sort each bin by atom index (deterministic order) and reset its counters.
__global__ void k_bin_sort(Dev d, const int* bin_rep) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.n_bins) return;
    if (!d.st[bin_rep[b]].rebuild) return;
    int n = d.bin_count[b];
    if (n > 1) {
        int* p = d.sort_buf + d.bin_start[b];
        for (int i = 1; i < n; ++i) {
            int v = p[i];
            int j = i - 1;
            while (j >= 0 && p[j] > v) {
                p[j + 1] = p[j];
                --j;
            }
            p[j + 1] = v;
        }
    }
    d.bin_count[b] = 0;
    d.bin_fill[b] = 0;
}

// R5: tiles -- slot<->atom maps, reference positions, bounding boxes, mirror.
__global__ void k_tiles(Dev d) {
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= d.n_tiles) return;
    const int r = d.tile_rep[t];
    RepState* s = d.st + r;
    if (!s->rebuild) return;
    const Rep& R = d.rep[r];
    const double L = s->L;
    const int slot = 32 * t + lane;
    const int local = slot - 32 * R.tile_begin;
    const int a = (local < R.n_atoms) ? d.sort_buf[slot] : -1;
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
    if (d.xq32) {
        d.xq32[slot] = (a >= 0) ? make_float4(static_cast<float>(w[0] - c[0]), static_cast<float>(w[1] - c[1]),
                                              static_cast<float>(w[2] - c[2]), static_cast<float>(qa))
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (d.xq64) d.xq64[slot] = make_double4(xa, ya, za, qa);
}

// Entry encoding: bits 0..25 j slot, 26..31 image shift (mx+1, my+1, mz+1), 2 bits each.
//
// R6: chunk list.  A block of BW warps per i-tile; candidate j-tiles (J >= I,
// same replica) come from a conservative bounding-box test and are dealt
// round-robin to the warps.  Per pair: FP32 on tile-local coordinates, the
// reference's FP64 expression within 1e-5 of the cutoff.  Each warp packs its
// (j, mask) entries into 32-entry chunks; leftovers are merged through shared
// memory so each i-tile ends with at most one partial chunk.
constexpr int BW = 4;

__global__ void __launch_bounds__(32 * BW) k_build_pairs(Dev d) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int I = blockIdx.x;
    __shared__ float s_lx[32], s_ly[32], s_lz[32];
    __shared__ int s_a[32];
    __shared__ uint32_t s_e[BW][64], s_m[BW][64];
    __shared__ int s_left[BW];
    if (I >= d.n_tiles) return;
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
        s_a[lane] = a;
        s_lx[lane] = a >= 0 ? static_cast<float>((d.x[a] - d.imgx[a] * L) - cIx) : 0.f;
        s_ly[lane] = a >= 0 ? static_cast<float>((d.y[a] - d.imgy[a] * L) - cIy) : 0.f;
        s_lz[lane] = a >= 0 ? static_cast<float>((d.z[a] - d.imgz[a] * L) - cIz) : 0.f;
    }
    __syncthreads();
    const float hIx = d.thx[I], hIy = d.thy[I], hIz = d.thz[I];
    const int t_end = R.tile_begin + R.n_tiles;
    int nbuf = 0;        // entries buffered in s_e/s_m[wib] (warp-uniform)
    int cand_seen = 0;   // candidates enumerated so far (round-robin over warps)

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

    for (int J0 = I; J0 < t_end; J0 += 32) {
        const int Jl = J0 + lane;
        bool cand = false;
        if (Jl < t_end) {
            double dx = d.tcx[Jl] - cIx, dy = d.tcy[Jl] - cIy, dz = d.tcz[Jl] - cIz;
            dx -= L * round(dx * invL);
            dy -= L * round(dy * invL);
            dz -= L * round(dz * invL);
            double gx = fmax(fabs(dx) - (double)(hIx + d.thx[Jl]), 0.0);
            double gy = fmax(fabs(dy) - (double)(hIy + d.thy[Jl]), 0.0);
            double gz = fmax(fabs(dz) - (double)(hIz + d.thz[Jl]), 0.0);
            cand = gx * gx + gy * gy + gz * gz <= bb_rc2;
        }
        uint32_t cb = __ballot_sync(FULL, cand);
        while (cb) {
            const int J = J0 + __ffs(cb) - 1;
            cb &= cb - 1;
            if ((cand_seen++ % BW) != wib) continue;
            const int js = 32 * J + lane;
            const int aj = d.atom_of_slot[js];
            const double ddx = d.tcx[J] - cIx, ddy = d.tcy[J] - cIy, ddz = d.tcz[J] - cIz;
            const double rx0 = round(ddx * invL), ry0 = round(ddy * invL), rz0 = round(ddz * invL);
            // j atom in i-tile-local frame (centre image), exclusion partners
            float jx = 0.f, jy = 0.f, jz = 0.f;
            int ex[8];
            int nex = 0, e0 = 0, e1 = 0;
            if (aj >= 0) {
                const double wjx = d.x[aj] - d.imgx[aj] * L, wjy = d.y[aj] - d.imgy[aj] * L,
                             wjz = d.z[aj] - d.imgz[aj] * L;
                jx = static_cast<float>(wjx - cIx - rx0 * L);
                jy = static_cast<float>(wjy - cIy - ry0 * L);
                jz = static_cast<float>(wjz - cIz - rz0 * L);
                e0 = d.ex_start[aj];
                e1 = d.ex_start[aj + 1];
                if (phys) nex = e1 - e0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) ex[k] = (k < nex) ? d.ex_list[e0 + k] : -1;
            // Pairs of one j atom normally share one periodic image; in small boxes
            // (tile extent ~ L/4) several can occur.  Each pass emits the entry of
            // one image code and leaves the i atoms with other codes for the next.
            uint32_t todo = 0;
            if (aj >= 0) todo = (J == I) ? ((1u << lane) - 1u) : 0xffffffffu;
            while (__any_sync(FULL, todo != 0)) {
                uint32_t bits = 0, rest = 0, code0 = 0xffffffffu;
                for (uint32_t t = todo; t; t &= t - 1) {
                    const int i = __ffs(t) - 1;
                    const int ai = s_a[i];
                    if (ai < 0) continue;
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
                        double ex_ = __dsub_rn(d.x[aj], d.x[ai]), ey = __dsub_rn(d.y[aj], d.y[ai]),
                               ez = __dsub_rn(d.z[aj], d.z[ai]);
                        const double qx = round(__dmul_rn(ex_, invL)), qy = round(__dmul_rn(ey, invL)),
                                     qz = round(__dmul_rn(ez, invL));
                        ex_ = __dsub_rn(ex_, __dmul_rn(qx, L));
                        ey = __dsub_rn(ey, __dmul_rn(qy, L));
                        ez = __dsub_rn(ez, __dmul_rn(qz, L));
                        if (!(r2_ref(ex_, ey, ez) < rc2)) continue;
                        mx = d.imgx[aj] - d.imgx[ai] - static_cast<int>(qx);
                        my = d.imgy[aj] - d.imgy[ai] - static_cast<int>(qy);
                        mz = d.imgz[aj] - d.imgz[ai] - static_cast<int>(qz);
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
                            for (int k = 0; k < 8; ++k) excluded |= (ex[k] == ai);
                        } else {
                            for (int e = e0; e < e1; ++e) excluded |= (d.ex_list[e] == ai);
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
        }
    }
    // merge the warps' leftovers: warp 0 collects them and flushes
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
        if (nbuf > 0) flush_chunk(s_e[0], s_m[0], nbuf);
    }
}

// R7: close the rebuild -- capacity check, counters, flat chunk numbering.
__global__ void k_rebuild_finish(Dev d, int in_graph) {
    if (threadIdx.x != 0) return;
    if (in_graph) d.st[0].body_runs += 1;
    int run = 0;
    for (int r = 0; r < d.n_rep; ++r) {
        RepState* s = d.st + r;
        if (s->rebuild) {
            if (s->n_chunks > d.rep[r].chunk_cap) {
                s->status |= ST_CAPACITY;
                s->n_chunks = d.rep[r].chunk_cap;
            }
            s->rebuild = 0;
            s->lj_counter = 0;
            s->list_builds += 1;
        }
        d.chunk_prefix[r] = run;
        run += s->n_chunks;
    }
    d.chunk_prefix[d.n_rep] = run;
}

// R0: reset chunk counters of replicas about to rebuild; when the step runs as
// a CUDA graph, also set the IF-node condition that gates R1..R7.
__global__ void k_rebuild_begin(Dev d, cudaGraphConditionalHandle cond, int use_cond) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int r = threadIdx.x; r < d.n_rep; r += blockDim.x) {
        if (d.st[r].rebuild) {
            d.st[r].n_chunks = 0;
            any = 1;
        }
    }
    __syncthreads();
    if (use_cond && threadIdx.x == 0) cudaGraphSetConditional(cond, any ? 1u : 0u);
}

void launch_rebuild_flag(const Dev& d, cudaGraphConditionalHandle cond, bool use_cond, cudaStream_t st,
                         long long* nlaunch) {
    k_rebuild_begin<<<1, 256, 0, st>>>(d, cond, use_cond ? 1 : 0);
    *nlaunch += 1;
}

void launch_rebuild_body(const Dev& d, const int* bin_rep, bool in_graph, cudaStream_t st,
                         long long* nlaunch) {
    const int T = 256;
    k_bin_atoms<<<(d.n_atoms + T - 1) / T, T, 0, st>>>(d);
    k_bin_scan<<<d.n_rep, 1024, 0, st>>>(d);
    k_bin_scatter<<<(d.n_atoms + T - 1) / T, T, 0, st>>>(d);
    k_bin_sort<<<(d.n_bins + T - 1) / T, T, 0, st>>>(d, bin_rep);
    k_tiles<<<(d.n_tiles * 32 + T - 1) / T, T, 0, st>>>(d);
    k_build_pairs<<<d.n_tiles, 32 * BW, 0, st>>>(d);
    k_rebuild_finish<<<1, 32, 0, st>>>(d, in_graph ? 1 : 0);
    *nlaunch += 7;
}

}  // namespace dmd
