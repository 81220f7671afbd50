// noalloc.cu -- non-bonded force evaluation that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc -- hosts whose device
// memory is owned by another allocator or pool (a framework's caching
// allocator, a fixed arena on an embedded or real-time system, where a stray
// cudaMalloc would fragment or exceed the arena), and callers that must not
// pay allocation latency or risk an allocation failure in the middle of a
// run.  They pass their own device buffers for the inputs and outputs; every
// intermediate buffer of the evaluation -- the spatial sort, the tiles, the
// pair list and the fixed-point force accumulators -- lives in one file-scope
// static device array of scratch_bytes() (about 6 MB for the limits in
// dmdgpu.h) that each GPU holds from the moment the library is loaded on it
// until the process exits.
//
// The call is synchronous: it copies small host tables into the array from
// pageable memory and ends with cudaStreamSynchronize on the caller's stream
// to read the status word, so it cannot be issued while that stream is being
// captured into a CUDA graph.
//
// The work is the same as dmdgpu_component_compute for the Lennard-Jones and
// real-space Coulomb components: the same kernels, run over a batch of one
// system whose arrays are carved out of the static array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/dmdgpu.h"
#include "device.cuh"
#include "launch.h"

namespace dmd {

namespace {

constexpr int NA = DMDGPU_NOALLOC_MAX_ATOMS;        // atoms (and sorted slots)
constexpr int NT = NA / 32;                          // tiles
constexpr int NB = DMDGPU_NOALLOC_MAX_SORT_CELLS;    // sort cells
constexpr int NC = DMDGPU_NOALLOC_MAX_CHUNKS;        // pair-list chunks
constexpr int NTY = DMDGPU_NOALLOC_MAX_TYPES;
constexpr int NEX = DMDGPU_NOALLOC_MAX_EXCLUSIONS;   // exclusion pairs

constexpr size_t up256(size_t b) { return (b + 255) & ~static_cast<size_t>(255); }

// Byte layout of the scratch array (every piece 256-byte aligned).
struct Layout {
    size_t off = 0;
    size_t take(size_t bytes) {
        size_t o = off;
        off += up256(bytes);
        return o;
    }
};

constexpr size_t scratch_bytes() {
    size_t b = 0;
    b += up256(sizeof(Rep)) + up256(sizeof(RepState)) + up256(8 * sizeof(int));  // rep, state, prefix
    b += 3 * up256(NA * sizeof(int));              // imgx/y/z
    b += 3 * up256(NA * sizeof(double));           // xr/yr/zr
    b += 3 * up256(NA * sizeof(int));              // atom_rep, slot_of_atom, atom_bin
    b += up256(NA * sizeof(int));                  // validated copy of the caller's types
    b += up256(NA * sizeof(int)) * 3;              // atom_of_slot, type_s, sort_buf
    b += up256(NA * sizeof(double4));              // xq (float4 or double4)
    b += up256(NA * sizeof(float4));               // xl32 (build-frame copy, FP64 mode)
    b += 3 * up256(NA * sizeof(long long));        // fnx/fny/fnz
    b += 3 * up256(NT * sizeof(double)) + 3 * up256(NT * sizeof(float)) + up256(NT * sizeof(int));
    b += 5 * up256(NB * sizeof(int));              // bin count/start/fill, vox_rank, bin_rep
    b += up256((NA + 1) * sizeof(int)) + up256(2 * NEX * sizeof(int));  // exclusion CSR
    b += up256(NC * sizeof(int)) + 2 * up256(static_cast<size_t>(NC) * 32 * sizeof(uint32_t));
    b += up256(NTY * NTY * sizeof(double2)) + up256(NTY * NTY * sizeof(float4));
    return b;
}

}  // namespace

// The scratch array.  In host code `g_nb_scratch` is only a host-side stand-in
// for the symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_nb_scratch[scratch_bytes()];

namespace {

std::mutex g_mu;
void* g_addr[64] = {};  // device address of g_nb_scratch per device ordinal

// Per-device set-up: with the device current, resolve the array's address once.
// The address is cached per device ordinal, so calls must run in the device's
// primary context (the runtime API's default); a caller that switches to
// another context on the same device, or resets the device, would be handed
// the old context's address.
int scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) return DMDGPU_ERR_PARM;
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_nb_scratch) != cudaSuccess || !p) return DMDGPU_ERR_GPU;
        g_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[dev]);
    return DMDGPU_OK;
}

// Copy the caller's LJ types, flagging (and clamping) any outside [0, n_types),
// so no kernel indexes the LJ table out of range.
__global__ void k_noalloc_types(const int32_t* in, int* out, int n, int n_types, RepState* st) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    int t = in[a];
    if (t < 0 || t >= n_types) {
        set_status(st, ST_LIST);
        t = 0;
    }
    out[a] = t;
}

// Forces from slot order (fixed point) to the caller's atom order; energies out.
__global__ void k_noalloc_out(Dev d, double* fx, double* fy, double* fz, double* energies) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < d.n_atoms) {
        const int s = d.slot_of_atom[a];
        fx[a] = from_fix(d.fnx[s], FSCALE);
        fy[a] = from_fix(d.fny[s], FSCALE);
        fz[a] = from_fix(d.fnz[s], FSCALE);
    }
    if (a == 0 && energies) {
        energies[0] = from_fix(d.st[0].e_acc[E_LJ], ESCALE);
        energies[1] = from_fix(d.st[0].e_acc[E_CREAL], ESCALE);
    }
}

}  // namespace

}  // namespace dmd

extern "C" int dmdgpu_nonbonded_noalloc(const dmdgpu_nb_params* p, const double* d_x, const double* d_y,
                                        const double* d_z, const double* d_q, const int32_t* d_type,
                                        double* d_fx, double* d_fy, double* d_fz, double* d_energies,
                                        void* stream_ptr) {
    using namespace dmd;
    if (!p || !d_x || !d_y || !d_z || !d_q || !d_type || !d_fx || !d_fy || !d_fz) return DMDGPU_ERR_INVALID;
    const int n = p->n_atoms;
    // sizes beyond the static maxima are rejected
    if (n <= 0 || n > NA) return DMDGPU_ERR_PARM;
    if (p->n_types <= 0 || p->n_types > NTY || !p->lj_sigma || !p->lj_epsilon) return DMDGPU_ERR_PARM;
    if (p->n_excl < 0 || p->n_excl > NEX || (p->n_excl && (!p->excl_i || !p->excl_j))) return DMDGPU_ERR_PARM;
    if (!(p->box > 0) || !(p->lj_cutoff >= 0) || !(p->coul_cutoff >= 0)) return DMDGPU_ERR_PARM;
    const bool phys = p->profile == DMDGPU_PROFILE_PHYS;
    const bool fp64 = p->precision == DMDGPU_PRECISION_FP64;
    cudaStream_t st = static_cast<cudaStream_t>(stream_ptr);
    // an error left pending by the caller's earlier work is reported before any
    // work is issued and is not cleared, so it is not mistaken for this call's
    if (cudaPeekAtLastError() != cudaSuccess) return DMDGPU_ERR_GPU;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DMDGPU_ERR_GPU;
    unsigned char* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc) return rc;

    // sort grid as in the engine, shrunk until it fits the static sort cells
    const double L = p->box;
    const double rho = n / (L * L * L);
    int nvx = std::min(std::max(static_cast<int>(std::floor(L / (1.2 * std::cbrt(32.0 / rho)))), 1), 256);
    int nvz = std::min(std::max(static_cast<int>(std::floor(L / 0.1)), 1), 1024);
    while (static_cast<long long>(nvx) * nvx * nvz > NB) {
        if (nvz > nvx) nvz = std::max(1, nvz / 2);
        else nvx = std::max(1, nvx - 1);
    }
    const int nbins = nvx * nvx * nvz;
    const int ntiles = (n + 31) / 32;

    Layout lay;
    auto at = [&](size_t bytes) { return base + lay.take(bytes); };
    Dev d{};
    d.n_rep = 1;
    d.n_atoms = n;
    d.n_tiles = ntiles;
    d.n_slots = 32 * ntiles;
    d.n_bins = nbins;
    Rep* d_rep = reinterpret_cast<Rep*>(at(sizeof(Rep)));
    RepState* d_st = reinterpret_cast<RepState*>(at(sizeof(RepState)));
    d.chunk_prefix = reinterpret_cast<int*>(at(8 * sizeof(int)));
    d.build_prefix = d.chunk_prefix + 8;  // [3][2]: words 8..13 of the 256-byte block
    d.nb_work = d.chunk_prefix + 4;  // zeroed with the prefix below
    d.nb_work_mi = d.chunk_prefix + 3;  // words 0, 1: the chunk prefix of the one replica
    d.build_work = d.chunk_prefix + 5;
    d.grid_bar = reinterpret_cast<unsigned*>(d.chunk_prefix + 6);  // [2]: words 6, 7
    d.rep = d_rep;
    d.st = d_st;
    d.x = const_cast<double*>(d_x);
    d.y = const_cast<double*>(d_y);
    d.z = const_cast<double*>(d_z);
    d.q = d_q;
    int* types = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.type = types;
    d.imgx = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.imgy = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.imgz = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.xr = reinterpret_cast<double*>(at(NA * sizeof(double)));
    d.yr = reinterpret_cast<double*>(at(NA * sizeof(double)));
    d.zr = reinterpret_cast<double*>(at(NA * sizeof(double)));
    int* atom_rep = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.atom_rep = atom_rep;
    d.slot_of_atom = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.atom_bin = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.atom_of_slot = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.type_s = reinterpret_cast<int*>(at(NA * sizeof(int)));
    d.sort_buf = reinterpret_cast<int*>(at(NA * sizeof(int)));
    unsigned char* xq = at(NA * sizeof(double4));
    if (fp64) d.xq64 = reinterpret_cast<double4*>(xq);
    else d.xq32 = reinterpret_cast<float4*>(xq);
    unsigned char* xl = at(NA * sizeof(float4));
    d.xl32 = fp64 ? reinterpret_cast<float4*>(xl) : d.xq32;
    d.fnx = reinterpret_cast<long long*>(at(NA * sizeof(long long)));
    d.fny = reinterpret_cast<long long*>(at(NA * sizeof(long long)));
    d.fnz = reinterpret_cast<long long*>(at(NA * sizeof(long long)));
    d.tcx = reinterpret_cast<double*>(at(NT * sizeof(double)));
    d.tcy = reinterpret_cast<double*>(at(NT * sizeof(double)));
    d.tcz = reinterpret_cast<double*>(at(NT * sizeof(double)));
    d.thx = reinterpret_cast<float*>(at(NT * sizeof(float)));
    d.thy = reinterpret_cast<float*>(at(NT * sizeof(float)));
    d.thz = reinterpret_cast<float*>(at(NT * sizeof(float)));
    int* tile_rep = reinterpret_cast<int*>(at(NT * sizeof(int)));
    d.tile_rep = tile_rep;
    d.bin_count = reinterpret_cast<int*>(at(NB * sizeof(int)));
    d.bin_start = reinterpret_cast<int*>(at(NB * sizeof(int)));
    d.bin_fill = reinterpret_cast<int*>(at(NB * sizeof(int)));
    int* vox_rank = reinterpret_cast<int*>(at(NB * sizeof(int)));
    d.vox_rank = vox_rank;
    int* bin_rep = reinterpret_cast<int*>(at(NB * sizeof(int)));
    int* ex_start = reinterpret_cast<int*>(at((NA + 1) * sizeof(int)));
    int* ex_list = reinterpret_cast<int*>(at(2 * NEX * sizeof(int)));
    d.ex_start = ex_start;
    d.ex_list = ex_list;
    d.chunk_itile = reinterpret_cast<int*>(at(NC * sizeof(int)));
    d.chunk_j = reinterpret_cast<uint32_t*>(at(static_cast<size_t>(NC) * 32 * sizeof(uint32_t)));
    d.chunk_mask = reinterpret_cast<uint32_t*>(at(static_cast<size_t>(NC) * 32 * sizeof(uint32_t)));
    double2* lj64 = reinterpret_cast<double2*>(at(NTY * NTY * sizeof(double2)));
    float4* lj32 = reinterpret_cast<float4*>(at(NTY * NTY * sizeof(float4)));
    d.lj64 = lj64;
    d.lj32 = lj32;
    d.n_lj = p->n_types * p->n_types;

    if (lay.off > scratch_bytes()) return DMDGPU_ERR_GPU;  // layout and size disagree

    // host-side tables (no device allocation: all go into the static array)
    const int nt = p->n_types;
    std::vector<double2> h64(nt * nt);
    std::vector<float4> h32(nt * nt);
    for (int k = 0; k < nt * nt; ++k) {
        const double sg = p->lj_sigma[k], ep = p->lj_epsilon[k];
        const double sig2 = sg * sg, sig6 = sig2 * sig2 * sig2;
        h64[k] = make_double2(ep, sig6);
        h32[k] = lj_coeffs32(ep, sig6);
    }
    std::vector<int> hvr(nbins);
    for (int ix = 0; ix < nvx; ++ix)
        for (int iy = 0; iy < nvx; ++iy) {
            const int col = ix * nvx + ((ix & 1) ? nvx - 1 - iy : iy);
            for (int iz = 0; iz < nvz; ++iz)
                hvr[(ix * nvx + iy) * nvz + iz] = col * nvz + ((col & 1) ? nvz - 1 - iz : iz);
        }
    std::vector<int> hes(n + 1, 0), hel;
    if (phys && p->n_excl) {
        std::vector<std::vector<int>> lists(n);
        for (int k = 0; k < p->n_excl; ++k) {
            const int a = p->excl_i[k], b = p->excl_j[k];
            if (a < 0 || a >= n || b < 0 || b >= n) return DMDGPU_ERR_PARM;
            if (a != b) {
                lists[a].push_back(b);
                lists[b].push_back(a);
            }
        }
        for (int a = 0; a < n; ++a) {
            std::sort(lists[a].begin(), lists[a].end());
            lists[a].erase(std::unique(lists[a].begin(), lists[a].end()), lists[a].end());
            hes[a + 1] = hes[a] + static_cast<int>(lists[a].size());
            hel.insert(hel.end(), lists[a].begin(), lists[a].end());
        }
    }
    Rep R{};
    R.n_atoms = n;
    R.n_tiles = ntiles;
    R.nvx = nvx;
    R.nvz = nvz;
    R.chunk_cap = NC;
    R.n_types = nt;
    R.flags = F_LJ | (phys ? (F_PHYS | (p->coul_cutoff > 0 ? F_COUL_REAL : 0)) : 0);
    R.profile = phys ? 1 : 0;
    R.rc_lj = p->lj_cutoff;
    R.rc_c = p->coul_cutoff;
    R.rc_lj2 = p->lj_cutoff * p->lj_cutoff;
    R.rc_c2 = p->coul_cutoff * p->coul_cutoff;
    R.rc_list = phys ? std::max(p->lj_cutoff, (R.flags & F_COUL_REAL) ? p->coul_cutoff : 0.0) + p->skin
                     : p->lj_cutoff;
    R.rc_list2 = R.rc_list * R.rc_list;
    R.alpha = p->ewald_coeff;
    // a box narrower than twice the list cutoff: minimum image per evaluation
    d.mi_split = L * L < 4.0 * R.rc_list2 ? 1 : 0;
    d.any_coul = (R.flags & F_COUL_REAL) ? 1 : 0;
    RepState S{};
    S.L = L;
    S.invL = 1.0 / L;
    S.rebuild = 1;
    S.eval = 1;
    S.want_e = 1;
    S.active = 1;
    S.vscale = 1.0;
    S.pscale = 1.0;

    // clear what must start at zero (the array keeps the last call's contents)
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    bool good = ok(cudaMemcpyAsync(d_rep, &R, sizeof(R), cudaMemcpyHostToDevice, st)) &&
                ok(cudaMemcpyAsync(d_st, &S, sizeof(S), cudaMemcpyHostToDevice, st)) &&
                ok(cudaMemcpyAsync(lj64, h64.data(), sizeof(double2) * h64.size(), cudaMemcpyHostToDevice, st)) &&
                ok(cudaMemcpyAsync(lj32, h32.data(), sizeof(float4) * h32.size(), cudaMemcpyHostToDevice, st)) &&
                ok(cudaMemcpyAsync(vox_rank, hvr.data(), sizeof(int) * nbins, cudaMemcpyHostToDevice, st)) &&
                ok(cudaMemcpyAsync(ex_start, hes.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st)) &&
                (hel.empty() ||
                 ok(cudaMemcpyAsync(ex_list, hel.data(), sizeof(int) * hel.size(), cudaMemcpyHostToDevice, st))) &&
                ok(cudaMemsetAsync(atom_rep, 0, sizeof(int) * n, st)) &&
                ok(cudaMemsetAsync(tile_rep, 0, sizeof(int) * ntiles, st)) &&
                ok(cudaMemsetAsync(bin_rep, 0, sizeof(int) * nbins, st)) &&
                ok(cudaMemsetAsync(d.bin_count, 0, sizeof(int) * nbins, st)) &&
                ok(cudaMemsetAsync(d.bin_fill, 0, sizeof(int) * nbins, st)) &&
                ok(cudaMemsetAsync(d.fnx, 0, sizeof(long long) * 32 * ntiles, st)) &&
                ok(cudaMemsetAsync(d.fny, 0, sizeof(long long) * 32 * ntiles, st)) &&
                ok(cudaMemsetAsync(d.fnz, 0, sizeof(long long) * 32 * ntiles, st)) &&
                ok(cudaMemsetAsync(d.chunk_prefix, 0, 8 * sizeof(int), st));
    if (!good) return DMDGPU_ERR_GPU;
    long long nl = 0;
    // every launch is checked as soon as it is issued
    k_noalloc_types<<<(n + 255) / 256, 256, 0, st>>>(d_type, types, n, nt, d_st);
    if (cudaGetLastError() != cudaSuccess) return DMDGPU_ERR_GPU;
    int n_sm = 148;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DMDGPU_ERR_GPU;
    launch_rebuild(d, bin_rep, n_sm, st, &nl);
    if (cudaGetLastError() != cudaSuccess) return DMDGPU_ERR_GPU;
    launch_nonbonded(d, fp64, phys, n_sm, 2, NB_CHUNK32, st, &nl);
    if (cudaGetLastError() != cudaSuccess) return DMDGPU_ERR_GPU;
    k_noalloc_out<<<(n + 255) / 256, 256, 0, st>>>(d, d_fx, d_fy, d_fz, d_energies);
    if (cudaGetLastError() != cudaSuccess) return DMDGPU_ERR_GPU;
    // the call is synchronous: the status word says whether the list fitted
    RepState out{};
    if (!ok(cudaMemcpyAsync(&out, d_st, sizeof(out), cudaMemcpyDeviceToHost, st)) ||
        !ok(cudaStreamSynchronize(st)))
        return DMDGPU_ERR_GPU;
    // a list build whose bounded grid barrier gave up left a partial list
    if (out.status & ST_TIMEOUT) return DMDGPU_ERR_GPU;
    if (out.status & ST_LIST) return DMDGPU_ERR_PARM;  // an atom type outside [0, n_types)
    if (out.status & ST_CAPACITY) return DMDGPU_ERR_CAPACITY;
    if (out.status & ST_NAN) return DMDGPU_ERR_NAN;
    if (out.status & ST_RANGE) return DMDGPU_ERR_BOND_EXPLOSION;
    return DMDGPU_OK;
}
