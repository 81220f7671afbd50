// engine.cu -- host orchestration of the device path.
//
// A Batch owns one packed device table of replicas (a single system is a batch
// of one).  It replaces, on the host side, build_simulation / build_force_engine
// (src/sim/simulation_engine.cpp:147-386), SimulationEngine::step / run
// (:53-106) and checkpoint save / load (src/sim/checkpoint.cpp).  Steps are
// issued as CUDA graphs; run_n(k) is k graph replays with no host sync in
// between.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <mutex>
#include <stdexcept>
#include <tuple>

#include "engine.h"
#include "launch.h"

namespace dmd {

void SlabStore::prepare(size_t expect) {
    const size_t n1 = slabs.size();
    // keep a single slab that holds the table and is not more than 4x too big
    if (n1 == 1 && slabs[0].cap >= expect && slabs[0].cap <= 4 * expect + (size_t(64) << 20)) return;
    release();
    const size_t cap = ((expect + expect / 4 + (size_t(8) << 20)) + 0xFFFFF) & ~size_t(0xFFFFF);
    void* p = nullptr;
    if (cudaMalloc(&p, cap) != cudaSuccess) {
        cudaGetLastError();
        return;  // DeviceArena::alloc makes smaller slabs as it goes
    }
    slabs.push_back({static_cast<char*>(p), cap});
}

void SlabStore::release() {
    for (auto& sl : slabs) cudaFree(sl.p);
    slabs.clear();
}

template <typename T>
T* DeviceArena::alloc(size_t n) {
    if (n == 0) n = 1;
    const size_t want = (n * sizeof(T) + 255) & ~size_t(255);
    for (;;) {
        if (slab < store->slabs.size()) {
            SlabStore::Slab& sl = store->slabs[slab];
            if (off + want <= sl.cap) {
                char* p = sl.p + off;
                off += want;
                bytes += want;
                if (cudaMemsetAsync(p, 0, want, stream) != cudaSuccess) throw std::runtime_error("memset failed");
                return reinterpret_cast<T*>(p);
            }
            ++slab;
            off = 0;
            continue;
        }
        // the table outgrew the slabs: another one (the next rebuild makes one
        // slab of the whole size)
        void* p = nullptr;
        const size_t cap = std::max(want, size_t(64) << 20);
        if (cudaMalloc(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("cudaMalloc failed");
        }
        store->slabs.push_back({static_cast<char*>(p), cap});
    }
}

void* PinnedStaging::put(const void* src, size_t bytes) {
    const size_t want = (bytes + 255) & ~size_t(255);
    while (blk < blocks.size() && off + want > blocks[blk].second) {
        ++blk;
        off = 0;
    }
    if (blk == blocks.size()) {
        void* p = nullptr;
        const size_t cap = std::max(want, size_t(64) << 20);
        if (cudaMallocHost(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("pinned staging alloc failed");
        }
        blocks.emplace_back(static_cast<char*>(p), cap);
        off = 0;
    }
    char* dst = blocks[blk].first + off;
    std::memcpy(dst, src, bytes);
    off += want;
    return dst;
}

void PinnedStaging::trim(size_t keep) {
    size_t held = 0;
    size_t k = 0;
    for (; k < blocks.size() && held + blocks[k].second <= keep; ++k) held += blocks[k].second;
    for (size_t m = k; m < blocks.size(); ++m) cudaFreeHost(blocks[m].first);
    blocks.resize(k);
    reset();
}

namespace {

template <typename T>
std::vector<T> vec_of(const T* p, int n) {
    if (!p || n <= 0) return {};
    return std::vector<T>(p, p + n);
}

// Sort grid: square x-y columns 1.2x the edge of a 32-atom cube, z slabs of
// 0.1 nm; columns and slabs are visited in a snake order (see vox_rank), so
// 32 consecutive atoms are a compact tile.
void sort_grid(int n, double L, int& nvx, int& nvz) {
    const double rho = n / (L * L * L);
    const double a = 1.2 * std::cbrt(32.0 / std::max(rho, 1e-12));
    nvx = std::min(std::max(static_cast<int>(std::floor(L / a)), 1), 256);
    nvz = std::min(std::max(static_cast<int>(std::floor(L / 0.1)), 1), 1024);
}

}  // namespace

// ---------------------------------------------------------------------------
// Autotuner cache: the pair kernel's launch shape chosen for a kind of batch,
// shared by every batch of the process (the serving loop repacks often).
// Key: device, precision, whether a PME chain runs beside the pair kernel, and
// the batch's atom count in powers of four (a served stream's table changes
// size with every admission; nearby sizes share a shape).
namespace {
struct TuneKey {
    int device, fp64, pme, bucket, forced, dens;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, fp64, pme, bucket, forced, dens) <
               std::tie(o.device, o.fp64, o.pme, o.bucket, o.forced, o.dens);
    }
};
// A choice: the pair-kernel form (NbForm) and its blocks of 256 threads per SM.
struct TuneChoice {
    int form, bps;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune;
constexpr int kTuneSteps = 6;               // timed steps per candidate
// (4 blocks per SM: the LJ-only chunk kernel only, which a table without
// real-space Coulomb runs; for the others the launch takes 3)
constexpr TuneChoice kTuneCand[] = {{NB_CLUSTER8, 1}, {NB_CLUSTER8, 2}, {NB_CHUNK32, 2}, {NB_CHUNK32, 3},
                                    {NB_CHUNK32, 4}};

// forced: the caller's dmdgpu_options.nb_form (0: the default form)
// bucket: atom count in powers of four; dens: the table's atoms per nm^3 in
// powers of two (LJ fluids ~16-22, water ~100)
TuneKey tune_key(int device, bool fp64, bool pme, long long n_atoms, int forced, double density) {
    int b = 0;
    while ((1LL << (2 * b + 2)) <= n_atoms) ++b;
    const int dens = density > 0.0 ? static_cast<int>(std::floor(std::log2(density))) : 0;
    return TuneKey{device, fp64 ? 1 : 0, pme ? 1 : 0, b, forced, dens};
}

// DMDGPU_NB_* of the options -> NbForm, or -1 for the default form
int forced_form(int nb_form) {
    return nb_form == DMDGPU_NB_CHUNK32 ? NB_CHUNK32 : (nb_form == DMDGPU_NB_CLUSTER8 ? NB_CLUSTER8 : -1);
}
}  // namespace

// The 8-atom i-cluster form runs only when the options ask for it: measured on
// one B200, its pair kernel is faster alone (water 30k: 62.7 vs 66.8 us per
// launch in the step) but it holds every register of its SMs, so the SPME
// chain no longer runs beside it, and regrouping the list adds ~70 us to each
// rebuild; the 32-wide chunk form is the default.  The cluster rows and their
// bookkeeping are allocated (and built) only for that form.
bool Batch::uses_clusters() const { return !fp64_ && forced_form(opt_.nb_form) == NB_CLUSTER8; }

Batch::Batch(const dmdgpu_options& opt, long long budget) : opt_(opt), budget_(budget) {
    fp64_ = opt.precision == DMDGPU_PRECISION_FP64;
    phys_ = opt.profile == DMDGPU_PROFILE_PHYS;
    device_ = opt.device;
    if (cudaSetDevice(device_) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
    cudaDeviceGetAttribute(&n_sm_, cudaDevAttrMultiProcessorCount, device_);
    // The pair kernel is the longest branch of a force evaluation; the bonded
    // terms and the PME chain (a sequence of short kernels ending in the
    // gather, which the step waits for) run beside it.  The PME and bonded
    // streams have the higher priority, so that their blocks are dispatched
    // first wherever an SM has room (the main stream's own kernels are
    // ordered by dependencies); in the step graph every kernel node but the
    // pair kernel's gets the higher priority.
    configure_nonbonded_kernels();
    int prio_lo = 0, prio_hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&aux_stream_, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&bond_stream_, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join_b_, cudaEventDisableTiming) != cudaSuccess)
        throw std::runtime_error("cudaStreamCreate failed");
    prio_lo_ = prio_lo;
    prio_hi_ = prio_hi;
}

Batch::~Batch() {
    cudaSetDevice(device_);
    free_frames();
    free_device();
    for (auto& kv : plans_) {
        cufftDestroy(kv.second.first);
        cufftDestroy(kv.second.second);
    }
    plans_.clear();
    if (flush_buf_) cudaFree(flush_buf_);
    if (h_st_) cudaFreeHost(h_st_);
    if (h_tgt_) cudaFreeHost(h_tgt_);
    if (h_and_flag_) cudaFreeHost(h_and_flag_);
    if (h_and_v_) cudaFreeHost(h_and_v_);
    for (cudaEvent_t e : ev_pool_) cudaEventDestroy(e);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (ev_join_b_) cudaEventDestroy(ev_join_b_);
    if (bond_stream_) cudaStreamDestroy(bond_stream_);
    if (aux_stream_) cudaStreamDestroy(aux_stream_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Batch::free_device() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    // cuFFT plans depend only on the mesh size: they are kept across table
    // rebuilds (an admission or release rebuilds the table) and destroyed with
    // the batch
    // the pinned mirrors are kept (cudaFreeHost synchronises the device and
    // costs milliseconds); the next table grows them when it needs more
    arena_.reset();
    st_fresh_ = false;
    packed_ = false;
    used_bytes_ = 0;
}

int Batch::fail(int code, const std::string& msg) {
    err_ = msg;
    return code;
}

int Batch::check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return DMDGPU_OK;
    return fail(DMDGPU_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        int rc__ = check_cuda((call), #call);                      \
        if (rc__) return rc__;                                     \
    } while (0)

// ---------------------------------------------------------------------------
// Host replica construction (build_simulation, simulation_engine.cpp:248-386)
// ---------------------------------------------------------------------------
int Batch::build_host(HostRep& hr, unsigned mask) {
    HostSystem& s = hr.sys;
    Rep& R = hr.rep;
    R = Rep{};
    const int n = s.n;
    R.n_atoms = n;
    R.n_tiles = (n + 31) / 32;
    R.profile = phys_ ? 1 : 0;
    bool anyq = false;
    for (double v : s.q) anyq |= (v != 0.0);
    int flags = 0;
    if (s.use_lj && (mask & C_LJ)) flags |= F_LJ;
    if (phys_) flags |= F_PHYS;
    if (phys_ && anyq && (mask & C_CREAL)) flags |= F_COUL_REAL;
    if (s.coulomb_type == 1 && (mask & C_PME)) flags |= F_PME;
    if ((s.coulomb_type == 1 || !s.ei.empty()) && (mask & C_EXCL)) flags |= F_EXCL;
    R.flags = flags;
    R.rc_lj = s.lj_cutoff;
    R.rc_c = s.coul_cutoff;
    R.rc_lj2 = s.lj_cutoff * s.lj_cutoff;
    R.rc_c2 = s.coul_cutoff * s.coul_cutoff;
    if (phys_) {
        double rc = 0.0;
        if (s.use_lj) rc = std::max(rc, s.lj_cutoff);
        if (anyq) rc = std::max(rc, s.coul_cutoff);
        R.rc_list = rc + opt_.skin;
    } else {
        R.rc_list = s.lj_cutoff;  // the LennardJones list (no skin)
    }
    R.rc_list2 = R.rc_list * R.rc_list;
    R.half_skin2 = 0.25 * opt_.skin * opt_.skin;
    R.alpha = s.ewald;
    R.dt = s.dt;
    R.thermostat = s.thermostat;
    R.t_temp = s.t_temp;
    R.t_tau = s.t_tau;
    R.t_freq = s.t_freq;
    double dof = 3.0 * static_cast<double>(n) - 3.0;  // nose_hoover.cpp:9-13
    if (dof < 1.0) dof = 1.0;
    R.nh_Q = dof * KB * s.t_temp * s.t_tau * s.t_tau;
    R.barostat = s.barostat;
    R.b_pressure = s.b_pressure;
    R.b_tau = s.b_tau;
    R.b_compress = s.b_compress;
    R.piston_W = dof * KB * s.b_pressure * s.b_tau * s.b_tau;  // andersen_barostat.cpp:8-14
    R.cons_tol = s.ctol;
    R.n_types = std::max(s.n_types, 1);
    sort_grid(n, s.box, R.nvx, R.nvz);
    if (s.coulomb_type == 1) {
        s.pme_K = std::max(8, static_cast<int>(s.box / s.spacing + 0.5));  // simulation_engine.cpp:183-185
    }
    R.pme_K = (flags & F_PME) ? s.pme_K : 0;
    double sum_q2 = 0.0;  // CoulombPME::calc_self_energy (coulomb_pme.cpp:71-75)
    for (double v : s.q) sum_q2 += v * v;
    R.e_self = (flags & F_PME) ? -KE * s.ewald / std::sqrt(M_PI) * sum_q2 : 0.0;
    const uint64_t key = opt_.rng_seed;
    R.key0 = static_cast<uint32_t>(key);
    R.key1 = static_cast<uint32_t>(key >> 32);

    RepState& st = hr.init;
    st = RepState{};
    st.L = s.box;
    st.invL = 1.0 / s.box;
    st.vscale = 1.0;
    st.pscale = 1.0;
    st.rebuild = 1;
    st.lj_counter = 10;  // LennardJones::step_since_rebuild_ initial value (lennard_jones.cpp:10)
    st.L_build = s.box;
    return DMDGPU_OK;
}

long long Batch::footprint(const HostSystem& s) const {
    const long long n = s.n, tiles = (n + 31) / 32;
    const double rho = n / (s.box * s.box * s.box);
    long long per_atom = 8 * 6 + 8 * 2 + 4 * 2 + 8 * 3 + 4 + 8 * 3 + 4 * 4;
    long long per_slot = 4 + 32 + 4 + 8 * 3;
    long long chunks = tiles * 64;
    (void)rho;
    long long b = n * per_atom + tiles * 32 * per_slot + chunks * (4 + 32 * 8) + tiles * 64;
    // mixed precision: the list regrouped by 8-atom i-cluster (rows of 32 entry
    // words and 32 byte masks, up to 4 per chunk and 4 per tile) and its
    // per-tile bookkeeping
    if (uses_clusters()) b += (4 * chunks + 4 * tiles) * (32 * 4 + 32) + chunks * 8 + tiles * (12 + 4 * 8);
    b += static_cast<long long>(s.ci.size()) * (8 + 8 + 8);  // constraints and their groups
    if (s.coulomb_type == 1) {
        long long K = std::max(8, static_cast<int>(s.box / s.spacing + 0.5));
        b += K * K * (K + 2) * 8 + K * K * K * 8 + K * K * (K / 2 + 1) * 16 + 3 * K * K * K * 8;
    }
    return b + (2 << 20);
}

int Batch::add(const dmdgpu_system& in, long long n_steps, unsigned comp_mask, int* out_slot) {
    *out_slot = -1;
    if (in.n_atoms <= 0) return fail(DMDGPU_ERR_PARM, "n_atoms must be positive");
    if (!(in.box_size > 0)) return fail(DMDGPU_ERR_PARM, "box_size must be positive");
    if (!in.masses || !in.pos_x || !in.pos_y || !in.pos_z)
        return fail(DMDGPU_ERR_PARM, "masses and positions are required");
    if (in.constraint_type < 0 || in.constraint_type > 1)
        return fail(DMDGPU_ERR_PARM, "Unknown constraint type");
    if (in.constraint_type == 1 && in.thermostat_type == DMDGPU_THERMO_ANDERSEN)
        return fail(DMDGPU_ERR_PARM, "SHAKE/RATTLE constraints with the Andersen thermostat are not supported");
    if (in.thermostat_type < 0 || in.thermostat_type > 3)
        return fail(DMDGPU_ERR_PARM, "Unknown thermostat type");
    if (in.barostat_type < 0 || in.barostat_type > 2)
        return fail(DMDGPU_ERR_PARM, "Unknown barostat type");
    if (in.barostat_type == DMDGPU_BARO_ANDERSEN && phys_)
        return fail(DMDGPU_ERR_PARM, "the Andersen barostat runs in the ref profile only");
    if (in.n_atoms >= (1 << 26)) return fail(DMDGPU_ERR_PARM, "more than 2^26 atoms in one system");
    auto hr = std::make_unique<HostRep>();
    HostSystem& s = hr->sys;
    const int n = in.n_atoms;
    s.n = n;
    s.box = in.box_size;
    s.mass = vec_of(in.masses, n);
    s.q = in.charges ? vec_of(in.charges, n) : std::vector<double>(n, 0.0);
    s.x = vec_of(in.pos_x, n);
    s.y = vec_of(in.pos_y, n);
    s.z = vec_of(in.pos_z, n);
    s.vx = in.vel_x ? vec_of(in.vel_x, n) : std::vector<double>(n, 0.0);
    s.vy = in.vel_y ? vec_of(in.vel_y, n) : std::vector<double>(n, 0.0);
    s.vz = in.vel_z ? vec_of(in.vel_z, n) : std::vector<double>(n, 0.0);
    s.type = in.atom_types ? vec_of(in.atom_types, n) : std::vector<int>(n, 0);
    s.use_lj = in.use_lj;
    s.n_types = in.lj_n_types;
    s.lj_cutoff = in.lj_cutoff;
    if (s.use_lj) {
        if (s.n_types <= 0 || !in.lj_sigma || !in.lj_epsilon)
            return fail(DMDGPU_ERR_PARM, "LJ enabled without a type table");
        s.sigma = vec_of(in.lj_sigma, s.n_types * s.n_types);
        s.eps = vec_of(in.lj_epsilon, s.n_types * s.n_types);
        for (int t : s.type)
            if (t < 0 || t >= s.n_types) return fail(DMDGPU_ERR_PARM, "atom type outside the LJ table");
    }
    auto check_idx = [&](const int32_t* p, int m) {
        for (int k = 0; k < m; ++k)
            if (p[k] < 0 || p[k] >= n) return false;
        return true;
    };
    if (in.n_bonds > 0) {
        if (!check_idx(in.bond_i, in.n_bonds) || !check_idx(in.bond_j, in.n_bonds))
            return fail(DMDGPU_ERR_PARM, "bond index out of range");
        s.bi = vec_of(in.bond_i, in.n_bonds);
        s.bj = vec_of(in.bond_j, in.n_bonds);
        s.bk = vec_of(in.bond_k, in.n_bonds);
        s.br0 = vec_of(in.bond_r0, in.n_bonds);
    }
    if (in.n_angles > 0) {
        if (!check_idx(in.angle_i, in.n_angles) || !check_idx(in.angle_j, in.n_angles) ||
            !check_idx(in.angle_k, in.n_angles))
            return fail(DMDGPU_ERR_PARM, "angle index out of range");
        s.ai = vec_of(in.angle_i, in.n_angles);
        s.aj = vec_of(in.angle_j, in.n_angles);
        s.ak = vec_of(in.angle_k, in.n_angles);
        s.akt = vec_of(in.angle_k_theta, in.n_angles);
        s.at0 = vec_of(in.angle_theta0, in.n_angles);
    }
    if (in.n_dihedrals > 0) {
        const int m = in.n_dihedrals;
        if (!check_idx(in.dihedral_i, m) || !check_idx(in.dihedral_j, m) ||
            !check_idx(in.dihedral_k, m) || !check_idx(in.dihedral_l, m))
            return fail(DMDGPU_ERR_PARM, "dihedral index out of range");
        s.di = vec_of(in.dihedral_i, m);
        s.dj = vec_of(in.dihedral_j, m);
        s.dk = vec_of(in.dihedral_k, m);
        s.dl = vec_of(in.dihedral_l, m);
        s.dn = vec_of(in.dihedral_periodicity, m);
        s.dkp = vec_of(in.dihedral_k_phi, m);
        s.dp0 = vec_of(in.dihedral_phi0, m);
    }
    if (in.n_impropers > 0) {
        const int m = in.n_impropers;
        if (!in.improper_i || !in.improper_j || !in.improper_k || !in.improper_l ||
            !in.improper_k_phi || !in.improper_phi0)
            return fail(DMDGPU_ERR_PARM, "improper arrays missing");
        if (!check_idx(in.improper_i, m) || !check_idx(in.improper_j, m) ||
            !check_idx(in.improper_k, m) || !check_idx(in.improper_l, m))
            return fail(DMDGPU_ERR_PARM, "improper index out of range");
        s.ii = vec_of(in.improper_i, m);
        s.ij = vec_of(in.improper_j, m);
        s.ik = vec_of(in.improper_k, m);
        s.il = vec_of(in.improper_l, m);
        s.ikp = vec_of(in.improper_k_phi, m);
        s.ip0 = vec_of(in.improper_phi0, m);
    }
    if (in.n_excl > 0) {
        if (!check_idx(in.excl_i, in.n_excl) || !check_idx(in.excl_j, in.n_excl))
            return fail(DMDGPU_ERR_PARM, "exclusion index out of range");
        s.ei = vec_of(in.excl_i, in.n_excl);
        s.ej = vec_of(in.excl_j, in.n_excl);
    }
    if (in.constraint_type == 1 && in.n_constraints > 0) {
        const int m = in.n_constraints;
        if (!in.constraint_i || !in.constraint_j || !in.constraint_dist)
            return fail(DMDGPU_ERR_PARM, "constraint arrays missing");
        if (!check_idx(in.constraint_i, m) || !check_idx(in.constraint_j, m))
            return fail(DMDGPU_ERR_PARM, "constraint index out of range");
        s.ci = vec_of(in.constraint_i, m);
        s.cj = vec_of(in.constraint_j, m);
        s.cd = vec_of(in.constraint_dist, m);
        s.ctol = in.constraint_tolerance;
    }
    s.coulomb_type = in.coulomb_type;
    s.coul_cutoff = in.coulomb_cutoff;
    s.ewald = in.ewald_coeff;
    s.spacing = in.pme_grid_spacing;
    s.pme_order = in.pme_order;
    if (s.coulomb_type == 1 && !(s.spacing > 0)) return fail(DMDGPU_ERR_PARM, "pme_grid_spacing must be positive");
    s.dt = in.dt;
    s.n_steps = in.n_steps;
    s.thermostat = in.thermostat_type;
    s.t_temp = in.thermo_temperature;
    s.t_tau = in.thermo_tau;
    s.t_freq = in.thermo_frequency;
    s.barostat = in.barostat_type;
    s.b_pressure = in.baro_pressure;
    s.b_tau = in.baro_tau;
    s.b_compress = in.baro_compressibility;
    s.checkpoint_interval = in.checkpoint_interval;
    if (in.checkpoint_path) s.checkpoint_path = in.checkpoint_path;
    // Maxwell-Boltzmann velocities exactly as build_simulation (simulation_engine.cpp:339-383)
    if (in.gen_vel && n > 0) {
        std::mt19937 rng(in.seed);
        std::normal_distribution<double> normal(0.0, 1.0);
        double kBT = KB * in.init_temperature;
        for (int i = 0; i < n; ++i) {
            double sigma = std::sqrt(kBT / s.mass[i]);
            s.vx[i] = normal(rng) * sigma;
            s.vy[i] = normal(rng) * sigma;
            s.vz[i] = normal(rng) * sigma;
        }
        double cx = 0, cy = 0, cz = 0, tm = 0;
        for (int i = 0; i < n; ++i) {
            cx += s.mass[i] * s.vx[i];
            cy += s.mass[i] * s.vy[i];
            cz += s.mass[i] * s.vz[i];
            tm += s.mass[i];
        }
        cx /= tm;
        cy /= tm;
        cz /= tm;
        for (int i = 0; i < n; ++i) {
            s.vx[i] -= cx;
            s.vy[i] -= cy;
            s.vz[i] -= cz;
        }
        if (in.init_temperature > 0) {
            double ek = 0;
            for (int i = 0; i < n; ++i)
                ek += 0.5 * s.mass[i] * (s.vx[i] * s.vx[i] + s.vy[i] * s.vy[i] + s.vz[i] * s.vz[i]);
            double ta = (n < 2) ? 0.0 : 2.0 * ek / ((3.0 * static_cast<double>(n) - 3.0) * KB);
            double lam = std::sqrt(in.init_temperature / ta);
            for (int i = 0; i < n; ++i) {
                s.vx[i] *= lam;
                s.vy[i] *= lam;
                s.vz[i] *= lam;
            }
        }
    }
    int rc = build_host(*hr, comp_mask);
    if (rc) return rc;
    hr->target = n_steps;
    if (budget_ > 0) {
        // admitted systems count from admission on, packed or not yet
        long long committed = 0;
        for (const auto& r : reps_)
            if (r) committed += footprint(r->sys);
        if (std::max(used_bytes_, committed) + footprint(s) > budget_)
            return fail(DMDGPU_ERR_BUDGET, "HBM budget exceeded");
    }
    // reuse a free slot id
    int slot = -1;
    for (size_t k = 0; k < reps_.size(); ++k)
        if (!reps_[k]) { slot = static_cast<int>(k); break; }
    if (slot < 0) {
        slot = static_cast<int>(reps_.size());
        reps_.emplace_back();
    }
    // the cuFFT plans of a new mesh size are made here, at admission, not in
    // the table rebuild of the next step (a plan takes tens of ms to make)
    if (hr->rep.flags & F_PME) {
        CK(cudaSetDevice(device_));
        int rc = ensure_plans(hr->rep.pme_K);
        if (rc) return rc;
    }
    reps_[slot] = std::move(hr);
    packed_ = false;
    *out_slot = slot;
    return DMDGPU_OK;
}

int Batch::ensure_plans(int K) {
    if (plans_.count(K)) return DMDGPU_OK;
    cufftHandle f, b;
    if (cufftPlan3d(&f, K, K, K, fp64_ ? CUFFT_D2Z : CUFFT_R2C) != CUFFT_SUCCESS)
        return fail(DMDGPU_ERR_GPU, "cufftPlan3d failed");
    if (cufftPlan3d(&b, K, K, K, fp64_ ? CUFFT_Z2D : CUFFT_C2R) != CUFFT_SUCCESS) {
        cufftDestroy(f);
        return fail(DMDGPU_ERR_GPU, "cufftPlan3d failed");
    }
    cufftSetStream(f, aux_stream_);
    cufftSetStream(b, aux_stream_);
    plans_[K] = {f, b};
    return DMDGPU_OK;
}

int Batch::release(int slot) {
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    reps_[slot].reset();
    packed_ = false;
    return DMDGPU_OK;
}

// What a running replica goes through when another slot is admitted or released:
// the table is rebuilt with its state carried over bit for bit, its pair list is
// rebuilt in the frame of its last build and its forces are evaluated again at
// the same positions; the trajectory continues unchanged.
int Batch::repack() {
    CK(cudaSetDevice(device_));
    packed_ = false;
    return pack();
}

int Batch::replica_index(int slot) const {
    for (size_t k = 0; k < order_.size(); ++k)
        if (order_[k] == slot) return static_cast<int>(k);
    return -1;
}

// ---------------------------------------------------------------------------
// Packing: host replicas -> one device table
// ---------------------------------------------------------------------------
int Batch::pack() {
    CK(cudaSetDevice(device_));
    // carry the device state of replicas that were already packed
    if (arena_) {
        CK(cudaStreamSynchronize(stream_));
        launch_finalize_velocities(dev_, stream_, &launches_);
        CK(cudaMemcpyAsync(h_st_, d_st_, sizeof(RepState) * order_.size(), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (size_t k = 0; k < order_.size(); ++k) {
            // a released slot may already hold a newly admitted system: only
            // replicas that were packed carry device state over
            if (!reps_[order_[k]] || !reps_[order_[k]]->on_device) continue;
            HostRep& o = *reps_[order_[k]];
            HostSystem& s = o.sys;
            const int a0 = o.rep.atom_begin, n = s.n;
            CK(cudaMemcpy(s.x.data(), dev_.x + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.y.data(), dev_.y + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.z.data(), dev_.z + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.vx.data(), dev_.vx + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.vy.data(), dev_.vy + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.vz.data(), dev_.vz + a0, n * 8, cudaMemcpyDeviceToHost));
            // the positions of the last list build: the list is rebuilt in that
            // frame (rebuild_in_frame), so the carried replica continues exactly
            // as it would have in the old table
            s.xr.resize(n);
            s.yr.resize(n);
            s.zr.resize(n);
            CK(cudaMemcpy(s.xr.data(), dev_.xr + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.yr.data(), dev_.yr + a0, n * 8, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(s.zr.data(), dev_.zr + a0, n * 8, cudaMemcpyDeviceToHost));
            RepState st = h_st_[k];
            st.have_forces = 0;      // forces are evaluated again at the same positions
            st.n_chunks = 0;
            st.n_cl = 0;
            st.green_L = 0.0;        // the new arena holds no PME influence function yet
            o.init = st;
        }
    }
    free_device();
    order_.clear();
    for (size_t k = 0; k < reps_.size(); ++k)
        if (reps_[k]) order_.push_back(static_cast<int>(k));
    const int R = static_cast<int>(order_.size());
    if (R == 0) {
        packed_ = true;
        return DMDGPU_OK;
    }
    // offsets
    long long n_atoms = 0, n_tiles = 0, n_bins = 0, n_chunks = 0, n_lj = 0, n_bond = 0, n_ang = 0,
              n_dih = 0, n_imp = 0, n_excl = 0, mesh_fix = 0, mesh_real = 0, mesh_cplx = 0, n_bsp = 0,
              n_cl = 0;
    int pme_blocks = 0, conv_blocks = 0;
    any_pme_ = any_baro_ = any_narrow_ = any_ref_lj_ = any_andersen_ref_ = any_andersen_phys_ = false;
    for (int k = 0; k < R; ++k) {
        HostRep& h = *reps_[order_[k]];
        HostSystem& s = h.sys;
        Rep& P = h.rep;
        P.atom_begin = static_cast<int>(n_atoms);
        P.tile_begin = static_cast<int>(n_tiles);
        P.bin_begin = static_cast<int>(n_bins);
        P.lj_off = static_cast<int>(n_lj);
        // chunk capacity: j atoms within rc_list of a tile's box (half), 1.5x margin
        {
            const double rho = s.n / (s.box * s.box * s.box);
            const double at = std::cbrt(32.0 / rho);
            const double reach = P.rc_list + 1.2 * at;
            double nj = 0.5 * rho * 4.18879 * reach * reach * reach;
            nj = std::min(nj, static_cast<double>(s.n));
            long long per_tile = static_cast<long long>(nj / 32.0) + 3;
            P.chunk_cap = static_cast<int>(std::max<long long>(1, P.n_tiles * per_tile * 3 / 2 + 8));
            if (P.rc_list <= 0) P.chunk_cap = 1;
        }
        P.chunk_begin = static_cast<int>(n_chunks);
        // i-cluster rows: each of a tile's chunks adds at most 32 entries to each
        // of its four clusters, so 4 rows per chunk plus one partial row per
        // cluster always suffice
        P.cl_cap = uses_clusters() ? static_cast<int>(std::min<long long>(4LL * P.chunk_cap + 4LL * P.n_tiles, INT32_MAX / 64)) : 0;
        P.cl_begin = static_cast<int>(n_cl);
        n_cl += P.cl_cap;
        n_atoms += s.n;
        n_tiles += P.n_tiles;
        n_bins += static_cast<long long>(P.nvx) * P.nvx * P.nvz;
        n_chunks += P.chunk_cap;
        n_lj += static_cast<long long>(P.n_types) * P.n_types;
        n_bond += s.bi.size();
        n_ang += s.ai.size();
        n_dih += s.di.size();
        n_imp += s.ii.size();
        n_excl += s.ei.size();
        if (P.flags & F_PME) {
            const int K = P.pme_K;
            // every replica's meshes start on a 64-element boundary: cuFFT reads a
            // real array that is not 8-byte aligned (odd K^3 offsets) incorrectly
            auto align64 = [](long long v) { return (v + 63) & ~63LL; };
            P.mesh_fix_off = mesh_fix;
            P.mesh_fix_n = phys_ ? static_cast<long long>(K) * K * K
                                 : static_cast<long long>(K) * K * 2 * (K / 2 + 1);
            mesh_fix = align64(mesh_fix + P.mesh_fix_n);
            P.mesh_real_off = mesh_real;
            mesh_real = align64(mesh_real + static_cast<long long>(K) * K * K + 64);
            P.mesh_cplx_off = mesh_cplx;
            mesh_cplx = align64(mesh_cplx + static_cast<long long>(K) * K * (K / 2 + 1) + 64);
            P.bsp_off = static_cast<int>(n_bsp);
            n_bsp += K;
            P.pme_block_begin = pme_blocks;
            P.pme_blocks = static_cast<int>((static_cast<long long>(K) * K * (K / 2 + 1) + 255) / 256);
            pme_blocks += P.pme_blocks;
            P.conv_block_begin = conv_blocks;
            P.conv_blocks = static_cast<int>((P.mesh_fix_n + 1023) / 1024);
            conv_blocks += P.conv_blocks;
            any_pme_ = true;
        }
        if (s.barostat) any_baro_ = true;
        // a box narrower than twice the list cutoff (or one a barostat may
        // shrink): the pair kernels take the minimum image per evaluation
        if (s.barostat || s.box * s.box < 4.0 * P.rc_list2) any_narrow_ = true;
        if (!phys_ && (P.flags & F_LJ)) any_ref_lj_ = true;
        if (s.thermostat == 3 && !phys_) any_andersen_ref_ = true;
        if (s.thermostat == 3 && phys_) any_andersen_phys_ = true;
    }
    n_pme_blocks_ = pme_blocks;
    n_conv_blocks_ = conv_blocks;
    // one slab for the table, sized from the footprint estimates scaled by
    // what the last table actually took of its estimate
    size_t fp_sum = 0;
    for (int k = 0; k < R; ++k) fp_sum += static_cast<size_t>(footprint(reps_[order_[k]]->sys));
    slabs_.prepare(static_cast<size_t>(static_cast<double>(fp_sum) * std::max(1.0, fp_ratio_)));
    staging_.reset();
    try {
        arena_ = std::make_unique<DeviceArena>();
        arena_->store = &slabs_;
        arena_->stream = stream_;
        DeviceArena& A = *arena_;
        Dev& d = dev_;
        d = Dev{};
        d.n_rep = R;
        d.n_atoms = static_cast<int>(n_atoms);
        d.n_tiles = static_cast<int>(n_tiles);
        d.n_slots = static_cast<int>(n_tiles * 32);
        d.n_bins = static_cast<int>(n_bins);
        d_rep_ = A.alloc<Rep>(R);
        d_st_ = A.alloc<RepState>(R);
        d.rep = d_rep_;
        d.st = d_st_;
        d.x = A.alloc<double>(n_atoms);
        d.y = A.alloc<double>(n_atoms);
        d.z = A.alloc<double>(n_atoms);
        d.vx = A.alloc<double>(n_atoms);
        d.vy = A.alloc<double>(n_atoms);
        d.vz = A.alloc<double>(n_atoms);
        double* mass = A.alloc<double>(n_atoms);
        double* q = A.alloc<double>(n_atoms);
        int* type = A.alloc<int>(n_atoms);
        int* atom_rep = A.alloc<int>(n_atoms);
        d.mass = mass;
        d.q = q;
        d.type = type;
        d.atom_rep = atom_rep;
        d.fbx = A.alloc<long long>(n_atoms);
        d.fby = A.alloc<long long>(n_atoms);
        d.fbz = A.alloc<long long>(n_atoms);
        d.slot_of_atom = A.alloc<int>(n_atoms);
        d.xr = A.alloc<double>(n_atoms);
        d.yr = A.alloc<double>(n_atoms);
        d.zr = A.alloc<double>(n_atoms);
        d.imgx = A.alloc<int>(n_atoms);
        d.imgy = A.alloc<int>(n_atoms);
        d.imgz = A.alloc<int>(n_atoms);
        d.atom_bin = A.alloc<int>(n_atoms);
        d.atom_of_slot = A.alloc<int>(d.n_slots);
        if (fp64_) d.xq64 = A.alloc<double4>(d.n_slots);
        else d.xq32 = A.alloc<float4>(d.n_slots);
        d.xl32 = fp64_ ? A.alloc<float4>(d.n_slots) : d.xq32;
        d.type_s = A.alloc<int>(d.n_slots);
        d.fnx = A.alloc<long long>(d.n_slots);
        d.fny = A.alloc<long long>(d.n_slots);
        d.fnz = A.alloc<long long>(d.n_slots);
        d.tcx = A.alloc<double>(n_tiles);
        d.tcy = A.alloc<double>(n_tiles);
        d.tcz = A.alloc<double>(n_tiles);
        d.thx = A.alloc<float>(n_tiles);
        d.thy = A.alloc<float>(n_tiles);
        d.thz = A.alloc<float>(n_tiles);
        int* tile_rep = A.alloc<int>(n_tiles);
        d.tile_rep = tile_rep;
        d.tile_ke = A.alloc<double>(n_tiles);
        d.tile_vir = A.alloc<double>(n_tiles);
        d.bin_count = A.alloc<int>(n_bins);
        d.bin_start = A.alloc<int>(n_bins);
        d.bin_fill = A.alloc<int>(n_bins);
        int* vox_rank = A.alloc<int>(n_bins);
        d.vox_rank = vox_rank;
        d_bin_rep_ = A.alloc<int>(n_bins);
        d.sort_buf = A.alloc<int>(d.n_slots);
        d.chunk_itile = A.alloc<int>(n_chunks);
        d.chunk_j = A.alloc<uint32_t>(n_chunks * 32);
        d.chunk_mask = A.alloc<uint32_t>(n_chunks * 32);
        d.chunk_prefix = A.alloc<int>(R + 4);
        d.nb_work = d.chunk_prefix + R + 1;
        d.build_work = d.chunk_prefix + R + 2;
        d.nb_work_mi = d.chunk_prefix + R + 3;
        d.mi_split = any_narrow_ ? 1 : 0;
        {
            double vol = 0.0;
            for (int k = 0; k < R; ++k) {
                const double L = reps_[order_[k]]->sys.box;
                vol += L * L * L;
            }
            density_ = vol > 0.0 ? static_cast<double>(n_atoms) / vol : 0.0;
        }
        d.any_coul = 0;
        for (int k = 0; k < R; ++k)
            if (reps_[order_[k]]->rep.flags & F_COUL_REAL) d.any_coul = 1;
        d.grid_bar = A.alloc<unsigned>(2);
        d.build_prefix = A.alloc<int>(4 * (R + 1));
        if (uses_clusters()) {
            d.tile_nch = A.alloc<int>(n_tiles);
            d.tile_c0 = A.alloc<int>(n_tiles);
            d.tile_fill = A.alloc<int>(n_tiles);
            d.chunk_order = A.alloc<int>(n_chunks);
            d.chunk_sorted = A.alloc<int>(n_chunks);
            d.cl_j = A.alloc<uint32_t>(n_cl * 32);
            d.cl_m = A.alloc<uint8_t>(n_cl * 32);
            d.cl_job = A.alloc<int2>(4 * n_tiles);
        }
        // host-side staging
        std::vector<double> hm(n_atoms), hq(n_atoms), hx(n_atoms), hy(n_atoms), hz(n_atoms), hvx(n_atoms),
            hvy(n_atoms), hvz(n_atoms), hxr(n_atoms), hyr(n_atoms), hzr(n_atoms);
        std::vector<int> ht(n_atoms), har(n_atoms), htr(n_tiles), hvr(n_bins), hbr(n_bins);
        std::vector<double2> lj64(n_lj);
        std::vector<float4> lj32(n_lj);
        std::vector<int2> bij;
        std::vector<double2> bkr;
        std::vector<int4> aijk;
        std::vector<double2> akt;
        std::vector<int4> dijkl;
        std::vector<int> dn;
        std::vector<double2> dkp;
        std::vector<int4> iijkl;
        std::vector<double2> ikp;
        std::vector<int2> ex;
        std::vector<int2> cij;              // constraints grouped by connected atom set
        std::vector<double> cdist;
        std::vector<int> cgb(1, 0), cgr;    // group begin offsets, group replica
        std::vector<int> cgab(1, 0), cga;   // each group's distinct atoms
        std::vector<double> bsp(std::max<long long>(n_bsp, 1));
        std::vector<int> pbr(std::max(pme_blocks, 1));
        std::vector<int> cbr(std::max(conv_blocks, 1));
        std::vector<Rep> hrep(R);
        for (int k = 0; k < R; ++k) {
            HostRep& h = *reps_[order_[k]];
            HostSystem& s = h.sys;
            Rep& P = h.rep;
            const int a0 = P.atom_begin;
            for (int i = 0; i < s.n; ++i) {
                hm[a0 + i] = s.mass[i];
                hq[a0 + i] = s.q[i];
                hx[a0 + i] = s.x[i];
                hy[a0 + i] = s.y[i];
                hz[a0 + i] = s.z[i];
                const bool framed = !s.xr.empty();
                hxr[a0 + i] = framed ? s.xr[i] : s.x[i];
                hyr[a0 + i] = framed ? s.yr[i] : s.y[i];
                hzr[a0 + i] = framed ? s.zr[i] : s.z[i];
                hvx[a0 + i] = s.vx[i];
                hvy[a0 + i] = s.vy[i];
                hvz[a0 + i] = s.vz[i];
                ht[a0 + i] = s.type[i];
                har[a0 + i] = k;
            }
            for (int t = 0; t < P.n_tiles; ++t) htr[P.tile_begin + t] = k;
            // snake rank of the replica's sort cells: columns in boustrophedon order
            // over (x, y), z reversed in every other column, so consecutive cells touch
            const int nvx = P.nvx, nvz = P.nvz;
            const int nb = nvx * nvx * nvz;
            for (int ix = 0; ix < nvx; ++ix)
                for (int iy = 0; iy < nvx; ++iy) {
                    const int col = ix * nvx + ((ix & 1) ? nvx - 1 - iy : iy);
                    for (int iz = 0; iz < nvz; ++iz) {
                        const int v = (ix * nvx + iy) * nvz + iz;
                        hvr[P.bin_begin + v] = col * nvz + ((col & 1) ? nvz - 1 - iz : iz);
                    }
                }
            for (int b = 0; b < nb; ++b) hbr[P.bin_begin + b] = k;
            // LJ tables: (eps, sig^6) with sig2*sig2*sig2 as in lennard_jones.cpp:75-77
            for (int ti = 0; ti < P.n_types; ++ti)
                for (int tj = 0; tj < P.n_types; ++tj) {
                    double sg = 1.0, ep = 0.0;
                    if (s.use_lj && !s.sigma.empty()) {
                        sg = s.sigma[ti * s.n_types + tj];
                        ep = s.eps[ti * s.n_types + tj];
                    }
                    const double sig2 = sg * sg;
                    const double sig6 = sig2 * sig2 * sig2;
                    lj64[P.lj_off + ti * P.n_types + tj] = make_double2(ep, sig6);
                    lj32[P.lj_off + ti * P.n_types + tj] = lj_coeffs32(ep, sig6);
                }
            for (size_t t = 0; t < s.bi.size(); ++t) {
                bij.push_back(make_int2(a0 + s.bi[t], a0 + s.bj[t]));
                bkr.push_back(make_double2(s.bk[t], s.br0[t]));
            }
            for (size_t t = 0; t < s.ai.size(); ++t) {
                aijk.push_back(make_int4(a0 + s.ai[t], a0 + s.aj[t], a0 + s.ak[t], 0));
                akt.push_back(make_double2(s.akt[t], s.at0[t]));
            }
            for (size_t t = 0; t < s.di.size(); ++t) {
                dijkl.push_back(make_int4(a0 + s.di[t], a0 + s.dj[t], a0 + s.dk[t], a0 + s.dl[t]));
                dn.push_back(s.dn[t]);
                dkp.push_back(make_double2(s.dkp[t], s.dp0[t]));
            }
            for (size_t t = 0; t < s.ii.size(); ++t) {
                iijkl.push_back(make_int4(a0 + s.ii[t], a0 + s.ij[t], a0 + s.ik[t], a0 + s.il[t]));
                ikp.push_back(make_double2(s.ikp[t], s.ip0[t]));
            }
            if (!s.ci.empty()) {
                // connected atom sets of the constraint graph (union-find); groups in
                // order of their first constraint, each group's constraints in the
                // order given: sweeping every group on its own reproduces the
                // reference's Gauss-Seidel sweeps over all constraints, which never
                // couple two groups
                std::vector<int> root(s.n);
                for (int i = 0; i < s.n; ++i) root[i] = i;
                auto find = [&](int v) {
                    while (root[v] != v) v = root[v] = root[root[v]];
                    return v;
                };
                for (size_t t = 0; t < s.ci.size(); ++t) {
                    const int ra = find(s.ci[t]), rb = find(s.cj[t]);
                    if (ra != rb) root[std::max(ra, rb)] = std::min(ra, rb);
                }
                std::vector<int> gid(s.n, -1);
                std::vector<std::vector<int>> members;
                for (size_t t = 0; t < s.ci.size(); ++t) {
                    const int g0 = find(s.ci[t]);
                    if (gid[g0] < 0) {
                        gid[g0] = static_cast<int>(members.size());
                        members.emplace_back();
                    }
                    members[gid[g0]].push_back(static_cast<int>(t));
                }
                std::vector<char> seen(s.n, 0);
                for (const auto& mem : members) {
                    for (int t : mem) {
                        cij.push_back(make_int2(a0 + s.ci[t], a0 + s.cj[t]));
                        cdist.push_back(s.cd[t]);
                        for (int a : {s.ci[t], s.cj[t]})
                            if (!seen[a]) {
                                seen[a] = 1;
                                cga.push_back(a0 + a);
                            }
                    }
                    cgb.push_back(static_cast<int>(cij.size()));
                    cgab.push_back(static_cast<int>(cga.size()));
                    cgr.push_back(k);
                }
            }
            for (size_t t = 0; t < s.ei.size(); ++t) ex.push_back(make_int2(a0 + s.ei[t], a0 + s.ej[t]));
            if (P.flags & F_PME) {
                const int K = P.pme_K;
                for (int kk = 0; kk < K; ++kk) {
                    const int m = (kk <= K / 2) ? kk : kk - K;
                    double b;
                    if (phys_) {
                        const double c = 2.0 / 3.0 + std::cos(2.0 * PI * m / K) / 3.0;
                        b = 1.0 / (c * c);
                    } else {  // b_factor (coulomb_pme.cpp:159-163)
                        if (m == 0) b = 1.0;
                        else {
                            const double t = M_PI * std::abs(m) / K;
                            b = std::pow(std::sin(t) / t, 2 * s.pme_order);
                        }
                    }
                    bsp[P.bsp_off + kk] = b;
                }
                for (int b = 0; b < P.pme_blocks; ++b) pbr[P.pme_block_begin + b] = k;
                for (int b = 0; b < P.conv_blocks; ++b) cbr[P.conv_block_begin + b] = k;
            }
            hrep[k] = P;
        }
        // exclusion CSR: each atom's excluded partners, ascending, without
        // repeats (counted, filled, then each short row sorted in place)
        std::vector<int> ex_start(n_atoms + 1, 0), ex_list;
        {
            std::vector<int> cnt(n_atoms + 1, 0);
            for (const int2& e : ex)
                if (e.x != e.y) {
                    ++cnt[e.x + 1];
                    ++cnt[e.y + 1];
                }
            for (long long a = 0; a < n_atoms; ++a) cnt[a + 1] += cnt[a];
            std::vector<int> raw(cnt[n_atoms]);
            std::vector<int> fill(cnt.begin(), cnt.end() - 1);
            for (const int2& e : ex)
                if (e.x != e.y) {
                    raw[fill[e.x]++] = e.y;
                    raw[fill[e.y]++] = e.x;
                }
            ex_list.reserve(raw.size());
            for (long long a = 0; a < n_atoms; ++a) {
                auto b = raw.begin() + cnt[a], e = raw.begin() + cnt[a + 1];
                std::sort(b, e);
                e = std::unique(b, e);
                ex_list.insert(ex_list.end(), b, e);
                ex_start[a + 1] = static_cast<int>(ex_list.size());
            }
        }
        // staged in pinned memory, copied in order on the main stream after the
        // zero fills of the arena
        auto up = [&](void* dst, const void* src, size_t bytes) {
            if (!bytes) return;
            const void* h = staging_.put(src, bytes);
            if (cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, stream_) != cudaSuccess)
                throw std::runtime_error("upload failed");
        };
        up(d.x, hx.data(), 8 * n_atoms);
        up(d.y, hy.data(), 8 * n_atoms);
        up(d.z, hz.data(), 8 * n_atoms);
        up(d.vx, hvx.data(), 8 * n_atoms);
        up(d.vy, hvy.data(), 8 * n_atoms);
        up(d.vz, hvz.data(), 8 * n_atoms);
        up(d.xr, hxr.data(), 8 * n_atoms);
        up(d.yr, hyr.data(), 8 * n_atoms);
        up(d.zr, hzr.data(), 8 * n_atoms);
        up(mass, hm.data(), 8 * n_atoms);
        up(q, hq.data(), 8 * n_atoms);
        up(type, ht.data(), 4 * n_atoms);
        up(atom_rep, har.data(), 4 * n_atoms);
        up(tile_rep, htr.data(), 4 * n_tiles);
        up(vox_rank, hvr.data(), 4 * n_bins);
        up(d_bin_rep_, hbr.data(), 4 * n_bins);
        double2* dlj64 = A.alloc<double2>(n_lj);
        float4* dlj32 = A.alloc<float4>(n_lj);
        up(dlj64, lj64.data(), sizeof(double2) * n_lj);
        up(dlj32, lj32.data(), sizeof(float4) * n_lj);
        d.lj64 = dlj64;
        d.lj32 = dlj32;
        d.n_lj = static_cast<int>(n_lj);
        d.n_bonds = static_cast<int>(bij.size());
        d.n_angles = static_cast<int>(aijk.size());
        d.n_dih = static_cast<int>(dijkl.size());
        d.n_imp = static_cast<int>(iijkl.size());
        d.n_excl = static_cast<int>(ex.size());
        int2* dbij = A.alloc<int2>(bij.size());
        double2* dbkr = A.alloc<double2>(bkr.size());
        int4* daijk = A.alloc<int4>(aijk.size());
        double2* dakt = A.alloc<double2>(akt.size());
        int4* ddijkl = A.alloc<int4>(dijkl.size());
        int* ddn = A.alloc<int>(dn.size());
        double2* ddkp = A.alloc<double2>(dkp.size());
        int4* diijkl = A.alloc<int4>(iijkl.size());
        double2* dikp = A.alloc<double2>(ikp.size());
        int2* dex = A.alloc<int2>(ex.size());
        int* dexs = A.alloc<int>(ex_start.size());
        int* dexl = A.alloc<int>(ex_list.size());
        up(dbij, bij.data(), sizeof(int2) * bij.size());
        up(dbkr, bkr.data(), sizeof(double2) * bkr.size());
        up(daijk, aijk.data(), sizeof(int4) * aijk.size());
        up(dakt, akt.data(), sizeof(double2) * akt.size());
        up(ddijkl, dijkl.data(), sizeof(int4) * dijkl.size());
        up(ddn, dn.data(), sizeof(int) * dn.size());
        up(ddkp, dkp.data(), sizeof(double2) * dkp.size());
        up(diijkl, iijkl.data(), sizeof(int4) * iijkl.size());
        up(dikp, ikp.data(), sizeof(double2) * ikp.size());
        up(dex, ex.data(), sizeof(int2) * ex.size());
        up(dexs, ex_start.data(), sizeof(int) * ex_start.size());
        up(dexl, ex_list.data(), sizeof(int) * ex_list.size());
        d.bond_ij = dbij;
        d.bond_kr = dbkr;
        d.ang_ijk = daijk;
        d.ang_kt = dakt;
        d.dih_ijkl = ddijkl;
        d.dih_n = ddn;
        d.dih_kp = ddkp;
        d.imp_ijkl = diijkl;
        d.imp_kp = dikp;
        d.excl = dex;
        d.ex_start = dexs;
        d.ex_list = dexl;
        d.n_cgroups = static_cast<int>(cgr.size());
        any_cons_ = d.n_cgroups > 0;
        if (any_cons_) {
            int* dcgb = A.alloc<int>(cgb.size());
            int* dcgr = A.alloc<int>(cgr.size());
            int2* dcij = A.alloc<int2>(cij.size());
            double* dcd = A.alloc<double>(cdist.size());
            up(dcgb, cgb.data(), sizeof(int) * cgb.size());
            up(dcgr, cgr.data(), sizeof(int) * cgr.size());
            up(dcij, cij.data(), sizeof(int2) * cij.size());
            up(dcd, cdist.data(), sizeof(double) * cdist.size());
            int* dcgab = A.alloc<int>(cgab.size());
            int* dcga = A.alloc<int>(cga.size());
            up(dcgab, cgab.data(), sizeof(int) * cgab.size());
            up(dcga, cga.data(), sizeof(int) * cga.size());
            d.cgroup_begin = dcgb;
            d.cgroup_rep = dcgr;
            d.cons_ij = dcij;
            d.cons_d = dcd;
            d.cgroup_atom_begin = dcgab;
            d.cgroup_atoms = dcga;
            d.cons_x0 = A.alloc<double>(3 * static_cast<size_t>(n_atoms));
        }
        if (any_pme_) {
            d.mesh_fix = A.alloc<long long>(mesh_fix);
            if (fp64_) {
                d.mesh_real = A.alloc<double>(mesh_real);
                d.mesh_cplx = A.alloc<double2>(mesh_cplx);
                d.pme_green = A.alloc<double>(mesh_cplx);
            } else {
                d.mesh_real = A.alloc<float>(mesh_real);
                d.mesh_cplx = A.alloc<float2>(mesh_cplx);
                d.pme_green = A.alloc<float>(mesh_cplx);
            }
            double* dbsp = A.alloc<double>(bsp.size());
            up(dbsp, bsp.data(), 8 * bsp.size());
            d.bsp = dbsp;
            d.pme_part = A.alloc<double>(2 * static_cast<size_t>(pme_blocks));
            int* dpbr = A.alloc<int>(pbr.size());
            up(dpbr, pbr.data(), 4 * pbr.size());
            d.pme_block_rep = dpbr;
            int* dcbr = A.alloc<int>(cbr.size());
            up(dcbr, cbr.data(), 4 * cbr.size());
            d.conv_block_rep = dcbr;
        }
        if (any_andersen_ref_) {
            d_and_flag_ = A.alloc<int>(n_atoms);
            d_and_v_ = A.alloc<double>(3 * n_atoms);
            d.and_flag = d_and_flag_;
            d.and_v = d_and_v_;
            if (n_atoms > h_and_cap_) {
                if (h_and_flag_) cudaFreeHost(h_and_flag_);
                if (h_and_v_) cudaFreeHost(h_and_v_);
                h_and_flag_ = nullptr;
                h_and_v_ = nullptr;
                h_and_cap_ = 0;
                const long long cap = n_atoms + n_atoms / 4;
                if (cudaMallocHost(&h_and_flag_, 4 * cap) != cudaSuccess ||
                    cudaMallocHost(&h_and_v_, 24 * cap) != cudaSuccess)
                    throw std::runtime_error("pinned alloc failed");
                h_and_cap_ = cap;
            }
        }
        up(d_rep_, hrep.data(), sizeof(Rep) * R);
        std::vector<RepState> hst(R);
        for (int k = 0; k < R; ++k) {
            HostRep& h = *reps_[order_[k]];
            hst[k] = h.init;
            hst[k].target_step = h.target;
        }
        up(d_st_, hst.data(), sizeof(RepState) * R);
        used_bytes_ = static_cast<long long>(A.bytes);
        fp_ratio_ = fp_sum ? static_cast<double>(A.bytes) / static_cast<double>(fp_sum) : 1.0;
    } catch (const std::exception& e) {
        cudaStreamSynchronize(stream_);
        arena_.reset();
        return fail(DMDGPU_ERR_OOM, std::string("device allocation/upload failed: ") + e.what());
    }
    // every zero fill and upload done; the staging blocks beyond 256 MB go back
    CK(cudaStreamSynchronize(stream_));
    staging_.trim(size_t(256) << 20);
    if (R > h_st_cap_) {
        if (h_st_) cudaFreeHost(h_st_);
        if (h_tgt_) cudaFreeHost(h_tgt_);
        h_st_ = nullptr;
        h_tgt_ = nullptr;
        h_st_cap_ = 0;
        const int cap = (R + 63) & ~63;
        CK(cudaMallocHost(&h_st_, sizeof(RepState) * cap));
        CK(cudaMallocHost(&h_tgt_, sizeof(long long) * cap));
        h_st_cap_ = cap;
    }
    st_fresh_ = false;
    // cuFFT plans per mesh size (normally made at admission already)
    for (int k = 0; k < R; ++k) {
        const Rep& P = reps_[order_[k]]->rep;
        if (P.flags & F_PME) {
            int rc = ensure_plans(P.pme_K);
            if (rc) return rc;
        }
    }
    for (int k : order_) reps_[k]->on_device = true;
    {
        // every replica's list, built in the frame of its last build (a new
        // replica: its current positions and box)
        std::vector<char> all(R, 1);
        int rc = rebuild_in_frame(all);
        if (rc) return rc;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        const TuneKey key = tune_key(device_, fp64_, any_pme_, dev_.n_atoms, opt_.nb_form, density_);
        auto it = g_tune.find(key);
        if (it == g_tune.end()) {
            // a table of a size not tuned yet takes the shape tuned for the
            // nearest size of the same kind, so a serving loop whose table size
            // changes with every admission tunes once, not at every rebuild
            int best = 1 << 30;
            for (auto jt = g_tune.begin(); jt != g_tune.end(); ++jt) {
                const TuneKey& k = jt->first;
                if (k.device != key.device || k.fp64 != key.fp64 || k.pme != key.pme || k.forced != key.forced)
                    continue;
                const int dist = 4 * std::abs(k.dens - key.dens) + std::abs(k.bucket - key.bucket);
                if (dist < best) {
                    best = dist;
                    it = jt;
                }
            }
        }
        tuned_ = fp64_ || it != g_tune.end();
        nb_form_ = uses_clusters() ? NB_CLUSTER8 : NB_CHUNK32;
        nb_blocks_per_sm_ = (it != g_tune.end()) ? it->second.bps : ((any_pme_ || nb_form_ == NB_CLUSTER8) ? 2 : 3);
    }
    packed_ = true;
    graph_dirty_ = true;
    return DMDGPU_OK;
}

// ---------------------------------------------------------------------------
// Step orchestration
// ---------------------------------------------------------------------------
void Batch::enqueue_eval(int pass) {
    Dev& d = dev_;
    launch_eval_begin(d, pass, stream_, &launches_);
    if (pass != PASS_SECOND) launch_clear_forces(d, stream_, &launches_);
    // The list rebuild (a cooperative launch: it needs the whole GPU) goes first;
    // it returns at once on steps without a rebuild.
    enqueue_rebuild();
    // Bonded terms and PME depend on atom positions only (not on the sorted slots),
    // so they run on two more streams concurrently with the pair kernel; all force
    // and energy sums are fixed-point atomics (order-free).  The pair kernel (the
    // longest branch, persistent) is issued first so its blocks take their SM
    // slots before the short PME and bonded blocks fill the rest.
    cudaEventRecord(ev_fork_, stream_);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof_nb_) {
        e0 = next_event();
        record(e0, stream_);
    }
    launch_nonbonded(d, fp64_, phys_, n_sm_, nb_blocks_per_sm_, nb_form_, stream_, &launches_);
    if (prof_nb_) {
        e1 = next_event();
        record(e1, stream_);
        prof_nb_->emplace_back(e0, e1);
    }
    cudaStreamWaitEvent(aux_stream_, ev_fork_, 0);
    cudaStreamWaitEvent(bond_stream_, ev_fork_, 0);
    if (any_pme_) {
        if (prof_pme_) {
            e0 = next_event();
            record(e0, aux_stream_);
        }
        launch_pme_spread(d, fp64_, aux_stream_, &launches_);
        launch_pme_convert(d, fp64_, n_conv_blocks_, aux_stream_, &launches_);
        for (int k : order_) {
            const Rep& P = reps_[k]->rep;
            if (!(P.flags & F_PME)) continue;
            auto& pl = plans_[P.pme_K];
            if (fp64_) {
                cufftExecD2Z(pl.first, static_cast<double*>(d.mesh_real) + P.mesh_real_off,
                             static_cast<cufftDoubleComplex*>(d.mesh_cplx) + P.mesh_cplx_off);
            } else {
                cufftExecR2C(pl.first, static_cast<float*>(d.mesh_real) + P.mesh_real_off,
                             static_cast<cufftComplex*>(d.mesh_cplx) + P.mesh_cplx_off);
            }
        }
        launch_pme_influence(d, fp64_, n_pme_blocks_, aux_stream_, &launches_);
        for (int k : order_) {
            const Rep& P = reps_[k]->rep;
            if (!(P.flags & F_PME)) continue;
            auto& pl = plans_[P.pme_K];
            if (fp64_) {
                cufftExecZ2D(pl.second, static_cast<cufftDoubleComplex*>(d.mesh_cplx) + P.mesh_cplx_off,
                             static_cast<double*>(d.mesh_real) + P.mesh_real_off);
            } else {
                cufftExecC2R(pl.second, static_cast<cufftComplex*>(d.mesh_cplx) + P.mesh_cplx_off,
                             static_cast<float*>(d.mesh_real) + P.mesh_real_off);
            }
        }
        launch_pme_gather(d, fp64_, aux_stream_, &launches_);
        if (prof_pme_) {
            e1 = next_event();
            record(e1, aux_stream_);
            prof_pme_->emplace_back(e0, e1);
        }
    }
    cudaEventRecord(ev_join_, aux_stream_);
    launch_bonded(d, fp64_, phys_, bond_stream_, &launches_);
    cudaEventRecord(ev_join_b_, bond_stream_);
    cudaStreamWaitEvent(stream_, ev_join_, 0);
    cudaStreamWaitEvent(stream_, ev_join_b_, 0);
    // the second pass of a step is closed by k_replica_update
    if (pass != PASS_SECOND) launch_eval_end(d, stream_, &launches_);
}

// Neighbour-list rebuild: one cooperative launch that returns at once unless
// some replica's rebuild flag is set.
void Batch::enqueue_rebuild() { launch_rebuild(dev_, d_bin_rep_, n_sm_, stream_, &launches_); }

void Batch::enqueue_step() {
    // The first evaluation repeats the previous step's second one unless the
    // barostat moved the atoms, the REF list cadence rebuilds now, or no forces
    // exist yet; only then is it issued (its kernels skip replicas that do not need it).
    if (need_eval1_) enqueue_eval(PASS_FIRST);
    launch_kick_drift(dev_, fp64_, stream_, &launches_);
    if (any_cons_) launch_shake(dev_, stream_, &launches_);
    enqueue_eval(PASS_SECOND);
    launch_kick2(dev_, any_andersen_ref_, any_andersen_phys_, stream_, &launches_);
    if (any_cons_) launch_rattle(dev_, stream_, &launches_);
    launch_replica_update(dev_, stream_, &launches_);
    if (any_baro_ && !phys_) launch_apply_scale(dev_, fp64_, stream_, &launches_);
}

// AndersenThermostat::apply (andersen.cpp:14-32): the REF profile reproduces the
// reference's mt19937_64 stream on the host and uploads the resampled velocities.
void Batch::andersen_ref_prepare() {
    std::memset(h_and_flag_, 0, sizeof(int) * dev_.n_atoms);
    for (int k : order_) {
        HostRep& h = *reps_[k];
        const HostSystem& s = h.sys;
        if (s.thermostat != 3) continue;
        const double prob = s.t_freq * s.dt;
        if (prob <= 0.0) continue;
        std::mt19937_64 rng(h.andersen_seed);
        std::uniform_real_distribution<double> uni(0.0, 1.0);
        std::normal_distribution<double> nd(0.0, 1.0);
        const int a0 = h.rep.atom_begin;
        for (int i = 0; i < s.n; ++i) {
            if (uni(rng) < prob) {
                double sigma = std::sqrt(KB * s.t_temp / s.mass[i]);
                h_and_flag_[a0 + i] = 1;
                h_and_v_[3 * (a0 + i)] = nd(rng) * sigma;
                h_and_v_[3 * (a0 + i) + 1] = nd(rng) * sigma;
                h_and_v_[3 * (a0 + i) + 2] = nd(rng) * sigma;
            }
        }
        ++h.andersen_seed;
    }
    cudaMemcpyAsync(d_and_flag_, h_and_flag_, sizeof(int) * dev_.n_atoms, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(d_and_v_, h_and_v_, sizeof(double) * 3 * dev_.n_atoms, cudaMemcpyHostToDevice, stream_);
}

// Kernel-node priorities of a captured step: the pair kernel low, every other
// kernel (bonded terms, the PME chain, cuFFT's kernels, integration) high.
// The graph is instantiated with cudaGraphInstantiateFlagUseNodePriority.
void Batch::set_node_priorities(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return;
    }
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(node, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp{};
        bool nb = false;
        if (cudaGraphKernelNodeGetParams(node, &kp) == cudaSuccess) nb = is_nonbonded_kernel(kp.func);
        else cudaGetLastError();  // a kernel launched through the driver API (cuFFT)
        cudaKernelNodeAttrValue v{};
        v.priority = nb ? prio_lo_ : prio_hi_;
        if (cudaGraphKernelNodeSetAttribute(node, cudaKernelNodeAttributePriority, &v) != cudaSuccess)
            cudaGetLastError();
    }
}

int Batch::run_steps(int n) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    if (n <= 0) return DMDGPU_OK;
    static const bool eager = [] {
        const char* e = std::getenv("DMD_EAGER");
        return e && e[0] == '1';
    }();
    if (eager && !any_andersen_ref_) {
        // every launch issued from the host (profilers see each kernel); same work
        need_eval1_ = true;
        for (int i = 0; i < n; ++i) {
            enqueue_step();
            CK(cudaGetLastError());
            if (i == 0) need_eval1_ = (any_baro_ && !phys_) || any_ref_lj_;
        }
        graph_dirty_ = true;
        return DMDGPU_OK;
    }
    if (any_andersen_ref_) {
        // host-generated random stream per step: no graph
        need_eval1_ = true;
        for (int i = 0; i < n; ++i) {
            andersen_ref_prepare();
            CK(cudaStreamSynchronize(stream_));
            enqueue_step();
            CK(cudaGetLastError());
        }
        return DMDGPU_OK;
    }
    if (graph_dirty_ || !graph_) {
        // first step eagerly (initial list + forces), then capture the steady-state step
        need_eval1_ = true;
        enqueue_step();
        CK(cudaGetLastError());
        need_eval1_ = (any_baro_ && !phys_) || any_ref_lj_;
        --n;
        if (!tuned_) {
            int used = 0;
            int rc = autotune(n, &used);
            if (rc) return rc;
            n -= used;
        }
        if (graph_) cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
        cudaGraph_t g;
        long long before = launches_;
        capture_error_ = false;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        enqueue_step();
        CK(cudaStreamEndCapture(stream_, &g));
        if (capture_error_) {
            cudaGraphDestroy(g);
            return fail(DMDGPU_ERR_GPU, "conditional-node capture failed");
        }
        per_step_launches_ = launches_ - before;
        set_node_priorities(g);
        CK(cudaGraphInstantiate(&graph_, g, cudaGraphInstantiateFlagUseNodePriority));
        cudaGraphDestroy(g);
        graph_dirty_ = false;
    }
    for (int i = 0; i < n; ++i) {
        CK(cudaGraphLaunch(graph_, stream_));
        launches_ += per_step_launches_;
    }
    return DMDGPU_OK;
}

// Pair-kernel launch shape by measurement: each candidate runs kTuneSteps real
// steps (eagerly, in the same order as the captured step) timed with events on
// the main stream, which the bonded / PME stream joins every step; the fastest
// median step wins and is cached for this kind of batch.  The candidates give
// bit-identical results, so tuning steps are ordinary steps of the run.  Runs
// only when the call has enough steps to spare.
int Batch::autotune(int max_steps, int* used) {
    *used = 0;
    // The form itself is not tuned: its FP32 summation order differs, so a
    // choice made by timing would make results differ from run to run and
    // between a system alone and the same system in a batch.  Only the launch
    // shape, which changes no result bit, is chosen by measurement.
    const int form = uses_clusters() ? NB_CLUSTER8 : NB_CHUNK32;
    std::vector<TuneChoice> cand;
    for (const TuneChoice& c : kTuneCand)
        if (c.form == form) cand.push_back(c);
    const int n_cand = static_cast<int>(cand.size());
    if (max_steps < n_cand * kTuneSteps) return DMDGPU_OK;
    std::vector<cudaEvent_t> ev(kTuneSteps + 1);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    TuneChoice best{nb_form_, nb_blocks_per_sm_};
    float best_ms = 1e30f;
    for (int c = 0; c < n_cand; ++c) {
        nb_form_ = cand[c].form;
        nb_blocks_per_sm_ = cand[c].bps;
        std::vector<float> t(kTuneSteps);
        CK(cudaEventRecord(ev[0], stream_));
        for (int i = 0; i < kTuneSteps; ++i) {
            enqueue_step();
            CK(cudaEventRecord(ev[i + 1], stream_));
        }
        CK(cudaGetLastError());
        CK(cudaEventSynchronize(ev[kTuneSteps]));
        for (int i = 0; i < kTuneSteps; ++i) CK(cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
        std::sort(t.begin(), t.end());
        const float med = t[kTuneSteps / 2];
        if (med < best_ms) {
            best_ms = med;
            best = cand[c];
        }
        *used += kTuneSteps;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    nb_form_ = best.form;
    nb_blocks_per_sm_ = best.bps;
    tuned_ = true;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(device_, fp64_, any_pme_, dev_.n_atoms, opt_.nb_form, density_)] = best;
    return DMDGPU_OK;
}

// Pair lists of the selected replicas (packed indices) rebuilt in the frame of
// their last build: positions xr/yr/zr (already on the device) and box L_build.
// The slot order, tile centres, frozen images and chunk lists then equal the
// ones the replica had, so a table rebuild or a checkpoint restart continues
// bit for bit.  Afterwards the current box and counters are restored, forces
// are marked for evaluation and the mirror is rewritten from the positions.
int Batch::rebuild_in_frame(const std::vector<char>& sel) {
    const int R = static_cast<int>(order_.size());
    if (R == 0) return DMDGPU_OK;
    std::vector<RepState> cur(R), tmp(R);
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(cur.data(), d_st_, sizeof(RepState) * R, cudaMemcpyDeviceToHost));
    tmp = cur;
    for (int k = 0; k < R; ++k) {
        tmp[k].rebuild = sel[k] ? 1 : 0;
        if (sel[k]) {
            tmp[k].L = cur[k].L_build;
            tmp[k].invL = 1.0 / cur[k].L_build;
        }
    }
    CK(cudaMemcpy(d_st_, tmp.data(), sizeof(RepState) * R, cudaMemcpyHostToDevice));
    Dev frame = dev_;
    frame.x = dev_.xr;
    frame.y = dev_.yr;
    frame.z = dev_.zr;
    launch_rebuild(frame, d_bin_rep_, n_sm_, stream_, &launches_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(tmp.data(), d_st_, sizeof(RepState) * R, cudaMemcpyDeviceToHost));
    for (int k = 0; k < R; ++k) {
        if (!sel[k]) {
            tmp[k] = cur[k];
            continue;
        }
        RepState& f = tmp[k];
        f.L = cur[k].L;
        f.invL = cur[k].invL;
        f.L_build = cur[k].L_build;
        f.lj_counter = cur[k].lj_counter;
        // a replica that had built before keeps a pending rebuild request; a new
        // one has just been built at its current positions
        f.rebuild = cur[k].list_builds > 0 ? cur[k].rebuild : 0;
        f.list_builds = std::max(cur[k].list_builds, 1LL);
        f.have_forces = 0;
    }
    CK(cudaMemcpy(d_st_, tmp.data(), sizeof(RepState) * R, cudaMemcpyHostToDevice));
    launch_write_mirror(dev_, fp64_, stream_, &launches_);
    CK(cudaGetLastError());
    st_fresh_ = false;
    graph_dirty_ = true;
    return DMDGPU_OK;
}

int Batch::sync_status() {
    if (!packed_ || order_.empty()) return DMDGPU_OK;
    CK(cudaMemcpyAsync(h_st_, d_st_, sizeof(RepState) * order_.size(), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    st_fresh_ = true;
    int rc = DMDGPU_OK;
    for (size_t k = 0; k < order_.size(); ++k) {
        HostRep& h = *reps_[order_[k]];
        const int st = h_st_[k].status;
        // the cause first: a truncated list makes every force after it meaningless
        if (st & ST_TIMEOUT) {
            failed_ = true;
            rc = fail(DMDGPU_ERR_GPU, "list-build grid barrier timed out");
        } else if (st & ST_CAPACITY) rc = fail(DMDGPU_ERR_CAPACITY, "pair list capacity exceeded");
        else if (st & ST_NAN) rc = fail(DMDGPU_ERR_NAN, "non-finite force or energy on device");
        else if (st & ST_RANGE) rc = fail(DMDGPU_ERR_BOND_EXPLOSION, "force outside the fixed-point range");
        if (!h.done && h.target > 0 && h_st_[k].step >= h.target) {
            h.done = true;
            finished_.push_back(order_[k]);
        }
    }
    return rc;
}

int Batch::step(int n) {
    CK(cudaSetDevice(device_));
    if (failed_) return fail(DMDGPU_ERR_GPU, "a list build timed out earlier; the table is unusable");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    if (order_.empty()) return DMDGPU_OK;
    if (frame_fn_ && frame_interval_ > 0 && order_.size() == 1) {
        // steps in runs that end on frame steps, a frame issued after each
        if (!st_fresh_) {
            CK(cudaMemcpyAsync(h_st_, d_st_, sizeof(RepState), cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            st_fresh_ = true;
        }
        long long s = h_st_[0].step;
        const long long I = frame_interval_;
        int left = n;
        while (left > 0) {
            const long long next = (s / I + 1) * I;
            const int k = static_cast<int>(std::min<long long>(left, next - s));
            int rc = run_steps(k);
            if (rc) return rc;
            s += k;
            left -= k;
            if (s == next) {
                rc = enqueue_frame();
                if (rc) return rc;
            }
        }
        return sync_status();
    }
    int rc = run_steps(n);
    if (rc) return rc;
    return sync_status();
}

// ---------------------------------------------------------------------------
// Trajectory frames.  The snapshot kernel reads the state the last step left
// (positions, velocities with the pending thermostat scale, step, time, box)
// and changes nothing, so exporting leaves the trajectory bit for bit as it is.
// Slot k is reused only after the copy stream has delivered its previous
// frame (frame_done_), so the main stream waits only when the writer is
// DMDGPU_FRAME_SLOTS frames behind.
// ---------------------------------------------------------------------------
int Batch::set_frame_writer(int interval, dmdgpu_frame_fn fn, void* user) {
    CK(cudaSetDevice(device_));
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    free_frames();
    if (interval <= 0 || !fn) return DMDGPU_OK;
    if (order_.size() != 1) return fail(DMDGPU_ERR_INVALID, "frames are exported for a single-system context");
    frame_n_ = reps_[order_[0]]->sys.n;
    const size_t bytes = sizeof(double) * (3 + 6 * static_cast<size_t>(frame_n_));
    CK(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    for (int k = 0; k < DMDGPU_FRAME_SLOTS; ++k) {
        CK(cudaMalloc(&frame_dev_[k], bytes));
        CK(cudaMallocHost(&frame_host_[k], bytes));
        CK(cudaEventCreateWithFlags(&frame_snap_[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&frame_done_[k], cudaEventDisableTiming));
        CK(cudaEventRecord(frame_done_[k], copy_stream_));
        frame_slot_[k] = FrameSlot{this, k};
    }
    frame_interval_ = interval;
    frame_fn_ = fn;
    frame_user_ = user;
    frame_count_ = 0;
    return DMDGPU_OK;
}

int Batch::flush_frames() {
    if (copy_stream_) CK(cudaStreamSynchronize(copy_stream_));
    return DMDGPU_OK;
}

void Batch::free_frames() {
    if (copy_stream_) cudaStreamSynchronize(copy_stream_);
    for (int k = 0; k < DMDGPU_FRAME_SLOTS; ++k) {
        if (frame_dev_[k]) cudaFree(frame_dev_[k]);
        if (frame_host_[k]) cudaFreeHost(frame_host_[k]);
        if (frame_snap_[k]) cudaEventDestroy(frame_snap_[k]);
        if (frame_done_[k]) cudaEventDestroy(frame_done_[k]);
        frame_dev_[k] = nullptr;
        frame_host_[k] = nullptr;
        frame_snap_[k] = nullptr;
        frame_done_[k] = nullptr;
    }
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
    copy_stream_ = nullptr;
    frame_fn_ = nullptr;
    frame_interval_ = 0;
}

int Batch::enqueue_frame() {
    const int k = static_cast<int>(frame_count_ % DMDGPU_FRAME_SLOTS);
    const size_t bytes = sizeof(double) * (3 + 6 * static_cast<size_t>(frame_n_));
    CK(cudaStreamWaitEvent(stream_, frame_done_[k], 0));
    launch_frame_snapshot(dev_, 0, frame_n_, frame_dev_[k], stream_, &launches_);
    CK(cudaGetLastError());
    CK(cudaEventRecord(frame_snap_[k], stream_));
    CK(cudaStreamWaitEvent(copy_stream_, frame_snap_[k], 0));
    CK(cudaMemcpyAsync(frame_host_[k], frame_dev_[k], bytes, cudaMemcpyDeviceToHost, copy_stream_));
    CK(cudaLaunchHostFunc(copy_stream_, &Batch::deliver_frame, &frame_slot_[k]));
    CK(cudaEventRecord(frame_done_[k], copy_stream_));
    ++frame_count_;
    st_fresh_ = false;
    return DMDGPU_OK;
}

void CUDART_CB Batch::deliver_frame(void* p) {
    const FrameSlot* fs = static_cast<const FrameSlot*>(p);
    const Batch* b = fs->self;
    const double* h = b->frame_host_[fs->index];
    const int n = b->frame_n_;
    dmdgpu_frame f;
    f.step = static_cast<int64_t>(h[0]);
    f.time = h[1];
    f.box = h[2];
    f.n_atoms = n;
    f.x = h + 3;
    f.y = h + 3 + n;
    f.z = h + 3 + 2 * n;
    f.vx = h + 3 + 3 * n;
    f.vy = h + 3 + 4 * n;
    f.vz = h + 3 + 5 * n;
    b->frame_fn_(&f, b->frame_user_);
}

cudaEvent_t Batch::next_event() {
    if (ev_used_ == ev_pool_.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ev_pool_.push_back(e);
    }
    return ev_pool_[ev_used_++];
}

int Batch::extend_targets(long long n) {
    CK(cudaSetDevice(device_));
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    if (order_.empty()) return DMDGPU_OK;
    // The step counters come from the host mirror when nothing ran since it was
    // read (the common run_n loop: no device round trip); the new targets go
    // to the device asynchronously from pinned memory, ahead of the next step.
    if (!st_fresh_) {
        CK(cudaMemcpyAsync(h_st_, d_st_, sizeof(RepState) * order_.size(), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        st_fresh_ = true;
    }
    for (size_t k = 0; k < order_.size(); ++k) {
        const long long tgt = h_st_[k].step + n;
        h_tgt_[k] = tgt;
        h_st_[k].target_step = tgt;
        CK(cudaMemcpyAsync(&d_st_[k].target_step, h_tgt_ + k, 8, cudaMemcpyHostToDevice, stream_));
        reps_[order_[k]]->target = tgt;
        reps_[order_[k]]->done = false;
    }
    return DMDGPU_OK;
}

// Event record usable for timing inside a captured graph: an external event
// node (a plain record during capture only becomes a graph dependency).
void Batch::record(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else cudaEventRecord(e, st);
}

// n steps with device timing.  Every step is one launch of a one-step graph,
// between two events recorded on the main stream (the optional L2 flush goes
// before the first event).  Seven of every eight launches are of the step
// graph run_n uses; every eighth is of a copy with event record nodes around
// every pair-kernel launch and every PME chain, whose nodes are pointed at
// fresh events before each launch (cudaGraphExecEventRecordNodeSetEvent), so
// the pair kernel's and the PME chain's durations are those of the sampled
// steps.  Event nodes on the critical path add a few microseconds to their
// step, and capturing all n steps into one graph with their events changed
// how the branches were scheduled (water 30k: a step period of ~143 us
// against ~124 us for run_n's graph), hence one step graph and sampling.
int Batch::step_timed(int n, long long flush_bytes, dmdgpu_timing* out) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    std::memset(out, 0, sizeof(*out));
    if (failed_) return fail(DMDGPU_ERR_GPU, "a list build timed out earlier; the table is unusable");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    if (n <= 0) return DMDGPU_OK;
    if (graph_dirty_ || !graph_ || any_andersen_ref_) {
        int rc = run_steps(1);  // initial forces / steady-state configuration
        if (rc) return rc;
        CK(cudaStreamSynchronize(stream_));
        --n;
        if (n == 0) return sync_status();
    }
    if (any_andersen_ref_) return fail(DMDGPU_ERR_INVALID, "timed steps need the step graph (not with a host-drawn Andersen stream)");
    if (flush_bytes > 0 && flush_bytes != flush_bytes_) {
        if (flush_buf_) cudaFree(flush_buf_);
        flush_buf_ = nullptr;
        CK(cudaMalloc(&flush_buf_, flush_bytes));
        flush_bytes_ = flush_bytes;
    }
    // capture one step with its pair-kernel and PME events
    ev_used_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> nb0, pme0;
    prof_nb_ = &nb0;
    prof_pme_ = &pme0;
    cudaGraph_t g;
    const long long before = launches_;
    capture_error_ = false;
    cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_step();
        e = cudaStreamEndCapture(stream_, &g);
    }
    prof_nb_ = nullptr;
    prof_pme_ = nullptr;
    if (e != cudaSuccess || capture_error_) {
        cudaGetLastError();
        return fail(DMDGPU_ERR_GPU, std::string("timed capture failed: ") + cudaGetErrorString(e));
    }
    const long long per_step = launches_ - before;
    launches_ = before;
    // the event record nodes, in the order of nb0 / pme0 (start, end)
    std::vector<cudaGraphNode_t> nb_nodes(2 * nb0.size()), pme_nodes(2 * pme0.size());
    {
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(g, nodes.data(), &nn);
        for (cudaGraphNode_t node : nodes) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(node, &t) != cudaSuccess || t != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev = nullptr;
            if (cudaGraphEventRecordNodeGetEvent(node, &ev) != cudaSuccess) continue;
            for (size_t k = 0; k < nb0.size(); ++k) {
                if (ev == nb0[k].first) nb_nodes[2 * k] = node;
                if (ev == nb0[k].second) nb_nodes[2 * k + 1] = node;
            }
            for (size_t k = 0; k < pme0.size(); ++k) {
                if (ev == pme0[k].first) pme_nodes[2 * k] = node;
                if (ev == pme0[k].second) pme_nodes[2 * k + 1] = node;
            }
        }
        for (cudaGraphNode_t node : nb_nodes)
            if (!node) {
                cudaGraphDestroy(g);
                return fail(DMDGPU_ERR_GPU, "timed capture: pair-kernel event nodes not found");
            }
        for (cudaGraphNode_t node : pme_nodes)
            if (!node) {
                cudaGraphDestroy(g);
                return fail(DMDGPU_ERR_GPU, "timed capture: PME event nodes not found");
            }
    }
    set_node_priorities(g);
    cudaGraphExec_t ge;
    e = cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return check_cuda(e, "cudaGraphInstantiate");
    }
    // g (whose nodes name the exec graph's event nodes) lives until the end
    // events for every launch: the step's pair, then the nodes' pairs
    const size_t per_launch = 2 + nb_nodes.size() + pme_nodes.size();
    const size_t need = ev_used_ + per_launch * static_cast<size_t>(n);
    while (ev_pool_.size() < need) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        ev_pool_.push_back(ev);
    }
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> nb, pme, steps;
    auto point = [&](const std::vector<cudaGraphNode_t>& nodes, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& out) {
        for (size_t k = 0; k < nodes.size() && e == cudaSuccess; k += 2) {
            const cudaEvent_t x = next_event(), y = next_event();
            e = cudaGraphExecEventRecordNodeSetEvent(ge, nodes[k], x);
            if (e == cudaSuccess) e = cudaGraphExecEventRecordNodeSetEvent(ge, nodes[k + 1], y);
            out.emplace_back(x, y);
        }
    };
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        if (flush_buf_) cudaMemsetAsync(flush_buf_, i & 0xff, flush_bytes_, stream_);
        const cudaEvent_t a = next_event(), b = next_event();
        const bool sampled = (i % 8) == 7 || (n < 8 && i == n - 1);
        if (sampled) {
            point(nb_nodes, nb);
            point(pme_nodes, pme);
            if (e != cudaSuccess) break;
        }
        cudaEventRecord(a, stream_);
        e = cudaGraphLaunch(sampled ? ge : graph_, stream_);
        cudaEventRecord(b, stream_);
        steps.emplace_back(a, b);
        launches_ += per_step;
    }
    const cudaError_t e_sync = cudaStreamSynchronize(stream_);
    if (e == cudaSuccess) e = e_sync;
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return check_cuda(e, "timed steps");
    float ms = 0.f;
    for (auto& pr : steps) {
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        out->step_ms += ms;
    }
    for (auto& pr : nb) {
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        out->nonbonded_ms += ms;
    }
    for (auto& pr : pme) {
        CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        out->pme_ms += ms;
    }
    out->nonbonded_launches = static_cast<long long>(nb.size());
    out->sampled_steps = static_cast<long long>(nb_nodes.empty() ? 0 : nb.size() / (nb_nodes.size() / 2));
    int rc = sync_status();
    out->kernel_launches = per_step * n;
    return rc;
}

void Batch::launch_info(dmdgpu_launch_info* out) const {
    *out = dmdgpu_launch_info{};
    out->packed = packed_ && !order_.empty() ? 1 : 0;
    if (!out->packed) return;
    out->nb_form = nb_form_ == NB_CLUSTER8 ? DMDGPU_NB_CLUSTER8 : DMDGPU_NB_CHUNK32;
    out->nb_blocks_per_sm = fp64_ ? 8 : nb_blocks_per_sm_;
    out->tuned = tuned_ ? 1 : 0;
    out->min_image_kernel = fp64_ ? 0 : dev_.mi_split;  // the FP64 kernel always takes it
    out->n_replicas = static_cast<int32_t>(order_.size());
    out->n_atoms = dev_.n_atoms;
    out->launches_per_step = per_step_launches_;
}

int Batch::active() const {
    int c = 0;
    for (int k : order_)
        if (reps_[k] && !reps_[k]->done) ++c;
    return c;
}

// Failure-path test hooks.  Both act on the host: they only change what the
// next list build is given, and every wait they make run out is bounded.
//  BARRIER_TIMEOUT: the grid barrier waits for one arrival more than the grid
//    has blocks, so no arrival completes it; each wait gives up after 20 ms,
//    records ST_TIMEOUT and the blocks leave the kernel.  The forces of that
//    step come from the previous (still intact) list.
//  LIST_CAPACITY: every replica's chunk capacity becomes 1, so the next build
//    overflows; the builders write no chunk beyond the capacity.
int Batch::inject(int what) {
    CK(cudaSetDevice(device_));
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    if (order_.empty()) return fail(DMDGPU_ERR_INVALID, "empty batch");
    CK(cudaStreamSynchronize(stream_));
    st_fresh_ = false;
    if (what == DMDGPU_INJECT_BARRIER_TIMEOUT) {
        dev_.bar_extra = 1;
        dev_.bar_limit_ns = 20000000ull;
    } else if (what == DMDGPU_INJECT_LIST_CAPACITY) {
        for (size_t k = 0; k < order_.size(); ++k) {
            reps_[order_[k]]->rep.chunk_cap = 1;
            const int one = 1;
            CK(cudaMemcpy(&d_rep_[k].chunk_cap, &one, 4, cudaMemcpyHostToDevice));
        }
    } else {
        return fail(DMDGPU_ERR_PARM, "unknown injection");
    }
    for (size_t k = 0; k < order_.size(); ++k) {
        const int one = 1;
        CK(cudaMemcpy(&d_st_[k].rebuild, &one, 4, cudaMemcpyHostToDevice));
    }
    graph_dirty_ = true;  // the kernels take the changed table by value
    return DMDGPU_OK;
}

int Batch::poll(int32_t* slots, int cap, int* n_done) {
    int c = 0;
    for (int s : finished_) {
        if (c < cap && slots) slots[c] = s;
        ++c;
    }
    *n_done = c;
    finished_.clear();
    return DMDGPU_OK;
}

// ---------------------------------------------------------------------------
// State access
// ---------------------------------------------------------------------------
int Batch::get_state(int slot, int which, double* x, double* y, double* z) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    const int k = replica_index(slot);
    const HostRep& h = *reps_[slot];
    const int a0 = h.rep.atom_begin, n = h.sys.n;
    if (which == 0) {
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(x, dev_.x + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(y, dev_.y + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(z, dev_.z + a0, 8 * n, cudaMemcpyDeviceToHost));
    } else if (which == 1) {
        launch_finalize_velocities(dev_, stream_, &launches_);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(x, dev_.vx + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(y, dev_.vy + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(z, dev_.vz + a0, 8 * n, cudaMemcpyDeviceToHost));
    } else if (which == 2) {
        CK(cudaStreamSynchronize(stream_));
        const Rep& P = h.rep;
        const int s0 = 32 * P.tile_begin, ns = 32 * P.n_tiles;
        std::vector<long long> fb(3 * n), fn(3 * ns);
        std::vector<int> sl(n);
        CK(cudaMemcpy(fb.data(), dev_.fbx + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fb.data() + n, dev_.fby + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fb.data() + 2 * n, dev_.fbz + a0, 8 * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fn.data(), dev_.fnx + s0, 8 * ns, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fn.data() + ns, dev_.fny + s0, 8 * ns, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fn.data() + 2 * ns, dev_.fnz + s0, 8 * ns, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(sl.data(), dev_.slot_of_atom + a0, 4 * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) {
            const int s = sl[i] - s0;
            x[i] = static_cast<double>(fb[i] + fn[s]) * (1.0 / FSCALE);
            y[i] = static_cast<double>(fb[n + i] + fn[ns + s]) * (1.0 / FSCALE);
            z[i] = static_cast<double>(fb[2 * n + i] + fn[2 * ns + s]) * (1.0 / FSCALE);
        }
    } else {
        return fail(DMDGPU_ERR_PARM, "which must be 0, 1 or 2");
    }
    (void)k;
    return DMDGPU_OK;
}

int Batch::set_state(int slot, int which, const double* x, const double* y, const double* z) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    HostRep& h = *reps_[slot];
    const int a0 = h.rep.atom_begin, n = h.sys.n;
    const int k = replica_index(slot);
    CK(cudaStreamSynchronize(stream_));
    if (which == 0) {
        CK(cudaMemcpy(dev_.x + a0, x, 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dev_.y + a0, y, 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dev_.z + a0, z, 8 * n, cudaMemcpyHostToDevice));
        // new positions: rebuild the list and recompute forces before the next kick
        int one = 1, zero = 0;
        CK(cudaMemcpy(&d_st_[k].rebuild, &one, 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(&d_st_[k].have_forces, &zero, 4, cudaMemcpyHostToDevice));
        graph_dirty_ = true;  // the next step must evaluate forces first
    } else if (which == 1) {
        launch_finalize_velocities(dev_, stream_, &launches_);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(dev_.vx + a0, x, 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dev_.vy + a0, y, 8 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dev_.vz + a0, z, 8 * n, cudaMemcpyHostToDevice));
    } else {
        return fail(DMDGPU_ERR_PARM, "which must be 0 or 1");
    }
    return DMDGPU_OK;
}

int Batch::get_scalars(int slot, dmdgpu_scalars* out) {
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    const int k = replica_index(slot);
    if (!st_fresh_) {
        CK(cudaMemcpyAsync(h_st_ + k, d_st_ + k, sizeof(RepState), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    const RepState& s = h_st_[k];
    const HostRep& h = *reps_[slot];
    const Rep& P = h.rep;
    std::memset(out, 0, sizeof(*out));
    out->step = s.step;
    out->time = s.time;
    out->box = s.L;
    double e[9];
    e[0] = static_cast<double>(s.e_acc[E_LJ]) / ESCALE;
    e[1] = static_cast<double>(s.e_acc[E_CREAL]) / ESCALE;
    e[2] = (P.flags & F_PME) ? s.e_recip : 0.0;
    e[3] = (P.flags & F_PME) ? P.e_self : 0.0;
    e[4] = static_cast<double>(s.e_acc[E_CEXCL]) / ESCALE;
    e[5] = static_cast<double>(s.e_acc[E_BOND]) / ESCALE;
    e[6] = static_cast<double>(s.e_acc[E_ANGLE]) / ESCALE;
    e[7] = static_cast<double>(s.e_acc[E_DIH]) / ESCALE;
    e[8] = static_cast<double>(s.e_acc[E_IMP]) / ESCALE;
    double pe = 0.0;
    for (int t = 0; t < 9; ++t) {
        out->e_terms[t] = e[t];
        pe += e[t];
    }
    out->potential_energy = pe;
    out->kinetic_energy = s.ke;
    const double nn = static_cast<double>(h.sys.n);
    out->temperature = h.sys.n < 2 ? 0.0 : 2.0 * s.ke / ((3.0 * nn - 3.0) * KB);
    out->pressure = s.pressure;
    out->virial = s.virial;
    out->zeta = s.zeta;
    out->list_builds = s.list_builds;
    out->lj_step_since_rebuild = s.lj_counter;
    out->status = s.status;
    out->list_chunks = s.n_chunks;
    return DMDGPU_OK;
}

int Batch::compute_forces(int slot, double* fx, double* fy, double* fz, double* e_terms) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (failed_) return fail(DMDGPU_ERR_GPU, "a list build timed out earlier; the table is unusable");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    const int k = replica_index(slot);
    int one = 1;
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&d_st_[k].rebuild, &one, 4, cudaMemcpyHostToDevice));
    enqueue_eval(PASS_SINGLE);
    launch_energy_reduce(dev_, stream_, &launches_);
    CK(cudaGetLastError());
    int rc = sync_status();
    if (rc) return rc;
    if (fx) {
        rc = get_state(slot, 2, fx, fy, fz);
        if (rc) return rc;
    }
    if (e_terms) {
        dmdgpu_scalars s;
        rc = get_scalars(slot, &s);
        if (rc) return rc;
        std::memcpy(e_terms, s.e_terms, sizeof(double) * 9);
    }
    return DMDGPU_OK;
}

int Batch::pair_list(int slot, int32_t* pi, int32_t* pj, long long cap, long long* count) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    const int k = replica_index(slot);
    const HostRep& h = *reps_[slot];
    const Rep& P = h.rep;
    CK(cudaStreamSynchronize(stream_));
    RepState st;
    CK(cudaMemcpy(&st, d_st_ + k, sizeof(RepState), cudaMemcpyDeviceToHost));
    const int nc = st.n_chunks;
    std::vector<int> it(nc);
    std::vector<uint32_t> je(32LL * nc), mk(32LL * nc);
    std::vector<int> aos(32 * P.n_tiles);
    if (nc) {
        CK(cudaMemcpy(it.data(), dev_.chunk_itile + P.chunk_begin, 4 * nc, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(je.data(), dev_.chunk_j + 32LL * P.chunk_begin, 128LL * nc, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(mk.data(), dev_.chunk_mask + 32LL * P.chunk_begin, 128LL * nc, cudaMemcpyDeviceToHost));
    }
    CK(cudaMemcpy(aos.data(), dev_.atom_of_slot + 32 * P.tile_begin, 4 * 32 * P.n_tiles, cudaMemcpyDeviceToHost));
    const int s0 = 32 * P.tile_begin, a0 = P.atom_begin;
    std::vector<std::pair<int, int>> pairs;
    for (int c = 0; c < nc; ++c) {
        const int I = it[c];
        for (int l = 0; l < 32; ++l) {
            uint32_t m = mk[32LL * c + l];
            if (!m) continue;
            const int js = static_cast<int>(je[32LL * c + l] & 0x03FFFFFFu);
            const int aj = aos[js - s0] - a0;
            for (; m; m &= m - 1) {
                const int i = __builtin_ctz(m);
                const int ai = aos[32 * I + i - s0] - a0;
                pairs.emplace_back(std::min(ai, aj), std::max(ai, aj));
            }
        }
    }
    std::sort(pairs.begin(), pairs.end());
    if (dev_.cl_j && nc) {
        // the i-cluster rows must encode exactly the same pair set
        std::vector<int2> job(4LL * P.n_tiles);
        CK(cudaMemcpy(job.data(), dev_.cl_job + 4LL * P.tile_begin, sizeof(int2) * job.size(),
                      cudaMemcpyDeviceToHost));
        const int rows = st.n_cl;
        std::vector<uint32_t> cj(32LL * rows);
        std::vector<uint8_t> cm(32LL * rows);
        if (rows) {
            CK(cudaMemcpy(cj.data(), dev_.cl_j + 32LL * P.cl_begin, 4LL * cj.size(), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(cm.data(), dev_.cl_m + 32LL * P.cl_begin, cm.size(), cudaMemcpyDeviceToHost));
        }
        std::vector<std::pair<int, int>> cp;
        cp.reserve(pairs.size());
        for (int t = 0; t < P.n_tiles; ++t)
            for (int k = 0; k < 4; ++k) {
                const int2 jb = job[4 * t + k];
                for (int g = jb.x; g < jb.x + jb.y; ++g) {
                    const long long row = g - P.cl_begin;
                    if (row < 0 || row >= rows) return fail(DMDGPU_ERR_MISMATCH, "i-cluster row out of range");
                    for (int l = 0; l < 32; ++l) {
                        const uint32_t m = cm[32 * row + l];
                        if (!m) continue;
                        const int js = static_cast<int>(cj[32 * row + l] & 0x03FFFFFFu);
                        const int aj = aos[js - s0] - a0;
                        for (int i = 0; i < 8; ++i)
                            if ((m >> i) & 1u) {
                                const int ai = aos[32 * (P.tile_begin + t) + 8 * k + i - s0] - a0;
                                cp.emplace_back(std::min(ai, aj), std::max(ai, aj));
                            }
                    }
                }
            }
        std::sort(cp.begin(), cp.end());
        if (cp != pairs) return fail(DMDGPU_ERR_MISMATCH, "i-cluster rows differ from the chunk list");
    }
    *count = static_cast<long long>(pairs.size());
    for (long long p = 0; p < std::min<long long>(cap, *count); ++p) {
        pi[p] = pairs[p].first;
        pj[p] = pairs[p].second;
    }
    return DMDGPU_OK;
}

// ---------------------------------------------------------------------------
// Checkpoints: v1 layout of src/sim/checkpoint.cpp:9-38 plus a trailer.
// ---------------------------------------------------------------------------
namespace {
constexpr uint32_t CK_MAGIC = 0x444D4450;   // checkpoint.cpp:6
constexpr uint32_t CK_VERSION = 1;           // checkpoint.cpp:7
constexpr uint32_t TR_MAGIC = 0x32474D44;    // trailer tag
}  // namespace

int Batch::save_checkpoint(int slot, const char* path) {
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    const HostRep& h = *reps_[slot];
    const int n = h.sys.n;
    std::vector<double> px(n), py(n), pz(n), vx(n), vy(n), vz(n), fx(n), fy(n), fz(n);
    int rc = get_state(slot, 0, px.data(), py.data(), pz.data());
    if (!rc) rc = get_state(slot, 1, vx.data(), vy.data(), vz.data());
    if (!rc) rc = get_state(slot, 2, fx.data(), fy.data(), fz.data());
    if (rc) return rc;
    dmdgpu_scalars sc;
    rc = get_scalars(slot, &sc);
    if (rc) return rc;
    std::ofstream os(path, std::ios::binary);
    if (!os) return fail(DMDGPU_ERR_PARM, std::string("cannot open ") + path);
    uint64_t nn = static_cast<uint64_t>(n);
    uint64_t stp = static_cast<uint64_t>(sc.step);
    double tm = sc.time, pe = sc.potential_energy;
    os.write(reinterpret_cast<const char*>(&CK_MAGIC), 4);
    os.write(reinterpret_cast<const char*>(&CK_VERSION), 4);
    os.write(reinterpret_cast<const char*>(&nn), 8);
    os.write(reinterpret_cast<const char*>(&stp), 8);
    os.write(reinterpret_cast<const char*>(&tm), 8);
    os.write(reinterpret_cast<const char*>(&pe), 8);
    for (auto* v : {&px, &py, &pz, &vx, &vy, &vz, &fx, &fy, &fz})
        os.write(reinterpret_cast<const char*>(v->data()), 8 * n);
    os.write(reinterpret_cast<const char*>(h.sys.mass.data()), 8 * n);
    os.write(reinterpret_cast<const char*>(h.sys.q.data()), 8 * n);
    os.write(reinterpret_cast<const char*>(h.sys.type.data()), 4 * n);
    int32_t ljc = sc.lj_step_since_rebuild;
    os.write(reinterpret_cast<const char*>(&ljc), 4);
    // trailer: box, Nose-Hoover zeta, Andersen call counter, profile, (v3) the
    // PHYS barostat scale still to be applied with the next drift, (v4) the
    // frame of the last list build (box edge, build count, positions) and the
    // pending-rebuild flag, so a restart rebuilds the very same list, (v5) the
    // Andersen barostat's piston velocity
    uint32_t tv = 5;
    double box = sc.box, zeta = sc.zeta;
    int k = replica_index(slot);
    int64_t acalls = h_st_[k].andersen_calls;
    int32_t prof = phys_ ? 1 : 0;
    uint32_t aseed = h.andersen_seed;
    os.write(reinterpret_cast<const char*>(&TR_MAGIC), 4);
    os.write(reinterpret_cast<const char*>(&tv), 4);
    os.write(reinterpret_cast<const char*>(&box), 8);
    os.write(reinterpret_cast<const char*>(&zeta), 8);
    os.write(reinterpret_cast<const char*>(&acalls), 8);
    os.write(reinterpret_cast<const char*>(&aseed), 4);
    os.write(reinterpret_cast<const char*>(&prof), 4);
    double pscale = phys_ ? h_st_[k].pscale : 1.0;
    os.write(reinterpret_cast<const char*>(&pscale), 8);
    {
        const RepState& st = h_st_[k];
        const double lb = st.L_build;
        const int64_t nb = st.list_builds;
        const int32_t pending = st.rebuild;
        os.write(reinterpret_cast<const char*>(&lb), 8);
        os.write(reinterpret_cast<const char*>(&nb), 8);
        os.write(reinterpret_cast<const char*>(&pending), 4);
        std::vector<double> f(n);
        const int a0 = h.rep.atom_begin;
        for (double* src : {dev_.xr, dev_.yr, dev_.zr}) {
            CK(cudaMemcpy(f.data(), src + a0, 8 * n, cudaMemcpyDeviceToHost));
            os.write(reinterpret_cast<const char*>(f.data()), 8 * n);
        }
        const double ed = st.eps_dot;
        os.write(reinterpret_cast<const char*>(&ed), 8);
    }
    return os.good() ? DMDGPU_OK : fail(DMDGPU_ERR_PARM, "checkpoint write failed");
}

int Batch::load_checkpoint(int slot, const char* path) {
    st_fresh_ = false;  // device work follows: the host mirror is stale
    CK(cudaSetDevice(device_));
    if (!has(slot)) return fail(DMDGPU_ERR_INVALID, "no such slot");
    if (!packed_) {
        int rc = pack();
        if (rc) return rc;
    }
    std::ifstream is(path, std::ios::binary);
    if (!is) return fail(DMDGPU_ERR_PARM, std::string("cannot open ") + path);
    HostRep& h = *reps_[slot];
    const int n = h.sys.n;
    uint32_t magic = 0, version = 0;
    uint64_t nn = 0, stp = 0;
    double tm = 0, pe = 0;
    is.read(reinterpret_cast<char*>(&magic), 4);
    is.read(reinterpret_cast<char*>(&version), 4);
    // the reference writes both words and never reads them back
    // (src/sim/checkpoint.cpp:40-47); a file with other values is refused here
    if (!is || magic != CK_MAGIC) return fail(DMDGPU_ERR_MISMATCH, "not a DMD checkpoint (bad magic)");
    if (version != CK_VERSION) return fail(DMDGPU_ERR_MISMATCH, "unsupported checkpoint version");
    is.read(reinterpret_cast<char*>(&nn), 8);
    if (!is || nn != static_cast<uint64_t>(n))
        return fail(DMDGPU_ERR_MISMATCH, "checkpoint atom count differs from the system");
    is.read(reinterpret_cast<char*>(&stp), 8);
    is.read(reinterpret_cast<char*>(&tm), 8);
    is.read(reinterpret_cast<char*>(&pe), 8);
    std::vector<double> v[11];
    for (int i = 0; i < 11; ++i) {
        v[i].resize(n);
        is.read(reinterpret_cast<char*>(v[i].data()), 8 * n);
    }
    std::vector<int> types(n);
    is.read(reinterpret_cast<char*>(types.data()), 4 * n);
    int32_t ljc = 0;
    is.read(reinterpret_cast<char*>(&ljc), 4);
    if (!is) return fail(DMDGPU_ERR_MISMATCH, "truncated checkpoint");
    uint32_t tmagic = 0, tv = 0;
    double box = 0, zeta = 0;
    int64_t acalls = 0;
    uint32_t aseed = 42;
    int32_t prof = -1;
    double pscale = 1.0;
    bool trailer = false;
    if (is.read(reinterpret_cast<char*>(&tmagic), 4) && tmagic == TR_MAGIC) {
        is.read(reinterpret_cast<char*>(&tv), 4);
        is.read(reinterpret_cast<char*>(&box), 8);
        is.read(reinterpret_cast<char*>(&zeta), 8);
        is.read(reinterpret_cast<char*>(&acalls), 8);
        is.read(reinterpret_cast<char*>(&aseed), 4);
        is.read(reinterpret_cast<char*>(&prof), 4);
        trailer = static_cast<bool>(is);
        if (trailer && (tv < 1 || tv > 5)) return fail(DMDGPU_ERR_MISMATCH, "unsupported checkpoint trailer version");
        if (trailer && tv >= 3 && !is.read(reinterpret_cast<char*>(&pscale), 8)) pscale = 1.0;
    }
    // v4: the frame of the last list build
    bool framed = false;
    double lbuild = 0.0;
    int64_t nbuilds = 0;
    int32_t pending = 0;
    std::vector<double> fr[3];
    if (trailer && tv >= 4) {
        is.read(reinterpret_cast<char*>(&lbuild), 8);
        is.read(reinterpret_cast<char*>(&nbuilds), 8);
        is.read(reinterpret_cast<char*>(&pending), 4);
        for (auto& f : fr) {
            f.resize(n);
            is.read(reinterpret_cast<char*>(f.data()), 8 * n);
        }
        framed = static_cast<bool>(is) && lbuild > 0.0;
    }
    double eps_dot = 0.0;  // v5
    if (trailer && tv >= 5 && !is.read(reinterpret_cast<char*>(&eps_dot), 8)) eps_dot = 0.0;
    const int k = replica_index(slot);
    const int a0 = h.rep.atom_begin;
    CK(cudaStreamSynchronize(stream_));
    double* dst[6] = {dev_.x, dev_.y, dev_.z, dev_.vx, dev_.vy, dev_.vz};
    for (int i = 0; i < 6; ++i) CK(cudaMemcpy(dst[i] + a0, v[i].data(), 8 * n, cudaMemcpyHostToDevice));
    // SystemData masses are restored (checkpoint.cpp:66); the components keep the
    // charges / types they were built with.
    h.sys.mass = v[9];
    CK(cudaMemcpy(const_cast<double*>(dev_.mass) + a0, v[9].data(), 8 * n, cudaMemcpyHostToDevice));
    RepState st;
    CK(cudaMemcpy(&st, d_st_ + k, sizeof(RepState), cudaMemcpyDeviceToHost));
    st.step = static_cast<long long>(stp);
    st.time = tm;
    st.lj_counter = ljc;
    st.rebuild = 1;
    st.have_forces = 0;
    st.vscale = 1.0;
    st.target_step = st.step;
    if (trailer) {
        st.L = box;
        st.invL = 1.0 / box;
        st.zeta = zeta;
        st.andersen_calls = acalls;
        h.andersen_seed = aseed;
        st.pscale = phys_ ? pscale : 1.0;
        st.eps_dot = eps_dot;
    }
    if (framed) {
        // the saved list frame: the list is rebuilt as it was, not at the loaded positions
        st.L_build = lbuild;
        st.list_builds = nbuilds;
        st.rebuild = pending;
        double* fdst[3] = {dev_.xr, dev_.yr, dev_.zr};
        for (int i = 0; i < 3; ++i) CK(cudaMemcpy(fdst[i] + a0, fr[i].data(), 8 * n, cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(d_st_ + k, &st, sizeof(RepState), cudaMemcpyHostToDevice));
    if (framed) {
        std::vector<char> sel(order_.size(), 0);
        sel[k] = 1;
        int rc = rebuild_in_frame(sel);
        if (rc) return rc;
    }
    h.target = st.step;
    h.done = false;
    graph_dirty_ = true;  // the next step must evaluate forces first
    return DMDGPU_OK;
}

}  // namespace dmd
