// layout.h -- device data layout shared by the kernels and the host engine.
//
// A "batch" packs R independent systems (replicas) into one set of device
// arrays.  Replica r owns
//   atoms  [atom_begin, atom_begin + n_atoms)          reference atom order, FP64 state
//   tiles  [tile_begin, tile_begin + n_tiles)          32 sorted slots per tile
//   slots  [32*tile_begin, 32*(tile_begin + n_tiles))  spatially sorted mirror
//   bins   [bin_begin, bin_begin + nvx^2 nvz)          snake-ranked sort cells
//   chunks [chunk_begin, chunk_begin + chunk_cap)      pair list segment
//   mesh   PME buffers at per-replica offsets
// A single system is a batch of one.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dmd {

constexpr double KB = 0.008314462618;   // kJ mol^-1 K^-1 (src/core/constants.h:6)
constexpr double KE = 138.935456;       // kJ mol^-1 nm e^-2 (coulomb_pme.h:45)
constexpr double PI = 3.14159265358979323846;
constexpr double BAR = 0.0602214086;    // kJ mol^-1 nm^-3 per bar

// Fixed-point scales (int64 two's complement accumulators).
constexpr double FSCALE = 4294967296.0;        // 2^32 per kJ mol^-1 nm^-1 (forces)
constexpr double ESCALE = 4294967296.0;        // 2^32 per kJ mol^-1 (energies, virial)
constexpr double MSCALE = 1099511627776.0;     // 2^40 per e (PME mesh charge)
constexpr double FMAX = 1.0e9;                 // |F| above this -> BondExplosion status

enum RepFlags : int {
    F_LJ = 1,          // Lennard-Jones component present
    F_COUL_REAL = 2,   // real-space Ewald on the shared list (phys)
    F_PME = 4,         // SPME reciprocal part
    F_EXCL = 8,        // exclusion correction component
    F_PHYS = 16,       // gradient-consistent profile
    F_BONDED = 32,
};

enum Status : int {
    ST_NAN = 1, ST_RANGE = 2, ST_CAPACITY = 4, ST_LIST = 8, ST_TIMEOUT = 16,
};

enum ETerm : int { E_LJ = 0, E_CREAL = 1, E_CRECIP = 2, E_CSELF = 3, E_CEXCL = 4, E_BOND = 5,
                   E_ANGLE = 6, E_DIH = 7, E_IMP = 8, E_VIR = 9, N_EACC = 10 };

// Per-replica constants.
struct Rep {
    int atom_begin, n_atoms, tile_begin, n_tiles;
    int bin_begin, nvx, nvz;            // sort grid: nvx x nvx columns, nvz slabs
    int chunk_begin, chunk_cap;
    int cl_begin, cl_cap;               // 8-atom i-cluster lists (mixed precision)
    int n_types, lj_off;
    int flags, profile;
    int thermostat, barostat;
    int pme_K;
    long long mesh_fix_off, mesh_fix_n;  // int64 spread buffer (REF: K*K*2(K/2+1), PHYS: K^3)
    long long mesh_real_off;             // K^3 reals
    long long mesh_cplx_off;             // K*K*(K/2+1) complex
    int bsp_off;                         // K doubles: B-spline factor per mesh index
    int pme_block_begin, pme_blocks;     // influence-kernel blocks
    int conv_block_begin, conv_blocks;   // convert-kernel blocks (1,024 mesh points each)
    double rc_lj, rc_c, rc_list;
    double rc_lj2, rc_c2, rc_list2, half_skin2;
    double alpha;
    double dt;
    double t_temp, t_tau, t_freq, nh_Q;
    double b_pressure, b_tau, b_compress;
    double piston_W;                     // Andersen barostat piston mass
    double cons_tol;                     // constraint tolerance (SHAKE on r^2 - d^2, RATTLE on r.v)
    double e_self;
    uint32_t key0, key1;                 // Andersen (phys) Philox key
};

// FP32 LJ coefficients of one type pair, (c6, c12, 6 c6, 12 c12) with
// c6 = 4 eps sig^6 and c12 = 4 eps sig^12, each rounded once from FP64.
inline float4 lj_coeffs32(double eps, double sig6) {
    const double c6 = 4.0 * eps * sig6, c12 = 4.0 * eps * sig6 * sig6;
    return make_float4(static_cast<float>(c6), static_cast<float>(c12), static_cast<float>(6.0 * c6),
                       static_cast<float>(12.0 * c12));
}

// Per-replica mutable state.
struct RepState {
    double L, invL;
    double zeta;
    double vscale;        // pending thermostat velocity scale (applied in the next kick)
    double pscale;        // pending barostat position scale
    double eps_dot;       // Andersen barostat piston velocity (strain rate)
    double ke, pressure, virial;
    double e_recip, vir_recip;
    double time;
    long long e_acc[N_EACC];
    long long step, target_step;
    long long andersen_calls;
    long long list_builds;
    int active;           // advances this step
    int eval;             // forces evaluated in the current evaluation pass
    int rebuild;          // neighbour list rebuild requested
    int lj_counter;       // LennardJones::step_since_rebuild_ (REF cadence)
    int have_forces;
    int status;
    int n_chunks;
    int n_cl;             // i-cluster list rows in use
    int want_e;           // the current evaluation's pair energies / virial are read
    int green_ok;         // the cached PME influence function matches the box
    double green_L;       // box edge the cached influence function was made for
    double L_build;       // box edge at the last list build (with xr/yr/zr: the list's frame)
};

// Kernel view of the whole batch (passed by value).
struct Dev {
    int n_rep, n_atoms, n_tiles, n_slots, n_bins;
    const Rep* rep;
    RepState* st;
    // atoms (reference order)
    double *x, *y, *z, *vx, *vy, *vz;
    const double *mass, *q;
    const int *type, *atom_rep;
    long long *fbx, *fby, *fbz;        // bonded + PME + exclusion forces (fixed point)
    int* slot_of_atom;
    double *xr, *yr, *zr;              // positions at the last list build
    int *imgx, *imgy, *imgz;           // periodic image frozen at the last build
    int* atom_bin;
    // sorted slots
    int* atom_of_slot;
    float4* xq32;                      // tile-local FP32 coordinates + charge
    float4* xl32;                      // the same at the last list build (aliases xq32 when mixed)
    double4* xq64;                     // unwrapped FP64 coordinates + charge
    int* type_s;
    long long *fnx, *fny, *fnz;        // non-bonded forces (fixed point, slot order)
    // tiles
    double *tcx, *tcy, *tcz;
    float *thx, *thy, *thz;
    const int* tile_rep;
    double *tile_ke, *tile_vir;
    // voxel bins
    int *bin_count, *bin_start, *bin_fill;
    const int* vox_rank;
    int* sort_buf;                     // slot-indexed scratch for the counting sort
    // exclusions
    const int *ex_start, *ex_list;     // CSR per atom (global indices)
    int n_excl;
    const int2* excl;
    // pair list
    int* chunk_itile;
    uint32_t *chunk_j, *chunk_mask;
    int* chunk_prefix;                 // [n_rep + 1] flat chunk numbering
    // The same pair list regrouped by 8-atom i-cluster (a quarter of an
    // i-tile: slots 32 I + 8 k .. + 7, cluster index 4 I + k).  A row holds 32
    // j entries (the chunk entry words) and one 8-bit mask per entry over the
    // cluster's atoms; a cluster's rows are contiguous, the entries in the
    // order of its tile's chunks sorted by their first entry word.  Built after
    // every list build when the arrays exist (mixed precision), not otherwise.
    int* tile_nch;                     // [n_tiles] chunks of each i-tile
    int* tile_c0;                      // [n_tiles] first position of its chunk ids in chunk_order
    int* tile_fill;                    // [n_tiles] scatter counter
    int* chunk_order;                  // chunk ids grouped by i-tile (chunk capacity)
    int* chunk_sorted;                 // the same, each tile's ids in canonical order
    uint32_t* cl_j;                    // [rows][32] entry words
    uint8_t* cl_m;                     // [rows][32] masks (bit k: cluster atom k)
    int2* cl_job;                      // [4 n_tiles] per cluster: first row, row count
    void* pme_green;                   // cached PME influence function (mesh_cplx layout, T)
    int* nb_work;                      // pair-kernel chunk counter (reset per evaluation)
    int* nb_work_mi;                   // the same for the narrow-box pair kernel
    int mi_split;                      // narrow-box replicas go to their own pair kernel
    int any_coul;                      // some replica has real-space Coulomb (F_COUL_REAL)
    int* build_work;                   // list-build i-tile counter (reset per rebuild)
    int* build_prefix;                 // [3][n_rep + 1] prefixes of the rebuilding replicas'
                                       // atoms, sort cells and tiles
    unsigned* grid_bar;                // [2] rebuild grid barrier: arrivals, generation
    unsigned long long bar_limit_ns;   // a barrier wait gives up after this long (0: one second)
    unsigned bar_extra;                // arrivals a barrier needs beyond the grid's blocks (0;
                                       // only the failure-path test hook sets it)
    // bonded terms (global atom indices)
    int n_bonds, n_angles, n_dih, n_imp;
    const int2* bond_ij;
    const double2* bond_kr;
    const int4* ang_ijk;
    const double2* ang_kt;
    const int4* dih_ijkl;
    const int* dih_n;
    const double2* dih_kp;
    const int4* imp_ijkl;
    const double2* imp_kp;             // (k, chi0)
    // distance constraints, grouped by connected atom set (a molecule), each
    // group's constraints in their sweep order (global atom indices)
    int n_cgroups;
    const int* cgroup_begin;           // [n_cgroups + 1] into cons_ij / cons_d
    const int* cgroup_rep;
    const int2* cons_ij;
    const double* cons_d;              // target distance
    const int* cgroup_atom_begin;      // [n_cgroups + 1] into cgroup_atoms
    const int* cgroup_atoms;           // each group's distinct atoms
    double* cons_x0;                   // [3][n_atoms] positions before SHAKE (PHYS)
    // LJ tables per type pair
    const double2* lj64;               // (eps, sig^6)
    const float4* lj32;                // (c6, c12, 6 c6, 12 c12), c6 = 4 eps sig^6, c12 = 4 eps sig^12
    int n_lj;                          // entries of the LJ tables (all replicas)
    // PME
    long long* mesh_fix;
    void* mesh_real;
    void* mesh_cplx;
    const double* bsp;
    double* pme_part;                  // per influence block: energy, virial
    const int* pme_block_rep;
    const int* conv_block_rep;         // replica of each convert-kernel block
    // Andersen (REF): host-generated overrides
    const int* and_flag;
    const double* and_v;
};

}  // namespace dmd
