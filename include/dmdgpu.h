/*
 * dmdgpu.h -- C ABI of the B200 (sm_100a) implementation of DMD's per-step
 * force-and-integrate path.
 *
 * Plain C: POD descriptors, plain pointers and sizes, int status codes, no
 * exceptions and no torch types across the boundary.  Every array passed in
 * is owned by the caller and copied during the call.  A context owns its
 * device memory, CUDA stream, cuFFT plans and CUDA graphs.  Calls on one
 * context are not re-entrant; distinct contexts are independent.
 *
 * Units are the reference's: nm, ps, amu, kJ/mol, e, K; k_B = 0.008314462618
 * kJ mol^-1 K^-1, k_e = 138.935456 kJ mol^-1 nm e^-2.
 */
#ifndef DMDGPU_H
#define DMDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..5 mirror ForceError (src/core/error.h:6-12); a non-zero
 * status leaves a message in dmdgpu_last_error(). */
enum {
    DMDGPU_OK = 0,
    DMDGPU_ERR_NAN = 1,            /* ForceError::NaN: non-finite force/energy seen on device */
    DMDGPU_ERR_BOND_EXPLOSION = 2, /* ForceError::BondExplosion: fixed-point force range exceeded */
    DMDGPU_ERR_MISMATCH = 3,       /* ForceError::Mismatch: array sizes / checkpoint disagree */
    DMDGPU_ERR_PARM = 4,           /* ForceError::ParmError: invalid parameter */
    DMDGPU_ERR_GPU = 5,            /* ForceError::GPUError: CUDA / cuFFT failure */
    DMDGPU_ERR_OOM = 6,            /* device allocation failed */
    DMDGPU_ERR_BUDGET = 7,         /* batch admission: HBM budget or slot table full */
    DMDGPU_ERR_INVALID = 8,        /* bad handle / call order */
    DMDGPU_ERR_CAPACITY = 9        /* neighbour-list capacity exceeded on device */
};

/* coulomb_type (SimulationConfig::coulomb_type, src/sim/simulation_config.h:62) */
enum { DMDGPU_COULOMB_CUTOFF = 0, /* "cutoff" / "direct" */ DMDGPU_COULOMB_PME = 1 };
/* ThermostatConfig::type (src/sim/simulation_config.h:11-16) */
enum { DMDGPU_THERMO_NONE = 0, DMDGPU_THERMO_BERENDSEN = 1, DMDGPU_THERMO_NOSE_HOOVER = 2,
       DMDGPU_THERMO_ANDERSEN = 3 };
/* BarostatConfig::type (src/sim/simulation_config.h:18-23); "andersen"
 * (src/barostat/andersen_barostat.cpp:8-45) runs in the REF profile only.
 * Constraints (constraint_type 1, src/integrate/constraints.cpp:9-91): SHAKE
 * after the drift, RATTLE after the second half kick (PHYS also gives SHAKE's
 * displacement to the half-step velocities); not with the Andersen thermostat. */
enum { DMDGPU_BARO_NONE = 0, DMDGPU_BARO_BERENDSEN = 1, DMDGPU_BARO_ANDERSEN = 2 };
/* Semantic profile: REF reproduces the reference's formulas (quirks included);
 * PHYS uses gradient-consistent forces (skin list, erfc real space with
 * exclusions, textbook SPME, analytic bonded gradients, atomic virial). */
enum { DMDGPU_PROFILE_REF = 0, DMDGPU_PROFILE_PHYS = 1 };
/* MIXED: FP32 pair/mesh/bonded arithmetic, int64 fixed-point force accumulation,
 * FP64 integration and reductions.  FP64: every stage in FP64. */
enum { DMDGPU_PRECISION_MIXED = 0, DMDGPU_PRECISION_FP64 = 1 };

/*
 * System + run description.  Mirrors SimulationConfig
 * (src/sim/simulation_config.h:27-84) as filled by SystemBuilder/apply_config
 * (python/dmd/system.py, python/dmd/config.py): a cubic box, per-atom SoA
 * arrays, one bond / angle / dihedral / improper term set each.  vel_* may be NULL (zero
 * velocities); atom_types may be NULL (all type 0).
 */
typedef struct dmdgpu_system {
    int32_t n_atoms;
    double box_size;
    const double *masses, *charges;
    const double *pos_x, *pos_y, *pos_z;
    const double *vel_x, *vel_y, *vel_z;
    const int32_t *atom_types;
    /* Lennard-Jones: n_types x n_types row-major sigma / epsilon */
    int32_t use_lj, lj_n_types;
    const double *lj_sigma, *lj_epsilon;
    double lj_cutoff;
    /* bonded terms */
    int32_t n_bonds;
    const int32_t *bond_i, *bond_j;
    const double *bond_k, *bond_r0;
    int32_t n_angles;
    const int32_t *angle_i, *angle_j, *angle_k;
    const double *angle_k_theta, *angle_theta0;
    int32_t n_dihedrals;
    const int32_t *dihedral_i, *dihedral_j, *dihedral_k, *dihedral_l, *dihedral_periodicity;
    const double *dihedral_k_phi, *dihedral_phi0;
    /* HarmonicImproper (src/force/harmonic_improper.cpp:10-130): E = k/2 (chi - chi0)^2 */
    int32_t n_impropers;
    const int32_t *improper_i, *improper_j, *improper_k, *improper_l;
    const double *improper_k_phi, *improper_phi0;
    /* electrostatics */
    int32_t coulomb_type;
    double coulomb_cutoff, ewald_coeff, pme_grid_spacing;
    int32_t pme_order;
    /* exclusions (1-2, 1-3, 1-4 pairs) */
    int32_t n_excl;
    const int32_t *excl_i, *excl_j;
    /* run control */
    double dt;
    int32_t n_steps, gen_vel, seed;
    double init_temperature;
    int32_t thermostat_type;
    double thermo_temperature, thermo_tau, thermo_frequency;
    int32_t barostat_type;
    double baro_pressure, baro_tau, baro_compressibility;
    int32_t constraint_type; /* 0 "none", 1 "shake" (SHAKE + RATTLE) */
    int32_t checkpoint_interval;
    const char *checkpoint_path; /* may be NULL */
    /* distance constraints (ConstraintsParams, src/integrate/constraints.h:8-12),
     * used when constraint_type is 1 */
    int32_t n_constraints;
    const int32_t *constraint_i, *constraint_j;
    const double *constraint_dist;
    double constraint_tolerance;
} dmdgpu_system;

typedef struct dmdgpu_options {
    int32_t profile;    /* DMDGPU_PROFILE_* */
    int32_t precision;  /* DMDGPU_PRECISION_* */
    double skin;        /* Verlet skin (nm), PHYS only; REF uses the reference's no-skin list */
    int32_t device;     /* CUDA device ordinal */
    uint64_t rng_seed;  /* PHYS Andersen thermostat stream key */
    int32_t nb_form;    /* mixed-precision pair-kernel form: DMDGPU_NB_* (results do not
                           depend on it beyond FP32 summation order) */
} dmdgpu_options;

#define DMDGPU_NB_AUTO 0      /* the default form (32 x 32 chunks); the autotuner picks only
                                 its launch shape, which changes no result bit */
#define DMDGPU_NB_CHUNK32 1   /* one warp per 32 x 32 (i-tile, j entries) chunk */
#define DMDGPU_NB_CLUSTER8 2  /* one warp per 8-atom i-cluster over its 32-entry rows */

/* Scalars of the last force evaluation / current state. */
typedef struct dmdgpu_scalars {
    int64_t step;
    double time;
    double potential_energy; /* SystemData::potential_energy after the last evaluation */
    double box;
    double kinetic_energy, temperature, pressure, virial;
    double zeta;             /* Nose-Hoover friction */
    /* energy terms: lj, coul_real, coul_recip, coul_self, coul_excl, bond, angle, dihedral,
     * improper */
    double e_terms[9];
    int64_t list_builds;
    int32_t lj_step_since_rebuild; /* LennardJones::step_since_rebuild (REF cadence) */
    int32_t status;
    int64_t list_chunks;           /* 32-entry pair-list chunks of the current list */
} dmdgpu_scalars;

typedef struct dmdgpu_ctx dmdgpu_ctx;

/* Replaces build_simulation (src/sim/simulation_engine.cpp:248-386) +
 * EngineWrapper::EngineWrapper (python/dmd/core.cpp:21-25).  Velocities are
 * generated as the reference does when gen_vel != 0 (std::mt19937(seed),
 * std::normal_distribution, COM removal, rescale; simulation_engine.cpp:339-383). */
int dmdgpu_create(const dmdgpu_system *sys, const dmdgpu_options *opt, dmdgpu_ctx **out);

/* Replaces SimulationEngine::step x n (src/sim/simulation_engine.cpp:53-86) and
 * EngineWrapper::run_n (python/dmd/core.cpp:29-44): n steps on the device, one call. */
int dmdgpu_step(dmdgpu_ctx *ctx, int32_t n_steps);

/* Replaces SimulationEngine::run (simulation_engine.cpp:88-106): n_steps steps with
 * a checkpoint every checkpoint_interval steps (when a path is set). */
int dmdgpu_run(dmdgpu_ctx *ctx);

/* State copies in the reference's atom order.  which: 0 positions, 1 velocities,
 * 2 forces (of the last evaluation).  Replaces the EngineWrapper getters
 * positions / velocities / forces (python/dmd/core.cpp:49-90). */
int dmdgpu_get_state(dmdgpu_ctx *ctx, int32_t which, double *x, double *y, double *z);
/* Overwrite positions (which=0) or velocities (which=1). */
int dmdgpu_set_state(dmdgpu_ctx *ctx, int32_t which, const double *x, const double *y,
                     const double *z);
int dmdgpu_get_scalars(dmdgpu_ctx *ctx, dmdgpu_scalars *out);

/* Single-point evaluation of every component at the current positions
 * (ForceEngine::compute, src/force/force_engine.cpp:10-25) with a freshly built
 * list.  Forces are written (not accumulated); e_terms receives 9 doubles
 * (see dmdgpu_scalars.e_terms) and may be NULL. */
int dmdgpu_compute_forces(dmdgpu_ctx *ctx, double *fx, double *fy, double *fz, double *e_terms);

/* One force component at caller positions, accumulated into caller arrays --
 * the ForceComponent::compute contract (src/force/force_component.h:12-21):
 * forces are added (never zeroed) and the energy is added to *energy.
 * component: 0 LennardJones, 1 HarmonicBond, 2 HarmonicAngle, 3 PeriodicDihedral,
 * 4 CoulombDirect (real-space Ewald), 5 CoulombPME (reciprocal + self),
 * 6 CoulombExclusion, 7 HarmonicImproper.  The context's own positions are left
 * unchanged. */
int dmdgpu_component_compute(dmdgpu_ctx *ctx, int32_t component, const double *pos_x,
                             const double *pos_y, const double *pos_z, double box,
                             double *forces_x, double *forces_y, double *forces_z,
                             double *energy);

/* The current short-range pair list as sorted (i<j) atom pairs: REF = the
 * LennardJones list (pairs within lj_cutoff at the last rebuild,
 * lennard_jones.cpp:18-41); PHYS = pairs within max cutoff + skin, exclusions
 * removed.  Copies min(count, cap) pairs; *count receives the total. */
int dmdgpu_pair_list(dmdgpu_ctx *ctx, int32_t *pi, int32_t *pj, int64_t cap, int64_t *count);

/* Binary checkpoint v1 (src/sim/checkpoint.cpp:9-75) plus a trailer the v1
 * reader ignores (box, Nose-Hoover zeta, thermostat call counter, profile, the
 * pending PHYS barostat scale, the frame of the last pair-list build: its
 * box edge and positions, and the Andersen barostat's piston velocity).  A restart rebuilds the list in that frame, so N
 * steps equal N/2 + save/load + N/2 bit for bit in both profiles and both
 * precisions.  Replaces SimulationEngine::save_checkpoint / load_checkpoint
 * (:108-137). */
int dmdgpu_save_checkpoint(dmdgpu_ctx *ctx, const char *path);
int dmdgpu_load_checkpoint(dmdgpu_ctx *ctx, const char *path);

/* Device bytes a context for this system would hold (admission accounting). */
int64_t dmdgpu_footprint_bytes(const dmdgpu_system *sys, const dmdgpu_options *opt);

/* Rebuild this context's device table with its state carried over bit for bit:
 * the pair list is rebuilt in the frame of its last build and forces are
 * evaluated again at the current positions before the next step.  This is what
 * a running slot of a batch goes through when another slot is admitted or
 * released; the trajectory continues bit for bit, so a batched job equals the
 * same job run alone.  No counterpart in the reference. */
int dmdgpu_repack(dmdgpu_ctx *ctx);

/* Kernel launches issued by this context so far (this library's own kernels). */
int64_t dmdgpu_kernel_launches(dmdgpu_ctx *ctx);

/* The CUDA stream (cudaStream_t) every launch of this context is issued on, so a
 * caller can order its own work or record timing events on it. */
void *dmdgpu_stream(dmdgpu_ctx *ctx);

/* The launch configuration the current device table runs with: the knobs the
 * autotuner chose (or took from its cache) and the forms the options and the
 * systems select.  Valid after the first step (the table is built then). */
typedef struct dmdgpu_launch_info {
    int32_t packed;            /* 1: a device table exists (the fields below describe it) */
    int32_t nb_form;           /* DMDGPU_NB_CHUNK32 or DMDGPU_NB_CLUSTER8 (FP64: CHUNK32) */
    int32_t nb_blocks_per_sm;  /* persistent pair-kernel blocks per SM */
    int32_t tuned;             /* 1: blocks per SM measured (now or cached) for this kind
                                  of table; 0: the untuned default */
    int32_t min_image_kernel;  /* 1: boxes narrower than twice the list cutoff (or under
                                  a barostat) also run the minimum-image pair kernel */
    int32_t n_replicas;
    int64_t n_atoms;
    int64_t launches_per_step; /* kernels in one captured step */
} dmdgpu_launch_info;

int dmdgpu_get_launch_info(dmdgpu_ctx *ctx, dmdgpu_launch_info *out);

/* Device timing of a run of steps. */
typedef struct dmdgpu_timing {
    double step_ms;            /* summed device time of the n steps (flushes excluded) */
    double nonbonded_ms;       /* summed device time of the non-bonded pair-kernel launches of
                                  the sampled steps (every eighth step, and the last of a short run) */
    double pme_ms;             /* summed device time of the sampled steps' PME chains (spread .. gather) */
    int64_t nonbonded_launches; /* pair-kernel launches of the sampled steps */
    int64_t kernel_launches;   /* this library's kernels executed during the n steps */
    int64_t sampled_steps;     /* steps whose pair-kernel and PME launches were timed */
} dmdgpu_timing;

/* dmdgpu_step with device timing: the step graph (the one dmdgpu_step launches,
 * with event records around every non-bonded launch and every PME chain) is
 * launched n times, each launch between two events on the context's stream.
 * When l2_flush_bytes > 0 a buffer of that size is overwritten between steps
 * (outside the timed intervals) so each step starts with a cold L2.  Not
 * available for a REF Andersen thermostat (its random stream is drawn on the
 * host every step). */
int dmdgpu_step_timed(dmdgpu_ctx *ctx, int32_t n_steps, int64_t l2_flush_bytes, dmdgpu_timing *out);

/* Trajectory frames, exported while the run continues.  Replaces the frame
 * writing inside the reference's run loop (EngineWrapper::run_n,
 * python/dmd/core.cpp:29-44, and SimulationEngine::run,
 * src/sim/simulation_engine.cpp:88-104): after every step whose step counter
 * is a multiple of `interval`, the step, time, box and the positions and
 * velocities of that step (what H5MDWriter::write_frame,
 * src/trajectory/h5md_writer.cpp:191, records) are copied on the device into
 * one of a few staging buffers, then to pinned host memory on a copy stream
 * while the next steps compute, and `fn` is called with them in step order.
 * The run waits for the writer only when it falls DMDGPU_FRAME_SLOTS frames
 * behind.
 *
 * `fn` runs on a CUDA host-callback thread: it must not call CUDA or any
 * dmdgpu_ function, and the arrays it receives are valid only during the
 * call (copy what you keep).  dmdgpu_step / dmdgpu_run return without
 * waiting for frames still in flight; dmdgpu_flush_frames waits for them (so
 * does dmdgpu_destroy).  interval <= 0 or fn == NULL turns export off.
 * Exporting changes no bit of the trajectory.  No counterpart in the
 * reference for the callback itself: the reference writes HDF5 inline. */
#define DMDGPU_FRAME_SLOTS 4
typedef struct dmdgpu_frame {
    int64_t step;
    double time;                 /* ps */
    double box;                  /* cubic box edge (nm) */
    int32_t n_atoms;
    const double *x, *y, *z;     /* positions (nm), unwrapped as the engine keeps them */
    const double *vx, *vy, *vz;  /* velocities (nm/ps) */
} dmdgpu_frame;
typedef void (*dmdgpu_frame_fn)(const dmdgpu_frame *frame, void *user);
int dmdgpu_set_frame_writer(dmdgpu_ctx *ctx, int32_t interval, dmdgpu_frame_fn fn, void *user);
int dmdgpu_flush_frames(dmdgpu_ctx *ctx);

/* Test-only fault injection, done on the host; no counterpart in the reference.
 * It changes only what the next list build is given, so the failure paths can
 * be exercised without faulting, trapping or hanging the GPU:
 *   DMDGPU_INJECT_BARRIER_TIMEOUT  the next build's grid barrier can never be
 *     completed and each bounded wait gives up after 20 ms: that step returns
 *     DMDGPU_ERR_GPU and every later step or force call on the context returns
 *     DMDGPU_ERR_GPU without issuing work (state can still be read);
 *   DMDGPU_INJECT_LIST_CAPACITY  the pair-list capacity becomes one chunk: the
 *     next build returns DMDGPU_ERR_CAPACITY (no chunk is written past it). */
#define DMDGPU_INJECT_BARRIER_TIMEOUT 1
#define DMDGPU_INJECT_LIST_CAPACITY 2
int dmdgpu_test_inject(dmdgpu_ctx *ctx, int32_t what);

const char *dmdgpu_last_error(const dmdgpu_ctx *ctx);
void dmdgpu_destroy(dmdgpu_ctx *ctx);

/* ---------------------------------------------------------------------------
 * Batched replicas and continuous serving.  A batch packs many independent
 * systems ("slots") into one device table; one dmdgpu_batch_step advances every
 * running slot with the same kernel launches.  Slots are admitted while the
 * HBM budget allows and released when done; results of a slot do not depend
 * on which other slots share the batch.  No counterpart in the reference
 * (which is one SimulationEngine per process).
 * ------------------------------------------------------------------------- */
typedef struct dmdgpu_batch dmdgpu_batch;

int dmdgpu_batch_create(int64_t budget_bytes, const dmdgpu_options *opt, dmdgpu_batch **out);
/* Admit a system to run n_steps steps; *slot receives its id.  Returns
 * DMDGPU_ERR_BUDGET (nothing admitted) when it does not fit. */
int dmdgpu_batch_admit(dmdgpu_batch *b, const dmdgpu_system *sys, int64_t n_steps, int32_t *slot);
/* Advance every running slot by up to n_steps (a slot stops at its own n_steps). */
int dmdgpu_batch_step(dmdgpu_batch *b, int32_t n_steps);
/* dmdgpu_batch_step with device timing, as dmdgpu_step_timed does for one
 * context (one CUDA graph, events around every step and every non-bonded / PME
 * launch, optional L2 flush between steps); slots stop at their own targets. */
int dmdgpu_batch_step_timed(dmdgpu_batch *b, int32_t n_steps, int64_t l2_flush_bytes,
                            dmdgpu_timing *out);
/* Slots that finished since the last poll: copies up to cap ids into slots. */
int dmdgpu_batch_poll(dmdgpu_batch *b, int32_t *slots, int32_t cap, int32_t *n_done);
int dmdgpu_batch_get_state(dmdgpu_batch *b, int32_t slot, int32_t which, double *x, double *y,
                           double *z);
int dmdgpu_batch_get_scalars(dmdgpu_batch *b, int32_t slot, dmdgpu_scalars *out);
int dmdgpu_batch_release(dmdgpu_batch *b, int32_t slot);
int64_t dmdgpu_batch_used_bytes(dmdgpu_batch *b);
int dmdgpu_batch_get_launch_info(dmdgpu_batch *b, dmdgpu_launch_info *out);
int32_t dmdgpu_batch_active(dmdgpu_batch *b);
const char *dmdgpu_batch_last_error(const dmdgpu_batch *b);
void dmdgpu_batch_destroy(dmdgpu_batch *b);

/* ---------------------------------------------------------------------------
 * Non-bonded forces without any device allocation.
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts whose device memory belongs to another allocator or a fixed arena (a
 * framework's caching allocator, an embedded or real-time system that sizes
 * its memory up front), callers that must not pay for, or risk the failure
 * of, an allocation per call.  It computes what dmdgpu_component_compute gives for
 * components 0 (Lennard-Jones) and 4 (real-space Coulomb) -- the same kernels --
 * on caller-owned device buffers: d_x/d_y/d_z (positions), d_q (charges) and
 * d_type (LJ type per atom) in; d_fx/d_fy/d_fz (forces, written, not
 * accumulated) and d_energies (2 doubles: LJ, real-space Coulomb; may be NULL)
 * out.  Every intermediate buffer lives in one static device array of about
 * 6 MB that each GPU holds from the first use of the library until the process
 * exits; no device memory is allocated or freed.  Atom types must lie in
 * [0, n_types): a type outside it returns DMDGPU_ERR_PARM (and is never used
 * to index the LJ table).
 *
 * Limits (sizes beyond them return DMDGPU_ERR_PARM): n_atoms <=
 * DMDGPU_NOALLOC_MAX_ATOMS, n_types <= DMDGPU_NOALLOC_MAX_TYPES, n_excl <=
 * DMDGPU_NOALLOC_MAX_EXCLUSIONS; a pair list longer than
 * DMDGPU_NOALLOC_MAX_CHUNKS chunks returns DMDGPU_ERR_CAPACITY.
 *
 * The first call on a device resolves the array's device address (one-time
 * set-up) and caches it per device ordinal, so calls must run in the device's
 * primary context (the runtime API's default).  Calls run on `stream` (a
 * cudaStream_t, NULL = legacy default stream) and are synchronous: they copy
 * small host tables from pageable memory and return after the stream has
 * synchronised, so they cannot be issued while that stream is being captured.
 * An error left pending by the caller's earlier work is returned as
 * DMDGPU_ERR_GPU before any work is issued (and is not cleared); a list build
 * whose bounded wait gave up returns DMDGPU_ERR_GPU.  All calls share the one
 * array: calls that overlap on the GPU (other threads, other streams) race and
 * must be serialised by the caller.
 */
#define DMDGPU_NOALLOC_MAX_ATOMS 8192
#define DMDGPU_NOALLOC_MAX_TYPES 16
#define DMDGPU_NOALLOC_MAX_EXCLUSIONS 32768
#define DMDGPU_NOALLOC_MAX_SORT_CELLS 32768
#define DMDGPU_NOALLOC_MAX_CHUNKS 16384

typedef struct dmdgpu_nb_params {
    int32_t n_atoms;
    double box;                        /* cubic box length */
    int32_t n_types;
    const double *lj_sigma, *lj_epsilon; /* host, n_types x n_types */
    double lj_cutoff, coul_cutoff, ewald_coeff;
    int32_t n_excl;                    /* exclusion pairs (host); PHYS skips them */
    const int32_t *excl_i, *excl_j;
    int32_t profile;                   /* DMDGPU_PROFILE_* */
    int32_t precision;                 /* DMDGPU_PRECISION_* */
    double skin;                       /* PHYS list skin (nm) */
} dmdgpu_nb_params;

int dmdgpu_nonbonded_noalloc(const dmdgpu_nb_params *p, const double *d_x, const double *d_y,
                             const double *d_z, const double *d_q, const int32_t *d_type,
                             double *d_fx, double *d_fy, double *d_fz, double *d_energies,
                             void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DMDGPU_H */
