// launch.h -- host-side launchers of the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "layout.h"

namespace dmd {

// k_list.cu: spatial sort + pair-list build for replicas whose `rebuild` flag
// is set, as one cooperative launch (returns at once when no replica rebuilds).
void launch_rebuild(const Dev& d, const int* bin_rep, int n_sm, cudaStream_t st, long long* nlaunch);

// k_nonbonded.cu: LJ + real-space Ewald over the pair list (replicas with `eval`).
// Pair energies and virial are summed only for replicas whose `want_e` is set.
// The mixed-precision kernels are persistent with blocks_per_sm blocks of 256
// threads per SM (1..3) and come in two forms -- one warp per 32 x 32 chunk,
// or one warp per 8-atom i-cluster over its rows (needs d.cl_j) -- both chosen
// by the engine's autotuner; results do not depend on the launch shape (one
// warp per work item, fixed-point sums).
enum NbForm { NB_CHUNK32 = 0, NB_CLUSTER8 = 1 };
void launch_nonbonded(const Dev& d, bool fp64, bool phys, int n_sm, int blocks_per_sm, int form,
                      cudaStream_t st, long long* nlaunch);
// Whether a kernel function (cudaGraphKernelNodeGetParams' func) is one of the
// pair kernels: the step graph gives every other kernel the higher priority.
bool is_nonbonded_kernel(const void* func);
// Per-device function attributes of the pair kernels (the shared-memory
// carveout); called once per context before the first launch.
void configure_nonbonded_kernels();

// k_forces.cu
// bonds, angles, dihedrals and the exclusion correction in one launch
void launch_bonded(const Dev& d, bool fp64, bool phys, cudaStream_t st, long long* nlaunch);
void launch_pme_spread(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch);
void launch_pme_convert(const Dev& d, bool fp64, int n_blocks, cudaStream_t st, long long* nlaunch);
void launch_pme_influence(const Dev& d, bool fp64, int n_blocks, cudaStream_t st,
                          long long* nlaunch);
void launch_pme_gather(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch);

// k_integrate.cu
enum EvalPass { PASS_FIRST = 1, PASS_SECOND = 2, PASS_SINGLE = 3 };
void launch_eval_begin(const Dev& d, int pass, cudaStream_t st, long long* nlaunch);
void launch_clear_forces(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_eval_end(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_kick_drift(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch);
void launch_kick2(const Dev& d, bool andersen_ref, bool andersen_phys, cudaStream_t st,
                  long long* nlaunch);
void launch_shake(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_rattle(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_replica_update(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_apply_scale(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch);
void launch_finalize_velocities(const Dev& d, cudaStream_t st, long long* nlaunch);
void launch_energy_reduce(const Dev& d, cudaStream_t st, long long* nlaunch);
// replica r's frame (step, time, box, positions, velocities) into `out`
// (3 + 6 n_atoms doubles), state unchanged
void launch_frame_snapshot(const Dev& d, int r, int n_atoms, double* out, cudaStream_t st, long long* nlaunch);
void launch_write_mirror(const Dev& d, bool fp64, cudaStream_t st, long long* nlaunch);

}  // namespace dmd
