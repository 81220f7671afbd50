// engine.h -- host orchestration of the device path (one Batch = one packed table).
#pragma once

#include <cufft.h>

#include <map>
#include <utility>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dmdgpu.h"
#include "layout.h"

namespace dmd {

// Component selection for single-component evaluation (ForceComponent parity).
enum CompMask : unsigned {
    C_LJ = 1u << 0, C_BOND = 1u << 1, C_ANGLE = 1u << 2, C_DIH = 1u << 3, C_CREAL = 1u << 4,
    C_PME = 1u << 5, C_EXCL = 1u << 6, C_IMP = 1u << 7, C_ALL = 0xffu
};

// Host copy of one system (a SimulationConfig) plus its packing metadata.
struct HostSystem {
    int n = 0;
    double box = 0;
    std::vector<double> mass, q, x, y, z, vx, vy, vz;
    std::vector<int> type;
    int use_lj = 0, n_types = 0;
    std::vector<double> sigma, eps;
    double lj_cutoff = 1.2;
    std::vector<int> bi, bj;
    std::vector<double> bk, br0;
    std::vector<int> ai, aj, ak;
    std::vector<double> akt, at0;
    std::vector<int> di, dj, dk, dl, dn;
    std::vector<double> dkp, dp0;
    std::vector<double> xr, yr, zr;   // positions of the last list build (empty: never built)
    std::vector<int> ii, ij, ik, il;
    std::vector<double> ikp, ip0;
    std::vector<int> ei, ej;
    std::vector<int> ci, cj;              // distance constraints (SHAKE / RATTLE), in sweep order
    std::vector<double> cd;
    double ctol = 1e-6;
    int coulomb_type = 0;
    double coul_cutoff = 1.2, ewald = 0.34, spacing = 0.12;
    int pme_order = 4, pme_K = 0;
    double dt = 0.002;
    int n_steps = 0;
    int thermostat = 0;
    double t_temp = 300, t_tau = 0.1, t_freq = 10;
    int barostat = 0;
    double b_pressure = 1, b_tau = 1, b_compress = 4.5e-5;
    int checkpoint_interval = 0;
    std::string checkpoint_path;
};

// Per-replica bookkeeping kept on the host.
struct HostRep {
    HostSystem sys;
    Rep rep{};
    RepState init{};
    long long target = 0;      // step count to reach (served jobs)
    unsigned andersen_seed = 42;
    bool done = false;
    bool polled = false;
    bool on_device = false;    // packed into the current device table (its state lives there)
};

// Device memory of the packed table: slabs kept by the batch across table
// rebuilds, handed out by a bump pointer.  A serving loop rebuilds its table at
// every admission and release; cudaMalloc and cudaFree of every array each
// time stall the device (cudaFree waits for it and unmaps: measured up to
// ~0.7 s in one rebuild), so the table reuses one slab while it fits and a
// new slab is made only when it grows (or shrinks far below it).
struct SlabStore {
    struct Slab {
        char* p;
        size_t cap;
    };
    std::vector<Slab> slabs;
    void prepare(size_t expect);  // one slab of at least `expect` bytes
    void release();
    ~SlabStore() { release(); }
};

struct DeviceArena {
    SlabStore* store = nullptr;
    cudaStream_t stream = nullptr;  // zero fills are issued here, before the uploads
    size_t slab = 0, off = 0;       // bump position
    size_t bytes = 0;               // bytes handed out (budget accounting)
    template <typename T>
    T* alloc(size_t n);
};

// Pinned host blocks the table uploads are staged in (kept across rebuilds):
// every upload is one asynchronous copy on the main stream, with one
// synchronisation for all of them.
struct PinnedStaging {
    std::vector<std::pair<char*, size_t>> blocks;
    size_t blk = 0, off = 0;
    void* put(const void* src, size_t bytes);
    void reset() { blk = off = 0; }
    void trim(size_t keep);       // frees the later blocks beyond `keep` bytes
    ~PinnedStaging() { trim(0); }
};

class Batch {
  public:
    Batch(const dmdgpu_options& opt, long long budget_bytes);
    ~Batch();

    // Replica management (host side; the device table is rebuilt by pack()).
    int add(const dmdgpu_system& sys, long long n_steps, unsigned comp_mask, int* slot);
    int release(int slot);
    int pack();                 // (re)build the packed device table from host replicas
    int repack();               // rebuild the table now, carrying every replica's state
    long long footprint(const HostSystem& s) const;

    int step(int n);            // advance every running replica by up to n steps
    int extend_targets(long long n);  // single-system API: allow n more steps
    int step_timed(int n, long long flush_bytes, dmdgpu_timing* out);
    cudaStream_t stream() const { return stream_; }
    int compute_forces(int slot, double* fx, double* fy, double* fz, double* e_terms);
    int get_state(int slot, int which, double* x, double* y, double* z);
    int set_state(int slot, int which, const double* x, const double* y, const double* z);
    int get_scalars(int slot, dmdgpu_scalars* out);
    int pair_list(int slot, int32_t* pi, int32_t* pj, long long cap, long long* count);
    int save_checkpoint(int slot, const char* path);
    int load_checkpoint(int slot, const char* path);
    int poll(int32_t* slots, int cap, int* n_done);
    // Host-side fault injection for the failure-path tests (DMDGPU_INJECT_*).
    int inject(int what);
    bool uses_clusters() const;  // the options select the 8-atom i-cluster pair form
    // Trajectory frames of a single-system table (dmdgpu_set_frame_writer).
    int set_frame_writer(int interval, dmdgpu_frame_fn fn, void* user);
    int flush_frames();

    long long used_bytes() const { return used_bytes_; }
    long long launches() const { return launches_; }
    void launch_info(dmdgpu_launch_info* out) const;
    int active() const;
    const std::string& error() const { return err_; }
    int fail(int code, const std::string& msg);
    const HostSystem& system(int slot) const { return reps_.at(slot)->sys; }
    bool has(int slot) const { return slot >= 0 && slot < (int)reps_.size() && reps_[slot]; }

  private:
    int check_cuda(cudaError_t e, const char* what);
    int build_host(HostRep& hr, unsigned comp_mask);
    void enqueue_eval(int pass);
    void enqueue_rebuild();
    void enqueue_step();
    int run_steps(int n);
    int autotune(int max_steps, int* used);
    int rebuild_in_frame(const std::vector<char>& sel);
    int sync_status();
    int replica_index(int slot) const;
    void free_device();
    void andersen_ref_prepare();
    int ensure_plans(int K);  // cuFFT R2C/C2R plans of mesh size K, made once per batch

    dmdgpu_options opt_;
    long long budget_;
    bool fp64_, phys_;
    int device_ = 0, n_sm_ = 148;
    cudaStream_t stream_ = nullptr;
    // bonded + PME run on aux_stream_, forked from and joined back to stream_
    cudaStream_t aux_stream_ = nullptr;
    // bonded terms on a third stream, beside both
    cudaStream_t bond_stream_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr, ev_join_b_ = nullptr;
    bool capture_error_ = false;
    std::vector<std::unique_ptr<HostRep>> reps_;   // indexed by slot (nullptr = free)
    std::vector<int> order_;                        // packed replica index -> slot
    SlabStore slabs_;                                // declared before arena_: outlives it
    std::unique_ptr<DeviceArena> arena_;
    PinnedStaging staging_;
    double fp_ratio_ = 1.0;                          // last table's bytes / its footprint estimate
    Dev dev_{};
    Rep* d_rep_ = nullptr;
    RepState* d_st_ = nullptr;
    RepState* h_st_ = nullptr;                      // pinned mirror of the state table
    bool st_fresh_ = false;                         // h_st_ equals the device table (no work since)
    long long* h_tgt_ = nullptr;                    // pinned step targets for extend_targets
    int h_st_cap_ = 0;                              // replicas h_st_ / h_tgt_ hold
    int* d_bin_rep_ = nullptr;
    int n_pme_blocks_ = 0, n_conv_blocks_ = 0;
    bool any_cons_ = false;  // some replica has distance constraints
    bool any_pme_ = false, any_baro_ = false, any_narrow_ = false, any_ref_lj_ = false, any_andersen_ref_ = false,
         any_andersen_phys_ = false;
    std::map<int, std::pair<cufftHandle, cufftHandle>> plans_;
    cudaGraphExec_t graph_ = nullptr;
    bool packed_ = false;
    // a list build timed out: its sort and list buffers are in an unknown
    // state, so no further device work is issued on this table
    bool failed_ = false;
    bool graph_dirty_ = true;
    bool need_eval1_ = true;
    int nb_blocks_per_sm_ = 2;  // pair-kernel launch shape (autotuned)
    int prio_lo_ = 0, prio_hi_ = 0;  // stream priority range
    double density_ = 0.0;           // table atoms per nm^3 (autotuner cache key)
    void set_node_priorities(cudaGraph_t g);
    int nb_form_ = 1;           // pair-kernel form (NbForm; autotuned)
    bool tuned_ = false;
    long long launches_ = 0;
    long long per_step_launches_ = 0;
    long long used_bytes_ = 0;
    // per-kernel timing (step_profiled): event pairs recorded around launches
    std::vector<cudaEvent_t> ev_pool_;
    size_t ev_used_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* prof_nb_ = nullptr;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* prof_pme_ = nullptr;
    void* flush_buf_ = nullptr;
    long long flush_bytes_ = 0;
    void record(cudaEvent_t e, cudaStream_t st);
    // frame export: a device snapshot on the main stream into one of
    // DMDGPU_FRAME_SLOTS staging buffers, then a copy to pinned host memory and
    // the writer call on copy_stream_
    struct FrameSlot {
        Batch* self;
        int index;
    };
    int enqueue_frame();
    void free_frames();
    static void CUDART_CB deliver_frame(void* p);
    int frame_interval_ = 0;
    dmdgpu_frame_fn frame_fn_ = nullptr;
    void* frame_user_ = nullptr;
    int frame_n_ = 0;
    cudaStream_t copy_stream_ = nullptr;
    double* frame_dev_[DMDGPU_FRAME_SLOTS] = {};
    double* frame_host_[DMDGPU_FRAME_SLOTS] = {};
    cudaEvent_t frame_snap_[DMDGPU_FRAME_SLOTS] = {};
    cudaEvent_t frame_done_[DMDGPU_FRAME_SLOTS] = {};
    FrameSlot frame_slot_[DMDGPU_FRAME_SLOTS] = {};
    long long frame_count_ = 0;
    cudaEvent_t next_event();
    std::string err_;
    std::vector<int> finished_;
    // Andersen REF override buffers
    int* h_and_flag_ = nullptr;
    double* h_and_v_ = nullptr;
    long long h_and_cap_ = 0;                       // atoms h_and_flag_ / h_and_v_ hold
    int* d_and_flag_ = nullptr;
    double* d_and_v_ = nullptr;
};

}  // namespace dmd
