// wenofv_engine.h -- host-side engine behind the C ABI: a set of instances on one device
// advanced together by the fused stage kernels.  A single-grid context is an engine with one
// instance; the batch API exposes several; the server adds and removes instances in slots.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/wenofv.h"
#include "wenofv_types.h"

namespace wenofv {

void set_error(const char *fmt, ...);
const char *last_error_text();
int cuda_fail(cudaError_t e, const char *what);
#define WENOFV_CUDA(call)                                                   \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #call);                 \
    } while (0)

int validate(const wenofv_config *cfg, const wenofv_eq_params *eq);
int nvar_of(int eq_kind);
// the device-side equation parameters (for the stiffened-gas model with the linearised sound
// speeds of its first guess)
EqParams eq_params_of(const wenofv_eq_params &e);
// the reference's grid metric (src/WENOFV.cpp:89-123), see wenofv_create
void grid_metric(const wenofv_config &c, double *dxc, double *dxl, double *dy);

// buffer roles of one RK stage for a step starting at parity p (the state returns to
// buffer 0 after two steps, so a captured pair of steps has fixed roles)
struct Roles { int bin, bun, bout; };
Roles stage_roles(int rk, int parity, int stage);
int stage_count(int rk);
void stage_coeffs(int rk, int stage, double &A, double &B, double &C);

class Engine {
public:
    ~Engine();
    // all instances live (context and batch)
    int init(int n, const wenofv_config *cfgs, const wenofv_eq_params *eqs);

    int upload(int i, const double *U, int layout);
    int download(int i, double *U, int layout);
    int compute_dt(double *dt_out);                // per instance, synchronises
    int step(double dt);                           // one manual RK step of every instance
    int rhs(double *out, int layout);              // instance 0
    int advance(const double *t0, const double *t_end, int64_t max_steps, double *t_out, int64_t *nsteps);
    int status(int i, uint32_t *flags, int64_t *cell);
    int set_tiling(int rows, int ctas_per_sm);
    int autotune(int *rows, int *ctas_per_sm, double *best_ms);
    // puts states, buffer rotation, loop state and tiling back after a tuning search
    void restore_after_tune(int rows, int ctas, int nt, int cur, const InstState *st, const std::vector<double *> &saved);
    int set_threads(int nt);                           // 0: per instance by the width model; 128 or 256
    void tiling(int *rows, int *ctas, int *nt) const;  // the current settings (0 = automatic)
    int device_state(int i, double **U, int *pitch);
    int set_frame(int i, const double *frame); // NEUMANN2 ghost averages, SoA [v][ny+8][nx+8]
    int theta_flags(int i, unsigned char *out, int layout); // the final stage's limiter record per cell
    int snapshot_begin(int i, double *host, int layout);     // async copy of the current state
    int snapshot_wait();                                     // blocks until that copy has landed
    int init_testcase(int i, const wenofv_testcase *tc);                      // wenofv_init.cu
    int accuracy(int i, const wenofv_testcase *tc, double t, double *norms); // wenofv_init.cu

    // ---- slots (serving): capacity fixed at init_slots, instances added and removed ----
    // arena_bytes > 0: every slot's device memory comes from one arena allocated here, so that
    // adding a slot calls no cudaMalloc
    int init_slots(int capacity, int device, int rk_method, size_t arena_bytes = 0);
    int add(const wenofv_config &cfg, const wenofv_eq_params &eq, int *slot);
    int remove(int slot);
    int start(int slot, double t_end, int64_t max_steps); // device loop of one slot: t = 0 -> t_end
    // start several slots at once: one CFL launch per launch group over the new slots only
    int start_many(const std::vector<int> &slots, const std::vector<double> &t_end, const std::vector<int64_t> &max_steps);
    int run_pairs(int K);                                 // K pairs of steps of every live, unfinished slot
    int run_graph_pairs(int K);                           // the same, as one captured graph
    int refresh();                                        // pull the device loop state
    size_t arena_free_bytes() const;
    const InstState &slot_state(int slot) const { return h_state_[slot]; }
    bool live(int slot) const { return slot >= 0 && slot < cap_ && live_[slot]; }
    static size_t bytes_needed(const wenofv_config &cfg, const wenofv_eq_params &eq);

    cudaStream_t stream = nullptr;
    int device = 0;
    int n = 0;
    int rk = 2;
    bool slot_mode = false;    // serving: every slot keeps its own current buffer
    bool theta_record = false; // contexts: keep the limiter's per-cell record (wenofv_theta_flags)
    bool solo = false;         // contexts: one instance alone on the GPU (instance_nt)

private:
    // one persistent launch per RK stage for the instances of one template key; the work
    // list, the finalize list and their counts live in device buffers that are rewritten in
    // place while they fit, so a captured graph stays valid when instances come and go
    struct Group {
        long key = 0;
        int ns_strict, fp32, eq, recon, scheme, flux, nt = 128;
        std::vector<int> inst;
        WorkItem *d_work = nullptr;
        int nwork = 0, cap_work = 0;
        int *d_fin = nullptr;
        int cap_fin = 0;
        int *d_counts = nullptr; // {nwork, nfin} (+ {init nwork, init nfin} for start_many)
        WorkItem *d_init_work = nullptr;
        int *d_init_fin = nullptr;
        int cap_init_work = 0, cap_init_fin = 0;
        unsigned int *d_counter = nullptr;
        int grid = 0;
        cudaStream_t gstream = nullptr; // the group's branch inside a captured graph
        cudaEvent_t joined = nullptr;
    };
    struct Block { size_t off, size; };
    int build_work();
    void free_work();
    long group_key(int i) const;
    int instance_nt(int i) const;
    int item_rows(const std::vector<int> &inst, int tx, int slots) const;
    double waves_of(const std::vector<int> &inst, int tx, int slots, int s) const;
    int group_launch(const Group &g, StageLaunch &L) const;
    int arena_alloc(size_t bytes, size_t *off);
    void arena_free(size_t off);
    int ensure_work();
    int alloc_instance(int i, const wenofv_config &c, const wenofv_eq_params &e);
    void free_instance(int i);
    int launch_stage_all(int parity, int stage, double *rhs_out);
    int check_frames() const;
    int ensure_stage(size_t bytes);
    int launch_cfl_all();
    int pull_state();
    int push_state();
    int normalize_buffers();
    int run_graph(int double_steps);
    void drop_graphs();

    std::vector<wenofv_config> cfg_;
    std::vector<wenofv_eq_params> eq_;
    std::vector<InstDesc> desc_;
    std::vector<double *> dmem_;    // per instance: 3 state buffers
    std::vector<double *> dmetric_; // per instance: dxc, dxl, dy
    std::vector<double *> dframe_;  // per NEUMANN2 instance: its ghost frame
    std::vector<unsigned char *> dtheta_; // per instance: the limiter's per-cell theta record [ny][nx]
    // snapshot: a device copy of one state, read back on a copy stream while the next steps run
    double *d_snap_ = nullptr;
    double *h_snap_ = nullptr; // pinned read-back of the snapshot (pitched), repacked by snapshot_wait
    size_t snap_bytes_ = 0;
    cudaStream_t copy_stream_ = nullptr;
    cudaEvent_t snap_ready_ = nullptr, snap_done_ = nullptr;
    double *snap_host_ = nullptr;
    int snap_layout_ = 0, snap_nv_ = 0, snap_nx_ = 0, snap_ny_ = 0, snap_pitch_ = 0;
    bool snap_pending_ = false;
    std::vector<char> frame_set_;
    std::vector<char> live_;
    std::vector<Group> groups_;
    InstDesc *d_desc_ = nullptr;
    InstState *d_state_ = nullptr;
    InstState *h_state_ = nullptr; // pinned mirror
    double *h_stage_ = nullptr;    // pinned staging for upload/download
    size_t h_stage_bytes_ = 0;
    double *d_rhs_ = nullptr;
    int rows_per_item_ = 0, ctas_per_sm_ = 0;
    int nt_override_ = 0; // 0: CTA width per instance by the width model; 128 or 256: forced
    int sms_ = 148;
    int cap_ = 0;
    int cur_ = 0; // buffer holding every instance's state between calls (context/batch)
    bool work_dirty_ = true;
    std::map<int, cudaGraphExec_t> graphs_;
    std::map<int, cudaGraph_t> graph_defs_;
    cudaEvent_t fork_ = nullptr;
    bool capturing_ = false; // launch_stage_all puts each group on its own branch
    // slot arena: one allocation, first-fit blocks of 256-byte granularity
    char *arena_ = nullptr;
    size_t arena_bytes_ = 0;
    std::map<size_t, size_t> arena_freelist_; // offset -> size of the free blocks
    std::map<size_t, size_t> arena_used_;     // offset -> size of the allocated blocks
    std::vector<size_t> slot_off_;            // per slot: offset of its block (arena mode)
};

} // namespace wenofv
