// engine_state.cuh -- host-side state of one batched replica engine
// (struct bd_engine of the C ABI), shared by the translation units that
// implement bd_engine_* entry points.
#pragma once
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <vector>

#include "engine.cuh"
#include "runtime.cuh"

struct bd_engine {
    int dev = 0;
    cudaStream_t stream = nullptr;
    int R = 0;
    std::vector<bd_system_desc> desc;
    std::vector<bd::SysDev> sysh;
    bd::SysDev *d_sys = nullptr;
    std::vector<int4> bricks_h;
    int4 *d_bricks = nullptr;
    int nbricks = 0;
    int bx = 4, by = 4, bz = 3, cap = 16, threads = 128, smax = 0, mode = BD_MODE_PLAIN, cluster = 8;
    size_t smem = 0, smem_census = 0;
    size_t lsmem = 0;  // list build (kListBuildThreads per CTA)
    long long C = 0, P = 0;
    int *cnt[3] = {nullptr, nullptr, nullptr};
    float4 *pos[3] = {nullptr, nullptr, nullptr};
    int cur = 0;
    float *lo[3] = {nullptr, nullptr, nullptr};
    double *dsp[3] = {nullptr, nullptr, nullptr};
    int *gid_of = nullptr, *rep_of_sid = nullptr, *rep_of_gid = nullptr;
    double *x0 = nullptr, *obs = nullptr;
    float4 *snap = nullptr;
    int *nbr_count = nullptr;
    unsigned long long *nbr_hash = nullptr;
    curandState *cr = nullptr;
    float *noise = nullptr;
    unsigned long long *rn_ring = nullptr, *rn_lcg = nullptr;  // rannew64 streams by storage id
    long long rn_ni0 = 0;
    unsigned *status = nullptr;
    long long *d_ni = nullptr;
    float *out_pos = nullptr, *out_raw = nullptr;
    long long ni = 0, ni_first = 0;
    int rng = BD_RNG_PHILOX;
    unsigned rng_stream = 0;
    float qmax = 6.2831853f;
    bool loaded = false;
    int graph_steps = 96;
    cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};  // one per rotation phase e->cur
    int autotune = 0;
    bool tuned = false;
    int lvar = 0;            // list-step launch variant (ListVariant<lvar>)
    bool tune_lvar = false;  // the autotuner chooses lvar
    // persistent mode: replicas packed into cluster bins
    std::vector<int> cl_start_h, cl_bricks_h;
    int *d_cl_start = nullptr, *d_cl_bricks = nullptr;
    int nclusters = 0, max_clusters = 0;
    float tuned_ms = 0.f;
    // displacement snapshots for waiting-time correlations: slot k holds the
    // FP64 displacement of every storage id, [k][axis][P]
    double *snaps = nullptr;
    int nslots = 0;
    std::vector<long long> snap_ni;   // step index at which each slot was taken
    std::vector<long long> snap_gen;  // set_positions generation of each slot
    long long generation = 0;
    // correlation reduction: segment table and scratch
    int2 *d_segs = nullptr;
    int *d_seg_first = nullptr;
    int nsegs = 0;
    double *corr_part = nullptr, *corr_out = nullptr;
    size_t corr_part_cap = 0, corr_out_cap = 0;
    // neighbour-list mode (plain mode with generated noise): positions by
    // storage id (double-buffered, e->cur selects), build positions, lists
    bool list = false;
    bool extra_pot = false;  // some replica uses a potential other than the modified WCA
    float skin = 0.f;
    float4 *lpos[2] = {nullptr, nullptr};
    float4 *pbuild = nullptr;
    int *nbr = nullptr, *nnb = nullptr;
    int *lflag = nullptr, *d_one = nullptr;
    long long *d_builds = nullptr;  // [0] replica list builds, [1] steps that rebuilt
    int *img = nullptr;             // [3][P] face crossings since the origin (displacement on demand)
    float *amp_tab = nullptr;       // [graph_steps][R][2] noise amplitudes of a launch batch
    int *d_rep_order = nullptr;     // per-replica launch (variants 3-5): replica of each block
    size_t lrep_smem = 0;           // variant 5: shared memory of an in-block rebuild (0: from global memory)
    int *d_step_rebuilt = nullptr;  // [graph_steps] steps of such a launch that rebuilt a replica
    // set_positions scratch (storage order computed on the device)
    float *ld_in = nullptr;        // [P][3] positions as given
    float4 *ld_staged = nullptr;   // [P] in storage order
    int *ld_slot = nullptr, *ld_bucket = nullptr;  // [P]
    int *ld_cnt = nullptr, *ld_start = nullptr;    // [slots]: count, first storage id
    int *ld_bsum = nullptr;                         // [slots / kScanBlock + 1]
    unsigned *ld_bad = nullptr;
    long long ld_slots = 0;        // capacity of ld_cnt
};


namespace bd {

// cell-bounded g(r) (gder.cu): stencil reach of a replica (-1: region would
// wrap) and the launch over the replicas with m_of[r] >= 0; replicas it
// cannot count come back with m_of[r] = -1
int gder_cell_reach(const SysDev &S, float range);
int launch_gder_cells(bd_engine *e, std::vector<int> &m_of, int nbins, float range, const float *d_thr,
                      unsigned long long *d_counts);

// cell-bucket buffer holding the current state (list mode rebuilds buffer 0
// before every observation pass)
inline int obs_buf(const bd_engine *e) { return e->list ? 0 : e->cur; }

// list mode keeps no per-step displacement: rebuild dsp[] from the state
// before anything reads it (a no-op in the other modes)
int sync_dsp(bd_engine *e);

inline int engine_status(bd_engine *e) {
    unsigned bits = 0;
    BD_CUDA_TRY(cudaMemcpyAsync(&bits, e->status, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    BD_CUDA_TRY(cudaStreamSynchronize(e->stream));
    return status_from_bits(bits);
}

}  // namespace bd
