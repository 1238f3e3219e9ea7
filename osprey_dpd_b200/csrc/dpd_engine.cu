// dpd_engine.cu -- host runtime of the B200 DPD step engine and its C ABI
// (include/dpd_engine.h).  It owns the device state, queues one timestep as a
// fixed sequence of kernels on one CUDA stream, and translates between the
// reference's bead-object view (bead-vector order, FP64 xyz triplets) and the
// device's cell-sorted structure-of-arrays.
#include "../../include/dpd_engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "dpd_kernels.cuh"
#include "pair_forces.cuh"
#include "pair_staged.cuh"
#include "slice_stress.cuh"
#include "monitor.cuh"
#include "upload.cuh"
#include "builder.cuh"
#include "slab.cuh"
#include <climits>

using namespace dpd;

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// One z-slab of a decomposed box (dpd_engine_slab_*): the geometry, the pack's
// scratch and the whole box's topology on the device.
struct SlabState {
    SlabGeom geom{};
    int* d_bcount = nullptr;             // kSlabOuts block counts, then their offsets
    size_t cap_bcount = 0;
    int* d_total = nullptr;              // kSlabOuts stream totals
    double* d_keep = nullptr;            // staying owned beads' records (local frame)
    double* d_mine = nullptr;            // own migrants' records (local frame)
    size_t cap_keep = 0, cap_mine = 0;
    int* h_sizes = nullptr;              // k_slab_sizes' output, mapped pinned memory
    int* d_sizes = nullptr;
    bool packed = false;                 // a pack waits for its unpack
    // topology of the whole box, by bond / bond-pair index and by bead id
    bool topo = false;
    int nb = 0, na = 0, id_max = 0;
    size_t nterm = 0;
    int *d_head_id = nullptr, *d_tail_id = nullptr, *d_first = nullptr, *d_second = nullptr;
    int *d_gptr = nullptr, *d_gterm = nullptr;
    unsigned long long* d_idmap = nullptr;
    unsigned version = 0;
    int* d_cnt = nullptr;
    int* d_bsum = nullptr;
    size_t cap_cnt = 0, cap_bsum = 0, cap_bb = 0;
};

}  // namespace

struct dpd_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;          // bonded-force branch, forked from and joined to s()
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    dpd_params params{};
    int precision = DPD_PRECISION_MIXED;
    std::vector<double> a, gamma, gamma_backup, a_backup;   // host copies of the tables
    bool thermostat_on = true, conservative_on = true;
    int32_t ntypes = 0;
    int64_t ncell = 0;
    int nchunk = 0;
    int64_t n = 0;
    int64_t cap_n = 0;          // beads the per-bead buffers hold
    double n_headroom = 1.0;    // their growth factor (a slab's bead count changes every step)
    SlabState* slab = nullptr;  // set by dpd_engine_slab_setup
    bool host_ids_stale = false;   // h_id / h_type lag an upload from device memory
    int64_t launches = 0;
    bool uploaded = false;
    bool stepped = false;
    int64_t last_step = 0;      // m_SimTime of the state on the device
    int cur = 0;                // which of the double buffers holds the state
    std::string err;

    // boxes: one for a single simulation, one per replica for a batch
    std::vector<Box> hboxes;
    std::vector<double> box_a, box_g;   // nboxes * ntypes^2 each
    Box* d_boxes = nullptr;
    double* d_box_obs = nullptr;        // nboxes * kObsTerms, filled on demand
    bool box_obs_valid = false;

    // device state
    StepConst* d_K = nullptr;
    void* d_tab = nullptr;      // 3 * T*T of real: a, gamma, sigma
    int64_t* d_step = nullptr;
    unsigned* d_status = nullptr;
    double* d_x[2] = {nullptr, nullptr};
    double* d_v[2] = {nullptr, nullptr};
    int* d_bid[2] = {nullptr, nullptr};
    int* d_tf[2] = {nullptr, nullptr};
    uint32_t* d_img[2] = {nullptr, nullptr};
    int* d_cell[2] = {nullptr, nullptr};
    // UpdatePos of the next call's first step, done by the last k_update_mom of
    // a call into these buffers (the visible state keeps the step's own x, img, cell)
    double* d_xa = nullptr;
    uint32_t* d_imga = nullptr;
    int* d_cella = nullptr;
    bool ahead_valid = false;    // d_xa/d_imga/d_cella and the arrival counts hold the next drift
    // upload staging: the caller's arrays as given, and per-bead scratch by upload index
    double* d_up = nullptr;
    size_t cap_up = 0;
    int* d_up_cell = nullptr;
    uint32_t* d_up_img = nullptr;
    double* d_up_off = nullptr;
    int* d_up_perm = nullptr;
    int* d_up_err = nullptr;           // error slots, residual flag, changed bits, type counts
    int64_t* d_prev_id = nullptr;      // ids and types of the last upload (upload order)
    int* d_prev_type = nullptr;
    size_t cap_prev_id = 0, cap_prev_type = 0;
    int64_t prev_n = -1;               // bead count whose d_prev_* hold a complete upload (-1: none)
    size_t cap_up_cell = 0, cap_up_img = 0, cap_up_off = 0, cap_up_perm = 0, cap_up_err = 0;
    bool ahead_enabled = true;
    bool pdl = true;             // programmatic dependent launch of the step kernels
    void* d_F = nullptr;        // current force, slot order (real)
    void* d_Fold = nullptr;     // previous force, slot order (real)
    void* d_stress = nullptr;   // per-bead virial of the last sample step (real, 9 planes)
    void* d_pos4 = nullptr;
    void* d_vel4 = nullptr;
    int* d_rank = nullptr;
    int* d_perm = nullptr;
    int* d_pid[2] = {nullptr, nullptr};   // noise id (reference bead id) in slot order
    int* d_pid_of = nullptr;              // noise id by upload index
    double4* d_ubuf = nullptr;            // unPBC position of bonded beads by upload index (FP64)
    int* d_bb = nullptr;                  // bonded beads' upload indices, ascending
    int64_t nbb = 0;
    int64_t topo_nb = 0, topo_na = 0;     // bonds and bond pairs of the uploaded topology

    // slice stress profile (CMonitor::AddBeadStress & co.), built on sample steps
    int slice_S = 0, slice_nbt = 0, slice_nbpt = 0;
    double* d_slice = nullptr;            // pair | bond | bondpair bins, one allocation
    // the profile's pair list (kSliceListPerBead entries a bead) and its counters
    uint2* d_slice_list = nullptr;
    unsigned* d_slice_cnt = nullptr;
    double* d_slice_part = nullptr;      // k_slice_eval's per-block partial sums
    size_t cap_slice_list = 0, cap_slice_cnt = 0, cap_slice_part = 0;
    size_t cap_slice = 0;
    int* d_slice_bt = nullptr;            // bond type per bond
    int* d_slice_bpt = nullptr;           // bond-pair type per bond pair
    size_t cap_slice_bt = 0, cap_slice_bpt = 0;
    bool slice_sampled = false;           // a sample step has filled the bins

    // CMonitor sample data on request (dpd_engine_set_monitor / dpd_engine_monitor)
    std::vector<int64_t> type_count;      // beads per type at the last upload
    std::vector<int64_t> h_id;            // bead ids and types by upload index (restart files)
    std::vector<int32_t> h_type;
    uint64_t ids_version = 0;             // advanced when an upload brings other bead ids
    // the inputs of the last topology build, which the staging buffer still
    // holds: an identical upload for the same bead ids reuses it
    struct TopoInputs {
        std::vector<int64_t> bh, bt, f, sc;
        std::vector<double> k2, l0, k3, phi0;
        uint64_t ids_version = ~0ull;
        int64_t n = 0, nbl = 0;
        bool valid = false;
    } topo_in;
    // restart-file layout: file order of the beads (upload indices), their polymer id and type
    std::vector<int64_t> rs_order, rs_poly_id;
    std::vector<int32_t> rs_poly_type;
    std::vector<double> rs_radius;        // per bead type
    std::vector<double> h_ang_phi0;       // bond-pair phi0 of the uploaded topology
    bool mon_set = false;
    int mon_nbt = 0, mon_npt = 0, mon_nbpt = 0;
    int64_t mon_np = 0;
    std::vector<int64_t> mon_bcount, mon_pcount, mon_bpcount;
    int *d_mon_bt = nullptr, *d_mon_bpt = nullptr, *d_mon_ph = nullptr, *d_mon_pt = nullptr, *d_mon_ptype = nullptr;
    double *d_mon_phi0 = nullptr, *d_mon_u0 = nullptr, *d_mon_xu = nullptr, *d_mon_sums = nullptr;
    double4* d_Fb = nullptr;              // bonded force by upload index (FP64)
    double* d_Sb = nullptr;               // bond virial, 9 planes by upload index (sample steps)
    double* d_off = nullptr;
    int* d_count = nullptr;
    int* d_start = nullptr;
    int* d_block_count = nullptr;
    double* d_partials = nullptr;
    double* d_obs = nullptr;
    double* d_renorm = nullptr;     // kinetic sums of dpd_engine_renormalise_mom (kObsTerms)
    // download staging
    double* d_out = nullptr;    // 3n x, 3n u, 3n v, 3n f, 9n stress
    int* d_out_cell = nullptr;
    // topology (buffers grow but never move for same-size uploads, so
    // captured graphs stay valid)
    size_t cap_csr_ptr = 0, cap_csr_term = 0, cap_bond = 0, cap_ang = 0, cap_off = 0, cap_ubuf = 0, cap_bb = 0,
           cap_Fb = 0, cap_Sb = 0;
    bool off_active = false;
    int* d_csr_ptr = nullptr;
    int* d_csr_term = nullptr;
    int* d_bond_h = nullptr;
    int* d_bond_t = nullptr;
    double* d_bond_k2 = nullptr;
    double* d_bond_l0 = nullptr;
    int* d_ang[4] = {nullptr, nullptr, nullptr, nullptr};
    double* d_ang_k3 = nullptr;
    double* d_ang_cos0 = nullptr;
    double* d_ang_sin0 = nullptr;
    // pinned host
    unsigned* h_status = nullptr;
    // status word as of the start of the latest call's device work, written by
    // that call's first kernel into mapped pinned memory (d_seen is its device
    // address); read by dpd_engine_step without waiting
    unsigned* h_seen = nullptr;
    unsigned* d_seen = nullptr;
    // the value the device step counter holds once every queued step has run
    // (each step's k_update_mom advances it); INT64_MIN: unknown
    int64_t dev_step = INT64_MIN;
    double* h_obs = nullptr;
    // pinned staging for the host-built topology arrays (grown as needed)
    unsigned char* h_stage = nullptr;
    size_t cap_h_stage = 0;
    bool obs_valid = false;
    bool obs_has_virial = false;
    int64_t sample_period = 0;      // 0: sample at the last step of every call
    bool sampled = false;           // a sample step has run since the last upload
    int64_t last_sample_step = 0;

    std::vector<void*> allocations;

    // caller-provided stream (dpd_engine_set_stream) and kernel timing
    cudaStream_t user_stream = nullptr;
    bool profiling = false;
    struct ProfRec { int kernel; cudaEvent_t a, b; };
    std::vector<ProfRec> prof;          // recorded since profiling was switched on
    std::vector<cudaEvent_t> event_pool;

    cudaStream_t s() const { return user_stream ? user_stream : stream; }

    // captured multi-step sequences (DPD_GRAPHS=0 disables)
    struct Graph {
        int nsteps, parity;
        bool from_ahead, to_ahead;
        std::vector<char> samples;
        cudaStream_t stream;
        cudaGraphExec_t exec;
        int64_t launches;          // kernels per replay
    };
    std::vector<Graph> graphs;
    bool graphs_enabled = true;

    // pair-kernel launch shape (DPD_TUNE="hitcap=32,bps=8,carveout=50"; 0 = automatic)
    int sms = 148;
    int pair_hitcap = 32;
    int pair_bps = 0;          // resident blocks per SM for the persistent grid
    int pair_carveout = -1;    // preferred shared-memory carveout in percent, -1 = driver default
    int pair_scheme = DPD_PAIR_FULL_SHELL;   // DPD_PAIR_*: full shell (reproducible), half shell, staged half shell
    int pair_tile = kHalfBlock;              // beads per block of the half-shell kernel (64 or 128)
    bool pair_attr_set[2][2] = {{false, false}, {false, false}};   // [fp64][sample]; one box kind per engine
};

namespace {

int fail(dpd_engine* e, int code, const std::string& msg)
{
    if (e) e->err = msg;
    return code;
}

#define CU(call)                                                                            \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess)                                                              \
            return fail(e, DPD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

template <typename T>
int dalloc(dpd_engine* e, T** p, size_t count)
{
    void* q = nullptr;
    cudaError_t rc = cudaMalloc(&q, count ? count * sizeof(T) : sizeof(T));
    if (rc != cudaSuccess) return fail(e, DPD_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(rc));
    e->allocations.push_back(q);
    *p = static_cast<T*>(q);
    return DPD_OK;
}

void dfree(dpd_engine* e, void* p)
{
    if (!p) return;
    auto it = std::find(e->allocations.begin(), e->allocations.end(), p);
    if (it != e->allocations.end()) {
        cudaFree(p);
        e->allocations.erase(it);
    }
}

// Grows *p to hold count elements (allocating max(count, room) when it grows);
// sets *moved when the address changes.
template <typename T>
int ensure(dpd_engine* e, T** p, size_t& cap, size_t count, bool* moved, size_t room = 0)
{
    if (*p && count <= cap) return DPD_OK;
    dfree(e, *p);
    *p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(std::max<size_t>(count, room), 1);
    const int rc = dalloc(e, p, want);
    if (rc) return rc;
    cap = want;
    *moved = true;
    return DPD_OK;
}

// The allocation for count elements of a buffer whose count changes every
// upload (a slab): n_headroom times count.
size_t with_room(const dpd_engine* e, size_t count) { return (size_t)((double)count * e->n_headroom); }

size_t real_size(const dpd_engine* e) { return e->precision == DPD_PRECISION_FP64 ? sizeof(double) : sizeof(float); }

int check_launch(dpd_engine* e, const char* what)
{
    ++e->launches;
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess) return fail(e, DPD_E_CUDA, std::string(what) + ": " + cudaGetErrorString(rc));
    return DPD_OK;
}

// Host mirror of StepConst, the box table and the pair tables
// (CCNTCell::SetTimeStepConstants, CNTCell.cpp:180-203;
// sigma_ij = sqrt(gamma_ij) * sqrt(24 kT / dt), CNTCell.cpp:190,1220).
// Forget a drift done ahead by the last call (its arrival counts included),
// before anything that changes what that drift computed.
int drop_ahead(dpd_engine* e)
{
    if (!e->ahead_valid) return DPD_OK;
    CU(cudaMemsetAsync(e->d_count, 0, sizeof(int) * (size_t)e->ncell, e->s()));
    CU(cudaMemsetAsync(e->d_block_count, 0, sizeof(int) * (size_t)e->nchunk, e->s()));
    e->ahead_valid = false;
    return DPD_OK;
}

int push_constants(dpd_engine* e)
{
    int rc0;
    if ((rc0 = drop_ahead(e))) return rc0;   // the drift done ahead used the old constants
    const dpd_params& p = e->params;
    StepConst K{};
    K.dt = p.dt;
    K.halfdt = 0.5 * p.dt;
    K.halfdt2 = 0.5 * p.dt * p.dt;
    K.lamdt = p.lambda * p.dt;
    K.invrootdt = std::sqrt(24.0 * p.kT / p.dt);
    const Box& b0 = e->hboxes[0];
    for (int d = 0; d < 3; ++d) {
        K.nc[d] = b0.nc[d];
        K.w[d] = b0.w[d];
        K.L[d] = b0.L[d];
    }
    K.ntypes = e->ntypes;
    K.seed = b0.seed;
    const int m = e->ntypes * e->ntypes;
    const size_t nb = e->hboxes.size();
    std::vector<double> tab(3 * (size_t)m * nb);
    for (size_t bx = 0; bx < nb; ++bx) {
        double* t = tab.data() + 3 * (size_t)m * bx;
        e->hboxes[bx].tab = (int)(3 * (size_t)m * bx);
        for (int k = 0; k < m; ++k) {
            const double a = e->conservative_on ? e->box_a[bx * m + k] : 0.0;
            const double g = e->thermostat_on ? e->box_g[bx * m + k] : 0.0;
            t[k] = a;
            t[m + k] = g;
            t[2 * m + k] = std::sqrt(g) * K.invrootdt;
        }
    }
    CU(cudaStreamSynchronize(e->s()));   // tables may be in use by queued work
    CU(cudaMemcpy(e->d_K, &K, sizeof K, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(e->d_boxes, e->hboxes.data(), nb * sizeof(Box), cudaMemcpyHostToDevice));
    if (e->precision == DPD_PRECISION_FP64) {
        CU(cudaMemcpy(e->d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> tf(tab.begin(), tab.end());
        CU(cudaMemcpy(e->d_tab, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return DPD_OK;
}

// Single-bead sums of every box: one block per box over its contiguous slot
// range, fixed order (deterministic).  The virial is the per-bead stress of the
// latest sample step.
template <typename real>
__global__ void __launch_bounds__(256) k_box_sums(const Box* __restrict__ boxes, const int* __restrict__ start,
                                                  int n, const double* __restrict__ x, const double* __restrict__ v,
                                                  const real* __restrict__ stress, double* __restrict__ out)
{
    const Box& B = boxes[blockIdx.x];
    const int s0 = start[B.cell_base], s1 = start[B.cell_base + B.nc[0] * B.nc[1] * B.nc[2]];
    double acc[kObsTerms];
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) acc[q] = 0.0;
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const double xs[3] = {x[s], x[n + s], x[2 * n + s]};
        const double vs[3] = {v[s], v[n + s], v[2 * n + s]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            acc[d] += vs[d];
            acc[3 + d] += vs[d] * vs[d];
            acc[15 + d] += xs[d];
        }
        if (stress) {
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[6 + q] += (double)stress[q * n + s];
        }
        acc[18] += xs[1] * vs[2] - xs[2] * vs[1];
        acc[19] += -xs[0] * vs[2] + xs[2] * vs[0];
        acc[20] += xs[0] * vs[1] - xs[1] * vs[0];
    }
    __shared__ double red[8][kObsTerms];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) {
        double a = acc[q];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) red[wid][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < kObsTerms) {
        double a = 0.0;
        for (int w = 0; w < 8; ++w) a += red[w][threadIdx.x];
        out[blockIdx.x * kObsTerms + threadIdx.x] = a;
    }
}

cudaEvent_t take_event(dpd_engine* e)
{
    if (!e->event_pool.empty()) {
        cudaEvent_t ev = e->event_pool.back();
        e->event_pool.pop_back();
        return ev;
    }
    cudaEvent_t ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    return ev;
}

// Brackets one kernel launch with events when profiling is on.
struct Timed {
    dpd_engine* e;
    int kernel;
    cudaEvent_t a = nullptr;
    Timed(dpd_engine* eng, int k) : e(eng), kernel(k)
    {
        if (e->profiling && (a = take_event(e))) cudaEventRecord(a, e->s());
    }
    ~Timed()
    {
        if (!a) return;
        cudaEvent_t b = take_event(e);
        if (!b) { e->event_pool.push_back(a); return; }
        cudaEventRecord(b, e->s());
        e->prof.push_back({kernel, a, b});
    }
};

// The pair kernel variant for (box table, sample step, pair scheme).
template <typename real>
auto pair_kernel(bool multi, bool sample, int scheme, int tile)
{
    if (scheme == DPD_PAIR_STAGED)
        return multi ? (sample ? k_pair_forces_staged<real, true, true> : k_pair_forces_staged<real, false, true>)
                     : (sample ? k_pair_forces_staged<real, true, false> : k_pair_forces_staged<real, false, false>);
    if (scheme == DPD_PAIR_HALF_SHELL && tile == kPairBlock)
        return multi ? (sample ? k_pair_forces_half<real, true, true, kPairBlock>
                               : k_pair_forces_half<real, false, true, kPairBlock>)
                     : (sample ? k_pair_forces_half<real, true, false, kPairBlock>
                               : k_pair_forces_half<real, false, false, kPairBlock>);
    if (scheme == DPD_PAIR_HALF_SHELL)
        return multi ? (sample ? k_pair_forces_half<real, true, true> : k_pair_forces_half<real, false, true>)
                     : (sample ? k_pair_forces_half<real, true, false> : k_pair_forces_half<real, false, false>);
    return multi ? (sample ? k_pair_forces<real, true, true> : k_pair_forces<real, false, true>)
                 : (sample ? k_pair_forces<real, true, false> : k_pair_forces<real, false, false>);
}

// Dynamic shared memory of the engine's pair kernel.
template <typename real>
size_t pair_dyn_bytes(const dpd_engine* e, bool multi)
{
    if (e->pair_scheme == DPD_PAIR_STAGED) return StgLayout<real>(e->ntypes, e->pair_hitcap, multi).total;
    if (e->pair_scheme == DPD_PAIR_HALF_SHELL)
        return e->pair_tile == kPairBlock ? half_smem_bytes<real, kPairBlock>(e->ntypes, e->pair_hitcap, multi)
                                          : half_smem_bytes<real, kHalfBlock>(e->ntypes, e->pair_hitcap, multi);
    return pair_smem_bytes<real>(e->ntypes, e->pair_hitcap, multi);
}

// Dynamic shared memory and carveout of the pair kernel's variants (outside
// any stream capture).
template <typename real>
int set_pair_attributes(dpd_engine* e)
{
    const bool multi = e->hboxes.size() > 1;
    const int pv = sizeof(real) == 8 ? 1 : 0;
    for (int sv = 0; sv < 2; ++sv) {
        if (e->pair_attr_set[pv][sv]) continue;
        auto kern = pair_kernel<real>(multi, sv != 0, e->pair_scheme, e->pair_tile);
        const size_t dyn = pair_dyn_bytes<real>(e, multi);
        CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        if (e->pair_carveout >= 0)
            CU(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, e->pair_carveout));
        e->pair_attr_set[pv][sv] = true;
    }
    return DPD_OK;
}

// A step kernel launched with programmatic stream serialization (when the
// engine allows it): it may be scheduled while its predecessor drains and
// waits in pdl_wait() for that predecessor's results.
template <typename... KArgs, typename... Args>
cudaError_t launch_step(const dpd_engine* e, void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem,
                        cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = e->pdl ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Slice-profile parameters of the engine (S = 0 when off).
SliceParams slice_params(const dpd_engine* e)
{
    SliceParams sp{};
    if (!e->slice_S) return sp;
    const int S = e->slice_S, KT = e->ntypes * e->ntypes;
    sp.S = S;
    sp.width = e->hboxes[0].L[2] / (double)S;   // m_GridZCellWidth, Monitor.cpp:247
    sp.inv = 1.0 / sp.width;                    // m_invSliceWidth, Monitor.cpp:2185
    sp.nbt = e->slice_nbt;
    sp.nbpt = e->slice_nbpt;
    sp.pair = e->d_slice;
    sp.bond = e->d_slice + (size_t)S * KT * 9;
    sp.bondpair = sp.bond + (size_t)S * e->slice_nbt * 9;
    sp.bond_type = e->d_slice_bt;
    sp.bondpair_type = e->d_slice_bpt;
    return sp;
}

size_t slice_bins(const dpd_engine* e)
{
    return (size_t)e->slice_S * 9 * ((size_t)e->ntypes * e->ntypes + e->slice_nbt + e->slice_nbpt);
}

constexpr size_t kSliceSmemMax = 160 * 1024;   // block-private pair bins up to this size

// One timestep.  The first step of a call starts with k_update_pos; the
// others had their UpdatePos fused into the k_update_mom before them, which
// does so for every step but the last of the call.
template <typename real>
int queue_step(dpd_engine* e, bool sample, bool first, bool last, bool from_ahead, bool to_ahead)
{
    typedef typename Vec4<real>::type V4;
    const int n = (int)e->n;
    const int a = e->cur, b = 1 - e->cur;
    const int nb = blocks_for(n, kThreads);
    cudaStream_t st = e->s();
    int rc;
    // the first step of a call drifts here unless the previous call's last
    // k_update_mom did it already (from_ahead: x, img, cell from the ahead buffers)
    const bool ahead_in = first && from_ahead;
    double* x_in = ahead_in ? e->d_xa : e->d_x[a];
    uint32_t* img_in = ahead_in ? e->d_imga : e->d_img[a];
    int* cell_in = ahead_in ? e->d_cella : e->d_cell[a];
    // The full shell keeps every cell's beads in the order of their previous
    // slots (bitwise reproducible forces): arrival ranks, a permutation, then a
    // gather.  The half-shell schemes add forces with atomics in no fixed order
    // anyway: their beads are scattered into the cells by k_gather, one kernel
    // less, and without ranks the counting atomics return nothing.
    const bool stable = e->pair_scheme == DPD_PAIR_FULL_SHELL;
    int* rank_out = stable ? e->d_rank : nullptr;
    if (first && !from_ahead) {
        {
            Timed t(e, DPD_KERNEL_UPDATE_POS);
            CU(launch_step(e, k_update_pos<real>, nb, kThreads, 0, st, n, e->d_K, e->d_boxes, e->d_x[a], e->d_v[a],
                           (const real*)e->d_F, e->d_tf[a], e->d_img[a], e->d_cell[a], rank_out, e->d_count,
                           e->d_block_count, e->d_status, first ? e->d_seen : (unsigned*)nullptr));
        }
        if ((rc = check_launch(e, "k_update_pos"))) return rc;
    }
    {
        Timed t(e, DPD_KERNEL_SCAN_CELLS);
        // the call's first kernel publishes the status word (k_update_pos when it runs)
        CU(launch_step(e, k_scan_cells, e->nchunk, kScanThreads, 0, st, (int)e->ncell, n, e->d_count,
                       e->d_block_count, e->d_start, (const unsigned*)e->d_status,
                       (first && from_ahead) ? e->d_seen : (unsigned*)nullptr, stable ? 1 : 0));
    }
    if ((rc = check_launch(e, "k_scan_cells"))) return rc;
    if (stable) {
        {
            Timed t(e, DPD_KERNEL_PERMUTE);
            CU(launch_step(e, k_permute, blocks_for(std::max<int64_t>(n, e->nchunk), kThreads), kThreads, 0, st, n,
                           e->nchunk, cell_in, e->d_rank, e->d_start, e->d_perm, e->d_block_count));
        }
        if ((rc = check_launch(e, "k_permute"))) return rc;
    }
    {
        Timed t(e, DPD_KERNEL_GATHER);
        // the half-shell schemes accumulate into F with atomics: k_gather clears it
        const int zero_F = stable ? 0 : 1;
        CU(launch_step(e, k_gather<real>, blocks_for(std::max<int64_t>(n, stable ? 0 : e->nchunk), kThreads), kThreads,
                       0, st, n, e->d_K, e->d_boxes, e->d_perm, e->d_start, x_in, e->d_v[a], (real*)e->d_F,
                       e->d_bid[a], e->d_tf[a], img_in, cell_in, e->d_x[b], e->d_v[b], (real*)e->d_Fold,
                       e->d_bid[b], e->d_tf[b], e->d_img[b], e->d_cell[b], e->d_pid[a], e->d_pid[b], (V4*)e->d_pos4,
                       (V4*)e->d_vel4, e->d_ubuf, (const double*)(e->off_active ? e->d_off : nullptr), zero_F,
                       (int)e->nchunk, e->d_block_count, stable ? (int*)nullptr : e->d_count));
    }
    if ((rc = check_launch(e, "k_gather"))) return rc;
    // bond and bond-pair forces: a branch beside the pair kernel (on the
    // launching stream itself while profiling, so every kernel is timed)
    const bool slices = sample && e->slice_S > 0;
    const SliceParams sp = slices ? slice_params(e) : SliceParams{};
    if (slices) CU(cudaMemsetAsync(e->d_slice, 0, slice_bins(e) * sizeof(double), st));
    const Topology topo{e->d_csr_ptr, e->d_csr_term, e->d_bond_h, e->d_bond_t, e->d_bond_k2, e->d_bond_l0,
                        e->d_ang[0], e->d_ang[1], e->d_ang[2], e->d_ang[3], e->d_ang_k3, e->d_ang_cos0,
                        e->d_ang_sin0, e->d_ubuf, sp};
    const bool fork = e->nbb > 0 && !e->profiling;
    if (e->nbb > 0) {
        cudaStream_t bst = st;
        if (fork) {
            CU(cudaEventRecord(e->ev_fork, st));
            CU(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
            bst = e->side;
        }
        {
            Timed t(e, DPD_KERNEL_BONDED);
            auto kern = sample ? k_bonds<true> : k_bonds<false>;
            kern<<<blocks_for(e->nbb, kThreads), kThreads, 0, bst>>>((int)e->nbb, n, e->d_bb, topo, e->d_Fb, e->d_Sb);
        }
        if ((rc = check_launch(e, "k_bonds"))) return rc;
        if (slices && e->topo_nb + e->topo_na > 0) {
            // the profile's bond and bond-pair part, bonds and bond pairs in whole warps each
            Timed t(e, DPD_KERNEL_BONDED);
            const int64_t threads = ((e->topo_nb + 31) & ~(int64_t)31) + ((e->topo_na + 31) & ~(int64_t)31);
            k_bonded_slices<<<blocks_for(threads, kThreads), kThreads, 0, bst>>>((int)e->topo_nb, (int)e->topo_na,
                                                                                 topo);
            if ((rc = check_launch(e, "k_bonded_slices"))) return rc;
        }
        if (fork) CU(cudaEventRecord(e->ev_join, e->side));
    }
    {
        const bool multi = e->hboxes.size() > 1;
        auto kern = pair_kernel<real>(multi, sample, e->pair_scheme, e->pair_tile);
        const size_t dyn = pair_dyn_bytes<real>(e, multi);
        if ((rc = set_pair_attributes<real>(e))) return rc;
        // the half shell accumulates into F with atomics
        // the half-shell kernels add each owner's pair virial in pieces
        if (sample && e->pair_scheme != DPD_PAIR_FULL_SHELL)
            CU(cudaMemsetAsync(e->d_stress, 0, (size_t)9 * n * sizeof(real), st));
        // one tile per block by default; bps > 0 selects a persistent grid of
        // sms * bps blocks walking contiguous tiles
        const int block = e->pair_scheme == DPD_PAIR_HALF_SHELL ? e->pair_tile : kPairBlock;
        const int tiles = blocks_for(n, block);
        const int tpb = e->pair_bps > 0 ? std::max(1, blocks_for(tiles, (int64_t)e->sms * e->pair_bps)) : 1;
        Timed t(e, DPD_KERNEL_PAIR_FORCES);
        CU(launch_step(e, kern, blocks_for(tiles, tpb), block, dyn, st, n, e->d_K, e->d_boxes, e->d_step,
                       (const real*)e->d_tab, e->d_cell[b], e->d_start, (const V4*)e->d_pos4, (const V4*)e->d_vel4,
                       (real*)e->d_F, (real*)e->d_stress, e->pair_hitcap, tpb, e->d_status,
                       (const double*)e->d_x[b]));
    }
    if ((rc = check_launch(e, "k_pair_forces"))) return rc;
    if (slices) {
        const int KT = e->ntypes * e->ntypes;
        const int sb = slice_smem_bytes<real>(e->slice_S, KT, true) <= kSliceSmemMax;
        const size_t smem = slice_smem_bytes<real>(e->slice_S, KT, sb != 0);
        Timed t(e, DPD_KERNEL_SLICES);
        // pairs listed by the test, then evaluated from the list; the
        // one-kernel form runs instead when the list cannot hold them
        const SliceList L{e->d_slice_list, e->d_slice_cnt, (int)std::min<size_t>(e->cap_slice_list, INT_MAX)};
        const bool listed = e->d_slice_list && e->cap_slice_list >= (size_t)kSliceListPerBead * (size_t)n;
        if (listed) {
            CU(cudaMemsetAsync(e->d_slice_cnt, 0, 2 * sizeof(unsigned), st));
            CU(launch_step(e, k_slice_pairs<real>, e->sms * 4, kSliceBlock, slice_smem_bytes<real>(e->slice_S, KT, false),
                           st, n, e->d_K, e->d_boxes, e->d_step, (const real*)e->d_tab, e->d_cell[b], e->d_start,
                           (const V4*)e->d_pos4, (const V4*)e->d_vel4, (const double*)e->d_x[b], sp, 0, L,
                           (int)kSliceList));
            if ((rc = check_launch(e, "k_slice_pairs"))) return rc;
            const int nbins = e->slice_S * KT * 9;
            const int eblocks = e->sms * kSliceEvalBlocksPerSM;
            CU(launch_step(e, k_slice_eval<real>, eblocks, kSliceEvalBlock,
                           slice_eval_smem_bytes<real>(e->slice_S, KT, sb != 0), st, n, e->d_K, e->d_boxes, e->d_step,
                           (const real*)e->d_tab, (const V4*)e->d_pos4, (const V4*)e->d_vel4,
                           (const double*)e->d_x[b], sp, sb, L, (real*)e->d_slice_part));
            if ((rc = check_launch(e, "k_slice_eval"))) return rc;
            CU(launch_step(e, k_slice_sum<real>, blocks_for(nbins, 32), 256, 0, st, nbins, sb ? eblocks : 0,
                           (const real*)e->d_slice_part, (const unsigned*)e->d_slice_cnt, sp.pair));
            if ((rc = check_launch(e, "k_slice_sum"))) return rc;
        }
        CU(launch_step(e, k_slice_pairs<real>, e->sms * 4, kSliceBlock, smem, st, n, e->d_K, e->d_boxes, e->d_step,
                       (const real*)e->d_tab, e->d_cell[b], e->d_start, (const V4*)e->d_pos4, (const V4*)e->d_vel4,
                       (const double*)e->d_x[b], sp, sb, L, (int)(listed ? kSliceFallback : kSliceOne)));
        if ((rc = check_launch(e, "k_slice_pairs"))) return rc;
        e->slice_sampled = true;
    }
    if (fork) CU(cudaStreamWaitEvent(st, e->ev_join, 0));
    {
        Timed t(e, DPD_KERNEL_UPDATE_MOM);
        // the next step's drift: in place between the steps of a call, into
        // the ahead buffers after the last one (or not at all)
        const bool pos = !last || to_ahead;
        auto kern = sample ? (pos ? k_update_mom<real, true, true> : k_update_mom<real, true, false>)
                           : (pos ? k_update_mom<real, false, true> : k_update_mom<real, false, false>);
        double* xo = last ? e->d_xa : e->d_x[b];
        uint32_t* imgo = last ? e->d_imga : e->d_img[b];
        int* cello = last ? e->d_cella : e->d_cell[b];
        CU(launch_step(e, kern, nb, kThreads, 0, st, n, e->d_K, e->d_boxes, e->d_step, (const double*)e->d_x[b],
                       e->d_v[b], (real*)e->d_F, (const real*)e->d_Fold, e->d_bid[b], e->d_tf[b],
                       (const double4*)e->d_Fb, (const double*)e->d_Sb, (real*)e->d_stress, e->d_partials,
                       (const uint32_t*)e->d_img[b], (const int*)e->d_cell[b], rank_out, e->d_count,
                       e->d_block_count, e->d_status, xo, imgo, cello));
    }
    if ((rc = check_launch(e, "k_update_mom"))) return rc;
    if (sample) {
        {
            Timed t(e, DPD_KERNEL_REDUCE_OBS);
            CU(launch_step(e, k_reduce_obs, 1, 32 * kObsTerms, 0, st, nb, (const double*)e->d_partials, e->d_obs));
        }
        if ((rc = check_launch(e, "k_reduce_obs"))) return rc;
    }
    e->cur = b;
    return DPD_OK;
}

// "hitcap=32,bps=8,carveout=50,half=1,scheme=2": pair-kernel hit-list
// capacity (8..64), resident blocks per SM for its persistent grid, preferred
// shared-memory carveout (%), half-shell kernel, pair scheme (DPD_PAIR_*).
void parse_tuning(dpd_engine* e, const char* spec)
{
    std::string str(spec);
    size_t pos = 0;
    while (pos < str.size()) {
        size_t end = str.find(',', pos);
        if (end == std::string::npos) end = str.size();
        const std::string item = str.substr(pos, end - pos);
        const size_t eq = item.find('=');
        if (eq != std::string::npos) {
            const std::string key = item.substr(0, eq);
            const int val = atoi(item.c_str() + eq + 1);
            if (key == "hitcap") e->pair_hitcap = std::min(std::max(val, 8), (int)kHitCapMax);
            else if (key == "bps") e->pair_bps = std::max(val, 0);
            else if (key == "carveout") e->pair_carveout = std::min(std::max(val, -1), 100);
            else if (key == "half") e->pair_scheme = val ? DPD_PAIR_HALF_SHELL : DPD_PAIR_FULL_SHELL;
            else if (key == "scheme" && val >= DPD_PAIR_FULL_SHELL && val <= DPD_PAIR_STAGED) e->pair_scheme = val;
            else if (key == "tile" && (val == kHalfBlock || val == kPairBlock)) e->pair_tile = val;
            else if (key == "ahead") e->ahead_enabled = val != 0;
            else if (key == "pdl") e->pdl = val != 0;
        }
        pos = end + 1;
    }
}

void drop_graphs(dpd_engine* e)
{
    for (auto& g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
}

void release_topology(dpd_engine* e)
{
    int** ip[] = {&e->d_csr_ptr, &e->d_csr_term, &e->d_bond_h, &e->d_bond_t,
                  &e->d_ang[0], &e->d_ang[1], &e->d_ang[2], &e->d_ang[3]};
    for (auto q : ip) { dfree(e, *q); *q = nullptr; }
    double** dp[] = {&e->d_bond_k2, &e->d_bond_l0, &e->d_ang_k3, &e->d_ang_cos0, &e->d_ang_sin0};
    for (auto q : dp) { dfree(e, *q); *q = nullptr; }
    e->cap_csr_ptr = e->cap_csr_term = e->cap_bond = e->cap_ang = 0;
    e->topo_in.valid = false;
}

// Empty topology: csr_ptr all zero.  With keep_bonded (same bead count as
// before) the bonded branch keeps its bead list and stays in the captured
// graphs: with no terms it writes zero bonded forces, which k_update_mom
// ignores for beads without kFlagBonded (all of them after a bead upload).
int empty_topology(dpd_engine* e, bool keep_bonded)
{
    bool moved = false;
    int rc;
    if ((rc = ensure(e, &e->d_csr_ptr, e->cap_csr_ptr, (size_t)e->n + 1, &moved, with_room(e, (size_t)e->n) + 1)))
        return rc;
    CU(cudaMemsetAsync(e->d_csr_ptr, 0, sizeof(int) * ((size_t)e->n + 1), e->s()));
    if (moved || (e->nbb && !keep_bonded)) {
        drop_graphs(e);
        e->nbb = 0;
    }
    if (moved || !keep_bonded) e->topo_in.valid = false;
    e->topo_nb = e->topo_na = 0;
    return DPD_OK;
}

// The host copies of the bead ids and types, fetched after an upload from
// device memory (d_prev_id / d_prev_type hold the last upload's, upload order).
int host_ids(dpd_engine* e)
{
    if (!e->host_ids_stale) return DPD_OK;
    const size_t n = (size_t)e->n;
    e->h_id.resize(n);
    e->h_type.resize(n);
    CU(cudaMemcpyAsync(e->h_id.data(), e->d_prev_id, n * sizeof(int64_t), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaMemcpyAsync(e->h_type.data(), e->d_prev_type, n * sizeof(int), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    e->host_ids_stale = false;
    return DPD_OK;
}

}  // namespace

// ===================================================================== C ABI

extern "C" {

static bool box_ok(int32_t nx, int32_t ny, int32_t nz, double wx, double wy, double wz)
{
    return nx >= 3 && ny >= 3 && nz >= 3 && wx >= 1.0 && wy >= 1.0 && wz >= 1.0;
}

// Shared by the single-box and the batch constructors.
static int create_impl(const dpd_params* p, int32_t nboxes, const dpd_box* bx, dpd_engine** out)
{
    dpd_engine* e = nullptr;
    if (!out) return DPD_E_ARG;
    *out = nullptr;
    if (!p || !(p->dt > 0.0) || p->lambda < 0.0 || p->kT < 0.0 || p->ntypes < 1 || p->ntypes > kMaxTypes ||
        (p->precision != DPD_PRECISION_MIXED && p->precision != DPD_PRECISION_FP64) || nboxes < 1 ||
        nboxes > kMaxBoxes || !bx)
        return DPD_E_ARG;
    int64_t ncell = 0;
    for (int32_t k = 0; k < nboxes; ++k) {
        if (!box_ok(bx[k].nx, bx[k].ny, bx[k].nz, bx[k].wx, bx[k].wy, bx[k].wz) || !bx[k].a || !bx[k].gamma)
            return DPD_E_ARG;
        ncell += (int64_t)bx[k].nx * bx[k].ny * bx[k].nz;
    }
    if (ncell > (int64_t)1 << 30) return DPD_E_ARG;
    e = new (std::nothrow) dpd_engine();
    if (!e) return DPD_E_NOMEM;
    e->params = *p;
    e->params.a = nullptr;
    e->params.gamma = nullptr;
    e->params.nx = bx[0].nx; e->params.ny = bx[0].ny; e->params.nz = bx[0].nz;
    e->params.wx = bx[0].wx; e->params.wy = bx[0].wy; e->params.wz = bx[0].wz;
    e->params.seed = bx[0].seed;
    e->precision = p->precision;
    e->ntypes = p->ntypes;
    const int m = p->ntypes * p->ntypes;
    int64_t base = 0;
    for (int32_t k = 0; k < nboxes; ++k) {
        Box b{};
        b.nc[0] = bx[k].nx; b.nc[1] = bx[k].ny; b.nc[2] = bx[k].nz;
        b.w[0] = bx[k].wx; b.w[1] = bx[k].wy; b.w[2] = bx[k].wz;
        for (int d = 0; d < 3; ++d) b.L[d] = (double)b.nc[d] * b.w[d];
        b.cell_base = (int)base;
        b.seed = bx[k].seed;
        set_cell_division(b);
        base += (int64_t)b.nc[0] * b.nc[1] * b.nc[2];
        e->hboxes.push_back(b);
        e->box_a.insert(e->box_a.end(), bx[k].a, bx[k].a + m);
        e->box_g.insert(e->box_g.end(), bx[k].gamma, bx[k].gamma + m);
    }
    e->a.assign(bx[0].a, bx[0].a + m);
    e->gamma.assign(bx[0].gamma, bx[0].gamma + m);
    e->ncell = ncell;
    e->nchunk = (int)((ncell + kScanChunk - 1) / kScanChunk);
    int rc = DPD_OK;
    do {
        if (p->device >= 0) {
            if (cudaSetDevice(p->device) != cudaSuccess) { rc = fail(e, DPD_E_CUDA, "cudaSetDevice failed"); break; }
            e->device = p->device;
        } else if (cudaGetDevice(&e->device) != cudaSuccess) {
            rc = fail(e, DPD_E_CUDA, "no CUDA device");
            break;
        }
        cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device);
        if (const char* tune = getenv("DPD_TUNE")) parse_tuning(e, tune);
        if (const char* g = getenv("DPD_GRAPHS")) e->graphs_enabled = atoi(g) != 0;
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming) != cudaSuccess) {
            rc = fail(e, DPD_E_CUDA, "cudaStreamCreate failed");
            break;
        }
        if ((rc = dalloc(e, &e->d_K, 1))) break;
        if ((rc = dalloc(e, &e->d_boxes, (size_t)nboxes))) break;
        if ((rc = dalloc(e, &e->d_box_obs, (size_t)nboxes * kObsTerms))) break;
        // a single box may later grow its type table (AddDPDBeadType); a batch keeps its types
        const size_t tab_m = nboxes == 1 ? (size_t)kMaxTypes * kMaxTypes : (size_t)m;
        if ((rc = dalloc(e, (char**)&e->d_tab, 3 * tab_m * nboxes * sizeof(double)))) break;
        if ((rc = dalloc(e, &e->d_step, 1))) break;
        if ((rc = dalloc(e, &e->d_status, 1))) break;
        if ((rc = dalloc(e, &e->d_count, (size_t)ncell))) break;
        if ((rc = dalloc(e, &e->d_start, (size_t)ncell + 1))) break;
        if ((rc = dalloc(e, &e->d_block_count, (size_t)e->nchunk))) break;
        if ((rc = dalloc(e, &e->d_obs, kObsTerms))) break;
        if ((rc = dalloc(e, &e->d_renorm, kObsTerms))) break;
        if (cudaMallocHost(&e->h_status, sizeof(unsigned)) != cudaSuccess ||
            cudaMallocHost(&e->h_obs, kObsTerms * sizeof(double)) != cudaSuccess ||
            cudaHostAlloc(&e->h_seen, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess) {
            rc = fail(e, DPD_E_NOMEM, "cudaMallocHost failed");
            break;
        }
        *e->h_seen = 0u;
        if (cudaHostGetDevicePointer((void**)&e->d_seen, e->h_seen, 0) != cudaSuccess || !e->d_seen) {
            rc = fail(e, DPD_E_CUDA, "cudaHostGetDevicePointer failed");
            break;
        }
        if (cudaMemset(e->d_status, 0, sizeof(unsigned)) != cudaSuccess ||
            cudaMemset(e->d_count, 0, sizeof(int) * ncell) != cudaSuccess ||
            cudaMemset(e->d_block_count, 0, sizeof(int) * e->nchunk) != cudaSuccess ||
            cudaMemset(e->d_step, 0, sizeof(int64_t)) != cudaSuccess) {
            rc = fail(e, DPD_E_CUDA, "cudaMemset failed");
            break;
        }
        if ((rc = push_constants(e))) break;
    } while (0);
    if (rc != DPD_OK) {
        // keep the message readable through a half-built engine
        fprintf(stderr, "dpd_engine_create: %s\n", e->err.c_str());
        dpd_engine_destroy(e);
        return rc;
    }
    *out = e;
    return DPD_OK;
}

int dpd_engine_create(const dpd_params* p, dpd_engine** out)
{
    if (!out) return DPD_E_ARG;
    *out = nullptr;
    if (!p || !p->a || !p->gamma) return DPD_E_ARG;
    const dpd_box b{p->nx, p->ny, p->nz, p->wx, p->wy, p->wz, p->a, p->gamma, p->seed};
    return create_impl(p, 1, &b, out);
}

int dpd_batch_create(const dpd_params* shared, int32_t nboxes, const dpd_box* boxes, dpd_engine** out)
{
    return create_impl(shared, nboxes, boxes, out);
}

void dpd_engine_destroy(dpd_engine* e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->user_stream) cudaStreamSynchronize(e->user_stream);
    drop_graphs(e);
    for (auto& r : e->prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (cudaEvent_t ev : e->event_pool) cudaEventDestroy(ev);
    for (void* p : e->allocations) cudaFree(p);
    e->allocations.clear();
    if (e->slab) {
        if (e->slab->h_sizes) cudaFreeHost(e->slab->h_sizes);
        delete e->slab;
    }
    if (e->h_status) cudaFreeHost(e->h_status);
    if (e->h_obs) cudaFreeHost(e->h_obs);
    if (e->h_stage) cudaFreeHost(e->h_stage);
    if (e->h_seen) cudaFreeHost(e->h_seen);
    if (e->side) cudaStreamSynchronize(e->side);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    if (e->side) cudaStreamDestroy(e->side);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* dpd_engine_last_error(const dpd_engine* e) { return e ? e->err.c_str() : "null engine"; }

int dpd_engine_set_launch_shape(dpd_engine* e, int32_t hitcap, int32_t persistent_blocks_per_sm,
                                int32_t smem_carveout)
{
    if (!e) return DPD_E_ARG;
    if (hitcap < 8 || hitcap > kHitCapMax || persistent_blocks_per_sm < 0 || smem_carveout < -1 ||
        smem_carveout > 100)
        return fail(e, DPD_E_ARG, "launch shape out of range");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    e->pair_hitcap = hitcap;
    e->pair_bps = persistent_blocks_per_sm;
    e->pair_carveout = smem_carveout;
    memset(e->pair_attr_set, 0, sizeof e->pair_attr_set);
    drop_graphs(e);
    return DPD_OK;
}

int dpd_engine_set_pair_tile(dpd_engine* e, int32_t beads_per_block)
{
    if (!e) return DPD_E_ARG;
    if (beads_per_block == 0) beads_per_block = kHalfBlock;
    if (beads_per_block != kHalfBlock && beads_per_block != kPairBlock)
        return fail(e, DPD_E_ARG, "half-shell tiles hold 64 or 128 beads");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    e->pair_tile = beads_per_block;
    memset(e->pair_attr_set, 0, sizeof e->pair_attr_set);
    drop_graphs(e);
    return DPD_OK;
}

int dpd_engine_set_pair_scheme(dpd_engine* e, int32_t scheme)
{
    if (!e) return DPD_E_ARG;
    if (scheme != DPD_PAIR_FULL_SHELL && scheme != DPD_PAIR_HALF_SHELL && scheme != DPD_PAIR_STAGED)
        return fail(e, DPD_E_ARG, "unknown pair scheme");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    // a drift done ahead counted arrivals for the old scheme's gather (ranks or not)
    if (int rc0 = drop_ahead(e)) return rc0;
    e->pair_scheme = scheme;
    memset(e->pair_attr_set, 0, sizeof e->pair_attr_set);
    drop_graphs(e);
    return DPD_OK;
}

int dpd_engine_set_sample_period(dpd_engine* e, int64_t period)
{
    if (!e) return DPD_E_ARG;
    if (period < 0) return fail(e, DPD_E_ARG, "negative sample period");
    e->sample_period = period;
    return DPD_OK;
}

int dpd_engine_set_stream(dpd_engine* e, void* cuda_stream)
{
    if (!e) return DPD_E_ARG;
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));   // finish work queued on the old stream
    e->user_stream = static_cast<cudaStream_t>(cuda_stream);
    drop_graphs(e);
    return DPD_OK;
}

int dpd_engine_profile(dpd_engine* e, int32_t on)
{
    if (!e) return DPD_E_ARG;
    CU(cudaSetDevice(e->device));
    if (on) {
        CU(cudaStreamSynchronize(e->s()));
        for (auto& r : e->prof) { e->event_pool.push_back(r.a); e->event_pool.push_back(r.b); }
        e->prof.clear();
    }
    e->profiling = on != 0;
    return DPD_OK;
}

int dpd_engine_profile_read(dpd_engine* e, double* total_ms, int64_t* launches)
{
    if (!e) return DPD_E_ARG;
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    double ms[DPD_NUM_KERNELS] = {0};
    int64_t cnt[DPD_NUM_KERNELS] = {0};
    for (auto& r : e->prof) {
        float t = 0.f;
        CU(cudaEventElapsedTime(&t, r.a, r.b));
        if (r.kernel >= 0 && r.kernel < DPD_NUM_KERNELS) {
            ms[r.kernel] += t;
            cnt[r.kernel] += 1;
        }
    }
    for (int k = 0; k < DPD_NUM_KERNELS; ++k) {
        if (total_ms) total_ms[k] = ms[k];
        if (launches) launches[k] = cnt[k];
    }
    return DPD_OK;
}

int64_t dpd_engine_launch_count(const dpd_engine* e) { return e ? e->launches : -1; }

// Staging buffers of a bead upload; layout in doubles: x, unPBC, v, F (3n
// each, xyz interleaved, bead order), id (n int64), then int type[n], box[n]
// and the movable bytes.
static int stage_buffers(dpd_engine* e, int64_t n)
{
    int rc;
    bool smoved = false;
    // room for the bead counts of the next uploads too when they change every step (a slab)
    const size_t m = (size_t)n;
    if ((rc = ensure(e, &e->d_up, e->cap_up, 15 * m + 8, &smoved, 15 * with_room(e, m) + 8))) return rc;
    if ((rc = ensure(e, &e->d_up_cell, e->cap_up_cell, m, &smoved, with_room(e, m)))) return rc;
    if ((rc = ensure(e, &e->d_up_img, e->cap_up_img, m, &smoved, with_room(e, m)))) return rc;
    if ((rc = ensure(e, &e->d_up_off, e->cap_up_off, 3 * m, &smoved, 3 * with_room(e, m)))) return rc;
    if ((rc = ensure(e, &e->d_up_perm, e->cap_up_perm, m, &smoved, with_room(e, m)))) return rc;
    if ((rc = ensure(e, &e->d_up_err, e->cap_up_err, (size_t)kUpErrors + 2 + kMaxTypes, &smoved))) return rc;
    bool pmoved = false;
    if ((rc = ensure(e, &e->d_prev_id, e->cap_prev_id, m, &pmoved, with_room(e, m)))) return rc;
    if ((rc = ensure(e, &e->d_prev_type, e->cap_prev_type, m, &pmoved, with_room(e, m)))) return rc;
    if (pmoved) e->prev_n = -1;
    return DPD_OK;
}

static int upload_staged(dpd_engine* e, int64_t n, const int32_t* box, const int64_t* id, const int32_t* type,
                         const UploadIn& in);

// The per-bead state buffers for n beads: (re)allocated when too small
// (strides follow the bead count, so smaller counts fit; n_headroom leaves
// room for counts that change every upload); new addresses or another bead
// count invalidate the captured graphs.
static int ensure_beads(dpd_engine* e, int64_t n)
{
    if (n != e->n) drop_graphs(e);
    if (n > e->cap_n) {
        // a slab keeps the whole box's topology arrays across its uploads
        if (!e->slab) release_topology(e);
        void** bufs[] = {(void**)&e->d_x[0], (void**)&e->d_x[1], (void**)&e->d_v[0], (void**)&e->d_v[1],
                         (void**)&e->d_bid[0], (void**)&e->d_bid[1], (void**)&e->d_tf[0], (void**)&e->d_tf[1],
                         (void**)&e->d_img[0], (void**)&e->d_img[1], (void**)&e->d_cell[0], (void**)&e->d_cell[1],
                         &e->d_F, &e->d_Fold, &e->d_stress, &e->d_pos4, &e->d_vel4, (void**)&e->d_rank,
                         (void**)&e->d_perm, (void**)&e->d_pid[0], (void**)&e->d_pid[1], (void**)&e->d_pid_of,
                         (void**)&e->d_partials,
                         (void**)&e->d_out, (void**)&e->d_out_cell, (void**)&e->d_xa, (void**)&e->d_imga,
                         (void**)&e->d_cella};
        for (auto q : bufs) { dfree(e, *q); *q = nullptr; }
        const size_t rs = real_size(e);
        const int64_t cap = std::max<int64_t>(n, (int64_t)((double)n * e->n_headroom));
        e->cap_n = 0;
        int rc;
        if ((rc = dalloc(e, &e->d_xa, 3 * (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_imga, (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_cella, (size_t)cap))) return rc;
        for (int k = 0; k < 2; ++k) {
            if ((rc = dalloc(e, &e->d_x[k], 3 * (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_v[k], 3 * (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_bid[k], (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_tf[k], (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_img[k], (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_cell[k], (size_t)cap))) return rc;
            if ((rc = dalloc(e, &e->d_pid[k], (size_t)cap))) return rc;
        }
        if ((rc = dalloc(e, (char**)&e->d_F, 3 * rs * (size_t)cap))) return rc;
        if ((rc = dalloc(e, (char**)&e->d_Fold, 3 * rs * (size_t)cap))) return rc;
        if ((rc = dalloc(e, (char**)&e->d_stress, 9 * rs * (size_t)cap))) return rc;
        if ((rc = dalloc(e, (char**)&e->d_pos4, 4 * rs * (size_t)cap))) return rc;
        if ((rc = dalloc(e, (char**)&e->d_vel4, 4 * rs * (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_rank, (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_perm, (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_pid_of, (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_partials, (size_t)blocks_for(cap, kThreads) * kObsTerms))) return rc;
        if ((rc = dalloc(e, &e->d_out, 21 * (size_t)cap))) return rc;
        if ((rc = dalloc(e, &e->d_out_cell, (size_t)cap))) return rc;
        e->cap_n = cap;
    }
    return DPD_OK;
}


static int upload_impl(dpd_engine* e, int64_t n, const int32_t* box, const int64_t* id, const int32_t* type,
                       const uint8_t* movable, const double* x3, const double* unpbc3, const double* v3,
                       const double* f3)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "a slab's beads come from its exchange (dpd_engine_slab_unpack)");
    if (n < 1 || n > ((int64_t)1 << 30) || !id || !type || !x3 || !v3) return fail(e, DPD_E_ARG, "bad bead arrays");
    if (!box && e->hboxes.size() > 1) return fail(e, DPD_E_ARG, "a batch needs the box of every bead");
    CU(cudaSetDevice(e->device));
    if (int rc0 = drop_ahead(e)) return rc0;   // the new state replaces the drifted one
    CU(cudaStreamSynchronize(e->s()));
    cudaStream_t st = e->s();
    // the caller's arrays, copied as they are (pinned buffers make these DMA
    // copies) into the staging buffers
    int rc;
    if ((rc = stage_buffers(e, n))) return rc;
    double* up = e->d_up;
    int* upi = reinterpret_cast<int*>(up + 13 * (size_t)n);
    unsigned char* upm = reinterpret_cast<unsigned char*>(upi + 2 * (size_t)n);
    const size_t v3b = 3 * sizeof(double) * (size_t)n;
    UploadIn in{};
    in.x = up;
    CU(cudaMemcpyAsync(up, x3, v3b, cudaMemcpyHostToDevice, st));
    if (unpbc3) { in.u = up + 3 * (size_t)n; CU(cudaMemcpyAsync(up + 3 * (size_t)n, unpbc3, v3b, cudaMemcpyHostToDevice, st)); }
    in.v = up + 6 * (size_t)n;
    CU(cudaMemcpyAsync(up + 6 * (size_t)n, v3, v3b, cudaMemcpyHostToDevice, st));
    if (f3) { in.f = up + 9 * (size_t)n; CU(cudaMemcpyAsync(up + 9 * (size_t)n, f3, v3b, cudaMemcpyHostToDevice, st)); }
    in.id = reinterpret_cast<const int64_t*>(up + 12 * (size_t)n);
    CU(cudaMemcpyAsync(up + 12 * (size_t)n, id, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
    in.type = upi;
    CU(cudaMemcpyAsync(upi, type, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    if (box) { in.box = upi + n; CU(cudaMemcpyAsync(upi + n, box, sizeof(int) * n, cudaMemcpyHostToDevice, st)); }
    if (movable) { in.movable = upm; CU(cudaMemcpyAsync(upm, movable, (size_t)n, cudaMemcpyHostToDevice, st)); }
    return upload_staged(e, n, box, id, type, in);
}

// Validation, binning and placement of a staged bead set (in: device arrays
// in the staging buffers; id and type: the same beads on the host, or null
// for an upload from device memory).
static int upload_staged(dpd_engine* e, int64_t n, const int32_t* box, const int64_t* id, const int32_t* type,
                         const UploadIn& in)
{
    cudaStream_t st = e->s();
    int rc;
    // validation and binning (CSimBox::AssignBeadstoCells, SimBox.cpp:715-762:
    // ix = (long)(x/w), box-local coordinates); nothing of the state changes yet
    // herr: the first bead of each error kind, any residual unPBC offset,
    // the bits of ids / types that differ from the previous upload, and the
    // beads per type
    int herr[kUpErrors + 2 + kMaxTypes];
    for (int k = 0; k < kUpErrors; ++k) herr[k] = INT_MAX;
    for (int k = kUpErrors; k < kUpErrors + 2 + kMaxTypes; ++k) herr[k] = 0;
    CU(cudaMemcpyAsync(e->d_up_err, herr, sizeof herr, cudaMemcpyHostToDevice, st));
    const UploadPrev prev{e->d_prev_id, e->d_prev_type, reinterpret_cast<unsigned*>(e->d_up_err + kUpErrors + 1),
                          e->d_up_err + kUpErrors + 2};
    const bool prev_ok = e->prev_n == n;   // d_prev_* hold the last complete upload of n beads
    k_up_check<<<blocks_for(n, kThreads), kThreads, 0, st>>>((int)n, (int)e->hboxes.size(), e->ntypes, e->d_boxes, in,
                                                            e->d_up_cell, e->d_up_img, e->d_up_off, e->d_count,
                                                            e->d_block_count, e->d_up_err, e->d_up_err + kUpErrors,
                                                            prev);
    if ((rc = check_launch(e, "k_up_check"))) return rc;
    CU(cudaMemcpyAsync(herr, e->d_up_err, sizeof herr, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    e->prev_n = -1;   // d_prev_* now hold this upload, complete only once it succeeds
    int bad = INT_MAX, kind = -1;
    for (int k = 0; k < kUpErrors; ++k)
        if (herr[k] < bad) { bad = herr[k]; kind = k; }
    if (kind >= 0) {
        CU(cudaMemset(e->d_count, 0, sizeof(int) * (size_t)e->ncell));
        CU(cudaMemset(e->d_block_count, 0, sizeof(int) * (size_t)e->nchunk));
        switch (kind) {
            case kUpType: return fail(e, DPD_E_ARG, "bead type out of range");
            case kUpId: return fail(e, DPD_E_ARG, "bead id outside 1..2^31-1");
            case kUpBox: return fail(e, DPD_E_ARG, "bead box index out of range");
            case kUpNonFinite: return fail(e, DPD_E_BOX, "non-finite bead state");
            case kUpOutside: {
                char msg[160];
                if (id)
                    snprintf(msg, sizeof msg, "bead %lld (id %lld) lies outside the box", (long long)bad,
                             (long long)id[bad]);
                else
                    snprintf(msg, sizeof msg, "bead %lld lies outside the box", (long long)bad);
                return fail(e, DPD_E_BOX, msg);
            }
            default: return fail(e, DPD_E_ARG, "unPBC more than 511 box lengths from x");
        }
    }
    const bool any_off = herr[kUpErrors] != 0;
    const bool same_n = e->n == n;
    if ((rc = ensure_beads(e, n))) return rc;
    e->n = n;
    // cell starts, then the slot order: by cell, inside a cell by upload index
    k_scan_cells<<<e->nchunk, kScanThreads, 0, st>>>((int)e->ncell, (int)n, e->d_count, e->d_block_count, e->d_start,
                                                     (const unsigned*)e->d_status, (unsigned*)nullptr, 1);
    if ((rc = check_launch(e, "k_scan_cells"))) return rc;
    CU(cudaMemsetAsync(e->d_block_count, 0, sizeof(int) * (size_t)e->nchunk, st));
    k_up_scatter<<<blocks_for(n, kThreads), kThreads, 0, st>>>((int)n, e->d_up_cell, e->d_start, e->d_count,
                                                              e->d_up_perm);
    if ((rc = check_launch(e, "k_up_scatter"))) return rc;
    const int c = e->cur;
    if (e->precision == DPD_PRECISION_FP64)
        k_up_place<double><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            (int)n, in, e->d_up_cell, e->d_up_img, e->d_start, e->d_up_perm, e->d_x[c], e->d_v[c], (double*)e->d_F,
            e->d_bid[c], e->d_tf[c], e->d_cell[c], e->d_img[c], e->d_pid[c], e->d_pid_of);
    else
        k_up_place<float><<<blocks_for(n, kThreads), kThreads, 0, st>>>(
            (int)n, in, e->d_up_cell, e->d_up_img, e->d_start, e->d_up_perm, e->d_x[c], e->d_v[c], (float*)e->d_F,
            e->d_bid[c], e->d_tf[c], e->d_cell[c], e->d_img[c], e->d_pid[c], e->d_pid_of);
    if ((rc = check_launch(e, "k_up_place"))) return rc;
    CU(cudaMemsetAsync(e->d_count, 0, sizeof(int) * (size_t)e->ncell, st));
    if (any_off) {
        bool moved = false;
        if ((rc = ensure(e, &e->d_off, e->cap_off, 3 * (size_t)e->cap_n, &moved))) return rc;
        CU(cudaMemcpyAsync(e->d_off, e->d_up_off, 3 * sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st));
        if (moved || !e->off_active) drop_graphs(e);
    } else if (e->off_active) {
        drop_graphs(e);        // the kernels' offset pointer becomes null
    }
    e->off_active = any_off;
    CU(cudaMemsetAsync(e->d_stress, 0, 9 * real_size(e) * (size_t)n, st));
    CU(cudaMemsetAsync(e->d_status, 0, sizeof(unsigned), st));
    // host copies of ids and types, refreshed only when the device saw them
    // change; beads per type counted by k_up_check
    const unsigned changed = prev_ok ? (unsigned)herr[kUpErrors + 1] : 3u;
    e->type_count.assign(herr + kUpErrors + 2, herr + kUpErrors + 2 + e->ntypes);
    if (!id || !type) {
        // an upload from device memory: the host copies are fetched when needed
        if (changed & 3u) {
            e->host_ids_stale = true;
            ++e->ids_version;
        }
    } else {
        if (e->host_ids_stale || (changed & 1u) || e->h_id.size() != (size_t)n) {
            e->h_id.assign(id, id + n);
            ++e->ids_version;
        }
        if (e->host_ids_stale || (changed & 2u) || e->h_type.size() != (size_t)n) e->h_type.assign(type, type + n);
        e->host_ids_stale = false;
    }
    CU(cudaStreamSynchronize(st));
    *(volatile unsigned*)e->h_seen = 0u;   // no kernel of the engine is in flight after the sync
    rc = empty_topology(e, same_n);
    if (rc) return rc;
    e->uploaded = true;
    e->prev_n = n;
    e->rs_order.clear();   // the restart layout refers to the old beads
    e->mon_set = false;   // the monitor's polymers and initial positions refer to the old beads
    e->stepped = false;
    e->sampled = false;
    e->obs_valid = false;
    e->box_obs_valid = false;
    return DPD_OK;
}

int dpd_engine_upload_beads(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type,
                            const uint8_t* movable, const double* x3, const double* unpbc3, const double* v3,
                            const double* f3)
{
    return upload_impl(e, n, nullptr, id, type, movable, x3, unpbc3, v3, f3);
}

int dpd_batch_upload_beads(dpd_engine* e, int64_t n, const int32_t* box, const int64_t* id, const int32_t* type,
                           const uint8_t* movable, const double* x3, const double* unpbc3, const double* v3,
                           const double* f3)
{
    if (!box) return fail(e, DPD_E_ARG, "null box array");
    return upload_impl(e, n, box, id, type, movable, x3, unpbc3, v3, f3);
}

// CBuilder::MaxwellDist (Builder.cpp:104-126): max(n, 10^7) magnitudes from a
// sequential recurrence through the C library's log and exp, computed on the
// host the way the reference does (same operations, same order) and kept for
// the process.
static const std::vector<double>& maxwell_table(int64_t n)
{
    static std::mutex mu;
    static std::vector<double> tab;
    std::lock_guard<std::mutex> lock(mu);
    const int64_t M = std::max<int64_t>(n, 10000000);
    if ((int64_t)tab.size() != M) {
        tab.assign((size_t)M, 0.0);
        const double dM = (double)M;
        double factor = 1.0;
        for (int64_t j = 0; j < M - 1; ++j) {
            const double vel = std::sqrt(2.0 * std::log(dM * factor / (dM - factor)));
            factor = std::exp(0.5 * vel * vel);
            tab[(size_t)j] = vel;
        }
        tab[(size_t)(M - 1)] = tab[(size_t)(M - 2)];
    }
    return tab;
}

int dpd_engine_build_random(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type, uint64_t rng_seed,
                            int64_t rng_skip, int64_t nb, const int64_t* bond_head, const int64_t* bond_tail,
                            double* x3_out, double* v3_out)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "a slab's beads come from its exchange (dpd_engine_slab_unpack)");
    if (n < 1 || n > ((int64_t)1 << 30) || !id || !type || rng_skip < 0 || nb < 0 ||
        (nb > 0 && (!bond_head || !bond_tail)))
        return fail(e, DPD_E_ARG, "bad arguments");
    if (e->hboxes.size() != 1) return fail(e, DPD_E_ARG, "the random builder fills a single box");
    for (int64_t k = 0; k < nb; ++k)
        if (bond_head[k] < 0 || bond_head[k] >= n || bond_tail[k] < 0 || bond_tail[k] >= n ||
            bond_head[k] == bond_tail[k])
            return fail(e, DPD_E_ARG, "bond bead index out of range");
    // connected components of the bond graph (union-find on bead indices);
    // each component's bonds keep their order
    std::vector<int64_t> comp_ptr(1, 0), comp_bonds;
    if (nb > 0) {
        std::vector<int64_t> parent((size_t)n);
        for (int64_t b = 0; b < n; ++b) parent[(size_t)b] = b;
        auto find = [&](int64_t a) {
            while (parent[(size_t)a] != a) {
                parent[(size_t)a] = parent[(size_t)parent[(size_t)a]];
                a = parent[(size_t)a];
            }
            return a;
        };
        for (int64_t k = 0; k < nb; ++k) {
            const int64_t ra = find(bond_head[k]), rb = find(bond_tail[k]);
            if (ra != rb) parent[(size_t)std::max(ra, rb)] = std::min(ra, rb);
        }
        std::vector<int64_t> root((size_t)nb), count;
        std::unordered_map<int64_t, int64_t> slot;
        for (int64_t k = 0; k < nb; ++k) {
            const int64_t r = find(bond_head[k]);
            auto it = slot.find(r);
            if (it == slot.end()) { it = slot.emplace(r, (int64_t)count.size()).first; count.push_back(0); }
            root[(size_t)k] = it->second;
            count[(size_t)it->second]++;
        }
        comp_ptr.assign(count.size() + 1, 0);
        for (size_t c = 0; c < count.size(); ++c) comp_ptr[c + 1] = comp_ptr[c] + count[c];
        std::vector<int64_t> fill(comp_ptr.begin(), comp_ptr.end() - 1);
        comp_bonds.resize((size_t)nb);
        for (int64_t k = 0; k < nb; ++k) comp_bonds[(size_t)fill[(size_t)root[(size_t)k]]++] = k;
    }
    const int ncomp = (int)comp_ptr.size() - 1;
    const std::vector<double>& tab = maxwell_table(n);
    CU(cudaSetDevice(e->device));
    if (int rc0 = drop_ahead(e)) return rc0;   // the new state replaces the drifted one
    CU(cudaStreamSynchronize(e->s()));
    cudaStream_t st = e->s();
    int rc;
    if ((rc = stage_buffers(e, n))) return rc;
    double* up = e->d_up;
    int* upi = reinterpret_cast<int*>(up + 13 * (size_t)n);
    const int nblk = blocks_for(n, kRbThreads);
    // scratch of the build, released at the end: table, partial sums, bonds
    double* d_tab = nullptr;
    double* d_part = nullptr;
    int64_t* d_bonds = nullptr;
    auto release = [&]() { dfree(e, d_tab); dfree(e, d_part); dfree(e, d_bonds); };
    const size_t nbw = nb > 0 ? 2 * (size_t)nb + (size_t)ncomp + 1 + (size_t)nb : 1;
    if ((rc = dalloc(e, &d_tab, tab.size())) || (rc = dalloc(e, &d_part, 3 * (size_t)nblk + 8)) ||
        (rc = dalloc(e, &d_bonds, nbw))) {
        release();
        return rc;
    }
    UploadIn in{};
    in.x = up;
    in.v = up + 6 * (size_t)n;
    in.id = reinterpret_cast<const int64_t*>(up + 12 * (size_t)n);
    in.type = upi;
    auto run = [&]() -> int {
        CU(cudaMemcpyAsync(up + 12 * (size_t)n, id, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(upi, type, sizeof(int) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st));
        const Box& B = e->hboxes[0];
        k_rb_beads<<<nblk, kRbThreads, 0, st>>>((int)n, rng_seed, (uint64_t)rng_skip, B.L[0], B.L[1], B.L[2], d_tab,
                                                (int64_t)tab.size(), up, up + 6 * (size_t)n, d_part);
        if (int r = check_launch(e, "k_rb_beads")) return r;
        if (nb > 0) {
            int64_t* dh = d_bonds;
            int64_t* dt = dh + nb;
            int64_t* dp = dt + nb;
            int64_t* dc = dp + ncomp + 1;
            CU(cudaMemcpyAsync(dh, bond_head, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dt, bond_tail, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dp, comp_ptr.data(), sizeof(int64_t) * (ncomp + 1), cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dc, comp_bonds.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
            k_rb_bonds<<<blocks_for(ncomp, kRbThreads), kRbThreads, 0, st>>>(ncomp, dp, dc, dh, dt, up);
            if (int r = check_launch(e, "k_rb_bonds")) return r;
        }
        double* stats = d_part + 3 * (size_t)nblk;   // vcm[3], vtotal
        k_rb_vcm<<<1, 32, 0, st>>>(nblk, (int)n, d_part, stats);
        k_rb_center<<<nblk, kRbThreads, 0, st>>>((int)n, stats, up + 6 * (size_t)n, d_part);
        k_rb_vtotal<<<1, 32, 0, st>>>(nblk, (int)n, d_part, stats);
        k_rb_scale<<<blocks_for(3 * n, kRbThreads), kRbThreads, 0, st>>>((int)n, std::sqrt(e->params.kT), stats,
                                                                         up + 6 * (size_t)n);
        if (int r = check_launch(e, "k_rb_scale")) return r;
        if (x3_out) CU(cudaMemcpyAsync(x3_out, up, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        if (v3_out) CU(cudaMemcpyAsync(v3_out, up + 6 * (size_t)n, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        return DPD_OK;
    };
    rc = run();
    release();
    if (rc) return rc;
    return upload_staged(e, n, nullptr, id, type, in);
}

int dpd_engine_build_lamella(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type, int64_t npoly,
                             const int64_t* poly_first, const int32_t* poly_type, int32_t lipid_type,
                             int32_t head_offset, int32_t tail_offset, int32_t normal, double centre_frac,
                             double thickness, int32_t linearise, double upper_fraction, uint64_t rng_seed,
                             int64_t rng_skip, int64_t nb, const int64_t* bond_head, const int64_t* bond_tail,
                             double* x3_out, double* v3_out)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "a slab's beads come from its exchange (dpd_engine_slab_unpack)");
    if (n < 1 || n > ((int64_t)1 << 30) || !id || !type || npoly < 1 || npoly > n || !poly_first || !poly_type ||
        rng_skip < 0 || nb < 0 || (nb > 0 && (!bond_head || !bond_tail)) || normal < 0 || normal > 2 ||
        !(thickness > 0.0) || !(upper_fraction >= 0.0 && upper_fraction <= 1.0))
        return fail(e, DPD_E_ARG, "bad arguments");
    if (e->hboxes.size() != 1) return fail(e, DPD_E_ARG, "the lamella builder fills a single box");
    if (poly_first[0] != 0 || poly_first[npoly] != n) return fail(e, DPD_E_ARG, "polymers must cover the beads");
    for (int64_t p = 0; p < npoly; ++p)
        if (poly_first[p + 1] <= poly_first[p]) return fail(e, DPD_E_ARG, "empty or unordered polymer");
    for (int64_t k = 0; k < nb; ++k)
        if (bond_head[k] < 0 || bond_head[k] >= n || bond_tail[k] < 0 || bond_tail[k] >= n ||
            bond_head[k] == bond_tail[k])
            return fail(e, DPD_E_ARG, "bond bead index out of range");
    const Box& B = e->hboxes[0];
    // InitialStateLamella.cpp:705-770: lattice lengths, mid-plane, head planes
    LamellaParams P{};
    P.normal = normal;
    P.p0 = normal == 0 ? 1 : (normal == 1 ? 2 : 0);   // LamellaBuilder.cpp:440-600
    P.p1 = normal == 0 ? 2 : (normal == 1 ? 0 : 1);
    for (int d = 0; d < 3; ++d) P.L[d] = B.L[d];
    const double l1 = normal == 0 ? B.L[1] : B.L[0], l2 = normal == 2 ? B.L[1] : B.L[2], Ln = B.L[normal];
    const double centre = centre_frac * Ln;
    if (centre + 0.5 * thickness > Ln || centre - 0.5 * thickness < 0.0)
        return fail(e, DPD_E_ARG, "the bilayer does not fit the box");
    double lower = centre - 0.5 * thickness, upper = centre + 0.5 * thickness;
    const double area = l1 * l2;
    // the bilayer polymers (type lipid_type, in polymer order), all one size
    std::vector<int64_t> lip;
    int64_t size = 0;
    for (int64_t p = 0; p < npoly; ++p)
        if (poly_type[p] == lipid_type) {
            const int64_t m = poly_first[p + 1] - poly_first[p];
            if (lip.empty()) size = m;
            else if (m != size) return fail(e, DPD_E_ARG, "bilayer polymers of different sizes");
            lip.push_back(p);
        }
    const int64_t total = (int64_t)lip.size();
    if (total == 0 || head_offset < 0 || tail_offset < 0 || head_offset >= size || tail_offset >= size ||
        head_offset == tail_offset)
        return fail(e, DPD_E_ARG, "no bilayer polymers, or bad head / tail offsets");
    int64_t counter = 0;   // beads head..tail inclusive (LamellaBuilder.cpp:300-336)
    {
        bool bcount = false;
        int64_t pend = -1;
        for (int64_t k = 0; k < size; ++k) {
            if (k == head_offset && !bcount) { bcount = true; pend = tail_offset; counter++; }
            else if (k == tail_offset && !bcount) { bcount = true; pend = head_offset; counter++; }
            else if (k == pend) { bcount = false; counter++; }
            else if (bcount) counter++;
        }
    }
    // monolayers (LamellaBuilder.cpp:180-222) and their lattices (:250-290)
    int64_t mtot[2], mfirst[2], lat[2];
    P.msign[0] = 1.0;
    P.msign[1] = -1.0;
    mtot[0] = (int64_t)(upper_fraction * (double)total);
    mtot[1] = total - mtot[0];
    const bool mono1 = mtot[0] == 0 || mtot[1] == 0;
    if (mtot[0] == 0) {
        mfirst[0] = mfirst[1] = 0; lat[0] = 0; lat[1] = mtot[1];
        P.mhead[0] = 0.0; P.mhead[1] = lower; upper = centre;
    } else if (mtot[1] == 0) {
        mfirst[0] = mfirst[1] = 0; lat[0] = mtot[0]; lat[1] = 0;
        P.mhead[0] = upper; P.mhead[1] = 0.0; lower = centre;
    } else {
        mfirst[0] = 0; mfirst[1] = mtot[0]; lat[0] = mtot[0]; lat[1] = mtot[1];
        P.mhead[0] = upper; P.mhead[1] = lower;
    }
    double hs[2];
    if (mono1) {
        if (mtot[0] == 0) { hs[0] = 0.0; hs[1] = 0.999 * std::sqrt(1.1547 * area / (double)lat[1]); }
        else { hs[0] = 0.999 * std::sqrt(1.1547 * area / (double)lat[0]); hs[1] = 0.0; }
    } else {
        hs[0] = 0.999 * std::sqrt(1.1547 * area / (double)lat[0]);
        hs[1] = 0.999 * std::sqrt(1.1547 * area / (double)lat[1]);
    }
    double e2x[2];
    for (int mi = 0; mi < 2; ++mi) {
        P.e1x[mi] = hs[mi];
        e2x[mi] = 0.5 * hs[mi];
        P.e2y[mi] = 0.866025 * hs[mi];
    }
    P.cspace[0] = 0.5 * thickness / (double)(counter - 1);
    P.cspace[1] = P.cspace[0];
    P.centre = centre;
    P.thickness = thickness;
    P.size = (int)size;
    P.head_offset = head_offset;
    P.tail_offset = tail_offset;
    P.lipid_type = lipid_type;
    P.linearise = linearise ? 1 : 0;
    // the lattice walk of each monolayer (LamellaBuilder.cpp:382-650): the
    // site of every bilayer polymer, in the reference's floating-point order
    std::vector<double> site(2 * (size_t)total);
    std::vector<int> mono((size_t)total);
    for (int mi = 0; mi < 2; ++mi) {
        double hexp[2] = {0.001 * P.e1x[mi], 0.001 * P.e2y[mi]};
        double xp[2] = {hexp[0], hexp[1]};
        int64_t rowCounter = 0;
        for (int64_t iv = mfirst[mi]; iv < mfirst[mi] + lat[mi]; ++iv) {
            site[2 * (size_t)iv] = xp[0];
            site[2 * (size_t)iv + 1] = xp[1];
            mono[(size_t)iv] = mi;
            hexp[0] += P.e1x[mi];
            if (hexp[0] > l1 + (double)rowCounter * e2x[mi]) {
                rowCounter++;
                hexp[0] = (double)rowCounter * e2x[mi];
                hexp[1] += P.e2y[mi];
                xp[0] = hexp[0];
                xp[1] = hexp[1];
                if (hexp[1] >= l2) return fail(e, DPD_E_ARG, "lamella lattice outside the box");
            } else if (hexp[0] > l1) {
                xp[0] = hexp[0] - l1;
            } else {
                xp[0] = hexp[0];
                xp[1] = hexp[1];
            }
        }
    }
    // each polymer's first draw: the bilayer polymers in order (three per
    // scattered bead), then the other polymers in polymer order (one, then
    // three per bead); the velocities after all of them
    std::vector<int64_t> pdraw((size_t)npoly);
    std::vector<int> plip((size_t)npoly, -1), bpoly((size_t)n), ptype(poly_type, poly_type + npoly);
    const int64_t per_lipid = P.linearise ? 0 : 3 * (size - 2);
    for (int64_t j = 0; j < total; ++j) {
        pdraw[(size_t)lip[(size_t)j]] = per_lipid * j;
        plip[(size_t)lip[(size_t)j]] = (int)j;
    }
    int64_t draws = per_lipid * total;
    for (int64_t p = 0; p < npoly; ++p) {
        for (int64_t b = poly_first[p]; b < poly_first[p + 1]; ++b) bpoly[(size_t)b] = (int)p;
        if (poly_type[p] == lipid_type) continue;
        pdraw[(size_t)p] = draws;
        draws += 1 + 3 * (poly_first[p + 1] - poly_first[p]);
    }
    P.vel_base = (uint64_t)draws;
    P.seed = rng_seed;
    P.skip = (uint64_t)rng_skip;
    // the free regions along the normal (LamellaBuilder.cpp:960-990, Builder.cpp:350-372)
    const double ex[6] = {0.0, 0.0, lower, upper, Ln - 0.0, Ln};
    for (int k = 0; k < 6; ++k) P.ex[k] = ex[k];
    {
        double freeLength = 0.0, cum = 0.0;
        for (int i = 1; i < 3; ++i) freeLength += ex[2 * i] - ex[2 * i - 1];
        for (int i = 1; i < 3; ++i) { cum += (ex[2 * i] - ex[2 * i - 1]) / freeLength; P.ratio[i - 1] = cum; }
    }
    // the other polymers' bonds (shortened per polymer in its bond order)
    std::vector<int64_t> comp_ptr(1, 0), comp_bonds;
    {
        int64_t cur = -1;
        for (int64_t k = 0; k < nb; ++k) {
            const int64_t p = bpoly[(size_t)bond_head[k]];
            if (poly_type[p] == lipid_type) continue;
            if (bpoly[(size_t)bond_tail[k]] != p) return fail(e, DPD_E_ARG, "a bond joins two polymers");
            if (p < cur) return fail(e, DPD_E_ARG, "bonds not in polymer order");
            if (p != cur) {
                if (cur >= 0) comp_ptr.push_back((int64_t)comp_bonds.size());
                cur = p;
            }
            comp_bonds.push_back(k);
        }
        if (cur >= 0) comp_ptr.push_back((int64_t)comp_bonds.size());
    }
    const int ncomp = (int)comp_ptr.size() - 1;
    const std::vector<double>& tab = maxwell_table(n);
    P.ntab = (int64_t)tab.size();
    CU(cudaSetDevice(e->device));
    if (int rc0 = drop_ahead(e)) return rc0;   // the new state replaces the drifted one
    CU(cudaStreamSynchronize(e->s()));
    cudaStream_t st = e->s();
    int rc;
    if ((rc = stage_buffers(e, n))) return rc;
    double* up = e->d_up;
    int* upi = reinterpret_cast<int*>(up + 13 * (size_t)n);
    const int nblk = blocks_for(n, kRbThreads);
    // scratch of the build, released at the end
    double* d_tab = nullptr;
    double* d_part = nullptr;
    double* d_site = nullptr;
    int64_t* d_i64 = nullptr;   // pfirst (npoly + 1), pdraw (npoly), bond heads, tails, comp_ptr, comp_bonds
    int* d_i32 = nullptr;       // bpoly (n), ptype, plip (npoly), mono (total)
    auto release = [&]() { dfree(e, d_tab); dfree(e, d_part); dfree(e, d_site); dfree(e, d_i64); dfree(e, d_i32); };
    const size_t n64 = (size_t)(2 * npoly + 1) + (nb > 0 ? 2 * (size_t)nb + comp_ptr.size() + comp_bonds.size() : 0);
    const size_t n32 = (size_t)n + 2 * (size_t)npoly + (size_t)total;
    if ((rc = dalloc(e, &d_tab, tab.size())) || (rc = dalloc(e, &d_part, 3 * (size_t)nblk + 8)) ||
        (rc = dalloc(e, &d_site, site.size())) || (rc = dalloc(e, &d_i64, n64)) || (rc = dalloc(e, &d_i32, n32))) {
        release();
        return rc;
    }
    UploadIn in{};
    in.x = up;
    in.v = up + 6 * (size_t)n;
    in.id = reinterpret_cast<const int64_t*>(up + 12 * (size_t)n);
    in.type = upi;
    auto run = [&]() -> int {
        int64_t* dpf = d_i64;
        int64_t* dpd = dpf + npoly + 1;
        int* dbp = d_i32;
        int* dpt = dbp + n;
        int* dpl = dpt + npoly;
        int* dmo = dpl + npoly;
        CU(cudaMemcpyAsync(up + 12 * (size_t)n, id, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(upi, type, sizeof(int) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_site, site.data(), sizeof(double) * site.size(), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dpf, poly_first, sizeof(int64_t) * (npoly + 1), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dpd, pdraw.data(), sizeof(int64_t) * npoly, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dbp, bpoly.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dpt, ptype.data(), sizeof(int) * npoly, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dpl, plip.data(), sizeof(int) * npoly, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dmo, mono.data(), sizeof(int) * total, cudaMemcpyHostToDevice, st));
        k_lb_beads<<<nblk, kRbThreads, 0, st>>>((int)n, P, dbp, dpf, dpt, dpd, dpl, d_site, dmo, d_tab, up,
                                                up + 6 * (size_t)n, d_part);
        if (int r = check_launch(e, "k_lb_beads")) return r;
        if (ncomp > 0) {
            int64_t* dh = dpd + npoly;
            int64_t* dt = dh + nb;
            int64_t* dp = dt + nb;
            int64_t* dc = dp + comp_ptr.size();
            CU(cudaMemcpyAsync(dh, bond_head, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dt, bond_tail, sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dp, comp_ptr.data(), sizeof(int64_t) * comp_ptr.size(), cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(dc, comp_bonds.data(), sizeof(int64_t) * comp_bonds.size(), cudaMemcpyHostToDevice,
                               st));
            k_rb_bonds<<<blocks_for(ncomp, kRbThreads), kRbThreads, 0, st>>>(ncomp, dp, dc, dh, dt, up);
            if (int r = check_launch(e, "k_rb_bonds")) return r;
        }
        double* stats = d_part + 3 * (size_t)nblk;   // vcm[3], vtotal
        k_rb_vcm<<<1, 32, 0, st>>>(nblk, (int)n, d_part, stats);
        k_rb_center<<<nblk, kRbThreads, 0, st>>>((int)n, stats, up + 6 * (size_t)n, d_part);
        k_lb_vtotal<<<1, 32, 0, st>>>(nblk, (int)n, e->params.kT, d_part, stats);
        k_lb_scale<<<nblk, kRbThreads, 0, st>>>((int)n, normal, stats, up + 6 * (size_t)n);
        if (int r = check_launch(e, "k_lb_scale")) return r;
        if (x3_out) CU(cudaMemcpyAsync(x3_out, up, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        if (v3_out) CU(cudaMemcpyAsync(v3_out, up + 6 * (size_t)n, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        return DPD_OK;
    };
    rc = run();
    release();
    if (rc) return rc;
    return upload_staged(e, n, nullptr, id, type, in);
}

int dpd_engine_upload_topology(dpd_engine* e, int64_t nb, const int64_t* bond_head_id, const int64_t* bond_tail_id,
                               const double* k2, const double* l0, int64_t na, const int64_t* first_bond,
                               const int64_t* second_bond, const double* k3, const double* phi0)
{
    if (!e) return DPD_E_ARG;
    if (!e->uploaded) return fail(e, DPD_E_STATE, "upload beads before the topology");
    if (e->hboxes.size() > 1 && (nb > 0 || na > 0))
        return fail(e, DPD_E_STATE, "bonds are not supported in a replica batch");
    if (nb < 0 || na < 0 || (nb && (!bond_head_id || !bond_tail_id || !k2 || !l0)) ||
        (na && (!first_bond || !second_bond || !k3 || !phi0)))
        return fail(e, DPD_E_ARG, "bad topology arrays");
    if (e->slab) return fail(e, DPD_E_STATE, "a slab takes its topology in dpd_engine_slab_setup");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    if (int rc0 = host_ids(e)) return rc0;
    const int64_t n = e->n;
    // The device arrays are built on the host in one pinned staging buffer
    // and copied asynchronously; the call waits once, at the end.
    const size_t nterm = (size_t)(2 * nb + 3 * na);
    if (nb * 2 + na * 3 > ((int64_t)1 << 28)) return fail(e, DPD_E_ARG, "topology too large");
    auto words = [](size_t k, size_t w) { return (k * w + 15) / 16 * 16; };   // 16-byte aligned pieces
    const size_t stage = words(2 * (size_t)nb, 4) + words(2 * (size_t)nb, 8) + words(4 * (size_t)na, 4) +
                         words(3 * (size_t)na, 8) + words((size_t)n + 1, 4) + words(nterm, 4) + words((size_t)n, 4);
    if (stage > e->cap_h_stage) {
        if (e->h_stage) cudaFreeHost(e->h_stage);
        e->h_stage = nullptr;
        e->cap_h_stage = 0;
        if (cudaHostAlloc((void**)&e->h_stage, stage, cudaHostAllocDefault) != cudaSuccess) {
            e->h_stage = nullptr;
            return fail(e, DPD_E_CUDA, "pinned staging allocation failed");
        }
        e->cap_h_stage = stage;
    }
    unsigned char* arena = e->h_stage;
    auto carve = [&](size_t k, size_t w) {
        unsigned char* q = arena;
        arena += words(k, w);
        return q;
    };
    int* bh = reinterpret_cast<int*>(carve(2 * (size_t)nb, 4));
    int* bt = bh + nb;
    double* bk = reinterpret_cast<double*>(carve(2 * (size_t)nb, 8));   // k2, then l0
    int* a4 = reinterpret_cast<int*>(carve(4 * (size_t)na, 4));          // four planes of na
    double* ak = reinterpret_cast<double*>(carve(3 * (size_t)na, 8));    // k3, cos(phi0), sin(phi0)
    int* cnt = reinterpret_cast<int*>(carve((size_t)n + 1, 4));
    int* terms = reinterpret_cast<int*>(carve(nterm, 4));
    int* bbl = reinterpret_cast<int*>(carve((size_t)n, 4));
    // The same topology for the same bead ids as the last build: the staging
    // buffer still holds that build, so only the copies are made again (a
    // bead upload clears the term offsets and the bonded flags).
    dpd_engine::TopoInputs& tin = e->topo_in;
    auto same_i = [](const std::vector<int64_t>& v, const int64_t* q, int64_t k) {
        return (int64_t)v.size() == k && (k == 0 || memcmp(v.data(), q, sizeof(int64_t) * (size_t)k) == 0);
    };
    auto same_d = [](const std::vector<double>& v, const double* q, int64_t k) {
        return (int64_t)v.size() == k && (k == 0 || memcmp(v.data(), q, sizeof(double) * (size_t)k) == 0);
    };
    const bool reuse = tin.valid && tin.ids_version == e->ids_version && tin.n == n &&
                       same_i(tin.bh, bond_head_id, nb) && same_i(tin.bt, bond_tail_id, nb) &&
                       same_d(tin.k2, k2, nb) && same_d(tin.l0, l0, nb) && same_i(tin.f, first_bond, na) &&
                       same_i(tin.sc, second_bond, na) && same_d(tin.k3, k3, na) && same_d(tin.phi0, phi0, na);
    int64_t nbl = reuse ? tin.nbl : 0;
    if (!reuse) {
    tin.valid = false;   // the staging buffer is rewritten below
    // bead id -> upload index (the ids kept from the bead upload)
    const std::vector<int64_t>& hpid = e->h_id;
    bool identity = true;
    for (int64_t b = 0; b < n && identity; ++b) identity = (hpid[b] == b + 1);
    std::unordered_map<int64_t, int> by_id;
    if (!identity && (nb || na)) {
        by_id.reserve((size_t)n);
        for (int64_t b = 0; b < n; ++b) by_id.emplace(hpid[b], (int)b);
    }
    auto index_of = [&](int64_t idv) -> int {
        if (identity) return (idv >= 1 && idv <= n) ? (int)(idv - 1) : -1;
        const auto it = by_id.find(idv);
        return it == by_id.end() ? -1 : it->second;
    };
    for (int64_t i = 0; i < nb; ++i) {
        bh[i] = index_of(bond_head_id[i]);
        bt[i] = index_of(bond_tail_id[i]);
        if (bh[i] < 0 || bt[i] < 0) return fail(e, DPD_E_ARG, "bond refers to an unknown bead id");
        if (bh[i] == bt[i]) return fail(e, DPD_E_ARG, "bond joins a bead to itself");
        bk[i] = k2[i];
        bk[nb + i] = l0[i];
    }
    for (int64_t i = 0; i < na; ++i) {
        if (first_bond[i] < 0 || first_bond[i] >= nb || second_bond[i] < 0 || second_bond[i] >= nb)
            return fail(e, DPD_E_ARG, "bond pair refers to an unknown bond");
        a4[i] = bh[first_bond[i]];
        a4[na + i] = bt[first_bond[i]];
        a4[2 * na + i] = bh[second_bond[i]];
        a4[3 * na + i] = bt[second_bond[i]];
        // CBondPair ctor caches cos/sin of phi0; the phi0 > 0 branch of
        // BondPair.cpp:178-188 is selected by sin0 != 0
        ak[i] = k3[i];
        ak[na + i] = phi0[i] > 0.0 ? std::cos(phi0[i]) : 1.0;
        ak[2 * na + i] = phi0[i] > 0.0 ? std::sin(phi0[i]) : 0.0;
    }
    // per-bead term lists (CSR by upload index); terms in bond order then pair order
    std::fill(cnt, cnt + n + 1, 0);
    for (int64_t i = 0; i < nb; ++i) { cnt[bh[i] + 1]++; cnt[bt[i] + 1]++; }
    for (int64_t i = 0; i < na; ++i) { cnt[a4[na + i] + 1]++; cnt[a4[i] + 1]++; cnt[a4[2 * na + i] + 1]++; }
    for (int64_t b = 0; b < n; ++b) cnt[b + 1] += cnt[b];
    std::vector<int> fillp(cnt, cnt + n);
    for (int64_t i = 0; i < nb; ++i) {
        terms[fillp[bh[i]]++] = (int)(i * 8 + kBondHead);
        terms[fillp[bt[i]]++] = (int)(i * 8 + kBondTail);
    }
    for (int64_t i = 0; i < na; ++i) {
        terms[fillp[a4[na + i]]++] = (int)(i * 8 + kAngle0);    // first bond's tail: force [0]
        terms[fillp[a4[i]]++] = (int)(i * 8 + kAngle1);         // middle bead:       force [1]
        terms[fillp[a4[2 * na + i]]++] = (int)(i * 8 + kAngle2);  // second bond's head: force [2]
    }
    for (int64_t b = 0; b < n; ++b)
        if (cnt[b + 1] > cnt[b]) bbl[nbl++] = (int)b;
    }
    bool moved = false;
    int rc;
    cudaStream_t st = e->s();
    if (nbl) {
        if ((rc = ensure(e, &e->d_ubuf, e->cap_ubuf, (size_t)n, &moved))) return rc;
        if ((rc = ensure(e, &e->d_Fb, e->cap_Fb, (size_t)n, &moved))) return rc;
        if ((rc = ensure(e, &e->d_Sb, e->cap_Sb, 9 * (size_t)n, &moved))) return rc;
        if ((rc = ensure(e, &e->d_bb, e->cap_bb, (size_t)nbl, &moved))) return rc;
        CU(cudaMemcpyAsync(e->d_bb, bbl, (size_t)nbl * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    if (nbl != e->nbb) drop_graphs(e);   // the bonded branch appears or changes size
    e->nbb = nbl;
    if ((rc = ensure(e, &e->d_csr_ptr, e->cap_csr_ptr, (size_t)n + 1, &moved))) return rc;
    if ((rc = ensure(e, &e->d_csr_term, e->cap_csr_term, nterm, &moved))) return rc;
    CU(cudaMemcpyAsync(e->d_csr_ptr, cnt, ((size_t)n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    if (nterm) CU(cudaMemcpyAsync(e->d_csr_term, terms, nterm * sizeof(int), cudaMemcpyHostToDevice, st));
    // mark the beads that have terms (kFlagBonded) so k_update_mom skips the
    // topology lookup for all others, and k_gather writes their unPBC
    // position into the FP64 buffer the bonded terms read
    k_mark_bonded<<<blocks_for(n, kThreads), kThreads, 0, st>>>((int)n, e->d_bid[e->cur], e->d_csr_ptr,
                                                                e->d_tf[e->cur]);
    if ((rc = check_launch(e, "k_mark_bonded"))) return rc;
    if (nb) {
        size_t c = e->cap_bond;
        if ((rc = ensure(e, &e->d_bond_h, c, nb, &moved))) return rc;
        c = e->cap_bond;
        if ((rc = ensure(e, &e->d_bond_t, c, nb, &moved))) return rc;
        c = e->cap_bond;
        if ((rc = ensure(e, &e->d_bond_k2, c, nb, &moved))) return rc;
        c = e->cap_bond;
        if ((rc = ensure(e, &e->d_bond_l0, c, nb, &moved))) return rc;
        e->cap_bond = std::max(e->cap_bond, (size_t)nb);
        CU(cudaMemcpyAsync(e->d_bond_h, bh, nb * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(e->d_bond_t, bt, nb * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(e->d_bond_k2, bk, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(e->d_bond_l0, bk + nb, nb * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    if (na) {
        const size_t c0 = e->cap_ang;
        for (int k = 0; k < 4; ++k) {
            size_t c = c0;
            if ((rc = ensure(e, &e->d_ang[k], c, na, &moved))) return rc;
            CU(cudaMemcpyAsync(e->d_ang[k], a4 + k * na, na * sizeof(int), cudaMemcpyHostToDevice, st));
        }
        size_t c = c0;
        if ((rc = ensure(e, &e->d_ang_k3, c, na, &moved))) return rc;
        c = c0;
        if ((rc = ensure(e, &e->d_ang_cos0, c, na, &moved))) return rc;
        c = c0;
        if ((rc = ensure(e, &e->d_ang_sin0, c, na, &moved))) return rc;
        e->cap_ang = std::max(c0, (size_t)na);
        CU(cudaMemcpyAsync(e->d_ang_k3, ak, na * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(e->d_ang_cos0, ak + na, na * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(e->d_ang_sin0, ak + 2 * na, na * sizeof(double), cudaMemcpyHostToDevice, st));
        e->h_ang_phi0.assign(phi0, phi0 + na);
    }
    CU(cudaStreamSynchronize(st));   // the staging buffer is reused by the next call
    if (!reuse) {
        tin.bh.assign(bond_head_id, bond_head_id + nb);
        tin.bt.assign(bond_tail_id, bond_tail_id + nb);
        tin.k2.assign(k2, k2 + nb);
        tin.l0.assign(l0, l0 + nb);
        tin.f.assign(first_bond, first_bond + na);
        tin.sc.assign(second_bond, second_bond + na);
        tin.k3.assign(k3, k3 + na);
        tin.phi0.assign(phi0, phi0 + na);
        tin.ids_version = e->ids_version;
        tin.n = n;
        tin.nbl = nbl;
        tin.valid = true;
    }
    e->topo_nb = nb;
    e->topo_na = na;
    e->mon_set = false;   // the monitor's bond types refer to the previous topology
    // the slice profile's bond types refer to the previous topology
    if (e->slice_S) { e->slice_S = 0; drop_graphs(e); }
    if (moved) drop_graphs(e);
    return DPD_OK;
}

int dpd_engine_set_slice_stress(dpd_engine* e, int32_t nslices, int32_t nbondtypes, const int32_t* bond_type,
                                int32_t nbptypes, const int32_t* bondpair_type)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "the slice profile covers a whole box; a slab also holds ghosts");
    if (e->hboxes.size() > 1) return fail(e, DPD_E_STATE, "the slice stress profile needs a single-box engine");
    if (!e->uploaded) return fail(e, DPD_E_STATE, "upload beads (and the topology) before the slice profile");
    if (nslices < 0 || nslices > 65536 || nbondtypes < 0 || nbptypes < 0 || nbondtypes > 65536 || nbptypes > 65536)
        return fail(e, DPD_E_ARG, "slice profile sizes out of range");
    if (nslices > 0 && ((e->topo_nb > 0 && !bond_type) || (e->topo_na > 0 && !bondpair_type)))
        return fail(e, DPD_E_ARG, "bond and bond-pair types are required for the uploaded topology");
    for (int64_t i = 0; nslices > 0 && i < e->topo_nb; ++i)
        if (bond_type[i] < 0 || bond_type[i] >= nbondtypes) return fail(e, DPD_E_ARG, "bond type out of range");
    for (int64_t i = 0; nslices > 0 && i < e->topo_na; ++i)
        if (bondpair_type[i] < 0 || bondpair_type[i] >= nbptypes)
            return fail(e, DPD_E_ARG, "bond-pair type out of range");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    drop_graphs(e);
    e->slice_S = 0;
    e->slice_sampled = false;
    if (nslices == 0) return DPD_OK;
    e->slice_nbt = nbondtypes;
    e->slice_nbpt = nbptypes;
    e->slice_S = nslices;
    int rc;
    bool moved = false;
    if ((rc = ensure(e, &e->d_slice, e->cap_slice, slice_bins(e), &moved))) { e->slice_S = 0; return rc; }
    if (e->topo_nb) {
        if ((rc = ensure(e, &e->d_slice_bt, e->cap_slice_bt, (size_t)e->topo_nb, &moved))) { e->slice_S = 0; return rc; }
        CU(cudaMemcpy(e->d_slice_bt, bond_type, sizeof(int) * e->topo_nb, cudaMemcpyHostToDevice));
    }
    if (e->topo_na) {
        if ((rc = ensure(e, &e->d_slice_bpt, e->cap_slice_bpt, (size_t)e->topo_na, &moved))) { e->slice_S = 0; return rc; }
        CU(cudaMemcpy(e->d_slice_bpt, bondpair_type, sizeof(int) * e->topo_na, cudaMemcpyHostToDevice));
    }
    CU(cudaMemset(e->d_slice, 0, slice_bins(e) * sizeof(double)));
    // the pair list (best effort: without it the profile is built by one kernel)
    if (ensure(e, &e->d_slice_list, e->cap_slice_list, (size_t)kSliceListPerBead * (size_t)e->n, &moved) != DPD_OK ||
        ensure(e, &e->d_slice_cnt, e->cap_slice_cnt, 2, &moved) != DPD_OK ||
        ensure(e, &e->d_slice_part, e->cap_slice_part,
               (size_t)e->sms * kSliceEvalBlocksPerSM * (size_t)nslices * e->ntypes * e->ntypes * 9, &moved) !=
            DPD_OK) {
        dfree(e, e->d_slice_list);
        e->d_slice_list = nullptr;
        e->cap_slice_list = 0;
    }
    // dynamic shared memory of the pair part: bins (when they fit) and hit lists
    const int KT = e->ntypes * e->ntypes;
    const bool bf = slice_smem_bytes<float>(nslices, KT, true) <= kSliceSmemMax;
    const bool bd = slice_smem_bytes<double>(nslices, KT, true) <= kSliceSmemMax;
    CU(cudaFuncSetAttribute(k_slice_pairs<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)slice_smem_bytes<float>(nslices, KT, bf)));
    CU(cudaFuncSetAttribute(k_slice_pairs<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)slice_smem_bytes<double>(nslices, KT, bd)));
    CU(cudaFuncSetAttribute(k_slice_eval<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)slice_eval_smem_bytes<float>(nslices, KT, bf)));
    CU(cudaFuncSetAttribute(k_slice_eval<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)slice_eval_smem_bytes<double>(nslices, KT, bd)));
    return DPD_OK;
}

int dpd_engine_slice_stress(dpd_engine* e, double* pair, double* bond, double* bondpair)
{
    if (!e) return DPD_E_ARG;
    if (!e->slice_S) return fail(e, DPD_E_STATE, "the slice stress profile is off");
    if (!e->slice_sampled) return fail(e, DPD_E_STATE, "no sample step has built the slice stress profile yet");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    const SliceParams sp = slice_params(e);
    const size_t S = (size_t)e->slice_S;
    if (pair) CU(cudaMemcpy(pair, sp.pair, S * e->ntypes * e->ntypes * 9 * sizeof(double), cudaMemcpyDeviceToHost));
    if (bond) CU(cudaMemcpy(bond, sp.bond, S * e->slice_nbt * 9 * sizeof(double), cudaMemcpyDeviceToHost));
    if (bondpair)
        CU(cudaMemcpy(bondpair, sp.bondpair, S * e->slice_nbpt * 9 * sizeof(double), cudaMemcpyDeviceToHost));
    return DPD_OK;
}

int dpd_engine_set_monitor(dpd_engine* e, int32_t nbondtypes, const int32_t* bond_type, int32_t nbptypes,
                           const int32_t* bondpair_type, int64_t npoly, const int64_t* poly_head_id,
                           const int64_t* poly_tail_id, const int32_t* poly_type, int32_t npolytypes,
                           const double* initial_unpbc3)
{
    if (!e) return DPD_E_ARG;
    if (!e->uploaded) return fail(e, DPD_E_STATE, "upload beads (and the topology) before the monitor");
    if (e->slab) return fail(e, DPD_E_STATE, "the monitor covers a whole box; a slab also holds ghosts");
    if (e->hboxes.size() > 1) return fail(e, DPD_E_STATE, "the monitor needs a single-box engine");
    if (nbondtypes < 0 || nbptypes < 0 || npolytypes < 0 || npoly < 0 || nbondtypes > 65536 || nbptypes > 65536 ||
        npolytypes > 65536 || (e->topo_nb && !bond_type) || (e->topo_na && !bondpair_type) ||
        (npoly && (!poly_head_id || !poly_tail_id || !poly_type)))
        return fail(e, DPD_E_ARG, "bad monitor arrays");
    std::vector<int64_t> bc(nbondtypes, 0), bpc(nbptypes, 0), pc(npolytypes, 0);
    for (int64_t i = 0; i < e->topo_nb; ++i) {
        if (bond_type[i] < 0 || bond_type[i] >= nbondtypes) return fail(e, DPD_E_ARG, "bond type out of range");
        bc[bond_type[i]]++;
    }
    for (int64_t i = 0; i < e->topo_na; ++i) {
        if (bondpair_type[i] < 0 || bondpair_type[i] >= nbptypes) return fail(e, DPD_E_ARG, "bond-pair type out of range");
        bpc[bondpair_type[i]]++;
    }
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    const int64_t n = e->n;
    // bead id -> upload index, as in the topology upload
    std::vector<int> hpid(n);
    CU(cudaMemcpy(hpid.data(), e->d_pid_of, n * sizeof(int), cudaMemcpyDeviceToHost));
    std::unordered_map<int64_t, int> by_id;
    by_id.reserve((size_t)n);
    for (int64_t b = 0; b < n; ++b) by_id.emplace((int64_t)hpid[b], (int)b);
    std::vector<int> ph(npoly), pt(npoly), pty(npoly);
    for (int64_t k = 0; k < npoly; ++k) {
        const auto ih = by_id.find(poly_head_id[k]), it = by_id.find(poly_tail_id[k]);
        if (ih == by_id.end() || it == by_id.end()) return fail(e, DPD_E_ARG, "polymer refers to an unknown bead id");
        if (poly_type[k] < 0 || poly_type[k] >= npolytypes) return fail(e, DPD_E_ARG, "polymer type out of range");
        ph[k] = ih->second;
        pt[k] = it->second;
        pty[k] = poly_type[k];
        pc[poly_type[k]]++;
    }
    int rc;
    auto upload_ints = [&](int** d, const int* h, int64_t cnt) -> int {
        dfree(e, *d);
        *d = nullptr;
        if ((rc = dalloc(e, d, (size_t)std::max<int64_t>(cnt, 1)))) return rc;
        if (cnt) CU(cudaMemcpy(*d, h, sizeof(int) * cnt, cudaMemcpyHostToDevice));
        return DPD_OK;
    };
    if ((rc = upload_ints(&e->d_mon_bt, bond_type, e->topo_nb))) return rc;
    if ((rc = upload_ints(&e->d_mon_bpt, bondpair_type, e->topo_na))) return rc;
    if ((rc = upload_ints(&e->d_mon_ph, ph.data(), npoly))) return rc;
    if ((rc = upload_ints(&e->d_mon_pt, pt.data(), npoly))) return rc;
    if ((rc = upload_ints(&e->d_mon_ptype, pty.data(), npoly))) return rc;
    double** dd[] = {&e->d_mon_phi0, &e->d_mon_u0, &e->d_mon_xu, &e->d_mon_sums};
    for (auto q : dd) { dfree(e, *q); *q = nullptr; }
    if ((rc = dalloc(e, &e->d_mon_phi0, (size_t)std::max<int64_t>(e->topo_na, 1)))) return rc;
    if (e->topo_na) CU(cudaMemcpy(e->d_mon_phi0, e->h_ang_phi0.data(), sizeof(double) * e->topo_na, cudaMemcpyHostToDevice));
    if ((rc = dalloc(e, &e->d_mon_u0, 3 * (size_t)n))) return rc;
    if ((rc = dalloc(e, &e->d_mon_xu, 6 * (size_t)n))) return rc;
    const size_t nsums = 6 + (size_t)e->ntypes + nbondtypes + 2 + npolytypes + 5 * (size_t)nbptypes;
    if ((rc = dalloc(e, &e->d_mon_sums, nsums))) return rc;
    if (initial_unpbc3) {
        CU(cudaMemcpy(e->d_mon_u0, initial_unpbc3, 3 * sizeof(double) * n, cudaMemcpyHostToDevice));
    } else {   // the current unPBC positions, as k_download forms them
        const int c = e->cur;
        const int nbk = blocks_for(n, kThreads);
        if (e->precision == DPD_PRECISION_FP64)
            k_download<double><<<nbk, kThreads, 0, e->s()>>>((int)n, e->d_boxes, e->d_tf[c], e->d_bid[c], e->d_x[c],
                                                             e->d_v[c], (const double*)e->d_F, e->d_img[c],
                                                             e->off_active ? e->d_off : nullptr, nullptr, e->d_cell[c],
                                                             nullptr, e->d_mon_u0, nullptr, nullptr, nullptr, nullptr);
        else
            k_download<float><<<nbk, kThreads, 0, e->s()>>>((int)n, e->d_boxes, e->d_tf[c], e->d_bid[c], e->d_x[c],
                                                            e->d_v[c], (const float*)e->d_F, e->d_img[c],
                                                            e->off_active ? e->d_off : nullptr, nullptr, e->d_cell[c],
                                                            nullptr, e->d_mon_u0, nullptr, nullptr, nullptr, nullptr);
        if ((rc = check_launch(e, "k_download"))) return rc;
        CU(cudaStreamSynchronize(e->s()));
    }
    e->mon_nbt = nbondtypes;
    e->mon_nbpt = nbptypes;
    e->mon_npt = npolytypes;
    e->mon_np = npoly;
    e->mon_bcount = bc;
    e->mon_bpcount = bpc;
    e->mon_pcount = pc;
    e->mon_set = true;
    return DPD_OK;
}

int dpd_engine_monitor(dpd_engine* e, dpd_monitor* out, double* msd, double* bond_length, double* end_to_end,
                       double* bondpair)
{
    if (!e) return DPD_E_ARG;
    if (!out) return fail(e, DPD_E_ARG, "null output");
    if (!e->mon_set) return fail(e, DPD_E_STATE, "dpd_engine_set_monitor has not been called for these beads");
    CU(cudaSetDevice(e->device));
    const int n = (int)e->n, T = e->ntypes;
    const size_t nsums = 6 + (size_t)T + e->mon_nbt + 2 + e->mon_npt + 5 * (size_t)e->mon_nbpt;
    CU(cudaMemsetAsync(e->d_mon_sums, 0, nsums * sizeof(double), e->s()));
    const int c = e->cur;
    k_monitor_beads<<<blocks_for(n, kThreads), kThreads, 0, e->s()>>>(n, T, e->d_boxes, e->d_tf[c], e->d_bid[c],
                                                                       e->d_x[c], e->d_img[c],
                                                                       e->off_active ? e->d_off : nullptr,
                                                                       e->d_mon_u0, e->d_mon_xu, e->d_mon_sums);
    int rc;
    if ((rc = check_launch(e, "k_monitor_beads"))) return rc;
    MonitorTerms M{};
    M.nb = (int)e->topo_nb;
    M.np = (int)e->mon_np;
    M.na = (int)e->topo_na;
    M.bond_h = e->d_bond_h; M.bond_t = e->d_bond_t; M.bond_type = e->d_mon_bt;
    M.poly_h = e->d_mon_ph; M.poly_t = e->d_mon_pt; M.poly_type = e->d_mon_ptype;
    M.ang_b1h = e->d_ang[0]; M.ang_b1t = e->d_ang[1]; M.ang_b2h = e->d_ang[2]; M.ang_b2t = e->d_ang[3];
    M.ang_type = e->d_mon_bpt; M.ang_phi0 = e->d_mon_phi0; M.ang_cos0 = e->d_ang_cos0; M.ang_sin0 = e->d_ang_sin0;
    M.nbt = e->mon_nbt; M.npt = e->mon_npt; M.nbpt = e->mon_nbpt;
    for (int d = 0; d < 3; ++d) M.L[d] = e->hboxes[0].L[d];
    M.sums = e->d_mon_sums + 6 + T;
    const int64_t terms = (int64_t)M.nb + M.np + M.na;
    const size_t tsm = (M.nbt + 2 + M.npt + 5 * (size_t)M.nbpt) * sizeof(double);
    if (terms > 0) {
        if (tsm > 48 * 1024) return fail(e, DPD_E_LIMIT, "too many bond, polymer and bond-pair types for the monitor");
        k_monitor_terms<<<blocks_for(terms, kThreads), kThreads, tsm, e->s()>>>(M, e->d_mon_xu, n);
        if ((rc = check_launch(e, "k_monitor_terms"))) return rc;
    }
    std::vector<double> h(nsums);
    CU(cudaMemcpyAsync(h.data(), e->d_mon_sums, nsums * sizeof(double), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    memset(out, 0, sizeof *out);
    out->step = e->stepped ? e->last_step : 0;
    out->n = e->n;
    // m_totalInertia / N (Monitor.cpp:999-1007), symmetric completion
    const double N = (double)e->n;
    const int idx[6] = {0, 1, 2, 4, 5, 8};
    for (int k = 0; k < 6; ++k) out->inertia[idx[k]] = h[k] / N;
    out->inertia[3] = out->inertia[1];
    out->inertia[6] = out->inertia[2];
    out->inertia[7] = out->inertia[5];
    // m_vBeadMSD / (6 dt t N_type) (Monitor.cpp:943-964); at step 0 only / N_type
    const double pre = 6.0 * e->params.dt * (double)out->step;
    for (int t = 0; t < T && msd; ++t) {
        const double cnt = (double)e->type_count[t];
        msd[t] = cnt > 0 ? h[6 + t] / ((pre > 0 ? pre : 1.0) * cnt) : 0.0;
    }
    const double* hb = h.data() + 6 + T;
    int64_t nbt = 0;
    for (int k = 0; k < e->mon_nbt; ++k) nbt += e->mon_bcount[k];
    for (int k = 0; k < e->mon_nbt && bond_length; ++k)
        bond_length[k] = e->mon_bcount[k] ? hb[k] / (double)e->mon_bcount[k] : 0.0;
    out->bonds = nbt;
    out->mean_bond_length = nbt ? hb[e->mon_nbt] / (double)nbt : 0.0;
    out->mean_sq_bond_length = nbt ? hb[e->mon_nbt + 1] / (double)nbt : 0.0;
    const double* hp = hb + e->mon_nbt + 2;
    for (int k = 0; k < e->mon_npt && end_to_end; ++k)
        end_to_end[k] = e->mon_pcount[k] ? hp[k] / (double)e->mon_pcount[k] : 0.0;
    const double* ha = hp + e->mon_npt;
    for (int k = 0; k < e->mon_nbpt && bondpair; ++k) {
        const int64_t cnt = e->mon_bpcount[k];
        double* o = bondpair + 6 * k;
        for (int q = 0; q < 6; ++q) o[q] = 0.0;
        if (!cnt) continue;
        const double inv = 1.0 / (double)cnt;   // Monitor.cpp:1210-1222
        o[0] = ha[5 * k] * inv;       // P2
        o[1] = ha[5 * k + 1] * inv;   // first bond length
        o[2] = ha[5 * k + 2] * inv;   // second bond length
        o[3] = ha[5 * k + 3] * inv;   // phi - phi0
        o[4] = ha[5 * k + 4] * inv;   // (phi - phi0)^2
        o[5] = o[3] > 0.0 ? o[4] / (o[3] * o[3]) : 0.0;   // m_vBondPairPhiRatio
    }
    return DPD_OK;
}

static int run_download(dpd_engine* e, double* x3, double* u3, double* v3, double* f3, double* st9, int32_t* cell);

int dpd_engine_set_restart_layout(dpd_engine* e, int64_t n, const int64_t* order, const int64_t* poly_id,
                                  const int32_t* poly_type, const double* radius_by_type)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "restart files cover a whole box; a slab also holds ghosts");
    if (!e->uploaded) return fail(e, DPD_E_STATE, "upload beads before the restart layout");
    if (n != e->n || !order || !poly_id || !poly_type || !radius_by_type)
        return fail(e, DPD_E_ARG, "the restart layout needs every bead, its polymer id and type, and the radii");
    std::vector<char> seen((size_t)n, 0);
    for (int64_t k = 0; k < n; ++k) {
        if (order[k] < 0 || order[k] >= n || seen[(size_t)order[k]])
            return fail(e, DPD_E_ARG, "restart order is not a permutation of the upload indices");
        seen[(size_t)order[k]] = 1;
    }
    e->rs_order.assign(order, order + n);
    e->rs_poly_id.assign(poly_id, poly_id + n);
    e->rs_poly_type.assign(poly_type, poly_type + n);
    e->rs_radius.assign(radius_by_type, radius_by_type + e->ntypes);
    return DPD_OK;
}

int dpd_engine_write_restart(dpd_engine* e, const char* path, int32_t wall, int32_t gravity, int32_t shear)
{
    if (!e) return DPD_E_ARG;
    if (!path) return fail(e, DPD_E_ARG, "null path");
    if (e->rs_order.empty() || (int64_t)e->rs_order.size() != e->n)
        return fail(e, DPD_E_STATE, "dpd_engine_set_restart_layout has not been called for these beads");
    if (e->hboxes.size() > 1) return fail(e, DPD_E_STATE, "restart files are written for single-box engines");
    const int64_t n = e->n;
    std::vector<double> x(3 * n), u(3 * n), v(3 * n), f(3 * n);
    int rc = run_download(e, x.data(), u.data(), v.data(), f.data(), nullptr, nullptr);
    if (rc) return rc;
    if ((rc = host_ids(e))) return rc;
    const double* L = e->hboxes[0].L;
    // CRestartState::CheckBeadWithinBox (RestartState.cpp:488-530): a
    // coordinate past the box length is an error, one within 0.001 of a face
    // is written as 0.001
    const double lim = 0.001;
    for (int64_t b = 0; b < n; ++b)
        for (int d = 0; d < 3; ++d) {
            double& c = x[3 * b + d];
            if (c > L[d]) return fail(e, DPD_E_BOX, "bead coordinate outside the box writing a restart state");
            if (c > L[d] - lim || c < lim) c = lim;
        }
    // CRestartState::Serialize (RestartState.cpp:113-163): the constraint
    // flags, then one line per bead in polymer order with the stream's default
    // 6-significant-digit formatting; lines formatted in parallel chunks
    const int nth = (int)std::max<unsigned>(1, std::min<unsigned>(16, std::thread::hardware_concurrency()));
    std::vector<std::string> parts(nth);
    auto work = [&](int t) {
        const int64_t k0 = n * t / nth, k1 = n * (t + 1) / nth;
        std::string& out = parts[t];
        out.reserve((size_t)(k1 - k0) * 200);
        char line[512];
        for (int64_t k = k0; k < k1; ++k) {
            const int64_t b = e->rs_order[k];
            const double* X = &x[3 * b];
            const double* U = &u[3 * b];
            const double* V = &v[3 * b];
            const double* F = &f[3 * b];
            const int len = snprintf(line, sizeof line,
                                     "%lld %d %lld %d %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g %.6g\n",
                                     (long long)e->rs_poly_id[k], e->rs_poly_type[k], (long long)e->h_id[b],
                                     e->h_type[b], e->rs_radius[e->h_type[b]], X[0], X[1], X[2], U[0], U[1], U[2],
                                     V[0], V[1], V[2], F[0], F[1], F[2]);
            out.append(line, (size_t)len);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    FILE* fp = fopen(path, "wb");
    if (!fp) return fail(e, DPD_E_ARG, std::string("cannot open ") + path);
    bool ok = fprintf(fp, "%d %d %d\n", wall ? 1 : 0, gravity ? 1 : 0, shear ? 1 : 0) > 0;
    for (auto& pstr : parts) ok = ok && fwrite(pstr.data(), 1, pstr.size(), fp) == pstr.size();
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return fail(e, DPD_E_ARG, std::string("write failed: ") + path);
    return DPD_OK;
}

// The Paraview snapshot of CCurrentState::Serialize with CParaviewFormat
// (CurrentState.cpp:163-244, ParaviewFormat.cpp:72-112) for n beads in file
// order: the format's header lines (with their trailing tabs and spaces), one
// "x y z" line per bead with the stream's default 6-significant-digit
// formatting, the vertex list and one display id per bead.
static bool write_paraview_file(const char* path, int64_t n, const double* x3, const int32_t* display_id)
{
    const int nth = (int)std::max<unsigned>(1, std::min<unsigned>(16, std::thread::hardware_concurrency()));
    std::vector<std::string> parts(nth);
    auto work = [&](int t) {
        const int64_t k0 = n * t / nth, k1 = n * (t + 1) / nth;
        std::string& out = parts[t];
        out.reserve((size_t)(k1 - k0) * 40);
        char line[128];
        for (int64_t k = k0; k < k1; ++k) {
            const int len = snprintf(line, sizeof line, "%.6g %.6g %.6g\n", x3[3 * k], x3[3 * k + 1], x3[3 * k + 2]);
            out.append(line, (size_t)len);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    FILE* fp = fopen(path, "wb");
    if (!fp) return false;
    bool ok = fprintf(fp,
                      "# vtk DataFile Version 2.0\t\t\t    \n"
                      "data\t\t\t\t\t\t\t\t\t\t\n"
                      "ASCII\t\t\t\t\t\t\t\t\t\n"
                      "DATASET POLYDATA\t\t\t\t\t\t    \n"
                      "POINTS %lld double\t\t\n",
                      (long long)n) > 0;
    for (auto& pstr : parts) ok = ok && fwrite(pstr.data(), 1, pstr.size(), fp) == pstr.size();
    ok = ok && fprintf(fp, "VERTICES  %lld %lld\n", (long long)n, (long long)(2 * n)) > 0;
    std::string tail;
    tail.reserve((size_t)n * 12 + 64);
    char line[64];
    for (int64_t k = 0; k < n; ++k) tail.append(line, (size_t)snprintf(line, sizeof line, "1 %lld\n", (long long)k));
    tail.append("POINT_DATA ");
    tail.append(std::to_string((long long)n));
    tail.append("\nSCALARS ptype float 1\nLOOKUP_TABLE  default\n");
    for (int64_t k = 0; k < n; ++k) tail.append(line, (size_t)snprintf(line, sizeof line, "%d\n", display_id[k]));
    ok = ok && fwrite(tail.data(), 1, tail.size(), fp) == tail.size();
    ok = (fclose(fp) == 0) && ok;
    return ok;
}

int dpd_write_paraview(const char* path, int64_t n, const double* x3, const int32_t* display_id)
{
    if (!path || n < 0 || (n > 0 && (!x3 || !display_id))) return DPD_E_ARG;
    return write_paraview_file(path, n, x3, display_id) ? DPD_OK : DPD_E_ARG;
}

int dpd_engine_write_paraview(dpd_engine* e, const char* path, const uint8_t* type_visible, const int32_t* display_id)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "snapshots cover a whole box; a slab also holds ghosts");
    if (!path) return fail(e, DPD_E_ARG, "null path");
    if (e->hboxes.size() > 1) return fail(e, DPD_E_STATE, "snapshots are written for single-box engines");
    const int64_t n = e->n;
    std::vector<double> x(3 * (size_t)n);
    std::vector<int32_t> cell((size_t)n);
    int rc = run_download(e, x.data(), nullptr, nullptr, nullptr, nullptr, cell.data());
    if (rc) return rc;
    if ((rc = host_ids(e))) return rc;
    // CSimBox::GetAllBeadsInCNTCells (SimBox.cpp:5883-5895): cells in index
    // order; inside a cell the reference keeps its list order, the engine the
    // upload order.  Beads of invisible types are left out (CurrentState.cpp:
    // 207-223).
    std::vector<int64_t> order;
    order.reserve((size_t)n);
    for (int64_t b = 0; b < n; ++b)
        if (!type_visible || type_visible[e->h_type[(size_t)b]]) order.push_back(b);
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t p, int64_t q) { return cell[(size_t)p] < cell[(size_t)q]; });
    const int64_t m = (int64_t)order.size();
    std::vector<double> xo(3 * (size_t)m);
    std::vector<int32_t> ids((size_t)m);
    for (int64_t k = 0; k < m; ++k) {
        const int64_t b = order[(size_t)k];
        for (int d = 0; d < 3; ++d) xo[3 * (size_t)k + d] = x[3 * (size_t)b + d];
        // the reference's default display id is the bead type (Monitor.cpp:277)
        ids[(size_t)k] = display_id ? display_id[b] : e->h_type[(size_t)b];
    }
    if (!write_paraview_file(path, m, xo.data(), ids.data()))
        return fail(e, DPD_E_ARG, std::string("write failed: ") + path);
    return DPD_OK;
}

int dpd_engine_set_pair_params(dpd_engine* e, int32_t ntypes, const double* a, const double* gamma)
{
    if (!e) return DPD_E_ARG;
    if (ntypes < 1 || ntypes > kMaxTypes || !a || !gamma) return fail(e, DPD_E_ARG, "bad pair tables");
    if (ntypes < e->ntypes) return fail(e, DPD_E_ARG, "bead types cannot be removed");
    const int m = ntypes * ntypes;
    for (int i = 0; i < ntypes; ++i)
        for (int j = 0; j < ntypes; ++j)
            if (a[i * ntypes + j] != a[j * ntypes + i] || gamma[i * ntypes + j] != gamma[j * ntypes + i])
                return fail(e, DPD_E_ARG, "pair tables must be symmetric");
    if (ntypes != e->ntypes && e->hboxes.size() > 1) return fail(e, DPD_E_ARG, "a batch keeps its bead types");
    if (ntypes != e->ntypes) {
        // the pair kernel's shared-memory size and the captured graphs depend on ntypes
        memset(e->pair_attr_set, 0, sizeof e->pair_attr_set);
        CU(cudaSetDevice(e->device));
        CU(cudaStreamSynchronize(e->s()));
        drop_graphs(e);
    }
    e->ntypes = ntypes;
    e->a.assign(a, a + m);
    e->gamma.assign(gamma, gamma + m);
    if (e->hboxes.size() == 1) {
        e->box_a = e->a;
        e->box_g = e->gamma;
    } else {
        for (size_t k = 0; k < e->hboxes.size(); ++k) {
            std::copy(a, a + m, e->box_a.begin() + k * m);
            std::copy(gamma, gamma + m, e->box_g.begin() + k * m);
        }
    }
    CU(cudaSetDevice(e->device));
    return push_constants(e);
}

int dpd_engine_set_dt(dpd_engine* e, double dt)
{
    if (!e) return DPD_E_ARG;
    if (!(dt > 0.0)) return DPD_OK;   // ChangeTimeStepConstants ignores dt <= 0 (CNTCell.cpp:359)
    e->params.dt = dt;
    CU(cudaSetDevice(e->device));
    return push_constants(e);
}

int dpd_engine_set_thermostat(dpd_engine* e, int32_t on)
{
    if (!e) return DPD_E_ARG;
    e->thermostat_on = on != 0;
    CU(cudaSetDevice(e->device));
    return push_constants(e);
}

int dpd_engine_set_conservative(dpd_engine* e, int32_t on)
{
    if (!e) return DPD_E_ARG;
    e->conservative_on = on != 0;
    CU(cudaSetDevice(e->device));
    return push_constants(e);
}

int dpd_engine_renormalise_mom(dpd_engine* e)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "a slab holds ghosts: renormalise through the ranks' owned sums");
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    if (e->hboxes.size() != 1) return fail(e, DPD_E_ARG, "momentum renormalisation is for single-box engines");
    if (!(e->params.kT > 0.0)) return fail(e, DPD_E_ARG, "momentum renormalisation needs kT > 0");
    CU(cudaSetDevice(e->device));
    int rc;
    // the next step's drift, if done ahead, used the old momenta
    if ((rc = drop_ahead(e))) return rc;
    const int n = (int)e->n;
    const int nb = blocks_for(n, kThreads);
    double* v = e->d_v[e->cur];
    k_kinetic_partials<<<nb, kThreads, 0, e->s()>>>(n, e->d_x[e->cur], v, e->d_partials);
    if ((rc = check_launch(e, "k_kinetic_partials"))) return rc;
    k_reduce_obs<<<1, 32 * kObsTerms, 0, e->s()>>>(nb, e->d_partials, e->d_renorm);
    if ((rc = check_launch(e, "k_reduce_obs"))) return rc;
    k_renorm_scale<<<nb, kThreads, 0, e->s()>>>(n, v, e->d_renorm, 3.0 * (double)n * e->params.kT);
    if ((rc = check_launch(e, "k_renorm_scale"))) return rc;
    e->obs_valid = false;
    return DPD_OK;
}

int dpd_engine_step(dpd_engine* e, int64_t first_step, int32_t nsteps)
{
    if (!e) return DPD_E_ARG;
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    if (nsteps < 0) return fail(e, DPD_E_ARG, "negative step count");
    // The status word as published by the latest call whose device work has
    // started (no wait): a fatal bit stops the run here, as the reference's
    // CLogSimErrorTrace + ccStopNoSave would (SimBox.cpp:436-445), and no
    // further work is queued on the invalid state.
    const unsigned seen = *(volatile unsigned*)e->h_seen;
    if (seen & DPD_STATUS_FATAL_MASK) {
        char msg[160];
        snprintf(msg, sizeof msg, "device status 0x%x: %s%s%s%s", seen,
                 (seen & DPD_STATUS_NONFINITE) ? "non-finite position, velocity or force; " : "",
                 (seen & DPD_STATUS_IMAGE_OVERFLOW) ? "periodic image counter overflow; " : "",
                 (seen & DPD_STATUS_INTERNAL) ? "internal capacity check; " : "",
                 (seen & DPD_STATUS_SLAB_REACH) ? "a bond reaches beyond the slab's ghost layers" : "");
        return fail(e, DPD_E_STATUS, msg);
    }
    if (nsteps == 0) return DPD_OK;
    CU(cudaSetDevice(e->device));
    // the step counter keys the pair noise; it is advanced on the device by
    // every step's k_update_mom, so it is set only when this call does not
    // continue where the queued work ends
    const bool continues = first_step == e->dev_step;
    e->dev_step = INT64_MIN;   // until this call's steps are all queued
    if (!continues) {
        k_set_step<<<1, 1, 0, e->s()>>>(e->d_step, first_step, e->d_status, e->d_seen);
        CU(cudaGetLastError());
        e->launches += 1;
    }
    std::vector<char> samples(nsteps);
    const bool from_ahead = e->ahead_valid, to_ahead = e->ahead_enabled;
    for (int32_t k = 0; k < nsteps; ++k) {
        const int64_t t = first_step + k;
        // ISimState::TimeToSample (ISimState.cpp:468-471): m_SimTime % SamplePeriod == 0
        samples[k] = e->sample_period > 0 ? (t % e->sample_period == 0) : (k == nsteps - 1);
    }
    auto queue_all = [&](void) -> int {
        for (int32_t k = 0; k < nsteps; ++k) {
            const bool first = k == 0, last = k == nsteps - 1;
            const int rc = (e->precision == DPD_PRECISION_FP64)
                               ? queue_step<double>(e, samples[k], first, last, from_ahead, to_ahead)
                               : queue_step<float>(e, samples[k], first, last, from_ahead, to_ahead);
            if (rc) return rc;
        }
        return DPD_OK;
    };
    const int parity = e->cur;
    if (e->graphs_enabled && !e->profiling) {
        // one captured graph per (step count, buffer parity, sample pattern, stream)
        dpd_engine::Graph* g = nullptr;
        for (auto& cand : e->graphs)
            if (cand.nsteps == nsteps && cand.parity == parity && cand.samples == samples && cand.stream == e->s() &&
                cand.from_ahead == from_ahead && cand.to_ahead == to_ahead)
                g = &cand;
        if (!g) {
            if (e->graphs.size() >= 16) drop_graphs(e);
            // kernel attributes are set outside the capture
            const int rc0 = (e->precision == DPD_PRECISION_FP64) ? set_pair_attributes<double>(e)
                                                                  : set_pair_attributes<float>(e);
            if (rc0) return rc0;
            cudaGraph_t graph = nullptr;
            CU(cudaStreamBeginCapture(e->s(), cudaStreamCaptureModeThreadLocal));
            const int64_t launches0 = e->launches;
            const int rc = queue_all();
            cudaError_t ce = cudaStreamEndCapture(e->s(), &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                e->cur = parity;
                return rc;
            }
            if (ce != cudaSuccess) return fail(e, DPD_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            cudaGraphExec_t exec = nullptr;
            ce = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) return fail(e, DPD_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
            e->graphs.push_back({nsteps, parity, from_ahead, to_ahead, samples, e->s(), exec, e->launches - launches0});
            g = &e->graphs.back();
            e->launches = launches0;   // counted per replay below
            e->cur = parity;
        }
        CU(cudaGraphLaunch(g->exec, e->s()));
        e->launches += g->launches;
        e->cur = (nsteps % 2) ? 1 - parity : parity;
    } else {
        const int rc = queue_all();
        if (rc) return rc;
    }
    for (int32_t k = nsteps - 1; k >= 0; --k)
        if (samples[k]) {
            e->sampled = true;
            e->last_sample_step = first_step + k;
            break;
        }
    e->ahead_valid = to_ahead;
    e->dev_step = first_step + nsteps;
    e->stepped = true;
    e->obs_valid = false;
    e->box_obs_valid = false;
    e->obs_has_virial = true;
    e->last_step = first_step + nsteps - 1;
    return DPD_OK;
}

int dpd_engine_status(dpd_engine* e, uint32_t* bits)
{
    if (!e) return DPD_E_ARG;
    CU(cudaSetDevice(e->device));
    CU(cudaMemcpyAsync(e->h_status, e->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    if (bits) *bits = *e->h_status;
    *(volatile unsigned*)e->h_seen = *e->h_status;   // nothing in flight: the next step call sees it at once
    return DPD_OK;
}

static int run_download(dpd_engine* e, double* x3, double* u3, double* v3, double* f3, double* st9, int32_t* cell)
{
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    CU(cudaSetDevice(e->device));
    const int n = (int)e->n;
    double* o = e->d_out;
    double *ox = x3 ? o : nullptr, *ou = u3 ? o + 3 * (size_t)n : nullptr, *ov = v3 ? o + 6 * (size_t)n : nullptr,
           *of = f3 ? o + 9 * (size_t)n : nullptr, *ost = st9 ? o + 12 * (size_t)n : nullptr;
    const int c = e->cur;
    if (e->precision == DPD_PRECISION_FP64)
        k_download<double><<<blocks_for(n, kThreads), kThreads, 0, e->s()>>>(
            n, e->d_boxes, e->d_tf[c], e->d_bid[c], e->d_x[c], e->d_v[c], (const double*)e->d_F, e->d_img[c], e->off_active ? e->d_off : nullptr,
            e->sampled ? (const double*)e->d_stress : nullptr, e->d_cell[c], ox, ou, ov, of, ost,
            cell ? e->d_out_cell : nullptr);
    else
        k_download<float><<<blocks_for(n, kThreads), kThreads, 0, e->s()>>>(
            n, e->d_boxes, e->d_tf[c], e->d_bid[c], e->d_x[c], e->d_v[c], (const float*)e->d_F, e->d_img[c], e->off_active ? e->d_off : nullptr,
            e->sampled ? (const float*)e->d_stress : nullptr, e->d_cell[c], ox, ou, ov, of, ost,
            cell ? e->d_out_cell : nullptr);
    int rc = check_launch(e, "k_download");
    if (rc) return rc;
    if (x3) CU(cudaMemcpyAsync(x3, ox, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, e->s()));
    if (u3) CU(cudaMemcpyAsync(u3, ou, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, e->s()));
    if (v3) CU(cudaMemcpyAsync(v3, ov, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, e->s()));
    if (f3) CU(cudaMemcpyAsync(f3, of, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, e->s()));
    if (st9) CU(cudaMemcpyAsync(st9, ost, 9 * sizeof(double) * n, cudaMemcpyDeviceToHost, e->s()));
    if (cell) CU(cudaMemcpyAsync(cell, e->d_out_cell, sizeof(int) * n, cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    return DPD_OK;
}

int dpd_engine_download(dpd_engine* e, double* x3, double* unpbc3, double* v3, double* f3, double* stress9)
{
    if (!e) return DPD_E_ARG;
    return run_download(e, x3, unpbc3, v3, f3, stress9, nullptr);
}

int dpd_engine_bead_ids(dpd_engine* e, int64_t* id, int32_t* type)
{
    if (!e) return DPD_E_ARG;
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    CU(cudaSetDevice(e->device));
    if (int rc = host_ids(e)) return rc;
    if (id) memcpy(id, e->h_id.data(), sizeof(int64_t) * (size_t)e->n);
    if (type) memcpy(type, e->h_type.data(), sizeof(int32_t) * (size_t)e->n);
    return DPD_OK;
}

int dpd_engine_cells(dpd_engine* e, int32_t* cell)
{
    if (!e) return DPD_E_ARG;
    if (!cell) return fail(e, DPD_E_ARG, "null cell array");
    return run_download(e, nullptr, nullptr, nullptr, nullptr, nullptr, cell);
}

int dpd_engine_observables(dpd_engine* e, dpd_obs* out)
{
    if (!e) return DPD_E_ARG;
    if (e->slab) return fail(e, DPD_E_STATE, "a slab also holds ghosts: dpd_engine_slab_observables");
    if (!out) return fail(e, DPD_E_ARG, "null output");
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    CU(cudaSetDevice(e->device));
    const int n = (int)e->n;
    if (!e->sampled) {
        const int nb = blocks_for(n, kThreads);
        k_kinetic_partials<<<nb, kThreads, 0, e->s()>>>(n, e->d_x[e->cur], e->d_v[e->cur], e->d_partials);
        int rc = check_launch(e, "k_kinetic_partials");
        if (rc) return rc;
        k_reduce_obs<<<1, 32 * kObsTerms, 0, e->s()>>>(nb, e->d_partials, e->d_obs);
        if ((rc = check_launch(e, "k_reduce_obs"))) return rc;
    }
    CU(cudaMemcpyAsync(e->h_obs, e->d_obs, kObsTerms * sizeof(double), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    const double* h = e->h_obs;
    memset(out, 0, sizeof *out);
    out->step = e->sampled ? e->last_sample_step : (e->stepped ? e->last_step : 0);
    out->n = e->n;
    for (int d = 0; d < 3; ++d) {
        out->sum_v[d] = h[d];
        out->sum_v2[d] = h[3 + d];
        out->sum_x[d] = h[15 + d];
        out->ang_mom[d] = h[18 + d];
    }
    out->has_virial = e->sampled ? 1 : 0;
    for (int q = 0; q < 9; ++q) out->virial[q] = e->sampled ? h[6 + q] : 0.0;
    const dpd_params& p = e->params;
    const double V = (p.nx * p.wx) * (p.ny * p.wy) * (p.nz * p.wz);
    const double v2 = out->sum_v2[0] + out->sum_v2[1] + out->sum_v2[2];
    out->kT = v2 / (3.0 * (double)e->n);
    out->pressure = 0.3333333333 * (1.0 / V) * (v2 + out->virial[0] + out->virial[4] + out->virial[8]);
    return DPD_OK;
}

int dpd_batch_observables(dpd_engine* e, int32_t box, dpd_obs* out)
{
    if (!e) return DPD_E_ARG;
    if (!out) return fail(e, DPD_E_ARG, "null output");
    if (!e->uploaded) return fail(e, DPD_E_STATE, "no beads uploaded");
    if (box < 0 || box >= (int32_t)e->hboxes.size()) return fail(e, DPD_E_ARG, "box index out of range");
    CU(cudaSetDevice(e->device));
    const int nb = (int)e->hboxes.size();
    if (!e->box_obs_valid) {
        const int c = e->cur;
        if (e->precision == DPD_PRECISION_FP64)
            k_box_sums<double><<<nb, 256, 0, e->s()>>>(e->d_boxes, e->d_start, (int)e->n, e->d_x[c], e->d_v[c],
                                                       e->sampled ? (const double*)e->d_stress : nullptr,
                                                       e->d_box_obs);
        else
            k_box_sums<float><<<nb, 256, 0, e->s()>>>(e->d_boxes, e->d_start, (int)e->n, e->d_x[c], e->d_v[c],
                                                      e->sampled ? (const float*)e->d_stress : nullptr,
                                                      e->d_box_obs);
        int rc = check_launch(e, "k_box_sums");
        if (rc) return rc;
        e->box_obs_valid = true;
    }
    double h[kObsTerms];
    CU(cudaMemcpyAsync(h, e->d_box_obs + (size_t)box * kObsTerms, sizeof h, cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    int64_t nbox = 0;
    {
        int se[2];
        const Box& B = e->hboxes[box];
        CU(cudaMemcpy(&se[0], e->d_start + B.cell_base, sizeof(int), cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(&se[1], e->d_start + B.cell_base + B.nc[0] * B.nc[1] * B.nc[2], sizeof(int),
                      cudaMemcpyDeviceToHost));
        nbox = se[1] - se[0];
    }
    memset(out, 0, sizeof *out);
    out->step = e->sampled ? e->last_sample_step : (e->stepped ? e->last_step : 0);
    out->n = nbox;
    for (int d = 0; d < 3; ++d) {
        out->sum_v[d] = h[d];
        out->sum_v2[d] = h[3 + d];
        out->sum_x[d] = h[15 + d];
        out->ang_mom[d] = h[18 + d];
    }
    out->has_virial = e->sampled ? 1 : 0;
    for (int q = 0; q < 9; ++q) out->virial[q] = h[6 + q];
    const Box& B = e->hboxes[box];
    const double V = B.L[0] * B.L[1] * B.L[2];
    const double v2 = out->sum_v2[0] + out->sum_v2[1] + out->sum_v2[2];
    out->kT = nbox > 0 ? v2 / (3.0 * (double)nbox) : 0.0;
    out->pressure = 0.3333333333 * (1.0 / V) * (v2 + out->virial[0] + out->virial[4] + out->virial[8]);
    return DPD_OK;
}

// ===================================================== z-slab decomposition

// The local box's bonds and bond pairs: the whole box's terms whose beads are
// all in the local box, per bead in the single-box build's order, with the
// bead indices of the current upload (k_slab_* in slab.cuh).  With check, an
// owned bead that loses a term sets DPD_STATUS_SLAB_REACH (not at setup,
// before the first exchange has brought the ghosts).
static int slab_topology(dpd_engine* e, bool check)
{
    SlabState& S = *e->slab;
    const int n = (int)e->n;
    cudaStream_t st = e->s();
    int rc;
    bool moved = false;
    if (++S.version == 0) {   // the map's entries carry the version: a wrap clears it
        CU(cudaMemsetAsync(S.d_idmap, 0, sizeof(unsigned long long) * ((size_t)S.id_max + 1), st));
        S.version = 1;
    }
    const SlabTopo T{S.nb, S.na, S.id_max, S.d_head_id, S.d_tail_id, S.d_first, S.d_second, S.d_gptr, S.d_gterm};
    k_slab_idmap<<<blocks_for(n, kThreads), kThreads, 0, st>>>(n, S.id_max, e->d_pid_of, S.version, S.d_idmap);
    if ((rc = check_launch(e, "k_slab_idmap"))) return rc;
    const int m = std::max(S.nb, S.na);
    if (m > 0) {
        k_slab_endpoints<<<blocks_for(m, kThreads), kThreads, 0, st>>>(T, S.d_idmap, S.version, e->d_bond_h,
                                                                      e->d_bond_t, e->d_ang[0], e->d_ang[1],
                                                                      e->d_ang[2], e->d_ang[3]);
        if ((rc = check_launch(e, "k_slab_endpoints"))) return rc;
    }
    const int nblk = blocks_for(n, kThreads);
    const size_t room = with_room(e, (size_t)n);   // the count changes every step
    if ((rc = ensure(e, &S.d_cnt, S.cap_cnt, (size_t)n, &moved, room))) return rc;
    if ((rc = ensure(e, &S.d_bsum, S.cap_bsum, (size_t)nblk, &moved, (size_t)blocks_for(room, kThreads)))) return rc;
    if ((rc = ensure(e, &e->d_csr_ptr, e->cap_csr_ptr, (size_t)n + 1, &moved, room + 1))) return rc;
    if ((rc = ensure(e, &e->d_csr_term, e->cap_csr_term, std::max<size_t>(S.nterm, 1), &moved))) return rc;
    k_slab_term_count<<<nblk, kThreads, 0, st>>>(n, check ? S.geom.n_owned : 0, T, e->d_pid_of, e->d_bond_h, e->d_bond_t,
                                                 e->d_ang[0], e->d_ang[1], e->d_ang[2], e->d_ang[3], S.d_cnt,
                                                 e->d_status);
    if ((rc = check_launch(e, "k_slab_term_count"))) return rc;
    k_scan_block_sums<<<nblk, kThreads, 0, st>>>(n, S.d_cnt, S.d_bsum);
    if ((rc = check_launch(e, "k_scan_block_sums"))) return rc;
    k_scan_top<<<1, 1024, 0, st>>>(nblk, S.d_bsum);
    if ((rc = check_launch(e, "k_scan_top"))) return rc;
    k_scan_apply<<<nblk, kThreads, 0, st>>>(n, S.d_cnt, S.d_bsum, e->d_csr_ptr);
    if ((rc = check_launch(e, "k_scan_apply"))) return rc;
    k_slab_term_write<<<nblk, kThreads, 0, st>>>(n, T, e->d_pid_of, e->d_bond_h, e->d_bond_t, e->d_ang[0],
                                                 e->d_ang[1], e->d_ang[2], e->d_ang[3], e->d_csr_ptr, e->d_csr_term,
                                                 (int)std::min<size_t>(e->cap_csr_term, INT_MAX));
    if ((rc = check_launch(e, "k_slab_term_write"))) return rc;
    // every local bead runs through the bonded kernel (beads without terms
    // leave it at once): the bonded-bead list is 0..n-1
    if ((rc = ensure(e, &e->d_ubuf, e->cap_ubuf, (size_t)n, &moved, room))) return rc;
    if ((rc = ensure(e, &e->d_Fb, e->cap_Fb, (size_t)n, &moved, room))) return rc;
    if ((rc = ensure(e, &e->d_Sb, e->cap_Sb, 9 * (size_t)n, &moved, 9 * room))) return rc;
    if (!e->d_bb || S.cap_bb < (size_t)n) {
        if ((rc = ensure(e, &e->d_bb, e->cap_bb, (size_t)n, &moved, room))) return rc;
        k_iota<<<blocks_for(e->cap_bb, kThreads), kThreads, 0, st>>>((int)e->cap_bb, e->d_bb);
        if ((rc = check_launch(e, "k_iota"))) return rc;
        S.cap_bb = e->cap_bb;
    }
    e->nbb = n;
    k_mark_bonded<<<nblk, kThreads, 0, st>>>(n, e->d_bid[e->cur], e->d_csr_ptr, e->d_tf[e->cur]);
    if ((rc = check_launch(e, "k_mark_bonded"))) return rc;
    e->topo_nb = S.nb;
    e->topo_na = S.na;
    return DPD_OK;
}

int dpd_engine_slab_setup(dpd_engine* e, int32_t nz_global, int32_t z0, int32_t z1, int32_t ghost, int64_t n_owned,
                          int64_t id_max, int64_t nb, const int64_t* bond_head_id, const int64_t* bond_tail_id,
                          const double* k2, const double* l0, int64_t na, const int64_t* first_bond,
                          const int64_t* second_bond, const double* k3, const double* phi0)
{
    if (!e) return DPD_E_ARG;
    if (!e->uploaded) return fail(e, DPD_E_STATE, "upload the slab's owned beads first");
    if (e->hboxes.size() > 1) return fail(e, DPD_E_STATE, "a slab is a single-box engine");
    if (e->slab) return fail(e, DPD_E_STATE, "the engine is a slab already");
    const Box& B = e->hboxes[0];
    const int own = z1 - z0;
    if (ghost < 1 || z0 < 0 || own < 2 * ghost || z1 > nz_global || own + 2 * ghost > nz_global ||
        B.nc[2] != own + 2 * ghost)
        return fail(e, DPD_E_ARG, "slab layers: 0 <= z0, 2*ghost <= z1 - z0, (z1 - z0) + 2*ghost <= nz_global, "
                                  "and the engine's box holds z1 - z0 + 2*ghost layers");
    if (n_owned < 0 || n_owned > e->n) return fail(e, DPD_E_ARG, "owned beads outside 0..n");
    if (nb < 0 || na < 0 || (nb && (!bond_head_id || !bond_tail_id || !k2 || !l0)) ||
        (na && (!first_bond || !second_bond || !k3 || !phi0)))
        return fail(e, DPD_E_ARG, "bad topology arrays");
    if ((nb || na) && (id_max < 1 || id_max > 0x7fffffff)) return fail(e, DPD_E_ARG, "id_max outside 1..2^31-1");
    if (nb * 2 + na * 3 > ((int64_t)1 << 28)) return fail(e, DPD_E_ARG, "topology too large");
    for (int64_t i = 0; i < nb; ++i)
        if (bond_head_id[i] < 1 || bond_head_id[i] > id_max || bond_tail_id[i] < 1 || bond_tail_id[i] > id_max ||
            bond_head_id[i] == bond_tail_id[i])
            return fail(e, DPD_E_ARG, "bond refers to a bead id outside 1..id_max or joins a bead to itself");
    for (int64_t i = 0; i < na; ++i)
        if (first_bond[i] < 0 || first_bond[i] >= nb || second_bond[i] < 0 || second_bond[i] >= nb)
            return fail(e, DPD_E_ARG, "bond pair refers to an unknown bond");
    CU(cudaSetDevice(e->device));
    CU(cudaStreamSynchronize(e->s()));
    if (int rc0 = drop_ahead(e)) return rc0;
    drop_graphs(e);
    release_topology(e);
    if (int rc0 = empty_topology(e, false)) return rc0;
    std::unique_ptr<SlabState> S(new SlabState());
    S->geom.z0 = z0;
    S->geom.z1 = z1;
    S->geom.g = ghost;
    S->geom.nzg = nz_global;
    S->geom.w = B.w[2];
    S->geom.Lz = (double)nz_global * B.w[2];
    S->geom.c = (double)(z0 - ghost) * B.w[2];
    S->geom.n_owned = (int)n_owned;
    if (cudaHostAlloc((void**)&S->h_sizes, 16 * sizeof(int), cudaHostAllocMapped) != cudaSuccess)
        return fail(e, DPD_E_CUDA, "pinned allocation failed");
    if (cudaHostGetDevicePointer((void**)&S->d_sizes, S->h_sizes, 0) != cudaSuccess) {
        cudaFreeHost(S->h_sizes);
        return fail(e, DPD_E_CUDA, "mapped pinned memory unavailable");
    }
    memset(S->h_sizes, 0, 16 * sizeof(int));
    int rc;
    if ((rc = dalloc(e, &S->d_total, (size_t)kSlabOuts))) { cudaFreeHost(S->h_sizes); return rc; }
    S->topo = nb > 0 || na > 0;
    if (S->topo) {
        S->nb = (int)nb;
        S->na = (int)na;
        S->id_max = (int)id_max;
        // the whole box's term lists by bead id, in the single-box build's
        // order (bonds by index, head and tail; then bond pairs by index)
        std::vector<int> cnt((size_t)id_max + 2, 0);
        for (int64_t i = 0; i < nb; ++i) { cnt[(size_t)bond_head_id[i] + 1]++; cnt[(size_t)bond_tail_id[i] + 1]++; }
        for (int64_t i = 0; i < na; ++i) {
            cnt[(size_t)bond_tail_id[first_bond[i]] + 1]++;
            cnt[(size_t)bond_head_id[first_bond[i]] + 1]++;
            cnt[(size_t)bond_head_id[second_bond[i]] + 1]++;
        }
        for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
        S->nterm = (size_t)cnt.back();
        std::vector<int> gterm(std::max<size_t>(S->nterm, 1)), fillp(cnt.begin(), cnt.end() - 1);
        for (int64_t i = 0; i < nb; ++i) {
            gterm[(size_t)fillp[(size_t)bond_head_id[i]]++] = (int)(i * 8 + kBondHead);
            gterm[(size_t)fillp[(size_t)bond_tail_id[i]]++] = (int)(i * 8 + kBondTail);
        }
        for (int64_t i = 0; i < na; ++i) {
            gterm[(size_t)fillp[(size_t)bond_tail_id[first_bond[i]]]++] = (int)(i * 8 + kAngle0);
            gterm[(size_t)fillp[(size_t)bond_head_id[first_bond[i]]]++] = (int)(i * 8 + kAngle1);
            gterm[(size_t)fillp[(size_t)bond_head_id[second_bond[i]]]++] = (int)(i * 8 + kAngle2);
        }
        std::vector<int> hid((size_t)std::max<int64_t>(nb, 1)), tid((size_t)std::max<int64_t>(nb, 1));
        for (int64_t i = 0; i < nb; ++i) { hid[(size_t)i] = (int)bond_head_id[i]; tid[(size_t)i] = (int)bond_tail_id[i]; }
        std::vector<int> fb((size_t)std::max<int64_t>(na, 1)), sb((size_t)std::max<int64_t>(na, 1));
        std::vector<double> ak(3 * (size_t)std::max<int64_t>(na, 1));
        for (int64_t i = 0; i < na; ++i) {
            fb[(size_t)i] = (int)first_bond[i];
            sb[(size_t)i] = (int)second_bond[i];
            // as the single-box build: cos/sin of phi0, sin0 = 0 selecting the phi0 <= 0 branch
            ak[(size_t)i] = k3[i];
            ak[(size_t)na + i] = phi0[i] > 0.0 ? std::cos(phi0[i]) : 1.0;
            ak[2 * (size_t)na + i] = phi0[i] > 0.0 ? std::sin(phi0[i]) : 0.0;
        }
        const size_t nbs = (size_t)std::max<int64_t>(nb, 1), nas = (size_t)std::max<int64_t>(na, 1);
        bool moved = false;
        size_t c;
        if ((rc = dalloc(e, &S->d_head_id, nbs)) || (rc = dalloc(e, &S->d_tail_id, nbs)) ||
            (rc = dalloc(e, &S->d_first, nas)) || (rc = dalloc(e, &S->d_second, nas)) ||
            (rc = dalloc(e, &S->d_gptr, cnt.size())) || (rc = dalloc(e, &S->d_gterm, gterm.size())) ||
            (rc = dalloc(e, &S->d_idmap, (size_t)id_max + 1))) {
            cudaFreeHost(S->h_sizes);
            return rc;
        }
        c = 0; if ((rc = ensure(e, &e->d_bond_h, c, nbs, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        c = 0; if ((rc = ensure(e, &e->d_bond_t, c, nbs, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        c = 0; if ((rc = ensure(e, &e->d_bond_k2, c, nbs, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        c = 0; if ((rc = ensure(e, &e->d_bond_l0, c, nbs, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        e->cap_bond = nbs;
        for (int k = 0; k < 4; ++k) {
            c = 0;
            if ((rc = ensure(e, &e->d_ang[k], c, nas, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        }
        c = 0; if ((rc = ensure(e, &e->d_ang_k3, c, nas, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        c = 0; if ((rc = ensure(e, &e->d_ang_cos0, c, nas, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        c = 0; if ((rc = ensure(e, &e->d_ang_sin0, c, nas, &moved))) { cudaFreeHost(S->h_sizes); return rc; }
        e->cap_ang = nas;
        cudaStream_t st = e->s();
        CU(cudaMemcpyAsync(S->d_head_id, hid.data(), nbs * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S->d_tail_id, tid.data(), nbs * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S->d_first, fb.data(), nas * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S->d_second, sb.data(), nas * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S->d_gptr, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(S->d_gterm, gterm.data(), gterm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CU(cudaMemsetAsync(S->d_idmap, 0, sizeof(unsigned long long) * ((size_t)id_max + 1), st));
        if (nb) {
            CU(cudaMemcpyAsync(e->d_bond_k2, k2, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(e->d_bond_l0, l0, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        if (na) {
            CU(cudaMemcpyAsync(e->d_ang_k3, ak.data(), (size_t)na * sizeof(double), cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(e->d_ang_cos0, ak.data() + na, (size_t)na * sizeof(double), cudaMemcpyHostToDevice, st));
            CU(cudaMemcpyAsync(e->d_ang_sin0, ak.data() + 2 * (size_t)na, (size_t)na * sizeof(double),
                               cudaMemcpyHostToDevice, st));
            e->h_ang_phi0.assign(phi0, phi0 + na);
        }
        CU(cudaStreamSynchronize(st));
    }
    // every step's bead set is new: no captured graphs, and no drift done
    // ahead by the last k_update_mom (the upload would discard it)
    e->graphs_enabled = false;
    e->ahead_enabled = false;
    e->n_headroom = 1.25;
    e->mon_set = false;
    if (e->slice_S) e->slice_S = 0;
    e->slab = S.release();
    if (e->slab->topo) {
        if ((rc = slab_topology(e, false))) return rc;
        CU(cudaStreamSynchronize(e->s()));
    }
    return DPD_OK;
}

int dpd_engine_slab_pack(dpd_engine* e, double* send_below, double* send_above, int64_t capacity)
{
    if (!e) return DPD_E_ARG;
    if (!e->slab) return fail(e, DPD_E_STATE, "not a slab (dpd_engine_slab_setup)");
    if (!send_below || !send_above || send_below == send_above || capacity < 1 || capacity > (1 << 26) ||
        ((uintptr_t)send_below & 15) || ((uintptr_t)send_above & 15))
        return fail(e, DPD_E_ARG, "two distinct 16-byte aligned send buffers of capacity >= 1 records");
    SlabState& S = *e->slab;
    CU(cudaSetDevice(e->device));
    const int n = (int)e->n;
    const int nblk = blocks_for(n, kThreads);
    int rc;
    bool moved = false;
    const size_t room = with_room(e, (size_t)n);   // the count changes every step
    if ((rc = ensure(e, &S.d_bcount, S.cap_bcount, (size_t)kSlabOuts * nblk, &moved,
                     (size_t)kSlabOuts * blocks_for(room, kThreads))))
        return rc;
    if ((rc = ensure(e, &S.d_keep, S.cap_keep, (size_t)kSlabRec * n, &moved, (size_t)kSlabRec * room))) return rc;
    if ((rc = ensure(e, &S.d_mine, S.cap_mine, (size_t)kSlabRec * n, &moved, (size_t)kSlabRec * room))) return rc;
    S.geom.cap = (int)capacity;
    cudaStream_t st = e->s();
    const int c = e->cur;
    k_slab_count<<<nblk, kThreads, 0, st>>>(n, S.geom, e->d_x[c], e->d_bid[c], S.d_bcount);
    if ((rc = check_launch(e, "k_slab_count"))) return rc;
    k_slab_offsets<<<1, 1024, 0, st>>>(nblk, S.d_bcount, S.d_total, send_below, send_above, (int)capacity);
    if ((rc = check_launch(e, "k_slab_offsets"))) return rc;
    const double* off = e->off_active ? e->d_off : nullptr;
    if (e->precision == DPD_PRECISION_FP64)
        k_slab_write<double><<<nblk, kThreads, 0, st>>>(n, S.geom, e->d_boxes, e->d_x[c], e->d_v[c],
                                                         (const double*)e->d_F, e->d_img[c], off, e->d_tf[c],
                                                         e->d_bid[c], e->d_pid[c], S.d_bcount, S.d_total, send_below,
                                                         send_above, S.d_keep, S.d_mine);
    else
        k_slab_write<float><<<nblk, kThreads, 0, st>>>(n, S.geom, e->d_boxes, e->d_x[c], e->d_v[c],
                                                        (const float*)e->d_F, e->d_img[c], off, e->d_tf[c],
                                                        e->d_bid[c], e->d_pid[c], S.d_bcount, S.d_total, send_below,
                                                        send_above, S.d_keep, S.d_mine);
    if ((rc = check_launch(e, "k_slab_write"))) return rc;
    S.packed = true;
    return DPD_OK;
}

int dpd_engine_slab_unpack(dpd_engine* e, const double* recv_below, const double* recv_above, int64_t* n_owned,
                           int64_t* n_local)
{
    if (!e) return DPD_E_ARG;
    if (!e->slab) return fail(e, DPD_E_STATE, "not a slab (dpd_engine_slab_setup)");
    SlabState& S = *e->slab;
    if (!S.packed) return fail(e, DPD_E_STATE, "dpd_engine_slab_pack first");
    if (!recv_below || !recv_above || ((uintptr_t)recv_below & 15) || ((uintptr_t)recv_above & 15))
        return fail(e, DPD_E_ARG, "two 16-byte aligned receive buffers");
    CU(cudaSetDevice(e->device));
    cudaStream_t st = e->s();
    k_slab_sizes<<<1, 1, 0, st>>>(recv_below, recv_above, S.d_total, e->d_status, S.geom.cap, S.d_sizes);
    int rc = check_launch(e, "k_slab_sizes");
    if (rc) return rc;
    CU(cudaStreamSynchronize(st));
    int hs[16];
    memcpy(hs, (const void*)S.h_sizes, sizeof hs);
    S.packed = false;
    if (hs[2] || hs[3] || hs[11] || hs[6] + hs[8] > S.geom.cap || hs[7] + hs[9] > S.geom.cap)
        return fail(e, DPD_E_LIMIT, "more boundary beads than the exchange buffers hold");
    const unsigned status = (unsigned)hs[4];
    if (status & DPD_STATUS_FATAL_MASK) {
        *(volatile unsigned*)e->h_seen = status;
        char msg[96];
        snprintf(msg, sizeof msg, "fatal device status 0x%x before the exchange", status);
        return fail(e, DPD_E_STATUS, msg);
    }
    const int64_t nn = hs[1];
    if (nn < 1) return fail(e, DPD_E_STATE, "the slab would hold no beads");
    // The next local box goes straight into the step's input arrays in upload
    // order; the next step's drift, cell scan and gather bin it (no upload
    // kernels, no further host wait).  The drift of a slab's steps is never
    // done ahead, so the arrival counts are zero here.
    if ((rc = drop_ahead(e))) return rc;
    const bool same_n = e->n == nn;
    if ((rc = ensure_beads(e, nn))) return rc;
    bool moved = false;
    if ((rc = ensure(e, &e->d_off, e->cap_off, 3 * (size_t)e->cap_n, &moved))) return rc;
    if ((rc = ensure(e, &e->d_prev_id, e->cap_prev_id, (size_t)nn, &moved, with_room(e, (size_t)nn)))) return rc;
    if ((rc = ensure(e, &e->d_prev_type, e->cap_prev_type, (size_t)nn, &moved, with_room(e, (size_t)nn)))) return rc;
    // the status word starts the next step with the step's non-fatal bits (cell skips)
    CU(cudaMemsetAsync(e->d_status, 0, sizeof(unsigned), st));
    if (status) {
        k_slab_status<<<1, 1, 0, st>>>(e->d_status, status);
        if ((rc = check_launch(e, "k_slab_status"))) return rc;
    }
    const int c = e->cur;
    if (e->precision == DPD_PRECISION_FP64)
        k_slab_place_state<double><<<blocks_for(nn, kThreads), kThreads, 0, st>>>(
            (int)nn, e->ntypes, S.geom, e->d_boxes, S.d_sizes + 5, S.d_keep, recv_below, recv_above, S.d_mine,
            e->d_x[c], e->d_v[c], (double*)e->d_F, e->d_bid[c], e->d_tf[c], e->d_cell[c], e->d_img[c], e->d_pid[c],
            e->d_pid_of, e->d_off, e->d_prev_id, e->d_prev_type, e->d_status);
    else
        k_slab_place_state<float><<<blocks_for(nn, kThreads), kThreads, 0, st>>>(
            (int)nn, e->ntypes, S.geom, e->d_boxes, S.d_sizes + 5, S.d_keep, recv_below, recv_above, S.d_mine,
            e->d_x[c], e->d_v[c], (float*)e->d_F, e->d_bid[c], e->d_tf[c], e->d_cell[c], e->d_img[c], e->d_pid[c],
            e->d_pid_of, e->d_off, e->d_prev_id, e->d_prev_type, e->d_status);
    if ((rc = check_launch(e, "k_slab_place_state"))) return rc;
    CU(cudaMemsetAsync(e->d_stress, 0, 9 * real_size(e) * (size_t)nn, st));
    e->n = nn;
    e->off_active = true;
    e->host_ids_stale = true;   // bead_ids() reads d_prev_id
    ++e->ids_version;
    e->prev_n = nn;
    *(volatile unsigned*)e->h_seen = 0u;   // every kernel before the exchange has finished (the size read)
    if ((rc = empty_topology(e, same_n))) return rc;
    e->uploaded = true;
    e->rs_order.clear();
    e->mon_set = false;
    e->stepped = false;
    e->sampled = false;
    e->obs_valid = false;
    e->box_obs_valid = false;
    S.geom.n_owned = hs[0];
    if (S.topo && (rc = slab_topology(e, true))) return rc;
    if (n_owned) *n_owned = hs[0];
    if (n_local) *n_local = nn;
    return DPD_OK;
}

int dpd_engine_slab_observables(dpd_engine* e, dpd_obs* out)
{
    if (!e) return DPD_E_ARG;
    if (!e->slab) return fail(e, DPD_E_STATE, "not a slab (dpd_engine_slab_setup)");
    if (!out) return fail(e, DPD_E_ARG, "null output");
    if (e->slab->packed) return fail(e, DPD_E_STATE, "the sums are taken after a step, before the exchange");
    CU(cudaSetDevice(e->device));
    const int n = (int)e->n;
    const int nb = blocks_for(n, kThreads);
    // the virial of the latest step when it was a sample step; a pair's counts
    // once over the ranks only when both beads hold half of it (full shell)
    const bool virial = e->sampled && e->stepped && e->pair_scheme == DPD_PAIR_FULL_SHELL;
    const int c = e->cur;
    if (e->precision == DPD_PRECISION_FP64)
        k_slab_obs_partials<double><<<nb, kThreads, 0, e->s()>>>(n, e->slab->geom.n_owned, e->d_bid[c], e->d_x[c],
                                                                e->d_v[c],
                                                                virial ? (const double*)e->d_stress : nullptr,
                                                                e->d_partials);
    else
        k_slab_obs_partials<float><<<nb, kThreads, 0, e->s()>>>(n, e->slab->geom.n_owned, e->d_bid[c], e->d_x[c],
                                                               e->d_v[c], virial ? (const float*)e->d_stress : nullptr,
                                                               e->d_partials);
    int rc = check_launch(e, "k_slab_obs_partials");
    if (rc) return rc;
    k_reduce_obs<<<1, 32 * kObsTerms, 0, e->s()>>>(nb, e->d_partials, e->d_obs);
    if ((rc = check_launch(e, "k_reduce_obs"))) return rc;
    CU(cudaMemcpyAsync(e->h_obs, e->d_obs, kObsTerms * sizeof(double), cudaMemcpyDeviceToHost, e->s()));
    CU(cudaStreamSynchronize(e->s()));
    e->obs_valid = false;   // d_obs now holds the owned beads' sums
    const double* h = e->h_obs;
    memset(out, 0, sizeof *out);
    out->step = e->stepped ? e->last_step : 0;
    out->n = e->slab->geom.n_owned;
    for (int d = 0; d < 3; ++d) {
        out->sum_v[d] = h[d];
        out->sum_v2[d] = h[3 + d];
        out->sum_x[d] = h[15 + d];
        out->ang_mom[d] = h[18 + d];
    }
    out->has_virial = virial ? 1 : 0;
    for (int q = 0; q < 9; ++q) out->virial[q] = virial ? h[6 + q] : 0.0;
    return DPD_OK;   // kT and pressure are the whole box's: left to the caller's sums over the ranks
}

int dpd_engine_slab_counts(dpd_engine* e, int64_t* n_owned, int64_t* n_local)
{
    if (!e) return DPD_E_ARG;
    if (!e->slab) return fail(e, DPD_E_STATE, "not a slab (dpd_engine_slab_setup)");
    if (n_owned) *n_owned = e->slab->geom.n_owned;
    if (n_local) *n_local = e->n;
    return DPD_OK;
}

}  // extern "C"
