// dpd_noalloc.cu -- a DPD pair-force evaluation that allocates no memory.
//
// Who needs it: code that is not allowed to call cudaMalloc (or any
// allocator) at the point where it wants forces.  Typical cases are a host
// application that hands the GPU to a memory pool it does not control (the
// pool owns all device memory, so a stray cudaMalloc fails or fragments it),
// real-time loops where an allocation would stall the device, and plug-ins
// embedded in a program whose allocator policy forbids library-side
// allocations.  Such a caller already owns device buffers for its beads and
// its forces; it only lacks the cell-list scratch that the engine
// (dpd_engine_*) allocates for itself.  The call waits for its own work (it
// synchronises the caller's stream before it returns).
//
// Here that scratch lives in one file-scope __device__ array of fixed size,
// so the call needs nothing but the caller's input and output buffers.  The
// limits are DPD_NOALLOC_MAX_BEADS beads and DPD_NOALLOC_MAX_CELLS CNT
// cells; larger systems are rejected with DPD_E_LIMIT.  Every GPU that loads
// the library holds the array (about 4.5 MB) until the process exits.
//
// The work is the engine's own: beads are binned into CNT cells with the
// reference's (long)(x/w) rule, sorted by cell and, inside a cell, by bead
// index, and the engine's pair-force kernel (k_pair_forces_ref, FP32 forces)
// evaluates the conservative, dissipative and random forces; the result is
// written back in the caller's bead order as FP64.
#include "../../include/dpd_engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "dpd_kernels.cuh"

using namespace dpd;

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxDevices = 64;

// Byte layout of the scratch array; every region starts on a 256-byte boundary.
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffK = 0;
constexpr size_t kOffTab = align256(kOffK + sizeof(StepConst));
constexpr size_t kOffStep = align256(kOffTab + 3 * sizeof(float) * kMaxTypes * kMaxTypes);
constexpr size_t kOffStatus = align256(kOffStep + sizeof(int64_t));
constexpr size_t kMaxChunks = (DPD_NOALLOC_MAX_CELLS + kScanChunk - 1) / kScanChunk;
constexpr size_t kOffChunk = align256(kOffStatus + sizeof(unsigned));
constexpr size_t kOffCount = align256(kOffChunk + sizeof(int) * kMaxChunks);
constexpr size_t kOffStart = align256(kOffCount + sizeof(int) * DPD_NOALLOC_MAX_CELLS);
constexpr size_t kOffCell = align256(kOffStart + sizeof(int) * (DPD_NOALLOC_MAX_CELLS + 1));
constexpr size_t kOffRank = align256(kOffCell + sizeof(int) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffPerm = align256(kOffRank + sizeof(int) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffOrder = align256(kOffPerm + sizeof(int) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffSlotCell = align256(kOffOrder + sizeof(int) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffPos = align256(kOffSlotCell + sizeof(int) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffVel = align256(kOffPos + sizeof(float4) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kOffF = align256(kOffVel + sizeof(float4) * DPD_NOALLOC_MAX_BEADS);
constexpr size_t kScratchBytes = align256(kOffF + 3 * sizeof(float) * DPD_NOALLOC_MAX_BEADS);

}  // namespace

// The scratch itself.  Host code must not pass this name to a kernel: on the
// host it is only a stand-in symbol, not a device address.  Its device
// address comes from cudaGetSymbolAddress (noalloc_scratch_for_current_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mutex;
void* g_scratch_addr[kNaMaxDevices] = {};

// Once per device, with that device current: the device address of the array.
// The address is kept for the life of the process, so a context reset
// (cudaDeviceReset) between calls is not supported.
int noalloc_scratch_for_current_device(unsigned char** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return DPD_E_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DPD_E_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return DPD_OK;
}

// Clears what must start at zero: the cell counts, the per-chunk totals and
// the status word (the array keeps whatever the previous call left in it).
__global__ void k_na_clear(int ncell, int nchunk, int* __restrict__ count, int* __restrict__ chunk,
                           unsigned* __restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ncell) count[i] = 0;
    if (i < nchunk) chunk[i] = 0;
    if (i == 0) *status = 0u;
}

// CSimBox::AssignBeadstoCells rule (SimBox.cpp:738-750).  A bead outside the
// box sets status bit 1 and is filed in cell 0 so every access stays in bounds.
__global__ void k_na_bin(int n, const StepConst* __restrict__ K, const double* __restrict__ x3,
                         int* __restrict__ cell, int* __restrict__ rank, int* __restrict__ count,
                         int* __restrict__ chunk, unsigned* __restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long ci[3];
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xv = x3[3 * i + d];
        ci[d] = (long long)(xv / K->w[d]);
        inside = inside && (xv >= 0.0) && ci[d] >= 0 && ci[d] < K->nc[d];
    }
    int c = 0;
    if (inside) c = (int)(ci[0] + (long long)K->nc[0] * (ci[1] + (long long)K->nc[1] * ci[2]));
    else atomicOr(status, 1u);
    cell[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
    atomicAdd(&chunk[c / kScanChunk], 1);
}

__global__ void k_na_place(int n, const int* __restrict__ cell, const int* __restrict__ rank,
                           const int* __restrict__ start, int* __restrict__ perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[start[cell[i]] + rank[i]] = i;
}

// Final slot = cell start + rank of the bead index among the cell's beads;
// writes the force kernel's shadows (position relative to the cell origin,
// type; velocity, noise id).  A type outside 0..ntypes-1 would index past the
// pair tables: it sets status bit 2 and is replaced by type 0.
__global__ void k_na_shadows(int n, const StepConst* __restrict__ K, const int* __restrict__ perm,
                             const int* __restrict__ cell, const int* __restrict__ start,
                             const double* __restrict__ x3, const double* __restrict__ v3,
                             const int32_t* __restrict__ type, const int32_t* __restrict__ id,
                             int* __restrict__ order, int* __restrict__ slot_cell, float4* __restrict__ pos4,
                             float4* __restrict__ vel4, unsigned* __restrict__ status)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int i = perm[d];
    const int c = cell[i];
    const int beg = start[c], end = start[c + 1];
    int k = 0;
    for (int e = beg; e < end; ++e) k += (perm[e] < i);
    const int o = beg + k;
    const int nx = K->nc[0], ny = K->nc[1];
    const int ci[3] = {c % nx, (c / nx) % ny, c / (nx * ny)};
    float4 p, w;
    p.x = (float)__dadd_rn(x3[3 * i], -__dmul_rn((double)ci[0], K->w[0]));
    p.y = (float)__dadd_rn(x3[3 * i + 1], -__dmul_rn((double)ci[1], K->w[1]));
    p.z = (float)__dadd_rn(x3[3 * i + 2], -__dmul_rn((double)ci[2], K->w[2]));
    int ti = type[i];
    if (ti < 0 || ti >= K->ntypes) {
        atomicOr(status, 2u);
        ti = 0;
    }
    p.w = __int_as_float(ti);
    w.x = (float)v3[3 * i];
    w.y = (float)v3[3 * i + 1];
    w.z = (float)v3[3 * i + 2];
    w.w = __int_as_float(id[i]);
    pos4[o] = p;
    vel4[o] = w;
    order[o] = i;
    slot_cell[o] = c;
}

__global__ void k_na_scatter(int n, const int* __restrict__ order, const float* __restrict__ F,
                             double* __restrict__ f3)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int i = order[d];
    f3[3 * i] = (double)F[d];
    f3[3 * i + 1] = (double)F[n + d];
    f3[3 * i + 2] = (double)F[2 * n + d];
}

inline int nblk(int64_t n) { return (int)((n + kNaThreads - 1) / kNaThreads); }

}  // namespace

static int pair_forces_on_current_device(const dpd_params* p, int64_t step, int64_t n, int64_t ncell,
                                         const double* x3, const double* v3, const int32_t* type,
                                         const int32_t* id, double* f3, void* cuda_stream);

extern "C" DPD_API int dpd_pair_forces_noalloc(const dpd_params* p, int64_t step, int64_t n,
                                               const double* x3, const double* v3, const int32_t* type,
                                               const int32_t* id, double* f3, void* cuda_stream)
{
    if (!p || !x3 || !v3 || !type || !id || !f3 || n < 1) return DPD_E_ARG;
    if (p->nx < 3 || p->ny < 3 || p->nz < 3 || !(p->wx >= 1.0) || !(p->wy >= 1.0) || !(p->wz >= 1.0) ||
        !(p->dt > 0.0) || p->kT < 0.0 || p->ntypes < 1 || p->ntypes > kMaxTypes || !p->a || !p->gamma)
        return DPD_E_ARG;
    const int64_t ncell = (int64_t)p->nx * p->ny * p->nz;
    if (n > DPD_NOALLOC_MAX_BEADS || ncell > DPD_NOALLOC_MAX_CELLS) return DPD_E_LIMIT;
    // the caller's current device is restored on every return below
    int caller_dev = -1;
    if (cudaGetDevice(&caller_dev) != cudaSuccess) return DPD_E_CUDA;
    if (p->device >= 0 && p->device != caller_dev && cudaSetDevice(p->device) != cudaSuccess) return DPD_E_CUDA;
    const int rc = pair_forces_on_current_device(p, step, n, ncell, x3, v3, type, id, f3, cuda_stream);
    if (p->device >= 0 && p->device != caller_dev && cudaSetDevice(caller_dev) != cudaSuccess) return DPD_E_CUDA;
    return rc;
}

// The work of dpd_pair_forces_noalloc with its device already current.
static int pair_forces_on_current_device(const dpd_params* p, int64_t step, int64_t n, int64_t ncell,
                                         const double* x3, const double* v3, const int32_t* type,
                                         const int32_t* id, double* f3, void* cuda_stream)
{
    unsigned char* base = nullptr;
    int rc = noalloc_scratch_for_current_device(&base);
    if (rc != DPD_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    // constants and pair tables (stack copies, then into the scratch)
    StepConst K{};
    K.dt = p->dt;
    K.halfdt = 0.5 * p->dt;
    K.halfdt2 = 0.5 * p->dt * p->dt;
    K.lamdt = p->lambda * p->dt;
    K.invrootdt = std::sqrt(24.0 * p->kT / p->dt);
    K.nc[0] = p->nx; K.nc[1] = p->ny; K.nc[2] = p->nz;
    K.w[0] = p->wx; K.w[1] = p->wy; K.w[2] = p->wz;
    for (int d = 0; d < 3; ++d) K.L[d] = (double)K.nc[d] * K.w[d];
    K.ntypes = p->ntypes;
    K.seed = p->seed;
    const int m = p->ntypes * p->ntypes;
    float tab[3 * kMaxTypes * kMaxTypes];
    for (int k = 0; k < m; ++k) {
        tab[k] = (float)p->a[k];
        tab[m + k] = (float)p->gamma[k];
        tab[2 * m + k] = (float)(std::sqrt(p->gamma[k]) * K.invrootdt);
    }
    int64_t step_h = step;
    StepConst* dK = reinterpret_cast<StepConst*>(base + kOffK);
    float* dTab = reinterpret_cast<float*>(base + kOffTab);
    int64_t* dStep = reinterpret_cast<int64_t*>(base + kOffStep);
    unsigned* dStatus = reinterpret_cast<unsigned*>(base + kOffStatus);
    int* dChunk = reinterpret_cast<int*>(base + kOffChunk);
    int* dCount = reinterpret_cast<int*>(base + kOffCount);
    int* dStart = reinterpret_cast<int*>(base + kOffStart);
    int* dCell = reinterpret_cast<int*>(base + kOffCell);
    int* dRank = reinterpret_cast<int*>(base + kOffRank);
    int* dPerm = reinterpret_cast<int*>(base + kOffPerm);
    int* dOrder = reinterpret_cast<int*>(base + kOffOrder);
    int* dSlotCell = reinterpret_cast<int*>(base + kOffSlotCell);
    float4* dPos = reinterpret_cast<float4*>(base + kOffPos);
    float4* dVel = reinterpret_cast<float4*>(base + kOffVel);
    float* dF = reinterpret_cast<float*>(base + kOffF);

    if (cudaMemcpyAsync(dK, &K, sizeof K, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dTab, tab, 3 * sizeof(float) * m, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dStep, &step_h, sizeof step_h, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return DPD_E_CUDA;
    const int nn = (int)n, nc = (int)ncell, nchunk = (int)((ncell + kScanChunk - 1) / kScanChunk);
    k_na_clear<<<nblk(std::max(nc, 1)), kNaThreads, 0, st>>>(nc, nchunk, dCount, dChunk, dStatus);
    k_na_bin<<<nblk(nn), kNaThreads, 0, st>>>(nn, dK, x3, dCell, dRank, dCount, dChunk, dStatus);
    k_scan_cells<<<nchunk, kScanThreads, 0, st>>>(nc, nn, dCount, dChunk, dStart, (const unsigned*)nullptr,
                                                  (unsigned*)nullptr, 1);
    k_na_place<<<nblk(nn), kNaThreads, 0, st>>>(nn, dCell, dRank, dStart, dPerm);
    k_na_shadows<<<nblk(nn), kNaThreads, 0, st>>>(nn, dK, dPerm, dCell, dStart, x3, v3, type, id, dOrder,
                                                  dSlotCell, dPos, dVel, dStatus);
    k_pair_forces_ref<float, false><<<(nn + 127) / 128, 128, 0, st>>>(nn, dK, dStep, dTab, dSlotCell, dStart,
                                                                      dPos, dVel, dF, nullptr);
    k_na_scatter<<<nblk(nn), kNaThreads, 0, st>>>(nn, dOrder, dF, f3);
    if (cudaGetLastError() != cudaSuccess) return DPD_E_CUDA;
    unsigned status = 0;
    if (cudaMemcpyAsync(&status, dStatus, sizeof status, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return DPD_E_CUDA;
    if (status & 2u) return DPD_E_ARG;   // a bead type outside 0..ntypes-1
    return (status & 1u) ? DPD_E_BOX : DPD_OK;
}
