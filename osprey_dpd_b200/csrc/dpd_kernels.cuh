// dpd_kernels.cuh -- sm_100a kernels of one DPD timestep.
//
// Device layout ("slot order"): beads sorted by CNT cell, cells in the
// reference's index order nx*(ny*iz+iy)+ix (SimBox.cpp:888-920).  Under the
// full-shell pair scheme the beads of a cell keep the order of their
// previous slots (a stable counting sort), so the order -- and every
// floating-point sum -- is deterministic; the half-shell schemes add forces
// with atomics in no fixed order anyway and scatter each cell's beads in
// any order.  Per-bead arrays are structure-of-arrays; 3-vectors are three
// planes of n values.
//
// One step, in the reference's order (CSimBox::Evolve, SimBox.cpp:977-1120):
//   k_update_pos   UpdatePos: drift, incremental cell move + PBC wrap,
//                  per-cell arrival counts         (CNTCell.cpp:1634-2262);
//                  first step of a call only, the others drift in the
//                  k_update_mom before them
//   k_scan_cells   cell start offsets (exclusive prefix sum of the counts)
//   k_permute      arrival slot -> new slot map (full shell only)
//   k_gather       permutes the state into the new slot order (half shell:
//                  slots claimed from the counts), writes the cell-relative
//                  FP32/FP64 shadows the force kernel reads
//   k_bonds        bond and bond-pair forces, FP64, beside the pair kernel
//                  (Bond.cpp:111-162, BondPair.cpp:138-286)
//   pair kernel    conservative + dissipative + random pair forces over the
//                  neighbour cells (pair_forces.cuh; CNTCell.cpp:1103-1572)
//   k_update_mom   adds the bonded forces, UpdateMom, FP64 sums on sample
//                  steps, then the next step's UpdatePos
//                  (CNTCell.cpp:2280-2310, Monitor.cpp:790-1040)
// Non-template kernels have internal linkage so that more than one
// translation unit of the library can include this header.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "philox.cuh"

namespace dpd {

// Programmatic dependent launch (sm_90 and later): a kernel launched with the
// programmatic-serialization attribute may be scheduled while the kernel
// ahead of it in the stream is still running.  pdl_wait() blocks until that
// kernel has completed and its writes are visible; pdl_launch() lets the next
// kernel be scheduled once every block of this one has started.  Both are
// no-ops for an ordinary launch.  Every step kernel calls both first thing,
// before it reads any global memory.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

constexpr int kMaxTypes = 32;
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 4;
constexpr int kScanChunk = kScanThreads * kScanPerThread;   // cells per scan block
constexpr int kObsTerms = 21;   // sum_v[3] sum_v2[3] virial[9] sum_x[3] angmom[3]

// Image counters: three signed 10-bit fields (bias 512) in one word.
__host__ __device__ __forceinline__ uint32_t img_pack(int ix, int iy, int iz)
{
    return (uint32_t)(ix + 512) | ((uint32_t)(iy + 512) << 10) | ((uint32_t)(iz + 512) << 20);
}
__host__ __device__ __forceinline__ int img_get(uint32_t w, int d)
{
    return (int)((w >> (10 * d)) & 1023u) - 512;
}

// Time-step constants and the first box; lives in device memory so that a
// parameter change needs no relaunch configuration (CCNTCell statics,
// CNTCell.cpp:42-75).
struct StepConst {
    double dt, halfdt, halfdt2, lamdt, invrootdt;
    double L[3], w[3];
    int nc[3];
    int ntypes;
    uint64_t seed;
};

// One simulation box (CCNTCell::SetSimBoxLengths, CNTCell.cpp:143-158).  An
// engine holds a packed table of them: one for a single simulation, one per
// replica for a batch.  Global cell index = cell_base + nx*(ny*iz+iy)+ix.
struct Box {
    int nc[3];
    int cell_base;
    double w[3];
    double L[3];
    uint64_t seed;     // pair-noise seed of this box
    int tab;           // offset of this box's pair tables (3 * ntypes^2 reals)
    int pad;
    double iw[3];      // 1 / w
    // division of a box-local cell index c < 2^31 by nx and by nx*ny as a
    // multiply and shift (set_cell_division)
    unsigned long long mx, mxy;
    int kx, kxy;
};

// Division by an invariant integer d (1 <= d < 2^31) for numerators below
// 2^31 as floor(c * m / 2^k), k = 31 + ceil(log2 d), m = ceil(2^k / d)
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, with N = 31 numerator bits): exact, since
// c * (m d - 2^k) / (d 2^k) < 1/d.
__host__ __device__ inline void division_magic(unsigned d, unsigned long long& m, int& k)
{
    int l = 0;
    while ((1ull << l) < d) ++l;
    k = 31 + l;
    m = ((1ull << k) + d - 1) / d;
}
inline void set_cell_division(Box& b)
{
    division_magic((unsigned)b.nc[0], b.mx, b.kx);
    division_magic((unsigned)b.nc[0] * (unsigned)b.nc[1], b.mxy, b.kxy);
    for (int d = 0; d < 3; ++d) b.iw[d] = 1.0 / b.w[d];
}
// Cell coordinates (ix, iy, iz) of box-local cell index cl = nx*(ny*iz+iy)+ix.
__device__ __forceinline__ void cell_coords(const Box& B, int cl, int ci[3])
{
    const int q = (int)(((unsigned long long)(unsigned)cl * B.mx) >> B.kx);     // cl / nx
    ci[2] = (int)(((unsigned long long)(unsigned)cl * B.mxy) >> B.kxy);         // cl / (nx ny)
    ci[0] = cl - q * B.nc[0];
    ci[1] = q - ci[2] * B.nc[1];
}

// Bead flags word: type in bits 0..7, box in bits 8..23, frozen (never
// moves) in bit 24, has bond or bond-pair terms in bit 25.  The force
// kernel's position shadow carries bits 0..23.
__host__ __device__ __forceinline__ int flag_type(int tf) { return tf & 0xFF; }
__host__ __device__ __forceinline__ int flag_box(int tf) { return (tf >> 8) & 0xFFFF; }
__device__ __forceinline__ bool flag_frozen(int tf) { return (tf >> 24) & 1; }
__device__ __forceinline__ bool flag_bonded(int tf) { return (tf >> 25) & 1; }
constexpr int kFlagFrozen = 1 << 24;
constexpr int kFlagBonded = 1 << 25;
constexpr int kShadowMask = 0x00FFFFFF;
constexpr int kMaxBoxes = 1 << 16;

template <typename real> struct Vec4;
template <> struct Vec4<float> { typedef float4 type; };
template <> struct Vec4<double> { typedef double4 type; };

__device__ __forceinline__ float as_real_bits(int v, float) { return __int_as_float(v); }
__device__ __forceinline__ double as_real_bits(int v, double) { return __longlong_as_double((long long)v); }
__device__ __forceinline__ int real_bits(float v) { return __float_as_int(v); }
__device__ __forceinline__ int real_bits(double v) { return (int)__double_as_longlong(v); }

// The first kernel of a call copies the status word of all work queued
// before it (its predecessors have completed: a call's first kernel waits
// for them in full) to `seen`, a word of mapped pinned host memory that the
// host reads without waiting; seen = NULL in every other launch.
__device__ __forceinline__ void publish_status(const unsigned* status, unsigned* seen)
{
    if (seen && blockIdx.x == 0 && threadIdx.x == 0) *(volatile unsigned*)seen = *(const volatile unsigned*)status;
}

// ------------------------------------------------------------- UpdatePos

// One bead's drift and cell move; returns its new cell and writes x, img and
// cell of slot s (a frozen bead's unchanged ones too: the output may be the
// separate buffers of a drift done ahead).  x0, v0, f0 are the bead's
// position, velocity and force.
__device__ __forceinline__ int drift_and_move(const StepConst* __restrict__ K, const Box* __restrict__ boxes,
                                              int n, int s, int c, int tfl, const double x0[3], const double v0[3],
                                              const double f0[3], uint32_t im0, double* __restrict__ x,
                                              uint32_t* __restrict__ img, int* __restrict__ cell, unsigned& bad)
{
    if (flag_frozen(tfl)) {
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d * n + s] = x0[d];
        img[s] = im0;
        cell[s] = c;
        return c;
    }
    const Box& B = boxes[flag_box(tfl)];
    int cnew = c;
    const double dt = K->dt, h2 = K->halfdt2;
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    const int cl = c - B.cell_base;
    int ci[3];
    cell_coords(B, cl, ci);
    const bool ext = ci[0] == 0 || ci[0] == nx - 1 || ci[1] == 0 || ci[1] == ny - 1 ||
                     ci[2] == 0 || ci[2] == nz - 1;
    double xn[3];
    int mv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        // x += dt*v + dt^2/2*F with the reference's rounding (no fused multiply-add)
        const double dx = __dadd_rn(__dmul_rn(dt, v0[d]), __dmul_rn(h2, f0[d]));
        xn[d] = __dadd_rn(x0[d], dx);
        const double BL = __dmul_rn((double)ci[d], B.w[d]);   // CCNTCell ctor, CNTCell.cpp:598-604
        const double TR = __dadd_rn(BL, B.w[d]);
        mv[d] = (xn[d] > TR) ? 1 : ((xn[d] < BL) ? -1 : 0);
    }
    uint32_t im = im0;
    if (mv[0] | mv[1] | mv[2]) {
        int nci[3];
        for (int d = 0; d < 3; ++d) {
            nci[d] = ci[d] + mv[d];
            if (nci[d] < 0) nci[d] += B.nc[d];
            else if (nci[d] >= B.nc[d]) nci[d] -= B.nc[d];
        }
        const bool next = nci[0] == 0 || nci[0] == nx - 1 || nci[1] == 0 || nci[1] == ny - 1 ||
                          nci[2] == 0 || nci[2] == nz - 1;
        if (ext && next) {
            int ii[3] = {img_get(im, 0), img_get(im, 1), img_get(im, 2)};
            for (int d = 0; d < 3; ++d) {
                if (mv[d] > 0 && xn[d] > B.L[d]) { xn[d] -= B.L[d]; ++ii[d]; }
                else if (mv[d] < 0 && xn[d] < 0.0) { xn[d] += B.L[d]; --ii[d]; }
                if (ii[d] < -511 || ii[d] > 511) bad |= 0x4u;
            }
            im = img_pack(ii[0], ii[1], ii[2]);
        }
        cnew = B.cell_base + nci[0] + nx * (nci[1] + ny * nci[2]);
    }
    // CCNTCell::CheckBeadsinCell audit (CNTCell.cpp:2636-2650), run by the
    // reference after every step (SimBox.cpp:1322): (long)(x / w) per axis,
    // from x * (1/w) (within 2 ulp of x / w) except within 1e-9 of a cell
    // face, where the truncation could differ and the division is done
    long long a[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double q = xn[d] * B.iw[d];
        a[d] = (long long)q;
        if (fabs(q - rint(q)) < 1e-9) a[d] = (long long)(xn[d] / B.w[d]);
    }
    if (B.cell_base + (long long)nx * ((long long)ny * a[2] + a[1]) + a[0] != cnew) bad |= 0x1u;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!isfinite(xn[d])) bad |= 0x2u;
        x[d * n + s] = xn[d];
    }
    img[s] = im;
    cell[s] = cnew;
    return cnew;
}

// Warp-aggregated counting of the beads arriving in each cell: lanes bound
// for the same cell take one atomic (beads are cell-sorted, so a warp spans
// ~11 cells); with `rank`, each bead's rank inside its cell (lane order inside
// the group) for a gather in a fixed order, else the count alone, by
// reductions that return nothing (k_gather then claims the slots).  One
// reduction per scan chunk per warp as well.  Called by every lane of the warp.
__device__ __forceinline__ void count_arrival(bool live, int s, int cnew, int* __restrict__ rank,
                                              int* __restrict__ count, int* __restrict__ block_count)
{
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (live) {
        const int lane = threadIdx.x & 31;
        const unsigned peers = __match_any_sync(act, cnew);
        const int leader = __ffs(peers) - 1;
        if (rank) {
            int base = 0;
            if (lane == leader) base = atomicAdd(&count[cnew], __popc(peers));
            base = __shfl_sync(act, base, leader);
            rank[s] = base + __popc(peers & ((1u << lane) - 1u));
        } else if (lane == leader) {
            atomicAdd(&count[cnew], __popc(peers));   // result unused: a reduction
        }
        const int chunk = cnew / kScanChunk;
        const unsigned cpeers = __match_any_sync(act, chunk);
        if (lane == __ffs(cpeers) - 1) atomicAdd(&block_count[chunk], __popc(cpeers));   // result unused: a reduction
    }
}

// Drift and cell migration of every bead (CCNTCell::UpdatePos) for the first
// step of a call; later steps run it fused into k_update_mom of the step
// before.  The reference's 27-way decision tree moves a bead by one cell
// along each axis where x > TR (+1) or x < BL (-1), TR = BL + w with
// BL = ix*w (CNTCell.cpp:598-604, 1768-2254), wrapping the moved coordinates
// only when both cells lie on the box boundary.  Frozen beads keep their cell.
template <typename real>
__global__ void __launch_bounds__(256, 6) k_update_pos(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, double* __restrict__ x,
    const double* __restrict__ v,
    const real* __restrict__ F, const int* __restrict__ tf, uint32_t* __restrict__ img,
    int* __restrict__ cell, int* __restrict__ rank, int* __restrict__ count,
    int* __restrict__ block_count, unsigned* __restrict__ status, unsigned* seen)
{
    pdl_wait();
    pdl_launch();
    publish_status(status, seen);
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < n;
    int cnew = 0;
    unsigned bad = 0;
    if (live) {
        // every load first, so one memory round trip covers them all
        const int c = cell[s];
        const int tfl = tf[s];
        double x0[3], v0[3], f0[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x0[d] = x[d * n + s];
            v0[d] = v[d * n + s];
            f0[d] = (double)F[d * n + s];
        }
        const uint32_t im0 = img[s];
        cnew = drift_and_move(K, boxes, n, s, c, tfl, x0, v0, f0, im0, x, img, cell, bad);
    }
    count_arrival(live, s, cnew, rank, count, block_count);
    if (bad) atomicOr(status, bad);
}

// ------------------------------------------------------------------ scan

// start[c] = sum of count[0..c); one block per chunk of kScanChunk cells.  The
// chunk's base is the sum of the per-chunk totals counted by k_update_pos.
// With clear, the counts are cleared for the next step.
static __global__ void __launch_bounds__(kScanThreads) k_scan_cells(
    int ncell, int n, int* __restrict__ count, const int* __restrict__ block_count,
    int* __restrict__ start, const unsigned* status, unsigned* seen, int clear)
{
    pdl_wait();
    pdl_launch();
    publish_status(status, seen);
    __shared__ int warp_sum[kScanThreads / 32];
    __shared__ int base_s;
    const int b = blockIdx.x, t = threadIdx.x, lane = t & 31, wid = t >> 5;
    // this thread's cell counts first (one 16-byte load), so their memory
    // round trip overlaps the one of the chunk totals below
    const int c0 = b * kScanChunk + t * kScanPerThread;
    int vals[kScanPerThread];
    static_assert(kScanPerThread == 4, "one int4 per thread");
    if (c0 + kScanPerThread <= ncell) {
        const int4 q = *reinterpret_cast<const int4*>(count + c0);
        vals[0] = q.x; vals[1] = q.y; vals[2] = q.z; vals[3] = q.w;
    } else {
#pragma unroll
        for (int k = 0; k < kScanPerThread; ++k) vals[k] = (c0 + k < ncell) ? count[c0 + k] : 0;
    }
    int acc = 0;
    for (int k = t; k < b; k += kScanThreads) acc += block_count[k];
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) warp_sum[wid] = acc;
    __syncthreads();
    if (t == 0) {
        int s = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) s += warp_sum[w];
        base_s = s;
    }
    __syncthreads();
    const int base = base_s;
    int tot = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) tot += vals[k];
    // exclusive scan of per-thread totals across the block
    int inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    __syncthreads();
    if (lane == 31) warp_sum[wid] = inc;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < wid; ++w) wbase += warp_sum[w];
    int run = base + wbase + inc - tot;
    // clear = 0 leaves the counts for k_gather to claim slots from (it
    // returns them to zero)
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
        const int c = c0 + k;
        if (c < ncell) {
            start[c] = run;
            if (clear) count[c] = 0;
        }
        run += vals[k];
    }
    if (b == gridDim.x - 1 && t == 0) start[ncell] = n;
}

// new arrival slot -> old slot; also clears the per-chunk totals.
static __global__ void __launch_bounds__(256) k_permute(
    int n, int nchunk, const int* __restrict__ cell, const int* __restrict__ rank,
    const int* __restrict__ start, int* __restrict__ perm, int* __restrict__ block_count)
{
    pdl_wait();
    pdl_launch();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nchunk) block_count[s] = 0;
    if (s < n) perm[start[cell[s]] + rank[s]] = s;
}

// Stable order inside each cell (by previous slot), state permutation, the
// force kernel's shadows (position relative to the bead's own cell origin
// and intermediate velocity v~ = v + lambda*dt*F_old (CNTCell.cpp:1743-1747),
// with the bead type and the noise id in the fourth component) and, with
// zero_F, the cleared force accumulator.
template <typename real>
__global__ void __launch_bounds__(256, 6) k_gather(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int* __restrict__ perm,
    const int* __restrict__ start,
    const double* __restrict__ x_in, const double* __restrict__ v_in, real* __restrict__ F_in,
    const int* __restrict__ bid_in, const int* __restrict__ tf_in, const uint32_t* __restrict__ img_in,
    const int* __restrict__ cell_in, double* __restrict__ x_out, double* __restrict__ v_out,
    real* __restrict__ Fold_out, int* __restrict__ bid_out, int* __restrict__ tf_out,
    uint32_t* __restrict__ img_out, int* __restrict__ cell_out, const int* __restrict__ pid_in,
    int* __restrict__ pid_out, typename Vec4<real>::type* __restrict__ pos4,
    typename Vec4<real>::type* __restrict__ vel4, double4* __restrict__ ubuf, const double* __restrict__ off,
    int zero_F, int nchunk, int* __restrict__ block_count, int* __restrict__ claim)
{
    pdl_wait();
    pdl_launch();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    // Scatter mode (claim = the arrival counts): thread t moves source slot t
    // into its cell, to a slot that the warp's beads bound for the cell take
    // from the count by one atomic subtraction (in no fixed order inside the
    // cell), which leaves every count at zero for the next step; the arrival
    // permutation (k_permute) is not needed, and the per-chunk totals are
    // cleared for the next step.  Gather mode: thread t fills slot t from
    // perm, in the order of the beads' previous slots.
    if (claim && t < nchunk) block_count[t] = 0;
    const unsigned act = claim ? __ballot_sync(0xffffffffu, t < n) : 0u;
    if (t >= n) return;
    const int s = claim ? t : perm[t];
    // the bead's state is independent of its final slot: load it before the
    // rank scan so both memory round trips overlap
    const int c = cell_in[s];
    const int b = bid_in[s];
    const int tfl = tf_in[s];
    const uint32_t im = img_in[s];
    const int pid = pid_in[s];
    double xs[3], vs[3];
    real fs[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        xs[q] = x_in[q * n + s];
        vs[q] = v_in[q * n + s];
        fs[q] = F_in[q * n + s];
    }
    int o;
    if (claim) {
        const int lane = threadIdx.x & 31;
        const unsigned peers = __match_any_sync(act, c);
        const int leader = __ffs(peers) - 1, k = __popc(peers);
        int top = 0;
        if (lane == leader) top = atomicSub(&claim[c], k);
        top = __shfl_sync(peers, top, leader);
        o = start[c] + top - k + __popc(peers & ((1u << lane) - 1u));
    } else {
        const int beg = start[c], end = start[c + 1];
        int k = 0;
        for (int e = beg; e < end; ++e) k += (perm[e] < s);
        o = beg + k;
    }
    const Box& B = boxes[flag_box(tfl)];
    int ci[3];
    cell_coords(B, c - B.cell_base, ci);
    const bool frozen = flag_frozen(tfl);
    real rel[3], vt[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double xv = xs[q];
        const double vv = vs[q];
        const real fv = fs[q];
        x_out[q * n + o] = xv;
        v_out[q * n + o] = vv;
        Fold_out[q * n + o] = fv;
        rel[q] = (real)__dadd_rn(xv, -__dmul_rn((double)ci[q], B.w[q]));
        vt[q] = frozen ? (real)vv : (real)__dadd_rn(vv, __dmul_rn(K->lamdt, (double)fv));
    }
    bid_out[o] = b;
    tf_out[o] = tfl;
    img_out[o] = im;
    cell_out[o] = c;
    pid_out[o] = pid;
    typedef typename Vec4<real>::type V4;
    V4 p, w;
    p.x = rel[0]; p.y = rel[1]; p.z = rel[2]; p.w = as_real_bits(tfl & kShadowMask, real(0));
    w.x = vt[0]; w.y = vt[1]; w.z = vt[2]; w.w = as_real_bits(pid, real(0));
    pos4[o] = p;
    vel4[o] = w;
    if (flag_bonded(tfl)) {
        // unPBC position (x + image*L + upload offset) for the bonded terms,
        // stored by upload index: chain partners sit in the same lines
        double u[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) u[q] = xs[q] + (double)img_get(im, q) * B.L[q] + (off ? off[q * n + b] : 0.0);
        ubuf[b] = make_double4(u[0], u[1], u[2], xs[2]);   // w: wrapped z, for the slice stress profile
    }
    // the half-shell pair kernels add into F: each old slot was read above by
    // exactly one thread, which clears it last (no separate memset)
    if (zero_F) {
#pragma unroll
        for (int q = 0; q < 3; ++q) F_in[q * n + s] = real(0);
    }
}

// ------------------------------------------------------------ pair forces

// Pair-parameter tables staged per block: a_ij, gamma_ij and
// sigma_ij = sqrt(gamma_ij) * sqrt(24 kT / dt).
template <typename real>
struct PairTables {
    real a[kMaxTypes * kMaxTypes];
    real g[kMaxTypes * kMaxTypes];
    real sig[kMaxTypes * kMaxTypes];
};

template <typename real>
__device__ __forceinline__ void load_tables(PairTables<real>& T, const real* __restrict__ tab, int nt)
{
    const int m = nt * nt;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        T.a[k] = tab[k];
        T.g[k] = tab[m + k];
        T.sig[k] = tab[2 * m + k];
    }
}

__device__ __forceinline__ float noise_centered(uint32_t r, float)
{
    // 0.5 - r * 2^-32, formed exactly in integers before the conversion
    return (float)(int)(0x80000000u - r) * 2.3283064365386963e-10f;
}
__device__ __forceinline__ double noise_centered(uint32_t r, double)
{
    return 0.5 - (double)r * 2.3283064365386963e-10;
}

// Reference force kernel: one thread per bead, full 27-cell shell, every
// pair evaluated from both sides (no atomics, deterministic).  The DPD force
// of CNTCell.cpp:1192-1220 with rc = 1:
//   w = 1 - r; F = (a_ij w - gamma_ij w^2 (r.v)/r + sigma_ij w (0.5 - U)) r_vec / r
template <typename real, bool VIRIAL>
__global__ void __launch_bounds__(128) k_pair_forces_ref(
    int n, const StepConst* __restrict__ K, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress)
{
    __shared__ PairTables<real> T;
    const int nt = K->ntypes;
    load_tables(T, tab, nt);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t key = philox_step_key(K->seed, *step_ptr);
    const int nx = K->nc[0], ny = K->nc[1], nz = K->nc[2];
    const int c = cell[i];
    const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
    const typename Vec4<real>::type pi = pos4[i], vi = vel4[i];
    const int ti = real_bits(pi.w) & 0xFF;
    const uint32_t idi = (uint32_t)real_bits(vi.w);
    real fx = 0, fy = 0, fz = 0;
    real s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int oz = -1; oz <= 1; ++oz) {
        int z2 = cz + oz;
        z2 += (z2 < 0) ? nz : ((z2 >= nz) ? -nz : 0);
        for (int oy = -1; oy <= 1; ++oy) {
            int y2 = cy + oy;
            y2 += (y2 < 0) ? ny : ((y2 >= ny) ? -ny : 0);
            for (int ox = -1; ox <= 1; ++ox) {
                int x2 = cx + ox;
                x2 += (x2 < 0) ? nx : ((x2 >= nx) ? -nx : 0);
                const int c2 = x2 + nx * (y2 + ny * z2);
                const real sx = (real)(ox * K->w[0]), sy = (real)(oy * K->w[1]), sz = (real)(oz * K->w[2]);
                const int jb = start[c2], je = start[c2 + 1];
                for (int j = jb; j < je; ++j) {
                    if (j == i) continue;
                    const typename Vec4<real>::type pj = pos4[j];
                    const real dx = (pi.x - pj.x) - sx;
                    const real dy = (pi.y - pj.y) - sy;
                    const real dz = (pi.z - pj.z) - sz;
                    const real r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < real(1) && r2 > real(1e-18)) {
                        const typename Vec4<real>::type vj = vel4[j];
                        const real r = sqrt(r2);
                        const real inv = real(1) / r;
                        const real wr = real(1) - r;
                        const int tj = real_bits(pj.w) & 0xFF;
                        const int tt = ti * nt + tj;
                        const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
                        const uint32_t idj = (uint32_t)real_bits(vj.w);
                        const uint32_t u = philox2x32_10(min(idi, idj), max(idi, idj), key);
                        const real mag = T.a[tt] * wr - T.g[tt] * wr * wr * rdotv +
                                         T.sig[tt] * wr * noise_centered(u, real(0));
                        const real m = mag * inv;
                        const real gx = m * dx, gy = m * dy, gz = m * dz;
                        fx += gx; fy += gy; fz += gz;
                        if (VIRIAL) {
                            s[0] += dx * gx; s[1] += dy * gx; s[2] += dz * gx;
                            s[3] += dx * gy; s[4] += dy * gy; s[5] += dz * gy;
                            s[6] += dx * gz; s[7] += dy * gz; s[8] += dz * gz;
                        }
                    }
                }
            }
        }
    }
    F[i] = fx;
    F[n + i] = fy;
    F[2 * n + i] = fz;
    if (VIRIAL) {
#pragma unroll
        for (int q = 0; q < 9; ++q) stress[q * n + i] = real(0.5) * s[q];
    }
}

// -------------------------------------------------------------- UpdateMom

// ------------------------------------------------- slice stress profile
// CMonitor::AddBeadStress / AddBondStress / AddBondPairStress
// (Monitor.cpp:1900-2755); see slice_stress.cuh.

struct SliceParams {
    int S;              // slices (0 = off)
    double width;       // L_z / S (Monitor.cpp:247)
    double inv;         // 1 / width (Monitor.cpp:2185)
    int nbt, nbpt;      // bond and bond-pair types
    double* pair;       // [S][T*T][9]
    double* bond;       // [S][nbt][9]
    double* bondpair;   // [S][nbpt][9]
    const int* bond_type;       // per bond
    const int* bondpair_type;   // per bond pair
};

__device__ __forceinline__ void outer9(const double f[3], const double d[3], double o[9])
{
    o[0] = f[0] * d[0]; o[1] = f[0] * d[1]; o[2] = f[0] * d[2];
    o[3] = f[1] * d[0]; o[4] = f[1] * d[1]; o[5] = f[1] * d[2];
    o[6] = f[2] * d[0]; o[7] = f[2] * d[1]; o[8] = f[2] * d[2];
}

struct Topology {
    const int* csr_ptr;     // per bead (upload index): first term
    const int* csr_term;    // term = index * 8 + code
    const int* bond_h;      // bond head / tail bead (upload index)
    const int* bond_t;
    const double* bond_k2;
    const double* bond_l0;
    const int* ang_b1h;     // first bond head (middle bead), first bond tail,
    const int* ang_b1t;     // second bond head, second bond tail
    const int* ang_b2h;
    const int* ang_b2t;
    const double* ang_k3;
    const double* ang_cos0; // cos(phi0); 1 when phi0 <= 0
    const double* ang_sin0; // sin(phi0); exactly 0 when phi0 <= 0 (the k3/|b1||b2| branch)
    const double4* ubuf;    // unPBC position by upload index (w: wrapped z), written by k_gather for bonded beads
    SliceParams sp;         // slice stress profile on sample steps (sp.S = 0: off)
};

enum TermCode { kBondHead = 0, kBondTail = 1, kAngle0 = 2, kAngle1 = 3, kAngle2 = 4 };

__device__ __forceinline__ void unwrapped(const double4* __restrict__ ubuf, int b, double u[3])
{
    const double4 q = ubuf[b];
    u[0] = q.x;
    u[1] = q.y;
    u[2] = q.z;
}

// CBond::AddForce (Bond.cpp:123-160, the serial build's unPBC coordinates):
// the bond vector b = head - tail and the force g on the head bead.
__device__ __forceinline__ void bond_force(const Topology& topo, int idx, double b[3], double g[3])
{
    double uh[3], ut[3];
    unwrapped(topo.ubuf, topo.bond_h[idx], uh);
    unwrapped(topo.ubuf, topo.bond_t[idx], ut);
    const double bx = uh[0] - ut[0], by = uh[1] - ut[1], bz = uh[2] - ut[2];
    const double len = sqrt(bx * bx + by * by + bz * bz);
    const double k2 = topo.bond_k2[idx], l0 = topo.bond_l0[idx];
    b[0] = bx; b[1] = by; b[2] = bz;
    g[0] = k2 * (l0 - len) * bx / len;
    g[1] = k2 * (l0 - len) * by / len;
    g[2] = k2 * (l0 - len) * bz / len;
}

// CBondPair::AddForce (BondPair.cpp:140-285): the unPBC positions of the
// first bond's tail and head and the second bond's head, and the forces on
// the first bond's tail (G0) and the second bond's head (G2); the middle bead
// takes -G0 - G2.  Zero forces for a degenerate pair (|b1||b2| <= 1e-4).
__device__ __forceinline__ void bondpair_force(const Topology& topo, int idx, double u1t[3], double u1h[3],
                                               double u2h[3], double G0[3], double G2[3])
{
    double u2t[3];
    unwrapped(topo.ubuf, topo.ang_b1h[idx], u1h);
    unwrapped(topo.ubuf, topo.ang_b1t[idx], u1t);
    unwrapped(topo.ubuf, topo.ang_b2h[idx], u2h);
    unwrapped(topo.ubuf, topo.ang_b2t[idx], u2t);
    double b1[3], b2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        b1[d] = u1h[d] - u1t[d];
        b2[d] = u2h[d] - u2t[d];
        G0[d] = 0.0;
        G2[d] = 0.0;
    }
    const double l1 = sqrt(b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2]);
    const double l2 = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    const double mag = l1 * l2;
    if (mag > 0.0001) {
        const double dot = b1[0] * b2[0] + b1[1] * b2[1] + b1[2] * b2[2];
        const double o1 = dot / (l1 * l1), o2 = dot / (l2 * l2);
        const double k3 = topo.ang_k3[idx];
        double fm = k3 / mag;
        const double s0 = topo.ang_sin0[idx];
        if (s0 != 0.0 && fabs(dot) > 0.000001) {
            const double pre = sqrt(1.0 / (o1 * o2) - 1.0);
            fm = k3 * (topo.ang_cos0[idx] - s0 / pre) / mag;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            G0[d] = fm * (o1 * b1[d] - b2[d]);
            G2[d] = fm * (b1[d] - o2 * b2[d]);
        }
    }
}

// Bond and bond-pair forces of one bonded bead each, in upload order (chains
// are contiguous there, so the partners' positions and the term tables are
// read as whole lines), FP64 in both precision modes: the bond-pair force
// with phi0 > 0 divides by sqrt(1/cos^2 - 1), which FP32 cannot resolve for
// nearly straight chains.  Each bond is evaluated by both of its beads and
// each bond pair by its three beads, so no atomics.  Writes the bonded force
// (and on sample steps the bond virial of the head bead) by upload index.
// The slice stress profile's bonded part is k_bonded_slices.
template <bool SAMPLE>
__global__ void __launch_bounds__(256) k_bonds(int nbb, int n, const int* __restrict__ bb, Topology topo,
                                               double4* __restrict__ Fb, double* __restrict__ Sb)
{
    pdl_wait();
    pdl_launch();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nbb) {
        const int b = bb[k];
        double bf[3] = {0.0, 0.0, 0.0};
        double bs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int t0 = topo.csr_ptr[b], t1 = topo.csr_ptr[b + 1];
        for (int t = t0; t < t1; ++t) {
            const int term = topo.csr_term[t];
            const int code = term & 7, idx = term >> 3;
            if (code <= kBondTail) {
                double bv[3], g[3];
                bond_force(topo, idx, bv, g);
                if (code == kBondHead) {
                    bf[0] += g[0]; bf[1] += g[1]; bf[2] += g[2];
                    if (SAMPLE) {
                        bs[0] += bv[0] * g[0]; bs[1] += bv[1] * g[0]; bs[2] += bv[2] * g[0];
                        bs[3] += bv[0] * g[1]; bs[4] += bv[1] * g[1]; bs[5] += bv[2] * g[1];
                        bs[6] += bv[0] * g[2]; bs[7] += bv[1] * g[2]; bs[8] += bv[2] * g[2];
                    }
                } else {
                    bf[0] -= g[0]; bf[1] -= g[1]; bf[2] -= g[2];
                }
            } else {
                double u1t[3], u1h[3], u2h[3], G0[3], G2[3];
                bondpair_force(topo, idx, u1t, u1h, u2h, G0, G2);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (code == kAngle0) bf[d] += G0[d];
                    else if (code == kAngle2) bf[d] += G2[d];
                    else bf[d] += -G0[d] - G2[d];
                }
            }
        }
        Fb[b] = make_double4(bf[0], bf[1], bf[2], 0.0);
        if (SAMPLE) {
#pragma unroll
            for (int q = 0; q < 9; ++q) Sb[(size_t)q * n + b] = bs[q];
        }
    }
}

// The slices one contribution spreads over (CMonitor::AddBeadStress /
// AddBondStress / AddBondPairStress, Monitor.cpp:2180-2755, with the same
// branch structure and arithmetic): za is the z of the bead the separation
// points to (bead 1, bond head, bead j+1), zb the other's, zDiff the
// separation's z component.  kind 0: none (a z rounded up to L_z, or a type
// out of range); 1: one slice whole; 2: two halves (both beads on one slice
// face); 3: a span of `n_inner` slices crossed whole (weight width/|dz|),
// then the lower end slice and, when covered, the upper one.
struct SliceSpan {
    int kind, ui, li, n_inner;
    double ur, lr, inner;
};

__device__ __forceinline__ SliceSpan slice_span(const SliceParams& sp, int K, int idx, double zDiff, double za,
                                                double zb)
{
    SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
    double up, lo;
    if (zDiff > 0.00001) {
        up = za * sp.inv;
        lo = zb * sp.inv;
    } else if (zDiff < -0.00001) {
        zDiff = -zDiff;
        up = zb * sp.inv;
        lo = za * sp.inv;
    } else {
        up = za * sp.inv;
        lo = up;
    }
    const int S = sp.S;
    s.ui = (int)up;
    s.ur = up - (double)s.ui;
    s.li = (int)lo;
    s.lr = lo - (double)s.li;
    if (s.ui < 0 || s.ui >= S || s.li < 0 || s.li >= S || idx < 0 || idx >= K) return s;
    if (s.ui == s.li) {
        s.kind = (up != lo || s.ur > 0.00001) ? 1 : 2;
    } else {
        s.kind = 3;
        s.inner = sp.width / zDiff;
        s.n_inner = s.ui > s.li ? s.ui - s.li - 1 : S + s.ui - s.li - 1;
    }
    return s;
}

__device__ __forceinline__ int span_count(const SliceSpan& s)
{
    return s.kind == 0 ? 0 : (s.kind == 1 ? 1 : (s.kind == 2 ? 2 : s.n_inner + 1 + (s.ur > 0.000001 ? 1 : 0)));
}

// Entry t of the span: slice and weight (1.0 for a slice taken whole).
__device__ __forceinline__ void span_entry(const SliceSpan& s, int S, int t, int& sl, double& fac)
{
    if (s.kind == 1) {
        sl = s.li;
        fac = 1.0;
    } else if (s.kind == 2) {
        sl = t == 0 ? s.ui : (s.li == 0 ? S - 1 : s.li - 1);
        fac = 0.5;
    } else if (t < s.n_inner) {
        const int k = s.li + 1 + t;
        sl = k >= S ? k - S : k;
        fac = s.inner;
    } else if (t == s.n_inner) {
        sl = s.li;
        fac = s.lr > 0.000001 ? (1.0 - s.lr) * s.inner : s.inner;
    } else {
        sl = s.ui;
        fac = s.ur * s.inner;
    }
}

// Adds v (9 components) to the FP64 bins arr[key * 9 ...] for every lane of
// the warp with key >= 0: the lanes sharing a key are summed by shuffles and
// one of them adds the sum, so lanes that meet on one bin (the bonds of a
// membrane leaflet share a few slices) take one atomic instead of queueing
// on it.  Called by all 32 lanes.
__device__ __forceinline__ void warp_bin_add(double* __restrict__ arr, int key, const double v[9])
{
    const int lane = threadIdx.x & 31;
    unsigned pending = __ballot_sync(0xffffffffu, key >= 0);
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const int kl = __shfl_sync(0xffffffffu, key, leader);
        const unsigned grp = __ballot_sync(0xffffffffu, key == kl);
        const bool mine = (grp >> lane) & 1u;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            double a = mine ? v[c] : 0.0;
#pragma unroll
            for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
            if (lane == leader) atomicAdd(arr + (size_t)kl * 9 + c, a);
        }
        pending &= ~grp;
    }
}

// One contribution of every lane (fdx over the span of slices between its
// beads) into bins arr[S][K][9]; lanes with cnt = 0 add nothing.
__device__ __forceinline__ void warp_span_add(const SliceParams& sp, double* __restrict__ arr, int K, int idx,
                                              const SliceSpan& s, const double fdx[9])
{
    const int cnt = span_count(s);
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    for (int t = 0; t < trip; ++t) {
        int key = -1;
        double v[9];
        if (t < cnt) {
            int sl;
            double fac;
            span_entry(s, sp.S, t, sl, fac);
            key = sl * K + idx;
#pragma unroll
            for (int c = 0; c < 9; ++c) v[c] = fdx[c] * fac;
        } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) v[c] = 0.0;
        }
        warp_bin_add(arr, key, v);
    }
}

// The bonded part of the slice stress profile on a sample step: one thread
// per bond (CMonitor::AddBondStress, the bond's force on its head x the bond
// vector, Monitor.cpp:2220-2470) and per bond pair (AddBondPairStress: the
// segments first tail -> first head -> second head -> first tail with force
// 0.33333333 (F[j+1] - F[j]), Monitor.cpp:2480-2755), the forces recomputed
// as k_bonds computes them.  Threads [0, nbp) are bonds and [nbp, nbp + na)
// bond pairs, nbp = nb rounded up to whole warps, so every warp runs one
// kind of term and the span loops are warp-uniform.  A degenerate bond pair
// adds zero, where the reference would reuse its last forces.
static __global__ void __launch_bounds__(256) k_bonded_slices(int nb, int na, Topology topo)
{
    const SliceParams& sp = topo.sp;
    const int nbp = (nb + 31) & ~31;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nbp) {
        const bool live = k < nb;
        double fdx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
        int type = 0;
        if (live) {
            double bv[3], g[3];
            bond_force(topo, k, bv, g);
            outer9(g, bv, fdx);
            type = sp.bond_type[k];
            s = slice_span(sp, sp.nbt, type, bv[2], topo.ubuf[topo.bond_h[k]].w, topo.ubuf[topo.bond_t[k]].w);
        }
        warp_span_add(sp, sp.bond, sp.nbt, type, s, fdx);
    } else if (k < nbp + ((na + 31) & ~31)) {
        const int a = k - nbp;
        const bool live = a < na;
        double U[4][3], FF[4][3], Z[4] = {0.0, 0.0, 0.0, 0.0};
        int type = 0;
        if (live) {
            double G0[3], G2[3];
            bondpair_force(topo, a, U[0], U[1], U[2], G0, G2);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                U[3][d] = U[0][d];
                FF[0][d] = G0[d];
                FF[1][d] = -G0[d] - G2[d];
                FF[2][d] = G2[d];
                FF[3][d] = G0[d];
            }
            Z[0] = topo.ubuf[topo.ang_b1t[a]].w;
            Z[1] = topo.ubuf[topo.ang_b1h[a]].w;
            Z[2] = topo.ubuf[topo.ang_b2h[a]].w;
            Z[3] = Z[0];
            type = sp.bondpair_type[a];
        }
        for (int j = 0; j < 3; ++j) {
            double fdx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
            if (live) {
                double dv[3], fo[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    dv[d] = U[j + 1][d] - U[j][d];
                    fo[d] = 0.33333333 * (FF[j + 1][d] - FF[j][d]);
                }
                outer9(fo, dv, fdx);
                s = slice_span(sp, sp.nbpt, type, dv[2], Z[j + 1], Z[j]);
            }
            warp_span_add(sp, sp.bondpair, sp.nbpt, type, s, fdx);
        }
    }
}

// The bonded force of k_bonds added per bead, then the velocity update of
// CCNTCell::UpdateMom: v = v_old + dt/2 (F + F_old) for movable beads.
// Non-movable beads keep v and, as in the reference (whose UpdatePos skips
// them), keep accumulating force.  On sample steps the FP64 single-bead sums
// are reduced per block.  With POS the same thread goes on with the next
// step's UpdatePos (drift, cell move, arrival counts), which saves a launch
// and a second pass over x, v, F and the flags; the drifted x, img and cell
// go to xo, imgo, cello -- the state arrays themselves between the steps of
// a call, separate buffers after its last step (the state the caller sees
// stays the step's own).  Each thread reads slot s before it writes it.
template <typename real, bool SAMPLE, bool POS>
__global__ void __launch_bounds__(256, 4) k_update_mom(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, int64_t* __restrict__ step_ptr,
    const double* x, double* __restrict__ v, real* __restrict__ F,
    const real* __restrict__ Fold, const int* __restrict__ bid, const int* __restrict__ tf,
    const double4* __restrict__ Fb, const double* __restrict__ Sb,
    real* __restrict__ stress, double* __restrict__ partials, const uint32_t* img, const int* cell,
    int* __restrict__ rank, int* __restrict__ count, int* __restrict__ block_count, unsigned* __restrict__ status,
    double* xo, uint32_t* imgo, int* cello)
{
    pdl_wait();
    pdl_launch();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < n;
    double acc[kObsTerms];
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) acc[q] = 0.0;
    int cnew = 0;
    unsigned bad = 0;
    if (live) {
        const int b = bid[s];
        const int tfl = tf[s];
        const bool frozen = flag_frozen(tfl);
        real f[3] = {F[s], F[n + s], F[2 * n + s]};
        real fo[3] = {Fold[s], Fold[n + s], Fold[2 * n + s]};
        const double v0[3] = {v[s], v[n + s], v[2 * n + s]};
        double xs[3] = {0.0, 0.0, 0.0};
        int c = 0;
        uint32_t im0 = 0;
        if (SAMPLE || POS) {
#pragma unroll
            for (int d = 0; d < 3; ++d) xs[d] = x[d * n + s];
        }
        if (POS) {
            c = cell[s];
            im0 = img[s];
        }
        if (frozen) { f[0] += fo[0]; f[1] += fo[1]; f[2] += fo[2]; }
        // Bonded terms (k_bonds, FP64) are added once, rounded into the
        // force accumulator.
        double bf[3] = {0.0, 0.0, 0.0};
        double bs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const bool bonded = flag_bonded(tfl);
        if (bonded) {
            const double4 g = Fb[b];
            bf[0] = g.x; bf[1] = g.y; bf[2] = g.z;
            if (SAMPLE) {
#pragma unroll
                for (int q = 0; q < 9; ++q) bs[q] = Sb[(size_t)q * n + b];
            }
        }
        if (bonded) {
#pragma unroll
            for (int d = 0; d < 3; ++d) f[d] = (real)((double)f[d] + bf[d]);
        }
        if (frozen || bonded) {   // otherwise F holds the pair force, the total already
            F[s] = f[0];
            F[n + s] = f[1];
            F[2 * n + s] = f[2];
        }
        if (!isfinite((double)f[0]) || !isfinite((double)f[1]) || !isfinite((double)f[2])) bad |= 0x2u;
        double vn[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            vn[d] = v0[d];
            if (!frozen) {
                vn[d] = __dadd_rn(vn[d], __dmul_rn(K->halfdt, __dadd_rn((double)f[d], (double)fo[d])));
                v[d * n + s] = vn[d];
            }
        }
        if (POS) {
            // UpdatePos of the next step (the drift uses this step's v and F)
            const double f0[3] = {(double)f[0], (double)f[1], (double)f[2]};
            cnew = drift_and_move(K, boxes, n, s, c, tfl, xs, vn, f0, im0, xo, imgo, cello, bad);
        }
        if (SAMPLE) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const real st = (real)((double)stress[q * n + s] + bs[q]);
                stress[q * n + s] = st;
                acc[6 + q] = (double)st;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                acc[d] = vn[d];
                acc[3 + d] = vn[d] * vn[d];
                acc[15 + d] = xs[d];
            }
            acc[18] = xs[1] * vn[2] - xs[2] * vn[1];
            acc[19] = -xs[0] * vn[2] + xs[2] * vn[0];
            acc[20] = xs[0] * vn[1] - xs[1] * vn[0];
        }
    }
    if (SAMPLE) {
        __shared__ double red[256 / 32][kObsTerms];
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
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += red[w][threadIdx.x];
            partials[threadIdx.x * gridDim.x + blockIdx.x] = a;   // term-major
        }
    }
    if (POS) count_arrival(live, s, cnew, rank, count, block_count);
    if (bad) atomicOr(status, bad);
    if (s == 0) *step_ptr += 1;
}

// Sets the step counter that keys the pair noise (a launch argument, so the
// host queues it without waiting for earlier work) when a call does not
// continue where the previous one ended, and publishes the status word of
// all work queued before it to `seen` (see publish_status).
static __global__ void k_set_step(int64_t* __restrict__ step_ptr, int64_t value, const unsigned* __restrict__ status,
                                  unsigned* seen)
{
    *step_ptr = value;
    *(volatile unsigned*)seen = *status;
}

// Fixed-order sum of the per-block partials (deterministic): one warp per
// term, coalesced reads of the term-major partials into four running sums per
// lane, then a fixed shuffle tree.
static __global__ void __launch_bounds__(32 * kObsTerms) k_reduce_obs(int nblocks, const double* __restrict__ partials,
                                                                       double* __restrict__ out)
{
    pdl_wait();
    pdl_launch();
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* p = partials + (size_t)q * nblocks;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int b = lane;
    for (; b + 96 < nblocks; b += 128) {
        a0 += p[b];
        a1 += p[b + 32];
        a2 += p[b + 64];
        a3 += p[b + 96];
    }
    for (; b < nblocks; b += 32) a0 += p[b];
    double a = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) out[q] = a;
}

// Kinetic sums without a force evaluation (state just uploaded).
static __global__ void __launch_bounds__(256) k_kinetic_partials(int n, const double* __restrict__ x,
                                                           const double* __restrict__ v,
                                                           double* __restrict__ partials)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kObsTerms];
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) acc[q] = 0.0;
    if (s < n) {
        const double xs[3] = {x[s], x[n + s], x[2 * n + s]};
        const double vs[3] = {v[s], v[n + s], v[2 * n + s]};
        for (int d = 0; d < 3; ++d) {
            acc[d] = vs[d];
            acc[3 + d] = vs[d] * vs[d];
            acc[15 + d] = xs[d];
        }
        acc[18] = xs[1] * vs[2] - xs[2] * vs[1];
        acc[19] = -xs[0] * vs[2] + xs[2] * vs[0];
        acc[20] = xs[0] * vs[1] - xs[1] * vs[0];
    }
    __shared__ double red[256 / 32][kObsTerms];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < kObsTerms; ++q) {
        double a = acc[q];
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) red[wid][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < kObsTerms) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += red[w][threadIdx.x];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = a;   // term-major
    }
}

// CSimBox::UpdateRenormalisedMom (SimBox.cpp:3177-3225): every momentum
// component divided by sqrt(sum v^2 / denom), denom = 3 N kT; sums[3..5] are
// the per-axis squared-momentum sums of k_kinetic_partials + k_reduce_obs.
static __global__ void __launch_bounds__(256) k_renorm_scale(int n, double* __restrict__ v,
                                                           const double* __restrict__ sums, double denom)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double scale = sqrt((sums[3] + sums[4] + sums[5]) / denom);
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d * n + s] = v[d * n + s] / scale;
}

// ---------------------------------------------------------------- download

// Slot order -> upload order, FP64, xyz interleaved; unPBC = x + img*L + off.
template <typename real>
__global__ void __launch_bounds__(256) k_download(
    int n, const Box* __restrict__ boxes, const int* __restrict__ tf, const int* __restrict__ bid,
    const double* __restrict__ x,
    const double* __restrict__ v, const real* __restrict__ F, const uint32_t* __restrict__ img,
    const double* __restrict__ off, const real* __restrict__ stress, const int* __restrict__ cell,
    double* __restrict__ ox, double* __restrict__ ou, double* __restrict__ ov, double* __restrict__ of,
    double* __restrict__ ost, int* __restrict__ ocell)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = bid[s];
    const uint32_t im = img[s];
    const Box& B = boxes[flag_box(tf[s])];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xv = x[d * n + s];
        if (ox) ox[3 * b + d] = xv;
        if (ou) ou[3 * b + d] = xv + (double)img_get(im, d) * B.L[d] + (off ? off[d * n + b] : 0.0);
        if (ov) ov[3 * b + d] = v[d * n + s];
        if (of) of[3 * b + d] = (double)F[d * n + s];
    }
    if (ost) {
#pragma unroll
        for (int q = 0; q < 9; ++q) ost[9 * b + q] = stress ? (double)stress[q * n + s] : 0.0;
    }
    if (ocell) ocell[b] = cell[s] - B.cell_base;
}

}  // namespace dpd
