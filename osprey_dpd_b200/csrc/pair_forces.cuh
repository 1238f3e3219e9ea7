// pair_forces.cuh -- the engine's DPD pair-force kernel (CCNTCell::UpdateForce,
// DPD branch, CNTCell.cpp:1103-1572) with warp-level hit compaction.
//
// Only ~15% of the candidates in the 27 neighbour cells lie inside the cut-off
// (rho = 3: 81 candidates, 12.6 partners per bead), so evaluating the force
// where the distance test passes would run the expensive body (sqrt, Philox,
// ~80 instructions) with a few lanes active on almost every iteration.  The
// kernel therefore splits the work in two phases inside each warp:
//
//   test   : every lane owns one bead i (a slot in cell order) and walks its
//            9 neighbour rows; a row (cells x-1, x, x+1 at fixed y', z') is one
//            contiguous slot range in the cell-sorted layout, split in two
//            only where it wraps around the x boundary.  Passing candidates are
//            appended to a per-warp queue in shared memory (ballot + popc).
//   force  : whenever 32 hits are queued, all 32 lanes evaluate one pair each
//            and add the force to the owning lane's accumulator in shared
//            memory.
//
// Every pair is evaluated from both sides (full shell), so bead i only ever
// accumulates its own force: no global atomics, and the result depends only on
// the cell-sorted order, which is deterministic.
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

constexpr int kPairWarps = 4;
constexpr int kPairBlock = 32 * kPairWarps;
// Resident blocks per SM the pair kernels are compiled for: 8 (64 registers,
// 32 warps) in FP32; the FP64 variants keep 6 to avoid spills.
template <typename real> struct PairOcc { static constexpr int value = sizeof(real) == 4 ? 8 : 6; };
constexpr int kHitCapMax = 64;           // upper bound of the run-time hit-list capacity

template <typename real> struct RealOps;
template <> struct RealOps<float> {
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
};
template <> struct RealOps<double> {
    static __device__ __forceinline__ double rsqrt(double x) { return 1.0 / sqrt(x); }
};

// Dynamic shared memory of one block: pair tables, then the hit lists
// (entry k of thread t at lists[k * kPairBlock + t], so a warp's stores and
// loads of one k hit 32 consecutive words).
template <typename real>
__host__ __device__ constexpr size_t pair_tables_bytes(int nt)
{
    return ((3 * sizeof(real) * (size_t)nt * nt + 15) / 16) * 16;
}
template <typename real>
__host__ __device__ constexpr size_t pair_smem_bytes(int nt, int hitcap, bool multi)
{
    return (multi ? 0 : pair_tables_bytes<real>(nt)) + sizeof(uint32_t) * hitcap * kPairBlock;
}

// Hit entry: candidate slot in bits 0..25, cell offsets + 1 (x, y, z) in
// 2-bit fields at bits 26, 28, 30.
__device__ __forceinline__ uint32_t hit_pack(int j, int ox1, int oy1, int oz1)
{
    return (uint32_t)j | ((uint32_t)ox1 << 26) | ((uint32_t)oy1 << 28) | ((uint32_t)oz1 << 30);
}

// Evaluates this lane's listed hits (the DPD force of CNTCell.cpp:1192-1220
// with rc = 1) and adds them, in list order, to the lane's own accumulator.
template <typename real, bool VIRIAL>
__device__ __forceinline__ void pair_force_pass(int cnt, const uint32_t* __restrict__ list,
                                                const typename Vec4<real>::type& pi,
                                                const typename Vec4<real>::type& vi, const real* __restrict__ T,
                                                int nt, real wx, real wy, real wz, const uint32_t* keys,
                                                const typename Vec4<real>::type* __restrict__ pos4,
                                                const typename Vec4<real>::type* __restrict__ vel4, real* acc)
{
    typedef typename Vec4<real>::type V4;
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    const int ti = (real_bits(pi.w) & 0xFF) * nt;
    const uint32_t idi = (uint32_t)real_bits(vi.w);
    const int m2 = nt * nt;
    for (int k = 0; k < trip; ++k) {
        if (k < cnt) {
            const uint32_t e = list[k * kPairBlock];
            const int j = (int)(e & 0x03FFFFFFu);
            const V4 pj = pos4[j];
            const V4 vj = vel4[j];
            const real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
            const real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
            const real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
            const real r2 = dx * dx + dy * dy + dz * dz;
            const real inv = RealOps<real>::rsqrt(r2);
            const real wr = real(1) - r2 * inv;
            const int tt = ti + (real_bits(pj.w) & 0xFF);
            const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
            const uint32_t idj = (uint32_t)real_bits(vj.w);
            uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                const uint64_t prod = (uint64_t)0xD256D193u * c0;   // one wide multiply per round
                c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
                c1 = (uint32_t)prod;
            }
            const real mag = T[tt] * wr - T[m2 + tt] * wr * wr * rdotv +
                             T[2 * m2 + tt] * wr * noise_centered(c0, real(0));
            const real m = mag * inv;
            const real gx = m * dx, gy = m * dy, gz = m * dz;
            acc[0] += gx; acc[1] += gy; acc[2] += gz;
            if (VIRIAL) {
                acc[3] += dx * gx; acc[4] += dy * gx; acc[5] += dz * gx;
                acc[6] += dx * gy; acc[7] += dy * gy; acc[8] += dz * gy;
                acc[9] += dx * gz; acc[10] += dy * gz; acc[11] += dz * gz;
            }
        }
    }
}

// Slot range of row segment `seg` (0 or 1) for a bead in cell column cx: the
// row's cells x-1, x, x+1 are one contiguous range except where the row wraps
// around the x boundary, which splits it in two.  Cell offset of slot j:
// -1 below b1, 0 in [b1, b2), +1 from b2.
__device__ __forceinline__ void row_segment(bool live, int seg, int rb, int cx, int nx, const int* __restrict__ start,
                                            int& lo, int& hi, int& b1, int& b2)
{
    if (!live) {
        lo = hi = b1 = b2 = 0;
    } else if (cx > 0 && cx < nx - 1) {
        if (seg == 0) {
            lo = start[rb + cx - 1]; b1 = start[rb + cx]; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2];
        } else {
            lo = hi = b1 = b2 = 0;
        }
    } else if (cx == 0) {
        if (seg == 0) { lo = b1 = start[rb]; b2 = start[rb + 1]; hi = start[rb + 2]; }
        else { lo = start[rb + nx - 1]; hi = b1 = b2 = start[rb + nx]; }
    } else {
        if (seg == 0) { lo = start[rb + nx - 2]; b1 = start[rb + nx - 1]; hi = b2 = start[rb + nx]; }
        else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; }
    }
}

// Persistent blocks: block b evaluates the contiguous tiles [b*tpb, (b+1)*tpb)
// of kPairBlock slots, so consecutive tiles of one block walk neighbouring
// cells and reuse the neighbour rows already in its SM's L1.
// MULTI: beads of many boxes (a replica batch); each bead takes its box, pair
// tables and noise key from the packed box table, tables are read through the
// read-only cache.  Otherwise one box whose tables are staged in shared memory.
template <typename real, bool VIRIAL, bool MULTI>
__global__ void __launch_bounds__(kPairBlock, PairOcc<real>::value) k_pair_forces(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, int tiles_per_block,
    unsigned* __restrict__ status)
{
    typedef typename Vec4<real>::type V4;
    extern __shared__ __align__(16) unsigned char pair_dyn[];
    const int nt = K->ntypes;
    real* Tsh = reinterpret_cast<real*>(pair_dyn);    // a, gamma, sigma: 3 * ntypes^2
    uint32_t* list = reinterpret_cast<uint32_t*>(pair_dyn + (MULTI ? 0 : pair_tables_bytes<real>(nt))) + threadIdx.x;
    if (!MULTI)
        for (int k = threadIdx.x; k < 3 * nt * nt; k += kPairBlock) Tsh[k] = tab[k];
    const int64_t step = *step_ptr;
    __syncthreads();   // tables
    const int tile0 = blockIdx.x * tiles_per_block;
    for (int tile = tile0; tile < tile0 + tiles_per_block; ++tile) {
    const int i = tile * kPairBlock + threadIdx.x;
    if (tile * kPairBlock >= n) break;
    const bool live = i < n;
    V4 pi, vi;
    int cx = 0, cy = 0, cz = 0;
    if (live) {
        pi = pos4[i];
        vi = vel4[i];
    } else {
        pi.x = pi.y = pi.z = pi.w = vi.x = vi.y = vi.z = vi.w = real(0);
    }
    const Box& B = boxes[MULTI ? flag_box(real_bits(pi.w)) : 0];
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    if (live) {
        const int c = cell[i] - B.cell_base;
        cx = c % nx;
        cy = (c / nx) % ny;
        cz = c / (nx * ny);
    }
    const real* T = MULTI ? tab + B.tab : Tsh;
    uint32_t keys[10];
    {
        uint32_t k = philox_step_key(B.seed, step);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
    }
    const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
    // home x shifted into the frame of the row's cells x-1, x, x+1
    const real pxm = pi.x + wx, px0 = pi.x, pxp = pi.x - wx;
    constexpr int NACC = VIRIAL ? 12 : 3;
    real acc[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) acc[q] = real(0);
    int cnt = 0;
    for (int r = 0; r < 9; ++r) {
        const int dy = r % 3 - 1, dz = r / 3 - 1;
        int y2 = cy + dy, z2 = cz + dz;
        y2 += (y2 < 0) ? ny : ((y2 >= ny) ? -ny : 0);
        z2 += (z2 < 0) ? nz : ((z2 >= nz) ? -nz : 0);
        const int rb = B.cell_base + nx * (y2 + ny * z2);
        const real piy = pi.y - (real)dy * wy, piz = pi.z - (real)dz * wz;
        const uint32_t rowbits = ((uint32_t)(dy + 1) << 28) | ((uint32_t)(dz + 1) << 30);
        for (int seg = 0; seg < 2; ++seg) {
            // slots [lo, hi): cell offset -1 below b1, 0 in [b1, b2), +1 from b2
            int lo, hi, b1, b2;
            row_segment(live, seg, rb, cx, nx, start, lo, hi, b1, b2);
            const int len = hi - lo;
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            // chunks of at most hitcap candidates, so a list can never overflow
            for (int base = 0; base < trip; base += hitcap) {
                const int clen = min(max(len - base, 0), hitcap);
                if (__any_sync(0xffffffffu, cnt + clen > hitcap)) {
                    pair_force_pass<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc);
                    cnt = 0;
                }
                const int tend = base + min(trip - base, hitcap);
                // Two candidates per iteration (independent loads in flight).
                // The bead itself (r2 = 0) fails r2 > 1e-18, the reference's
                // dr > 1e-9 test (CNTCell.cpp:1202), so no separate j != i test.
                // cnt + clen <= hitcap holds here, so the stores stay in range.
                for (int t = base; t < tend; t += 2) {
                    const int j0 = lo + t, j1 = j0 + 1;
                    const bool h0 = t < len, h1 = t + 1 < len && t + 1 < tend;
                    V4 p0, p1;
                    if (h0) p0 = pos4[j0];
                    if (h1) p1 = pos4[j1];
                    if (h0) {
                        const bool ge1 = j0 >= b1, ge2 = j0 >= b2;
                        const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p0.x;
                        const real ddy = piy - p0.y, ddz = piz - p0.z;
                        const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        if ((r2 < real(1)) && (r2 > real(1e-18))) {
                            list[cnt * kPairBlock] = (uint32_t)j0 | ((uint32_t)(ge1 + ge2) << 26) | rowbits;
                            ++cnt;
                        }
                    }
                    if (h1) {
                        const bool ge1 = j1 >= b1, ge2 = j1 >= b2;
                        const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p1.x;
                        const real ddy = piy - p1.y, ddz = piz - p1.z;
                        const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        if ((r2 < real(1)) && (r2 > real(1e-18))) {
                            list[cnt * kPairBlock] = (uint32_t)j1 | ((uint32_t)(ge1 + ge2) << 26) | rowbits;
                            ++cnt;
                        }
                    }
                }
            }
        }
    }
    pair_force_pass<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc);
    if (live) {
        F[i] = acc[0];
        F[n + i] = acc[1];
        F[2 * n + i] = acc[2];
        if (VIRIAL) {
#pragma unroll
            for (int q = 0; q < 9; ++q) stress[q * n + i] = real(0.5) * acc[3 + q];
        }
    }
    }
}

// ------------------------------------------------------------ half shell

// This lane's listed pairs, each evaluated once: the force goes to the lane's
// own accumulator and, negated, to the partner through atomics.
template <typename real, bool VIRIAL>
__device__ __forceinline__ void pair_force_pass_half(int cnt, const uint32_t* __restrict__ list,
                                                     const typename Vec4<real>::type& pi,
                                                     const typename Vec4<real>::type& vi, const real* __restrict__ T,
                                                     int nt, real wx, real wy, real wz, const uint32_t* keys,
                                                     const typename Vec4<real>::type* __restrict__ pos4,
                                                     const typename Vec4<real>::type* __restrict__ vel4, real* acc,
                                                     real* __restrict__ F, int n)
{
    typedef typename Vec4<real>::type V4;
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    const int ti = (real_bits(pi.w) & 0xFF) * nt;
    const uint32_t idi = (uint32_t)real_bits(vi.w);
    const int m2 = nt * nt;
    for (int k = 0; k < trip; ++k) {
        if (k < cnt) {
            const uint32_t e = list[k * kPairBlock];
            const int j = (int)(e & 0x03FFFFFFu);
            const V4 pj = pos4[j];
            const V4 vj = vel4[j];
            const real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
            const real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
            const real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
            const real r2 = dx * dx + dy * dy + dz * dz;
            const real inv = RealOps<real>::rsqrt(r2);
            const real wr = real(1) - r2 * inv;
            const int tt = ti + (real_bits(pj.w) & 0xFF);
            const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
            const uint32_t idj = (uint32_t)real_bits(vj.w);
            uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                const uint64_t prod = (uint64_t)0xD256D193u * c0;
                c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
                c1 = (uint32_t)prod;
            }
            const real mag = T[tt] * wr - T[m2 + tt] * wr * wr * rdotv +
                             T[2 * m2 + tt] * wr * noise_centered(c0, real(0));
            const real m = mag * inv;
            const real gx = m * dx, gy = m * dy, gz = m * dz;
            acc[0] += gx; acc[1] += gy; acc[2] += gz;
            atomicAdd(F + j, -gx);
            atomicAdd(F + n + j, -gy);
            atomicAdd(F + 2 * n + j, -gz);
            if (VIRIAL) {
                acc[3] += dx * gx; acc[4] += dy * gx; acc[5] += dz * gx;
                acc[6] += dx * gy; acc[7] += dy * gy; acc[8] += dz * gy;
                acc[9] += dx * gz; acc[10] += dy * gz; acc[11] += dz * gz;
            }
        }
    }
}

// Half-shell variant: every pair once, as CCNTCell::UpdateForce visits them
// (CNTCell.cpp:1103-1572, m_aIntNNCells): the beads after bead i in its own cell and the 13
// cells of the half shell (dz = +1: all nine; dz = 0: dy = +1 row; dy = 0:
// the cell at dx = +1).  In slot terms: own row [i+1, end of cell x+1), the
// (dy=+1, dz=0) row and the three dz=+1 rows.  Half the distance tests and
// force bodies of the full shell; the partner's share is added with global
// atomics, so the FP32 summation order (and the last bits) vary from run to
// run.  F must be zero on entry.  The pair virial goes whole to bead i, the
// reference's convention (CNTCell.cpp:1283-1301).
template <typename real, bool VIRIAL, bool MULTI>
__global__ void __launch_bounds__(kPairBlock, PairOcc<real>::value) k_pair_forces_half(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, int tiles_per_block,
    unsigned* __restrict__ status)
{
    typedef typename Vec4<real>::type V4;
    extern __shared__ __align__(16) unsigned char pair_dyn[];
    const int nt = K->ntypes;
    real* Tsh = reinterpret_cast<real*>(pair_dyn);
    uint32_t* list = reinterpret_cast<uint32_t*>(pair_dyn + (MULTI ? 0 : pair_tables_bytes<real>(nt))) + threadIdx.x;
    if (!MULTI)
        for (int k = threadIdx.x; k < 3 * nt * nt; k += kPairBlock) Tsh[k] = tab[k];
    const int64_t step = *step_ptr;
    __syncthreads();   // tables
    const int tile0 = blockIdx.x * tiles_per_block;
    for (int tile = tile0; tile < tile0 + tiles_per_block; ++tile) {
        const int i = tile * kPairBlock + threadIdx.x;
        if (tile * kPairBlock >= n) break;
        const bool live = i < n;
        V4 pi, vi;
        int cx = 0, cy = 0, cz = 0;
        if (live) {
            pi = pos4[i];
            vi = vel4[i];
        } else {
            pi.x = pi.y = pi.z = pi.w = vi.x = vi.y = vi.z = vi.w = real(0);
        }
        const Box& B = boxes[MULTI ? flag_box(real_bits(pi.w)) : 0];
        const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
        if (live) {
            const int c = cell[i] - B.cell_base;
            cx = c % nx;
            cy = (c / nx) % ny;
            cz = c / (nx * ny);
        }
        const real* T = MULTI ? tab + B.tab : Tsh;
        uint32_t keys[10];
        {
            uint32_t k = philox_step_key(B.seed, step);
#pragma unroll
            for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
        }
        const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
        const real pxm = pi.x + wx, px0 = pi.x, pxp = pi.x - wx;
        constexpr int NACC = VIRIAL ? 12 : 3;
        real acc[NACC];
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q] = real(0);
        int cnt = 0;
        for (int r = 0; r < 5; ++r) {
            const int dy = r == 0 ? 0 : (r == 1 ? 1 : r - 3);
            const int dz = r < 2 ? 0 : 1;
            int y2 = cy + dy, z2 = cz + dz;
            y2 += (y2 >= ny) ? -ny : 0;
            z2 += (z2 >= nz) ? -nz : 0;
            y2 += (y2 < 0) ? ny : 0;
            const int rb = B.cell_base + nx * (y2 + ny * z2);
            const real piy = pi.y - (real)dy * wy, piz = pi.z - (real)dz * wz;
            const uint32_t rowbits = ((uint32_t)(dy + 1) << 28) | ((uint32_t)(dz + 1) << 30);
            for (int seg = 0; seg < 2; ++seg) {
                int lo, hi, b1, b2;
                if (r > 0) {
                    row_segment(live, seg, rb, cx, nx, start, lo, hi, b1, b2);
                } else if (!live) {
                    lo = hi = b1 = b2 = 0;
                } else if (cx < nx - 1) {
                    // own cell after i, then cell x+1 (offset +1 from b2)
                    if (seg == 0) { lo = b1 = i + 1; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2]; }
                    else { lo = hi = b1 = b2 = 0; }
                } else {
                    // cx = nx-1: own cell after i, then cell 0 across the boundary
                    if (seg == 0) { lo = b1 = i + 1; b2 = hi = start[rb + cx + 1]; }
                    else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; }
                }
                const int len = hi - lo;
                const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
                for (int base = 0; base < trip; base += hitcap) {
                    const int clen = min(max(len - base, 0), hitcap);
                    if (__any_sync(0xffffffffu, cnt + clen > hitcap)) {
                        pair_force_pass_half<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4,
                                                           acc, F, n);
                        cnt = 0;
                    }
                    const int tend = base + min(trip - base, hitcap);
                    for (int t = base; t < tend; t += 2) {
                        const int j0 = lo + t, j1 = j0 + 1;
                        const bool h0 = t < len, h1 = t + 1 < len && t + 1 < tend;
                        V4 p0, p1;
                        if (h0) p0 = pos4[j0];
                        if (h1) p1 = pos4[j1];
                        if (h0) {
                            const bool ge1 = j0 >= b1, ge2 = j0 >= b2;
                            const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p0.x;
                            const real ddy = piy - p0.y, ddz = piz - p0.z;
                            const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            if ((r2 < real(1)) && (r2 > real(1e-18))) {
                                list[cnt * kPairBlock] = (uint32_t)j0 | ((uint32_t)(ge1 + ge2) << 26) | rowbits;
                                ++cnt;
                            }
                        }
                        if (h1) {
                            const bool ge1 = j1 >= b1, ge2 = j1 >= b2;
                            const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p1.x;
                            const real ddy = piy - p1.y, ddz = piz - p1.z;
                            const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            if ((r2 < real(1)) && (r2 > real(1e-18))) {
                                list[cnt * kPairBlock] = (uint32_t)j1 | ((uint32_t)(ge1 + ge2) << 26) | rowbits;
                                ++cnt;
                            }
                        }
                    }
                }
            }
        }
        pair_force_pass_half<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc, F, n);
        if (live) {
            atomicAdd(F + i, acc[0]);
            atomicAdd(F + n + i, acc[1]);
            atomicAdd(F + 2 * n + i, acc[2]);
            if (VIRIAL) {
#pragma unroll
                for (int q = 0; q < 9; ++q) stress[q * n + i] = acc[3 + q];
            }
        }
    }
}

}  // namespace dpd
