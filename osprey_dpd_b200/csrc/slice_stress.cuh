// slice_stress.cuh -- the slice stress profile of CMonitor (AddBeadStress,
// AddBondStress, AddBondPairStress, Monitor.cpp:1900-2755) on the device.
//
// The reference adds, for every interacting pair, bond and bond-pair segment,
// the 9 products force x separation to the z slices between the two beads
// (the Goetz-Lipowsky contour: a slice fully crossed gets width / |dz|, the
// end slices their covered fraction, beads in one slice give it the whole
// product), per type pair / bond type / bond-pair type.  It zeroes the
// profile every step (SimBox.cpp:999) and only the stress-profile analysis
// reads it, at sample time (aaStressTensor1d.cpp:150-200), so the engine
// builds it on sample steps only.
//
// Pairs are enumerated over the reference's own half shell (CSimBox::
// MakeCNTCells, SimBox.cpp:845-856: dz = +1; dz = 0, dx = +1; dz = dx = 0,
// dy = +1), so the reference's "bead 1" (type index t1 * T + t2, and the z
// used when |dz| <= 1e-5) is reproduced for every pair in different cells;
// for a pair inside one cell the reference's order is its linked-list order,
// and the engine takes the lower slot as bead 1.
// SliceParams and the contour split itself (slice_span, span_entry) live in
// dpd_kernels.cuh, shared with the bonded kernel.
#pragma once
#include "pair_forces.cuh"

namespace dpd {

// Pair part on a sample step, in two phases per 128-bead tile (one lane per
// bead i).  Test: the lane walks its own cell (beads after i) and the 13 cells
// of the reference's half shell, one cell at a time (a constant cell shift),
// and lists the candidates inside the cut-off in its column of shared memory.
// Evaluate: the lane takes its listed pairs, computes the DPD pair force of the
// force kernels (same Philox draw) and splits force x separation over the
// slices (slice_span).  Only listed pairs pay for the force and the split, so
// no lane idles through another's force work on the ~85 % of candidates that
// miss.  Bins are block-private in shared memory when they fit (sbins) --
// FP32 partial sums in a mixed-precision engine, FP64 in an FP64 engine --
// and added once per block to the FP64 profile; else they go straight to
// global memory.  Grid-stride loop over warps; each lane's beads lie in its
// own 32nd of the box (see below).
constexpr int kSliceBlock = 128;
constexpr int kSliceHits = 32;   // list entries per lane before an evaluation pass
constexpr int kSliceListPerBead = 16;   // capacity of the profile's pair list (6.3 pairs a bead at rho = 3)

template <typename real>
__host__ __device__ constexpr size_t slice_bin_bytes(int S, int KT)
{
    return ((sizeof(real) * (size_t)S * KT * 9 + 15) / 16) * 16;
}
template <typename real>
__host__ __device__ constexpr size_t slice_smem_bytes(int S, int KT, bool sbins)
{
    return (sbins ? slice_bin_bytes<real>(S, KT) : 0) + sizeof(uint32_t) * (kSliceHits + 1) * kSliceBlock;
}

// The contribution of pair (i, j) to the profile, i the reference's bead 1:
// the DPD pair force of the force kernels (same Philox draw), force x
// separation (fdx) and the slices it spreads over (s, kind 0 when the pair
// lies at or beyond the cut-off: the test's rounding differs there).  e is a
// hit-list entry (partner slot and cell offsets + 1).
template <typename real>
__device__ __forceinline__ void slice_pair(uint32_t e, int i, int n, const typename Vec4<real>::type& pi,
                                           const typename Vec4<real>::type& vi, double zi,
                                           const real* __restrict__ tab, int nt, const uint32_t* keys, real wx,
                                           real wy, real wz, const typename Vec4<real>::type* __restrict__ pos4,
                                           const typename Vec4<real>::type* __restrict__ vel4,
                                           const double* __restrict__ x, const SliceParams& sp, const double* L,
                                           double fdx[9], SliceSpan& s, int& tt)
{
    typedef typename Vec4<real>::type V4;
    const int m2 = nt * nt;
    const int j = (int)(e & 0x03FFFFFFu);
    const V4 pj = pos4[j];
    const V4 vj = vel4[j];
    real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
    real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
    real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
    const real r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 < real(1) && r2 > real(1e-18))) return;
    const real inv = RealOps<real>::rsqrt(r2);
    const real wr = real(1) - r2 * inv;
    tt = (real_bits(pi.w) & 0xFF) * nt + (real_bits(pj.w) & 0xFF);
    const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
    const uint32_t idi = (uint32_t)real_bits(vi.w), idj = (uint32_t)real_bits(vj.w);
    uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
    for (int q = 0; q < 10; ++q) {
        const uint64_t prod = (uint64_t)0xD256D193u * c0;
        c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
        c1 = (uint32_t)prod;
    }
    const real ta = tab[tt], tg = tab[m2 + tt], ts = tab[2 * m2 + tt], noise = noise_centered(c0, real(0));
    real m = (ta * wr - tg * wr * wr * rdotv + ts * wr * noise) * inv;
    close_pair_fix(dx, dy, dz, m, r2, x, n, i, j, L, vi, vj, ta, tg, ts, noise);
    const double f[3] = {(double)(m * dx), (double)(m * dy), (double)(m * dz)};
    const double d[3] = {(double)dx, (double)dy, (double)dz};
    outer9(f, d, fdx);
    s = slice_span(sp, nt * nt, tt, d[2], zi, x[2 * (size_t)n + j]);
}

// Every lane's contribution into the bins, the adds of one slice issued
// together (warp-uniform loop over the longest span).  Called by all 32 lanes.
template <typename bin_t>
__device__ __forceinline__ void slice_add_span(bin_t* bins, int KT, int S, int tt, const SliceSpan& s,
                                               const double fdx[9])
{
    const int ms = span_count(s);
    const int mt = (int)__reduce_max_sync(0xffffffffu, (unsigned)ms);
    for (int t = 0; t < mt; ++t) {
        if (t < ms) {
            int sl;
            double fac;
            span_entry(s, S, t, sl, fac);
            bin_t* q = bins + ((size_t)sl * KT + tt) * 9;
#pragma unroll
            for (int c = 0; c < 9; ++c) atomicAdd(q + c, (bin_t)(fdx[c] * fac));
        }
    }
}

// The listed pairs of the warp's lanes, one pair per lane per iteration (the
// loop runs to the longest list, so it is warp-uniform).  Called by all 32
// lanes.  bins: the block's shared bins (real) or the global FP64 profile.
template <typename real, typename bin_t>
__device__ __forceinline__ void slice_eval(int cnt, const uint32_t* __restrict__ list, int i, int n,
                                           const typename Vec4<real>::type& pi, const typename Vec4<real>::type& vi,
                                           double zi, const real* __restrict__ tab, int nt, const uint32_t* keys,
                                           real wx, real wy, real wz, const typename Vec4<real>::type* __restrict__ pos4,
                                           const typename Vec4<real>::type* __restrict__ vel4,
                                           const double* __restrict__ x, const SliceParams& sp, bin_t* bins,
                                           const double* L)
{
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    for (int k = 0; k < trip; ++k) {
        double fdx[9];
        SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
        int tt = 0;
        if (k < cnt)
            slice_pair<real>(list[k * kSliceBlock], i, n, pi, vi, zi, tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp, L,
                             fdx, s, tt);
        slice_add_span(bins, nt * nt, sp.S, tt, s, fdx);
    }
}

// Global list of the profile's pairs (bead 1 slot, hit entry), filled by
// k_slice_pairs in list mode and evaluated by k_slice_eval.  count[0]:
// entries appended (may pass cap), count[1]: nonzero when an append did not
// fit, in which case k_slice_pairs in fallback mode builds the profile the
// one-kernel way.
struct SliceList {
    uint2* pairs;
    unsigned* count;
    int cap;
};

// The warp's per-lane hit lists appended to the global list: one atomic per
// warp (prefix of the lane counts).  Called by all 32 lanes.
__device__ __forceinline__ void slice_flush(int cnt, const uint32_t* __restrict__ list, int i, const SliceList& L)
{
    const int lane = threadIdx.x & 31;
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    const int total = __shfl_sync(0xffffffffu, inc, 31);
    if (total == 0) return;
    unsigned base = 0;
    if (lane == 31) base = atomicAdd(L.count, (unsigned)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    if ((long long)base + total > (long long)L.cap) {   // warp-uniform
        if (lane == 0) atomicOr(L.count + 1, 1u);
        return;
    }
    const unsigned o = base + (unsigned)(inc - cnt);
    for (int k = 0; k < cnt; ++k) {
        const uint32_t e = list[k * kSliceBlock];
        // x code 3 (unused by offsets): the reference's bead 1 is the partner,
        // which sees slot i at cell offset (+1, -1, 0)
        L.pairs[o + k] = ((e >> 26) & 3u) == 3u
                             ? make_uint2(e & 0x03FFFFFFu, (unsigned)i | (2u << 26) | (0u << 28) | (1u << 30))
                             : make_uint2((unsigned)i, e);
    }
}

// List mode's test for the 128 slots of one tile (lane = slot, consecutive
// slots per warp): the half shell of the force kernels (own row: cell x after
// slot i and cell x+1; the row dy = +1; the three rows dz = +1), row windows
// pruned as there and four candidates in flight.  That half shell and the
// reference's (CSimBox::MakeCNTCells, SimBox.cpp:845-856) differ in one cell
// offset, (-1, +1, 0) against (+1, -1, 0): such pairs are listed with the
// partner as bead 1 (x code 3, decoded by slice_flush), so every pair is
// listed once, oriented as the reference orients it.
template <typename real>
__device__ __forceinline__ void slice_list_tile(int i, int n, const Box& B, const int* __restrict__ cell,
                                                const int* __restrict__ start,
                                                const typename Vec4<real>::type* __restrict__ pos4,
                                                uint32_t* list, const SliceList& L)
{
    typedef typename Vec4<real>::type V4;
    const bool live = i < n;
    V4 pi;
    int cx = 0, cy = 0, cz = 0;
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    if (live) {
        pi = pos4[i];
        int cc[3];
        cell_coords(B, cell[i] - B.cell_base, cc);
        cx = cc[0];
        cy = cc[1];
        cz = cc[2];
    } else {
        pi.x = pi.y = pi.z = pi.w = real(0);
    }
    const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
    const real pxm = pi.x + wx, px0 = pi.x, pxp = pi.x - wx;
    int cnt = 0;
    const int nseg = __any_sync(0xffffffffu, live && (cx == 0 || cx == nx - 1)) ? 2 : 1;
    for (int r = 0; r < 5; ++r) {
        int dy, dz;
        stg_row_shift(r, dy, dz);
        int y2 = cy + dy, z2 = cz + dz;
        y2 += (y2 >= ny) ? -ny : 0;
        z2 += (z2 >= nz) ? -nz : 0;
        y2 += (y2 < 0) ? ny : 0;
        const int rb = B.cell_base + nx * (y2 + ny * z2);
        const real piy = pi.y - (real)dy * wy, piz = pi.z - (real)dz * wz;
        const uint32_t rowbits = ((uint32_t)(dy + 1) << 28) | ((uint32_t)(dz + 1) << 30);
        // cell x-1 of the row dy = +1, dz = 0 is the offset the reference lists from the partner's side
        const uint32_t code_m = r == 1 ? (3u << 26) : rowbits, code_0 = rowbits | (1u << 26),
                       code_p = rowbits | (2u << 26);
        const real gy = dy > 0 ? wy - pi.y : (dy < 0 ? pi.y : real(0));
        const real gz = dz > 0 ? wz - pi.z : real(0);
        const real gyz = gy * gy + gz * gz;
        const real gxp = wx - pi.x;
        const bool keep_0 = gyz < kPruneR2;
        const bool keep_m = pi.x * pi.x + gyz < kPruneR2;
        const bool keep_p = gxp * gxp + gyz < kPruneR2;
        for (int seg = 0; seg < nseg; ++seg) {
            int lo, hi, b1, b2;
            if (r > 0) {
                row_segment(live, seg, rb, cx, nx, start, lo, hi, b1, b2);
            } else if (!live) {
                lo = hi = b1 = b2 = 0;
            } else if (cx < nx - 1) {
                if (seg == 0) { lo = b1 = i + 1; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2]; }
                else { lo = hi = b1 = b2 = 0; }
            } else {
                if (seg == 0) { lo = b1 = i + 1; b2 = hi = start[rb + cx + 1]; }
                else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; }
            }
            lo = keep_m ? lo : b1;
            hi = keep_p ? hi : b2;
            hi = keep_0 ? hi : lo;
            const int len = max(hi - lo, 0);
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            for (int base = 0; base < trip; base += kSliceHits) {
                const int clen = min(max(len - base, 0), kSliceHits);
                if (__any_sync(0xffffffffu, cnt + clen > kSliceHits)) {
                    slice_flush(cnt, list, i, L);
                    cnt = 0;
                }
                const int tend = base + min(trip - base, kSliceHits);
                const int lim = min(len, tend);
                const int tend4 = base + ((tend - base) & ~3);
                int t = base;
                for (; t < tend4; t += 4) {
                    const int j0 = lo + t, rem = lim - t;
                    V4 p[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) p[q] = pos4[min(j0 + q, n - 1)];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int jq = j0 + q;
                        const bool ge1 = jq >= b1, ge2 = jq >= b2;
                        const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p[q].x;
                        const real ddy = piy - p[q].y, ddz = piz - p[q].z;
                        const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        list[cnt * kSliceBlock] = (uint32_t)min(jq, n - 1) | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                        cnt += (r2 < real(1) && r2 > real(1e-18) && q < rem) ? 1 : 0;
                    }
                }
                for (; t < tend; ++t) {
                    const int jq = lo + t;
                    const V4 pq = pos4[min(jq, n - 1)];
                    const bool ge1 = jq >= b1, ge2 = jq >= b2;
                    const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - pq.x;
                    const real ddy = piy - pq.y, ddz = piz - pq.z;
                    const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    list[cnt * kSliceBlock] = (uint32_t)min(jq, n - 1) | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                    cnt += (r2 < real(1) && r2 > real(1e-18) && t < lim) ? 1 : 0;
                }
            }
        }
    }
    slice_flush(cnt, list, i, L);
}

// mode kSliceOne: test and evaluate (the profile in one kernel); kSliceList:
// test only, the pairs appended to L; kSliceFallback: kSliceOne when L
// overflowed, else nothing.
enum SliceMode { kSliceOne = 0, kSliceList = 1, kSliceFallback = 2 };

template <typename real>
__global__ void __launch_bounds__(kSliceBlock, 4) k_slice_pairs(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    const double* __restrict__ x, SliceParams sp, int sbins, SliceList L, int mode)
{
    pdl_wait();
    pdl_launch();
    if (mode == kSliceFallback && *(volatile unsigned*)(L.count + 1) == 0u) return;   // the list held every pair
    const bool to_list = mode == kSliceList;
    typedef typename Vec4<real>::type V4;
    extern __shared__ __align__(16) unsigned char slice_dyn[];
    const int nt = K->ntypes, KT = nt * nt;
    const int nbins = sp.S * KT * 9;
    real* sbin = reinterpret_cast<real*>(slice_dyn);
    uint32_t* lists = reinterpret_cast<uint32_t*>(slice_dyn + (sbins ? slice_bin_bytes<real>(sp.S, KT) : 0));
    uint32_t* list = lists + threadIdx.x;
    if (sbins) {
        for (int k = threadIdx.x; k < nbins; k += blockDim.x) sbin[k] = real(0);
        __syncthreads();
    }
    const Box& B = boxes[0];
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
    uint32_t keys[10];
    {
        uint32_t k = philox_step_key(B.seed, *step_ptr);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
    }
    // Lane l of a warp takes its beads from the l-th 32nd of the slot range
    // (slots are cell-sorted, z-major): the 32 lanes sit at 32 different
    // heights and rarely add into the same slice bins at the same time, where
    // the beads of one cell row would all meet on a few (shared-memory float
    // atomics retry on every collision).  Listing only, a warp takes 32
    // consecutive slots, whose neighbour cells it shares.
    const int lane = threadIdx.x & 31;
    const int P = (n + 31) / 32;
    const int nwarps = gridDim.x * (kSliceBlock / 32);
    if (to_list) {   // list mode: the force kernels' row windows, one tile of consecutive slots per warp
        for (int v = blockIdx.x * (kSliceBlock / 32) + (threadIdx.x >> 5); v < P; v += nwarps)
            slice_list_tile<real>(v * 32 + lane, n, B, cell, start, pos4, list, L);
        return;
    }
    for (int v = blockIdx.x * (kSliceBlock / 32) + (threadIdx.x >> 5); v < P; v += nwarps) {
        const int i = lane * P + v;
        const bool live = i < n;
        V4 pi, vi;
        int cx = 0, cy = 0, cz = 0;
        double zi = 0.0;
        if (live) {
            pi = pos4[i];
            vi = vel4[i];
            const int c = cell[i] - B.cell_base;
            int cc[3];
            cell_coords(B, c, cc);
            cx = cc[0];
            cy = cc[1];
            cz = cc[2];
            zi = x[2 * (size_t)n + i];
        } else {
            pi.x = pi.y = pi.z = pi.w = vi.x = vi.y = vi.z = vi.w = real(0);
        }
        int cnt = 0;
        // o = 0: own cell after i; o = 1..13: (dx, dy, dz) of the reference's half
        // shell (CSimBox::MakeCNTCells, SimBox.cpp:845-856)
        for (int o = 0; o < 14; ++o) {
            int ox = 0, oy = 0, oz = 0;
            if (o >= 1 && o <= 9) { ox = (o - 1) % 3 - 1; oy = (o - 1) / 3 - 1; oz = 1; }
            else if (o >= 10 && o <= 12) { ox = 1; oy = o - 11; oz = 0; }
            else if (o == 13) { ox = 0; oy = 1; oz = 0; }
            int x2 = cx + ox, y2 = cy + oy, z2 = cz + oz;
            x2 += x2 < 0 ? nx : (x2 >= nx ? -nx : 0);
            y2 += y2 < 0 ? ny : (y2 >= ny ? -ny : 0);
            z2 += z2 >= nz ? -nz : 0;
            const int c2 = B.cell_base + x2 + nx * (y2 + ny * z2);
            int jb = 0, je = 0;
            if (live) {
                jb = o == 0 ? i + 1 : start[c2];
                je = start[c2 + 1];
            }
            const int len = max(je - jb, 0);
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            const real pxs = pi.x - (real)ox * wx, pys = pi.y - (real)oy * wy, pzs = pi.z - (real)oz * wz;
            const uint32_t code = ((uint32_t)(ox + 1) << 26) | ((uint32_t)(oy + 1) << 28) | ((uint32_t)(oz + 1) << 30);
            for (int base = 0; base < trip; base += kSliceHits) {
                const int clen = min(max(len - base, 0), kSliceHits);
                if (__any_sync(0xffffffffu, cnt + clen > kSliceHits)) {
                    if (sbins)
                        slice_eval<real>(cnt, list, i, n, pi, vi, zi, tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp,
                                         sbin, B.L);
                    else
                        slice_eval<real>(cnt, list, i, n, pi, vi, zi, tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp,
                                         sp.pair, B.L);
                    cnt = 0;
                }
                const int tend = base + min(trip - base, kSliceHits);
                // four candidates per iteration (loads in flight together),
                // then the last 1-3 singly; the entry is stored always and
                // kept by advancing cnt (cnt + clen <= kSliceHits: at most the
                // spare row)
                const int tend4 = base + ((tend - base) & ~3);
                int t = base;
                for (; t < tend4; t += 4) {
                    V4 p[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) p[q] = pos4[min(jb + t + q, n - 1)];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const real dx = pxs - p[q].x, dy = pys - p[q].y, dz = pzs - p[q].z;
                        const real r2 = dx * dx + dy * dy + dz * dz;
                        list[cnt * kSliceBlock] = (uint32_t)min(jb + t + q, n - 1) | code;
                        cnt += (t + q < len && r2 < real(1) && r2 > real(1e-18)) ? 1 : 0;
                    }
                }
                for (; t < tend; ++t) {
                    const int j = min(jb + t, n - 1);
                    const V4 pj = pos4[j];
                    const real dx = pxs - pj.x, dy = pys - pj.y, dz = pzs - pj.z;
                    const real r2 = dx * dx + dy * dy + dz * dz;
                    list[cnt * kSliceBlock] = (uint32_t)j | code;
                    cnt += (t < len && r2 < real(1) && r2 > real(1e-18)) ? 1 : 0;
                }
            }
        }
        if (sbins)
            slice_eval<real>(cnt, list, i, n, pi, vi, zi, tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp, sbin, B.L);
        else
            slice_eval<real>(cnt, list, i, n, pi, vi, zi, tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp, sp.pair, B.L);
    }
    if (sbins) {
        __syncthreads();
        for (int k = threadIdx.x; k < nbins; k += blockDim.x)
            if (sbin[k] != real(0)) atomicAdd(sp.pair + k, (double)sbin[k]);
    }
}

// The listed pairs of the profile, one pair per lane: lane l of a warp takes
// the entries of the l-th 32nd of the list, so a warp's lanes hold pairs from
// unrelated parts of the box and rarely add into the same bins at once.
// Bins block-private in shared memory when they fit, added once per block to
// the FP64 profile.  Does nothing when the list overflowed (the fallback
// builds the profile then).
constexpr int kSliceEvalBlock = 256;
constexpr int kSliceEvalBlocksPerSM = 4;   // one wave at 64 registers

template <typename real>
__host__ __device__ constexpr size_t slice_eval_smem_bytes(int S, int KT, bool sbins)
{
    return sbins ? slice_bin_bytes<real>(S, KT) : 0;
}

// One lane's running sum for one bin (slice * KT + type pair) of the pair
// part: the 6 distinct products of the symmetric pair tensor (the force is
// parallel to the separation: (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)), added to
// the bins when the lane moves to another bin.
struct SliceRun {
    int key;
    double v[6];
};
template <typename bin_t>
__device__ __forceinline__ void slice_run_flush(SliceRun& a, bin_t* bins)
{
    if (a.key >= 0) {
        bin_t* q = bins + (size_t)a.key * 9;
        atomicAdd(q + 0, (bin_t)a.v[0]);
        atomicAdd(q + 1, (bin_t)a.v[1]);
        atomicAdd(q + 2, (bin_t)a.v[2]);
        atomicAdd(q + 4, (bin_t)a.v[3]);
        atomicAdd(q + 5, (bin_t)a.v[4]);
        atomicAdd(q + 8, (bin_t)a.v[5]);
    }
}
template <typename bin_t>
__device__ __forceinline__ void slice_run_add(SliceRun& a, bin_t* bins, int key, const double fdx[9], double fac)
{
    if (key != a.key) {
        slice_run_flush(a, bins);
        a.key = key;
#pragma unroll
        for (int c = 0; c < 6; ++c) a.v[c] = 0.0;
    }
    a.v[0] += fdx[0] * fac;
    a.v[1] += fdx[1] * fac;
    a.v[2] += fdx[2] * fac;
    a.v[3] += fdx[4] * fac;
    a.v[4] += fdx[5] * fac;
    a.v[5] += fdx[8] * fac;
}

// The listed pairs of the profile, one pair per lane: lane l of a warp takes
// entries from the l-th 32nd of the list, so a warp's lanes hold pairs from
// unrelated parts of the box and rarely add into the same bins at once, and
// walks consecutive entries (the pairs of one bead 1 in a row), whose
// products mostly fall in the bin of the previous pair and are summed in
// registers first (SliceRun).  The upper triangle of each bin is added
// (k_slice_sum mirrors it).  Bins block-private in shared memory when they
// fit, written once per block to its row of the partial sums.  Does nothing
// when the list overflowed (the fallback builds the profile then).
template <typename real>
__global__ void __launch_bounds__(kSliceEvalBlock, 4) k_slice_eval(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const typename Vec4<real>::type* __restrict__ pos4,
    const typename Vec4<real>::type* __restrict__ vel4, const double* __restrict__ x, SliceParams sp, int sbins,
    SliceList L, real* __restrict__ partial)
{
    pdl_wait();
    pdl_launch();
    typedef typename Vec4<real>::type V4;
    if (*(volatile unsigned*)(L.count + 1) != 0u) return;   // overflowed: the fallback builds the profile
    extern __shared__ __align__(16) unsigned char slice_dyn[];
    const int nt = K->ntypes, KT = nt * nt;
    const int nbins = sp.S * KT * 9;
    real* sbin = reinterpret_cast<real*>(slice_dyn);
    if (sbins) {
        for (int k = threadIdx.x; k < nbins; k += blockDim.x) sbin[k] = real(0);
        __syncthreads();
    }
    const Box& B = boxes[0];
    const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
    uint32_t keys[10];
    {
        uint32_t k = philox_step_key(B.seed, *step_ptr);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
    }
    const int total = (int)min(*(volatile unsigned*)L.count, (unsigned)L.cap);
    const int lane = threadIdx.x & 31;
    const int P = (total + 31) / 32;                              // entries a lane column holds
    const int nwarps = gridDim.x * (kSliceEvalBlock / 32);
    const int Q = (P + nwarps - 1) / nwarps;                      // consecutive entries a warp walks
    const int w = blockIdx.x * (kSliceEvalBlock / 32) + (threadIdx.x >> 5);
    SliceRun run;
    run.key = -1;
    for (int v = w * Q; v < min((w + 1) * Q, P); ++v) {
        const int k = lane * P + v;
        double fdx[9];
        SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
        int tt = 0;
        if (k < total) {
            const uint2 pe = L.pairs[k];
            const int i = (int)pe.x;
            const V4 pi = pos4[i];
            const V4 vi = vel4[i];
            slice_pair<real>(pe.y, i, n, pi, vi, x[2 * (size_t)n + i], tab, nt, keys, wx, wy, wz, pos4, vel4, x, sp,
                             B.L, fdx, s, tt);
        }
        // the span's slices in a warp-uniform loop, so the lanes that move to
        // another bin at the same step add their runs together
        const int ms = span_count(s);
        const int mt = (int)__reduce_max_sync(0xffffffffu, (unsigned)ms);
        for (int t = 0; t < mt; ++t) {
            int sl = 0;
            double fac = 0.0;
            if (t < ms) span_entry(s, sp.S, t, sl, fac);
            if (t < ms) {
                if (sbins) slice_run_add(run, sbin, sl * KT + tt, fdx, fac);
                else slice_run_add(run, sp.pair, sl * KT + tt, fdx, fac);
            }
        }
    }
    if (sbins) slice_run_flush(run, sbin);
    else slice_run_flush(run, sp.pair);
    if (sbins) {   // this block's bins to its row of the partial sums (k_slice_sum adds the rows)
        __syncthreads();
        real* row = partial + (size_t)blockIdx.x * nbins;
        for (int k = threadIdx.x; k < nbins; k += blockDim.x) row[k] = sbin[k];
    }
}

// The pair part of the profile from the partial-sum rows of k_slice_eval:
// each block adds 32 consecutive bins over all rows (8 groups of rows, then
// the groups in a fixed order) and mirrors the upper triangle of every 3x3
// bin, which is all k_slice_eval adds.  Nothing when the list overflowed.
// With bins straight in global memory (no rows), only the mirror.
template <typename real>
__global__ void __launch_bounds__(256) k_slice_sum(int nbins, int nrows, const real* __restrict__ partial,
                                                   const unsigned* __restrict__ count, double* __restrict__ pair)
{
    pdl_wait();
    pdl_launch();
    if (*(volatile const unsigned*)(count + 1) != 0u) return;
    __shared__ double part[8][33];
    const int b = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int k0 = blockIdx.x * 32;
    const int k = k0 + b;
    double a = 0.0;
    if (nrows > 0 && k < nbins) {
        int r = g;
        for (; r + 24 < nrows; r += 32) {   // four rows of this group in flight
            const real p0 = partial[(size_t)r * nbins + k], p1 = partial[(size_t)(r + 8) * nbins + k];
            const real p2 = partial[(size_t)(r + 16) * nbins + k], p3 = partial[(size_t)(r + 24) * nbins + k];
            a += (double)p0;
            a += (double)p1;
            a += (double)p2;
            a += (double)p3;
        }
        for (; r < nrows; r += 8) a += (double)partial[(size_t)r * nbins + k];
    }
    part[g][b] = a;
    __syncthreads();
    if (g == 0 && k < nbins) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) t += part[q][b];
        part[0][b] = t + pair[k];   // the direct adds (bins not in shared memory) already hold theirs
    }
    __syncthreads();
    // mirror: component 3r+c below the diagonal takes 3c+r; blocks cover 32
    // bins, so a 3x3 group may straddle two blocks: the block holding an
    // upper entry writes it and its mirror, lower entries are written by no
    // one else (nothing was added to them)
    if (g == 0 && k < nbins) {
        const int c9 = k % 9, r = c9 / 3, c = c9 % 3;
        if (r <= c) pair[k] = part[0][b];
        if (r < c) pair[k - c9 + 3 * c + r] = part[0][b];
    }
}

}  // namespace dpd
