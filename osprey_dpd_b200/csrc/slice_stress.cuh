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

// The listed pairs of the warp's lanes, one pair per lane per iteration (the
// loop runs to the longest list, so it is warp-uniform): the force, then the
// slices it spreads over, every lane's adds to one slice issued together
// (slice_span / span_entry).  Called by all 32 lanes.  bins: the block's shared bins (real) or the global FP64 profile.
template <typename real, typename bin_t>
__device__ __forceinline__ void slice_eval(int cnt, const uint32_t* __restrict__ list, int i, int n,
                                           const typename Vec4<real>::type& pi, const typename Vec4<real>::type& vi,
                                           double zi, const real* __restrict__ tab, int nt, const uint32_t* keys,
                                           real wx, real wy, real wz, const typename Vec4<real>::type* __restrict__ pos4,
                                           const typename Vec4<real>::type* __restrict__ vel4,
                                           const double* __restrict__ x, const SliceParams& sp, bin_t* bins,
                                           const double* L)
{
    typedef typename Vec4<real>::type V4;
    const int m2 = nt * nt, KT = nt * nt;
    const int ti = real_bits(pi.w) & 0xFF;
    const uint32_t idi = (uint32_t)real_bits(vi.w);
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    for (int k = 0; k < trip; ++k) {
        double fdx[9];
        SliceSpan s{0, 0, 0, 0, 0.0, 0.0, 0.0};
        int tt = 0;
        if (k < cnt) {
            const uint32_t e = list[k * kSliceBlock];
            const int j = (int)(e & 0x03FFFFFFu);
            const V4 pj = pos4[j];
            const V4 vj = vel4[j];
            real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
            real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
            real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
            const real r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < real(1) && r2 > real(1e-18)) {   // the test's rounding differs at the cut-off
                const real inv = RealOps<real>::rsqrt(r2);
                const real wr = real(1) - r2 * inv;
                const int tj = real_bits(pj.w) & 0xFF;
                tt = ti * nt + tj;
                const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
                const uint32_t idj = (uint32_t)real_bits(vj.w);
                uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
                for (int q = 0; q < 10; ++q) {
                    const uint64_t prod = (uint64_t)0xD256D193u * c0;
                    c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
                    c1 = (uint32_t)prod;
                }
                const real ta = tab[tt], tg = tab[m2 + tt], ts = tab[2 * m2 + tt],
                           noise = noise_centered(c0, real(0));
                real m = (ta * wr - tg * wr * wr * rdotv + ts * wr * noise) * inv;
                close_pair_fix(dx, dy, dz, m, r2, x, n, i, j, L, vi, vj, ta, tg, ts, noise);
                const double f[3] = {(double)(m * dx), (double)(m * dy), (double)(m * dz)};
                const double d[3] = {(double)dx, (double)dy, (double)dz};
                outer9(f, d, fdx);
                s = slice_span(sp, KT, tt, d[2], zi, x[2 * (size_t)n + j]);
            }
        }
        const int ms = span_count(s);
        const int mt = (int)__reduce_max_sync(0xffffffffu, (unsigned)ms);
        for (int t = 0; t < mt; ++t) {
            if (t < ms) {
                int sl;
                double fac;
                span_entry(s, sp.S, t, sl, fac);
                bin_t* q = bins + ((size_t)sl * KT + tt) * 9;
#pragma unroll
                for (int c = 0; c < 9; ++c) atomicAdd(q + c, (bin_t)(fdx[c] * fac));
            }
        }
    }
}

template <typename real>
__global__ void __launch_bounds__(kSliceBlock, 4) k_slice_pairs(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    const double* __restrict__ x, SliceParams sp, int sbins)
{
    pdl_wait();
    pdl_launch();
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
    // atomics retry on every collision).
    const int lane = threadIdx.x & 31;
    const int P = (n + 31) / 32;
    const int nwarps = gridDim.x * (kSliceBlock / 32);
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
                for (int t = base; t < tend; ++t) {
                    // the entry is stored always and kept by advancing cnt
                    // (cnt + clen <= kSliceHits: at most the spare row)
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

}  // namespace dpd
