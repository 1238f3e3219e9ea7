// pair_forces.cuh -- the engine's DPD pair-force kernels (CCNTCell::UpdateForce,
// DPD branch, CNTCell.cpp:1103-1572) with per-lane hit lists.
//
// Only ~15% of the candidates in the neighbour cells lie inside the cut-off
// (rho = 3: 81 candidates in the full shell, 12.6 partners per bead), so
// evaluating the force where the distance test passes would run the expensive
// body (sqrt, Philox, ~80 instructions) with a few lanes active on almost
// every iteration.  The kernels therefore split the work in two phases:
//
//   test   : every lane owns one bead i (a slot in cell order) and walks its
//            neighbour rows; a row (cells x-1, x, x+1 at fixed y', z') is one
//            contiguous slot range in the cell-sorted layout, split in two
//            only where it wraps around the x boundary.  Passing candidates
//            are appended to the lane's own list column in shared memory.
//   force  : the listed pairs are evaluated.  Full shell (k_pair_forces):
//            every lane walks its own list, every pair is evaluated from both
//            sides, so bead i only accumulates its own force -- no atomics,
//            and the result depends only on the deterministic cell-sorted
//            order.  Half shell (k_pair_forces_half): every pair once, the
//            warp's lists are cut into 32 equal runs so all lanes evaluate
//            the same number of pairs, and forces are added with atomics.
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

constexpr int kPairWarps = 4;
constexpr int kPairBlock = 32 * kPairWarps;   // full-shell and staged tiles
// Half-shell tiles: two warps by default (dpd_engine_set_pair_tile selects
// 64 or 128 beads per block at run time).  Measured on the B200 against four
// and eight warps (same registers per SM): the mixed-precision kernel 2-3 %
// faster (bilayer 77.1 vs 79.2 us, melt 886 vs 901 us), FP64 even; one warp
// slower.
constexpr int kHalfBlock = 64;
// Resident blocks per SM the pair kernels are compiled for: 8 (64 registers,
// 32 warps) in FP32; the FP64 variants keep 6 to limit spills.
template <typename real, bool MULTI = false> struct PairOcc {
    static constexpr int value = sizeof(real) == 8 ? 6 : 8;
};
// The same warps per SM for the half-shell kernel's tiles of BLOCK beads.
template <typename real, bool MULTI = false, int BLOCK = kHalfBlock> struct HalfOcc {
    static constexpr int value = PairOcc<real, MULTI>::value * kPairBlock / BLOCK;
};
constexpr int kHitCapMax = 64;           // upper bound of the run-time hit-list capacity
// Cell pruning threshold on the squared distance to a cell's nearest point:
// the cut-off (1) plus a margin far above the FP32 rounding of r2.
constexpr float kPruneR2 = 1.0f + 1e-5f;

template <typename real> struct RealOps;
template <> struct RealOps<float> {
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float rnd(float x) { return rintf(x); }
};
template <> struct RealOps<double> {
    static __device__ __forceinline__ double rsqrt(double x) { return 1.0 / sqrt(x); }
    static __device__ __forceinline__ double rnd(double x) { return rint(x); }
};

// Pairs closer than 0.1 take their separation from the FP64 positions
// (slot order, three planes of n; minimum image in a box of lengths L): the
// FP32 cell-relative shadows carry ~6e-8 absolute error, which for beads a
// few 1e-3 apart (random initial states of millions of beads) turns the pair
// direction by ~1e-5.  Rare, so the branch costs little.  The pair is first
// evaluated as every other pair; close_pair_fix then replaces its separation
// and force scalar m (a, g, s: a_ij, gamma_ij, sigma_ij; noise: 0.5 - U), and
// the callers accumulate m * separation with explicit round-to-nearest
// operations, so the arithmetic of ordinary pairs does not depend on the
// presence of this branch (a replica batch and a single box round alike).
// FP64 shadows are exact already.
constexpr float kCloseR2 = 0.01f;
template <typename V4>
__device__ __forceinline__ void close_pair_fix(double&, double&, double&, double&, double, const double*, int, int, int,
                                               const double*, const V4&, const V4&, double, double, double, double)
{
}
template <typename V4>
__device__ __forceinline__ void close_pair_fix(float& dx, float& dy, float& dz, float& m, float r2,
                                               const double* __restrict__ xs, int n, int i, int j, const double* L,
                                               const V4& vi, const V4& vj, float a, float g, float s, float noise)
{
    if (r2 < kCloseR2 && xs) {
        float d[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            double e = xs[(size_t)q * n + i] - xs[(size_t)q * n + j];
            e = e > 0.5 * L[q] ? e - L[q] : (e < -0.5 * L[q] ? e + L[q] : e);
            d[q] = (float)e;
        }
        dx = d[0]; dy = d[1]; dz = d[2];
        const float rr = dx * dx + dy * dy + dz * dz;
        const float inv = rsqrtf(rr);
        const float wr = 1.f - rr * inv;
        const float rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
        m = rr > 1e-18f ? (a * wr - g * wr * wr * rdotv + s * wr * noise) * inv : 0.f;
    }
}

// The pair's force m * (dx, dy, dz) added to acc (and the virial terms), with
// explicit roundings (see close_pair_fix); returns the force in g.
template <typename real, bool VIRIAL>
__device__ __forceinline__ void pair_accumulate(real m, real dx, real dy, real dz, real* acc, real g[3])
{
    g[0] = m * dx;
    g[1] = m * dy;
    g[2] = m * dz;
    if (sizeof(real) == 4) {
        g[0] = __fmul_rn((float)m, (float)dx);
        g[1] = __fmul_rn((float)m, (float)dy);
        g[2] = __fmul_rn((float)m, (float)dz);
        acc[0] = __fadd_rn((float)acc[0], (float)g[0]);
        acc[1] = __fadd_rn((float)acc[1], (float)g[1]);
        acc[2] = __fadd_rn((float)acc[2], (float)g[2]);
        if (VIRIAL) {
            const float d[3] = {(float)dx, (float)dy, (float)dz};
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    acc[3 + 3 * r + c] = __fadd_rn((float)acc[3 + 3 * r + c], __fmul_rn(d[c], (float)g[r]));
        }
    } else {
        acc[0] += g[0]; acc[1] += g[1]; acc[2] += g[2];
        if (VIRIAL) {
            acc[3] += dx * g[0]; acc[4] += dy * g[0]; acc[5] += dz * g[0];
            acc[6] += dx * g[1]; acc[7] += dy * g[1]; acc[8] += dz * g[1];
            acc[9] += dx * g[2]; acc[10] += dy * g[2]; acc[11] += dz * g[2];
        }
    }
}

// Dynamic shared memory of one block: pair tables, then the hit lists
// (entry k of thread t at lists[k * kPairBlock + t], so a warp's stores and
// loads of one k hit 32 consecutive words).
template <typename real>
__host__ __device__ constexpr size_t pair_tables_bytes(int nt)
{
    return ((3 * sizeof(real) * (size_t)nt * nt + 15) / 16) * 16;
}
template <typename real, int BLOCK = kPairBlock>
__host__ __device__ constexpr size_t pair_smem_bytes(int nt, int hitcap, bool multi)
{
    return (multi ? 0 : pair_tables_bytes<real>(nt)) + sizeof(uint32_t) * hitcap * BLOCK;
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
                                                const typename Vec4<real>::type* __restrict__ vel4, real* acc,
                                                const double* __restrict__ xs, int n, int i, const double* L)
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
            real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
            real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
            real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
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
            const real ta = T[tt], tg = T[m2 + tt], ts = T[2 * m2 + tt], noise = noise_centered(c0, real(0));
            real m = (ta * wr - tg * wr * wr * rdotv + ts * wr * noise) * inv;
            close_pair_fix(dx, dy, dz, m, r2, xs, n, i, j, L, vi, vj, ta, tg, ts, noise);
            real g[3];
            pair_accumulate<real, VIRIAL>(m, dx, dy, dz, acc, g);
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
__global__ void __launch_bounds__(kPairBlock, PairOcc<real, MULTI>::value) k_pair_forces(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, int tiles_per_block,
    unsigned* __restrict__ status, const double* __restrict__ xs)
{
    pdl_wait();
    pdl_launch();
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
        int cc[3];
        cell_coords(B, c, cc);
        cx = cc[0];
        cy = cc[1];
        cz = cc[2];
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
                    pair_force_pass<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc, xs, n,
                                                  i, B.L);
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
    pair_force_pass<real, VIRIAL>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc, xs, n, i, B.L);
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

// Per-warp scratch of the balanced force pass in shared memory: the home
// beads' shadows (read by whichever lane evaluates their pairs) and the hit
// counts with their exclusive prefix.
template <typename real>
struct HalfShared {
    typename Vec4<real>::type* hpos;   // one entry per thread of the block
    typename Vec4<real>::type* hvel;   // one entry per thread
    real* hxw;                         // one entry per thread (staged scheme only)
    int* wcnt;                         // hits of each thread
    int* wexc;                         // exclusive prefix of the hits inside the warp
};

// Hit-list entry formats of the two half-shell kernels.
// Unstaged: candidate slot in bits 0..25, cell offsets + 1 (x, y, z) in 2-bit
// fields at bits 26, 28, 30.  Staged: staged index in bits 0..11, window
// (row offset, see stg_row_shift) in bits 12..14.
__device__ __forceinline__ void stg_row_shift(int r, int& dy, int& dz)
{
    dy = r == 0 ? 0 : (r == 1 ? 1 : r - 3);
    dz = r >= 2 ? 1 : 0;
}

// Force phase of one warp for the half-shell schemes, called by all 32 lanes
// with cnt = this lane's listed hits.  The warp's lists are read as one
// owner-major sequence (lane 0's hits, then lane 1's, ...) cut into 32 equal
// runs, one per lane, so every lane evaluates the same number of pairs
// whatever the per-bead hit counts.  A lane keeps the partial force of its
// current owner in registers and adds it to the owner's global force with
// atomics when the owner changes (or the run ends); the partner's share is
// added with atomics.  The pair force is CNTCell.cpp:1192-1220 with rc = 1:
//   w = 1 - r; F = (a_ij w - gamma_ij w^2 (r.v)/r + sigma_ij w (0.5 - U)) r_vec / r
// w0 holds the cell widths of a single-box engine; a replica batch (MULTI)
// reloads widths, tables and noise key per owner.  F (and on sample steps
// stress) must be zero before the kernel.
template <typename real, bool VIRIAL, bool MULTI, bool STAGED, int BLOCK = kPairBlock>
__device__ __forceinline__ void balanced_force_pass(
    int cnt, const uint32_t* __restrict__ lists, const HalfShared<real>& sh,
    const typename Vec4<real>::type* stg, int tile_base, const Box* __restrict__ boxes, const real* Tsh,
    const real* __restrict__ tab, int nt, const uint32_t* keys0, const real* w0, int64_t step,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int n, const double* __restrict__ xs)
{
    typedef typename Vec4<real>::type V4;
    const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
    const int tot = (int)__reduce_add_sync(0xffffffffu, (unsigned)cnt);
    if (tot == 0) return;
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    int* wcnt = sh.wcnt + wbase;
    int* wexc = sh.wexc + wbase;
    wcnt[lane] = cnt;
    wexc[lane] = inc - cnt;
    __syncwarp();
    const int per = (tot + 31) >> 5;
    int f = lane * per;
    const int f1 = min(f + per, tot);
    if (f < f1) {
        // owner of entry f: the last lane whose exclusive offset is <= f
        int o = 0;
#pragma unroll
        for (int s = 16; s; s >>= 1)
            if (wexc[o + s] <= f) o += s;
        int e = f - wexc[o], co = wcnt[o];
        const int m2 = nt * nt;
        V4 pi, vi;
        real xwi = real(0), wx = w0[0], wy = w0[1], wz = w0[2], iw = STAGED ? real(1) / w0[0] : real(0);
        int islot, ti;
        uint32_t idi;
        const real* T = Tsh;
        uint32_t keys[10];
        if (!MULTI) {
#pragma unroll
            for (int q = 0; q < 10; ++q) keys[q] = keys0[q];
        }
        int cur_box = -1;
        const double* Lb = boxes[0].L;   // the owner's box lengths (MULTI: reloaded with the box)
        auto load_owner = [&](int oo) {
            const int to = wbase + oo;
            pi = sh.hpos[to];
            vi = sh.hvel[to];
            if (STAGED) xwi = sh.hxw[to];
            islot = tile_base + to;
            ti = (real_bits(pi.w) & 0xFF) * nt;
            idi = (uint32_t)real_bits(vi.w);
            // the owner's box (cell widths, pair tables, noise key), reloaded
            // only when it changes: a batch's boxes are contiguous in slot order
            if (MULTI && flag_box(real_bits(pi.w)) != cur_box) {
                cur_box = flag_box(real_bits(pi.w));
                const Box& B = boxes[cur_box];
                wx = (real)B.w[0]; wy = (real)B.w[1]; wz = (real)B.w[2];
                Lb = B.L;
                if (STAGED) iw = real(1) / wx;
                T = tab + B.tab;
                uint32_t k = philox_step_key(B.seed, step);
#pragma unroll
                for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
            }
        };
        load_owner(o);
        constexpr int NACC = VIRIAL ? 12 : 3;
        real acc[NACC];
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q] = real(0);
        for (; f < f1; ++f) {
            if (e == co) {
                atomicAdd(F + islot, acc[0]);
                atomicAdd(F + n + islot, acc[1]);
                atomicAdd(F + 2 * n + islot, acc[2]);
                if (VIRIAL) {
#pragma unroll
                    for (int q = 0; q < 9; ++q) atomicAdd(stress + q * n + islot, acc[3 + q]);
                }
#pragma unroll
                for (int q = 0; q < NACC; ++q) acc[q] = real(0);
                do { ++o; } while (o < 31 && wcnt[o] == 0);   // a later owner holds entry f, since f < tot
                e = 0;
                co = wcnt[o];
                load_owner(o);
            }
            const uint32_t ent = lists[e * BLOCK + wbase + o];
            ++e;
            int j;
            real dx, dy, dz;
            V4 pj;
            if (STAGED) {
                const V4 sj = stg[ent & 0xFFFu];
                int dyi, dzi;
                stg_row_shift((int)(ent >> 12), dyi, dzi);
                j = real_bits(sj.w);
                pj = pos4[j];
                const real bx = pi.x - pj.x;
                const real ox = RealOps<real>::rnd((bx - (xwi - sj.x)) * iw);   // cell x offset of j
                dx = bx - ox * wx;
                dy = (pi.y - pj.y) - (real)dyi * wy;
                dz = (pi.z - pj.z) - (real)dzi * wz;
            } else {
                j = (int)(ent & 0x03FFFFFFu);
                pj = pos4[j];
                dx = (pi.x - pj.x) - (real)((int)((ent >> 26) & 3u) - 1) * wx;
                dy = (pi.y - pj.y) - (real)((int)((ent >> 28) & 3u) - 1) * wy;
                dz = (pi.z - pj.z) - (real)((int)(ent >> 30) - 1) * wz;
            }
            const V4 vj = vel4[j];
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
            const real ta = T[tt], tg = T[m2 + tt], ts = T[2 * m2 + tt], noise = noise_centered(c0, real(0));
            // the staged test decides pairs at the cut-off from rounded window
            // coordinates: the exact cut-off is applied here, and coincident
            // beads (r2 <= 1e-18) are left to this pass
            real m = (r2 < real(1) && r2 > real(1e-18)) ? (ta * wr - tg * wr * wr * rdotv + ts * wr * noise) * inv
                                                          : real(0);
            close_pair_fix(dx, dy, dz, m, r2, xs, n, islot, j, Lb, vi, vj, ta, tg, ts, noise);
            real g[3];
            pair_accumulate<real, VIRIAL>(m, dx, dy, dz, acc, g);
            atomicAdd(F + j, -g[0]);
            atomicAdd(F + n + j, -g[1]);
            atomicAdd(F + 2 * n + j, -g[2]);
        }
        atomicAdd(F + islot, acc[0]);
        atomicAdd(F + n + islot, acc[1]);
        atomicAdd(F + 2 * n + islot, acc[2]);
        if (VIRIAL) {
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(stress + q * n + islot, acc[3 + q]);
        }
    }
    __syncwarp();   // every lane is done with the lists before they are refilled
}

// This lane's listed pairs, each evaluated once: the force goes to the lane's
// own accumulator and, negated, to the partner through atomics.
template <typename real, bool VIRIAL, int BLOCK>
__device__ __forceinline__ void pair_force_pass_half(int cnt, const uint32_t* __restrict__ list,
                                                     const typename Vec4<real>::type& pi,
                                                     const typename Vec4<real>::type& vi, const real* __restrict__ T,
                                                     int nt, real wx, real wy, real wz, const uint32_t* keys,
                                                     const typename Vec4<real>::type* __restrict__ pos4,
                                                     const typename Vec4<real>::type* __restrict__ vel4, real* acc,
                                                     real* __restrict__ F, int n, const double* __restrict__ xs,
                                                     int i, const double* L)
{
    typedef typename Vec4<real>::type V4;
    const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
    const int ti = (real_bits(pi.w) & 0xFF) * nt;
    const uint32_t idi = (uint32_t)real_bits(vi.w);
    const int m2 = nt * nt;
    for (int k = 0; k < trip; ++k) {
        if (k < cnt) {
            const uint32_t e = list[k * BLOCK];
            const int j = (int)(e & 0x03FFFFFFu);
            const V4 pj = pos4[j];
            const V4 vj = vel4[j];
            real dx = (pi.x - pj.x) - (real)((int)((e >> 26) & 3u) - 1) * wx;
            real dy = (pi.y - pj.y) - (real)((int)((e >> 28) & 3u) - 1) * wy;
            real dz = (pi.z - pj.z) - (real)((int)(e >> 30) - 1) * wz;
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
            const real ta = T[tt], tg = T[m2 + tt], ts = T[2 * m2 + tt], noise = noise_centered(c0, real(0));
            real m = (ta * wr - tg * wr * wr * rdotv + ts * wr * noise) * inv;
            close_pair_fix(dx, dy, dz, m, r2, xs, n, i, j, L, vi, vj, ta, tg, ts, noise);
            real g[3];
            pair_accumulate<real, VIRIAL>(m, dx, dy, dz, acc, g);
            atomicAdd(F + j, -g[0]);
            atomicAdd(F + n + j, -g[1]);
            atomicAdd(F + 2 * n + j, -g[2]);
        }
    }
}

// The same tile with the per-lane force pass of the previous kernel
// generation: every lane evaluates its own hits (the warp runs as long as
// its busiest lane) and keeps bead i's force in registers.  Measured faster
// than the balanced pass for the FP64 and replica-batch variants, whose
// register budgets the balanced pass exceeds.
template <typename real, bool VIRIAL, bool MULTI, int BLOCK>
__device__ __forceinline__ void half_shell_tile_lanes(
    int tile, int n, int nt, const Box* __restrict__ boxes, int64_t step, const real* __restrict__ tab,
    const real* Tsh, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, uint32_t* lists, const double* __restrict__ xs)
{
    typedef typename Vec4<real>::type V4;
    uint32_t* list = lists + threadIdx.x;
    {
        const int i = tile * BLOCK + threadIdx.x;
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
            int cc[3];
            cell_coords(B, c, cc);
            cx = cc[0];
            cy = cc[1];
            cz = cc[2];
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
        // the periodic-boundary segment of a row only for warps with a bead in
        // the first or last cell column (as in half_shell_tile)
        const int nseg = __any_sync(0xffffffffu, live && (cx == 0 || cx == nx - 1)) ? 2 : 1;
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
            const uint32_t code_m = rowbits, code_0 = rowbits | (1u << 26), code_p = rowbits | (2u << 26);
            // cell pruning as in half_shell_tile
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
                    // own cell after i, then cell x+1 (offset +1 from b2)
                    if (seg == 0) { lo = b1 = i + 1; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2]; }
                    else { lo = hi = b1 = b2 = 0; }
                } else {
                    // cx = nx-1: own cell after i, then cell 0 across the boundary
                    if (seg == 0) { lo = b1 = i + 1; b2 = hi = start[rb + cx + 1]; }
                    else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; }
                }
                lo = keep_m ? lo : b1;
                hi = keep_p ? hi : b2;
                hi = keep_0 ? hi : lo;
                const int len = max(hi - lo, 0);
                const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
                for (int base = 0; base < trip; base += hitcap) {
                    const int clen = min(max(len - base, 0), hitcap);
                    if (__any_sync(0xffffffffu, cnt + clen > hitcap)) {
                        pair_force_pass_half<real, VIRIAL, BLOCK>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4,
                                                           acc, F, n, xs, i, B.L);
                        cnt = 0;
                    }
                    const int tend = base + min(trip - base, hitcap);
                    const int lim = min(len, tend);
                    // two candidates per iteration, then the last one singly,
                    // without branches (clamped loads, masked results, the
                    // entry stored at the list's count, which stays within the
                    // spare row: cnt + clen <= hitcap)
                    const int tend2 = base + ((tend - base) & ~1);
                    int t = base;
                    for (; t < tend2; t += 2) {
                        const int j0 = lo + t, rem = lim - t;
                        V4 p[2];
#pragma unroll
                        for (int q = 0; q < 2; ++q) p[q] = pos4[min(j0 + q, n - 1)];
#pragma unroll
                        for (int q = 0; q < 2; ++q) {
                            const int jq = j0 + q;
                            const bool ge1 = jq >= b1, ge2 = jq >= b2;
                            const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - p[q].x;
                            const real ddy = piy - p[q].y, ddz = piz - p[q].z;
                            const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            list[cnt * BLOCK] = (uint32_t)jq | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                            cnt += (r2 < real(1) && r2 > real(1e-18) && q < rem) ? 1 : 0;
                        }
                    }
                    if (t < tend) {
                        const int jq = lo + t;
                        const V4 pq = pos4[min(jq, n - 1)];
                        const bool ge1 = jq >= b1, ge2 = jq >= b2;
                        const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - pq.x;
                        const real ddy = piy - pq.y, ddz = piz - pq.z;
                        const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        list[cnt * BLOCK] = (uint32_t)jq | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                        cnt += (r2 < real(1) && r2 > real(1e-18) && t < lim) ? 1 : 0;
                    }
                }
            }
        }
        pair_force_pass_half<real, VIRIAL, BLOCK>(cnt, list, pi, vi, T, nt, wx, wy, wz, keys, pos4, vel4, acc, F, n, xs, i,
                                           B.L);
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

// Dynamic shared memory of k_pair_forces_half: pair tables (single box), hit
// lists (hitcap rows plus the spare row of the branch-free test loop), then
// the balanced pass's per-thread scratch.
template <typename real, int BLOCK>
__host__ __device__ constexpr size_t half_scratch_bytes()
{
    return (2 * 4 * sizeof(real) + 2 * sizeof(int)) * (size_t)BLOCK;
}
template <typename real, int BLOCK>
__host__ __device__ constexpr size_t half_smem_bytes(int nt, int hitcap, bool multi)
{
    return pair_smem_bytes<real, BLOCK>(nt, hitcap + 1, multi) + half_scratch_bytes<real, BLOCK>();
}
template <typename real, int BLOCK>
__device__ __forceinline__ HalfShared<real> half_shared(unsigned char* base)
{
    typedef typename Vec4<real>::type V4;
    HalfShared<real> sh;
    sh.hpos = reinterpret_cast<V4*>(base);
    sh.hvel = sh.hpos + BLOCK;
    sh.hxw = nullptr;
    sh.wcnt = reinterpret_cast<int*>(sh.hvel + BLOCK);
    sh.wexc = sh.wcnt + BLOCK;
    return sh;
}

// Half-shell scheme: every pair once, over the beads after bead i in its own
// cell and 13 neighbour cells (dz = +1: all nine; dz = 0: the dy = +1 row;
// dz = dy = 0: the cell at dx = +1) -- one of the two symmetric halves of the
// 26 neighbours, as CCNTCell::UpdateForce visits each pair once through its
// m_aIntNNCells half shell (CNTCell.cpp:1103-1572).  In slot terms: own row
// [i+1, end of cell x+1), the (dy=+1, dz=0) row and the three dz=+1 rows.
// The partner's share is added with global atomics, so the FP32 summation
// order (and the last bits) vary from run to run.  The pair virial goes whole
// to bead i, the reference's convention (CNTCell.cpp:1283-1301).
// One tile of BLOCK slots; `lists` the block's hit lists (this thread's
// column at lists + threadIdx.x), Tsh the staged pair tables (single box), sh
// the balanced pass's scratch.  Called by every thread of the block for the
// same tile.
template <typename real, bool VIRIAL, bool MULTI, int BLOCK>
__device__ __forceinline__ void half_shell_tile(
    int tile, int n, int nt, const Box* __restrict__ boxes, int64_t step, const real* __restrict__ tab,
    const real* Tsh, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, uint32_t* lists, const HalfShared<real>& sh,
    const uint32_t* keys0, const double* __restrict__ xs)
{
    typedef typename Vec4<real>::type V4;
    uint32_t* list = lists + threadIdx.x;
    const int i = tile * BLOCK + threadIdx.x;
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
        int cc[3];
        cell_coords(B, c, cc);
        cx = cc[0];
        cy = cc[1];
        cz = cc[2];
    }
    sh.hpos[threadIdx.x] = pi;
    sh.hvel[threadIdx.x] = vi;
    const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
    const real w0[3] = {wx, wy, wz};   // the box of a single-box engine (MULTI reloads per owner)
    const real pxm = pi.x + wx, px0 = pi.x, pxp = pi.x - wx;
    const int tile_base = tile * BLOCK;
    int cnt = 0;
    // a row's second segment (the cell across the periodic x boundary) exists
    // only for beads in the first or last cell column: warps with none skip it
    const int nseg = __any_sync(0xffffffffu, live && (cx == 0 || cx == nx - 1)) ? 2 : 1;
    __syncwarp();   // home shadows visible to the warp
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
        const uint32_t code_m = rowbits, code_0 = rowbits | (1u << 26), code_p = rowbits | (2u << 26);
        // Cell pruning: the nearest point of a row cell lies g_yz away in y-z
        // (0 where the row spans the bead's own y or z) and, for the cells at
        // x-1 and x+1, a further pi.x or wx - pi.x in x.  A cell whose nearest
        // point is at or beyond the cut-off (with a margin far above the FP32
        // rounding of r2) holds no partner and is cut from the window.
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
                // own cell after i, then cell x+1 (offset +1 from b2)
                if (seg == 0) { lo = b1 = i + 1; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2]; }
                else { lo = hi = b1 = b2 = 0; }
            } else {
                // cx = nx-1: own cell after i, then cell 0 across the boundary
                if (seg == 0) { lo = b1 = i + 1; b2 = hi = start[rb + cx + 1]; }
                else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; }
            }
            // [lo, b1) is cell x-1, [b1, b2) cell x, [b2, hi) cell x+1
            lo = keep_m ? lo : b1;
            hi = keep_p ? hi : b2;
            hi = keep_0 ? hi : lo;
            const int len = max(hi - lo, 0);
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            // chunks of at most hitcap candidates, so a list can never overflow
            for (int base = 0; base < trip; base += hitcap) {
                const int clen = min(max(len - base, 0), hitcap);
                if (__any_sync(0xffffffffu, cnt + clen > hitcap)) {
                    balanced_force_pass<real, VIRIAL, MULTI, false, BLOCK>(cnt, lists, sh, nullptr, tile_base, boxes, Tsh,
                                                                    tab, nt, keys0, w0, step, pos4, vel4, F, stress,
                                                                    n, xs);
                    cnt = 0;
                }
                const int tend = base + min(trip - base, hitcap);
                const int lim = min(len, tend);
                // Four candidates per iteration (then the last 1-3 singly, so
                // no group runs past the warp's longest window), without
                // branches: every lane runs all four (a lane past the end of
                // its window loads a clamped slot and its result is masked),
                // so their loads are issued together and four L1/L2 round
                // trips overlap.  The entry is stored whether or not the candidate passes and kept
                // by advancing cnt: cnt + clen <= hitcap holds here, so the
                // store goes at most to the list's spare row (index hitcap).
                // The own-cell window starts after i; coincident beads (the
                // reference's dr > 1e-9 test, CNTCell.cpp:1202) are left to
                // the force pass.
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
                        list[cnt * BLOCK] = (uint32_t)jq | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                        cnt += (r2 < real(1) && q < rem) ? 1 : 0;
                    }
                }
                for (; t < tend; ++t) {   // the last 1-3 candidates of the warp's longest window
                    const int jq = lo + t;
                    const V4 pq = pos4[min(jq, n - 1)];
                    const bool ge1 = jq >= b1, ge2 = jq >= b2;
                    const real ddx = (ge2 ? pxp : (ge1 ? px0 : pxm)) - pq.x;
                    const real ddy = piy - pq.y, ddz = piz - pq.z;
                    const real r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    list[cnt * BLOCK] = (uint32_t)jq | (ge2 ? code_p : (ge1 ? code_0 : code_m));
                    cnt += (r2 < real(1) && t < lim) ? 1 : 0;
                }
            }
        }
    }
    balanced_force_pass<real, VIRIAL, MULTI, false, BLOCK>(cnt, lists, sh, nullptr, tile_base, boxes, Tsh, tab, nt, keys0,
                                                    w0, step, pos4, vel4, F, stress, n, xs);
}

// Which force pass a k_pair_forces_half instantiation uses: the balanced pass
// for one FP32 box, the per-lane pass for FP64 and replica batches (each the
// faster of the two on a B200).
template <typename real, bool MULTI>
constexpr bool kHalfBalanced = sizeof(real) == 4 && !MULTI;

// F must be zero on entry, and on sample steps (VIRIAL) the stress array too.
template <typename real, bool VIRIAL, bool MULTI, int BLOCK = kHalfBlock>
__global__ void __launch_bounds__(BLOCK, HalfOcc<real, MULTI, BLOCK>::value) k_pair_forces_half(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    real* __restrict__ F, real* __restrict__ stress, int hitcap, int tiles_per_block,
    unsigned* __restrict__ status, const double* __restrict__ xs)
{
    pdl_wait();
    pdl_launch();
    extern __shared__ __align__(16) unsigned char pair_dyn[];
    const int nt = K->ntypes;
    real* Tsh = reinterpret_cast<real*>(pair_dyn);
    unsigned char* lbase = pair_dyn + (MULTI ? 0 : pair_tables_bytes<real>(nt));
    uint32_t* lists = reinterpret_cast<uint32_t*>(lbase);
    const HalfShared<real> sh = half_shared<real, BLOCK>(lbase + sizeof(uint32_t) * (size_t)(hitcap + 1) * BLOCK);
    if (!MULTI)
        for (int k = threadIdx.x; k < 3 * nt * nt; k += BLOCK) Tsh[k] = tab[k];
    const int64_t step = *step_ptr;
    uint32_t keys0[10];
    {
        uint32_t k = philox_step_key(boxes[0].seed, step);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys0[q] = k; k += 0x9E3779B9u; }
    }
    __syncthreads();   // tables
    const int tile0 = blockIdx.x * tiles_per_block;
    for (int tile = tile0; tile < tile0 + tiles_per_block; ++tile) {
        if (tile * BLOCK >= n) break;
        if (kHalfBalanced<real, MULTI>)
            half_shell_tile<real, VIRIAL, MULTI, BLOCK>(tile, n, nt, boxes, step, tab, Tsh, cell, start, pos4, vel4, F,
                                                 stress, hitcap, lists, sh, keys0, xs);
        else
            half_shell_tile_lanes<real, VIRIAL, MULTI, BLOCK>(tile, n, nt, boxes, step, tab, Tsh, cell, start, pos4, vel4,
                                                       F, stress, hitcap, lists, xs);
    }
}

}  // namespace dpd
