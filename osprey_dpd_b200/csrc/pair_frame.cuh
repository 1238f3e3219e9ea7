// pair_frame.cuh -- half-shell DPD pair forces (CCNTCell::UpdateForce, DPD
// branch, CNTCell.cpp:1103-1572) with the candidate test in the frame of the
// box's x axis, single box, FP32 forces.
//
// Same work layout as k_pair_forces_half (pair_forces.cuh): one lane per bead
// of a 128-slot tile walks its five half-shell neighbour rows, each a
// contiguous slot range (two where it wraps around the x boundary); hits go
// to the lane's list column in shared memory; the warp's hits are then cut
// into 32 equal runs for the force phase.  The difference is what the test
// reads.  The cell-relative shadows make the x separation depend on which of
// the row's three cells a candidate sits in (a compare and select per
// candidate, plus the matching entry code).  Here the test reads the "frame
// shadow" (K->tst4: FP32 absolute x, cell-relative y and z), so inside a row
// segment the x shift is one constant -- zero, or a box length for the
// segment across the periodic boundary -- and a candidate costs a load,
// three subtractions, the squared distance, one compare and the branch-free
// list store.  The frame shadow is padded past the last bead (kFramePad far
// away entries), so lanes past their window read in bounds without a
// per-candidate clamp.
//
// FP32 absolute x carries ~4e-6 rounding in a 64-cell box (~8e-6 at 128), so
// the test keeps r^2 < 1 + 1e-4; the force pass takes the x separation
// exactly from the FP64 positions (x_i - x_j minus the entry's image shift
// times L_x) and y, z from the cell-relative shadows, and applies the exact
// cut-off.  Entry: slot | (image shift + 1) << 26 | (dy + 1) << 28 |
// (dz + 1) << 30.  F (and on sample steps the stress array) must be zero on
// entry.
#pragma once
#include "pair_forces.cuh"

namespace dpd {

constexpr int kFramePad = kHitCapMax + 8;   // padding entries of the frame shadow past the last bead
constexpr float kFrameTestR2 = 1.0001f;

// Force phase of one warp (all 32 lanes), owner-major runs of equal length as
// balanced_force_pass, with the x separation from the FP64 positions.
template <bool VIRIAL>
__device__ __forceinline__ void frame_force_pass(int cnt, const uint32_t* __restrict__ lists,
                                                 const HalfShared<float>& sh, int tile_base, const Box& B,
                                                 const float* Tsh, int nt, const uint32_t* keys,
                                                 const float4* __restrict__ pos4, const float4* __restrict__ vel4,
                                                 const double* __restrict__ xs, float* __restrict__ F,
                                                 float* __restrict__ stress, int n)
{
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
        const float wy = (float)B.w[1], wz = (float)B.w[2];
        const double Lx = B.L[0];
        float4 pi, vi;
        double xi = 0.0;
        int islot, ti;
        uint32_t idi;
        auto load_owner = [&](int oo) {
            const int to = wbase + oo;
            pi = sh.hpos[to];
            vi = sh.hvel[to];
            islot = tile_base + to;
            xi = xs[islot];
            ti = (__float_as_int(pi.w) & 0xFF) * nt;
            idi = __float_as_uint(vi.w);
        };
        load_owner(o);
        constexpr int NACC = VIRIAL ? 12 : 3;
        float acc[NACC];
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q] = 0.f;
        for (; f < f1; ++f) {
            if (e == co) {
                atomicAdd(F + islot, acc[0]);
                atomicAdd(F + n + islot, acc[1]);
                atomicAdd(F + 2 * n + islot, acc[2]);
                if (VIRIAL) {
#pragma unroll
                    for (int q = 0; q < 9; ++q) atomicAdd(stress + (size_t)q * n + islot, acc[3 + q]);
                }
#pragma unroll
                for (int q = 0; q < NACC; ++q) acc[q] = 0.f;
                do { ++o; } while (o < 31 && wcnt[o] == 0);   // a later owner holds entry f, since f < tot
                e = 0;
                co = wcnt[o];
                load_owner(o);
            }
            const uint32_t ent = lists[e * kPairBlock + wbase + o];
            ++e;
            const int j = (int)(ent & 0x03FFFFFFu);
            const float4 pj = pos4[j];
            const float4 vj = vel4[j];
            const double xj = xs[j];
            float dx = (float)((xi - xj) - (double)((int)((ent >> 26) & 3u) - 1) * Lx);
            float dy = (pi.y - pj.y) - (float)((int)((ent >> 28) & 3u) - 1) * wy;
            float dz = (pi.z - pj.z) - (float)((int)(ent >> 30) - 1) * wz;
            float r2 = dx * dx + dy * dy + dz * dz;
            refine_close(dx, dy, dz, r2, xs, n, islot, j, B.L);
            const float inv = RealOps<float>::rsqrt(r2);
            const float wr = 1.f - r2 * inv;
            const int tt = ti + (__float_as_int(pj.w) & 0xFF);
            const float rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
            const uint32_t idj = __float_as_uint(vj.w);
            uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                const uint64_t prod = (uint64_t)0xD256D193u * c0;   // one wide multiply per round
                c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
                c1 = (uint32_t)prod;
            }
            const float mag = Tsh[tt] * wr - Tsh[m2 + tt] * wr * wr * rdotv +
                              Tsh[2 * m2 + tt] * wr * noise_centered(c0, 0.f);
            // the exact cut-off (the test's was widened) and no coincident beads
            const float m = (r2 < 1.f && r2 > 1e-18f) ? mag * inv : 0.f;
            const float gx = m * dx, gy = m * dy, gz = m * dz;
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
        atomicAdd(F + islot, acc[0]);
        atomicAdd(F + n + islot, acc[1]);
        atomicAdd(F + 2 * n + islot, acc[2]);
        if (VIRIAL) {
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(stress + (size_t)q * n + islot, acc[3 + q]);
        }
    }
    __syncwarp();   // every lane is done with the lists before they are refilled
}

template <bool VIRIAL>
__global__ void __launch_bounds__(kPairBlock, 8) k_pair_forces_frame(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const float* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const float4* __restrict__ pos4, const float4* __restrict__ vel4, float* __restrict__ F,
    float* __restrict__ stress, int hitcap, int tiles_per_block, unsigned* __restrict__ status,
    const double* __restrict__ xs)
{
    pdl_wait();
    pdl_launch();
    extern __shared__ __align__(16) unsigned char pair_dyn[];
    const int nt = K->ntypes;
    const float4* __restrict__ tst4 = K->tst4;
    float* Tsh = reinterpret_cast<float*>(pair_dyn);
    unsigned char* lbase = pair_dyn + pair_tables_bytes<float>(nt);
    uint32_t* lists = reinterpret_cast<uint32_t*>(lbase);
    const HalfShared<float> sh = half_shared<float>(lbase + sizeof(uint32_t) * (size_t)(hitcap + 1) * kPairBlock);
    for (int k = threadIdx.x; k < 3 * nt * nt; k += kPairBlock) Tsh[k] = tab[k];
    uint32_t keys[10];
    {
        uint32_t k = philox_step_key(boxes[0].seed, *step_ptr);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
    }
    __syncthreads();   // tables
    const int tile_base = blockIdx.x * kPairBlock;
    const int i = tile_base + threadIdx.x;
    const bool live = i < n;
    const Box& B = boxes[0];
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    const float wx = (float)B.w[0], wy = (float)B.w[1], wz = (float)B.w[2];
    const float Lxf = (float)B.L[0];
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vi = pi;
    float Xi = 0.f;
    int cx = 0, cy = 0, cz = 0;
    if (live) {
        pi = pos4[i];
        vi = vel4[i];
        Xi = tst4[i].x;
        const int c = cell[i];
        cx = c % nx;
        cy = (c / nx) % ny;
        cz = c / (nx * ny);
    }
    sh.hpos[threadIdx.x] = pi;
    sh.hvel[threadIdx.x] = vi;
    uint32_t* list = lists + threadIdx.x;
    int cnt = 0;
    // the periodic-boundary segment of a row only in warps with a bead in the
    // first or last cell column
    const int nseg = __any_sync(0xffffffffu, live && (cx == 0 || cx == nx - 1)) ? 2 : 1;
    __syncwarp();   // home shadows visible to the warp
    for (int r = 0; r < 5; ++r) {
        const int dy = r == 0 ? 0 : (r == 1 ? 1 : r - 3);
        const int dz = r < 2 ? 0 : 1;
        int y2 = cy + dy, z2 = cz + dz;
        y2 += (y2 >= ny) ? -ny : 0;
        z2 += (z2 >= nz) ? -nz : 0;
        y2 += (y2 < 0) ? ny : 0;
        const int rb = nx * (y2 + ny * z2);
        const float Yr = pi.y - (float)dy * wy, Zr = pi.z - (float)dz * wz;
        const uint32_t rowbits = ((uint32_t)(dy + 1) << 28) | ((uint32_t)(dz + 1) << 30);
        // cell pruning as in half_shell_tile: a row cell whose nearest point
        // lies at or beyond the cut-off holds no partner
        const float gy = dy > 0 ? wy - pi.y : (dy < 0 ? pi.y : 0.f);
        const float gz = dz > 0 ? wz - pi.z : 0.f;
        const float gyz = gy * gy + gz * gz;
        const float gxp = wx - pi.x;
        const bool keep_0 = gyz < kPruneR2;
        const bool keep_m = pi.x * pi.x + gyz < kPruneR2;
        const bool keep_p = gxp * gxp + gyz < kPruneR2;
        for (int seg = 0; seg < nseg; ++seg) {
            int lo, hi, b1, b2, img = 0;
            if (r > 0) {
                row_segment(live, seg, rb, cx, nx, start, lo, hi, b1, b2);
                img = seg == 0 ? 0 : (cx == 0 ? -1 : 1);
            } else if (!live) {
                lo = hi = b1 = b2 = 0;
            } else if (cx < nx - 1) {
                // own cell after i, then cell x+1 (offset +1 from b2)
                if (seg == 0) { lo = b1 = i + 1; b2 = start[rb + cx + 1]; hi = start[rb + cx + 2]; }
                else { lo = hi = b1 = b2 = 0; }
            } else {
                // cx = nx-1: own cell after i, then cell 0 across the boundary
                if (seg == 0) { lo = b1 = i + 1; b2 = hi = start[rb + cx + 1]; }
                else { lo = b1 = b2 = start[rb]; hi = start[rb + 1]; img = 1; }
            }
            // [lo, b1) is cell x-1, [b1, b2) cell x, [b2, hi) cell x+1
            lo = keep_m ? lo : b1;
            hi = keep_p ? hi : b2;
            hi = keep_0 ? hi : lo;
            const int len = max(hi - lo, 0);
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
            // candidate j's x separation in this segment: (Xi - img L) - X_j
            const float Xs = Xi - (float)img * Lxf;
            const uint32_t ebase = ((uint32_t)lo | ((uint32_t)(img + 1) << 26)) | rowbits;
            for (int base = 0; base < trip; base += hitcap) {
                const int clen = min(max(len - base, 0), hitcap);
                if (__any_sync(0xffffffffu, cnt + clen > hitcap)) {
                    frame_force_pass<VIRIAL>(cnt, lists, sh, tile_base, B, Tsh, nt, keys, pos4, vel4, xs, F, stress,
                                             n);
                    cnt = 0;
                }
                const int tend = base + min(trip - base, hitcap);
                const int lim = min(len, tend);
                // where this lane reads: its window while part of it lies in
                // this chunk (then at most hitcap - 1 entries past lo + len <=
                // n, inside the padding), else the shadow's start (t < trip <=
                // n); either way in bounds, and results past lim are masked
                const float4* __restrict__ src = lim > base ? tst4 + lo : tst4;
                // four candidates per iteration, without branches: a lane past
                // its window reads the next shadows (the padding past the last
                // bead keeps it in bounds) and its results are masked; the entry
                // is stored always and kept by advancing cnt (cnt + clen <=
                // hitcap: at most the spare row)
                int t = base;
                for (; t + 4 <= tend; t += 4) {
                    float4 q[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) q[u] = src[t + u];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const float ex = Xs - q[u].x, ey = Yr - q[u].y, ez = Zr - q[u].z;
                        const float r2 = ex * ex + ey * ey + ez * ez;
                        list[cnt * kPairBlock] = ebase + (uint32_t)(t + u);
                        cnt += (r2 < kFrameTestR2 && t + u < lim) ? 1 : 0;
                    }
                }
                for (; t < tend; ++t) {   // the last 1-3 candidates of the warp's longest window
                    const float4 q = src[t];
                    const float ex = Xs - q.x, ey = Yr - q.y, ez = Zr - q.z;
                    const float r2 = ex * ex + ey * ey + ez * ez;
                    list[cnt * kPairBlock] = ebase + (uint32_t)t;
                    cnt += (r2 < kFrameTestR2 && t < lim) ? 1 : 0;
                }
            }
        }
    }
    frame_force_pass<VIRIAL>(cnt, lists, sh, tile_base, B, Tsh, nt, keys, pos4, vel4, xs, F, stress, n);
}

}  // namespace dpd
