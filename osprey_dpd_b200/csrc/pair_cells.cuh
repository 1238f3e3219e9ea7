// pair_cells.cuh -- half-shell DPD pair forces (CCNTCell::UpdateForce, DPD
// branch, CNTCell.cpp:1103-1572) with the lanes of a warp over the candidates
// of one home cell, single box, FP32 forces.
//
// The per-bead kernels give every lane one bead and walk its neighbour
// windows; a warp then runs as long as its busiest lane, and with ~3 beads a
// cell the windows of the 32 lanes differ enough that most lane slots idle.
// Here the roles are swapped.  A warp owns 32 consecutive slots (its "home"
// beads, grouped into runs of one CNT cell each).  For one home cell the
// candidates -- the beads of the 14 cells of the reference's half shell: the
// own cell, cell x+1, and cells x-1..x+1 of the rows (y+1, z), (y-1, z+1),
// (y, z+1), (y+1, z+1) -- are spread over the lanes, 32 at a time, already
// shifted into the home cell's frame; the home beads of the run are then
// broadcast one by one and every lane tests its candidate.  Each lane-test is
// a real candidate pair, so no lane waits on another's window.  Hits are
// compacted into the warp's list with a ballot (owner-major, since the home
// beads are taken in order).
//
// Force phase: the list is cut into 32 equal runs, one per lane; a lane keeps
// the partial force of its current owner in registers and adds it to the
// owner's global force when the owner changes; the partner's share is added
// with atomics.  F (and on sample steps the stress array) must be zero on
// entry.  No block barrier after the pair tables are staged: every warp works
// alone.
#pragma once
#include <climits>

#include "pair_forces.cuh"

namespace dpd {

constexpr int kCellRanges = 14;          // own cell, cell x+1, four rows of three cells
constexpr int kCellHitCap = 512;         // warp list entries before a force pass (a multiple of 32)
constexpr float kCellTestR2 = 1.0001f;   // the test's cut-off; the force pass applies the exact one

struct CellWarp {
    uint2 hits[kCellHitCap];    // (slot | cell offsets + 1 in bits 26..31, owner lane)
    int4 rng[16];               // per candidate range: (first candidate, first slot, code bits, own cell);
                                // entries 14, 15: sentinels for the search
    float4 rsh[16];             // per range: the shift into the home cell's frame
    float4 hpos[32];            // the warp's home beads: cell-relative position, type
    float4 hvel[32];            // v~ and noise id
};

__host__ __device__ constexpr size_t cells_smem_bytes(int nt, int nwarps)
{
    return pair_tables_bytes<float>(nt) + sizeof(CellWarp) * (size_t)nwarps;
}

// Force phase over the warp's list (all 32 lanes call it): entries [0, nhits),
// lane L takes the contiguous run [L*per, (L+1)*per).
template <bool VIRIAL>
__device__ __forceinline__ void cells_force_pass(int nhits, const CellWarp* cw, int base, const float* Tsh, int nt,
                                                 uint32_t key0, float wx, float wy, float wz,
                                                 const double* L, const float4* __restrict__ pos4,
                                                 const float4* __restrict__ vel4, const double* __restrict__ xs,
                                                 float* __restrict__ F, float* __restrict__ stress, int n)
{
    __syncwarp();   // the list is complete
    uint32_t keys[10];   // the Philox round keys of this step (kept out of the test phase's registers)
    {
        uint32_t k = key0;
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys[q] = k; k += 0x9E3779B9u; }
    }
    const int lane = threadIdx.x & 31;
    const int per = (nhits + 31) >> 5;
    int f = lane * per;
    const int f1 = min(f + per, nhits);
    const int m2 = nt * nt;
    constexpr int NACC = VIRIAL ? 12 : 3;
    float acc[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) acc[q] = 0.f;
    int cur = -1, islot = 0, ti = 0;
    uint32_t idi = 0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vi = pi;
    auto flush = [&]() {
        atomicAdd(F + islot, acc[0]);
        atomicAdd(F + n + islot, acc[1]);
        atomicAdd(F + 2 * n + islot, acc[2]);
        if (VIRIAL) {
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(stress + (size_t)q * n + islot, acc[3 + q]);
        }
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[q] = 0.f;
    };
    for (; f < f1; ++f) {
        const uint2 e = cw->hits[f];
        const int a = (int)e.y;
        if (a != cur) {
            if (cur >= 0) flush();
            cur = a;
            pi = cw->hpos[a];
            vi = cw->hvel[a];
            islot = base + a;
            ti = (__float_as_int(pi.w) & 0xFF) * nt;
            idi = __float_as_uint(vi.w);
        }
        const int j = (int)(e.x & 0x03FFFFFFu);
        const float4 pj = pos4[j];
        const float4 vj = vel4[j];
        float dx = (pi.x - pj.x) - (float)((int)((e.x >> 26) & 3u) - 1) * wx;
        float dy = (pi.y - pj.y) - (float)((int)((e.x >> 28) & 3u) - 1) * wy;
        float dz = (pi.z - pj.z) - (float)((int)(e.x >> 30) - 1) * wz;
        float r2 = dx * dx + dy * dy + dz * dz;
        refine_close(dx, dy, dz, r2, xs, n, islot, j, L);
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
        // the test used a widened cut-off in the shifted frame: the exact one
        // is applied here, and coincident beads (r2 <= 1e-18) are dropped
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
    if (cur >= 0) flush();
    __syncwarp();   // every lane is done with the list before it is refilled
}

template <bool VIRIAL>
__global__ void __launch_bounds__(kPairBlock, 8) k_pair_forces_cells(
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
    float* Tsh = reinterpret_cast<float*>(pair_dyn);
    CellWarp* cw = reinterpret_cast<CellWarp*>(pair_dyn + pair_tables_bytes<float>(nt)) + (threadIdx.x >> 5);
    for (int k = threadIdx.x; k < 3 * nt * nt; k += kPairBlock) Tsh[k] = tab[k];
    const uint32_t key0 = philox_step_key(boxes[0].seed, *step_ptr);
    __syncthreads();   // tables; from here on every warp works alone
    const int lane = threadIdx.x & 31;
    const int base = blockIdx.x * kPairBlock + (threadIdx.x & ~31);
    if (base >= n) return;   // the whole warp past the end
    const int i = base + lane;
    const bool live = i < n;
    const Box& B = boxes[0];
    const int nx = B.nc[0], ny = B.nc[1], nz = B.nc[2];
    const float wx = (float)B.w[0], wy = (float)B.w[1], wz = (float)B.w[2];
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vi = pi;
    int c = -1;
    if (live) {
        pi = pos4[i];
        vi = vel4[i];
        c = cell[i];
    }
    cw->hpos[lane] = pi;
    cw->hvel[lane] = vi;
    if (lane < 2) cw->rng[kCellRanges + lane] = make_int4(INT_MAX, 0, 0, 0);   // search sentinels
    // runs of one home cell: slots are cell-sorted
    const int prev = __shfl_up_sync(0xffffffffu, c, 1);
    const unsigned firsts = __ballot_sync(0xffffffffu, live && (lane == 0 || prev != c));
    const int nlive = __popc(__ballot_sync(0xffffffffu, live));
    int nhits = 0;
    unsigned rem = firsts;
    while (rem) {
        const int a0 = __ffs(rem) - 1;
        rem &= rem - 1;
        const int a1 = rem ? __ffs(rem) - 1 : nlive;   // the run is lanes [a0, a1)
        const int hc = __shfl_sync(0xffffffffu, c, a0);
        // candidate ranges, one cell each, written by lanes 0..13
        int len = 0;
        if (lane < kCellRanges) {
            const int hx = hc % nx, hy = (hc / nx) % ny, hz = hc / (nx * ny);
            int ox, oy, oz;
            if (lane < 2) {
                ox = lane; oy = 0; oz = 0;
            } else {
                const int rr = (lane - 2) / 3;
                ox = (lane - 2) - 3 * rr - 1;
                oy = rr == 0 ? 1 : rr - 2;
                oz = rr == 0 ? 0 : 1;
            }
            int x2 = hx + ox, y2 = hy + oy, z2 = hz + oz;
            x2 += x2 < 0 ? nx : (x2 >= nx ? -nx : 0);
            y2 += y2 < 0 ? ny : (y2 >= ny ? -ny : 0);
            z2 += z2 >= nz ? -nz : 0;
            const int cc = x2 + nx * (y2 + ny * z2);
            const int lo = start[cc];
            len = start[cc + 1] - lo;
            int inc = len;
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) {
                const int y = __shfl_up_sync(0x3FFFu, inc, o, 16);
                if (lane >= o) inc += y;
            }
            cw->rng[lane] = make_int4(inc - len, lo,
                                      (int)(((uint32_t)(ox + 1) << 26) | ((uint32_t)(oy + 1) << 28) |
                                            ((uint32_t)(oz + 1) << 30)),
                                      lane == 0 ? 1 : 0);
            cw->rsh[lane] = make_float4((float)ox * wx, (float)oy * wy, (float)oz * wz, 0.f);
            len = inc;
        }
        const int ncand = __shfl_sync(0xffffffffu, len, kCellRanges - 1);
        __syncwarp();   // range table written
        // home beads in chunks of at most 16, so one round adds at most 512
        // entries and the list is emptied before a round, never inside it
        for (int ab = a0; ab < a1; ab += 16) {
        const int ae = min(a1, ab + 16);
        for (int k0 = 0; k0 < ncand; k0 += 32) {
            if (nhits + 32 * (ae - ab) > kCellHitCap) {
                cells_force_pass<VIRIAL>(nhits, cw, base, Tsh, nt, key0, wx, wy, wz, B.L, pos4, vel4, xs, F, stress,
                                         n);
                nhits = 0;
            }
            const int k = k0 + lane;
            const bool valid = k < ncand;
            // the range of candidate k: the last range whose first candidate is <= k
            int r = 0;
#pragma unroll
            for (int s = 8; s; s >>= 1)
                if (cw->rng[r + s].x <= k) r += s;
            const int4 R = cw->rng[r];
            const float4 S = cw->rsh[r];
            const int j = R.y + (k - R.x);
            float4 q = make_float4(1e30f, 1e30f, 1e30f, 0.f);
            if (valid) q = pos4[j];
            const float cx = q.x + S.x, cy = q.y + S.y, cz = q.z + S.z;
            const uint32_t ent = (uint32_t)j | (uint32_t)R.z;
            const bool own = R.w != 0;
            for (int a = ab; a < ae; ++a) {
                const float4 h = cw->hpos[a];
                const float ex = h.x - cx, ey = h.y - cy, ez = h.z - cz;
                const float r2 = ex * ex + ey * ey + ez * ez;
                const bool hit = valid && r2 < kCellTestR2 && (!own || j > base + a);
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (hit) cw->hits[nhits + __popc(m & ((1u << lane) - 1u))] = make_uint2(ent, (uint32_t)a);
                nhits += __popc(m);
            }
        }
        }
        __syncwarp();   // the range table is read before the next run rewrites it
    }
    cells_force_pass<VIRIAL>(nhits, cw, base, Tsh, nt, key0, wx, wy, wz, B.L, pos4, vel4, xs, F, stress, n);
}

}  // namespace dpd
