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
// SliceParams and the contour split itself (slice_add) live in
// dpd_kernels.cuh, shared with the bonded kernel.
#pragma once
#include "pair_forces.cuh"

namespace dpd {

// Pair part on a sample step: one thread per bead i over its own cell (beads
// after i) and the 13 cells of the reference's half shell, the DPD pair force
// of the force kernels (same Philox draw), accumulated into block-private
// bins in shared memory when they fit (sbins), else straight into global.
// Grid-stride loop; the bins are flushed once per block.
template <typename real>
__global__ void __launch_bounds__(256) k_slice_pairs(
    int n, const StepConst* __restrict__ K, const Box* __restrict__ boxes, const int64_t* __restrict__ step_ptr,
    const real* __restrict__ tab, const int* __restrict__ cell, const int* __restrict__ start,
    const typename Vec4<real>::type* __restrict__ pos4, const typename Vec4<real>::type* __restrict__ vel4,
    const double* __restrict__ x, SliceParams sp, int sbins)
{
    pdl_wait();
    pdl_launch();
    typedef typename Vec4<real>::type V4;
    extern __shared__ double sbin[];
    const int nt = K->ntypes, KT = nt * nt;
    const int nbins = sp.S * KT * 9;
    double* bins = sbins ? sbin : sp.pair;
    if (sbins) {
        for (int k = threadIdx.x; k < nbins; k += blockDim.x) sbin[k] = 0.0;
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
    const int m2 = nt * nt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V4 pi = pos4[i], vi = vel4[i];
        const int c = cell[i] - B.cell_base;
        const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
        const int ti = real_bits(pi.w) & 0xFF;
        const uint32_t idi = (uint32_t)real_bits(vi.w);
        const double zi = x[2 * (size_t)n + i];
        // o = 0: own cell after i; o = 1..13: (dx, dy, dz) of the reference's half shell
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
            const int jb = o == 0 ? i + 1 : start[c2], je = start[c2 + 1];
            for (int j = jb; j < je; ++j) {
                const V4 pj = pos4[j];
                const real dx = (pi.x - pj.x) - (real)ox * wx;
                const real dy = (pi.y - pj.y) - (real)oy * wy;
                const real dz = (pi.z - pj.z) - (real)oz * wz;
                const real r2 = dx * dx + dy * dy + dz * dz;
                if (!(r2 < real(1) && r2 > real(1e-18))) continue;
                const V4 vj = vel4[j];
                const real inv = RealOps<real>::rsqrt(r2);
                const real wr = real(1) - r2 * inv;
                const int tj = real_bits(pj.w) & 0xFF;
                const int tt = ti * nt + tj;
                const real rdotv = (dx * (vi.x - vj.x) + dy * (vi.y - vj.y) + dz * (vi.z - vj.z)) * inv;
                const uint32_t idj = (uint32_t)real_bits(vj.w);
                uint32_t c0 = min(idi, idj), c1 = max(idi, idj);
#pragma unroll
                for (int q = 0; q < 10; ++q) {
                    const uint64_t prod = (uint64_t)0xD256D193u * c0;
                    c0 = (uint32_t)(prod >> 32) ^ keys[q] ^ c1;
                    c1 = (uint32_t)prod;
                }
                const real mag = tab[tt] * wr - tab[m2 + tt] * wr * wr * rdotv +
                                 tab[2 * m2 + tt] * wr * noise_centered(c0, real(0));
                const real m = mag * inv;
                const double f[3] = {(double)(m * dx), (double)(m * dy), (double)(m * dz)};
                const double d[3] = {(double)dx, (double)dy, (double)dz};
                double fdx[9];
                outer9(f, d, fdx);
                slice_add(sp, bins, KT, tt, fdx, d[2], zi, x[2 * (size_t)n + j]);
            }
        }
    }
    if (sbins) {
        __syncthreads();
        for (int k = threadIdx.x; k < nbins; k += blockDim.x)
            if (sbin[k] != 0.0) atomicAdd(sp.pair + k, sbin[k]);
    }
}

}  // namespace dpd
