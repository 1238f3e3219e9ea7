// builder.cuh -- the random initial state of CRandomBuilder::Assemble
// (RandomBuilder.cpp:71-361, no walls, three dimensions) built on the device.
//
// The reference draws six numbers per bead, in bead order, from one 64-bit
// LCG (CCNTCell::Randf / lcg, CNTCell.cpp:2454-2466): the index into the
// velocity-magnitude table, x, y, z, then the polar and azimuthal angles of
// the velocity.  k_rb_beads gives every bead its own thread: the generator's
// state before the bead's first draw is the seed advanced by skip + 6 i steps,
// found in O(log) multiplications by the arbitrary-stride method for linear
// congruential generators (F. B. Brown, "Random number generation with
// arbitrary strides", Trans. Am. Nucl. Soc. 71 (1994) 202).  Positions use the
// reference's own operations in its order with explicit round-to-nearest
// intrinsics (no fused multiply-add), so they equal the reference's bit for
// bit; velocities go through the device's acos/sin/cos and a tree sum, and
// agree to a few ulps.
//
// Bonds are shortened per connected component of the bond graph (one thread
// each, bonds in the reference's polymer order), the centre-of-mass velocity
// is removed and the velocities are scaled to kT with the 3N normalisation.
// The velocity-magnitude table (CBuilder::MaxwellDist, Builder.cpp:104-126)
// is a sequential recurrence through the C library's exp and log; the host
// computes it exactly as the reference does and uploads it.
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

constexpr uint64_t kLcgMul = 6364136223846793005ull;   // CCNTCell::lcg, CNTCell.cpp:2461-2465
constexpr int kRbThreads = 256;

// The LCG state after k steps from s (state' = kLcgMul * state + 1, mod 2^64).
__device__ __forceinline__ uint64_t lcg_advance(uint64_t s, uint64_t k)
{
    uint64_t am = 1, ap = 0, cm = kLcgMul, cp = 1;
    while (k) {
        if (k & 1) {
            am *= cm;
            ap = ap * cm + cp;
        }
        cp = (cm + 1) * cp;
        cm *= cm;
        k >>= 1;
    }
    return am * s + ap;
}

__device__ __forceinline__ double lcg_draw(uint64_t& s)
{
    s = kLcgMul * s + 1ull;
    return (double)(uint32_t)(s >> 32) * (1.0 / 4294967296.0);   // CCNTCell::Randf, CNTCell.cpp:2454-2457
}

// Per bead: position (x3, interleaved, bead order) and unscaled velocity
// (v3); per block, the velocity sums in part[3 * blockIdx.x + d].
__global__ void __launch_bounds__(kRbThreads) k_rb_beads(int n, uint64_t seed, uint64_t skip, double Lx, double Ly,
                                                         double Lz, const double* __restrict__ tab, int64_t ntab,
                                                         double* __restrict__ x3, double* __restrict__ v3,
                                                         double* __restrict__ part)
{
    __shared__ double red[kRbThreads / 32][3];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vp[3] = {0.0, 0.0, 0.0};
    if (i < n) {
        uint64_t s = lcg_advance(seed, skip + 6ull * (uint64_t)i);
        // RandomBuilder.cpp:139-140: index = (long)(table size * u)
        const int64_t index = (int64_t)__dmul_rn((double)ntab, lcg_draw(s));
        const double vmag = tab[min(index, ntab - 1)];
        const double L[3] = {Lx, Ly, Lz};
        double xp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // wall width (0) + bulk length * u, moved to 0 within 1e-4 of the
            // upper face (RandomBuilder.cpp:142-191)
            xp[d] = __dadd_rn(0.0, __dmul_rn(L[d], lcg_draw(s)));
            if (__dadd_rn(L[d], -xp[d]) < 0.0001) xp[d] = 0.0;
        }
        // RandomBuilder.cpp:201-208
        const double vtheta = acos(__dadd_rn(1.0, -__dmul_rn(2.0, lcg_draw(s))));
        const double vphi = __dmul_rn(2.0 * 3.141592653589793238, lcg_draw(s));   // xxBase::m_globalTwoPI
        const double st = sin(vtheta);
        vp[0] = __dmul_rn(__dmul_rn(vmag, st), cos(vphi));
        vp[1] = __dmul_rn(__dmul_rn(vmag, st), sin(vphi));
        vp[2] = __dmul_rn(vmag, cos(vtheta));
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x3[3 * (size_t)i + d] = xp[d];
            v3[3 * (size_t)i + d] = vp[d];
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double a = vp[d];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) red[w][d] = a;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int k = 0; k < kRbThreads / 32; ++k) a += red[k][threadIdx.x];
        part[3 * blockIdx.x + threadIdx.x] = a;
    }
}

// Bond shortening (RandomBuilder.cpp:241-311): one thread per connected
// component of the bond graph walks its bonds (comp_bonds[comp_ptr[c] ..
// comp_ptr[c+1]), bead indices, the reference's polymer order) and, where a
// component of tail - head exceeds 1 in magnitude, sets the tail's coordinate
// to head + the unit vector's component.
__global__ void __launch_bounds__(kRbThreads) k_rb_bonds(int ncomp, const int64_t* __restrict__ comp_ptr,
                                                         const int64_t* __restrict__ comp_bonds,
                                                         const int64_t* __restrict__ head,
                                                         const int64_t* __restrict__ tail, double* __restrict__ x3)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    for (int64_t q = comp_ptr[c]; q < comp_ptr[c + 1]; ++q) {
        const int64_t k = comp_bonds[q];
        const double* h = x3 + 3 * head[k];
        double* t = x3 + 3 * tail[k];
        const double rd[3] = {__dadd_rn(t[0], -h[0]), __dadd_rn(t[1], -h[1]), __dadd_rn(t[2], -h[2])};
        const double rmag =
            sqrt(__dadd_rn(__dadd_rn(__dmul_rn(rd[0], rd[0]), __dmul_rn(rd[1], rd[1])), __dmul_rn(rd[2], rd[2])));
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (fabs(rd[d]) > 1.0) t[d] = __dadd_rn(h[d], __ddiv_rn(rd[d], rmag));
    }
}

// One block: sums the per-block partials of k_rb_beads in block order and
// leaves the centre-of-mass velocity (sum / n) in out[0..3).
__global__ void __launch_bounds__(32) k_rb_vcm(int nblocks, int n, const double* __restrict__ part,
                                               double* __restrict__ out)
{
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int b = 0; b < nblocks; ++b) a += part[3 * b + threadIdx.x];
        out[threadIdx.x] = a / (double)n;
    }
}

// v -= vcm (RandomBuilder.cpp:326-336); per block, the sum of v.v of the
// centred velocities in part[blockIdx.x].
__global__ void __launch_bounds__(kRbThreads) k_rb_center(int n, const double* __restrict__ vcm,
                                                          double* __restrict__ v3, double* __restrict__ part)
{
    __shared__ double red[kRbThreads / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double a = 0.0;
    if (i < n) {
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = __dadd_rn(v3[3 * (size_t)i + d], -vcm[d]);
            v3[3 * (size_t)i + d] = v[d];
        }
        a = __dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2]));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kRbThreads / 32; ++k) s += red[k];
        part[blockIdx.x] = s;
    }
}

// One block: vtotal = sqrt(sum v.v / 3N) (RandomBuilder.cpp:345-349) into out[3].
__global__ void __launch_bounds__(32) k_rb_vtotal(int nblocks, int n, const double* __restrict__ part,
                                                  double* __restrict__ out)
{
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int b = 0; b < nblocks; ++b) a += part[b];
        out[3] = sqrt(a / (double)(3 * (int64_t)n));
    }
}

// v = sqrt(kT) v / vtotal (RandomBuilder.cpp:356-358).
__global__ void __launch_bounds__(kRbThreads) k_rb_scale(int n, double rootkT, const double* __restrict__ stats,
                                                         double* __restrict__ v3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n) return;
    v3[i] = __ddiv_rn(__dmul_rn(rootkT, v3[i]), stats[3]);
}

// ---------------------------------------------------------------- lamella
//
// CLamellaBuilder::Assemble (LamellaBuilder.cpp:126-1010, no walls, no
// polymerised bonds) with the in-plane Maxwell velocities of
// CBuilder::AssignMaxwellVelocities (Builder.cpp:4207-4330).  The host walks
// the hexagonal lattice of each monolayer (a short sequential recurrence in
// the reference's floating-point order) and counts every polymer's draws;
// k_lb_beads then gives every bead its own thread: a bilayer polymer's bead on
// the head-tail line (straight chains, no draws) or scattered about it (three
// draws), a solvent bead in the free region its polymer drew (one draw per
// polymer, three per bead), and two draws for the velocity, each at its place
// in the reference's single generator stream (lcg_advance).

struct LamellaParams {
    int normal, p0, p1;           // normal axis; axes taking the lattice's first and second coordinate
    int size, head_offset, tail_offset, lipid_type, linearise;
    double L[3];
    double centre, thickness;
    double mhead[2], msign[2], e1x[2], e2y[2], cspace[2];
    double ex[6];                 // excluded regions along the normal (Builder.cpp:293-360)
    double ratio[2];              // cumulative shares of the free length of the two free regions
    uint64_t seed, skip, vel_base;   // generator seed; draws before the builder; draws before the velocities
    int64_t ntab;
};

// Per bead: position (x3) and unscaled in-plane velocity (v3: VX, VY, 0);
// per block, the velocity sums in part[3 * blockIdx.x + d].
__global__ void __launch_bounds__(kRbThreads) k_lb_beads(int n, LamellaParams P, const int* __restrict__ bpoly,
                                                         const int64_t* __restrict__ pfirst,
                                                         const int* __restrict__ ptype,
                                                         const int64_t* __restrict__ pdraw,
                                                         const int* __restrict__ plip,
                                                         const double* __restrict__ site,
                                                         const int* __restrict__ mono,
                                                         const double* __restrict__ tab, double* __restrict__ x3,
                                                         double* __restrict__ v3, double* __restrict__ part)
{
    __shared__ double red[kRbThreads / 32][3];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double vp[3] = {0.0, 0.0, 0.0};
    if (b < n) {
        const int p = bpoly[b];
        const int k = (int)(b - pfirst[p]);
        double q[3];
        if (ptype[p] == P.lipid_type) {
            const int j = plip[p];
            const int mi = mono[j];
            const double xp0 = site[2 * (size_t)j], xp1 = site[2 * (size_t)j + 1];
            const double sg = P.msign[mi];
            if (k == P.tail_offset || k == P.head_offset || P.linearise) {
                q[P.p0] = xp0;
                q[P.p1] = xp1;
                if (k == P.tail_offset) {
                    q[P.normal] = __dadd_rn(P.centre, __dmul_rn(sg, 0.2));      // LamellaBuilder.cpp:567
                } else if (k == P.head_offset) {
                    q[P.normal] = P.mhead[mi];
                } else {
                    // the k-th bead's place among the beads between: head z - sign * counter * spacing
                    const double bc = (double)(k - (P.head_offset < k) - (P.tail_offset < k) + 1);
                    q[P.normal] = __dadd_rn(P.mhead[mi], -__dmul_rn(__dmul_rn(sg, bc), P.cspace[mi]));
                }
            } else {
                const int ii = k - (P.head_offset < k) - (P.tail_offset < k);
                uint64_t s = lcg_advance(P.seed, P.skip + (uint64_t)pdraw[p] + 3ull * (uint64_t)ii);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double u = lcg_draw(s);
                    if (d == P.normal)
                        q[d] = __dadd_rn(P.centre, __dmul_rn(__dmul_rn(__dmul_rn(0.5, sg), P.thickness), u));
                    else if (d == P.p0)
                        q[d] = __dadd_rn(xp0, __dmul_rn(__dmul_rn(0.5, P.e1x[mi]), u));
                    else
                        q[d] = __dadd_rn(xp1, __dmul_rn(__dmul_rn(0.5, P.e2y[mi]), u));
                }
                if (q[P.p0] > P.L[P.p0]) q[P.p0] = __dadd_rn(q[P.p0], -__dmul_rn(0.5, P.e1x[mi]));
                if (q[P.p1] > P.L[P.p1]) q[P.p1] = __dadd_rn(q[P.p1], -__dmul_rn(0.5, P.e2y[mi]));
            }
        } else {
            // the polymer's free region (Builder.cpp:383-406), then this bead's three draws
            uint64_t s = lcg_advance(P.seed, P.skip + (uint64_t)pdraw[p]);
            const double rindex = lcg_draw(s);
            const int index = rindex <= P.ratio[0] ? 0 : (rindex <= P.ratio[1] ? 1 : 0);
            const double width = __dadd_rn(P.ex[2 * index + 2], -P.ex[2 * index + 1]);
            s = lcg_advance(P.seed, P.skip + (uint64_t)pdraw[p] + 1ull + 3ull * (uint64_t)k);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double u = lcg_draw(s);
                q[d] = d == P.normal ? __dadd_rn(P.ex[2 * index + 1], __dmul_rn(width, u))
                                     : __dmul_rn(__dmul_rn(0.95, P.L[d]), u);
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) x3[3 * (size_t)b + d] = q[d];
        // Builder.cpp:4262-4275: table index, phi = 2 pi u, (vmag cos phi, vmag sin phi)
        uint64_t s = lcg_advance(P.seed, P.skip + P.vel_base + 2ull * (uint64_t)b);
        const int64_t index = (int64_t)__dmul_rn((double)P.ntab, lcg_draw(s));
        const double vmag = tab[min(index, P.ntab - 1)];
        const double vphi = __dmul_rn(2.0 * 3.141592653589793238, lcg_draw(s));   // xxBase::m_globalTwoPI
        vp[0] = __dmul_rn(vmag, cos(vphi));
        vp[1] = __dmul_rn(vmag, sin(vphi));
#pragma unroll
        for (int d = 0; d < 3; ++d) v3[3 * (size_t)b + d] = vp[d];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double a = vp[d];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) red[w][d] = a;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int k = 0; k < kRbThreads / 32; ++k) a += red[k][threadIdx.x];
        part[3 * blockIdx.x + threadIdx.x] = a;
    }
}

// One block: vtotal = sqrt(sum v.v / (2 N kT)) (Builder.cpp:4298-4302, 2-d) into out[3].
__global__ void __launch_bounds__(32) k_lb_vtotal(int nblocks, int n, double kT, const double* __restrict__ part,
                                                  double* __restrict__ out)
{
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int b = 0; b < nblocks; ++b) a += part[b];
        out[3] = sqrt(__ddiv_rn(a, __dmul_rn(__dmul_rn(2.0, (double)n), kT)));
    }
}

// V = V / vtotal, placed in the in-plane axes (Builder.cpp:4306-4330):
// normal x: (0, VY, VX); y: (VX, 0, VY); z: (VX, VY, 0).
__global__ void __launch_bounds__(kRbThreads) k_lb_scale(int n, int normal, const double* __restrict__ stats,
                                                         double* __restrict__ v3)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    double* v = v3 + 3 * (size_t)b;
    const double VX = __ddiv_rn(v[0], stats[3]), VY = __ddiv_rn(v[1], stats[3]);
    if (normal == 0) { v[0] = 0.0; v[1] = VY; v[2] = VX; }
    else if (normal == 1) { v[0] = VX; v[1] = 0.0; v[2] = VY; }
    else { v[0] = VX; v[1] = VY; v[2] = 0.0; }
}

}  // namespace dpd
