// monitor.cuh -- the sample data of the reference's CMonitor that are not
// single-bead sums of the step kernels, computed on the device from the
// current state on request (dpd_engine_monitor):
//
//   CMonitor::CalculateSingleBeadData     Monitor.cpp:790-1040  inertia tensor,
//                                         per-type mean square displacement
//   CMonitor::CalculateSinglePolymerData  Monitor.cpp:708-788   per-type mean
//                                         end-to-end distance (minimum image)
//   CMonitor::CalculateSingleBondData     Monitor.cpp:1052-1174 per-type and
//                                         global bond length (minimum image)
//   CMonitor::CalculateSingleBondPairData Monitor.cpp:1176-1273 per-type P2,
//                                         bond lengths, phi - phi0 and its
//                                         square, from CBondPair::AddForce's
//                                         observables (BondPair.cpp:140-199)
//
// Sums are FP64 and reduced per block in shared memory before one global
// atomic per bin and block; the host divides by the counts as the reference
// does.
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

// Slot-order pass over the beads: writes each bead's wrapped and unPBC
// position by upload index (xu: 6 planes of n) for the term kernels, and adds
// the inertia sums (6) and the per-type squared displacement from u0 (T) to
// sums[0..6+T).
__global__ void __launch_bounds__(256) k_monitor_beads(int n, int ntypes, const Box* __restrict__ boxes,
                                                       const int* __restrict__ tf, const int* __restrict__ bid,
                                                       const double* __restrict__ x, const uint32_t* __restrict__ img,
                                                       const double* __restrict__ off, const double* __restrict__ u0,
                                                       double* __restrict__ xu, double* __restrict__ sums)
{
    __shared__ double bin[6 + kMaxTypes];
    for (int k = threadIdx.x; k < 6 + ntypes; k += blockDim.x) bin[k] = 0.0;
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        const int b = bid[s];
        const int tfl = tf[s];
        const Box& B = boxes[flag_box(tfl)];
        const uint32_t im = img[s];
        double p[3], u[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            p[d] = x[d * n + s];
            u[d] = p[d] + (double)img_get(im, d) * B.L[d] + (off ? off[d * n + b] : 0.0);
            xu[d * n + b] = p[d];
            xu[(3 + d) * n + b] = u[d];
        }
        // m_totalInertia (Monitor.cpp:885-893): [0], [1], [2], [4], [5], [8]
        atomicAdd(&bin[0], p[1] * p[1] + p[2] * p[2]);
        atomicAdd(&bin[1], -p[0] * p[1]);
        atomicAdd(&bin[2], -p[0] * p[2]);
        atomicAdd(&bin[3], p[0] * p[0] + p[2] * p[2]);
        atomicAdd(&bin[4], -p[1] * p[2]);
        atomicAdd(&bin[5], p[0] * p[0] + p[1] * p[1]);
        // m_vBeadMSD (Monitor.cpp:838-843)
        const double d0 = u[0] - u0[3 * b], d1 = u[1] - u0[3 * b + 1], d2 = u[2] - u0[3 * b + 2];
        atomicAdd(&bin[6 + flag_type(tfl)], d0 * d0 + d1 * d1 + d2 * d2);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 6 + ntypes; k += blockDim.x)
        if (bin[k] != 0.0) atomicAdd(sums + k, bin[k]);
}

__device__ __forceinline__ double min_image(double d, double L)
{
    // Monitor.cpp:733-752: one correction by the box length past half of it
    if (d > 0.5 * L) return d - L;
    if (d < -0.5 * L) return d + L;
    return d;
}

struct MonitorTerms {
    int nb, np, na;
    const int* bond_h;         // upload indices
    const int* bond_t;
    const int* bond_type;
    const int* poly_h;         // polymer head / tail, upload indices
    const int* poly_t;
    const int* poly_type;
    const int* ang_b1h;        // first bond head (middle), first tail, second head, second tail
    const int* ang_b1t;
    const int* ang_b2h;
    const int* ang_b2t;
    const int* ang_type;
    const double* ang_phi0;
    const double* ang_cos0;
    const double* ang_sin0;
    int nbt, npt, nbpt;
    double L[3];
    // bins in sums: bonds [nbt], then bond length sum and square sum (2),
    // polymers [npt], bond pairs [nbpt][5] (P2, first, second, phi, phi^2)
    double* sums;
};

// One thread per bond, polymer and bond pair (grid over nb + np + na).
__global__ void __launch_bounds__(256) k_monitor_terms(MonitorTerms M, const double* __restrict__ xu, int n)
{
    extern __shared__ double tbin[];
    const int nbins = M.nbt + 2 + M.npt + 5 * M.nbpt;
    for (int k = threadIdx.x; k < nbins; k += blockDim.x) tbin[k] = 0.0;
    __syncthreads();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const double* px = xu;               // wrapped, plane d at d * n
    const double* pu = xu + 3 * (size_t)n;
    if (g < M.nb) {
        // CMonitor::CalculateSingleBondData, Monitor.cpp:1066-1098
        const int h = M.bond_h[g], t = M.bond_t[g];
        double r2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double dx = min_image(px[d * n + h] - px[d * n + t], M.L[d]);
            r2 += dx * dx;
        }
        const double r = sqrt(r2);
        atomicAdd(&tbin[M.bond_type[g]], r);
        atomicAdd(&tbin[M.nbt], r);
        atomicAdd(&tbin[M.nbt + 1], r * r);
    } else if (g < M.nb + M.np) {
        // CMonitor::CalculateSinglePolymerData, Monitor.cpp:719-756
        const int k = g - M.nb;
        const int h = M.poly_h[k], t = M.poly_t[k];
        double r2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double dx = min_image(px[d * n + h] - px[d * n + t], M.L[d]);
            r2 += dx * dx;
        }
        atomicAdd(&tbin[M.nbt + 2 + M.poly_type[k]], sqrt(r2));
    } else if (g < M.nb + M.np + M.na) {
        // CBondPair::AddForce observables (BondPair.cpp:140-199) on the unPBC
        // bond vectors, summed as CMonitor::CalculateSingleBondPairData
        const int k = g - M.nb - M.np;
        const int a1h = M.ang_b1h[k], a1t = M.ang_b1t[k], a2h = M.ang_b2h[k], a2t = M.ang_b2t[k];
        double b1[3], b2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            b1[d] = pu[d * n + a1h] - pu[d * n + a1t];
            b2[d] = pu[d * n + a2h] - pu[d * n + a2t];
        }
        const double l1 = sqrt(b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2]);
        const double l2 = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
        double P2 = 0.0, phid = 0.0, phid2 = 0.0;
        if (l1 * l2 > 0.0001) {
            const double dot = b1[0] * b2[0] + b1[1] * b2[1] + b1[2] * b2[2];
            const double o1 = dot / (l1 * l1), o2 = dot / (l2 * l2);
            const double cos2 = o1 * o2;
            const double phi0 = M.ang_phi0[k];
            if (fabs(dot) > 0.000001) {
                const double pre = sqrt(1.0 / cos2 - 1.0);
                P2 = phi0 > 0.0 ? 0.5 * (3.0 * cos2 * (M.ang_cos0[k] + M.ang_sin0[k] * pre) - 1.0)
                                : 0.5 * (3.0 * cos2 - 1.0);
            } else {
                P2 = -0.5;
            }
            phid = acos(cos2) - phi0;
            phid2 = phid * phid;
        }
        double* q = tbin + M.nbt + 2 + M.npt + 5 * M.ang_type[k];
        atomicAdd(q, P2);
        atomicAdd(q + 1, l1);
        atomicAdd(q + 2, l2);
        atomicAdd(q + 3, phid);
        atomicAdd(q + 4, phid2);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nbins; k += blockDim.x)
        if (tbin[k] != 0.0) atomicAdd(M.sums + k, tbin[k]);
}

}  // namespace dpd
