// upload.cuh -- bead upload on the device (CSimBox::AssignBeadstoCells,
// SimBox.cpp:715-762): the caller's arrays are copied once as they are
// (bead order, xyz interleaved), then
//   k_up_check   validates every bead, files it in its CNT cell
//                (ix = (long)(x/w)), splits unPBC - x into periodic images
//                and a residual offset, and counts the beads per cell;
//   k_scan_cells (dpd_kernels.cuh) turns the counts into cell starts;
//   k_up_scatter drops every bead into its cell's slot range;
//   k_up_place   orders each cell's beads by upload index (the slot order the
//                host counting sort used: by cell, then by upload index) and
//                writes the structure-of-arrays state in slot order.
// Nothing of the engine's state is written before k_up_check has passed.
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

// Error kinds of k_up_check, each recording the lowest failing bead index.
enum UploadError { kUpType = 0, kUpId, kUpBox, kUpNonFinite, kUpOutside, kUpImage, kUpErrors };

struct UploadIn {
    const double* x;        // 3 per bead, bead order
    const double* u;        // unPBC, or null
    const double* v;
    const double* f;        // or null
    const int64_t* id;
    const int* type;
    const int* box;         // or null (single box)
    const unsigned char* movable;   // or null
};

// The previous upload's bead ids and types (upload order), compared with
// the new ones so the host refreshes its copies only when they change.
struct UploadPrev {
    int64_t* id;           // n entries, overwritten with the new ids
    int* type;
    unsigned* changed;     // bit 0: an id differs, bit 1: a type differs
    int* type_count;       // beads per type (ntypes entries, zeroed by the caller)
};

// Validation and binning of an uploaded bead set: cell[b] receives the bead's
// CNT cell and the cells are counted; the first bead of each error kind is
// recorded in err; every valid bead's type is counted (block histogram).
__global__ void __launch_bounds__(256) k_up_check(int n, int nboxes, int ntypes, const Box* __restrict__ boxes,
                                                  UploadIn in, int* __restrict__ cell, uint32_t* __restrict__ img,
                                                  double* __restrict__ off, int* __restrict__ count,
                                                  int* __restrict__ block_count, int* __restrict__ err,
                                                  int* __restrict__ any_off, UploadPrev prev)
{
    __shared__ int hist[kMaxTypes];
    for (int k = threadIdx.x; k < ntypes; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned diff = 0;
    int c = -1;   // the bead's cell once it has passed every check
    if (b < n) {
        const int t = in.type[b];
        const int64_t idv = in.id[b];
        diff = (prev.id[b] != idv ? 1u : 0u) | (prev.type[b] != t ? 2u : 0u);
        prev.id[b] = idv;
        prev.type[b] = t;
        do {
            if (t < 0 || t >= ntypes) { atomicMin(&err[kUpType], b); break; }
            if (idv < 1 || idv > 0x7fffffff) { atomicMin(&err[kUpId], b); break; }
            const int bx = in.box ? in.box[b] : 0;
            if (bx < 0 || bx >= nboxes) { atomicMin(&err[kUpBox], b); break; }
            const Box& B = boxes[bx];
            long long ci[3];
            bool bad = false;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double xv = in.x[3 * b + d];
                if (!isfinite(xv) || !isfinite(in.v[3 * b + d])) { atomicMin(&err[kUpNonFinite], b); bad = true; break; }
                ci[d] = (long long)(xv / B.w[d]);
                if (xv < 0.0 || ci[d] < 0 || ci[d] >= B.nc[d]) { atomicMin(&err[kUpOutside], b); bad = true; break; }
            }
            if (bad) break;
            int ii[3] = {0, 0, 0};
            bool residual = false;
            double r[3] = {0.0, 0.0, 0.0};
            if (in.u) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double du = in.u[3 * b + d] - in.x[3 * b + d];
                    const double k = nearbyint(du / B.L[d]);
                    if (!(fabs(k) <= 511.0)) { atomicMin(&err[kUpImage], b); bad = true; break; }
                    ii[d] = (int)k;
                    r[d] = du - k * B.L[d];
                    residual |= r[d] != 0.0;
                }
            }
            if (bad) break;
            c = (int)(B.cell_base + ci[0] + (long long)B.nc[0] * (ci[1] + (long long)B.nc[1] * ci[2]));
            cell[b] = c;
            img[b] = img_pack(ii[0], ii[1], ii[2]);
#pragma unroll
            for (int d = 0; d < 3; ++d) off[(size_t)d * n + b] = r[d];
            if (residual) *any_off = 1;
            atomicAdd(&hist[t], 1);
        } while (false);
    }
    // cell and chunk counts, one atomic per distinct cell (chunk) and warp:
    // beads uploaded in cell order (a slab's exchange) share them
    const unsigned act = __ballot_sync(0xffffffffu, c >= 0);
    if (c >= 0) {
        const int lane = threadIdx.x & 31;
        const unsigned peers = __match_any_sync(act, c);
        if (lane == __ffs(peers) - 1) atomicAdd(&count[c], __popc(peers));
        const int chunk = c / kScanChunk;
        const unsigned cpeers = __match_any_sync(act, chunk);
        if (lane == __ffs(cpeers) - 1) atomicAdd(&block_count[chunk], __popc(cpeers));
    }
    const unsigned wdiff = __reduce_or_sync(0xffffffffu, diff);
    if ((threadIdx.x & 31) == 0 && wdiff) atomicOr(prev.changed, wdiff);
    __syncthreads();
    for (int k = threadIdx.x; k < ntypes; k += blockDim.x)
        if (hist[k]) atomicAdd(&prev.type_count[k], hist[k]);
}

__global__ void __launch_bounds__(256) k_up_scatter(int n, const int* __restrict__ cell,
                                                    const int* __restrict__ start, int* __restrict__ cursor,
                                                    int* __restrict__ perm)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int c = cell[b];
    perm[start[c] + atomicAdd(&cursor[c], 1)] = b;
}

template <typename real>
__global__ void __launch_bounds__(256) k_up_place(int n, UploadIn in, const int* __restrict__ cell,
                                                  const uint32_t* __restrict__ img, const int* __restrict__ start,
                                                  const int* __restrict__ perm, double* __restrict__ x,
                                                  double* __restrict__ v, real* __restrict__ F, int* __restrict__ bid,
                                                  int* __restrict__ tf, int* __restrict__ ocell,
                                                  uint32_t* __restrict__ oimg, int* __restrict__ pid,
                                                  int* __restrict__ pid_of)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = perm[s];
    const int c = cell[b];
    const int beg = start[c], end = start[c + 1];
    int k = 0;
    for (int q = beg; q < end; ++q) k += perm[q] < b;
    const int o = beg + k;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        x[(size_t)d * n + o] = in.x[3 * b + d];
        v[(size_t)d * n + o] = in.v[3 * b + d];
        F[(size_t)d * n + o] = in.f ? (real)in.f[3 * b + d] : real(0);
    }
    bid[o] = b;
    tf[o] = in.type[b] | ((in.box ? in.box[b] : 0) << 8) | ((in.movable && !in.movable[b]) ? kFlagFrozen : 0);
    ocell[o] = c;
    oimg[o] = img[b];
    pid[o] = (int)in.id[b];
    pid_of[b] = (int)in.id[b];
}

// kFlagBonded for the beads with bond or bond-pair terms (csr_ptr by upload
// index), in slot order.
__global__ void __launch_bounds__(256) k_mark_bonded(int n, const int* __restrict__ bid,
                                                     const int* __restrict__ csr_ptr, int* __restrict__ tf)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int b = bid[s];
    tf[s] = (tf[s] & ~kFlagBonded) | (csr_ptr[b + 1] > csr_ptr[b] ? kFlagBonded : 0);
}

}  // namespace dpd
