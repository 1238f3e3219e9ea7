// slab.cuh -- one box split into z-slabs over ranks, each rank's slab kept on
// its GPU between steps (the reference's mps* decomposition: SimBox.cpp:481-567,
// mpsSimBox.cpp:796-860; its per-processor force loop CNTCell.cpp:3598).
//
// Each rank's engine steps a local box of its own cell layers [z0, z1) plus
// g ghost layers on either side.  In upload order the local beads are the
// owned ones first (upload indices [0, n_owned)), then the ghosts.  After a
// step, one exchange per neighbour carries
//   * migrants: owned beads that left [z0, z1); the receiver owns them from
//     now on, and the sender keeps them as ghosts (they lie in its ghost
//     layer next to the face they crossed);
//   * ghosts: owned beads that stay and lie within g layers of the face, the
//     neighbour's ghosts for the next step.
// This single exchange equals the two of the host form (ghosts before the
// step, migrants after it): the beads a neighbour needs as ghosts for the next
// step are its neighbour's owned beads in the boundary layers after the
// migration, which are either staying beads (sent as ghosts) or beads that
// just migrated out of the neighbour itself (kept by it as ghosts).
//
// Kernels here: classification and ordered compaction of the records to
// send (k_slab_count / k_slab_offsets / k_slab_write, slot order, so the
// result does not depend on thread timing), the sizes of the next local box
// (k_slab_sizes), its placement into the step's input arrays
// (k_slab_place_state), and the device topology filter that keeps the bonds and
// bond pairs whose beads are all in the local box (k_slab_idmap,
// k_slab_endpoints, k_slab_term_count, k_slab_term_write, with the scan
// kernels k_scan_*).
#pragma once
#include "dpd_kernels.cuh"

namespace dpd {

// DPD_STATUS_SLAB_REACH of the C ABI
constexpr unsigned kStatusSlabReach = 0x10u;

// a bead record: id, type, movable, kind (0 migrant, 1 ghost), x, unPBC, v, F
constexpr int kSlabRec = 16;
enum SlabField { kRecId = 0, kRecType = 1, kRecMovable = 2, kRecKind = 3, kRecX = 4, kRecU = 7, kRecV = 10,
                 kRecF = 13 };
// record 0 of an exchange buffer is its header: beads, of them migrants
// (stored first), overflow flag (more beads than the buffer's capacity)
enum SlabHeader { kHdrCount = 0, kHdrMigrants = 1, kHdrOverflow = 2 };
// the classification's output streams
enum SlabOut { kToBelowMig = 0, kToBelowGhost, kToAboveMig, kToAboveGhost, kKeep, kSlabOuts };

struct SlabGeom {
    int z0, z1, g, nzg;    // owned global layers [z0, z1), ghost layers per side, global layers
    double w, Lz, c;       // layer width, global box length in z, (z0 - g) * w (local origin, global frame)
    int n_owned;           // upload indices [0, n_owned) are owned
    int cap;               // records one exchange buffer holds (besides its header)
};

// Where an owned bead in local layer lz goes (bits over SlabOut); ghosts go
// nowhere (the owner sends them again).  With at least 2g owned layers no
// bead is a ghost for both neighbours.
__host__ __device__ __forceinline__ unsigned slab_classify(int lz, bool owned, int g, int own)
{
    if (!owned) return 0u;
    if (lz < g) return 1u << kToBelowMig;
    if (lz >= g + own) return 1u << kToAboveMig;
    unsigned m = 1u << kKeep;
    if (lz < 2 * g) m |= 1u << kToBelowGhost;
    if (lz >= own) m |= 1u << kToAboveGhost;
    return m;
}

// local cell layer of a wrapped local z: (long)(z / w), the upload's binning rule
__device__ __forceinline__ int slab_layer(double z, double w) { return (int)(long long)(z / w); }

// Per block: beads of each output stream (block counts, nblocks per stream).
__global__ void __launch_bounds__(256) k_slab_count(int n, SlabGeom G, const double* __restrict__ x,
                                                    const int* __restrict__ bid, int* __restrict__ bcount)
{
    __shared__ int cnt[kSlabOuts];
    if (threadIdx.x < kSlabOuts) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned m = 0;
    if (s < n) m = slab_classify(slab_layer(x[2 * (size_t)n + s], G.w), bid[s] < G.n_owned, G.g, G.z1 - G.z0);
#pragma unroll
    for (int k = 0; k < kSlabOuts; ++k) {
        const unsigned b = __ballot_sync(0xffffffffu, (m >> k) & 1u);
        if ((threadIdx.x & 31) == 0 && b) atomicAdd(&cnt[k], __popc(b));
    }
    __syncthreads();
    if (threadIdx.x < kSlabOuts) bcount[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// One block: exclusive scan of every stream's block counts (in place) and
// the totals; writes the two send headers.
__global__ void __launch_bounds__(1024) k_slab_offsets(int nblocks, int* __restrict__ bcount,
                                                       int* __restrict__ total, double* __restrict__ send_below,
                                                       double* __restrict__ send_above, int cap)
{
    __shared__ int wsum[32];
    __shared__ int carry;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    for (int k = 0; k < kSlabOuts; ++k) {
        int* a = bcount + (size_t)k * nblocks;
        if (t == 0) carry = 0;
        __syncthreads();
        for (int base = 0; base < nblocks; base += 1024) {
            const int i = base + t;
            const int v = i < nblocks ? a[i] : 0;
            int inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) wsum[wid] = inc;
            __syncthreads();
            if (wid == 0) {
                int ws = wsum[lane];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, ws, o);
                    if (lane >= o) ws += y;
                }
                wsum[lane] = ws;   // inclusive over warps
            }
            __syncthreads();
            const int before = carry + (wid ? wsum[wid - 1] : 0) + inc - v;
            if (i < nblocks) a[i] = before;
            __syncthreads();
            if (t == 1023) carry = before + v;
            __syncthreads();
        }
        if (t == 0) total[k] = carry;
        __syncthreads();
    }
    if (t == 0) {
        const int bm = total[kToBelowMig], bg = total[kToBelowGhost];
        const int am = total[kToAboveMig], ag = total[kToAboveGhost];
        send_below[kHdrCount] = (double)(bm + bg);
        send_below[kHdrMigrants] = (double)bm;
        send_below[kHdrOverflow] = (bm + bg > cap) ? 1.0 : 0.0;
        send_above[kHdrCount] = (double)(am + ag);
        send_above[kHdrMigrants] = (double)am;
        send_above[kHdrOverflow] = (am + ag > cap) ? 1.0 : 0.0;
        for (int q = 3; q < kSlabRec; ++q) send_below[q] = send_above[q] = 0.0;
    }
}

// The record of the bead in slot s (the state dpd_engine_download reads),
// local frame.
template <typename real>
__device__ __forceinline__ void slab_record(int n, int s, const Box& B, const double* __restrict__ x,
                                            const double* __restrict__ v, const real* __restrict__ F,
                                            const uint32_t* __restrict__ img, const double* __restrict__ off,
                                            const int* __restrict__ tf, const int* __restrict__ bid,
                                            const int* __restrict__ pid, double r[kSlabRec])
{
    const int b = bid[s];
    const int tfl = tf[s];
    const uint32_t im = img[s];
    r[kRecId] = (double)pid[s];
    r[kRecType] = (double)(tfl & 0xFF);
    r[kRecMovable] = flag_frozen(tfl) ? 0.0 : 1.0;
    r[kRecKind] = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xv = x[(size_t)d * n + s];
        r[kRecX + d] = xv;
        r[kRecU + d] = xv + (double)img_get(im, d) * B.L[d] + (off ? off[(size_t)d * n + b] : 0.0);
        r[kRecV + d] = v[(size_t)d * n + s];
        r[kRecF + d] = (double)F[(size_t)d * n + s];
    }
}

__device__ __forceinline__ void slab_store(double* __restrict__ dst, const double r[kSlabRec])
{
    double2* q = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int k = 0; k < kSlabRec / 2; ++k) q[k] = make_double2(r[2 * k], r[2 * k + 1]);
}

// Writes every owned bead's record(s) at its place in slot order: migrants
// and ghosts into the send buffers (global frame), staying beads into keep
// and migrants also into mine (local frame; the sender's ghosts next step).
template <typename real>
__global__ void __launch_bounds__(256) k_slab_write(
    int n, SlabGeom G, const Box* __restrict__ boxes, const double* __restrict__ x, const double* __restrict__ v,
    const real* __restrict__ F, const uint32_t* __restrict__ img, const double* __restrict__ off,
    const int* __restrict__ tf, const int* __restrict__ bid, const int* __restrict__ pid,
    const int* __restrict__ boff, const int* __restrict__ total, double* __restrict__ send_below,
    double* __restrict__ send_above, double* __restrict__ keep, double* __restrict__ mine)
{
    __shared__ int wbase[kSlabOuts][8];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned m = 0;
    if (s < n) m = slab_classify(slab_layer(x[2 * (size_t)n + s], G.w), bid[s] < G.n_owned, G.g, G.z1 - G.z0);
    unsigned ball[kSlabOuts];
#pragma unroll
    for (int k = 0; k < kSlabOuts; ++k) {
        ball[k] = __ballot_sync(0xffffffffu, (m >> k) & 1u);
        if (lane == 0) wbase[k][wid] = __popc(ball[k]);
    }
    __syncthreads();
    if (!m) return;
    int pos[kSlabOuts];
#pragma unroll
    for (int k = 0; k < kSlabOuts; ++k) {
        int before = 0;
        for (int w = 0; w < wid; ++w) before += wbase[k][w];
        pos[k] = boff[(size_t)k * gridDim.x + blockIdx.x] + before + __popc(ball[k] & ((1u << lane) - 1u));
    }
    double r[kSlabRec];
    slab_record<real>(n, s, boxes[0], x, v, F, img, off, tf, bid, pid, r);
    if (m & (1u << kKeep)) slab_store(keep + (size_t)kSlabRec * pos[kKeep], r);
    if (m & ((1u << kToBelowMig) | (1u << kToAboveMig))) {
        const int k = (m & (1u << kToBelowMig)) ? pos[kToBelowMig] : total[kToBelowMig] + pos[kToAboveMig];
        slab_store(mine + (size_t)kSlabRec * k, r);
    }
    // to the global frame: z + c, wrapped into [0, Lz); unPBC z + c
    double zg = r[kRecX + 2] + G.c;
    if (zg < 0.0) zg += G.Lz;
    else if (zg >= G.Lz) zg -= G.Lz;
    r[kRecX + 2] = zg;
    r[kRecU + 2] += G.c;
    const int bm = total[kToBelowMig], am = total[kToAboveMig];
    if (m & (1u << kToBelowMig)) {
        if (pos[kToBelowMig] < G.cap) slab_store(send_below + (size_t)kSlabRec * (1 + pos[kToBelowMig]), r);
    }
    if (m & (1u << kToAboveMig)) {
        if (pos[kToAboveMig] < G.cap) slab_store(send_above + (size_t)kSlabRec * (1 + pos[kToAboveMig]), r);
    }
    r[kRecKind] = 1.0;
    if (m & (1u << kToBelowGhost)) {
        const int k = bm + pos[kToBelowGhost];
        if (k < G.cap) slab_store(send_below + (size_t)kSlabRec * (1 + k), r);
    }
    if (m & (1u << kToAboveGhost)) {
        const int k = am + pos[kToAboveGhost];
        if (k < G.cap) slab_store(send_above + (size_t)kSlabRec * (1 + k), r);
    }
}

// Sizes of the next local box, from the two received headers and this
// rank's own counts: out[0] owned beads, out[1] all beads, out[2..3] the
// received headers' overflow flags, out[4] the device status word, out[5..10]
// the segment lengths (keep, migrants from below, from above, ghosts from
// below, from above, mine), out[11] this rank's own send overflow.
__global__ void k_slab_sizes(const double* __restrict__ recv_below, const double* __restrict__ recv_above,
                             const int* __restrict__ total, const unsigned* __restrict__ status, int cap,
                             int* __restrict__ out)
{
    const int mb = (int)recv_below[kHdrMigrants], gb = (int)recv_below[kHdrCount] - mb;
    const int ma = (int)recv_above[kHdrMigrants], ga = (int)recv_above[kHdrCount] - ma;
    const int keep = total[kKeep], mine = total[kToBelowMig] + total[kToAboveMig];
    out[0] = keep + mb + ma;
    out[1] = keep + mb + ma + gb + ga + mine;
    out[2] = recv_below[kHdrOverflow] != 0.0;
    out[3] = recv_above[kHdrOverflow] != 0.0;
    out[4] = (int)*status;
    out[5] = keep; out[6] = mb; out[7] = ma; out[8] = gb; out[9] = ga; out[10] = mine;
    out[11] = total[kToBelowMig] + total[kToBelowGhost] > cap || total[kToAboveMig] + total[kToAboveGhost] > cap;
}

// The next local box written straight into the step's input arrays in
// upload order (slot o = upload index o; the next step's drift, cell scan
// and gather bin them, as after any step): the record's x, v and F, its
// type and movability, its CNT cell by the upload's rule ix = (long)(x/w),
// its periodic images (unPBC - x in whole box lengths) and the residual in
// off, its id (noise id, pid_of, and the previous-upload copy the host reads
// ids from).  Order of the beads: the kept owned beads, migrants from below,
// from above (the owned beads), ghosts from below, from above, this rank's
// own migrants; received records come in the global frame: z - c, wrapped
// into [0, Lz) (a ghost from across the global z face takes the periodic
// shift), unPBC z - c.  The records are the engine's own: a bead outside the
// box, of an unknown type or with an image count beyond +-511 is filed in
// range and sets DPD_STATUS_INTERNAL.
template <typename real>
__global__ void __launch_bounds__(256) k_slab_place_state(
    int n, int ntypes, SlabGeom G, const Box* __restrict__ boxes, const int* __restrict__ seg,
    const double* __restrict__ keep, const double* __restrict__ recv_below, const double* __restrict__ recv_above,
    const double* __restrict__ mine, double* __restrict__ x, double* __restrict__ v, real* __restrict__ F,
    int* __restrict__ bid, int* __restrict__ tf, int* __restrict__ cell, uint32_t* __restrict__ img,
    int* __restrict__ pid, int* __restrict__ pid_of, double* __restrict__ off, int64_t* __restrict__ prev_id,
    int* __restrict__ prev_type, unsigned* __restrict__ status)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int nkeep = seg[0], mb = seg[1], ma = seg[2], gb = seg[3], ga = seg[4];
    const double* src;
    bool received = true;
    int k = o;
    if (k < nkeep) { src = keep + (size_t)kSlabRec * k; received = false; }
    else if ((k -= nkeep) < mb) src = recv_below + (size_t)kSlabRec * (1 + k);
    else if ((k -= mb) < ma) src = recv_above + (size_t)kSlabRec * (1 + k);
    else if ((k -= ma) < gb) src = recv_below + (size_t)kSlabRec * (1 + mb + k);
    else if ((k -= gb) < ga) src = recv_above + (size_t)kSlabRec * (1 + ma + k);
    else { src = mine + (size_t)kSlabRec * (k - ga); received = false; }
    double r[kSlabRec];
    const double2* q = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int j = 0; j < kSlabRec / 2; ++j) {
        const double2 p = q[j];
        r[2 * j] = p.x;
        r[2 * j + 1] = p.y;
    }
    if (received) {
        double z = r[kRecX + 2] - G.c;
        if (z < 0.0) z += G.Lz;
        else if (z >= G.Lz) z -= G.Lz;
        r[kRecX + 2] = z;
        r[kRecU + 2] -= G.c;
    }
    const Box& B = boxes[0];
    bool bad = false;
    int ci[3], ii[3];
    const size_t N = (size_t)n;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xv = r[kRecX + d];
        long long c = (long long)(xv / B.w[d]);
        if (!(xv >= 0.0) || c < 0 || c >= B.nc[d]) {
            bad = true;
            c = c < 0 ? 0 : (c >= B.nc[d] ? B.nc[d] - 1 : c);
        }
        ci[d] = (int)c;
        const double du = r[kRecU + d] - xv;
        double kk = nearbyint(du / B.L[d]);
        if (!(fabs(kk) <= 511.0)) { bad = true; kk = 0.0; }
        ii[d] = (int)kk;
        off[(size_t)d * N + o] = du - kk * B.L[d];
        x[(size_t)d * N + o] = xv;
        v[(size_t)d * N + o] = r[kRecV + d];
        F[(size_t)d * N + o] = (real)r[kRecF + d];
    }
    int t = (int)r[kRecType];
    if (t < 0 || t >= ntypes) { bad = true; t = 0; }
    const int id = (int)r[kRecId];
    bid[o] = o;
    tf[o] = t | (r[kRecMovable] != 0.0 ? 0 : kFlagFrozen);
    cell[o] = B.cell_base + ci[0] + B.nc[0] * (ci[1] + B.nc[1] * ci[2]);
    img[o] = img_pack(ii[0], ii[1], ii[2]);
    pid[o] = id;
    pid_of[o] = id;
    prev_id[o] = id;
    prev_type[o] = t;
    if (bad) atomicOr(status, 0x8u);
}

__global__ void k_slab_status(unsigned* __restrict__ status, unsigned bits) { *status |= bits; }

// Single-bead sums over the owned beads only (upload indices below n_owned),
// per block and term (term-major, the layout k_reduce_obs reads): momentum,
// squared momentum, the per-bead virial (when stress is given), position and
// angular momentum.  Summed over the ranks they are the whole box's: every
// bead is owned once, and the per-bead virial counts a pair once when each
// bead of it holds half (the full-shell kernel) and a bond or bond pair at
// the one bead that holds it.
template <typename real>
__global__ void __launch_bounds__(256) k_slab_obs_partials(int n, int n_owned, const int* __restrict__ bid,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ v,
                                                           const real* __restrict__ stress,
                                                           double* __restrict__ partials)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kObsTerms];
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) acc[q] = 0.0;
    if (s < n && bid[s] < n_owned) {
        const double xs[3] = {x[s], x[n + s], x[2 * (size_t)n + s]};
        const double vs[3] = {v[s], v[n + s], v[2 * (size_t)n + s]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            acc[d] = vs[d];
            acc[3 + d] = vs[d] * vs[d];
            acc[15 + d] = xs[d];
        }
        if (stress) {
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[6 + q] = (double)stress[(size_t)q * n + s];
        }
        acc[18] = xs[1] * vs[2] - xs[2] * vs[1];
        acc[19] = -xs[0] * vs[2] + xs[2] * vs[0];
        acc[20] = xs[0] * vs[1] - xs[1] * vs[0];
    }
    __shared__ double red[8][kObsTerms];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q) {
        double a = acc[q];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) red[wid][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < kObsTerms) {
        double a = 0.0;
        for (int w = 0; w < 8; ++w) a += red[w][threadIdx.x];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = a;
    }
}

// ---------------------------------------------------------- topology filter

// The whole box's topology, by bond and bond-pair index and by bead id.
struct SlabTopo {
    int nb, na, id_max;
    const int* head_id;     // per bond
    const int* tail_id;
    const int* first;       // per bond pair: its first and second bond
    const int* second;
    const int* gptr;        // per bead id 1..id_max: its terms (index*8 + code) in
    const int* gterm;       // the single-box build's order (bonds, then bond pairs)
};

// idmap[id] = (version << 32) | upload index of the local bead with that id
// (ids above id_max belong to no bond).
__global__ void __launch_bounds__(256) k_slab_idmap(int n, int id_max, const int* __restrict__ pid_of,
                                                    unsigned version, unsigned long long* __restrict__ idmap)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int id = pid_of[b];
    if (id >= 1 && id <= id_max) idmap[id] = ((unsigned long long)version << 32) | (unsigned)b;
}

__device__ __forceinline__ int slab_lookup(const unsigned long long* __restrict__ idmap, unsigned version, int id)
{
    const unsigned long long e = idmap[id];
    return (unsigned)(e >> 32) == version ? (int)(unsigned)e : -1;
}

// Upload indices of every bond's and bond pair's beads (-1: not in the local box).
__global__ void __launch_bounds__(256) k_slab_endpoints(SlabTopo T, const unsigned long long* __restrict__ idmap,
                                                        unsigned version, int* __restrict__ bond_h,
                                                        int* __restrict__ bond_t, int* __restrict__ a0,
                                                        int* __restrict__ a1, int* __restrict__ a2,
                                                        int* __restrict__ a3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < T.nb) {
        bond_h[i] = slab_lookup(idmap, version, T.head_id[i]);
        bond_t[i] = slab_lookup(idmap, version, T.tail_id[i]);
    }
    if (i < T.na) {
        const int f = T.first[i], s2 = T.second[i];
        a0[i] = slab_lookup(idmap, version, T.head_id[f]);    // first bond's head (middle bead)
        a1[i] = slab_lookup(idmap, version, T.tail_id[f]);    // first bond's tail
        a2[i] = slab_lookup(idmap, version, T.head_id[s2]);   // second bond's head
        a3[i] = slab_lookup(idmap, version, T.tail_id[s2]);   // second bond's tail
    }
}

__device__ __forceinline__ bool slab_term_present(int term, const int* __restrict__ bond_h,
                                                  const int* __restrict__ bond_t, const int* __restrict__ a0,
                                                  const int* __restrict__ a1, const int* __restrict__ a2,
                                                  const int* __restrict__ a3)
{
    const int code = term & 7, idx = term >> 3;
    if (code <= kBondTail) return bond_h[idx] >= 0 && bond_t[idx] >= 0;
    return a0[idx] >= 0 && a1[idx] >= 0 && a2[idx] >= 0 && a3[idx] >= 0;
}

// Terms of each local bead whose beads are all local (per upload index).  An
// owned bead must keep every term (its partners lie within the ghost
// layers); one that loses a term sets DPD_STATUS_SLAB_REACH (fatal): a bond
// reaches beyond the ghost layers.
__global__ void __launch_bounds__(256) k_slab_term_count(int n, int n_owned, SlabTopo T,
                                                         const int* __restrict__ pid_of,
                                                         const int* __restrict__ bond_h,
                                                         const int* __restrict__ bond_t, const int* __restrict__ a0,
                                                         const int* __restrict__ a1, const int* __restrict__ a2,
                                                         const int* __restrict__ a3, int* __restrict__ cnt,
                                                         unsigned* __restrict__ status)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int id = pid_of[b];
    int c = 0, all = 0;
    if (id >= 1 && id <= T.id_max) {
        all = T.gptr[id + 1] - T.gptr[id];
        for (int t = T.gptr[id]; t < T.gptr[id + 1]; ++t)
            c += slab_term_present(T.gterm[t], bond_h, bond_t, a0, a1, a2, a3);
    }
    cnt[b] = c;
    if (b < n_owned && c != all) atomicOr(status, kStatusSlabReach);
}

__global__ void __launch_bounds__(256) k_slab_term_write(int n, SlabTopo T, const int* __restrict__ pid_of,
                                                         const int* __restrict__ bond_h,
                                                         const int* __restrict__ bond_t, const int* __restrict__ a0,
                                                         const int* __restrict__ a1, const int* __restrict__ a2,
                                                         const int* __restrict__ a3, const int* __restrict__ csr_ptr,
                                                         int* __restrict__ csr_term, int cap)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int id = pid_of[b];
    int o = csr_ptr[b];
    if (id >= 1 && id <= T.id_max)
        for (int t = T.gptr[id]; t < T.gptr[id + 1]; ++t) {
            const int term = T.gterm[t];
            // (a bead id uploaded twice could list a term twice: never past the array)
            if (slab_term_present(term, bond_h, bond_t, a0, a1, a2, a3) && o < cap) csr_term[o++] = term;
        }
}

__global__ void __launch_bounds__(256) k_iota(int n, int* __restrict__ a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// ------------------------------------------------------------ exclusive scan
// out[0..n] = exclusive prefix sums of in[0..n) (out[n] = the total), in three
// launches: block sums, one block scanning them, per-block application.

__global__ void __launch_bounds__(256) k_scan_block_sums(int n, const int* __restrict__ in, int* __restrict__ bsum)
{
    __shared__ int ws[8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int v = i < n ? in[i] : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < 8; ++w) s += ws[w];
        bsum[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(1024) k_scan_top(int nblocks, int* __restrict__ bsum)
{
    __shared__ int wsum[32];
    __shared__ int carry;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nblocks; base += 1024) {
        const int i = base + t;
        const int v = i < nblocks ? bsum[i] : 0;
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            int ws = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            wsum[lane] = ws;
        }
        __syncthreads();
        const int before = carry + (wid ? wsum[wid - 1] : 0) + inc - v;
        if (i < nblocks) bsum[i] = before;
        __syncthreads();
        if (t == 1023) carry = before + v;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_scan_apply(int n, const int* __restrict__ in, const int* __restrict__ bsum,
                                                    int* __restrict__ out)
{
    __shared__ int ws[8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int v = i < n ? in[i] : 0;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) ws[wid] = inc;
    __syncthreads();
    int before = bsum[blockIdx.x];
    for (int w = 0; w < wid; ++w) before += ws[w];
    before += inc - v;
    if (i < n) out[i] = before;
    if (i == n - 1) out[n] = before + v;
}

}  // namespace dpd
