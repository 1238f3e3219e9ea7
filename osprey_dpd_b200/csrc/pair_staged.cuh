// pair_staged.cuh -- half-shell DPD pair forces (CCNTCell::UpdateForce, DPD
// branch, CNTCell.cpp:1103-1572) with each tile's neighbour rows staged in
// shared memory.
//
// A tile is kPairBlock consecutive slots of the cell-sorted layout.  Its beads
// lie in one or more "home rows" (cells of one (y, z), consecutive in x).  For
// every home row the block copies five windows of the cell grid into shared
// memory with coalesced loads:
//
//   r = 0  row (y,   z)   cells xa-1 .. xb+1   (own cell after i, and cell x+1)
//   r = 1  row (y+1, z)   cells xa-1 .. xb+1
//   r = 2  row (y-1, z+1) cells xa-1 .. xb+1
//   r = 3  row (y,   z+1) cells xa-1 .. xb+1
//   r = 4  row (y+1, z+1) cells xa-1 .. xb+1
//
// where xa..xb are the x columns of the tile's beads in that row.  The copy is
// in logical x order (a window that crosses the periodic x boundary is copied
// as up to three slot ranges), so the candidates of a bead in cell x are ONE
// contiguous range per window: cells x-1, x, x+1.  The 14 cells are the half
// shell (each unordered cell pair once) of the engine's half-shell scheme.
//
// Staged x is stored relative to the window's first cell (x_w = x_loc +
// l * w), so the distance test needs no per-candidate cell shift; the force
// itself is recomputed from the exact cell-relative coordinates, with the x
// cell offset recovered as rint((x_loc,i - x_loc,j - (x_w,i - x_w,j)) / w).
// The test's rounding (~4e-6 at 45 cells) only decides pairs within that
// distance of the cut-off, where the force is below a_ij * 4e-6; the exact
// cut-off is re-applied in the force evaluation.
//
// Test phase: one lane per home bead walks its five windows and appends hits
// (staged index + window) to its own list column in shared memory.  Force
// phase: balanced_force_pass (pair_forces.cuh), the warp's hits cut into 32
// equal runs.  F (and on sample steps the stress array) must be zero on
// entry.
//
// A tile whose windows do not fit (more than kStgRows home rows, more staged
// beads or table entries than the buffers hold) is evaluated by the unstaged
// half-shell tile code instead, so any bead distribution is handled.
//
// Measured on a B200 this scheme is slower than the unstaged half shell: the
// per-tile staging (block barriers and dependent global round trips of the
// row geometry with four-warp blocks) costs more than the shared-memory
// candidate loads save.  It stays selectable (DPD_PAIR_STAGED) for that
// comparison.
#pragma once
#include "pair_forces.cuh"

namespace dpd {

constexpr int kStgRows = 25;                 // home rows per tile (5 windows each, one thread per window)
constexpr int kStgWin = 5 * kStgRows;
static_assert(kStgWin <= kPairBlock, "one thread per window");
constexpr int kStgCells = 768;               // window cell-offset table entries per tile
template <typename real> struct StgCap { static constexpr int value = sizeof(real) == 4 ? 1280 : 896; };
template <typename real> struct StgOcc { static constexpr int value = sizeof(real) == 4 ? 5 : 4; };

// Byte offsets of the dynamic shared memory of k_pair_forces_staged.
template <typename real>
struct StgLayout {
    size_t tabs, stg, hpos, hvel, hxw, lists, coff, total;
    __host__ __device__ StgLayout(int nt, int hitcap, bool multi)
    {
        const size_t v4 = 4 * sizeof(real);
        size_t o = 0;
        tabs = o; o += multi ? 0 : pair_tables_bytes<real>(nt);
        stg = o; o += v4 * StgCap<real>::value;
        hpos = o; o += v4 * kPairBlock;
        hvel = o; o += v4 * kPairBlock;
        hxw = o; o += ((sizeof(real) * kPairBlock + 15) / 16) * 16;
        lists = o; o += sizeof(uint32_t) * (size_t)(hitcap + 1) * kPairBlock;   // + the spare row of half_shell_tile
        coff = o; o += sizeof(int) * kStgCells;
        total = o;
    }
};

template <typename real, bool VIRIAL, bool MULTI>
__global__ void __launch_bounds__(kPairBlock, StgOcc<real>::value) k_pair_forces_staged(
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
    __shared__ int key_s[kPairBlock];
    __shared__ int wtmp_s[kPairWarps];
    __shared__ long long wscan_s[kPairWarps];
    __shared__ int rkey_s[kStgRows], rxa_s[kStgRows], rxb_s[kStgRows], rbox_s[kStgRows];
    __shared__ int wrc_s[kStgWin], wcf_s[kStgWin], wms_s[kStgWin], wmid_s[kStgWin], wtot_s[kStgWin];
    __shared__ int wbase_s[kStgWin], tbase_s[kStgWin];
    __shared__ int wcnt_s[kPairBlock], wexc_s[kPairBlock];

    const int nt = K->ntypes;
    const StgLayout<real> L(nt, hitcap, MULTI);
    real* Tsh = reinterpret_cast<real*>(pair_dyn + L.tabs);
    V4* stg = reinterpret_cast<V4*>(pair_dyn + L.stg);
    V4* hpos = reinterpret_cast<V4*>(pair_dyn + L.hpos);
    V4* hvel = reinterpret_cast<V4*>(pair_dyn + L.hvel);
    real* hxw = reinterpret_cast<real*>(pair_dyn + L.hxw);
    uint32_t* lists = reinterpret_cast<uint32_t*>(pair_dyn + L.lists);
    int* coff = reinterpret_cast<int*>(pair_dyn + L.coff);
    const HalfShared<real> sh{hpos, hvel, hxw, wcnt_s, wexc_s};
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int cap = StgCap<real>::value;
    if (!MULTI)
        for (int k = t; k < 3 * nt * nt; k += kPairBlock) Tsh[k] = tab[k];
    const int64_t step = *step_ptr;
    uint32_t keys0[10];
    {
        uint32_t k = philox_step_key(boxes[0].seed, step);
#pragma unroll
        for (int q = 0; q < 10; ++q) { keys0[q] = k; k += 0x9E3779B9u; }
    }
    const int tile0 = blockIdx.x * tiles_per_block;
    for (int tile = tile0; tile < tile0 + tiles_per_block; ++tile) {
        if (tile * kPairBlock >= n) break;
        __syncthreads();   // the previous tile is done with the shared buffers (and the tables are in)
        const int i = tile * kPairBlock + t;
        const bool live = i < n;
        V4 pi, vi;
        int c = 0;
        if (live) {
            pi = pos4[i];
            vi = vel4[i];
            c = cell[i];
        } else {
            pi.x = pi.y = pi.z = pi.w = vi.x = vi.y = vi.z = vi.w = real(0);
        }
        const int bx = MULTI ? flag_box(real_bits(pi.w)) : 0;
        const Box& B = boxes[bx];
        int cx = 0, rowkey = -1;
        if (live) {
            const int cl = c - B.cell_base;
            cx = cl % B.nc[0];
            rowkey = c - cx;   // global index of the row's x = 0 cell
        }
        key_s[t] = rowkey;
        __syncthreads();
        // home rows: slots are cell-sorted, so a row's beads are consecutive
        const bool first = live && (t == 0 || key_s[t - 1] != rowkey);
        const bool last = live && (t == kPairBlock - 1 || key_s[t + 1] != rowkey);
        const unsigned fb = __ballot_sync(0xffffffffu, first);
        if (lane == 0) wtmp_s[warp] = __popc(fb);
        __syncthreads();
        int H = 0, before = 0;
#pragma unroll
        for (int w = 0; w < kPairWarps; ++w) {
            const int v = wtmp_s[w];
            H += v;
            before += w < warp ? v : 0;
        }
        if (H > kStgRows) {   // block-uniform
            half_shell_tile<real, VIRIAL, MULTI, kPairBlock>(tile, n, nt, boxes, step, tab, Tsh, cell, start, pos4,
                                                             vel4, F, stress, hitcap, lists, sh, keys0, xs);
            continue;
        }
        const int h = before + __popc(fb & ((2u << lane) - 1u)) - 1;
        if (first) { rkey_s[h] = rowkey; rxa_s[h] = cx; rbox_s[h] = bx; }
        if (last) rxb_s[h] = cx;
        __syncthreads();
        // window geometry, one thread per window w = 5 * row + r
        int wtot = 0, wtab = 0;
        if (t < 5 * H) {
            const int hh = t / 5, r = t - 5 * hh;
            const Box& Bh = boxes[rbox_s[hh]];
            const int hnx = Bh.nc[0], hny = Bh.nc[1], hnz = Bh.nc[2];
            const int xa = rxa_s[hh], xb = rxb_s[hh];
            const int rl = (rkey_s[hh] - Bh.cell_base) / hnx;
            int dy, dz;
            stg_row_shift(r, dy, dz);
            int y2 = rl % hny + dy, z2 = rl / hny + dz;
            y2 += y2 < 0 ? hny : (y2 >= hny ? -hny : 0);
            z2 += z2 >= hnz ? -hnz : 0;
            const int rc = Bh.cell_base + hnx * (y2 + hny * z2);
            const int m0 = max(xa - 1, 0), m1 = min(xb + 1, hnx - 1);
            // pieces in logical x order: cell nx-1 when xa = 0, cells m0..m1, cell 0 when xb = nx-1
            const int cf = xa == 0 ? start[rc + hnx] - start[rc + hnx - 1] : 0;
            const int ms = start[rc + m0];
            const int mid = start[rc + m1 + 1] - ms;
            const int cb = xb == hnx - 1 ? start[rc + 1] - start[rc] : 0;
            wtot = cf + mid + cb;
            wtab = xb - xa + 4;   // logical cells xa-1 .. xb+1 and the end
            wrc_s[t] = rc; wcf_s[t] = cf; wms_s[t] = ms; wmid_s[t] = mid; wtot_s[t] = wtot;
        }
        // block exclusive scan of (staged beads, table entries); beads clamped
        // to cap + 1 so the packed sum cannot carry into the table count
        const long long pv = ((long long)min(wtot, cap + 1) << 32) | (long long)wtab;
        long long inc = pv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wscan_s[warp] = inc;
        __syncthreads();
        long long wb0 = 0, all = 0;
#pragma unroll
        for (int w = 0; w < kPairWarps; ++w) {
            const long long v = wscan_s[w];
            all += v;
            wb0 += w < warp ? v : 0;
        }
        const int S = (int)(all >> 32), NT = (int)(all & 0xFFFFFFFFll);
        if (S > cap || NT > kStgCells) {   // block-uniform
            half_shell_tile<real, VIRIAL, MULTI, kPairBlock>(tile, n, nt, boxes, step, tab, Tsh, cell, start, pos4,
                                                             vel4, F, stress, hitcap, lists, sh, keys0, xs);
            continue;
        }
        if (t < 5 * H) {
            const long long ex = wb0 + inc - pv;
            wbase_s[t] = (int)(ex >> 32);
            tbase_s[t] = (int)(ex & 0xFFFFFFFFll);
        }
        __syncthreads();
        // cell-offset tables and the staged copy, one warp per window
        for (int w = warp; w < 5 * H; w += kPairWarps) {
            const int hh = w / 5;
            const Box& Bh = boxes[rbox_s[hh]];
            const int hnx = Bh.nc[0];
            const int xa = rxa_s[hh], xb = rxb_s[hh];
            const int rc = wrc_s[w], cf = wcf_s[w], ms = wms_s[w], mid = wmid_s[w], tw = wtot_s[w];
            const int wb = wbase_s[w], tb = tbase_s[w];
            const int m1 = min(xb + 1, hnx - 1);
            for (int l = lane; l <= xb - xa + 3; l += 32) {
                const int x = xa - 1 + l;
                const int off = x < 0 ? 0 : (x <= m1 + 1 ? cf + start[rc + x] - ms : tw);
                coff[tb + l] = wb + off;
            }
            const real wxr = (real)Bh.w[0];
            const int fs = cf ? start[rc + hnx - 1] : 0;
            const int bs = tw > cf + mid ? start[rc] : 0;
            for (int k = lane; k < tw; k += 32) {
                int slot, lc;
                if (k < cf) {
                    slot = fs + k;
                    lc = 0;
                } else if (k < cf + mid) {
                    slot = ms + (k - cf);
                    lc = cell[slot] - rc - xa + 1;
                } else {
                    slot = bs + (k - cf - mid);
                    lc = hnx - xa + 1;
                }
                V4 p = pos4[slot];
                p.x += (real)lc * wxr;
                p.w = as_real_bits(slot, real(0));
                stg[wb + k] = p;
            }
        }
        const real wx = (real)B.w[0], wy = (real)B.w[1], wz = (real)B.w[2];
        const real w0[3] = {wx, wy, wz};
        int li = 0;
        real xwi = real(0);
        if (live) {
            li = cx - rxa_s[h] + 1;
            xwi = pi.x + (real)li * wx;
        }
        hpos[t] = pi;
        hvel[t] = vi;
        hxw[t] = xwi;
        __syncthreads();   // staged windows, tables and home beads are in place
        int ownpos = 0;
        if (live) ownpos = coff[tbase_s[5 * h] + li] + (i - start[c]);
        uint32_t* mylist = lists + t;
        int cnt = 0;
        for (int r = 0; r < 5; ++r) {
            int lo = 0, hi = 0;
            if (live) {
                const int tb = tbase_s[5 * h + r];
                hi = coff[tb + li + 2];
                lo = r == 0 ? ownpos + 1 : coff[tb + li - 1];
            }
            int dy, dz;
            stg_row_shift(r, dy, dz);
            const real py = pi.y - (real)dy * wy, pz = pi.z - (real)dz * wz;
            const uint32_t tag = (uint32_t)r << 12;
            const int len = hi - lo;
            const int trip = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(len, 0));
            for (int u = 0; u < trip; u += 2) {
                if (__any_sync(0xffffffffu, cnt > hitcap - 2)) {
                    balanced_force_pass<real, VIRIAL, MULTI, true>(cnt, lists, sh, stg, tile * kPairBlock, boxes,
                                                                   Tsh, tab, nt, keys0, w0, step, pos4, vel4, F,
                                                                   stress, n, xs);
                    cnt = 0;
                }
                const bool v0 = u < len, v1 = u + 1 < len;
                V4 s0, s1;
                if (v0) s0 = stg[lo + u];
                if (v1) s1 = stg[lo + u + 1];
                if (v0) {
                    const real ex = xwi - s0.x, ey = py - s0.y, ez = pz - s0.z;
                    const real r2 = ex * ex + ey * ey + ez * ez;
                    if (r2 < real(1) && r2 > real(1e-18)) {
                        mylist[cnt * kPairBlock] = (uint32_t)(lo + u) | tag;
                        ++cnt;
                    }
                }
                if (v1) {
                    const real ex = xwi - s1.x, ey = py - s1.y, ez = pz - s1.z;
                    const real r2 = ex * ex + ey * ey + ez * ez;
                    if (r2 < real(1) && r2 > real(1e-18)) {
                        mylist[cnt * kPairBlock] = (uint32_t)(lo + u + 1) | tag;
                        ++cnt;
                    }
                }
            }
        }
        balanced_force_pass<real, VIRIAL, MULTI, true>(cnt, lists, sh, stg, tile * kPairBlock, boxes, Tsh, tab, nt,
                                                       keys0, w0, step, pos4, vel4, F, stress, n, xs);
    }
}

}  // namespace dpd
