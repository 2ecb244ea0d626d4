// Device helpers shared by the kernel sources (vlj_grid.cu, vlj_forces.cu).
#pragma once

#include <cuda_runtime.h>

#include "vlj_internal.cuh"

namespace vlj {

// Host side: grid size for n threads, and launch bookkeeping (vlj_grid.cu).
inline unsigned blocks_for(uint64_t n, int threads = kBlock) {
    uint64_t b = (n + (uint64_t)threads - 1) / (uint64_t)threads;
    return b ? (unsigned)b : 1u;
}
cudaError_t after_launch(unsigned n = 1);
// Streaming multiprocessors of the current device (cached per device): the
// grid of the kernels that loop over the step's work list.
int sm_count();
cudaError_t launch_build_list(const Arena& a, cudaStream_t s);  // vlj_build.cu

__device__ __forceinline__ uint32_t box_of_slot(const Arena& a, uint32_t slot) {
    return a.box_of_slot ? a.box_of_slot[slot] : 0u;
}

__device__ __forceinline__ uint32_t box_of_cell(const Arena& a, uint32_t cell) {
    return a.box_of_cell ? a.box_of_cell[cell] : 0u;
}

// Every kernel counts its own launch once, so the number of this library's
// kernels that ran (graph nodes skipped by a condition do not) is exact.
__device__ __forceinline__ void count_kernel(const Arena& a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.glob->kernels, 1ull);
}

// A step starts: the decision taken for it (if a step kernel took it) is
// used up. Block 0 clears the flag before it counts itself finished, so the
// last block's decision for the next step lands after the clear.
__device__ __forceinline__ void consume_decision(const Arena& a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) a.glob->decided = 0u;
}

__device__ __forceinline__ bool rebuilding(const Arena& a, uint32_t b) {
    return a.ctrl[b].rebuild != 0u;
}

// The step's work list: its length, and entry t (the dense cells first).
__device__ __forceinline__ uint32_t work_total(const Arena& a) {
    return a.glob->work_front + a.glob->work_back;
}

__device__ __forceinline__ uint32_t work_item(const Arena& a, uint32_t front, uint32_t t) {
    return t < front ? a.work[t] : a.work[a.work_cap - 1u - (t - front)];
}

// A box under five cells wide on some axis: the list build tests on encoded
// words there, and splits each cell's home particles into parts.
__device__ __forceinline__ bool narrow_box(const Box& bx) {
    return bx.cells[0] < 5u || bx.cells[1] < 5u || bx.cells[2] < 5u;
}

// Work-list entries of a cell of m particles.
__device__ __forceinline__ uint32_t cell_parts(uint32_t m, bool narrow) {
    if (m == 0u) return 0u;
    return narrow ? min(kMaxParts, (m + kPartHomes - 1u) / kPartHomes) : 1u;
}

// ---- cell tiles (tile_step_kernel, and the list build that indexes them) ----
// A brick is cells x0 .. x0 + w - 1 of the x-row (y, z) of a box. Its tile is
// the nine x-rows (y + dy, z + dz), dz, dy = -1..1 in that order, each over
// the rx cells x_start, x_start + 1, ... (mod nx): the whole row when the row
// is one brick, else the brick's cells and one more on each side. Each cell
// brings its particles in sorted order, so the tile holds every home
// particle's neighbour cells, and the cells of one row are at most two runs
// of the sorted order.
struct Brick {
    uint32_t x0, w, rx, x_start;
    uint32_t y, z;
    bool full;  // the row is one brick
};

// Bricks per x-row r_n = brick_cols: widths nx / r_n, the first nx % r_n one more.
__device__ __forceinline__ void brick_span(const Box& bx, uint32_t r, uint32_t& x0, uint32_t& w) {
    const uint32_t nx = bx.cells[0], cols = bx.brick_cols;
    const uint32_t q = nx / cols, rem = nx % cols;
    w = q + (r < rem ? 1u : 0u);
    x0 = r * q + min(r, rem);
}

__device__ __forceinline__ uint32_t brick_col_of(const Box& bx, uint32_t cx) {
    const uint32_t nx = bx.cells[0], cols = bx.brick_cols;
    const uint32_t q = nx / cols, rem = nx % cols;
    const uint32_t wide = rem * (q + 1u);
    return cx < wide ? cx / (q + 1u) : rem + (cx - wide) / q;
}

__device__ __forceinline__ Brick make_brick(const Box& bx, uint32_t r, uint32_t y, uint32_t z) {
    Brick k;
    brick_span(bx, r, k.x0, k.w);
    k.y = y;
    k.z = z;
    k.full = bx.brick_cols == 1u;
    const uint32_t nx = bx.cells[0];
    k.rx = k.full ? nx : k.w + 2u;
    k.x_start = k.full ? 0u : (k.x0 + nx - 1u) % nx;
    return k;
}

// Brick `index` of a box: (z * ny + y) * brick_cols + r.
__device__ __forceinline__ Brick brick_at(const Box& bx, uint32_t index) {
    const uint32_t cols = bx.brick_cols;
    const uint32_t r = index % cols, yz = index / cols;
    return make_brick(bx, r, yz % bx.cells[1], yz / bx.cells[1]);
}

// First cell of tile row rho (0..8: dz = rho / 3 - 1, dy = rho % 3 - 1).
__device__ __forceinline__ uint32_t tile_row_cell(const Box& bx, const Brick& k, uint32_t rho) {
    const uint32_t ny = bx.cells[1], nz = bx.cells[2];
    const uint32_t y = (k.y + ny + (rho % 3u) - 1u) % ny;
    const uint32_t z = (k.z + nz + (rho / 3u) - 1u) % nz;
    return bx.cell_base + (z * ny + y) * bx.cells[0];
}

// Particles in the first xp cells of a tile row whose cells start at `row`
// (xp <= rx): one run of the sorted order, or two where the row wraps.
__device__ __forceinline__ uint32_t tile_row_prefix(const uint32_t* __restrict__ cs,
                                                    const Box& bx, const Brick& k, uint32_t row,
                                                    uint32_t xp) {
    const uint32_t nx = bx.cells[0];
    const uint32_t end = k.x_start + xp;
    if (end <= nx) return cs[row + end] - cs[row + k.x_start];
    return cs[row + nx] - cs[row + k.x_start] + cs[row + end - nx] - cs[row];
}

// Tile column of home cell cx's neighbour at dx (-1, 0, 1).
__device__ __forceinline__ uint32_t tile_col(const Box& bx, const Brick& k, uint32_t cx, int32_t dx) {
    const uint32_t nx = bx.cells[0];
    return k.full ? (cx + nx + (uint32_t)dx) % nx : cx - k.x0 + 1u + (uint32_t)dx;
}

// Whether the cell grid is rebuilt this step: with the lists, or on every
// step when grid_every_step is set (a single box).
__device__ __forceinline__ bool grid_pass(const Arena& a) {
    return a.glob->any != 0u || a.glob->grid_every_step != 0u;
}

// ---- decide (lennard_jones.wgsl:281-307), by one whole block ----
// Finishes the previous step's bookkeeping (flip the position copy, advance
// the step counter), then per box: rebuild when something moved more than
// skin / 2 since the last build, or never built; reorder on every
// reorder_every-th rebuild (counted before the increment, as the reference).
// With `set`, the decision (some box rebuilds) becomes the value of the graph
// conditional `handle`.
// A step kernel's last block takes the next step's decision itself
// (`folded`) and leaves Global::decided set; the step that follows consumes
// it (its step kernel clears the flag). A decide that finds such a decision
// not yet consumed keeps it -- the displacements it came from were reset --
// and only adds the boxes whose rebuild was forced since.
__device__ __forceinline__ void decide_block(const Arena& a, cudaGraphConditionalHandle handle,
                                             bool set, bool folded = false) {
    __shared__ int s_any, s_keep;
    Global* g = a.glob;
    if (threadIdx.x == 0) {
        s_any = 0;
        s_keep = !folded && g->decided != 0u;
        g->decided = folded ? 1u : 0u;
        g->work_front = 0u;
        g->work_back = 0u;
        g->next_build = 0u;
        if (g->pending) {
            g->phase ^= 1u;
            g->step += 1ull;
            g->pending = 0u;
        }
    }
    __syncthreads();
    const bool keep = s_keep != 0;
    for (uint32_t b = threadIdx.x; b < a.nboxes; b += blockDim.x) {
        Control& c = a.ctrl[b];
        const Box& bx = a.boxes[b];
        if (keep && c.rebuild) {
            // decided at the end of the last step
            c.forced = 0u;
            s_any = 1;
            continue;
        }
        const float moved = keep ? 0.0f : __uint_as_float(c.max_disp);
        if (!keep) c.max_disp = 0u;
        const bool rebuild = moved > bx.half_skin2 || c.built == 0u || c.forced != 0u;
        c.forced = 0u;
        c.rebuild = rebuild ? 1u : 0u;
        if (rebuild) {
            c.reorder = (c.rebuilds % bx.reorder_every == 0u) ? 1u : 0u;
            c.rebuilds += 1u;
            c.built = 1u;
            s_any = 1;
        } else {
            c.reorder = 0u;
        }
    }
    __syncthreads();
    if (a.nboxes == 1u) {
        if (threadIdx.x == 0) {
            // the particles the grid kernels cover: the box's, when its lists
            // rebuild or its grid is rebuilt every step
            const bool r = a.ctrl[0].rebuild != 0u || g->grid_every_step != 0u;
            a.rb_box[0] = 0u;
            a.rb_first[0] = 0u;
            a.rb_first[r ? 1 : 0] = r ? a.boxes[0].n : 0u;
            g->rb_boxes = r ? 1u : 0u;
            g->rb_slots = r ? a.boxes[0].n : 0u;
            g->any = (uint32_t)s_any;
            if (set) cudaGraphSetConditional(handle, (unsigned)s_any);
        }
        return;
    }
    // the rebuilding boxes, compacted in box order, with their particle counts
    // summed before each: two block-wide exclusive scans per pass
    __shared__ uint32_t s_wbox[32], s_wslot[32], s_cbox, s_cslot;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    if (threadIdx.x == 0) s_cbox = s_cslot = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < a.nboxes; base += blockDim.x) {
        const uint32_t b = base + threadIdx.x;
        const bool flag = b < a.nboxes && a.ctrl[b].rebuild != 0u;
        const uint32_t nb = flag ? a.boxes[b].n : 0u;
        uint32_t ib = flag ? 1u : 0u, is = nb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t tb = __shfl_up_sync(0xffffffffu, ib, o);
            const uint32_t ts = __shfl_up_sync(0xffffffffu, is, o);
            if (lane >= (uint32_t)o) {
                ib += tb;
                is += ts;
            }
        }
        if (lane == 31u) {
            s_wbox[warp] = ib;
            s_wslot[warp] = is;
        }
        __syncthreads();
        uint32_t pb = s_cbox, ps = s_cslot;
        for (uint32_t w = 0; w < warp; w++) {
            pb += s_wbox[w];
            ps += s_wslot[w];
        }
        if (flag) {
            const uint32_t k = pb + ib - 1u;
            a.rb_box[k] = b;
            a.rb_first[k] = ps + is - nb;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (uint32_t w = 0; w < warps; w++) {
                s_cbox += s_wbox[w];
                s_cslot += s_wslot[w];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.rb_first[s_cbox] = s_cslot;
        g->rb_boxes = s_cbox;
        g->rb_slots = s_cslot;
        g->any = (uint32_t)s_any;
        if (set) cudaGraphSetConditional(handle, (unsigned)s_any);
    }
}

// Runs body(slot, box) for every particle of the boxes that rebuild this step
// (Global::rb_slots of them), over a resident grid: each block takes 256
// consecutive particles of the compacted list at a time, finds the first one's
// box by bisection, and its threads step on from there. Every thread of the
// block must call this.
template <class F>
__device__ __forceinline__ void for_rebuild_slots(const Arena& a, F body) {
    __shared__ uint32_t s_k0;
    const uint32_t total = a.glob->rb_slots, boxes = a.glob->rb_boxes;
    for (uint32_t start = blockIdx.x * blockDim.x; start < total; start += gridDim.x * blockDim.x) {
        if (threadIdx.x == 0) {
            uint32_t lo = 0, hi = boxes;  // last k with rb_first[k] <= start
            while (hi - lo > 1u) {
                const uint32_t m = (lo + hi) >> 1;
                if (a.rb_first[m] <= start) lo = m; else hi = m;
            }
            s_k0 = lo;
        }
        __syncthreads();
        const uint32_t t = start + threadIdx.x;
        if (t < total) {
            uint32_t k = s_k0;
            while (a.rb_first[k + 1] <= t) k++;
            const uint32_t b = a.rb_box[k];
            body(a.boxes[b].first + (t - a.rb_first[k]), b);
        }
        __syncthreads();
    }
}

// Whether every valid thread of the block belongs to the box of the block's
// first slot; that box in *ref. Call from every thread of the block.
__device__ __forceinline__ bool block_in_one_box(const Arena& a, bool valid, uint32_t b,
                                                 uint32_t first_slot, uint32_t* ref) {
    __shared__ uint32_t s_ref;
    __shared__ int s_mixed;
    if (threadIdx.x == 0) {
        s_mixed = 0;
        s_ref = box_of_slot(a, first_slot);
    }
    __syncthreads();
    if (valid && b != s_ref) s_mixed = 1;
    __syncthreads();
    *ref = s_ref;
    return s_mixed == 0;
}

// Largest value over the block into each box's max_disp: one atomicMax when
// the block lies in one box (the usual case), one per thread otherwise.
__device__ __forceinline__ void block_max_per_box(const Arena& a, bool valid, uint32_t b,
                                                  uint32_t first_slot, float value) {
    __shared__ uint32_t s_val[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t bits = valid ? __float_as_uint(value) : 0u;
    uint32_t ref;
    if (!block_in_one_box(a, valid, b, first_slot, &ref)) {
        if (valid) atomicMax(&a.ctrl[b].max_disp, bits);
        return;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bits = max(bits, __shfl_xor_sync(0xffffffffu, bits, o));
    if (lane == 0) s_val[warp] = bits;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = max(m, s_val[w]);
        atomicMax(&a.ctrl[ref].max_disp, m);
    }
}

// Sum of kSlots 64-bit integers over the block into each box's accumulators,
// with the same one-box shortcut. Integer sums: the order does not matter.
__device__ __forceinline__ void block_sum_slots(const Arena& a, bool valid, uint32_t b,
                                                uint32_t first_slot, long long (&v)[kSlots]) {
    __shared__ long long s_sum[kBlock / 32][kSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t ref;
    if (!block_in_one_box(a, valid, b, first_slot, &ref)) {
        if (valid)
            for (int k = 0; k < kSlots; k++)
                if (v[k]) atomicAdd(&a.accum[b * kSlots + k], (unsigned long long)v[k]);
        return;
    }
#pragma unroll
    for (int k = 0; k < kSlots; k++) {
        long long x = valid ? v[k] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) s_sum[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < kSlots) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_sum[w][threadIdx.x];
        if (t) atomicAdd(&a.accum[ref * kSlots + threadIdx.x], (unsigned long long)t);
    }
}

// Error-free sum s + e = a + b (Knuth's two-sum; df64.rs:15-22).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// One Nose-Hoover half step of (xi, eta) (lennard_jones.wgsl:341-377): xi a
// quarter step with the kinetic energy ke, the velocity scale
// s = exp(-xi dt / 2), eta a half step, xi another quarter step with the
// kinetic energy after scaling. Returns s; ke becomes ke s^2.
__device__ __forceinline__ double nh_half(const Box& bx, double& xi, double& eta, double& ke) {
    const double quarter = 0.5 * bx.half_dt;
    xi += (2.0 * ke - bx.nh_gkt) / bx.nh_q * quarter;
    const double s = exp(-xi * bx.half_dt);
    eta += xi * bx.half_dt;
    ke = ke * s * s;
    xi += (2.0 * ke - bx.nh_gkt) / bx.nh_q * quarter;
    return s;
}

// Canonical velocity component k of slot i: the stored one plus the closing
// half kick (velocities half a kick behind), or the stored one itself when the
// box keeps canonical velocities -- times Nose-Hoover's pending end-half scale.
__device__ __forceinline__ double canonical_velocity(const Arena& a, const Box& bx, uint32_t b,
                                                     uint32_t i, int k, float acc) {
    const double v = a.v[(size_t)k * a.seg + i];
    if (bx.canonical) return bx.thermostat == 2 ? v * a.nh[b].scale : v;
    return v + (double)acc * bx.half_dt;
}

// Periodic wrap of an f64 coordinate that moved less than one side.
__device__ __forceinline__ double wrap(double x, double side) {
    if (x >= side) x -= side;
    if (x < 0.0) x += side;
    if (x >= side) x -= side;
    return x;
}

}  // namespace vlj
