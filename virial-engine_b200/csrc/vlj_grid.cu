// CUDA kernels of the cell grid and the Verlet lists, sm_100a.
//
// A step starts with `decide` (one block: flip the position copy, pick the
// boxes that rebuild). The rebuild chain that follows -- bin, scan, scatter,
// per-cell order with the optional reorder, copy back, list build --
// sits under a conditional graph node, so it runs only on steps where some
// box crossed the skin / 2 trigger; launched directly, each kernel returns at
// once when nothing rebuilds. Reference kernels are cited at each kernel.
#include <cuda_runtime.h>

#include <atomic>

#include "vlj_device.cuh"
#include "vlj_internal.cuh"

namespace vlj {

static std::atomic<unsigned long long> g_launches{0};
unsigned long long launches() { return g_launches.load(); }

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

cudaError_t after_launch(unsigned n) {
    g_launches += n;
    return cudaGetLastError();
}

// ---- encode positions into the current cache copy ----
__global__ void encode_kernel(Arena a) {
    count_kernel(a);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    const Box& bx = a.boxes[box_of_slot(a, i)];
    uint4 w;
    w.x = encode(a.x[i], bx.enc[0]);
    w.y = encode(a.x[a.seg + i], bx.enc[1]);
    w.z = encode(a.x[2 * a.seg + i], bx.enc[2]);
    w.w = 0u;
    a.cache[a.glob->phase][i] = w;
}

// ---- particles in and out (lennard_jones.rs:1354-1374; input order) ----
__global__ void load_particles_kernel(Arena a) {
    count_kernel(a);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    const Box& bx = a.boxes[0];
    const double* p = a.aos + 6 * (size_t)i;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double x = p[k], v = p[3 + k];
        finite = finite && isfinite(x) && isfinite(v);
        // rem_euclid: fmod is exact, so this is the host's result to the bit
        double r = fmod(x, bx.box[k]);
        if (r < 0.0) r += bx.box[k];
        a.x[(size_t)k * a.seg + i] = r;
        a.v[(size_t)k * a.seg + i] = v;
    }
    a.id[i] = i;
    if (!finite) atomicCAS(&a.glob->fault, 0u, kFaultNonFinite);
}

__global__ void store_particles_kernel(Arena a) {
    count_kernel(a);
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nslots) return;
    double* p = a.aos + 6 * (size_t)a.id[s];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        p[k] = a.x[(size_t)k * a.seg + s];
        p[3 + k] = a.vcanon[(size_t)k * a.seg + s];
    }
}

// ---- decide (lennard_jones.wgsl:281-307) ----
// One block. Finishes the previous step's bookkeeping (flip the position
// copy, advance the step counter), then per box: rebuild when something moved
// more than skin / 2 since the last build, or never built; reorder on every
// reorder_every-th rebuild (counted before the increment, as the reference).
template <bool SET_CONDITION>
__global__ void decide_kernel(Arena a, cudaGraphConditionalHandle handle) {
    count_kernel(a);
    decide_block(a, handle, SET_CONDITION);
}

// ---- bin (grid.wgsl:11-38): cell of each slot from its f32 position ----
__global__ void bin_kernel(Arena a) {
    count_kernel(a);
    if (!grid_pass(a)) return;
    for_rebuild_slots(a, [&](uint32_t i, uint32_t b) {
        const Box& bx = a.boxes[b];
        int32_t c[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float hi = (float)a.x[k * a.seg + i];
            int32_t v = (int32_t)floorf(__fdiv_rn(hi, bx.cell_size_f[k]));
            int32_t m = (int32_t)bx.cells[k] - 1;
            c[k] = v < 0 ? 0 : (v > m ? m : v);
        }
        uint32_t cell = bx.cell_base +
            ((uint32_t)c[2] * bx.cells[1] + (uint32_t)c[1]) * bx.cells[0] + (uint32_t)c[0];
        a.cell_of_slot[i] = cell;
        atomicAdd(&a.count[cell], 1u);
#if !VLJ_LIST_STREAM
        // a force block wholly inside this box restarts its staged-row count
        if (i % kForceThreads == 0u && rebuilding(a, b)) {
            const uint32_t end = min(i + (uint32_t)kForceThreads, a.nslots);
            if (i >= bx.first && end <= bx.first + bx.n) a.block_rows[i / kForceThreads] = 0u;
        }
#endif
    });
}

// ---- scan (grid.wgsl:43-117): one block per box, exclusive prefix sum of
// the counts offset by the box's first slot; counts become zeroed cursors.
// The box's non-empty cells join the step's work list for the sort and the
// list build as entries cell * 8 + part: cells of kDenseCell particles or
// more at its front, the others at its back; in a narrow box every non-empty
// cell's parts (kPartHomes home particles each) at its front. Each warp takes
// kScanPer runs of 32 consecutive cells, a lane
// per cell, so every load and store of a run is one coalesced line; shuffles
// scan within the warp, warp 0 scans the warps' totals, and one atomic per
// block and class reserves its work-list entries.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 16;  // runs of 32 cells per warp: 16,384 cells per pass

__global__ void __launch_bounds__(kScanThreads) scan_kernel(Arena a) {
    count_kernel(a);
    if (!grid_pass(a)) return;
    const uint32_t b = blockIdx.x;
    if (b >= a.nboxes || !(rebuilding(a, b) || a.glob->grid_every_step)) return;
    const Box& bx = a.boxes[b];
    __shared__ uint32_t s_sum[kScanThreads / 32], s_nd[kScanThreads / 32], s_ns[kScanThreads / 32];
    __shared__ uint32_t s_carry, s_tile;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    if (threadIdx.x == 0) s_carry = bx.first;
    __syncthreads();
    const uint32_t total = bx.total_cells, base = bx.cell_base;
    const bool narrow = narrow_box(bx);
    for (uint32_t tile = 0; tile < total; tile += (uint32_t)kScanThreads * kScanPer) {
        const uint32_t first = tile + warp * 32u * (uint32_t)kScanPer;
        uint32_t excl[kScanPer];  // within the warp's cells, before this lane's
        // nibble r: front entries of this lane's cell of run r (its parts,
        // when it holds kDenseCell particles or more or the box is narrow)
        unsigned long long front_parts = 0ull;
        uint32_t sparse = 0;      // bit r: one back entry (a cell of fewer, but some)
        uint32_t sum = 0, nd = 0, ns = 0;
        // the runs that reach into the box (warp-uniform; a small box has
        // fewer cells than one pass covers)
        const uint32_t runs = first >= total ? 0u : min((uint32_t)kScanPer, (total - first + 31u) / 32u);
        // every run's count is read before the first shuffle, so the warp
        // waits for the loads once rather than once a run
#pragma unroll
        for (int r = 0; r < kScanPer; r++) {
            const uint32_t c = first + 32u * (uint32_t)r + lane;
            excl[r] = c < total ? a.count[base + c] : 0u;
        }
#pragma unroll
        for (int r = 0; r < kScanPer; r++) {
            if ((uint32_t)r >= runs) continue;
            const uint32_t v = excl[r];
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += t;
            }
            excl[r] = sum + x - v;
            sum += __shfl_sync(0xffffffffu, x, 31);
            if (narrow) {
                // every non-empty cell's parts go to the front
                const uint32_t parts = cell_parts(v, true);
                front_parts |= (unsigned long long)parts << (4 * r);
                nd += __reduce_add_sync(0xffffffffu, parts);
            } else {
                const bool d = v >= kDenseCell, sp = v != 0u && v < kDenseCell;
                front_parts |= (unsigned long long)(d ? 1u : 0u) << (4 * r);
                sparse |= (sp ? 1u : 0u) << r;
                nd += (uint32_t)__popc(__ballot_sync(0xffffffffu, d));
                ns += (uint32_t)__popc(__ballot_sync(0xffffffffu, sp));
            }
        }
        if (lane == 0) {
            s_sum[warp] = sum;
            s_nd[warp] = nd;
            s_ns[warp] = ns;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t ws = s_sum[lane], wd = s_nd[lane], wp = s_ns[lane];
            uint32_t is = ws, id = wd, ip = wp;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t ts = __shfl_up_sync(0xffffffffu, is, o);
                const uint32_t td = __shfl_up_sync(0xffffffffu, id, o);
                const uint32_t tp = __shfl_up_sync(0xffffffffu, ip, o);
                if (lane >= (uint32_t)o) {
                    is += ts;
                    id += td;
                    ip += tp;
                }
            }
            const uint32_t block_d = __shfl_sync(0xffffffffu, id, 31);
            const uint32_t block_p = __shfl_sync(0xffffffffu, ip, 31);
            uint32_t at_d = 0, at_p = 0;
            if (lane == 0 && block_d) at_d = atomicAdd(&a.glob->work_front, block_d);
            if (lane == 0 && block_p) at_p = atomicAdd(&a.glob->work_back, block_p);
            at_d = __shfl_sync(0xffffffffu, at_d, 0);
            at_p = __shfl_sync(0xffffffffu, at_p, 0);
            s_sum[lane] = is - ws;
            s_nd[lane] = at_d + id - wd;
            s_ns[lane] = at_p + ip - wp;
            if (lane == 31u) s_tile = is;
        }
        __syncthreads();
        const uint32_t before = s_carry + s_sum[warp];
        uint32_t at_d = s_nd[warp], at_p = s_ns[warp];
#pragma unroll
        for (int r = 0; r < kScanPer; r++) {
            if ((uint32_t)r >= runs) continue;
            const uint32_t c = first + 32u * (uint32_t)r + lane;
            if (c < total) {
                a.cell_start[base + c] = before + excl[r];
                a.count[base + c] = 0u;
            }
            // costly cells' parts from the front of the work list, the
            // others from its back
            const uint32_t kd = (uint32_t)(front_parts >> (4 * r)) & 15u;
            if (narrow) {
                // several parts a cell: an exclusive scan of the counts
                uint32_t incl = kd;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= (uint32_t)o) incl += t;
                }
                for (uint32_t q = 0; q < kd; q++) a.work[at_d + incl - kd + q] = (base + c) * 8u + q;
                at_d += __shfl_sync(0xffffffffu, incl, 31);
            } else {
                // one entry at most: a ballot ranks them
                const unsigned md = __ballot_sync(0xffffffffu, kd != 0u);
                if (kd) a.work[at_d + (uint32_t)__popc(md & below)] = (base + c) * 8u;
                at_d += (uint32_t)__popc(md);
            }
            const bool sp = (sparse >> r) & 1u;
            const unsigned mp = __ballot_sync(0xffffffffu, sp);
            if (sp) a.work[a.work_cap - 1u - (at_p + (uint32_t)__popc(mp & below))] = (base + c) * 8u;
            at_p += (uint32_t)__popc(mp);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += s_tile;
        __syncthreads();
    }
}

// ---- scatter (grid.wgsl:119-127): slot into its cell's next free place ----
__global__ void scatter_kernel(Arena a) {
    count_kernel(a);
    if (!grid_pass(a)) return;
    for_rebuild_slots(a, [&](uint32_t i, uint32_t) {
        const uint32_t c = a.cell_of_slot[i];
        a.sorted[a.cell_start[c] + atomicAdd(&a.count[c], 1u)] = i;
    });
}

// ---- per-cell order (grid.wgsl:129-148) ----
// A warp per cell of the step's work list (the resident grid's warps stride
// through it): each slot's rank is the number of smaller slots in the cell, so
// the cell ends up sorted by slot index whatever order the scatter's atomics
// produced. With reorder, every particle is also copied to the slot
// it takes in cell order (lennard_jones.wgsl:419-433).
constexpr int kSortRegs = 8;  // cells up to 256 particles rank in registers

__device__ __forceinline__ void move_to_scratch(const Arena& a, uint32_t from, uint32_t to,
                                                uint32_t cell) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        a.sx[k * a.seg + to] = a.x[k * a.seg + from];
        a.sv[k * a.seg + to] = a.v[k * a.seg + from];
    }
    a.sid[to] = a.id[from];
    a.scell[to] = cell;
}

// A cell of more than 32 particles: ranks in registers up to 32 * kSortRegs,
// else (improbably full cells) lane 0's insertion sort, as the reference.
__device__ __forceinline__ void sort_big_cell(const Arena& a, uint32_t cell, uint32_t start,
                                              uint32_t m, bool reorder, uint32_t lane) {
    const uint32_t end = start + m;
    if (m <= 32u * kSortRegs) {
        uint32_t key[kSortRegs], rank[kSortRegs];
#pragma unroll
        for (int r = 0; r < kSortRegs; r++) {
            uint32_t t = r * 32 + lane;
            key[r] = t < m ? a.sorted[start + t] : 0xffffffffu;
            rank[r] = 0;
        }
        for (int rr = 0; rr < kSortRegs; rr++) {
            if ((uint32_t)rr * 32u >= m) break;
            for (int src = 0; src < 32; src++) {
                uint32_t other = __shfl_sync(0xffffffffu, key[rr], src);
#pragma unroll
                for (int r = 0; r < kSortRegs; r++) rank[r] += other < key[r] ? 1u : 0u;
            }
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < kSortRegs; r++) {
            uint32_t t = r * 32 + lane;
            if (t < m) {
                a.sorted[start + rank[r]] = key[r];
                if (reorder) move_to_scratch(a, key[r], start + rank[r], cell);
            }
        }
    } else if (lane == 0) {
        for (uint32_t s = start + 1; s < end; s++) {
            uint32_t key = a.sorted[s];
            uint32_t t = s;
            while (t > start && a.sorted[t - 1] > key) {
                a.sorted[t] = a.sorted[t - 1];
                t -= 1;
            }
            a.sorted[t] = key;
        }
        if (reorder)
            for (uint32_t s = start; s < end; s++) move_to_scratch(a, a.sorted[s], s, cell);
    }
}

__global__ void __launch_bounds__(kBlock, 4) sort_kernel(Arena a) {
    count_kernel(a);
    if (!grid_pass(a)) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t cells = work_total(a), front = a.glob->work_front;
    // A warp takes work entries w and w + warps together, so the two cells'
    // chains of dependent loads (entry, range, slots, particles) overlap.
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < cells; w += 2u * warps) {
        uint32_t cell[2], start[2] = {0u, 0u}, m[2] = {0u, 0u}, key[2], rank[2] = {0u, 0u};
        bool live[2], reorder[2] = {false, false};
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const uint32_t t = w + (uint32_t)k * warps;
            const uint32_t entry = t < cells ? work_item(a, front, t) : 1u;
            live[k] = (entry & 7u) == 0u;  // a cell sorts once, with its first part
            cell[k] = entry >> 3;
        }
#pragma unroll
        for (int k = 0; k < 2; k++)
            if (live[k]) {
                start[k] = a.cell_start[cell[k]];
                m[k] = a.cell_start[cell[k] + 1] - start[k];
                reorder[k] = a.ctrl[box_of_cell(a, cell[k])].reorder != 0u;
                if (lane == 0) a.count[cell[k]] = 0u;
            }
        // the usual cell: one key per lane, ranked against the m keys (a
        // lane past m holds the largest key, which ranks below no one)
        bool small[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            small[k] = live[k] && m[k] <= 32u;
            key[k] = small[k] && lane < m[k] ? a.sorted[start[k] + lane] : 0xffffffffu;
        }
        const uint32_t mm = max(small[0] ? m[0] : 0u, small[1] ? m[1] : 0u);
        for (uint32_t src = 0; src < mm; src++) {
            rank[0] += __shfl_sync(0xffffffffu, key[0], src) < key[0] ? 1u : 0u;
            rank[1] += __shfl_sync(0xffffffffu, key[1], src) < key[1] ? 1u : 0u;
        }
        __syncwarp();
        // with reorder, both cells' particles are read before any is written
        double px[2][3], pv[2][3];
        uint32_t pid[2];
        bool moves[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            moves[k] = small[k] && lane < m[k] && reorder[k];
            if (moves[k]) {
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    px[k][d] = a.x[d * a.seg + key[k]];
                    pv[k][d] = a.v[d * a.seg + key[k]];
                }
                pid[k] = a.id[key[k]];
            }
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            if (!(small[k] && lane < m[k])) continue;
            const uint32_t to = start[k] + rank[k];
            a.sorted[to] = key[k];
            if (moves[k]) {
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    a.sx[d * a.seg + to] = px[k][d];
                    a.sv[d * a.seg + to] = pv[k][d];
                }
                a.sid[to] = pid[k];
                a.scell[to] = cell[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 2; k++)
            if (live[k] && m[k] > 32u) sort_big_cell(a, cell[k], start[k], m[k], reorder[k], lane);
        __syncwarp();
    }
}

// ---- reorder copy back (lennard_jones.wgsl:435-452) ----
__global__ void reorder_kernel(Arena a) {
    count_kernel(a);
    if (!a.glob->any) return;
    for_rebuild_slots(a, [&](uint32_t s, uint32_t b) {
        if (!a.ctrl[b].reorder) return;
        const Box& bx = a.boxes[b];
        uint4 w;
        double xs[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            xs[k] = a.sx[k * a.seg + s];
            a.x[k * a.seg + s] = xs[k];
            a.v[k * a.seg + s] = a.sv[k * a.seg + s];
        }
        a.id[s] = a.sid[s];
        a.cell_of_slot[s] = a.scell[s];
        a.sorted[s] = s;
        w.x = encode(xs[0], bx.enc[0]);
        w.y = encode(xs[1], bx.enc[1]);
        w.z = encode(xs[2], bx.enc[2]);
        w.w = 0u;
        a.cache[a.glob->phase][s] = w;
    });
}

// ---- launchers ----
cudaError_t launch_encode(const Arena& a, cudaStream_t s) {
    encode_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_load_particles(const Arena& a, cudaStream_t s) {
    load_particles_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_store_particles(const Arena& a, cudaStream_t s) {
    store_particles_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_decide(const Arena& a, cudaStream_t s, unsigned long long cond_handle) {
    if (cond_handle)
        decide_kernel<true><<<1, kBlock, 0, s>>>(a, (cudaGraphConditionalHandle)cond_handle);
    else
        decide_kernel<false><<<1, kBlock, 0, s>>>(a, (cudaGraphConditionalHandle)0);
    return after_launch();
}

cudaError_t launch_grid(const Arena& a, cudaStream_t s) {
    // the per-particle kernels cover the rebuilding boxes' particles from a
    // resident grid
    const unsigned slots = (unsigned)sm_count() * 8u;
    bin_kernel<<<slots, kBlock, 0, s>>>(a);
    scan_kernel<<<a.nboxes, kScanThreads, 0, s>>>(a);
    scatter_kernel<<<slots, kBlock, 0, s>>>(a);
    sort_kernel<<<(unsigned)sm_count() * 8u, kBlock, 0, s>>>(a);
    return after_launch(4);
}

cudaError_t launch_lists(const Arena& a, cudaStream_t s) {
    reorder_kernel<<<(unsigned)sm_count() * 8u, kBlock, 0, s>>>(a);
    launch_build_list(a, s);  // vlj_build.cu
    return after_launch(2);
}

cudaError_t launch_rebuild(const Arena& a, cudaStream_t s) {
    const cudaError_t e = launch_grid(a, s);
    return e != cudaSuccess ? e : launch_lists(a, s);
}

}  // namespace vlj
