// Internal structures and device helpers of the B200 Lennard-Jones library.
//
// Layout in HBM (one "arena" holds one box, or many independent boxes for the
// batched path, each box a contiguous run of slots and of cells):
//   x, v      f64, structure of arrays: x[k * seg + slot], k = 0, 1, 2.
//             v is stored half a kick behind (see the step kernel), so one
//             force pass serves the closing half kick of a step and the
//             opening half kick of the next; with Nose-Hoover or the heat
//             exchange it is canonical and the last forces are kept in acc.
//   cache[2]  uint4 per slot: the position as 32-bit fractions of the box
//             (X = round(x / L * 2^32) mod 2^32). Two copies: the step kernel
//             reads one and writes the other; `phase` says which is current.
//             Differences of these words wrap modulo 2^32, which is the
//             minimum image for free, at 32-bit resolution on any box size.
//   snap      uint4 per slot: the cache word at the last list build, for the
//             skin / 2 displacement trigger.
//   (no copy of the reference's packed positions is kept: the list build
//   settles all but a thin shell of candidates on the 32-bit words and, for
//   that shell, derives the reference's f32 hi / packed lo parts from x and
//   applies the reference's f32 predicate, so lists match it bit for bit)
//   list      u32 slot indices, interleaved by four: entry k of slot i at
//             list[((k / 4) * seg + i) * 4 + k % 4], counts in list_count[i];
//             the last row's unused places hold i itself. A row of the list
//             (four entries of one slot) is 16 B, so a thread reads a row with
//             one load and a warp reads 512 contiguous bytes; the force
//             kernels stream rows per thread past L1 (or, as a tuning option,
//             stage row tiles into shared memory with TMA).
//   cells     per cell: count (atomic cursor) and start. Boxes own contiguous
//             runs of slots and cells, so one start array of ncells + 1 entries
//             serves every box: box b's last cell ends where box b + 1 begins.
//   work      per step, the non-empty cells of the rebuilding boxes; rb_box /
//             rb_first the rebuilding boxes and their particle offsets.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vlj {

constexpr int kBlock = 256;
constexpr int kSlots = 8;  // measurement accumulators per box
// Force kernels: one thread per particle, kForceThreads per block. With the
// TMA tile ring (VLJ_LIST_STREAM=0) each tile holds kTileRows list rows (4
// entries each) of the block's particles; the ring's shared memory comes out
// of the same 256 KB per SM as the L1 that serves the neighbour gathers, so
// its depth is a tuning knob (tune.py sweeps it).
#ifndef VLJ_TILE_ROWS
#define VLJ_TILE_ROWS 4
#endif
#ifndef VLJ_TILE_SLOTS
#define VLJ_TILE_SLOTS 3
#endif
// 1: each force-kernel thread streams its own list rows from global memory
// with loads that do not allocate in L1 (leaving all of L1 to the gathers)
// instead of the TMA tile ring in shared memory.
#ifndef VLJ_LIST_STREAM
#define VLJ_LIST_STREAM 1
#endif
// 1: the pair force's reciprocal (square root) as the flush-to-zero PTX
// approximation (rsqrt_pair / rcp_pair below); 0: rsqrtf / __fdividef.
#ifndef VLJ_FTZ_PAIR
#define VLJ_FTZ_PAIR 1
#endif
// 1: with streamed rows, issue the next row's neighbour gathers before
// computing this row's pairs (twice the loads in flight, more registers).
#ifndef VLJ_GATHER_AHEAD
#define VLJ_GATHER_AHEAD 0
#endif
// Cell tiles of the step kernel (tile_step_kernel): 1 stages f32 offsets
// from the brick's centre instead of the encoded words (the separation is a
// plain f32 difference, not the same bits as the list kernels); 1 reads the
// next list row's neighbours while computing this row's pairs.
#ifndef VLJ_TILE_F32
#define VLJ_TILE_F32 0
#endif
// 1: the step kernel's blocks that share an SM take neighbouring runs of
// particles (their neighbourhoods overlap in that SM's L1)
#ifndef VLJ_STEP_REMAP
#define VLJ_STEP_REMAP 0
#endif
#ifndef VLJ_TILE_PIPE
#define VLJ_TILE_PIPE 0
#endif
constexpr int kForceThreads = 128;
constexpr uint32_t kDenseCell = 8;  // particles in a cell the list build takes first
// In a box under five cells wide on some axis (a batched replica) a cell
// holds many particles and its candidate stream is most of the box, so its
// home particles split into parts of kPartHomes (at most kMaxParts, the
// last taking the rest), each a work-list entry of its own: entry = cell * 8
// + part.
#ifndef VLJ_PART_HOMES
#define VLJ_PART_HOMES 8
#endif
constexpr uint32_t kPartHomes = VLJ_PART_HOMES;
constexpr uint32_t kMaxParts = 8;
constexpr int kTileRows = VLJ_TILE_ROWS;
constexpr int kTileSlots = VLJ_TILE_SLOTS;  // tiles in flight per block
// measurement slots: 0 kinetic, 1 potential, 2 virial, 3-5 momentum,
// 6 condensed count, 7 unused (lennard_jones.wgsl:576-626)

// Constants of one box. Read by every kernel from device memory, so a
// setter changes them without re-capturing graphs.
struct Box {
    double box[3];       // sides, rounded to f32 (lennard_jones.rs:450)
    double enc[3];       // 2^32 / side
    double dt, half_dt;
    double c1, c2;       // Langevin v <- c1 v + c2 xi (lennard_jones.rs:520-523)
    double nh_gkt, nh_q; // Nose-Hoover g k T and Q (lennard_jones.rs:516-528)
    double hex_energy;   // heat exchange: energy moved per step (its f32 value)
    float dec[3];        // side / 2^32, exact in f32
    float box_f[3];
    float cell_size_f[3];
    float rc2, list_r2, half_skin2;
    float shift, force_shift, rc;
    float energy_scale, momentum_scale;
    float bin_width;
    float inv_box_f[3];  // 1 / box_f, for nearest_ref_fast
    float hex_slabs[4];  // heat exchange: hot lo, hi, cold lo, hi in z
    float prefilter_r2;  // list_r2 widened past any encoding difference
    float accept_r2;     // list_r2 narrowed past any encoding difference
    float reach_r2;      // prefilter_r2 widened past binning round-off
    uint32_t cells[3];
    uint32_t total_cells;
    uint32_t cell_base;  // first cell of this box
    uint32_t first;      // first slot of this box
    uint32_t n;
    uint32_t capacity;   // list entries per particle
    int32_t thermostat;  // 0 constant energy, 1 Langevin, 2 Nose-Hoover
    uint32_t seed;
    uint32_t near_count;
    uint32_t drawn;
    uint32_t reorder_every;
    uint32_t profile_bins;
    uint32_t canonical;  // velocities stored canonical (Nose-Hoover, heat exchange)
    // Cell tiles of the step kernel (0 bricks: off for this box). A brick is
    // a run of cells along x in one row (y, z): each x-row holds brick_cols
    // bricks of nx / brick_cols cells (the first nx % brick_cols one more);
    // brick_base is the first brick of this box in the arena's numbering.
    uint32_t brick_cols;
    uint32_t brick_base;
    uint32_t pad[3];
};

// Mutable per-box words.
struct Control {
    uint32_t max_disp;   // f32 bits of the largest squared displacement
    uint32_t rebuild;    // this step rebuilds
    uint32_t reorder;    // this rebuild also moves particles into cell order
    uint32_t rebuilds;   // rebuilds so far (lennard_jones.wgsl:299-305)
    uint32_t overflow;   // largest neighbour count that did not fit
    uint32_t built;      // 0 until the first build
    uint32_t forced;     // rebuild at the next decision whatever moved
    uint32_t pad;
};

// Words shared by every box of an arena.
struct Global {
    uint32_t phase;      // which cache copy holds the current positions
    uint32_t pending;    // a step finished since the last decision
    uint32_t any;        // some box rebuilds this step
    uint32_t fault;      // first error a kernel recorded (0 none)
    unsigned long long step;     // steps taken: the counter of the noise stream
    unsigned long long kernels;  // kernels of this arena that ran
    uint32_t grid_every_step;    // 1: bin, scan, scatter and sort every step (one box)
    uint32_t work_front;         // Arena::work entries at its front: cells of kDenseCell or more
    uint32_t work_back;          // entries at its back (work[ncells - 1 - k]): the other non-empty cells
    uint32_t next_build;         // next work entry the list build takes
    uint32_t blocks_done;        // step-kernel blocks finished (the last one decides)
    uint32_t rb_boxes;           // boxes that rebuild this step (Arena::rb_box)
    uint32_t rb_slots;           // their particles, in all
    uint32_t heat_next;          // heat-current samples written to the series so far
    uint32_t decided;            // a step kernel took the next step's decision, not yet consumed
    uint32_t tiles_ready;        // the 16-bit tile lists match the box's bricks (a build wrote them)
};

// Nose-Hoover state of a box (Tuckerman's splitting, lennard_jones.wgsl:309-397).
// A step is: start half step (scale by s1), half kick, drift, lists, forces,
// half kick, end half step (scale by s2). The force kernel does the end half
// step's thermostat update once every block has added its kinetic energy
// (the last block to finish), but leaves the scaling pending: the velocities
// stay unscaled, `scale` holds s2, and whatever reads velocities at the step
// boundary (the measurement, the next step's start) applies it.
struct Thermo {
    double xi_s, eta_s;  // after the last start half step
    double xi_m, eta_m;  // after the last end half step (what a measurement sees)
    double ke_m;         // kinetic energy after the end half step's scaling
    double scale;        // s2: the end half step's scale, not yet applied
    unsigned long long ke_raw;  // this force pass's kinetic energy, 32.32 x energy scale
    uint32_t blocks_done;       // force blocks that added their part
    uint32_t pad;
};

// Heat exchange state of a box (eHEX/a, lennard_jones.wgsl:732-893): per
// slab (0 hot, 1 cold) the force pass's exact sums -- count, momentum (3),
// sum of v^2, sum of f . v, sum of f (3) -- in 32.32 fixed point (momentum
// and force times the momentum scale, the others times the energy scale),
// then what the last block to finish works out of them for the apply pass.
struct Exchange {
    unsigned long long sums[2][9];
    double com[2][3];     // centre-of-mass velocity
    double mean_f[2][3];  // mean force
    double s_minus_1[2];  // velocity scale about the centre of mass, minus one
    double c_v[2], c_f[2];  // eq. 20's position-correction coefficients
    uint32_t blocks_done;
    uint32_t pad;
};

// Fault codes in Global::fault (the first one recorded wins).
constexpr uint32_t kFaultTmaTimeout = 1;  // a TMA tile never arrived
constexpr uint32_t kFaultNonFinite = 2;   // an uploaded coordinate was not finite

// Every pointer a kernel needs; passed by value (it sits in the constant
// bank), so captured graphs see fixed pointers and read the mutable state
// through Control and Global.
struct Arena {
    const Box* boxes;
    Control* ctrl;
    Global* glob;
    uint32_t nboxes;
    uint32_t nslots;     // particles in all boxes
    uint32_t seg;        // padded slot count (list row length)
    uint32_t ncells;     // cells in all boxes
    const uint32_t* box_of_slot;  // null for a single box
    const uint32_t* box_of_cell;  // null for a single box
    double* x;
    double* v;
    uint32_t* id;
    uint4* cache[2];
    uint4* snap;
    uint32_t* cell_of_slot;
    uint32_t* sorted;
    uint32_t* cell_start;  // ncells + 1
    uint32_t* count;
    // the non-empty cells of the boxes that rebuild this step, as entries
    // cell * 8 + part (one part per cell but in narrow boxes): those of
    // kDenseCell particles or more and every part of a narrow box's cell
    // from the front, the others from the back, so the list build takes the
    // costly work first and ends on cheap work (work_item below)
    uint32_t* work;
    uint32_t work_cap;   // entries of room in work
    // the boxes that rebuild this step (rb_boxes of them, ascending) and the
    // running count of their particles before each (rb_first[rb_boxes] =
    // rb_slots): the per-particle rebuild kernels cover only these
    uint32_t* rb_box;
    uint32_t* rb_first;
    uint32_t* list_count;
    uint32_t* list;
    // The same lists as 16-bit indices into the cell tile of the home
    // particle's brick (tile_step_kernel), by sorted position: entry k of the
    // particle at sorted position p at list16[((k / 8) * seg + p) * 8 + k % 8]
    // (a row of eight entries is 16 B); the last row's unused places hold the
    // particle's own tile index. Null when no box uses cell tiles.
    uint16_t* list16;
    uint32_t bricks;     // bricks in all boxes: the tile step kernel's grid
    uint32_t tile_cap;   // tile entries (16 B each) a block stages in shared memory
    uint32_t tile_threads;  // threads of a tile step block
    uint32_t step_threads;  // particles per block of the step kernel: 64, 128 or 256
    uint32_t step_lanes;    // lanes per particle of the step kernel: 0 by grid size, 1 or 2
    uint32_t remap_sms, remap_per_sm;  // the step kernel's first-wave block layout (VLJ_STEP_REMAP)
    // per force block (kForceThreads slots), for the TMA tile ring only: rows
    // (four entries each) of the longest list in it, so a block stages only
    // the rows its particles use. Reset at each rebuild of
    // the box that holds the whole block; a block across two boxes keeps the
    // largest value it ever had (more rows staged, never fewer).
    uint32_t* block_rows;
    // particles as the API passes them (pos[3], vel[3] per particle, input
    // order), staged for upload and read-back
    double* aos;
    // reorder scratch
    double* sx;
    double* sv;
    uint32_t* sid;
    uint32_t* scell;
    // steps on canonical velocities (Nose-Hoover, heat exchange): the
    // thermostat and exchange state, and the last forces
    Thermo* nh;
    Exchange* hex;
    float4* acc;
    // measurements
    unsigned long long* accum;  // nboxes * kSlots
    float* pe_half;  // (hi, lo) per slot
    float* w_half;   // (hi, lo) per slot
    float4* vel4;
    double* vcanon;             // canonical velocities (3 * seg), on request
    // profiles / heat current
    unsigned long long* profile;  // bins * 8 + 3 per box
    unsigned long long* series;   // 1 + 3 * capacity
    uint32_t series_capacity;
};

// ---- fixed point: 32.32, round to nearest even ----
// For f32 x with |x| < 2^31 this equals the reference's integer split
// (fixed.wgsl:20-55): x * 2^32 is exact in f64 and the conversion rounds to
// nearest even.
__device__ __forceinline__ long long fixed_raw_f32(float x) {
    return __double2ll_rn((double)x * 4294967296.0);
}
__device__ __forceinline__ long long fixed_raw_f64(double x) {
    return __double2ll_rn(x * 4294967296.0);
}

// ---- position encoding ----
__device__ __forceinline__ uint32_t encode(double x, double enc) {
    return (uint32_t)(unsigned long long)__double2ll_rn(x * enc);
}
__device__ __forceinline__ float decode_diff(uint32_t a, uint32_t b, float dec) {
    return (float)(int32_t)(a - b) * dec;
}

// ---- the reference's packed positions (lennard_jones.wgsl:128-152), IEEE
// f32 operations exactly as written (no contraction) ----
__device__ __forceinline__ float last_bit(float h) {
    uint32_t e = (__float_as_uint(h) >> 23) & 0xffu;
    e = e < 24u ? 24u : e;
    return __uint_as_float((e - 23u) << 23);
}

// One axis of the reference's packed lo part: the f32 lo part as a 9-bit
// fraction q / 510 of the hi part's last bit, and back (pack_lo / unpack_lo,
// lennard_jones.wgsl:128-152). `q510` holds q / 510 for q = -256..255.
__device__ __forceinline__ float packed_lo(float h, float l, const float* q510) {
    const float unit = last_bit(h);
    float t = __fdiv_rn(l, unit);
    t = fminf(fmaxf(t, -0.5f), 0.5f);
    const int32_t q = (int32_t)rintf(__fmul_rn(t, 510.0f));
    return __fmul_rn(q510[q + 256], unit);
}

// nearest image, lennard_jones.wgsl:199-202
__device__ __forceinline__ float nearest_ref(float d, float side) {
    return __fsub_rn(d, __fmul_rn(side, rintf(__fdiv_rn(d, side))));
}

// ---- Philox-4x32-10 (Salmon et al., SC'11) of counter c and key k ----
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    uint32_t c0 = c.x, c1 = c.y, c2 = c.z, c3 = c.w;
    uint32_t k0 = k.x, k1 = k.y;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}

// The Langevin noise stream: counter (id, step lo, step hi, 0), key (seed,
// "LJV1"), one Philox block per particle and step.
__device__ __forceinline__ uint4 philox(uint32_t id, unsigned long long step, uint32_t seed) {
    return philox4x32_10(make_uint4(id, (uint32_t)step, (uint32_t)(step >> 32), 0u),
                         make_uint2(seed, 0x4C4A5631u));
}

// r . F and U of a pair at r2 < rc2 (lennard_jones.wgsl:533-545), for the
// energy and virial sums. The reciprocal and the square root are correctly
// rounded: on a lattice every pair at one distance rounds the same way, so a
// bias of a few ulp would add up coherently over all pairs, and the virial
// (a difference of repulsive and attractive terms) would show it.
template <bool SHIFTED_FORCE>
__device__ __forceinline__ void lj_pair(float r2, const Box& b, float& rf, float& u) {
    float inv2 = __frcp_rn(r2);
    float s6 = inv2 * inv2 * inv2;
    float s12 = s6 * s6;
    rf = 24.0f * (2.0f * s12 - s6);
    u = 4.0f * (s12 - s6) - b.shift;
    if (SHIFTED_FORCE) {
        float r = __fsqrt_rn(r2);
        rf -= r * b.force_shift;
        u += (r - b.rc) * b.force_shift;
    }
}

// 1 / sqrt(x) and 1 / x as the PTX approximations rsqrtf and __fdividef(1, x)
// use, in their flush-to-zero forms: the same values for normal inputs, without
// the subnormal-range handling around the hardware instruction. A list entry's
// r^2 is never subnormal: it is at least a few tenths (pairs closer than that
// have energies far beyond any simulated state) or exactly 0 for the padding,
// whose result the cutoff test drops either way.
__device__ __forceinline__ float rsqrt_pair(float x) {
#if VLJ_FTZ_PAIR
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
#else
    return rsqrtf(x);
#endif
}

__device__ __forceinline__ float rcp_pair(float x) {
#if VLJ_FTZ_PAIR
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
#else
    return __fdividef(1.0f, x);
#endif
}

// The pair energy at r2 < rc2 with the force kernels' reciprocal (the same
// approximations as lj_force_over_r2, so a pass computes both from one).
template <bool SHIFTED_FORCE>
__device__ __forceinline__ float lj_energy_fast(float r2, const Box& b) {
    if (SHIFTED_FORCE) {
        const float inv_r = rsqrt_pair(r2);
        const float inv2 = inv_r * inv_r;
        const float s6 = inv2 * inv2 * inv2;
        return 4.0f * s6 * (s6 - 1.0f) - b.shift + (r2 * inv_r - b.rc) * b.force_shift;
    }
    const float inv2 = rcp_pair(r2);
    const float s6 = inv2 * inv2 * inv2;
    return 4.0f * s6 * (s6 - 1.0f) - b.shift;
}

// |F| / r of a pair at r2 < rc2: the factor that multiplies the separation.
// Every operation is spelled out (no contraction left to the compiler), so
// each kernel that computes it, whatever else it computes beside, gets the
// same bits.
template <bool SHIFTED_FORCE>
__device__ __forceinline__ float lj_force_over_r2(float r2, float force_shift) {
    if (SHIFTED_FORCE) {
        // one reciprocal square root gives both 1/r^2 and r
        const float inv_r = rsqrt_pair(r2);
        const float inv2 = __fmul_rn(inv_r, inv_r);
        const float s6 = __fmul_rn(__fmul_rn(inv2, inv2), inv2);
        const float lj = __fmul_rn(__fmul_rn(24.0f, s6), __fmaf_rn(2.0f, s6, -1.0f));
        const float rf = __fmaf_rn(-__fmul_rn(r2, inv_r), force_shift, lj);
        return __fmul_rn(rf, inv2);
    }
    const float inv2 = rcp_pair(r2);
    const float s6 = __fmul_rn(__fmul_rn(inv2, inv2), inv2);
    return __fmul_rn(__fmul_rn(__fmul_rn(24.0f, s6), __fmaf_rn(2.0f, s6, -1.0f)), inv2);
}

// Squared length of a separation, the force kernels' way (spelled out).
__device__ __forceinline__ float sep_r2(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// The reference's nearest image d - side * round(d / side) with the IEEE
// quotient, computed through the reciprocal: d * (1 / side) is within 2e-7 of
// d / side for |d| <= side, so both round to the same integer unless the
// quotient is within 1e-6 of a half-integer, where the exact division is
// taken. Bit-identical to nearest_ref.
__device__ __forceinline__ float nearest_ref_fast(float d, float side, float inv_side) {
    float q = d * inv_side;
    float aq = fabsf(q);
    float r;
    if (aq < 1.25f && fabsf(aq - 0.5f) > 1e-6f)
        r = rintf(q);
    else
        r = rintf(__fdiv_rn(d, side));
    return __fsub_rn(d, __fmul_rn(side, r));
}

// Squared length of an encoded separation (the force kernels' arithmetic).
__device__ __forceinline__ float encoded_r2(uint4 a, uint4 b, const float dec[3]) {
    float dx = decode_diff(a.x, b.x, dec[0]);
    float dy = decode_diff(a.y, b.y, dec[1]);
    float dz = decode_diff(a.z, b.z, dec[2]);
    return dx * dx + dy * dy + dz * dz;
}

// ---- launchers (vlj_kernels.cu); every kernel takes the Arena by value ----
cudaError_t launch_encode(const Arena& a, cudaStream_t s);
// Particles from a.aos (input order) into the state of a single box: positions
// wrapped into the box, ids the input order; a non-finite coordinate records
// kFaultNonFinite. And back: positions and canonical velocities (a.vcanon)
// into a.aos in input order.
cudaError_t launch_load_particles(const Arena& a, cudaStream_t s);
cudaError_t launch_store_particles(const Arena& a, cudaStream_t s);
cudaError_t launch_decide(const Arena& a, cudaStream_t s, unsigned long long cond_handle);
cudaError_t launch_rebuild(const Arena& a, cudaStream_t s);
// The two halves of launch_rebuild: the cell grid (bin, scan, scatter, sort)
// and the lists (reorder copy-back, list build).
cudaError_t launch_grid(const Arena& a, cudaStream_t s);
cudaError_t launch_lists(const Arena& a, cudaStream_t s);
// The force kernels read list rows through `list_map`: a 2D TMA tensor map
// over the list viewed as u64 pairs of entries (inner dimension 2 * seg,
// outer one row per four entries) whose box is kTileRows rows of
// kForceThreads slots.
cudaError_t launch_prime(const Arena& a, const CUtensorMap& list_map, bool shifted_force,
                         cudaStream_t s);
// `next_decision`, when not 0, is the graph conditional of the next step's
// rebuild: the step kernel's last block to finish then takes the next step's
// decision itself (in place of a decide launch) and sets it.
// With `heat`, the same kernel also takes the pending heat-current sample of
// the state it starts from (series slot Global::heat_next, then advanced):
// the force pass has every pair's separation and force, and the canonical
// velocity v + a dt / 2 is known once the particle's forces are summed.
cudaError_t launch_step(const Arena& a, const CUtensorMap& list_map, bool shifted_force,
                        cudaStream_t s, unsigned long long next_decision = 0, bool heat = false);
cudaError_t launch_measure(const Arena& a, const CUtensorMap& list_map, bool shifted_force,
                           bool canonical, cudaStream_t s);
// Steps on canonical velocities (one box): begin applies Nose-Hoover's
// pending scale s2 and this step's s1, kicks and drifts; canon_force computes
// the forces and then, by `pass`: kPrime records them (and the starting
// kinetic energy) without a kick; kNoseHoover kicks and does the end half
// step's thermostat update; kExchange kicks and sums the exchange slabs;
// kKick only kicks. hex_apply moves the energy between the slabs.
enum CanonPass { kPrime = 0, kNoseHoover = 1, kExchange = 2, kKick = 3 };
cudaError_t launch_begin(const Arena& a, cudaStream_t s);
cudaError_t launch_canon_force(const Arena& a, const CUtensorMap& list_map, bool shifted_force,
                               CanonPass pass, cudaStream_t s);
cudaError_t launch_hex_apply(const Arena& a, cudaStream_t s);
// Back from canonical velocities to half a kick behind (v -= a dt / 2).
cudaError_t launch_half_kick_back(const Arena& a, cudaStream_t s);
// Sampling kernels (vlj_sampling.cu): one profile sample added into
// a.profile, one heat-current sample into a.series slot 1 + 3 * sample.
cudaError_t launch_profile(const Arena& a, uint32_t bins, bool shifted_force, cudaStream_t s);
// After a measurement, each particle's local temperature into vel4.w:
// m v^2 / 3 averaged over it and its neighbours within the cutoff.
cudaError_t launch_drawn_temperature(const Arena& a, cudaStream_t s);
cudaError_t launch_heat_current(const Arena& a, bool shifted_force, uint32_t sample,
                                cudaStream_t s);
cudaError_t launch_fp32_peak(float* out, int blocks, int iters, cudaStream_t s);
// Philox-4x32-10 of n (counter, key) pairs and the Langevin noise the step
// kernel draws for each (id, step, seed) read from them (vlj_debug_philox).
cudaError_t launch_philox_check(const uint4* ctr, const uint2* key, uint32_t n, uint4* out,
                                float4* noise, cudaStream_t s);
unsigned long long launches();

}  // namespace vlj
