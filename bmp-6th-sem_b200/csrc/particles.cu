// particles.cu -- cell binning, CIC deposit and gather + Boris push for
// sm_100a.
//
// Reference operators replaced (SYCL-PIC-poissonsolver):
//   * hashmap binning: InsertKernel (src/particles.cpp:227-237), map
//     delete/insert inside MoverKernel (src/mover.cpp:353-364), cleanup_map
//     (src/utils.cpp:30-44) and compact_particles (src/utils.cpp:249-372);
//   * interpolate() (src/interpolation.cpp:13-171);
//   * deterministic_mover() + MoverKernel (src/mover.cpp:103-176, 304-366).
//
// Layout: the particles of a species live in a double buffer of 20-byte
// slots, float4 {fx, fy, vx, vy} (in-cell offsets in [0,1), velocities in
// m/s) plus float vz.  Cell c (c = gy*nx + gx) owns the slots base[c] ..
// base[c+1] of both buffers with slack: its particles are a front run (the
// ones that stayed in the cell at the last push) and a back run (the ones
// that moved in), with a free gap between them.
//
// One push of a species is ONE pass over its particles (k_cells<kPush>): a
// warp walks a cell, gathers E and Bz, pushes, and
//   * writes a particle that stays in its cell to the front of the cell's
//     slots in the other buffer, at its rank among the cell's stayers
//     (ballot + popc: no atomics);
//   * appends a particle that moves to a neighbouring cell to the back of
//     that cell's slots: lanes moving the same way form a group
//     (match.any), the group leader reserves the slots with one atomic on
//     the target's back count.  The reservation is capped at the target's
//     capacity minus its current count (the most stayers it can have), so
//     front and back runs never meet;
//   * deposits the new position: stayers accumulate per-lane integer
//     moments reduced once per cell, movers add their four fixed-point
//     corner weights with 64-bit RED.
// A mover whose target is full, or which jumped more than one cell, goes to
// a side list; a small kernel (k_fixup) then places it in the free space of
// its target cell, or keeps it on the list (still part of the state: it is
// pushed and deposited from there at the next step).  When the list grows,
// the host rebuilds the layout from the per-cell counts (k_relayout_*).
// Per particle-step the HBM traffic is 20 B read + 20 B written.
//
// Determinism: the charge and energy deposits are sums of integers, so they
// do not depend on the order in which particles are processed or placed;
// the set of particles in each cell is deterministic, their order within
// the back run is not.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "pic_internal.h"

namespace picb200 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = kWarps * 32;
constexpr int kCellBlocksPerSM = 4;           // k_cells residency (register budget)
constexpr int kScanTile = 2048;               // cells per scan block
constexpr uint32_t kAxisOne = 1u << kAxisBits;
constexpr float kAxisScale = (float)(1u << kAxisBits);
constexpr float kOneBelow = 0x1.fffffep-1f;   // largest float < 1
constexpr float kEnergyScale = 4194304.0f;    // eV -> 2^-22 eV units
constexpr float kFloorMagic = 12582912.0f;    // 1.5 * 2^23
constexpr uint32_t kFloorMagicBits = 0x4B400000u;
constexpr int kFixupBlocks = 296;

enum Mode { kPush = 0, kDeposit = 1 };
constexpr int kFar = 9;       // moved more than one cell in x or y

// list_counts slots
enum { kOvf = 0, kLoose0 = 1, kLoose1 = 2 };

struct ListDev {
    float4* a;
    float* vz;
    uint32_t* cell;
    uint32_t* count;
    uint32_t cap;
};

__host__ __forceinline__ ListDev list_dev(const LooseList& L) {
    return ListDev{L.a, L.vz, L.cell, L.count, L.cap};
}

struct KArgs {
    int nx, ny, GX;
    int64_t ncells;
    SpeciesConsts k;
    const float4* __restrict__ fld;
    const float4* __restrict__ src_a;
    const float* __restrict__ src_vz;
    float4* __restrict__ dst_a;
    float* __restrict__ dst_vz;
    const uint32_t* __restrict__ base;
    const uint32_t* __restrict__ front_src;
    const uint32_t* __restrict__ back_src;
    uint32_t* front_dst;
    uint32_t* back_dst;
    ListDev ovf;
    unsigned long long* acc_q;
    unsigned long long* acc_e;
    unsigned long long* counters;  // [0] left exits, [1] cell limit, [2] lost particles
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Asynchronous global -> shared copies (cp.async) to a shared-space address;
// a false predicate copies nothing and fills the destination with zeros.
// Only the wait orders them against the shared-memory reads of the data.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool pred) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(pred ? 16 : 0));
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, bool pred) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src),
                 "r"(pred ? 4 : 0));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Result of one gather + Boris + position update.
struct Pushed {
    float fx, fy, vx, vy;
    float px, py;  // new position in units of the old cell (its corner at 0)
    int sx, sy;    // cell step: 0, 0 exactly when the particle keeps its cell
    // set by resolve_move
    int gx, gy;
    int dir;  // 0: moved at most one cell in x and y, kFar: farther, -1: absorbed
    bool left;
};

// Bilinear gather of E (and Bz) from the cell's four nodes plus the Boris
// push of deterministic_mover (src/mover.cpp:123-174) in FP32.  Weights:
// (1-fx)(1-fy), fx(1-fy), (1-fx)fy, fx*fy == the reference's unnormalised
// weights divided by dx*dy.  Every operation is an explicit _rn intrinsic:
// the result does not depend on how the compiler contracts the code.
//
// push_move does the arithmetic of every particle; resolve_move the cell
// bookkeeping that only particles leaving their cell need.
__device__ __forceinline__ Pushed push_move(float4 a, float4 n00, float4 n10, float4 n01,
                                            float4 n11, const SpeciesConsts& k) {
    const float fx = a.x, fy = a.y;
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    const float w00 = __fmul_rn(ofx, ofy), w10 = __fmul_rn(fx, ofy);
    const float w01 = __fmul_rn(ofx, fy), w11 = __fmul_rn(fx, fy);
    const float ex = __fmaf_rn(w11, n11.x, __fmaf_rn(w01, n01.x, __fmaf_rn(w10, n10.x, __fmul_rn(w00, n00.x))));
    const float ey = __fmaf_rn(w11, n11.y, __fmaf_rn(w01, n01.y, __fmaf_rn(w10, n10.y, __fmul_rn(w00, n00.y))));
    // Boris rotation about z (src/mover.cpp:151-162): t = h Bz, s = 2t/(1+t^2)
    float t, s;
    if (k.bzu) {
        t = k.bt;
        s = k.bs;
    } else {
        const float bz = __fmaf_rn(w11, n11.z, __fmaf_rn(w01, n01.z, __fmaf_rn(w10, n10.z, __fmul_rn(w00, n00.z))));
        t = __fmul_rn(k.h, bz);
        // approximate reciprocal: ~1 ulp, far below the FP32 state's error
        s = __fdividef(__fmul_rn(2.0f, t), __fmaf_rn(t, t, 1.0f));
    }
    const float ax = __fmul_rn(k.h, ex), ay = __fmul_rn(k.h, ey);
    const float vxm = __fadd_rn(a.z, ax), vym = __fadd_rn(a.w, ay);
    const float vxp = __fmaf_rn(vym, t, vxm);
    const float vyp = __fmaf_rn(-vxm, t, vym);
    Pushed o;
    o.vx = __fadd_rn(__fmaf_rn(vyp, s, vxm), ax);
    o.vy = __fadd_rn(__fmaf_rn(-vxp, s, vym), ay);
    // Position update in cell units (src/mover.cpp:164-165), then re-cell:
    // the integer part moves the cell, the remainder is the new offset.
    const float px = __fmaf_rn(o.vx, k.dtdx, fx);
    const float py = __fmaf_rn(o.vy, k.dtdy, fy);
    o.px = px;
    o.py = py;
    // floor without the conversion unit: for |p| < 2^22, p + 1.5*2^23
    // rounded down is floor(p) + 1.5*2^23 exactly, an integer held in the
    // low mantissa bits; subtracting 1.5*2^23 again is exact.  The step's
    // bits are 0 exactly when floor(p) == 0: for NaN or |p| >= 2^22 the sum
    // is not 1.5*2^23, so those never read as staying.
    const float tx = __fadd_rd(px, kFloorMagic), ty = __fadd_rd(py, kFloorMagic);
    const float fsx = __fsub_rn(tx, kFloorMagic), fsy = __fsub_rn(ty, kFloorMagic);
    o.fx = fminf(__fsub_rn(px, fsx), kOneBelow);
    o.fy = fminf(__fsub_rn(py, fsy), kOneBelow);
    o.sx = (int)(__float_as_uint(tx) - kFloorMagicBits);
    o.sy = (int)(__float_as_uint(ty) - kFloorMagicBits);
    return o;
}

// Cell bookkeeping of a pushed particle that was in cell (gx, gy).
__device__ __forceinline__ void resolve_move(Pushed& o, const SpeciesConsts& k, int gx, int gy,
                                             int nx, int ny) {
    const float px = o.px, py = o.py;
    // beyond 2^20 cells (or NaN) a particle is lost whatever the grid
    const bool ok = fabsf(px) < 1048576.0f && fabsf(py) < 1048576.0f;
    const int sx = ok ? o.sx : 0;
    const int sy = ok ? o.sy : 0;
    o.gx = gx + sx;
    o.gy = gy + sy;
    // periodic in y (modulo(y, H), src/mover.cpp:317-320): the cell row
    // wraps, the offset stays
    if (k.pery && (unsigned)o.gy >= (unsigned)ny) {
        o.gy %= ny;
        if (o.gy < 0) o.gy += ny;
    }
    // absorbing walls (src/mover.cpp:325): outside [0,W) x [0,H)
    const bool alive = ok && (unsigned)o.gx < (unsigned)nx && (unsigned)o.gy < (unsigned)ny;
    o.left = ok ? (o.gx < 0) : (px < 0.0f);
    const bool near = (unsigned)(sx + 1) < 3u && (unsigned)(sy + 1) < 3u;
    o.dir = !alive ? -1 : (near ? 0 : kFar);
}

__device__ __forceinline__ Pushed push_one(float4 a, float4 n00, float4 n10, float4 n01,
                                           float4 n11, const SpeciesConsts& k, int gx, int gy,
                                           int nx, int ny) {
    Pushed o = push_move(a, n00, n10, n01, n11, k);
    resolve_move(o, k, gx, gy, nx, ny);
    return o;
}

// round(f * 2^20) for f in [0, 1): exact scaling, then the 1.5*2^23 addition
// rounds to nearest-even in the mantissa (integer ALU, no conversion unit).
__device__ __forceinline__ uint32_t axis_fixed(float f) {
    const float t = __fadd_rn(__fmul_rn(f, kAxisScale), 12582912.0f);
    return __float_as_uint(t) - 0x4B400000u;
}

// Kinetic energy in eV (0.5 v^2/|q/m|, src/interpolation.cpp:88-89), clamped.
__device__ __forceinline__ float energy_ev(float vx, float vy, float vz, float half_inv_abs_qm) {
    const float v2 = __fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx)));
    return fminf(__fmul_rn(v2, half_inv_abs_qm), kEnergyClampEv);
}

// Energy-weighted corner weights of one particle, rounded to integers of
// 2^-22 eV (each below 2^32): e00 <-> (gx,gy), e10 <-> (gx+1,gy),
// e01 <-> (gx,gy+1), e11 <-> (gx+1,gy+1).
struct EWeights {
    uint32_t e00, e10, e01, e11;
};

__device__ __forceinline__ EWeights energy_weights(float fx, float fy, float en) {
    const float es = __fmul_rn(en, kEnergyScale);
    const float a = __fmul_rn(es, __fsub_rn(1.0f, fx)), b = __fmul_rn(es, fx);
    const float ofy = __fsub_rn(1.0f, fy);
    EWeights w;
    w.e00 = __float2uint_rn(__fmul_rn(a, ofy));
    w.e10 = __float2uint_rn(__fmul_rn(b, ofy));
    w.e01 = __float2uint_rn(__fmul_rn(a, fy));
    w.e11 = __float2uint_rn(__fmul_rn(b, fy));
    return w;
}

// Global 64-bit integer reductions (fire-and-forget RED) into the node
// accumulators.
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long v) {
    atomicAdd(p, v);
}

// Deposit of one particle straight into the node accumulators: its four
// charge corner weights are the exact 40-bit products of the 20-bit axis
// weights (they sum to exactly 2^40).
template <bool ENERGY>
__device__ __forceinline__ void deposit_one(unsigned long long* acc_q, unsigned long long* acc_e,
                                            int GX, uint32_t n, float fx, float fy, float en) {
    const uint32_t ax = axis_fixed(fx), ay = axis_fixed(fy);
    const uint32_t bx = kAxisOne - ax, by = kAxisOne - ay;
    red_add(acc_q + n, (unsigned long long)bx * by);
    red_add(acc_q + n + 1, (unsigned long long)ax * by);
    red_add(acc_q + n + GX, (unsigned long long)bx * ay);
    red_add(acc_q + n + GX + 1, (unsigned long long)ax * ay);
    if (ENERGY) {
        const EWeights e = energy_weights(fx, fy, en);
        red_add(acc_e + n, e.e00);
        red_add(acc_e + n + 1, e.e10);
        red_add(acc_e + n + GX, e.e01);
        red_add(acc_e + n + GX + 1, e.e11);
    }
}

// Per-lane sums of the particles that stay in the warp's cell.  Charge as
// moments of the 20-bit axis weights -- count N (the warp's stayer count,
// kept by the caller), sum ax, sum ay, sum ax*ay -- from which the four
// corner sums follow exactly:
//   Q00 = N 2^40 - (SX + SY) 2^20 + SXY,  Q10 = SX 2^20 - SXY,
//   Q01 = SY 2^20 - SXY,                   Q11 = SXY.
// A lane holds at most kMaxPerCell/32 = 2^11 particles: SX, SY < 2^31,
// SXY < 2^51.  The energy mesh (a diagnostic) sums its corner weights per
// lane in FP32, in 2^-22 eV units (< 2^43), rounded to integers once per
// lane and cell: exact integer sums from there on, but the per-lane FP32
// rounding depends on the order of the lane's particles.
struct StayAcc {
    uint32_t sx, sy;
    unsigned long long sxy;
    float e[4];
};

__device__ __forceinline__ void acc_zero(StayAcc& s) {
    s.sx = s.sy = 0u;
    s.sxy = 0ull;
#pragma unroll
    for (int k = 0; k < 4; ++k) s.e[k] = 0.f;
}

template <bool ENERGY>
__device__ __forceinline__ void acc_add(StayAcc& s, float fx, float fy, float en) {
    const uint32_t ax = axis_fixed(fx), ay = axis_fixed(fy);
    s.sx += ax;
    s.sy += ay;
    s.sxy += (unsigned long long)ax * ay;
    if (ENERGY) {
        const float es = __fmul_rn(en, kEnergyScale);
        const float a = __fmul_rn(es, __fsub_rn(1.0f, fx)), b = __fmul_rn(es, fx);
        const float ofy = __fsub_rn(1.0f, fy);
        s.e[0] = __fmaf_rn(a, ofy, s.e[0]);
        s.e[1] = __fmaf_rn(b, ofy, s.e[1]);
        s.e[2] = __fmaf_rn(a, fy, s.e[2]);
        s.e[3] = __fmaf_rn(b, fy, s.e[3]);
    }
}

// Warp sum of a value below 2^(LO+27) as two 32-bit limbs (redux.sync).
template <int LO>
__device__ __forceinline__ unsigned long long warp_sum_limbs(unsigned long long v) {
    const uint32_t lo = (uint32_t)(v & ((1ull << LO) - 1ull));
    const uint32_t hi = (uint32_t)(v >> LO);
    return (unsigned long long)__reduce_add_sync(kFull, lo) +
           ((unsigned long long)__reduce_add_sync(kFull, hi) << LO);
}

// Warp-reduce the cell's stayer sums and add them to its four nodes (lane 0).
// N: the cell's stayer count (known to the whole warp).
template <bool ENERGY>
__device__ __forceinline__ void acc_flush(StayAcc& s, const KArgs& A, int gx, int gy, int lane,
                                          unsigned long long N) {
    const unsigned long long SX = warp_sum_limbs<26>(s.sx);
    const unsigned long long SY = warp_sum_limbs<26>(s.sy);
    const unsigned long long SXY = warp_sum_limbs<26>(s.sxy);
    unsigned long long E[4] = {0ull, 0ull, 0ull, 0ull};
    if (ENERGY) {
#pragma unroll
        for (int k = 0; k < 4; ++k) E[k] = warp_sum_limbs<22>(__float2ull_rn(s.e[k]));
    }
    if (lane == 0 && N) {
        const int64_t n = (int64_t)gy * A.GX + gx;
        red_add(A.acc_q + n, (N << 40) - ((SX + SY) << 20) + SXY);
        red_add(A.acc_q + n + 1, (SX << 20) - SXY);
        red_add(A.acc_q + n + A.GX, (SY << 20) - SXY);
        red_add(A.acc_q + n + A.GX + 1, SXY);
        if (ENERGY) {
            red_add(A.acc_e + n, E[0]);
            red_add(A.acc_e + n + 1, E[1]);
            red_add(A.acc_e + n + A.GX, E[2]);
            red_add(A.acc_e + n + A.GX + 1, E[3]);
        }
    }
    acc_zero(s);
}

__device__ __forceinline__ void store_slot(float4* dst_a, float* dst_vz, uint32_t slot,
                                           const Pushed& p, float vz) {
    __stcs(dst_a + slot, make_float4(p.fx, p.fy, p.vx, p.vy));
    __stcs(dst_vz + slot, vz);
}

// Appends the lanes with `on` set to a side list (one atomic per warp).
__device__ __forceinline__ void list_append(const ListDev& L, bool on, uint32_t cell,
                                            const Pushed& p, float vz, unsigned lt, int lane,
                                            unsigned long long* lost) {
    const unsigned m = __ballot_sync(kFull, on);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    uint32_t b = 0;
    if (lane == leader) b = atomicAdd(L.count, (uint32_t)__popc(m));
    b = __shfl_sync(kFull, b, leader);
    if (on) {
        const uint32_t s = b + __popc(m & lt);
        if (s < L.cap) {
            L.a[s] = make_float4(p.fx, p.fy, p.vx, p.vy);
            L.vz[s] = vz;
            L.cell[s] = cell;
        } else {
            atomicOr(lost, 1ull);
        }
    }
}

// One kernel body for the two uses:
//   kPush    -- push, place every particle in the other buffer, deposit the
//               new positions;
//   kDeposit -- deposit the current positions (no push, nothing moves).
// A block owns a kTileX x kTileY tile of cells.  Its prologue stages the
// tile's per-cell slot metadata and the node fields in shared memory; then
// each warp streams through the particles of its cells (tile cells warp,
// warp + kWarps, ...) in chunks of 32.  The chunks travel through a per-warp
// ring of kDepth chunk buffers in shared memory filled by cp.async, kDepth-1
// chunks ahead of the one being processed -- across cell boundaries, so the
// load pipeline never drains.
constexpr int kDepth = 4;
static_assert((kDepth & (kDepth - 1)) == 0, "ring depth: a power of two");

struct CellMeta {
    uint32_t b0, b1, nf, nb;
};

// Movers wait in a per-warp queue in shared memory and are placed 32 at a
// time (all lanes busy): deposit, grouping by target cell (match.any), one
// slot reservation per group, store.
constexpr int kQueue = 64;

struct MoverQueue {
    float4 a[kQueue];
    float vz[kQueue];
    uint2 g[kQueue];  // target cell (gx, gy)
};

// A cell strictly inside its block's tile (not on the tile's border, not on
// the periodic seam) receives direct placements only from cells of the
// same tile: one-cell movers from elsewhere cannot reach it, and longer
// jumps into it from other tiles go to the side list.  Its back count is
// kept in shared memory and written out when the block ends, instead of a
// global atomic per group of movers.  (lx, ly): the cell's position in its
// tile; gy: its row.
template <int TX, int TY>
__device__ __forceinline__ bool tile_owned(int lx, int ly, int gy, const KArgs& A) {
    return TY > 2 && lx >= 1 && lx <= TX - 2 && ly >= 1 && ly <= TY - 2 &&
           !(A.k.pery && (gy == 0 || gy == A.ny - 1));
}

// Places `count` (<= 32) queued movers, entries 0..count-1, from the block
// of tile (tgx0, tgy0): all lanes busy on the target's bookkeeping.
template <bool ENERGY, int TX, int TY>
__device__ __forceinline__ void place_movers(const KArgs& A, MoverQueue& q,
                                             const CellMeta* __restrict__ s_meta,
                                             uint32_t* s_back, int tgx0, int tgy0, int count,
                                             int lane, unsigned lt) {
    __syncwarp();
    const bool on = lane < count;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    float vz = 0.f;
    uint2 g = make_uint2(0u, 0u);
    if (on) {
        a = q.a[lane];
        vz = q.vz[lane];
        g = q.g[lane];
    }
    const uint32_t t = g.y * (uint32_t)A.nx + g.x;
    const float en = (ENERGY && on) ? energy_ev(a.z, a.w, vz, A.k.half_inv_abs_qm) : 0.f;
    // movers bound for the same cell form a group; its leader reserves the
    // group's slots at the back of the cell, capped at the cell's capacity
    // minus its current count (the most stayers it can have)
    const unsigned grp = __match_any_sync(kFull, on ? t : (0x80000000u | (uint32_t)lane));
    const int leader = __ffs(grp) - 1;
    uint32_t old = 0, lim = 0, top = 0;
    if (on && lane == leader) {
        const uint32_t cnt = __popc(grp);
        const int lx = (int)g.x - tgx0, ly = (int)g.y - tgy0;
        const bool in_tile = (unsigned)lx < (unsigned)TX && (unsigned)ly < (unsigned)TY;
        // the target's slots and source counts: from the tile's shared
        // metadata when it lies in this block's tile (most movers go one
        // cell), else from global memory
        CellMeta m;
        if (in_tile) {
            m = s_meta[ly * TX + lx];
        } else {
            m.b0 = A.base[t];
            m.b1 = A.base[t + 1];
            m.nf = A.front_src[t];
            m.nb = A.back_src[t];
        }
        lim = (m.b1 - m.b0) - (m.nf + m.nb);
        top = m.b1;
        // the back count: in shared memory for a cell this block owns
        uint32_t* ctr = (in_tile && tile_owned<TX, TY>(lx, ly, (int)g.y, A)) ? s_back + (ly * TX + lx)
                                                                              : A.back_dst + t;
        old = atomicAdd(ctr, cnt);
        // give back what does not fit (the count then ends at
        // min(requested, lim) with slots 0.. taken)
        if (old + cnt > lim) atomicSub(ctr, old >= lim ? cnt : old + cnt - lim);
    }
    if (on) deposit_one<ENERGY>(A.acc_q, A.acc_e, A.GX, g.y * (uint32_t)A.GX + g.x, a.x, a.y, en);
    old = __shfl_sync(kFull, old, leader);
    lim = __shfl_sync(kFull, lim, leader);
    top = __shfl_sync(kFull, top, leader);
    bool spill = false;
    Pushed p;
    p.fx = a.x; p.fy = a.y; p.vx = a.z; p.vy = a.w;
    if (on) {
        const uint32_t k = old + __popc(grp & lt);
        if (k < lim) store_slot(A.dst_a, A.dst_vz, top - 1u - k, p, vz);
        else spill = true;
    }
    list_append(A.ovf, spill, t, p, vz, lt, lane, A.counters + 2);
}

template <int MODE, bool ENERGY, int TX, int TY>
__device__ __forceinline__ void cells_body(const KArgs& A, int tile_x, int tile_y) {
    constexpr int kTileX = TX, kTileY = TY;
    constexpr int kTileCells = kTileX * kTileY;
    constexpr int kTileNodesX = kTileX + 1;
    constexpr int kTileNodes = (kTileX + 1) * (kTileY + 1);
    __shared__ CellMeta s_meta[kTileCells];
    __shared__ float4 s_fld[MODE == kPush ? kTileNodes : 1];
    __shared__ MoverQueue s_q[MODE == kPush ? kWarps : 1];
    // tiles of one or two rows own no cell
    __shared__ uint32_t s_back[MODE == kPush && kTileY > 2 ? kTileCells : 1];
    __shared__ float4 s_ring_a[kWarps][kDepth][32];
    __shared__ float s_ring_vz[kWarps][kDepth][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tgx0 = tile_x * kTileX, tgy0 = tile_y * kTileY;
    const unsigned lt = lanemask_lt();
    // tile cell (lx, ly) is owned: inside the grid, off the tile's border
    // and off the periodic seam (rows 0 and ny-1 exchange wrapped movers)
    auto owned = [&](int lx, int ly) {
        return tgx0 + lx < A.nx && tgy0 + ly < A.ny && tile_owned<TX, TY>(lx, ly, tgy0 + ly, A);
    };
    if (MODE == kPush && kTileY > 2)
        for (int i = threadIdx.x; i < kTileCells; i += kThreads) s_back[i] = 0u;
    for (int i = threadIdx.x; i < kTileCells; i += kThreads) {
        const int gx = tgx0 + (i % kTileX), gy = tgy0 + (i / kTileX);
        CellMeta m{0u, 0u, 0u, 0u};
        if (gx < A.nx && gy < A.ny) {
            const int64_t c = (int64_t)gy * A.nx + gx;
            m.b0 = A.base[c];
            m.b1 = A.base[c + 1];
            m.nf = A.front_src[c];
            m.nb = A.back_src[c];
        }
        s_meta[i] = m;
    }
    if (MODE == kPush) {
        for (int i = threadIdx.x; i < kTileNodes; i += kThreads) {
            const int x = tgx0 + (i % kTileNodesX), y = tgy0 + (i / kTileNodesX);
            s_fld[i] = (x < A.GX && y < A.ny + 1) ? __ldg(A.fld + (int64_t)y * A.GX + x)
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    __syncthreads();

    uint32_t left_exits = 0;  // per lane
    // the warp's cells are lc = warp + kWarps*k; empty ones only get their
    // front count written
    auto next_cell = [&](int lc, bool mark_empty) {
        for (; lc < kTileCells; lc += kWarps) {
            const CellMeta m = s_meta[lc];
            if (m.nf + m.nb) break;
            const int gx = tgx0 + (lc % kTileX), gy = tgy0 + (lc / kTileX);
            if (MODE == kPush && mark_empty && lane == 0 && gx < A.nx && gy < A.ny)
                A.front_dst[(int64_t)gy * A.nx + gx] = 0u;
        }
        return lc;
    };
    // producer: issues the copies of the chunk (plc, pj0) into ring slot r
    // and advances; every call commits one (possibly empty) copy group
    // the producer's cell as the source index of its j-th particle: the
    // front run for j < nf, then the back run (index back + j)
    struct ProdCell {
        uint32_t front, back, nf, n;
    };
    auto prod_cell = [&](int c) {
        const CellMeta pm = c < kTileCells ? s_meta[c] : CellMeta{0u, 0u, 0u, 0u};
        return ProdCell{pm.b0, pm.b1 - pm.nb - pm.nf, pm.nf, pm.nf + pm.nb};
    };
    int plc = next_cell(warp, false);
    ProdCell pc = prod_cell(plc);
    uint32_t pj0 = 0;
    const uint32_t ring_a0 = smem_u32(&s_ring_a[warp][0][lane]);
    const uint32_t ring_vz0 = smem_u32(&s_ring_vz[warp][0][lane]);
    auto issue = [&](int r) {
        if (plc < kTileCells) {
            const uint32_t jj = pj0 + lane;
            const bool v = jj < pc.n;
            const uint32_t i = !v ? 0u : (jj < pc.nf ? pc.front : pc.back) + jj;
            cp_async16(ring_a0 + (uint32_t)r * (32u * 16u), A.src_a + i, v);
            cp_async4(ring_vz0 + (uint32_t)r * (32u * 4u), A.src_vz + i, v);
            if (pj0 + 32 >= pc.n) {
                plc = next_cell(plc + kWarps, false);
                pc = prod_cell(plc);
                pj0 = 0;
            } else {
                pj0 += 32;
            }
        }
        cp_async_commit();
    };

    MoverQueue& q = s_q[MODE == kPush ? warp : 0];
    int queued = 0;  // warp-uniform
    int lc = next_cell(warp, true);
    if (lc < kTileCells) {
#pragma unroll
        for (int r = 0; r < kDepth - 1; ++r) issue(r);
        // the consumer's cell: particle count, coordinates, its field
        // corner in the shared tile, and the next free front slot
        uint32_t n, front;
        int gx, gy;
        const float4* f;
        auto enter = [&](int c) {
            const CellMeta m = s_meta[c];
            n = m.nf + m.nb;
            front = m.b0;
            const int lx = c % kTileX, ly = c / kTileX;
            gx = tgx0 + lx;
            gy = tgy0 + ly;
            f = s_fld + ly * kTileNodesX + lx;
        };
        enter(lc);
        uint32_t j0 = 0, front0 = front;
        int r = 0;
        StayAcc acc;
        acc_zero(acc);
        for (;;) {
            const bool last = j0 + 32 >= n;
            // the next chunk: same cell, or the warp's next non-empty cell
            const int lcn = last ? next_cell(lc + kWarps, true) : lc;
            // refill the slot freed by the previous chunk, then wait for this one
            issue((r + kDepth - 1) & (kDepth - 1));
            cp_async_wait<kDepth - 1>();
            const float4 a = s_ring_a[warp][r][lane];
            const float vz = s_ring_vz[warp][r][lane];
            r = (r + 1) & (kDepth - 1);

            const bool valid = j0 + lane < n;
            Pushed p;
            bool stay;
            if (MODE == kDeposit) {
                p.fx = a.x; p.fy = a.y; p.vx = a.z; p.vy = a.w;
                stay = valid;
            } else {
                p = push_move(a, f[0], f[1], f[kTileNodesX], f[kTileNodesX + 1], A.k);
                stay = valid && (p.sx | p.sy) == 0;
            }
            const float en = (ENERGY && stay) ? energy_ev(p.vx, p.vy, vz, A.k.half_inv_abs_qm) : 0.f;
            if (stay) acc_add<ENERGY>(acc, p.fx, p.fy, en);
            if (MODE == kPush) {
                const unsigned sm = __ballot_sync(kFull, stay);
                if (stay) store_slot(A.dst_a, A.dst_vz, front + __popc(sm & lt), p, vz);
                front += __popc(sm);
                // the cell bookkeeping of the rest (absorbed or moving), only
                // in chunks that have any (most chunks of slow species do not)
                const bool other = valid && !stay;
                if (__any_sync(kFull, other)) {
                    bool mv = false, far = false;
                    if (other) {
                        resolve_move(p, A.k, gx, gy, A.nx, A.ny);
                        mv = p.dir >= 0;
                        // a jump of more than one cell into a cell that
                        // another block owns: deposited here, placed from
                        // the side list after the pass (rare)
                        if (kTileY > 2 && p.dir == kFar) {
                            const int olx = p.gx % kTileX, oly = p.gy % kTileY;
                            const bool mine = p.gx - olx == tgx0 && p.gy - oly == tgy0;
                            far = !mine && tile_owned<TX, TY>(olx, oly, p.gy, A);
                            mv = mv && !far;
                        }
                        left_exits += (p.dir < 0 && p.left) ? 1u : 0u;
                    }
                    if (kTileY > 2 && __any_sync(kFull, far)) {
                        const uint32_t tc = (uint32_t)(p.gy * A.nx + p.gx);
                        if (far) {
                            const float ef = ENERGY ? energy_ev(p.vx, p.vy, vz, A.k.half_inv_abs_qm) : 0.f;
                            deposit_one<ENERGY>(A.acc_q, A.acc_e, A.GX, (uint32_t)(p.gy * A.GX + p.gx),
                                                p.fx, p.fy, ef);
                        }
                        list_append(A.ovf, far, tc, p, vz, lt, lane, A.counters + 2);
                    }
                    const unsigned mm = __ballot_sync(kFull, mv);
                    if (mm) {  // warp-uniform: queue the movers
                        if (mv) {
                            const int e = queued + __popc(mm & lt);
                            q.a[e] = make_float4(p.fx, p.fy, p.vx, p.vy);
                            q.vz[e] = vz;
                            q.g[e] = make_uint2((uint32_t)p.gx, (uint32_t)p.gy);
                        }
                        queued += __popc(mm);
                        if (queued >= 32) {
                            place_movers<ENERGY, TX, TY>(A, q, s_meta, s_back, tgx0, tgy0, 32, lane, lt);
                            // the rest (< 32) moves to the front of the queue
                            queued -= 32;
                            __syncwarp();
                            if (lane < queued) {
                                q.a[lane] = q.a[32 + lane];
                                q.vz[lane] = q.vz[32 + lane];
                                q.g[lane] = q.g[32 + lane];
                            }
                            __syncwarp();
                        }
                    }
                }
            }
            if (last) {
                const uint32_t stayers = front - front0;
                acc_flush<ENERGY>(acc, A, gx, gy, lane, MODE == kPush ? stayers : n);
                if (MODE == kPush && lane == 0) A.front_dst[(int64_t)gy * A.nx + gx] = stayers;
                if (lcn >= kTileCells) break;
                enter(lcn);
                front0 = front;
                j0 = 0;
            } else {
                j0 += 32;
            }
            lc = lcn;
        }
        cp_async_wait<0>();
    }
    if (MODE == kPush && queued > 0)
        place_movers<ENERGY, TX, TY>(A, q, s_meta, s_back, tgx0, tgy0, queued, lane, lt);
    if (MODE == kPush) {
        const uint32_t left = __reduce_add_sync(kFull, left_exits);
        if (lane == 0 && left) atomicAdd(A.counters, (unsigned long long)left);
        // the owned cells' back counts (no other block placed into them)
        if (kTileY > 2) {
            __syncthreads();
            for (int i = threadIdx.x; i < kTileCells; i += kThreads) {
                const int lx = i % kTileX, ly = i / kTileX;
                if (owned(lx, ly) && s_back[i])
                    A.back_dst[(int64_t)(tgy0 + ly) * A.nx + tgx0 + lx] = s_back[i];
            }
        }
    }
}

// Tile shapes the kernels are built for (cells per block in x, y); every
// shape has 256 cells.
#define PIC_TILE_SHAPES(X) X(64, 4) X(256, 1) X(128, 2) X(16, 16)
constexpr int kNumTileShapes = 4;
constexpr int kTileShapeX[kNumTileShapes] = {64, 256, 128, 16};
constexpr int kTileShapeY[kNumTileShapes] = {4, 1, 2, 16};

template <int MODE, bool ENERGY, int TX, int TY>
__global__ void __launch_bounds__(kThreads, kCellBlocksPerSM) k_cells(KArgs A) {
    cells_body<MODE, ENERGY, TX, TY>(A, blockIdx.x, blockIdx.y);
}

// One launch over many instances: block b works on tile (work[b].y & 0xffff,
// work[b].y >> 16) of instance work[b].x, whose arguments are args[work[b].x].
template <int MODE, bool ENERGY, int TX, int TY>
__global__ void __launch_bounds__(kThreads, kCellBlocksPerSM) k_cells_batch(const KArgs* __restrict__ args,
                                                             const uint2* __restrict__ work) {
    __shared__ KArgs s_args;
    const uint2 w = work[blockIdx.x];
    static_assert(sizeof(KArgs) % 8 == 0, "KArgs copy");
    for (int i = threadIdx.x; i < (int)(sizeof(KArgs) / 8); i += kThreads)
        reinterpret_cast<unsigned long long*>(&s_args)[i] =
            reinterpret_cast<const unsigned long long*>(args + w.x)[i];
    __syncthreads();
    cells_body<MODE, ENERGY, TX, TY>(s_args, (int)(w.y & 0xffffu), (int)(w.y >> 16));
}

// ---- side lists ---------------------------------------------------------------

struct FixArgs {
    int nx, ny, GX;
    SpeciesConsts k;
    const float4* __restrict__ fld;
    float4* dst_a;
    float* dst_vz;
    const uint32_t* __restrict__ base;
    const uint32_t* __restrict__ front;  // final front counts of the new buffer
    uint32_t* back;                      // back counts of the new buffer
    ListDev ovf;    // pushed this step, not yet placed
    ListDev prev;   // part of the state before the push, not yet pushed
    ListDev next;   // output: pushed, did not fit
    unsigned long long* acc_q;
    unsigned long long* acc_e;
    unsigned long long* counters;
};

// Pushes (and deposits) the particles of the previous side list, then tries
// to place them and this push's spilled movers in the free gap of their
// target cells; what does not fit goes to the next side list.
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_fixup(FixArgs F) {
    const uint32_t n_prev = min(*F.prev.count, F.prev.cap);
    const uint32_t n_ovf = min(*F.ovf.count, F.ovf.cap);
    const uint32_t total = n_prev + n_ovf;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        Pushed p;
        float vz;
        uint32_t t;
        if (i < n_prev) {
            const uint32_t c = F.prev.cell[i];
            const int gx = (int)(c % (uint32_t)F.nx), gy = (int)(c / (uint32_t)F.nx);
            const int64_t n0 = (int64_t)gy * F.GX + gx;
            vz = F.prev.vz[i];
            p = push_one(F.prev.a[i], F.fld[n0], F.fld[n0 + 1], F.fld[n0 + F.GX], F.fld[n0 + F.GX + 1],
                         F.k, gx, gy, F.nx, F.ny);
            if (p.dir < 0) {
                if (p.left) atomicAdd(F.counters, 1ull);
                continue;
            }
            const float en = ENERGY ? energy_ev(p.vx, p.vy, vz, F.k.half_inv_abs_qm) : 0.f;
            deposit_one<ENERGY>(F.acc_q, F.acc_e, F.GX, (uint32_t)(p.gy * F.GX + p.gx), p.fx, p.fy, en);
            t = (uint32_t)(p.gy * F.nx + p.gx);
        } else {
            const uint32_t e = i - n_prev;
            const float4 a = F.ovf.a[e];
            p.fx = a.x; p.fy = a.y; p.vx = a.z; p.vy = a.w;
            vz = F.ovf.vz[e];
            t = F.ovf.cell[e];
        }
        const uint32_t lim = (F.base[t + 1] - F.base[t]) - F.front[t];
        const uint32_t k = atomicAdd(F.back + t, 1u);
        if (k < lim) {
            store_slot(F.dst_a, F.dst_vz, F.base[t + 1] - 1u - k, p, vz);
        } else {
            atomicSub(F.back + t, 1u);
            const uint32_t s = atomicAdd(F.next.count, 1u);
            if (s < F.next.cap) {
                F.next.a[s] = make_float4(p.fx, p.fy, p.vx, p.vy);
                F.next.vz[s] = vz;
                F.next.cell[s] = t;
            } else {
                atomicOr(F.counters + 2, 1ull);
            }
        }
    }
}

// Deposit of the particles on a side list (stand-alone deposit).
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_list_deposit(ListDev L, int nx, int GX, float half_inv_abs_qm,
                                                      unsigned long long* acc_q, unsigned long long* acc_e) {
    const uint32_t n = min(*L.count, L.cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = L.a[i];
        const uint32_t c = L.cell[i];
        const float en = ENERGY ? energy_ev(a.z, a.w, L.vz[i], half_inv_abs_qm) : 0.f;
        deposit_one<ENERGY>(acc_q, acc_e, GX, c + c / (uint32_t)nx, a.x, a.y, en);  // node = c + gy
    }
}

// ---- layouts: counts, exclusive scans ------------------------------------------
//
// Slot capacity of a cell holding n particles: n + n/2 + 16 (room for a
// step's incoming movers and for the count to drift between re-layouts).
__host__ __device__ __forceinline__ uint32_t cell_capacity(uint32_t n) { return n + n / 2u + 16u; }

// cnt[c] = front[c] + back[c]
__global__ void k_cell_counts(const uint32_t* front, const uint32_t* back, int64_t ncells, uint32_t* cnt) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncells) cnt[c] = front[c] + back[c];
}

// cnt[cell] += 1 for each side-list entry
__global__ void k_list_counts(ListDev L, uint32_t* cnt) {
    const uint32_t n = min(*L.count, L.cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(cnt + L.cell[i], 1u);
}

template <bool CAP>
__device__ __forceinline__ uint32_t scan_value(const uint32_t* in, int64_t t) {
    return CAP ? cell_capacity(in[t]) : in[t];
}

template <bool CAP>
__global__ void __launch_bounds__(256) k_scan_partials(const uint32_t* in, int64_t n, uint32_t* partials) {
    __shared__ uint32_t red[8];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (int j = threadIdx.x; j < kScanTile; j += 256) {
        const int64_t t = base + j;
        if (t >= n) break;
        s += scan_value<CAP>(in, t);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += red[w];
        partials[blockIdx.x] = t;
    }
}

// out[t] = sum of values before t, out[n] = total.  With CAP the values are
// cell capacities, and cells above kMaxPerCell raise counters[1].
template <bool CAP>
__global__ void __launch_bounds__(256) k_scan_apply(const uint32_t* in, int64_t n,
                                                    const uint32_t* partials, uint32_t* out,
                                                    unsigned long long* counters) {
    __shared__ uint32_t red[8];
    __shared__ uint32_t wsum[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t pre = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += 256) pre += partials[j];
    for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(kFull, pre, o);
    if (lane == 0) red[warp] = pre;
    __syncthreads();
    uint32_t block_pre = 0;
    for (int w = 0; w < 8; ++w) block_pre += red[w];
    // each thread owns 8 consecutive entries
    const int64_t c0 = (int64_t)blockIdx.x * kScanTile + threadIdx.x * 8;
    uint32_t v[8];
    uint32_t tsum = 0, vmax = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        v[j] = (c0 + j < n) ? scan_value<CAP>(in, c0 + j) : 0u;
        tsum += v[j];
        vmax = max(vmax, v[j]);
    }
    uint32_t incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += wsum[w];
    uint32_t run = block_pre + wpre + incl - tsum;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t t = c0 + j;
        if (t < n) out[t] = run;
        run += v[j];
        if (t == n - 1) out[n] = run;
    }
    if (CAP && vmax > kMaxPerCell) atomicOr(counters + 1, 1ull);
}

// Copies every cell's particles (front run, then back run) from the old
// layout to the front of its slots in the new one; new_front = count.
__global__ void k_relayout_cells(const float4* __restrict__ src_a, const float* __restrict__ src_vz,
                                 const uint32_t* __restrict__ base, const uint32_t* __restrict__ front,
                                 const uint32_t* __restrict__ back, const uint32_t* __restrict__ nbase,
                                 int64_t ncells, float4* dst_a, float* dst_vz, uint32_t* nfront,
                                 uint32_t* nback) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const uint32_t nf = front[c], nb = back[c], b0 = base[c], back0 = base[c + 1] - nb;
    const uint32_t d0 = nbase[c];
    for (uint32_t j = lane; j < nf + nb; j += 32) {
        const uint32_t i = j < nf ? b0 + j : back0 + (j - nf);
        dst_a[d0 + j] = src_a[i];
        dst_vz[d0 + j] = src_vz[i];
    }
    if (lane == 0) {
        nfront[c] = nf + nb;
        nback[c] = 0u;
    }
}

// Side-list particles into the new layout, after the cell's own particles.
__global__ void k_relayout_list(ListDev L, const uint32_t* __restrict__ nbase, uint32_t* nfront,
                                float4* dst_a, float* dst_vz) {
    const uint32_t n = min(*L.count, L.cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = L.cell[i];
        const uint32_t s = nbase[c] + atomicAdd(nfront + c, 1u);
        dst_a[s] = L.a[i];
        dst_vz[s] = L.vz[i];
    }
}

// ---- import / export ------------------------------------------------------

// Reference Point -> cell.  The cell follows InsertKernel: gx = (int)(x *
// (1/dx)) in FP64 (src/particles.cpp:230-235); dead (pointer == -1) and
// out-of-domain points get no cell.
// Import of records (converted from reference Points on the host): count
// per cell, then place each record in its cell's front run.
__global__ void k_import_count(const PointRec* __restrict__ recs, int64_t n, uint32_t* cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t cell = recs[i].cell;
    if (cell != kNoCell) atomicAdd(cnt + cell, 1u);
}

__global__ void k_import_place(const PointRec* __restrict__ recs, int64_t n,
                               const uint32_t* __restrict__ base, uint32_t* front, float4* dst_a,
                               float* dst_vz) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PointRec r = recs[i];
    if (r.cell == kNoCell) return;
    const uint32_t d = base[r.cell] + atomicAdd(front + r.cell, 1u);
    dst_a[d] = make_float4(r.fx, r.fy, r.vx, r.vy);
    dst_vz[d] = r.vz;
}

// Layout -> records in cell order (dense[c] = particles before cell c); the
// host expands them into reference Points.
__global__ void k_export(const float4* __restrict__ a, const float* __restrict__ vz,
                         const uint32_t* __restrict__ base, const uint32_t* __restrict__ front,
                         const uint32_t* __restrict__ back, const uint32_t* __restrict__ dense,
                         int64_t ncells, PointRec* out) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const uint32_t nf = front[c], nb = back[c], b0 = base[c], back0 = base[c + 1] - nb, d0 = dense[c];
    for (uint32_t j = lane; j < nf + nb; j += 32) {
        const uint32_t i = j < nf ? b0 + j : back0 + (j - nf);
        const float4 v = a[i];
        PointRec r;
        r.cell = (uint32_t)c;
        r.fx = v.x;
        r.fy = v.y;
        r.vx = v.z;
        r.vy = v.w;
        r.vz = vz[i];
        out[d0 + j] = r;
    }
}

// Layout -> raw arrays (cell, fx, fy, vx, vy, vz) in cell order.
__global__ void k_export_state(const float4* __restrict__ a, const float* __restrict__ vz,
                               const uint32_t* __restrict__ base, const uint32_t* __restrict__ front,
                               const uint32_t* __restrict__ back, const uint32_t* __restrict__ dense,
                               int64_t ncells, int32_t* cell, float* fx, float* fy, float* vx,
                               float* vy, float* vzo) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const uint32_t nf = front[c], nb = back[c], b0 = base[c], back0 = base[c + 1] - nb, d0 = dense[c];
    for (uint32_t j = lane; j < nf + nb; j += 32) {
        const uint32_t i = j < nf ? b0 + j : back0 + (j - nf);
        const float4 v = a[i];
        const uint32_t o = d0 + j;
        cell[o] = (int32_t)c;
        fx[o] = v.x;
        fy[o] = v.y;
        vx[o] = v.z;
        vy[o] = v.w;
        vzo[o] = vz[i];
    }
}

// Live particles per reference bucket key gy*GRID_X + gx.
__global__ void k_bin_counts(const uint32_t* __restrict__ cnt, int nx, int ny, int GX, int32_t* counts) {
    const int64_t nodes = (int64_t)GX * (ny + 1);
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    const int gx = (int)(k % GX), gy = (int)(k / GX);
    counts[k] = (gx < nx && gy < ny) ? (int32_t)cnt[(int64_t)gy * nx + gx] : 0;
}

// ---- accumulators -> meshes -------------------------------------------------

// final_mesh = weighing * sum of unnormalised corner weights; rho += final *
// (-q/eps) (src/interpolation.cpp:139-171).  Resets the accumulators.
// The conversion of one species' accumulators into its final/energy mesh
// (and rho += final * chrg).
struct FlushEntry {
    int64_t nodes;
    unsigned long long* acc_q;
    unsigned long long* acc_e;
    double qscale, escale, chrg;
    double* final_mesh;
    double* energy_mesh;
    double* rho;
    int energy;
};

// kFlushNodes nodes from i0 on, `stride` apart (coalesced across a block),
// all loads issued before any store: the arrays are distinct, so the loads
// need not wait on each other's stores, and several are in flight at once.
constexpr int kFlushNodes = 4;

__device__ __forceinline__ void flush_nodes(const FlushEntry& F, int64_t i0, int stride) {
    unsigned long long q[kFlushNodes], e[kFlushNodes];
    double r[kFlushNodes];
#pragma unroll
    for (int u = 0; u < kFlushNodes; ++u) {
        const int64_t i = i0 + (int64_t)u * stride;
        const bool in = i < F.nodes;
        q[u] = in ? F.acc_q[i] : 0ull;
        e[u] = (in && F.energy) ? F.acc_e[i] : 0ull;
        r[u] = in ? F.rho[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kFlushNodes; ++u) {
        const int64_t i = i0 + (int64_t)u * stride;
        if (i >= F.nodes) break;
        const double f = (double)q[u] * F.qscale;
        F.acc_q[i] = 0ull;
        F.final_mesh[i] = f;
        if (F.energy) {
            F.energy_mesh[i] = (double)e[u] * F.escale;
            F.acc_e[i] = 0ull;
        } else {
            F.energy_mesh[i] = 0.0;
        }
        F.rho[i] = r[u] + f * F.chrg;
    }
}

__global__ void k_flush(FlushEntry F) {
    flush_nodes(F, (int64_t)blockIdx.x * blockDim.x * kFlushNodes + threadIdx.x, blockDim.x);
}

// ---- device plasma loading (Philox-4x32-10, Salmon et al., SC'11) ----------

__device__ __forceinline__ uint4 philox(uint4 ctr, uint2 key) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * ctr.x, hi0 = __umulhi(0xD2511F53u, ctr.x);
        const uint32_t lo1 = 0xCD9E8D57u * ctr.z, hi1 = __umulhi(0xCD9E8D57u, ctr.z);
        ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
        key.x += 0x9E3779B9u;
        key.y += 0xBB67AE85u;
    }
    return ctr;
}

__device__ __forceinline__ float u01(uint32_t u) { return (float)(u >> 8) * 0x1p-24f; }
__device__ __forceinline__ float u01_open(uint32_t u) { return (float)((u >> 8) + 1u) * 0x1p-24f; }

struct PlasmaArgs {
    int nx, ny;
    int ppc;
    double blob_peak, blob_cx, blob_cy, inv_two_sig2;
    float sigma_v, drift_vx, drift_vy;
    uint2 key;
    uint32_t species;
};

__device__ __forceinline__ uint32_t blob_count(const PlasmaArgs& P, int64_t c) {
    if (P.blob_peak <= 0.0) return 0;
    const int gx = (int)(c % P.nx), gy = (int)(c / P.nx);
    const double rx = gx + 0.5 - P.blob_cx, ry = gy + 0.5 - P.blob_cy;
    const double m = P.blob_peak * exp(-(rx * rx + ry * ry) * P.inv_two_sig2);
    const uint4 r = philox(make_uint4((uint32_t)c, (uint32_t)(c >> 32), P.species, 0xB10Bu), P.key);
    return (uint32_t)floor(m + (double)u01(r.x));
}

__global__ void k_plasma_counts(PlasmaArgs P, int64_t ncells, uint32_t* cnt) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    cnt[c] = (uint32_t)P.ppc + blob_count(P, c);
}

// Particle j of cell c gets the Philox counter dense[c] + j (its index in
// cell order) and the slot base[c] + j.
__global__ void k_plasma_generate(PlasmaArgs P, const uint32_t* __restrict__ dense,
                                  const uint32_t* __restrict__ base, int64_t ncells, float4* a,
                                  float* vz, uint32_t* front, uint32_t* back) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const uint32_t beg = dense[c], end = dense[c + 1], b0 = base[c];
    for (uint32_t i = beg + lane; i < end; i += 32) {
        const uint4 r0 = philox(make_uint4(i, P.species, 0u, 0x5EEDu), P.key);
        const uint4 r1 = philox(make_uint4(i, P.species, 1u, 0x5EEDu), P.key);
        const float fx = u01(r0.x), fy = u01(r0.y);
        // Box-Muller, per-component sigma = sqrt(e*T/m)
        const float m1 = P.sigma_v * sqrtf(-2.0f * logf(u01_open(r0.z)));
        const float m2 = P.sigma_v * sqrtf(-2.0f * logf(u01_open(r1.x)));
        float s1, c1, s2, c2;
        sincospif(2.0f * u01(r0.w), &s1, &c1);
        sincospif(2.0f * u01(r1.y), &s2, &c2);
        const bool blob = (i - beg) >= (uint32_t)P.ppc;
        float vx = m1 * c1, vy = m1 * s1, vzz = m2 * c2;
        if (blob) {
            vx += P.drift_vx;
            vy += P.drift_vy;
        }
        const uint32_t s = b0 + (i - beg);
        a[s] = make_float4(fx, fy, vx, vy);
        vz[s] = vzz;
    }
    if (lane == 0) {
        front[c] = end - beg;
        back[c] = 0u;
    }
}

inline unsigned grid1d(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// out[0..n] = exclusive scan of in (CAP: of cell capacities); returns the
// total through *total when not null (synchronises).
template <bool CAP>
int scan_cells(pic_ctx* c, Species& sp, const uint32_t* in, uint32_t* out, uint32_t* total) {
    const int64_t n = c->ncells;
    const int nparts = (int)((n + kScanTile - 1) / kScanTile);
    k_scan_partials<CAP><<<nparts, 256, 0, c->stream>>>(in, n, c->scan_partials);
    k_scan_apply<CAP><<<nparts, 256, 0, c->stream>>>(in, n, c->scan_partials, out, sp.counters);
    c->launches += 2;
    PIC_CUDA(cudaGetLastError());
    if (total) {
        PIC_CUDA(cudaMemcpyAsync(total, out + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
    }
    return PIC_OK;
}

// Species constants for a push, with the Boris factors of a uniform Bz.
SpeciesConsts push_consts(const pic_ctx* c, const Species& sp) {
    SpeciesConsts k = sp.k;
    k.bzu = c->bz_uniform ? 1 : 0;
    k.pery = c->periodic ? 1 : 0;
    const float t = k.h * (float)c->bz_value;
    k.bt = t;
    k.bs = (float)(2.0 * (double)t / (1.0 + (double)t * (double)t));
    return k;
}

KArgs make_args(pic_ctx* c, Species& sp) {
    KArgs A{};
    A.nx = c->nx;
    A.ny = c->ny;
    A.GX = c->GX;
    A.ncells = c->ncells;
    A.k = push_consts(c, sp);
    A.fld = c->fld;
    A.src_a = sp.buf[sp.cur].a;
    A.src_vz = sp.buf[sp.cur].vz;
    A.dst_a = sp.buf[sp.cur ^ 1].a;
    A.dst_vz = sp.buf[sp.cur ^ 1].vz;
    A.base = sp.base;
    A.front_src = sp.front[sp.cur];
    A.back_src = sp.back[sp.cur];
    A.front_dst = sp.front[sp.cur ^ 1];
    A.back_dst = sp.back[sp.cur ^ 1];
    A.ovf = list_dev(sp.ovf);
    A.acc_q = sp.acc_q;
    A.acc_e = sp.acc_e;
    A.counters = sp.counters;
    return A;
}

dim3 tile_grid(const pic_ctx* c, int shape) {
    return dim3((unsigned)((c->nx + kTileShapeX[shape] - 1) / kTileShapeX[shape]),
                (unsigned)((c->ny + kTileShapeY[shape] - 1) / kTileShapeY[shape]));
}

// Launch of k_cells with the tile shape `shape` (index into kTileShape*).
template <int MODE, bool ENERGY>
void launch_cells(int shape, dim3 grid, cudaStream_t st, const KArgs& A) {
    switch (shape) {
        case 1: k_cells<MODE, ENERGY, 256, 1><<<grid, kThreads, 0, st>>>(A); break;
        case 2: k_cells<MODE, ENERGY, 128, 2><<<grid, kThreads, 0, st>>>(A); break;
        case 3: k_cells<MODE, ENERGY, 16, 16><<<grid, kThreads, 0, st>>>(A); break;
        default: k_cells<MODE, ENERGY, 64, 4><<<grid, kThreads, 0, st>>>(A); break;
    }
}

template <int MODE, bool ENERGY>
void launch_cells_batch(int shape, unsigned nblocks, cudaStream_t st, const KArgs* args,
                        const uint2* work) {
    switch (shape) {
        case 1: k_cells_batch<MODE, ENERGY, 256, 1><<<nblocks, kThreads, 0, st>>>(args, work); break;
        case 2: k_cells_batch<MODE, ENERGY, 128, 2><<<nblocks, kThreads, 0, st>>>(args, work); break;
        case 3: k_cells_batch<MODE, ENERGY, 16, 16><<<nblocks, kThreads, 0, st>>>(args, work); break;
        default: k_cells_batch<MODE, ENERGY, 64, 4><<<nblocks, kThreads, 0, st>>>(args, work); break;
    }
}

template <typename K>
cudaError_t max_shared(K k) {
    return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
}

// Four blocks of the particle kernels per SM need ~4 x 44 KB of shared memory.
template <int MODE, bool ENERGY>
cudaError_t carveouts() {
    cudaError_t e = cudaSuccess;
#define PIC_CARVE(TX, TY)                                                           \
    if (e == cudaSuccess) e = max_shared(k_cells<MODE, ENERGY, TX, TY>);           \
    if (e == cudaSuccess) e = max_shared(k_cells_batch<MODE, ENERGY, TX, TY>);
    PIC_TILE_SHAPES(PIC_CARVE)
#undef PIC_CARVE
    return e;
}

int check_flags(pic_ctx* c, Species& sp, bool sync);

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static int list_alloc(LooseList& L, uint32_t cap, uint32_t* count) {
    cudaFree(L.a);
    cudaFree(L.vz);
    cudaFree(L.cell);
    L = LooseList{};
    PIC_CUDA(cudaMalloc(&L.a, (size_t)cap * sizeof(float4)));
    PIC_CUDA(cudaMalloc(&L.vz, (size_t)cap * sizeof(float)));
    PIC_CUDA(cudaMalloc(&L.cell, (size_t)cap * sizeof(uint32_t)));
    L.cap = cap;
    L.count = count;
    return PIC_OK;
}

static void list_free(LooseList& L) {
    cudaFree(L.a);
    cudaFree(L.vz);
    cudaFree(L.cell);
    L = LooseList{};
}

static int grow_store(pic_ctx* c, int s, int64_t capacity);
static int grow_lists(pic_ctx* c, int s);

// Side lists hold up to 1/16 of the slots (at least 2^20 particles).
static uint32_t list_capacity(int64_t slots) {
    return (uint32_t)std::min<int64_t>(std::max<int64_t>(slots / 16, 1 << 20), 0x40000000ll);
}

int species_setup(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    sp.desc = c->cfg.species[s];
    if (sp.desc.mass <= 0 || sp.desc.sim_count <= 0)
        return fail(PIC_ERR_CONFIG, "species mass and SimulationParticles must be positive");
    sp.ctom = sp.desc.charge / sp.desc.mass;  // initCtoM, src/particles.cpp:298-300
    const double surf = c->cfg.surf_area > 0 ? c->cfg.surf_area : c->cfg.xmax * c->cfg.ymax;
    // updateWeighingFactor, src/particles.cpp:303-305
    sp.weighing = sp.desc.actual_count * surf / (sp.desc.sim_count * c->dx * c->dy * c->dx * c->dy);
    sp.k.h = (float)(0.5 * sp.ctom * c->cfg.dt);
    sp.k.dtdx = (float)(c->cfg.dt / c->dx);
    sp.k.dtdy = (float)(c->cfg.dt / c->dy);
    sp.k.half_inv_abs_qm = sp.ctom != 0 ? (float)(0.5 / std::fabs(sp.ctom)) : 0.f;
    const size_t nc = (size_t)c->ncells;
    PIC_CUDA(cudaMalloc(&sp.base, (nc + 1) * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.base_next, (nc + 1) * sizeof(uint32_t)));
    for (int b = 0; b < 2; ++b) {
        PIC_CUDA(cudaMalloc(&sp.front[b], nc * sizeof(uint32_t)));
        PIC_CUDA(cudaMalloc(&sp.back[b], nc * sizeof(uint32_t)));
        PIC_CUDA(cudaMemsetAsync(sp.front[b], 0, nc * sizeof(uint32_t), c->stream));
        PIC_CUDA(cudaMemsetAsync(sp.back[b], 0, nc * sizeof(uint32_t), c->stream));
    }
    PIC_CUDA(cudaMalloc(&sp.cnt, nc * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.dense, (nc + 1) * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.list_counts, 4 * sizeof(uint32_t)));
    PIC_CUDA(cudaMemsetAsync(sp.list_counts, 0, 4 * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMalloc(&sp.acc_q, (size_t)c->nodes * sizeof(unsigned long long)));
    PIC_CUDA(cudaMalloc(&sp.acc_e, (size_t)c->nodes * sizeof(unsigned long long)));
    PIC_CUDA(cudaMalloc(&sp.final_mesh, (size_t)c->nodes * sizeof(double)));
    PIC_CUDA(cudaMalloc(&sp.energy_mesh, (size_t)c->nodes * sizeof(double)));
    PIC_CUDA(cudaMalloc(&sp.counters, 4 * sizeof(unsigned long long)));
    PIC_CUDA(cudaMallocHost(&sp.host_flags, 16 * sizeof(uint32_t)));
    std::memset(sp.host_flags, 0, 16 * sizeof(uint32_t));
    PIC_CUDA(cudaEventCreateWithFlags(&sp.flags_ev, cudaEventDisableTiming));
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.final_mesh, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.energy_mesh, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.counters, 0, 4 * sizeof(unsigned long long), c->stream));
    // an empty layout: every cell owns cell_capacity(0) slots
    PIC_CUDA(cudaMemsetAsync(sp.cnt, 0, nc * sizeof(uint32_t), c->stream));
    uint32_t total = 0;
    PIC_TRY(scan_cells<true>(c, sp, sp.cnt, sp.base, &total));
    PIC_TRY(grow_store(c, s, total));
    PIC_TRY(grow_lists(c, s));
    PIC_CUDA((carveouts<kPush, true>()));
    PIC_CUDA((carveouts<kPush, false>()));
    PIC_CUDA((carveouts<kDeposit, true>()));
    PIC_CUDA((carveouts<kDeposit, false>()));
    sp.acc_fresh = true;  // zero particles: the zero accumulator is their deposit
    return PIC_OK;
}

void species_free(Species& sp) {
    cudaFree(sp.store);
    cudaFree(sp.base);
    cudaFree(sp.base_next);
    for (int b = 0; b < 2; ++b) {
        cudaFree(sp.front[b]);
        cudaFree(sp.back[b]);
    }
    cudaFree(sp.cnt);
    cudaFree(sp.dense);
    cudaFree(sp.list_counts);
    list_free(sp.ovf);
    list_free(sp.loose[0]);
    list_free(sp.loose[1]);
    if (sp.host_flags) cudaFreeHost(sp.host_flags);
    if (sp.flags_ev) cudaEventDestroy(sp.flags_ev);
    cudaFree(sp.acc_q);
    cudaFree(sp.acc_e);
    cudaFree(sp.final_mesh);
    cudaFree(sp.energy_mesh);
    cudaFree(sp.counters);
    sp = Species{};
}

// Grows the buffers to `capacity` slots each, keeping the current buffer's
// contents (same layout).
static int grow_store(pic_ctx* c, int s, int64_t capacity) {
    Species& sp = c->sp[s];
    if (capacity <= sp.capacity && sp.store) return PIC_OK;
    // multiples of 64 slots keep both buffers' float4 arrays 256-byte aligned
    capacity = (capacity + 63) & ~(int64_t)63;
    if (capacity > (int64_t)0xF0000000ll)
        return fail(PIC_ERR_CAPACITY, "a species holds at most 4.0e9 particle slots (32-bit indices)");
    float* store = nullptr;
    PIC_CUDA(cudaMalloc(&store, (size_t)capacity * 2 * 5 * sizeof(float)));
    ParticleSoA nb[2];
    for (int b = 0; b < 2; ++b) {
        nb[b].a = reinterpret_cast<float4*>(store + (size_t)b * capacity * 5);
        nb[b].vz = store + (size_t)b * capacity * 5 + (size_t)capacity * 4;
    }
    if (sp.store && sp.capacity > 0) {
        PIC_CUDA(cudaMemcpyAsync(nb[sp.cur].a, sp.buf[sp.cur].a, (size_t)sp.capacity * sizeof(float4),
                                 cudaMemcpyDeviceToDevice, c->stream));
        PIC_CUDA(cudaMemcpyAsync(nb[sp.cur].vz, sp.buf[sp.cur].vz, (size_t)sp.capacity * sizeof(float),
                                 cudaMemcpyDeviceToDevice, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
    }
    cudaFree(sp.store);
    sp.store = store;
    sp.buf[0] = nb[0];
    sp.buf[1] = nb[1];
    sp.capacity = capacity;
    return PIC_OK;
}

// Sizes the side lists for the current capacity; only called while they
// are empty.
static int grow_lists(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    const uint32_t lc = list_capacity(sp.capacity);
    if (lc <= sp.ovf.cap) return PIC_OK;
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    PIC_TRY(list_alloc(sp.ovf, lc, sp.list_counts + kOvf));
    PIC_TRY(list_alloc(sp.loose[0], lc, sp.list_counts + kLoose0));
    PIC_TRY(list_alloc(sp.loose[1], lc, sp.list_counts + kLoose1));
    return PIC_OK;
}

static int normalize(pic_ctx* c, int s);

int species_reserve(pic_ctx* c, int s, int64_t capacity) {
    Species& sp = c->sp[s];
    if (sp.store) PIC_TRY(normalize(c, s));  // side lists empty before they are resized
    PIC_TRY(grow_store(c, s, capacity));
    return grow_lists(c, s);
}

namespace {

// Reads the loose-list count and error flags recorded after the last push.
// sync: wait for them; otherwise only look when they are already there.
int check_flags(pic_ctx* c, Species& sp, bool sync) {
    if (!sp.flags_pending) return PIC_OK;
    if (sync) {
        PIC_CUDA(cudaEventSynchronize(sp.flags_ev));
    } else {
        const cudaError_t e = cudaEventQuery(sp.flags_ev);
        if (e == cudaErrorNotReady) return PIC_OK;
        if (e != cudaSuccess) return fail(PIC_ERR_CUDA, std::string("flags event: ") + cudaGetErrorString(e));
    }
    sp.flags_pending = false;
    const unsigned long long* fl = reinterpret_cast<const unsigned long long*>(sp.host_flags + 4);
    if (fl[1]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    if (fl[2]) return fail(PIC_ERR_CAPACITY, "particle side list overflowed: particles were lost");
    return PIC_OK;
}

}  // namespace

// Rebuilds the layout from the current per-cell counts (cell runs plus the
// side list): every cell gets cell_capacity(count) slots with its particles
// at the front.  Synchronises.
static int relayout(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    const int64_t nc = c->ncells;
    const int src = sp.cur;
    const ListDev L = list_dev(sp.loose[sp.lcur]);
    k_cell_counts<<<grid1d(nc, 256), 256, 0, c->stream>>>(sp.front[src], sp.back[src], nc, sp.cnt);
    k_list_counts<<<kFixupBlocks, 256, 0, c->stream>>>(L, sp.cnt);
    c->launches += 2;
    uint32_t total = 0;
    PIC_TRY(scan_cells<true>(c, sp, sp.cnt, sp.base_next, &total));
    const int dst = src ^ 1;
    if ((int64_t)total > sp.capacity) {
        // grow: a fresh store, the old current buffer copied into its buffer
        // `src` first (same layout), then rebuilt into `dst` as usual
        PIC_TRY(grow_store(c, s, (int64_t)total + total / 8));
    }
    k_relayout_cells<<<grid1d(nc, 8), 256, 0, c->stream>>>(
        sp.buf[src].a, sp.buf[src].vz, sp.base, sp.front[src], sp.back[src], sp.base_next, nc,
        sp.buf[dst].a, sp.buf[dst].vz, sp.front[dst], sp.back[dst]);
    k_relayout_list<<<kFixupBlocks, 256, 0, c->stream>>>(L, sp.base_next, sp.front[dst], sp.buf[dst].a,
                                                         sp.buf[dst].vz);
    c->launches += 2;
    PIC_CUDA(cudaGetLastError());
    PIC_CUDA(cudaMemsetAsync(sp.list_counts, 0, 4 * sizeof(uint32_t), c->stream));
    std::swap(sp.base, sp.base_next);
    sp.cur = dst;
    sp.lcur = 0;
    sp.flags_pending = false;
    sp.host_flags[0] = 0u;
    unsigned long long flags[3] = {0, 0, 0};
    PIC_CUDA(cudaMemcpyAsync(flags, sp.counters, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (flags[1]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    if (flags[2]) return fail(PIC_ERR_CAPACITY, "particle side list overflowed: particles were lost");
    return grow_lists(c, s);
}

// Every particle in a cell run (side list empty).  Synchronises.
static int normalize(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    PIC_TRY(check_flags(c, sp, true));
    uint32_t n = 0;
    PIC_CUDA(cudaMemcpyAsync(&n, sp.list_counts + kLoose0 + sp.lcur, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (n > 0) PIC_TRY(relayout(c, s));
    return PIC_OK;
}

// cnt = particles per cell, dense = its exclusive scan; *total = particles.
static int count_cells(pic_ctx* c, int s, int64_t* total) {
    Species& sp = c->sp[s];
    PIC_TRY(normalize(c, s));
    k_cell_counts<<<grid1d(c->ncells, 256), 256, 0, c->stream>>>(sp.front[sp.cur], sp.back[sp.cur],
                                                                 c->ncells, sp.cnt);
    c->launches += 1;
    uint32_t t = 0;
    PIC_TRY(scan_cells<false>(c, sp, sp.cnt, sp.dense, &t));
    *total = t;
    return PIC_OK;
}

int ensure_staging(pic_ctx* c, size_t bytes) {
    if (bytes <= c->staging_bytes) return PIC_OK;
    // whole 32 MiB granules: requests of nearly the same size (an export,
    // then an import of the same particles) reuse the buffer
    constexpr size_t kGranule = 32u << 20;
    bytes = (bytes + kGranule - 1) / kGranule * kGranule;
    cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    PIC_CUDA(cudaMalloc(&c->staging, bytes));
    c->staging_bytes = bytes;
    return PIC_OK;
}

int particles_import_staging(pic_ctx* c, int64_t n, PointRec** dev_recs) {
    PIC_TRY(ensure_staging(c, (size_t)n * sizeof(PointRec)));
    *dev_recs = static_cast<PointRec*>(c->staging);
    return PIC_OK;
}

// Installs a fresh layout from sp.cnt (particles per cell): base from the
// cell capacities, growing the buffers when needed.  The current buffer's
// contents are dropped.
static int fresh_layout(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    uint32_t total = 0;
    PIC_TRY(scan_cells<true>(c, sp, sp.cnt, sp.base, &total));
    PIC_CUDA(cudaMemsetAsync(sp.list_counts, 0, 4 * sizeof(uint32_t), c->stream));
    sp.lcur = 0;
    sp.flags_pending = false;
    sp.host_flags[0] = 0u;
    if ((int64_t)total > sp.capacity) {
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(sp.store);
        sp.store = nullptr;
        sp.capacity = 0;
        PIC_TRY(grow_store(c, s, total));
    }
    PIC_TRY(grow_lists(c, s));
    unsigned long long flags[2] = {0, 0};
    PIC_CUDA(cudaMemcpyAsync(flags, sp.counters, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (flags[1]) {
        PIC_CUDA(cudaMemsetAsync(sp.counters + 1, 0, 8, c->stream));
        return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    }
    return PIC_OK;
}

int particles_import(pic_ctx* c, int s, int64_t n) {
    Species& sp = c->sp[s];
    if ((size_t)n * sizeof(PointRec) > c->staging_bytes)
        return fail(PIC_ERR_STATE, "import staging too small");
    const PointRec* recs = static_cast<const PointRec*>(c->staging);
    PIC_CUDA(cudaMemsetAsync(sp.cnt, 0, (size_t)c->ncells * 4, c->stream));
    if (n > 0) k_import_count<<<grid1d(n, 256), 256, 0, c->stream>>>(recs, n, sp.cnt);
    PIC_TRY(fresh_layout(c, s));
    const int b = sp.cur;
    PIC_CUDA(cudaMemsetAsync(sp.front[b], 0, (size_t)c->ncells * 4, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.back[b], 0, (size_t)c->ncells * 4, c->stream));
    if (n > 0)
        k_import_place<<<grid1d(n, 256), 256, 0, c->stream>>>(recs, n, sp.base, sp.front[b],
                                                              sp.buf[b].a, sp.buf[b].vz);
    c->launches += 2;
    PIC_CUDA(cudaGetLastError());
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_export(pic_ctx* c, int s, PointRec* dev_out, int64_t* n_out) {
    Species& sp = c->sp[s];
    int64_t n = 0;
    PIC_TRY(count_cells(c, s, &n));
    *n_out = n;
    if (n == 0) return PIC_OK;
    const int b = sp.cur;
    k_export<<<grid1d(c->ncells, 8), 256, 0, c->stream>>>(sp.buf[b].a, sp.buf[b].vz, sp.base,
                                                          sp.front[b], sp.back[b], sp.dense,
                                                          c->ncells, dev_out);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int particles_export_state(pic_ctx* c, int s, void* dev, int64_t n) {
    Species& sp = c->sp[s];
    int64_t m = 0;
    PIC_TRY(count_cells(c, s, &m));
    if (m != n) return fail(PIC_ERR_STATE, "particle count changed during export");
    if (n == 0) return PIC_OK;
    int32_t* cell = static_cast<int32_t*>(dev);
    float* f = reinterpret_cast<float*>(cell + n);
    const int b = sp.cur;
    k_export_state<<<grid1d(c->ncells, 8), 256, 0, c->stream>>>(
        sp.buf[b].a, sp.buf[b].vz, sp.base, sp.front[b], sp.back[b], sp.dense, c->ncells, cell, f,
        f + n, f + 2 * n, f + 3 * n, f + 4 * n);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int particles_count(pic_ctx* c, int s, int64_t* n) { return count_cells(c, s, n); }

int particles_bin_counts(pic_ctx* c, int s, int32_t* dev_counts) {
    Species& sp = c->sp[s];
    int64_t n = 0;
    PIC_TRY(count_cells(c, s, &n));
    k_bin_counts<<<grid1d(c->nodes, 256), 256, 0, c->stream>>>(sp.cnt, c->nx, c->ny, c->GX, dev_counts);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int particles_load_plasma(pic_ctx* c, int s, const pic_plasma_desc* d) {
    Species& sp = c->sp[s];
    if (d->ppc < 0 || d->temperature_ev < 0 || d->blob_peak_ppc < 0)
        return fail(PIC_ERR_ARG, "plasma description has a negative count or temperature");
    PlasmaArgs P{};
    P.nx = c->nx;
    P.ny = c->ny;
    P.ppc = d->ppc;
    P.blob_peak = d->blob_peak_ppc;
    P.blob_cx = d->blob_cx;
    P.blob_cy = d->blob_cy;
    P.inv_two_sig2 = d->blob_sigma > 0 ? 1.0 / (2.0 * d->blob_sigma * d->blob_sigma) : 0.0;
    P.sigma_v = (float)std::sqrt(1.602176634e-19 * d->temperature_ev / sp.desc.mass);
    P.drift_vx = (float)d->drift_vx;
    P.drift_vy = (float)d->drift_vy;
    P.key = make_uint2((uint32_t)d->seed, (uint32_t)(d->seed >> 32));
    P.species = (uint32_t)s;
    k_plasma_counts<<<grid1d(c->ncells, 256), 256, 0, c->stream>>>(P, c->ncells, sp.cnt);
    c->launches += 1;
    PIC_TRY(scan_cells<false>(c, sp, sp.cnt, sp.dense, nullptr));
    PIC_TRY(fresh_layout(c, s));
    const int b = sp.cur;
    k_plasma_generate<<<grid1d(c->ncells, 8), 256, 0, c->stream>>>(P, sp.dense, sp.base, c->ncells,
                                                                    sp.buf[b].a, sp.buf[b].vz,
                                                                    sp.front[b], sp.back[b]);
    c->launches += 1;
    PIC_CUDA(cudaGetLastError());
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_deposit(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    KArgs A = make_args(c, sp);
    const bool energy = c->cfg.deposit_energy != 0;
    const ListDev L = list_dev(sp.loose[sp.lcur]);
    prof_begin(c, PIC_PHASE_DEPOSIT);
    const int sh = c->tile_shape;
    if (energy) {
        launch_cells<kDeposit, true>(sh, tile_grid(c, sh), c->stream, A);
        k_list_deposit<true><<<kFixupBlocks, 256, 0, c->stream>>>(L, c->nx, c->GX, sp.k.half_inv_abs_qm,
                                                                  sp.acc_q, sp.acc_e);
    } else {
        launch_cells<kDeposit, false>(sh, tile_grid(c, sh), c->stream, A);
        k_list_deposit<false><<<kFixupBlocks, 256, 0, c->stream>>>(L, c->nx, c->GX, sp.k.half_inv_abs_qm,
                                                                   sp.acc_q, sp.acc_e);
    }
    prof_end(c, PIC_PHASE_DEPOSIT);
    c->launches += 2;
    PIC_CUDA(cudaGetLastError());
    sp.acc_fresh = true;
    return PIC_OK;
}

int particles_flush_rho(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    const double area = c->dx * c->dy;
    const double qscale = kChargeUnit * area * sp.weighing;
    const double escale = kEnergyUnit * area * sp.weighing;
    const double chrg = -sp.desc.charge / c->cfg.epsilon;
    prof_begin(c, PIC_PHASE_FLUSH);
    c->launches += 1;
    const FlushEntry F{c->nodes, sp.acc_q, sp.acc_e, qscale, escale, chrg, sp.final_mesh,
                       sp.energy_mesh, c->rho, c->cfg.deposit_energy ? 1 : 0};
    k_flush<<<grid1d(c->nodes, 256 * kFlushNodes), 256, 0, c->stream>>>(F);
    prof_end(c, PIC_PHASE_FLUSH);
    PIC_CUDA(cudaGetLastError());
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_push(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    // a side list that keeps growing means the layout no longer fits the
    // particle distribution: rebuild it (looked at without waiting)
    PIC_TRY(check_flags(c, sp, false));
    if (!sp.flags_pending && sp.host_flags[0] > sp.loose[0].cap / 8u) {
        prof_begin(c, PIC_PHASE_RELAYOUT);
        PIC_TRY(relayout(c, s));
        prof_end(c, PIC_PHASE_RELAYOUT);
    }
    KArgs A = make_args(c, sp);
    const int sh = c->tile_shape;
    const dim3 g = tile_grid(c, sh);
    const bool energy = c->cfg.deposit_energy != 0;
    const int dst = sp.cur ^ 1;
    PIC_CUDA(cudaMemsetAsync(sp.back[dst], 0, (size_t)c->ncells * 4, c->stream));
    // the accumulators collect the deposit of the new positions
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    prof_begin(c, PIC_PHASE_PUSH);
    if (energy)
        launch_cells<kPush, true>(sh, g, c->stream, A);
    else
        launch_cells<kPush, false>(sh, g, c->stream, A);
    prof_end(c, PIC_PHASE_PUSH);
    PIC_CUDA(cudaGetLastError());
    FixArgs F{};
    F.nx = c->nx;
    F.ny = c->ny;
    F.GX = c->GX;
    F.k = push_consts(c, sp);
    F.fld = c->fld;
    F.dst_a = sp.buf[dst].a;
    F.dst_vz = sp.buf[dst].vz;
    F.base = sp.base;
    F.front = sp.front[dst];
    F.back = sp.back[dst];
    F.ovf = list_dev(sp.ovf);
    F.prev = list_dev(sp.loose[sp.lcur]);
    F.next = list_dev(sp.loose[sp.lcur ^ 1]);
    F.acc_q = sp.acc_q;
    F.acc_e = sp.acc_e;
    F.counters = sp.counters;
    prof_begin(c, PIC_PHASE_FIXUP);
    if (energy)
        k_fixup<true><<<kFixupBlocks, 256, 0, c->stream>>>(F);
    else
        k_fixup<false><<<kFixupBlocks, 256, 0, c->stream>>>(F);
    prof_end(c, PIC_PHASE_FIXUP);
    PIC_CUDA(cudaGetLastError());
    c->launches += 2;
    // the consumed lists start empty next time
    PIC_CUDA(cudaMemsetAsync(sp.list_counts + kOvf, 0, sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.list_counts + kLoose0 + sp.lcur, 0, sizeof(uint32_t), c->stream));
    sp.lcur ^= 1;
    sp.cur = dst;
    // side-list size and error flags, read back without waiting
    PIC_CUDA(cudaMemcpyAsync(sp.host_flags, sp.list_counts + kLoose0 + sp.lcur, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaMemcpyAsync(sp.host_flags + 4, sp.counters, 3 * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaEventRecord(sp.flags_ev, c->stream));
    sp.flags_pending = true;
    sp.acc_fresh = true;
    return PIC_OK;
}

}  // namespace picb200

// ---------------------------------------------------------------------------
// Tile-shape autotuning
// ---------------------------------------------------------------------------
namespace picb200 {

int particles_num_tile_shapes() { return kNumTileShapes; }

// Times `reps` push passes of every species with each tile shape on the
// current particles, without committing them (no buffer swap, no side-list
// placement), then restores what the passes touched: the side-list count,
// the counters, and the accumulators (marked stale, so the next
// charge_deposition redeposits).  ms[k] = mean milliseconds of one pass over
// all species with shape k.
int particles_time_shapes(pic_ctx* c, int reps, double* ms) {
    if (!c->fields_valid) PIC_TRY(fields_from_phi(c));
    const int ns = c->cfg.num_species;
    unsigned long long* saved = nullptr;
    PIC_CUDA(cudaMalloc(&saved, (size_t)ns * 4 * sizeof(unsigned long long)));
    for (int s = 0; s < ns; ++s)
        PIC_CUDA(cudaMemcpyAsync(saved + 4 * s, c->sp[s].counters, 4 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, c->stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PIC_CUDA(cudaEventCreate(&e0));
    PIC_CUDA(cudaEventCreate(&e1));
    int status = PIC_OK;
    const bool energy = c->cfg.deposit_energy != 0;
    for (int sh = 0; sh < kNumTileShapes && status == PIC_OK; ++sh) {
        float total = 0.f;
        for (int r = -1; r < reps; ++r) {  // r = -1: warm-up
            cudaEventRecord(e0, c->stream);
            for (int s = 0; s < ns; ++s) {
                Species& sp = c->sp[s];
                KArgs A = make_args(c, sp);
                cudaMemsetAsync(sp.back[sp.cur ^ 1], 0, (size_t)c->ncells * 4, c->stream);
                cudaMemsetAsync(sp.list_counts + kOvf, 0, sizeof(uint32_t), c->stream);
                if (energy)
                    launch_cells<kPush, true>(sh, tile_grid(c, sh), c->stream, A);
                else
                    launch_cells<kPush, false>(sh, tile_grid(c, sh), c->stream, A);
            }
            cudaEventRecord(e1, c->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
                status = fail(PIC_ERR_CUDA, "autotune: push launch failed");
                break;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r >= 0) total += t;
        }
        if (ms) ms[sh] = total / (float)std::max(reps, 1);
    }
    for (int s = 0; s < ns; ++s) {
        Species& sp = c->sp[s];
        cudaMemcpyAsync(sp.counters, saved + 4 * s, 4 * sizeof(unsigned long long),
                        cudaMemcpyDeviceToDevice, c->stream);
        cudaMemsetAsync(sp.list_counts + kOvf, 0, sizeof(uint32_t), c->stream);
        sp.acc_fresh = false;
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(saved);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PIC_CUDA(cudaGetLastError());
    return status;
}

}  // namespace picb200

// ---------------------------------------------------------------------------
// Batched particle phases: one launch per phase over the contexts of an
// ensemble (same device, same stream).  Per-instance arguments live in
// device tables rebuilt by the host before each step; the kernels only read
// them, so a captured step replays with the tables of the next step.
// ---------------------------------------------------------------------------
namespace picb200 {
namespace {

struct ZeroEntry {
    uint32_t* ptr;
    uint64_t words;  // 4-byte words
};

__global__ void k_batch_zero(const ZeroEntry* __restrict__ e, int n) {
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t gsize = (int64_t)gridDim.x * blockDim.x;
    for (int i = 0; i < n; ++i) {
        const ZeroEntry z = e[i];
        for (int64_t w = gtid; w < (int64_t)z.words; w += gsize) z.ptr[w] = 0u;
    }
}

// Every species of every instance: block (x, i) works on kFlushNodes x 256
// nodes of instance i, each thread on the same nodes of every species in
// turn (species order, as rho sums them one species at a time).
// e[s * n + i]: species s of instance i.
__global__ void k_batch_flush(const FlushEntry* __restrict__ e, int n, int ns) {
    const int i = blockIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x * kFlushNodes + threadIdx.x;
    if (i0 >= e[i].nodes) return;
    for (int s = 0; s < ns; ++s) flush_nodes(e[(size_t)s * n + i], i0, blockDim.x);
}

constexpr int kFixupBlocksPerInstance = 4;

template <bool ENERGY>
__global__ void __launch_bounds__(256) k_fixup_batch(const FixArgs* __restrict__ args) {
    // the single-instance body reads blockIdx.x / gridDim.x: emulate them
    const int inst = blockIdx.x / kFixupBlocksPerInstance;
    const FixArgs F = args[inst];
    const uint32_t n_prev = min(*F.prev.count, F.prev.cap);
    const uint32_t n_ovf = min(*F.ovf.count, F.ovf.cap);
    const uint32_t total = n_prev + n_ovf;
    const uint32_t b = blockIdx.x % kFixupBlocksPerInstance;
    for (uint32_t i = b * blockDim.x + threadIdx.x; i < total; i += kFixupBlocksPerInstance * blockDim.x) {
        Pushed p;
        float vz;
        uint32_t t;
        if (i < n_prev) {
            const uint32_t c = F.prev.cell[i];
            const int gx = (int)(c % (uint32_t)F.nx), gy = (int)(c / (uint32_t)F.nx);
            const int64_t n0 = (int64_t)gy * F.GX + gx;
            vz = F.prev.vz[i];
            p = push_one(F.prev.a[i], F.fld[n0], F.fld[n0 + 1], F.fld[n0 + F.GX], F.fld[n0 + F.GX + 1],
                         F.k, gx, gy, F.nx, F.ny);
            if (p.dir < 0) {
                if (p.left) atomicAdd(F.counters, 1ull);
                continue;
            }
            const float en = ENERGY ? energy_ev(p.vx, p.vy, vz, F.k.half_inv_abs_qm) : 0.f;
            deposit_one<ENERGY>(F.acc_q, F.acc_e, F.GX, (uint32_t)(p.gy * F.GX + p.gx), p.fx, p.fy, en);
            t = (uint32_t)(p.gy * F.nx + p.gx);
        } else {
            const uint32_t e = i - n_prev;
            const float4 a = F.ovf.a[e];
            p.fx = a.x; p.fy = a.y; p.vx = a.z; p.vy = a.w;
            vz = F.ovf.vz[e];
            t = F.ovf.cell[e];
        }
        const uint32_t lim = (F.base[t + 1] - F.base[t]) - F.front[t];
        const uint32_t k = atomicAdd(F.back + t, 1u);
        if (k < lim) {
            store_slot(F.dst_a, F.dst_vz, F.base[t + 1] - 1u - k, p, vz);
        } else {
            atomicSub(F.back + t, 1u);
            const uint32_t s = atomicAdd(F.next.count, 1u);
            if (s < F.next.cap) {
                F.next.a[s] = make_float4(p.fx, p.fy, p.vx, p.vy);
                F.next.vz[s] = vz;
                F.next.cell[s] = t;
            } else {
                atomicOr(F.counters + 2, 1ull);
            }
        }
    }
}

// flags[i] = {loose count (new current list), left exits lo/hi, cell-limit, lost}
struct FlagEntry {
    const uint32_t* loose_count;
    const unsigned long long* counters;
};

__global__ void k_batch_flags(const FlagEntry* __restrict__ e, int n, unsigned long long* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[4 * i] = *e[i].loose_count;
    out[4 * i + 1] = e[i].counters[0];
    out[4 * i + 2] = e[i].counters[1];
    out[4 * i + 3] = e[i].counters[2];
}

}  // namespace

struct ParticleBatchImpl {
    int n = 0, ns = 0;
    uint2* work[kNumTileShapes] = {};
    unsigned nblocks[kNumTileShapes] = {};
    KArgs* d_args = nullptr;      // [ns][n]
    FixArgs* d_fix = nullptr;     // [ns][n]
    FlushEntry* d_flush = nullptr;  // [ns][n]
    ZeroEntry* d_zero = nullptr;  // [ns][3n] before each push, [ns][2n] after, [n] rho
    FlagEntry* d_flagsrc = nullptr;  // [ns][n]
    unsigned long long* d_flags = nullptr;  // [ns][n][4]
    // pinned host mirrors (one upload per step)
    char* h_tables = nullptr;
    char* d_tables = nullptr;
    size_t table_bytes = 0;
    unsigned long long* h_flags = nullptr;
    int64_t max_nodes = 0;  // nodes of the largest instance
};

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int batch_create(pic_ctx** cs, int n, ParticleBatchImpl** out) {
    auto* B = new ParticleBatchImpl();
    *out = B;
    B->n = n;
    B->ns = cs[0]->cfg.num_species;
    for (int i = 0; i < n; ++i) B->max_nodes = std::max<int64_t>(B->max_nodes, cs[i]->nodes);
    for (int sh = 0; sh < kNumTileShapes; ++sh) {
        std::vector<uint2> w;
        for (int i = 0; i < n; ++i) {
            const dim3 g = tile_grid(cs[i], sh);
            for (unsigned y = 0; y < g.y; ++y)
                for (unsigned x = 0; x < g.x; ++x) w.push_back(make_uint2((uint32_t)i, x | (y << 16)));
        }
        B->nblocks[sh] = (unsigned)w.size();
        PIC_CUDA(cudaMalloc(&B->work[sh], w.size() * sizeof(uint2)));
        PIC_CUDA(cudaMemcpy(B->work[sh], w.data(), w.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    const int ns = B->ns;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        const size_t o = off;
        off += align256(bytes);
        return o;
    };
    const size_t o_args = carve(sizeof(KArgs) * ns * n), o_fix = carve(sizeof(FixArgs) * ns * n);
    const size_t o_flush = carve(sizeof(FlushEntry) * ns * n), o_zero = carve(sizeof(ZeroEntry) * (ns * 5 * n + n));
    const size_t o_flag = carve(sizeof(FlagEntry) * ns * n);
    B->table_bytes = off;
    PIC_CUDA(cudaMalloc(&B->d_tables, off));
    PIC_CUDA(cudaMallocHost(&B->h_tables, off));
    std::memset(B->h_tables, 0, off);
    B->d_args = reinterpret_cast<KArgs*>(B->d_tables + o_args);
    B->d_fix = reinterpret_cast<FixArgs*>(B->d_tables + o_fix);
    B->d_flush = reinterpret_cast<FlushEntry*>(B->d_tables + o_flush);
    B->d_zero = reinterpret_cast<ZeroEntry*>(B->d_tables + o_zero);
    B->d_flagsrc = reinterpret_cast<FlagEntry*>(B->d_tables + o_flag);
    PIC_CUDA(cudaMalloc(&B->d_flags, sizeof(unsigned long long) * 4 * ns * n));
    PIC_CUDA(cudaMallocHost(&B->h_flags, sizeof(unsigned long long) * 4 * ns * n));
    std::memset(B->h_flags, 0, sizeof(unsigned long long) * 4 * ns * n);
    return PIC_OK;
}

void batch_destroy(ParticleBatchImpl* B) {
    if (!B) return;
    for (auto* w : B->work) cudaFree(w);
    cudaFree(B->d_tables);
    cudaFree(B->d_flags);
    if (B->h_tables) cudaFreeHost(B->h_tables);
    if (B->h_flags) cudaFreeHost(B->h_flags);
    delete B;
}

// Host part before a step: side-list checks (and rare re-layouts) per
// instance, then the tables of this step, uploaded on `st`.
int batch_prepare(ParticleBatchImpl* B, pic_ctx** cs, cudaStream_t st) {
    const int n = B->n, ns = B->ns;
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < ns; ++s) {
            Species& sp = cs[i]->sp[s];
            const unsigned long long* f = B->h_flags + 4 * ((size_t)s * n + i);
            if (f[2]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
            if (f[3]) return fail(PIC_ERR_CAPACITY, "particle side list overflowed: particles were lost");
            if (f[0] > sp.loose[0].cap / 8u) {
                PIC_TRY(relayout(cs[i], s));
                B->h_flags[4 * ((size_t)s * n + i)] = 0;
            }
        }
    const size_t o_args = 0, o_fix = align256(sizeof(KArgs) * ns * n);
    const size_t o_flush = o_fix + align256(sizeof(FixArgs) * ns * n);
    const size_t o_zero = o_flush + align256(sizeof(FlushEntry) * ns * n);
    const size_t o_flag = o_zero + align256(sizeof(ZeroEntry) * (ns * 5 * n + n));
    KArgs* ha = reinterpret_cast<KArgs*>(B->h_tables + o_args);
    FixArgs* hf = reinterpret_cast<FixArgs*>(B->h_tables + o_fix);
    FlushEntry* hl = reinterpret_cast<FlushEntry*>(B->h_tables + o_flush);
    ZeroEntry* hz = reinterpret_cast<ZeroEntry*>(B->h_tables + o_zero);
    FlagEntry* hg = reinterpret_cast<FlagEntry*>(B->h_tables + o_flag);
    for (int i = 0; i < n; ++i) {
        pic_ctx* c = cs[i];
        hz[(size_t)ns * 5 * n + i] = ZeroEntry{reinterpret_cast<uint32_t*>(c->rho), (uint64_t)c->nodes * 2};
        for (int s = 0; s < ns; ++s) {
            Species& sp = c->sp[s];
            const size_t k = (size_t)s * n + i;
            const int dst = sp.cur ^ 1;
            ha[k] = make_args(c, sp);
            FixArgs& F = hf[k];
            F = FixArgs{};
            F.nx = c->nx;
            F.ny = c->ny;
            F.GX = c->GX;
            F.k = push_consts(c, sp);
            F.fld = c->fld;
            F.dst_a = sp.buf[dst].a;
            F.dst_vz = sp.buf[dst].vz;
            F.base = sp.base;
            F.front = sp.front[dst];
            F.back = sp.back[dst];
            F.ovf = list_dev(sp.ovf);
            F.prev = list_dev(sp.loose[sp.lcur]);
            F.next = list_dev(sp.loose[sp.lcur ^ 1]);
            F.acc_q = sp.acc_q;
            F.acc_e = sp.acc_e;
            F.counters = sp.counters;
            const double area = c->dx * c->dy;
            hl[k] = FlushEntry{c->nodes, sp.acc_q, sp.acc_e, kChargeUnit * area * sp.weighing,
                               kEnergyUnit * area * sp.weighing, -sp.desc.charge / c->cfg.epsilon,
                               sp.final_mesh, sp.energy_mesh, c->rho, c->cfg.deposit_energy ? 1 : 0};
            // before the push: back counts of the new buffer, the accumulators
            ZeroEntry* zb = hz + (size_t)s * 5 * n;
            zb[i] = ZeroEntry{sp.back[dst], (uint64_t)c->ncells};
            zb[n + i] = ZeroEntry{reinterpret_cast<uint32_t*>(sp.acc_q), (uint64_t)c->nodes * 2};
            zb[2 * n + i] = ZeroEntry{reinterpret_cast<uint32_t*>(sp.acc_e), (uint64_t)c->nodes * 2};
            // after the fix-up: the consumed side lists
            zb[3 * n + i] = ZeroEntry{sp.list_counts + kOvf, 1};
            zb[4 * n + i] = ZeroEntry{sp.list_counts + kLoose0 + sp.lcur, 1};
            hg[k] = FlagEntry{sp.list_counts + kLoose0 + (sp.lcur ^ 1), sp.counters};
        }
    }
    PIC_CUDA(cudaMemcpyAsync(B->d_tables, B->h_tables, B->table_bytes, cudaMemcpyHostToDevice, st));
    return PIC_OK;
}

// zero rho of every instance; flush the accumulators of every species into
// final/energy mesh and rho (charge_deposition).
int batch_deposit(ParticleBatchImpl* B, cudaStream_t st) {
    const int n = B->n, ns = B->ns;
    k_batch_zero<<<296, 256, 0, st>>>(B->d_zero + (size_t)ns * 5 * n, n);
    const dim3 fg(grid1d(B->max_nodes, 256 * kFlushNodes), (unsigned)n);
    k_batch_flush<<<fg, 256, 0, st>>>(B->d_flush, n, ns);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

// push every species of every instance, then gather the side-list counts and
// flags for the host (copied into B->h_flags on `st`).
int batch_push(ParticleBatchImpl* B, int shape, bool energy, cudaStream_t st) {
    const int n = B->n, ns = B->ns;
    for (int s = 0; s < ns; ++s) {
        k_batch_zero<<<296, 256, 0, st>>>(B->d_zero + (size_t)s * 5 * n, 3 * n);
        if (energy)
            launch_cells_batch<kPush, true>(shape, B->nblocks[shape], st, B->d_args + (size_t)s * n, B->work[shape]);
        else
            launch_cells_batch<kPush, false>(shape, B->nblocks[shape], st, B->d_args + (size_t)s * n, B->work[shape]);
        if (energy)
            k_fixup_batch<true><<<n * kFixupBlocksPerInstance, 256, 0, st>>>(B->d_fix + (size_t)s * n);
        else
            k_fixup_batch<false><<<n * kFixupBlocksPerInstance, 256, 0, st>>>(B->d_fix + (size_t)s * n);
        k_batch_zero<<<1, 256, 0, st>>>(B->d_zero + (size_t)s * 5 * n + 3 * n, 2 * n);
    }
    k_batch_flags<<<(ns * n + 127) / 128, 128, 0, st>>>(B->d_flagsrc, ns * n, B->d_flags);
    PIC_CUDA(cudaMemcpyAsync(B->h_flags, B->d_flags, sizeof(unsigned long long) * 4 * ns * n,
                             cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

// Host bookkeeping after a step (the buffers and lists every push flips).
void batch_commit(pic_ctx** cs, int n) {
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < cs[i]->cfg.num_species; ++s) {
            Species& sp = cs[i]->sp[s];
            sp.cur ^= 1;
            sp.lcur ^= 1;
            sp.acc_fresh = true;
            sp.flags_pending = false;
        }
}

}  // namespace picb200

namespace picb200 {

// Times `reps` batched push passes of all species with each tile shape on the
// current particles of every instance, without committing them; restores
// the counters and side-list counts the passes touched and marks the
// accumulators stale.  Tables must be prepared (batch_prepare).
int batch_time_shapes(ParticleBatchImpl* B, pic_ctx** cs, cudaStream_t st, int reps, bool energy,
                      double* ms) {
    const int n = B->n, ns = B->ns;
    unsigned long long* saved = nullptr;
    PIC_CUDA(cudaMalloc(&saved, (size_t)n * ns * 4 * sizeof(unsigned long long)));
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < ns; ++s)
            PIC_CUDA(cudaMemcpyAsync(saved + 4 * ((size_t)i * ns + s), cs[i]->sp[s].counters,
                                     4 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PIC_CUDA(cudaEventCreate(&e0));
    PIC_CUDA(cudaEventCreate(&e1));
    int status = PIC_OK;
    for (int sh = 0; sh < kNumTileShapes && status == PIC_OK; ++sh) {
        float total = 0.f;
        for (int r = -1; r < reps; ++r) {
            cudaEventRecord(e0, st);
            for (int s = 0; s < ns; ++s) {
                k_batch_zero<<<296, 256, 0, st>>>(B->d_zero + (size_t)s * 5 * n, 3 * n);
                k_batch_zero<<<1, 256, 0, st>>>(B->d_zero + (size_t)s * 5 * n + 3 * n, n);  // ovf counts
                if (energy)
                    launch_cells_batch<kPush, true>(sh, B->nblocks[sh], st, B->d_args + (size_t)s * n, B->work[sh]);
                else
                    launch_cells_batch<kPush, false>(sh, B->nblocks[sh], st, B->d_args + (size_t)s * n, B->work[sh]);
            }
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
                status = fail(PIC_ERR_CUDA, "autotune: batched push launch failed");
                break;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r >= 0) total += t;
        }
        if (ms) ms[sh] = total / (float)std::max(reps, 1);
    }
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < ns; ++s) {
            Species& sp = cs[i]->sp[s];
            cudaMemcpyAsync(sp.counters, saved + 4 * ((size_t)i * ns + s), 4 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToDevice, st);
            cudaMemsetAsync(sp.list_counts + kOvf, 0, sizeof(uint32_t), st);
            sp.acc_fresh = false;
        }
    cudaStreamSynchronize(st);
    cudaFree(saved);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PIC_CUDA(cudaGetLastError());
    return status;
}

}  // namespace picb200

// ---------------------------------------------------------------------------
// Particle sources: generate_new_electrons and generate_pairs
// (SYCL-PIC-poissonsolver/src/utils.cpp:374-777, called per step by
// src/sycl_pic_ctypes.cpp:212-236).  New particles are drawn on the device
// (Philox-4x32-10, counter = (call, particle, stream)) and appended to the
// species' side list: they are part of the state at once (deposited into
// the accumulators when those hold the current positions) and are placed in
// their cells by the next push or re-layout.
// ---------------------------------------------------------------------------
namespace picb200 {
namespace {

struct SourceArgs {
    int nx, ny, GX;
    double dx, dy, W, H;
    double x_reinject;
    double x11, x22, xm;
    double ve, vi;  // sqrt(2|q/m|T) of electrons and ions
    uint32_t n_reinject, n_pairs;
    uint2 key;
    uint32_t call;
    ListDev e_list, i_list;
    unsigned long long* e_acc_q;
    unsigned long long* e_acc_e;
    unsigned long long* i_acc_q;
    unsigned long long* i_acc_e;
    int deposit_e, deposit_i, energy;
    float e_half_inv_abs_qm, i_half_inv_abs_qm;
    unsigned long long* e_counters;
    unsigned long long* i_counters;
    unsigned* accepted;  // pairs created
};

__device__ __forceinline__ double u01d(uint32_t a, uint32_t b) {
    // 53-bit uniform in [0, 1)
    return (double)(((uint64_t)a << 21) ^ (uint64_t)(b >> 11)) * (1.0 / 9007199254740992.0);
}

// the reference's Maxwellian draw: v * sqrt(-ln u) * (cos, sin)(2 pi u'),
// u clamped below at 1e-10 as ran2 (src/utils.cpp:51-56)
__device__ __forceinline__ void maxwell(double v, uint4 r0, uint4 r1, double& vx, double& vy, double& vz) {
    const double u1 = fmax(u01d(r0.x, r0.y), 1e-10), u2 = u01d(r0.z, r0.w);
    const double u3 = fmax(u01d(r1.x, r1.y), 1e-10), u4 = u01d(r1.z, r1.w);
    const double z1 = sqrt(-log(u1)), z3 = sqrt(-log(u3));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    vx = v * z1 * c;
    vy = v * z1 * s;
    sincospi(2.0 * u4, &s, &c);
    vz = v * z3 * c;
}

// Appends one particle (FP64 position) to a side list, deposit included.
template <bool ENERGY>
__device__ __forceinline__ void append_point(const SourceArgs& S, const ListDev& L, double x, double y,
                                             double vx, double vy, double vz, bool deposit,
                                             unsigned long long* acc_q, unsigned long long* acc_e,
                                             float half_inv_abs_qm, unsigned long long* counters) {
    const double sx = x * (1.0 / S.dx), sy = y * (1.0 / S.dy);
    if (!(sx >= 0.0 && sy >= 0.0 && sx < (double)S.nx && sy < (double)S.ny)) return;
    const int gx = (int)sx, gy = (int)sy;
    const float fx = fminf((float)(sx - gx), kOneBelow), fy = fminf((float)(sy - gy), kOneBelow);
    const uint32_t s = atomicAdd(L.count, 1u);
    if (s >= L.cap) {
        atomicOr(counters + 2, 1ull);
        return;
    }
    L.a[s] = make_float4(fx, fy, (float)vx, (float)vy);
    L.vz[s] = (float)vz;
    L.cell[s] = (uint32_t)(gy * S.nx + gx);
    if (deposit) {
        const float en = ENERGY ? energy_ev((float)vx, (float)vy, (float)vz, half_inv_abs_qm) : 0.f;
        deposit_one<ENERGY>(acc_q, acc_e, S.GX, (uint32_t)(gy * S.GX + gx), fx, fy, en);
    }
}

template <bool ENERGY>
__global__ void k_sources(SourceArgs S) {
    const uint32_t total = S.n_reinject + S.n_pairs;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const uint4 r0 = philox(make_uint4(k, S.call, 0u, 0x50u), S.key);
        const uint4 r1 = philox(make_uint4(k, S.call, 1u, 0x50u), S.key);
        if (k < S.n_reinject) {
            // generate_new_electrons (src/utils.cpp:397-425): x fixed, y uniform
            double vx, vy, vz;
            maxwell(S.ve, r0, r1, vx, vy, vz);
            const uint4 r2 = philox(make_uint4(k, S.call, 2u, 0x50u), S.key);
            append_point<ENERGY>(S, S.e_list, S.x_reinject, S.H * u01d(r2.x, r2.y), vx, vy, vz, S.deposit_e,
                                 S.e_acc_q, S.e_acc_e, S.e_half_inv_abs_qm, S.e_counters);
        } else {
            // generate_pairs (src/utils.cpp:517-566): one electron and one
            // ion at x = xm + asin(2u-1)(x22-x11)/pi, y uniform, kept inside (0, W)
            const uint4 r2 = philox(make_uint4(k, S.call, 2u, 0x50u), S.key);
            const uint4 r3 = philox(make_uint4(k, S.call, 3u, 0x50u), S.key);
            const uint4 r4 = philox(make_uint4(k, S.call, 4u, 0x50u), S.key);
            const double x = S.xm + asin(2.0 * u01d(r2.x, r2.y) - 1.0) * (S.x22 - S.x11) * (1.0 / 3.14159265358979323846);
            const double y = S.H * u01d(r2.z, r2.w);
            if (!(x > 0.0 && x < S.W)) continue;
            double vx, vy, vz;
            maxwell(S.ve, r0, r1, vx, vy, vz);
            append_point<ENERGY>(S, S.e_list, x, y, vx, vy, vz, S.deposit_e, S.e_acc_q, S.e_acc_e,
                                 S.e_half_inv_abs_qm, S.e_counters);
            maxwell(S.vi, r3, r4, vx, vy, vz);
            append_point<ENERGY>(S, S.i_list, x, y, vx, vy, vz, S.deposit_i, S.i_acc_q, S.i_acc_e,
                                 S.i_half_inv_abs_qm, S.i_counters);
            atomicAdd(S.accepted, 1u);
        }
    }
}

}  // namespace

int particles_generate(pic_ctx* c, const pic_source_desc* d, int64_t* n_e, int64_t* n_p) {
    if (c->cfg.num_species < 2) return fail(PIC_ERR_STATE, "particle sources need electrons (species 0) and ions (1)");
    Species& E = c->sp[0];
    Species& I = c->sp[1];
    // re-injection count: electron exits through x < 0 beyond the ions'
    unsigned long long ex[2] = {0, 0};
    PIC_CUDA(cudaMemcpyAsync(&ex[0], E.counters, 8, cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaMemcpyAsync(&ex[1], I.counters, 8, cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    int64_t num_new = 0;
    if (d->reinject) {
        num_new = std::max<int64_t>((int64_t)ex[0] - (int64_t)ex[1], 0);
        PIC_CUDA(cudaMemsetAsync(E.counters, 0, 8, c->stream));
        PIC_CUDA(cudaMemsetAsync(I.counters, 0, 8, c->stream));
    }
    int64_t target = 0;
    if (d->pairs) {
        // fn = H dt (2/pi) (x22 - x11) ionimax / rate_div (src/utils.cpp:502)
        const double fn = c->cfg.ymax * c->cfg.dt * (2.0 / 3.14159265358979323846) * (d->x22 - d->x11) *
                          d->ionimax / d->rate_div;
        if (fn > 0) target = (int64_t)std::ceil(fn);
    }
    if (n_e) *n_e = 0;
    if (n_p) *n_p = 0;
    if (num_new + target == 0) return PIC_OK;
    if (num_new + target > 0x7fffffffll) return fail(PIC_ERR_CAPACITY, "too many new particles in one call");
    // the side lists must hold them: make room first if needed
    for (Species* sp : {&E, &I}) {
        uint32_t n = 0;
        PIC_CUDA(cudaMemcpy(&n, sp->list_counts + 1 + sp->lcur, 4, cudaMemcpyDeviceToHost));
        if ((int64_t)n + num_new + target > (int64_t)sp->loose[sp->lcur].cap)
            return fail(PIC_ERR_CAPACITY, "particle sources: more new particles than the side list holds");
    }
    unsigned* accepted = nullptr;
    PIC_CUDA(cudaMalloc(&accepted, sizeof(unsigned)));
    PIC_CUDA(cudaMemsetAsync(accepted, 0, sizeof(unsigned), c->stream));
    SourceArgs S{};
    S.nx = c->nx;
    S.ny = c->ny;
    S.GX = c->GX;
    S.dx = c->dx;
    S.dy = c->dy;
    S.W = c->cfg.xmax;
    S.H = c->cfg.ymax;
    S.x_reinject = d->reinject_x;
    S.x11 = d->x11;
    S.x22 = d->x22;
    S.xm = d->xm;
    S.ve = std::sqrt(2.0 * std::fabs(E.ctom) * d->te_ev);
    S.vi = std::sqrt(2.0 * std::fabs(I.ctom) * d->ti_ev);
    S.n_reinject = (uint32_t)num_new;
    S.n_pairs = (uint32_t)target;
    S.key = make_uint2((uint32_t)d->seed, (uint32_t)(d->seed >> 32));
    S.call = (uint32_t)c->source_calls++;
    S.e_list = list_dev(E.loose[E.lcur]);
    S.i_list = list_dev(I.loose[I.lcur]);
    S.e_acc_q = E.acc_q;
    S.e_acc_e = E.acc_e;
    S.i_acc_q = I.acc_q;
    S.i_acc_e = I.acc_e;
    S.deposit_e = E.acc_fresh ? 1 : 0;
    S.deposit_i = I.acc_fresh ? 1 : 0;
    S.e_half_inv_abs_qm = E.k.half_inv_abs_qm;
    S.i_half_inv_abs_qm = I.k.half_inv_abs_qm;
    S.e_counters = E.counters;
    S.i_counters = I.counters;
    S.accepted = accepted;
    const unsigned blocks = (unsigned)std::min<int64_t>((num_new + target + 255) / 256, 148 * 8);
    if (c->cfg.deposit_energy)
        k_sources<true><<<blocks, 256, 0, c->stream>>>(S);
    else
        k_sources<false><<<blocks, 256, 0, c->stream>>>(S);
    c->launches += 1;
    unsigned acc_h = 0;
    cudaMemcpyAsync(&acc_h, accepted, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(accepted);
    if (e != cudaSuccess) return fail(PIC_ERR_CUDA, std::string("particle sources: ") + cudaGetErrorString(e));
    // the new particles make the side lists' host-side counts stale
    E.flags_pending = I.flags_pending = false;
    if (n_e) *n_e = num_new;
    if (n_p) *n_p = acc_h;
    return PIC_OK;
}

}  // namespace picb200
