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
// Layout: particles of a species live cell-sorted in a double buffer.  The
// cell of a particle is implied by its position in the buffer: off[c] ..
// off[c+1] is cell c (c = gy*nx + gx).  Each particle is 20 bytes:
//   float4 {fx, fy, vx, vy} (in-cell offsets in [0,1), velocities in m/s)
//   float  vz
//
// One push step of a species is four launches:
//   1. k_particles<COUNT>   -- gather + Boris for every particle, classify as
//      stayer / mover / dead, count stayers per cell and movers per target
//      cell.  Nothing per particle is written.
//   2. k_scan_partials, k_scan_apply -- exclusive scan of the new per-cell
//      counts into the new segment table.
//   3. k_particles<SCATTER> -- the same push again (bit-identical: every
//      float operation is an explicit round-to-nearest intrinsic, so the two
//      passes cannot contract differently), scatter into the other buffer and
//      deposit the NEW positions into the 64-bit fixed-point accumulators.
// The deposit of positions x_{n+1} therefore rides on the push of step n; the
// next charge_deposition only converts the accumulators.  Per particle-step
// the traffic is 20 B (pass 1) + 40 B (pass 2) of HBM.
//
// Work decomposition: a block owns a kTileX x kTileY tile of cells; each warp
// walks whole cells of the tile (field values of the cell's four nodes are
// warp-uniform loads).  Stayers accumulate their deposit in registers and are
// reduced once per cell; movers deposit with shared atomics into the block's
// node tile (kHalo cells of margin) or global atomics beyond it.  The tile is
// flushed once to HBM with 64-bit integer atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "pic_internal.h"

namespace picb200 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = kWarps * 32;
constexpr int kScanTile = 2048;               // cells per scan block
constexpr uint32_t kAxisOne = 1u << kAxisBits;
constexpr float kAxisScale = (float)(1u << kAxisBits);
constexpr float kOneBelow = 0x1.fffffep-1f;   // largest float < 1

enum Mode { kCount = 0, kScatter = 1, kDeposit = 2 };
constexpr int kDirs = 9;      // 3x3 neighbourhood, d = (sy+1)*3 + (sx+1)
constexpr int kStay = 4;      // d of a particle that keeps its cell
constexpr int kFar = 9;       // moved more than one cell in x or y

struct KArgs {
    int nx, ny, GX;
    int64_t ncells;
    SpeciesConsts k;
    const float4* __restrict__ fld;
    const float4* __restrict__ src_a;
    const float* __restrict__ src_vz;
    float4* __restrict__ dst_a;
    float* __restrict__ dst_vz;
    const uint32_t* __restrict__ off;
    uint32_t* dcount;   // [9][ncells]
    const uint32_t* __restrict__ sub;  // [10][ncells]
    uint32_t* farin;
    uint32_t* farcur;
    unsigned long long* acc_q;
    unsigned long long* acc_e;
    unsigned long long* counters;  // [0] left exits, [1] cell overflow, [2] scatter guard
    uint32_t cap;                  // particles the destination buffer holds
    int energy;
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Result of one gather + Boris + position update.
struct Pushed {
    float fx, fy, vx, vy;
    int gx, gy;
    int dir;  // 0..8 near (4 = same cell), kFar, or -1 when absorbed
    bool left;
};

// Bilinear gather of E and Bz from the cell's four nodes plus the Boris push
// of deterministic_mover (src/mover.cpp:123-174) in FP32.  Weights:
// (1-fx)(1-fy), fx(1-fy), (1-fx)fy, fx*fy == the reference's unnormalised
// weights divided by dx*dy.  Every operation is an explicit _rn intrinsic so
// the COUNT and SCATTER passes produce identical bits.
__device__ __forceinline__ Pushed push_one(float4 a, float4 n00, float4 n10, float4 n01,
                                           float4 n11, const SpeciesConsts& k, int gx, int gy,
                                           int nx, int ny) {
    const float fx = a.x, fy = a.y;
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    const float w00 = __fmul_rn(ofx, ofy), w10 = __fmul_rn(fx, ofy);
    const float w01 = __fmul_rn(ofx, fy), w11 = __fmul_rn(fx, fy);
    const float ex = __fmaf_rn(w11, n11.x, __fmaf_rn(w01, n01.x, __fmaf_rn(w10, n10.x, __fmul_rn(w00, n00.x))));
    const float ey = __fmaf_rn(w11, n11.y, __fmaf_rn(w01, n01.y, __fmaf_rn(w10, n10.y, __fmul_rn(w00, n00.y))));
    const float bz = __fmaf_rn(w11, n11.z, __fmaf_rn(w01, n01.z, __fmaf_rn(w10, n10.z, __fmul_rn(w00, n00.z))));
    // Boris rotation about z (src/mover.cpp:151-162).
    const float ax = __fmul_rn(k.h, ex), ay = __fmul_rn(k.h, ey);
    const float vxm = __fadd_rn(a.z, ax), vym = __fadd_rn(a.w, ay);
    const float t = __fmul_rn(k.h, bz);
    const float vxp = __fmaf_rn(vym, t, vxm);
    const float vyp = __fmaf_rn(-vxm, t, vym);
    // s = 2t/(1+t^2) with the approximate reciprocal: both passes compute the
    // same bits, and its error (~1 ulp) is far below the FP32 state's
    const float s = __fdividef(__fmul_rn(2.0f, t), __fmaf_rn(t, t, 1.0f));
    Pushed o;
    o.vx = __fadd_rn(__fmaf_rn(vyp, s, vxm), ax);
    o.vy = __fadd_rn(__fmaf_rn(-vxp, s, vym), ay);
    // Position update in cell units (src/mover.cpp:164-165), then re-cell.
    const float px = __fmaf_rn(o.vx, k.dtdx, fx);
    const float py = __fmaf_rn(o.vy, k.dtdy, fy);
    if (px >= -1.0f && px < 2.0f && py >= -1.0f && py < 2.0f) {
        // moved at most one cell per axis: floor(p) in {-1, 0, 1}
        const int sx = (px >= 1.0f) - (px < 0.0f);
        const int sy = (py >= 1.0f) - (py < 0.0f);
        const int ngx = gx + sx, ngy = gy + sy;
        // absorbing walls (src/mover.cpp:325): outside [0,W) x [0,H)
        const bool alive = ngx >= 0 && ngx < nx && ngy >= 0 && ngy < ny;
        o.left = ngx < 0;
        o.gx = ngx;
        o.gy = ngy;
        o.dir = alive ? (sy + 1) * 3 + (sx + 1) : -1;
        const float fsx = (px >= 1.0f) ? 1.0f : ((px < 0.0f) ? -1.0f : 0.0f);
        const float fsy = (py >= 1.0f) ? 1.0f : ((py < 0.0f) ? -1.0f : 0.0f);
        o.fx = fminf(__fsub_rn(px, fsx), kOneBelow);
        o.fy = fminf(__fsub_rn(py, fsy), kOneBelow);
    } else {
        // far jump, or NaN (which lands outside)
        const float fsx = floorf(px), fsy = floorf(py);
        const float ngx = __fadd_rn((float)gx, fsx), ngy = __fadd_rn((float)gy, fsy);
        const bool alive = (ngx >= 0.0f) && (ngx < (float)nx) && (ngy >= 0.0f) && (ngy < (float)ny);
        o.left = !(ngx >= 0.0f);
        o.gx = alive ? (int)ngx : gx;
        o.gy = alive ? (int)ngy : gy;
        const int ix = o.gx - gx, iy = o.gy - gy;
        o.dir = !alive ? -1 : ((ix < -1 || ix > 1 || iy < -1 || iy > 1) ? kFar : (iy + 1) * 3 + (ix + 1));
        o.fx = fminf(__fsub_rn(px, fsx), kOneBelow);
        o.fy = fminf(__fsub_rn(py, fsy), kOneBelow);
    }
    return o;
}

// round(f * 2^20) for f in [0, 1): exact scaling, then the 1.5*2^23 addition
// rounds to nearest-even in the mantissa (integer ALU, no conversion unit).
__device__ __forceinline__ uint32_t axis_fixed(float f) {
    const float t = __fadd_rn(__fmul_rn(f, kAxisScale), 12582912.0f);
    return __float_as_uint(t) - 0x4B400000u;
}

// Fixed-point corner weights of a particle at offsets (fx, fy): exact 40-bit
// products summing to exactly 2^40; e_* are the energy-weighted weights in
// units of 2^-24 eV (en * q/2^40 * 2^24, rounded half up).
struct Weights {
    unsigned long long q00, q10, q01, q11;
    unsigned long long e00, e10, e01, e11;
};

template <bool ENERGY>
__device__ __forceinline__ Weights fixed_weights(float fx, float fy, float en) {
    const uint32_t ax = axis_fixed(fx), ay = axis_fixed(fy);
    const uint32_t bx = kAxisOne - ax, by = kAxisOne - ay;
    Weights w;
    w.q00 = (unsigned long long)bx * by;
    w.q10 = (unsigned long long)ax * by;
    w.q01 = (unsigned long long)bx * ay;
    w.q11 = (unsigned long long)ax * ay;
    if (ENERGY) {
        // energy in units of 2^-22 eV (32 bits, clamped below 1024 eV) times
        // 16-bit axis weights: e = E * wx16 * wy16 / 2^32 < 2^32
        const uint32_t E = __float2uint_rn(__fmul_rn(en, 4194304.0f));
        const uint32_t ax16 = (ax + 8u) >> 4, ay16 = (ay + 8u) >> 4;
        const uint32_t bx16 = 65536u - ax16, by16 = 65536u - ay16;
        const unsigned long long ea = (unsigned long long)E * ax16;
        const unsigned long long eb = (unsigned long long)E * bx16;
        // round to nearest: the products stay below 2^64 - 2^32
        w.e00 = (eb * by16 + 0x80000000ull) >> 32;
        w.e10 = (ea * by16 + 0x80000000ull) >> 32;
        w.e01 = (eb * ay16 + 0x80000000ull) >> 32;
        w.e11 = (ea * ay16 + 0x80000000ull) >> 32;
    } else {
        w.e00 = w.e10 = w.e01 = w.e11 = 0ull;
    }
    return w;
}

// Kinetic energy in eV (0.5 v^2/|q/m|, src/interpolation.cpp:88-89), clamped.
__device__ __forceinline__ float energy_ev(float vx, float vy, float vz, float half_inv_abs_qm) {
    const float v2 = __fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx)));
    return fminf(__fmul_rn(v2, half_inv_abs_qm), kEnergyClampEv);
}

// Global 64-bit integer reductions (fire-and-forget RED) into the node
// accumulators.
__device__ __forceinline__ void red_add(unsigned long long* p, unsigned long long v) {
    atomicAdd(p, v);
}

__device__ __forceinline__ void global_add(const KArgs& A, int gx, int gy, const Weights& w,
                                           bool energy) {
    const int64_t n = (int64_t)gy * A.GX + gx;
    red_add(A.acc_q + n, w.q00);
    red_add(A.acc_q + n + 1, w.q10);
    red_add(A.acc_q + n + A.GX, w.q01);
    red_add(A.acc_q + n + A.GX + 1, w.q11);
    if (energy) {
        red_add(A.acc_e + n, w.e00);
        red_add(A.acc_e + n + 1, w.e10);
        red_add(A.acc_e + n + A.GX, w.e01);
        red_add(A.acc_e + n + A.GX + 1, w.e11);
    }
}

__device__ __forceinline__ void store_particle(const KArgs& A, uint32_t dst, const Pushed& p,
                                               float vz) {
    if (dst < A.cap) {
        __stcs(A.dst_a + dst, make_float4(p.fx, p.fy, p.vx, p.vy));
        __stcs(A.dst_vz + dst, vz);
    } else {
        atomicOr(A.counters + 2, 1ull);
    }
}

// Per-lane fixed-point sums of the stayers of the current cell (64-bit).  A
// cell holds at most kMaxPerCell = 2^16 particles, so a lane sums at most
// 2^11 of them: charge sums stay below 2^51, energy sums below 2^43.  The
// per-cell warp reduction runs on two 32-bit limbs per value with
// redux.sync (26/22-bit low limbs keep every limb sum below 2^32).
struct StayAcc {
    unsigned long long q[4];
    unsigned long long e[4];
};

__device__ __forceinline__ void acc_zero(StayAcc& s) {
#pragma unroll
    for (int k = 0; k < 4; ++k) s.q[k] = s.e[k] = 0ull;
}

template <bool ENERGY>
__device__ __forceinline__ void acc_add(StayAcc& s, const Weights& w) {
    s.q[0] += w.q00; s.q[1] += w.q10; s.q[2] += w.q01; s.q[3] += w.q11;
    if (ENERGY) {
        s.e[0] += w.e00; s.e[1] += w.e10; s.e[2] += w.e01; s.e[3] += w.e11;
    }
}

template <int LO>
__device__ __forceinline__ unsigned long long warp_sum_limbs(unsigned long long v) {
    const uint32_t lo = (uint32_t)(v & ((1ull << LO) - 1ull));
    const uint32_t hi = (uint32_t)(v >> LO);
    return (unsigned long long)__reduce_add_sync(kFull, lo) +
           ((unsigned long long)__reduce_add_sync(kFull, hi) << LO);
}

// Warp-reduce and add the cell's four node sums (lane 0).
template <bool ENERGY>
__device__ __forceinline__ void acc_flush(StayAcc& s, const KArgs& A, int gx, int gy, int lane) {
    Weights w;
    w.q00 = warp_sum_limbs<26>(s.q[0]);
    w.q10 = warp_sum_limbs<26>(s.q[1]);
    w.q01 = warp_sum_limbs<26>(s.q[2]);
    w.q11 = warp_sum_limbs<26>(s.q[3]);
    w.e00 = w.e10 = w.e01 = w.e11 = 0ull;
    if (ENERGY) {
        w.e00 = warp_sum_limbs<22>(s.e[0]);
        w.e10 = warp_sum_limbs<22>(s.e[1]);
        w.e01 = warp_sum_limbs<22>(s.e[2]);
        w.e11 = warp_sum_limbs<22>(s.e[3]);
    }
    if (lane == 0) global_add(A, gx, gy, w, ENERGY);
    acc_zero(s);
}

// One kernel body for the three uses:
//   kCount   -- push, count leavers per direction (plain stores), far movers
//               per target (atomics);
//   kScatter -- push again, place every particle at its deterministic slot
//               (sub-segment of its target cell for its direction + rank
//               within the direction), deposit the new positions;
//   kDeposit -- deposit the current positions (no push).
// A block owns a kTileX x kTileY tile of cells and each warp walks whole
// cells of it: the cell's segment bounds, its four node fields and (scatter)
// the nine destination sub-segment starts are warp-uniform loads; particles
// stream through in chunks of 32 with the next chunk's loads issued before
// the current chunk is processed.
template <int MODE, bool ENERGY>
__global__ void __launch_bounds__(kThreads, (MODE == kScatter && ENERGY) ? 3 : 4) k_particles(KArgs A) {
    constexpr bool kDep = (MODE != kCount);
    __shared__ uint32_t run_s[kWarps][kDirs + 1];
    __shared__ uint32_t base_s[MODE == kScatter ? kWarps : 1][kDirs + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tgx0 = blockIdx.x * kTileX, tgy0 = blockIdx.y * kTileY;
    const unsigned lt = lanemask_lt();
    unsigned long long left_exits = 0;

    for (int lc = warp; lc < kTileX * kTileY; lc += kWarps) {
        const int gx = tgx0 + (lc % kTileX), gy = tgy0 + (lc / kTileX);
        if (gx >= A.nx || gy >= A.ny) continue;  // warp-uniform
        const int64_t c = (int64_t)gy * A.nx + gx;
        const uint32_t beg = A.off[c], end = A.off[c + 1];
        if (beg == end) {
            if (MODE == kCount && lane < kDirs) A.dcount[(int64_t)lane * A.ncells + c] = 0u;
            continue;
        }
        // first chunk's loads go out before the per-cell tables
        uint32_t i = beg + lane;
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        float vz = 0.f;
        if (i < end) {
            a = __ldcs(A.src_a + i);
            if (MODE != kCount) vz = __ldcs(A.src_vz + i);
        }
        float4 f00 = make_float4(0, 0, 0, 0), f10 = f00, f01 = f00, f11 = f00;
        if (MODE != kDeposit) {
            const int64_t n0 = (int64_t)gy * A.GX + gx;
            f00 = __ldg(A.fld + n0);
            f10 = __ldg(A.fld + n0 + 1);
            f01 = __ldg(A.fld + n0 + A.GX);
            f11 = __ldg(A.fld + n0 + A.GX + 1);
        }
        if (lane < kDirs) {
            run_s[warp][lane] = 0u;
            if (MODE == kScatter) {
                const int tx = gx + lane % 3 - 1, ty = gy + lane / 3 - 1;
                base_s[warp][lane] = (tx >= 0 && ty >= 0 && tx < A.nx && ty < A.ny)
                                         ? __ldg(A.sub + (int64_t)lane * A.ncells + (int64_t)ty * A.nx + tx)
                                         : 0u;
            }
        }
        __syncwarp();
        StayAcc acc;
        acc_zero(acc);

        for (uint32_t i0 = beg; i0 < end; i0 += 32) {
            const bool valid = i < end;
            const uint32_t inext = i + 32;
            float4 an = make_float4(0.f, 0.f, 0.f, 0.f);
            float vzn = 0.f;
            if (inext < end) {
                an = __ldcs(A.src_a + inext);
                if (MODE != kCount) vzn = __ldcs(A.src_vz + inext);
            }
            Pushed p;
            if (MODE == kDeposit) {
                p.fx = a.x; p.fy = a.y; p.vx = a.z; p.vy = a.w;
                p.gx = gx; p.gy = gy; p.dir = kStay; p.left = false;
            } else {
                p = push_one(a, f00, f10, f01, f11, A.k, gx, gy, A.nx, A.ny);
            }
            const int dir = valid ? p.dir : -1;
            if (MODE == kScatter) left_exits += __popc(__ballot_sync(kFull, valid && dir < 0 && p.left));
            // rank among this cell's particles leaving in the same direction
            // (warp multi-split: lanes with equal direction bits form a group)
            uint32_t rank = 0;
            {
                const bool ranked = dir >= 0 && dir < kDirs;
                unsigned same = __ballot_sync(kFull, ranked);
#pragma unroll
                for (int bit = 0; bit < 4; ++bit) {
                    const unsigned b = __ballot_sync(kFull, (dir >> bit) & 1);
                    same &= ((dir >> bit) & 1) ? b : ~b;
                }
                const uint32_t before = __popc(same & lt);
                const uint32_t r0 = ranked ? run_s[warp][dir] : 0u;
                rank = r0 + before;
                __syncwarp();
                if (ranked && before == 0) run_s[warp][dir] = r0 + __popc(same);
                __syncwarp();
            }
            if (kDep) {
                const bool live = dir >= 0;
                const float en = (ENERGY && live) ? energy_ev(p.vx, p.vy, vz, A.k.half_inv_abs_qm) : 0.f;
                const Weights w = fixed_weights<ENERGY>(p.fx, p.fy, en);
                if (dir == kStay) acc_add<ENERGY>(acc, w);
                if (MODE == kScatter && live && dir != kStay) global_add(A, p.gx, p.gy, w, ENERGY);
            }
            if (MODE == kScatter && dir >= 0) {
                uint32_t dst;
                if (dir == kFar) {
                    const int64_t nc = (int64_t)p.gy * A.nx + p.gx;
                    dst = __ldg(A.sub + (int64_t)kFar * A.ncells + nc) + atomicAdd(A.farcur + nc, 1u);
                } else {
                    dst = base_s[warp][dir] + rank;
                }
                store_particle(A, dst, p, vz);
            }
            if (MODE == kCount && dir == kFar)
                atomicAdd(A.farin + (int64_t)p.gy * A.nx + p.gx, 1u);
            i = inext;
            a = an;
            vz = vzn;
        }
        if (kDep) acc_flush<ENERGY>(acc, A, gx, gy, lane);
        if (MODE == kCount && lane < kDirs) A.dcount[(int64_t)lane * A.ncells + c] = run_s[warp][lane];
        __syncwarp();
    }
    if (MODE == kScatter && lane == 0 && left_exits) atomicAdd(A.counters, left_exits);
}

// ---- exclusive scan of the new per-cell counts ------------------------------
//
// Cell t receives, from each direction d, the particles that left cell
// t - dir(d) in direction d, plus its far movers.  Its new segment is laid
// out by direction (d = 0..8, then far), so every particle has a
// deterministic slot except far movers (atomic cursor).

struct ScanArgs {
    const uint32_t* dcount;
    uint32_t* farin;
    uint32_t* farcur;
    uint32_t* sub;
    uint32_t* off_next;
    int nx, ny;
    int64_t ncells;
};

__device__ __forceinline__ void incoming(const ScanArgs& S, int64_t t, uint32_t (&in)[kDirs + 1]) {
    const int tx = (int)(t % S.nx), ty = (int)(t / S.nx);
#pragma unroll
    for (int d = 0; d < kDirs; ++d) {
        const int sx = tx - (d % 3 - 1), sy = ty - (d / 3 - 1);
        in[d] = (sx >= 0 && sy >= 0 && sx < S.nx && sy < S.ny)
                    ? S.dcount[(int64_t)d * S.ncells + (int64_t)sy * S.nx + sx]
                    : 0u;
    }
    in[kDirs] = S.farin[t];
}

__global__ void __launch_bounds__(256) k_scan_partials(ScanArgs S, uint32_t* partials) {
    __shared__ uint32_t red[8];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (int j = threadIdx.x; j < kScanTile; j += 256) {
        const int64_t t = base + j;
        if (t >= S.ncells) break;
        uint32_t in[kDirs + 1];
        incoming(S, t, in);
#pragma unroll
        for (int d = 0; d <= kDirs; ++d) s += in[d];
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

// off_next[t] = particles in cells before t; sub[d][t] = start of the part of
// t's segment fed from direction d; off_next[ncells] = total.  Zeroes the far
// counters for the next step and flags cells above kMaxPerCell.
__global__ void __launch_bounds__(256) k_scan_apply(ScanArgs S, const uint32_t* partials,
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
    // each thread owns 8 consecutive cells
    const int64_t c0 = (int64_t)blockIdx.x * kScanTile + threadIdx.x * 8;
    uint32_t tot[8];
    uint32_t tsum = 0, vmax = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        tot[j] = 0;
        if (c0 + j < S.ncells) {
            uint32_t in[kDirs + 1];
            incoming(S, c0 + j, in);
#pragma unroll
            for (int d = 0; d <= kDirs; ++d) tot[j] += in[d];
        }
        tsum += tot[j];
        vmax = max(vmax, tot[j]);
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
        if (t < S.ncells) {
            S.off_next[t] = run;
            uint32_t in[kDirs + 1];
            incoming(S, t, in);
            uint32_t r = run;
#pragma unroll
            for (int d = 0; d <= kDirs; ++d) {
                S.sub[(int64_t)d * S.ncells + t] = r;
                r += in[d];
            }
            S.farin[t] = 0;
            S.farcur[t] = 0;
        }
        run += tot[j];
        if (t == S.ncells - 1) S.off_next[S.ncells] = run;
    }
    if (vmax > kMaxPerCell) atomicOr(counters + 1, 1ull);
}

// ---- import / export ------------------------------------------------------

// Reference Point -> cell + FP32 offsets.  The cell follows InsertKernel:
// gx = (int)(x * (1/dx)) in FP64 (src/particles.cpp:230-235).
__global__ void k_import_convert(const pic_point* __restrict__ pts, int64_t n, int nx, int ny,
                                 double inv_dx, double inv_dy, float4* tmp_a, float* tmp_vz,
                                 uint32_t* cell_of, uint32_t* farin) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const pic_point p = pts[i];
    uint32_t cell = 0xffffffffu;
    if (p.pointer != -1) {
        const double sx = p.x * inv_dx, sy = p.y * inv_dy;
        if (sx >= 0.0 && sy >= 0.0 && sx < (double)nx && sy < (double)ny) {
            const int gx = (int)sx, gy = (int)sy;
            cell = (uint32_t)gy * (uint32_t)nx + (uint32_t)gx;
            const float fx = fminf((float)(sx - gx), kOneBelow);
            const float fy = fminf((float)(sy - gy), kOneBelow);
            tmp_a[i] = make_float4(fx, fy, (float)p.vx, (float)p.vy);
            tmp_vz[i] = (float)p.vz;
        }
    }
    cell_of[i] = cell;
    if (cell != 0xffffffffu) atomicAdd(farin + cell, 1u);
}

__global__ void k_import_scatter(const float4* __restrict__ tmp_a, const float* __restrict__ tmp_vz,
                                 const uint32_t* __restrict__ cell_of, int64_t n,
                                 const uint32_t* __restrict__ off, uint32_t* farcur,
                                 float4* dst_a, float* dst_vz) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = cell_of[i];
    if (c == 0xffffffffu) return;
    const uint32_t d = off[c] + atomicAdd(farcur + c, 1u);
    dst_a[d] = tmp_a[i];
    dst_vz[d] = tmp_vz[i];
}

// Sorted SoA -> reference Point AoS.  x = (gx + fx)*dx in FP64.
__global__ void k_export(const float4* __restrict__ a, const float* __restrict__ vz,
                         const uint32_t* __restrict__ off, int nx, int64_t ncells, double dx,
                         double dy, pic_point* out) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const int gx = (int)(c % nx), gy = (int)(c / nx);
    for (uint32_t i = off[c] + lane; i < off[c + 1]; i += 32) {
        const float4 v = a[i];
        pic_point p;
        p.x = ((double)gx + (double)v.x) * dx;
        p.y = ((double)gy + (double)v.y) * dy;
        p.z = 0.0;
        p.vx = v.z;
        p.vy = v.w;
        p.vz = vz[i];
        p.pointer = (int32_t)i;
        p.pad_ = 0;
        out[i] = p;
    }
}

// Sorted state -> raw arrays (cell, fx, fy, vx, vy, vz), storage order.
__global__ void k_export_state(const float4* __restrict__ a, const float* __restrict__ vz,
                               const uint32_t* __restrict__ off, int64_t ncells, int64_t n,
                               int32_t* cell, float* fx, float* fy, float* vx, float* vy,
                               float* vzo) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    for (uint32_t i = off[c] + lane; i < off[c + 1]; i += 32) {
        const float4 v = a[i];
        cell[i] = (int32_t)c;
        fx[i] = v.x;
        fy[i] = v.y;
        vx[i] = v.z;
        vy[i] = v.w;
        vzo[i] = vz[i];
    }
    (void)n;
}

// Live particles per reference bucket key gy*GRID_X + gx.
__global__ void k_bin_counts(const uint32_t* __restrict__ off, int nx, int ny, int GX,
                             int32_t* counts) {
    const int64_t nodes = (int64_t)GX * (ny + 1);
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    const int gx = (int)(k % GX), gy = (int)(k / GX);
    int32_t v = 0;
    if (gx < nx && gy < ny) {
        const int64_t c = (int64_t)gy * nx + gx;
        v = (int32_t)(off[c + 1] - off[c]);
    }
    counts[k] = v;
}

// ---- accumulators -> meshes -------------------------------------------------

// final_mesh = weighing * sum of unnormalised corner weights; rho += final *
// (-q/eps) (src/interpolation.cpp:139-171).  Resets the accumulators.
__global__ void k_flush(int64_t nodes, unsigned long long* acc_q, unsigned long long* acc_e,
                        double qscale, double escale, double chrg, double* final_mesh,
                        double* energy_mesh, double* rho, int energy) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const double f = (double)acc_q[i] * qscale;
    acc_q[i] = 0ull;
    final_mesh[i] = f;
    if (energy) {
        energy_mesh[i] = (double)acc_e[i] * escale;
        acc_e[i] = 0ull;
    } else {
        energy_mesh[i] = 0.0;
    }
    rho[i] += f * chrg;
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

// counts enter as the "stay" direction of each cell
__global__ void k_plasma_counts(PlasmaArgs P, int64_t ncells, uint32_t* stay_count) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    stay_count[c] = (uint32_t)P.ppc + blob_count(P, c);
}

__global__ void k_plasma_generate(PlasmaArgs P, const uint32_t* __restrict__ off, int64_t ncells,
                                  float4* a, float* vz) {
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (c >= ncells) return;
    const int lane = threadIdx.x & 31;
    const uint32_t beg = off[c], end = off[c + 1];
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
        a[i] = make_float4(fx, fy, vx, vy);
        vz[i] = vzz;
    }
}

inline unsigned grid1d(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int scan_counts(pic_ctx* c, Species& sp) {
    const int64_t ncells = c->ncells;
    const int nparts = (int)((ncells + kScanTile - 1) / kScanTile);
    ScanArgs S{sp.dcount, sp.farin, sp.farcur, sp.sub, sp.off_next, c->nx, c->ny, ncells};
    k_scan_partials<<<nparts, 256, 0, c->stream>>>(S, c->scan_partials);
    k_scan_apply<<<nparts, 256, 0, c->stream>>>(S, c->scan_partials, sp.counters);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

KArgs make_args(pic_ctx* c, Species& sp) {
    KArgs A{};
    A.nx = c->nx;
    A.ny = c->ny;
    A.GX = c->GX;
    A.ncells = c->ncells;
    A.k = sp.k;
    A.fld = c->fld;
    A.src_a = sp.buf[sp.cur].a;
    A.src_vz = sp.buf[sp.cur].vz;
    A.dst_a = sp.buf[sp.cur ^ 1].a;
    A.dst_vz = sp.buf[sp.cur ^ 1].vz;
    A.off = sp.off;
    A.dcount = sp.dcount;
    A.sub = sp.sub;
    A.farin = sp.farin;
    A.farcur = sp.farcur;
    A.acc_q = sp.acc_q;
    A.acc_e = sp.acc_e;
    A.counters = sp.counters;
    A.cap = (uint32_t)sp.capacity;
    A.energy = c->cfg.deposit_energy ? 1 : 0;
    return A;
}

dim3 tile_grid(pic_ctx* c) {
    return dim3((unsigned)((c->nx + kTileX - 1) / kTileX), (unsigned)((c->ny + kTileY - 1) / kTileY));
}

void swap_buffers(Species& sp) {
    sp.cur ^= 1;
    std::swap(sp.off, sp.off_next);
}

}  // namespace

// ---------------------------------------------------------------------------
// host entry points
// ---------------------------------------------------------------------------

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
    PIC_CUDA(cudaMalloc(&sp.off, (nc + 1) * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.off_next, (nc + 1) * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.dcount, 9 * nc * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.sub, 10 * nc * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.farin, nc * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.farcur, nc * sizeof(uint32_t)));
    PIC_CUDA(cudaMalloc(&sp.acc_q, (size_t)c->nodes * sizeof(unsigned long long)));
    PIC_CUDA(cudaMalloc(&sp.acc_e, (size_t)c->nodes * sizeof(unsigned long long)));
    PIC_CUDA(cudaMalloc(&sp.final_mesh, (size_t)c->nodes * sizeof(double)));
    PIC_CUDA(cudaMalloc(&sp.energy_mesh, (size_t)c->nodes * sizeof(double)));
    PIC_CUDA(cudaMalloc(&sp.counters, 4 * sizeof(unsigned long long)));
    PIC_CUDA(cudaMemsetAsync(sp.off, 0, (nc + 1) * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.off_next, 0, (nc + 1) * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.dcount, 0, 9 * nc * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.sub, 0, 10 * nc * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.farin, 0, nc * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.farcur, 0, nc * sizeof(uint32_t), c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.final_mesh, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.energy_mesh, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.counters, 0, 4 * sizeof(unsigned long long), c->stream));
    sp.acc_fresh = true;  // zero particles: the zero accumulator is their deposit
    return PIC_OK;
}

void species_free(Species& sp) {
    cudaFree(sp.store);
    cudaFree(sp.off);
    cudaFree(sp.off_next);
    cudaFree(sp.dcount);
    cudaFree(sp.sub);
    cudaFree(sp.farin);
    cudaFree(sp.farcur);
    cudaFree(sp.acc_q);
    cudaFree(sp.acc_e);
    cudaFree(sp.final_mesh);
    cudaFree(sp.energy_mesh);
    cudaFree(sp.counters);
    sp = Species{};
}

int species_reserve(pic_ctx* c, int s, int64_t capacity) {
    Species& sp = c->sp[s];
    if (capacity <= sp.capacity) return PIC_OK;
    // multiples of 64 particles keep both buffers' float4 arrays 256-byte aligned
    capacity = (capacity + 63) & ~(int64_t)63;
    if (capacity > (int64_t)0xF0000000ll)
        return fail(PIC_ERR_CAPACITY, "a species holds at most 4.0e9 particles (32-bit offsets)");
    int64_t live = 0;
    if (sp.store) PIC_TRY(particles_count(c, s, &live));
    float* store = nullptr;
    PIC_CUDA(cudaMalloc(&store, (size_t)capacity * 2 * 5 * sizeof(float)));
    ParticleSoA nb[2];
    for (int b = 0; b < 2; ++b) {
        nb[b].a = reinterpret_cast<float4*>(store + (size_t)b * capacity * 5);
        nb[b].vz = store + (size_t)b * capacity * 5 + (size_t)capacity * 4;
    }
    if (sp.store && live > 0) {
        PIC_CUDA(cudaMemcpyAsync(nb[0].a, sp.buf[sp.cur].a, (size_t)live * sizeof(float4),
                                 cudaMemcpyDeviceToDevice, c->stream));
        PIC_CUDA(cudaMemcpyAsync(nb[0].vz, sp.buf[sp.cur].vz, (size_t)live * sizeof(float),
                                 cudaMemcpyDeviceToDevice, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
    }
    cudaFree(sp.store);
    sp.store = store;
    sp.buf[0] = nb[0];
    sp.buf[1] = nb[1];
    sp.cur = 0;
    sp.capacity = capacity;
    return PIC_OK;
}

int ensure_staging(pic_ctx* c, size_t bytes) {
    if (bytes <= c->staging_bytes) return PIC_OK;
    cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    PIC_CUDA(cudaMalloc(&c->staging, bytes));
    c->staging_bytes = bytes;
    return PIC_OK;
}

static size_t aligned_points_bytes(int64_t n) {
    return ((size_t)n * sizeof(pic_point) + 255) & ~(size_t)255;
}

int particles_import_staging(pic_ctx* c, int64_t n, pic_point** dev_points) {
    PIC_TRY(ensure_staging(c, aligned_points_bytes(n) + (size_t)n * 4 + 256));
    *dev_points = static_cast<pic_point*>(c->staging);
    return PIC_OK;
}

int particles_import(pic_ctx* c, int s, int64_t n) {
    Species& sp = c->sp[s];
    PIC_TRY(species_reserve(c, s, std::max<int64_t>(n, 1)));
    if (aligned_points_bytes(n) + (size_t)n * 4 > c->staging_bytes)
        return fail(PIC_ERR_STATE, "import staging too small");
    const pic_point* dev_points = static_cast<const pic_point*>(c->staging);
    uint32_t* cell_of =
        reinterpret_cast<uint32_t*>(static_cast<char*>(c->staging) + aligned_points_bytes(n));
    const ParticleSoA tmp = sp.buf[sp.cur ^ 1];
    const ParticleSoA dst = sp.buf[sp.cur];
    // every imported particle enters as a "far mover" of its cell
    PIC_CUDA(cudaMemsetAsync(sp.farin, 0, (size_t)c->ncells * 4, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.dcount, 0, (size_t)c->ncells * 4 * 9, c->stream));
    if (n > 0)
        k_import_convert<<<grid1d(n, 256), 256, 0, c->stream>>>(dev_points, n, c->nx, c->ny,
                                                                1.0 / c->dx, 1.0 / c->dy, tmp.a,
                                                                tmp.vz, cell_of, sp.farin);
    PIC_TRY(scan_counts(c, sp));
    if (n > 0)
        k_import_scatter<<<grid1d(n, 256), 256, 0, c->stream>>>(tmp.a, tmp.vz, cell_of, n,
                                                                sp.sub + 9 * c->ncells,
                                                                sp.farcur, dst.a,
                                                                dst.vz);
    PIC_CUDA(cudaGetLastError());
    std::swap(sp.off, sp.off_next);
    PIC_CUDA(cudaMemsetAsync(sp.farcur, 0, (size_t)c->ncells * 4, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    unsigned long long flags[2] = {0, 0};
    PIC_CUDA(cudaMemcpyAsync(flags, sp.counters, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (flags[1]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_export(pic_ctx* c, int s, pic_point* dev_out, int64_t* n_out) {
    Species& sp = c->sp[s];
    int64_t n = 0;
    PIC_TRY(particles_count(c, s, &n));
    *n_out = n;
    if (n == 0 || !sp.store) return PIC_OK;
    const int wpb = 8;
    k_export<<<grid1d(c->ncells, wpb), wpb * 32, 0, c->stream>>>(
        sp.buf[sp.cur].a, sp.buf[sp.cur].vz, sp.off, c->nx, c->ncells, c->dx, c->dy, dev_out);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int particles_export_state(pic_ctx* c, int s, void* dev, int64_t n) {
    Species& sp = c->sp[s];
    if (n == 0 || !sp.store) return PIC_OK;
    int32_t* cell = static_cast<int32_t*>(dev);
    float* f = reinterpret_cast<float*>(cell + n);
    k_export_state<<<grid1d(c->ncells, 8), 256, 0, c->stream>>>(
        sp.buf[sp.cur].a, sp.buf[sp.cur].vz, sp.off, c->ncells, n, cell, f, f + n, f + 2 * n,
        f + 3 * n, f + 4 * n);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int particles_count(pic_ctx* c, int s, int64_t* n) {
    Species& sp = c->sp[s];
    uint32_t v = 0;
    unsigned long long flags[3] = {0, 0, 0};
    PIC_CUDA(cudaMemcpyAsync(&v, sp.off + c->ncells, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             c->stream));
    PIC_CUDA(cudaMemcpyAsync(flags, sp.counters, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    *n = v;
    if (flags[1]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    if (flags[2]) return fail(PIC_ERR_STATE, "push passes disagreed: a scatter write was refused");
    return PIC_OK;
}

int particles_bin_counts(pic_ctx* c, int s, int32_t* dev_counts) {
    Species& sp = c->sp[s];
    k_bin_counts<<<grid1d(c->nodes, 256), 256, 0, c->stream>>>(sp.off, c->nx, c->ny, c->GX,
                                                               dev_counts);
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
    PIC_CUDA(cudaMemsetAsync(sp.dcount, 0, (size_t)c->ncells * 4 * 9, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.farin, 0, (size_t)c->ncells * 4, c->stream));
    k_plasma_counts<<<grid1d(c->ncells, 256), 256, 0, c->stream>>>(P, c->ncells,
                                                                   sp.dcount + 4 * c->ncells);
    PIC_TRY(scan_counts(c, sp));
    std::swap(sp.off, sp.off_next);
    int64_t n = 0;
    PIC_TRY(particles_count(c, s, &n));
    unsigned long long flags[2] = {0, 0};
    PIC_CUDA(cudaMemcpyAsync(flags, sp.counters, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (flags[1]) return fail(PIC_ERR_CAPACITY, "a cell exceeds the per-cell particle limit");
    if (n > sp.capacity) {
        // the old particles are replaced: drop them before growing
        sp.capacity = 0;
        cudaFree(sp.store);
        sp.store = nullptr;
        PIC_TRY(species_reserve(c, s, n));
    }
    k_plasma_generate<<<grid1d(c->ncells, 8), 256, 0, c->stream>>>(P, sp.off, c->ncells,
                                                                    sp.buf[sp.cur].a,
                                                                    sp.buf[sp.cur].vz);
    PIC_CUDA(cudaGetLastError());
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_deposit(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    if (!sp.store) {
        sp.acc_fresh = true;
        return PIC_OK;
    }
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    KArgs A = make_args(c, sp);
    prof_begin(c, PIC_PHASE_DEPOSIT);
    if (A.energy)
        k_particles<kDeposit, true><<<tile_grid(c), kThreads, 0, c->stream>>>(A);
    else
        k_particles<kDeposit, false><<<tile_grid(c), kThreads, 0, c->stream>>>(A);
    prof_end(c, PIC_PHASE_DEPOSIT);
    c->launches += 1;
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
    k_flush<<<grid1d(c->nodes, 256), 256, 0, c->stream>>>(c->nodes, sp.acc_q, sp.acc_e, qscale,
                                                          escale, chrg, sp.final_mesh,
                                                          sp.energy_mesh, c->rho,
                                                          c->cfg.deposit_energy ? 1 : 0);
    prof_end(c, PIC_PHASE_FLUSH);
    PIC_CUDA(cudaGetLastError());
    sp.acc_fresh = false;
    return PIC_OK;
}

int particles_push(pic_ctx* c, int s) {
    Species& sp = c->sp[s];
    if (!sp.store) return PIC_OK;
    KArgs A = make_args(c, sp);
    const dim3 g = tile_grid(c);
    prof_begin(c, PIC_PHASE_PUSH_COUNT);
    k_particles<kCount, false><<<g, kThreads, 0, c->stream>>>(A);
    prof_end(c, PIC_PHASE_PUSH_COUNT);
    PIC_CUDA(cudaGetLastError());
    prof_begin(c, PIC_PHASE_SCAN);
    PIC_TRY(scan_counts(c, sp));
    prof_end(c, PIC_PHASE_SCAN);
    // the accumulators collect the deposit of the new positions
    PIC_CUDA(cudaMemsetAsync(sp.acc_q, 0, (size_t)c->nodes * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(sp.acc_e, 0, (size_t)c->nodes * 8, c->stream));
    prof_begin(c, PIC_PHASE_PUSH_SCATTER);
    if (A.energy)
        k_particles<kScatter, true><<<g, kThreads, 0, c->stream>>>(A);
    else
        k_particles<kScatter, false><<<g, kThreads, 0, c->stream>>>(A);
    prof_end(c, PIC_PHASE_PUSH_SCATTER);
    c->launches += 4;
    PIC_CUDA(cudaGetLastError());
    swap_buffers(sp);
    sp.acc_fresh = true;
    return PIC_OK;
}

}  // namespace picb200
