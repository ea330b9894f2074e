// warmstart.cu -- learned initial guess for the Poisson PCG solve.
//
// Takes the place of the reference's ML Poisson surrogate
// (SYCL-PIC-poissonsolver/src/poisson_ml_bridge.py:55-106,
// src/predict_poisson_ml.py:194-221), which replaced the solve.  Here the
// network only proposes phi_n as the starting point of PCG, which always runs
// to the same tolerance afterwards: the converged answer does not depend on
// the network.
//
// Network (the 3-level / 32-channel / 3x3 / two-convs-per-level encoder-
// decoder), on the node grid zero-padded to P x P (P a multiple of 4):
//   x0  = [phi_{n-1}/s0, db*dx^2/s1, mask]                  (3 channels)
//   a1  = relu(conv3x3_3->32(x0)),  a2 = relu(conv(a1))        level 0
//   p1  = avgpool2(a2); a3 = relu(conv(p1)), a4 = relu(conv(a3))   level 1
//   p2  = avgpool2(a4); a5 = relu(conv(p2)), a6 = relu(conv(a5))   level 2
//   u1  = up2(a6) + a4; a7 = relu(conv(u1)), a8 = relu(conv(a7))   level 1
//   u0  = up2(a8) + a2; a9 = relu(conv(u0)), a10 = relu(conv(a9))  level 0
//   out = conv3x3_32->1(a10)                   predicted (phi_n-phi_{n-1})/s2
// db is the change of the solve's right-hand side between the two steps, so
// by linearity the target is A_red^-1 db.
//
// Storage: activations and their gradients NHWC bf16 (32 channels), weights
// bf16 with FP32 master copies and Adam moments.  Convolutions are implicit
// GEMMs on the tensor cores, bf16 operands and FP32 accumulation (K = 9 taps
// x 32 channels for the 32->32 layers): the 32->32 layers forward and their
// data gradients on tcgen05 with TMEM accumulators (k_conv_rows: the average
// pools fused into the forward epilogue, the relu gates into the gradient
// one) and their weight gradients on tcgen05 as well (k_wgrad_rows, MN-major
// operands); the forward 3->32 input and 32->1 output layers with
// mma.sync.m16n8k16 (K = 12 taps x 4 channels, and N = 8 of which one column
// is used), their bf16 weights prepacked as B fragments; the outer layers'
// gradients on the FP32 cores.
// Weight gradients are reduced through per-block partials in a fixed order,
// so training is deterministic.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pic_internal.h"

namespace picb200 {
namespace {

constexpr int C = 32;        // channels of the inner layers
constexpr int TH = 8, TW = 32;  // output tile (pixels) of the tensor-core kernels
constexpr int CP = 40;       // padded channel stride in shared memory (bank-conflict free)
constexpr int kWgradBlocks = 296;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                        uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// x += c for 8 bf16 channels, each sum rounded to bf16
__device__ __forceinline__ void add_bf16x8(uint4& x, const uint4& c) {
    __nv_bfloat162* px = reinterpret_cast<__nv_bfloat162*>(&x);
    const __nv_bfloat162* pc = reinterpret_cast<const __nv_bfloat162*>(&c);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float2 a = __bfloat1622float2(pc[e]), b = __bfloat1622float2(px[e]);
        px[e] = __floats2bfloat162_rn(a.x + b.x, a.y + b.y);
    }
}

// Asynchronous global -> shared copies; with valid == false the destination
// is zero-filled and nothing is read.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Start the copy of a (TH+2) x (TW+2) x 32 halo tile of an NHWC bf16 image
// into shared memory ([row][col][CP]); pixels outside the image read as zero.
__device__ __forceinline__ void load_halo_async(__nv_bfloat16* dst, const __nv_bfloat16* src, int P,
                                                int y0, int x0) {
    constexpr int kChunks = (TH + 2) * (TW + 2) * (C / 8);  // 16-byte chunks
    for (int i = threadIdx.x; i < kChunks; i += blockDim.x) {
        const int q = i & 3, pix = i >> 2;
        const int r = pix / (TW + 2), col = pix % (TW + 2);
        const int y = y0 + r - 1, x = x0 + col - 1;
        const bool in = y >= 0 && x >= 0 && y < P && x < P;
        cp_async16(dst + pix * CP + q * 8, in ? src + ((int64_t)y * P + x) * C + q * 8 : src, in);
    }
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers
// ---------------------------------------------------------------------------
__device__ int g_ws_fault;  // a bounded wait of the warm-start kernels gave up
// Bound of the tensor-core kernels' pipeline waits, in SM clock cycles (about
// a second by default); a test lowers it to make the waits give up.
constexpr long long kWsWaitCycles = 1ll << 31;
__device__ long long g_ws_wait_cycles = kWsWaitCycles;

__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// u = up2(coarse) + skip, 16 bytes a thread (P = fine size; each sum rounded to bf16)
__global__ void k_up_add8(const __nv_bfloat16* coarse, const __nv_bfloat16* skip, int P, __nv_bfloat16* u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * P * 4) return;
    const int q = i & 3, p = i >> 2, y = p / P, x = p % P, Q = P / 2;
    uint4 v = reinterpret_cast<const uint4*>(skip)[i];
    add_bf16x8(v, *reinterpret_cast<const uint4*>(coarse + ((int64_t)(y >> 1) * Q + (x >> 1)) * C + q * 8));
    reinterpret_cast<uint4*>(u)[i] = v;
}

// ---------------------------------------------------------------------------
// Block-streaming 32->32 convolution on tcgen05 (the forward 32->32 layers).
//
// Implicit GEMM over blocks of 4 output rows x 30 output columns.  Its input,
// image rows y - 1 .. y + 4 by columns x0 - 1 .. x0 + 30 (x0 = 30 s for column
// strip s, y a multiple of 4), arrives as ONE TMA box of 6 rows x 32 pixels x
// 32 channels (64 bytes a pixel, 64-byte swizzle, zero filled outside the
// image): tile row i = 32 r + p holds row y - 1 + r, column x0 - 1 + p.  The
// four-row window starting at box row dy is the A operand of row tap dy -- a
// 2 KB offset in shared memory -- so for every block
//   D[32 r + p][32 dx + co] = sum_{dy, ci} in[y + r + dy - 1][x0 - 1 + p][ci] W[dy][dx][ci][co]
// is six MMAs of M = 128, N = 96, K = 16 (three row taps x two halves of the
// input channels), FP32 accumulators in TMEM.  The column taps are summed in
// the epilogue, where warp r of a warpgroup reads TMEM lanes 32 r .. 32 r + 31
// (output row y + r, one pixel a lane): lane p = 1..30 outputs column
// x0 + p - 1,
//   out[co] = D[i - 1][co] + D[i][32 + co] + D[i + 1][64 + co],
// the neighbours' values taken by warp shuffles.  One TMA box per 120
// outputs keeps the copy engine's per-box cost off the critical path (1.6x
// the output's bytes are read, the halo rows and columns mostly from L2).
//
// Roles, 12 warps:
//   warp 0   TMA producer (one lane), a ring of block slots;
//   warp 1   TMEM allocation, MMA issue (one lane), four accumulators;
//   warps 4-7 and 8-11  two epilogue warpgroups, each taking every block for
//            one half of the output channels: bias, relu, bf16 store and,
//            for the encoder layers, the 2x2 average pool (rows y + 2k and
//            y + 2k + 1 meet through shared memory, columns through a
//            shuffle).
// Every wait is bounded (g_ws_wait_cycles); a role that gives up records
// g_ws_fault, the CTA's roles leave their loops, the MMA lane waits (fixed
// bound) for the MMAs it issued and the producer for its copies before the
// tensor memory is freed.
// ---------------------------------------------------------------------------
constexpr int kRwCols = 30;                   // output columns a strip
constexpr int kRwBlk = 4;                     // output rows a block
constexpr int kRwSlots = 8;                   // block slots
constexpr int kRwBoxRows = kRwBlk + 2;
constexpr int kRwSlotBytes = kRwBoxRows * 32 * 64;   // 6 rows x 32 px x 32 ch bf16 (12 KB)
constexpr int kRwWBytes = 6 * 2 * 96 * 16;    // weights: [dy][kc][g][n 96][8 ci] bf16
constexpr int kRwThreads = 12 * 32;
// shared memory: head @0 (full[8] @0, empty[8] @64, accf[4] @128, acce[4]
// @160, drain @192, TMEM address @200, abort @204), bias @512, weights
// @1024, block slots (1024-aligned), pool exchange [half][buf][pair][32][8] words
constexpr int kRwOffBias = 512;
constexpr int kRwOffW = 1024;
constexpr int kRwOffSlots = kRwOffW + kRwWBytes;
constexpr int kRwOffX = kRwOffSlots + kRwSlots * kRwSlotBytes;
constexpr int kRwXchgBytes = 2 * 2 * 2 * 32 * 8 * 4;
constexpr int kRwSmemUsed = kRwOffX + kRwXchgBytes;
static_assert(kRwOffSlots % 1024 == 0 && kRwSlotBytes % 1024 == 0, "block slots 1024-aligned");
// more than half an SM's shared memory: one CTA an SM (its TMEM is all 512 columns)
constexpr int kRwSmem = 140 * 1024;
static_assert(kRwSmemUsed + 1024 <= kRwSmem, "row-conv shared memory");
// kind::f16: FP32 accumulator, bf16 A and B, both K-major, N = 96, M = 128
constexpr uint32_t kRwIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((96u >> 3) << 17) | ((128u >> 4) << 24);

// Forward layers: out = relu(conv + bias) (and its pool).  Data gradients
// (weights flipped and transposed, see k_pack_rows_w): out = conv, each
// value kept where gate > 0 (the forward activation), else 0.
struct RowConvArgs {
    const __nv_bfloat16* w;     // packed [dy][kc][g][n][8]
    const float* bias;          // [32] or null (0)
    __nv_bfloat16* out;         // [P][P][32]
    __nv_bfloat16* pool;        // [P/2][P/2][32] or null
    const __nv_bfloat16* gate;  // [P][P][32] or null
    int P;
    int relu;
};

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* tmap, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// K-major operand in the 64-byte swizzle layout (rows of 64 bytes, 16-byte
// chunks permuted within each 512-byte group of 8 rows, as TMA's 64-byte
// swizzle writes them): stride between 8-row groups 512 bytes; a K block of
// 16 bf16 at byte k * 32 of the row is addressed by the start address.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(512u >> 4) << 32) |
           (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ void rw_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(kRwIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The CTA's share [g0, g1) of the (strip, block) units, strip-major.
__device__ __forceinline__ void rw_share(int units, int& g0, int& g1) {
    const int b = blockIdx.x, n = gridDim.x;
    g0 = (int)(((int64_t)units * b) / n);
    g1 = (int)(((int64_t)units * (b + 1)) / n);
}

__global__ void __launch_bounds__(kRwThreads, 1) k_conv_rows(const __grid_constant__ CUtensorMap tmap,
                                                            RowConvArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // offsets below are from the first 1024-byte boundary of the buffer
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_u32(smem);
    const uint32_t full0 = sbase, empty0 = sbase + 64, accf0 = sbase + 128, acce0 = sbase + 160;
    const uint32_t drain = sbase + 192;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 200);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 204);
    float* sbias = reinterpret_cast<float*>(smem + kRwOffBias);
    unsigned char* wsm = smem + kRwOffW;
    unsigned char* slots = smem + kRwOffSlots;
    uint32_t* xch = reinterpret_cast<uint32_t*>(smem + kRwOffX);
    const long long wl = g_ws_wait_cycles;
    const int P = A.P;
    const int nblk = (P + kRwBlk - 1) / kRwBlk;
    const int units = ((P + kRwCols - 1) / kRwCols) * nblk;
    const int pool = A.pool != nullptr;
    int g0, g1;
    rw_share(units, g0, g1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(smem_u32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRwSlots; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int a = 0; a < 4; ++a) {
            mbar_init(accf0 + 8 * a, 1);
            mbar_init(acce0 + 8 * a, 8);  // the eight epilogue warps
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // launched with programmatic stream serialisation: everything above ran
    // while the kernel before was finishing; from here on its results are
    // read (the weights too: the packing kernel may be the one before)
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    // weights and bias into shared memory (generic stores, then a fence to
    // the async proxy the MMAs read through)
    for (int i = threadIdx.x; i < kRwWBytes / 16; i += kRwThreads)
        reinterpret_cast<uint4*>(wsm)[i] = reinterpret_cast<const uint4*>(A.w)[i];
    if (threadIdx.x < 32) sbias[threadIdx.x] = A.bias ? A.bias[threadIdx.x] : 0.f;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;
    auto give_up = [&]() {
        if (!*abort_flag) atomicExch(&g_ws_fault, 1);
        *abort_flag = 1;
    };

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int k = 0;
            for (int u = g0; u < g1; ++u, ++k) {
                const int s = k % kRwSlots;
                if (k >= kRwSlots && !mbar_wait_bounded(empty0 + 8 * s, ((k / kRwSlots) & 1) ^ 1, wl)) {
                    give_up();
                    break;
                }
                if (*abort_flag) break;
                const int x0 = (u / nblk) * kRwCols, y = (u % nblk) * kRwBlk;
                mbar_expect_tx(full0 + 8 * s, kRwSlotBytes);
                tma_load_3d(smem_u32(slots + s * kRwSlotBytes), &tmap, 0, x0 - 1, y - 1, full0 + 8 * s);
            }
            // every copy issued has landed before the CTA leaves (the last
            // use of each slot; fixed bound)
            for (int j = max(0, k - kRwSlots); j < k; ++j)
                if (!mbar_wait_bounded(full0 + 8 * (j % kRwSlots), (j / kRwSlots) & 1, kWsWaitCycles))
                    atomicExch(&g_ws_fault, 1);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0) {
            const uint32_t slots_u32 = smem_u32(slots), w_u32 = smem_u32(wsm);
            bool quit = false;
            int k = 0;
            for (int u = g0; u < g1; ++u, ++k) {
                const int s = k % kRwSlots, q = k & 3;
                if (!mbar_wait_bounded(full0 + 8 * s, (k / kRwSlots) & 1, wl) ||
                    (k >= 4 && !mbar_wait_bounded(acce0 + 8 * q, ((k >> 2) & 1) ^ 1, wl))) {
                    give_up();
                    quit = true;
                    break;
                }
                if (*abort_flag) {
                    quit = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t sb = slots_u32 + s * kRwSlotBytes;
#pragma unroll
                for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                    for (int kc = 0; kc < 2; ++kc)
                        rw_mma(tmem + q * 128, sw64_desc(sb + dy * 2048 + kc * 32),
                               tc_desc(w_u32 + (dy * 2 + kc) * 3072, 1536, 128), (dy | kc) ? 1u : 0u);
                tc_commit(accf0 + 8 * q);
                tc_commit(empty0 + 8 * s);
            }
            if (quit) {  // MMAs the epilogue will not wait for may still run
                tc_commit(drain);
                if (!mbar_wait_bounded(drain, 0, kWsWaitCycles)) atomicExch(&g_ws_fault, 1);
            }
        }
        __syncwarp();
    }
    else if (warp >= 4) {
        // ---------------- epilogue ----------------
        const int h = (warp - 4) >> 2;    // output channels 16 h .. 16 h + 15
        const int r = warp & 3;           // TMEM lanes 32 r .. 32 r + 31 = output row y + r
        const int Q = P / 2;
        float bias[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) bias[c] = sbias[16 * h + c];
        int k = 0;
        for (int u = g0; u < g1; ++u, ++k) {
            const int q = k & 3;
            const int x = (u / nblk) * kRwCols + lane - 1, y = (u % nblk) * kRwBlk + r;
            const bool valid = lane >= 1 && lane <= kRwCols && x < P && y < P;
            const bool ok = __all_sync(kFull, !*abort_flag && mbar_wait_bounded(accf0 + 8 * q, (k >> 2) & 1, wl));
            if (!ok && lane == 0) give_up();
            uint32_t quit;  // the same decision in the whole warpgroup (it meets at barriers below)
            asm volatile(
                "{\n.reg .pred p, t;\nsetp.ne.u32 p, %1, 0;\nbar.red.or.pred t, %2, 128, p;\nselp.u32 %0, 1, 0, t;\n}\n"
                : "=r"(quit)
                : "r"(ok ? 0u : 1u), "r"(1 + h)
                : "memory");
            if (quit) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            float v0[16], v1[16], v2[16];
            const uint32_t ta = tmem + ((uint32_t)(32 * r) << 16) + (uint32_t)(q * 128 + 16 * h);
            tc_ld16(ta, v0);
            tc_ld16(ta + 32, v1);
            tc_ld16(ta + 64, v2);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(acce0 + 8 * q);  // this warp's part of the accumulator is read
            uint32_t pk[8];
#pragma unroll
            for (int c = 0; c < 16; c += 2) {
                const float l0 = __shfl_up_sync(kFull, v0[c], 1), l1 = __shfl_up_sync(kFull, v0[c + 1], 1);
                const float r0v = __shfl_down_sync(kFull, v2[c], 1), r1v = __shfl_down_sync(kFull, v2[c + 1], 1);
                const float s0 = l0 + v1[c] + r0v + bias[c], s1 = l1 + v1[c + 1] + r1v + bias[c + 1];
                pk[c / 2] = A.relu ? pack_bf16x2(fmaxf(s0, 0.f), fmaxf(s1, 0.f)) : pack_bf16x2(s0, s1);
            }
            if (A.gate && valid) {
                const uint4* gp = reinterpret_cast<const uint4*>(A.gate + ((int64_t)y * P + x) * C + 16 * h);
                const uint4 ga = gp[0], gb = gp[1];
                const uint32_t gw[8] = {ga.x, ga.y, ga.z, ga.w, gb.x, gb.y, gb.z, gb.w};
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pk[e]));
                    const float2 g = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&gw[e]));
                    pk[e] = pack_bf16x2(g.x > 0.f ? f.x : 0.f, g.y > 0.f ? f.y : 0.f);
                }
            }
            if (valid) {
                uint4* dst = reinterpret_cast<uint4*>(A.out + ((int64_t)y * P + x) * C + 16 * h);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            if (pool) {
                // rows y (r even) and y + 1 meet in shared memory (double
                // buffered by block: one barrier a block)
                uint4* xb = reinterpret_cast<uint4*>(xch + (((h * 2 + (k & 1)) * 2 + (r >> 1)) * 32 + lane) * 8);
                if ((r & 1) == 0) {
                    xb[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    xb[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
                asm volatile("bar.sync %0, 128;\n" ::"r"(1 + h) : "memory");
                if (r & 1) {
                    // 0.25 (v(y-1, x) + v(y-1, x+1) + v(y, x) + v(y, x+1)) of the
                    // bf16 values; lane l + 1 holds column x + 1
                    uint32_t pp[8], pe[8];
                    *reinterpret_cast<uint4*>(pe) = xb[0];
                    *reinterpret_cast<uint4*>(pe + 4) = xb[1];
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const uint32_t pv = pe[c];
                        const uint32_t pr = __shfl_down_sync(kFull, pv, 1);
                        const uint32_t cr = __shfl_down_sync(kFull, pk[c], 1);
                        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pv));
                        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pr));
                        const float2 d = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pk[c]));
                        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&cr));
                        pp[c] = pack_bf16x2(0.25f * (a.x + b.x + d.x + f.x), 0.25f * (a.y + b.y + d.y + f.y));
                    }
                    if (valid && (lane & 1) && (x >> 1) < Q) {
                        uint4* dst = reinterpret_cast<uint4*>(A.pool + ((int64_t)(y >> 1) * Q + (x >> 1)) * C + 16 * h);
                        dst[0] = make_uint4(pp[0], pp[1], pp[2], pp[3]);
                        dst[1] = make_uint4(pp[4], pp[5], pp[6], pp[7]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem) : "memory");
    }
}

// FP32 masters [tap][ci][co] of the 32->32 layers (stride apart) -> the B
// operand layout [dy][kc][g][n = 32 dx + co][8 ci] in bf16 (ci = 16 kc + 8 g
// + e), for the forward layers (out) and for their data gradients (out_t:
// taps flipped, channels swapped, W'[tap][ci][co] = W[8 - tap][co][ci], since
// dX[p][ci] = sum_tap sum_co dY[p - d(tap)][co] W[tap][ci][co] and
// d(8 - tap) = -d(tap)).
constexpr int kRwWElems = 6 * 2 * 96 * 8;
__global__ void k_pack_rows_w(const float* w, int64_t stride, int layers, __nv_bfloat16* out,
                              __nv_bfloat16* out_t) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (int64_t)layers * kRwWElems) return;
    const int l = (int)(j / kRwWElems), i = (int)(j % kRwWElems);
    const int e = i & 7, n = (i >> 3) % 96, gk = i / (8 * 96);  // gk = (dy * 2 + kc) * 2 + g
    const int g = gk & 1, kc = (gk >> 1) & 1, dy = gk >> 2;
    const int dx = n / 32, co = n % 32, ci = 16 * kc + 8 * g + e;
    const int tap = dy * 3 + dx;
    const float* wl = w + l * stride;
    out[j] = __float2bfloat16_rn(wl[(tap * C + ci) * C + co]);
    out_t[j] = __float2bfloat16_rn(wl[((8 - tap) * C + co) * C + ci]);
}

// ---------------------------------------------------------------------------
// 32 -> 32 weight gradient on tcgen05 (training).
//
//   dW[dy][dx][ci][co] = sum_{y, x} X[y + dy - 1][x + dx - 1][ci] dY[y][x][co],
//   db[co] = sum_{y, x} dY[y][x][co]
//
// The reduction runs over pixels, so both operands are MN-major: a pixel's
// 32 channels (64 bytes) are the M (or N) extent of one swizzle atom and
// consecutive pixels its K rows, which is exactly how the TMA boxes of the
// NHWC images land in shared memory (64-byte swizzle, 8 pixels a 512-byte
// atom).  A unit is 4 rows x 32 pixels of dY (rows y0 .. y0 + 3, pixels
// x0 .. x0 + 31): its dY box (4 rows) and, for each column tap dx, a box of
// X rows y0 - 1 .. y0 + 5 shifted by dx - 1 pixels (zero filled outside the
// image).  For dY row r the A operand is X rows r .. r + 3 of the dx box --
// four 32-channel atoms 2 KB apart (LBO), so M = 128 = (dy = 0..3) x 32 ci,
// the fourth row tap unused -- and B is dY row r (N = 32 co); K = 16 pixels
// an MMA (two 8-pixel groups 512 bytes apart, SBO).  Every unit adds its
// 24 MMAs (4 rows x 3 dx x 2 K blocks) into three TMEM accumulators
// (D_dx[dy ci][co]), which the CTA writes out once at the end as its
// per-block partial; the partials are summed in a fixed order afterwards.
//
// Roles, 8 warps: warp 0 TMA producer (one lane), warp 1 TMEM allocation and
// MMA issue (one lane), warps 4-7 the bias gradient (each unit's dY box from
// shared memory, a channel and a quarter of the pixels a thread) and the
// final TMEM read-out (warp 4 + dy reads lanes 32 dy ..).  Every wait is
// bounded as in k_conv_rows.
// ---------------------------------------------------------------------------
constexpr int kWgStages = 3;
constexpr int kWgXRows = 7;                              // X rows of a box
constexpr int kWgXBytes = kWgXRows * 32 * 64;            // 14 KB
constexpr int kWgDBytes = 4 * 32 * 64;                   // 8 KB
constexpr int kWgStageBytes = 3 * kWgXBytes + kWgDBytes; // 50 KB
constexpr int kWgOffStages = 2048;
// a 4 KB pad after the ring keeps every operand address an MMA can form
// inside the allocation
constexpr int kWgSmemUsed = kWgOffStages + kWgStages * kWgStageBytes + 4096;
constexpr int kWgSmem = kWgSmemUsed + 1024;              // + alignment slack
static_assert(kWgStageBytes % 1024 == 0, "stages 1024-aligned");
static_assert(kWgSmem <= 227 * 1024, "weight-gradient shared memory");
constexpr int kWgThreads = 8 * 32;
// kind::f16: FP32 accumulator, bf16 A and B, both MN-major, N = 32, M = 128
constexpr uint32_t kWgIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                              ((32u >> 3) << 17) | ((128u >> 4) << 24);

// MN-major operand, 64-byte swizzle: 32-element atoms `lbo` bytes apart in
// M/N, 8-row K groups `sbo` bytes apart
__device__ __forceinline__ uint64_t sw64_mn_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ void wg_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(kWgIdesc), "r"(accumulate)
        : "memory");
}

__global__ void __launch_bounds__(kWgThreads, 1) k_wgrad_rows(const __grid_constant__ CUtensorMap tmx,
                                                             const __grid_constant__ CUtensorMap tmd,
                                                             int P, float* partial) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_u32(smem);
    // head: full[3] @0, empty[3] @32, accf @64, TMEM address @80, abort @84;
    // bias exchange [4][32] floats @1024; stages from @2048
    const uint32_t full0 = sbase, empty0 = sbase + 32, accf = sbase + 64;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 80);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + 84);
    float* sdb = reinterpret_cast<float*>(smem + 1024);
    unsigned char* stages = smem + kWgOffStages;
    const long long wl = g_ws_wait_cycles;
    const int nrb = (P + 3) / 4;  // row blocks; rows past P read as zero
    const int units = nrb * ((P + 31) / 32);
    int g0, g1;
    rw_share(units, g0, g1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;\n" ::"r"(smem_u32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kWgStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 5);  // the MMA commit and the four bias warps
        }
        mbar_init(accf, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;
    auto give_up = [&]() {
        if (!*abort_flag) atomicExch(&g_ws_fault, 1);
        *abort_flag = 1;
    };

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int k = 0;
            for (int u = g0; u < g1; ++u, ++k) {
                const int s = k % kWgStages;
                if (k >= kWgStages && !mbar_wait_bounded(empty0 + 8 * s, ((k / kWgStages) & 1) ^ 1, wl)) {
                    give_up();
                    break;
                }
                if (*abort_flag) break;
                const int x0 = (u / nrb) * 32, y0 = (u % nrb) * 4;
                const uint32_t st = smem_u32(stages + s * kWgStageBytes);
                mbar_expect_tx(full0 + 8 * s, kWgStageBytes);
#pragma unroll
                for (int dx = 0; dx < 3; ++dx)
                    tma_load_3d(st + dx * kWgXBytes, &tmx, 0, x0 + dx - 1, y0 - 1, full0 + 8 * s);
                tma_load_3d(st + 3 * kWgXBytes, &tmd, 0, x0, y0, full0 + 8 * s);
            }
            // every copy issued has landed before the CTA leaves (fixed bound)
            for (int j = max(0, k - kWgStages); j < k; ++j)
                if (!mbar_wait_bounded(full0 + 8 * (j % kWgStages), (j / kWgStages) & 1, kWsWaitCycles))
                    atomicExch(&g_ws_fault, 1);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0) {
            int k = 0;
            for (int u = g0; u < g1; ++u, ++k) {
                const int s = k % kWgStages;
                if (!mbar_wait_bounded(full0 + 8 * s, (k / kWgStages) & 1, wl)) {
                    give_up();
                    break;
                }
                if (*abort_flag) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t st = smem_u32(stages + s * kWgStageBytes);
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                        for (int kb = 0; kb < 2; ++kb)
                            wg_mma(tmem + dx * 32, sw64_mn_desc(st + dx * kWgXBytes + r * 2048 + kb * 1024, 2048, 512),
                                   sw64_mn_desc(st + 3 * kWgXBytes + r * 2048 + kb * 1024, 2048, 512),
                                   (k | r | kb) ? 1u : 0u);
                tc_commit(empty0 + 8 * s);
            }
            // all issued MMAs have completed when this arrives (also on the
            // give-up path, before the tensor memory is freed)
            tc_commit(accf);
        }
        __syncwarp();
    } else if (warp >= 4) {
        // ---------------- bias gradient, then the read-out ----------------
        const int q = warp - 4;  // pixels 8q .. 8q + 7 of each row; TMEM lanes 32q ..
        const int chunk = lane >> 3, e = lane & 7;
        float dbs = 0.f;
        int k = 0;
        for (int u = g0; u < g1; ++u, ++k) {
            const int s = k % kWgStages;
            const bool ok = __all_sync(kFull, !*abort_flag && mbar_wait_bounded(full0 + 8 * s, (k / kWgStages) & 1, wl));
            if (!ok) {
                if (lane == 0) give_up();
                break;
            }
            const unsigned char* dyb = stages + s * kWgStageBytes + 3 * kWgXBytes;
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int p = 0; p < 8; ++p) {
                    // channel `lane` of pixel 8q + p in row r: 64-byte rows,
                    // 16-byte chunk index XOR (row >> 1) & 3 (the 64-byte swizzle)
                    const int row = r * 32 + 8 * q + p;
                    const int off = row * 64 + ((chunk ^ ((row >> 1) & 3)) << 4) + 2 * e;
                    dbs += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(dyb + off));
                }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * s);
        }
        sdb[q * 32 + lane] = dbs;
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        float* out = partial + (int64_t)blockIdx.x * (9 * C * C + C);
        if (q == 0) out[9 * C * C + lane] = ((sdb[lane] + sdb[32 + lane]) + sdb[64 + lane]) + sdb[96 + lane];
        const bool done = __all_sync(kFull, mbar_wait_bounded(accf, 0, kWsWaitCycles));
        const bool good = __all_sync(kFull, done && !*abort_flag && g1 > g0);
        if (!done && lane == 0) give_up();
        if (q < 3) {
            // row tap dy = q, input channel ci = lane; column dx * 32 + co
            const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16);
            float v[16];
#pragma unroll 1
            for (int cb = 0; cb < 6; ++cb) {
                if (good) {
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    tc_ld16(ta + cb * 16, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = 0.f;
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = cb * 16 + j, dx = col >> 5, co = col & 31;
                    out[((q * 3 + dx) * C + co) * C + lane] = v[j];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;\n" ::"r"(tmem) : "memory");
    }
}

// Sums per-block partials into grad[n] (n values per block) in a fixed
// order.  Many outputs: a block takes 32 consecutive outputs, its warp w
// sums blocks w, w + 8, ... (coalesced rows), and the eight warp sums are
// added in order; few outputs: a warp an output, lane l summing blocks l,
// l + 32, ..., then a fixed shuffle tree.
constexpr int kSumWide = 256;  // outputs from which the first form is used
__global__ void __launch_bounds__(256) k_sum_partials(const float* partial, int nblocks, int n, float* grad) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (n >= kSumWide) {
        __shared__ float red[8][32];
        const int i = blockIdx.x * 32 + lane;
        float v = 0.f;
        if (i < n)
            for (int b = warp; b < nblocks; b += 8) v += partial[(int64_t)b * n + i];
        red[warp][lane] = v;
        __syncthreads();
        if (warp == 0 && i < n)
            grad[i] = ((red[0][lane] + red[1][lane]) + (red[2][lane] + red[3][lane])) +
                      ((red[4][lane] + red[5][lane]) + (red[6][lane] + red[7][lane]));
        return;
    }
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;  // whole warps leave together
    float v = 0.f;
    for (int b = lane; b < nblocks; b += 32) v += partial[(int64_t)b * n + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if (lane == 0) grad[i] = v;
}

// launch shape of k_sum_partials (256 threads a block) for n outputs
inline unsigned sum_blocks(int n) { return n >= kSumWide ? (unsigned)((n + 31) / 32) : (unsigned)((n * 32 + 255) / 256); }

// ---------------------------------------------------------------------------
// Input conv 3->32, output conv 32->1
// ---------------------------------------------------------------------------
// Both are implicit GEMMs on the tensor cores over TH x TW output tiles (warp
// = tile row, two m16 tiles of pixels), with the input tile and its halo
// staged in shared memory and the weights as bf16 B fragments prepacked per
// lane by k_pack_frags (FP32 accumulation).
//
// Input: x0 is [P][P][4] bf16 (channel 3 zero); K index = tap*4 + ci over 12
// taps (taps 9..11 zero), three k16 steps; N = 32 output channels.
// out = relu(b + sum_K W[K][:] x0[p+tap][ci]), stored through a shared-memory
// stage so that the 64-byte pixels leave in 16-byte chunks.
constexpr int kInSteps = 3, kOutSteps = 18;  // k16 steps of the two GEMMs

__global__ void __launch_bounds__(256) k_conv_in(const __nv_bfloat16* x0, const uint2* wfrag,
                                                 const float* bias, int P, __nv_bfloat16* out) {
    __shared__ __align__(16) uint2 xs[(TH + 2) * (TW + 2)];
    __shared__ __align__(16) __nv_bfloat16 os[TH * TW * CP];
    const int y0 = blockIdx.y * TH, x0p = blockIdx.x * TW;
    for (int i = threadIdx.x; i < (TH + 2) * (TW + 2); i += blockDim.x) {
        const int y = y0 + i / (TW + 2) - 1, x = x0p + i % (TW + 2) - 1;
        const bool in = y >= 0 && x >= 0 && y < P && x < P;
        cp_async8(xs + i, in ? x0 + ((int64_t)y * P + x) * 4 : x0, in);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    uint2 b[kInSteps][4];
#pragma unroll
    for (int s = 0; s < kInSteps; ++s)
#pragma unroll
        for (int n = 0; n < 4; ++n) b[s][n] = wfrag[(s * 4 + n) * 32 + lane];
    cp_async_wait_all();
    __syncthreads();
    const uint32_t* xw = reinterpret_cast<const uint32_t*>(xs);
    float acc[2][4][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;
#pragma unroll
    for (int s = 0; s < kInSteps; ++s) {
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            uint32_t a[4];
#pragma unroll
            for (int h = 0; h < 2; ++h) {  // k offset 0 / 8 of the step
                const int tap = 4 * s + 2 * h + (t >> 1);
#pragma unroll
                for (int r = 0; r < 2; ++r) {  // pixel row g / g + 8 of the m tile
                    const int px = m * 16 + g + 8 * r;
                    a[h * 2 + r] = tap < 9 ? xw[2 * ((warp + tap / 3) * (TW + 2) + px + tap % 3) + (t & 1)] : 0u;
                }
            }
#pragma unroll
            for (int n = 0; n < 4; ++n) mma_bf16(acc[m][n], a[0], a[1], a[2], a[3], b[s][n].x, b[s][n].y);
        }
    }
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int px = m * 16 + g + 8 * r, ch = n * 8 + 2 * t;
                const float v0 = fmaxf(acc[m][n][2 * r] + bias[ch], 0.f);
                const float v1 = fmaxf(acc[m][n][2 * r + 1] + bias[ch + 1], 0.f);
                *reinterpret_cast<__nv_bfloat162*>(os + (warp * TW + px) * CP + ch) = __floats2bfloat162_rn(v0, v1);
            }
    __syncthreads();
    for (int i = threadIdx.x; i < TH * TW * (C / 8); i += blockDim.x) {
        const int q = i & 3, pix = i >> 2;
        const int y = y0 + pix / TW, x = x0p + pix % TW;
        if (y >= P || x >= P) continue;
        *reinterpret_cast<uint4*>(out + ((int64_t)y * P + x) * C + q * 8) =
            *reinterpret_cast<const uint4*>(os + pix * CP + q * 8);
    }
}

// Output: out[p] = b + sum_tap sum_ci w[tap][ci] a[p+tap][ci]; K = tap*32 + ci,
// eighteen k16 steps; N = 8 with only column 0 non-zero (lanes t == 0 hold
// the result).
__global__ void __launch_bounds__(256) k_conv_out(const __nv_bfloat16* a, const uint2* wfrag,
                                                  const float* bias, int P, float* out) {
    __shared__ __align__(16) __nv_bfloat16 in_s[(TH + 2) * (TW + 2) * CP];
    const int y0 = blockIdx.y * TH, x0 = blockIdx.x * TW;
    load_halo_async(in_s, a, P, y0, x0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    cp_async_wait_all();
    __syncthreads();
    float acc[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[m][e] = 0.f;
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
            const uint2 b = wfrag[(tap * 2 + kc) * 32 + lane];
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                uint32_t f[4];
                const int r = (lane & 7) + ((lane >> 3) & 1) * 8;
                const int koff = (lane >> 4) * 8;
                ldsm_x4(smem_u32(in_s + ((warp + dy) * (TW + 2) + m * 16 + r + dx) * CP + kc * 16 + koff),
                        f[0], f[1], f[2], f[3]);
                mma_bf16(acc[m], f[0], f[1], f[2], f[3], b.x, b.y);
            }
        }
    }
    if ((lane & 3) == 0) {
        const int g = lane >> 2, y = y0 + warp;
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int x = x0 + m * 16 + g + 8 * r;
                if (y < P && x < P) out[(int64_t)y * P + x] = acc[m][2 * r] + bias[0];
            }
    }
}

// dA[p][ci] = (sum_tap w[tap][ci] dout[p - tap]) gated by (a[p][ci] > 0)
__global__ void k_conv_out_dx(const float* dout, const float* w, const __nv_bfloat16* a, int P,
                              __nv_bfloat16* da) {
    __shared__ float ws[9 * C];
    for (int i = threadIdx.x; i < 9 * C; i += blockDim.x) ws[i] = w[i];
    __syncthreads();
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)P * P) return;
    const int y = (int)(p / P), x = (int)(p % P);
    float d[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int yy = y - (tap / 3 - 1), xx = x - (tap % 3 - 1);
        d[tap] = (yy < 0 || xx < 0 || yy >= P || xx >= P) ? 0.f : dout[(int64_t)yy * P + xx];
    }
    const uint4* ap = reinterpret_cast<const uint4*>(a + p * C);
    uint4* dst = reinterpret_cast<uint4*>(da + p * C);
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // channels 8q .. 8q + 7
        const uint4 av = ap[q];
        const uint32_t aw[4] = {av.x, av.y, av.z, av.w};
        uint32_t o[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int c0 = 8 * q + 2 * h;
            float s0 = 0.f, s1 = 0.f;
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                // (a tap outside the image adds 0: the same sum)
                s0 = fmaf(ws[tap * C + c0], d[tap], s0);
                s1 = fmaf(ws[tap * C + c0 + 1], d[tap], s1);
            }
            const float2 g = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&aw[h]));
            o[h] = pack_bf16x2(g.x > 0.f ? s0 : 0.f, g.y > 0.f ? s1 : 0.f);
        }
        dst[q] = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// Small weight gradients on FP32 cores, persistent blocks over TH x TW tiles
// staged in shared memory; each thread owns fixed output entries and keeps
// their sums in registers; one partial per block, summed afterwards.
//   input conv:  g[(tap*3+ci)*32+co] = sum_p x0[p+tap][ci] * dY[p][co], g[864+co] = sum_p dY[p][co]
//   output conv: g[tap*32+ci] = sum_p a[p+tap][ci] * dout[p],           g[288] = sum_p dout[p]
constexpr int kSmallWgradBlocks = 296;
constexpr int kInOut = 9 * 3 * C + C;   // 896 input-conv gradient entries
constexpr int kOutOut = 9 * C + 1;      // 289 output-conv gradient entries

__global__ void __launch_bounds__(256) k_wgrad_in(const __nv_bfloat16* x0, const __nv_bfloat16* dY,
                                                  int P, float* partial) {
    __shared__ float xs[TH + 2][TW + 2][3];
    __shared__ float ds[TH * TW][C + 1];
    const int tiles_x = (P + TW - 1) / TW, tiles_y = (P + TH - 1) / TH;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};  // outputs threadIdx.x + 256*j
    for (int tile = blockIdx.x; tile < tiles_x * tiles_y; tile += gridDim.x) {
        const int y0 = (tile / tiles_x) * TH, x0p = (tile % tiles_x) * TW;
        __syncthreads();
        for (int i = threadIdx.x; i < (TH + 2) * (TW + 2); i += blockDim.x) {
            const int r = i / (TW + 2), col = i % (TW + 2);
            const int y = y0 + r - 1, x = x0p + col - 1;
            const bool in = y >= 0 && x >= 0 && y < P && x < P;
            for (int ci = 0; ci < 3; ++ci)
                xs[r][col][ci] = in ? __bfloat162float(x0[((int64_t)y * P + x) * 4 + ci]) : 0.f;
        }
        for (int i = threadIdx.x; i < TH * TW * C; i += blockDim.x) {
            const int pix = i / C, co = i % C;
            const int y = y0 + pix / TW, x = x0p + pix % TW;
            ds[pix][co] = (y < P && x < P) ? __bfloat162float(dY[((int64_t)y * P + x) * C + co]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int o = threadIdx.x + 256 * j;
            if (o >= kInOut) break;
            float s = 0.f;
            if (o < 9 * 3 * C) {
                const int tap = o / (3 * C), ci = (o / C) % 3, co = o % C;
                const int dy = tap / 3, dx = tap % 3;
                for (int r = 0; r < TH; ++r)
                    for (int col = 0; col < TW; ++col)
                        s = fmaf(xs[r + dy][col + dx][ci], ds[r * TW + col][co], s);
            } else {
                const int co = o - 9 * 3 * C;
                for (int pix = 0; pix < TH * TW; ++pix) s += ds[pix][co];
            }
            acc[j] += s;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int o = threadIdx.x + 256 * j;
        if (o < kInOut) partial[(int64_t)blockIdx.x * kInOut + o] = acc[j];
    }
}

__global__ void __launch_bounds__(256) k_wgrad_out(const __nv_bfloat16* a, const float* dout, int P,
                                                   float* partial) {
    __shared__ float as[TH + 2][TW + 2][C + 1];
    __shared__ float ds[TH * TW];
    const int tiles_x = (P + TW - 1) / TW, tiles_y = (P + TH - 1) / TH;
    float acc[2] = {0.f, 0.f};
    for (int tile = blockIdx.x; tile < tiles_x * tiles_y; tile += gridDim.x) {
        const int y0 = (tile / tiles_x) * TH, x0p = (tile % tiles_x) * TW;
        __syncthreads();
        for (int i = threadIdx.x; i < (TH + 2) * (TW + 2) * C; i += blockDim.x) {
            const int pix = i / C, ci = i % C;
            const int r = pix / (TW + 2), col = pix % (TW + 2);
            const int y = y0 + r - 1, x = x0p + col - 1;
            as[r][col][ci] = (y >= 0 && x >= 0 && y < P && x < P)
                                 ? __bfloat162float(a[((int64_t)y * P + x) * C + ci])
                                 : 0.f;
        }
        for (int i = threadIdx.x; i < TH * TW; i += blockDim.x) {
            const int y = y0 + i / TW, x = x0p + i % TW;
            ds[i] = (y < P && x < P) ? dout[(int64_t)y * P + x] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int o = threadIdx.x + 256 * j;
            if (o >= kOutOut) break;
            float s = 0.f;
            if (o < 9 * C) {
                const int tap = o / C, ci = o % C, dy = tap / 3, dx = tap % 3;
                for (int r = 0; r < TH; ++r)
                    for (int col = 0; col < TW; ++col)
                        s = fmaf(as[r + dy][col + dx][ci], ds[r * TW + col], s);
            } else {
                for (int pix = 0; pix < TH * TW; ++pix) s += ds[pix];
            }
            acc[j] += s;
        }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int o = threadIdx.x + 256 * j;
        if (o < kOutOut) partial[(int64_t)blockIdx.x * kOutOut + o] = acc[j];
    }
}


// ---------------------------------------------------------------------------
// Pooling, upsampling, gates
// ---------------------------------------------------------------------------
// dcoarse[Y][X] = sum of the 2x2 fine gradients, gated by (act > 0)
__global__ void k_down_sum_gate(const __nv_bfloat16* dfine, const __nv_bfloat16* act, int P,
                                __nv_bfloat16* dcoarse) {
    const int Q = P / 2;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)Q * Q * C) return;
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int Y = (int)(q / Q), X = (int)(q % Q);
    auto at = [&](int y, int x) { return __bfloat162float(dfine[((int64_t)y * P + x) * C + c]); };
    const float s = at(2 * Y, 2 * X) + at(2 * Y, 2 * X + 1) + at(2 * Y + 1, 2 * X) + at(2 * Y + 1, 2 * X + 1);
    dcoarse[i] = __float2bfloat16_rn(__bfloat162float(act[i]) > 0.f ? s : 0.f);
}

// d = (dskip + 0.25 * dpooled[y/2][x/2]) gated by (act > 0)   (P = fine size)
__global__ void k_skip_pool_gate(const __nv_bfloat16* dskip, const __nv_bfloat16* dpooled,
                                 const __nv_bfloat16* act, int P, __nv_bfloat16* d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)P * P * C) return;
    const int c = (int)(i % C);
    const int64_t p = i / C;
    const int y = (int)(p / P), x = (int)(p % P), Q = P / 2;
    const float v = __bfloat162float(dskip[i]) +
                    0.25f * __bfloat162float(dpooled[((int64_t)(y / 2) * Q + x / 2) * C + c]);
    d[i] = __float2bfloat16_rn(__bfloat162float(act[i]) > 0.f ? v : 0.f);
}

// ---------------------------------------------------------------------------
// Inputs, loss, output, optimiser
// ---------------------------------------------------------------------------
// x0 = [phi/s0, db*dx^2/s1, mask] on the padded grid (zero outside)
__global__ void k_make_input(const double* phi, const double* db, const uint8_t* mask, int GX,
                             int GY, int P, float inv_s0, float s1f, __nv_bfloat16* x0) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)P * P) return;
    const int y = (int)(p / P), x = (int)(p % P);
    float c0 = 0.f, c1 = 0.f, c2 = 0.f;
    if (y < GY && x < GX) {
        const int64_t k = (int64_t)y * GX + x;
        c0 = (float)phi[k] * inv_s0;
        c1 = mask[k] ? 0.f : (float)db[k] * s1f;
        c2 = mask[k] ? 1.f : 0.f;
    }
    __nv_bfloat16* d = x0 + p * 4;
    d[0] = __float2bfloat16_rn(c0);
    d[1] = __float2bfloat16_rn(c1);
    d[2] = __float2bfloat16_rn(c2);
    d[3] = __float2bfloat16_rn(0.f);
}

// The loss is the starting residual of PCG from the network's guess, in
// scaled units.  With the guess phi_prev + s2*out on non-electrode nodes, the
// residual of the reduced system is (s1/dx^2) * r with
//   r = rhs - kappa * L(u),  rhs = (b_n - b_{n-1}) dx^2 / s1,  kappa = s2/s1,
//   L(u) = (2 + 2 beta) u - (u_w + u_e) - beta (u_s + u_n),  beta = dx^2/dy^2,
// u = out on non-electrode nodes and 0 on electrodes (every wall node is an
// electrode, so a free node's four neighbours are inside the grid).
// loss = sum over free nodes of r^2 / nodes.
__device__ __forceinline__ bool free_node(const uint8_t* mask, int GX, int GY, int y, int x) {
    return y > 0 && x > 0 && y < GY - 1 && x < GX - 1 && !mask[(int64_t)y * GX + x];
}

__global__ void k_resid(const float* out, const float* rhs, const uint8_t* mask, int GX, int GY,
                        int P, float kappa, float beta, float inv_count, float* resid,
                        float* loss_partial) {
    __shared__ float red[8];
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (k < (int64_t)GX * GY) {
        const int y = (int)(k / GX), x = (int)(k % GX);
        float r = 0.f;
        if (free_node(mask, GX, GY, y, x)) {
            auto u = [&](int yy, int xx) {
                return mask[(int64_t)yy * GX + xx] ? 0.f : out[(int64_t)yy * P + xx];
            };
            const float Lu = (2.f + 2.f * beta) * u(y, x) - (u(y, x - 1) + u(y, x + 1)) -
                             beta * (u(y - 1, x) + u(y + 1, x));
            r = rhs[k] - kappa * Lu;
        }
        resid[k] = r;
        l = r * r * inv_count;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(kFull, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += red[w];
        loss_partial[blockIdx.x] = s;
    }
}

// dloss/dout = -(2 kappa / nodes) L(r) on free nodes, 0 elsewhere (L is
// symmetric on the free nodes; r is 0 on electrodes).
__global__ void k_resid_grad(const float* resid, const uint8_t* mask, int GX, int GY, int P,
                             float kappa, float beta, float inv_count, float* dout) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)P * P) return;
    const int y = (int)(p / P), x = (int)(p % P);
    float d = 0.f;
    if (y < GY && x < GX && free_node(mask, GX, GY, y, x)) {
        auto r = [&](int yy, int xx) { return resid[(int64_t)yy * GX + xx]; };
        const float Lr = (2.f + 2.f * beta) * r(y, x) - (r(y, x - 1) + r(y, x + 1)) -
                         beta * (r(y - 1, x) + r(y + 1, x));
        d = -2.f * kappa * inv_count * Lr;
    }
    dout[p] = d;
}

// guess = phi_prev + out * s2 on non-electrode nodes
__global__ void k_make_guess(const double* phi_prev, const float* out, const uint8_t* mask, int GX,
                             int GY, int P, float s2, float* guess) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)GX * GY) return;
    const int y = (int)(k / GX), x = (int)(k % GX);
    guess[k] = mask[k] ? 0.f : (float)phi_prev[k] + out[(int64_t)y * P + x] * s2;
}

// Adam on the FP32 master weights; refreshes the bf16 or fp32 working copy.
__global__ void k_adam(float* w, float* m, float* v, const float* g, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2, float gscale,
                       __nv_bfloat16* w_bf16, float* w_f32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    if (w_bf16) w_bf16[i] = __float2bfloat16_rn(wi);
    if (w_f32) w_f32[i] = wi;
}

// Records a training pair: db = b_n - b_prev (RHS change) on the node grid
// and the input image.
__global__ void k_diff(const double* a, const double* b, int64_t n, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] - b[i];
}

// rhs = (b_n - b_{n-1}) dx^2 / s1 on free nodes, 0 on electrodes
__global__ void k_rhs(const double* db, const uint8_t* mask, int64_t n, double dx2_over_s1, float* t) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) t[i] = mask[i] ? 0.f : (float)(db[i] * dx2_over_s1);
}

// Sums of squares over non-electrode nodes of phi_prev, db*dx^2 and
// phi - phi_prev, and the number of those nodes: one partial quadruple per
// block (summed on the host in block order).
__global__ void k_sumsq4(const double* phi_prev, const double* db, const double* phi,
                         const uint8_t* mask, int64_t n, double dx2, double* partial) {
    __shared__ double red[4][8];
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (mask[i]) continue;
        const double a = phi_prev[i], b = db[i] * dx2, d = phi[i] - phi_prev[i];
        s[0] += a * a;
        s[1] += b * b;
        s[2] += d * d;
        s[3] += 1.0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[threadIdx.x][w];
        partial[blockIdx.x * 4 + threadIdx.x] = v;
    }
}

inline unsigned g1(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
// Network state
// ---------------------------------------------------------------------------

// parameter blocks: 0 = input conv, 1..9 = 32->32 convs, 10 = output conv
constexpr int kNumConv32 = 9;
constexpr int kInW = 9 * 3 * C, kInB = C;
constexpr int kW32 = 9 * C * C, kB32 = C;
constexpr int kOutW = 9 * C, kOutB = 1;
constexpr int kParams = kInW + kInB + kNumConv32 * (kW32 + kB32) + kOutW + kOutB;

struct Net {
    int P = 0, GX = 0, GY = 0;
    int sms = 148;  // streaming multiprocessors of the device (persistent grids)
    float s0 = 1, s1 = 1, s2 = 1;  // input / target scales
    // parameters (fp32 master, Adam moments, gradient)
    float* w = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* g = nullptr;
    int64_t adam_t = 0;
    // bf16 B fragments of the input and output convolutions (k_pack_frags)
    uint2* in_frag = nullptr;
    uint2* out_frag = nullptr;
    // the 32->32 layers' weights in k_conv_rows' B layout (forward, and
    // flipped and transposed for the data gradients), the TMA descriptors of
    // the forward inputs (a1, p1, a3, p2, a5, u1, a7, u0, a9) and of the
    // gradient buffers the backward convolutions read (d_big[0..1],
    // d_mid[0..1], d_small[0..1])
    __nv_bfloat16* wrows = nullptr;
    __nv_bfloat16* wrows_t = nullptr;
    CUtensorMap tm_in[9];
    CUtensorMap tm_grad[6];
    CUtensorMap tm_wx[9], tm_wd[6];  // the same images in k_wgrad_rows' boxes
    // activations (P = fine, Q = P/2, R = P/4)
    __nv_bfloat16 *x0 = nullptr, *a[11] = {}, *p1 = nullptr, *p2 = nullptr, *u0 = nullptr, *u1 = nullptr;
    float* out = nullptr;
    const __nv_bfloat16* xin = nullptr;  // input image of the current pass (x0 or a recorded pair)
    // gradients
    __nv_bfloat16 *d_big[3] = {}, *d_mid[3] = {}, *d_small[2] = {};
    float* dout = nullptr;
    float* resid = nullptr;  // scaled starting residual on the node grid
    float* partial = nullptr;
    size_t partial_floats = 0;
    float* gsum = nullptr;  // summed 32->32 weight gradient before re-layout
    float* loss_acc = nullptr;  // per-pair loss of the current epoch
    float* loss_partial = nullptr;
    // dataset of recorded pairs: x0 image (bf16, P*P*4) and target (f32, GX*GY)
    int64_t cap_pairs = 0, n_pairs = 0, next_pair = 0;
    __nv_bfloat16* ds_x = nullptr;
    float* ds_t = nullptr;
    // recording scratch
    double* phi_prev = nullptr;
    double* b_prev = nullptr;
    double* db = nullptr;
    bool have_prev = false;
    bool trained = false;
    bool packed = false;      // the bf16 weights match the masters
    bool auto_scale = false;  // take s0, s1, s2 from the first recorded pair
};

static int64_t param_off(int block) {
    if (block == 0) return 0;
    if (block <= kNumConv32) return kInW + kInB + (int64_t)(block - 1) * (kW32 + kB32);
    return kInW + kInB + (int64_t)kNumConv32 * (kW32 + kB32);
}

static void net_free(Net& N) {
    cudaFree(N.w); cudaFree(N.m); cudaFree(N.v); cudaFree(N.g);
    cudaFree(N.in_frag); cudaFree(N.out_frag); cudaFree(N.wrows); cudaFree(N.wrows_t);
    cudaFree(N.x0);
    for (auto* p : N.a) cudaFree(p);
    cudaFree(N.p1); cudaFree(N.p2); cudaFree(N.u0); cudaFree(N.u1); cudaFree(N.out);
    for (auto* p : N.d_big) cudaFree(p);
    for (auto* p : N.d_mid) cudaFree(p);
    for (auto* p : N.d_small) cudaFree(p);
    cudaFree(N.dout); cudaFree(N.resid); cudaFree(N.partial); cudaFree(N.loss_partial); cudaFree(N.gsum); cudaFree(N.loss_acc);
    cudaFree(N.ds_x); cudaFree(N.ds_t);
    cudaFree(N.phi_prev); cudaFree(N.b_prev); cudaFree(N.db);
    N = Net{};
}

// Deterministic initialisation (He-style uniform from a hashed index).
static void init_params(std::vector<float>& w) {
    auto u = [](uint64_t i) {
        uint64_t z = i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E5Full;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    w.assign(kParams, 0.f);
    for (int blk = 0; blk <= kNumConv32 + 1; ++blk) {
        const int64_t off = param_off(blk);
        const int fan_in = blk == 0 ? 27 : 9 * C;
        const int nw = blk == 0 ? kInW : (blk <= kNumConv32 ? kW32 : kOutW);
        const double bound = std::sqrt(6.0 / fan_in) * (blk == kNumConv32 + 1 ? 0.1 : 1.0);
        for (int i = 0; i < nw; ++i) w[off + i] = (float)(bound * u(off + i));
    }
}

}  // namespace picb200

using namespace picb200;

struct pic_ws {
    Net net;
};

namespace picb200 {

// TMA descriptor of an NHWC bf16 image of P x P pixels and 32 channels,
// read in boxes of 32 channels x 32 pixels x 6 rows (64 bytes a pixel,
// 64-byte swizzle, zero filled outside).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int make_row_tmap(CUtensorMap* tm, const __nv_bfloat16* base, int P, int rows = kRwBoxRows) {
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !f)
            return fail(PIC_ERR_CUDA, "warm start: cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<EncodeTiledFn>(f);
    }
    const cuuint64_t dims[3] = {(cuuint64_t)C, (cuuint64_t)P, (cuuint64_t)P};
    const cuuint64_t strides[2] = {(cuuint64_t)C * 2, (cuuint64_t)P * C * 2};
    const cuuint32_t box[3] = {(cuuint32_t)C, 32, (cuuint32_t)rows};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(base), dims,
                              strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(PIC_ERR_CUDA, "warm start: TMA descriptor encoding failed (" + std::to_string((int)r) + ")");
    return PIC_OK;
}

static int ws_alloc(pic_ctx* c) {
    if (c->ws) return PIC_OK;
    auto* W = new pic_ws();
    c->ws = W;
    Net& N = W->net;
    N.GX = c->GX;
    N.GY = c->GY;
    N.P = ((std::max(c->GX, c->GY) + 3) / 4) * 4;
    if (cudaDeviceGetAttribute(&N.sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || N.sms < 1)
        return fail(PIC_ERR_CUDA, "warm start: device query failed");
    const int64_t P = N.P, Q = P / 2, R = P / 4;
    auto balloc = [&](__nv_bfloat16** p, int64_t n) {
        return cudaMalloc(p, (size_t)n * sizeof(__nv_bfloat16));
    };
    if (cudaMalloc(&N.w, kParams * 4) || cudaMalloc(&N.m, kParams * 4) ||
        cudaMalloc(&N.v, kParams * 4) || cudaMalloc(&N.g, kParams * 4) ||
        cudaMalloc(&N.in_frag, kInSteps * 4 * 32 * sizeof(uint2)) ||
        cudaMalloc(&N.out_frag, kOutSteps * 32 * sizeof(uint2)) ||
        balloc(&N.x0, P * P * 4))
        return fail(PIC_ERR_CUDA, "warm start: parameter allocation failed");
    const int64_t sizes[11] = {P, P, Q, Q, R, R, Q, Q, P, P, 0};  // a1..a10 at index 1..10
    for (int i = 1; i <= 10; ++i)
        if (balloc(&N.a[i], sizes[i - 1] * sizes[i - 1] * C))
            return fail(PIC_ERR_CUDA, "warm start: activation allocation failed");
    if (balloc(&N.p1, Q * Q * C) || balloc(&N.p2, R * R * C) || balloc(&N.u0, P * P * C) ||
        balloc(&N.u1, Q * Q * C) || cudaMalloc(&N.out, P * P * 4) || cudaMalloc(&N.dout, P * P * 4) ||
        cudaMalloc(&N.resid, (size_t)c->nodes * 4))
        return fail(PIC_ERR_CUDA, "warm start: activation allocation failed");
    for (auto*& p : N.d_big)
        if (balloc(&p, P * P * C)) return fail(PIC_ERR_CUDA, "warm start: gradient allocation failed");
    for (auto*& p : N.d_mid)
        if (balloc(&p, Q * Q * C)) return fail(PIC_ERR_CUDA, "warm start: gradient allocation failed");
    for (auto*& p : N.d_small)
        if (balloc(&p, R * R * C)) return fail(PIC_ERR_CUDA, "warm start: gradient allocation failed");
    // per-block partials of the 32->32 weight gradients; per-row partials of
    // the outer layers'
    N.partial_floats = (size_t)std::max(kWgradBlocks, kSmallWgradBlocks) * (9 * C * C + C);
    if (cudaMalloc(&N.partial, N.partial_floats * 4) || cudaMalloc(&N.loss_partial, g1(std::max<int64_t>(P * P, c->nodes)) * 4) ||
        cudaMalloc(&N.gsum, (9 * C * C + C) * 4))
        return fail(PIC_ERR_CUDA, "warm start: scratch allocation failed");
    const size_t nodes = (size_t)c->nodes;
    if (cudaMalloc(&N.phi_prev, nodes * 8) || cudaMalloc(&N.b_prev, nodes * 8) ||
        cudaMalloc(&N.db, nodes * 8))
        return fail(PIC_ERR_CUDA, "warm start: scratch allocation failed");
    std::vector<float> w;
    init_params(w);
    PIC_CUDA(cudaMemcpy(N.w, w.data(), kParams * 4, cudaMemcpyHostToDevice));
    PIC_CUDA(cudaMemset(N.m, 0, kParams * 4));
    PIC_CUDA(cudaMemset(N.v, 0, kParams * 4));
    PIC_CUDA(cudaFuncSetAttribute(k_conv_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kRwSmem));
    if (cudaMalloc(&N.wrows, (size_t)kNumConv32 * kRwWBytes) || cudaMalloc(&N.wrows_t, (size_t)kNumConv32 * kRwWBytes))
        return fail(PIC_ERR_CUDA, "warm start: parameter allocation failed");
    {
        const __nv_bfloat16* ins[9] = {N.a[1], N.p1, N.a[3], N.p2, N.a[5], N.u1, N.a[7], N.u0, N.a[9]};
        const int sz[9] = {(int)P, (int)Q, (int)Q, (int)R, (int)R, (int)Q, (int)Q, (int)P, (int)P};
        for (int l = 0; l < 9; ++l) PIC_TRY(make_row_tmap(&N.tm_in[l], ins[l], sz[l]));
        const __nv_bfloat16* gr[6] = {N.d_big[0], N.d_big[1], N.d_mid[0], N.d_mid[1], N.d_small[0], N.d_small[1]};
        const int gs[6] = {(int)P, (int)P, (int)Q, (int)Q, (int)R, (int)R};
        for (int i = 0; i < 6; ++i) PIC_TRY(make_row_tmap(&N.tm_grad[i], gr[i], gs[i]));
        // the weight gradients' boxes: X rows y0 - 1 .. y0 + 5, dY rows y0 .. y0 + 3
        for (int l = 0; l < 9; ++l) PIC_TRY(make_row_tmap(&N.tm_wx[l], ins[l], sz[l], kWgXRows));
        for (int i = 0; i < 6; ++i) PIC_TRY(make_row_tmap(&N.tm_wd[i], gr[i], gs[i], 4));
    }
    PIC_CUDA(cudaFuncSetAttribute(k_wgrad_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
    return PIC_OK;
}

// B fragments (m16n8k16, per lane: {k 2t, 2t+1 | k 2t+8, 2t+9} of column g)
// of the input and output convolutions, from the FP32 masters.
//   input  [step s][n tile][lane]: B[K][co] = w_in[tap][ci][co], K = 16s + k =
//          tap*4 + ci, zero for ci == 3 or tap >= 9;
//   output [step j = tap*2 + kc][lane]: B[K][0] = w_out[tap][kc*16 + k], other
//          columns zero.
__global__ void k_pack_frags(const float* w_in, const float* w_out, uint2* in_frag, uint2* out_frag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = i & 31, g = lane >> 2, t = lane & 3;
    if (i < kInSteps * 4 * 32) {
        const int s = i / 128, n = (i / 32) % 4, co = n * 8 + g;
        auto w = [&](int k) {
            const int K = 16 * s + k, tap = K / 4, ci = K % 4;
            return (ci < 3 && tap < 9) ? w_in[(tap * 3 + ci) * C + co] : 0.f;
        };
        in_frag[i] = make_uint2(pack_bf16x2(w(2 * t), w(2 * t + 1)), pack_bf16x2(w(2 * t + 8), w(2 * t + 9)));
    } else if (i < kInSteps * 4 * 32 + kOutSteps * 32) {
        const int j = (i - kInSteps * 4 * 32) / 32, tap = j / 2, kc = j % 2;
        const float* wt = w_out + tap * C + kc * 16;
        out_frag[j * 32 + lane] = g == 0 ? make_uint2(pack_bf16x2(wt[2 * t], wt[2 * t + 1]),
                                                      pack_bf16x2(wt[2 * t + 8], wt[2 * t + 9]))
                                         : make_uint2(0u, 0u);
    }
}

// Refresh the bf16 working weights and their transposes from the masters
// (only after the masters changed).
static int ws_pack(pic_ctx* c) {
    Net& N = c->ws->net;
    if (N.packed) return PIC_OK;
    k_pack_frags<<<g1((kInSteps * 4 + kOutSteps) * 32), 256, 0, c->stream>>>(
        N.w, N.w + param_off(kNumConv32 + 1), N.in_frag, N.out_frag);
    k_pack_rows_w<<<g1((int64_t)kNumConv32 * kRwWElems), 256, 0, c->stream>>>(
        N.w + param_off(1), kW32 + kB32, kNumConv32, N.wrows, N.wrows_t);
    c->launches += 2;
    PIC_CUDA(cudaGetLastError());
    N.packed = true;
    return PIC_OK;
}

static void conv_rows(pic_ctx* c, int layer, __nv_bfloat16* out, int P, __nv_bfloat16* pool,
                      const __nv_bfloat16* up = nullptr, const __nv_bfloat16* skip = nullptr,
                      __nv_bfloat16* u = nullptr) {
    Net& N = c->ws->net;
    if (up) {
        k_up_add8<<<g1((int64_t)P * P * 4), 256, 0, c->stream>>>(up, skip, P, u);
        c->launches += 1;
    }
    const int units = ((P + kRwCols - 1) / kRwCols) * ((P + kRwBlk - 1) / kRwBlk);
    const int grid = std::max(1, std::min(N.sms, (units + 3) / 4));
    RowConvArgs A;
    A.w = N.wrows + (int64_t)layer * (kRwWBytes / 2);
    A.bias = N.w + param_off(layer + 1) + kW32;
    A.out = out;
    A.pool = pool;
    A.gate = nullptr;
    A.P = P;
    A.relu = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kRwThreads);
    cfg.dynamicSmemBytes = kRwSmem;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_conv_rows, N.tm_in[layer], A);
    c->launches += 1;
}

// Data gradient of 32->32 layer `layer` on tcgen05: out = conv(grad input
// tm_grad[g], flipped and transposed weights), kept where gate > 0.
static void conv_rows_grad(pic_ctx* c, int layer, int g, __nv_bfloat16* out, int P, const __nv_bfloat16* gate) {
    Net& N = c->ws->net;
    const int units = ((P + kRwCols - 1) / kRwCols) * ((P + kRwBlk - 1) / kRwBlk);
    const int grid = std::max(1, std::min(N.sms, (units + 3) / 4));
    RowConvArgs A;
    A.w = N.wrows_t + (int64_t)layer * (kRwWBytes / 2);
    A.bias = nullptr;
    A.out = out;
    A.pool = nullptr;
    A.gate = gate;
    A.P = P;
    A.relu = 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kRwThreads);
    cfg.dynamicSmemBytes = kRwSmem;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_conv_rows, N.tm_grad[g], A);
    c->launches += 1;
}

// The solve's guess buffer, allocated when a network becomes usable (so
// that no allocation falls inside a timed solve).
static int ws_guess_buffer(pic_ctx* c) {
    if (!c->ps.net_guess) PIC_CUDA(cudaMalloc(&c->ps.net_guess, (size_t)c->nodes * 4));
    return PIC_OK;
}

// Bound of the tensor-core kernels' waits on the current device; cycles <= 0
// restores the default.
int ws_set_wait_limit(int64_t cycles) {
    const long long v = cycles > 0 ? (long long)cycles : kWsWaitCycles;
    PIC_CUDA(cudaMemcpyToSymbol(g_ws_wait_cycles, &v, sizeof(v)));
    return PIC_OK;
}

// A bounded device wait of the warm-start kernels gave up (read after a
// synchronisation; clears the flag).
int ws_check_fault() {
    int f = 0;
    PIC_CUDA(cudaMemcpyFromSymbol(&f, g_ws_fault, sizeof(int)));
    if (f) {
        const int z = 0;
        PIC_CUDA(cudaMemcpyToSymbol(g_ws_fault, &z, sizeof(int)));
        return fail(PIC_ERR_TIMEOUT, "warm start: a tensor-core wait timed out");
    }
    return PIC_OK;
}

// [tap][co][ci] (+ bias) -> the parameter layout [tap][ci][co] (+ bias)
__global__ void k_scatter_wgrad(const float* src, float* g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * C * C + C) return;
    if (i < 9 * C * C) {
        const int tap = i / (C * C), co = (i / C) % C, ci = i % C;
        g[(tap * C + ci) * C + co] = src[i];
    } else {
        g[i] = src[i];
    }
}

// Weight gradient of 32->32 layer `layer` from its forward input (tm_wx)
// and the gradient image tm_wd[g] of its output, on tcgen05.
static void wgrad32(pic_ctx* c, int layer, int g, int P) {
    Net& N = c->ws->net;
    const int units = ((P + 3) / 4) * ((P + 31) / 32);
    const int grid = std::max(1, std::min(N.sms, units));
    k_wgrad_rows<<<grid, kWgThreads, kWgSmem, c->stream>>>(N.tm_wx[layer], N.tm_wd[g], P, N.partial);
    k_sum_partials<<<sum_blocks(9 * C * C + C), 256, 0, c->stream>>>(N.partial, grid, 9 * C * C + C,
                                                             N.gsum);
    k_scatter_wgrad<<<g1(9 * C * C + C), 256, 0, c->stream>>>(N.gsum, N.g + param_off(layer + 1));
}

// Forward pass on the image N.xin; result in N.out.  Thirteen launches: the
// pools run inside the 32->32 convolutions, the decoder's upsample-and-skip
// sums (kept in u0, u1 for the backward pass) as vector kernels before them.
static void forward(pic_ctx* c) {
    Net& N = c->ws->net;
    const int P = N.P, Q = P / 2, R = P / 4;
    const dim3 gP((P + TW - 1) / TW, (P + TH - 1) / TH);
    k_conv_in<<<gP, 256, 0, c->stream>>>(N.xin, N.in_frag, N.w + kInW, P, N.a[1]);
    conv_rows(c, 0, N.a[2], P, N.p1);
    conv_rows(c, 1, N.a[3], Q, nullptr);
    conv_rows(c, 2, N.a[4], Q, N.p2);
    conv_rows(c, 3, N.a[5], R, nullptr);
    conv_rows(c, 4, N.a[6], R, nullptr);
    conv_rows(c, 5, N.a[7], Q, nullptr, N.a[6], N.a[4], N.u1);
    conv_rows(c, 6, N.a[8], Q, nullptr);
    conv_rows(c, 7, N.a[9], P, nullptr, N.a[8], N.a[2], N.u0);
    conv_rows(c, 8, N.a[10], P, nullptr);
    const int64_t ob = param_off(kNumConv32 + 1);
    k_conv_out<<<gP, 256, 0, c->stream>>>(N.a[10], N.out_frag, N.w + ob + kOutW, P, N.out);
    c->launches += 2;
}

// Loss of the guess N.out against the scaled right-hand-side change rhs
// (free nodes of the node grid): residual, its sum into *loss_slot, and
// dloss/dout into N.dout.
static void enqueue_loss(pic_ctx* c, const float* rhs, float* loss_slot) {
    Net& N = c->ws->net;
    const int64_t nodes = c->nodes;
    const float kappa = N.s2 / N.s1;
    const float beta = (float)((c->dx * c->dx) / (c->dy * c->dy));
    const float inv_count = 1.f / (float)nodes;
    k_resid<<<g1(nodes), 256, 0, c->stream>>>(N.out, rhs, c->mask, N.GX, N.GY, N.P, kappa, beta,
                                              inv_count, N.resid, N.loss_partial);
    k_sum_partials<<<sum_blocks(1), 256, 0, c->stream>>>(N.loss_partial, (int)g1(nodes), 1, loss_slot);
    k_resid_grad<<<g1((int64_t)N.P * N.P), 256, 0, c->stream>>>(N.resid, c->mask, N.GX, N.GY, N.P,
                                                                kappa, beta, inv_count, N.dout);
    c->launches += 3;
}

// Backward pass from N.dout (dloss/dout) into N.g (overwrites the gradient).
static void backward(pic_ctx* c) {
    Net& N = c->ws->net;
    const int P = N.P, Q = P / 2, R = P / 4;
    const int64_t ob = param_off(kNumConv32 + 1);
    __nv_bfloat16 *B0 = N.d_big[0], *B1 = N.d_big[1], *B2 = N.d_big[2];
    __nv_bfloat16 *M0 = N.d_mid[0], *M1 = N.d_mid[1], *M2 = N.d_mid[2];
    __nv_bfloat16 *S0 = N.d_small[0], *S1 = N.d_small[1];
    // output conv
    k_wgrad_out<<<kSmallWgradBlocks, 256, 0, c->stream>>>(N.a[10], N.dout, P, N.partial);
    k_sum_partials<<<sum_blocks(kOutOut), 256, 0, c->stream>>>(N.partial, kSmallWgradBlocks, kOutOut, N.g + ob);
    k_conv_out_dx<<<g1((int64_t)P * P, 128), 128, 0, c->stream>>>(N.dout, N.w + ob, N.a[10], P, B0);
    // B0 = dPre10
    wgrad32(c, 8, 0, P);
    conv_rows_grad(c, 8, 0, B1, P, N.a[9]);        // B1 = dPre9
    wgrad32(c, 7, 1, P);
    conv_rows_grad(c, 7, 1, B2, P, nullptr);       // B2 = dU0
    k_down_sum_gate<<<g1((int64_t)Q * Q * C), 256, 0, c->stream>>>(B2, N.a[8], P, M0);  // M0 = dPre8
    wgrad32(c, 6, 2, Q);
    conv_rows_grad(c, 6, 2, M1, Q, N.a[7]);        // M1 = dPre7
    wgrad32(c, 5, 3, Q);
    conv_rows_grad(c, 5, 3, M2, Q, nullptr);       // M2 = dU1
    k_down_sum_gate<<<g1((int64_t)R * R * C), 256, 0, c->stream>>>(M2, N.a[6], Q, S0);  // S0 = dPre6
    wgrad32(c, 4, 4, R);
    conv_rows_grad(c, 4, 4, S1, R, N.a[5]);        // S1 = dPre5
    wgrad32(c, 3, 5, R);
    conv_rows_grad(c, 3, 5, S0, R, nullptr);       // S0 = dP2
    k_skip_pool_gate<<<g1((int64_t)Q * Q * C), 256, 0, c->stream>>>(M2, S0, N.a[4], Q, M0);  // M0 = dPre4
    wgrad32(c, 2, 2, Q);
    conv_rows_grad(c, 2, 2, M1, Q, N.a[3]);        // M1 = dPre3
    wgrad32(c, 1, 3, Q);
    conv_rows_grad(c, 1, 3, M0, Q, nullptr);       // M0 = dP1
    k_skip_pool_gate<<<g1((int64_t)P * P * C), 256, 0, c->stream>>>(B2, M0, N.a[2], P, B0);  // B0 = dPre2
    wgrad32(c, 0, 0, P);
    conv_rows_grad(c, 0, 0, B1, P, N.a[1]);        // B1 = dPre1
    k_wgrad_in<<<kSmallWgradBlocks, 256, 0, c->stream>>>(N.xin, B1, P, N.partial);
    k_sum_partials<<<sum_blocks(kInOut), 256, 0, c->stream>>>(N.partial, kSmallWgradBlocks, kInOut, N.g);
    c->launches += 2 + 1 + 10 * 3 + 4 + 2;
}

}  // namespace picb200

// ---------------------------------------------------------------------------
// Hooks used by the Poisson solve and the C ABI
// ---------------------------------------------------------------------------
namespace picb200 {

// A trained network (or a recording in progress) needs phi_{n-1} and b_{n-1}
// at every solve, whichever warm start the solve itself uses.
bool ws_tracking(const pic_ctx* c) { return c->ws && (c->ws_record || c->ws->net.trained); }

void ws_free(pic_ctx* c) {
    if (!c->ws) return;
    net_free(c->ws->net);
    delete c->ws;
    c->ws = nullptr;
}

// Before the solve: remember phi_{n-1} and b_{n-1} (after overwriteRho the
// device rho holds b).  Called with the new b already in place.
int ws_before_solve(pic_ctx* c, bool want_guess) {
    if (!c->ws) PIC_TRY(ws_alloc(c));
    Net& N = c->ws->net;
    const int64_t n = c->nodes;
    if (N.have_prev) k_diff<<<g1(n), 256, 0, c->stream>>>(c->rho, N.b_prev, n, N.db);
    PIC_CUDA(cudaMemcpyAsync(N.phi_prev, c->phi, (size_t)n * 8, cudaMemcpyDeviceToDevice, c->stream));
    if (want_guess && N.have_prev && N.trained) {
        PIC_TRY(ws_pack(c));
        k_make_input<<<g1((int64_t)N.P * N.P), 256, 0, c->stream>>>(
            N.phi_prev, N.db, c->mask, N.GX, N.GY, N.P, 1.f / N.s0, (float)(c->dx * c->dx) / N.s1, N.x0);
        N.xin = N.x0;
        forward(c);
        PIC_TRY(ws_guess_buffer(c));
        k_make_guess<<<g1(n), 256, 0, c->stream>>>(N.phi_prev, N.out, c->mask, N.GX, N.GY, N.P, N.s2,
                                                   c->ps.net_guess);
        c->launches += 3;
        PIC_CUDA(cudaGetLastError());
        return 1;  // guess available
    }
    return 0;
}

// After the solve: record (input, target) when recording, keep b for the
// next step.
int ws_after_solve(pic_ctx* c, bool record) {
    Net& N = c->ws->net;
    const int64_t n = c->nodes;
    if (record && N.have_prev && N.cap_pairs > 0) {
        if (N.auto_scale) {
            // root-mean-square of each quantity over the non-electrode nodes
            constexpr int kB = 148;
            double* part = reinterpret_cast<double*>(N.partial);
            k_sumsq4<<<kB, 256, 0, c->stream>>>(N.phi_prev, N.db, c->phi, c->mask, n, c->dx * c->dx, part);
            c->launches += 1;
            double h[kB * 4];
            PIC_CUDA(cudaMemcpyAsync(h, part, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
            PIC_CUDA(cudaStreamSynchronize(c->stream));
            double t[4] = {0, 0, 0, 0};
            for (int b = 0; b < kB; ++b)
                for (int k = 0; k < 4; ++k) t[k] += h[b * 4 + k];
            float sc[3];
            for (int k = 0; k < 3; ++k) {
                const double rms = std::sqrt(t[k] / std::max(t[3], 1.0));
                sc[k] = (rms > 0 && std::isfinite(rms)) ? (float)rms : 1.f;
            }
            N.s0 = sc[0];
            N.s1 = sc[1];
            N.s2 = sc[2];
            N.auto_scale = false;
        }
        const int64_t slot = N.next_pair;
        k_make_input<<<g1((int64_t)N.P * N.P), 256, 0, c->stream>>>(
            N.phi_prev, N.db, c->mask, N.GX, N.GY, N.P, 1.f / N.s0, (float)(c->dx * c->dx) / N.s1,
            N.ds_x + slot * (int64_t)N.P * N.P * 4);
        k_rhs<<<g1(n), 256, 0, c->stream>>>(N.db, c->mask, n, c->dx * c->dx / N.s1, N.ds_t + slot * n);
        N.next_pair = (N.next_pair + 1) % N.cap_pairs;
        N.n_pairs = std::min(N.n_pairs + 1, N.cap_pairs);
    }
    PIC_CUDA(cudaMemcpyAsync(N.b_prev, c->rho, (size_t)n * 8, cudaMemcpyDeviceToDevice, c->stream));
    N.have_prev = true;
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

}  // namespace picb200

extern "C" {

int pic_ws_record(pic_ctx* c, int64_t max_pairs, double phi_scale, double db_scale,
                  double target_scale) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (max_pairs == 0) {  // stop recording, keep the dataset and the scales
        c->ws_record = false;
        return PIC_OK;
    }
    if (c->periodic && max_pairs > 0)
        return fail(PIC_ERR_CONFIG, "periodic in y: the learned warm start is not available");
    PIC_TRY(ws_alloc(c));
    Net& N = c->ws->net;
    if (max_pairs < 0) {  // stop and release the dataset
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(N.ds_x);
        cudaFree(N.ds_t);
        N.ds_x = nullptr;
        N.ds_t = nullptr;
        N.cap_pairs = N.n_pairs = N.next_pair = 0;
        c->ws_record = false;
        return PIC_OK;
    }
    const bool autos = phi_scale == 0 && db_scale == 0 && target_scale == 0;
    if (!autos && (!(phi_scale > 0) || !(db_scale > 0) || !(target_scale > 0)))
        return fail(PIC_ERR_ARG, "warm start: scales must all be positive, or all 0 (automatic)");
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(N.ds_x);
    cudaFree(N.ds_t);
    cudaFree(N.loss_acc);
    N.ds_x = nullptr;
    N.ds_t = nullptr;
    N.loss_acc = nullptr;
    N.cap_pairs = N.n_pairs = N.next_pair = 0;
    c->ws_record = false;
    if (cudaMalloc(&N.ds_x, (size_t)max_pairs * N.P * N.P * 4 * 2) ||
        cudaMalloc(&N.ds_t, (size_t)max_pairs * c->nodes * 4) ||
        cudaMalloc(&N.loss_acc, (size_t)max_pairs * 4)) {
        cudaGetLastError();
        cudaFree(N.ds_x);
        cudaFree(N.ds_t);
        cudaFree(N.loss_acc);
        N.ds_x = nullptr;
        N.ds_t = nullptr;
        N.loss_acc = nullptr;
        return fail(PIC_ERR_CAPACITY, "warm start: dataset does not fit in device memory");
    }
    N.s0 = (float)phi_scale;
    N.s1 = (float)db_scale;
    N.s2 = (float)target_scale;
    N.auto_scale = autos;
    N.cap_pairs = max_pairs;
    c->ws_record = true;
    return PIC_OK;
}

int pic_ws_pairs(pic_ctx* c, int64_t* n) {
    if (!c || !n) return fail(PIC_ERR_ARG, "null argument");
    *n = c->ws ? c->ws->net.n_pairs : 0;
    return PIC_OK;
}

// Adam over the recorded pairs, one pair a step, the pairs of each epoch in
// an order drawn afresh (a seeded permutation: training is repeatable); the
// step size follows lr(t) = lr_min + (lr_max - lr_min) (1 + cos(pi t / T)) / 2
// over the T steps of the call (constant when lr_min == lr_max).
static int ws_train(pic_ctx* c, int epochs, double lr_max, double lr_min, double* loss_out) {
    if (!c || epochs < 0 || !(lr_max > 0) || !(lr_min > 0) || lr_min > lr_max)
        return fail(PIC_ERR_ARG, "warm start: bad training arguments");
    if (!c->ws || c->ws->net.n_pairs == 0) return fail(PIC_ERR_STATE, "warm start: no recorded pairs");
    Net& N = c->ws->net;
    const int P = N.P;
    const int64_t np = N.n_pairs, total = (int64_t)epochs * np;
    std::vector<int64_t> order((size_t)np);
    double last = 0;
    int64_t t = 0;
    for (int e = 0; e < epochs; ++e) {
        for (int64_t s = 0; s < np; ++s) order[(size_t)s] = s;
        uint64_t z = 0x9E3779B97F4A7C15ull * (uint64_t)(N.adam_t + 1) + (uint64_t)e;
        for (int64_t s = np - 1; s > 0; --s) {  // Fisher-Yates with splitmix64 draws
            z += 0x9E3779B97F4A7C15ull;
            uint64_t r = z;
            r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
            r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
            r ^= r >> 31;
            std::swap(order[(size_t)s], order[(size_t)(r % (uint64_t)(s + 1))]);
        }
        double ep = 0;
        for (int64_t k = 0; k < np; ++k, ++t) {
            const int64_t s = order[(size_t)k];
            PIC_TRY(ws_pack(c));
            N.xin = N.ds_x + s * (int64_t)P * P * 4;
            forward(c);
            enqueue_loss(c, N.ds_t + s * c->nodes, N.loss_acc + s);
            backward(c);
            N.adam_t += 1;
            const double lr = lr_min + (lr_max - lr_min) * 0.5 *
                                           (1.0 + std::cos(3.141592653589793 * (double)t / (double)std::max<int64_t>(total, 1)));
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f / (1.f - std::pow(b1, (float)N.adam_t));
            const float c2 = 1.f / (1.f - std::pow(b2, (float)N.adam_t));
            k_adam<<<g1(kParams), 256, 0, c->stream>>>(N.w, N.m, N.v, N.g, kParams, (float)lr, b1, b2,
                                                       1e-8f, c1, c2, 1.f, nullptr, nullptr);
            N.packed = false;
            c->launches += 1;
        }
        std::vector<float> ls((size_t)np);
        PIC_CUDA(cudaMemcpyAsync(ls.data(), N.loss_acc, ls.size() * 4, cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        PIC_TRY(ws_check_fault());
        for (float v : ls) ep += v;
        last = ep / (double)np;
    }
    N.trained = true;
    PIC_TRY(ws_guess_buffer(c));
    if (loss_out) *loss_out = last;
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int pic_ws_train(pic_ctx* c, int epochs, double lr, double* loss_out) {
    return ws_train(c, epochs, lr, lr, loss_out);
}

int pic_ws_train_cosine(pic_ctx* c, int epochs, double lr_max, double lr_min, double* loss_out) {
    return ws_train(c, epochs, lr_max, lr_min, loss_out);
}

int pic_ws_get_params(pic_ctx* c, float* host, int64_t n) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    if (n < kParams) return fail(PIC_ERR_CAPACITY, "warm start: parameter buffer too small");
    PIC_TRY(ws_alloc(c));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    PIC_CUDA(cudaMemcpy(host, c->ws->net.w, kParams * 4, cudaMemcpyDeviceToHost));
    return PIC_OK;
}

int pic_ws_set_params(pic_ctx* c, const float* host, int64_t n, double phi_scale, double db_scale,
                      double target_scale) {
    if (!c || !host || n != kParams) return fail(PIC_ERR_ARG, "warm start: parameter count mismatch");
    PIC_TRY(ws_alloc(c));
    Net& N = c->ws->net;
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    PIC_CUDA(cudaMemcpy(N.w, host, kParams * 4, cudaMemcpyHostToDevice));
    N.packed = false;
    N.s0 = (float)phi_scale;
    N.s1 = (float)db_scale;
    N.s2 = (float)target_scale;
    N.trained = true;
    PIC_TRY(ws_guess_buffer(c));
    return PIC_OK;
}

int64_t pic_ws_num_params(void) { return kParams; }

// One forward + backward on a caller-given input image and scaled
// right-hand-side change, for gradient checks: x0 host [P*P*3] (channels phi,
// RHS change, mask, already scaled), rhs host [GX*GY]; returns out [P*P],
// gradient [kParams], loss.  Uses the network's current scales for kappa.
int pic_ws_debug_step(pic_ctx* c, const float* x0_host, const float* rhs_host, float* out_host,
                      float* grad_host, double* loss) {
    if (!c || !x0_host || !rhs_host) return fail(PIC_ERR_ARG, "null argument");
    PIC_TRY(ws_alloc(c));
    Net& N = c->ws->net;
    const int P = N.P;
    std::vector<__nv_bfloat16> x((size_t)P * P * 4);
    for (int64_t p = 0; p < (int64_t)P * P; ++p) {
        for (int ch = 0; ch < 3; ++ch) x[p * 4 + ch] = __float2bfloat16(x0_host[p * 3 + ch]);
        x[p * 4 + 3] = __float2bfloat16(0.f);
    }
    float* t = nullptr;
    float* l = nullptr;
    PIC_CUDA(cudaMalloc(&t, (size_t)c->nodes * 4));
    PIC_CUDA(cudaMalloc(&l, 4));
    PIC_CUDA(cudaMemcpy(N.x0, x.data(), x.size() * 2, cudaMemcpyHostToDevice));
    PIC_CUDA(cudaMemcpy(t, rhs_host, (size_t)c->nodes * 4, cudaMemcpyHostToDevice));
    PIC_TRY(ws_pack(c));
    N.xin = N.x0;
    forward(c);
    enqueue_loss(c, t, l);
    backward(c);
    float lh = 0.f;
    PIC_CUDA(cudaMemcpyAsync(&lh, l, 4, cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(t);
    cudaFree(l);
    PIC_TRY(ws_check_fault());
    if (out_host) PIC_CUDA(cudaMemcpy(out_host, N.out, (size_t)P * P * 4, cudaMemcpyDeviceToHost));
    if (grad_host) PIC_CUDA(cudaMemcpy(grad_host, N.g, kParams * 4, cudaMemcpyDeviceToHost));
    if (loss) *loss = lh;
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int pic_ws_scales(pic_ctx* c, double* scales) {
    if (!c || !scales) return fail(PIC_ERR_ARG, "null argument");
    if (!c->ws) return fail(PIC_ERR_STATE, "warm start: no network");
    const Net& N = c->ws->net;
    scales[0] = N.s0;
    scales[1] = N.s1;
    scales[2] = N.s2;
    return PIC_OK;
}

int pic_ws_grid(pic_ctx* c, int* P) {
    if (!c || !P) return fail(PIC_ERR_ARG, "null argument");
    *P = ((std::max(c->GX, c->GY) + 3) / 4) * 4;
    return PIC_OK;
}

}  // extern "C"
