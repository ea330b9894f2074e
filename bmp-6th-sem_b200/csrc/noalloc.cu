// noalloc.cu -- charge deposition of reference Points that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they need a
// deposit: a host framework that owns a fixed device-memory budget and hands
// plugins only the buffers it has already sized, or a time-critical loop
// that must not call cudaMalloc/cudaFree because those may synchronise the
// whole device.  pic_deposit_points_noalloc serves them: the caller passes
// the particles and the output grids, and the one scratch buffer the
// deposit needs (the 64-bit fixed-point node accumulators) is a file-scope
// __device__ array of fixed size that every GPU loading this library keeps
// until the process exits.
//
// The arithmetic is the library's own deposit: the cell of a Point is
// (int)(x*(1/dx)), the FP32 in-cell offset is the FP64 remainder, each axis
// offset is rounded to 20 bits and the four corner weights are exact 40-bit
// products summed in 64-bit integers -- so the result is bit-for-bit the
// final_mesh / rho that pic_import_points + pic_charge_deposition produce.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "pic_internal.h"

namespace picb200 {
namespace {

// 2^19 nodes = 4 MiB of accumulators, e.g. up to 724 x 724 nodes.
constexpr int64_t kNoAllocMaxNodes = 1ll << 19;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned long long g_noalloc_acc[kNoAllocMaxNodes];

std::mutex g_mu;
// Per device: the device address of the scratch array and the unique id of
// the CUDA context it was looked up in.  The address belongs to the module
// as loaded into that context; after cudaDeviceReset the next primary
// context loads the module again, possibly at another address, so a change
// of context id means a new lookup.
struct ScratchSlot {
    unsigned long long ctx_id;
    unsigned long long* addr;
};
ScratchSlot g_slot[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The current context's unique id through the driver entry points (no link
// against libcuda); 0 when the driver cannot tell, which disables the cache.
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
            get_id = reinterpret_cast<CtxGetIdFn>(f2);
        }
        cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array on the current device (the host-side
// name of the array is not a device address), looked up with the device
// current once per device and context.
int scratch_address(unsigned long long** out) {
    int dev = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(PIC_ERR_NO_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    // 0 before the runtime has made the device's primary context current: the
    // lookup below does that, and the id is read again after it
    const unsigned long long id = current_context_id();
    ScratchSlot& slot = g_slot[dev];
    if (!slot.addr || id == 0 || slot.ctx_id != id) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
        if (e != cudaSuccess) {
            slot.addr = nullptr;
            return fail(PIC_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_acc): ") +
                                          cudaGetErrorString(e));
        }
        slot.addr = static_cast<unsigned long long*>(p);
        slot.ctx_id = current_context_id();
    }
    *out = slot.addr;
    return PIC_OK;
}

__global__ void k_na_clear(unsigned long long* acc, int64_t nodes) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nodes) acc[i] = 0ull;
}

__device__ __forceinline__ uint32_t na_axis(float f) {
    const float t = __fadd_rn(__fmul_rn(f, (float)(1u << kAxisBits)), 12582912.0f);
    return __float_as_uint(t) - 0x4B400000u;
}

__global__ void k_na_deposit(const pic_point* __restrict__ pts, int64_t n, int nx, int ny, int GX,
                             double inv_dx, double inv_dy, unsigned long long* acc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const pic_point p = pts[i];
    if (p.pointer == -1) return;
    const double sx = p.x * inv_dx, sy = p.y * inv_dy;
    if (!(sx >= 0.0 && sy >= 0.0 && sx < (double)nx && sy < (double)ny)) return;
    const int gx = (int)sx, gy = (int)sy;
    const float one_below = 0x1.fffffep-1f;
    const float fx = fminf((float)(sx - gx), one_below);
    const float fy = fminf((float)(sy - gy), one_below);
    const uint32_t ax = na_axis(fx), ay = na_axis(fy);
    const uint32_t bx = (1u << kAxisBits) - ax, by = (1u << kAxisBits) - ay;
    unsigned long long* q = acc + (int64_t)gy * GX + gx;
    atomicAdd(q, (unsigned long long)bx * by);
    atomicAdd(q + 1, (unsigned long long)ax * by);
    atomicAdd(q + GX, (unsigned long long)bx * ay);
    atomicAdd(q + GX + 1, (unsigned long long)ax * ay);
}

__global__ void k_na_finish(const unsigned long long* acc, int64_t nodes, double qscale,
                            double chrg, double* final_mesh, double* rho) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const double f = (double)acc[i] * qscale;
    final_mesh[i] = f;
    if (rho) rho[i] += f * chrg;
}

}  // namespace
}  // namespace picb200

using namespace picb200;

extern "C" int pic_deposit_points_noalloc(const pic_point* dev_points, int64_t n, int32_t nx,
                                          int32_t ny, double xmax, double ymax,
                                          const pic_species_desc* species, double surf_area,
                                          double epsilon, double* dev_final_mesh,
                                          double* dev_rho, void* cuda_stream) {
    if (n < 0 || (n > 0 && !dev_points) || !species || !dev_final_mesh)
        return fail(PIC_ERR_ARG, "pic_deposit_points_noalloc: null pointer or negative count");
    if (nx < 1 || ny < 1 || !(xmax > 0) || !(ymax > 0) || !(epsilon > 0) ||
        !(species->sim_count > 0))
        return fail(PIC_ERR_CONFIG, "pic_deposit_points_noalloc: bad grid or species description");
    const int64_t GX = (int64_t)nx + 1, nodes = GX * ((int64_t)ny + 1);
    if (nodes > kNoAllocMaxNodes)
        return fail(PIC_ERR_CAPACITY,
                    "pic_deposit_points_noalloc: grid of " + std::to_string(nodes) +
                        " nodes exceeds the fixed scratch of " + std::to_string(kNoAllocMaxNodes) +
                        " nodes");
    unsigned long long* acc = nullptr;
    PIC_TRY(scratch_address(&acc));
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    const double dx = xmax / nx, dy = ymax / ny;
    const double surf = surf_area > 0 ? surf_area : xmax * ymax;
    // updateWeighingFactor, src/particles.cpp:303-305
    const double weighing = species->actual_count * surf / (species->sim_count * dx * dy * dx * dy);
    const double qscale = kChargeUnit * (dx * dy) * weighing;  // as the context's flush rounds it
    const double chrg = -species->charge / epsilon;  // RhoKernel, src/interpolation.cpp:164-170
    k_na_clear<<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(acc, nodes);
    if (n > 0)
        k_na_deposit<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dev_points, n, nx, ny, (int)GX,
                                                                  1.0 / dx, 1.0 / dy, acc);
    k_na_finish<<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(acc, nodes, qscale, chrg,
                                                                 dev_final_mesh, dev_rho);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}
