// gpe_calc_fi3d_noalloc: the dipolar potential without any device allocation.
//
// Some callers cannot call cudaMalloc: a host framework that owns all device
// memory through its own allocator (a caching allocator or a pre-reserved
// pool), or a time-critical loop that must not add the device-wide
// synchronisation cudaMalloc/cudaFree can cause.  For them this entry point
// computes phi = calc_fi3d(psi) (same kernels as the handle-based path) with
// every intermediate in one file-scope __device__ array of fixed size.  The
// caller passes device pointers to psi (complex64) and phi (float); nothing
// else is allocated, on the device or in pinned host memory.
//
// Limits and sharing:
//  * scratch holds the pruned dipolar spectrum (nx * 2ny * (nz+1) complex64),
//    the V_dd(k) table ((nx+1) * (ny+1) * (nz+1) floats) and three twiddle
//    tables with their rounding remainders; grids needing more than GPE_NOALLOC_SCRATCH_BYTES are rejected
//    with GPE_ERR_SIZE (128 x 128 x 32 needs about 10.9 MB);
//   * the array lives on every GPU that loads the library until the process
//    exits, and every call on a GPU shares it: calls that overlap on that GPU
//    (other streams, other threads) race.  Every call rebuilds the twiddle and
//    V_dd(k) tables it needs before its passes (a few microseconds): no state
//    carries over from one call to the next, whatever stream or grid the
//    previous call used;
//  * the first call on each device does a one-time set-up on the host (looks
//    up the array's device address with cudaGetSymbolAddress and raises the
//    kernels' shared-memory limit to the device's opt-in maximum); make that
//    first call before any stream capture on that device.
#include "../../include/gpe_b200.h"
#include "kernels.cuh"
#include "plan.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

namespace gpe {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GPE_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

struct NoallocSlot {
    bool ready          = false;
    unsigned char *base = nullptr; // device address of g_noalloc_scratch
    size_t smem_max     = 0;       // dynamic shared memory the kernels may use on this device
};

std::mutex g_noalloc_mu;
NoallocSlot g_noalloc_slots[kMaxDevices];

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// exp(-2 pi i m / L) in FP64, rounded to float2 (tw) with the rounding
// remainder in twlo (the FFT stages multiply by tw + twlo, compensated).
__global__ void k_na_twiddles(float2 *tw, float2 *twlo, int L) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)L, &s, &c);
        const float ch = (float)c, sh = (float)-s;
        tw[m]          = make_float2(ch, sh);
        twlo[m]        = make_float2((float)(c - (double)ch), (float)(-s - (double)sh));
    }
}

// V_dd(k) = kz^2 / k^2 on the (2nx, 2ny, 2nz) box, reduced by |kx|, |ky| symmetry
// (fftw_poisson_solver.cpp:12-49), FP64 then rounded to float.
__global__ void k_na_vdip(float *vk, int nx, int ny, int nz, double dx, double dy, double dz) {
    const int H = nz + 1, px = 2 * nx, py = 2 * ny, pz = 2 * nz;
    const double dkx = 2. * M_PI / (px * dx), dky = 2. * M_PI / (py * dy), dkz = 2. * M_PI / (pz * dz);
    const size_t total = (size_t)(nx + 1) * (ny + 1) * H;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % H), j = (int)((q / H) % (ny + 1)), i = (int)(q / ((size_t)H * (ny + 1)));
        const double kx = i * dkx, ky = j * dky, kz = k * dkz;
        const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
        vk[q]           = (k2 > 1e-30) ? (float)__ddiv_rn(__dmul_rn(kz, kz), k2) : 0.0f;
    }
}

struct Layout {
    size_t a_off, vk_off, twx_off, twy_off, twz_off, total;
    // each twiddle region holds the table followed by its remainder table
};

Layout layout(int nx, int ny, int nz) {
    Layout l{};
    const int H = nz + 1;
    size_t off = 0;
    l.a_off    = off;
    off += align256(sizeof(float2) * (size_t)nx * 2 * ny * H);
    l.vk_off = off;
    off += align256(sizeof(float) * (size_t)(nx + 1) * (ny + 1) * H);
    l.twx_off = off;
    off += align256(sizeof(float2) * 2 * 2 * (size_t)nx);
    l.twy_off = off;
    off += align256(sizeof(float2) * 2 * 2 * (size_t)ny);
    l.twz_off = off;
    off += align256(sizeof(float2) * 2 * 2 * (size_t)nz);
    l.total = off;
    return l;
}

int tile_for(int L, int pad) {
    int TB = 32;
    while (TB > 1 && 2 * sizeof(float2) * (size_t)(TB + pad) * L > 64 * 1024)
        TB >>= 1;
    return TB;
}

LinePlan line(int L, const float2 *tw) {
    LinePlan p{};
    std::vector<int> r = factor_line(L);
    p.L                = L;
    p.nstages          = (int)r.size();
    for (size_t s = 0; s < r.size(); ++s)
        p.radix[s] = r[s];
    p.tw = tw;
    return p;
}

int fail(int code, const std::string &msg) {
    last_error() = msg;
    return code;
}

} // namespace
} // namespace gpe

extern "C" int gpe_calc_fi3d_noalloc(const void *psi_c64_dev, float *fi3d_dev, int nx, int ny, int nz,
                                     double dx, double dy, double dz, double n_atoms,
                                     void *cuda_stream) {
    using namespace gpe;
    if (!psi_c64_dev || !fi3d_dev)
        return fail(GPE_ERR_ARG, "gpe_calc_fi3d_noalloc: null device pointer");
    if (nx < 1 || ny < 1 || nz < 1 || !(dx > 0) || !(dy > 0) || !(dz > 0))
        return fail(GPE_ERR_ARG, "gpe_calc_fi3d_noalloc: grid dimensions and spacings must be positive");
    const Layout lay = layout(nx, ny, nz);
    if (lay.total > (size_t)GPE_NOALLOC_SCRATCH_BYTES)
        return fail(GPE_ERR_SIZE, "gpe_calc_fi3d_noalloc: a " + std::to_string(nx) + "x" +
                                      std::to_string(ny) + "x" + std::to_string(nz) + " grid needs " +
                                      std::to_string(lay.total) + " bytes of scratch, above the " +
                                      std::to_string((size_t)GPE_NOALLOC_SCRATCH_BYTES) +
                                      "-byte limit");
    LinePlan lx, ly, lz;
    try {
        lx = line(2 * nx, nullptr);
        ly = line(2 * ny, nullptr);
        lz = line(2 * nz, nullptr);
    } catch (const Error &e) {
        return fail(e.code, std::string("gpe_calc_fi3d_noalloc: ") + e.what());
    }
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess)
        return fail(GPE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(GPE_ERR_ARG, "gpe_calc_fi3d_noalloc: device ordinal out of range");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const int TBx = tile_for(lx.L, 0), TBy = tile_for(ly.L, 0), TBz = tile_for(lz.L, 1);
    const size_t smx = 2 * sizeof(float2) * (size_t)TBx * lx.L;
    const size_t smy = 2 * sizeof(float2) * (size_t)TBy * ly.L;
    const size_t smz = 2 * sizeof(float2) * (size_t)(TBz + 1) * lz.L; // z tiles: odd stride TB + 1

    NoallocSlot &slot = g_noalloc_slots[dev];
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!slot.ready) {
            // One-time set-up on this device: the host-side name of the array is
            // not its device address, so look the address up.
            void *p = nullptr;
            err     = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (err != cudaSuccess)
                return fail(GPE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
            int optin = 0;
            err       = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (err != cudaSuccess)
                return fail(GPE_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(err));
            const void *kern[] = {(const void *)k_dip_z_fwd<float>, (const void *)k_dip_y<-1, float>,
                                  (const void *)k_dip_y<+1, float>, (const void *)k_dip_x<float>,
                                  (const void *)k_dip_z_inv<float>};
            for (const void *f : kern) {
                err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
                if (err != cudaSuccess)
                    return fail(GPE_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
            }
            slot.base     = static_cast<unsigned char *>(p);
            slot.smem_max = (size_t)optin;
            slot.ready    = true;
        }
    }
    if (smx > slot.smem_max || smy > slot.smem_max || smz > slot.smem_max)
        return fail(GPE_ERR_SIZE, "gpe_calc_fi3d_noalloc: the line tiles of this grid need more shared memory "
                                  "than the device allows per block");
    // An error left by earlier, unrelated work would be reported as this call's:
    // refuse to start instead (the error stays pending for its owner).
    err = cudaPeekAtLastError();
    if (err != cudaSuccess)
        return fail(GPE_ERR_CUDA, std::string("gpe_calc_fi3d_noalloc: a CUDA error from earlier work is pending: ") +
                                      cudaGetErrorString(err));
    unsigned char *base = slot.base;
    float2 *A           = reinterpret_cast<float2 *>(base + lay.a_off);
    float *vk           = reinterpret_cast<float *>(base + lay.vk_off);
    float2 *twx         = reinterpret_cast<float2 *>(base + lay.twx_off);
    float2 *twy         = reinterpret_cast<float2 *>(base + lay.twy_off);
    float2 *twz         = reinterpret_cast<float2 *>(base + lay.twz_off);
    lx.tw               = twx;
    ly.tw               = twy;
    lz.tw               = twz;
    lx.twlo             = twx + 2 * nx;
    ly.twlo             = twy + 2 * ny;
    lz.twlo             = twz + 2 * nz;
    const int H         = nz + 1;

    // the tables of this grid, rebuilt by every call (in stream order before the
    // passes that read them)
    k_na_twiddles<<<(2 * nx + 255) / 256, 256, 0, s>>>(twx, twx + 2 * nx, 2 * nx);
    k_na_twiddles<<<(2 * ny + 255) / 256, 256, 0, s>>>(twy, twy + 2 * ny, 2 * ny);
    k_na_twiddles<<<(2 * nz + 255) / 256, 256, 0, s>>>(twz, twz + 2 * nz, 2 * nz);
    k_na_vdip<<<592, 256, 0, s>>>(vk, nx, ny, nz, dx, dy, dz);
    // The pruned dipolar convolution: every element of A that a pass reads was
    // written by the pass before it in this call, so nothing needs clearing.
    const int lines = nx * ny;
    const float2 *psi = static_cast<const float2 *>(psi_c64_dev);
    k_dip_z_fwd<float><<<(lines + TBz - 1) / TBz, 256, smz, s>>>(psi, nullptr, 0, A, nx, ny, nz,
                                                                 (float)n_atoms, lz, TBz);
    k_dip_y<-1, float><<<dim3((H + TBy - 1) / TBy, nx), 256, smy, s>>>(A, ny, H, ny, 2 * ny, ly, TBy);
    k_dip_x<float><<<(2 * ny * H + TBx - 1) / TBx, 256, smx, s>>>(A, vk, nx, ny, H, 1.0f, lx, TBx);
    k_dip_y<+1, float><<<dim3((H + TBy - 1) / TBy, nx), 256, smy, s>>>(A, ny, H, 2 * ny, ny, ly, TBy);
    k_dip_z_inv<float><<<(lines + TBz - 1) / TBz, 256, smz, s>>>(
        A, fi3d_dev, nx, ny, nz, (float)(1.0 / (8.0 * (double)nx * ny * nz)), lz, TBz);
    err = cudaGetLastError();
    if (err != cudaSuccess)
        return fail(GPE_ERR_CUDA, std::string("gpe_calc_fi3d_noalloc launch: ") + cudaGetErrorString(err));
    return GPE_OK;
}
