// Learned warm start for imaginary time: a small network maps the physical
// parameters (edd, n_atoms, omega_r, omega_z) to a ground-state amplitude
// |psi_0| on the solver grid; imaginary time then refines that guess instead of
// starting from a Gaussian.  The reference has no counterpart (it always starts
// from its initialisers); plain Gaussian-start imaginary time stays the
// fallback and the reference answer the prediction is measured against.
//
// Network (weights BF16, arithmetic FP32):
//   dense 4 -> H, SiLU;  dense H -> C0 * X0 * Y0 * Z0 (the latent volume), SiLU
//   `levels` stages of: nearest-neighbour upsampling x2 in x, y, z, 3x3x3
//   convolution (zero padding) C_s -> C_{s+1}, SiLU
//   a last 3x3x3 convolution C_L -> 1 at full resolution: the amplitude
//   (linear: a saturating output such as softplus stalls at zero, where the
//   targets are zero over most of the box)
// Volumes are [channel][x][y][z] with z fastest, the solver's layout.
//
// Training minimises the mean squared amplitude error against ground states
// that imaginary time produced, with Adam on FP32 master weights; the BF16
// copies are refreshed after every step.  All of it is memory- and
// latency-bound (few channels, large volumes): the kernels are plain SIMT with
// FP32 accumulation, and none of the products is a dense contraction worth a
// tensor-core tile.
#include "../../include/gpe_b200.h"
#include "plan.hpp"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <random>
#include <type_traits>
#include <string>
#include <vector>

namespace gpe {
namespace {

#define WS_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw Error(e_ == cudaErrorMemoryAllocation ? GPE_ERR_NOMEM : GPE_ERR_CUDA,            \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

template <class T> struct Buf {
    T *p     = nullptr;
    size_t n = 0;
    void alloc(size_t k) {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = k;
        if (k)
            WS_CUDA(cudaMalloc(&p, sizeof(T) * k));
    }
    ~Buf() {
        if (p)
            cudaFree(p);
    }
};

__device__ __forceinline__ float silu(float y) { return y / (1.f + __expf(-y)); }
__device__ __forceinline__ float silu_grad(float y) {
    const float s = 1.f / (1.f + __expf(-y));
    return s * (1.f + y * (1.f - s));
}

// ---------------------------------------------------------------------------
// dense layers: Y[b][o] = sum_i W[o][i] X[b][i] + bias[o]
// ---------------------------------------------------------------------------
__global__ void k_dense_fwd(const float *__restrict__ X, const __nv_bfloat16 *__restrict__ W,
                            const __nv_bfloat16 *__restrict__ bias, float *__restrict__ Ypre,
                            float *__restrict__ Y, int B, int I, int O) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (o >= O || b >= B)
        return;
    float acc = __bfloat162float(bias[o]);
    const __nv_bfloat16 *w = W + (size_t)o * I;
    const float *x         = X + (size_t)b * I;
    for (int i = 0; i < I; ++i)
        acc = fmaf(__bfloat162float(w[i]), x[i], acc);
    Ypre[(size_t)b * O + o] = acc;
    Y[(size_t)b * O + o]    = silu(acc);
}

// G[b][o] = dL/dY[b][o] * silu'(Ypre)  (in place)
__global__ void k_silu_back(float *__restrict__ G, const float *__restrict__ Ypre, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        G[e] *= silu_grad(Ypre[e]);
}

// dW[o][i] = sum_b G[b][o] X[b][i];  db[o] = sum_b G[b][o]
__global__ void k_dense_wgrad(const float *__restrict__ G, const float *__restrict__ X, float *__restrict__ dW,
                              float *__restrict__ db, int B, int I, int O) {
    const size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (e >= (size_t)O * I)
        return;
    const int o = (int)(e / I), i = (int)(e % I);
    float acc = 0.f;
    for (int b = 0; b < B; ++b)
        acc = fmaf(G[(size_t)b * O + o], X[(size_t)b * I + i], acc);
    dW[e] = acc;
    if (i == 0) {
        float s = 0.f;
        for (int b = 0; b < B; ++b)
            s += G[(size_t)b * O + o];
        db[o] = s;
    }
}

// dX[b][i] = sum_o W[o][i] G[b][o]
__global__ void k_dense_xgrad(const float *__restrict__ G, const __nv_bfloat16 *__restrict__ W,
                              float *__restrict__ dX, int B, int I, int O) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (i >= I || b >= B)
        return;
    float acc = 0.f;
    for (int o = 0; o < O; ++o)
        acc = fmaf(__bfloat162float(W[(size_t)o * I + i]), G[(size_t)b * O + o], acc);
    dX[(size_t)b * I + i] = acc;
}

// ---------------------------------------------------------------------------
// 3x3x3 convolution of the (optionally x2 nearest-upsampled) input
// ---------------------------------------------------------------------------
struct ConvGeom {
    int cin, cout;
    int X, Y, Z;    // output (fine) grid
    int up;         // 1: input is (X/2, Y/2, Z/2), read through nearest upsampling
};

// input value of channel c at fine position (x, y, z), zero outside
__device__ __forceinline__ float conv_in(const float *__restrict__ in, const ConvGeom &g, int c, int x, int y,
                                         int z) {
    if (x < 0 || y < 0 || z < 0 || x >= g.X || y >= g.Y || z >= g.Z)
        return 0.f;
    if (g.up) {
        const int Xc = g.X >> 1, Yc = g.Y >> 1, Zc = g.Z >> 1;
        return __ldg(&in[(((size_t)c * Xc + (x >> 1)) * Yc + (y >> 1)) * Zc + (z >> 1)]);
    }
    return __ldg(&in[(((size_t)c * g.X + x) * g.Y + y) * g.Z + z]);
}

constexpr int kMaxCout = 32;

// one thread per output voxel and group of COUT output channels (blockIdx.y =
// sample * groups + group: small volumes spread their channels over more
// threads); weights [o][c][27] BF16 staged in shared memory as FP32.  pre =
// the pre-activation, out = SiLU(pre) (act = 0: out = pre).
template <int COUT>
__global__ void k_conv_fwd(const float *__restrict__ in, const __nv_bfloat16 *__restrict__ W,
                           const __nv_bfloat16 *__restrict__ bias, float *__restrict__ pre,
                           float *__restrict__ out, ConvGeom g, int act, size_t in_stride, size_t out_stride) {
    const int groups = g.cout / COUT;
    const int smp = blockIdx.y / groups, o0 = (blockIdx.y % groups) * COUT;
    extern __shared__ float ws[];
    const int nw = g.cout * g.cin * 27;
    for (int e = threadIdx.x; e < nw; e += blockDim.x)
        ws[e] = __bfloat162float(W[e]);
    __syncthreads();
    const size_t nv = (size_t)g.X * g.Y * g.Z;
    const float *inb = in + smp * in_stride;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(v % g.Z), y = (int)((v / g.Z) % g.Y), x = (int)(v / ((size_t)g.Z * g.Y));
        float acc[COUT];
#pragma unroll
        for (int o = 0; o < COUT; ++o)
            acc[o] = __bfloat162float(bias[o0 + o]);
        for (int c = 0; c < g.cin; ++c)
            for (int t = 0; t < 27; ++t) {
                const int dx = t / 9 - 1, dy = (t / 3) % 3 - 1, dz = t % 3 - 1;
                const float u = conv_in(inb, g, c, x + dx, y + dy, z + dz);
#pragma unroll
                for (int o = 0; o < COUT; ++o)
                    acc[o] = fmaf(ws[((o0 + o) * g.cin + c) * 27 + t], u, acc[o]);
            }
#pragma unroll
        for (int o = 0; o < COUT; ++o) {
            const size_t q = smp * out_stride + (size_t)(o0 + o) * nv + v;
            pre[q]         = acc[o];
            out[q]         = act ? silu(acc[o]) : acc[o];
        }
    }
}

// The same convolution on 8x8x8 output tiles, one voxel per thread (512
// threads): the input tile with its halo is staged in shared memory once
// (zeros outside the volume), the 27 taps and CIN channels unroll, so a voxel
// costs CIN x 27 shared loads and CIN x 27 x COUT FMAs without per-tap index
// arithmetic.  For volumes with all sizes multiples of 8 and the channel
// counts instantiated below.  blockIdx.y = sample.
template <int CIN, int COUT, int UP>
__global__ void __launch_bounds__(512)
    k_conv_fwd_tile(const float *__restrict__ in, const __nv_bfloat16 *__restrict__ W,
                    const __nv_bfloat16 *__restrict__ bias, float *__restrict__ pre, float *__restrict__ out,
                    ConvGeom g, int act, size_t in_stride, size_t out_stride) {
    constexpr int T = UP ? 6 : 10; // staged input tile edge
    __shared__ float ws[COUT * CIN * 27];
    __shared__ float ts[CIN * T * T * T];
    const int tid = threadIdx.x;
    for (int e = tid; e < COUT * CIN * 27; e += 512)
        ws[e] = __bfloat162float(W[e]);
    const int tx = g.X / 8, ty = g.Y / 8;
    const int bx = blockIdx.x / (ty * (g.Z / 8)), rem = blockIdx.x % (ty * (g.Z / 8));
    const int by = rem / (g.Z / 8), bz = rem % (g.Z / 8);
    (void)tx;
    const int x0 = bx * 8, y0 = by * 8, z0 = bz * 8;
    const float *inb = in + blockIdx.y * in_stride;
    // input origin of the tile (coarse grid when UP)
    const int Xi = UP ? g.X / 2 : g.X, Yi = UP ? g.Y / 2 : g.Y, Zi = UP ? g.Z / 2 : g.Z;
    const int ox = UP ? x0 / 2 - 1 : x0 - 1, oy = UP ? y0 / 2 - 1 : y0 - 1, oz = UP ? z0 / 2 - 1 : z0 - 1;
    for (int e = tid; e < CIN * T * T * T; e += 512) {
        const int c = e / (T * T * T), r = e % (T * T * T);
        const int ix = ox + r / (T * T), iy = oy + (r / T) % T, iz = oz + r % T;
        float v = 0.f;
        if (ix >= 0 && iy >= 0 && iz >= 0 && ix < Xi && iy < Yi && iz < Zi)
            v = __ldg(&inb[(((size_t)c * Xi + ix) * Yi + iy) * Zi + iz]);
        ts[e] = v;
    }
    __syncthreads();
    const int lx = tid / 64, ly = (tid / 8) % 8, lz = tid % 8;
    // tile offsets of the three neighbours along each axis
    int ax[3], ay[3], az[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ax[d] = UP ? ((lx + d - 1) >> 1) + 1 : lx + d;
        ay[d] = UP ? ((ly + d - 1) >> 1) + 1 : ly + d;
        az[d] = UP ? ((lz + d - 1) >> 1) + 1 : lz + d;
    }
    float acc[COUT];
#pragma unroll
    for (int o = 0; o < COUT; ++o)
        acc[o] = __bfloat162float(bias[o]);
#pragma unroll
    for (int c = 0; c < CIN; ++c) {
#pragma unroll
        for (int t = 0; t < 27; ++t) {
            const float u = ts[c * T * T * T + (ax[t / 9] * T + ay[(t / 3) % 3]) * T + az[t % 3]];
#pragma unroll
            for (int o = 0; o < COUT; ++o)
                acc[o] = fmaf(ws[(o * CIN + c) * 27 + t], u, acc[o]);
        }
    }
    const size_t nv = (size_t)g.X * g.Y * g.Z;
    const size_t v  = ((size_t)(x0 + lx) * g.Y + (y0 + ly)) * g.Z + (z0 + lz);
#pragma unroll
    for (int o = 0; o < COUT; ++o) {
        const size_t q = blockIdx.y * out_stride + (size_t)o * nv + v;
        pre[q]         = acc[o];
        out[q]         = act ? silu(acc[o]) : acc[o];
    }
}

// weight and bias gradients, stage 1: per chunk of voxels, per output channel o,
// partial[chunk][o][c][t] = sum_v gy[o][v] * u[c][v + t]; partial bias in slot
// [chunk][o][cin * 27].  blockIdx.x = chunk, blockIdx.y = o, blockIdx.z = sample.
constexpr int kChunk = 2048;
__global__ void k_conv_wgrad_partial(const float *__restrict__ in, const float *__restrict__ gy,
                                     float *__restrict__ partial, ConvGeom g, size_t in_stride, size_t g_stride,
                                     int nchunks) {
    __shared__ float gs[kChunk];
    const size_t nv = (size_t)g.X * g.Y * g.Z;
    const int o     = blockIdx.y;
    const size_t v0 = (size_t)blockIdx.x * kChunk;
    const int cnt   = (int)min((size_t)kChunk, nv - v0);
    const float *gyo = gy + blockIdx.z * g_stride + (size_t)o * nv + v0;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x)
        gs[e] = gyo[e];
    __syncthreads();
    const float *inb = in + blockIdx.z * in_stride;
    const int nk     = g.cin * 27 + 1;
    float *dst = partial + (((size_t)blockIdx.z * nchunks + blockIdx.x) * g.cout + o) * nk;
    for (int k = threadIdx.x; k < nk; k += blockDim.x) {
        float acc = 0.f;
        if (k == nk - 1) {
            for (int e = 0; e < cnt; ++e)
                acc += gs[e];
        } else {
            const int c = k / 27, t = k % 27;
            const int dx = t / 9 - 1, dy = (t / 3) % 3 - 1, dz = t % 3 - 1;
            for (int e = 0; e < cnt; ++e) {
                const size_t v = v0 + e;
                const int z = (int)(v % g.Z), y = (int)((v / g.Z) % g.Y), x = (int)(v / ((size_t)g.Z * g.Y));
                acc = fmaf(gs[e], conv_in(inb, g, c, x + dx, y + dy, z + dz), acc);
            }
        }
        dst[k] = acc;
    }
}

// stage 2: dW[o][c][t] = sum over samples and chunks (fixed order); db[o] likewise
__global__ void k_conv_wgrad_reduce(const float *__restrict__ partial, float *__restrict__ dW,
                                    float *__restrict__ db, int cout, int cin, int nparts) {
    const int nk = cin * 27 + 1;
    const int e  = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cout * nk)
        return;
    const int o = e / nk, k = e % nk;
    float acc = 0.f;
    for (int p = 0; p < nparts; ++p)
        acc += partial[((size_t)p * cout + o) * nk + k];
    if (k == nk - 1)
        db[o] = acc;
    else
        dW[(size_t)o * cin * 27 + k] = acc;
}

// input gradient: dU[c][v] = sum_o sum_t W[o][c][t] gy[o][v - t] on the fine
// grid, summed over the 8 fine children of each coarse voxel when the input was
// upsampled.  One thread per input voxel, all input channels (<= 32).
template <int CIN>
__global__ void k_conv_xgrad(const float *__restrict__ gy, const __nv_bfloat16 *__restrict__ W,
                             float *__restrict__ dx, ConvGeom g, size_t g_stride, size_t dx_stride) {
    extern __shared__ float ws[];
    const int nw = g.cout * g.cin * 27;
    for (int e = threadIdx.x; e < nw; e += blockDim.x)
        ws[e] = __bfloat162float(W[e]);
    __syncthreads();
    const int Xi = g.up ? g.X >> 1 : g.X, Yi = g.up ? g.Y >> 1 : g.Y, Zi = g.up ? g.Z >> 1 : g.Z;
    const size_t ni = (size_t)Xi * Yi * Zi, nv = (size_t)g.X * g.Y * g.Z;
    const float *gyb = gy + blockIdx.y * g_stride;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ni; q += (size_t)gridDim.x * blockDim.x) {
        const int zi = (int)(q % Zi), yi = (int)((q / Zi) % Yi), xi = (int)(q / ((size_t)Zi * Yi));
        float acc[CIN];
#pragma unroll
        for (int c = 0; c < CIN; ++c)
            acc[c] = 0.f;
        const int nch = g.up ? 8 : 1;
        for (int ch = 0; ch < nch; ++ch) {
            const int x = g.up ? 2 * xi + (ch >> 2) : xi;
            const int y = g.up ? 2 * yi + ((ch >> 1) & 1) : yi;
            const int z = g.up ? 2 * zi + (ch & 1) : zi;
            for (int t = 0; t < 27; ++t) {
                // output voxel w = v - tap reads u[v] through tap t
                const int ox = x - (t / 9 - 1), oy = y - ((t / 3) % 3 - 1), oz = z - (t % 3 - 1);
                if (ox < 0 || oy < 0 || oz < 0 || ox >= g.X || oy >= g.Y || oz >= g.Z)
                    continue;
                const size_t w = ((size_t)ox * g.Y + oy) * g.Z + oz;
                for (int o = 0; o < g.cout; ++o) {
                    const float gv = __ldg(&gyb[(size_t)o * nv + w]);
#pragma unroll
                    for (int c = 0; c < CIN; ++c)
                        acc[c] = fmaf(ws[(o * CIN + c) * 27 + t], gv, acc[c]);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < CIN; ++c)
            dx[blockIdx.y * dx_stride + (size_t)c * ni + q] = acc[c];
    }
}

// loss partials of (u - target)^2 per block and gu = dL/du = 2 (u - t) / (B n)
__global__ void k_loss(const float *__restrict__ u, const float *__restrict__ t, float *__restrict__ gu,
                       double *__restrict__ part, size_t n_total, float inv_n) {
    double acc = 0.;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n_total; e += (size_t)gridDim.x * blockDim.x) {
        const float d = u[e] - t[e];
        acc += (double)d * d;
        gu[e] = 2.f * d * inv_n;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        part[blockIdx.x] = red[0];
}


// Adam (Kingma and Ba, 2015) on the FP32 master weights, then the BF16 copy.
__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, __nv_bfloat16 *__restrict__ wb, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float ge = g[e];
        const float me = b1 * m[e] + (1.f - b1) * ge;
        const float ve = b2 * v[e] + (1.f - b2) * ge * ge;
        m[e]           = me;
        v[e]           = ve;
        const float we = w[e] - lr * (me / c1) / (sqrtf(ve / c2) + eps);
        w[e]           = we;
        wb[e]          = __float2bfloat16_rn(we);
    }
}

__global__ void k_to_bf16(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, size_t n) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        wb[e] = __float2bfloat16_rn(w[e]);
}

int grid_for(size_t n, int bs = 256) { return (int)std::min<size_t>((n + bs - 1) / bs, 148 * 16); }

// channel counts the kernels are compiled for
bool channels_ok(int c) { return c == 1 || c == 2 || c == 4 || c == 8 || c == 16 || c == 32; }

template <class F> void by_channels(int c, F &&f) {
    switch (c) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: f(std::integral_constant<int, 32>{}); break;
    }
}

} // namespace
} // namespace gpe

using gpe::Buf;

struct gpe_warm {
    gpe_warm_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    // parameter layout (offsets into the flat weight vector)
    struct Layer {
        size_t w = 0, b = 0; // offsets
        int cin = 0, cout = 0;
        gpe::ConvGeom g{};
    };
    size_t d1w = 0, d1b = 0, d2w = 0, d2b = 0, nweights = 0;
    int latent = 0;
    std::vector<Layer> conv; // levels upsampling stages + the last one
    Buf<float> w, m, v, grad;
    Buf<__nv_bfloat16> wb;
    // activations (max_batch samples)
    Buf<float> x, h1pre, h1, h2pre, h2, gh1, gh2;
    std::vector<Buf<float>> pre, act, gact; // per conv layer output
    Buf<float> partial, target_scratch;
    Buf<double> lpart;
    long step = 0;

    size_t vox(int l) const { return (size_t)conv[l].g.X * conv[l].g.Y * conv[l].g.Z; }
};

namespace {

int wbad(const char *msg) {
    gpe::last_error() = msg;
    return GPE_ERR_ARG;
}

template <class F> int wguard(F &&f) {
    try {
        f();
        return GPE_OK;
    } catch (const gpe::Error &e) {
        gpe::last_error() = e.what();
        return e.code;
    } catch (const std::exception &e) {
        gpe::last_error() = e.what();
        return GPE_ERR_CUDA;
    }
}

using gpe::Error;

void forward(gpe_warm *W, int B) {
    using namespace gpe;
    const auto &c = W->cfg;
    cudaStream_t s = W->stream;
    const __nv_bfloat16 *wb = W->wb.p;
    k_dense_fwd<<<dim3((c.hidden + 127) / 128, B), 128, 0, s>>>(W->x.p, wb + W->d1w, wb + W->d1b, W->h1pre.p,
                                                                 W->h1.p, B, c.n_inputs, c.hidden);
    k_dense_fwd<<<dim3((W->latent + 127) / 128, B), 128, 0, s>>>(W->h1.p, wb + W->d2w, wb + W->d2b, W->h2pre.p,
                                                                  W->h2.p, B, c.hidden, W->latent);
    const float *in = W->h2.p;
    size_t in_stride = W->latent;
    for (size_t l = 0; l < W->conv.size(); ++l) {
        const auto &L  = W->conv[l];
        const size_t n = W->vox((int)l) * L.cout;
        const size_t sm = sizeof(float) * L.cin * L.cout * 27;
        const int last  = l + 1 == W->conv.size();
        const size_t nvox = W->vox((int)l);
        if (L.g.X % 8 == 0 && L.g.Y % 8 == 0 && L.g.Z % 8 == 0 && nvox >= 32768) {
            const int tiles = (L.g.X / 8) * (L.g.Y / 8) * (L.g.Z / 8);
            bool done = false;
            auto go = [&](auto CI, auto CO, auto UPc) {
                constexpr int ci = decltype(CI)::value, co = decltype(CO)::value, up = decltype(UPc)::value;
                if (L.cin == ci && L.cout == co && L.g.up == up) {
                    gpe::k_conv_fwd_tile<ci, co, up><<<dim3(tiles, B), 512, 0, s>>>(
                        in, wb + L.w, wb + L.b, W->pre[l].p, W->act[l].p, L.g, last ? 0 : 1, in_stride, n);
                    done = true;
                }
            };
            using I4 = std::integral_constant<int, 4>;
            using I8 = std::integral_constant<int, 8>;
            using I16 = std::integral_constant<int, 16>;
            using I1 = std::integral_constant<int, 1>;
            using U0 = std::integral_constant<int, 0>;
            using U1 = std::integral_constant<int, 1>;
            go(I16{}, I8{}, U1{});
            go(I8{}, I8{}, U1{});
            go(I8{}, I4{}, U1{});
            go(I4{}, I4{}, U1{});
            go(I8{}, I1{}, U0{});
            go(I4{}, I1{}, U0{});
            go(I8{}, I8{}, U0{});
            if (done) {
                in        = W->act[l].p;
                in_stride = n;
                continue;
            }
        }
        // output channels per thread: all of them on large volumes, fewer on
        // small ones, so that a layer runs at least ~64 k threads
        int per = L.cout;
        while (per > 1 && nvox * B * (L.cout / per) < 65536)
            per >>= 1;
        const int groups = L.cout / per;
        gpe::by_channels(per, [&](auto CO) {
            k_conv_fwd<decltype(CO)::value><<<dim3(gpe::grid_for(nvox), B * groups), 256, sm, s>>>(
                in, wb + L.w, wb + L.b, W->pre[l].p, W->act[l].p, L.g, last ? 0 : 1, in_stride, n);
        });
        in        = W->act[l].p;
        in_stride = n;
    }
    WS_CUDA(cudaGetLastError());
}

// gradients of the mean squared amplitude error against `targets` (device,
// B x N floats); returns the loss (host)
double backward(gpe_warm *W, int B, const float *targets) {
    using namespace gpe;
    const auto &c   = W->cfg;
    cudaStream_t s  = W->stream;
    const __nv_bfloat16 *wb = W->wb.p;
    const int nl    = (int)W->conv.size();
    const size_t N  = W->vox(nl - 1);
    const int lb    = 148 * 4;
    k_loss<<<lb, 256, 0, s>>>(W->pre[nl - 1].p, targets, W->gact[nl - 1].p, W->lpart.p, (size_t)B * N,
                              1.f / (float)((size_t)B * N));
    for (int l = nl - 1; l >= 0; --l) {
        const auto &L  = W->conv[l];
        const size_t n = W->vox(l) * L.cout;
        float *gy      = W->gact[l].p; // dL/d(pre-activation) after the line below
        if (l != nl - 1)
            k_silu_back<<<gpe::grid_for((size_t)B * n), 256, 0, s>>>(gy, W->pre[l].p, (size_t)B * n);
        const float *in  = l == 0 ? W->h2.p : W->act[l - 1].p;
        const size_t ins = l == 0 ? (size_t)W->latent : W->vox(l - 1) * W->conv[l - 1].cout;
        const int nchunks = (int)((W->vox(l) + kChunk - 1) / kChunk);
        k_conv_wgrad_partial<<<dim3(nchunks, L.cout, B), 256, 0, s>>>(in, gy, W->partial.p, L.g, ins, n, nchunks);
        const int nk = L.cin * 27 + 1;
        k_conv_wgrad_reduce<<<(L.cout * nk + 255) / 256, 256, 0, s>>>(W->partial.p, W->grad.p + L.w,
                                                                       W->grad.p + L.b, L.cout, L.cin,
                                                                       nchunks * B);
        float *dx = l == 0 ? W->gh2.p : W->gact[l - 1].p;
        const size_t ni = l == 0 ? (size_t)W->latent / L.cin : W->vox(l - 1);
        const size_t sm = sizeof(float) * L.cin * L.cout * 27;
        gpe::by_channels(L.cin, [&](auto CI) {
            k_conv_xgrad<decltype(CI)::value><<<dim3(gpe::grid_for(ni), B), 256, sm, s>>>(gy, wb + L.w, dx, L.g, n,
                                                                                       ni * L.cin);
        });
    }
    // dense 2 and dense 1
    k_silu_back<<<gpe::grid_for((size_t)B * W->latent), 256, 0, s>>>(W->gh2.p, W->h2pre.p, (size_t)B * W->latent);
    k_dense_wgrad<<<(int)(((size_t)W->latent * c.hidden + 255) / 256), 256, 0, s>>>(
        W->gh2.p, W->h1.p, W->grad.p + W->d2w, W->grad.p + W->d2b, B, c.hidden, W->latent);
    k_dense_xgrad<<<dim3((c.hidden + 127) / 128, B), 128, 0, s>>>(W->gh2.p, wb + W->d2w, W->gh1.p, B, c.hidden,
                                                                   W->latent);
    k_silu_back<<<gpe::grid_for((size_t)B * c.hidden), 256, 0, s>>>(W->gh1.p, W->h1pre.p, (size_t)B * c.hidden);
    k_dense_wgrad<<<(int)(((size_t)c.hidden * c.n_inputs + 255) / 256), 256, 0, s>>>(
        W->gh1.p, W->x.p, W->grad.p + W->d1w, W->grad.p + W->d1b, B, c.n_inputs, c.hidden);
    WS_CUDA(cudaGetLastError());
    std::vector<double> lp(lb);
    WS_CUDA(cudaMemcpyAsync(lp.data(), W->lpart.p, sizeof(double) * lb, cudaMemcpyDeviceToHost, s));
    WS_CUDA(cudaStreamSynchronize(s));
    double loss = 0.;
    for (double v : lp)
        loss += v;
    return loss / (double)((size_t)B * N);
}

void upload_inputs(gpe_warm *W, const float *params_host, int B) {
    WS_CUDA(cudaMemcpyAsync(W->x.p, params_host, sizeof(float) * B * W->cfg.n_inputs, cudaMemcpyHostToDevice,
                            W->stream));
}

} // namespace

extern "C" {

int gpe_warm_create(const gpe_warm_config *cfg, int device, gpe_warm **out) {
    if (!cfg || !out)
        return wbad("null argument");
    *out = nullptr;
    const auto &c = *cfg;
    if (c.levels < 0 || c.levels > 6 || c.hidden <= 0 || c.n_inputs <= 0 || c.max_batch <= 0)
        return wbad("bad network configuration");
    const int f = 1 << c.levels;
    if (c.nx % f || c.ny % f || c.nz % f)
        return wbad("grid sizes must be divisible by 2^levels");
    for (int s = 0; s <= c.levels; ++s)
        if (!gpe::channels_ok(c.channels[s]))
            return wbad("channels must be 1, 2, 4, 8, 16 or 32");
    return wguard([&] {
        auto W    = std::make_unique<gpe_warm>();
        W->cfg    = c;
        W->device = device;
        WS_CUDA(cudaSetDevice(device));
        WS_CUDA(cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking));
        const int X0 = c.nx / f, Y0 = c.ny / f, Z0 = c.nz / f;
        W->latent    = c.channels[0] * X0 * Y0 * Z0;
        size_t off   = 0;
        W->d1w = off, off += (size_t)c.hidden * c.n_inputs;
        W->d1b = off, off += c.hidden;
        W->d2w = off, off += (size_t)W->latent * c.hidden;
        W->d2b = off, off += W->latent;
        int X = X0, Y = Y0, Z = Z0;
        for (int s = 0; s <= c.levels; ++s) {
            gpe_warm::Layer L;
            L.cin  = c.channels[s];
            L.cout = s < c.levels ? c.channels[s + 1] : 1;
            const int up = s < c.levels;
            if (up)
                X *= 2, Y *= 2, Z *= 2;
            L.g = gpe::ConvGeom{L.cin, L.cout, X, Y, Z, up};
            L.w = off, off += (size_t)L.cout * L.cin * 27;
            L.b = off, off += L.cout;
            W->conv.push_back(L);
        }
        W->nweights = off;
        W->w.alloc(off);
        W->m.alloc(off);
        W->v.alloc(off);
        W->grad.alloc(off);
        W->wb.alloc(off);
        WS_CUDA(cudaMemset(W->w.p, 0, sizeof(float) * off));
        WS_CUDA(cudaMemset(W->m.p, 0, sizeof(float) * off));
        WS_CUDA(cudaMemset(W->v.p, 0, sizeof(float) * off));
        const int B = c.max_batch;
        W->x.alloc((size_t)B * c.n_inputs);
        W->h1pre.alloc((size_t)B * c.hidden);
        W->h1.alloc((size_t)B * c.hidden);
        W->gh1.alloc((size_t)B * c.hidden);
        W->h2pre.alloc((size_t)B * W->latent);
        W->h2.alloc((size_t)B * W->latent);
        W->gh2.alloc((size_t)B * W->latent);
        size_t maxpart = 0;
        W->pre.resize(W->conv.size());
        W->act.resize(W->conv.size());
        W->gact.resize(W->conv.size());
        for (size_t l = 0; l < W->conv.size(); ++l) {
            const size_t n = W->vox((int)l) * W->conv[l].cout * B;
            W->pre[l].alloc(n);
            W->act[l].alloc(n);
            W->gact[l].alloc(n);
            const size_t nch = (W->vox((int)l) + gpe::kChunk - 1) / gpe::kChunk;
            maxpart = std::max(maxpart, nch * B * W->conv[l].cout * (W->conv[l].cin * 27 + 1));
        }
        W->partial.alloc(maxpart);
        W->lpart.alloc(148 * 4);
        // weights staged in shared memory: up to 32 x 32 x 27 floats
        const int smax = (int)(sizeof(float) * gpe::kMaxCout * gpe::kMaxCout * 27);
        for (int ch : {1, 2, 4, 8, 16, 32})
            gpe::by_channels(ch, [&](auto C) {
                WS_CUDA(cudaFuncSetAttribute((const void *)gpe::k_conv_fwd<decltype(C)::value>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
                WS_CUDA(cudaFuncSetAttribute((const void *)gpe::k_conv_xgrad<decltype(C)::value>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
            });
        *out = W.release();
    });
}

int gpe_warm_destroy(gpe_warm *W) {
    if (!W)
        return GPE_OK;
    cudaSetDevice(W->device);
    cudaStreamSynchronize(W->stream);
    cudaStream_t s = W->stream;
    delete W;
    cudaStreamDestroy(s);
    return GPE_OK;
}

int gpe_warm_num_weights(gpe_warm *W, size_t *n) {
    if (!W || !n)
        return wbad("null argument");
    *n = W->nweights;
    return GPE_OK;
}

int gpe_warm_set_weights(gpe_warm *W, const float *host, size_t n) {
    if (!W || !host || n != W->nweights)
        return wbad("weight count mismatch");
    return wguard([&] {
        WS_CUDA(cudaSetDevice(W->device));
        WS_CUDA(cudaMemcpyAsync(W->w.p, host, sizeof(float) * n, cudaMemcpyHostToDevice, W->stream));
        gpe::k_to_bf16<<<gpe::grid_for(n), 256, 0, W->stream>>>(W->w.p, W->wb.p, n);
        WS_CUDA(cudaMemsetAsync(W->m.p, 0, sizeof(float) * n, W->stream));
        WS_CUDA(cudaMemsetAsync(W->v.p, 0, sizeof(float) * n, W->stream));
        WS_CUDA(cudaStreamSynchronize(W->stream));
        W->step = 0;
    });
}

int gpe_warm_get_weights(gpe_warm *W, float *host, size_t n) {
    if (!W || !host || n != W->nweights)
        return wbad("weight count mismatch");
    return wguard([&] {
        WS_CUDA(cudaSetDevice(W->device));
        WS_CUDA(cudaMemcpyAsync(host, W->w.p, sizeof(float) * n, cudaMemcpyDeviceToHost, W->stream));
        WS_CUDA(cudaStreamSynchronize(W->stream));
    });
}

int gpe_warm_init_weights(gpe_warm *W, unsigned long long seed) {
    if (!W)
        return wbad("null network");
    // He-style uniform initialisation scaled by fan-in, zero biases
    std::vector<float> h(W->nweights, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, size_t n, int fan_in) {
        const float a = std::sqrt(3.f / (float)fan_in);
        std::uniform_real_distribution<float> U(-a, a);
        for (size_t e = 0; e < n; ++e)
            h[off + e] = U(rng);
    };
    const auto &c = W->cfg;
    fill(W->d1w, (size_t)c.hidden * c.n_inputs, c.n_inputs);
    fill(W->d2w, (size_t)W->latent * c.hidden, c.hidden);
    for (const auto &L : W->conv)
        fill(L.w, (size_t)L.cout * L.cin * 27, L.cin * 27);
    return gpe_warm_set_weights(W, h.data(), h.size());
}

int gpe_warm_forward(gpe_warm *W, const float *params_host, int B, float *amp_dev) {
    if (!W || !params_host || !amp_dev || B <= 0 || B > W->cfg.max_batch)
        return wbad("bad forward arguments");
    return wguard([&] {
        WS_CUDA(cudaSetDevice(W->device));
        upload_inputs(W, params_host, B);
        forward(W, B);
        const int nl   = (int)W->conv.size();
        const size_t n = (size_t)B * W->vox(nl - 1);
        WS_CUDA(cudaMemcpyAsync(amp_dev, W->pre[nl - 1].p, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                W->stream));
        WS_CUDA(cudaStreamSynchronize(W->stream));
    });
}

int gpe_warm_gradients(gpe_warm *W, const float *params_host, const float *targets_dev, int B, float *grad_host,
                       double *loss) {
    if (!W || !params_host || !targets_dev || B <= 0 || B > W->cfg.max_batch)
        return wbad("bad gradient arguments");
    return wguard([&] {
        WS_CUDA(cudaSetDevice(W->device));
        upload_inputs(W, params_host, B);
        forward(W, B);
        const double l = backward(W, B, targets_dev);
        if (loss)
            *loss = l;
        if (grad_host) {
            WS_CUDA(cudaMemcpyAsync(grad_host, W->grad.p, sizeof(float) * W->nweights, cudaMemcpyDeviceToHost,
                                    W->stream));
            WS_CUDA(cudaStreamSynchronize(W->stream));
        }
    });
}

int gpe_warm_train_step(gpe_warm *W, const float *params_host, const float *targets_dev, int B, float lr,
                        double *loss) {
    if (!W || !params_host || !targets_dev || B <= 0 || B > W->cfg.max_batch || !(lr > 0))
        return wbad("bad training arguments");
    return wguard([&] {
        WS_CUDA(cudaSetDevice(W->device));
        upload_inputs(W, params_host, B);
        forward(W, B);
        const double l = backward(W, B, targets_dev);
        if (loss)
            *loss = l;
        ++W->step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)W->step), c2 = 1.f - std::pow(b2, (float)W->step);
        gpe::k_adam<<<gpe::grid_for(W->nweights), 256, 0, W->stream>>>(W->w.p, W->m.p, W->v.p, W->grad.p, W->wb.p,
                                                                        W->nweights, lr, b1, b2, 1e-8f, c1, c2);
        WS_CUDA(cudaGetLastError());
    });
}

} // extern "C"
