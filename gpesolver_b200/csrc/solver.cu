// gpe_b200: host runtime of the B200 GPE solver backend and its C ABI.
//
// One Solver<R> per handle owns the device fields, the FFT plans and tables, a
// CUDA stream and a cache of instantiated CUDA graphs (one per chunk of fused
// iterations).  All work is enqueued on the handle's stream; the host only
// waits where the reference's interface returns a value (norm, energies,
// exported fields).
#include "../../include/gpe_b200.h"
#include "fused_yz.cuh"
#include "plane_pair.cuh"
#include "init.cuh"
#include "kernels.cuh"
#include "plan.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace gpe {

// ---------------------------------------------------------------------------
// Non-template kernels
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_norm_finalize(const double *__restrict__ partial, int nparts, double dV,
                    double *__restrict__ norm_state, int *__restrict__ status) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int t = threadIdx.x; t < nparts; t += blockDim.x)
        acc += partial[t];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double x = red[0] * dV;
        norm_state[0]  = x;
        norm_state[1]  = x;
        if (!(x > 0.0) || !isfinite(x))
            status[0] = 1;
    }
}

__global__ void __launch_bounds__(256)
    k_energy_finalize(const double *__restrict__ partial, int nparts, double *__restrict__ out) {
    __shared__ double red[256];
    for (int t = 0; t < 5; ++t) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < nparts; b += blockDim.x)
            acc += partial[(size_t)t * nparts + b];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s)
                red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[t] = red[0];
        __syncthreads();
    }
}

__global__ void k_advance(int *counter, int by) { counter[0] += by; }

__global__ void k_set_f64(double *p, double v) { p[0] = v; }

// ---------------------------------------------------------------------------
// Error helpers
// ---------------------------------------------------------------------------
std::string &last_error() {
    static thread_local std::string msg;
    return msg;
}

#define GPE_CUDA(call)                                                                             \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw Error(e_ == cudaErrorMemoryAllocation ? GPE_ERR_NOMEM : GPE_ERR_CUDA,            \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

template <class T> struct DevBuf {
    T *p     = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        n = count;
        GPE_CUDA(cudaMalloc(&p, sizeof(T) * (count ? count : 1)));
        GPE_CUDA(cudaMemset(p, 0, sizeof(T) * (count ? count : 1)));
    }
    ~DevBuf() {
        if (p)
            cudaFree(p);
    }
};

// ---------------------------------------------------------------------------
// Solver interface (precision-erased)
// ---------------------------------------------------------------------------
class SolverBase {
  public:
    virtual ~SolverBase() = default;
    virtual void set_stream(cudaStream_t s)                  = 0;
    virtual cudaStream_t stream() const                      = 0;
    virtual void load_psi(const double *psi)                 = 0;
    virtual void import_psi(const double *psi)               = 0;
    virtual void load_potential(const double *V)             = 0;
    virtual void export_psi(double *out)                     = 0;
    virtual void export_fi3d(double *out)                    = 0;
    virtual void load_fi3d(const double *fi3d)               = 0;
    virtual void calc_fi3d()                                 = 0;
    virtual void imag_linear()                               = 0;
    virtual void imag_nonlinear()                            = 0;
    virtual double calc_norm(bool to_host)                   = 0;
    virtual void normalize()                                 = 0;
    virtual void potential_half_step()                       = 0;
    virtual void kinetic_step()                              = 0;
    virtual void energy(double *out6)                        = 0;
    virtual void set_coeffs(double ggp11, double gamma)      = 0;
    virtual void imag_steps(long k)                          = 0;
    virtual void imag_steps_energies(long k, int checks, double *e_total) = 0;
    virtual void real_steps(long k, long first_iter)         = 0;
    virtual long long launches() const                       = 0;
    virtual void time_kernel(int which, int reps, double *ms, double *bytes) = 0;
    virtual size_t n() const                                 = 0;
    // device-side initial state and potential (same semantics as load_psi /
    // load_potential of the host-computed arrays)
    virtual void init_potential(const PotCoef &c)            = 0;
    virtual void init_psi(const PsiCoef &c)                  = 0;
    virtual void export_potential(double *out)               = 0;
    virtual void export_amplitude_device(float *amp)         = 0;
    virtual void export_psi_async(double *host)              = 0;
    virtual void export_wait()                               = 0;
    virtual void load_amplitude_device(const float *amp)     = 0;
    // batched imaginary time (gpe_batch): the solver's fused IT graph pieces
    // captured as one branch of a batch graph
    virtual bool batchable() const                           = 0;
    virtual void it_batch_begin()                            = 0;
    virtual long long capture_it_branch(int kind, int count, cudaEvent_t fork, cudaStream_t root) = 0;
    virtual void it_batch_after(int kind, int count, long long nodes) = 0;
    virtual void it_batch_end()                              = 0;
    virtual const void *psi_ptr() const                      = 0;
    virtual void x_tiles(int *kin_lines, int *dip_lines) const  = 0;
    virtual const char *plane_kernel() const                 = 0;
    virtual int device() const                               = 0;
};

// update_edd (src/parameters/parameters.cpp:53-59), FP64, same expression order.
static void edd_at(const gpe_params &p, long iter, double *edd, double *ggp11, double *gamma) {
    const double e = p.edd_start + (p.edd_stop - p.edd_start) * (unsigned)iter /
                                       (double)(size_t)p.iter_real;
    const double a = p.add / e;
    *edd           = e;
    *ggp11         = 4 * M_PI * a / p.m;
    *gamma         = 128. * std::sqrt(M_PI) * std::pow(a, 2.5) / 3. / p.m * (1. + 1.5 * std::pow(e, 2));
}

template <class R>
__global__ void k_amplitude_out(const cplx<R> *__restrict__ psi, const double *__restrict__ divisor,
                                float *__restrict__ amp, size_t n) {
    const double sc = 1.0 / sqrt(divisor[0]);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const cplx<R> p = psi[e];
        amp[e]          = (float)(sqrt((double)p.x * p.x + (double)p.y * p.y) * sc);
    }
}

// psi_0 = max(amp, 0) on the interior, zero on the boundary cells (where the
// reference's initialisers leave it: imaginary time never updates the boundary,
// so a non-zero boundary would stay and hold norm)
__global__ void k_amplitude_in(const float *__restrict__ amp, double *__restrict__ psi_c128, int nx, int ny,
                               int nz) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % nz), j = (int)((e / nz) % ny), i = (int)(e / ((size_t)nz * ny));
        const bool in = i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
        psi_c128[2 * e]     = in ? fmax((double)amp[e], 0.0) : 0.0;
        psi_c128[2 * e + 1] = 0.0;
    }
}

template <class R> class Solver final : public SolverBase {
    using C = cplx<R>;

    // A planned line transform plus its launch tile.
    struct Line {
        LinePlan plan{};
        DevBuf<C> tw, twlo;
        int TB  = 1;
        int pad = 0; // z-pass tiles use the odd stride TB + 1
        size_t smem() const { return 2 * sizeof(C) * (size_t)(TB + pad) * plan.L; }
    };

  public:
    explicit Solver(const gpe_params &p) : P(p) {
        nx = p.nx;
        ny = p.ny;
        nz = p.nz;
        if (nx < 1 || ny < 1 || nz < 1)
            throw Error(GPE_ERR_ARG, "grid dimensions must be positive");
        if (!(p.dx > 0 && p.dy > 0 && p.dz > 0 && p.m > 0))
            throw Error(GPE_ERR_ARG, "grid spacings and mass must be positive");
        if ((long long)nx * ny * nz > (1LL << 30))
            throw Error(GPE_ERR_SIZE, "grid larger than 2^30 points");
        N = (size_t)nx * ny * nz;
        H = nz + 1;
        GPE_CUDA(cudaSetDevice(p.device));
        GPE_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        GPE_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        GPE_CUDA(cudaStreamCreateWithFlags(&cap_stream2, cudaStreamNonBlocking));
        GPE_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        GPE_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        cur = own_stream;

        plan_line(kz, nz, 16, 1);
        plan_line(ky, ny, 32, 0);
        plan_line(kx, nx, 32, 0);
        plan_line(dz, 2 * nz, 16, 1);
        plan_line(dy, 2 * ny, 32, 0);
        plan_line(dx, 2 * nx, 32, 0);

        psi.alloc(N);
        psii.alloc(N);
        bnd.alloc(N);
        V.alloc(N);
        phi.alloc(N);
        A.alloc((size_t)nx * 2 * ny * H);
        staging.alloc(2 * N);
        norm_state.alloc(4);
        status.alloc(4);
        iter_zero.alloc(1);
        iter_base.alloc(1);
        cur_coef.alloc(1);
        eout.alloc(8);

        nblk_elem = 148 * 8;
        partial.alloc(nblk_elem);
        epartial.alloc(5 * (size_t)nblk_elem);

        build_tables();
        fused = std::is_same<R, float>::value && p.schedule == 0 && fused_dim_xy(nx) &&
                fused_dim_xy(ny) && fused_dim_z(nz);
        if (fused) {
            S2.alloc((size_t)nx * 2 * ny * nz);
            psir.alloc(N);
            GPE_CUDA(cudaMemsetAsync(psir.p, 0, sizeof(C) * N, cur)); // defined before any RT call
            // per-CTA partial norms: one per 32 rows (four-kernel z pass), one per
            // CTA of a plane kernel (2 nx with two CTAs per plane)
            zpartial.alloc(std::max<size_t>((size_t)(nx * ny + 31) / 32, (size_t)2 * nx));
            ticket.alloc(1);
            build_vk2();
        }
        set_coeffs(p.ggp11, p.gamma);
        set_divisor_one();
        GPE_CUDA(cudaStreamSynchronize(cur));
        set_smem_attrs();
        if (fused) {
            set_fused_attrs();
            autotune_x();
        }
    }

    ~Solver() override {
        if (ev_copied) {
            cudaEventSynchronize(ev_copied);
            cudaEventDestroy(ev_copied);
            cudaEventDestroy(ev_widened);
            cudaStreamDestroy(copy_stream);
        }
        for (auto &kv : graphs)
            cudaGraphExecDestroy(kv.second);
        if (coef_host)
            cudaFreeHost(coef_host);
        if (coef_event)
            cudaEventDestroy(coef_event);
        cudaStreamSynchronize(cur);
        cudaEventDestroy(ev_fork);
        cudaEventDestroy(ev_join);
        cudaStreamDestroy(cap_stream2);
        cudaStreamDestroy(cap_stream);
        cudaStreamDestroy(own_stream);
    }

    void set_stream(cudaStream_t s) override { cur = s ? s : own_stream; }
    cudaStream_t stream() const override { return cur; }
    long long launches() const override { return n_launch; }
    size_t n() const override { return N; }

    // ---- data in / out ----------------------------------------------------
    void load_psi(const double *h) override {
        GPE_CUDA(cudaMemcpyAsync(staging.p, h, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, cur));
        load_psi_staged();
    }

    // load_buffer of the complex128 values in `staging`
    void load_psi_staged() {
        launch(k_from_f64<R>, grid_elem(2 * N), 256, 0, cur, (const double *)staging.p,
               reinterpret_cast<R *>(psi.p), 2 * N);
        GPE_CUDA(cudaMemcpyAsync(psii.p, psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(bnd.p, psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        // calc_norm + normalize: the normalisation is held as the lazy divisor.
        enqueue_norm(cur, psi.p, /*set_divisor=*/true);
        lazy = true;
        check_status();
    }

    void import_psi(const double *h) override {
        GPE_CUDA(cudaMemcpyAsync(staging.p, h, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, cur));
        launch(k_from_f64<R>, grid_elem(2 * N), 256, 0, cur, (const double *)staging.p,
               reinterpret_cast<R *>(psi.p), 2 * N);
        GPE_CUDA(cudaMemcpyAsync(psii.p, psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(bnd.p, psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        set_divisor_one();
        lazy = false;
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    void load_potential(const double *h) override {
        GPE_CUDA(cudaMemcpyAsync(staging.p, h, sizeof(double) * N, cudaMemcpyHostToDevice, cur));
        launch(k_from_f64<R>, grid_elem(N), 256, 0, cur, (const double *)staging.p, V.p, N);
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    InitGeom geom() const { return InitGeom{nx, ny, nz, P.dx, P.dy, P.dz}; }

    void init_potential(const PotCoef &c) override {
        launch(k_init_potential, grid_elem(N), 256, 0, cur, staging.p, geom(), c);
        launch(k_from_f64<R>, grid_elem(N), 256, 0, cur, (const double *)staging.p, V.p, N);
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    void init_psi(const PsiCoef &c) override {
        launch(k_init_psi, grid_elem(N), 256, 0, cur, staging.p, geom(), c);
        load_psi_staged();
    }

    // export_psi without waiting: psi is widened to complex128 on the device into
    // a buffer of its own (on the compute stream, before any later iteration),
    // then copied to `host` on a copy stream while the compute stream goes on.
    // `host` should be pinned for the copy to overlap.
    void export_psi_async(double *host) override {
        if (!export_buf.p) {
            export_buf.alloc(2 * N);
            GPE_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
            GPE_CUDA(cudaEventCreateWithFlags(&ev_widened, cudaEventDisableTiming));
            GPE_CUDA(cudaEventCreateWithFlags(&ev_copied, cudaEventDisableTiming));
        } else {
            GPE_CUDA(cudaEventSynchronize(ev_copied)); // the buffer of the previous export
        }
        launch(k_to_f64<R>, grid_elem(2 * N), 256, 0, cur, reinterpret_cast<const R *>(psi.p), export_buf.p,
               2 * N, (const double *)(norm_state.p + 1), 1);
        GPE_CUDA(cudaEventRecord(ev_widened, cur));
        GPE_CUDA(cudaStreamWaitEvent(copy_stream, ev_widened, 0));
        GPE_CUDA(cudaMemcpyAsync(host, export_buf.p, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, copy_stream));
        GPE_CUDA(cudaEventRecord(ev_copied, copy_stream));
    }
    void export_wait() override {
        if (export_buf.p)
            GPE_CUDA(cudaEventSynchronize(ev_copied));
    }

    // |psi| of the normalised psi, FP32, into a device buffer
    void export_amplitude_device(float *amp) override {
        launch(k_amplitude_out<R>, grid_elem(N), 256, 0, cur, (const C *)psi.p, (const double *)(norm_state.p + 1),
               amp, N);
        GPE_CUDA(cudaStreamSynchronize(cur));
    }
    // load_buffer of a real, non-negative amplitude (FP32, device), boundary zero
    void load_amplitude_device(const float *amp) override {
        launch(k_amplitude_in, grid_elem(N), 256, 0, cur, amp, staging.p, nx, ny, nz);
        load_psi_staged();
    }

    void export_potential(double *h) override {
        launch(k_to_f64<R>, grid_elem(N), 256, 0, cur, (const R *)V.p, staging.p, N,
               (const double *)one_ptr(), 1);
        GPE_CUDA(cudaMemcpyAsync(h, staging.p, sizeof(double) * N, cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    // ---- batched imaginary time ----------------------------------------------
    bool batchable() const override { return fused; }
    const void *psi_ptr() const override { return psi.p; }
    int device() const override { return P.device; }
    void it_batch_begin() override {
        if (!lazy)
            set_divisor_one();
        // members of a batch run side by side: fewer, larger CTAs of the dipolar
        // x pencils pay there (64-member sweep: 76.8 k against 75.7 k
        // member-iterations/s with the widths tuned for a solve alone)
        if (std::getenv("GPE_X_TILES") == nullptr)
            xd_lines = 16;
    }
    // Records this solver's fused IT graph piece (kind 20: prologue, 21: `count`
    // iterations, 23: the prologue and `count` iterations) on its capture stream
    // as a branch from `fork` that joins `root`.
    long long capture_it_branch(int kind, int count, cudaEvent_t fork, cudaStream_t root) override {
        const long long before = n_launch;
        GPE_CUDA(cudaStreamWaitEvent(cap_stream, fork, 0));
        if (kind == 23) {
            capture_fused(20, 0);
            capture_fused(21, count);
        } else {
            capture_fused(kind, count);
        }
        GPE_CUDA(cudaEventRecord(ev_join, cap_stream));
        GPE_CUDA(cudaStreamWaitEvent(root, ev_join, 0));
        const long long nodes = n_launch - before;
        n_launch              = before;
        return nodes;
    }
    void it_batch_after(int kind, int count, long long nodes) override {
        n_launch += nodes;
        if ((kind == 21 || kind == 23) && (count & 1))
            std::swap(psi.p, psii.p);
    }
    void it_batch_end() override {
        lazy = true;
        check_status();
    }

    void export_psi(double *h) override {
        launch(k_to_f64<R>, grid_elem(2 * N), 256, 0, cur, reinterpret_cast<const R *>(psi.p),
               staging.p, 2 * N, (const double *)(norm_state.p + 1), 1);
        GPE_CUDA(cudaMemcpyAsync(h, staging.p, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    void export_fi3d(double *h) override {
        launch(k_to_f64<R>, grid_elem(N), 256, 0, cur, (const R *)phi.p, staging.p, N,
               (const double *)one_ptr(), 1);
        GPE_CUDA(cudaMemcpyAsync(h, staging.p, sizeof(double) * N, cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    void load_fi3d(const double *h) override {
        GPE_CUDA(cudaMemcpyAsync(staging.p, h, sizeof(double) * N, cudaMemcpyHostToDevice, cur));
        launch(k_from_f64<R>, grid_elem(N), 256, 0, cur, (const double *)staging.p, phi.p, N);
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    // ---- the reference's virtuals ------------------------------------------
    void calc_fi3d() override { enqueue_dipolar(cur, psi.p); }

    void imag_linear() override { enqueue_it_update(cur, psi.p, psii.p); }

    void imag_nonlinear() override {
        std::swap(psi.p, psii.p);
        set_divisor_one();
        lazy = false;
    }

    // Reference semantics: no error on a zero or non-finite norm here (the
    // reference's initialize() normalises the still-zero psi); the fused paths
    // and load_psi report them.
    double calc_norm(bool to_host) override {
        materialize();
        enqueue_norm(cur, psi.p, /*set_divisor=*/false);
        set_divisor_one();
        if (!to_host)
            return 0.0;
        double x = 0;
        GPE_CUDA(cudaMemcpyAsync(&x, norm_state.p, sizeof(double), cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
        return x;
    }

    void normalize() override {
        // psi /= sqrt(xnorma): held lazily as the divisor norm_state[1] = xnorma.
        GPE_CUDA(cudaMemcpyAsync(norm_state.p + 1, norm_state.p, sizeof(double),
                                 cudaMemcpyDeviceToDevice, cur));
        lazy = true;
    }

    void potential_half_step() override {
        materialize();
        enqueue_phase(cur, cur_coef.p, iter_zero.p, 0);
    }

    void kinetic_step() override {
        materialize();
        enqueue_kinetic(cur);
    }

    void energy(double *out) override {
        const int nb = nblk_elem;
        launch(k_energy_partial<R>, nb, 256, 0, cur, (const C *)psi.p, (const R *)V.p,
               (const R *)phi.p, (const double *)(norm_state.p + 1), 1, epartial.p, nx, ny, nz,
               1.0 / (P.dx * P.dx), 1.0 / (P.dy * P.dy), 1.0 / (P.dz * P.dz), ggp11_cur, P.cdd,
               P.n_atoms, gamma_cur);
        launch(k_energy_finalize, 1, 256, 0, cur, (const double *)epartial.p, nb, eout.p);
        double e[5];
        GPE_CUDA(cudaMemcpyAsync(e, eout.p, sizeof(e), cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
        // Post-scaling of CpuGrossPitaevskiSolver::calc_energy (cpu_solver.cpp:185-191).
        const double dV = P.dx * P.dy * P.dz, w = P.n_atoms;
        out[0]          = e[0] * (dV / (2 * P.m) * w);
        out[1]          = e[1] * (dV * w);
        out[2]          = e[2] * (dV * std::pow(w, 2));
        out[3]          = e[3] * dV;
        out[4]          = e[4] * (dV * std::pow(w, 2.5));
        out[5]          = out[0] + out[1] + out[2] + out[3] + out[4];
        for (int t = 0; t < 6; ++t)
            if (!std::isfinite(out[t]))
                throw Error(GPE_ERR_NUMERIC, "non-finite energy");
    }

    // `checks` times: k imaginary-time iterations, then the total energy into a
    // device history; one host synchronisation at the end.
    void imag_steps_energies(long k, int checks, double *e_total) override {
        if (k <= 0 || checks <= 0)
            throw Error(GPE_ERR_ARG, "iterations and checks must be positive");
        if (ehist.n < (size_t)5 * checks)
            ehist.alloc((size_t)5 * checks);
        const int nb = nblk_elem;
        for (int c = 0; c < checks; ++c) {
            if (!lazy)
                set_divisor_one();
            if (fused) {
                // the energy kernels between checks only read psi: one prologue
                fused_imag(k, c == 0);
            } else {
                long done = 0;
                while (k - done >= kItChunk) {
                    run_graph(0, kItChunk);
                    done += kItChunk;
                }
                if (k - done > 0)
                    run_graph(0, (int)(k - done));
            }
            lazy = true;
            launch(k_energy_partial<R>, nb, 256, 0, cur, (const C *)psi.p, (const R *)V.p, (const R *)phi.p,
                   (const double *)(norm_state.p + 1), 1, epartial.p, nx, ny, nz, 1.0 / (P.dx * P.dx),
                   1.0 / (P.dy * P.dy), 1.0 / (P.dz * P.dz), ggp11_cur, P.cdd, P.n_atoms, gamma_cur);
            launch(k_energy_finalize, 1, 256, 0, cur, (const double *)epartial.p, nb, ehist.p + 5 * c);
        }
        std::vector<double> e((size_t)5 * checks);
        GPE_CUDA(cudaMemcpyAsync(e.data(), ehist.p, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, cur));
        check_status();
        const double dV = P.dx * P.dy * P.dz, w = P.n_atoms;
        for (int c = 0; c < checks; ++c) {
            const double *x = &e[(size_t)5 * c];
            e_total[c] = x[0] * (dV / (2 * P.m) * w) + x[1] * (dV * w) + x[2] * (dV * std::pow(w, 2)) + x[3] * dV +
                         x[4] * (dV * std::pow(w, 2.5));
            if (!std::isfinite(e_total[c]))
                throw Error(GPE_ERR_NUMERIC, "non-finite energy");
        }
    }

    void set_coeffs(double ggp11, double gamma) override {
        ggp11_cur = ggp11;
        gamma_cur = gamma;
        StepCoef c{(ggp11 - P.cdd / 3) * P.n_atoms, gamma * P.w_15};
        host_coef = c;
        GPE_CUDA(cudaMemcpyAsync(cur_coef.p, &host_coef, sizeof(StepCoef), cudaMemcpyHostToDevice, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
    }

    // ---- fused iterations ---------------------------------------------------
    void imag_steps(long k) override {
        if (k <= 0)
            return;
        if (!lazy)
            set_divisor_one();
        if (fused) {
            fused_imag(k);
            lazy = true;
            check_status();
            return;
        }
        const int CH = kItChunk;
        long done    = 0;
        while (k - done >= CH) {
            run_graph(0, CH);
            done += CH;
        }
        if (k - done > 0)
            run_graph(0, (int)(k - done));
        lazy = true;
        check_status();
    }

    void real_steps(long k, long first_iter) override {
        if (k <= 0)
            return;
        materialize();
        // Per-iteration coefficients (update_edd when ramping), FP64 on the host.
        ensure_coef_capacity(k);
        if (coef_event)
            GPE_CUDA(cudaEventSynchronize(coef_event));
        for (long t = 0; t < k; ++t) {
            double g = ggp11_cur, gm = gamma_cur;
            if (!P.const_edd) {
                double e;
                edd_at(P, first_iter + t, &e, &g, &gm);
            }
            coef_host[t] = StepCoef{(g - P.cdd / 3) * P.n_atoms, gm * P.w_15};
            if (t == k - 1 && !P.const_edd)
                set_coeffs(g, gm);
        }
        GPE_CUDA(cudaMemcpyAsync(coef_dev.p, coef_host, sizeof(StepCoef) * k, cudaMemcpyHostToDevice, cur));
        GPE_CUDA(cudaEventRecord(coef_event, cur));
        GPE_CUDA(cudaMemsetAsync(iter_base.p, 0, sizeof(int), cur));
        if (fused) {
            fused_real(k);
            check_status();
            return;
        }
        const int CH = kRtChunk;
        long done    = 0;
        while (k - done >= CH) {
            run_graph(1, CH);
            done += CH;
        }
        if (k - done > 0)
            run_graph(1, (int)(k - done));
        check_status();
    }

    void time_kernel(int which, int reps, double *ms, double *bytes) override {
        if (which < 0 || which >= GPE_K_COUNT || reps < 1)
            throw Error(GPE_ERR_ARG, "bad kernel id or repetition count");
        materialize();
        // save the state the kernels modify
        DevBuf<C> save_psi, save_A, save_S2;
        DevBuf<R> save_phi;
        save_psi.alloc(N);
        save_A.alloc(A.n);
        save_phi.alloc(N);
        GPE_CUDA(cudaMemcpyAsync(save_psi.p, psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(save_A.p, A.p, sizeof(C) * A.n, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(save_phi.p, phi.p, sizeof(R) * N, cudaMemcpyDeviceToDevice, cur));
        if (fused) {
            save_S2.alloc(S2.n);
            GPE_CUDA(cudaMemcpyAsync(save_S2.p, S2.p, sizeof(C) * S2.n, cudaMemcpyDeviceToDevice, cur));
        }
        if (which == GPE_K_F_Z || which == GPE_K_F_YZ) {
            // the merged phase reads the coefficients of two consecutive iterations
            ensure_coef_capacity(2);
            GPE_CUDA(cudaEventSynchronize(coef_event));
            coef_host[0] = coef_host[1] = host_coef;
            GPE_CUDA(cudaMemcpyAsync(coef_dev.p, coef_host, 2 * sizeof(StepCoef), cudaMemcpyHostToDevice, cur));
            GPE_CUDA(cudaEventRecord(coef_event, cur));
            GPE_CUDA(cudaMemsetAsync(iter_base.p, 0, sizeof(int), cur));
        }
        cudaEvent_t e0, e1;
        GPE_CUDA(cudaEventCreate(&e0));
        GPE_CUDA(cudaEventCreate(&e1));
        const double F = (double)sizeof(C) * N, Rb = (double)sizeof(R) * N;
        const double I = (double)sizeof(C) * nx * 2 * ny * H, half = (double)sizeof(C) * nx * ny * H;
        double b = 0;
        auto one = [&]() {
            const int lines = nx * ny;
            switch (which) {
            case GPE_K_DIP_Z_FWD:
                launch(k_dip_z_fwd<R>, (lines + dz.TB - 1) / dz.TB, 256, dz.smem(), cur, (const C *)psi.p,
                       (const double *)(norm_state.p + 1), 1, A.p, nx, ny, nz, (R)P.n_atoms, dz.plan, dz.TB);
                b = F + half;
                break;
            case GPE_K_DIP_Y_FWD:
                launch(k_dip_y<-1, R>, dim3((H + dy.TB - 1) / dy.TB, nx), 256, dy.smem(), cur, A.p, ny, H,
                       ny, 2 * ny, dy.plan, dy.TB);
                b = half + I;
                break;
            case GPE_K_DIP_X:
                launch(k_dip_x<R>, (2 * ny * H + dx.TB - 1) / dx.TB, 256, dx.smem(), cur, A.p,
                       (const R *)vk.p, nx, ny, H, (R)1, dx.plan, dx.TB);
                b = 2 * I;
                break;
            case GPE_K_DIP_Y_INV:
                launch(k_dip_y<+1, R>, dim3((H + dy.TB - 1) / dy.TB, nx), 256, dy.smem(), cur, A.p, ny, H,
                       2 * ny, ny, dy.plan, dy.TB);
                b = I + half;
                break;
            case GPE_K_DIP_Z_INV:
                launch(k_dip_z_inv<R>, (lines + dz.TB - 1) / dz.TB, 256, dz.smem(), cur, (const C *)A.p, phi.p,
                       nx, ny, nz, (R)(1.0 / (8.0 * (double)N)), dz.plan, dz.TB);
                b = half + Rb;
                break;
            case GPE_K_KIN_Z_FWD:
            case GPE_K_KIN_Z_INV:
                if (which == GPE_K_KIN_Z_FWD)
                    launch(k_kin_z<-1, R>, (lines + kz.TB - 1) / kz.TB, 256, kz.smem(), cur, psi.p, lines, nz,
                           kz.plan, kz.TB);
                else
                    launch(k_kin_z<+1, R>, (lines + kz.TB - 1) / kz.TB, 256, kz.smem(), cur, psi.p, lines, nz,
                           kz.plan, kz.TB);
                b = 2 * F;
                break;
            case GPE_K_KIN_Y_FWD:
            case GPE_K_KIN_Y_INV:
                if (which == GPE_K_KIN_Y_FWD)
                    launch(k_kin_y<-1, R>, dim3((nz + ky.TB - 1) / ky.TB, nx), 256, ky.smem(), cur, psi.p, ny,
                           nz, ky.plan, ky.TB);
                else
                    launch(k_kin_y<+1, R>, dim3((nz + ky.TB - 1) / ky.TB, nx), 256, ky.smem(), cur, psi.p, ny,
                           nz, ky.plan, ky.TB);
                b = 2 * F;
                break;
            case GPE_K_KIN_X:
                launch(k_kin_x<R>, (ny * nz + kx.TB - 1) / kx.TB, 256, kx.smem(), cur, psi.p,
                       (const C *)ex.p, (const C *)ey.p, (const C *)ez.p, inv_hi, inv_lo, nx, ny, nz, kx.plan, kx.TB);
                b = 2 * F;
                break;
            case GPE_K_PHASE:
                enqueue_phase(cur, cur_coef.p, iter_zero.p, 0);
                b = 2 * F + 2 * Rb;
                break;
            case GPE_K_F_X:
            case GPE_K_F_YINV:
            case GPE_K_F_Z:
            case GPE_K_F_YFWD:
            case GPE_K_F_XK:
            case GPE_K_F_XD:
            case GPE_K_F_YZ: {
                if (!fused)
                    throw Error(GPE_ERR_STATE, "the fused pipeline is not available for this grid");
                if (which == GPE_K_F_YZ && !yz_plane())
                    throw Error(GPE_ERR_STATE, "no yz plane kernel for this grid");
                const double S2b = (double)sizeof(C) * nx * 2 * ny * nz;
                const double S2h = (double)sizeof(C) * nx * ny * nz;
                if (which == GPE_K_F_XK) {
                    f_x(cur, true, nullptr, 1);
                    b = 2 * F; // psi spectrum in and out
                } else if (which == GPE_K_F_XD) {
                    f_x(cur, false, nullptr);
                    b = 2 * S2h + (double)sizeof(R) * (nx + 1) * (ny + 1) * nz; // + the V_dd table
                } else if (which == GPE_K_F_YZ) {
                    f_yz<ZM_RT_MID>(cur, psi.p, psi.p, coef_dev.p, 0);
                    // kinetic increment R+W, real-space psi R+W, spectrum (2ny
                    // rows) R+W, V read (phi is written only by the last
                    // iteration of a call)
                    b = 4 * F + 2 * S2b + Rb;
                } else if (which == GPE_K_F_X) {
                    f_x(cur, true, nullptr);
                    b = 2 * F + 2 * S2h; // kinetic R+W; dipolar reads and writes nx of 2nx planes
                } else if (which == GPE_K_F_YINV) {
                    f_y<+1>(cur, true);
                    b = 2 * F + S2b + S2h;
                } else if (which == GPE_K_F_YFWD) {
                    f_y<-1>(cur, true);
                    b = 2 * F + S2h + S2b;
                } else {
                    f_z<ZM_RT_MID>(cur, psi.p, psi.p, coef_dev.p, 0);
                    // increment R+W, real-space psi R+W, spectrum R+W, V read, phi write
                    b = 4 * F + 2 * S2h + Rb + Rb;
                }
                break;
            }
            default:
                enqueue_it_update(cur, psi.p, psii.p);
                b = 2 * F + 2 * Rb;
                break;
            }
        };
        one(); // warm-up
        GPE_CUDA(cudaEventRecord(e0, cur));
        for (int r = 0; r < reps; ++r)
            one();
        GPE_CUDA(cudaEventRecord(e1, cur));
        GPE_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        GPE_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        GPE_CUDA(cudaMemcpyAsync(psi.p, save_psi.p, sizeof(C) * N, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(A.p, save_A.p, sizeof(C) * A.n, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaMemcpyAsync(phi.p, save_phi.p, sizeof(R) * N, cudaMemcpyDeviceToDevice, cur));
        if (fused)
            GPE_CUDA(cudaMemcpyAsync(S2.p, save_S2.p, sizeof(C) * S2.n, cudaMemcpyDeviceToDevice, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
        *ms    = (double)t / reps;
        *bytes = b;
    }

  private:
    // ---- fused pipeline ---------------------------------------------------
    static bool fused_dim_xy(int n) { return n == 32 || n == 64 || n == 96 || n == 128 || n == 256; }
    static bool fused_dim_z(int n) { return n == 8 || n == 16 || n == 24 || n == 32 || n == 64; }

    // V_dd(k) for kz = 1..nz (the kz = 0 plane is identically zero), reduced by
    // |kx|, |ky| symmetry, FP64 as fftw_poisson_solver.cpp:12-49.
    void build_vk2() {
        const int px = 2 * nx, py = 2 * ny, pz = 2 * nz;
        const double dkx = 2. * M_PI / (px * P.dx), dky = 2. * M_PI / (py * P.dy),
                     dkz = 2. * M_PI / (pz * P.dz);
        std::vector<R> t((size_t)(nx + 1) * (ny + 1) * nz);
        for (int i = 0; i <= nx; ++i) {
            const double kxv = i * dkx;
            for (int j = 0; j <= ny; ++j) {
                const double kyv = j * dky;
                for (int k = 1; k <= nz; ++k) {
                    const double kzv = k * dkz;
                    const double k2  = kxv * kxv + kyv * kyv + kzv * kzv;
                    t[((size_t)i * (ny + 1) + j) * nz + (k - 1)] = (R)((k2 > 1e-30) ? (kzv * kzv / k2) : 0.0);
                }
            }
        }
        vk2.alloc(t.size());
        GPE_CUDA(cudaMemcpy(vk2.p, t.data(), sizeof(R) * t.size(), cudaMemcpyHostToDevice));
    }

    static Twid twid(const Line &l) { return Twid{l.plan.tw, l.plan.twlo}; }

#define GPE_XY_CASES(M) M(32) M(64) M(96) M(128) M(256)
#define GPE_Z_CASES(M) M(8) M(16) M(24) M(32) M(64)
#define GPE_YZ_CASES(M) M(32, 16) M(64, 16) M(64, 32) M(96, 24) M(128, 32)

    void set_fused_attrs() {
        if constexpr (std::is_same<R, float>::value) {
            auto set = [](const void *f, size_t bytes) {
                if (bytes > 48 * 1024)
                    GPE_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
            };
#define GPE_SETX(N)                                                                                \
    if (nx == N) {                                                                                 \
        set_x_attrs<N, 8>(set);                                                                    \
        set_x_attrs<N, 16>(set);                                                                   \
    }
#define GPE_SETY1(N, CNT, SIGN)                                                                    \
    {                                                                                              \
        using Y = YShape<R, N, CNT>;                                                               \
        set((const void *)k3_y_kin<R, N, SIGN, CNT, Y::NTK>, Y::SK);                               \
        set((const void *)k3_y_dip<R, N, SIGN, CNT, Y::NTD>, Y::SD);                               \
    }
#define GPE_SETY(N)                                                                                \
    if (ny == N) {                                                                                 \
        GPE_SETY1(N, 8, -1) GPE_SETY1(N, 8, +1) GPE_SETY1(N, 16, -1) GPE_SETY1(N, 16, +1)          \
    }
#define GPE_SETZ(N)                                                                                \
    if (nz == N) {                                                                                 \
        set((const void *)k2_z<R, N, ZM_RT_PRO>, z_smem<R, N>());                                   \
        set((const void *)k2_z<R, N, ZM_RT_MID>, z_smem<R, N>());                                   \
        set((const void *)k2_z<R, N, ZM_RT_EPI>, z_smem<R, N>());                                   \
        set((const void *)k2_z<R, N, ZM_IT_PRO>, z_smem<R, N>());                                   \
        set((const void *)k2_z<R, N, ZM_IT_MID>, z_smem<R, N>());                                   \
    }
#define GPE_SETYZ(A, B)                                                                            \
    if (ny == A && nz == B) {                                                                      \
        using G = YZShape<R, A, B>;                                                                \
        set((const void *)k4_yz<R, A, B, ZM_RT_PRO>, G::template smem<ZM_RT_PRO>());               \
        set((const void *)k4_yz<R, A, B, ZM_RT_MID>, G::template smem<ZM_RT_MID>());               \
        set((const void *)k4_yz<R, A, B, ZM_RT_EPI>, G::template smem<ZM_RT_EPI>());               \
        set((const void *)k4_yz<R, A, B, ZM_IT_PRO>, G::template smem<ZM_IT_PRO>());               \
        set((const void *)k4_yz<R, A, B, ZM_IT_MID>, G::template smem<ZM_IT_MID>());               \
        set((const void *)k4_yz<R, A, B, ZM_IT_MID, false>, G::template smem<ZM_IT_MID>());        \
        set((const void *)k5_yz_pair<R, A, B>, PairShape<R, A, B>::SMEM);                          \
        set((const void *)k5_yz_pair_it<R, A, B>, PairShapeIT<R, A, B>::SMEM);                     \
    }
            GPE_YZ_CASES(GPE_SETYZ)
#undef GPE_SETYZ
            GPE_XY_CASES(GPE_SETX)
            GPE_XY_CASES(GPE_SETY)
            GPE_Z_CASES(GPE_SETZ)
#undef GPE_SETX
#undef GPE_SETY1
#undef GPE_SETY
#undef GPE_SETZ
        }
    }

    // part: 0 both, 1 kinetic only, 2 dipolar only
    // X pass: kinetic pencils (kin, part 0 or 1) and dipolar pencils (part 0, or !kin).
    // x-pass launches for nx = NN with CNT lines per CTA (the autotuned choice)
    template <int NN, int CNT, class Set> static void set_x_attrs(Set &set) {
        set((const void *)k3_x_kin<R, NN, CNT, pass_threads<NN, CNT>()>, xy_smem<R, NN, CNT>());
        set((const void *)k3_x_dip<R, NN, CNT, pass_threads<2 * NN, CNT>()>, x_dip_smem<R, NN, CNT>());
    }
    template <int NN, int CNT> void launch_xk(cudaStream_t s) {
        constexpr int NT = pass_threads<NN, CNT>();
        launch(k3_x_kin<R, NN, CNT, NT>, (ny * nz + CNT - 1) / CNT, NT, xy_smem<R, NN, CNT>(), s, psi.p,
               (const C *)ex.p, (const C *)ey.p, (const C *)ez.p, inv_hi, inv_lo, ny, nz, twid(kx));
    }
    template <int NN, int CNT> void launch_xd(cudaStream_t s, const double *divisor, double dscale) {
        constexpr int NT = pass_threads<2 * NN, CNT>();
        launch(k3_x_dip<R, NN, CNT, NT>, (2 * ny * nz + CNT - 1) / CNT, NT, x_dip_smem<R, NN, CNT>(), s, S2.p,
               (const R *)vk2.p, divisor, dscale, ny, nz, twid(dx));
    }
    template <int NN> void f_x_n(cudaStream_t s, bool kin, const double *divisor, int part, double dscale) {
        if (kin) {
            if (xk_lines == 8)
                launch_xk<NN, 8>(s);
            else
                launch_xk<NN, 16>(s);
        }
        if (!kin || part == 0) {
            if (xd_lines == 8)
                launch_xd<NN, 8>(s, divisor, dscale);
            else
                launch_xd<NN, 16>(s, divisor, dscale);
        }
    }
    void f_x(cudaStream_t s, bool kin, const double *divisor, int part = 0) {
        if constexpr (std::is_same<R, float>::value) {
            const double dscale = 1.0 / (8.0 * (double)N);
#define GPE_LX(NN)                                                                                 \
    if (nx == NN)                                                                                  \
        f_x_n<NN>(s, kin, divisor, part, dscale);
            GPE_XY_CASES(GPE_LX)
#undef GPE_LX
        }
    }

    // Autotuner of the pencil passes: lines per CTA (8 or 16) of the kinetic
    // and of the dipolar x pencils, and (four-kernel schedule, nz >= 16) z
    // columns per CTA of the y lines, each timed alone (CUDA events around each
    // of 20 launches after one warm-up, on zeroed buffers) when the first
    // solver of a grid is created on a device; later solvers of that grid and
    // device reuse the choice.  GPE_X_TILES="k,d" and GPE_Y_LINES=c (values 8 or
    // 16) fix them.
    void autotune_x() {
        y_lines = nz >= 16 ? 16 : 8;
        bool fix_x = false, fix_y = false, fix_p = false;
        if (const char *env = std::getenv("GPE_PLANE_PAIR")) {
            if (env[0] == '0' || env[0] == '1') {
                pair_rt = pair_it = yz_plane() && env[0] == '1';
                fix_p             = true;
            }
        }
        // GPE_IT_WIDE=0|1 fixes the one-CTA imaginary-time kernel's block
        bool fix_w = false;
        if (const char *env = std::getenv("GPE_IT_WIDE")) {
            if (env[0] == '0' || env[0] == '1') {
                it_wide = env[0] == '1';
                fix_w   = true;
            }
        }
        const bool tune_p = yz_plane() && !fix_p;
        if (const char *env = std::getenv("GPE_X_TILES")) {
            int k = 0, d = 0;
            if (std::sscanf(env, "%d,%d", &k, &d) == 2 && (k == 8 || k == 16) && (d == 8 || d == 16)) {
                xk_lines = k;
                xd_lines = d;
                fix_x    = true;
            }
        }
        if (const char *env = std::getenv("GPE_Y_LINES")) {
            const int c = std::atoi(env);
            if ((c == 8 || c == 16) && c <= nz) {
                y_lines = c;
                fix_y   = true;
            }
        }
        const bool tune_y = !fix_y && !yz_plane() && nz >= 16;
        if (fix_x && !tune_y && !tune_p)
            return;
        static std::mutex mu;
        // keyed by the schedule too: the plane schedule never tunes y_lines, so a
        // four-kernel solver of the same grid must not reuse its untuned value
        static std::map<std::tuple<int, int, int, int, bool>, std::tuple<int, int, int, int>> chosen;
        // the plane decomposition alone, measured also by solvers whose x widths
        // are fixed: every solver of a grid then runs the same plane kernels (the
        // one-CTA and two-CTA real-time kernels agree to rounding, not to the bit)
        static std::map<std::tuple<int, int, int, int>, int> chosen_p;
        const auto key  = std::make_tuple(P.device, nx, ny, nz, yz_plane());
        const auto keyp = std::make_tuple(P.device, nx, ny, nz);
        std::lock_guard<std::mutex> lock(mu);
        const auto it = chosen.find(key);
        if (it != chosen.end()) {
            if (!fix_x) {
                xk_lines = std::get<0>(it->second);
                xd_lines = std::get<1>(it->second);
            }
            if (tune_y)
                y_lines = std::get<2>(it->second);
            if (tune_p) {
                pair_rt = (std::get<3>(it->second) & 1) != 0;
                pair_it = (std::get<3>(it->second) & 2) != 0;
                if (!fix_w)
                    it_wide = (std::get<3>(it->second) & 4) == 0;
            }
            return;
        }
        bool measure_p = tune_p;
        if (tune_p) {
            const auto ip = chosen_p.find(keyp);
            if (ip != chosen_p.end()) {
                pair_rt   = (ip->second & 1) != 0;
                pair_it   = (ip->second & 2) != 0;
                if (!fix_w)
                    it_wide = (ip->second & 4) == 0;
                measure_p = false;
                if (fix_x && !tune_y)
                    return;
            }
        }
        GPE_CUDA(cudaMemsetAsync(psi.p, 0, sizeof(C) * N, cur));
        GPE_CUDA(cudaMemsetAsync(S2.p, 0, sizeof(C) * S2.n, cur));
        cudaEvent_t e0, e1;
        GPE_CUDA(cudaEventCreate(&e0));
        GPE_CUDA(cudaEventCreate(&e1));
        // Grids whose fields (~40 bytes a point: psi, the kept psi, the dipolar
        // spectrum, V, phi) outgrow half the L2 run their passes from DRAM: time
        // those candidates with the L2 flushed before every launch, the others
        // L2-resident, as the pipeline runs them.
        int l2 = 0;
        GPE_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, P.device));
        const bool cold = 40.0 * (double)N > 0.5 * (double)l2;
        DevBuf<unsigned char> flush;
        if (cold)
            flush.alloc(2 * (size_t)l2);
        auto time_of = [&](auto &&run) {
            run();
            float total = 0.f;
            for (int r = 0; r < 20; ++r) {
                if (cold)
                    GPE_CUDA(cudaMemsetAsync(flush.p, r, flush.n, cur));
                GPE_CUDA(cudaEventRecord(e0, cur));
                run();
                GPE_CUDA(cudaEventRecord(e1, cur));
                GPE_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                GPE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                total += ms;
            }
            return total;
        };
        int best_k = xk_lines, best_d = xd_lines, best_y = y_lines;
        if (!fix_x) {
            // each width timed twice, alternated, the faster time of each kept;
            // 8 lines replace 16 only when 3% faster: choices within the
            // timing noise stay at the default and do not flip run to run
            float tk[2] = {0.f, 0.f}, td[2] = {0.f, 0.f}; // [16 lines, 8 lines]
            for (int rep = 0; rep < 2; ++rep) {
                for (int v = 0; v < 2; ++v) {
                    xk_lines = xd_lines = v == 0 ? 16 : 8;
                    const float a = time_of([&] { f_x(cur, true, nullptr, 1); });
                    const float b = time_of([&] { f_x(cur, false, nullptr, 1); });
                    tk[v]         = rep == 0 ? a : std::min(tk[v], a);
                    td[v]         = rep == 0 ? b : std::min(td[v], b);
                }
            }
            best_k = tk[1] < 0.97f * tk[0] ? 8 : 16;
            best_d = td[1] < 0.97f * td[0] ? 8 : 16;
        }
        if (tune_y) {
            float ty = 0.f;
            for (int c : {16, 8}) {
                y_lines       = c;
                const float a = time_of([&] {
                    f_y<+1>(cur, true);
                    f_y<-1>(cur, true);
                });
                if (c == 16 || a < 0.97f * ty) {
                    ty     = a;
                    best_y = c;
                }
            }
        }
        if (measure_p) {
            // the plane kernel of the middle iterations: one CTA per x plane
            // (k4_yz) or a two-CTA cluster per plane (k5_yz_pair[_it]), each
            // timed on the zeroed fields with a zero coefficient table; the
            // imaginary-time launches leave a zero norm behind, which is reset
            DevBuf<StepCoef> tcoef;
            tcoef.alloc(2);
            GPE_CUDA(cudaMemsetAsync(tcoef.p, 0, sizeof(StepCoef) * 2, cur));
            GPE_CUDA(cudaMemsetAsync(iter_base.p, 0, sizeof(int), cur));
            // the one-CTA imaginary-time kernel's block: twice the real-time
            // count or the real-time count (narrow only when 1% faster: the two
            // agree to 1e-9, and the gap where the narrow block wins is ~2.5%)
            pair_rt = pair_it = false;
            if (!fix_w) {
                // alternated twice, the faster of each pair kept: the candidates
                // are a few per cent apart, within a drift of the clocks
                float tw_ = 0.f, tn_ = 0.f;
                for (int rep = 0; rep < 2; ++rep) {
                    it_wide        = true;
                    const float a_ = time_of([&] { f_yz<ZM_IT_MID>(cur, psi.p, psii.p, tcoef.p, 0); });
                    it_wide        = false;
                    const float b_ = time_of([&] { f_yz<ZM_IT_MID>(cur, psi.p, psii.p, tcoef.p, 0); });
                    tw_            = rep == 0 ? a_ : std::min(tw_, a_);
                    tn_            = rep == 0 ? b_ : std::min(tn_, b_);
                }
                it_wide = !(tn_ < 0.99f * tw_);
            }
            float trt[2], tit[2]; // twice, alternated, the faster time of each kept
            for (int rep = 0; rep < 2; ++rep) {
                for (int v = 0; v < 2; ++v) {
                    pair_rt = pair_it = v == 1;
                    const float a = time_of([&] { f_yz<ZM_RT_MID>(cur, psi.p, psi.p, tcoef.p, 0); });
                    const float b = time_of([&] { f_yz<ZM_IT_MID>(cur, psi.p, psii.p, tcoef.p, 0); });
                    trt[v]        = rep == 0 ? a : std::min(trt[v], a);
                    tit[v]        = rep == 0 ? b : std::min(tit[v], b);
                }
            }
            GPE_CUDA(cudaStreamSynchronize(cur));
            // the pair replaces the one-CTA kernel only when 3% faster
            pair_rt = trt[1] < 0.97f * trt[0];
            pair_it = tit[1] < 0.97f * tit[0];
            // The imaginary-time launches divide by the zero norm they leave
            // behind, so the fields they wrote hold NaN: clear every field the
            // tuning touched, the norm state and the status, as at creation.
            GPE_CUDA(cudaMemsetAsync(psi.p, 0, sizeof(C) * N, cur));
            GPE_CUDA(cudaMemsetAsync(psii.p, 0, sizeof(C) * N, cur));
            GPE_CUDA(cudaMemsetAsync(psir.p, 0, sizeof(C) * N, cur));
            GPE_CUDA(cudaMemsetAsync(S2.p, 0, sizeof(C) * S2.n, cur));
            GPE_CUDA(cudaMemsetAsync(phi.p, 0, sizeof(R) * N, cur));
            GPE_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int) * 4, cur));
            GPE_CUDA(cudaMemcpyAsync(norm_state.p, one_buf.p, sizeof(double), cudaMemcpyDeviceToDevice, cur));
            set_divisor_one();
            GPE_CUDA(cudaStreamSynchronize(cur));
            if (!fix_w) // only measured choices are shared
                chosen_p[keyp] = (pair_rt ? 1 : 0) | (pair_it ? 2 : 0) | (it_wide ? 0 : 4);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        xk_lines = best_k;
        xd_lines = best_d;
        y_lines  = best_y;
        if (!fix_x && !fix_y && !fix_p && !fix_w) // only measured choices are shared
            chosen[key] = std::make_tuple(best_k, best_d, best_y,
                                          (pair_rt ? 1 : 0) | (pair_it ? 2 : 0) | (it_wide ? 0 : 4));
    }
    void x_tiles(int *k, int *d) const override {
        *k = xk_lines;
        *d = xd_lines;
    }
    const char *plane_kernel() const override { return pair_rt ? "k5_yz_pair" : (yz_plane() ? "k4_yz" : ""); }

    // Y pass (SIGN < 0 forward, > 0 inverse): kinetic lines (kin, part 0 or 1)
    // and dipolar lines (part 0, or !kin).  Tiles of 16 z columns (8 when nz = 8).
    template <int SIGN> void f_y(cudaStream_t s, bool kin, int part = 0) {
        if constexpr (std::is_same<R, float>::value) {
            if (y_lines == 16)
                f_y_cnt<SIGN, 16>(s, kin, part);
            else
                f_y_cnt<SIGN, 8>(s, kin, part);
        }
    }
    template <int SIGN, int CNT> void f_y_cnt(cudaStream_t s, bool kin, int part) {
        const dim3 grid((nz + CNT - 1) / CNT, nx);
#define GPE_LY(NN)                                                                                 \
    if (ny == NN) {                                                                                \
        using Y = YShape<R, NN, CNT>;                                                              \
        if (kin)                                                                                   \
            launch(k3_y_kin<R, NN, SIGN, CNT, Y::NTK>, grid, Y::NTK, Y::SK, s, psi.p, nz, twid(ky)); \
        if (!kin || part == 0)                                                                     \
            launch(k3_y_dip<R, NN, SIGN, CNT, Y::NTD>, grid, Y::NTD, Y::SD, s, S2.p, nz, twid(dy));  \
    }
        GPE_XY_CASES(GPE_LY)
#undef GPE_LY
    }

    ZArgs zargs(C *pin, C *pout, const StepCoef *coef, int local) {
        ZArgs a{};
        a.psi_in     = pin;
        a.psi_out    = pout;
        a.psi_r      = psir.p;
        a.bnd        = bnd.p;
        a.S          = S2.p;
        a.V          = V.p;
        a.phi        = phi.p;
        a.norm_state = norm_state.p;
        a.partial    = zpartial.p;
        a.ticket     = ticket.p;
        a.status     = status.p;
        a.dV         = P.dx * P.dy * P.dz;
        a.step       = StepIdx{coef, iter_base.p, local};
        a.half_dt    = P.real_time_dt / 2.;
        a.cdd        = P.cdd;
        a.w_atoms    = P.n_atoms;
        a.cx         = -0.5 / (P.m * P.dx * P.dx);
        a.cy         = 0.5 / (P.m * P.dy * P.dy);
        a.cz         = 0.5 / (P.m * P.dz * P.dz);
        a.dtau       = P.imag_time_dt;
        a.nx         = nx;
        a.ny         = ny;
        return a;
    }

    template <int MODE> void f_z(cudaStream_t s, C *pin, C *pout, const StepCoef *coef, int local) {
        if constexpr (std::is_same<R, float>::value) {
            const ZArgs a  = zargs(pin, pout, coef, local);
            const int grid = (nx * ny + 31) / 32;
#define GPE_LZ(NN)                                                                                 \
    if (nz == NN)                                                                                  \
        launch(k2_z<R, NN, MODE>, grid, 256, z_smem<R, NN>(), s, a, twid(kz), twid(dz));
            GPE_Z_CASES(GPE_LZ)
#undef GPE_LZ
        }
    }

    // The y passes and the z rows of one iteration as one kernel per x plane
    // (grids whose ny x nz planes fit in shared memory).
    bool yz_plane() const {
        bool ok = false;
#define GPE_YZOK(A, B) ok = ok || (ny == A && nz == B);
        GPE_YZ_CASES(GPE_YZOK)
#undef GPE_YZOK
        return fused && ok;
    }
    template <int MODE> void f_yz(cudaStream_t s, C *pin, C *pout, const StepCoef *coef, int local) {
        if constexpr (std::is_same<R, float>::value) {
            const ZArgs a = zargs(pin, pout, coef, local);
            const YZTwid t{twid(ky), twid(kz), twid(dy), twid(dz)};
#define GPE_LYZ(A, B)                                                                              \
    if (ny == A && nz == B) {                                                                      \
        using G = YZShape<R, A, B>;                                                                \
        if (MODE == ZM_RT_MID && pair_rt)                                                          \
            launch(k5_yz_pair<R, A, B>, 2 * nx, PairShape<R, A, B>::NT, PairShape<R, A, B>::SMEM,  \
                   s, a, t);                                                                       \
        else if (MODE == ZM_IT_MID && pair_it)                                                     \
            launch(k5_yz_pair_it<R, A, B>, 2 * nx, PairShape<R, A, B>::NT,                         \
                   PairShapeIT<R, A, B>::SMEM, s, a, t);                                           \
        else if (MODE == ZM_IT_MID && !it_wide)                                                    \
            launch(k4_yz<R, A, B, ZM_IT_MID, false>, nx, G::template nt<ZM_IT_MID, false>(),       \
                   G::template smem<ZM_IT_MID>(), s, a, t);                                        \
        else                                                                                       \
            launch(k4_yz<R, A, B, MODE>, nx, G::template nt<MODE>(), G::template smem<MODE>(), s, a, t); \
    }
            GPE_YZ_CASES(GPE_LYZ)
#undef GPE_LYZ
        }
    }

    // kind 10: RT prologue; 11: C mid RT iterations; 12: `count` mid + the last;
    // kind 20: IT prologue; 21: `count` IT iterations.
    void capture_fused(int kind, int count) {
        if (yz_plane()) {
            capture_fused_yz(kind, count);
            return;
        }
        cudaStream_t s = cap_stream;
        if (kind == 10) {
            f_z<ZM_RT_PRO>(s, psi.p, psi.p, coef_dev.p, 0);
            f_y<-1>(s, true);
        } else if (kind == 11 || kind == 12) {
            // the kinetic (s) and dipolar (s2) chains are independent until the Z
            // kernel; they run as two branches of the graph
            cudaStream_t s2 = cap_stream2;
            for (int t = 0; t <= count; ++t) {
                if (t == count && kind == 11)
                    break;
                GPE_CUDA(cudaEventRecord(ev_fork, s));
                GPE_CUDA(cudaStreamWaitEvent(s2, ev_fork, 0));
                f_x(s, true, nullptr, 1);
                f_x(s2, false, nullptr);
                f_y<+1>(s, true, 1);
                f_y<+1>(s2, false);
                GPE_CUDA(cudaEventRecord(ev_join, s2));
                GPE_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
                if (t == count) {
                    f_z<ZM_RT_EPI>(s, psi.p, psi.p, coef_dev.p, count);
                    break;
                }
                f_z<ZM_RT_MID>(s, psi.p, psi.p, coef_dev.p, t);
                GPE_CUDA(cudaEventRecord(ev_fork, s));
                GPE_CUDA(cudaStreamWaitEvent(s2, ev_fork, 0));
                f_y<-1>(s, true, 1);
                f_y<-1>(s2, false);
                GPE_CUDA(cudaEventRecord(ev_join, s2));
                GPE_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
            }
            if (kind == 12) {
            } else {
                launch(k_advance, 1, 1, 0, s, iter_base.p, count);
            }
        } else if (kind == 20) {
            f_z<ZM_IT_PRO>(s, psi.p, psi.p, cur_coef.p, 0);
            f_y<-1>(s, false);
        } else {
            C *a = psi.p, *b = psii.p;
            for (int t = 0; t < count; ++t) {
                f_x(s, false, norm_state.p + 1);
                f_y<+1>(s, false);
                f_z<ZM_IT_MID>(s, a, b, cur_coef.p, 0);
                f_y<-1>(s, false);
                std::swap(a, b);
            }
        }
    }

    // Two kernels per iteration: x pass (kinetic and dipolar pencils as two graph
    // branches in real time), then the yz plane kernel.
    void capture_fused_yz(int kind, int count) {
        cudaStream_t s = cap_stream;
        if (kind == 10) {
            f_yz<ZM_RT_PRO>(s, psi.p, psi.p, coef_dev.p, 0);
        } else if (kind == 11 || kind == 12) {
            cudaStream_t s2 = cap_stream2;
            for (int t = 0; t <= count; ++t) {
                if (t == count && kind == 11)
                    break;
                GPE_CUDA(cudaEventRecord(ev_fork, s));
                GPE_CUDA(cudaStreamWaitEvent(s2, ev_fork, 0));
                f_x(s, true, nullptr, 1);
                f_x(s2, false, nullptr);
                GPE_CUDA(cudaEventRecord(ev_join, s2));
                GPE_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
                if (t == count) {
                    f_yz<ZM_RT_EPI>(s, psi.p, psi.p, coef_dev.p, count);
                    break;
                }
                f_yz<ZM_RT_MID>(s, psi.p, psi.p, coef_dev.p, t);
            }
            if (kind == 11)
                launch(k_advance, 1, 1, 0, s, iter_base.p, count);
        } else if (kind == 20) {
            f_yz<ZM_IT_PRO>(s, psi.p, psi.p, cur_coef.p, 0);
        } else {
            C *a = psi.p, *b = psii.p;
            for (int t = 0; t < count; ++t) {
                f_x(s, false, norm_state.p + 1);
                f_yz<ZM_IT_MID>(s, a, b, cur_coef.p, 0);
                std::swap(a, b);
            }
        }
    }

    void run_fused_graph(int kind, int count) {
        auto key = std::make_tuple(kind, count, (const void *)psi.p);
        auto it  = graphs.find(key);
        if (it == graphs.end()) {
            const long long before = n_launch;
            GPE_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
            try {
                capture_fused(kind, count);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(cap_stream, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g;
            GPE_CUDA(cudaStreamEndCapture(cap_stream, &g));
            cudaGraphExec_t ge;
            GPE_CUDA(cudaGraphInstantiate(&ge, g, 0));
            cudaGraphDestroy(g);
            graphs[key]      = ge;
            graph_nodes[key] = (int)(n_launch - before);
            n_launch         = before;
            it               = graphs.find(key);
        }
        GPE_CUDA(cudaGraphLaunch(it->second, cur));
        n_launch += graph_nodes[key];
        if (kind == 21 && (count & 1))
            std::swap(psi.p, psii.p);
    }

    void fused_real(long k) {
        run_fused_graph(10, 0);
        const long mid = k - 1;
        const int CH   = kRtChunk;
        long done      = 0;
        while (mid - done >= CH) {
            run_fused_graph(11, CH);
            done += CH;
        }
        run_fused_graph(12, (int)(mid - done));
    }

    // prologue = false: the dipolar spectrum is already that of the stored psi
    // (the previous call ended with an IT iteration and nothing has written psi
    // since); the prologue would recompute it bit for bit.
    void fused_imag(long k, bool prologue = true) {
        if (prologue)
            run_fused_graph(20, 0);
        const int CH = kItChunk;
        long done    = 0;
        while (k - done >= CH) {
            run_fused_graph(21, CH);
            done += CH;
        }
        if (k - done > 0)
            run_fused_graph(21, (int)(k - done));
    }

    static constexpr int kItChunk = 64;
    static constexpr int kRtChunk = 32;

    gpe_params P;
    int nx, ny, nz, H;
    size_t N;
    Line kz, ky, kx, dz, dy, dx;
    DevBuf<C> psi, psii, bnd, A, ex, ey, ez;
    DevBuf<R> V, phi, vk;
    DevBuf<double> staging, norm_state, partial, epartial, eout;
    DevBuf<double> export_buf; // asynchronous exports
    DevBuf<double> ehist;      // energy history of imag_steps_energies
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_widened = nullptr, ev_copied = nullptr;
    DevBuf<int> status, iter_zero, iter_base;
    // fused pipeline (compile-time line lengths; complex64 only)
    bool fused = false;
    // middle real- / imaginary-time iterations on the two-CTA plane kernels
    // (k5_yz_pair, k5_yz_pair_it) instead of k4_yz: picked by autotune_x
    bool pair_rt = false, pair_it = false;
    // imaginary-time k4_yz with twice the real-time block (at most 1024
    // threads) or the real-time block: picked by autotune_x
    bool it_wide = true;
    DevBuf<C> S2;
    DevBuf<C> psir; // real time: psi in real space after the last phase step
    int xk_lines = 16, xd_lines = 16; // x-pass lines per CTA (autotune_x)
    int y_lines = 16;                 // y-pass z columns per CTA (four-kernel schedule; autotune_x)
    DevBuf<R> vk2;
    DevBuf<double> zpartial;
    DevBuf<unsigned> ticket;
    DevBuf<StepCoef> cur_coef, coef_dev;
    StepCoef host_coef{};
    StepCoef *coef_host   = nullptr;
    size_t coef_cap       = 0;
    cudaEvent_t coef_event = nullptr;
    DevBuf<double> one_buf;
    cudaStream_t own_stream = nullptr, cap_stream = nullptr, cap_stream2 = nullptr, cur = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::map<std::tuple<int, int, const void *>, cudaGraphExec_t> graphs;
    std::map<std::tuple<int, int, const void *>, int> graph_nodes;
    int nblk_elem = 0;
    R inv_hi = 0, inv_lo = 0;
    bool lazy     = false;
    double ggp11_cur = 0, gamma_cur = 0;
    long long n_launch = 0;

    int grid_elem(size_t n) const {
        size_t b = (n + 255) / 256;
        return (int)std::min<size_t>(b, (size_t)nblk_elem);
    }

    template <class K, class... Args>
    void launch(K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
        kernel<<<grid, block, smem, s>>>(args...);
        GPE_CUDA(cudaGetLastError());
        ++n_launch;
    }

    void plan_line(Line &ln, int L, int tbmax, int pad) {
        std::vector<int> r = factor_line(L);
        ln.plan.L          = L;
        ln.plan.nstages    = (int)r.size();
        ln.pad             = pad;
        for (size_t s = 0; s < r.size(); ++s)
            ln.plan.radix[s] = r[s];
        std::vector<double> t = twiddles(L);
        std::vector<C> tc(L), tl(L);
        for (int m = 0; m < L; ++m) {
            tc[m] = C{(R)t[2 * m], (R)t[2 * m + 1]};
            tl[m] = C{(R)(t[2 * m] - (double)tc[m].x), (R)(t[2 * m + 1] - (double)tc[m].y)};
        }
        ln.tw.alloc(L);
        ln.twlo.alloc(L);
        GPE_CUDA(cudaMemcpy(ln.tw.p, tc.data(), sizeof(C) * L, cudaMemcpyHostToDevice));
        GPE_CUDA(cudaMemcpy(ln.twlo.p, tl.data(), sizeof(C) * L, cudaMemcpyHostToDevice));
        ln.plan.tw   = ln.tw.p;
        ln.plan.twlo = ln.twlo.p;
        // Tile: two Stockham buffers of TB lines within a 64 KiB budget per CTA.
        const size_t budget = 64 * 1024;
        int TB              = tbmax;
        while (TB > 1 && 2 * sizeof(C) * (size_t)(TB + pad) * L > budget)
            TB >>= 1;
        if (2 * sizeof(C) * (size_t)(TB + pad) * L > 200 * 1024)
            throw Error(GPE_ERR_SIZE, "FFT line of length " + std::to_string(L) + " too long");
        ln.TB = TB;
    }

    void set_smem_attrs() {
        auto set = [](const void *f, size_t bytes) {
            if (bytes > 48 * 1024)
                GPE_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        };
        set((const void *)k_dip_z_fwd<R>, dz.smem());
        set((const void *)k_dip_y<-1, R>, dy.smem());
        set((const void *)k_dip_y<+1, R>, dy.smem());
        set((const void *)k_dip_x<R>, dx.smem());
        set((const void *)k_dip_z_inv<R>, dz.smem());
        set((const void *)k_kin_z<-1, R>, kz.smem());
        set((const void *)k_kin_z<+1, R>, kz.smem());
        set((const void *)k_kin_y<-1, R>, ky.smem());
        set((const void *)k_kin_y<+1, R>, ky.smem());
        set((const void *)k_kin_x<R>, kx.smem());
    }

    // FP64 tables: V_dd(k) (fftw_poisson_solver.cpp:12-49) reduced by |kx|,|ky|
    // symmetry, and the separable kinetic phase (fftw_split_solver.cpp:11-42).
    void build_tables() {
        {
            const int px = 2 * nx, py = 2 * ny, pz = 2 * nz;
            const double dkx = 2. * M_PI / (px * P.dx);
            const double dky = 2. * M_PI / (py * P.dy);
            const double dkz = 2. * M_PI / (pz * P.dz);
            std::vector<R> t((size_t)(nx + 1) * (ny + 1) * H);
            for (int i = 0; i <= nx; ++i) {
                const double kxv = (i <= (px / 2)) ? i * dkx : (i - px) * dkx;
                for (int j = 0; j <= ny; ++j) {
                    const double kyv = (j <= (py / 2)) ? j * dky : (j - py) * dky;
                    for (int k = 0; k < H; ++k) {
                        const double kzv = (k <= (pz / 2)) ? k * dkz : (k - pz) * dkz;
                        const double k2  = kxv * kxv + kyv * kyv + kzv * kzv;
                        const double v   = (k2 > 1e-30) ? (kzv * kzv / k2) : 0.0;
                        t[((size_t)i * (ny + 1) + j) * H + k] = (R)v;
                    }
                }
            }
            vk.alloc(t.size());
            GPE_CUDA(cudaMemcpy(vk.p, t.data(), sizeof(R) * t.size(), cudaMemcpyHostToDevice));
        }
        {
            // Per-axis exp(i theta) - 1 with theta = -dt/(2m) k^2 (k as in
            // fftw_split_solver.cpp:26-31), in FP64; the kernel combines the three
            // axes and applies the factor as v + v*w.
            const double dt = P.real_time_dt, fac = -dt / (2.0 * P.m);
            auto axis = [&](int n, double d, DevBuf<C> &out) {
                std::vector<C> t(n);
                for (int i = 0; i < n; ++i) {
                    const double kv = (i <= n / 2) ? (2.0 * M_PI * i / (n * d))
                                                   : (2.0 * M_PI * (i - n) / (n * d));
                    const double f  = fac * (kv * kv);
                    const double sh = std::sin(0.5 * f);
                    t[i]            = C{(R)(-2.0 * sh * sh), (R)std::sin(f)};
                }
                out.alloc(n);
                GPE_CUDA(cudaMemcpy(out.p, t.data(), sizeof(C) * n, cudaMemcpyHostToDevice));
            };
            axis(nx, P.dx, ex);
            axis(ny, P.dy, ey);
            axis(nz, P.dz, ez);
            const double inv = 1.0 / (double)N;
            inv_hi           = (R)inv;
            inv_lo           = (R)(inv - (double)inv_hi);
        }
        one_buf.alloc(1);
        const double one = 1.0;
        GPE_CUDA(cudaMemcpy(one_buf.p, &one, sizeof(double), cudaMemcpyHostToDevice));
    }

    const double *one_ptr() const { return one_buf.p; }

    void set_divisor_one() {
        GPE_CUDA(cudaMemcpyAsync(norm_state.p + 1, one_buf.p, sizeof(double), cudaMemcpyDeviceToDevice, cur));
    }

    void materialize() {
        if (!lazy)
            return;
        launch(k_scale<R>, grid_elem(N), 256, 0, cur, psi.p, N, (const double *)(norm_state.p + 1));
        set_divisor_one();
        lazy = false;
    }

    // status[0]: a non-finite or non-positive norm; status[1]: a bulk copy into
    // shared memory that a plane kernel stopped waiting for
    void check_status() {
        int st[2] = {0, 0};
        GPE_CUDA(cudaMemcpyAsync(st, status.p, sizeof(st), cudaMemcpyDeviceToHost, cur));
        GPE_CUDA(cudaStreamSynchronize(cur));
        if (st[0] != 0 || st[1] != 0) {
            GPE_CUDA(cudaMemset(status.p, 0, sizeof(st)));
            if (st[1] != 0)
                throw Error(GPE_ERR_CUDA, "a plane kernel's bulk copy into shared memory did not complete");
            throw Error(GPE_ERR_NUMERIC, "non-finite or non-positive norm of psi");
        }
    }

    void ensure_coef_capacity(long k) {
        if ((size_t)k <= coef_cap)
            return;
        if (coef_event)
            GPE_CUDA(cudaEventSynchronize(coef_event));
        if (coef_host)
            cudaFreeHost(coef_host);
        size_t cap = std::max<size_t>((size_t)k, 1024);
        GPE_CUDA(cudaMallocHost(&coef_host, sizeof(StepCoef) * cap));
        coef_dev.~DevBuf();
        new (&coef_dev) DevBuf<StepCoef>();
        coef_dev.alloc(cap);
        coef_cap = cap;
        if (!coef_event)
            GPE_CUDA(cudaEventCreateWithFlags(&coef_event, cudaEventDisableTiming));
        // cached real-time graphs (split schedule: kind 1; fused: kinds 10-12)
        // hold the address of the old coefficient buffer
        for (auto it = graphs.begin(); it != graphs.end();) {
            const int kind = std::get<0>(it->first);
            if (kind == 1 || (kind >= 10 && kind <= 12)) {
                cudaGraphExecDestroy(it->second);
                graph_nodes.erase(it->first);
                it = graphs.erase(it);
            } else {
                ++it;
            }
        }
    }

    // ---- enqueue helpers (usable while capturing) ---------------------------
    void enqueue_norm(cudaStream_t s, const C *p, bool set_divisor) {
        launch(k_norm_partial<R>, nblk_elem, 256, 0, s, p, N, partial.p);
        launch(k_norm_finalize, 1, 256, 0, s, (const double *)partial.p, nblk_elem,
               P.dx * P.dy * P.dz, norm_state.p, status.p);
        if (!set_divisor)
            return;
    }

    void enqueue_dipolar(cudaStream_t s, const C *p) {
        const int lines = nx * ny;
        launch(k_dip_z_fwd<R>, (lines + dz.TB - 1) / dz.TB, 256, dz.smem(), s, p,
               (const double *)(norm_state.p + 1), 1, A.p, nx, ny, nz, (R)P.n_atoms, dz.plan, dz.TB);
        launch(k_dip_y<-1, R>, dim3((H + dy.TB - 1) / dy.TB, nx), 256, dy.smem(), s, A.p, ny, H, ny,
               2 * ny, dy.plan, dy.TB);
        const int cols = 2 * ny * H;
        launch(k_dip_x<R>, (cols + dx.TB - 1) / dx.TB, 256, dx.smem(), s, A.p, (const R *)vk.p, nx,
               ny, H, (R)1, dx.plan, dx.TB);
        launch(k_dip_y<+1, R>, dim3((H + dy.TB - 1) / dy.TB, nx), 256, dy.smem(), s, A.p, ny, H,
               2 * ny, ny, dy.plan, dy.TB);
        const R inv_n = (R)(1.0 / (8.0 * (double)N));
        launch(k_dip_z_inv<R>, (lines + dz.TB - 1) / dz.TB, 256, dz.smem(), s, (const C *)A.p, phi.p,
               nx, ny, nz, inv_n, dz.plan, dz.TB);
    }

    void enqueue_kinetic(cudaStream_t s) {
        const int lines = nx * ny;
        launch(k_kin_z<-1, R>, (lines + kz.TB - 1) / kz.TB, 256, kz.smem(), s, psi.p, lines, nz,
               kz.plan, kz.TB);
        launch(k_kin_y<-1, R>, dim3((nz + ky.TB - 1) / ky.TB, nx), 256, ky.smem(), s, psi.p, ny, nz,
               ky.plan, ky.TB);
        const int cols = ny * nz;
        launch(k_kin_x<R>, (cols + kx.TB - 1) / kx.TB, 256, kx.smem(), s, psi.p, (const C *)ex.p,
               (const C *)ey.p, (const C *)ez.p, inv_hi, inv_lo, nx, ny, nz, kx.plan, kx.TB);
        launch(k_kin_y<+1, R>, dim3((nz + ky.TB - 1) / ky.TB, nx), 256, ky.smem(), s, psi.p, ny, nz,
               ky.plan, ky.TB);
        launch(k_kin_z<+1, R>, (lines + kz.TB - 1) / kz.TB, 256, kz.smem(), s, psi.p, lines, nz,
               kz.plan, kz.TB);
    }

    void enqueue_phase(cudaStream_t s, const StepCoef *coef, const int *base, int local) {
        launch(k_phase<R>, grid_elem(N), 256, 0, s, psi.p, (const R *)V.p, (const R *)phi.p, coef,
               base, local, nx, ny, nz, (R)(P.real_time_dt / 2.), (R)P.cdd);
    }

    void enqueue_it_update(cudaStream_t s, const C *in, C *out) {
        const double m = P.m;
        launch(k_it_update<R>, nblk_elem, 256, 0, s, in, out, (const C *)bnd.p, (const R *)V.p,
               (const R *)phi.p, (const double *)(norm_state.p + 1), (const StepCoef *)cur_coef.p,
               partial.p, nx, ny, nz, (R)(-0.5 / (m * P.dx * P.dx)), (R)(0.5 / (m * P.dy * P.dy)),
               (R)(0.5 / (m * P.dz * P.dz)), (R)P.imag_time_dt, (R)P.cdd);
    }

    // One fused imaginary-time iteration from psi `in` into `out`:
    // calc_fi3d -> Euler update -> calc_norm (normalize held as the divisor).
    void enqueue_it_step(cudaStream_t s, const C *in, C *out) {
        enqueue_dipolar(s, in);
        enqueue_it_update(s, in, out);
        launch(k_norm_finalize, 1, 256, 0, s, (const double *)partial.p, nblk_elem,
               P.dx * P.dy * P.dz, norm_state.p, status.p);
    }

    // One fused real-time iteration (real_time_iter) on psi in place.
    void enqueue_rt_step(cudaStream_t s, int local) {
        enqueue_phase(s, coef_dev.p, iter_base.p, local);
        enqueue_dipolar(s, psi.p);
        enqueue_kinetic(s);
        enqueue_phase(s, coef_dev.p, iter_base.p, local);
    }

    // kind 0: `count` IT iterations; kind 1: `count` RT iterations.
    void run_graph(int kind, int count) {
        auto key = std::make_tuple(kind, count, (const void *)psi.p);
        auto it  = graphs.find(key);
        if (it == graphs.end()) {
            const long long before = n_launch;
            GPE_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
            try {
                if (kind == 0) {
                    C *a = psi.p, *b = psii.p;
                    for (int t = 0; t < count; ++t) {
                        enqueue_it_step(cap_stream, a, b);
                        std::swap(a, b);
                    }
                } else {
                    for (int t = 0; t < count; ++t)
                        enqueue_rt_step(cap_stream, t);
                    launch(k_advance, 1, 1, 0, cap_stream, iter_base.p, count);
                }
            } catch (...) {
                cudaGraph_t g;
                cudaStreamEndCapture(cap_stream, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g;
            GPE_CUDA(cudaStreamEndCapture(cap_stream, &g));
            cudaGraphExec_t ge;
            GPE_CUDA(cudaGraphInstantiate(&ge, g, 0));
            cudaGraphDestroy(g);
            graphs[key]      = ge;
            graph_nodes[key] = (int)(n_launch - before);
            n_launch         = before;
            it               = graphs.find(key);
        }
        GPE_CUDA(cudaGraphLaunch(it->second, cur));
        n_launch += graph_nodes[key];
        if (kind == 0 && (count & 1))
            std::swap(psi.p, psii.p);
    }
};

} // namespace gpe

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct gpe_handle {
    std::unique_ptr<gpe::SolverBase> impl;
    int device = 0;
    gpe_params params{};
};

namespace {

template <class F> int guarded(F &&f) {
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

int bad(const char *msg) {
    gpe::last_error() = msg;
    return GPE_ERR_ARG;
}

#define GPE_HANDLE(h)                                                                              \
    if (!(h) || !(h)->impl)                                                                        \
        return bad("null handle");                                                                 \
    if (cudaSetDevice((h)->device) != cudaSuccess)                                                 \
        return bad("cudaSetDevice failed");

} // namespace

extern "C" {

const char *gpe_last_error(void) { return gpe::last_error().c_str(); }
int gpe_abi_version(void) { return GPE_B200_ABI_VERSION; }

int gpe_params_derive(gpe_params *p) {
    if (!p)
        return bad("null params");
    if (!(p->m > 0) || !(p->edd > 0))
        return bad("mass and edd must be positive");
    // PhysicalParameters::init_parameters (src/parameters/parameters.cpp:37-51).
    p->add          = 131.;
    p->cdd          = 12. * M_PI * p->add / p->m;
    const double a  = p->add / p->edd;
    p->ggp11        = 4. * M_PI * a / p->m;
    p->gamma        = 128. * std::sqrt(M_PI) * std::pow(a, 2.5) / 3. / p->m * (1. + 1.5 * std::pow(p->edd, 2));
    p->w_15         = std::pow(p->n_atoms, 1.5);
    p->real_time_dt = 1.00e10;
    p->imag_time_dt = 1.25e11;
    return GPE_OK;
}

int gpe_params_edd_at(const gpe_params *p, long iter, double *out3) {
    if (!p || !out3)
        return bad("null argument");
    if (p->iter_real <= 0)
        return bad("iter_real must be positive for an edd ramp");
    gpe::edd_at(*p, iter, &out3[0], &out3[1], &out3[2]);
    return GPE_OK;
}

int gpe_create(const gpe_params *p, gpe_handle **out) {
    if (!p || !out)
        return bad("null argument");
    *out = nullptr;
    if (p->precision != GPE_PREC_C64 && p->precision != GPE_PREC_C128)
        return bad("unknown precision");
    if (!p->const_edd && p->iter_real <= 0)
        return bad("iter_real must be positive when edd is ramped");
    return guarded([&] {
        auto h    = std::make_unique<gpe_handle>();
        h->device = p->device;
        h->params = *p;
        if (p->precision == GPE_PREC_C64)
            h->impl.reset(new gpe::Solver<float>(*p));
        else
            h->impl.reset(new gpe::Solver<double>(*p));
        *out = h.release();
    });
}

} // extern "C"

using gpe::Error; // for GPE_CUDA outside namespace gpe

struct gpe_batch {
    std::vector<gpe_handle *> members;
    int device          = 0;
    cudaStream_t own    = nullptr; // the batch's own stream
    cudaStream_t cur    = nullptr;
    cudaStream_t root   = nullptr; // capture origin
    cudaEvent_t fork    = nullptr;
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        std::vector<long long> nodes; // kernel launches per member
    };
    std::map<std::tuple<int, int, std::vector<const void *>>, Graph> graphs;

    ~gpe_batch() {
        cudaSetDevice(device);
        if (cur)
            cudaStreamSynchronize(cur);
        for (auto &kv : graphs)
            cudaGraphExecDestroy(kv.second.exec);
        for (auto *m : members)
            delete m;
        if (fork)
            cudaEventDestroy(fork);
        if (root)
            cudaStreamDestroy(root);
        if (own)
            cudaStreamDestroy(own);
    }

    // iterations of every member per graph launch (GPE_BATCH_CHUNK overrides):
    // a call of up to 1024 iterations is one launch, each member an independent
    // chain of its prologue and iterations (a 64-member sweep of 1000
    // iterations: 0.761-0.764 s against 0.766-0.767 s in launches of 64)
    long chunk = 1024;

    // One launch of the batch graph for (kind, count): kind 20 the IT prologue,
    // 21 `count` IT iterations of every member, 23 the prologue and `count`
    // iterations.
    void run(int kind, int count) {
        std::vector<const void *> sig;
        for (auto *m : members)
            sig.push_back(m->impl->psi_ptr());
        auto key = std::make_tuple(kind, count, sig);
        auto it  = graphs.find(key);
        if (it == graphs.end()) {
            Graph g;
            GPE_CUDA(cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal));
            try {
                GPE_CUDA(cudaEventRecord(fork, root));
                for (auto *m : members)
                    g.nodes.push_back(m->impl->capture_it_branch(kind, count, fork, root));
            } catch (...) {
                cudaGraph_t gr = nullptr;
                cudaStreamEndCapture(root, &gr);
                if (gr)
                    cudaGraphDestroy(gr);
                throw;
            }
            cudaGraph_t gr;
            GPE_CUDA(cudaStreamEndCapture(root, &gr));
            GPE_CUDA(cudaGraphInstantiate(&g.exec, gr, 0));
            cudaGraphDestroy(gr);
            it = graphs.emplace(key, std::move(g)).first;
        }
        GPE_CUDA(cudaGraphLaunch(it->second.exec, cur));
        for (size_t m = 0; m < members.size(); ++m)
            members[m]->impl->it_batch_after(kind, count, it->second.nodes[m]);
    }
};

namespace {

// PsiCoef of DataInitializer::init_with_* (initializer.cpp:46-219), host FP64
// with the reference's expressions.
gpe::PsiCoef psi_coef(const gpe_params &p, int strategy, const gpe_init_params &ip) {
    gpe::PsiCoef c{};
    c.strategy = strategy;
    if (strategy == GPE_INIT_COS) {
        c.rrr = (static_cast<int>(p.nx / 2) * p.dx);
        c.dd  = ip.dd;
    } else if (strategy == GPE_INIT_GAUSS) {
        c.sx = (p.nx * p.dx) / 10.;
        c.sy = (p.ny * p.dy) / 10.;
        c.sz = (p.nz * p.dz) / 10.;
    } else if (strategy == GPE_INIT_MULTIPLE_GAUSS) {
        c.sx = (p.nx * p.dx) / 20.;
        c.sy = (p.ny * p.dy) / 20.;
        c.sz = (p.nz * p.dz) / 20.;
        const int n = ip.n_gauss_max;
        if (n < 0 || n > gpe::kMaxGaussCentres)
            throw gpe::Error(GPE_ERR_ARG, "n_gauss_max must be in 0..64");
        c.ncent = n;
        const double y0 = (0 - (static_cast<int>(p.ny / 2))) * p.dy;
        for (int idx = 0; idx < n; ++idx) {
            c.cx[idx] = idx % 2 ? ip.dd : -ip.dd;
            if (n % 2 == 1) {
                const int center_y_idx = n / 2;
                c.cy[idx]              = (idx - center_y_idx) * (p.ny * p.dy) / 2. / (n + 1.);
            } else {
                const int y_idx = (idx / 2 + 1), y_maximas = (n / 2 + 1);
                c.cy[idx]       = y0 + y_idx * (p.ny * p.dy) / y_maximas;
            }
        }
    } else if (strategy == GPE_INIT_SETUP_GAUSS) {
        c.sx = (p.nx * p.dx) / 20.;
        c.sy = (p.ny * p.dy) / 20.;
        c.sz = (p.nz * p.dz) / 20.;
        const int bx = ip.bec_droplets_x, by = ip.bec_droplets_y, bz = ip.bec_droplets_z;
        if (bx < 0 || by < 0 || bz < 0 || (long)bx * by * bz > gpe::kMaxGaussCentres)
            throw gpe::Error(GPE_ERR_ARG, "bec_droplets_x * _y * _z must be in 0..64");
        c.ncent = bx * by * bz;
        c.zcent = 1;
        const double x_tot = p.nx * p.dx, y_tot = p.ny * p.dy, z_tot = p.nz * p.dz;
        for (int i = 0; i < bx; ++i)
            for (int j = 0; j < by; ++j)
                for (int k = 0; k < bz; ++k) {
                    const int idx          = i * by * bz + j * bz + k;
                    const double spacing_x = x_tot / static_cast<double>(bx + 1);
                    const double spacing_y = y_tot / static_cast<double>(by + 1);
                    const double spacing_z = z_tot / static_cast<double>(bz + 1);
                    c.cx[idx]              = -x_tot / 2 + spacing_x * (i + 1);
                    c.cy[idx]              = -y_tot / 2 + spacing_y * (j + 1);
                    c.cz[idx]              = -z_tot / 2 + spacing_z * (k + 1);
                }
    } else {
        throw gpe::Error(GPE_ERR_ARG, "unknown initial-state strategy");
    }
    return c;
}

} // namespace

extern "C" {

int gpe_init_potential(gpe_handle *h, int pote, const gpe_init_params *ip) {
    GPE_HANDLE(h);
    if (!ip)
        return bad("null init params");
    if (pote < 0 || pote >= gpe::POT_COUNT)
        return bad("unknown potential");
    return guarded([&] {
        const gpe_params &p = h->params;
        gpe::PotCoef c{};
        c.key = pote;
        c.m   = p.m;
        c.wx = ip->omega_x, c.wy = ip->omega_y, c.wz = ip->omega_z;
        c.aa = ip->aa, c.b = ip->b;
        if (pote == GPE_POT_MEXICAN_ASYMETRIC || pote == GPE_POT_MEXICAN_ASYMETRIC_FREE) {
            // potentials.hpp:133-137
            const double conv = 27211.4 * 11.6 * 1e9;
            const double nK25 = 0.25 / conv;
            c.slope           = nK25 / ip->dd;
        }
        h->impl->init_potential(c);
    });
}

int gpe_init_psi(gpe_handle *h, int strategy, const gpe_init_params *ip) {
    GPE_HANDLE(h);
    if (!ip)
        return bad("null init params");
    return guarded([&] { h->impl->init_psi(psi_coef(h->params, strategy, *ip)); });
}

int gpe_export_potential(gpe_handle *h, double *V, size_t n) {
    GPE_HANDLE(h);
    if (!V || n != h->impl->n())
        return bad("potential buffer size mismatch");
    return guarded([&] { h->impl->export_potential(V); });
}

int gpe_imag_steps_energies(gpe_handle *h, long k, int checks, double *e_total) {
    GPE_HANDLE(h);
    if (!e_total)
        return bad("null argument");
    return guarded([&] { h->impl->imag_steps_energies(k, checks, e_total); });
}

int gpe_export_psi_async(gpe_handle *h, double *psi_c128, size_t n) {
    GPE_HANDLE(h);
    if (!psi_c128 || n != h->impl->n())
        return bad("psi buffer size mismatch");
    return guarded([&] { h->impl->export_psi_async(psi_c128); });
}

int gpe_export_wait(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->export_wait(); });
}

int gpe_export_amplitude_device(gpe_handle *h, float *amp, size_t n) {
    GPE_HANDLE(h);
    if (!amp || n != h->impl->n())
        return bad("amplitude buffer size mismatch");
    return guarded([&] { h->impl->export_amplitude_device(amp); });
}

int gpe_load_amplitude_device(gpe_handle *h, const float *amp, size_t n) {
    GPE_HANDLE(h);
    if (!amp || n != h->impl->n())
        return bad("amplitude buffer size mismatch");
    return guarded([&] { h->impl->load_amplitude_device(amp); });
}

int gpe_batch_create(const gpe_params *members, int count, gpe_batch **out) {
    if (!members || !out || count <= 0)
        return bad("null argument or empty batch");
    *out = nullptr;
    for (int m = 0; m < count; ++m)
        if (members[m].device != members[0].device)
            return bad("batch members must share one device");
    return guarded([&] {
        auto b    = std::make_unique<gpe_batch>();
        b->device = members[0].device;
        GPE_CUDA(cudaSetDevice(b->device));
        GPE_CUDA(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
        GPE_CUDA(cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking));
        GPE_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        b->cur = b->own;
        if (const char *e = std::getenv("GPE_BATCH_CHUNK")) {
            const long c = std::atol(e);
            if (c < 1 || c > 4096)
                throw gpe::Error(GPE_ERR_ARG, "GPE_BATCH_CHUNK must be in 1..4096");
            b->chunk = c;
        }
        for (int m = 0; m < count; ++m) {
            gpe_handle *h = nullptr;
            const int rc  = gpe_create(&members[m], &h);
            if (rc != GPE_OK)
                throw gpe::Error(rc, "batch member " + std::to_string(m) + ": " + gpe::last_error());
            b->members.push_back(h);
            if (!h->impl->batchable())
                throw gpe::Error(GPE_ERR_STATE, "batch member " + std::to_string(m) +
                                                    ": needs complex64 and a grid with the fused pipeline");
            h->impl->set_stream(b->cur);
        }
        *out = b.release();
    });
}

int gpe_batch_destroy(gpe_batch *b) {
    delete b;
    return GPE_OK;
}

int gpe_batch_member(gpe_batch *b, int m, gpe_handle **h) {
    if (!b || !h || m < 0 || m >= (int)b->members.size())
        return bad("bad batch or member index");
    *h = b->members[m];
    return GPE_OK;
}

int gpe_batch_set_stream(gpe_batch *b, void *s) {
    if (!b)
        return bad("null batch");
    if (cudaSetDevice(b->device) != cudaSuccess)
        return bad("cudaSetDevice failed");
    return guarded([&] {
        b->cur = s ? (cudaStream_t)s : b->own;
        for (auto *m : b->members)
            m->impl->set_stream(b->cur);
    });
}

int gpe_batch_imag_steps(gpe_batch *b, long k) {
    if (!b)
        return bad("null batch");
    if (k < 0)
        return bad("negative iteration count");
    if (cudaSetDevice(b->device) != cudaSuccess)
        return bad("cudaSetDevice failed");
    if (k == 0)
        return GPE_OK;
    return guarded([&] {
        for (auto *m : b->members)
            m->impl->it_batch_begin();
        // the fused imaginary-time schedule of every member (fused_imag):
        // prologue, chunks of 64 iterations, remainder
        const long CH = b->chunk;
        long done     = std::min(k, CH);
        b->run(23, (int)done);
        while (k - done >= CH) {
            b->run(21, (int)CH);
            done += CH;
        }
        if (k - done > 0)
            b->run(21, (int)(k - done));
        for (auto *m : b->members)
            m->impl->it_batch_end();
    });
}

int gpe_destroy(gpe_handle *h) {
    if (!h)
        return GPE_OK;
    cudaSetDevice(h->device);
    delete h;
    return GPE_OK;
}

int gpe_set_stream(gpe_handle *h, void *s) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->set_stream((cudaStream_t)s); });
}

int gpe_get_stream(gpe_handle *h, void **s) {
    GPE_HANDLE(h);
    if (!s)
        return bad("null argument");
    *s = (void *)h->impl->stream();
    return GPE_OK;
}

int gpe_synchronize(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] {
        cudaError_t e = cudaStreamSynchronize(h->impl->stream());
        if (e != cudaSuccess)
            throw gpe::Error(GPE_ERR_CUDA, cudaGetErrorString(e));
    });
}

int gpe_load_psi(gpe_handle *h, const double *psi, size_t n) {
    GPE_HANDLE(h);
    if (!psi || n != h->impl->n())
        return bad("gpe_load_psi: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->load_psi(psi); });
}

int gpe_load_potential(gpe_handle *h, const double *V, size_t n) {
    GPE_HANDLE(h);
    if (!V || n != h->impl->n())
        return bad("gpe_load_potential: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->load_potential(V); });
}

int gpe_export_psi(gpe_handle *h, double *psi, size_t n) {
    GPE_HANDLE(h);
    if (!psi || n != h->impl->n())
        return bad("gpe_export_psi: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->export_psi(psi); });
}

int gpe_export_fi3d(gpe_handle *h, double *fi3d, size_t n) {
    GPE_HANDLE(h);
    if (!fi3d || n != h->impl->n())
        return bad("gpe_export_fi3d: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->export_fi3d(fi3d); });
}

int gpe_load_fi3d(gpe_handle *h, const double *fi3d, size_t n) {
    GPE_HANDLE(h);
    if (!fi3d || n != h->impl->n())
        return bad("gpe_load_fi3d: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->load_fi3d(fi3d); });
}

int gpe_calc_fi3d(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->calc_fi3d(); });
}

int gpe_imag_iter_linear_step(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->imag_linear(); });
}

int gpe_imag_iter_nonlinear_step(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->imag_nonlinear(); });
}

int gpe_calc_norm(gpe_handle *h, double *x) {
    GPE_HANDLE(h);
    return guarded([&] {
        double v = h->impl->calc_norm(x != nullptr);
        if (x)
            *x = v;
    });
}

int gpe_import_psi(gpe_handle *h, const double *psi, size_t n) {
    GPE_HANDLE(h);
    if (!psi || n != h->impl->n())
        return bad("gpe_import_psi: null pointer or n != nx*ny*nz");
    return guarded([&] { h->impl->import_psi(psi); });
}

int gpe_normalize(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->normalize(); });
}

int gpe_real_fft_potential_half_step(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->potential_half_step(); });
}

int gpe_real_fft_kinetic_step(gpe_handle *h) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->kinetic_step(); });
}

int gpe_calc_energy(gpe_handle *h, double *out6) {
    GPE_HANDLE(h);
    if (!out6)
        return bad("null argument");
    return guarded([&] { h->impl->energy(out6); });
}

int gpe_set_coeffs(gpe_handle *h, double ggp11, double gamma) {
    GPE_HANDLE(h);
    return guarded([&] { h->impl->set_coeffs(ggp11, gamma); });
}

int gpe_imag_steps(gpe_handle *h, long k) {
    GPE_HANDLE(h);
    if (k < 0)
        return bad("negative iteration count");
    return guarded([&] { h->impl->imag_steps(k); });
}

int gpe_real_steps(gpe_handle *h, long k, long first_iter) {
    GPE_HANDLE(h);
    if (k < 0 || first_iter < 0)
        return bad("negative iteration count");
    return guarded([&] { h->impl->real_steps(k, first_iter); });
}

int gpe_time_kernel(gpe_handle *h, int which, int reps, double *ms, double *bytes) {
    GPE_HANDLE(h);
    if (!ms || !bytes)
        return bad("null argument");
    return guarded([&] { h->impl->time_kernel(which, reps, ms, bytes); });
}

const char *gpe_kernel_name(int which) {
    static const char *names[] = {"k_dip_z_fwd", "k_dip_y", "k_dip_x", "k_dip_y", "k_dip_z_inv",
                                  "k_kin_z", "k_kin_y", "k_kin_x", "k_kin_y", "k_kin_z",
                                  "k_phase", "k_it_update", "k3_x", "k3_y", "k2_z", "k3_y",
                                  "k3_x_kin", "k3_x_dip", "k4_yz"};
    if (which < 0 || which >= GPE_K_COUNT)
        return "";
    return names[which];
}

const char *gpe_plane_kernel_name(gpe_handle *h) {
    if (!h || !h->impl)
        return "";
    return h->impl->plane_kernel();
}

int gpe_launch_count(gpe_handle *h, long long *count) {
    GPE_HANDLE(h);
    if (!count)
        return bad("null argument");
    *count = h->impl->launches();
    return GPE_OK;
}

int gpe_x_tiles(gpe_handle *h, int *kin_lines, int *dip_lines) {
    GPE_HANDLE(h);
    if (!kin_lines || !dip_lines)
        return bad("null argument");
    h->impl->x_tiles(kin_lines, dip_lines);
    return GPE_OK;
}

} // extern "C"
