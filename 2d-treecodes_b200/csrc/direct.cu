// direct.cu -- O(N M) FP64 direct sums on the GPU (accuracy reference at sizes where the CPU
// direct sum of main.cpp:201-245 would take minutes) and an FMA-throughput probe used as the
// FP64 / FP32 pipe peak of the roofline.
#include <algorithm>
#include <cfloat>

#include "tc_internal.h"
#include "tc_math.cuh"

namespace tc {

constexpr int DS_THREADS = 256;

// main.cpp:213-221: s += log(sqrt(r^2 + eps)) * v
__global__ __launch_bounds__(DS_THREADS) void k_direct_potential(
    const double *__restrict__ xs, const double *__restrict__ ys, const double *__restrict__ vs,
    int n, const double *__restrict__ xt, const double *__restrict__ yt, int m,
    double *__restrict__ out) {
    __shared__ double sx[DS_THREADS], sy[DS_THREADS], sv[DS_THREADS];
    const double eps = DBL_EPSILON * 10;
    const int i = blockIdx.x * DS_THREADS + threadIdx.x;
    const double x = i < m ? xt[i] : 0, y = i < m ? yt[i] : 0;
    double s = 0;
    for (int j0 = 0; j0 < n; j0 += DS_THREADS) {
        const int cnt = min(DS_THREADS, n - j0);
        __syncthreads();
        if (threadIdx.x < cnt) {
            sx[threadIdx.x] = xs[j0 + threadIdx.x];
            sy[threadIdx.x] = ys[j0 + threadIdx.x];
            sv[threadIdx.x] = vs[j0 + threadIdx.x];
        }
        __syncthreads();
        for (int k = 0; k < cnt; ++k) {
            const double xr = x - sx[k], yr = y - sy[k];
            s += log(sqrt(xr * xr + yr * yr + eps)) * sv[k];
        }
    }
    if (i < m) out[i] = s;
}

// main.cpp:232-243: (xs, ys) += v (xr, yr) / (r^2 + eps)
__global__ __launch_bounds__(DS_THREADS) void k_direct_force(
    const double *__restrict__ xs, const double *__restrict__ ys, const double *__restrict__ vs,
    int n, const double *__restrict__ xt, const double *__restrict__ yt, int m,
    double *__restrict__ xo, double *__restrict__ yo) {
    __shared__ double sx[DS_THREADS], sy[DS_THREADS], sv[DS_THREADS];
    const double eps = DBL_EPSILON * 10;
    const int i = blockIdx.x * DS_THREADS + threadIdx.x;
    const double x = i < m ? xt[i] : 0, y = i < m ? yt[i] : 0;
    double ax = 0, ay = 0;
    for (int j0 = 0; j0 < n; j0 += DS_THREADS) {
        const int cnt = min(DS_THREADS, n - j0);
        __syncthreads();
        if (threadIdx.x < cnt) {
            sx[threadIdx.x] = xs[j0 + threadIdx.x];
            sy[threadIdx.x] = ys[j0 + threadIdx.x];
            sv[threadIdx.x] = vs[j0 + threadIdx.x];
        }
        __syncthreads();
        for (int k = 0; k < cnt; ++k) {
            const double xr = x - sx[k], yr = y - sy[k];
            const double f = sv[k] / (xr * xr + yr * yr + eps);
            ax += xr * f;
            ay += yr * f;
        }
    }
    if (i < m) {
        xo[i] = ax;
        yo[i] = ay;
    }
}

int direct_potential(Context &c, const double *xs, const double *ys, const double *vs, int n,
                     const double *xt, const double *yt, int m, double *out) {
    if (m == 0) return TC_OK;
    k_direct_potential<<<(m + DS_THREADS - 1) / DS_THREADS, DS_THREADS, 0, c.stream>>>(
        xs, ys, vs, n, xt, yt, m, out);
    TC_KERNEL_CHECK();
    return TC_OK;
}

int direct_force(Context &c, const double *xs, const double *ys, const double *vs, int n,
                 const double *xt, const double *yt, int m, double *xo, double *yo) {
    if (m == 0) return TC_OK;
    k_direct_force<<<(m + DS_THREADS - 1) / DS_THREADS, DS_THREADS, 0, c.stream>>>(
        xs, ys, vs, n, xt, yt, m, xo, yo);
    TC_KERNEL_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------- log probe
// out[2i] = log_pos(x[i]) (the potential kernels' logarithm), out[2i + 1] = the library log.
__global__ void k_log_probe(const double *__restrict__ x, int n, double *__restrict__ out) {
    __shared__ double s_neg_log_c[LOG_NTAB];
    load_log_table(s_neg_log_c);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[2 * i] = log_pos(x[i], s_neg_log_c);
        out[2 * i + 1] = log(x[i]);
    }
}

int log_probe(Context &c, const double *x, int n, double *out) {
    if (n <= 0) return TC_OK;
    k_log_probe<<<(int)std::min<long long>((n + 255) / 256, 148 * 8), 256, 0, c.stream>>>(x, n, out);
    TC_KERNEL_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------- FMA probe
// Eight independent FMA chains per thread; flops = 2 * 8 * iters per thread.
template <class T>
__global__ void k_fma_peak(T *out, int iters, T b, T cst) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, cst);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == (T)-1.2345) out[blockIdx.x] = s;   // keeps the chains alive
}

int measure_fma_peak(int fp64, double *tflops) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void *out = nullptr;
    TC_CUDA_TRY(cudaMalloc(&out, 1 << 20));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = sms * 8, iters = fp64 ? 8192 : 16384;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (fp64)
            k_fma_peak<double><<<blocks, threads>>>((double *)out, iters, 0.9999999, 1e-7);
        else
            k_fma_peak<float><<<blocks, threads>>>((float *)out, iters, 0.99999f, 1e-5f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) {
        set_error(TC_ERR_CUDA, "fma probe: %s", cudaGetErrorString(err));
        return TC_ERR_CUDA;
    }
    const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return TC_OK;
}

void kernels_direct(KernelList &v) {
    v.insert(v.end(), {(const void *)k_direct_potential, (const void *)k_direct_force,
                       (const void *)k_log_probe, (const void *)k_fma_peak<float>,
                       (const void *)k_fma_peak<double>});
}

}  // namespace tc
