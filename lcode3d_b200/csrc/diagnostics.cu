// The reference's density-noise diagnostic on the device (lcode.py:979-987,
// diags_ro_zn):
//     blurred = gaussian_filter(ro, sigma = 0.25 / h)      (scipy.ndimage)
//     zn = mean |ro - blurred| / 4.23045376e-04
// The Gaussian is scipy's: weights exp(-k^2 / (2 sigma^2)) for |k| <= r,
// r = int(4 sigma + 0.5), normalised to sum 1, applied along axis 0 then
// axis 1 with the 'reflect' boundary (d c b a | a b c d | d c b a). One
// pass per axis; the mean is a fixed-order reduction (block partial sums,
// then one block), so the result is deterministic.

#include <cmath>
#include <vector>

#include "lc3d_internal.cuh"

namespace {

constexpr int ZN_THREADS = 256;
constexpr int ZN_BLOCKS = 296;
constexpr int ZN_MAX_R = 1024;

__device__ __forceinline__ int reflect(int i, int n) {
    // scipy 'reflect' (half-sample symmetric) for |overhang| < n
    if (i < 0) i = -i - 1;
    if (i >= n) i = 2 * n - 1 - i;
    return i;
}

// out[i][j] = sum_k w[k] in[reflect(i + k - r)][j]   (axis 0), or along j (axis 1)
__global__ void __launch_bounds__(ZN_THREADS) blur_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                          const double* __restrict__ w, int r, int N, int axis) {
    const int k = blockIdx.x * ZN_THREADS + threadIdx.x;
    if (k >= N * N) return;
    const int i = k / N, j = k - i * N;
    double s = 0.0;
    if (axis == 0) {
        for (int t = -r; t <= r; ++t) s += __ldg(w + t + r) * __ldg(in + (size_t)reflect(i + t, N) * N + j);
    } else {
        const double* row = in + (size_t)i * N;
        for (int t = -r; t <= r; ++t) s += __ldg(w + t + r) * __ldg(row + reflect(j + t, N));
    }
    out[k] = s;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int h = ZN_THREADS / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    return sh[0];
}

__global__ void __launch_bounds__(ZN_THREADS) absdiff_partial_kernel(const double* __restrict__ a,
                                                                     const double* __restrict__ b, int n,
                                                                     double* __restrict__ partial) {
    __shared__ double sh[ZN_THREADS];
    double v = 0.0;
    for (int k = blockIdx.x * ZN_THREADS + threadIdx.x; k < n; k += ZN_BLOCKS * ZN_THREADS) v += fabs(a[k] - b[k]);
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(ZN_THREADS) zn_final_kernel(const double* __restrict__ partial, double scale,
                                                              double* out) {
    __shared__ double sh[ZN_THREADS];
    double v = 0.0;
    for (int k = threadIdx.x; k < ZN_BLOCKS; k += ZN_THREADS) v += partial[k];
    const double s = block_sum(v, sh);
    if (threadIdx.x == 0) *out = s * scale;
}

}  // namespace

int diag_init(lc3d_ctx* c) {
    const double sigma = 0.25 / c->p.grid_step_size;
    int r = (int)(4.0 * sigma + 0.5);
    if (r > ZN_MAX_R) r = ZN_MAX_R;
    if (r >= c->N) r = c->N - 1;   // 'reflect' indexing above covers one mirror image
    std::vector<double> w(2 * (size_t)r + 1 + ZN_BLOCKS);
    double sum = 0.0;
    for (int t = -r; t <= r; ++t) {
        const double v = std::exp(-0.5 * (double)t * (double)t / (sigma * sigma));
        w[t + r] = v;
        sum += v;
    }
    for (int t = 0; t <= 2 * r; ++t) w[t] /= sum;
    c->diag_r = r;
    LC3D_CUDA_TRY(cudaMalloc(&c->diag_w, w.size() * sizeof(double)));
    LC3D_CUDA_TRY(cudaMemcpy(c->diag_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
    LC3D_CUDA_TRY(cudaMalloc(&c->diag_buf, 2 * (size_t)c->N * c->N * sizeof(double)));
    return LC3D_OK;
}

void diag_free(lc3d_ctx* c) {
    if (c->diag_w) cudaFree(c->diag_w);
    if (c->diag_buf) cudaFree(c->diag_buf);
    c->diag_w = nullptr;
    c->diag_buf = nullptr;
}

extern "C" int lc3d_diag_zn(lc3d_ctx* c, const double* ro, double* zn, void* stream) {
    if (!c || !ro || !zn || !c->diag_w) return LC3D_ERR_PARAM;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != c->device) cudaSetDevice(c->device);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int N = c->N, n = N * N, r = c->diag_r;
    double* t0 = c->diag_buf;
    double* t1 = c->diag_buf + n;
    double* partial = c->diag_w + 2 * r + 1;
    const unsigned grid = (unsigned)((n + ZN_THREADS - 1) / ZN_THREADS);
    int rc = LC3D_OK;
    {
        ProfScope ps(c, LC3D_STAGE_OTHER, s);
        blur_kernel<<<grid, ZN_THREADS, 0, s>>>(ro, t0, c->diag_w, r, N, 0);
        blur_kernel<<<grid, ZN_THREADS, 0, s>>>(t0, t1, c->diag_w, r, N, 1);
        absdiff_partial_kernel<<<ZN_BLOCKS, ZN_THREADS, 0, s>>>(ro, t1, n, partial);
        zn_final_kernel<<<1, ZN_THREADS, 0, s>>>(partial, 1.0 / ((double)n * 4.23045376e-04), zn);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            lc3d_set_last_cuda_error(e, "lc3d_diag_zn", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
        }
    }
    if (dev >= 0 && dev != c->device) cudaSetDevice(dev);
    return rc;
}
