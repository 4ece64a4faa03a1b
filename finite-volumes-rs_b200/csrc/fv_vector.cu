// DistributedVector operations (linalg/dvector.rs:46-160): dot / dot_smaller
// and sum with a fixed reduction order (each thread sums a fixed strided set
// of entries, then a fixed shuffle tree, then the block partials in block
// order, so a result depends only on n and the data), and the elementwise
// updates +=, -=, *= (scalar), inv and set, which are exact.
#include <algorithm>

#include "fv_internal.cuh"

namespace {

constexpr int kVB = 256;

inline int vec_grid(int64_t n) {
    const int64_t b = (n + kVB - 1) / kVB;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 4));
}

__device__ __forceinline__ double block_sum(double v, double *sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kVB / 32; ++w) t += sm[w];
    return t;
}

// mode 0: sum x_i y_i; mode 1: sum x_i
__global__ void __launch_bounds__(kVB) k_vec_partial(int64_t n, const double *__restrict__ x,
                                                     const double *__restrict__ y, int mode,
                                                     double *__restrict__ partial) {
    __shared__ double sm[kVB / 32];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * kVB + threadIdx.x; i < n; i += (int64_t)gridDim.x * kVB)
        acc += mode == 0 ? x[i] * y[i] : x[i];
    const double t = block_sum(acc, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

__global__ void k_vec_final(int nb, const double *__restrict__ partial, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += partial[b];
    *out = t;
}

// op 0: y += x; 1: y -= x; 2: y *= a; 3: y = 1 / y; 4: y = x
__global__ void k_vec_update(int64_t n, double *__restrict__ y, const double *__restrict__ x, double a, int op) {
    for (int64_t i = (int64_t)blockIdx.x * kVB + threadIdx.x; i < n; i += (int64_t)gridDim.x * kVB) {
        switch (op) {
        case 0: y[i] = y[i] + x[i]; break;
        case 1: y[i] = y[i] - x[i]; break;
        case 2: y[i] = y[i] * a; break;
        case 3: y[i] = 1.0 / y[i]; break;
        default: y[i] = x[i]; break;
        }
    }
}

fv_status reduce(int64_t n, const double *x, const double *y, int mode, void *stream, double *out) {
    if (n < 0 || !out) return FV_ERR_INVALID;
    if (n == 0) {  // empty vectors: no data pointer is needed
        *out = 0.0;
        return FV_OK;
    }
    if (!x || (mode == 0 && !y)) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int G = vec_grid(n);
    double *buf = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&buf, sizeof(double) * (G + 1), st));
    fv_note_launch();
    k_vec_partial<<<G, kVB, 0, st>>>(n, x, y, mode, buf);
    fv_note_launch();
    k_vec_final<<<1, 32, 0, st>>>(G, buf, buf + G);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf + G, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    FV_CUDA_TRY(e);
    return FV_OK;
}

}  // namespace

extern "C" fv_status fv_vec_dot(int64_t n, const double *x, const double *y, void *stream, double *out) {
    return reduce(n, x, y, 0, stream, out);
}

extern "C" fv_status fv_vec_sum(int64_t n, const double *x, void *stream, double *out) {
    return reduce(n, x, nullptr, 1, stream, out);
}

extern "C" fv_status fv_vec_update(int64_t n, double *y, const double *x, double a, int32_t op, void *stream) {
    if (n < 0 || op < 0 || op > 4) return FV_ERR_INVALID;
    if (n == 0) return FV_OK;
    if (!y || ((op == 0 || op == 1 || op == 4) && !x)) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    fv_note_launch();
    k_vec_update<<<vec_grid(n), kVB, 0, st>>>(n, y, x, a, op);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}
