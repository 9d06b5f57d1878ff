// bm_debug.cu — test-only entry points: the device math the step kernels use,
// run on caller-given inputs so that tests can compare it with the reference
// directly rather than through whole steps.
#include "bm_world.h"
#include "bm_math.cuh"

using namespace bm;

namespace {

// One 3x3 SVD per thread (bm::svd3, the step kernels' SVD::compute).
template <bool Fast>
__global__ void k_svd3(int64_t n, const float* __restrict__ F, float* __restrict__ U, float* __restrict__ S,
                       float* __restrict__ V) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[9], u[9], s[3], v[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = F[9 * i + q];
    svd3<Fast>(f, u, s, v);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        U[9 * i + q] = u[q];
        V[9 * i + q] = v[q];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) S[3 * i + q] = s[q];
}

}  // namespace

extern "C" {

BM_API bm_status_t bm_debug_svd3(int64_t n, const float* F, float* U, float* S, float* V, int32_t fast_math) {
    if (n < 0 || (n > 0 && (!F || !U || !S || !V))) return invalid_arg("bad SVD arrays");
    if (n == 0) return BM_OK;
    float* d = nullptr;
    const size_t b9 = sizeof(float) * 9 * (size_t)n, b3 = sizeof(float) * 3 * (size_t)n;
    BM_CHECK_CUDA(cudaMalloc((void**)&d, 3 * b9 + b3));
    float *dF = d, *dU = d + 9 * n, *dV = d + 18 * n, *dS = d + 27 * n;
    bm_status_t st = BM_OK;
    cudaError_t e = cudaMemcpy(dF, F, b9, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const unsigned blocks = (unsigned)((n + 127) / 128);
        if (fast_math) k_svd3<true><<<blocks, 128>>>(n, dF, dU, dS, dV);
        else k_svd3<false><<<blocks, 128>>>(n, dF, dU, dS, dV);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(U, dU, b9, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(V, dV, b9, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(S, dS, b3, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_last_error(std::string("bm_debug_svd3: ") + cudaGetErrorString(e));
        st = BM_ERR_CUDA;
    }
    cudaFree(d);
    return st;
}

}  // extern "C"
