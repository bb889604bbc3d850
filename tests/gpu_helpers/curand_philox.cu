// Test helper: first outputs of cuRAND's Philox4_32_10 generator for given (seed, subsequence),
// and the CUDA math library's sinf/cosf/logf/expf, for comparison with the engine's own
// counter-based Philox and series-based elementary functions.
#include <curand_kernel.h>
#include <cuda_runtime.h>

__global__ void philox_kernel(unsigned long long seed, const unsigned long long* subseq, uint4* out, int n, int per) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandStatePhilox4_32_10_t s;
    curand_init(seed, subseq[i], 0, &s);
    for (int k = 0; k < per; ++k) out[i * per + k] = curand4(&s);
}

__global__ void math_kernel(int which, const float* x, float* y, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = x[i];
    y[i] = which == 0 ? sinf(v) : which == 1 ? cosf(v) : which == 2 ? logf(v) : expf(v);
}

extern "C" int curand_philox(unsigned long long seed, const unsigned long long* subseq, unsigned int* out, int n, int per) {
    unsigned long long* ds; uint4* dout;
    if (cudaMalloc(&ds, n * sizeof(unsigned long long)) != cudaSuccess) return 1;
    if (cudaMalloc(&dout, (size_t)n * per * sizeof(uint4)) != cudaSuccess) return 1;
    cudaMemcpy(ds, subseq, n * sizeof(unsigned long long), cudaMemcpyHostToDevice);
    philox_kernel<<<(n + 127) / 128, 128>>>(seed, ds, dout, n, per);
    cudaMemcpy(out, dout, (size_t)n * per * sizeof(uint4), cudaMemcpyDeviceToHost);
    cudaFree(ds); cudaFree(dout);
    return cudaGetLastError() != cudaSuccess;
}

extern "C" int cuda_math(int which, const float* x, float* y, int n) {
    float *dx, *dy;
    if (cudaMalloc(&dx, n * 4) != cudaSuccess || cudaMalloc(&dy, n * 4) != cudaSuccess) return 1;
    cudaMemcpy(dx, x, n * 4, cudaMemcpyHostToDevice);
    math_kernel<<<(n + 255) / 256, 256>>>(which, dx, dy, n);
    cudaMemcpy(y, dy, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(dx); cudaFree(dy);
    return cudaGetLastError() != cudaSuccess;
}
