// sincos against sin and cos on the device, bit for bit, in double and float: the
// neighbour kernel takes an anchor's trig row from one sincos per lane where the
// reference calls sin and cos, and the two must give the same values.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace {

__device__ __noinline__ double f_sin(double x) { return sin(x); }
__device__ __noinline__ double f_cos(double x) { return cos(x); }
__device__ __noinline__ float g_sin(float x) { return sinf(x); }
__device__ __noinline__ float g_cos(float x) { return cosf(x); }

__device__ uint64_t mix(uint64_t &s) {  // splitmix64
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// mode 0: angles of the path, [-0.5, 6.5); 1: arguments up to 1e6 in magnitude;
// 2: any finite double (and its float where finite)
__global__ void k_check(int mode, int per_thread, unsigned long long *bad) {
    const unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    uint64_t s = 77 + t * 0x9E3779B97F4A7C15ULL + (uint64_t)mode;
    unsigned long long nb = 0;
    for (int i = 0; i < per_thread; ++i) {
        const uint64_t r = mix(s);
        double x;
        if (mode == 0) x = (double)(r >> 11) * 0x1.0p-53 * 7.0 - 0.5;
        else if (mode == 1) x = ((double)(r >> 11) * 0x1.0p-53 - 0.5) * 2e6;
        else x = __longlong_as_double((long long)(r & 0x7FEFFFFFFFFFFFFFULL));
        double s1, c1;
        sincos(x, &s1, &c1);
        if (__double_as_longlong(s1) != __double_as_longlong(f_sin(x)) ||
            __double_as_longlong(c1) != __double_as_longlong(f_cos(x)))
            ++nb;
        const float xf = (float)x;
        if (isinf(xf)) continue;
        float s3, c3;
        sincosf(xf, &s3, &c3);
        if (__float_as_int(s3) != __float_as_int(g_sin(xf)) || __float_as_int(c3) != __float_as_int(g_cos(xf))) ++nb;
    }
    atomicAdd(bad, nb);
}

}  // namespace

int main() {
    unsigned long long *bad = nullptr, h = 0;
    if (cudaMalloc(&bad, sizeof(h)) != cudaSuccess) {
        printf("error allocation\n");
        return 1;
    }
    const int blocks = 148 * 8, threads = 256, per = 2048;
    for (int mode = 0; mode < 3; ++mode) {
        cudaMemset(bad, 0, sizeof(h));
        k_check<<<blocks, threads>>>(mode, per, bad);
        cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost);
        printf("check mode %d arguments %lld mismatches %llu\n", mode, (long long)blocks * threads * per, h);
    }
    const cudaError_t err = cudaDeviceSynchronize();
    printf("status %s\n", cudaGetErrorString(err));
    cudaFree(bad);
    return err == cudaSuccess ? 0 : 1;
}
