// Two quotients with one divisor, a1 / b and a2 / b, by Markstein's method on a
// shared reciprocal, against two IEEE divisions: throughput, and a bit-for-bit
// comparison on the device. The bundle transport has such a pair in every cell
// (its two k_dx bounds share the divisor e1); this probe measures what sharing
// the reciprocal would save there.
//
// The sequence (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990; J.-M. Muller et
// al., Handbook of Floating-Point Arithmetic, Birkhauser, ch. on FMA-based
// division), binary64, round to nearest even, all steps single FMAs:
//   y  = RN(1/b)                 (__drcp_rn, CUDA's correctly rounded reciprocal)
//   q0 = RN(a y)
//   r0 = RN(a - b q0),  q1 = RN(q0 + r0 y)
//   r1 = RN(a - b q1),  q2 = RN(q1 + r1 y)   = RN(a / b)
// Why q2 is a / b correctly rounded, scaled to 1 <= a, b < 2 (powers of two scale
// every step exactly while nothing under- or overflows), a, b > 0, b > 1 (b = 1
// is exact), Q = a / b in (1/2, 2):
//  1. |y - 1/b| <= 2^-54, so e = b y - 1 has |e| <= b 2^-54 < 2^-53.
//  2. |q0 - Q| <= a |y - 1/b| + (rounding of a y) < 2^-52.
//  3. r0 = b (Q - q0)(1 + d), |d| <= 2^-53, so q0 + r0 y = Q + (Q - q0) h with
//     |h| < 2^-52 + 2^-106: q1 = RN(Q + D1), |D1| < 2^-103.99, is one of the two
//     doubles around Q (faithful).
//  4. A faithful q1 makes r1 = a - b q1 exact, so q1 + r1 y = Q + (Q - q1) e.
//  5. Q is never a midpoint of two doubles (a = b m with m of 54 significant bits
//     would need more than 53 bits in a), and its distance to the nearest one is
//     at least 2^-106 / b for Q < 1 (2^-105 / b for Q >= 1): a - b m is a nonzero
//     multiple of 2^-106 (2^-105).
//  6. |Q - q1| <= ulp(Q)/2 + 2^-104 and |e| <= b 2^-54 give |(Q - q1) e| below that
//     distance whenever b^2 (1 + 2^-50) < 4, i.e. for every b below 2 - 4 ulp.
//     Then no midpoint lies between Q and Q + (Q - q1) e, and q2 = RN(Q).
// The guard sends everything else to '/': a divisor with one of the four largest
// significands, any operand outside [2^-500, 2^500] in magnitude (zeros,
// subnormals, infinities and NaN included), so that no step under- or overflows.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ double two_corrections(double a, double b, double y) {
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-b, q1, a);
    return fma(r1, y, q1);
}
__device__ __forceinline__ double one_correction(double a, double b, double y) {
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    return fma(r0, y, q0);
}
// exponent field in [523, 1523]: |x| in [2^-500, 2^501)
__device__ __forceinline__ bool in_range(double x) {
    const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7FFu;
    return e - 523u <= 1000u;
}
__device__ __forceinline__ bool divisor_ok(double b) {
    const unsigned hi = (unsigned)__double2hiint(b), lo = (unsigned)__double2loint(b);
    return in_range(b) && !((hi & 0xFFFFFu) == 0xFFFFFu && lo >= 0xFFFFFFFCu);
}
__device__ __forceinline__ void shared_quotients(double a1, double a2, double b, double &q1, double &q2) {
    const double y = __drcp_rn(b);
    q1 = two_corrections(a1, b, y);
    q2 = two_corrections(a2, b, y);
    if (!(divisor_ok(b) && in_range(a1) && in_range(a2))) {
        q1 = a1 / b;
        q2 = a2 / b;
    }
}

// V 0: two IEEE divisions; 1: shared reciprocal, two corrections, no guard;
// 2: shared reciprocal, one correction (no proof; timing only); 3: the guarded form
template <int V>
__global__ void k_time(const double *A, const double *B, double *out, int iters) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double a1 = A[2 * t], a2 = A[2 * t + 1], b = B[t];
    double acc = 0.0;
    for (int k = 0; k < iters; ++k) {
        double q1, q2;
        if (V == 0) {
            q1 = a1 / b;
            q2 = a2 / b;
        } else if (V == 1 || V == 2) {
            const double y = __drcp_rn(b);
            q1 = V == 1 ? two_corrections(a1, b, y) : one_correction(a1, b, y);
            q2 = V == 1 ? two_corrections(a2, b, y) : one_correction(a2, b, y);
        } else {
            shared_quotients(a1, a2, b, q1, q2);
        }
        acc += q1;
        acc += q2;
        b += 0.0078125;
        a1 += 0.015625;
    }
    out[t] = acc;
}

__device__ uint64_t mix(uint64_t &s) {  // splitmix64
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__device__ double u01(uint64_t &s) { return (double)(mix(s) >> 11) * 0x1.0p-53; }

__device__ bool same_bits(double x, double y) {
    return __double_as_longlong(x) == __double_as_longlong(y) || (x != x && y != y);
}

// mode 0: the transport's ranges (divisors in [-10, 190], half of them scaled by
// 2^-40 as cancelled sums; numerators in [-20, 20]); 1: random significands,
// exponents in [-60, 60]; 2: divisors with significands within 2^16 ulp of 1 or of
// 2; 3: special operands mixed with random ones; 4: the 64 largest significands
__global__ void k_check(int mode, int per_thread, unsigned long long *bad) {
    const unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    uint64_t s = 0x1234567ULL + t * 0x9E3779B97F4A7C15ULL + (uint64_t)mode * 7919ULL;
    const double sp[] = {0.0, -0.0, 0x1p-1074, -0x1p-1060, 0x1.8p-1022, 0x1p-501, 0x1p-500,
                         0x1.fffffffffffffp-501, 0x1p500, 0x1.fffffffffffffp500, 0x1p501, 1e300, -1e308,
                         __longlong_as_double(0x7FF0000000000000LL), __longlong_as_double(0xFFF0000000000000LL),
                         __longlong_as_double(0x7FF8000000000000LL), 0x1.fffffffffffffp0, 0x1.ffffffffffffep0,
                         0x1.ffffffffffffdp0, 0x1.ffffffffffffcp0, 0x1.ffffffffffffbp0, -0x1.fffffffffffffp-3,
                         1.0, -1.0, 3.0, 0.1};
    const int ns = (int)(sizeof(sp) / sizeof(sp[0]));
    unsigned long long nb = 0;
    for (int i = 0; i < per_thread; ++i) {
        double a, b;
        const uint64_t r = mix(s);
        if (mode == 0) {
            b = u01(s) * 200.0 - 10.0;
            a = u01(s) * 40.0 - 20.0;
            if (r & 1) b *= 0x1p-40;
        } else if (mode == 1) {
            b = ldexp(1.0 + u01(s), (int)(mix(s) % 121) - 60) * ((r & 1) ? -1.0 : 1.0);
            a = ldexp(1.0 + u01(s), (int)(mix(s) % 121) - 60) * ((r & 2) ? -1.0 : 1.0);
        } else if (mode == 2 || mode == 4) {
            const uint64_t m = mode == 4 ? 0xFFFFFFFFFFFFFULL - ((r >> 2) % 64)
                                         : ((r & 1) ? 0xFFFFFFFFFFFFFULL - ((r >> 2) % 65536) : (r >> 2) % 65536);
            const uint64_t bb = ((0x3FFULL + (mix(s) % 41) - 20) << 52) | m;
            memcpy(&b, &bb, 8);
            if (r & 2) b = -b;
            a = ldexp(1.0 + u01(s), (int)(mix(s) % 41) - 20) * ((r & 4) ? -1.0 : 1.0);
        } else {
            b = ((r & 3) == 0) ? sp[(r >> 2) % ns] : ldexp(1.0 + u01(s), (int)(mix(s) % 41) - 20);
            a = ((r & 12) == 0) ? sp[(r >> 5) % ns]
                                : ldexp(1.0 + u01(s), (int)(mix(s) % 41) - 20) * ((r & 16) ? -1.0 : 1.0);
        }
        double q1, q2;
        shared_quotients(a, -0.75 * a, b, q1, q2);
        if (!same_bits(q1, a / b) || !same_bits(q2, (-0.75 * a) / b)) ++nb;
    }
    atomicAdd(bad, nb);
}

}  // namespace

int main() {
    const int blocks = 148 * 8, threads = 256, n = blocks * threads, iters = 4096;
    double *A = nullptr, *B = nullptr, *out = nullptr;
    unsigned long long *bad = nullptr;
    if (cudaMalloc(&A, sizeof(double) * 2 * n) != cudaSuccess || cudaMalloc(&B, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&out, sizeof(double) * n) != cudaSuccess || cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess) {
        printf("error allocation\n");
        return 1;
    }
    double *hA = new double[2 * n], *hB = new double[n];
    uint64_t s = 42;
    for (int i = 0; i < n; ++i) {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        hB[i] = 0.5 + (double)(s >> 11) * 0x1.0p-53 * 10.0;
        hA[2 * i] = (double)((s >> 20) & 0xffff) / 4096.0 - 8.0;
        hA[2 * i + 1] = hA[2 * i] + 1.2;
    }
    cudaMemcpy(A, hA, sizeof(double) * 2 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(B, hB, sizeof(double) * n, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const char *names[] = {"two_divisions", "shared_two_corrections", "shared_one_correction", "shared_guarded"};
    float best[4] = {1e30f, 1e30f, 1e30f, 1e30f};
    for (int rep = 0; rep < 4; ++rep) {
        for (int v = 0; v < 4; ++v) {
            cudaEventRecord(e0);
            if (v == 0) k_time<0><<<blocks, threads>>>(A, B, out, iters);
            if (v == 1) k_time<1><<<blocks, threads>>>(A, B, out, iters);
            if (v == 2) k_time<2><<<blocks, threads>>>(A, B, out, iters);
            if (v == 3) k_time<3><<<blocks, threads>>>(A, B, out, iters);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && ms < best[v]) best[v] = ms;  // the first round warms up
        }
    }
    for (int v = 0; v < 4; ++v)
        printf("time %s %.4f ms %.1f G_pairs_per_s\n", names[v], best[v], (double)n * iters / (best[v] * 1e6));
    const int per = 4096;
    for (int mode = 0; mode < 5; ++mode) {
        unsigned long long hb = 0;
        cudaMemset(bad, 0, sizeof(hb));
        k_check<<<blocks, threads>>>(mode, per, bad);
        cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost);
        printf("check mode %d operands %lld mismatches %llu\n", mode, (long long)n * per, hb);
    }
    const cudaError_t err = cudaDeviceSynchronize();
    printf("status %s\n", cudaGetErrorString(err));
    delete[] hA;
    delete[] hB;
    return err == cudaSuccess ? 0 : 1;
}
