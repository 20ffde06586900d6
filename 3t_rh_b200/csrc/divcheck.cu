// Diagnostic (no reference counterpart): the shared-reciprocal divisions of
// divrn.cuh against the IEEE quotient, bit for bit, on operands generated on
// the device: random ones, divisors with all-ones significands, quotients
// next to a rounding midpoint, operands at and beyond the fast path's
// exponent range, and special values; and the reciprocals of a face's
// L-row divisors that roe_div (physics.cuh) forms by scaling 1/(12 c^2).
#include <cstdint>

#include <cuda_runtime.h>

#include "physics.cuh"

namespace rh3t {

__device__ __forceinline__ uint64_t mix64(uint64_t x) { // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// a double with random sign, random 52-bit fraction and exponent e (e in [-1023, 1023])
__device__ __forceinline__ double make_double(uint64_t h, int e) {
    const uint64_t frac = h & 0x000fffffffffffffull;
    const uint64_t sign = (h >> 63) << 63;
    return __longlong_as_double((long long)(sign | ((uint64_t)(e + 1023) << 52) | frac));
}

// a value whose quotient by b lies next to a rounding midpoint: RN(b mu),
// mu = q + ulp(q) / 2 for a random q with exponent e, moved by up to 3 ulps
__device__ __forceinline__ double near_midpoint(double b, uint64_t hq, int e, int shift) {
    const double q = make_double(hq & ~(1ull << 63), e);
    const double half_ulp = __longlong_as_double((long long)((__double_as_longlong(q) & 0x7ff0000000000000ll) -
                                                             (53ll << 52)));
    const double a = __fma_rn(b, q, b * half_ulp);
    return __longlong_as_double(__double_as_longlong(a) + shift);
}

__device__ __forceinline__ bool same_bits(double x, double y) {
    if (isnan(x) && isnan(y)) return true;
    return __double_as_longlong(x) == __double_as_longlong(y);
}

constexpr int DIV_CATEGORIES = 7;

// category of case k: 0 random, 1 all-ones divisors, 2 near-midpoint
// quotients, 3 range edges and special values, 4 a / 3, 5 a / 6, 6 the
// reciprocals of 6 c^2 and 3 c^2 in roe_div (c^2 > 0 with exponents over and
// beyond the fast range, all-ones significands among them)
__global__ void k_div_check(long long n, unsigned long long seed, unsigned long long* bad, double* first) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int cat = (int)(k % DIV_CATEGORIES);
        const uint64_t h1 = mix64(seed ^ (uint64_t)k), h2 = mix64(h1), h3 = mix64(h2);
        double a, b, got;
        if (cat == 0) {
            a = make_double(h1, (int)(h3 % 941) - 470);
            b = make_double(h2, (int)((h3 >> 16) % 941) - 470);
        } else if (cat == 1) {
            a = make_double(h1, (int)(h3 % 401) - 200);
            const uint64_t frac = 0x000fffffffffffffull - (h2 & 0xffull) - (((h3 >> 40) & 1) ? ((h2 >> 8) & 0xffffull) : 0);
            b = __longlong_as_double((long long)(((uint64_t)((int)((h3 >> 16) % 401) - 200 + 1023) << 52) | frac));
        } else if (cat == 2) {
            b = make_double(h1, (int)(h3 % 201) - 100);
            a = near_midpoint(b, h2, (int)((h3 >> 16) % 201) - 100, (int)((h3 >> 40) % 7) - 3);
        } else if (cat == 3) {
            const double specials[12] = {0.0, -0.0, INFINITY, -INFINITY, NAN, 4.9e-324, 2.2250738585072014e-308,
                                         1.7976931348623157e308, 0x1p-450, 0x1p450, 0x1.fffffffffffffp-451,
                                         0x1.fffffffffffffp450};
            a = (h3 & 3) == 0 ? specials[h1 % 12] : make_double(h1, (int)(h3 % 2047) - 1023);
            b = (h3 & 12) == 0 ? specials[h2 % 12] : make_double(h2, (int)((h3 >> 16) % 2047) - 1023);
            // next to the fast path's exponent range [-450, 450], on both sides
            if ((h3 >> 20) % 5 == 0) a = make_double(h1, ((h3 >> 44) & 1 ? 1 : -1) * ((int)((h3 >> 24) % 7) + 447));
            if ((h3 >> 28) % 5 == 0) b = make_double(h2, ((h3 >> 45) & 1 ? 1 : -1) * ((int)((h3 >> 32) % 7) + 447));
        } else if (cat == 6) {
            uint64_t hc = h1 & ~(1ull << 63);
            if ((h3 & 7) == 0) hc |= 0x000fffffffffffffull;
            const double cs2 = make_double(hc, (int)(h3 % 921) - 460);
            Roe q{};
            q.cs2 = cs2;
            q.den = 12.0 * cs2;
            q.b = 1.0;
            DevParams P{};
            P.gamma_e = 5.0 / 3.0;
            P.gamma_i = 5.0 / 3.0;
            P.gamma_r = 4.0 / 3.0;
            const RoeDiv rd = roe_div(q, P);
            const double w6 = __ddiv_rn(1.0, 6.0 * cs2), w3 = __ddiv_rn(1.0, 3.0 * cs2);
            a = cs2;
            b = 6.0 * cs2;
            if (!same_bits(rd.c6.y, w6) || !same_bits(rd.c3.y, w3) || rd.c6.b != 6.0 * cs2 || rd.c3.b != 3.0 * cs2) {
                atomicAdd(&bad[cat], 1ull);
                if (atomicAdd(&bad[DIV_CATEGORIES], 1ull) == 0) {
                    first[0] = a;
                    first[1] = b;
                    first[2] = same_bits(rd.c6.y, w6) ? rd.c3.y : rd.c6.y;
                }
            }
            continue;
        } else {
            b = cat == 4 ? 3.0 : 6.0;
            if ((h3 & 1) == 0) a = make_double(h1, (int)(h3 % 1001) - 500);
            else a = near_midpoint(b, h2, (int)((h3 >> 16) % 201) - 100, (int)((h3 >> 40) % 7) - 3);
        }
        const double want = __ddiv_rn(a, b);
        if (cat == 4) got = div3_rn(a);
        else if (cat == 5) got = div6_rn(a);
        else got = div_rn(a, recip(b));
        if (!same_bits(got, want)) {
            atomicAdd(&bad[cat], 1ull);
            if (atomicAdd(&bad[DIV_CATEGORIES], 1ull) == 0) {
                first[0] = a;
                first[1] = b;
                first[2] = got;
            }
        }
    }
}

} // namespace rh3t

// counts[0..6]: mismatches per category (0 random, 1 all-ones divisors, 2
// near-midpoint quotients, 3 range edges and special values, 4 a / 3,
// 5 a / 6, 6 roe_div's reciprocals of 6 c^2 and 3 c^2); first[3]: a, b and
// the routine's quotient of one mismatch (category 6: c^2, 6 c^2 and the
// reciprocal)
extern "C" int rh3t_div_check(int32_t device, int64_t n, uint64_t seed, int64_t* counts, double* first) {
    if (!counts || !first || n < 0) return 7; // RH3T_ERR_INVALID_ARGUMENT
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return 10; // RH3T_ERR_NO_DEVICE
    if (cudaSetDevice(device) != cudaSuccess) return 8;
    unsigned long long* d_bad = nullptr;
    double* d_first = nullptr;
    if (cudaMalloc(&d_bad, (rh3t::DIV_CATEGORIES + 1) * sizeof(unsigned long long)) != cudaSuccess) return 8;
    if (cudaMalloc(&d_first, 3 * sizeof(double)) != cudaSuccess) {
        cudaFree(d_bad);
        return 8;
    }
    cudaError_t e = cudaMemset(d_bad, 0, (rh3t::DIV_CATEGORIES + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d_first, 0, 3 * sizeof(double));
    if (e == cudaSuccess && n > 0) {
        rh3t::k_div_check<<<148 * 16, 256>>>((long long)n, (unsigned long long)seed, d_bad, d_first);
        e = cudaGetLastError();
    }
    unsigned long long h[rh3t::DIV_CATEGORIES + 1] = {0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d_bad, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(first, d_first, 3 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_bad);
    cudaFree(d_first);
    if (e != cudaSuccess) return 8; // RH3T_ERR_CUDA
    for (int k = 0; k < rh3t::DIV_CATEGORIES; ++k) counts[k] = (int64_t)h[k];
    return 0;
}
