// hea_device.cuh -- device primitives of the swap search (sm_100a).
//
// The random streams, the bounded draws, the shuffle permutation and the
// fitness summation order defined here are the contract the CPU oracle
// restates; any change here must be made there too.
#pragma once
#include <cstdint>

namespace hea {

constexpr int kMaxTypes = 6;        // packed 5-bit histogram fields: 6 * 5 = 30 bits
constexpr int kMaxShells = 3;       // pyhea builds three shells (pyhea/lattice/lattice.py:471-475)
constexpr int kMaxShellPad = 28;    // padded shell length must stay below 32 (5-bit fields)
constexpr uint32_t kPhiloxCallsPerDraw = 1u << 19;  // two attempts per call (four with 16-bit draws)
constexpr int kFeistelRounds = 6;
constexpr uint32_t kInitStream = 0xFFFFFFFFu;

// Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3", SC'11).
struct u32x4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}

// Lemire's multiply-and-reject bounded draw: exactly uniform on [0, n) when it accepts.
__device__ __forceinline__ bool bounded_draw(uint32_t x, uint32_t n, uint32_t reject_below, uint32_t &v)
{
    v = __umulhi(x, n);
    return x * n >= reject_below;
}

// The same on a 16-bit word h (n <= 2^16): accept iff low16(h n) >= 2^16 mod n; value high16(h n).
__device__ __forceinline__ bool bounded_draw16(uint32_t h, uint32_t n, uint32_t reject16, uint32_t &v)
{
    const uint32_t m = h * n;
    v = m >> 16;
    return (m & 0xFFFFu) >= reject16;
}

// Whether proposals of a structure of n sites use 16-bit draws (four attempts
// per Philox call): n <= 2^16 and at most 1/16 of the 16-bit words rejected.
__host__ __device__ __forceinline__ bool use_draw16(uint32_t n) { return n <= 65536u && (65536u % n) <= 4096u; }

// murmur3 finaliser, the Feistel round function.
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

__host__ __device__ __forceinline__ uint32_t feistel(uint32_t x, int h, const uint32_t *rk)
{
    const uint32_t mask = (h >= 32) ? 0xFFFFFFFFu : ((1u << h) - 1u);
    uint32_t l = x >> h, r = x & mask;
#pragma unroll
    for (int i = 0; i < kFeistelRounds; ++i) {
        const uint32_t nl = r;
        r = l ^ (fmix32(r ^ rk[i]) & mask);
        l = nl;
    }
    return (l << h) | r;
}

// Half width of the Feistel domain covering [0, n): 2h >= bits(n - 1), h >= 1.
inline int feistel_half_bits(uint32_t n)
{
    int b = 0;
    for (uint32_t m = n > 1 ? n - 1 : 0; m; m >>= 1) ++b;
    if (b < 2) b = 2;
    return (b + 1) / 2;
}

// Device wall clock in nanoseconds (the %globaltimer register).
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace hea
