// Counter-based Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11) and Box-Muller normals in FP64.
//
// A thermal field value is a pure function of (seed, member, noise index, cell,
// component): the stochastic integrators regenerate the previous step's field
// instead of storing it, and every ensemble member has its own stream.
#pragma once
#include <cstdint>

namespace mafb {

struct Philox4 {
    uint32_t v[4];
};

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// 10 rounds of Philox-4x32 on counter c with key k (constants from the paper)
__host__ __device__ __forceinline__ Philox4 philox4x32_10(Philox4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(M0, c.v[0], hi0, lo0);
        mulhilo32(M1, c.v[2], hi1, lo1);
        Philox4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform in (0, 1] from 64 random bits, 53-bit resolution
__host__ __device__ __forceinline__ double u01_53(uint32_t hi, uint32_t lo) {
    const uint64_t x = ((uint64_t)hi << 21) ^ (uint64_t)(lo >> 11);  // 53 bits
    return ((double)(x & ((1ull << 53) - 1)) + 1.0) * (1.0 / 9007199254740992.0);
}

// Three standard normals for (cell, noise index) of one stream:
// counter = (cell lo, cell hi, index lo, index hi), key = (seed lo ^ member, seed hi).
__device__ __forceinline__ void normal3(uint64_t seed, uint32_t member, uint64_t index, uint64_t cell, double out[3]) {
    Philox4 c;
    c.v[0] = (uint32_t)cell;
    c.v[1] = (uint32_t)(cell >> 32);
    c.v[2] = (uint32_t)index;
    c.v[3] = (uint32_t)(index >> 32);
    const uint32_t k0 = (uint32_t)seed ^ (member * 0x9E3779B9u);
    const uint32_t k1 = (uint32_t)(seed >> 32);
    const Philox4 r = philox4x32_10(c, k0, k1);
    c.v[1] ^= 0x80000000u;  // second, independent block for the third normal
    const Philox4 s = philox4x32_10(c, k0, k1);
    const double u1 = u01_53(r.v[0], r.v[1]);
    const double u2 = u01_53(r.v[2], r.v[3]);
    const double u3 = u01_53(s.v[0], s.v[1]);
    const double u4 = u01_53(s.v[2], s.v[3]);
    const double r1 = sqrt(-2.0 * log(u1));
    const double r2 = sqrt(-2.0 * log(u3));
    double s1, c1, s2, c2;
    sincospi(2.0 * u2, &s1, &c1);
    sincospi(2.0 * u4, &s2, &c2);
    out[0] = r1 * c1;
    out[1] = r1 * s1;
    out[2] = r2 * c2;
}

}  // namespace mafb
