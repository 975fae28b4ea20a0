// Counter-based random numbers for seeded initialisation (beams on the host, thermal plasma
// momenta on the device): Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11), uniforms with 53 random bits and Box-Muller normals.
// Counter = (particle index, sub-stream); key = seed. Usable from host and device code.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define HPQ_RNG_HD __host__ __device__
#else
#define HPQ_RNG_HD
#endif

namespace hpq {

class Philox {
public:
    HPQ_RNG_HD explicit Philox(uint64_t seed) : k0_((uint32_t)seed), k1_((uint32_t)(seed >> 32)) {}

    HPQ_RNG_HD void block(uint64_t ctr, uint32_t sub, uint32_t out[4]) const {
        uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), sub, 0x5eedu};
        uint32_t k0 = k0_, k1 = k1_;
        for (int r = 0; r < 10; ++r) {
            const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
            const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
            const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
            const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
            c[0] = hi1 ^ c[1] ^ k0;
            c[1] = lo1;
            c[2] = hi0 ^ c[3] ^ k1;
            c[3] = lo0;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        for (int i = 0; i < 4; ++i) out[i] = c[i];
    }
    // two uniforms in [0, 1) from one block
    HPQ_RNG_HD void uniforms2(uint64_t ctr, uint32_t sub, double u[2]) const {
        uint32_t r[4];
        block(ctr, sub, r);
        u[0] = ((r[0] >> 5) * 67108864.0 + (r[1] >> 6)) * (1.0 / 9007199254740992.0);
        u[1] = ((r[2] >> 5) * 67108864.0 + (r[3] >> 6)) * (1.0 / 9007199254740992.0);
    }
    HPQ_RNG_HD double uniform(uint64_t ctr, uint32_t k) const {
        double u[2];
        uniforms2(ctr, 2 + k, u);
        return u[0];
    }
    // four standard normals (two Box-Muller pairs)
    HPQ_RNG_HD void normals(uint64_t ctr, double out[4]) const {
        for (uint32_t s = 0; s < 2; ++s) {
            double u[2];
            uniforms2(ctr, s, u);
            const double r = ::sqrt(-2.0 * ::log(1.0 - u[0]));
            const double t = 6.283185307179586476925 * u[1];
            out[2 * s] = r * ::cos(t);
            out[2 * s + 1] = r * ::sin(t);
        }
    }

private:
    uint32_t k0_, k1_;
};

// Thermal momentum draw of the plasma (PlasmaParticleContainerInit.cpp:282,
// ParticleUtil.H:113-124: u = u_mean + u_std * N(0, 1) per component). The plasma is created
// anew every step, so the draw has a stream per (species, step): key from the deck's seed and the
// species, counter = (step << 40) | index of the particle in the species' lattice order.
HPQ_RNG_HD inline uint64_t plasma_thermal_seed(uint64_t random_seed, int species) {
    return random_seed * 1000003ull + (uint64_t)species * 7919ull + 424242ull;
}
HPQ_RNG_HD inline void plasma_thermal_u(const Philox& rng, int step, long long i, const double mean[3],
                                        const double stdv[3], double u[3]) {
    double g[4];
    rng.normals(((uint64_t)(uint32_t)step << 40) | (uint64_t)i, g);
    for (int d = 0; d < 3; ++d) u[d] = mean[d] + stdv[d] * g[d];
}

}  // namespace hpq
