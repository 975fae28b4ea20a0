// DST-I Poisson solve of the single-precision path as dense sine-basis GEMMs on the 5th-generation
// tensor cores (tcgen05, accumulators in tensor memory, operands staged by TMA).
//
// Same operator as the FP64 solvers (FFTPoissonSolverDirichletFast.cpp:196-328): DST-I along x and
// y, division by the 5-point Laplacian eigenvalues (normalisation folded in), inverse transforms.
// Each 1-D transform of a batch of rows is D = A * S with S[k][n] = sin(pi (k+1)(n+1) / (n_axis+1)),
// A row-major with the transform axis contiguous. The four GEMMs of a solve of `nrhs` right-hand
// sides (k = right-hand side, i/j = x/y index, P_x/P_y = padded row pitches):
//   G1  stage[k][j][i]  * Sx -> w1[k][i][j]   (transposed store)
//   G2  w1[k][i][j]     * Sy -> w2[k][i][j]   (times the eigenvalue, stored in place order)
//   G3  w2[k][i][j]     * Sy -> w3[k][j][i]   (transposed store)
//   G4  w3[k][j][i]     * Sx -> field k       (scatter into the slice arrays)
// so every GEMM has M = nrhs * n rows, N = K = n, K-major A and B (S is symmetric).
//
// Split precision ("TF32x3"): a = a_hi + a_lo with a_hi = tf32(a), a_lo = tf32(a - a_hi), and
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32. Relative error per product
// ~2^-20, against 2^-11 for a single TF32 product. The S splits are made on the host (from the
// FP64 sines); A is split in shared memory by the converter warps after each TMA load.
//
// Kernel roles (6 warps, one 128 x BN output tile per CTA):
//   warp 4      TMA producer: A tile 128 x 32 and S_hi, S_lo tiles BN x 32 per k-block
//   warps 0-3   split A into hi/lo in place, then the epilogue (TMEM lanes 32w .. 32w+31)
//   warp 5      TMEM allocation and the MMA issue (one thread), 12 MMAs (3 products x K 32/8)
// Pipelines: full[s] (TMA bytes) -> conv[s] (4 converter warps) -> empty[s] (MMA commit).
// Every wait is bounded in time; on a timeout the CTA records an error code, waits for its own
// copies and MMAs, frees its tensor memory and returns.
#pragma once

#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace hpq {
namespace tc {

constexpr int BM = 128;             // tile rows (TMEM lanes)
constexpr int BK = 32;              // fp32 per 128-byte swizzled row
constexpr int kThreads = 192;
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s

enum EpiMode : int { EPI_ROW = 0, EPI_TRANS = 1, EPI_EIG = 2, EPI_FIELD = 3 };

// r = output row, k = r / na (right-hand side), a = r % na, n = output column (< nb)
struct Epi {
    int mode;
    float* out;
    int ldo;
    int na, nb;
    const float* eigT;  // EPI_EIG: eigT[a * lde + n]
    int lde;
    float* base;        // EPI_FIELD: base[comp[k] * cstride + (a + G) * pitch + (n + G)]
    size_t cstride;
    int pitch;
    int comp[4];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait until the phase of parity `parity` has completed. Gives up (false) after kWaitNs, or at
// once when another role of the CTA has raised `abort`.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
    if (mbar_test(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_test(b, parity)) return true;
        if (abort && *abort) return false;
        if (global_ns() - t0 > kWaitNs) return false;
        __nanosleep(20);
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major operand in the 128-byte swizzle: 8-row groups 1024 bytes apart (SBO), version 1
// (tcgen05), layout type 2 (SWIZZLE_128B). The tile base is 1024-byte aligned; the k-th MMA of a
// 32-float row starts 32 * k bytes further.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor: D f32, A and B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive 32-bit columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// round to the nearest tf32 (10 explicit mantissa bits), ties away from zero
__host__ __device__ __forceinline__ uint32_t tf32_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }


// one row's 16 consecutive output columns nb0 .. nb0+15 of a tile, through the epilogue mode
__device__ __forceinline__ void epilogue16(const Epi& epi, int r, int k, int a, int nb0, float (&v)[16]) {
    if (epi.mode == EPI_ROW || epi.mode == EPI_EIG) {
        if (epi.mode == EPI_EIG) {
            const float* e = epi.eigT + (size_t)a * epi.lde + nb0;
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (nb0 + q < epi.nb) v[q] *= e[q];
        }
        float* o = epi.out + (size_t)r * epi.ldo + nb0;
        if (nb0 + 16 <= epi.nb) {
#pragma unroll
            for (int q = 0; q < 16; q += 4)
                *reinterpret_cast<float4*>(o + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if (nb0 + q < epi.nb) o[q] = v[q];
        }
    } else if (epi.mode == EPI_TRANS) {
        float* o = epi.out + ((size_t)k * epi.nb + nb0) * epi.ldo + a;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (nb0 + q < epi.nb) o[(size_t)q * epi.ldo] = v[q];
    } else {
        float* o = epi.base + (size_t)epi.comp[k] * epi.cstride + (size_t)(a + kGuardAlloc) * epi.pitch +
                   kGuardAlloc + nb0;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (nb0 + q < epi.nb) o[q] = v[q];
    }
}

template <int BN, int ST>
struct Smem {
    static constexpr int A_BYTES = BM * BK * 4;
    static constexpr int B_BYTES = BN * BK * 4;
    static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;  // A_hi, A_lo, S_hi, S_lo
    static constexpr int BAR_OFF = ST * STAGE;
    static constexpr int NBAR = 3 * ST + 2;                  // full, conv, empty, accf, spare
    static constexpr int TOTAL = BAR_OFF + 8 * NBAR + 16 + 1024;  // + tmem slot, abort flag, alignment
};

__device__ __forceinline__ uint32_t split_hi(uint32_t b) { return tf32_bits(b); }
__device__ __forceinline__ uint32_t split_lo(uint32_t b, uint32_t hi) {
    return tf32_bits(__float_as_uint(__uint_as_float(b) - __uint_as_float(hi)));
}

template <int BN, int ST>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mBh,
              const __grid_constant__ CUtensorMap mBl, int M, int num_kb, Epi epi, int* err) {
    HPQ_PDL_ENTRY();
    using L = Smem<BN, ST>;
    extern __shared__ unsigned char smem_dyn[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + L::BAR_OFF);
    uint64_t* conv = full + ST;
    uint64_t* empty = conv + ST;
    uint64_t* accf = empty + ST;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + L::NBAR);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(full + s, 1);
            mbar_init(conv + s, 4);
            mbar_init(empty + s, 1);
        }
        mbar_init(accf, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    auto raise = [&](int code) {
        *abort = 1;
        atomicExch(err, code);
    };

    if (warp == 4) {
        // ---------------- TMA producer
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < num_kb; ++kb) {
                const int s = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (kb >= ST && !mbar_wait(empty + s, ph ^ 1u, abort)) {
                    if (!*abort) raise(1);
                    break;
                }
                unsigned char* st = sm + s * L::STAGE;
                mbar_expect_tx(full + s, (uint32_t)(L::A_BYTES + 2 * L::B_BYTES));
                tma_load_2d(st, &mA, full + s, kb * BK, m0);
                tma_load_2d(st + 2 * L::A_BYTES, &mBh, full + s, kb * BK, n0);
                tma_load_2d(st + 2 * L::A_BYTES + L::B_BYTES, &mBl, full + s, kb * BK, n0);
                issued = kb + 1;
            }
            // the last copy into each stage has landed before the CTA may leave
            for (int kb = (issued > ST ? issued - ST : 0); kb < issued; ++kb)
                mbar_wait(full + kb % ST, (uint32_t)(kb / ST) & 1u, nullptr);
        }
    } else if (warp == 5) {
        // ---------------- MMA issue (one thread)
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_tf32(BM, BN);
            for (int kb = 0; kb < num_kb; ++kb) {
                const int s = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (!mbar_wait(conv + s, ph, abort)) {
                    if (!*abort) raise(2);
                    break;
                }
                tc_fence_after();
                const uint32_t ah = smem_u32(sm + s * L::STAGE);
                const uint32_t al = ah + L::A_BYTES;
                const uint32_t bh = ah + 2 * L::A_BYTES;
                const uint32_t bl = bh + L::B_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK / 8; ++kk) {
                    const uint32_t o = 32u * kk;
                    mma_tf32(tmem, desc_sw128(ah + o), desc_sw128(bh + o), idesc, (kb | kk) != 0 ? 1u : 0u);
                    mma_tf32(tmem, desc_sw128(ah + o), desc_sw128(bl + o), idesc, 1u);
                    mma_tf32(tmem, desc_sw128(al + o), desc_sw128(bh + o), idesc, 1u);
                }
                mma_commit(empty + s);
            }
            mma_commit(accf);  // arrives once every MMA issued above has completed
        }
    } else {
        // ---------------- warps 0-3: split A into tf32 hi/lo in place, then the epilogue
        bool ok = true;
        for (int kb = 0; kb < num_kb && ok; ++kb) {
            const int s = kb % ST;
            const uint32_t ph = (uint32_t)(kb / ST) & 1u;
            ok = mbar_wait(full + s, ph, abort);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0 && !*abort) raise(3);
                ok = false;
                break;
            }
            uint4* h = reinterpret_cast<uint4*>(sm + s * L::STAGE);
            uint4* l = reinterpret_cast<uint4*>(sm + s * L::STAGE + L::A_BYTES);
#pragma unroll 4
            for (int e = threadIdx.x; e < L::A_BYTES / 16; e += 128) {
                const uint4 v = h[e];
                uint4 hi, lo;
                hi.x = split_hi(v.x); lo.x = split_lo(v.x, hi.x);
                hi.y = split_hi(v.y); lo.y = split_lo(v.y, hi.y);
                hi.z = split_hi(v.z); lo.z = split_lo(v.z, hi.z);
                hi.w = split_hi(v.w); lo.w = split_lo(v.w, hi.w);
                h[e] = hi;
                l[e] = lo;
            }
            // generic-proxy writes become visible to the tensor core's reads
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(conv + s);
        }
        if (ok) {
            ok = mbar_wait(accf, 0, abort);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0 && !*abort) raise(4);
                ok = false;
            }
        }
        if (ok) {
            tc_fence_after();
            const int r = m0 + warp * 32 + lane;
            const bool rv = r < M;
            const int k = rv ? r / epi.na : 0, a = rv ? r - k * epi.na : 0;
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
                if (!rv) continue;
                epilogue16(epi, r, k, a, n0 + c, v);
            }
        }
    }
    // ---------------- teardown: every MMA has completed before the tensor memory is freed
    if (warp == 5 && lane == 0) mbar_wait(accf, 0, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
    }
}

// ------------------------------------------------------------------------------------------
// BF16x3 variant of the same GEMM: a = a_hi + a_lo with a_hi = bf16(a), a_lo = bf16(a - a_hi),
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32 by tcgen05.mma kind::f16 (both
// operands bf16). A k-block is 64 elements: two FP32 TMA boxes of 128 x 32 land in shared memory
// and the converter warps write the bf16 hi and lo tiles (128 x 64, one 128-byte row per tile
// row, in the same 128-byte swizzle: 16-byte chunk c of row r at chunk c ^ (r % 8)); B hi/lo are
// bf16 on the host and arrive by TMA. 4 MMAs of K = 16 per product and k-block.
// Relative error per product ~2^-16 (TF32x3: ~2^-20), at twice the tensor rate of TF32.
// ------------------------------------------------------------------------------------------
constexpr int BK16 = 64;  // bf16 per 128-byte swizzled row

// instruction descriptor: D f32, A and B bf16 (kind::f16), both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// round-to-nearest-even bf16 of an fp32 bit pattern (finite inputs)
__host__ __device__ __forceinline__ uint32_t bf16_bits(uint32_t b) { return (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16; }
__device__ __forceinline__ uint32_t bf16_hi_lo(float a, uint32_t& lo) {
    const uint32_t h = bf16_bits(__float_as_uint(a));
    const float r = a - __uint_as_float(h << 16);
    lo = bf16_bits(__float_as_uint(r));
    return h;
}

template <int BN, int ST>
struct Smem16 {
    static constexpr int F_BYTES = BM * 32 * 4;                    // one fp32 TMA box (128 x 32)
    static constexpr int A_BYTES = BM * BK16 * 2;                  // one bf16 A tile (128 x 64)
    static constexpr int B_BYTES = BN * BK16 * 2;                  // one bf16 B tile
    static constexpr int STAGE = 2 * F_BYTES + 2 * A_BYTES + 2 * B_BYTES;  // F0, F1, A_hi, A_lo, B_hi, B_lo
    static constexpr int BAR_OFF = ST * STAGE;
    static constexpr int NBAR = 3 * ST + 2;
    static constexpr int TOTAL = BAR_OFF + 8 * NBAR + 16 + 1024;
};

template <int BN, int ST>
__global__ void __launch_bounds__(kThreads, 1)
    k_tc_gemm_bf16(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mBh,
                   const __grid_constant__ CUtensorMap mBl, int M, int num_kb, Epi epi, int* err) {
    HPQ_PDL_ENTRY();
    using L = Smem16<BN, ST>;
    extern __shared__ unsigned char smem_dyn[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + L::BAR_OFF);
    uint64_t* conv = full + ST;
    uint64_t* empty = conv + ST;
    uint64_t* accf = empty + ST;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + L::NBAR);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(full + s, 1);
            mbar_init(conv + s, 4);
            mbar_init(empty + s, 1);
        }
        mbar_init(accf, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    auto raise = [&](int code) {
        *abort = 1;
        atomicExch(err, code);
    };

    if (warp == 4) {
        // ---------------- TMA producer: two fp32 boxes of A, the bf16 B hi/lo tiles
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < num_kb; ++kb) {
                const int s = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (kb >= ST && !mbar_wait(empty + s, ph ^ 1u, abort)) {
                    if (!*abort) raise(11);
                    break;
                }
                unsigned char* st = sm + s * L::STAGE;
                mbar_expect_tx(full + s, (uint32_t)(2 * L::F_BYTES + 2 * L::B_BYTES));
                tma_load_2d(st, &mA, full + s, kb * BK16, m0);
                tma_load_2d(st + L::F_BYTES, &mA, full + s, kb * BK16 + 32, m0);
                unsigned char* bst = st + 2 * L::F_BYTES + 2 * L::A_BYTES;
                tma_load_2d(bst, &mBh, full + s, kb * BK16, n0);
                tma_load_2d(bst + L::B_BYTES, &mBl, full + s, kb * BK16, n0);
                issued = kb + 1;
            }
            for (int kb = (issued > ST ? issued - ST : 0); kb < issued; ++kb)
                mbar_wait(full + kb % ST, (uint32_t)(kb / ST) & 1u, nullptr);
        }
    } else if (warp == 5) {
        // ---------------- MMA issue (one thread)
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(BM, BN);
            for (int kb = 0; kb < num_kb; ++kb) {
                const int s = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (!mbar_wait(conv + s, ph, abort)) {
                    if (!*abort) raise(12);
                    break;
                }
                tc_fence_after();
                const uint32_t ah = smem_u32(sm + s * L::STAGE + 2 * L::F_BYTES);
                const uint32_t al = ah + L::A_BYTES;
                const uint32_t bh = ah + 2 * L::A_BYTES;
                const uint32_t bl = bh + L::B_BYTES;
#pragma unroll
                for (int kk = 0; kk < BK16 / 16; ++kk) {
                    const uint32_t o = 32u * kk;
                    mma_bf16(tmem, desc_sw128(ah + o), desc_sw128(bh + o), idesc, (kb | kk) != 0 ? 1u : 0u);
                    mma_bf16(tmem, desc_sw128(ah + o), desc_sw128(bl + o), idesc, 1u);
                    mma_bf16(tmem, desc_sw128(al + o), desc_sw128(bh + o), idesc, 1u);
                }
                mma_commit(empty + s);
            }
            mma_commit(accf);
        }
    } else {
        // ---------------- warps 0-3: fp32 boxes -> bf16 hi/lo tiles, then the epilogue
        bool ok = true;
        for (int kb = 0; kb < num_kb && ok; ++kb) {
            const int s = kb % ST;
            const uint32_t ph = (uint32_t)(kb / ST) & 1u;
            ok = mbar_wait(full + s, ph, abort);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0 && !*abort) raise(13);
                ok = false;
                break;
            }
            const unsigned char* f = sm + s * L::STAGE;
            unsigned char* hi = sm + s * L::STAGE + 2 * L::F_BYTES;
            unsigned char* lo = hi + L::A_BYTES;
            // output chunk (r, c): bf16 k = 8c .. 8c+7 of row r, from fp32 box c / 4, fp32 chunks
            // 2 (c % 4) and 2 (c % 4) + 1 of that row
#pragma unroll 2
            for (int e = threadIdx.x; e < BM * 8; e += 128) {
                const int r = e >> 3, c = e & 7;
                const int sw = r & 7;
                const unsigned char* box = f + (c >> 2) * L::F_BYTES + r * 128;
                const int q0 = 2 * (c & 3);
                const float4 v0 = *reinterpret_cast<const float4*>(box + ((q0 ^ sw) << 4));
                const float4 v1 = *reinterpret_cast<const float4*>(box + (((q0 + 1) ^ sw) << 4));
                const float a[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
                uint32_t h[8], l[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) h[t] = bf16_hi_lo(a[t], l[t]);
                const uint4 hv = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
                const uint4 lv = make_uint4(l[0] | (l[1] << 16), l[2] | (l[3] << 16), l[4] | (l[5] << 16), l[6] | (l[7] << 16));
                *reinterpret_cast<uint4*>(hi + r * 128 + ((c ^ sw) << 4)) = hv;
                *reinterpret_cast<uint4*>(lo + r * 128 + ((c ^ sw) << 4)) = lv;
            }
            // generic-proxy writes become visible to the tensor core's reads; the MMA waits for
            // the arrivals of all four converter warps
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(conv + s);
        }
        if (ok) {
            ok = mbar_wait(accf, 0, abort);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0 && !*abort) raise(14);
                ok = false;
            }
        }
        if (ok) {
            tc_fence_after();
            const int r = m0 + warp * 32 + lane;
            const bool rv = r < M;
            const int k = rv ? r / epi.na : 0, a = rv ? r - k * epi.na : 0;
#pragma unroll 1
            for (int c = 0; c < BN; c += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
                if (!rv) continue;
                epilogue16(epi, r, k, a, n0 + c, v);
            }
        }
    }
    if (warp == 5 && lane == 0) mbar_wait(accf, 0, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
    }
}


inline float host_tf32(double x) {
    float f = (float)x;
    uint32_t b;
    std::memcpy(&b, &f, 4);
    b = tf32_bits(b);
    std::memcpy(&f, &b, 4);
    return f;
}

// bf16 of a double, rounded to nearest even through fp32
inline uint16_t host_bf16(double x) {
    const float f = (float)x;
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return (uint16_t)bf16_bits(b);
}
inline double bf16_value(uint16_t h) {
    const uint32_t b = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        HPQ_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) throw CudaError("cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// row-major fp32 matrix `rows` x `inner` (inner = row pitch, a multiple of 4), tiles of
// box_rows x 32 in the 128-byte swizzle; reads outside the matrix return zeros
inline CUtensorMap make_map(const float* ptr, int inner, int rows, int box_rows) {
    if (inner % 4 || (reinterpret_cast<uintptr_t>(ptr) & 15)) throw CudaError("tensor map: unaligned operand");
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode_tiled()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), dims, strides,
                                      box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

// row-major bf16 matrix `rows` x `inner` (inner = row pitch, a multiple of 8), tiles of
// box_rows x 64 in the 128-byte swizzle; reads outside the matrix return zeros
inline CUtensorMap make_map16(const uint16_t* ptr, int inner, int rows, int box_rows) {
    if (inner % 8 || (reinterpret_cast<uintptr_t>(ptr) & 15)) throw CudaError("tensor map: unaligned operand");
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(uint16_t)};
    const cuuint32_t box[2] = {(cuuint32_t)BK16, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode_tiled()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t*>(ptr), dims,
                                      strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace tc

// Host side of the tensor-core DST solve (single precision). Buffers: stage [k][j][i] (pitch px),
// w1/w2 [k][i][j] (pitch py), w3 [k][j][i] (pitch px); pitches are padded to multiples of 4 floats
// (16-byte TMA strides) and the padding stays zero, as do the sine rows beyond n.
class TcDST {
public:
    int nx = 0, ny = 0, nrhs = 0, px = 0, py = 0;
    float *stage = nullptr, *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    float *sxh = nullptr, *sxl = nullptr, *syh = nullptr, *syl = nullptr, *eigT = nullptr;
    int* err = nullptr;  // device error code of the last failing CTA (0 = none)
    CUtensorMap m_stage{}, m_w1{}, m_w2{}, m_w3{}, m_sxh{}, m_sxl{}, m_syh{}, m_syl{};
    int bn = 128;
    // BF16x3 form (kind::f16 MMAs on bf16 hi/lo splits): the sines are bf16 tables with row
    // pitches padded to multiples of 8 (16-byte TMA strides)
    bool bf16 = false;
    uint16_t *bxh = nullptr, *bxl = nullptr, *byh = nullptr, *byl = nullptr;

    static bool supported(int nx, int ny) { return nx >= 16 && ny >= 16; }

    void init(int nx_, int ny_, double dx, double dy, int nrhs_, int* err_dev, bool bf16_ = false) {
        nx = nx_; ny = ny_; nrhs = nrhs_; err = err_dev; bf16 = bf16_;
        px = (nx + 3) & ~3;
        py = (ny + 3) & ~3;
        const double pi = 3.14159265358979323846;
        auto sine = [&](int n, int p, std::vector<float>& hi, std::vector<float>& lo) {
            hi.assign((size_t)p * p, 0.f);
            lo.assign((size_t)p * p, 0.f);
            for (int a = 0; a < n; ++a)
                for (int b = 0; b < n; ++b) {
                    const double v = sin(pi * (double)(a + 1) * (b + 1) / (n + 1));
                    const float h = tc::host_tf32(v);
                    hi[(size_t)a * p + b] = h;
                    lo[(size_t)a * p + b] = tc::host_tf32(v - (double)h);
                }
        };
        auto sine16 = [&](int n, int p, std::vector<uint16_t>& hi, std::vector<uint16_t>& lo) {
            hi.assign((size_t)p * p, 0);
            lo.assign((size_t)p * p, 0);
            for (int a = 0; a < n; ++a)
                for (int b = 0; b < n; ++b) {
                    const double v = sin(pi * (double)(a + 1) * (b + 1) / (n + 1));
                    const uint16_t h = tc::host_bf16(v);
                    hi[(size_t)a * p + b] = h;
                    lo[(size_t)a * p + b] = tc::host_bf16(v - tc::bf16_value(h));
                }
        };
        std::vector<float> hxh, hxl, hyh, hyl;
        if (!bf16) {
            sine(nx, px, hxh, hxl);
            sine(ny, py, hyh, hyl);
        }
        std::vector<float> he((size_t)nx * py, 0.f);
        const double sxf = pi / (2. * (nx + 1)), syf = pi / (2. * (ny + 1));
        const double norm = (2.0 / (nx + 1)) * (2.0 / (ny + 1));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                double a = sin((i + 1) * sxf), b = sin((j + 1) * syf);
                a *= a; b *= b;
                he[(size_t)i * py + j] = (float)(norm / (-4.0 * (a / (dx * dx) + b / (dy * dy))));
            }
        auto upload = [&](float*& d, const std::vector<float>& h) {
            HPQ_CUDA(cudaMalloc(&d, h.size() * sizeof(float)));
            HPQ_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
        };
        upload(eigT, he);
        if (!bf16) {
            upload(sxh, hxh); upload(sxl, hxl); upload(syh, hyh); upload(syl, hyl);
        } else {
            const int qx = (nx + 7) & ~7, qy = (ny + 7) & ~7;
            auto upload16 = [&](uint16_t*& d, const std::vector<uint16_t>& h) {
                HPQ_CUDA(cudaMalloc(&d, h.size() * sizeof(uint16_t)));
                HPQ_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
            };
            std::vector<uint16_t> h, l;
            sine16(nx, qx, h, l); upload16(bxh, h); upload16(bxl, l);
            sine16(ny, qy, h, l); upload16(byh, h); upload16(byl, l);
        }
        auto zeros = [&](float*& d, size_t n) {
            HPQ_CUDA(cudaMalloc(&d, n * sizeof(float)));
            HPQ_CUDA(cudaMemset(d, 0, n * sizeof(float)));
        };
        zeros(stage, (size_t)nrhs * ny * px);
        zeros(w1, (size_t)nrhs * nx * py);
        zeros(w2, (size_t)nrhs * nx * py);
        zeros(w3, (size_t)nrhs * ny * px);
        // the smallest grid decides the tile width: 128 columns once it fills the GPU
        int dev = 0, sms = 148;
        HPQ_CUDA(cudaGetDevice(&dev));
        HPQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int mt = (nrhs * std::min(nx, ny) + tc::BM - 1) / tc::BM;
        bn = (mt * ((std::min(nx, ny) + 127) / 128) >= sms) ? 128 : 64;
        m_stage = tc::make_map(stage, px, nrhs * ny, tc::BM);
        m_w1 = tc::make_map(w1, py, nrhs * nx, tc::BM);
        m_w2 = tc::make_map(w2, py, nrhs * nx, tc::BM);
        m_w3 = tc::make_map(w3, px, nrhs * ny, tc::BM);
        if (!bf16) {
            m_sxh = tc::make_map(sxh, px, px, bn);
            m_sxl = tc::make_map(sxl, px, px, bn);
            m_syh = tc::make_map(syh, py, py, bn);
            m_syl = tc::make_map(syl, py, py, bn);
            set_attrs<128, 3>();
            set_attrs<64, 4>();
        } else {
            const int qx = (nx + 7) & ~7, qy = (ny + 7) & ~7;
            m_sxh = tc::make_map16(bxh, qx, qx, bn);
            m_sxl = tc::make_map16(bxl, qx, qx, bn);
            m_syh = tc::make_map16(byh, qy, qy, bn);
            m_syl = tc::make_map16(byl, qy, qy, bn);
            set_attrs16<128, 2>();
            set_attrs16<64, 2>();
        }
    }
    void release() {
        for (float* p : {stage, w1, w2, w3, sxh, sxl, syh, syl, eigT}) if (p) cudaFree(p);
        for (uint16_t* p : {bxh, bxl, byh, byl}) if (p) cudaFree(p);
        stage = w1 = w2 = w3 = sxh = sxl = syh = syl = eigT = nullptr;
        bxh = bxl = byh = byl = nullptr;
    }
    template <int BN, int ST>
    static void set_attrs16() {
        static bool done = false;
        if (done) return;
        HPQ_CUDA(cudaFuncSetAttribute(tc::k_tc_gemm_bf16<BN, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      tc::Smem16<BN, ST>::TOTAL));
        done = true;
    }

    template <int BN, int ST>
    static void set_attrs() {
        static bool done = false;
        if (done) return;
        HPQ_CUDA(cudaFuncSetAttribute(tc::k_tc_gemm<BN, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      tc::Smem<BN, ST>::TOTAL));
        done = true;
    }

    void gemm(cudaStream_t st, const CUtensorMap& a, const CUtensorMap& bh, const CUtensorMap& bl, int M, int N, int K,
              const tc::Epi& e) {
        if (bf16) {
            const int nkb = (K + tc::BK16 - 1) / tc::BK16;
            if (bn == 128) {
                dim3 grid((M + tc::BM - 1) / tc::BM, (N + 127) / 128);
                hpq_launch(tc::k_tc_gemm_bf16<128, 2>, grid, dim3(tc::kThreads), (size_t)tc::Smem16<128, 2>::TOTAL, st,
                           a, bh, bl, M, nkb, e, err);
            } else {
                dim3 grid((M + tc::BM - 1) / tc::BM, (N + 63) / 64);
                hpq_launch(tc::k_tc_gemm_bf16<64, 2>, grid, dim3(tc::kThreads), (size_t)tc::Smem16<64, 2>::TOTAL, st,
                           a, bh, bl, M, nkb, e, err);
            }
            HPQ_LAUNCH_CHECK();
            return;
        }
        const int nkb = (K + tc::BK - 1) / tc::BK;
        if (bn == 128) {
            dim3 grid((M + tc::BM - 1) / tc::BM, (N + 127) / 128);
            hpq_launch(tc::k_tc_gemm<128, 3>, grid, dim3(tc::kThreads), (size_t)tc::Smem<128, 3>::TOTAL, st, a, bh, bl, M,
                       nkb, e, err);
        } else {
            dim3 grid((M + tc::BM - 1) / tc::BM, (N + 63) / 64);
            hpq_launch(tc::k_tc_gemm<64, 4>, grid, dim3(tc::kThreads), (size_t)tc::Smem<64, 4>::TOTAL, st, a, bh, bl, M,
                       nkb, e, err);
        }
        HPQ_LAUNCH_CHECK();
    }

    // `n` right-hand sides in stage (element (k, j, i) at stage[(k * ny + j) * px + i]); solutions
    // into the interiors of field components comps[k] of the slice arrays
    void solve(cudaStream_t st, int n, float* base, size_t cstride, int pitch, const int* comps) {
        tc::Epi e{};
        // G1: rows (k, j), x-transform, stored as w1[(k * nx + i) * py + j]
        e.mode = tc::EPI_TRANS; e.out = w1; e.ldo = py; e.na = ny; e.nb = nx;
        gemm(st, m_stage, m_sxh, m_sxl, n * ny, nx, nx, e);
        // G2: rows (k, i), y-transform, times the eigenvalue
        e = tc::Epi{};
        e.mode = tc::EPI_EIG; e.out = w2; e.ldo = py; e.na = nx; e.nb = ny; e.eigT = eigT; e.lde = py;
        gemm(st, m_w1, m_syh, m_syl, n * nx, ny, ny, e);
        // G3: rows (k, i), inverse y-transform, stored as w3[(k * ny + j) * px + i]
        e = tc::Epi{};
        e.mode = tc::EPI_TRANS; e.out = w3; e.ldo = px; e.na = nx; e.nb = ny;
        gemm(st, m_w2, m_syh, m_syl, n * nx, ny, ny, e);
        // G4: rows (k, j), inverse x-transform into the fields
        e = tc::Epi{};
        e.mode = tc::EPI_FIELD; e.na = ny; e.nb = nx; e.base = base; e.cstride = cstride; e.pitch = pitch;
        for (int k = 0; k < n; ++k) e.comp[k] = comps[k];
        gemm(st, m_w3, m_sxh, m_sxl, n * ny, nx, nx, e);
    }
};

}  // namespace hpq
