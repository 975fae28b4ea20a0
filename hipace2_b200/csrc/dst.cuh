// Dirichlet Poisson solver with DST-I written as dense sine-basis GEMMs.
//
// The reference solves Lap(u) = f on the nx x ny interior with homogeneous Dirichlet values one
// cell outside the box by DST-I in x, DST-I in y, division by the 5-point Laplacian eigenvalues
// and the inverse transforms (FFTPoissonSolverDirichletFast.cpp:196-328, FFTW RODFT00 in
// FFTPoissonSolverDirichletDirect). Here each 1-D DST of a batch of rows is one GEMM with the
// symmetric matrix S[k][i] = sin(pi (i+1)(k+1) / (n+1)); the normalisation of the two transforms
// per axis (2/(n+1) each) is folded into the eigenvalues. Several right-hand sides are solved
// together: stage layout is [j][k][i] (row j, right-hand side k, column i), so
//   y-transform:  Y(ny x K*nx)   = Sy(ny x ny) * X(ny x K*nx)
//   x-transform:  Z(K*ny x nx)   = Y(K*ny x nx) * Sx(nx x nx)
// are both plain row-major GEMMs on the same buffer.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "fftdst.cuh"
#include "tcdst.cuh"

namespace hpq {

// C = A * B (+ epilogue). Row-major, arbitrary M, N, K. Tile BM x BN x BK, 256 threads, each
// thread a TM x TN register block.
template <class R, int BM, int BN, int BK, int TM, int TN, class Epi>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const R* __restrict__ A, int lda,
                                              const R* __restrict__ B, int ldb, Epi epi) {
    HPQ_PDL_ENTRY();
    static_assert((BM / TM) * (BN / TN) == 256, "tile/thread mismatch");
    __shared__ R As[BK][BM + 1];
    __shared__ R Bs[BK][BN];
    const int tid = threadIdx.x;
    const int tr = tid / (BN / TN), tc = tid % (BN / TN);
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    R acc[TM][TN];
#pragma unroll
    for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = R(0);
    for (int k0 = 0; k0 < K; k0 += BK) {
        for (int e = tid; e < BM * BK; e += 256) {
            const int r = e / BK, c = e % BK;
            const int gm = m0 + r, gk = k0 + c;
            As[c][r] = (gm < M && gk < K) ? A[(size_t)gm * lda + gk] : R(0);
        }
        for (int e = tid; e < BK * BN; e += 256) {
            const int r = e / BN, c = e % BN;
            const int gk = k0 + r, gn = n0 + c;
            Bs[r][c] = (gk < K && gn < N) ? B[(size_t)gk * ldb + gn] : R(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            R av[TM], bv[TN];
#pragma unroll
            for (int a = 0; a < TM; ++a) av[a] = As[kk][tr * TM + a];
#pragma unroll
            for (int b = 0; b < TN; ++b) bv[b] = Bs[kk][tc + b * (BN / TN)];
#pragma unroll
            for (int a = 0; a < TM; ++a)
#pragma unroll
                for (int b = 0; b < TN; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) {
            const int gm = m0 + tr * TM + a, gn = n0 + tc + b * (BN / TN);
            if (gm < M && gn < N) epi(gm, gn, acc[a][b]);
        }
}

// plain store
template <class R>
struct EpiStore {
    R* C;
    int ldc;
    __device__ void operator()(int m, int n, R v) const { C[(size_t)m * ldc + n] = v; }
};
// store times eigenvalue: rows are (j, k) with K right-hand sides per j
template <class R>
struct EpiEig {
    R* C;
    int ldc, nrhs;
    const R* eig;
    int lde;
    __device__ void operator()(int m, int n, R v) const {
        C[(size_t)m * ldc + n] = v * eig[(size_t)(m / nrhs) * lde + n];
    }
};
// scatter the solution of right-hand side k = n / nx into field component comp[k]
template <class R>
struct EpiField {
    R* base;
    size_t cstride;
    int pitch, nx;
    int comp[4];
    __device__ void operator()(int m, int n, R v) const {
        const int k = n / nx, i = n - k * nx;
        base[(size_t)comp[k] * cstride + (size_t)(m + kGuardAlloc) * pitch + (i + kGuardAlloc)] = v;
    }
};

template <class R>
class PoissonDST {
public:
    int nx = 0, ny = 0, nrhs_max = 0;
    R *sx = nullptr, *sy = nullptr, *eig = nullptr, *stage = nullptr, *work = nullptr;
    R* stage_simt = nullptr;  // the stage of the SIMT-GEMM and FFT forms
    bool use_fft = false, use_tc = false;
    FastDST<R> fast;
    TcDST tcd;  // tensor-core form, single precision only
    double dx_ = 0, dy_ = 0;
    // stage element (rhs k, row j, column i) is stage[k * sk + j * sj + i]
    int sk = 0, sj = 0;
    void set_mode(bool fft) {
        use_tc = false;
        stage = stage_simt;
        use_fft = fft && FastDST<R>::supported(nx, ny);
        if (use_fft) { sk = nx * ny; sj = nx; }
        else { sk = nx; sj = nrhs_max * nx; }
    }
    // tensor-core sine GEMMs (TF32x3, or BF16x3 with bf16) for the single-precision path; err
    // receives the kernels' error code
    void set_tensor_mode(int* err, bool bf16 = false) {
        if constexpr (std::is_same<R, float>::value) {
            if (!TcDST::supported(nx, ny)) return;
            if (tcd.stage && tcd.bf16 != bf16) tcd.release();
            if (!tcd.stage) tcd.init(nx, ny, dx_, dy_, nrhs_max, err, bf16);
            use_tc = true;
            use_fft = false;
            stage = tcd.stage;
            sk = ny * tcd.px;
            sj = tcd.px;
        } else {
            (void)err;
        }
    }

    void init(int nx_, int ny_, double dx, double dy, int nrhs_max_) {
        nx = nx_; ny = ny_; nrhs_max = nrhs_max_;
        dx_ = dx; dy_ = dy;
        std::vector<R> hx((size_t)nx * nx), hy((size_t)ny * ny), he((size_t)nx * ny);
        const double pi = 3.14159265358979323846;
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nx; ++k) hx[(size_t)i * nx + k] = (R)sin(pi * (double)(i + 1) * (k + 1) / (nx + 1));
        for (int i = 0; i < ny; ++i)
            for (int k = 0; k < ny; ++k) hy[(size_t)i * ny + k] = (R)sin(pi * (double)(i + 1) * (k + 1) / (ny + 1));
        const double sxf = pi / (2. * (nx + 1)), syf = pi / (2. * (ny + 1));
        const double norm = (2.0 / (nx + 1)) * (2.0 / (ny + 1));
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double a = sin((i + 1) * sxf), b = sin((j + 1) * syf);
                a *= a; b *= b;
                he[(size_t)j * nx + i] = (R)((a != 0 && b != 0) ? norm / (-4.0 * (a / (dx * dx) + b / (dy * dy))) : 0.0);
            }
        HPQ_CUDA(cudaMalloc(&sx, hx.size() * sizeof(R)));
        HPQ_CUDA(cudaMalloc(&sy, hy.size() * sizeof(R)));
        HPQ_CUDA(cudaMalloc(&eig, he.size() * sizeof(R)));
        HPQ_CUDA(cudaMalloc(&stage_simt, (size_t)nx * ny * nrhs_max * sizeof(R)));
        stage = stage_simt;
        HPQ_CUDA(cudaMalloc(&work, (size_t)nx * ny * nrhs_max * sizeof(R)));
        HPQ_CUDA(cudaMemcpy(sx, hx.data(), hx.size() * sizeof(R), cudaMemcpyHostToDevice));
        HPQ_CUDA(cudaMemcpy(sy, hy.data(), hy.size() * sizeof(R), cudaMemcpyHostToDevice));
        HPQ_CUDA(cudaMemcpy(eig, he.data(), he.size() * sizeof(R), cudaMemcpyHostToDevice));
        if (FastDST<R>::supported(nx, ny)) fast.init(nx, ny);
        set_mode(true);
    }
    void release() {
        for (R* p : {sx, sy, eig, stage_simt, work}) if (p) cudaFree(p);
        sx = sy = eig = stage = stage_simt = work = nullptr;
        fast.release();
        tcd.release();
    }

    template <class Epi>
    static void gemm(cudaStream_t st, int M, int N, int K, const R* A, int lda, const R* B, int ldb, Epi e) {
        constexpr int BM = 64, BN = 64, BK = 16;
        dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
        hpq_launch(k_gemm<R, BM, BN, BK, 4, 4, Epi>, dim3(grid), dim3(256), 0, st, M, N, K, A, lda, B, ldb, e);
        HPQ_LAUNCH_CHECK();
    }

    // Solve for `nrhs` right-hand sides already in `stage` ([j][k][i]); results go to field
    // components comps[k] of the slab (interior only).
    void solve(cudaStream_t st, int nrhs, R* base, size_t cstride, int pitch, const int* comps) {
        if constexpr (std::is_same<R, float>::value) {
            if (use_tc) {
                tcd.solve(st, nrhs, base, cstride, pitch, comps);
                return;
            }
        }
        if (use_fft) {
            fast.solve(st, nrhs, stage, work, eig, base, cstride, pitch, comps);
            return;
        }
        // GEMM path: layout [j][k][i] with nrhs_max planes interleaved per row
        const int W = nrhs * nx;
        if (nrhs != nrhs_max) throw CudaError("GEMM DST expects all right-hand sides");
        // forward: y then x (with eigenvalues)
        gemm(st, ny, W, ny, sy, ny, stage, W, EpiStore<R>{work, W});
        gemm(st, nrhs * ny, nx, nx, work, nx, sx, nx, EpiEig<R>{stage, nx, nrhs, eig, nx});
        // inverse: x then y (scatter to the fields)
        gemm(st, nrhs * ny, nx, nx, stage, nx, sx, nx, EpiStore<R>{work, nx});
        EpiField<R> ef{base, cstride, pitch, nx, {0, 0, 0, 0}};
        for (int k = 0; k < nrhs; ++k) ef.comp[k] = comps[k];
        gemm(st, ny, W, ny, sy, ny, work, W, ef);
    }
};

}  // namespace hpq
