// DST-I through shared-memory FFTs, for grids with 2(n+1) a power of two (n = 31, 63, 127,
// 255, 511, 1023, 2047): the reference's fast Dirichlet solver evaluates the same transforms with
// real-to-complex repacking and cuFFT (FFTPoissonSolverDirichletFast.cpp:34-72, 196-328).
//
// Two real rows a, b (length n) are packed as one complex odd extension of length M = 2(n+1):
//   z[0] = z[n+1] = 0, z[j] = a[j-1] + i b[j-1], z[M-j] = -z[j]   (j = 1..n)
// whose DFT is Z[k] = -2i S(a)[k] + 2 S(b)[k] with S(v)[k] = sum_j v[j-1] sin(pi j k / (n+1)),
// i.e. the DST-I of both rows from one radix-2 FFT. A Poisson solve is three kernels:
//   x-pass (rows along x, transposed write)  ->  y-pass, eigenvalue divide, y-pass (transposed
//   write back)  ->  x-pass with the scatter into the field components.
#pragma once

#include <vector>

#include "common.cuh"

namespace hpq {

template <class R>
struct Cx {
    R re, im;
};

// rows per block by transform length (shared memory: RB/2 complex arrays of M elements); passes
// with fewer than 2 blocks per SM at that size run 2 rows per block instead
template <int M>
struct DstCfg {
    static constexpr int RB = M <= 2048 ? 4 : 2;
};
constexpr int kDstSmallRows = 2 * 148 * 4;  // rows below which a pass uses 2 rows per block

template <class R>
__device__ __forceinline__ Cx<R> cmul(const Cx<R>& v0, const Cx<R>& w) {
    return {v0.re * w.re - v0.im * w.im, v0.re * w.im + v0.im * w.re};
}

// In-place radix-2 DIT FFT of nfft rows of length M held in bit-reversed order. Pairs of
// consecutive radix-2 stages (lengths 2h and 4h) are done by one thread on 4 elements (a
// radix-4 step with the same operations as the two radix-2 stages), so a length-2^k transform
// needs ceil(k/2) block barriers instead of k; stage sizes are compile-time, indices are shifts.
template <class R, int M, int LOGM>
__device__ __forceinline__ void fft_block(Cx<R>* z, int nfft, const Cx<R>* __restrict__ tw) {
    static_assert((1 << LOGM) == M, "M = 2^LOGM");
    int s = 0;  // stage length 2h with h = 2^s
    if (LOGM & 1) {
        for (int t = threadIdx.x; t < nfft * (M / 2); t += blockDim.x) {
            const int f = t >> (LOGM - 1), b = t & (M / 2 - 1);
            Cx<R>* zz = z + f * M;
            const int i0 = 2 * b, i1 = i0 + 1;
            const Cx<R> w = tw[0];
            const Cx<R> u = zz[i0], v = cmul(zz[i1], w);
            zz[i0] = {u.re + v.re, u.im + v.im};
            zz[i1] = {u.re - v.re, u.im - v.im};
        }
        __syncthreads();
        s = 1;
    }
#pragma unroll
    for (int ss = LOGM & 1; ss < LOGM; ss += 2) {
        s = ss;
        const int h = 1 << s;
        for (int t = threadIdx.x; t < nfft * (M / 4); t += blockDim.x) {
            const int f = t >> (LOGM - 2), b = t & (M / 4 - 1);
            const int grp = b >> s, pos = b & (h - 1);
            Cx<R>* zz = z + f * M;
            const int i0 = grp * 4 * h + pos, i1 = i0 + h, i2 = i0 + 2 * h, i3 = i0 + 3 * h;
            const Cx<R> wa = tw[pos * (M / (2 * h))];
            const Cx<R> wb0 = tw[pos * (M / (4 * h))], wb1 = tw[(pos + h) * (M / (4 * h))];
            Cx<R> x0 = zz[i0], x1 = zz[i1], x2 = zz[i2], x3 = zz[i3];
            // stage of length 2h: (i0, i1) and (i2, i3)
            Cx<R> v = cmul(x1, wa);
            x1 = {x0.re - v.re, x0.im - v.im};
            x0 = {x0.re + v.re, x0.im + v.im};
            v = cmul(x3, wa);
            x3 = {x2.re - v.re, x2.im - v.im};
            x2 = {x2.re + v.re, x2.im + v.im};
            // stage of length 4h: (i0, i2) and (i1, i3)
            v = cmul(x2, wb0);
            zz[i2] = {x0.re - v.re, x0.im - v.im};
            zz[i0] = {x0.re + v.re, x0.im + v.im};
            v = cmul(x3, wb1);
            zz[i3] = {x1.re - v.re, x1.im - v.im};
            zz[i1] = {x1.re + v.re, x1.im + v.im};
        }
        __syncthreads();
    }
    (void)s;
}

template <int LOGM>
__device__ __forceinline__ int brev(int j) {
    return (int)(__brev((unsigned)j) >> (32 - LOGM));
}

// odd extension of row values (val(row, e), e in [0, n)) into bit-reversed order
template <class R, int M, int LOGM, class Get>
__device__ __forceinline__ void load_odd(Cx<R>* z, int nfft, int n, Get get) {
    for (int t = threadIdx.x; t < nfft * M; t += blockDim.x) {
        const int f = t / M, j = t - f * M;
        R re = 0, im = 0;
        if (j >= 1 && j <= n) { re = get(2 * f, j - 1); im = get(2 * f + 1, j - 1); }
        else if (j >= n + 2) { re = -get(2 * f, M - j - 1); im = -get(2 * f + 1, M - j - 1); }
        z[f * M + brev<LOGM>(j)] = {re, im};
    }
    __syncthreads();
}

// DST-I value of element e of block row r after the FFT
template <class R, int M>
__device__ __forceinline__ R dst_val(const Cx<R>* z, int r, int e) {
    const Cx<R> v = z[(r >> 1) * M + e + 1];
    return (r & 1) ? v.re * R(0.5) : -v.im * R(0.5);
}

// Pass over rows: out(row, e) = DST-I(in row)[e]; written transposed:
// out[(row / rows_per_plane) * n * rows_per_plane + e * rows_per_plane + row % rows_per_plane]
template <class R, int M, int LOGM, int RB>
__global__ void __launch_bounds__(256) k_dst_pass_t(const R* __restrict__ in, int nrows, int n, int rows_per_plane,
                                                    R* __restrict__ out, const Cx<R>* __restrict__ tw) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    load_odd<R, M, LOGM>(z, RB / 2, n, get);
    fft_block<R, M, LOGM>(z, RB / 2, tw);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t % RB, e = t / RB;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int pl = row / rows_per_plane, rr = row - pl * rows_per_plane;
        out[((size_t)pl * n + e) * rows_per_plane + rr] = dst_val<R, M>(z, r, e);
    }
}

// y-pass, eigenvalue multiply, y-pass; rows are (plane, i) of length n = ny; eig is [j][i] with
// row length nxe; written transposed back to [plane][j][i]
template <class R, int M, int LOGM, int RB>
__global__ void __launch_bounds__(256) k_dst_pass_eig(const R* __restrict__ in, int nrows, int n, int rows_per_plane,
                                                      const R* __restrict__ eig, R* __restrict__ out,
                                                      const Cx<R>* __restrict__ tw) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    R* tmp = reinterpret_cast<R*>(z + (RB / 2) * M);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    load_odd<R, M, LOGM>(z, RB / 2, n, get);
    fft_block<R, M, LOGM>(z, RB / 2, tw);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t / n, e = t - r * n;
        const int row = r0 + r;
        const int i = row % rows_per_plane;
        tmp[t] = row < nrows ? dst_val<R, M>(z, r, e) * eig[(size_t)e * rows_per_plane + i] : R(0);
    }
    __syncthreads();
    auto get2 = [&](int r, int e) -> R { return tmp[r * n + e]; };
    load_odd<R, M, LOGM>(z, RB / 2, n, get2);
    fft_block<R, M, LOGM>(z, RB / 2, tw);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t % RB, e = t / RB;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int pl = row / rows_per_plane, rr = row - pl * rows_per_plane;
        out[((size_t)pl * n + e) * rows_per_plane + rr] = dst_val<R, M>(z, r, e);
    }
}

// final x-pass: rows are (plane k, j) of length nx; result scattered into field component comp[k]
template <class R, int M, int LOGM, int RB>
__global__ void __launch_bounds__(256) k_dst_pass_field(const R* __restrict__ in, int nrows, int n, int ny, R* base,
                                                        size_t cstride, int pitch, int c0, int c1, int c2,
                                                        const Cx<R>* __restrict__ tw) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    load_odd<R, M, LOGM>(z, RB / 2, n, get);
    fft_block<R, M, LOGM>(z, RB / 2, tw);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t / n, e = t - r * n;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int k = row / ny, j = row - k * ny;
        const int comp = k == 0 ? c0 : (k == 1 ? c1 : c2);
        base[(size_t)comp * cstride + (size_t)(j + kGuardAlloc) * pitch + (e + kGuardAlloc)] = dst_val<R, M>(z, r, e);
    }
}

// ------------------------------------------------------------------------------------------
// Any length: Bluestein's chirp-z algorithm (L. Bluestein, "A linear filtering approach to the
// computation of the discrete Fourier transform", 1970). With d_m = exp(-i pi m^2 / M), the DFT of
// the odd extension z (length M = 2(n+1), not a power of two) is
//   Z[k] = d_k sum_j (z_j d_j) conj(d_{k-j}),
// a circular convolution of length L (a power of two >= 2M - 1) done with two radix-2 FFTs of
// length L: the forward one decimated in frequency (natural order in, bit-reversed out), the
// product with B = FFT(conj(d)) held in bit-reversed order, and the inverse through
// conj(FFT(conj(.))) decimated in time (bit-reversed in, natural out). No permutation pass.
// ------------------------------------------------------------------------------------------
template <class R>
struct BluAxis {
    const Cx<R>* d;    // chirp d_m, m < M
    const Cx<R>* B;    // FFT_L of the chirp filter conj(d_|m|), bit-reversed order
    const Cx<R>* tw;   // exp(-2 pi i t / L), t < L/2
    int M;
};

// In-place radix-2 DIF FFT of nfft rows of length L (natural order in, bit-reversed order out)
template <class R, int L, int LOGL>
__device__ __forceinline__ void fft_block_dif(Cx<R>* z, int nfft, const Cx<R>* __restrict__ tw) {
#pragma unroll 1
    for (int s = LOGL - 1; s >= 0; --s) {
        const int h = 1 << s;
        for (int t = threadIdx.x; t < nfft * (L / 2); t += blockDim.x) {
            const int f = t >> (LOGL - 1), b = t & (L / 2 - 1);
            const int grp = b >> s, pos = b & (h - 1);
            Cx<R>* zz = z + f * L;
            const int i0 = grp * 2 * h + pos, i1 = i0 + h;
            const Cx<R> u = zz[i0], v = zz[i1];
            zz[i0] = {u.re + v.re, u.im + v.im};
            zz[i1] = cmul(Cx<R>{u.re - v.re, u.im - v.im}, tw[pos << (LOGL - 1 - s)]);
        }
        __syncthreads();
    }
}

// DFT of the odd extensions of nfft row pairs into z (row f: complex z[f * L + k] such that
// blu_val reads the DST-I); get(r, e) returns element e of block row r
template <class R, int L, int LOGL, class Get>
__device__ __forceinline__ void blu_forward(Cx<R>* z, int nfft, int n, const BluAxis<R>& A, Get get) {
    const int M = A.M;
    for (int t = threadIdx.x; t < nfft * L; t += blockDim.x) {
        const int f = t >> LOGL, j = t & (L - 1);
        Cx<R> v{R(0), R(0)};
        if (j < M) {
            R re = 0, im = 0;
            if (j >= 1 && j <= n) { re = get(2 * f, j - 1); im = get(2 * f + 1, j - 1); }
            else if (j >= n + 2) { re = -get(2 * f, M - j - 1); im = -get(2 * f + 1, M - j - 1); }
            v = cmul(Cx<R>{re, im}, A.d[j]);
        }
        z[t] = v;
    }
    __syncthreads();
    fft_block_dif<R, L, LOGL>(z, nfft, A.tw);
    for (int t = threadIdx.x; t < nfft * L; t += blockDim.x) {
        const Cx<R> p = cmul(z[t], A.B[t & (L - 1)]);
        z[t] = {p.re, -p.im};
    }
    __syncthreads();
    fft_block<R, L, LOGL>(z, nfft, A.tw);
}

// DST-I value of element e of block row r: Z[k] = d_k conj(y[k]) / L at k = e + 1
template <class R, int L>
__device__ __forceinline__ R blu_val(const Cx<R>* z, const BluAxis<R>& A, int r, int e) {
    const Cx<R> y = z[(r >> 1) * L + e + 1];
    const Cx<R> zk = cmul(Cx<R>{y.re, -y.im}, A.d[e + 1]);
    return (r & 1) ? zk.re * (R(0.5) / R(L)) : -zk.im * (R(0.5) / R(L));
}

template <class R, int L, int LOGL, int RB>
__global__ void __launch_bounds__(256) k_dstb_pass_t(const R* __restrict__ in, int nrows, int n, int rows_per_plane,
                                                     R* __restrict__ out, BluAxis<R> A) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    blu_forward<R, L, LOGL>(z, RB / 2, n, A, get);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t % RB, e = t / RB;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int pl = row / rows_per_plane, rr = row - pl * rows_per_plane;
        out[((size_t)pl * n + e) * rows_per_plane + rr] = blu_val<R, L>(z, A, r, e);
    }
}

template <class R, int L, int LOGL, int RB>
__global__ void __launch_bounds__(256) k_dstb_pass_eig(const R* __restrict__ in, int nrows, int n, int rows_per_plane,
                                                       const R* __restrict__ eig, R* __restrict__ out, BluAxis<R> A) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    R* tmp = reinterpret_cast<R*>(z + (RB / 2) * L);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    blu_forward<R, L, LOGL>(z, RB / 2, n, A, get);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t / n, e = t - r * n;
        const int row = r0 + r;
        const int i = row % rows_per_plane;
        tmp[t] = row < nrows ? blu_val<R, L>(z, A, r, e) * eig[(size_t)e * rows_per_plane + i] : R(0);
    }
    __syncthreads();
    auto get2 = [&](int r, int e) -> R { return tmp[r * n + e]; };
    blu_forward<R, L, LOGL>(z, RB / 2, n, A, get2);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t % RB, e = t / RB;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int pl = row / rows_per_plane, rr = row - pl * rows_per_plane;
        out[((size_t)pl * n + e) * rows_per_plane + rr] = blu_val<R, L>(z, A, r, e);
    }
}

template <class R, int L, int LOGL, int RB>
__global__ void __launch_bounds__(256) k_dstb_pass_field(const R* __restrict__ in, int nrows, int n, int ny, R* base,
                                                         size_t cstride, int pitch, int c0, int c1, int c2, BluAxis<R> A) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    Cx<R>* z = reinterpret_cast<Cx<R>*>(smem_raw);
    const int r0 = blockIdx.x * RB;
    auto get = [&](int r, int e) -> R { const int row = r0 + r; return row < nrows ? in[(size_t)row * n + e] : R(0); };
    blu_forward<R, L, LOGL>(z, RB / 2, n, A, get);
    for (int t = threadIdx.x; t < RB * n; t += blockDim.x) {
        const int r = t / n, e = t - r * n;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const int k = row / ny, j = row - k * ny;
        const int comp = k == 0 ? c0 : (k == 1 ? c1 : c2);
        base[(size_t)comp * cstride + (size_t)(j + kGuardAlloc) * pitch + (e + kGuardAlloc)] = blu_val<R, L>(z, A, r, e);
    }
}

// rows per block of a Bluestein pass: the L-point complex rows of the row pairs must fit
template <class R, int L>
struct BluCfg {
    static constexpr int RB = (size_t)2 * L * sizeof(Cx<R>) <= 96 * 1024 ? 4 : 2;
};

template <class R>
class FastDST {
public:
    int nx = 0, ny = 0, Mx = 0, My = 0;  // radix-2 lengths 2(n+1), or 0 on a Bluestein axis
    int Lx = 0, Ly = 0;                  // Bluestein lengths, or 0 on a radix-2 axis
    Cx<R>* twx = nullptr;
    Cx<R>* twy = nullptr;
    BluAxis<R> bx{}, by{};

    static int pow2_len(int n) {
        const int m = 2 * (n + 1);
        return (m >= 64 && m <= 4096 && (m & (m - 1)) == 0) ? m : 0;
    }
    // Bluestein convolution length: the smallest power of two >= 2M - 1, M = 2(n+1); up to n = 2047
    static int blu_len(int n) {
        if (n < 1) return 0;
        const int m = 2 * (n + 1);
        int l = 64;
        while (l < 2 * m - 1) l <<= 1;
        return l <= 8192 ? l : 0;
    }
    static bool axis_ok(int n) { return pow2_len(n) || blu_len(n); }
    static bool supported(int nx, int ny) { return axis_ok(nx) && axis_ok(ny); }
    static bool radix2(int nx, int ny) { return pow2_len(nx) && pow2_len(ny); }

    // chirp, filter spectrum (bit-reversed) and twiddles of a Bluestein axis, from FP64 tables
    static BluAxis<R> blu_axis(int n, int L) {
        const int M = 2 * (n + 1);
        const double pi = 3.14159265358979323846;
        std::vector<double> dre(M), dim(M);
        for (int m = 0; m < M; ++m) {
            const long long q = ((long long)m * m) % (2LL * M);  // d_m = exp(-i pi m^2 / M), m^2 mod 2M exact
            dre[m] = std::cos(pi * (double)q / M);
            dim[m] = -std::sin(pi * (double)q / M);
        }
        // b_m = conj(d_|m|) on the circle of length L, then its DFT (iterative radix 2, FP64)
        std::vector<double> br(L, 0.0), bi(L, 0.0);
        for (int m = 0; m < M; ++m) { br[m] = dre[m]; bi[m] = -dim[m]; }
        for (int m = 1; m < M; ++m) { br[L - m] = dre[m]; bi[L - m] = -dim[m]; }
        int logl = 0;
        while ((1 << logl) < L) ++logl;
        auto rev = [&](int j) {
            int r = 0;
            for (int b = 0; b < logl; ++b) r |= ((j >> b) & 1) << (logl - 1 - b);
            return r;
        };
        for (int j = 0; j < L; ++j) {
            const int r = rev(j);
            if (r > j) { std::swap(br[j], br[r]); std::swap(bi[j], bi[r]); }
        }
        for (int len = 2; len <= L; len <<= 1)
            for (int i0 = 0; i0 < L; i0 += len)
                for (int k = 0; k < len / 2; ++k) {
                    const double c = std::cos(2 * pi * k / len), sn = -std::sin(2 * pi * k / len);
                    const int a = i0 + k, b = a + len / 2;
                    const double vr = br[b] * c - bi[b] * sn, vi = br[b] * sn + bi[b] * c;
                    br[b] = br[a] - vr; bi[b] = bi[a] - vi;
                    br[a] += vr; bi[a] += vi;
                }
        std::vector<Cx<R>> hd(M), hB(L);
        for (int m = 0; m < M; ++m) hd[m] = {(R)dre[m], (R)dim[m]};
        for (int q = 0; q < L; ++q) hB[q] = {(R)br[rev(q)], (R)bi[rev(q)]};  // bit-reversed order
        BluAxis<R> A{};
        Cx<R>*d = nullptr, *B = nullptr;
        HPQ_CUDA(cudaMalloc(&d, M * sizeof(Cx<R>)));
        HPQ_CUDA(cudaMalloc(&B, L * sizeof(Cx<R>)));
        HPQ_CUDA(cudaMemcpy(d, hd.data(), M * sizeof(Cx<R>), cudaMemcpyHostToDevice));
        HPQ_CUDA(cudaMemcpy(B, hB.data(), L * sizeof(Cx<R>), cudaMemcpyHostToDevice));
        A.d = d;
        A.B = B;
        A.tw = twiddles(L);
        A.M = M;
        return A;
    }
    static void free_axis(BluAxis<R>& A) {
        if (A.d) cudaFree(const_cast<Cx<R>*>(A.d));
        if (A.B) cudaFree(const_cast<Cx<R>*>(A.B));
        if (A.tw) cudaFree(const_cast<Cx<R>*>(A.tw));
        A = BluAxis<R>{};
    }

    static Cx<R>* twiddles(int M) {
        std::vector<Cx<R>> h(M / 2);
        const double pi = 3.14159265358979323846;
        for (int k = 0; k < M / 2; ++k) h[k] = {(R)std::cos(2 * pi * k / M), (R)(-std::sin(2 * pi * k / M))};
        Cx<R>* d;
        HPQ_CUDA(cudaMalloc(&d, h.size() * sizeof(Cx<R>)));
        HPQ_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(Cx<R>), cudaMemcpyHostToDevice));
        return d;
    }
    void init(int nx_, int ny_) {
        nx = nx_; ny = ny_;
        Mx = pow2_len(nx); My = pow2_len(ny);
        Lx = Mx ? 0 : blu_len(nx);
        Ly = My ? 0 : blu_len(ny);
        if (!(Mx || Lx) || !(My || Ly)) throw CudaError("FastDST: grid too large for the FFT DST");
        if (Mx) twx = twiddles(Mx); else bx = blu_axis(nx, Lx);
        if (My) twy = twiddles(My); else by = blu_axis(ny, Ly);
        set_attrs<64, 6>(); set_attrs<128, 7>(); set_attrs<256, 8>(); set_attrs<512, 9>();
        set_attrs<1024, 10>(); set_attrs<2048, 11>(); set_attrs<4096, 12>();
        if (Lx || Ly) {
            set_attrs_blu<64, 6>(); set_attrs_blu<128, 7>(); set_attrs_blu<256, 8>(); set_attrs_blu<512, 9>();
            set_attrs_blu<1024, 10>(); set_attrs_blu<2048, 11>(); set_attrs_blu<4096, 12>(); set_attrs_blu<8192, 13>();
        }
    }
    void release() {
        if (twx) cudaFree(twx);
        if (twy) cudaFree(twy);
        twx = twy = nullptr;
        free_axis(bx);
        free_axis(by);
    }
    template <int L, int LOGL>
    static void set_attrs_blu() {
        constexpr int RB = BluCfg<R, L>::RB;
        const int big = 220 * 1024;
        HPQ_CUDA(cudaFuncSetAttribute(k_dstb_pass_t<R, L, LOGL, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        HPQ_CUDA(cudaFuncSetAttribute(k_dstb_pass_eig<R, L, LOGL, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        HPQ_CUDA(cudaFuncSetAttribute(k_dstb_pass_field<R, L, LOGL, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    }
    template <int L>
    static size_t smem_blu() { return (size_t)(BluCfg<R, L>::RB / 2) * L * sizeof(Cx<R>); }
    template <int L, int LOGL>
    void bpass_t(cudaStream_t st, const R* in, int nrows, int n, int rpp, R* out, const BluAxis<R>& A) {
        constexpr int RB = BluCfg<R, L>::RB;
        hpq_launch(k_dstb_pass_t<R, L, LOGL, RB>, dim3((nrows + RB - 1) / RB), dim3(256), smem_blu<L>(), st, in, nrows, n, rpp, out, A);
        HPQ_LAUNCH_CHECK();
    }
    template <int L, int LOGL>
    void bpass_eig(cudaStream_t st, const R* in, int nrows, int n, int rpp, const R* eig, R* out, const BluAxis<R>& A) {
        constexpr int RB = BluCfg<R, L>::RB;
        hpq_launch(k_dstb_pass_eig<R, L, LOGL, RB>, dim3((nrows + RB - 1) / RB), dim3(256),
                   smem_blu<L>() + (size_t)RB * n * sizeof(R), st, in, nrows, n, rpp, eig, out, A);
        HPQ_LAUNCH_CHECK();
    }
    template <int L, int LOGL>
    void bpass_field(cudaStream_t st, const R* in, int nrows, int n, R* base, size_t cs, int pitch, const int* comps,
                     int nrhs, const BluAxis<R>& A) {
        constexpr int RB = BluCfg<R, L>::RB;
        hpq_launch(k_dstb_pass_field<R, L, LOGL, RB>, dim3((nrows + RB - 1) / RB), dim3(256), smem_blu<L>(), st,
                   in, nrows, n, ny, base, cs, pitch, comps[0], nrhs > 1 ? comps[1] : comps[0],
                   nrhs > 2 ? comps[2] : comps[0], A);
        HPQ_LAUNCH_CHECK();
    }
    template <int M, int RB>
    static size_t smem_fft() { return (size_t)(RB / 2) * M * sizeof(Cx<R>); }
    template <int M, int RB>
    static size_t smem_eig(int n) { return smem_fft<M, RB>() + (size_t)RB * n * sizeof(R); }
    template <int M, int LOGM, int RB>
    static void set_attrs_rb() {
        const int big = 200 * 1024;
        HPQ_CUDA(cudaFuncSetAttribute(k_dst_pass_t<R, M, LOGM, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        HPQ_CUDA(cudaFuncSetAttribute(k_dst_pass_eig<R, M, LOGM, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        HPQ_CUDA(cudaFuncSetAttribute(k_dst_pass_field<R, M, LOGM, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    }
    template <int M, int LOGM>
    static void set_attrs() {
        set_attrs_rb<M, LOGM, DstCfg<M>::RB>();
        if (DstCfg<M>::RB != 2) set_attrs_rb<M, LOGM, 2>();
    }

    template <int M, int LOGM, int RB>
    void pass_t_rb(cudaStream_t st, const R* in, int nrows, int n, int rpp, R* out, const Cx<R>* tw) {
        hpq_launch(k_dst_pass_t<R, M, LOGM, RB>, dim3((nrows + RB - 1) / RB), dim3(256), smem_fft<M, RB>(), st, in, nrows, n, rpp, out, tw);
        HPQ_LAUNCH_CHECK();
    }
    template <int M, int LOGM>
    void pass_t(cudaStream_t st, const R* in, int nrows, int n, int rpp, R* out, const Cx<R>* tw) {
        if (nrows < kDstSmallRows) pass_t_rb<M, LOGM, 2>(st, in, nrows, n, rpp, out, tw);
        else pass_t_rb<M, LOGM, DstCfg<M>::RB>(st, in, nrows, n, rpp, out, tw);
    }
    template <int M, int LOGM, int RB>
    void pass_eig_rb(cudaStream_t st, const R* in, int nrows, int n, int rpp, const R* eig, R* out, const Cx<R>* tw) {
        hpq_launch(k_dst_pass_eig<R, M, LOGM, RB>, dim3((nrows + RB - 1) / RB), dim3(256), smem_eig<M, RB>(n), st, in, nrows, n, rpp, eig, out, tw);
        HPQ_LAUNCH_CHECK();
    }
    template <int M, int LOGM>
    void pass_eig(cudaStream_t st, const R* in, int nrows, int n, int rpp, const R* eig, R* out, const Cx<R>* tw) {
        if (nrows < kDstSmallRows) pass_eig_rb<M, LOGM, 2>(st, in, nrows, n, rpp, eig, out, tw);
        else pass_eig_rb<M, LOGM, DstCfg<M>::RB>(st, in, nrows, n, rpp, eig, out, tw);
    }
    template <int M, int LOGM, int RB>
    void pass_field_rb(cudaStream_t st, const R* in, int nrows, int n, R* base, size_t cs, int pitch, const int* comps,
                       int nrhs, const Cx<R>* tw) {
        hpq_launch(k_dst_pass_field<R, M, LOGM, RB>, dim3((nrows + RB - 1) / RB), dim3(256), smem_fft<M, RB>(), st,
            in, nrows, n, ny, base, cs, pitch, comps[0], nrhs > 1 ? comps[1] : comps[0], nrhs > 2 ? comps[2] : comps[0], tw);
        HPQ_LAUNCH_CHECK();
    }
    template <int M, int LOGM>
    void pass_field(cudaStream_t st, const R* in, int nrows, int n, R* base, size_t cs, int pitch, const int* comps,
                    int nrhs, const Cx<R>* tw) {
        if (nrows < kDstSmallRows) pass_field_rb<M, LOGM, 2>(st, in, nrows, n, base, cs, pitch, comps, nrhs, tw);
        else pass_field_rb<M, LOGM, DstCfg<M>::RB>(st, in, nrows, n, base, cs, pitch, comps, nrhs, tw);
    }

#define HPQ_DST_DISPATCH(Mval, CALL)                       \
    switch (Mval) {                                        \
        case 64: CALL(64, 6); break;                       \
        case 128: CALL(128, 7); break;                     \
        case 256: CALL(256, 8); break;                     \
        case 512: CALL(512, 9); break;                     \
        case 1024: CALL(1024, 10); break;                  \
        case 2048: CALL(2048, 11); break;                  \
        case 4096: CALL(4096, 12); break;                  \
        default: throw CudaError("unsupported DST length"); \
    }

#define HPQ_DSTB_DISPATCH(Lval, CALL)                      \
    switch (Lval) {                                        \
        case 64: CALL(64, 6); break;                       \
        case 128: CALL(128, 7); break;                     \
        case 256: CALL(256, 8); break;                     \
        case 512: CALL(512, 9); break;                     \
        case 1024: CALL(1024, 10); break;                  \
        case 2048: CALL(2048, 11); break;                  \
        case 4096: CALL(4096, 12); break;                  \
        case 8192: CALL(8192, 13); break;                  \
        default: throw CudaError("unsupported Bluestein length"); \
    }

    // stage: nrhs planes [k][j][i] (nx contiguous); work: scratch of the same size; eig [j][i]
    void solve(cudaStream_t st, int nrhs, R* stage, R* work, const R* eig, R* base, size_t cs, int pitch,
               const int* comps) {
        if (Mx) {
#define CALL1(M, L) pass_t<M, L>(st, stage, nrhs * ny, nx, ny, work, twx)
            HPQ_DST_DISPATCH(Mx, CALL1)
#undef CALL1
        } else {
#define CALL1(L, G) bpass_t<L, G>(st, stage, nrhs * ny, nx, ny, work, bx)
            HPQ_DSTB_DISPATCH(Lx, CALL1)
#undef CALL1
        }
        if (My) {
#define CALL2(M, L) pass_eig<M, L>(st, work, nrhs * nx, ny, nx, eig, stage, twy)
            HPQ_DST_DISPATCH(My, CALL2)
#undef CALL2
        } else {
#define CALL2(L, G) bpass_eig<L, G>(st, work, nrhs * nx, ny, nx, eig, stage, by)
            HPQ_DSTB_DISPATCH(Ly, CALL2)
#undef CALL2
        }
        if (Mx) {
#define CALL3(M, L) pass_field<M, L>(st, stage, nrhs * ny, nx, base, cs, pitch, comps, nrhs, twx)
            HPQ_DST_DISPATCH(Mx, CALL3)
#undef CALL3
        } else {
#define CALL3(L, G) bpass_field<L, G>(st, stage, nrhs * ny, nx, base, cs, pitch, comps, nrhs, bx)
            HPQ_DSTB_DISPATCH(Lx, CALL3)
#undef CALL3
        }
    }
};

}  // namespace hpq
