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

template <class R>
class FastDST {
public:
    int nx = 0, ny = 0, Mx = 0, My = 0;
    Cx<R>* twx = nullptr;
    Cx<R>* twy = nullptr;

    static int pow2_len(int n) {
        const int m = 2 * (n + 1);
        return (m >= 64 && m <= 4096 && (m & (m - 1)) == 0) ? m : 0;
    }
    static bool supported(int nx, int ny) { return pow2_len(nx) && pow2_len(ny); }

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
        twx = twiddles(Mx);
        twy = twiddles(My);
        set_attrs<64, 6>(); set_attrs<128, 7>(); set_attrs<256, 8>(); set_attrs<512, 9>();
        set_attrs<1024, 10>(); set_attrs<2048, 11>(); set_attrs<4096, 12>();
    }
    void release() {
        if (twx) cudaFree(twx);
        if (twy) cudaFree(twy);
        twx = twy = nullptr;
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

    // stage: nrhs planes [k][j][i] (nx contiguous); work: scratch of the same size; eig [j][i]
    void solve(cudaStream_t st, int nrhs, R* stage, R* work, const R* eig, R* base, size_t cs, int pitch,
               const int* comps) {
#define CALL1(M, L) pass_t<M, L>(st, stage, nrhs * ny, nx, ny, work, twx)
        HPQ_DST_DISPATCH(Mx, CALL1)
#undef CALL1
#define CALL2(M, L) pass_eig<M, L>(st, work, nrhs * nx, ny, nx, eig, stage, twy)
        HPQ_DST_DISPATCH(My, CALL2)
#undef CALL2
#define CALL3(M, L) pass_field<M, L>(st, stage, nrhs * ny, nx, base, cs, pitch, comps, nrhs, twx)
        HPQ_DST_DISPATCH(Mx, CALL3)
#undef CALL3
    }
};

}  // namespace hpq
