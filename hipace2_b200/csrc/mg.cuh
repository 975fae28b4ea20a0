// Geometric multigrid for the explicit Bx/By equation  -chi*B + Lap(B) = S  (two components
// sharing one coefficient), homogeneous Dirichlet boundaries. Restates hpmg::MultiGrid system
// type 1 (mg_solver/HpMultiGrid.cpp):
//   * levels: cell-centred when n is even (Dirichlet on the cell face with the 4/3 closure,
//     :162-183, 265-294), node-centred otherwise (Dirichlet on the first guard node) (:1043-1100)
//   * smoother: 4 red-black Gauss-Seidel colour sweeps, optionally followed by the residual,
//     computed tile-by-tile in shared memory with a 5-cell halo (:412-592)
//   * V-cycle: smooth+residual, restrict down to the levels that fit one block; a single block
//     does those levels including 16 bottom sweeps (:854-1040); interpolate and smooth back up
//     (:1429-1512)
//   * convergence: max-norm residual <= max(tol_abs, tol_rel * max(|rhs|, |res0|)) (:1340-1398)
// The iteration count is decided on the device (Ctl::mg_go), so the whole solve can sit inside
// a CUDA graph with a conditional while node.
#pragma once

#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace hpq {

// view of a two-component array in level index space: element (i, j, c)
template <class R>
struct MV {
    R* p[2];
    int pitch;
    int off;
    __device__ R& operator()(int i, int j, int c) const { return p[c][(ptrdiff_t)(j + off) * pitch + (i + off)]; }
};

struct MGLev {
    int w, h;               // full box (cell: n; node: N+2)
    int vlo, vhi_i, vhi_j;  // valid box [vlo, vhi]
};

template <class R, bool CELL>
__device__ __forceinline__ R mg_lap(const MGLev& L, int i, int j, R pc, R pim, R pip, R pjm, R pjp, R facx, R facy) {
    R l = R(-2.) * (facx + facy) * pc;
    if (CELL && i == 0) l += facx * (R(4. / 3.) * pip - R(2.) * pc);
    else if (CELL && i == L.w - 1) l += facx * (R(4. / 3.) * pim - R(2.) * pc);
    else l += facx * (pim + pip);
    if (CELL && j == 0) l += facy * (R(4. / 3.) * pjp - R(2.) * pc);
    else if (CELL && j == L.h - 1) l += facy * (R(4. / 3.) * pjm - R(2.) * pc);
    else l += facy * (pjm + pjp);
    return l;
}

template <class R, bool CELL>
__device__ __forceinline__ R mg_gs(const MGLev& L, int i, int j, R pim, R pip, R pjm, R pjp, R rhs, R a, R facx,
                                   R facy) {
    R l;
    R c0 = -(a + R(2.) * (facx + facy));
    if (CELL && i == 0) { l = facx * R(4. / 3.) * pip; c0 -= R(2.) * facx; }
    else if (CELL && i == L.w - 1) { l = facx * R(4. / 3.) * pim; c0 -= R(2.) * facx; }
    else l = facx * (pim + pip);
    if (CELL && j == 0) { l += facy * R(4. / 3.) * pjp; c0 -= R(2.) * facy; }
    else if (CELL && j == L.h - 1) { l += facy * R(4. / 3.) * pjm; c0 -= R(2.) * facy; }
    else l += facy * (pjm + pjp);
    const R c0_inv = R(1.) / c0;
    return (rhs - l) * c0_inv;
}

// restrict_cc / restrict_nd (HpMultiGrid.cpp:29-53) for `nc` components
template <class R, bool CELL>
__device__ __forceinline__ R mg_restrict1(const MV<R>& f, int i, int j, int c) {
    if (CELL)
        return R(0.25) * (f(2 * i, 2 * j, c) + f(2 * i + 1, 2 * j, c) + f(2 * i, 2 * j + 1, c) + f(2 * i + 1, 2 * j + 1, c));
    return R(1. / 16.) * (f(2 * i - 1, 2 * j - 1, c) + R(2.) * f(2 * i, 2 * j - 1, c) + f(2 * i + 1, 2 * j - 1, c) +
                          R(2.) * f(2 * i - 1, 2 * j, c) + R(4.) * f(2 * i, 2 * j, c) + R(2.) * f(2 * i + 1, 2 * j, c) +
                          f(2 * i - 1, 2 * j + 1, c) + R(2.) * f(2 * i, 2 * j + 1, c) + f(2 * i + 1, 2 * j + 1, c));
}

template <class R, bool CELL>
__global__ void k_mg_restrict(MGLev C, MV<R> crse, MV<R> fine, int nc) {
    HPQ_PDL_ENTRY();
    const int vw = C.vhi_i - C.vlo + 1, vh = C.vhi_j - C.vlo + 1;
    for (long long k = gtid(); k < (long long)vw * vh; k += gstride()) {
        const int i = C.vlo + (int)(k % vw), j = C.vlo + (int)(k / vw);
        for (int c = 0; c < nc; ++c) crse(i, j, c) = mg_restrict1<R, CELL>(fine, i, j, c);
    }
}

// interpcpy (HpMultiGrid.cpp:79-120): out = fin + I(crse)
template <class R, bool CELL>
__device__ __forceinline__ R mg_interp1(const MV<R>& crse, int i, int j, int c) {
    const int ic = i >> 1, jc = j >> 1;  // i, j >= 0 on every level
    if (CELL) return crse(ic, jc, c);
    const bool io = (ic * 2 != i), jo = (jc * 2 != j);
    if (io && jo) return (crse(ic, jc, c) + crse(ic + 1, jc, c) + crse(ic, jc + 1, c) + crse(ic + 1, jc + 1, c)) * R(0.25);
    if (io) return (crse(ic, jc, c) + crse(ic + 1, jc, c)) * R(0.5);
    if (jo) return (crse(ic, jc, c) + crse(ic, jc + 1, c)) * R(0.5);
    return crse(ic, jc, c);
}

template <class R, bool CELL>
__global__ void k_mg_interp(MGLev F, MV<R> out, MV<R> fin, MV<R> crse) {
    HPQ_PDL_ENTRY();
    const int vw = F.vhi_i - F.vlo + 1, vh = F.vhi_j - F.vlo + 1;
    for (long long k = gtid(); k < (long long)vw * vh; k += gstride()) {
        const int i = F.vlo + (int)(k % vw), j = F.vlo + (int)(k / vw);
        for (int c = 0; c < 2; ++c) out(i, j, c) = fin(i, j, c) + mg_interp1<R, CELL>(crse, i, j, c);
    }
}

// ------------------------------------------------------------------------------------------
// Fused tile smoother. One launch does, on a T x T output tile with a 6-cell halo in shared
// memory:
//   load    phi = 0 | phi_in | phi_in + I(coarse)   (zero init / initial guess / the
//           interpolation of the up-sweep, HpMultiGrid.cpp:79-120, applied on the fly)
//   smooth  4 red-black Gauss-Seidel colour sweeps (gs1, :265-294)
//   store   phi_out on the tile
//   RES     residual rhs + a*phi - Lap(phi) on the tile and a one-cell ring (:185-198)
//   RESTR   restriction of that residual to the coarse points whose centre lies in the tile
//           (:29-53), i.e. the next level's right-hand side
//   NORM    max |residual| of the tile -> atomic max; the last block to finish takes the
//           convergence decision of solve_doit (:1340-1398) and sets the graph condition
// A cell at distance d from the edge of the loaded region is exact after 4 colour sweeps when
// d >= 4, so the residual is exact on the tile and its ring with a halo of 6.
// ------------------------------------------------------------------------------------------
enum { MG_INIT_ZERO = 0, MG_INIT_VIEW = 1, MG_INIT_INTERP = 2 };
enum { MG_NORM_NONE = 0, MG_NORM_ITER = 1, MG_NORM_FIRST = 2 };

template <class R>
struct SmoothArgs {
    MGLev L, Lc;
    MV<R> out, rhs, acf, in, crse_in, crse_res;
    // ping-pong: when set, iteration parity (Ctl::mg_iter & 1) == 1 swaps in/out for in2/out2
    MV<R> in2, out2;
    int pingpong;
    R facx, facy;
    Ctl* ctl;
    unsigned int* counter;
    double tol_rel, tol_abs;
    int maxiter;
    unsigned long long cond;
    int use_cond;
};

__device__ __forceinline__ double atomic_read(double* p) {
    return __longlong_as_double((long long)atomicAdd(reinterpret_cast<unsigned long long*>(p), 0ull));
}

__device__ __forceinline__ void mg_decide_first(Ctl* ctl, double resnorm0, double rhsnorm0, double tol_rel,
                                                double tol_abs, unsigned long long cond, int use_cond) {
    const double max_norm = (rhsnorm0 >= resnorm0) ? rhsnorm0 : resnorm0;
    ctl->mg_maxnorm = max_norm;
    ctl->mg_target = fmax(tol_abs, fmax(tol_rel, 1.e-16) * max_norm);
    ctl->mg_go = !(resnorm0 <= ctl->mg_target);
    ctl->mg_iter = 0;
    ctl->mg_norm = 0;
#if CUDART_VERSION >= 12040
    if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, ctl->mg_go);
#endif
}

__device__ __forceinline__ void mg_decide_iter(Ctl* ctl, double norminf, int maxiter, unsigned long long cond,
                                               int use_cond) {
    ctl->mg_norm = 0;
    ctl->mg_iter += 1;
    ctl->mg_total_iters += 1;
    int go = 1;
    if (norminf <= ctl->mg_target) go = 0;
    else if (norminf > 1.e20 * ctl->mg_maxnorm) { go = 0; if (!ctl->mg_status) ctl->mg_status = 2; }
    else if (ctl->mg_iter >= maxiter) { go = 0; if (!ctl->mg_status) ctl->mg_status = 1; }
    ctl->mg_go = go;
#if CUDART_VERSION >= 12040
    if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, go);
#endif
}

template <int T, int NSW>
struct SmoothSmem {
    static constexpr int H = NSW + 2;  // exact residual on the tile and its ring after NSW sweeps
    static constexpr int E = T + 2 * H;
    static constexpr int Q = T + 2;
    template <class R>
    static constexpr size_t bytes() { return (size_t)(5 * E * E + 2 * Q * Q) * sizeof(R); }
};

template <class R, bool CELL, int T, int INIT, bool RES, bool RESTR, int NORM, int NSW>
__global__ void __launch_bounds__(256) k_mg_smooth(SmoothArgs<R> A) {
    HPQ_PDL_ENTRY();
    using SM = SmoothSmem<T, NSW>;
    constexpr int H = SM::H;
    constexpr int E = SM::E;
    constexpr int Q = SM::Q;  // residual tile with its ring
    extern __shared__ unsigned char smem_raw[];
    R (*sp)[E * E] = reinterpret_cast<R (*)[E * E]>(smem_raw);                 // phi, 2 comps
    R (*srh)[E * E] = reinterpret_cast<R (*)[E * E]>(smem_raw + 2 * E * E * sizeof(R));  // rhs
    R* sa = reinterpret_cast<R*>(smem_raw + 4 * E * E * sizeof(R));             // coefficient
    R (*sr)[Q * Q] = reinterpret_cast<R (*)[Q * Q]>(smem_raw + 5 * E * E * sizeof(R));   // residual
    __shared__ double wmax[8], wrhs[8];
    const MGLev& L = A.L;
    const int t0i = L.vlo + blockIdx.x * T, t0j = L.vlo + blockIdx.y * T;
    const int ti0 = t0i - H, tj0 = t0j - H;
    const bool swap = A.pingpong && (A.ctl->mg_iter & 1);
    const MV<R> vin = swap ? A.in2 : A.in;
    const MV<R> vout = swap ? A.out2 : A.out;
    // every global read of the block happens here, all in flight together
    for (int e = threadIdx.x; e < E * E; e += blockDim.x) {
        const int i = ti0 + e % E, j = tj0 + e / E;
        const bool v = i >= L.vlo && i <= L.vhi_i && j >= L.vlo && j <= L.vhi_j;
        sa[e] = v ? A.acf(i, j, 0) : R(0);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            R val = R(0);
            if (v) {
                if (INIT == MG_INIT_VIEW) val = vin(i, j, c);
                else if (INIT == MG_INIT_INTERP) val = vin(i, j, c) + mg_interp1<R, CELL>(A.crse_in, i, j, c);
            }
            sp[c][e] = val;
            srh[c][e] = v ? A.rhs(i, j, c) : R(0);
        }
    }
    __syncthreads();
    for (int s = 0; s < NSW; ++s) {
        for (int e = threadIdx.x; e < E * E; e += blockDim.x) {
            const int li = e % E, lj = e / E;
            if (li == 0 || lj == 0 || li == E - 1 || lj == E - 1) continue;
            const int i = ti0 + li, j = tj0 + lj;
            if (((i + j + s) & 1) != 0) continue;
            if (i < L.vlo || i > L.vhi_i || j < L.vlo || j > L.vhi_j) continue;
            const R a = sa[e];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const R* q = sp[c];
                sp[c][e] = mg_gs<R, CELL>(L, i, j, q[e - 1], q[e + 1], q[e - E], q[e + E], srh[c][e], a, A.facx, A.facy);
            }
        }
        __syncthreads();
    }
    double bmax = 0, brhs = 0;
    if (RES) {
        for (int e = threadIdx.x; e < Q * Q; e += blockDim.x) {
            const int ri = e % Q, rj = e / Q;
            const int i = t0i - 1 + ri, j = t0j - 1 + rj;
            const bool v = i >= L.vlo && i <= L.vhi_i && j >= L.vlo && j <= L.vhi_j;
            const bool in_tile = ri >= 1 && ri <= T && rj >= 1 && rj <= T;
            const int k = (rj + H - 1) * E + (ri + H - 1);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                R r = R(0);
                if (v) {
                    const R* q = sp[c];
                    const R rh = srh[c][k];
                    r = rh + sa[k] * q[k] - mg_lap<R, CELL>(L, i, j, q[k], q[k - 1], q[k + 1], q[k - E], q[k + E], A.facx, A.facy);
                    if (NORM != MG_NORM_NONE && in_tile) {
                        bmax = fmax(bmax, fabs((double)r));
                        if (NORM == MG_NORM_FIRST) brhs = fmax(brhs, fabs((double)rh));
                    }
                }
                sr[c][e] = r;
            }
        }
    }
    for (int e = threadIdx.x; e < T * T; e += blockDim.x) {
        const int li = e % T, lj = e / T;
        const int i = t0i + li, j = t0j + lj;
        if (i > L.vhi_i || j > L.vhi_j) continue;
        const int k = (lj + H) * E + (li + H);
        vout(i, j, 0) = sp[0][k];
        vout(i, j, 1) = sp[1][k];
    }
    if (RESTR) {
        __syncthreads();
        const MGLev& C = A.Lc;
        // coarse points whose centre 2I lies in this tile
        const int ci0 = max(C.vlo, (t0i + 1) >> 1), cj0 = max(C.vlo, (t0j + 1) >> 1);
        const int ci1 = min(C.vhi_i, (t0i + T - 1) >> 1), cj1 = min(C.vhi_j, (t0j + T - 1) >> 1);
        const int cw = ci1 - ci0 + 1, ch = cj1 - cj0 + 1;
        if (cw > 0 && ch > 0) {
            for (int e = threadIdx.x; e < cw * ch; e += blockDim.x) {
                const int I = ci0 + e % cw, J = cj0 + e / cw;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    // residual at fine (i, j) is sr[c][(j - t0j + 1) * Q + (i - t0i + 1)]
                    auto f = [&](int i, int j) -> R { return sr[c][(j - t0j + 1) * Q + (i - t0i + 1)]; };
                    R v;
                    if (CELL) {
                        v = R(0.25) * (f(2 * I, 2 * J) + f(2 * I + 1, 2 * J) + f(2 * I, 2 * J + 1) + f(2 * I + 1, 2 * J + 1));
                    } else {
                        v = R(1. / 16.) * (f(2 * I - 1, 2 * J - 1) + R(2.) * f(2 * I, 2 * J - 1) + f(2 * I + 1, 2 * J - 1) +
                                           R(2.) * f(2 * I - 1, 2 * J) + R(4.) * f(2 * I, 2 * J) + R(2.) * f(2 * I + 1, 2 * J) +
                                           f(2 * I - 1, 2 * J + 1) + R(2.) * f(2 * I, 2 * J + 1) + f(2 * I + 1, 2 * J + 1));
                    }
                    A.crse_res(I, J, c) = v;
                }
            }
        }
    }
    if (NORM != MG_NORM_NONE) {
        for (int d = 16; d > 0; d >>= 1) {
            bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, d));
            brhs = fmax(brhs, __shfl_xor_sync(0xffffffffu, brhs, d));
        }
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) { wmax[warp] = bmax; wrhs[warp] = brhs; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { bmax = fmax(bmax, wmax[w]); brhs = fmax(brhs, wrhs[w]); }
            Ctl* ctl = A.ctl;
            atomic_max_nonneg(&ctl->mg_norm, bmax);
            if (NORM == MG_NORM_FIRST) atomic_max_nonneg(&ctl->mg_maxnorm, brhs);
            __threadfence();
            const unsigned total = gridDim.x * gridDim.y;
            const unsigned prev = atomicAdd(A.counter, 1u);
            if (prev == total - 1) {
                __threadfence();
                *A.counter = 0;
                const double norm = atomic_read(&ctl->mg_norm);
                if (NORM == MG_NORM_FIRST)
                    mg_decide_first(ctl, norm, atomic_read(&ctl->mg_maxnorm), A.tol_rel, A.tol_abs, A.cond, A.use_cond);
                else
                    mg_decide_iter(ctl, norm, A.maxiter, A.cond, A.use_cond);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// The coarse levels [sb, nl) in one block with shared memory (bottomsolve_gpu,
// HpMultiGrid.cpp:854-1040): down with 4 sweeps + residual + restriction per level, 16 sweeps
// on the coarsest level, up with interpolation + 4 sweeps. The coefficient of the levels below
// sb is restricted here as well (average_down_acoef, :1640-1700).
// ------------------------------------------------------------------------------------------
struct MGCoarse {
    int nl;
    MGLev L[16];
    size_t off[16];  // level offsets (elements) in the shared-memory arena
};

template <class R, bool CELL>
__device__ __forceinline__ void blk_sweeps(const MGLev& L, const R* acf, const R* res, R* cor, int nsweeps, R facx,
                                           R facy) {
    const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
    const int plane = L.w * L.h;
    for (int s = 0; s < nsweeps; ++s) {
        for (int k = threadIdx.x; k < vw * vh; k += blockDim.x) {
            const int i = L.vlo + k % vw, j = L.vlo + k / vw;
            if (((i + j + s) & 1) != 0) continue;
            const int id = j * L.w + i;
            const int im = i > 0 ? id - 1 : id, ip = i < L.w - 1 ? id + 1 : id;
            const int jm = j > 0 ? id - L.w : id, jp = j < L.h - 1 ? id + L.w : id;
            const R a = acf[id];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                R* p = cor + c * plane;
                p[id] = mg_gs<R, CELL>(L, i, j, p[im], p[ip], p[jm], p[jp], res[c * plane + id], a, facx, facy);
            }
        }
        __syncthreads();
    }
}

template <class R, bool CELL>
__global__ void __launch_bounds__(1024) k_mg_bottom(MGCoarse M, const R* __restrict__ res_g, const R* __restrict__ acf_g,
                                                    R* __restrict__ cor_g, R facx0, R facy0) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    R* arena = reinterpret_cast<R*>(smem_raw);
    // level l: cor (2n), res (2n), rescor (2n), acf (n)
    auto cor = [&](int l) { return arena + M.off[l]; };
    auto res = [&](int l) { return arena + M.off[l] + 2 * (size_t)M.L[l].w * M.L[l].h; };
    auto rsc = [&](int l) { return arena + M.off[l] + 4 * (size_t)M.L[l].w * M.L[l].h; };
    auto acf = [&](int l) { return arena + M.off[l] + 6 * (size_t)M.L[l].w * M.L[l].h; };
    {
        const int n0 = M.L[0].w * M.L[0].h;
        for (int k = threadIdx.x; k < n0; k += blockDim.x) {
            res(0)[k] = res_g[k];
            res(0)[n0 + k] = res_g[n0 + k];
            acf(0)[k] = acf_g[k];
        }
        for (int l = 1; l < M.nl; ++l) {
            const int n = M.L[l].w * M.L[l].h;
            for (int k = threadIdx.x; k < 7 * n; k += blockDim.x) cor(l)[k] = R(0);
        }
        __syncthreads();
        // coefficient hierarchy below sb
        for (int l = 1; l < M.nl; ++l) {
            const MGLev& C = M.L[l];
            const MGLev& F = M.L[l - 1];
            MV<R> fine{{acf(l - 1), acf(l - 1)}, F.w, 0};
            const int cw = C.vhi_i - C.vlo + 1, ch = C.vhi_j - C.vlo + 1;
            for (int k = threadIdx.x; k < cw * ch; k += blockDim.x) {
                const int i = C.vlo + k % cw, j = C.vlo + k / cw;
                acf(l)[j * C.w + i] = mg_restrict1<R, CELL>(fine, i, j, 0);
            }
            __syncthreads();
        }
    }
    R facx = facx0, facy = facy0;
    for (int l = 0; l < M.nl; ++l) {
        const MGLev& L = M.L[l];
        const int plane = L.w * L.h;
        for (int k = threadIdx.x; k < 2 * plane; k += blockDim.x) cor(l)[k] = R(0);
        __syncthreads();
        if (l == M.nl - 1) {
            blk_sweeps<R, CELL>(L, acf(l), res(l), cor(l), 16, facx, facy);
            break;
        }
        blk_sweeps<R, CELL>(L, acf(l), res(l), cor(l), 4, facx, facy);
        const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
        for (int k = threadIdx.x; k < vw * vh; k += blockDim.x) {
            const int i = L.vlo + k % vw, j = L.vlo + k / vw;
            const int id = j * L.w + i;
            const int im = i > 0 ? id - 1 : id, ip = i < L.w - 1 ? id + 1 : id;
            const int jm = j > 0 ? id - L.w : id, jp = j < L.h - 1 ? id + L.w : id;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const R* p = cor(l) + c * plane;
                rsc(l)[c * plane + id] = res(l)[c * plane + id] + acf(l)[id] * p[id] -
                                         mg_lap<R, CELL>(L, i, j, p[id], p[im], p[ip], p[jm], p[jp], facx, facy);
            }
        }
        __syncthreads();
        const MGLev& C = M.L[l + 1];
        const int cw = C.vhi_i - C.vlo + 1, ch = C.vhi_j - C.vlo + 1;
        MV<R> fine{{rsc(l), rsc(l) + plane}, L.w, 0};
        const int cplane = C.w * C.h;
        for (int k = threadIdx.x; k < cw * ch; k += blockDim.x) {
            const int i = C.vlo + k % cw, j = C.vlo + k / cw;
#pragma unroll
            for (int c = 0; c < 2; ++c) res(l + 1)[c * cplane + j * C.w + i] = mg_restrict1<R, CELL>(fine, i, j, c);
        }
        __syncthreads();
        facx *= R(0.25);
        facy *= R(0.25);
    }
    for (int l = M.nl - 2; l >= 0; --l) {
        facx *= R(4.);
        facy *= R(4.);
        const MGLev& L = M.L[l];
        const MGLev& C = M.L[l + 1];
        const int plane = L.w * L.h;
        MV<R> crse{{cor(l + 1), cor(l + 1) + C.w * C.h}, C.w, 0};
        const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
        for (int k = threadIdx.x; k < vw * vh; k += blockDim.x) {
            const int i = L.vlo + k % vw, j = L.vlo + k / vw;
#pragma unroll
            for (int c = 0; c < 2; ++c) cor(l)[c * plane + j * L.w + i] += mg_interp1<R, CELL>(crse, i, j, c);
        }
        __syncthreads();
        blk_sweeps<R, CELL>(L, acf(l), res(l), cor(l), 4, facx, facy);
    }
    const int n0 = 2 * M.L[0].w * M.L[0].h;
    for (int k = threadIdx.x; k < n0; k += blockDim.x) cor_g[k] = cor(0)[k];
}

template <class R>
__global__ void k_mg_copy_out(MGLev L, MV<R> sol, MV<R> cor_even, MV<R> cor_odd, const Ctl* ctl) {
    HPQ_PDL_ENTRY();
    const MV<R> cor = (ctl->mg_iter & 1) ? cor_odd : cor_even;
    const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
    for (long long k = gtid(); k < (long long)vw * vh; k += gstride()) {
        const int i = L.vlo + (int)(k % vw), j = L.vlo + (int)(k / vw);
        sol(i, j, 0) = cor(i, j, 0);
        sol(i, j, 1) = cor(i, j, 1);
    }
}

// ------------------------------------------------------------------------------------------
template <class R>
class Multigrid {
public:
    bool cell = true;
    double dx = 0, dy = 0;
    std::vector<MGLev> lev;
    std::vector<R*> acf, res, cor, up;  // level 0: acf/res are views into the slab; up = up-sweep result
    unsigned int* counter = nullptr;
    int sb = 1;  // first level of the single-block bottom solve
    int nl = 0;
    size_t bottom_smem = 0;
    MGCoarse coarse{};

    void init(int nx, int ny, double dx_, double dy_) {
        dx = dx_; dy = dy_;
        cell = (nx % 2 == 0);
        int lx, ly;
        if (cell) { lx = nx - 1; ly = ny - 1; } else { lx = nx + 1; ly = ny + 1; }
        for (int l = 0; l < 40; ++l) {
            MGLev L;
            L.w = lx + 1; L.h = ly + 1;
            if (cell) { L.vlo = 0; L.vhi_i = lx; L.vhi_j = ly; }
            else { L.vlo = 1; L.vhi_i = lx - 1; L.vhi_j = ly - 1; }
            lev.push_back(L);
            const int len_x = lx + 1, len_y = ly + 1, minw = cell ? 2 : 4;
            if (len_x < 2 * minw || len_y < 2 * minw) break;
            if (cell) { if (len_x % 2 || len_y % 2) break; lx = len_x / 2 - 1; ly = len_y / 2 - 1; }
            else { if (lx % 2 || ly % 2) break; lx /= 2; ly /= 2; }
        }
        nl = (int)lev.size();
        if (nl < 2) throw CudaError("hpmg: the domain cannot be coarsened (need at least 2 levels)");
        // single-block levels: from the first level (>= 1) whose hierarchy fits 160 KB of shared memory
        auto smem_from = [&](int s0) {
            size_t tot = 0;
            for (int l = s0; l < nl; ++l) tot += 7 * (size_t)lev[l].w * lev[l].h;
            return tot * sizeof(R);
        };
        sb = nl - 1;
        for (int l = 1; l < nl; ++l) if (smem_from(l) <= 160 * 1024 && (long long)lev[l].w * lev[l].h <= 4096) { sb = l; break; }
        if (nl - sb > 16) sb = nl - 16;
        bottom_smem = smem_from(sb);
        coarse.nl = nl - sb;
        size_t off = 0;
        for (int l = sb; l < nl; ++l) {
            coarse.L[l - sb] = lev[l];
            coarse.off[l - sb] = off;
            off += 7 * (size_t)lev[l].w * lev[l].h;
        }
        acf.assign(nl, nullptr); res.assign(nl, nullptr); cor.assign(nl, nullptr); up.assign(nl, nullptr);
        for (int l = 0; l < nl; ++l) {
            const size_t n = (size_t)lev[l].w * lev[l].h;
            if (l > 0) {
                HPQ_CUDA(cudaMalloc(&acf[l], n * sizeof(R)));
                HPQ_CUDA(cudaMalloc(&res[l], 2 * n * sizeof(R)));
                HPQ_CUDA(cudaMemset(acf[l], 0, n * sizeof(R)));
                HPQ_CUDA(cudaMemset(res[l], 0, 2 * n * sizeof(R)));
            }
            HPQ_CUDA(cudaMalloc(&cor[l], 2 * n * sizeof(R)));
            HPQ_CUDA(cudaMalloc(&up[l], 2 * n * sizeof(R)));
            HPQ_CUDA(cudaMemset(cor[l], 0, 2 * n * sizeof(R)));
            HPQ_CUDA(cudaMemset(up[l], 0, 2 * n * sizeof(R)));
        }
        HPQ_CUDA(cudaMalloc(&counter, sizeof(unsigned int)));
        HPQ_CUDA(cudaMemset(counter, 0, sizeof(unsigned int)));
        if (cell) HPQ_CUDA(cudaFuncSetAttribute(k_mg_bottom<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bottom_smem));
        else HPQ_CUDA(cudaFuncSetAttribute(k_mg_bottom<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bottom_smem));
    }
    void release() {
        for (int l = 0; l < nl; ++l) {
            if (l > 0) { cudaFree(acf[l]); cudaFree(res[l]); }
            cudaFree(cor[l]); cudaFree(up[l]);
        }
        if (counter) cudaFree(counter);
        counter = nullptr;
        lev.clear(); nl = 0;
    }
    MV<R> own(std::vector<R*>& v, int l, int ncomp = 2) const {
        const size_t n = (size_t)lev[l].w * lev[l].h;
        return {{v[l], ncomp > 1 ? v[l] + n : v[l]}, lev[l].w, 0};
    }
    MV<R> slab_view(const Slab<R>& S, int c0, int c1) const {
        const int o = cell ? 0 : 1;
        return {{S.c(c0).p, S.c(c1).p}, S.pitch, kGuardAlloc - o};
    }
    double fac(int l, double d) const { const double f = (double)(1 << l); return 1. / ((d * f) * (d * f)); }

    template <bool CELL, int INIT, bool RES, bool RESTR, int NORM, int NSW = 4>
    void smooth(cudaStream_t st, int l, SmoothArgs<R> a) {
        const MGLev& L = lev[l];
        a.L = L;
        if (l + 1 < nl) a.Lc = lev[l + 1];
        a.facx = (R)fac(l, dx);
        a.facy = (R)fac(l, dy);
        a.counter = counter;
        const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
        dim3 grid((vw + 15) / 16, (vh + 15) / 16);
        constexpr size_t smem = SmoothSmem<16, NSW>::template bytes<R>();
        auto kern = k_mg_smooth<R, CELL, 16, INIT, RES, RESTR, NORM, NSW>;
        static bool attr_done = false;  // one per instantiation
        if (!attr_done) {
            HPQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_done = true;
        }
        hpq_launch(kern, grid, dim3(256), smem, st, a);
        HPQ_LAUNCH_CHECK();
    }

    SmoothArgs<R> base_args(Ctl* ctl, double tol_rel, double tol_abs, int maxiter, unsigned long long cond,
                            int use_cond) const {
        SmoothArgs<R> a{};
        a.ctl = ctl; a.tol_rel = tol_rel; a.tol_abs = tol_abs; a.maxiter = maxiter; a.cond = cond; a.use_cond = use_cond;
        return a;
    }

    // coefficient hierarchy down to sb, first smoothing, norms and the initial decision
    template <bool CELL>
    void pre(cudaStream_t st, const Slab<R>& S, Ctl* ctl, double tol_rel, double tol_abs, int maxiter,
             unsigned long long cond, int use_cond) {
        MV<R> sol = slab_view(S, C_BX, C_BY), rhs = slab_view(S, C_SY, C_SX), a0 = slab_view(S, C_CHI, C_CHI);
        for (int l = 1; l <= sb; ++l) {
            MV<R> fine = (l == 1) ? a0 : own(acf, l - 1, 1);
            const long long n = (long long)lev[l].w * lev[l].h;
            hpq_launch(k_mg_restrict<R, CELL>, dim3(blocks_for(n, 256)), dim3(256), 0, st, lev[l], own(acf, l, 1), fine, 1);
            HPQ_LAUNCH_CHECK();
        }
        HPQ_CUDA(cudaMemsetAsync(&ctl->mg_norm, 0, sizeof(double), st));
        HPQ_CUDA(cudaMemsetAsync(&ctl->mg_maxnorm, 0, sizeof(double), st));
        SmoothArgs<R> a = base_args(ctl, tol_rel, tol_abs, maxiter, cond, use_cond);
        a.out = own(cor, 0); a.rhs = rhs; a.acf = a0; a.in = sol; a.crse_res = own(res, 1);
        smooth<CELL, MG_INIT_VIEW, true, true, MG_NORM_FIRST>(st, 0, a);
    }

    // one V-cycle; its last kernel computes the residual norm and the decision
    template <bool CELL>
    void vcycle(cudaStream_t st, const Slab<R>& S, Ctl* ctl, int maxiter, unsigned long long cond, int use_cond) {
        MV<R> sol = slab_view(S, C_BX, C_BY), rhs = slab_view(S, C_SY, C_SX), a0 = slab_view(S, C_CHI, C_CHI);
        const SmoothArgs<R> b = base_args(ctl, 0, 0, maxiter, cond, use_cond);
        for (int l = 1; l < sb; ++l) {
            SmoothArgs<R> a = b;
            a.out = own(cor, l); a.rhs = own(res, l); a.acf = own(acf, l, 1); a.crse_res = own(res, l + 1);
            smooth<CELL, MG_INIT_ZERO, true, true, MG_NORM_NONE>(st, l, a);
        }
        if (cell) hpq_launch(k_mg_bottom<R, true>, dim3(1), dim3(1024), bottom_smem, st, coarse, res[sb], acf[sb], cor[sb], (R)fac(sb, dx), (R)fac(sb, dy));
        else hpq_launch(k_mg_bottom<R, false>, dim3(1), dim3(1024), bottom_smem, st, coarse, res[sb], acf[sb], cor[sb], (R)fac(sb, dx), (R)fac(sb, dy));
        HPQ_LAUNCH_CHECK();
        for (int l = sb - 1; l >= 1; --l) {
            SmoothArgs<R> a = b;
            a.out = own(up, l); a.rhs = own(res, l); a.acf = own(acf, l, 1); a.in = own(cor, l);
            a.crse_in = (l + 1 == sb) ? own(cor, sb) : own(up, l + 1);
            smooth<CELL, MG_INIT_INTERP, false, false, MG_NORM_NONE>(st, l, a);
        }
        {
            // level 0: the up-sweep smoothing (cor0 + I(coarse) -> sol) and the closing
            // smoothing + residual (sol -> cor0) are 8 consecutive colour sweeps; sol between the
            // two is not read anywhere else, so one kernel does both (solve_doit copies cor0
            // into the solution after the last cycle)
            SmoothArgs<R> a = b;
            // cor0 is read over halos and written per tile: iterations alternate between cor[0] and
            // up[0] by the device-side iteration parity
            a.in = own(cor, 0); a.out = own(up, 0);
            a.in2 = own(up, 0); a.out2 = own(cor, 0);
            a.pingpong = 1;
            a.rhs = rhs; a.acf = a0;
            a.crse_in = (sb == 1) ? own(cor, 1) : own(up, 1);
            a.crse_res = own(res, 1);
            smooth<CELL, MG_INIT_INTERP, true, true, MG_NORM_ITER, 8>(st, 0, a);
        }
    }

    template <bool CELL>
    void post(cudaStream_t st, const Slab<R>& S, const Ctl* ctl) {
        MV<R> sol = slab_view(S, C_BX, C_BY);
        const long long n0 = (long long)lev[0].w * lev[0].h;
        hpq_launch(k_mg_copy_out<R>, dim3(blocks_for(n0, 256)), dim3(256), 0, st, lev[0], sol, own(cor, 0), own(up, 0), ctl);
        HPQ_LAUNCH_CHECK();
    }
};

}  // namespace hpq
