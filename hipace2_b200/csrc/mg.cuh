// Geometric multigrid for the explicit Bx/By equation  -chi*B + Lap(B) = S  (two components
// sharing one coefficient), homogeneous Dirichlet boundaries. Restates hpmg::MultiGrid system
// type 1 (mg_solver/HpMultiGrid.cpp):
//   * levels: cell-centred when n is even (Dirichlet on the cell face with the 4/3 closure,
//     :162-183, 265-294), node-centred otherwise (Dirichlet on the first guard node) (:1043-1100)
//   * smoother: 4 red-black Gauss-Seidel colour sweeps, optionally followed by the residual,
//     computed tile-by-tile in shared memory with a 5-cell halo (:412-592)
//   * V-cycle: smooth+residual, restrict down to the levels that fit one block's shared memory;
//     those levels, including max(16, longest side) bottom sweeps, run in one block per
//     component in the persistent solve (one block for both in the multi-kernel form)
//     (:854-1040, 1584-1592); interpolate and smooth back up (:1429-1512)
//   * convergence: max-norm residual <= max(tol_abs, tol_rel * max(|rhs|, |res0|)) (:1340-1398)
// The iteration count is decided on the device (Ctl::mg_go), so the whole solve can sit inside
// a CUDA graph with a conditional while node.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <type_traits>
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

// Gauss-Seidel point update (gs1, HpMultiGrid.cpp:265-294) split in two: the inverse of the
// diagonal, which depends only on the coefficient and the position, is computed once per point
// and reused by every colour sweep.
template <class R, bool CELL>
__device__ __forceinline__ R mg_diag_inv(const MGLev& L, int i, int j, R a, R facx, R facy) {
    R c0 = -(a + R(2.) * (facx + facy));
    if (CELL && (i == 0 || i == L.w - 1)) c0 -= R(2.) * facx;
    if (CELL && (j == 0 || j == L.h - 1)) c0 -= R(2.) * facy;
    return R(1.) / c0;
}
template <class R, bool CELL>
__device__ __forceinline__ R mg_gs_inv(const MGLev& L, int i, int j, R pim, R pip, R pjm, R pjp, R rhs, R c0_inv,
                                       R facx, R facy) {
    R l;
    if (CELL && i == 0) l = facx * R(4. / 3.) * pip;
    else if (CELL && i == L.w - 1) l = facx * R(4. / 3.) * pim;
    else l = facx * (pim + pip);
    if (CELL && j == 0) l += facy * R(4. / 3.) * pjp;
    else if (CELL && j == L.h - 1) l += facy * R(4. / 3.) * pjm;
    else l += facy * (pjm + pjp);
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
// initial guess of a smoothing pass: zero, the input view, the input view plus the interpolated
// coarse correction, or zero plus the interpolated coarse correction
enum { MG_INIT_ZERO = 0, MG_INIT_VIEW = 1, MG_INIT_INTERP = 2, MG_INIT_INTERP0 = 3 };
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

// Asynchronous global -> shared copy of one element (cp.async, 4 or 8 bytes); with `valid` false
// nothing is read and the element is zero-filled. All copies of a tile are in flight together.
template <class R>
__device__ __forceinline__ void cp_async_el(R* dst, const R* src, bool valid) {
    static_assert(sizeof(R) == 4 || sizeof(R) == 8, "element size");
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if (sizeof(R) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// interpcpy (HpMultiGrid.cpp:79-120) with the coarse values read through an accessor c(ic, jc)
template <class R, bool CELL, class C>
__device__ __forceinline__ R mg_interp1f(const C& crse, int i, int j) {
    const int ic = i >> 1, jc = j >> 1;
    if (CELL) return crse(ic, jc);
    const bool io = (ic * 2 != i), jo = (jc * 2 != j);
    if (io && jo) return (crse(ic, jc) + crse(ic + 1, jc) + crse(ic, jc + 1) + crse(ic + 1, jc + 1)) * R(0.25);
    if (io) return (crse(ic, jc) + crse(ic + 1, jc)) * R(0.5);
    if (jo) return (crse(ic, jc) + crse(ic, jc + 1)) * R(0.5);
    return crse(ic, jc);
}

template <int T, int NSW>
struct SmoothSmem {
    static constexpr int H = NSW + 2;  // exact residual on the tile and its ring after NSW sweeps
    static constexpr int E = T + 2 * H;
    static constexpr int Q = T + 2;
    static constexpr int EC = E / 2 + 3;  // coarse points under the loaded region (interpolation)
    // phi (2), rhs (2), coefficient, 1/diagonal, then the coarse correction (2, read before the
    // sweeps); the residual (2 Q^2) reuses the 1/diagonal and coarse planes after the sweeps
    static constexpr int TAIL = (E * E + 2 * EC * EC > 2 * Q * Q) ? E * E + 2 * EC * EC : 2 * Q * Q;
    template <class R>
    static constexpr size_t bytes() { return (size_t)(5 * E * E + TAIL) * sizeof(R); }
};

// One T x T tile (tile coordinates bx, by) of the fused smoother. `swap` selects in2/out2 for
// in/out. The tile's residual and |rhs| max norms are folded into the caller's bmax / brhs.
template <class R, bool CELL, int T, int INIT, bool RES, bool RESTR, int NORM, int NSW>
__device__ __forceinline__ void mg_smooth_tile(const SmoothArgs<R>& A, int bx, int by, bool swap,
                                               unsigned char* smem_raw, double& bmax, double& brhs) {
    using SM = SmoothSmem<T, NSW>;
    constexpr int H = SM::H;
    constexpr int E = SM::E;
    constexpr int Q = SM::Q;  // residual tile with its ring
    constexpr int NT = 256;   // threads of every smoother launch
    R (*sp)[E * E] = reinterpret_cast<R (*)[E * E]>(smem_raw);                 // phi, 2 comps
    R (*srh)[E * E] = reinterpret_cast<R (*)[E * E]>(smem_raw + 2 * E * E * sizeof(R));  // rhs
    R* sa = reinterpret_cast<R*>(smem_raw + 4 * E * E * sizeof(R));             // coefficient
    R* sinv = reinterpret_cast<R*>(smem_raw + 5 * E * E * sizeof(R));           // 1 / diagonal
    constexpr int EC = SM::EC;
    R (*sc)[EC * EC] = reinterpret_cast<R (*)[EC * EC]>(smem_raw + 6 * E * E * sizeof(R));  // coarse (set-up only)
    // residual: written after the last sweep's barrier, over the 1/diagonal and coarse planes
    R (*sr)[Q * Q] = reinterpret_cast<R (*)[Q * Q]>(smem_raw + 5 * E * E * sizeof(R));
    const MGLev& L = A.L;
    const int t0i = L.vlo + bx * T, t0j = L.vlo + by * T;
    const int ti0 = t0i - H, tj0 = t0j - H;
    const MV<R> vin = swap ? A.in2 : A.in;
    const MV<R> vout = swap ? A.out2 : A.out;
    __syncthreads();  // shared memory of the previous tile of this block
    // every global read of the tile is an asynchronous copy issued here, all in flight together
    // (cells outside the valid box are zero-filled)
    const int ci0 = (ti0 >> 1) - 1, cj0 = (tj0 >> 1) - 1;  // coarse origin of the interpolation
#pragma unroll
    for (int e0 = 0; e0 < E * E; e0 += NT) {
        const int e = e0 + threadIdx.x;
        if (e >= E * E) break;
        const int i = ti0 + e % E, j = tj0 + e / E;
        const bool v = i >= L.vlo && i <= L.vhi_i && j >= L.vlo && j <= L.vhi_j;
        cp_async_el<R>(&sa[e], v ? &A.acf(i, j, 0) : A.acf.p[0], v);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            cp_async_el<R>(&srh[c][e], v ? &A.rhs(i, j, c) : A.rhs.p[c], v);
            if (INIT == MG_INIT_ZERO || INIT == MG_INIT_INTERP0) sp[c][e] = R(0);
            else cp_async_el<R>(&sp[c][e], v ? &vin(i, j, c) : vin.p[c], v);
        }
    }
    if (INIT == MG_INIT_INTERP || INIT == MG_INIT_INTERP0) {
        const MGLev& C = A.Lc;
        for (int e = threadIdx.x; e < EC * EC; e += NT) {
            const int ic = ci0 + e % EC, jc = cj0 + e / EC;
            const bool v = ic >= 0 && ic < C.w && jc >= 0 && jc < C.h;
#pragma unroll
            for (int c = 0; c < 2; ++c) cp_async_el<R>(&sc[c][e], v ? &A.crse_in(ic, jc, c) : A.crse_in.p[c], v);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // inverse diagonals; the interpolated coarse correction added to the initial guess
#pragma unroll
    for (int e0 = 0; e0 < E * E; e0 += NT) {
        const int e = e0 + threadIdx.x;
        if (e >= E * E) break;
        const int i = ti0 + e % E, j = tj0 + e / E;
        const bool v = i >= L.vlo && i <= L.vhi_i && j >= L.vlo && j <= L.vhi_j;
        sinv[e] = v ? mg_diag_inv<R, CELL>(L, i, j, sa[e], A.facx, A.facy) : R(0);
        if ((INIT == MG_INIT_INTERP || INIT == MG_INIT_INTERP0) && v) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const R* q = sc[c];
                sp[c][e] = sp[c][e] + mg_interp1f<R, CELL>([&](int ic, int jc) { return q[(jc - cj0) * EC + (ic - ci0)]; }, i, j);
            }
        }
    }
    __syncthreads();
    // colour sweeps over the interior of the loaded region (its outer ring stays fixed): only
    // the points of the sweep's colour are visited, (E-2)/2 per row
    constexpr int HW = (E - 2) / 2;
    for (int s = 0; s < NSW; ++s) {
#pragma unroll
        for (int q0 = 0; q0 < (E - 2) * HW; q0 += NT) {
            const int q = q0 + threadIdx.x;
            if (q >= (E - 2) * HW) break;
            const int lj = 1 + q / HW, k = q - (lj - 1) * HW;
            const int par = (s + ti0 + tj0 + lj) & 1;  // parity of li for (i + j + s) even
            const int li = (par ? 1 : 2) + 2 * k;
            const int i = ti0 + li, j = tj0 + lj;
            if (i < L.vlo || i > L.vhi_i || j < L.vlo || j > L.vhi_j) continue;
            const int e = lj * E + li;
            const R inv = sinv[e];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const R* qq = sp[c];
                sp[c][e] = mg_gs_inv<R, CELL>(L, i, j, qq[e - 1], qq[e + 1], qq[e - E], qq[e + E], srh[c][e], inv, A.facx, A.facy);
            }
        }
        __syncthreads();
    }
    if (RES) {
        for (int e = threadIdx.x; e < Q * Q; e += NT) {
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
    for (int e = threadIdx.x; e < T * T; e += NT) {
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
            for (int e = threadIdx.x; e < cw * ch; e += NT) {
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
}

// max over the block of two per-thread values; the result is valid in thread 0
__device__ __forceinline__ void block_max2(double& a, double& b) {
    __shared__ double wa[32], wb[32];
    for (int d = 16; d > 0; d >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, d));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, d));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) { wa[warp] = a; wb[warp] = b; }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { a = fmax(a, wa[w]); b = fmax(b, wb[w]); }
}

// one tile per block; with NORM the last block to finish takes the convergence decision of
// solve_doit (:1340-1398) and sets the graph condition
template <class R, bool CELL, int T, int INIT, bool RES, bool RESTR, int NORM, int NSW>
__global__ void __launch_bounds__(256) k_mg_smooth(SmoothArgs<R> A) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    double bmax = 0, brhs = 0;
    const bool swap = A.pingpong && (A.ctl->mg_iter & 1);
    mg_smooth_tile<R, CELL, T, INIT, RES, RESTR, NORM, NSW>(A, blockIdx.x, blockIdx.y, swap, smem_raw, bmax, brhs);
    if (NORM != MG_NORM_NONE) {
        block_max2(bmax, brhs);
        if (threadIdx.x == 0) {
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
// The coarse levels [sb, nl) in one block with shared memory, for one or both components
// (bottomsolve_gpu, HpMultiGrid.cpp:854-1040): down with 4 sweeps + residual + restriction per
// level, max(16, longest side) sweeps on the coarsest level, up with interpolation + 4 sweeps.
// The coefficient of the levels below sb is restricted here as well (average_down_acoef,
// :1640-1700).
// ------------------------------------------------------------------------------------------
struct MGCoarse {
    int nl;
    int lw;          // first level run by one warp (levels of at most kWarpLevelPoints points)
    int ns_bottom;   // sweeps of the coarsest level: max(16, its longest side rounded up to even)
    // arena of the coarse levels in global memory when they do not fit in shared memory (grids
    // that stop coarsening at a large level, e.g. 300^2 -> 75^2), else null
    void* garena;
    MGLev L[16];
    // level l starts (3 NC + 2) poff[l] elements into the arena, poff[l] = the points of the
    // levels before it (NC: components per bottom block)
    size_t poff[16];
};
constexpr int kWarpLevelPoints = 128;
constexpr size_t kBottomSmemMax = 200 * 1024;  // shared memory of the single-block bottom solve

// 2-D loops over the valid points of a level (threads as 16 columns x blockDim/16 rows, no
// integer division), all points or those of one colour ((i + j + s) even)
template <class F>
__device__ __forceinline__ void for_valid(const MGLev& L, F f) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, nty = blockDim.x >> 4;
    for (int j = L.vlo + ty; j <= L.vhi_j; j += nty)
        for (int i = L.vlo + tx; i <= L.vhi_i; i += 16) f(i, j);
}
template <class F>
__device__ __forceinline__ void for_colour(const MGLev& L, int s, F f) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, nty = blockDim.x >> 4;
    for (int j = L.vlo + ty; j <= L.vhi_j; j += nty) {
        const int i0 = L.vlo + ((L.vlo + j + s) & 1);
        for (int i = i0 + 2 * tx; i <= L.vhi_i; i += 32) f(i, j);
    }
}


// The coarse levels in one block. With `init` the coefficient hierarchy and the inverse
// diagonals are built in the arena; without it they are the ones of an earlier call of the same
// solve, still resident in this block's shared memory. The global arrays are plain (not
// restrict/read-only) pointers: in the persistent solve other blocks write them earlier in the
// same launch.
// Thread groups of the coarse levels: the whole block (loops over 16 columns x blockDim/16 rows,
// block barriers), or warp 0 alone for the smallest levels (lane-strided loops, warp barriers:
// a level of a few dozen points is then a handful of instructions per step instead of a block
// barrier). A colour sweep updates points of one colour from the other colour only, so the
// order of the points, and the group, do not change the result.
struct BlockGroup {
    __device__ static void sync() { __syncthreads(); }
    template <class F>
    __device__ static void valid(const MGLev& L, F f) { for_valid(L, f); }
    template <class F>
    __device__ static void colour(const MGLev& L, int s, F f) { for_colour(L, s, f); }
};
struct WarpGroup {
    __device__ static void sync() { __syncwarp(); }
    template <class F>
    __device__ static void valid(const MGLev& L, F f) {
        const int vw = L.vhi_i - L.vlo + 1, n = vw * (L.vhi_j - L.vlo + 1);
        for (int k = threadIdx.x & 31; k < n; k += 32) f(L.vlo + k % vw, L.vlo + k / vw);
    }
    template <class F>
    __device__ static void colour(const MGLev& L, int s, F f) {
        valid(L, [&](int i, int j) {
            if (((i + j + s) & 1) == 0) f(i, j);
        });
    }
};

// one coarse level in the shared-memory arena: correction, right-hand side, residual,
// coefficient, inverse diagonal (two components each for the first three)
template <class R>
struct CoarseLevel {
    MGLev L;
    R *cor, *res, *rsc, *acf, *dinv;
    R facx, facy;
};

// NC: the components one group carries (2, or 1 when the two components of the coarse levels
// are solved by two blocks side by side); every load of a point's components comes before
// any of its stores, so the NC update chains overlap
template <class G, class R, bool CELL, int NC>
__device__ __forceinline__ void coarse_sweeps(const CoarseLevel<R>& A, int nsweeps) {
    const MGLev& L = A.L;
    const int plane = L.w * L.h;
    for (int s = 0; s < nsweeps; ++s) {
        G::colour(L, s, [&](int i, int j) {
            const int id = j * L.w + i;
            const int im = i > 0 ? id - 1 : id, ip = i < L.w - 1 ? id + 1 : id;
            const int jm = j > 0 ? id - L.w : id, jp = j < L.h - 1 ? id + L.w : id;
            // a colour sweep reads only the other colour: the components' chains are independent
            const R inv = A.dinv[id];
            R a[NC], b[NC], c[NC], d[NC], r[NC], v[NC];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const R* p = A.cor + q * plane;
                a[q] = p[im]; b[q] = p[ip]; c[q] = p[jm]; d[q] = p[jp]; r[q] = A.res[q * plane + id];
            }
#pragma unroll
            for (int q = 0; q < NC; ++q) v[q] = mg_gs_inv<R, CELL>(L, i, j, a[q], b[q], c[q], d[q], r[q], inv, A.facx, A.facy);
#pragma unroll
            for (int q = 0; q < NC; ++q) A.cor[q * plane + id] = v[q];
        });
        G::sync();
    }
}

// The colour sweeps of a level of at most 32 valid points in warp 0 with the values in
// registers: lane k holds valid point k (row-major in the valid box) and reads its neighbours of
// the other colour with shuffles, or from the arena where a neighbour lies outside the valid box
// (those values do not change during the sweeps). The same point updates in the same order of
// colours as coarse_sweeps, so the values are the same; the result goes back to the arena. Call
// with all 32 lanes of warp 0.
template <class R, bool CELL, int NC>
__device__ __forceinline__ void coarse_sweeps_lanes(const CoarseLevel<R>& A, int nsweeps) {
    const MGLev& L = A.L;
    const int plane = L.w * L.h;
    const int lane = threadIdx.x & 31;
    const int vw = L.vhi_i - L.vlo + 1, np = vw * (L.vhi_j - L.vlo + 1);
    const bool mine = lane < np;
    const int k = mine ? lane : 0;
    const int i = L.vlo + k % vw, j = L.vlo + k / vw;
    const int id = j * L.w + i;
    const int im = i > 0 ? id - 1 : id, ip = i < L.w - 1 ? id + 1 : id;
    const int jm = j > 0 ? id - L.w : id, jp = j < L.h - 1 ? id + L.w : id;
    // neighbour inside the valid box: the lane holding it, else -1 (value from the arena)
    const int lm = (i - 1 >= L.vlo && im != id) ? k - 1 : -1, lp = (i + 1 <= L.vhi_i && ip != id) ? k + 1 : -1;
    const int ljm = (j - 1 >= L.vlo && jm != id) ? k - vw : -1, ljp = (j + 1 <= L.vhi_j && jp != id) ? k + vw : -1;
    const R inv = A.dinv[id];
    R v[NC], r[NC], em[NC], ep[NC], ejm[NC], ejp[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const R* p = A.cor + q * plane;
        v[q] = p[id];
        r[q] = A.res[q * plane + id];
        em[q] = p[im]; ep[q] = p[ip]; ejm[q] = p[jm]; ejp[q] = p[jp];
    }
    for (int s = 0; s < nsweeps; ++s) {
        const bool upd = mine && ((i + j + s) & 1) == 0;
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const R a = __shfl_sync(0xffffffffu, v[q], lm < 0 ? lane : lm);
            const R b = __shfl_sync(0xffffffffu, v[q], lp < 0 ? lane : lp);
            const R c = __shfl_sync(0xffffffffu, v[q], ljm < 0 ? lane : ljm);
            const R d = __shfl_sync(0xffffffffu, v[q], ljp < 0 ? lane : ljp);
            const R nv = mg_gs_inv<R, CELL>(L, i, j, lm < 0 ? em[q] : a, lp < 0 ? ep[q] : b, ljm < 0 ? ejm[q] : c,
                                            ljp < 0 ? ejp[q] : d, r[q], inv, A.facx, A.facy);
            if (upd) v[q] = nv;
        }
    }
    if (mine) {
#pragma unroll
        for (int q = 0; q < NC; ++q) A.cor[q * plane + id] = v[q];
    }
}

// 4 sweeps, the residual, and its restriction into the next level's right-hand side
template <class G, class R, bool CELL, int NC>
__device__ __forceinline__ void coarse_down(const CoarseLevel<R>& A, const CoarseLevel<R>& C) {
    coarse_sweeps<G, R, CELL, NC>(A, 4);
    const MGLev& L = A.L;
    const int plane = L.w * L.h;
    G::valid(L, [&](int i, int j) {
        const int id = j * L.w + i;
        const int im = i > 0 ? id - 1 : id, ip = i < L.w - 1 ? id + 1 : id;
        const int jm = j > 0 ? id - L.w : id, jp = j < L.h - 1 ? id + L.w : id;
        const R ac = A.acf[id];
        R e[NC], a[NC], b[NC], c[NC], d[NC], r[NC], q[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const R* p = A.cor + k * plane;
            e[k] = p[id]; a[k] = p[im]; b[k] = p[ip]; c[k] = p[jm]; d[k] = p[jp]; r[k] = A.res[k * plane + id];
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) q[k] = r[k] + ac * e[k] - mg_lap<R, CELL>(L, i, j, e[k], a[k], b[k], c[k], d[k], A.facx, A.facy);
#pragma unroll
        for (int k = 0; k < NC; ++k) A.rsc[k * plane + id] = q[k];
    });
    G::sync();
    MV<R> fine{{A.rsc, A.rsc + (NC > 1 ? plane : 0)}, L.w, 0};
    const int cplane = C.L.w * C.L.h;
    G::valid(C.L, [&](int i, int j) {
        R q[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) q[k] = mg_restrict1<R, CELL>(fine, i, j, k);
#pragma unroll
        for (int k = 0; k < NC; ++k) C.res[k * cplane + j * C.L.w + i] = q[k];
    });
    G::sync();
}

// interpolation of the coarser correction, then 4 sweeps
template <class G, class R, bool CELL, int NC>
__device__ __forceinline__ void coarse_up(const CoarseLevel<R>& A, const CoarseLevel<R>& C) {
    const MGLev& L = A.L;
    const int plane = L.w * L.h;
    MV<R> crse{{C.cor, C.cor + (NC > 1 ? C.L.w * C.L.h : 0)}, C.L.w, 0};
    G::valid(L, [&](int i, int j) {
        const int id = j * L.w + i;
        R u[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) u[k] = A.cor[k * plane + id] + mg_interp1<R, CELL>(crse, i, j, k);
#pragma unroll
        for (int k = 0; k < NC; ++k) A.cor[k * plane + id] = u[k];
    });
    G::sync();
    coarse_sweeps<G, R, CELL, NC>(A, 4);
}

__device__ __forceinline__ unsigned long long tc_clock_ns();

// bt (tracing only): thread 0 records the global timer at the start, after the set-up, after each
// level of the down sweep, after the coarsest level, after each level of the up sweep and at the
// end: bt[0] = count, bt[1..]
// NC = 2: both components (res_g, cor_g: two planes of the first level); NC = 1: one component
// (res_g, cor_g point at its plane), the other one solved by another block
// Coefficient hierarchy of the coarse levels in a bottom block's arena (NC components per
// level): from the coefficient of the first coarse level, already in acf(0) (the rest of the
// arena zero), the restrictions to the coarser levels (average_down_acoef, :1640-1700) and the
// inverse diagonals of every level.
template <class R, bool CELL, int NC>
__device__ __forceinline__ void mg_coarse_coef(const MGCoarse& M, R* arena, R facx0, R facy0) {
    auto nn = [&](int l) { return (size_t)M.L[l].w * M.L[l].h; };
    auto acf = [&](int l) { return arena + (3 * NC + 2) * M.poff[l] + 3 * NC * nn(l); };
    auto dinv = [&](int l) { return arena + (3 * NC + 2) * M.poff[l] + (3 * NC + 1) * nn(l); };
    for (int l = 1; l < M.nl; ++l) {
        const MGLev& C = M.L[l];
        MV<R> fine{{acf(l - 1), acf(l - 1)}, M.L[l - 1].w, 0};
        for_valid(C, [&](int i, int j) { acf(l)[j * C.w + i] = mg_restrict1<R, CELL>(fine, i, j, 0); });
        __syncthreads();
    }
    R fx = facx0, fy = facy0;
    for (int l = 0; l < M.nl; ++l) {
        const MGLev& L = M.L[l];
        for_valid(L, [&](int i, int j) {
            dinv(l)[j * L.w + i] = mg_diag_inv<R, CELL>(L, i, j, acf(l)[j * L.w + i], fx, fy);
        });
        fx *= R(0.25);
        fy *= R(0.25);
    }
}

// The same hierarchy built ahead of the first bottom solve of a persistent solve, by a bottom
// block during the phase before it: the first coarse level's coefficient is restricted here from
// the finer level's `fine` (the same restriction, on the same values, as the grid-wide one that
// writes it to global memory in that phase).
template <class R, bool CELL, int NC>
__device__ __forceinline__ void mg_bottom_prebuild(const MGCoarse& M, const MV<R>& fine, R facx0, R facy0,
                                                   unsigned char* smem_raw) {
    __syncthreads();
    R* arena = reinterpret_cast<R*>(smem_raw);
    for (int l = 0; l < M.nl; ++l) {
        const int n = M.L[l].w * M.L[l].h;
        R* a = arena + (3 * NC + 2) * M.poff[l];
        for (int k = threadIdx.x; k < (3 * NC + 2) * n; k += blockDim.x) a[k] = R(0);
    }
    __syncthreads();
    const MGLev& C = M.L[0];
    R* acf0 = arena + 3 * NC * (size_t)C.w * C.h;
    for_valid(C, [&](int i, int j) { acf0[j * C.w + i] = mg_restrict1<R, CELL>(fine, i, j, 0); });
    __syncthreads();
    mg_coarse_coef<R, CELL, NC>(M, arena, facx0, facy0);
    __syncthreads();
}

// LANES: a coarsest level of at most 32 points is swept in registers of warp 0
// (coarse_sweeps_lanes) instead of by the block
template <class R, bool CELL, bool GA = false, int NC = 2, bool LANES = false>
__device__ __forceinline__ void mg_bottom_block(const MGCoarse& M, const R* res_g, const R* acf_g, R* cor_g, R facx0,
                                                R facy0, unsigned char* smem_raw, bool init,
                                                unsigned long long* bt = nullptr) {
    int nbt = 0;
    auto bstamp = [&]() {
        if (bt && threadIdx.x == 0 && nbt < 60) bt[1 + nbt++] = tc_clock_ns();
    };
    bstamp();
    __syncthreads();  // the block may have used the shared memory just before
    // GA: the arena in global memory (M.garena), else in shared memory, known at compile time
    R* arena = GA ? static_cast<R*>(M.garena) : reinterpret_cast<R*>(smem_raw);
    // level l (n points, 3 NC + 2 planes from (3 NC + 2) M.poff[l]): cor (NC n), res (NC n),
    // rescor (NC n), acf (n), 1/diagonal (n)
    auto nn = [&](int l) { return (size_t)M.L[l].w * M.L[l].h; };
    auto cor = [&](int l) { return arena + (3 * NC + 2) * M.poff[l]; };
    auto res = [&](int l) { return cor(l) + NC * nn(l); };
    auto rsc = [&](int l) { return cor(l) + 2 * NC * nn(l); };
    auto acf = [&](int l) { return cor(l) + 3 * NC * nn(l); };
    auto dinv = [&](int l) { return cor(l) + (3 * NC + 1) * nn(l); };
    const int n0 = M.L[0].w * M.L[0].h;
    if (init) {
        for (int l = 0; l < M.nl; ++l) {
            const int n = M.L[l].w * M.L[l].h;
            for (int k = threadIdx.x; k < (3 * NC + 2) * n; k += blockDim.x) cor(l)[k] = R(0);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < n0; k += blockDim.x) acf(0)[k] = acf_g[k];
        __syncthreads();
        // coefficient hierarchy below sb
        mg_coarse_coef<R, CELL, NC>(M, arena, facx0, facy0);
    } else {
        for (int l = 0; l < M.nl; ++l) {
            const int n = M.L[l].w * M.L[l].h;
            for (int k = threadIdx.x; k < NC * n; k += blockDim.x) cor(l)[k] = R(0);
        }
    }
    for (int k = threadIdx.x; k < NC * n0; k += blockDim.x) res(0)[k] = res_g[k];
    __syncthreads();
    bstamp();
    // down to the first warp level (block-wide), the smallest levels by warp 0 alone (down,
    // coarsest, up: no block barrier between their short steps), then the block-wide up-sweep
    const int lw = M.lw < M.nl ? M.lw : M.nl;
    auto fac = [&](int l, R f0) {
        for (int k = 0; k < l; ++k) f0 *= R(0.25);
        return f0;
    };
    auto arena_level = [&](int l) {
        return CoarseLevel<R>{M.L[l], cor(l), res(l), rsc(l), acf(l), dinv(l), fac(l, facx0), fac(l, facy0)};
    };
    for (int l = 0; l < lw && l < M.nl - 1; ++l) {
        coarse_down<BlockGroup, R, CELL, NC>(arena_level(l), arena_level(l + 1));
        bstamp();
    }
    if (lw >= M.nl - 1 && lw == M.nl) {
        const MGLev& Lc = M.L[M.nl - 1];
        if (LANES && (Lc.vhi_i - Lc.vlo + 1) * (Lc.vhi_j - Lc.vlo + 1) <= 32) {
            // a coarsest level of at most 32 points: its sweeps in registers of warp 0
            if (threadIdx.x < 32) coarse_sweeps_lanes<R, CELL, NC>(arena_level(M.nl - 1), M.ns_bottom);
            __syncthreads();
        } else if (M.ns_bottom == 16) {
            coarse_sweeps<BlockGroup, R, CELL, NC>(arena_level(M.nl - 1), 16);
        } else {
            coarse_sweeps<BlockGroup, R, CELL, NC>(arena_level(M.nl - 1), M.ns_bottom);
        }
        bstamp();
    } else {
        if (threadIdx.x < 32) {
            for (int l = lw; l < M.nl - 1; ++l) coarse_down<WarpGroup, R, CELL, NC>(arena_level(l), arena_level(l + 1));
            coarse_sweeps<WarpGroup, R, CELL, NC>(arena_level(M.nl - 1), M.ns_bottom);
            for (int l = M.nl - 2; l >= lw; --l) coarse_up<WarpGroup, R, CELL, NC>(arena_level(l), arena_level(l + 1));
        }
        __syncthreads();
        bstamp();
    }
    for (int l = (lw < M.nl ? lw : M.nl - 1) - 1; l >= 0; --l) {
        coarse_up<BlockGroup, R, CELL, NC>(arena_level(l), arena_level(l + 1));
        bstamp();
    }
    for (int k = threadIdx.x; k < NC * n0; k += blockDim.x) cor_g[k] = cor(0)[k];
    bstamp();
    if (bt && threadIdx.x == 0) bt[0] = nbt;
}

template <class R, bool CELL>
__global__ void __launch_bounds__(1024) k_mg_bottom(MGCoarse M, const R* __restrict__ res_g, const R* __restrict__ acf_g,
                                                    R* __restrict__ cor_g, R facx0, R facy0) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    if (M.garena) mg_bottom_block<R, CELL, true>(M, res_g, acf_g, cor_g, facx0, facy0, smem_raw, true);
    else mg_bottom_block<R, CELL, false>(M, res_g, acf_g, cor_g, facx0, facy0, smem_raw, true);
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
// Persistent solve: the whole of solve_doit (first smoothing, every V-cycle, the convergence
// decisions and the copy into the solution) in ONE cooperative launch. Each phase of the
// multi-kernel V-cycle above becomes a loop over its tiles, separated by grid barriers; the
// arithmetic per point is the same device code, so both forms give identical results.
// ------------------------------------------------------------------------------------------
constexpr int kMGMaxLevels = 16;
constexpr double kRefineTol = 1e-5;  // relative tolerance below which single precision refines in FP64
constexpr long long kBarrierSpins = 1ll << 24;  // >= ~1 s of polling before giving up
constexpr long long kBarrierFastSpins = 0;      // polls without a sleep in between (256 measured slower)

template <class R>
struct MGSolveArgs {
    int nl, sb;
    MGLev lev[kMGMaxLevels];
    R facx[kMGMaxLevels], facy[kMGMaxLevels];
    MV<R> sol, rhs, a0;  // level-0 views into the slice arrays
    R* acf[kMGMaxLevels];
    R* res[kMGMaxLevels];
    R* cor[kMGMaxLevels];
    R* up[kMGMaxLevels];
    MGCoarse coarse;
    Ctl* ctl;
    double tol_rel, tol_abs;
    int maxiter;
    // single precision: level-0 solution in FP64 and the FP32 right-hand side of the level-0
    // correction equation, two slots each (by iteration parity)
    double* x64[2];
    R* r32[2];
    // optional phase trace (HPQ_MG_TRACE): block 0 records the global timer after each barrier
    unsigned long long* trace;
    // single precision: 1 = level 0 with FP64 iterative refinement, 0 = plain FP32 V-cycles
    int refine;
    // 32^2 form: bit l set = level l >= 1 in 32^2 tiles as well
    unsigned int l32_mask;
    // level 0 of a V-cycle as two phases of 4 sweeps (interpolation + up-sweeps, then the next
    // down-sweeps + residual) instead of one phase of 8: each 16^2 tile then sweeps a 28^2
    // region 4 + 4 times instead of a 36^2 region 8 times (40 % fewer point updates, one more
    // grid barrier). Same sweeps in the same order, so the same results.
    int split0;
};

__device__ __forceinline__ unsigned long long tc_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier for a cooperative launch (all blocks co-resident). Arrival is one release
// reduction per block on a counter that only grows during a solve (cleared before every
// launch): a block's n-th barrier is passed once the counter reaches n x (blocks in the grid),
// which the waiting blocks read from the counter itself with acquire loads, so the last block to
// arrive has nothing more to publish. Bounded: a block that polls longer than kBarrierSpins, or
// sees the error flag, sets the flag and returns false; every block then leaves the kernel at
// its next barrier. `seq` counts the barriers this block has passed (thread 0's copy is used).
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, int* err, unsigned int& seq) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int* verr = err;
        const unsigned int target = ++seq * (gridDim.x * gridDim.y * gridDim.z);
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        long long it = 0;
        while (ld_acquire(bar) < target) {
            if (*verr) break;
            if (++it > kBarrierSpins) { atomicExch(err, 1); break; }
            if (it > kBarrierFastSpins) __nanosleep(32);
        }
        s_ok = (*verr == 0);
    }
    __syncthreads();
    return s_ok != 0;
}

template <class R>
__device__ __forceinline__ MV<R> mg_own(R* const* v, const MGLev* lev, int l, int ncomp = 2) {
    const size_t n = (size_t)lev[l].w * lev[l].h;
    return {{v[l], ncomp > 1 ? v[l] + n : v[l]}, lev[l].w, 0};
}

// ------------------------------------------------------------------------------------------
// Level 0 of the single-precision solve with FP64 iterative refinement. The solution x is held
// in FP64; the colour sweeps run in FP32 on the correction d of the level-0 correction equation
// (Lap - a) d = r, whose right-hand side r = rhs + a x - Lap(x) is recomputed in FP64 from x.
// Because every smoothing step is affine and keeps the exact solution fixed, sweeping d from
// zero (or from the coarse-grid correction) with right-hand side r and then adding d to x gives
// the same iterates as sweeping x itself (the reference's form), up to FP32 rounding of d; the
// residual, its norm and the stopping test are FP64, so the solve converges to tolerances that
// an all-FP32 multigrid cannot reach.
//   FIRST: x = initial guess (the slice arrays), r from x, 4 sweeps on d from zero.
//   else:  x, r from the previous iteration, d from the interpolated coarse correction, 8 sweeps
//          (the up-sweep of this V-cycle and the down-sweep of the next).
// Both end with x += d, the new FP64 residual on the tile and its ring, its max norm, the FP32
// residual of the tile (next right-hand side) and its restriction to level 1.
// ------------------------------------------------------------------------------------------
template <int T, int NSW>
struct RefineSmem {
    static constexpr int H = NSW + 2;
    static constexpr int E = T + 2 * H;
    static constexpr int Q = T + 2;
    static constexpr int EC = E / 2 + 3;
    static constexpr size_t bytes() {
        return (size_t)2 * E * E * sizeof(double) + (size_t)(6 * E * E + 2 * Q * Q + 2 * EC * EC) * sizeof(float);
    }
};

// DIN: the correction d starts from P.up[0] (the first 4 sweeps of the split level-0 phase)
// instead of the interpolated coarse correction
template <bool CELL, bool FIRST, int NSW, bool DIN = false>
__device__ __forceinline__ void mg_refine_tile(const MGSolveArgs<float>& P, int slot_in, int bx, int by,
                                               unsigned char* smem_raw, double& bmax, double& brhs) {
    constexpr int T = 16, NT = 256;
    using SM = RefineSmem<T, NSW>;
    constexpr int H = SM::H, E = SM::E, Q = SM::Q;
    double (*sx)[E * E] = reinterpret_cast<double (*)[E * E]>(smem_raw);                     // x, 2 comps
    float* fbase = reinterpret_cast<float*>(smem_raw + 2 * E * E * sizeof(double));
    float (*sd)[E * E] = reinterpret_cast<float (*)[E * E]>(fbase);                          // d
    float (*srh)[E * E] = reinterpret_cast<float (*)[E * E]>(fbase + 2 * E * E);             // r (rhs of d)
    float* sa = fbase + 4 * E * E;                                                            // coefficient
    float* sinv = fbase + 5 * E * E;                                                          // 1 / diagonal
    float (*sr)[Q * Q] = reinterpret_cast<float (*)[Q * Q]>(fbase + 6 * E * E);              // new residual
    constexpr int EC = SM::EC;
    float (*sc)[EC * EC] = reinterpret_cast<float (*)[EC * EC]>(fbase + 6 * E * E + 2 * Q * Q);  // coarse
    const MGLev& L = P.lev[0];
    const float facx = P.facx[0], facy = P.facy[0];
    const double dfx = (double)facx, dfy = (double)facy;
    const int t0i = L.vlo + bx * T, t0j = L.vlo + by * T;
    const int ti0 = t0i - H, tj0 = t0j - H;
    const MV<float> crse = (P.sb == 1) ? MV<float>{{P.cor[1], P.cor[1] + (size_t)P.lev[1].w * P.lev[1].h}, P.lev[1].w, 0}
                                       : MV<float>{{P.up[1], P.up[1] + (size_t)P.lev[1].w * P.lev[1].h}, P.lev[1].w, 0};
    const size_t n0 = (size_t)L.w * L.h;
    const double* xin = P.x64[slot_in];
    const float* rin = P.r32[slot_in];
    double* xout = P.x64[slot_in ^ (FIRST ? 0 : 1)];
    float* rout = P.r32[slot_in ^ (FIRST ? 0 : 1)];
    auto inside = [&](int i, int j) { return i >= L.vlo && i <= L.vhi_i && j >= L.vlo && j <= L.vhi_j; };
    const int ci0 = (ti0 >> 1) - 1, cj0 = (tj0 >> 1) - 1;  // coarse origin of the interpolation
    __syncthreads();
    // asynchronous copies of everything the tile reads (zero-filled outside the valid box); in
    // FIRST the FP32 initial guess lands in sd and is widened below
#pragma unroll
    for (int e0 = 0; e0 < E * E; e0 += NT) {
        const int e = e0 + threadIdx.x;
        if (e >= E * E) break;
        const int i = ti0 + e % E, j = tj0 + e / E;
        const bool v = inside(i, j);
        const size_t id = v ? (size_t)j * L.w + i : 0;
        cp_async_el<float>(&sa[e], v ? &P.a0(i, j, 0) : P.a0.p[0], v);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (FIRST) {
                cp_async_el<float>(&sd[c][e], v ? &P.sol(i, j, c) : P.sol.p[c], v);
                cp_async_el<float>(&srh[c][e], v ? &P.rhs(i, j, c) : P.rhs.p[c], v);  // f for now, r below
            } else {
                cp_async_el<double>(&sx[c][e], xin + c * n0 + id, v);
                cp_async_el<float>(&srh[c][e], rin + c * n0 + id, v);
                if (DIN) cp_async_el<float>(&sd[c][e], P.up[0] + c * n0 + id, v);
            }
        }
    }
    if (!FIRST && !DIN) {
        const MGLev& C = P.lev[1];
        for (int e = threadIdx.x; e < EC * EC; e += NT) {
            const int ic = ci0 + e % EC, jc = cj0 + e / EC;
            const bool v = ic >= 0 && ic < C.w && jc >= 0 && jc < C.h;
#pragma unroll
            for (int c = 0; c < 2; ++c) cp_async_el<float>(&sc[c][e], v ? &crse(ic, jc, c) : crse.p[c], v);
        }
    }
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int e0 = 0; e0 < E * E; e0 += NT) {
        const int e = e0 + threadIdx.x;
        if (e >= E * E) break;
        const int i = ti0 + e % E, j = tj0 + e / E;
        const bool v = inside(i, j);
        sinv[e] = v ? mg_diag_inv<float, CELL>(L, i, j, sa[e], facx, facy) : 0.f;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (FIRST) {
                sx[c][e] = (double)sd[c][e];
                sd[c][e] = 0.f;
            } else if (!DIN) {
                const float* q = sc[c];
                sd[c][e] = v ? mg_interp1f<float, CELL>([&](int ic, int jc) { return q[(jc - cj0) * EC + (ic - ci0)]; }, i, j) : 0.f;
            }
        }
    }
    __syncthreads();
    if (FIRST) {
        // r = f + a x - Lap(x) in FP64 wherever the sweeps read it (all but the outer ring)
        float rr[(E * E + NT - 1) / NT][2];
#pragma unroll
        for (int e0 = 0, q = 0; e0 < E * E; e0 += NT, ++q) {
            const int e = e0 + threadIdx.x;
            rr[q][0] = rr[q][1] = 0.f;
            if (e >= E * E) break;
            const int li = e % E, lj = e / E;
            const int i = ti0 + li, j = tj0 + lj;
            if (li == 0 || lj == 0 || li == E - 1 || lj == E - 1 || !inside(i, j)) continue;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double* x = sx[c];
                const double r = (double)srh[c][e] + (double)sa[e] * x[e] -
                                 mg_lap<double, CELL>(L, i, j, x[e], x[e - 1], x[e + 1], x[e - E], x[e + E], dfx, dfy);
                rr[q][c] = (float)r;
                if (li >= H && li < H + T && lj >= H && lj < H + T) brhs = fmax(brhs, fabs((double)srh[c][e]));
            }
        }
        __syncthreads();
#pragma unroll
        for (int e0 = 0, q = 0; e0 < E * E; e0 += NT, ++q) {
            const int e = e0 + threadIdx.x;
            if (e >= E * E) break;
            srh[0][e] = rr[q][0];
            srh[1][e] = rr[q][1];
        }
        __syncthreads();
    }
    constexpr int HW = (E - 2) / 2;  // points of one colour per interior row
    for (int s = 0; s < NSW; ++s) {
#pragma unroll
        for (int q0 = 0; q0 < (E - 2) * HW; q0 += NT) {
            const int q = q0 + threadIdx.x;
            if (q >= (E - 2) * HW) break;
            const int lj = 1 + q / HW, k = q - (lj - 1) * HW;
            const int par = (s + ti0 + tj0 + lj) & 1;
            const int li = (par ? 1 : 2) + 2 * k;
            const int i = ti0 + li, j = tj0 + lj;
            if (!inside(i, j)) continue;
            const int e = lj * E + li;
            const float inv = sinv[e];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const float* qq = sd[c];
                sd[c][e] = mg_gs_inv<float, CELL>(L, i, j, qq[e - 1], qq[e + 1], qq[e - E], qq[e + E], srh[c][e], inv, facx, facy);
            }
        }
        __syncthreads();
    }
    // x += d where d is exact (distance >= NSW from the edge of the loaded region)
#pragma unroll
    for (int e0 = 0; e0 < E * E; e0 += NT) {
        const int e = e0 + threadIdx.x;
        if (e >= E * E) break;
        const int li = e % E, lj = e / E;
        if (li < NSW || lj < NSW || li >= E - NSW || lj >= E - NSW) continue;
        sx[0][e] += (double)sd[0][e];
        sx[1][e] += (double)sd[1][e];
    }
    __syncthreads();
    // FP64 residual of the new x with the original right-hand side f on the tile and its ring
    for (int e = threadIdx.x; e < Q * Q; e += NT) {
        const int ri = e % Q, rj = e / Q;
        const int i = t0i - 1 + ri, j = t0j - 1 + rj;
        const bool v = inside(i, j);
        const bool in_tile = ri >= 1 && ri <= T && rj >= 1 && rj <= T;
        const int k = (rj + H - 1) * E + (ri + H - 1);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            float rf = 0.f;
            if (v) {
                const double* x = sx[c];
                const double f = (double)P.rhs(i, j, c);
                const double r = f + (double)sa[k] * x[k] -
                                 mg_lap<double, CELL>(L, i, j, x[k], x[k - 1], x[k + 1], x[k - E], x[k + E], dfx, dfy);
                if (in_tile) bmax = fmax(bmax, fabs(r));
                rf = (float)r;
            }
            sr[c][e] = rf;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < T * T; e += NT) {
        const int li = e % T, lj = e / T;
        const int i = t0i + li, j = t0j + lj;
        if (i > L.vhi_i || j > L.vhi_j) continue;
        const int k = (lj + H) * E + (li + H);
        const size_t id = (size_t)j * L.w + i;
        const int kr = (lj + 1) * Q + (li + 1);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            xout[c * n0 + id] = sx[c][k];
            rout[c * n0 + id] = sr[c][kr];
        }
    }
    {
        const MGLev& C = P.lev[1];
        MV<float> cres{{P.res[1], P.res[1] + (size_t)C.w * C.h}, C.w, 0};
        const int ci0 = max(C.vlo, (t0i + 1) >> 1), cj0 = max(C.vlo, (t0j + 1) >> 1);
        const int ci1 = min(C.vhi_i, (t0i + T - 1) >> 1), cj1 = min(C.vhi_j, (t0j + T - 1) >> 1);
        const int cw = ci1 - ci0 + 1, ch = cj1 - cj0 + 1;
        if (cw > 0 && ch > 0) {
            for (int e = threadIdx.x; e < cw * ch; e += NT) {
                const int I = ci0 + e % cw, J = cj0 + e / cw;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    auto f = [&](int i, int j) -> float { return sr[c][(j - t0j + 1) * Q + (i - t0i + 1)]; };
                    float v;
                    if (CELL) {
                        v = 0.25f * (f(2 * I, 2 * J) + f(2 * I + 1, 2 * J) + f(2 * I, 2 * J + 1) + f(2 * I + 1, 2 * J + 1));
                    } else {
                        v = (1.f / 16.f) * (f(2 * I - 1, 2 * J - 1) + 2.f * f(2 * I, 2 * J - 1) + f(2 * I + 1, 2 * J - 1) +
                                            2.f * f(2 * I - 1, 2 * J) + 4.f * f(2 * I, 2 * J) + 2.f * f(2 * I + 1, 2 * J) +
                                            f(2 * I - 1, 2 * J + 1) + 2.f * f(2 * I, 2 * J + 1) + f(2 * I + 1, 2 * J + 1));
                    }
                    cres(I, J, c) = v;
                }
            }
        }
    }
}

// T0: tile edge of level 0 (16, or 32 on large grids: a 4-sweep phase then loads 44^2 points per
// 32^2 tile instead of 28^2 per 16^2, 1.6x less halo work; the sweeps give the same values). With
// T0 = 32 level 0 runs without FP64 refinement, and in double precision in the split form.
// TB: the coarsest level is too large for one block's shared memory (Multigrid::tile_bottom) and
// its sweeps run as grid-wide tile phases; a separate instance, so that the common one keeps its
// register allocation.
template <class R, bool CELL, int T0 = 16, bool TB = false>
__global__ void __launch_bounds__(256, 2) k_mg_solve(MGSolveArgs<R> P) {
    HPQ_PDL_ENTRY();
    extern __shared__ unsigned char smem_raw[];
    __shared__ int s_go;
    __shared__ double s_target, s_maxn;
    constexpr bool kFloat = std::is_same<R, float>::value;
    constexpr bool kRefinable = kFloat && T0 == 16;
    const bool refine = kRefinable && P.refine != 0;  // FP64 refinement of level 0 (tight tolerances)
    const bool split = (T0 != 16 && !kFloat) || P.split0 != 0;
    Ctl* ctl = P.ctl;
    unsigned int* bar = ctl->mgp_bar;  // arrivals (mgp_bar[1] unused)
    int* err = &ctl->mgp_bar_err;
    unsigned int bseq = 0;  // grid barriers passed
    const int nb = gridDim.x;
    // trace: [0] count, [1..127] block 0 after each grid barrier; [128] count, [129..255] the
    // moment the phase's work of block 2, the first tile block, is done
    int nstamp = 0, nwork = 0;
    auto stamp = [&]() {
        if (P.trace && blockIdx.x == 0 && threadIdx.x == 0 && nstamp < 126) P.trace[1 + nstamp++] = tc_clock_ns();
    };
    auto wstamp = [&](int who) {
        if (P.trace && threadIdx.x == 0 && (int)blockIdx.x == who && nwork < 126) P.trace[129 + nwork++] = tc_clock_ns();
    };
    stamp();
    auto base = [&](int l) {
        SmoothArgs<R> a{};
        a.L = P.lev[l];
        if (l + 1 < P.nl) a.Lc = P.lev[l + 1];
        a.facx = P.facx[l];
        a.facy = P.facy[l];
        a.ctl = ctl;
        return a;
    };
    // blocks 0 and 1 run the coarse levels, one component each, and keep them resident in their
    // shared memory; the tiles go to the other blocks (the launch has at least 3 blocks)
    const int tb = (int)blockIdx.x - 2, ntb = nb - 2;
    const bool tile_block = blockIdx.x >= 2;
    // levels >= 1 also take 32^2 tiles in the 32^2 form where there are enough of them
    // (bit l of P.l32_mask)
    auto big = [&](int l) { return T0 == 32 && ((P.l32_mask >> l) & 1u) != 0; };
    auto ntiles = [&](int l, int& ntx) {
        const MGLev& L = P.lev[l];
        const int T = l == 0 ? T0 : big(l) ? 32 : 16;
        ntx = (L.vhi_i - L.vlo + T) / T;
        return ntx * ((L.vhi_j - L.vlo + T) / T);
    };
    // coefficient of level l from level l-1 (average_down_acoef), grid-stride
    auto restrict_acf = [&](int l) {
        const MGLev& C = P.lev[l];
        MV<R> fine = (l == 1) ? P.a0 : mg_own<R>(P.acf, P.lev, l - 1, 1);
        MV<R> crse = mg_own<R>(P.acf, P.lev, l, 1);
        const int vw = C.vhi_i - C.vlo + 1, vh = C.vhi_j - C.vlo + 1;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < vw * vh; k += nb * blockDim.x) {
            const int i = C.vlo + k % vw, j = C.vlo + k / vw;
            crse(i, j, 0) = mg_restrict1<R, CELL>(fine, i, j, 0);
        }
    };
    // the bottom blocks build their coefficient hierarchy in the phase before the first bottom
    // solve (they have no tiles there): from the coefficient of level sb - 1, written grid-wide in
    // the phase before that (level 0's is an input)
    auto prebuild = [&]() {
        if constexpr (!TB) {
            if (blockIdx.x < 2) {
                const int l = P.sb - 1;
                const MV<R> fine = (l == 0) ? P.a0 : mg_own<R>(P.acf, P.lev, l, 1);
                mg_bottom_prebuild<R, CELL, 1>(P.coarse, fine, P.facx[P.sb], P.facy[P.sb], smem_raw);
            }
        }
    };
    double bmax = 0, brhs = 0;
    // ---- first smoothing of level 0 (residual, restriction, norms) and the level-1 coefficient
    {
        SmoothArgs<R> a = base(0);
        a.out = mg_own<R>(P.cor, P.lev, 0); a.rhs = P.rhs; a.acf = P.a0; a.in = P.sol;
        a.crse_res = mg_own<R>(P.res, P.lev, 1);
        int ntx;
        const int nt = ntiles(0, ntx);
        for (int t = tb; tile_block && t < nt; t += ntb) {
            bool done = false;
            if constexpr (kRefinable) {
                if (refine) { mg_refine_tile<CELL, true, 4>(P, 0, t % ntx, t / ntx, smem_raw, bmax, brhs); done = true; }
            }
            if (!done)
                mg_smooth_tile<R, CELL, T0, MG_INIT_VIEW, true, true, MG_NORM_FIRST, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
        }
        restrict_acf(1);
        if (P.sb == 1) prebuild();
        block_max2(bmax, brhs);
        if (threadIdx.x == 0) {
            atomic_max_nonneg(&ctl->mgp_norm[0], bmax);
            atomic_max_nonneg(&ctl->mgp_rhsnorm, brhs);
        }
    }
    if (!grid_barrier(bar, err, bseq)) return;
    stamp();
    if (threadIdx.x == 0) {
        const double r0 = atomic_read(&ctl->mgp_norm[0]), m0 = atomic_read(&ctl->mgp_rhsnorm);
        s_maxn = (m0 >= r0) ? m0 : r0;
        s_target = fmax(P.tol_abs, fmax(P.tol_rel, 1.e-16) * s_maxn);
        s_go = !(r0 <= s_target);
        if (blockIdx.x == 0) { ctl->mg_target = s_target; ctl->mg_maxnorm = s_maxn; }
    }
    __syncthreads();
    int it = 0;
    while (s_go) {
        // down: levels 1 .. sb-1 (zero initial guess), residual restricted to the next level
        for (int l = 1; l < P.sb; ++l) {
            SmoothArgs<R> a = base(l);
            a.out = mg_own<R>(P.cor, P.lev, l); a.rhs = mg_own<R>(P.res, P.lev, l);
            a.acf = mg_own<R>(P.acf, P.lev, l, 1); a.crse_res = mg_own<R>(P.res, P.lev, l + 1);
            int ntx;
            const int nt = ntiles(l, ntx);
            bool done = false;
            if constexpr (T0 == 32) {
                if (big(l)) {
                    for (int t = tb; tile_block && t < nt; t += ntb)
                        mg_smooth_tile<R, CELL, 32, MG_INIT_ZERO, true, true, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                    done = true;
                }
            }
            if (!done)
                for (int t = tb; tile_block && t < nt; t += ntb)
                    mg_smooth_tile<R, CELL, 16, MG_INIT_ZERO, true, true, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
            if (it == 0) restrict_acf(l + 1);
            if (it == 0 && l == P.sb - 1) prebuild();
            wstamp(2);
            if (!grid_barrier(bar, err, bseq)) return;
            stamp();
        }
        if constexpr (TB) {
            // the coarsest level: ns_bottom sweeps from a zero guess as grid-wide phases of 4
            // sweeps (the last of 2 when ns_bottom is not a multiple of 4) on 16^2 tiles with
            // their halos, alternating between up and cor so that the last phase writes cor
            const int l = P.sb;
            const MGLev& L = P.lev[l];
            const int ns = P.coarse.ns_bottom, n2 = (ns % 4) ? 1 : 0, nph = ns / 4 + n2;
            const int ntx = (L.vhi_i - L.vlo + 16) / 16, nt = ntx * ((L.vhi_j - L.vlo + 16) / 16);
            for (int ph = 0; ph < nph; ++ph) {
                const bool to_cor = ((nph - 1 - ph) & 1) == 0;
                SmoothArgs<R> a = base(l);
                a.rhs = mg_own<R>(P.res, P.lev, l);
                a.acf = mg_own<R>(P.acf, P.lev, l, 1);
                a.out = to_cor ? mg_own<R>(P.cor, P.lev, l) : mg_own<R>(P.up, P.lev, l);
                a.in = to_cor ? mg_own<R>(P.up, P.lev, l) : mg_own<R>(P.cor, P.lev, l);
                const bool two = n2 && ph == nph - 1;
                for (int t = tb; tile_block && t < nt; t += ntb) {
                    if (ph == 0) {
                        if (two) mg_smooth_tile<R, CELL, 16, MG_INIT_ZERO, false, false, MG_NORM_NONE, 2>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                        else mg_smooth_tile<R, CELL, 16, MG_INIT_ZERO, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                    } else {
                        if (two) mg_smooth_tile<R, CELL, 16, MG_INIT_VIEW, false, false, MG_NORM_NONE, 2>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                        else mg_smooth_tile<R, CELL, 16, MG_INIT_VIEW, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                    }
                }
                if (ph + 1 < nph && !grid_barrier(bar, err, bseq)) return;
            }
        } else if (blockIdx.x < 2) {
            // levels sb .. nl-1: component c in block c (the components share the operator and
            // are coupled only through the norms, which are taken on level 0)
            const int c = (int)blockIdx.x;
            const size_t nsb = (size_t)P.lev[P.sb].w * P.lev[P.sb].h;
            // (the lane form in every persistent kernel but the single-precision 32^2 one, which
            // has no registers to spare; the multi-kernel form keeps the block form, and the
            // persistent solve is checked against it)
            mg_bottom_block<R, CELL, false, 1, (sizeof(R) == 8 || T0 == 16)>(P.coarse, P.res[P.sb] + c * nsb, P.acf[P.sb], P.cor[P.sb] + c * nsb,
                                               P.facx[P.sb], P.facy[P.sb], smem_raw, false,
                                               (P.trace && c == 0) ? P.trace + 256 : nullptr);
        }
        wstamp(2);
        if (!grid_barrier(bar, err, bseq)) return;
        stamp();
        // up: levels sb-1 .. 1, interpolation of the coarser correction + 4 sweeps
        for (int l = P.sb - 1; l >= 1; --l) {
            SmoothArgs<R> a = base(l);
            a.out = mg_own<R>(P.up, P.lev, l); a.rhs = mg_own<R>(P.res, P.lev, l);
            a.acf = mg_own<R>(P.acf, P.lev, l, 1); a.in = mg_own<R>(P.cor, P.lev, l);
            a.crse_in = (l + 1 == P.sb) ? mg_own<R>(P.cor, P.lev, P.sb) : mg_own<R>(P.up, P.lev, l + 1);
            int ntx;
            const int nt = ntiles(l, ntx);
            bool done = false;
            if constexpr (T0 == 32) {
                if (big(l)) {
                    for (int t = tb; tile_block && t < nt; t += ntb)
                        mg_smooth_tile<R, CELL, 32, MG_INIT_INTERP, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                    done = true;
                }
            }
            if (!done)
                for (int t = tb; tile_block && t < nt; t += ntb)
                    mg_smooth_tile<R, CELL, 16, MG_INIT_INTERP, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
            wstamp(2);
            if (!grid_barrier(bar, err, bseq)) return;
            stamp();
        }
        // level 0, split form (double precision on large grids): interpolation + 4 up-sweeps
        // from cor[0] into up[0], barrier, 4 down-sweeps + residual + restriction + norm from
        // up[0] back into cor[0]
        // (single precision: the first 4 sweeps of the correction d, from the interpolated coarse
        // correction with the FP32 residual as right-hand side, go to up[0]; the second pass
        // reloads d, sweeps 4 more times, adds it to the FP64 solution and forms the residual)
        if (split) {
            {
                SmoothArgs<R> a = base(0);
                a.crse_in = (P.sb == 1) ? mg_own<R>(P.cor, P.lev, 1) : mg_own<R>(P.up, P.lev, 1);
                a.out = mg_own<R>(P.up, P.lev, 0);
                a.acf = P.a0;
                int ntx;
                const int nt = ntiles(0, ntx);
                bool done = false;
                if constexpr (kRefinable) {
                    if (refine) {
                        const size_t n0 = (size_t)P.lev[0].w * P.lev[0].h;
                        a.rhs = MV<R>{{P.r32[it & 1], P.r32[it & 1] + n0}, P.lev[0].w, 0};
                        for (int t = tb; tile_block && t < nt; t += ntb)
                            mg_smooth_tile<R, CELL, 16, MG_INIT_INTERP0, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                        done = true;
                    }
                }
                if (!done) {
                    a.in = mg_own<R>(P.cor, P.lev, 0);
                    a.rhs = P.rhs;
                    for (int t = tb; tile_block && t < nt; t += ntb)
                        mg_smooth_tile<R, CELL, T0, MG_INIT_INTERP, false, false, MG_NORM_NONE, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                }
                wstamp(2);
            }
            if (!grid_barrier(bar, err, bseq)) return;
            stamp();
            {
                int ntx;
                const int nt = ntiles(0, ntx);
                bmax = 0;
                bool done = false;
                if constexpr (kRefinable) {
                    if (refine) {
                        for (int t = tb; tile_block && t < nt; t += ntb)
                            mg_refine_tile<CELL, false, 4, true>(P, it & 1, t % ntx, t / ntx, smem_raw, bmax, brhs);
                        done = true;
                    }
                }
                if (!done) {
                    SmoothArgs<R> a = base(0);
                    a.in = mg_own<R>(P.up, P.lev, 0); a.out = mg_own<R>(P.cor, P.lev, 0);
                    a.rhs = P.rhs; a.acf = P.a0;
                    a.crse_res = mg_own<R>(P.res, P.lev, 1);
                    for (int t = tb; tile_block && t < nt; t += ntb)
                        mg_smooth_tile<R, CELL, T0, MG_INIT_VIEW, true, true, MG_NORM_ITER, 4>(a, t % ntx, t / ntx, false, smem_raw, bmax, brhs);
                }
                block_max2(bmax, brhs);
                if (threadIdx.x == 0) atomic_max_nonneg(&ctl->mgp_norm[(it + 1) & 1], bmax);
                wstamp(2);
            }
        } else
        // level 0: up-sweep and the next down-sweep (8 colour sweeps), residual, restriction,
        // norm; the solution alternates between cor[0] and up[0] by iteration parity
        {
            SmoothArgs<R> a = base(0);
            a.in = mg_own<R>(P.cor, P.lev, 0); a.out = mg_own<R>(P.up, P.lev, 0);
            a.in2 = mg_own<R>(P.up, P.lev, 0); a.out2 = mg_own<R>(P.cor, P.lev, 0);
            a.rhs = P.rhs; a.acf = P.a0;
            a.crse_in = (P.sb == 1) ? mg_own<R>(P.cor, P.lev, 1) : mg_own<R>(P.up, P.lev, 1);
            a.crse_res = mg_own<R>(P.res, P.lev, 1);
            int ntx;
            const int nt = ntiles(0, ntx);
            bmax = 0;
            for (int t = tb; tile_block && t < nt; t += ntb) {
                bool done = false;
                if constexpr (kRefinable) {
                    if (refine) { mg_refine_tile<CELL, false, 8>(P, it & 1, t % ntx, t / ntx, smem_raw, bmax, brhs); done = true; }
                }
                if constexpr (T0 == 16 || kFloat) {
                    if (!done)
                        mg_smooth_tile<R, CELL, T0, MG_INIT_INTERP, true, true, MG_NORM_ITER, 8>(a, t % ntx, t / ntx, (it & 1) != 0, smem_raw, bmax, brhs);
                }
            }
            block_max2(bmax, brhs);
            if (threadIdx.x == 0) atomic_max_nonneg(&ctl->mgp_norm[(it + 1) & 1], bmax);
            wstamp(2);
        }
        if (!grid_barrier(bar, err, bseq)) return;
        stamp();
        ++it;
        if (threadIdx.x == 0) {
            const double norm = atomic_read(&ctl->mgp_norm[it & 1]);
            int go = 1, status = 0;
            if (norm <= s_target) go = 0;
            else if (norm > 1.e20 * s_maxn) { go = 0; status = 2; }
            else if (it >= P.maxiter) { go = 0; status = 1; }
            s_go = go;
            if (blockIdx.x == 0) {
                ctl->mgp_norm[(it + 1) & 1] = 0;  // read by every block at the previous decision
                ctl->mg_total_iters += 1;
                if (status && !ctl->mg_status) ctl->mg_status = status;
                __threadfence();
            }
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->mg_iter = it;
        ctl->mg_go = 0;
        if (P.trace) P.trace[0] = nstamp;
    }
    if (P.trace && blockIdx.x == 2 && threadIdx.x == 0) P.trace[128] = nwork;
    // solution: the last level-0 output (cor[0] after an even number of cycles, else up[0]; the
    // FP64 solution slot it & 1 in single precision)
    const MV<R> fin = ((it & 1) && !split) ? mg_own<R>(P.up, P.lev, 0) : mg_own<R>(P.cor, P.lev, 0);
    const MGLev& L = P.lev[0];
    const int vw = L.vhi_i - L.vlo + 1, vh = L.vhi_j - L.vlo + 1;
    const size_t n0 = (size_t)L.w * L.h;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < vw * vh; k += nb * blockDim.x) {
        const int i = L.vlo + k % vw, j = L.vlo + k / vw;
        if (refine) {
            const double* x = P.x64[it & 1];
            P.sol(i, j, 0) = (R)x[(size_t)j * L.w + i];
            P.sol(i, j, 1) = (R)x[n0 + (size_t)j * L.w + i];
        } else {
            P.sol(i, j, 0) = fin(i, j, 0);
            P.sol(i, j, 1) = fin(i, j, 1);
        }
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
    size_t bottom_smem = 0;   // single-block bottom solve, both components (k_mg_bottom)
    size_t bottom_smem1 = 0;  // one component (each bottom block of the persistent solve)
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
            for (int l = s0; l < nl; ++l) tot += 8 * (size_t)lev[l].w * lev[l].h;
            return tot * sizeof(R);
        };
        sb = nl - 1;
        for (int l = 1; l < nl; ++l) if (smem_from(l) <= 160 * 1024 && (long long)lev[l].w * lev[l].h <= 4096) { sb = l; break; }
        if (nl - sb > 16) sb = nl - 16;
        bottom_smem = smem_from(sb);
        // the persistent solve's two bottom blocks carry one component each: 5 planes per level
        bottom_smem1 = bottom_smem / 8 * 5;
        coarse.garena = nullptr;
        if (bottom_smem > kBottomSmemMax) {
            // the coarsest level alone is too large for shared memory: the bottom block works on
            // the same arena in global memory (L2-resident), with the same arithmetic
            HPQ_CUDA(cudaMalloc(&coarse.garena, bottom_smem));
            HPQ_CUDA(cudaMemset(coarse.garena, 0, bottom_smem));
            bottom_smem = 0;
            bottom_smem1 = 0;
        }
        coarse.nl = nl - sb;
        // the bottom solve of HpMultiGrid's CPU build (HpMultiGrid.cpp:1584-1592): 16 sweeps, or
        // the longest side of the coarsest level rounded up to an even count when that is more
        // (grids that stop coarsening early, e.g. 100 x 72 -> 25 x 18)
        coarse.ns_bottom = std::max(16, (std::max(lev[nl - 1].w, lev[nl - 1].h) + 1) / 2 * 2);
        // HPQ_MG_WARP=1 in the environment runs the smallest coarse levels on one warp (measured
        // slower at 255^2: 10.8 us instead of 7.0 for levels 9^2 and 5^2, so off by default)
        const char* ew = getenv("HPQ_MG_WARP");
        coarse.lw = coarse.nl;
        if (ew && ew[0] == '1')
            for (int l = sb; l < nl; ++l)
                if ((long long)lev[l].w * lev[l].h <= kWarpLevelPoints) { coarse.lw = l - sb; break; }
        size_t off = 0;
        for (int l = sb; l < nl; ++l) {
            coarse.L[l - sb] = lev[l];
            coarse.poff[l - sb] = off;
            off += (size_t)lev[l].w * lev[l].h;
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
        if (cell) setup_persistent<true>(); else setup_persistent<false>();
    }

    // persistent solve: one cooperative launch with as many co-resident blocks as there are
    // level-0 tiles, at most (HPQ_MG=kernels in the environment selects the multi-kernel form)
    bool coop_ok = false;
    int coop_blocks = 0;
    size_t coop_smem = 0;
    double* x64[2] = {nullptr, nullptr};  // single precision: FP64 level-0 solution (refinement)
    R* r32[2] = {nullptr, nullptr};
    unsigned long long* trace = nullptr;  // HPQ_MG_TRACE=1: phase timestamps of the last solve
    bool split0 = false;                  // level-0 phase split in two (MGSolveArgs::split0)
    int refine_force = -1;                // single precision: -1 by tolerance, 0 plain FP32, 1 FP64 refinement
    bool use32 = false;                   // level-0 tiles of 32^2 (k_mg_solve<R, CELL, 32>) for unrefined solves
    bool tile_bottom = false;             // the coarsest level's sweeps as grid-wide tile phases (TB)
    int coop_blocks32 = 0;
    size_t coop_smem32 = 0;
    bool split32 = true;                  // level 0 of the 32^2 form as two 4-sweep passes
    unsigned int l32_mask = 0;            // levels >= 1 of the 32^2 form in 32^2 tiles too (bit l)

    // Prints the phase durations of the last persistent solve (microseconds) to stderr.
    void print_trace() const {
        if (!trace) return;
        std::vector<unsigned long long> h(320);
        if (cudaMemcpy(h.data(), trace, 320 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess) return;
        const int n = (int)std::min<unsigned long long>(h[0], 126);
        std::string line = "hpmg phases (us):", work = "hpmg work done at (us):";
        for (int k = 1; k < n; ++k) {
            char buf[32];
            snprintf(buf, sizeof(buf), " %.2f", (double)(h[1 + k] - h[k]) / 1000.0);
            line += buf;
        }
        // block 2 (the first tile block) finished the work of phase w + 2 (the first smoothing, phase 1, has no stamp)
        // at h[129 + w]; relative to the start of that phase (the barrier before it)
        const int nw = (int)std::min<unsigned long long>(h[128], 126);
        for (int w = 0; w < nw && w + 2 < n; ++w) {
            char buf[32];
            snprintf(buf, sizeof(buf), " %.2f", ((double)h[129 + w] - (double)h[w + 2]) / 1000.0);
            work += buf;
        }
        // the last coarse-level solve: set-up, each level down, coarsest, each level up, store
        std::string bot = "hpmg bottom steps (us):";
        const int nb = (int)std::min<unsigned long long>(h[256], 60);
        for (int k = 1; k < nb; ++k) {
            char buf[32];
            snprintf(buf, sizeof(buf), " %.2f", (double)(h[257 + k] - h[256 + k]) / 1000.0);
            bot += buf;
        }
        fprintf(stderr, "%s\n%s\n%s\n", line.c_str(), work.c_str(), bot.c_str());
    }

    template <bool CELL>
    void setup_persistent() {
        coop_ok = false;
        const char* e = getenv("HPQ_MG");
        if (e && std::string(e) == "kernels") return;
        if (nl > kMGMaxLevels) return;
        coop_smem = std::max({SmoothSmem<16, 8>::template bytes<R>(), SmoothSmem<16, 4>::template bytes<R>(), bottom_smem1});
        if (const char* t = getenv("HPQ_MG_TRACE")) {
            if (t[0] == '1') {
                HPQ_CUDA(cudaMalloc(&trace, 320 * sizeof(unsigned long long)));
                HPQ_CUDA(cudaMemset(trace, 0, 320 * sizeof(unsigned long long)));
            }
        }
        if (std::is_same<R, float>::value) {
            coop_smem = std::max({coop_smem, RefineSmem<16, 8>::bytes(), RefineSmem<16, 4>::bytes()});
            const size_t n0 = (size_t)lev[0].w * lev[0].h;
            for (int k = 0; k < 2; ++k) {
                HPQ_CUDA(cudaMalloc(&x64[k], 2 * n0 * sizeof(double)));
                HPQ_CUDA(cudaMalloc(&r32[k], 2 * n0 * sizeof(R)));
                HPQ_CUDA(cudaMemset(x64[k], 0, 2 * n0 * sizeof(double)));
                HPQ_CUDA(cudaMemset(r32[k], 0, 2 * n0 * sizeof(R)));
            }
        }
        // a global-memory arena only ever holds the coarsest level alone (sb == nl - 1): the
        // persistent kernel then sweeps it as grid-wide tile phases, and otherwise its bottom block
        // works in shared memory
        if (coarse.garena != nullptr && sb != nl - 1)
            throw CudaError("hpmg: coarse levels exceed shared memory below the coarsest level");
        tile_bottom = coarse.garena != nullptr;
        auto kern = tile_bottom ? k_mg_solve<R, CELL, 16, true> : k_mg_solve<R, CELL, 16, false>;
        HPQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coop_smem));
        int dev = 0, sms = 0, coop = 0, per = 0;
        HPQ_CUDA(cudaGetDevice(&dev));
        HPQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        HPQ_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        HPQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, coop_smem));
        const MGLev& L = lev[0];
        const int nt0 = ((L.vhi_i - L.vlo + 16) / 16) * ((L.vhi_j - L.vlo + 16) / 16);
        coop_blocks = std::min(per * sms, nt0 + 2);  // + blocks 0 and 1 for the coarse levels
        coop_ok = coop && per > 0 && coop_blocks >= 3;
        // split level-0 phase once every tile block sweeps at least 4 tiles (HPQ_MG_SPLIT=0/1
        // in the environment forces either form)
        const char* es = getenv("HPQ_MG_SPLIT");
        split0 = es ? (es[0] == '1') : (nt0 >= 4 * std::max(coop_blocks - 2, 1));
        // single precision: HPQ_MG_REFINE=0/1 forces plain FP32 V-cycles or FP64 refinement
        const char* er = getenv("HPQ_MG_REFINE");
        refine_force = er ? (er[0] == '1' ? 1 : 0) : -1;
        // 32^2 level-0 tiles in single precision once there are two per tile block
        // (HPQ_MG_T0=16/32 forces either form)
        const int nt32 = ((L.vhi_i - L.vlo + 32) / 32) * ((L.vhi_j - L.vlo + 32) / 32);
        const char* e32 = getenv("HPQ_MG_T0");
        // (the 32^2 form is taken where it keeps the blocks per SM of the 16^2 form)
        use32 = coop_ok && (e32 ? std::atoi(e32) == 32 : nt32 >= 2 * std::max(coop_blocks - 2, 1));
        if (use32) {
            coop_smem32 = std::max({SmoothSmem<32, 4>::template bytes<R>(), SmoothSmem<16, 4>::template bytes<R>(), bottom_smem1});
            // single precision may run level 0 as one 8-sweep pass of 32^2 tiles
            if (std::is_same<R, float>::value) coop_smem32 = std::max(coop_smem32, SmoothSmem<32, 8>::template bytes<R>());
            const char* es32 = getenv("HPQ_MG_SPLIT");
            split32 = std::is_same<R, float>::value ? (es32 ? es32[0] == '1' : true) : true;
            auto k32 = tile_bottom ? k_mg_solve<R, CELL, 32, true> : k_mg_solve<R, CELL, 32, false>;
            HPQ_CUDA(cudaFuncSetAttribute(k32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coop_smem32));
            int per32 = 0;
            HPQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k32, 256, coop_smem32));
            coop_blocks32 = std::min(per32 * sms, nt32 + 2);
            use32 = per32 > 0 && coop_blocks32 >= 3 && (e32 || per32 >= per);
            // levels >= 1 in 32^2 tiles once they occupy at least half of the tile blocks
            // (HPQ_MG_L1=16/32 forces either form on level 1)
            l32_mask = 0;
            const char* el1 = getenv("HPQ_MG_L1");
            for (int l = 1; l < std::min(sb, 32); ++l) {
                const MGLev& Ll = lev[l];
                const int ntl = ((Ll.vhi_i - Ll.vlo + 32) / 32) * ((Ll.vhi_j - Ll.vlo + 32) / 32);
                const bool on = (l == 1 && el1) ? std::atoi(el1) == 32 : 2 * ntl >= coop_blocks32 - 2;
                if (on) l32_mask |= 1u << l;
            }
        }
    }

    template <bool CELL>
    void solve_persistent(cudaStream_t st, const Slab<R>& S, Ctl* ctl, double tol_rel, double tol_abs, int maxiter) {
        MGSolveArgs<R> P{};
        P.nl = nl;
        P.sb = sb;
        for (int l = 0; l < nl; ++l) {
            P.lev[l] = lev[l];
            P.facx[l] = (R)fac(l, dx);
            P.facy[l] = (R)fac(l, dy);
            P.acf[l] = acf[l]; P.res[l] = res[l]; P.cor[l] = cor[l]; P.up[l] = up[l];
        }
        P.sol = slab_view(S, C_BX, C_BY);
        P.rhs = slab_view(S, C_SY, C_SX);
        P.a0 = slab_view(S, C_CHI, C_CHI);
        P.coarse = coarse;
        P.ctl = ctl;
        P.tol_rel = tol_rel; P.tol_abs = tol_abs; P.maxiter = maxiter;
        P.x64[0] = x64[0]; P.x64[1] = x64[1];
        P.r32[0] = r32[0]; P.r32[1] = r32[1];
        P.trace = trace;
        P.split0 = split0 ? 1 : 0;
        // single precision refines level 0 in FP64 only where the tolerance asks for it: an FP32
        // V-cycle reaches relative residuals well below kRefineTol on its own
        P.refine = std::is_same<R, float>::value && (refine_force >= 0 ? refine_force == 1 : tol_rel < kRefineTol);
        // norms and barrier state; the timeout flag stays set until the step ends, so that after
        // a timeout the remaining solves of the step leave at their first barrier
        static_assert(offsetof(Ctl, mgp_bar_err) - offsetof(Ctl, mgp_rhsnorm) == 32, "Ctl layout");
        HPQ_CUDA(cudaMemsetAsync(&ctl->mgp_rhsnorm, 0, 32, st));
        const bool t32 = use32 && !P.refine;
        if (t32) P.split0 = split32 ? 1 : 0;
        P.l32_mask = t32 ? l32_mask : 0u;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(t32 ? coop_blocks32 : coop_blocks);
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = t32 ? coop_smem32 : coop_smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        void (*kern)(MGSolveArgs<R>) = tile_bottom ? (t32 ? k_mg_solve<R, CELL, 32, true> : k_mg_solve<R, CELL, 16, true>)
                                                   : (t32 ? k_mg_solve<R, CELL, 32, false> : k_mg_solve<R, CELL, 16, false>);
        HPQ_CUDA(cudaLaunchKernelEx(&cfg, kern, P));
        HPQ_LAUNCH_CHECK();
    }
    void release() {
        for (int l = 0; l < nl; ++l) {
            if (l > 0) { cudaFree(acf[l]); cudaFree(res[l]); }
            cudaFree(cor[l]); cudaFree(up[l]);
        }
        if (counter) cudaFree(counter);
        counter = nullptr;
        if (coarse.garena) cudaFree(coarse.garena);
        coarse.garena = nullptr;
        if (trace) cudaFree(trace);
        trace = nullptr;
        for (int k = 0; k < 2; ++k) {
            if (x64[k]) cudaFree(x64[k]);
            if (r32[k]) cudaFree(r32[k]);
            x64[k] = nullptr; r32[k] = nullptr;
        }
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
