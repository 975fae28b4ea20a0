// Slice-loop kernels: plasma initialisation, deposition, explicit Sx/Sy deposition, push;
// beam deposition, push and slice partition; elementwise field kernels.
//
// Every kernel reads the per-slice control block `Ctl` from device memory (slice index, step
// parity, beam counters) so that one captured CUDA graph replays any slice of any step.
#pragma once

#include "common.cuh"
#include "inputs.hpp"
#include "rng.hpp"

namespace hpq {

// ------------------------------------------------------------------------------------------
// Field components of the slice slab. Names follow Fields.cpp:49-148 (explicit and
// predictor-corrector layouts); "N"/"P" prefixes are the Next/Previous slices.
// ------------------------------------------------------------------------------------------
enum Comp : int {
    C_CHI = 0, C_SY, C_SX, C_EXMBY, C_EYPBX, C_EZ, C_BX, C_BY, C_BZ, C_PSI,
    C_JXB, C_JYB, C_JZB, C_JX, C_JY, C_RHOMJZ, C_RHO, C_RHOMJZB,
    C_NJXB, C_NJYB, C_PJXB, C_PJYB, C_IONS,
    C_JZ, C_NJX, C_NJY, C_PBX, C_PBY, C_PJX, C_PJY, C_PCIBX, C_PCIBY, C_PCPBX, C_PCPBY,
    C_NCOMP
};

template <class R>
struct Slab {
    R* base = nullptr;
    int nx = 0, ny = 0, pitch = 0, rows = 0;
    size_t cstride = 0;
    __host__ __device__ F2<R> c(int comp) const { return {base + (size_t)comp * cstride, pitch}; }
};

constexpr int kMaxBeams = 4;
constexpr int kMaxPlasmas = 4;

struct BeamBuf {
    double *x, *y, *z, *w, *ux, *uy, *uz;
    long long* id;
    int* nsub;
    uint8_t* valid;
};

struct BeamDev {
    BeamBuf buf[2];     // stores of the previous and the current step (by step parity)
    BeamBuf carry[2];   // slipped particles handed from one slice to the next (by slice parity)
    int* start[2];      // per-slice start/count in buf[.]
    int* count[2];
    double charge, mass;
    int n_subcycles;
    int do_z_push;
    long long cap;
    // external fields Ex Ey Ez Bx By Bz (x, y, z, t) of the beam push in device memory, or null
    // (<beam>.external_E/B(x,y,z,t), BeamParticleContainer.cpp:72-86)
    const Expr* ext;
};

template <class R>
struct PlasmaDev {
    R *x, *y, *w, *ux, *uy, *psi, *xp, *yp, *uxh, *uyh, *psih;
    // Single precision only: the particle's lattice point in cell units (exact in FP32, e.g.
    // 130.5). x, y, xp, yp then hold the displacement from that point and psi, psih hold psi - 1,
    // so the cell fraction that the shape factors use and the deviation of psi from 1 keep full
    // FP32 precision instead of the precision of |x| and of 1. Null in double precision, where
    // x, y and psi are stored as they are.
    float *ru, *rv;
    uint8_t* valid;
    long long n;
    double charge, mass, qsa_max;
    int n_subcycles;
    int neutralize;
};

// dynamic per-slice state (device memory)
struct Ctl {
    int islice;
    int step_parity;        // buf[step_parity] is read, buf[1-step_parity] is written
    int carry_n[kMaxBeams][2];
    int cursor[kMaxBeams];
    int err;
    // multigrid
    double mg_target, mg_maxnorm, mg_norm;
    int mg_iter, mg_go, mg_status, mg_pad;
    long long mg_total_iters;
    // predictor-corrector
    double pc_err, pc_err_prev, pc_sum[2], pc_w[2], pc_mix;
    int pc_iter, pc_go, pc_mixnow, pc_pad;
    unsigned int pc_cnt[2];  // arrivals of the blocks of the norm and mix kernels (last block decides)
    // persistent multigrid solve (one cooperative launch): |rhs| max, residual norms by
    // iteration parity and the grid barrier's arrival counter (mgp_bar[0]; [1] unused), cleared
    // before every solve; the barrier's timeout flag, cleared when a step begins
    double mgp_rhsnorm, mgp_norm[2];
    unsigned int mgp_bar[2];
    int mgp_bar_err, mgp_pad;
    int tc_err, tc_pad;  // error code of the tensor-core DST kernels (a timed-out wait)
    // in-situ reductions on this step (set when the step begins)
    int insitu_beam[kMaxBeams];
    int insitu_fields, insitu_pad;
    // adjoint forward: checkpoints of segment heads are written while set
    int adj_ckpt, adj_pad;
    // beam time step of this step (hipace.dt, shortened to end on hipace.max_time)
    double beam_dt;
    // physical time at the start of this step (external beam fields)
    double phys_time;
};

struct Geo {
    int nx, ny, nz;
    double plo[3], phi[3], dx[3], dxi[3];
    double xoff, yoff;          // GetPosOffset for the 2-guard slice box (Fields.H:72-76)
    double plo_p[2], phi_p[2];  // particle boundary
    int bc;                     // ParticleBC
    double c, ep0, mu0;
    int normalized;
};

// ------------------------------------------------------------------------------------------
// EnforceBC (GetAndSetPosition.H:29-99). Returns false when the particle is absorbed.
// ------------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ bool enforce_bc(const Geo& g, T& x, T& y, T& ux, T& uy) {
    const T plo0 = (T)g.plo_p[0], plo1 = (T)g.plo_p[1], phi0 = (T)g.phi_p[0], phi1 = (T)g.phi_p[1];
    if (x < plo0 || y < plo1 || x > phi0 || y > phi1) {
        const T lx = phi0 - plo0, ly = phi1 - plo1;
        if (g.bc == 0) {
            x = fmod(x - plo0, T(2) * lx); if (x < 0) x += T(2) * lx; x += plo0;
            if (x > phi0) { x = T(2) * phi0 - x; ux = -ux; }
            y = fmod(y - plo1, T(2) * ly); if (y < 0) y += T(2) * ly; y += plo1;
            if (y > phi1) { y = T(2) * phi1 - y; uy = -uy; }
            return true;
        } else if (g.bc == 1) {
            x = fmod(x - plo0, lx); if (x < 0) x += lx; x += plo0;
            y = fmod(y - plo1, ly); if (y < 0) y += ly; y += plo1;
            return true;
        }
        return false;
    }
    return true;
}

// ------------------------------------------------------------------------------------------
// Plasma initialisation (PlasmaParticleContainerInit.cpp:17-310): the particle list of one
// species is fixed on the host (lattice positions that pass the domain/radius tests); the
// kernel evaluates the density expression at c*t and resets all attributes.
// ------------------------------------------------------------------------------------------
// Thermal momenta (u_std != 0) are drawn per particle from the counter-based stream of rng.hpp
// (plasma_thermal_u), keyed by the particle's lattice index and the step. Particles are put back
// in lattice order (a reorder during the previous step permuted them), including their lattice
// points in cell units in single precision.
struct PlasmaMomenta {
    double mean[3], stdv[3];
    uint64_t seed;
    int step;
    int thermal;
};
template <class R>
__global__ void k_plasma_reset(PlasmaDev<R> P, const double* __restrict__ x0, const double* __restrict__ y0,
                               Expr density, double c_t, double scale, PlasmaMomenta m, double clight, double xoff,
                               double dxi, double yoff, double dyi) {
    HPQ_PDL_ENTRY();
    const Philox rng(m.seed);
    for (long long i = gtid(); i < P.n; i += gstride()) {
        const double x = x0[i], y = y0[i];
        double v[3] = {x, y, c_t};
        const double w = density.eval(v) * scale;
        double u[3] = {m.mean[0], m.mean[1], m.mean[2]};
        if (m.thermal) plasma_thermal_u(rng, m.step, i, m.mean, m.stdv, u);
        const double psi = sqrt(1. + u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) - u[2];
        const R xs = P.ru ? R(0) : (R)x, ys = P.ru ? R(0) : (R)y;
        P.x[i] = xs; P.y[i] = ys; P.xp[i] = xs; P.yp[i] = ys;
        if (P.ru) {
            P.ru[i] = (float)((x - xoff) * dxi);
            P.rv[i] = (float)((y - yoff) * dyi);
        }
        P.w[i] = (R)w;
        P.ux[i] = (R)(u[0] * clight); P.uy[i] = (R)(u[1] * clight);
        P.uxh[i] = (R)(u[0] * clight); P.uyh[i] = (R)(u[1] * clight);
        const R psis = P.ru ? (R)(psi - 1.0) : (R)psi;
        P.psi[i] = psis; P.psih[i] = psis;
        P.valid[i] = 1;
    }
}

// ------------------------------------------------------------------------------------------
// Plasma reorder (PlasmaParticleContainer::ReorderParticles, PlasmaParticleContainer.cpp:197-208):
// every reorder_period slices the particles are sorted by the cell (or node) they sit in, which
// gives the deposit's atomics cell locality once the plasma response has scattered them. The
// sort is a stable counting sort, so that runs are reproducible: keys and per-bin counts, an
// exclusive scan over the bins, a scatter into the bins, each bin's indices put back in
// ascending order (bins hold a few particles), then a gather of every attribute into scratch
// arrays and a copy back (the slice graph keeps the attribute pointers).
// Bin of a particle: cell centres sit at integer t = (x - xoff) / dx, so the cell is
// floor(t + 1/2) in [0, n-1] and the nearest node floor(t + 1) in [0, n]; key = j (nx + 1) + i.
// ------------------------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ int reorder_bin(bool has_ref, float r0, R x, double off, double dxi, int n, int node) {
    const double t = has_ref ? (double)r0 + (double)x * dxi : ((double)x - off) * dxi;
    const double f = floor(t + (node ? 1.0 : 0.5));
    const int hi = node ? n : n - 1;
    return f < 0 ? 0 : (f > hi ? hi : (int)f);
}

template <class R>
__global__ void k_reorder_keys(PlasmaDev<R> P, Geo g, int node_x, int node_y, int* __restrict__ key,
                               int* __restrict__ cnt) {
    HPQ_PDL_ENTRY();
    for (long long i = gtid(); i < P.n; i += gstride()) {
        const int bi = reorder_bin<R>(P.ru != nullptr, P.ru ? P.ru[i] : 0.f, P.x[i], g.xoff, g.dxi[0], g.nx, node_x);
        const int bj = reorder_bin<R>(P.rv != nullptr, P.rv ? P.rv[i] : 0.f, P.y[i], g.yoff, g.dxi[1], g.ny, node_y);
        const int k = bj * (g.nx + 1) + bi;
        key[i] = k;
        atomicAdd(&cnt[k], 1);
    }
}

// exclusive scan of n ints in three launches: per-block scans (1024 per block) with block
// totals, the scan of the block totals (one block), and the block offsets added (also written to
// `fill`, the scatter cursors)
__device__ __forceinline__ int block_exclusive_scan_1024(int v, int& total) {
    __shared__ int ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    __syncthreads();
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    int before = 0;
    total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        if (w < warp) before += ws[w];
        total += ws[w];
    }
    return before + x - v;
}
__global__ void __launch_bounds__(1024) k_scan_blocks(const int* __restrict__ in, int* __restrict__ out,
                                                      int* __restrict__ bsum, long long n) {
    HPQ_PDL_ENTRY();
    const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
    int total;
    const int e = block_exclusive_scan_1024(i < n ? in[i] : 0, total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) k_scan_totals(int* __restrict__ bsum, int nb) {
    HPQ_PDL_ENTRY();
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        const int v = b < nb ? bsum[b] : 0;
        int total;
        const int e = block_exclusive_scan_1024(v, total);
        const int base = carry;
        if (b < nb) bsum[b] = base + e;
        __syncthreads();
        if (threadIdx.x == 0) carry = base + total;
        __syncthreads();
    }
}
__global__ void k_scan_add(int* __restrict__ out, const int* __restrict__ bsum, int* __restrict__ fill, long long n) {
    HPQ_PDL_ENTRY();
    for (long long i = gtid(); i < n; i += gstride()) {
        const int v = out[i] + bsum[i / 1024];
        out[i] = v;
        fill[i] = v;
    }
}

__global__ void k_reorder_scatter(const int* __restrict__ key, long long n, int* __restrict__ fill, int* __restrict__ perm) {
    HPQ_PDL_ENTRY();
    for (long long i = gtid(); i < n; i += gstride()) perm[atomicAdd(&fill[key[i]], 1)] = (int)i;
}

// one thread per bin: insertion sort of the bin's particle indices (ascending = stable)
__global__ void k_reorder_bins(const int* __restrict__ start, const int* __restrict__ cnt, long long nbins,
                               int* __restrict__ perm) {
    HPQ_PDL_ENTRY();
    for (long long b = gtid(); b < nbins; b += gstride()) {
        const int s0 = start[b], m = cnt[b];
        for (int a = 1; a < m; ++a) {
            const int v = perm[s0 + a];
            int c = a - 1;
            while (c >= 0 && perm[s0 + c] > v) {
                perm[s0 + c + 1] = perm[s0 + c];
                --c;
            }
            perm[s0 + c + 1] = v;
        }
    }
}

// dst[k] = src[perm[k]] for every attribute (to = 1), or the copy back src[k] = dst[k] (to = 0)
template <class R>
__global__ void k_reorder_move(PlasmaDev<R> P, PlasmaDev<R> T, const int* __restrict__ perm, int to) {
    HPQ_PDL_ENTRY();
    for (long long k = gtid(); k < P.n; k += gstride()) {
        if (to) {
            const int i = perm[k];
            T.x[k] = P.x[i]; T.y[k] = P.y[i]; T.w[k] = P.w[i]; T.ux[k] = P.ux[i]; T.uy[k] = P.uy[i];
            T.psi[k] = P.psi[i]; T.xp[k] = P.xp[i]; T.yp[k] = P.yp[i]; T.uxh[k] = P.uxh[i]; T.uyh[k] = P.uyh[i];
            T.psih[k] = P.psih[i]; T.valid[k] = P.valid[i];
            if (P.ru) { T.ru[k] = P.ru[i]; T.rv[k] = P.rv[i]; }
        } else {
            P.x[k] = T.x[k]; P.y[k] = T.y[k]; P.w[k] = T.w[k]; P.ux[k] = T.ux[k]; P.uy[k] = T.uy[k];
            P.psi[k] = T.psi[k]; P.xp[k] = T.xp[k]; P.yp[k] = T.yp[k]; P.uxh[k] = T.uxh[k]; P.uyh[k] = T.uyh[k];
            P.psih[k] = T.psih[k]; P.valid[k] = T.valid[k];
            if (P.ru) { P.ru[k] = T.ru[k]; P.rv[k] = T.rv[k]; }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Plasma current deposition, order 2 (PlasmaDepositCurrent.cpp:22-259). Null outputs are
// skipped. QSA-violating particles (gamma/psi outside (0, max]) are invalidated (:199-206).
// ------------------------------------------------------------------------------------------
template <class R>
struct DepOut {
    R *jx, *jy, *jz, *rho, *chi, *rhomjz;
    int pitch;
    int merge;  // order 2, floating-point atomics: warp-merged stencils (plasma_deposit_merged)
};

// Deterministic deposition (hpq_set_deterministic). Floating-point atomics give sums whose last
// bits depend on the order in which threads arrive. In deterministic mode every deposited value v
// is split into three 64-bit fixed-point words,
//   a = rint(v 2^10),  b = rint((v - a 2^-10) 2^50),  c = rint((v - a 2^-10 - b 2^-50) 2^90),
// added with integer atomics into slab-shaped shadow arrays. Integer addition is associative, so
// the totals do not depend on the arrival order, and k_det_flush turns them back into one
// floating-point value per cell, the same on every run. Range: |sum| < 2^53; resolution 2^-91
// per deposited value (below the FP64 rounding of any value above 1e-12).
struct DetAcc {
    long long* w[3];   // shadow words (null: plain floating-point atomics)
    const void* base;  // slab base the deposited planes belong to
};

template <class R>
__device__ __forceinline__ void addc(const DetAcc& d, R* base, int pitch, int i, int j, R v) {
    const ptrdiff_t off = (ptrdiff_t)(j + kGuardAlloc) * pitch + (i + kGuardAlloc);
    double r = (double)v;
    if (d.w[0] == nullptr || !isfinite(r)) {
        atomicAdd(base + off, v);
        return;
    }
    const ptrdiff_t e = (base - static_cast<const R*>(d.base)) + off;
    const double a = rint(r * 0x1p10);
    r -= a * 0x1p-10;
    const double b = rint(r * 0x1p50);
    r -= b * 0x1p-50;
    const double c = rint(r * 0x1p90);
    atomicAdd(reinterpret_cast<unsigned long long*>(d.w[0] + e), (unsigned long long)(long long)a);
    atomicAdd(reinterpret_cast<unsigned long long*>(d.w[1] + e), (unsigned long long)(long long)b);
    atomicAdd(reinterpret_cast<unsigned long long*>(d.w[2] + e), (unsigned long long)(long long)c);
}

// addc with the mode fixed at compile time: plain floating-point atomics without deterministic
// accumulation (no per-deposit branch)
template <bool DET, class R>
__device__ __forceinline__ void addd(const DetAcc& d, R* base, int pitch, int i, int j, R v) {
    if constexpr (DET) addc(d, base, pitch, i, j, v);
    else atomicAdd(base + (ptrdiff_t)(j + kGuardAlloc) * pitch + (i + kGuardAlloc), v);
}

// Cell-unit coordinate of a plasma position along one axis as base + t: with a reference lattice
// coordinate (single precision) t = frac(u0) + x * dxi is a small number and the integer part
// goes to `base`; without one, base = 0 and t = (x - off) * dxi. Clamped to [-1, n - 1/2] like
// clamp_mid.
template <class R>
__device__ __forceinline__ R plasma_mid_v(bool has_ref, float u0, R x, R off, R dxi, int n, int& base) {
    if (!has_ref) {
        base = 0;
        return clamp_mid<R>((x - off) * dxi, n);
    }
    const float fb = floorf(u0);
    const R t = (R)(u0 - fb) + x * dxi;
    const R tot = (R)fb + t;
    if (!(tot >= R(-1) && tot <= R(n) - R(0.5))) {
        base = 0;
        return clamp_mid<R>(tot, n);
    }
    base = (int)fb;
    return t;
}
template <class R>
__device__ __forceinline__ R plasma_mid(const float* ref, long long ip, R x, R off, R dxi, int n, int& base) {
    return plasma_mid_v<R>(ref != nullptr, ref ? ref[ip] : 0.f, x, off, dxi, n, base);
}

// Warp-merged order-2 plasma deposition. The lanes of a warp hold consecutive particles; in a
// plasma still in lattice (or reorder) order, lane l + 1 sits one cell to the right of lane l in
// the same row, and their 3 x 3 stencils share two columns. Each lane then deposits its centre
// column with the right column of lane l - 1 and the left column of lane l + 1 added in (their
// shapes and weights come by shuffle); a lane deposits its own left/right column only where it has
// no such neighbour. Lattice-ordered rows need a third of the atomics of the plain deposit; the
// sums per cell are the same terms in another order.
template <class R>
__device__ __forceinline__ void plasma_deposit_merged(const PlasmaDev<R>& P, const DepOut<R>& o, const Geo& g,
                                                      R charge_invvol, R q_mu0_mass_ratio) {
    const R clight = (R)g.c, clightinv = (R)(1.0 / g.c);
    const R xoff = (R)g.xoff, yoff = (R)g.yoff, dxi = (R)g.dxi[0], dyi = (R)g.dxi[1];
    const R qsa = (R)P.qsa_max;
    const int lane = threadIdx.x & 31;
    const long long stride = gstride();
    const DetAcc nodet{};
    for (long long base = gtid() - lane; base < P.n; base += stride) {
        const long long ip = base + lane;
        bool act = ip < P.n && P.valid[ip];
        R qv = 0, f[5] = {0, 0, 0, 0, 0}, sxs[3] = {0, 0, 0}, sys[3] = {0, 0, 0};
        int cx = 0, cy = 0;
        if (act) {
            const R psis = P.psi[ip];
            const R psi_inv = P.ru ? R(1) / (R(1) + psis) : R(1) / psis;
            const R vx_c = P.ux[ip] * psi_inv, vy_c = P.uy[ip] * psi_inv;
            int bx, by;
            const R xmid = plasma_mid<R>(P.ru, ip, P.x[ip], xoff, dxi, g.nx, bx);
            const R ymid = plasma_mid<R>(P.rv, ip, P.y[ip], yoff, dyi, g.ny, by);
            const R gamma_psi = R(0.5) * (psi_inv * psi_inv + vx_c * vx_c * clightinv * clightinv +
                                          vy_c * vy_c * clightinv * clightinv + R(1));
            const R gpm1 = P.ru ? R(0.5) * (-psis * (R(2) + psis) * psi_inv * psi_inv + vx_c * vx_c * clightinv * clightinv +
                                            vy_c * vy_c * clightinv * clightinv)
                                : gamma_psi - R(1);
            if (gamma_psi < R(0) || gamma_psi > qsa || psi_inv < R(0)) {
                P.w[ip] = R(0);
                P.valid[ip] = 0;
                act = false;
            } else {
                qv = charge_invvol * P.w[ip];
                f[0] = vx_c; f[1] = vy_c; f[2] = gpm1 * clight; f[3] = gamma_psi; f[4] = q_mu0_mass_ratio * psi_inv;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const Sh<R> a = shape2<R>(xmid, k), b = shape2<R>(ymid, k);
                    sxs[k] = a.s; sys[k] = b.s;
                    if (k == 1) { cx = a.cell + bx; cy = b.cell + by; }
                }
            }
        }
        // links to the right neighbour, and from the left one
        const int cxn = __shfl_down_sync(0xffffffffu, cx, 1), cyn = __shfl_down_sync(0xffffffffu, cy, 1);
        const bool actn = __shfl_down_sync(0xffffffffu, act, 1);
        const bool right = act && lane < 31 && actn && cyn == cy && cxn == cx + 1;
        const bool left = __shfl_up_sync(0xffffffffu, right, 1) && lane > 0;
        // the neighbours' weights: right lane's left column, left lane's right column
        const R qn = __shfl_down_sync(0xffffffffu, qv * sxs[0], 1), qp = __shfl_up_sync(0xffffffffu, qv * sxs[2], 1);
        R syn[3], syp[3], fn[5], fp[5];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            syn[k] = __shfl_down_sync(0xffffffffu, sys[k], 1);
            syp[k] = __shfl_up_sync(0xffffffffu, sys[k], 1);
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            fn[k] = __shfl_down_sync(0xffffffffu, f[k], 1);
            fp[k] = __shfl_up_sync(0xffffffffu, f[k], 1);
        }
        if (!act) continue;
        R* planes[5] = {o.jx, o.jy, o.jz, o.rho, o.chi};
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const int j = cy - 1 + iy;
            const R wc = qv * sxs[1] * sys[iy];
            const R wr = right ? qn * syn[iy] : R(0);
            const R wl = left ? qp * syp[iy] : R(0);
            const R w0 = qv * sxs[0] * sys[iy], w2 = qv * sxs[2] * sys[iy];
#pragma unroll
            for (int p = 0; p < 5; ++p) {
                if (!planes[p]) continue;
                addd<false>(nodet, planes[p], o.pitch, cx, j, wc * f[p] + wr * fn[p] + wl * fp[p]);
                if (!left) addd<false>(nodet, planes[p], o.pitch, cx - 1, j, w0 * f[p]);
                if (!right) addd<false>(nodet, planes[p], o.pitch, cx + 1, j, w2 * f[p]);
            }
            if (o.rhomjz) {
                addd<false>(nodet, o.rhomjz, o.pitch, cx, j, wc + wr + wl);
                if (!left) addd<false>(nodet, o.rhomjz, o.pitch, cx - 1, j, w0);
                if (!right) addd<false>(nodet, o.rhomjz, o.pitch, cx + 1, j, w2);
            }
        }
    }
}

template <class R, bool DET, int ORD = 2>
__global__ void __launch_bounds__(256) k_plasma_deposit(PlasmaDev<R> P, DepOut<R> o, Geo g, double charge,
                                                        const int* gate, DetAcc det) {
    HPQ_PDL_ENTRY();
    if (gate && !*gate) return;
    const R invvol = g.normalized ? (R)(g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1]) : (R)(g.dxi[0] * g.dxi[1] * g.dxi[2]);
    const R clight = (R)g.c, clightinv = (R)(1.0 / g.c);
    const R charge_invvol = (R)charge * invvol;
    const R q_mu0_mass_ratio = (R)(charge * g.mu0 / P.mass);
    const R xoff = (R)g.xoff, yoff = (R)g.yoff, dxi = (R)g.dxi[0], dyi = (R)g.dxi[1];
    const R qsa = (R)P.qsa_max;
    if constexpr (!DET && ORD == 2) {
        if (o.merge) {
            plasma_deposit_merged<R>(P, o, g, charge_invvol, q_mu0_mass_ratio);
            return;
        }
    }
    // the attributes of the thread's next particle are loaded before the atomics of the current
    // one, so that two particles' loads are in flight per thread
    struct Pt {
        R x, y, w, ux, uy, psi;
        float ru, rv;
        uint8_t v;
    };
    auto load = [&](long long ip) {
        Pt q;
        q.v = P.valid[ip];
        q.x = P.x[ip]; q.y = P.y[ip]; q.w = P.w[ip];
        q.ux = P.ux[ip]; q.uy = P.uy[ip]; q.psi = P.psi[ip];
        q.ru = P.ru ? P.ru[ip] : 0.f;
        q.rv = P.rv ? P.rv[ip] : 0.f;
        return q;
    };
    const long long stride = gstride();
    long long ip = gtid();
    Pt cur{};
    if (ip < P.n) cur = load(ip);
    for (; ip < P.n; ip += stride) {
        Pt nxt{};
        if (ip + stride < P.n) nxt = load(ip + stride);
        if (cur.v) {
            const R psis = cur.psi;
            const R psi_inv = P.ru ? R(1) / (R(1) + psis) : R(1) / psis;
            const R vx_c = cur.ux * psi_inv;
            const R vy_c = cur.uy * psi_inv;
            const R q_invvol = charge_invvol * cur.w;
            int bx, by;
            const R xmid = plasma_mid_v<R>(P.ru != nullptr, cur.ru, cur.x, xoff, dxi, g.nx, bx);
            const R ymid = plasma_mid_v<R>(P.rv != nullptr, cur.rv, cur.y, yoff, dyi, g.ny, by);
            const R gamma_psi = R(0.5) * (psi_inv * psi_inv + vx_c * vx_c * clightinv * clightinv +
                                          vy_c * vy_c * clightinv * clightinv + R(1));
            // gamma/psi - 1; with psi - 1 stored, (1/psi)^2 - 1 = -(psi - 1)(psi + 1)/psi^2 avoids
            // the cancellation of two numbers close to 1
            const R gpm1 = P.ru ? R(0.5) * (-psis * (R(2) + psis) * psi_inv * psi_inv + vx_c * vx_c * clightinv * clightinv +
                                            vy_c * vy_c * clightinv * clightinv)
                                : gamma_psi - R(1);
            if (gamma_psi < R(0) || gamma_psi > qsa || psi_inv < R(0)) {
                P.w[ip] = R(0);
                P.valid[ip] = 0;
            } else {
                constexpr int NP = ORD + 1;
                Sh<R> sx[NP], sy[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    sx[k] = shapeN<R, ORD>(xmid, k); sy[k] = shapeN<R, ORD>(ymid, k);
                    sx[k].cell += bx; sy[k].cell += by;
                }
#pragma unroll
                for (int iy = 0; iy < NP; ++iy)
#pragma unroll
                    for (int ix = 0; ix < NP; ++ix) {
                        const int i = sx[ix].cell, j = sy[iy].cell;
                        const R cd = q_invvol * sx[ix].s * sy[iy].s;
                        if (o.jx) { addd<DET>(det, o.jx, o.pitch, i, j, cd * vx_c); addd<DET>(det, o.jy, o.pitch, i, j, cd * vy_c); }
                        if (o.jz) addd<DET>(det, o.jz, o.pitch, i, j, cd * gpm1 * clight);
                        if (o.rho) addd<DET>(det, o.rho, o.pitch, i, j, cd * gamma_psi);
                        if (o.chi) addd<DET>(det, o.chi, o.pitch, i, j, cd * q_mu0_mass_ratio * psi_inv);
                        if (o.rhomjz) addd<DET>(det, o.rhomjz, o.pitch, i, j, cd);
                    }
            }
        }
        cur = nxt;
    }
}

// ------------------------------------------------------------------------------------------
// Explicit Sx/Sy deposition (ExplicitDeposition.cpp:20-265, no laser)
// ------------------------------------------------------------------------------------------
// Bz, Ez, ExmBy, EypBx of one cell side by side, so that the explicit deposition reads a cell's
// four fields with one vector load instead of four scalar loads
template <class R>
struct alignas(4 * sizeof(R)) Quad {
    R bz, ez, ex, ey;
};
template <class R>
__global__ void k_pack_explicit(Slab<R> S, Quad<R>* __restrict__ q) {
    HPQ_PDL_ENTRY();
    const R* bz = S.c(C_BZ).p;
    const R* ez = S.c(C_EZ).p;
    const R* ex = S.c(C_EXMBY).p;
    const R* ey = S.c(C_EYPBX).p;
    for (long long k = gtid(); k < (long long)S.cstride; k += gstride()) q[k] = Quad<R>{bz[k], ez[k], ex[k], ey[k]};
}

template <class R, int DT, bool DET, int ORD = 2>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 2 : 3) k_explicit_deposit(PlasmaDev<R> P, Slab<R> S, Geo g,
                                                                                    const Quad<R>* __restrict__ quad,
                                                                                    DetAcc det) {
    HPQ_PDL_ENTRY();
    const R invvol = g.normalized ? (R)(g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1]) : (R)(g.dxi[0] * g.dxi[1] * g.dxi[2]);
    const R a_clight = (R)g.c, clight_inv = (R)(1.0 / g.c);
    const R charge_invvol_mu0 = (R)(P.charge * (double)invvol * g.mu0);
    const R q_mass_ratio = (R)(P.charge / P.mass);
    const R xoff = (R)g.xoff, yoff = (R)g.yoff, dxi = (R)g.dxi[0], dyi = (R)g.dxi[1];
    R* Sx = S.c(C_SX).p;
    R* Sy = S.c(C_SY).p;
    constexpr int NS = dshape_points<DT, ORD>();
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        const R psis = P.psi[ip];
        const R psi_inv = P.ru ? R(1) / (R(1) + psis) : R(1) / psis;
        const R vx = P.ux[ip] * psi_inv * clight_inv;
        const R vy = P.uy[ip] * psi_inv * clight_inv;
        const R cdm = charge_invvol_mu0 * P.w[ip];
        int bx, by;
        const R xmid = plasma_mid<R>(P.ru, ip, P.x[ip], xoff, dxi, g.nx, bx);
        const R ymid = plasma_mid<R>(P.rv, ip, P.y[ip], yoff, dyi, g.ny, by);
        const R gamma_psi = R(0.5) * (psi_inv * psi_inv + vx * vx + vy * vy + R(1));
        // gamma/psi - 1 - v_y^2 and gamma/psi - 1 - v_x^2 (see k_plasma_deposit for psi - 1)
        const R gpm1 = P.ru ? R(0.5) * (-psis * (R(2) + psis) * psi_inv * psi_inv + vx * vx + vy * vy) : R(0);
        const R gmy = P.ru ? gpm1 - vy * vy : gamma_psi - vy * vy - R(1);
        const R gmx = P.ru ? gpm1 - vx * vx : gamma_psi - vx * vx - R(1);
        DSh<R> sx[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            sx[k] = dshapeN<R, DT, ORD>(xmid, k);
            sx[k].cell += bx;
        }
        // one row of the stencil at a time (the y shape of the row is formed in the loop, which
        // keeps the register count low enough for two blocks per SM)
#pragma unroll 1
        for (int iy = 0; iy < NS; ++iy) {
            DSh<R> syr = dshapeN<R, DT, ORD>(ymid, iy);
            syr.cell += by;
#pragma unroll
            for (int ix = 0; ix < NS; ++ix) {
                if (DT == 2 && (ix == 0 || ix == NS - 1) && (iy == 0 || iy == NS - 1)) continue;
                const int i = sx[ix].cell, j = syr.cell;
                const Quad<R> fq = quad[(ptrdiff_t)(j + kGuardAlloc) * S.pitch + (i + kGuardAlloc)];
                const R Bz_v = fq.bz, Ez_v = fq.ez, ExmBy_v = fq.ex, EypBx_v = fq.ey;
                const R sxs = sx[ix].s, sys = syr.s, sxd = sx[ix].ds, syd = syr.ds;
                const R vsy = cdm * (-sxs * sys * (-Bz_v * vx + (Ez_v * vy + ExmBy_v * (-vx * vy) + EypBx_v * (gamma_psi - vy * vy)) * clight_inv) * q_mass_ratio * psi_inv +
                                     (-sxd * sys * dxi * (-vx * vy) - sxs * syd * dyi * gmy) * a_clight);
                const R vsx = cdm * (+sxs * sys * (+Bz_v * vy + (Ez_v * vx + ExmBy_v * (gamma_psi - vx * vx) + EypBx_v * (-vx * vy)) * clight_inv) * q_mass_ratio * psi_inv +
                                     (+sxd * sys * dxi * gmx + sxs * syd * dyi * (-vx * vy)) * a_clight);
                addd<DET>(det, Sy, S.pitch, i, j, vsy);
                addd<DET>(det, Sx, S.pitch, i, j, vsx);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Field gather (FieldGather.H:45-96, derivative type 1: (ORD + 2)^2 stencil, 4x4 at order 2)
// ------------------------------------------------------------------------------------------
// x, y in cell units, as base + fraction (bx, by integer)
template <class R, class T, int ORD = 2>
__device__ __forceinline__ void gather_mid(const Slab<R>& S, const Geo& g, T x, T y, int bx, int by, T& ExmBy,
                                           T& EypBx, T& Ez, T& Bx, T& By, T& Bz) {
    const T dxi = (T)g.dxi[0], dyi = (T)g.dxi[1];
    const F2<R> Psi = S.c(C_PSI), FEz = S.c(C_EZ), FBx = S.c(C_BX), FBy = S.c(C_BY), FBz = S.c(C_BZ);
    constexpr int NG = ORD + 2;
    DSh<T> sx[NG], sy[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) {
        sx[k] = dshapeN<T, 1, ORD>(x, k); sy[k] = dshapeN<T, 1, ORD>(y, k);
        sx[k].cell += bx; sy[k].cell += by;
    }
#pragma unroll
    for (int iy = 0; iy < NG; iy++)
#pragma unroll
        for (int ix = 0; ix < NG; ix++) {
            const int i = sx[ix].cell, j = sy[iy].cell;
            const T psi = (T)Psi(i, j);
            ExmBy += (sx[ix].ds * sy[iy].s) * psi * dxi;
            EypBx += (sx[ix].s * sy[iy].ds) * psi * dyi;
            const T s = sx[ix].s * sy[iy].s;
            Ez += s * (T)FEz(i, j);
            Bx += s * (T)FBx(i, j);
            By += s * (T)FBy(i, j);
            Bz += s * (T)FBz(i, j);
        }
}

template <class R, class T, int ORD = 2>
__device__ __forceinline__ void gather(const Slab<R>& S, const Geo& g, T xp, T yp, T& ExmBy, T& EypBx, T& Ez,
                                       T& Bx, T& By, T& Bz) {
    const T x = clamp_mid<T>((xp - (T)g.xoff) * (T)g.dxi[0], g.nx), y = clamp_mid<T>((yp - (T)g.yoff) * (T)g.dxi[1], g.ny);
    gather_mid<R, T, ORD>(S, g, x, y, 0, 0, ExmBy, EypBx, Ez, Bx, By, Bz);
}

// ------------------------------------------------------------------------------------------
// Plasma push (PlasmaParticleAdvance.cpp:29-217; PlasmaMomentumPush PushPlasmaParticles.H:39-75)
// Leapfrog in zeta: 4 Taylor sub-steps (second order through the derivative of the right-hand
// side along the trajectory) for u and psi from -1/2 to +1/2, full position step, 2 more
// sub-steps to the slice.
// ------------------------------------------------------------------------------------------
template <class R, int ORD = 2>
__global__ void __launch_bounds__(256) k_plasma_push(PlasmaDev<R> P, Slab<R> S, Geo g, int temp,
                                                     const int* gate) {
    HPQ_PDL_ENTRY();
    if (gate && !*gate) return;
    const R clight = (R)g.c, ci = (R)(1. / g.c);
    const R qmc = (R)(P.charge / (P.mass * g.c));
    const int nsubc = P.n_subcycles;
    const R dzs = (R)(g.dx[2] / nsubc);
    const R sdz = dzs / R(4);
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        for (int isc = 0; isc < nsubc; ++isc) {
            R xp = P.xp[ip], yp = P.yp[ip];
            R Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
            {
                int bx, by;
                const R xm = plasma_mid<R>(P.ru, ip, xp, (R)g.xoff, (R)g.dxi[0], g.nx, bx);
                const R ym = plasma_mid<R>(P.rv, ip, yp, (R)g.yoff, (R)g.dxi[1], g.ny, by);
                gather_mid<R, R, ORD>(S, g, xm, ym, bx, by, Ex, Ey, Ez, Bx, By, Bz);
            }
            Bx *= clight; By *= clight;
            R ux = P.uxh[ip], uy = P.uyh[ip], psi = P.psih[ip];
            const R pb = P.ru ? R(1) : R(0);  // psi = pb + stored value
            // u += h f(u) + h^2/2 Df(u) f(u): the second-order term is the derivative of the
            // right-hand side along the trajectory (the reference evaluates it with dual numbers,
            // PushPlasmaParticles.H:39-75; the fields are constant along it, so it is written out)
            const R c2 = ci * ci, hh = R(0.5) * sdz * sdz;
            auto substep = [&]() {
                const R pi = R(1) / (pb + psi);
                const R a2 = R(1) + (ux * ux + uy * uy) * c2;
                const R gp = R(0.5) * pi * pi * a2 + R(0.5);
                const R ue = ux * Ex + uy * Ey;
                const R d0 = qmc * (gp * Ex + By + (uy * Bz) * pi);
                const R d1 = qmc * (gp * Ey - Bx - (ux * Bz) * pi);
                const R d2 = qmc * ci * (ue * ci * pi - Ez);
                const R dpi = -(pi * pi) * d2;
                const R dgp = pi * dpi * a2 + pi * pi * c2 * (ux * d0 + uy * d1);
                const R e0 = qmc * (dgp * Ex + Bz * (d1 * pi + uy * dpi));
                const R e1 = qmc * (dgp * Ey - Bz * (d0 * pi + ux * dpi));
                const R e2 = qmc * c2 * ((d0 * Ex + d1 * Ey) * pi + ue * dpi);
                ux += sdz * d0 + hh * e0;
                uy += sdz * d1 + hh * e1;
                psi += sdz * d2 + hh * e2;
            };
#pragma unroll
            for (int k = 0; k < 4; ++k) substep();
            xp += dzs * ci * (ux * (R(1) / (pb + psi)));
            yp += dzs * ci * (uy * (R(1) / (pb + psi)));
            if (P.ru) {
                // displacements: the boundary test needs the absolute position
                const R x0 = (R)(g.xoff + (double)P.ru[ip] * g.dx[0]), y0 = (R)(g.yoff + (double)P.rv[ip] * g.dx[1]);
                R xa = x0 + xp, ya = y0 + yp;
                const R xa0 = xa, ya0 = ya;
                if (!enforce_bc<R>(g, xa, ya, ux, uy)) { P.w[ip] = R(0); P.valid[ip] = 0; break; }
                if (xa != xa0) xp = xa - x0;
                if (ya != ya0) yp = ya - y0;
            } else if (!enforce_bc<R>(g, xp, yp, ux, uy)) { P.w[ip] = R(0); P.valid[ip] = 0; break; }
            P.x[ip] = xp; P.y[ip] = yp;
            if (!temp) {
                P.uxh[ip] = ux; P.uyh[ip] = uy; P.psih[ip] = psi;
                P.xp[ip] = xp; P.yp[ip] = yp;
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) substep();
            P.ux[ip] = ux; P.uy[ip] = uy; P.psi[ip] = psi;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Beam deposition (BeamDepositCurrent.cpp:21-196): the non-slipped particles of slice
// `ctl->islice - which` of the current store.
// ------------------------------------------------------------------------------------------
template <class R, int ORD = 2>
__global__ void __launch_bounds__(256) k_beam_deposit(BeamDev B, const Ctl* __restrict__ ctl, int which, R* jx, R* jy,
                                                      R* jz, R* rmj, int pitch, Geo g, int gated, DetAcc det) {
    HPQ_PDL_ENTRY();
    if (gated && !ctl->pc_go) return;
    const int s = ctl->islice - which;
    if (s < 0) return;
    const int par = ctl->step_parity;
    const int start = B.start[par][s], n = B.count[par][s];
    const BeamBuf b = B.buf[par];
    const double invvol = g.normalized ? 1.0 : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double clightinv = 1.0 / g.c, clightsq = 1.0 / (g.c * g.c);
    for (long long k = gtid(); k < n; k += gstride()) {
        const long long ip = start + k;
        if (!b.valid[ip]) continue;
        const double ux = b.ux[ip], uy = b.uy[ip], uz = b.uz[ip];
        const double gaminv = 1.0 / sqrt(1.0 + ux * ux * clightsq + uy * uy * clightsq + uz * uz * clightsq);
        const double wq = B.charge * b.w[ip] * invvol;
        const double vx = ux * gaminv, vy = uy * gaminv, vz = uz * gaminv;
        const double wqx = wq * vx, wqy = wq * vy, wqz = wq * vz, wqr = wq * (1. - vz * clightinv);
        const double xmid = clamp_mid<double>((b.x[ip] - g.xoff) * g.dxi[0], g.nx);
        const double ymid = clamp_mid<double>((b.y[ip] - g.yoff) * g.dxi[1], g.ny);
        constexpr int NP = ORD + 1;
        Sh<double> sx[NP], sy[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) { sx[q] = shapeN<double, ORD>(xmid, q); sy[q] = shapeN<double, ORD>(ymid, q); }
#pragma unroll
        for (int iy = 0; iy < NP; ++iy)
#pragma unroll
            for (int ix = 0; ix < NP; ++ix) {
                const double S = sx[ix].s * sy[iy].s;
                const int i = sx[ix].cell, j = sy[iy].cell;
                if (jx) { addc<R>(det, jx, pitch, i, j, (R)(S * wqx)); addc<R>(det, jy, pitch, i, j, (R)(S * wqy)); }
                if (jz) addc<R>(det, jz, pitch, i, j, (R)(S * wqz));
                if (rmj) addc<R>(det, rmj, pitch, i, j, (R)(S * wqr));
            }
    }
}

// Both beam depositions of the explicit solver in one launch: jz_beam (and rhomjz_beam) from the
// non-slipped particles of this slice, jx_beam/jy_beam of the next slice from its particles.
template <class R, int ORD = 2>
__global__ void __launch_bounds__(256) k_beam_deposit_this_next(BeamDev B, const Ctl* __restrict__ ctl, R* jz, R* rmj,
                                                                R* njx, R* njy, int pitch, Geo g, DetAcc det) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice;
    const int par = ctl->step_parity;
    const int st0 = B.start[par][s], n0 = B.count[par][s];
    const int st1 = s > 0 ? B.start[par][s - 1] : 0, n1 = (s > 0 && njx) ? B.count[par][s - 1] : 0;
    const BeamBuf b = B.buf[par];
    const double invvol = g.normalized ? 1.0 : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double clightinv = 1.0 / g.c, clightsq = 1.0 / (g.c * g.c);
    for (long long k = gtid(); k < n0 + n1; k += gstride()) {
        const bool nxt = k >= n0;
        const long long ip = nxt ? st1 + (k - n0) : st0 + k;
        if (!b.valid[ip]) continue;
        const double ux = b.ux[ip], uy = b.uy[ip], uz = b.uz[ip];
        const double gaminv = 1.0 / sqrt(1.0 + ux * ux * clightsq + uy * uy * clightsq + uz * uz * clightsq);
        const double wq = B.charge * b.w[ip] * invvol;
        const double vx = ux * gaminv, vy = uy * gaminv, vz = uz * gaminv;
        const double wqx = wq * vx, wqy = wq * vy, wqz = wq * vz, wqr = wq * (1. - vz * clightinv);
        const double xmid = clamp_mid<double>((b.x[ip] - g.xoff) * g.dxi[0], g.nx);
        const double ymid = clamp_mid<double>((b.y[ip] - g.yoff) * g.dxi[1], g.ny);
        constexpr int NP = ORD + 1;
        Sh<double> sx[NP], sy[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) { sx[q] = shapeN<double, ORD>(xmid, q); sy[q] = shapeN<double, ORD>(ymid, q); }
#pragma unroll
        for (int iy = 0; iy < NP; ++iy)
#pragma unroll
            for (int ix = 0; ix < NP; ++ix) {
                const double S = sx[ix].s * sy[iy].s;
                const int i = sx[ix].cell, j = sy[iy].cell;
                if (nxt) {
                    addc<R>(det, njx, pitch, i, j, (R)(S * wqx));
                    addc<R>(det, njy, pitch, i, j, (R)(S * wqy));
                } else {
                    addc<R>(det, jz, pitch, i, j, (R)(S * wqz));
                    if (rmj) addc<R>(det, rmj, pitch, i, j, (R)(S * wqr));
                }
            }
    }
}

// ------------------------------------------------------------------------------------------
// Beam push (BeamParticleAdvance.cpp:19-336; FP64 throughout). Pushes the non-slipped
// particles of slice ctl->islice + lag and the particles that slipped in from the slice before
// it, resuming at their sub-cycle count; a particle stops when it leaves the slice (z < slice
// lower edge). S holds that slice's fields (the slice driver runs the push of a slice beside the
// next slice's solve, on a saved copy of the fields); lag 1 beyond the box head does nothing.
// ------------------------------------------------------------------------------------------
template <class R, int ORD = 2>
__global__ void __launch_bounds__(256) k_beam_push(BeamDev B, const Ctl* __restrict__ ctl, int bi, Slab<R> S, Geo g,
                                                   int lag) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice + lag;
    if (s < 0 || s >= g.nz) return;
    const int par = ctl->step_parity;
    const int start = B.start[par][s], na = B.count[par][s];
    const int cin = (s + 1) & 1;
    const int nc = ctl->carry_n[bi][cin];
    const BeamBuf a = B.buf[par];
    const BeamBuf c = B.carry[cin];
    const int nsubc = B.n_subcycles;
    const double dtb = ctl->beam_dt / nsubc;
    const double clight = g.c, inv_c2 = 1. / (g.c * g.c);
    const double cmr = B.charge / B.mass;
    const double min_z = g.plo[2] + s * g.dx[2];
    for (long long k = gtid(); k < na + nc; k += gstride()) {
        const BeamBuf& bb = k < na ? a : c;
        const long long ip = k < na ? start + k : k - na;
        if (!bb.valid[ip]) continue;
        double xp = bb.x[ip], yp = bb.y[ip], zp = bb.z[ip], ux = bb.ux[ip], uy = bb.uy[ip], uz = bb.uz[ip];
        int i = bb.nsub[ip];
        bool absorbed = false;
        for (; i < nsubc; i++) {
            if (zp < min_z) break;
            const double gpi = 1. / sqrt(1. + (ux * ux + uy * uy + uz * uz) * inv_c2);
            xp += dtb * 0.5 * ux * gpi;
            yp += dtb * 0.5 * uy * gpi;
            if (!enforce_bc<double>(g, xp, yp, ux, uy)) { absorbed = true; break; }
            double Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
            gather<R, double, ORD>(S, g, xp, yp, Ex, Ey, Ez, Bx, By, Bz);
            if (B.ext) {
                // ApplyExternalField (ExternalFields.H:29-56) at the step's start time; Ex, Ey
                // here are ExmBy, EypBx
                const double at[4] = {xp, yp, zp, ctl->phys_time};
                double f[6];
#pragma unroll
                for (int q = 0; q < 6; ++q) f[q] = B.ext[q].eval(at);
                Ex += f[0] - clight * f[4];
                Ey += f[1] + clight * f[3];
                Ez += f[2];
                Bx += f[3];
                By += f[4];
                Bz += f[5];
            }
            const double uxn = ux + dtb * cmr * (Ex + (clight - uz * gpi) * By + uy * gpi * Bz);
            const double uyn = uy + dtb * cmr * (Ey + (uz * gpi - clight) * Bx - ux * gpi * Bz);
            const double uxi = (uxn + ux) * 0.5, uyi = (uyn + uy) * 0.5;
            const double uzi = uz + dtb * 0.5 * cmr * Ez;
            const double gii = 1. / sqrt(1. + (uxi * uxi + uyi * uyi + uzi * uzi) * inv_c2);
            const double uzn = uz + dtb * cmr * (Ez + (uxi * By - uyi * Bx) * gii);
            const double gni = 1. / sqrt(1. + (uxn * uxn + uyn * uyn + uzn * uzn) * inv_c2);
            xp += dtb * 0.5 * uxn * gni;
            yp += dtb * 0.5 * uyn * gni;
            if (B.do_z_push) zp += dtb * (uzn * gni - clight);
            ux = uxn; uy = uyn; uz = uzn;
        }
        if (absorbed || !enforce_bc<double>(g, xp, yp, ux, uy)) { bb.w[ip] = 0; bb.valid[ip] = 0; continue; }
        bb.x[ip] = xp; bb.y[ip] = yp; bb.z[ip] = zp; bb.nsub[ip] = i;
        bb.ux[ip] = ux; bb.uy[ip] = uy; bb.uz[ip] = uz;
    }
}

// ------------------------------------------------------------------------------------------
// Slice partition after the beam push (SliceSort.cpp:13-64 with the MultiBuffer hand-off,
// MultiBuffer.cpp:806-926) of slice ctl->islice + lag: invalid particles are dropped, particles
// still on the slice are appended to the next step's store (sub-cycle count reset), slipped
// particles go to the carry buffer of the next slice. One block; stable order via block-wide
// prefix sums.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void copy_particle(const BeamBuf& d, long long di, const BeamBuf& s, long long si, int nsub) {
    d.x[di] = s.x[si]; d.y[di] = s.y[si]; d.z[di] = s.z[si]; d.w[di] = s.w[si];
    d.ux[di] = s.ux[si]; d.uy[di] = s.uy[si]; d.uz[di] = s.uz[si];
    d.id[di] = s.id[si]; d.nsub[di] = nsub; d.valid[di] = 1;
}

// ------------------------------------------------------------------------------------------
// In-situ reductions (BeamParticleContainer.cpp:476-548, Fields.cpp:1289-1346), one block per
// slice so that the sums are taken in a fixed order (bit-identical run to run). Raw sums per
// slice go to out[islice * NV + k]; the host normalises them.
// ------------------------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&a)[NV], double* out) {
    __shared__ double ws[32][NV];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int d = 16; d > 0; d >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], d);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) ws[warp][k] = a[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
}

// beam "This" slice: the slice's own particles and those that slipped in from the previous slice
__global__ void __launch_bounds__(1024) k_beam_insitu(BeamDev B, const Ctl* __restrict__ ctl, int bi, double r2,
                                                      double clight_inv, double* out, int lag, int nz) {
    HPQ_PDL_ENTRY();
    if (!ctl->insitu_beam[bi]) return;
    const int s = ctl->islice + lag;
    if (s < 0 || s >= nz) return;
    const int par = ctl->step_parity;
    const int start = B.start[par][s], na = B.count[par][s];
    const int cin = (s + 1) & 1;
    const int nc = ctl->carry_n[bi][cin];
    double a[23];
#pragma unroll
    for (int k = 0; k < 23; ++k) a[k] = 0;
    for (int k = threadIdx.x; k < na + nc; k += blockDim.x) {
        const BeamBuf& bb = k < na ? B.buf[par] : B.carry[cin];
        const long long ip = k < na ? start + k : k - na;
        const double x = bb.x[ip], y = bb.y[ip];
        if (!bb.valid[ip] || x * x + y * y > r2) continue;
        const double z = bb.z[ip], w = bb.w[ip];
        const double ux = bb.ux[ip] * clight_inv, uy = bb.uy[ip] * clight_inv, uz = bb.uz[ip] * clight_inv;
        const double uz_inv = uz == 0. ? 0. : 1. / uz;
        const double gamma = sqrt(1.0 + ux * ux + uy * uy + uz * uz);
        a[0] += w; a[1] += w * x; a[2] += w * x * x; a[3] += w * y; a[4] += w * y * y; a[5] += w * z;
        a[6] += w * z * z; a[7] += w * ux; a[8] += w * ux * ux; a[9] += w * uy; a[10] += w * uy * uy;
        a[11] += w * uz; a[12] += w * uz * uz; a[13] += w * x * ux; a[14] += w * y * uy; a[15] += w * z * uz;
        a[16] += w * x * uy; a[17] += w * y * ux; a[18] += w * ux * uz_inv; a[19] += w * uy * uz_inv;
        a[20] += w * gamma; a[21] += w * gamma * gamma; a[22] += 1.0;
    }
    block_sum_store<23>(a, out + (size_t)s * 23);
}

template <class R>
__global__ void __launch_bounds__(1024) k_field_insitu(Slab<R> S, const Ctl* __restrict__ ctl, double clight,
                                                       double* out) {
    HPQ_PDL_ENTRY();
    if (!ctl->insitu_fields) return;
    const F2<R> ex = S.c(C_EXMBY), ey = S.c(C_EYPBX), ez = S.c(C_EZ), bx = S.c(C_BX), by = S.c(C_BY), bz = S.c(C_BZ),
                jzb = S.c(C_JZB);
    double a[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) a[k] = 0;
    for (int k = threadIdx.x; k < S.nx * S.ny; k += blockDim.x) {
        const int i = k % S.nx, j = k / S.nx;
        const double vex = ex(i, j), vey = ey(i, j), vez = ez(i, j), vbx = bx(i, j), vby = by(i, j), vbz = bz(i, j),
                     vj = jzb(i, j);
        const double t0 = vex + vby * clight, t1 = vey - vbx * clight;
        a[0] += t0 * t0; a[1] += t1 * t1; a[2] += vez * vez; a[3] += vbx * vbx; a[4] += vby * vby; a[5] += vbz * vbz;
        a[6] += vex * vex; a[7] += vey * vey; a[8] += vj; a[9] += vez * vj;
    }
    block_sum_store<10>(a, out + (size_t)ctl->islice * 10);
}

// ------------------------------------------------------------------------------------------
// Slice binning of an uploaded beam (BoxSort.cpp:14-78): slice = int((z - plo_z) dzi), particles
// outside [0, nz) dropped, slices stored top-down (nz-1 first), input order kept within a slice.
// A stable counting sort in four launches: per-chunk histograms, per-slice scans across chunks,
// the scan over slices, and a scatter in which one warp walks its chunk in order, ranking equal
// slices within each group of 32 with __match_any_sync.
// ------------------------------------------------------------------------------------------
constexpr int kBinChunk = 8192;  // particles per chunk (one block of the histogram and scatter)

// key[i] = slice of particle i or -1; hist[k * nb + b] = particles of chunk b in slice k
__global__ void __launch_bounds__(256) k_bin_hist(const double* __restrict__ z, long long n, double plo, double dzi,
                                                  int nz, int* __restrict__ key, int* __restrict__ hist, int nb) {
    HPQ_PDL_ENTRY();
    extern __shared__ int sh[];
    for (int k = threadIdx.x; k < nz; k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const long long i0 = (long long)blockIdx.x * kBinChunk;
    const long long i1 = i0 + kBinChunk < n ? i0 + kBinChunk : n;
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int s = (int)((z[i] - plo) * dzi);
        const int k = (s < 0 || s >= nz) ? -1 : s;
        key[i] = k;
        if (k >= 0) atomicAdd(&sh[k], 1);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nz; k += blockDim.x) hist[(size_t)k * nb + blockIdx.x] = sh[k];
}

// one block per slice: exclusive prefix of the slice's chunk counts (in place) and its total
__global__ void __launch_bounds__(256) k_bin_scan_chunks(int* __restrict__ hist, int nb, int* __restrict__ count) {
    HPQ_PDL_ENTRY();
    __shared__ int ws[8];
    __shared__ int carry;
    int* h = hist + (size_t)blockIdx.x * nb;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        const int v = b < nb ? h[b] : 0;
        int x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += t;
        }
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        int wsum = 0;
        for (int w = 0; w < warp; ++w) wsum += ws[w];
        const int base = carry;
        if (b < nb) h[b] = base + wsum + x - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = base + wsum + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) count[blockIdx.x] = carry;
}

// one block: start of every slice, top slice first
__global__ void __launch_bounds__(1024) k_bin_scan_slices(const int* __restrict__ count, int nz, int* __restrict__ start,
                                                          long long* __restrict__ total) {
    HPQ_PDL_ENTRY();
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r0 = 0; r0 < nz; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;  // rank from the top: slice nz-1-r
        const int v = r < nz ? count[nz - 1 - r] : 0;
        int x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += t;
        }
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        int wsum = 0;
        for (int w = 0; w < warp; ++w) wsum += ws[w];
        const int base = carry;
        if (r < nz) start[nz - 1 - r] = base + wsum + x - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = base + wsum + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// one warp per chunk, in input order: perm[start[k] + hist[k][b] + rank] = i
__global__ void __launch_bounds__(32) k_bin_scatter(const int* __restrict__ key, long long n, const int* __restrict__ hist,
                                                    int nb, const int* __restrict__ start, int nz, int* __restrict__ perm) {
    HPQ_PDL_ENTRY();
    extern __shared__ int cnt[];
    const int b = blockIdx.x, lane = threadIdx.x;
    for (int k = lane; k < nz; k += 32) cnt[k] = start[k] + hist[(size_t)k * nb + b];
    __syncwarp();
    const long long i0 = (long long)b * kBinChunk;
    const long long i1 = i0 + kBinChunk < n ? i0 + kBinChunk : n;
    const unsigned lt = (1u << lane) - 1u;
    for (long long g0 = i0; g0 < i1; g0 += 32) {
        const long long i = g0 + lane;
        const int k = i < i1 ? key[i] : -2;
        const unsigned m = __match_any_sync(0xffffffffu, k);
        const int rank = __popc(m & lt);
        if (k >= 0) perm[cnt[k] + rank] = (int)i;
        __syncwarp();
        if (k >= 0 && (m & lt) == 0) cnt[k] += __popc(m);
        __syncwarp();
    }
}

// particles received for one slice (time-step pipeline): sub-cycle count 0, valid where w != 0
__global__ void k_beam_slice_flags(BeamBuf dst, long long c0, long long n) {
    HPQ_PDL_ENTRY();
    for (long long k = gtid(); k < n; k += gstride()) {
        dst.nsub[c0 + k] = 0;
        dst.valid[c0 + k] = dst.w[c0 + k] != 0.0;
    }
}

// initial store of a beam: dst[k] = src[perm[k]] for k < *n (stable slice binning order)
__global__ void k_beam_gather(BeamBuf dst, const BeamBuf src, const int* __restrict__ perm, const long long* n_dev,
                              int has_id) {
    HPQ_PDL_ENTRY();
    const long long n = *n_dev;
    for (long long k = gtid(); k < n; k += gstride()) {
        const int i = perm[k];
        dst.x[k] = src.x[i]; dst.y[k] = src.y[i]; dst.z[k] = src.z[i]; dst.w[k] = src.w[i];
        dst.ux[k] = src.ux[i]; dst.uy[k] = src.uy[i]; dst.uz[k] = src.uz[i];
        dst.id[k] = has_id ? src.id[i] : (long long)i + 1;
        dst.nsub[k] = 0;
        dst.valid[k] = src.w[i] != 0.0;
    }
}

__global__ void __launch_bounds__(1024) k_beam_partition(BeamDev B, Ctl* ctl, int bi, Geo g, int keep_store, int lag) {
    HPQ_PDL_ENTRY();
    constexpr int IT = 8;  // consecutive particles per thread and round
    __shared__ int sst[32], ssl[32];
    __shared__ int base_stay, base_slip;
    const int s = ctl->islice + lag;
    if (s < 0 || s >= g.nz) return;
    const int par = ctl->step_parity;
    const int start = B.start[par][s], na = B.count[par][s];
    const int cin = (s + 1) & 1, cout = s & 1;
    const int nc = ctl->carry_n[bi][cin];
    const BeamBuf a = B.buf[par];
    const BeamBuf c = B.carry[cin];
    const BeamBuf o = B.buf[1 - par];
    const BeamBuf co = B.carry[cout];
    const double min_z = g.plo[2] + s * g.dx[2];
    const int cursor = ctl->cursor[bi];
    if (threadIdx.x == 0) { base_stay = 0; base_slip = 0; }
    __syncthreads();
    const int total = na + nc;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int round = 0; round < total; round += blockDim.x * IT) {
        const int first = round + threadIdx.x * IT;
        unsigned stay_m = 0, slip_m = 0;
#pragma unroll
        for (int q = 0; q < IT; ++q) {
            const int k = first + q;
            if (k >= total) break;
            const BeamBuf& bb = k < na ? a : c;
            const long long ip = k < na ? start + k : k - na;
            if (bb.valid[ip]) {
                if (bb.z[ip] >= min_z) stay_m |= 1u << q; else slip_m |= 1u << q;
            }
        }
        const int ns = __popc(stay_m), nl = __popc(slip_m);
        // block-wide exclusive scans of the per-thread counts
        int vs = ns, vl = nl;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int t1 = __shfl_up_sync(0xffffffffu, vs, d), t2 = __shfl_up_sync(0xffffffffu, vl, d);
            if (lane >= d) { vs += t1; vl += t2; }
        }
        if (lane == 31) { sst[warp] = vs; ssl[warp] = vl; }
        __syncthreads();
        if (warp == 0) {
            int ws = lane < nwarps ? sst[lane] : 0;
            int wl = lane < nwarps ? ssl[lane] : 0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                int t1 = __shfl_up_sync(0xffffffffu, ws, d), t2 = __shfl_up_sync(0xffffffffu, wl, d);
                if (lane >= d) { ws += t1; wl += t2; }
            }
            sst[lane] = ws; ssl[lane] = wl;
        }
        __syncthreads();
        int os = base_stay + (warp ? sst[warp - 1] : 0) + vs - ns;
        int ol = base_slip + (warp ? ssl[warp - 1] : 0) + vl - nl;
#pragma unroll
        for (int q = 0; q < IT; ++q) {
            const int k = first + q;
            const bool st_ = (stay_m >> q) & 1u, sl_ = (slip_m >> q) & 1u;
            if (!st_ && !sl_) continue;
            const BeamBuf& bb = k < na ? a : c;
            const long long ip = k < na ? start + k : k - na;
            if (st_) { if (keep_store) copy_particle(o, cursor + os, bb, ip, 0); ++os; }
            else { copy_particle(co, ol, bb, ip, bb.nsub[ip]); ++ol; }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            base_stay += sst[nwarps - 1];
            base_slip += ssl[nwarps - 1];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        B.start[1 - par][s] = cursor;
        B.count[1 - par][s] = keep_store ? base_stay : 0;
        if (keep_store) ctl->cursor[bi] = cursor + base_stay;
        ctl->carry_n[bi][cout] = base_slip;
    }
}

// ------------------------------------------------------------------------------------------
// Elementwise field kernels
// ------------------------------------------------------------------------------------------
struct CompList {
    int n;
    int c[24];
};

// deterministic deposition: listed planes += fixed-point totals (see addc), shadows cleared
template <class R>
__global__ void k_det_flush(Slab<R> S, DetAcc d, CompList L) {
    HPQ_PDL_ENTRY();
    const size_t n = S.cstride;
    for (long long k = gtid(); k < (long long)n; k += gstride())
        for (int q = 0; q < L.n; ++q) {
            const size_t e = (size_t)L.c[q] * S.cstride + k;
            const long long a = d.w[0][e], b = d.w[1][e], c = d.w[2][e];
            if ((a | b | c) == 0) continue;
            const double v = ((double)c * 0x1p-90 + (double)b * 0x1p-50) + (double)a * 0x1p-10;
            S.base[e] += (R)v;
            d.w[0][e] = 0; d.w[1][e] = 0; d.w[2][e] = 0;
        }
}

// zero listed components over the whole allocated slice (setVal on growntilebox)
template <class R>
__global__ void k_zero_comps(Slab<R> S, CompList L) {
    HPQ_PDL_ENTRY();
    const size_t n = S.cstride;
    for (long long k = gtid(); k < (long long)n; k += gstride())
#pragma unroll 4
        for (int q = 0; q < L.n; ++q) S.base[(size_t)L.c[q] * S.cstride + k] = R(0);
}

// dst[q] = src[q] over the whole allocated slice (Fields::shift / duplicate)
struct CopyList {
    int n;
    int dst[8], src[8];
};
template <class R>
__global__ void k_copy_comps(Slab<R> S, CopyList L) {
    HPQ_PDL_ENTRY();
    const size_t n = S.cstride;
    for (long long k = gtid(); k < (long long)n; k += gstride())
        for (int q = 0; q < L.n; ++q) S.base[(size_t)L.dst[q] * S.cstride + k] = S.base[(size_t)L.src[q] * S.cstride + k];
}

// AddRhoIons + the three right-hand sides of SolvePoissonPsiExmByEypBxEzBz
// (Fields.cpp:606-615, 840-903). Staging layout: stage[(j*3 + k)*ldx + i], k = Psi, Ez, Bz.
template <class R>
__global__ void k_rhs3(Slab<R> S, Geo g, R* __restrict__ stage, int sk, int sj, int add_ions, int add_rho, int add_rmb) {
    HPQ_PDL_ENTRY();
    const int ax = S.nx + 2 * kGuardAlloc;
    const long long ntot = (long long)ax * S.rows;
    const F2<R> rm = S.c(C_RHOMJZ), jx = S.c(C_JX), jy = S.c(C_JY), ions = S.c(C_IONS), rho = S.c(C_RHO),
                rmb = S.c(C_RHOMJZB);
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]);
    const R fe = (R)(1. / (g.ep0 * g.c)), mu0 = (R)g.mu0, mep = (R)(-1. / g.ep0);
    for (long long k = gtid(); k < ntot; k += gstride()) {
        const int i = (int)(k % ax) - kGuardAlloc, j = (int)(k / ax) - kGuardAlloc;
        R r = rm(i, j);
        if (add_ions) { r += ions(i, j); if (add_rho) rho(i, j) += ions(i, j); }
        if (add_rmb) r += rmb(i, j);
        if (add_ions || add_rmb) rm(i, j) = r;
        if (i >= 0 && i < S.nx && j >= 0 && j < S.ny) {
            R* st = stage + (size_t)j * sj + i;
            st[0] = mep * r;
            st[sk] = fe * ((jx(i + 1, j) - jx(i - 1, j)) * hx) + fe * ((jy(i, j + 1) - jy(i, j - 1)) * hy);
            st[2 * (size_t)sk] = mu0 * ((jx(i, j + 1) - jx(i, j - 1)) * hy) + (-mu0) * ((jy(i + 1, j) - jy(i - 1, j)) * hx);
        }
    }
}

// ExmBy = -dPsi/dx, EypBx = -dPsi/dy on the box grown by one guard (Fields.cpp:931-956)
template <class R>
__global__ void k_grad_psi(Slab<R> S, Geo g) {
    HPQ_PDL_ENTRY();
    const int w = S.nx + 2, h = S.ny + 2;
    const F2<R> Psi = S.c(C_PSI), Ex = S.c(C_EXMBY), Ey = S.c(C_EYPBX);
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]);
    for (long long k = gtid(); k < (long long)w * h; k += gstride()) {
        const int i = (int)(k % w) - 1, j = (int)(k / w) - 1;
        Ex(i, j) = -(Psi(i + 1, j) - Psi(i - 1, j)) * hx;
        Ey(i, j) = -(Psi(i, j + 1) - Psi(i, j - 1)) * hy;
    }
}

// ExmBy/EypBx = -grad Psi (Fields.cpp:931-956) and the beam part of Sx, Sy
// (Hipace.cpp:744-790) in one launch
template <class R>
__global__ void k_grad_psi_sxsy(Slab<R> S, Geo g) {
    HPQ_PDL_ENTRY();
    const int w = S.nx + 2, h = S.ny + 2;
    const F2<R> Psi = S.c(C_PSI), Ex = S.c(C_EXMBY), Ey = S.c(C_EYPBX);
    const F2<R> jzb = S.c(C_JZB), pjx = S.c(C_PJXB), pjy = S.c(C_PJYB), njx = S.c(C_NJXB), njy = S.c(C_NJYB),
                Sx = S.c(C_SX), Sy = S.c(C_SY);
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]);
    const R mu0 = (R)g.mu0;
    const R dx2 = (R)(2. * g.dx[0]), dy2 = (R)(2. * g.dx[1]), dz2 = (R)(2. * g.dx[2]);
    for (long long k = gtid(); k < (long long)w * h; k += gstride()) {
        const int i = (int)(k % w) - 1, j = (int)(k / w) - 1;
        Ex(i, j) = -(Psi(i + 1, j) - Psi(i - 1, j)) * hx;
        Ey(i, j) = -(Psi(i, j + 1) - Psi(i, j - 1)) * hy;
        if (i >= 0 && i < S.nx && j >= 0 && j < S.ny) {
            const R dx_jzb = (jzb(i + 1, j) - jzb(i - 1, j)) / dx2;
            const R dy_jzb = (jzb(i, j + 1) - jzb(i, j - 1)) / dy2;
            const R dz_jxb = (pjx(i, j) - njx(i, j)) / dz2;
            const R dz_jyb = (pjy(i, j) - njy(i, j)) / dz2;
            Sy(i, j) = mu0 * (-dy_jzb + dz_jyb);
            Sx(i, j) = -mu0 * (-dx_jzb + dz_jxb);
        }
    }
}

// Sx, Sy from the beam currents (Hipace.cpp:744-790)
template <class R>
__global__ void k_sxsy_beam(Slab<R> S, Geo g) {
    HPQ_PDL_ENTRY();
    const F2<R> jzb = S.c(C_JZB), pjx = S.c(C_PJXB), pjy = S.c(C_PJYB), njx = S.c(C_NJXB), njy = S.c(C_NJYB),
                Sx = S.c(C_SX), Sy = S.c(C_SY);
    const R mu0 = (R)g.mu0;
    const R dx2 = (R)(2. * g.dx[0]), dy2 = (R)(2. * g.dx[1]), dz2 = (R)(2. * g.dx[2]);
    for (long long k = gtid(); k < (long long)S.nx * S.ny; k += gstride()) {
        const int i = (int)(k % S.nx), j = (int)(k / S.nx);
        const R dx_jzb = (jzb(i + 1, j) - jzb(i - 1, j)) / dx2;
        const R dy_jzb = (jzb(i, j + 1) - jzb(i, j - 1)) / dy2;
        const R dz_jxb = (pjx(i, j) - njx(i, j)) / dz2;
        const R dz_jyb = (pjy(i, j) - njy(i, j)) / dz2;
        Sy(i, j) = mu0 * (-dy_jzb + dz_jyb);
        Sx(i, j) = -mu0 * (-dx_jzb + dz_jxb);
    }
}

// PC: right-hand sides of Bx, By (Fields.cpp:1008-1078) into stage rows k = 0 (Bx), 1 (By)
template <class R>
__global__ void k_rhs_bxby(Slab<R> S, Geo g, R* __restrict__ stage, int sk, int sj) {
    HPQ_PDL_ENTRY();
    const F2<R> jz = S.c(C_JZ), pjx = S.c(C_PJX), pjy = S.c(C_PJY), njx = S.c(C_NJX), njy = S.c(C_NJY);
    const R mu0 = (R)g.mu0;
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]), hz = (R)(0.5 * g.dxi[2]);
    for (long long k = gtid(); k < (long long)S.nx * S.ny; k += gstride()) {
        const int i = (int)(k % S.nx), j = (int)(k / S.nx);
        R* st = stage + (size_t)j * sj + i;
        st[0] = -mu0 * ((jz(i, j + 1) - jz(i, j - 1)) * hy) + mu0 * ((pjy(i, j) - njy(i, j)) * hz);
        st[sk] = mu0 * ((jz(i + 1, j) - jz(i - 1, j)) * hx) + (-mu0) * ((pjx(i, j) - njx(i, j)) * hz);
    }
}

// copy interior of listed components into the 3-D diagnostic buffer at the current slice
// out layout: [q][nz][ny][nx]
// diagnostic plane of a slice: the whole slice (type 0), or the row (type 1, xz) / column
// (type 2, yz) at the domain centre, interpolated between cells lo and hi with weights wlo, whi
struct DiagSel {
    int type, lo, hi;
    double wlo, whi;
};
template <class R>
__global__ void k_diag_copy(Slab<R> S, const Ctl* ctl, CompList L, double* __restrict__ out, int nz, DiagSel d) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice;
    const long long np = d.type == 0 ? (long long)S.nx * S.ny : d.type == 1 ? S.nx : S.ny;
    for (long long k = gtid(); k < np * L.n; k += gstride()) {
        const int q = (int)(k / np);
        const long long r = k % np;
        const F2<R> f = S.c(L.c[q]);
        double v;
        if (d.type == 0) v = (double)f((int)(r % S.nx), (int)(r / S.nx));
        else if (d.type == 1) v = d.wlo * (double)f((int)r, d.lo) + d.whi * (double)f((int)r, d.hi);
        else v = d.wlo * (double)f(d.lo, (int)r) + d.whi * (double)f(d.hi, (int)r);
        out[((size_t)q * nz + s) * np + r] = v;
    }
}

}  // namespace hpq
