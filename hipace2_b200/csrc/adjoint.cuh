// Adjoint of one step of the explicit slice march in double precision (hpq_adjoint_grad).
//
// The reference has no adjoint. The objective and parameters are defined by hpq::AdjointConfig
// (config.hpp): the current-weighted variance of Ez over the witness slices, differentiated with
// respect to the knots of the witness current profile and of the plasma density multiplier.
//
// Forward: the slice march of one step without the beam push (which only feeds the next step).
// Every K-th slice (adjoint.checkpoint_interval) the plasma state and the slab are saved; within
// a segment of K slices each slice's plasma state (after the deposit's QSA test) and the fields
// the reverse sweep reads are recorded. Reverse: segments from the tail of the box to its head,
// each recomputed from its checkpoint (the last one is still recorded from the forward), then
// swept slice by slice from the tail up:
//   plasma push      per particle: tangent passes through gather + push (5 seeds on the state,
//                    6 on the gathered fields); field adjoints scattered by the gather shapes
//                    (the adjoint of a gather is a deposit)
//   objective        dJ/dEz = 2 jz (Ez - Ebar)/S0, dJ/djz = ((Ez - Ebar)^2 - J)/S0
//   multigrid        the transposed operator is W A W^-1 (W = 3/4 on the boundary rows of the
//                    cell-centred 4/3 closure, 1 elsewhere), so one solve of the forward
//                    multigrid with right-hand side W^-1 lambda_B gives mu = W A^-1 W^-1 lambda_B;
//                    dJ/dchi = mu B
//   explicit Sx/Sy   per particle: tangent passes; field adjoints in closed form
//   Sx/Sy beam part, ExmBy/EypBx = -grad Psi, Poisson right-hand sides: transposed difference
//                    stencils (gather form, no atomics); the DST solve is symmetric
//   plasma deposit   per particle: tangent passes (the adjoint of a deposit is a gather)
//   beam deposits    linear in the witness weights
// The oracle (oracle/oracle.cpp, adjoint_grad) restates the same sweep on the CPU; both are
// checked against central finite differences of the forward.
#pragma once

#include "kernels.cuh"

namespace hpq {

// ------------------------------------------------------------------------------------------
// Tangent numbers (value, one directional derivative)
// ------------------------------------------------------------------------------------------
struct Tn { double v, d; };
__device__ __forceinline__ Tn operator+(Tn a, Tn b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Tn operator-(Tn a, Tn b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Tn operator*(Tn a, Tn b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Tn operator/(Tn a, Tn b) { const double q = a.v / b.v; return {q, (a.d - q * b.d) / b.v}; }
__device__ __forceinline__ Tn operator-(Tn a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Tn operator+(Tn a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Tn operator+(double a, Tn b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Tn operator-(Tn a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Tn operator-(double a, Tn b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Tn operator*(Tn a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Tn operator*(double a, Tn b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Tn operator/(Tn a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Tn operator/(double a, Tn b) { const double q = a / b.v; return {q, -q * b.d / b.v}; }
__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Tn a) { return a.v; }
__device__ __forceinline__ Tn tseed(double v, bool on) { return {v, on ? 1.0 : 0.0}; }

template <class T> struct ASh { T s; int cell; };
template <class T> struct ADSh { T s, ds; int cell; };

// clamp_mid on a generic scalar: a clamped coordinate is constant
template <class T>
__device__ __forceinline__ T a_clamp(T x, int n) {
    if (val(x) < -1.0) return 0.0 * x - 1.0;
    if (val(x) > (double)n) return 0.0 * x + (double)n;
    return x;
}
// shape2 and dshape2 (common.cuh) on a generic scalar, same expressions
template <class T>
__device__ __forceinline__ ASh<T> a_shape2(T xmid, int ix) {
    const double xfloor = floor(val(xmid) + 0.5);
    const T xint = xmid - xfloor;
    const int c = (int)xfloor;
    if (ix == 0) return {0.5 * (0.5 - xint) * (0.5 - xint), c - 1};
    if (ix == 1) return {0.75 - xint * xint, c};
    return {0.5 * (0.5 + xint) * (0.5 + xint), c + 1};
}
template <class T>
__device__ __forceinline__ ADSh<T> a_dshape2(int type, T xmid, int ix) {
    if (type == 0) {
        xmid = xmid + 0.5;
        const double xfloor = floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        const int c = (int)xfloor - 1 + ix;
        if (ix == 0) return {0.5 * x2 - xint + 0.5, -(xint - 1.0), c};
        if (ix == 1) return {-x2 + xint + 0.5, -(1.0 - 2.0 * xint), c};
        return {0.5 * x2, -xint, c};
    } else if (type == 1) {
        const double xfloor = floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        const bool lo = val(xint) < 0.5;
        const T zero = 0.0 * xint;
        const int c = (int)xfloor - 1 + ix;
        if (ix == 0) return {lo ? 0.5 * x2 - 0.5 * xint + 1.0 / 8.0 : zero, -(-0.5 * x2 + xint - 0.5), c};
        if (ix == 1) return {lo ? 0.75 - x2 : 0.5 * x2 - 1.5 * xint + 9.0 / 8.0, -(1.5 * x2 - 2.0 * xint), c};
        if (ix == 2) return {lo ? 0.5 * x2 + 0.5 * xint + 1.0 / 8.0 : -x2 + 2.0 * xint - 0.25, -(-1.5 * x2 + xint + 0.5), c};
        return {lo ? zero : 0.5 * x2 - 0.5 * xint + 1.0 / 8.0, -(0.5 * x2), c};
    } else {
        xmid = xmid + 0.5;
        const double xfloor = floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        const T zero = 0.0 * xint;
        const int c = (int)xfloor - 2 + ix;
        if (ix == 0) return {zero, -(-0.25 * x2 + 0.5 * xint - 0.25), c};
        if (ix == 1) return {0.5 * x2 - xint + 0.5, -(0.5 * x2 - 0.5 * xint - 0.25), c};
        if (ix == 2) return {-x2 + xint + 0.5, -(0.25 - 0.5 * xint), c};
        if (ix == 3) return {0.5 * x2, -(-0.5 * x2 + 0.5 * xint + 0.25), c};
        return {zero, -(0.25 * x2), c};
    }
}

// ------------------------------------------------------------------------------------------
// Records and adjoint arrays
// ------------------------------------------------------------------------------------------
enum RecField : int { RF_PSI = 0, RF_EZ, RF_BZ, RF_BX, RF_BY, RF_EXMBY, RF_EYPBX, RF_CHI, RF_JZB, RF_N };
// slab components recorded per slice, in RecField order
constexpr int kRecComp[RF_N] = {C_PSI, C_EZ, C_BZ, C_BX, C_BY, C_EXMBY, C_EYPBX, C_CHI, C_JZB};

// adjoint slab: lambda of each slice field, plus the three Poisson adjoint solutions (V*)
enum AdjComp : int {
    A_PSI = 0, A_EZ, A_BZ, A_BX, A_BY, A_EXMBY, A_EYPBX, A_SX, A_SY, A_CHI, A_JX, A_JY, A_RM, A_JZB,
    A_PJX, A_PJY, A_NJX, A_NJY, A_VPSI, A_VEZ, A_VBZ, A_NCOMP
};

// plasma state of one slice: positions, half-step and deposited momenta and psi after the
// deposit of the slice (invalidated particles have valid = 0); weights of the step
struct AdjPlasma {
    const double *x, *y, *uxh, *uyh, *psih, *ux, *uy, *psi, *w;
    const uint8_t* valid;
    long long n;
    double charge, mass;
};
// adjoint of the plasma state (same attributes)
struct AdjLam {
    double *x, *y, *uxh, *uyh, *psih, *ux, *uy, *psi;
};
struct AdjRecF {
    F2<double> f[RF_N];
};

// ------------------------------------------------------------------------------------------
// Per-particle maps on a generic scalar (double for values, Tn for derivatives)
// ------------------------------------------------------------------------------------------
// FieldGather (derivative type 1, 4x4): G = ExmBy, EypBx, Ez, c Bx, c By, Bz
template <class T>
__device__ __forceinline__ void a_gather(const AdjRecF& F, const Geo& g, T xp, T yp, T* G) {
    const T x = a_clamp((xp - g.xoff) * g.dxi[0], g.nx), y = a_clamp((yp - g.yoff) * g.dxi[1], g.ny);
    const double dxi = g.dxi[0], dyi = g.dxi[1];
#pragma unroll
    for (int c = 0; c < 6; ++c) G[c] = 0.0 * x;
#pragma unroll 1
    for (int iy = 0; iy < 4; iy++) {
        const ADSh<T> sy = a_dshape2<T>(1, y, iy);
#pragma unroll
        for (int ix = 0; ix < 4; ix++) {
            const ADSh<T> sx = a_dshape2<T>(1, x, ix);
            const int i = sx.cell, j = sy.cell;
            const double psi = F.f[RF_PSI](i, j);
            G[0] = G[0] + (sx.ds * sy.s) * (psi * dxi);
            G[1] = G[1] + (sx.s * sy.ds) * (psi * dyi);
            const T s = sx.s * sy.s;
            G[2] = G[2] + s * F.f[RF_EZ](i, j);
            G[3] = G[3] + s * F.f[RF_BX](i, j);
            G[4] = G[4] + s * F.f[RF_BY](i, j);
            G[5] = G[5] + s * F.f[RF_BZ](i, j);
        }
    }
    G[3] = G[3] * g.c;
    G[4] = G[4] * g.c;
}

// EnforceBC on a generic scalar: the wrap is a shift by a constant, the reflection flips signs
template <class T>
__device__ __forceinline__ bool a_enforce_bc(const Geo& g, T& x, T& y, T& ux, T& uy) {
    const double plo0 = g.plo_p[0], plo1 = g.plo_p[1], phi0 = g.phi_p[0], phi1 = g.phi_p[1];
    if (val(x) < plo0 || val(y) < plo1 || val(x) > phi0 || val(y) > phi1) {
        if (g.bc != 0 && g.bc != 1) return false;
        const bool refl = g.bc == 0;
        const double lx = phi0 - plo0, ly = phi1 - plo1;
        const double px = refl ? 2 * lx : lx, py = refl ? 2 * ly : ly;
        double m = fmod(val(x) - plo0, px);
        if (m < 0) m += px;
        x = x + ((m + plo0) - val(x));
        m = fmod(val(y) - plo1, py);
        if (m < 0) m += py;
        y = y + ((m + plo1) - val(y));
        if (refl && val(x) > phi0) { x = 2 * phi0 - x; ux = -ux; }
        if (refl && val(y) > phi1) { y = 2 * phi1 - y; uy = -uy; }
    }
    return true;
}

template <class T> struct ADu { T v, e; };
template <class T> __device__ __forceinline__ ADu<T> operator+(ADu<T> a, ADu<T> b) { return {a.v + b.v, a.e + b.e}; }
template <class T> __device__ __forceinline__ ADu<T> operator-(ADu<T> a, ADu<T> b) { return {a.v - b.v, a.e - b.e}; }
template <class T> __device__ __forceinline__ ADu<T> operator*(ADu<T> a, ADu<T> b) { return {a.v * b.v, a.e * b.v + a.v * b.e}; }

// plasma push of one particle (n_subcycles 1) with gathered fields G. out: x, y, ux_h, uy_h,
// psi_h, ux, uy, psi. Returns false if the particle is absorbed.
template <class T>
__device__ __forceinline__ bool a_push(const Geo& g, double qmc, T x, T y, T ux, T uy, T psi, const T* G, T* out) {
    const double ci = 1. / g.c, dzs = g.dx[2];
    const double sdz = dzs / 4;
    auto substep = [&]() {
        const T pi = 1.0 / psi;
        const T gp = 0.5 * pi * pi * (1.0 + ux * ux * (ci * ci) + uy * uy * (ci * ci)) + 0.5;
        const T d0 = qmc * (gp * G[0] + G[4] + (uy * G[5]) * pi);
        const T d1 = qmc * (gp * G[1] - G[3] - (ux * G[5]) * pi);
        const T d2 = qmc * ci * ((ux * G[0] + uy * G[1]) * ci * pi - G[2]);
        const T z = 0.0 * psi;
        const ADu<T> dux{ux, d0}, duy{uy, d1}, dpi{pi, -pi * pi * d2};
        const ADu<T> c2{z + ci * ci, z}, one{z + 1.0, z}, half{z + 0.5, z}, q{z + qmc, z}, cc{z + ci, z};
        const ADu<T> E0{G[0], z}, E1{G[1], z}, E2{G[2], z}, B0{G[3], z}, B1{G[4], z}, B2{G[5], z};
        const ADu<T> gpd = half * dpi * dpi * (one + dux * dux * c2 + duy * duy * c2) + half;
        const ADu<T> e0 = q * (gpd * E0 + B1 + (duy * B2) * dpi);
        const ADu<T> e1 = q * (gpd * E1 - B0 - (dux * B2) * dpi);
        const ADu<T> e2 = q * cc * ((dux * E0 + duy * E1) * cc * dpi - E2);
        ux = ux + sdz * d0 + 0.5 * sdz * sdz * e0.e;
        uy = uy + sdz * d1 + 0.5 * sdz * sdz * e1.e;
        psi = psi + sdz * d2 + 0.5 * sdz * sdz * e2.e;
    };
#pragma unroll 1
    for (int k = 0; k < 4; ++k) substep();
    x = x + dzs * ci * (ux * (1.0 / psi));
    y = y + dzs * ci * (uy * (1.0 / psi));
    if (!a_enforce_bc(g, x, y, ux, uy)) return false;
    out[0] = x; out[1] = y; out[2] = ux; out[3] = uy; out[4] = psi;
#pragma unroll 1
    for (int k = 0; k < 2; ++k) substep();
    out[5] = ux; out[6] = uy; out[7] = psi;
    return true;
}

// ------------------------------------------------------------------------------------------
// Forward hooks (captured in the adjoint slice graph)
// ------------------------------------------------------------------------------------------
// a list of arrays copied into slot buffers (dst + slot * n)
template <class R>
struct AdjCopy {
    static constexpr int kMax = 20;
    const R* src[kMax];
    R* dst[kMax];
    long long n[kMax];
    int na;
    const uint8_t* vsrc;
    uint8_t* vdst;
    long long nv;
    int nz, K;
};

// checkpoint of the state entering slice islice when it starts a segment (and checkpoints are on)
template <class R>
__global__ void k_adj_checkpoint(const Ctl* __restrict__ ctl, AdjCopy<R> a) {
    HPQ_PDL_ENTRY();
    if (!ctl->adj_ckpt) return;
    const int d = a.nz - 1 - ctl->islice;
    if (d % a.K) return;
    const long long c = d / a.K;
    for (int k = 0; k < a.na; ++k)
        for (long long i = gtid(); i < a.n[k]; i += gstride()) a.dst[k][c * a.n[k] + i] = a.src[k][i];
    for (long long i = gtid(); i < a.nv; i += gstride()) a.vdst[c * a.nv + i] = a.vsrc[i];
}

// record of slice islice in its segment slot
template <class R>
__global__ void k_adj_record(const Ctl* __restrict__ ctl, AdjCopy<R> a) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice;
    const int c = (a.nz - 1 - s) / a.K;
    const int hi = a.nz - 1 - c * a.K;
    const int lo = hi - a.K + 1 > 0 ? hi - a.K + 1 : 0;
    const long long slot = s - lo;
    for (int k = 0; k < a.na; ++k)
        for (long long i = gtid(); i < a.n[k]; i += gstride()) a.dst[k][slot * a.n[k] + i] = a.src[k][i];
    for (long long i = gtid(); i < a.nv; i += gstride()) a.vdst[slot * a.nv + i] = a.vsrc[i];
}

// objective sums S0 = sum jz_beam, S1 = sum jz_beam Ez, S2 = sum jz_beam Ez^2 over the interior of
// an objective slice (zero elsewhere); one block, fixed order
template <class R>
__global__ void __launch_bounds__(1024) k_adj_objective_sums(Slab<R> S, const Ctl* __restrict__ ctl, Geo g,
                                                             double zlo, double zhi, double* out) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice;
    const double zc = g.plo[2] + (s + 0.5) * g.dx[2];
    double a[3] = {0, 0, 0};
    if (zc >= zlo && zc <= zhi) {
        const F2<R> jz = S.c(C_JZB), ez = S.c(C_EZ);
        for (long long k = threadIdx.x; k < (long long)S.nx * S.ny; k += blockDim.x) {
            const int i = (int)(k % S.nx), j = (int)(k / S.nx);
            const double q = (double)jz(i, j), e = (double)ez(i, j);
            a[0] += q; a[1] += q * e; a[2] += q * e * e;
        }
    }
    block_sum_store<3>(a, out + (size_t)s * 3);
}

// slice cursor and checkpoint switch of the adjoint forward; in-situ reductions stay off
__global__ void k_adj_set_slice(Ctl* ctl, int islice, int ckpt) {
    HPQ_PDL_ENTRY();
    ctl->islice = islice;
    ctl->adj_ckpt = ckpt;
    ctl->insitu_fields = 0;
    for (int b = 0; b < kMaxBeams; ++b) ctl->insitu_beam[b] = 0;
}

// ------------------------------------------------------------------------------------------
// Parameters
// ------------------------------------------------------------------------------------------
// witness weights of the read store: w = w0 * profile(z)
__global__ void k_adj_profile(BeamDev B, int par, int nz, const double* __restrict__ w0,
                              const double* __restrict__ knots, double lo, double hi, int n) {
    HPQ_PDL_ENTRY();
    const int s = blockIdx.y;
    if (s >= nz) return;
    const int start = B.start[par][s], cnt = B.count[par][s];
    const BeamBuf b = B.buf[par];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const long long ip = start + k;
        const double z = b.z[ip];
        double p = 0;
        if (z >= lo && z <= hi) {
            double t = (z - lo) / (hi - lo) * (n - 1);
            int kk = (int)t;
            if (kk > n - 2) kk = n - 2;
            const double f = t - kk;
            p = (1.0 - f) * knots[kk] + f * knots[kk + 1];
        }
        b.w[ip] = w0[ip] * p;
    }
}

// dJ/dknot_k = sum over witness particles of lambda_w * w0 * hat_k(z); one block per knot
__global__ void __launch_bounds__(256) k_adj_knot_grad(BeamDev B, int par, int nz, const double* __restrict__ lw,
                                                       const double* __restrict__ w0, double lo, double hi, int n,
                                                       double* grad) {
    HPQ_PDL_ENTRY();
    const int knot = blockIdx.x;
    const BeamBuf b = B.buf[par];
    double a[1] = {0};
    for (int s = 0; s < nz; ++s) {
        const int start = B.start[par][s], cnt = B.count[par][s];
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
            const long long ip = start + k;
            const double z = b.z[ip];
            if (!(z >= lo && z <= hi) || lw[ip] == 0.0) continue;
            double t = (z - lo) / (hi - lo) * (n - 1);
            int kk = (int)t;
            if (kk > n - 2) kk = n - 2;
            const double f = t - kk;
            const double gp = lw[ip] * w0[ip];
            if (kk == knot) a[0] += (1.0 - f) * gp;
            if (kk + 1 == knot) a[0] += f * gp;
        }
    }
    block_sum_store<1>(a, grad + knot);
}

// sum_p lambda_w[p] * w[p] (plasma weights of the step); one block
__global__ void __launch_bounds__(1024) k_adj_dot(const double* __restrict__ a, const double* __restrict__ b,
                                                  long long n, double* out) {
    HPQ_PDL_ENTRY();
    double s[1] = {0};
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s[0] += a[i] * b[i];
    block_sum_store<1>(s, out);
}

// interior dot product of two planes (the ion background term); one block
__global__ void __launch_bounds__(1024) k_adj_plane_dot(F2<double> a, F2<double> b, int nx, int ny, double* out) {
    HPQ_PDL_ENTRY();
    double s[1] = {0};
    for (long long k = threadIdx.x; k < (long long)nx * ny; k += blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        s[0] += a(i, j) * b(i, j);
    }
    block_sum_store<1>(s, out);
}

// ------------------------------------------------------------------------------------------
// Reverse sweep kernels (one slice)
// ------------------------------------------------------------------------------------------
struct AdjL {
    F2<double> f[A_NCOMP];
};

// plasma push: lin(x, y, ux_h, uy_h, psi_h) = J^T lout; lin(ux, uy, psi) = 0; field adjoints
// scattered by the gather shapes
__global__ void __launch_bounds__(128) k_adj_push(AdjPlasma P, AdjLam lout, AdjLam lin, AdjRecF F, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    const double qmc = P.charge / (P.mass * g.c);
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        lin.ux[ip] = 0; lin.uy[ip] = 0; lin.psi[ip] = 0;
        double lo[8] = {lout.x[ip], lout.y[ip], lout.uxh[ip], lout.uyh[ip], lout.psih[ip],
                        lout.ux[ip], lout.uy[ip], lout.psi[ip]};
        bool any = false;
#pragma unroll
        for (int o = 0; o < 8; ++o) any = any || lo[o] != 0.0;
        if (!P.valid[ip] || !any) {
            lin.x[ip] = 0; lin.y[ip] = 0; lin.uxh[ip] = 0; lin.uyh[ip] = 0; lin.psih[ip] = 0;
            continue;
        }
        const double in[5] = {P.x[ip], P.y[ip], P.uxh[ip], P.uyh[ip], P.psih[ip]};
        double d[5];
        bool alive = true;
#pragma unroll 1
        for (int k = 0; k < 5 && alive; ++k) {
            Tn t[5], G[6], out[8];
#pragma unroll
            for (int m = 0; m < 5; ++m) t[m] = tseed(in[m], m == k);
            a_gather<Tn>(F, g, t[0], t[1], G);
            alive = a_push<Tn>(g, qmc, t[0], t[1], t[2], t[3], t[4], G, out);
            double s = 0;
#pragma unroll
            for (int o = 0; o < 8; ++o) s += lo[o] * out[o].d;
            d[k] = s;
        }
        if (!alive) {
            lin.x[ip] = 0; lin.y[ip] = 0; lin.uxh[ip] = 0; lin.uyh[ip] = 0; lin.psih[ip] = 0;
            continue;
        }
        double Gv[6];
        a_gather<double>(F, g, in[0], in[1], Gv);
        double lG[6];
#pragma unroll 1
        for (int c = 0; c < 6; ++c) {
            Tn G[6], out[8];
#pragma unroll
            for (int m = 0; m < 6; ++m) G[m] = tseed(Gv[m], m == c);
            a_push<Tn>(g, qmc, tseed(in[0], false), tseed(in[1], false), tseed(in[2], false), tseed(in[3], false),
                       tseed(in[4], false), G, out);
            double s = 0;
#pragma unroll
            for (int o = 0; o < 8; ++o) s += lo[o] * out[o].d;
            lG[c] = s;
        }
        lin.x[ip] = d[0]; lin.y[ip] = d[1]; lin.uxh[ip] = d[2]; lin.uyh[ip] = d[3]; lin.psih[ip] = d[4];
        // adjoint of the gather: a deposit with the gather shapes
        const double x = a_clamp((in[0] - g.xoff) * g.dxi[0], g.nx), y = a_clamp((in[1] - g.yoff) * g.dxi[1], g.ny);
        const double dxi = g.dxi[0], dyi = g.dxi[1];
#pragma unroll 1
        for (int iy = 0; iy < 4; iy++) {
            const ADSh<double> sy = a_dshape2<double>(1, y, iy);
#pragma unroll
            for (int ix = 0; ix < 4; ix++) {
                const ADSh<double> sx = a_dshape2<double>(1, x, ix);
                const int i = sx.cell, j = sy.cell;
                const double s = sx.s * sy.s;
                atomicAdd(L.f[A_PSI].ptr(i, j), lG[0] * sx.ds * sy.s * dxi + lG[1] * sx.s * sy.ds * dyi);
                atomicAdd(L.f[A_EZ].ptr(i, j), lG[2] * s);
                atomicAdd(L.f[A_BX].ptr(i, j), lG[3] * g.c * s);
                atomicAdd(L.f[A_BY].ptr(i, j), lG[4] * g.c * s);
                atomicAdd(L.f[A_BZ].ptr(i, j), lG[5] * s);
            }
        }
    }
}

// objective: lambda_Ez += 2 jz (Ez - Ebar)/S0, lambda_jz += ((Ez - Ebar)^2 - J)/S0 (interior)
__global__ void k_adj_objective(AdjL L, AdjRecF F, int nx, int ny, double J, double Ebar, double S0) {
    HPQ_PDL_ENTRY();
    for (long long k = gtid(); k < (long long)nx * ny; k += gstride()) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        const double jz = F.f[RF_JZB](i, j), e = F.f[RF_EZ](i, j) - Ebar;
        L.f[A_EZ](i, j) += 2.0 * jz * e / S0;
        L.f[A_JZB](i, j) += (e * e - J) / S0;
    }
}

__device__ __forceinline__ double adj_mg_weight(int i, int j, int nx, int ny, int cellc) {
    double w = 1.0;
    if (cellc && (i == 0 || i == nx - 1)) w *= 0.75;
    if (cellc && (j == 0 || j == ny - 1)) w *= 0.75;
    return w;
}

// multigrid slab for the transposed solve: chi, rhs = W^-1 lambda_B (interior), zero guess
__global__ void k_adj_mg_pre(Slab<double> M, AdjL L, AdjRecF F, int cellc) {
    HPQ_PDL_ENTRY();
    const int ax = M.nx + 2 * kGuardAlloc;
    for (long long k = gtid(); k < (long long)ax * M.rows; k += gstride()) {
        const int i = (int)(k % ax) - kGuardAlloc, j = (int)(k / ax) - kGuardAlloc;
        const bool in = i >= 0 && j >= 0 && i < M.nx && j < M.ny;
        const double w = adj_mg_weight(i, j, M.nx, M.ny, cellc);
        M.c(C_CHI)(i, j) = F.f[RF_CHI](i, j);
        M.c(C_SY)(i, j) = in ? L.f[A_BX](i, j) / w : 0.0;
        M.c(C_SX)(i, j) = in ? L.f[A_BY](i, j) / w : 0.0;
        M.c(C_BX)(i, j) = 0.0;
        M.c(C_BY)(i, j) = 0.0;
    }
}
// mu = W * solution: lambda_Sy = mu_x, lambda_Sx = mu_y, lambda_chi = mu . B (interior)
__global__ void k_adj_mg_post(Slab<double> M, AdjL L, AdjRecF F, int cellc) {
    HPQ_PDL_ENTRY();
    for (long long k = gtid(); k < (long long)M.nx * M.ny; k += gstride()) {
        const int i = (int)(k % M.nx), j = (int)(k / M.nx);
        const double w = adj_mg_weight(i, j, M.nx, M.ny, cellc);
        const double mx = M.c(C_BX)(i, j) * w, my = M.c(C_BY)(i, j) * w;
        L.f[A_SY](i, j) = mx;
        L.f[A_SX](i, j) = my;
        L.f[A_CHI](i, j) = mx * F.f[RF_BX](i, j) + my * F.f[RF_BY](i, j);
    }
}

// explicit Sx/Sy deposit: lambda of the particle (+=) and of Bz, Ez, ExmBy, EypBx (scattered)
template <class T, int DT>
__device__ __forceinline__ T a_explicit_L(const AdjRecF& F, const AdjL& L, const Geo& g, double charge, double mass,
                                          double w, T x, T y, T ux, T uy, T psi, bool scatter) {
    const double invvol = g.normalized ? g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1] : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double a_clight = g.c, ci = 1. / g.c;
    const double cdm = charge * invvol * g.mu0 * w;
    const double qm = charge / mass;
    const double dxi = g.dxi[0], dyi = g.dxi[1];
    const T pi = 1.0 / psi;
    const T vx = ux * pi * ci, vy = uy * pi * ci;
    const T xmid = a_clamp((x - g.xoff) * dxi, g.nx), ymid = a_clamp((y - g.yoff) * dyi, g.ny);
    const T gp = 0.5 * (pi * pi + vx * vx + vy * vy + 1.0);
    constexpr int NS = 3 + DT;
    T acc = 0.0 * x;
#pragma unroll 1
    for (int iy = 0; iy < NS; ++iy) {
        const ADSh<T> sy = a_dshape2<T>(DT, ymid, iy);
#pragma unroll 1
        for (int ix = 0; ix < NS; ++ix) {
            if (DT == 2 && (ix == 0 || ix == 4) && (iy == 0 || iy == 4)) continue;
            const ADSh<T> sx = a_dshape2<T>(DT, xmid, ix);
            const int i = sx.cell, j = sy.cell;
            const double Bz = F.f[RF_BZ](i, j), Ez = F.f[RF_EZ](i, j), Ex = F.f[RF_EXMBY](i, j), Ey = F.f[RF_EYPBX](i, j);
            const double lsy = L.f[A_SY](i, j), lsx = L.f[A_SX](i, j);
            if (lsy == 0.0 && lsx == 0.0) continue;
            const T ss = sx.s * sy.s;
            const T vsy = cdm * (-ss * (-Bz * vx + (Ez * vy + Ex * (-vx * vy) + Ey * (gp - vy * vy)) * ci) * qm * pi +
                                 (-sx.ds * sy.s * dxi * (-vx * vy) - sx.s * sy.ds * dyi * (gp - vy * vy - 1.0)) * a_clight);
            const T vsx = cdm * (ss * (Bz * vy + (Ez * vx + Ex * (gp - vx * vx) + Ey * (-vx * vy)) * ci) * qm * pi +
                                 (sx.ds * sy.s * dxi * (gp - vx * vx - 1.0) + sx.s * sy.ds * dyi * (-vx * vy)) * a_clight);
            acc = acc + lsy * vsy + lsx * vsx;
            if (scatter) {
                const double K = val(ss * pi) * cdm * qm;
                const double a = val(vx), b = val(vy), gpv = val(gp);
                atomicAdd(L.f[A_BZ].ptr(i, j), lsy * K * a + lsx * K * b);
                atomicAdd(L.f[A_EZ].ptr(i, j), -lsy * K * b * ci + lsx * K * a * ci);
                atomicAdd(L.f[A_EXMBY].ptr(i, j), lsy * K * a * b * ci + lsx * K * (gpv - a * a) * ci);
                atomicAdd(L.f[A_EYPBX].ptr(i, j), -lsy * K * (gpv - b * b) * ci - lsx * K * a * b * ci);
            }
        }
    }
    return acc;
}

template <int DT>
__global__ void __launch_bounds__(128) k_adj_explicit(AdjPlasma P, AdjLam lin, double* lw, AdjRecF F, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        const double in[5] = {P.x[ip], P.y[ip], P.ux[ip], P.uy[ip], P.psi[ip]};
        double d[5];
#pragma unroll 1
        for (int k = 0; k < 5; ++k) {
            Tn t[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) t[m] = tseed(in[m], m == k);
            d[k] = a_explicit_L<Tn, DT>(F, L, g, P.charge, P.mass, P.w[ip], t[0], t[1], t[2], t[3], t[4], false).d;
        }
        lin.x[ip] += d[0]; lin.y[ip] += d[1]; lin.ux[ip] += d[2]; lin.uy[ip] += d[3]; lin.psi[ip] += d[4];
        lw[ip] += a_explicit_L<double, DT>(F, L, g, P.charge, P.mass, 1.0, in[0], in[1], in[2], in[3], in[4], false);
        a_explicit_L<double, DT>(F, L, g, P.charge, P.mass, P.w[ip], in[0], in[1], in[2], in[3], in[4], true);
    }
}

// Sx/Sy beam part (gather form): lambda_jz_beam on [-1, n], lambda of the previous/next slice's
// beam jx, jy (interior); and the Poisson stage: lambda_Psi (with the transposed -grad of
// ExmBy/EypBx), lambda_Ez, lambda_Bz on the interior
__global__ void k_adj_sxsy_stage(AdjL L, Geo g, int nx, int ny, double* stage, int sk, int sj) {
    HPQ_PDL_ENTRY();
    const double mu0 = g.mu0, dx = g.dx[0], dy = g.dx[1], dz = g.dx[2];
    const double hx = 0.5 * g.dxi[0], hy = 0.5 * g.dxi[1];
    const int w = nx + 2, h = ny + 2;
    for (long long k = gtid(); k < (long long)w * h; k += gstride()) {
        const int i = (int)(k % w) - 1, j = (int)(k / w) - 1;
        const F2<double> lsx = L.f[A_SX], lsy = L.f[A_SY];
        L.f[A_JZB](i, j) += -mu0 / (2 * dy) * lsy(i, j - 1) + mu0 / (2 * dy) * lsy(i, j + 1) +
                            mu0 / (2 * dx) * lsx(i - 1, j) - mu0 / (2 * dx) * lsx(i + 1, j);
        if (i >= 0 && j >= 0 && i < nx && j < ny) {
            const double ly = lsy(i, j), lx = lsx(i, j);
            L.f[A_PJY](i, j) = mu0 / (2 * dz) * ly;
            L.f[A_NJY](i, j) = -mu0 / (2 * dz) * ly;
            L.f[A_PJX](i, j) = -mu0 / (2 * dz) * lx;
            L.f[A_NJX](i, j) = mu0 / (2 * dz) * lx;
            const F2<double> ex = L.f[A_EXMBY], ey = L.f[A_EYPBX];
            double* st = stage + (size_t)j * sj + i;
            st[0] = L.f[A_PSI](i, j) - hx * ex(i - 1, j) + hx * ex(i + 1, j) - hy * ey(i, j - 1) + hy * ey(i, j + 1);
            st[sk] = L.f[A_EZ](i, j);
            st[2 * (size_t)sk] = L.f[A_BZ](i, j);
        }
    }
}

// transposed right-hand sides of the Psi, Ez, Bz solves (gather form on [-1, n]); V* are the
// adjoint solutions (zero outside the interior)
__global__ void k_adj_rhs_t(AdjL L, Geo g, int nx, int ny) {
    HPQ_PDL_ENTRY();
    const double hx = 0.5 * g.dxi[0], hy = 0.5 * g.dxi[1];
    const double fe = 1. / (g.ep0 * g.c), mu0 = g.mu0, mep = -1. / g.ep0;
    const F2<double> vp = L.f[A_VPSI], ve = L.f[A_VEZ], vb = L.f[A_VBZ];
    const int w = nx + 2, h = ny + 2;
    for (long long k = gtid(); k < (long long)w * h; k += gstride()) {
        const int i = (int)(k % w) - 1, j = (int)(k / w) - 1;
        L.f[A_JX](i, j) += fe * hx * (ve(i - 1, j) - ve(i + 1, j)) + mu0 * hy * (vb(i, j - 1) - vb(i, j + 1));
        L.f[A_JY](i, j) += fe * hy * (ve(i, j - 1) - ve(i, j + 1)) + mu0 * hx * (vb(i + 1, j) - vb(i - 1, j));
        if (i >= 0 && j >= 0 && i < nx && j < ny) L.f[A_RM](i, j) += mep * vp(i, j);
    }
}

// plasma deposit (jx, jy, chi, rho - jz): lambda of the particle (+=)
template <class T>
__device__ __forceinline__ T a_deposit_L(const AdjL& L, const Geo& g, double charge, double mass, double w, T x, T y,
                                         T ux, T uy, T psi) {
    const double invvol = g.normalized ? g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1] : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double q_invvol = charge * invvol * w;
    const double qm = charge * g.mu0 / mass;
    const T pi = 1.0 / psi;
    const T vx = ux * pi, vy = uy * pi;
    const T xmid = a_clamp((x - g.xoff) * g.dxi[0], g.nx), ymid = a_clamp((y - g.yoff) * g.dxi[1], g.ny);
    T acc = 0.0 * x;
#pragma unroll
    for (int iy = 0; iy < 3; ++iy) {
        const ASh<T> sy = a_shape2<T>(ymid, iy);
#pragma unroll
        for (int ix = 0; ix < 3; ++ix) {
            const ASh<T> sx = a_shape2<T>(xmid, ix);
            const int i = sx.cell, j = sy.cell;
            const T cd = q_invvol * sx.s * sy.s;
            acc = acc + cd * (vx * L.f[A_JX](i, j) + vy * L.f[A_JY](i, j) + qm * pi * L.f[A_CHI](i, j) + L.f[A_RM](i, j));
        }
    }
    return acc;
}

__global__ void __launch_bounds__(128) k_adj_deposit(AdjPlasma P, AdjLam lin, double* lw, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        const double in[5] = {P.x[ip], P.y[ip], P.ux[ip], P.uy[ip], P.psi[ip]};
        double d[5];
#pragma unroll 1
        for (int k = 0; k < 5; ++k) {
            Tn t[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) t[m] = tseed(in[m], m == k);
            d[k] = a_deposit_L<Tn>(L, g, P.charge, P.mass, P.w[ip], t[0], t[1], t[2], t[3], t[4]).d;
        }
        lin.x[ip] += d[0]; lin.y[ip] += d[1]; lin.ux[ip] += d[2]; lin.uy[ip] += d[3]; lin.psi[ip] += d[4];
        lw[ip] += a_deposit_L<double>(L, g, P.charge, P.mass, 1.0, in[0], in[1], in[2], in[3], in[4]);
    }
}

// beam deposits of store slice k (witness): lambda_w += q/V sum S (vz ljz + (1 - vz/c) lrm +
// vx ljx + vy ljy); null planes are skipped
__global__ void __launch_bounds__(256) k_adj_beam(BeamDev B, int par, int k, const double* ljz, const double* lrm,
                                                  const double* ljx, const double* ljy, int pitch, Geo g,
                                                  double* lw) {
    HPQ_PDL_ENTRY();
    const int start = B.start[par][k], cnt = B.count[par][k];
    const BeamBuf b = B.buf[par];
    const double invvol = g.normalized ? 1.0 : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double ci = 1.0 / g.c, ci2 = ci * ci;
    const F2<double> Fz{const_cast<double*>(ljz), pitch}, Fr{const_cast<double*>(lrm), pitch},
        Fx{const_cast<double*>(ljx), pitch}, Fy{const_cast<double*>(ljy), pitch};
    for (long long q = gtid(); q < cnt; q += gstride()) {
        const long long ip = start + q;
        if (!b.valid[ip]) continue;
        const double gaminv = 1.0 / sqrt(1.0 + b.ux[ip] * b.ux[ip] * ci2 + b.uy[ip] * b.uy[ip] * ci2 + b.uz[ip] * b.uz[ip] * ci2);
        const double vx = b.ux[ip] * gaminv, vy = b.uy[ip] * gaminv, vz = b.uz[ip] * gaminv;
        const double xmid = clamp_mid<double>((b.x[ip] - g.xoff) * g.dxi[0], g.nx);
        const double ymid = clamp_mid<double>((b.y[ip] - g.yoff) * g.dxi[1], g.ny);
        double acc = 0;
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const Sh<double> sy = shape2<double>(ymid, iy);
#pragma unroll
            for (int ix = 0; ix < 3; ++ix) {
                const Sh<double> sx = shape2<double>(xmid, ix);
                const int i = sx.cell, j = sy.cell;
                double l = 0;
                if (ljz) l += vz * Fz(i, j);
                if (lrm) l += (1.0 - vz * ci) * Fr(i, j);
                if (ljx) l += vx * Fx(i, j) + vy * Fy(i, j);
                acc += sx.s * sy.s * l;
            }
        }
        lw[ip] += B.charge * invvol * acc;
    }
}

}  // namespace hpq
