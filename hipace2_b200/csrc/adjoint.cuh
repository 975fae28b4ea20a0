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
// (bit 0/1 of *reflected: x/y reflected)
template <class T>
__device__ __forceinline__ bool a_enforce_bc(const Geo& g, T& x, T& y, T& ux, T& uy, int* reflected = nullptr) {
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
        int r = 0;
        if (refl && val(x) > phi0) { x = 2 * phi0 - x; ux = -ux; r |= 1; }
        if (refl && val(y) > phi1) { y = 2 * phi1 - y; uy = -uy; r |= 2; }
        if (reflected) *reflected = r;
    }
    return true;
}

// plasma push of one particle (n_subcycles 1) with gathered fields G. out: x, y, ux_h, uy_h,
// psi_h, ux, uy, psi. Returns false if the particle is absorbed. Each sub-step is
//   u += h f(u) + h^2/2 (Df(u) f(u)),
// f the momentum right-hand side of k_plasma_push and Df f its derivative along the trajectory
// (the dual-number term of the forward, written out: the fields are constant along it).
template <class T>
__device__ __forceinline__ bool a_push(const Geo& g, double qmc, T x, T y, T ux, T uy, T psi, const T* G, T* out,
                                       int* reflected = nullptr) {
    const double ci = 1. / g.c, c2 = ci * ci, dzs = g.dx[2];
    const double sdz = dzs / 4, hh = 0.5 * sdz * sdz;
    auto substep = [&]() {
        const T pi = 1.0 / psi;
        const T a2 = 1.0 + (ux * ux + uy * uy) * c2;
        const T gp = 0.5 * pi * pi * a2 + 0.5;
        const T ue = ux * G[0] + uy * G[1];
        const T d0 = qmc * (gp * G[0] + G[4] + (uy * G[5]) * pi);
        const T d1 = qmc * (gp * G[1] - G[3] - (ux * G[5]) * pi);
        const T d2 = qmc * ci * (ue * ci * pi - G[2]);
        // derivatives along (d0, d1, d2): dpi = -pi^2 d2
        const T dpi = -(pi * pi) * d2;
        const T dgp = pi * dpi * a2 + pi * pi * c2 * (ux * d0 + uy * d1);
        const T e0 = qmc * (dgp * G[0] + G[5] * (d1 * pi + uy * dpi));
        const T e1 = qmc * (dgp * G[1] - G[5] * (d0 * pi + ux * dpi));
        const T e2 = qmc * c2 * ((d0 * G[0] + d1 * G[1]) * pi + ue * dpi);
        ux = ux + sdz * d0 + hh * e0;
        uy = uy + sdz * d1 + hh * e1;
        psi = psi + sdz * d2 + hh * e2;
    };
#pragma unroll 1
    for (int k = 0; k < 4; ++k) substep();
    x = x + dzs * ci * (ux * (1.0 / psi));
    y = y + dzs * ci * (uy * (1.0 / psi));
    if (reflected) *reflected = 0;
    if (!a_enforce_bc(g, x, y, ux, uy, reflected)) return false;
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

// record of a single-precision forward, widened to double for the reverse sweep: positions as
// the particle's lattice point plus its stored displacement, psi as 1 + the stored psi - 1, the
// field planes converted
struct AdjRecMixed {
    const float* pl[8];  // x, y, ux_h, uy_h, psi_h, ux, uy, psi (displacements, psi - 1)
    const float* ru;
    const float* rv;
    double xoff, yoff, dx, dy;
    double* dst[8];
    const float* f[RF_N];
    double* fdst[RF_N];
    long long n, cs;
    const uint8_t* vsrc;
    uint8_t* vdst;
    int nz, K;
};
__global__ void k_adj_record_mixed(const Ctl* __restrict__ ctl, AdjRecMixed a) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice;
    const int c = (a.nz - 1 - s) / a.K;
    const int hi = a.nz - 1 - c * a.K;
    const int lo = hi - a.K + 1 > 0 ? hi - a.K + 1 : 0;
    const long long slot = s - lo;
    for (long long i = gtid(); i < a.n; i += gstride()) {
        const size_t o = slot * a.n + i;
        a.dst[0][o] = a.xoff + (double)a.ru[i] * a.dx + (double)a.pl[0][i];
        a.dst[1][o] = a.yoff + (double)a.rv[i] * a.dy + (double)a.pl[1][i];
        a.dst[2][o] = (double)a.pl[2][i];
        a.dst[3][o] = (double)a.pl[3][i];
        a.dst[4][o] = 1.0 + (double)a.pl[4][i];
        a.dst[5][o] = (double)a.pl[5][i];
        a.dst[6][o] = (double)a.pl[6][i];
        a.dst[7][o] = 1.0 + (double)a.pl[7][i];
        a.vdst[o] = a.vsrc[i];
    }
    for (int k = 0; k < RF_N; ++k)
        for (long long i = gtid(); i < a.cs; i += gstride()) a.fdst[k][slot * a.cs + i] = (double)a.f[k][i];
}
// dst = src in double
template <class R>
__global__ void k_adj_widen(const R* __restrict__ src, double* __restrict__ dst, long long n) {
    HPQ_PDL_ENTRY();
    for (long long i = gtid(); i < n; i += gstride()) dst[i] = (double)src[i];
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
template <class R>
__global__ void __launch_bounds__(1024) k_adj_plane_dot(F2<double> a, F2<R> b, int nx, int ny, double* out) {
    HPQ_PDL_ENTRY();
    double s[1] = {0};
    for (long long k = threadIdx.x; k < (long long)nx * ny; k += blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        s[0] += a(i, j) * (double)b(i, j);
    }
    block_sum_store<1>(s, out);
}

// ------------------------------------------------------------------------------------------
// Reverse sweep kernels (one slice)
// ------------------------------------------------------------------------------------------
struct AdjL {
    F2<double> f[A_NCOMP];
};

// plasma push: lin += J^T lout for (x, y, ux_h, uy_h, psi_h) (lin zeroed before); field
// adjoints scattered by the gather shapes. One thread per (particle, seed): seeds 0-2
// differentiate the push with respect to ux_h, uy_h, psi_h, seeds 3-8 with respect to the six
// gathered values G. The positions enter the push only through G and the position update
// x' = x + dz ux/(c psi) (+-1 under a reflection), so dL/dx = sum_c dL/dG_c dG_c/dx + lout_x' (+-1):
// the thread of G_c adds its term (gather shapes differentiated in x and y) and deposits dL/dG_c
// on the plane of G_c (the adjoint of a gather is a deposit).
constexpr int kPushSeeds = 9;
__global__ void __launch_bounds__(256) k_adj_push(AdjPlasma P, AdjLam lout, AdjLam lin, AdjRecF F, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    const double qmc = P.charge / (P.mass * g.c);
    const long long total = P.n * kPushSeeds;
    for (long long t = gtid(); t < total; t += gstride()) {
        const long long ip = t / kPushSeeds;
        const int k = (int)(t - ip * kPushSeeds);
        const double lo[8] = {lout.x[ip], lout.y[ip], lout.uxh[ip], lout.uyh[ip], lout.psih[ip],
                              lout.ux[ip], lout.uy[ip], lout.psi[ip]};
        bool any = false;
#pragma unroll
        for (int o = 0; o < 8; ++o) any = any || lo[o] != 0.0;
        if (!P.valid[ip] || !any) continue;
        const double in[5] = {P.x[ip], P.y[ip], P.uxh[ip], P.uyh[ip], P.psih[ip]};
        double Gv[6];
        a_gather<double>(F, g, in[0], in[1], Gv);
        Tn G[6], out[8];
#pragma unroll
        for (int m = 0; m < 6; ++m) G[m] = tseed(Gv[m], m == k - 3);
        int refl = 0;
        const bool alive = a_push<Tn>(g, qmc, tseed(in[0], false), tseed(in[1], false), tseed(in[2], k == 0),
                                      tseed(in[3], k == 1), tseed(in[4], k == 2), G, out, &refl);
        if (!alive) continue;
        double sum = 0;
#pragma unroll
        for (int o = 0; o < 8; ++o) sum += lo[o] * out[o].d;
        if (k < 3) {
            double* const lk = k == 0 ? lin.uxh : k == 1 ? lin.uyh : lin.psih;
            lk[ip] += sum;
            if (k == 0) {
                atomicAdd(lin.x + ip, (refl & 1) ? -lo[0] : lo[0]);
                atomicAdd(lin.y + ip, (refl & 2) ? -lo[1] : lo[1]);
            }
            continue;
        }
        if (sum == 0.0) continue;
        const int c = k - 3;
        const F2<double> dstp = L.f[c <= 1 ? A_PSI : c == 2 ? A_EZ : c == 3 ? A_BX : c == 4 ? A_BY : A_BZ];
        const F2<double> src = F.f[c <= 1 ? RF_PSI : c == 2 ? RF_EZ : c == 3 ? RF_BX : c == 4 ? RF_BY : RF_BZ];
        const double fac = (c == 3 || c == 4) ? g.c : 1.0;
        const double dxi = g.dxi[0], dyi = g.dxi[1];
        // cell coordinates with their derivatives d/dx (x pass) and d/dy (y pass)
        const Tn xm = a_clamp((tseed(in[0], true) - g.xoff) * dxi, g.nx);
        const Tn ym = a_clamp((tseed(in[1], true) - g.yoff) * dyi, g.ny);
        double gx = 0, gy = 0;
#pragma unroll 1
        for (int iy = 0; iy < 4; iy++) {
            const ADSh<Tn> sy = a_dshape2<Tn>(1, ym, iy);
#pragma unroll
            for (int ix = 0; ix < 4; ix++) {
                const ADSh<Tn> sx = a_dshape2<Tn>(1, xm, ix);
                const int i = sx.cell, j = sy.cell;
                double w, wx, wy;
                if (c == 0) { w = sx.ds.v * sy.s.v * dxi; wx = sx.ds.d * sy.s.v * dxi; wy = sx.ds.v * sy.s.d * dxi; }
                else if (c == 1) { w = sx.s.v * sy.ds.v * dyi; wx = sx.s.d * sy.ds.v * dyi; wy = sx.s.v * sy.ds.d * dyi; }
                else { w = sx.s.v * sy.s.v; wx = sx.s.d * sy.s.v; wy = sx.s.v * sy.s.d; }
                const double f = src(i, j);
                gx += wx * f;
                gy += wy * f;
                atomicAdd(dstp.ptr(i, j), sum * fac * w);
            }
        }
        atomicAdd(lin.x + ip, sum * fac * gx);
        atomicAdd(lin.y + ip, sum * fac * gy);
    }
}

// The same map in reverse mode, one thread per particle: the forward push in double keeping the
// state entering each of the 6 sub-steps, then the adjoint of each sub-step in reverse order
// (a_substep_rev: the sub-step's expressions differentiated by hand, last operation first), of the
// boundary condition (a reflection flips x and u) and of the position update. All nine input
// adjoints (u_h, and the six gathered values) come out of one pass, where the forward-mode form
// re-runs the push nine times. Same results as k_adj_push up to the order of the sums.
struct SubstepC {
    double qmc, ci, c2, sdz, hh;
};
__device__ __forceinline__ void a_substep_fwd(const SubstepC& k, const double* G, double& ux, double& uy,
                                              double& psi) {
    const double pi = 1.0 / psi;
    const double a2 = 1.0 + (ux * ux + uy * uy) * k.c2;
    const double gp = 0.5 * pi * pi * a2 + 0.5;
    const double ue = ux * G[0] + uy * G[1];
    const double d0 = k.qmc * (gp * G[0] + G[4] + (uy * G[5]) * pi);
    const double d1 = k.qmc * (gp * G[1] - G[3] - (ux * G[5]) * pi);
    const double d2 = k.qmc * k.ci * (ue * k.ci * pi - G[2]);
    const double dpi = -(pi * pi) * d2;
    const double dgp = pi * dpi * a2 + pi * pi * k.c2 * (ux * d0 + uy * d1);
    const double e0 = k.qmc * (dgp * G[0] + G[5] * (d1 * pi + uy * dpi));
    const double e1 = k.qmc * (dgp * G[1] - G[5] * (d0 * pi + ux * dpi));
    const double e2 = k.qmc * k.c2 * ((d0 * G[0] + d1 * G[1]) * pi + ue * dpi);
    ux = ux + k.sdz * d0 + k.hh * e0;
    uy = uy + k.sdz * d1 + k.hh * e1;
    psi = psi + k.sdz * d2 + k.hh * e2;
}
// (ux, uy, psi): the state entering the sub-step; (lux, luy, lpsi): the adjoint of the state
// after it on entry, of the state before it on exit; lG accumulates the field adjoints
__device__ __forceinline__ void a_substep_rev(const SubstepC& k, const double* G, double ux, double uy, double psi,
                                              double& lux, double& luy, double& lpsi, double* lG) {
    const double pi = 1.0 / psi;
    const double a2 = 1.0 + (ux * ux + uy * uy) * k.c2;
    const double gp = 0.5 * pi * pi * a2 + 0.5;
    const double ue = ux * G[0] + uy * G[1];
    const double d0 = k.qmc * (gp * G[0] + G[4] + (uy * G[5]) * pi);
    const double d1 = k.qmc * (gp * G[1] - G[3] - (ux * G[5]) * pi);
    const double d2 = k.qmc * k.ci * (ue * k.ci * pi - G[2]);
    const double dpi = -(pi * pi) * d2;
    const double dgp = pi * dpi * a2 + pi * pi * k.c2 * (ux * d0 + uy * d1);
    // u' = u + sdz d + hh e
    double ld0 = k.sdz * lux, ld1 = k.sdz * luy, ld2 = k.sdz * lpsi;
    const double le0 = k.hh * lux, le1 = k.hh * luy, le2 = k.hh * lpsi;
    double lpi = 0, lue = 0, ldpi = 0, ldgp = 0, lgp = 0, la2 = 0;
    // e2 = qmc c2 ((d0 G0 + d1 G1) pi + ue dpi)
    const double k2 = k.qmc * k.c2 * le2;
    ld0 += k2 * G[0] * pi; lG[0] += k2 * d0 * pi;
    ld1 += k2 * G[1] * pi; lG[1] += k2 * d1 * pi;
    lpi += k2 * (d0 * G[0] + d1 * G[1]); lue += k2 * dpi; ldpi += k2 * ue;
    // e1 = qmc (dgp G1 - G5 (d0 pi + ux dpi))
    const double k1 = k.qmc * le1;
    ldgp += k1 * G[1]; lG[1] += k1 * dgp; lG[5] -= k1 * (d0 * pi + ux * dpi);
    ld0 -= k1 * G[5] * pi; lpi -= k1 * G[5] * d0; lux -= k1 * G[5] * dpi; ldpi -= k1 * G[5] * ux;
    // e0 = qmc (dgp G0 + G5 (d1 pi + uy dpi))
    const double k0 = k.qmc * le0;
    ldgp += k0 * G[0]; lG[0] += k0 * dgp; lG[5] += k0 * (d1 * pi + uy * dpi);
    ld1 += k0 * G[5] * pi; lpi += k0 * G[5] * d1; luy += k0 * G[5] * dpi; ldpi += k0 * G[5] * uy;
    // dgp = pi dpi a2 + pi^2 c2 (ux d0 + uy d1)
    const double pp = pi * pi * k.c2;
    lpi += ldgp * (dpi * a2 + 2.0 * pi * k.c2 * (ux * d0 + uy * d1));
    ldpi += ldgp * pi * a2; la2 += ldgp * pi * dpi;
    lux += ldgp * pp * d0; ld0 += ldgp * pp * ux;
    luy += ldgp * pp * d1; ld1 += ldgp * pp * uy;
    // dpi = -pi^2 d2
    lpi -= ldpi * 2.0 * pi * d2; ld2 -= ldpi * pi * pi;
    // d2 = qmc ci (ue ci pi - G2)
    const double kd2 = k.qmc * k.ci * ld2;
    lue += kd2 * k.ci * pi; lpi += kd2 * ue * k.ci; lG[2] -= kd2;
    // d1 = qmc (gp G1 - G3 - ux G5 pi)
    const double kd1 = k.qmc * ld1;
    lgp += kd1 * G[1]; lG[1] += kd1 * gp; lG[3] -= kd1;
    lux -= kd1 * G[5] * pi; lG[5] -= kd1 * ux * pi; lpi -= kd1 * ux * G[5];
    // d0 = qmc (gp G0 + G4 + uy G5 pi)
    const double kd0 = k.qmc * ld0;
    lgp += kd0 * G[0]; lG[0] += kd0 * gp; lG[4] += kd0;
    luy += kd0 * G[5] * pi; lG[5] += kd0 * uy * pi; lpi += kd0 * uy * G[5];
    // ue = ux G0 + uy G1; gp = pi^2 a2 / 2 + 1/2; a2 = 1 + (ux^2 + uy^2) c2; pi = 1/psi
    lux += lue * G[0]; lG[0] += lue * ux; luy += lue * G[1]; lG[1] += lue * uy;
    lpi += lgp * pi * a2; la2 += lgp * 0.5 * pi * pi;
    lux += la2 * 2.0 * ux * k.c2; luy += la2 * 2.0 * uy * k.c2;
    lpsi -= lpi * pi * pi;
}

__global__ void __launch_bounds__(256) k_adj_push_rev(AdjPlasma P, AdjLam lout, AdjLam lin, AdjRecF F, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    SubstepC k;
    k.qmc = P.charge / (P.mass * g.c);
    k.ci = 1. / g.c;
    k.c2 = k.ci * k.ci;
    const double dzs = g.dx[2];
    k.sdz = dzs / 4;
    k.hh = 0.5 * k.sdz * k.sdz;
    const double dxi = g.dxi[0], dyi = g.dxi[1];
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        const double lo[8] = {lout.x[ip], lout.y[ip], lout.uxh[ip], lout.uyh[ip], lout.psih[ip],
                              lout.ux[ip], lout.uy[ip], lout.psi[ip]};
        bool any = false;
#pragma unroll
        for (int o = 0; o < 8; ++o) any = any || lo[o] != 0.0;
        if (!P.valid[ip] || !any) continue;
        const double x0 = P.x[ip], y0 = P.y[ip];
        double G[6];
        a_gather<double>(F, g, x0, y0, G);
        // forward, keeping the state entering each sub-step
        double su[6], sv[6], sp[6];
        double ux = P.uxh[ip], uy = P.uyh[ip], psi = P.psih[ip];
#pragma unroll
        for (int q = 0; q < 4; ++q) { su[q] = ux; sv[q] = uy; sp[q] = psi; a_substep_fwd(k, G, ux, uy, psi); }
        const double ux4 = ux, uy4 = uy, psi4 = psi;
        double x = x0 + dzs * k.ci * (ux * (1.0 / psi));
        double y = y0 + dzs * k.ci * (uy * (1.0 / psi));
        int refl = 0;
        if (!a_enforce_bc<double>(g, x, y, ux, uy, &refl)) continue;
#pragma unroll
        for (int q = 4; q < 6; ++q) { su[q] = ux; sv[q] = uy; sp[q] = psi; a_substep_fwd(k, G, ux, uy, psi); }
        // reverse
        double lux = lo[5], luy = lo[6], lpsi = lo[7];
        double lG[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 5; q >= 4; --q) a_substep_rev(k, G, su[q], sv[q], sp[q], lux, luy, lpsi, lG);
        lux += lo[2]; luy += lo[3]; lpsi += lo[4];
        double lx = lo[0], ly = lo[1];
        if (refl & 1) { lx = -lx; lux = -lux; }
        if (refl & 2) { ly = -ly; luy = -luy; }
        // x' = x + dz ux / (c psi), y' likewise, at the state after 4 sub-steps
        const double pinv = 1.0 / psi4, f = dzs * k.ci;
        lux += lx * f * pinv;
        luy += ly * f * pinv;
        lpsi -= (lx * ux4 + ly * uy4) * f * pinv * pinv;
#pragma unroll
        for (int q = 3; q >= 0; --q) a_substep_rev(k, G, su[q], sv[q], sp[q], lux, luy, lpsi, lG);
        lin.uxh[ip] += lux;
        lin.uyh[ip] += luy;
        lin.psih[ip] += lpsi;
        // field adjoints by the gather shapes, and the positions' share through the gathered values
        lG[3] *= g.c;
        lG[4] *= g.c;
        const Tn xm = a_clamp((tseed(x0, true) - g.xoff) * dxi, g.nx);
        const Tn ym = a_clamp((tseed(y0, true) - g.yoff) * dyi, g.ny);
        double gx = 0, gy = 0;
#pragma unroll 1
        for (int iy = 0; iy < 4; iy++) {
            const ADSh<Tn> sy = a_dshape2<Tn>(1, ym, iy);
#pragma unroll
            for (int ix = 0; ix < 4; ix++) {
                const ADSh<Tn> sx = a_dshape2<Tn>(1, xm, ix);
                const int i = sx.cell, j = sy.cell;
                const double w = sx.s.v * sy.s.v, wx = sx.s.d * sy.s.v, wy = sx.s.v * sy.s.d;
                // Psi through ExmBy (x derivative shape) and EypBx (y derivative shape)
                const double wp = lG[0] * sx.ds.v * sy.s.v * dxi + lG[1] * sx.s.v * sy.ds.v * dyi;
                const double wpx = lG[0] * sx.ds.d * sy.s.v * dxi + lG[1] * sx.s.d * sy.ds.v * dyi;
                const double wpy = lG[0] * sx.ds.v * sy.s.d * dxi + lG[1] * sx.s.v * sy.ds.d * dyi;
                const double fpsi = F.f[RF_PSI](i, j), fez = F.f[RF_EZ](i, j), fbx = F.f[RF_BX](i, j),
                             fby = F.f[RF_BY](i, j), fbz = F.f[RF_BZ](i, j);
                gx += wpx * fpsi + wx * (lG[2] * fez + lG[3] * fbx + lG[4] * fby + lG[5] * fbz);
                gy += wpy * fpsi + wy * (lG[2] * fez + lG[3] * fbx + lG[4] * fby + lG[5] * fbz);
                if (wp != 0.0) atomicAdd(L.f[A_PSI].ptr(i, j), wp);
                if (lG[2] != 0.0) atomicAdd(L.f[A_EZ].ptr(i, j), lG[2] * w);
                if (lG[3] != 0.0) atomicAdd(L.f[A_BX].ptr(i, j), lG[3] * w);
                if (lG[4] != 0.0) atomicAdd(L.f[A_BY].ptr(i, j), lG[4] * w);
                if (lG[5] != 0.0) atomicAdd(L.f[A_BZ].ptr(i, j), lG[5] * w);
            }
        }
        lin.x[ip] += lx + gx;
        lin.y[ip] += ly + gy;
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

// multigrid slab for the transposed solve: chi, rhs = W^-1 lambda_B (interior), zero initial guess (the
// previous slice's solution is a worse start: lambda_B changes its pattern from slice to slice)
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

// explicit Sx/Sy deposit. With a = lambda_Sx, b = lambda_Sy, S = sx sy, Dx = sx' sy, Dy = sx sy'
// (shape and derivative shape) and the node fields, the particle's contribution to the adjoint
// objective is cdm * Phi with
//   Phi = qm pi [vy m1 + ci vx m2 + ci (gp - vx^2) m3 - ci vx vy m4 + vx m5 - ci vy m6
//                + ci vx vy m7 - ci (gp - vy^2) m8]
//       + c [dxi (gp - vx^2 - 1) d1 + dxi vx vy d2 - dyi vx vy d3 - dyi (gp - vy^2 - 1) d4],
//   m1..m4 = sum S a (Bz, Ez, ExmBy, EypBx), m5..m8 = sum S b (...), d1 = sum Dx a, d2 = sum Dx b,
//   d3 = sum Dy a, d4 = sum Dy b
// (the expression of k_explicit_deposit regrouped). Phi is linear in the 12 stencil moments, so
// dPhi/dx is Phi of the moments' x-derivatives (one pass with the shapes differentiated in x),
// likewise y; the velocity variables enter Phi only through (pi, vx, vy, gp).
template <class V, class M>
__device__ __forceinline__ V a_explicit_phi(const Geo& g, double qm, V pi, V vx, V vy, V gp, const M* m) {
    const double ci = 1. / g.c, dxi = g.dxi[0], dyi = g.dxi[1];
    return qm * pi * (vy * m[0] + ci * vx * m[1] + ci * (gp - vx * vx) * m[2] - ci * vx * vy * m[3] + vx * m[4] -
                      ci * vy * m[5] + ci * vx * vy * m[6] - ci * (gp - vy * vy) * m[7]) +
           g.c * (dxi * (gp - vx * vx - 1.0) * m[8] + dxi * vx * vy * m[9] - dyi * vx * vy * m[10] -
                  dyi * (gp - vy * vy - 1.0) * m[11]);
}
template <int DT>
__device__ __forceinline__ void a_explicit_moments(const AdjRecF& F, const AdjL& L, const Geo& g, Tn xm, Tn ym,
                                                   Tn* m) {
#pragma unroll
    for (int q = 0; q < 12; ++q) m[q] = Tn{0.0, 0.0};
    constexpr int NS = 3 + DT;
#pragma unroll 1
    for (int iy = 0; iy < NS; ++iy) {
        const ADSh<Tn> sy = a_dshape2<Tn>(DT, ym, iy);
#pragma unroll 1
        for (int ix = 0; ix < NS; ++ix) {
            if (DT == 2 && (ix == 0 || ix == 4) && (iy == 0 || iy == 4)) continue;
            const ADSh<Tn> sx = a_dshape2<Tn>(DT, xm, ix);
            const int i = sx.cell, j = sy.cell;
            const double a = L.f[A_SX](i, j), b = L.f[A_SY](i, j);
            if (a == 0.0 && b == 0.0) continue;
            const Tn S = sx.s * sy.s, Dx = sx.ds * sy.s, Dy = sx.s * sy.ds;
            const double Bz = F.f[RF_BZ](i, j), Ez = F.f[RF_EZ](i, j), Ex = F.f[RF_EXMBY](i, j), Ey = F.f[RF_EYPBX](i, j);
            const Tn Sa = S * a, Sb = S * b;
            m[0] = m[0] + Sa * Bz; m[1] = m[1] + Sa * Ez; m[2] = m[2] + Sa * Ex; m[3] = m[3] + Sa * Ey;
            m[4] = m[4] + Sb * Bz; m[5] = m[5] + Sb * Ez; m[6] = m[6] + Sb * Ex; m[7] = m[7] + Sb * Ey;
            m[8] = m[8] + Dx * a; m[9] = m[9] + Dx * b; m[10] = m[10] + Dy * a; m[11] = m[11] + Dy * b;
        }
    }
}

template <int DT>
__global__ void __launch_bounds__(256) k_adj_explicit(AdjPlasma P, AdjLam lin, double* lw, AdjRecF F, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    const double invvol = g.normalized ? g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1] : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double ci = 1. / g.c, dxi = g.dxi[0], dyi = g.dxi[1];
    const double cdm1 = P.charge * invvol * g.mu0;  // cdm per unit weight
    const double qm = P.charge / P.mass;
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        const double x = P.x[ip], y = P.y[ip], ux = P.ux[ip], uy = P.uy[ip], psi = P.psi[ip], w = P.w[ip];
        const double cdm = cdm1 * w;
        Tn mx[12], my[12];
        a_explicit_moments<DT>(F, L, g, a_clamp((tseed(x, true) - g.xoff) * dxi, g.nx),
                               a_clamp((tseed(y, false) - g.yoff) * dyi, g.ny), mx);
        a_explicit_moments<DT>(F, L, g, a_clamp((tseed(x, false) - g.xoff) * dxi, g.nx),
                               a_clamp((tseed(y, true) - g.yoff) * dyi, g.ny), my);
        double mv[12], mdx[12], mdy[12];
#pragma unroll
        for (int q = 0; q < 12; ++q) { mv[q] = mx[q].v; mdx[q] = mx[q].d; mdy[q] = my[q].d; }
        const double pi = 1.0 / psi, vx = ux * pi * ci, vy = uy * pi * ci;
        const double gp = 0.5 * (pi * pi + vx * vx + vy * vy + 1.0);
        lin.x[ip] += cdm * a_explicit_phi<double, double>(g, qm, pi, vx, vy, gp, mdx);
        lin.y[ip] += cdm * a_explicit_phi<double, double>(g, qm, pi, vx, vy, gp, mdy);
        double dv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const Tn tux = tseed(ux, k == 0), tuy = tseed(uy, k == 1), tps = tseed(psi, k == 2);
            const Tn tpi = 1.0 / tps, tvx = tux * tpi * ci, tvy = tuy * tpi * ci;
            const Tn tgp = 0.5 * (tpi * tpi + tvx * tvx + tvy * tvy + 1.0);
            dv[k] = a_explicit_phi<Tn, double>(g, qm, tpi, tvx, tvy, tgp, mv).d;
        }
        lin.ux[ip] += cdm * dv[0];
        lin.uy[ip] += cdm * dv[1];
        lin.psi[ip] += cdm * dv[2];
        lw[ip] += cdm1 * a_explicit_phi<double, double>(g, qm, pi, vx, vy, gp, mv);
        // field adjoints (closed form per node)
        const double xm = a_clamp((x - g.xoff) * dxi, g.nx), ym = a_clamp((y - g.yoff) * dyi, g.ny);
        constexpr int NS = 3 + DT;
#pragma unroll 1
        for (int iy = 0; iy < NS; ++iy) {
            const ADSh<double> sy = a_dshape2<double>(DT, ym, iy);
#pragma unroll 1
            for (int ix = 0; ix < NS; ++ix) {
                if (DT == 2 && (ix == 0 || ix == 4) && (iy == 0 || iy == 4)) continue;
                const ADSh<double> sx = a_dshape2<double>(DT, xm, ix);
                const int i = sx.cell, j = sy.cell;
                const double lsx = L.f[A_SX](i, j), lsy = L.f[A_SY](i, j);
                if (lsx == 0.0 && lsy == 0.0) continue;
                const double K = sx.s * sy.s * pi * cdm * qm;
                atomicAdd(L.f[A_BZ].ptr(i, j), lsy * K * vx + lsx * K * vy);
                atomicAdd(L.f[A_EZ].ptr(i, j), -lsy * K * vy * ci + lsx * K * vx * ci);
                atomicAdd(L.f[A_EXMBY].ptr(i, j), lsy * K * vx * vy * ci + lsx * K * (gp - vx * vx) * ci);
                atomicAdd(L.f[A_EYPBX].ptr(i, j), -lsy * K * (gp - vy * vy) * ci - lsx * K * vx * vy * ci);
            }
        }
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

// plasma deposit (jx, jy, chi, rho - jz). The particle's contribution to the adjoint objective is
// q_invvol * (vx m0 + vy m1 + qm pi m2 + m3) with vx = ux pi, vy = uy pi, pi = 1/psi and the
// moments m = sum S (lambda_jx, lambda_jy, lambda_chi, lambda_rhomjz) over the 3x3 stencil;
// x and y derivatives from the moments of the differentiated shapes.
__device__ __forceinline__ void a_deposit_moments(const AdjL& L, Tn xm, Tn ym, Tn* m) {
#pragma unroll
    for (int q = 0; q < 4; ++q) m[q] = Tn{0.0, 0.0};
#pragma unroll
    for (int iy = 0; iy < 3; ++iy) {
        const ASh<Tn> sy = a_shape2<Tn>(ym, iy);
#pragma unroll
        for (int ix = 0; ix < 3; ++ix) {
            const ASh<Tn> sx = a_shape2<Tn>(xm, ix);
            const int i = sx.cell, j = sy.cell;
            const Tn S = sx.s * sy.s;
            m[0] = m[0] + S * L.f[A_JX](i, j);
            m[1] = m[1] + S * L.f[A_JY](i, j);
            m[2] = m[2] + S * L.f[A_CHI](i, j);
            m[3] = m[3] + S * L.f[A_RM](i, j);
        }
    }
}
template <class V, class M>
__device__ __forceinline__ V a_deposit_phi(double qm, V ux, V uy, V psi, const M* m) {
    const V pi = 1.0 / psi;
    return ux * pi * m[0] + uy * pi * m[1] + qm * pi * m[2] + m[3];
}

__global__ void __launch_bounds__(256) k_adj_deposit(AdjPlasma P, AdjLam lin, double* lw, AdjL L, Geo g) {
    HPQ_PDL_ENTRY();
    const double invvol = g.normalized ? g.dx[0] * g.dx[1] * g.dxi[0] * g.dxi[1] : g.dxi[0] * g.dxi[1] * g.dxi[2];
    const double q1 = P.charge * invvol;  // q_invvol per unit weight
    const double qm = P.charge * g.mu0 / P.mass;
    const double dxi = g.dxi[0], dyi = g.dxi[1];
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        const double x = P.x[ip], y = P.y[ip], ux = P.ux[ip], uy = P.uy[ip], psi = P.psi[ip];
        const double qw = q1 * P.w[ip];
        Tn mx[4], my[4];
        a_deposit_moments(L, a_clamp((tseed(x, true) - g.xoff) * dxi, g.nx), a_clamp((tseed(y, false) - g.yoff) * dyi, g.ny), mx);
        a_deposit_moments(L, a_clamp((tseed(x, false) - g.xoff) * dxi, g.nx), a_clamp((tseed(y, true) - g.yoff) * dyi, g.ny), my);
        double mv[4], mdx[4], mdy[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) { mv[q] = mx[q].v; mdx[q] = mx[q].d; mdy[q] = my[q].d; }
        lin.x[ip] += qw * a_deposit_phi<double, double>(qm, ux, uy, psi, mdx);
        lin.y[ip] += qw * a_deposit_phi<double, double>(qm, ux, uy, psi, mdy);
        lin.ux[ip] += qw * a_deposit_phi<Tn, double>(qm, tseed(ux, true), tseed(uy, false), tseed(psi, false), mv).d;
        lin.uy[ip] += qw * a_deposit_phi<Tn, double>(qm, tseed(ux, false), tseed(uy, true), tseed(psi, false), mv).d;
        lin.psi[ip] += qw * a_deposit_phi<Tn, double>(qm, tseed(ux, false), tseed(uy, false), tseed(psi, true), mv).d;
        lw[ip] += q1 * a_deposit_phi<double, double>(qm, ux, uy, psi, mv);
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
