// SALAME beam loading (src/salame/Salame.cpp): kernels of the SALAME slice. The SALAME slice is
// a second set of slab components (component C_NCOMP + c of the slab), so every slab kernel runs
// on it through a Slab view whose base is offset by C_NCOMP planes; the extra planes of the
// reference's WhichSlice::Salame (Ez_target, Ez_no_salame, Sy_back, Sx_back) sit in components
// that the SALAME slice does not otherwise use.
#pragma once

#include "kernels.cuh"

namespace hpq {

// SALAME-slice components with no counterpart in the slice layout (Fields.cpp:117-128)
constexpr int kSalEzTarget = C_PSI;
constexpr int kSalEzNoSalame = C_BZ;
constexpr int kSalSyBack = C_EXMBY;
constexpr int kSalSxBack = C_EYPBX;

// Right-hand side of Fields::SolvePoissonEz (Fields.cpp:960-1005) from jx, jy of slab V into
// stage slot 0: (d_x jx + d_y jy) / (ep0 c), centred differences.
template <class R>
__global__ void k_sal_rhs_ez(Slab<R> V, Geo g, R* __restrict__ stage, int sj) {
    HPQ_PDL_ENTRY();
    const F2<R> jx = V.c(C_JX), jy = V.c(C_JY);
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]);
    const R fe = (R)(1. / (g.ep0 * g.c));
    for (long long k = gtid(); k < (long long)V.nx * V.ny; k += gstride()) {
        const int i = (int)(k % V.nx), j = (int)(k / V.nx);
        stage[(size_t)j * sj + i] = fe * ((jx(i + 1, j) - jx(i - 1, j)) * hx) + fe * ((jy(i, j + 1) - jy(i, j - 1)) * hy);
    }
}

// SalameInitializeSxSyWithBeam (Salame.cpp:189-220): Sy = mu0 (-d_y jz_beam),
// Sx = -mu0 (-d_x jz_beam) of the SALAME beam alone, interior cells.
template <class R>
__global__ void k_sal_sxsy(Slab<R> V, Geo g) {
    HPQ_PDL_ENTRY();
    const F2<R> jzb = V.c(C_JZB), Sx = V.c(C_SX), Sy = V.c(C_SY);
    const R hx = (R)(0.5 * g.dxi[0]), hy = (R)(0.5 * g.dxi[1]), mu0 = (R)g.mu0;
    for (long long k = gtid(); k < (long long)V.nx * V.ny; k += gstride()) {
        const int i = (int)(k % V.nx), j = (int)(k / V.nx);
        const R dx_jzb = (jzb(i + 1, j) - jzb(i - 1, j)) * hx;
        const R dy_jzb = (jzb(i, j + 1) - jzb(i, j - 1)) * hy;
        Sy(i, j) = mu0 * (-dy_jzb);
        Sx(i, j) = -mu0 * (-dx_jzb);
    }
}

// SalameGetJxJyFromBxBy (Salame.cpp:223-255): jx = 1.5 dz chi By / mu0, jy = -1.5 dz chi Bx / mu0
// with chi of this slice and Bx, By of the SALAME slice, interior cells.
template <class R>
__global__ void k_sal_jxjy_from_b(Slab<R> S, Slab<R> V, Geo g) {
    HPQ_PDL_ENTRY();
    const F2<R> chi = S.c(C_CHI), Bx = V.c(C_BX), By = V.c(C_BY), jx = V.c(C_JX), jy = V.c(C_JY);
    const R dz = (R)(1.5 * g.dx[2]), mu0_inv = (R)(1. / g.mu0);
    for (long long k = gtid(); k < (long long)V.nx * V.ny; k += gstride()) {
        const int i = (int)(k % V.nx), j = (int)(k / V.nx);
        jx(i, j) = dz * chi(i, j) * By(i, j) * mu0_inv;
        jy(i, j) = -dz * chi(i, j) * Bx(i, j) * mu0_inv;
    }
}

// SalameOnlyAdvancePlasma (Salame.cpp:257-331): the plasma momenta from the SALAME-only Bx, By
// gathered (deposit shape of order ORD, doBxByGatherShapeN, FieldGather.H:183-216) at the
// previous position: ux = 1.5 dz q/m By, uy = -1.5 dz q/m Bx.
template <class R, int ORD = 2>
__global__ void __launch_bounds__(256) k_sal_only_push(PlasmaDev<R> P, Slab<R> V, Geo g) {
    HPQ_PDL_ENTRY();
    const F2<R> FBx = V.c(C_BX), FBy = V.c(C_BY);
    const R f = (R)(1.5 * g.dx[2] * P.charge / P.mass);
    for (long long ip = gtid(); ip < P.n; ip += gstride()) {
        if (!P.valid[ip]) continue;
        int bx, by;
        const R xm = plasma_mid<R>(P.ru, ip, P.xp[ip], (R)g.xoff, (R)g.dxi[0], g.nx, bx);
        const R ym = plasma_mid<R>(P.rv, ip, P.yp[ip], (R)g.yoff, (R)g.dxi[1], g.ny, by);
        constexpr int NP = ORD + 1;
        Sh<R> sx[NP], sy[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            sx[q] = shapeN<R, ORD>(xm, q); sy[q] = shapeN<R, ORD>(ym, q);
            sx[q].cell += bx; sy[q].cell += by;
        }
        R bxp = 0, byp = 0;
#pragma unroll
        for (int iy = 0; iy < NP; ++iy)
#pragma unroll
            for (int ix = 0; ix < NP; ++ix) {
                const R s = sx[ix].s * sy[iy].s;
                bxp += s * FBx(sx[ix].cell, sy[iy].cell);
                byp += s * FBy(sx[ix].cell, sy[iy].cell);
            }
        P.ux[ip] = f * byp;
        P.uy[ip] = -f * bxp;
    }
}

// SalameGetW sums (Salame.cpp:334-388) over the interior cells in a fixed order (one block):
// out = {sum jz Ez_target, sum jz Ez_no_salame, sum jz Ez, sum jz} of the SALAME slice.
template <class R>
__global__ void __launch_bounds__(1024) k_sal_sums(Slab<R> V, double* __restrict__ out) {
    HPQ_PDL_ENTRY();
    __shared__ double red[4][32];
    const F2<R> jz = V.c(C_JZB), et = V.c(kSalEzTarget), eno = V.c(kSalEzNoSalame), ez = V.c(C_EZ);
    double a[4] = {0, 0, 0, 0};
    for (long long k = threadIdx.x; k < (long long)V.nx * V.ny; k += blockDim.x) {
        const int i = (int)(k % V.nx), j = (int)(k / V.nx);
        const double q = (double)jz(i, j);
        a[0] += q * (double)et(i, j);
        a[1] += q * (double)eno(i, j);
        a[2] += q * (double)ez(i, j);
        a[3] += q;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        for (int d = 16; d > 0; d >>= 1) a[c] += __shfl_xor_sync(0xffffffffu, a[c], d);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 4; ++c) red[c][warp] = a[c];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

// SalameMultiplyBeamWeight (Salame.cpp:403-437): the non-slipped particles of slice ctl->islice
// of a SALAME beam get w *= W, or are invalidated when W = 0.
__global__ void k_sal_weight(BeamDev B, const Ctl* __restrict__ ctl, double W) {
    HPQ_PDL_ENTRY();
    const int s = ctl->islice, par = ctl->step_parity;
    const int start = B.start[par][s], n = B.count[par][s];
    const BeamBuf b = B.buf[par];
    for (long long k = gtid(); k < n; k += gstride()) {
        const long long ip = start + k;
        if (!b.valid[ip]) continue;
        if (W == 0) { b.valid[ip] = 0; continue; }
        b.w[ip] *= W;
    }
}

// dst += src for component pairs of one slab (Fields::add, Fields.H:431-456), guards included
template <class R>
__global__ void k_add_comps(Slab<R> S, CopyList L) {
    HPQ_PDL_ENTRY();
    for (long long k = gtid(); k < (long long)S.cstride; k += gstride())
        for (int q = 0; q < L.n; ++q) S.base[(size_t)L.dst[q] * S.cstride + k] += S.base[(size_t)L.src[q] * S.cstride + k];
}

}  // namespace hpq
