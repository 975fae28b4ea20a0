// ORACLE — test infrastructure only. Not part of the product and never linked into it.
//
// A plain FP64 CPU restatement of HiPACE++'s quasi-static slice loop (explicit and
// predictor-corrector Bx/By solvers, Dirichlet fields, transverse shape order 2), used by the
// tests to check the CUDA implementation and by bench.py as the timed CPU baseline.
// Each routine cites the reference file:line it restates. Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this library.
//
// The reference itself (AMReX + FFTW + MPI) cannot be built here; parity of this oracle is
// pinned instead against the reference's own checksum goldens
// (tests/checksum/benchmarks_json/*.json), see tests/test_oracle_golden.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../hipace2_b200/csrc/config.hpp"
#include "../hipace2_b200/csrc/rng.hpp"

using hpq::SimConfig;

namespace oracle {

// ------------------------------------------------------------------------------------------
// Shape factors (ShapeFactors.H:122-171 order 2, :212-468 derivative shapes)
// ------------------------------------------------------------------------------------------
struct Shape { double s; int cell; };
struct DShape { double s, ds; int cell; };

static inline Shape shape2(double xmid, int ix) {
    const double xfloor = std::floor(xmid + 0.5);
    const double xint = xmid - xfloor;
    if (ix == 0) return {0.5 * (0.5 - xint) * (0.5 - xint), (int)xfloor - 1};
    if (ix == 1) return {0.75 - xint * xint, (int)xfloor};
    return {0.5 * (0.5 + xint) * (0.5 + xint), (int)xfloor + 1};
}

// derivative shapes for order 2; returns {s_x, -sdx, cell} like the reference
static inline DShape dshape2(int type, double xmid, int ix) {
    if (type == 0) {
        xmid += 0.5;
        const double xfloor = std::floor(xmid);
        const double xint = xmid - xfloor, x2 = xint * xint;
        if (ix == 0) return {0.5 * x2 - 1.0 * xint + 0.5, -(xint - 1.0), (int)xfloor - 1 + ix};
        if (ix == 1) return {-x2 + 1.0 * xint + 0.5, -(1.0 - 2 * xint), (int)xfloor - 1 + ix};
        return {0.5 * x2, -xint, (int)xfloor - 1 + ix};
    } else if (type == 1) {
        const double xfloor = std::floor(xmid);
        const double xint = xmid - xfloor, x2 = xint * xint;
        const bool lo = xint < 0.5;
        if (ix == 0) return {lo ? 0.5 * x2 - 0.5 * xint + 1.0 / 8.0 : 0,
                             -(-0.5 * x2 + xint - 0.5), (int)xfloor - 1 + ix};
        if (ix == 1) return {lo ? 3.0 / 4.0 - x2 : 0.5 * x2 - 1.5 * xint + 9.0 / 8.0,
                             -(1.5 * x2 - 2 * xint), (int)xfloor - 1 + ix};
        if (ix == 2) return {lo ? 0.5 * x2 + 0.5 * xint + 1.0 / 8.0 : -x2 + 2 * xint - 1.0 / 4.0,
                             -(-1.5 * x2 + xint + 0.5), (int)xfloor - 1 + ix};
        return {lo ? 0 : 0.5 * x2 - 0.5 * xint + 1.0 / 8.0, -(0.5 * x2), (int)xfloor - 1 + ix};
    } else {
        xmid += 0.5;
        const double xfloor = std::floor(xmid);
        const double xint = xmid - xfloor, x2 = xint * xint;
        if (ix == 0) return {0, -(-0.25 * x2 + 0.5 * xint - 0.25), (int)xfloor - 2 + ix};
        if (ix == 1) return {0.5 * x2 - xint + 0.5, -(0.5 * x2 - 0.5 * xint - 0.25), (int)xfloor - 2 + ix};
        if (ix == 2) return {-x2 + xint + 0.5, -(0.25 - 0.5 * xint), (int)xfloor - 2 + ix};
        if (ix == 3) return {0.5 * x2, -(-0.5 * x2 + 0.5 * xint + 0.25), (int)xfloor - 2 + ix};
        return {0, -(0.25 * x2), (int)xfloor - 2 + ix};
    }
}

// Orders 0..3 (ShapeFactors.H:130-197 compute_single_shape_factor, :212-468
// single_derivative_shape_factor): B-splines of order 0, 1, 3 and their analytic (type 0), nodal
// (1) and centred (2) derivative forms; order 2 is shape2 / dshape2 above.
static inline Shape shapeN(int ord, double xmid, int ix) {
    if (ord == 2) return shape2(xmid, ix);
    if (ord == 0) return {1.0, (int)std::floor(xmid + 0.5)};
    const double xfloor = std::floor(xmid), xint = xmid - xfloor;
    if (ord == 1) return {ix == 0 ? 1.0 - xint : xint, (int)xfloor + ix};
    const int c = (int)xfloor - 1 + ix;
    if (ix == 0) return {1.0 / 6.0 * (1.0 - xint) * (1.0 - xint) * (1.0 - xint), c};
    if (ix == 1) return {2.0 / 3.0 - xint * xint * (1.0 - xint / 2.0), c};
    if (ix == 2) return {2.0 / 3.0 - (1.0 - xint) * (1.0 - xint) * (1.0 - 0.5 * (1.0 - xint)), c};
    return {1.0 / 6.0 * xint * xint * xint, c};
}
static inline int dshape_points(int type, int ord) { return type == 2 ? ord + 3 : ord + type + 1; }
static inline DShape dshapeN(int type, int ord, double xmid, int ix) {
    if (ord == 2) return dshape2(type, xmid, ix);
    if (type == 0) {
        if (ord == 0) return {1.0, 0.0, (int)std::floor(xmid + 0.5)};
        const double xfloor = std::floor(xmid), x = xmid - xfloor, x2 = x * x, x3 = x2 * x;
        if (ord == 1) return ix == 0 ? DShape{1.0 - x, 1.0, (int)xfloor} : DShape{x, -1.0, (int)xfloor + 1};
        const int c = (int)xfloor - 1 + ix;
        if (ix == 0) return {-1.0 / 6.0 * x3 + 0.5 * x2 - 0.5 * x + 1.0 / 6.0, -(-0.5 * x2 + x - 0.5), c};
        if (ix == 1) return {0.5 * x3 - x2 + 2.0 / 3.0, -(1.5 * x2 - 2 * x), c};
        if (ix == 2) return {-0.5 * x3 + 0.5 * x2 + 0.5 * x + 1.0 / 6.0, -(-1.5 * x2 + x + 0.5), c};
        return {1.0 / 6.0 * x3, -(0.5 * x2), c};
    }
    if (type == 1) {
        if (ord == 0) {
            const double xfloor = std::floor(xmid), x = xmid - xfloor;
            const bool lo = x < 0.5;
            return ix == 0 ? DShape{lo ? 1.0 : 0.0, 1.0, (int)xfloor} : DShape{lo ? 0.0 : 1.0, -1.0, (int)xfloor + 1};
        }
        const double xm = xmid + 0.5, xfloor = std::floor(xm), x = xm - xfloor, x2 = x * x, x3 = x2 * x;
        const bool lo = x < 0.5;
        if (ord == 1) {
            const int c = (int)xfloor - 1 + ix;
            if (ix == 0) return {lo ? 0.5 - x : 0.0, -(x - 1), c};
            if (ix == 1) return {lo ? x + 0.5 : 1.5 - x, -(1 - 2 * x), c};
            return {lo ? 0.0 : x - 0.5, -x, c};
        }
        const int c = (int)xfloor - 2 + ix;
        if (ix == 0) return {lo ? -1.0 / 6.0 * x3 + 0.25 * x2 - 0.125 * x + 1.0 / 48.0 : 0.0,
                             -(1.0 / 6.0 * x3 - 0.5 * x2 + 0.5 * x - 1.0 / 6.0), c};
        if (ix == 1) return {lo ? 0.5 * x3 - 0.25 * x2 - 0.625 * x + 23.0 / 48.0 : -1.0 / 6.0 * x3 + 0.75 * x2 - 1.125 * x + 9.0 / 16.0,
                             -(-2.0 / 3.0 * x3 + 1.5 * x2 - 0.5 * x - 0.5), c};
        if (ix == 2) return {lo ? -0.5 * x3 - 0.25 * x2 + 0.625 * x + 23.0 / 48.0 : 0.5 * x3 - 1.75 * x2 + 1.375 * x + 17.0 / 48.0,
                             -(x3 - 1.5 * x2 - 0.5 * x + 0.5), c};
        if (ix == 3) return {lo ? 1.0 / 6.0 * x3 + 0.25 * x2 + 0.125 * x + 1.0 / 48.0 : -0.5 * x3 + 1.25 * x2 - 0.375 * x + 5.0 / 48.0,
                             -(-2.0 / 3.0 * x3 + 0.5 * x2 + 0.5 * x + 1.0 / 6.0), c};
        return {lo ? 0.0 : 1.0 / 6.0 * x3 - 0.25 * x2 + 0.125 * x - 1.0 / 48.0, -(1.0 / 6.0 * x3), c};
    }
    if (ord == 0) {
        const int c = (int)std::floor(xmid + 0.5) - 1 + ix;
        if (ix == 0) return {0.0, 0.5, c};
        if (ix == 1) return {1.0, 0.0, c};
        return {0.0, -0.5, c};
    }
    const double xfloor = std::floor(xmid), x = xmid - xfloor, x2 = x * x, x3 = x2 * x;
    if (ord == 1) {
        const int c = (int)xfloor - 1 + ix;
        if (ix == 0) return {0.0, -(0.5 * x - 0.5), c};
        if (ix == 1) return {1 - x, -(-0.5 * x), c};
        if (ix == 2) return {x, -(0.5 - 0.5 * x), c};
        return {0.0, -(0.5 * x), c};
    }
    const int c = (int)xfloor - 2 + ix;
    if (ix == 0) return {0.0, -(1.0 / 12.0 * x3 - 0.25 * x2 + 0.25 * x - 1.0 / 12.0), c};
    if (ix == 1) return {-1.0 / 6.0 * x3 + 0.5 * x2 - 0.5 * x + 1.0 / 6.0, -(-0.25 * x3 + 0.5 * x2 - 1.0 / 3.0), c};
    if (ix == 2) return {0.5 * x3 - x2 + 2.0 / 3.0, -(1.0 / 6.0 * x3 - 0.5 * x), c};
    if (ix == 3) return {-0.5 * x3 + 0.5 * x2 + 0.5 * x + 1.0 / 6.0, -(1.0 / 6.0 * x3 - 0.5 * x2 + 1.0 / 3.0), c};
    if (ix == 4) return {1.0 / 6.0 * x3, -(-0.25 * x3 + 0.25 * x2 + 0.25 * x + 1.0 / 12.0), c};
    return {0.0, -(1.0 / 12.0 * x3), c};
}

// ------------------------------------------------------------------------------------------
// Slice field storage: nx x ny interior plus guard cells (the reference uses
// (depos_order+1)/2+1 = 2 guards, Fields.cpp:63; one more is allocated so that stencils that
// touch a zero-weight cell beyond the guard stay in bounds).
// ------------------------------------------------------------------------------------------
struct Grid {
    int nx, ny, g;
    int px;  // pitch
    size_t size() const { return (size_t)(nx + 2 * g) * (ny + 2 * g); }
    size_t idx(int i, int j) const { return (size_t)(j + g) * px + (i + g); }
};

struct Field {
    std::vector<double> a;
    Grid gr;
    void init(const Grid& g) { gr = g; a.assign(g.size(), 0.0); }
    double& operator()(int i, int j) { return a[gr.idx(i, j)]; }
    double operator()(int i, int j) const { return a[gr.idx(i, j)]; }
    void zero() { std::fill(a.begin(), a.end(), 0.0); }
};

struct Plasma {
    std::vector<double> x, y, w, ux, uy, psi, x_prev, y_prev, ux_h, uy_h, psi_h;
    std::vector<uint8_t> valid;
    size_t n() const { return x.size(); }
};

struct BeamParticle {
    double x, y, z, w, ux, uy, uz;
    int64_t id;
    int nsub;
    bool valid;
};

struct BeamSlice {
    std::vector<BeamParticle> p;
    size_t num_nonslipped = 0;
};

// ------------------------------------------------------------------------------------------
// Complex DFT of any length N, out_k = sum_j in_j exp(-2 pi i j k / N), on split real/imaginary
// arrays: iterative radix-2 (bit reversal, then butterflies) when N is a power of two, else
// recursive mixed-radix Cooley-Tukey decimation in time over the prime factors of N (a prime
// factor p costs O(p^2) per butterfly group). Used for the DST-I below.
// ------------------------------------------------------------------------------------------
struct FFTPlan {
    int N = 0;
    bool pow2 = false;
    std::vector<int> f;         // prime factors of N (mixed radix)
    std::vector<double> wr, wi;  // exp(-2 pi i t / N), t < N
    std::vector<int> rev;       // bit reversal (radix 2)
    int pmax = 1;
    void init(int n) {
        N = n;
        pow2 = n >= 2 && (n & (n - 1)) == 0;
        f.clear();
        for (int m = n, p = 2; m > 1;) {
            if (m % p == 0) { f.push_back(p); m /= p; continue; }
            p = (p == 2) ? 3 : p + 2;
            if ((long long)p * p > m) { f.push_back(m); break; }
        }
        pmax = 1;
        for (int p : f) pmax = std::max(pmax, p);
        wr.resize(N);
        wi.resize(N);
        const double pi = 3.14159265358979323846;
        for (int t = 0; t < N; ++t) { wr[t] = std::cos(2 * pi * t / N); wi[t] = -std::sin(2 * pi * t / N); }
        if (pow2) {
            rev.resize(N);
            int bits = 0;
            while ((1 << bits) < N) ++bits;
            for (int i = 0; i < N; ++i) {
                int r = 0;
                for (int k = 0; k < bits; ++k) r |= ((i >> k) & 1) << (bits - 1 - k);
                rev[i] = r;
            }
        }
    }
    // in place on (re, im); tmp holds 2 * (N + pmax) doubles
    void forward(double* re, double* im, double* tmp) const {
        if (pow2) {
            for (int i = 0; i < N; ++i)
                if (rev[i] > i) { std::swap(re[i], re[rev[i]]); std::swap(im[i], im[rev[i]]); }
            for (int len = 2; len <= N; len <<= 1) {
                const int half = len >> 1, step = N / len;
                for (int i0 = 0; i0 < N; i0 += len)
                    for (int k = 0; k < half; ++k) {
                        const double c = wr[k * step], s = wi[k * step];
                        const int a = i0 + k, b = a + half;
                        const double vr = re[b] * c - im[b] * s, vi = re[b] * s + im[b] * c;
                        re[b] = re[a] - vr; im[b] = im[a] - vi;
                        re[a] += vr; im[a] += vi;
                    }
            }
            return;
        }
        double* orr = tmp;
        double* oi = tmp + N;
        rec(orr, oi, re, im, N, 1, 0, tmp + 2 * N);
        std::copy(orr, orr + N, re);
        std::copy(oi, oi + N, im);
    }
    void rec(double* outr, double* outi, const double* inr, const double* ini, int n, int s, int fi, double* t) const {
        const int p = f[fi], m = n / p;
        if (m == 1) for (int r = 0; r < p; ++r) { outr[r] = inr[(size_t)r * s]; outi[r] = ini[(size_t)r * s]; }
        else for (int r = 0; r < p; ++r) rec(outr + (size_t)r * m, outi + (size_t)r * m, inr + (size_t)r * s, ini + (size_t)r * s, m, s * p, fi + 1, t);
        const int sn = N / n, sp = N / p;
        double* tr = t;
        double* ti = t + p;
        for (int k1 = 0; k1 < m; ++k1) {
            for (int r = 0; r < p; ++r) {
                const size_t w = (size_t)r * k1 * sn;  // < N
                const double ar = outr[(size_t)r * m + k1], ai = outi[(size_t)r * m + k1];
                tr[r] = ar * wr[w] - ai * wi[w];
                ti[r] = ar * wi[w] + ai * wr[w];
            }
            for (int k2 = 0; k2 < p; ++k2) {
                double accr = 0, acci = 0;
                size_t w = 0;
                const size_t dw = (size_t)k2 * sp;
                for (int r = 0; r < p; ++r) {
                    accr += tr[r] * wr[w] - ti[r] * wi[w];
                    acci += tr[r] * wi[w] + ti[r] * wr[w];
                    w += dw;
                    if (w >= (size_t)N) w -= N;
                }
                outr[(size_t)k2 * m + k1] = accr;
                outi[(size_t)k2 * m + k1] = acci;
            }
        }
    }
};

// Unnormalised DST-I (FFTW RODFT00): y_k = 2 sum_j x_j sin(pi (j+1)(k+1) / (n+1)). The odd
// extension z of length N = 2(n+1) (z_0 = z_{n+1} = 0, z_{j+1} = x_j, z_{N-1-j} = -x_j) has
// DFT(z)_{k+1} = -i y_k. Two real rows a, b go through one complex DFT of z_a + i z_b:
// y_a = -Im, y_b = Re.
struct DST1 {
    int n = 0;
    FFTPlan plan;
    void init(int n_) { n = n_; plan.init(2 * (n + 1)); }
    size_t work_size() const { return (size_t)2 * plan.N + 2 * ((size_t)plan.N + plan.pmax); }
    // rows a and b (b may be null), strided; in place
    void apply2(double* a, double* b, size_t st, double* work) const {
        const int N = plan.N;
        double* re = work;
        double* im = work + N;
        re[0] = im[0] = re[n + 1] = im[n + 1] = 0;
        for (int j = 0; j < n; ++j) {
            const double va = a[(size_t)j * st], vb = b ? b[(size_t)j * st] : 0.0;
            re[j + 1] = va; re[N - 1 - j] = -va;
            im[j + 1] = vb; im[N - 1 - j] = -vb;
        }
        plan.forward(re, im, work + 2 * N);
        for (int k = 0; k < n; ++k) {
            a[(size_t)k * st] = -im[k + 1];
            if (b) b[(size_t)k * st] = re[k + 1];
        }
    }
};

// ------------------------------------------------------------------------------------------
// Dirichlet Poisson solver: DST-I in x and y, eigenvalue divide, DST-I back
// (FFTPoissonSolverDirichletFast.cpp:196-328; FFTW RODFT00 in FFTPoissonSolverDirichletDirect).
// The transforms are the FFT-based DST-I above (O(n^2 log n) per solve, like FFTW); the
// normalisation 1/(4(nx+1)(ny+1)) of two unnormalised RODFT00 transforms per axis is folded
// into the eigenvalues.
// ------------------------------------------------------------------------------------------
struct PoissonDST {
    int nx = 0, ny = 0;
    DST1 tx, ty;
    std::vector<double> eig;  // eigenvalues (ny x nx)
    void init(int nx_, int ny_, double dx, double dy) {
        nx = nx_; ny = ny_;
        const double pi = 3.14159265358979323846;
        tx.init(nx);
        ty.init(ny);
        const double sxf = pi / (2. * (nx + 1)), syf = pi / (2. * (ny + 1));
        const double norm = 0.5 / (2 * ((nx + 1) * (ny + 1)));
        eig.resize((size_t)nx * ny);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double a = std::sin((i + 1) * sxf), b = std::sin((j + 1) * syf);
                a *= a; b *= b;
                eig[(size_t)j * nx + i] = (a != 0 && b != 0) ? norm / (-4.0 * (a / (dx * dx) + b / (dy * dy))) : 0.0;
            }
    }
    // in/out: row-major ny x nx
    // rows (x) or columns (y) in pairs, one complex DFT per pair
    void transform_x(std::vector<double>& v) const {
#pragma omp parallel
        {
            std::vector<double> work(tx.work_size());
#pragma omp for schedule(static)
            for (int j = 0; j < ny; j += 2)
                tx.apply2(&v[(size_t)j * nx], j + 1 < ny ? &v[(size_t)(j + 1) * nx] : nullptr, 1, work.data());
        }
    }
    void transform_y(std::vector<double>& v) const {
#pragma omp parallel
        {
            std::vector<double> work(ty.work_size());
#pragma omp for schedule(static)
            for (int i = 0; i < nx; i += 2) ty.apply2(&v[i], i + 1 < nx ? &v[i + 1] : nullptr, nx, work.data());
        }
    }
    void solve(std::vector<double>& v) const {
        transform_x(v);
        transform_y(v);
        for (size_t k = 0; k < v.size(); ++k) v[k] *= eig[k];
        transform_y(v);
        transform_x(v);
    }
};

// ------------------------------------------------------------------------------------------
// Geometric multigrid for -a*u + Lap(u) = f, two components sharing a (HpMultiGrid.cpp,
// system type 1). Cell-centred levels when n is even (Dirichlet on the cell face, 4/3 closure
// :162-183, 265-294), node-centred otherwise (Dirichlet on the first guard node, :1054-1066).
// ------------------------------------------------------------------------------------------
struct MGLevel {
    int lo_i, hi_i, lo_j, hi_j;  // full box (cell: 0..n-1; node: 0..N+1)
    int vlo_i, vhi_i, vlo_j, vhi_j;  // valid loop box
    int w, h;
    std::vector<double> acf, res[2], cor[2], rescor[2];
    size_t id(int i, int j) const { return (size_t)(j - lo_j) * w + (i - lo_i); }
};

struct Multigrid {
    bool cell = true;
    double dx = 0, dy = 0;
    std::vector<MGLevel> L;
    int total_vcycles = 0;

    void init(int nx, int ny, double dx_, double dy_) {
        dx = dx_; dy = dy_;
        cell = (nx % 2 == 0);
        L.clear();
        int lx, ly;  // box bounds
        if (cell) { lx = nx - 1; ly = ny - 1; } else { lx = nx + 1; ly = ny + 1; }
        for (int lev = 0; lev < 40; ++lev) {
            MGLevel m;
            m.lo_i = 0; m.lo_j = 0; m.hi_i = lx; m.hi_j = ly;
            m.w = lx + 1; m.h = ly + 1;
            if (cell) { m.vlo_i = 0; m.vlo_j = 0; m.vhi_i = lx; m.vhi_j = ly; }
            else { m.vlo_i = 1; m.vlo_j = 1; m.vhi_i = lx - 1; m.vhi_j = ly - 1; }
            const size_t n = (size_t)m.w * m.h;
            m.acf.assign(n, 0.0);
            for (int c = 0; c < 2; ++c) { m.res[c].assign(n, 0.0); m.cor[c].assign(n, 0.0); m.rescor[c].assign(n, 0.0); }
            L.push_back(std::move(m));
            // coarsenable with min width 2 (cell) or 4 (node)  (HpMultiGrid.cpp:1067-1074)
            const int len_x = lx + 1, len_y = ly + 1;
            const int minw = cell ? 2 : 4;
            if (len_x < 2 * minw || len_y < 2 * minw) break;
            if (cell) {
                if (len_x % 2 || len_y % 2) break;
                lx = len_x / 2 - 1; ly = len_y / 2 - 1;
            } else {
                if (lx % 2 || ly % 2) break;
                lx = lx / 2; ly = ly / 2;
            }
        }
    }

    static inline double lap(const MGLevel& m, const std::vector<double>& p, int i, int j,
                             double facx, double facy, bool cellc) {
        double l = -2.0 * (facx + facy) * p[m.id(i, j)];
        if (cellc && i == m.lo_i) l += facx * (4. / 3. * p[m.id(i + 1, j)] - 2. * p[m.id(i, j)]);
        else if (cellc && i == m.hi_i) l += facx * (4. / 3. * p[m.id(i - 1, j)] - 2. * p[m.id(i, j)]);
        else l += facx * (p[m.id(i - 1, j)] + p[m.id(i + 1, j)]);
        if (cellc && j == m.lo_j) l += facy * (4. / 3. * p[m.id(i, j + 1)] - 2. * p[m.id(i, j)]);
        else if (cellc && j == m.hi_j) l += facy * (4. / 3. * p[m.id(i, j - 1)] - 2. * p[m.id(i, j)]);
        else l += facy * (p[m.id(i, j - 1)] + p[m.id(i, j + 1)]);
        return l;
    }
    // gs1 (HpMultiGrid.cpp:265-294)
    static inline void gs(const MGLevel& m, std::vector<double>& p, int i, int j, double rhs, double a,
                          double facx, double facy, bool cellc) {
        double l;
        double c0 = -(a + 2. * (facx + facy));
        if (cellc && i == m.lo_i) { l = facx * (4. / 3.) * p[m.id(i + 1, j)]; c0 -= 2. * facx; }
        else if (cellc && i == m.hi_i) { l = facx * (4. / 3.) * p[m.id(i - 1, j)]; c0 -= 2. * facx; }
        else l = facx * (p[m.id(i - 1, j)] + p[m.id(i + 1, j)]);
        if (cellc && j == m.lo_j) { l += facy * (4. / 3.) * p[m.id(i, j + 1)]; c0 -= 2. * facy; }
        else if (cellc && j == m.hi_j) { l += facy * (4. / 3.) * p[m.id(i, j - 1)]; c0 -= 2. * facy; }
        else l += facy * (p[m.id(i, j - 1)] + p[m.id(i, j + 1)]);
        const double c0_inv = 1. / c0;
        p[m.id(i, j)] = (rhs - l) * c0_inv;
    }
    // gsrb_4_residual (HpMultiGrid.cpp:697-850): phi_out = 4 red-black colour sweeps starting
    // from phi_in (or zero), then optionally res_out = rhs - L(phi_out).
    void smooth4(int lev, std::vector<double>* phi_out, std::vector<double>* const* rhs,
                 const std::vector<double>* const* phi_in, std::vector<double>* const* res_out,
                 int nsweeps = 4) {
        MGLevel& m = L[lev];
        const double f = (double)(1 << lev);
        const double ddx = dx * f, ddy = dy * f;
        const double facx = 1. / (ddx * ddx), facy = 1. / (ddy * ddy);
        for (int c = 0; c < 2; ++c) {
            std::vector<double>& p = phi_out[c];
            for (int j = m.lo_j; j <= m.hi_j; ++j)
                for (int i = m.lo_i; i <= m.hi_i; ++i) {
                    const bool v = i >= m.vlo_i && i <= m.vhi_i && j >= m.vlo_j && j <= m.vhi_j;
                    p[m.id(i, j)] = (v && phi_in) ? (*phi_in[c])[m.id(i, j)] : 0.0;
                }
        }
        for (int is = 0; is < nsweeps; ++is) {
            for (int c = 0; c < 2; ++c) {
                std::vector<double>& p = phi_out[c];
                const std::vector<double>& r = *rhs[c];
#pragma omp parallel for schedule(static)
                for (int j = m.vlo_j; j <= m.vhi_j; ++j)
                    for (int i = m.vlo_i; i <= m.vhi_i; ++i)
                        if ((i + j + is) % 2 == 0) gs(m, p, i, j, r[m.id(i, j)], m.acf[m.id(i, j)], facx, facy, cell);
            }
        }
        if (res_out) {
            for (int c = 0; c < 2; ++c) {
                const std::vector<double>& p = phi_out[c];
                const std::vector<double>& r = *rhs[c];
                std::vector<double>& o = *res_out[c];
#pragma omp parallel for schedule(static)
                for (int j = m.vlo_j; j <= m.vhi_j; ++j)
                    for (int i = m.vlo_i; i <= m.vhi_i; ++i) {
                        const size_t k = m.id(i, j);
                        o[k] = r[k] + m.acf[k] * p[k] - lap(m, p, i, j, facx, facy, cell);
                    }
            }
        }
    }
    // restrict_cc / restrict_nd (HpMultiGrid.cpp:29-53)
    void restrict_to(int lev_c, const std::vector<double>& fine, std::vector<double>& crse) {
        const MGLevel& C = L[lev_c];
        const MGLevel& F = L[lev_c - 1];
        for (int j = C.vlo_j; j <= C.vhi_j; ++j)
            for (int i = C.vlo_i; i <= C.vhi_i; ++i) {
                if (cell) {
                    crse[C.id(i, j)] = 0.25 * (fine[F.id(2 * i, 2 * j)] + fine[F.id(2 * i + 1, 2 * j)] +
                                               fine[F.id(2 * i, 2 * j + 1)] + fine[F.id(2 * i + 1, 2 * j + 1)]);
                } else {
                    crse[C.id(i, j)] = (1. / 16.) * (fine[F.id(2 * i - 1, 2 * j - 1)] + 2. * fine[F.id(2 * i, 2 * j - 1)] +
                                                     fine[F.id(2 * i + 1, 2 * j - 1)] + 2. * fine[F.id(2 * i - 1, 2 * j)] +
                                                     4. * fine[F.id(2 * i, 2 * j)] + 2. * fine[F.id(2 * i + 1, 2 * j)] +
                                                     fine[F.id(2 * i - 1, 2 * j + 1)] + 2. * fine[F.id(2 * i, 2 * j + 1)] +
                                                     fine[F.id(2 * i + 1, 2 * j + 1)]);
                }
            }
    }
    // interpcpy_cc / interpcpy_nd (HpMultiGrid.cpp:79-120): out = fine_in + I(crse)
    void interp_add(int lev_f, const std::vector<double>& fin, const std::vector<double>& crse,
                    std::vector<double>& out) {
        const MGLevel& F = L[lev_f];
        const MGLevel& C = L[lev_f + 1];
        auto cdiv = [](int i) { return i >= 0 ? i / 2 : -((-i + 1) / 2); };
        for (int j = F.vlo_j; j <= F.vhi_j; ++j)
            for (int i = F.vlo_i; i <= F.vhi_i; ++i) {
                const int ic = cdiv(i), jc = cdiv(j);
                const size_t k = F.id(i, j);
                if (cell) { out[k] = fin[k] + crse[C.id(ic, jc)]; continue; }
                const bool io = ic * 2 != i, jo = jc * 2 != j;
                if (io && jo) out[k] = fin[k] + (crse[C.id(ic, jc)] + crse[C.id(ic + 1, jc)] + crse[C.id(ic, jc + 1)] + crse[C.id(ic + 1, jc + 1)]) * 0.25;
                else if (io) out[k] = fin[k] + (crse[C.id(ic, jc)] + crse[C.id(ic + 1, jc)]) * 0.5;
                else if (jo) out[k] = fin[k] + (crse[C.id(ic, jc)] + crse[C.id(ic, jc + 1)]) * 0.5;
                else out[k] = fin[k] + crse[C.id(ic, jc)];
            }
    }

    // one V-cycle (HpMultiGrid.cpp:1429-1512 with the bottom solve :1514-1595)
    void vcycle(std::vector<double>* sol, std::vector<double>* const* rhs0) {
        const int nl = (int)L.size();
        for (int lev = 0; lev < nl - 1; ++lev) {
            if (lev > 0) {
                std::vector<double>* r[2] = {&L[lev].res[0], &L[lev].res[1]};
                std::vector<double>* o[2] = {&L[lev].rescor[0], &L[lev].rescor[1]};
                smooth4(lev, L[lev].cor, r, nullptr, o);
            }
            for (int c = 0; c < 2; ++c) restrict_to(lev + 1, L[lev].rescor[c], L[lev + 1].res[c]);
        }
        {   // bottom: zero initial guess, 16 sweeps
            const int lev = nl - 1;
            std::vector<double>* r[2] = {&L[lev].res[0], &L[lev].res[1]};
            const int len = std::max(L[lev].w, L[lev].h);
            const int ns = std::max(16, (len + 1) / 2 * 2);
            smooth4(lev, L[lev].cor, r, nullptr, nullptr, ns);
        }
        for (int lev = nl - 2; lev >= 0; --lev) {
            for (int c = 0; c < 2; ++c) interp_add(lev, L[lev].cor[c], L[lev + 1].cor[c], L[lev].rescor[c]);
            const std::vector<double>* in[2] = {&L[lev].rescor[0], &L[lev].rescor[1]};
            if (lev == 0) {
                smooth4(0, sol, rhs0, in, nullptr);
            } else {
                std::vector<double>* r[2] = {&L[lev].res[0], &L[lev].res[1]};
                smooth4(lev, L[lev].cor, r, in, nullptr);
            }
        }
        const std::vector<double>* in[2] = {&sol[0], &sol[1]};
        std::vector<double>* o[2] = {&L[0].rescor[0], &L[0].rescor[1]};
        smooth4(0, L[0].cor, rhs0, in, o);
        total_vcycles++;
    }

    double maxabs_valid(int lev, const std::vector<double>* a) const {
        const MGLevel& m = L[lev];
        double r = 0;
        for (int c = 0; c < 2; ++c)
            for (int j = m.vlo_j; j <= m.vhi_j; ++j)
                for (int i = m.vlo_i; i <= m.vhi_i; ++i) r = std::max(r, std::fabs(a[c][m.id(i, j)]));
        return r;
    }

    // solve1 + solve_doit (HpMultiGrid.cpp:1169-1427). Field layout: cell (i,j) of the slice maps
    // to MG index (i,j) for cell-centred and (i+1,j+1) for node-centred levels.
    // Returns 0 on success, 1 if not converged within maxiter, 2 on divergence.
    int solve(Field& Bx, Field& By, const Field& Sy, const Field& Sx, const Field& chi,
              double tol_rel, double tol_abs, int maxiter, int* iters_out) {
        MGLevel& m0 = L[0];
        const int off = cell ? 0 : 1;
        auto map_in = [&](const Field& f, std::vector<double>& dst) {
            for (int j = m0.lo_j; j <= m0.hi_j; ++j)
                for (int i = m0.lo_i; i <= m0.hi_i; ++i) dst[m0.id(i, j)] = f(i - off, j - off);
        };
        map_in(chi, m0.acf);
        // average_down_acoef (HpMultiGrid.cpp:1640-1700)
        for (size_t lev = 1; lev < L.size(); ++lev) restrict_to((int)lev, L[lev - 1].acf, L[lev].acf);
        std::vector<double> sol[2], rhs[2];
        for (int c = 0; c < 2; ++c) { sol[c].assign(m0.acf.size(), 0.0); rhs[c].assign(m0.acf.size(), 0.0); }
        map_in(Bx, sol[0]); map_in(By, sol[1]);
        map_in(Sy, rhs[0]); map_in(Sx, rhs[1]);
        std::vector<double>* rp[2] = {&rhs[0], &rhs[1]};
        const std::vector<double>* sp[2] = {&sol[0], &sol[1]};
        std::vector<double>* op[2] = {&m0.rescor[0], &m0.rescor[1]};
        smooth4(0, m0.cor, rp, sp, op);
        const double resnorm0 = maxabs_valid(0, m0.rescor);
        const double rhsnorm0 = maxabs_valid(0, rhs);
        const double max_norm = (rhsnorm0 >= resnorm0) ? rhsnorm0 : resnorm0;
        const double res_target = std::max(tol_abs, std::max(tol_rel, 1.e-16) * max_norm);
        int status = 0, it = 0;
        if (!(resnorm0 <= res_target)) {
            bool converged = false;
            for (int iter = 0; iter < maxiter; ++iter) {
                vcycle(sol, rp);
                it = iter + 1;
                const double norminf = maxabs_valid(0, m0.rescor);
                converged = norminf <= res_target;
                if (converged) break;
                if (norminf > 1.e20 * max_norm) { status = 2; break; }
            }
            if (!converged && status == 0) status = 1;
        }
        if (iters_out) *iters_out = it;
        for (int j = m0.vlo_j; j <= m0.vhi_j; ++j)
            for (int i = m0.vlo_i; i <= m0.vhi_i; ++i) {
                Bx(i - off, j - off) = m0.cor[0][m0.id(i, j)];
                By(i - off, j - off) = m0.cor[1][m0.id(i, j)];
            }
        return status;
    }
};

// ------------------------------------------------------------------------------------------
// Forward-mode tangent numbers for the adjoint: value and one directional derivative. The
// per-particle maps (deposit, explicit deposit, gather + push) are written once for a generic
// scalar type; the adjoint of a particle's contribution L = sum(lambda * output) with respect to
// one input is L's tangent when that input is seeded with 1.
// ------------------------------------------------------------------------------------------
struct Tn { double v, d; };
static inline Tn operator+(Tn a, Tn b) { return {a.v + b.v, a.d + b.d}; }
static inline Tn operator-(Tn a, Tn b) { return {a.v - b.v, a.d - b.d}; }
static inline Tn operator*(Tn a, Tn b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
static inline Tn operator/(Tn a, Tn b) { const double q = a.v / b.v; return {q, (a.d - q * b.d) / b.v}; }
static inline Tn operator-(Tn a) { return {-a.v, -a.d}; }
static inline Tn operator+(Tn a) { return a; }
static inline Tn operator+(Tn a, double b) { return {a.v + b, a.d}; }
static inline Tn operator+(double a, Tn b) { return {a + b.v, b.d}; }
static inline Tn operator-(Tn a, double b) { return {a.v - b, a.d}; }
static inline Tn operator-(double a, Tn b) { return {a - b.v, -b.d}; }
static inline Tn operator*(Tn a, double b) { return {a.v * b, a.d * b}; }
static inline Tn operator*(double a, Tn b) { return {a * b.v, a * b.d}; }
static inline Tn operator/(Tn a, double b) { return {a.v / b, a.d / b}; }
static inline Tn operator/(double a, Tn b) { const double q = a / b.v; return {q, -q * b.d / b.v}; }
static inline double val(double a) { return a; }
static inline double val(Tn a) { return a.v; }
static inline Tn seed(double v, bool on) { return {v, on ? 1.0 : 0.0}; }

template <class T> struct ShapeT { T s; int cell; };
template <class T> struct DShapeT { T s, ds; int cell; };

// shape2 / dshape2 above on a generic scalar (same expressions)
template <class T>
static inline ShapeT<T> shape2t(T xmid, int ix) {
    const double xfloor = std::floor(val(xmid) + 0.5);
    const T xint = xmid - xfloor;
    if (ix == 0) return {0.5 * (0.5 - xint) * (0.5 - xint), (int)xfloor - 1};
    if (ix == 1) return {0.75 - xint * xint, (int)xfloor};
    return {0.5 * (0.5 + xint) * (0.5 + xint), (int)xfloor + 1};
}
template <class T>
static inline DShapeT<T> dshape2t(int type, T xmid, int ix) {
    if (type == 0) {
        xmid = xmid + 0.5;
        const double xfloor = std::floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        if (ix == 0) return {0.5 * x2 - 1.0 * xint + 0.5, -(xint - 1.0), (int)xfloor - 1 + ix};
        if (ix == 1) return {-x2 + 1.0 * xint + 0.5, -(1.0 - 2 * xint), (int)xfloor - 1 + ix};
        return {0.5 * x2, -xint, (int)xfloor - 1 + ix};
    } else if (type == 1) {
        const double xfloor = std::floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        const bool lo = val(xint) < 0.5;
        const T zero = 0.0 * xint;
        if (ix == 0) return {lo ? 0.5 * x2 - 0.5 * xint + 1.0 / 8.0 : zero, -(-0.5 * x2 + xint - 0.5), (int)xfloor - 1 + ix};
        if (ix == 1) return {lo ? 0.75 - x2 : 0.5 * x2 - 1.5 * xint + 9.0 / 8.0, -(1.5 * x2 - 2 * xint), (int)xfloor - 1 + ix};
        if (ix == 2) return {lo ? 0.5 * x2 + 0.5 * xint + 1.0 / 8.0 : -x2 + 2 * xint - 0.25, -(-1.5 * x2 + xint + 0.5), (int)xfloor - 1 + ix};
        return {lo ? zero : 0.5 * x2 - 0.5 * xint + 1.0 / 8.0, -(0.5 * x2), (int)xfloor - 1 + ix};
    } else {
        xmid = xmid + 0.5;
        const double xfloor = std::floor(val(xmid));
        const T xint = xmid - xfloor, x2 = xint * xint;
        const T zero = 0.0 * xint;
        if (ix == 0) return {zero, -(-0.25 * x2 + 0.5 * xint - 0.25), (int)xfloor - 2 + ix};
        if (ix == 1) return {0.5 * x2 - xint + 0.5, -(0.5 * x2 - 0.5 * xint - 0.25), (int)xfloor - 2 + ix};
        if (ix == 2) return {-x2 + xint + 0.5, -(0.25 - 0.5 * xint), (int)xfloor - 2 + ix};
        if (ix == 3) return {0.5 * x2, -(-0.5 * x2 + 0.5 * xint + 0.25), (int)xfloor - 2 + ix};
        return {zero, -(0.25 * x2), (int)xfloor - 2 + ix};
    }
}

// Taylor dual (value, d/dzeta) over a generic scalar, as in the plasma push
template <class T> struct DuT { T v, e; };
template <class T> static inline DuT<T> tadd(DuT<T> a, DuT<T> b) { return {a.v + b.v, a.e + b.e}; }
template <class T> static inline DuT<T> tsub(DuT<T> a, DuT<T> b) { return {a.v - b.v, a.e - b.e}; }
template <class T> static inline DuT<T> tmul(DuT<T> a, DuT<T> b) { return {a.v * b.v, a.e * b.v + a.v * b.e}; }

// ------------------------------------------------------------------------------------------
// The simulation
// ------------------------------------------------------------------------------------------
class Sim {
public:
    SimConfig cfg;
    Grid gr{};
    int nx = 0, ny = 0, nz = 0;
    double dx = 0, dy = 0, dz = 0, dxi = 0, dyi = 0, dzi = 0;
    double xoff = 0, yoff = 0;  // GetPosOffset for the guarded slice box
    std::map<std::string, Field> F;
    std::vector<Plasma> plasmas;
    // beams: per beam, per slice storage for the next step
    std::vector<std::vector<BeamSlice>> store;
    std::vector<BeamSlice> bthis, bnext;
    std::vector<bool> store_valid;
    PoissonDST dst;
    Multigrid mg;
    double physical_time = 0;
    double step_dt = 0, next_time = 0;  // this step's dt and end time (hpq::step_time)
    std::string error;
    int mg_status = 0;
    // SALAME state (Hipace.H:290-295) and a record of (slice, iteration, W) of every iteration
    int sal_last = -1;
    bool sal_overloaded = false;
    double sal_zeta0 = 0;
    std::vector<double> salame_log;
    long long mg_iters_total = 0;
    // diagnostics: requested components, 3-D arrays (nz x ny x nx) for the last solved step
    std::vector<std::string> diag_names;
    std::map<std::string, std::vector<double>> diag;
    std::vector<double> pc_errors;

    explicit Sim(const SimConfig& c) : cfg(c) {
        nx = c.n_cell[0]; ny = c.n_cell[1]; nz = c.n_cell[2];
        dx = (c.prob_hi[0] - c.prob_lo[0]) / nx;
        dy = (c.prob_hi[1] - c.prob_lo[1]) / ny;
        dz = (c.prob_hi[2] - c.prob_lo[2]) / nz;
        dxi = 1. / dx; dyi = 1. / dy; dzi = 1. / dz;
        gr.nx = nx; gr.ny = ny; gr.g = 3; gr.px = nx + 2 * gr.g;
        // GetPosOffset with the 2-guard slice box (Fields.H:72-76)
        xoff = 0.5 * (c.prob_lo[0] + c.prob_hi[0] - dx * ((-2) + (nx + 1)));
        yoff = 0.5 * (c.prob_lo[1] + c.prob_hi[1] - dy * ((-2) + (ny + 1)));
        const char* names_explicit[] = {
            "chi", "Sy", "Sx", "ExmBy", "EypBx", "Ez", "Bx", "By", "Bz", "Psi", "jx_beam", "jy_beam",
            "jz_beam", "jx", "jy", "rhomjz", "rho", "rhomjz_beam", "Next.jx_beam", "Next.jy_beam",
            "Prev.jx_beam", "Prev.jy_beam", "Ions.rhomjz"};
        const char* names_pc[] = {
            "ExmBy", "EypBx", "Ez", "Bx", "By", "Bz", "Psi", "jx", "jy", "jz", "rhomjz", "rho",
            "Next.jx", "Next.jy", "Prev.Bx", "Prev.By", "Prev.jx", "Prev.jy", "PCIter.Bx",
            "PCIter.By", "PCPrevIter.Bx", "PCPrevIter.By", "Ions.rhomjz"};
        if (c.explicit_solver) for (auto* n : names_explicit) F[n].init(gr);
        // the SALAME slice (Fields.cpp:117-128)
        if (c.explicit_solver && c.any_salame())
            for (auto* n : {"Salame.Ez_target", "Salame.Ez_no_salame", "Salame.Ez", "Salame.jx", "Salame.jy",
                            "Salame.jz_beam", "Salame.Bx", "Salame.By", "Salame.Sy", "Salame.Sx", "Salame.Sy_back",
                            "Salame.Sx_back"})
                F[n].init(gr);
        else for (auto* n : names_pc) F[n].init(gr);
        g_psi = &f("Psi"); g_ez = &f("Ez"); g_bx = &f("Bx"); g_by = &f("By"); g_bz = &f("Bz");
        dst.init(nx, ny, dx, dy);
        if (c.explicit_solver) mg.init(nx, ny, dx, dy);
        store.resize(c.beams.size());
        for (auto& s : store) s.resize(nz);
        store_valid.assign(c.beams.size(), false);
        bthis.resize(c.beams.size());
        bnext.resize(c.beams.size());
    }

    Field& f(const char* n) { return F.at(n); }

    // -------------------------------------------------------------- beam initialisation
    // BoxSort.cpp:14-78: slice = int((z - plo_z) * dzi); outside [0, nz) is dropped. Within a
    // slice the input order is kept.
    void set_beam(int b, const double* x, const double* y, const double* z, const double* w,
                  const double* ux, const double* uy, const double* uz, const int64_t* id, int64_t n) {
        auto& st = store[b];
        for (auto& s : st) { s.p.clear(); s.num_nonslipped = 0; }
        for (int64_t i = 0; i < n; ++i) {
            int s = (int)((z[i] - cfg.prob_lo[2]) * dzi);
            if (s < 0 || s >= nz) continue;
            BeamParticle p{x[i], y[i], z[i], w[i], ux[i], uy[i], uz[i], id ? id[i] : (int64_t)(i + 1), 0, true};
            if (p.w == 0.0) p.valid = false;
            st[s].p.push_back(p);
        }
        for (auto& s : st) s.num_nonslipped = s.p.size();
        store_valid[b] = true;
    }

    // InitBeamFixedPPCSlice (BeamParticleContainerInit.cpp:199-345) for all slices at once
    void init_beam_fixed_ppc(int b) {
        const hpq::BeamSpecies& B = cfg.beams[b];
        auto& st = store[b];
        const int nppc = B.ppc[0] * B.ppc[1] * B.ppc[2];
        const double scale = cfg.normalized_units ? 1. / nppc : dx * dy * dz / nppc;
        int64_t pid = 1;
        for (int k = 0; k < nz; ++k) {
            BeamSlice& s = st[k];
            s.p.clear();
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int ip = 0; ip < nppc; ++ip) {
                        const int nyp = B.ppc[1], nzp = B.ppc[2];
                        const int ixp = ip / (nyp * nzp);
                        const int iyp = (ip % (nyp * nzp)) % nyp;
                        const int izp = (ip % (nyp * nzp)) / nyp;
                        const double r0 = (0.5 + ixp) / B.ppc[0], r1 = (0.5 + iyp) / B.ppc[1], r2 = (0.5 + izp) / B.ppc[2];
                        const double x = cfg.prob_lo[0] + (i + r0) * dx;
                        const double y = cfg.prob_lo[1] + (j + r1) * dy;
                        const double z = cfg.prob_lo[2] + (k + r2) * dz;
                        if (z >= B.zmax || z < B.zmin ||
                            ((x - B.position_mean[0]) * (x - B.position_mean[0]) + (y - B.position_mean[1]) * (y - B.position_mean[1])) > B.radius * B.radius)
                            continue;
                        double dens;
                        if (B.profile == hpq::BeamProfile::Gaussian) {
                            const double ddx = (x - B.position_mean[0]) / B.position_std[0];
                            const double ddy = (y - B.position_mean[1]) / B.position_std[1];
                            const double ddz = (z - B.position_mean[2]) / B.position_std[2];
                            dens = B.density * std::exp(-0.5 * ddx * ddx) * std::exp(-0.5 * ddy * ddy) * std::exp(-0.5 * ddz * ddz);
                        } else {
                            dens = B.density;
                        }
                        if (dens <= B.min_density) continue;
                        BeamParticle p{};
                        double xp = x, yp = y;
                        double uxp = B.u_mean[0] * cfg.pc.c, uyp = B.u_mean[1] * cfg.pc.c;
                        bool valid = enforce_bc(xp, yp, uxp, uyp);
                        p.x = xp; p.y = yp; p.z = z;
                        p.ux = uxp; p.uy = uyp; p.uz = B.u_mean[2] * cfg.pc.c;
                        p.w = valid ? std::fabs(dens * scale) : 0.0;
                        p.id = pid++;
                        p.nsub = 0;
                        p.valid = valid;
                        s.p.push_back(p);
                    }
            s.num_nonslipped = s.p.size();
        }
        store_valid[b] = true;
    }

    // InitBeamFixedWeight3D (BeamParticleContainerInit.cpp:349-476): Gaussian (or can) beam of
    // num_particles equal weights Q / (N q). The reference draws from AMReX's random stream,
    // which is not reproduced; this draw uses the counter-based Philox4x32-10 stream of
    // ../hipace2_b200/csrc/rng.hpp with the seed derivation of the library's beam injection, so
    // that the oracle and the library start from the same particles without exchanging them
    // (per particle i: normals of counters 2i and 2i+1; z of a can beam from uniform(2i+1, 3)).
    void init_beam_fixed_weight(int b) {
        const hpq::BeamSpecies& B = cfg.beams[b];
        const int64_t n = B.num_particles;
        std::vector<double> x, y, z, w, ux, uy, uz;
        std::vector<int64_t> id;
        if (n > 0) {
            const int64_t nbase = B.do_symmetrize ? n / 4 : n;
            const uint64_t seed = (uint64_t)(cfg.has_random_seed ? cfg.random_seed : 0) * 1000003ull +
                                  (uint64_t)b * 7919ull + 12345ull;
            const hpq::Philox rng(seed);
            const bool can = B.profile == hpq::BeamProfile::Can;
            const double z_mean = can ? 0.5 * (B.zmin + B.zmax) : B.position_mean[2];
            const double weight = B.total_charge / (B.num_particles * B.charge);
            const int ncopy = B.do_symmetrize ? 4 : 1;
            const size_t cap = (size_t)nbase * ncopy;
            for (auto* v : {&x, &y, &z, &w, &ux, &uy, &uz}) v->reserve(cap);
            id.reserve(cap);
            int64_t pid = 1;
            for (int64_t i = 0; i < nbase; ++i) {
                double g[8];
                rng.normals(2 * (uint64_t)i, g);
                rng.normals(2 * (uint64_t)i + 1, g + 4);
                const double zc = can ? rng.uniform(2 * (uint64_t)i + 1, 3) * (B.zmax - B.zmin) + B.zmin
                                      : z_mean + B.position_std[2] * g[0];
                double px = B.position_std[0] * g[1], py = B.position_std[1] * g[2];
                double u[3] = {B.u_mean[0] + B.u_std[0] * g[3], B.u_mean[1] + B.u_std[1] * g[4],
                               B.u_mean[2] + B.u_std[2] * g[5]};
                u[2] += (zc - z_mean) * B.duz_per_uz0_dzeta * B.u_mean[2];
                const bool inside = !(zc < B.zmin || zc > B.zmax || px * px + py * py > B.radius * B.radius);
                px -= B.z_foc * u[0] / u[2];
                py -= B.z_foc * u[1] / u[2];
                for (int q = 0; q < ncopy; ++q) {
                    const double sx = (q & 1) ? -1 : 1, sy = (q & 2) ? -1 : 1;
                    double xp = B.position_mean[0] + sx * px, yp = B.position_mean[1] + sy * py;
                    double uxp = sx * u[0] * cfg.pc.c, uyp = sy * u[1] * cfg.pc.c;
                    const bool ok = enforce_bc(xp, yp, uxp, uyp) && inside;
                    x.push_back(xp); y.push_back(yp); z.push_back(zc);
                    w.push_back(ok ? std::fabs(weight) : 0.0);
                    ux.push_back(uxp); uy.push_back(uyp); uz.push_back(u[2] * cfg.pc.c);
                    id.push_back(pid++);
                }
            }
        }
        set_beam(b, x.data(), y.data(), z.data(), w.data(), ux.data(), uy.data(), uz.data(), id.data(),
                 (int64_t)x.size());
    }

    // EnforceBC (GetAndSetPosition.H:29-99); returns false if the particle is absorbed
    bool enforce_bc(double& x, double& y, double& ux, double& uy) const {
        const double plo0 = cfg.particle_lo[0], plo1 = cfg.particle_lo[1];
        const double phi0 = cfg.particle_hi[0], phi1 = cfg.particle_hi[1];
        if (x < plo0 || y < plo1 || x > phi0 || y > phi1) {
            const double lx = phi0 - plo0, ly = phi1 - plo1;
            if (cfg.particle_bc == hpq::ParticleBC::Reflecting) {
                x = std::fmod(x - plo0, 2 * lx); if (x < 0) x += 2 * lx; x += plo0;
                if (x > phi0) { x = 2 * phi0 - x; ux = -ux; }
                y = std::fmod(y - plo1, 2 * ly); if (y < 0) y += 2 * ly; y += plo1;
                if (y > phi1) { y = 2 * phi1 - y; uy = -uy; }
                return true;
            } else if (cfg.particle_bc == hpq::ParticleBC::Periodic) {
                x = std::fmod(x - plo0, lx); if (x < 0) x += lx; x += plo0;
                y = std::fmod(y - plo1, ly); if (y < 0) y += ly; y += plo1;
                return true;
            }
            return false;
        }
        return true;
    }

    // -------------------------------------------------------------- plasma initialisation
    // PlasmaParticleContainerInit.cpp:17-310 (no fine patch, no symmetrize). Particle order:
    // loop over i_part outside, cells in x-fastest order inside.
    void init_plasmas() {
        plasmas.assign(cfg.plasmas.size(), Plasma{});
        const double c_t = cfg.pc.c * physical_time;
        for (size_t s = 0; s < cfg.plasmas.size(); ++s) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[s];
            Plasma& pl = plasmas[s];
            const int nppc = P.ppc[0] * P.ppc[1];
            const double scale = nppc <= 0 ? 0. : (cfg.normalized_units ? 1. / nppc : dx * dy * dz / nppc);
            int ilo = 0, ihi = nx - 1, jlo = 0, jhi = ny - 1;
            double xo = 0, yo = 0;
            if (P.prevent_centered_particle) {
                if (nx % 2 == 1 && P.ppc[0] % 2 == 1) { ilo = 1; ihi = nx - 1; xo = -0.5; }
                if (ny % 2 == 1 && P.ppc[1] % 2 == 1) { jlo = 1; jhi = ny - 1; yo = -0.5; }
            }
            if (P.radius < 1e299) {
                ilo = std::max(ilo, (int)std::round((-P.radius - cfg.prob_lo[0]) / dx - 2));
                jlo = std::max(jlo, (int)std::round((-P.radius - cfg.prob_lo[1]) / dy - 2));
                ihi = std::min(ihi, (int)std::round((P.radius - cfg.prob_lo[0]) / dx + 2));
                jhi = std::min(jhi, (int)std::round((P.radius - cfg.prob_lo[1]) / dy + 2));
            }
            const hpq::Philox rng(hpq::plasma_thermal_seed((uint64_t)(cfg.has_random_seed ? cfg.random_seed : 0), (int)s));
            for (int ip = 0; ip < nppc; ++ip) {
                const int ixp = ip % P.ppc[0], iyp = ip / P.ppc[0];
                const double r0 = (0.5 + ixp) / P.ppc[0], r1 = (0.5 + iyp) / P.ppc[1];
                for (int j = jlo; j <= jhi; ++j)
                    for (int i = ilo; i <= ihi; ++i) {
                        const double x = cfg.prob_lo[0] + (i + r0 + xo) * dx;
                        const double y = cfg.prob_lo[1] + (j + r1 + yo) * dy;
                        const double rsq = x * x + y * y;
                        double v[3] = {x, y, c_t};
                        if (x >= cfg.particle_hi[0] || x < cfg.particle_lo[0] || y >= cfg.particle_hi[1] ||
                            y < cfg.particle_lo[1] || rsq > P.radius * P.radius ||
                            rsq < P.hollow_core_radius * P.hollow_core_radius || P.density.eval(v) <= P.min_density)
                            continue;
                        // get_gaussian_random_momentum (ParticleUtil.H:113-124) from the
                        // counter-based stream shared with the library (rng.hpp); the counter is
                        // the particle's index in this lattice order and the step
                        double u[3] = {P.u_mean[0], P.u_mean[1], P.u_mean[2]};
                        if (P.thermal) hpq::plasma_thermal_u(rng, cur_step, (long long)pl.x.size(), P.u_mean, P.u_std, u);
                        const double u0 = u[0], u1 = u[1], u2 = u[2];
                        pl.x.push_back(x); pl.y.push_back(y);
                        pl.w.push_back(P.density.eval(v) * scale);
                        pl.ux.push_back(u0 * cfg.pc.c); pl.uy.push_back(u1 * cfg.pc.c);
                        const double psi = std::sqrt(1. + u0 * u0 + u1 * u1 + u2 * u2) - u2;
                        pl.psi.push_back(psi);
                        pl.x_prev.push_back(x); pl.y_prev.push_back(y);
                        pl.ux_h.push_back(u0 * cfg.pc.c); pl.uy_h.push_back(u1 * cfg.pc.c);
                        pl.psi_h.push_back(psi);
                        pl.valid.push_back(1);
                    }
            }
        }
    }

    // -------------------------------------------------------------- threaded deposition
    // The deposits run over the particles grouped in bands of kBand cell rows (by the row of
    // the particle's position). A deposit stencil reaches at most 3 rows from that row, so the
    // bands of one parity touch disjoint rows: the even bands deposit in parallel, then the odd
    // ones. Within a band the particles keep their order, so the sums do not depend on the number
    // of threads. (The reference's OpenMP build tiles its deposition in the same spirit,
    // PlasmaDepositCurrent.cpp:90-130.)
    static constexpr int kBand = 8;
    template <class Body>
    void for_particles_banded(const Plasma& pl, const std::vector<double>& ypos, Body body) {
        const size_t n = pl.n();
        const int nb = (gr.ny + 2 * gr.g) / kBand + 2;
        std::vector<int> band(n);
        std::vector<size_t> start(nb + 1, 0);
        for (size_t ip = 0; ip < n; ++ip) {
            const int row = (int)std::floor((ypos[ip] - yoff) * dyi) + gr.g;
            band[ip] = std::min(std::max(row / kBand, 0), nb - 1);
            ++start[band[ip] + 1];
        }
        for (int b = 0; b < nb; ++b) start[b + 1] += start[b];
        std::vector<size_t> idx(n), fill(start.begin(), start.end() - 1);
        for (size_t ip = 0; ip < n; ++ip) idx[fill[band[ip]]++] = ip;
        for (int parity = 0; parity < 2; ++parity) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int b = parity; b < nb; b += 2)
                for (size_t k = start[b]; k < start[b + 1]; ++k) body(idx[k]);
        }
    }

    // -------------------------------------------------------------- plasma deposition
    // PlasmaDepositCurrent.cpp:22-259, order 2. `which`: 0 = This, 1 = Next, 2 = ions.
    void plasma_deposit(int which, bool jxjy, bool jz, bool rho, bool chi, bool rhomjz) {
        for (size_t s = 0; s < plasmas.size(); ++s) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[s];
            Plasma& pl = plasmas[s];
            const double charge = (which == 2) ? -P.charge : P.charge;
            const double invvol = cfg.normalized_units ? dx * dy * dxi * dyi : dxi * dyi * dzi;
            const double clight = cfg.pc.c, clightinv = 1.0 / cfg.pc.c;
            const double charge_invvol = charge * invvol;
            const double charge_mu0_mass_ratio = charge * cfg.pc.mu0 / P.mass;
            Field *Fjx = nullptr, *Fjy = nullptr, *Fjz = nullptr, *Frho = nullptr, *Fchi = nullptr, *Frm = nullptr;
            if (which == 2) { Frm = &f("Ions.rhomjz"); }
            else if (which == 3) { Fjx = &f("Salame.jx"); Fjy = &f("Salame.jy"); }
            else if (cfg.explicit_solver) {
                if (which == 0) {
                    if (jxjy) { Fjx = &f("jx"); Fjy = &f("jy"); }
                    if (rho) Frho = &f("rho");
                    if (chi) Fchi = &f("chi");
                    if (rhomjz) Frm = &f("rhomjz");
                }
            } else {
                if (which == 0) {
                    if (jxjy) { Fjx = &f("jx"); Fjy = &f("jy"); }
                    if (jz) Fjz = &f("jz");
                    if (rho) Frho = &f("rho");
                    if (rhomjz) Frm = &f("rhomjz");
                } else {
                    if (jxjy) { Fjx = &f("Next.jx"); Fjy = &f("Next.jy"); }
                }
            }
            for_particles_banded(pl, pl.y, [&](size_t ip) {
                if (!pl.valid[ip]) return;
                const double psi_inv = 1.0 / pl.psi[ip];
                const double xp = pl.x[ip], yp = pl.y[ip];
                const double vx_c = pl.ux[ip] * psi_inv;
                const double vy_c = pl.uy[ip] * psi_inv;
                const double q_invvol = charge_invvol * pl.w[ip];
                const double q_mu0_mass_ratio = charge_mu0_mass_ratio;
                const double xmid = (xp - xoff) * dxi;
                const double ymid = (yp - yoff) * dyi;
                const double gamma_psi = 0.5 * ((1.0 + 0.5 * 0.0) * psi_inv * psi_inv +
                                                vx_c * vx_c * clightinv * clightinv +
                                                vy_c * vy_c * clightinv * clightinv + 1.0);
                if (gamma_psi < 0.0 || gamma_psi > P.max_qsa_weighting_factor || psi_inv < 0.0) {
                    pl.w[ip] = 0.0;
                    pl.valid[ip] = 0;
                    return;
                }
                const int ord = cfg.depos_order_xy;
                for (int iy = 0; iy <= ord; ++iy)
                    for (int ix = 0; ix <= ord; ++ix) {
                        Shape sx = shapeN(ord, xmid, ix), sy = shapeN(ord, ymid, iy);
                        const int i = sx.cell, j = sy.cell;
                        const double cd = q_invvol * sx.s * sy.s;
                        if (Fjx) { (*Fjx)(i, j) += cd * vx_c; (*Fjy)(i, j) += cd * vy_c; }
                        if (Fjz) (*Fjz)(i, j) += cd * (gamma_psi - 1.0) * clight;
                        if (Frho) (*Frho)(i, j) += cd * gamma_psi;
                        if (Fchi) (*Fchi)(i, j) += cd * q_mu0_mass_ratio * psi_inv;
                        if (Frm) (*Frm)(i, j) += cd;
                    }
            });
        }
    }

    // -------------------------------------------------------------- explicit deposition
    // ExplicitDeposition.cpp:20-265 (no laser): Sx, Sy += plasma contribution
    void explicit_deposit() {
        const int dt = cfg.depos_derivative_type;
        const int ord = cfg.depos_order_xy;
        const int ns = dshape_points(dt, ord) - 1;  // stencil extent - 1
        Field& Sx = f("Sx"); Field& Sy = f("Sy");
        const Field& Bz = f("Bz"); const Field& Ez = f("Ez");
        const Field& ExmBy = f("ExmBy"); const Field& EypBx = f("EypBx");
        for (size_t s = 0; s < plasmas.size(); ++s) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[s];
            Plasma& pl = plasmas[s];
            const double invvol = cfg.normalized_units ? dx * dy * dxi * dyi : dxi * dyi * dzi;
            const double a_clight = cfg.pc.c, clight_inv = 1. / cfg.pc.c;
            const double charge_invvol_mu0 = P.charge * invvol * cfg.pc.mu0;
            const double q_mass_ratio = P.charge / P.mass;
            for_particles_banded(pl, pl.y, [&](size_t ip) {
                if (!pl.valid[ip]) return;
                const double psi_inv = 1. / pl.psi[ip];
                const double xp = pl.x[ip], yp = pl.y[ip];
                const double vx = pl.ux[ip] * psi_inv * clight_inv;
                const double vy = pl.uy[ip] * psi_inv * clight_inv;
                const double cdm = charge_invvol_mu0 * pl.w[ip];
                const double xmid = (xp - xoff) * dxi, ymid = (yp - yoff) * dyi;
                const double gamma_psi = 0.5 * ((1. + 0.5 * 0.0) * psi_inv * psi_inv + vx * vx + vy * vy + 1.);
                DShape shx[6], shy[6];
                for (int k = 0; k <= ns; ++k) { shx[k] = dshapeN(dt, ord, xmid, k); shy[k] = dshapeN(dt, ord, ymid, k); }
                for (int iy = 0; iy <= ns; ++iy)
                    for (int ix = 0; ix <= ns; ++ix) {
                        if (dt == 2 && (ix == 0 || ix == ns) && (iy == 0 || iy == ns)) continue;
                        const DShape& sy = shy[iy];
                        const DShape& sx = shx[ix];
                        const int i = sx.cell, j = sy.cell;
                        const double Bz_v = Bz(i, j), Ez_v = Ez(i, j), ExmBy_v = ExmBy(i, j), EypBx_v = EypBx(i, j);
                        Sy(i, j) += cdm * (-sx.s * sy.s * (-Bz_v * vx + (Ez_v * vy + ExmBy_v * (-vx * vy) + EypBx_v * (gamma_psi - vy * vy)) * clight_inv - 0.25 * 0.0 * q_mass_ratio * psi_inv) * q_mass_ratio * psi_inv +
                                           (-sx.ds * sy.s * dxi * (-vx * vy) - sx.s * sy.ds * dyi * (gamma_psi - vy * vy - 1.)) * a_clight);
                        Sx(i, j) += cdm * (+sx.s * sy.s * (+Bz_v * vy + (Ez_v * vx + ExmBy_v * (gamma_psi - vx * vx) + EypBx_v * (-vx * vy)) * clight_inv - 0.25 * 0.0 * q_mass_ratio * psi_inv) * q_mass_ratio * psi_inv +
                                           (+sx.ds * sy.s * dxi * (gamma_psi - vx * vx - 1.) + sx.s * sy.ds * dyi * (-vx * vy)) * a_clight);
                    }
            });
        }
    }

    // -------------------------------------------------------------- beam deposition
    // BeamDepositCurrent.cpp:21-196: deposits the non-slipped particles of a beam slice
    void beam_deposit(const BeamSlice& bs, double q, Field* jx, Field* jy, Field* jz, Field* rmj) {
        const double invvol = cfg.normalized_units ? 1.0 : dxi * dyi * dzi;
        const double clightinv = 1.0 / cfg.pc.c, clightsq = 1.0 / (cfg.pc.c * cfg.pc.c);
        for (size_t ip = 0; ip < bs.num_nonslipped; ++ip) {
            const BeamParticle& p = bs.p[ip];
            if (!p.valid) continue;
            const double gaminv = 1.0 / std::sqrt(1.0 + p.ux * p.ux * clightsq + p.uy * p.uy * clightsq + p.uz * p.uz * clightsq);
            const double wq = q * p.w * invvol;
            const double vx = p.ux * gaminv, vy = p.uy * gaminv, vz = p.uz * gaminv;
            const double wqx = wq * vx, wqy = wq * vy, wqz = wq * vz, wqr = wq * (1. - vz * clightinv);
            const double xmid = (p.x - xoff) * dxi, ymid = (p.y - yoff) * dyi;
            const int ord = cfg.depos_order_xy;
            for (int iy = 0; iy <= ord; ++iy)
                for (int ix = 0; ix <= ord; ++ix) {
                    Shape sx = shapeN(ord, xmid, ix), sy = shapeN(ord, ymid, iy);
                    const double S = sx.s * sy.s;
                    const int i = sx.cell, j = sy.cell;
                    if (jx) { (*jx)(i, j) += S * wqx; (*jy)(i, j) += S * wqy; }
                    if (jz) (*jz)(i, j) += S * wqz;
                    if (rmj) (*rmj)(i, j) += S * wqr;
                }
        }
    }

    // -------------------------------------------------------------- field solves
    // Fields.cpp:840-957: Psi, Ez, Bz Poisson solves and ExmBy/EypBx = -grad Psi
    void solve_psi_ez_bz() {
        const hpq::PhysConst& pc = cfg.pc;
        if (cfg.explicit_solver && cfg.do_beam_jz_minus_rho) {
            Field& r = f("rhomjz"); const Field& b = f("rhomjz_beam");
            for (size_t k = 0; k < r.a.size(); ++k) r.a[k] += b.a[k];
        }
        const Field& rm = f("rhomjz");
        const Field& jx = f("jx");
        const Field& jy = f("jy");
        std::vector<double> st((size_t)nx * ny);
        auto solve_into = [&](Field& out) {
            dst.solve(st);
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) out(i, j) = st[(size_t)j * nx + i];
        };
        const double hx = 0.5 * dxi, hy = 0.5 * dyi;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) st[(size_t)j * nx + i] = -1. / pc.ep0 * rm(i, j);
        solve_into(f("Psi"));
        const double fe = 1. / (pc.ep0 * pc.c);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                st[(size_t)j * nx + i] = fe * ((jx(i + 1, j) - jx(i - 1, j)) * hx) + fe * ((jy(i, j + 1) - jy(i, j - 1)) * hy);
        solve_into(f("Ez"));
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                st[(size_t)j * nx + i] = pc.mu0 * ((jx(i, j + 1) - jx(i, j - 1)) * hy) + (-pc.mu0) * ((jy(i + 1, j) - jy(i - 1, j)) * hx);
        solve_into(f("Bz"));
        const Field& Psi = f("Psi");
        Field& Ex = f("ExmBy"); Field& Ey = f("EypBx");
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i) {
                Ex(i, j) = -(Psi(i + 1, j) - Psi(i - 1, j)) * hx;
                Ey(i, j) = -(Psi(i, j + 1) - Psi(i, j - 1)) * hy;
            }
    }

    // Fields.cpp:1008-1078: PC Bx, By from jz (This) and d/dzeta of jx, jy (Previous, Next)
    void solve_bxby_pc() {
        const hpq::PhysConst& pc = cfg.pc;
        const Field& jz = f("jz");
        const Field& pjx = f("Prev.jx"); const Field& pjy = f("Prev.jy");
        const Field& njx = f("Next.jx"); const Field& njy = f("Next.jy");
        std::vector<double> st((size_t)nx * ny);
        const double hx = 0.5 * dxi, hy = 0.5 * dyi, hz = 0.5 * dzi;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                st[(size_t)j * nx + i] = -pc.mu0 * ((jz(i, j + 1) - jz(i, j - 1)) * hy) + pc.mu0 * ((pjy(i, j) - njy(i, j)) * hz);
        dst.solve(st);
        Field& bx = f("PCIter.Bx");
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) bx(i, j) = st[(size_t)j * nx + i];
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                st[(size_t)j * nx + i] = pc.mu0 * ((jz(i + 1, j) - jz(i - 1, j)) * hx) + (-pc.mu0) * ((pjx(i, j) - njx(i, j)) * hz);
        dst.solve(st);
        Field& by = f("PCIter.By");
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) by(i, j) = st[(size_t)j * nx + i];
    }

    // Hipace.cpp:744-790
    void init_sxsy_with_beam() {
        const double mu0 = cfg.pc.mu0;
        const Field& jzb = f("jz_beam");
        const Field& pjx = f("Prev.jx_beam"); const Field& pjy = f("Prev.jy_beam");
        const Field& njx = f("Next.jx_beam"); const Field& njy = f("Next.jy_beam");
        Field& Sx = f("Sx"); Field& Sy = f("Sy");
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double dx_jzb = (jzb(i + 1, j) - jzb(i - 1, j)) / (2. * dx);
                const double dy_jzb = (jzb(i, j + 1) - jzb(i, j - 1)) / (2. * dy);
                const double dz_jxb = (pjx(i, j) - njx(i, j)) / (2. * dz);
                const double dz_jyb = (pjy(i, j) - njy(i, j)) / (2. * dz);
                Sy(i, j) = mu0 * (-dy_jzb + dz_jyb);
                Sx(i, j) = -mu0 * (-dx_jzb + dz_jxb);
            }
    }

    // -------------------------------------------------------------- plasma push
    // PlasmaParticleAdvance.cpp:29-217 with doGatherShapeN (FieldGather.H:45-96, derivative
    // type 1) and PlasmaMomentumPush (PushPlasmaParticles.H:39-75); leapfrog, 4+2 Taylor substeps.
    struct Deriv { double ux, uy, psi; };
    static inline Deriv mom(double ux, double uy, double psi_inv, double ExmBy, double EypBx, double Ez,
                            double Bxc, double Byc, double Bz, double ci, double qmc) {
        const double gamma_psi = 0.5 * psi_inv * psi_inv * (1.0 + 0.0 + ux * ux * (ci * ci) + uy * uy * (ci * ci)) + 0.5;
        return {qmc * (gamma_psi * ExmBy + Byc + (uy * Bz) * psi_inv) - 0.0 * psi_inv,
                qmc * (gamma_psi * EypBx - Bxc - (ux * Bz) * psi_inv) - 0.0 * psi_inv,
                qmc * ci * ((ux * ExmBy + uy * EypBx) * ci * psi_inv - Ez)};
    }
    // the same expression evaluated on dual numbers (value, epsilon) (DualNumbers.H)
    struct Dual { double v, e; };
    static inline Dual dadd(Dual a, Dual b) { return {a.v + b.v, a.e + b.e}; }
    static inline Dual dsub(Dual a, Dual b) { return {a.v - b.v, a.e - b.e}; }
    static inline Dual dmul(Dual a, Dual b) { return {a.v * b.v, a.e * b.v + a.v * b.e}; }
    static inline void mom_dual(Dual ux, Dual uy, Dual pi, double ExmBy, double EypBx, double Ez, double Bxc,
                                double Byc, double Bz, double ci, double qmc, Dual& dux, Dual& duy, Dual& dpsi) {
        const Dual c2{ci * ci, 0};
        Dual t = dadd(dadd(dadd(Dual{1.0, 0}, Dual{0.0, 0}), dmul(dmul(ux, ux), c2)), dmul(dmul(uy, uy), c2));
        Dual gp = dadd(dmul(dmul(dmul(Dual{0.5, 0}, pi), pi), t), Dual{0.5, 0});
        dux = dsub(dmul(Dual{qmc, 0}, dadd(dadd(dmul(gp, Dual{ExmBy, 0}), Dual{Byc, 0}), dmul(dmul(uy, Dual{Bz, 0}), pi))), dmul(Dual{0.0, 0}, pi));
        duy = dsub(dmul(Dual{qmc, 0}, dsub(dsub(dmul(gp, Dual{EypBx, 0}), Dual{Bxc, 0}), dmul(dmul(ux, Dual{Bz, 0}), pi))), dmul(Dual{0.0, 0}, pi));
        dpsi = dmul(dmul(Dual{qmc, 0}, Dual{ci, 0}), dsub(dmul(dmul(dadd(dmul(ux, Dual{ExmBy, 0}), dmul(uy, Dual{EypBx, 0})), Dual{ci, 0}), pi), Dual{Ez, 0}));
    }

    // the gathered planes, looked up once (std::map nodes do not move)
    const Field *g_psi = nullptr, *g_ez = nullptr, *g_bx = nullptr, *g_by = nullptr, *g_bz = nullptr;
    void gather(double xp, double yp, double& ExmBy, double& EypBx, double& Ez, double& Bx, double& By, double& Bz) {
        const Field& Psi = *g_psi; const Field& FEz = *g_ez;
        const Field& FBx = *g_bx; const Field& FBy = *g_by; const Field& FBz = *g_bz;
        const double x = (xp - xoff) * dxi, y = (yp - yoff) * dyi;
        const int ord = cfg.depos_order_xy;
        DShape shx[5], shy[5];
        for (int k = 0; k <= ord + 1; k++) { shx[k] = dshapeN(1, ord, x, k); shy[k] = dshapeN(1, ord, y, k); }
        for (int iy = 0; iy <= ord + 1; iy++)
            for (int ix = 0; ix <= ord + 1; ix++) {
                const DShape& sy = shy[iy];
                const DShape& sx = shx[ix];
                const int i = sx.cell, j = sy.cell;
                ExmBy += (sx.ds * sy.s) * Psi(i, j) * dxi;
                EypBx += (sx.s * sy.ds) * Psi(i, j) * dyi;
                Ez += (sx.s * sy.s) * FEz(i, j);
                Bx += (sx.s * sy.s) * FBx(i, j);
                By += (sx.s * sy.s) * FBy(i, j);
                Bz += (sx.s * sy.s) * FBz(i, j);
            }
    }

    void plasma_push(bool temp) {
        for (size_t s = 0; s < plasmas.size(); ++s) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[s];
            Plasma& pl = plasmas[s];
            const double clight = cfg.pc.c, ci = 1. / cfg.pc.c;
            const double qmc = P.charge / (P.mass * cfg.pc.c);
            const int nsubc = P.n_subcycles;
            const double dzs = dz / nsubc;
#pragma omp parallel for schedule(static)
            for (long long ip = 0; ip < (long long)pl.n(); ++ip) {
                if (!pl.valid[ip]) continue;
                double ExmBy = 0, EypBx = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
                for (int isc = 0; isc < nsubc; ++isc) {
                    double xp = pl.x_prev[ip], yp = pl.y_prev[ip];
                    ExmBy = 0; EypBx = 0; Ez = 0; Bx = 0; By = 0; Bz = 0;
                    gather(xp, yp, ExmBy, EypBx, Ez, Bx, By, Bz);
                    Bx *= clight; By *= clight;
                    const int nsub = 4;
                    const double sdz = dzs / nsub;
                    double ux = pl.ux_h[ip], uy = pl.uy_h[ip], psi = pl.psi_h[ip];
                    auto substep = [&]() {
                        const double psi_inv = 1. / psi;
                        Deriv d = mom(ux, uy, psi_inv, ExmBy, EypBx, Ez, Bx, By, Bz, ci, qmc);
                        Dual dux, duy, dps;
                        mom_dual({ux, d.ux}, {uy, d.uy}, {psi_inv, -psi_inv * psi_inv * d.psi}, ExmBy, EypBx, Ez, Bx, By, Bz, ci, qmc, dux, duy, dps);
                        ux += sdz * d.ux + 0.5 * sdz * sdz * dux.e;
                        uy += sdz * d.uy + 0.5 * sdz * sdz * duy.e;
                        psi += sdz * d.psi + 0.5 * sdz * sdz * dps.e;
                    };
                    for (int k = 0; k < nsub; ++k) substep();
                    xp += dzs * ci * (ux * (1. / psi));
                    yp += dzs * ci * (uy * (1. / psi));
                    if (!enforce_bc(xp, yp, ux, uy)) { pl.w[ip] = 0; pl.valid[ip] = 0; break; }
                    pl.x[ip] = xp; pl.y[ip] = yp;
                    if (!temp) {
                        pl.ux_h[ip] = ux; pl.uy_h[ip] = uy; pl.psi_h[ip] = psi;
                        pl.x_prev[ip] = xp; pl.y_prev[ip] = yp;
                    }
                    for (int k = 0; k < nsub / 2; ++k) substep();
                    pl.ux[ip] = ux; pl.uy[ip] = uy; pl.psi[ip] = psi;
                }
            }
        }
    }

    // -------------------------------------------------------------- beam push
    // BeamParticleAdvance.cpp:19-336 (no external fields, spin or radiation reaction)
    void beam_push(int b, BeamSlice& bs, int islice) {
        const hpq::BeamSpecies& B = cfg.beams[b];
        const double dtb = step_dt / B.n_subcycles;
        const double clight = cfg.pc.c, inv_c2 = 1. / (cfg.pc.c * cfg.pc.c);
        const double cmr = B.charge / B.mass;
        const double min_z = cfg.prob_lo[2] + (islice - 0) * dz;
#pragma omp parallel for schedule(static) if (bs.p.size() > 2048)
        for (size_t ip = 0; ip < bs.p.size(); ++ip) {
            BeamParticle& p = bs.p[ip];
            if (!p.valid) continue;
            double xp = p.x, yp = p.y, zp = p.z, ux = p.ux, uy = p.uy, uz = p.uz;
            int i = p.nsub;
            bool absorbed = false;
            for (; i < B.n_subcycles; i++) {
                if (zp < min_z) break;
                const double gammap_inv = 1. / std::sqrt(1. + (ux * ux + uy * uy + uz * uz) * inv_c2);
                xp += dtb * 0.5 * ux * gammap_inv;
                yp += dtb * 0.5 * uy * gammap_inv;
                if (!enforce_bc(xp, yp, ux, uy)) { absorbed = true; break; }
                double ExmBy = 0, EypBx = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
                gather(xp, yp, ExmBy, EypBx, Ez, Bx, By, Bz);
                if (B.use_external) {
                    // ApplyExternalField (ExternalFields.H:29-56), at the step's start time
                    const double a[4] = {xp, yp, zp, physical_time};
                    double f[6];
                    for (int k = 0; k < 6; ++k) f[k] = B.external[k].eval(a);
                    ExmBy += f[0] - clight * f[4];
                    EypBx += f[1] + clight * f[3];
                    Ez += f[2];
                    Bx += f[3];
                    By += f[4];
                    Bz += f[5];
                }
                const double ux_next = ux + dtb * cmr * (ExmBy + (clight - uz * gammap_inv) * By + uy * gammap_inv * Bz);
                const double uy_next = uy + dtb * cmr * (EypBx + (uz * gammap_inv - clight) * Bx - ux * gammap_inv * Bz);
                const double uxi = (ux_next + ux) * 0.5, uyi = (uy_next + uy) * 0.5;
                const double uzi = uz + dtb * 0.5 * cmr * Ez;
                const double gii = 1. / std::sqrt(1. + (uxi * uxi + uyi * uyi + uzi * uzi) * inv_c2);
                const double uz_next = uz + dtb * cmr * (Ez + (uxi * By - uyi * Bx) * gii);
                const double gni = 1. / std::sqrt(1. + (ux_next * ux_next + uy_next * uy_next + uz_next * uz_next) * inv_c2);
                xp += dtb * 0.5 * ux_next * gni;
                yp += dtb * 0.5 * uy_next * gni;
                if (B.do_z_push) zp += dtb * (uz_next * gni - clight);
                ux = ux_next; uy = uy_next; uz = uz_next;
            }
            if (absorbed || !enforce_bc(xp, yp, ux, uy)) { p.w = 0; p.valid = false; continue; }
            p.x = xp; p.y = yp; p.z = zp; p.nsub = i;
            p.ux = ux; p.uy = uy; p.uz = uz;
        }
    }

    // SliceSort.cpp:13-64: drop invalid particles, keep z >= min_z on this slice (stable), move
    // the rest to the next slice behind the non-slipped ones there
    void shift_slipped(int b, int islice) {
        BeamSlice& T = bthis[b];
        BeamSlice& N = bnext[b];
        const double min_z = cfg.prob_lo[2] + islice * dz;
        std::vector<BeamParticle> stay, slip;
        for (auto& p : T.p) {
            if (!p.valid) continue;
            if (p.z >= min_z) stay.push_back(p); else slip.push_back(p);
        }
        T.p = stay;
        T.num_nonslipped = stay.size();
        if (!slip.empty()) {
            N.p.resize(N.num_nonslipped);
            for (auto& p : slip) N.p.push_back(p);
        }
    }

    void load_beam_slice(int b, int islice, BeamSlice& dst_slice) {
        dst_slice = store[b][islice];
        for (auto& p : dst_slice.p) p.nsub = 0;
        dst_slice.num_nonslipped = dst_slice.p.size();
    }

    // -------------------------------------------------------------- PC helpers
    double rel_b_error(const char* bx, const char* by, const char* bxi, const char* byi) {
        const Field& Bx = f(bx); const Field& By = f(by);
        const Field& Bxi = f(bxi); const Field& Byi = f(byi);
        double nb = 0, nd = 0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                nb += std::sqrt(Bx(i, j) * Bx(i, j) + By(i, j) * By(i, j));
                nd += std::sqrt((Bx(i, j) - Bxi(i, j)) * (Bx(i, j) - Bxi(i, j)) + (By(i, j) - Byi(i, j)) * (By(i, j) - Byi(i, j)));
            }
        return nb > 0 ? nd / nb : 0.0;
    }
    static void lincomb(Field& dst, double a, const Field& x, double b, const Field& y) {
        for (size_t k = 0; k < dst.a.size(); ++k) dst.a[k] = a * x.a[k] + b * y.a[k];
    }
    static void copy(Field& dst, const Field& src) { dst.a = src.a; }

    // Hipace.cpp:935-1031
    void pc_loop(int islice) {
        (void)islice;
        double err_prev = 1.0;
        double err = rel_b_error("Prev.Bx", "Prev.By", "PCPrevIter.Bx", "PCPrevIter.By");
        // InitialBfieldGuess (Fields.cpp:1149-1171)
        const double tol = cfg.predcorr_B_error_tolerance;
        const double mix = std::exp(-0.5 * std::pow(err / (2.5 * tol), 2));
        lincomb(f("Bx"), 1. + mix, f("Prev.Bx"), -mix, f("PCPrevIter.Bx"));
        lincomb(f("By"), 1. + mix, f("Prev.By"), -mix, f("PCPrevIter.By"));
        f("PCIter.Bx").zero(); f("PCIter.By").zero();
        copy(f("PCPrevIter.Bx"), f("Bx")); copy(f("PCPrevIter.By"), f("By"));
        int it = 0;
        err = 1.0;
        while (err > tol && it < cfg.predcorr_max_iterations) {
            it++;
            plasma_push(true);
            plasma_deposit(1, true, false, false, false, false);
            for (size_t b = 0; b < cfg.beams.size(); ++b)
                if (cfg.do_beam_jx_jy_deposition)
                    beam_deposit(bnext[b], cfg.beams[b].charge, &f("Next.jx"), &f("Next.jy"), nullptr, nullptr);
            solve_bxby_pc();
            err = rel_b_error("Bx", "By", "PCIter.Bx", "PCIter.By");
            if (it == 1) err_prev = err;
            // MixAndShiftBfields (Fields.cpp:1173-1226)
            double wi, wp;
            if (err != 0. || err_prev != 0.) { wi = err_prev / (err + err_prev); wp = err / (err + err_prev); }
            else { wi = 0.5; wp = 0.5; }
            lincomb(f("PCPrevIter.Bx"), wi, f("PCIter.Bx"), wp, f("PCPrevIter.Bx"));
            lincomb(f("PCPrevIter.By"), wi, f("PCIter.By"), wp, f("PCPrevIter.By"));
            const double a = cfg.predcorr_B_mixing_factor;
            lincomb(f("Bx"), 1. - a, f("Bx"), a, f("PCPrevIter.Bx"));
            lincomb(f("By"), 1. - a, f("By"), a, f("PCPrevIter.By"));
            copy(f("PCPrevIter.Bx"), f("PCIter.Bx")); copy(f("PCPrevIter.By"), f("PCIter.By"));
            f("Next.jx").zero(); f("Next.jy").zero();
            err_prev = err;
        }
        pc_errors.push_back(err);
    }

    // -------------------------------------------------------------- one slice
    // Hipace::SolveOneSlice (Hipace.cpp:556-728), level 0 only
    // PlasmaParticleContainer::ReorderParticles (PlasmaParticleContainer.cpp:197-208; the CPU
    // build's SortParticlesByCell): a stable sort of the particles by the cell (index type 0) or
    // nearest node (1) they sit in. Cell centres sit at integer t = (x - xoff) / dx, so the cell is
    // floor(t + 1/2) in [0, n-1], the node floor(t + 1) in [0, n]; key = j (nx + 1) + i.
    void reorder_plasma(int s) {
        Plasma& pl = plasmas[s];
        const hpq::PlasmaSpecies& P = cfg.plasmas[s];
        const size_t n = pl.n();
        auto bin = [](double t, int node, int nc) {
            const double f = std::floor(t + (node ? 1.0 : 0.5));
            const int hi = node ? nc : nc - 1;
            return f < 0 ? 0 : (f > hi ? hi : (int)f);
        };
        std::vector<long long> key(n);
        for (size_t i = 0; i < n; ++i)
            key[i] = (long long)bin((pl.y[i] - yoff) * dyi, P.reorder_idx_type[1], ny) * (nx + 1) +
                     bin((pl.x[i] - xoff) * dxi, P.reorder_idx_type[0], nx);
        std::vector<size_t> perm(n);
        for (size_t i = 0; i < n; ++i) perm[i] = i;
        std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
        for (auto* v : {&pl.x, &pl.y, &pl.w, &pl.ux, &pl.uy, &pl.psi, &pl.x_prev, &pl.y_prev, &pl.ux_h, &pl.uy_h, &pl.psi_h}) {
            std::vector<double> t(n);
            for (size_t k = 0; k < n; ++k) t[k] = (*v)[perm[k]];
            v->swap(t);
        }
        std::vector<uint8_t> t(n);
        for (size_t k = 0; k < n; ++k) t[k] = pl.valid[perm[k]];
        pl.valid.swap(t);
    }

    void solve_one_slice(int islice, int step) {
        const bool ex = cfg.explicit_solver;
        // ReorderParticles(islice) at the start of SolveOneSlice (Hipace.cpp:594-595)
        for (size_t s = 0; s < plasmas.size(); ++s) {
            const int period = cfg.plasmas[s].reorder_period;
            if (period > 0 && islice % period == 0) reorder_plasma((int)s);
        }
        if (islice == nz - 1)
            for (size_t b = 0; b < cfg.beams.size(); ++b) load_beam_slice((int)b, islice, bthis[b]);
        // InitializeSlices (Fields.cpp:535-586)
        if (ex) {
            for (auto n : {"chi", "Sy", "Sx", "ExmBy", "EypBx", "jz_beam", "rhomjz", "Next.jx_beam", "Next.jy_beam", "rhomjz_beam"}) f(n).zero();
        } else {
            for (auto n : {"ExmBy", "EypBx", "jx", "jy", "jz", "rhomjz"}) f(n).zero();
        }
        if (cfg.deposit_rho) f("rho").zero();
        // deposition on This
        if (ex) {
            plasma_deposit(0, true, false, cfg.deposit_rho, true, true);
            // SALAME beams deposit only jz in step 0 (MultiBeam.cpp:50-56)
            for (size_t b = 0; b < cfg.beams.size(); ++b)
                beam_deposit(bthis[b], cfg.beams[b].charge, nullptr, nullptr, &f("jz_beam"),
                             cfg.do_beam_jz_minus_rho && !is_salame(b, step) ? &f("rhomjz_beam") : nullptr);
        } else {
            plasma_deposit(0, true, true, cfg.deposit_rho, false, true);
            for (size_t b = 0; b < cfg.beams.size(); ++b)
                beam_deposit(bthis[b], cfg.beams[b].charge,
                             cfg.do_beam_jx_jy_deposition ? &f("jx") : nullptr,
                             cfg.do_beam_jx_jy_deposition ? &f("jy") : nullptr, &f("jz"),
                             cfg.do_beam_jz_minus_rho ? &f("rhomjz") : nullptr);
        }
        // AddRhoIons (Fields.cpp:606-615)
        if (cfg.any_neutralize_background()) {
            Field& r = f("rhomjz"); const Field& ions = f("Ions.rhomjz");
            for (size_t k = 0; k < r.a.size(); ++k) r.a[k] += ions.a[k];
            if (cfg.deposit_rho) { Field& rr = f("rho"); for (size_t k = 0; k < rr.a.size(); ++k) rr.a[k] += ions.a[k]; }
        }
        solve_psi_ez_bz();
        if (islice - 1 >= 0)
            for (size_t b = 0; b < cfg.beams.size(); ++b) load_beam_slice((int)b, islice - 1, bnext[b]);
        if (ex) {
            for (size_t b = 0; b < cfg.beams.size(); ++b)
                if (cfg.do_beam_jx_jy_deposition && !is_salame(b, step))
                    beam_deposit(bnext[b], cfg.beams[b].charge, &f("Next.jx_beam"), &f("Next.jy_beam"), nullptr, nullptr);
            init_sxsy_with_beam();
            explicit_deposit();
            int iters = 0;
            const int st = mg.solve(f("Bx"), f("By"), f("Sy"), f("Sx"), f("chi"), cfg.mg_tol_rel, cfg.mg_tol_abs,
                                    cfg.mg_max_iters, &iters);
            mg_iters_total += iters;
            if (st != 0 && mg_status == 0) mg_status = st;
            if (salame_now(step)) salame_module(islice);
        } else {
            pc_loop(islice);
        }
        // in-situ reductions (after SALAME, before the beam push, Hipace.cpp:681-685)
        insitu_compute(islice);
        // diagnostics (after all fields are known, before the pushes)
        for (auto& n : diag_names) {
            auto& d = diag[n];
            const Field& src = f(n.c_str());
            int lo, hi;
            double wlo, whi;
            if (cfg.diag_type == 0) {
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) d[((size_t)islice * ny + j) * nx + i] = src(i, j);
            } else if (cfg.diag_type == 1) {
                hpq::mid_plane(ny, lo, hi, wlo, whi);
                for (int i = 0; i < nx; ++i) d[(size_t)islice * nx + i] = wlo * src(i, lo) + whi * src(i, hi);
            } else {
                hpq::mid_plane(nx, lo, hi, wlo, whi);
                for (int j = 0; j < ny; ++j) d[(size_t)islice * ny + j] = wlo * src(lo, j) + whi * src(hi, j);
            }
        }
        plasma_push(false);
        for (size_t b = 0; b < cfg.beams.size(); ++b) {
            beam_push((int)b, bthis[b], islice);
            shift_slipped((int)b, islice);
            const bool is_last_step = (step == cfg.max_step);
            if (!is_last_step) store[b][islice] = bthis[b];
            else store[b][islice] = bthis[b];  // kept for inspection after the run
            store[b][islice].num_nonslipped = store[b][islice].p.size();
        }
        // ShiftSlices (Fields.cpp:588-604)
        if (ex) {
            copy(f("Prev.jx_beam"), f("jx_beam")); copy(f("Prev.jy_beam"), f("jy_beam"));
            copy(f("jx_beam"), f("Next.jx_beam")); copy(f("jy_beam"), f("Next.jy_beam"));
            copy(f("jx"), f("Next.jx_beam")); copy(f("jy"), f("Next.jy_beam"));
        } else {
            copy(f("PCPrevIter.Bx"), f("Prev.Bx")); copy(f("PCPrevIter.By"), f("Prev.By"));
            copy(f("Prev.Bx"), f("Bx")); copy(f("Prev.By"), f("By"));
            copy(f("Prev.jx"), f("jx")); copy(f("Prev.jy"), f("jy"));
        }
        for (size_t b = 0; b < cfg.beams.size(); ++b) {
            bthis[b] = bnext[b];
            bnext[b].p.clear();
            bnext[b].num_nonslipped = 0;
        }
    }

    // -------------------------------------------------------------- one step
    // Hipace::Evolve per-step body (Hipace.cpp:401-492), one rank, fixed dt shortened to end on
    // max_time (Hipace.cpp:424-435)
    void begin_step(int step) {
        for (auto& kv : F) kv.second.zero();  // ResetAllQuantities
        cur_step = step;
        const hpq::StepTime T = hpq::step_time(physical_time, cfg.dt, cfg.max_time);
        step_dt = T.dt;
        next_time = T.next;
        insitu_beam.resize(cfg.beams.size());
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (insitu_beam_on(b)) insitu_beam[b].assign((size_t)nz * 23, 0.0);
        if (insitu_fields_on()) insitu_fields.assign((size_t)nz * 10, 0.0);
        init_plasmas();
        if (cfg.any_neutralize_background()) {
            // DepositNeutralizingBackground: rhomjz of ions with the opposite charge
            std::vector<hpq::PlasmaSpecies> saved = cfg.plasmas;
            plasma_deposit_ions();
        }
        const size_t plane = cfg.diag_type == 0 ? (size_t)nx * ny : cfg.diag_type == 1 ? (size_t)nx : (size_t)ny;
        for (auto& n : diag_names) diag[n].assign(plane * nz, 0.0);
    }
    void plasma_deposit_ions() {
        // only species with neutralize_background deposit (MultiPlasma.cpp:103-115)
        std::vector<Plasma> saved = plasmas;
        for (size_t s = 0; s < plasmas.size(); ++s)
            if (!cfg.plasmas[s].neutralize_background) plasmas[s].valid.assign(plasmas[s].n(), 0);
        plasma_deposit(2, false, false, false, false, true);
        // the ion deposit may invalidate QSA-violating particles (same test as the plasma)
        for (size_t s = 0; s < plasmas.size(); ++s)
            if (!cfg.plasmas[s].neutralize_background) { plasmas[s].valid = saved[s].valid; plasmas[s].w = saved[s].w; }
    }
    void end_step() { physical_time = next_time; }

    // -------------------------------------------------------------- SALAME (Salame.cpp)
    bool is_salame(size_t b, int step) const { return cfg.beams[b].do_salame && step == 0; }
    // MultiBeam::isSalameNow (MultiBeam.cpp:128-139): step 0 and a SALAME beam has particles in
    // this slice (slipped ones not counted)
    bool salame_now(int step) const {
        if (step != 0) return false;
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (cfg.beams[b].do_salame && bthis[b].num_nonslipped > 0) return true;
        return false;
    }
    int mg_solve_fields(const char* bx, const char* by, const char* sy, const char* sx) {
        int iters = 0;
        const int st = mg.solve(f(bx), f(by), f(sy), f(sx), f("chi"), cfg.mg_tol_rel, cfg.mg_tol_abs, cfg.mg_max_iters, &iters);
        mg_iters_total += iters;
        if (st != 0 && mg_status == 0) mg_status = st;
        return st;
    }
    // Fields::SolvePoissonEz (Fields.cpp:960-1005) on the SALAME slice
    void salame_solve_ez() {
        const Field& jx = f("Salame.jx"); const Field& jy = f("Salame.jy");
        std::vector<double> st((size_t)nx * ny);
        const double hx = 0.5 * dxi, hy = 0.5 * dyi, fe = 1. / (cfg.pc.ep0 * cfg.pc.c);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                st[(size_t)j * nx + i] = fe * ((jx(i + 1, j) - jx(i - 1, j)) * hx) + fe * ((jy(i, j + 1) - jy(i, j - 1)) * hy);
        dst.solve(st);
        Field& ez = f("Salame.Ez");
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) ez(i, j) = st[(size_t)j * nx + i];
    }
    void salame_deposit_jz(Field& jz) {
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (cfg.beams[b].do_salame) beam_deposit(bthis[b], cfg.beams[b].charge, nullptr, nullptr, &jz, nullptr);
    }
    // SalameModule (Salame.cpp:14-185): one level, no grid current
    void salame_module(int islice) {
        const double zoff = cfg.prob_lo[2] + 0.5 * dz;  // GetPosOffset(2, geom, domain)
        // always use the Ez field from before SALAME started (:21-29)
        if (islice + 1 != sal_last) {
            copy(f("Salame.Ez_target"), f("Ez"));
            sal_overloaded = false;
            sal_zeta0 = islice * dz + zoff;
        }
        sal_last = islice;
        // plasma-only Sx, Sy, kept for step 4 (:32-39)
        f("Sy").zero(); f("Sx").zero();
        explicit_deposit();
        copy(f("Salame.Sy_back"), f("Sy")); copy(f("Salame.Sx_back"), f("Sx"));
        for (int iter = 0; iter < cfg.salame_n_iter; ++iter) {
            const int it0 = iter;
            // step 1: Ez of the next slice with the current SALAME weights (:43-76)
            plasma_push(true);
            copy(f("Salame.jx"), f("Next.jx_beam")); copy(f("Salame.jy"), f("Next.jy_beam"));
            plasma_deposit(3, true, false, false, false, false);
            for (auto n : {"Salame.Ez", "Salame.jz_beam", "Salame.Sy", "Salame.Sx", "Salame.Bx", "Salame.By"}) f(n).zero();
            salame_solve_ez();
            copy(f("Salame.Ez_no_salame"), f("Salame.Ez"));
            // step 2: the Ez response to the SALAME beam alone (:78-123)
            salame_deposit_jz(f("Salame.jz_beam"));
            {
                // SalameInitializeSxSyWithBeam (:189-220)
                const Field& jzb = f("Salame.jz_beam");
                Field& Sx = f("Salame.Sx"); Field& Sy = f("Salame.Sy");
                const double dxih = 0.5 * dxi, dyih = 0.5 * dyi, mu0 = cfg.pc.mu0;
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const double dx_jzb = (jzb(i + 1, j) - jzb(i - 1, j)) * dxih;
                        const double dy_jzb = (jzb(i, j + 1) - jzb(i, j - 1)) * dyih;
                        Sy(i, j) = mu0 * (-dy_jzb);
                        Sx(i, j) = -mu0 * (-dx_jzb);
                    }
            }
            mg_solve_fields("Salame.Bx", "Salame.By", "Salame.Sy", "Salame.Sx");
            for (auto n : {"Salame.Ez", "Salame.jx", "Salame.jy"}) f(n).zero();
            if (cfg.salame_do_advance) {
                salame_only_advance();
                plasma_deposit(3, true, false, false, false, false);
            } else {
                // SalameGetJxJyFromBxBy (:223-255)
                const double dzf = 1.5 * dz, mu0_inv = 1. / cfg.pc.mu0;
                const Field& chi = f("chi"); const Field& bx = f("Salame.Bx"); const Field& by = f("Salame.By");
                Field& jx = f("Salame.jx"); Field& jy = f("Salame.jy");
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        jx(i, j) = dzf * chi(i, j) * by(i, j) * mu0_inv;
                        jy(i, j) = -dzf * chi(i, j) * bx(i, j) * mu0_inv;
                    }
            }
            salame_solve_ez();
            // step 3: the weight factor (:125-158, SalameGetW :334-400)
            f("Salame.jz_beam").zero();
            salame_deposit_jz(f("Salame.jz_beam"));
            double s_t = 0, s_no = 0, s_only = 0, s_jz = 0;
            {
                const Field& jz = f("Salame.jz_beam"); const Field& et = f("Salame.Ez_target");
                const Field& eno = f("Salame.Ez_no_salame"); const Field& ez = f("Salame.Ez");
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        s_t += jz(i, j) * et(i, j);
                        s_no += jz(i, j) * eno(i, j);
                        s_only += jz(i, j) * ez(i, j);
                        s_jz += jz(i, j);
                    }
            }
            s_t /= s_jz; s_no /= s_jz; s_only /= s_jz;
            const double zeta = (islice - 1) * dz + zoff;  // the Ez of the next slice
            const double args[3] = {zeta, sal_zeta0, s_t};
            s_t = cfg.salame_target.eval(args);
            double W = (s_t - s_no) / s_only + 1.0;
            if (W < 0 || sal_overloaded) {
                W = 0;
                iter = cfg.salame_n_iter - 1;
                sal_overloaded = true;
            }
            salame_log.insert(salame_log.end(), {(double)islice, (double)it0, W});
            if (!sal_overloaded && iter >= 1 && std::abs(W - 1.) < cfg.salame_relative_tolerance) iter = cfg.salame_n_iter - 1;
            // SalameMultiplyBeamWeight (:403-437)
            for (size_t b = 0; b < cfg.beams.size(); ++b) {
                if (!cfg.beams[b].do_salame) continue;
                for (size_t ip = 0; ip < bthis[b].num_nonslipped; ++ip) {
                    BeamParticle& p = bthis[b].p[ip];
                    if (!p.valid) continue;
                    if (W == 0) { p.valid = false; continue; }
                    p.w *= W;
                }
            }
            // step 4: Bx, By of this slice with the new weights (:160-183)
            f("jz_beam").zero(); f("Sy").zero(); f("Sx").zero();
            for (size_t b = 0; b < cfg.beams.size(); ++b)
                beam_deposit(bthis[b], cfg.beams[b].charge, nullptr, nullptr, &f("jz_beam"), nullptr);
            init_sxsy_with_beam();
            {
                Field& Sy = f("Sy"); Field& Sx = f("Sx");
                const Field& by = f("Salame.Sy_back"); const Field& bx = f("Salame.Sx_back");
                for (size_t k = 0; k < Sy.a.size(); ++k) { Sy.a[k] += by.a[k]; Sx.a[k] += bx.a[k]; }
            }
            mg_solve_fields("Bx", "By", "Sy", "Sx");
        }
    }
    // SalameOnlyAdvancePlasma (Salame.cpp:257-331): momenta from the SALAME-only Bx, By at the
    // previous position
    void salame_only_advance() {
        const Field& FBx = f("Salame.Bx"); const Field& FBy = f("Salame.By");
        for (size_t s = 0; s < plasmas.size(); ++s) {
            Plasma& pl = plasmas[s];
            const double qm = cfg.plasmas[s].charge / cfg.plasmas[s].mass;
            for (size_t ip = 0; ip < pl.n(); ++ip) {
                if (!pl.valid[ip]) continue;
                const double x = (pl.x_prev[ip] - xoff) * dxi, y = (pl.y_prev[ip] - yoff) * dyi;
                double bxp = 0, byp = 0;
                const int ord = cfg.depos_order_xy;
                for (int iy = 0; iy <= ord; ++iy)
                    for (int ix = 0; ix <= ord; ++ix) {
                        Shape sx = shapeN(ord, x, ix), sy = shapeN(ord, y, iy);
                        bxp += sx.s * sy.s * FBx(sx.cell, sy.cell);
                        byp += sx.s * sy.s * FBy(sx.cell, sy.cell);
                    }
                pl.ux[ip] = 1.5 * dz * qm * byp;
                pl.uy[ip] = -1.5 * dz * qm * bxp;
            }
        }
    }

    // ---- in-situ diagnostics (BeamParticleContainer.cpp:476-548, Fields.cpp:1289-1346)
    int cur_step = 0;
    std::vector<std::vector<double>> insitu_beam;  // per beam: per slice 22 sums + Np
    std::vector<double> insitu_fields;             // per slice 10 sums (times dx dy dz)
    bool insitu_beam_on(size_t b) const {
        return hpq::do_diagnostics(cfg.beams[b].insitu_period, cur_step, cfg.max_step, physical_time, cfg.max_time);
    }
    bool insitu_fields_on() const {
        return hpq::do_diagnostics(cfg.fields_insitu_period, cur_step, cfg.max_step, physical_time, cfg.max_time);
    }
    void insitu_compute(int islice) {
        const double cinv = 1.0 / cfg.pc.c;
        for (size_t b = 0; b < cfg.beams.size(); ++b) {
            if (!insitu_beam_on(b)) continue;
            const double r2 = cfg.beams[b].insitu_radius * cfg.beams[b].insitu_radius;
            double a[23] = {0};
            for (const BeamParticle& q : bthis[b].p) {
                if (!q.valid || q.x * q.x + q.y * q.y > r2) continue;
                const double x = q.x, y = q.y, z = q.z, w = q.w;
                const double ux = q.ux * cinv, uy = q.uy * cinv, uz = q.uz * cinv;
                const double uz_inv = uz == 0. ? 0. : 1. / uz;
                const double gamma = std::sqrt(1.0 + ux * ux + uy * uy + uz * uz);
                const double v[23] = {w, w * x, w * x * x, w * y, w * y * y, w * z, w * z * z, w * ux, w * ux * ux,
                                      w * uy, w * uy * uy, w * uz, w * uz * uz, w * x * ux, w * y * uy, w * z * uz,
                                      w * x * uy, w * y * ux, w * ux * uz_inv, w * uy * uz_inv, w * gamma,
                                      w * gamma * gamma, 1.0};
                for (int k = 0; k < 23; ++k) a[k] += v[k];
            }
            for (int k = 0; k < 23; ++k) insitu_beam[b][(size_t)islice * 23 + k] = a[k];
        }
        if (insitu_fields_on()) {
            const double c = cfg.pc.c, dv = dx * dy * dz;
            const Field &ex = f("ExmBy"), &ey = f("EypBx"), &ez = f("Ez"), &bx = f("Bx"), &by = f("By"), &bz = f("Bz"),
                        &jzb = f("jz_beam");
            double a[10] = {0};
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double v[10] = {std::pow(ex(i, j) + by(i, j) * c, 2), std::pow(ey(i, j) - bx(i, j) * c, 2),
                                          std::pow(ez(i, j), 2), std::pow(bx(i, j), 2), std::pow(by(i, j), 2),
                                          std::pow(bz(i, j), 2), std::pow(ex(i, j), 2), std::pow(ey(i, j), 2),
                                          jzb(i, j), ez(i, j) * jzb(i, j)};
                    for (int k = 0; k < 10; ++k) a[k] += v[k];
                }
            for (int k = 0; k < 10; ++k) insitu_fields[(size_t)islice * 10 + k] = a[k] * dv;
        }
    }

    // ======================================================================================
    // Adjoint of one step (explicit solver) with respect to the witness current-profile knots
    // and the plasma-density knots (hpq::AdjointConfig). The forward is the slice march of
    // solve_one_slice without the beam push (the beam push of this step only feeds the next
    // step); every slice's plasma state and fields are kept (small cases only), then the
    // slices are swept backwards:
    //   push            -> tangent passes of gather + push, field adjoints scattered by the
    //                      gather shapes (gather-adjoint = deposit)
    //   objective       -> dJ/dEz = 2 jz (Ez - Ebar)/S0, dJ/djz = ((Ez - Ebar)^2 - J)/S0
    //   multigrid       -> one solve with the transposed operator (W A W^-1, W = 3/4 on the
    //                      cell-centred boundary rows of the 4/3 closure, else 1); dJ/dchi = mu B
    //   explicit Sx/Sy  -> tangent passes per particle; field adjoints in closed form
    //   Sx/Sy beam part -> transposed centred differences
    //   Psi, Ez, Bz     -> the DST solve is symmetric; transposed gradient/divergence/curl
    //   deposit         -> tangent passes per particle (deposit-adjoint = gather)
    //   beam deposits   -> linear in the witness weights
    // ======================================================================================
    const double* adj_theta = nullptr;  // parameters during an adjoint evaluation
    double adj_sigma = 1.0;             // plasma density multiplier of the step

    double adj_profile(double z) const {
        const hpq::AdjointConfig& a = cfg.adjoint;
        return hpq::knot_value(adj_theta, z, a.profile_lo, a.profile_hi, a.n_profile, false);
    }

    struct AdjSlice {
        std::vector<Plasma> plasma;  // state entering the slice
        Field Psi, Ez, Bz, Bx, By, ExmBy, EypBx, chi, jzb;
    };

    // one slice of the forward without the beam push (explicit solver); objective sums added
    void adj_forward_slice(int islice, double* S) {
        for (auto n : {"chi", "Sy", "Sx", "ExmBy", "EypBx", "jz_beam", "rhomjz", "Next.jx_beam", "Next.jy_beam", "rhomjz_beam"}) f(n).zero();
        if (cfg.deposit_rho) f("rho").zero();
        if (islice == nz - 1)
            for (size_t b = 0; b < cfg.beams.size(); ++b) adj_load((int)b, islice, bthis[b]);
        plasma_deposit(0, true, false, cfg.deposit_rho, true, true);
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            beam_deposit(bthis[b], cfg.beams[b].charge, nullptr, nullptr, &f("jz_beam"),
                         cfg.do_beam_jz_minus_rho ? &f("rhomjz_beam") : nullptr);
        if (cfg.any_neutralize_background()) {
            Field& r = f("rhomjz"); const Field& ions = f("Ions.rhomjz");
            for (size_t k = 0; k < r.a.size(); ++k) r.a[k] += ions.a[k];
            if (cfg.deposit_rho) { Field& rr = f("rho"); for (size_t k = 0; k < rr.a.size(); ++k) rr.a[k] += ions.a[k]; }
        }
        solve_psi_ez_bz();
        if (islice - 1 >= 0)
            for (size_t b = 0; b < cfg.beams.size(); ++b) adj_load((int)b, islice - 1, bnext[b]);
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (cfg.do_beam_jx_jy_deposition && islice - 1 >= 0)
                beam_deposit(bnext[b], cfg.beams[b].charge, &f("Next.jx_beam"), &f("Next.jy_beam"), nullptr, nullptr);
        init_sxsy_with_beam();
        explicit_deposit();
        int iters = 0;
        const int st = mg.solve(f("Bx"), f("By"), f("Sy"), f("Sx"), f("chi"), cfg.mg_tol_rel, cfg.mg_tol_abs,
                                cfg.mg_max_iters, &iters);
        mg_iters_total += iters;
        if (st != 0 && mg_status == 0) mg_status = st;
        if (adj_objective_slice(islice)) {
            const Field& jz = f("jz_beam"); const Field& Ez = f("Ez");
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double a = jz(i, j), e = Ez(i, j);
                    S[0] += a; S[1] += a * e; S[2] += a * e * e;
                }
        }
        plasma_push(false);
        copy(f("Prev.jx_beam"), f("jx_beam")); copy(f("Prev.jy_beam"), f("jy_beam"));
        copy(f("jx_beam"), f("Next.jx_beam")); copy(f("jy_beam"), f("Next.jy_beam"));
        copy(f("jx"), f("Next.jx_beam")); copy(f("jy"), f("Next.jy_beam"));
        for (size_t b = 0; b < cfg.beams.size(); ++b) { bthis[b] = bnext[b]; bnext[b].p.clear(); bnext[b].num_nonslipped = 0; }
    }
    bool adj_objective_slice(int islice) const {
        const double zc = cfg.prob_lo[2] + (islice + 0.5) * dz;
        return zc >= cfg.adjoint.objective_lo && zc <= cfg.adjoint.objective_hi;
    }
    // beam slice with the witness weights multiplied by the profile
    void adj_load(int b, int islice, BeamSlice& dst_slice) {
        load_beam_slice(b, islice, dst_slice);
        if (b == cfg.adjoint.witness)
            for (auto& p : dst_slice.p) p.w *= adj_profile(p.z);
    }

    // the step's start: fields reset, plasma created and scaled by the density multiplier
    void adj_begin(const double* theta, Field* ions0) {
        adj_theta = theta;
        const hpq::AdjointConfig& a = cfg.adjoint;
        adj_sigma = hpq::knot_value(theta + a.n_profile, cfg.pc.c * physical_time, a.density_lo, a.density_hi,
                                    a.n_density, true);
        for (auto& kv : F) kv.second.zero();
        init_plasmas();
        if (cfg.any_neutralize_background()) plasma_deposit_ions();
        if (ions0) *ions0 = f("Ions.rhomjz");
        for (auto& pl : plasmas) for (auto& w : pl.w) w *= adj_sigma;
        for (auto& v : f("Ions.rhomjz").a) v *= adj_sigma;
    }

    double adj_objective(const double* S) const {
        if (S[0] == 0.0) return 0.0;
        const double m = S[1] / S[0];
        return S[2] / S[0] - m * m;
    }

    // forward only: the objective for parameters theta
    double adjoint_objective(const double* theta) {
        adj_begin(theta, nullptr);
        double S[3] = {0, 0, 0};
        for (int isl = nz - 1; isl >= 0; --isl) adj_forward_slice(isl, S);
        adj_theta = nullptr;
        return adj_objective(S);
    }

    // ---- per-particle maps on a generic scalar
    template <class T>
    void gather_t(T xp, T yp, T* G) {
        const Field& Psi = f("Psi"); const Field& FEz = f("Ez");
        const Field& FBx = f("Bx"); const Field& FBy = f("By"); const Field& FBz = f("Bz");
        const T x = (xp - xoff) * dxi, y = (yp - yoff) * dyi;
        for (int c = 0; c < 6; ++c) G[c] = 0.0 * x;
        for (int iy = 0; iy <= 3; iy++)
            for (int ix = 0; ix <= 3; ix++) {
                DShapeT<T> sy = dshape2t(1, y, iy);
                DShapeT<T> sx = dshape2t(1, x, ix);
                const int i = sx.cell, j = sy.cell;
                G[0] = G[0] + (sx.ds * sy.s) * Psi(i, j) * dxi;
                G[1] = G[1] + (sx.s * sy.ds) * Psi(i, j) * dyi;
                G[2] = G[2] + (sx.s * sy.s) * FEz(i, j);
                G[3] = G[3] + (sx.s * sy.s) * FBx(i, j);
                G[4] = G[4] + (sx.s * sy.s) * FBy(i, j);
                G[5] = G[5] + (sx.s * sy.s) * FBz(i, j);
            }
        G[3] = G[3] * cfg.pc.c;
        G[4] = G[4] * cfg.pc.c;
    }
    template <class T>
    bool enforce_bc_t(T& x, T& y, T& ux, T& uy) const {
        const double plo0 = cfg.particle_lo[0], plo1 = cfg.particle_lo[1];
        const double phi0 = cfg.particle_hi[0], phi1 = cfg.particle_hi[1];
        if (val(x) < plo0 || val(y) < plo1 || val(x) > phi0 || val(y) > phi1) {
            const double lx = phi0 - plo0, ly = phi1 - plo1;
            if (cfg.particle_bc == hpq::ParticleBC::Absorbing) return false;
            const bool refl = cfg.particle_bc == hpq::ParticleBC::Reflecting;
            const double px = refl ? 2 * lx : lx, py = refl ? 2 * ly : ly;
            double m = std::fmod(val(x) - plo0, px); if (m < 0) m += px;
            x = x + ((m + plo0) - val(x));
            m = std::fmod(val(y) - plo1, py); if (m < 0) m += py;
            y = y + ((m + plo1) - val(y));
            if (refl && val(x) > phi0) { x = 2 * phi0 - x; ux = -ux; }
            if (refl && val(y) > phi1) { y = 2 * phi1 - y; uy = -uy; }
        }
        return true;
    }
    // gather fields G (ExmBy, EypBx, Ez, c Bx, c By, Bz) given; push of one particle, n_subcycles 1.
    // out: x, y, ux_h, uy_h, psi_h, ux, uy, psi
    template <class T>
    bool push_t(T x, T y, T ux, T uy, T psi, const T* G, double qmc, T* out) const {
        const double ci = 1. / cfg.pc.c, dzs = dz;
        const double sdz = dzs / 4;
        auto substep = [&]() {
            const T psi_inv = 1. / psi;
            const T gamma_psi = 0.5 * psi_inv * psi_inv * (1.0 + ux * ux * (ci * ci) + uy * uy * (ci * ci)) + 0.5;
            const T d_ux = qmc * (gamma_psi * G[0] + G[4] + (uy * G[5]) * psi_inv);
            const T d_uy = qmc * (gamma_psi * G[1] - G[3] - (ux * G[5]) * psi_inv);
            const T d_psi = qmc * ci * ((ux * G[0] + uy * G[1]) * ci * psi_inv - G[2]);
            const T zero = 0.0 * psi;
            DuT<T> dx_{ux, d_ux}, dy_{uy, d_uy}, dp{psi_inv, -psi_inv * psi_inv * d_psi};
            const DuT<T> c2{zero + ci * ci, zero}, one{zero + 1.0, zero}, half{zero + 0.5, zero};
            const DuT<T> q{zero + qmc, zero}, cc{zero + ci, zero};
            const DuT<T> E0{G[0], zero}, E1{G[1], zero}, E2{G[2], zero}, B0{G[3], zero}, B1{G[4], zero}, B2{G[5], zero};
            DuT<T> t = tadd(tadd(one, tmul(tmul(dx_, dx_), c2)), tmul(tmul(dy_, dy_), c2));
            DuT<T> gp = tadd(tmul(tmul(tmul(half, dp), dp), t), half);
            DuT<T> dux = tmul(q, tadd(tadd(tmul(gp, E0), B1), tmul(tmul(dy_, B2), dp)));
            DuT<T> duy = tmul(q, tsub(tsub(tmul(gp, E1), B0), tmul(tmul(dx_, B2), dp)));
            DuT<T> dps = tmul(tmul(q, cc), tsub(tmul(tmul(tadd(tmul(dx_, E0), tmul(dy_, E1)), cc), dp), E2));
            ux = ux + sdz * d_ux + 0.5 * sdz * sdz * dux.e;
            uy = uy + sdz * d_uy + 0.5 * sdz * sdz * duy.e;
            psi = psi + sdz * d_psi + 0.5 * sdz * sdz * dps.e;
        };
        for (int k = 0; k < 4; ++k) substep();
        x = x + dzs * ci * (ux * (1. / psi));
        y = y + dzs * ci * (uy * (1. / psi));
        if (!enforce_bc_t(x, y, ux, uy)) return false;
        out[0] = x; out[1] = y; out[2] = ux; out[3] = uy; out[4] = psi;
        for (int k = 0; k < 2; ++k) substep();
        out[5] = ux; out[6] = uy; out[7] = psi;
        return true;
    }

    struct AdjFields {
        Field Psi, Ez, Bz, Bx, By, ExmBy, EypBx, Sx, Sy, chi, jx, jy, rm, jzb, Pjx, Pjy, Njx, Njy;
        void init(const Grid& g) {
            for (Field* q : {&Psi, &Ez, &Bz, &Bx, &By, &ExmBy, &EypBx, &Sx, &Sy, &chi, &jx, &jy, &rm, &jzb, &Pjx, &Pjy, &Njx, &Njy}) q->init(g);
        }
        void zero() {
            for (Field* q : {&Psi, &Ez, &Bz, &Bx, &By, &ExmBy, &EypBx, &Sx, &Sy, &chi, &jx, &jy, &rm, &jzb, &Pjx, &Pjy, &Njx, &Njy}) q->zero();
        }
    };
    struct PlasmaAdj { std::vector<double> x, y, uhx, uhy, psih, ux, uy, psi, w; };

    static void zero_outside_interior(Field& q, int nx_, int ny_) {
        const int g = q.gr.g;
        for (int j = -g; j < ny_ + g; ++j)
            for (int i = -g; i < nx_ + g; ++i)
                if (i < 0 || j < 0 || i >= nx_ || j >= ny_) q(i, j) = 0.0;
    }

    // adjoint of the beam deposits of beam slice k of the witness: dJ/dw_eff per particle
    void adj_beam(int k, const Field* ljz, const Field* lrm, const Field* ljx, const Field* ljy,
                  std::vector<std::vector<double>>& lw) {
        if (k < 0 || k >= nz) return;
        const int b = cfg.adjoint.witness;
        const BeamSlice& bs = store[b][k];
        const double invvol = cfg.normalized_units ? 1.0 : dxi * dyi * dzi;
        const double ci = 1.0 / cfg.pc.c, ci2 = ci * ci;
        const double q = cfg.beams[b].charge;
        for (size_t ip = 0; ip < bs.p.size(); ++ip) {
            const BeamParticle& p = bs.p[ip];
            if (!p.valid) continue;
            const double gaminv = 1.0 / std::sqrt(1.0 + p.ux * p.ux * ci2 + p.uy * p.uy * ci2 + p.uz * p.uz * ci2);
            const double vx = p.ux * gaminv, vy = p.uy * gaminv, vz = p.uz * gaminv;
            const double xmid = (p.x - xoff) * dxi, ymid = (p.y - yoff) * dyi;
            double acc = 0;
            for (int iy = 0; iy <= 2; ++iy)
                for (int ix = 0; ix <= 2; ++ix) {
                    Shape sx = shape2(xmid, ix), sy = shape2(ymid, iy);
                    const double S = sx.s * sy.s;
                    const int i = sx.cell, j = sy.cell;
                    double l = 0;
                    if (ljz) l += vz * (*ljz)(i, j);
                    if (lrm) l += (1. - vz * ci) * (*lrm)(i, j);
                    if (ljx) l += vx * (*ljx)(i, j) + vy * (*ljy)(i, j);
                    acc += S * l;
                }
            lw[k][ip] += q * invvol * acc;
        }
    }

    // gradient of the objective; returns J
    double adjoint_grad(const double* theta, double* grad) {
        const hpq::AdjointConfig& A = cfg.adjoint;
        Field ions0; ions0.init(gr);
        adj_begin(theta, &ions0);
        double S[3] = {0, 0, 0};
        std::vector<AdjSlice> rec(nz);
        std::vector<std::vector<double>> w0(plasmas.size());
        for (size_t sp = 0; sp < plasmas.size(); ++sp) {
            w0[sp] = plasmas[sp].w;
            for (auto& w : w0[sp]) w = adj_sigma != 0 ? w / adj_sigma : 0.0;
        }
        for (int isl = nz - 1; isl >= 0; --isl) {
            rec[isl].plasma = plasmas;
            adj_forward_slice(isl, S);
            AdjSlice& r = rec[isl];
            r.Psi = f("Psi"); r.Ez = f("Ez"); r.Bz = f("Bz"); r.Bx = f("Bx"); r.By = f("By");
            r.ExmBy = f("ExmBy"); r.EypBx = f("EypBx"); r.chi = f("chi"); r.jzb = f("jz_beam");
        }
        const double J = adj_objective(S);
        const double S0 = S[0], Ebar = S0 != 0 ? S[1] / S0 : 0.0;
        const double mu0 = cfg.pc.mu0, ep0 = cfg.pc.ep0, cl = cfg.pc.c, ci = 1. / cl;
        const double hx = 0.5 * dxi, hy = 0.5 * dyi;
        // adjoint state
        AdjFields L; L.init(gr);
        std::vector<PlasmaAdj> lp(plasmas.size());
        for (size_t sp = 0; sp < plasmas.size(); ++sp) {
            const size_t n = plasmas[sp].n();
            for (auto* v : {&lp[sp].x, &lp[sp].y, &lp[sp].uhx, &lp[sp].uhy, &lp[sp].psih, &lp[sp].ux, &lp[sp].uy, &lp[sp].psi, &lp[sp].w})
                v->assign(n, 0.0);
        }
        std::vector<std::vector<double>> lwb(nz);
        const int wb = A.witness;
        for (int k = 0; k < nz; ++k) lwb[k].assign(store[wb][k].p.size(), 0.0);
        double dsigma_ions = 0;
        Field sol[2], rhs[2];
        for (int c = 0; c < 2; ++c) { sol[c].init(gr); rhs[c].init(gr); }

        for (int isl = 0; isl < nz; ++isl) {
            AdjSlice& r = rec[isl];
            // the forward fields of this slice become current (gather/explicit read them)
            f("Psi") = r.Psi; f("Ez") = r.Ez; f("Bz") = r.Bz; f("Bx") = r.Bx; f("By") = r.By;
            f("ExmBy") = r.ExmBy; f("EypBx") = r.EypBx;
            L.zero();
            std::vector<PlasmaAdj> lin(plasmas.size());
            for (size_t sp = 0; sp < plasmas.size(); ++sp) {
                const size_t n = plasmas[sp].n();
                for (auto* v : {&lin[sp].x, &lin[sp].y, &lin[sp].uhx, &lin[sp].uhy, &lin[sp].psih, &lin[sp].ux, &lin[sp].uy, &lin[sp].psi})
                    v->assign(n, 0.0);
            }
            // (1) plasma push
            for (size_t sp = 0; sp < plasmas.size(); ++sp) {
                const hpq::PlasmaSpecies& P = cfg.plasmas[sp];
                const Plasma& pl = r.plasma[sp];
                const PlasmaAdj& lo = lp[sp];
                const double qmc = P.charge / (P.mass * cl);
                for (size_t ip = 0; ip < pl.n(); ++ip) {
                    if (!pl.valid[ip] || !adj_alive(P, pl, ip)) continue;
                    const double lout[8] = {lo.x[ip], lo.y[ip], lo.uhx[ip], lo.uhy[ip], lo.psih[ip], lo.ux[ip], lo.uy[ip], lo.psi[ip]};
                    bool any = false;
                    for (double v : lout) any = any || v != 0.0;
                    if (!any) continue;
                    const double in[5] = {pl.x_prev[ip], pl.y_prev[ip], pl.ux_h[ip], pl.uy_h[ip], pl.psi_h[ip]};
                    double dl[5];
                    bool alive = true;
                    for (int k = 0; k < 5 && alive; ++k) {
                        Tn t[5];
                        for (int m = 0; m < 5; ++m) t[m] = seed(in[m], m == k);
                        Tn G[6], out[8];
                        gather_t(t[0], t[1], G);
                        alive = push_t(t[0], t[1], t[2], t[3], t[4], G, qmc, out);
                        double d = 0;
                        for (int o = 0; o < 8; ++o) d += lout[o] * out[o].d;
                        dl[k] = d;
                    }
                    if (!alive) continue;
                    double Gv[6];
                    gather_t(in[0], in[1], Gv);
                    double lG[6];
                    for (int c = 0; c < 6; ++c) {
                        Tn t[5], G[6], out[8];
                        for (int m = 0; m < 5; ++m) t[m] = seed(in[m], false);
                        for (int m = 0; m < 6; ++m) G[m] = seed(Gv[m], m == c);
                        push_t(t[0], t[1], t[2], t[3], t[4], G, qmc, out);
                        double d = 0;
                        for (int o = 0; o < 8; ++o) d += lout[o] * out[o].d;
                        lG[c] = d;
                    }
                    PlasmaAdj& li = lin[sp];
                    li.x[ip] += dl[0]; li.y[ip] += dl[1]; li.uhx[ip] += dl[2]; li.uhy[ip] += dl[3]; li.psih[ip] += dl[4];
                    // gather adjoint: scatter by the gather shapes
                    const double x = (in[0] - xoff) * dxi, y = (in[1] - yoff) * dyi;
                    for (int iy = 0; iy <= 3; iy++)
                        for (int ix = 0; ix <= 3; ix++) {
                            DShape sy = dshape2(1, y, iy), sx = dshape2(1, x, ix);
                            const int i = sx.cell, j = sy.cell;
                            const double Sv = sx.s * sy.s;
                            L.Psi(i, j) += lG[0] * sx.ds * sy.s * dxi + lG[1] * sx.s * sy.ds * dyi;
                            L.Ez(i, j) += lG[2] * Sv;
                            L.Bx(i, j) += lG[3] * cl * Sv;
                            L.By(i, j) += lG[4] * cl * Sv;
                            L.Bz(i, j) += lG[5] * Sv;
                        }
                }
            }
            // (2) objective
            if (adj_objective_slice(isl) && S0 != 0) {
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const double jz = r.jzb(i, j), e = r.Ez(i, j) - Ebar;
                        L.Ez(i, j) += 2 * jz * e / S0;
                        L.jzb(i, j) += (e * e - J) / S0;
                    }
            }
            // (3) multigrid: mu = W A^-1 W^-1 lambda_B
            for (Field* q : {&L.Bx, &L.By}) zero_outside_interior(*q, nx, ny);
            const bool cellc = mg.cell;
            auto wgt = [&](int i, int j) {
                double w = 1;
                if (cellc && (i == 0 || i == nx - 1)) w *= 0.75;
                if (cellc && (j == 0 || j == ny - 1)) w *= 0.75;
                return w;
            };
            for (int c = 0; c < 2; ++c) { sol[c].zero(); rhs[c].zero(); }
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    rhs[0](i, j) = L.Bx(i, j) / wgt(i, j);
                    rhs[1](i, j) = L.By(i, j) / wgt(i, j);
                }
            {
                int iters = 0;
                mg.solve(sol[0], sol[1], rhs[0], rhs[1], r.chi, cfg.mg_tol_rel, cfg.mg_tol_abs, cfg.mg_max_iters, &iters);
            }
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double mx = sol[0](i, j) * wgt(i, j), my = sol[1](i, j) * wgt(i, j);
                    L.Sy(i, j) = mx;
                    L.Sx(i, j) = my;
                    L.chi(i, j) += mx * r.Bx(i, j) + my * r.By(i, j);
                }
            // (4) explicit deposit
            adj_explicit(r, L, lin);
            // (5) Sx/Sy beam part (Hipace.cpp:744-790)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double ly_ = L.Sy(i, j), lx_ = L.Sx(i, j);
                    L.jzb(i, j + 1) += -mu0 / (2 * dy) * ly_;
                    L.jzb(i, j - 1) += mu0 / (2 * dy) * ly_;
                    L.jzb(i + 1, j) += mu0 / (2 * dx) * lx_;
                    L.jzb(i - 1, j) += -mu0 / (2 * dx) * lx_;
                    L.Pjy(i, j) += mu0 / (2 * dz) * ly_;
                    L.Njy(i, j) += -mu0 / (2 * dz) * ly_;
                    L.Pjx(i, j) += -mu0 / (2 * dz) * lx_;
                    L.Njx(i, j) += mu0 / (2 * dz) * lx_;
                }
            // (6) ExmBy, EypBx = -grad Psi on [-1, n]
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    const double a = L.ExmBy(i, j), b = L.EypBx(i, j);
                    L.Psi(i + 1, j) += -a * hx; L.Psi(i - 1, j) += a * hx;
                    L.Psi(i, j + 1) += -b * hy; L.Psi(i, j - 1) += b * hy;
                }
            // (7) Poisson solves (symmetric), then transposed right-hand sides
            std::vector<double> st((size_t)nx * ny);
            auto solve_from = [&](const Field& q) {
                for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) st[(size_t)j * nx + i] = q(i, j);
                dst.solve(st);
            };
            solve_from(L.Psi);
            for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) L.rm(i, j) += -1. / ep0 * st[(size_t)j * nx + i];
            const double fe = 1. / (ep0 * cl);
            solve_from(L.Ez);
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double v = st[(size_t)j * nx + i];
                    L.jx(i + 1, j) += fe * hx * v; L.jx(i - 1, j) -= fe * hx * v;
                    L.jy(i, j + 1) += fe * hy * v; L.jy(i, j - 1) -= fe * hy * v;
                }
            solve_from(L.Bz);
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double v = st[(size_t)j * nx + i];
                    L.jx(i, j + 1) += mu0 * hy * v; L.jx(i, j - 1) -= mu0 * hy * v;
                    L.jy(i + 1, j) -= mu0 * hx * v; L.jy(i - 1, j) += mu0 * hx * v;
                }
            // (8) plasma deposit
            adj_deposit(r, L, lin);
            // ions and beam
            for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) dsigma_ions += L.rm(i, j) * ions0(i, j);
            adj_beam(isl, &L.jzb, cfg.do_beam_jz_minus_rho ? &L.rm : nullptr,
                     (cfg.do_beam_jx_jy_deposition && isl <= nz - 2) ? &L.jx : nullptr, &L.jy, lwb);
            if (cfg.do_beam_jx_jy_deposition) {
                if (isl + 1 <= nz - 2) adj_beam(isl + 1, nullptr, nullptr, &L.Pjx, &L.Pjy, lwb);
                if (isl - 1 >= 0) adj_beam(isl - 1, nullptr, nullptr, &L.Njx, &L.Njy, lwb);
            }
            for (size_t sp = 0; sp < plasmas.size(); ++sp) {
                PlasmaAdj& a = lp[sp];
                a.x = lin[sp].x; a.y = lin[sp].y; a.uhx = lin[sp].uhx; a.uhy = lin[sp].uhy; a.psih = lin[sp].psih;
                a.ux = lin[sp].ux; a.uy = lin[sp].uy; a.psi = lin[sp].psi;
                for (size_t ip = 0; ip < a.w.size(); ++ip) a.w[ip] += lin[sp].w.empty() ? 0.0 : lin[sp].w[ip];
            }
        }
        // parameters
        const int np = A.n_params();
        for (int k = 0; k < np; ++k) grad[k] = 0;
        for (int k = 0; k < nz; ++k) {
            const BeamSlice& bs = store[wb][k];
            for (size_t ip = 0; ip < bs.p.size(); ++ip) {
                if (!bs.p[ip].valid || lwb[k][ip] == 0.0) continue;
                int kk; double fr;
                if (!hpq::knot_interval(bs.p[ip].z, A.profile_lo, A.profile_hi, A.n_profile, false, kk, fr)) continue;
                const double g = lwb[k][ip] * bs.p[ip].w;
                grad[kk] += (1 - fr) * g;
                grad[kk + 1] += fr * g;
            }
        }
        double dsigma = dsigma_ions;
        for (size_t sp = 0; sp < plasmas.size(); ++sp)
            for (size_t ip = 0; ip < w0[sp].size(); ++ip) dsigma += lp[sp].w[ip] * w0[sp][ip];
        {
            int kk; double fr;
            if (hpq::knot_interval(cfg.pc.c * physical_time, A.density_lo, A.density_hi, A.n_density, true, kk, fr)) {
                if (A.n_density == 1) grad[A.n_profile] += dsigma;
                else { grad[A.n_profile + kk] += (1 - fr) * dsigma; grad[A.n_profile + kk + 1] += fr * dsigma; }
            }
        }
        adj_theta = nullptr;
        return J;
    }

    // the deposit's QSA test (PlasmaDepositCurrent.cpp:164-247) on the stored state
    bool adj_alive(const hpq::PlasmaSpecies& P, const Plasma& pl, size_t ip) const {
        const double psi_inv = 1.0 / pl.psi[ip];
        const double ci = 1.0 / cfg.pc.c;
        const double vx = pl.ux[ip] * psi_inv * ci, vy = pl.uy[ip] * psi_inv * ci;
        const double gamma_psi = 0.5 * (psi_inv * psi_inv + vx * vx + vy * vy + 1.0);
        return !(gamma_psi < 0.0 || gamma_psi > P.max_qsa_weighting_factor || psi_inv < 0.0);
    }

    template <class T>
    T dep_L(const hpq::PlasmaSpecies& P, T x, T y, T ux, T uy, T psi, double w, const AdjFields& L) const {
        const double invvol = cfg.normalized_units ? dx * dy * dxi * dyi : dxi * dyi * dzi;
        const double clightinv = 1.0 / cfg.pc.c;
        const double q_invvol = P.charge * invvol * w;
        const double qm = P.charge * cfg.pc.mu0 / P.mass;
        const T psi_inv = 1.0 / psi;
        const T vx_c = ux * psi_inv, vy_c = uy * psi_inv;
        (void)clightinv;
        const T xmid = (x - xoff) * dxi, ymid = (y - yoff) * dyi;
        T acc = 0.0 * x;
        for (int iy = 0; iy <= 2; ++iy)
            for (int ix = 0; ix <= 2; ++ix) {
                ShapeT<T> sx = shape2t(xmid, ix), sy = shape2t(ymid, iy);
                const int i = sx.cell, j = sy.cell;
                const T cd = q_invvol * sx.s * sy.s;
                acc = acc + cd * (vx_c * L.jx(i, j) + vy_c * L.jy(i, j) + qm * psi_inv * L.chi(i, j) + L.rm(i, j));
            }
        return acc;
    }
    void adj_deposit(const AdjSlice& r, const AdjFields& L, std::vector<PlasmaAdj>& lin) {
        for (size_t sp = 0; sp < plasmas.size(); ++sp) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[sp];
            const Plasma& pl = r.plasma[sp];
            PlasmaAdj& li = lin[sp];
            if (li.w.empty()) li.w.assign(pl.n(), 0.0);
            for (size_t ip = 0; ip < pl.n(); ++ip) {
                if (!pl.valid[ip] || !adj_alive(P, pl, ip)) continue;
                const double in[5] = {pl.x[ip], pl.y[ip], pl.ux[ip], pl.uy[ip], pl.psi[ip]};
                double d[5];
                for (int k = 0; k < 5; ++k) {
                    Tn t[5];
                    for (int m = 0; m < 5; ++m) t[m] = seed(in[m], m == k);
                    d[k] = dep_L(P, t[0], t[1], t[2], t[3], t[4], pl.w[ip], L).d;
                }
                li.x[ip] += d[0]; li.y[ip] += d[1]; li.ux[ip] += d[2]; li.uy[ip] += d[3]; li.psi[ip] += d[4];
                li.w[ip] += dep_L(P, in[0], in[1], in[2], in[3], in[4], 1.0, L);
            }
        }
    }

    template <class T>
    T ex_L(const hpq::PlasmaSpecies& P, T x, T y, T ux, T uy, T psi, double w, const AdjFields& L,
           AdjFields* scatter) {
        const int dt = cfg.depos_derivative_type;
        const int ns = 2 + dt;
        const Field& Bz = f("Bz"); const Field& Ez = f("Ez");
        const Field& ExmBy = f("ExmBy"); const Field& EypBx = f("EypBx");
        const double invvol = cfg.normalized_units ? dx * dy * dxi * dyi : dxi * dyi * dzi;
        const double a_clight = cfg.pc.c, ci = 1. / cfg.pc.c;
        const double cdm = P.charge * invvol * cfg.pc.mu0 * w;
        const double qm = P.charge / P.mass;
        const T psi_inv = 1. / psi;
        const T vx = ux * psi_inv * ci, vy = uy * psi_inv * ci;
        const T xmid = (x - xoff) * dxi, ymid = (y - yoff) * dyi;
        const T gamma_psi = 0.5 * (psi_inv * psi_inv + vx * vx + vy * vy + 1.);
        T acc = 0.0 * x;
        for (int iy = 0; iy <= ns; ++iy)
            for (int ix = 0; ix <= ns; ++ix) {
                if (dt == 2 && (ix == 0 || ix == 4) && (iy == 0 || iy == 4)) continue;
                DShapeT<T> sy = dshape2t(dt, ymid, iy);
                DShapeT<T> sx = dshape2t(dt, xmid, ix);
                const int i = sx.cell, j = sy.cell;
                const double Bz_v = Bz(i, j), Ez_v = Ez(i, j), ExmBy_v = ExmBy(i, j), EypBx_v = EypBx(i, j);
                const T Sy_c = cdm * (-sx.s * sy.s * (-Bz_v * vx + (Ez_v * vy + ExmBy_v * (-vx * vy) + EypBx_v * (gamma_psi - vy * vy)) * ci) * qm * psi_inv +
                                      (-sx.ds * sy.s * dxi * (-vx * vy) - sx.s * sy.ds * dyi * (gamma_psi - vy * vy - 1.)) * a_clight);
                const T Sx_c = cdm * (+sx.s * sy.s * (+Bz_v * vy + (Ez_v * vx + ExmBy_v * (gamma_psi - vx * vx) + EypBx_v * (-vx * vy)) * ci) * qm * psi_inv +
                                      (+sx.ds * sy.s * dxi * (gamma_psi - vx * vx - 1.) + sx.s * sy.ds * dyi * (-vx * vy)) * a_clight);
                const double lSy = L.Sy(i, j), lSx = L.Sx(i, j);
                acc = acc + lSy * Sy_c + lSx * Sx_c;
                if (scatter) {
                    const double K = val(cdm * sx.s * sy.s * qm * psi_inv);
                    const double vxv = val(vx), vyv = val(vy), gp = val(gamma_psi);
                    scatter->Bz(i, j) += lSy * K * vxv + lSx * K * vyv;
                    scatter->Ez(i, j) += -lSy * K * vyv * ci + lSx * K * vxv * ci;
                    scatter->ExmBy(i, j) += lSy * K * vxv * vyv * ci + lSx * K * (gp - vxv * vxv) * ci;
                    scatter->EypBx(i, j) += -lSy * K * (gp - vyv * vyv) * ci - lSx * K * vxv * vyv * ci;
                }
            }
        return acc;
    }
    void adj_explicit(const AdjSlice& r, AdjFields& L, std::vector<PlasmaAdj>& lin) {
        for (size_t sp = 0; sp < plasmas.size(); ++sp) {
            const hpq::PlasmaSpecies& P = cfg.plasmas[sp];
            const Plasma& pl = r.plasma[sp];
            PlasmaAdj& li = lin[sp];
            if (li.w.empty()) li.w.assign(pl.n(), 0.0);
            for (size_t ip = 0; ip < pl.n(); ++ip) {
                if (!pl.valid[ip] || !adj_alive(P, pl, ip)) continue;
                const double in[5] = {pl.x[ip], pl.y[ip], pl.ux[ip], pl.uy[ip], pl.psi[ip]};
                double d[5];
                for (int k = 0; k < 5; ++k) {
                    Tn t[5];
                    for (int m = 0; m < 5; ++m) t[m] = seed(in[m], m == k);
                    d[k] = ex_L(P, t[0], t[1], t[2], t[3], t[4], pl.w[ip], L, nullptr).d;
                }
                li.x[ip] += d[0]; li.y[ip] += d[1]; li.ux[ip] += d[2]; li.uy[ip] += d[3]; li.psi[ip] += d[4];
                li.w[ip] += ex_L(P, in[0], in[1], in[2], in[3], in[4], 1.0, L, nullptr);
                ex_L(P, in[0], in[1], in[2], in[3], in[4], pl.w[ip], L, &L);
            }
        }
    }

    int step(int s) {
        begin_step(s);
        for (int isl = nz - 1; isl >= 0; --isl) solve_one_slice(isl, s);
        end_step();
        return mg_status;
    }
};

}  // namespace oracle

// ------------------------------------------------------------------------------------------
// C interface used by the tests (ctypes)
// ------------------------------------------------------------------------------------------
struct OracleHandle {
    std::unique_ptr<oracle::Sim> sim;
    std::string err;
};

extern "C" {

int oracle_create(const char* input_text, OracleHandle** out, char* err, int errlen) {
    try {
        hpq::InputStore in;
        in.parse_text(input_text);
        hpq::SimConfig cfg = hpq::build_config(in);
        auto* h = new OracleHandle;
        h->sim.reset(new oracle::Sim(cfg));
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        if (err && errlen > 0) { strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return 1;
    }
}
void oracle_destroy(OracleHandle* h) { delete h; }

int oracle_init_beams(OracleHandle* h) {
    auto& s = *h->sim;
    for (size_t b = 0; b < s.cfg.beams.size(); ++b) {
        if (s.cfg.beams[b].injection == hpq::BeamInjection::FixedPPC) s.init_beam_fixed_ppc((int)b);
        else if (s.store_valid[b]) continue;  // particles given with oracle_set_beam
        else if (s.cfg.beams[b].injection == hpq::BeamInjection::FixedWeight) s.init_beam_fixed_weight((int)b);
        else return 2;  // fixed_weight_pdf beams must be provided
    }
    return 0;
}

int oracle_set_beam(OracleHandle* h, int b, const double* x, const double* y, const double* z, const double* w,
                    const double* ux, const double* uy, const double* uz, const int64_t* id, int64_t n) {
    auto& s = *h->sim;
    if (b < 0 || b >= (int)s.cfg.beams.size()) return 1;
    s.set_beam(b, x, y, z, w, ux, uy, uz, id, n);
    return 0;
}

// Time-step pipeline hand-off (MultiBuffer.cpp:181-430): after slice islice of a step, store
// slice islice holds what it hands to the next step; a rank that runs the next step puts the
// received particles there (slices from the head down, nz-1 first, which empties the store).
int64_t oracle_beam_slice_count(OracleHandle* h, int b, int islice) {
    return (int64_t)h->sim->store.at(b).at(islice).p.size();
}
int oracle_get_beam_slice(OracleHandle* h, int b, int islice, double* x, double* y, double* z, double* w, double* ux,
                          double* uy, double* uz, int64_t* id) {
    const auto& v = h->sim->store.at(b).at(islice).p;
    for (size_t k = 0; k < v.size(); ++k) {
        x[k] = v[k].x; y[k] = v[k].y; z[k] = v[k].z; w[k] = v[k].w;
        ux[k] = v[k].ux; uy[k] = v[k].uy; uz[k] = v[k].uz; id[k] = v[k].id;
    }
    return 0;
}
int oracle_put_beam_slice(OracleHandle* h, int b, int islice, const double* x, const double* y, const double* z,
                          const double* w, const double* ux, const double* uy, const double* uz, const int64_t* id,
                          int64_t n) {
    auto& st = h->sim->store.at(b);
    if (islice == (int)st.size() - 1)
        for (auto& sl : st) { sl.p.clear(); sl.num_nonslipped = 0; }
    auto& sl = st.at(islice);
    sl.p.clear();
    for (int64_t k = 0; k < n; ++k) sl.p.push_back({x[k], y[k], z[k], w[k], ux[k], uy[k], uz[k], id[k], 0, w[k] != 0.0});
    sl.num_nonslipped = sl.p.size();
    return 0;
}
void oracle_set_time(OracleHandle* h, double t) { h->sim->physical_time = t; }

// number of stored particles of beam b (all slices), and a copy in slice-descending order
int64_t oracle_beam_count(OracleHandle* h, int b) {
    auto& s = *h->sim;
    int64_t n = 0;
    for (auto& sl : s.store[b]) n += (int64_t)sl.p.size();
    return n;
}
int oracle_get_beam(OracleHandle* h, int b, double* x, double* y, double* z, double* w, double* ux, double* uy,
                    double* uz, int64_t* id) {
    auto& s = *h->sim;
    int64_t k = 0;
    for (int sl = s.nz - 1; sl >= 0; --sl)
        for (auto& p : s.store[b][sl].p) {
            // invalid particles are reported with weight 0 (as hpq_get_beam does)
            x[k] = p.x; y[k] = p.y; z[k] = p.z; w[k] = p.valid ? p.w : 0.0; ux[k] = p.ux; uy[k] = p.uy; uz[k] = p.uz;
            if (id) id[k] = p.id;
            ++k;
        }
    return 0;
}

int oracle_set_diag(OracleHandle* h, const char* names) {
    auto& s = *h->sim;
    s.diag_names.clear();
    std::string t(names);
    std::istringstream in(t);
    std::string n;
    while (in >> n) {
        if (!s.F.count(n)) return 1;
        s.diag_names.push_back(n);
    }
    return 0;
}
int oracle_get_diag(OracleHandle* h, const char* name, double* out) {
    auto& s = *h->sim;
    auto it = s.diag.find(name);
    if (it == s.diag.end()) return 1;
    std::memcpy(out, it->second.data(), it->second.size() * sizeof(double));
    return 0;
}

int oracle_step(OracleHandle* h, int step) { return h->sim->step(step); }
int oracle_begin_step(OracleHandle* h, int step) { h->sim->begin_step(step); return 0; }
int oracle_solve_slice(OracleHandle* h, int islice, int step) { h->sim->solve_one_slice(islice, step); return h->sim->mg_status; }
int oracle_end_step(OracleHandle* h) { h->sim->end_step(); return 0; }
double oracle_time(OracleHandle* h) { return h->sim->physical_time; }
// The Dirichlet Poisson solve of the slice loop on its own, Lap(u) = f on an nx x ny grid (x
// fastest) with u = 0 one cell outside, by the sine transform of PoissonDST (known-answer tests)
int oracle_poisson_dirichlet(const double* f, double* u, int nx, int ny, double dx, double dy) {
    if (nx < 1 || ny < 1) return 1;
    oracle::PoissonDST d;
    d.init(nx, ny, dx, dy);
    std::vector<double> v(f, f + (size_t)nx * ny);
    d.solve(v);
    std::copy(v.begin(), v.end(), u);
    return 0;
}
// DST-I of length n as used by the solver: out_k = sum_i 2 sin(pi (i+1)(k+1) / (n+1)) in_i
int oracle_dst1(const double* in, double* out, int n) {
    if (n < 1) return 1;
    oracle::PoissonDST d;
    d.init(n, 1, 1.0, 1.0);
    std::vector<double> v(in, in + n);
    d.transform_x(v);
    std::copy(v.begin(), v.end(), out);
    return 0;
}

// One shape factor of the restated ShapeFactors.H: type -1 the deposit shape of order `ord`,
// types 0/1/2 the derivative shapes (known-answer tests)
int oracle_shape_factor(int type, int ord, double xmid, int ix, double* sv, double* dsv, int* cell) {
    if (ord < 0 || ord > 3 || type < -1 || type > 2) return 1;
    if (type < 0) {
        const oracle::Shape r = oracle::shapeN(ord, xmid, ix);
        *sv = r.s; *dsv = 0; *cell = r.cell;
    } else {
        const oracle::DShape r = oracle::dshapeN(type, ord, xmid, ix);
        *sv = r.s; *dsv = r.ds; *cell = r.cell;
    }
    return 0;
}

// SALAME record: (slice, iteration, weight factor) triples; returns the number of doubles
long long oracle_salame_log(OracleHandle* h, double* out) {
    const auto& v = h->sim->salame_log;
    if (out) std::memcpy(out, v.data(), v.size() * sizeof(double));
    return (long long)v.size();
}

// interior nx*ny values of a slice component (current slice state)
int oracle_get_field(OracleHandle* h, const char* name, double* out) {
    auto& s = *h->sim;
    auto it = s.F.find(name);
    if (it == s.F.end()) return 1;
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i) out[(size_t)j * s.nx + i] = it->second(i, j);
    return 0;
}

// particles of plasma species sp in the current step (0 before the first step begins)
int64_t oracle_plasma_count(OracleHandle* h, int sp) {
    const auto& p = h->sim->plasmas;
    return (sp >= 0 && sp < (int)p.size()) ? (int64_t)p[sp].n() : 0;
}
// attributes: x y w ux uy psi x_prev y_prev ux_half uy_half psi_half valid
int oracle_get_plasma(OracleHandle* h, int sp, double* out12) {
    auto& pl = h->sim->plasmas[sp];
    const size_t n = pl.n();
    const std::vector<double>* a[11] = {&pl.x, &pl.y, &pl.w, &pl.ux, &pl.uy, &pl.psi, &pl.x_prev, &pl.y_prev, &pl.ux_h, &pl.uy_h, &pl.psi_h};
    for (int k = 0; k < 11; ++k) std::memcpy(out12 + k * n, a[k]->data(), n * sizeof(double));
    for (size_t i = 0; i < n; ++i) out12[11 * n + i] = pl.valid[i];
    return 0;
}

long long oracle_mg_iterations(OracleHandle* h) { return h->sim->mg_iters_total; }
int oracle_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
const char* oracle_error(OracleHandle* h) { return h->sim->error.c_str(); }

// In-situ data of the last diagnostic step: "fields" or a beam name. Layout (the reference's
// reduced-diagnostic arrays, value index outer, slice inner): beam: 22 x nz values (entry 0 the
// sum of weights, the others divided by it), nz particle counts, 22 sums over slices, the total
// count; fields: 10 x nz values, 10 sums.
int oracle_n_cell(OracleHandle* h, int* n) {
    for (int d = 0; d < 3; ++d) n[d] = h->sim->cfg.n_cell[d];
    return 0;
}
int oracle_adjoint_nparams(OracleHandle* h) {
    return h->sim->cfg.adjoint.witness < 0 ? 0 : h->sim->cfg.adjoint.n_params();
}
// objective (and its gradient when grad != NULL) for parameters theta; 0 on success
int oracle_adjoint(OracleHandle* h, const double* theta, double* grad, double* J) {
    oracle::Sim& s = *h->sim;
    if (s.cfg.adjoint.witness < 0) return 1;
    for (size_t b = 0; b < s.cfg.beams.size(); ++b) if (!s.store_valid[b]) return 2;
    *J = grad ? s.adjoint_grad(theta, grad) : s.adjoint_objective(theta);
    return s.mg_status;
}
long long oracle_insitu_size(OracleHandle* h, const char* what) {
    auto& s = *h->sim;
    if (std::string(what) == "fields") return 11LL * s.nz;
    for (size_t b = 0; b < s.cfg.beams.size(); ++b)
        if (s.cfg.beams[b].name == what) return 23LL * s.nz + 23;
    return -1;
}
int oracle_get_insitu(OracleHandle* h, const char* what, double* out) {
    auto& s = *h->sim;
    const int nz = s.nz;
    if (std::string(what) == "fields") {
        if (s.insitu_fields.empty()) return 1;
        std::vector<double> sum(10, 0.0);
        for (int isl = nz - 1; isl >= 0; --isl)
            for (int k = 0; k < 10; ++k) sum[k] += s.insitu_fields[(size_t)isl * 10 + k];
        for (int k = 0; k < 10; ++k)
            for (int isl = 0; isl < nz; ++isl) out[(size_t)k * nz + isl] = s.insitu_fields[(size_t)isl * 10 + k];
        for (int k = 0; k < 10; ++k) out[(size_t)10 * nz + k] = sum[k];
        return 0;
    }
    for (size_t b = 0; b < s.cfg.beams.size(); ++b) {
        if (s.cfg.beams[b].name != what) continue;
        const auto& r = s.insitu_beam[b];
        if (r.empty()) return 1;
        std::vector<double> sum(23, 0.0);
        for (int isl = nz - 1; isl >= 0; --isl)
            for (int k = 0; k < 23; ++k) sum[k] += r[(size_t)isl * 23 + k];
        for (int isl = 0; isl < nz; ++isl) {
            const double sw = r[(size_t)isl * 23];
            const double inv = sw <= 0. ? 0. : 1. / sw;
            for (int k = 0; k < 22; ++k) out[(size_t)k * nz + isl] = r[(size_t)isl * 23 + k] * (k == 0 ? 1. : inv);
            out[(size_t)22 * nz + isl] = r[(size_t)isl * 23 + 22];
        }
        for (int k = 0; k < 23; ++k) out[(size_t)23 * nz + k] = sum[k];
        return 0;
    }
    return 2;
}

}  // extern "C"
