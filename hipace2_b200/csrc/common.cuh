// Device-side building blocks shared by the slice-loop kernels: shape factors, field views,
// atomics and launch helpers. Everything here is written for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <stdexcept>
#include <string>
#include <utility>

namespace hpq {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define HPQ_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::hpq::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) +      \
                                   " (" __FILE__ ":" + std::to_string(__LINE__) + ")");       \
    } while (0)

// kernel launches issued by this thread (each launch site is followed by one check)
inline thread_local long long g_launches = 0;
#define HPQ_LAUNCH_CHECK()                  \
    do {                                    \
        HPQ_CUDA(cudaGetLastError());       \
        ++::hpq::g_launches;                \
    } while (0)

// Programmatic dependent launch: every kernel starts with this prologue. It lets the next kernel
// of the stream (or graph) launch once all blocks of this one are running, then waits until the
// previous kernel has completed and its memory is visible. Without a programmatic predecessor
// both instructions return at once.
#define HPQ_PDL_ENTRY()                                                         \
    do {                                                                        \
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");         \
        asm volatile("griddepcontrol.wait;" ::: "memory");                      \
    } while (0)

// launches with the programmatic-serialization attribute (HPQ_PDL=0 in the environment turns it off)
inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = getenv("HPQ_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}
template <typename... KArgs, typename... Args>
inline void hpq_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    HPQ_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

constexpr int kGuardAlloc = 3;   // allocated guard cells per side
constexpr int kGuardPhys = 2;    // guard cells of the reference slice arrays (Fields.cpp:63)

// 2-D view of one field component: element (i, j) of the interior index space.
template <class R>
struct F2 {
    R* p;
    int pitch;
    __host__ __device__ R& operator()(int i, int j) const {
        return p[(ptrdiff_t)(j + kGuardAlloc) * pitch + (i + kGuardAlloc)];
    }
    __host__ __device__ R* ptr(int i, int j) const {
        return p + (ptrdiff_t)(j + kGuardAlloc) * pitch + (i + kGuardAlloc);
    }
};

// ------------------------------------------------------------------------------------------
// Shape factors, transverse order 2 (ShapeFactors.H:150-171 and the derivative shapes of
// :212-468). Each returns weight and cell index for stencil point ix.
// ------------------------------------------------------------------------------------------
template <class R>
struct Sh { R s; int cell; };
template <class R>
struct DSh { R s, ds; int cell; };

template <class R>
__device__ __forceinline__ Sh<R> shape2(R xmid, int ix) {
    const R xfloor = floor(xmid + R(0.5));
    const R xint = xmid - xfloor;
    const int c = (int)xfloor;
    if (ix == 0) return {R(0.5) * (R(0.5) - xint) * (R(0.5) - xint), c - 1};
    if (ix == 1) return {R(0.75) - xint * xint, c};
    return {R(0.5) * (R(0.5) + xint) * (R(0.5) + xint), c + 1};
}

// derivative type 1 ("nodal"), 4 points; used by the field gather (FieldGather.H:67)
template <class R>
__device__ __forceinline__ DSh<R> dshape_nodal2(R xmid, int ix) {
    const R xfloor = floor(xmid);
    const R xint = xmid - xfloor, x2 = xint * xint;
    const bool lo = xint < R(0.5);
    const int c = (int)xfloor - 1 + ix;
    if (ix == 0) return {lo ? R(0.5) * x2 - R(0.5) * xint + R(1.0 / 8.0) : R(0), -(R(-0.5) * x2 + xint - R(0.5)), c};
    if (ix == 1) return {lo ? R(3.0 / 4.0) - x2 : R(0.5) * x2 - R(1.5) * xint + R(9.0 / 8.0), -(R(1.5) * x2 - R(2) * xint), c};
    if (ix == 2) return {lo ? R(0.5) * x2 + R(0.5) * xint + R(1.0 / 8.0) : -x2 + R(2) * xint - R(1.0 / 4.0), -(R(-1.5) * x2 + xint + R(0.5)), c};
    return {lo ? R(0) : R(0.5) * x2 - R(0.5) * xint + R(1.0 / 8.0), -(R(0.5) * x2), c};
}

// derivative types 0 (analytic, 3 points), 1 (nodal, 4) and 2 (centred, 5) for the explicit
// Sx/Sy deposition (ExplicitDeposition.cpp:173-176)
template <class R, int TYPE>
__device__ __forceinline__ DSh<R> dshape2(R xmid, int ix) {
    if constexpr (TYPE == 0) {
        xmid += R(0.5);
        const R xfloor = floor(xmid);
        const R xint = xmid - xfloor, x2 = xint * xint;
        const int c = (int)xfloor - 1 + ix;
        if (ix == 0) return {R(0.5) * x2 - xint + R(0.5), -(xint - R(1)), c};
        if (ix == 1) return {-x2 + xint + R(0.5), -(R(1) - R(2) * xint), c};
        return {R(0.5) * x2, -xint, c};
    } else if constexpr (TYPE == 1) {
        return dshape_nodal2<R>(xmid, ix);
    } else {
        xmid += R(0.5);
        const R xfloor = floor(xmid);
        const R xint = xmid - xfloor, x2 = xint * xint;
        const int c = (int)xfloor - 2 + ix;
        if (ix == 0) return {R(0), -(R(-0.25) * x2 + R(0.5) * xint - R(0.25)), c};
        if (ix == 1) return {R(0.5) * x2 - xint + R(0.5), -(R(0.5) * x2 - R(0.5) * xint - R(0.25)), c};
        if (ix == 2) return {-x2 + xint + R(0.5), -(R(0.25) - R(0.5) * xint), c};
        if (ix == 3) return {R(0.5) * x2, -(R(-0.5) * x2 + R(0.5) * xint + R(0.25)), c};
        return {R(0), -(R(0.25) * x2), c};
    }
}

// Shape factors of any transverse order 0..3 (ShapeFactors.H:130-197 for the deposits,
// :212-468 for the derivative shapes of the gather and the explicit deposition): the quadratic
// ones are the functions above, the others the B-splines of order 0, 1 and 3 and their
// derivative forms (analytic, nodal, centred). Stencil points: ORD + 1 for shapeN,
// ORD + TYPE + 1 for dshapeN (ORD + 3 for the centred type 2).
template <class R, int ORD>
__device__ __forceinline__ Sh<R> shapeN(R xmid, int ix) {
    if constexpr (ORD == 2) {
        return shape2<R>(xmid, ix);
    } else if constexpr (ORD == 0) {
        return {R(1), (int)floor(xmid + R(0.5))};
    } else if constexpr (ORD == 1) {
        const R xf = floor(xmid), xi = xmid - xf;
        return {ix == 0 ? R(1) - xi : xi, (int)xf + ix};
    } else {
        const R xf = floor(xmid), xi = xmid - xf, xm = R(1) - xi;
        const int c = (int)xf - 1 + ix;
        if (ix == 0) return {R(1.0 / 6.0) * xm * xm * xm, c};
        if (ix == 1) return {R(2.0 / 3.0) - xi * xi * (R(1) - xi / R(2)), c};
        if (ix == 2) return {R(2.0 / 3.0) - xm * xm * (R(1) - R(0.5) * xm), c};
        return {R(1.0 / 6.0) * xi * xi * xi, c};
    }
}
template <int TYPE, int ORD>
__host__ __device__ constexpr int dshape_points() { return TYPE == 2 ? ORD + 3 : ORD + TYPE + 1; }

template <class R, int TYPE, int ORD>
__device__ __forceinline__ DSh<R> dshapeN(R xmid, int ix) {
    if constexpr (ORD == 2) {
        return dshape2<R, TYPE>(xmid, ix);
    } else if constexpr (TYPE == 0) {  // analytic derivative
        if constexpr (ORD == 0) {
            return {R(1), R(0), (int)floor(xmid + R(0.5))};
        } else if constexpr (ORD == 1) {
            const R xf = floor(xmid), xi = xmid - xf;
            return ix == 0 ? DSh<R>{R(1) - xi, R(1), (int)xf} : DSh<R>{xi, R(-1), (int)xf + 1};
        } else {
            const R xf = floor(xmid), xi = xmid - xf, x2 = xi * xi, x3 = x2 * xi;
            const int c = (int)xf - 1 + ix;
            if (ix == 0) return {R(-1.0 / 6.0) * x3 + R(0.5) * x2 - R(0.5) * xi + R(1.0 / 6.0), -(R(-0.5) * x2 + xi - R(0.5)), c};
            if (ix == 1) return {R(0.5) * x3 - x2 + R(2.0 / 3.0), -(R(1.5) * x2 - R(2) * xi), c};
            if (ix == 2) return {R(-0.5) * x3 + R(0.5) * x2 + R(0.5) * xi + R(1.0 / 6.0), -(R(-1.5) * x2 + xi + R(0.5)), c};
            return {R(1.0 / 6.0) * x3, -(R(0.5) * x2), c};
        }
    } else if constexpr (TYPE == 1) {  // nodal derivative
        if constexpr (ORD == 0) {
            const R xf = floor(xmid), xi = xmid - xf;
            const bool lo = xi < R(0.5);
            return ix == 0 ? DSh<R>{lo ? R(1) : R(0), R(1), (int)xf} : DSh<R>{lo ? R(0) : R(1), R(-1), (int)xf + 1};
        } else if constexpr (ORD == 1) {
            const R xm = xmid + R(0.5), xf = floor(xm), xi = xm - xf;
            const bool lo = xi < R(0.5);
            const int c = (int)xf - 1 + ix;
            if (ix == 0) return {lo ? R(0.5) - xi : R(0), -(xi - R(1)), c};
            if (ix == 1) return {lo ? xi + R(0.5) : R(1.5) - xi, -(R(1) - R(2) * xi), c};
            return {lo ? R(0) : xi - R(0.5), -xi, c};
        } else {
            const R xm = xmid + R(0.5), xf = floor(xm), xi = xm - xf, x2 = xi * xi, x3 = x2 * xi;
            const bool lo = xi < R(0.5);
            const int c = (int)xf - 2 + ix;
            if (ix == 0)
                return {lo ? R(-1.0 / 6.0) * x3 + R(0.25) * x2 - R(0.125) * xi + R(1.0 / 48.0) : R(0),
                        -(R(1.0 / 6.0) * x3 - R(0.5) * x2 + R(0.5) * xi - R(1.0 / 6.0)), c};
            if (ix == 1)
                return {lo ? R(0.5) * x3 - R(0.25) * x2 - R(0.625) * xi + R(23.0 / 48.0)
                           : R(-1.0 / 6.0) * x3 + R(0.75) * x2 - R(1.125) * xi + R(9.0 / 16.0),
                        -(R(-2.0 / 3.0) * x3 + R(1.5) * x2 - R(0.5) * xi - R(0.5)), c};
            if (ix == 2)
                return {lo ? R(-0.5) * x3 - R(0.25) * x2 + R(0.625) * xi + R(23.0 / 48.0)
                           : R(0.5) * x3 - R(1.75) * x2 + R(1.375) * xi + R(17.0 / 48.0),
                        -(x3 - R(1.5) * x2 - R(0.5) * xi + R(0.5)), c};
            if (ix == 3)
                return {lo ? R(1.0 / 6.0) * x3 + R(0.25) * x2 + R(0.125) * xi + R(1.0 / 48.0)
                           : R(-0.5) * x3 + R(1.25) * x2 - R(0.375) * xi + R(5.0 / 48.0),
                        -(R(-2.0 / 3.0) * x3 + R(0.5) * x2 + R(0.5) * xi + R(1.0 / 6.0)), c};
            return {lo ? R(0) : R(1.0 / 6.0) * x3 - R(0.25) * x2 + R(0.125) * xi - R(1.0 / 48.0), -(R(1.0 / 6.0) * x3), c};
        }
    } else {  // centred derivative
        if constexpr (ORD == 0) {
            const R xf = floor(xmid + R(0.5));
            const int c = (int)xf - 1 + ix;
            if (ix == 0) return {R(0), R(0.5), c};
            if (ix == 1) return {R(1), R(0), c};
            return {R(0), R(-0.5), c};
        } else if constexpr (ORD == 1) {
            const R xf = floor(xmid), xi = xmid - xf;
            const int c = (int)xf - 1 + ix;
            if (ix == 0) return {R(0), -(R(0.5) * xi - R(0.5)), c};
            if (ix == 1) return {R(1) - xi, -(R(-0.5) * xi), c};
            if (ix == 2) return {xi, -(R(0.5) - R(0.5) * xi), c};
            return {R(0), -(R(0.5) * xi), c};
        } else {
            const R xf = floor(xmid), xi = xmid - xf, x2 = xi * xi, x3 = x2 * xi;
            const int c = (int)xf - 2 + ix;
            if (ix == 0) return {R(0), -(R(1.0 / 12.0) * x3 - R(0.25) * x2 + R(0.25) * xi - R(1.0 / 12.0)), c};
            if (ix == 1)
                return {R(-1.0 / 6.0) * x3 + R(0.5) * x2 - R(0.5) * xi + R(1.0 / 6.0), -(R(-0.25) * x3 + R(0.5) * x2 - R(1.0 / 3.0)), c};
            if (ix == 2) return {R(0.5) * x3 - x2 + R(2.0 / 3.0), -(R(1.0 / 6.0) * x3 - R(0.5) * xi), c};
            if (ix == 3)
                return {R(-0.5) * x3 + R(0.5) * x2 + R(0.5) * xi + R(1.0 / 6.0), -(R(1.0 / 6.0) * x3 - R(0.5) * x2 + R(1.0 / 3.0)), c};
            if (ix == 4)
                return {R(1.0 / 6.0) * x3, -(R(-0.25) * x3 + R(0.25) * x2 + R(0.25) * xi + R(1.0 / 12.0)), c};
            return {R(0), -(R(1.0 / 12.0) * x3), c};
        }
    }
}

// Position in cell units clamped to [-1, n - 1/2]: identity for particles inside the domain
// (xmid in [-0.5, n-0.5]); keeps NaN/inf positions from indexing outside the three guard cells
// with any stencil of order <= 3.
template <class R>
__device__ __forceinline__ R clamp_mid(R xmid, int n) {
    return fmin(fmax(xmid, R(-1)), R(n) - R(0.5));
}

// grid-stride loop helpers
__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

inline int blocks_for(long long n, int threads, int max_blocks = 148 * 16) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

// atomicMax on non-negative doubles through their bit pattern (monotone for x >= 0)
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
    atomicMax(reinterpret_cast<unsigned int*>(addr), (unsigned int)__float_as_int(v));
}

}  // namespace hpq
