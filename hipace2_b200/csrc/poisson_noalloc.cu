// Allocation-free Dirichlet Poisson solve (hpq_poisson_dirichlet_noalloc in include/hpq.h).
//
// Some callers of this library cannot call cudaMalloc: code that runs while a CUDA stream is
// being captured into a graph (allocation is not a capturable operation), plugins of host
// frameworks that own the device memory pool and forbid side allocations, and real-time loops
// that must not pay for or fail on an allocation at solve time. This entry point serves them:
// the caller passes the right-hand side and the solution buffer; the temporaries of the solve
// (the transformed intermediate, the eigenvalues and the FFT twiddles) live in one file-scope
// device array of fixed size. CUDA loads the library's device code lazily, so the array's
// memory is committed on a device by the first call on that device (which can therefore fail
// with HPQ_ERR_CUDA when the device is already full) and held until the process exits.
//
// Limit: nx and ny of the form 2^k - 1 with 31 <= n <= 1023 (the shared-memory FFT path of the
// DST-I), i.e. at most 1023 x 1023 cells; the scratch array is 16.1 MiB.
// All calls share the array and it keeps the contents of the last call. Every element a solve
// reads is written earlier in the same solve, so nothing needs clearing between calls; two
// calls whose kernels overlap on the GPU (different streams, or different host threads on one
// stream without ordering) race on the array and give wrong results.
// Errors: a CUDA error already pending when the call starts is left to the caller (the call
// returns HPQ_ERR_CUDA without launching or clearing it); each launch is checked right after it
// is made.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hpq.h"
#include "fftdst.cuh"

namespace {

constexpr int kMaxN = 1023;
constexpr size_t kPlane = (size_t)kMaxN * kMaxN;          // one nx x ny plane
constexpr size_t kTw = 2048;                               // complex twiddles: M/2 for x and y
constexpr size_t kScratchDoubles = 2 * kPlane + 2 * kTw;   // work plane, eigenvalues, twiddles

static __device__ __align__(256) double g_poisson_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

cudaError_t set_smem_attributes();

// Set-up, once per device with that device current: the host address of the array is only a
// stand-in, kernels must be given the device address returned here. The shared-memory limits of
// the pass kernels are raised at the same time, so later calls make no set-up call at all.
int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HPQ_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_poisson_scratch) != cudaSuccess || !p) return HPQ_ERR_CUDA;
        if (set_smem_attributes() != cudaSuccess) return HPQ_ERR_CUDA;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return HPQ_OK;
}

// eigenvalues of the 5-point Laplacian with the normalisation of the two DST-I per axis
__global__ void k_fill_eig(double* eig, int nx, int ny, double dx, double dy) {
    const double pi = 3.14159265358979323846;
    const double sxf = pi / (2. * (nx + 1)), syf = pi / (2. * (ny + 1));
    const double norm = (2.0 / (nx + 1)) * (2.0 / (ny + 1));
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < (long long)nx * ny;
         k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        double a = sin((i + 1) * sxf), b = sin((j + 1) * syf);
        a *= a;
        b *= b;
        eig[k] = norm / (-4.0 * (a / (dx * dx) + b / (dy * dy)));
    }
}

__global__ void k_fill_twiddles(hpq::Cx<double>* tw, int M) {
    const double pi = 3.14159265358979323846;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M / 2; k += gridDim.x * blockDim.x)
        tw[k] = {cos(2 * pi * k / M), -sin(2 * pi * k / M)};
}

// shared memory of one block of a pass: rb/2 complex rows of length M (the eigenvalue pass adds
// rb rows of n <= kMaxN reals)
template <int M>
constexpr size_t smem_t() { return (size_t)(hpq::DstCfg<M>::RB / 2) * M * sizeof(hpq::Cx<double>); }

template <int M, int LOGM>
cudaError_t set_attrs_for() {
    constexpr int RB = hpq::DstCfg<M>::RB;
    cudaError_t e = cudaFuncSetAttribute(hpq::k_dst_pass_t<double, M, LOGM, RB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t<M>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hpq::k_dst_pass_eig<double, M, LOGM, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(smem_t<M>() + (size_t)RB * kMaxN * sizeof(double)));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hpq::k_dst_pass_field<double, M, LOGM, RB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t<M>());
    return e;
}

cudaError_t set_smem_attributes() {
    cudaError_t e = set_attrs_for<64, 6>();
    if (e == cudaSuccess) e = set_attrs_for<128, 7>();
    if (e == cudaSuccess) e = set_attrs_for<256, 8>();
    if (e == cudaSuccess) e = set_attrs_for<512, 9>();
    if (e == cudaSuccess) e = set_attrs_for<1024, 10>();
    if (e == cudaSuccess) e = set_attrs_for<2048, 11>();
    return e;
}

template <int M, int LOGM>
cudaError_t pass_t(cudaStream_t st, const double* in, int nrows, int n, int rpp, double* out,
                   const hpq::Cx<double>* tw) {
    const int rb = hpq::DstCfg<M>::RB;
    const size_t smem = smem_t<M>();
    hpq::k_dst_pass_t<double, M, LOGM, hpq::DstCfg<M>::RB><<<(nrows + rb - 1) / rb, 256, smem, st>>>(in, nrows, n, rpp, out, tw);
    return cudaGetLastError();
}

template <int M, int LOGM>
cudaError_t pass_eig(cudaStream_t st, const double* in, int nrows, int n, int rpp, const double* eig,
                     double* out, const hpq::Cx<double>* tw) {
    const int rb = hpq::DstCfg<M>::RB;
    const size_t smem = smem_t<M>() + (size_t)rb * n * sizeof(double);
    hpq::k_dst_pass_eig<double, M, LOGM, hpq::DstCfg<M>::RB><<<(nrows + rb - 1) / rb, 256, smem, st>>>(in, nrows, n, rpp, eig, out, tw);
    return cudaGetLastError();
}

// The last x-pass writes a plain nx x ny plane (the caller's solution buffer): a slab view with
// no guard cells, i.e. pitch nx and the guard offset removed from the base pointer.
template <int M, int LOGM>
cudaError_t pass_plane(cudaStream_t st, const double* in, int nrows, int n, int ny, double* out,
                       const hpq::Cx<double>* tw) {
    const int rb = hpq::DstCfg<M>::RB;
    const size_t smem = smem_t<M>();
    const int G = hpq::kGuardAlloc;
    double* base = out - ((ptrdiff_t)G * n + G);  // element (i, j) -> out[j * n + i]
    hpq::k_dst_pass_field<double, M, LOGM, hpq::DstCfg<M>::RB><<<(nrows + rb - 1) / rb, 256, smem, st>>>(
        in, nrows, n, ny, base, 0, n, 0, 0, 0, tw);
    return cudaGetLastError();
}

int pow2_len(int n) {
    const int m = 2 * (n + 1);
    return (n >= 31 && n <= kMaxN && (m & (m - 1)) == 0) ? m : 0;
}

#define HPQ_NOALLOC_DISPATCH(Mval, CALL) \
    switch (Mval) {                      \
        case 64: e = CALL(64, 6); break;   \
        case 128: e = CALL(128, 7); break; \
        case 256: e = CALL(256, 8); break; \
        case 512: e = CALL(512, 9); break; \
        case 1024: e = CALL(1024, 10); break; \
        case 2048: e = CALL(2048, 11); break; \
        default: return HPQ_ERR_ARG;     \
    }

}  // namespace

extern "C" int hpq_poisson_dirichlet_noalloc(const double* f, double* u, int nx, int ny, double dx, double dy,
                                             void* stream) {
    if (!f || !u || !(dx > 0) || !(dy > 0)) return HPQ_ERR_ARG;
    if (nx > kMaxN || ny > kMaxN) return HPQ_ERR_TOO_LARGE;
    const int Mx = pow2_len(nx), My = pow2_len(ny);
    if (!Mx || !My) return HPQ_ERR_ARG;
    // an error left pending by the caller's earlier work stays the caller's: nothing is launched
    // and it is not cleared
    if (cudaPeekAtLastError() != cudaSuccess) return HPQ_ERR_CUDA;
    double* scratch = nullptr;
    if (int r = scratch_for_current_device(&scratch)) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* work = scratch;                        // y-transformed intermediate, nx*ny
    double* eig = scratch + kPlane;                // eigenvalues, nx*ny
    auto* twx = reinterpret_cast<hpq::Cx<double>*>(scratch + 2 * kPlane);  // Mx/2 complex
    auto* twy = twx + kTw / 2;                                              // My/2 complex
    k_fill_eig<<<148, 256, 0, st>>>(eig, nx, ny, dx, dy);
    if (cudaGetLastError() != cudaSuccess) return HPQ_ERR_CUDA;
    k_fill_twiddles<<<4, 256, 0, st>>>(twx, Mx);
    if (cudaGetLastError() != cudaSuccess) return HPQ_ERR_CUDA;
    k_fill_twiddles<<<4, 256, 0, st>>>(twy, My);
    if (cudaGetLastError() != cudaSuccess) return HPQ_ERR_CUDA;
    cudaError_t e = cudaSuccess;
    // x-pass of f -> u (transposed, u serves as the temporary); y-pass * eig * y-pass of u ->
    // work; x-pass of work -> u. No pass reads and writes the same buffer.
#define CALL1(M, L) pass_t<M, L>(st, f, ny, nx, ny, u, twx)
    HPQ_NOALLOC_DISPATCH(Mx, CALL1)
#undef CALL1
    if (e != cudaSuccess) return HPQ_ERR_CUDA;
#define CALL2(M, L) pass_eig<M, L>(st, u, nx, ny, nx, eig, work, twy)
    HPQ_NOALLOC_DISPATCH(My, CALL2)
#undef CALL2
    if (e != cudaSuccess) return HPQ_ERR_CUDA;
#define CALL3(M, L) pass_plane<M, L>(st, work, ny, nx, ny, u, twx)
    HPQ_NOALLOC_DISPATCH(Mx, CALL3)
#undef CALL3
    if (e != cudaSuccess) return HPQ_ERR_CUDA;
    return HPQ_OK;
}
