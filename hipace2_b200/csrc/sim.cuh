// The slice-loop driver: owns device memory, initialises plasma and beams, and sequences the
// kernels of one slice (Hipace::SolveOneSlice, Hipace.cpp:556-728) for the explicit and the
// predictor-corrector Bx/By solvers. R is the field/plasma precision (double: plain FP64 path;
// float: mixed path); beam particles are always FP64.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "common.cuh"
#include "salame.cuh"
#include "config.hpp"
#include "dst.cuh"
#include <type_traits>
#include "kernels.cuh"
#include "mg.cuh"
#include "rng.hpp"

namespace hpq {

struct HostBeam {
    std::vector<double> x, y, z, w, ux, uy, uz;
    std::vector<long long> id;
    size_t size() const { return x.size(); }
    void push(double a, double b, double c, double ww, double d, double e, double f, long long i) {
        x.push_back(a); y.push_back(b); z.push_back(c); w.push_back(ww); ux.push_back(d); uy.push_back(e); uz.push_back(f); id.push_back(i);
    }
};

struct Stats {
    long long mg_vcycles = 0;
    int mg_status = 0;
    long long plasma_pushes = 0;
    long long beam_particles = 0;
    long long slices = 0;
    long long launches = 0;
};

class SimBase {
public:
    virtual ~SimBase() = default;
    virtual void init() = 0;
    virtual void set_beam(int b, const double* x, const double* y, const double* z, const double* w, const double* ux,
                          const double* uy, const double* uz, const long long* id, long long n) = 0;
    virtual long long beam_count(int b) = 0;
    // time-step pipeline hand-off (MultiBuffer.cpp:181-430): the particles that slice islice of
    // the current (or last) step hands to the next step, and the particles of slice islice of the
    // current step received from the rank that ran the previous step
    virtual long long beam_slice_count(int b, int islice) = 0;
    virtual void get_beam_slice(int b, int islice, double* x, double* y, double* z, double* w, double* ux, double* uy,
                                double* uz, long long* id) = 0;
    virtual void put_beam_slice(int b, int islice, const double* x, const double* y, const double* z, const double* w,
                                const double* ux, const double* uy, const double* uz, const long long* id,
                                long long n) = 0;
    virtual void set_time(double t) = 0;
    virtual void get_beam(int b, double* x, double* y, double* z, double* w, double* ux, double* uy, double* uz,
                          long long* id) = 0;
    virtual void begin_step(int step) = 0;
    virtual void solve_slice(int islice) = 0;
    virtual void end_step() = 0;
    virtual void get_field(const std::string& name, double* out) = 0;
    virtual void set_diag(const std::vector<std::string>& names) = 0;
    virtual void get_diag(const std::string& name, double* out) = 0;
    virtual long long plasma_count(int sp) = 0;
    virtual void get_plasma(int sp, double* out12) = 0;
    virtual void synchronize() = 0;
    virtual cudaStream_t stream() = 0;
    virtual Stats stats() = 0;
    virtual void set_graphs(bool on) = 0;
    virtual void set_deterministic(bool on) = 0;
    // in-situ data of the last diagnostic step ("fields" or a beam name); size < 0: unknown name
    virtual long long insitu_size(const std::string& what) = 0;
    virtual bool get_insitu(const std::string& what, double* out) = 0;
    virtual void set_profiling(bool on) = 0;
    virtual bool get_profile(const std::string& name, double* ms, long long* n) = 0;
    // adjoint of one step (double precision): number of parameters, objective and gradient
    virtual int adjoint_nparams() const = 0;
    virtual double adjoint(const double* theta, double* grad) = 0;
    virtual std::string profile_names() = 0;
    // physical time at which the next step starts (infinite once the step at max_time ran)
    virtual double time() const = 0;
    // SALAME record: (slice, iteration, weight factor) of every iteration since hpq_init
    virtual const std::vector<double>& salame_record() const = 0;
    const SimConfig& config() const { return cfg; }
    SimConfig cfg;
};

inline int comp_from_name(const std::string& n, bool explicit_solver) {
    static const std::map<std::string, int> ex = {
        {"chi", C_CHI}, {"Sy", C_SY}, {"Sx", C_SX}, {"ExmBy", C_EXMBY}, {"EypBx", C_EYPBX}, {"Ez", C_EZ},
        {"Bx", C_BX}, {"By", C_BY}, {"Bz", C_BZ}, {"Psi", C_PSI}, {"jx_beam", C_JXB}, {"jy_beam", C_JYB},
        {"jz_beam", C_JZB}, {"jx", C_JX}, {"jy", C_JY}, {"rhomjz", C_RHOMJZ}, {"rho", C_RHO},
        {"rhomjz_beam", C_RHOMJZB}, {"Next.jx_beam", C_NJXB}, {"Next.jy_beam", C_NJYB},
        {"Prev.jx_beam", C_PJXB}, {"Prev.jy_beam", C_PJYB}, {"Ions.rhomjz", C_IONS}};
    static const std::map<std::string, int> pc = {
        {"ExmBy", C_EXMBY}, {"EypBx", C_EYPBX}, {"Ez", C_EZ}, {"Bx", C_BX}, {"By", C_BY}, {"Bz", C_BZ},
        {"Psi", C_PSI}, {"jx", C_JX}, {"jy", C_JY}, {"jz", C_JZ}, {"rhomjz", C_RHOMJZ}, {"rho", C_RHO},
        {"Next.jx", C_NJX}, {"Next.jy", C_NJY}, {"Prev.Bx", C_PBX}, {"Prev.By", C_PBY}, {"Prev.jx", C_PJX},
        {"Prev.jy", C_PJY}, {"PCIter.Bx", C_PCIBX}, {"PCIter.By", C_PCIBY}, {"PCPrevIter.Bx", C_PCPBX},
        {"PCPrevIter.By", C_PCPBY}, {"Ions.rhomjz", C_IONS}};
    const auto& m = explicit_solver ? ex : pc;
    auto it = m.find(n);
    if (it == m.end()) throw InputError("unknown field component '" + n + "'");
    return it->second;
}

// ------------------------------------------------------------------------------------------
// PC helper kernels (Fields.cpp:1149-1286)
// ------------------------------------------------------------------------------------------
// first error of a slice -> initial-guess mixing factor (InitialBfieldGuess)
__device__ __forceinline__ void pc_guess_factor(Ctl* ctl, double tol) {
    const double err = ctl->pc_sum[0] > 0 ? ctl->pc_sum[1] / ctl->pc_sum[0] : 0.0;
    ctl->pc_sum[0] = ctl->pc_sum[1] = 0;
    ctl->pc_mix = exp(-0.5 * pow(err / (2.5 * tol), 2));
    ctl->pc_iter = 0;
    ctl->pc_err = 1.0;
    ctl->pc_err_prev = 1.0;
    ctl->pc_go = 1.0 > tol;
}
// error of one iteration -> mixing weights and whether to continue (MixAndShiftBfields)
__device__ __forceinline__ void pc_iter_factor(Ctl* ctl) {
    const double err = ctl->pc_sum[0] > 0 ? ctl->pc_sum[1] / ctl->pc_sum[0] : 0.0;
    ctl->pc_sum[0] = ctl->pc_sum[1] = 0;
    ctl->pc_iter += 1;
    double prev = ctl->pc_err_prev;
    if (ctl->pc_iter == 1) prev = err;
    double wi, wp;
    if (err != 0. || prev != 0.) { wi = prev / (err + prev); wp = err / (err + prev); }
    else { wi = 0.5; wp = 0.5; }
    ctl->pc_w[0] = wi; ctl->pc_w[1] = wp;
    ctl->pc_err = err;
    ctl->pc_err_prev = err;
    ctl->pc_mixnow = 1;
}

// Norms of (B) and (B - B_iter) summed over the interior into Ctl::pc_sum; the last block to
// finish turns them into the guess factor (gated == 0, the first norms of a slice) or the
// iteration weights (gated == 1, skipped with the whole kernel once the loop has stopped)
template <class R>
__global__ void k_pc_norms(Slab<R> S, int bx, int by, int bxi, int byi, Ctl* ctl, int gated, double tol) {
    HPQ_PDL_ENTRY();
    if (gated && !ctl->pc_go) return;
    const F2<R> Bx = S.c(bx), By = S.c(by), Bxi = S.c(bxi), Byi = S.c(byi);
    double nb = 0, nd = 0;
    for (long long k = gtid(); k < (long long)S.nx * S.ny; k += gstride()) {
        const int i = (int)(k % S.nx), j = (int)(k / S.nx);
        const double a = Bx(i, j), b = By(i, j), c = Bxi(i, j), d = Byi(i, j);
        nb += sqrt(a * a + b * b);
        nd += sqrt((a - c) * (a - c) + (b - d) * (b - d));
    }
    for (int o = 16; o > 0; o >>= 1) { nb += __shfl_xor_sync(0xffffffffu, nb, o); nd += __shfl_xor_sync(0xffffffffu, nd, o); }
    __shared__ double wb[32], wd[32];
    __shared__ int last;
    if (gridDim.x > 1) {
        if ((threadIdx.x & 31) == 0) { atomicAdd(&ctl->pc_sum[0], nb); atomicAdd(&ctl->pc_sum[1], nd); }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            last = atomicAdd(&ctl->pc_cnt[0], 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (!last || threadIdx.x != 0) return;
        __threadfence();
        ctl->pc_sum[0] = atomic_read(&ctl->pc_sum[0]);
        ctl->pc_sum[1] = atomic_read(&ctl->pc_sum[1]);
        ctl->pc_cnt[0] = 0;
    } else {
        // one block (deterministic mode): warp sums added in warp order by one thread
        if ((threadIdx.x & 31) == 0) { wb[threadIdx.x >> 5] = nb; wd[threadIdx.x >> 5] = nd; }
        __syncthreads();
        if (threadIdx.x != 0) return;
        double sb = 0, sd = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { sb += wb[w]; sd += wd[w]; }
        ctl->pc_sum[0] += sb;
        ctl->pc_sum[1] += sd;
    }
    if (gated) pc_iter_factor(ctl);
    else pc_guess_factor(ctl, tol);
}
template <class R>
__global__ void k_pc_guess(Slab<R> S, const Ctl* ctl) {
    HPQ_PDL_ENTRY();
    const R mix = (R)ctl->pc_mix;
    R *B = S.c(C_BX).p, *By = S.c(C_BY).p, *PB = S.c(C_PBX).p, *PBy = S.c(C_PBY).p;
    R *PCP = S.c(C_PCPBX).p, *PCPy = S.c(C_PCPBY).p, *PCI = S.c(C_PCIBX).p, *PCIy = S.c(C_PCIBY).p;
    for (long long k = gtid(); k < (long long)S.cstride; k += gstride()) {
        const R bx = (R(1) + mix) * PB[k] + (-mix) * PCP[k];
        const R by = (R(1) + mix) * PBy[k] + (-mix) * PCPy[k];
        B[k] = bx; By[k] = by;
        PCI[k] = 0; PCIy[k] = 0;
        PCP[k] = bx; PCPy[k] = by;
    }
}
// B = (1 - a) B + a (wi B_iter + wp B_previter); the last block to finish ends the iteration
// (clears the mix flag, decides whether the loop goes on)
template <class R>
__global__ void k_pc_mix(Slab<R> S, Ctl* ctl, double a, double tol, int maxit) {
    HPQ_PDL_ENTRY();
    if (!ctl->pc_mixnow) return;
    const R wi = (R)ctl->pc_w[0], wp = (R)ctl->pc_w[1], ra = (R)a;
    R *B = S.c(C_BX).p, *By = S.c(C_BY).p;
    R *PCP = S.c(C_PCPBX).p, *PCPy = S.c(C_PCPBY).p, *PCI = S.c(C_PCIBX).p, *PCIy = S.c(C_PCIBY).p;
    R *NJX = S.c(C_NJX).p, *NJY = S.c(C_NJY).p;
    for (long long k = gtid(); k < (long long)S.cstride; k += gstride()) {
        const R px = wi * PCI[k] + wp * PCP[k];
        const R py = wi * PCIy[k] + wp * PCPy[k];
        B[k] = (R(1) - ra) * B[k] + ra * px;
        By[k] = (R(1) - ra) * By[k] + ra * py;
        PCP[k] = PCI[k]; PCPy[k] = PCIy[k];
        NJX[k] = 0; NJY[k] = 0;
    }
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&ctl->pc_cnt[1], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    ctl->pc_cnt[1] = 0;
    ctl->pc_mixnow = 0;
    ctl->pc_go = (ctl->pc_err > tol) && (ctl->pc_iter < maxit);
}

__global__ void k_slice_done(Ctl* ctl) {
    HPQ_PDL_ENTRY(); ctl->islice -= 1; }

// ------------------------------------------------------------------------------------------
template <class R>
class Sim final : public SimBase {
public:
    explicit Sim(const SimConfig& c) { cfg = c; }
    ~Sim() override { release(); }

    Geo g{};
    int nx = 0, ny = 0, nz = 0;
    cudaStream_t st = nullptr;
    Slab<R> S;
    PoissonDST<R> dst;
    PoissonDST<R> pc_dst;  // the two Bx/By solves of the predictor-corrector loop
    PoissonDST<R> sal_dst;  // the Ez solves of the SALAME slice
    // slab components allocated: the slice, plus the SALAME slice when a beam does SALAME
    int ncomp_alloc = C_NCOMP;
    // SALAME state (Hipace.H:284-301): this step runs it, the last SALAME slice, overloading,
    // the zeta where it started, per-beam particle counts of the step's slices (host copy), the
    // device sums of SalameGetW and a record of (slice, iteration, W)
    bool sal_step = false;
    int sal_last = -1;
    bool sal_overloaded = false;
    double sal_zeta0 = 0;
    std::vector<std::vector<int>> sal_count;
    double* sal_sums_d = nullptr;
    double* sal_sums_h = nullptr;
    std::vector<double> salame_log;
    Multigrid<R> mg;
    std::vector<PlasmaDev<R>> pl;
    // plasma reorder (allocated at the first reorder): attribute scratch, keys, permutation and
    // per-bin counts, starts and cursors, scan block totals
    PlasmaDev<R> ro_tmp{};
    int *ro_key = nullptr, *ro_perm = nullptr, *ro_cnt = nullptr, *ro_start = nullptr, *ro_fill = nullptr,
        *ro_bsum = nullptr;
    long long ro_cap = 0, ro_bins = 0;
    std::vector<bool> reordered;  // species reordered since its last reset (lattice order lost)
    std::vector<double*> px0, py0;
    std::vector<std::vector<double>> hx0, hy0;  // lattice points on the host (output of displacements)
    std::vector<BeamDev> bm;
    std::vector<HostBeam> pending_beams;
    std::vector<bool> beam_set;
    Ctl* ctl = nullptr;
    Ctl* ctl_h = nullptr;
    int parity = 0;
    int cur_step = 0;
    int cur_islice = 0;
    double physical_time = 0;
    double next_time = 0;  // physical time after the current step (step_time)
    bool use_graphs = false;
    bool capturing = false;
    cudaStream_t st2 = nullptr;
    // side stream of the two forks of a slice (beam deposit | plasma deposit, beam push and
    // partition | plasma push and copies); not used while profiling, which times kernels serially
    cudaStream_t sts = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // second side stream: the beam push and partition of slice s run beside the solve of slice
    // s - 1 (their results only feed the next step), on a copy SB of slice s's gathered fields
    // (planes C_EZ .. C_PSI); the last slice's beam work runs when the step ends
    cudaStream_t stb = nullptr;
    cudaEvent_t ev_bfork = nullptr, ev_bjoin = nullptr;
    Slab<R> SB;
    cudaStream_t beam_begin() {
        if (profiling) return st;
        HPQ_CUDA(cudaEventRecord(ev_bfork, st));
        HPQ_CUDA(cudaStreamWaitEvent(stb, ev_bfork, 0));
        return stb;
    }
    void beam_end() {
        if (profiling) return;
        HPQ_CUDA(cudaEventRecord(ev_bjoin, stb));
        HPQ_CUDA(cudaStreamWaitEvent(st, ev_bjoin, 0));
    }
    cudaStream_t side_begin() {
        if (profiling) return st;
        HPQ_CUDA(cudaEventRecord(ev_fork, st));
        HPQ_CUDA(cudaStreamWaitEvent(sts, ev_fork, 0));
        return sts;
    }
    void side_end() {
        if (profiling) return;
        HPQ_CUDA(cudaEventRecord(ev_join, sts));
        HPQ_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    }
    // launches of the enclosed code go to stream t (every launch site uses the member `st`)
    struct OnStream {
        Sim* s;
        cudaStream_t old;
        OnStream(Sim* s_, cudaStream_t t) : s(s_), old(s_->st) { s->st = t; }
        ~OnStream() { s->st = old; }
    };
    cudaGraph_t slice_graph = nullptr;
    cudaGraphExec_t slice_exec = nullptr;
    long long graph_nodes = 0;
    long long launches_top = 0, launches_body = 0;  // kernels per slice graph / per V-cycle body
    long long launches_total = 0;                   // kernels launched or replayed so far
    long long body_launch_offset = 0;
    // per-kernel-class timing with CUDA events on the launching stream
    struct ProfEntry {
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
        double ms = 0;
        long long n = 0;
    };
    std::map<std::string, ProfEntry> prof;
    std::vector<cudaEvent_t> ev_pool;
    bool profiling = false;
    cudaEvent_t ev_get() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            HPQ_CUDA(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    struct Scope {
        Sim* s;
        const char* name;
        cudaEvent_t a = nullptr, b = nullptr;
        Scope(Sim* s_, const char* n) : s(s_), name(n) {
            if (s->profiling) { a = s->ev_get(); b = s->ev_get(); HPQ_CUDA(cudaEventRecord(a, s->st)); }
        }
        ~Scope() {
            if (a) { cudaEventRecord(b, s->st); s->prof[name].pending.push_back({a, b}); }
        }
    };
    void prof_collect() {
        for (auto& kv : prof) {
            for (auto& pr : kv.second.pending) {
                float ms = 0;
                HPQ_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
                kv.second.ms += ms;
                kv.second.n += 1;
                ev_pool.push_back(pr.first);
                ev_pool.push_back(pr.second);
            }
            kv.second.pending.clear();
        }
    }
    void set_profiling(bool on) override {
        synchronize();
        prof_collect();
        prof.clear();
        profiling = on;
    }
    bool get_profile(const std::string& name, double* ms, long long* n) override {
        synchronize();
        prof_collect();
        auto it = prof.find(name);
        if (it == prof.end()) { *ms = 0; *n = 0; return false; }
        *ms = it->second.ms;
        *n = it->second.n;
        return true;
    }
    double time() const override { return physical_time; }
    const std::vector<double>& salame_record() const override { return salame_log; }

    std::string profile_names() override {
        std::string r;
        for (auto& kv : prof) r += kv.first + " ";
        return r;
    }
    // diagnostics
    std::vector<std::string> diag_names;
    CompList diag_list{};
    double* diag_buf = nullptr;
    Stats st_host{};

    cudaStream_t stream() override { return st; }
    void set_graphs(bool on) override {
        use_graphs = on;
        if (!on) invalidate_graph();
    }

    void release() {
        if (st) cudaStreamSynchronize(st);
        if (S.base) cudaFree(S.base);
        S.base = nullptr;
        if (SB.base) cudaFree(SB.base);
        SB.base = nullptr;
        if (quad) cudaFree(quad);
        quad = nullptr;
        if (bin_key) cudaFree(bin_key);
        if (bin_hist) cudaFree(bin_hist);
        if (bin_total) cudaFree(bin_total);
        if (valid_h) cudaFreeHost(valid_h);
        valid_h = nullptr;
        valid_cap = valid_n = 0;
        bin_key = bin_hist = nullptr;
        bin_total = nullptr;
        bin_key_cap = bin_hist_cap = 0;
        dst.release();
        pc_dst.release();
        sal_dst.release();
        if (sal_sums_d) cudaFree(sal_sums_d);
        if (sal_sums_h) cudaFreeHost(sal_sums_h);
        sal_sums_d = nullptr;
        sal_sums_h = nullptr;
        mg.release();
        for (auto& p : pl)
            for (void* q : {(void*)p.x, (void*)p.y, (void*)p.w, (void*)p.ux, (void*)p.uy, (void*)p.psi, (void*)p.xp,
                            (void*)p.yp, (void*)p.uxh, (void*)p.uyh, (void*)p.psih, (void*)p.valid, (void*)p.ru,
                            (void*)p.rv})
                if (q) cudaFree(q);
        pl.clear();
        release_reorder();
        hx0.clear(); hy0.clear();
        for (auto* q : px0) cudaFree(q);
        for (auto* q : py0) cudaFree(q);
        px0.clear(); py0.clear();
        for (auto& b : bm) free_beam(b);
        bm.clear();
        for (double* p : insitu_beam_d) if (p) cudaFree(p);
        insitu_beam_d.clear();
        if (insitu_fields_d) cudaFree(insitu_fields_d);
        insitu_fields_d = nullptr;
        if (det_mem) cudaFree(det_mem);
        det_mem = nullptr;
        det = DetAcc{};
        if (ctl) cudaFree(ctl);
        if (ctl_h) cudaFreeHost(ctl_h);
        ctl = nullptr; ctl_h = nullptr;
        if (diag_buf) cudaFree(diag_buf);
        diag_buf = nullptr;
        adj_release();
        for (auto& kv : prof)
            for (auto& pr : kv.second.pending) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
        prof.clear();
        for (auto e : ev_pool) cudaEventDestroy(e);
        ev_pool.clear();
        invalidate_graph();
        if (st2) cudaStreamDestroy(st2);
        st2 = nullptr;
        if (sts) cudaStreamDestroy(sts);
        sts = nullptr;
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        ev_fork = ev_join = nullptr;
        if (stb) cudaStreamDestroy(stb);
        stb = nullptr;
        if (ev_bfork) cudaEventDestroy(ev_bfork);
        if (ev_bjoin) cudaEventDestroy(ev_bjoin);
        ev_bfork = ev_bjoin = nullptr;
        if (st) cudaStreamDestroy(st);
        st = nullptr;
    }

    // ----------------------------------------------------------------------------- init
    void init() override {
        nx = cfg.n_cell[0]; ny = cfg.n_cell[1]; nz = cfg.n_cell[2];
        g.nx = nx; g.ny = ny; g.nz = nz;
        for (int d = 0; d < 3; ++d) {
            g.plo[d] = cfg.prob_lo[d]; g.phi[d] = cfg.prob_hi[d];
            g.dx[d] = (cfg.prob_hi[d] - cfg.prob_lo[d]) / cfg.n_cell[d];
            g.dxi[d] = 1. / g.dx[d];
        }
        g.xoff = 0.5 * (cfg.prob_lo[0] + cfg.prob_hi[0] - g.dx[0] * ((-2) + (nx + 1)));
        g.yoff = 0.5 * (cfg.prob_lo[1] + cfg.prob_hi[1] - g.dx[1] * ((-2) + (ny + 1)));
        g.plo_p[0] = cfg.particle_lo[0]; g.plo_p[1] = cfg.particle_lo[1];
        g.phi_p[0] = cfg.particle_hi[0]; g.phi_p[1] = cfg.particle_hi[1];
        g.bc = (int)cfg.particle_bc;
        g.c = cfg.pc.c; g.ep0 = cfg.pc.ep0; g.mu0 = cfg.pc.mu0;
        g.normalized = cfg.normalized_units;
        if ((int)cfg.beams.size() > kMaxBeams) throw InputError("at most 4 beam species are supported");

        HPQ_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        HPQ_CUDA(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        HPQ_CUDA(cudaStreamCreateWithFlags(&sts, cudaStreamNonBlocking));
        HPQ_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        HPQ_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        HPQ_CUDA(cudaStreamCreateWithFlags(&stb, cudaStreamNonBlocking));
        HPQ_CUDA(cudaEventCreateWithFlags(&ev_bfork, cudaEventDisableTiming));
        HPQ_CUDA(cudaEventCreateWithFlags(&ev_bjoin, cudaEventDisableTiming));
        // slab
        S.nx = nx; S.ny = ny;
        S.pitch = ((nx + 2 * kGuardAlloc + 7) / 8) * 8;
        S.rows = ny + 2 * kGuardAlloc;
        S.cstride = (size_t)S.pitch * S.rows;
        ncomp_alloc = (cfg.explicit_solver && cfg.any_salame()) ? 2 * C_NCOMP : C_NCOMP;
        HPQ_CUDA(cudaMalloc(&S.base, S.cstride * ncomp_alloc * sizeof(R)));
        HPQ_CUDA(cudaMemset(S.base, 0, S.cstride * ncomp_alloc * sizeof(R)));
        SB = S;
        HPQ_CUDA(cudaMalloc(&SB.base, S.cstride * (C_PSI + 1) * sizeof(R)));
        if (cfg.explicit_solver) HPQ_CUDA(cudaMalloc(&quad, S.cstride * sizeof(Quad<R>)));
        HPQ_CUDA(cudaMemset(SB.base, 0, S.cstride * (C_PSI + 1) * sizeof(R)));
        dst.init(nx, ny, g.dx[0], g.dx[1], 3);
        if (!cfg.explicit_solver) pc_dst.init(nx, ny, g.dx[0], g.dx[1], 2);
        if (cfg.explicit_solver) mg.init(nx, ny, g.dx[0], g.dx[1]);
        if (ncomp_alloc > C_NCOMP) {
            sal_dst.init(nx, ny, g.dx[0], g.dx[1], 1);
            HPQ_CUDA(cudaMalloc(&sal_sums_d, 4 * sizeof(double)));
            HPQ_CUDA(cudaMallocHost(&sal_sums_h, 4 * sizeof(double)));
        }
        HPQ_CUDA(cudaMalloc(&ctl, sizeof(Ctl)));
        HPQ_CUDA(cudaMemset(ctl, 0, sizeof(Ctl)));
        HPQ_CUDA(cudaMallocHost(&ctl_h, sizeof(Ctl)));
        std::memset(ctl_h, 0, sizeof(Ctl));
        // Poisson form: single precision uses the radix-2 FP32 FFT on 2^k - 1 grids (at 255^2 as
        // fast as the tensor-core GEMMs, 3438 vs 3429 slices/s, with 2.5x less error in Ez: 5.2e-4
        // vs 1.3e-3 of FP64 in the blowout; at 2047^2 faster, 266 vs 249; at 1023^2 4 % slower,
        // 582 vs 608) and the tensor-core sine GEMMs (TF32x3) on other grids up to 1023^2;
        // HPQ_DST=tc / tc_bf16 (BF16x3 tensor-core GEMMs) / fft / gemm (SIMT sine GEMMs on every
        // grid, cross-checks) forces a form;
        // double precision uses the radix-2 FFT on 2^k - 1 grids, the SIMT sine GEMMs on other
        // grids up to 1024 (measured whole steps on a B200 against the Bluestein FFT: equal or
        // faster from 48 to 1000, e.g. 13.8 vs 20.0 ms at 128^2 x 40 slices, 20.9 vs 29.0 at 256^2,
        // 102.6 vs 110.2 at 600^2 x 16, the linear-wake predictor-corrector case at 64^2 3053 vs
        // 1912 slices/s; up to 7 % slower on explicit decks below 128) and the Bluestein FFT beyond
        const char* env = getenv("HPQ_DST");
        std::string dmode = env ? env : "";
        if (dmode.empty() && std::is_same<R, float>::value && FastDST<R>::radix2(nx, ny)) dmode = "fft";
        if (dmode.empty() && std::is_same<R, double>::value && !FastDST<R>::radix2(nx, ny) && std::max(nx, ny) <= 1024)
            dmode = "gemm";
        if (dmode == "gemm") { dst.set_mode(false); pc_dst.set_mode(false); if (sal_dst.nx) sal_dst.set_mode(false); }
        else if (dmode != "fft" && std::is_same<R, float>::value) {
            const bool bf16 = dmode == "tc_bf16";
            dst.set_tensor_mode(&ctl->tc_err, bf16);
            pc_dst.set_tensor_mode(&ctl->tc_err, bf16);
            if (sal_dst.nx) sal_dst.set_tensor_mode(&ctl->tc_err, bf16);
        }
        init_plasma_lattices();
        insitu_alloc();
        // beams: fixed_ppc generated here, fixed_weight drawn from the seeded generator unless
        // the caller provides particles with set_beam before the first step
        beam_set.assign(cfg.beams.size(), false);
        pending_beams.assign(cfg.beams.size(), HostBeam{});
        bm.resize(cfg.beams.size());
        for (size_t b = 0; b < cfg.beams.size(); ++b) {
            const BeamInjection inj = cfg.beams[b].injection;
            HostBeam hb = inj == BeamInjection::FixedPPC      ? make_fixed_ppc((int)b)
                          : inj == BeamInjection::FixedWeight ? make_fixed_weight((int)b)
                                                              : make_fixed_weight_pdf((int)b);
            upload_beam((int)b, hb);
        }
        // the set-up above zeroes and fills buffers with synchronous cudaMemset / cudaMemcpy calls
        // on the legacy default stream, which the library's non-blocking streams do not wait
        // for (a memset returns before it runs, a pageable upload before its DMA lands): finish
        // them before the first launch on those streams
        HPQ_CUDA(cudaDeviceSynchronize());
    }

    void init_plasma_lattices() {
        for (size_t s = 0; s < cfg.plasmas.size(); ++s) {
            const PlasmaSpecies& P = cfg.plasmas[s];
            std::vector<double> hx, hy;
            const int nppc = P.ppc[0] * P.ppc[1];
            int ilo = 0, ihi = nx - 1, jlo = 0, jhi = ny - 1;
            double xo = 0, yo = 0;
            if (P.prevent_centered_particle) {
                if (nx % 2 == 1 && P.ppc[0] % 2 == 1) { ilo = 1; xo = -0.5; }
                if (ny % 2 == 1 && P.ppc[1] % 2 == 1) { jlo = 1; yo = -0.5; }
            }
            if (P.radius < 1e299) {
                ilo = std::max(ilo, (int)std::round((-P.radius - cfg.prob_lo[0]) / g.dx[0] - 2));
                jlo = std::max(jlo, (int)std::round((-P.radius - cfg.prob_lo[1]) / g.dx[1] - 2));
                ihi = std::min(ihi, (int)std::round((P.radius - cfg.prob_lo[0]) / g.dx[0] + 2));
                jhi = std::min(jhi, (int)std::round((P.radius - cfg.prob_lo[1]) / g.dx[1] + 2));
            }
            // particles whose density is below min_density at t=0 are dropped; the density of a
            // kept particle is re-evaluated at c*t every step
            for (int ip = 0; ip < nppc; ++ip) {
                const int ixp = ip % P.ppc[0], iyp = ip / P.ppc[0];
                const double r0 = (0.5 + ixp) / P.ppc[0], r1 = (0.5 + iyp) / P.ppc[1];
                for (int j = jlo; j <= jhi; ++j)
                    for (int i = ilo; i <= ihi; ++i) {
                        const double x = cfg.prob_lo[0] + (i + r0 + xo) * g.dx[0];
                        const double y = cfg.prob_lo[1] + (j + r1 + yo) * g.dx[1];
                        const double rsq = x * x + y * y;
                        double v[3] = {x, y, 0.0};
                        if (x >= cfg.particle_hi[0] || x < cfg.particle_lo[0] || y >= cfg.particle_hi[1] ||
                            y < cfg.particle_lo[1] || rsq > P.radius * P.radius ||
                            rsq < P.hollow_core_radius * P.hollow_core_radius || P.density.eval(v) <= P.min_density)
                            continue;
                        hx.push_back(x); hy.push_back(y);
                    }
            }
            PlasmaDev<R> d{};
            d.n = (long long)hx.size();
            d.charge = P.charge; d.mass = P.mass; d.qsa_max = P.max_qsa_weighting_factor;
            d.n_subcycles = P.n_subcycles; d.neutralize = P.neutralize_background;
            const size_t nb = std::max<size_t>(1, hx.size());
            R** arrs[] = {&d.x, &d.y, &d.w, &d.ux, &d.uy, &d.psi, &d.xp, &d.yp, &d.uxh, &d.uyh, &d.psih};
            for (R** a : arrs) HPQ_CUDA(cudaMalloc(a, nb * sizeof(R)));
            HPQ_CUDA(cudaMalloc(&d.valid, nb));
            double *dx0, *dy0;
            HPQ_CUDA(cudaMalloc(&dx0, nb * sizeof(double)));
            HPQ_CUDA(cudaMalloc(&dy0, nb * sizeof(double)));
            if (!hx.empty()) {
                HPQ_CUDA(cudaMemcpy(dx0, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice));
                HPQ_CUDA(cudaMemcpy(dy0, hy.data(), hy.size() * sizeof(double), cudaMemcpyHostToDevice));
            }
            d.ru = d.rv = nullptr;
            if (std::is_same<R, float>::value) {
                // lattice points in cell units (exact in FP32); positions become displacements
                std::vector<float> hu(nb, 0.f), hv(nb, 0.f);
                for (size_t i = 0; i < hx.size(); ++i) {
                    hu[i] = (float)((hx[i] - g.xoff) * g.dxi[0]);
                    hv[i] = (float)((hy[i] - g.yoff) * g.dxi[1]);
                }
                float *du, *dv;
                HPQ_CUDA(cudaMalloc(&du, nb * sizeof(float)));
                HPQ_CUDA(cudaMalloc(&dv, nb * sizeof(float)));
                HPQ_CUDA(cudaMemcpy(du, hu.data(), nb * sizeof(float), cudaMemcpyHostToDevice));
                HPQ_CUDA(cudaMemcpy(dv, hv.data(), nb * sizeof(float), cudaMemcpyHostToDevice));
                d.ru = du; d.rv = dv;
            }
            pl.push_back(d);
            px0.push_back(dx0); py0.push_back(dy0);
            hx0.push_back(std::move(hx)); hy0.push_back(std::move(hy));
        }
    }

    // InitBeamFixedPPCSlice for all slices (BeamParticleContainerInit.cpp:199-345)
    HostBeam make_fixed_ppc(int b) {
        const BeamSpecies& B = cfg.beams[b];
        HostBeam hb;
        const int nppc = B.ppc[0] * B.ppc[1] * B.ppc[2];
        const double scale = cfg.normalized_units ? 1. / nppc : g.dx[0] * g.dx[1] * g.dx[2] / nppc;
        long long pid = 1;
        for (int k = 0; k < nz; ++k) {
            const double z0 = cfg.prob_lo[2] + k * g.dx[2];
            if (z0 + g.dx[2] < B.zmin || z0 > B.zmax) continue;
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int ip = 0; ip < nppc; ++ip) {
                        const int nyp = B.ppc[1], nzp = B.ppc[2];
                        const int ixp = ip / (nyp * nzp), iyp = (ip % (nyp * nzp)) % nyp, izp = (ip % (nyp * nzp)) / nyp;
                        const double x = cfg.prob_lo[0] + (i + (0.5 + ixp) / B.ppc[0]) * g.dx[0];
                        const double y = cfg.prob_lo[1] + (j + (0.5 + iyp) / B.ppc[1]) * g.dx[1];
                        const double z = cfg.prob_lo[2] + (k + (0.5 + izp) / B.ppc[2]) * g.dx[2];
                        if (z >= B.zmax || z < B.zmin ||
                            ((x - B.position_mean[0]) * (x - B.position_mean[0]) + (y - B.position_mean[1]) * (y - B.position_mean[1])) > B.radius * B.radius)
                            continue;
                        double dens;
                        if (B.profile == BeamProfile::Gaussian) {
                            const double a = (x - B.position_mean[0]) / B.position_std[0];
                            const double bb = (y - B.position_mean[1]) / B.position_std[1];
                            const double c = (z - B.position_mean[2]) / B.position_std[2];
                            dens = B.density * std::exp(-0.5 * a * a) * std::exp(-0.5 * bb * bb) * std::exp(-0.5 * c * c);
                        } else {
                            dens = B.density;
                        }
                        if (dens <= B.min_density) continue;
                        double xp = x, yp = y, uxp = B.u_mean[0] * cfg.pc.c, uyp = B.u_mean[1] * cfg.pc.c;
                        const bool ok = host_bc(xp, yp, uxp, uyp);
                        hb.push(xp, yp, z, ok ? std::fabs(dens * scale) : 0.0, uxp, uyp, B.u_mean[2] * cfg.pc.c, pid++);
                    }
        }
        return hb;
    }

    // InitBeamFixedWeight3D/Slice (BeamParticleContainerInit.cpp:349-476) with this build's own
    // counter-based generator (Philox4x32-10); AMReX's random stream is not reproduced.
    HostBeam make_fixed_weight(int b) {
        const BeamSpecies& B = cfg.beams[b];
        HostBeam hb;
        long long n = B.num_particles;
        if (n <= 0) return hb;
        const long long nbase = B.do_symmetrize ? n / 4 : n;
        const uint64_t seed = (uint64_t)(cfg.has_random_seed ? cfg.random_seed : 0) * 1000003ull + (uint64_t)b * 7919ull + 12345ull;
        Philox rng(seed);
        const bool can = B.profile == BeamProfile::Can;
        const double z_mean = can ? 0.5 * (B.zmin + B.zmax) : B.position_mean[2];
        const double weight = B.total_charge / (B.num_particles * B.charge);
        long long pid = 1;
        for (long long i = 0; i < nbase; ++i) {
            double nrm[8];
            rng.normals(2 * (uint64_t)i, nrm);
            rng.normals(2 * (uint64_t)i + 1, nrm + 4);
            const double zc = can ? rng.uniform(2 * (uint64_t)i + 1, 3) * (B.zmax - B.zmin) + B.zmin
                                  : z_mean + B.position_std[2] * nrm[0];
            double x = B.position_std[0] * nrm[1];
            double y = B.position_std[1] * nrm[2];
            double u[3] = {B.u_mean[0] + B.u_std[0] * nrm[3], B.u_mean[1] + B.u_std[1] * nrm[4],
                           B.u_mean[2] + B.u_std[2] * nrm[5]};
            u[2] += (zc - z_mean) * B.duz_per_uz0_dzeta * B.u_mean[2];
            bool valid = !(zc < B.zmin || zc > B.zmax || x * x + y * y > B.radius * B.radius);
            x -= B.z_foc * u[0] / u[2];
            y -= B.z_foc * u[1] / u[2];
            const double cx = B.position_mean[0], cy = B.position_mean[1];
            const int ncopy = B.do_symmetrize ? 4 : 1;
            for (int q = 0; q < ncopy; ++q) {
                const double sx = (q & 1) ? -1 : 1, sy = (q & 2) ? -1 : 1;
                double xp = cx + sx * x, yp = cy + sy * y, uxp = sx * u[0] * cfg.pc.c, uyp = sy * u[1] * cfg.pc.c;
                const bool ok = host_bc(xp, yp, uxp, uyp) && valid;
                hb.push(xp, yp, zc, ok ? std::fabs(weight) : 0.0, uxp, uyp, u[2] * cfg.pc.c, pid++);
            }
        }
        return hb;
    }

    // fixed_weight_pdf (InitBeamFixedWeightPDF3D and InitBeamFixedWeightPDFSlice,
    // BeamParticleContainerInit.cpp:479-678): particle counts per pdf sub-slice drawn from Poisson
    // distributions with the pdf's means (redrawn on the remainder until the total is exact), z
    // inside a sub-slice from the inverse of the trapezoidal pdf, Gaussian x, y, u with z-dependent
    // means and widths, constant weights. The random streams are this library's (std::mt19937_64
    // for the counts, Philox for the particles), not AMReX's.
    HostBeam make_fixed_weight_pdf(int b) {
        const BeamSpecies& B = cfg.beams[b];
        HostBeam hb;
        if (B.num_particles <= 0) return hb;
        const long long nadd = B.do_symmetrize ? B.num_particles / 4 : B.num_particles;
        const int ref = B.pdf_ref_ratio;
        const int nsl = nz * ref;
        const double z0 = cfg.prob_lo[2], zs = g.dx[2] / ref;
        const double pi = 3.14159265358979323846;
        auto fz = [](const Expr& e, double z) { return e.eval(&z); };
        std::vector<double> lw(nsl);
        double integral = 0, maxd = 0;
        for (int s = nsl - 1; s >= 0; --s) {
            const double zmin = z0 + s * zs, zmax = z0 + (s + 1) * zs, zmid = 0.5 * (zmin + zmax);
            const double a = fz(B.pdf, zmin), c = fz(B.pdf, zmax);
            if (!(a >= 0 && c >= 0)) throw InputError("PDF must be >= 0 everywhere");
            lw[s] = 0.5 * (a + c);
            if (B.peak_density_specified)
                maxd = std::max(maxd, lw[s] / (zs * fz(B.pdf_pos[2], zmid) * fz(B.pdf_pos[3], zmid) * 2.0 * pi));
            integral += lw[s];
        }
        if (!(integral > 0)) throw InputError("the pdf of beam " + B.name + " is zero over the box");
        double total_weight = B.peak_density_specified ? B.density * integral / maxd : B.total_charge / std::fabs(B.charge);
        if (cfg.normalized_units) total_weight *= g.dxi[0] * g.dxi[1] * g.dxi[2];
        const uint64_t seed = (uint64_t)(cfg.has_random_seed ? cfg.random_seed : 0) * 1000003ull + (uint64_t)b * 7919ull + 54321ull;
        std::mt19937_64 gen(seed);
        std::vector<long long> cnt(nsl, 0);
        long long added = 0;
        while (added != nadd) {
            const long long now = nadd - added;
            for (int s = nsl - 1; s >= 0; --s) {
                const double mean = (double)now * lw[s] / integral;
                if (mean > 0) {
                    const long long n = std::poisson_distribution<long long>(mean)(gen);
                    cnt[s] += n;
                    added += n;
                } else if (mean < 0) {
                    const long long n = std::min(std::poisson_distribution<long long>(-mean)(gen), cnt[s]);
                    cnt[s] -= n;
                    added -= n;
                }
            }
        }
        const double weight = total_weight / B.num_particles;
        const Philox rng(seed ^ 0x9e3779b97f4a7c15ull);
        constexpr int kTries = 1000;  // transverse redraws inside the radius (the reference loops until one fits)
        long long idx = 0, pid = 1;
        for (int s = nsl - 1; s >= 0; --s) {
            if (cnt[s] == 0) continue;
            const double zmin = z0 + s * zs, zmax = z0 + (s + 1) * zs;
            const double lo = fz(B.pdf, zmin), hi = fz(B.pdf, zmax);
            // the exact inverse is ill-conditioned for lo close to hi: Taylor form within 10 %
            const bool taylor = std::min(lo, hi) * 1.1 > std::max(lo, hi);
            const double inv = taylor ? 1.0 / (hi + lo) : 1.0 / (hi - lo);
            for (long long q = 0; q < cnt[s]; ++q, ++idx) {
                const uint64_t ctr = (uint64_t)idx * 1024;
                const double w = rng.uniform(ctr, 0);
                const double z = zmin + (taylor ? zs * (w - w * (w - 1.0) * (hi - lo) * inv)
                                                : zs * ((std::sqrt(lo * lo + w * (hi * hi - lo * lo)) - lo) * inv));
                const double xm = fz(B.pdf_pos[0], z), ym = fz(B.pdf_pos[1], z);
                const double xs = fz(B.pdf_pos[2], z), ys = fz(B.pdf_pos[3], z);
                double x = 0, y = 0, nrm[4];
                bool valid = false;
                for (int t = 0; t < kTries; ++t) {
                    rng.normals(ctr + t, nrm);
                    x = xs * nrm[0];
                    y = ys * nrm[1];
                    valid = x * x + y * y <= B.radius * B.radius;
                    if (valid || B.peak_density_specified) break;
                }
                rng.normals(ctr + 1023, nrm);
                double u[3];
                for (int d = 0; d < 3; ++d) u[d] = fz(B.pdf_u[d], z) + fz(B.pdf_u[d + 3], z) * nrm[d];
                x -= B.z_foc * u[0] / u[2];
                y -= B.z_foc * u[1] / u[2];
                const int ncopy = B.do_symmetrize ? 4 : 1;
                for (int k = 0; k < ncopy; ++k) {
                    const double sx = (k & 1) ? -1 : 1, sy = (k & 2) ? -1 : 1;
                    double xp = xm + sx * x, yp = ym + sy * y, uxp = sx * u[0] * cfg.pc.c, uyp = sy * u[1] * cfg.pc.c;
                    const bool ok = host_bc(xp, yp, uxp, uyp) && valid;
                    hb.push(xp, yp, z, ok ? std::fabs(weight) : 0.0, uxp, uyp, u[2] * cfg.pc.c, pid++);
                }
            }
        }
        return hb;
    }

    bool host_bc(double& x, double& y, double& ux, double& uy) const {
        const double plo0 = cfg.particle_lo[0], plo1 = cfg.particle_lo[1], phi0 = cfg.particle_hi[0], phi1 = cfg.particle_hi[1];
        if (x < plo0 || y < plo1 || x > phi0 || y > phi1) {
            const double lx = phi0 - plo0, ly = phi1 - plo1;
            if (cfg.particle_bc == ParticleBC::Reflecting) {
                x = std::fmod(x - plo0, 2 * lx); if (x < 0) x += 2 * lx; x += plo0;
                if (x > phi0) { x = 2 * phi0 - x; ux = -ux; }
                y = std::fmod(y - plo1, 2 * ly); if (y < 0) y += 2 * ly; y += plo1;
                if (y > phi1) { y = 2 * phi1 - y; uy = -uy; }
                return true;
            } else if (cfg.particle_bc == ParticleBC::Periodic) {
                x = std::fmod(x - plo0, lx); if (x < 0) x += lx; x += plo0;
                y = std::fmod(y - plo1, ly); if (y < 0) y += ly; y += plo1;
                return true;
            }
            return false;
        }
        return true;
    }

    static void alloc_buf(BeamBuf& b, long long cap) {
        const size_t n = (size_t)std::max<long long>(cap, 1);
        double** d[] = {&b.x, &b.y, &b.z, &b.w, &b.ux, &b.uy, &b.uz};
        for (double** p : d) HPQ_CUDA(cudaMalloc(p, n * sizeof(double)));
        HPQ_CUDA(cudaMalloc(&b.id, n * sizeof(long long)));
        HPQ_CUDA(cudaMalloc(&b.nsub, n * sizeof(int)));
        HPQ_CUDA(cudaMalloc(&b.valid, n));
    }
    static void free_buf(BeamBuf& b) {
        for (void* p : {(void*)b.x, (void*)b.y, (void*)b.z, (void*)b.w, (void*)b.ux, (void*)b.uy, (void*)b.uz,
                        (void*)b.id, (void*)b.nsub, (void*)b.valid})
            if (p) cudaFree(p);
        std::memset(&b, 0, sizeof(b));
    }
    static void free_beam(BeamDev& d) {
        if (d.ext) cudaFree(const_cast<Expr*>(d.ext));
        d.ext = nullptr;
        for (int q = 0; q < 2; ++q) {
            free_buf(d.buf[q]); free_buf(d.carry[q]);
            if (d.start[q]) cudaFree(d.start[q]);
            if (d.count[q]) cudaFree(d.count[q]);
            d.start[q] = d.count[q] = nullptr;
        }
    }

    // BoxSort (BoxSort.cpp:14-78): slice = int((z - lo) / dz); particles outside [0, nz) are
    // dropped; stable within a slice. Slices are stored top-down like the slice march. The host
    // computes only the order (a counting sort of indices); the particle data go to the device
    // as they are (from the caller's buffers, pinned or not) and are gathered there.
    // scratch of the device slice binning: keys, per-chunk histograms, the in-box count
    int* bin_key = nullptr;
    int* bin_hist = nullptr;
    long long* bin_total = nullptr;
    long long bin_key_cap = 0, bin_hist_cap = 0;

    void upload_beam(int b, const double* x, const double* y, const double* z, const double* w, const double* ux,
                     const double* uy, const double* uz, const long long* id, long long nin) {
        BeamDev& d = bm[b];
        const BeamSpecies& B = cfg.beams[b];
        d.charge = B.charge; d.mass = B.mass; d.n_subcycles = B.n_subcycles; d.do_z_push = B.do_z_push;
        if (nin > INT32_MAX) throw InputError("beam too large");
        // device buffers are kept when the new beam fits (captured slice graphs stay valid)
        if (d.buf[0].x == nullptr || nin > d.cap) {
            free_beam(d);
            invalidate_graph();
            if (B.use_external) {
                Expr* e = nullptr;
                HPQ_CUDA(cudaMalloc(&e, 6 * sizeof(Expr)));
                HPQ_CUDA(cudaMemcpyAsync(e, B.external, 6 * sizeof(Expr), cudaMemcpyHostToDevice, st));
                d.ext = e;
            }
            d.cap = std::max<long long>(nin, 1);
            for (int q = 0; q < 2; ++q) {
                alloc_buf(d.buf[q], d.cap);
                alloc_buf(d.carry[q], d.cap);
                HPQ_CUDA(cudaMalloc(&d.start[q], nz * sizeof(int)));
                HPQ_CUDA(cudaMalloc(&d.count[q], nz * sizeof(int)));
            }
        }
        const int nb = (int)std::max<long long>((nin + kBinChunk - 1) / kBinChunk, 1);
        if (bin_key_cap < nin || !bin_key) {
            if (bin_key) cudaFree(bin_key);
            bin_key_cap = std::max<long long>(nin, 1);
            HPQ_CUDA(cudaMalloc(&bin_key, bin_key_cap * sizeof(int)));
        }
        if (bin_hist_cap < (long long)nz * nb || !bin_hist) {
            if (bin_hist) cudaFree(bin_hist);
            bin_hist_cap = (long long)nz * nb;
            HPQ_CUDA(cudaMalloc(&bin_hist, bin_hist_cap * sizeof(int)));
        }
        if (!bin_total) HPQ_CUDA(cudaMalloc(&bin_total, sizeof(long long)));
        for (int q = 0; q < 2; ++q) {
            HPQ_CUDA(cudaMemsetAsync(d.start[q], 0, nz * sizeof(int), st));
            HPQ_CUDA(cudaMemsetAsync(d.count[q], 0, nz * sizeof(int), st));
        }
        // the carry buffers are free between steps: carry[0] stages the input arrays, the sub-cycle
        // array of carry[1] the order
        const BeamBuf& sg = d.carry[0];
        if (nin > 0) {
            const double* src[7] = {x, y, z, w, ux, uy, uz};
            double* dstp[7] = {sg.x, sg.y, sg.z, sg.w, sg.ux, sg.uy, sg.uz};
            for (int k = 0; k < 7; ++k)
                HPQ_CUDA(cudaMemcpyAsync(dstp[k], src[k], nin * sizeof(double), cudaMemcpyHostToDevice, st));
            if (id) HPQ_CUDA(cudaMemcpyAsync(sg.id, id, nin * sizeof(long long), cudaMemcpyHostToDevice, st));
            // slice binning on the device (stable counting sort, top slice first)
            const size_t ksm = (size_t)nz * sizeof(int);
            if (ksm > 48 * 1024) {
                HPQ_CUDA(cudaFuncSetAttribute(k_bin_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ksm));
                HPQ_CUDA(cudaFuncSetAttribute(k_bin_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ksm));
            }
            hpq_launch(k_bin_hist, dim3(nb), dim3(256), ksm, st, (const double*)sg.z, nin, cfg.prob_lo[2], g.dxi[2], nz,
                       bin_key, bin_hist, nb);
            HPQ_LAUNCH_CHECK();
            hpq_launch(k_bin_scan_chunks, dim3(nz), dim3(256), 0, st, bin_hist, nb, d.count[parity]);
            HPQ_LAUNCH_CHECK();
            hpq_launch(k_bin_scan_slices, dim3(1), dim3(1024), 0, st, (const int*)d.count[parity], nz, d.start[parity], bin_total);
            HPQ_LAUNCH_CHECK();
            hpq_launch(k_bin_scatter, dim3(nb), dim3(32), ksm, st, (const int*)bin_key, nin, (const int*)bin_hist, nb,
                       (const int*)d.start[parity], nz, d.carry[1].nsub);
            HPQ_LAUNCH_CHECK();
            hpq_launch(k_beam_gather, dim3(blocks_for(nin, 256)), dim3(256), 0, st, d.buf[parity], (const BeamBuf)sg,
                       (const int*)d.carry[1].nsub, (const long long*)bin_total, id ? 1 : 0);
            HPQ_LAUNCH_CHECK();
        }
        HPQ_CUDA(cudaStreamSynchronize(st));  // the caller's buffers are released
        st_host.beam_particles = 0;
        ++beam_gen;
    }
    void upload_beam(int b, const HostBeam& hb) {
        upload_beam(b, hb.x.data(), hb.y.data(), hb.z.data(), hb.w.data(), hb.ux.data(), hb.uy.data(), hb.uz.data(),
                    hb.id.data(), (long long)hb.size());
    }

    void set_beam(int b, const double* x, const double* y, const double* z, const double* w, const double* ux,
                  const double* uy, const double* uz, const long long* id, long long n) override {
        if (b < 0 || b >= (int)cfg.beams.size()) throw InputError("beam index out of range");
        HPQ_CUDA(cudaStreamSynchronize(st));
        upload_beam(b, x, y, z, w, ux, uy, uz, id, n);
    }

    // calls f(std::integral_constant<int, ORD>{}) for the deck's transverse shape order
    // (hipace.depos_order_xy, 0..3): the deposits, gathers and pushes are compiled per order
    template <class F>
    void with_order(F&& f) const {
        switch (cfg.depos_order_xy) {
            case 0: f(std::integral_constant<int, 0>{}); break;
            case 1: f(std::integral_constant<int, 1>{}); break;
            case 3: f(std::integral_constant<int, 3>{}); break;
            default: f(std::integral_constant<int, 2>{}); break;
        }
    }

    // ---- time-step pipeline hand-off
    // out_par: parity of the store the current (or last) step writes for the next step
    int out_par = 1;
    std::vector<long long> put_cursor;
    long long beam_slice_count(int b, int islice) override {
        HPQ_CUDA(cudaStreamSynchronize(st));
        int n = 0;
        HPQ_CUDA(cudaMemcpy(&n, bm.at(b).count[out_par] + islice, sizeof(int), cudaMemcpyDeviceToHost));
        return n;
    }
    void get_beam_slice(int b, int islice, double* x, double* y, double* z, double* w, double* ux, double* uy,
                        double* uz, long long* id) override {
        HPQ_CUDA(cudaStreamSynchronize(st));
        const BeamDev& d = bm.at(b);
        int n = 0, s0 = 0;
        HPQ_CUDA(cudaMemcpy(&n, d.count[out_par] + islice, sizeof(int), cudaMemcpyDeviceToHost));
        HPQ_CUDA(cudaMemcpy(&s0, d.start[out_par] + islice, sizeof(int), cudaMemcpyDeviceToHost));
        if (n == 0) return;
        const BeamBuf& src = d.buf[out_par];
        double* outs[7] = {x, y, z, w, ux, uy, uz};
        const double* ins[7] = {src.x, src.y, src.z, src.w, src.ux, src.uy, src.uz};
        for (int a = 0; a < 7; ++a)
            HPQ_CUDA(cudaMemcpy(outs[a], ins[a] + s0, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
        HPQ_CUDA(cudaMemcpy(id, src.id + s0, (size_t)n * sizeof(long long), cudaMemcpyDeviceToHost));
    }
    // Appends the particles of slice islice to the store the current step reads. Slices come from
    // the head down; the first one of a step (nz - 1) empties the store. Each must arrive before
    // the slice graph that reads it: slice islice is read by the solves of slices islice + 1 (its
    // jx/jy beam deposit) and islice.
    void put_beam_slice(int b, int islice, const double* x, const double* y, const double* z, const double* w,
                        const double* ux, const double* uy, const double* uz, const long long* id,
                        long long n) override {
        BeamDev& d = bm.at(b);
        if (put_cursor.size() < bm.size()) put_cursor.resize(bm.size(), 0);
        if (islice == nz - 1) {
            put_cursor[b] = 0;
            HPQ_CUDA(cudaMemsetAsync(d.count[parity], 0, nz * sizeof(int), st));
            HPQ_CUDA(cudaMemsetAsync(d.start[parity], 0, nz * sizeof(int), st));
        }
        const long long c0 = put_cursor[b];
        if (c0 + n > d.cap)
            throw InputError("hpq_put_beam_slice: the received particles exceed the beam's store (" +
                             std::to_string(d.cap) + ")");
        const BeamBuf& dst = d.buf[parity];
        if (n > 0) {
            const double* ins[7] = {x, y, z, w, ux, uy, uz};
            double* outs[7] = {dst.x, dst.y, dst.z, dst.w, dst.ux, dst.uy, dst.uz};
            for (int a = 0; a < 7; ++a)
                HPQ_CUDA(cudaMemcpyAsync(outs[a] + c0, ins[a], (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
            HPQ_CUDA(cudaMemcpyAsync(dst.id + c0, id, (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, st));
            hpq_launch(k_beam_slice_flags, dim3(blocks_for(n, 256)), dim3(256), 0, st, dst, c0, n);
            HPQ_LAUNCH_CHECK();
        }
        const int s0 = (int)c0, cnt = (int)n;
        HPQ_CUDA(cudaMemcpyAsync(d.start[parity] + islice, &s0, sizeof(int), cudaMemcpyHostToDevice, st));
        HPQ_CUDA(cudaMemcpyAsync(d.count[parity] + islice, &cnt, sizeof(int), cudaMemcpyHostToDevice, st));
        put_cursor[b] = c0 + n;
        HPQ_CUDA(cudaStreamSynchronize(st));  // the caller's buffers (and s0, cnt) are released
    }
    void set_time(double t) override { physical_time = t; }

    long long beam_count(int b) override {
        HPQ_CUDA(cudaStreamSynchronize(st));
        std::vector<int> cnt(nz);
        HPQ_CUDA(cudaMemcpy(cnt.data(), bm[b].count[parity], nz * sizeof(int), cudaMemcpyDeviceToHost));
        long long n = 0;
        for (int c : cnt) n += c;
        return n;
    }
    // particles of the current store in slice-descending order; invalid particles (absorbed at a
    // boundary, removed by SALAME) are reported with weight 0, which hpq_set_beam reads back as
    // invalid
    // validity flags of the last read-back (pinned, so that their copy is a plain DMA)
    uint8_t* valid_h = nullptr;
    long long valid_cap = 0, valid_n = 0;
    void get_beam(int b, double* x, double* y, double* z, double* w, double* ux, double* uy, double* uz,
                  long long* id) override {
        get_beam_raw(b, x, y, z, w, ux, uy, uz, id);
        // eight flags at a time: runs of valid particles (flag 1) are skipped with one compare
        long long k = 0;
        for (; k + 8 <= valid_n; k += 8) {
            uint64_t q;
            std::memcpy(&q, valid_h + k, 8);
            if (q == 0x0101010101010101ull) continue;
            for (int t = 0; t < 8; ++t)
                if (!valid_h[k + t]) w[k + t] = 0.0;
        }
        for (; k < valid_n; ++k)
            if (!valid_h[k]) w[k] = 0.0;
    }
    void get_beam_raw(int b, double* x, double* y, double* z, double* w, double* ux, double* uy, double* uz,
                      long long* id) {
        HPQ_CUDA(cudaStreamSynchronize(st));
        BeamDev& d = bm[b];
        std::vector<int> cnt(nz), start(nz);
        HPQ_CUDA(cudaMemcpy(cnt.data(), d.count[parity], nz * sizeof(int), cudaMemcpyDeviceToHost));
        HPQ_CUDA(cudaMemcpy(start.data(), d.start[parity], nz * sizeof(int), cudaMemcpyDeviceToHost));
        const BeamBuf& s = d.buf[parity];
        double* outs[7] = {x, y, z, w, ux, uy, uz};
        double* ins[7] = {s.x, s.y, s.z, s.w, s.ux, s.uy, s.uz};
        // the slices of a store are consecutive (top-down, no gaps): one copy per array
        bool contiguous = true;
        long long total = 0;
        for (int sl = nz - 1; sl >= 0; --sl) {
            if (cnt[sl] && start[sl] != start[nz - 1] + total) contiguous = false;
            total += cnt[sl];
        }
        if (total > valid_cap) {
            if (valid_h) HPQ_CUDA(cudaFreeHost(valid_h));
            valid_h = nullptr;
            valid_cap = 0;
            HPQ_CUDA(cudaMallocHost(&valid_h, (size_t)total));
            valid_cap = total;
        }
        valid_n = total;
        if (contiguous) {
            if (total > 0) {
                const size_t o = start[nz - 1];
                for (int a = 0; a < 7; ++a)
                    HPQ_CUDA(cudaMemcpyAsync(outs[a], ins[a] + o, total * sizeof(double), cudaMemcpyDeviceToHost, st));
                if (id) HPQ_CUDA(cudaMemcpyAsync(id, s.id + o, total * sizeof(long long), cudaMemcpyDeviceToHost, st));
                HPQ_CUDA(cudaMemcpyAsync(valid_h, s.valid + o, total, cudaMemcpyDeviceToHost, st));
                HPQ_CUDA(cudaStreamSynchronize(st));
            }
            return;
        }
        long long k = 0;
        for (int sl = nz - 1; sl >= 0; --sl) {
            const size_t n = cnt[sl], o = start[sl];
            if (!n) continue;
            for (int a = 0; a < 7; ++a) HPQ_CUDA(cudaMemcpy(outs[a] + k, ins[a] + o, n * sizeof(double), cudaMemcpyDeviceToHost));
            if (id) HPQ_CUDA(cudaMemcpy(id + k, s.id + o, n * sizeof(long long), cudaMemcpyDeviceToHost));
            HPQ_CUDA(cudaMemcpy(valid_h + k, s.valid + o, n, cudaMemcpyDeviceToHost));
            k += n;
        }
    }

    // ----------------------------------------------------------------------------- step
    // Hipace::Evolve per-step body (Hipace.cpp:401-480): reset slices, re-create the plasma,
    // deposit the ion background
    void begin_step(int step) override {
        cur_step = step;
        out_par = 1 - parity;
        HPQ_CUDA(cudaMemsetAsync(S.base, 0, S.cstride * ncomp_alloc * sizeof(R), st));
        // SALAME runs in step 0 only (MultiBeam::isSalameNow, MultiBeam.cpp:128-139); the host
        // needs each SALAME beam's particle count per slice to decide slice by slice
        sal_step = ncomp_alloc > C_NCOMP && step == 0;
        sal_count.assign(bm.size(), {});
        if (sal_step)
            for (size_t b = 0; b < bm.size(); ++b) {
                if (!cfg.beams[b].do_salame) continue;
                sal_count[b].resize(nz);
                HPQ_CUDA(cudaMemcpyAsync(sal_count[b].data(), bm[b].count[parity], nz * sizeof(int), cudaMemcpyDeviceToHost, st));
            }
        if (sal_step) HPQ_CUDA(cudaStreamSynchronize(st));
        const double c_t = cfg.pc.c * physical_time;
        for (size_t s = 0; s < pl.size(); ++s) {
            const PlasmaSpecies& P = cfg.plasmas[s];
            const int nppc = P.ppc[0] * P.ppc[1];
            const double scale = adj_plasma_scale *
                                 (nppc <= 0 ? 0. : (cfg.normalized_units ? 1. / nppc : g.dx[0] * g.dx[1] * g.dx[2] / nppc));
            if (pl[s].n == 0) continue;
            PlasmaMomenta m{};
            for (int d = 0; d < 3; ++d) { m.mean[d] = P.u_mean[d]; m.stdv[d] = P.u_std[d]; }
            m.thermal = P.thermal ? 1 : 0;
            m.seed = plasma_thermal_seed((uint64_t)(cfg.has_random_seed ? cfg.random_seed : 0), (int)s);
            m.step = step;
            hpq_launch(k_plasma_reset<R>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], px0[s], py0[s], P.density, c_t, scale,
                       m, cfg.pc.c, g.xoff, g.dxi[0], g.yoff, g.dxi[1]);
            HPQ_LAUNCH_CHECK();
            if (s < reordered.size()) reordered[s] = false;
        }
        for (size_t s = 0; s < pl.size(); ++s) {
            if (!pl[s].neutralize || pl[s].n == 0) continue;
            DepOut<R> o{nullptr, nullptr, nullptr, nullptr, nullptr, S.c(C_IONS).p, S.pitch};
            with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(det.w[0] ? k_plasma_deposit<R, true, ORD> : k_plasma_deposit<R, false, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], o, g, -pl[s].charge, (const int*)nullptr, det); });
            HPQ_LAUNCH_CHECK();
            det_flush({C_IONS});
        }
        // control block for the slice march
        std::memset(ctl_h, 0, sizeof(Ctl));
        ctl_h->islice = nz - 1;
        ctl_h->step_parity = parity;
        const StepTime T = step_time(physical_time, cfg.dt, cfg.max_time);
        ctl_h->beam_dt = T.dt;
        ctl_h->phys_time = physical_time;
        next_time = T.next;
        for (size_t b = 0; b < cfg.beams.size() && b < (size_t)kMaxBeams; ++b) {
            const bool on = insitu_beam_d[b] && do_diagnostics(cfg.beams[b].insitu_period, step, cfg.max_step,
                                                               physical_time, cfg.max_time);
            ctl_h->insitu_beam[b] = on;
            if (on) insitu_beam_has[b] = 1;
        }
        {
            const bool on = insitu_fields_d && do_diagnostics(cfg.fields_insitu_period, step, cfg.max_step,
                                                              physical_time, cfg.max_time);
            ctl_h->insitu_fields = on;
            if (on) insitu_fields_has = true;
        }
        HPQ_CUDA(cudaMemcpyAsync(ctl, ctl_h, sizeof(Ctl), cudaMemcpyHostToDevice, st));
        cur_islice = nz - 1;
    }

    void end_step() override {
        if (!bm.empty()) {
            // beam work of the last slice (slice 0: the counter stands at -1)
            const long long l0 = g_launches;
            beam_work(1);
            launches_total += g_launches - l0;
        }
        physical_time = next_time;
        parity = 1 - parity;
        ++beam_gen;
        HPQ_CUDA(cudaMemcpyAsync(ctl_h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        HPQ_CUDA(cudaStreamSynchronize(st));
        prof_collect();
        st_host.mg_vcycles += ctl_h->mg_total_iters;
        if (use_graphs && !profiling) launches_total += ctl_h->mg_total_iters * launches_body;
        st_host.launches = launches_total;
        if (ctl_h->mg_status && !st_host.mg_status) st_host.mg_status = ctl_h->mg_status;
        st_host.slices += nz;
        for (auto& p : pl) st_host.plasma_pushes += p.n * nz;
        if (cfg.explicit_solver) mg.print_trace();
        if (ctl_h->tc_err) throw CudaError("tensor-core DST: a pipeline wait timed out (code " + std::to_string(ctl_h->tc_err) + ")");
        if (ctl_h->mgp_bar_err) throw CudaError("hpmg: grid barrier of the persistent multigrid solve timed out");
        if (st_host.mg_status == 1) throw CudaError("hpmg: failed to converge within the iteration limit");
        if (st_host.mg_status == 2) throw CudaError("hpmg: diverged");
    }

    // warp-merged order-2 plasma deposit (plasma_deposit_merged); HPQ_DEPOSIT_MERGE=1/0 in the
    // environment switches it on/off
    int deposit_merge = -1;
    void deposit_plasma(int sp, R* jx, R* jy, R* jz, R* rho, R* chi, R* rhomjz) {
        if (pl[sp].n == 0) return;
        if (deposit_merge < 0) {
            const char* e = getenv("HPQ_DEPOSIT_MERGE");
            deposit_merge = (e && e[0] == '1') ? 1 : 0;
        }
        DepOut<R> o{jx, jy, jz, rho, chi, rhomjz, S.pitch, deposit_merge};
        Scope sc(this, "plasma_deposit");
        with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(det.w[0] ? k_plasma_deposit<R, true, ORD> : k_plasma_deposit<R, false, ORD>, dim3(blocks_for(pl[sp].n, 256)), dim3(256), 0, st, pl[sp], o, g, pl[sp].charge, (const int*)nullptr, det); });
        HPQ_LAUNCH_CHECK();
        det_flush_ptrs({jx, jy, jz, rho, chi, rhomjz});
    }
    void deposit_beam(int b, int which, R* jx, R* jy, R* jz, R* rmj) {
        Scope sc(this, "beam_deposit");
        with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_beam_deposit<R, ORD>, dim3(148 * 2), dim3(256), 0, st, bm[b], (const Ctl*)ctl, which, jx, jy, jz, rmj, S.pitch, g, 0, det); });
        HPQ_LAUNCH_CHECK();
        det_flush_ptrs({jx, jy, jz, rmj});
    }
    // ---- in-situ reductions (raw per-slice sums on the device; normalised on the host)
    std::vector<double*> insitu_beam_d;  // per beam: nz x 23
    double* insitu_fields_d = nullptr;   // nz x 10
    std::vector<char> insitu_beam_has;   // the last diagnostic step filled the arrays
    bool insitu_fields_has = false;
    void insitu_alloc() {
        insitu_beam_d.assign(cfg.beams.size(), nullptr);
        insitu_beam_has.assign(cfg.beams.size(), 0);
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (cfg.beams[b].insitu_period > 0) {
                HPQ_CUDA(cudaMalloc(&insitu_beam_d[b], (size_t)nz * 23 * sizeof(double)));
                HPQ_CUDA(cudaMemset(insitu_beam_d[b], 0, (size_t)nz * 23 * sizeof(double)));
            }
        if (cfg.fields_insitu_period > 0) {
            HPQ_CUDA(cudaMalloc(&insitu_fields_d, (size_t)nz * 10 * sizeof(double)));
            HPQ_CUDA(cudaMemset(insitu_fields_d, 0, (size_t)nz * 10 * sizeof(double)));
        }
    }
    long long insitu_size(const std::string& what) override {
        if (what == "fields") return cfg.fields_insitu_period > 0 ? 11LL * nz : -1;
        for (size_t b = 0; b < cfg.beams.size(); ++b)
            if (cfg.beams[b].name == what) return cfg.beams[b].insitu_period > 0 ? 23LL * nz + 23 : -1;
        return -1;
    }
    // layout of the reference's reduced diagnostics: value index outer, slice inner; beams: 22 x nz
    // values (entry 0 the sum of weights, the others divided by it), nz counts, 22 + 1 sums over
    // slices; fields: 10 x nz values (times dx dy dz), 10 sums
    bool get_insitu(const std::string& what, double* out) override {
        HPQ_CUDA(cudaStreamSynchronize(st));
        if (what == "fields") {
            if (!insitu_fields_d || !insitu_fields_has) return false;
            std::vector<double> r((size_t)nz * 10);
            HPQ_CUDA(cudaMemcpy(r.data(), insitu_fields_d, r.size() * sizeof(double), cudaMemcpyDeviceToHost));
            const double dv = g.dx[0] * g.dx[1] * g.dx[2];
            std::vector<double> sum(10, 0.0);
            for (int isl = nz - 1; isl >= 0; --isl)
                for (int k = 0; k < 10; ++k) sum[k] += r[(size_t)isl * 10 + k] * dv;
            for (int k = 0; k < 10; ++k)
                for (int isl = 0; isl < nz; ++isl) out[(size_t)k * nz + isl] = r[(size_t)isl * 10 + k] * dv;
            for (int k = 0; k < 10; ++k) out[(size_t)10 * nz + k] = sum[k];
            return true;
        }
        for (size_t b = 0; b < cfg.beams.size(); ++b) {
            if (cfg.beams[b].name != what) continue;
            if (!insitu_beam_d[b] || !insitu_beam_has[b]) return false;
            std::vector<double> r((size_t)nz * 23);
            HPQ_CUDA(cudaMemcpy(r.data(), insitu_beam_d[b], r.size() * sizeof(double), cudaMemcpyDeviceToHost));
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
            return true;
        }
        throw InputError("unknown in-situ diagnostic '" + what + "'");
    }

    // ---- deterministic deposition (fixed-point shadows, see addc)
    DetAcc det{};
    long long* det_mem = nullptr;
    void set_deterministic(bool on) override {
        if (on == (det.w[0] != nullptr)) return;
        invalidate_graph();
        if (on) {
            const size_t n = (size_t)ncomp_alloc * S.cstride;
            HPQ_CUDA(cudaMalloc(&det_mem, 3 * n * sizeof(long long)));
            HPQ_CUDA(cudaMemsetAsync(det_mem, 0, 3 * n * sizeof(long long), st));
            for (int k = 0; k < 3; ++k) det.w[k] = det_mem + k * n;
            det.base = S.base;
        } else {
            HPQ_CUDA(cudaDeviceSynchronize());
            cudaFree(det_mem);
            det_mem = nullptr;
            det = DetAcc{};
        }
    }
    void det_flush(std::initializer_list<int> comps) {
        if (!det.w[0]) return;
        CompList L{};
        for (int c : comps) L.c[L.n++] = c;
        hpq_launch(k_det_flush<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 4)), dim3(256), 0, st, S, det, L);
        HPQ_LAUNCH_CHECK();
    }
    void det_flush_ptrs(std::initializer_list<R*> planes) {
        if (!det.w[0]) return;
        CompList L{};
        for (R* p : planes)
            if (p) L.c[L.n++] = (int)((p - S.base) / (ptrdiff_t)S.cstride);
        if (L.n == 0) return;
        hpq_launch(k_det_flush<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 4)), dim3(256), 0, st, S, det, L);
        HPQ_LAUNCH_CHECK();
    }

    void zero(std::initializer_list<int> comps) {
        CompList L{};
        for (int c : comps) L.c[L.n++] = c;
        hpq_launch(k_zero_comps<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 8)), dim3(256), 0, st, S, L);
        HPQ_LAUNCH_CHECK();
    }
    void copies(std::initializer_list<std::pair<int, int>> pairs) {
        CopyList L{};
        for (auto& p : pairs) { L.dst[L.n] = p.first; L.src[L.n] = p.second; L.n++; }
        hpq_launch(k_copy_comps<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 8)), dim3(256), 0, st, S, L);
        HPQ_LAUNCH_CHECK();
    }
    void field_solve_psi_ez_bz() {
        const long long ntot = (long long)(nx + 2 * kGuardAlloc) * S.rows;
        Scope sc(this, "poisson_psi_ez_bz");
        hpq_launch(k_rhs3<R>, dim3(blocks_for(ntot, 256)), dim3(256), 0, st, S, g, dst.stage, dst.sk, dst.sj, cfg.any_neutralize_background(),
                                                         cfg.deposit_rho && cfg.any_neutralize_background(),
                                                         cfg.explicit_solver && cfg.do_beam_jz_minus_rho);
        HPQ_LAUNCH_CHECK();
        const int comps[3] = {C_PSI, C_EZ, C_BZ};
        dst.solve(st, 3, S.base, S.cstride, S.pitch, comps);
        if (cfg.explicit_solver) hpq_launch(k_grad_psi_sxsy<R>, dim3(blocks_for((long long)(nx + 2) * (ny + 2), 256)), dim3(256), 0, st, S, g);
        else hpq_launch(k_grad_psi<R>, dim3(blocks_for((long long)(nx + 2) * (ny + 2), 256)), dim3(256), 0, st, S, g);
        HPQ_LAUNCH_CHECK();
    }

    // ExplicitDeposition (ExplicitDeposition.cpp:20-265): Sx, Sy += the plasma contribution;
    // the four fields it gathers are first packed cell by cell (Quad)
    Quad<R>* quad = nullptr;
    void explicit_deposit() {
        bool packed = false;
        for (size_t s = 0; s < pl.size(); ++s) {
            if (pl[s].n == 0) continue;
            Scope sc(this, "explicit_deposit");
            if (!packed) {
                hpq_launch(k_pack_explicit<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 8)), dim3(256), 0, st, S, quad);
                HPQ_LAUNCH_CHECK();
                packed = true;
            }
            const int nb = blocks_for(pl[s].n, 256);
            const bool d = det.w[0] != nullptr;
            const Quad<R>* q = quad;
            if (cfg.depos_derivative_type == 0) with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(d ? k_explicit_deposit<R, 0, true, ORD> : k_explicit_deposit<R, 0, false, ORD>, dim3(nb), dim3(256), 0, st, pl[s], S, g, q, det); });
            else if (cfg.depos_derivative_type == 1) with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(d ? k_explicit_deposit<R, 1, true, ORD> : k_explicit_deposit<R, 1, false, ORD>, dim3(nb), dim3(256), 0, st, pl[s], S, g, q, det); });
            else with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(d ? k_explicit_deposit<R, 2, true, ORD> : k_explicit_deposit<R, 2, false, ORD>, dim3(nb), dim3(256), 0, st, pl[s], S, g, q, det); });
            HPQ_LAUNCH_CHECK();
            det_flush({C_SX, C_SY});
        }
    }

    // ---- SALAME (Salame.cpp). The SALAME slice is slab components C_NCOMP + c (view SV).
    bool salame_slice(int islice) const {
        for (size_t b = 0; b < bm.size(); ++b)
            if (cfg.beams[b].do_salame && !sal_count[b].empty() && sal_count[b][islice] > 0) return true;
        return false;
    }
    Slab<R> salame_view() const {
        Slab<R> V = S;
        V.base = S.base + (size_t)C_NCOMP * S.cstride;
        return V;
    }
    // Fields::SolvePoissonEz on the SALAME slice
    void salame_ez(const Slab<R>& V) {
        hpq_launch(k_sal_rhs_ez<R>, dim3(blocks_for((long long)nx * ny, 256)), dim3(256), 0, st, V, g, sal_dst.stage, sal_dst.sj);
        HPQ_LAUNCH_CHECK();
        const int comps[1] = {C_EZ};
        sal_dst.solve(st, 1, V.base, V.cstride, V.pitch, comps);
    }
    void salame_deposit_jz(R* jz) {
        for (size_t b = 0; b < bm.size(); ++b)
            if (cfg.beams[b].do_salame) deposit_beam((int)b, 0, nullptr, nullptr, jz, nullptr);
    }
    // SalameModule (Salame.cpp:14-185), one level, no grid current; W is decided on the host
    // like the reference's (its print of the weight factor becomes a record in salame_log)
    void salame(int islice) {
        constexpr int N = C_NCOMP;
        const Slab<R> V = salame_view();
        const double zoff = g.plo[2] + 0.5 * g.dx[2];  // GetPosOffset(2, geom, domain)
        // the target is Ez of the first SALAME slice of a contiguous run, before SALAME (:21-29)
        if (islice + 1 != sal_last) {
            copies({{N + kSalEzTarget, C_EZ}});
            sal_overloaded = false;
            sal_zeta0 = islice * g.dx[2] + zoff;
        }
        sal_last = islice;
        // the plasma part of Sx, Sy alone, kept for step 4 (:32-39)
        zero({C_SY, C_SX});
        explicit_deposit();
        copies({{N + kSalSyBack, C_SY}, {N + kSalSxBack, C_SX}});
        for (int iter = 0; iter < cfg.salame_n_iter; ++iter) {
            const int it0 = iter;
            // step 1: Ez of the next slice with the present weights (:43-76)
            for (size_t s = 0; s < pl.size(); ++s) {
                if (pl[s].n == 0) continue;
                with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_plasma_push<R, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], S, g, 1, (const int*)nullptr); });
                HPQ_LAUNCH_CHECK();
            }
            copies({{N + C_JX, C_NJXB}, {N + C_JY, C_NJYB}});
            for (size_t s = 0; s < pl.size(); ++s)
                deposit_plasma((int)s, V.c(C_JX).p, V.c(C_JY).p, nullptr, nullptr, nullptr, nullptr);
            zero({N + C_EZ, N + C_JZB, N + C_SY, N + C_SX, N + C_BX, N + C_BY});
            salame_ez(V);
            copies({{N + kSalEzNoSalame, N + C_EZ}});
            // step 2: the Ez of the next slice from the SALAME beam alone (:78-123)
            salame_deposit_jz(V.c(C_JZB).p);
            hpq_launch(k_sal_sxsy<R>, dim3(blocks_for((long long)nx * ny, 256)), dim3(256), 0, st, V, g);
            HPQ_LAUNCH_CHECK();
            copies({{N + C_CHI, C_CHI}});  // the solve takes chi of this slice
            if (mg.cell) mg_solve_t<true>(V); else mg_solve_t<false>(V);
            zero({N + C_EZ, N + C_JX, N + C_JY});
            if (cfg.salame_do_advance) {
                for (size_t s = 0; s < pl.size(); ++s) {
                    if (pl[s].n == 0) continue;
                    with_order([&](auto o_) {
                        constexpr int ORD = decltype(o_)::value;
                        hpq_launch(k_sal_only_push<R, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], V, g);
                    });
                    HPQ_LAUNCH_CHECK();
                    deposit_plasma((int)s, V.c(C_JX).p, V.c(C_JY).p, nullptr, nullptr, nullptr, nullptr);
                }
            } else {
                hpq_launch(k_sal_jxjy_from_b<R>, dim3(blocks_for((long long)nx * ny, 256)), dim3(256), 0, st, S, V, g);
                HPQ_LAUNCH_CHECK();
            }
            salame_ez(V);
            // step 3: the weight factor (:125-158, SalameGetW :334-400)
            zero({N + C_JZB});
            salame_deposit_jz(V.c(C_JZB).p);
            hpq_launch(k_sal_sums<R>, dim3(1), dim3(1024), 0, st, V, sal_sums_d);
            HPQ_LAUNCH_CHECK();
            HPQ_CUDA(cudaMemcpyAsync(sal_sums_h, sal_sums_d, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
            HPQ_CUDA(cudaStreamSynchronize(st));
            const double sjz = sal_sums_h[3];
            double s_t = sal_sums_h[0] / sjz;
            const double s_no = sal_sums_h[1] / sjz, s_only = sal_sums_h[2] / sjz;
            const double args[3] = {(islice - 1) * g.dx[2] + zoff, sal_zeta0, s_t};  // Ez of the next slice
            s_t = cfg.salame_target.eval(args);
            double W = (s_t - s_no) / s_only + 1.0;
            if (W < 0 || sal_overloaded) {
                W = 0;
                iter = cfg.salame_n_iter - 1;
                sal_overloaded = true;
            }
            salame_log.insert(salame_log.end(), {(double)islice, (double)it0, W});
            if (!sal_overloaded && iter >= 1 && std::abs(W - 1.) < cfg.salame_relative_tolerance) iter = cfg.salame_n_iter - 1;
            for (size_t b = 0; b < bm.size(); ++b) {
                if (!cfg.beams[b].do_salame) continue;
                hpq_launch(k_sal_weight, dim3(148), dim3(256), 0, st, bm[b], (const Ctl*)ctl, W);
                HPQ_LAUNCH_CHECK();
            }
            // step 4: Bx, By of this slice with the new weights (:160-183)
            zero({C_JZB, C_SY, C_SX});
            for (size_t b = 0; b < bm.size(); ++b) deposit_beam((int)b, 0, nullptr, nullptr, S.c(C_JZB).p, nullptr);
            // (recomputes ExmBy, EypBx from the unchanged Psi: the same values)
            hpq_launch(k_grad_psi_sxsy<R>, dim3(blocks_for((long long)(nx + 2) * (ny + 2), 256)), dim3(256), 0, st, S, g);
            HPQ_LAUNCH_CHECK();
            {
                CopyList L{};
                L.n = 2;
                L.dst[0] = C_SY; L.src[0] = N + kSalSyBack;
                L.dst[1] = C_SX; L.src[1] = N + kSalSxBack;
                hpq_launch(k_add_comps<R>, dim3(blocks_for((long long)S.cstride, 256, 148 * 8)), dim3(256), 0, st, S, L);
                HPQ_LAUNCH_CHECK();
            }
            mg_solve();
        }
    }

    void mg_solve() {
        Scope sc(this, "multigrid");
        if (mg.cell) mg_solve_t<true>(S); else mg_solve_t<false>(S);
    }
    // the multigrid reads Sy, Sx, chi and writes Bx, By of slab MS
    template <bool CELL>
    void mg_solve_t(const Slab<R>& MS) { mg_run<CELL>(mg, MS); }
    template <bool CELL, class MGT, class RS>
    void mg_run(MGT& mg, const Slab<RS>& MS) {
        if (mg.coop_ok) {
            // the whole solve, iterations and decisions included, is one cooperative kernel
            mg.template solve_persistent<CELL>(st, MS, ctl, cfg.mg_tol_rel, cfg.mg_tol_abs, cfg.mg_max_iters);
            return;
        }
        if (capturing) {
            // inside the slice graph: a conditional WHILE node repeats the V-cycle body for as
            // long as the device-side decision (k_mg_init_decide / k_mg_decide) says so
            cudaStreamCaptureStatus cs;
            cudaGraph_t cg;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            HPQ_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps));
            cudaGraphConditionalHandle handle;
            HPQ_CUDA(cudaGraphConditionalHandleCreate(&handle, cg, 0, cudaGraphCondAssignDefault));
            mg.template pre<CELL>(st, MS, ctl, cfg.mg_tol_rel, cfg.mg_tol_abs, cfg.mg_max_iters, (unsigned long long)handle, 1);
            HPQ_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps));
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cnode;
            HPQ_CUDA(cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            HPQ_CUDA(cudaStreamBeginCaptureToGraph(st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            const long long l0 = g_launches;
            mg.template vcycle<CELL>(st2, MS, ctl, cfg.mg_max_iters, (unsigned long long)handle, 1);
            launches_body = g_launches - l0;
            body_launch_offset += launches_body;
            cudaGraph_t body_out;
            HPQ_CUDA(cudaStreamEndCapture(st2, &body_out));
            HPQ_CUDA(cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies));
            mg.template post<CELL>(st, MS, ctl);
            return;
        }
        mg.template pre<CELL>(st, MS, ctl, cfg.mg_tol_rel, cfg.mg_tol_abs, cfg.mg_max_iters, 0, 0);
        // the device decides after every V-cycle (Ctl::mg_go); without graphs the host reads
        // the decision back each cycle, like the reference's host-side max reduction
        HPQ_CUDA(cudaMemcpyAsync(&ctl_h->mg_go, &ctl->mg_go, sizeof(int), cudaMemcpyDeviceToHost, st));
        HPQ_CUDA(cudaStreamSynchronize(st));
        for (int it = 0; it < cfg.mg_max_iters && ctl_h->mg_go; ++it) {
            mg.template vcycle<CELL>(st, MS, ctl, cfg.mg_max_iters, 0, 0);
            HPQ_CUDA(cudaMemcpyAsync(&ctl_h->mg_go, &ctl->mg_go, sizeof(int), cudaMemcpyDeviceToHost, st));
            HPQ_CUDA(cudaStreamSynchronize(st));
        }
        mg.template post<CELL>(st, MS, ctl);
    }

    // ------------------------------------------------------------------ adjoint (adjoint.cuh)
    static bool adj_push_tangent() {
        static const bool on = [] {
            const char* e = getenv("HPQ_ADJ_PUSH");
            return e && std::string(e) == "tangent";
        }();
        return on;
    }
    bool adj_fwd = false;           // the slice graph is the adjoint forward (hooks, no beam push)
    double adj_plasma_scale = 1.0;  // plasma density multiplier applied when a step begins
    long long beam_gen = 0;         // changes whenever the beam stores change
    struct AdjBuf {
        int K = 0, C = 0;                 // slices per segment, segments (checkpoints)
        long long n = 0, cap = -1;        // plasma particles, witness store capacity
        double* rec_pl[8] = {};           // K slots: x, y, ux_h, uy_h, psi_h, ux, uy, psi
        uint8_t* rec_valid = nullptr;
        double* rec_f[RF_N] = {};         // K slots of each recorded field plane
        double* ck_pl[11] = {};           // C slots of the 11 plasma attributes
        uint8_t* ck_valid = nullptr;
        double* ck_slab = nullptr;        // C slots of the whole slab
        Slab<double> L{}, M{};            // adjoint planes; multigrid planes of the transposed solve
        double* lam[2][8] = {};           // adjoint of the plasma state (out / in, swapped per slice)
        double* lw = nullptr;             // adjoint of the plasma weights (accumulated)
        double* w_step = nullptr;         // plasma weights of the step
        double* lwb = nullptr;            // adjoint of the witness weights (store order)
        double* w0 = nullptr;             // witness weights before the profile
        long long w0_gen = -1;
        double* obj = nullptr;            // nz x 3 objective sums
        double* ions = nullptr;           // nz ion-background terms of dJ/dsigma
        double* knots = nullptr;          // parameters
        double* grad = nullptr;           // profile-knot gradient
        double* sig = nullptr;            // sum lambda_w w
        AdjCopy<R> ck_args{}, rec_args{};
        AdjRecMixed rec_mixed{};          // single precision: the record widened to double
        std::vector<void*> owned;
    } adjb;
    // single precision: the reverse sweep runs in double with its own multigrid and DST
    Multigrid<double>* mg64 = nullptr;
    PoissonDST<double>* dst64 = nullptr;

    int adjoint_nparams() const override { return cfg.adjoint.witness < 0 ? 0 : cfg.adjoint.n_params(); }

    template <class T>
    T* adj_alloc1(size_t count) {
        void* p = nullptr;
        HPQ_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        HPQ_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), st));
        adjb.owned.push_back(p);
        return static_cast<T*>(p);
    }
    void adj_release() {
        for (void* p : adjb.owned) cudaFree(p);
        adjb = AdjBuf{};
        if (mg64) { mg64->release(); delete mg64; mg64 = nullptr; }
        if (dst64) { dst64->release(); delete dst64; dst64 = nullptr; }
    }
    // buffers of the adjoint (once per simulation; the witness arrays follow the store capacity)
    void adj_setup() {
        AdjBuf& a = adjb;
        const int wb = cfg.adjoint.witness;
        if (a.K == 0) {
            const PlasmaDev<R>& P = pl[0];
            a.n = P.n;
            a.K = std::min(cfg.adjoint.checkpoint_interval, nz);
            a.C = (nz + a.K - 1) / a.K;
            const size_t n = (size_t)a.n, cs = S.cstride;
            for (auto& q : a.rec_pl) q = adj_alloc1<double>(n * a.K);
            a.rec_valid = adj_alloc1<uint8_t>(n * a.K);
            for (auto& q : a.rec_f) q = adj_alloc1<double>(cs * a.K);
            for (auto& q : a.ck_pl) q = adj_alloc1<double>(n * a.C);
            a.ck_valid = adj_alloc1<uint8_t>(n * a.C);
            a.ck_slab = adj_alloc1<double>(cs * C_NCOMP * a.C);
            for (Slab<double>* q : {&a.L, &a.M}) {
                q->nx = nx; q->ny = ny; q->pitch = S.pitch; q->rows = S.rows; q->cstride = cs;
            }
            a.L.base = adj_alloc1<double>(cs * A_NCOMP);
            a.M.base = adj_alloc1<double>(cs * (C_BY + 1));
            for (auto& side : a.lam)
                for (auto& q : side) q = adj_alloc1<double>(n);
            a.lw = adj_alloc1<double>(n);
            a.w_step = adj_alloc1<double>(n);
            a.obj = adj_alloc1<double>((size_t)nz * 3);
            a.ions = adj_alloc1<double>(nz);
            a.knots = adj_alloc1<double>(cfg.adjoint.n_params());
            a.grad = adj_alloc1<double>(cfg.adjoint.n_profile);
            a.sig = adj_alloc1<double>(1);
            // checkpoint: the 11 plasma attributes, the valid flags and the whole slab
            AdjCopy<R>& c = a.ck_args;
            c = AdjCopy<R>{};
            const R* src[11] = {P.x, P.y, P.w, P.ux, P.uy, P.psi, P.xp, P.yp, P.uxh, P.uyh, P.psih};
            for (int k = 0; k < 11; ++k) { c.src[k] = src[k]; c.dst[k] = (R*)a.ck_pl[k]; c.n[k] = a.n; }
            c.src[11] = S.base; c.dst[11] = (R*)a.ck_slab; c.n[11] = (long long)(cs * C_NCOMP);
            c.na = 12;
            c.vsrc = P.valid; c.vdst = a.ck_valid; c.nv = a.n;
            c.nz = nz; c.K = a.K;
            // record: the plasma state the reverse sweep reads and the recorded field planes
            AdjCopy<R>& r = a.rec_args;
            r = AdjCopy<R>{};
            const R* rsrc[8] = {P.x, P.y, P.uxh, P.uyh, P.psih, P.ux, P.uy, P.psi};
            for (int k = 0; k < 8; ++k) { r.src[k] = rsrc[k]; r.dst[k] = (R*)a.rec_pl[k]; r.n[k] = a.n; }
            for (int k = 0; k < RF_N; ++k) {
                r.src[8 + k] = S.c(kRecComp[k]).p; r.dst[8 + k] = (R*)a.rec_f[k]; r.n[8 + k] = (long long)cs;
            }
            r.na = 8 + RF_N;
            r.vsrc = P.valid; r.vdst = a.rec_valid; r.nv = a.n;
            r.nz = nz; r.K = a.K;
            if constexpr (std::is_same<R, float>::value) {
                AdjRecMixed& m = a.rec_mixed;
                m = AdjRecMixed{};
                for (int k = 0; k < 8; ++k) { m.pl[k] = rsrc[k]; m.dst[k] = a.rec_pl[k]; }
                m.ru = P.ru; m.rv = P.rv;
                m.xoff = g.xoff; m.yoff = g.yoff; m.dx = g.dx[0]; m.dy = g.dx[1];
                for (int k = 0; k < RF_N; ++k) { m.f[k] = S.c(kRecComp[k]).p; m.fdst[k] = a.rec_f[k]; }
                m.n = a.n; m.cs = (long long)cs;
                m.vsrc = P.valid; m.vdst = a.rec_valid;
                m.nz = nz; m.K = a.K;
                // the transposed multigrid and the Poisson solves of the reverse sweep, in double
                mg64 = new Multigrid<double>();
                mg64->init(nx, ny, g.dx[0], g.dx[1]);
                dst64 = new PoissonDST<double>();
                dst64->init(nx, ny, g.dx[0], g.dx[1], 3);
            }
            // the set-up above ran synchronous copies on the legacy stream
            HPQ_CUDA(cudaDeviceSynchronize());
        }
        if (a.cap != bm[wb].cap) {
            // the witness store grew: new per-particle arrays (freed with the others at release)
            a.lwb = adj_alloc1<double>((size_t)bm[wb].cap);
            a.w0 = adj_alloc1<double>((size_t)bm[wb].cap);
            a.cap = bm[wb].cap;
            a.w0_gen = -1;
        }
    }

    // objective J (and its gradient when grad != nullptr) for the parameters theta
    // In single precision the forward (and the recomputation of each segment) runs in FP32 and
    // records its state widened to double; the reverse sweep, the objective sums and the knot
    // reductions are FP64.
    double adjoint(const double* theta, double* grad) override {
        {
            const AdjointConfig& A = cfg.adjoint;
            if (A.witness < 0) throw InputError("no adjoint configured (adjoint.witness)");
            if (pl.size() != 1 || pl[0].n == 0) throw InputError("the adjoint needs exactly one plasma species");
            const int wb = A.witness;
            adj_setup();
            AdjBuf& a = adjb;
            const int np = A.n_params();
            HPQ_CUDA(cudaMemcpyAsync(a.knots, theta, np * sizeof(double), cudaMemcpyHostToDevice, st));
            const double ct = cfg.pc.c * physical_time;
            const double sigma = knot_value(theta + A.n_profile, ct, A.density_lo, A.density_hi, A.n_density, true);
            if (sigma == 0.0) throw InputError("the plasma density multiplier is zero at z = c t");
            // witness weights w0 * profile(z) in the read store
            BeamDev& W = bm[wb];
            if (a.w0_gen != beam_gen) {
                HPQ_CUDA(cudaMemcpyAsync(a.w0, W.buf[parity].w, W.cap * sizeof(double), cudaMemcpyDeviceToDevice, st));
                a.w0_gen = beam_gen;
            }
            hpq_launch(k_adj_profile, dim3(8, nz), dim3(256), 0, st, W, parity, nz, (const double*)a.w0,
                       (const double*)a.knots, A.profile_lo, A.profile_hi, A.n_profile);
            HPQ_LAUNCH_CHECK();
            // ---- forward: the march without the beam push, checkpoints and records. The slice
            // graph of the adjoint forward replaces the step's graph until this call returns.
            struct Restore {
                Sim* s;
                ~Restore() {
                    cudaStreamSynchronize(s->st);
                    s->adj_fwd = false;
                    s->adj_plasma_scale = 1.0;
                    s->invalidate_graph();
                }
            } restore{this};
            invalidate_graph();
            adj_fwd = true;
            adj_plasma_scale = sigma;
            begin_step(cur_step);
            adj_plasma_scale = 1.0;
            hpq_launch(k_adj_set_slice, dim3(1), dim3(1), 0, st, ctl, nz - 1, 1);
            HPQ_LAUNCH_CHECK();
            if constexpr (std::is_same<R, double>::value) {
                HPQ_CUDA(cudaMemcpyAsync(a.w_step, pl[0].w, a.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            } else {
                hpq_launch(k_adj_widen<R>, dim3(blocks_for(a.n, 256, 148 * 4)), dim3(256), 0, st, (const R*)pl[0].w,
                           a.w_step, a.n);
                HPQ_LAUNCH_CHECK();
            }
            for (int s = nz - 1; s >= 0; --s) solve_slice(s);
            std::vector<double> obj((size_t)nz * 3);
            HPQ_CUDA(cudaMemcpyAsync(obj.data(), a.obj, obj.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            HPQ_CUDA(cudaStreamSynchronize(st));
            double S0 = 0, S1 = 0, S2 = 0;
            for (int s = nz - 1; s >= 0; --s) { S0 += obj[3 * s]; S1 += obj[3 * s + 1]; S2 += obj[3 * s + 2]; }
            const double Ebar = S0 != 0 ? S1 / S0 : 0.0;
            const double J = S0 != 0 ? S2 / S0 - Ebar * Ebar : 0.0;
            if (grad) {
                adj_reverse(J, Ebar, S0);
                std::vector<double> gp(A.n_profile), ions(nz);
                double sig = 0;
                HPQ_CUDA(cudaMemcpyAsync(gp.data(), a.grad, A.n_profile * sizeof(double), cudaMemcpyDeviceToHost, st));
                HPQ_CUDA(cudaMemcpyAsync(ions.data(), a.ions, nz * sizeof(double), cudaMemcpyDeviceToHost, st));
                HPQ_CUDA(cudaMemcpyAsync(&sig, a.sig, sizeof(double), cudaMemcpyDeviceToHost, st));
                HPQ_CUDA(cudaStreamSynchronize(st));
                for (int k = 0; k < np; ++k) grad[k] = k < A.n_profile ? gp[k] : 0.0;
                double dsig = sig;
                for (int s = 0; s < nz; ++s) dsig += ions[s];
                dsig /= sigma;
                int kk; double fr;
                if (knot_interval(ct, A.density_lo, A.density_hi, A.n_density, true, kk, fr)) {
                    if (A.n_density == 1) grad[A.n_profile] += dsig;
                    else { grad[A.n_profile + kk] += (1 - fr) * dsig; grad[A.n_profile + kk + 1] += fr * dsig; }
                }
            }
            HPQ_CUDA(cudaMemcpyAsync(ctl_h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
            HPQ_CUDA(cudaStreamSynchronize(st));
            if (ctl_h->mgp_bar_err) throw CudaError("hpmg: grid barrier of the persistent multigrid solve timed out");
            if (ctl_h->mg_status == 1) throw CudaError("hpmg: failed to converge within the iteration limit");
            if (ctl_h->mg_status == 2) throw CudaError("hpmg: diverged");
            return J;
        }
    }

    void adj_reverse(double J, double Ebar, double S0) {
        AdjBuf& a = adjb;
        const AdjointConfig& A = cfg.adjoint;
        const int wb = A.witness;
        const size_t n = (size_t)a.n;
        for (auto* q : a.lam[0]) HPQ_CUDA(cudaMemsetAsync(q, 0, n * sizeof(double), st));
        HPQ_CUDA(cudaMemsetAsync(a.lw, 0, n * sizeof(double), st));
        HPQ_CUDA(cudaMemsetAsync(a.lwb, 0, a.cap * sizeof(double), st));
        HPQ_CUDA(cudaMemsetAsync(a.ions, 0, nz * sizeof(double), st));
        HPQ_CUDA(cudaMemsetAsync(a.M.base, 0, a.M.cstride * (C_BY + 1) * sizeof(double), st));
        // slices behind the first objective slice do not influence J: their adjoints are zero
        int smin = nz;
        for (int s = 0; s < nz; ++s) {
            const double zc = cfg.prob_lo[2] + (s + 0.5) * g.dx[2];
            if (zc >= A.objective_lo && zc <= A.objective_hi) { smin = s; break; }
        }
        int cur = 0;
        for (int c = a.C - 1; c >= 0; --c) {
            const int hi = nz - 1 - c * a.K, lo_seg = std::max(hi - a.K + 1, 0), lo = std::max(lo_seg, smin);
            if (hi < lo) continue;
            if (c != a.C - 1) {
                // recompute the segment from its checkpoint (records only)
                for (int k = 0; k < 11; ++k)
                    HPQ_CUDA(cudaMemcpyAsync((void*)a.ck_args.src[k], (const R*)a.ck_pl[k] + (size_t)c * n, n * sizeof(R),
                                             cudaMemcpyDeviceToDevice, st));
                HPQ_CUDA(cudaMemcpyAsync(pl[0].valid, a.ck_valid + (size_t)c * n, n, cudaMemcpyDeviceToDevice, st));
                HPQ_CUDA(cudaMemcpyAsync(S.base, (const R*)a.ck_slab + (size_t)c * S.cstride * C_NCOMP,
                                         S.cstride * C_NCOMP * sizeof(R), cudaMemcpyDeviceToDevice, st));
                hpq_launch(k_adj_set_slice, dim3(1), dim3(1), 0, st, ctl, hi, 0);
                HPQ_LAUNCH_CHECK();
                cur_islice = hi;
                for (int s = hi; s >= lo; --s) solve_slice(s);
            }
            for (int s = lo; s <= hi; ++s) {
                adj_reverse_slice(s, s - lo_seg, cur, J, Ebar, S0);
                cur = 1 - cur;
            }
        }
        // parameters: witness profile knots and the plasma weight term of dJ/dsigma
        hpq_launch(k_adj_knot_grad, dim3(A.n_profile), dim3(256), 0, st, bm[wb], parity, nz, (const double*)a.lwb,
                   (const double*)a.w0, A.profile_lo, A.profile_hi, A.n_profile, a.grad);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_adj_dot, dim3(1), dim3(1024), 0, st, (const double*)a.lw, (const double*)a.w_step, a.n, a.sig);
        HPQ_LAUNCH_CHECK();
    }

    void adj_reverse_slice(int s, int slot, int cur, double J, double Ebar, double S0) {
        AdjBuf& a = adjb;
        const AdjointConfig& A = cfg.adjoint;
        const int wb = A.witness;
        const size_t n = (size_t)a.n, cs = S.cstride;
        const PlasmaDev<R>& P0 = pl[0];
        AdjPlasma P{a.rec_pl[0] + slot * n, a.rec_pl[1] + slot * n, a.rec_pl[2] + slot * n, a.rec_pl[3] + slot * n,
                    a.rec_pl[4] + slot * n, a.rec_pl[5] + slot * n, a.rec_pl[6] + slot * n, a.rec_pl[7] + slot * n,
                    a.w_step, a.rec_valid + slot * n, a.n, P0.charge, P0.mass};
        AdjRecF F;
        for (int k = 0; k < RF_N; ++k) F.f[k] = F2<double>{a.rec_f[k] + slot * cs, S.pitch};
        AdjL L;
        for (int k = 0; k < A_NCOMP; ++k) L.f[k] = a.L.c(k);
        AdjLam lout{a.lam[cur][0], a.lam[cur][1], a.lam[cur][2], a.lam[cur][3], a.lam[cur][4], a.lam[cur][5],
                    a.lam[cur][6], a.lam[cur][7]};
        AdjLam lin{a.lam[1 - cur][0], a.lam[1 - cur][1], a.lam[1 - cur][2], a.lam[1 - cur][3], a.lam[1 - cur][4],
                   a.lam[1 - cur][5], a.lam[1 - cur][6], a.lam[1 - cur][7]};
        Geo gg = g;
        const int nbp = blocks_for(a.n * kPushSeeds, 256), nbd = blocks_for(a.n, 256);
        HPQ_CUDA(cudaMemsetAsync(a.L.base, 0, cs * A_NCOMP * sizeof(double), st));
        for (int k = 0; k < 8; ++k) HPQ_CUDA(cudaMemsetAsync(a.lam[1 - cur][k], 0, n * sizeof(double), st));
        // plasma push: reverse mode, one thread per particle (HPQ_ADJ_PUSH=tangent in the
        // environment selects the forward-mode form, one thread per particle and seed, for
        // cross-checks)
        Scope sc_push(this, "adj_push");
        if (adj_push_tangent()) hpq_launch(k_adj_push, dim3(nbp), dim3(256), 0, st, P, lout, lin, F, L, gg);
        else hpq_launch(k_adj_push_rev, dim3(nbd), dim3(256), 0, st, P, lout, lin, F, L, gg);
        HPQ_LAUNCH_CHECK();
        // objective
        const double zc = cfg.prob_lo[2] + (s + 0.5) * g.dx[2];
        if (zc >= A.objective_lo && zc <= A.objective_hi && S0 != 0.0) {
            hpq_launch(k_adj_objective, dim3(blocks_for((long long)nx * ny, 256)), dim3(256), 0, st, L, F, nx, ny, J, Ebar, S0);
            HPQ_LAUNCH_CHECK();
        }
        // multigrid (transposed solve)
        Scope sc_mg(this, "adj_multigrid");
        const int ncell = (int)cs;
        hpq_launch(k_adj_mg_pre, dim3(blocks_for(ncell, 256)), dim3(256), 0, st, a.M, L, F, (int)mg.cell);
        HPQ_LAUNCH_CHECK();
        if constexpr (std::is_same<R, double>::value) {
            if (mg.cell) mg_run<true>(mg, a.M); else mg_run<false>(mg, a.M);
        } else {
            if (mg64->cell) mg_run<true>(*mg64, a.M); else mg_run<false>(*mg64, a.M);
        }
        hpq_launch(k_adj_mg_post, dim3(blocks_for((long long)nx * ny, 256)), dim3(256), 0, st, a.M, L, F, (int)mg.cell);
        HPQ_LAUNCH_CHECK();
        // explicit Sx/Sy deposit
        Scope sc_ex(this, "adj_explicit");
        if (cfg.depos_derivative_type == 0) hpq_launch(k_adj_explicit<0>, dim3(nbd), dim3(256), 0, st, P, lin, a.lw, F, L, gg);
        else if (cfg.depos_derivative_type == 1) hpq_launch(k_adj_explicit<1>, dim3(nbd), dim3(256), 0, st, P, lin, a.lw, F, L, gg);
        else hpq_launch(k_adj_explicit<2>, dim3(nbd), dim3(256), 0, st, P, lin, a.lw, F, L, gg);
        HPQ_LAUNCH_CHECK();
        // beam part of Sx/Sy, -grad Psi, Poisson stage; the three solves; right-hand sides
        Scope sc_f(this, "adj_fields");
        {
            PoissonDST<double>* d64 = nullptr;
            if constexpr (std::is_same<R, double>::value) d64 = &dst;
            else d64 = dst64;
            hpq_launch(k_adj_sxsy_stage, dim3(blocks_for((long long)(nx + 2) * (ny + 2), 256)), dim3(256), 0, st, L, gg, nx, ny,
                       d64->stage, d64->sk, d64->sj);
            HPQ_LAUNCH_CHECK();
            const int comps[3] = {A_VPSI, A_VEZ, A_VBZ};
            d64->solve(st, 3, a.L.base, a.L.cstride, a.L.pitch, comps);
        }
        hpq_launch(k_adj_rhs_t, dim3(blocks_for((long long)(nx + 2) * (ny + 2), 256)), dim3(256), 0, st, L, gg, nx, ny);
        HPQ_LAUNCH_CHECK();
        // plasma deposit
        Scope sc_dep(this, "adj_deposit");
        hpq_launch(k_adj_deposit, dim3(nbd), dim3(256), 0, st, P, lin, a.lw, L, gg);
        HPQ_LAUNCH_CHECK();
        // ion background (scaled by the density multiplier like the plasma)
        if (cfg.any_neutralize_background()) {
            hpq_launch(k_adj_plane_dot<R>, dim3(1), dim3(1024), 0, st, L.f[A_RM], S.c(C_IONS), nx, ny, a.ions + s);
            HPQ_LAUNCH_CHECK();
        }
        // beam deposits of the witness: jz (and rho - jz) of this slice's particles, their jx/jy
        // (deposited one slice earlier into this slice's jx/jy), and the jx/jy of the previous and
        // next slices' particles read by the beam part of Sx/Sy
        Scope sc_b(this, "adj_beam");
        const bool jxy = cfg.do_beam_jx_jy_deposition;
        const int pitch = S.pitch;
        hpq_launch(k_adj_beam, dim3(148), dim3(256), 0, st, bm[wb], parity, s, (const double*)L.f[A_JZB].p,
                   cfg.do_beam_jz_minus_rho ? (const double*)L.f[A_RM].p : (const double*)nullptr,
                   (jxy && s <= nz - 2) ? (const double*)L.f[A_JX].p : (const double*)nullptr,
                   (const double*)L.f[A_JY].p, pitch, gg, a.lwb);
        HPQ_LAUNCH_CHECK();
        if (jxy && s + 1 <= nz - 2) {
            hpq_launch(k_adj_beam, dim3(148), dim3(256), 0, st, bm[wb], parity, s + 1, (const double*)nullptr,
                       (const double*)nullptr, (const double*)L.f[A_PJX].p, (const double*)L.f[A_PJY].p, pitch, gg, a.lwb);
            HPQ_LAUNCH_CHECK();
        }
        if (jxy && s - 1 >= 0) {
            hpq_launch(k_adj_beam, dim3(148), dim3(256), 0, st, bm[wb], parity, s - 1, (const double*)nullptr,
                       (const double*)nullptr, (const double*)L.f[A_NJX].p, (const double*)L.f[A_NJY].p, pitch, gg, a.lwb);
            HPQ_LAUNCH_CHECK();
        }
    }

    // Stable sort of species sp by bin (k_reorder_* in kernels.cuh), on the library's stream.
    void reorder_plasma(int sp) {
        PlasmaDev<R>& P = pl[sp];
        if (P.n == 0) return;
        const long long bins = (long long)(nx + 1) * (ny + 1);
        if (ro_cap < P.n || ro_bins < bins) {
            release_reorder();
            ro_cap = 0;
            for (auto& q : pl) ro_cap = std::max(ro_cap, q.n);
            ro_bins = bins;
            const size_t n = (size_t)ro_cap;
            R** arrs[] = {&ro_tmp.x, &ro_tmp.y, &ro_tmp.w, &ro_tmp.ux, &ro_tmp.uy, &ro_tmp.psi, &ro_tmp.xp, &ro_tmp.yp,
                          &ro_tmp.uxh, &ro_tmp.uyh, &ro_tmp.psih};
            for (R** a : arrs) HPQ_CUDA(cudaMalloc(a, n * sizeof(R)));
            HPQ_CUDA(cudaMalloc(&ro_tmp.valid, n));
            if (std::is_same<R, float>::value) {
                HPQ_CUDA(cudaMalloc(&ro_tmp.ru, n * sizeof(float)));
                HPQ_CUDA(cudaMalloc(&ro_tmp.rv, n * sizeof(float)));
            }
            HPQ_CUDA(cudaMalloc(&ro_key, n * sizeof(int)));
            HPQ_CUDA(cudaMalloc(&ro_perm, n * sizeof(int)));
            HPQ_CUDA(cudaMalloc(&ro_cnt, (size_t)bins * sizeof(int)));
            HPQ_CUDA(cudaMalloc(&ro_start, (size_t)bins * sizeof(int)));
            HPQ_CUDA(cudaMalloc(&ro_fill, (size_t)bins * sizeof(int)));
            HPQ_CUDA(cudaMalloc(&ro_bsum, (size_t)((bins + 1023) / 1024) * sizeof(int)));
        }
        PlasmaDev<R> T = ro_tmp;
        T.n = P.n;
        if (!P.ru) T.ru = T.rv = nullptr;
        const PlasmaSpecies& S_ = cfg.plasmas[sp];
        const int nblk = (int)((bins + 1023) / 1024);
        const unsigned pb = blocks_for(P.n, 256);
        HPQ_CUDA(cudaMemsetAsync(ro_cnt, 0, (size_t)bins * sizeof(int), st));
        hpq_launch(k_reorder_keys<R>, dim3(pb), dim3(256), 0, st, P, g, S_.reorder_idx_type[0], S_.reorder_idx_type[1],
                   ro_key, ro_cnt);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_scan_blocks, dim3(nblk), dim3(1024), 0, st, (const int*)ro_cnt, ro_start, ro_bsum, bins);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_scan_totals, dim3(1), dim3(1024), 0, st, ro_bsum, nblk);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_scan_add, dim3(blocks_for(bins, 256)), dim3(256), 0, st, ro_start, (const int*)ro_bsum, ro_fill, bins);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_reorder_scatter, dim3(pb), dim3(256), 0, st, (const int*)ro_key, P.n, ro_fill, ro_perm);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_reorder_bins, dim3(blocks_for(bins, 256)), dim3(256), 0, st, (const int*)ro_start,
                   (const int*)ro_cnt, bins, ro_perm);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_reorder_move<R>, dim3(pb), dim3(256), 0, st, P, T, (const int*)ro_perm, 1);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_reorder_move<R>, dim3(pb), dim3(256), 0, st, P, T, (const int*)ro_perm, 0);
        HPQ_LAUNCH_CHECK();
        if (reordered.size() < pl.size()) reordered.resize(pl.size(), false);
        reordered[sp] = true;
    }
    void release_reorder() {
        for (void* q : {(void*)ro_tmp.x, (void*)ro_tmp.y, (void*)ro_tmp.w, (void*)ro_tmp.ux, (void*)ro_tmp.uy,
                        (void*)ro_tmp.psi, (void*)ro_tmp.xp, (void*)ro_tmp.yp, (void*)ro_tmp.uxh, (void*)ro_tmp.uyh,
                        (void*)ro_tmp.psih, (void*)ro_tmp.valid, (void*)ro_tmp.ru, (void*)ro_tmp.rv, (void*)ro_key,
                        (void*)ro_perm, (void*)ro_cnt, (void*)ro_start, (void*)ro_fill, (void*)ro_bsum})
            if (q) cudaFree(q);
        ro_tmp = PlasmaDev<R>{};
        ro_key = ro_perm = ro_cnt = ro_start = ro_fill = ro_bsum = nullptr;
        ro_cap = ro_bins = 0;
    }

    // one slice: replay the captured graph, or launch kernel by kernel (profiling mode)
    void solve_slice(int islice) override {
        if (islice != cur_islice) throw InputError("slices must be solved from the head (nz-1) to the tail (0)");
        // ReorderParticles(islice) at the start of SolveOneSlice (Hipace.cpp:594-595); not in the
        // adjoint forward, whose reverse sweep follows particles by index from slice to slice
        if (!adj_fwd)
            for (size_t sp = 0; sp < pl.size(); ++sp) {
                const int period = cfg.plasmas[sp].reorder_period;
                if (period > 0 && islice % period == 0) reorder_plasma((int)sp);
            }
        // the SALAME step runs kernel by kernel: its iterations end on host decisions
        if (use_graphs && !profiling && !sal_step) {
            if (!slice_exec) capture_slice();
            HPQ_CUDA(cudaGraphLaunch(slice_exec, st));
            launches_total += launches_top;
        } else {
            const long long l0 = g_launches;
            record_slice();
            launches_total += g_launches - l0;
        }
        cur_islice--;
    }
    void capture_slice() {
        invalidate_graph();
        HPQ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        const long long l0 = g_launches;
        body_launch_offset = 0;
        try {
            record_slice();
        } catch (...) {
            capturing = false;
            cudaGraph_t g0;
            cudaStreamEndCapture(st, &g0);
            if (g0) cudaGraphDestroy(g0);
            cudaGetLastError();
            throw;
        }
        capturing = false;
        launches_top = g_launches - l0 - body_launch_offset;
        HPQ_CUDA(cudaStreamEndCapture(st, &slice_graph));
        HPQ_CUDA(cudaGraphInstantiate(&slice_exec, slice_graph, 0));
        size_t nn = 0;
        HPQ_CUDA(cudaGraphGetNodes(slice_graph, nullptr, &nn));
        graph_nodes = (long long)nn;
    }
    void invalidate_graph() {
        if (slice_exec) { cudaGraphExecDestroy(slice_exec); slice_exec = nullptr; }
        if (slice_graph) { cudaGraphDestroy(slice_graph); slice_graph = nullptr; }
    }

    // Hipace::SolveOneSlice (Hipace.cpp:556-728)
    // beam in-situ reductions, push and partition of slice ctl->islice + lag (Hipace.cpp:680-700)
    void beam_work(int lag) {
        for (size_t b = 0; b < bm.size(); ++b) {
            // beam in-situ reductions before the push (Hipace.cpp:680-681)
            if (insitu_beam_d[b]) {
                const double r = cfg.beams[b].insitu_radius;
                hpq_launch(k_beam_insitu, dim3(1), dim3(1024), 0, st, bm[b], (const Ctl*)ctl, (int)b,
                           r < 1e150 ? r * r : 1e300, 1.0 / cfg.pc.c, insitu_beam_d[b], lag, nz);
                HPQ_LAUNCH_CHECK();
            }
            {
                Scope sc(this, "beam_push");
                with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_beam_push<R, ORD>, dim3(148 * 2), dim3(256), 0, st, bm[b], ctl, (int)b, SB, g, lag); });
                HPQ_LAUNCH_CHECK();
            }
            Scope sc2(this, "beam_partition");
            hpq_launch(k_beam_partition, dim3(1), dim3(1024), 0, st, bm[b], ctl, (int)b, g, 1, lag);
            HPQ_LAUNCH_CHECK();
        }
    }

    void record_slice() {
        const bool ex = cfg.explicit_solver;
        if (adj_fwd) {
            // adjoint forward: the state entering a segment head is checkpointed
            hpq_launch(k_adj_checkpoint<R>, dim3(148 * 4), dim3(256), 0, st, (const Ctl*)ctl, adjb.ck_args);
            HPQ_LAUNCH_CHECK();
        }
        // (the adjoint forward leaves the beam as it is: its push only feeds the next step)
        const bool beams = !adj_fwd && !bm.empty();
        if (beams) {
            // the previous slice's beam push and partition, beside this slice's solve (nothing
            // at the head of the box)
            OnStream on(this, beam_begin());
            beam_work(1);
        }
        if (ex) {
            if (cfg.deposit_rho) zero({C_CHI, C_SY, C_SX, C_EXMBY, C_EYPBX, C_JZB, C_RHOMJZ, C_NJXB, C_NJYB, C_RHOMJZB, C_RHO});
            else zero({C_CHI, C_SY, C_SX, C_EXMBY, C_EYPBX, C_JZB, C_RHOMJZ, C_NJXB, C_NJYB, C_RHOMJZB});
            // beam deposits (own components) run beside the plasma deposit
            {
                OnStream on(this, side_begin());
                // jz_beam of this slice and jx_beam/jy_beam of the next slice (the reference
                // deposits the latter after the Psi/Ez/Bz solve, Hipace.cpp:656-657; the two are
                // independent)
                for (size_t b = 0; b < bm.size(); ++b) {
                    Scope sc(this, "beam_deposit");
                    // a SALAME beam deposits only jz in the SALAME step (MultiBeam.cpp:50-56)
                    const bool sal = sal_step && cfg.beams[b].do_salame;
                    const bool nj = cfg.do_beam_jx_jy_deposition && !sal;
                    with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_beam_deposit_this_next<R, ORD>, dim3(148 * 2), dim3(256), 0, st,
                        bm[b], ctl, S.c(C_JZB).p, cfg.do_beam_jz_minus_rho && !sal ? S.c(C_RHOMJZB).p : nullptr,
                        nj ? S.c(C_NJXB).p : nullptr, nj ? S.c(C_NJYB).p : nullptr, S.pitch, g, det); });
                    HPQ_LAUNCH_CHECK();
                    det_flush({C_JZB, C_RHOMJZB, C_NJXB, C_NJYB});
                }
            }
            for (size_t s = 0; s < pl.size(); ++s)
                deposit_plasma((int)s, S.c(C_JX).p, S.c(C_JY).p, nullptr, cfg.deposit_rho ? S.c(C_RHO).p : nullptr,
                               S.c(C_CHI).p, S.c(C_RHOMJZ).p);
            side_end();
        } else {
            if (cfg.deposit_rho) zero({C_EXMBY, C_EYPBX, C_JX, C_JY, C_JZ, C_RHOMJZ, C_RHO});
            else zero({C_EXMBY, C_EYPBX, C_JX, C_JY, C_JZ, C_RHOMJZ});
            for (size_t s = 0; s < pl.size(); ++s)
                deposit_plasma((int)s, S.c(C_JX).p, S.c(C_JY).p, S.c(C_JZ).p, cfg.deposit_rho ? S.c(C_RHO).p : nullptr,
                               nullptr, S.c(C_RHOMJZ).p);
            for (size_t b = 0; b < bm.size(); ++b)
                deposit_beam((int)b, 0, cfg.do_beam_jx_jy_deposition ? S.c(C_JX).p : nullptr,
                             cfg.do_beam_jx_jy_deposition ? S.c(C_JY).p : nullptr, S.c(C_JZ).p,
                             cfg.do_beam_jz_minus_rho ? S.c(C_RHOMJZ).p : nullptr);
        }
        field_solve_psi_ez_bz();
        if (ex) {
            explicit_deposit();
            mg_solve();
            if (sal_step && !capturing && salame_slice(cur_islice)) salame(cur_islice);
        } else {
            pc_loop();
        }
        if (adj_fwd) {
            // adjoint forward: objective sums and the record of this slice (plasma state after the
            // deposit's QSA test, the fields the reverse sweep reads)
            hpq_launch(k_adj_objective_sums<R>, dim3(1), dim3(1024), 0, st, S, (const Ctl*)ctl, g,
                       cfg.adjoint.objective_lo, cfg.adjoint.objective_hi, adjb.obj);
            HPQ_LAUNCH_CHECK();
            if constexpr (std::is_same<R, double>::value)
                hpq_launch(k_adj_record<R>, dim3(148 * 4), dim3(256), 0, st, (const Ctl*)ctl, adjb.rec_args);
            else
                hpq_launch(k_adj_record_mixed, dim3(148 * 4), dim3(256), 0, st, (const Ctl*)ctl, adjb.rec_mixed);
            HPQ_LAUNCH_CHECK();
        }
        if (diag_list.n > 0) {
            hpq_launch(k_diag_copy<R>, dim3(blocks_for((long long)diag_plane() * diag_list.n, 256)), dim3(256), 0, st, S, ctl,
                       diag_list, diag_buf, nz, diag_sel());
            HPQ_LAUNCH_CHECK();
        }
        // field in-situ reductions after every field of the slice is known (Hipace.cpp:684-685)
        if (insitu_fields_d) {
            hpq_launch(k_field_insitu<R>, dim3(1), dim3(1024), 0, st, S, (const Ctl*)ctl, cfg.pc.c, insitu_fields_d);
            HPQ_LAUNCH_CHECK();
        }
        // the beam push and partition (beam arrays, Ctl) run beside the plasma push and the
        // component shifts (plasma arrays, slab planes the pushes do not read)
        if (beams) {
            // this slice's gathered fields for its beam push (behind the previous slice's beam
            // work on the same side stream, beside the plasma push)
            OnStream on(this, beam_begin());
            HPQ_CUDA(cudaMemcpyAsync(SB.c(C_EZ).p, S.c(C_EZ).p, (size_t)(C_PSI - C_EZ + 1) * S.cstride * sizeof(R),
                                     cudaMemcpyDeviceToDevice, st));
        }
        if (ex) {
            // ShiftSlices (Fields.cpp:588-604) beside the plasma push: the push reads Psi, Ez, Bx,
            // By, Bz, none of the shifted planes
            OnStream on(this, side_begin());
            copies({{C_PJXB, C_JXB}, {C_PJYB, C_JYB}, {C_JXB, C_NJXB}, {C_JYB, C_NJYB}, {C_JX, C_NJXB}, {C_JY, C_NJYB}});
        }
        for (size_t s = 0; s < pl.size(); ++s) {
            if (pl[s].n == 0) continue;
            Scope sc(this, "plasma_push");
            with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_plasma_push<R, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], S, g, 0, (const int*)nullptr); });
            HPQ_LAUNCH_CHECK();
        }
        if (ex) {
            side_end();
        } else {
            copies({{C_PCPBX, C_PBX}, {C_PCPBY, C_PBY}, {C_PBX, C_BX}, {C_PBY, C_BY}, {C_PJX, C_JX}, {C_PJY, C_JY}});
        }
        if (beams) beam_end();
        hpq_launch(k_slice_done, dim3(1), dim3(1), 0, st, ctl);
        HPQ_LAUNCH_CHECK();
    }

    // Hipace::PredictorCorrectorLoopToSolveBxBy (Hipace.cpp:935-1031)
    void pc_loop() {
        const long long nxy = (long long)nx * ny;
        const double tol = cfg.predcorr_B_error_tolerance;
        const int maxit = cfg.predcorr_max_iterations;
        HPQ_CUDA(cudaMemsetAsync(&ctl->pc_sum[0], 0, 2 * sizeof(double), st));
        hpq_launch(k_pc_norms<R>, dim3(det.w[0] ? 1 : blocks_for(nxy, 256, 148 * 4)), dim3(det.w[0] ? 1024 : 256), 0, st, S, C_PBX, C_PBY, C_PCPBX, C_PCPBY, ctl, 0, tol);
        HPQ_LAUNCH_CHECK();
        hpq_launch(k_pc_guess<R>, dim3(blocks_for((long long)S.cstride, 256)), dim3(256), 0, st, S, ctl);
        HPQ_LAUNCH_CHECK();
        for (int it = 0; it < maxit; ++it) {
            // iterations after convergence are predicated off on the device (Ctl::pc_go)
            for (size_t s = 0; s < pl.size(); ++s) {
                if (pl[s].n == 0) continue;
                with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_plasma_push<R, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], S, g, 1, &ctl->pc_go); });
                HPQ_LAUNCH_CHECK();
                DepOut<R> o{S.c(C_NJX).p, S.c(C_NJY).p, nullptr, nullptr, nullptr, nullptr, S.pitch};
                with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(det.w[0] ? k_plasma_deposit<R, true, ORD> : k_plasma_deposit<R, false, ORD>, dim3(blocks_for(pl[s].n, 256)), dim3(256), 0, st, pl[s], o, g, pl[s].charge, &ctl->pc_go, det); });
                HPQ_LAUNCH_CHECK();
                det_flush({C_NJX, C_NJY});
            }
            if (cfg.do_beam_jx_jy_deposition)
                for (size_t b = 0; b < bm.size(); ++b) deposit_beam_if((int)b);
            const int comps[2] = {C_PCIBX, C_PCIBY};
            hpq_launch(k_rhs_bxby<R>, dim3(blocks_for(nxy, 256)), dim3(256), 0, st, S, g, pc_dst.stage, pc_dst.sk, pc_dst.sj);
            HPQ_LAUNCH_CHECK();
            pc_dst.solve(st, 2, S.base, S.cstride, S.pitch, comps);
            hpq_launch(k_pc_norms<R>, dim3(det.w[0] ? 1 : blocks_for(nxy, 256, 148 * 4)), dim3(det.w[0] ? 1024 : 256), 0, st, S, C_BX, C_BY, C_PCIBX, C_PCIBY, ctl, 1, tol);
            HPQ_LAUNCH_CHECK();
            hpq_launch(k_pc_mix<R>, dim3(blocks_for((long long)S.cstride, 256)), dim3(256), 0, st, S, ctl, cfg.predcorr_B_mixing_factor, tol, maxit);
            HPQ_LAUNCH_CHECK();
        }
    }
    void deposit_beam_if(int b) {
        with_order([&](auto o_) { constexpr int ORD = decltype(o_)::value; hpq_launch(k_beam_deposit<R, ORD>, dim3(148 * 2), dim3(256), 0, st, bm[b], ctl, 1, S.c(C_NJX).p, S.c(C_NJY).p, nullptr, nullptr, S.pitch, g, 1, det); });
        HPQ_LAUNCH_CHECK();
        det_flush({C_NJX, C_NJY});
    }

    // ----------------------------------------------------------------------------- io
    void get_field(const std::string& name, double* out) override {
        const int c = comp_from_name(name, cfg.explicit_solver);
        HPQ_CUDA(cudaStreamSynchronize(st));
        std::vector<R> tmp(S.cstride);
        HPQ_CUDA(cudaMemcpy(tmp.data(), S.c(c).p, S.cstride * sizeof(R), cudaMemcpyDeviceToHost));
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) out[(size_t)j * nx + i] = (double)tmp[(size_t)(j + kGuardAlloc) * S.pitch + i + kGuardAlloc];
    }
    long long diag_plane() const { return cfg.diag_type == 0 ? (long long)nx * ny : cfg.diag_type == 1 ? nx : ny; }
    DiagSel diag_sel() const {
        DiagSel d{cfg.diag_type, 0, 0, 1.0, 0.0};
        if (cfg.diag_type == 1) mid_plane(ny, d.lo, d.hi, d.wlo, d.whi);
        if (cfg.diag_type == 2) mid_plane(nx, d.lo, d.hi, d.wlo, d.whi);
        return d;
    }
    void set_diag(const std::vector<std::string>& names) override {
        if (names.size() > 24) throw InputError("at most 24 diagnostic components");
        synchronize();
        invalidate_graph();
        diag_names = names;
        diag_list = CompList{};
        for (auto& n : names) diag_list.c[diag_list.n++] = comp_from_name(n, cfg.explicit_solver);
        if (diag_buf) { cudaFree(diag_buf); diag_buf = nullptr; }
        if (!names.empty()) {
            const size_t n = (size_t)names.size() * diag_plane() * nz;
            HPQ_CUDA(cudaMalloc(&diag_buf, n * sizeof(double)));
            // on the library's stream, ahead of the slices that fill it
            HPQ_CUDA(cudaMemsetAsync(diag_buf, 0, n * sizeof(double), st));
        }
    }
    void get_diag(const std::string& name, double* out) override {
        auto it = std::find(diag_names.begin(), diag_names.end(), name);
        if (it == diag_names.end()) throw InputError("component '" + name + "' is not in the diagnostic list");
        const size_t q = it - diag_names.begin();
        const size_t n = (size_t)diag_plane() * nz;
        HPQ_CUDA(cudaStreamSynchronize(st));
        HPQ_CUDA(cudaMemcpy(out, diag_buf + q * n, n * sizeof(double), cudaMemcpyDeviceToHost));
    }
    long long plasma_count(int sp) override { return pl.at(sp).n; }
    void get_plasma(int sp, double* out12) override {
        HPQ_CUDA(cudaStreamSynchronize(st));
        const PlasmaDev<R>& p = pl.at(sp);
        const size_t n = p.n;
        const R* arr[11] = {p.x, p.y, p.w, p.ux, p.uy, p.psi, p.xp, p.yp, p.uxh, p.uyh, p.psih};
        std::vector<R> tmp(n);
        // lattice points of the particles in their current order: the host copy, or, after a
        // reorder, the points in cell units carried by the particles
        std::vector<double> lx, ly;
        const bool perm = p.ru && sp < (int)reordered.size() && reordered[sp];
        if (perm) {
            std::vector<float> f(n);
            lx.resize(n);
            ly.resize(n);
            HPQ_CUDA(cudaMemcpy(f.data(), p.ru, n * sizeof(float), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) lx[i] = g.xoff + (double)f[i] * g.dx[0];
            HPQ_CUDA(cudaMemcpy(f.data(), p.rv, n * sizeof(float), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) ly[i] = g.yoff + (double)f[i] * g.dx[1];
        }
        for (int k = 0; k < 11; ++k) {
            HPQ_CUDA(cudaMemcpy(tmp.data(), arr[k], n * sizeof(R), cudaMemcpyDeviceToHost));
            // x, y, xp, yp are displacements from the lattice point, psi, psih are psi - 1 when
            // p.ru is set
            const std::vector<double>* ref = nullptr;
            if (p.ru && (k == 0 || k == 6)) ref = perm ? &lx : &hx0.at(sp);
            if (p.ru && (k == 1 || k == 7)) ref = perm ? &ly : &hy0.at(sp);
            const double off = (p.ru && (k == 5 || k == 10)) ? 1.0 : 0.0;
            for (size_t i = 0; i < n; ++i) out12[k * n + i] = (double)tmp[i] + (ref ? (*ref)[i] : 0.0) + off;
        }
        std::vector<uint8_t> v(n);
        HPQ_CUDA(cudaMemcpy(v.data(), p.valid, n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) out12[11 * n + i] = v[i];
    }
    void synchronize() override { HPQ_CUDA(cudaStreamSynchronize(st)); }
    Stats stats() override { return st_host; }
};

}  // namespace hpq
