// C ABI of the slice loop (declared in include/hpq.h). All exceptions stop here and turn into
// status codes plus a message kept on the handle.
#include <algorithm>
#include <cmath>
#include <memory>
#include <sstream>
#include <string>

#include "../../include/hpq.h"
#include "config.hpp"
#include "sim.cuh"

struct hpq_handle {
    hpq::SimConfig cfg;
    std::unique_ptr<hpq::SimBase> sim;
    int precision = HPQ_PLAIN_FP64;
    bool graphs = false;
    bool deterministic = false;
    bool initialised = false;
    bool in_step = false;
    std::string err;
};

namespace {
thread_local std::string g_create_error;

template <class F>
int guarded(hpq_handle* h, F&& f) {
    if (!h) return HPQ_ERR_ARG;
    try {
        h->err.clear();
        return f();
    } catch (const hpq::InputError& e) {
        h->err = e.what();
        return HPQ_ERR_INPUT;
    } catch (const hpq::CudaError& e) {
        h->err = e.what();
        const std::string m = e.what();
        if (m.find("failed to converge") != std::string::npos) return HPQ_ERR_NOT_CONVERGED;
        if (m.find("diverged") != std::string::npos) return HPQ_ERR_DIVERGED;
        return HPQ_ERR_CUDA;
    } catch (const std::exception& e) {
        h->err = e.what();
        return HPQ_ERR_CUDA;
    }
}

int need_init(hpq_handle* h) {
    if (!h->initialised) { h->err = "hpq_init has not been called"; return HPQ_ERR_STATE; }
    return 0;
}
}  // namespace

extern "C" {

int hpq_create(const char* input_text, hpq_handle** out) {
    if (!input_text || !out) return HPQ_ERR_ARG;
    try {
        hpq::InputStore in;
        in.parse_text(input_text);
        auto h = std::make_unique<hpq_handle>();
        h->cfg = hpq::build_config(in);
        *out = h.release();
        g_create_error.clear();
        return HPQ_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        *out = nullptr;
        return HPQ_ERR_INPUT;
    }
}

const char* hpq_create_error(void) { return g_create_error.c_str(); }

void hpq_destroy(hpq_handle* h) { delete h; }

const char* hpq_last_error(const hpq_handle* h) { return h ? h->err.c_str() : "null handle"; }

int hpq_n_cell(const hpq_handle* h, int n_cell[3]) {
    if (!h || !n_cell) return HPQ_ERR_ARG;
    for (int d = 0; d < 3; ++d) n_cell[d] = h->cfg.n_cell[d];
    return HPQ_OK;
}

const char* hpq_beam_name(const hpq_handle* h, int beam) {
    if (!h || beam < 0 || beam >= (int)h->cfg.beams.size()) return nullptr;
    return h->cfg.beams[(size_t)beam].name.c_str();
}

int hpq_salame_log(hpq_handle* h, double* out, int64_t* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!n) return (int)HPQ_ERR_ARG;
        const std::vector<double>& v = h->sim->salame_record();
        if (out) std::copy(v.begin(), v.end(), out);
        *n = (int64_t)v.size();
        return (int)HPQ_OK;
    });
}

int hpq_max_step(const hpq_handle* h, int* max_step) {
    if (!h || !max_step) return HPQ_ERR_ARG;
    *max_step = h->cfg.max_step;
    return HPQ_OK;
}

int hpq_time(hpq_handle* h, double* t) {
    return guarded(h, [&] {
        if (!t) return (int)HPQ_ERR_ARG;
        *t = h->sim ? h->sim->time() : 0.0;
        return (int)HPQ_OK;
    });
}

int hpq_diag_count(const hpq_handle* h, int64_t* n) {
    if (!h || !n) return HPQ_ERR_ARG;
    const hpq::SimConfig& c = h->cfg;
    const int64_t plane = c.diag_type == 0 ? (int64_t)c.n_cell[0] * c.n_cell[1] : c.diag_type == 1 ? c.n_cell[0] : c.n_cell[1];
    *n = plane * c.n_cell[2];
    return HPQ_OK;
}

int hpq_set_precision(hpq_handle* h, int mode) {
    return guarded(h, [&] {
        if (h->initialised) { h->err = "hpq_set_precision must come before hpq_init"; return (int)HPQ_ERR_STATE; }
        if (mode != HPQ_PLAIN_FP64 && mode != HPQ_MIXED) { h->err = "unknown precision mode"; return (int)HPQ_ERR_ARG; }
        h->precision = mode;
        return (int)HPQ_OK;
    });
}

int hpq_init(hpq_handle* h) {
    return guarded(h, [&] {
        if (h->initialised) { h->err = "hpq_init called twice"; return (int)HPQ_ERR_STATE; }
        if (h->precision == HPQ_MIXED) h->sim.reset(new hpq::Sim<float>(h->cfg));
        else h->sim.reset(new hpq::Sim<double>(h->cfg));
        h->sim->init();
        h->sim->set_graphs(h->graphs);
        h->sim->set_deterministic(h->deterministic);
        h->initialised = true;
        return (int)HPQ_OK;
    });
}

int hpq_set_beam(hpq_handle* h, int beam, const double* x, const double* y, const double* z, const double* w,
                 const double* ux, const double* uy, const double* uz, const int64_t* id, int64_t n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (n < 0 || (n > 0 && (!x || !y || !z || !w || !ux || !uy || !uz))) return (int)HPQ_ERR_ARG;
        if (h->in_step) { h->err = "hpq_set_beam inside a step"; return (int)HPQ_ERR_STATE; }
        h->sim->set_beam(beam, x, y, z, w, ux, uy, uz, (const long long*)id, n);
        return (int)HPQ_OK;
    });
}

int hpq_beam_count(hpq_handle* h, int beam, int64_t* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!n || beam < 0 || beam >= (int)h->cfg.beams.size()) return (int)HPQ_ERR_ARG;
        *n = h->sim->beam_count(beam);
        return (int)HPQ_OK;
    });
}

int hpq_get_beam(hpq_handle* h, int beam, double* x, double* y, double* z, double* w, double* ux, double* uy,
                 double* uz, int64_t* id) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (beam < 0 || beam >= (int)h->cfg.beams.size()) return (int)HPQ_ERR_ARG;
        h->sim->get_beam(beam, x, y, z, w, ux, uy, uz, (long long*)id);
        return (int)HPQ_OK;
    });
}

int hpq_beam_slice_count(hpq_handle* h, int beam, int islice, int64_t* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!n || beam < 0 || beam >= (int)h->cfg.beams.size() || islice < 0 || islice >= h->cfg.n_cell[2])
            return (int)HPQ_ERR_ARG;
        *n = h->sim->beam_slice_count(beam, islice);
        return (int)HPQ_OK;
    });
}

int hpq_get_beam_slice(hpq_handle* h, int beam, int islice, double* x, double* y, double* z, double* w, double* ux,
                       double* uy, double* uz, int64_t* id) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (beam < 0 || beam >= (int)h->cfg.beams.size() || islice < 0 || islice >= h->cfg.n_cell[2])
            return (int)HPQ_ERR_ARG;
        h->sim->get_beam_slice(beam, islice, x, y, z, w, ux, uy, uz, (long long*)id);
        return (int)HPQ_OK;
    });
}

int hpq_put_beam_slice(hpq_handle* h, int beam, int islice, const double* x, const double* y, const double* z,
                       const double* w, const double* ux, const double* uy, const double* uz, const int64_t* id,
                       int64_t n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (beam < 0 || beam >= (int)h->cfg.beams.size() || islice < 0 || islice >= h->cfg.n_cell[2] || n < 0 ||
            (n > 0 && (!x || !y || !z || !w || !ux || !uy || !uz || !id)))
            return (int)HPQ_ERR_ARG;
        if (!h->in_step) { h->err = "hpq_put_beam_slice outside a step"; return (int)HPQ_ERR_STATE; }
        h->sim->put_beam_slice(beam, islice, x, y, z, w, ux, uy, uz, (const long long*)id, n);
        return (int)HPQ_OK;
    });
}

int hpq_set_time(hpq_handle* h, double t) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (h->in_step) { h->err = "hpq_set_time inside a step"; return (int)HPQ_ERR_STATE; }
        if (!std::isfinite(t)) return (int)HPQ_ERR_ARG;
        h->sim->set_time(t);
        return (int)HPQ_OK;
    });
}

int hpq_begin_step(hpq_handle* h, int step) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (h->in_step) { h->err = "hpq_begin_step inside a step"; return (int)HPQ_ERR_STATE; }
        if (std::isinf(h->sim->time())) {
            h->err = "the step at hipace.max_time has run; the simulation has ended";
            return (int)HPQ_ERR_STATE;
        }
        h->sim->begin_step(step);
        h->in_step = true;
        return (int)HPQ_OK;
    });
}

int hpq_solve_slice(hpq_handle* h, int islice) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!h->in_step) { h->err = "hpq_solve_slice outside a step"; return (int)HPQ_ERR_STATE; }
        if (islice < 0 || islice >= h->cfg.n_cell[2]) return (int)HPQ_ERR_ARG;
        h->sim->solve_slice(islice);
        return (int)HPQ_OK;
    });
}

int hpq_end_step(hpq_handle* h) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!h->in_step) { h->err = "hpq_end_step outside a step"; return (int)HPQ_ERR_STATE; }
        h->in_step = false;
        h->sim->end_step();
        return (int)HPQ_OK;
    });
}

int hpq_step(hpq_handle* h, int step) {
    int r = hpq_begin_step(h, step);
    if (r) return r;
    for (int s = h->cfg.n_cell[2] - 1; s >= 0; --s) {
        r = hpq_solve_slice(h, s);
        if (r) { h->in_step = false; return r; }
    }
    return hpq_end_step(h);
}

int hpq_get_field(hpq_handle* h, const char* comp, double* out) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!comp || !out) return (int)HPQ_ERR_ARG;
        h->sim->get_field(comp, out);
        return (int)HPQ_OK;
    });
}

int hpq_set_diag(hpq_handle* h, const char* comps) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!comps) return (int)HPQ_ERR_ARG;
        std::istringstream in(comps);
        std::vector<std::string> v;
        std::string s;
        while (in >> s) v.push_back(s);
        h->sim->set_diag(v);
        return (int)HPQ_OK;
    });
}

int hpq_get_diag(hpq_handle* h, const char* comp, double* out) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!comp || !out) return (int)HPQ_ERR_ARG;
        h->sim->get_diag(comp, out);
        return (int)HPQ_OK;
    });
}

int hpq_insitu_size(hpq_handle* h, const char* what, int64_t* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!what || !n) return (int)HPQ_ERR_ARG;
        const long long k = h->sim->insitu_size(what);
        if (k < 0) { h->err = std::string("no in-situ diagnostic '") + what + "'"; return (int)HPQ_ERR_ARG; }
        *n = k;
        return (int)HPQ_OK;
    });
}

int hpq_get_insitu(hpq_handle* h, const char* what, double* out) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!what || !out) return (int)HPQ_ERR_ARG;
        if (h->in_step) { h->err = "hpq_get_insitu inside a step"; return (int)HPQ_ERR_STATE; }
        if (h->sim->insitu_size(what) < 0) { h->err = std::string("no in-situ diagnostic '") + what + "'"; return (int)HPQ_ERR_ARG; }
        if (!h->sim->get_insitu(what, out)) { h->err = "no diagnostic step has run yet"; return (int)HPQ_ERR_STATE; }
        return (int)HPQ_OK;
    });
}

int hpq_plasma_count(hpq_handle* h, int sp, int64_t* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!n || sp < 0 || sp >= (int)h->cfg.plasmas.size()) return (int)HPQ_ERR_ARG;
        *n = h->sim->plasma_count(sp);
        return (int)HPQ_OK;
    });
}

int hpq_get_plasma(hpq_handle* h, int sp, double* out) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!out || sp < 0 || sp >= (int)h->cfg.plasmas.size()) return (int)HPQ_ERR_ARG;
        h->sim->get_plasma(sp, out);
        return (int)HPQ_OK;
    });
}

int hpq_set_graphs(hpq_handle* h, int on) {
    return guarded(h, [&] {
        h->graphs = on != 0;
        if (h->sim) h->sim->set_graphs(h->graphs);
        return (int)HPQ_OK;
    });
}

int hpq_set_deterministic(hpq_handle* h, int on) {
    return guarded(h, [&] {
        if (h->in_step) { h->err = "hpq_set_deterministic inside a step"; return (int)HPQ_ERR_STATE; }
        h->deterministic = on != 0;
        if (h->sim) h->sim->set_deterministic(h->deterministic);
        return (int)HPQ_OK;
    });
}

int hpq_adjoint_nparams(hpq_handle* h, int* n) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!n) return (int)HPQ_ERR_ARG;
        *n = h->sim->adjoint_nparams();
        return (int)HPQ_OK;
    });
}

int hpq_adjoint_grad(hpq_handle* h, const double* knots, double* grad, double* objective) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!knots || !objective) return (int)HPQ_ERR_ARG;
        if (h->in_step) { h->err = "hpq_adjoint_grad inside a step"; return (int)HPQ_ERR_STATE; }
        if (h->sim->adjoint_nparams() == 0) { h->err = "no adjoint configured (adjoint.witness)"; return (int)HPQ_ERR_INPUT; }
        *objective = h->sim->adjoint(knots, grad);
        return (int)HPQ_OK;
    });
}

int hpq_synchronize(hpq_handle* h) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        h->sim->synchronize();
        return (int)HPQ_OK;
    });
}

int hpq_set_profiling(hpq_handle* h, int on) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        h->sim->set_profiling(on != 0);
        return (int)HPQ_OK;
    });
}

int hpq_get_profile(hpq_handle* h, const char* kernel_class, double* total_ms, int64_t* launches) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        if (!kernel_class || !total_ms || !launches) return (int)HPQ_ERR_ARG;
        long long n = 0;
        h->sim->get_profile(kernel_class, total_ms, &n);
        *launches = n;
        return (int)HPQ_OK;
    });
}

void* hpq_stream(hpq_handle* h) { return (h && h->sim) ? (void*)h->sim->stream() : nullptr; }

int hpq_get_counters(hpq_handle* h, int64_t* mg_vcycles, int64_t* slices, int64_t* plasma_pushes,
                     int64_t* kernel_launches) {
    return guarded(h, [&] {
        if (int r = need_init(h)) return r;
        hpq::Stats s = h->sim->stats();
        if (mg_vcycles) *mg_vcycles = s.mg_vcycles;
        if (slices) *slices = s.slices;
        if (plasma_pushes) *plasma_pushes = s.plasma_pushes;
        if (kernel_launches) *kernel_launches = s.launches;
        return (int)HPQ_OK;
    });
}

}  // extern "C"
