// hpq — command-line driver of libhpq, the counterpart of the reference's executable
// (src/main.cpp: amrex::Initialize(argc, argv) reads the input file named first and the
// `key = value` overrides after it, then Hipace::InitData() and Hipace::Evolve()).
//
//   hpq <inputs> [key=value ...] [--precision fp64|mixed] [--no-graphs] [--deterministic]
//       [--checksum [comps]] [--quiet] [--dry-run]
//
// Overrides follow ParmParse's command-line form: a token containing '=' (or followed by a token
// that starts with '=') opens a new `key = value` line and later tokens continue its value, so
// `amr.n_cell=64 64 100`, `amr.n_cell="64 64 100"` and `max_step = 3` all work; they are appended
// after the file, where later lines override earlier ones. Steps run 0 .. max_step and the loop
// ends after the step at hipace.max_time (Hipace.cpp:401-419). --checksum prints, after the
// last step, the reference's regression checksum (tests/checksum: sum of |Q| over the 3-D output
// of each field component of the last iteration, and sums of |attribute| over each beam) as one
// JSON object. --dry-run parses and validates the inputs, prints the grid and max_step and exits
// without touching the GPU. Errors print hpq_last_error and exit 1 (the reference aborts).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hpq.h"

namespace {

const char* kAllComps =
    "Bx By Bz ExmBy EypBx Ez Psi Sx Sy chi jx jx_beam jy jy_beam jz_beam rho rhomjz";

int usage() {
    std::fprintf(stderr,
                 "usage: hpq <inputs> [key=value ...] [--precision fp64|mixed] [--no-graphs]\n"
                 "           [--deterministic] [--checksum [\"comp comp ...\"]] [--quiet] [--dry-run]\n");
    return 2;
}

void fail(hpq_handle* h, int rc, const char* what) {
    std::fprintf(stderr, "hpq: %s failed (code %d): %s\n", what, rc, h ? hpq_last_error(h) : hpq_create_error());
    if (h) hpq_destroy(h);
    std::exit(1);
}

// ParmParse command-line tokens -> input lines
std::string override_lines(const std::vector<std::string>& tok) {
    std::string out, line;
    for (size_t i = 0; i < tok.size(); ++i) {
        const std::string& t = tok[i];
        const bool key_here = t.find('=') != std::string::npos && t[0] != '=';
        const bool key_next = i + 1 < tok.size() && !tok[i + 1].empty() && tok[i + 1][0] == '=';
        if ((key_here || key_next) && !line.empty()) {
            out += line + "\n";
            line.clear();
        }
        line += (line.empty() ? "" : " ") + t;
    }
    if (!line.empty()) out += line + "\n";
    return out;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2 || !std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help")) return usage();
    std::ifstream f(argv[1]);
    if (!f) {
        std::fprintf(stderr, "hpq: cannot read input file %s\n", argv[1]);
        return 1;
    }
    std::stringstream text;
    text << f.rdbuf() << "\n";
    int precision = HPQ_PLAIN_FP64, graphs = 1, deterministic = 0, quiet = 0, dry = 0;
    bool checksum = false;
    std::string comps = kAllComps;
    std::vector<std::string> tok;
    for (int i = 2; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--precision" && i + 1 < argc) {
            const std::string p = argv[++i];
            if (p == "fp64") precision = HPQ_PLAIN_FP64;
            else if (p == "mixed") precision = HPQ_MIXED;
            else return usage();
        } else if (a == "--no-graphs") {
            graphs = 0;
        } else if (a == "--deterministic") {
            deterministic = 1;
        } else if (a == "--quiet") {
            quiet = 1;
        } else if (a == "--dry-run") {
            dry = 1;
        } else if (a == "--checksum") {
            checksum = true;
            if (i + 1 < argc && std::strncmp(argv[i + 1], "--", 2) && !std::strchr(argv[i + 1], '=')) comps = argv[++i];
        } else if (a.compare(0, 2, "--") == 0) {
            return usage();
        } else {
            tok.push_back(a);
        }
    }
    text << override_lines(tok);

    hpq_handle* h = nullptr;
    int rc = hpq_create(text.str().c_str(), &h);
    if (rc) fail(nullptr, rc, "reading the inputs");
    if ((rc = hpq_set_precision(h, precision))) fail(h, rc, "hpq_set_precision");
    if ((rc = hpq_set_graphs(h, graphs))) fail(h, rc, "hpq_set_graphs");
    if ((rc = hpq_set_deterministic(h, deterministic))) fail(h, rc, "hpq_set_deterministic");
    int n_cell[3] = {0, 0, 0}, max_step = 0;
    hpq_n_cell(h, n_cell);
    hpq_max_step(h, &max_step);
    if (dry) {
        std::printf("n_cell %d %d %d  max_step %d\n", n_cell[0], n_cell[1], n_cell[2], max_step);
        for (int b = 0; hpq_beam_name(h, b); ++b) std::printf("beam %s\n", hpq_beam_name(h, b));
        hpq_destroy(h);
        return 0;
    }
    if ((rc = hpq_init(h))) fail(h, rc, "hpq_init");
    if (checksum && (rc = hpq_set_diag(h, comps.c_str()))) fail(h, rc, "hpq_set_diag");

    using clock = std::chrono::steady_clock;
    const auto t_start = clock::now();
    for (int step = 0; step <= max_step; ++step) {
        double t = 0;
        hpq_time(h, &t);
        if (std::isinf(t)) break;
        const auto t0 = clock::now();
        if ((rc = hpq_step(h, step))) fail(h, rc, "hpq_step");
        if ((rc = hpq_synchronize(h))) fail(h, rc, "hpq_synchronize");
        const double s = std::chrono::duration<double>(clock::now() - t0).count();
        if (!quiet)
            std::printf("step %d  time %.10g  %.3f ms  %.1f slices/s\n", step, t, s * 1e3, n_cell[2] / s);
    }
    const double total = std::chrono::duration<double>(clock::now() - t_start).count();
    if (!quiet) std::printf("total %.3f s\n", total);

    if (checksum) {
        int64_t n = 0;
        hpq_diag_count(h, &n);
        std::vector<double> buf((size_t)n);
        std::printf("{\n  \"lev=0\": {");
        std::istringstream in(comps);
        std::string c;
        bool first = true;
        while (in >> c) {
            if ((rc = hpq_get_diag(h, c.c_str(), buf.data()))) fail(h, rc, "hpq_get_diag");
            double sum = 0;
            for (double v : buf) sum += std::fabs(v);
            std::printf("%s\n    \"%s\": %.14g", first ? "" : ",", c.c_str(), sum);
            first = false;
        }
        std::printf("\n  }");
        for (int b = 0;; ++b) {
            const char* name = hpq_beam_name(h, b);
            if (!name) break;
            int64_t nb = 0;
            if ((rc = hpq_beam_count(h, b, &nb))) fail(h, rc, "hpq_beam_count");
            std::vector<double> a[7];
            for (auto& v : a) v.resize((size_t)nb);
            std::vector<int64_t> id((size_t)nb);
            if ((rc = hpq_get_beam(h, b, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data(),
                                   a[6].data(), id.data())))
                fail(h, rc, "hpq_get_beam");
            static const char* names[7] = {"x", "y", "z", "w", "ux", "uy", "uz"};
            std::printf(",\n  \"%s\": {\n    \"num_particles\": %lld", name, (long long)nb);
            long long ids = 0;
            for (int64_t k = 0; k < nb; ++k) ids += id[(size_t)k];
            std::printf(",\n    \"id\": %lld", ids);
            for (int k = 0; k < 7; ++k) {
                double sum = 0;
                for (double v : a[k]) sum += std::fabs(v);
                std::printf(",\n    \"%s\": %.14g", names[k], sum);
            }
            std::printf("\n  }");
        }
        std::printf("\n}\n");
    }
    hpq_destroy(h);
    return 0;
}
