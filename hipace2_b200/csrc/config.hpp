// Simulation parameters of the quasi-static slice loop, read from reference-style input keys.
//
// Keys, defaults and meanings follow the reference:
//   hipace.*      Hipace.cpp:33-60, 74-244 and Hipace.H:180-300 (defaults)
//   amr.*, geometry.*, boundary.*   Hipace.cpp:176-230, 297-391
//   fields.*      Fields.cpp:29-47
//   <plasma>.*    PlasmaParticleContainer.cpp:27-187, PlasmaParticleContainer.H:151-200
//   <beam>.*      BeamParticleContainer.cpp:41-290, BeamParticleContainer.H:206-300
// Features that the reference has but this slice loop does not implement (mesh refinement,
// lasers, ionization, collisions, periodic/open field boundaries, adaptive dt, openPMD
// beams) are rejected with an explicit error instead of being silently ignored.
#pragma once

#include <limits>
#include <string>
#include <vector>

#include "inputs.hpp"

namespace hpq {

enum class ParticleBC : int { Reflecting = 0, Periodic = 1, Absorbing = 2 };

struct PhysConst {
    double c, ep0, mu0, q_e, m_e, m_p;
};

inline PhysConst constants_normalized() { return {1.0, 1.0, 1.0, 1.0, 1.0, 1836.15267343}; }
inline PhysConst constants_SI() {
    return {299792458.0, 8.8541878128e-12, 1.25663706212e-06, 1.602176634e-19,
            9.1093837015e-31, 1.67262192369e-27};
}

struct PlasmaSpecies {
    std::string name;
    double charge = 0, mass = 0;
    Expr density;             // density(x,y,z), z = c*t
    int ppc[2] = {0, 0};
    double u_mean[3] = {0, 0, 0};
    double u_std[3] = {0, 0, 0};
    double radius = 1e300;    // +inf in the reference
    double hollow_core_radius = 0;
    double max_qsa_weighting_factor = 35.0;
    double min_density = 0;
    int n_subcycles = 1;
    bool neutralize_background = true;
    bool prevent_centered_particle = false;
    bool thermal = false;     // u_std != 0: momenta drawn every step (rng.hpp plasma_thermal_u)
    // reorder by cell every reorder_period slices (PlasmaParticleContainer.cpp:197-208), binned
    // to cells (0) or nodes (1) per axis
    int reorder_period = 0;
    int reorder_idx_type[2] = {0, 0};
};

enum class BeamInjection : int { FixedPPC = 0, FixedWeight = 1, FixedWeightPDF = 2 };
enum class BeamProfile : int { Gaussian = 0, Flattop = 1, Can = 2 };

struct BeamSpecies {
    std::string name;
    BeamInjection injection = BeamInjection::FixedWeight;
    BeamProfile profile = BeamProfile::Gaussian;
    double charge = 0, mass = 0;
    double density = 0;              // peak density (fixed_ppc: profile density)
    double zmin = -1e300, zmax = 1e300, radius = 1e300;
    bool do_salame = false;          // <beam>.do_salame (BeamParticleContainer.cpp:66)
    // external fields of the beam push, Ex Ey Ez Bx By Bz as functions of (x, y, z, t)
    // (<beam>.external_E/B(x,y,z,t), BeamParticleContainer.cpp:72-86)
    bool use_external = false;
    Expr external[6];
    double position_mean[3] = {0, 0, 0};
    double position_std[3] = {0, 0, 0};
    int ppc[3] = {1, 1, 1};
    double u_mean[3] = {0, 0, 0};
    double u_std[3] = {0, 0, 0};
    long long num_particles = 0;
    double total_charge = 0;         // fixed_weight: Q (normalized: already divided by dV)
    double z_foc = 0;
    double duz_per_uz0_dzeta = 0;
    bool do_symmetrize = false;
    bool do_z_push = true;
    int n_subcycles = 10;
    double min_density = 0;
    // in-situ diagnostics (BeamParticleContainer.cpp:61-63, 476-548)
    int insitu_period = 0;
    double insitu_radius = 1e300;
    // fixed_weight_pdf (BeamParticleContainer.cpp:200-249): longitudinal pdf(z); mean x, mean y,
    // std x, std y of z; u_mean x y z and u_std x y z of z; pdf sub-slices per slice
    Expr pdf;
    Expr pdf_pos[4];
    Expr pdf_u[6];
    int pdf_ref_ratio = 4;
    bool peak_density_specified = false;
};

// Adjoint of one step of the explicit slice march with respect to a beam-loading objective.
// The reference has no adjoint; these keys belong to this library. The parameter vector is
//   theta[0 .. n_profile)                 witness current-profile knots: the witness weights are
//                                         multiplied by the piecewise-linear profile through
//                                         these values at n_profile equidistant points of
//                                         [profile_lo, profile_hi] in zeta (zero outside);
//   theta[n_profile .. n_profile+n_density) plasma-density knots: the plasma (and neutralising
//                                         ion) weights are multiplied by the piecewise-linear
//                                         profile through these values over [density_lo,
//                                         density_hi] in z = c t, clamped to the end values.
// Objective: the current-weighted variance of Ez over the slices whose centre lies in
// [objective_lo, objective_hi]: J = S2/S0 - (S1/S0)^2, S_n = sum jz_beam * Ez^n.
struct AdjointConfig {
    int witness = -1;  // beam index; -1: no adjoint configured
    double profile_lo = -7, profile_hi = -5;
    int n_profile = 64;
    double density_lo = 0, density_hi = 1;
    int n_density = 8;
    double objective_lo = -7, objective_hi = -5;
    int checkpoint_interval = 32;
    int n_params() const { return n_profile + n_density; }
};

// Piecewise-linear interpolation on n equidistant knots over [lo, hi]: value = (1-f) v[k] +
// f v[k+1]. Returns false outside [lo, hi] unless `clamp`, which then holds the end value.
inline bool knot_interval(double z, double lo, double hi, int n, bool clamp, int& k, double& f) {
    if (n < 1) return false;
    if (n == 1) { k = 0; f = 0; return clamp || (z >= lo && z <= hi); }
    if (z < lo || z > hi) {
        if (!clamp) return false;
        k = z < lo ? 0 : n - 2;
        f = z < lo ? 0.0 : 1.0;
        return true;
    }
    const double t = (z - lo) / (hi - lo) * (n - 1);
    k = (int)t;
    if (k > n - 2) k = n - 2;
    f = t - k;
    return true;
}
inline double knot_value(const double* v, double z, double lo, double hi, int n, bool clamp) {
    int k; double f;
    if (!knot_interval(z, lo, hi, n, clamp, k, f)) return 0.0;
    if (n == 1) return v[0];
    return (1.0 - f) * v[k] + f * v[k + 1];
}

struct SimConfig {
    bool normalized_units = false;
    PhysConst pc{};
    int n_cell[3] = {0, 0, 0};
    double prob_lo[3] = {0, 0, 0};
    double prob_hi[3] = {0, 0, 0};
    double dx[3] = {0, 0, 0};
    ParticleBC particle_bc = ParticleBC::Absorbing;
    double particle_lo[2] = {0, 0};
    double particle_hi[2] = {0, 0};
    int max_step = 0;
    double dt = 0;
    double max_time = 1e300;
    long long random_seed = 0;
    bool has_random_seed = false;
    int depos_order_xy = 2;
    int depos_derivative_type = 2;
    bool explicit_solver = true;
    double mg_tol_rel = 1.e-4;
    double mg_tol_abs = 2.2250738585072014e-308;  // numeric_limits<double>::min()
    int mg_max_iters = 200;
    double predcorr_B_error_tolerance = 4e-2;
    int predcorr_max_iterations = 30;
    double predcorr_B_mixing_factor = 0.05;
    bool do_beam_jx_jy_deposition = true;
    bool do_beam_jz_minus_rho = false;
    bool deposit_rho = false;
    int fields_insitu_period = 0;  // fields.insitu_period (Fields.cpp:41, 1289-1346)
    int diag_type = 0;             // diagnostic.diag_type: 0 xyz, 1 xz, 2 yz (see mid_plane)
    AdjointConfig adjoint;
    // SALAME beam-loading weights (Hipace.cpp:137-143, Hipace.H:284-301)
    int salame_n_iter = 5;
    bool salame_do_advance = true;
    Expr salame_target;  // hipace.salame_Ez_target(zeta,zeta_initial,Ez_initial)
    double salame_relative_tolerance = 1e-4;
    std::vector<PlasmaSpecies> plasmas;
    std::vector<BeamSpecies> beams;
    bool any_neutralize_background() const {
        for (auto& p : plasmas) if (p.neutralize_background) return true;
        return false;
    }
    bool any_salame() const {
        for (auto& b : beams) if (b.do_salame) return true;
        return false;
    }
};

// diagnostic.diag_type (Diagnostic.cpp:51-61): 0 xyz (whole slices), 1 xz (the plane y = domain
// centre), 2 yz (x = domain centre). The plane value is Fields::Copy's order-1 interpolation
// (Fields.cpp:413-533) at the centre of n cells: the middle cell for odd n, the mean of the two
// middle cells for even n.
inline void mid_plane(int n, int& lo, int& hi, double& wlo, double& whi) {
    if (n % 2) { lo = hi = (n - 1) / 2; wlo = 1.0; whi = 0.0; }
    else { lo = n / 2 - 1; hi = n / 2; wlo = 0.5; whi = 0.5; }
}

// Time step of the step that starts at time t (Hipace::Evolve, Hipace.cpp:424-435): a step that
// starts at max_time is a last step with dt = 0, after which the time is infinite and the step
// loop ends (Hipace.cpp:413-419); a step that would cross max_time is shortened to end on it.
struct StepTime {
    double dt, next;
};
inline StepTime step_time(double t, double dt, double max_time) {
    if (t == max_time) return {0.0, std::numeric_limits<double>::infinity()};
    if ((t + dt >= max_time && t < max_time) || (t + dt <= max_time && t > max_time)) return {max_time - t, max_time};
    return {dt, t + dt};
}

// utils::doDiagnostics (IOUtil.cpp:75-82)
inline bool do_diagnostics(int period, int step, int max_step, double time, double max_time) {
    return period > 0 && (time == max_time || step == max_step || step % period == 0);
}

namespace detail {
inline bool query_alt_str(const InputStore& in, const std::string& name, const std::string& alt,
                          const std::string& key, std::string& v) {
    return in.query_str(name + "." + key, v) || in.query_str(alt + "." + key, v);
}
template <class T>
inline bool query_alt(const InputStore& in, const std::string& name, const std::string& alt,
                      const std::string& key, T& v) {
    return in.query(name + "." + key, v) || in.query(alt + "." + key, v);
}
template <class T, size_t N>
inline bool query_alt_arr(const InputStore& in, const std::string& name, const std::string& alt,
                          const std::string& key, T (&v)[N]) {
    return in.query_arr(name + "." + key, v) || in.query_arr(alt + "." + key, v);
}
inline void reject(const InputStore& in, const std::string& key, const std::string& why) {
    if (in.contains(key)) throw InputError("input '" + key + "' is not supported: " + why);
}
// a species key that the reference also reads under the shared prefix (queryWithParserAlt):
// <species>.key and <alt>.key are both rejected
inline void reject_alt(const InputStore& in, const std::string& name, const std::string& alt,
                       const std::string& key, const std::string& why) {
    reject(in, name + "." + key, why);
    reject(in, alt + "." + key, why);
}
}  // namespace detail

inline SimConfig build_config(const InputStore& in) {
    using namespace detail;
    SimConfig c;
    int nu = 0;
    in.query("hipace.normalized_units", nu);
    c.normalized_units = nu != 0;
    c.pc = c.normalized_units ? constants_normalized() : constants_SI();

    int max_level = 0;
    in.query("amr.max_level", max_level);
    if (max_level != 0) throw InputError("amr.max_level > 0 (mesh refinement) is not supported");
    in.get_arr("amr.n_cell", c.n_cell);
    in.get_arr("geometry.prob_lo", c.prob_lo);
    in.get_arr("geometry.prob_hi", c.prob_hi);
    for (int d = 0; d < 3; ++d) {
        if (c.n_cell[d] <= 0) throw InputError("amr.n_cell must be positive");
        if (!(c.prob_hi[d] > c.prob_lo[d])) throw InputError("geometry.prob_hi must exceed prob_lo");
        c.dx[d] = (c.prob_hi[d] - c.prob_lo[d]) / c.n_cell[d];
    }
    if (c.n_cell[0] % 2 != c.n_cell[1] % 2)
        throw InputError("amr.n_cell in x and y must both be even or both be odd (multigrid)");

    std::string fb;
    if (!in.query_str("boundary.field", fb)) throw InputError("missing required input 'boundary.field'");
    if (fb != "Dirichlet")
        throw InputError("boundary.field = " + fb + " is not supported (only Dirichlet)");
    std::string pb;
    if (!in.query_str("boundary.particle", pb)) throw InputError("missing required input 'boundary.particle'");
    if (pb == "Reflecting") c.particle_bc = ParticleBC::Reflecting;
    else if (pb == "Periodic") c.particle_bc = ParticleBC::Periodic;
    else if (pb == "Absorbing") c.particle_bc = ParticleBC::Absorbing;
    else throw InputError("Unknown particle boundary '" + pb + "'");
    c.particle_lo[0] = c.prob_lo[0]; c.particle_lo[1] = c.prob_lo[1];
    c.particle_hi[0] = c.prob_hi[0]; c.particle_hi[1] = c.prob_hi[1];
    in.query_arr("boundary.particle_lo", c.particle_lo);
    in.query_arr("boundary.particle_hi", c.particle_hi);
    if (c.particle_lo[0] < c.prob_lo[0] || c.particle_lo[1] < c.prob_lo[1] ||
        c.particle_hi[0] > c.prob_hi[0] || c.particle_hi[1] > c.prob_hi[1])
        throw InputError("Particle boundary must be contained within the simulation domain");

    in.query("max_step", c.max_step);
    in.query("fields.insitu_period", c.fields_insitu_period);
    {
        std::string dt;
        if (in.query_str("diagnostic.diag_type", dt)) {
            if (dt == "xyz") c.diag_type = 0;
            else if (dt == "xz") c.diag_type = 1;
            else if (dt == "yz") c.diag_type = 2;
            else throw InputError("Unknown diagnostics type: must be xyz, xz or yz.");
        }
    }
    std::string dts;
    if (in.query_str("hipace.dt", dts)) {
        if (dts == "adaptive") throw InputError("hipace.dt = adaptive is not supported");
        in.query("hipace.dt", c.dt);
    }
    if (in.query("hipace.max_time", c.max_time)) {
        c.max_time = std::copysign(c.max_time, c.dt);
    }
    if (in.query("random_seed", c.random_seed)) c.has_random_seed = true;

    in.query("hipace.depos_order_xy", c.depos_order_xy);
    if (c.depos_order_xy < 0 || c.depos_order_xy > 3)
        throw InputError("hipace.depos_order_xy = " + std::to_string(c.depos_order_xy) +
                         " is not supported (0, 1, 2 or 3)");
    int dz_order = 0;
    in.query("hipace.depos_order_z", dz_order);
    if (dz_order != 0) throw InputError("hipace.depos_order_z must be 0");
    in.query("hipace.depos_derivative_type", c.depos_derivative_type);
    if (c.depos_derivative_type < 0 || c.depos_derivative_type > 2)
        throw InputError("hipace.depos_derivative_type must be 0, 1 or 2");

    std::string solver = "explicit";
    in.query_str("hipace.bxby_solver", solver);
    if (solver != "explicit" && solver != "predictor-corrector")
        throw InputError("hipace.bxby_solver must be explicit or predictor-corrector");
    c.explicit_solver = solver == "explicit";
    in.query("hipace.MG_tolerance_rel", c.mg_tol_rel);
    in.query("hipace.MG_tolerance_abs", c.mg_tol_abs);
    in.query("hipace.predcorr_B_error_tolerance", c.predcorr_B_error_tolerance);
    in.query("hipace.predcorr_max_iterations", c.predcorr_max_iterations);
    in.query("hipace.predcorr_B_mixing_factor", c.predcorr_B_mixing_factor);
    in.query_bool("hipace.do_beam_jx_jy_deposition", c.do_beam_jx_jy_deposition);
    in.query_bool("hipace.do_beam_jz_minus_rho", c.do_beam_jz_minus_rho);
    // diagnostics that name rho switch on its deposition (Diagnostic::needsRho)
    for (auto& s : in.query_strs("diagnostic.field_data")) if (s == "rho") c.deposit_rho = true;
    in.query_bool("hipace.deposit_rho", c.deposit_rho);

    std::string ps = "FFTDirichletFast";
    in.query_str("fields.poisson_solver", ps);
    if (ps != "FFTDirichletFast" && ps != "FFTDirichletDirect" && ps != "FFTDirichletExpanded")
        throw InputError("fields.poisson_solver = " + ps + " is not supported (Dirichlet FFT solvers only)");

    reject(in, "lasers.names", "laser envelope solver is outside the slice loop");
    reject(in, "hipace.collisions", "collisions are outside the slice loop");
    reject(in, "hipace.use_amrex_mlmg", "the AMReX MLMG path is not part of this build");
    {
        bool individual = false;
        if (in.query_bool("hipace.deposit_rho_individual", individual) && individual)
            throw InputError("input 'hipace.deposit_rho_individual' is not supported: per-species rho diagnostics are not implemented");
    }
    reject(in, "fields.do_symmetrize", "field symmetrization is not implemented");
    bool bb = false;
    if (in.query_bool("hipace.interpolate_neutralizing_background", bb) && bb)
        throw InputError("hipace.interpolate_neutralizing_background needs mesh refinement");

    const PhysConst& pc = c.pc;
    // ---------------- plasmas
    std::vector<std::string> pnames = in.query_strs("plasmas.names");
    if (!pnames.empty() && pnames[0] == "no_plasma") pnames.clear();
    for (auto& name : pnames) {
        PlasmaSpecies p;
        p.name = name;
        std::string element;
        in.query_str(name + ".element", element);
        double mass_Da = 0;
        if (element == "electron") { p.charge = -pc.q_e; p.mass = pc.m_e; }
        else if (element == "positron") { p.charge = pc.q_e; p.mass = pc.m_e; }
        else if (element == "proton") { p.charge = pc.q_e; p.mass = pc.m_p; }
        else if (!element.empty())
            throw InputError(name + ".element = " + element + " is not supported (electron, positron, proton)");
        if (in.query(name + ".mass_Da", mass_Da) && mass_Da != 0) p.mass = pc.m_p * mass_Da / 1.007276466621;
        in.query(name + ".mass", p.mass);
        if (p.mass == 0) throw InputError("The plasma particle mass must be specified");
        in.query(name + ".charge", p.charge);
        if (p.charge == 0) throw InputError("The plasma particle charge must be specified");
        reject(in, name + ".can_ionize", "ionization is outside the slice loop");
        reject(in, name + ".ionization_product", "ionization is outside the slice loop");
        reject_alt(in, name, "plasmas", "fine_ppc", "fine plasma patches need mesh refinement");
        reject_alt(in, name, "plasmas", "fine_patch(x,y)", "fine plasma patches need mesh refinement");
        reject_alt(in, name, "plasmas", "fine_transition_cells", "fine plasma patches need mesh refinement");
        reject_alt(in, name, "plasmas", "do_symmetrize", "symmetrized plasma loading is not implemented");
        {
            int period = 0;
            if (query_alt(in, name, "plasmas", "insitu_period", period) && period != 0)
                throw InputError("input '" + name + ".insitu_period' is not supported: plasma in-situ diagnostics are not implemented");
        }
        reject(in, name + ".density_table_file", "density tables are not implemented");

        int ion_lev = -1;
        if (in.query(name + ".initial_ion_level", ion_lev)) p.charge *= ion_lev;
        query_alt(in, name, "plasmas", "n_subcycles", p.n_subcycles);
        if (p.n_subcycles < 1) throw InputError("n_subcycles must be larger or equal to 1");
        query_alt(in, name, "plasmas", "neutralize_background", p.neutralize_background);
        std::string dens = "0.";
        query_alt_str(in, name, "plasmas", "density(x,y,z)", dens);
        p.density = in.function(dens, {"x", "y", "z"});
        query_alt(in, name, "plasmas", "min_density", p.min_density);
        query_alt(in, name, "plasmas", "radius", p.radius);
        query_alt(in, name, "plasmas", "hollow_core_radius", p.hollow_core_radius);
        if (!(p.hollow_core_radius < p.radius))
            throw InputError("The hollow core plasma radius must be smaller than the plasma radius");
        query_alt(in, name, "plasmas", "max_qsa_weighting_factor", p.max_qsa_weighting_factor);
        if (!query_alt_arr(in, name, "plasmas", "ppc", p.ppc))
            throw InputError("missing required input '" + name + ".ppc'");
        in.query_arr(name + ".u_mean", p.u_mean);
        const bool has_u_std = in.query_arr(name + ".u_std", p.u_std);
        double temperature_ev = 0;
        const bool has_t = in.query(name + ".temperature_in_ev", temperature_ev);
        if (has_u_std && has_t)
            throw InputError("Please specify exlusively either a temperature or the thermal momentum");
        if (has_t) {
            // PlasmaParticleContainer.cpp:135-144: u_std = sqrt(T e / (m c^2)) in SI
            const double q_e_si = 1.602176634e-19, m_e_si = 9.1093837015e-31, c_si = 299792458.0;
            const double m_si = p.mass * (m_e_si / pc.m_e);
            for (int d = 0; d < 3; ++d) p.u_std[d] = std::sqrt(temperature_ev * q_e_si / (m_si * c_si * c_si));
        }
        p.thermal = p.u_std[0] != 0 || p.u_std[1] != 0 || p.u_std[2] != 0;
        query_alt(in, name, "plasmas", "prevent_centered_particle", p.prevent_centered_particle);
        query_alt(in, name, "plasmas", "reorder_period", p.reorder_period);
        if (p.reorder_period < 0) throw InputError(name + ".reorder_period must be >= 0");
        p.reorder_idx_type[0] = p.reorder_idx_type[1] = c.depos_order_xy % 2;
        query_alt_arr(in, name, "plasmas", "reorder_idx_type", p.reorder_idx_type);
        for (int d = 0; d < 2; ++d)
            if (p.reorder_idx_type[d] != 0 && p.reorder_idx_type[d] != 1)
                throw InputError(name + ".reorder_idx_type must be 0 (cells) or 1 (nodes) per axis");
        c.plasmas.push_back(p);
    }
    // ---------------- beams
    std::vector<std::string> bnames = in.query_strs("beams.names");
    if (!bnames.empty() && bnames[0] == "no_beam") bnames.clear();
    for (auto& name : bnames) {
        BeamSpecies b;
        b.name = name;
        std::string element = "electron";
        in.query_str(name + ".element", element);
        if (element == "electron") { b.charge = -pc.q_e; b.mass = pc.m_e; }
        else if (element == "proton") { b.charge = pc.q_e; b.mass = pc.m_p; }
        else if (element == "positron") { b.charge = pc.q_e; b.mass = pc.m_e; }
        in.query(name + ".charge", b.charge);
        in.query(name + ".mass", b.mass);
        if (b.mass == 0) throw InputError("The beam particle mass must not be 0");
        std::string inj;
        if (!in.query_str(name + ".injection_type", inj))
            throw InputError("missing required input '" + name + ".injection_type'");
        in.query(name + ".n_subcycles", b.n_subcycles);
        if (b.n_subcycles < 1) throw InputError("n_subcycles must be >= 1");
        in.query_bool(name + ".do_z_push", b.do_z_push);
        in.query(name + ".duz_per_uz0_dzeta", b.duz_per_uz0_dzeta);
        query_alt(in, name, "beams", "insitu_period", b.insitu_period);
        query_alt(in, name, "beams", "insitu_radius", b.insitu_radius);
        in.query_bool(name + ".do_salame", b.do_salame);
        reject_alt(in, name, "beams", "do_spin_tracking", "spin tracking is outside the slice loop");
        reject_alt(in, name, "beams", "do_radiation_reaction", "radiation reaction is outside the slice loop");
        for (int f = 0; f < 2; ++f) {
            const std::string key = f == 0 ? "external_E(x,y,z,t)" : "external_B(x,y,z,t)";
            std::vector<std::string> e = in.query_strs(name + "." + key);
            if (e.empty()) e = in.query_strs("beams." + key);
            if (!e.empty() && e.size() != 3) throw InputError(name + "." + key + " expects 3 expressions");
            for (int d = 0; d < 3; ++d)
                b.external[3 * f + d] = in.function(e.empty() ? std::string("0") : e[d], {"x", "y", "z", "t"});
            if (!e.empty()) b.use_external = true;
        }
        if (inj != "fixed_weight_pdf") {
            in.query_arr(name + ".u_mean", b.u_mean);
            in.query_arr(name + ".u_std", b.u_std);
        }
        std::string profile;
        if (inj == "fixed_weight_pdf") {
            // BeamParticleContainer.cpp:200-249: every profile quantity is a function of z
            b.injection = BeamInjection::FixedWeightPDF;
            std::string pdf;
            if (!in.query_str(name + ".pdf", pdf)) throw InputError("missing required input '" + name + ".pdf'");
            b.pdf = in.function(pdf, {"z"});
            auto funcs = [&](const std::string& key, Expr* out, size_t n) {
                const std::vector<std::string> v = in.query_strs(name + "." + key);
                if (v.size() != n)
                    throw InputError("input '" + name + "." + key + "' expects " + std::to_string(n) + " values");
                for (size_t i = 0; i < n; ++i) out[i] = in.function(v[i], {"z"});
            };
            Expr pm[2], ps[2], um[3], us[3];
            funcs("position_mean", pm, 2);
            funcs("position_std", ps, 2);
            funcs("u_mean", um, 3);
            funcs("u_std", us, 3);
            b.pdf_pos[0] = pm[0]; b.pdf_pos[1] = pm[1]; b.pdf_pos[2] = ps[0]; b.pdf_pos[3] = ps[1];
            for (int i = 0; i < 3; ++i) { b.pdf_u[i] = um[i]; b.pdf_u[i + 3] = us[i]; }
            in.get(name + ".num_particles", b.num_particles);
            in.query(name + ".radius", b.radius);
            in.query(name + ".z_foc", b.z_foc);
            in.query_bool(name + ".do_symmetrize", b.do_symmetrize);
            in.query(name + ".pdf_ref_ratio", b.pdf_ref_ratio);
            if (b.pdf_ref_ratio < 1) throw InputError(name + ".pdf_ref_ratio must be >= 1");
            if (b.do_symmetrize && b.num_particles % 4 != 0)
                throw InputError("To symmetrize the beam, please specify a beam particle number divisible by 4.");
            const bool has_q = in.query(name + ".total_charge", b.total_charge);
            const bool has_n = in.query(name + ".density", b.density);
            if (has_q && c.normalized_units)
                throw InputError("The option 'beam.total_charge' is only valid in SI units.");
            if ((int)has_q + (int)has_n != 1)
                throw InputError("Please specify exlusively either total_charge or density of the beam");
            b.peak_density_specified = has_n;
            b.density = std::fabs(b.density);
            b.total_charge = std::fabs(b.total_charge);
        } else if (inj == "fixed_ppc") {
            b.injection = BeamInjection::FixedPPC;
            in.query_arr(name + ".ppc", b.ppc);
            in.get(name + ".zmin", b.zmin);
            in.get(name + ".zmax", b.zmax);
            in.get(name + ".radius", b.radius);
            in.query_arr(name + ".position_mean", b.position_mean);
            in.query(name + ".min_density", b.min_density);
            b.min_density = std::fabs(b.min_density);
            int rnd[3] = {0, 0, 0};
            if (in.query_arr(name + ".random_ppc", rnd) && (rnd[0] || rnd[1] || rnd[2]))
                throw InputError(name + ".random_ppc is not supported");
            if (!in.query_str(name + ".profile", profile))
                throw InputError("missing required input '" + name + ".profile'");
            if (profile == "gaussian") {
                b.profile = BeamProfile::Gaussian;
                in.get(name + ".density", b.density);
                in.query_arr(name + ".position_std", b.position_std);
            } else if (profile == "flattop") {
                b.profile = BeamProfile::Flattop;
                in.get(name + ".density", b.density);
            } else {
                throw InputError(name + ".profile = " + profile + " is not supported for fixed_ppc");
            }
            b.density = std::fabs(b.density);
            if (b.duz_per_uz0_dzeta != 0.)
                throw InputError("Tilted beams and correlated energy spreads are only implemented for fixed weight beams");
        } else if (inj == "fixed_weight") {
            b.injection = BeamInjection::FixedWeight;
            profile = "gaussian";
            in.query_str(name + ".profile", profile);
            in.query(name + ".radius", b.radius);
            if (profile == "can") {
                b.profile = BeamProfile::Can;
                in.get(name + ".zmin", b.zmin);
                in.get(name + ".zmax", b.zmax);
            } else if (profile == "gaussian") {
                b.profile = BeamProfile::Gaussian;
                in.query(name + ".zmin", b.zmin);
                in.query(name + ".zmax", b.zmax);
                if (b.do_salame && (b.zmin <= -1e300 || b.zmax >= 1e300))
                    throw InputError("For the SALAME algorithm it is mandatory to either use a 'can' profile or "
                                     "'zmin' and 'zmax' with a gaussian profile");
            } else {
                throw InputError("Only gaussian and can are supported with fixed_weight beam injection");
            }
            std::vector<std::string> pm = in.query_strs(name + ".position_mean");
            if (pm.size() != 3) throw InputError(name + ".position_mean expects 3 values");
            for (int d = 0; d < 3; ++d) {
                Expr e = in.function(pm[d], {"z"});
                if (!e.is_constant())
                    throw InputError(name + ".position_mean depending on z is not supported");
                b.position_mean[d] = e.eval(nullptr);
            }
            in.get_arr(name + ".position_std", b.position_std);
            in.get(name + ".num_particles", b.num_particles);
            in.query(name + ".z_foc", b.z_foc);
            bool has_q = in.query(name + ".total_charge", b.total_charge);
            bool has_n = in.query(name + ".density", b.density);
            if (has_q && c.normalized_units)
                throw InputError("The option 'beam.total_charge' is only valid in SI units.");
            if ((int)has_q + (int)has_n != 1)
                throw InputError("Please specify exlusively either total_charge or density of the beam");
            in.query_bool(name + ".do_symmetrize", b.do_symmetrize);
            if (b.do_symmetrize && b.num_particles % 4 != 0)
                throw InputError("To symmetrize the beam, please specify a beam particle number divisible by 4.");
            // total charge from the peak density (BeamParticleContainer.cpp:179-190)
            if (has_n) {
                b.total_charge = b.density * b.charge;
                for (int d = 0; d < 3; ++d) b.total_charge *= b.position_std[d] * std::sqrt(2. * 3.14159265358979323846);
            }
            if (c.normalized_units) b.total_charge *= 1.0 / (c.dx[0] * c.dx[1] * c.dx[2]);
        } else {
            throw InputError(name + ".injection_type = " + inj +
                             " is not supported (fixed_ppc, fixed_weight, fixed_weight_pdf)");
        }
        c.beams.push_back(b);
    }
    if (c.fields_insitu_period > 0 && !c.explicit_solver)
        throw InputError("Must use explicit solver for field insitu diagnostic");
    in.query("hipace.salame_n_iter", c.salame_n_iter);
    in.query_bool("hipace.salame_do_advance", c.salame_do_advance);
    {
        std::string t = "Ez_initial";
        in.query_str("hipace.salame_Ez_target(zeta,zeta_initial,Ez_initial)", t);
        c.salame_target = in.function(t, {"zeta", "zeta_initial", "Ez_initial"});
    }
    in.query("hipace.salame_relative_tolerance", c.salame_relative_tolerance);
    if (c.any_salame() && !c.explicit_solver)
        throw InputError("Cannot use SALAME algorithm with predictor-corrector solver");
    std::string witness;
    if (in.query_str("adjoint.witness", witness)) {
        AdjointConfig& a = c.adjoint;
        for (size_t b = 0; b < c.beams.size(); ++b)
            if (c.beams[b].name == witness) a.witness = (int)b;
        if (a.witness < 0) throw InputError("adjoint.witness = " + witness + " is not in beams.names");
        if (!c.explicit_solver) throw InputError("the adjoint needs the explicit Bx/By solver");
        if (c.any_salame()) throw InputError("the adjoint does not differentiate SALAME");
        if (c.depos_order_xy != 2)
            throw InputError("the adjoint is written for the quadratic shapes (hipace.depos_order_xy = 2)");
        for (auto& p : c.plasmas)
            if (p.n_subcycles != 1) throw InputError("the adjoint needs plasma n_subcycles = 1");
        double r[2];
        if (in.query_arr("adjoint.profile_zeta", r)) { a.profile_lo = r[0]; a.profile_hi = r[1]; }
        if (in.query_arr("adjoint.density_z", r)) { a.density_lo = r[0]; a.density_hi = r[1]; }
        if (in.query_arr("adjoint.objective_zeta", r)) { a.objective_lo = r[0]; a.objective_hi = r[1]; }
        in.query("adjoint.n_profile_knots", a.n_profile);
        in.query("adjoint.n_density_knots", a.n_density);
        in.query("adjoint.checkpoint_interval", a.checkpoint_interval);
        if (a.n_profile < 2 || a.n_density < 1 || a.checkpoint_interval < 1 ||
            !(a.profile_hi > a.profile_lo) || !(a.density_hi > a.density_lo) ||
            !(a.objective_hi >= a.objective_lo))
            throw InputError("invalid adjoint.* ranges or knot counts");
    }
    return c;
}

}  // namespace hpq
