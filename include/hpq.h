/*
 * hpq — C ABI of the B200 quasi-static slice loop (HiPACE++ slice solver, drop-in).
 *
 * Conventions (all entry points):
 *   - return 0 on success, a non-zero HPQ_ERR_* code otherwise; hpq_last_error() gives the text.
 *     No C++ exception crosses this boundary. The reference terminates the process through
 *     amrex::Abort on the same conditions.
 *   - the handle owns all device memory and one CUDA stream; host buffers belong to the caller.
 *   - one handle is driven by one host thread at a time (the reference: one host thread per
 *     rank driving amrex::Gpu::gpuStream()).
 * Input text uses the reference's input-file syntax and keys (hipace.*, amr.*, geometry.*,
 * boundary.*, plasmas.*, beams.*, <species>.*, my_constants.*; docs/source/run/parameters.rst).
 */
#ifndef HPQ_H_
#define HPQ_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hpq_handle hpq_handle;

enum {
    HPQ_OK = 0,
    HPQ_ERR_INPUT = 1,          /* bad or unsupported input key/value */
    HPQ_ERR_CUDA = 2,           /* CUDA runtime error */
    HPQ_ERR_STATE = 3,          /* call out of order (e.g. slice before hpq_begin_step) */
    HPQ_ERR_NOT_CONVERGED = 4,  /* multigrid hit its iteration limit (hpmg "failed") */
    HPQ_ERR_DIVERGED = 5,       /* multigrid residual grew by 1e20 (hpmg "failing") */
    HPQ_ERR_ARG = 6,            /* bad argument (index, name, null pointer, unsupported shape) */
    HPQ_ERR_TOO_LARGE = 7       /* grid larger than a fixed-size scratch area allows */
};

enum { HPQ_PLAIN_FP64 = 0, HPQ_MIXED = 1 };

/* Parse and validate an input deck; replaces Hipace::Hipace() (src/Hipace.cpp:74-244) reading
 * amrex::ParmParse. `input_text` holds the file content, later lines override earlier ones
 * (command-line overrides can be appended as extra lines). */
int hpq_create(const char* input_text, hpq_handle** out);
void hpq_destroy(hpq_handle* h);
const char* hpq_last_error(const hpq_handle* h);
/* Grid size (amr.n_cell, after my_constants and expressions are evaluated), valid after
 * hpq_create (Hipace.cpp:176-230 reads the same key). */
int hpq_n_cell(const hpq_handle* h, int n_cell[3]);
/* max_step of the input (the last step of Hipace::Evolve's loop, Hipace.cpp:401). */
int hpq_max_step(const hpq_handle* h, int* max_step);
/* Physical time at which the next step starts (0 before the first step). Steps follow the
 * reference's max_time rule (Hipace.cpp:413-435): a step that would cross hipace.max_time is
 * shortened to end on it, the step that starts on it runs with dt = 0, after which the time is
 * +infinity and hpq_begin_step / hpq_step return HPQ_ERR_STATE (the reference leaves its step
 * loop there). */
int hpq_time(hpq_handle* h, double* t);
/* Number of doubles hpq_get_diag writes per component: nz*ny*nx (diagnostic.diag_type = xyz),
 * nz*nx (xz) or nz*ny (yz). */
int hpq_diag_count(const hpq_handle* h, int64_t* n);
/* Text of the last hpq_create failure (no handle exists then). */
const char* hpq_create_error(void);

/* Field/plasma arithmetic: HPQ_PLAIN_FP64 (the reference's FP64 path) or HPQ_MIXED (FP32
 * plasma, fields and multigrid; FP64 beam). Call before hpq_init. */
int hpq_set_precision(hpq_handle* h, int mode);

/* Allocate device data and inject the beams; replaces Hipace::InitData()
 * (src/Hipace.cpp:246-295): fixed_ppc beams follow InitBeamFixedPPCSlice
 * (src/particles/beam/BeamParticleContainerInit.cpp:199-345); fixed_weight beams are drawn
 * from this library's seeded Philox stream (hpq_set_beam overrides them). */
int hpq_init(hpq_handle* h);

/* Replace all particles of beam `beam` (FP64 SoA, momenta are gamma*beta*c like the reference
 * BeamIdx::ux..uz, src/particles/beam/BeamParticleContainer.H:23-41). Particles are binned
 * into slices as BoxSorter::sortParticlesByBox (src/particles/sorting/BoxSort.cpp:14-78).
 * `id` may be NULL. */
int hpq_set_beam(hpq_handle* h, int beam, const double* x, const double* y, const double* z,
                 const double* w, const double* ux, const double* uy, const double* uz,
                 const int64_t* id, int64_t n);
/* Name of beam `beam` (beams.names order), or NULL past the last beam. */
const char* hpq_beam_name(const hpq_handle* h, int beam);
/* Number of stored particles of a beam and a copy of them (slices from head to tail). Invalid
 * particles (absorbed at a boundary, removed by SALAME) are reported with weight 0; hpq_set_beam
 * treats weight-0 particles as invalid, so the two round-trip. */
int hpq_beam_count(hpq_handle* h, int beam, int64_t* n);
int hpq_get_beam(hpq_handle* h, int beam, double* x, double* y, double* z, double* w,
                 double* ux, double* uy, double* uz, int64_t* id);

/* Time-step pipeline across processes (one GPU each): rank r runs steps r, r+N, ... and hands
 * each finished beam slice to rank r+1, which replaces the reference's MultiBuffer transfers
 * (src/utils/MultiBuffer.cpp:181-430, put_data/get_data around SolveOneSlice,
 * src/Hipace.cpp:581-583, 700-705). The transport is the caller's (hipace2_b200/pipeline.py).
 * hpq_beam_slice_count / hpq_get_beam_slice: the particles that slice `islice` of the current
 *   (or last) step hands to the next step, after the slice's beam push and slip bookkeeping;
 *   final once slice islice - 1 has been solved (hpq_solve_slice), or after hpq_end_step for
 *   slice 0.
 * hpq_put_beam_slice: inside a step, the particles of slice `islice` of this step received
 *   from the rank that ran the previous step (the step's own beam is replaced). Slices are put
 *   from the head (nz-1) down, nz-1 first, and slice islice must be put before
 *   hpq_solve_slice(islice + 1) (its jx/jy beam deposit reads it). Weight-0 particles are
 *   invalid. HPQ_ERR_INPUT if the particles exceed the beam's store.
 * hpq_set_time: physical time at which the next step starts (each rank runs every N-th step). */
int hpq_beam_slice_count(hpq_handle* h, int beam, int islice, int64_t* n);
int hpq_get_beam_slice(hpq_handle* h, int beam, int islice, double* x, double* y, double* z, double* w,
                       double* ux, double* uy, double* uz, int64_t* id);
int hpq_put_beam_slice(hpq_handle* h, int beam, int islice, const double* x, const double* y,
                       const double* z, const double* w, const double* ux, const double* uy,
                       const double* uz, const int64_t* id, int64_t n);
int hpq_set_time(hpq_handle* h, double t);

/* One full time step (all slices, head to tail); replaces the body of the step loop of
 * Hipace::Evolve (src/Hipace.cpp:401-492). */
int hpq_step(hpq_handle* h, int step);
/* The per-slice surface: begin a step (ResetAllQuantities, plasma re-initialisation,
 * neutralising background; src/Hipace.cpp:403-472), solve one slice — replaces
 * Hipace::SolveOneSlice(islice, step) (src/Hipace.H:119, src/Hipace.cpp:556-728); slices must
 * be solved from nz-1 down to 0 — then end the step. */
int hpq_begin_step(hpq_handle* h, int step);
int hpq_solve_slice(hpq_handle* h, int islice);
int hpq_end_step(hpq_handle* h);

/* Interior (ny x nx, x fastest) of a slice field component of the current slice, by the
 * reference component name (Fields::getField, src/fields/Fields.H:436; names of
 * src/fields/Fields.cpp:76-148, e.g. "Ez", "Psi", "Bx", "jz_beam", "chi"). */
int hpq_get_field(hpq_handle* h, const char* comp, double* out);

/* 3-D field diagnostic: record the listed components (space separated) of every slice of the
 * following steps into nz x ny x nx arrays (replaces Fields::Copy into the openPMD diagnostic,
 * src/fields/Fields.cpp:413-533, for diag_type=xyz without coarsening). */
int hpq_set_diag(hpq_handle* h, const char* comps);
int hpq_get_diag(hpq_handle* h, const char* comp, double* out);

/* In-situ reduced diagnostics of the last diagnostic step (keys <beam>.insitu_period,
 * <beam>.insitu_radius, beams.insitu_*, fields.insitu_period). Replaces the per-slice reductions
 * BeamParticleContainer::InSituComputeDiags (BeamParticleContainer.cpp:476-548) and
 * Fields::InSituComputeDiags (Fields.cpp:1289-1346) with the arrays their InSituWriteToFile
 * writes. `what` is a beam name or "fields". Layout, value index outer and slice inner:
 *   beam (23 nz + 23 doubles): 22 x nz per-slice values ([0] sum of weights, [1..21] the
 *     weighted means [x], [x^2], [y], [y^2], [z], [z^2], [ux], [ux^2], [uy], [uy^2], [uz],
 *     [uz^2], [x*ux], [y*uy], [z*uz], [x*uy], [y*ux], [ux/uz], [uy/uz], [ga], [ga^2]), nz particle
 *     counts, then the 22 raw sums and the particle count over all slices;
 *   fields (11 nz doubles): 10 x nz per-slice sums times dx dy dz ([Ex^2], [Ey^2], [Ez^2],
 *     [Bx^2], [By^2], [Bz^2], [ExmBy^2], [EypBx^2], [jz_beam], [Ez*jz_beam]), then the 10 sums. */
int hpq_insitu_size(hpq_handle* h, const char* what, int64_t* n);
int hpq_get_insitu(hpq_handle* h, const char* what, double* out);

/* Plasma species `sp`: particle count and the 11 real attributes of PlasmaIdx
 * (src/particles/plasma/PlasmaParticleContainer.H:21-46) plus the valid flag, as 12 blocks of
 * `n` doubles: x y w ux uy psi x_prev y_prev ux_half_step uy_half_step psi_half_step valid. */
int hpq_plasma_count(hpq_handle* h, int sp, int64_t* n);
int hpq_get_plasma(hpq_handle* h, int sp, double* out);

/* Capture each slice in a CUDA graph (default on) or launch kernel by kernel. */
int hpq_set_graphs(hpq_handle* h, int on);
/* Deterministic deposition (default off): current and charge deposits are accumulated with
 * order-independent fixed-point integer atomics and every reduction runs in a fixed order, so
 * two runs on the same inputs give bit-identical fields, beams and plasma. The reference deposits
 * with floating-point atomics (PlasmaDepositCurrent.cpp:164-247, BeamDepositCurrent.cpp:130-190)
 * and has no such mode; the values agree with the default mode to FP64 rounding. Allowed between
 * steps. */
int hpq_set_deterministic(hpq_handle* h, int on);
/* Adjoint of one step (the reference has no adjoint). In plain FP64 everything runs in double;
 * with HPQ_MIXED the forward and its segment recomputations run in single precision and record
 * their state widened to double, and the reverse sweep is FP64. Configured with the
 * adjoint.* input keys: the objective is the current-weighted variance of Ez over the slices
 * whose centre lies in adjoint.objective_zeta,
 *   J = S2/S0 - (S1/S0)^2,  S_n = sum over those slices and cells of jz_beam * Ez^n,
 * and the parameters are n_profile + n_density knot values:
 *   knots[0, n_profile): the witness beam (adjoint.witness) current profile, piecewise linear on
 *     n_profile equidistant points of adjoint.profile_zeta, multiplying the witness weights
 *     given by hpq_set_beam or the injection (zero outside the range);
 *   knots[n_profile, n_profile + n_density): the plasma density multiplier, piecewise linear on
 *     adjoint.density_z, evaluated at z = c t of the step (end values held outside).
 * hpq_adjoint_grad runs the forward of the next step (without advancing time or the beam; the
 * witness weights of the store are left multiplied by the profile) and, if grad is not NULL, the
 * reverse sweep with checkpoints every adjoint.checkpoint_interval slices, writing dJ/dknots.
 * The forward map replaces, for the gradient, the step of Hipace::Evolve (Hipace.cpp:393-554) and
 * the slice loop of Hipace::SolveOneSlice (Hipace.cpp:556-728). Explicit solver, one plasma
 * species with n_subcycles 1. */
int hpq_adjoint_nparams(hpq_handle* h, int* n);
int hpq_adjoint_grad(hpq_handle* h, const double* knots, double* grad, double* objective);
/* SALAME (<beam>.do_salame, hipace.salame_*; src/salame/Salame.cpp): in step 0 the weights of
 * the SALAME beams are rescaled slice by slice so that the current-weighted Ez of the next slice
 * follows hipace.salame_Ez_target(zeta,zeta_initial,Ez_initial). The reference prints the weight
 * factor W of every iteration (Salame.cpp:146-157); here they are kept as (slice, iteration, W)
 * triples: *n receives the number of doubles (3 per iteration) and `out`, if not NULL, the
 * values. */
int hpq_salame_log(hpq_handle* h, double* out, int64_t* n);
/* Wait for all work of the handle. */
int hpq_synchronize(hpq_handle* h);
/* Per-kernel-class timing with CUDA events on the launching stream (kernel launch mode only).
 * Classes: plasma_deposit, beam_deposit, poisson_psi_ez_bz, explicit_deposit, multigrid,
 * plasma_push, beam_push, beam_partition. hpq_get_profile returns the accumulated device time
 * and number of timed regions since profiling was switched on. */
int hpq_set_profiling(hpq_handle* h, int on);
int hpq_get_profile(hpq_handle* h, const char* kernel_class, double* total_ms, int64_t* launches);
/* The handle's CUDA stream (cudaStream_t), for timing with events on the launching stream. */
void* hpq_stream(hpq_handle* h);
/* Counters since hpq_init, updated at the end of each step: multigrid V-cycles, slices solved,
 * plasma particle pushes (the reference's performance counters, src/Hipace.H:275-282) and
 * kernels launched by this library (graph replays included). Any pointer may be NULL. */
int hpq_get_counters(hpq_handle* h, int64_t* mg_vcycles, int64_t* slices, int64_t* plasma_pushes,
                     int64_t* kernel_launches);

/* Allocation-free Dirichlet Poisson solve, Lap(u) = f on an nx x ny grid (x fastest) with
 * cell sizes dx, dy and u = 0 one cell outside the grid, by DST-I; the same solve as the slice
 * loop's Psi/Ez/Bz solves. No counterpart in the reference: it exists for callers that cannot
 * allocate device memory when they solve — code running under CUDA stream capture, plugins whose
 * host framework owns the memory pool, real-time loops that must not allocate. f and u are
 * device pointers owned by the caller (u may not alias f); `stream` is a cudaStream_t (NULL =
 * default stream). Nothing is allocated: the temporaries live in a 16.1 MiB device array inside
 * the library. CUDA loads the library's device code lazily, so the first call on each device
 * commits that array's memory there (and may fail with HPQ_ERR_CUDA if the device is full); it is
 * held until the process exits. Limit: nx, ny of the form 2^k - 1 with 31 <= n <= 1023; larger
 * grids return HPQ_ERR_TOO_LARGE, other shapes HPQ_ERR_ARG. The first call on a device also
 * looks up the device address of that array and sets the kernels' shared-memory limits (once per
 * device, with the device current), so make the first call on each device before any stream
 * capture. All calls share the array: calls whose kernels overlap on the GPU race and give wrong
 * results; serialise them (one stream, or events). A CUDA error already pending when the call
 * starts is not touched: the call returns HPQ_ERR_CUDA without launching anything; each of its
 * own launches is checked as it is made. */
int hpq_poisson_dirichlet_noalloc(const double* f, double* u, int nx, int ny, double dx, double dy,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HPQ_H_ */
