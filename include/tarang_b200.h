/*
 * tarang_b200 — C ABI of the B200 pseudo-spectral IF-RK4 hot path.
 *
 * Drop-in replacement for the nonlinear-term + RK4 step of the Tarang-2
 * reference (anandogc/tarang, paths below are inside its trunk/lib/).  The
 * reference binds these through its C++ seams: the abstract basis `Universal`
 * (basis/basicfn/universal.h:48-), the static `Nlin_incompress` functions
 * (fluid/incompressible/nlin/Nlin.h:69-101) and `Time_advance_incompress`
 * (fluid/incompressible/time_advance/Time_advance.h:69-187).
 *
 * Conventions
 *  - Every function returns a ts_status and never aborts (the reference prints
 *    and calls exit/MPI_Abort, e.g. basis/FFF/pencil/FFF_pencil.cc:84-87).
 *  - Spectral fields use the reference layout: complex (Nx, Ny, Nz/2+1), C
 *    order, kx and ky in FFT order (FFF_pencil_inline.h:63-111); a vector field
 *    is its three components V1, V2, V3 stored back to back.  Complex = two
 *    reals (re, im) of the plan's precision (double for TS_F64, float for TS_F32).
 *  - Real fields use the reference's padded layout (Nx, Ny, Nz+2)
 *    (FFF_pencil.cc:212); the two pad values per line are ignored on input and
 *    written as 0 on output.
 *  - Normalisation (inferred from the reference's energy functions): forward
 *    transforms divide by Nx*Ny*Nz (FFF) or by 2Nx*Ny*Nz (SFF); inverses are
 *    unnormalised.
 *  - Field pointers may be device pointers or host pointers; host pointers are
 *    staged through plan-owned device buffers (copies inside the call).
 *  - A plan is used by one host thread at a time; distinct plans are independent.
 */
#ifndef TARANG_B200_H
#define TARANG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TS_OK = 0,
  TS_ERR_ARG = 1,         /* invalid argument / unsupported size */
  TS_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  TS_ERR_NAN = 3,         /* a NaN / Inf was detected in the state */
  TS_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
  TS_ERR_UNSUPPORTED = 5, /* valid but not implemented for this basis / precision */
  TS_ERR_NOMEM = 6        /* device allocation failed */
} ts_status;

/* TS_BASIS_SSF (sin/cos along x and y, Fourier along z; basis/SSF/pencil) offers the
 * transforms (ts_fft_forward / ts_fft_inverse with parities "SCF", "CSF", "SSF", "CCF"),
 * ts_rk4_step for the conservative, unforced fluid (sincostr_switch "SCF":
 * Vx = SCF, Vy = CSF, Vz = CCF), ts_rk4_step_rbc, ts_energy, ts_nusselt, ts_max_div,
 * ts_shell_spectrum and ts_flux; the other calls on an SSF plan return
 * TS_ERR_UNSUPPORTED. */
/* TS_BASIS_SSS (sin/cos along every axis; basis/SSS/pencil) stores real coefficients in
 * the padded real layout (Nx, Ny, Nz + 2) of each component (the complex buffer viewed
 * as reals, as SSS_PENCIL does) and offers the transforms (parities [SC][SC][SC]) and
 * ts_rk4_step for the conservative, unforced fluid (sincostr_switch "SCC": Vx = SCC,
 * Vy = CSC, Vz = CCS), ts_rk4_step_rbc, ts_energy, ts_nusselt, ts_max_div,
 * ts_shell_spectrum, ts_flux and ts_dealias_field. */
typedef enum { TS_BASIS_FFF = 0, TS_BASIS_SFF = 1, TS_BASIS_SSF = 2, TS_BASIS_SSS = 3 } ts_basis;
typedef enum { TS_F64 = 0, TS_F32 = 1 } ts_precision;
typedef enum { TS_NLIN_CONSERVATIVE = 0, TS_NLIN_ROTATIONAL = 1 } ts_nlin_form;
typedef enum { TS_DEALIAS_NONE = 0, TS_DEALIAS_REFERENCE_CORNER = 1, TS_DEALIAS_TWO_THIRDS = 2 } ts_dealias;
typedef enum { TS_FORCE_NONE = 0, TS_FORCE_CARATI_ENERGY_SUPPLY = 1, TS_FORCE_RBC = 51 } ts_force;
/* PHYSICS.Pr_option and PHYSICS.Uscaling of an RBC run (Global_read.cc; the
 * coefficients of compute_force_RBC.cc:104-150 and Correlation.cc:144-176).  PRZERO and
 * PRINFTY slave one field to the other (Single_time_step_RBC, Tadvance_functions.cc:
 * 380-395): under PRZERO only U is advanced and T = U.V1 / K^2 after every stage; under
 * PRINFTY only T is advanced and U = vs P(T x) / K^2 (FluidVF.cc:228-272).  They step on
 * SFF plans (ts_rk4_step_rbc); SSF / SSS plans and ensembles refuse them with
 * TS_ERR_UNSUPPORTED. */
typedef enum { TS_PR_LARGE = 0, TS_PR_SMALL = 1, TS_PR_ZERO = 2, TS_PR_INFTY = 3 } ts_pr_option;
typedef enum { TS_U_LARGE = 0, TS_U_SMALL = 1 } ts_uscaling;

/* Solver configuration.  Field names follow the reference's para.yaml keys
 * where one exists (global/Global.h:65-259). */
typedef struct {
  int basis;            /* ts_basis (program.basis_type) */
  int N[3];             /* field.N, powers of two 16..1024 */
  double kfactor[3];    /* field.kfactor (reference kfactor[1..3]) */
  int precision;        /* ts_precision (build option -DREAL) */
  int nlin_form;        /* ts_nlin_form */
  int dealias_mode;     /* ts_dealias (program.alias_option) */
  int reality_fix;      /* program.apply_strong_realitycond_alltime_switch */
  double nu;            /* field.diss_coefficients[0] (velocity) */
  double kappa;         /* field.diss_coefficients[1] (scalar) */
  double dt;            /* time.dt_fixed */
  int force_type;       /* ts_force (force.field_procedure) */
  double force_inner_radius, force_outer_radius; /* Carati band (force.parameters) */
  const double* energy_supply;   /* per shell ceil|K| (in/forcing.txt), copied at create */
  const double* helicity_supply; /* may be NULL */
  int n_supply;
  double Ra, Pr;        /* PHYSICS.Rayleigh, PHYSICS.Prandtl (RBC) */
  int Pr_option;        /* ts_pr_option (RBC; default PRLARGE) */
  int Uscaling;         /* ts_uscaling (RBC; default ULARGE) */
} ts_config;

typedef struct ts_plan ts_plan;

/* Fill *cfg with defaults: FFF, N = 64^3, kfactor 1, F64, conservative,
 * reference-corner dealias, reality fix on, nu = 0.01, dt = 1e-3, no force. */
void ts_config_default(ts_config* cfg);

/* Replaces the FFF_PENCIL / SFF_PENCIL constructor + fftk.Init
 * (FFF_pencil.cc:31-135, SFF_pencil.cc:38-): allocates twiddles and workspace. */
int ts_plan_create(const ts_config* cfg, ts_plan** plan);
int ts_plan_destroy(ts_plan* plan);
/* Stream for every later call (cudaStream_t; NULL = legacy default stream). */
int ts_plan_set_stream(ts_plan* plan, void* stream);
/* Complex elements per component (Nx*Ny*(Nz/2+1)) and bytes per complex. */
int ts_plan_sizes(const ts_plan* plan, long long* elems_per_comp, int* bytes_per_complex);
/* Number of shells of E(k): Min_radius_outside()+1 (FFF_pencil_inline.h:497-504). */
int ts_plan_num_shells(const ts_plan* plan, int* n_shells);
/* A zeroed device field of ncomp components in the plan's spectral layout
 * (ncomp * elems_per_comp complex elements of the plan's precision), the storage
 * PlainCVF / CVF allocate for their V1..V3 (fields/plainCvf.cc:52) and CSF for F.
 * The caller owns it and releases it with ts_free_field. */
int ts_alloc_field(const ts_plan* plan, int ncomp, void** field);
int ts_free_field(void* field);
/* Wait for the plan's stream and report the plan's health word: a bounded device
 * wait that gave up in any earlier call (TS_ERR_TIMEOUT), else a NaN or Inf that a
 * step wrote into the state (TS_ERR_NAN; every step's stage-4 store checks the
 * values it writes, the device-side form of the reference's abort on a NaN total
 * energy, Ifluid_main.cc:127-129).  The stepping calls report the same at their
 * next call, without stepping.  The word stays set until ts_plan_clear_status. */
int ts_plan_status(ts_plan* plan);
/* Clear the plan's health word (after the caller has replaced a bad state).  No
 * reference counterpart. */
int ts_plan_clear_status(ts_plan* plan);
/* Test of the timeout path: one block waits, with the library's bounded wait and
 * `polls` polls, on an mbarrier that nothing arrives on and no copy completes, so
 * the wait gives up, sets the plan's timeout bit and the kernel returns.  Then
 * ts_plan_status reports TS_ERR_TIMEOUT and the context stays usable.  No
 * reference counterpart. */
int ts_plan_expire_wait(ts_plan* plan, int polls);
/* Set the fixed time step (global.time.dt). */
int ts_plan_set_dt(ts_plan* plan, double dt);

/* Universal::Forward_transform / Inverse_transform (FFF_pencil_tr.cc:43-66,
 * SFF_pencil_tr.cc:43-68).  parity replaces global.program.sincostr_switch:
 * "FFF" for FFF; "SFF" (sine along x) or "CFF" (cosine along x) for SFF.
 * real: (Nx,Ny,Nz+2) padded; spec: (Nx,Ny,Nz/2+1).  ncomp fields back to back. */
int ts_fft_forward(ts_plan* plan, const char* parity, const void* real_in, void* spec_out, int ncomp);
int ts_fft_inverse(ts_plan* plan, const char* parity, const void* spec_in, void* real_out, int ncomp);

/* Nlin_incompress::Compute_nlin(FluidVF&) (compute_nlin.cc:58-109): dealias U
 * in place (as the reference does), then nlin_i = sum_j i K_j F[u_i u_j]
 * (conservative) or -F[u x omega] (rotational).  u_hat, nlin_hat: 3 components. */
int ts_nlin(ts_plan* plan, void* u_hat, void* nlin_hat);

/* Time_advance_incompress::RK4(U,P,F) (RK.cc:91-170) + strong reality fix
 * (Time_advance.cc:59-60), nsteps times, in place on u_hat (3 components).
 * FFF with force_type NONE or CARATI_ENERGY_SUPPLY. */
int ts_rk4_step(ts_plan* plan, void* u_hat, int nsteps);

/* RK4(U,T,P,F) for RBC (RK_SF.cc:97-221), PRLARGE/ULARGE buoyancy
 * (compute_force_RBC.cc:104-150): on an SFF plan, and on SSF / SSS plans
 * (conservative, unforced; T takes the Vx parity, SCF / SCC, with the products
 * u_i T in Vi2 / VxVy / VxVz, Global_process_basic_vars.cc:108-116; on SSS, T_hat
 * is one component of real coefficients in the padded real layout). */
int ts_rk4_step_rbc(ts_plan* plan, void* u_hat, void* T_hat, int nsteps);
/* RK4(U,T,P,F) (RK_SF.cc:97-221) with a passive scalar (program.kind SCALAR_INCOMPRESS,
 * Compute_force_TO_rhs_scalar, Tadvance_functions.cc:464-474, no force) on an FFF
 * plan, conservative form: U with nu, T with kappa; T_hat one component in the
 * state layout.  Replaces that RK4 call for kind SCALAR_INCOMPRESS. */
int ts_rk4_step_scalar(ts_plan* plan, void* u_hat, void* T_hat, int nsteps);
/* Time_advance_incompress::RK4(U, W, P, F) for incompressible MHD (RK_VF_MHD.cc:126-186,
 * Compute_nlin(U, W) compute_nlin_VF_MHD.cc:40-95 in Elsasser form) + the strong
 * reality condition on U and B (Time_advance.cc:126-129), FFF plan, no force:
 * U with nu, B = W with eta = the plan's kappa (diss_coefficients[1]); b_hat three
 * components in the state layout. */
int ts_rk4_step_mhd(ts_plan* plan, void* u_hat, void* b_hat, int nsteps);

/* Temperature perturbation for RBC (SFF): amplitude amp and uniform random
 * phases (this project's splitmix64 generator, counter = linear mode index) on
 * the modes with grid radius |(m, ky, kz)| <= kmax and m >= 1, then the strong
 * reality condition.  The reference's RBC ICs are read from files or set per
 * mode (init_cond_main.cc:48-78); this is the benchmark's seeded stand-in. */
int ts_init_temperature_perturbation(ts_plan* plan, double amp, double kmax, uint64_t seed, void* T_hat);

/* CVF::Compute_total_energy (Cvf.cc:213-221): sum over ncomp components, with the
 * basis's weights (FFF_pencil_energy.cc, SFF_pencil_energy.cc:76-95, and on SSF / SSS
 * the Multiplicity_factor weights 4 / 2 / 1 / 1/2 of SSF_pencil_energy.cc:76-103,
 * SSS_pencil_energy.cc:69-98; SSS coefficients real in the padded layout, whose two
 * padding reals per line are not summed). */
int ts_energy(ts_plan* plan, const void* a_hat, int ncomp, double* energy);
/* Universal::Compute_shell_spectrum (universal_energy.cc:279-366), summed over
 * ncomp components: Ek[n_shells]. */
int ts_shell_spectrum(ts_plan* plan, const void* a_hat, int ncomp, double* Ek, int n_shells);
/* EnergyTr::Compute_flux(U) (compute_flux.cc:51-65): the energy flux Pi(R_i) out of
 * each sphere |K| <= R_i, at most 63 radii (in any order: the reference's default
 * radii do not ascend on small grids; the one-pass form runs for ascending radii).  Corner-box or no dealiasing:
 * the reference's per-sphere algorithm, one giver nonlinear term per sphere
 * (Fill_in_sphere fill_space.cc:56-64, Compute_nlin(U, Giver) compute_nlin_ET_VF.cc:
 * 71-87) and Pi(R) = -sum_{|K| > R} 2 mult Re(N . conj(D U)) (prod_nlinV.cc:61-69).
 * Two-thirds dealiasing: the same value from one nonlinear term, Pi(R) =
 * sum_{|K| <= R} 2 mult Re(N . conj(D U)), N = F[(u.grad)u] (there the products
 * alias only onto modes D U does not hold, so the two forms agree).  FP64 sums in a
 * fixed order.  u_hat is not modified (the reference dealiases U in place here:
 * call ts_dealias_field first to reproduce that side effect).  FFF, SFF and SSF plans
 * (on SFF and SSF the per-sphere algorithm in every dealias mode, through the sin/cos
 * passes with each product's parities; on SFF the velocity flux of an RBC plan, in three
 * dimensions or two), and SSS plans (the per-sphere algorithm on the real coefficients,
 * sphere fill and outside sum over the real z index, SSS_pencil_ET.cc:50-70, 662-678). */
int ts_flux(ts_plan* plan, const void* u_hat, const double* radii, int n_radii, double* Pi);
/* Universal::Dealias on ncomp components in place (FFF_pencil_basic.cc:87-90 corner
 * box, or the plan's two-thirds rule; nothing for dealias NONE; on SSS plans the real
 * coefficients by the real z index). */
int ts_dealias_field(ts_plan* plan, void* a_hat, int ncomp);
/* Raw shell sums for the reference's text outputs: sums[k] = sum over modes with
 * ceil|K| = k of mult K^2 Re(A . conj(B)) (B = NULL: |A|^2), counts[k] = sum of
 * 2 mult (Compute_local_shell_spectrum / _force, universal_energy.cc:196-229,
 * 279-310; E(k) = sums 4 pi / (counts kf1 kf2 kf3)).  Device pointers; either
 * output may be NULL. */
int ts_shell_sums(ts_plan* plan, const void* a_hat, const void* b_hat, int ncomp, double* sums, double* counts,
                  int n_shells);
/* The Carati force of state u_hat (FORCE::Compute_force, compute_force_Carati.cc:158-205)
 * as a full spectral field f_hat (3 components, zero outside the forcing band);
 * device pointers. */
int ts_force_field(ts_plan* plan, const void* u_hat, void* f_hat);
/* max |div U| (universal_basic.cc:343-356), with the basis's derivatives (SSF / SSS:
 * sine +K, cosine -K along the sin/cos axes; SSS padding reals skipped). */
int ts_max_div(ts_plan* plan, const void* u_hat, double* max_div);
/* Nusselt number nu0 + nuc <U1, T> with the factors of the plan's scaling
 * (Correlation.cc:144-176; PRLARGE/ULARGE: 1 + 2 sqrt(Ra Pr) <U1, T>; PRZERO reports
 * 2 <U1, T>), on SFF, SSF and SSS plans. */
int ts_nusselt(ts_plan* plan, const void* u_hat, const void* T_hat, double* Nu);
/* The slaved field of a PRZERO / PRINFTY state on an SFF plan, in place: PRZERO sets
 * T_hat = U.V1 / K^2 (Zero_Prandtl_number_compute_temperature, FluidVF.cc:228-232);
 * PRINFTY sets u_hat = vs P(T x) / K^2 (Infinite_Prandtl_number_compute_velocity,
 * FluidVF.cc:235-272) -- what the reference does after an initial condition
 * (init_cond_energy.cc:242-258).  TS_ERR_ARG for the other scalings. */
int ts_rbc_slave(ts_plan* plan, void* u_hat, void* T_hat);

/* Random-phase solenoidal FFF field with shell energies E_ic[n] (construction of
 * init_cond_energy.cc:67-120; counter-based splitmix64 phases from seed), then the
 * strong reality fix and a rescale to total energy target_energy (<= 0: no rescale). */
int ts_init_energy_spectrum(ts_plan* plan, const double* E_ic, int n, uint64_t seed, double target_energy,
                            void* u_hat);

/* Ensemble of independent Boussinesq (RBC, SFF) runs of uneven sizes: a batching
 * layer with no reference counterpart (the reference runs one field per MPI job).
 * Each member has its own plan (N, Ra, Pr; nu and kappa of base.Pr_option / base.Uscaling,
 * PRLARGE or PRSMALL: PRZERO / PRINFTY return TS_ERR_UNSUPPORTED) and device state; the
 * other settings come from `base`.  Members of one grid size advance as one batch;
 * ts_ensemble_run advances every member by nsteps with one CUDA graph launch per eight
 * steps (plus one per remaining step), whose parallel branches are the size groups.
 * Asynchronous: ts_ensemble_synchronize / ts_ensemble_nusselt wait for it. */
typedef struct {
  int N[3];
  double Ra, Pr;
} ts_member;
typedef struct ts_ensemble ts_ensemble;
int ts_ensemble_create(const ts_config* base, const ts_member* members, int count, ts_ensemble** ens);
int ts_ensemble_destroy(ts_ensemble* ens);
/* the member's plan and its device state u_hat (3 components) and T_hat */
int ts_ensemble_member(ts_ensemble* ens, int member, ts_plan** plan, void** u_hat, void** T_hat);
/* u = 0 and a temperature perturbation (ts_init_temperature_perturbation, seed + member) */
int ts_ensemble_init_temperature(ts_ensemble* ens, double amp, double kmax, uint64_t seed);
int ts_ensemble_run(ts_ensemble* ens, int nsteps);
int ts_ensemble_synchronize(ts_ensemble* ens);
/* Nusselt number of every member (Correlation.cc:154-156) */
int ts_ensemble_nusselt(ts_ensemble* ens, double* Nu);
/* Per-member health after the steps run so far (waits for them): status[m] =
 * TS_OK, TS_ERR_NAN (the member's step wrote a NaN or Inf into its U or T) or
 * TS_ERR_TIMEOUT (a bounded wait of its size group gave up).  Members are
 * independent: a bad member does not change the others.  clear != 0 resets the
 * words afterwards.  No reference counterpart (one run per reference process). */
int ts_ensemble_health(ts_ensemble* ens, int* status, int clear);

/* Discrete adjoint of the FFF IF-RK4 step (rotational form, unforced plans).
 * No reference counterpart: the reference has no adjoint.  Cotangents are
 * complex fields in the state's layout, in the real inner product
 * <A, B> = Re sum A conj(B) over the stored half spectrum (torch's convention
 * for the gradient of a real loss with respect to a complex tensor).
 * Device pointers only, 16-byte aligned.
 *
 * ts_rk4_step_keep: one ts_rk4_step that writes the new state to u_next (may be
 *   u_hat) and keeps the stage fields U1, U2, U3 (9 components) in `stages`.
 * ts_adjoint_step: lam_hat <- (d step / d u_hat)^T lam_hat, u_hat = the state
 *   at the start of the step, `stages` = its stage fields.
 * ts_adjoint_window: checkpointed form.  Recomputes nsteps steps from u_start,
 *   keeping every step's state and stage fields in `work`, then runs the nsteps
 *   adjoint steps backwards: lam_hat enters as the cotangent of the state after
 *   nsteps and leaves as the cotangent of u_start.
 * ts_adjoint_work_bytes: size of `work` for nsteps (12 components per step). */
int ts_rk4_step_keep(ts_plan* plan, const void* u_hat, void* u_next, void* stages);
int ts_adjoint_step(ts_plan* plan, const void* u_hat, const void* stages, void* lam_hat);
int ts_adjoint_work_bytes(const ts_plan* plan, int nsteps, size_t* bytes);
int ts_adjoint_window(ts_plan* plan, const void* u_start, int nsteps, void* lam_hat, void* work, size_t work_bytes);

/* Launch tuning (no reference counterpart: the reference leaves the FFT plan
 * to FFTW's planner).  Each right-hand side runs five pass classes; for each
 * the library holds a fixed rule (candidate 0) and up to five other kernel
 * candidates that change the radix schedule (elements per thread, so the
 * Stockham passes' radices), the column-tile width, the staging depth (y passes:
 * candidate 4 keeps two items in flight ahead of the one transformed; at 1024 points
 * in FP32 the y forward rule is one tile per block with 32 elements per thread and
 * candidate 5 swaps it with the y inverse rule's form), or the kernel form (z:
 * shared-memory slot kernels, and at 1024 points in FP32 candidate 4 loads each
 * component just before its transform; FFF inverse x at 1024 points in FP32 under
 * two-thirds dealiasing: candidate 5 swaps the staged rule kernel with the
 * direct-load one; FFF forward x: split x FFF + elementwise epilogue; SFF forward x:
 * the other fused/split choice), plus a
 * blocks-per-SM count for the persistent launches (y passes, fused FFF
 * forward x; 0 = the rule).  Every candidate computes the same transform;
 * results differ from the rule's in rounding only.
 * ts_tuning_candidates: bit v of *mask set when candidate v of class cls exists
 *   for this plan; *blocks != 0 when the class takes a blocks-per-SM count.
 * ts_plan_set_tuning: TS_ERR_ARG if a candidate does not exist for the plan.
 * ts_plan_autotune: coordinate descent, class by class: times whole IF-RK4 steps
 *   of a scratch state on the plan's stream with CUDA events (best of `reps`
 *   trials, enough steps per trial for about 3 ms), keeps a candidate only when
 *   it is at least 1 % faster.  The caller's fields are not touched; the plan's
 *   work buffers are.  report (may be NULL): a JSON summary of every timing.
 *   The incumbent is re-timed at the start of every class, and the picks are
 *   kept only if, timed twice against the rule (interleaved), they are still at
 *   least 1 % faster ("confirm" and "final" in the report).
 * ts_ensemble_autotune: the same for every size group of an ensemble, timing
 *   whole ensemble steps (one graph launch each, about 30 ms per trial); the
 *   members' states are saved and restored. */
typedef enum {
  TS_TUNE_X_INV = 0,
  TS_TUNE_Y_INV = 1,
  TS_TUNE_Z = 2,
  TS_TUNE_Y_FWD = 3,
  TS_TUNE_X_FWD = 4,
  TS_TUNE_NCLASS = 5
} ts_tune_class;
typedef struct {
  int variant[TS_TUNE_NCLASS];
  int blocks_per_sm[TS_TUNE_NCLASS];
} ts_tuning;
int ts_tuning_candidates(const ts_plan* plan, int cls, int* mask, int* blocks);
int ts_plan_get_tuning(const ts_plan* plan, ts_tuning* tuning);
int ts_plan_set_tuning(ts_plan* plan, const ts_tuning* tuning);
int ts_plan_autotune(ts_plan* plan, int reps, char* report, size_t report_len);
/* the tuning of the size group holding member m (its plan's tuning) */
int ts_ensemble_get_tuning(ts_ensemble* ens, int member, ts_tuning* tuning);
int ts_ensemble_set_tuning(ts_ensemble* ens, int member, const ts_tuning* tuning);
int ts_ensemble_autotune(ts_ensemble* ens, int reps, char* report, size_t report_len);

/* Kernel classes of one right-hand-side evaluation, for ts_profile_read. */
typedef enum {
  TS_KCLASS_INV_X = 0,  /* dealias + inverse FFT along x (+ vorticity) */
  TS_KCLASS_Y_INV = 1,  /* inverse FFT along y */
  TS_KCLASS_Z = 2,      /* C2R z + real-space products + R2C z */
  TS_KCLASS_Y_FWD = 3,  /* forward FFT along y */
  TS_KCLASS_FWD_X = 4,  /* forward FFT along x + projection + RK stage update */
  TS_KCLASS_OTHER = 5,  /* forcing and reality kernels */
  TS_KCLASS_COUNT = 6
} ts_kernel_class;

/* Per-kernel-class timing with CUDA events recorded on the plan's stream around
 * every launch of ts_rk4_step (no reference counterpart: the reference times
 * the whole run with time(), main.cc:105-109).  bytes_per_launch is the
 * algorithmic traffic of one launch (every field read or written once). */
int ts_profile_enable(ts_plan* plan, int enable);
int ts_profile_reset(ts_plan* plan);
int ts_profile_read(ts_plan* plan, int kernel_class, double* total_ms, long long* launches,
                    double* bytes_per_launch);

/* Shell spectrum E(k) without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when they
 * need the diagnostic (a stepping loop that has reserved nearly all of the GPU's
 * memory for its fields, or one that must not let cudaMalloc / cudaFree
 * synchronize the device).  Same result as ts_shell_spectrum, but it needs no
 * plan: the caller passes the geometry, the device field a_hat (ncomp
 * components) and a device array Ek[n_shells], which receives the normalised
 * spectrum.  The shell accumulators (the result and the per-block partial
 * sums of the shell kernel's 32 blocks) are a file-scope __device__ array for
 * TS_NOALLOC_MAX_SHELLS shells (2.06 MiB, held on every GPU that loads the
 * library until exit); more shells than that return TS_ERR_ARG with a message
 * on stderr.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture.  Calls share the array and each overwrites what it
 * reads on `stream` before reading it, so calls that overlap on the GPU race:
 * order them.  The sums are added in a fixed order (same field, same bits). */
#define TS_NOALLOC_MAX_SHELLS 4096
int ts_shell_spectrum_noalloc(int basis, int precision, const int N[3], const double kfactor[3], const void* a_hat,
                              int ncomp, double* Ek, int n_shells, void* stream);

/* Number of kernels this library has launched since load (diagnostics). */
long long ts_kernel_launch_count(void);
/* Last CUDA error string seen by the library ("" if none). */
const char* ts_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
