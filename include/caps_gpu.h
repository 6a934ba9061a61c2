/* caps_gpu.h — C ABI of the B200 engine for CAPS's MD force-and-integrate step.
 *
 * This is the drop-in boundary between CAPS's C++ core and the device. Only plain C types cross it: pointers, sizes,
 * doubles and POD structs. Every entry point returns 0 on success or a negative status; caps_gpu_error() gives the text,
 * which is the text the CPU path would have thrown (FieldError messages) so the caller can rethrow it unchanged.
 *
 * What each entry point replaces in the reference (paths inside MuhammadUzairRiaz/CAPS):
 *   caps_gpu_create     Evaluator::Evaluator(const ForceField&, const EnergyOptions&)   core/include/caps/field.hpp:332
 *   caps_gpu_set_options Evaluator::set_options(const EnergyOptions&)                    core/include/caps/field.hpp:337
 *   caps_gpu_energies   Evaluator::energies(bool)                                       core/include/caps/field.hpp:344
 *   caps_gpu_compute    Evaluator::compute(x, cell, f) -> EnergyTerms                    core/include/caps/field.hpp:340
 *   caps_gpu_list_builds Evaluator::list_builds()                                       core/include/caps/field.hpp:341
 *   caps_gpu_reload     Evaluator::reload()                                              core/include/caps/field.hpp:349-352
 *   caps_gpu_freeze_pairs Evaluator::freeze_pairs(x, cell) / unfreeze()                 core/include/caps/field.hpp:341-347
 *   caps_gpu_pairs      Evaluator::pairs()                                               core/include/caps/field.hpp:348
 *   caps_gpu_threads    Evaluator::threads()                                             core/include/caps/field.hpp:333
 *   caps_gpu_run        run_dynamics(System&, const DynamicsOptions&, DynamicsReport*)   core/include/caps/dynamics.hpp:180
 *   caps_gpu_destroy    Evaluator::~Evaluator()                                          core/include/caps/field.hpp:333
 *   caps_gpu_traj_*     write_trajectory(const Trajectory&, path, dt_fs)                 core/include/caps/io.hpp:142, io_traj.cpp:47
 *   caps_gpu_request_stop request_stop(bool)                                            core/include/caps/live.hpp:29
 *   caps_gpu_error      FieldError text / caps_last_error()                              capi/include/caps_c.h:63
 *
 * Units are the reference's (LAMMPS "real"): Å, fs, kcal/mol, e, g/mol, K, atm.
 */
#ifndef CAPS_GPU_H
#define CAPS_GPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CAPS_GPU_ABI_VERSION 5

/* Status codes (negative). The text is in caps_gpu_error(). */
#define CAPS_GPU_OK 0
#define CAPS_GPU_EINVAL (-1)      /* bad argument: sizes, options the engine does not take */
#define CAPS_GPU_ECUDA (-2)       /* a CUDA call failed */
#define CAPS_GPU_EFIELD (-3)      /* FieldError: FENE overstretch, cell too small, non-finite coordinates */
#define CAPS_GPU_ECONSTRAINT (-4) /* SHAKE/RATTLE did not converge or a bond turned past 90 degrees */
#define CAPS_GPU_ECANCEL (-5)     /* the progress callback asked to stop (DynamicsCancelled) */
#define CAPS_GPU_ENODEV (-6)      /* no CUDA device: there is no CPU fallback */
#define CAPS_GPU_ESTOPPED (-7)    /* a stop was asked for (caps_gpu_request_stop): DynamicsInterrupted; the state is the
                                     stopped step's */

/* The force field as the device path consumes it: the subset of caps::ForceField (core/include/caps/field.hpp:154-249)
 * that the MD hot path reads, flattened to arrays. Pair coefficients are given per type pair after mixing
 * (caps::mixed_pair, field.cpp:2588), so the mixing rule stays on the host. Term lists keep the reference's order;
 * dihedral and improper Fourier terms of one quadruple stay adjacent, as the reference groups them
 * (field.cpp:1875-1920). Arrays are read during caps_gpu_create and not kept. */
typedef struct {
  int32_t natoms;
  int32_t ntypes;
  const int32_t* type_index; /* [natoms] */
  const double* charge;      /* [natoms] e (already divided by sqrt(dielectric) if the model has one) */
  const double* mass;        /* [natoms] g/mol */
  const double* pair_eps;    /* [ntypes*ntypes] kcal/mol, after mixing; <= 0: the pair does not interact */
  const double* pair_sigma;  /* [ntypes*ntypes] Å */
  int32_t nbonds;            /* harmonic bonds k (r - r0)^2 */
  const uint32_t* bond_ij;   /* [2*nbonds] */
  const double* bond_k_r0;   /* [2*nbonds] */
  int32_t nangles;           /* harmonic angles kt (theta - theta0)^2, j the vertex, theta0 in radians */
  const uint32_t* angle_ijk; /* [3*nangles] */
  const double* angle_kt_theta0;
  int32_t ndihedrals;        /* v [1 + cos(n phi - delta)], IUPAC phi */
  const uint32_t* dihedral_ijkl; /* [4*ndihedrals] */
  const double* dihedral_v_delta; /* [2*ndihedrals] */
  const int32_t* dihedral_n;      /* [ndihedrals] */
  int32_t nimpropers;             /* same form as the dihedrals (AMBER/OPLS order) */
  const uint32_t* improper_ijkl;
  const double* improper_v_delta;
  const int32_t* improper_n;
  int32_t npairs14;               /* 1-4 pairs: LJ scaled by lj14 (or per pair), Coulomb handled with the exclusions */
  const uint32_t* pair14_ij;      /* [2*npairs14] */
  const double* pair14_lj;        /* [npairs14] per-pair LJ scale, or NULL for lj14 */
  const double* pair14_coul;      /* [npairs14] per-pair Coulomb scale, or NULL for coul14 */
  double lj14, coul14;
  const uint32_t* excl_offset;    /* [natoms+1] CSR of ForceField::excluded (1-2, 1-3, 1-4 partners, sorted) */
  const uint32_t* excl_list;
  int32_t nfene;                  /* BondX form 3: -0.5 K R0^2 ln(1-(r/R0)^2) + WCA(eps, sigma) below 2^(1/6) sigma */
  const uint32_t* fene_ij;        /* [2*nfene] */
  const double* fene_k_r0_eps_sigma; /* [4*nfene] */
  int32_t lj_shift;               /* ForceField::lj_shift: LJ shifted to zero at the cut-off, no tail correction */
  double model_cutoff;            /* ForceField::cutoff: > 0 replaces the options' cut-off */
  int32_t lj_form;                /* ForceField::pair_form (field.cpp:505-506): 0 "lj12-6" 4 eps ((s/r)^12 - (s/r)^6), 1 "lj9-6"
                                   * (class II) eps (2 (s/r)^9 - 3 (s/r)^6); pair_eps / pair_sigma are the mixed values either way */
  /* ABI 5: ForceField::pair_func (field.hpp:68, 174), non-LJ forms for type pairs, on the FP64 path (a force field with any
   * runs every evaluation in FP64, as the reference's mixed path falls back to its FP64 pair loop for them; field.cpp:848).
   * Per entry: the type pair (a <= b) and (form, a, b, c, rc): 1 Buckingham A e^(-r/rho) - C/r^6 (A, rho, C); 2 Morse
   * D (e^(-2 alpha (r - r0)) - 2 e^(-alpha (r - r0))) (D, alpha, r0); 3 Rydberg (A + C r) e^(-r/rho) (A, rho, C); rc > 0
   * the pair's own cut-off. The tabulated, cosine-squared, lj/gromacs and SDK forms are refused. */
  int32_t npair_func;
  const int32_t* pair_func_ab;    /* [2*npair_func] */
  const double* pair_func_p;      /* [5*npair_func] form, a, b, c, rc */
  /* forms 11-14 SDK C eps ((s/r)^m - (s/r)^n) (a eps, b sigma; 9-6, 12-4, 12-6, 12-5), 20 LJ 12-6 with GROMACS's force
   * switch from lj_inner to the cut-off (a eps, b sigma), 31 / 32 cosine-squared attraction, 32 with WCA below sigma
   * (a eps, b sigma, c its cut-off), 40 tabulated (a the table's index): the reference's codes (field.hpp:61-75) */
  double lj_inner;                /* ForceField::lj_inner (Å): where the lj/gromacs and CHARMM switches start */
  int32_t lj_fsw;                 /* ForceField::lj_fsw: every 12-6 pair with CHARMM's force switch from lj_inner to the cut-off
                                   * (field.cpp:1455-1469), no shift and no tail; runs the FP64 path */
  int32_t ntables;                /* ForceField::tables (field.hpp:75-76, 175) */
  const int32_t* table_n;         /* [ntables] points of each table */
  const double* table_r0_dr;      /* [2*ntables] first point and spacing (Å) */
  const double* table_e;          /* the tables' energies, one after another (kcal/mol) */
  const double* table_f;          /* the tables' forces -dE/dr (kcal/mol/Å), the same layout */
} caps_gpu_ff;

/* caps::EnergyOptions (field.hpp:274-308), the fields the device path takes. */
typedef struct {
  double cutoff;        /* Å, LJ and Coulomb (default 10) */
  double skin;          /* Å, Verlet buffer (default 2) */
  int32_t coulomb;      /* electrostatics on */
  int32_t electrostatics; /* 0 damped shifted force, 1 PME */
  double dsf_alpha;     /* 1/Å (0.2) */
  double ewald_rtol;    /* erfc(beta rc) = rtol (1e-5) */
  double pme_spacing;   /* Å (1.0) */
  int32_t pme_order;    /* B-spline order, 3..8 (reference default 5; the configs use 4) */
  int32_t tail;         /* LJ tail correction */
  int32_t precision;    /* 0 mixed: FP32 arithmetic, int64 fixed-point forces; 1 double: FP64 throughout */
  double force_cap;     /* > 0: LJ continued linearly inside the radius where |F| reaches this (push-off); FP64 only */
  int32_t parts;        /* 1 bonded, 2 non-bonded, 3 both (r-RESPA splits) */
} caps_gpu_opts;

/* caps::EnergyTerms (field.hpp:310-320). */
typedef struct {
  double bond, angle, dihedral, improper, vdw, coulomb;
  double virial;        /* sum r.f, kcal/mol */
  double w[6];          /* virial tensor xx yy zz xy xz yz */
  double tail_energy, tail_virial;
} caps_gpu_terms;

/* Called with each checkpoint: positions (3N, unwrapped), velocities (3N, Å/fs), cell[12] and step (with step_offset).
 * DynamicsOptions::checkpoint (core/include/caps/dynamics.hpp:143-146). */
typedef void (*caps_gpu_checkpoint_fn)(const double* x, const double* v, const double* cell, int64_t step, void* user);

/* caps::DynamicsOptions (dynamics.hpp:60-154), the fields the device step takes. */
typedef struct {
  double dt;                /* fs */
  int64_t steps;
  double temperature;       /* K */
  double temperature_end;   /* K; >= 0 ramps the target linearly over the run */
  int32_t thermostat;       /* 0 none (NVE), 1 Bussi, 2 Langevin (BAOAB), 3 Nose-Hoover chain of 3 */
  double tau_t;             /* fs */
  int32_t barostat;         /* 0 none, 1 stochastic cell rescaling, 2 Berendsen, 3 MTK (the reference's CRescale, Berendsen
                               and MTK; MTK every step, isotropic, without constraints, with Nose-Hoover or no thermostat) */
  double pressure;          /* atm */
  double tau_p;             /* fs */
  double compressibility;   /* 1/atm */
  int32_t barostat_every;
  int32_t constraints;      /* 0 none, 1 bonds to hydrogen and rigid water (SHAKE/RATTLE; SETTLE for waters) */
  int32_t new_velocities;   /* draw Maxwell-Boltzmann velocities even when given some */
  uint64_t seed;
  int32_t thermo_every;
  int32_t frame_every;      /* 0 none */
  int64_t step_offset;
  int32_t respa;            /* r-RESPA inner steps (1 off) */
  const int8_t* is_hydrogen; /* [natoms] element == 1, for the constraint set; NULL: mass < 1.6 */
  const int8_t* is_oxygen;   /* [natoms] element == 8, for rigid waters; NULL: none */
  int32_t respa_split;      /* with respa > 1: 0 bonded forces every dt/respa (the reference's split, dynamics.cpp:113);
                               1 PME every dt, everything else every dt/respa (a split the reference does not have) */
  int64_t checkpoint_every; /* 0 none; at steps s % checkpoint_every == 0, s < steps, whose x and v are finite
                               (dynamics.cpp:758-763) */
  caps_gpu_checkpoint_fn checkpoint;   /* NULL none */
  void* checkpoint_user;
  /* ABI 4 */
  double hmr;               /* > 0: hydrogen mass repartitioning to this mass in u (DynamicsOptions::hmr, dynamics.cpp:125-147) */
  int32_t anisotropic;      /* with the Berendsen barostat: each Cartesian axis scaled on its own (dynamics.cpp:668-687) */
  int32_t couple_axes;      /* with anisotropic: bit k couples axis k (DynamicsOptions::couple_axis); 0 means all three */
  int32_t axis_pressure_set; /* with anisotropic: bit k set: axis k's target is axis_pressure[k], otherwise pressure */
  double axis_pressure[3];  /* atm */
  /* ABI 5 */
  int32_t constraint_algorithm; /* 0 SHAKE, 1 LINCS (order 4) for the positions; RATTLE for the velocities either way
                                   (DynamicsOptions::constraint_algorithm, constraints.cpp:125-185) */
} caps_gpu_md_opts;

/* caps::ThermoRow (dynamics.hpp:28-43), the fields the device step fills. */
typedef struct {
  int64_t step;
  double time_ps, temperature, potential, kinetic, total, conserved, pressure, volume, density;
  double target_temperature;
  double p[6];
  caps_gpu_terms terms;
} caps_gpu_thermo;

/* Called with each thermo row; non-zero cancels the run (DynamicsCancelled). */
typedef int32_t (*caps_gpu_progress_fn)(const caps_gpu_thermo* row, void* user);
/* Called with each recorded frame: positions (3N, unwrapped), cell[12] (origin, a, b, c) and step.
 * Frames and checkpoints leave the device asynchronously: a recorded step's state is copied aside on the device, moved to
 * pinned host memory on a copy stream while the next steps run, and handed to the callbacks on the calling thread at the
 * next step that reports or records, or at the end of the run. The order of the calls is the reference's: the thermo row
 * of a step, then its frame, then its checkpoint; every frame and checkpoint before the next row. The pointers are valid
 * during the call only. */
typedef void (*caps_gpu_frame_fn)(const double* x, const double* cell, int64_t step, void* user);

/* The state a run works on, in place: positions (3N unwrapped), velocities (3N, Å/fs; may be NULL to draw them),
 * cell[12] (origin, a, b, c). On return they hold the end state. */
typedef struct {
  double* x;
  double* v;
  double* cell;
  int32_t has_velocities;
} caps_gpu_state;

typedef struct caps_gpu_engine caps_gpu_engine;

int32_t caps_gpu_abi_version(void);
/* Number of CUDA devices visible (0: none). Needs no engine. */
int32_t caps_gpu_device_count(void);

/* Builds the engine on the current CUDA device: uploads the force field, sizes the buffers. NULL on error, with the
 * text in caps_gpu_error(NULL). Replaces Evaluator::Evaluator (core/include/caps/field.hpp:332). */
caps_gpu_engine* caps_gpu_create(const caps_gpu_ff* ff, const caps_gpu_opts* opts);
/* Replaces Evaluator::set_options (field.hpp:337): a new cut-off or skin rebuilds the list at the next call. */
int32_t caps_gpu_set_options(caps_gpu_engine* e, const caps_gpu_opts* opts);
/* Replaces Evaluator::energies(bool) (field.hpp:344): 0 lets later calls skip the pair energies (forces unchanged). */
int32_t caps_gpu_energies(caps_gpu_engine* e, int32_t on);
/* Energy, forces and virial at x (3N, Å, host memory) in cell[12]; f (3N host) is overwritten. Replaces
 * Evaluator::compute (field.hpp:340, field.cpp:1249-2539). */
int32_t caps_gpu_compute(caps_gpu_engine* e, const double* x, const double* cell, double* f, caps_gpu_terms* out);
/* The same with x and f already in device memory (3N doubles each): no host copies. */
int32_t caps_gpu_compute_device(caps_gpu_engine* e, const double* d_x, const double* cell, double* d_f, caps_gpu_terms* out);
/* Replaces Evaluator::list_builds (field.hpp:341). */
int32_t caps_gpu_list_builds(const caps_gpu_engine* e);
/* Replaces Evaluator::reload (field.hpp:349-352): the force field changed (bonds, types, charges, bonded terms or
 * exclusions; the same number of atoms): everything taken from it is set up again from `ff`, with the engine's options,
 * and the list is rebuilt at the next call. A frozen list ends. */
int32_t caps_gpu_reload(caps_gpu_engine* e, const caps_gpu_ff* ff);
/* Replace Evaluator::freeze_pairs / unfreeze (field.hpp:341-347): later calls take exactly the atom pairs inside the
 * cut-off at (x, cell), whatever their distance then (a pair beyond the cut-off takes the closed-form Coulomb term),
 * on the FP64 path, and never rebuild the list; the cell may deform. Dynamics refuses a frozen engine. */
int32_t caps_gpu_freeze_pairs(caps_gpu_engine* e, const double* x, const double* cell);
int32_t caps_gpu_unfreeze(caps_gpu_engine* e);
/* Replaces Evaluator::pairs (field.hpp:348): the atom pairs of the FP64 pair list (within cut-off + skin at its last
 * build); on the mixed path, as the reference's cluster path, those of the last freeze_pairs (0 without one). -1 on error. */
int64_t caps_gpu_pairs(caps_gpu_engine* e);
/* Replaces Evaluator::threads (field.hpp:333): the device's streaming multiprocessors, the engine's parallel workers. */
int32_t caps_gpu_threads(const caps_gpu_engine* e);
/* Molecular dynamics in place on `state` (host memory). Replaces run_dynamics (dynamics.hpp:180; dynamics.cpp:71-815)
 * for the options above. progress and frame may be NULL. report (may be NULL) receives a short text summary. */
int32_t caps_gpu_run(caps_gpu_engine* e, caps_gpu_state* state, const caps_gpu_md_opts* md, caps_gpu_progress_fn progress,
                     caps_gpu_frame_fn frame, void* user, char* report, int32_t report_cap);
/* Independent replicas in lock step, one engine each (own force field, state and dynamics options; the same number of
 * steps; all engines created on the current device). Replaces running run_dynamics once per replica (core/src/dynamics.cpp:71, called in turn for each rung of a
 * Tg ladder or each seed of a protocol, e.g. core/src/mechanics.cpp:1381): a step on which no replica reports, records
 * a frame, rescales its cell or refills its thermostat draws is one CUDA graph launch for all replicas. progress and
 * frame receive user[r] for replica r. Errors: caps_gpu_error(engines[0]). Afterwards every engine's
 * caps_gpu_last_steps_per_second is the batch's. */
int32_t caps_gpu_run_batch(caps_gpu_engine* const* engines, caps_gpu_state* const* states, const caps_gpu_md_opts* const* md, int32_t count,
                           caps_gpu_progress_fn progress, caps_gpu_frame_fn frame, void* const* user);
/* A stop asked for from outside (caps::request_stop, core/include/caps/live.hpp:27-29): process-wide. A run checks it at
 * every step; at the first step s < steps that sees it, it takes a checkpoint of step s (when it has a checkpoint
 * callback and the state is finite), writes that state back and returns CAPS_GPU_ESTOPPED with the text
 * "stopped at step N (a stop was asked for)" (DynamicsInterrupted, dynamics.hpp:173-176). A batch stops every replica. */
void caps_gpu_request_stop(int32_t on);
int32_t caps_gpu_stop_requested(void);
/* The last run's throughput: steps per second over the step loop (first force excluded, as dynamics.cpp:601,776). */
double caps_gpu_last_steps_per_second(const caps_gpu_engine* e);
void caps_gpu_destroy(caps_gpu_engine* e);
/* Text of the last error on this engine (or of the last failed caps_gpu_create when e is NULL). */
const char* caps_gpu_error(const caps_gpu_engine* e);

/* Trajectory writers, frame by frame (write_trajectory, core/src/io_traj.cpp:47; write_dcd, core/src/io_binary.cpp:415;
 * write_lammps_dump, core/src/io_lammps.cpp:612): the file the reference writes for the same frames, byte for byte, but
 * written as the frames arrive instead of from a Trajectory held in memory. The format is the path's extension:
 * .lammpstrj / .dump (LAMMPS text dump: id mol type xu yu zu, the cell turned into LAMMPS's form), .dcd (LAMMPS's
 * CHARMM-style DCD with a unit-cell record per frame; the frame count and step range in the header are completed by
 * caps_gpu_traj_close; the unit-cell flag is the first frame's), .trr (GROMACS, single precision, nm).
 * ids, mols: [natoms] LAMMPS atom and molecule ids (NULL: 1..N and 1); types: [natoms] 1-based types (NULL: 1);
 * title: the DCD's second title line (NULL: empty); dt_fs: the time step, for DCD's time unit and TRR's times.
 * NULL on error with the text in caps_gpu_error(NULL). Host code: no device needed. */
typedef struct caps_gpu_traj caps_gpu_traj;
caps_gpu_traj* caps_gpu_traj_open(const char* path, int32_t natoms, const int64_t* ids, const int64_t* mols, const int32_t* types,
                                  const char* title, double dt_fs);
/* One frame: x (3N, Å), cell[12] (origin, a, b, c; a zero cell is no cell), step. */
int32_t caps_gpu_traj_append(caps_gpu_traj* t, const double* x, const double* cell, int64_t step);
/* A caps_gpu_frame_fn that appends to the writer passed as user: caps_gpu_run(..., caps_gpu_traj_frame, writer, ...)
 * streams a run's frames to the file with no other code in between. A write error is kept and returned by close. */
void caps_gpu_traj_frame(const double* x, const double* cell, int64_t step, void* user);
int64_t caps_gpu_traj_frames(const caps_gpu_traj* t);
/* Completes the header, closes the file and frees the writer; the first error met while writing, if any. */
int32_t caps_gpu_traj_close(caps_gpu_traj* t);

/* Kinetic energy and kinetic tensor of n atoms, computed without allocating any device memory. No counterpart in the
 * reference: it is for callers that may not call cudaMalloc, such as a host whose memory manager owns all device memory
 * and hands out its own buffers, or code running beside a long stream-ordered pipeline that an allocation would
 * synchronise. d_v (3n doubles, Å/fs), d_mass (n doubles, g/mol) and d_out (7 doubles) are device pointers the caller
 * owns; on completion d_out[0] = sum 0.5 m v² and d_out[1..6] = sum m v_a v_b (xx yy zz xy xz yz), in kcal/mol.
 * stream: a cudaStream_t passed as a pointer (NULL: the default stream); the call only enqueues work on it.
 * Limits: 1 <= n <= 1,048,576 (larger n is rejected with CAPS_GPU_EINVAL). The working memory is one fixed array of
 * about 230 KB per GPU, held from the library's load until the process exits, and shared by every call on that GPU: calls
 * whose work overlaps on the device (different streams, or other host threads) race on it and must be serialised by the
 * caller. The first call on each device looks up that array's device address; make that first call before any stream
 * capture. The address is kept for the life of the process: after cudaDeviceReset, or any other teardown of a device's
 * primary context, the library must be reloaded before this entry point is used on that device again.
 * Errors: caps_gpu_error(NULL). */
int32_t caps_gpu_kinetic_noalloc(const double* d_v, const double* d_mass, int32_t n, double* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CAPS_GPU_H */
