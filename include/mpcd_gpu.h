/*
 * mpcd_gpu.h -- C ABI of libmpcd_gpu.so, the B200 (sm_100a) solvent timestep
 * of multi-particle collision dynamics (MPCD).
 *
 * The library replaces one call of the reference program, the serial solvent
 * timestep
 *
 *   void timestep(cell ***CL, particleMPC *SRDparticles, spec SP[], bc WALL[],
 *                 simptr simMD, specSwimmer *SS, swimmer swimmers[],
 *                 double AVNOW[3], double AVV[3], double avDIR[3],
 *                 inputList in, double *KBTNOW, double *AVS, int runtime,
 *                 int MD_mode, outputFlagsList outFlags,
 *                 outputFilesList outFiles);
 *
 * (mpcd/headers/mpc.h:16, mpcd/subroutines/mpc.c:4496), called once per
 * iteration from mpcd/mpcd.c:268 (warm-up) and mpcd/mpcd.c:298 (main loop).
 * Where the reference keeps its state in host structures (particles in a
 * 128-byte AoS array threaded through per-cell linked lists, globals such as
 * DIM/XYZ/GnDNST, a static RNG), a handle here owns the state in device
 * memory, and every entry point takes plain pointers and sizes.
 *
 * Conventions: every function returns an int status, 0 on success and a
 * negative MPCD_ERR_* code on failure (the reference prints and calls exit(1)
 * instead, e.g. mpc.c:2805-2808, bc.c:700-711).  Nothing here calls exit().
 * A handle is used by one host thread at a time; its GPU work is ordered on
 * one CUDA stream owned by the handle.
 */
#ifndef MPCD_GPU_H
#define MPCD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPCD_ABI_VERSION 4

#define MPCD_MAX_SPECIES 10 /* reference MAXSPECI, definitions.h:66 */
#define MPCD_MAX_WALLS 16

/* status codes */
#define MPCD_OK 0
#define MPCD_ERR_ARG (-1)         /* bad argument / null pointer            */
#define MPCD_ERR_UNSUPPORTED (-2) /* option outside the GPU path            */
#define MPCD_ERR_CUDA (-3)        /* CUDA runtime error                     */
#define MPCD_ERR_NOMEM (-4)       /* device allocation failed               */
#define MPCD_ERR_STATE (-5)       /* call out of order (e.g. no particles)  */
#define MPCD_ERR_SIZE (-6)        /* size above a compiled-in maximum       */

/* collision operators: the reference's collOp codes (definitions.h:261-303)
 * that this library implements */
#define MPCD_COLL_ARBAXIS 0        /* SRD, random axis                     */
#define MPCD_COLL_ORTHAXIS 1       /* SRD, random Cartesian axis           */
#define MPCD_COLL_VICSEK 7         /* Vicsek alignment in the cell (vicsek) */
#define MPCD_COLL_CHATE 8          /* nematic Vicsek (chate), 2D           */
#define MPCD_COLL_MPCAT 2          /* Andersen MPC-AT                      */
#define MPCD_COLL_LANG 4           /* Langevin MPC (langevinMPC)           */
#define MPCD_COLL_RAT 3            /* Andersen MPC-AT+a                    */
#define MPCD_COLL_ACT_ARBAXIS 9    /* active SRD, random axis (activeSRD)  */
#define MPCD_COLL_ACT_ORTHAXIS 10  /* active SRD, random Cartesian axis    */
#define MPCD_COLL_VICSEK_MPCAT 11  /* MPC-AT with Vicsek alignment          */
#define MPCD_COLL_VICSEK_LANG 12   /* Langevin MPC with Vicsek alignment    */
#define MPCD_COLL_CHATE_MPCAT 13   /* MPC-AT with Chate alignment, 2D       */
#define MPCD_COLL_DIPOLE_DIR_SUM 16 /* nematic, dipole activity summed    */
#define MPCD_COLL_DIPOLE_DIR_AV 17  /* nematic, dipole activity averaged  */

/* nematic switch: the reference's in.LC values (definitions.h:194-200) */
#define MPCD_LC_ISOTROPIC 0
#define MPCD_LC_LOCAL 1

/* precision of the particle state */
#define MPCD_PREC_FP64 0  /* positions and velocities in FP64 (reference) */
#define MPCD_PREC_MIXED 1 /* int cell + FP32 offset, FP32 velocity;
                             cell sums and 3x3 inverses in FP64          */

/* One species of MPCD particle: the fields of the reference's spec struct
 * (SRDclss.h:56-83) that the timestep reads. */
typedef struct mpcd_species {
    double mass;        /* MASS   (json 'mass')      */
    double damp;        /* DAMP   (json 'damp')      */
    double rfc;         /* RFC    (json 'rfc')       */
    double tumble;      /* TUMBLE (json 'tumble')    */
    double chihi;       /* CHIHI  (json 'shearSusc') */
    double act;         /* ACT    (json 'act')       */
    double mfpot;       /* MFPOT  (json 'mfpot')     */
    double sigwidth;    /* SIGWIDTH                  */
    double sigpos;      /* SIGPOS                    */
    double minactratio; /* MINACTRATIO               */
} mpcd_species;

/* One planar boundary: the fields of the reference's bc struct
 * (SRDclss.h:140-200) used for a static, axis-aligned plane (P = 1,
 * exactly one non-zero component of A; PLANAR flag of read.c:1417-1428).
 * Surface W = sum_i A_i (x_i - Q_i) - R, times -1 if inv (calcW_PLANE,
 * bc.c:306-316); a particle is inside the wall when W < 0. */
typedef struct mpcd_wall {
    double A[3];     /* normal (1/aInv), points into the fluid             */
    double Q[3];     /* point on the plane                                 */
    double R;        /* offset                                             */
    int inv;         /* INV                                                */
    int phantom;     /* PHANTOM: ghost particles fill cut cells            */
    int coll_type;   /* COLL_TYPE: only 1 (BC_SURF_RULES) is implemented   */
    int pad_;
    double DN, DT;   /* position shift normal / tangential                 */
    double DVN, DVT; /* velocity shift normal / tangential                 */
    double MVN, MVT; /* velocity multiplier normal / tangential            */
    double DVxyz[3]; /* cartesian velocity shift                           */
    double MUN, MUT; /* orientation multiplier normal / tangential         */
    double MUxyz[3]; /* cartesian orientation multiplier                   */
    double DUxyz[3]; /* cartesian orientation shift                        */
    int inter[MPCD_MAX_SPECIES]; /* INTER: 1 if species interacts       */
} mpcd_wall;

/* Simulation parameters: the parts of the reference's inputList
 * (SRDclss.h:389-425) and globals (globals.h:24-65) the timestep uses. */
typedef struct mpcd_config {
    int dim;          /* DIM: 2 or 3                                       */
    int L[3];         /* XYZ: box size in cells (L[2] = 1 in 2D)            */
    double dt;        /* in.dt                                             */
    double kbt;       /* in.KBT                                            */
    int coll_op;      /* in.RTECH, one of MPCD_COLL_*                      */
    int lc;           /* in.LC, MPCD_LC_*                                  */
    double rot_ang;   /* in.RA in radians (SRD rotation angle)             */
    int galinv;       /* in.GALINV: 1 = random grid shift each step        */
    int precision;    /* MPCD_PREC_*                                       */
    double grav[3];   /* in.GRAV                                           */
    double gndnst;    /* GnDNST; <= 0 means: compute at upload as
                         globalDensities (init.c:1002-1018) does           */
    uint64_t seed;    /* key of the counter-based generator               */
    uint32_t replica; /* replica index folded into every draw              */
    int n_species;
    mpcd_species species[MPCD_MAX_SPECIES];
    int n_walls;
    mpcd_wall walls[MPCD_MAX_WALLS];
    int capacity;     /* maximum number of particles                       */
    double fricco;    /* in.FRICCO: friction of the Langevin operators     */
    double relax;     /* in.TAU: RELAX of the Vicsek-aligned operators     */
} mpcd_config;

/* Per-handle error counters (the reference prints warnings instead). */
typedef struct mpcd_status {
    uint64_t steps;         /* steps executed                               */
    uint64_t escaped;       /* particles that left the grid: re-placed at
                               the end of their step as the reference's
                               re-bin does (bin(), mpc.c:969-982), or, at
                               a shifted binning, clamped to the grid      */
    uint64_t bounce_limit;  /* particles that exceeded NBOUNCE wall
                               collisions in a step (bcCNT, bc.c:1461-1492);
                               the reference's remedies are applied: longer
                               rewinds, then re-thermalisation            */
    uint64_t nonfinite;     /* non-finite velocities seen by the step       */
    uint64_t overflow;      /* particles of cells too populous for one tile
                               (streamed without collision)                 */
    uint64_t sync_timeout;  /* bounded waits inside a kernel that gave up
                               (the step's results are then invalid)       */
} mpcd_status;

typedef struct mpcd_handle mpcd_handle;

/* Library version (MPCD_ABI_VERSION). */
int mpcd_abi_version(void);

/* Create a handle on the current CUDA device.  Replaces the reference's
 * readJson (read.c:973) + initializeSIM (init.c:2048) state set-up; the
 * particles are supplied separately by mpcd_upload_state.
 * MPCD_ERR_UNSUPPORTED for a collision operator outside MPCD_COLL_*, for
 * MPCD_COLL_CHATE, MPCD_COLL_CHATE_MPCAT or a nematic outside 2D, and for
 * active SRD whose species differ in activity (the reference takes the
 * cell's activity from the last particle of its list, an order set by its
 * re-binning history);
 * MPCD_ERR_ARG for a negative fricco with a Langevin operator. */
int mpcd_create(const mpcd_config *cfg, mpcd_handle **out);

/* Release all device memory of the handle. */
int mpcd_destroy(mpcd_handle *h);

/* Copy n particles (AoS, 3 doubles per vector; U and spid may be NULL) to
 * the device.  Replaces binin (mpc.c:924) and the initial localPROP. */
int mpcd_upload_state(mpcd_handle *h, int n, const double *Q, const double *V,
                      const double *U, const int *spid);

/* Same, reading an array of records with a byte stride, so a caller can pass
 * the reference's particleMPC array (SRDclss.h:34-44) directly:
 * stride = sizeof(particleMPC), offsets = offsetof(particleMPC, Q/V/U/SPID).
 * off_U may be (size_t)-1 to skip orientations (nematic states then start
 * every orientation at (1, 0)); off_spid (size_t)-1 gives every particle
 * species 0. */
int mpcd_upload_particles_strided(mpcd_handle *h, int n, const void *base,
                                  size_t stride, size_t off_Q, size_t off_V,
                                  size_t off_U, size_t off_spid);

/* Initial velocity distributions: the reference's vDist codes
 * (definitions.h:149-157, push init.c:1261-1291).  READ (1) is an upload. */
#define MPCD_VDIST_RANDVEL 0  /* uniform, each component in +-sqrt(kT/m)  */
#define MPCD_VDIST_HOMO 2     /* speed sqrt(DIM kT/m), random direction     */
#define MPCD_VDIST_HOMOAXIS 3 /* each component +-sqrt(DIM kT/m)           */
#define MPCD_VDIST_GAUSS 4    /* Maxwell-Boltzmann                          */

/* Initial orientation distributions: the reference's oDist codes
 * (definitions.h:165-183, orient init.c:1307-1405). */
#define MPCD_ODIST_RANDORIENT 0
#define MPCD_ODIST_ALIGNX 1
#define MPCD_ODIST_ALIGNY 2
#define MPCD_ODIST_ALIGNZ 3
#define MPCD_ODIST_ALIGN45 4
#define MPCD_ODIST_PLANEZ 5
#define MPCD_ODIST_PLANEY 6
#define MPCD_ODIST_PLANEX 7
#define MPCD_ODIST_ALIGNTR 8
#define MPCD_ODIST_ALIGNDEFECTPAIR 9

/* The initial state the reference builds from its JSON species entries. */
typedef struct mpcd_init_params {
    int population[MPCD_MAX_SPECIES]; /* POP (json 'pop', or 'dens' times
                                         the accessible volume)           */
    int vdist[MPCD_MAX_SPECIES];      /* VDIST (json 'vDist')             */
    int odist[MPCD_MAX_SPECIES];      /* ODIST (json 'oDist'), nematic    */
    int rframe;                       /* in.RFRAME (json 'rFrame')        */
    int pad_;
} mpcd_init_params;

/* Build the initial particle state on the device, as setcoord
 * (init.c:1565-1600), galileantrans (mtools.c:673-711, when rframe and more
 * than 2 particles) and the VSC temperature scaling (scaleT, therm.c:106-143)
 * of initializeSIM (init.c:2092-2170) do: the first population[0] particles
 * are species 0, and so on; positions uniform in the box, placed anew while
 * any interacting wall has W <= TOL; velocities from vdist; orientations
 * (nematic configs) from odist at the first position; then V scaled so that
 * TEMP about the initial mean velocity is kbt.  Random draws are keyed by
 * (seed, replica) at step 0.  *kbtnow (may be NULL) receives TEMP after the
 * scaling, what the reference computes at init.c:2170.  The state replaces
 * any uploaded one and downloads like an upload.  MPCD_ERR_ARG if a species
 * with particles has no accessible volume (the reference loops for ever
 * there) or a particle is still inside a wall after the attempts its
 * species' accessible fraction allows (64 / fraction, at least 256).
 * MPCD_ERR_UNSUPPORTED for vdist READ, and for a 2D nematic, the odist
 * codes ALIGNZ, PLANEY and PLANEX: they give the orientation a z component,
 * which the reference keeps and rotates back into the plane, but a 2D state
 * here does not hold. */
int mpcd_init_state(mpcd_handle *h, const mpcd_init_params *p, double *kbtnow);

/* The species' velocity distributions (VDIST codes, one per species; all
 * RANDVEL, the reference's JSON default, until set).  A particle that
 * exceeds the bounce limit at the walls is given a fresh velocity of its
 * species' distribution (bc.c:1477-1488).  mpcd_init_state sets them from
 * its parameters. */
int mpcd_set_species_vdist(mpcd_handle *h, const int *vdist);

/* Volume accessible to species 'species': the box volume (XYZ[2] = 1 in 2D)
 * less the parts where some wall the species interacts with has W < 0.
 * The reference estimates it by Monte Carlo with 1000 points per unit volume
 * (accessibleVolume, init.c:954-989); with axis-aligned planar walls it is a
 * product of per-axis intervals, computed here exactly.  Host only: no
 * device work. */
int mpcd_accessible_volume(const mpcd_config *cfg, int species, double *vol);

/* Copy the particle state back in the caller's original particle order. */
int mpcd_download_state(mpcd_handle *h, double *Q, double *V, double *U);

/* The species id of every particle, in the caller's original order. */
int mpcd_download_species(mpcd_handle *h, int *spid);

/* The handle's configuration, with gndnst the global number density in use
 * (given, or computed at the last upload). */
int mpcd_get_config(const mpcd_handle *h, mpcd_config *cfg);

/* Number of particles in the handle's state. */
int mpcd_particle_count(const mpcd_handle *h, int *n);

/* Strided counterpart of mpcd_download_state: writes the Q and V fields of
 * each record and, for a nematic state (lc != 0) with off_U != (size_t)-1,
 * the U field (the orientation, third component 0 in 2D); other bytes of the
 * records are left as they are. */
int mpcd_download_particles_strided(mpcd_handle *h, void *base, size_t stride,
                                    size_t off_Q, size_t off_V, size_t off_U);

/* Enqueue nsteps timesteps with step numbers step0, step0+1, ...  The step
 * number keys every random draw.  Asynchronous on the handle's stream. */
int mpcd_step(mpcd_handle *h, int nsteps, uint32_t step0);

/* Drop-in for one call of timestep() (mpc.c:4496): one step numbered
 * 'runtime', then the step's global measures copied to the host:
 * AVNOW = avVel (therm.c:362-367), KBTNOW = TEMP (therm.c:209-235). */
int mpcd_timestep(mpcd_handle *h, uint32_t runtime, double AVNOW[3],
                  double *KBTNOW);

/* nsteps timesteps numbered step0, step0+1, ... (as mpcd_step) with every
 * step's global measures returned: kbtnow[k] = TEMP and avnow[3k..3k+2] =
 * avVel of step step0 + k (therm.c:209-235, 362-367), what nsteps calls of
 * mpcd_timestep return.  The measures come back in batches, read while the
 * next batch runs, so the host does not wait for each step as it does with
 * mpcd_timestep.  Returns when the last step has finished. */
int mpcd_step_record(mpcd_handle *h, int nsteps, uint32_t step0, double *kbtnow,
                     double *avnow);

/* Global measures of the last executed step (blocks until it finishes). */
int mpcd_globals(mpcd_handle *h, double *kbtnow, double avnow[3]);

/* Re-bin on the unshifted grid and compute per-cell properties for output
 * (the re-bin + localPROP at the end of timestep, mpc.c:4936-4942), on the
 * device; only the cell arrays are copied back.  Arrays hold
 * (L0+1)(L1+1)(L2+1) cells, index (a*(L1+1)+b)*(L2+1)+c; any pointer may be
 * NULL.  vcm/cm hold 3 doubles per cell (CM = sum m Q / M, computed for
 * every operator; the reference fills it for MPC-AT+a and nematics only,
 * mpc.c:75).  The FP64 sums are added in arrival order, so they agree with
 * the reference's list-order sums to rounding. */
int mpcd_cell_props(mpcd_handle *h, int *pop, double *mass, double *vcm,
                    double *cm);

/* Parity check (no counterpart in the reference): the population of every
 * cell of the NEXT step's shifted grid (step last + 1, (L+1)^D cells in the
 * layout of mpcd_cell_props), exactly as the step's own kernels hold it for
 * that step's collision (the counting sort's offsets, or the resident
 * families' population sums).  They are the cell lists the reference's
 * bin() (mpc.c:948-992) builds at the start of that step.
 * MPCD_ERR_STATE before the first step after an upload. */
int mpcd_debug_cell_counts(mpcd_handle *h, int *pop);

/* Transverse momentum modes of the smallest wavevectors (an analysis
 * helper with no counterpart in the reference): for each ordered pair of
 * axes (a, b), a != b (b outer, a inner), j = sum_i v_i,a exp(-2 pi i
 * x_i,b / L_b), written as (Re, Im) pairs to out[0 .. 2*nmodes-1] (at most
 * 12 doubles; nmodes = 6 in 3D, 2 in 2D).  Their decay measures the
 * kinematic viscosity. */
int mpcd_transverse_modes(mpcd_handle *h, double *out, int *nmodes);

/* Error counters accumulated so far. */
int mpcd_get_status(mpcd_handle *h, mpcd_status *st);

/* Use the caller's CUDA stream (cudaStream_t passed as void*) from now on. */
int mpcd_set_stream(mpcd_handle *h, void *stream);

/* Number of kernel launches the last mpcd_step issued per step. */
int mpcd_launches_per_step(mpcd_handle *h);

/* Timing of the step's particle pass (the kernel that reads and writes every
 * particle; no counterpart in the reference): while enabled, each step
 * records a CUDA event pair around that launch on the handle's stream.
 * mpcd_kernel_time synchronizes, returns the summed duration (ms) and the
 * number of timed launches since timing was enabled or last queried, and
 * starts a new interval. */
int mpcd_set_timing(mpcd_handle *h, int enable);
int mpcd_kernel_time(mpcd_handle *h, double *ms_total, int *launches);

/* Execution strategy of the per-step pipeline (no counterpart in the
 * reference, which has one serial path):
 *   MPCD_STRATEGY_SCATTER   fused cell kernel writes in place, a scatter
 *                           kernel reorders the state (one pass of compute);
 *   MPCD_STRATEGY_RECOMPUTE the fused cell kernel runs twice, first only
 *                           counting the next step's cells, then writing each
 *                           particle directly to its sorted slot (fewer
 *                           bytes moved, twice the arithmetic).
 * strategy -1 restores the default; tile_particles (0 = default) sets the
 * average number of particles staged per thread block. */
#define MPCD_STRATEGY_SCATTER 0
#define MPCD_STRATEGY_RECOMPUTE 1
int mpcd_set_strategy(mpcd_handle *h, int strategy, int tile_particles);

/* Cell-kernel family (no counterpart in the reference).  For the SRD
 * operator without phantom walls:
 *   MPCD_KERNEL_RESIDENT the particles stay in place: a thread-per-cell
 *                      pass turns the cell sums into each cell's
 *                      centre-of-mass velocity and rotation, and a
 *                      thread-per-particle pass collides, streams, writes the
 *                      particle back and adds it to the next step's cell
 *                      sums.  Mixed precision (the default there): sums in
 *                      64-bit fixed point, results independent of the
 *                      particle order.  FP64: FP64 atomic sums, which agree
 *                      with the sorted-order sums to rounding;
 *   MPCD_KERNEL_SPLIT  the same two passes over a state kept sorted by cell,
 *                      re-binned every step;
 *   MPCD_KERNEL_GROUP  one warp per group of 32 cells does both, staging the
 *                      group in shared memory;
 *   MPCD_KERNEL_TILE   one block per tile of cells (the kernel every other
 *                      operator uses).
 * For every operator but the nematic ones, FP64 form:
 *   MPCD_KERNEL_PERSIST one persistent cooperative launch (a block per SM at
 *                      most) holds the whole box in its blocks' shared memory
 *                      and runs all the steps of an mpcd_step call, the
 *                      blocks meeting at a grid barrier twice per step; for
 *                      small boxes, whose steps are otherwise bound by
 *                      launch latency.  mpcd_step returns
 *                      MPCD_ERR_UNSUPPORTED when the box does not fit.
 * MPCD_KERNEL_AUTO picks PERSIST for FP64 boxes of at most two particles per
 * thread of the launch (about 75,000 particles on a B200), RESIDENT for other
 * SRD boxes without phantom walls, and TILE elsewhere. */
#define MPCD_KERNEL_AUTO 0
#define MPCD_KERNEL_TILE 1
#define MPCD_KERNEL_GROUP 2
#define MPCD_KERNEL_SPLIT 3
#define MPCD_KERNEL_RESIDENT 4
#define MPCD_KERNEL_PERSIST 5
int mpcd_set_kernel(mpcd_handle *h, int kernel);

/* MPCD_KERNEL_RESIDENT re-sorts the state by cell every 'steps' steps
 * (default 30) to keep particles that are close in space close in memory;
 * the sort changes no result, only the speed.  The call starts a new cycle:
 * the next step re-sorts.  No counterpart in the reference. */
int mpcd_set_sort_interval(mpcd_handle *h, int steps);

/* ---------------------------------------------------------------------
 * Autotuner (no counterpart in the reference, which has one serial path).
 * mpcd_autotune times the execution plans that apply to the handle's
 * configuration on its current state -- kernel family, write-out strategy,
 * tile size, re-sort interval -- for trial_steps steps each (0: 60) after 3
 * warm-up steps, applies the fastest, and restores the state, error counters
 * and step bookkeeping, so that the trajectory continues as if the call had
 * not been made (its draws are keyed by the caller's step numbers).  With a
 * cache_path (may be NULL) the choice is looked up first, by device name and
 * workload (mpcd_tune_key), and stored after a tuning; a cached choice is
 * applied without trials.  Every plan gives the same results to the form's
 * rounding. */
typedef struct mpcd_tune_choice {
    int kernel;          /* MPCD_KERNEL_*                                    */
    int strategy;        /* MPCD_STRATEGY_*, -1 for the default              */
    int tile_particles;  /* particles per tile, 0 for the default            */
    int sort_interval;   /* steps between re-sorts (resident families)       */
    double us_per_step;  /* measured step time of the chosen plan            */
    int from_cache;      /* 1: taken from the cache file without trials      */
    int candidates;      /* plans timed (0 when taken from the cache)        */
} mpcd_tune_choice;
int mpcd_autotune(mpcd_handle *h, int trial_steps, const char *cache_path,
                  mpcd_tune_choice *out);
/* The cache key of a workload on a device (needs no GPU): device name, dim,
 * box, particle count, operator, nematic switch, precision, walls, species,
 * gravity.  MPCD_ERR_SIZE if it does not fit in len bytes. */
int mpcd_tune_key(const mpcd_config *cfg, int n, const char *device, char *key,
                  size_t len);
/* Cache file access (needs no GPU): lookup returns 1 and fills *out if the
 * key has an entry (the last one), 0 if not; store appends an entry. */
int mpcd_tune_cache_lookup(const char *path, const char *key,
                           mpcd_tune_choice *out);
int mpcd_tune_cache_store(const char *path, const char *key,
                          const mpcd_tune_choice *c);

/* ---------------------------------------------------------------------
 * Ensembles: many independent periodic 3D SRD boxes of different sizes
 * stepped together (mixed precision).  No counterpart in the reference,
 * which runs one box per process.  Every kernel of a step runs once for the
 * whole ensemble, driven by per-box offset tables; the step counter lives in
 * device memory and each step is one replay of a captured CUDA graph.  Box b
 * uses the generator key (seeds[b], replica b): its trajectory equals, bit
 * for bit, that of a single-box handle (MPCD_KERNEL_RESIDENT) created with
 * seed = seeds[b] and replica = b.
 * base: dim 3, MPCD_COLL_ARBAXIS, one species, no gravity, MPCD_PREC_MIXED;
 * its L and walls are ignored (every box is periodic).  L holds 3 sizes per
 * box; seeds may be NULL (base->seed for every box). */
typedef struct mpcd_batch mpcd_batch;
int mpcd_batch_create(const mpcd_config *base, int nboxes, const int *L,
                      const uint64_t *seeds, mpcd_batch **out);
int mpcd_batch_destroy(mpcd_batch *b);
/* npart[b] particles per box; Q, V: the boxes' arrays concatenated in box
 * order (3 doubles per particle); step0 numbers the first step. */
int mpcd_batch_upload(mpcd_batch *b, const int *npart, const double *Q, const double *V,
                      uint32_t step0);
int mpcd_batch_step(mpcd_batch *b, int nsteps);
int mpcd_batch_download(mpcd_batch *b, double *Q, double *V);
/* per-box TEMP (kbt[b]) and avVel (avv[3b..3b+2]) of the last step */
int mpcd_batch_globals(mpcd_batch *b, double *kbt, double *avv);
int mpcd_batch_set_sort_interval(mpcd_batch *b, int steps);
int mpcd_batch_set_stream(mpcd_batch *b, void *stream);
/* particles, particle slots (with padding) and cells (with padding) */
int mpcd_batch_info(mpcd_batch *b, int *n, int *slots, int *cells);

/* One SRD timestep that allocates no memory, device or host (no
 * counterpart in the reference, whose timestep works on host memory).  For
 * callers that cannot allocate at step time: a program whose allocator owns
 * all device memory, code running under CUDA stream capture (where cudaMalloc
 * is not allowed), or a plugin that must not allocate behind its host
 * framework's memory manager.  Q and V are the caller's DEVICE arrays of n
 * particles (3 doubles each, AoS), updated in place in the caller's order;
 * globals, if not NULL, is a device array of 4 doubles receiving
 * KBTNOW and AVNOW[3] (TEMP and avVel); counters, if not NULL, is a device
 * array of MPCD_NOALLOC_COUNTERS uint64 to which the step ADDS its error
 * counts (escaped, bounce_limit, nonfinite, as in mpcd_status), so a caller
 * that zeroes it once accumulates over calls.  cfg must select the SRD
 * operator (MPCD_COLL_ARBAXIS) in FP64 form with one species, without
 * phantom walls or nematic order (MPCD_ERR_UNSUPPORTED otherwise).
 * All scratch is one fixed device array of this library (11.6 MiB, held on
 * every GPU that loads it until exit), so n is limited to
 * MPCD_NOALLOC_MAX_PARTICLES and the (L+1)^D cell grid to
 * MPCD_NOALLOC_MAX_CELLS; larger sizes return MPCD_ERR_SIZE.  The first call
 * in a CUDA context (on each device, and again after a device reset) looks up
 * the array's device address; make that first call before any stream
 * capture.  Calls share the array: work of two calls that overlaps on the GPU
 * races and must be serialised by the caller.  stream is a cudaStream_t
 * (NULL: the default stream); the call is asynchronous. */
#define MPCD_NOALLOC_MAX_PARTICLES 65536
#define MPCD_NOALLOC_MAX_CELLS 32768
#define MPCD_NOALLOC_COUNTERS 3
int mpcd_srd_step_noalloc(const mpcd_config *cfg, int n, double *Q, double *V,
                          uint32_t step, double *globals, unsigned long long *counters,
                          void *stream);

/* ---- output fields ----------------------------------------------------
 * Per-species populations of the end-of-step cells (as mpcd_cell_props
 * re-bins them): counts[s * ncells + c], cells of the (L+1)^D grid in
 * row-major order; with one species, the cell populations. */
int mpcd_cell_species(mpcd_handle *h, int *counts);

/* The flow field's running sum (localFLOW + sumFLOW, mpc.c:226-246, which
 * the reference runs after every step while flow output is on): enable = 1
 * starts an empty sum (and every following step adds the end-of-step cell
 * velocities to it), 0 stops and frees it. */
int mpcd_flow_enable(mpcd_handle *h, int enable);

/* Copy the flow sum (3 doubles per cell of the (L+1)^D grid) and the number
 * of steps in it; reset = 1 empties it, as flowout does after writing
 * (pout.c:1695).  MPCD_ERR_STATE when the flow sum is off. */
int mpcd_flow_read(mpcd_handle *h, double *flow, long long *nsteps, int reset);

/* Sum over the particles of m v^2 / 2 (enout's MPCD_kin, pout.c:1393-1399). */
int mpcd_kinetic_energy(mpcd_handle *h, double *ke);

/* The reference's output files, printed from host arrays as its writers
 * print them (cells of the L^D box in x -> y -> z order; arrays over the
 * (L+1)^D grid as the calls above return them).  header = 1 creates the
 * file with the reference's banner and column header (openBasic,
 * init.c:51-63); header = 0 appends one block.  t is the time printed
 * (runtime * dt, as outputResults passes it). */
int mpcd_write_coarse(const char *path, const mpcd_config *cfg, double t, const int *pop,
                      const double *vcm, const int *spc, int header);      /* coarseout */
int mpcd_write_velfield(const char *path, const mpcd_config *cfg, double t, const double *vcm,
                        int header);                                       /* velout */
int mpcd_write_densityfield(const char *path, const mpcd_config *cfg, double t, const int *pop,
                            const double *mass, const int *spc, int header); /* densityout */
int mpcd_write_flowfield(const char *path, const mpcd_config *cfg, double t, const double *flow,
                         int interval, int header);                        /* flowout */
int mpcd_write_avvel(const char *path, double t, const double avnow[3], double kbtnow,
                     const double grad[9], int header);          /* avveloutWithGradVel */
int mpcd_write_energy(const char *path, double t, double kinetic, double kbtnow,
                      int header);                                         /* enout */

/* The velocity gradient of localVelGrad (lc.c:2054-2162: D3Q15 or D2Q9
 * weights over the bulk, edges copied from their inner neighbour) from the
 * cell velocities, into E (9 doubles per cell of the (L+1)^D grid, zero at
 * first; entries outside the bulk and the copies, corners of the extra
 * layer, keep what they held, as the reference's cells do), and its mean
 * over the L^D box (grad, row-major; may be NULL), what avVel.dat prints. */
int mpcd_vel_grad(const mpcd_config *cfg, const double *vcm, double *E, double grad[9]);

/* avVel (therm.c:362-367) of cell velocities: their sum over the (L+1)^D
 * grid / VOL, the AVNOW that outputResults recomputes after its re-bin and
 * prints in avVel.dat. */
int mpcd_av_vel(const mpcd_config *cfg, const double *vcm, double avnow[3]);

/* ---- checkpoints in the reference's format ----------------------------
 * The reference checkpoints a run as text: checkpoint (pout.c:2325-2396)
 * writes, and readchckpnt (read.c:669-834) reads, the run's counters, input
 * parameters, output flags, species, walls, every particle (S_flag, SPID, q,
 * Q, V, U, T) and the swimmers.  An mpcd_ckpt holds every field of such a
 * file.  The library reads the fields it uses (configuration, counters,
 * particles), replaces them from a handle, and carries all others through
 * unchanged, so a run can move between the reference program and this
 * library in either direction.  Host only, except the two calls that take a
 * handle. */
typedef struct mpcd_ckpt mpcd_ckpt;

/* Counters and global measures of a checkpoint (the first lines of the
 * file): in.simSteps, in.warmupSteps, runtime, warmtime, KBTNOW, AVV,
 * AVNOW. */
typedef struct mpcd_ckpt_run {
    int sim_steps, warmup_steps;
    int runtime, warmtime;
    double kbtnow;
    double avv[3], avnow[3];
} mpcd_ckpt_run;

/* Parse a checkpoint file; *out is freed with mpcd_ckpt_free.  MPCD_ERR_ARG
 * for a file that ends early or holds a field that is not a number. */
int mpcd_ckpt_read(const char *path, mpcd_ckpt **out);

/* A checkpoint of cfg with no particles: the fields the library does not
 * own take the values a JSON run with the defaults of readJson would hold
 * (no thermostat, no outputs, static walls, no swimmers). */
int mpcd_ckpt_create(const mpcd_config *cfg, mpcd_ckpt **out);

int mpcd_ckpt_free(mpcd_ckpt *ck);

/* Write the checkpoint.  precise = 0 prints every field as checkpoint does
 * (doubles with "%lf", six decimals): a file read and written again is
 * identical byte for byte.  precise = 1 prints doubles with 17 significant
 * digits, which readchckpnt reads back exactly (a lossless checkpoint in the
 * same layout). */
int mpcd_ckpt_write(const mpcd_ckpt *ck, const char *path, int precise);

/* The configuration the checkpoint describes (seed = in.seed, gndnst =
 * GnDNST, capacity 0).  MPCD_ERR_UNSUPPORTED when the run uses something
 * outside this library: MD coupling, swimmers, a thermostat, moving,
 * rotating or non-planar walls, an external magnetic field, or another
 * collision operator. */
int mpcd_ckpt_config(const mpcd_ckpt *ck, mpcd_config *cfg);

int mpcd_ckpt_get_run(const mpcd_ckpt *ck, mpcd_ckpt_run *run);
int mpcd_ckpt_set_run(mpcd_ckpt *ck, const mpcd_ckpt_run *run);

/* Particle count, and the particles (any output may be NULL; 3 doubles per
 * vector). */
int mpcd_ckpt_count(const mpcd_ckpt *ck, int *n);
int mpcd_ckpt_particles(const mpcd_ckpt *ck, double *Q, double *V, double *U, int *spid);

/* Replace the checkpoint's particles (n of them; U and spid may be NULL for
 * zero orientations and species 0); the species populations follow.
 * Particles keep their S_flag, q and T where the count is unchanged; new
 * ones get S_flag 1 (STREAM) and zero q and T. */
int mpcd_ckpt_set_particles(mpcd_ckpt *ck, int n, const double *Q, const double *V,
                            const double *U, const int *spid);

/* The checkpoint's particles into the handle (mpcd_upload_state), as
 * initializeRecovery (init.c:2193-2215) bins them after readchckpnt. */
int mpcd_ckpt_upload(const mpcd_ckpt *ck, mpcd_handle *h);

/* The handle's particles into the checkpoint (mpcd_ckpt_set_particles with
 * the handle's positions, velocities, species and, for a nematic state,
 * orientations; an isotropic state leaves the file's orientations), and the
 * handle's GnDNST. */
int mpcd_ckpt_capture(mpcd_ckpt *ck, mpcd_handle *h);

#ifdef __cplusplus
}
#endif

#endif /* MPCD_GPU_H */
