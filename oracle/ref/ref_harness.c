/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY.  Drives the reference program's
 * own solvent timestep (NIAMH-MPCD, compiled unmodified from its sources into
 * oracle/_ref/) on state built here, so its outputs can pin the CPU oracle and
 * be committed as golden fixtures.  Nothing in the product links this file.
 *
 * Two builds of this file exist (oracle/ref/Makefile):
 *
 *  - libmpcdref.so (REF_INJECT defined): the reference's rand.c is replaced by
 *    the functions below, which hand out the counter-based draws of
 *    niamh-mpcd_b200/csrc/mpcd_rng.h.  The reference visits cells and
 *    particles in its own serial order, so the harness interposes the
 *    per-cell entry points (MPCcollision, ghostPart, LCcollision,
 *    genrand_maierSaupe) to learn which cell or particle a draw belongs to.
 *    Interposition works because the reference objects are built -fPIC with
 *    GCC's default semantic interposition: their calls to these global
 *    functions go through the PLT and resolve to the definitions here first.
 *
 *  - libmpcdref_time.so: the reference's own rand.c (Mersenne Twister) and
 *    no interposers, built -fno-semantic-interposition, to time the
 *    reference's serial timestep as the CPU baseline.
 *
 * State is built directly (positions, velocities, walls) instead of through
 * readJson, skipping accessibleVolume (init.c:954-989), which takes minutes.
 * Walls are filled as readJson fills a JSON "BC" entry (read.c:1141-1428).
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* product headers first: the reference headers define macros named e, pi
 * and real (definitions.h:73-75, md/mdtypes.h:52) */
#include "mpcd_gpu.h"
#include "mpcd_rng.h"

#include "definitions.h"
#include "SRDclss.h"
#include "mpc.h"
#include "init.h"
#include "therm.h"
#include "pout.h"
#include "read.h"
#include "lc.h"

/* reference globals (globals.h:24-65, common symbols of the core library) */
extern int DBUG, DIM, MDmode, GPOP, NSPECI, NBC, NS;
extern double VOL, GnDNST, GmDNST, GMASS;
extern int XYZ[_3D], XYZ_P1[_3D], XYZPBC[_3D], maxXYZ;
extern int BMHASSPARE;
extern double BMSPARE;

void setPBC(bc *WALL);                         /* read.c:584 */
void galileantrans(particleMPC *pp, bc WALL[], simptr simMD, spec SP[], double KBT,
                   double VEL[], int POP, int NBC, int MDmode, int dimension); /* mtools.c:673 */
double calcW(bc WALL, particleMPC P);          /* bc.c:55    */
void crossprod(double x[3], double y[3], double result[3]);          /* mtools.c:177  */
double absAngle(double v1[], double v2[], int dimension);           /* mtools.c:365  */
void rodriguesRotation(double vec[], double rotAx[], double theta); /* mtools.c:1572 */
unsigned long RandomSeedSRD(unsigned long s);  /* rand.c:293 */

/* ------------------------------------------------------------------ state */
static cell ***g_CL = NULL;
static cell *g_cells = NULL;
static particleMPC *g_pp = NULL;
static spec *g_SP = NULL;
static bc *g_WALL = NULL;
static specSwimmer *g_SS = NULL;
static inputList g_in;
static outputFlagsList g_oflags;
static outputFilesList g_ofiles;
static double g_AVNOW[3], g_AVV[3], g_avDIR[3], g_KBTNOW, g_AVS;
static int g_ncells = 0;

/* draw bookkeeping */
static uint64_t g_seed = 0;
static uint32_t g_replica = 0, g_step = 0;
enum { PH_NONE = 0, PH_COLLIDE, PH_GHOST, PH_LC, PH_INIT, PH_RETHERM, PH_ESCAPE, PH_CONE };
static int g_phase = PH_NONE;
static int g_cell = 0;
static int g_rtech = 0;  /* RTECH of the collision in progress */
static int g_ccount = 0; /* its uniform draws so far */
static int g_last = 0;   /* the particle whose thermal draws ended last */
static particleMPC *g_cursor = NULL;
static int g_comp = 0;
static uint32_t g_stream = 0; /* PH_INIT: the stream of the current draws */
static int *g_attempt = NULL; /* PH_INIT: placement attempts per particle */
static int *g_retherm = NULL; /* re-thermalisations per particle this step */
static int g_retherm_n = 0;
static int g_pid = 0;
static uint32_t g_k = 0;
static int *g_ghost = NULL;
static int g_ghost_n = 0, g_ghost_pos = 0;
static long g_unexpected = 0;

static int cell_id(const cell *c) { return (int)(c - g_cells); }

/* ------------------------------------------------------------ set-up/API */
static int g_clx = 0; /* rows of g_CL as allocated (readchckpnt rewrites XYZ_P1) */
int ref_free(void) {
    if (g_CL) {
        for (int i = 0; i < g_clx; i++) free(g_CL[i]);
        free(g_CL);
    }
    free(g_cells);
    free(g_pp);
    free(g_SP);
    free(g_WALL);
    free(g_SS);
    free(g_ghost);
    g_CL = NULL;
    g_cells = NULL;
    g_pp = NULL;
    g_SP = NULL;
    g_WALL = NULL;
    g_SS = NULL;
    g_ghost = NULL;
    return 0;
}

/* Build the reference's state from a config and particle arrays (AoS, 3
 * doubles per vector).  Returns 0 on success. */
int ref_init(const mpcd_config *cfg, int n, const double *Q, const double *V,
             const double *U, const int *spid) {
    int i, j, d;
    ref_free();
    DBUG = 0;
    DIM = cfg->dim;
    MDmode = 0;
    NS = 0;
    GPOP = n;
    NSPECI = cfg->n_species;
    NBC = cfg->n_walls;
    for (d = 0; d < 3; d++) {
        XYZ[d] = (d < DIM) ? cfg->L[d] : 1; /* read.c:1040-1044 */
        XYZ_P1[d] = XYZ[d] + 1;
    }
    VOL = 1.0;
    for (d = 0; d < DIM; d++) VOL *= XYZ[d];
    maxXYZ = (int)sqrt((double)(XYZ[0] * XYZ[0] + XYZ[1] * XYZ[1] + XYZ[2] * XYZ[2]));
    BMHASSPARE = 0;
    BMSPARE = 0.0;

    g_SP = (spec *)calloc((size_t)NSPECI, sizeof(spec));
    for (i = 0; i < NSPECI; i++) {
        const mpcd_species *s = &cfg->species[i];
        g_SP[i].MASS = s->mass;
        g_SP[i].DAMP = s->damp;
        g_SP[i].RFC = s->rfc;
        g_SP[i].TUMBLE = s->tumble;
        g_SP[i].CHIHI = s->chihi;
        g_SP[i].ACT = s->act;
        g_SP[i].MFPOT = s->mfpot;
        g_SP[i].SIGWIDTH = s->sigwidth;
        g_SP[i].SIGPOS = s->sigpos;
        g_SP[i].MINACTRATIO = s->minactratio;
        g_SP[i].LEN = 0.007;
        g_SP[i].POP = 0;
    }
    for (i = 0; i < n; i++) g_SP[spid ? spid[i] : 0].POP++;

    g_WALL = (bc *)calloc((size_t)(NBC > 0 ? NBC : 1), sizeof(bc));
    for (i = 0; i < NBC; i++) {
        const mpcd_wall *w = &cfg->walls[i];
        bc *b = &g_WALL[i];
        b->COLL_TYPE = w->coll_type;
        b->PHANTOM = w->phantom;
        b->E = -1.0;
        for (d = 0; d < 3; d++) {
            b->Q[d] = w->Q[d];
            b->A[d] = w->A[d];
            b->AINV[d] = (w->A[d] != 0.0) ? 1.0 / w->A[d] : 0.0;
            b->DVxyz[d] = w->DVxyz[d];
            b->MUxyz[d] = w->MUxyz[d];
            b->DUxyz[d] = w->DUxyz[d];
        }
        for (d = 0; d < 4; d++) b->P[d] = 1.0;
        b->ROTSYMM[0] = 4.0;
        b->ROTSYMM[1] = 4.0;
        b->R = w->R;
        b->INV = w->inv;
        b->DN = w->DN;
        b->DT = w->DT;
        b->DVN = w->DVN;
        b->DVT = w->DVT;
        b->MVN = w->MVN;
        b->MVT = w->MVT;
        b->MUN = w->MUN;
        b->MUT = w->MUT;
        b->KBT = 1.0;
        b->MASS = 1.0;
        b->DSPLC = 0;
        b->REORIENT = 0; /* init.c:2063-2065: static walls with O = 0 */
        for (j = 0; j < MAXSPECI; j++) b->INTER[j] = w->inter[j];
        b->INTER[MAXSPECI] = BCON;
        b->INTER[MAXSPECI + 1] = BCON;
        /* PLANAR flag as read.c:1417-1428 */
        b->PLANAR = 0;
        if ((b->A[0] != 0.0) + (b->A[1] != 0.0) + (b->A[2] != 0.0) == 1) b->PLANAR = 1;
    }
    for (d = 0; d < 3; d++) XYZPBC[d] = 0;
    for (i = 0; i < NBC; i++) setPBC(&g_WALL[i]);

    g_pp = (particleMPC *)calloc((size_t)(n > 0 ? n : 1), sizeof(particleMPC));
    for (i = 0; i < n; i++) {
        for (d = 0; d < 3; d++) {
            g_pp[i].Q[d] = Q[3 * i + d];
            g_pp[i].V[d] = V[3 * i + d];
            g_pp[i].U[d] = U ? U[3 * i + d] : 0.0;
        }
        g_pp[i].SPID = spid ? spid[i] : 0;
        g_pp[i].S_flag = STREAM;
    }

    g_ncells = XYZ_P1[0] * XYZ_P1[1] * XYZ_P1[2];
    g_cells = (cell *)calloc((size_t)g_ncells, sizeof(cell));
    g_CL = (cell ***)malloc((size_t)XYZ_P1[0] * sizeof(cell **));
    g_clx = XYZ_P1[0];
    for (i = 0; i < XYZ_P1[0]; i++) {
        g_CL[i] = (cell **)malloc((size_t)XYZ_P1[1] * sizeof(cell *));
        for (j = 0; j < XYZ_P1[1]; j++)
            g_CL[i][j] = g_cells + ((size_t)i * XYZ_P1[1] + j) * XYZ_P1[2];
    }
    g_ghost = (int *)malloc((size_t)g_ncells * sizeof(int));
    g_SS = (specSwimmer *)calloc(1, sizeof(specSwimmer));

    memset(&g_in, 0, sizeof(g_in));
    g_in.KBT = cfg->kbt;
    g_in.dt = cfg->dt;
    g_in.RA = cfg->rot_ang;
    g_in.C = cos(cfg->rot_ang); /* initvar, init.c:1194-1195 */
    g_in.S = sin(cfg->rot_ang);
    g_in.RTECH = cfg->coll_op;
    g_in.FRICCO = cfg->fricco;
    g_in.LC = cfg->lc;
    g_in.GALINV = cfg->galinv;
    g_in.TSTECH = NOTHERM;
    g_in.TAU = cfg->relax;
    g_in.noHI = HION;
    g_in.inCOMP = INCOMPOFF;
    g_in.MULTIPHASE = MPHOFF;
    g_in.seed = (unsigned long)cfg->seed;
    for (d = 0; d < 3; d++) g_in.GRAV[d] = cfg->grav[d];
    g_in.GRAV_FLAG = (fabs(g_in.GRAV[0]) >= TOL || fabs(g_in.GRAV[1]) >= TOL ||
                      fabs(g_in.GRAV[2]) >= TOL);
    memset(&g_oflags, 0, sizeof(g_oflags));
    memset(&g_ofiles, 0, sizeof(g_ofiles));
    for (d = 0; d < 3; d++) g_AVNOW[d] = g_AVV[d] = g_avDIR[d] = 0.0;
    g_KBTNOW = 0.0;
    g_AVS = 0.0;

    g_seed = cfg->seed;
    g_replica = cfg->replica;
#ifndef REF_INJECT
    RandomSeedSRD((unsigned long)(cfg->seed ? cfg->seed : 1));
#endif
    binin(g_pp, g_CL);
    localPROP(g_CL, g_SP, *g_SS, g_in.RTECH, g_in.LC);
    globalDensities(g_CL, g_SP);
    if (cfg->gndnst > 0.0) GnDNST = cfg->gndnst;
    return 0;
}

double ref_gndnst(void) { return GnDNST; }

/* The reference's analytic transport coefficients, theory_trans
 * (init.c:800-942), for one species of mass m at number density n in DIM
 * dimensions: returns the kinematic viscosity VISC / (n m) (the value
 * synopsis.dat prints), *sdiff the self-diffusion coefficient and *mfp the
 * mean free path.  The globals it reads (DIM, GPOP) are set for the call
 * and restored. */
double ref_theory_visc(int rtech, int dim, double n, double ra, double dt, double kbt,
                       double m, double *sdiff, double *mfp) {
    double MFP = 0, VISC = 0, THERMD = 0, SDIFF = 0, SOS = 0;
    const int dim0 = DIM, gpop0 = GPOP;
    DIM = dim;
    GPOP = 1000;
    theory_trans(&MFP, &VISC, &THERMD, &SDIFF, &SOS, ra, 0.0, kbt, dt, m * (double)GPOP, rtech,
                 n, n * m, 0, NULL);
    DIM = dim0;
    GPOP = gpop0;
    if (sdiff) *sdiff = SDIFF;
    if (mfp) *mfp = MFP;
    return VISC / (n * m);
}
int ref_ncells(void) { return g_ncells; }

/* The reference's initial particle state: setcoord (init.c:1565-1600),
 * galileantrans when rframe and GPOP > 2, TEMP and the VSC scaling, in the
 * order of initializeSIM (init.c:2092-2170), then the first binning so that
 * ref_step can continue from it.  With the injected draws the positions,
 * velocities and orientations use the counter-based streams at step 0.
 * Writes Q, V, U (3 doubles per particle), spid and TEMP after scaling. */
int ref_init_state(const mpcd_config *cfg, const mpcd_init_params *p, double *Q, double *V,
                   double *U, int *spid, double *kbt_after) {
    int n = 0, i, s, d, k = 0;
    for (s = 0; s < cfg->n_species; s++) n += p->population[s];
    int *sp = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    double *z = (double *)calloc((size_t)(n > 0 ? n : 1) * 3, sizeof(double));
    for (s = 0; s < cfg->n_species; s++)
        for (i = 0; i < p->population[s]; i++) sp[k++] = s;
    ref_init(cfg, n, z, z, NULL, sp);
    free(z);
    free(sp);
    for (s = 0; s < NSPECI; s++) {
        g_SP[s].QDIST = PRF;
        g_SP[s].VDIST = p->vdist[s];
        g_SP[s].ODIST = p->odist[s];
    }
    free(g_attempt);
    g_attempt = (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int));
    char dir[4] = "";
    g_step = 0;
    g_phase = PH_INIT;
    setcoord(dir, g_SP, g_pp, g_in.KBT, g_AVV, g_WALL, NULL, 0, g_in.LC);
    g_phase = PH_NONE;
    free(g_attempt);
    g_attempt = NULL;
    if (p->rframe && GPOP > 2)
        galileantrans(g_pp, g_WALL, NULL, g_SP, g_in.KBT, g_AVV, GPOP, NBC, 0, DIM);
    g_KBTNOW = TEMP(g_pp, g_SP, g_WALL, g_AVV);
    scaleT(g_in.KBT, g_KBTNOW, g_in.dt, g_in.TAU, g_AVV, g_AVNOW, VSC, g_SP, g_in.LC, g_WALL,
           g_pp, g_CL);
    g_KBTNOW = TEMP(g_pp, g_SP, g_WALL, g_AVV);
    if (kbt_after) *kbt_after = g_KBTNOW;
    for (i = 0; i < n; i++) {
        for (d = 0; d < 3; d++) {
            Q[3 * i + d] = g_pp[i].Q[d];
            V[3 * i + d] = g_pp[i].V[d];
            if (U) U[3 * i + d] = g_pp[i].U[d];
        }
        spid[i] = g_pp[i].SPID;
    }
    /* the state's first binning, as ref_init does for uploaded particles */
    for (i = 0; i < g_ncells; i++) g_cells[i].pp = NULL;
    binin(g_pp, g_CL);
    localPROP(g_CL, g_SP, *g_SS, g_in.RTECH, g_in.LC);
    globalDensities(g_CL, g_SP);
    if (cfg->gndnst > 0.0) GnDNST = cfg->gndnst;
    for (d = 0; d < 3; d++) g_AVV[d] = 0.0;
    return 0;
}

/* The reference's own checkpoint writer (checkpoint, pout.c:2325-2396) on
 * the current state, with run counters runtime and warmtime. */
int ref_checkpoint_write(const char *path, int runtime, int warmtime) {
    if (!g_pp) return -1;
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    kinTheory *th = (kinTheory *)calloc((size_t)(NSPECI > 0 ? NSPECI : 1), sizeof(kinTheory));
    kinTheory thg;
    memset(&thg, 0, sizeof(thg));
    g_in.simSteps = 1000;
    g_in.stepsMD = 20;
    checkpoint(f, g_in, g_SP, g_pp, 0, g_WALL, g_oflags, runtime, warmtime, 0.0, g_AVS, g_avDIR,
               0.0, 0.0, g_KBTNOW, g_AVV, g_AVNOW, th, thg, *g_SS, NULL);
    fclose(f);
    free(th);
    return 0;
}

/* The reference's own checkpoint reader (readchckpnt, read.c:669-834) on a
 * file: the configuration as the reference holds it after reading (into
 * cfg), the particle count, run counters, KBTNOW and AVNOW; the particles
 * stay for ref_checkpoint_particles.  Overwrites the reference's globals. */
static particleMPC *g_rd = NULL;
static int g_rd_n = 0;
int ref_checkpoint_read(const char *path, mpcd_config *cfg, int *n, int *runtime, int *warmtime,
                        double *kbtnow, double *avnow) {
    inputList in;
    memset(&in, 0, sizeof(in));
    in.chckpntInputFile = (char *)path;
    spec *SP = NULL;
    particleMPC *pp = NULL;
    cell ***CL = NULL;
    int md = 0, i, j, d;
    bc *WALL = (bc *)calloc(MAXBC, sizeof(bc));
    outputFlagsList out;
    memset(&out, 0, sizeof(out));
    kinTheory *th = (kinTheory *)calloc(MAXSPECI, sizeof(kinTheory));
    kinTheory thg;
    double AVVEL, AVS, avDIR[3], S4, stdN, AVV[3];
    specSwimmer ss;
    memset(&ss, 0, sizeof(ss));
    swimmer *sw = NULL;
    readchckpnt(&in, &SP, &pp, &CL, &md, &WALL, &out, runtime, warmtime, &th, &thg, &AVVEL, &AVS,
                avDIR, &S4, &stdN, kbtnow, AVV, avnow, &ss, &sw);
    memset(cfg, 0, sizeof(*cfg));
    cfg->dim = DIM;
    for (d = 0; d < 3; d++) {
        cfg->L[d] = XYZ[d];
        cfg->grav[d] = in.GRAV[d];
    }
    cfg->dt = in.dt;
    cfg->kbt = in.KBT;
    cfg->coll_op = in.RTECH;
    cfg->fricco = in.FRICCO;
    cfg->relax = in.TAU;
    cfg->lc = in.LC;
    cfg->rot_ang = in.RA;
    cfg->galinv = in.GALINV;
    cfg->gndnst = GnDNST;
    cfg->seed = (uint64_t)in.seed;
    cfg->n_species = NSPECI;
    for (i = 0; i < NSPECI && i < MPCD_MAX_SPECIES; i++) {
        mpcd_species *s = &cfg->species[i];
        s->mass = SP[i].MASS;
        s->damp = SP[i].DAMP;
        s->rfc = SP[i].RFC;
        s->tumble = SP[i].TUMBLE;
        s->chihi = SP[i].CHIHI;
        s->act = SP[i].ACT;
        s->mfpot = SP[i].MFPOT;
        s->sigwidth = SP[i].SIGWIDTH;
        s->sigpos = SP[i].SIGPOS;
        s->minactratio = SP[i].MINACTRATIO;
    }
    cfg->n_walls = NBC;
    for (i = 0; i < NBC && i < MPCD_MAX_WALLS; i++) {
        mpcd_wall *w = &cfg->walls[i];
        const bc *b = &WALL[i];
        for (d = 0; d < 3; d++) {
            w->A[d] = b->A[d];
            w->Q[d] = b->Q[d];
            w->DVxyz[d] = b->DVxyz[d];
            w->MUxyz[d] = b->MUxyz[d];
            w->DUxyz[d] = b->DUxyz[d];
        }
        w->R = b->R;
        w->inv = b->INV;
        w->phantom = b->PHANTOM;
        w->coll_type = b->COLL_TYPE;
        w->DN = b->DN;
        w->DT = b->DT;
        w->DVN = b->DVN;
        w->DVT = b->DVT;
        w->MVN = b->MVN;
        w->MVT = b->MVT;
        w->MUN = b->MUN;
        w->MUT = b->MUT;
        for (j = 0; j < MPCD_MAX_SPECIES; j++) w->inter[j] = b->INTER[j];
    }
    free(g_rd);
    g_rd = pp;
    g_rd_n = GPOP;
    *n = GPOP;
    for (i = 0; i < XYZ_P1[0]; i++) {
        for (j = 0; j < XYZ_P1[1]; j++) free(CL[i][j]);
        free(CL[i]);
    }
    free(CL);
    free(SP);
    free(WALL);
    free(th);
    free(sw);
    return 0;
}

int ref_checkpoint_particles(double *Q, double *V, double *U, int *spid) {
    for (int i = 0; i < g_rd_n; i++) {
        for (int d = 0; d < 3; d++) {
            if (Q) Q[3 * i + d] = g_rd[i].Q[d];
            if (V) V[3 * i + d] = g_rd[i].V[d];
            if (U) U[3 * i + d] = g_rd[i].U[d];
        }
        if (spid) spid[i] = g_rd[i].SPID;
    }
    return 0;
}

/* The species' VDIST (the distribution of a re-thermalised velocity). */
int ref_set_vdist(const int *vdist) {
    for (int s = 0; s < NSPECI; s++) g_SP[s].VDIST = vdist[s];
    return 0;
}

/* Flow output on: timestep() then sums every step's cell velocities into
 * FLOW (localFLOW + sumFLOW, mpc.c:4946-4951). */
int ref_set_flow(int on) {
    g_oflags.FLOWOUT = on ? OUT : 0;
    return 0;
}
int ref_get_flow(double *flow) {
    for (int c = 0; c < g_ncells; c++)
        for (int d = 0; d < 3; d++) flow[3 * c + d] = g_cells[c].FLOW[d];
    return 0;
}
int ref_get_cell_species(int *spc) {
    for (int s = 0; s < NSPECI; s++)
        for (int c = 0; c < g_ncells; c++) spc[(size_t)s * g_ncells + c] = g_cells[c].SP[s];
    return 0;
}

/* The reference's own writers of the cell fields and global measures, as
 * outputResults (pout.c:2518-2600) calls them after a step: re-bin,
 * localPROP, avVel, then coarseout, velout, densityout, flowout (which
 * empties FLOW), localVelGrad + avveloutWithGradVel, enout.  Files in dir
 * (ending in '/'), created with their headers when header is set. */
static FILE *ref_open(void (*opener)(FILE **, char *, char *, char *), const char *dir,
                      const char *name, int header) {
    FILE *f = NULL;
    char d[4096], nm[256], ext[8] = ".dat";
    snprintf(d, sizeof d, "%s", dir);
    snprintf(nm, sizeof nm, "%s", name);
    if (header) {
        opener(&f, d, nm, ext);
    } else {
        char path[4400];
        snprintf(path, sizeof path, "%s%s.dat", dir, name);
        f = fopen(path, "a");
    }
    return f;
}
int ref_write_outputs(const char *dir, int runtime, int flow_interval, int header) {
    if (!g_pp) return -1;
    const double t = runtime * g_in.dt;
    FILE *f;
    int a, b, c, i, j;
    bin(g_CL, g_SP, g_WALL, g_in.KBT, g_in.LC, 0);
    localPROP(g_CL, g_SP, *g_SS, g_in.RTECH, g_in.LC);
    avVel(g_CL, g_AVNOW);
    if (!(f = ref_open(opencoarse, dir, "coarsegrain", header))) return -1;
    coarseout(f, t, g_CL);
    fclose(f);
    if (!(f = ref_open(openvel, dir, "velfield", header))) return -1;
    velout(f, g_CL, t);
    fclose(f);
    if (!(f = ref_open(opendensity, dir, "densityfield", header))) return -1;
    densityout(f, g_CL, t);
    fclose(f);
    if (flow_interval > 0) {
        if (!(f = ref_open(openflow, dir, "flowfield", header))) return -1;
        flowout(f, g_CL, flow_interval, t);
        fclose(f);
    }
    double grad[3][3];
    localVelGrad(g_CL);
    for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++) grad[i][j] = 0.;
    for (a = 0; a < XYZ[0]; a++)
        for (b = 0; b < XYZ[1]; b++)
            for (c = 0; c < XYZ[2]; c++)
                for (i = 0; i < 3; i++)
                    for (j = 0; j < 3; j++) grad[i][j] += g_CL[a][b][c].E[i][j];
    for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++) grad[i][j] /= VOL;
    if (!(f = ref_open(openavvel, dir, "avVel", header))) return -1;
    avveloutWithGradVel(f, t, g_AVNOW, g_KBTNOW, grad);
    fclose(f);
    if (!(f = ref_open(openenergy, dir, "energy", header))) return -1;
    enout(f, g_pp, g_SP, g_WALL, t, g_KBTNOW, 0.0);
    fclose(f);
    return 0;
}

/* The reference's Monte Carlo accessible volume (init.c:954-989) of species
 * 'spid' for the walls of the last ref_init; with the reference's own
 * generator (libmpcdref_time.so) it is the value readJson computes. */
double ref_accessible_volume(int spid) { return accessibleVolume(g_WALL, spid); }
long ref_unexpected_draws(void) { return g_unexpected; }

/* One call of the reference timestep() (mpc.c:4496) numbered 'step'. */
int ref_step(uint32_t step) {
    if (!g_pp) return -1;
    g_step = step;
    if (g_retherm_n != GPOP) {
        free(g_retherm);
        g_retherm = (int *)calloc((size_t)(GPOP > 0 ? GPOP : 1), sizeof(int));
        g_retherm_n = GPOP;
    } else if (g_retherm) {
        memset(g_retherm, 0, (size_t)GPOP * sizeof(int));
    }
    timestep(g_CL, g_pp, g_SP, g_WALL, NULL, g_SS, NULL, g_AVNOW, g_AVV, g_avDIR,
             g_in, &g_KBTNOW, &g_AVS, (int)step, 0, g_oflags, g_ofiles);
    return 0;
}

/* Run nsteps and return the elapsed wall time in seconds (CPU baseline). */
double ref_run_timed(int nsteps, uint32_t step0) {
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int s = 0; s < nsteps; s++) ref_step(step0 + (uint32_t)s);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

int ref_get_particles(double *Q, double *V, double *U) {
    for (int i = 0; i < GPOP; i++)
        for (int d = 0; d < 3; d++) {
            if (Q) Q[3 * i + d] = g_pp[i].Q[d];
            if (V) V[3 * i + d] = g_pp[i].V[d];
            if (U) U[3 * i + d] = g_pp[i].U[d];
        }
    return 0;
}

int ref_get_globals(double *kbtnow, double *avnow) {
    *kbtnow = g_KBTNOW;
    for (int d = 0; d < 3; d++) avnow[d] = g_AVNOW[d];
    return 0;
}

/* Cell properties as left by the last timestep (re-bin + localPROP on the
 * unshifted grid, mpc.c:4936-4942), cells in (a,b,c) row-major order. */
int ref_get_cells(int *pop, double *mass, double *vcm, double *cm) {
    for (int c = 0; c < g_ncells; c++) {
        if (pop) pop[c] = g_cells[c].POP;
        if (mass) mass[c] = g_cells[c].MASS;
        for (int d = 0; d < 3; d++) {
            if (vcm) vcm[3 * c + d] = g_cells[c].VCM[d];
            if (cm) cm[3 * c + d] = g_cells[c].CM[d];
        }
    }
    return 0;
}

#ifdef REF_INJECT
/* ======================================================================
 * Replacement of mpcd/subroutines/rand.c: every symbol another reference
 * translation unit calls, serving the counter-based draws.
 * ====================================================================== */
static float next_normal(void) {
    float g = 0.0f;
    if (g_phase == PH_INIT) {
        g = mpcd_rng_normal(g_seed, g_replica, 0u, MPCD_STREAM_INIT_VEL, (uint32_t)g_pid,
                            (uint32_t)g_comp++);
    } else if (g_phase == PH_RETHERM) {
        g = mpcd_rng_normal(g_seed, g_replica, g_step, MPCD_STREAM_RETHERM, (uint32_t)g_pid,
                            (uint32_t)g_comp++);
    } else if (g_phase == PH_ESCAPE) {
        g = mpcd_rng_normal(g_seed, g_replica, g_step, MPCD_STREAM_ESCAPE_VEL, (uint32_t)g_pid,
                            (uint32_t)g_comp++);
    } else if (g_phase == PH_COLLIDE && g_cursor) {
        int pid = (int)(g_cursor - g_pp);
        g = mpcd_rng_normal(g_seed, g_replica, g_step, MPCD_STREAM_THERMAL,
                            (uint32_t)pid, (uint32_t)g_comp);
        if (++g_comp == DIM) {
            g_comp = 0;
            g_last = pid;
            g_cursor = g_cursor->next;
        }
    } else if (g_phase == PH_GHOST && g_ghost_pos < g_ghost_n) {
        g = mpcd_rng_normal(g_seed, g_replica, g_step, MPCD_STREAM_GHOST,
                            (uint32_t)g_ghost[g_ghost_pos], (uint32_t)g_comp);
        if (++g_comp == DIM) {
            g_comp = 0;
            g_ghost_pos++;
        }
    } else {
        g_unexpected++;
    }
    return g;
}

unsigned long RandomSeedSRD(unsigned long seed) { return seed; }
void init_genrand(unsigned long s) { (void)s; }
unsigned long genrand_int32(void) {
    g_unexpected++;
    return 0x80000000ul;
}
long genrand_int31(void) { return (long)(genrand_int32() >> 1); }

double genrand_real(void) {
    if (g_phase == PH_INIT)
        return mpcd_rng_uniform(g_seed, g_replica, 0u, g_stream, (uint32_t)g_pid, g_k++);
    if (g_phase == PH_RETHERM)
        return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_RETHERM, (uint32_t)g_pid,
                                g_k++);
    if (g_phase == PH_LC)
        return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_LC,
                                (uint32_t)g_pid, g_k++);
    if (g_phase == PH_ESCAPE)
        return mpcd_rng_uniform(g_seed, g_replica, g_step, g_stream, (uint32_t)g_pid, g_k++);
    if (g_phase == PH_CONE)
        return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_VICSEK, (uint32_t)g_pid,
                                g_k++);
    /* stochrotMPC draws a uniform for the orthogonal axis (ORTHAXIS only,
     * mpc.c:1289) and then one for the rotation sign, which
     * (long)genrand_real() truncates to 0 (mpc.c:1291) */
    if (g_phase == PH_COLLIDE) {
        /* chate's genrand_pmOne: the last cone particle's next uniform */
        if (g_rtech == CHATE)
            return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_VICSEK,
                                    (uint32_t)g_pid, g_k++);
        /* chateAndersenMPC's genrand_pmOne follows the particle's normals */
        if (g_rtech == CHATE_MPCAT)
            return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_VICSEK,
                                    (uint32_t)g_last, 0u);
        if ((g_rtech == ORTHAXIS || g_rtech == ACT_ORTHAXIS) && g_ccount++ == 0)
            return mpcd_rng_uniform(g_seed, g_replica, g_step, MPCD_STREAM_ORTH,
                                    (uint32_t)g_cell, 0u);
        return 0.0;
    }
    g_unexpected++;
    return 0.5;
}
double genrand_pmOne(void) { return genrand_real() <= 0.5 ? -1.0 : 1.0; }
float genrand_gauss(void) { return next_normal(); }
double genrand_gaussMB(double KBT, double M) {
    double sigma = sqrt(KBT / M);
    return sigma * next_normal();
}
double genrand_gaussGen(double mu, double sigma) { return sigma * next_normal() + mu; }
double genrand_exp(double lambda) {
    g_unexpected++;
    return lambda;
}
int genrand_poisson(double lambda) {
    g_unexpected++;
    return (int)lambda;
}
float genrand_rayleigh(float std) {
    g_unexpected++;
    return std;
}
void genrand_sphere(double vec[], int dimension) {
    g_unexpected++;
    for (int i = 0; i < dimension; i++) vec[i] = (i == 0);
}
void genrand_coneNP(double vec[], double theta, int dimension) {
    if (g_phase == PH_ESCAPE) {
        /* the orientation of an escaped nematic: the particle's own stream */
        g_stream = MPCD_STREAM_ESCAPE_ORI;
        g_k = 0;
    } else if (g_phase != PH_INIT && g_phase != PH_CONE) {
        genrand_sphere(vec, dimension);
        return;
    }
    /* rand.c:397-425, restated: it lives in the replaced rand.c */
    double z, phi, ct = cos(theta);
    if (dimension == _3D) {
        z = genrand_real() * (1.0 - ct) + ct;
        phi = genrand_real() * 2.0 * pi;
        vec[0] = z;
        vec[1] = sqrt(1.0 - z * z) * cos(phi);
        vec[2] = sqrt(1.0 - z * z) * sin(phi);
    } else if (dimension == _2D) {
        phi = theta * (1. - 2. * genrand_real());
        vec[0] = cos(phi);
        vec[1] = sin(phi);
    } else {
        g_unexpected++;
    }
}
/* rand.c:438-454, restated: a draw on the cone about the x axis, then
 * Rodrigues' rotation about axis x x-hat by the angle between them, with the
 * reference's own crossprod, absAngle and rodriguesRotation.  In a collision
 * (vicsek, mpc.c:2098-2135, one draw per listed particle) the uniforms are
 * the particle's own stream. */
void genrand_cone(double axis[], double vecOut[], double theta, int dimension) {
    double rotAx[_3D], randVec[_3D] = {0.0}, xaxis[_3D] = {0.0};
    int cone = g_phase == PH_COLLIDE && g_cursor;
    if (cone) {
        g_pid = (int)(g_cursor - g_pp);
        g_k = 0;
        g_phase = PH_CONE;
    }
    xaxis[0] = 1.0;
    genrand_coneNP(randVec, theta, dimension);
    crossprod(axis, xaxis, rotAx);
    double angle = absAngle(axis, xaxis, _3D);
    rodriguesRotation(randVec, rotAx, angle);
    for (int i = 0; i < dimension; i++) vecOut[i] = randVec[i];
    if (cone) {
        g_phase = PH_COLLIDE;
        g_cursor = g_cursor->next;
    }
}
double *ranvec3D(double *v) {
    mpcd_rng_axis3(g_seed, g_replica, g_step, (uint32_t)g_cell, v);
    return v;
}
double *ranvec2D(double *v) {
    v[0] = 1.0;
    v[1] = 0.0;
    return v;
}
double *ranvec(double *v, int dimension) {
    if (g_phase != PH_COLLIDE) g_unexpected++;
    if (dimension == _3D) ranvec3D(v);
    if (dimension == _2D) ranvec2D(v);
    return v;
}
double *ranshift(double *v, int doShift, int dimension) {
    if (doShift) {
        mpcd_rng_shift(g_seed, g_replica, g_step, dimension, v);
    } else {
        v[0] = v[1] = v[2] = 0.0;
    }
    return v;
}
int rand_particle(int POP) {
    g_unexpected++;
    return POP / 2;
}

/* ======================================================================
 * Interposers: set the cursor, then call the reference's own function.
 * ====================================================================== */
typedef void (*mpccoll_fn)(cell *, spec *, specSwimmer, double, int, double,
                           double, double, double, int, int, double, double *,
                           int);
void MPCcollision(cell *CL, spec *SP, specSwimmer SS, double KBT, int RTECH,
                  double C, double S, double FRICCO, double TimeStep,
                  int MD_mode, int LC, double RELAX, double *CLQ, int outP) {
    static mpccoll_fn orig = NULL;
    if (!orig) orig = (mpccoll_fn)dlsym(RTLD_NEXT, "MPCcollision");
    g_phase = PH_COLLIDE;
    g_cell = cell_id(CL);
    g_cursor = CL->pp;
    g_comp = 0;
    g_rtech = RTECH;
    g_ccount = 0;
    orig(CL, SP, SS, KBT, RTECH, C, S, FRICCO, TimeStep, MD_mode, LC, RELAX, CLQ,
         outP);
    g_phase = PH_NONE;
}

/* The cells ghostPart (mpc.c:351-567) fills: cut by a phantom wall (some
 * corner with W < 0) and 0 < POP < GnDNST, in its x->y->z order. */
typedef void (*ghost_fn)(cell ***, bc *, double, int, spec *);
void ghostPart(cell ***CL, bc WALL[], double KBT, int LC, spec *SP) {
    static ghost_fn orig = NULL;
    if (!orig) orig = (ghost_fn)dlsym(RTLD_NEXT, "ghostPart");
    int ncorner = 1 << DIM;
    particleMPC tp;
    memset(&tp, 0, sizeof(tp));
    g_ghost_n = 0;
    for (int a = 0; a <= XYZ[0]; a++)
        for (int b = 0; b <= XYZ[1]; b++)
            for (int c = 0; c <= XYZ[2]; c++) {
                cell *cl = &CL[a][b][c];
                if (cl->POP <= 0) continue;
                int flagW = 0;
                for (int i = 0; i < NBC; i++) {
                    if (!WALL[i].PHANTOM) continue;
                    for (int j = 0; j < ncorner; j++) {
                        tp.Q[0] = (double)a + (double)(j & 1);
                        tp.Q[1] = (double)b + (double)((j >> 1) & 1);
                        tp.Q[2] = (double)c + (double)((j >> 2) & 1);
                        if (calcW(WALL[i], tp) < 0.0) flagW = 1;
                    }
                }
                if (flagW && cl->POP < GnDNST && cl->POP > 0)
                    g_ghost[g_ghost_n++] = cell_id(cl);
            }
    g_phase = PH_GHOST;
    g_ghost_pos = 0;
    g_comp = 0;
    orig(CL, WALL, KBT, LC, SP);
    if (g_ghost_pos != g_ghost_n) g_unexpected++;
    g_phase = PH_NONE;
}

typedef void (*lccoll_fn)(cell *, spec *, double, int, double, double, int);
void LCcollision(cell *CL, spec *SP, double KBT, int zeroMFPot, double dt,
                 double SG, int LC) {
    static lccoll_fn orig = NULL;
    if (!orig) orig = (lccoll_fn)dlsym(RTLD_NEXT, "LCcollision");
    g_phase = PH_LC;
    g_cell = cell_id(CL);
    orig(CL, SP, KBT, zeroMFPot, dt, SG, LC);
    g_phase = PH_NONE;
}

typedef void (*ms_fn)(double *, double *, double, double *, double, double,
                      double);
void genrand_maierSaupe(double DIR[], double rotAx[], double rotAngle,
                        double U[], double KBT, double S, double effM) {
    static ms_fn orig = NULL;
    if (!orig) orig = (ms_fn)dlsym(RTLD_NEXT, "genrand_maierSaupe");
    particleMPC *p =
        (particleMPC *)((char *)U - offsetof(particleMPC, U));
    g_pid = (int)(p - g_pp);
    g_k = 0;
    orig(DIR, rotAx, rotAngle, U, KBT, S, effM);
}
/* The escape rule of bin() (mpc.c:969-982): replacePos_WithCheck re-places a
 * particle that left the grid from the particle's position stream of the
 * step; the velocity (genrand_gaussMB) and orientation (genrand_coneNP)
 * draws that bin() makes next come from its velocity and orientation
 * streams.  bin() ends the phase. */
typedef void (*rpwc_fn)(particleMPC *, bc *);
void replacePos_WithCheck(particleMPC *pp, bc WALL[]) {
    static rpwc_fn orig = NULL;
    if (!orig) orig = (rpwc_fn)dlsym(RTLD_NEXT, "replacePos_WithCheck");
    g_phase = PH_ESCAPE;
    g_pid = (int)(pp - g_pp);
    g_stream = MPCD_STREAM_ESCAPE_POS;
    g_k = 0;
    g_comp = 0;
    orig(pp, WALL);
}
typedef void (*bin_fn)(cell ***, spec *, bc *, double, int, int);
void bin(cell ***CL, spec *SP, bc WALL[], double KBT, int LC, int shifted) {
    static bin_fn orig = NULL;
    if (!orig) orig = (bin_fn)dlsym(RTLD_NEXT, "bin");
    orig(CL, SP, WALL, KBT, LC, shifted);
    if (g_phase == PH_ESCAPE) g_phase = PH_NONE;
}

/* Initialisation: place, push, orient and replace (init.c:1219-1405) learn
 * their particle from the address they are given. */
static int pid_of(const void *field, size_t off) {
    return (int)(((const char *)field - off - (const char *)g_pp) / sizeof(particleMPC));
}
typedef void (*place_fn)(double *, int, FILE *);
void place(double Q[], int PL, FILE *fin) {
    static place_fn orig = NULL;
    if (!orig) orig = (place_fn)dlsym(RTLD_NEXT, "place");
    g_pid = pid_of(Q, offsetof(particleMPC, Q));
    g_stream = MPCD_STREAM_INIT_POS;
    g_k = 0;
    if (g_attempt) g_attempt[g_pid] = 0;
    orig(Q, PL, fin);
}
typedef void (*replace_fn)(particleMPC *);
void replace(particleMPC *p) {
    static replace_fn orig = NULL;
    if (!orig) orig = (replace_fn)dlsym(RTLD_NEXT, "replace");
    if (g_phase == PH_ESCAPE) {
        /* attempt a of replacePos_WithCheck: uniforms DIM a .. (g_k runs on) */
        orig(p);
        return;
    }
    g_pid = (int)(p - g_pp);
    g_stream = MPCD_STREAM_INIT_POS;
    g_k = 4u * (uint32_t)(g_attempt ? ++g_attempt[g_pid] : 1);
    orig(p);
}
typedef void (*push_fn)(double *, double, int, double, FILE *);
void push(double V[], double KBT, int PL, double MASS, FILE *fin) {
    static push_fn orig = NULL;
    if (!orig) orig = (push_fn)dlsym(RTLD_NEXT, "push");
    g_pid = pid_of(V, offsetof(particleMPC, V));
    if (g_phase == PH_INIT) {
        g_stream = MPCD_STREAM_INIT_VEL;
        g_k = 0;
        g_comp = 0;
        orig(V, KBT, PL, MASS, fin);
        return;
    }
    /* a bounce-limit re-thermalisation inside MPC_BCcollision
     * (bc.c:1482): draws 4c.. of the particle's stream this step */
    const int prev = g_phase;
    const int c = (g_retherm && g_pid >= 0 && g_pid < g_retherm_n) ? g_retherm[g_pid]++ : 0;
    g_phase = PH_RETHERM;
    g_k = 4u * (uint32_t)c;
    g_comp = 4 * c;
    orig(V, KBT, PL, MASS, fin);
    g_phase = prev;
}
typedef void (*orient_fn)(double *, double *, int);
void orient(double U[], double Q[], int PL) {
    static orient_fn orig = NULL;
    if (!orig) orig = (orient_fn)dlsym(RTLD_NEXT, "orient");
    g_pid = pid_of(U, offsetof(particleMPC, U));
    g_stream = MPCD_STREAM_INIT_ORI;
    g_k = 0;
    orig(U, Q, PL);
}
#endif /* REF_INJECT */
