/*
 * dropin_timestep.c -- TEST INFRASTRUCTURE: the drop-in binding of the GPU
 * library exercised on the reference program itself.
 *
 * The reference (NIAMH-MPCD) is built unmodified from its sources into a
 * shared library with GCC's default semantic interposition (oracle/ref/
 * Makefile, target dropin).  This file defines timestep() with the
 * reference's signature (mpcd/headers/mpc.h:16); linked ahead of that
 * library, it answers the calls of the reference's own main()
 * (mpcd/mpcd.c:268, 298).  So the reference's JSON reader, initialisation,
 * output writers and checkpointing run as they are, and only the solvent
 * timestep comes from libmpcd_gpu.so:
 *
 *   first call  build an mpcd_config from the reference's state (inputList,
 *               species, walls, globals), create a handle and upload the
 *               particles (mpcd_upload_particles_strided, reading the
 *               reference's particleMPC array in place);
 *   each call   mpcd_timestep (AVNOW, KBTNOW); on the steps whose output
 *               or checkpoint reads the particles (need_host_state), the
 *               particles are downloaded into the reference's array and the
 *               end of the reference's timestep runs for the output
 *               writers: re-bin, localPROP and the flow sums
 *               (mpc.c:4936-4958).
 *
 * Configurations outside the GPU path (MD coupling, swimmers, moving or
 * non-planar walls, thermostats, other collision operators, 3D or global
 * nematic order) make mpcd_create fail or are refused here, and so does a machine without a
 * usable GPU; every call then goes to the reference's own timestep (found
 * with dlsym(RTLD_NEXT)), and the run is the reference's.
 *
 * Environment: MPCD_DROPIN_PRECISION = fp64 (default) or mixed;
 * MPCD_DROPIN_SYNC set downloads on every step;
 * MPCD_DROPIN_OFF set runs the reference's own timestep throughout (the same
 * executable as its CPU control).
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* product header first: the reference headers define macros named e, pi
 * and real (definitions.h:73-75) */
#include "mpcd_gpu.h"

#include "definitions.h"
#include "SRDclss.h"
#include "mpc.h"
#include "therm.h"
#include "pout.h"

extern int DIM, GPOP, NSPECI, NBC, NS, MDmode;
extern double GnDNST;
extern int XYZ[_3D];

typedef void (*timestep_fn)(cell ***, particleMPC *, spec[], bc[], simptr, specSwimmer *,
                            swimmer[], double[_3D], double[_3D], double[_3D], inputList,
                            double *, double *, int, int, outputFlagsList, outputFilesList);

static int g_state = 0; /* 0 untried, 1 GPU, -1 reference */
static mpcd_handle *g_h = NULL;
static uint32_t g_step = 0;

static int fill_config(mpcd_config *c, inputList in, spec SP[], bc WALL[]) {
    int s, w, d;
    memset(c, 0, sizeof(*c));
    c->dim = DIM;
    for (d = 0; d < 3; d++) c->L[d] = XYZ[d];
    c->dt = in.dt;
    c->kbt = in.KBT;
    c->coll_op = in.RTECH;
    c->fricco = in.FRICCO;
    c->relax = in.TAU;
    c->lc = in.LC;
    c->rot_ang = in.RA;
    c->galinv = in.GALINV;
    for (d = 0; d < 3; d++) c->grav[d] = in.GRAV[d];
    c->gndnst = GnDNST;
    c->seed = (uint64_t)in.seed;
    c->replica = 0;
    {
        const char *p = getenv("MPCD_DROPIN_PRECISION");
        c->precision = (p && strcmp(p, "mixed") == 0) ? MPCD_PREC_MIXED : MPCD_PREC_FP64;
    }
    if (NSPECI > MPCD_MAX_SPECIES || NBC > MPCD_MAX_WALLS) return 0;
    c->n_species = NSPECI;
    for (s = 0; s < NSPECI; s++) {
        c->species[s].mass = SP[s].MASS;
        c->species[s].damp = SP[s].DAMP;
        c->species[s].rfc = SP[s].RFC;
        c->species[s].tumble = SP[s].TUMBLE;
        c->species[s].chihi = SP[s].CHIHI;
        c->species[s].act = SP[s].ACT;
        c->species[s].mfpot = SP[s].MFPOT;
        c->species[s].sigwidth = SP[s].SIGWIDTH;
        c->species[s].sigpos = SP[s].SIGPOS;
        c->species[s].minactratio = SP[s].MINACTRATIO;
    }
    c->n_walls = NBC;
    for (w = 0; w < NBC; w++) {
        const bc *b = &WALL[w];
        mpcd_wall *o = &c->walls[w];
        /* static planes only */
        if (!b->PLANAR || b->DSPLC || b->ABS) return 0;
        for (d = 0; d < 4; d++)
            if (b->P[d] != 1.0) return 0;
        for (d = 0; d < 3; d++) {
            o->A[d] = b->A[d];
            o->Q[d] = b->Q[d];
            o->DVxyz[d] = b->DVxyz[d];
            o->MUxyz[d] = b->MUxyz[d];
            o->DUxyz[d] = b->DUxyz[d];
        }
        o->R = b->R;
        o->inv = b->INV;
        o->phantom = b->PHANTOM;
        o->coll_type = b->COLL_TYPE;
        o->DN = b->DN;
        o->DT = b->DT;
        o->DVN = b->DVN;
        o->DVT = b->DVT;
        o->MVN = b->MVN;
        o->MVT = b->MVT;
        o->MUN = b->MUN;
        o->MUT = b->MUT;
        for (s = 0; s < MPCD_MAX_SPECIES; s++) o->inter[s] = b->INTER[s];
    }
    c->capacity = GPOP;
    return 1;
}

static int setup(particleMPC *pp, spec SP[], bc WALL[], inputList in) {
    mpcd_config c;
    /* options the GPU path does not carry: MD, swimmers, the thermostats,
     * multiphase and incompressibility collisions, the no-hydrodynamics
     * scramble, activity layers (mpc.c:4706-4760), and the periodic return
     * to the rest frame that outputResults applies to the host particles
     * (pout.c:2557); nematic order other than the local 2D form makes
     * mpcd_create fail */
    if (getenv("MPCD_DROPIN_OFF")) return 0;
    if (MDmode || NS > 0 || in.TSTECH != 0 || in.MULTIPHASE != MPHOFF ||
        in.inCOMP != INCOMPOFF || in.noHI == HIOFF || in.MFPLAYERH > 0 || in.RFRAME)
        return 0;
    if (!fill_config(&c, in, SP, WALL)) return 0;
    if (mpcd_create(&c, &g_h) != MPCD_OK) return 0;
    {
        /* the species' VDIST re-thermalises particles past the bounce
         * limit (bc.c:1482); READ (1) has no file at that point */
        int vd[MPCD_MAX_SPECIES] = {0};
        int s;
        for (s = 0; s < NSPECI && s < MPCD_MAX_SPECIES; s++)
            vd[s] = SP[s].VDIST == 1 ? MPCD_VDIST_RANDVEL : SP[s].VDIST;
        if (mpcd_set_species_vdist(g_h, vd) != MPCD_OK) {
            mpcd_destroy(g_h);
            g_h = NULL;
            return 0;
        }
    }
    if (mpcd_upload_particles_strided(g_h, GPOP, pp, sizeof(particleMPC),
                                      offsetof(particleMPC, Q), offsetof(particleMPC, V),
                                      offsetof(particleMPC, U),
                                      offsetof(particleMPC, SPID)) != MPCD_OK) {
        mpcd_destroy(g_h);
        g_h = NULL;
        return 0;
    }
    fprintf(stderr, "dropin: solvent timestep on the GPU (%s, %d particles)\n",
            c.precision == MPCD_PREC_MIXED ? "mixed" : "fp64", GPOP);
    return 1;
}

/* Whether the caller reads the particles or the cell lists after this step:
 * on the main loop's output and histogram steps (writeOutput,
 * writeHistograms: mpcd.c:302-307), on checkpoint steps of either loop
 * (mpcd.c:272, 310), on the last step, and on every step while the flow
 * field is averaged (the per-step flow sums, mpc.c:4950-4958).  On the other
 * steps the state stays on the GPU.  MPCD_DROPIN_SYNC set downloads on every
 * step (the device state evolves the same either way). */
static int need_host_state(int runtime, inputList in, outputFlagsList f) {
    if (getenv("MPCD_DROPIN_SYNC")) return 1;
    if (f.FLOWOUT >= OUT || f.SWFLOWOUT >= OUT) return 1;
    if (f.CHCKPNT >= OUT && runtime % f.CHCKPNT == 0) return 1;
    if (in.warmupSteps) return 0;
    return writeOutput(runtime, f, in.RFRAME, in.zeroNetMom) || writeHistograms(runtime, f) ||
           runtime >= in.simSteps;
}

void timestep(cell ***CL, particleMPC *SRDparticles, spec SP[], bc WALL[], simptr simMD,
              specSwimmer *SS, swimmer swimmers[], double AVNOW[_3D], double AVV[_3D],
              double avDIR[_3D], inputList in, double *KBTNOW, double *AVS, int runtime,
              int MD_mode, outputFlagsList outFlags, outputFilesList outFiles) {
    if (g_state == 0) g_state = setup(SRDparticles, SP, WALL, in) ? 1 : -1;
    if (g_state < 0) {
        timestep_fn ref = (timestep_fn)dlsym(RTLD_NEXT, "timestep");
        if (!ref) {
            fprintf(stderr, "dropin: reference timestep not found\n");
            exit(1);
        }
        ref(CL, SRDparticles, SP, WALL, simMD, SS, swimmers, AVNOW, AVV, avDIR, in, KBTNOW,
            AVS, runtime, MD_mode, outFlags, outFiles);
        return;
    }
    /* one monotonically increasing step number keys the draws (warm-up and
     * main loop both count runtime from zero) */
    if (mpcd_timestep(g_h, g_step++, AVNOW, KBTNOW) != MPCD_OK) {
        fprintf(stderr, "dropin: GPU timestep failed\n");
        exit(1);
    }
    if (!need_host_state(runtime, in, outFlags)) return;
    if (mpcd_download_particles_strided(g_h, SRDparticles, sizeof(particleMPC),
                                        offsetof(particleMPC, Q), offsetof(particleMPC, V),
                                        offsetof(particleMPC, U)) != MPCD_OK) {
        fprintf(stderr, "dropin: GPU download failed\n");
        exit(1);
    }
    /* the end of the reference's timestep, for its output writers */
    bin(CL, SP, WALL, in.KBT, in.LC, 0);
    localPROP(CL, SP, *SS, in.RTECH, in.LC);
    if ((outFlags.FLOWOUT >= OUT || outFlags.SWFLOWOUT >= OUT) && !in.warmupSteps) {
        localFLOW(CL, SP);
        if (outFlags.FLOWOUT >= OUT) sumFLOW(CL);
    }
    /* AVNOW and KBTNOW came from mpcd_timestep: avVel after the collision
     * and TEMP against AVV, which is zero without the MAXV thermostat
     * (init.c:2074-2078), as the reference's timestep leaves them */
    (void)AVV;
    (void)runtime;
    (void)avDIR;
    (void)AVS;
}

/* the reference program's main(), renamed at its compilation */
int mpcd_reference_main(int argc, char *argv[]);
int main(int argc, char *argv[]) {
    const int r = mpcd_reference_main(argc, argv);
    if (g_h) mpcd_destroy(g_h);
    return r;
}
