// mpcd_out.cpp -- the reference's output files of the per-cell fields and
// global measures, written from the library's arrays.
//
// The reference's writers (pout.c) print, for the cells of the L^D box in
// x -> y -> z order, the end-of-step centre-of-mass velocity, population,
// mass and per-species populations that localPROP leaves after the re-bin
// (mpc.c:4936-4942), the flow field's running sum (sumFLOW, mpc.c:241-246),
// and the global velocity, temperature, mean velocity gradient and kinetic
// energy.  Here the same lines are printed, character for character, from
// the arrays mpcd_cell_props, mpcd_cell_species and mpcd_flow_read return
// (cells of the (L+1)^D grid in row-major order, vectors as 3 doubles).
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mpcd_gpu.h"

namespace {

// The banner every output file of the reference starts with (outheader,
// pout.c:40-52; written by openBasic, init.c:51-63).
void banner(FILE *f) {
    static const char *const kLines[] = {
        " **********************************************\n",
        " **********************************************\n",
        " **********************************************\n",
        " ***************** NIAMH-MPCD *****************\n",
        " **********************************************\n",
        " **************** Shendruk Lab ****************\n",
        " ********** University of Edinburgh ***********\n",
        " ************ Code begun Oct. 2008 ************\n",
        " **********************************************\n",
        " **********************************************\n",
        " **********************************************\n\n",
    };
    for (const char *l : kLines) fputs(l, f);
}

struct Grid {
    int dim, L[3], N1[3], ns;
    bool ok;
    explicit Grid(const mpcd_config *c) {
        ok = c && (c->dim == 2 || c->dim == 3) && c->n_species >= 1 &&
             c->n_species <= MPCD_MAX_SPECIES;
        if (!ok) return;
        dim = c->dim;
        ns = c->n_species;
        for (int d = 0; d < 3; d++) {
            L[d] = d < dim ? c->L[d] : 1;
            N1[d] = L[d] + 1;
            ok = ok && L[d] >= 1;
        }
    }
    size_t cells() const { return (size_t)N1[0] * N1[1] * N1[2]; }
    size_t at(int i, int j, int k) const { return ((size_t)i * N1[1] + j) * N1[2] + k; }
};

FILE *open_out(const char *path, int header) {
    return fopen(path, header ? "w" : "a");
}

int close_out(FILE *f) {
    const bool bad = ferror(f) != 0;
    return (fclose(f) != 0 || bad) ? MPCD_ERR_ARG : MPCD_OK;
}

}  // namespace

extern "C" int mpcd_write_coarse(const char *path, const mpcd_config *cfg, double t,
                                 const int *pop, const double *vcm, const int *spc, int header) {
    const Grid g(cfg);
    if (!path || !g.ok || !pop || !vcm || (g.ns > 1 && !spc)) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // coarseheader, pout.c:80-85
        banner(f);
        fprintf(f, "t\t\t\t\tQX\t\tQY\t\tQZ\tVcmX\t\t\tVcmY\t\t\tVcmZ\t\t\t\tPOP");
        for (int n = 0; n < g.ns; n++) fprintf(f, "\t\tSP%d", n);
        fprintf(f, "\n");
    }
    // coarseout, pout.c:640-658
    for (int i = 0; i < g.L[0]; i++)
        for (int j = 0; j < g.L[1]; j++)
            for (int k = 0; k < g.L[2]; k++) {
                const size_t c = g.at(i, j, k);
                fprintf(f, "%.2f\t", t);
                fprintf(f, "%5d\t%5d\t%5d\t", i, j, k);
                if (pop[c] == 0) {
                    fprintf(f, "%12.5e\t%12.5e\t%12.5e\t%5i", 0., 0., 0., 0);
                    for (int n = 0; n < g.ns; n++) fprintf(f, "\t%5i", 0);
                } else {
                    fprintf(f, "%12.5e\t%12.5e\t%12.5e\t%5i", vcm[3 * c], vcm[3 * c + 1],
                            vcm[3 * c + 2], pop[c]);
                    for (int n = 0; n < g.ns; n++)
                        fprintf(f, "\t%5i", g.ns > 1 ? spc[(size_t)n * g.cells() + c] : pop[c]);
                }
                fprintf(f, "\n");
            }
    return close_out(f);
}

extern "C" int mpcd_write_velfield(const char *path, const mpcd_config *cfg, double t,
                                   const double *vcm, int header) {
    const Grid g(cfg);
    if (!path || !g.ok || !vcm) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // flowheader, pout.c:355-357
        banner(f);
        fprintf(f, "   t\t   QX\t   QY\t   QZ\tVcmX\t\tVcmY\t\tVcmZ\n");
    }
    // velout, pout.c:1715-1731
    double vel[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < g.L[0]; i++)
        for (int j = 0; j < g.L[1]; j++)
            for (int k = 0; k < g.L[2]; k++) {
                const size_t c = g.at(i, j, k);
                for (int h = 0; h < g.dim; h++) vel[h] = vcm[3 * c + h];
                fprintf(f, "%12.5e\t", t);
                fprintf(f, "%5d\t%5d\t%5d\t", i, j, k);
                fprintf(f, "%12.5e\t%12.5e\t%12.5e\n", vel[0], vel[1], vel[2]);
            }
    return close_out(f);
}

extern "C" int mpcd_write_densityfield(const char *path, const mpcd_config *cfg, double t,
                                       const int *pop, const double *mass, const int *spc,
                                       int header) {
    const Grid g(cfg);
    if (!path || !g.ok || !pop || !mass || (g.ns > 1 && !spc)) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // densityheader, pout.c:372-377
        banner(f);
        fprintf(f, "   t\t   QX\t   QY\t   QZ\tpop\t\tmass\t\tpopSRD\t\tpopMD\t\tpopSW");
        for (int n = 0; n < g.ns; n++) fprintf(f, "\t\tSP%d", n);
        fprintf(f, "\n");
    }
    // densityout, pout.c:1744-1758: MPCD particles only (POPSRD = POP,
    // POPMD = POPSW = 0)
    for (int i = 0; i < g.L[0]; i++)
        for (int j = 0; j < g.L[1]; j++)
            for (int k = 0; k < g.L[2]; k++) {
                const size_t c = g.at(i, j, k);
                fprintf(f, "%12.5e\t", t);
                fprintf(f, "%5d\t%5d\t%5d\t", i, j, k);
                fprintf(f, "%5d\t%12.5e\t%5d\t%5d\t%5d\t", pop[c], mass[c], pop[c], 0, 0);
                for (int n = 0; n < g.ns; n++)
                    fprintf(f, "\t%5d", g.ns > 1 ? spc[(size_t)n * g.cells() + c] : pop[c]);
                fprintf(f, "\n");
            }
    return close_out(f);
}

extern "C" int mpcd_write_flowfield(const char *path, const mpcd_config *cfg, double t,
                                    const double *flow, int interval, int header) {
    const Grid g(cfg);
    if (!path || !g.ok || !flow || interval == 0) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // flowheader, pout.c:355-357
        banner(f);
        fprintf(f, "   t\t   QX\t   QY\t   QZ\tVcmX\t\tVcmY\t\tVcmZ\n");
    }
    // flowout, pout.c:1681-1701: the sum over the interval's steps / interval
    const double dint = (double)interval;
    double av[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < g.L[0]; i++)
        for (int j = 0; j < g.L[1]; j++)
            for (int k = 0; k < g.L[2]; k++) {
                const size_t c = g.at(i, j, k);
                for (int h = 0; h < g.dim; h++) av[h] = flow[3 * c + h] / dint;
                fprintf(f, "%12.5e\t", t);
                fprintf(f, "%5d\t%5d\t%5d\t", i, j, k);
                fprintf(f, "%12.5e\t%12.5e\t%12.5e\n", av[0], av[1], av[2]);
            }
    return close_out(f);
}

extern "C" int mpcd_vel_grad(const mpcd_config *cfg, const double *vcm, double *E,
                             double grad[9]) {
    const Grid g(cfg);
    if (!g.ok || !vcm || !E) return MPCD_ERR_ARG;
    // localVelGrad (lc.c:2054-2060): D3Q15 (lc.c:2070-2123) or D2Q9
    // (lc.c:2134-2162) lattice-Boltzmann weights, E[i][j] = dv_i/dx_j over
    // the bulk cells [1, L), then the edges copied from their inner
    // neighbour in x, y, z order; entries neither reaches (corners of the
    // extra layer) keep what they held, as the reference's cell array does.
    static const int u3[14][3] = {{1, 0, 0},   {0, 1, 0},   {-1, 0, 0}, {0, -1, 0},
                                  {0, 0, 1},   {0, 0, -1},  {1, 1, 1},  {-1, 1, 1},
                                  {1, -1, 1},  {-1, -1, 1}, {1, 1, -1}, {-1, 1, -1},
                                  {1, -1, -1}, {-1, -1, -1}};
    static const int u2[8][3] = {{1, 0, 0},  {0, 1, 0},  {-1, 0, 0}, {0, -1, 0},
                                 {1, 1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}};
    const double w3[14] = {1. / 9.,  1. / 9.,  1. / 9.,  1. / 9.,  1. / 9.,
                           1. / 9.,  1. / 72., 1. / 72., 1. / 72., 1. / 72.,
                           1. / 72., 1. / 72., 1. / 72., 1. / 72.};
    const double w2[8] = {1. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
    const int D = g.dim, nn = D == 3 ? 14 : 8;
    const int(*uv)[3] = D == 3 ? u3 : u2;
    const double *w = D == 3 ? w3 : w2;
    const int X = g.L[0], Y = g.L[1], Z = g.L[2];
    auto e = [&](int a, int b, int c, int i, int j) -> double & {
        return E[9 * g.at(a, b, c) + 3 * i + j];
    };
    const int zlo = D == 3 ? 1 : 0, zhi = D == 3 ? Z : 1;
    for (int a = 1; a < X; a++)
        for (int b = 1; b < Y; b++)
            for (int c = zlo; c < zhi; c++)
                for (int i = 0; i < D; i++)
                    for (int j = 0; j < D; j++) {
                        double s = 0.;
                        for (int k = 0; k < nn; k++)
                            s += w[k] * uv[k][j] *
                                 vcm[3 * g.at(a + uv[k][0], b + uv[k][1], c + uv[k][2]) + i];
                        e(a, b, c, i, j) = s * 3.;
                    }
    auto copy = [&](int a, int b, int c, int a2, int b2, int c2) {
        for (int i = 0; i < D; i++)
            for (int j = 0; j < D; j++) e(a, b, c, i, j) = e(a2, b2, c2, i, j);
    };
    for (int b = 0; b < Y; b++)
        for (int c = 0; c < zhi; c++) copy(0, b, c, 1, b, c);
    for (int b = 0; b < Y; b++)
        for (int c = 0; c < zhi; c++) copy(X, b, c, X - 1, b, c);
    for (int a = 0; a < X; a++)
        for (int c = 0; c < zhi; c++) copy(a, 0, c, a, 1, c);
    for (int a = 0; a < X; a++)
        for (int c = 0; c < zhi; c++) copy(a, Y, c, a, Y - 1, c);
    if (D == 3) {
        for (int a = 0; a < X; a++)
            for (int b = 0; b < Y; b++) copy(a, b, 0, a, b, 1);
        for (int a = 0; a < X; a++)
            for (int b = 0; b < Y; b++) copy(a, b, Z, a, b, Z - 1);
    }
    if (grad) {
        // the box mean (outputResults, pout.c:2572-2577): the L^D cells / VOL
        double vol = 1.0;
        for (int d = 0; d < D; d++) vol *= g.L[d];
        for (int q = 0; q < 9; q++) grad[q] = 0.;
        for (int a = 0; a < X; a++)
            for (int b = 0; b < Y; b++)
                for (int c = 0; c < Z; c++)
                    for (int q = 0; q < 9; q++) grad[q] += E[9 * g.at(a, b, c) + q];
        for (int q = 0; q < 9; q++) grad[q] /= vol;
    }
    return MPCD_OK;
}

extern "C" int mpcd_av_vel(const mpcd_config *cfg, const double *vcm, double avnow[3]) {
    const Grid g(cfg);
    if (!g.ok || !vcm || !avnow) return MPCD_ERR_ARG;
    // avVel (therm.c:362-367): every cell of the (L+1)^D grid, over VOL
    double vol = 1.0;
    for (int d = 0; d < g.dim; d++) vol *= g.L[d];
    for (int d = 0; d < 3; d++) avnow[d] = 0.0;
    for (size_t c = 0; c < g.cells(); c++)
        for (int d = 0; d < g.dim; d++) avnow[d] += vcm[3 * c + d];
    for (int d = 0; d < g.dim; d++) avnow[d] /= vol;
    return MPCD_OK;
}

extern "C" int mpcd_write_avvel(const char *path, double t, const double avnow[3], double kbtnow,
                                const double grad[9], int header) {
    if (!path || !avnow || !grad) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // avvelWithGradVelheader, pout.c:156-158
        banner(f);
        fprintf(f,
                "t\t VcmX\t\tVcmY\t\tVcmZ\t\tKBT\t\tdVXX\t\tdVXY\t\tdVXZ\t\tdVYX\t\tdVYY\t\tdVYZ"
                "\t\tdVZX\t\tdVZY\t\tdVZZ\t\n");
    }
    // avveloutWithGradVel, pout.c:1590-1596
    fprintf(f, "%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\t", t, avnow[0], avnow[1], avnow[2], kbtnow);
    fprintf(f, "%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\t%12.5e\n", grad[0],
            grad[1], grad[2], grad[3], grad[4], grad[5], grad[6], grad[7], grad[8]);
    return close_out(f);
}

extern "C" int mpcd_write_energy(const char *path, double t, double kinetic, double kbtnow,
                                 int header) {
    if (!path) return MPCD_ERR_ARG;
    FILE *f = open_out(path, header);
    if (!f) return MPCD_ERR_ARG;
    if (header) {  // energyheader, pout.c:517-519
        banner(f);
        fprintf(f, "t\t\tMPCD_kin\t\tMPCD_nem\t\tBC_kin\t\tBC_rot\t\tTotal\t\tKBT\n");
    }
    // enout, pout.c:1389-1425, for static walls and an isotropic fluid:
    // no wall or nematic energies
    const double wmf = 0.0, bck = 0.0, bcr = 0.0;
    fprintf(f, "%lf\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", t, kinetic, wmf, bck, bcr,
            kinetic + bck + bcr + wmf, kbtnow);
    return close_out(f);
}
