// mpcd_ckpt.cpp -- checkpoints in the reference's text format.
//
// The reference writes a checkpoint with checkpoint() (pout.c:2325-2396) and
// reads it back with readchckpnt() (read.c:669-834).  A checkpoint here is
// the file's fields in the writer's line layout: each line a list of typed
// fields, held as parsed, so that a file read and written again is the same
// byte for byte, and the fields this library does not use (output flags,
// swimmers, theory values, ...) pass through.  The library reads and
// replaces the fields it owns: the configuration, the run counters and the
// particles.
//
// Field types, as the writer prints them:
//   'i' int "%d", 'I' int "%i" (readchckpnt reads these with %i, which also
//   accepts octal and hex), 'l' long "%ld", 'f' double "%lf", 'g' float
//   "%f" (CHCKPNTTIMER; always six decimals, also in the precise form,
//   because readchckpnt reads one integer more than the writer writes on
//   that line and relies on the decimal point to resynchronise, read.c:718).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mpcd_gpu.h"

namespace {

struct Field {
    char t;
    long long i;
    double f;
};

struct Line {
    std::vector<Field> v;
    bool trail;  // the writer ends this line with a space before the newline
};

// Line layouts of the writer, in order (pout.c:2328-2393).
const char *const kHead[] = {
    "i",            // simSteps
    "if",           // warmupSteps dt
    "l",            // seed
    "iiiiff",       // DIM XYZ[3] KBT KBTNOW
    "iiiiii",       // RFRAME zeroNetMom GALINV TSTECH RTECH LC
    "fff",          // TAU RA FRICCO
    "iiii",         // noHI inCOMP MULTIPHASE MFPLAYERH
    "fff",          // GRAV
    "fff",          // MAG
    "ii",           // MD_mode stepsMD
    "ii",           // GPOP NSPECI
    "iiffiif",      // runtime warmtime C S GRAV_FLAG MAG_FLAG tolD
    "ffffffff",     // AVVEL AVS avDIR[3] S4 stdN VOL
    "ffffff",       // AVV[3] AVNOW[3]
    "ffffff",       // theoryGl: MFP VISC THERMD SDIFF SPEEDOFSOUND sumM
    "ii",           // chckpntIn MDmode
    "iiiiiiiiiiiiiiiiiiiiiiiiiiiiiiig",  // DBUG + 30 output flags, CHCKPNTTIMER
    "ii",           // SPOUT PRESOUT
    "iiiiiii",      // histogram outputs
    "iiiii",        // spectra, topology, defects, disclinations
    "iii",          // swimmer outputs
};
constexpr int kNHead = sizeof(kHead) / sizeof(kHead[0]);
// species: MASS POP QDIST VDIST ODIST, RFC LEN TUMBLE CHIHI CHIA ACT MFPOT
// SIGWIDTH SIGPOS DAMP, VOL nDNST mDNST MINACTRATIO BS; then M[NSPECI]; then
// the species' theory values
const char *const kSpec = "fIIIIfffffffffffffff";
const char *const kSpecTheory = "ffffff";
const char *const kDens = "fffi";  // GnDNST GmDNST GMASS maxXYZ
// walls (8 lines each)
const char *const kWall[] = {
    "iiffffffffff",          // COLL_TYPE PHANTOM E Q[3] V[3] O[3]
    "ffffffffffffffffffff",  // L[3] G[3] A[3] AINV[3] P[4] R B[3]
    "ffffffffffffff",        // DN DT DVN DVT DVxyz[3] MVN MVT MUN MUT MUxyz[3]
    "ffffiif",               // DUxyz[3] KBT DSPLC INV MASS
    "fffffffffffffffff",     // W VOL Q_old[3] O_old[3] I[3][3]
    "iiiff",                 // PLANAR REORIENT ABS ROTSYMM[2]
    "ffffff",                // dV[3] dL[3]
};
const char *const kPart = "iifffffffffffff";  // S_flag SPID q Q[3] V[3] U[3] T[3]
const char *const kSwimSpec[] = {"iiiiiiffii", "ffffffffffffiffffif"};
const char *const kSwimmer[] = {"ifffiifffff", "ifffffffff", "ifffffffff"};

constexpr int L_STEPS = 0, L_WARM = 1, L_SEED = 2, L_DIM = 3, L_FLAGS = 4, L_ANG = 5,
              L_HI = 6, L_GRAV = 7, L_MAG = 8, L_MD = 9, L_POP = 10, L_RUN = 11, L_AVG = 12,
              L_AVV = 13, L_THEORY = 14, L_CKIN = 15;

}  // namespace

struct mpcd_ckpt {
    std::vector<Line> lines;
    int nspec = 0, nbc = 0, gpop = 0, ns = 0;
    int spec0 = 0;  // first species line
    int dens = 0;   // GnDNST line
    int wall0 = 0;  // first wall line
    int part0 = 0;  // first particle line
    int swim0 = 0;  // swimmer species line

    Field &at(int l, int k) { return lines[(size_t)l].v[(size_t)k]; }
    const Field &at(int l, int k) const { return lines[(size_t)l].v[(size_t)k]; }
    double f(int l, int k) const { return at(l, k).f; }
    long long i(int l, int k) const { return at(l, k).i; }
    void set_f(int l, int k, double x) { at(l, k).f = x; }
    void set_i(int l, int k, long long x) { at(l, k).i = x; }
    int spec_line(int s) const { return spec0 + 3 * s; }
    int wall_line(int w, int k) const { return wall0 + 8 * w + k; }
    int part_line(int p) const { return part0 + p; }
};

namespace {

Line blank_line(const char *types, int repeat_f = 0, bool trail = false) {
    Line ln;
    ln.trail = trail;
    if (repeat_f > 0) {
        for (int k = 0; k < repeat_f; k++) ln.v.push_back(Field{types[0], 0, 0.0});
    } else {
        for (const char *p = types; *p; ++p) ln.v.push_back(Field{*p, 0, 0.0});
    }
    return ln;
}

// Token reader over the whole file.
struct Tokens {
    std::string buf;
    size_t pos = 0;
    bool next(std::string &tok) {
        while (pos < buf.size() && isspace((unsigned char)buf[pos])) pos++;
        if (pos >= buf.size()) return false;
        size_t s = pos;
        while (pos < buf.size() && !isspace((unsigned char)buf[pos])) pos++;
        tok.assign(buf, s, pos - s);
        return true;
    }
};

bool parse_field(const std::string &tok, Field &f) {
    char *end = nullptr;
    errno = 0;
    if (f.t == 'f' || f.t == 'g') {
        f.f = strtod(tok.c_str(), &end);
    } else {
        f.i = strtoll(tok.c_str(), &end, f.t == 'I' ? 0 : 10);
    }
    return end && *end == '\0' && errno == 0;
}

bool read_line(Tokens &tk, Line &ln) {
    std::string tok;
    for (Field &f : ln.v)
        if (!tk.next(tok) || !parse_field(tok, f)) return false;
    return true;
}

void print_field(FILE *fp, const Field &f, bool precise) {
    switch (f.t) {
        case 'l':
            fprintf(fp, "%lld", f.i);
            break;
        case 'f':
            if (precise)
                fprintf(fp, "%.17g", f.f);
            else
                fprintf(fp, "%lf", f.f);
            break;
        case 'g':
            fprintf(fp, "%f", f.f);
            break;
        default:
            fprintf(fp, "%d", (int)f.i);
    }
}

// The layout after the header, once the counts are known.
void lay_out(mpcd_ckpt &c) {
    c.lines.resize(kNHead);
    c.spec0 = kNHead;
    for (int s = 0; s < c.nspec; s++) {
        c.lines.push_back(blank_line(kSpec));
        c.lines.push_back(blank_line("f", c.nspec, true));
        c.lines.push_back(blank_line(kSpecTheory));
    }
    c.dens = (int)c.lines.size();
    c.lines.push_back(blank_line(kDens));
    c.lines.push_back(blank_line("i"));  // NBC
    c.wall0 = (int)c.lines.size();
    for (int w = 0; w < c.nbc; w++) {
        for (const char *t : kWall) c.lines.push_back(blank_line(t));
        c.lines.push_back(blank_line("I", MPCD_MAX_SPECIES + 2, true));
    }
    c.part0 = (int)c.lines.size();
    for (int p = 0; p < c.gpop; p++) c.lines.push_back(blank_line(kPart));
    c.swim0 = (int)c.lines.size();
    c.lines.push_back(blank_line(kSwimSpec[0]));
    c.lines.push_back(blank_line(kSwimSpec[1]));
    for (int k = 0; k < c.ns; k++)
        for (const char *t : kSwimmer) c.lines.push_back(blank_line(t));
}

bool feq0(double x) { return std::fabs(x) < 1e-8; }

}  // namespace

extern "C" int mpcd_ckpt_read(const char *path, mpcd_ckpt **out) {
    if (!path || !out) return MPCD_ERR_ARG;
    *out = nullptr;
    FILE *fp = fopen(path, "rb");
    if (!fp) return MPCD_ERR_ARG;
    Tokens tk;
    char chunk[65536];
    size_t got;
    while ((got = fread(chunk, 1, sizeof chunk, fp)) > 0) tk.buf.append(chunk, got);
    fclose(fp);
    mpcd_ckpt *c = new mpcd_ckpt();
    bool ok = true;
    for (int l = 0; l < kNHead && ok; l++) {
        c->lines.push_back(blank_line(kHead[l]));
        ok = read_line(tk, c->lines.back());
    }
    // species (their count, then populations fix the particle count, as
    // readchckpnt does), densities, walls, particles, swimmers: each block
    // is read before the counts of the next are known
    if (ok) {
        c->nspec = (int)c->i(L_POP, 1);
        ok = c->nspec >= 0 && c->nspec <= 64;
    }
    if (ok) {
        c->spec0 = kNHead;
        for (int s = 0; s < c->nspec && ok; s++) {
            c->lines.push_back(blank_line(kSpec));
            ok = read_line(tk, c->lines.back());
            c->lines.push_back(blank_line("f", c->nspec, true));
            ok = ok && read_line(tk, c->lines.back());
            c->lines.push_back(blank_line(kSpecTheory));
            ok = ok && read_line(tk, c->lines.back());
        }
    }
    long long gpop = 0;
    for (int s = 0; ok && s < c->nspec; s++) gpop += c->i(c->spec_line(s), 1);
    ok = ok && gpop >= 0 && gpop <= 0x7FFFFFFF;
    if (ok) {
        c->dens = (int)c->lines.size();
        c->lines.push_back(blank_line(kDens));
        ok = read_line(tk, c->lines.back());
        c->lines.push_back(blank_line("i"));
        ok = ok && read_line(tk, c->lines.back());
    }
    if (ok) {
        c->nbc = (int)c->lines.back().v[0].i;
        ok = c->nbc >= 0 && c->nbc <= 4096;
    }
    c->wall0 = (int)c->lines.size();
    for (int w = 0; ok && w < c->nbc; w++) {
        for (const char *t : kWall) {
            c->lines.push_back(blank_line(t));
            ok = ok && read_line(tk, c->lines.back());
        }
        c->lines.push_back(blank_line("I", MPCD_MAX_SPECIES + 2, true));
        ok = ok && read_line(tk, c->lines.back());
    }
    c->gpop = (int)gpop;
    c->part0 = (int)c->lines.size();
    if (ok) c->lines.reserve(c->lines.size() + (size_t)c->gpop + 8);
    for (int p = 0; ok && p < c->gpop; p++) {
        c->lines.push_back(blank_line(kPart));
        ok = read_line(tk, c->lines.back());
    }
    c->swim0 = (int)c->lines.size();
    for (int k = 0; ok && k < 2; k++) {
        c->lines.push_back(blank_line(kSwimSpec[k]));
        ok = read_line(tk, c->lines.back());
    }
    if (ok) {
        c->ns = (int)c->i(c->swim0, 0);
        ok = c->ns >= 0 && c->ns <= (1 << 24);
    }
    for (int k = 0; ok && k < c->ns; k++)
        for (const char *t : kSwimmer) {
            c->lines.push_back(blank_line(t));
            ok = ok && read_line(tk, c->lines.back());
        }
    if (!ok) {
        delete c;
        return MPCD_ERR_ARG;
    }
    // the header's GPOP follows the species populations (read.c:763-768)
    c->set_i(L_POP, 0, c->gpop);
    *out = c;
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_free(mpcd_ckpt *ck) {
    delete ck;
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_write(const mpcd_ckpt *ck, const char *path, int precise) {
    if (!ck || !path) return MPCD_ERR_ARG;
    FILE *fp = fopen(path, "wb");
    if (!fp) return MPCD_ERR_ARG;
    for (const Line &ln : ck->lines) {
        for (size_t k = 0; k < ln.v.size(); k++) {
            if (k) fputc(' ', fp);
            print_field(fp, ln.v[k], precise != 0);
        }
        if (ln.trail && !ln.v.empty()) fputc(' ', fp);
        fputc('\n', fp);
    }
    const bool bad = ferror(fp) != 0;
    return (fclose(fp) != 0 || bad) ? MPCD_ERR_ARG : MPCD_OK;
}

extern "C" int mpcd_ckpt_create(const mpcd_config *cfg, mpcd_ckpt **out) {
    if (!cfg || !out) return MPCD_ERR_ARG;
    *out = nullptr;
    double vol0;
    int r = mpcd_accessible_volume(cfg, 0, &vol0);  // validates cfg
    if (r != MPCD_OK) return r;
    mpcd_ckpt *c = new mpcd_ckpt();
    for (int l = 0; l < kNHead; l++) c->lines.push_back(blank_line(kHead[l]));
    c->nspec = cfg->n_species;
    c->nbc = cfg->n_walls;
    c->gpop = 0;
    c->ns = 0;
    lay_out(*c);
    const int D = cfg->dim;
    int XYZ[3];
    for (int d = 0; d < 3; d++) XYZ[d] = d < D ? cfg->L[d] : 1;
    c->set_f(L_WARM, 1, cfg->dt);
    c->set_i(L_SEED, 0, (long long)cfg->seed);
    c->set_i(L_DIM, 0, D);
    for (int d = 0; d < 3; d++) c->set_i(L_DIM, 1 + d, XYZ[d]);
    c->set_f(L_DIM, 4, cfg->kbt);
    c->set_f(L_DIM, 5, cfg->kbt);
    c->set_i(L_FLAGS, 2, cfg->galinv);
    c->set_i(L_FLAGS, 4, cfg->coll_op);
    c->set_i(L_FLAGS, 5, cfg->lc);
    c->set_i(L_STEPS, 0, 2000);  // readJson defaults (read.c:1058-1130)
    c->set_f(L_ANG, 0, cfg->relax);  // TAU
    c->set_f(L_ANG, 1, cfg->rot_ang);
    c->set_f(L_ANG, 2, cfg->fricco);  // FRICCO
    for (int d = 0; d < 3; d++) c->set_f(L_GRAV, d, cfg->grav[d]);
    c->set_i(L_MD, 1, 20);  // stepsMD
    c->set_i(L_POP, 1, cfg->n_species);
    c->set_f(L_RUN, 2, std::cos(cfg->rot_ang));  // initvar (init.c:1194-1195)
    c->set_f(L_RUN, 3, std::sin(cfg->rot_ang));
    c->set_i(L_RUN, 4, !(feq0(cfg->grav[0]) && feq0(cfg->grav[1]) && feq0(cfg->grav[2])));
    c->set_f(L_RUN, 6, 0.01);  // tolD
    double box = 1.0;
    for (int d = 0; d < D; d++) box *= XYZ[d];
    c->set_f(L_AVG, 7, box);  // VOL
    for (int s = 0; s < cfg->n_species; s++) {
        const mpcd_species &sp = cfg->species[s];
        const int l = c->spec_line(s);
        const double vals[20] = {sp.mass, 0, 0, 0, 0, sp.rfc, 0.007, sp.tumble, sp.chihi, 0,
                                 sp.act, sp.mfpot, sp.sigwidth, sp.sigpos, sp.damp, 0, 0, 0,
                                 sp.minactratio, 0};
        for (int k = 0; k < 20; k++) {
            if (k >= 1 && k <= 4) continue;  // POP QDIST VDIST ODIST: integers
            c->set_f(l, k, vals[k]);
        }
        c->set_i(l, 4, 2);  // ODIST (readJson default)
        double v = 0.0;
        mpcd_accessible_volume(cfg, s, &v);
        c->set_f(l, 15, v);
    }
    c->set_f(c->dens, 0, cfg->gndnst);
    c->set_i(c->dens, 3, (int)std::sqrt((double)(XYZ[0] * XYZ[0] + XYZ[1] * XYZ[1] + XYZ[2] * XYZ[2])));
    c->set_i(c->dens + 1, 0, cfg->n_walls);
    for (int w = 0; w < cfg->n_walls; w++) {
        const mpcd_wall &wl = cfg->walls[w];
        c->set_i(c->wall_line(w, 0), 0, wl.coll_type);
        c->set_i(c->wall_line(w, 0), 1, wl.phantom);
        c->set_f(c->wall_line(w, 0), 2, -1.0);  // E
        for (int d = 0; d < 3; d++) {
            c->set_f(c->wall_line(w, 0), 3 + d, wl.Q[d]);
            c->set_f(c->wall_line(w, 1), 6 + d, wl.A[d]);
            c->set_f(c->wall_line(w, 1), 9 + d, wl.A[d] != 0.0 ? 1.0 / wl.A[d] : 0.0);
            c->set_f(c->wall_line(w, 2), 4 + d, wl.DVxyz[d]);
            c->set_f(c->wall_line(w, 2), 11 + d, wl.MUxyz[d]);
            c->set_f(c->wall_line(w, 3), d, wl.DUxyz[d]);
        }
        for (int k = 0; k < 4; k++) c->set_f(c->wall_line(w, 1), 12 + k, 1.0);  // P
        c->set_f(c->wall_line(w, 1), 16, wl.R);
        const double w3[4] = {wl.DN, wl.DT, wl.DVN, wl.DVT};
        for (int k = 0; k < 4; k++) c->set_f(c->wall_line(w, 2), k, w3[k]);
        c->set_f(c->wall_line(w, 2), 7, wl.MVN);
        c->set_f(c->wall_line(w, 2), 8, wl.MVT);
        c->set_f(c->wall_line(w, 2), 9, wl.MUN);
        c->set_f(c->wall_line(w, 2), 10, wl.MUT);
        c->set_f(c->wall_line(w, 3), 3, 1.0);  // KBT
        c->set_i(c->wall_line(w, 3), 5, wl.inv);
        c->set_f(c->wall_line(w, 3), 6, 1.0);  // MASS
        c->set_i(c->wall_line(w, 5), 0, 1);    // PLANAR
        c->set_f(c->wall_line(w, 5), 3, 4.0);  // ROTSYMM
        c->set_f(c->wall_line(w, 5), 4, 4.0);
        for (int s = 0; s < MPCD_MAX_SPECIES; s++) c->set_i(c->wall_line(w, 7), s, wl.inter[s]);
        c->set_i(c->wall_line(w, 7), MPCD_MAX_SPECIES, 1);  // BCON for the MD and swimmer slots
        c->set_i(c->wall_line(w, 7), MPCD_MAX_SPECIES + 1, 1);
    }
    *out = c;
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_config(const mpcd_ckpt *ck, mpcd_config *cfg) {
    if (!ck || !cfg) return MPCD_ERR_ARG;
    memset(cfg, 0, sizeof(*cfg));
    const int D = (int)ck->i(L_DIM, 0);
    if (D != 2 && D != 3) return MPCD_ERR_UNSUPPORTED;
    if (ck->nspec < 1 || ck->nspec > MPCD_MAX_SPECIES || ck->nbc > MPCD_MAX_WALLS)
        return MPCD_ERR_UNSUPPORTED;
    // features outside the library's timestep
    if (ck->i(L_MD, 0) != 0 || ck->ns != 0) return MPCD_ERR_UNSUPPORTED;  // MD, swimmers
    if (ck->i(L_FLAGS, 3) != 0) return MPCD_ERR_UNSUPPORTED;              // thermostat
    if (ck->i(L_HI, 0) != 0 || ck->i(L_HI, 1) != 0 || ck->i(L_HI, 2) != 0)
        return MPCD_ERR_UNSUPPORTED;  // noHI, incompressibility, multiphase
    for (int d = 0; d < 3; d++)
        if (!feq0(ck->f(L_MAG, d))) return MPCD_ERR_UNSUPPORTED;  // magnetic field
    cfg->dim = D;
    for (int d = 0; d < 3; d++) cfg->L[d] = (int)ck->i(L_DIM, 1 + d);
    cfg->dt = ck->f(L_WARM, 1);
    cfg->kbt = ck->f(L_DIM, 4);
    cfg->galinv = (int)ck->i(L_FLAGS, 2);
    cfg->coll_op = (int)ck->i(L_FLAGS, 4);
    cfg->lc = (int)ck->i(L_FLAGS, 5);
    cfg->rot_ang = ck->f(L_ANG, 1);
    cfg->fricco = ck->f(L_ANG, 2);
    cfg->relax = ck->f(L_ANG, 0);
    for (int d = 0; d < 3; d++) cfg->grav[d] = ck->f(L_GRAV, d);
    cfg->gndnst = ck->f(ck->dens, 0);
    cfg->seed = (uint64_t)ck->i(L_SEED, 0);
    cfg->precision = MPCD_PREC_FP64;
    cfg->n_species = ck->nspec;
    for (int s = 0; s < ck->nspec; s++) {
        const int l = ck->spec_line(s);
        mpcd_species &sp = cfg->species[s];
        sp.mass = ck->f(l, 0);
        sp.rfc = ck->f(l, 5);
        sp.tumble = ck->f(l, 7);
        sp.chihi = ck->f(l, 8);
        sp.act = ck->f(l, 10);
        sp.mfpot = ck->f(l, 11);
        sp.sigwidth = ck->f(l, 12);
        sp.sigpos = ck->f(l, 13);
        sp.damp = ck->f(l, 14);
        sp.minactratio = ck->f(l, 18);
    }
    cfg->n_walls = ck->nbc;
    for (int w = 0; w < ck->nbc; w++) {
        mpcd_wall &wl = cfg->walls[w];
        // static, unrotated planes only: no displacement, velocity, angular
        // velocity or orientation, powers 1 (a plane)
        if (ck->i(ck->wall_line(w, 3), 4) != 0) return MPCD_ERR_UNSUPPORTED;  // DSPLC
        for (int d = 0; d < 3; d++)
            if (!feq0(ck->f(ck->wall_line(w, 0), 6 + d)) ||
                !feq0(ck->f(ck->wall_line(w, 0), 9 + d)) ||
                !feq0(ck->f(ck->wall_line(w, 1), d)))
                return MPCD_ERR_UNSUPPORTED;
        for (int k = 0; k < 4; k++)
            if (!feq0(ck->f(ck->wall_line(w, 1), 12 + k) - 1.0)) return MPCD_ERR_UNSUPPORTED;
        wl.coll_type = (int)ck->i(ck->wall_line(w, 0), 0);
        wl.phantom = (int)ck->i(ck->wall_line(w, 0), 1);
        for (int d = 0; d < 3; d++) {
            wl.Q[d] = ck->f(ck->wall_line(w, 0), 3 + d);
            wl.A[d] = ck->f(ck->wall_line(w, 1), 6 + d);
            wl.DVxyz[d] = ck->f(ck->wall_line(w, 2), 4 + d);
            wl.MUxyz[d] = ck->f(ck->wall_line(w, 2), 11 + d);
            wl.DUxyz[d] = ck->f(ck->wall_line(w, 3), d);
        }
        wl.R = ck->f(ck->wall_line(w, 1), 16);
        wl.DN = ck->f(ck->wall_line(w, 2), 0);
        wl.DT = ck->f(ck->wall_line(w, 2), 1);
        wl.DVN = ck->f(ck->wall_line(w, 2), 2);
        wl.DVT = ck->f(ck->wall_line(w, 2), 3);
        wl.MVN = ck->f(ck->wall_line(w, 2), 7);
        wl.MVT = ck->f(ck->wall_line(w, 2), 8);
        wl.MUN = ck->f(ck->wall_line(w, 2), 9);
        wl.MUT = ck->f(ck->wall_line(w, 2), 10);
        wl.inv = (int)ck->i(ck->wall_line(w, 3), 5);
        for (int s = 0; s < MPCD_MAX_SPECIES; s++)
            wl.inter[s] = (int)ck->i(ck->wall_line(w, 7), s);
    }
    // the timestep's own checks (collision operator, wall forms, sizes)
    double v;
    return mpcd_accessible_volume(cfg, 0, &v);
}

extern "C" int mpcd_ckpt_get_run(const mpcd_ckpt *ck, mpcd_ckpt_run *run) {
    if (!ck || !run) return MPCD_ERR_ARG;
    run->sim_steps = (int)ck->i(L_STEPS, 0);
    run->warmup_steps = (int)ck->i(L_WARM, 0);
    run->runtime = (int)ck->i(L_RUN, 0);
    run->warmtime = (int)ck->i(L_RUN, 1);
    run->kbtnow = ck->f(L_DIM, 5);
    for (int d = 0; d < 3; d++) {
        run->avv[d] = ck->f(L_AVV, d);
        run->avnow[d] = ck->f(L_AVV, 3 + d);
    }
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_set_run(mpcd_ckpt *ck, const mpcd_ckpt_run *run) {
    if (!ck || !run) return MPCD_ERR_ARG;
    ck->set_i(L_STEPS, 0, run->sim_steps);
    ck->set_i(L_WARM, 0, run->warmup_steps);
    ck->set_i(L_RUN, 0, run->runtime);
    ck->set_i(L_RUN, 1, run->warmtime);
    ck->set_f(L_DIM, 5, run->kbtnow);
    for (int d = 0; d < 3; d++) {
        ck->set_f(L_AVV, d, run->avv[d]);
        ck->set_f(L_AVV, 3 + d, run->avnow[d]);
    }
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_count(const mpcd_ckpt *ck, int *n) {
    if (!ck || !n) return MPCD_ERR_ARG;
    *n = ck->gpop;
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_particles(const mpcd_ckpt *ck, double *Q, double *V, double *U,
                                   int *spid) {
    if (!ck) return MPCD_ERR_ARG;
    for (int p = 0; p < ck->gpop; p++) {
        const int l = ck->part_line(p);
        for (int d = 0; d < 3; d++) {
            if (Q) Q[3 * (size_t)p + d] = ck->f(l, 3 + d);
            if (V) V[3 * (size_t)p + d] = ck->f(l, 6 + d);
            if (U) U[3 * (size_t)p + d] = ck->f(l, 9 + d);
        }
        if (spid) spid[p] = (int)ck->i(l, 1);
    }
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_upload(const mpcd_ckpt *ck, mpcd_handle *h) {
    if (!ck || !h) return MPCD_ERR_ARG;
    const size_t n = (size_t)ck->gpop;
    std::vector<double> Q(3 * n), V(3 * n), U(3 * n);
    std::vector<int> sp(n);
    mpcd_ckpt_particles(ck, Q.data(), V.data(), U.data(), sp.data());
    // the species' VDIST for the bounce-limit re-thermalisation
    int vdist[MPCD_MAX_SPECIES] = {0};
    for (int s = 0; s < ck->nspec && s < MPCD_MAX_SPECIES; s++) {
        vdist[s] = (int)ck->i(ck->spec_line(s), 3);
        // READ (1) has no file to read from at a re-thermalisation (the
        // reference would read from a null file there): uniform instead
        if (vdist[s] == 1) vdist[s] = MPCD_VDIST_RANDVEL;
    }
    int r = mpcd_set_species_vdist(h, vdist);
    if (r != MPCD_OK) return r;
    return mpcd_upload_state(h, ck->gpop, Q.data(), V.data(), U.data(), sp.data());
}

// Replace the particle block; U == nullptr keeps the file's orientations
// (zero for new particles).
static int set_particles(mpcd_ckpt *ck, int n, const double *Q, const double *V, const double *U,
                         const int *spid) {
    for (int p = 0; p < n; p++)
        if (spid && (spid[p] < 0 || spid[p] >= ck->nspec)) return MPCD_ERR_ARG;
    if (n != ck->gpop) {
        // rebuild the particle block for the new count
        std::vector<Line> swim(ck->lines.begin() + ck->swim0, ck->lines.end());
        ck->lines.resize((size_t)ck->part0);
        for (int p = 0; p < n; p++) {
            Line ln = blank_line(kPart);
            ln.v[0].i = 1;  // S_flag = STREAM (init.c:1601)
            ck->lines.push_back(ln);
        }
        ck->swim0 = (int)ck->lines.size();
        ck->lines.insert(ck->lines.end(), swim.begin(), swim.end());
        ck->gpop = n;
    }
    std::vector<long long> pop((size_t)ck->nspec, 0);
    for (int p = 0; p < n; p++) {
        const int l = ck->part_line(p);
        const int sp = spid ? spid[p] : 0;
        ck->set_i(l, 1, sp);
        pop[(size_t)sp]++;
        for (int d = 0; d < 3; d++) {
            ck->set_f(l, 3 + d, Q[3 * (size_t)p + d]);
            ck->set_f(l, 6 + d, V[3 * (size_t)p + d]);
            if (U) ck->set_f(l, 9 + d, U[3 * (size_t)p + d]);
        }
    }
    ck->set_i(L_POP, 0, n);
    for (int s = 0; s < ck->nspec; s++) ck->set_i(ck->spec_line(s), 1, pop[(size_t)s]);
    return MPCD_OK;
}

extern "C" int mpcd_ckpt_set_particles(mpcd_ckpt *ck, int n, const double *Q, const double *V,
                                       const double *U, const int *spid) {
    if (!ck || n < 0 || (n > 0 && (!Q || !V))) return MPCD_ERR_ARG;
    if (U) return set_particles(ck, n, Q, V, U, spid);
    // no orientations given: zero
    std::vector<double> Z(3 * (size_t)n, 0.0);
    return set_particles(ck, n, Q, V, Z.data(), spid);
}

extern "C" int mpcd_ckpt_capture(mpcd_ckpt *ck, mpcd_handle *h) {
    if (!ck || !h) return MPCD_ERR_ARG;
    int n = 0;
    int r = mpcd_particle_count(h, &n);
    if (r != MPCD_OK) return r;
    const size_t N = (size_t)n;
    std::vector<double> Q(3 * N), V(3 * N), U(3 * N);
    std::vector<int> sp(N);
    if ((r = mpcd_download_state(h, Q.data(), V.data(), U.data())) != MPCD_OK) return r;
    if ((r = mpcd_download_species(h, sp.data())) != MPCD_OK) return r;
    mpcd_config hc;
    if ((r = mpcd_get_config(h, &hc)) != MPCD_OK) return r;
    ck->set_f(ck->dens, 0, hc.gndnst);  // GnDNST, as the reference carries it
    // an isotropic state downloads zero orientations: keep the file's then
    bool oriented = false;
    for (size_t k = 0; k < 3 * N && !oriented; k++) oriented = U[k] != 0.0;
    if (!oriented && n == ck->gpop) return set_particles(ck, n, Q.data(), V.data(), nullptr, sp.data());
    return set_particles(ck, n, Q.data(), V.data(), U.data(), sp.data());
}
