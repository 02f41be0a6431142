// mpcd_tune.cu -- the autotuner's cache: execution plans chosen by
// mpcd_autotune, keyed by device and workload, kept in a text file between
// runs.  Host code only (no GPU needed), so the cache logic is testable
// anywhere.
//
// File format: one plan per line, tab-separated:
//   key  kernel  strategy  tile_particles  sort_interval  us_per_step
// Lines that do not parse are skipped; the last line of a key wins, so a
// re-tune appends rather than rewrites.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "mpcd_gpu.h"

extern "C" int mpcd_tune_key(const mpcd_config *cfg, int n, const char *device, char *key,
                             size_t len) {
    if (!cfg || !device || !key || len == 0 || n < 0) return MPCD_ERR_ARG;
    int solid = 0, phantom = 0;
    for (int w = 0; w < cfg->n_walls && w < MPCD_MAX_WALLS; w++) {
        const mpcd_wall &wl = cfg->walls[w];
        const bool periodic = wl.MVN > 0.0 && wl.MVT > 0.0 && (wl.DN != 0.0 || wl.DT != 0.0);
        if (!periodic) solid++;
        if (wl.phantom) phantom++;
    }
    const bool grav = cfg->grav[0] != 0.0 || cfg->grav[1] != 0.0 || cfg->grav[2] != 0.0;
    std::string dev(device);
    for (char &ch : dev)
        if (ch == '\t' || ch == '\n' || ch == '|') ch = '_';
    const int w = snprintf(key, len, "%s|dim=%d|L=%dx%dx%d|n=%d|op=%d|lc=%d|prec=%d|solid=%d|"
                                     "phantom=%d|species=%d|grav=%d",
                           dev.c_str(), cfg->dim, cfg->L[0], cfg->L[1],
                           cfg->dim == 3 ? cfg->L[2] : 1, n, cfg->coll_op, cfg->lc,
                           cfg->precision, solid, phantom, cfg->n_species, grav ? 1 : 0);
    return (w < 0 || (size_t)w >= len) ? MPCD_ERR_SIZE : MPCD_OK;
}

extern "C" int mpcd_tune_cache_lookup(const char *path, const char *key, mpcd_tune_choice *out) {
    if (!path || !key || !out) return MPCD_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return 0;
    char line[1024];
    int found = 0;
    const size_t klen = strlen(key);
    while (fgets(line, sizeof(line), f)) {
        if (strncmp(line, key, klen) != 0 || line[klen] != '\t') continue;
        mpcd_tune_choice c;
        memset(&c, 0, sizeof(c));
        if (sscanf(line + klen + 1, "%d\t%d\t%d\t%d\t%lf", &c.kernel, &c.strategy,
                   &c.tile_particles, &c.sort_interval, &c.us_per_step) != 5)
            continue;
        if (c.kernel < MPCD_KERNEL_AUTO || c.kernel > MPCD_KERNEL_PERSIST) continue;
        c.from_cache = 1;
        *out = c;
        found = 1;
    }
    fclose(f);
    return found;
}

extern "C" int mpcd_tune_cache_store(const char *path, const char *key,
                                     const mpcd_tune_choice *c) {
    if (!path || !key || !c || strchr(key, '\t') || strchr(key, '\n')) return MPCD_ERR_ARG;
    FILE *f = fopen(path, "a");
    if (!f) return MPCD_ERR_ARG;
    const int w = fprintf(f, "%s\t%d\t%d\t%d\t%d\t%.3f\n", key, c->kernel, c->strategy,
                          c->tile_particles, c->sort_interval, c->us_per_step);
    const int e = fclose(f);
    return (w < 0 || e != 0) ? MPCD_ERR_ARG : MPCD_OK;
}
