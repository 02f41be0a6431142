// mpcd_api.cu -- the C ABI of libmpcd_gpu.so (declared in include/mpcd_gpu.h).
//
// A handle owns the particle state in device memory, two state buffers (the
// counting sort writes the cell-ordered copy into the other one), the cell
// count/start arrays and the per-step accumulators, all on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mpcd_gpu.h"
#include "mpcd_device.cuh"
#include "mpcd_fp64.cuh"
#include "mpcd_mixed.cuh"
#include "mpcd_tile.cuh"
#include "mpcd_group.cuh"
#include "mpcd_split.cuh"
#include "mpcd_resident.cuh"
#include "mpcd_resident64.cuh"
#include "mpcd_lc.cuh"
#include "mpcd_xfer.cuh"
#include "mpcd_persist.cuh"
#include "mpcd_init.cuh"

using namespace mpcd;

struct mpcd_handle {
    mpcd_config cfg;
    DevCfg dc;
    int device;
    cudaStream_t stream;
    bool own_stream;
    int n;
    int cap;
    int prec;
    Fp64State f[2];  // FP64 state, two buffers (the sort writes the other)
    MixState mx[2];  // mixed state, two buffers
    int cur;
    int *key, *rank, *count, *fill, *start[2], *part;
    int *perm;  // destination -> source index of a reordering (mixed state)
    int scur;        // which start[] belongs to the current order
    double *acc;     // 2 x ACC_WORDS, by step parity
    unsigned long long *status;
    int nscan;       // scan tiles of the largest key space
    int nkeys;       // keys the counting sort may use: cells, or the bricks' slots
    int sm_count;
    int smem_optin;  // largest dynamic shared memory a block may opt in to
    int launches;
    int strategy;    // MPCD_STRATEGY_*
    int tile_target; // expected particles per tile
    int kernel;      // MPCD_KERNEL_*: cell kernel family
    void *crec;      // per-cell SRD records (split kernel family)
    LcCells lcc;     // per-cell nematic arrays (lc != 0)
    double *lcbuf;
    double *modes;   // transverse momentum modes (mpcd_transverse_modes)
    bool stepped;        // a step ran since the last upload (mpcd_debug_cell_counts)
    double *props;       // mpcd_cell_props accumulators: 7 doubles + (1 + species) ints per cell
    double *flow;        // flow field running sum, 3 doubles per cell (null: off)
    long long flow_steps;  // steps summed into flow
    double *host_ring;   // pinned: per-step globals of mpcd_step_record
    int per_blocks;      // persistent family: blocks of the launch (0: not planned, -1: unfit)
    int per_planned_n;   // particle count the plan was made for
    int *per_pop;        // persistent family: populations of the next step's cells
    void *per_work;      // persistent family: sums, populations, records, barrier counter
    int64_t per_pop_for; // step whose cells per_pop counts; -1 none
    bool res_attr;       // the resident kernels' shared-memory attributes are set
    int r64_per_sm;      // resident blocks per SM of the FP64 particle pass (0: not yet known)
    void *xfer;          // device staging of FP64 uploads and downloads (mixed form)
    size_t xfer_bytes;
    int64_t sorted_for;  // step whose shifted grid the current order bins; -1 none
    ResSum *rsum;              // resident family: cell sums, two steps by parity
    double *r64sum;            // FP64 resident family: M, p[3] sums (4 x nc), two steps by parity
    int *r64pop;               // FP64 resident family: populations, two steps by parity
    unsigned long long *rmsum;  // resident family: mass sums (several species)
    int64_t sums_for;          // step whose cell sums rsum holds; -1 none
    int sort_interval;         // resident family: steps between re-sorts
    int sort_age;              // steps since the last sort; -1 unknown
    uint32_t last_step;
    uint64_t steps;
    double *host_acc;  // pinned
    // optional timing of the step's particle pass (the dominant kernel):
    // an event pair around each of its launches, summed on request
    bool timing;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tev;
};

static void time_begin(mpcd_handle *h) {
    if (!h->timing) return;
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return;
    }
    cudaEventRecord(a, h->stream);
    h->tev.emplace_back(a, b);
}
static void time_end(mpcd_handle *h) {
    if (!h->timing || h->tev.empty()) return;
    cudaEventRecord(h->tev.back().second, h->stream);
}
static void time_clear(mpcd_handle *h) {
    for (auto &p : h->tev) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    h->tev.clear();
}

// Per-step global accumulators (ACC_KE, ACC_VCM) live in a ring of
// kAccRing slots indexed by the step number: the kernels of step t clear
// the slot of step t + 1, so the slots of the last kAccRing - 1 steps stay
// readable (mpcd_step_record reads them in batches).
constexpr int kAccRing = 128;
constexpr int kRecordBatch = 32;  // steps per read-back of mpcd_step_record
static_assert(2 * kRecordBatch < kAccRing, "a batch is read while the next one runs");
static double *acc_at(const mpcd_handle *h, uint32_t step) {
    return h->acc + (size_t)(step % (uint32_t)kAccRing) * ACC_WORDS;
}

#define CK(call)                                                        \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) {                                        \
            fprintf(stderr, "mpcd: %s failed: %s\n", #call,             \
                    cudaGetErrorString(e_));                            \
            return MPCD_ERR_CUDA;                                       \
        }                                                               \
    } while (0)

static int dev_alloc(void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? MPCD_ERR_NOMEM : MPCD_ERR_CUDA;
    }
    return MPCD_OK;
}

#define ALLOC(ptr, bytes)                                        \
    do {                                                         \
        int r_ = dev_alloc((void **)&(ptr), (bytes));            \
        if (r_ != MPCD_OK) {                                     \
            mpcd_destroy(h);                                     \
            return r_;                                           \
        }                                                        \
    } while (0)

static bool is_periodic_wall(const mpcd_wall &w) {
    // setPBC, read.c:584-603
    for (int d = 0; d < 3; d++)
        if (std::fabs(std::fabs(w.A[d]) - 1.0) <= kTol && w.MVN > 0.0 && w.MVT > 0.0 &&
            (std::fabs(w.DN) >= kTol || std::fabs(w.DT) >= kTol))
            return true;
    return false;
}

static int build_devcfg(const mpcd_config *cfg, DevCfg *dc) {
    memset(dc, 0, sizeof(*dc));
    if (cfg->dim != 2 && cfg->dim != 3) return MPCD_ERR_UNSUPPORTED;
    if (cfg->n_species < 1 || cfg->n_species > MPCD_MAX_SPECIES) return MPCD_ERR_ARG;
    if (cfg->n_walls < 0 || cfg->n_walls > MPCD_MAX_WALLS) return MPCD_ERR_ARG;
    if (!(cfg->dt > 0.0) || !(cfg->kbt >= 0.0)) return MPCD_ERR_ARG;
    if (cfg->lc != MPCD_LC_ISOTROPIC && !(cfg->lc == MPCD_LC_LOCAL && cfg->dim == 2))
        return MPCD_ERR_UNSUPPORTED;
    if (cfg->lc == MPCD_LC_ISOTROPIC && !is_vcm_op(cfg->coll_op) &&
        !is_mpcat_op(cfg->coll_op) && cfg->coll_op != MPCD_COLL_RAT &&
        !is_lang_op(cfg->coll_op))
        return MPCD_ERR_UNSUPPORTED;
    if (is_lang_op(cfg->coll_op) && !(cfg->fricco >= 0.0)) return MPCD_ERR_ARG;
    // Chate's director needs the order tensor's eigenvectors: 2x2 only here
    if ((cfg->coll_op == MPCD_COLL_CHATE || cfg->coll_op == MPCD_COLL_CHATE_MPCAT) &&
        cfg->dim != 2)
        return MPCD_ERR_UNSUPPORTED;
    dc->dim = cfg->dim;
    dc->op = cfg->coll_op;
    dc->lc = cfg->lc;
    dc->galinv = cfg->galinv;
    for (int d = 0; d < 3; d++) {
        int L = d < cfg->dim ? cfg->L[d] : 1;
        if (L < 1) return MPCD_ERR_ARG;
        dc->L[d] = L;
        dc->N1[d] = L + 1;
    }
    long long nc = (long long)dc->N1[0] * dc->N1[1] * dc->N1[2];
    if (nc > (1LL << 30)) return MPCD_ERR_SIZE;
    dc->ncells = (int)nc;
    dc->vol = 1.0;
    for (int d = 0; d < cfg->dim; d++) dc->vol *= dc->L[d];
    dc->n_species = cfg->n_species;
    for (int s = 0; s < cfg->n_species; s++) {
        if (!(cfg->species[s].mass > 0.0)) return MPCD_ERR_ARG;
        dc->mass[s] = cfg->species[s].mass;
        dc->sig[s] = std::sqrt(cfg->kbt / cfg->species[s].mass);
        {
            // as langevinMPC and vicsekLangevinMPC evaluate them (mpc.c:1744-1745)
            const double M = cfg->species[s].mass, F = cfg->fricco, step = cfg->dt;
            dc->lang_a[s] = (M - F * step * 0.5) / (M + 0.5 * F * step);
            dc->lang_b[s] = std::sqrt(F * step) / (M + 0.5 * F * step);
            if (cfg->coll_op == MPCD_COLL_VICSEK_MPCAT) {
                // V' = VCM + (RV - RS) + alignment: the Langevin update's form
                dc->lang_a[s] = 0.0;
                dc->lang_b[s] = 1.0;
            }
        }
        // the Vicsek- and Chate-aligned operators apply no damping (mpc.c:2204-2480)
        dc->damp[s] = is_vicsek_op(cfg->coll_op) || cfg->coll_op == MPCD_COLL_CHATE_MPCAT
                          ? 0.0
                          : cfg->species[s].damp;
        dc->rfc[s] = cfg->species[s].rfc;
        dc->tumble[s] = cfg->species[s].tumble;
        dc->chihi[s] = cfg->species[s].chihi;
        dc->act[s] = cfg->species[s].act;
        dc->mfpot[s] = cfg->species[s].mfpot;
        dc->sigwidth[s] = cfg->species[s].sigwidth;
        dc->sigpos[s] = cfg->species[s].sigpos;
        dc->minactratio[s] = cfg->species[s].minactratio;
    }
    // activeSRD takes the cell's activity from the last particle of the
    // cell's linked list (sumACT = ACT, mpc.c:2058-2062), an order that the
    // reference's re-binning history sets: only species of one activity give
    // a result that does not depend on it.
    dc->act_srd = cfg->lc == MPCD_LC_ISOTROPIC && (cfg->coll_op == MPCD_COLL_ACT_ARBAXIS ||
                                                   cfg->coll_op == MPCD_COLL_ACT_ORTHAXIS);
    if (dc->act_srd)
        for (int s = 1; s < cfg->n_species; s++)
            if (cfg->species[s].act != cfg->species[0].act) return MPCD_ERR_UNSUPPORTED;
    dc->dt = cfg->dt;
    dc->kbt = cfg->kbt;
    dc->relax = cfg->relax;
    dc->cosA = std::cos(cfg->rot_ang);
    dc->sinA = -1.0 * std::sin(cfg->rot_ang);  // rotation sign draw is always 0
    for (int d = 0; d < 3; d++) dc->grav[d] = cfg->grav[d];
    dc->grav_flag = std::fabs(cfg->grav[0]) >= kTol || std::fabs(cfg->grav[1]) >= kTol ||
                    std::fabs(cfg->grav[2]) >= kTol;
    dc->seed = cfg->seed;
    dc->replica = cfg->replica;
    dc->n_walls = cfg->n_walls;
    for (int w = 0; w < cfg->n_walls; w++) {
        const mpcd_wall &src = cfg->walls[w];
        DevWall &dst = dc->walls[w];
        int nz = 0, ax = 0;
        for (int d = 0; d < 3; d++)
            if (src.A[d] != 0.0) {
                nz++;
                ax = d;
            }
        // static axis-aligned planes with rule-based collisions only
        if (nz != 1 || src.coll_type != 1) return MPCD_ERR_UNSUPPORTED;
        for (int d = 0; d < 3; d++) {
            dst.A[d] = src.A[d];
            dst.Q[d] = src.Q[d];
            dst.DVxyz[d] = src.DVxyz[d];
            dst.MUxyz[d] = src.MUxyz[d];
            dst.DUxyz[d] = src.DUxyz[d];
        }
        dst.MUN = src.MUN;
        dst.MUT = src.MUT;
        // nematic anchoring by phantom walls (ghostPart's ghost anchoring) is
        // not implemented
        if (cfg->lc && src.phantom && (std::fabs(src.MUN) <= kTol || std::fabs(src.MUT) <= kTol))
            return MPCD_ERR_UNSUPPORTED;
        dst.R = src.R;
        dst.DN = src.DN;
        dst.DT = src.DT;
        dst.DVN = src.DVN;
        dst.DVT = src.DVT;
        dst.MVN = src.MVN;
        dst.MVT = src.MVT;
        dst.inv = src.inv;
        dst.phantom = src.phantom;
        dst.axis = ax;
        dst.periodic = is_periodic_wall(src) ? 1 : 0;
        uint32_t m = 0;
        for (int s = 0; s < MPCD_MAX_SPECIES; s++)
            if (src.inter[s]) m |= 1u << s;
        dst.inter = m;
        if (dst.phantom) dc->any_phantom = 1;
        if (!dst.periodic) dc->n_solid++;
        if (dst.periodic) dc->pbc[ax] = 1;
    }
    dc->gndnst = cfg->gndnst;
    dc->all_periodic = dc->n_solid == 0;
    for (int d = 0; d < cfg->dim; d++)
        if (!dc->pbc[d]) dc->all_periodic = 0;
    res_slot_bits(dc->dim, dc->L, dc->res_shift, dc->res_mask);
    return MPCD_OK;
}

// Configuration check and device form, shared with the allocation-free
// entry point (mpcd_noalloc.cu).
int mpcd_build_devcfg(const mpcd_config *cfg, DevCfg *dc) { return build_devcfg(cfg, dc); }

extern "C" int mpcd_abi_version(void) { return MPCD_ABI_VERSION; }

extern "C" int mpcd_destroy(mpcd_handle *h) {
    if (!h) return MPCD_ERR_ARG;
    for (int b = 0; b < 2; b++) {
        for (int d = 0; d < 3; d++) {
            cudaFree(h->f[b].q[d]);
            cudaFree(h->f[b].v[d]);
        }
        cudaFree(h->f[b].pid);
        cudaFree(h->f[b].sp);
        cudaFree(h->f[b].u[0]);
        cudaFree(h->f[b].u[1]);
        mix_free(h->mx[b]);
    }
    cudaFree(h->key);
    cudaFree(h->rank);
    cudaFree(h->perm);
    cudaFree(h->count);
    cudaFree(h->fill);
    cudaFree(h->start[0]);
    cudaFree(h->start[1]);
    cudaFree(h->part);
    cudaFree(h->acc);
    cudaFree(h->status);
    cudaFree(h->crec);
    cudaFree(h->modes);
    cudaFree(h->xfer);
    cudaFree(h->rsum);
    cudaFree(h->rmsum);
    cudaFree(h->r64sum);
    cudaFree(h->r64pop);
    cudaFree(h->lcbuf);
    cudaFree(h->props);
    cudaFree(h->flow);
    cudaFree(h->per_pop);
    cudaFree(h->per_work);
    if (h->host_acc) cudaFreeHost(h->host_acc);
    if (h->host_ring) cudaFreeHost(h->host_ring);
    time_clear(h);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MPCD_OK;
}

extern "C" int mpcd_create(const mpcd_config *cfg, mpcd_handle **out) {
    if (!cfg || !out) return MPCD_ERR_ARG;
    *out = nullptr;
    DevCfg dc;
    int r = build_devcfg(cfg, &dc);
    if (r != MPCD_OK) return r;
    if (cfg->capacity < 0) return MPCD_ERR_ARG;
    if (cfg->precision != MPCD_PREC_FP64 && cfg->precision != MPCD_PREC_MIXED)
        return MPCD_ERR_ARG;
    if (cfg->precision == MPCD_PREC_MIXED) {
        r = mix_check(dc);
        if (r != MPCD_OK) return r;
    }
    mpcd_handle *h = new mpcd_handle();
    h->cfg = *cfg;
    h->dc = dc;
    h->prec = cfg->precision;
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return MPCD_ERR_CUDA;
    }
    h->own_stream = true;
    int nc = dc.ncells;
    // the 3D resident family sorts by brick (k_key_res3): its key space
    h->nkeys = nc;
    if (cfg->precision == MPCD_PREC_MIXED && !dc.lc && dc.dim == 3)
        h->nkeys = std::max(nc, res_brick_keys(dc.N1));
    const int nk = h->nkeys;
    h->nscan = (nk + kScanTile - 1) / kScanTile;
    ALLOC(h->count, sizeof(int) * nk);
    ALLOC(h->fill, sizeof(int) * nk);
    ALLOC(h->start[0], sizeof(int) * (nk + 1));
    ALLOC(h->start[1], sizeof(int) * (nk + 1));
    ALLOC(h->part, sizeof(int) * h->nscan);
    ALLOC(h->acc, sizeof(double) * kAccRing * ACC_WORDS);
    ALLOC(h->status, sizeof(unsigned long long) * ST_WORDS);
    ALLOC(h->crec, (size_t)nc * 128);
    if (cfg->precision == MPCD_PREC_MIXED && !dc.lc) {
        ALLOC(h->rsum, sizeof(ResSum) * 2 * (size_t)nc);
        if (dc.n_species > 1) ALLOC(h->rmsum, sizeof(unsigned long long) * 2 * (size_t)nc);
    }
    if (cfg->precision == MPCD_PREC_FP64 && !dc.lc) {
        ALLOC(h->r64sum, sizeof(double) * 8 * (size_t)nc);
        ALLOC(h->r64pop, sizeof(int) * 2 * (size_t)nc);
    }
    if (dc.lc) {
        ALLOC(h->lcbuf, (size_t)nc * 13 * sizeof(double));
        if (cudaMemsetAsync(h->lcbuf, 0, (size_t)nc * 13 * sizeof(double), h->stream) !=
            cudaSuccess) {
            mpcd_destroy(h);
            return MPCD_ERR_CUDA;
        }
        double *b = h->lcbuf;
        h->lcc.vcm = b;
        h->lcc.cm = b + 2 * (size_t)nc;
        h->lcc.izz = b + 4 * (size_t)nc;
        h->lcc.mass = b + 5 * (size_t)nc;
        h->lcc.S = b + 6 * (size_t)nc;
        h->lcc.dir = b + 7 * (size_t)nc;
        h->lcc.E = b + 9 * (size_t)nc;
    }
    h->sorted_for = -1;
    h->sums_for = -1;
    h->per_pop_for = -1;
    h->sort_interval = 30;
    h->sort_age = -1;
    h->strategy = -1;
    h->tile_target = 0;
    if (cudaMemsetAsync(h->count, 0, sizeof(int) * nk, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->fill, 0, sizeof(int) * nk, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->status, 0, sizeof(unsigned long long) * ST_WORDS, h->stream) !=
            cudaSuccess ||
        cudaMemsetAsync(h->acc, 0, sizeof(double) * kAccRing * ACC_WORDS, h->stream) !=
            cudaSuccess) {
        mpcd_destroy(h);
        return MPCD_ERR_CUDA;
    }
    // pinned host buffers of the globals read-back (allocated here: a
    // pinned allocation costs milliseconds, too much inside a caller's loop)
    if (cudaMallocHost((void **)&h->host_acc, sizeof(double) * ACC_WORDS) != cudaSuccess ||
        cudaMallocHost((void **)&h->host_ring, sizeof(double) * 2 * kRecordBatch * ACC_WORDS) !=
            cudaSuccess) {
        mpcd_destroy(h);
        return MPCD_ERR_NOMEM;
    }
    *out = h;
    return MPCD_OK;
}

// (Re)allocate the per-particle arrays for n particles.
static int ensure_capacity(mpcd_handle *h, int n) {
    int want = n > h->cfg.capacity ? n : h->cfg.capacity;
    if (want <= h->cap) return MPCD_OK;
    for (int b = 0; b < 2; b++) {
        for (int d = 0; d < 3; d++) {
            cudaFree(h->f[b].q[d]);
            cudaFree(h->f[b].v[d]);
            h->f[b].q[d] = h->f[b].v[d] = nullptr;
        }
        cudaFree(h->f[b].pid);
        cudaFree(h->f[b].sp);
        h->f[b].pid = h->f[b].sp = nullptr;
        for (int d = 0; d < 2; d++) {
            cudaFree(h->f[b].u[d]);
            h->f[b].u[d] = nullptr;
        }
        mix_free(h->mx[b]);
    }
    cudaFree(h->key);
    cudaFree(h->rank);
    cudaFree(h->perm);
    h->key = h->rank = h->perm = nullptr;
    size_t N = (size_t)want;
    int r;
    for (int b = 0; b < 2; b++) {
        if (h->prec == MPCD_PREC_FP64) {
            for (int d = 0; d < h->dc.dim; d++) {
                if ((r = dev_alloc((void **)&h->f[b].q[d], N * sizeof(double)))) return r;
                if ((r = dev_alloc((void **)&h->f[b].v[d], N * sizeof(double)))) return r;
            }
            if ((r = dev_alloc((void **)&h->f[b].pid, N * sizeof(int)))) return r;
            if (h->dc.lc)
                for (int d = 0; d < 2; d++)
                    if ((r = dev_alloc((void **)&h->f[b].u[d], N * sizeof(double)))) return r;
            if (h->dc.n_species > 1)
                if ((r = dev_alloc((void **)&h->f[b].sp, N * sizeof(int)))) return r;
        } else {
            if ((r = mix_alloc(h->mx[b], N, h->dc))) return r;
        }
    }
    if ((r = dev_alloc((void **)&h->key, N * sizeof(int)))) return r;
    if ((r = dev_alloc((void **)&h->rank, N * sizeof(int)))) return r;
    if ((r = dev_alloc((void **)&h->perm, N * sizeof(int))))
        return r;
    h->cap = want;
    return MPCD_OK;
}

// Reset of the per-state bookkeeping for n uploaded particles.
static int upload_common(mpcd_handle *h, int n) {
    int r = ensure_capacity(h, n);
    if (r != MPCD_OK) return r;
    h->n = n;
    h->cur = 0;
    h->sorted_for = -1;
    h->sums_for = -1;
    h->sort_age = -1;
    h->stepped = false;
    h->per_pop_for = -1;
    return MPCD_OK;
}

static int grid_for(const mpcd_handle *h, int n) {
    int g = (n + 255) / 256;
    int cap = h->sm_count * 8;
    if (g > cap) g = cap;
    return g < 1 ? 1 : g;
}

// Device staging buffer of at least 'bytes' (grown, never shrunk).
static int xfer_reserve(mpcd_handle *h, size_t bytes) {
    if (bytes <= h->xfer_bytes) return MPCD_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->xfer);
    h->xfer = nullptr;
    h->xfer_bytes = 0;
    if (cudaMalloc(&h->xfer, bytes) != cudaSuccess) return MPCD_ERR_NOMEM;
    h->xfer_bytes = bytes;
    return MPCD_OK;
}

// Staging layout of an upload or download of N particles: Q, V (and U) as
// 3 doubles per particle, the species ids, and 32 bytes of flags and sums.
struct Staging {
    double *Q, *V, *U;
    int *sp;
    int *err;
    unsigned long long *sums;  // GnDNST: occupied cells, particles
};
static int staging(mpcd_handle *h, size_t N, bool withU, bool withSp, Staging *x) {
    const size_t vec = (N * 24 + 255) / 256 * 256, ids = (N * 4 + 255) / 256 * 256;
    int r = xfer_reserve(h, 2 * vec + (withU ? vec : 0) + (withSp ? ids : 0) + 256);
    if (r != MPCD_OK) return r;
    char *p = (char *)h->xfer;
    x->Q = (double *)p;
    x->V = (double *)(p + vec);
    p += 2 * vec;
    x->U = withU ? (double *)p : nullptr;
    if (withU) p += vec;
    x->sp = withSp ? (int *)p : nullptr;
    if (withSp) p += ids;
    x->err = (int *)p;
    x->sums = (unsigned long long *)(p + 16);
    return MPCD_OK;
}

// Staged particles (caller order, 3 doubles per vector) -> the handle's
// state, and the global number density.  Waits for the stream; a rejected
// state (non-finite values, species out of range, a particle the
// initialisation could not place) leaves no state.
static int upload_from_staging(mpcd_handle *h, int n, const Staging &x) {
    const int g = grid_for(h, n);
    if (h->prec == MPCD_PREC_FP64) {
        if (h->dc.dim == 3)
            k_f64_from_aos<3><<<g, 256, 0, h->stream>>>(h->f[0], h->dc, n, x.Q, x.V, x.U, x.sp,
                                                        x.err);
        else
            k_f64_from_aos<2><<<g, 256, 0, h->stream>>>(h->f[0], h->dc, n, x.Q, x.V, x.U, x.sp,
                                                        x.err);
    } else {
        k_mix_from_f64<<<g, 256, 0, h->stream>>>(h->mx[0], h->dc, n, x.Q, x.V, x.U, x.sp, x.err);
    }
    // global number density as globalDensities (init.c:1002-1018) unless
    // given; phantom walls and the nematic activity use it
    const bool density = !(h->cfg.gndnst > 0.0) && (h->dc.any_phantom || h->dc.lc);
    if (density) {
        k_pop_unshifted<<<g, 256, 0, h->stream>>>(h->dc, n, x.Q, h->count);
        k_gndnst_reduce<<<grid_for(h, h->dc.ncells), 256, 0, h->stream>>>(h->dc, h->count,
                                                                         x.sums);
    }
    CK(cudaGetLastError());
    int herr[8];
    CK(cudaMemcpyAsync(herr, x.err, 32, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (herr[0]) {
        h->n = 0;  // a rejected upload leaves no state
        return MPCD_ERR_ARG;
    }
    if (density) {
        unsigned long long occ, sum;
        memcpy(&occ, &herr[4], 8);
        memcpy(&sum, &herr[6], 8);
        h->dc.gndnst = occ > 0 ? (double)sum / (double)occ : 0.0;
    }
    return MPCD_OK;
}

extern "C" int mpcd_upload_state(mpcd_handle *h, int n, const double *Q, const double *V,
                                 const double *U, const int *spid) {
    if (!h || n < 0 || (n > 0 && (!Q || !V))) return MPCD_ERR_ARG;
    int r = upload_common(h, n);
    if (r != MPCD_OK) return r;
    if (n == 0) return MPCD_OK;
    const size_t N = (size_t)n;
    // species ids are checked whenever given (with one species every id
    // must be 0)
    const bool withU = U && h->dc.lc, withSp = spid != nullptr;
    // several species without ids: every particle species 0 (the kernels
    // read a null id array as species 0 only with one species)
    const bool zeroSp = !spid && h->dc.n_species > 1;
    Staging x;
    r = staging(h, N, withU, withSp || zeroSp, &x);
    if (r != MPCD_OK) return r;
    CK(cudaMemcpyAsync(x.Q, Q, N * 24, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(x.V, V, N * 24, cudaMemcpyHostToDevice, h->stream));
    if (withU) CK(cudaMemcpyAsync(x.U, U, N * 24, cudaMemcpyHostToDevice, h->stream));
    if (withSp) CK(cudaMemcpyAsync(x.sp, spid, N * 4, cudaMemcpyHostToDevice, h->stream));
    if (zeroSp) CK(cudaMemsetAsync(x.sp, 0, N * 4, h->stream));
    CK(cudaMemsetAsync(x.err, 0, 256, h->stream));
    return upload_from_staging(h, n, x);
}

// Exact accessible volume for axis-aligned planar walls: each wall the
// species interacts with bounds one axis (W = A (x - Q) - R, negated when
// inverted, is >= 0 on one side of x0 = Q + R/A); the volume is the product
// of the remaining intervals.  A wall whose normal lies outside the first
// DIM axes has the constant W = -R (R when inverted) there.
static double accessible_volume(const DevCfg &dc, const mpcd_config *cfg, int species) {
    double lo[3] = {0.0, 0.0, 0.0}, hi[3];
    for (int d = 0; d < 3; d++) hi[d] = (double)dc.L[d];
    for (int j = 0; j < dc.n_walls; j++) {
        if (!cfg->walls[j].inter[species]) continue;
        const DevWall &w = dc.walls[j];
        const int ax = w.axis;
        if (ax >= dc.dim) {
            const double W = w.inv ? w.R : -w.R;
            if (W < 0.0) return 0.0;
            continue;
        }
        const double A = w.A[ax], x0 = w.Q[ax] + w.R / A;
        const bool above = (A > 0.0) != (w.inv != 0);
        if (above)
            lo[ax] = std::max(lo[ax], x0);
        else
            hi[ax] = std::min(hi[ax], x0);
    }
    double v = 1.0;
    for (int d = 0; d < 3; d++) v *= std::max(0.0, hi[d] - lo[d]);
    return v;
}

extern "C" int mpcd_accessible_volume(const mpcd_config *cfg, int species, double *vol) {
    if (!cfg || !vol) return MPCD_ERR_ARG;
    DevCfg dc;
    int r = build_devcfg(cfg, &dc);
    if (r != MPCD_OK) return r;
    if (species < 0 || species >= cfg->n_species) return MPCD_ERR_ARG;
    *vol = accessible_volume(dc, cfg, species);
    return MPCD_OK;
}

extern "C" int mpcd_init_state(mpcd_handle *h, const mpcd_init_params *p, double *kbtnow) {
    if (!h || !p) return MPCD_ERR_ARG;
    const DevCfg &dc = h->dc;
    InitPlan plan;
    memset(&plan, 0, sizeof(plan));
    long long total = 0;
    const double box = (double)dc.L[0] * dc.L[1] * dc.L[2];
    for (int s = 0; s < MPCD_MAX_SPECIES; s++) {
        const int pop = p->population[s];
        if (pop < 0 || (s >= dc.n_species && pop != 0)) return MPCD_ERR_ARG;
        plan.off[s] = (int)std::min<long long>(total, INT32_MAX);
        total += pop;
        if (s >= dc.n_species) continue;
        const int vd = p->vdist[s], od = p->odist[s];
        if (vd != MPCD_VDIST_RANDVEL && vd != MPCD_VDIST_HOMO && vd != MPCD_VDIST_HOMOAXIS &&
            vd != MPCD_VDIST_GAUSS)
            return MPCD_ERR_UNSUPPORTED;
        if (dc.lc && (od < MPCD_ODIST_RANDORIENT || od > MPCD_ODIST_ALIGNDEFECTPAIR))
            return MPCD_ERR_UNSUPPORTED;
        // the 2D nematic state holds the orientation's x and y only: the
        // codes that give a 2D orientation a z component are refused
        if (dc.lc && dc.dim == 2 &&
            (od == MPCD_ODIST_ALIGNZ || od == MPCD_ODIST_PLANEY || od == MPCD_ODIST_PLANEX))
            return MPCD_ERR_UNSUPPORTED;
        plan.vdist[s] = vd;
        plan.odist[s] = od;
        if (pop > 0) {
            const double frac = accessible_volume(dc, &h->cfg, s) / box;
            if (!(frac > 0.0)) return MPCD_ERR_ARG;
            plan.max_attempts[s] = (int)std::min(std::max(64.0 / frac, 256.0), 4194304.0);
        }
    }
    plan.off[MPCD_MAX_SPECIES] = (int)std::min<long long>(total, INT32_MAX);
    // the species' velocity distributions also serve the bounce-limit
    // re-thermalisation from now on (VDIST, bc.c:1482)
    for (int s = 0; s < dc.n_species; s++) h->dc.vdist[s] = p->vdist[s];
    if (total > INT32_MAX) return MPCD_ERR_SIZE;
    const int n = (int)total;
    plan.rframe = p->rframe && n > 2;  // init.c:2140-2143
    int r = upload_common(h, n);
    if (r != MPCD_OK) return r;
    if (n == 0) {
        if (kbtnow) *kbtnow = 0.0;
        return MPCD_OK;
    }
    Staging x;
    r = staging(h, (size_t)n, dc.lc != 0, dc.n_species > 1, &x);
    if (r != MPCD_OK) {
        h->n = 0;
        return r;
    }
    const int g = grid_for(h, n);
    double *work = nullptr;  // block partials (8 per block), then 3 x 8 sums
    if (cudaMalloc((void **)&work, sizeof(double) * (8 * (size_t)g + 24)) != cudaSuccess) {
        h->n = 0;
        return MPCD_ERR_NOMEM;
    }
    double *part = work, *sums = work + 8 * (size_t)g;
    cudaError_t e = cudaMemsetAsync(x.err, 0, 256, h->stream);
    k_init_gen<<<g, 256, 0, h->stream>>>(dc, plan, n, x.Q, x.V, x.U, x.sp, x.err, part);
    k_init_reduce<<<1, 256, 0, h->stream>>>(part, g, 7, sums);
    k_init_adjust<<<g, 256, 0, h->stream>>>(dc, plan, n, x.V, sums, nullptr, part);
    k_init_reduce<<<1, 256, 0, h->stream>>>(part, g, 1, sums + 8);
    k_init_adjust<<<g, 256, 0, h->stream>>>(dc, plan, n, x.V, sums, sums + 8, part);
    k_init_reduce<<<1, 256, 0, h->stream>>>(part, g, 1, sums + 16);
    double t_after = 0.0;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&t_after, sums + 16, sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) r = upload_from_staging(h, n, x);
    cudaStreamSynchronize(h->stream);
    cudaFree(work);
    if (e != cudaSuccess || r != MPCD_OK) {
        h->n = 0;
        return e != cudaSuccess ? MPCD_ERR_CUDA : r;
    }
    if (kbtnow) *kbtnow = t_after / ((double)n * dc.dim);
    return MPCD_OK;
}

extern "C" int mpcd_upload_particles_strided(mpcd_handle *h, int n, const void *base,
                                             size_t stride, size_t off_Q, size_t off_V,
                                             size_t off_U, size_t off_spid) {
    if (!h || n < 0 || (n > 0 && !base) || stride == 0) return MPCD_ERR_ARG;
    const bool has_U = off_U != (size_t)-1, has_sp = off_spid != (size_t)-1;
    std::vector<double> Q((size_t)3 * n), V((size_t)3 * n), U(has_U ? (size_t)3 * n : 0);
    std::vector<int> sp((size_t)n);
    const char *b = (const char *)base;
    for (int i = 0; i < n; i++) {
        const char *rec = b + (size_t)i * stride;
        memcpy(&Q[3 * (size_t)i], rec + off_Q, 3 * sizeof(double));
        memcpy(&V[3 * (size_t)i], rec + off_V, 3 * sizeof(double));
        if (has_U) memcpy(&U[3 * (size_t)i], rec + off_U, 3 * sizeof(double));
        if (has_sp)
            memcpy(&sp[i], rec + off_spid, sizeof(int));
        else
            sp[i] = 0;
    }
    return mpcd_upload_state(h, n, Q.data(), V.data(), has_U ? U.data() : nullptr, sp.data());
}

// The state in the caller's original particle order; any output may be
// null (then not gathered).
static int download_impl(mpcd_handle *h, double *Q, double *V, double *U, int *spid) {
    if (!h) return MPCD_ERR_ARG;
    const int n = h->n;
    const size_t N = (size_t)n;
    if (n == 0) return MPCD_OK;
    Staging x;
    int r = staging(h, N, U != nullptr, spid != nullptr, &x);
    if (r != MPCD_OK) return r;
    CK(cudaMemsetAsync(x.err, 0, sizeof(int), h->stream));
    const int g = grid_for(h, n);
    // the inverse of the state's order (into the sort's scratch), then a
    // gather in the caller's order: coalesced stores to the caller's arrays
    int *inv = h->perm;
    CK(cudaMemsetAsync(inv, 0xFF, N * sizeof(int), h->stream));  // -1: no slot yet
    if (h->prec == MPCD_PREC_FP64)
        k_inv_pid_f64<<<g, 256, 0, h->stream>>>(h->f[h->cur].pid, n, inv, x.err);
    else
        k_inv_pid_mix<<<g, 256, 0, h->stream>>>(h->mx[h->cur].W, n, inv, x.err);
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, x.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (herr) return MPCD_ERR_STATE;  // not a permutation: nothing to gather
    if (h->prec == MPCD_PREC_FP64) {
        if (h->dc.dim == 3)
            k_f64_gather_aos<3><<<g, 256, 0, h->stream>>>(h->f[h->cur], n, inv, x.Q, x.V, x.U,
                                                          x.sp, x.err);
        else
            k_f64_gather_aos<2><<<g, 256, 0, h->stream>>>(h->f[h->cur], n, inv, x.Q, x.V, x.U,
                                                          x.sp, x.err);
    } else {
        k_mix_gather_aos<<<g, 256, 0, h->stream>>>(h->mx[h->cur], h->dc, n, inv, x.Q, x.V, x.U,
                                                   x.sp, x.err);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&herr, x.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (Q) CK(cudaMemcpyAsync(Q, x.Q, N * 24, cudaMemcpyDeviceToHost, h->stream));
    if (V) CK(cudaMemcpyAsync(V, x.V, N * 24, cudaMemcpyDeviceToHost, h->stream));
    if (U) CK(cudaMemcpyAsync(U, x.U, N * 24, cudaMemcpyDeviceToHost, h->stream));
    if (spid) CK(cudaMemcpyAsync(spid, x.sp, N * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return herr ? MPCD_ERR_STATE : MPCD_OK;
}

extern "C" int mpcd_download_state(mpcd_handle *h, double *Q, double *V, double *U) {
    return download_impl(h, Q, V, U, nullptr);
}

extern "C" int mpcd_download_species(mpcd_handle *h, int *spid) {
    if (!h || (h->n > 0 && !spid)) return MPCD_ERR_ARG;
    return download_impl(h, nullptr, nullptr, nullptr, spid);
}

extern "C" int mpcd_set_species_vdist(mpcd_handle *h, const int *vdist) {
    if (!h || !vdist) return MPCD_ERR_ARG;
    for (int s = 0; s < h->dc.n_species; s++)
        if (vdist[s] != MPCD_VDIST_RANDVEL && vdist[s] != MPCD_VDIST_HOMO &&
            vdist[s] != MPCD_VDIST_HOMOAXIS && vdist[s] != MPCD_VDIST_GAUSS)
            return MPCD_ERR_UNSUPPORTED;
    for (int s = 0; s < h->dc.n_species; s++) h->dc.vdist[s] = vdist[s];
    return MPCD_OK;
}

extern "C" int mpcd_get_config(const mpcd_handle *h, mpcd_config *cfg) {
    if (!h || !cfg) return MPCD_ERR_ARG;
    *cfg = h->cfg;
    cfg->gndnst = h->dc.gndnst;
    return MPCD_OK;
}

extern "C" int mpcd_particle_count(const mpcd_handle *h, int *n) {
    if (!h || !n) return MPCD_ERR_ARG;
    *n = h->n;
    return MPCD_OK;
}

extern "C" int mpcd_download_particles_strided(mpcd_handle *h, void *base, size_t stride,
                                               size_t off_Q, size_t off_V, size_t off_U) {
    if (!h || (h->n > 0 && !base) || stride == 0) return MPCD_ERR_ARG;
    int n = h->n;
    // orientations only where the state carries them (nematic order): an
    // isotropic fluid's records keep whatever U the caller holds
    const bool has_U = off_U != (size_t)-1 && h->dc.lc;
    std::vector<double> Q((size_t)3 * n), V((size_t)3 * n), U(has_U ? (size_t)3 * n : 0);
    int r = mpcd_download_state(h, Q.data(), V.data(), has_U ? U.data() : nullptr);
    if (r != MPCD_OK) return r;
    char *b = (char *)base;
    for (int i = 0; i < n; i++) {
        char *rec = b + (size_t)i * stride;
        memcpy(rec + off_Q, &Q[3 * (size_t)i], 3 * sizeof(double));
        memcpy(rec + off_V, &V[3 * (size_t)i], 3 * sizeof(double));
        if (has_U) memcpy(rec + off_U, &U[3 * (size_t)i], 3 * sizeof(double));
    }
    return MPCD_OK;
}


// Tile geometry: cells per tile so that a tile holds about 'target'
// particles on average; staging capacity 1.5x that plus a margin.
static void tile_geometry(const mpcd_handle *h, int target, int *ct, int *cap) {
    double vol = 1.0;
    for (int d = 0; d < h->dc.dim; d++) vol *= h->dc.L[d];
    double ppc = h->n > 0 ? (double)h->n / vol : 10.0;
    if (ppc < 1.0) ppc = 1.0;
    int c = 1;
    while (c * 2 <= 256 && (double)(c * 2) * ppc <= (double)target) c *= 2;
    *ct = c;
    *cap = (int)(1.5 * (double)c * ppc) + 128;
}

// Staging capacity of a warp's 32-cell group: mean + ~4 sigma + margin.
static int group_capacity(const mpcd_handle *h) {
    double vol = 1.0;
    for (int d = 0; d < h->dc.dim; d++) vol *= h->dc.L[d];
    double mean = 32.0 * (h->n > 0 ? (double)h->n / vol : 10.0);
    int capw = (int)(mean + 4.0 * std::sqrt(mean) + 32.0);
    capw = (capw + 31) / 32 * 32;
    return capw < 64 ? 64 : (capw > 2048 ? 2048 : capw);
}

template <int DIM, class T>
static int launch_group(mpcd_handle *h, int mode, const typename T::State &a,
                        const typename T::State &b, const TileBufs &tb, const StepArgs &sa) {
    int capw = group_capacity(h);
    // clamp the staging capacity to what a block may hold (larger groups
    // report overflow)
    while (capw > 32 &&
           GroupLayout<T>::kWarps * GroupLayout<T>::per_warp_bytes(capw) > h->smem_optin - 1024)
        capw -= 32;
    int bytes = GroupLayout<T>::kWarps * GroupLayout<T>::per_warp_bytes(capw);
    int groups = (h->dc.ncells + 31) / 32;
    int grid = (groups + GroupLayout<T>::kWarps - 1) / GroupLayout<T>::kWarps;
    const DevCfg &c = h->dc;
    cudaError_t e = cudaSuccess;
#define MPCD_LAUNCH_GROUP(MODEV)                                                         \
    do {                                                                                 \
        auto kfn = k_group<DIM, T, MODEV>;                                               \
        e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); \
        if (e == cudaSuccess)                                                            \
            e = cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, \
                                     100);                                               \
        if (e == cudaSuccess)                                                            \
            kfn<<<grid, 32 * GroupLayout<T>::kWarps, bytes, h->stream>>>(c, a, b, tb, sa, capw); \
    } while (0)
    if (mode == MODE_INPLACE)
        MPCD_LAUNCH_GROUP(MODE_INPLACE);
    else if (mode == MODE_COUNT)
        MPCD_LAUNCH_GROUP(MODE_COUNT);
    else
        MPCD_LAUNCH_GROUP(MODE_FINAL);
#undef MPCD_LAUNCH_GROUP
    if (e != cudaSuccess) return MPCD_ERR_CUDA;
    return MPCD_OK;
}

// The persistent family's plan for the current state: blocks of the
// cooperative launch (one per SM at most), or -1 if the box does not fit in
// their shared memory (FP64 form, isotropic fluids only).  `wanted` is set
// when the box is small enough for the family to be the default: at most
// two particles per thread.
static int per_plan(mpcd_handle *h, bool *wanted = nullptr) {
    if (wanted) *wanted = false;
    if (h->per_planned_n != h->n || h->per_blocks == 0) {
        h->per_planned_n = h->n;
        h->per_blocks = -1;
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
        if (h->prec == MPCD_PREC_FP64 && !h->dc.lc && h->n > 0 && coop) {
            bool fits = true;
            for (int d = 0; d < 3; d++) fits = fits && h->dc.N1[d] <= 1024;
            const int blocks =
                std::max(1, std::min(h->sm_count, (h->n + kPerThreads - 1) / kPerThreads));
            const PerLayout l = h->dc.dim == 3
                                    ? per_layout<3>(h->n, h->dc.op, h->dc.n_species, blocks)
                                    : per_layout<2>(h->n, h->dc.op, h->dc.n_species, blocks);
            auto kfn = h->dc.dim == 3 ? k_persist<3> : k_persist<2>;
            int per_sm = 0;
            if (fits && l.bytes <= h->smem_optin &&
                cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, l.bytes) ==
                    cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kPerThreads,
                                                              l.bytes) == cudaSuccess &&
                per_sm >= 1)
                h->per_blocks = blocks;
            cudaGetLastError();
        }
    }
    if (wanted && h->per_blocks > 0)
        *wanted = (h->n + h->per_blocks - 1) / h->per_blocks <= 2 * kPerThreads;
    return h->per_blocks;
}

static int kernel_family(mpcd_handle *h) {
    // the nematic and Chate (the cells' director) run on the tile kernel only
    if (h->dc.lc || h->dc.op == MPCD_COLL_CHATE || h->dc.op == MPCD_COLL_CHATE_MPCAT)
        return MPCD_KERNEL_TILE;
    if (h->kernel == MPCD_KERNEL_PERSIST) return MPCD_KERNEL_PERSIST;
    bool wanted = false;
    if (h->kernel == MPCD_KERNEL_AUTO && h->prec == MPCD_PREC_FP64 && per_plan(h, &wanted) > 0 &&
        wanted)
        return MPCD_KERNEL_PERSIST;
    bool srd_plain = h->dc.op == MPCD_COLL_ARBAXIS && !h->dc.any_phantom;
    if (!srd_plain) return MPCD_KERNEL_TILE;
    if (h->kernel == MPCD_KERNEL_AUTO) return MPCD_KERNEL_RESIDENT;
    return h->kernel;
}

// nsteps steps of the persistent family: one cooperative launch that keeps
// the whole box in its blocks' shared memory.
template <int DIM>
static int run_steps_per(mpcd_handle *h, int nsteps, uint32_t step0) {
    const int blocks = per_plan(h);
    if (blocks <= 0) return MPCD_ERR_UNSUPPORTED;
    const PerLayout l = per_layout<DIM>(h->n, h->dc.op, h->dc.n_species, blocks);
    const size_t nc = (size_t)h->dc.ncells;
    // sums (the largest operator's rows), populations, records, record
    // populations and the barrier counter
    const size_t bytes = nc * (kPerRowsMax * 8 + 4 + kPerRecMax * 8 + 4) + 64;
    if (!h->per_work) {
        CK(cudaMalloc(&h->per_work, bytes));
        CK(cudaMemsetAsync(h->per_work, 0, bytes, h->stream));
    }
    if (!h->per_pop) CK(cudaMalloc((void **)&h->per_pop, sizeof(int) * nc));
    PerGlobal g;
    g.sum = (double *)h->per_work;
    g.rec = g.sum + kPerRowsMax * nc;
    g.pop = (int *)(g.rec + kPerRecMax * nc);
    g.rpop = g.pop + nc;
    g.bar = (unsigned long long *)(((uintptr_t)(g.rpop + nc) + 15) & ~(uintptr_t)15);
    g.ncells = (int)nc;
    CK(cudaMemsetAsync(h->per_pop, 0, sizeof(int) * nc, h->stream));
    CK(cudaMemsetAsync(g.bar, 0, sizeof(unsigned long long), h->stream));
    // a launch that continues the previous one finds its first binning
    // counted already
    const int count_first = h->per_pop_for == (int64_t)step0 ? 0 : 1;
    Fp64State st = h->f[h->cur];
    int n = h->n, ring = kAccRing;
    double *acc = h->acc;
    int *pop = h->per_pop;
    unsigned long long *status = h->status;
    DevCfg dc = h->dc;
    void *args[] = {&dc, &st, &n, (void *)&l, &g, &step0, &nsteps, &acc, &ring, &pop, &status,
                    (void *)&count_first};
    time_begin(h);
    CK(cudaLaunchCooperativeKernel((void *)k_persist<DIM>, dim3((unsigned)blocks),
                                   dim3((unsigned)kPerThreads), args, (size_t)l.bytes, h->stream));
    time_end(h);
    h->sorted_for = -1;
    h->sums_for = -1;
    h->per_pop_for = (int64_t)step0 + nsteps;
    h->launches = 1;
    return MPCD_OK;
}

template <int DIM, class T>
static int launch_srd_cells(mpcd_handle *h, const typename T::State &a, const int *start,
                            const StepArgs &sa, double *acc) {
    int grid = (h->dc.ncells + 255) / 256;
    k_srd_cells<DIM, T><<<grid, 256, 0, h->stream>>>(
        h->dc, a, start, (typename SrdCell<T>::Rec *)h->crec, sa, acc);
    return cudaGetLastError() == cudaSuccess ? MPCD_OK : MPCD_ERR_CUDA;
}

template <int DIM, class T>
static int launch_srd_parts(mpcd_handle *h, int mode, const typename T::State &a,
                            const typename T::State &b, const TileBufs &tb,
                            const StepArgs &sa) {
    int grid = (h->n + 255) / 256;
    const typename SrdCell<T>::Rec *cr = (const typename SrdCell<T>::Rec *)h->crec;
    if (mode == MODE_INPLACE)
        k_srd_parts<DIM, T, MODE_INPLACE><<<grid, 256, 0, h->stream>>>(h->dc, a, b, h->n, cr, tb, sa);
    else if (mode == MODE_COUNT)
        k_srd_parts<DIM, T, MODE_COUNT><<<grid, 256, 0, h->stream>>>(h->dc, a, b, h->n, cr, tb, sa);
    else
        k_srd_parts<DIM, T, MODE_FINAL><<<grid, 256, 0, h->stream>>>(h->dc, a, b, h->n, cr, tb, sa);
    return cudaGetLastError() == cudaSuccess ? MPCD_OK : MPCD_ERR_CUDA;
}

template <int DIM, class T>
static int launch_tile(mpcd_handle *h, int mode, const typename T::State &a,
                       const typename T::State &b, const TileBufs &tb, const StepArgs &sa) {
    int fam = kernel_family(h);
    if (fam == MPCD_KERNEL_SPLIT) return launch_srd_parts<DIM, T>(h, mode, a, b, tb, sa);
    if (fam == MPCD_KERNEL_GROUP) return launch_group<DIM, T>(h, mode, a, b, tb, sa);
    int ct, capp;
    tile_geometry(h, h->tile_target, &ct, &capp);
    TileLayout lay = tile_layout<T>(ct, capp, h->dc.op, h->dc.n_species);
    while (lay.bytes > 200 * 1024 && capp > 256) {
        capp = capp * 3 / 4;
        lay = tile_layout<T>(ct, capp, h->dc.op, h->dc.n_species);
    }
    int grid = (h->dc.ncells + ct - 1) / ct;
    const DevCfg &c = h->dc;
    cudaError_t e = cudaSuccess;
#define MPCD_LAUNCH_TILE(MODEV)                                                          \
    do {                                                                                 \
        auto kfn = k_tile<DIM, T, MODEV>;                                                \
        e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 lay.bytes);                                             \
        if (e == cudaSuccess)                                                            \
            e = cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, \
                                     100);                                               \
        if (e == cudaSuccess) kfn<<<grid, 256, lay.bytes, h->stream>>>(c, a, b, tb, sa, lay); \
    } while (0)
    if (mode == MODE_INPLACE)
        MPCD_LAUNCH_TILE(MODE_INPLACE);
    else if (mode == MODE_COUNT)
        MPCD_LAUNCH_TILE(MODE_COUNT);
    else
        MPCD_LAUNCH_TILE(MODE_FINAL);
#undef MPCD_LAUNCH_TILE
    if (e != cudaSuccess) return MPCD_ERR_CUDA;
    return MPCD_OK;
}

// Exclusive scan of the first nkeys counts (default: one per cell).
static void launch_scan(mpcd_handle *h, int *start, int *fill, double *acc_zero,
                        int nkeys = -1) {
    if (nkeys < 0) nkeys = h->dc.ncells;
    const int tiles = (nkeys + kScanTile - 1) / kScanTile;
    k_scan_partial<<<tiles, 256, 0, h->stream>>>(h->count, nkeys, h->part);
    k_scan_apply<<<tiles, 256, 0, h->stream>>>(h->count, nkeys, h->part, start, fill, acc_zero);
}

template <int DIM, class T>
static void launch_key(mpcd_handle *h, const typename T::State &a, const StepArgs &sa);
template <>
void launch_key<3, MixT<3>>(mpcd_handle *h, const MixState &a, const StepArgs &sa) {
    k_key_mix<3><<<grid_for(h, h->n), 256, 0, h->stream>>>(h->dc, a, h->n, h->key, h->rank,
                                                           h->count, sa, h->status);
}
template <>
void launch_key<2, MixT<2>>(mpcd_handle *h, const MixState &a, const StepArgs &sa) {
    k_key_mix<2><<<grid_for(h, h->n), 256, 0, h->stream>>>(h->dc, a, h->n, h->key, h->rank,
                                                           h->count, sa, h->status);
}
template <>
void launch_key<3, F64T<3>>(mpcd_handle *h, const Fp64State &a, const StepArgs &sa) {
    k_key_f64<3><<<grid_for(h, h->n), 256, 0, h->stream>>>(h->dc, a, h->n, h->key, h->rank,
                                                           h->count, sa, h->status);
}
template <>
void launch_key<2, F64T<2>>(mpcd_handle *h, const Fp64State &a, const StepArgs &sa) {
    k_key_f64<2><<<grid_for(h, h->n), 256, 0, h->stream>>>(h->dc, a, h->n, h->key, h->rank,
                                                           h->count, sa, h->status);
}

// Reorder the state into counting-sort order; returns the launch count.
static int launch_scatter(mpcd_handle *h, const MixState &a, const MixState &b,
                          const int *start) {
    k_perm<<<grid_for(h, h->n), 256, 0, h->stream>>>(h->n, h->key, h->rank, start, h->perm);
    k_gather_mix<<<grid_for(h, h->n), 256, 0, h->stream>>>(a, b, h->n, h->perm);
    return 2;
}
// The FP64 state's reorder is a gather too: each 8-byte element scattered
// to its sorted place would write a part of a 32-byte sector.
static int launch_scatter(mpcd_handle *h, const Fp64State &a, const Fp64State &b,
                          const int *start) {
    k_perm<<<grid_for(h, h->n), 256, 0, h->stream>>>(h->n, h->key, h->rank, start, h->perm);
    if (h->dc.dim == 3)
        k_gather_f64<3><<<grid_for(h, h->n), 256, 0, h->stream>>>(a, b, h->n, h->perm);
    else
        k_gather_f64<2><<<grid_for(h, h->n), 256, 0, h->stream>>>(a, b, h->n, h->perm);
    return 2;
}

static void host_shift(const mpcd_handle *h, uint32_t step, double s[3]) {
    s[0] = s[1] = s[2] = 0.0;
    if (h->dc.galinv) mpcd_rng_shift(h->dc.seed, h->dc.replica, step, h->dc.dim, s);
}

// One solvent timestep.  Particles enter sorted by cell of this step's
// shifted grid (established here if they are not) and leave sorted for the
// next step's.
template <int DIM, class T>
static int run_step(mpcd_handle *h, typename T::State *st, uint32_t step) {
    StepArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.step = step;
    host_shift(h, step, sa.s);
    host_shift(h, step + 1u, sa.sn);
    for (int d = 0; d < 3; d++) {  // s = k * 2^-32 exactly
        // the mixed form's position words carry 22 fraction bits
        sa.ks[d] = (uint32_t)(sa.s[d] * 4294967296.0) & kShiftMask;
        sa.ksn[d] = (uint32_t)(sa.sn[d] * 4294967296.0) & kShiftMask;
    }
    double *acc_cur = acc_at(h, step);
    double *acc_nxt = acc_at(h, step + 1u);
    int launches = 0;
    if (h->sorted_for != (int64_t)step) {
        launch_key<DIM, T>(h, st[h->cur], sa);
        launch_scan(h, h->start[h->scur], nullptr, acc_cur);
        launches += 3 + launch_scatter(h, st[h->cur], st[1 - h->cur], h->start[h->scur]);
        h->cur = 1 - h->cur;
    }
    TileBufs tb;
    memset(&tb, 0, sizeof(tb));
    tb.start = h->start[h->scur];
    tb.start_next = h->start[1 - h->scur];
    tb.count_next = h->count;
    tb.fill = h->fill;
    tb.key = h->key;
    tb.rank = h->rank;
    tb.acc = acc_cur;
    tb.status = h->status;
    int r;
    if (kernel_family(h) == MPCD_KERNEL_SPLIT) {
        r = launch_srd_cells<DIM, T>(h, st[h->cur], tb.start, sa, acc_cur);
        if (r != MPCD_OK) return r;
        launches += 1;
    }
    if (h->strategy == MPCD_STRATEGY_SCATTER) {
        time_begin(h);
        r = launch_tile<DIM, T>(h, MODE_INPLACE, st[h->cur], st[1 - h->cur], tb, sa);
        time_end(h);
        if (r != MPCD_OK) return r;
        launch_scan(h, h->start[1 - h->scur], nullptr, acc_nxt);
        launches += launch_scatter(h, st[h->cur], st[1 - h->cur], h->start[1 - h->scur]) - 1;
    } else {
        r = launch_tile<DIM, T>(h, MODE_COUNT, st[h->cur], st[1 - h->cur], tb, sa);
        if (r != MPCD_OK) return r;
        launch_scan(h, h->start[1 - h->scur], h->fill, acc_nxt);
        time_begin(h);
        r = launch_tile<DIM, T>(h, MODE_FINAL, st[h->cur], st[1 - h->cur], tb, sa);
        time_end(h);
        if (r != MPCD_OK) return r;
    }
    launches += 4;
    CK(cudaGetLastError());
    h->cur = 1 - h->cur;
    h->scur = 1 - h->scur;
    h->sorted_for = (int64_t)step + 1;
    h->sums_for = -1;
    h->launches = launches;
    return MPCD_OK;
}

// One SRD timestep with the particles resident in place (mixed precision):
// an occasional re-sort for locality, the cell pass and the particle pass.
// The cell and particle passes are launched as programmatic dependents
// (launch_pdl): each may start while the kernel before it finishes, doing the
// work that reads nothing that kernel writes (the cell pass's axis draws, the
// particle pass's table set-up) before it waits for it.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem,
                              cudaStream_t stream, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int DIM>
static int run_step_res(mpcd_handle *h, uint32_t step) {
    StepArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.step = step;
    host_shift(h, step, sa.s);
    host_shift(h, step + 1u, sa.sn);
    for (int d = 0; d < 3; d++) {
        // the mixed form's position words carry 22 fraction bits
        sa.ks[d] = (uint32_t)(sa.s[d] * 4294967296.0) & kShiftMask;
        sa.ksn[d] = (uint32_t)(sa.sn[d] * 4294967296.0) & kShiftMask;
    }
    const DevCfg &c = h->dc;
    const size_t nc = (size_t)c.ncells;
    double *acc_cur = acc_at(h, step);
    double *acc_nxt = acc_at(h, step + 1u);
    const ResPlanes sum_cur{(long long *)(h->rsum + (step & 1u) * nc), (int)nc};
    const ResPlanes sum_nxt{(long long *)(h->rsum + ((step + 1u) & 1u) * nc), (int)nc};
    unsigned long long *ms_cur = h->rmsum ? h->rmsum + (step & 1u) * nc : nullptr;
    unsigned long long *ms_nxt = h->rmsum ? h->rmsum + ((step + 1u) & 1u) * nc : nullptr;
    int launches = 0;
    if (h->sorted_for == (int64_t)step) {
        h->sort_age = 0;
    } else if (h->sort_age < 0 || h->sort_age >= h->sort_interval) {
        if (DIM == 3) {
            k_key_res3<<<grid_for(h, h->n), 256, 0, h->stream>>>(
                h->dc, h->mx[h->cur], h->n, h->key, h->rank, h->count, sa, h->status);
            launch_scan(h, h->start[h->scur], nullptr, nullptr, res_brick_keys(h->dc.N1));
        } else {
            launch_key<DIM, MixT<DIM>>(h, h->mx[h->cur], sa);
            launch_scan(h, h->start[h->scur], nullptr, nullptr);
        }
        launches += 3 + launch_scatter(h, h->mx[h->cur], h->mx[1 - h->cur], h->start[h->scur]);
        h->cur = 1 - h->cur;
        h->sort_age = 0;
    }
    const int pgrid = (int)((h->n + kResChunk - 1) / kResChunk);
    const int pbytes = res_table_bytes(h->rmsum ? DIM + 1 : DIM);
    typedef ResRec CRec;
    if (!h->res_attr) {
        // once per handle (the driver keeps them for the device): the
        // largest table any handle may use (several species) and the
        // carve-out, for each variant of the particle pass
        for (auto k : {k_res_parts<DIM, RES_SUM, false>, k_res_parts<DIM, RES_STEP, true>,
                       k_res_parts<DIM, RES_STEP, false>}) {
            CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    res_table_bytes(DIM + 1)));
            CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        }
        h->res_attr = true;
    }
    if (h->sums_for != (int64_t)step) {
        CK(cudaMemsetAsync(h->rsum, 0, sizeof(ResSum) * 2 * nc, h->stream));
        if (h->rmsum)
            CK(cudaMemsetAsync(h->rmsum, 0, sizeof(unsigned long long) * 2 * nc, h->stream));
        CK(cudaMemsetAsync(acc_cur, 0, sizeof(double) * ACC_WORDS, h->stream));
        auto ksum = k_res_parts<DIM, RES_SUM, false>;
        ksum<<<pgrid, kResThreads, pbytes, h->stream>>>(c, h->mx[h->cur], h->n,
                                                        (const CRec *)h->crec, sum_cur, ms_cur,
                                                        acc_cur, h->status, sa);
        launches += 1;
    }
    CK(launch_pdl(k_res_cells<DIM>, (int)((nc + 256 * kResCellsPer - 1) / (256 * kResCellsPer)),
                  256, 0, h->stream, c, sum_cur, ms_cur, (CRec *)h->crec, sa, acc_cur, acc_nxt));
    const bool lean = c.all_periodic && !h->rmsum && !c.grav_flag;
    auto kstep = lean ? k_res_parts<DIM, RES_STEP, true> : k_res_parts<DIM, RES_STEP, false>;
    time_begin(h);
    CK(launch_pdl(kstep, pgrid, kResThreads, pbytes, h->stream, c, h->mx[h->cur], h->n,
                  (const CRec *)h->crec, sum_nxt, ms_nxt, acc_cur, h->status, sa));
    time_end(h);
    launches += 2;
    CK(cudaGetLastError());
    h->sums_for = (int64_t)step + 1;
    h->sorted_for = -1;
    h->sort_age++;
    h->launches = launches;
    return MPCD_OK;
}

// One step of the FP64 resident family (mpcd_resident64.cuh): an occasional
// re-sort for locality (the FP64 counting sort), the cell pass and the
// particle pass, both launched as programmatic dependents.
template <int DIM>
static int run_step_r64(mpcd_handle *h, uint32_t step) {
    StepArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.step = step;
    host_shift(h, step, sa.s);
    host_shift(h, step + 1u, sa.sn);
    const DevCfg &c = h->dc;
    const size_t nc = (size_t)c.ncells;
    double *acc_cur = acc_at(h, step);
    double *acc_nxt = acc_at(h, step + 1u);
    auto sums_of = [&](uint32_t parity) {
        R64Sums r;
        double *b = h->r64sum + (size_t)(parity & 1u) * 4 * nc;
        r.M = b;
        for (int d = 0; d < 3; d++) r.p[d] = b + (size_t)(d + 1) * nc;
        r.pop = h->r64pop + (size_t)(parity & 1u) * nc;
        return r;
    };
    const R64Sums sum_cur = sums_of(step), sum_nxt = sums_of(step + 1u);
    using Rec = R64Rec;
    int launches = 0;
    if (h->sorted_for == (int64_t)step) {
        h->sort_age = 0;
    } else if (h->sort_age < 0 || h->sort_age >= h->sort_interval) {
        launch_key<DIM, F64T<DIM>>(h, h->f[h->cur], sa);
        launch_scan(h, h->start[h->scur], nullptr, nullptr);
        launches += 3 + launch_scatter(h, h->f[h->cur], h->f[1 - h->cur], h->start[h->scur]);
        h->cur = 1 - h->cur;
        h->sort_age = 0;
    }
    // one wave: the blocks of the particle pass that fit on the handle's
    // device at once (the kernel strides over the particles); the grid also
    // fixes the order of the FP64 KE sums, so KE rounding depends on it
    // a box periodic on every axis runs the particle pass without the
    // re-placement of particles that leave the grid (they cannot)
    const bool open = !c.all_periodic;
    auto kstep = open ? k_r64_parts<DIM, RES_STEP, true> : k_r64_parts<DIM, RES_STEP, false>;
    if (h->r64_per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kstep, 256, 0) != cudaSuccess ||
            b < 1)
            b = 1;
        h->r64_per_sm = b;
    }
    const long long pwant = ((long long)h->n + 255) / 256,
                    pcap = (long long)h->sm_count * h->r64_per_sm;
    const int pgrid = (int)(pwant < pcap ? pwant : pcap);
    if (h->sums_for != (int64_t)step) {
        CK(cudaMemsetAsync(h->r64sum, 0, sizeof(double) * 8 * nc, h->stream));
        CK(cudaMemsetAsync(h->r64pop, 0, sizeof(int) * 2 * nc, h->stream));
        CK(cudaMemsetAsync(acc_cur, 0, sizeof(double) * ACC_WORDS, h->stream));
        k_r64_parts<DIM, RES_SUM, false><<<pgrid, 256, 0, h->stream>>>(
            c, h->f[h->cur], h->n, (const Rec *)h->crec, sum_cur, acc_cur, h->status, sa);
        launches += 1;
    }
    CK(launch_pdl(k_r64_cells<DIM>, (int)((nc + 255) / 256), 256, 0, h->stream, c, sum_cur,
                  (Rec *)h->crec, sa, acc_cur, acc_nxt));
    time_begin(h);
    CK(launch_pdl(kstep, pgrid, 256, 0, h->stream, c, h->f[h->cur], h->n,
                  (const Rec *)h->crec, sum_nxt, acc_cur, h->status, sa));
    time_end(h);
    launches += 2;
    CK(cudaGetLastError());
    h->sums_for = (int64_t)step + 1;
    h->sorted_for = -1;
    h->sort_age++;
    h->launches = launches;
    return MPCD_OK;
}

static int default_strategy(const mpcd_handle *h) {
    // recompute (96 B/particle) wins when the collision is cheap to redo
    return is_vcm_op(h->dc.op) ? MPCD_STRATEGY_RECOMPUTE : MPCD_STRATEGY_SCATTER;
}

// One nematic (2D) timestep: moments + order parameter, velocity gradient,
// the tile kernel (orientation update, collision, streaming), re-sort.
template <class T>
static int run_step_lc(mpcd_handle *h, typename T::State *st, uint32_t step) {
    StepArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.step = step;
    host_shift(h, step, sa.s);
    host_shift(h, step + 1u, sa.sn);
    for (int d = 0; d < 3; d++) {
        // the mixed form's position words carry 22 fraction bits
        sa.ks[d] = (uint32_t)(sa.s[d] * 4294967296.0) & kShiftMask;
        sa.ksn[d] = (uint32_t)(sa.sn[d] * 4294967296.0) & kShiftMask;
    }
    double *acc_cur = acc_at(h, step);
    double *acc_nxt = acc_at(h, step + 1u);
    int launches = 0;
    if (h->sorted_for != (int64_t)step) {
        launch_key<2, T>(h, st[h->cur], sa);
        launch_scan(h, h->start[h->scur], nullptr, acc_cur);
        launches += 3 + launch_scatter(h, st[h->cur], st[1 - h->cur], h->start[h->scur]);
        h->cur = 1 - h->cur;
    }
    const DevCfg &c = h->dc;
    const int *start = h->start[h->scur];
    k_lc_moments<T><<<(c.ncells + 255) / 256, 256, 0, h->stream>>>(c, st[h->cur], start,
                                                                   h->lcc, sa, acc_cur);
    int nb = (c.L[0] - 1) * (c.L[1] - 1);
    if (nb > 0) k_lc_grad<<<(nb + 255) / 256, 256, 0, h->stream>>>(c, h->lcc);
    k_lc_edges<<<(c.L[1] + 255) / 256, 256, 0, h->stream>>>(c, h->lcc, 0);
    k_lc_edges<<<(c.L[0] + 255) / 256, 256, 0, h->stream>>>(c, h->lcc, 1);
    // tile: about 512 particles by default (mpcd_step); with three blocks
    // per SM (80 registers) this measured 0.639 ms per 256^2 mixed step,
    // against 0.654 ms for 1024 particles at two blocks per SM (118
    // registers), whose per-particle phases left the block's warps waiting
    // at its barriers
    int ct, capp;
    tile_geometry(h, h->tile_target > 0 ? h->tile_target : 512, &ct, &capp);
    LcTileLayout lay;
    lay.ct = ct;
    lay.cap = capp;
    lay.bytes = (int)((size_t)capp * sizeof(LcPart) + (size_t)((ct + 1) * 4 + 15) / 16 * 16 +
                      (size_t)ct * 9 * sizeof(double) + (size_t)capp + 16);
    while (lay.bytes > 200 * 1024 && lay.cap > 256) {
        lay.cap = lay.cap * 3 / 4;
        lay.bytes = (int)((size_t)lay.cap * sizeof(LcPart) + (size_t)((ct + 1) * 4 + 15) / 16 * 16 +
                          (size_t)ct * 9 * sizeof(double) + (size_t)lay.cap + 16);
    }
    TileBufs tb;
    memset(&tb, 0, sizeof(tb));
    tb.start = start;
    tb.count_next = h->count;
    tb.key = h->key;
    tb.rank = h->rank;
    tb.acc = acc_cur;
    tb.status = h->status;
    auto kfn = k_lc_tile<T>;
    CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.bytes));
    time_begin(h);
    kfn<<<(c.ncells + ct - 1) / ct, 256, lay.bytes, h->stream>>>(c, st[h->cur], h->lcc, tb, sa,
                                                                 lay);
    time_end(h);
    launch_scan(h, h->start[1 - h->scur], nullptr, acc_nxt);
    launches += 8 + launch_scatter(h, st[h->cur], st[1 - h->cur], h->start[1 - h->scur]);
    CK(cudaGetLastError());
    h->cur = 1 - h->cur;
    h->scur = 1 - h->scur;
    h->sorted_for = (int64_t)step + 1;
    h->sums_for = -1;
    h->launches = launches;
    return MPCD_OK;
}

static int flow_accumulate(mpcd_handle *h);

extern "C" int mpcd_step(mpcd_handle *h, int nsteps, uint32_t step0) {
    if (!h || nsteps < 0) return MPCD_ERR_ARG;
    if (h->n <= 0) return MPCD_ERR_STATE;
    if (h->strategy < 0) h->strategy = default_strategy(h);
    if (h->tile_target <= 0)
        h->tile_target = h->dc.lc ? 512 : (h->prec == MPCD_PREC_MIXED ? 1024 : 768);
    if (nsteps > 0 && !h->dc.lc && kernel_family(h) == MPCD_KERNEL_PERSIST) {
        // all steps in one launch, or one launch per step while the flow
        // field is summed
        const int chunk = h->flow ? 1 : nsteps;
        for (int k = 0; k < nsteps; k += chunk) {
            const uint32_t s0 = step0 + (uint32_t)k;
            int r = h->dc.dim == 3 ? run_steps_per<3>(h, chunk, s0)
                                         : run_steps_per<2>(h, chunk, s0);
            if (r != MPCD_OK) return r;
            h->last_step = s0 + (uint32_t)(chunk - 1);
            h->steps += (uint64_t)chunk;
            h->stepped = true;
            if (h->flow && (r = flow_accumulate(h)) != MPCD_OK) return r;
        }
        return MPCD_OK;
    }
    for (int k = 0; k < nsteps; k++) {
        uint32_t step = step0 + (uint32_t)k;
        int r;
        if (h->dc.lc)
            r = h->prec == MPCD_PREC_FP64 ? run_step_lc<F64T<2>>(h, h->f, step)
                                          : run_step_lc<MixT<2>>(h, h->mx, step);
        else if (h->prec == MPCD_PREC_FP64 && kernel_family(h) == MPCD_KERNEL_RESIDENT)
            r = h->dc.dim == 3 ? run_step_r64<3>(h, step) : run_step_r64<2>(h, step);
        else if (h->prec == MPCD_PREC_FP64)
            r = h->dc.dim == 3 ? run_step<3, F64T<3>>(h, h->f, step)
                               : run_step<2, F64T<2>>(h, h->f, step);
        else if (kernel_family(h) == MPCD_KERNEL_RESIDENT)
            r = h->dc.dim == 3 ? run_step_res<3>(h, step) : run_step_res<2>(h, step);
        else
            r = h->dc.dim == 3 ? run_step<3, MixT<3>>(h, h->mx, step)
                               : run_step<2, MixT<2>>(h, h->mx, step);
        if (r != MPCD_OK) return r;
        h->last_step = step;
        h->steps++;
        h->stepped = true;
        if (h->flow && (r = flow_accumulate(h)) != MPCD_OK) return r;
    }
    return MPCD_OK;
}

extern "C" int mpcd_set_kernel(mpcd_handle *h, int kernel) {
    if (!h || kernel < MPCD_KERNEL_AUTO || kernel > MPCD_KERNEL_PERSIST) return MPCD_ERR_ARG;
    h->kernel = kernel;
    return MPCD_OK;
}

extern "C" int mpcd_set_sort_interval(mpcd_handle *h, int steps) {
    if (!h || steps < 1) return MPCD_ERR_ARG;
    h->sort_interval = steps;
    h->sort_age = -1;  // a new cycle: the next step re-sorts
    return MPCD_OK;
}

extern "C" int mpcd_set_strategy(mpcd_handle *h, int strategy, int tile_particles) {
    if (!h) return MPCD_ERR_ARG;
    if (strategy != MPCD_STRATEGY_SCATTER && strategy != MPCD_STRATEGY_RECOMPUTE &&
        strategy != -1)
        return MPCD_ERR_ARG;
    if (tile_particles != 0 && (tile_particles < 32 || tile_particles > 8192)) return MPCD_ERR_ARG;
    h->strategy = strategy;
    h->tile_target = tile_particles;
    return MPCD_OK;
}

extern "C" int mpcd_globals(mpcd_handle *h, double *kbtnow, double avnow[3]) {
    if (!h) return MPCD_ERR_ARG;
    CK(cudaMemcpyAsync(h->host_acc, acc_at(h, h->last_step),
                       sizeof(double) * ACC_WORDS,
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int dim = h->dc.dim;
    if (kbtnow) *kbtnow = h->n > 0 ? h->host_acc[ACC_KE] / (double)(h->n * dim) : 0.0;
    if (avnow)
        for (int d = 0; d < 3; d++)
            avnow[d] = d < dim ? h->host_acc[ACC_VCM + d] / h->dc.vol : 0.0;
    return MPCD_OK;
}

extern "C" int mpcd_timestep(mpcd_handle *h, uint32_t runtime, double AVNOW[3],
                             double *KBTNOW) {
    int r = mpcd_step(h, 1, runtime);
    if (r != MPCD_OK) return r;
    return mpcd_globals(h, KBTNOW, AVNOW);
}

extern "C" int mpcd_step_record(mpcd_handle *h, int nsteps, uint32_t step0, double *kbtnow,
                                double *avnow) {
    if (!h || nsteps < 0 || (nsteps > 0 && (!kbtnow || !avnow))) return MPCD_ERR_ARG;
    if (h->n <= 0) return MPCD_ERR_STATE;
    if (!h->host_ring &&
        cudaMallocHost((void **)&h->host_ring, sizeof(double) * 2 * kRecordBatch * ACC_WORDS) !=
            cudaSuccess)
        return MPCD_ERR_NOMEM;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto &e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            for (auto &f : ev)
                if (f) cudaEventDestroy(f);
            return MPCD_ERR_CUDA;
        }
    const int dim = h->dc.dim;
    const double inv_nd = 1.0 / (double)((long long)h->n * dim);
    // the globals of batch b in host half b & 1, converted while batch b + 1
    // runs on the GPU
    auto convert = [&](int b, int cnt) {
        CK(cudaEventSynchronize(ev[b & 1]));
        const double *src = h->host_ring + (size_t)(b & 1) * kRecordBatch * ACC_WORDS;
        for (int j = 0; j < cnt; j++) {
            const size_t k = (size_t)b * kRecordBatch + (size_t)j;
            kbtnow[k] = src[j * ACC_WORDS + ACC_KE] * inv_nd;
            for (int d = 0; d < 3; d++)
                avnow[3 * k + d] = d < dim ? src[j * ACC_WORDS + ACC_VCM + d] / h->dc.vol : 0.0;
        }
        return MPCD_OK;
    };
    int r = MPCD_OK;
    const int nb = (nsteps + kRecordBatch - 1) / kRecordBatch;
    for (int b = 0; b < nb && r == MPCD_OK; b++) {
        const int cnt = std::min(kRecordBatch, nsteps - b * kRecordBatch);
        const uint32_t s0 = step0 + (uint32_t)(b * kRecordBatch);
        r = mpcd_step(h, cnt, s0);
        if (r != MPCD_OK) break;
        // the batch's ring slots, in at most two contiguous pieces
        double *dst = h->host_ring + (size_t)(b & 1) * kRecordBatch * ACC_WORDS;
        int done = 0;
        while (done < cnt && r == MPCD_OK) {
            const uint32_t slot = (s0 + (uint32_t)done) % (uint32_t)kAccRing;
            const int piece = std::min(cnt - done, kAccRing - (int)slot);
            if (cudaMemcpyAsync(dst + (size_t)done * ACC_WORDS, h->acc + (size_t)slot * ACC_WORDS,
                                sizeof(double) * ACC_WORDS * piece, cudaMemcpyDeviceToHost,
                                h->stream) != cudaSuccess)
                r = MPCD_ERR_CUDA;
            done += piece;
        }
        if (r == MPCD_OK && cudaEventRecord(ev[b & 1], h->stream) != cudaSuccess)
            r = MPCD_ERR_CUDA;
        if (r == MPCD_OK && b > 0) r = convert(b - 1, kRecordBatch);
    }
    if (r == MPCD_OK && nb > 0) r = convert(nb - 1, nsteps - (nb - 1) * kRecordBatch);
    for (auto &e : ev) cudaEventDestroy(e);
    return r;
}

extern "C" int mpcd_get_status(mpcd_handle *h, mpcd_status *st) {
    if (!h || !st) return MPCD_ERR_ARG;
    unsigned long long w[ST_WORDS];
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(w, h->status, sizeof(w), cudaMemcpyDeviceToHost));
    st->steps = h->steps;
    st->escaped = w[ST_ESCAPED];
    st->bounce_limit = w[ST_BOUNCE];
    st->nonfinite = w[ST_NONFINITE];
    st->overflow = w[ST_OVERFLOW];
    st->sync_timeout = w[ST_SYNC];
    return MPCD_OK;
}

extern "C" int mpcd_set_stream(mpcd_handle *h, void *stream) {
    if (!h) return MPCD_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return MPCD_OK;
}

extern "C" int mpcd_launches_per_step(mpcd_handle *h) { return h ? h->launches : 0; }

extern "C" int mpcd_set_timing(mpcd_handle *h, int enable) {
    if (!h) return MPCD_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    time_clear(h);
    h->timing = enable != 0;
    return MPCD_OK;
}

extern "C" int mpcd_kernel_time(mpcd_handle *h, double *ms_total, int *launches) {
    if (!h || !ms_total || !launches) return MPCD_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    double t = 0.0;
    for (auto &p : h->tev) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p.first, p.second));
        t += ms;
    }
    *ms_total = t;
    *launches = (int)h->tev.size();
    time_clear(h);
    return MPCD_OK;
}

// Transverse momentum modes of the smallest wavevectors: for each ordered
// pair (a, b), a != b, j = sum_i v_i,a exp(-2 pi i x_i,b / L_b), accumulated
// as (Re, Im) in FP64 (phases in FP32).  Pair order: b outer, a inner.
template <int DIM>
__global__ void __launch_bounds__(256) k_modes_mix(const __grid_constant__ DevCfg c, MixState s,
                                                   int n, double *out) {
    constexpr int NM = DIM * (DIM - 1);
    double acc[2 * NM];
    for (int j = 0; j < 2 * NM; j++) acc[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 W = s.W[i];
        int ci[3];
        uint32_t f[3];
        pos_unpack(s.P[i], ci, f);
        const float v[3] = {W.x, W.y, W.z};
        int m = 0;
        for (int b = 0; b < DIM; b++) {
            const float x = (float)ci[b] + (float)((double)f[b] * kFxInv);
            float sn, cs;
            sincospif(2.0f * x / (float)c.L[b], &sn, &cs);
            for (int a = 0; a < DIM; a++) {
                if (a == b) continue;
                acc[2 * m] += (double)(v[a] * cs);
                acc[2 * m + 1] -= (double)(v[a] * sn);
                m++;
            }
        }
    }
    for (int j = 0; j < 2 * NM; j++) {
        double t = acc[j];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&out[j], t);
    }
}
template <int DIM>
__global__ void __launch_bounds__(256) k_modes_f64(const __grid_constant__ DevCfg c,
                                                   Fp64State s, int n, double *out) {
    constexpr int NM = DIM * (DIM - 1);
    double acc[2 * NM];
    for (int j = 0; j < 2 * NM; j++) acc[j] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int m = 0;
        for (int b = 0; b < DIM; b++) {
            double sn, cs;
            sincospi(2.0 * s.q[b][i] / (double)c.L[b], &sn, &cs);
            for (int a = 0; a < DIM; a++) {
                if (a == b) continue;
                acc[2 * m] += s.v[a][i] * cs;
                acc[2 * m + 1] -= s.v[a][i] * sn;
                m++;
            }
        }
    }
    for (int j = 0; j < 2 * NM; j++) {
        double t = acc[j];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&out[j], t);
    }
}

extern "C" int mpcd_transverse_modes(mpcd_handle *h, double *out, int *nmodes) {
    if (!h || !out) return MPCD_ERR_ARG;
    if (h->n <= 0) return MPCD_ERR_STATE;
    const int dim = h->dc.dim, nm = dim * (dim - 1);
    if (!h->modes) CK(cudaMalloc((void **)&h->modes, sizeof(double) * 12));
    CK(cudaMemsetAsync(h->modes, 0, sizeof(double) * 12, h->stream));
    const int grid = grid_for(h, h->n);
    if (h->prec == MPCD_PREC_MIXED) {
        if (dim == 3)
            k_modes_mix<3><<<grid, 256, 0, h->stream>>>(h->dc, h->mx[h->cur], h->n, h->modes);
        else
            k_modes_mix<2><<<grid, 256, 0, h->stream>>>(h->dc, h->mx[h->cur], h->n, h->modes);
    } else {
        if (dim == 3)
            k_modes_f64<3><<<grid, 256, 0, h->stream>>>(h->dc, h->f[h->cur], h->n, h->modes);
        else
            k_modes_f64<2><<<grid, 256, 0, h->stream>>>(h->dc, h->f[h->cur], h->n, h->modes);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, h->modes, sizeof(double) * 2 * nm, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (nmodes) *nmodes = nm;
    return MPCD_OK;
}

// The end-of-step cell properties on the unshifted grid (re-bin + the
// per-cell moments) into h->props, on the handle's stream; returns the
// views into it.
static int props_compute(mpcd_handle *h, CellProps *out) {
    const int n = h->n, dim = h->dc.dim, ns = h->dc.n_species;
    const size_t nc = (size_t)h->dc.ncells;
    const size_t bytes = nc * (7 * sizeof(double) + (size_t)(1 + (ns > 1 ? ns : 0)) * sizeof(int));
    if (!h->props && cudaMalloc((void **)&h->props, bytes) != cudaSuccess) return MPCD_ERR_NOMEM;
    CellProps p;
    p.mass = h->props;
    p.sv = p.mass + nc;
    p.sq = p.sv + 3 * nc;
    p.pop = (int *)(p.sq + 3 * nc);
    p.spc = ns > 1 ? p.pop + nc : nullptr;
    CK(cudaMemsetAsync(h->props, 0, bytes, h->stream));
    if (n > 0) {
        const int g = grid_for(h, n);
        if (h->prec == MPCD_PREC_FP64) {
            if (dim == 3)
                k_props_f64<3><<<g, 256, 0, h->stream>>>(h->dc, h->f[h->cur], n, p);
            else
                k_props_f64<2><<<g, 256, 0, h->stream>>>(h->dc, h->f[h->cur], n, p);
        } else {
            if (dim == 3)
                k_props_mix<3><<<g, 256, 0, h->stream>>>(h->dc, h->mx[h->cur], n, p);
            else
                k_props_mix<2><<<g, 256, 0, h->stream>>>(h->dc, h->mx[h->cur], n, p);
        }
        k_props_finish<<<grid_for(h, (int)nc), 256, 0, h->stream>>>(h->dc, p);
    }
    CK(cudaGetLastError());
    *out = p;
    return MPCD_OK;
}

extern "C" int mpcd_cell_props(mpcd_handle *h, int *pop, double *mass, double *vcm,
                               double *cm) {
    if (!h) return MPCD_ERR_ARG;
    // the re-bin on the unshifted grid and the per-cell moments, on the
    // device; only the cell arrays come back
    const size_t nc = (size_t)h->dc.ncells;
    CellProps p;
    int r = props_compute(h, &p);
    if (r != MPCD_OK) return r;
    if (pop) CK(cudaMemcpyAsync(pop, p.pop, nc * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (mass)
        CK(cudaMemcpyAsync(mass, p.mass, nc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (vcm)
        CK(cudaMemcpyAsync(vcm, p.sv, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
    if (cm)
        CK(cudaMemcpyAsync(cm, p.sq, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPCD_OK;
}

extern "C" int mpcd_cell_species(mpcd_handle *h, int *counts) {
    if (!h || !counts) return MPCD_ERR_ARG;
    const size_t nc = (size_t)h->dc.ncells;
    CellProps p;
    int r = props_compute(h, &p);
    if (r != MPCD_OK) return r;
    if (p.spc)
        CK(cudaMemcpyAsync(counts, p.spc, (size_t)h->dc.n_species * nc * sizeof(int),
                           cudaMemcpyDeviceToHost, h->stream));
    else  // one species: its populations are the cells'
        CK(cudaMemcpyAsync(counts, p.pop, nc * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPCD_OK;
}

extern "C" int mpcd_kinetic_energy(mpcd_handle *h, double *ke) {
    if (!h || !ke) return MPCD_ERR_ARG;
    *ke = 0.0;
    if (h->n <= 0) return MPCD_OK;
    int r = xfer_reserve(h, 256);
    if (r != MPCD_OK) return r;
    double *out = (double *)h->xfer;
    CK(cudaMemsetAsync(out, 0, sizeof(double), h->stream));
    const int g = grid_for(h, h->n);
    if (h->prec == MPCD_PREC_FP64)
        k_kinetic<<<g, 256, 0, h->stream>>>(h->dc, h->f[h->cur], h->n, out);
    else
        k_kinetic<<<g, 256, 0, h->stream>>>(h->dc, h->mx[h->cur], h->n, out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ke, out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPCD_OK;
}

extern "C" int mpcd_flow_enable(mpcd_handle *h, int enable) {
    if (!h) return MPCD_ERR_ARG;
    if (!enable) {
        cudaFree(h->flow);
        h->flow = nullptr;
        h->flow_steps = 0;
        return MPCD_OK;
    }
    const size_t bytes = 3 * (size_t)h->dc.ncells * sizeof(double);
    if (!h->flow && cudaMalloc((void **)&h->flow, bytes) != cudaSuccess) return MPCD_ERR_NOMEM;
    CK(cudaMemsetAsync(h->flow, 0, bytes, h->stream));
    h->flow_steps = 0;
    return MPCD_OK;
}

// One step's contribution to the flow field: the end-of-step cell
// velocities (the re-bin and localPROP of mpc.c:4936-4942) added to the sum.
static int flow_accumulate(mpcd_handle *h) {
    CellProps p;
    int r = props_compute(h, &p);
    if (r != MPCD_OK) return r;
    k_flow_add<<<grid_for(h, h->dc.ncells), 256, 0, h->stream>>>(h->dc, p.sv, h->flow);
    CK(cudaGetLastError());
    h->flow_steps++;
    return MPCD_OK;
}

extern "C" int mpcd_flow_read(mpcd_handle *h, double *flow, long long *nsteps, int reset) {
    if (!h) return MPCD_ERR_ARG;
    if (!h->flow) return MPCD_ERR_STATE;
    const size_t bytes = 3 * (size_t)h->dc.ncells * sizeof(double);
    if (flow) CK(cudaMemcpyAsync(flow, h->flow, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (nsteps) *nsteps = h->flow_steps;
    if (reset) {
        CK(cudaMemsetAsync(h->flow, 0, bytes, h->stream));
        h->flow_steps = 0;
    }
    CK(cudaStreamSynchronize(h->stream));
    return MPCD_OK;
}

extern "C" int mpcd_debug_cell_counts(mpcd_handle *h, int *pop) {
    if (!h || !pop) return MPCD_ERR_ARG;
    if (!h->stepped || h->n <= 0) return MPCD_ERR_STATE;
    const int nc = h->dc.ncells;
    const int64_t next = (int64_t)h->last_step + 1;
    int r = xfer_reserve(h, (size_t)nc * sizeof(int) + 256);
    if (r != MPCD_OK) return r;
    int *out = (int *)h->xfer;
    const int g = grid_for(h, nc);
    const size_t snc = (size_t)nc;
    if (h->sums_for == next && h->rsum) {
        const long long *plane = (const long long *)(h->rsum + (size_t)(next & 1) * snc) + 3 * snc;
        k_counts_plane<<<g, 256, 0, h->stream>>>(plane, nc, out);
    } else if (h->sums_for == next && h->r64sum) {
        const double *M = h->r64sum + (size_t)(next & 1) * 4 * snc;
        const int *cnt = h->dc.n_species > 1 ? h->r64pop + (size_t)(next & 1) * snc : nullptr;
        k_counts_r64<<<g, 256, 0, h->stream>>>(M, cnt, h->dc.mass[0], nc, out);
    } else if (h->per_pop_for == next && h->per_pop) {
        CK(cudaMemcpyAsync(out, h->per_pop, snc * sizeof(int), cudaMemcpyDeviceToDevice,
                           h->stream));
    } else if (h->sorted_for == next) {
        k_counts_start<<<g, 256, 0, h->stream>>>(h->start[h->scur], nc, out);
    } else {
        return MPCD_ERR_STATE;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(pop, out, snc * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MPCD_OK;
}

// The device arrays of state buffer b that a step reads and writes, with
// their sizes for the current particle count.
static void state_views(const mpcd_handle *h, int b, std::vector<std::pair<void *, size_t>> &v) {
    const size_t N = (size_t)h->n;
    v.clear();
    if (h->prec == MPCD_PREC_FP64) {
        const Fp64State &f = h->f[b];
        for (int d = 0; d < h->dc.dim; d++) {
            v.emplace_back(f.q[d], N * 8);
            v.emplace_back(f.v[d], N * 8);
        }
        v.emplace_back(f.pid, N * 4);
        if (f.sp) v.emplace_back(f.sp, N * 4);
        for (int d = 0; d < 2; d++)
            if (f.u[d]) v.emplace_back(f.u[d], N * 8);
    } else {
        const MixState &m = h->mx[b];
        v.emplace_back(m.P, N * 16);
        v.emplace_back(m.W, N * 16);
        if (m.sp) v.emplace_back(m.sp, N * 4);
        if (m.U) v.emplace_back(m.U, N * 8);
    }
}

static void apply_choice(mpcd_handle *h, const mpcd_tune_choice &c) {
    h->kernel = c.kernel;
    h->strategy = c.strategy;
    h->tile_target = c.tile_particles;
    h->sort_interval = c.sort_interval > 0 ? c.sort_interval : 30;
    h->sort_age = -1;
}

extern "C" int mpcd_autotune(mpcd_handle *h, int trial_steps, const char *cache_path,
                             mpcd_tune_choice *out) {
    if (!h || !out || trial_steps < 0) return MPCD_ERR_ARG;
    if (h->n <= 0) return MPCD_ERR_STATE;
    if (trial_steps == 0) trial_steps = 60;
    memset(out, 0, sizeof(*out));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, h->device));
    char key[512];
    int r = mpcd_tune_key(&h->cfg, h->n, prop.name, key, sizeof(key));
    if (r != MPCD_OK) return r;
    if (cache_path && mpcd_tune_cache_lookup(cache_path, key, out) == 1) {
        apply_choice(h, *out);
        return MPCD_OK;
    }
    // the plans that apply to this configuration
    std::vector<mpcd_tune_choice> cands;
    auto add = [&](int kernel, int strategy, int tile, int sort) {
        mpcd_tune_choice c;
        memset(&c, 0, sizeof(c));
        c.kernel = kernel;
        c.strategy = strategy;
        c.tile_particles = tile;
        c.sort_interval = sort;
        cands.push_back(c);
    };
    if (h->dc.lc) {
        for (int t : {320, 512, 1024}) add(MPCD_KERNEL_TILE, -1, t, 30);
    } else {
        if (h->prec == MPCD_PREC_FP64 && per_plan(h) > 0) add(MPCD_KERNEL_PERSIST, -1, 0, 30);
        if (h->dc.op == MPCD_COLL_ARBAXIS && !h->dc.any_phantom) {
            for (int si : {10, 20, 30, 60}) add(MPCD_KERNEL_RESIDENT, -1, 0, si);
            for (int st : {MPCD_STRATEGY_SCATTER, MPCD_STRATEGY_RECOMPUTE})
                add(MPCD_KERNEL_SPLIT, st, 0, 30);
        }
        for (int t : {512, 1024, 2048})
            for (int st : {MPCD_STRATEGY_SCATTER, MPCD_STRATEGY_RECOMPUTE})
                add(MPCD_KERNEL_TILE, st, t, 30);
        for (int st : {MPCD_STRATEGY_SCATTER, MPCD_STRATEGY_RECOMPUTE})
            add(MPCD_KERNEL_GROUP, st, 0, 30);
    }
    // snapshot of the state, the error counters and the bookkeeping
    CK(cudaStreamSynchronize(h->stream));
    std::vector<std::pair<void *, size_t>> views;
    state_views(h, h->cur, views);
    size_t total = sizeof(unsigned long long) * ST_WORDS;
    for (auto &vw : views) total += (vw.second + 255) / 256 * 256;
    char *snap = nullptr;
    if (cudaMalloc((void **)&snap, total) != cudaSuccess) return MPCD_ERR_NOMEM;
    {
        size_t o = 0;
        for (auto &vw : views) {
            CK(cudaMemcpyAsync(snap + o, vw.first, vw.second, cudaMemcpyDeviceToDevice, h->stream));
            o += (vw.second + 255) / 256 * 256;
        }
        CK(cudaMemcpyAsync(snap + o, h->status, sizeof(unsigned long long) * ST_WORDS,
                           cudaMemcpyDeviceToDevice, h->stream));
    }
    const int kernel0 = h->kernel, strategy0 = h->strategy, tile0 = h->tile_target,
              sort0 = h->sort_interval;
    const uint64_t steps0 = h->steps;
    const uint32_t last0 = h->last_step;
    const bool stepped0 = h->stepped;
    auto restore = [&]() -> int {
        state_views(h, 0, views);
        size_t o = 0;
        for (auto &vw : views) {
            if (cudaMemcpyAsync(vw.first, snap + o, vw.second, cudaMemcpyDeviceToDevice,
                                h->stream) != cudaSuccess)
                return MPCD_ERR_CUDA;
            o += (vw.second + 255) / 256 * 256;
        }
        if (cudaMemcpyAsync(h->status, snap + o, sizeof(unsigned long long) * ST_WORDS,
                            cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
            return MPCD_ERR_CUDA;
        h->cur = 0;
        h->sorted_for = -1;
        h->sums_for = -1;
        h->sort_age = -1;
        h->per_pop_for = -1;
        h->steps = steps0;
        h->last_step = last0;
        h->stepped = stepped0;
        return MPCD_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const uint32_t base = last0 + 1u;
    int best = -1, timed = 0;
    float best_ms = 0.f;
    for (size_t i = 0; i < cands.size() && r == MPCD_OK; i++) {
        r = restore();
        if (r != MPCD_OK) break;
        apply_choice(h, cands[i]);
        if (mpcd_step(h, 3, base) != MPCD_OK) {  // this plan does not apply: skip it
            cudaGetLastError();
            continue;
        }
        // the timed window starts with a re-sort and covers at least one
        // interval, so each plan pays its re-sorts at (or above) their
        // steady-state rate
        const int steps = cands[i].kernel == MPCD_KERNEL_RESIDENT
                              ? std::max(trial_steps, cands[i].sort_interval)
                              : trial_steps;
        h->sort_age = -1;
        cudaEventRecord(e0, h->stream);
        if (mpcd_step(h, steps, base + 3u) != MPCD_OK) {
            cudaGetLastError();
            cudaStreamSynchronize(h->stream);
            continue;
        }
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            r = MPCD_ERR_CUDA;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)steps;
        cands[i].us_per_step = 1e3 * (double)ms;
        timed++;
        if (best < 0 || ms < best_ms) {
            best = (int)i;
            best_ms = ms;
        }
    }
    const int rr = restore();
    if (r == MPCD_OK) r = rr;
    if (r == MPCD_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) r = MPCD_ERR_CUDA;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(snap);
    if (r != MPCD_OK || best < 0) {
        h->kernel = kernel0;
        h->strategy = strategy0;
        h->tile_target = tile0;
        h->sort_interval = sort0;
        return r != MPCD_OK ? r : MPCD_ERR_STATE;
    }
    *out = cands[best];
    out->candidates = timed;
    apply_choice(h, *out);
    if (cache_path) mpcd_tune_cache_store(cache_path, key, out);
    return MPCD_OK;
}
