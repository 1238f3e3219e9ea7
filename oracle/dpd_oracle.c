/* dpd_oracle.c -- CPU restatement of Osprey-DPD's per-timestep DPD loop.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  See dpd_oracle.h for the list of
 * reference functions restated here.  The code keeps the reference's data
 * structures where they fix the floating-point operation order: one doubly
 * linked bead list per CNT cell with push_front insertion, cells visited in
 * index order, the same-cell reverse scan and the 13-cell half shell in the
 * reference's neighbour order.  Everything is FP64 as in the reference.
 *
 * Compiled with -ffp-contract=off so that no multiply-add is fused; the
 * reference's own x86-64 build has no FMA either, which makes the LCG mode
 * bit-identical to the reference binary.
 */
#include "dpd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct dpdo_sim {
    dpdo_params p;
    double L[3], halfL[3], w[3];
    double halfdt, halfdt2, invrootdt, lamdt;   /* SetTimeStepConstants, CNTCell.cpp:180-203 */
    double* a;                                   /* owned copies of the type tables */
    double* g;
    int32_t T;

    int64_t ncell;
    int32_t* head;         /* first bead of each cell list, -1 if empty */
    int32_t* tail;         /* last bead of each cell list */
    uint8_t* ext;          /* cell lies on a box face (SimBox.cpp:789-798) */
    int32_t* nn27;         /* m_aNNCells, index 13+alpha+3beta+9gamma (SimBox.cpp:925-940) */
    int32_t* nn13;         /* m_aIntNNCells in the reference's insertion order (SimBox.cpp:845-856) */
    int32_t* cbl;          /* cell integer coordinates, 3 per cell */

    int64_t n;
    int64_t* id;
    int32_t* type;
    uint8_t* frozen;       /* !movable at upload: never moves (CBead::SetMovable, Bead.cpp:114-120) */
    uint8_t* movable;      /* per-step m_bIsMovable */
    int32_t* next;
    int32_t* prev;
    int32_t* cell;
    double *x, *u, *v, *f, *xo, *vo, *fo, *st;

    int64_t nb;
    int32_t *bh, *bt;
    double *k2, *l0, *bdx, *blen;
    int64_t na;
    int32_t *af, *as;
    double *k3, *phi0;

    /* slice stress profile (CMonitor::AddBeadStress / AddBondStress /
     * AddBondPairStress, Monitor.cpp:1900-2755), S = 0 when off */
    int32_t S, nbt, nbpt;
    double swidth, sinv;
    int32_t *btype, *bptype;       /* bond type per bond, bondpair type per bond pair */
    double *ssp, *ssb, *ssbp;      /* [S][T*T][9], [S][nbt][9], [S][nbpt][9] */
    double *bpf;                   /* per bond pair the forces on its beads, [4][3]; kept
                                      between steps like m_BeadXForce (BondPair.h:82) */
    int64_t slice_errors;

    uint64_t lcg;
    int64_t step;          /* m_SimTime of the step being evaluated */
    int64_t pairs;
    int64_t cell_errors;
};

/* ---------------------------------------------------------------- RNG --- */

/* CCNTCell::lcg / Randf, CNTCell.cpp:2454-2465. */
static double lcg_randf(uint64_t* state)
{
    *state = 6364136223846793005ull * (*state) + 1ull;
    const uint32_t r = (uint32_t)(*state >> 32);
    return (double)r * (1.0 / 4294967296.0);
}

/* Philox2x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 64-bit counter, 32-bit
 * key; per round (L,R) -> (hi(M*L) ^ k ^ R, lo(M*L)), k += W. */
static uint32_t philox2x32_10(uint32_t c0, uint32_t c1, uint32_t k)
{
    const uint32_t M = 0xD256D193u, W = 0x9E3779B9u;
    for (int r = 0; r < 10; ++r) {
        const uint64_t prod = (uint64_t)M * (uint64_t)c0;
        const uint32_t hi = (uint32_t)(prod >> 32), lo = (uint32_t)prod;
        c0 = hi ^ k ^ c1;
        c1 = lo;
        k += W;
    }
    return c0;
}

/* Key of the pair stream for one step: a 32-bit mix of the seed plus the step
 * times an odd constant, so distinct steps of one run get distinct keys. */
static uint32_t philox_step_key(uint64_t seed, int64_t step)
{
    uint32_t s = (uint32_t)seed ^ (uint32_t)(seed >> 32) * 0x85EBCA6Bu;
    s ^= s >> 16;
    s *= 0x7FEB352Du;
    s ^= s >> 15;
    return s + (uint32_t)step * 0xC2B2AE35u;
}

uint32_t dpdo_philox_pair(uint64_t seed, int64_t step, uint32_t id_lo, uint32_t id_hi)
{
    return philox2x32_10(id_lo, id_hi, philox_step_key(seed, step));
}

/* ------------------------------------------------------------- set-up --- */

static void set_step_constants(dpdo_sim* s)
{
    s->halfdt = 0.5 * s->p.dt;
    s->halfdt2 = 0.5 * s->p.dt * s->p.dt;
    s->invrootdt = sqrt(24.0 * s->p.kT / s->p.dt);
    s->lamdt = s->p.lambda * s->p.dt;
}

/* CSimBox::MapCelltoIndex, SimBox.cpp:888-920. */
static int64_t map_cell(const dpdo_sim* s, int64_t i, int64_t j, int64_t k, int alpha, int beta, int gamma)
{
    const int64_t nx = s->p.nx, ny = s->p.ny, nxy = nx * ny, total = s->ncell;
    int64_t idx = i + j * nx + k * nxy;
    idx += alpha;
    if (idx >= nx * (1 + j + k * ny)) idx -= nx;
    else if (idx < nx * (j + k * ny)) idx += nx;
    idx += beta * nx;
    if (idx >= (1 + k) * nxy) idx -= nxy;
    else if (idx < k * nxy) idx += nxy;
    idx += gamma * nxy;
    if (idx >= total) idx -= total;
    else if (idx < 0) idx += total;
    return idx;
}

dpdo_sim* dpdo_create(const dpdo_params* p)
{
    if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1 || p->ntypes < 1 || !p->a || !p->gamma) return NULL;
    dpdo_sim* s = (dpdo_sim*)calloc(1, sizeof *s);
    if (!s) return NULL;
    s->p = *p;
    s->T = p->ntypes;
    s->a = (double*)malloc(sizeof(double) * s->T * s->T);
    s->g = (double*)malloc(sizeof(double) * s->T * s->T);
    memcpy(s->a, p->a, sizeof(double) * s->T * s->T);
    memcpy(s->g, p->gamma, sizeof(double) * s->T * s->T);
    s->p.a = s->a;
    s->p.gamma = s->g;
    s->w[0] = p->wx; s->w[1] = p->wy; s->w[2] = p->wz;
    /* CCNTCell::SetSimBoxLengths, CNTCell.cpp:143-158 */
    s->L[0] = (double)p->nx * p->wx;
    s->L[1] = (double)p->ny * p->wy;
    s->L[2] = (double)p->nz * p->wz;
    for (int d = 0; d < 3; ++d) s->halfL[d] = 0.5 * s->L[d];
    set_step_constants(s);
    s->lcg = p->seed;

    s->ncell = (int64_t)p->nx * p->ny * p->nz;
    s->head = (int32_t*)malloc(sizeof(int32_t) * s->ncell);
    s->tail = (int32_t*)malloc(sizeof(int32_t) * s->ncell);
    s->ext = (uint8_t*)malloc(s->ncell);
    s->nn27 = (int32_t*)malloc(sizeof(int32_t) * s->ncell * 27);
    s->nn13 = (int32_t*)malloc(sizeof(int32_t) * s->ncell * 13);
    s->cbl = (int32_t*)malloc(sizeof(int32_t) * s->ncell * 3);
    /* CSimBox::MakeCNTCells, SimBox.cpp:767-877 */
    for (int64_t k = 0; k < p->nz; ++k)
        for (int64_t j = 0; j < p->ny; ++j)
            for (int64_t i = 0; i < p->nx; ++i) {
                const int64_t c = p->nx * (p->ny * k + j) + i;
                s->head[c] = s->tail[c] = -1;
                s->ext[c] = (i == 0 || i == p->nx - 1 || j == 0 || j == p->ny - 1 || k == 0 || k == p->nz - 1);
                s->cbl[3 * c] = (int32_t)i; s->cbl[3 * c + 1] = (int32_t)j; s->cbl[3 * c + 2] = (int32_t)k;
            }
    for (int64_t c = 0; c < s->ncell; ++c) {
        int nint = 0;
        const int64_t i = s->cbl[3 * c], j = s->cbl[3 * c + 1], k = s->cbl[3 * c + 2];
        for (int gamma = -1; gamma < 2; ++gamma)
            for (int beta = -1; beta < 2; ++beta)
                for (int alpha = -1; alpha < 2; ++alpha) {
                    const int64_t nb = map_cell(s, i, j, k, alpha, beta, gamma);
                    s->nn27[27 * c + 13 + alpha + 3 * beta + 9 * gamma] = (int32_t)nb;
                    if (gamma == 1 || (gamma == 0 && (alpha == 1 || (alpha == 0 && beta == 1))))
                        s->nn13[13 * c + nint++] = (int32_t)nb;
                }
    }
    return s;
}

static void free_beads(dpdo_sim* s)
{
    free(s->id); free(s->type); free(s->frozen); free(s->movable); free(s->next); free(s->prev);
    free(s->cell); free(s->x); free(s->u); free(s->v); free(s->f); free(s->xo); free(s->vo);
    free(s->fo); free(s->st);
    s->id = NULL;
}

static void free_slices(dpdo_sim* s)
{
    free(s->btype); free(s->bptype); free(s->ssp); free(s->ssb); free(s->ssbp);
    s->btype = s->bptype = NULL;
    s->ssp = s->ssb = s->ssbp = NULL;
    s->S = 0;
}

static void free_topo(dpdo_sim* s)
{
    free(s->bh); free(s->bt); free(s->k2); free(s->l0); free(s->bdx); free(s->blen);
    free(s->af); free(s->as); free(s->k3); free(s->phi0); free(s->bpf);
    s->bpf = NULL;
    free_slices(s);
    s->bh = NULL; s->nb = 0; s->na = 0;
}

void dpdo_destroy(dpdo_sim* s)
{
    if (!s) return;
    free_beads(s);
    free_topo(s);
    free(s->head); free(s->tail); free(s->ext); free(s->nn27); free(s->nn13); free(s->cbl);
    free(s->a); free(s->g);
    free(s);
}

/* std::list::push_front (CCNTCell::AddBeadtoCell, CNTCell.cpp:2339-2342). */
static void push_front(dpdo_sim* s, int64_t c, int32_t b)
{
    s->prev[b] = -1;
    s->next[b] = s->head[c];
    if (s->head[c] >= 0) s->prev[s->head[c]] = b;
    else s->tail[c] = b;
    s->head[c] = b;
    s->cell[b] = (int32_t)c;
}

static void erase(dpdo_sim* s, int64_t c, int32_t b)
{
    if (s->prev[b] >= 0) s->next[s->prev[b]] = s->next[b];
    else s->head[c] = s->next[b];
    if (s->next[b] >= 0) s->prev[s->next[b]] = s->prev[b];
    else s->tail[c] = s->prev[b];
}

int dpdo_set_beads(dpdo_sim* s, int64_t n, const int64_t* id, const int32_t* type,
                   const uint8_t* movable, const double* x3, const double* unpbc3,
                   const double* v3, const double* f3)
{
    if (!s || n < 0 || (n > 0 && (!id || !type || !x3 || !v3))) return -1;
    free_beads(s);
    s->n = n;
    s->id = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
    s->type = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    s->frozen = (uint8_t*)malloc(n ? n : 1);
    s->movable = (uint8_t*)malloc(n ? n : 1);
    s->next = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    s->prev = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    s->cell = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    double** arrs[] = {&s->x, &s->u, &s->v, &s->f, &s->xo, &s->vo, &s->fo};
    for (int k = 0; k < 7; ++k) *arrs[k] = (double*)calloc(3 * (n ? n : 1), sizeof(double));
    s->st = (double*)calloc(9 * (n ? n : 1), sizeof(double));
    for (int64_t c = 0; c < s->ncell; ++c) s->head[c] = s->tail[c] = -1;
    for (int64_t b = 0; b < n; ++b) {
        if (type[b] < 0 || type[b] >= s->T) return -2;
        s->id[b] = id[b];
        s->type[b] = type[b];
        s->frozen[b] = movable ? !movable[b] : 0;
        s->movable[b] = !s->frozen[b];
        for (int d = 0; d < 3; ++d) {
            s->x[3 * b + d] = x3[3 * b + d];
            s->u[3 * b + d] = unpbc3 ? unpbc3[3 * b + d] : x3[3 * b + d];
            s->v[3 * b + d] = v3[3 * b + d];
            s->f[3 * b + d] = f3 ? f3[3 * b + d] : 0.0;
        }
    }
    /* CSimBox::AssignBeadstoCells, SimBox.cpp:715-762: bead-vector order, push_front. */
    for (int64_t b = 0; b < n; ++b) {
        const int64_t ix = (int64_t)(s->x[3 * b] / s->p.wx);
        const int64_t iy = (int64_t)(s->x[3 * b + 1] / s->p.wy);
        const int64_t iz = (int64_t)(s->x[3 * b + 2] / s->p.wz);
        const int64_t c = (int64_t)s->p.nx * ((int64_t)s->p.ny * iz + iy) + ix;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= s->p.nx || iy >= s->p.ny || iz >= s->p.nz || c >= s->ncell)
            return -3;
        push_front(s, c, (int32_t)b);
    }
    return 0;
}

static int32_t find_id(const dpdo_sim* s, int64_t idv)
{
    /* Ids are 1..N in bead order for every state the reference builds
     * (InitialState.cpp:490-500); fall back to a scan otherwise. */
    if (idv >= 1 && idv <= s->n && s->id[idv - 1] == idv) return (int32_t)(idv - 1);
    for (int64_t b = 0; b < s->n; ++b)
        if (s->id[b] == idv) return (int32_t)b;
    return -1;
}

int dpdo_set_topology(dpdo_sim* s, int64_t nb, const int64_t* head_id, const int64_t* tail_id,
                      const double* k2, const double* l0, int64_t na,
                      const int64_t* first_bond, const int64_t* second_bond,
                      const double* k3, const double* phi0)
{
    if (!s || nb < 0 || na < 0 || !s->id) return -1;
    free_topo(s);
    s->nb = nb;
    s->na = na;
    s->bh = (int32_t*)malloc(sizeof(int32_t) * (nb ? nb : 1));
    s->bt = (int32_t*)malloc(sizeof(int32_t) * (nb ? nb : 1));
    s->k2 = (double*)malloc(sizeof(double) * (nb ? nb : 1));
    s->l0 = (double*)malloc(sizeof(double) * (nb ? nb : 1));
    s->bdx = (double*)calloc(3 * (nb ? nb : 1), sizeof(double));
    s->blen = (double*)calloc(nb ? nb : 1, sizeof(double));
    s->af = (int32_t*)malloc(sizeof(int32_t) * (na ? na : 1));
    s->as = (int32_t*)malloc(sizeof(int32_t) * (na ? na : 1));
    s->k3 = (double*)malloc(sizeof(double) * (na ? na : 1));
    s->phi0 = (double*)malloc(sizeof(double) * (na ? na : 1));
    s->bpf = (double*)calloc(12 * (na ? na : 1), sizeof(double));
    for (int64_t i = 0; i < nb; ++i) {
        s->bh[i] = find_id(s, head_id[i]);
        s->bt[i] = find_id(s, tail_id[i]);
        if (s->bh[i] < 0 || s->bt[i] < 0) return -2;
        s->k2[i] = k2[i];
        s->l0[i] = l0[i];
    }
    for (int64_t i = 0; i < na; ++i) {
        if (first_bond[i] < 0 || first_bond[i] >= nb || second_bond[i] < 0 || second_bond[i] >= nb) return -3;
        s->af[i] = (int32_t)first_bond[i];
        s->as[i] = (int32_t)second_bond[i];
        s->k3[i] = k3[i];
        s->phi0[i] = phi0[i];
    }
    return 0;
}

int dpdo_set_dt(dpdo_sim* s, double dt)
{
    if (!s || !(dt > 0.0)) return -1;   /* ChangeTimeStepConstants ignores dt <= 0 */
    s->p.dt = dt;
    set_step_constants(s);
    return 0;
}

int dpdo_set_pair(dpdo_sim* s, int32_t ti, int32_t tj, double a, double gamma)
{
    if (!s || ti < 0 || tj < 0 || ti >= s->T || tj >= s->T) return -1;
    s->a[ti * s->T + tj] = s->a[tj * s->T + ti] = a;
    s->g[ti * s->T + tj] = s->g[tj * s->T + ti] = gamma;
    return 0;
}

/* --------------------------------------------------------- the step --- */

/* CCNTCell::UpdatePos, DPD branch and migration, CNTCell.cpp:1634-2262. */
static void update_pos(dpdo_sim* s)
{
    const double dt = s->p.dt;
    for (int64_t c = 0; c < s->ncell; ++c) {
        double BL[3], TR[3];
        for (int d = 0; d < 3; ++d) {
            BL[d] = (double)s->cbl[3 * c + d] * s->w[d];   /* CCNTCell ctor, CNTCell.cpp:598-604 */
            TR[d] = BL[d] + s->w[d];
        }
        int32_t b = s->head[c];
        while (b >= 0) {
            const int32_t nextb = s->next[b];
            if (!s->movable[b]) { b = nextb; continue; }
            double* x = s->x + 3 * b;
            double* v = s->v + 3 * b;
            double* f = s->f + 3 * b;
            double dx[3];
            for (int d = 0; d < 3; ++d) {
                s->xo[3 * b + d] = x[d];
                s->vo[3 * b + d] = v[d];
                s->fo[3 * b + d] = f[d];
            }
            for (int d = 0; d < 3; ++d) dx[d] = dt * v[d] + s->halfdt2 * f[d];
            for (int d = 0; d < 3; ++d) x[d] += dx[d];
            for (int d = 0; d < 3; ++d) s->u[3 * b + d] += dx[d];
            for (int d = 0; d < 3; ++d) v[d] = s->vo[3 * b + d] + s->lamdt * s->fo[3 * b + d];
            for (int d = 0; d < 3; ++d) f[d] = 0.0;

            /* The 27-way decision tree reduces to an independent test per axis:
             * x > TR moves +1, else x < BL moves -1 (CNTCell.cpp:1768-2254). */
            int mv[3];
            for (int d = 0; d < 3; ++d) mv[d] = (x[d] > TR[d]) ? 1 : ((x[d] < BL[d]) ? -1 : 0);
            s->movable[b] = 0;   /* SetNotMovable in every branch */
            if (mv[0] || mv[1] || mv[2]) {
                const int32_t nb = s->nn27[27 * c + 13 + mv[0] + 3 * mv[1] + 9 * mv[2]];
                if (s->ext[c] && s->ext[nb]) {
                    for (int d = 0; d < 3; ++d) {
                        if (mv[d] > 0 && x[d] > s->L[d]) x[d] -= s->L[d];
                        else if (mv[d] < 0 && x[d] < 0.0) x[d] += s->L[d];
                    }
                }
                /* m_aNNCells[..]->m_lBeads.push_front(bead); m_lBeads.erase(it):
                 * unlink first because both lists share the bead's links here */
                erase(s, c, b);
                push_front(s, nb, b);
            }
            b = nextb;
        }
    }
}

/* One interacting pair, CNTCell.cpp:1192-1301 (same cell) and 1363-1522 (neighbour cell). */
/* ------------------------------------------------- slice stress profile --- */

/* The shared body of CMonitor::AddBeadStress (Monitor.cpp:1900-2107),
 * AddBondStress (2283-2518) and AddBondPairStress (2520-2755): the
 * Goetz-Lipowsky split of one contribution fdx (force x separation, 9
 * components) over the z slices between two beads.  za is the z of the bead
 * the separation points to (bead 1, the bond head, bead j+1), zb the other's;
 * zDiff the z separation.  arr is [S][K][9]; idx the type index. */
static void slice_add(dpdo_sim* s, double* arr, int64_t K, int64_t idx, const double fdx[9], double zDiff,
                      double za, double zb)
{
    double up, lo;
    if (zDiff > 0.00001) {
        up = za * s->sinv;
        lo = zb * s->sinv;
    } else if (zDiff < -0.00001) {
        zDiff = -zDiff;
        up = zb * s->sinv;
        lo = za * s->sinv;
    } else {
        up = za * s->sinv;
        lo = up;
    }
    const int64_t S = s->S;
    int64_t ui = (int64_t)up;
    const double ur = up - (double)ui;
    int64_t li = (int64_t)lo;
    const double lr = lo - (double)li;
    if (ui < 0 || ui >= S || li < 0 || li >= S || idx < 0 || idx >= K) { s->slice_errors++; return; }
#define SLICE_ADD(sl, fac) do { double* q_ = arr + ((sl) * K + idx) * 9; \
        for (int c_ = 0; c_ < 9; ++c_) q_[c_] += fdx[c_] * (fac); } while (0)
    if (ui == li) {
        if (up != lo || ur > 0.00001) {
            double* q = arr + (li * K + idx) * 9;
            for (int c = 0; c < 9; ++c) q[c] += fdx[c];
        } else {
            SLICE_ADD(ui, 0.5);
            if (--li < 0) li += S;
            SLICE_ADD(li, 0.5);
        }
    } else {
        const double inner = s->swidth / zDiff;
        if (ui > li) {
            for (int64_t k = li + 1; k <= ui - 1; ++k) SLICE_ADD(k, inner);
        } else {
            for (int64_t kp = li + 1; kp <= S + ui - 1; ++kp) {
                int64_t k = kp;
                if (k >= S) k -= S;
                SLICE_ADD(k, inner);
            }
        }
        if (lr > 0.000001) SLICE_ADD(li, (1.0 - lr) * inner);
        else SLICE_ADD(li, inner);
        if (ur > 0.000001) SLICE_ADD(ui, ur * inner);
    }
#undef SLICE_ADD
}

static void outer9(const double f[3], const double d[3], double o[9])
{
    o[0] = f[0] * d[0]; o[1] = f[0] * d[1]; o[2] = f[0] * d[2];
    o[3] = f[1] * d[0]; o[4] = f[1] * d[1]; o[5] = f[1] * d[2];
    o[6] = f[2] * d[0]; o[7] = f[2] * d[1]; o[8] = f[2] * d[2];
}

int dpdo_set_slice_stress(dpdo_sim* s, int32_t nslices, int32_t nbondtypes, const int32_t* bond_type,
                          int32_t nbptypes, const int32_t* bondpair_type)
{
    if (!s || nslices < 0 || nbondtypes < 0 || nbptypes < 0) return -1;
    free_slices(s);
    if (nslices == 0) return 0;
    if ((s->nb > 0 && !bond_type) || (s->na > 0 && !bondpair_type)) return -1;
    s->S = nslices;
    s->nbt = nbondtypes;
    s->nbpt = nbptypes;
    /* m_GridZCellWidth = m_SimBoxZLength / GridZCellNo (Monitor.cpp:247), inverse as Monitor.cpp:2185 */
    s->swidth = s->L[2] / (double)nslices;
    s->sinv = 1.0 / s->swidth;
    s->btype = (int32_t*)malloc(sizeof(int32_t) * (s->nb ? s->nb : 1));
    s->bptype = (int32_t*)malloc(sizeof(int32_t) * (s->na ? s->na : 1));
    for (int64_t i = 0; i < s->nb; ++i) s->btype[i] = bond_type[i];
    for (int64_t i = 0; i < s->na; ++i) s->bptype[i] = bondpair_type[i];
    s->ssp = (double*)calloc((size_t)nslices * s->T * s->T * 9, sizeof(double));
    s->ssb = (double*)calloc((size_t)nslices * (nbondtypes ? nbondtypes : 1) * 9, sizeof(double));
    s->ssbp = (double*)calloc((size_t)nslices * (nbptypes ? nbptypes : 1) * 9, sizeof(double));
    return 0;
}

int dpdo_get_slice_stress(const dpdo_sim* s, double* pair, double* bond, double* bondpair)
{
    if (!s || !s->S) return -1;
    if (pair) memcpy(pair, s->ssp, sizeof(double) * (size_t)s->S * s->T * s->T * 9);
    if (bond) memcpy(bond, s->ssb, sizeof(double) * (size_t)s->S * s->nbt * 9);
    if (bondpair) memcpy(bondpair, s->ssbp, sizeof(double) * (size_t)s->S * s->nbpt * 9);
    return 0;
}

int64_t dpdo_slice_errors(const dpdo_sim* s) { return s ? s->slice_errors : -1; }

/* CMonitor::ZeroSliceStress (Monitor.cpp:2109), called at the start of every
 * step (SimBox.cpp:999). */
static void zero_slices(dpdo_sim* s)
{
    if (!s->S) return;
    memset(s->ssp, 0, sizeof(double) * (size_t)s->S * s->T * s->T * 9);
    memset(s->ssb, 0, sizeof(double) * (size_t)s->S * (s->nbt ? s->nbt : 1) * 9);
    memset(s->ssbp, 0, sizeof(double) * (size_t)s->S * (s->nbpt ? s->nbpt : 1) * 9);
}

static void pair_force(dpdo_sim* s, int32_t b1, int32_t b2, int minimg)
{
    double dx[3], dv[3], nf[3];
    for (int d = 0; d < 3; ++d) {
        dx[d] = s->x[3 * b1 + d] - s->x[3 * b2 + d];
        dv[d] = s->v[3 * b1 + d] - s->v[3 * b2 + d];
    }
    if (minimg) {
        for (int d = 0; d < 3; ++d) {
            if (dx[d] > s->halfL[d]) dx[d] = dx[d] - s->L[d];
            else if (dx[d] < -s->halfL[d]) dx[d] = dx[d] + s->L[d];
        }
    }
    const double dr2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
    if (!(dr2 < 1.0)) return;
    const double dr = sqrt(dr2);
    if (!(dr > 0.000000001)) return;
    const double wr = 1.0 - dr;
    const double wr2 = wr * wr;
    const int32_t t1 = s->type[b1], t2 = s->type[b2];
    const double conForce = s->a[t1 * s->T + t2] * wr;
    const double rdotv = (dx[0] * dv[0] + dx[1] * dv[1] + dx[2] * dv[2]) / dr;
    const double gammap = s->g[t1 * s->T + t2] * wr2;
    const double dissForce = -gammap * rdotv;
    double u;
    if (s->p.noise == DPDO_NOISE_LCG) {
        u = lcg_randf(&s->lcg);
    } else {
        const int64_t i1 = s->id[b1], i2 = s->id[b2];
        const uint32_t lo = (uint32_t)(i1 < i2 ? i1 : i2), hi = (uint32_t)(i1 < i2 ? i2 : i1);
        u = (double)dpdo_philox_pair(s->p.seed, s->step, lo, hi) * (1.0 / 4294967296.0);
    }
    const double randForce = sqrt(gammap) * s->invrootdt * (0.5 - u);
    for (int d = 0; d < 3; ++d) nf[d] = (conForce + dissForce + randForce) * dx[d] / dr;
    s->pairs++;
    for (int d = 0; d < 3; ++d) s->f[3 * b1 + d] += nf[d];
    for (int d = 0; d < 3; ++d) s->f[3 * b2 + d] -= nf[d];
    double* st = s->st + 9 * b1;
    st[0] += dx[0] * nf[0]; st[1] += dx[1] * nf[0]; st[2] += dx[2] * nf[0];
    st[3] += dx[0] * nf[1]; st[4] += dx[1] * nf[1]; st[5] += dx[2] * nf[1];
    st[6] += dx[0] * nf[2]; st[7] += dx[1] * nf[2]; st[8] += dx[2] * nf[2];
    if (s->S) {   /* CMonitor::AddBeadStress(bead1, bead2, newForce, dx), CNTCell.cpp:1310 */
        double fdx[9];
        outer9(nf, dx, fdx);
        slice_add(s, s->ssp, (int64_t)s->T * s->T, (int64_t)t1 * s->T + t2, fdx, dx[2], s->x[3 * b1 + 2],
                  s->x[3 * b2 + 2]);
    }
}

/* CCNTCell::UpdateForce, DPD branch, CNTCell.cpp:1103-1572. */
static void update_force(dpdo_sim* s)
{
    s->pairs = 0;
    for (int64_t c = 0; c < s->ncell; ++c) {
        for (int32_t b1 = s->head[c]; b1 >= 0; b1 = s->next[b1]) {
            for (int k = 0; k < 9; ++k) s->st[9 * b1 + k] = 0.0;
            /* reverse scan of the same cell until bead 1 is reached */
            for (int32_t b2 = s->tail[c]; b2 >= 0 && s->id[b2] != s->id[b1]; b2 = s->prev[b2])
                pair_force(s, b1, b2, 0);
            for (int k = 0; k < 13; ++k) {
                const int32_t nc = s->nn13[13 * c + k];
                const int minimg = s->ext[c] && s->ext[nc];
                for (int32_t b2 = s->head[nc]; b2 >= 0; b2 = s->next[b2]) pair_force(s, b1, b2, minimg);
            }
        }
    }
}

/* CBond::AddForce (serial build), Bond.cpp:111-162. */
static void bond_forces(dpdo_sim* s)
{
    for (int64_t i = 0; i < s->nb; ++i) {
        const int32_t h = s->bh[i], t = s->bt[i];
        double* bd = s->bdx + 3 * i;
        bd[0] = s->u[3 * h] - s->u[3 * t];
        bd[1] = s->u[3 * h + 1] - s->u[3 * t + 1];
        bd[2] = s->u[3 * h + 2] - s->u[3 * t + 2];
        const double len = sqrt(bd[0] * bd[0] + bd[1] * bd[1] + bd[2] * bd[2]);
        s->blen[i] = len;
        const double fx = s->k2[i] * (s->l0[i] - len) * bd[0] / len;
        const double fy = s->k2[i] * (s->l0[i] - len) * bd[1] / len;
        const double fz = s->k2[i] * (s->l0[i] - len) * bd[2] / len;
        s->f[3 * h] += fx; s->f[3 * h + 1] += fy; s->f[3 * h + 2] += fz;
        s->f[3 * t] -= fx; s->f[3 * t + 1] -= fy; s->f[3 * t + 2] -= fz;
        double* st = s->st + 9 * h;
        st[0] += bd[0] * fx; st[1] += bd[1] * fx; st[2] += bd[2] * fx;
        st[3] += bd[0] * fy; st[4] += bd[1] * fy; st[5] += bd[2] * fy;
        st[6] += bd[0] * fz; st[7] += bd[1] * fz; st[8] += bd[2] * fz;
        if (s->S) {   /* CMonitor::AddBondStress, Polymer.cpp:677-680 */
            const double fb[3] = {fx, fy, fz};
            double fdx[9];
            outer9(fb, bd, fdx);
            slice_add(s, s->ssb, s->nbt, s->btype[i], fdx, bd[2], s->x[3 * h + 2], s->x[3 * t + 2]);
        }
    }
}

/* CMonitor::AddBondPairStress (Monitor.cpp:2520-2755) of bond pair i: the
 * three bead pairs first.tail -> first.head -> second.head -> first.tail,
 * separation = unPBC difference, force = 0.33333333 * (F[j+1] - F[j]). */
static void bondpair_slices(dpdo_sim* s, int64_t i)
{
    if (!s->S) return;
    const int32_t b1 = s->af[i], b2 = s->as[i];
    const int32_t bead[4] = {s->bt[b1], s->bh[b1], s->bh[b2], s->bt[b1]};
    const double* bp = s->bpf + 12 * i;
    for (int j = 0; j < 3; ++j) {
        const int jp1 = j + 1;
        double dx[3], fo[3], fdx[9];
        for (int d = 0; d < 3; ++d) dx[d] = s->u[3 * bead[jp1] + d] - s->u[3 * bead[j] + d];
        for (int d = 0; d < 3; ++d) fo[d] = 0.33333333 * (bp[3 * jp1 + d] - bp[3 * j + d]);
        outer9(fo, dx, fdx);
        slice_add(s, s->ssbp, s->nbpt, s->bptype[i], fdx, dx[2], s->x[3 * bead[jp1] + 2], s->x[3 * bead[j] + 2]);
    }
}

/* CBondPair::AddForce, BondPair.cpp:138-286 (the P2 / phi observables are
 * not forces and are left out). */
static void bondpair_forces(dpdo_sim* s)
{
    for (int64_t i = 0; i < s->na; ++i) {
        const int32_t b1 = s->af[i], b2 = s->as[i];
        const double firstLength = s->blen[b1], secondLength = s->blen[b2];
        const double magProduct = firstLength * secondLength;
        if (!(magProduct > 0.0001)) {
            bondpair_slices(s, i);   /* stale m_BeadXForce, as the reference */
            continue;
        }
        const double* first = s->bdx + 3 * b1;
        const double* second = s->bdx + 3 * b2;
        const double b1MagSq = firstLength * firstLength;
        const double b2MagSq = secondLength * secondLength;
        const double b1Dotb2 = first[0] * second[0] + first[1] * second[1] + first[2] * second[2];
        const double b1b2Overb1Sq = b1Dotb2 / b1MagSq;
        const double b1b2Overb2Sq = b1Dotb2 / b2MagSq;
        const double cosPhiSq = b1b2Overb1Sq * b1b2Overb2Sq;
        double forceMag;
        if (fabs(b1Dotb2) > 0.000001) {
            const double prefactor = sqrt(1.0 / cosPhiSq - 1.0);
            if (s->phi0[i] > 0.0)
                forceMag = s->k3[i] * (cos(s->phi0[i]) - sin(s->phi0[i]) / prefactor) / magProduct;
            else
                forceMag = s->k3[i] / magProduct;
        } else {
            forceMag = s->k3[i] / magProduct;
        }
        double f0[3], f2[3], f1[3];
        for (int d = 0; d < 3; ++d) f0[d] = forceMag * (b1b2Overb1Sq * first[d] - second[d]);
        for (int d = 0; d < 3; ++d) f2[d] = forceMag * (first[d] - b1b2Overb2Sq * second[d]);
        for (int d = 0; d < 3; ++d) f1[d] = -f0[d] - f2[d];
        const int32_t ft = s->bt[b1], sh = s->bh[b2], fh = s->bh[b1];
        for (int d = 0; d < 3; ++d) s->f[3 * ft + d] += f0[d];
        for (int d = 0; d < 3; ++d) s->f[3 * sh + d] += f2[d];
        for (int d = 0; d < 3; ++d) s->f[3 * fh + d] += f1[d];
        double* bp = s->bpf + 12 * i;   /* m_BeadXForce[0..3], [3] = [0] (BondPair.cpp:231-262) */
        for (int d = 0; d < 3; ++d) { bp[d] = f0[d]; bp[3 + d] = f1[d]; bp[6 + d] = f2[d]; bp[9 + d] = f0[d]; }
        bondpair_slices(s, i);
    }
}

/* CCNTCell::UpdateMom, CNTCell.cpp:2280-2310 (angular momentum is an
 * observable only and is not kept). */
static void update_mom(dpdo_sim* s)
{
    for (int64_t c = 0; c < s->ncell; ++c)
        for (int32_t b = s->head[c]; b >= 0; b = s->next[b]) {
            s->movable[b] = !s->frozen[b];
            if (!s->movable[b]) continue;
            for (int d = 0; d < 3; ++d)
                s->v[3 * b + d] = s->vo[3 * b + d] + s->halfdt * (s->f[3 * b + d] + s->fo[3 * b + d]);
        }
}

/* CSimBox::UpdateRenormalisedMom, SimBox.cpp:3177-3225: the squared momenta
 * of all beads in the CNT cells, summed cell by cell in list order (x, y, z
 * of a bead in turn), give the scale sqrt(sum / (3 N kT)) that every
 * momentum component is divided by. */
int dpdo_renormalise_mom(dpdo_sim* s)
{
    if (!s || s->n <= 0 || !(s->p.kT > 0.0)) return -1;
    double sum = 0.0;
    for (int64_t c = 0; c < s->ncell; ++c)
        for (int32_t b = s->head[c]; b >= 0; b = s->next[b]) {
            sum += s->v[3 * b] * s->v[3 * b];
            sum += s->v[3 * b + 1] * s->v[3 * b + 1];
            sum += s->v[3 * b + 2] * s->v[3 * b + 2];
        }
    const double scale = sqrt(sum / (3.0 * (double)s->n * s->p.kT));
    for (int64_t c = 0; c < s->ncell; ++c)
        for (int32_t b = s->head[c]; b >= 0; b = s->next[b])
            for (int d = 0; d < 3; ++d) s->v[3 * b + d] = s->v[3 * b + d] / scale;
    return 0;
}

/* CCNTCell::CheckBeadsinCell, CNTCell.cpp:2628-2700. */
static void check_cells(dpdo_sim* s)
{
    s->cell_errors = 0;
    for (int64_t b = 0; b < s->n; ++b) {
        const int64_t ix = (int64_t)(s->x[3 * b] / s->p.wx);
        const int64_t iy = (int64_t)(s->x[3 * b + 1] / s->p.wy);
        const int64_t iz = (int64_t)(s->x[3 * b + 2] / s->p.wz);
        if ((int64_t)s->p.nx * ((int64_t)s->p.ny * iz + iy) + ix != s->cell[b]) s->cell_errors++;
    }
}

int dpdo_step(dpdo_sim* s, int64_t first_step, int32_t nsteps)
{
    if (!s || !s->id || nsteps < 0) return -1;
    for (int32_t k = 0; k < nsteps; ++k) {
        s->step = first_step + k;
        update_pos(s);
        zero_slices(s);
        update_force(s);
        bond_forces(s);
        bondpair_forces(s);
        update_mom(s);
        check_cells(s);
    }
    return 0;
}

int dpdo_get(const dpdo_sim* s, double* x3, double* unpbc3, double* v3, double* f3, double* stress9)
{
    if (!s || !s->id) return -1;
    const size_t n3 = sizeof(double) * 3 * (size_t)s->n;
    if (x3) memcpy(x3, s->x, n3);
    if (unpbc3) memcpy(unpbc3, s->u, n3);
    if (v3) memcpy(v3, s->v, n3);
    if (f3) memcpy(f3, s->f, n3);
    if (stress9) memcpy(stress9, s->st, 3 * n3);
    return 0;
}

int dpdo_get_cells(const dpdo_sim* s, int32_t* cell)
{
    if (!s || !s->id || !cell) return -1;
    memcpy(cell, s->cell, sizeof(int32_t) * (size_t)s->n);
    return 0;
}

int64_t dpdo_cell_errors(const dpdo_sim* s) { return s ? s->cell_errors : -1; }
int64_t dpdo_pair_count(const dpdo_sim* s) { return s ? s->pairs : -1; }

/* ---------------------------------------------------------------- random initial state
 *
 * CRandomBuilder::Assemble (RandomBuilder.cpp:71-361) for a box without
 * walls, in three dimensions, restated operation by operation:
 *   - the velocity-magnitude table CBuilder::MaxwellDist (Builder.cpp:104-126):
 *     max(n, 10^7) entries from the recurrence vel = sqrt(2 log(M f/(M - f))),
 *     f = exp(vel^2/2), the last entry repeating the one before;
 *   - per bead i in bead order, six draws of the reference's LCG
 *     (CCNTCell::Randf / lcg, CNTCell.cpp:2454-2466; state' = 6364136223846793005
 *     state + 1, draw = (state' >> 32) / 2^32): table index, x, y, z (each
 *     L * u, set to 0 when within 1e-4 of the upper face, RandomBuilder.cpp:
 *     139-191), then theta = acos(1 - 2u), phi = 2 pi u, v = vmag (sin theta
 *     cos phi, sin theta sin phi, cos theta) (RandomBuilder.cpp:201-208);
 *   - bonds in polymer order: where a component of tail - head exceeds 1 in
 *     magnitude the tail's coordinate becomes head + the unit vector's
 *     component (RandomBuilder.cpp:241-311); the unPBC position equals x;
 *   - centre-of-mass velocity removed and the velocities scaled to kT with
 *     the 3N normalisation (RandomBuilder.cpp:315-361), sums in bead order.
 * `skip` draws of the generator are consumed first (the reference's draws
 * before the builder runs).  Returns 0, or -1 - i for bead i drawn outside
 * the box (the reference's "coord outside box" error). */
static double rb_draw(uint64_t* st)
{
    *st = 6364136223846793005ull * *st + 1ull;
    return (double)(uint32_t)(*st >> 32) * (1.0 / 4294967296.0);
}

int dpdo_random_state(int64_t n, const double L[3], double kT, uint64_t seed, int64_t skip, int64_t nb,
                      const int64_t* bond_head, const int64_t* bond_tail, double* x3, double* v3)
{
    const int64_t M = n > 10000000 ? n : 10000000;
    double* tab = (double*)malloc(sizeof(double) * (size_t)M);
    if (!tab) return -1000000000;
    const double dM = (double)M;
    double factor = 1.0;
    for (int64_t j = 0; j < M - 1; ++j) {
        const double vel = sqrt(2.0 * log(dM * factor / (dM - factor)));
        factor = exp(0.5 * vel * vel);
        tab[j] = vel;
    }
    tab[M - 1] = tab[M - 2];
    uint64_t st = seed;
    for (int64_t k = 0; k < skip; ++k) (void)rb_draw(&st);
    const double twopi = 2.0 * 3.141592653589793238;   /* xxBase::m_globalTwoPI, xxBase.cpp:30-31 */
    double vcm[3] = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < n; ++i) {
        const int64_t index = (int64_t)((double)(size_t)M * rb_draw(&st));
        const double vmag = tab[index];
        double xp[3];
        for (int d = 0; d < 3; ++d) {
            xp[d] = 0.0 + L[d] * rb_draw(&st);
            if (xp[d] > L[d]) { free(tab); return (int)(-1 - i); }
            if (L[d] - xp[d] < 0.0001) xp[d] = 0.0;
        }
        const double vtheta = acos(1.0 - 2.0 * rb_draw(&st));
        const double vphi = twopi * rb_draw(&st);
        double* v = v3 + 3 * i;
        v[0] = vmag * sin(vtheta) * cos(vphi);
        v[1] = vmag * sin(vtheta) * sin(vphi);
        v[2] = vmag * cos(vtheta);
        vcm[0] += v[0];
        vcm[1] += v[1];
        vcm[2] += v[2];
        for (int d = 0; d < 3; ++d) x3[3 * i + d] = xp[d];
    }
    free(tab);
    for (int64_t k = 0; k < nb; ++k) {
        double* h = x3 + 3 * bond_head[k];
        double* t = x3 + 3 * bond_tail[k];
        const double rd[3] = {t[0] - h[0], t[1] - h[1], t[2] - h[2]};
        const double rmag = sqrt(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
        const double ru[3] = {rd[0] / rmag, rd[1] / rmag, rd[2] / rmag};
        for (int d = 0; d < 3; ++d)
            if (fabs(rd[d]) > 1.0) t[d] = h[d] + ru[d];
    }
    for (int d = 0; d < 3; ++d) vcm[d] /= (double)n;
    double vtotal = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double* v = v3 + 3 * i;
        v[0] -= vcm[0];
        v[1] -= vcm[1];
        v[2] -= vcm[2];
        vtotal = vtotal + v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    }
    vtotal = sqrt(vtotal / (double)(3 * n));
    for (int64_t i = 0; i < 3 * n; ++i) v3[i] = sqrt(kT) * v3[i] / vtotal;
    return 0;
}

/* ---------------------------------------------------------------- lamella initial state
 *
 * CLamellaBuilder::Assemble (LamellaBuilder.cpp:126-1010) with the geometry
 * of CInitialStateLamella::ValidateData (InitialStateLamella.cpp:705-770),
 * no walls and no polymerised bonds, restated operation by operation:
 *   - the bilayer polymers (type lipid_type, in polymer order) split into the
 *     upper monolayer (the first (long)(upper_fraction * total)) and the
 *     lower one; each monolayer's polymers sit on the vertices of a hexagonal
 *     lattice of spacing 0.999 sqrt(1.1547 area / count), walked row by row
 *     from (0.001 e1x, 0.001 e2y) (LamellaBuilder.cpp:250-290, 382-650);
 *   - per polymer: the tail at centre + sign 0.2, the head at the monolayer's
 *     head plane, the beads between on the head-tail line spaced
 *     0.5 thickness / (beads head..tail - 1) (linearise), or scattered about
 *     the axis with three draws each;
 *   - the other polymers, in polymer order, in the free regions below and
 *     above the bilayer (CBuilder::isRandom::Assemble, Builder.cpp:293-480):
 *     one draw choosing the region by its share of the free length, three
 *     draws per bead ((0.95 L) u in-plane, region start + width u along the
 *     normal), then the polymer's bonds shortened as the random builder's;
 *   - unPBC = x (Builder.cpp:4391-4404);
 *   - in-plane Maxwell velocities (CBuilder::AssignMaxwellVelocities, 2-d
 *     branch, Builder.cpp:4207-4330): per bead the table index and
 *     phi = 2 pi u, v = vmag (cos phi, sin phi); centre-of-mass velocity
 *     removed, velocities divided by sqrt(sum v.v / (2 N kT)), the pair placed
 *     in the two in-plane axes (normal x: (0, VY, VX); y: (VX, 0, VY);
 *     z: (VX, VY, 0)).
 * Beads: n in polymer order; polymer p holds beads [poly_first[p],
 * poly_first[p+1]); head_offset / tail_offset are the bilayer polymer's head
 * and tail bead offsets; normal 0, 1, 2 = x, y, z; bonds as bead indices in
 * polymer order.  Returns 0, -1 for bad arguments, -2 when the bilayer does
 * not fit the box, -3 when the lattice runs out of the box (the reference's
 * "lamella lattice outside SimBox"). */
int dpdo_lamella_state(int64_t n, const double L[3], double kT, uint64_t seed, int64_t skip, int64_t npoly,
                       const int64_t* poly_first, const int32_t* poly_type, int32_t lipid_type,
                       int32_t head_offset, int32_t tail_offset, int32_t normal, double centre_frac,
                       double thickness, int32_t linearise, double upper_fraction, int64_t nb,
                       const int64_t* bond_head, const int64_t* bond_tail, double* x3, double* v3)
{
    if (n < 1 || npoly < 1 || normal < 0 || normal > 2 || poly_first[0] != 0 || poly_first[npoly] != n) return -1;
    /* the lattice lengths (InitialStateLamella.cpp:705-730) and the axes that
     * take the lattice's two coordinates (LamellaBuilder.cpp:440-600: normal x:
     * y, z; normal y: z, x; normal z: x, y) */
    const double l1 = normal == 0 ? L[1] : L[0], l2 = normal == 2 ? L[1] : L[2], Ln = L[normal];
    const int p0 = normal == 0 ? 1 : (normal == 1 ? 2 : 0), p1 = normal == 0 ? 2 : (normal == 1 ? 0 : 1);
    const double centre = centre_frac * Ln;
    if (centre + 0.5 * thickness > Ln || centre - 0.5 * thickness < 0.0) return -2;
    double lower = centre - 0.5 * thickness, upper = centre + 0.5 * thickness;
    const double area = l1 * l2;
    int64_t total = 0, first_lipid = -1, size = 0;
    for (int64_t p = 0; p < npoly; ++p)
        if (poly_type[p] == lipid_type) {
            if (first_lipid < 0) { first_lipid = p; size = poly_first[p + 1] - poly_first[p]; }
            else if (poly_first[p + 1] - poly_first[p] != size) return -1;
            ++total;
        }
    if (total == 0 || head_offset < 0 || tail_offset < 0 || head_offset >= size || tail_offset >= size ||
        head_offset == tail_offset)
        return -1;
    /* beads head..tail inclusive (LamellaBuilder.cpp:300-336) */
    int64_t counter = 0;
    {
        int bcount = 0, pend = -1;
        for (int64_t k = 0; k < size; ++k) {
            if (k == head_offset && !bcount) { bcount = 1; pend = tail_offset; counter++; }
            else if (k == tail_offset && !bcount) { bcount = 1; pend = head_offset; counter++; }
            else if (k == pend) { bcount = 0; counter++; }
            else if (bcount) counter++;
        }
    }
    int64_t mtot[2], mfirst[2], lat[2];
    double mhead[2];
    const double msign[2] = {1.0, -1.0};
    mtot[0] = (int64_t)(upper_fraction * (double)total);
    mtot[1] = total - mtot[0];
    int mono = 0;
    if (mtot[0] == 0) {
        mono = 1; mfirst[0] = 0; mfirst[1] = 0; lat[0] = 0; lat[1] = mtot[1];
        mhead[0] = 0.0; mhead[1] = lower; upper = centre;
    } else if (mtot[1] == 0) {
        mono = 1; mfirst[0] = 0; mfirst[1] = 0; lat[0] = mtot[0]; lat[1] = 0;
        mhead[0] = upper; mhead[1] = 0.0; lower = centre;
    } else {
        mfirst[0] = 0; mfirst[1] = mtot[0]; lat[0] = mtot[0]; lat[1] = mtot[1];
        mhead[0] = upper; mhead[1] = lower;
    }
    double hs[2];
    if (mono) {
        if (mtot[0] == 0) { hs[0] = 0.0; hs[1] = 0.999 * sqrt(1.1547 * area / (double)lat[1]); }
        else { hs[0] = 0.999 * sqrt(1.1547 * area / (double)lat[0]); hs[1] = 0.0; }
    } else {
        hs[0] = 0.999 * sqrt(1.1547 * area / (double)lat[0]);
        hs[1] = 0.999 * sqrt(1.1547 * area / (double)lat[1]);
    }
    const double e1x[2] = {hs[0], hs[1]}, e2x[2] = {0.5 * hs[0], 0.5 * hs[1]};
    const double e2y[2] = {0.866025 * hs[0], 0.866025 * hs[1]};
    double cspace[2];
    cspace[0] = 0.5 * thickness / (double)(counter - 1);
    cspace[1] = cspace[0];
    /* the bilayer polymers in polymer order */
    int64_t* lip = (int64_t*)malloc(sizeof(int64_t) * (size_t)total);
    if (!lip) return -1;
    for (int64_t p = 0, k = 0; p < npoly; ++p)
        if (poly_type[p] == lipid_type) lip[k++] = p;
    uint64_t st = seed;
    for (int64_t k = 0; k < skip; ++k) (void)rb_draw(&st);
    for (int mi = 0; mi < 2; ++mi) {
        double hexp[3] = {0.001 * e1x[mi], 0.001 * e2y[mi], 0.0};
        double xp[3] = {hexp[0], hexp[1], hexp[2]};
        int64_t rowCounter = 0;
        for (int64_t iv = mfirst[mi]; iv < mfirst[mi] + lat[mi]; ++iv) {
            const int64_t b0 = poly_first[lip[iv]];
            double* head = x3 + 3 * (b0 + head_offset);
            double* tail = x3 + 3 * (b0 + tail_offset);
            tail[p0] = xp[0];
            tail[p1] = xp[1];
            tail[normal] = centre + msign[mi] * 0.2;
            head[p0] = xp[0];
            head[p1] = xp[1];
            head[normal] = mhead[mi];
            double beadCounter = 1.0;
            for (int64_t k = 0; k < size; ++k) {
                if (k == head_offset || k == tail_offset) continue;
                double* q = x3 + 3 * (b0 + k);
                if (linearise) {
                    q[p0] = xp[0];
                    q[p1] = xp[1];
                    q[normal] = head[normal] - msign[mi] * beadCounter * cspace[mi];
                    beadCounter += 1.0;
                } else {
                    /* three draws, axes in x, y, z order as the reference's statements */
                    for (int d = 0; d < 3; ++d) {
                        if (d == normal) q[d] = centre + 0.5 * msign[mi] * thickness * rb_draw(&st);
                        else if (d == p0) q[d] = xp[0] + 0.5 * e1x[mi] * rb_draw(&st);
                        else q[d] = xp[1] + 0.5 * e2y[mi] * rb_draw(&st);
                    }
                    if (q[p0] > L[p0]) q[p0] -= 0.5 * e1x[mi];
                    if (q[p1] > L[p1]) q[p1] -= 0.5 * e2y[mi];
                }
            }
            /* the next vertex (LamellaBuilder.cpp:605-650) */
            hexp[0] += e1x[mi];
            if (hexp[0] > l1 + (double)rowCounter * e2x[mi]) {
                rowCounter++;
                hexp[0] = (double)rowCounter * e2x[mi];
                hexp[1] += e2y[mi];
                xp[0] = hexp[0];
                xp[1] = hexp[1];
                if (hexp[1] >= l2) { free(lip); return -3; }
            } else if (hexp[0] > l1) {
                xp[0] = hexp[0] - l1;
            } else {
                xp[0] = hexp[0];
                xp[1] = hexp[1];
            }
        }
    }
    free(lip);
    /* the other polymers in the free regions (Builder.cpp:293-480) */
    const double ex[6] = {0.0, 0.0, lower, upper, Ln - 0.0, Ln};
    double freeLength = 0.0, ratio[2];
    for (int i = 1; i < 3; ++i) freeLength += ex[2 * i] - ex[2 * i - 1];
    {
        double cum = 0.0;
        for (int i = 1; i < 3; ++i) { cum += (ex[2 * i] - ex[2 * i - 1]) / freeLength; ratio[i - 1] = cum; }
    }
    int64_t bq = 0;   /* bonds in polymer order: the next bond to look at */
    for (int64_t p = 0; p < npoly; ++p) {
        const int64_t b0 = poly_first[p], b1 = poly_first[p + 1];
        while (bq < nb && bond_head[bq] < b0) ++bq;
        if (poly_type[p] == lipid_type) continue;
        const double rindex = rb_draw(&st);
        int index = 0, unassigned = 1;
        for (int k = 0; k < 2; ++k)
            if (unassigned && rindex <= ratio[k]) { unassigned = 0; index = k; }
        const double width = ex[2 * index + 2] - ex[2 * index + 1];
        for (int64_t b = b0; b < b1; ++b) {
            double xp[3];
            for (int d = 0; d < 3; ++d) {
                if (d == normal) xp[d] = ex[2 * index + 1] + width * rb_draw(&st);
                else xp[d] = 0.95 * L[d] * rb_draw(&st);
            }
            for (int d = 0; d < 3; ++d) x3[3 * b + d] = xp[d];
        }
        for (int64_t k = bq; k < nb && bond_head[k] < b1 && bond_head[k] >= b0; ++k) {
            double* h = x3 + 3 * bond_head[k];
            double* t = x3 + 3 * bond_tail[k];
            const double rd[3] = {t[0] - h[0], t[1] - h[1], t[2] - h[2]};
            const double rmag = sqrt(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
            const double ru[3] = {rd[0] / rmag, rd[1] / rmag, rd[2] / rmag};
            for (int d = 0; d < 3; ++d)
                if (fabs(rd[d]) > 1.0) t[d] = h[d] + ru[d];
        }
    }
    /* in-plane Maxwell velocities (Builder.cpp:4207-4330, 2-d branch) */
    const int64_t M = n > 10000000 ? n : 10000000;
    double* tab = (double*)malloc(sizeof(double) * (size_t)M);
    double* vx = (double*)malloc(sizeof(double) * (size_t)n);
    double* vy = (double*)malloc(sizeof(double) * (size_t)n);
    if (!tab || !vx || !vy) { free(tab); free(vx); free(vy); return -1; }
    {
        const double dM = (double)M;
        double factor = 1.0;
        for (int64_t j = 0; j < M - 1; ++j) {
            const double vel = sqrt(2.0 * log(dM * factor / (dM - factor)));
            factor = exp(0.5 * vel * vel);
            tab[j] = vel;
        }
        tab[M - 1] = tab[M - 2];
    }
    const double twopi = 2.0 * 3.141592653589793238;   /* xxBase::m_globalTwoPI */
    double vcm[3] = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < n; ++i) {
        const int64_t index = (int64_t)((double)(size_t)M * rb_draw(&st));
        const double vmag = tab[index];
        const double vphi = twopi * rb_draw(&st);
        vx[i] = vmag * cos(vphi);
        vy[i] = vmag * sin(vphi);
        vcm[0] += vx[i];
        vcm[1] += vy[i];
    }
    free(tab);
    const double dn = (double)n;
    vcm[0] /= dn;
    vcm[1] /= dn;
    vcm[2] /= dn;
    double vtotal = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        vx[i] -= vcm[0];
        vy[i] -= vcm[1];
        const double vz = 0.0 - vcm[2];
        vtotal = vtotal + vx[i] * vx[i] + vy[i] * vy[i] + vz * vz;
    }
    vtotal = sqrt(vtotal / (2.0 * dn * kT));
    for (int64_t i = 0; i < n; ++i) {
        const double VX = vx[i] / vtotal, VY = vy[i] / vtotal;
        double* v = v3 + 3 * i;
        if (normal == 0) { v[0] = 0.0; v[1] = VY; v[2] = VX; }
        else if (normal == 1) { v[0] = VX; v[1] = 0.0; v[2] = VY; }
        else { v[0] = VX; v[1] = VY; v[2] = 0.0; }
    }
    free(vx);
    free(vy);
    return 0;
}
