/*
 * ref_harness.c -- parity checker built from the reference's OWN sources.
 *
 * TEST INFRASTRUCTURE ONLY.  Linked with the reference's hot-path C files
 * (compiled in place from the reference tree by oracle/Makefile) into
 * oracle/_ref/libmplb_ref.so.  Only tests/, the smoke check and bench.py's
 * CPU-baseline leg load it.
 *
 * The harness builds the reference's host structures (latticeMesh,
 * macroFields, lbeField) in memory from the flat descriptors of
 * include/mplb_gpu.h instead of reading dictionary and mesh files, and then
 * calls the reference's functions in the order of its solver:
 *   start-up   multiPhasePP.c:122-147 (equilibrium f, g; interForce; heatSource)
 *   time step  multiPhasePP.c:157-240 (collision/lbstream/updateBoundaries f, g;
 *              macroDensity; heatSource; macroTemperature; interForce;
 *              macroVelocity), with updateTime() semantics for time.current
 *              (src/IO/time/timeOptions.c:35-64).
 * Results are copied out as doubles, so no float-precision writer is involved
 * in the lattice checks; ref_write_field runs the reference's field writers
 * for the byte-for-byte check of the library's writers.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <pthread.h>

#include <latticeMesh.h>
#include <macroFields.h>
#include <lbeField.h>
#include <latticeModel.h>
#include <basic.h>
#include <generalLbe.h>
#include <pseudoPot.h>
#include <asciiRaw.h>
#include <binaryRaw.h>
#include <pvtu.h>

#include "../include/mplb_gpu.h"

typedef struct ref_case {
    latticeMesh mesh;
    macroFields mf;
    lbeField f, g;
    int has_f, has_g;
    int Q;
    uint32_t n;
} ref_case;

static double** rows_alloc(uint32_t n, uint32_t m) {
    double** r = (double**)malloc((size_t)n * sizeof(double*));
    for (uint32_t i = 0; i < n; i++) r[i] = (double*)calloc(m, sizeof(double));
    return r;
}

static void rows_free(double** r, uint32_t n) {
    if (!r) return;
    for (uint32_t i = 0; i < n; i++) free(r[i]);
    free(r);
}

static void setup_field(ref_case* c, lbeField* fl, const mplb_field_desc* d) {
    memset(fl, 0, sizeof(*fl));
    fl->value = rows_alloc(c->n, c->Q);
    fl->swap = rows_alloc(c->n, c->Q);
    fl->scalarSource = (scalar*)calloc(c->n, sizeof(scalar));
    fl->model = (lbeModel)d->model;
    fl->update = d->update ? 1 : 0;
    scalar* lam = (scalar*)calloc(MPLB_MAX_Q, sizeof(scalar));
    for (int k = 0; k < MPLB_MAX_Q; k++) lam[k] = d->Lambda[k];
    switch (d->model) {
    case MPLB_LIMRT:
        fl->lbparam.liMRT.Lambda = lam;
        fl->lbparam.liMRT.sigma = d->sigma;
        fl->lbparam.liMRT.surfaceTension = d->surface_tension ? liSurfTen : no_st;
        fl->lbparam.liMRT.kappa_st = d->kappa_st;
        break;
    case MPLB_XUMRT:
        fl->lbparam.xuMRT.Lambda = lam;
        fl->lbparam.xuMRT.sigma = d->sigma;
        fl->lbparam.xuMRT.surfaceTension = d->surface_tension ? xuSurfTen : noXuSurf;
        fl->lbparam.xuMRT.kappa_st = d->kappa_st;
        break;
    case MPLB_LITEMPMRT:
        fl->lbparam.liTempMRT.Lambda = lam;
        break;
    case MPLB_MYMRT:
        fl->lbparam.myMRT.Lambda = lam;
        fl->lbparam.myMRT.alpha_1 = d->alpha_1;
        fl->lbparam.myMRT.alpha_2 = d->alpha_2;
        break;
    default:
        fl->lbparam.liMRT.Lambda = lam;
        break;
    }
    uint32_t np = c->mesh.mesh.bd.nbd;
    fl->boundary = (bdField*)calloc(np ? np : 1, sizeof(bdField));
    for (uint32_t p = 0; p < np; p++) {
        fl->boundary[p].type = d->bc_type ? (bdType)d->bc_type[p] : periodic;
        if (d->bc_type && d->bc_value) {
            if (d->bc_type[p] == MPLB_BC_FIXEDT) fl->boundary[p].param.ft.T = d->bc_value[3 * p];
            if (d->bc_type[p] == MPLB_BC_FIXEDU)
                for (int j = 0; j < 3; j++) fl->boundary[p].param.fu.U[j] = d->bc_value[3 * p + j];
            if (d->bc_type[p] == MPLB_BC_FIXEDRANDOMT) {
                /* readFixedRandomTParam.c:14-75: value, pert, duration */
                fl->boundary[p].param.frdt.T = d->bc_value[3 * p];
                fl->boundary[p].param.frdt.p = d->bc_value[3 * p + 1];
                fl->boundary[p].param.frdt.psteps = (int)d->bc_value[3 * p + 2];
                fl->boundary[p].param.frdt.localTStep = 0;
            }
        }
    }
    fl->nreq = 0;
}

ref_case* ref_create(const mplb_mesh_desc* md, const mplb_eos_desc* ed,
                     const mplb_field_desc* fd, const mplb_field_desc* gd, uint32_t start_time) {
    ref_case* c = (ref_case*)calloc(1, sizeof(ref_case));
    DdQq model = md->lattice == MPLB_D3Q15 ? D3Q15 : D2Q9;
    c->n = md->n_points;

    /* Lattice tables exactly as setLatticeInfo() assigns them (setLatticeInfo.c:68-84). */
    latticeInfo* L = &c->mesh.lattice;
    L->model = model;
    L->cs2 = cs2(model);
    L->Q = latticeQ(model);
    L->d = latticeD(model);
    L->vel = latticeVelocities(model);
    L->reverse = latticeReverseDir(model);
    L->omega = latticeWeights(model);
    L->weights = ppWeights(model);
    L->M = MRTMatrix(model);
    L->invM = MRTInvMatrix(model);
    c->Q = L->Q;

    /* Single rank, no ghosts. */
    c->mesh.parallel.pid = 0;
    c->mesh.parallel.worldSize = 1;
    c->mesh.parallel.nlocal = c->n;
    c->mesh.parallel.nghosts = 0;
    c->mesh.parallel.nrg = (uint*)calloc(1, sizeof(uint));
    c->mesh.parallel.nsg = (uint*)calloc(1, sizeof(uint));

    basicMesh* m = &c->mesh.mesh;
    m->nPoints = c->n;
    m->Q = c->Q;
    m->nb = (int**)malloc((size_t)c->n * sizeof(int*));
    m->isOnBnd = (uint*)malloc((size_t)c->n * sizeof(uint));
    m->points = (int**)malloc((size_t)c->n * sizeof(int*));
    for (uint32_t i = 0; i < c->n; i++) {
        m->nb[i] = (int*)malloc((size_t)c->Q * sizeof(int));
        m->points[i] = (int*)calloc(3, sizeof(int));
        uint is_b = 0;
        for (int k = 0; k < c->Q; k++) {
            m->nb[i][k] = md->nb[(size_t)i * c->Q + k];
            if (m->nb[i][k] == -1) is_b++;
        }
        /* readLatticeMesh.c:171-203: any missing neighbour marks the node. */
        m->isOnBnd[i] = is_b ? 1 : 0;
        if (md->points)
            for (int j = 0; j < 3; j++) m->points[i][j] = md->points[(size_t)i * 3 + j];
    }
    m->bd.nbd = md->n_patches;
    m->bd.nbdelem = (uint*)calloc(md->n_patches ? md->n_patches : 1, sizeof(uint));
    m->bd.bdPoints = (uint**)calloc(md->n_patches ? md->n_patches : 1, sizeof(uint*));
    size_t off = 0;
    for (uint32_t p = 0; p < md->n_patches; p++) {
        m->bd.nbdelem[p] = md->patch_count[p];
        m->bd.bdPoints[p] = (uint*)malloc((size_t)(md->patch_count[p] ? md->patch_count[p] : 1) * sizeof(uint));
        for (uint32_t i = 0; i < md->patch_count[p]; i++) m->bd.bdPoints[p][i] = md->patch_nodes[off + i];
        off += md->patch_count[p];
        snprintf(m->bd.bdNames[p], 100, "P%u", p);
    }

    EOSInfo* E = &c->mesh.EOS;
    E->etype = (eosType)ed->type;
    switch (ed->type) {
    case MPLB_EOS_CS: E->eParam.csp.a = ed->a; E->eParam.csp.b = ed->b; break;
    case MPLB_EOS_PR: E->eParam.prp.a = ed->a; E->eParam.prp.b = ed->b; E->eParam.prp.omega = ed->w; break;
    case MPLB_EOS_VDW: E->eParam.vdwparam.a = ed->a; E->eParam.vdwparam.b = ed->b; break;
    default: break;
    }
    E->R = ed->R; E->G = ed->G; E->M = ed->M; E->Cv = ed->Cv; E->rho_0 = ed->rho_0;
    E->g = (scalar*)malloc(3 * sizeof(scalar));
    E->fext = (scalar*)malloc(3 * sizeof(scalar));
    for (int j = 0; j < 3; j++) { E->g[j] = ed->g[j]; E->fext[j] = ed->fext[j]; }

    c->mesh.time.start = start_time;
    c->mesh.time.current = start_time;
    c->mesh.time.end = 0xffffffffu;
    c->mesh.time.writeInterval = 0xffffffffu;
    c->mesh.time.stp = 0;

    c->mf.rho = (scalar*)calloc(c->n, sizeof(scalar));
    c->mf.T = (scalar*)calloc(c->n, sizeof(scalar));
    c->mf.p = (scalar*)calloc(c->n, sizeof(scalar));
    c->mf.U = rows_alloc(c->n, 3);
    c->mf.Fi = rows_alloc(c->n, 3);
    c->mf.Ft = rows_alloc(c->n, 3);

    c->has_f = fd && fd->model != MPLB_NO_MODEL;
    c->has_g = gd && gd->model != MPLB_NO_MODEL;
    mplb_field_desc none;
    memset(&none, 0, sizeof(none));
    none.model = MPLB_LIMRT;
    setup_field(c, &c->f, c->has_f ? fd : &none);
    setup_field(c, &c->g, c->has_g ? gd : &none);
    if (!c->has_f) c->f.update = 0;
    if (!c->has_g) c->g.update = 0;
    return c;
}

void ref_destroy(ref_case* c) {
    if (!c) return;
    rows_free(c->f.value, c->n); rows_free(c->f.swap, c->n);
    rows_free(c->g.value, c->n); rows_free(c->g.swap, c->n);
    free(c->f.scalarSource); free(c->g.scalarSource);
    rows_free(c->mf.U, c->n); rows_free(c->mf.Fi, c->n); rows_free(c->mf.Ft, c->n);
    free(c->mf.rho); free(c->mf.T); free(c->mf.p);
    free(c);
}

static void put_rows(double** r, const double* src, uint32_t n, int m) {
    for (uint32_t i = 0; i < n; i++)
        for (int j = 0; j < m; j++) r[i][j] = src[(size_t)i * m + j];
}

static void get_rows(double* dst, double** r, uint32_t n, int m) {
    for (uint32_t i = 0; i < n; i++)
        for (int j = 0; j < m; j++) dst[(size_t)i * m + j] = r[i][j];
}

int ref_upload(ref_case* c, const double* rho, const double* U, const double* T,
               const double* f, const double* g, const double* S,
               const double* Fi, const double* Ft) {
    if (rho) memcpy(c->mf.rho, rho, c->n * sizeof(double));
    if (T) memcpy(c->mf.T, T, c->n * sizeof(double));
    if (U) put_rows(c->mf.U, U, c->n, 3);
    if (Fi) put_rows(c->mf.Fi, Fi, c->n, 3);
    if (Ft) put_rows(c->mf.Ft, Ft, c->n, 3);
    if (f) put_rows(c->f.value, f, c->n, c->Q);
    if (g) put_rows(c->g.value, g, c->n, c->Q);
    if (S) memcpy(c->g.scalarSource, S, c->n * sizeof(double));
    return 0;
}

int ref_download(ref_case* c, double* rho, double* U, double* T, double* Fi, double* Ft,
                 double* S, double* f, double* g) {
    if (rho) memcpy(rho, c->mf.rho, c->n * sizeof(double));
    if (T) memcpy(T, c->mf.T, c->n * sizeof(double));
    if (U) get_rows(U, c->mf.U, c->n, 3);
    if (Fi) get_rows(Fi, c->mf.Fi, c->n, 3);
    if (Ft) get_rows(Ft, c->mf.Ft, c->n, 3);
    if (f) get_rows(f, c->f.value, c->n, c->Q);
    if (g) get_rows(g, c->g.value, c->n, c->Q);
    if (S) memcpy(S, c->g.scalarSource, c->n * sizeof(double));
    return 0;
}

void ref_set_time(ref_case* c, uint32_t t) { c->mesh.time.current = t; }
void ref_set_rank(ref_case* c, int32_t pid) { c->mesh.parallel.pid = pid; }
uint32_t ref_get_time(ref_case* c) { return c->mesh.time.current; }

/* Owner rank per node from the reference partitioner's default method
 * (applications/mesh/latticeMeshPartition/standardDecomp.c), which reads only
 * the node count.  The caller keeps 1 <= np <= n. */
void standardDecomp(uint* owner, basicMesh* mesh, uint np);
void ref_standard_decomp(uint32_t n, uint32_t np, uint32_t* owner) {
    basicMesh m;
    memset(&m, 0, sizeof(m));
    m.nPoints = n;
    standardDecomp((uint*)owner, &m, np);
}
void ref_set_rho0(ref_case* c, double r) { c->mesh.EOS.rho_0 = r; }
double ref_average_rho0(ref_case* c) {
    c->mesh.EOS.rho_0 = averageScalarField(&c->mesh, c->mf.rho);
    return c->mesh.EOS.rho_0;
}

/* Start-up block of the solver (multiPhasePP.c:122-147). */
int ref_initialize(ref_case* c) {
    equilibrium(&c->mesh, &c->mf, &c->f);
    equilibrium(&c->mesh, &c->mf, &c->g);
    interForce(&c->mesh, &c->mf);
    heatSource(&c->mesh, &c->mf, &c->g);
    return 0;
}

/* One pass of the time loop body (multiPhasePP.c:157-240), writes excluded.
 * The --frozen / --nht switches act through the update flags exactly as
 * mp.frozen / mp.ht do in the solver. */
int ref_step(ref_case* c, uint32_t nsteps) {
    latticeMesh* m = &c->mesh;
    for (uint32_t s = 0; s < nsteps; s++) {
        ++m->time.current;
        collision(m, &c->mf, &c->f);
        lbstream(m, &c->f);
        updateBoundaries(m, &c->mf, &c->f);
        collision(m, &c->mf, &c->g);
        lbstream(m, &c->g);
        updateBoundaries(m, &c->mf, &c->g);
        macroDensity(m, &c->mf, &c->f, 0, m->parallel.nlocal);
        macroDensity(m, &c->mf, &c->f, m->parallel.nlocal, m->mesh.nPoints);
        if (c->g.update != 0) heatSource(m, &c->mf, &c->g);
        macroTemperature(m, &c->mf, &c->g, 0, m->mesh.nPoints);
        if (c->f.update != 0) interForce(m, &c->mf);
        macroVelocity(m, &c->mf, &c->f, 0, m->mesh.nPoints);
    }
    return 0;
}

/* Single reference operators, for operator-level parity. */
enum { OP_EQUILIBRIUM = 0, OP_COLLISION, OP_LBSTREAM, OP_BOUNDARIES, OP_DENSITY,
       OP_VELOCITY, OP_TEMPERATURE, OP_INTERFORCE, OP_HEATSOURCE, OP_PRESSURE };

int ref_op(ref_case* c, int op, int field, uint32_t start, uint32_t end) {
    lbeField* fl = field == MPLB_FIELD_G ? &c->g : &c->f;
    latticeMesh* m = &c->mesh;
    switch (op) {
    case OP_EQUILIBRIUM: equilibrium(m, &c->mf, fl); break;
    case OP_COLLISION: collision(m, &c->mf, fl); break;
    case OP_LBSTREAM: lbstream(m, fl); break;
    case OP_BOUNDARIES: updateBoundaries(m, &c->mf, fl); break;
    case OP_DENSITY: macroDensity(m, &c->mf, &c->f, start, end); break;
    case OP_VELOCITY: macroVelocity(m, &c->mf, &c->f, start, end); break;
    case OP_TEMPERATURE: macroTemperature(m, &c->mf, &c->g, start, end); break;
    case OP_INTERFORCE: interForce(m, &c->mf); break;
    case OP_HEATSOURCE: heatSource(m, &c->mf, &c->g); break;
    case OP_PRESSURE: macroPressure(m, &c->mf, &c->f); break;  /* multiPhasePP.c:264 */
    default: return -1;
    }
    return 0;
}

/* Pressure field (macroFields.p), filled by OP_PRESSURE. */
void ref_get_p(ref_case* c, double* p) { memcpy(p, c->mf.p, c->n * sizeof(double)); }

/* The reference structures of a case, for the adapter check. */
void ref_structs(ref_case* c, latticeMesh** m, macroFields** mf, lbeField** f, lbeField** g) {
    *m = &c->mesh;
    *mf = &c->mf;
    *f = &c->f;
    *g = &c->g;
}

/* p_eos and potential as scalar functions, for EOS-level checks. */
double ref_p_eos(ref_case* c, double rho, double T) { return p_eos(&c->mesh.EOS, rho, T); }
double ref_potential(ref_case* c, double rho, double T) { return potential(&c->mesh, rho, T); }

/*
 * The reference's own field writers (src/IO/asciiRaw, binaryRaw, pvtu) on a
 * host array: format 0 asciiRaw, 1 binaryRaw, 2 pvtu (include/dataTypes.h:53);
 * scalar != 0 takes writeScalarTo*, else writeArrayTo* with vsize columns.
 * Files go to processor<pid>/<time>/ under the CURRENT folder, as in the
 * reference; pvtu appends to an existing fields.vtu there.  field is
 * [n][vsize] doubles.  Never called with a NaN (the reference's NaN check
 * lives in writeScalarField, which exits).
 */
int ref_write_field(int format, int scalar, const char* name, const double* field, uint32_t n, uint32_t vsize,
                    int pid, uint32_t time) {
    latticeMesh mesh;
    memset(&mesh, 0, sizeof mesh);
    mesh.mesh.nPoints = n;
    mesh.parallel.pid = pid;
    mesh.time.current = time;
    char nm[100];
    snprintf(nm, sizeof nm, "%s", name);
    if (scalar) {
        double* v = (double*)malloc((n ? n : 1) * sizeof(double));
        memcpy(v, field, n * sizeof(double));
        switch (format) {
        case 0: writeScalarToAsciiRaw(nm, v, &mesh); break;
        case 1: writeScalarToBinaryRaw(nm, v, &mesh); break;
        case 2: writeScalarToPvtu(nm, v, &mesh); break;
        default: free(v); return -1;
        }
        free(v);
        return 0;
    }
    double** r = rows_alloc(n, vsize);
    put_rows(r, field, n, (int)vsize);
    switch (format) {
    case 0: writeArrayToAsciiRaw(nm, r, &mesh, vsize); break;
    case 1: writeArrayToBinaryRaw(nm, r, &mesh, vsize); break;
    case 2: writeArrayToPvtu(nm, r, &mesh, vsize); break;
    default: rows_free(r, n); return -1;
    }
    rows_free(r, n);
    return 0;
}

/* ------------------------------------------------------------------------
 * Several ranks of a partitioned mesh, each a ref_case, run by the
 * reference's own exchange code (sendPdfField / recvPdfField,
 * syncScalarField, syncVectorField, and syncPdfField inside the
 * surface-tension collisions) with one thread per rank and the stub's
 * in-process messages.  The caller creates every rank's case from its own
 * nodes (owned first, then ghosts), then sets its place here. */

/* mpiInfo of rank `pid` of `world` as readLatticeMesh fills it
 * (readLatticeMesh.c:299-425): nrg[s] ghosts received from s, listed in recv
 * (peer by peer), nsg[s] owned nodes sent to s, listed in send, and the
 * buffers of the exchange; the fields' PDF buffers as createLbeField sizes
 * them. */
int ref_set_parallel(ref_case* c, uint32_t pid, uint32_t world, uint32_t nlocal, const uint32_t* nrg,
                     const uint32_t* recv, const uint32_t* nsg, const uint32_t* send) {
    if (world < 1 || pid >= world || nlocal > c->n) return -1;
    mpiInfo* P = &c->mesh.parallel;
    P->pid = pid;
    P->worldSize = world;
    P->nlocal = nlocal;
    P->nghosts = c->n - nlocal;
    free(P->nrg);
    free(P->nsg);
    P->nrg = (uint*)calloc(world, sizeof(uint));
    P->nsg = (uint*)calloc(world, sizeof(uint));
    P->recvGhosts = (uint**)calloc(world, sizeof(uint*));
    P->sendGhosts = (uint**)calloc(world, sizeof(uint*));
    P->sbuf = (scalar**)calloc(world, sizeof(scalar*));
    P->rbuf = (scalar**)calloc(world, sizeof(scalar*));
    P->vsbuf = (scalar**)calloc(world, sizeof(scalar*));
    P->vrbuf = (scalar**)calloc(world, sizeof(scalar*));
    lbeField* fl[2] = {&c->f, &c->g};
    for (int w = 0; w < 2; w++) {
        fl[w]->sbuf = (scalar**)calloc(world, sizeof(scalar*));
        fl[w]->rbuf = (scalar**)calloc(world, sizeof(scalar*));
        fl[w]->nreq = 0;
    }
    size_t ro = 0, so = 0;
    for (uint32_t s = 0; s < world; s++) {
        P->nrg[s] = nrg[s];
        P->nsg[s] = nsg[s];
        P->recvGhosts[s] = (uint*)malloc((nrg[s] ? nrg[s] : 1) * sizeof(uint));
        P->sendGhosts[s] = (uint*)malloc((nsg[s] ? nsg[s] : 1) * sizeof(uint));
        for (uint32_t i = 0; i < nrg[s]; i++) {
            if (recv[ro + i] < nlocal || recv[ro + i] >= c->n) return -2;  /* a ghost is not owned */
            P->recvGhosts[s][i] = recv[ro + i];
        }
        for (uint32_t i = 0; i < nsg[s]; i++) {
            if (send[so + i] >= nlocal) return -3;  /* only owned nodes are sent */
            P->sendGhosts[s][i] = send[so + i];
        }
        ro += nrg[s];
        so += nsg[s];
        size_t rq = (size_t)(nrg[s] ? nrg[s] : 1) * c->Q, sq = (size_t)(nsg[s] ? nsg[s] : 1) * c->Q;
        P->rbuf[s] = (scalar*)calloc(rq, sizeof(scalar));
        P->sbuf[s] = (scalar*)calloc(sq, sizeof(scalar));
        P->vrbuf[s] = (scalar*)calloc((size_t)(nrg[s] ? nrg[s] : 1) * 3, sizeof(scalar));
        P->vsbuf[s] = (scalar*)calloc((size_t)(nsg[s] ? nsg[s] : 1) * 3, sizeof(scalar));
        for (int w = 0; w < 2; w++) {
            fl[w]->rbuf[s] = (scalar*)calloc(rq, sizeof(scalar));
            fl[w]->sbuf[s] = (scalar*)calloc(sq, sizeof(scalar));
        }
    }
    return 0;
}

/* multiPhasePP.c:122-147 with the exchanges of a multi-rank run. */
static void rank_initialize(ref_case* c) {
    latticeMesh* m = &c->mesh;
    equilibrium(m, &c->mf, &c->f);
    equilibrium(m, &c->mf, &c->g);
    interForce(m, &c->mf);
    syncVectorField(m, c->mf.Fi);
    syncVectorField(m, c->mf.Ft);
    heatSource(m, &c->mf, &c->g);
    syncScalarField(m, c->g.scalarSource);
}

/* fixedRandomT seeds the C library's single rand() state with its rank's
 * pid at every application (fixedRandomT.c) and then draws from it.  Separate
 * processes each own that state; rank threads share it, so each thread's
 * boundary update runs alone, which gives every rank the draws it would get
 * in its own process.  updateBoundaries sends no message, so holding the
 * lock across it cannot stall another rank's exchange. */
static pthread_mutex_t boundary_mu = PTHREAD_MUTEX_INITIALIZER;

static void rank_boundaries(latticeMesh* m, macroFields* mf, lbeField* fl) {
    pthread_mutex_lock(&boundary_mu);
    updateBoundaries(m, mf, fl);
    pthread_mutex_unlock(&boundary_mu);
}

/* multiPhasePP.c:157-240 with its exchanges; the solver's --frozen / --nht
 * switches are the fields' update flags (multiPhasePP.c:106,116). */
static void rank_steps(ref_case* c, uint32_t nsteps) {
    latticeMesh* m = &c->mesh;
    for (uint32_t s = 0; s < nsteps; s++) {
        ++m->time.current;
        collision(m, &c->mf, &c->f);
        lbstream(m, &c->f);
        rank_boundaries(m, &c->mf, &c->f);
        if (c->f.update != 0) sendPdfField(m, &c->f);
        collision(m, &c->mf, &c->g);
        lbstream(m, &c->g);
        rank_boundaries(m, &c->mf, &c->g);
        if (c->g.update != 0) sendPdfField(m, &c->g);
        macroDensity(m, &c->mf, &c->f, 0, m->parallel.nlocal);
        if (c->f.update != 0) recvPdfField(m, &c->f);
        macroDensity(m, &c->mf, &c->f, m->parallel.nlocal, m->mesh.nPoints);
        if (c->g.update != 0) recvPdfField(m, &c->g);
        if (c->g.update != 0) {
            heatSource(m, &c->mf, &c->g);
            syncScalarField(m, c->g.scalarSource);
        }
        macroTemperature(m, &c->mf, &c->g, 0, m->mesh.nPoints);
        if (c->f.update != 0) {
            interForce(m, &c->mf);
            syncVectorField(m, c->mf.Fi);
            syncVectorField(m, c->mf.Ft);
        }
        macroVelocity(m, &c->mf, &c->f, 0, m->mesh.nPoints);
    }
}

enum { JOB_STEPS = 0, JOB_INIT = 1, JOB_AVERAGE_RHO0 = 2 };

typedef struct {
    ref_case* c;
    uint32_t nsteps;
    int kind;
    double result;
} rank_job;

static void* rank_thread(void* a) {
    rank_job* j = (rank_job*)a;
    mplb_stub_set_rank((int)j->c->mesh.parallel.pid);
    if (j->kind == JOB_INIT) rank_initialize(j->c);
    else if (j->kind == JOB_AVERAGE_RHO0) {
        /* the write step's buoyancy reference (multiPhasePP.c:271) */
        j->result = averageScalarField(&j->c->mesh, j->c->mf.rho);
        j->c->mesh.EOS.rho_0 = j->result;
    } else rank_steps(j->c, j->nsteps);
    return NULL;
}

static int ranks_run(ref_case** cases, uint32_t nranks, int kind, uint32_t nsteps, double* results);

/* Every rank's start-up (init != 0) or nsteps time steps, one thread per
 * rank; cases[r] is rank r.  0, or -1 when a message went missing. */
int ref_ranks_run(ref_case** cases, uint32_t nranks, int init, uint32_t nsteps) {
    return ranks_run(cases, nranks, init ? JOB_INIT : JOB_STEPS, nsteps, NULL);
}

/* averageScalarField of every rank's density, as the write step calls it
 * (local serial sums, MPI_Allreduce of the sums and of the node counts),
 * stored as each rank's rho_0; out[r] = rank r's result. */
int ref_ranks_average_rho0(ref_case** cases, uint32_t nranks, double* out) {
    return ranks_run(cases, nranks, JOB_AVERAGE_RHO0, 0, out);
}

static int ranks_run(ref_case** cases, uint32_t nranks, int kind, uint32_t nsteps, double* results) {
    for (uint32_t r = 0; r < nranks; r++)
        if (cases[r]->mesh.parallel.pid != r || cases[r]->mesh.parallel.worldSize != nranks) return -2;
    mplb_stub_reset();
    mplb_stub_set_world((int)nranks);
    pthread_t* th = (pthread_t*)calloc(nranks, sizeof(pthread_t));
    rank_job* jobs = (rank_job*)calloc(nranks, sizeof(rank_job));
    uint32_t started = 0;
    for (uint32_t r = 0; r < nranks; r++) {
        jobs[r].c = cases[r];
        jobs[r].nsteps = nsteps;
        jobs[r].kind = kind;
        if (pthread_create(&th[r], NULL, rank_thread, &jobs[r]) != 0) break;
        started++;
    }
    for (uint32_t r = 0; r < started; r++) pthread_join(th[r], NULL);
    if (results)
        for (uint32_t r = 0; r < started; r++) results[r] = jobs[r].result;
    free(th);
    free(jobs);
    mplb_stub_set_world(1);
    if (started != nranks) return -3;
    return mplb_stub_failures() ? -1 : 0;
}
