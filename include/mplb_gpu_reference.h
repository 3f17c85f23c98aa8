/*
 * mplb_gpu_reference.h -- adapter from the reference's host structures to
 * the C-ABI of mplb_gpu.h.  Header-only: it is compiled inside the reference
 * driver, after the reference's own headers, so this library never depends
 * on the layout of latticeMesh / macroFields / lbeField (which embed MPI
 * types whose size depends on the MPI implementation).
 *
 *   #include <latticeMesh.h>
 *   #include <macroFields.h>
 *   #include <lbeField.h>
 *   #include "mplb_gpu_reference.h"
 *
 * Requires the DP build (scalar == double, src/dataTypes/dataTypes.h:19-21).
 * A mesh is one rank's: the whole lattice at one rank (nPoints == nlocal),
 * or a rank of a partitioned mesh (nlocal owned nodes, then the ghosts, which
 * get no neighbours); mplb_ref_ghost_runs turns the ranks' ghost lists into
 * the exchange of mplb_ranks_step.  What it reads, with the reference
 * definitions it follows:
 *   mesh->mesh.nb, points, bd            basicMesh   (src/dataTypes/basicMesh.h:19-70)
 *   mesh->parallel.pid, worldSize,
 *   nlocal, nrg, recvGhosts, nsg,
 *   sendGhosts                           mpiInfo     (src/dataTypes/mpiInfo.h)
 *   mesh->EOS                            EOSInfo     (src/EOS/EOSInfo.h:80-102)
 *   field->model, lbparam, update,
 *   boundary[p].type / param             lbeField    (src/dataTypes/lbeField.h:32-108)
 *   mfields->rho, U, T, Fi, Ft           macroFields (src/dataTypes/macroFields.h:19-62)
 */
#ifndef MPLB_GPU_REFERENCE_H
#define MPLB_GPU_REFERENCE_H

#include <stdlib.h>
#include <string.h>

#include "mplb_gpu.h"

typedef struct mplb_ref_descs {
    mplb_mesh_desc mesh;
    mplb_eos_desc eos;
    mplb_field_desc field[2];
    int32_t* nb;
    int32_t* points;
    uint32_t* patch_count;
    uint32_t* patch_nodes;
    int32_t* bc_type[2];
    double* bc_value[2];
} mplb_ref_descs;

static inline void mplb_ref_free(mplb_ref_descs* d) {
    free(d->nb);
    free(d->points);
    free(d->patch_count);
    free(d->patch_nodes);
    for (int i = 0; i < 2; i++) {
        free(d->bc_type[i]);
        free(d->bc_value[i]);
    }
    memset(d, 0, sizeof(*d));
}

/* lbParameters union (src/lbEquation/lbParameters.h:16-31) -> field descriptor. */
static inline void mplb_ref_pack_field(const latticeMesh* mesh, const lbeField* fl, mplb_ref_descs* d, int which) {
    mplb_field_desc* fd = &d->field[which];
    uint32_t np = mesh->mesh.bd.nbd;
    const scalar* lam = NULL;
    memset(fd, 0, sizeof(*fd));
    if (!fl) {
        fd->model = MPLB_NO_MODEL;
        return;
    }
    fd->model = (int32_t)fl->model;
    fd->update = fl->update ? 1 : 0;
    switch (fl->model) {
    case liMRT:
        lam = fl->lbparam.liMRT.Lambda;
        fd->sigma = fl->lbparam.liMRT.sigma;
        fd->surface_tension = fl->lbparam.liMRT.surfaceTension != no_st;
        fd->kappa_st = fl->lbparam.liMRT.kappa_st;
        break;
    case xuMRT:
        lam = fl->lbparam.xuMRT.Lambda;
        fd->sigma = fl->lbparam.xuMRT.sigma;
        fd->surface_tension = fl->lbparam.xuMRT.surfaceTension != noXuSurf;
        fd->kappa_st = fl->lbparam.xuMRT.kappa_st;
        break;
    case liTempMRT:
        lam = fl->lbparam.liTempMRT.Lambda;
        break;
    case myMRT:
        lam = fl->lbparam.myMRT.Lambda;
        fd->alpha_1 = fl->lbparam.myMRT.alpha_1;
        fd->alpha_2 = fl->lbparam.myMRT.alpha_2;
        break;
    default:
        lam = fl->lbparam.myMRT.Lambda;
        break;
    }
    for (int k = 0; k < mesh->lattice.Q && k < MPLB_MAX_Q; k++) fd->Lambda[k] = lam ? lam[k] : 0.0;
    d->bc_type[which] = (int32_t*)calloc(np ? np : 1, sizeof(int32_t));
    d->bc_value[which] = (double*)calloc(3 * (np ? np : 1), sizeof(double));
    for (uint32_t p = 0; p < np; p++) {
        d->bc_type[which][p] = (int32_t)fl->boundary[p].type;
        if (fl->boundary[p].type == ft) d->bc_value[which][3 * p] = fl->boundary[p].param.ft.T;
        if (fl->boundary[p].type == fu)
            for (int j = 0; j < 3; j++) d->bc_value[which][3 * p + j] = fl->boundary[p].param.fu.U[j];
        if (fl->boundary[p].type == frdt) {
            d->bc_value[which][3 * p] = fl->boundary[p].param.frdt.T;
            d->bc_value[which][3 * p + 1] = fl->boundary[p].param.frdt.p;
            d->bc_value[which][3 * p + 2] =
                (double)fl->boundary[p].param.frdt.psteps - (double)fl->boundary[p].param.frdt.localTStep;
        }
    }
    fd->bc_type = d->bc_type[which];
    fd->bc_value = d->bc_value[which];
}

/* Pack the reference's structures into descriptors (no device work). */
static inline int mplb_ref_pack(const latticeMesh* mesh, const lbeField* f, const lbeField* g, mplb_ref_descs* d) {
    memset(d, 0, sizeof(*d));
    /* A rank of a partitioned mesh holds nlocal owned nodes, then its ghosts;
     * readLatticeMesh.c:135-160 reads neighbours for the owned nodes only. */
    if (mesh->parallel.worldSize < 1 || mesh->parallel.nlocal > mesh->mesh.nPoints ||
        (mesh->parallel.worldSize == 1 && mesh->parallel.nlocal != mesh->mesh.nPoints))
        return MPLB_E_UNSUPPORTED;
    uint32_t n = mesh->mesh.nPoints, nlocal = mesh->parallel.nlocal;
    int Q = mesh->lattice.Q;
    d->nb = (int32_t*)malloc((size_t)n * Q * sizeof(int32_t));
    d->points = (int32_t*)malloc((size_t)n * 3 * sizeof(int32_t));
    if (!d->nb || !d->points) { mplb_ref_free(d); return MPLB_E_ARG; }
    for (uint32_t i = 0; i < n; i++) {
        for (int k = 0; k < Q; k++) d->nb[(size_t)i * Q + k] = i < nlocal ? mesh->mesh.nb[i][k] : -1;
        for (int j = 0; j < 3; j++) d->points[(size_t)i * 3 + j] = mesh->mesh.points[i][j];
    }
    uint32_t np = mesh->mesh.bd.nbd, tot = 0;
    d->patch_count = (uint32_t*)calloc(np ? np : 1, sizeof(uint32_t));
    for (uint32_t p = 0; p < np; p++) tot += (d->patch_count[p] = mesh->mesh.bd.nbdelem[p]);
    d->patch_nodes = (uint32_t*)malloc((tot ? tot : 1) * sizeof(uint32_t));
    for (uint32_t p = 0, o = 0; p < np; p++)
        for (uint32_t i = 0; i < d->patch_count[p]; i++) d->patch_nodes[o++] = mesh->mesh.bd.bdPoints[p][i];
    d->mesh.lattice = mesh->lattice.model == D3Q15 ? MPLB_D3Q15 : MPLB_D2Q9;
    d->mesh.n_points = n;
    d->mesh.nb = d->nb;
    d->mesh.points = d->points;
    d->mesh.n_patches = np;
    d->mesh.patch_count = d->patch_count;
    d->mesh.patch_nodes = d->patch_nodes;

    const EOSInfo* e = &mesh->EOS;
    d->eos.type = (int32_t)e->etype;
    switch (e->etype) {
    case CarStar: d->eos.a = e->eParam.csp.a; d->eos.b = e->eParam.csp.b; break;
    case PengRob: d->eos.a = e->eParam.prp.a; d->eos.b = e->eParam.prp.b; d->eos.w = e->eParam.prp.omega; break;
    case VdW: d->eos.a = e->eParam.vdwparam.a; d->eos.b = e->eParam.vdwparam.b; break;
    default: break;
    }
    d->eos.R = e->R;
    d->eos.G = e->G;
    d->eos.M = e->M;
    d->eos.Cv = e->Cv;
    d->eos.rho_0 = e->rho_0;
    for (int j = 0; j < 3; j++) {
        d->eos.g[j] = e->g ? e->g[j] : 0.0;
        d->eos.fext[j] = e->fext ? e->fext[j] : 0.0;
    }
    mplb_ref_pack_field(mesh, f, d, 0);
    mplb_ref_pack_field(mesh, g, d, 1);
    return 0;
}

/* Row arrays (matrixDoubleAlloc layout) <-> contiguous [n][m]. */
static inline double* mplb_ref_rows_to_flat(scalar** rows, uint32_t n, int m) {
    double* a = (double*)malloc((size_t)n * m * sizeof(double));
    if (!a) return NULL;
    for (uint32_t i = 0; i < n; i++) memcpy(a + (size_t)i * m, rows[i], m * sizeof(double));
    return a;
}
static inline void mplb_ref_flat_to_rows(const double* a, scalar** rows, uint32_t n, int m) {
    for (uint32_t i = 0; i < n; i++) memcpy(rows[i], a + (size_t)i * m, m * sizeof(double));
}

/* Create a handle from the reference's state and upload rho, U, T, f, g,
 * scalarSource, Fi, Ft (those present).  The caller then runs
 * mplb_gpu_initialize (or not, when resuming an already initialised state). */
static inline int mplb_ref_create(const latticeMesh* mesh, const macroFields* mf, const lbeField* f,
                                  const lbeField* g, const mplb_opts* opts, mplb_gpu_t** out) {
    mplb_ref_descs d;
    int rc = mplb_ref_pack(mesh, f, g, &d);
    if (rc) return rc;
    mplb_opts o;
    if (opts) o = *opts;
    else {
        memset(&o, 0, sizeof(o));
        o.device = -1;
        o.start_time = mesh->time.current;
    }
    o.rank = mesh->parallel.pid;  /* fixedRandomT seeds rand() with it */
    rc = mplb_gpu_create(&d.mesh, &d.eos, &d.field[0], &d.field[1], &o, out);
    if (rc == 0) {
        uint32_t n = mesh->mesh.nPoints;
        int Q = mesh->lattice.Q;
        double* U = mf->U ? mplb_ref_rows_to_flat(mf->U, n, 3) : NULL;
        double* Fi = mf->Fi ? mplb_ref_rows_to_flat(mf->Fi, n, 3) : NULL;
        double* Ft = mf->Ft ? mplb_ref_rows_to_flat(mf->Ft, n, 3) : NULL;
        double* fv = (f && f->value) ? mplb_ref_rows_to_flat(f->value, n, Q) : NULL;
        double* gv = (g && g->value) ? mplb_ref_rows_to_flat(g->value, n, Q) : NULL;
        rc = mplb_gpu_upload(*out, mf->rho, U, mf->T, fv, gv, g ? g->scalarSource : NULL, Fi, Ft);
        free(U); free(Fi); free(Ft); free(fv); free(gv);
        if (rc) { mplb_gpu_destroy(*out); *out = NULL; }
    }
    mplb_ref_free(&d);
    return rc;
}

/* Device state -> the reference's host structures (write steps). */
static inline int mplb_ref_download(mplb_gpu_t* h, const latticeMesh* mesh, macroFields* mf, lbeField* f, lbeField* g) {
    uint32_t n = mesh->mesh.nPoints;
    int Q = mesh->lattice.Q;
    double* U = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* Fi = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* Ft = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* fv = (double*)malloc((size_t)n * Q * sizeof(double));
    double* gv = (double*)malloc((size_t)n * Q * sizeof(double));
    int rc = (U && Fi && Ft && fv && gv) ? 0 : MPLB_E_ARG;
    if (!rc) rc = mplb_gpu_download(h, mf->rho, U, mf->T, Fi, Ft, g ? g->scalarSource : NULL, fv, gv);
    if (!rc) {
        if (mf->U) mplb_ref_flat_to_rows(U, mf->U, n, 3);
        if (mf->Fi) mplb_ref_flat_to_rows(Fi, mf->Fi, n, 3);
        if (mf->Ft) mplb_ref_flat_to_rows(Ft, mf->Ft, n, 3);
        if (f && f->value) mplb_ref_flat_to_rows(fv, f->value, n, Q);
        if (g && g->value) mplb_ref_flat_to_rows(gv, g->value, n, Q);
    }
    free(U); free(Fi); free(Ft); free(fv); free(gv);
    return rc;
}

/* The ghost exchange of nranks ranks driven from one process
 * (mplb_ranks_initialize / mplb_ranks_step), from their partitioned meshes:
 * meshes[r] is rank r's mesh (readLatticeMesh(r)).  The i-th node of rank r's
 * recvGhosts[s] is filled from the i-th node of rank s's sendGhosts[r], the
 * pairing of the reference's exchange (sendPdfField.c:23-35 packs
 * sendGhosts[pid] in order, recvPdfField.c:29-41 unpacks into
 * recvGhosts[pid] in order).  Nodes that step by one on both sides merge
 * into one run.  *runs is malloc'd (release it with free()).  Returns
 * MPLB_E_ARG when a rank's pid or world size disagrees with its place in
 * meshes[], or when rank r receives a different number of ghosts from s
 * than s sends to r. */
static inline int mplb_ref_ghost_runs(const latticeMesh* const* meshes, uint32_t nranks, mplb_ghost_run** runs,
                                      uint32_t* nruns) {
    *runs = NULL;
    *nruns = 0;
    uint32_t cap = 0;
    for (uint32_t r = 0; r < nranks; r++)
        if (meshes[r]->parallel.pid != r || meshes[r]->parallel.worldSize != nranks) return MPLB_E_ARG;
    for (uint32_t r = 0; r < nranks; r++) {
        const mpiInfo* pr = &meshes[r]->parallel;
        for (uint32_t s = 0; s < nranks; s++) {
            const mpiInfo* ps = &meshes[s]->parallel;
            if (pr->nrg[s] != ps->nsg[r]) {
                free(*runs);
                *runs = NULL;
                *nruns = 0;
                return MPLB_E_ARG;
            }
            for (uint32_t i = 0; i < pr->nrg[s]; i++) {
                uint32_t d0 = pr->recvGhosts[s][i], s0 = ps->sendGhosts[r][i];
                mplb_ghost_run* last = (i > 0) ? &(*runs)[*nruns - 1] : NULL;
                if (last && last->dst_start + last->count == d0 && last->src_start + last->count == s0) {
                    last->count++;
                    continue;
                }
                if (*nruns == cap) {
                    cap = 2 * cap + 16;
                    mplb_ghost_run* grown = (mplb_ghost_run*)realloc(*runs, cap * sizeof(mplb_ghost_run));
                    if (!grown) {
                        free(*runs);
                        *runs = NULL;
                        *nruns = 0;
                        return MPLB_E_ARG;
                    }
                    *runs = grown;
                }
                mplb_ghost_run run = {r, d0, s, s0, 1};
                (*runs)[(*nruns)++] = run;
            }
        }
    }
    return 0;
}

/* The write step's buoyancy reference across nranks ranks driven from one
 * process (multiPhasePP.c:271), as averageScalarField computes it
 * (src/basic/averageScalarField.c): 0 when the configured rho_0 is <= 0,
 * else each rank's serial sum of rho over its nlocal owned nodes, the sums
 * and counts combined as its MPI_Allreduce combines them (here in rank
 * order; with two ranks every order gives the same bits), and the division.
 * meshes[r] and mf[r] are rank r's, with rho downloaded (mplb_ref_download). */
static inline double mplb_ref_average_rho0(const latticeMesh* const* meshes, const macroFields* const* mf,
                                           uint32_t nranks) {
    if (nranks == 0 || meshes[0]->EOS.rho_0 <= 0) return 0.0;
    double total = 0.0;
    uint32_t count = 0;
    for (uint32_t r = 0; r < nranks; r++) {
        double local = 0.0;
        for (uint32_t i = 0; i < meshes[r]->parallel.nlocal; i++) local += mf[r]->rho[i];
        total = r ? total + local : local;
        count += meshes[r]->parallel.nlocal;
    }
    return total / count;
}

#endif /* MPLB_GPU_REFERENCE_H */
