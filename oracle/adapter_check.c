/*
 * adapter_check.c -- exercises include/mplb_gpu_reference.h on the
 * reference's own structures.  TEST INFRASTRUCTURE ONLY.
 *
 * Built by oracle/Makefile (target `adapter`) against the reference's headers
 * and linked with oracle/_ref/libmplb_ref.so (the harness that builds the
 * reference structs in memory) and the GPU library.
 *
 *   adapter_pack_check  packs a reference case and compares the descriptors
 *                       with the structures field by field (no GPU needed)
 *   adapter_gpu_run     the drop-in loop: reference structs -> GPU handle ->
 *                       nsteps on the GPU -> results written back into the
 *                       same reference structs
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <latticeMesh.h>
#include <macroFields.h>
#include <lbeField.h>

#include "../include/mplb_gpu_reference.h"

typedef struct ref_case ref_case;
void ref_structs(ref_case* c, latticeMesh** m, macroFields** mf, lbeField** f, lbeField** g);

/* 0 when every packed value equals its source in the reference structures. */
int adapter_pack_check(ref_case* c) {
    latticeMesh* m;
    macroFields* mf;
    lbeField *f, *g;
    ref_structs(c, &m, &mf, &f, &g);
    mplb_ref_descs d;
    int rc = mplb_ref_pack(m, f, g, &d);
    if (rc) return 100 + (-rc);
    int bad = 0;
    uint32_t n = m->mesh.nPoints;
    if (d.mesh.n_points != n || d.mesh.lattice != (m->lattice.model == D3Q15 ? MPLB_D3Q15 : MPLB_D2Q9)) bad |= 1;
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < m->lattice.Q; k++)
            if (d.nb[(size_t)i * m->lattice.Q + k] != m->mesh.nb[i][k]) bad |= 2;
    uint32_t o = 0;
    if (d.mesh.n_patches != m->mesh.bd.nbd) bad |= 4;
    for (uint32_t p = 0; p < m->mesh.bd.nbd; p++)
        for (uint32_t i = 0; i < m->mesh.bd.nbdelem[p]; i++)
            if (d.patch_nodes[o++] != m->mesh.bd.bdPoints[p][i]) bad |= 8;
    if (d.eos.type != (int)m->EOS.etype || d.eos.R != m->EOS.R || d.eos.G != m->EOS.G || d.eos.rho_0 != m->EOS.rho_0) bad |= 16;
    for (int j = 0; j < 3; j++)
        if (d.eos.g[j] != m->EOS.g[j] || d.eos.fext[j] != m->EOS.fext[j]) bad |= 32;
    lbeField* fl[2] = {f, g};
    for (int w = 0; w < 2; w++) {
        if (d.field[w].model != (int)fl[w]->model || d.field[w].update != (int)fl[w]->update) bad |= 64;
        for (uint32_t p = 0; p < m->mesh.bd.nbd; p++)
            if (d.field[w].bc_type[p] != (int)fl[w]->boundary[p].type) bad |= 128;
    }
    if (f->model == liMRT)
        for (int k = 0; k < 9; k++)
            if (d.field[0].Lambda[k] != f->lbparam.liMRT.Lambda[k]) bad |= 256;
    if (g->model == myMRT) {
        if (d.field[1].alpha_1 != g->lbparam.myMRT.alpha_1 || d.field[1].alpha_2 != g->lbparam.myMRT.alpha_2) bad |= 512;
        for (int k = 0; k < m->lattice.Q; k++)
            if (d.field[1].Lambda[k] != g->lbparam.myMRT.Lambda[k]) bad |= 512;
    }
    for (int w = 0; w < 2; w++)
        for (uint32_t p = 0; p < m->mesh.bd.nbd; p++)
            if (fl[w]->boundary[p].type == frdt &&
                (d.field[w].bc_value[3 * p] != fl[w]->boundary[p].param.frdt.T ||
                 d.field[w].bc_value[3 * p + 1] != fl[w]->boundary[p].param.frdt.p ||
                 d.field[w].bc_value[3 * p + 2] != (double)(fl[w]->boundary[p].param.frdt.psteps -
                                                            fl[w]->boundary[p].param.frdt.localTStep)))
                bad |= 1024;
    mplb_ref_free(&d);
    return bad;
}

/* The drop-in loop on the reference structures.  Returns 0 or the error code. */
int adapter_gpu_run(ref_case* c, uint32_t nsteps, int path, uint32_t start_time) {
    latticeMesh* m;
    macroFields* mf;
    lbeField *f, *g;
    ref_structs(c, &m, &mf, &f, &g);
    mplb_opts o;
    memset(&o, 0, sizeof(o));
    o.precision = MPLB_FP64;
    o.path = path;
    o.device = -1;
    o.start_time = start_time;
    mplb_gpu_t* h = NULL;
    int rc = mplb_ref_create(m, mf, f, g, &o, &h);
    if (rc) {
        fprintf(stderr, "create: %s\n", mplb_gpu_last_error());
        return rc;
    }
    rc = mplb_gpu_step(h, nsteps);
    if (!rc) rc = mplb_ref_download(h, m, mf, f, g);
    if (rc) fprintf(stderr, "run: %s\n", mplb_gpu_last_error());
    mplb_gpu_destroy(h);
    return rc;
}

/* One rank of a partitioned mesh packed by mplb_ref_pack: the reference case's
 * lattice, EOS and fields with the rank's own nodes (npts = nlocal owned +
 * ghosts; nb_owned holds the owned nodes' neighbours, as readLatticeMesh reads
 * them) and no patches.  0 when the descriptor holds the owned neighbours,
 * no neighbours for the ghosts and every point; 1000 + code when the pack
 * refuses. */
int adapter_pack_part_check(ref_case* c, uint32_t npts, uint32_t nlocal, const int32_t* nb_owned,
                            const int32_t* points, uint32_t pid, uint32_t world) {
    latticeMesh* m;
    macroFields* mf;
    lbeField *f, *g;
    ref_structs(c, &m, &mf, &f, &g);
    const int Q = m->lattice.Q;
    latticeMesh lm = *m;
    int** nbrows = (int**)malloc((nlocal ? nlocal : 1) * sizeof(int*));
    int** ptrows = (int**)malloc((npts ? npts : 1) * sizeof(int*));
    for (uint32_t i = 0; i < nlocal; i++) nbrows[i] = (int*)(nb_owned + (size_t)i * Q);
    for (uint32_t i = 0; i < npts; i++) ptrows[i] = (int*)(points + (size_t)i * 3);
    lm.mesh.nPoints = npts;
    lm.mesh.nb = nbrows;
    lm.mesh.points = ptrows;
    lm.mesh.bd.nbd = 0;
    lm.parallel.pid = pid;
    lm.parallel.worldSize = world;
    lm.parallel.nlocal = nlocal;
    lm.parallel.nghosts = npts - nlocal;
    mplb_ref_descs d;
    int rc = mplb_ref_pack(&lm, f, g, &d);
    int bad = 0;
    if (rc) bad = 1000 + (-rc);
    else {
        if (d.mesh.n_points != npts || d.mesh.n_patches != 0) bad |= 1;
        for (uint32_t i = 0; i < npts; i++) {
            for (int k = 0; k < Q; k++)
                if (d.nb[(size_t)i * Q + k] != (i < nlocal ? nb_owned[(size_t)i * Q + k] : -1)) bad |= 2;
            for (int j = 0; j < 3; j++)
                if (d.points[(size_t)i * 3 + j] != points[(size_t)i * 3 + j]) bad |= 4;
        }
        mplb_ref_free(&d);
    }
    free(nbrows);
    free(ptrows);
    return bad;
}

/* mplb_ref_ghost_runs over nranks meshes that carry only their mpiInfo:
 * nrg[r * nranks + s] ghosts of rank r come from rank s, listed in recv (rank
 * major, peer minor); nsg and send likewise.  pid_of[r] is rank r's pid.
 * The runs (dst, dst_start, src, src_start, count) go to out, at most cap. */
int adapter_ghost_runs(uint32_t nranks, const uint32_t* pid_of, const uint32_t* nrg, const uint32_t* recv,
                       const uint32_t* nsg, const uint32_t* send, uint32_t* out, uint32_t cap, uint32_t* nout) {
    latticeMesh* ms = (latticeMesh*)calloc(nranks, sizeof(latticeMesh));
    const latticeMesh** mp = (const latticeMesh**)malloc(nranks * sizeof(latticeMesh*));
    uint** rg = (uint**)malloc((size_t)nranks * nranks * sizeof(uint*));
    uint** sg = (uint**)malloc((size_t)nranks * nranks * sizeof(uint*));
    size_t ro = 0, so = 0;
    for (uint32_t r = 0; r < nranks; r++) {
        mpiInfo* p = &ms[r].parallel;
        p->pid = pid_of[r];
        p->worldSize = nranks;
        p->nrg = (uint*)(nrg + (size_t)r * nranks);
        p->nsg = (uint*)(nsg + (size_t)r * nranks);
        p->recvGhosts = rg + (size_t)r * nranks;
        p->sendGhosts = sg + (size_t)r * nranks;
        for (uint32_t s = 0; s < nranks; s++) {
            p->recvGhosts[s] = (uint*)(recv + ro);
            p->sendGhosts[s] = (uint*)(send + so);
            ro += nrg[(size_t)r * nranks + s];
            so += nsg[(size_t)r * nranks + s];
        }
        mp[r] = &ms[r];
    }
    mplb_ghost_run* runs = NULL;
    uint32_t nruns = 0;
    int rc = mplb_ref_ghost_runs(mp, nranks, &runs, &nruns);
    *nout = nruns;
    for (uint32_t i = 0; i < nruns && i < cap; i++) {
        out[5 * i] = runs[i].dst;
        out[5 * i + 1] = runs[i].dst_start;
        out[5 * i + 2] = runs[i].src;
        out[5 * i + 3] = runs[i].src_start;
        out[5 * i + 4] = runs[i].count;
    }
    free(runs);
    free(rg);
    free(sg);
    free(mp);
    free(ms);
    return rc;
}

/* mplb_ref_ghost_runs and mplb_ref_pack on the harness's ranks (reference
 * structures whose mpiInfo ref_set_parallel filled): the runs go to out as
 * in adapter_ghost_runs; every rank must pack, with its ghost rows carrying
 * no neighbours.  0, the ghost-runs error, or 2000 + the first rank that
 * does not pack as expected. */
int adapter_ghost_runs_of_ranks(ref_case** cs, uint32_t nranks, uint32_t* out, uint32_t cap, uint32_t* nout) {
    const latticeMesh** mp = (const latticeMesh**)malloc(nranks * sizeof(latticeMesh*));
    int bad = 0;
    for (uint32_t r = 0; r < nranks; r++) {
        latticeMesh* m;
        macroFields* mf;
        lbeField *f, *g;
        ref_structs(cs[r], &m, &mf, &f, &g);
        mp[r] = m;
        mplb_ref_descs d;
        if (!bad && mplb_ref_pack(m, f, g, &d) == 0) {
            const int Q = m->lattice.Q;
            for (uint32_t i = m->parallel.nlocal; i < m->mesh.nPoints; i++)
                for (int k = 0; k < Q; k++)
                    if (d.nb[(size_t)i * Q + k] != -1) bad = 2000 + (int)r;
            if (d.mesh.n_points != m->mesh.nPoints) bad = 2000 + (int)r;
            mplb_ref_free(&d);
        } else if (!bad) {
            bad = 2000 + (int)r;
        }
    }
    mplb_ghost_run* runs = NULL;
    uint32_t nruns = 0;
    int rc = mplb_ref_ghost_runs(mp, nranks, &runs, &nruns);
    *nout = nruns;
    for (uint32_t i = 0; i < nruns && i < cap; i++) {
        out[5 * i] = runs[i].dst;
        out[5 * i + 1] = runs[i].dst_start;
        out[5 * i + 2] = runs[i].src;
        out[5 * i + 3] = runs[i].src_start;
        out[5 * i + 4] = runs[i].count;
    }
    free(runs);
    free(mp);
    return rc ? rc : bad;
}

/* mplb_ref_average_rho0 on the harness's ranks (reference structures). */
double adapter_average_rho0_of_ranks(ref_case** cs, uint32_t nranks) {
    const latticeMesh** mp = (const latticeMesh**)malloc(nranks * sizeof(latticeMesh*));
    const macroFields** mfp = (const macroFields**)malloc(nranks * sizeof(macroFields*));
    for (uint32_t r = 0; r < nranks; r++) {
        latticeMesh* m;
        macroFields* mf;
        lbeField *f, *g;
        ref_structs(cs[r], &m, &mf, &f, &g);
        mp[r] = m;
        mfp[r] = mf;
    }
    double v = mplb_ref_average_rho0(mp, mfp, nranks);
    free(mp);
    free(mfp);
    return v;
}
