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
