/*
 * mplb_oracle.c -- CPU restatement of multiphaseLB's lattice update.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared
 * against.  Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it (through oracle/oracle.py); the library never does.
 *
 * It restates, in plain C and flat [node][k] arrays, every function on the
 * reference's time-step path.  Each function names the reference file:line
 * it follows.  Floating-point expressions are written with the reference's
 * evaluation order (C left-to-right, no contraction: build with
 * -ffp-contract=off) so the results can be compared bit for bit with the
 * reference compiled from its own sources (oracle/_ref).
 *
 * Lattice tables are derived, not transcribed: velocities are the standard
 * D2Q9 / D3Q15 sets in the reference's order, the MRT matrix rows are the
 * usual moment polynomials evaluated on those velocities, and the inverse is
 * M^T diag(1/|row|^2) (the rows are orthogonal).  Every entry of that inverse
 * is a correctly rounded quotient of small integers, which equals the
 * reference's transcribed constants (e.g. c1/4 == 1/36 in binary64).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/mplb_gpu.h"

typedef struct orc {
    int lat, Q, D;
    uint32_t n;
    int32_t* nb;      /* [n][Q] */
    uint8_t* onb;     /* isOnBnd */
    uint32_t npatch;
    uint32_t* pcount;
    uint32_t* poff;
    uint32_t* pnodes;
    mplb_eos_desc eos;
    mplb_field_desc fd[2];
    int32_t* bct[2];
    double* bcv[2];
    int has[2];
    double *rho, *T, *U, *Fi, *Ft, *S, *p; /* U/Fi/Ft: [n][3] */
    double *pdf[2], *swap;             /* [n][Q] */
    uint32_t current;
    int32_t rank;                      /* parallel.pid (fixedRandomT's srand seed) */
    int64_t frdt_step[2][MPLB_MAX_PATCHES];  /* fixedRandomT localTStep per field and patch */
    /* lattice tables */
    int c[MPLB_MAX_Q][3];
    int rev[MPLB_MAX_Q];
    double w[MPLB_MAX_Q], ppw[MPLB_MAX_Q], M[MPLB_MAX_Q][MPLB_MAX_Q], Mi[MPLB_MAX_Q][MPLB_MAX_Q], cs2;
    int fd_a[3], fd_b[3];  /* finite-difference directions per axis */
} orc;

/* ------------------------------------------------------------ lattice tables */
static const int C9[9][3] = {{0,0,0},{1,0,0},{0,1,0},{-1,0,0},{0,-1,0},{1,1,0},{-1,1,0},{-1,-1,0},{1,-1,0}};
static const int C15[15][3] = {{0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1},
    {1,1,1},{-1,1,1},{1,-1,1},{-1,-1,1},{1,1,-1},{-1,1,-1},{1,-1,-1},{-1,-1,-1}};

/* Moment rows: D2Q9 Lallemand-Luo basis (D2Q9_MRT.c:20-108), D3Q15
 * d'Humieres basis (D3Q15_MRT.c), evaluated on the velocity set. */
static int moment_row(int lat, int r, const int* c) {
    int cx = c[0], cy = c[1], cz = c[2], c2 = cx * cx + cy * cy + cz * cz;
    if (lat == MPLB_D2Q9) {
        switch (r) {
        case 0: return 1;
        case 1: return -4 + 3 * c2;
        case 2: return (8 - 21 * c2 + 9 * c2 * c2) / 2;
        case 3: return cx;
        case 4: return (-5 + 3 * c2) * cx;
        case 5: return cy;
        case 6: return (-5 + 3 * c2) * cy;
        case 7: return cx * cx - cy * cy;
        default: return cx * cy;
        }
    }
    switch (r) {
    case 0: return 1;
    case 1: return c2 - 2;
    case 2: return (15 * c2 * c2 - 55 * c2 + 32) / 2;
    case 3: return cx;
    case 4: return (5 * c2 - 13) * cx / 2;
    case 5: return cy;
    case 6: return (5 * c2 - 13) * cy / 2;
    case 7: return cz;
    case 8: return (5 * c2 - 13) * cz / 2;
    case 9: return 3 * cx * cx - c2;
    case 10: return cy * cy - cz * cz;
    case 11: return cx * cy;
    case 12: return cy * cz;
    case 13: return cx * cz;
    default: return cx * cy * cz;
    }
}

static void tables(orc* o) {
    int Q = o->Q;
    const int (*C)[3] = o->lat == MPLB_D2Q9 ? C9 : C15;
    for (int k = 0; k < Q; k++)
        for (int j = 0; j < 3; j++) o->c[k][j] = C[k][j];
    for (int k = 0; k < Q; k++)
        for (int q = 0; q < Q; q++)
            if (C[q][0] == -C[k][0] && C[q][1] == -C[k][1] && C[q][2] == -C[k][2]) o->rev[k] = q;
    o->cs2 = 1.0 / 3.0;                                     /* D2Q9_cs2.c, D3Q15_cs2.c */
    for (int k = 0; k < Q; k++) {
        int c2 = C[k][0] * C[k][0] + C[k][1] * C[k][1] + C[k][2] * C[k][2];
        if (o->lat == MPLB_D2Q9) {                          /* D2Q9_omega.c, D2Q9_ppw.c */
            o->w[k] = c2 == 0 ? 4.0 / 9.0 : (c2 == 1 ? 1.0 / 9.0 : 1.0 / 36.0);
            o->ppw[k] = c2 == 0 ? 0.0 : (c2 == 1 ? 1.0 / 3 : 1.0 / 12);
        } else {                                            /* D3Q15_omega.c, D3Q15_ppw.c */
            o->w[k] = c2 == 0 ? 2.0 / 9.0 : (c2 == 1 ? 1.0 / 9.0 : 1.0 / 72.0);
            o->ppw[k] = c2 == 0 ? 0.0 : (c2 == 1 ? 1.0 / 3.0 : 1.0 / 24.0);
        }
    }
    for (int r = 0; r < Q; r++) {
        int norm = 0;
        for (int k = 0; k < Q; k++) {
            int m = moment_row(o->lat, r, C[k]);
            o->M[r][k] = (double)m;
            norm += m * m;
        }
        for (int k = 0; k < Q; k++) o->Mi[k][r] = o->M[r][k] / (double)norm;
    }
    /* Axis finite differences: a = direction whose pull source is x + e_d,
     * b = the one whose source is x - e_d (scalarGradient.c:22-23,62-63,108-109,...). */
    for (int d = 0; d < 3; d++) {
        o->fd_a[d] = o->fd_b[d] = -1;
        for (int k = 0; k < Q; k++) {
            int unit = 1;
            for (int j = 0; j < 3; j++) if (j != d && C[k][j] != 0) unit = 0;
            if (!unit) continue;
            if (C[k][d] == -1) o->fd_a[d] = k;
            if (C[k][d] == 1) o->fd_b[d] = k;
        }
    }
}

/* ---------------------------------------------------------------- arithmetic */
/* matVecMult.c:4-20: dense row sums, left to right, from 0. */
static void matvec(const orc* o, const double (*A)[MPLB_MAX_Q], const double* v, double* r) {
    for (int i = 0; i < o->Q; i++) {
        double s = 0;
        for (int j = 0; j < o->Q; j++) s += A[i][j] * v[j];
        r[i] = s;
    }
}

/* p_eos.c:7-64 */
static double p_eos(const mplb_eos_desc* e, double rho, double T) {
    double p = 0, al, be;
    switch (e->type) {
    case MPLB_EOS_IDEAL:
        p = rho * e->R * T;
        break;
    case MPLB_EOS_CS:
        al = e->b * rho / 4.0;
        be = 1 - al;
        p = rho * e->R * T * ((1 + al + al * al - al * al * al) / (be * be * be)) - e->a * rho * rho;
        break;
    case MPLB_EOS_PR:
        al = 0.170151343 * e->a / (e->b * e->R);
        be = (1 + (0.37464 + 1.5422 * e->w - 0.26992 * e->w * e->w) * (1 - sqrt(T / al)));
        p = rho * e->R * T / (1 - e->b * rho) - e->a * be * be * rho * rho / (1 + 2 * e->b * rho - e->b * rho * e->b * rho);
        break;
    case MPLB_EOS_VDW:
        p = rho * e->R * T / (e->M - rho * e->b) - e->a * rho * rho / (e->M * e->M);
        break;
    }
    return p;
}

/* potential.c:7-13 */
static double psi(const orc* o, double rho, double T) {
    return sqrt(2 * (p_eos(&o->eos, rho, T) - rho * o->cs2) / (o->eos.G));
}

/* liMRTEquilibrium.c:3-29 (xuMRTEquilibrium.c is the same formula) */
static void eq_flow(const orc* o, double rho, const double* v, double* f) {
    for (int k = 0; k < o->Q; k++) {
        double al = 0, be = 0;
        for (int j = 0; j < 3; j++) {
            al += o->c[k][j] * v[j];
            be += v[j] * v[j];
        }
        f[k] = rho * o->w[k] * (1 + al / o->cs2 + 0.5 * al * al / (o->cs2 * o->cs2) - 0.5 * be / o->cs2);
    }
}

/* liTempMRTEquilibrium.c:5-44 (D2Q9 only) */
static void eq_heat(const orc* o, double T, const double* U, double* g) {
    double n[MPLB_MAX_Q] = {0};
    n[0] = T;
    n[1] = -2.0 * T;
    n[2] = 2.0 * T;
    n[3] = T * U[0];
    n[4] = T * (-U[0]);
    n[5] = T * U[1];
    n[6] = T * (-U[1]);
    n[7] = 0;
    n[8] = 0;
    matvec(o, o->Mi, n, g);
}

/* myMRTEquilibrium.c:5-95: moments T, a1 T, a2 T, T U_x, T (-U_x), T U_y,
 * T (-U_y) [, T U_z, -(T U_z)], zeros; then M^-1. */
static void neq_my(const orc* o, double T, const double* U, double* n) {
    const mplb_field_desc* d = &o->fd[1];
    for (int k = 0; k < MPLB_MAX_Q; k++) n[k] = 0;
    n[0] = T;
    n[1] = d->alpha_1 * T;
    n[2] = d->alpha_2 * T;
    n[3] = T * U[0];
    n[4] = T * (-U[0]);
    n[5] = T * U[1];
    n[6] = T * (-U[1]);
    if (o->lat == MPLB_D3Q15) {
        n[7] = T * U[2];
        n[8] = -(T * U[2]);
    }
}

static void eq_my(const orc* o, double T, const double* U, double* g) {
    double n[MPLB_MAX_Q];
    neq_my(o, T, U, n);
    matvec(o, o->Mi, n, g);
}

/* ---------------------------------------------------------------- operators */
/* Surface-tension moments of one node: liMRTSurfaceTension.c:7-150 (D2Q9)
 * and xuMRTSurfaceTension.c:7-168 (D3Q15).  Q_ij = sum_k w_k (psi(x + c_k) -
 * psi(x)) c_ki c_kj with w the pseudopotential weights (lattice.weights is
 * ppWeights, setLatticeInfo.c:80; the neighbour is nb[id][rev k]), scaled by
 * 0.5 psi G kappa; C = 0 on a node with any missing neighbour.  D2Q9 fills
 * the whole 2x2 tensor, D3Q15 its upper triangle. */
static void surface_tension(const orc* o, uint32_t id, double* C) {
    for (int k = 0; k < o->Q; k++) C[k] = 0;
    int noneigh = 0;
    for (int k = 1; k < o->Q; k++)
        if (o->nb[(size_t)id * o->Q + k] == -1) noneigh++;
    if (noneigh) return;
    const int D = o->lat == MPLB_D2Q9 ? 2 : 3;
    double Qt[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double ps = psi(o, o->rho[id], o->T[id]);
    for (int k = 1; k < o->Q; k++) {
        int nid = o->nb[(size_t)id * o->Q + o->rev[k]];
        double alpha = o->ppw[k] * (psi(o, o->rho[nid], o->T[nid]) - ps);
        for (int i = 0; i < D; i++)
            for (int j = (D == 2 ? 0 : i); j < D; j++) Qt[i][j] += alpha * o->c[k][i] * o->c[k][j];
    }
    const double kap = o->fd[0].kappa_st;
    for (int i = 0; i < D; i++)
        for (int j = (D == 2 ? 0 : i); j < D; j++) Qt[i][j] = Qt[i][j] * 0.5 * ps * o->eos.G * kap;
    const double* L = o->fd[0].Lambda;
    if (D == 2) {
        C[1] = 1.5 * L[1] * (Qt[0][0] + Qt[1][1]);
        C[2] = -1.5 * L[2] * (Qt[0][0] + Qt[1][1]);
        C[7] = -L[8] * (Qt[0][0] - Qt[1][1]);
        C[8] = -L[8] * Qt[0][1];
    } else {
        C[1] = 4.0 * L[1] * (Qt[0][0] + Qt[1][1] + Qt[2][2]) / 5.0;
        C[9] = -L[10] * (2 * Qt[0][0] - Qt[1][1] - Qt[2][2]);
        C[10] = -L[10] * (Qt[1][1] - Qt[2][2]);
        C[11] = -L[10] * Qt[0][1];
        C[12] = -L[10] * Qt[1][2];
        C[13] = -L[10] * Qt[0][2];
    }
}

/* liMRTCollision.c:43-109 with liMRTForce.c:10-44 */
static void collide_limrt(orc* o) {
    const double* L = o->fd[0].Lambda;
    double sg = o->fd[0].sigma;
    for (uint32_t id = 0; id < o->n; id++) {
        const double* U = o->U + 3 * id;
        double rho = o->rho[id];
        double um = 0;
        for (int k = 0; k < 3; k++) um += U[k] * U[k];
        double meq[9], m[9], S[9];
        meq[0] = rho;
        meq[1] = rho * (-2 + 3 * um);
        meq[2] = rho * (1 - 3 * um);
        meq[3] = rho * U[0];
        meq[4] = rho * (-U[0]);
        meq[5] = rho * U[1];
        meq[6] = rho * (-U[1]);
        meq[7] = rho * (U[0] * U[0] - U[1] * U[1]);
        meq[8] = rho * U[0] * U[1];
        double* f = o->pdf[0] + 9 * id;
        matvec(o, o->M, f, m);
        const double* F = o->Ft + 3 * id;
        const double* Fi = o->Fi + 3 * id;
        double ps = psi(o, rho, o->T[id]);
        S[0] = 0;
        S[1] = 6 * (U[0] * F[0] + U[1] * F[1]) + 12 * sg * (Fi[0] * Fi[0] + Fi[1] * Fi[1]) / (ps * ps * ((1 / L[1]) - 0.5));
        S[2] = -6 * (U[0] * F[0] + U[1] * F[1]) - 12 * sg * (Fi[0] * Fi[0] + Fi[1] * Fi[1]) / (ps * ps * ((1 / L[2]) - 0.5));
        S[3] = F[0];
        S[4] = -F[0];
        S[5] = F[1];
        S[6] = -F[1];
        S[7] = 2 * (U[0] * F[0] - U[1] * F[1]);
        S[8] = U[0] * F[1] + U[1] * F[0];
        double Cst[9];
        if (o->fd[0].surface_tension) surface_tension(o, id, Cst);
        for (int k = 0; k < 9; k++) {
            m[k] = m[k] - L[k] * (m[k] - meq[k]) + (1 - 0.5 * L[k]) * S[k];
            if (o->fd[0].surface_tension) m[k] = m[k] + Cst[k];
        }
        matvec(o, o->Mi, m, f);
    }
}

/* xuMRTCollision.c:42-92, xuMRTEquilibriumMS.c:8-55, xuMRTForce.c:9-71 */
static void collide_xumrt(orc* o) {
    const double* L = o->fd[0].Lambda;
    double sg = o->fd[0].sigma;
    for (uint32_t id = 0; id < o->n; id++) {
        double U[3] = {o->U[3 * id], o->U[3 * id + 1], o->U[3 * id + 2]};
        double rho = o->rho[id];
        double um = 0;
        for (int k = 0; k < 3; k++) um += U[k] * U[k];
        double meq[15], m[15], S[15], F[3];
        meq[0] = rho;
        meq[1] = rho * (-1.0 + um);
        meq[2] = rho * (1.0 - 5.0 * um);
        meq[3] = rho * U[0];
        meq[4] = rho * -7.0 * U[0] / 3.0;
        meq[5] = rho * U[1];
        meq[6] = rho * -7.0 * U[1] / 3.0;
        meq[7] = rho * U[2];
        meq[8] = rho * -7.0 * U[2] / 3.0;
        meq[9] = rho * (2.0 * U[0] * U[0] - U[1] * U[1] - U[2] * U[2]);
        meq[10] = rho * (U[1] * U[1] - U[2] * U[2]);
        meq[11] = rho * U[0] * U[1];
        meq[12] = rho * U[1] * U[2];
        meq[13] = rho * U[0] * U[2];
        meq[14] = 0;
        double* f = o->pdf[0] + 15 * id;
        matvec(o, o->M, f, m);
        for (int j = 0; j < 3; j++) F[j] = o->Fi[3 * id + j] + (rho - o->eos.rho_0) * o->eos.g[j];
        double ps = psi(o, rho, o->T[id]);
        double uf = U[0] * F[0] + U[1] * F[1] + U[2] * F[2];
        double f2 = 0;
        for (int k = 0; k < 3; k++) f2 += F[k] * F[k];
        S[0] = 0;
        S[1] = 2.0 * uf + (6.0 * sg * f2) / (ps * ps * ((1 / L[1]) - 0.5));
        S[2] = -10.0 * uf;
        S[3] = F[0];
        S[4] = -7.0 * F[0] / 3.0;
        S[5] = F[1];
        S[6] = -7.0 * F[1] / 3.0;
        S[7] = F[2];
        S[8] = -7.0 * F[2] / 3.0;
        S[9] = 4.0 * U[0] * F[0] - 2.0 * U[1] * F[1] - 2.0 * U[2] * F[2];
        S[10] = 2.0 * U[1] * F[1] - 2.0 * U[2] * F[2];
        S[11] = U[0] * F[1] + U[1] * F[0];
        S[12] = U[1] * F[2] + U[2] * F[1];
        S[13] = U[0] * F[2] + U[2] * F[0];
        S[14] = 0;
        double Cst[15];
        if (o->fd[0].surface_tension) surface_tension(o, id, Cst);
        for (int k = 0; k < 15; k++) {
            m[k] = m[k] - L[k] * (m[k] - meq[k]) + (1 - 0.5 * L[k]) * S[k];
            if (o->fd[0].surface_tension) m[k] = m[k] + Cst[k];
        }
        matvec(o, o->Mi, m, f);
    }
}

/* liTempMRTCollision.c:31-87, liTempMRTEquilibriumMS.c:20-41, liTempMRTSource.c:17-24 */
static void collide_litemp(orc* o) {
    const double* L = o->fd[1].Lambda;
    for (uint32_t id = 0; id < o->n; id++) {
        const double* U = o->U + 3 * id;
        double T = o->T[id];
        double neq[9], n[9], G[9];
        neq[0] = T;
        neq[1] = -2.0 * T;
        neq[2] = 2.0 * T;
        neq[3] = T * U[0];
        neq[4] = T * (-U[0]);
        neq[5] = T * U[1];
        neq[6] = T * (-U[1]);
        neq[7] = 0;
        neq[8] = 0;
        double* g = o->pdf[1] + 9 * id;
        matvec(o, o->M, g, n);
        for (int k = 0; k < 9; k++) G[k] = 0;
        G[0] = o->S[id];
        double n4 = n[4], n6 = n[6];
        for (int k = 0; k < 9; k++) n[k] = n[k] - L[k] * (n[k] - neq[k]) + G[k];
        n[3] = n[3] + (1 - L[3] / 2) * L[4] * n4;
        n[5] = n[5] + (1 - L[5] / 2) * L[6] * n6;
        matvec(o, o->Mi, n, g);
    }
}

/* sparseMatVecMult.c:4-28: diagonal products, then the listed pairs added. */
static void sparse_mv(int Q, const double (*A)[MPLB_MAX_Q], const double* v, double* r, const int (*nz)[2],
                      int nnz) {
    for (int i = 0; i < Q; i++) r[i] = A[i][i] * v[i];
    for (int i = 0; i < nnz; i++) r[nz[i][0]] = r[nz[i][0]] + A[nz[i][0]][nz[i][1]] * v[nz[i][1]];
}

/* myMRTCollision.c:8-260: Q = diag(Lambda) with Q[3][4], Q[5][6] (and
 * Q[7][8] on D3Q15) = Q[j+1][j+1] (Q[j][j]/2 - 1); n = M g; n <- n -
 * Q (n - n_eq) + (I - Q/2) Gamma with Gamma = (S, 0, ...); g = M^-1 n. */
static void collide_my(orc* o) {
    const double* L = o->fd[1].Lambda;
    const int Q = o->Q;
    static const int nz[3][2] = {{3, 4}, {5, 6}, {7, 8}};
    const int nnz = o->lat == MPLB_D2Q9 ? 2 : 3;
    double A[MPLB_MAX_Q][MPLB_MAX_Q], B[MPLB_MAX_Q][MPLB_MAX_Q];
    memset(A, 0, sizeof A);
    for (int k = 0; k < Q; k++) A[k][k] = L[k];
    for (int i = 0; i < nnz; i++) A[nz[i][0]][nz[i][1]] = A[nz[i][1]][nz[i][1]] * (A[nz[i][0]][nz[i][0]] / 2.0 - 1.0);
    for (int j = 0; j < Q; j++)
        for (int k = 0; k < Q; k++) {
            B[j][k] = -0.5 * A[j][k];
            if (j == k) B[j][k] = 1.0 + B[j][k];
        }
    for (uint32_t id = 0; id < o->n; id++) {
        double ne[MPLB_MAX_Q], n[MPLB_MAX_Q], G[MPLB_MAX_Q], a1[MPLB_MAX_Q], a2[MPLB_MAX_Q];
        neq_my(o, o->T[id], o->U + 3 * (size_t)id, ne);
        double* g = o->pdf[1] + (size_t)Q * id;
        matvec(o, o->M, g, n);
        for (int k = 0; k < Q; k++) G[k] = 0;
        G[0] = o->S[id];
        for (int k = 0; k < Q; k++) a2[k] = n[k] - ne[k];
        sparse_mv(Q, (const double (*)[MPLB_MAX_Q])A, a2, a1, nz, nnz);
        sparse_mv(Q, (const double (*)[MPLB_MAX_Q])B, G, a2, nz, nnz);
        for (int k = 0; k < Q; k++) n[k] = n[k] - a1[k] + a2[k];
        matvec(o, o->Mi, n, g);
    }
}

/* general/collision.c:6-67 */
static int op_collision(orc* o, int fi) {
    if (!o->fd[fi].update) return 0;
    switch (o->fd[fi].model) {
    case MPLB_LIMRT: if (fi != 0) return -1; collide_limrt(o); return 0;
    case MPLB_XUMRT: if (fi != 0) return -1; collide_xumrt(o); return 0;
    case MPLB_LITEMPMRT: if (fi != 1) return -1; collide_litemp(o); return 0;
    case MPLB_MYMRT: if (fi != 1) return -1; collide_my(o); return 0;
    default: return -1;
    }
}

/* general/lbstream.c:5-72: copy, pull where nb != -1, copy back. */
static void op_stream(orc* o, int fi) {
    if (!o->fd[fi].update) return;
    int Q = o->Q;
    double* v = o->pdf[fi];
    memcpy(o->swap, v, (size_t)o->n * Q * sizeof(double));
    for (uint32_t id = 0; id < o->n; id++)
        for (int k = 0; k < Q; k++) {
            int s = o->nb[(size_t)id * Q + k];
            if (s != -1) o->swap[(size_t)id * Q + k] = v[(size_t)s * Q + k];
        }
    memcpy(v, o->swap, (size_t)o->n * Q * sizeof(double));
}

/* boundary/bounceBack/bounceBack.c:7-77: in place, k ascending. */
static void bc_bounceback(orc* o, double* v, uint32_t p) {
    int Q = o->Q, nax = o->lat == MPLB_D2Q9 ? 4 : 6;
    for (uint32_t i = 0; i < o->pcount[p]; i++) {
        uint32_t id = o->pnodes[o->poff[p] + i];
        double* f = v + (size_t)id * Q;
        const int32_t* nb = o->nb + (size_t)id * Q;
        for (int k = 0; k < Q; k++) {
            if (nb[k] == -1) {
                f[k] = f[o->rev[k]];
            } else if (nb[o->rev[k]] != -1 && k >= 1 && k <= nax) {
                f[k] = 0.5 * f[k] + 0.5 * f[o->rev[k]];
                f[o->rev[k]] = f[k];
            }
        }
    }
}

/* boundary/fixedT/fixedT.c:15-142 with liTempMRTEquilibrium or myMRTEquilibrium. */
static void bc_fixedt(orc* o, double* v, uint32_t p, double Tw) {
    int Q = o->Q;
    double fn[MPLB_MAX_Q], fb[MPLB_MAX_Q];
    for (uint32_t i = 0; i < o->pcount[p]; i++) {
        uint32_t id = o->pnodes[o->poff[p] + i];
        const int32_t* nb = o->nb + (size_t)id * Q;
        for (int k = 0; k < Q; k++) {
            if (nb[k] != -1) continue;
            int nbid = nb[o->rev[k]];
            if (nbid == -1) continue;
            if (o->fd[1].model == MPLB_MYMRT) {
                eq_my(o, o->T[nbid], o->U + 3 * (size_t)nbid, fn);
                eq_my(o, Tw, o->U + 3 * (size_t)nbid, fb);
            } else {
                eq_heat(o, o->T[nbid], o->U + 3 * (size_t)nbid, fn);
                eq_heat(o, Tw, o->U + 3 * (size_t)nbid, fb);
            }
            double eq_nb = fn[k];
            double eq_bnd = fb[k];
            v[(size_t)id * Q + k] = eq_bnd + (v[(size_t)nbid * Q + k] - eq_nb);
        }
    }
}

/* boundary/fixedU/fixedU.c:7-143 (liMRT only). */
static void bc_fixedu(orc* o, double* v, uint32_t p, const double* Uw) {
    int Q = o->Q;
    double fn[MPLB_MAX_Q], fb[MPLB_MAX_Q];
    for (uint32_t i = 0; i < o->pcount[p]; i++) {
        uint32_t id = o->pnodes[o->poff[p] + i];
        const int32_t* nb = o->nb + (size_t)id * Q;
        for (int k = 0; k < Q; k++) {
            if (nb[k] != -1) continue;
            int nbid = nb[o->rev[k]];
            if (nbid == -1) continue;
            double lv[3] = {0, 0, 0}, nbrho = 0, F[3];
            const double* fv = v + (size_t)nbid * Q;
            for (int j = 0; j < 3; j++)
                F[j] = o->Fi[3 * (size_t)nbid + j] + (o->rho[nbid] - o->eos.rho_0) * o->eos.g[j];
            for (int j = 0; j < 3; j++)
                for (int q = 0; q < Q; q++) lv[j] += o->c[q][j] * fv[q];
            for (int q = 0; q < Q; q++) nbrho += fv[q];
            for (int j = 0; j < 3; j++) lv[j] = (lv[j] + F[j] * 0.5) / nbrho;
            eq_flow(o, nbrho, lv, fn);
            eq_flow(o, nbrho, Uw, fb);
            v[(size_t)id * Q + k] = fb[k] + (v[(size_t)nbid * Q + k] - fn[k]);
        }
    }
}

/* rand() of the GNU C library after srand(seed) (fixedRandomT.c:37,81),
 * restated from its published description (P. Selinger, "The GLIBC
 * pseudo-random number generator", 2007): r_0 = seed (0 -> 1), r_i = 16807
 * r_{i-1} mod (2^31 - 1) for i < 31, r_i = r_{i-31} for i = 31..33, then
 * r_i = r_{i-3} + r_{i-31} mod 2^32; the k-th output is r_{k+344} >> 1. */
typedef struct { uint32_t r[34]; uint64_t i; } gnu_rand;  /* the last 34 words, r_i at r[i % 34] */

static int gnu_rand_step(gnu_rand* g) {
    uint32_t v = g->r[(g->i - 31) % 34] + g->r[(g->i - 3) % 34];
    g->r[g->i % 34] = v;
    g->i++;
    return (int)(v >> 1);
}

static void gnu_srand(gnu_rand* g, uint32_t seed) {
    int64_t w = seed == 0 ? 1 : seed;
    g->r[0] = (uint32_t)w;
    for (int i = 1; i < 31; i++) {
        w = (16807 * w) % 2147483647;
        g->r[i] = (uint32_t)w;
    }
    for (int i = 31; i < 34; i++) g->r[i] = g->r[i - 31];
    g->i = 34;
    for (int i = 34; i < 344; i++) gnu_rand_step(g);
}

static int gnu_rand_next(gnu_rand* g) { return gnu_rand_step(g); }

/* boundary/fixedRandomT/fixedRandomT.c:15-125 (myMRT): while localTStep <
 * psteps the wall temperature of each (node, missing direction) is drawn
 * uniformly in T (1 -+ p/100), with srand(pid) at every call. */
static void bc_fixedrandomt(orc* o, double* v, uint32_t p, const double* bcv, int64_t* local_step) {
    int Q = o->Q;
    double fn[MPLB_MAX_Q], fb[MPLB_MAX_Q];
    static gnu_rand g;
    gnu_srand(&g, (uint32_t)o->rank);
    double T0 = bcv[0], pc = bcv[1];
    double minT = T0 * (100.0 - pc) / 100.0;
    double maxT = T0 * (100.0 + pc) / 100.0;
    int64_t psteps = (int64_t)bcv[2];
    for (uint32_t i = 0; i < o->pcount[p]; i++) {
        uint32_t id = o->pnodes[o->poff[p] + i];
        const int32_t* nb = o->nb + (size_t)id * Q;
        for (int k = 0; k < Q; k++) {
            if (nb[k] != -1) continue;
            int nbid = nb[o->rev[k]];
            if (nbid == -1) continue;
            eq_my(o, o->T[nbid], o->U + 3 * (size_t)nbid, fn);
            double eq_nb = fn[k];
            if (*local_step < psteps) {
                double r = (double)gnu_rand_next(&g) / 2147483647;
                double Tb = minT + (maxT - minT) * r;
                eq_my(o, Tb, o->U + 3 * (size_t)nbid, fb);
            } else {
                eq_my(o, T0, o->U + 3 * (size_t)nbid, fb);
            }
            v[(size_t)id * Q + k] = fb[k] + (v[(size_t)nbid * Q + k] - eq_nb);
        }
    }
    (*local_step)++;
}

/* boundary/outflow/outflow.c:12-208: the normal is the sum of the velocities
 * whose node x + c_k is missing, normalised in float; ln the last direction
 * equal to its (int) truncation; the unknown populations are advected from
 * the inner neighbour nb[id][ln] with its normal velocity (force-corrected,
 * from the previous step's Fi and rho). */
static int bc_outflow(orc* o, double* v, uint32_t p) {
    int Q = o->Q;
    for (uint32_t i = 0; i < o->pcount[p]; i++) {
        uint32_t id = o->pnodes[o->poff[p] + i];
        const int32_t* nb = o->nb + (size_t)id * Q;
        float normal[3] = {0, 0, 0};
        for (int k = 0; k < Q; k++)
            if (nb[o->rev[k]] == -1)
                for (int j = 0; j < 3; j++) normal[j] += o->c[k][j];
        float nmag = 0;
        for (int j = 0; j < 3; j++) nmag += normal[j] * normal[j];
        if (nmag == 0) return -1;
        nmag = sqrt(nmag);
        for (int j = 0; j < 3; j++) normal[j] = normal[j] / nmag;
        int ln = 0;
        for (int k = 0; k < Q; k++)
            if (o->c[k][0] == (int)normal[0] && o->c[k][1] == (int)normal[1] && o->c[k][2] == (int)normal[2]) ln = k;
        int m = nb[ln];
        if (m == -1) continue;
        const double* fm = v + (size_t)m * Q;
        double F[3], nbv[3] = {0, 0, 0}, nbrho = 0, uadv = 0;
        for (int j = 0; j < 3; j++)
            F[j] = o->Fi[3 * (size_t)m + j] + (o->rho[m] - o->eos.rho_0) * o->eos.g[j];
        for (int j = 0; j < 3; j++)
            for (int q = 0; q < Q; q++) nbv[j] += o->c[q][j] * fm[q];
        for (int q = 0; q < Q; q++) nbrho += fm[q];
        for (int j = 0; j < 3; j++) nbv[j] = (nbv[j] + F[j] * 0.5) / nbrho;
        for (int j = 0; j < 3; j++) uadv += normal[j] * nbv[j];
        for (int k = 0; k < Q; k++)
            if (nb[k] == -1) v[(size_t)id * Q + k] = (v[(size_t)id * Q + k] + uadv * fm[k]) / (1 + uadv);
    }
    return 0;
}

/* general/updateBoundaries.c:6-75: patches in file order. */
static int op_boundaries(orc* o, int fi) {
    if (!o->fd[fi].update) return 0;
    for (uint32_t p = 0; p < o->npatch; p++) {
        int t = o->bct[fi][p];
        switch (t) {
        case MPLB_BC_PERIODIC: break;
        case MPLB_BC_BOUNCEBACK: bc_bounceback(o, o->pdf[fi], p); break;
        case MPLB_BC_FIXEDT:
            if (fi != 1 || (o->fd[fi].model != MPLB_LITEMPMRT && o->fd[fi].model != MPLB_MYMRT)) return -1;
            bc_fixedt(o, o->pdf[fi], p, o->bcv[fi][3 * p]);
            break;
        case MPLB_BC_FIXEDRANDOMT:
            if (fi != 1 || o->fd[fi].model != MPLB_MYMRT) return -1;
            bc_fixedrandomt(o, o->pdf[fi], p, o->bcv[fi] + 3 * p, &o->frdt_step[fi][p]);
            break;
        case MPLB_BC_OUTFLOW:
            if (bc_outflow(o, o->pdf[fi], p)) return -1;
            break;
        case MPLB_BC_FIXEDU:
            if (o->fd[fi].model == MPLB_LIMRT) bc_fixedu(o, o->pdf[fi], p, o->bcv[fi] + 3 * p);
            break;
        default: return -1;
        }
    }
    return 0;
}

/* macroDensity.c:7-75, liMRTDensity.c:3-19 */
static void op_density(orc* o, uint32_t s, uint32_t e) {
    if (!o->fd[0].update) return;
    for (uint32_t id = s; id < e; id++) {
        double r = 0;
        for (int k = 0; k < o->Q; k++) r += o->pdf[0][(size_t)id * o->Q + k];
        o->rho[id] = r;
    }
}

/* macroVelocity.c:6-65, liMRTVelocity.c:6-55, xuMRTVelocity.c:6-55 */
static void op_velocity(orc* o, uint32_t s, uint32_t e) {
    if (!o->fd[0].update) return;
    for (uint32_t id = s; id < e; id++) {
        double F[3], lv[3] = {0, 0, 0};
        for (int j = 0; j < 3; j++)
            F[j] = o->fd[0].model == MPLB_XUMRT
                       ? o->Fi[3 * (size_t)id + j] + (o->rho[id] - o->eos.rho_0) * o->eos.g[j]
                       : o->Ft[3 * (size_t)id + j];
        const double* f = o->pdf[0] + (size_t)id * o->Q;
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < o->Q; k++) lv[j] += o->c[k][j] * f[k];
        for (int j = 0; j < 3; j++) lv[j] = (lv[j] + F[j] * 0.5) / o->rho[id];
        for (int j = 0; j < 3; j++) o->U[3 * (size_t)id + j] = lv[j];
    }
}

/* macroTemperature.c:7-68, liTempMRTTemperature.c:5-26, myMRTTemperature.c:5-37 */
static void op_temperature(orc* o, uint32_t s, uint32_t e) {
    if (!o->fd[1].update) return;
    for (uint32_t id = s; id < e; id++) {
        double T = 0;
        for (int k = 0; k < o->Q; k++) T += o->pdf[1][(size_t)id * o->Q + k];
        if (o->fd[1].model == MPLB_MYMRT) T = T + 0.5 * o->S[id];  /* myMRTTemperature.c:22-31 */
        o->T[id] = T;
    }
}

/* interForce.c:7-52 with interactionForce.c:8-84 */
static void op_interforce(orc* o) {
    int Q = o->Q;
    for (uint32_t id = 0; id < o->n; id++) {
        double F[3] = {0.0, 0.0, 0.0}, Ff[3] = {0, 0, 0};
        if (o->onb[id] == 0) {
            for (int k = 1; k < Q; k++) {
                int nbid = o->nb[(size_t)id * Q + o->rev[k]];
                double al = o->ppw[k] * psi(o, o->rho[nbid], o->T[nbid]);
                for (int i = 0; i < 3; i++) F[i] += al * (double)o->c[k][i];
            }
            double be = -o->eos.G * psi(o, o->rho[id], o->T[id]);
            for (int i = 0; i < 3; i++) Ff[i] = F[i] * be;
        }
        for (int j = 0; j < 3; j++) {
            o->Fi[3 * (size_t)id + j] = Ff[j];
            o->Ft[3 * (size_t)id + j] = Ff[j] + (o->rho[id] - o->eos.rho_0) * o->eos.g[j];
            if (o->onb[id] == 0) o->Ft[3 * (size_t)id + j] += o->eos.fext[j];
        }
    }
}

/* finiteDifference/scalarGradient.c, invScalarGradient.c, vectorDivergence.c:
 * central difference where both axis neighbours exist, one-sided otherwise. */
static double fd_diff(const orc* o, const double* fld, int stride, int comp, uint32_t id, int d,
                      int inv, int* present) {
    int a = o->nb[(size_t)id * o->Q + o->fd_a[d]];
    int b = o->nb[(size_t)id * o->Q + o->fd_b[d]];
#define VAL(i) (inv ? 1.0 / fld[(size_t)(i) * stride + comp] : fld[(size_t)(i) * stride + comp])
    *present = 1;
    if (a != -1 && b != -1) return 0.5 * (VAL(a) - VAL(b));
    if (a == -1 && b != -1) return VAL(id) - VAL(b);
    if (a != -1 && b == -1) return VAL(a) - VAL(id);
    *present = 0;
    return 0;
#undef VAL
}

/* general/heatSource.c:28-168 (myMRT and liTempMRT branches) */
static int op_heatsource(orc* o) {
    if (!o->fd[1].update) return 0;
    const int my = o->fd[1].model == MPLB_MYMRT;
    if (o->fd[1].model != MPLB_LITEMPMRT && !my) return -1;
    const double* L = o->fd[1].Lambda;
    const double a1 = o->fd[1].alpha_1, a2 = o->fd[1].alpha_2;
    double Cv = o->eos.Cv;
    int D = o->D;
    for (uint32_t id = 0; id < o->n; id++) {
        double lambda;
        if (!my) lambda = o->rho[id] * Cv * (1 / L[3] - 0.5);
        else if (o->lat == MPLB_D2Q9) lambda = o->rho[id] * Cv * (1 / L[3] - 0.5) * (4.0 + 3.0 * a1 + 2.0 * a2) / 6.0;
        else lambda = o->rho[id] * Cv * (1 / L[3] - 0.5) * (6.0 + 11.0 * a1 + a2) / 9.0;
        double gT[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, div = 0, dot = 0;
        int pr;
        for (int d = 0; d < D; d++) {
            gT[d] = fd_diff(o, o->T, 1, 0, id, d, 0, &pr);
            gR[d] = fd_diff(o, o->rho, 1, 0, id, d, 1, &pr);
            double dv = fd_diff(o, o->U, 3, d, id, d, 0, &pr);
            if (pr) div += dv;
        }
        for (int k = 0; k < 3; k++) dot += gT[k] * gR[k];
        double T = o->T[id], rho = o->rho[id];
        double dpdT = p_eos(&o->eos, rho, 1.1 * T) - p_eos(&o->eos, rho, 0.9 * T);
        dpdT = dpdT / (0.2 * T);
        double s = -lambda * dot / Cv + div * T * (1.0 - dpdT / (rho * Cv));
        if (my) {
            o->S[id] = s;
        } else {
            double old = o->current == 0 ? 0 : o->S[id];
            o->S[id] = s + 0.5 * (s - old);
        }
    }
    return 0;
}

/* liMRTPressure.c:6-253 (D2Q9): rho cs2 + G psi^2/2 + G psi lap(psi)/12
 * + 2 G^2 sigma |grad psi|^2, with one-sided second differences at a missing
 * neighbour; xuMRTPressure.c:6-22 (D3Q15) keeps rho cs2 + G psi^2/2. */
static double pressure_node(orc* o, uint32_t id) {
    const int Q = o->Q;
    double ps = psi(o, o->rho[id], o->T[id]);
    double p = o->rho[id] * o->cs2 + 0.5 * o->eos.G * ps * ps;
    if (o->lat != MPLB_D2Q9) return p;
#define PSI(i) psi(o, o->rho[i], o->T[i])
#define NB(i, k) o->nb[(size_t)(i) * Q + (k)]
    /* x term assigns lap, y term adds to it left to right:
     * lap = lap + psi_a + psi_b - 2 psi (liMRTPressure.c:27-110). */
    double lap = 0;
    for (int d = 0; d < 2; d++) {
        int ka = o->fd_a[d], kb = o->fd_b[d];
        int a = NB(id, ka), b = NB(id, kb);
        double s0 = d == 0 ? 0.0 : lap;
        if (a != -1 && b != -1) {
            lap = d == 0 ? PSI(a) + PSI(b) - 2 * PSI(id) : s0 + PSI(a) + PSI(b) - 2 * PSI(id);
        } else if (a == -1 && b != -1) {
            int c = NB(b, kb);
            lap = d == 0 ? PSI(c) - 2 * PSI(b) + PSI(id) : s0 + PSI(c) - 2 * PSI(b) + PSI(id);
        } else if (a != -1 && b == -1) {
            int c = NB(a, ka);
            lap = d == 0 ? PSI(c) - 2 * PSI(a) + PSI(id) : s0 + PSI(c) - 2 * PSI(a) + PSI(id);
        } else if (d == 0) {
            lap = 0;
        }
    }
    p = p + o->eos.G * ps * lap / 12;
    double grad[3] = {0, 0, 0};
    for (int d = 0; d < 2; d++) {
        int a = NB(id, o->fd_a[d]), b = NB(id, o->fd_b[d]);
        if (a != -1 && b != -1) grad[d] = 0.5 * (PSI(a) - PSI(b));
        else if (a == -1 && b != -1) grad[d] = (PSI(id) - PSI(b));
        else if (a != -1 && b == -1) grad[d] = (PSI(a) - PSI(id));
        else grad[d] = 0;
    }
#undef PSI
#undef NB
    double g2 = 0;
    for (int k = 0; k < 3; k++) g2 += grad[k] * grad[k];
    return p + 2.0 * o->eos.G * o->eos.G * o->fd[0].sigma * g2;
}

/* general/macroPressure.c:8-69 */
static int op_pressure(orc* o) {
    if (!o->fd[0].update) return 0;
    if (o->fd[0].model != MPLB_LIMRT && o->fd[0].model != MPLB_XUMRT) return -1;
    for (uint32_t id = 0; id < o->n; id++) o->p[id] = pressure_node(o, id);
    return 0;
}

/* general/equilibrium.c:6-90 */
static int op_equilibrium(orc* o, int fi) {
    if (!o->fd[fi].update) return 0;
    for (uint32_t id = 0; id < o->n; id++) {
        double* v = o->pdf[fi] + (size_t)id * o->Q;
        switch (o->fd[fi].model) {
        case MPLB_LIMRT:
        case MPLB_XUMRT: eq_flow(o, o->rho[id], o->U + 3 * (size_t)id, v); break;
        case MPLB_LITEMPMRT: if (o->lat != MPLB_D2Q9) return -1; eq_heat(o, o->T[id], o->U + 3 * (size_t)id, v); break;
        case MPLB_MYMRT: if (fi != 1) return -1; eq_my(o, o->T[id], o->U + 3 * (size_t)id, v); break;
        default: return -1;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ handle API */
orc* orc_create(const mplb_mesh_desc* md, const mplb_eos_desc* ed, const mplb_field_desc* fd,
                const mplb_field_desc* gd, uint32_t start_time) {
    orc* o = (orc*)calloc(1, sizeof(orc));
    o->lat = md->lattice;
    o->Q = o->lat == MPLB_D2Q9 ? 9 : 15;
    o->D = o->lat == MPLB_D2Q9 ? 2 : 3;
    o->n = md->n_points;
    tables(o);
    size_t nq = (size_t)o->n * o->Q;
    o->nb = (int32_t*)malloc(nq * sizeof(int32_t));
    memcpy(o->nb, md->nb, nq * sizeof(int32_t));
    o->onb = (uint8_t*)calloc(o->n, 1);
    for (uint32_t i = 0; i < o->n; i++)
        for (int k = 0; k < o->Q; k++) if (o->nb[(size_t)i * o->Q + k] == -1) o->onb[i] = 1;
    o->npatch = md->n_patches;
    o->pcount = (uint32_t*)calloc(o->npatch + 1, sizeof(uint32_t));
    o->poff = (uint32_t*)calloc(o->npatch + 1, sizeof(uint32_t));
    uint32_t tot = 0;
    for (uint32_t p = 0; p < o->npatch; p++) { o->pcount[p] = md->patch_count[p]; o->poff[p] = tot; tot += md->patch_count[p]; }
    o->pnodes = (uint32_t*)malloc((tot + 1) * sizeof(uint32_t));
    if (tot) memcpy(o->pnodes, md->patch_nodes, tot * sizeof(uint32_t));
    o->eos = *ed;
    const mplb_field_desc* src[2] = {fd, gd};
    for (int i = 0; i < 2; i++) {
        o->has[i] = src[i] && src[i]->model != MPLB_NO_MODEL;
        if (o->has[i]) o->fd[i] = *src[i];
        else { memset(&o->fd[i], 0, sizeof(o->fd[i])); o->fd[i].model = MPLB_NO_MODEL; }
        o->bct[i] = (int32_t*)calloc(o->npatch + 1, sizeof(int32_t));
        o->bcv[i] = (double*)calloc(3 * (o->npatch + 1), sizeof(double));
        for (uint32_t p = 0; p < o->npatch; p++) {
            o->bct[i][p] = o->has[i] && src[i]->bc_type ? src[i]->bc_type[p] : MPLB_BC_PERIODIC;
            for (int j = 0; j < 3; j++)
                o->bcv[i][3 * p + j] = o->has[i] && src[i]->bc_value ? src[i]->bc_value[3 * p + j] : 0.0;
        }
        o->pdf[i] = (double*)calloc(nq, sizeof(double));
    }
    o->swap = (double*)calloc(nq, sizeof(double));
    o->rho = (double*)calloc(o->n, sizeof(double));
    o->T = (double*)calloc(o->n, sizeof(double));
    o->S = (double*)calloc(o->n, sizeof(double));
    o->p = (double*)calloc(o->n, sizeof(double));
    o->U = (double*)calloc(3 * (size_t)o->n, sizeof(double));
    o->Fi = (double*)calloc(3 * (size_t)o->n, sizeof(double));
    o->Ft = (double*)calloc(3 * (size_t)o->n, sizeof(double));
    o->current = start_time;
    return o;
}

void orc_destroy(orc* o) {
    if (!o) return;
    free(o->nb); free(o->onb); free(o->pcount); free(o->poff); free(o->pnodes);
    for (int i = 0; i < 2; i++) { free(o->bct[i]); free(o->bcv[i]); free(o->pdf[i]); }
    free(o->swap); free(o->rho); free(o->T); free(o->S); free(o->p); free(o->U); free(o->Fi); free(o->Ft);
    free(o);
}

int orc_upload(orc* o, const double* rho, const double* U, const double* T, const double* f,
               const double* g, const double* S, const double* Fi, const double* Ft) {
    size_t n = o->n, nq = n * o->Q;
    if (rho) memcpy(o->rho, rho, n * sizeof(double));
    if (U) memcpy(o->U, U, 3 * n * sizeof(double));
    if (T) memcpy(o->T, T, n * sizeof(double));
    if (f) memcpy(o->pdf[0], f, nq * sizeof(double));
    if (g) memcpy(o->pdf[1], g, nq * sizeof(double));
    if (S) memcpy(o->S, S, n * sizeof(double));
    if (Fi) memcpy(o->Fi, Fi, 3 * n * sizeof(double));
    if (Ft) memcpy(o->Ft, Ft, 3 * n * sizeof(double));
    return 0;
}

int orc_download(orc* o, double* rho, double* U, double* T, double* Fi, double* Ft, double* S,
                 double* f, double* g) {
    size_t n = o->n, nq = n * o->Q;
    if (rho) memcpy(rho, o->rho, n * sizeof(double));
    if (U) memcpy(U, o->U, 3 * n * sizeof(double));
    if (T) memcpy(T, o->T, n * sizeof(double));
    if (Fi) memcpy(Fi, o->Fi, 3 * n * sizeof(double));
    if (Ft) memcpy(Ft, o->Ft, 3 * n * sizeof(double));
    if (S) memcpy(S, o->S, n * sizeof(double));
    if (f) memcpy(f, o->pdf[0], nq * sizeof(double));
    if (g) memcpy(g, o->pdf[1], nq * sizeof(double));
    return 0;
}

void orc_set_time(orc* o, uint32_t t) { o->current = t; }
void orc_set_rank(orc* o, int32_t pid) { o->rank = pid; }
uint32_t orc_get_time(orc* o) { return o->current; }
void orc_set_rho0(orc* o, double r) { o->eos.rho_0 = r; }

/* averageScalarField.c:4-78, one rank. */
double orc_average_rho0(orc* o) {
    double avg = 0;
    if (!(o->eos.rho_0 <= 0)) {
        double s = 0;
        for (uint32_t i = 0; i < o->n; i++) s += o->rho[i];
        avg = s / (int)o->n;
    }
    o->eos.rho_0 = avg;
    return avg;
}

/* multiPhasePP.c:122-147 */
int orc_initialize(orc* o) {
    if (op_equilibrium(o, 0) || op_equilibrium(o, 1)) return -1;
    op_interforce(o);
    return op_heatsource(o);
}

/* multiPhasePP.c:157-240, writes excluded. */
int orc_step(orc* o, uint32_t nsteps) {
    for (uint32_t s = 0; s < nsteps; s++) {
        ++o->current;
        if (op_collision(o, 0) && o->fd[0].update) return -1;
        op_stream(o, 0);
        if (op_boundaries(o, 0)) return -1;
        if (op_collision(o, 1) && o->fd[1].update) return -1;
        op_stream(o, 1);
        if (op_boundaries(o, 1)) return -1;
        op_density(o, 0, o->n);
        if (o->fd[1].update && op_heatsource(o)) return -1;
        op_temperature(o, 0, o->n);
        if (o->fd[0].update) op_interforce(o);
        op_velocity(o, 0, o->n);
    }
    return 0;
}

int orc_op(orc* o, int op, int field, uint32_t start, uint32_t end) {
    int fi = field == MPLB_FIELD_G ? 1 : 0;
    switch (op) {
    case 0: return op_equilibrium(o, fi);
    case 1: return op_collision(o, fi);
    case 2: op_stream(o, fi); return 0;
    case 3: return op_boundaries(o, fi);
    case 4: op_density(o, start, end); return 0;
    case 5: op_velocity(o, start, end); return 0;
    case 6: op_temperature(o, start, end); return 0;
    case 7: op_interforce(o); return 0;
    case 8: return op_heatsource(o);
    case 9: return op_pressure(o);
    default: return -1;
    }
}

void orc_get_p(orc* o, double* p) { memcpy(p, o->p, o->n * sizeof(double)); }
double orc_p_eos(orc* o, double rho, double T) { return p_eos(&o->eos, rho, T); }
double orc_potential(orc* o, double rho, double T) { return psi(o, rho, T); }
