/*
 * mpi_stub.c -- in-process point-to-point messages for the MPI stand-in
 * (oracle/mpi_stub/mpi.h).  TEST INFRASTRUCTURE ONLY.
 *
 * The harness runs the ranks of a partitioned mesh as threads of one
 * process.  A send copies its buffer into a mailbox at once (MPI's buffered
 * mode; the reference reuses its send buffers only after MPI_Waitall, so
 * either mode gives the same data).  A receive is recorded in the calling
 * thread's table and filled in MPI_Waitall by the oldest message from its
 * source rank with its tag, as MPI's non-overtaking order fills it.  Each
 * wait gives up after MPLB_STUB_WAIT_S seconds, counts a failure and
 * returns non-zero, so a checker that loses a message ends with an error
 * instead of hanging.
 */
#include <errno.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mpi.h"

#define MPLB_STUB_WAIT_S 20
#define MPLB_STUB_MAX_RECV 1024

typedef struct msg {
    int src, dst, tag;
    size_t bytes;
    struct msg* next;
    unsigned char data[];
} msg;

static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t cv = PTHREAD_COND_INITIALIZER;
static msg* head = NULL;
static msg* tail = NULL;
static int failures = 0;

typedef struct {
    void* buf;
    size_t bytes;
    int src, tag, used;
} pending;

static __thread int my_rank = 0;
static __thread pending table[MPLB_STUB_MAX_RECV];

void mplb_stub_set_rank(int rank) { my_rank = rank; }

int mplb_stub_failures(void) {
    pthread_mutex_lock(&mu);
    int f = failures;
    pthread_mutex_unlock(&mu);
    return f;
}

void mplb_stub_reset(void) {
    pthread_mutex_lock(&mu);
    while (head) {
        msg* m = head;
        head = m->next;
        free(m);
    }
    tail = NULL;
    failures = 0;
    pthread_mutex_unlock(&mu);
}

int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* r) {
    (void)c;
    size_t bytes = (size_t)n * mplb_stub_size(t);
    msg* m = (msg*)malloc(sizeof(msg) + (bytes ? bytes : 1));
    if (!m) return 1;
    m->src = my_rank;
    m->dst = d;
    m->tag = tag;
    m->bytes = bytes;
    m->next = NULL;
    memcpy(m->data, b, bytes);
    pthread_mutex_lock(&mu);
    if (tail) tail->next = m;
    else head = m;
    tail = m;
    pthread_cond_broadcast(&cv);
    pthread_mutex_unlock(&mu);
    *r = 0;
    return 0;
}

int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* r) {
    (void)c;
    for (int i = 0; i < MPLB_STUB_MAX_RECV; i++) {
        if (!table[i].used) {
            table[i].buf = b;
            table[i].bytes = (size_t)n * mplb_stub_size(t);
            table[i].src = s;
            table[i].tag = tag;
            table[i].used = 1;
            *r = i + 1;
            return 0;
        }
    }
    *r = 0;
    pthread_mutex_lock(&mu);
    failures++;
    pthread_mutex_unlock(&mu);
    return 1;
}

/* Take the oldest message for this thread from `src` with `tag`; mu held. */
static msg* take(int src, int tag) {
    msg* prev = NULL;
    for (msg* m = head; m; prev = m, m = m->next) {
        if (m->dst == my_rank && m->src == src && m->tag == tag) {
            if (prev) prev->next = m->next;
            else head = m->next;
            if (tail == m) tail = prev;
            return m;
        }
    }
    return NULL;
}

/* MPI_Allreduce (MPI_SUM) over the rank threads: every rank leaves its
 * contribution, the last to arrive folds them in rank order
 * (((r0 + r1) + r2) + ...), and all leave with that result.  An MPI library
 * may fold in another order; with two ranks every order gives the same
 * bits. */
#define MPLB_STUB_MAX_RANKS 64
#define MPLB_STUB_MAX_ELEMS 8
static int world_size = 1;
static int ar_count = 0, ar_gen = 0;
static double ar_slot[MPLB_STUB_MAX_RANKS][MPLB_STUB_MAX_ELEMS];
static double ar_sum[MPLB_STUB_MAX_ELEMS];

void mplb_stub_set_world(int world) {
    pthread_mutex_lock(&mu);
    world_size = world < 1 ? 1 : world;
    ar_count = 0;
    pthread_mutex_unlock(&mu);
}

static double load_elem(const void* p, MPI_Datatype t, int i) {
    switch (t) {
    case MPI_INT: return (double)((const int*)p)[i];
    case MPI_FLOAT: return (double)((const float*)p)[i];
    default: return ((const double*)p)[i];
    }
}

static void store_elem(void* p, MPI_Datatype t, int i, double v) {
    switch (t) {
    case MPI_INT: ((int*)p)[i] = (int)v; break;
    case MPI_FLOAT: ((float*)p)[i] = (float)v; break;
    default: ((double*)p)[i] = v; break;
    }
}

int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op;
    (void)c;
    pthread_mutex_lock(&mu);
    int world = world_size;
    pthread_mutex_unlock(&mu);
    if (world <= 1) {
        memcpy(out, in, (size_t)n * mplb_stub_size(t));
        return 0;
    }
    if (n > MPLB_STUB_MAX_ELEMS || my_rank < 0 || my_rank >= world || world > MPLB_STUB_MAX_RANKS ||
        t == MPI_CHAR) {
        pthread_mutex_lock(&mu);
        failures++;
        pthread_mutex_unlock(&mu);
        return 1;
    }
    struct timespec deadline;
    clock_gettime(CLOCK_REALTIME, &deadline);
    deadline.tv_sec += MPLB_STUB_WAIT_S;
    pthread_mutex_lock(&mu);
    int gen = ar_gen;
    for (int i = 0; i < n; i++) ar_slot[my_rank][i] = load_elem(in, t, i);
    if (++ar_count == world) {
        for (int i = 0; i < n; i++) {
            /* the fold in the contribution's own type: ints sum exactly in a
             * double; floats are rounded back after every addition */
            double acc = ar_slot[0][i];
            for (int r = 1; r < world; r++) {
                acc += ar_slot[r][i];
                if (t == MPI_FLOAT) acc = (double)(float)acc;
            }
            ar_sum[i] = acc;
        }
        ar_count = 0;
        ar_gen++;
        pthread_cond_broadcast(&cv);
    } else {
        while (gen == ar_gen) {
            if (pthread_cond_timedwait(&cv, &mu, &deadline) == ETIMEDOUT) {
                failures++;
                pthread_mutex_unlock(&mu);
                return 1;
            }
        }
    }
    for (int i = 0; i < n; i++) store_elem(out, t, i, ar_sum[i]);
    pthread_mutex_unlock(&mu);
    return 0;
}

int MPI_Waitall(int n, MPI_Request* r, MPI_Status* st) {
    (void)st;
    int rc = 0;
    struct timespec deadline;
    clock_gettime(CLOCK_REALTIME, &deadline);
    deadline.tv_sec += MPLB_STUB_WAIT_S;
    pthread_mutex_lock(&mu);
    for (int i = 0; i < n; i++) {
        if (r[i] <= 0 || r[i] > MPLB_STUB_MAX_RECV) continue;  /* sends, or nothing posted */
        pending* p = &table[r[i] - 1];
        msg* m = NULL;
        while (!(m = take(p->src, p->tag))) {
            if (pthread_cond_timedwait(&cv, &mu, &deadline) == ETIMEDOUT) break;
        }
        if (m && m->bytes == p->bytes) memcpy(p->buf, m->data, m->bytes);
        else {
            failures++;
            rc = 1;
        }
        free(m);
        p->used = 0;
        r[i] = 0;
    }
    pthread_mutex_unlock(&mu);
    return rc;
}
