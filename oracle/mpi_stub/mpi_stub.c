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
