/*
 * Multi-process stand-in for the subset of MPI that pllcart3d.c and
 * pll_tridiag.c use (same interface as mpi.h / minimpi.c), for timing the
 * reference's own slab decomposition on the host cores.  Test and
 * measurement infrastructure only: never linked into the GPU library.
 *
 * The ranks are processes forked from one parent (shm_mpi_launch), sharing
 * one anonymous shared mapping:
 *   - point to point: one FIFO byte ring per directed pair that the
 *     reference uses (rank r to r+1, r+1 to r, and 0 to Size-1 for the
 *     inflow flux of velo_correction, pllcart3d.c:2188-2195, which is a
 *     message to itself on one rank); sends copy
 *     eagerly into the ring (blocking only while it is full), receives take
 *     the ring's head, whose tag must be the one asked for (every pair's
 *     messages are received in the order they were sent in this code);
 *   - collectives (Allreduce/Reduce with MPI_MAX, Gather, Bcast, Barrier)
 *     through per-rank slots and a sense-reversing barrier.
 * Waits spin and yield; every wait is bounded (~10 minutes), after which
 * the rank reports the stuck call and exits, so a mismatch cannot hang a
 * measurement.
 */
#include "mpi.h"

#include <sched.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define COLL_DOUBLES 65536
#define REQ_MAX 256
#define SPIN_LIMIT_S 600.0

typedef struct {
    volatile long head;   /* bytes consumed */
    volatile long tail;   /* bytes produced */
    char pad[48];
    char data[];          /* g_ring_bytes */
} ring_t;

/* ring capacity, set at launch: at least three of the largest messages a
 * rank sends before the receiver takes the first (a neighbour pair sends to
 * each other eagerly before either receives) */
static long g_ring_bytes = 16L << 20;
#define RING_BYTES g_ring_bytes
static size_t ring_stride(void) { return (sizeof(ring_t) + (size_t)g_ring_bytes + 4095) & ~(size_t)4095; }

typedef struct {
    int size;
    volatile int count;
    volatile int sense;
    volatile int failed;
    char pad[48];
    double coll[]; /* size * COLL_DOUBLES, then the rings */
} world_t;

static world_t *W;
static int g_rank = 0, g_size = 1;

typedef struct {
    int used, is_recv, src, tag, count;
    void *buf;
} req_t;
static req_t reqs[REQ_MAX];

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

static void die(const char *what)
{
    fprintf(stderr, "shmmpi rank %d: %s\n", g_rank, what);
    if (W) W->failed = 1;
    _exit(3);
}

static double g_spin_limit = SPIN_LIMIT_S;

static void spin_wait(double t0, const char *what)
{
    if (W->failed) die("another rank failed");
    if (now_s() - t0 > g_spin_limit) die(what);
    sched_yield();
}

static int n_rings(int size) { return 2 * (size - 1) + 1; }

/* ring of the directed pair (src, dst), or -1 when the pair is not one
 * the reference communicates over */
static int ring_index(int src, int dst)
{
    if (dst == src + 1) return 2 * src;
    if (dst == src - 1) return 2 * dst + 1;
    if (src == 0 && dst == g_size - 1) return 2 * (g_size - 1);
    return -1;
}

static ring_t *ring_at(int idx)
{
    char *base = (char *)W->coll + sizeof(double) * (size_t)g_size * COLL_DOUBLES;
    return (ring_t *)(base + (size_t)idx * ring_stride());
}

size_t shm_mpi_bytes(int size)
{
    return sizeof(world_t) + sizeof(double) * (size_t)size * COLL_DOUBLES + (size_t)n_rings(size) * ring_stride();
}

static void ring_put(ring_t *r, const void *p, long n)
{
    long off = 0;
    double t0 = now_s();
    while (off < n) {
        long room = RING_BYTES - (r->tail - r->head);
        long pos = r->tail % RING_BYTES;
        long chunk = n - off;
        if (chunk > room) chunk = room;
        if (chunk > RING_BYTES - pos) chunk = RING_BYTES - pos;
        if (chunk <= 0) {
            spin_wait(t0, "send: ring full for too long");
            continue;
        }
        memcpy(r->data + pos, (const char *)p + off, (size_t)chunk);
        __sync_synchronize();
        r->tail += chunk;
        off += chunk;
    }
}

static void ring_get(ring_t *r, void *p, long n)
{
    long off = 0;
    double t0 = now_s();
    while (off < n) {
        long avail = r->tail - r->head;
        long pos = r->head % RING_BYTES;
        long chunk = n - off;
        if (chunk > avail) chunk = avail;
        if (chunk > RING_BYTES - pos) chunk = RING_BYTES - pos;
        if (chunk <= 0) {
            spin_wait(t0, "receive: no message for too long");
            continue;
        }
        __sync_synchronize();
        memcpy((char *)p + off, r->data + pos, (size_t)chunk);
        __sync_synchronize();
        r->head += chunk;
        off += chunk;
    }
}

static void send_msg(const void *buf, int count, int dst, int tag)
{
    int idx, hdr[2];
    if (dst == MPI_PROC_NULL) return;
    idx = ring_index(g_rank, dst);
    if (idx < 0) die("send to a rank the reference never sends to");
    hdr[0] = tag;
    hdr[1] = count;
    ring_put(ring_at(idx), hdr, sizeof(hdr));
    ring_put(ring_at(idx), buf, (long)sizeof(double) * count);
}

static void recv_msg(void *buf, int count, int src, int tag)
{
    int idx, hdr[2];
    if (src == MPI_PROC_NULL) return;
    idx = ring_index(src, g_rank);
    if (idx < 0) die("receive from a rank the reference never receives from");
    ring_get(ring_at(idx), hdr, sizeof(hdr));
    if (hdr[0] != tag || hdr[1] != count) die("message out of order (tag or size)");
    ring_get(ring_at(idx), buf, (long)sizeof(double) * count);
}

static int new_req(void)
{
    int i;
    for (i = 1; i < REQ_MAX; i++)
        if (!reqs[i].used) {
            memset(&reqs[i], 0, sizeof(reqs[i]));
            reqs[i].used = 1;
            return i;
        }
    die("request table full");
    return 0;
}

static int g_sense = 0;   /* this rank's sense of the barrier in progress */

static void barrier(void)
{
    double t0 = now_s();
    g_sense = !g_sense;
    if (__sync_add_and_fetch(&W->count, 1) == g_size) {
        W->count = 0;
        __sync_synchronize();
        W->sense = g_sense;
    } else {
        while (W->sense != g_sense) spin_wait(t0, "barrier: a rank did not arrive");
    }
    __sync_synchronize();
}

/* ---- set-up ---------------------------------------------------------------- */

/* Fork `size` ranks sharing one mapping (rings of ring_bytes each); each
 * runs body(rank, arg) and exits with its return value.  Returns 0 when
 * every rank exited 0. */
int shm_mpi_launch(int size, long ring_bytes, int (*body)(int rank, void *arg), void *arg)
{
    int r, bad = 0;
    pid_t *pid;
    size_t bytes;
    g_ring_bytes = ring_bytes > (1L << 20) ? ring_bytes : (1L << 20);
    g_size = size;
    bytes = shm_mpi_bytes(size);
    void *m = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (m == MAP_FAILED) return -1;
    memset(m, 0, sizeof(world_t));
    W = (world_t *)m;
    W->size = size;
    pid = (pid_t *)calloc((size_t)size, sizeof(pid_t));
    fflush(stdout);
    fflush(stderr);
    for (r = 0; r < size; r++) {
        pid[r] = fork();
        if (pid[r] == 0) {
            const char *lim = getenv("PLL_SHMMPI_TIMEOUT_S");
            if (lim && atof(lim) > 0) g_spin_limit = atof(lim);
            g_rank = r;
            g_size = size;
            _exit(body(r, arg));
        }
        if (pid[r] < 0) {
            bad = 1;
            W->failed = 1;
            break;
        }
    }
    for (r = 0; r < size; r++) {
        int st = 0;
        if (pid[r] <= 0) continue;
        if (waitpid(pid[r], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) {
            bad = 1;
            W->failed = 1;
        }
    }
    free(pid);
    munmap(m, bytes);
    W = NULL;
    return bad ? -1 : 0;
}

/* ---- the MPI subset ------------------------------------------------------ */

int MPI_Init(int *argc, char ***argv)
{
    (void)argc;
    (void)argv;
    return MPI_SUCCESS;
}

int MPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
    (void)comm;
    *rank = g_rank;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    (void)comm;
    *size = g_size;
    return MPI_SUCCESS;
}

double MPI_Wtime(void) { return now_s(); }

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Status *st)
{
    (void)dt;
    (void)comm;
    recv_msg(buf, count, src, tag);
    if (st) {
        st->MPI_SOURCE = src;
        st->MPI_TAG = tag;
        st->MPI_ERROR = 0;
    }
    return MPI_SUCCESS;
}

/* Requests that are complete when posted (eager sends, receives from
 * MPI_PROC_NULL) take no table slot: the reference does not wait on all of
 * them (e.g. the inflow-flux send of velo_correction) */
#define REQ_DONE (-1)

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req)
{
    int i;
    (void)dt;
    (void)comm;
    if (src == MPI_PROC_NULL) {
        *req = REQ_DONE;
        return MPI_SUCCESS;
    }
    i = new_req();
    reqs[i].is_recv = 1;
    reqs[i].buf = buf;
    reqs[i].count = count;
    reqs[i].src = src;
    reqs[i].tag = tag;
    *req = i;
    return MPI_SUCCESS;
}

int MPI_Isend(void *buf, int count, MPI_Datatype dt, int dst, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)dt;
    (void)comm;
    send_msg(buf, count, dst, tag);   /* eager: complete on return */
    *req = REQ_DONE;
    return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *st)
{
    int i = *req;
    if (i == REQ_DONE) {
        if (st) st->MPI_ERROR = 0;
        return MPI_SUCCESS;
    }
    if (i <= 0 || i >= REQ_MAX || !reqs[i].used) die("MPI_Wait on an unknown request");
    if (reqs[i].is_recv) recv_msg(reqs[i].buf, reqs[i].count, reqs[i].src, reqs[i].tag);
    if (st) {
        st->MPI_SOURCE = reqs[i].src;
        st->MPI_TAG = reqs[i].tag;
        st->MPI_ERROR = 0;
    }
    reqs[i].used = 0;
    return MPI_SUCCESS;
}

static double *slot(int r) { return W->coll + (size_t)r * COLL_DOUBLES; }

int MPI_Allreduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm)
{
    int r, k;
    double *out = (double *)rbuf;
    (void)dt;
    (void)comm;
    if (op != MPI_MAX || count > COLL_DOUBLES) die("unsupported MPI_Allreduce");
    memcpy(slot(g_rank), sbuf, sizeof(double) * count);
    barrier();
    for (k = 0; k < count; k++) {
        double m = slot(0)[k];
        for (r = 1; r < g_size; r++)
            if (slot(r)[k] > m) m = slot(r)[k];
        out[k] = m;
    }
    barrier();
    return MPI_SUCCESS;
}

int MPI_Reduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm)
{
    int r, k;
    (void)dt;
    (void)comm;
    if (op != MPI_MAX || count > COLL_DOUBLES) die("unsupported MPI_Reduce");
    memcpy(slot(g_rank), sbuf, sizeof(double) * count);
    barrier();
    if (g_rank == root) {
        double *out = (double *)rbuf;
        for (k = 0; k < count; k++) {
            double m = slot(0)[k];
            for (r = 1; r < g_size; r++)
                if (slot(r)[k] > m) m = slot(r)[k];
            out[k] = m;
        }
    }
    barrier();
    return MPI_SUCCESS;
}

int MPI_Gather(void *sbuf, int scount, MPI_Datatype sdt, void *rbuf, int rcount, MPI_Datatype rdt, int root,
               MPI_Comm comm)
{
    int r;
    (void)sdt;
    (void)rdt;
    (void)comm;
    if (scount != rcount || scount > COLL_DOUBLES) die("unsupported MPI_Gather");
    memcpy(slot(g_rank), sbuf, sizeof(double) * scount);
    barrier();
    if (g_rank == root)
        for (r = 0; r < g_size; r++) memcpy((double *)rbuf + (size_t)r * rcount, slot(r), sizeof(double) * rcount);
    barrier();
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm)
{
    (void)dt;
    (void)comm;
    if (count > COLL_DOUBLES) die("unsupported MPI_Bcast");
    if (g_rank == root) memcpy(slot(root), buf, sizeof(double) * count);
    barrier();
    if (g_rank != root) memcpy(buf, slot(root), sizeof(double) * count);
    barrier();
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    barrier();
    return MPI_SUCCESS;
}
