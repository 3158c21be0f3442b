/*
 * Single-rank MPI stand-in (see mpi.h).  Test infrastructure only.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SELFQ_MAX 64
#define REQ_MAX 256

typedef struct {
    int used;
    int tag;
    int count;
    double data[4];
} self_msg;

typedef struct {
    int used;
    int pending_recv;
    void *buf;
    int count;
    int tag;
} req_slot;

static self_msg selfq[SELFQ_MAX];
static req_slot reqs[REQ_MAX];

static void die(const char *what)
{
    fprintf(stderr, "minimpi: unsupported use: %s\n", what);
    abort();
}

static int new_req(void)
{
    int i;
    for (i = 1; i < REQ_MAX; i++) {
        if (!reqs[i].used) {
            memset(&reqs[i], 0, sizeof(reqs[i]));
            reqs[i].used = 1;
            return i;
        }
    }
    die("request table full");
    return 0;
}

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
    *rank = 0;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    (void)comm;
    *size = 1;
    return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag,
             MPI_Comm comm, MPI_Status *st)
{
    (void)buf; (void)count; (void)dt; (void)tag; (void)comm; (void)st;
    if (src == MPI_PROC_NULL) return MPI_SUCCESS;
    die("blocking receive with one rank");
    return 1;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag,
              MPI_Comm comm, MPI_Request *req)
{
    int r;
    (void)dt; (void)comm;
    *req = 0; /* completes at once: no slot needed */
    if (src != MPI_PROC_NULL) {
        if (src != 0) die("receive from a rank other than 0");
        r = new_req();
        reqs[r].pending_recv = 1;
        reqs[r].buf = buf;
        reqs[r].count = count;
        reqs[r].tag = tag;
        *req = r;
    }
    return MPI_SUCCESS;
}

int MPI_Isend(void *buf, int count, MPI_Datatype dt, int dst, int tag,
              MPI_Comm comm, MPI_Request *req)
{
    int i;
    (void)dt; (void)comm;
    *req = 0; /* buffered or null: complete at once */
    if (dst == MPI_PROC_NULL) return MPI_SUCCESS;
    if (dst != 0) die("send to a rank other than 0");
    if (count > 4) die("self message longer than 4 doubles");
    for (i = 0; i < SELFQ_MAX; i++) {
        if (!selfq[i].used) {
            selfq[i].used = 1;
            selfq[i].tag = tag;
            selfq[i].count = count;
            memcpy(selfq[i].data, buf, sizeof(double) * (size_t)count);
            return MPI_SUCCESS;
        }
    }
    die("self queue full");
    return 1;
}

int MPI_Wait(MPI_Request *req, MPI_Status *st)
{
    int r = *req, i;
    (void)st;
    if (r <= 0 || r >= REQ_MAX || !reqs[r].used) return MPI_SUCCESS;
    if (reqs[r].pending_recv) {
        for (i = 0; i < SELFQ_MAX; i++) {
            if (selfq[i].used && selfq[i].tag == reqs[r].tag) {
                memcpy(reqs[r].buf, selfq[i].data,
                       sizeof(double) * (size_t)reqs[r].count);
                selfq[i].used = 0;
                break;
            }
        }
        if (i == SELFQ_MAX) die("wait on a receive with no matching send");
    }
    reqs[r].used = 0;
    return MPI_SUCCESS;
}

int MPI_Allreduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt,
                  MPI_Op op, MPI_Comm comm)
{
    (void)dt; (void)op; (void)comm;
    memcpy(rbuf, sbuf, sizeof(double) * (size_t)count);
    return MPI_SUCCESS;
}

int MPI_Reduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op,
               int root, MPI_Comm comm)
{
    (void)dt; (void)op; (void)root; (void)comm;
    memcpy(rbuf, sbuf, sizeof(double) * (size_t)count);
    return MPI_SUCCESS;
}

int MPI_Gather(void *sbuf, int scount, MPI_Datatype sdt, void *rbuf,
               int rcount, MPI_Datatype rdt, int root, MPI_Comm comm)
{
    (void)sdt; (void)rcount; (void)rdt; (void)root; (void)comm;
    memcpy(rbuf, sbuf, sizeof(double) * (size_t)scount);
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)dt; (void)root; (void)comm;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    return MPI_SUCCESS;
}
