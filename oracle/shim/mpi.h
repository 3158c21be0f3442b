/*
 * Single-rank stand-in for the subset of MPI that pllcart3d.c and
 * pll_tridiag.c use (MPI-2 C bindings, MPICH2 1.1 era, Makefile:6,35 of the
 * reference).  Test infrastructure only: it lets the reference's own C code
 * be compiled in this container (which has no MPI) so that its output can pin
 * the CPU restatement in oracle/.  It is never linked into the GPU library.
 *
 * Semantics are those of MPI with one process:
 *   - MPI_PROC_NULL sends/receives complete at once and move no data;
 *   - a send to rank 0 (ourselves) is buffered and matched by tag at the
 *     receiver's MPI_Wait (velo_correction, pllcart3d.c:2188-2213);
 *   - collectives copy send to receive buffers (MPI_MAX over one value).
 */
#ifndef PLL_SHIM_MPI_H
#define PLL_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0x44000000
#define MPI_DOUBLE 0x4c00080b
#define MPI_MAX 0x58000001
#define MPI_PROC_NULL (-1)
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
double MPI_Wtime(void);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag,
             MPI_Comm comm, MPI_Status *st);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Isend(void *buf, int count, MPI_Datatype dt, int dst, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Allreduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt,
                  MPI_Op op, MPI_Comm comm);
int MPI_Reduce(void *sbuf, void *rbuf, int count, MPI_Datatype dt, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Gather(void *sbuf, int scount, MPI_Datatype sdt, void *rbuf,
               int rcount, MPI_Datatype rdt, int root, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);

#endif
