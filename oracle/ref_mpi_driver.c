/*
 * The reference's own multi-rank time step (pllcart3d.c:158-195 on the
 * x-slab decomposition of grid_setup, pllcart3d.c:357-378, with its halo
 * exchanges and pll_tridiag's pipelined x solves), run as `ranks` processes
 * over the shared-memory MPI stand-in (shim/shmmpi.c) and timed.  Test and
 * measurement infrastructure only: it times the reference's CPU path on the
 * host cores; nothing of it reaches the GPU library.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

#include "mpi.h"

int shm_mpi_launch(int size, long ring_bytes, int (*body)(int rank, void *arg), void *arg);
int pllref_init_ranked(const char *rundir, int rank, int size);
int pllref_x_offset(void);
void pllref_dims(int *d);
int pllref_load_ic(const double *c, const double *u, const double *v, const double *w);
int pllref_steps(int n);
void pllref_set_fast_dct(int fast);
int pllref_get(const char *name, double *out);

typedef struct {
    const char *rundir;
    const double *c, *u, *v, *w;   /* the whole padded box, [x][y][z] */
    int warm, steps;
    double budget_s;               /* timed steps stop once this much time has passed (0: no limit) */
    double *out;                   /* shared: [0] timed seconds, [1] warm-up seconds, [2] set-up seconds,
                                      [3] timed steps run */
    double *c_all;                 /* shared, or NULL: c_new of the whole padded box after the steps */
} job_t;

static int rank_body(int rank, void *arg)
{
    job_t *J = (job_t *)arg;
    int size, d[6];
    long plane, off;
    double t0, t1, t2, t3;
    MPI_Comm_size(MPI_COMM_WORLD, &size);
    t0 = MPI_Wtime();
    if (pllref_init_ranked(J->rundir, rank, size) != 0) return 2;
    pllref_set_fast_dct(1);   /* FFT-speed DCT, as FFTW gives the reference */
    pllref_dims(d);
    plane = (long)d[1] * d[2];
    off = (long)pllref_x_offset() * plane;   /* this slab's first padded plane */
    if (pllref_load_ic(J->c + off, J->u + off, J->v + off, J->w + off) != 0) return 2;
    MPI_Barrier(MPI_COMM_WORLD);
    t1 = MPI_Wtime();
    pllref_steps(J->warm);
    MPI_Barrier(MPI_COMM_WORLD);
    t2 = MPI_Wtime();
    {
        int n;
        double go = 1.0;
        for (n = 0; n < J->steps && go > 0.0; ++n) {
            pllref_steps(1);
            /* rank 0 decides for all whether another step fits the budget */
            if (rank == 0) go = (J->budget_s <= 0.0 || MPI_Wtime() - t2 < J->budget_s) ? 1.0 : 0.0;
            MPI_Bcast(&go, 1, MPI_DOUBLE, 0, MPI_COMM_WORLD);
        }
        MPI_Barrier(MPI_COMM_WORLD);
        t3 = MPI_Wtime();
        if (rank == 0) {
            J->out[0] = t3 - t2;
            J->out[1] = t2 - t1;
            J->out[2] = t1 - t0;
            J->out[3] = n;
        }
    }
    if (J->c_all) {
        /* this slab's interior planes (and the outer ghosts on the end ranks) */
        double *loc = (double *)malloc(sizeof(double) * (size_t)d[0] * plane);
        int i0 = rank == 0 ? 0 : 3, i1 = rank == size - 1 ? d[0] : d[0] - 3;
        if (!loc) return 2;
        pllref_get("c_new", loc);
        memcpy(J->c_all + off + (long)i0 * plane, loc + (long)i0 * plane, sizeof(double) * (size_t)(i1 - i0) * plane);
        free(loc);
    }
    return 0;
}

/* Runs `warm` + up to `steps` whole steps on `ranks` processes from the
 * initial fields (the whole padded box), the timed steps ending early once
 * budget_s seconds have passed (0: no limit); out[0] = seconds of the timed
 * steps (max over ranks: they leave the last barrier together), out[3] the
 * timed steps run, out[1] warm-up,
 * out[2] set-up; the padded box has nelem doubles in nx_max_global planes;
 * c_out (nelem doubles, or NULL) receives c_new of the whole box.  Returns 0
 * on success. */
int pllref_mpi_run(int ranks, const char *rundir, const double *c, const double *u, const double *v,
                   const double *w, int warm, int steps, double budget_s, double *out, long nelem,
                   int nx_max_global, double *c_out)
{
    job_t J;
    int rc;
    double *c_all = NULL;
    if (c_out) {
        c_all = (double *)mmap(NULL, sizeof(double) * (size_t)nelem, PROT_READ | PROT_WRITE,
                               MAP_SHARED | MAP_ANONYMOUS, -1, 0);
        if (c_all == MAP_FAILED) return -1;
    }
    double *shared = (double *)mmap(NULL, 4096, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (shared == MAP_FAILED) return -1;
    memset(shared, 0, 4096);
    J.rundir = rundir;
    J.c = c;
    J.u = u;
    J.v = v;
    J.w = w;
    J.warm = warm;
    J.steps = steps;
    J.budget_s = budget_s;
    J.out = shared;
    J.c_all = c_all;
    /* the largest message is one halo exchange of four fields x 3 ghost
     * planes of the padded y-z plane (update_ghost_points); rings hold three
     * of them plus a pipelined x solve's per-line messages */
    {
        long plane = nelem / nx_max_global;
        long ring = 3L * 12 * plane * (long)sizeof(double) + (8L << 20);
        rc = shm_mpi_launch(ranks, ring, rank_body, &J);
    }
    if (c_all) {
        memcpy(c_out, c_all, sizeof(double) * (size_t)nelem);
        munmap(c_all, sizeof(double) * (size_t)nelem);
    }
    out[0] = shared[0];
    out[1] = shared[1];
    out[2] = shared[2];
    out[3] = shared[3];
    munmap(shared, 4096);
    return rc;
}
