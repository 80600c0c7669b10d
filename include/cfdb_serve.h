/*
 * cfdb serving loop: continuous batching of pressure solves on one GPU (no counterpart in the
 * reference, which solves one system at a time inside its time loop).
 *
 * Requests are queued at submit and taken by worker slots as soon as a slot is free; each mesh
 * keeps a resident persistent system (pattern, AMG hierarchy, the last matrix, right-hand side
 * and solution on the device, its own CUDA stream), so requests on different meshes overlap on
 * the GPU. Systems are admitted against an HBM budget (estimated footprint, then measured),
 * evicting idle systems least-recently-used first; requests that cannot fit yet wait.
 * matrix_key names a coefficient set: a request repeating the key of the matrix resident on its
 * mesh skips the matrix upload, and with warm_start it starts from the resident solution.
 */
#ifndef CFDB_SERVE_H
#define CFDB_SERVE_H

#include "cfdb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Order in which free worker slots take queued requests. */
enum {
    CFDB_SCHEDULE_FIFO = 0,      /* the first queued request whose mesh is free */
    CFDB_SCHEDULE_MOST_WORK = 1  /* the first queued request of the free mesh with the most
                                    queued cells (requests of one mesh stay in order) */
};

typedef struct {
    int slots;                  /* concurrent worker slots (streams), default 4 */
    double hbm_budget_bytes;    /* device bytes the resident systems may hold, default 150e9 */
    int precision;              /* cfdb_precision of the solves, default MIXED */
    cfdb_amg_settings settings; /* hierarchy settings */
    int max_age;                /* rebuild the hierarchy after this many solves (0: never), as
                                   the reference's AmgCache does; a request whose matrix is the
                                   one the hierarchy was built from (same matrix_key) does not
                                   trigger it, since the rebuild would reproduce the hierarchy */
    int pdl;                    /* programmatic dependent launch in the resident systems' solves
                                   (cfdb_tuning.pdl), default 0 (kernels scheduled early hold
                                   SM slots that other requests' kernels could use; on the
                                   box/tet serving mix with 6 slots it measured 3-8 % faster,
                                   and the benchmark turns it on) */
    int mixed_sweeps;           /* mixed precision: the V-cycle's smoother schedule */
    double mixed_weight;        /* (cfdb_tuning.mixed_sweeps / mixed_weight; 0: the hierarchy's) */
    int background_rebuild;     /* 1: an aged hierarchy is rebuilt off the request path, on a
                                   spare system per mesh, from a device copy of the triggering
                                   request's matrix; requests keep solving with the old one
                                   until the new one is swapped in (results then depend on
                                   timing, within the tolerance). 0 (default): rebuilt before
                                   the triggering request's solve, as the reference does */
    int schedule;               /* CFDB_SCHEDULE_*, default FIFO */
} cfdb_server_config;

typedef struct {
    int resident_systems;
    double resident_bytes;
    int queued;
    long long completed;
    long long evictions;
    long long rebuilds;            /* hierarchy rebuilds on the request path (age rule) */
    long long background_rebuilds; /* hierarchies built in the background and swapped in */
} cfdb_server_info_t;

typedef struct cfdb_server cfdb_server;

void cfdb_default_server_config(cfdb_server_config* c);
int cfdb_server_create(const cfdb_server_config* cfg, cfdb_server** out);
/* Drains the queue, joins the workers, frees every resident system. */
int cfdb_server_destroy(cfdb_server* s);
/* Registers mesh addressing (internal faces); returns its id. */
int cfdb_server_add_mesh(cfdb_server* s, int n_cells, int n_faces, const int* owner,
                         const int* neighbour, int* mesh_id);
/* Queues one solve A x = rhs to relative residual rel_tol (x0 = 0, or the resident solution of
 * the same matrix_key with warm_start). The host arrays are borrowed, as for an asynchronous
 * copy: diag / upper / lower / rhs must stay valid and unchanged, and x (n_cells, may be NULL)
 * receives the solution, by the time cfdb_server_wait returns for the ticket. Page-locked
 * arrays are copied at full link speed. */
int cfdb_server_submit(cfdb_server* s, int mesh_id, long long matrix_key, const double* diag,
                       const double* upper, const double* lower, const double* rhs, double* x,
                       int warm_start, double rel_tol, int max_iterations, long long* ticket);
/* Blocks until the ticket is done; times (3 doubles, may be NULL) receives the submit / start /
 * finish times in seconds since server creation. */
int cfdb_server_wait(cfdb_server* s, long long ticket, cfdb_stats* stats, double* times);
int cfdb_server_info(cfdb_server* s, cfdb_server_info_t* info);

#ifdef __cplusplus
}
#endif
#endif
