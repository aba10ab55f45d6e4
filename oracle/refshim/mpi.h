/* Single-rank stand-in for MPI, used only to compile the reference solver for oracle runs.
 * TEST INFRASTRUCTURE ONLY.  Collectives copy send -> receive buffers (device or host
 * pointers alike through cudaMemcpyDefault when built by nvcc); point-to-point calls are
 * never issued with one rank (zero neighbour ranks). */
#ifndef FG_REFSHIM_MPI_H
#define FG_REFSHIM_MPI_H
#include <string.h>
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct { int dummy; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
static inline int MPI_Init(int *a, char ***b) { (void)a; (void)b; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm c, int t, int k, MPI_Info i, MPI_Comm *o) { (void)c; (void)t; (void)k; (void)i; *o = 0; return 0; }
static inline int MPI_Comm_free(MPI_Comm *c) { (void)c; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Request_free(MPI_Request *r) { (void)r; return 0; }
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) { (void)n; (void)r; (void)s; return 0; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *r) { (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; (void)r; return 0; }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *r) { (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; (void)r; return 0; }
#ifdef __CUDACC__
#include <cuda_runtime.h>
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
    (void)o; (void)c;
    if (s == MPI_IN_PLACE) return 0;
    cudaMemcpy(r, s, (size_t)n * (size_t)t, cudaMemcpyDefault);
    return 0;
}
#else
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
    (void)o; (void)c;
    if (s == MPI_IN_PLACE) return 0;
    memcpy(r, s, (size_t)n * (size_t)t);
    return 0;
}
#endif
#endif
