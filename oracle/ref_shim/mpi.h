/* ORACLE test infrastructure: single-rank stand-in for the MPI calls the
 * reference makes, so that its sources compile and run as one process
 * without an MPI installation.  With one rank every collective is a copy
 * and no point-to-point call is reached (src/deviceclass.cpp:876,958,995
 * guard them with NumProcessors > 1). */
#ifndef ESDG_REF_MPI_STUB_H
#define ESDG_REF_MPI_STUB_H
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 4
#define MPI_FLOAT 104
#define MPI_DOUBLE 8
#define MPI_CHAR 1
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_REQUEST_NULL 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

static inline size_t esdg_mpi_size(MPI_Datatype t) { return t == MPI_FLOAT ? 4 : (size_t)(t % 100); }
static inline int MPI_Init(int* a, char*** b) { (void)a; (void)b; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* n) { (void)c; *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Get_processor_name(char* s, int* len) { strcpy(s, "localhost"); *len = 9; return 0; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
    (void)o; (void)c; memmove(r, s, (size_t)n * esdg_mpi_size(t)); return 0; }
static inline int MPI_Scatter(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
    (void)sn; (void)st; (void)root; (void)c; memmove(r, s, (size_t)rn * esdg_mpi_size(rt)); return 0; }
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) { (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 1; }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st) { (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 1; }
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* r) { (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *r = 0; return 1; }
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* r) { (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *r = 0; return 1; }
static inline int MPI_Wait(MPI_Request* r, MPI_Status* s) { (void)r; (void)s; return 0; }
static inline int MPI_Waitall(int n, MPI_Request* r, MPI_Status* s) { (void)n; (void)r; (void)s; return 0; }
#endif
