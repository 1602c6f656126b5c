/* Minimal single-process MPI stand-in used only to compile the reference
 * correlator sources (Configuration, Mode, Model) for the CPU oracle build.
 * Every call is a no-op that reports success: the oracle harness uses the
 * non-MPI Configuration constructor, so no message ever needs to move. */
#ifndef ORACLE_REFSTUB_MPI_H
#define ORACLE_REFSTUB_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_SUCCESS 0
#define MPI_INT 1
#define MPI_CHAR 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_COMM_WORLD 0
#ifdef __cplusplus
extern "C" {
#endif
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; (void)e; return MPI_SUCCESS; }
/* point-to-point calls of DataStream's send and receive paths, which the
 * harness never reaches: complete at once */
#define MPI_ANY_TAG (-1)
#define MPI_ANY_SOURCE (-1)
#define MPI_UNSIGNED_CHAR 5
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Issend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void)r; (void)s; return MPI_SUCCESS; }
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) { (void)n; (void)r; (void)s; return MPI_SUCCESS; }
static inline int MPI_Testall(int n, MPI_Request *r, int *flag, MPI_Status *s)
{ (void)n; (void)r; (void)s; *flag = 1; return MPI_SUCCESS; }
#ifdef __cplusplus
}
#endif
#endif
