/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference
 * library into the test oracle (oracle/_ref).  No MPI is installed in this
 * image; the oracle never calls the reference's MPI code paths (shot queue,
 * domain decomposition), it only needs the declarations to link.
 * Every call is a no-op that reports success on a world of one rank.
 *
 * Test infrastructure only: nothing in rockseis_b200/ includes this file.
 */
#ifndef RS_ORACLE_MPI_STUB_H
#define RS_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_COMM 5
#define MPI_ERR_COUNT 2
#define MPI_ERR_TYPE 3
#define MPI_ERR_TAG 4
#define MPI_ERR_RANK 6
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_TAG (-1)
#define MPI_ANY_SOURCE (-2)
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_UNSIGNED_LONG 4
#define MPI_LONG_INT 5
#define MPI_SUM 1
#define MPI_IN_PLACE ((void *)1)

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Get_processor_name(char *n, int *l) { strcpy(n, "oracle"); *l = 6; return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *s)
{ if (s) { s->MPI_SOURCE = 0; s->MPI_TAG = 0; s->MPI_ERROR = 0; } return 0; }
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype,
                               int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *n) { *n = 0; return 0; }
static inline int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *,
                                         MPI_Datatype *t) { *t = 100; return 0; }
static inline int MPI_Type_commit(MPI_Datatype *) { return 0; }

#endif
