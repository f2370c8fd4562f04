/*
 * One-rank MPI stand-in used ONLY to build the reference SALEc2d sources as a CPU oracle.
 *
 * Test infrastructure, not product code: the reference (src/mpi_vec/mpi_vec_types.h:7)
 * includes <mpi.h>, and this image has no MPI. Every communicator here has exactly one
 * rank (rank 0, size 1), so the reference's halo route tables are empty
 * (src/mpi_vec/mpi_vec.c:327-357) and collectives reduce to copies.
 *
 * Only the entry points the reference calls are provided (see oracle/mpi_shim/mpi_shim.c).
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Op;
typedef int MPI_Datatype;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

typedef int (MPI_Comm_copy_attr_function)(MPI_Comm, int, void *, void *, void *, int *);
typedef int (MPI_Comm_delete_attr_function)(MPI_Comm, int, void *, void *);

#define MPI_SUCCESS 0
#define MPI_COMM_NULL  ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_INFO_NULL ((MPI_Info)0)

#define MPI_CHAR   ((MPI_Datatype)1)
#define MPI_INT    ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)

#define MPI_MIN ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_SUM ((MPI_Op)3)

#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_MAX_PROCESSOR_NAME 256

#define MPI_COMM_NULL_COPY_FN ((MPI_Comm_copy_attr_function *)0)
#define MPI_COMM_NULL_DELETE_FN ((MPI_Comm_delete_attr_function *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Get_processor_name(char *name, int *len);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[], int reorder, MPI_Comm *cart);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Comm_create_keyval(MPI_Comm_copy_attr_function *copy_fn, MPI_Comm_delete_attr_function *delete_fn,
                           int *keyval, void *extra_state);
int MPI_Comm_set_attr(MPI_Comm comm, int keyval, void *attribute_val);
int MPI_Comm_get_attr(MPI_Comm comm, int keyval, void *attribute_val, int *flag);
int MPI_Comm_set_info(MPI_Comm comm, MPI_Info info);
int MPI_Info_create(MPI_Info *info);
int MPI_Info_set(MPI_Info info, const char *key, const char *value);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Iallreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm,
                   MPI_Request *req);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Send_init(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Startall(int count, MPI_Request reqs[]);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status stats[]);
int MPI_Wait(MPI_Request *req, MPI_Status *stat);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Status *stat);

#ifdef __cplusplus
}
#endif
#endif
