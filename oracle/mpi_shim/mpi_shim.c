/*
 * One-rank MPI stand-in for building the reference as a CPU oracle (test infrastructure).
 *
 * Semantics for a single process: rank 0 of size 1 on every communicator; reductions and
 * gathers copy the send buffer to the receive buffer; point-to-point calls are never
 * reached because the reference's route tables are empty with npgx = npgy = 1
 * (src/mpi_vec/mpi_vec.c:327-357) and abort loudly if they are.
 * Communicator attributes are stored per (communicator, key), as the reference's
 * field duplication relies on them (src/mpi_vec/mpi_vec.c:707-716, 753-756).
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SHIM_MAX_ATTR 4096

static int g_next_comm = 2;
static int g_next_key = 1;
static struct { MPI_Comm comm; int key; void *val; } g_attr[SHIM_MAX_ATTR];
static int g_nattr = 0;

static size_t dt_size(MPI_Datatype dt) { return (size_t)dt; }

static void shim_fail(const char *what)
{
    fprintf(stderr, "oracle mpi shim: %s is not supported with one rank\n", what);
    abort();
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }

int MPI_Get_processor_name(char *name, int *len)
{
    strcpy(name, "oracle");
    *len = (int)strlen(name);
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[], int reorder, MPI_Comm *cart)
{
    (void)old; (void)periods; (void)reorder;
    for (int k = 0; k < ndims; ++k)
        if (dims[k] != 1) shim_fail("a process grid larger than 1x1");
    *cart = g_next_comm++;
    return MPI_SUCCESS;
}

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) { (void)comm; *newcomm = g_next_comm++; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
    (void)comm; (void)color; (void)key;
    *newcomm = g_next_comm++;
    return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

int MPI_Comm_create_keyval(MPI_Comm_copy_attr_function *copy_fn, MPI_Comm_delete_attr_function *delete_fn,
                           int *keyval, void *extra_state)
{
    (void)copy_fn; (void)delete_fn; (void)extra_state;
    *keyval = g_next_key++;
    return MPI_SUCCESS;
}

int MPI_Comm_set_attr(MPI_Comm comm, int keyval, void *attribute_val)
{
    for (int k = 0; k < g_nattr; ++k)
        if (g_attr[k].comm == comm && g_attr[k].key == keyval) { g_attr[k].val = attribute_val; return MPI_SUCCESS; }
    if (g_nattr >= SHIM_MAX_ATTR) shim_fail("more communicator attributes than the shim table holds");
    g_attr[g_nattr].comm = comm;
    g_attr[g_nattr].key = keyval;
    g_attr[g_nattr].val = attribute_val;
    ++g_nattr;
    return MPI_SUCCESS;
}

int MPI_Comm_get_attr(MPI_Comm comm, int keyval, void *attribute_val, int *flag)
{
    for (int k = 0; k < g_nattr; ++k)
        if (g_attr[k].comm == comm && g_attr[k].key == keyval) {
            *(void **)attribute_val = g_attr[k].val;
            *flag = 1;
            return MPI_SUCCESS;
        }
    *flag = 0;
    return MPI_SUCCESS;
}

int MPI_Comm_set_info(MPI_Comm comm, MPI_Info info) { (void)comm; (void)info; return MPI_SUCCESS; }
int MPI_Info_create(MPI_Info *info) { *info = 1; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info info, const char *key, const char *value) { (void)info; (void)key; (void)value; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm;
    if (sendbuf != MPI_IN_PLACE && count > 0) memmove(recvbuf, sendbuf, (size_t)count * dt_size(dt));
    return MPI_SUCCESS;
}

int MPI_Iallreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm,
                   MPI_Request *req)
{
    if (req) *req = MPI_REQUEST_NULL;
    return MPI_Allreduce(sendbuf, recvbuf, count, dt, op, comm);
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm)
{
    (void)rcount; (void)rtype; (void)comm;
    if (sendbuf != MPI_IN_PLACE && scount > 0) memmove(recvbuf, sendbuf, (size_t)scount * dt_size(stype));
    return MPI_SUCCESS;
}

int MPI_Send_init(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)buf; (void)count; (void)dt; (void)dest; (void)tag; (void)comm; (void)req;
    shim_fail("MPI_Send_init");
    return 1;
}

int MPI_Recv_init(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)buf; (void)count; (void)dt; (void)src; (void)tag; (void)comm; (void)req;
    shim_fail("MPI_Recv_init");
    return 1;
}

int MPI_Startall(int count, MPI_Request reqs[]) { (void)reqs; if (count) shim_fail("MPI_Startall"); return MPI_SUCCESS; }
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status stats[]) { (void)reqs; (void)stats; if (count) shim_fail("MPI_Waitall"); return MPI_SUCCESS; }
int MPI_Wait(MPI_Request *req, MPI_Status *stat) { (void)req; (void)stat; return MPI_SUCCESS; }

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)buf; (void)count; (void)dt; (void)dest; (void)tag; (void)comm; (void)req;
    shim_fail("MPI_Isend");
    return 1;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)buf; (void)count; (void)dt; (void)src; (void)tag; (void)comm; (void)req;
    shim_fail("MPI_Irecv");
    return 1;
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm)
{
    (void)buf; (void)count; (void)dt; (void)dest; (void)tag; (void)comm;
    shim_fail("MPI_Send");
    return 1;
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Status *stat)
{
    (void)buf; (void)count; (void)dt; (void)src; (void)tag; (void)comm; (void)stat;
    shim_fail("MPI_Recv");
    return 1;
}
