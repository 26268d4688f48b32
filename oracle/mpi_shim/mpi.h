/* Thread-rank MPI stand-in used ONLY to build the reference CPU sources as a test oracle.
 *
 * Test infrastructure: nothing in the product links this.  No MPI library exists in this
 * image, so the reference's CPU path (src/step.cpp, src/communicate.cpp, src/static_ic.cpp,
 * ...) is compiled against this header.  Each "rank" is a host thread started by the oracle
 * harness (oracle/ref_harness.cpp); point-to-point messages go through in-process mailboxes
 * and collectives through a shared slot table.  Only the subset of MPI the reference calls is
 * provided: Init/Finalize/Comm_size/Comm_rank/Send/Recv/Sendrecv/Allreduce(MIN,MAX)/Bcast/
 * Abort and the constants they use.
 */
#ifndef R3D_ORACLE_MPI_SHIM_H
#define R3D_ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_MIN ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_SUM ((MPI_Op)3)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status* status);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int errorcode);

/* Harness control (not MPI): size the world and bind the calling thread to a rank. */
void r3d_shim_world_init(int nranks);
void r3d_shim_bind_rank(int rank);

#ifdef __cplusplus
}
#endif

#endif
