/* Single-rank MPI stand-in for building the reference library on one GPU.
 *
 * Test infrastructure only: it lets the reference sources (which declare
 * their single-GPU entry points only under HAVE_MPI, src/neurongpu.cu:284,
 * :426, :1093) compile without an MPI installation. Every process is rank 0
 * of a world of size 1; point-to-point calls are never reached in a
 * single-host run (they serve RemoteConnect / remote spikes) and return an
 * error if they are. */
#ifndef NGB200_REF_STUB_MPI_H
#define NGB200_REF_STUB_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_BYTE 4
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Finalized(int *flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
/* With one rank the root already holds the data. */
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_ERR_OTHER; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return MPI_ERR_OTHER; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
static inline int MPI_Test(MPI_Request *, int *flag, MPI_Status *) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype, int *count) { *count = st ? st->count : 0; return MPI_SUCCESS; }

#endif
